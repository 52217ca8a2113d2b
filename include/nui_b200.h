/*
 * nui_b200 -- C ABI of the B200 KinectFusion hot path.
 *
 * Replaces the device layer of hustztz/NatureUserInterfaceStudio for the per-frame path:
 * src/OpenCLUtilities (context/queue singleton, kernel manager, buffer manager) and the
 * OpenCL implementations of the tracker / frame / scene interfaces under
 * src/SLAM/VisualOdometry/DeviceSpecific.  Plain C types only: host pointers for the
 * session-level calls, device pointers (CUDA global memory of the context's device) for
 * the kernel-level calls, sizes as integers, an int status for every call.
 *
 * Threading: one session must not be called concurrently from two threads; different
 * sessions may be.  Every session-level call is synchronous with respect to the host
 * buffers it is given (they may be reused when the call returns).
 */
#ifndef NUI_B200_H
#define NUI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define NUI_API __attribute__((visibility("default")))
#else
#define NUI_API
#endif

/* ---------------------------------------------------------------- status codes
 * The reference returns bool and prints OpenCL errors to stderr
 * (src/OpenCLUtilities/NuiOpenCLUtil.h:10-13); here every call returns one of these. */
typedef enum {
  NUI_OK = 0,
  NUI_ERR_INVALID_ARG = 1,
  NUI_ERR_OOM = 2,
  NUI_ERR_TRACKING_LOST = 3, /* singular ICP system (NuiKinfuOpenCLDepthTracker.cpp:465-472) */
  NUI_ERR_HASH_FULL = 4,     /* voxel hash: a frame's allocation found the block pool or the
                              * excess list empty (or met a corrupted excess chain) and dropped
                              * blocks; the frame is otherwise complete (pose tracked, the
                              * allocated blocks integrated).  The reference drops them silently
                              * (KinfuHashScene.cl:155,171-172). */
  NUI_ERR_MESH_OVERFLOW = 5,
  NUI_ERR_TIMEOUT = 6,
  NUI_ERR_DEVICE = 7,
  NUI_ERR_UNSUPPORTED = 8
} nui_status;

/* TSDF storage formats of the dense volume.
 * NUI_TSDF_I16 is the reference's short2 (tsdf * 32766 truncated, int16 weight;
 * tsdfVolume.cl:31-190 with utils.cl:69-79).  The others store the same running average
 * without the 16-bit quantisation.  I16 and F32 sessions reproduce the reference's float
 * arithmetic bit for bit; the FP16 formats (the serving formats, for dense volumes and, as
 * half-precision sdf, voxel hashes) run tolerance-mode kernels for the bilateral filter,
 * dense integration and dense raycast: results agree with the reference within 1e-3
 * truncation units (TSDF) and 0.5 mm (raycast depth), not bit for bit. */
typedef enum {
  NUI_TSDF_I16 = 0,     /* 4 B/voxel: int16 tsdf, int16 weight                 */
  NUI_TSDF_F32 = 1,     /* 8 B/voxel: float tsdf, float weight                 */
  NUI_TSDF_F16_U8 = 2,  /* 3 B/voxel: half tsdf plane + uint8 weight plane     */
  NUI_TSDF_F16_F16 = 3  /* 4 B/voxel: half tsdf, half weight                   */
} nui_tsdf_format;

typedef enum { NUI_VOLUME_DENSE = 0, NUI_VOLUME_HASH = 1 } nui_volume_kind;

/* Session configuration.  Field meaning and defaults follow the reference configs:
 * NuiTrackerConfig (NuiTrackerConfig.cpp:5-24), NuiKinfuVolumeConfig
 * (NuiKinfuVolumeConfig.cpp:5-15), NuiCameraParams / NuiDepthFrame sensor range
 * (src/Frame/NuiDepthFrame.h:12-16) and the engine's integration gate
 * (NuiKinfuTrackingEngine.cpp:22). */
typedef struct {
  int width, height;
  float fx, fy, cx, cy;
  float depth_min, depth_max; /* metres; depth outside (min, max) is invalid */
  /* dense volume */
  int volume_kind;            /* nui_volume_kind */
  int tsdf_format;            /* nui_tsdf_format */
  int res[3];
  float dim[3];               /* metres; volume spans x,y in [-dim/2, dim/2], z in [0, dim] */
  float trunc_dist;           /* VolumeTrancDist; effective = max(trunc_dist, 2.1 * cell) */
  int color_volume;           /* VolumeHadColor */
  int max_color_weight;       /* MaxColorWeight */
  /* tracker */
  int levels;                 /* pyramid levels (<= 4) */
  int iterations[4];          /* ICP iterations per level, finest first */
  int filter_radius;          /* icp_filter_radius */
  float sigma_space2_inv_half;/* icp_sigma_space2_inv_half */
  float sigma_depth2_inv_half;/* icp_sigma_depth2_inv_half */
  float depth_threshold;      /* icp_depth_threshold */
  float dist_threshold;       /* icp_dist_threshold */
  float integration_threshold;/* m_integration_metric_threshold */
  /* voxel-block hash (volume_kind == NUI_VOLUME_HASH); NuiHashingSDFConfig
   * (NuiHashingSDFConfig.cpp:3-15).  Table sizes are runtime parameters here; the
   * reference fixes them at compile time (hashing_gpu_def.h:9-20).  tsdf_format selects
   * the voxel sdf storage: NUI_TSDF_I16 = the reference's int16 (sdf * 32767), anything
   * else = half; weights are uint8 (cap hash_max_weight) and colours RGB8. */
  float voxel_size;           /* m_virtualVoxelSize */
  float trunc_scale;          /* m_truncScale */
  int hash_buckets;           /* power of two; hash mask = buckets - 1 */
  int hash_excess;            /* excess (collision) list length */
  int hash_pool_blocks;       /* 8^3 voxel blocks in the pool */
  int hash_max_weight;        /* m_integrationWeightMax */
  /* colour tracking: weight of the photometric normal equations (the rows of
   * color_icp_block_kernel, colorIcp.cl:91-183, against the previous frame's colours at
   * the previous raycast's points) added to the point-to-plane ones in every ICP iteration
   * of the finest level; 0 = depth only.  Needs color_volume = 1 and BGRA frames whose
   * valid pixels have alpha 255.  Colours and gradients enter in units of 1/255. */
  float photometric_weight;
  /* shifting dense volume: the reference's eScene_ShiftingVolume (NuiKinfuOpenCLShiftScene,
   * NuiSLAMController.cpp:55-62; NuiKinfuVolumeConfig voxel_shift / translateBasis).  On an
   * integrating frame, every axis on which the tracked camera lies voxel_shift or more
   * voxels from shift_basis moves the volume by voxel_shift voxels before the integration:
   * the slab that leaves is fetched as points (fetchShiftVolumeKernel) into a device cache
   * of shift_point_cap points and cleared, the volume's voxel offset moves forward and the
   * session's (local) pose back.  Poses are then local to the volume: global = local +
   * offset (nui_shift_state).  0 = fixed volume (default); dense volumes only;
   * voxel_shift < res on every axis. */
  int voxel_shift;
  float shift_basis[3];
  int shift_point_cap;        /* default 2^20 (28 MB) */
  /* voxel hash: the global cache (NuiHashingSDFConfig::m_bUseSwapping,
   * NuiKinfuOpenCLHashGlobalCache).  Blocks that leave the view after being merged move to
   * a host store and their pool blocks are freed; blocks that come back are re-allocated
   * and merged with their stored copies, at most 4096 each way per frame.  The store is
   * pinned host memory mapped into the device, hash_store_blocks blocks of 512 voxels
   * (0 = one per hash entry, as the reference keeps); a full store leaves blocks in the
   * device pool (counted by nui_hash_swap_stats). */
  int hash_swapping;
  int hash_store_blocks;
  /* voxel hash: how the reference maps are rendered after each frame.  0 = raycast every
   * pixel (the reference's raycast path, NuiKinfuOpenCLHashScene::Raycast; the default
   * here).  1 = the reference's forward rendering (ForwardRender,
   * NuiKinfuOpenCLHashScene.cpp:991-1012, on by default in NuiSLAMController.cpp:47): the
   * previous maps' vertices are carried to the pixels they project to, only pixels nothing
   * lands on are raycast, and normals come from the vertex map; the reference projects the
   * vertices with the camera-to-world transform of the pose (forwardProject_kernel,
   * KinfuHashRaycast.cl:490), which mode 1 reproduces.  2 = forward rendering with the
   * vertices taken into the camera (world-to-camera).  Measured on the oracle (320x240 orbit,
   * 20 frames): ATE 4.0 mm with mode 0, 415 mm with mode 1 (tracking diverges once the
   * camera moves), 7.9 mm with mode 2. */
  int hash_forward_render;
} nui_session_cfg;

typedef struct nui_ctx nui_ctx;
typedef struct nui_session nui_session;

/* Fills the reference defaults (640x480, fx=fy=525, 256^3 over 3 m, 3 levels x 10 ICP
 * iterations, bilateral radius 3, thresholds of NuiTrackerConfig). */
NUI_API void nui_session_cfg_default(nui_session_cfg* cfg);

/* Last error message of the calling thread ("" if none). */
NUI_API const char* nui_last_error_string(void);

/* ---------------------------------------------------------------- context
 * Replaces NuiOpenCLGlobal::initializeOpenCL (NuiOpenCLGlobal.cpp:75-219): binds a CUDA
 * device and a stream.  nui_ctx_set_stream lets the caller supply its own stream
 * (cudaStream_t cast to void*); NULL restores the context's own stream. */
NUI_API nui_status nui_ctx_create(int device, nui_ctx** out);
NUI_API nui_status nui_ctx_destroy(nui_ctx* ctx);
NUI_API nui_status nui_ctx_set_stream(nui_ctx* ctx, void* cuda_stream);
NUI_API nui_status nui_ctx_synchronize(nui_ctx* ctx);
/* Session memory comes from a memory pool of the context, allocated and freed in stream
 * order (a destroyed session's memory stays in the pool for the next session, and serving
 * admissions never synchronise the device).  nui_ctx_trim waits for the context's stream and
 * returns the pool's unused memory to the device. */
NUI_API nui_status nui_ctx_trim(nui_ctx* ctx);

/* ---------------------------------------------------------------- sessions
 * A session holds one RGB-D stream's device state: frame pyramids, reference maps,
 * pose, volume.  Construction replaces NuiKinfuTrackingFactory::BuildTrackingEngine
 * (NuiKinfuTrackingFactory.h:23-50) + NuiSLAMController::setVolume
 * (NuiSLAMController.cpp:33-69).  Bytes of device memory it needs: */
NUI_API size_t nui_session_device_bytes(const nui_session_cfg* cfg);
NUI_API nui_status nui_session_create(nui_ctx* ctx, const nui_session_cfg* cfg, nui_session** out);
NUI_API nui_status nui_session_destroy(nui_session* s);
/* NuiKinfuScene::reset + NuiKinfuTrackingEngine::reset: empty volume, identity pose. */
NUI_API nui_status nui_reset(nui_session* s);

/* One frame of NuiKinfuTrackingEngine::RunTracking (NuiKinfuTrackingEngine.cpp:68-142):
 * upload + preprocess, then (frame 0) feedback maps + integrate, or (frame > 0) ICP,
 * gated integration and raycast.  depth_mm: width*height uint16; bgra: width*height*4
 * bytes or NULL.  pose_out (nullable): 12 floats, R row-major then t.
 * Returns NUI_ERR_TRACKING_LOST when ICP hits a singular system (the frame then leaves
 * the volume and pose untouched, as the reference's early `return false`). */
NUI_API nui_status nui_process_frame(nui_session* s, const uint16_t* depth_mm, const uint8_t* bgra,
                                     float* pose_out);
/* Same with the frame already in device memory. */
NUI_API nui_status nui_process_frame_device(nui_session* s, const uint16_t* d_depth_mm,
                                            const uint8_t* d_bgra, float* pose_out);

/* Step-wise calls mirroring the reference virtuals (for the C++ adaptor classes):
 *  NuiKinfuFrame::UpdateVertexBuffers / UpdateColorBuffers  -> nui_frame_upload
 *  NuiKinfuFeedbackFrame::UpdateBuffers                     -> nui_feedback_update
 *  NuiKinfuTracker::EstimatePose                            -> nui_track
 *  NuiKinfuScene::integrateVolume                           -> nui_integrate
 *  NuiKinfuScene::raycastRender                             -> nui_raycast
 *  NuiKinfuCameraState::UpdateCameraTransform / GetCameraPos-> nui_set_pose / nui_get_pose */
NUI_API nui_status nui_frame_upload(nui_session* s, const uint16_t* depth_mm, const uint8_t* bgra);
NUI_API nui_status nui_feedback_update(nui_session* s);
NUI_API nui_status nui_track(nui_session* s, float* err_out, int* count_out);
NUI_API nui_status nui_integrate(nui_session* s);
NUI_API nui_status nui_raycast(nui_session* s);
NUI_API nui_status nui_set_pose(nui_session* s, const float* pose12);
NUI_API nui_status nui_get_pose(nui_session* s, float* pose12);

/* Marching cubes over the dense volume (NuiKinfuScene::Volume2CLMesh,
 * NuiKinfuOpenCLScene.cpp:617-786), compacted by prefix sums into the deterministic order
 * of the reference's CPU extraction (y, then x, then z fastest).  pos: cap*3 floats,
 * col: cap*4 floats (either may be NULL); *nverts receives the full vertex count, and
 * NUI_ERR_MESH_OVERFLOW is returned (with the first cap vertices written) when it
 * exceeds cap. */
NUI_API nui_status nui_mesh(nui_session* s, float* pos, float* col, uint64_t cap, uint64_t* nverts);
/* Marching cubes of a dense session into caller-provided DEVICE buffers, without any
 * device allocation.  No counterpart in the reference: it exists for callers that cannot
 * call cudaMalloc while meshing, e.g. a host application that owns all device memory
 * through its own pool, or code running where allocation is forbidden or would stall the
 * GPU.  The per-column counts and block offsets the kernels need live in one file-scope
 * __device__ array of 1 MiB + 32 KiB (held by every GPU that loads the library until the
 * process exits), which bounds the volume to (res[0]-1)*(res[1]-1) <= 262144 columns and
 * (res[1]-1)*ceil((res[0]-1)/128) <= 4095 count blocks; larger volumes are rejected with
 * NUI_ERR_INVALID_ARG.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call outside any
 * stream capture.  The address is looked up again after nui_ctx_create on that device, so
 * a device reset (which invalidates it, with every session) followed by a new context
 * works.  All calls share the array: two calls that overlap on the GPU (other threads,
 * other streams) race on it.  The kernels run on the session's context stream with no
 * ordering against the caller's streams: the output buffers must be idle when the call is
 * made (synchronise whatever produces or reads them first); the call synchronises its
 * stream before it returns.  Buffers on another device are rejected.  The caller's current
 * device is restored on return.  Same order, capacity and overflow rules as nui_mesh;
 * d_pos: cap*3 floats, d_col: cap*4 floats, either may be NULL. */
NUI_API nui_status nui_mesh_device_noalloc(nui_session* s, float* d_pos, float* d_col, uint64_t cap,
                                           uint64_t* nverts);
/* Number of device and pinned-host allocations the library has made in this process (every
 * cudaMalloc / cudaMallocHost / cudaHostAlloc it issues).  No counterpart in the
 * reference; for tests that check an entry point allocates nothing. */
NUI_API nui_status nui_debug_allocation_count(uint64_t* n);
/* Marching-cubes case index of every cube, (res[0]-1)*(res[1]-1)*(res[2]-1) bytes in the
 * same (y, x, z) order; 0 for cubes skipped because a corner has no weight. */
NUI_API nui_status nui_mesh_cases(nui_session* s, uint8_t* cases, size_t bytes, uint64_t* nverts);

/* Debug / test readback of session buffers into host memory.  `what`:
 *   0 filtered depth L0 (f32, W*H)      1 scaled depth for integration (f32, W*H)
 *   2 vertex map level `level` (f32x4)  3 reference vertex map (f32x4, W*H, world)
 *   4 reference normal map (f32x4)       5 volume in the reference layout, short2
 *   6 raw volume storage of the session format   7 depth level `level` (f32)
 *   8 reference colour map (u8x4)        9 colour volume, reference layout (u8x4)
 *  10 model colours of colour tracking: the previous frame's (u8x4)
 *  11 / 12 x / y colour gradients of the current frame (u8x4, signed bytes; level 0)
 *  13 brick states (u8 per 8^3 brick, x fastest: 0 empty, 1 mixed, 2 positive, 3 awaiting
 *     re-classification, 4 positive with unweighted voxels)
 *  14 weight plane of NUI_TSDF_F16_U8 (u8, session layout x + rx*(y + ry*z)) */
NUI_API nui_status nui_debug_download(nui_session* s, int what, int level, void* host, size_t bytes);
/* Voxel-hash sessions: what = 20 entries (16 B each: short pos[3], pad, int ptr, uint
 * offset), 21 visible list (int, count = nui_hash_stats visible), 22 pool voxels in the
 * reference voxel layout (short sdf, uchar rgb[3], uchar weight; 6 B each), 23 expected
 * range image (float2 per pixel). */
NUI_API nui_status nui_hash_stats(nui_session* s, int* visible, int* last_free_block, int* last_free_excess,
                                  int* failed_allocs);
/* Writes a reference-layout short2 volume into the session (any format). */
NUI_API nui_status nui_debug_upload_volume(nui_session* s, const int16_t* ref_layout_short2);

/* ---------------------------------------------------------------- batched ticks
 * Advances n sessions by one frame each with one launch per stage for all of them
 * (captured once in a CUDA graph and replayed).  depths[i] / bgras[i]: host frames
 * (bgras may be NULL or have NULL entries).  per_session_status: n entries.
 * poses_out (nullable): n*12 floats. */
NUI_API nui_status nui_batch_tick(nui_ctx* ctx, nui_session* const* sessions, int n,
                                  const uint16_t* const* depths, const uint8_t* const* bgras,
                                  nui_status* per_session_status, float* poses_out);
/* Same with device-resident frames (d_depths[i]: device pointers). */
NUI_API nui_status nui_batch_tick_device(nui_ctx* ctx, nui_session* const* sessions, int n,
                                         const uint16_t* const* d_depths, const uint8_t* const* d_bgras,
                                         nui_status* per_session_status, float* poses_out);

/* ---------------------------------------------------------------- serving loop
 * Continuous batching of many RGB-D streams on one GPU.  No counterpart in the reference,
 * which runs one stream (NuiKinfuTrackingEngine on its tracking thread).
 *   admit    creates a session for a stream if its device bytes (nui_session_device_bytes)
 *            fit in what is left of the HBM budget and a slot is free (else NUI_ERR_OOM:
 *            the caller keeps the stream waiting and tries again after a release);
 *   submit   queues one frame of a stream (host pointers, read at the step that takes the
 *            frame; they must stay valid until its result is polled; pinned memory lets
 *            the upload overlap the previous batch);
 *   step     launches the next batch -- the oldest queued frame of every stream that has
 *            one, all streams in one batched tick -- after starting its uploads on a second
 *            stream, then collects the batch launched by the previous step;
 *   poll     returns the finished frames with their submit and completion times on the
 *            server clock (seconds; completion from CUDA events on the compute stream);
 *   release  ends a stream (a frame of it in flight is completed first); its session is
 *            kept for the next stream of the same configuration and freed when another
 *            stream needs its budget.
 * Streams join and leave between steps; the batch keeps every live stream (streams without
 * a queued frame sit the tick out), so its captured graph changes only when streams join
 * or leave.  One server per context; not thread-safe.  Between a step and the next step
 * (or drain) a tick of the server is in flight: the context runs no other tick
 * (nui_batch_tick*, nui_process_frame*) until nui_server_drain has returned. */
typedef struct nui_server nui_server;
typedef struct {
  int slot;
  int status;         /* nui_status of the frame */
  uint64_t tag;       /* as submitted */
  double t_submit;    /* server clock, seconds */
  double t_done;
  float pose[12];     /* R row-major, t */
} nui_server_result;
NUI_API nui_status nui_server_create(nui_ctx* ctx, size_t hbm_budget_bytes, int max_streams, nui_server** out);
NUI_API nui_status nui_server_destroy(nui_server* srv);
NUI_API double nui_server_clock(const nui_server* srv);
NUI_API nui_status nui_server_admit(nui_server* srv, const nui_session_cfg* cfg, int* slot);
NUI_API nui_status nui_server_release(nui_server* srv, int slot);
/* Creates `count` idle sessions of `cfg` (counted in the budget) that later admissions of
 * that configuration take without allocating; a released stream's session is kept the
 * same way until a new stream needs its memory. */
NUI_API nui_status nui_server_reserve(nui_server* srv, const nui_session_cfg* cfg, int count);
/* t_submit < 0: now on the server clock (else the caller's arrival time on that clock) */
NUI_API nui_status nui_server_submit(nui_server* srv, int slot, const uint16_t* depth_mm, const uint8_t* bgra,
                                     uint64_t tag, double t_submit);
NUI_API nui_status nui_server_step(nui_server* srv, int* frames_launched);
NUI_API nui_status nui_server_drain(nui_server* srv);
NUI_API nui_status nui_server_poll(nui_server* srv, nui_server_result* out, int cap, int* n);
NUI_API nui_status nui_server_stats(const nui_server* srv, size_t* bytes_used, int* streams, int* queued);
NUI_API nui_session* nui_server_session(nui_server* srv, int slot);

/* Per-stage device time of the last nui_batch_tick* / nui_process_frame* call of the
 * context, when timing is enabled (CUDA events on the context stream).
 * stage: 0 preprocess, 1 pyramid + feedback maps, 2 tracking (colour gradients, ICP, gate),
 * 3 shifting-volume shifts + dense integration kernel, 4 brick summaries (+ voxel-hash
 * allocation / integration), 5 raycast, 6 whole tick, 7 the dense raycast kernels alone,
 * 8 the voxel-hash sessions' work on the second stream (0 when it did not run there).
 * When the batch holds dense and voxel-hash sessions, the hash sessions' tracking,
 * allocation, integration and raycast run on a second stream beside stages 2-5 instead
 * (stage 2 then times the dense sessions' tracking, stage 8 all of the hash sessions'
 * work, tracking included; in a served batch, whose table mixes the two families, the
 * tracking of both stays in stage 2); stage 5 ends when both streams are done. */
NUI_API nui_status nui_ctx_enable_timing(nui_ctx* ctx, int enable);
NUI_API nui_status nui_ctx_stage_ms(nui_ctx* ctx, int stage, float* ms);
/* Kernel launches in the captured graph of the context's last graphed batch tick. */
NUI_API nui_status nui_ctx_last_tick_kernels(nui_ctx* ctx, int* n);
/* Launch shapes of a context's tick, chosen by nui_ctx_autotune (or set by hand).  No
 * choice changes a result bit except the two ICP shapes, which regroup the FP64 partial
 * sums of the normal equations (poses agree to the rounding of those sums).
 *   integrate_threads_log2   dense integration: each volume column is split into z chunks,
 *                            one thread each, until a session's launch has >= 2^this
 *                            threads (chunks of >= 16 slices); 14..22, default 18
 *   icp_pixels_per_thread    ICP block: 256 threads x this many pixels; 2, 4, 8 or 16 (4)
 *   icp_cluster_blocks       ICP: thread blocks of the cluster that tracks one session;
 *                            2..16 (12: six SMs at two blocks an SM, so that three
 *                            clusters fill an 18-SM GPC; above 8 a non-portable size)
 *   raycast_tile_width       dense raycast: a warp shades a tile this wide and 32 / this
 *                            high, a block 2 x 2 such tiles; 4, 8, 16 or 32 (8)
 *   hash_raycast_tile_width  the same for the voxel-hash raycast (8)
 * The reference fixes its work-group sizes per kernel in its OpenCL sources. */
typedef struct nui_tuning {
  int integrate_threads_log2;
  int icp_pixels_per_thread;
  int raycast_tile_width;
  int hash_raycast_tile_width;
  int icp_cluster_blocks;
} nui_tuning;
NUI_API nui_status nui_ctx_get_tuning(nui_ctx* ctx, nui_tuning* out);
NUI_API nui_status nui_ctx_set_tuning(nui_ctx* ctx, const nui_tuning* t);
/* Autotuner: creates n scratch sessions of cfgs (device memory for all n at once), runs
 * `frames` frames of each through batch ticks (frame f of session i: depth_mm[i * frames
 * + f], host u16; bgra likewise or NULL), then times every candidate of each parameter in
 * turn (coordinate descent: integration, ICP, dense raycast, hash raycast; parameters no
 * session uses are skipped) as the median device time over `repeats` ticks of the
 * integration stage (integration) or of the whole graphed tick (the others); a setting
 * keeps its current value unless a candidate is at least 2 % faster,
 * keeps the fastest in the context, frees the scratch sessions and reports the choice
 * (out) and the whole-tick median with it (out_tick_ms, nullable).  Takes the context's
 * stream for the whole call. */
NUI_API nui_status nui_ctx_autotune(nui_ctx* ctx, const nui_session_cfg* cfgs, int n,
                                    const uint16_t* const* depth_mm, const uint8_t* const* bgra, int frames,
                                    int repeats, nui_tuning* out, float* out_tick_ms);
/* Hash global cache: blocks merged from the store and swapped out by the last frame,
 * store blocks in use, and swap-outs the full store refused (all NULL-able). */
NUI_API nui_status nui_hash_swap_stats(nui_session* s, int* swapped_in, int* swapped_out, int* store_used,
                                       int* store_refused);
/* The stored copy of hash entry `entry`: 512 sdf values (int16, or half for a half-sdf
 * session), 512 weights, 512 colours (4 bytes, alpha unused; zeros without colour), in
 * the pool's voxel order; *found = 0 if the entry has none.  Any output may be NULL. */
NUI_API nui_status nui_hash_stored_block(nui_session* s, int entry, void* sdf, uint8_t* weight, uint8_t* rgb4,
                                         int* found);
/* Shifting volume state (NuiKinfuOpenCLShiftScene m_voxel_offset / getVoxelOffsetSize,
 * NuiKinfuOpenCLShiftScene.cpp:58-66): the volume's offset in voxels and metres (the
 * camera's global translation is its pose's translation plus offset_m) and how many points
 * the slabs that left the volume gave (more than shift_point_cap: the cache overflowed).
 * Any pointer may be NULL. */
NUI_API nui_status nui_shift_state(nui_session* s, int* voxel_offset, float* offset_m, uint64_t* points_found);
/* The point cache of a shifting volume (the reference appends the same points to its
 * NuiKinfuVertexCache, NuiKinfuOpenCLShiftScene.cpp:206-228): copies up to cap points to
 * host xyz (3 floats each) / rgba (4 floats each) and returns in *n how many the cache
 * holds.  Points come in no fixed order (the kernel appends them atomically, like the
 * reference's). */
NUI_API nui_status nui_shift_points(nui_session* s, float* xyz, float* rgba, uint64_t cap, uint64_t* n);
NUI_API nui_status nui_shift_points_clear(nui_session* s);
/* Point cloud of a session's scene, Volume2CLVertices of the reference's scenes.  Dense:
 * fetchVolumeKernel (extract.cl:4-79, NuiKinfuOpenCLScene), or fetchShiftVolumeKernel
 * (extract.cl:82-179) over the whole buffer of a shifting volume
 * (NuiKinfuOpenCLShiftScene.cpp:354-520): a point per voxel whose tsdf is exactly 0 and per
 * sign change between z-neighbours.  Voxel hash: fetchHashScene_kernel
 * (KinfuHashVisualization.cl:5-52, NuiKinfuOpenCLHashScene.cpp:1066-1180) over the last
 * frame's visible blocks: a point per weighted voxel within the truncation band.  Points
 * carry their colour / 255 (0,0,0,1 without colour).  Writes up to cap points to device
 * d_xyz (3 floats each, 4-byte aligned) / d_rgba (4 floats each, 16-byte aligned) in no
 * fixed order and returns in *found how many exist.  Synchronous. */
NUI_API nui_status nui_point_cloud_device(nui_session* s, float* d_xyz, float* d_rgba, uint64_t cap,
                                          uint64_t* found);
/* Session snapshot / restore (checkpointing; the reference keeps no such state on disk).
 * A snapshot holds everything a session carries from frame to frame: the volume or the
 * hash table and voxel pool, the tracker state and pose, the reference maps of the last
 * raycast, the colour-tracking model colours and a shifting volume's offset and point
 * cache.  nui_session_snapshot_bytes gives its size; nui_session_snapshot copies it to
 * host memory (waits for the session's stream); nui_session_restore loads it into a
 * session created with the same configuration (NUI_ERR_INVALID_ARG otherwise), after
 * which the session continues exactly as the snapshotted one would have. */
NUI_API size_t nui_session_snapshot_bytes(nui_session* s);
NUI_API nui_status nui_session_snapshot(nui_session* s, void* host, size_t bytes);
NUI_API nui_status nui_session_restore(nui_session* s, const void* host, size_t bytes);
/* Voxels read-modify-written by the last integration of a session. */
NUI_API nui_status nui_session_touched_voxels(nui_session* s, uint64_t* n);
/* Work the kernels counted for the session's last frame, from which the algorithmic bytes of
 * each launch follow (no counterpart in the reference): out[0] voxels updated by the
 * integration, out[1] 8^3 bricks the tolerance-mode integration re-classified, out[2] voxel
 * reads of the tolerance-mode dense raycast march, out[3] march samples it visited, out[4]
 * crossings it refined, out[5..8] ICP iterations run at levels 0..3, out[9] 32 x 8 x 8 voxel
 * tiles the tolerance-mode integration ran (those its cull kept).  10 values. */
NUI_API nui_status nui_session_work_counters(nui_session* s, uint64_t* out);

/* ---------------------------------------------------------------- kernel-level calls
 * One entry point per reference kernel launch on the hot path, on device pointers,
 * launched on the context's stream (asynchronous).  Vertex/normal maps are float4 per
 * pixel (xyz, w = 0); depth maps float; volumes in the session layout are reached
 * through sessions only. */
/* depth_passing_filter_kernel + bilateral_filter_depth_kernel + depth2vertex_kernel +
 * scaleDepthsKernel (filters.cl:9-23, bilateralFilter.cl:68-119, transformMaps.cl:18-42,
 * tsdfVolume.cl:8-29), fused: raw u16 -> filtered depth, vertex map (level 0) and the
 * ray-length depth used by integration. */
NUI_API nui_status nui_k_preprocess(nui_ctx* ctx, const uint16_t* d_raw, int W, int H, float fx, float fy,
                                    float cx, float cy, float dmin, float dmax, int radius,
                                    float sigma_space2_inv_half, float sigma_depth2_inv_half, float depth_thr,
                                    float* d_filtered, float* d_vertex4, float* d_scaled);
/* half_sample_kernel + depth2vertex_kernel for one pyramid level (transformMaps.cl:18-88). */
NUI_API nui_status nui_k_pyramid_level(nui_ctx* ctx, const float* d_src, int dW, int dH, float fx, float fy,
                                       float cx, float cy, int div, float depth_thr, float* d_dst,
                                       float* d_vertex4);
/* estimate_normals_simple_kernel + transform_maps_kernel (normalEstimation.cl:770-822,
 * transformMaps.cl:91-127): camera vertices -> world vertex and normal maps.
 * pose12: R row-major + t (host pointer). */
NUI_API nui_status nui_k_feedback_maps(nui_ctx* ctx, const float* d_vertex4, int W, int H, float depth_thr,
                                       const float* pose12, float* d_vref4, float* d_nref4);

/* half_sample_bgra_kernel + bgra_gradient_kernel over a whole colour pyramid
 * (transformMaps.cl:106-146, 514-560; NuiKinfuOpenCLColorTracker::SubSampleColors /
 * GradientBuffers, NuiKinfuOpenCLColorTracker.cpp:125-242): d_bgra (W x H BGRA) is level 0;
 * d_levels[l] (l >= 1) receives level l ((W >> l) x (H >> l) BGRA, radius-1 box mean,
 * alpha 255); d_gx[l] / d_gy[l] receive the Sobel / 8 gradients of level l as signed
 * bytes (alpha 255, border 0).  Host arrays of `levels` device pointers (d_levels[0] is
 * not used). */
NUI_API nui_status nui_k_color_pyramid(nui_ctx* ctx, const uint8_t* d_bgra, int W, int H, int levels,
                                       uint8_t* const* d_levels, uint8_t* const* d_gx, uint8_t* const* d_gy);

/* ---------------------------------------------------------------- recorded frames
 * The reference's frame file format (NuiFileIOUtilities.cpp:13-161): int64 timestamp,
 * uint32 width, uint32 height, uint32 stored size, then the raw pixels or -- when the
 * stored size differs from width * height * pixel bytes -- their zlib stream
 * (compress2 at Z_BEST_SPEED).  Camera files (.camIntri) hold fx, fy, cx, cy as floats.
 * A recording is a directory of <n>.depth (uint16 mm), <n>.color (BGRA), <n>.camIntri,
 * n = 0, 1, ... (NuiFrameLoader.cpp:26-92). */
NUI_API nui_status nui_frame_file_write(const char* path, int compressed, int64_t timestamp, uint32_t width,
                                        uint32_t height, const void* pixels, uint32_t pixel_bytes);
NUI_API nui_status nui_frame_file_header(const char* path, int64_t* timestamp, uint32_t* width, uint32_t* height);
NUI_API nui_status nui_frame_file_read(const char* path, void* pixels, uint32_t bytes);
NUI_API nui_status nui_camera_file_write(const char* path, const float* fx_fy_cx_cy);
NUI_API nui_status nui_camera_file_read(const char* path, float* fx_fy_cx_cy);
/* Frame `index` of a recording: whichever of depth / colour / intrinsics the directory has
 * and the caller asks for (null pointers skip); NUI_ERR_INVALID_ARG past the last frame or
 * when the stored size is not width x height. */
NUI_API nui_status nui_recording_frame(const char* dir, int index, uint16_t* depth_mm, uint8_t* bgra,
                                       float* fx_fy_cx_cy, int64_t* timestamp, uint32_t width, uint32_t height);

#ifdef __cplusplus
}
#endif
#endif /* NUI_B200_H */
