// Host runtime of the C ABI: context (device + stream), sessions (device-resident state),
// the per-frame launch schedule, batched ticks under a CUDA graph, and the entry points
// declared in include/nui_b200.h.
//
// One frame of a session (NuiKinfuTrackingEngine::RunTracking, NuiKinfuTrackingEngine.cpp:68-142)
// is this fixed sequence of launches, each covering every session of the batch
// (blockIdx.y = session):
//   k_preprocess, k_pyramid x (levels-1), k_feedback, k_icp x sum(iterations),
//   k_track_finalize, k_integrate<fmt>, k_raycast<fmt>
// Which session does what in a tick (first frame / tracking / inactive) is data in the
// session table, so the same sequence serves every tick and is captured once.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <deque>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/nui_b200.h"
#include "nui_device.cuh"

namespace nui {
__global__ void k_preprocess(const SessionDesc*);
__global__ void k_pyramid(const SessionDesc*, int);
__global__ void k_feedback(const SessionDesc*);
__global__ void k_vertex_map(const SessionDesc*, int, float4*);
template <int PPT>
__global__ void k_icp_cluster(const SessionDesc*, int);
__global__ void k_track_finalize(const SessionDesc*, int, int);
__global__ void k_ztab(const SessionDesc*);
__global__ void k_color_level(const SessionDesc*, int);
__global__ void k_color_grad(const SessionDesc*, int);
__global__ void k_color_keep(const SessionDesc*, int);
template <int F>
__global__ void k_integrate(const SessionDesc*);
template <int F>
__global__ void k_integrate_fast(const SessionDesc*);
template <int F>
__global__ void k_integrate_cull(const SessionDesc*);
template <int F>
__global__ void k_volume_init(const SessionDesc*);
template <int F>
__global__ void k_brick_summary(const SessionDesc*, int);
__global__ void k_super_summary(const SessionDesc*, int);
template <int F>
__global__ void k_raycast(const SessionDesc*, int);
template <int F>
__global__ void k_raycast_finish(const SessionDesc*);
template <int F>
__global__ void k_raycast_fast(const SessionDesc*, int);
template <int F>
__global__ void k_raycast_finish_fast(const SessionDesc*);
__global__ void k_publish(const SessionDesc*, int, float*, int*, int);
__global__ void k_tick_begin(const SessionDesc*, int);
__global__ void k_hash_health(const SessionDesc*, int, int*);
__global__ void k_occ_clear(const SessionDesc*);
__global__ void k_hash_prepare(const SessionDesc*);
__global__ void k_hash_walk(const SessionDesc*, int);
__global__ void k_hash_count(const SessionDesc*, int);
__global__ void k_hash_flag_count(const SessionDesc*, int);
__global__ void k_hash_scan(const SessionDesc*, int);
__global__ void k_hash_alloc(const SessionDesc*);
__global__ void k_hash_alloc_done(const SessionDesc*, int);
__global__ void k_hash_visible(const SessionDesc*);
__global__ void k_hash_compact(const SessionDesc*);
template <int F>
__global__ void k_hash_integrate(const SessionDesc*);
__global__ void k_hash_range(const SessionDesc*);
__global__ void k_hash_project(const SessionDesc*);
template <int F>
__global__ void k_hash_raycast(const SessionDesc*, int);
template <int F>
__global__ void k_hash_finish(const SessionDesc*);
__global__ void k_fwd_project(const SessionDesc*);
__global__ void k_fwd_fill(const SessionDesc*);
__global__ void k_fwd_scan(const SessionDesc*);
__global__ void k_fwd_commit(const SessionDesc*);
template <int F>
__global__ void k_fwd_raycast(const SessionDesc*);
template <int F>
__global__ void k_fwd_finish(const SessionDesc*);
__global__ void k_fwd_normals(const SessionDesc*);
__global__ void k_hash_reset(const SessionDesc*);
__global__ void k_hash_swap_lists(const SessionDesc*);
template <int F>
__global__ void k_hash_swap_in(const SessionDesc*);
__global__ void k_hash_swap_out_list(const SessionDesc*);
template <int F>
__global__ void k_hash_swap_out(const SessionDesc*);
__global__ void k_hash_swap_clean(const SessionDesc*);
__global__ void k_hash_export_voxels(const SessionDesc*, uint8_t*);
template <int F>
__global__ void k_shift_fetch(const SessionDesc*, int);
template <int F>
__global__ void k_fetch_volume(const SessionDesc*, float*, float*, long long, unsigned long long*);
template <int F>
__global__ void k_hash_fetch(const SessionDesc*, float*, float*, long long, unsigned long long*);
template <typename T>
__global__ void k_shift_roll_x(const SessionDesc*, int);
template <typename T>
__global__ void k_shift_roll_yz(const SessionDesc*, int, int);
__global__ void k_shift_dirty(const SessionDesc*);
template <int F>
__global__ void k_export_ref(const SessionDesc*, short2*, uchar4*);
template <int F>
__global__ void k_import_ref(const SessionDesc*, const short2*);
}  // namespace nui

using namespace nui;

namespace {
thread_local std::string g_err;
nui_status fail(nui_status st, const std::string& msg) {
  g_err = msg;
  return st;
}
#define NUI_CUDA(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess) return fail(NUI_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Every device or pinned-host allocation the library makes goes through these, so that
// tests can check that an entry point allocates nothing (nui_debug_allocation_count).
std::atomic<unsigned long long> g_allocations{0};
cudaError_t counted_malloc(void** p, size_t bytes) {
  g_allocations.fetch_add(1, std::memory_order_relaxed);
  return cudaMalloc(p, bytes);
}
template <typename T>
cudaError_t counted_malloc(T** p, size_t bytes) {
  return counted_malloc(reinterpret_cast<void**>(p), bytes);
}
cudaError_t counted_malloc_host(void** p, size_t bytes) {
  g_allocations.fetch_add(1, std::memory_order_relaxed);
  return cudaMallocHost(p, bytes);
}
template <typename T>
cudaError_t counted_malloc_host(T** p, size_t bytes) {
  return counted_malloc_host(reinterpret_cast<void**>(p), bytes);
}
// Session state comes from the context's memory pool in stream order: allocation and free
// are queued on the context stream and never synchronise the device (a served stream can
// join or leave while a tick runs).
cudaError_t counted_pool_alloc(void** p, size_t bytes, cudaMemPool_t pool, cudaStream_t st) {
  g_allocations.fetch_add(1, std::memory_order_relaxed);
  return cudaMallocFromPoolAsync(p, bytes, pool, st);
}
cudaError_t counted_host_alloc(void** p, size_t bytes, unsigned flags) {
  g_allocations.fetch_add(1, std::memory_order_relaxed);
  return cudaHostAlloc(p, bytes, flags);
}
template <typename T>
cudaError_t counted_host_alloc(T** p, size_t bytes, unsigned flags) {
  return counted_host_alloc(reinterpret_cast<void**>(p), bytes, flags);
}

void noalloc_forget(int device);  // defined with nui_mesh_device_noalloc

// stage intervals: 0-5 consecutive stages, 6 the whole tick, 7 the dense raycast kernels,
// 8 the voxel-hash work on the side stream; kEvents events mark them
constexpr int kStages = 9;
constexpr int kEvents = 11;
constexpr size_t kMaxGraphs = 64;  // captured tick graphs kept per context
}  // namespace

struct nui_session;

// Launch shape of a batch; the key of the graph cache (compared bytewise, so the
// constructor zeroes every byte, padding included).
struct BatchPlan {
  int n;
  int maxW, maxH, maxLevels;
  int maxIters[kMaxLevels];
  long maxIntegThreads[4];  // per format: columns * zchunks
  long maxBricks[4];        // per format: 8^3 bricks
  long maxHyper;            // 128^3 regions, all dense formats
  long maxHashBlk;          // scan blocks of 1024 entries
  int hashMask;             // bit per hash sdf format
  int fmtMask;
  int colorIcp;             // some dense (bit 0) / hash (bit 1) session tracks with the photometric term
  int shiftFmtMask;         // bit per dense format of the shifting sessions
  int shiftColor;           // some shifting session has a colour volume
  int hashSwap;             // some hash session swaps blocks to the host
  int hashFwd, hashPlain;   // some hash session renders forward / raycasts every pixel
  // descriptor ranges: a batch table lists its non-hash slots first, so the dense kernels
  // launch over the first n - hashTail descriptors and the hash kernels over the last
  // n - denseHead (0, 0: both families over the whole table)
  int hashTail, denseHead;
  int anyFirst;             // some session of the batch has its first frame (frame-0 maps)
  nui_tuning tune;          // the context's launch shapes
  BatchPlan() { std::memset(this, 0, sizeof(*this)); }
  bool operator<(const BatchPlan& o) const { return std::memcmp(this, &o, sizeof(BatchPlan)) < 0; }
};

struct nui_ctx {
  int device = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  // the voxel-hash sessions' integration and raycast run beside the dense ones: a second
  // stream forked from and joined back to `stream` within each tick (and its graph)
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  bool timing = false;
  bool side_timed = false;  // the last timed tick ran voxel-hash work on the side stream
  cudaEvent_t ev[kEvents] = {};
  float stage_ms[kStages] = {};
  // batch table (device + pinned staging) and per-session outputs (status + pose).  The
  // host sides come in two halves used by alternate ticks (`par`), so that a tick can be
  // launched while the previous one's results are still to be read; ev_tick[par] is
  // recorded behind the last tick that used half par.
  int cap = 0;
  SessionDesc* d_descs = nullptr;
  SessionDesc* h_descs = nullptr;  // 2 * cap
  float* d_pose = nullptr;  // cap * 14: R(9) t(3) err count
  int* d_status = nullptr;  // cap * 2: status, integrate
  float* h_pose = nullptr;  // 2 * cap * 14
  int* h_status = nullptr;  // 2 * cap * 2
  int par = 0;              // the half the next tick uses
  cudaEvent_t ev_tick[2] = {nullptr, nullptr};
  // scratch descriptor for kernel-level calls
  SessionDesc* d_kdesc = nullptr;
  TrackState* d_kts = nullptr;
  unsigned long long* d_count = nullptr;  // counter of the point-cloud fetch
  struct Graph {
    cudaGraphExec_t exec;
    int kernels;  // kernel launches per replay
  };
  std::map<BatchPlan, Graph> graphs;
  int last_kernels = 0;  // kernels of the last graphed tick
  nui_tuning tune = {18, 4, 8, 8, 12};
  cudaMemPool_t pool = nullptr;  // session state (stream-ordered; freed memory stays here)
};

struct nui_session {
  nui_ctx* ctx = nullptr;
  nui_session_cfg cfg;
  DevCam cam;
  float cell[3], trunc;
  unsigned icp_min_count[kMaxLevels] = {0, 0, 0, 0};
  float gauss[2 * kMaxRadius + 1];
  uint16_t* raw = nullptr;
  uint8_t* bgra = nullptr;
  float* dscaled = nullptr;
  float* dlev[kMaxLevels] = {};  // depth pyramid (vertices are rebuilt from it where used)
  float4 *vref = nullptr, *nref = nullptr;
  uchar4* cmap = nullptr;
  void* vol = nullptr;
  uint8_t* wvol = nullptr;
  uchar4* cvol = nullptr;
  uint8_t* occ = nullptr;
  uint8_t* occ2 = nullptr;
  float* ztab = nullptr;
  unsigned* fast_tiles = nullptr;
  uint8_t* occ3 = nullptr;
  float* tile_max = nullptr;
  TrackState* ts = nullptr;
  uchar4* cprev = nullptr;        // colour tracking: the previous frame's colours and the
  uchar4* cgx[kMaxLevels] = {};   // current frame's gradients (level 0)
  uchar4* cgy[kMaxLevels] = {};
  float* pts_xyz = nullptr;   // shifting volume: point cache of the slabs that left
  float* pts_rgba = nullptr;
  SessionDesc* d_desc1 = nullptr;
  // voxel-block hash
  bool hash = false;
  HEntry* entries = nullptr;
  void* hsdf = nullptr;
  uint8_t* hw = nullptr;
  uchar4* hrgb = nullptr;
  int *alloc_list = nullptr, *excess_list = nullptr, *hcount = nullptr, *vis_ids = nullptr;
  uint8_t *alloc_type = nullptr, *vis = nullptr;
  short4* coords = nullptr;
  unsigned long long* keys = nullptr;
  unsigned* blk = nullptr;
  float2* range = nullptr;  // one-entry table for the per-session path
  int *fwd_owner = nullptr, *fwd_ids = nullptr;  // forward rendering scratch
  unsigned* fwd_blk = nullptr;
  uchar4* fwd_col = nullptr;

  long frames = 0;
  bool color_frame = false;
  std::vector<void*> allocs;
  std::vector<void*> host_allocs;  // pinned, mapped (the hash global cache's store)
  // hash global cache
  uint8_t* swap = nullptr;
  int* store_slot = nullptr;
  int *swap_in_ids = nullptr, *swap_out_ids = nullptr;
  void* st_sdf = nullptr;  // device-mapped host pointers
  uint8_t* st_w = nullptr;
  uchar4* st_rgb = nullptr;
  void* h_st_sdf = nullptr;  // the same memory, host pointers
  uint8_t* h_st_w = nullptr;
  uchar4* h_st_rgb = nullptr;
  int st_cap = 0;
};

// ------------------------------------------------------------------ helpers
namespace {

size_t voxel_bytes(int fmt) { return fmt == NUI_TSDF_F32 ? 8 : (fmt == NUI_TSDF_F16_U8 ? 3 : 4); }

bool cfg_valid(const nui_session_cfg* c, std::string& why) {
  if (!c) return why = "null config", false;
  if (c->width <= 0 || c->height <= 0 || c->width > 4096 || c->height > 4096) return why = "bad image size", false;
  if (c->levels < 1 || c->levels > kMaxLevels) return why = "levels must be 1..4", false;
  for (int l = 0; l < c->levels; ++l) {
    if (c->iterations[l] < 0 || c->iterations[l] > 100) return why = "bad iteration count", false;
    if ((c->width >> l) < 2 || (c->height >> l) < 2) return why = "too many levels for the image", false;
    if (((c->width >> l) << l) != c->width || ((c->height >> l) << l) != c->height)
      return why = "image size must be divisible by 2^(levels-1)", false;
  }
  if (c->volume_kind != NUI_VOLUME_DENSE && c->volume_kind != NUI_VOLUME_HASH) return why = "bad volume kind", false;
  if (c->tsdf_format < 0 || c->tsdf_format > 3) return why = "bad tsdf format", false;
  if (c->volume_kind == NUI_VOLUME_HASH) {
    if (c->hash_buckets < 16 || (c->hash_buckets & (c->hash_buckets - 1))) return why = "hash buckets must be a power of two >= 16", false;
    if (c->hash_excess < 1 || c->hash_pool_blocks < 1 || (long)c->hash_buckets + c->hash_excess > (1L << 28))
      return why = "bad hash table sizes", false;
    if ((long)c->hash_pool_blocks > (1L << 22)) return why = "hash pool larger than 2^22 blocks", false;
    if (!(c->voxel_size > 0.f) || !(c->trunc_scale > 0.f)) return why = "voxel size / truncation must be positive", false;
    if (c->hash_max_weight < 1 || c->hash_max_weight > 255) return why = "hash max weight must be 1..255", false;
  }
  for (int i = 0; i < 3 && c->volume_kind == NUI_VOLUME_DENSE; ++i) {
    if (c->res[i] < 8 || c->res[i] > 1024) return why = "volume resolution must be 8..1024", false;
    if (!(c->dim[i] > 0.f)) return why = "volume size must be positive", false;
  }
  if (c->filter_radius < 0 || c->filter_radius > kMaxRadius) return why = "filter radius must be 0..7", false;
  if (!(c->fx > 0.f) || !(c->fy > 0.f)) return why = "focal lengths must be positive", false;
  if (!(c->photometric_weight >= 0.f) || !(c->photometric_weight < 1e30f))
    return why = "photometric weight must be finite and >= 0", false;
  if (c->photometric_weight > 0.f && !c->color_volume) return why = "colour tracking needs color_volume = 1", false;
  if (c->voxel_shift < 0 || c->shift_point_cap < 0) return why = "voxel shift and point cap must be >= 0", false;
  if (c->hash_swapping && c->volume_kind != NUI_VOLUME_HASH) return why = "swapping needs a voxel-hash volume", false;
  if (c->hash_store_blocks < 0) return why = "hash store blocks must be >= 0", false;
  if (c->hash_forward_render < 0 || c->hash_forward_render > 2) return why = "hash forward render must be 0, 1 or 2", false;
  if (c->hash_forward_render && c->volume_kind != NUI_VOLUME_HASH)
    return why = "forward rendering needs a voxel-hash volume", false;
  if (c->hash_forward_render && (long)c->width * c->height > 1024L * 1024L)
    return why = "forward rendering: images up to 2^20 pixels", false;
  if (c->voxel_shift > 0) {
    if (c->volume_kind != NUI_VOLUME_DENSE) return why = "a shifting volume must be dense", false;
    for (int i = 0; i < 3; ++i) {
      if (c->voxel_shift >= c->res[i]) return why = "voxel shift must be below the volume resolution", false;
      if (!(c->shift_basis[i] > -1e30f && c->shift_basis[i] < 1e30f)) return why = "shift basis must be finite", false;
    }
  }
  return true;
}

// ICP valid-count threshold per level.  The reference computes it from
// kernelGlobalSize[0], which after the first level still holds the global size of the
// last compute_sums launch (NuiKinfuOpenCLDepthTracker.cpp:309, 342, 368); reproduced.
void icp_thresholds(const nui_session_cfg& c, unsigned* out) {
  size_t g = (size_t)c.width * c.height;
  for (int lv = c.levels - 1; lv >= 0; --lv) {
    out[lv] = (unsigned)((double)(g >> (2 * lv)) * 0.1);
    if (c.iterations[lv] > 0) {
      size_t n = (size_t)(c.width >> lv) * (c.height >> lv);
      unsigned size = (unsigned)std::ceil((float)n / 128.f);
      unsigned nb = (unsigned)std::ceil((float)size / 128.f);
      g = (size_t)nb * 128;
    }
  }
}

// Integration z chunks of a volume: threads per launch >= 2^log2_threads, every chunk
// >= 16 slices.  The chunking changes no result (every chunk replays its column's sums).
int pick_zchunks(const nui_session_cfg& c, int log2_threads) {
  const long ncol = (long)c.res[0] * c.res[1], target = 1L << log2_threads;
  int z = (int)std::max(1L, (target + ncol - 1) / ncol);
  return std::min(z, std::max(1, c.res[2] / 16));
}

void fill_desc(const nui_session* s, SessionDesc& d, int kind, const uint16_t* raw, const uint8_t* bgra) {
  std::memset(&d, 0, sizeof(d));
  const nui_session_cfg& c = s->cfg;
  d.kind = kind;
  d.W = c.width;
  d.H = c.height;
  d.levels = c.levels;
  d.cam = s->cam;
  d.radius = c.filter_radius;
  d.sigma_depth = c.sigma_depth2_inv_half;
  d.depth_thr = c.depth_threshold;
  std::memcpy(d.gauss, s->gauss, sizeof(d.gauss));
  d.dist_thr = c.dist_threshold + c.dist_threshold / (float)c.levels;
  for (int l = 0; l < kMaxLevels; ++l) {
    d.iters[l] = l < c.levels ? c.iterations[l] : 0;
    d.icp_min_count[l] = s->icp_min_count[l];
    d.dlev[l] = s->dlev[l];
  }
  d.integ_thr = c.integration_threshold;
  d.raw = raw;
  d.bgra = bgra;
  d.dscaled = s->dscaled;
  d.vref = s->vref;
  d.nref = s->nref;
  d.cmap = s->cmap;
  d.tile_max = s->tile_max;
  d.fmt = c.tsdf_format;
  for (int i = 0; i < 3; ++i) {
    d.res[i] = c.res[i];
    d.dim[i] = c.dim[i];
    d.cell[i] = s->cell[i];
  }
  d.trunc = s->trunc;
  d.vol = s->vol;
  d.wvol = s->wvol;
  d.cvol = s->cvol;
  d.occ = s->occ;
  d.occ2 = s->occ2;
  d.ztab = s->ztab;
  d.tol = c.tsdf_format >= NUI_TSDF_F16_U8 ? 1 : 0;
  d.fast_tiles = s->fast_tiles;
  d.occ3 = s->occ3;
  d.max_cw = c.max_color_weight;
  d.zchunks = pick_zchunks(s->cfg, s->ctx->tune.integrate_threads_log2);
  d.voxel_shift = s->hash ? 0 : c.voxel_shift;
  for (int i = 0; i < 3; ++i) d.shift_basis[i] = c.shift_basis[i];
  d.pts_xyz = s->pts_xyz;
  d.pts_rgba = s->pts_rgba;
  d.pts_cap = s->pts_xyz ? c.shift_point_cap : 0;
  d.ts = s->ts;
  // colour tracking runs on frames that carry colour, once its buffers exist
  d.photo_w = (bgra && s->cgx[0] && s->cprev) ? s->cfg.photometric_weight : 0.f;
  d.cprev = s->cprev;
  for (int l = 0; l < kMaxLevels; ++l) {
    d.cpyr[l] = nullptr;
    d.cgx[l] = s->cgx[l];
    d.cgy[l] = s->cgy[l];
  }
  if (s->hash) {
    d.fmt = -1;  // dense kernels skip hash sessions
    d.hash = 1;
    d.hfmt = c.tsdf_format == NUI_TSDF_I16 ? 0 : 1;
    d.entries = s->entries;
    d.nb = c.hash_buckets;
    d.ne = c.hash_excess;
    d.np = c.hash_pool_blocks;
    d.hmask = (unsigned)(c.hash_buckets - 1);
    d.voxel = c.voxel_size;
    d.mu = c.trunc_scale;
    d.max_w = c.hash_max_weight;
    d.hsdf = s->hsdf;
    d.hw = s->hw;
    d.hrgb = s->hrgb;
    d.alloc_list = s->alloc_list;
    d.excess_list = s->excess_list;
    d.hcount = s->hcount;
    d.swapping = c.hash_swapping ? 1 : 0;
    d.swap = s->swap;
    d.store_slot = s->store_slot;
    d.swap_in_ids = s->swap_in_ids;
    d.swap_out_ids = s->swap_out_ids;
    d.st_sdf = s->st_sdf;
    d.st_w = s->st_w;
    d.st_rgb = s->st_rgb;
    d.st_cap = s->st_cap;
    d.alloc_type = s->alloc_type;
    d.vis = s->vis;
    d.coords = s->coords;
    d.keys = s->keys;
    d.vis_ids = s->vis_ids;
    d.blk = s->blk;
    d.range = s->range;
    d.fwd = c.hash_forward_render;
    d.fwd_owner = s->fwd_owner;
    d.fwd_ids = s->fwd_ids;
    d.fwd_blk = s->fwd_blk;
    d.fwd_col = s->fwd_col;
  }
}

void plan_add(BatchPlan& p, const nui_session* s) {
  const nui_session_cfg& c = s->cfg;
  p.tune = s->ctx->tune;
  p.maxW = std::max(p.maxW, c.width);
  p.maxH = std::max(p.maxH, c.height);
  p.maxLevels = std::max(p.maxLevels, c.levels);
  if (c.photometric_weight > 0.f) p.colorIcp |= s->hash ? 2 : 1;
  for (int l = 0; l < c.levels; ++l) p.maxIters[l] = std::max(p.maxIters[l], c.iterations[l]);
  if (s->hash) {
    p.hashMask |= 1 << (c.tsdf_format == NUI_TSDF_I16 ? 0 : 1);
    if (c.hash_swapping) p.hashSwap = 1;
    (c.hash_forward_render ? p.hashFwd : p.hashPlain) = 1;
    p.maxHashBlk = std::max(p.maxHashBlk, ((long)c.hash_buckets + c.hash_excess + 1023) / 1024);
    return;
  }
  long th = (long)c.res[0] * c.res[1] * pick_zchunks(c, p.tune.integrate_threads_log2);
  p.maxIntegThreads[c.tsdf_format] = std::max(p.maxIntegThreads[c.tsdf_format], th);
  p.fmtMask |= 1 << c.tsdf_format;
  const long nb = (long)((c.res[0] + 7) / 8) * ((c.res[1] + 7) / 8) * ((c.res[2] + 7) / 8);
  p.maxBricks[c.tsdf_format] = std::max(p.maxBricks[c.tsdf_format], nb);
  const long nh = (long)((c.res[0] + 127) / 128) * ((c.res[1] + 127) / 128) * ((c.res[2] + 127) / 128);
  p.maxHyper = std::max(p.maxHyper, nh);
  if (c.voxel_shift > 0) {
    p.shiftFmtMask |= 1 << c.tsdf_format;
    if (c.color_volume) p.shiftColor = 1;
  }
}

// Elementwise maximum of two launch shapes (n stays a's).
void plan_merge(BatchPlan& a, const BatchPlan& b) {
  a.maxW = std::max(a.maxW, b.maxW);
  a.maxH = std::max(a.maxH, b.maxH);
  a.maxLevels = std::max(a.maxLevels, b.maxLevels);
  for (int l = 0; l < kMaxLevels; ++l) a.maxIters[l] = std::max(a.maxIters[l], b.maxIters[l]);
  for (int f = 0; f < 4; ++f) {
    a.maxIntegThreads[f] = std::max(a.maxIntegThreads[f], b.maxIntegThreads[f]);
    a.maxBricks[f] = std::max(a.maxBricks[f], b.maxBricks[f]);
  }
  a.maxHyper = std::max(a.maxHyper, b.maxHyper);
  a.maxHashBlk = std::max(a.maxHashBlk, b.maxHashBlk);
  a.hashMask |= b.hashMask;
  a.fmtMask |= b.fmtMask;
  a.colorIcp |= b.colorIcp;
  a.shiftFmtMask |= b.shiftFmtMask;
  a.shiftColor |= b.shiftColor;
  a.hashSwap |= b.hashSwap;
}

unsigned cdiv(long a, long b) { return (unsigned)((a + b - 1) / b); }
unsigned dense_n(const BatchPlan& p) { return (unsigned)(p.n - p.hashTail); }



template <int F>
void launch_integrate(const BatchPlan& p, const SessionDesc* d, cudaStream_t st) {
  if (!(p.fmtMask & (1 << F))) return;
  if (F >= NUI_TSDF_F16_U8) {  // tolerance mode: cull the 32 x 8 x 8 tiles, then a warp per kept tile
    const long tiles = p.maxBricks[F] / 4 + 1;  // >= the tiles of any session of the format
    k_integrate_cull<F><<<dim3(cdiv(tiles, 256), dense_n(p)), 256, 0, st>>>(d);
    const long blocks = std::min<long>(cdiv(tiles, 32 * kFastWarps), 1024);
    const int smem = kFastWarps * kFastWarpSmem;
    static std::once_flag opt_in;  // more than 48 KB of dynamic shared memory a block
    std::call_once(opt_in, [&] { cudaFuncSetAttribute(k_integrate_fast<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); });
    k_integrate_fast<F><<<dim3((unsigned)std::max<long>(blocks, 1), dense_n(p)), 32 * kFastWarps, smem, st>>>(d);
    return;
  }
  k_integrate<F><<<dim3(cdiv(p.maxIntegThreads[F], 256), dense_n(p)), 256, 0, st>>>(d);
}
template <int F>
void launch_summary(const BatchPlan& p, const SessionDesc* d, cudaStream_t st, int force) {
  if (!(p.fmtMask & (1 << F))) return;
  // the tolerance-mode integration re-classifies the bricks it updates itself: bricks of
  // those formats are left dirty only by a shift (or an import, which forces the pass)
  if (F >= NUI_TSDF_F16_U8 && !force && !(p.shiftFmtMask & (1 << F))) return;
  k_brick_summary<F><<<dim3(cdiv(p.maxBricks[F], 1024), dense_n(p)), 256, 0, st>>>(d, force);
}
// Brick re-classification after integration, then the super-bricks it touched.
void launch_summaries(const BatchPlan& p, const SessionDesc* d, cudaStream_t st, int force) {
  launch_summary<0>(p, d, st, force);
  launch_summary<1>(p, d, st, force);
  launch_summary<2>(p, d, st, force);
  launch_summary<3>(p, d, st, force);
  if (p.fmtMask) k_super_summary<<<dim3((unsigned)p.maxHyper, dense_n(p)), 64, 0, st>>>(d, force);
}
// Blocks of the raycasts: 2 x 2 warps, each a tw x (32 / tw) pixel tile.
unsigned ray_blocks(const BatchPlan& p, int tw) { return cdiv(p.maxW, 2 * tw) * cdiv(p.maxH, 2 * (32 / tw)); }
template <int F>
void launch_raycast(const BatchPlan& p, const SessionDesc* d, cudaStream_t st) {
  if (!(p.fmtMask & (1 << F))) return;
  const int tw = p.tune.raycast_tile_width;
  if (F >= NUI_TSDF_F16_U8) {  // tolerance mode
    k_raycast_fast<F><<<dim3(ray_blocks(p, tw), dense_n(p)), 128, 0, st>>>(d, tw);
    k_raycast_finish_fast<F><<<dim3(cdiv((long)p.maxW * p.maxH, 256), dense_n(p)), 256, 0, st>>>(d);
    return;
  }
  k_raycast<F><<<dim3(ray_blocks(p, tw), dense_n(p)), 128, 0, st>>>(d, tw);
  k_raycast_finish<F><<<dim3(cdiv((long)p.maxW * p.maxH, 256), dense_n(p)), 256, 0, st>>>(d);
}

void launch_hash_integrate(const BatchPlan& p, const SessionDesc* d0, cudaStream_t st) {
  if (!p.hashMask) return;
  const SessionDesc* d = d0 + p.denseHead;
  const unsigned hn = (unsigned)(p.n - p.denseHead);
  const unsigned nb = (unsigned)p.maxHashBlk;
  k_hash_prepare<<<dim3(592, hn), 256, 0, st>>>(d);
  const unsigned pix = cdiv((long)p.maxW * p.maxH, 256);
  k_hash_walk<<<dim3(pix, hn), 256, 0, st>>>(d, 0);
  k_hash_walk<<<dim3(pix, hn), 256, 0, st>>>(d, 1);
  k_hash_flag_count<<<dim3(nb, hn), 64, 0, st>>>(d, 0);
  k_hash_scan<<<hn, 1024, 0, st>>>(d, 0);
  k_hash_alloc<<<dim3(nb, hn), 64, 0, st>>>(d);
  k_hash_alloc_done<<<cdiv(hn, 64), 64, 0, st>>>(d, (int)hn);
  k_hash_visible<<<dim3(592, hn), 256, 0, st>>>(d);
  k_hash_flag_count<<<dim3(nb, hn), 64, 0, st>>>(d, 1);
  k_hash_scan<<<hn, 1024, 0, st>>>(d, 1);
  k_hash_compact<<<dim3(nb, hn), 64, 0, st>>>(d);
  if (p.hashSwap) {  // global cache: re-allocations and the swap-in list
    k_hash_count<<<dim3(nb, hn), 256, 0, st>>>(d, 2);
    k_hash_scan<<<hn, 1024, 0, st>>>(d, 2);
    k_hash_swap_lists<<<dim3(nb, hn), 1024, 0, st>>>(d);
  }
  if (p.hashMask & 1) k_hash_integrate<0><<<dim3(1184, hn), 512, 0, st>>>(d);
  if (p.hashMask & 2) k_hash_integrate<1><<<dim3(1184, hn), 512, 0, st>>>(d);
  if (p.hashSwap) {  // global cache: swap in, then swap out
    if (p.hashMask & 1) k_hash_swap_in<0><<<dim3(1184, hn), 512, 0, st>>>(d);
    if (p.hashMask & 2) k_hash_swap_in<1><<<dim3(1184, hn), 512, 0, st>>>(d);
    k_hash_count<<<dim3(nb, hn), 256, 0, st>>>(d, 3);
    k_hash_scan<<<hn, 1024, 0, st>>>(d, 3);
    k_hash_swap_out_list<<<dim3(nb, hn), 1024, 0, st>>>(d);
    if (p.hashMask & 1) k_hash_swap_out<0><<<dim3(1184, hn), 512, 0, st>>>(d);
    if (p.hashMask & 2) k_hash_swap_out<1><<<dim3(1184, hn), 512, 0, st>>>(d);
    k_hash_swap_clean<<<hn, 1024, 0, st>>>(d);
  }
}
void launch_hash_raycast(const BatchPlan& p, const SessionDesc* d0, cudaStream_t st) {
  if (!p.hashMask) return;
  const SessionDesc* d = d0 + p.denseHead;
  const unsigned hn = (unsigned)(p.n - p.denseHead);
  k_hash_range<<<dim3(296, hn), 256, 0, st>>>(d);
  k_hash_project<<<dim3(296, hn), 256, 0, st>>>(d);
  const unsigned px = cdiv((long)p.maxW * p.maxH, 256);
  if (p.hashFwd) {  // forward rendering: land the previous vertices, cast the missing pixels
    const unsigned px1k = cdiv((long)p.maxW * p.maxH, 1024), pl = cdiv((long)p.maxW * p.maxH, 128);
    k_fwd_project<<<dim3(296, hn), 256, 0, st>>>(d);
    k_fwd_fill<<<dim3(px1k, hn), 1024, 0, st>>>(d);
    k_fwd_scan<<<dim3(1, hn), 1024, 0, st>>>(d);
    k_fwd_commit<<<dim3(px1k, hn), 1024, 0, st>>>(d);
    if (p.hashMask & 1) k_fwd_raycast<0><<<dim3(pl, hn), 128, 0, st>>>(d);
    if (p.hashMask & 2) k_fwd_raycast<1><<<dim3(pl, hn), 128, 0, st>>>(d);
    if (p.hashMask & 1) k_fwd_finish<0><<<dim3(px, hn), 256, 0, st>>>(d);
    if (p.hashMask & 2) k_fwd_finish<1><<<dim3(px, hn), 256, 0, st>>>(d);
    k_fwd_normals<<<dim3(px, hn), 256, 0, st>>>(d);
  }
  if (!p.hashPlain) return;
  const int tw = p.tune.hash_raycast_tile_width;
  const unsigned tiles = ray_blocks(p, tw);
  if (p.hashMask & 1) k_hash_raycast<0><<<dim3(tiles, hn), 128, 0, st>>>(d, tw);
  if (p.hashMask & 2) k_hash_raycast<1><<<dim3(tiles, hn), 128, 0, st>>>(d, tw);
  if (p.hashMask & 1) k_hash_finish<0><<<dim3(px, hn), 256, 0, st>>>(d);
  if (p.hashMask & 2) k_hash_finish<1><<<dim3(px, hn), 256, 0, st>>>(d);
}

// The shifts of the shifting volumes (after tracking, before integration): per axis, the
// leaving slab's points, then the roll of every per-voxel array; then all bricks dirty.
// Without a shift every launch returns at once.
constexpr unsigned kShiftBlocks = 592;
template <int F>
void launch_shift_fetch(const BatchPlan& p, const SessionDesc* d, cudaStream_t st, int axis) {
  if (p.shiftFmtMask & (1 << F)) k_shift_fetch<F><<<dim3(kShiftBlocks, dense_n(p)), 256, 0, st>>>(d, axis);
}
template <typename T>
void launch_roll(const BatchPlan& p, const SessionDesc* d, cudaStream_t st, int axis, int which) {
  if (axis == 0)
    k_shift_roll_x<T><<<dim3(kShiftBlocks, dense_n(p)), 256, 0, st>>>(d, which);
  else
    k_shift_roll_yz<T><<<dim3(kShiftBlocks, dense_n(p)), 256, 0, st>>>(d, axis, which);
}
void launch_shift(const BatchPlan& p, const SessionDesc* d, cudaStream_t st) {
  if (!p.shiftFmtMask) return;
  for (int axis = 0; axis < 3; ++axis) {
    launch_shift_fetch<0>(p, d, st, axis);
    launch_shift_fetch<1>(p, d, st, axis);
    launch_shift_fetch<2>(p, d, st, axis);
    launch_shift_fetch<3>(p, d, st, axis);
    if (p.shiftFmtMask & 0b1001) launch_roll<uint32_t>(p, d, st, axis, 0);  // short2, half2
    if (p.shiftFmtMask & 0b0010) launch_roll<unsigned long long>(p, d, st, axis, 0);  // float2
    if (p.shiftFmtMask & 0b0100) {  // half plane + u8 weight plane
      launch_roll<uint16_t>(p, d, st, axis, 0);
      launch_roll<uint8_t>(p, d, st, axis, 1);
    }
    if (p.shiftColor) launch_roll<uint32_t>(p, d, st, axis, 2);
  }
  k_shift_dirty<<<dim3(kShiftBlocks, dense_n(p)), 256, 0, st>>>(d);
}

// The ICP kernel over n sessions, one cluster of cl blocks each (cl = 16 is beyond the
// portable cluster size and needs the kernel's opt-in, given once per kernel).
void launch_icp_cluster(void (*kern)(const SessionDesc*, int), const SessionDesc* d, int n, int cl, int fam,
                        cudaStream_t st) {
  {
    static std::mutex mu;
    static std::vector<const void*> opted;
    std::lock_guard<std::mutex> lock(mu);
    if (std::find(opted.begin(), opted.end(), (const void*)kern) == opted.end()) {
      cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      opted.push_back((const void*)kern);
    }
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cl, n);
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cl;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, d, fam);
}

// Colour pyramid (if any session tracks with colour), the ICP iterations of every level,
// the integration gate and the published pose, for the sessions of family fam among the n
// descriptors at d.
void launch_track(const BatchPlan& p, const SessionDesc* d, int n, cudaStream_t st, float* d_pose, int* d_status,
                  bool color, int fam = kFamAll, bool tick = true) {
  if (n <= 0) return;
  const unsigned npix = cdiv((long)p.maxW * p.maxH, 256);
  if (color) k_color_grad<<<dim3(npix, n, 1), 256, 0, st>>>(d, fam);  // finest level
  // every level and iteration of every session in one launch: a cluster of
  // icp_cluster_blocks blocks per session
  const int ppt = p.tune.icp_pixels_per_thread;
  const int cl = p.tune.icp_cluster_blocks;
  if (ppt == 2) launch_icp_cluster(k_icp_cluster<2>, d, n, cl, fam, st);
  else if (ppt == 8) launch_icp_cluster(k_icp_cluster<8>, d, n, cl, fam, st);
  else if (ppt == 16) launch_icp_cluster(k_icp_cluster<16>, d, n, cl, fam, st);
  else launch_icp_cluster(k_icp_cluster<4>, d, n, cl, fam, st);
  k_track_finalize<<<n, 32, 0, st>>>(d, tick ? 1 : 0, fam);
  k_publish<<<cdiv(n, 64), 64, 0, st>>>(d, n, d_pose, d_status, fam);
  if (color) k_color_keep<<<dim3(cdiv(((long)p.maxW * p.maxH + 3) / 4, 256), n), 256, 0, st>>>(d, fam);
}

// The launch schedule of one tick.  ev: optional stage events (timing only).
void enqueue_tick(nui_ctx* ctx, const BatchPlan& p, const SessionDesc* d, float* d_pose, int* d_status, bool ev) {
  cudaStream_t st = ctx->stream;
  auto mark = [&](int i) {
    if (ev) cudaEventRecord(ctx->ev[i], st);
  };
  mark(0);
  k_tick_begin<<<cdiv(p.n, 64), 64, 0, st>>>(d, p.n);
  const unsigned tiles = cdiv(p.maxW, 32) * cdiv(p.maxH, 16);
  k_preprocess<<<dim3(tiles, p.n), dim3(kPreBlockX, kPreBlockY), 0, st>>>(d);
  mark(1);
  for (int l = 1; l < p.maxLevels; ++l)
    k_pyramid<<<dim3(cdiv((long)(p.maxW >> l) * (p.maxH >> l), 256), p.n), 256, 0, st>>>(d, l);
  if (p.anyFirst) k_feedback<<<dim3(cdiv((long)p.maxW * p.maxH, 256), p.n), 256, 0, st>>>(d);
  mark(2);
  // With dense and hash sessions in the batch, the hash sessions' tracking, allocation,
  // integration and raycast run on the side stream, beside the dense ones: the two sets of
  // kernels touch disjoint sessions, the dense integration starts as soon as the dense
  // sessions are tracked (instead of after the longer colour-tracked hash sessions), and
  // the many short kernels of the hash allocation fill the gaps of the dense integration.
  // A served batch, whose table keeps one launch shape while streams of either family come
  // and go, launches both trackings over the whole table, each skipping the other family.
  const bool fork = p.hashMask && p.fmtMask;
  const bool ranged = p.hashTail > 0 && p.denseHead > 0;
  cudaStream_t hs = fork ? ctx->side : st;
  if (fork) {
    cudaEventRecord(ctx->fork_ev, st);
    cudaStreamWaitEvent(hs, ctx->fork_ev, 0);
    if (ev) cudaEventRecord(ctx->ev[9], hs);
    if (ranged) {
      launch_track(p, d + p.denseHead, p.n - p.denseHead, hs, d_pose, d_status, (p.colorIcp & 2) != 0);
      launch_track(p, d, p.denseHead, st, d_pose, d_status, (p.colorIcp & 1) != 0);
    } else {
      launch_track(p, d, p.n, hs, d_pose, d_status, (p.colorIcp & 2) != 0, kFamHash);
      launch_track(p, d, p.n, st, d_pose, d_status, (p.colorIcp & 1) != 0, kFamDense);
    }
  } else {
    launch_track(p, d, p.n, st, d_pose, d_status, p.colorIcp != 0);
  }
  mark(3);
  if (ev) ctx->side_timed = fork;
  if (fork) {
    launch_hash_integrate(p, d, hs);
    launch_hash_raycast(p, d, hs);
    if (ev) cudaEventRecord(ctx->ev[10], hs);
  }
  launch_shift(p, d, st);
  launch_integrate<0>(p, d, st);
  launch_integrate<1>(p, d, st);
  launch_integrate<2>(p, d, st);
  launch_integrate<3>(p, d, st);
  mark(4);
  launch_summaries(p, d, st, 0);
  if (!fork) launch_hash_integrate(p, d, st);
  mark(5);
  mark(7);
  launch_raycast<0>(p, d, st);
  launch_raycast<1>(p, d, st);
  launch_raycast<2>(p, d, st);
  launch_raycast<3>(p, d, st);
  mark(8);
  if (fork) {
    cudaEventRecord(ctx->join_ev, hs);
    cudaStreamWaitEvent(st, ctx->join_ev, 0);
  } else {
    launch_hash_raycast(p, d, st);
  }
  if (p.hashMask) k_hash_health<<<cdiv(p.n, 64), 64, 0, st>>>(d, p.n, d_status);
  mark(6);
}

nui_status ensure_cap(nui_ctx* ctx, int n) {
  if (n <= ctx->cap) return NUI_OK;
  int cap = std::max(n, std::max(64, ctx->cap * 2));
  cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second.exec);
  ctx->graphs.clear();
  float* old_pose = ctx->h_pose;  // results of a tick not yet read move to the new arrays
  int* old_status = ctx->h_status;
  const int old_cap = ctx->cap;
  cudaFree(ctx->d_descs);
  cudaFreeHost(ctx->h_descs);
  cudaFree(ctx->d_pose);
  cudaFree(ctx->d_status);
  ctx->h_pose = nullptr;
  ctx->h_status = nullptr;
  NUI_CUDA(counted_malloc(&ctx->d_descs, sizeof(SessionDesc) * cap));
  NUI_CUDA(counted_malloc_host(&ctx->h_descs, sizeof(SessionDesc) * 2 * cap));
  NUI_CUDA(counted_malloc(&ctx->d_pose, sizeof(float) * 14 * cap));
  NUI_CUDA(counted_malloc(&ctx->d_status, sizeof(int) * 2 * cap));
  NUI_CUDA(counted_malloc_host(&ctx->h_pose, sizeof(float) * 2 * 14 * cap));
  NUI_CUDA(counted_malloc_host(&ctx->h_status, sizeof(int) * 2 * 2 * cap));
  for (int h = 0; h < 2 && old_pose; ++h) {
    std::memcpy(ctx->h_pose + (size_t)h * 14 * cap, old_pose + (size_t)h * 14 * old_cap, sizeof(float) * 14 * old_cap);
    std::memcpy(ctx->h_status + (size_t)h * 2 * cap, old_status + (size_t)h * 2 * old_cap, sizeof(int) * 2 * old_cap);
  }
  cudaFreeHost(old_pose);
  cudaFreeHost(old_status);
  ctx->cap = cap;
  return NUI_OK;
}

nui_status finish_timing(nui_ctx* ctx) {
  if (!ctx->timing) return NUI_OK;
  NUI_CUDA(cudaEventSynchronize(ctx->ev[6]));
  for (int i = 0; i < 6; ++i) cudaEventElapsedTime(&ctx->stage_ms[i], ctx->ev[i], ctx->ev[i + 1]);
  cudaEventElapsedTime(&ctx->stage_ms[6], ctx->ev[0], ctx->ev[6]);
  if (cudaEventElapsedTime(&ctx->stage_ms[7], ctx->ev[7], ctx->ev[8]) != cudaSuccess) ctx->stage_ms[7] = 0.f;
  if (!ctx->side_timed || cudaEventElapsedTime(&ctx->stage_ms[8], ctx->ev[9], ctx->ev[10]) != cudaSuccess)
    ctx->stage_ms[8] = 0.f;
  cudaGetLastError();
  return NUI_OK;
}

// Launches one batched tick on the context stream (asynchronous).  raws[i] == nullptr
// leaves session i out of this tick (inactive: every kernel skips it), so that a batch
// keeps its shape -- and its captured graph -- while some sessions have no frame.
// A null session is an empty slot: an inactive descriptor without buffers.  `floor`
// (nullable) is merged into the launch shape, so that a caller can keep one shape -- and
// its graph -- while sessions come and go.
nui_status tick_launch(nui_ctx* ctx, nui_session* const* ss, int n, const uint16_t* const* raws,
                       const uint8_t* const* bgras, bool use_graph, const BatchPlan* floor, int* par_out) {
  nui_status st = ensure_cap(ctx, n);
  if (st != NUI_OK) return st;
  // this tick's half of the host staging: the tick before last used it, and its table copy
  // and result copies are complete once its event is
  const int par = ctx->par;
  NUI_CUDA(cudaEventSynchronize(ctx->ev_tick[par]));
  SessionDesc* const hd = ctx->h_descs + (size_t)par * ctx->cap;
  BatchPlan p;
  p.n = n;
  // the table lists the non-hash slots first (empty ones included), then the hash sessions,
  // each group in slot order; a descriptor's slot is its row of the outputs
  int nhash = 0;
  for (int i = 0; i < n; ++i) nhash += ss[i] && ss[i]->hash;
  for (int i = 0, jd = 0, jh = n - nhash; i < n; ++i) {
    nui_session* s = ss[i];
    SessionDesc& dd = hd[s && s->hash ? jh++ : jd++];
    if (!s) {
      std::memset(&dd, 0, sizeof(SessionDesc));
      dd.kind = kInactive;
      dd.fmt = -1;
      dd.slot = i;
      continue;
    }
    plan_add(p, s);
    int kind = !raws[i] ? kInactive : s->frames == 0 ? kFirstFrame : kTrackFrame;
    if (kind == kFirstFrame) p.anyFirst = 1;
    fill_desc(s, dd, kind, raws[i], bgras ? bgras[i] : nullptr);
    dd.slot = i;
  }
  // the dense kernels launch over the rows before the hash sessions and the hash kernels
  // over theirs.  A served batch keeps its launch shape while streams come and go, but the
  // split follows the count of hash streams (a graph per count; empty slots sit among the
  // dense rows); with one family absent both launch over the whole table.
  if (!floor || (nhash > 0 && nhash < n)) {
    p.hashTail = nhash;
    p.denseHead = n - nhash;
  }
  if (floor) plan_merge(p, *floor);
  p.tune = ctx->tune;
  NUI_CUDA(cudaMemcpyAsync(ctx->d_descs, hd, sizeof(SessionDesc) * n, cudaMemcpyHostToDevice, ctx->stream));
  if (use_graph && !ctx->timing) {
    auto it = ctx->graphs.find(p);
    if (it == ctx->graphs.end()) {
      if (ctx->graphs.size() >= kMaxGraphs) {  // bounded cache: start over
        for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second.exec);
        ctx->graphs.clear();
      }
      cudaGraph_t g;
      NUI_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      enqueue_tick(ctx, p, ctx->d_descs, ctx->d_pose, ctx->d_status, false);
      NUI_CUDA(cudaStreamEndCapture(ctx->stream, &g));
      size_t nn = 0;
      NUI_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
      std::vector<cudaGraphNode_t> nodes(nn);
      NUI_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
      int kernels = 0;
      for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType ty;
        if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++kernels;
      }
      cudaGraphExec_t ge;
      NUI_CUDA(cudaGraphInstantiate(&ge, g, 0));
      cudaGraphDestroy(g);
      it = ctx->graphs.emplace(p, nui_ctx::Graph{ge, kernels}).first;
    }
    ctx->last_kernels = it->second.kernels;
    NUI_CUDA(cudaGraphLaunch(it->second.exec, ctx->stream));
  } else {
    enqueue_tick(ctx, p, ctx->d_descs, ctx->d_pose, ctx->d_status, ctx->timing);
    NUI_CUDA(cudaGetLastError());
  }
  NUI_CUDA(cudaMemcpyAsync(ctx->h_pose + (size_t)par * 14 * ctx->cap, ctx->d_pose, sizeof(float) * 14 * n,
                           cudaMemcpyDeviceToHost, ctx->stream));
  NUI_CUDA(cudaMemcpyAsync(ctx->h_status + (size_t)par * 2 * ctx->cap, ctx->d_status, sizeof(int) * 2 * n,
                           cudaMemcpyDeviceToHost, ctx->stream));
  NUI_CUDA(cudaEventRecord(ctx->ev_tick[par], ctx->stream));
  ctx->par = par ^ 1;
  if (par_out) *par_out = par;
  // a session's frame count advances when its frame is launched (a lost frame takes it
  // back when its result is read), so that the next tick can be launched before then
  for (int i = 0; i < n; ++i)
    if (ss[i] && raws[i]) ss[i]->frames += 1;
  return NUI_OK;
}

// Waits for the tick launched with staging half par and takes its per-session results.
nui_status tick_finish(nui_ctx* ctx, nui_session* const* ss, int n, const uint16_t* const* raws, nui_status* per,
                       float* poses, int par) {
  NUI_CUDA(cudaEventSynchronize(ctx->ev_tick[par]));
  nui_status st = finish_timing(ctx);
  if (st != NUI_OK) return st;
  const float* h_pose = ctx->h_pose + (size_t)par * 14 * ctx->cap;
  const int* h_status = ctx->h_status + (size_t)par * 2 * ctx->cap;
  nui_status agg = NUI_OK;
  auto note = [](nui_status r) {
    if (r == NUI_ERR_HASH_FULL)
      fail(r, "voxel hash: pool or excess list exhausted (or a corrupted chain); blocks dropped");
    else if (r == NUI_ERR_TRACKING_LOST)
      fail(r, "ICP system is singular");
  };
  for (int i = 0; i < n; ++i) {
    nui_session* s = ss[i];
    if (!s || !raws[i]) {
      if (per) per[i] = NUI_OK;
      continue;
    }
    int status = h_status[2 * i];
    if (status == 4) {  // tracked and integrated, but the voxel hash dropped blocks
      if (per) per[i] = NUI_ERR_HASH_FULL;
      if (agg == NUI_OK) {
        agg = NUI_ERR_HASH_FULL;
        note(agg);
      }
      if (poses) std::memcpy(poses + 12 * i, h_pose + 14 * i, 12 * sizeof(float));
      continue;
    }
    nui_status r = status == 0 ? NUI_OK : NUI_ERR_TRACKING_LOST;
    if (per) per[i] = r;
    if (r != NUI_OK) {
      agg = NUI_ERR_TRACKING_LOST;
      note(agg);
      // the device state stays on the previous frame, which the frame count follows; the
      // flag is cleared in stream order (every tick also clears it when it starts), so
      // that the next frame (after nui_reset or not) starts from a clean tracker
      s->frames -= 1;
      NUI_CUDA(cudaMemsetAsync(&s->ts->status, 0, sizeof(int), ctx->stream));
    }
    if (poses) std::memcpy(poses + 12 * i, h_pose + 14 * i, 12 * sizeof(float));
  }
  return agg;
}

nui_status run_tick(nui_ctx* ctx, nui_session* const* ss, int n, const uint16_t* const* raws,
                    const uint8_t* const* bgras, bool use_graph, nui_status* per, float* poses) {
  int par = 0;
  nui_status st = tick_launch(ctx, ss, n, raws, bgras, use_graph, nullptr, &par);
  if (st != NUI_OK) return st;
  return tick_finish(ctx, ss, n, raws, per, poses, par);
}

nui_status upload_frame(nui_session* s, const uint16_t* depth, const uint8_t* bgra) {
  const size_t N = (size_t)s->cfg.width * s->cfg.height;
  NUI_CUDA(cudaMemcpyAsync(s->raw, depth, N * 2, cudaMemcpyHostToDevice, s->ctx->stream));
  s->color_frame = false;
  if (bgra && s->bgra) {
    NUI_CUDA(cudaMemcpyAsync(s->bgra, bgra, N * 4, cudaMemcpyHostToDevice, s->ctx->stream));
    s->color_frame = true;
  }
  return NUI_OK;
}

template <int F>
void launch_init(nui_session* s) {
  k_volume_init<F><<<dim3(1184, 1), 256, 0, s->ctx->stream>>>(s->d_desc1);
}

// sync = false leaves the reset queued on the context stream (the host copies are staged
// by the runtime before the calls return).
nui_status reset_session(nui_session* s, bool sync = true) {
  SessionDesc d;
  fill_desc(s, d, kInactive, nullptr, nullptr);
  NUI_CUDA(cudaMemcpyAsync(s->d_desc1, &d, sizeof(d), cudaMemcpyHostToDevice, s->ctx->stream));
  if (s->hash) {
    k_hash_reset<<<1184, 256, 0, s->ctx->stream>>>(s->d_desc1);
  } else {
    switch (s->cfg.tsdf_format) {
      case 0: launch_init<0>(s); break;
      case 1: launch_init<1>(s); break;
      case 2: launch_init<2>(s); break;
      case 3: launch_init<3>(s); break;
    }
  }
  if (s->cprev)
    NUI_CUDA(cudaMemsetAsync(s->cprev, 0, (size_t)s->cfg.width * s->cfg.height * 4, s->ctx->stream));
  TrackState t;
  std::memset(&t, 0, sizeof(t));
  const float I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  std::memcpy(t.xf.R, I, sizeof(I));
  std::memcpy(t.xf.R_inv, I, sizeof(I));
  std::memcpy(t.R, I, sizeof(I));
  std::memcpy(t.lastR, I, sizeof(I));
  NUI_CUDA(cudaMemcpyAsync(s->ts, &t, sizeof(t), cudaMemcpyHostToDevice, s->ctx->stream));
  if (sync) NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  NUI_CUDA(cudaGetLastError());
  s->frames = 0;
  return NUI_OK;
}

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" {

NUI_API const char* nui_last_error_string(void) { return g_err.c_str(); }

NUI_API void nui_session_cfg_default(nui_session_cfg* c) {
  std::memset(c, 0, sizeof(*c));
  c->width = 640;
  c->height = 480;
  c->fx = c->fy = 525.f;
  c->cx = 319.5f;
  c->cy = 239.5f;
  c->depth_min = 0.5f;
  c->depth_max = 4.5f;
  c->volume_kind = NUI_VOLUME_DENSE;
  c->tsdf_format = NUI_TSDF_I16;
  c->res[0] = c->res[1] = c->res[2] = 256;
  c->dim[0] = c->dim[1] = c->dim[2] = 3.f;
  c->trunc_dist = 0.03f;
  c->color_volume = 0;
  c->max_color_weight = 128;
  c->levels = 3;
  c->iterations[0] = c->iterations[1] = c->iterations[2] = 10;
  c->filter_radius = 3;
  c->sigma_space2_inv_half = 0.08f;
  c->sigma_depth2_inv_half = 50.0f;
  c->depth_threshold = 0.3f;
  c->dist_threshold = 0.1f;
  c->integration_threshold = 0.15f;
  c->voxel_size = 0.005f;
  c->trunc_scale = 0.02f;
  c->hash_buckets = 1 << 20;
  c->hash_excess = 0x30000;
  c->hash_pool_blocks = 1 << 20;
  c->hash_max_weight = 255;
  c->voxel_shift = 0;
  c->shift_point_cap = 1 << 20;
}

NUI_API nui_status nui_ctx_create(int device, nui_ctx** out) {
  if (!out) return fail(NUI_ERR_INVALID_ARG, "out is null");
  int ndev = 0;
  NUI_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(NUI_ERR_INVALID_ARG, "no such device");
  NUI_CUDA(cudaSetDevice(device));
  noalloc_forget(device);
  nui_ctx* c = new nui_ctx();
  c->device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return fail(NUI_ERR_DEVICE, cudaGetErrorString(e));
  }
  c->stream = c->own;
  for (int i = 0; i < kEvents; ++i) cudaEventCreate(&c->ev[i]);
  if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_tick[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_tick[1], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return fail(NUI_ERR_DEVICE, "context streams");
  }
  if (counted_malloc(&c->d_kdesc, sizeof(SessionDesc)) != cudaSuccess ||
      counted_malloc(&c->d_kts, sizeof(TrackState)) != cudaSuccess ||
      counted_malloc(&c->d_count, sizeof(unsigned long long)) != cudaSuccess) {
    delete c;
    return fail(NUI_ERR_OOM, "context scratch");
  }
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  if (cudaMemPoolCreate(&c->pool, &props) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return fail(NUI_ERR_DEVICE, "context memory pool");
  }
  uint64_t keep = ~0ull;  // freed session memory stays in the pool for the next session
  cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  *out = c;
  return NUI_OK;
}

NUI_API nui_status nui_ctx_destroy(nui_ctx* c) {
  if (!c) return NUI_OK;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second.exec);
  for (int i = 0; i < kEvents; ++i) cudaEventDestroy(c->ev[i]);
  cudaFree(c->d_descs);
  cudaFreeHost(c->h_descs);
  cudaFree(c->d_pose);
  cudaFree(c->d_status);
  cudaFreeHost(c->h_pose);
  cudaFreeHost(c->h_status);
  cudaFree(c->d_kdesc);
  cudaFree(c->d_kts);
  cudaFree(c->d_count);
  cudaStreamDestroy(c->own);
  cudaStreamDestroy(c->side);
  cudaEventDestroy(c->fork_ev);
  cudaEventDestroy(c->join_ev);
  cudaEventDestroy(c->ev_tick[0]);
  cudaEventDestroy(c->ev_tick[1]);
  if (c->pool) {
    cudaDeviceSynchronize();
    cudaMemPoolDestroy(c->pool);
  }
  delete c;
  return NUI_OK;
}

NUI_API nui_status nui_ctx_set_stream(nui_ctx* c, void* stream) {
  if (!c) return fail(NUI_ERR_INVALID_ARG, "null context");
  NUI_CUDA(cudaStreamSynchronize(c->stream));
  c->stream = stream ? (cudaStream_t)stream : c->own;
  for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second.exec);
  c->graphs.clear();
  return NUI_OK;
}

NUI_API nui_status nui_ctx_trim(nui_ctx* c) {
  if (!c) return fail(NUI_ERR_INVALID_ARG, "null context");
  NUI_CUDA(cudaStreamSynchronize(c->stream));
  NUI_CUDA(cudaMemPoolTrimTo(c->pool, 0));
  return NUI_OK;
}

NUI_API nui_status nui_ctx_synchronize(nui_ctx* c) {
  if (!c) return fail(NUI_ERR_INVALID_ARG, "null context");
  NUI_CUDA(cudaStreamSynchronize(c->stream));
  return NUI_OK;
}

NUI_API nui_status nui_ctx_enable_timing(nui_ctx* c, int enable) {
  if (!c) return fail(NUI_ERR_INVALID_ARG, "null context");
  c->timing = enable != 0;
  return NUI_OK;
}

NUI_API nui_status nui_ctx_last_tick_kernels(nui_ctx* c, int* n) {
  if (!c || !n) return fail(NUI_ERR_INVALID_ARG, "null argument");
  *n = c->last_kernels;
  return NUI_OK;
}

bool tuning_valid(const nui_tuning& t) {
  auto tw_ok = [](int w) { return w == 4 || w == 8 || w == 16 || w == 32; };
  return t.integrate_threads_log2 >= 14 && t.integrate_threads_log2 <= 22 &&
         (t.icp_pixels_per_thread == 2 || t.icp_pixels_per_thread == 4 || t.icp_pixels_per_thread == 8 ||
          t.icp_pixels_per_thread == 16) &&
         (t.icp_cluster_blocks >= 2 && t.icp_cluster_blocks <= 16) &&
         tw_ok(t.raycast_tile_width) && tw_ok(t.hash_raycast_tile_width);
}

NUI_API nui_status nui_ctx_get_tuning(nui_ctx* c, nui_tuning* out) {
  if (!c || !out) return fail(NUI_ERR_INVALID_ARG, "null argument");
  *out = c->tune;
  return NUI_OK;
}

NUI_API nui_status nui_ctx_set_tuning(nui_ctx* c, const nui_tuning* t) {
  if (!c || !t) return fail(NUI_ERR_INVALID_ARG, "null argument");
  if (!tuning_valid(*t)) return fail(NUI_ERR_INVALID_ARG, "tuning out of range");
  c->tune = *t;  // the graph cache is keyed by the launch shape, tuning included
  return NUI_OK;
}

NUI_API nui_status nui_ctx_autotune(nui_ctx* c, const nui_session_cfg* cfgs, int n, const uint16_t* const* depth,
                                    const uint8_t* const* bgra, int frames, int repeats, nui_tuning* out,
                                    float* out_tick_ms) {
  if (!c || !cfgs || n <= 0 || !depth || frames < 2 || repeats < 1 || repeats > 101)
    return fail(NUI_ERR_INVALID_ARG, "autotune: bad argument (frames >= 2, 1 <= repeats <= 101)");
  for (int i = 0; i < n * frames; ++i)
    if (!depth[i]) return fail(NUI_ERR_INVALID_ARG, "autotune: null depth frame");
  std::vector<nui_session*> ss(n, nullptr);
  auto drop = [&]() {
    for (nui_session* s : ss)
      if (s) nui_session_destroy(s);
  };
  for (int i = 0; i < n; ++i) {
    nui_status st = nui_session_create(c, &cfgs[i], &ss[i]);
    if (st != NUI_OK) {
      const std::string why = g_err;
      drop();
      return fail(st, "autotune: scratch session: " + why);
    }
  }
  bool dense = false, hash = false;
  for (int i = 0; i < n; ++i) (ss[i]->hash ? hash : dense) = true;
  const bool timing = c->timing;
  c->timing = true;
  std::vector<const uint16_t*> raws(n);
  std::vector<const uint8_t*> cols(n);
  std::vector<nui_status> per(n);
  std::vector<float> poses(n * 12);
  // frame f of every session; past the sequence the last two frames alternate
  auto tick = [&](int f) -> nui_status {
    if (f >= frames) f = frames - 2 + ((f - frames) & 1);
    for (int i = 0; i < n; ++i) {
      raws[i] = depth[(size_t)i * frames + f];
      cols[i] = bgra ? bgra[(size_t)i * frames + f] : nullptr;
    }
    // a lost frame still ran the whole tick: it times like any other
    const nui_status r =
        nui_batch_tick(c, ss.data(), n, raws.data(), bgra ? cols.data() : nullptr, per.data(), poses.data());
    return (r == NUI_ERR_TRACKING_LOST || r == NUI_ERR_HASH_FULL) ? NUI_OK : r;
  };
  nui_status st = NUI_OK;
  int f = 0;
  for (; f < frames && st == NUI_OK; ++f) st = tick(f);
  // stage 6 (the whole tick) is timed as it runs in production: the captured graph between
  // two events on the context stream; the other stages by the stage events of an
  // un-graphed tick
  cudaEvent_t ta = nullptr, tb = nullptr;
  cudaEventCreate(&ta);
  cudaEventCreate(&tb);
  auto measure = [&](int stage, float* tick_ms) -> float {
    std::vector<float> t, w;
    for (int r = 0; r < repeats && st == NUI_OK; ++r) {
      if (stage == 6) {
        c->timing = false;
        cudaEventRecord(ta, c->stream);
        st = tick(f++);
        cudaEventRecord(tb, c->stream);
        float ms = 0.f;
        if (cudaEventSynchronize(tb) != cudaSuccess || cudaEventElapsedTime(&ms, ta, tb) != cudaSuccess) {
          cudaGetLastError();
          ms = 0.f;
        }
        c->timing = true;
        t.push_back(ms);
        w.push_back(ms);
        continue;
      }
      st = tick(f++);
      t.push_back(c->stage_ms[stage]);
      w.push_back(c->stage_ms[6]);
    }
    if (st != NUI_OK) return 0.f;
    std::sort(t.begin(), t.end());
    std::sort(w.begin(), w.end());
    if (tick_ms) *tick_ms = w[w.size() / 2];
    return t[t.size() / 2];
  };
  nui_tuning best = c->tune;
  // one parameter at a time: its stage's median over `repeats` ticks
  // The current value is timed first and stays unless a candidate beats it by 2 %: tick
  // times wander by a few per cent between otherwise equal runs, and a noise-driven switch
  // away from the default shape cost more than it ever gained.
  auto tune_one = [&](int nui_tuning::*field, std::initializer_list<int> cands, int stage) {
    const int cur = best.*field;
    c->tune = best;
    float best_ms = measure(stage, nullptr), cur_ms = best_ms;
    int pick = cur;
    for (int v : cands) {
      if (st != NUI_OK) return;
      if (v == cur) continue;
      c->tune = best;
      c->tune.*field = v;
      const float ms = measure(stage, nullptr);
      if (st == NUI_OK && ms < best_ms && ms < 0.98f * cur_ms) best_ms = ms, pick = v;
    }
    best.*field = pick;
  };
  if (dense) tune_one(&nui_tuning::integrate_threads_log2, {16, 17, 18, 19, 20}, 3);
  // the ICP shapes and ray tiles by the whole tick: with dense and hash sessions the hash
  // sessions' tracking and raycast run on the second stream, beside stages 2-5
  tune_one(&nui_tuning::icp_cluster_blocks, {8, 12, 16}, 6);
  tune_one(&nui_tuning::icp_pixels_per_thread, {2, 4, 8, 16}, 6);
  if (dense) tune_one(&nui_tuning::raycast_tile_width, {4, 8, 16, 32}, 6);
  if (hash) tune_one(&nui_tuning::hash_raycast_tile_width, {4, 8, 16, 32}, 6);
  float tick_ms = 0.f;
  if (st == NUI_OK) {
    c->tune = best;
    measure(6, &tick_ms);
  }
  const std::string why = g_err;
  c->timing = timing;
  cudaEventDestroy(ta);
  cudaEventDestroy(tb);
  drop();
  if (st != NUI_OK) {
    c->tune = best;
    return fail(st, "autotune: " + why);
  }
  if (out) *out = best;
  if (out_tick_ms) *out_tick_ms = tick_ms;
  return NUI_OK;
}

NUI_API nui_status nui_ctx_stage_ms(nui_ctx* c, int stage, float* ms) {
  if (!c || !ms || stage < 0 || stage >= kStages) return fail(NUI_ERR_INVALID_ARG, "bad stage");
  *ms = c->stage_ms[stage];
  return NUI_OK;
}

NUI_API size_t nui_session_device_bytes(const nui_session_cfg* c) {
  std::string why;
  if (!cfg_valid(c, why)) return 0;
  const size_t N = (size_t)c->width * c->height;
  size_t b = N * 2 + N * 4 /*bgra*/ + N * 4 /*scaled*/ + N * 16 * 2 /*ref maps*/ + N * 4 /*cmap*/;
  for (int l = 0; l < c->levels; ++l) b += (N >> (2 * l)) * 4;
  b += sizeof(TrackState) + sizeof(SessionDesc);
  b += (N / (kTile * kTile) + 64) * 4;
  if (c->volume_kind == NUI_VOLUME_HASH) {
    const size_t ne = (size_t)c->hash_buckets + c->hash_excess, nv = (size_t)c->hash_pool_blocks * 512;
    b += ne * (16 + 1 + 1 + 8 + 8 + 4) + ((ne + 1023) / 1024) * 16 + (size_t)c->hash_pool_blocks * 4 +
         (size_t)c->hash_excess * 4 + N * 8;
    b += nv * ((c->tsdf_format == NUI_TSDF_I16 ? 2 : 2) + 1 + (c->color_volume ? 4 : 0));
    if (c->hash_swapping) b += ne * 5 + 2 * 4096 * 4;  // the store itself is host memory
    if (c->hash_forward_render) b += N * (4 + 4 + (c->color_volume ? 4 : 0)) + ((N + 1023) / 1024 + 1) * 4;
    return b;
  }
  const size_t nv = (size_t)c->res[0] * c->res[1] * c->res[2];
  b += nv * voxel_bytes(c->tsdf_format);
  if (c->tsdf_format >= NUI_TSDF_F16_U8)  // tolerance-mode tile list
    b += (size_t)((c->res[0] + 31) / 32) * ((c->res[1] + 7) / 8) * ((c->res[2] + 7) / 8) * 4;
  if (c->color_volume) b += nv * 4;
  b += (size_t)((c->res[0] + 7) / 8) * ((c->res[1] + 7) / 8) * ((c->res[2] + 7) / 8);
  b += (size_t)((c->res[0] + 31) / 32) * ((c->res[1] + 31) / 32) * ((c->res[2] + 31) / 32);
  b += (size_t)((c->res[0] + 127) / 128) * ((c->res[1] + 127) / 128) * ((c->res[2] + 127) / 128);
  b += 2 * ((size_t)c->res[2] + 1) * sizeof(float);
  if (c->voxel_shift > 0) b += (size_t)c->shift_point_cap * 28;
  return b;
}

}  // extern "C"

namespace {
// Frees a session's memory in stream order (sync: wait for its stream first).
void session_free(nui_session* s, bool sync) {
  cudaStream_t st = s->ctx->stream;
  if (sync) cudaStreamSynchronize(st);
  for (void* p : s->allocs) cudaFreeAsync(p, st);
  for (void* p : s->host_allocs) cudaFreeHost(p);
  delete s;
}

// sync = false: the allocation and the reset are queued on the context stream and the call
// returns at once (the serving loop admits streams this way while a tick runs).
nui_status session_create(nui_ctx* ctx, const nui_session_cfg* cfg, nui_session** out, bool sync) {
  std::string why;
  if (!ctx || !out) return fail(NUI_ERR_INVALID_ARG, "null argument");
  if (!cfg_valid(cfg, why)) return fail(NUI_ERR_INVALID_ARG, why);
  NUI_CUDA(cudaSetDevice(ctx->device));
  nui_session* s = new nui_session();
  s->ctx = ctx;
  s->cfg = *cfg;
  const nui_session_cfg& c = s->cfg;
  s->cam = DevCam{c.fx, c.fy, 1 / c.fx, 1 / c.fy, c.cx, c.cy, c.width, c.height, c.depth_min, c.depth_max};
  for (int i = 0; i < 3; ++i) s->cell[i] = c.dim[i] / (float)c.res[i];
  s->trunc = std::max(c.trunc_dist, 2.1f * std::max(s->cell[0], std::max(s->cell[1], s->cell[2])));
  for (int i = 0; i < 2 * kMaxRadius + 1; ++i) s->gauss[i] = 0.f;
  for (int i = 0; i < 2 * c.filter_radius + 1; ++i) {
    int x = i - c.filter_radius;
    s->gauss[i] = std::exp((float)(-(x * x)) * c.sigma_space2_inv_half);
  }
  icp_thresholds(c, s->icp_min_count);
  const size_t N = (size_t)c.width * c.height;
  const size_t nv = (size_t)c.res[0] * c.res[1] * c.res[2];
  auto alloc = [&](void** p, size_t bytes) -> bool {
    if (counted_pool_alloc(p, bytes, ctx->pool, ctx->stream) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    s->allocs.push_back(*p);
    return true;
  };
  // pinned host memory mapped into the device: *h the host pointer, *d the device one
  auto host_alloc = [&](void** h, void** d, size_t bytes) -> bool {
    if (counted_host_alloc(h, bytes, cudaHostAllocMapped) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    s->host_allocs.push_back(*h);
    if (cudaHostGetDevicePointer(d, *h, 0) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return true;
  };
  s->hash = c.volume_kind == NUI_VOLUME_HASH;
  bool ok = alloc((void**)&s->raw, N * 2) && alloc((void**)&s->dscaled, N * 4) && alloc((void**)&s->vref, N * 16) &&
            alloc((void**)&s->nref, N * 16) && alloc((void**)&s->ts, sizeof(TrackState)) &&
            alloc((void**)&s->d_desc1, sizeof(SessionDesc));
  for (int l = 0; ok && l < c.levels; ++l)
    ok = alloc((void**)&s->dlev[l], (N >> (2 * l)) * 4);
  const size_t ntiles = (size_t)((c.width + kTile - 1) / kTile) * ((c.height + kTile - 1) / kTile);
  if (ok) ok = alloc((void**)&s->tile_max, ntiles * sizeof(float));
  if (s->hash) {
    const size_t ne = (size_t)c.hash_buckets + c.hash_excess, hv = (size_t)c.hash_pool_blocks * 512;
    ok = ok && alloc((void**)&s->entries, ne * sizeof(HEntry)) && alloc((void**)&s->hsdf, hv * 2) &&
         alloc((void**)&s->hw, hv) && alloc((void**)&s->alloc_list, (size_t)c.hash_pool_blocks * 4) &&
         alloc((void**)&s->excess_list, (size_t)c.hash_excess * 4) && alloc((void**)&s->hcount, 64) &&
         alloc((void**)&s->alloc_type, ne) && alloc((void**)&s->vis, ne) && alloc((void**)&s->coords, ne * 8) &&
         alloc((void**)&s->keys, ne * 8) && alloc((void**)&s->vis_ids, ne * 4) &&
         alloc((void**)&s->blk, ((ne + 1023) / 1024) * 16) && alloc((void**)&s->range, N * 8);
    if (ok && c.color_volume) ok = alloc((void**)&s->hrgb, hv * 4) && alloc((void**)&s->bgra, N * 4) && alloc((void**)&s->cmap, N * 4);
    if (ok && c.hash_forward_render)
      ok = alloc((void**)&s->fwd_owner, N * 4) && alloc((void**)&s->fwd_ids, N * 4) &&
           alloc((void**)&s->fwd_blk, ((N + 1023) / 1024 + 1) * 4) &&
           (!c.color_volume || alloc((void**)&s->fwd_col, N * 4));
    if (ok && c.hash_swapping) {
      // the global cache: swap state and store slot per entry, transfer lists, and the
      // store in pinned host memory mapped into the device (one slot per entry by default)
      s->st_cap = c.hash_store_blocks > 0 ? c.hash_store_blocks : (int)ne;
      const size_t sv = (size_t)s->st_cap * 512;
      ok = alloc((void**)&s->swap, ne) && alloc((void**)&s->store_slot, ne * 4) &&
           alloc((void**)&s->swap_in_ids, 4096 * 4) && alloc((void**)&s->swap_out_ids, 4096 * 4) &&
           host_alloc(&s->h_st_sdf, &s->st_sdf, sv * 2) && host_alloc((void**)&s->h_st_w, (void**)&s->st_w, sv) &&
           (!c.color_volume || host_alloc((void**)&s->h_st_rgb, (void**)&s->st_rgb, sv * 4));
    }
  } else {
    ok = ok && alloc((void**)&s->vol, nv * (c.tsdf_format == 2 ? 2 : voxel_bytes(c.tsdf_format)));
    if (ok && c.tsdf_format == NUI_TSDF_F16_U8) ok = alloc((void**)&s->wvol, nv);
    if (ok && c.tsdf_format >= NUI_TSDF_F16_U8)
      ok = alloc((void**)&s->fast_tiles, (size_t)((c.res[0] + 31) / 32) * ((c.res[1] + 7) / 8) * ((c.res[2] + 7) / 8) * 4);
    const size_t nbricks = (size_t)((c.res[0] + 7) / 8) * ((c.res[1] + 7) / 8) * ((c.res[2] + 7) / 8);
    const size_t nsuper = (size_t)((c.res[0] + 31) / 32) * ((c.res[1] + 31) / 32) * ((c.res[2] + 31) / 32);
    const size_t nhyper = (size_t)((c.res[0] + 127) / 128) * ((c.res[1] + 127) / 128) * ((c.res[2] + 127) / 128);
    if (ok) ok = alloc((void**)&s->occ, nbricks) && alloc((void**)&s->occ2, nsuper) && alloc((void**)&s->occ3, nhyper) &&
                 alloc((void**)&s->ztab, 2 * ((size_t)c.res[2] + 1) * sizeof(float));
    if (ok && c.color_volume) ok = alloc((void**)&s->cvol, nv * 4) && alloc((void**)&s->bgra, N * 4) && alloc((void**)&s->cmap, N * 4);
  }
  if (ok && c.photometric_weight > 0.f)
    ok = alloc((void**)&s->cprev, N * 4) && alloc((void**)&s->cgx[0], N * 4) && alloc((void**)&s->cgy[0], N * 4);
  if (ok && !s->hash && c.voxel_shift > 0 && c.shift_point_cap > 0)
    ok = alloc((void**)&s->pts_xyz, (size_t)c.shift_point_cap * 12) &&
         alloc((void**)&s->pts_rgba, (size_t)c.shift_point_cap * 16);
  if (!ok) {
    session_free(s, true);
    return fail(NUI_ERR_OOM, "device allocation failed");
  }
  cudaMemsetAsync(s->ts, 0, sizeof(TrackState), ctx->stream);
  nui_status st = reset_session(s, sync);
  if (st != NUI_OK) {
    session_free(s, true);
    return st;
  }
  *out = s;
  return NUI_OK;
}
}  // namespace

extern "C" {
NUI_API nui_status nui_session_create(nui_ctx* ctx, const nui_session_cfg* cfg, nui_session** out) {
  return session_create(ctx, cfg, out, true);
}

NUI_API nui_status nui_session_destroy(nui_session* s) {
  if (!s) return NUI_OK;
  session_free(s, true);
  return NUI_OK;
}

NUI_API nui_status nui_reset(nui_session* s) {
  if (!s) return fail(NUI_ERR_INVALID_ARG, "null session");
  return reset_session(s);
}

NUI_API nui_status nui_process_frame(nui_session* s, const uint16_t* depth, const uint8_t* bgra, float* pose) {
  if (!s || !depth) return fail(NUI_ERR_INVALID_ARG, "null argument");
  nui_status st = upload_frame(s, depth, bgra);
  if (st != NUI_OK) return st;
  const uint16_t* r = s->raw;
  const uint8_t* b = s->color_frame ? s->bgra : nullptr;
  nui_session* arr[1] = {s};
  nui_status per;
  return run_tick(s->ctx, arr, 1, &r, &b, false, &per, pose);
}

NUI_API nui_status nui_process_frame_device(nui_session* s, const uint16_t* d_depth, const uint8_t* d_bgra, float* pose) {
  if (!s || !d_depth) return fail(NUI_ERR_INVALID_ARG, "null argument");
  nui_session* arr[1] = {s};
  const uint8_t* b = (d_bgra && s->cmap) ? d_bgra : nullptr;
  nui_status per;
  return run_tick(s->ctx, arr, 1, &d_depth, &b, false, &per, pose);
}

NUI_API nui_status nui_batch_tick(nui_ctx* ctx, nui_session* const* ss, int n, const uint16_t* const* depths,
                                  const uint8_t* const* bgras, nui_status* per, float* poses) {
  if (!ctx || !ss || n <= 0 || !depths) return fail(NUI_ERR_INVALID_ARG, "bad batch");
  std::vector<const uint16_t*> r(n);
  std::vector<const uint8_t*> b(n);
  for (int i = 0; i < n; ++i) {
    if (!ss[i] || ss[i]->ctx != ctx || !depths[i]) return fail(NUI_ERR_INVALID_ARG, "bad session or frame");
    nui_status st = upload_frame(ss[i], depths[i], bgras ? bgras[i] : nullptr);
    if (st != NUI_OK) return st;
    r[i] = ss[i]->raw;
    b[i] = ss[i]->color_frame ? ss[i]->bgra : nullptr;
  }
  return run_tick(ctx, ss, n, r.data(), b.data(), true, per, poses);
}

NUI_API nui_status nui_batch_tick_device(nui_ctx* ctx, nui_session* const* ss, int n, const uint16_t* const* d_depths,
                                         const uint8_t* const* d_bgras, nui_status* per, float* poses) {
  if (!ctx || !ss || n <= 0 || !d_depths) return fail(NUI_ERR_INVALID_ARG, "bad batch");
  std::vector<const uint8_t*> b(n, nullptr);
  for (int i = 0; i < n; ++i) {
    if (!ss[i] || ss[i]->ctx != ctx || !d_depths[i]) return fail(NUI_ERR_INVALID_ARG, "bad session or frame");
    if (d_bgras && d_bgras[i] && ss[i]->cmap) b[i] = d_bgras[i];
  }
  return run_tick(ctx, ss, n, d_depths, b.data(), true, per, poses);
}

NUI_API nui_status nui_set_pose(nui_session* s, const float* pose12) {
  if (!s || !pose12) return fail(NUI_ERR_INVALID_ARG, "null argument");
  TrackState t;
  NUI_CUDA(cudaMemcpy(&t, s->ts, sizeof(t), cudaMemcpyDeviceToHost));
  double a[9];
  for (int i = 0; i < 9; ++i) a[i] = pose12[i];
  const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
  const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  const double inv[9] = {c00, a[2] * a[7] - a[1] * a[8], a[1] * a[5] - a[2] * a[4],
                         c01, a[0] * a[8] - a[2] * a[6], a[2] * a[3] - a[0] * a[5],
                         c02, a[1] * a[6] - a[0] * a[7], a[0] * a[4] - a[1] * a[3]};
  for (int i = 0; i < 9; ++i) {
    t.xf.R[i] = t.R[i] = pose12[i];
    t.xf.R_inv[i] = (float)(inv[i] / det);
  }
  for (int i = 0; i < 3; ++i) t.xf.t[i] = t.t[i] = pose12[9 + i];
  NUI_CUDA(cudaMemcpy(s->ts, &t, sizeof(t), cudaMemcpyHostToDevice));
  return NUI_OK;
}

NUI_API nui_status nui_get_pose(nui_session* s, float* pose12) {
  if (!s || !pose12) return fail(NUI_ERR_INVALID_ARG, "null argument");
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  TrackState t;
  NUI_CUDA(cudaMemcpy(&t, s->ts, sizeof(t), cudaMemcpyDeviceToHost));
  std::memcpy(pose12, t.xf.R, 9 * sizeof(float));
  std::memcpy(pose12 + 9, t.xf.t, 3 * sizeof(float));
  return NUI_OK;
}

}  // extern "C"

namespace {
// Device state a session carries from frame to frame: what a snapshot holds.  Per-frame
// scratch (depth pyramid, integration tables, hash allocation scratch, partial sums) is
// rebuilt by the next frame and left out.
std::vector<std::pair<void*, size_t>> state_segments(const nui_session* s) {
  const nui_session_cfg& c = s->cfg;
  const size_t N = (size_t)c.width * c.height;
  std::vector<std::pair<void*, size_t>> v;
  auto add = [&](void* p, size_t b) {
    if (p && b) v.emplace_back(p, b);
  };
  add(s->ts, sizeof(TrackState));
  add(s->vref, N * 16);
  add(s->nref, N * 16);
  add(s->cmap, N * 4);
  add(s->cprev, N * 4);
  if (s->hash) {
    const size_t ne = (size_t)c.hash_buckets + c.hash_excess, hv = (size_t)c.hash_pool_blocks * 512;
    add(s->entries, ne * sizeof(HEntry));
    add(s->hsdf, hv * 2);
    add(s->hw, hv);
    add(s->hrgb, hv * 4);
    add(s->alloc_list, (size_t)c.hash_pool_blocks * 4);
    add(s->excess_list, (size_t)c.hash_excess * 4);
    add(s->hcount, 64);
    add(s->vis, ne);
    add(s->vis_ids, ne * 4);
    add(s->swap, ne);
    add(s->store_slot, ne * 4);
    add(s->st_sdf, (size_t)s->st_cap * 512 * 2);
    add(s->st_w, (size_t)s->st_cap * 512);
    add(s->st_rgb, (size_t)s->st_cap * 512 * 4);
  } else {
    const size_t nv = (size_t)c.res[0] * c.res[1] * c.res[2];
    add(s->vol, nv * (c.tsdf_format == NUI_TSDF_F16_U8 ? 2 : voxel_bytes(c.tsdf_format)));
    add(s->wvol, nv);
    add(s->cvol, nv * 4);
    add(s->occ, (size_t)((c.res[0] + 7) / 8) * ((c.res[1] + 7) / 8) * ((c.res[2] + 7) / 8));
    add(s->occ2, (size_t)((c.res[0] + 31) / 32) * ((c.res[1] + 31) / 32) * ((c.res[2] + 31) / 32));
    add(s->occ3, (size_t)((c.res[0] + 127) / 128) * ((c.res[1] + 127) / 128) * ((c.res[2] + 127) / 128));
    add(s->pts_xyz, (size_t)c.shift_point_cap * 12);
    add(s->pts_rgba, (size_t)c.shift_point_cap * 16);
  }
  return v;
}

struct SnapshotHeader {
  char magic[8];  // "NUISNAP1"
  uint64_t bytes;  // whole snapshot
  nui_session_cfg cfg;
  int64_t frames;
};
}  // namespace

extern "C" {

NUI_API size_t nui_session_snapshot_bytes(nui_session* s) {
  if (!s) return 0;
  size_t b = sizeof(SnapshotHeader);
  for (auto& seg : state_segments(s)) b += seg.second;
  return b;
}

NUI_API nui_status nui_session_snapshot(nui_session* s, void* host, size_t bytes) {
  if (!s || !host) return fail(NUI_ERR_INVALID_ARG, "null argument");
  const size_t need = nui_session_snapshot_bytes(s);
  if (bytes < need) return fail(NUI_ERR_INVALID_ARG, "snapshot buffer too small");
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  SnapshotHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, "NUISNAP1", 8);
  h.bytes = need;
  h.cfg = s->cfg;
  h.frames = s->frames;
  std::memcpy(host, &h, sizeof(h));
  char* p = (char*)host + sizeof(h);
  for (auto& seg : state_segments(s)) {
    NUI_CUDA(cudaMemcpy(p, seg.first, seg.second, cudaMemcpyDefault));
    p += seg.second;
  }
  return NUI_OK;
}

NUI_API nui_status nui_session_restore(nui_session* s, const void* host, size_t bytes) {
  if (!s || !host) return fail(NUI_ERR_INVALID_ARG, "null argument");
  SnapshotHeader h;
  if (bytes < sizeof(h)) return fail(NUI_ERR_INVALID_ARG, "not a session snapshot");
  std::memcpy(&h, host, sizeof(h));
  if (std::memcmp(h.magic, "NUISNAP1", 8) != 0) return fail(NUI_ERR_INVALID_ARG, "not a session snapshot");
  if (h.bytes != nui_session_snapshot_bytes(s) || bytes < h.bytes)
    return fail(NUI_ERR_INVALID_ARG, "snapshot size does not match the session");
  if (std::memcmp(&h.cfg, &s->cfg, sizeof(nui_session_cfg)) != 0)
    return fail(NUI_ERR_INVALID_ARG, "snapshot of another configuration");
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  const char* p = (const char*)host + sizeof(h);
  for (auto& seg : state_segments(s)) {
    NUI_CUDA(cudaMemcpy(seg.first, p, seg.second, cudaMemcpyDefault));
    p += seg.second;
  }
  s->frames = h.frames;
  return NUI_OK;
}

NUI_API nui_status nui_hash_swap_stats(nui_session* s, int* swapped_in, int* swapped_out, int* store_used,
                                       int* store_refused) {
  if (!s || !s->hash || !s->swap) return fail(NUI_ERR_INVALID_ARG, "not a swapping hash session");
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  int c[9];
  NUI_CUDA(cudaMemcpy(c, s->hcount, sizeof(c), cudaMemcpyDeviceToHost));
  if (swapped_in) *swapped_in = c[4];
  if (swapped_out) *swapped_out = c[5];
  if (store_used) *store_used = std::min(c[7], s->st_cap);
  if (store_refused) *store_refused = c[8];
  return NUI_OK;
}

NUI_API nui_status nui_hash_stored_block(nui_session* s, int entry, void* sdf, uint8_t* weight, uint8_t* rgb4,
                                         int* found) {
  if (!s || !found || !s->hash || !s->swap) return fail(NUI_ERR_INVALID_ARG, "not a swapping hash session");
  const long ne = (long)s->cfg.hash_buckets + s->cfg.hash_excess;
  if (entry < 0 || entry >= ne) return fail(NUI_ERR_INVALID_ARG, "entry out of range");
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  int slot = -1;
  NUI_CUDA(cudaMemcpy(&slot, s->store_slot + entry, sizeof(int), cudaMemcpyDeviceToHost));
  *found = slot >= 0;
  if (slot < 0) return NUI_OK;
  const size_t o = (size_t)slot * 512;
  if (sdf) std::memcpy(sdf, (const char*)s->h_st_sdf + o * 2, 512 * 2);
  if (weight) std::memcpy(weight, s->h_st_w + o, 512);
  if (rgb4) {
    if (s->h_st_rgb)
      std::memcpy(rgb4, s->h_st_rgb + o, 512 * 4);
    else
      std::memset(rgb4, 0, 512 * 4);
  }
  return NUI_OK;
}

NUI_API nui_status nui_shift_state(nui_session* s, int* voxel_offset, float* offset_m, uint64_t* points_found) {
  if (!s) return fail(NUI_ERR_INVALID_ARG, "null session");
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  TrackState t;
  NUI_CUDA(cudaMemcpy(&t, s->ts, sizeof(t), cudaMemcpyDeviceToHost));
  for (int a = 0; a < 3; ++a) {
    if (voxel_offset) voxel_offset[a] = t.voff[a];
    if (offset_m) offset_m[a] = (float)t.voff[a] * s->cell[a];
  }
  if (points_found) *points_found = t.points;
  return NUI_OK;
}

NUI_API nui_status nui_shift_points(nui_session* s, float* xyz, float* rgba, uint64_t cap, uint64_t* n) {
  if (!s || !n || (cap && (!xyz || !rgba))) return fail(NUI_ERR_INVALID_ARG, "null argument");
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  unsigned long long found = 0;
  NUI_CUDA(cudaMemcpy(&found, &s->ts->points, sizeof(found), cudaMemcpyDeviceToHost));
  const uint64_t kept = s->pts_xyz ? std::min<uint64_t>(found, (uint64_t)s->cfg.shift_point_cap) : 0;
  const uint64_t k = std::min(kept, cap);
  if (k) {
    NUI_CUDA(cudaMemcpy(xyz, s->pts_xyz, k * 12, cudaMemcpyDeviceToHost));
    NUI_CUDA(cudaMemcpy(rgba, s->pts_rgba, k * 16, cudaMemcpyDeviceToHost));
  }
  *n = kept;
  return NUI_OK;
}

NUI_API nui_status nui_shift_points_clear(nui_session* s) {
  if (!s) return fail(NUI_ERR_INVALID_ARG, "null session");
  NUI_CUDA(cudaMemsetAsync(&s->ts->points, 0, sizeof(unsigned long long), s->ctx->stream));
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  return NUI_OK;
}

NUI_API nui_status nui_point_cloud_device(nui_session* s, float* d_xyz, float* d_rgba, uint64_t cap,
                                          uint64_t* found) {
  if (!s || !found || (cap && (!d_xyz || !d_rgba))) return fail(NUI_ERR_INVALID_ARG, "null argument");
  if (((uintptr_t)d_rgba & 15) || ((uintptr_t)d_xyz & 3)) return fail(NUI_ERR_INVALID_ARG, "misaligned buffers");
  nui_ctx* ctx = s->ctx;
  nui_status st = ensure_cap(ctx, 1);
  if (st != NUI_OK) return st;
  SessionDesc d;
  fill_desc(s, d, kInactive, nullptr, nullptr);
  NUI_CUDA(cudaMemcpyAsync(s->d_desc1, &d, sizeof(d), cudaMemcpyHostToDevice, ctx->stream));
  unsigned long long* counter = ctx->d_count;
  NUI_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), ctx->stream));
  const long long c = (long long)std::min<uint64_t>(cap, (uint64_t)1 << 62);
  if (s->hash) {
    if (s->cfg.tsdf_format == NUI_TSDF_I16)
      k_hash_fetch<0><<<1184, 512, 0, ctx->stream>>>(s->d_desc1, d_xyz, d_rgba, c, counter);
    else
      k_hash_fetch<1><<<1184, 512, 0, ctx->stream>>>(s->d_desc1, d_xyz, d_rgba, c, counter);
  } else switch (s->cfg.tsdf_format) {
    case 0: k_fetch_volume<0><<<1184, 256, 0, ctx->stream>>>(s->d_desc1, d_xyz, d_rgba, c, counter); break;
    case 1: k_fetch_volume<1><<<1184, 256, 0, ctx->stream>>>(s->d_desc1, d_xyz, d_rgba, c, counter); break;
    case 2: k_fetch_volume<2><<<1184, 256, 0, ctx->stream>>>(s->d_desc1, d_xyz, d_rgba, c, counter); break;
    default: k_fetch_volume<3><<<1184, 256, 0, ctx->stream>>>(s->d_desc1, d_xyz, d_rgba, c, counter); break;
  }
  NUI_CUDA(cudaGetLastError());
  unsigned long long n = 0;
  NUI_CUDA(cudaMemcpyAsync(&n, counter, sizeof(n), cudaMemcpyDeviceToHost, ctx->stream));
  NUI_CUDA(cudaStreamSynchronize(ctx->stream));
  *found = n;
  return NUI_OK;
}

NUI_API nui_status nui_session_work_counters(nui_session* s, uint64_t* out) {
  if (!s || !out) return fail(NUI_ERR_INVALID_ARG, "null argument");
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  TrackState t;
  NUI_CUDA(cudaMemcpy(&t, s->ts, sizeof(t), cudaMemcpyDeviceToHost));
  out[0] = t.touched;
  out[1] = t.bricks;
  out[2] = t.ray_reads;
  out[3] = t.ray_samples;
  out[4] = t.ray_hits;
  for (int l = 0; l < kMaxLevels; ++l) out[5 + l] = t.icp_iters[l];
  out[9] = t.tiles;
  return NUI_OK;
}

NUI_API nui_status nui_session_touched_voxels(nui_session* s, uint64_t* n) {
  if (!s || !n) return fail(NUI_ERR_INVALID_ARG, "null argument");
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  TrackState t;
  NUI_CUDA(cudaMemcpy(&t, s->ts, sizeof(t), cudaMemcpyDeviceToHost));
  *n = t.touched;
  return NUI_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ step-wise API, debug
namespace {
// Runs a subset of the tick on one session: `what` 0 = preprocess (+pyramid), 1 = track,
// 2 = integrate, 3 = raycast, 4 = feedback maps (frame-0 path).
nui_status run_stage(nui_session* s, int what) {
  nui_ctx* ctx = s->ctx;
  SessionDesc d;
  int kind = (what == 4 || (what == 2 && s->frames == 0)) ? kFirstFrame : kTrackFrame;
  fill_desc(s, d, kind, s->raw, s->color_frame ? s->bgra : nullptr);
  NUI_CUDA(cudaMemcpyAsync(s->d_desc1, &d, sizeof(d), cudaMemcpyHostToDevice, ctx->stream));
  BatchPlan p;
  p.n = 1;
  plan_add(p, s);
  cudaStream_t st = ctx->stream;
  const SessionDesc* dd = s->d_desc1;
  if (what == 0) {
    k_tick_begin<<<1, 64, 0, st>>>(dd, 1);
    k_preprocess<<<dim3(cdiv(p.maxW, 32) * cdiv(p.maxH, 16), 1), dim3(kPreBlockX, kPreBlockY), 0, st>>>(dd);
    for (int l = 1; l < p.maxLevels; ++l)
      k_pyramid<<<dim3(cdiv((long)(p.maxW >> l) * (p.maxH >> l), 256), 1), 256, 0, st>>>(dd, l);
  } else if (what == 1) {
    launch_track(p, dd, p.n, st, ctx->d_pose, ctx->d_status, p.colorIcp != 0, kFamAll, false);
  } else if (what == 2) {
    k_ztab<<<1, 32, 0, st>>>(dd);
    launch_shift(p, dd, st);
    launch_integrate<0>(p, dd, st);
    launch_integrate<1>(p, dd, st);
    launch_integrate<2>(p, dd, st);
    launch_integrate<3>(p, dd, st);
    launch_summaries(p, dd, st, 0);
    launch_hash_integrate(p, dd, st);
  } else if (what == 3) {
    launch_raycast<0>(p, dd, st);
    launch_raycast<1>(p, dd, st);
    launch_raycast<2>(p, dd, st);
    launch_raycast<3>(p, dd, st);
    launch_hash_raycast(p, dd, st);
  } else if (what == 4) {
    k_feedback<<<dim3(cdiv((long)p.maxW * p.maxH, 256), 1), 256, 0, st>>>(dd);
    if (p.colorIcp) k_color_keep<<<dim3(cdiv(((long)p.maxW * p.maxH + 3) / 4, 256), 1), 256, 0, st>>>(dd, kFamAll);
  }
  NUI_CUDA(cudaGetLastError());
  NUI_CUDA(cudaStreamSynchronize(st));
  return NUI_OK;
}

template <int F>
void launch_export(nui_session* s, short2* out, uchar4* cout) {
  k_export_ref<F><<<1184, 256, 0, s->ctx->stream>>>(s->d_desc1, out, cout);
}
template <int F>
void launch_import(nui_session* s, const short2* in) {
  k_import_ref<F><<<1184, 256, 0, s->ctx->stream>>>(s->d_desc1, in);
}
}  // namespace

extern "C" {

NUI_API nui_status nui_frame_upload(nui_session* s, const uint16_t* depth, const uint8_t* bgra) {
  if (!s || !depth) return fail(NUI_ERR_INVALID_ARG, "null argument");
  nui_status st = upload_frame(s, depth, bgra);
  if (st != NUI_OK) return st;
  return run_stage(s, 0);
}

NUI_API nui_status nui_feedback_update(nui_session* s) {
  if (!s) return fail(NUI_ERR_INVALID_ARG, "null session");
  return run_stage(s, 4);
}

NUI_API nui_status nui_track(nui_session* s, float* err, int* count) {
  if (!s) return fail(NUI_ERR_INVALID_ARG, "null session");
  nui_status st = ensure_cap(s->ctx, 1);
  if (st != NUI_OK) return st;
  // the track stage must run with the integration threshold of the session, and must
  // not integrate: k_track_finalize only decides the gate
  st = run_stage(s, 1);
  if (st != NUI_OK) return st;
  TrackState t;
  NUI_CUDA(cudaMemcpy(&t, s->ts, sizeof(t), cudaMemcpyDeviceToHost));
  if (err) *err = t.error;
  if (count) *count = (int)t.count;
  if (t.status != 0) {
    int zero = 0;
    cudaMemcpy(&s->ts->status, &zero, sizeof(int), cudaMemcpyHostToDevice);
    return fail(NUI_ERR_TRACKING_LOST, "ICP system is singular");
  }
  return NUI_OK;
}

NUI_API nui_status nui_integrate(nui_session* s) {
  if (!s) return fail(NUI_ERR_INVALID_ARG, "null session");
  int one = 1;
  NUI_CUDA(cudaMemcpy(&s->ts->integrate, &one, sizeof(int), cudaMemcpyHostToDevice));
  NUI_CUDA(cudaMemset(&s->ts->touched, 0, sizeof(unsigned long long)));
  if (!s->hash) return run_stage(s, 2);
  int before[16], after[16];
  NUI_CUDA(cudaMemcpy(before, s->hcount, sizeof(before), cudaMemcpyDeviceToHost));
  nui_status st = run_stage(s, 2);
  if (st != NUI_OK) return st;
  NUI_CUDA(cudaMemcpy(after, s->hcount, sizeof(after), cudaMemcpyDeviceToHost));
  if (after[kHashFailed] > before[kHashFailed] || after[kHashChainFaults] > before[kHashChainFaults])
    return fail(NUI_ERR_HASH_FULL, "voxel hash: pool or excess list exhausted (or a corrupted chain); blocks dropped");
  return NUI_OK;
}

NUI_API nui_status nui_raycast(nui_session* s) {
  if (!s) return fail(NUI_ERR_INVALID_ARG, "null session");
  return run_stage(s, 3);
}

NUI_API nui_status nui_debug_download(nui_session* s, int what, int level, void* host, size_t bytes) {
  if (!s || !host) return fail(NUI_ERR_INVALID_ARG, "null argument");
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  const nui_session_cfg& c = s->cfg;
  const size_t N = (size_t)c.width * c.height;
  const size_t nv = (size_t)c.res[0] * c.res[1] * c.res[2];
  if (level < 0 || level >= c.levels) return fail(NUI_ERR_INVALID_ARG, "bad level");
  if ((what == 5 || what == 6 || what == 9) && s->hash) return fail(NUI_ERR_INVALID_ARG, "not a dense session");
  if (what >= 20 && !s->hash) return fail(NUI_ERR_INVALID_ARG, "not a hash session");
  const size_t Nl = N >> (2 * level);
  const void* src = nullptr;
  size_t need = 0;
  switch (what) {
    case 0: src = s->dlev[0]; need = N * 4; break;
    case 1: src = s->dscaled; need = N * 4; break;
    case 2: {  // vertex map of a level, rebuilt from its depth
      need = Nl * 16;
      if (bytes < need) return fail(NUI_ERR_INVALID_ARG, "buffer too small");
      void* tmp = nullptr;
      NUI_CUDA(counted_malloc(&tmp, need));
      SessionDesc d;
      fill_desc(s, d, kInactive, nullptr, nullptr);
      cudaMemcpyAsync(s->d_desc1, &d, sizeof(d), cudaMemcpyHostToDevice, s->ctx->stream);
      k_vertex_map<<<dim3(cdiv((long)Nl, 256), 1), 256, 0, s->ctx->stream>>>(s->d_desc1, level, (float4*)tmp);
      cudaError_t e = cudaMemcpyAsync(host, tmp, need, cudaMemcpyDeviceToHost, s->ctx->stream);
      cudaStreamSynchronize(s->ctx->stream);
      cudaFree(tmp);
      if (e != cudaSuccess) return fail(NUI_ERR_DEVICE, cudaGetErrorString(e));
      return NUI_OK;
    }
    case 3: src = s->vref; need = N * 16; break;
    case 4: src = s->nref; need = N * 16; break;
    case 6: src = s->vol; need = nv * (c.tsdf_format == 2 ? 2 : voxel_bytes(c.tsdf_format)); break;
    case 7: src = s->dlev[level]; need = Nl * 4; break;
    case 8: src = s->cmap; need = N * 4; break;
    case 10: src = s->cprev; need = N * 4; break;
    case 11: src = s->cgx[level]; need = Nl * 4; break;
    case 12: src = s->cgy[level]; need = Nl * 4; break;
    case 13:  // brick states, one byte per 8^3 brick, x fastest
      if (s->hash) return fail(NUI_ERR_INVALID_ARG, "not a dense session");
      src = s->occ;
      need = (size_t)((c.res[0] + 7) / 8) * ((c.res[1] + 7) / 8) * ((c.res[2] + 7) / 8);
      break;
    case 14:  // the weight plane of NUI_TSDF_F16_U8
      if (s->hash || c.tsdf_format != NUI_TSDF_F16_U8) return fail(NUI_ERR_INVALID_ARG, "no weight plane");
      src = s->wvol;
      need = nv;
      break;
    case 20: src = s->entries; need = ((size_t)c.hash_buckets + c.hash_excess) * 16; break;
    case 21: {
      int cnt[4];
      NUI_CUDA(cudaMemcpy(cnt, s->hcount, 16, cudaMemcpyDeviceToHost));
      src = s->vis_ids;
      need = (size_t)cnt[2] * 4;
      break;
    }
    case 23: src = s->range; need = N * 8; break;
    case 24:  // the global cache's swap state per entry
      if (!s->swap) return fail(NUI_ERR_INVALID_ARG, "not a swapping hash session");
      src = s->swap;
      need = (size_t)c.hash_buckets + c.hash_excess;
      break;
    case 22: {
      if (!s->hash) return fail(NUI_ERR_INVALID_ARG, "not a hash session");
      need = (size_t)c.hash_pool_blocks * 512 * 6;
      if (bytes < need) return fail(NUI_ERR_INVALID_ARG, "buffer too small");
      void* tmp = nullptr;
      NUI_CUDA(counted_malloc(&tmp, need));
      SessionDesc d;
      fill_desc(s, d, kInactive, nullptr, nullptr);
      cudaMemcpyAsync(s->d_desc1, &d, sizeof(d), cudaMemcpyHostToDevice, s->ctx->stream);
      k_hash_export_voxels<<<1184, 256, 0, s->ctx->stream>>>(s->d_desc1, (uint8_t*)tmp);
      cudaError_t e = cudaMemcpyAsync(host, tmp, need, cudaMemcpyDeviceToHost, s->ctx->stream);
      cudaStreamSynchronize(s->ctx->stream);
      cudaFree(tmp);
      if (e != cudaSuccess) return fail(NUI_ERR_DEVICE, cudaGetErrorString(e));
      return NUI_OK;
    }
    case 5:
    case 9: {
      need = nv * 4;
      if (bytes < need) return fail(NUI_ERR_INVALID_ARG, "buffer too small");
      if (what == 9 && !s->cvol) return fail(NUI_ERR_INVALID_ARG, "no colour volume");
      void* tmp = nullptr;
      NUI_CUDA(counted_malloc(&tmp, need));
      SessionDesc d;
      fill_desc(s, d, kInactive, nullptr, nullptr);
      cudaMemcpyAsync(s->d_desc1, &d, sizeof(d), cudaMemcpyHostToDevice, s->ctx->stream);
      short2* vo = what == 5 ? (short2*)tmp : nullptr;
      uchar4* co = what == 9 ? (uchar4*)tmp : nullptr;
      switch (c.tsdf_format) {
        case 0: launch_export<0>(s, vo, co); break;
        case 1: launch_export<1>(s, vo, co); break;
        case 2: launch_export<2>(s, vo, co); break;
        case 3: launch_export<3>(s, vo, co); break;
      }
      cudaError_t e = cudaMemcpyAsync(host, tmp, need, cudaMemcpyDeviceToHost, s->ctx->stream);
      cudaStreamSynchronize(s->ctx->stream);
      cudaFree(tmp);
      if (e != cudaSuccess) return fail(NUI_ERR_DEVICE, cudaGetErrorString(e));
      return NUI_OK;
    }
    default:
      return fail(NUI_ERR_INVALID_ARG, "unknown buffer");
  }
  if (!src) return fail(NUI_ERR_INVALID_ARG, "buffer not present");
  if (bytes < need) return fail(NUI_ERR_INVALID_ARG, "buffer too small");
  NUI_CUDA(cudaMemcpy(host, src, need, cudaMemcpyDeviceToHost));
  return NUI_OK;
}

NUI_API nui_status nui_hash_stats(nui_session* s, int* visible, int* last_block, int* last_excess, int* failed) {
  if (!s || !s->hash) return fail(NUI_ERR_INVALID_ARG, "not a hash session");
  int cnt[4];
  NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  NUI_CUDA(cudaMemcpy(cnt, s->hcount, 16, cudaMemcpyDeviceToHost));
  if (visible) *visible = cnt[2];
  if (last_block) *last_block = cnt[0];
  if (last_excess) *last_excess = cnt[1];
  if (failed) *failed = cnt[3];
  return NUI_OK;
}

NUI_API nui_status nui_debug_upload_volume(nui_session* s, const int16_t* ref) {
  if (s && s->hash) return fail(NUI_ERR_UNSUPPORTED, "dense volumes only");
  if (!s || !ref) return fail(NUI_ERR_INVALID_ARG, "null argument");
  const size_t nv = (size_t)s->cfg.res[0] * s->cfg.res[1] * s->cfg.res[2];
  void* tmp = nullptr;
  NUI_CUDA(counted_malloc(&tmp, nv * 4));
  SessionDesc d;
  fill_desc(s, d, kInactive, nullptr, nullptr);
  cudaMemcpyAsync(s->d_desc1, &d, sizeof(d), cudaMemcpyHostToDevice, s->ctx->stream);
  cudaMemcpyAsync(tmp, ref, nv * 4, cudaMemcpyHostToDevice, s->ctx->stream);
  k_occ_clear<<<256, 256, 0, s->ctx->stream>>>(s->d_desc1);
  switch (s->cfg.tsdf_format) {
    case 0: launch_import<0>(s, (const short2*)tmp); break;
    case 1: launch_import<1>(s, (const short2*)tmp); break;
    case 2: launch_import<2>(s, (const short2*)tmp); break;
    case 3: launch_import<3>(s, (const short2*)tmp); break;
  }
  BatchPlan p;
  p.n = 1;
  plan_add(p, s);
  launch_summaries(p, s->d_desc1, s->ctx->stream, 1);
  cudaError_t e = cudaStreamSynchronize(s->ctx->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(NUI_ERR_DEVICE, cudaGetErrorString(e));
  return NUI_OK;
}

// ------------------------------------------------------------------ kernel-level calls
NUI_API nui_status nui_k_preprocess(nui_ctx* ctx, const uint16_t* d_raw, int W, int H, float fx, float fy, float cx,
                                    float cy, float dmin, float dmax, int radius, float ss2, float sd2, float thr,
                                    float* d_filtered, float* d_vertex4, float* d_scaled) {
  if (!ctx || !d_raw || !d_filtered || !d_vertex4 || !d_scaled || W <= 0 || H <= 0 || radius < 0 ||
      radius > kMaxRadius)
    return fail(NUI_ERR_INVALID_ARG, "bad argument");
  SessionDesc d;
  std::memset(&d, 0, sizeof(d));
  d.kind = kTrackFrame;
  d.W = W;
  d.H = H;
  d.levels = 1;
  d.cam = DevCam{fx, fy, 1 / fx, 1 / fy, cx, cy, W, H, dmin, dmax};
  d.radius = radius;
  d.sigma_depth = sd2;
  d.depth_thr = thr;
  for (int i = 0; i < 2 * radius + 1; ++i) {
    int x = i - radius;
    d.gauss[i] = std::exp((float)(-(x * x)) * ss2);
  }
  d.raw = d_raw;
  d.dlev[0] = d_filtered;
  d.vlev[0] = (float4*)d_vertex4;
  d.dscaled = d_scaled;
  NUI_CUDA(cudaMemcpyAsync(ctx->d_kdesc, &d, sizeof(d), cudaMemcpyHostToDevice, ctx->stream));
  k_preprocess<<<dim3(cdiv(W, 32) * cdiv(H, 16), 1), dim3(kPreBlockX, kPreBlockY), 0, ctx->stream>>>(ctx->d_kdesc);
  NUI_CUDA(cudaGetLastError());
  NUI_CUDA(cudaStreamSynchronize(ctx->stream));
  return NUI_OK;
}

NUI_API nui_status nui_k_pyramid_level(nui_ctx* ctx, const float* d_src, int dW, int dH, float fx, float fy, float cx,
                                       float cy, int div, float thr, float* d_dst, float* d_vertex4) {
  if (!ctx || !d_src || !d_dst || !d_vertex4 || dW <= 0 || dH <= 0) return fail(NUI_ERR_INVALID_ARG, "bad argument");
  int level = 0;
  while ((1 << level) < div) ++level;
  if ((1 << level) != div || level < 1 || level >= kMaxLevels) return fail(NUI_ERR_INVALID_ARG, "div must be 2, 4 or 8");
  SessionDesc d;
  std::memset(&d, 0, sizeof(d));
  d.kind = kTrackFrame;
  d.W = dW << level;
  d.H = dH << level;
  d.levels = level + 1;
  d.cam = DevCam{fx, fy, 1 / fx, 1 / fy, cx, cy, d.W, d.H, 0, 0};
  d.depth_thr = thr;
  d.dlev[level - 1] = const_cast<float*>(d_src);
  d.dlev[level] = d_dst;
  d.vlev[level] = (float4*)d_vertex4;
  NUI_CUDA(cudaMemcpyAsync(ctx->d_kdesc, &d, sizeof(d), cudaMemcpyHostToDevice, ctx->stream));
  k_pyramid<<<dim3(cdiv((long)dW * dH, 256), 1), 256, 0, ctx->stream>>>(ctx->d_kdesc, level);
  NUI_CUDA(cudaGetLastError());
  NUI_CUDA(cudaStreamSynchronize(ctx->stream));
  return NUI_OK;
}

NUI_API nui_status nui_k_color_pyramid(nui_ctx* ctx, const uint8_t* d_bgra, int W, int H, int levels,
                                       uint8_t* const* d_levels, uint8_t* const* d_gx, uint8_t* const* d_gy) {
  if (!ctx || !d_bgra || !d_levels || !d_gx || !d_gy || W <= 0 || H <= 0 || levels < 1 || levels > kMaxLevels)
    return fail(NUI_ERR_INVALID_ARG, "bad argument");
  if (((W >> (levels - 1)) << (levels - 1)) != W || ((H >> (levels - 1)) << (levels - 1)) != H)
    return fail(NUI_ERR_INVALID_ARG, "image size must be divisible by 2^(levels-1)");
  SessionDesc d;
  std::memset(&d, 0, sizeof(d));
  d.kind = kTrackFrame;
  d.W = W;
  d.H = H;
  d.levels = levels;
  d.photo_w = 1.f;
  d.bgra = d_bgra;
  for (int l = 0; l < levels; ++l) {
    if ((l > 0 && !d_levels[l]) || !d_gx[l] || !d_gy[l]) return fail(NUI_ERR_INVALID_ARG, "null level buffer");
    d.cpyr[l] = l > 0 ? (uchar4*)d_levels[l] : nullptr;
    d.cgx[l] = (uchar4*)d_gx[l];
    d.cgy[l] = (uchar4*)d_gy[l];
  }
  NUI_CUDA(cudaMemcpyAsync(ctx->d_kdesc, &d, sizeof(d), cudaMemcpyHostToDevice, ctx->stream));
  for (int l = 1; l < levels; ++l)
    k_color_level<<<dim3(cdiv((long)(W >> l) * (H >> l), 256), 1), 256, 0, ctx->stream>>>(ctx->d_kdesc, l);
  k_color_grad<<<dim3(cdiv((long)W * H, 256), 1, levels), 256, 0, ctx->stream>>>(ctx->d_kdesc, kFamAll);
  NUI_CUDA(cudaGetLastError());
  NUI_CUDA(cudaStreamSynchronize(ctx->stream));
  return NUI_OK;
}

NUI_API nui_status nui_k_feedback_maps(nui_ctx* ctx, const float* d_vertex4, int W, int H, float thr,
                                       const float* pose12, float* d_vref4, float* d_nref4) {
  if (!ctx || !d_vertex4 || !pose12 || !d_vref4 || !d_nref4 || W <= 0 || H <= 0)
    return fail(NUI_ERR_INVALID_ARG, "bad argument");
  TrackState t;
  std::memset(&t, 0, sizeof(t));
  std::memcpy(t.xf.R, pose12, 9 * sizeof(float));
  std::memcpy(t.xf.t, pose12 + 9, 3 * sizeof(float));
  SessionDesc d;
  std::memset(&d, 0, sizeof(d));
  d.kind = kFirstFrame;
  d.W = W;
  d.H = H;
  d.levels = 1;
  d.depth_thr = thr;
  d.vlev[0] = (float4*)const_cast<float*>(d_vertex4);
  d.vref = (float4*)d_vref4;
  d.nref = (float4*)d_nref4;
  d.ts = ctx->d_kts;
  NUI_CUDA(cudaMemcpyAsync(ctx->d_kts, &t, sizeof(t), cudaMemcpyHostToDevice, ctx->stream));
  NUI_CUDA(cudaMemcpyAsync(ctx->d_kdesc, &d, sizeof(d), cudaMemcpyHostToDevice, ctx->stream));
  k_feedback<<<dim3(cdiv((long)W * H, 256), 1), 256, 0, ctx->stream>>>(ctx->d_kdesc);
  NUI_CUDA(cudaGetLastError());
  NUI_CUDA(cudaStreamSynchronize(ctx->stream));
  return NUI_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ marching cubes
namespace {
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
}  // namespace
namespace nui {
void hash_mc_upload_tables(cudaStream_t st, const uint64_t* table);
template <int F>
__global__ void k_hash_mesh_count(const SessionDesc*, unsigned*);
__global__ void k_hash_mesh_scan(const unsigned*, unsigned long long*, int);
template <int F>
__global__ void k_hash_mesh_emit(const SessionDesc*, const unsigned long long*, float*, float*, unsigned long long);
}  // namespace nui
#include "nui_mc_tables.h"
namespace {
// Volume2CLMesh of the hash scene: the visible blocks of the last integration.
nui_status nui_hash_mesh_impl(nui_session* s, float* pos, float* col, uint64_t cap, uint64_t* nverts) {
  cudaStream_t st = s->ctx->stream;
  int cnt4[4];
  NUI_CUDA(cudaStreamSynchronize(st));
  NUI_CUDA(cudaMemcpy(cnt4, s->hcount, 16, cudaMemcpyDeviceToHost));
  const int nvis = cnt4[2];
  *nverts = 0;
  if (nvis == 0) return NUI_OK;
  SessionDesc d;
  fill_desc(s, d, kInactive, nullptr, nullptr);
  NUI_CUDA(cudaMemcpyAsync(s->d_desc1, &d, sizeof(d), cudaMemcpyHostToDevice, st));
  hash_mc_upload_tables(st, NUI_MC_TRI_PACKED);
  DevBuf cnt, off, dp, dc;
  NUI_CUDA(counted_malloc(&cnt.p, (size_t)nvis * 4));
  NUI_CUDA(counted_malloc(&off.p, ((size_t)nvis + 1) * 8));
  const int hf = d.hfmt;
  if (hf == 0)
    k_hash_mesh_count<0><<<1184, 512, 0, st>>>(s->d_desc1, (unsigned*)cnt.p);
  else
    k_hash_mesh_count<1><<<1184, 512, 0, st>>>(s->d_desc1, (unsigned*)cnt.p);
  k_hash_mesh_scan<<<1, 1024, 0, st>>>((const unsigned*)cnt.p, (unsigned long long*)off.p, nvis);
  unsigned long long total = 0;
  NUI_CUDA(cudaMemcpyAsync(&total, (unsigned long long*)off.p + nvis, 8, cudaMemcpyDeviceToHost, st));
  NUI_CUDA(cudaStreamSynchronize(st));
  *nverts = total;
  const unsigned long long k = total < cap ? total : cap;
  if (k > 0 && (pos || col)) {
    if (pos) NUI_CUDA(counted_malloc(&dp.p, k * 12));
    if (col) NUI_CUDA(counted_malloc(&dc.p, k * 16));
    if (hf == 0)
      k_hash_mesh_emit<0><<<1184, 512, 0, st>>>(s->d_desc1, (const unsigned long long*)off.p, (float*)dp.p, (float*)dc.p, k);
    else
      k_hash_mesh_emit<1><<<1184, 512, 0, st>>>(s->d_desc1, (const unsigned long long*)off.p, (float*)dp.p, (float*)dc.p, k);
    NUI_CUDA(cudaGetLastError());
    if (pos) NUI_CUDA(cudaMemcpyAsync(pos, dp.p, k * 12, cudaMemcpyDeviceToHost, st));
    if (col) NUI_CUDA(cudaMemcpyAsync(col, dc.p, k * 16, cudaMemcpyDeviceToHost, st));
    NUI_CUDA(cudaStreamSynchronize(st));
  }
  if (total > cap) return fail(NUI_ERR_MESH_OVERFLOW, "mesh larger than the output capacity");
  return NUI_OK;
}
}  // namespace
namespace nui {
void mc_upload_tables(cudaStream_t st);
template <int F>
__global__ void k_mc_count(const SessionDesc*, unsigned int*, unsigned long long*, uint8_t*);
__global__ void k_mc_scan(unsigned long long*, int);
template <int F>
__global__ void k_mc_emit(const SessionDesc*, const unsigned int*, const unsigned long long*, float*, float*,
                          unsigned long long);
}  // namespace nui

namespace {
template <int F>
void mc_count(nui_session* s, unsigned nb, unsigned* cc, unsigned long long* bt, uint8_t* cases) {
  k_mc_count<F><<<nb, 128, 0, s->ctx->stream>>>(s->d_desc1, cc, bt, cases);
}
template <int F>
void mc_emit(nui_session* s, unsigned nb, const unsigned* cc, const unsigned long long* bt, float* p, float* c,
             unsigned long long cap) {
  k_mc_emit<F><<<nb, 128, 0, s->ctx->stream>>>(s->d_desc1, cc, bt, p, c, cap);
}
// Count pass + block scan; returns the total vertex count.
nui_status mc_prepare(nui_session* s, DevBuf& cc, DevBuf& bt, unsigned& nb, uint8_t* d_cases,
                      unsigned long long& total) {
  const nui_session_cfg& c = s->cfg;
  cudaStream_t st = s->ctx->stream;
  SessionDesc d;
  fill_desc(s, d, kInactive, nullptr, nullptr);
  NUI_CUDA(cudaMemcpyAsync(s->d_desc1, &d, sizeof(d), cudaMemcpyHostToDevice, st));
  mc_upload_tables(st);
  const unsigned tilesX = cdiv(c.res[0] - 1, 128);
  nb = tilesX * (unsigned)(c.res[1] - 1);
  NUI_CUDA(counted_malloc(&cc.p, sizeof(unsigned) * (size_t)(c.res[0] - 1) * (c.res[1] - 1)));
  NUI_CUDA(counted_malloc(&bt.p, sizeof(unsigned long long) * (nb + 1)));
  switch (c.tsdf_format) {
    case 0: mc_count<0>(s, nb, (unsigned*)cc.p, (unsigned long long*)bt.p, d_cases); break;
    case 1: mc_count<1>(s, nb, (unsigned*)cc.p, (unsigned long long*)bt.p, d_cases); break;
    case 2: mc_count<2>(s, nb, (unsigned*)cc.p, (unsigned long long*)bt.p, d_cases); break;
    case 3: mc_count<3>(s, nb, (unsigned*)cc.p, (unsigned long long*)bt.p, d_cases); break;
  }
  k_mc_scan<<<1, 1024, 0, st>>>((unsigned long long*)bt.p, (int)nb);
  NUI_CUDA(cudaGetLastError());
  NUI_CUDA(cudaMemcpyAsync(&total, (unsigned long long*)bt.p + nb, sizeof(total), cudaMemcpyDeviceToHost, st));
  NUI_CUDA(cudaStreamSynchronize(st));
  return NUI_OK;
}
}  // namespace

extern "C" NUI_API nui_status nui_mesh(nui_session* s, float* pos, float* col, uint64_t cap, uint64_t* nverts) {
  if (!s || !nverts) return fail(NUI_ERR_INVALID_ARG, "null argument");
  if (s->hash) return nui_hash_mesh_impl(s, pos, col, cap, nverts);
  DevBuf cc, bt, dp, dc;
  unsigned nb = 0;
  unsigned long long total = 0;
  nui_status st = mc_prepare(s, cc, bt, nb, nullptr, total);
  if (st != NUI_OK) return st;
  *nverts = total;
  const unsigned long long k = total < cap ? total : cap;
  if (k > 0 && (pos || col)) {
    if (pos) NUI_CUDA(counted_malloc(&dp.p, k * 3 * sizeof(float)));
    if (col) NUI_CUDA(counted_malloc(&dc.p, k * 4 * sizeof(float)));
    switch (s->cfg.tsdf_format) {
      case 0: mc_emit<0>(s, nb, (unsigned*)cc.p, (unsigned long long*)bt.p, (float*)dp.p, (float*)dc.p, k); break;
      case 1: mc_emit<1>(s, nb, (unsigned*)cc.p, (unsigned long long*)bt.p, (float*)dp.p, (float*)dc.p, k); break;
      case 2: mc_emit<2>(s, nb, (unsigned*)cc.p, (unsigned long long*)bt.p, (float*)dp.p, (float*)dc.p, k); break;
      case 3: mc_emit<3>(s, nb, (unsigned*)cc.p, (unsigned long long*)bt.p, (float*)dp.p, (float*)dc.p, k); break;
    }
    NUI_CUDA(cudaGetLastError());
    if (pos) NUI_CUDA(cudaMemcpyAsync(pos, dp.p, k * 3 * sizeof(float), cudaMemcpyDeviceToHost, s->ctx->stream));
    if (col) NUI_CUDA(cudaMemcpyAsync(col, dc.p, k * 4 * sizeof(float), cudaMemcpyDeviceToHost, s->ctx->stream));
    NUI_CUDA(cudaStreamSynchronize(s->ctx->stream));
  }
  if (total > cap) return fail(NUI_ERR_MESH_OVERFLOW, "mesh larger than the output capacity");
  return NUI_OK;
}

extern "C" NUI_API nui_status nui_mesh_cases(nui_session* s, uint8_t* cases, size_t bytes, uint64_t* nverts) {
  if (!s || !cases) return fail(NUI_ERR_INVALID_ARG, "null argument");
  if (s->hash) return fail(NUI_ERR_UNSUPPORTED, "case indices of dense volumes only");
  const nui_session_cfg& c = s->cfg;
  const size_t need = (size_t)(c.res[0] - 1) * (c.res[1] - 1) * (c.res[2] - 1);
  if (bytes < need) return fail(NUI_ERR_INVALID_ARG, "buffer too small");
  DevBuf cc, bt, dcase;
  NUI_CUDA(counted_malloc(&dcase.p, need));
  unsigned nb = 0;
  unsigned long long total = 0;
  nui_status st = mc_prepare(s, cc, bt, nb, (uint8_t*)dcase.p, total);
  if (st != NUI_OK) return st;
  NUI_CUDA(cudaMemcpy(cases, dcase.p, need, cudaMemcpyDeviceToHost));
  if (nverts) *nverts = total;
  return NUI_OK;
}

// ------------------------------------------------------------------ meshing without allocation
// Scratch of nui_mesh_device_noalloc: per-column vertex counts (u32) and per-block offsets
// (u64).  A file-scope device array: host code reaches it only through the address that
// cudaGetSymbolAddress returns for the current device.
namespace {
constexpr size_t kNoAllocCols = 262144;   // (res[0]-1)*(res[1]-1) bound
constexpr size_t kNoAllocBlocks = 4096;   // count blocks + 1 bound
static __device__ __align__(256) unsigned char g_mesh_scratch[kNoAllocCols * 4 + kNoAllocBlocks * 8];
constexpr int kMaxDevices = 64;
unsigned char* g_mesh_scratch_addr[kMaxDevices] = {};
std::mutex g_mesh_scratch_mu;

// Restores the caller's current device when the entry point returns.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      prev = -1;
      cudaGetLastError();
    }
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Device address of the scratch array on `device` (current); looked up on the first call
// after the library loads or after a context is created on the device (nui_ctx_create
// forgets the cached address, so that a device reset followed by a new context looks it up
// again).  Nothing in the array needs to start at zero: the count pass writes every column
// count and every block total before the scan and the emit pass read them.
nui_status noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) return fail(NUI_ERR_INVALID_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(g_mesh_scratch_mu);
  if (!g_mesh_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_mesh_scratch);
    if (e != cudaSuccess) return fail(NUI_ERR_DEVICE, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_mesh_scratch_addr[device] = (unsigned char*)p;
  }
  *out = g_mesh_scratch_addr[device];
  return NUI_OK;
}

void noalloc_forget(int device) {
  if (device < 0 || device >= kMaxDevices) return;
  std::lock_guard<std::mutex> lock(g_mesh_scratch_mu);
  g_mesh_scratch_addr[device] = nullptr;
}
}  // namespace

extern "C" NUI_API nui_status nui_debug_allocation_count(uint64_t* n) {
  if (!n) return fail(NUI_ERR_INVALID_ARG, "null argument");
  *n = g_allocations.load(std::memory_order_relaxed);
  return NUI_OK;
}

extern "C" NUI_API nui_status nui_mesh_device_noalloc(nui_session* s, float* d_pos, float* d_col, uint64_t cap,
                                                      uint64_t* nverts) {
  if (!s || !nverts) return fail(NUI_ERR_INVALID_ARG, "null argument");
  if (s->hash) return fail(NUI_ERR_UNSUPPORTED, "dense sessions only");
  const nui_session_cfg& c = s->cfg;
  const size_t ncols = (size_t)(c.res[0] - 1) * (c.res[1] - 1);
  const unsigned nb = cdiv(c.res[0] - 1, 128) * (unsigned)(c.res[1] - 1);
  if (ncols > kNoAllocCols || (size_t)nb + 1 > kNoAllocBlocks)
    return fail(NUI_ERR_INVALID_ARG, "volume too large for the no-allocation mesh scratch");
  DeviceGuard guard;
  NUI_CUDA(cudaSetDevice(s->ctx->device));
  for (const float* q : {(const float*)d_pos, (const float*)d_col}) {
    if (!q) continue;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, q) != cudaSuccess ||
        (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)) {
      cudaGetLastError();
      return fail(NUI_ERR_INVALID_ARG, "output buffers must be device memory");
    }
    if (a.type == cudaMemoryTypeDevice && a.device != s->ctx->device)
      return fail(NUI_ERR_INVALID_ARG, "output buffers must be on the session's device");
  }
  unsigned char* base = nullptr;
  nui_status st0 = noalloc_scratch(s->ctx->device, &base);
  if (st0 != NUI_OK) return st0;
  unsigned* cc = (unsigned*)base;
  unsigned long long* bt = (unsigned long long*)(base + kNoAllocCols * 4);
  cudaStream_t st = s->ctx->stream;
  SessionDesc d;
  fill_desc(s, d, kInactive, nullptr, nullptr);
  NUI_CUDA(cudaMemcpyAsync(s->d_desc1, &d, sizeof(d), cudaMemcpyHostToDevice, st));
  mc_upload_tables(st);
  switch (c.tsdf_format) {
    case 0: mc_count<0>(s, nb, cc, bt, nullptr); break;
    case 1: mc_count<1>(s, nb, cc, bt, nullptr); break;
    case 2: mc_count<2>(s, nb, cc, bt, nullptr); break;
    case 3: mc_count<3>(s, nb, cc, bt, nullptr); break;
  }
  k_mc_scan<<<1, 1024, 0, st>>>(bt, (int)nb);
  NUI_CUDA(cudaGetLastError());
  unsigned long long total = 0;
  NUI_CUDA(cudaMemcpyAsync(&total, bt + nb, sizeof(total), cudaMemcpyDeviceToHost, st));
  NUI_CUDA(cudaStreamSynchronize(st));
  *nverts = total;
  const unsigned long long k = total < cap ? total : cap;
  if (k > 0 && (d_pos || d_col)) {
    switch (c.tsdf_format) {
      case 0: mc_emit<0>(s, nb, cc, bt, d_pos, d_col, k); break;
      case 1: mc_emit<1>(s, nb, cc, bt, d_pos, d_col, k); break;
      case 2: mc_emit<2>(s, nb, cc, bt, d_pos, d_col, k); break;
      case 3: mc_emit<3>(s, nb, cc, bt, d_pos, d_col, k); break;
    }
    NUI_CUDA(cudaGetLastError());
    NUI_CUDA(cudaStreamSynchronize(st));
  }
  if (total > cap) return fail(NUI_ERR_MESH_OVERFLOW, "mesh larger than the output capacity");
  return NUI_OK;
}

// ------------------------------------------------------------------ serving loop
// Every tick of the server covers all its slots (empty or idle ones sit out), with a
// launch shape that only grows as streams of new kinds are admitted: the captured graph
// of a tick is therefore reused while streams come and go.  Released sessions are kept
// for the next stream of the same configuration (a reset instead of a free and an
// allocation, which would synchronise the device); they are freed when a new stream
// needs their memory.
struct nui_server {
  struct Frame {
    const uint16_t* depth;
    const uint8_t* bgra;
    uint64_t tag;
    double t_submit;
  };
  struct Slot {
    nui_session* s = nullptr;
    size_t bytes = 0;
    std::deque<Frame> q;
    uint16_t* draw[2] = {nullptr, nullptr};  // device frame double buffer
    uint8_t* dbgra[2] = {nullptr, nullptr};
    size_t cap_px = 0;                       // pixels the buffers hold
    bool cap_bgra = false;
    int buf = 0;
  };
  struct Pooled {
    nui_session* s;
    size_t bytes;
  };
  nui_ctx* ctx = nullptr;
  size_t budget = 0, used = 0;  // live and pooled sessions
  cudaStream_t up = nullptr;
  cudaEvent_t ev_t0 = nullptr, ev_up = nullptr, ev_order = nullptr;
  cudaEvent_t ev_done[2] = {nullptr, nullptr};  // behind the tick of each host staging half
  std::chrono::steady_clock::time_point t0;
  std::vector<Slot> slots;
  std::vector<Pooled> pool;
  BatchPlan floor;
  // the batch in flight: every slot, with its session and frame (or none), and the
  // context's staging half it was launched with
  bool inflight = false;
  int bpar = 0;
  std::vector<nui_session*> bsess;
  std::vector<const uint16_t*> braw;
  std::vector<const uint8_t*> bbgra;
  std::vector<Frame> bframe;
  std::vector<nui_server_result> done;
  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {
nui_status server_collect(nui_server* v) {
  if (!v->inflight) return NUI_OK;
  v->inflight = false;
  NUI_CUDA(cudaEventSynchronize(v->ev_done[v->bpar]));
  float ms = 0.f;
  NUI_CUDA(cudaEventElapsedTime(&ms, v->ev_t0, v->ev_done[v->bpar]));
  const double t_done = ms * 1e-3;
  const int n = (int)v->bsess.size();
  std::vector<nui_status> per(n);
  std::vector<float> poses(12 * (size_t)n);
  nui_status st = tick_finish(v->ctx, v->bsess.data(), n, v->braw.data(), per.data(), poses.data(), v->bpar);
  if (st != NUI_OK && st != NUI_ERR_TRACKING_LOST && st != NUI_ERR_HASH_FULL) return st;
  for (int i = 0; i < n; ++i) {
    if (!v->bsess[i] || !v->braw[i]) continue;
    nui_server_result r;
    r.slot = i;
    r.status = per[i];
    r.tag = v->bframe[i].tag;
    r.t_submit = v->bframe[i].t_submit;
    r.t_done = t_done;
    std::memcpy(r.pose, poses.data() + 12 * i, sizeof(r.pose));
    v->done.push_back(r);
  }
  return NUI_OK;
}

// A slot's frame buffers come from the context's pool in the order of the upload stream:
// they are freed there behind the batch in flight (which may still read them) and the
// new ones allocated there before the first upload into them, so that neither waits for
// the device.
void server_free_slot_buffers(nui_server* v, nui_server::Slot& sl) {
  if (sl.draw[0] || sl.dbgra[0]) {
    cudaEventRecord(v->ev_order, v->ctx->stream);
    cudaStreamWaitEvent(v->up, v->ev_order, 0);
  }
  for (int b = 0; b < 2; ++b) {
    if (sl.draw[b]) cudaFreeAsync(sl.draw[b], v->up);
    if (sl.dbgra[b]) cudaFreeAsync(sl.dbgra[b], v->up);
    sl.draw[b] = nullptr;
    sl.dbgra[b] = nullptr;
  }
  sl.cap_px = 0;
  sl.cap_bgra = false;
}
}  // namespace

extern "C" {

NUI_API nui_status nui_server_create(nui_ctx* ctx, size_t budget, int max_streams, nui_server** out) {
  if (!ctx || !out || max_streams <= 0 || max_streams > 4096) return fail(NUI_ERR_INVALID_ARG, "bad argument");
  NUI_CUDA(cudaSetDevice(ctx->device));
  nui_server* v = new nui_server();
  v->ctx = ctx;
  v->budget = budget;
  v->slots.resize(max_streams);
  v->floor.n = max_streams;
  if (cudaStreamCreateWithFlags(&v->up, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&v->ev_t0) != cudaSuccess || cudaEventCreateWithFlags(&v->ev_up, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&v->ev_done[0]) != cudaSuccess || cudaEventCreate(&v->ev_done[1]) != cudaSuccess ||
      cudaEventCreateWithFlags(&v->ev_order, cudaEventDisableTiming) != cudaSuccess) {
    delete v;
    return fail(NUI_ERR_DEVICE, "stream / event creation failed");
  }
  // The budget is taken into the context's pool now (one allocation, freed at once: the
  // pool keeps the memory, its release threshold being unbounded), so that admissions
  // sub-allocate from memory the pool holds instead of mapping new memory while ticks run.
  // A budget above what the device has free is taken as far as it goes.
  {
    size_t free_b = 0, total_b = 0;
    NUI_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t margin = (size_t)2 << 30;
    const size_t take = std::min(budget, free_b > margin ? free_b - margin : 0);
    void* p = nullptr;
    if (take > 0 && counted_pool_alloc(&p, take, ctx->pool, ctx->stream) == cudaSuccess) {
      cudaFreeAsync(p, ctx->stream);
    } else {
      cudaGetLastError();
    }
  }
  // the server clock: host time of a recorded event, so device completion times map onto it
  NUI_CUDA(cudaStreamSynchronize(ctx->stream));
  NUI_CUDA(cudaEventRecord(v->ev_t0, ctx->stream));
  NUI_CUDA(cudaEventSynchronize(v->ev_t0));
  v->t0 = std::chrono::steady_clock::now();
  *out = v;
  return NUI_OK;
}

NUI_API nui_status nui_server_destroy(nui_server* v) {
  if (!v) return NUI_OK;
  server_collect(v);
  cudaStreamSynchronize(v->up);
  for (auto& sl : v->slots) {
    if (sl.s) nui_session_destroy(sl.s);
    server_free_slot_buffers(v, sl);
  }
  cudaStreamSynchronize(v->up);
  for (auto& p : v->pool) nui_session_destroy(p.s);
  nui_ctx_trim(v->ctx);  // the served sessions' memory goes back to the device
  cudaStreamDestroy(v->up);
  cudaEventDestroy(v->ev_t0);
  cudaEventDestroy(v->ev_up);
  cudaEventDestroy(v->ev_done[0]);
  cudaEventDestroy(v->ev_done[1]);
  cudaEventDestroy(v->ev_order);
  delete v;
  return NUI_OK;
}

NUI_API double nui_server_clock(const nui_server* v) { return v ? v->now() : 0.0; }

NUI_API nui_status nui_server_admit(nui_server* v, const nui_session_cfg* cfg, int* slot) {
  if (!v || !cfg || !slot) return fail(NUI_ERR_INVALID_ARG, "null argument");
  std::string why;
  if (!cfg_valid(cfg, why)) return fail(NUI_ERR_INVALID_ARG, why);
  const size_t need = nui_session_device_bytes(cfg) + (size_t)cfg->width * cfg->height * 12;
  int k = -1;
  for (int i = 0; i < (int)v->slots.size() && k < 0; ++i)
    if (!v->slots[i].s) k = i;
  if (k < 0) return fail(NUI_ERR_OOM, "no free stream slot");
  // a pooled session of the same configuration, else room for a new one
  nui_session* s = nullptr;
  size_t bytes = need;
  for (size_t i = 0; i < v->pool.size() && !s; ++i)
    if (std::memcmp(&v->pool[i].s->cfg, cfg, sizeof(nui_session_cfg)) == 0) {
      s = v->pool[i].s;
      bytes = v->pool[i].bytes;
      v->pool.erase(v->pool.begin() + i);
      nui_status st = reset_session(s, false);  // queued behind the batch in flight
      if (st != NUI_OK) return st;
    }
  if (!s) {
    // pooled sessions of other configurations make room; frees and the new session's
    // allocation and reset are queued on the context stream behind the tick in flight
    while (v->used + need > v->budget && !v->pool.empty()) {
      session_free(v->pool.front().s, false);
      v->used -= v->pool.front().bytes;
      v->pool.erase(v->pool.begin());
    }
    if (v->used + need > v->budget) return fail(NUI_ERR_OOM, "stream does not fit in the HBM budget");
    nui_status st = session_create(v->ctx, cfg, &s, false);
    if (st != NUI_OK) return st;
    v->used += need;
  }
  nui_server::Slot& sl = v->slots[k];
  const size_t N = (size_t)cfg->width * cfg->height;
  const bool col = s->cmap != nullptr;
  if (sl.cap_px < N || (col && !sl.cap_bgra)) {
    server_free_slot_buffers(v, sl);
    bool ok = true;
    for (int b = 0; b < 2 && ok; ++b) {
      ok = counted_pool_alloc((void**)&sl.draw[b], N * 2, v->ctx->pool, v->up) == cudaSuccess;
      if (ok && col) ok = counted_pool_alloc((void**)&sl.dbgra[b], N * 4, v->ctx->pool, v->up) == cudaSuccess;
    }
    if (!ok) {
      cudaGetLastError();
      server_free_slot_buffers(v, sl);
      v->pool.push_back(nui_server::Pooled{s, bytes});
      return fail(NUI_ERR_OOM, "device allocation failed");
    }
    sl.cap_px = N;
    sl.cap_bgra = col;
  }
  sl.s = s;
  sl.bytes = bytes;
  sl.buf = 0;
  sl.q.clear();
  plan_add(v->floor, s);
  *slot = k;
  return NUI_OK;
}

NUI_API nui_status nui_server_reserve(nui_server* v, const nui_session_cfg* cfg, int count) {
  if (!v || !cfg || count < 0) return fail(NUI_ERR_INVALID_ARG, "bad argument");
  std::string why;
  if (!cfg_valid(cfg, why)) return fail(NUI_ERR_INVALID_ARG, why);
  const size_t need = nui_session_device_bytes(cfg) + (size_t)cfg->width * cfg->height * 12;
  for (int i = 0; i < count; ++i) {
    if (v->used + need > v->budget) return fail(NUI_ERR_OOM, "reservation does not fit in the HBM budget");
    nui_session* s = nullptr;
    nui_status st = nui_session_create(v->ctx, cfg, &s);
    if (st != NUI_OK) return st;
    v->used += need;
    v->pool.push_back(nui_server::Pooled{s, need});
    // the tick's launch shape covers the reserved kinds from now on, so that their streams
    // join without a new graph capture
    plan_add(v->floor, s);
  }
  return NUI_OK;
}

NUI_API nui_status nui_server_release(nui_server* v, int slot) {
  if (!v || slot < 0 || slot >= (int)v->slots.size() || !v->slots[slot].s) return fail(NUI_ERR_INVALID_ARG, "bad slot");
  if (v->inflight && v->bsess[slot]) {
    nui_status st = server_collect(v);
    if (st != NUI_OK) return st;
  }
  nui_server::Slot& sl = v->slots[slot];
  v->pool.push_back(nui_server::Pooled{sl.s, sl.bytes});  // kept for the next stream like it
  sl.s = nullptr;
  sl.q.clear();
  sl.bytes = 0;
  return NUI_OK;
}

NUI_API nui_status nui_server_submit(nui_server* v, int slot, const uint16_t* depth, const uint8_t* bgra, uint64_t tag,
                                     double t_submit) {
  if (!v || !depth || slot < 0 || slot >= (int)v->slots.size() || !v->slots[slot].s)
    return fail(NUI_ERR_INVALID_ARG, "bad slot or frame");
  v->slots[slot].q.push_back(nui_server::Frame{depth, bgra, tag, t_submit < 0 ? v->now() : t_submit});
  return NUI_OK;
}

NUI_API nui_status nui_server_step(nui_server* v, int* launched) {
  if (!v) return fail(NUI_ERR_INVALID_ARG, "null server");
  const int ns = (int)v->slots.size();
  // the next batch: every slot, with the oldest queued frame of its stream if it has one
  std::vector<nui_session*> nsess(ns, nullptr);
  std::vector<const uint16_t*> nraw(ns, nullptr);
  std::vector<const uint8_t*> nbgra(ns, nullptr);
  std::vector<nui_server::Frame> nframe(ns, nui_server::Frame{nullptr, nullptr, 0, 0.0});
  int count = 0;
  for (int i = 0; i < ns; ++i) {
    nui_server::Slot& sl = v->slots[i];
    if (!sl.s) continue;
    nsess[i] = sl.s;
    if (sl.q.empty()) continue;
    nui_server::Frame f = sl.q.front();
    sl.q.pop_front();
    const int b = sl.buf ^ 1;  // the buffer the batch in flight does not read
    sl.buf = b;
    const size_t N = (size_t)sl.s->cfg.width * sl.s->cfg.height;
    NUI_CUDA(cudaMemcpyAsync(sl.draw[b], f.depth, N * 2, cudaMemcpyHostToDevice, v->up));
    if (f.bgra && sl.dbgra[b]) {
      NUI_CUDA(cudaMemcpyAsync(sl.dbgra[b], f.bgra, N * 4, cudaMemcpyHostToDevice, v->up));
      nbgra[i] = sl.dbgra[b];
    }
    nraw[i] = sl.draw[b];
    nframe[i] = f;
    ++count;
  }
  NUI_CUDA(cudaEventRecord(v->ev_up, v->up));
  if (launched) *launched = count;
  if (count == 0) return server_collect(v);
  // the new batch is queued behind the one in flight before that one is waited for, so
  // that the device goes from one tick to the next without waiting for the host
  NUI_CUDA(cudaStreamWaitEvent(v->ctx->stream, v->ev_up, 0));
  int par = 0;
  nui_status st = tick_launch(v->ctx, nsess.data(), ns, nraw.data(), nbgra.data(), true, &v->floor, &par);
  if (st != NUI_OK) {
    server_collect(v);
    return st;
  }
  NUI_CUDA(cudaEventRecord(v->ev_done[par], v->ctx->stream));
  st = server_collect(v);  // the batch launched by the previous step
  v->bsess.swap(nsess);
  v->braw.swap(nraw);
  v->bbgra.swap(nbgra);
  v->bframe.swap(nframe);
  v->bpar = par;
  v->inflight = true;
  return st;
}

NUI_API nui_status nui_server_drain(nui_server* v) {
  if (!v) return fail(NUI_ERR_INVALID_ARG, "null server");
  return server_collect(v);
}

NUI_API nui_status nui_server_poll(nui_server* v, nui_server_result* out, int cap, int* n) {
  if (!v || !n || (cap > 0 && !out)) return fail(NUI_ERR_INVALID_ARG, "null argument");
  const int k = std::min(cap, (int)v->done.size());
  for (int i = 0; i < k; ++i) out[i] = v->done[i];
  v->done.erase(v->done.begin(), v->done.begin() + k);
  *n = k;
  return NUI_OK;
}

NUI_API nui_status nui_server_stats(const nui_server* v, size_t* used, int* streams, int* queued) {
  if (!v) return fail(NUI_ERR_INVALID_ARG, "null server");
  int ns = 0, nq = 0;
  for (const auto& sl : v->slots)
    if (sl.s) {
      ++ns;
      nq += (int)sl.q.size();
    }
  if (used) *used = v->used;
  if (streams) *streams = ns;
  if (queued) *queued = nq;
  return NUI_OK;
}

NUI_API nui_session* nui_server_session(nui_server* v, int slot) {
  if (!v || slot < 0 || slot >= (int)v->slots.size()) return nullptr;
  return v->slots[slot].s;
}

}  // extern "C"
