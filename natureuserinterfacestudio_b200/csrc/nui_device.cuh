// Device-side types and helpers of the B200 KinectFusion path.
//
// The whole library is compiled with --fmad=false: every a*b+c in these kernels is a
// rounded multiply followed by a rounded add, in the order written, which is what makes
// the float results bit-identical to the CPU restatement of the reference kernels.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace nui {

constexpr int kMaxLevels = 4;
constexpr int kMaxRadius = 7;
constexpr int kIcpTerms = 29;  // 21 JtJ + 6 Jtr + r^2 + count  (icp.cl:122-160)
constexpr int kTile = 16;      // pixel tile of the depth bound used by integration culling
constexpr int kPreBlockX = 32, kPreBlockY = 8;  // k_preprocess block: 32 x 16 pixels, two a thread
constexpr int kFastWarps = 4;  // warps per block of the tolerance-mode integration
constexpr int kFastWarpSmem = 64 * 32 * 4 + 64 * 32 * 4;  // its shared memory per warp (bytes)

// Camera intrinsics block (gpu_def.h:13-27).
struct DevCam {
  float fx, fy, fx_inv, fy_inv, cx, cy;
  int W, H;
  float dmin, dmax;
};

// Rigid transform block (gpu_def.h:29-34): camera -> world rotation (row-major), its
// inverse, camera centre.
struct DevXform {
  float R[9], R_inv[9], t[3];
};

// Per-session tracking state, resident in device memory and updated by the kernels.
struct TrackState {
  DevXform xf;           // camera pose of the current frame (prev frame's during ICP)
  float R[9], t[3];      // ICP running estimate (Rcurr, tcurr)
  float Rg[9], tg[3];    // last accepted estimate of the level (Rgood, tgood)
  double good[27];       // accepted J^T J / J^T r sums
  float lambda, err_old; // Levenberg-Marquardt state of the level
  float error, count;    // NuiKinfuTracker::getError / getCount
  int level_done;        // the level's iteration loop has stopped early
  int status;            // 0 ok, 3 tracking lost
  int integrate;         // integration gate of this frame
  int iterations_run;
  float lastR[9], lastT[3];  // pose of the last integration (global translation: local +
                             // volume offset, NuiCameraPos.h:43)
  int dmax_bits;         // largest ray-length depth of the frame (float bits, >= 0)
  unsigned long long touched;
  // shifting volume: voxel offset of the volume (m_voxel_offset), this frame's shift in
  // voxels per axis (0: none), points found in the slabs that left the volume
  int voff[3];
  int shift[3];
  unsigned long long points;
  // work of the current frame counted by the kernels (the algorithmic bytes of a launch
  // follow from these): tolerance-mode raycast voxel reads, samples visited and refined
  // crossings; bricks re-classified by the tolerance-mode integration; ICP iterations run
  // per level
  unsigned long long ray_reads, ray_samples, ray_hits, bricks;
  unsigned long long tiles;  // 32 x 8 x 8 tiles the tolerance-mode integration ran
  unsigned int icp_iters[kMaxLevels];
  // tolerance-mode integration: tiles listed by the cull; blocks of the integration done
  // (both zero between integrations)
  unsigned int fast_count, fast_done;
};

// What one session does in the current tick (host-written, read by every kernel).
enum FrameKind : int { kInactive = -1, kFirstFrame = 0, kTrackFrame = 1 };

// hcount slots read by the frame's status check (k_hash_health)
constexpr int kHashFailed = 3, kHashChainFaults = 9, kHashFailedBefore = 10;

struct SessionDesc {
  int kind;  // FrameKind
  int slot;  // the session's row of the batch outputs (pose, status)
  int W, H, levels;
  DevCam cam;
  // preprocessing (NuiTrackerConfig)
  int radius;
  float sigma_depth, depth_thr;
  float gauss[2 * kMaxRadius + 1];
  // tracking
  float dist_thr;
  int iters[kMaxLevels];
  unsigned int icp_min_count[kMaxLevels];
  float integ_thr;
  // frame buffers
  const uint16_t* raw;
  const uint8_t* bgra;
  float* dscaled;                 // pass-filtered depth * ray scale (integration input)
  float* dlev[kMaxLevels];        // depth pyramid (level 0 = bilateral output)
  float4* vlev[kMaxLevels];       // camera-space vertex pyramid of the kernel-level calls (null in sessions)
  float4* vref;                   // world-space reference vertex map (W x H)
  float4* nref;                   // world-space reference normal map
  uchar4* cmap;                   // reference colour map (nullable)
  float* tile_max;                // per 16x16 pixel tile: largest ray-length depth (0 = none)
  // dense volume
  int fmt;                        // nui_tsdf_format
  int tol;                        // an FP16 serving format: the tolerance-mode kernels apply
  int res[3];
  float dim[3], cell[3], trunc;
  void* vol;                      // format storage, x-fastest: x + rx*(y + ry*z)
  uint8_t* wvol;                  // weight plane of NUI_TSDF_F16_U8
  uchar4* cvol;                   // colour volume (nullable), same layout
  uint8_t* occ;                   // per 8^3 brick state (kBrick*)
  uint8_t* occ2;                  // per 32^3 super-brick state (kSuper*)
  uint8_t* occ3;                  // per 128^3 region state (kSuper*, over its super-bricks)
  int max_cw;
  int zchunks;                    // integration: z chunks per column (one thread each)
  unsigned* fast_tiles;           // tolerance-mode integration: 32 x 8 x 8 tiles kept by the cull (list)
  float* ztab;                    // integration: running sums shared by all columns, 2 (rz + 1)
  // shifting volume (0: fixed): shift distance in voxels, basis translation, and the point
  // cache of the slabs that leave the volume (pts_cap points of xyz / rgba floats)
  int voxel_shift;
  float shift_basis[3];
  float* pts_xyz;
  float* pts_rgba;
  long long pts_cap;
  // colour tracking: weight of the photometric term (0: depth only); the previous frame's
  // colours (the model colours of the reference maps); the frame's colour pyramid (level 0
  // is bgra) and its x / y gradients per level (signed bytes)
  float photo_w;
  uchar4* cprev;
  uchar4* cpyr[kMaxLevels];
  uchar4* cgx[kMaxLevels];
  uchar4* cgy[kMaxLevels];
  // tracking state and ICP scratch
  TrackState* ts;
  // voxel-block hash (volume_kind == hash; fmt is then -1 so the dense kernels skip)
  int hash;                       // 1 for a hash session
  int hfmt;                       // 0: int16 sdf (reference), 1: half sdf
  struct HEntry* entries;         // buckets + excess entries
  int nb, ne, np;                 // buckets, excess list length, pool blocks
  unsigned int hmask;
  float voxel, mu;                // virtualVoxelSize, truncScale
  int max_w;                      // integrationWeightMax
  void* hsdf;                     // np * 512 sdf (int16 or half)
  uint8_t* hw;                    // np * 512 weights
  uchar4* hrgb;                   // np * 512 colours (nullable)
  int* alloc_list;                // free-block stack
  int* excess_list;               // free excess-slot stack
  int* hcount;                    // [0] last free block, [1] last free excess, [2] visible count, [3] failed
                                  // allocations, [4] swap-in count, [5] swap-out count, [6] free-list base
                                  // of the swap pass, [7] store blocks used, [8] store-full refusals,
                                  // [9] corrupted excess chains met this frame, [10] failed
                                  // allocations before this frame, [11] pixels the forward
                                  // render casts
  // forward rendering of the reference maps (0 off, 1 the reference's projection, 2 world to
  // camera): per pixel the last source pixel landing on it (+1), the missing pixels listed in
  // increasing order, per-1024-pixel-block counts then offsets, landed colours
  int fwd;
  int* fwd_owner;
  int* fwd_ids;
  unsigned* fwd_blk;
  uchar4* fwd_col;
  // global cache (hash swapping): per-entry swap state and store slot, the transfer lists,
  // and the host store (pinned, mapped: kernels read and write it directly)
  int swapping;
  uint8_t* swap;
  int* store_slot;
  int* swap_in_ids;               // kTransferBlocks
  int* swap_out_ids;              // kTransferBlocks
  void* st_sdf;                   // st_cap * 512 (int16 or half)
  uint8_t* st_w;                  // st_cap * 512
  uchar4* st_rgb;                 // st_cap * 512 (nullable)
  int st_cap;
  uint8_t* alloc_type;            // per entry
  uint8_t* vis;                   // per entry visible type
  short4* coords;                 // per entry block coordinates of a pending allocation
  unsigned long long* keys;       // per entry: last writer key of a pending allocation
  int* vis_ids;                   // visible list
  unsigned int* blk;              // scan scratch: per 1024 entries, 2 counts + 2 offsets
  float2* range;                  // expected range image
};

// Session families of a launch that covers the whole batch table: 0 every session, 1 the
// dense (non-hash) ones, 2 the voxel-hash ones.
constexpr int kFamAll = 0, kFamDense = 1, kFamHash = 2;
__device__ __forceinline__ bool in_family(const SessionDesc& s, int fam) {
  return fam == kFamAll || (fam == kFamHash) == (s.hash != 0);
}

// Hash entry (NuiKinfuHashEntry, hashing_gpu_def.h:49-63): 16 bytes.
struct __align__(16) HEntry {
  short pos[3];
  short pad;
  int ptr;
  unsigned int offset;
};

// ------------------------------------------------------------------ float helpers
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 mul3(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ bool isnan3(float3 v) { return isnan(v.x) || isnan(v.y) || isnan(v.z); }
// OpenCL normalize()/fast_normalize(): v / |v|, a zero vector is returned unchanged
__device__ __forceinline__ float3 normalize3(float3 v) {
  if (v.x == 0.f && v.y == 0.f && v.z == 0.f) return v;
  float l = sqrtf(dot3(v, v));
  return f3(v.x / l, v.y / l, v.z / l);
}
__device__ __forceinline__ float3 xyz(float4 v) { return f3(v.x, v.y, v.z); }
__device__ __forceinline__ float4 w0(float3 v) { return make_float4(v.x, v.y, v.z, 0.f); }
__device__ __forceinline__ float3 rot_rows(const float* M, float3 v) {
  return f3(dot3(f3(M[0], M[1], M[2]), v), dot3(f3(M[3], M[4], M[5]), v), dot3(f3(M[6], M[7], M[8]), v));
}
__device__ __forceinline__ float qnan() { return __int_as_float(0x7fc00000); }

// Camera-space vertex of pixel (x, y) of pyramid level `level` at depth d
// (depth2vertex_kernel, transformMaps.cl:18-42, with the level's intrinsics cx / 2^l and
// 2^l / fx as the reference's pyramid passes them); NaN where d is.  At level 0 the
// products are the full-resolution ones (2^0 / fx and cx / 2^0 are exact), so every
// consumer that rebuilds a vertex from the depth pyramid gets the bits the stored map had.
__device__ __forceinline__ float3 level_vertex(const DevCam& c, int level, int x, int y, float d) {
  const float div = (float)(1 << level);
  const float fxi = div * c.fx_inv, fyi = div * c.fy_inv, cxl = c.cx / div, cyl = c.cy / div;
  if (isnan(d)) return f3(qnan(), qnan(), qnan());
  return f3(d * (((float)x - cxl) * fxi), d * (((float)y - cyl) * fyi), d * 1.0f);
}

// exp() of the bilateral filter.  Method: x = k ln2 + r with a two-constant Cody-Waite
// split of ln2, exp(r) by Horner evaluation of the degree-7 Taylor polynomial
// (|r| <= ln2/2, truncation error < 1e-8 relative), scaled by 2^k in two exact steps.  The
// reduction and the polynomial use fused multiply-adds (explicit: the build turns automatic
// contraction off), which halves their instructions.  The CPU oracle implements the same
// method with the same fused operations, so both round identically.
__device__ __forceinline__ float nui_expf(float x) {
  if (isnan(x)) return x;
  if (x > 88.5f) return __int_as_float(0x7f800000);
  if (x < -103.5f) return 0.f;
  const float kf = rintf(x * 1.44269504088896341f);
  float r = __fmaf_rn(-kf, 0.693145751953125f, x);
  r = __fmaf_rn(-kf, 1.42860682030941723e-6f, r);
  float p = 1.98412698412698413e-4f;
  p = __fmaf_rn(p, r, 1.38888888888888889e-3f);
  p = __fmaf_rn(p, r, 8.33333333333333333e-3f);
  p = __fmaf_rn(p, r, 4.16666666666666667e-2f);
  p = __fmaf_rn(p, r, 1.66666666666666667e-1f);
  p = __fmaf_rn(p, r, 0.5f);
  p = __fmaf_rn(p, r, 1.0f);
  p = __fmaf_rn(p, r, 1.0f);
  int k = (int)kf;
  int k1 = k / 2, k2 = k - k1;
  float s1 = __int_as_float((k1 + 127) << 23), s2 = __int_as_float((k2 + 127) << 23);
  return (p * s1) * s2;
}

// nui_expf for -87 <= x <= 0, the range of every bilateral tap when the depth threshold
// and sigma keep thr^2 * sigma <= 87: no NaN, overflow or underflow tests, and one scale by
// 2^k, which is normal there (k >= -126).  The result is nui_expf's: p * 2^k1 is exact, so
// nui_expf's (p * 2^k1) * 2^k2 rounds the exact product p * 2^k once, as p * 2^k does.
__device__ __forceinline__ float nui_expf_neg(float x) {
  const float kf = rintf(x * 1.44269504088896341f);
  float r = __fmaf_rn(-kf, 0.693145751953125f, x);
  r = __fmaf_rn(-kf, 1.42860682030941723e-6f, r);
  float p = 1.98412698412698413e-4f;
  p = __fmaf_rn(p, r, 1.38888888888888889e-3f);
  p = __fmaf_rn(p, r, 8.33333333333333333e-3f);
  p = __fmaf_rn(p, r, 4.16666666666666667e-2f);
  p = __fmaf_rn(p, r, 1.66666666666666667e-1f);
  p = __fmaf_rn(p, r, 0.5f);
  p = __fmaf_rn(p, r, 1.0f);
  p = __fmaf_rn(p, r, 1.0f);
  return p * __int_as_float(((int)kf + 127) << 23);
}

// ------------------------------------------------------------------ voxel formats
// Each format exposes read(idx, F, W) -> true if W > 0, and write(idx, F, W).
template <int FMT>
struct Voxel;

template <>
struct Voxel<0> {  // NUI_TSDF_I16: short2, F = tsdf * 32766 truncated (utils.cl:69-79)
  static constexpr int kBytes = 4;
  __device__ static __forceinline__ void load(const SessionDesc& s, size_t i, float& F, int& W) {
    short2 v = reinterpret_cast<const short2*>(s.vol)[i];
    F = (float)v.x / 32766.f;
    W = v.y;
  }
  __device__ static __forceinline__ void store(const SessionDesc& s, size_t i, float F, int W) {
    reinterpret_cast<short2*>(s.vol)[i] = make_short2((short)__float2int_rz(F * 32766.f), (short)W);
  }
  __device__ static __forceinline__ void init(const SessionDesc& s, size_t i) {
    reinterpret_cast<short2*>(s.vol)[i] = make_short2(32767, 0);
  }
};
template <>
struct Voxel<1> {  // NUI_TSDF_F32: float2 (tsdf, weight)
  static constexpr int kBytes = 8;
  __device__ static __forceinline__ void load(const SessionDesc& s, size_t i, float& F, int& W) {
    float2 v = reinterpret_cast<const float2*>(s.vol)[i];
    F = v.x;
    W = (int)v.y;
  }
  __device__ static __forceinline__ void store(const SessionDesc& s, size_t i, float F, int W) {
    reinterpret_cast<float2*>(s.vol)[i] = make_float2(F, (float)W);
  }
  __device__ static __forceinline__ void init(const SessionDesc& s, size_t i) {
    reinterpret_cast<float2*>(s.vol)[i] = make_float2(1.f, 0.f);
  }
};
template <>
struct Voxel<2> {  // NUI_TSDF_F16_U8: half tsdf plane + uint8 weight plane
  static constexpr int kBytes = 3;
  __device__ static __forceinline__ void load(const SessionDesc& s, size_t i, float& F, int& W) {
    F = __half2float(reinterpret_cast<const __half*>(s.vol)[i]);
    W = s.wvol[i];
  }
  __device__ static __forceinline__ void store(const SessionDesc& s, size_t i, float F, int W) {
    reinterpret_cast<__half*>(s.vol)[i] = __float2half_rn(F);
    s.wvol[i] = (uint8_t)W;
  }
  __device__ static __forceinline__ void init(const SessionDesc& s, size_t i) {
    reinterpret_cast<__half*>(s.vol)[i] = __float2half_rn(1.f);
    s.wvol[i] = 0;
  }
};
template <>
struct Voxel<3> {  // NUI_TSDF_F16_F16: half2 (tsdf, weight)
  static constexpr int kBytes = 4;
  __device__ static __forceinline__ void load(const SessionDesc& s, size_t i, float& F, int& W) {
    __half2 v = reinterpret_cast<const __half2*>(s.vol)[i];
    F = __low2float(v);
    W = (int)__high2float(v);
  }
  __device__ static __forceinline__ void store(const SessionDesc& s, size_t i, float F, int W) {
    reinterpret_cast<__half2*>(s.vol)[i] = __floats2half2_rn(F, (float)W);
  }
  __device__ static __forceinline__ void init(const SessionDesc& s, size_t i) {
    reinterpret_cast<__half2*>(s.vol)[i] = __floats2half2_rn(1.f, 0.f);
  }
};

// The reference's voxelWrap component of a shifting volume at voxel offset `off` on an
// axis of r voxels (getVoxelWrap, NuiKinfuOpenCLShiftScene.cpp:44-56): voxel x of the
// volume sits at (x + wrap) % r of the reference's buffer.
__device__ __forceinline__ int ref_wrap(int off, int r) { return off >= 0 ? off : r - ((-off) % r); }

__device__ __forceinline__ size_t vox_index(const SessionDesc& s, int x, int y, int z) {
  return (size_t)x + (size_t)s.res[0] * ((size_t)y + (size_t)s.res[1] * (size_t)z);
}
// Brick states of 8^3 voxels (the voxels of a brick inside the volume).  Weights never
// decrease between resets, so an empty brick holds only weight-0 voxels; a positive brick
// has every voxel weighted with tsdf > 0; a no-negative brick mixes weight-0 voxels with
// weighted ones of tsdf > 0; a mixed brick has a weighted voxel with tsdf <= 0.
// Integration marks the bricks it touches dirty and k_brick_summary re-classifies them.
enum BrickState : uint8_t {
  kBrickEmpty = 0,
  kBrickMixed = 1,
  kBrickPositive = 2,
  kBrickDirty = 3,
  kBrickNoNeg = 4
};
// States of 32^3-voxel super-bricks (4^3 bricks): all bricks empty; some brick mixed or
// dirty; every brick empty, positive or no-negative (a march can cross it without a sign
// change); or awaiting re-classification.  128^3-voxel regions (4^3 super-bricks) use the
// same states over their super-bricks.
enum SuperState : uint8_t { kSuperEmpty = 0, kSuperMixed = 1, kSuperSkip = 2, kSuperDirty = 3 };
__device__ __forceinline__ size_t occ_index(const SessionDesc& s, int x, int y, int z) {
  const size_t bx = (size_t)(s.res[0] + 7) >> 3, by = (size_t)(s.res[1] + 7) >> 3;
  return (size_t)(x >> 3) + bx * ((size_t)(y >> 3) + by * (size_t)(z >> 3));
}
__device__ __forceinline__ size_t occ2_index(const SessionDesc& s, int x, int y, int z) {
  const size_t sx = (size_t)(s.res[0] + 31) >> 5, sy = (size_t)(s.res[1] + 31) >> 5;
  return (size_t)(x >> 5) + sx * ((size_t)(y >> 5) + sy * (size_t)(z >> 5));
}
// round(p / c) for a voxel coordinate, exactly as the IEEE quotient would round: the
// product with 1/c is within 2 ulp of the quotient, so unless it lies within 4 ulp of a
// rounding boundary (n + 0.5) both round alike; otherwise divide.  The nearest integer of
// the product comes from the 1.5 * 2^23 shift (adds and an integer subtract, no rounding
// or conversion instruction; exact for |q| < 2^22, and from |q| > 2^20 on every product
// lies within the boundary margin anyway).  Its distance |q - n| to the product is
// min(f, 1 - f) for the fraction f = q - floor(q), so the boundary test is unchanged, and
// away from a boundary round-to-nearest-even and round-half-away agree.
// Tolerance-mode rounding to the nearest integer: floor(q + 0.5).  At exact ties it rounds
// up, which is OpenCL's round() (half away from zero) for every q > -0.5; it differs from
// round() only within one ulp below a tie (where q + 0.5 itself rounds up) and at q = -0.5,
// both near ties that the tolerance admits.  Two instructions, no branch.
__device__ __forceinline__ int round_half_up(float q) { return __float2int_rd(q + 0.5f); }

__device__ __forceinline__ int round_div(float p, float c, float inv) {
  const float q = p * inv;
  const float big = 12582912.f;  // 1.5 * 2^23
  const float sh = q + big;
  const float f = q - (sh - big);  // q - n, exact
  if (fabsf(q) < 4194304.f && fabsf(fabsf(f) - 0.5f) > fabsf(q) * 4.8e-7f + 1e-6f)
    return __float_as_int(sh) - 0x4B400000;
  return (int)roundf(p / c);
}

}  // namespace nui
