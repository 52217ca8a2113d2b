// Frame preprocessing kernels.
//
//  k_preprocess   depth_passing_filter_kernel (filters.cl:9-23) + bilateral_filter_depth_kernel
//                 (bilateralFilter.cl:68-119) + depth2vertex_kernel at level 0
//                 (transformMaps.cl:18-42) + scaleDepthsKernel (tsdfVolume.cl:8-29), fused.
//                 One block per 32x16 output tile, two vertically adjacent pixels a thread;
//                 the pass-filtered depth of the tile and its radius-r halo is staged in
//                 shared memory once.
//                 Also writes the largest ray-length depth of each 16x16 tile (integration
//                 uses it to skip voxels that are behind every surface they can project to).
//  k_pyramid      half_sample_kernel (transformMaps.cl:44-88) + depth2vertex_kernel for one
//                 pyramid level.
//  k_feedback     estimate_normals_simple_kernel (normalEstimation.cl:770-822) +
//                 transform_maps_kernel (transformMaps.cl:91-127): frame-0 reference maps.
//
// Out-of-image taps are staged as NaN; the reference clamps its loops to the image
// instead, and since NaN taps are skipped the accumulated sequence is the same.
#include "nui_device.cuh"

namespace nui {

constexpr int kPreTX = kPreBlockX, kPreTY = 2 * kPreBlockY;
constexpr int kPreSW = kPreTX + 2 * kMaxRadius, kPreSH = kPreTY + 2 * kMaxRadius, kGW = 2 * kMaxRadius + 1;

// The bilateral sum of one pixel: taps in row-major window order, each weighted by its
// spatial weight times exp(-diff^2 sigma) when it is positive and within the depth
// threshold of the centre c (NaN taps fail both tests).  t points at the window's corner
// in the staged tile, g at the spatial weights.  KR > 0 unrolls a window of that radius;
// FAST takes nui_expf_neg, valid when thr^2 sigma <= 87.
template <int KR, bool FAST>
__device__ __forceinline__ float bilateral_px(const float* t, const float* g, int R, float c, float thr, float sig) {
  if (KR > 0) R = KR;
  float sd = 0.f, swt = 0.f;
#pragma unroll
  for (int dy = 0; dy <= 2 * R; ++dy) {
#pragma unroll
    for (int dx = 0; dx <= 2 * R; ++dx) {
      const float nr = t[dy * kPreSW + dx];
      const float diff = fabsf(c - nr);
      if (nr > 0.0f && diff < thr) {
        const float d2 = diff * diff;
        const float e = FAST ? nui_expf_neg(-(d2 * sig)) : nui_expf(-(d2 * sig));
        const float w = g[dy * kGW + dx] * e;
        sd += nr * w;
        swt += w;
      }
    }
  }
  return sd / swt;
}

// Tolerance mode (sessions in an FP16 serving format), radius 3: the same taps for two
// vertically adjacent pixels (centres c0, c1; t points at pixel 0's window corner, pixel 1's
// window starts one row lower), the eight staged rows read once for both.  A tap's weight
// g exp(-diff^2 sigma) is taken as one hardware base-2 exponential of
// log2(g) + diff^2 (-sigma log2(e)) (lg: log2 of the spatial weights, nk = -sigma log2(e)),
// with fused multiply-adds; the filtered depth differs from the reference's by a few ulps
// of the weights.
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ void bilateral_px2_tol(const float* t, const float* lg, float c0, float c1, float thr,
                                                  float nk, float& out0, float& out1) {
  constexpr int R = 3, G = 2 * R + 1;
  float sd0 = 0.f, sw0 = 0.f, sd1 = 0.f, sw1 = 0.f;
#pragma unroll
  for (int r = 0; r <= G; ++r) {
#pragma unroll
    for (int dx = 0; dx < G; ++dx) {
      const float nr = t[r * kPreSW + dx];
      if (r < G) {
        const float diff = c0 - nr;
        if (nr > 0.0f && fabsf(diff) < thr) {
          const float w = ex2_approx(__fmaf_rn(diff * diff, nk, lg[r * kGW + dx]));
          sd0 = __fmaf_rn(nr, w, sd0);
          sw0 += w;
        }
      }
      if (r > 0) {
        const float diff = c1 - nr;
        if (nr > 0.0f && fabsf(diff) < thr) {
          const float w = ex2_approx(__fmaf_rn(diff * diff, nk, lg[(r - 1) * kGW + dx]));
          sd1 = __fmaf_rn(nr, w, sd1);
          sw1 += w;
        }
      }
    }
  }
  out0 = __fdividef(sd0, sw0);
  out1 = __fdividef(sd1, sw1);
}

__global__ void __launch_bounds__(kPreBlockX* kPreBlockY, 4) k_preprocess(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind < 0) return;
  const int W = s.W, H = s.H, R = s.radius;
  const int tilesX = (W + kPreTX - 1) / kPreTX;
  const int tx0 = (blockIdx.x % tilesX) * kPreTX, ty0 = (blockIdx.x / tilesX) * kPreTY;
  if (ty0 >= H) return;
  __shared__ float tile[kPreSH][kPreSW];
  // spatial weights g[dx] * g[dy] of the taps (the products the tap loop would form), and
  // their base-2 logarithms for the tolerance-mode weights
  __shared__ float gw[kGW][kGW], lgw[kGW][kGW];
  const int tid = threadIdx.y * kPreBlockX + threadIdx.x;
  if (tid < (2 * R + 1) * (2 * R + 1)) {
    const int ty = tid / (2 * R + 1), tx = tid % (2 * R + 1);
    const float g = s.gauss[tx] * s.gauss[ty];
    gw[ty][tx] = g;
    lgw[ty][tx] = log2f(g);
  }
  const float dmin = s.cam.dmin, dmax = s.cam.dmax;
  const int sw = kPreTX + 2 * R, sh = kPreTY + 2 * R;
  for (int i = tid; i < sw * sh; i += kPreBlockX * kPreBlockY) {
    int ly = i / sw, lx = i - ly * sw;
    int gx = tx0 - R + lx, gy = ty0 - R + ly;
    float d = qnan();
    if (gx >= 0 && gy >= 0 && gx < W && gy < H) {
      float dp = (float)s.raw[(size_t)gy * W + gx] * 0.001f;
      if (dp > dmin && dp < dmax) d = dp;
    }
    tile[ly][lx] = d;
  }
  __syncthreads();
  const int ly0 = 2 * threadIdx.y;  // this thread's rows of the tile: ly0, ly0 + 1
  const int x = tx0 + threadIdx.x;
  float cs[2], outs[2];
  for (int k = 0; k < 2; ++k) {
    cs[k] = tile[ly0 + k + R][threadIdx.x + R];
    outs[k] = qnan();
  }
  const float thr = s.depth_thr, sig = s.sigma_depth;
  if (s.tol && R == 3) {
    if (!isnan(cs[0]) || !isnan(cs[1])) {
      bilateral_px2_tol(&tile[ly0][threadIdx.x], &lgw[0][0], cs[0], cs[1], thr, -sig * 1.44269504088896341f,
                        outs[0], outs[1]);
      for (int k = 0; k < 2; ++k)
        if (isnan(cs[k])) outs[k] = qnan();
    }
  } else {
    // every tap's exponent lies in [-thr^2 sigma, 0] (rounding is monotone)
    const bool fast = sig >= 0.f && thr * thr * sig <= 87.f;
    for (int k = 0; k < 2; ++k) {
      if (isnan(cs[k])) continue;
      const float* t = &tile[ly0 + k][threadIdx.x];
      if (fast && R == 3) outs[k] = bilateral_px<3, true>(t, &gw[0][0], R, cs[k], thr, sig);
      else if (fast) outs[k] = bilateral_px<0, true>(t, &gw[0][0], R, cs[k], thr, sig);
      else outs[k] = bilateral_px<0, false>(t, &gw[0][0], R, cs[k], thr, sig);
    }
  }
  float m = 0.f;  // largest ray-length depth of this thread's two pixels
  for (int k = 0; k < 2; ++k) {
    const int y = ty0 + ly0 + k;
    if (x >= W || y >= H) continue;
    const float c = cs[k], out = outs[k];
    const size_t i = (size_t)y * W + x;
    s.dlev[0][i] = out;
    const float xl = ((float)x - s.cam.cx) * s.cam.fx_inv;
    const float yl = ((float)y - s.cam.cy) * s.cam.fy_inv;
    if (s.vlev[0]) {  // the kernel-level call's vertex map (sessions rebuild vertices from depth)
      float4 v = make_float4(qnan(), qnan(), qnan(), 0.f);
      if (!isnan(out)) v = make_float4(out * xl, out * yl, out * 1.0f, 0.f);
      s.vlev[0][i] = v;
    }
    // ray-length depth for integration: the pass-filtered depth, not the bilateral output
    // (NuiKinfuOpenCLScene.cpp:218 passes GetDepthBuffer())
    float sc = c;
    if (!isnan(c)) sc = c * sqrtf(xl * xl + yl * yl + 1.f);
    s.dscaled[i] = sc;
    if (!isnan(sc)) m = fmaxf(m, sc);
  }
  // largest ray-length depth of each 16x16 tile (lanes 0-15 / 16-31 of a row are two
  // tiles) and of the frame: the bounds integration culls with
  for (int off = 8; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
  __shared__ float rowmax[kPreBlockY][2];
  if ((threadIdx.x & 15) == 0) rowmax[threadIdx.y][threadIdx.x >> 4] = m;
  __syncthreads();
  if (threadIdx.y == 0 && threadIdx.x < 2) {
    float t = 0.f;
    for (int r = 0; r < kPreBlockY; ++r) t = fmaxf(t, rowmax[r][threadIdx.x]);
    const int tcol = tx0 / kTile + threadIdx.x, trow = ty0 / kTile;
    const int ntx = (W + kTile - 1) / kTile;
    if (s.tile_max && tcol < ntx) s.tile_max[trow * ntx + tcol] = t;
    if (t > 0.f && s.ts) atomicMax(&s.ts->dmax_bits, __float_as_int(t));
  }
}

// One pyramid level: dst(x,y) = mean of the 3x3 taps around src(2x,2y) within the depth
// threshold of the centre (any valid tap if the centre is NaN); vertices with div = 2^l.
__global__ void k_pyramid(const SessionDesc* __restrict__ descs, int level) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind != kTrackFrame || level >= s.levels) return;
  const int dW = s.W >> level, dH = s.H >> level, sW = dW * 2, sH = dH * 2;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= dW * dH) return;
  const int x = idx % dW, y = idx / dW;
  const float* src = s.dlev[level - 1];
  const int sx = 2 * x, sy = 2 * y;
  const float c = src[(size_t)sy * sW + sx];
  const float thr = s.depth_thr;
  float sum = 0.f;
  int n = 0;
  for (int cy = max(sy - 1, 0); cy < min(sy + 2, sH); ++cy)
    for (int cx = max(sx - 1, 0); cx < min(sx + 2, sW); ++cx) {
      float nr = src[(size_t)cy * sW + cx];
      if (!isnan(nr) && (isnan(c) || fabsf(c - nr) < thr)) {
        sum += nr;
        n += 1;
      }
    }
  const float d = n > 0 ? sum / (float)n : qnan();
  s.dlev[level][idx] = d;
  if (s.vlev[level]) s.vlev[level][idx] = w0(level_vertex(s.cam, level, x, y, d));
}

// A level's vertex map from its depth, for downloads (sessions keep no vertex maps).
__global__ void k_vertex_map(const SessionDesc* __restrict__ descs, int level, float4* __restrict__ out) {
  const SessionDesc& s = descs[blockIdx.y];
  const int W = s.W >> level, H = s.H >> level;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= W * H) return;
  out[idx] = w0(level_vertex(s.cam, level, idx % W, idx / W, s.dlev[level][idx]));
}

// Frame-0 reference maps: simple normals from the level-0 vertex map, then both maps to
// world space with the current pose (NuiKinfuOpenCLFeedbackFrame::UpdateBuffers, :71-91).
__global__ void k_feedback(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind != kFirstFrame) return;
  const int W = s.W, H = s.H;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= W * H) return;
  const int x = idx % W, y = idx / W;
  // the level-0 vertices: the kernel-level call's map, else rebuilt from the depth
  const float4* V = s.vlev[0];
  auto vtx = [&](int j, int jx, int jy) {
    return V ? xyz(V[j]) : level_vertex(s.cam, 0, jx, jy, s.dlev[0][j]);
  };
  const float3 c = vtx(idx, x, y);
  const DevXform& m = s.ts->xf;
  if (isnan3(c)) {
    s.vref[idx] = make_float4(qnan(), qnan(), qnan(), 0.f);
    s.nref[idx] = make_float4(qnan(), qnan(), qnan(), 0.f);
    return;
  }
  const float thr = s.depth_thr;
  auto pick = [&](bool ok, int j, int jx, int jy) {
    if (!ok) return c;
    float3 q = vtx(j, jx, jy);
    if (isnan3(q) || fabsf(c.z - q.z) > thr) return c;
    return q;
  };
  const float3 l = pick(x > 0, idx - 1, x - 1, y), r = pick(x < W - 1, idx + 1, x + 1, y);
  const float3 u = pick(y > 0, idx - W, x, y - 1), d = pick(y < H - 1, idx + W, x, y + 1);
  const float3 n = normalize3(cross3(sub3(r, l), sub3(d, u)));
  const float3 vw = add3(rot_rows(m.R, c), f3(m.t[0], m.t[1], m.t[2]));
  s.vref[idx] = w0(vw);
  s.nref[idx] = isnan3(n) ? make_float4(qnan(), qnan(), qnan(), 0.f) : w0(rot_rows(m.R, n));
  if (s.cmap) {  // model colours of the first frame: the frame's (R, G, B order in hash scenes)
    uchar4 cc = s.bgra ? reinterpret_cast<const uchar4*>(s.bgra)[idx] : make_uchar4(0, 0, 0, 0);
    if (s.hash) cc = make_uchar4(cc.z, cc.y, cc.x, cc.w);
    s.cmap[idx] = cc;
  }
}

}  // namespace nui
