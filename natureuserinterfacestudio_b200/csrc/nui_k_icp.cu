// Point-to-plane ICP: every iteration of every level in one launch, one thread-block
// cluster per session, no host round trip.
//
// Per pixel (icp_block_kernel, icp.cl:222-292): rebuild the level's vertex from its depth,
// transform it by the running estimate, project into the previous camera with
// full-resolution intrinsics, bilinearly sample the world reference normal and vertex
// (icp.cl:192-220; a tap NaN -> no match), and if |q - p| < distThres form the row
// [n x p, n | n.(q - p)].  Each thread accumulates the 29 products of its pixels in FP64
// (exact products of the FP32 row values, fused multiply-adds);
// blocks reduce them with warp shuffles and shared memory; the cluster's first block adds
// the blocks' sums (distributed shared memory, fixed order) and runs the host step of
// NuiKinfuOpenCLDepthTracker::IterativeClosestPoint (NuiKinfuOpenCLDepthTracker.cpp:324-496):
// Levenberg-Marquardt accept/reject, FP64 determinant check and Cholesky solve, ZYX Euler
// increment composed in FP64.  The next iteration reads the updated estimate.
#include <cooperative_groups.h>

#include "nui_device.cuh"

namespace nui {

constexpr int kIcpThreads = 256;  // pixels per thread: the template parameter PPT (tuned)

// Bilinear sample with holes; taps whose linear index falls past the map read as holes.
__device__ __forceinline__ float3 bilinear_holes(const float4* __restrict__ src, float px, float py, int W,
                                                 int N) {
  const int ix = (int)floorf(px), iy = (int)floorf(py);
  const float dx = px - (float)ix, dy = py - (float)iy;
  const int ia = ix + iy * W, ib = (ix + 1) + iy * W, ic = ix + (iy + 1) * W, id = (ix + 1) + (iy + 1) * W;
  if (id >= N || ic >= N || ib >= N) return f3(qnan(), qnan(), qnan());
  const float3 a = xyz(__ldg(src + ia)), b = xyz(__ldg(src + ib)), c = xyz(__ldg(src + ic)),
               d = xyz(__ldg(src + id));
  if (isnan3(a) || isnan3(b) || isnan3(c) || isnan3(d)) return f3(qnan(), qnan(), qnan());
  const float ex = 1.0f - dx, ey = 1.0f - dy;
  float3 r;
  r.x = a.x * ex * ey + b.x * dx * ey + c.x * ex * dy + d.x * dx * dy;
  r.y = a.y * ex * ey + b.y * dx * ey + c.y * ex * dy + d.y * dx * dy;
  r.z = a.z * ex * ey + b.z * dx * ey + c.z * ex * dy + d.z * dx * dy;
  return r;
}

// ---------------------------------------------------------------- photometric rows
// One model point of the colour tracker's term (color_icp_block_kernel, colorIcp.cl:
// 119-178, in the tracker's convention), at the finest level: the world point m of the
// previous raycast, whose colour is the previous frame's at the same pixel (the raycast
// is rendered from the previous pose), is taken to the current camera by the running
// estimate, p = R^T (m - t), projected and rounded to a pixel of the current colour
// image; the residual is the colour difference (units of 1/255) and its derivative in
// each ICP parameter x_k is  grad(I) . d(proj)/dp . dp/dx_k  with dp/dx_k = R^T (e_k x m)
// for the rotations and -R^T e_k for the translations (the depth ICP's update
// R <- Rinc^-1 R, t <- Rinc^-1 t + tinc).  Colours count with alpha 255.  c receives the
// upper triangle of [D | -diff]^T [D | -diff] by rows (21 + 6), |diff|^2 and 1.
__device__ __forceinline__ bool color_row(const SessionDesc& s, int i, const float* R, const float3 t, float* c) {
  const float3 m = xyz(__ldg(s.vref + i));
  if (isnan3(m)) return false;
  const uchar4 mc = __ldg(s.cprev + i);
  if (mc.w != 255) return false;
  const float3 d = sub3(m, t);
  const float3 c0 = f3(R[0], R[3], R[6]), c1 = f3(R[1], R[4], R[7]), c2 = f3(R[2], R[5], R[8]);
  const float3 p = f3(dot3(c0, d), dot3(c1, d), dot3(c2, d));
  const float fx = s.cam.fx, fy = s.cam.fy, cx = s.cam.cx, cy = s.cam.cy;
  const int lw = s.W, lh = s.H;
  const int u = (int)roundf(p.x * fx / p.z + cx), v = (int)roundf(p.y * fy / p.z + cy);
  if (!(u >= 0 && u < lw && v >= 0 && v < lh)) return false;
  const int li = v * lw + u;
  const uchar4 co = __ldg(reinterpret_cast<const uchar4*>(s.bgra) + li);
  const uchar4 gx = __ldg(s.cgx[0] + li), gy = __ldg(s.cgy[0] + li);
  if (co.w != 255 || gx.w != 255 || gy.w != 255) return false;
  const float k255 = 1.0f / 255.0f;
  const float3 diff = mul3(f3((float)co.x - (float)mc.x, (float)co.y - (float)mc.y, (float)co.z - (float)mc.z), k255);
  const float3 g1 = mul3(f3((float)(signed char)gx.x, (float)(signed char)gx.y, (float)(signed char)gx.z), k255);
  const float3 g2 = mul3(f3((float)(signed char)gy.x, (float)(signed char)gy.y, (float)(signed char)gy.z), k255);
  float3 D[6];
  const float zz = p.z * p.z;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const float3 w = k == 0 ? f3(0.f, -m.z, m.y)
                   : k == 1 ? f3(m.z, 0.f, -m.x)
                   : k == 2 ? f3(-m.y, m.x, 0.f)
                   : k == 3 ? f3(-1.f, 0.f, 0.f)
                   : k == 4 ? f3(0.f, -1.f, 0.f)
                            : f3(0.f, 0.f, -1.f);
    const float3 dp = f3(dot3(c0, w), dot3(c1, w), dot3(c2, w));
    const float jx = fx * ((p.z * dp.x - dp.z * p.x) / zz);
    const float jy = fy * ((p.z * dp.y - dp.z * p.y) / zz);
    D[k] = f3(jx * g1.x + jy * g2.x, jx * g1.y + jy * g2.y, jx * g1.z + jy * g2.z);
  }
  const float3 nd = f3(-diff.x, -diff.y, -diff.z);
  int sh = 0;
#pragma unroll
  for (int a = 0; a < 6; ++a) {
#pragma unroll
    for (int b = a; b < 6; ++b) c[sh++] = dot3(D[a], D[b]);
    c[sh++] = dot3(D[a], nd);
  }
  c[27] = dot3(diff, diff);
  c[28] = 1.0f;
  return true;
}

// ---------------------------------------------------------------- FP64 host step
// The 6x6 algebra of the host step runs on one thread at the end of every ICP launch, so
// its latency is the launch's tail: every loop below is unrolled with constant indices,
// which keeps the matrices in registers (no local-memory round trips).

// Determinant by Gaussian elimination with partial pivoting (the first row holding the
// largest |entry| of the column); destroys A.
__device__ __forceinline__ double det6(double (&A)[6][6]) {
  double det = 1.0;
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    int piv = c;
    double best = fabs(A[c][c]);
#pragma unroll
    for (int r = c + 1; r < 6; ++r) {
      const double v = fabs(A[r][c]);
      if (v > best) {
        best = v;
        piv = r;
      }
    }
    if (best == 0.0) return 0.0;
    if (piv != c) {
#pragma unroll
      for (int r = c + 1; r < 6; ++r)
        if (piv == r) {
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            const double t = A[c][k];
            A[c][k] = A[r][k];
            A[r][k] = t;
          }
        }
      det = -det;
    }
    det *= A[c][c];
#pragma unroll
    for (int r = c + 1; r < 6; ++r) {
      const double f = A[r][c] / A[c][c];
#pragma unroll
      for (int k = c; k < 6; ++k) A[r][k] -= f * A[c][k];
    }
  }
  return det;
}

// Cholesky factorisation A = L L^T and the two triangular solves; false if a pivot is not
// positive.
__device__ __forceinline__ bool llt_solve6(const double (&A)[6][6], const double (&b)[6], double (&x)[6]) {
  double L[6][6];
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    double s = A[j][j];
#pragma unroll
    for (int k = 0; k < j; ++k) s -= L[j][k] * L[j][k];
    if (!(s > 0.0)) return false;
    L[j][j] = sqrt(s);
#pragma unroll
    for (int i = j + 1; i < 6; ++i) {
      double t = A[i][j];
#pragma unroll
      for (int k = 0; k < j; ++k) t -= L[i][k] * L[j][k];
      L[i][j] = t / L[j][j];
    }
  }
  double y[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    double t = b[i];
#pragma unroll
    for (int k = 0; k < i; ++k) t -= L[i][k] * y[k];
    y[i] = t / L[i][i];
  }
#pragma unroll
  for (int i = 5; i >= 0; --i) {
    double t = y[i];
#pragma unroll
    for (int k = i + 1; k < 6; ++k) t -= L[k][i] * x[k];
    x[i] = t / L[i][i];
  }
  return true;
}

// Rz(g) Ry(b) Rx(a) (AngleAxis composition at NuiKinfuOpenCLDepthTracker.cpp:486), from
// the angles' sines and cosines
__device__ __forceinline__ void euler_zyx(double sa, double ca, double sb, double cb, double sg, double cg,
                                          double (&R)[9]) {
  const double Rz[9] = {cg, -sg, 0, sg, cg, 0, 0, 0, 1};
  const double Ry[9] = {cb, 0, sb, 0, 1, 0, -sb, 0, cb};
  const double Rx[9] = {1, 0, 0, 0, ca, -sa, 0, sa, ca};
  double T[9];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double s = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k) s += Rz[i * 3 + k] * Ry[k * 3 + j];
      T[i * 3 + j] = s;
    }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double s = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k) s += T[i * 3 + k] * Rx[k * 3 + j];
      R[i * 3 + j] = s;
    }
}

// The tracker state the host step reads and writes: kept in block 0's shared memory for
// the whole ICP kernel (so that the single thread's step makes no global-memory round
// trips), copied in at the start and back at the end.
struct IcpLm {
  float R[9], t[3], Rg[9], tg[3];
  double good[27];
  float lambda, err_old, error, count;
  int level_done, status, iterations_run;
  unsigned icp_iters[kMaxLevels];
};

// Copies the fields (d <- s); T, U: TrackState or IcpLm.
template <class T, class U>
__device__ __forceinline__ void lm_copy(T* d, const U* s) {
  for (int k = 0; k < 9; ++k) d->R[k] = s->R[k], d->Rg[k] = s->Rg[k];
  for (int k = 0; k < 3; ++k) d->t[k] = s->t[k], d->tg[k] = s->tg[k];
  for (int k = 0; k < 27; ++k) d->good[k] = s->good[k];
  d->lambda = s->lambda;
  d->err_old = s->err_old;
  d->error = s->error;
  d->count = s->count;
  d->level_done = s->level_done;
  d->status = s->status;
  d->iterations_run = s->iterations_run;
  for (int k = 0; k < kMaxLevels; ++k) d->icp_iters[k] = s->icp_iters[k];
}

// The LM step on the reduced sums (NuiKinfuOpenCLDepthTracker.cpp:324-496), spread over
// the threads of the cluster's first block in phases separated by block barriers: the
// bookkeeping on one thread, the 27 normalised sums on 27 threads, the Cholesky solve and
// the determinant on two threads of different warps at once, the increments' sines and
// cosines on three threads, the composition on one.  Every value comes from the same FP64
// operations in the same order as a one-thread step; only their latencies overlap (one
// thread took ~8 us per iteration, while the cluster's other blocks waited).  All threads
// of the block call it.
struct IcpStepScratch {
  double A[6][6], b[6], x[6], det, sc[6];
  float cnt;
  int go, solved;
};
__device__ __noinline__ void icp_host_step(IcpLm* ts, IcpStepScratch& w, const double* sums, int iter,
                                              unsigned min_count) {
  const int tid = threadIdx.x;
  if (tid == 0) {  // bookkeeping: error, LM accept / reject
    float err = (float)sums[27];
    const float cnt = (float)sums[28];
    err = (cnt > 0.f) ? sqrtf(err) / cnt : 3.402823466e+38f;
    ts->error = err;
    ts->count = cnt;
    ts->iterations_run += 1;
    w.cnt = cnt;
    w.go = 1;
    if (iter == 0) {  // level start: lambda = 1, Rgood = Rcurr, errorOld = 1e20
      ts->lambda = 1.0f;
      for (int i = 0; i < 9; ++i) ts->Rg[i] = ts->R[i];
      for (int i = 0; i < 3; ++i) ts->tg[i] = ts->t[i];
      ts->err_old = 1e20f;
      ts->level_done = 0;
    }
    if (cnt < (float)min_count || err > ts->err_old) {
      ts->lambda *= 10.0f;
      for (int i = 0; i < 9; ++i) ts->R[i] = ts->Rg[i];
      for (int i = 0; i < 3; ++i) ts->t[i] = ts->tg[i];
      if (iter == 0) {
        ts->level_done = 1;
        w.go = 0;
      }
    } else {
      ts->lambda /= 10.0f;
      for (int i = 0; i < 9; ++i) ts->Rg[i] = ts->R[i];
      for (int i = 0; i < 3; ++i) ts->tg[i] = ts->t[i];
      ts->err_old = err;
      for (int k = 0; k < 27; ++k) ts->good[k] = sums[k];
    }
  }
  __syncthreads();
  if (!w.go) return;
  if (tid < 27) {  // sum sh = (i, j) of the upper triangle of [J|r] by rows, over the count
    int i = 0, j = tid;
    while (j >= 7 - i) j -= 7 - i, ++i;
    j += i;
    double v = ts->good[tid] / (double)w.cnt;
    if (j == 6) {
      w.b[i] = v;
    } else {
      if (i == j) v *= (double)(1.0f + ts->lambda);
      w.A[i][j] = v;
      w.A[j][i] = v;
    }
  }
  __syncthreads();
  // a singular system (|det| < 1e-15 or NaN) or a failed factorisation loses tracking; the
  // determinant's elimination works on a copy
  if (tid == 0) {
    double A[6][6], b[6], x[6];
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      b[r] = w.b[r];
#pragma unroll
      for (int c = 0; c < 6; ++c) A[r][c] = w.A[r][c];
    }
    w.solved = llt_solve6(A, b, x) ? 1 : 0;
#pragma unroll
    for (int r = 0; r < 6; ++r) w.x[r] = x[r];
  } else if (tid == 32) {
    double A[6][6];
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
      for (int c = 0; c < 6; ++c) A[r][c] = w.A[r][c];
    w.det = det6(A);
  }
  __syncthreads();
  if (tid == 0) {
    if (!w.solved || !(fabs(w.det) >= 1e-15)) {
      ts->status = 3;
      w.go = 0;
    } else {
      const float al = (float)w.x[0], be = (float)w.x[1], ga = (float)w.x[2];
      if (al * al + be * be + ga * ga < 1e-6f) {
        ts->level_done = 1;
        w.go = 0;
      }
    }
  }
  __syncthreads();
  if (!w.go) return;
  if (tid < 3) {  // sin and cos of the increment's angles (alpha, beta, gamma)
    double sn, cs;
    sincos((double)(float)w.x[tid], &sn, &cs);
    w.sc[2 * tid] = sn;
    w.sc[2 * tid + 1] = cs;
  }
  __syncthreads();
  if (tid == 0) {
    double Ri[9];
    euler_zyx(w.sc[0], w.sc[1], w.sc[2], w.sc[3], w.sc[4], w.sc[5], Ri);
    float t0[3], R0[9];
#pragma unroll
    for (int i = 0; i < 3; ++i) t0[i] = ts->t[i];
#pragma unroll
    for (int i = 0; i < 9; ++i) R0[i] = ts->R[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double s = 0;
#pragma unroll
      for (int k = 0; k < 3; ++k) s += Ri[k * 3 + i] * (double)t0[k];
      ts->t[i] = (float)(s + (double)(float)w.x[3 + i]);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        double s = 0;
#pragma unroll
        for (int k = 0; k < 3; ++k) s += Ri[k * 3 + i] * (double)R0[k * 3 + j];
        ts->R[i * 3 + j] = (float)s;
      }
  }
}

// The 29 sums of the depth rows of one block of pixels (kIcpThreads x PPT consecutive
// pixels of the level, index `vb`), added to this thread's FP64 accumulators.  sR / tc: the
// running estimate; sp: the previous camera pose (the reference maps' frame).
template <int PPT>
__device__ __forceinline__ void icp_depth_rows(const SessionDesc& s, int level, int vb, const float* sR, float3 tc,
                                               const DevXform& sp, double (&acc)[kIcpTerms]) {
  const int w = s.W >> level, n = w * (s.H >> level);
  const float* __restrict__ Dl = s.dlev[level];
  const float fx = s.cam.fx, fy = s.cam.fy, cx = s.cam.cx, cy = s.cam.cy;
  const int RW = s.W, RN = s.W * s.H;
  const float fW = (float)s.W, fH = (float)s.H;
  const float3 tp = f3(sp.t[0], sp.t[1], sp.t[2]);
  const int base = vb * kIcpThreads * PPT;
  // the depths of all the thread's pixels in flight at once, consumed from the front
  float dq[PPT];
#pragma unroll
  for (int k = 0; k < PPT; ++k) {
    const int i = base + k * kIcpThreads + threadIdx.x;
    dq[k] = i < n ? __ldg(Dl + i) : qnan();
  }
#pragma unroll 1
  for (int k = 0; k < PPT; ++k) {
    const float dep = dq[0];
#pragma unroll
    for (int j = 0; j + 1 < PPT; ++j) dq[j] = dq[j + 1];
    if (isnan(dep)) continue;
    const int i = base + k * kIcpThreads + threadIdx.x;
    const int py = i / w;
    const float3 v = level_vertex(s.cam, level, i - py * w, py, dep);
    const float3 pv = add3(rot_rows(sR, v), tc);
    const float3 pp = rot_rows(sp.R_inv, sub3(pv, tp));
    const float u = pp.x * fx / pp.z + cx;
    const float vv = pp.y * fy / pp.z + cy;
    if (!(u >= 0.0f && u < fW && vv >= 0.0f && vv < fH)) continue;
    // both maps sampled at once (their eight loads in flight together), then tested
    const float3 rn = bilinear_holes(s.nref, u, vv, RW, RN);
    const float3 rv = bilinear_holes(s.vref, u, vv, RW, RN);
    if (isnan3(rn) || isnan3(rv)) continue;
    const float3 diff = sub3(rv, pv);
    const float dist = sqrtf(dot3(diff, diff));
    if (!(dist < s.dist_thr)) continue;
    const float3 r0 = cross3(rn, pv);
    // the row's seven FP32 values widened once; each product is exact in FP64 and enters
    // its sum with one rounding (fused multiply-add)
    const double c7[7] = {(double)r0.x, (double)r0.y, (double)r0.z, (double)rn.x, (double)rn.y, (double)rn.z,
                          (double)dot3(rn, diff)};
    int sh = 0;
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
      for (int b = a; b < 7; ++b, ++sh) acc[sh] = fma(c7[a], c7[b], acc[sh]);
    acc[27] = fma(c7[6], c7[6], acc[27]);
    acc[28] += 1.0;
  }
}

// The photometric rows of one block of full-resolution model points (colour tracking).
template <int PPT>
__device__ __forceinline__ void icp_color_rows(const SessionDesc& s, int vb, const float* sR, float3 tc,
                                               double (&acc)[kIcpTerms]) {
  const int cbase = vb * kIcpThreads * PPT, NM = s.W * s.H;
#pragma unroll 1
  for (int k = 0; k < PPT; ++k) {
    const int i = cbase + k * kIcpThreads + threadIdx.x;
    if (i >= NM) break;
    float c[kIcpTerms];
    if (!color_row(s, i, sR, tc, c)) continue;
#pragma unroll
    for (int q = 0; q < kIcpTerms - 1; ++q) acc[q] += (double)c[q];
    acc[28] += 1.0;
  }
}

// Block sum of the threads' accumulators (a reduce-scatter over the 32 lanes of a warp,
// terms padded to 32 -- at each of five steps a lane keeps half of its values, sends the
// other half to its partner and adds what it receives, so lane k ends with the warp's sum
// of term k after 31 exchanges instead of 29 x 5 -- then the warps in shared memory, in a
// fixed order).  Threads 0..28 receive term threadIdx.x; all threads must call it.
__device__ __forceinline__ double icp_block_sum(const double (&acc)[kIcpTerms]) {
  constexpr int kWarps = kIcpThreads / 32;
  __shared__ double wsum[kWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double v[32];
#pragma unroll
  for (int k = 0; k < 32; ++k) v[k] = k < kIcpTerms ? acc[k] : 0.0;
#pragma unroll
  for (int half = 16; half > 0; half >>= 1) {
    const bool upper = lane & half;
#pragma unroll
    for (int j = 0; j < half; ++j) {
      const double send = upper ? v[j] : v[j + half];
      const double keep = upper ? v[j + half] : v[j];
      v[j] = keep + __shfl_xor_sync(0xffffffffu, send, half);
    }
  }
  wsum[warp][lane] = v[0];
  __syncthreads();
  double D = 0.0;
  if (threadIdx.x < kIcpTerms)
    for (int wi = 0; wi < kWarps; ++wi) D += wsum[wi][threadIdx.x];
  __syncthreads();  // wsum is reused by the next call
  return D;
}

// All ICP iterations of every level of one frame, one thread-block cluster per session
// (NuiKinfuOpenCLDepthTracker::IterativeClosestPoint, NuiKinfuOpenCLDepthTracker.cpp:240-504).
// The C blocks of a cluster (C = 2, 4, 8 or 16, a launch attribute: the ICP tuning's
// blocks per session) share the level's pixels (pixel blocks b = rank, rank + C, ...);
// every iteration each block reduces its FP64 sums into its own
// shared memory, a cluster barrier makes them visible, block 0 adds the blocks' sums in
// rank order through distributed shared memory and runs the host step (LM accept/reject,
// FP64 Cholesky, pose update) on one thread, and a second barrier publishes the new
// estimate, which every block reads from block 0's shared memory.  The hardware schedules
// a cluster's blocks together and its barriers need no polling; every block takes the same
// exits at the same points, since each decision comes from block 0's published state.
// One launch per tick replaces one launch per iteration, and sessions whose levels stop
// early leave their SMs to the others.
template <int PPT>
__global__ void __launch_bounds__(kIcpThreads, 2)
    k_icp_cluster(const SessionDesc* __restrict__ descs, int fam) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind != kTrackFrame || !in_family(s, fam)) return;  // the same for every block of the cluster
  TrackState* ts = s.ts;
  const int rank = (int)cluster.block_rank(), C = (int)cluster.num_blocks();
  __shared__ float sR[9], st[3];
  __shared__ DevXform sp;
  __shared__ double part[2][32];  // this block's depth / photometric sums
  __shared__ float bR[9], bt[3];  // block 0: the estimate after the host step
  __shared__ int bflags[2];       // block 0: status, level_done
  __shared__ double sums[kIcpTerms];
  __shared__ IcpLm lm;  // block 0: the tracker state during the kernel
  __shared__ IcpStepScratch hw;  // block 0: the LM step's intermediate values
  if (threadIdx.x < 9) sR[threadIdx.x] = ts->R[threadIdx.x];
  if (threadIdx.x < 3) st[threadIdx.x] = ts->t[threadIdx.x];
  if (threadIdx.x < 21) reinterpret_cast<float*>(&sp)[threadIdx.x] = reinterpret_cast<const float*>(&ts->xf)[threadIdx.x];
  const int status0 = ts->status;
  if (rank == 0 && threadIdx.x == 0) lm_copy(&lm, ts);
  // every block has read the initial state before block 0 writes any of it
  cluster.sync();
  if (status0 != 0) return;
  for (int level = s.levels - 1; level >= 0; --level) {
    const int n = (s.W >> level) * (s.H >> level);
    // the coarser levels in blocks of one pixel a thread: their few pixel blocks would
    // otherwise fall unevenly on the cluster's blocks (19 blocks of 1024 pixels for 16 at
    // 160 x 120), and a pass waits for its slowest block
    const int per_block = kIcpThreads * (level == 0 ? PPT : 1);
    const int nblocks = (n + per_block - 1) / per_block;
    const bool photo = s.photo_w > 0.f && level == 0;
    const int ncb = photo ? (s.W * s.H + per_block - 1) / per_block : 0;
    for (int iter = 0; iter < s.iters[level]; ++iter) {
      const float3 tc = f3(st[0], st[1], st[2]);
      double acc[kIcpTerms];
#pragma unroll
      for (int k = 0; k < kIcpTerms; ++k) acc[k] = 0.0;
      if (level == 0) {
        for (int vb = rank; vb < nblocks; vb += C) icp_depth_rows<PPT>(s, level, vb, sR, tc, sp, acc);
      } else {
        for (int vb = rank; vb < nblocks; vb += C) icp_depth_rows<1>(s, level, vb, sR, tc, sp, acc);
      }
      double D = icp_block_sum(acc);
      if (threadIdx.x < kIcpTerms) part[0][threadIdx.x] = D;
      if (photo) {
#pragma unroll
        for (int k = 0; k < kIcpTerms; ++k) acc[k] = 0.0;
        for (int vb = rank; vb < ncb; vb += C) icp_color_rows<PPT>(s, vb, sR, tc, acc);
        D = icp_block_sum(acc);
        if (threadIdx.x < kIcpTerms) part[1][threadIdx.x] = D;
      }
      cluster.sync();  // every block's sums are visible to block 0
      if (rank == 0) {
        if (threadIdx.x < kIcpTerms) {
          // the blocks' sums in rank order; the photometric normal equations and residual
          // enter weighted, the count stays the depth count
          double a = 0.0, c = 0.0;
          for (int r = 0; r < C; ++r) {
            const double* pr = cluster.map_shared_rank(&part[0][0], r);
            a += pr[threadIdx.x];
            if (photo) c += pr[32 + threadIdx.x];
          }
          if (photo && threadIdx.x < kIcpTerms - 1) a += (double)s.photo_w * c;
          sums[threadIdx.x] = a;
        }
        __syncthreads();
        if (threadIdx.x == 0) lm.icp_iters[level] += 1u;
        icp_host_step(&lm, hw, sums, iter, s.icp_min_count[level]);
        __syncthreads();
        if (threadIdx.x == 0) {
          for (int k = 0; k < 9; ++k) bR[k] = lm.R[k];
          for (int k = 0; k < 3; ++k) bt[k] = lm.t[k];
          bflags[0] = lm.status;
          bflags[1] = lm.level_done;
        }
      }
      cluster.sync();  // block 0's new estimate is visible to every block
      int flags[2];
      {
        const float* r0 = cluster.map_shared_rank(&bR[0], 0);
        const float* t0 = cluster.map_shared_rank(&bt[0], 0);
        const int* f0 = cluster.map_shared_rank(&bflags[0], 0);
        if (threadIdx.x < 9) sR[threadIdx.x] = r0[threadIdx.x];
        if (threadIdx.x < 3) st[threadIdx.x] = t0[threadIdx.x];
        flags[0] = f0[0];
        flags[1] = f0[1];
      }
      __syncthreads();
      if (flags[0] != 0) {  // tracking lost: every block leaves together
        if (rank == 0 && threadIdx.x == 0) lm_copy(ts, &lm);
        cluster.sync();     // (block 0's shared memory stays alive until all have read it)
        return;
      }
      if (flags[1]) break;
    }
  }
  if (rank == 0 && threadIdx.x == 0) lm_copy(ts, &lm);
  cluster.sync();  // no block leaves while another may still read block 0's shared memory
}

template __global__ void k_icp_cluster<2>(const SessionDesc*, int);
template __global__ void k_icp_cluster<4>(const SessionDesc*, int);
template __global__ void k_icp_cluster<8>(const SessionDesc*, int);
template __global__ void k_icp_cluster<16>(const SessionDesc*, int);

// After the last ICP launch (or on frame 0): publish the pose, decide the integration
// gate (NuiKinfuTrackingEngine.cpp:115-127) and reset the estimate for the next frame.
// Running sums of integrateTsdfVolumeKernel that do not depend on the voxel column
// (tsdfVolume.cl:74-79: v_g_z and z_scaled, both advanced by cell_z per slice), for the
// pose integration will use: ztab[z] and ztab[rz + 1 + z] after z additions.
__device__ void fill_ztab(const SessionDesc& s, const TrackState* ts) {
  if (!s.ztab) return;
  const int rz = s.res[2];
  const float c2 = s.cell[2];
  float vgz = 0.5f * c2 - ts->xf.t[2], zs = 0.f;
  for (int z = 0; z <= rz; ++z) {
    s.ztab[z] = vgz;
    s.ztab[rz + 1 + z] = zs;
    vgz += c2;
    zs += c2;
  }
}

// NuiKinfuOpenCLShiftScene::integrateVolume -> shiftVolume (NuiKinfuOpenCLShiftScene.cpp:
// 288-362): before a shifting volume integrates, every axis on which the camera lies
// voxel_shift or more voxels from the basis moves the volume by voxel_shift voxels; the
// camera's local translation moves back by the same distance and the offset forward.  The
// frame's shift is left in ts->shift for the fetch / roll kernels that follow.
__device__ void shift_decide(const SessionDesc& s, TrackState* ts) {
  ts->shift[0] = ts->shift[1] = ts->shift[2] = 0;
  const int vs = s.voxel_shift;
  if (vs <= 0 || s.fmt < 0) return;
  float st[3];
  int tr[3];
  for (int a = 0; a < 3; ++a) {
    st[a] = ts->xf.t[a] - s.shift_basis[a];
    const int f = (int)floorf(st[a] / s.cell[a]);
    tr[a] = st[a] < 0.f ? max(-vs, f) : min(vs, f);
  }
  for (int a = 0; a < 3; ++a)
    if (abs(tr[a]) >= vs) {
      ts->shift[a] = tr[a];
      ts->voff[a] += tr[a];
      st[a] -= (float)tr[a] * s.cell[a];
    }
  for (int a = 0; a < 3; ++a) {
    ts->xf.t[a] = st[a] + s.shift_basis[a];
    ts->t[a] = ts->xf.t[a];
  }
}

// The table for an integration the host requests directly (step-wise calls), after the
// shift that integration makes.
__global__ void k_ztab(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.x];
  if (threadIdx.x == 0 && s.kind >= 0) {
    shift_decide(s, s.ts);
    fill_ztab(s, s.ts);
  }
}

// shift_now: the tick's finalize makes the shifting volume's shift of an integrating
// frame here; the step-wise track leaves it to the integration call (k_ztab).
__global__ void k_track_finalize(const SessionDesc* __restrict__ descs, int shift_now, int fam) {
  const SessionDesc& s = descs[blockIdx.x];
  if (threadIdx.x != 0 || s.kind < 0 || !in_family(s, fam)) return;
  TrackState* ts = s.ts;
  if (s.kind == kFirstFrame) {
    ts->integrate = ts->status == 0 ? 1 : 0;
    ts->shift[0] = ts->shift[1] = ts->shift[2] = 0;
    if (ts->integrate) {
      if (shift_now) shift_decide(s, ts);
      fill_ztab(s, ts);
    }
    return;
  }
  ts->shift[0] = ts->shift[1] = ts->shift[2] = 0;
  if (ts->status != 0) {  // tracking lost: keep the previous pose, skip the rest
    for (int i = 0; i < 9; ++i) ts->R[i] = ts->xf.R[i];
    for (int i = 0; i < 3; ++i) ts->t[i] = ts->xf.t[i];
    ts->integrate = 0;
    return;
  }
  double a[9];
  for (int i = 0; i < 9; ++i) a[i] = ts->R[i];
  const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
  const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  const double inv[9] = {c00, a[2] * a[7] - a[1] * a[8], a[1] * a[5] - a[2] * a[4],
                         c01, a[0] * a[8] - a[2] * a[6], a[2] * a[3] - a[0] * a[5],
                         c02, a[1] * a[6] - a[0] * a[7], a[0] * a[4] - a[1] * a[3]};
  for (int i = 0; i < 9; ++i) {
    ts->xf.R[i] = ts->R[i];
    ts->xf.R_inv[i] = (float)(inv[i] / det);
  }
  for (int i = 0; i < 3; ++i) ts->xf.t[i] = ts->t[i];
  // rotation angle of R^-1 * R_last and translation distance
  double tr = 0;
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) tr += (double)ts->R[k * 3 + i] * (double)ts->lastR[k * 3 + i];
  const double cv = fmin(1.0, fmax(-1.0, (tr - 1.0) / 2.0));
  const double rn = acos(cv);
  // translations compared globally: local + the volume's offset (0 for a fixed volume)
  double tn = 0;
  for (int i = 0; i < 3; ++i) {
    const float g = ts->voff[i] ? ts->t[i] + (float)ts->voff[i] * s.cell[i] : ts->t[i];
    tn += ((double)(g - ts->lastT[i])) * ((double)(g - ts->lastT[i]));
  }
  tn = sqrt(tn);
  ts->integrate = ((float)((rn + tn) / 2) >= s.integ_thr) ? 1 : 0;
  if (ts->integrate) {
    if (shift_now) shift_decide(s, ts);
    fill_ztab(s, ts);
    for (int i = 0; i < 9; ++i) ts->lastR[i] = ts->R[i];
    for (int i = 0; i < 3; ++i) ts->lastT[i] = ts->voff[i] ? ts->t[i] + (float)ts->voff[i] * s.cell[i] : ts->t[i];
  }
}

}  // namespace nui
