// Dense raycast (raycastKernel, raycast.cl:128-277; interpolateTrilineary raycast.cl:36-120;
// getMinTime / getMaxTime raycast.cl:4-20).  One thread per pixel writes the world-space
// reference vertex / normal maps (and colour) that the next frame's ICP reads.
//
// Semantics kept from the reference: nearest-voxel sampling by round(p / cell) with voxel
// centres at (g + 0.5) cell, march step 0.8 * trunc accumulated in float, zero crossing
// refined by the two trilinear samples around it, central-difference normal; the
// trilinear weights pair the x-neighbour voxel with the y fraction and the y-neighbour
// with the x fraction, as the reference's index walk does (raycast.cl:66-119).
//
// Region skipping (exact): when a sample lands in an 8^3 brick, or a 32^3 super-brick,
// that holds no weighted voxel with tsdf <= 0, no two consecutive samples inside it can
// form a transition (each reads NaN or a positive value).  The samples that stay inside
// the region -- by a margin of 1% of a voxel -- are skipped: the march parameter jumps to
// the last of them along the exact float sequence t <- t + step (march_advance), and only
// that sample is read (its value, NaN or positive, is the next "previous" sample).  In an
// all-empty region, or a brick whose voxels are all weighted and positive, it is known
// without the read.
#include "nui_raycast.cuh"

namespace nui {

// t <- fl(t + step) repeated while fl(t + step) < Y (for Y <= cap this is also the
// plain loop's "while t < cap and fl(t + step) < Y"); returns the final t, the same value
// as the plain loop.  Inside one binade [2^e, 2^(e+1)) every element is a multiple of
// u = 2^(e-23), and as long as the sum stays in the binade fl(t + step) = t + M u with M
// the integer nearest step / u (on an exact tie, round to even: once t / u is even the
// increment is the even one of the two neighbours).  Runs of additions inside a binade
// are therefore counted in 32-bit integers (t / u < 2^24); the addition that leaves a
// binade is done plainly.
__device__ __forceinline__ float march_advance(float t, float step, float Y) {
  for (;;) {
    const float n = t + step;
    if (!(n < Y) || !(n > t)) return t;
    const int ex = ((__float_as_int(t) >> 23) & 0xff) - 127;  // t in [2^ex, 2^(ex+1))
    if (ex < -100 || ex > 100) {
      t = n;
      continue;
    }
    const float inv_u = __int_as_float((127 + 23 - ex) << 23);
    const float u = __int_as_float((127 - 23 + ex) << 23);
    const float q = step * inv_u;  // exact: scaling by a power of two
    if (!(q < 8388608.f)) {        // the step spans the binade
      t = n;
      continue;
    }
    const float fq = floorf(q), fr = q - fq;
    unsigned M = (unsigned)fq;
    const unsigned T = (unsigned)(t * inv_u);
    if (fr == 0.5f) {
      if (T & 1u) {  // the first tie may round up; afterwards t / u stays even
        t = n;
        continue;
      }
      M += (M & 1u);
    } else if (fr > 0.5f) {
      M += 1u;
    }
    const float ys = Y * inv_u;
    const unsigned L = ys < 16777216.f ? (unsigned)ceilf(ys) - 1u : 16777215u;  // results must stay <= L
    if (L < T + M) {  // the next addition leaves the binade
      t = n;
      continue;
    }
    const unsigned k = (L - T) / M;
    t = (float)(T + k * M) * u;
  }
}

// The plain loop, for the rare call whose cap lies below its bound.
__device__ __noinline__ float march_advance_capped(float t, float step, float Y, float cap) {
  for (;;) {
    if (!(t < cap)) return t;
    const float n = t + step;
    if (!(n < Y) || !(n > t)) return t;
    t = n;
  }
}

template <int FMT>
__global__ void __launch_bounds__(128) k_raycast(const SessionDesc* __restrict__ descs, int tw) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind != kTrackFrame || s.fmt != FMT || s.ts->status != 0) return;
  // each warp shades a tw x (32 / tw) pixel tile, a block 2 x 2 of them (neighbouring rays
  // march alike; tw is tuned)
  const int W = s.W, H = s.H;
  const int th = 32 / tw, bw = 2 * tw, bh = 2 * th;
  const int tiles_x = (W + bw - 1) / bw;
  if ((int)blockIdx.x >= tiles_x * ((H + bh - 1) / bh)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int px = ((int)blockIdx.x % tiles_x) * bw + (warp & 1) * tw + lane % tw;
  const int py = ((int)blockIdx.x / tiles_x) * bh + (warp >> 1) * th + lane / tw;
  if (px >= W || py >= H) return;
  const int id = py * W + px;
  const RayVol<FMT> V{s.vol, s.wvol, s.occ, s.res[0], s.res[1], s.res[2], (s.res[0] + 7) >> 3, (s.res[1] + 7) >> 3,
                      s.cell[0], s.cell[1], s.cell[2], 1.0f / s.cell[0], 1.0f / s.cell[1], 1.0f / s.cell[2]};
  const float D0 = s.dim[0], D1 = s.dim[1], D2 = s.dim[2];
  float3 start, dir, off;
  ray_of(s, px, py, start, dir, off);
  bool hit = false;  // a zero crossing between the samples at tc and tc + step
  float tc = 0.f;
  const float txmin = ((double)fabsf(dir.x) < 1e-14) ? 0.f : (((dir.x > 0 ? 0.f : D0) - start.x) / dir.x);
  const float tymin = ((double)fabsf(dir.y) < 1e-14) ? 0.f : (((dir.y > 0 ? 0.f : D1) - start.y) / dir.y);
  const float tzmin = ((double)fabsf(dir.z) < 1e-14) ? 0.f : (((dir.z > 0 ? 0.f : D2) - start.z) / dir.z);
  float tmin = fmaxf(fmaxf(txmin, tymin), tzmin);
  const float txmax = ((double)fabsf(dir.x) < 1e-14) ? 1e14f : (((dir.x > 0 ? D0 : 0.f) - start.x) / dir.x);
  const float tymax = ((double)fabsf(dir.y) < 1e-14) ? 1e14f : (((dir.y > 0 ? D1 : 0.f) - start.y) / dir.y);
  const float tzmax = ((double)fabsf(dir.z) < 1e-14) ? 1e14f : (((dir.z > 0 ? D2 : 0.f) - start.z) / dir.z);
  const float tmax = fminf(fminf(txmax, tymax), tzmax);
  tmin = fmaxf(tmin, 0.f);
  if (tmin < tmax) {
    tc = tmin;
    int gx, gy, gz;
    V.voxel_of(add3(start, mul3(dir, tc)), gx, gy, gz);
    gx = max(0, min(gx, V.rx - 1));
    gy = max(0, min(gy, V.ry - 1));
    gz = max(0, min(gz, V.rz - 1));
    float tsdf = qnan(), f;
    if (V.tsdf_at(gx, gy, gz, f)) tsdf = f;
    const float max_time = 3 * (D0 + D1 + D2);
    const float step = s.trunc * 0.8f;
    const int sx = (V.rx + 31) >> 5, sy = (V.ry + 31) >> 5;
    const int hx = (V.rx + 127) >> 7, hy = (V.ry + 127) >> 7;
    const float3 idir = f3(1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z);
    bool pend = false;  // tsdf stands for a skipped sample at tc whose class (NaN or > 0) is unread
    float tn = tc;
    while (tc < max_time) {
      float prev = tsdf;
      tn = tc + step;
      V.voxel_of(add3(start, mul3(dir, tn)), gx, gy, gz);
      if (!(gx >= 0 && gy >= 0 && gz >= 0 && gx < V.rx && gy < V.ry && gz < V.rz)) break;
      const uint8_t st = V.occ ? __ldg(V.occ + V.bidx(gx, gy, gz)) : (uint8_t)kBrickMixed;
      // only the class of a sample (NaN, < 0, 0, > 0) enters the march decisions
      if (st == kBrickEmpty) {
        tsdf = qnan();
      } else if (st == kBrickPositive) {
        tsdf = 1.0f;
      } else {
        tsdf = V.load(V.vidx(gx, gy, gz), f) ? f : qnan();
      }
      if ((st == kBrickEmpty || st == kBrickPositive || st == kBrickNoNeg) && (!(prev < 0.f) || isnan(tsdf))) {
        // no transition at this sample (its value is NaN or > 0 and prev is not negative,
        // or it is NaN), nor between any two samples of the region: skip to the last one
        int S = 128;
        bool uniform;
        const uint8_t s3 = __ldg(s.occ3 + (gx >> 7) + hx * ((gy >> 7) + hy * (gz >> 7)));
        if (s3 == kSuperEmpty || s3 == kSuperSkip) {
          uniform = s3 == kSuperEmpty;
        } else {
          const uint8_t s2 = __ldg(s.occ2 + (gx >> 5) + sx * ((gy >> 5) + sy * (gz >> 5)));
          if (s2 == kSuperEmpty || s2 == kSuperSkip) {
            S = 32;
            uniform = s2 == kSuperEmpty;
          } else {
            S = 8;
            uniform = st != kBrickNoNeg;
          }
        }
        const float te = V.region_exit(S, gx, gy, gz, start, dir, idir);
        const float tl = te <= max_time ? march_advance(tn, step, te) : march_advance_capped(tn, step, te, max_time);
        if (tl == tn || uniform) {
          pend = false;  // tsdf is the class of the sample at tl
        } else {
          pend = true;
          tsdf = 1.0f;
        }
        tc = tl;
        continue;
      }
      if (pend) {  // the previous sample was skipped: read its class now
        int lx, ly, lz;
        V.voxel_of(add3(start, mul3(dir, tc)), lx, ly, lz);
        prev = V.tsdf_at(lx, ly, lz, f) ? f : qnan();
        pend = false;
      }
      if (isnan(tsdf) || isnan(prev)) {
        tc = tn;
        continue;
      }
      if (prev < 0.f && tsdf > 0.f) break;
      if (prev >= 0.f && tsdf <= 0.f) {
        hit = true;
        break;
      }
      tc = tn;
    }
  }
  // the crossing waits in the vertex map for k_raycast_finish
  s.vref[id] = make_float4(tc, 0.f, 0.f, hit ? 1.f : 0.f);
}

// The zero-crossing refinement, normal and colour of every pixel after the march
// (raycast.cl:212-272): a kernel of its own, so that the march keeps fewer registers and the
// refining lanes of a warp run together.
template <int FMT>
__global__ void __launch_bounds__(256, 4) k_raycast_finish(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind != kTrackFrame || s.fmt != FMT || s.ts->status != 0) return;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= s.W * s.H) return;
  const float4 e = s.vref[id];
  const float4 nanv = make_float4(qnan(), qnan(), qnan(), 0.f);
  float4 vout = nanv, nout = nanv;
  uchar4 cout = make_uchar4(0, 0, 0, 0);
  if (e.w != 0.f) {
    const RayVol<FMT> V{s.vol, s.wvol, s.occ, s.res[0], s.res[1], s.res[2], (s.res[0] + 7) >> 3, (s.res[1] + 7) >> 3,
                        s.cell[0], s.cell[1], s.cell[2], 1.0f / s.cell[0], 1.0f / s.cell[1], 1.0f / s.cell[2]};
    float3 start, dir, off;
    ray_of(s, id % s.W, id / s.W, start, dir, off);
    const float step = s.trunc * 0.8f;
    const float tc = e.x, tn = tc + step;
    int gx, gy, gz;
    V.voxel_of(add3(start, mul3(dir, tn)), gx, gy, gz);
    const float Ftdt = V.trilinear(add3(start, mul3(dir, tn)));
    const float Ft = isnan(Ftdt) ? Ftdt : V.trilinear(add3(start, mul3(dir, tc)));
    if (!isnan(Ft)) {
      const float Ts = tc - step * Ft / (Ftdt - Ft);
      const float3 vf = add3(start, mul3(dir, Ts));
      vout = w0(sub3(vf, off));
      if (s.cvol) cout = s.cvol[V.vidx(gx, gy, gz)];
      int hx, hy, hz;
      V.voxel_of(add3(start, mul3(dir, tc)), hx, hy, hz);
      if (hx > 1 && hy > 1 && hz > 1 && hx < V.rx - 2 && hy < V.ry - 2 && hz < V.rz - 2) {
        float3 q, n;
        q = vf; q.x += s.cell[0]; const float fx1 = V.trilinear(q);
        q = vf; q.x -= s.cell[0]; const float fx2 = V.trilinear(q);
        n.x = fx1 - fx2;
        q = vf; q.y += s.cell[1]; const float fy1 = V.trilinear(q);
        q = vf; q.y -= s.cell[1]; const float fy2 = V.trilinear(q);
        n.y = fy1 - fy2;
        q = vf; q.z += s.cell[2]; const float fz1 = V.trilinear(q);
        q = vf; q.z -= s.cell[2]; const float fz2 = V.trilinear(q);
        n.z = fz1 - fz2;
        nout = w0(normalize3(n));
      }
    }
  }
  s.vref[id] = vout;
  s.nref[id] = nout;
  if (s.cmap) s.cmap[id] = cout;
}

template __global__ void k_raycast<0>(const SessionDesc*, int);
template __global__ void k_raycast<1>(const SessionDesc*, int);
template __global__ void k_raycast<2>(const SessionDesc*, int);
template __global__ void k_raycast<3>(const SessionDesc*, int);
template __global__ void k_raycast_finish<0>(const SessionDesc*);
template __global__ void k_raycast_finish<1>(const SessionDesc*);
template __global__ void k_raycast_finish<2>(const SessionDesc*);
template __global__ void k_raycast_finish<3>(const SessionDesc*);

}  // namespace nui
