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
#include "nui_device.cuh"

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
struct RayVol {
  const void* vol;
  const uint8_t* wvol;
  const uint8_t* occ;
  int rx, ry, rz, bx, by;
  float c0, c1, c2;
  float i0, i1, i2;  // 1 / cell
  __device__ __forceinline__ unsigned vidx(int x, int y, int z) const {
    return (unsigned)x + (unsigned)rx * ((unsigned)y + (unsigned)ry * (unsigned)z);
  }
  __device__ __forceinline__ unsigned bidx(int x, int y, int z) const {
    return (unsigned)(x >> 3) + (unsigned)bx * ((unsigned)(y >> 3) + (unsigned)by * (unsigned)(z >> 3));
  }
  __device__ __forceinline__ bool load(unsigned i, float& f) const {
    if (FMT == 0) {
      const short2 v = __ldg(reinterpret_cast<const short2*>(vol) + i);
      f = (float)v.x / 32766.f;
      return v.y > 0;
    } else if (FMT == 1) {
      const float2 v = __ldg(reinterpret_cast<const float2*>(vol) + i);
      f = v.x;
      return (int)v.y > 0;
    } else if (FMT == 2) {  // both planes read at once (no load waits on the other)
      const uint8_t w = __ldg(wvol + i);
      f = __half2float(__ldg(reinterpret_cast<const __half*>(vol) + i));
      return w != 0;
    } else {
      const __half2 v = reinterpret_cast<const __half2*>(vol)[i];
      f = __low2float(v);
      return (int)__high2float(v) > 0;
    }
  }
  // tsdf of a voxel if its weight is > 0
  __device__ __forceinline__ bool tsdf_at(int x, int y, int z, float& f) const {
    if (occ && __ldg(occ + bidx(x, y, z)) == kBrickEmpty) return false;
    return load(vidx(x, y, z), f);
  }
  __device__ __forceinline__ void voxel_of(float3 p, int& gx, int& gy, int& gz) const {
    gx = round_div(p.x, c0, i0);
    gy = round_div(p.y, c1, i1);
    gz = round_div(p.z, c2, i2);
  }
  // Out of line: called at eight places of the hit refinement, whose inlined copies
  // overflow the instruction cache.
  __device__ __noinline__ float trilinear(float3 p) const {
    int gx, gy, gz;
    voxel_of(p, gx, gy, gz);
    if (gx <= 0 || gx >= rx - 1) return qnan();
    if (gy <= 0 || gy >= ry - 1) return qnan();
    if (gz <= 0 || gz >= rz - 1) return qnan();
    const float vx = ((float)gx + 0.5f) * c0, vy = ((float)gy + 0.5f) * c1, vz = ((float)gz + 0.5f) * c2;
    gx = (p.x < vx) ? gx - 1 : gx;
    gy = (p.y < vy) ? gy - 1 : gy;
    gz = (p.z < vz) ? gz - 1 : gz;
    const float a = (p.x - ((float)gx + 0.5f) * c0) / c0;
    const float b = (p.y - ((float)gy + 0.5f) * c1) / c1;
    const float c = (p.z - ((float)gz + 0.5f) * c2) / c2;
    // The eight voxels read directly, all at once (a voxel of an empty brick has weight 0
    // anyway, so the brick test of tsdf_at would only add work here, next to the surface);
    // any unweighted one makes the sample NaN, whichever it is.
    float t000, t001, t011, t010, t110, t111, t101, t100;
    const unsigned i = vidx(gx, gy, gz), dy = (unsigned)rx, dz = (unsigned)rx * (unsigned)ry;
    bool ok = load(i, t000);
    ok &= load(i + dz, t001);
    ok &= load(i + 1 + dz, t011);
    ok &= load(i + 1, t010);
    ok &= load(i + 1 + dy, t110);
    ok &= load(i + 1 + dy + dz, t111);
    ok &= load(i + dy + dz, t101);
    ok &= load(i + dy, t100);
    if (!ok) return qnan();
    return t000 * (1 - a) * (1 - b) * (1 - c) + t001 * (1 - a) * (1 - b) * c + t010 * (1 - a) * b * (1 - c) +
           t011 * (1 - a) * b * c + t100 * a * (1 - b) * (1 - c) + t101 * a * (1 - b) * c +
           t110 * a * b * (1 - c) + t111 * a * b * c;
  }
  // Largest ray parameter up to which a sample stays (by 1% of a voxel) inside the
  // p-box of the aligned region of S^3 voxels (S a power of two) holding (gx, gy, gz),
  // clipped to the volume; samples with parameter below it map to voxels of that region.
  // The margin also absorbs the rounding of the reciprocal direction used here.
  __device__ __forceinline__ float region_exit(int S, int gx, int gy, int gz, float3 start, float3 dir,
                                               float3 idir) const {
    const int b[3] = {gx & ~(S - 1), gy & ~(S - 1), gz & ~(S - 1)};
    const int r[3] = {rx, ry, rz};
    const float c[3] = {c0, c1, c2};
    const float o[3] = {start.x, start.y, start.z};
    const float d[3] = {dir.x, dir.y, dir.z};
    const float id[3] = {idir.x, idir.y, idir.z};
    float te = 3.4e38f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float lo = ((float)b[a] - 0.5f + 0.01f) * c[a];
      const float hi = ((float)min(b[a] + S, r[a]) - 0.5f - 0.01f) * c[a];
      if (d[a] > 0.f) te = fminf(te, (hi - o[a]) * id[a]);
      else if (d[a] < 0.f) te = fminf(te, (lo - o[a]) * id[a]);
    }
    return te;
  }
};

// Camera ray of pixel (px, py) in volume coordinates (raycast.cl:150-162): its start (the
// camera centre), direction and the volume offset (half the x / y extent).
__device__ __forceinline__ void ray_of(const SessionDesc& s, int px, int py, float3& start, float3& dir, float3& off) {
  const DevXform& m = s.ts->xf;
  off = f3(s.dim[0] / 2.0f, s.dim[1] / 2.0f, 0.f);
  const float3 t = f3(m.t[0], m.t[1], m.t[2]);
  start = add3(t, off);
  float3 nx = f3(((float)px - s.cam.cx) * s.cam.fx_inv, ((float)py - s.cam.cy) * s.cam.fy_inv, 1.f);
  nx = add3(add3(rot_rows(m.R, nx), t), off);
  dir = normalize3(sub3(nx, start));
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
