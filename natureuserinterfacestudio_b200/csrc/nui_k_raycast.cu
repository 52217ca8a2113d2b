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
// Brick skipping (exact): when a sample lands in an 8^3 brick whose voxels are all
// unweighted (every sample there reads NaN) or all weighted with tsdf > 0 (every sample
// there is positive, so after the first one no transition can happen), the following
// samples that stay inside the brick -- by a margin of 1% of a voxel -- change nothing but
// the march parameter; they are skipped by advancing the parameter with the same float
// additions.
#include "nui_device.cuh"

namespace nui {

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
    } else if (FMT == 2) {
      if (__ldg(wvol + i) == 0) return false;
      f = __half2float(reinterpret_cast<const __half*>(vol)[i]);
      return true;
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
  __device__ float trilinear(float3 p) const {
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
    float t000, t001, t011, t010, t110, t111, t101, t100;
    if (!tsdf_at(gx, gy, gz, t000)) return qnan();
    if (!tsdf_at(gx, gy, gz + 1, t001)) return qnan();
    if (!tsdf_at(gx + 1, gy, gz + 1, t011)) return qnan();
    if (!tsdf_at(gx + 1, gy, gz, t010)) return qnan();
    if (!tsdf_at(gx + 1, gy + 1, gz, t110)) return qnan();
    if (!tsdf_at(gx + 1, gy + 1, gz + 1, t111)) return qnan();
    if (!tsdf_at(gx, gy + 1, gz + 1, t101)) return qnan();
    if (!tsdf_at(gx, gy + 1, gz, t100)) return qnan();
    return t000 * (1 - a) * (1 - b) * (1 - c) + t001 * (1 - a) * (1 - b) * c + t010 * (1 - a) * b * (1 - c) +
           t011 * (1 - a) * b * c + t100 * a * (1 - b) * (1 - c) + t101 * a * (1 - b) * c +
           t110 * a * b * (1 - c) + t111 * a * b * c;
  }
  // Largest ray parameter up to which a sample stays (by 1% of a voxel) inside the
  // p-box of brick (x>>3, y>>3, z>>3) clipped to the volume; samples with parameter below
  // it map to voxels of that brick.
  __device__ __forceinline__ float brick_exit(int gx, int gy, int gz, float3 start, float3 dir) const {
    const int b[3] = {gx & ~7, gy & ~7, gz & ~7};
    const int r[3] = {rx, ry, rz};
    const float c[3] = {c0, c1, c2};
    const float o[3] = {start.x, start.y, start.z};
    const float d[3] = {dir.x, dir.y, dir.z};
    float te = 3.4e38f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float lo = ((float)b[a] - 0.5f + 0.01f) * c[a];
      const float hi = ((float)min(b[a] + 8, r[a]) - 0.5f - 0.01f) * c[a];
      if (d[a] > 0.f) te = fminf(te, (hi - o[a]) / d[a]);
      else if (d[a] < 0.f) te = fminf(te, (lo - o[a]) / d[a]);
    }
    return te;
  }
};

template <int FMT>
__global__ void __launch_bounds__(128) k_raycast(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind != kTrackFrame || s.fmt != FMT || s.ts->status != 0) return;
  const int W = s.W, H = s.H;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= W * H) return;
  const int px = id % W, py = id / W;
  const float4 nanv = make_float4(qnan(), qnan(), qnan(), 0.f);
  float4 vout = nanv, nout = nanv;
  uchar4 cout = make_uchar4(0, 0, 0, 0);
  const RayVol<FMT> V{s.vol, s.wvol, s.occ, s.res[0], s.res[1], s.res[2], (s.res[0] + 7) >> 3, (s.res[1] + 7) >> 3,
                      s.cell[0], s.cell[1], s.cell[2], 1.0f / s.cell[0], 1.0f / s.cell[1], 1.0f / s.cell[2]};
  const DevXform& m = s.ts->xf;
  const float D0 = s.dim[0], D1 = s.dim[1], D2 = s.dim[2];
  const float3 off = f3(D0 / 2.0f, D1 / 2.0f, 0.f);
  const float3 t = f3(m.t[0], m.t[1], m.t[2]);
  const float3 start = add3(t, off);
  float3 nx = f3(((float)px - s.cam.cx) * s.cam.fx_inv, ((float)py - s.cam.cy) * s.cam.fy_inv, 1.f);
  nx = add3(add3(rot_rows(m.R, nx), t), off);
  const float3 dir = normalize3(sub3(nx, start));
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
    float tc = tmin;
    int gx, gy, gz;
    V.voxel_of(add3(start, mul3(dir, tc)), gx, gy, gz);
    gx = max(0, min(gx, V.rx - 1));
    gy = max(0, min(gy, V.ry - 1));
    gz = max(0, min(gz, V.rz - 1));
    float tsdf = qnan(), f;
    if (V.tsdf_at(gx, gy, gz, f)) tsdf = f;
    const float max_time = 3 * (D0 + D1 + D2);
    const float step = s.trunc * 0.8f;
    for (; tc < max_time; tc += step) {
      const float prev = tsdf;
      V.voxel_of(add3(start, mul3(dir, tc + step)), gx, gy, gz);
      if (!(gx >= 0 && gy >= 0 && gz >= 0 && gx < V.rx && gy < V.ry && gz < V.rz)) break;
      const uint8_t st = V.occ ? __ldg(V.occ + V.bidx(gx, gy, gz)) : (uint8_t)kBrickMixed;
      if (st == kBrickEmpty) {
        tsdf = qnan();
      } else {
        tsdf = V.load(V.vidx(gx, gy, gz), f) ? f : qnan();
      }
      if (st == kBrickEmpty || (st == kBrickPositive && !(prev < 0.f))) {
        // every further sample inside this brick reads the same kind of value: skip them
        const float te = V.brick_exit(gx, gy, gz, start, dir);
        for (;;) {
          const float tn = tc + step;
          if (!(tn < max_time) || !(tn + step < te)) break;
          tc = tn;
        }
        continue;
      }
      if (isnan(tsdf) || isnan(prev)) continue;
      if (prev < 0.f && tsdf > 0.f) break;
      if (prev >= 0.f && tsdf <= 0.f) {
        const float Ftdt = V.trilinear(add3(start, mul3(dir, tc + step)));
        if (isnan(Ftdt)) break;
        const float Ft = V.trilinear(add3(start, mul3(dir, tc)));
        if (isnan(Ft)) break;
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
        break;
      }
    }
  }
  s.vref[id] = vout;
  s.nref[id] = nout;
  if (s.cmap) s.cmap[id] = cout;
}

template __global__ void k_raycast<0>(const SessionDesc*);
template __global__ void k_raycast<1>(const SessionDesc*);
template __global__ void k_raycast<2>(const SessionDesc*);
template __global__ void k_raycast<3>(const SessionDesc*);

}  // namespace nui
