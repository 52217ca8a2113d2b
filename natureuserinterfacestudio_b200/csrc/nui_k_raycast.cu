// Dense raycast (raycastKernel, raycast.cl:128-277; interpolateTrilineary raycast.cl:36-120;
// getMinTime / getMaxTime raycast.cl:4-20).  One thread per pixel writes the world-space
// reference vertex / normal maps (and colour) that the next frame's ICP reads.
//
// Semantics kept from the reference: nearest-voxel sampling by round(p / cell) with voxel
// centres at (g + 0.5) cell, march step 0.8 * trunc, zero crossing refined by the two
// trilinear samples around it, central-difference normal; the trilinear weights pair the
// x-neighbour voxel with the y fraction and the y-neighbour with the x fraction, as the
// reference's index walk does (raycast.cl:66-119).
#include "nui_device.cuh"

namespace nui {

template <int FMT>
struct RayVol {
  const SessionDesc& s;
  int rx, ry, rz;
  float c0, c1, c2;
  float i0, i1, i2;  // 1 / cell
  // tsdf of a voxel if its weight is > 0; bricks never touched are answered from the
  // occupancy map without reading the voxel
  __device__ __forceinline__ bool tsdf_at(int x, int y, int z, float& f) const {
    if (s.occ && __ldg(s.occ + occ_index(s, x, y, z)) == 0) return false;
    const size_t i = vox_index(s, x, y, z);
    if (FMT == 2) {  // weight plane first: the tsdf plane is read only for weighted voxels
      if (__ldg(s.wvol + i) == 0) return false;
      f = __half2float(reinterpret_cast<const __half*>(s.vol)[i]);
      return true;
    }
    int W;
    Voxel<FMT>::load(s, i, f, W);
    return W > 0;
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
  const RayVol<FMT> V{s, s.res[0], s.res[1], s.res[2], s.cell[0], s.cell[1], s.cell[2],
                       1.0f / s.cell[0], 1.0f / s.cell[1], 1.0f / s.cell[2]};
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
      tsdf = V.tsdf_at(gx, gy, gz, f) ? f : qnan();
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
        if (s.cvol) cout = s.cvol[vox_index(s, gx, gy, gz)];
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
