// Volume access of the dense raycast (raycastKernel, raycast.cl:128-277;
// interpolateTrilineary raycast.cl:36-120), shared by the exact kernels (nui_k_raycast.cu)
// and the tolerance-mode kernels of the FP16 formats (nui_k_raycast_fast.cu).
#pragma once
#include "nui_device.cuh"

namespace nui {

// FAST: nearest voxel by a rounded product with 1/cell instead of the exactly rounded
// quotient, and trilinear fractions by that product too (tolerance mode).
template <int FMT, bool FAST = false>
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
    if (FAST) {
      gx = round_half_up(p.x * i0);  // exact ties up, as OpenCL's round()
      gy = round_half_up(p.y * i1);
      gz = round_half_up(p.z * i2);
    } else {
      gx = round_div(p.x, c0, i0);
      gy = round_div(p.y, c1, i1);
      gz = round_div(p.z, c2, i2);
    }
  }
  // Out of line: called at eight places of the exact hit refinement, whose inlined copies
  // overflow the instruction cache.
  __device__ __noinline__ float trilinear(float3 p) const { return trilinear_inl(p); }
  // Inlined form: the tolerance-mode refinement evaluates several samples in one
  // expression, so that their voxel loads are in flight together.
  __device__ __forceinline__ float trilinear_inl(float3 p) const {
    int gx, gy, gz;
    voxel_of(p, gx, gy, gz);
    if (gx <= 0 || gx >= rx - 1) return qnan();
    if (gy <= 0 || gy >= ry - 1) return qnan();
    if (gz <= 0 || gz >= rz - 1) return qnan();
    const float vx = ((float)gx + 0.5f) * c0, vy = ((float)gy + 0.5f) * c1, vz = ((float)gz + 0.5f) * c2;
    gx = (p.x < vx) ? gx - 1 : gx;
    gy = (p.y < vy) ? gy - 1 : gy;
    gz = (p.z < vz) ? gz - 1 : gz;
    float a, b, c;
    if (FAST) {
      a = p.x * i0 - ((float)gx + 0.5f);
      b = p.y * i1 - ((float)gy + 0.5f);
      c = p.z * i2 - ((float)gz + 0.5f);
    } else {
      a = (p.x - ((float)gx + 0.5f) * c0) / c0;
      b = (p.y - ((float)gy + 0.5f) * c1) / c1;
      c = (p.z - ((float)gz + 0.5f) * c2) / c2;
    }
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

}  // namespace nui
