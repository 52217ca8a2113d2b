// Dense TSDF integration in tolerance mode: the FP16 serving formats (NUI_TSDF_F16_U8,
// NUI_TSDF_F16_F16).  Same update as integrateTsdfVolumeKernel (tsdfVolume.cl:31-190) --
// project the voxel centre with R_inv, round to a pixel, sdf = ray depth - |voxel - camera|,
// update when sdf >= -trunc with tsdf = min(1, sdf / trunc), running average capped at
// weight 128, colour averaged inside the band -- evaluated with each voxel's position
// computed directly (fused multiply-adds, approximate reciprocal and square root) instead of
// the reference's incremental z sums.  Results agree with the reference within the TSDF
// tolerance (1e-3 truncation units, well above the half-precision quantum), not bit for bit;
// the int16 and FP32 formats keep the exact kernel (nui_k_tsdf.cu).  This file is compiled
// with contraction on.
//
// Work decomposition (HBM-bound by design): the volume is cut into tiles of 32 (x) x 8 (y)
// x 8 (z) voxels, one warp per tile, lane = x, so every row a warp touches is one
// contiguous 64 B run of the tsdf plane and 32 B of the weight plane.  A warp first culls
// its tile with eight lanes projecting the tile's corners: tiles entirely behind the
// camera, projecting outside the image, or farther from the camera than the largest ray
// depth of the pixel tiles they project to plus the truncation are skipped without a
// memory access.  Surviving tiles run two passes over their 64 rows: the update (only
// updated voxels are read and written), then -- for the 8^3 bricks of the tile that had
// an update -- the brick classification that the exact path leaves to k_brick_summary
// (every voxel of such a brick read once; the voxels just written come back from L2).
#include "nui_device.cuh"

namespace nui {

template <int FMT>
__device__ __forceinline__ void fast_load(const SessionDesc& s, size_t i, float& F, int& W) {
  if (FMT == 2) {
    F = __half2float(reinterpret_cast<const __half*>(s.vol)[i]);
    W = s.wvol[i];
  } else {
    const __half2 v = reinterpret_cast<const __half2*>(s.vol)[i];
    F = __low2float(v);
    W = (int)__high2float(v);
  }
}

template <int FMT>
__global__ void __launch_bounds__(32 * kFastWarps) k_integrate_fast(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind < 0 || s.fmt != FMT || !s.ts->integrate) return;
  const int rx = s.res[0], ry = s.res[1], rz = s.res[2];
  const int ntx = (rx + 31) >> 5, nty = (ry + 7) >> 3, ntz = (rz + 7) >> 3;
  const int ntiles = ntx * nty * ntz;
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * kFastWarps;
  const DevXform& m = s.ts->xf;
  float Ri[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) Ri[k] = m.R_inv[k];
  const float t0 = m.t[0], t1 = m.t[1], t2 = m.t[2];
  const float c0 = s.cell[0], c1 = s.cell[1], c2 = s.cell[2];
  const float fx = s.cam.fx, fy = s.cam.fy, ccx = s.cam.cx, ccy = s.cam.cy;
  const int W = s.W, H = s.H;
  const float fW = (float)W, fH = (float)H;
  const float trunc = s.trunc, tinv = 1.f / trunc;
  const float dmax = __int_as_float(s.ts->dmax_bits);
  const int ptx = (W + kTile - 1) / kTile;
  const float* __restrict__ depth = s.dscaled;
  const size_t slice = (size_t)rx * ry;
  const int hx = rx / 2, hy = ry / 2;
  unsigned int touched_total = 0, bricks = 0;

  for (int tile = blockIdx.x * kFastWarps + (threadIdx.x >> 5); tile < ntiles; tile += nwarps) {
    const int x0 = (tile % ntx) << 5, y0 = ((tile / ntx) % nty) << 3, z0 = (tile / (ntx * nty)) << 3;
    const int xn = min(32, rx - x0), yn = min(8, ry - y0), zn = min(8, rz - z0);
    // ---- cull: the tile's corner voxel centres, relative to the camera, in camera space
    bool skip;
    {
      const int cx = x0 + ((lane & 1) ? xn - 1 : 0), cy = y0 + ((lane & 2) ? yn - 1 : 0),
                cz = z0 + ((lane & 4) ? zn - 1 : 0);
      const float gx = ((float)(cx - hx) + 0.5f) * c0 - t0;
      const float gy = ((float)(cy - hy) + 0.5f) * c1 - t1;
      const float gz = ((float)cz + 0.5f) * c2 - t2;
      const float vx = Ri[0] * gx + Ri[1] * gy + Ri[2] * gz;
      const float vy = Ri[3] * gx + Ri[4] * gy + Ri[5] * gz;
      const float vz = Ri[6] * gx + Ri[7] * gy + Ri[8] * gz;
      const bool corner = lane < 8;
      const unsigned front = __ballot_sync(0xffffffffu, corner && vz > 1e-6f) & 0xffu;
      float u0 = 0.f, u1 = fW - 1.f, w0 = 0.f, w1 = fH - 1.f;
      if (front == 0u) {
        skip = true;  // the whole tile is behind the camera
      } else {
        if (front == 0xffu) {  // in front: the projections' bounding box bounds the tile's
          const float iz = __fdividef(1.f, vz);
          float ua = corner ? fx * vx * iz + ccx : 3.4e38f, ub = corner ? ua : -3.4e38f;
          float va = corner ? fy * vy * iz + ccy : 3.4e38f, vb = corner ? va : -3.4e38f;
#pragma unroll
          for (int o = 1; o < 8; o <<= 1) {
            ua = fminf(ua, __shfl_xor_sync(0xffffffffu, ua, o));
            ub = fmaxf(ub, __shfl_xor_sync(0xffffffffu, ub, o));
            va = fminf(va, __shfl_xor_sync(0xffffffffu, va, o));
            vb = fmaxf(vb, __shfl_xor_sync(0xffffffffu, vb, o));
          }
          ua = __shfl_sync(0xffffffffu, ua, 0);
          ub = __shfl_sync(0xffffffffu, ub, 0);
          va = __shfl_sync(0xffffffffu, va, 0);
          vb = __shfl_sync(0xffffffffu, vb, 0);
          u0 = fmaxf(ua - 1.f, 0.f);
          u1 = fminf(ub + 1.f, fW - 1.f);
          w0 = fmaxf(va - 1.f, 0.f);
          w1 = fminf(vb + 1.f, fH - 1.f);
        }
        skip = !(u0 <= u1 && w0 <= w1);
        if (!skip) {
          // largest ray depth over the pixel tiles of the footprint (the frame's largest
          // when the footprint spans more than 64 of them); 0 = no valid depth there
          const int a0 = (int)u0 / kTile, a1 = (int)u1 / kTile, b0 = (int)w0 / kTile, b1 = (int)w1 / kTile;
          const int na = a1 - a0 + 1, nt = na * (b1 - b0 + 1);
          float mx = 0.f;
          if (nt <= 64) {
            for (int k = lane; k < nt; k += 32) mx = fmaxf(mx, __ldg(s.tile_max + (b0 + k / na) * ptx + a0 + k % na));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
          } else {
            mx = dmax;
          }
          // nearest distance from the camera to the tile's box of voxel centres
          const float bx0 = ((float)(x0 - hx) + 0.5f) * c0 - t0, bx1 = bx0 + (float)(xn - 1) * c0;
          const float by0 = ((float)(y0 - hy) + 0.5f) * c1 - t1, by1 = by0 + (float)(yn - 1) * c1;
          const float bz0 = ((float)z0 + 0.5f) * c2 - t2, bz1 = bz0 + (float)(zn - 1) * c2;
          const float dx = fmaxf(fmaxf(bx0, -bx1), 0.f), dy = fmaxf(fmaxf(by0, -by1), 0.f),
                      dz = fmaxf(fmaxf(bz0, -bz1), 0.f);
          const float dmin = sqrtf(dx * dx + dy * dy + dz * dz);
          skip = !(mx > 0.f) || dmin > mx + trunc + 1e-3f * (1.f + dmin);
        }
      }
    }
    if (skip) continue;

    // ---- update pass: rows (y, z) of the tile, four at a time, lane = x
    const int x = x0 + lane;
    const bool xin = lane < xn;
    const float gx = ((float)(x - hx) + 0.5f) * c0 - t0;
    const float ax = Ri[0] * gx, ay = Ri[3] * gx, az = Ri[6] * gx;
    const float gx2 = gx * gx;
    unsigned int touched = 0;  // voxels this lane updated in the tile
#pragma unroll 1
    for (int r0 = 0; r0 < 64; r0 += 4) {
      float sdf[4];
      int pix[4];
      bool ok[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = r0 + q, yy = r & 7, zz = r >> 3;
        ok[q] = false;
        pix[q] = 0;
        sdf[q] = 0.f;
        if (!xin || yy >= yn || zz >= zn) continue;
        const float gy = ((float)(y0 + yy - hy) + 0.5f) * c1 - t1;
        const float gz = ((float)(z0 + zz) + 0.5f) * c2 - t2;
        const float vz = az + Ri[7] * gy + Ri[8] * gz;
        if (!(vz > 0.f)) continue;
        const float iz = __fdividef(1.f, vz);
        const float vx = ax + Ri[1] * gy + Ri[2] * gz;
        const float vy = ay + Ri[4] * gy + Ri[5] * gz;
        const int px = __float2int_rn(fx * vx * iz + ccx), py = __float2int_rn(fy * vy * iz + ccy);
        if (px < 0 || py < 0 || px >= W || py >= H) continue;
        const float r2 = gx2 + gy * gy + gz * gz;
        const float Dp = __ldg(depth + py * W + px);
        const float sd = Dp - r2 * rsqrtf(r2);
        if (!(sd >= -trunc)) continue;  // also false for a NaN depth
        ok[q] = true;
        sdf[q] = sd;
        pix[q] = py * W + px;
      }
      size_t idx[4];
      float F[4];
      int Wt[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = r0 + q;
        idx[q] = (size_t)x + (size_t)rx * (size_t)(y0 + (r & 7)) + slice * (size_t)(z0 + (r >> 3));
        if (ok[q]) fast_load<FMT>(s, idx[q], F[q], Wt[q]);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (!ok[q]) continue;
        const float tsdf = fminf(1.0f, sdf[q] * tinv);
        const float tn = __fdividef(F[q] * (float)Wt[q] + tsdf, (float)(Wt[q] + 1));
        const int wn = min(Wt[q] + 1, 128);
        if (FMT == 2) {
          reinterpret_cast<__half*>(s.vol)[idx[q]] = __float2half_rn(tn);
          s.wvol[idx[q]] = (uint8_t)wn;
        } else {
          reinterpret_cast<__half2*>(s.vol)[idx[q]] = __floats2half2_rn(tn, (float)wn);
        }
        touched += 1u;
        if (s.cvol && s.bgra && fabsf(sdf[q]) < trunc) {
          const uchar4 nc = reinterpret_cast<const uchar4*>(s.bgra)[pix[q]];
          if (nc.w != 0) {
            // the reference's arithmetic exactly (no product to contract, IEEE division):
            // colours agree bit for bit wherever the same voxels are updated
            const uchar4 vc = s.cvol[idx[q]];
            const float den = (float)vc.w + 1.f;
            uchar4 o;
            o.x = (unsigned char)fminf(fmaxf(((float)(vc.x * vc.w) + (float)nc.x) / den, 0.f), 255.f);
            o.y = (unsigned char)fminf(fmaxf(((float)(vc.y * vc.w) + (float)nc.y) / den, 0.f), 255.f);
            o.z = (unsigned char)fminf(fmaxf(((float)(vc.z * vc.w) + (float)nc.z) / den, 0.f), 255.f);
            o.w = min((unsigned char)s.max_cw, (unsigned char)(vc.w + 1));
            s.cvol[idx[q]] = o;
          }
        }
      }
    }
    touched_total += touched;
    // ---- classification of the bricks (lanes 8b .. 8b+7) that had an update
    const unsigned upd = __ballot_sync(0xffffffffu, touched != 0u);
    if (upd == 0u || !s.occ) continue;
    const bool mine = (upd >> (lane & ~7)) & 0xffu;
    bool weighted = false, unweighted = false, nonpos = false;
    if (mine && xin) {
#pragma unroll 4
      for (int r = 0; r < 64; ++r) {
        const int yy = r & 7, zz = r >> 3;
        if (yy >= yn || zz >= zn) continue;
        float F;
        int Wt;
        fast_load<FMT>(s, (size_t)x + (size_t)rx * (size_t)(y0 + yy) + slice * (size_t)(z0 + zz), F, Wt);
        if (Wt > 0) {
          weighted = true;
          if (!(F > 0.f)) nonpos = true;
        } else {
          unweighted = true;
        }
      }
    }
    const unsigned bw = __ballot_sync(0xffffffffu, weighted), bu = __ballot_sync(0xffffffffu, unweighted),
                   bn = __ballot_sync(0xffffffffu, nonpos);
    if ((lane & 7) == 0 && mine && xin) {
      const unsigned g = 0xffu << lane;
      const uint8_t st = (bn & g) ? kBrickMixed : !(bw & g) ? kBrickEmpty : (bu & g) ? kBrickNoNeg : kBrickPositive;
      s.occ[occ_index(s, x, y0, z0)] = st;
      ++bricks;
    }
    if (lane == 0 && s.occ2) s.occ2[occ2_index(s, x0, y0, z0)] = kSuperDirty;
  }
  const unsigned int t = __reduce_add_sync(0xffffffffu, touched_total);
  const unsigned int b = __reduce_add_sync(0xffffffffu, bricks);
  if (lane == 0 && t) atomicAdd(&s.ts->touched, (unsigned long long)t);
  if (lane == 0 && b) atomicAdd(&s.ts->bricks, (unsigned long long)b);
}

template __global__ void k_integrate_fast<2>(const SessionDesc*);
template __global__ void k_integrate_fast<3>(const SessionDesc*);

}  // namespace nui
