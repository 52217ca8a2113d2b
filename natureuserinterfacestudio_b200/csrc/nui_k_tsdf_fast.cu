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
// Work decomposition: the volume is cut into tiles of 32 (x) x 8 (y) x 8 (z) voxels.
// k_integrate_cull tests every tile on one thread: tiles entirely behind the camera,
// projecting outside the image, or farther from the camera than the largest ray depth of
// the pixel tiles they project to plus the truncation are dropped without a memory access;
// the kept ones are appended to the session's tile list.  k_integrate_fast deals the listed
// tiles round robin to its warps (the kept tiles cluster in the frustum, so a fixed
// tile-to-warp map would leave most warps idle), lane = x: a tile's depth pixels and voxel
// rows are brought into the warp's shared memory by asynchronous copies, all 64 rows at
// once, then updated from there (only updated voxels are written back), and the 8^3 bricks
// of the tile that had an update are re-classified from the same shared copy -- the brick
// summary the exact path leaves to k_brick_summary.
#include "nui_device.cuh"

namespace nui {

// Tile culling, one thread per tile: a tile can hold an updated voxel only if part of it
// is in front of the camera, projects into the image, and is no farther from the camera
// than the largest ray depth of the pixel tiles it projects to plus the truncation.  The
// corners' camera coordinates follow from one corner and the tile's three edge vectors.
template <int FMT>
__global__ void __launch_bounds__(256) k_integrate_cull(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind < 0 || s.fmt != FMT || !s.ts->integrate) return;
  const int rx = s.res[0], ry = s.res[1], rz = s.res[2];
  const int ntx = (rx + 31) >> 5, nty = (ry + 7) >> 3, ntz = (rz + 7) >> 3;
  const int tile = blockIdx.x * blockDim.x + threadIdx.x;
  if (tile >= ntx * nty * ntz) return;
  const DevXform& m = s.ts->xf;
  const float* Ri = m.R_inv;
  const float c0 = s.cell[0], c1 = s.cell[1], c2 = s.cell[2];
  const int x0 = (tile % ntx) << 5, y0 = ((tile / ntx) % nty) << 3, z0 = (tile / (ntx * nty)) << 3;
  const int xn = min(32, rx - x0), yn = min(8, ry - y0), zn = min(8, rz - z0);
  const float gx = ((float)(x0 - rx / 2) + 0.5f) * c0 - m.t[0];
  const float gy = ((float)(y0 - ry / 2) + 0.5f) * c1 - m.t[1];
  const float gz = ((float)z0 + 0.5f) * c2 - m.t[2];
  const float ex = (float)(xn - 1) * c0, ey = (float)(yn - 1) * c1, ez = (float)(zn - 1) * c2;
  const float3 v0 = f3(Ri[0] * gx + Ri[1] * gy + Ri[2] * gz, Ri[3] * gx + Ri[4] * gy + Ri[5] * gz,
                       Ri[6] * gx + Ri[7] * gy + Ri[8] * gz);
  const float3 dx = f3(Ri[0] * ex, Ri[3] * ex, Ri[6] * ex), dy = f3(Ri[1] * ey, Ri[4] * ey, Ri[7] * ey),
               dz = f3(Ri[2] * ez, Ri[5] * ez, Ri[8] * ez);
  const float fx = s.cam.fx, fy = s.cam.fy, ccx = s.cam.cx, ccy = s.cam.cy;
  const float fW = (float)s.W, fH = (float)s.H;
  float u0 = 3.4e38f, u1 = -3.4e38f, w0 = 3.4e38f, w1 = -3.4e38f;
  int front = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    float3 v = v0;
    if (k & 1) v = add3(v, dx);
    if (k & 2) v = add3(v, dy);
    if (k & 4) v = add3(v, dz);
    if (v.z > 1e-6f) {
      ++front;
      const float iz = __fdividef(1.f, v.z);
      const float u = fx * v.x * iz + ccx, w = fy * v.y * iz + ccy;
      u0 = fminf(u0, u);
      u1 = fmaxf(u1, u);
      w0 = fminf(w0, w);
      w1 = fmaxf(w1, w);
    }
  }
  bool keep = front > 0;
  if (keep) {
    if (front < 8) {  // straddles the camera plane: the footprint is unbounded
      u0 = 0.f, u1 = fW - 1.f, w0 = 0.f, w1 = fH - 1.f;
    } else {
      u0 = fmaxf(u0 - 1.f, 0.f), u1 = fminf(u1 + 1.f, fW - 1.f);
      w0 = fmaxf(w0 - 1.f, 0.f), w1 = fminf(w1 + 1.f, fH - 1.f);
    }
    keep = u0 <= u1 && w0 <= w1;
  }
  if (keep) {
    // largest ray depth over the pixel tiles of the footprint (the frame's largest when the
    // footprint spans more than 64 of them); 0 = no valid depth there
    const int ptx = (s.W + kTile - 1) / kTile;
    const int a0 = (int)u0 / kTile, a1 = (int)u1 / kTile, b0 = (int)w0 / kTile, b1 = (int)w1 / kTile;
    float mx = 0.f;
    if ((a1 - a0 + 1) * (b1 - b0 + 1) <= 64) {
      for (int b = b0; b <= b1; ++b)
        for (int a = a0; a <= a1; ++a) mx = fmaxf(mx, __ldg(s.tile_max + b * ptx + a));
    } else {
      mx = __int_as_float(s.ts->dmax_bits);
    }
    // nearest distance from the camera to the tile's box of voxel centres
    const float bx = fmaxf(fmaxf(gx, -(gx + ex)), 0.f), by = fmaxf(fmaxf(gy, -(gy + ey)), 0.f),
                bz = fmaxf(fmaxf(gz, -(gz + ez)), 0.f);
    const float dmin = sqrtf(bx * bx + by * by + bz * bz);
    keep = mx > 0.f && !(dmin > mx + s.trunc + 1e-3f * (1.f + dmin));
  }
  // append the kept tile to the session's list (one atomic per warp)
  const unsigned act = __activemask(), kept = __ballot_sync(act, keep);
  const int lane = threadIdx.x & 31;
  unsigned base = 0;
  if (kept && lane == __ffs(act) - 1) base = atomicAdd(&s.ts->fast_count, (unsigned)__popc(kept));
  base = __shfl_sync(act, base, __ffs(act) - 1);
  if (keep) s.fast_tiles[base + __popc(kept & ((1u << lane) - 1u))] = (unsigned)tile;
}

// Asynchronous copies global -> shared (cp.async): the data lands in shared memory without
// passing through registers, so a lane can have a whole tile's requests in flight.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
               "l"(gmem));
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(smem)),
               "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Shared memory of one warp (kFastWarpSmem bytes): the depth each voxel of the tile
// projects to (NaN: none), and the tile's voxels (64 rows of 32).
template <int FMT>
struct FastTileSmem {
  float* dep;  // [64][32]
  __half* fh;  // F16_U8: [64][32] tsdf
  uint8_t* wb; // F16_U8: [64][32] weight
  __half2* f2; // F16_F16: [64][32] (tsdf, weight)
  __device__ explicit FastTileSmem(unsigned char* base) {
    dep = reinterpret_cast<float*>(base);
    fh = reinterpret_cast<__half*>(base + 64 * 32 * 4);
    wb = base + 64 * 32 * 4 + 64 * 32 * 2;
    f2 = reinterpret_cast<__half2*>(base + 64 * 32 * 4);
  }
  __device__ __forceinline__ void get(int i, float& F, int& W) const {
    if (FMT == 2) {
      F = __half2float(fh[i]);
      W = wb[i];
    } else {
      const __half2 v = f2[i];
      F = __low2float(v);
      W = (int)__high2float(v);
    }
  }
};

// The tiles the cull listed, dealt round robin to the warps.  Per tile, in three phases:
//  1. every row of the tile is requested at once: each lane projects its voxel and copies
//     the depth pixel it lands on into shared memory (NaN when it lands on none), and the
//     row's voxels are copied as 16-byte pieces (4 + 2 lanes for FP16 + u8, 8 for FP16 +
//     FP16) -- 64 rows of requests in flight, one round trip for the tile;
//  2. the update from shared memory: sd = depth - |voxel - camera|, the running average,
//     stores of the updated voxels (and their new values into the shared copy);
//  3. the 8^3 bricks of the tile that had an update are re-classified from the shared copy.
// Rows that are not whole (a tile past the volume's x end) or not 16-byte aligned (x sizes
// not a multiple of 16) are loaded lane by lane instead.
template <int FMT>
__global__ void __launch_bounds__(32 * kFastWarps, 3) k_integrate_fast(const SessionDesc* __restrict__ descs) {
  extern __shared__ __align__(16) unsigned char fast_smem[];
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind < 0 || s.fmt != FMT || !s.ts->integrate) return;
  const int rx = s.res[0], ry = s.res[1], rz = s.res[2];
  const int ntx = (rx + 31) >> 5, nty = (ry + 7) >> 3;
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * kFastWarps;
  const FastTileSmem<FMT> sm(fast_smem + (threadIdx.x >> 5) * kFastWarpSmem);
  const DevXform& m = s.ts->xf;
  float Ri[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) Ri[k] = m.R_inv[k];
  const float t0 = m.t[0], t1 = m.t[1], t2 = m.t[2];
  const float c0 = s.cell[0], c1 = s.cell[1], c2 = s.cell[2];
  const float fx = s.cam.fx, fy = s.cam.fy, ccx = s.cam.cx, ccy = s.cam.cy;
  const int W = s.W, H = s.H;
  const float trunc = s.trunc, tinv = 1.f / trunc;
  const float* __restrict__ depth = s.dscaled;
  const size_t slice = (size_t)rx * ry;
  const int hx = rx / 2, hy = ry / 2;
  // whole rows start 16-byte aligned in every plane when the x size is a multiple of 16
  const bool aligned = (rx & 15) == 0 && ((reinterpret_cast<uintptr_t>(s.vol) | reinterpret_cast<uintptr_t>(s.wvol)) & 15) == 0;
  unsigned int touched_total = 0, bricks = 0;

  const unsigned count = *(volatile const unsigned*)&s.ts->fast_count;
  for (unsigned li = blockIdx.x * kFastWarps + (threadIdx.x >> 5); li < count; li += (unsigned)nwarps) {
    const int tile = (int)__ldg(s.fast_tiles + li);
    const int x0 = (tile % ntx) << 5, y0 = ((tile / ntx) % nty) << 3, z0 = (tile / (ntx * nty)) << 3;
    const int xn = min(32, rx - x0), yn = min(8, ry - y0), zn = min(8, rz - z0);
    const int x = x0 + lane;
    const bool xin = lane < xn;
    const bool whole = aligned && xn == 32;
    const float gx = ((float)(x - hx) + 0.5f) * c0 - t0;
    const float gy0 = ((float)(y0 - hy) + 0.5f) * c1 - t1;
    const float3 ey = f3(Ri[1] * c1, Ri[4] * c1, Ri[7] * c1);  // camera step of one y row

    // ---- 1. requests: voxel rows and depth pixels of the whole tile
    __syncwarp();  // the previous tile's shared copy is no longer read
    if (whole) {
      // the rows' 16-byte pieces dealt over the lanes (FP16 + u8: 4 tsdf + 2 weight pieces
      // a row; FP16 + FP16: 8 pieces), no lane idle and no branch per row
      constexpr int kPieces = FMT == 2 ? 6 : 8;
      const int nrow = zn * 8;  // rows of slices past the volume's y end are skipped below
      for (int j = lane; j < nrow * kPieces; j += 32) {
        const int r = j / kPieces, piece = j - r * kPieces, yy = r & 7, zz = r >> 3;
        if (yy >= yn) continue;
        const size_t rb = (size_t)x0 + (size_t)rx * (size_t)(y0 + yy) + slice * (size_t)(z0 + zz);
        if (FMT == 2) {
          if (piece < 4) cp_async16(sm.fh + r * 32 + piece * 8, reinterpret_cast<const __half*>(s.vol) + rb + piece * 8);
          else cp_async16(sm.wb + r * 32 + (piece - 4) * 16, s.wvol + rb + (piece - 4) * 16);
        } else {
          cp_async16(sm.f2 + r * 32 + piece * 4, reinterpret_cast<const __half2*>(s.vol) + rb + piece * 4);
        }
      }
    }
    const unsigned dep_s = (unsigned)__cvta_generic_to_shared(sm.dep + lane);  // this lane's column
#pragma unroll 1
    for (int zz = 0; zz < zn; ++zz) {
      const float gz = ((float)(z0 + zz) + 0.5f) * c2 - t2;
      float3 v = f3(Ri[0] * gx + Ri[1] * gy0 + Ri[2] * gz, Ri[3] * gx + Ri[4] * gy0 + Ri[5] * gz,
                    Ri[6] * gx + Ri[7] * gy0 + Ri[8] * gz);
      const size_t zbase = (size_t)x0 + (size_t)rx * (size_t)y0 + slice * (size_t)(z0 + zz);
#pragma unroll 2
      for (int yy = 0; yy < yn; ++yy) {
        const int r = zz * 8 + yy;
        bool got = false;
        if (xin && v.z > 0.f) {
          const float iz = __fdividef(1.f, v.z);
          // exact ties round up, as OpenCL's round(): they are frequent (pixel centres and
          // voxel centres sit on rational grids), and half-to-even would split them
          const int px = round_half_up(fx * v.x * iz + ccx), py = round_half_up(fy * v.y * iz + ccy);
          if (px >= 0 && py >= 0 && px < W && py < H) {
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dep_s + (unsigned)r * 128u),
                         "l"(depth + py * W + px));
            got = true;
          }
        }
        if (!got) sm.dep[r * 32 + lane] = __int_as_float(0x7fffffff);
        if (!whole && xin) {
          const size_t rb = zbase + (size_t)rx * yy;  // the row's first voxel
          if (FMT == 2) {
            sm.fh[r * 32 + lane] = reinterpret_cast<const __half*>(s.vol)[rb + lane];
            sm.wb[r * 32 + lane] = s.wvol[rb + lane];
          } else {
            sm.f2[r * 32 + lane] = reinterpret_cast<const __half2*>(s.vol)[rb + lane];
          }
        }
        v = add3(v, ey);
      }
    }
    cp_async_wait_all();
    __syncwarp();

    // ---- 2. the update, from shared memory
    unsigned int touched = 0;  // voxels this lane updated in the tile
    const float gx2 = gx * gx;
    if (xin) {
#pragma unroll 1
      for (int zz = 0; zz < zn; ++zz) {
        const float gz = ((float)(z0 + zz) + 0.5f) * c2 - t2;
        const float gz2 = gz * gz;
        const size_t zbase = (size_t)x + (size_t)rx * (size_t)y0 + slice * (size_t)(z0 + zz);
#pragma unroll 2
        for (int yy = 0; yy < yn; ++yy) {
          const int r = zz * 8 + yy, i = r * 32 + lane;
          const float gy = gy0 + (float)yy * c1;
          const float r2 = gx2 + gy * gy + gz2;
          const float sd = sm.dep[i] - r2 * rsqrtf(r2);
          if (!(sd >= -trunc)) continue;  // also a voxel without a depth (NaN)
          float F;
          int Wt;
          sm.get(i, F, Wt);
          const size_t vi = zbase + (size_t)rx * yy;
          const float tsdf = fminf(1.0f, sd * tinv);
          const float tn = __fdividef(F * (float)Wt + tsdf, (float)(Wt + 1));
          const int wn = min(Wt + 1, 128);
          if (FMT == 2) {
            const __half h = __float2half_rn(tn);
            reinterpret_cast<__half*>(s.vol)[vi] = h;
            s.wvol[vi] = (uint8_t)wn;
            sm.fh[i] = h;
            sm.wb[i] = (uint8_t)wn;
          } else {
            const __half2 h = __floats2half2_rn(tn, (float)wn);
            reinterpret_cast<__half2*>(s.vol)[vi] = h;
            sm.f2[i] = h;
          }
          touched += 1u;
          if (s.cvol && s.bgra && fabsf(sd) < trunc) {
            // the voxel's pixel again, by the same operations as in the request phase
            float3 v = f3(Ri[0] * gx + Ri[1] * gy0 + Ri[2] * gz, Ri[3] * gx + Ri[4] * gy0 + Ri[5] * gz,
                          Ri[6] * gx + Ri[7] * gy0 + Ri[8] * gz);
            for (int k = 0; k < yy; ++k) v = add3(v, ey);
            const float iz = __fdividef(1.f, v.z);
            const int px = round_half_up(fx * v.x * iz + ccx), py = round_half_up(fy * v.y * iz + ccy);
            const bool inimg = px >= 0 && py >= 0 && px < W && py < H;  // (a contraction may differ)
            const uchar4 nc = inimg ? reinterpret_cast<const uchar4*>(s.bgra)[py * W + px] : make_uchar4(0, 0, 0, 0);
            if (nc.w != 0) {
              // the reference's arithmetic exactly (no product to contract, IEEE division):
              // colours agree bit for bit wherever the same voxels are updated
              const uchar4 vc = s.cvol[vi];
              const float den = (float)vc.w + 1.f;
              uchar4 o;
              o.x = (unsigned char)fminf(fmaxf(((float)(vc.x * vc.w) + (float)nc.x) / den, 0.f), 255.f);
              o.y = (unsigned char)fminf(fmaxf(((float)(vc.y * vc.w) + (float)nc.y) / den, 0.f), 255.f);
              o.z = (unsigned char)fminf(fmaxf(((float)(vc.z * vc.w) + (float)nc.z) / den, 0.f), 255.f);
              o.w = min((unsigned char)s.max_cw, (unsigned char)(vc.w + 1));
              s.cvol[vi] = o;
            }
          }
        }
      }
    }
    touched_total += touched;
    // ---- 3. classification of the bricks (lanes 8b .. 8b+7) that had an update, from the
    // shared copy (which holds the values just written)
    const unsigned upd = __ballot_sync(0xffffffffu, touched != 0u);
    if (upd == 0u || !s.occ) continue;
    const bool mine = (upd >> (lane & ~7)) & 0xffu;
    bool weighted = false, unweighted = false, nonpos = false;
    if (mine && xin) {
#pragma unroll 1
      for (int zz = 0; zz < zn; ++zz)
#pragma unroll 4
        for (int yy = 0; yy < yn; ++yy) {
          float F;
          int Wt;
          sm.get((zz * 8 + yy) * 32 + lane, F, Wt);
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
  // the session's last block to finish empties the list for the next integration (every
  // block has read the count by then)
  __syncthreads();
  if (threadIdx.x == 0 && atomicAdd(&s.ts->fast_done, 1u) == gridDim.x - 1) {
    s.ts->tiles += count;
    s.ts->fast_count = 0u;
    s.ts->fast_done = 0u;
  }
}

template __global__ void k_integrate_cull<2>(const SessionDesc*);
template __global__ void k_integrate_cull<3>(const SessionDesc*);
template __global__ void k_integrate_fast<2>(const SessionDesc*);
template __global__ void k_integrate_fast<3>(const SessionDesc*);

}  // namespace nui
