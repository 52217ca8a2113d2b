// Dense TSDF integration (integrateTsdfVolumeKernel, tsdfVolume.cl:31-190) and volume reset
// (initializeVolume, tsdfVolume.cl:192-211).
//
// Layout: voxel (x, y, z) at x + rx*(y + ry*z), so the 32 lanes of a warp (consecutive x)
// touch one contiguous 128-256 B run of each z slice: every access is coalesced.  The
// reference keeps z fastest and loops z inside a thread, which strides a warp by rz voxels.
//
// Arithmetic: the reference advances the camera-space coordinates of a column
// incrementally along z (v_x += R_inv[2]*cell*fx, ...); rounding of that running sum
// decides which pixel a voxel projects to, so each thread replays the same additions.
// A thread owns one column and one chunk of z: it first replays the additions of the
// z values below its chunk (4 float adds per slice, no memory traffic), then integrates
// its chunk, evaluating the projections of kZUnroll slices before it issues their loads
// so that several voxel reads are in flight per thread.
#include "nui_device.cuh"

namespace nui {

constexpr int kTsdfThreads = 256;
constexpr int kZUnroll = 4;
constexpr int kChunk = 16;  // z slices per occlusion test

template <int FMT>
__global__ void __launch_bounds__(kTsdfThreads, 4) k_integrate(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind < 0 || s.fmt != FMT || !s.ts->integrate) return;
  const int rx = s.res[0], ry = s.res[1], rz = s.res[2];
  const int zchunks = s.zchunks;
  const long ncol = (long)rx * ry;
  const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= ncol * zchunks) return;
  const int chunk = (int)(tid / ncol);
  const long col = tid - (long)chunk * ncol;
  const int vx = (int)(col % rx), vy = (int)(col / rx);
  const int zlen = (rz + zchunks - 1) / zchunks;
  const int z0 = chunk * zlen, z1 = min(rz, z0 + zlen);

  const DevXform& m = s.ts->xf;
  const float* Ri = m.R_inv;
  const float c0 = s.cell[0], c1 = s.cell[1], c2 = s.cell[2];
  const float vgx = ((float)(vx - rx / 2) + 0.5f) * c0 - m.t[0];
  const float vgy = ((float)(vy - ry / 2) + 0.5f) * c1 - m.t[1];
  const float vgz0 = (0.5f) * c2 - m.t[2];
  const float* __restrict__ zt_vgz = s.ztab;            // v_g_z after z additions
  const float* __restrict__ zt_zs = s.ztab + rz + 1;    // z_scaled after z additions
  const float part = vgx * vgx + vgy * vgy;
  const float fx = s.cam.fx, fy = s.cam.fy, ccx = s.cam.cx, ccy = s.cam.cy;
  float v_x = (Ri[0] * vgx + Ri[1] * vgy + Ri[2] * vgz0) * fx;
  float v_y = (Ri[3] * vgx + Ri[4] * vgy + Ri[5] * vgz0) * fy;
  const float v_z = (Ri[6] * vgx + Ri[7] * vgy + Ri[8] * vgz0);
  const float trunc = s.trunc;
  const float tinv = 1.f / trunc;
  const float dx = Ri[2] * c2 * fx;
  const float dy = Ri[5] * c2 * fy;
  const float r8 = Ri[8];
  const int W = s.W, H = s.H;
  // Conservative z interval of this column: only voxels whose exact projection can land
  // inside the image (1.5 px margin) in front of the camera, and whose distance from the
  // camera can be within the frame's largest ray length + trunc, can be updated.  The
  // bounds come from the same affine recurrences the exact test uses, evaluated in
  // double; one voxel of margin on each side absorbs the float rounding of the running
  // sums, so every voxel outside the interval also fails the exact test below.
  int kb = z0, ke = z1;
  {
    const double X0 = v_x, dX = dx, Y0 = v_y, dY = dy, Z0 = v_z, dZ = (double)r8 * (double)c2;
    double lo = 0.0, hi = (double)(rz - 1);
    bool empty = false;
    auto ge = [&](double a, double b) {  // a + b k >= 0
      if (b > 0) lo = fmax(lo, -a / b);
      else if (b < 0) hi = fmin(hi, -a / b);
      else if (a < 0) empty = true;
    };
    const double m = 1.5;
    ge(X0 + ((double)ccx + m) * Z0, dX + ((double)ccx + m) * dZ);
    ge(-(X0 + ((double)ccx - (double)W - m) * Z0), -(dX + ((double)ccx - (double)W - m) * dZ));
    ge(Y0 + ((double)ccy + m) * Z0, dY + ((double)ccy + m) * dZ);
    ge(-(Y0 + ((double)ccy - (double)H - m) * Z0), -(dY + ((double)ccy - (double)H - m) * dZ));
    ge(Z0, dZ);
    const double rmax = (double)__int_as_float(s.ts->dmax_bits) + (double)trunc + 2.0 * (double)c2;
    const double s2 = rmax * rmax - (double)part;
    if (s2 < 0) {
      empty = true;
    } else {
      const double sr = sqrt(s2);
      ge((double)vgz0 + sr, (double)c2);
      ge(sr - (double)vgz0, -(double)c2);
    }
    if (empty || lo > hi) {
      kb = ke = z0;
    } else {
      kb = max(z0, (int)floor(lo) - 1);
      ke = min(z1, (int)ceil(hi) + 2);
      if (ke < kb) ke = kb;
    }
  }
  if (kb >= ke) return;  // nothing to update in this column chunk
  // v_x and v_y depend on the column: replay their additions below the interval
#pragma unroll 4
  for (int z = 0; z < kb; ++z) {
    v_x += dx;
    v_y += dy;
  }
  const float fW = (float)W, fH = (float)H;
  const float* __restrict__ depth = s.dscaled;
  const size_t slice = (size_t)rx * ry;
  const int ntx = (W + kTile - 1) / kTile, nty = (H + kTile - 1) / kTile;
  unsigned int touched = 0;

  for (int zc = kb; zc < ke; zc += kChunk) {
    const int zend = min(zc + kChunk, ke);
    // Occlusion test of the chunk: bound the pixels its voxels project to (the segment
    // between the projections of its end voxels, 2 px margin) and the largest ray length
    // over those pixels' tiles; if even the chunk's nearest voxel is farther than that
    // plus trunc, no voxel of the chunk passes sdf >= -trunc.
    bool skip = false;
    {
      // v_x, v_y and the table entries all stand at slice zc here
      const float k0 = 0.f, k1 = (float)(zend - 1 - zc);
      const float zs = zt_zs[zc], vgz = zt_vgz[zc];
      const float za = v_z + r8 * (zs + k0 * c2), zb2 = v_z + r8 * (zs + k1 * c2);
      if (za > 1e-3f && zb2 > 1e-3f) {
        const float ua = (v_x + k0 * dx) / za + ccx, ub = (v_x + k1 * dx) / zb2 + ccx;
        const float va = (v_y + k0 * dy) / za + ccy, vb = (v_y + k1 * dy) / zb2 + ccy;
        const float u0 = fmaxf(fminf(ua, ub) - 2.f, 0.f), u1 = fminf(fmaxf(ua, ub) + 2.f, fW - 1.f);
        const float w0_ = fmaxf(fminf(va, vb) - 2.f, 0.f), w1 = fminf(fmaxf(va, vb) + 2.f, fH - 1.f);
        if (u0 > u1 || w0_ > w1) {
          skip = true;  // projects outside the image
        } else {
          const int tx0 = (int)u0 / kTile, tx1 = (int)u1 / kTile, ty0 = (int)w0_ / kTile, ty1 = (int)w1 / kTile;
          if ((tx1 - tx0 + 1) * (ty1 - ty0 + 1) <= 16 && tx1 < ntx && ty1 < nty) {
            float mx = 0.f;
            for (int ty = ty0; ty <= ty1; ++ty)
              for (int tx = tx0; tx <= tx1; ++tx) mx = fmaxf(mx, __ldg(s.tile_max + ty * ntx + tx));
            const float g0 = vgz + k0 * c2, g1 = vgz + k1 * c2;
            const float gz = (g0 <= 0.f && g1 >= 0.f) ? 0.f : fminf(fabsf(g0), fabsf(g1));
            const float dmin = sqrtf(part + gz * gz);
            skip = dmin > mx + trunc + 1e-3f * (1.f + dmin);
          }
        }
      }
    }
    if (skip) {
#pragma unroll 4
      for (int z = zc; z < zend; ++z) {
        v_x += dx;
        v_y += dy;
      }
      continue;
    }
    size_t idx = (size_t)vx + (size_t)rx * vy + slice * (size_t)zc;
    for (int zb = zc; zb < zend; zb += kZUnroll) {
      float sdf[kZUnroll];
      int pix[kZUnroll];
      bool ok[kZUnroll];
#pragma unroll
      for (int u = 0; u < kZUnroll; ++u) {
        ok[u] = false;
        pix[u] = 0;
        sdf[u] = 0.f;
        if (zb + u < zend) {
          const float zs = zt_zs[zb + u], vgz = zt_vgz[zb + u];
          const float inv_z = __frcp_rn(v_z + r8 * zs);
          if (!(inv_z < 0.f)) {
            const float px = roundf(v_x * inv_z + ccx);
            const float py = roundf(v_y * inv_z + ccy);
            if (px >= 0.f && py >= 0.f && px < fW && py < fH) {
              const int p = (int)py * W + (int)px;
              const float Dp = __ldg(depth + p);
              const float sd = Dp - sqrtf(vgz * vgz + part);
              if (!isnan(Dp) && sd >= -trunc) {
                ok[u] = true;
                sdf[u] = sd;
                pix[u] = p;
              }
            }
          }
          v_x += dx;
          v_y += dy;
        }
      }
      float F[kZUnroll];
      int Wt[kZUnroll];
#pragma unroll
      for (int u = 0; u < kZUnroll; ++u)
        if (ok[u]) Voxel<FMT>::load(s, idx + (size_t)u * slice, F[u], Wt[u]);
#pragma unroll
      for (int u = 0; u < kZUnroll; ++u) {
        if (!ok[u]) continue;
        const float tsdf = fminf(1.0f, sdf[u] * tinv);
        const float tn = (F[u] * (float)Wt[u] + tsdf) / (float)(Wt[u] + 1);
        const int wn = min(Wt[u] + 1, 128);
        const size_t vi = idx + (size_t)u * slice;
        Voxel<FMT>::store(s, vi, tn, wn);
        ++touched;
        if (s.occ) s.occ[occ_index(s, vx, vy, zb + u)] = kBrickDirty;
        if (s.cvol && s.bgra && fabsf(sdf[u]) < trunc) {
          const uchar4 nc = reinterpret_cast<const uchar4*>(s.bgra)[pix[u]];
          if (nc.w != 0) {
            const uchar4 vc = s.cvol[vi];
            const float wr = 1.f;
            const float nx = ((float)(vc.x * vc.w) + wr * (float)nc.x) / ((float)vc.w + wr);
            const float ny = ((float)(vc.y * vc.w) + wr * (float)nc.y) / ((float)vc.w + wr);
            const float nz = ((float)(vc.z * vc.w) + wr * (float)nc.z) / ((float)vc.w + wr);
            const unsigned char wnew = (unsigned char)(vc.w + 1);
            uchar4 o;
            o.x = (unsigned char)fminf(fmaxf(nx, 0.f), 255.f);
            o.y = (unsigned char)fminf(fmaxf(ny, 0.f), 255.f);
            o.z = (unsigned char)fminf(fmaxf(nz, 0.f), 255.f);
            o.w = min((unsigned char)s.max_cw, wnew);
            s.cvol[vi] = o;
          }
        }
      }
      idx += (size_t)kZUnroll * slice;
    }
  }
  // warp-aggregated count of voxels read-modify-written
  const unsigned int mask = __activemask();
  const unsigned int t = __reduce_add_sync(mask, touched);
  if ((int)(threadIdx.x & 31) == __ffs(mask) - 1 && t) atomicAdd(&s.ts->touched, (unsigned long long)t);
}

// Re-classifies the bricks integration touched.  A block looks at 1024 bricks: it first
// compacts the dirty ones into a shared list, then each warp classifies listed bricks,
// every lane reading 16 of a brick's 512 voxels (8 consecutive x per row, so each row is
// one contiguous run).
template <int FMT>
__global__ void __launch_bounds__(256) k_brick_summary(const SessionDesc* __restrict__ descs, int force) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.fmt != FMT || !s.occ) return;
  if (!force && (s.kind < 0 || !s.ts->integrate)) return;
  const int bx = (s.res[0] + 7) >> 3, by = (s.res[1] + 7) >> 3, bz = (s.res[2] + 7) >> 3;
  const long nb = (long)bx * by * bz;
  const long b0 = (long)blockIdx.x * 1024;
  if (b0 >= nb) return;
  __shared__ int list[1024];
  __shared__ int count;
  if (threadIdx.x == 0) count = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) {
    const long b = b0 + i;
    if (b < nb && s.occ[b] == kBrickDirty) list[atomicAdd(&count, 1)] = i;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int sx = (s.res[0] + 31) >> 5, sy = (s.res[1] + 31) >> 5;
  for (int k = threadIdx.x >> 5; k < count; k += blockDim.x >> 5) {
    const long b = b0 + list[k];
    const int x0 = (int)(b % bx) * 8, y0 = (int)((b / bx) % by) * 8, z0 = (int)(b / ((long)bx * by)) * 8;
    bool weighted = false, unweighted = false, nonpos = false;
    // 64 rows (y, z) of 8 voxels, lane & 7 = x: four rows' voxels loaded before any is
    // tested
    for (int r0 = lane >> 3; r0 < 64; r0 += 16) {
      float F[4];
      int W[4];
      bool in[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = r0 + 4 * q;
        const int x = x0 + (lane & 7), y = y0 + (r & 7), z = z0 + (r >> 3);
        in[q] = x < s.res[0] && y < s.res[1] && z < s.res[2];
        if (in[q]) Voxel<FMT>::load(s, vox_index(s, x, y, z), F[q], W[q]);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (!in[q]) continue;
        if (W[q] > 0) {
          weighted = true;
          if (!(F[q] > 0.f)) nonpos = true;
        } else {
          unweighted = true;
        }
      }
    }
    const bool any_w = __any_sync(0xffffffffu, weighted), any_u = __any_sync(0xffffffffu, unweighted);
    const bool any_np = __any_sync(0xffffffffu, nonpos);
    if (lane == 0) {
      s.occ[b] = any_np ? kBrickMixed : !any_w ? kBrickEmpty : any_u ? kBrickNoNeg : kBrickPositive;
      if (s.occ2) s.occ2[(x0 >> 5) + (size_t)sx * ((y0 >> 5) + (size_t)sy * (z0 >> 5))] = kSuperDirty;
    }
  }
}

// Re-classifies the super-bricks whose bricks k_brick_summary changed, then the 128^3
// regions holding them: one block of 64 threads per region, one thread per super-brick.
__global__ void __launch_bounds__(64) k_super_summary(const SessionDesc* __restrict__ descs, int force) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.fmt < 0 || !s.occ2) return;
  if (!force && (s.kind < 0 || !s.ts->integrate)) return;
  const int sx = (s.res[0] + 31) >> 5, sy = (s.res[1] + 31) >> 5, sz = (s.res[2] + 31) >> 5;
  const int hx = (sx + 3) >> 2, hy = (sy + 3) >> 2, hz = (sz + 3) >> 2;
  const int h = blockIdx.x;
  if (h >= hx * hy * hz) return;
  const int HX = h % hx, HY = (h / hx) % hy, HZ = h / (hx * hy);
  const int X = 4 * HX + (threadIdx.x & 3), Y = 4 * HY + ((threadIdx.x >> 2) & 3), Z = 4 * HZ + (threadIdx.x >> 4);
  const bool live = X < sx && Y < sy && Z < sz;
  const size_t i = (size_t)X + (size_t)sx * (Y + (size_t)sy * Z);
  uint8_t st = kSuperEmpty;
  bool changed = false;
  if (live) {
    st = s.occ2[i];
    if (st == kSuperDirty) {
      changed = true;
      const int bx = (s.res[0] + 7) >> 3, by = (s.res[1] + 7) >> 3, bz = (s.res[2] + 7) >> 3;
      bool all_empty = true, mixed = false;
      for (int c = 4 * Z; c < min(4 * Z + 4, bz); ++c)
        for (int b = 4 * Y; b < min(4 * Y + 4, by); ++b)
          for (int a = 4 * X; a < min(4 * X + 4, bx); ++a) {
            const uint8_t bs = s.occ[a + (size_t)bx * (b + (size_t)by * c)];
            if (bs != kBrickEmpty) all_empty = false;
            if (bs == kBrickMixed || bs == kBrickDirty) mixed = true;
          }
      st = mixed ? kSuperMixed : all_empty ? kSuperEmpty : kSuperSkip;
      s.occ2[i] = st;
    }
  }
  const bool any_changed = __syncthreads_or(changed);
  if (!any_changed) return;
  const bool any_mixed = __syncthreads_or(st == kSuperMixed || st == kSuperDirty);
  const bool any_nonempty = __syncthreads_or(st != kSuperEmpty);
  if (threadIdx.x == 0) s.occ3[h] = any_mixed ? kSuperMixed : any_nonempty ? kSuperSkip : kSuperEmpty;
}

template <int FMT>
__global__ void k_volume_init(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  const size_t n = (size_t)s.res[0] * s.res[1] * s.res[2];
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    Voxel<FMT>::init(s, i);
    if (s.cvol) s.cvol[i] = make_uchar4(0, 0, 0, 0);
  }
  const size_t nb = (size_t)((s.res[0] + 7) >> 3) * ((s.res[1] + 7) >> 3) * ((s.res[2] + 7) >> 3);
  if (s.occ)
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += (size_t)gridDim.x * blockDim.x)
      s.occ[i] = kBrickEmpty;
  const size_t ns = (size_t)((s.res[0] + 31) >> 5) * ((s.res[1] + 31) >> 5) * ((s.res[2] + 31) >> 5);
  if (s.occ2)
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += (size_t)gridDim.x * blockDim.x)
      s.occ2[i] = kSuperEmpty;
  const size_t nh = (size_t)((s.res[0] + 127) >> 7) * ((s.res[1] + 127) >> 7) * ((s.res[2] + 127) >> 7);
  if (s.occ3)
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nh; i += (size_t)gridDim.x * blockDim.x)
      s.occ3[i] = kSuperEmpty;
}

template __global__ void k_integrate<0>(const SessionDesc*);
template __global__ void k_integrate<1>(const SessionDesc*);
template __global__ void k_integrate<2>(const SessionDesc*);
template __global__ void k_integrate<3>(const SessionDesc*);
template __global__ void k_brick_summary<0>(const SessionDesc*, int);
template __global__ void k_brick_summary<1>(const SessionDesc*, int);
template __global__ void k_brick_summary<2>(const SessionDesc*, int);
template __global__ void k_brick_summary<3>(const SessionDesc*, int);
template __global__ void k_volume_init<0>(const SessionDesc*);
template __global__ void k_volume_init<1>(const SessionDesc*);
template __global__ void k_volume_init<2>(const SessionDesc*);
template __global__ void k_volume_init<3>(const SessionDesc*);

}  // namespace nui
