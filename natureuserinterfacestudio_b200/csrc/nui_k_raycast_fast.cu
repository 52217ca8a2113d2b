// Dense raycast in tolerance mode: the FP16 serving formats (NUI_TSDF_F16_U8,
// NUI_TSDF_F16_F16).  The march of raycastKernel (raycast.cl:128-277) -- nearest-voxel
// samples every 0.8 * trunc from the volume entry, stop at the first + -> - transition,
// refine it with the two trilinear samples around it (with the reference's x / y-transposed
// trilinear weights, raycast.cl:36-120), central-difference normal, colour of the voxel at
// the crossing -- with the sample parameters computed directly as t0 + k * step (one
// rounding each, instead of the reference's running float sum), voxels found by a rounded
// product with 1 / cell, and empty space skipped by arithmetic on k: a sample that lands in
// a brick, super-brick or region without a weighted voxel of tsdf <= 0 jumps straight to
// the last sample inside it.  Depths agree with the reference within the 0.5 mm raycast
// tolerance; the int16 and FP32 formats keep the exact kernels (nui_k_raycast.cu).  This
// file is compiled with contraction on.
//
// Both kernels count their voxel reads (march samples read, refined crossings) into the
// session's work counters, from which the algorithmic bytes of the launch follow.
#include "nui_raycast.cuh"

namespace nui {

template <int FMT>
__global__ void __launch_bounds__(128) k_raycast_fast(const SessionDesc* __restrict__ descs, int tw) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind != kTrackFrame || s.fmt != FMT || s.ts->status != 0) return;
  const int W = s.W, H = s.H;
  const int th = 32 / tw, bw = 2 * tw, bh = 2 * th;
  const int tiles_x = (W + bw - 1) / bw;
  if ((int)blockIdx.x >= tiles_x * ((H + bh - 1) / bh)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int px = ((int)blockIdx.x % tiles_x) * bw + (warp & 1) * tw + lane % tw;
  const int py = ((int)blockIdx.x / tiles_x) * bh + (warp >> 1) * th + lane / tw;
  const bool live = px < W && py < H;
  unsigned reads = 0, visited = 0;
  if (live) {
    const int id = py * W + px;
    const RayVol<FMT, true> V{s.vol, s.wvol, s.occ, s.res[0], s.res[1], s.res[2], (s.res[0] + 7) >> 3,
                              (s.res[1] + 7) >> 3, s.cell[0], s.cell[1], s.cell[2], 1.0f / s.cell[0],
                              1.0f / s.cell[1], 1.0f / s.cell[2]};
    const float D0 = s.dim[0], D1 = s.dim[1], D2 = s.dim[2];
    float3 start, dir, off;
    ray_of(s, px, py, start, dir, off);
    bool hit = false;
    int kc = 0;  // index of the current sample: t = t0 + kc * step
    float t0 = 0.f;
    const float3 idir = f3(1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z);
    const float txmin = (fabsf(dir.x) < 1e-14f) ? 0.f : ((dir.x > 0 ? 0.f : D0) - start.x) * idir.x;
    const float tymin = (fabsf(dir.y) < 1e-14f) ? 0.f : ((dir.y > 0 ? 0.f : D1) - start.y) * idir.y;
    const float tzmin = (fabsf(dir.z) < 1e-14f) ? 0.f : ((dir.z > 0 ? 0.f : D2) - start.z) * idir.z;
    const float txmax = (fabsf(dir.x) < 1e-14f) ? 1e14f : ((dir.x > 0 ? D0 : 0.f) - start.x) * idir.x;
    const float tymax = (fabsf(dir.y) < 1e-14f) ? 1e14f : ((dir.y > 0 ? D1 : 0.f) - start.y) * idir.y;
    const float tzmax = (fabsf(dir.z) < 1e-14f) ? 1e14f : ((dir.z > 0 ? D2 : 0.f) - start.z) * idir.z;
    const float tmin = fmaxf(fmaxf(fmaxf(txmin, tymin), tzmin), 0.f);
    const float tmax = fminf(fminf(txmax, tymax), tzmax);
    if (tmin < tmax) {
      t0 = tmin;
      int gx, gy, gz;
      V.voxel_of(add3(start, mul3(dir, t0)), gx, gy, gz);
      gx = max(0, min(gx, V.rx - 1));
      gy = max(0, min(gy, V.ry - 1));
      gz = max(0, min(gz, V.rz - 1));
      float tsdf = qnan(), f;
      if (V.tsdf_at(gx, gy, gz, f)) tsdf = f;
      ++reads;
      const float max_time = 3 * (D0 + D1 + D2);
      const float step = s.trunc * 0.8f, inv_step = 1.0f / step;
      const int kmax = (int)ceilf((max_time - t0) * inv_step);  // first sample at or past max_time
      const int sx = (V.rx + 31) >> 5, sy = (V.ry + 31) >> 5;
      const int hx = (V.rx + 127) >> 7, hy = (V.ry + 127) >> 7;
      bool pend = false;  // tsdf stands for a skipped sample at kc whose class (NaN or > 0) is unread
      while (kc < kmax) {
        float prev = tsdf;
        const int kn = kc + 1;
        const float tn = fmaf((float)kn, step, t0);
        V.voxel_of(add3(start, mul3(dir, tn)), gx, gy, gz);
        // inside the volume on all three axes (one unsigned compare an axis)
        if (!((unsigned)gx < (unsigned)V.rx && (unsigned)gy < (unsigned)V.ry && (unsigned)gz < (unsigned)V.rz)) break;
        ++visited;
        const uint8_t st = V.occ ? __ldg(V.occ + V.bidx(gx, gy, gz)) : (uint8_t)kBrickMixed;
        if (st == kBrickEmpty) {
          tsdf = qnan();
        } else if (st == kBrickPositive) {
          tsdf = 1.0f;
        } else {
          tsdf = V.load(V.vidx(gx, gy, gz), f) ? f : qnan();
          ++reads;
        }
        // empty, positive or no-negative (states 0, 2, 4): a region the march may cross
        const bool crossable = (0x15u >> st) & 1u;
        if (crossable && (!(prev < 0.f) || isnan(tsdf))) {
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
          // the last sample strictly inside the region (its exit carries a 1% voxel margin)
          const float te = fminf(V.region_exit(S, gx, gy, gz, start, dir, idir), max_time + step);
          const int kl = min(max(kn, (int)ceilf((te - t0) * inv_step) - 1), kmax);
          if (kl == kn || uniform) {
            pend = false;  // tsdf is the class of the sample at kl
          } else {
            pend = true;
            tsdf = 1.0f;
          }
          kc = kl;
          continue;
        }
        if (pend) {  // the previous sample was skipped: read its class now
          int lx, ly, lz;
          V.voxel_of(add3(start, mul3(dir, fmaf((float)kc, step, t0))), lx, ly, lz);
          prev = V.tsdf_at(lx, ly, lz, f) ? f : qnan();
          ++reads;
          pend = false;
        }
        if (isnan(tsdf) || isnan(prev)) {
          kc = kn;
          continue;
        }
        if (prev < 0.f && tsdf > 0.f) break;
        if (prev >= 0.f && tsdf <= 0.f) {
          hit = true;
          break;
        }
        kc = kn;
      }
    }
    // the crossing (entry parameter, sample index) waits in the vertex map for the refinement
    s.vref[id] = make_float4(t0, (float)kc, 0.f, hit ? 1.f : 0.f);
  }
  // work counters: voxel reads of the march and samples visited (warp-aggregated)
  const unsigned r = __reduce_add_sync(0xffffffffu, reads), v = __reduce_add_sync(0xffffffffu, visited);
  if (lane == 0 && (r | v)) {
    atomicAdd(&s.ts->ray_reads, (unsigned long long)r);
    atomicAdd(&s.ts->ray_samples, (unsigned long long)v);
  }
}

// Zero-crossing refinement, normal and colour (raycast.cl:212-272) after the fast march.
template <int FMT>
__global__ void __launch_bounds__(256, 4) k_raycast_finish_fast(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind != kTrackFrame || s.fmt != FMT || s.ts->status != 0) return;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = id < s.W * s.H;
  bool refined = false;
  if (live) {
    const float4 e = s.vref[id];
    const float4 nanv = make_float4(qnan(), qnan(), qnan(), 0.f);
    float4 vout = nanv, nout = nanv;
    uchar4 cout = make_uchar4(0, 0, 0, 0);
    if (e.w != 0.f) {
      refined = true;
      const RayVol<FMT, true> V{s.vol, s.wvol, s.occ, s.res[0], s.res[1], s.res[2], (s.res[0] + 7) >> 3,
                                (s.res[1] + 7) >> 3, s.cell[0], s.cell[1], s.cell[2], 1.0f / s.cell[0],
                                1.0f / s.cell[1], 1.0f / s.cell[2]};
      float3 start, dir, off;
      ray_of(s, id % s.W, id / s.W, start, dir, off);
      const float step = s.trunc * 0.8f;
      const int kc = (int)e.y;
      const float tc = fmaf((float)kc, step, e.x), tn = fmaf((float)(kc + 1), step, e.x);
      int gx, gy, gz;
      V.voxel_of(add3(start, mul3(dir, tn)), gx, gy, gz);
      // both samples read together (the reference skips the second when the first is NaN;
      // the result is the same)
      const float Ftdt = V.trilinear_inl(add3(start, mul3(dir, tn)));
      const float Ftc = V.trilinear_inl(add3(start, mul3(dir, tc)));
      const float Ft = isnan(Ftdt) ? Ftdt : Ftc;
      if (!isnan(Ft)) {
        const float Ts = tc - step * __fdividef(Ft, Ftdt - Ft);
        const float3 vf = add3(start, mul3(dir, Ts));
        vout = w0(sub3(vf, off));
        if (s.cvol && gx >= 0 && gy >= 0 && gz >= 0 && gx < V.rx && gy < V.ry && gz < V.rz)
          cout = s.cvol[V.vidx(gx, gy, gz)];
        int hx, hy, hz;
        V.voxel_of(add3(start, mul3(dir, tc)), hx, hy, hz);
        if (hx > 1 && hy > 1 && hz > 1 && hx < V.rx - 2 && hy < V.ry - 2 && hz < V.rz - 2) {
          // the six samples in two groups of three, each group's 24 voxel reads in flight
          float3 n;
          const float fx1 = V.trilinear_inl(f3(vf.x + s.cell[0], vf.y, vf.z));
          const float fy1 = V.trilinear_inl(f3(vf.x, vf.y + s.cell[1], vf.z));
          const float fz1 = V.trilinear_inl(f3(vf.x, vf.y, vf.z + s.cell[2]));
          const float fx2 = V.trilinear_inl(f3(vf.x - s.cell[0], vf.y, vf.z));
          const float fy2 = V.trilinear_inl(f3(vf.x, vf.y - s.cell[1], vf.z));
          const float fz2 = V.trilinear_inl(f3(vf.x, vf.y, vf.z - s.cell[2]));
          n.x = fx1 - fx2;
          n.y = fy1 - fy2;
          n.z = fz1 - fz2;
          nout = w0(normalize3(n));
        }
      }
    }
    s.vref[id] = vout;
    s.nref[id] = nout;
    if (s.cmap) s.cmap[id] = cout;
  }
  const unsigned h = __popc(__ballot_sync(0xffffffffu, refined));
  if ((threadIdx.x & 31) == 0 && h) atomicAdd(&s.ts->ray_hits, (unsigned long long)h);
}

template __global__ void k_raycast_fast<2>(const SessionDesc*, int);
template __global__ void k_raycast_fast<3>(const SessionDesc*, int);
template __global__ void k_raycast_finish_fast<2>(const SessionDesc*);
template __global__ void k_raycast_finish_fast<3>(const SessionDesc*);

}  // namespace nui
