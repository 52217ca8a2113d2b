// Voxel-block hashing on the GPU (KinfuHashScene.cl, KinfuHashRaycast.cl; host
// NuiKinfuOpenCLHashScene.cpp AllocateSceneFromDepth / IntegrateIntoScene / raycastRender).
//
// Per frame, for every hash session of the batch:
//   k_hash_prepare      visible types of the last frame's list -> 3, allocation types -> 0
//   k_hash_walk(0)      per pixel: walk [d - mu, d + mu] along the ray in block units; mark
//                       found blocks visible, mark missing ones for allocation and keep, per
//                       entry slot, the largest (pixel, step) key that wanted it
//   k_hash_walk(1)      the walk again: the key owner writes its block coordinates (the
//                       block the last writer in raster order would have left)
//   k_hash_flag_count(0) + k_hash_scan + k_hash_alloc
//                       entries needing allocation, ranked in index order, pop blocks from
//                       the free stack (and excess slots for chain appends) in that order
//   k_hash_visible      previously visible entries (type 3): 8-corner frustum test
//   k_hash_flag_count(1) + k_hash_scan + k_hash_compact
//                       visible list = entries with visible type > 0 in index order
//   k_hash_integrate    one 512-thread block per visible entry, one voxel per thread
//   k_hash_range + k_hash_project + k_hash_raycast
//                       expected range image by atomic min/max of projected block boxes,
//                       then castRay per pixel
// Arithmetic follows the reference kernels operation by operation (the library is built
// without contraction), so all outputs match the CPU restatement bit for bit.
#include "nui_device.cuh"

namespace nui {

constexpr int kTransferBlocks = 4096;  // SDF_TRANSFER_BLOCK_NUM (hashing_gpu_def.h:16)

constexpr int kHashScanBlock = 1024;

__device__ __forceinline__ unsigned hash_index(unsigned mask, int x, int y, int z) {
  return (((unsigned)x * 73856093u) ^ ((unsigned)y * 19349669u) ^ ((unsigned)z * 83492791u)) & mask;
}
__device__ __forceinline__ HEntry load_entry(const HEntry* e, unsigned i) {
  const int4 v = __ldcg(reinterpret_cast<const int4*>(e) + i);
  HEntry r;
  r.pos[0] = (short)(v.x & 0xffff);
  r.pos[1] = (short)((unsigned)v.x >> 16);
  r.pos[2] = (short)(v.y & 0xffff);
  r.pad = (short)((unsigned)v.y >> 16);
  r.ptr = v.z;
  r.offset = (unsigned)v.w;
  return r;
}
__device__ __forceinline__ void store_entry(HEntry* e, unsigned i, const HEntry& r) {
  int4 v;
  v.x = (int)((unsigned short)r.pos[0] | ((unsigned)(unsigned short)r.pos[1] << 16));
  v.y = (int)((unsigned short)r.pos[2] | ((unsigned)(unsigned short)r.pad << 16));
  v.z = r.ptr;
  v.w = (int)r.offset;
  reinterpret_cast<int4*>(e)[i] = v;
}
__device__ __forceinline__ float3 xf_apply(const DevXform& m, float3 v) {
  return add3(rot_rows(m.R, v), f3(m.t[0], m.t[1], m.t[2]));
}
__device__ __forceinline__ float3 xf_inverse(const DevXform& m, float3 v) {
  return rot_rows(m.R_inv, sub3(v, f3(m.t[0], m.t[1], m.t[2])));
}
// pass-filtered z-depth of a pixel (depth_passing_filter_kernel, filters.cl:9-23)
__device__ __forceinline__ float pass_depth(const SessionDesc& s, int i) {
  const float dp = (float)s.raw[i] * 0.001f;
  return (dp > s.cam.dmin && dp < s.cam.dmax) ? dp : qnan();
}
// kinectDepthToSkeleton (cameraUtils.cl:46-53)
__device__ __forceinline__ float3 depth_to_point(const DevCam& c, int ux, int uy, float d) {
  const float x = ((float)ux - c.cx) / c.fx, y = ((float)uy - c.cy) / c.fy;
  return f3(d * x, d * y, d);
}
__device__ __forceinline__ bool hash_active(const SessionDesc& s) { return s.hash && s.kind >= 0 && s.ts->integrate; }

// ------------------------------------------------------------------ allocation
// The per-entry byte flags (alloc_type, vis) are scanned sixteen at a time: the bytes from
// entry i (a multiple of 16) in one 16-byte load when all lie below n, else byte by byte
// (bytes at or past n read as 0).  A 1024-entry scan block is 64 threads.
__device__ __forceinline__ uint4 load16(const uint8_t* p, unsigned i, unsigned n) {
  if (i + 16 <= n) return *reinterpret_cast<const uint4*>(p + i);
  unsigned w[4] = {0u, 0u, 0u, 0u};
  for (unsigned k = 0; k < 16 && i + k < n; ++k) w[k >> 2] |= (unsigned)p[i + k] << (8 * (k & 3));
  return make_uint4(w[0], w[1], w[2], w[3]);
}
// 0xff in every byte of w equal to / different from the matching byte of v
__device__ __forceinline__ uint4 eq16(uint4 w, unsigned v) {
  return make_uint4(__vcmpeq4(w.x, v), __vcmpeq4(w.y, v), __vcmpeq4(w.z, v), __vcmpeq4(w.w, v));
}
__device__ __forceinline__ uint4 ne16(uint4 w, unsigned v) {
  return make_uint4(__vcmpne4(w.x, v), __vcmpne4(w.y, v), __vcmpne4(w.z, v), __vcmpne4(w.w, v));
}
__device__ __forceinline__ unsigned count16(uint4 m) {
  return (__popc(m.x) + __popc(m.y) + __popc(m.z) + __popc(m.w)) >> 3;
}
__device__ __forceinline__ bool bit16(uint4 m, int k) {
  const unsigned w = k < 4 ? m.x : k < 8 ? m.y : k < 12 ? m.z : m.w;
  return (w >> (8 * (k & 3))) & 1u;
}
// Exclusive prefix of c over the 64 threads of a scan block, in thread order.
__device__ __forceinline__ unsigned scan64(unsigned c) {
  const int lane = threadIdx.x & 31;
  unsigned incl = c;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const unsigned o = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += o;
  }
  __shared__ unsigned w0;
  if (threadIdx.x == 31) w0 = incl;
  __syncthreads();
  return incl - c + (threadIdx.x >= 32 ? w0 : 0u);
}

__global__ void k_hash_prepare(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s)) return;
  const unsigned n = (unsigned)(s.nb + s.ne);
  for (unsigned i = 16 * (blockIdx.x * blockDim.x + threadIdx.x); i < n; i += 16 * gridDim.x * blockDim.x) {
    if (i + 16 <= n) {
      reinterpret_cast<uint4*>(s.alloc_type)[i >> 4] = make_uint4(0u, 0u, 0u, 0u);
      uint4* v = reinterpret_cast<uint4*>(s.vis) + (i >> 4);
      const uint4 m = ne16(*v, 0u);  // visible (any type) -> 3, else 0
      *v = make_uint4(m.x & 0x03030303u, m.y & 0x03030303u, m.z & 0x03030303u, m.w & 0x03030303u);
    } else {
      for (unsigned k = i; k < n; ++k) {
        s.alloc_type[k] = 0;
        s.vis[k] = s.vis[k] ? 3 : 0;
      }
    }
  }
}

// buildHashAllocAndVisibleType_kernel (KinfuHashScene.cl:52-136); pass 1 writes the
// coordinates of the last writer of each pending slot.
__global__ void __launch_bounds__(256) k_hash_walk(const SessionDesc* __restrict__ descs, int pass) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s)) return;
  const int W = s.W, H = s.H;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= W * H) return;
  const float Dp = pass_depth(s, id);
  if (isnan(Dp)) return;
  // pass 1 only walks the rays that requested a block in pass 0 (the table does not change
  // between the passes, so any other ray finds every block again); the flag is kept in the
  // range image, which the raycast rewrites before it reads it
  if (pass == 1 && s.range[id].x == 0.f) return;
  bool requested = false;
  const int px = id % W, py = id / W;
  const DevXform& m = s.ts->xf;
  const float3 pc = depth_to_point(s.cam, px, py, Dp);
  const float norm = s.mu / sqrtf(dot3(pc, pc));
  const float obs = 1.0f / (s.voxel * 8);
  float3 rmin = mul3(xf_apply(m, mul3(pc, 1.0f - norm)), obs);
  const float3 rmax = mul3(xf_apply(m, mul3(pc, 1.0f + norm)), obs);
  float3 rdir = sub3(rmax, rmin);
  const float rn = sqrtf(dot3(rdir, rdir));
  const int steps = (int)ceilf(2.0f * rn);
  const float dv = (float)(steps - 1);
  rdir = f3(rdir.x / dv, rdir.y / dv, rdir.z / dv);
  for (int i = 0; i < steps; ++i) {
    const short bx = (short)floorf(rmin.x), by = (short)floorf(rmin.y), bz = (short)floorf(rmin.z);
    unsigned hi = hash_index(s.hmask, bx, by, bz);
    HEntry en = load_entry(s.entries, hi);
    bool found = false;
    if (en.pos[0] == bx && en.pos[1] == by && en.pos[2] == bz && en.ptr >= -1) {
      if (pass == 0) s.vis[hi] = (en.ptr == -1) ? 2 : 1;
      found = true;
    }
    if (!found) {
      bool excess = false, broken = false;
      if (en.ptr >= -1) {
        // an excess chain holds at most ne entries, each link inside the excess list; a
        // link that breaks either rule is a corrupted table: counted (the tick reports
        // NUI_ERR_HASH_FULL) and the block is neither found nor requested
        int links = 0;
        while (en.offset >= 1) {
          if (en.offset > (unsigned)s.ne || ++links > s.ne) {
            if (pass == 0) atomicAdd(&s.hcount[kHashChainFaults], 1);
            broken = true;
            break;
          }
          hi = (unsigned)s.nb + en.offset - 1;
          en = load_entry(s.entries, hi);
          if (en.pos[0] == bx && en.pos[1] == by && en.pos[2] == bz && en.ptr >= -1) {
            if (pass == 0) s.vis[hi] = (en.ptr == -1) ? 2 : 1;
            found = true;
            break;
          }
        }
        excess = true;
      }
      if (!found && !broken) {
        const unsigned long long key = ((unsigned long long)(id + 1) << 16) | (unsigned long long)(i & 0xffff);
        if (pass == 0) {
          s.alloc_type[hi] = excess ? 2 : 1;
          s.vis[hi] = 1;
          atomicMax(&s.keys[hi], key);
          requested = true;
        } else if (__ldcg(&s.keys[hi]) == key) {
          s.coords[hi] = make_short4(bx, by, bz, 0);
        }
      }
    }
    rmin = add3(rmin, rdir);
  }
  if (pass == 0) s.range[id].x = requested ? 1.f : 0.f;
}

__device__ __forceinline__ int entry_ptr(const SessionDesc& s, unsigned i) {
  return reinterpret_cast<const int*>(s.entries)[4 * i + 2];
}
// buildSwapOutList_kernel (KinfuHashSwapping.cl:113-124): merged (2), holding a block other
// than block 0, not visible
__device__ __forceinline__ bool swap_out_flag(const SessionDesc& s, unsigned i) {
  return s.swap[i] == 2 && entry_ptr(s, i) > 0 && s.vis[i] == 0;
}

// Per 1024 entries: number of entries needing a block (type >= 1) and an excess slot
// (type 2) (which == 0); of visible entries (which == 1).  One 64-thread block per 1024
// entries, sixteen a thread.
__global__ void __launch_bounds__(64) k_hash_flag_count(const SessionDesc* __restrict__ descs, int which) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s)) return;
  const unsigned n = (unsigned)(s.nb + s.ne);
  const unsigned b0 = blockIdx.x * kHashScanBlock;
  if (b0 >= n) return;
  const unsigned i = b0 + 16 * threadIdx.x;
  unsigned a = 0, e = 0;
  if (i < n) {
    const uint4 w = load16(which == 0 ? s.alloc_type : s.vis, i, n);
    a = count16(ne16(w, 0u));
    if (which == 0) e = count16(eq16(w, 0x02020202u));
  }
  a = __reduce_add_sync(0xffffffffu, a);
  e = __reduce_add_sync(0xffffffffu, e);
  __shared__ unsigned sa, se;
  if (threadIdx.x == 32) {
    sa = a;
    se = e;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s.blk[4 * blockIdx.x] = a + sa;
    s.blk[4 * blockIdx.x + 1] = e + se;
  }
}

// With the global cache, per 1024 entries: number of visible entries whose block was
// swapped out and of entries to swap in (which == 2), of entries to swap out (which == 3).
__global__ void __launch_bounds__(256) k_hash_count(const SessionDesc* __restrict__ descs, int which) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s) || !s.swapping) return;
  const unsigned n = (unsigned)(s.nb + s.ne);
  const unsigned b0 = blockIdx.x * kHashScanBlock;
  if (b0 >= n) return;
  unsigned a = 0, e = 0;
  for (unsigned i = b0 + threadIdx.x; i < min(n, b0 + kHashScanBlock); i += blockDim.x) {
    if (which == 2) {  // re-allocations, swap-ins
      a += s.vis[i] > 0 && entry_ptr(s, i) == -1;
      e += s.swap[i] == 1;
    } else {  // swap-outs
      a += swap_out_flag(s, i);
    }
  }
  a = __reduce_add_sync(0xffffffffu, a);
  e = __reduce_add_sync(0xffffffffu, e);
  __shared__ unsigned sa[8], se[8];
  if ((threadIdx.x & 31) == 0) {
    sa[threadIdx.x >> 5] = a;
    se[threadIdx.x >> 5] = e;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned ta = 0, te = 0;
    for (int w = 0; w < 8; ++w) {
      ta += sa[w];
      te += se[w];
    }
    s.blk[4 * blockIdx.x] = ta;
    s.blk[4 * blockIdx.x + 1] = te;
  }
}

// Exclusive scan of the per-block counts of one session (one 1024-thread block per
// session); offsets go to blk[4b + 2], blk[4b + 3].  Totals: allocation -> updates the free
// stacks; visible -> visible count.
__global__ void __launch_bounds__(1024) k_hash_scan(const SessionDesc* __restrict__ descs, int which) {
  const SessionDesc& s = descs[blockIdx.x];
  if (!hash_active(s) || (which >= 2 && !s.swapping)) return;
  const int nblk = (s.nb + s.ne + kHashScanBlock - 1) / kHashScanBlock;
  __shared__ unsigned wa[32], we[32];
  __shared__ unsigned carry_a, carry_e;
  if (threadIdx.x == 0) carry_a = carry_e = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < nblk; base += 1024) {
    const int i = base + threadIdx.x;
    const unsigned va = i < nblk ? s.blk[4 * i] : 0u, ve = i < nblk ? s.blk[4 * i + 1] : 0u;
    unsigned ia = va, ie = ve;
    for (int off = 1; off < 32; off <<= 1) {
      const unsigned oa = __shfl_up_sync(0xffffffffu, ia, off), oe = __shfl_up_sync(0xffffffffu, ie, off);
      if (lane >= off) {
        ia += oa;
        ie += oe;
      }
    }
    if (lane == 31) {
      wa[warp] = ia;
      we[warp] = ie;
    }
    __syncthreads();
    if (warp == 0) {
      const unsigned a = wa[lane], e = we[lane];
      unsigned xa = a, xe = e;
      for (int off = 1; off < 32; off <<= 1) {
        const unsigned oa = __shfl_up_sync(0xffffffffu, xa, off), oe = __shfl_up_sync(0xffffffffu, xe, off);
        if (lane >= off) {
          xa += oa;
          xe += oe;
        }
      }
      wa[lane] = xa - a;
      we[lane] = xe - e;
    }
    __syncthreads();
    const unsigned ea = carry_a + wa[warp] + ia - va, ee = carry_e + we[warp] + ie - ve;
    __syncthreads();
    if (i < nblk) {
      s.blk[4 * i + 2] = ea;
      s.blk[4 * i + 3] = ee;
    }
    if (threadIdx.x == 1023) {
      carry_a = ea + va;
      carry_e = ee + ve;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (which == 1) s.hcount[2] = (int)carry_a;
    if (which == 2) {  // the re-allocations pop the free list in index order (atomic_dec)
      s.hcount[6] = s.hcount[0];
      s.hcount[0] -= (int)carry_a;
      s.hcount[4] = min((int)carry_e, kTransferBlocks);
    }
    if (which == 3) s.hcount[5] = min((int)carry_a, kTransferBlocks);
  }
}

// Rank of entry i among the entries of its 1024-block satisfying `pred` (block-wide scan in
// index order).  All threads of the block must call it.
template <class Pred>
__device__ __forceinline__ unsigned block_rank(unsigned i, unsigned n, Pred pred, bool& flag, unsigned& total) {
  __shared__ unsigned wsum[kHashScanBlock / 32];
  flag = i < n && pred(i);
  const unsigned ballot = __ballot_sync(0xffffffffu, flag);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) wsum[warp] = __popc(ballot);
  __syncthreads();
  unsigned before = 0;
  for (int w = 0; w < warp; ++w) before += wsum[w];
  total = 0;
  for (int w = 0; w < kHashScanBlock / 32; ++w) total += wsum[w];
  __syncthreads();
  return before + __popc(ballot & ((1u << lane) - 1u));
}

// allocateVoxelBlocksList_kernel (KinfuHashScene.cl:138-194) with the pops in index order:
// 256 threads a 1024-entry block, four entries each; an entry's ranks among the block's
// requests and excess requests are the counts of the threads before it (one scan of both
// counts packed in 16-bit halves) plus those of its own lower bytes.
__device__ __forceinline__ void alloc_one(const SessionDesc& s, unsigned i, int vba, int exl) {
  const uint8_t t = s.alloc_type[i];
  const short4 c = s.coords[i];
  s.keys[i] = 0ull;
  if (t == 1) {
    if (vba >= 0) {
      HEntry en;
      en.pos[0] = c.x;
      en.pos[1] = c.y;
      en.pos[2] = c.z;
      en.pad = 0;
      en.ptr = s.alloc_list[vba];
      en.offset = 0;
      store_entry(s.entries, i, en);
    } else {
      atomicAdd(&s.hcount[3], 1);
    }
  } else {
    if (vba >= 0 && exl >= 0) {
      HEntry en;
      en.pos[0] = c.x;
      en.pos[1] = c.y;
      en.pos[2] = c.z;
      en.pad = 0;
      en.ptr = s.alloc_list[vba];
      en.offset = 0;
      const int off = s.excess_list[exl];
      HEntry parent = load_entry(s.entries, i);
      parent.offset = (unsigned)off + 1;
      store_entry(s.entries, i, parent);
      store_entry(s.entries, (unsigned)s.nb + off, en);
      s.vis[s.nb + off] = 1;
    } else {
      atomicAdd(&s.hcount[3], 1);
    }
  }
}

__global__ void __launch_bounds__(64) k_hash_alloc(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s)) return;
  const unsigned n = (unsigned)(s.nb + s.ne);
  const unsigned b = blockIdx.x;
  if (b * kHashScanBlock >= n) return;
  if (s.blk[4 * b] == 0) return;  // no request among the block's entries (k_hash_flag_count)
  const unsigned i = b * kHashScanBlock + 16 * threadIdx.x;
  const uint4 w = i < n ? load16(s.alloc_type, i, n) : make_uint4(0u, 0u, 0u, 0u);
  const uint4 ma = ne16(w, 0u), me = eq16(w, 0x02020202u);
  const unsigned c = count16(ma) | (count16(me) << 16);
  const unsigned before = scan64(c);
  if (!count16(ma)) return;
  const int last_block = s.hcount[0], last_excess = s.hcount[1];
  unsigned ra = s.blk[4 * b + 2] + (before & 0xffffu), re = s.blk[4 * b + 3] + (before >> 16);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    if (!bit16(ma, k)) continue;
    const bool ex = bit16(me, k);
    alloc_one(s, i + k, last_block - (int)ra, ex ? last_excess - (int)re : 0);
    ++ra;
    if (ex) ++re;
  }
}

// After k_hash_alloc: pop the free stacks by the number of requests (as the reference's
// atomic_dec calls do, successful or not).
__global__ void k_hash_alloc_done(const SessionDesc* __restrict__ descs, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const SessionDesc& s = descs[k];
  if (!hash_active(s)) return;
  const int nblk = (s.nb + s.ne + kHashScanBlock - 1) / kHashScanBlock;
  const unsigned ta = s.blk[4 * (nblk - 1) + 2] + s.blk[4 * (nblk - 1)];
  const unsigned te = s.blk[4 * (nblk - 1) + 3] + s.blk[4 * (nblk - 1) + 1];
  s.hcount[0] -= (int)ta;
  s.hcount[1] -= (int)te;
}

// buildVisibleList_kernel + checkBlockVisibility (KinfuHashScene.cl:196-285).  With the
// global cache, buildVisibleEnlargedList_kernel (:358-385): its bounds are
// (-W/8, W + W/8, -H/8, H + H/8) held as unsigned numbers (:306-311), so the lower bound
// wraps above the upper one and the enlarged test never passes -- an entry seen only at the
// previous frame drops out; every entry visible at the start, unless already merged (2),
// is marked for swap-in.
__device__ __forceinline__ bool point_visible(const SessionDesc& s, const DevXform& m, float3 p) {
  const float3 q = xf_inverse(m, p);
  if (isnan3(q)) return false;
  const int sx = (int)(q.x * s.cam.fx / q.z + s.cam.cx + 0.5f), sy = (int)(q.y * s.cam.fy / q.z + s.cam.cy + 0.5f);
  return sx >= 0 && sx < s.W && sy >= 0 && sy < s.H;
}
__global__ void k_hash_visible(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s)) return;
  const unsigned n = (unsigned)(s.nb + s.ne);
  const DevXform& m = s.ts->xf;
  const float factor = 8.0f * s.voxel;
  if (s.swapping) {
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
      const uint8_t t = s.vis[i];
      if (t == 3) s.vis[i] = 0;
      if (t > 0 && s.swap[i] != 2) s.swap[i] = 1;
    }
    return;
  }
  for (unsigned i16 = 16 * (blockIdx.x * blockDim.x + threadIdx.x); i16 < n; i16 += 16 * gridDim.x * blockDim.x) {
    const uint4 m16 = eq16(load16(s.vis, i16, n), 0x03030303u);  // entries visible at the last frame
    for (int q = 0; q < 4; ++q) {
      unsigned m3 = q == 0 ? m16.x : q == 1 ? m16.y : q == 2 ? m16.z : m16.w;
      while (m3) {
        const int k = (__ffs(m3) - 1) >> 3;
        m3 &= ~(0xFFu << (8 * k));
        const unsigned i = i16 + 4 * q + (unsigned)k;
        const HEntry en = load_entry(s.entries, i);
        float3 p = f3((float)en.pos[0] * factor, (float)en.pos[1] * factor, (float)en.pos[2] * factor);
        bool v = point_visible(s, m, p);
        if (!v) { p.z += factor; v = point_visible(s, m, p); }
        if (!v) { p.y += factor; v = point_visible(s, m, p); }
        if (!v) { p.x += factor; v = point_visible(s, m, p); }
        if (!v) { p.z -= factor; v = point_visible(s, m, p); }
        if (!v) { p.y -= factor; v = point_visible(s, m, p); }
        if (!v) { p.x -= factor; p.y += factor; v = point_visible(s, m, p); }
        if (!v) { p.x += factor; p.y -= factor; p.z += factor; v = point_visible(s, m, p); }
        if (!v) s.vis[i] = 0;
      }
    }
  }
}

// The visible list in index order: a 64-thread block per 1024 entries, sixteen a thread;
// a thread's rank is the block offset (k_hash_scan) plus the visible entries of the
// threads before it.
__global__ void __launch_bounds__(64) k_hash_compact(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s)) return;
  const unsigned n = (unsigned)(s.nb + s.ne);
  const unsigned b = blockIdx.x;
  if (b * kHashScanBlock >= n) return;
  if (s.blk[4 * b] == 0) return;  // no visible entry in the block
  const unsigned i = b * kHashScanBlock + 16 * threadIdx.x;
  const uint4 m = i < n ? ne16(load16(s.vis, i, n), 0u) : make_uint4(0u, 0u, 0u, 0u);
  unsigned r = s.blk[4 * b + 2] + scan64(count16(m));
#pragma unroll
  for (int k = 0; k < 16; ++k)
    if (bit16(m, k)) s.vis_ids[r++] = (int)(i + k);
}

// ------------------------------------------------------------------ integration
template <int HF>
struct HVox;
template <>
struct HVox<0> {  // reference int16 sdf (KinfuHashScene.cl:438, 468)
  __device__ static __forceinline__ float load(const void* p, unsigned i) {
    return (float)reinterpret_cast<const short*>(p)[i] / 32767.0f;
  }
  __device__ static __forceinline__ void store(void* p, unsigned i, float f) {
    reinterpret_cast<short*>(p)[i] = (short)__float2int_rz(f * 32767.0f);
  }
};
template <>
struct HVox<1> {  // half sdf
  __device__ static __forceinline__ float load(const void* p, unsigned i) {
    return __half2float(reinterpret_cast<const __half*>(p)[i]);
  }
  __device__ static __forceinline__ void store(void* p, unsigned i, float f) {
    reinterpret_cast<__half*>(p)[i] = __float2half_rn(f);
  }
};

// One voxel of integrateIntoScene_kernel, given its entry, weight w and sdf oldF.  The
// reference's int16 format (HF 0) repeats its arithmetic operation for operation; the half
// format (HF 1, a serving format checked against tolerances) takes the same steps with fused
// multiply-adds and approximate reciprocals, which can move a voxel across a pixel's
// rounding edge or change its value by a few ulps, well inside the half quantum.
template <int HF>
__device__ __forceinline__ void integrate_voxel(const SessionDesc& s, const DevXform& m, const HEntry& en, int w,
                                                float oldF, int lid, int lx, int ly, int lz, unsigned& touched) {
  if (en.ptr < 0) return;
  const unsigned bid = (unsigned)en.ptr * 512u + (unsigned)lid;
  if (s.max_w == w) return;
  const float3 pm = mul3(f3((float)(en.pos[0] * 8 + lx), (float)(en.pos[1] * 8 + ly), (float)(en.pos[2] * 8 + lz)),
                         s.voxel);
  float3 pc;
  int ix, iy;
  if (HF == 0) {
    pc = xf_inverse(m, pm);
    if (pc.z <= 0) return;
    ix = (int)(pc.x * s.cam.fx / pc.z + s.cam.cx + 0.5f);
    iy = (int)(pc.y * s.cam.fy / pc.z + s.cam.cy + 0.5f);
  } else {
    const float dx = pm.x - m.t[0], dy = pm.y - m.t[1], dz = pm.z - m.t[2];
    const float* Ri = m.R_inv;
    pc = f3(__fmaf_rn(Ri[0], dx, __fmaf_rn(Ri[1], dy, Ri[2] * dz)), __fmaf_rn(Ri[3], dx, __fmaf_rn(Ri[4], dy, Ri[5] * dz)),
            __fmaf_rn(Ri[6], dx, __fmaf_rn(Ri[7], dy, Ri[8] * dz)));
    if (pc.z <= 0) return;
    const float iz = __fdividef(1.0f, pc.z);
    ix = (int)__fmaf_rn(pc.x * s.cam.fx, iz, s.cam.cx + 0.5f);
    iy = (int)__fmaf_rn(pc.y * s.cam.fy, iz, s.cam.cy + 0.5f);
  }
  if (ix < 0 || ix >= s.W || iy < 0 || iy >= s.H) return;
  const int sid = iy * s.W + ix;
  const float d = pass_depth(s, sid);
  if (isnan(d)) return;
  const float eta = d - pc.z;
  const float sdf = HF == 0 ? eta / s.mu : eta * __fdividef(1.0f, s.mu);
  if (eta < -s.mu) return;
  const float oldW = (float)w;
  float newF = fminf(1.0f, sdf);
  const float newW = 1.0f, cw = oldW + newW;
  if (s.bgra && s.hrgb && eta < s.mu && fabsf(sdf) < 0.25f) {
    const uchar4 col = reinterpret_cast<const uchar4*>(s.bgra)[sid];
    if (col.w == 255) {
      const uchar4 vc = s.hrgb[bid];
      float r, g, bl;
      if (HF == 0) {
        r = (oldW * (float)vc.x + newW * (float)col.z) / cw;
        g = (oldW * (float)vc.y + newW * (float)col.y) / cw;
        bl = (oldW * (float)vc.z + newW * (float)col.x) / cw;
      } else {
        const float icw = __fdividef(1.0f, cw);
        r = __fmaf_rn(oldW, (float)vc.x, (float)col.z) * icw;
        g = __fmaf_rn(oldW, (float)vc.y, (float)col.y) * icw;
        bl = __fmaf_rn(oldW, (float)vc.z, (float)col.x) * icw;
      }
      s.hrgb[bid] = make_uchar4((unsigned char)fminf(fmaxf(r, 0.f), 255.f), (unsigned char)fminf(fmaxf(g, 0.f), 255.f),
                                (unsigned char)fminf(fmaxf(bl, 0.f), 255.f), 0);
    }
  }
  if (HF == 0) {
    newF = oldW * oldF + newW * newF;
    newF /= cw;
  } else {
    newF = __fdividef(__fmaf_rn(oldW, oldF, newF), cw);
  }
  HVox<HF>::store(s.hsdf, bid, newF);
  s.hw[bid] = (uint8_t)min((int)(uint8_t)cw, s.max_w);
  ++touched;
}

// integrateIntoScene_kernel (KinfuHashScene.cl:387-470); blocks stride over the list.
template <int HF>
__global__ void __launch_bounds__(512, 3) k_hash_integrate(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s) || s.hfmt != HF) return;
  const int nvis = s.hcount[2];
  const DevXform& m = s.ts->xf;
  const int lid = threadIdx.x;
  const int lx = (lid % 64) % 8, ly = (lid % 64) / 8, lz = lid / 64;
  unsigned touched = 0;
  // Software pipeline over the block's list positions k, k + g, k + 2g, ...: while position
  // k is integrated, the voxel (weight and sdf) of k + g and the hash entry of k + 2g are
  // already in flight, so only the depth read waits inside an iteration.
  const int g = (int)gridDim.x, k0 = (int)blockIdx.x;
  auto entry_at = [&](int k) {
    HEntry e;
    e.ptr = -1;
    if (k < nvis) e = load_entry(s.entries, (unsigned)s.vis_ids[k]);
    return e;
  };
  HEntry en = entry_at(k0), en1 = entry_at(k0 + g);
  int w = 0;
  float oldF = 0.f;
  if (en.ptr >= 0) {
    w = s.hw[(unsigned)en.ptr * 512u + (unsigned)lid];
    oldF = HVox<HF>::load(s.hsdf, (unsigned)en.ptr * 512u + (unsigned)lid);
  }
  for (int k = k0; k < nvis; k += g) {
    const HEntry cur = en;
    const int cw0 = w;
    const float cF = oldF;
    en = en1;
    en1 = entry_at(k + 2 * g);
    if (en.ptr >= 0) {
      w = s.hw[(unsigned)en.ptr * 512u + (unsigned)lid];
      oldF = HVox<HF>::load(s.hsdf, (unsigned)en.ptr * 512u + (unsigned)lid);
    }
    integrate_voxel<HF>(s, m, cur, cw0, cF, lid, lx, ly, lz, touched);
  }
  const unsigned t = __reduce_add_sync(0xffffffffu, touched);
  if ((threadIdx.x & 31) == 0 && t) atomicAdd(&s.ts->touched, (unsigned long long)t);
}

// ------------------------------------------------------------------ raycast
__global__ void k_hash_range(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.hash || s.kind != kTrackFrame || s.ts->status != 0) return;
  const int n = s.W * s.H;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    s.range[i] = make_float2(999999.9f, 0.05f);
    if (s.fwd) s.fwd_owner[i] = 0;
  }
}

// project_minmax_depths_kernel (KinfuHashRaycast.cl:4-76) with atomic min / max per pixel
// (positive floats order like their bit patterns).  One warp per visible block: lanes 0-7
// project its corners, the warp reduces their bounds, and all lanes share the block's
// pixels.  The kernel's far depth is updated as zy = max(zx, z) after each corner, which
// leaves the depth of the last corner that projected (zx is then at most that depth).
__global__ void __launch_bounds__(256) k_hash_project(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.hash || s.kind != kTrackFrame || s.ts->status != 0) return;
  const int nvis = s.hcount[2];
  const DevXform& m = s.ts->xf;
  const int lane = threadIdx.x & 31;
  const int nwarps = gridDim.x * (blockDim.x >> 5);
  for (int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < nvis; k += nwarps) {
    const HEntry en = load_entry(s.entries, (unsigned)s.vis_ids[k]);
    if (en.ptr < 0) continue;
    int ulx = s.W, uly = s.H, lrx = 0, lry = 0;
    float zx = 999999.9f, pz = 0.f;
    bool valid = false;
    if (lane < 8) {
      const short cx = (short)(en.pos[0] + ((lane & 1) ? 1 : 0)), cy = (short)(en.pos[1] + ((lane & 2) ? 1 : 0)),
                  cz = (short)(en.pos[2] + ((lane & 4) ? 1 : 0));
      float3 p = mul3(mul3(f3((float)cx, (float)cy, (float)cz), 8.0f), s.voxel);
      p = xf_inverse(m, p);
      if (!(isnan3(p) || p.z < 1e-6)) {
        valid = true;
        const float u = p.x * s.cam.fx / p.z + s.cam.cx, v = p.y * s.cam.fy / p.z + s.cam.cy;
        ulx = (int)floorf(u);
        lrx = (int)ceilf(u);
        uly = (int)floorf(v);
        lry = (int)ceilf(v);
        zx = p.z;
        pz = p.z;
      }
    }
    const unsigned vb = __ballot_sync(0xffffffffu, valid);
    ulx = min(__reduce_min_sync(0xffffffffu, ulx), s.W);
    uly = min(__reduce_min_sync(0xffffffffu, uly), s.H);
    lrx = max(__reduce_max_sync(0xffffffffu, lrx), 0);
    lry = max(__reduce_max_sync(0xffffffffu, lry), 0);
    for (int off = 16; off > 0; off >>= 1) zx = fminf(zx, __shfl_xor_sync(0xffffffffu, zx, off));
    const float last = __shfl_sync(0xffffffffu, pz, vb ? 31 - __clz(vb) : 0);
    const float zy = vb ? last : 0.05f;
    if (ulx < 0) ulx = 0;
    if (uly < 0) uly = 0;
    if (lrx >= s.W) lrx = s.W - 1;
    if (lry >= s.H) lry = s.H - 1;
    if (zx < 0.05f) zx = 0.05f;
    const int bw = lrx - ulx + 1, bh = lry - uly + 1;
    if (bw <= 0 || bh <= 0) continue;
    // an atomic that cannot lower the pixel's near bound or raise its far bound is skipped:
    // the bounds only move one way, so a stale read costs an atomic, never a result
    for (int q = lane; q < bw * bh; q += 32) {
      float2* r = s.range + (uly + q / bw) * s.W + (ulx + q % bw);
      const float2 cur = __ldcg(r);
      if (__float_as_int(zx) < __float_as_int(cur.x)) atomicMin(reinterpret_cast<int*>(&r->x), __float_as_int(zx));
      if (__float_as_int(zy) > __float_as_int(cur.y)) atomicMax(reinterpret_cast<int*>(&r->y), __float_as_int(zy));
    }
  }
}

// Pool offset (block index * 512) of block (sx, sy, sz) or -1: the bucket, then its excess
// chain (findVoxelBlockIndex, KinfuHashRaycast.cl:78-111).
// The walk visits at most the bucket and ne excess entries and follows only links inside
// the excess list: a corrupted chain ends the lookup as "missing" and is counted.
__device__ __noinline__ int hash_block_lookup(const SessionDesc& s, short sx, short sy, short sz) {
  unsigned hi = hash_index(s.hmask, sx, sy, sz);
  for (int links = 0; links <= s.ne; ++links) {
    const HEntry en = load_entry(s.entries, hi);
    if (en.pos[0] == sx && en.pos[1] == sy && en.pos[2] == sz && en.ptr >= 0) return en.ptr * 512;
    if (en.offset < 1) return -1;
    if (en.offset > (unsigned)s.ne) break;
    hi = (unsigned)s.nb + en.offset - 1;
  }
  atomicAdd(&s.hcount[kHashChainFaults], 1);
  return -1;
}

// A warp's shared cache of block lookups: 64 direct-mapped 64-bit entries in shared memory,
// each the block's coordinates (14 bits an axis, offset by 8192; 16383 marks an empty
// entry) above its pool block index + 1 (22 bits; 0: not allocated).  The rays of a warp
// shade neighbouring pixels and walk largely the same blocks, so a lane finds most lookups
// another lane made.  An entry is written and read whole, so any lane sees a consistent
// (key, value) pair; the table does not change during the raycast.
constexpr int kWarpCache = 64;
__device__ __forceinline__ void warp_cache_clear(unsigned long long* wc) {
  const int lane = threadIdx.x & 31;
  wc[lane] = ~0ull;
  wc[lane + 32] = ~0ull;
  __syncwarp();
}

template <int HF>
struct HashRead {
  const SessionDesc& s;
  short cbx, cby, cbz;
  int cptr;  // cached block (findVoxelBlockIndex's cache; transparent to results)
  volatile unsigned long long* wc;  // the warp's shared lookup cache, or nullptr
  // Pool offset (block index * 512) of block (bx, by, bz), or -1 if it is not allocated.
  // The lookup itself is out of line: it is called from many places of the raycast, and
  // inlined copies of its chain walk overflow the instruction cache.
  __device__ __forceinline__ int block(int bx, int by, int bz) {
    const short sx = (short)bx, sy = (short)by, sz = (short)bz;
    if (cptr >= 0 && sx == cbx && sy == cby && sz == cbz) return cptr;
    const bool cacheable = wc && sx > -8192 && sx < 8191 && sy > -8192 && sy < 8191 && sz > -8192 && sz < 8191;
    unsigned long long key = 0;
    int slot = 0;
    int p;
    if (cacheable) {
      key = ((unsigned long long)(sx + 8192) << 28) | ((unsigned long long)(sy + 8192) << 14) |
            (unsigned long long)(sz + 8192);
      slot = (int)(hash_index(kWarpCache - 1, sx, sy, sz));
      const unsigned long long e = wc[slot];
      if ((e >> 22) == key) {
        p = (int)(e & 0x3fffffull) - 1;
        p = p < 0 ? -1 : p * 512;
        if (p >= 0) cbx = sx, cby = sy, cbz = sz, cptr = p;
        return p;
      }
    }
    p = hash_block_lookup(s, sx, sy, sz);
    if (cacheable) wc[slot] = (key << 22) | (unsigned long long)(p < 0 ? 0 : p / 512 + 1);
    if (p >= 0) {
      cbx = sx;
      cby = sy;
      cbz = sz;
      cptr = p;
    }
    return p;
  }
  // virtualVoxelPosToSDFBlock + the voxel's linear index (x + 8y + 64z); the reference's
  // rounding of negative coordinates toward -infinity is an arithmetic shift
  __device__ __forceinline__ int find(int vx, int vy, int vz) {
    const int b = block(vx >> 3, vy >> 3, vz >> 3);
    return b < 0 ? -1 : b + ((vx & 7) + 8 * (vy & 7) + 64 * (vz & 7));
  }
  // Neighbourhood reads.  Voxels (i + LO .. i + HI) on each axis span at most two blocks
  // per axis, so at most eight: each is looked up once, by every lane at the same call
  // site, and a voxel read then selects its block among them.  (Reading each neighbour
  // through its own lookup sent the lanes of a warp into two dozen separate divergent
  // calls.)
  struct Hood {
    int b0x, b0y, b0z;  // first block on each axis
    int P[8];           // pool offsets, index (bx - b0x) + 2 (by - b0y) + 4 (bz - b0z); -1: none
  };
  template <int LO, int HI>
  __device__ __forceinline__ void hood(Hood& h, int ix, int iy, int iz) {
    h.b0x = (ix + LO) >> 3;
    h.b0y = (iy + LO) >> 3;
    h.b0z = (iz + LO) >> 3;
    const int sx = ((ix + HI) >> 3) - h.b0x, sy = ((iy + HI) >> 3) - h.b0y, sz = ((iz + HI) >> 3) - h.b0z;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
      h.P[k] = (ox <= sx && oy <= sy && oz <= sz) ? block(h.b0x + ox, h.b0y + oy, h.b0z + oz) : -1;
    }
  }
  // pool index of voxel (x, y, z) of the neighbourhood, or -1 if its block is not allocated
  __device__ __forceinline__ int hood_index(const Hood& h, int x, int y, int z) const {
    const int sel = ((x >> 3) - h.b0x) + 2 * ((y >> 3) - h.b0y) + 4 * ((z >> 3) - h.b0z);
    int b = h.P[0];
#pragma unroll
    for (int k = 1; k < 8; ++k) b = sel == k ? h.P[k] : b;
    return b < 0 ? -1 : b + (x & 7) + 8 * (y & 7) + 64 * (z & 7);
  }
  __device__ __forceinline__ float hood_sdf(const Hood& h, int x, int y, int z) const {
    const int bi = hood_index(h, x, y, z);
    return bi < 0 ? 1.0f : HVox<HF>::load(s.hsdf, (unsigned)bi);
  }
};

// castRay + raycast_kernel (KinfuHashRaycast.cl:155-471): one thread per pixel.  The
// block cache of HashRead and the one-lookup neighbourhoods only save hash lookups; the
// values read are those of the reference's per-voxel findVoxelBlockIndex.

// The march of castRay (KinfuHashRaycast.cl:170-232) from (pr, total) until a surface
// (sdf <= 0) or the end of the range.
template <int HF>
__device__ __forceinline__ void hash_march(HashRead<HF>& R, const SessionDesc& s, float3& pr, float& total,
                                           const float totalMax, const float3 dir, const float stepScale, float& sdfv) {
  float stepLen;
  while (total < totalMax) {
    const int vx = (int)roundf(pr.x), vy = (int)roundf(pr.y), vz = (int)roundf(pr.z);
    const int bi = R.find(vx, vy, vz);
    if (bi < 0) {
      sdfv = 1.0f;
      stepLen = 8.0f;
    } else {
      sdfv = HVox<HF>::load(s.hsdf, (unsigned)bi);
      if (sdfv <= 0.1f && sdfv >= -0.5f) {
        const int ix = (int)floorf(pr.x), iy = (int)floorf(pr.y), iz = (int)floorf(pr.z);
        const float3 cf = f3(pr.x - (float)ix, pr.y - (float)iy, pr.z - (float)iz);
        typename HashRead<HF>::Hood h;
        R.template hood<0, 1>(h, ix, iy, iz);
        float v1 = R.hood_sdf(h, ix, iy, iz), v2 = R.hood_sdf(h, ix + 1, iy, iz);
        float r1 = (1.0f - cf.x) * v1 + cf.x * v2;
        v1 = R.hood_sdf(h, ix, iy + 1, iz);
        v2 = R.hood_sdf(h, ix + 1, iy + 1, iz);
        r1 = (1.0f - cf.y) * r1 + cf.y * ((1.0f - cf.x) * v1 + cf.x * v2);
        v1 = R.hood_sdf(h, ix, iy, iz + 1);
        v2 = R.hood_sdf(h, ix + 1, iy, iz + 1);
        float r2 = (1.0f - cf.x) * v1 + cf.x * v2;
        v1 = R.hood_sdf(h, ix, iy + 1, iz + 1);
        v2 = R.hood_sdf(h, ix + 1, iy + 1, iz + 1);
        r2 = (1.0f - cf.y) * r2 + cf.y * ((1.0f - cf.x) * v1 + cf.x * v2);
        sdfv = (1.0f - cf.z) * r1 + cf.z * r2;
      }
      if (sdfv <= 0.0f) return;
      stepLen = fmaxf(sdfv * stepScale, 1.0f);
    }
    pr = add3(pr, mul3(dir, stepLen));
    total += stepLen;
  }
}

// Ray of pixel pid: start and end of the expected range in voxel units, and direction.
template <int HF>
__device__ __forceinline__ void hash_ray(const SessionDesc& s, int pid, float3& ps, float& total, float& totalMax,
                                         float3& dir) {
  const int px = pid % s.W, py = pid / s.W;
  const DevXform& m = s.ts->xf;
  const float2 mm = s.range[pid];
  const float oov = 1.0f / s.voxel;
  ps = depth_to_point(s.cam, px, py, mm.x);
  total = sqrtf(dot3(ps, ps)) * oov;
  ps = mul3(xf_apply(m, ps), oov);
  float3 pe = depth_to_point(s.cam, px, py, mm.y);
  totalMax = sqrtf(dot3(pe, pe)) * oov;
  pe = mul3(xf_apply(m, pe), oov);
  dir = normalize3(sub3(pe, ps));
}

// The surface refinement, normal and colour of castRay / raycast_kernel
// (KinfuHashRaycast.cl:233-471) and the map writes of pixel pid.
template <int HF, bool NORMALS = true>
__device__ __forceinline__ void hash_finish(HashRead<HF>& R, const SessionDesc& s, int pid, float3 pr,
                                            const float3 dir, const float stepScale, float sdfv) {
  float stepLen;
  const float4 nanv = make_float4(qnan(), qnan(), qnan(), 0.f);
  float4 vout = nanv, nout = nanv;
  uchar4 col = make_uchar4(0, 0, 0, 0);
  if (sdfv <= 0.0f) {
    stepLen = sdfv * stepScale;
    pr = add3(pr, mul3(dir, stepLen));
    const int ix = (int)floorf(pr.x), iy = (int)floorf(pr.y), iz = (int)floorf(pr.z);
    const float3 cf = f3(pr.x - (float)ix, pr.y - (float)iy, pr.z - (float)iz);
    const float3 nc = f3(1.0f - cf.x, 1.0f - cf.y, 1.0f - cf.z);
    float fb[8];
    float nearest = 1.0e20f;
    // one neighbourhood for the corners and the gradient's outer samples
    typename HashRead<HF>::Hood h;
    R.template hood<-1, 2>(h, ix, iy, iz);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
      const int bi = R.hood_index(h, ix + ox, iy + oy, iz + oz);
      fb[k] = bi < 0 ? 1.0f : HVox<HF>::load(s.hsdf, (unsigned)bi);
      const float3 dd = f3(ox ? nc.x : cf.x, oy ? nc.y : cf.y, oz ? nc.z : cf.z);
      const float cd = sqrtf(dot3(dd, dd));
      if (s.cmap && s.hrgb && bi >= 0 && (k == 0 || nearest > cd)) {
        nearest = cd;
        const uchar4 v = s.hrgb[bi];
        col = make_uchar4(v.x, v.y, v.z, 255);
      }
    }
    sdfv = fb[0] * nc.x * nc.y * nc.z + fb[1] * cf.x * nc.y * nc.z + fb[2] * nc.x * cf.y * nc.z +
           fb[3] * cf.x * cf.y * nc.z + fb[4] * nc.x * nc.y * cf.z + fb[5] * cf.x * nc.y * cf.z +
           fb[6] * nc.x * cf.y * cf.z + fb[7] * cf.x * cf.y * cf.z;
    stepLen = sdfv * stepScale;
    pr = add3(pr, mul3(dir, stepLen));
    vout = w0(mul3(pr, s.voxel));
    if (!NORMALS) {  // the forward render casts without normals (genericRaycastMissingPoints_kernel)
      s.vref[pid] = vout;
      if (s.cmap) s.cmap[pid] = col;
      return;
    }
    float p1, p2, v1;
    auto nr = [&](int dx, int dy, int dz) { return R.hood_sdf(h, ix + dx, iy + dy, iz + dz); };
    float3 g;
    p1 = fb[0] * nc.y * nc.z + fb[2] * cf.y * nc.z + fb[4] * nc.y * cf.z + fb[6] * cf.y * cf.z;
    p2 = nr(-1, 0, 0) * nc.y * nc.z + nr(-1, +1, 0) * cf.y * nc.z +
         nr(-1, 0, +1) * nc.y * cf.z + nr(-1, +1, +1) * cf.y * cf.z;
    v1 = p1 * cf.x + p2 * nc.x;
    p1 = fb[1] * nc.y * nc.z + fb[3] * cf.y * nc.z + fb[5] * nc.y * cf.z + fb[7] * cf.y * cf.z;
    p2 = nr(+2, 0, 0) * nc.y * nc.z + nr(+2, +1, 0) * cf.y * nc.z +
         nr(+2, 0, +1) * nc.y * cf.z + nr(+2, +1, +1) * cf.y * cf.z;
    g.x = p1 * nc.x + p2 * cf.x - v1;
    p1 = fb[0] * nc.x * nc.z + fb[1] * cf.x * nc.z + fb[4] * nc.x * cf.z + fb[5] * cf.x * cf.z;
    p2 = nr(0, -1, 0) * nc.x * nc.z + nr(+1, -1, 0) * cf.x * nc.z +
         nr(0, -1, +1) * nc.x * cf.z + nr(+1, -1, +1) * cf.x * cf.z;
    v1 = p1 * cf.y + p2 * nc.y;
    p1 = fb[2] * nc.x * nc.z + fb[3] * cf.x * nc.z + fb[6] * nc.x * cf.z + fb[7] * cf.x * cf.z;
    p2 = nr(0, +2, 0) * nc.x * nc.z + nr(+1, +2, 0) * cf.x * nc.z +
         nr(0, +2, +1) * nc.x * cf.z + nr(+1, +2, +1) * cf.x * cf.z;
    g.y = p1 * nc.y + p2 * cf.y - v1;
    p1 = fb[0] * nc.x * nc.y + fb[1] * cf.x * nc.y + fb[2] * nc.x * cf.y + fb[3] * cf.x * cf.y;
    p2 = nr(0, 0, -1) * nc.x * nc.y + nr(+1, 0, -1) * cf.x * nc.y +
         nr(0, +1, -1) * nc.x * cf.y + nr(+1, +1, -1) * cf.x * cf.y;
    v1 = p1 * cf.z + p2 * nc.z;
    p1 = fb[4] * nc.x * nc.y + fb[5] * cf.x * nc.y + fb[6] * nc.x * cf.y + fb[7] * cf.x * cf.y;
    p2 = nr(0, 0, +2) * nc.x * nc.y + nr(+1, 0, +2) * cf.x * nc.y +
         nr(0, +1, +2) * nc.x * cf.y + nr(+1, +1, +2) * cf.x * cf.y;
    g.z = p1 * nc.z + p2 * cf.z - v1;
    nout = w0(normalize3(g));
  }
  s.vref[pid] = vout;
  if (NORMALS) s.nref[pid] = nout;
  if (s.cmap) s.cmap[pid] = col;
}

template <int HF>
__global__ void __launch_bounds__(128, 8) k_hash_raycast(const SessionDesc* __restrict__ descs, int tw) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.hash || s.fwd || s.hfmt != HF || s.kind != kTrackFrame || s.ts->status != 0) return;
  // each warp shades a tw x (32 / tw) pixel tile, a block 2 x 2 of them (neighbouring rays
  // march alike; tw is tuned)
  const int th = 32 / tw, bw = 2 * tw, bh = 2 * th;
  const int tiles_x = (s.W + bw - 1) / bw;
  if ((int)blockIdx.x >= tiles_x * ((s.H + bh - 1) / bh)) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ unsigned long long wcache[4][kWarpCache];
  warp_cache_clear(wcache[warp]);
  const int px = ((int)blockIdx.x % tiles_x) * bw + (warp & 1) * tw + lane % tw;
  const int py = ((int)blockIdx.x / tiles_x) * bh + (warp >> 1) * th + lane / tw;
  if (px >= s.W || py >= s.H) return;
  const int pid = py * s.W + px;
  HashRead<HF> R{s, 0, 0, 0, -1, wcache[warp]};
  const float stepScale = s.mu * (1.0f / s.voxel) * 0.6f;
  float3 pr, dir;
  float total, totalMax, sdfv = 1.0f;
  hash_ray<HF>(s, pid, pr, total, totalMax, dir);
  hash_march<HF>(R, s, pr, total, totalMax, dir, stepScale, sdfv);
  // the march's end point and last sdf wait in the vertex map for k_hash_finish
  s.vref[pid] = make_float4(pr.x, pr.y, pr.z, sdfv);
}

// The surface refinement, normal and colour of every pixel after the march: a kernel of
// its own, so that each of the two stays small in the instruction cache (the refinement's
// many neighbourhood reads and the march's lookups do not fit it together), and the
// refining lanes of a warp run together.
template <int HF>
__global__ void __launch_bounds__(256, 4) k_hash_finish(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.hash || s.fwd || s.hfmt != HF || s.kind != kTrackFrame || s.ts->status != 0) return;
  const int pid = blockIdx.x * blockDim.x + threadIdx.x;
  if (pid >= s.W * s.H) return;
  const float4 e = s.vref[pid];
  HashRead<HF> R{s, 0, 0, 0, -1};  // (a warp-shared lookup cache made this kernel slower)
  const float stepScale = s.mu * (1.0f / s.voxel) * 0.6f;
  float3 ps, dir;
  float total, totalMax;
  hash_ray<HF>(s, pid, ps, total, totalMax, dir);
  hash_finish<HF>(R, s, pid, f3(e.x, e.y, e.z), dir, stepScale, e.w);
}

// ------------------------------------------------------------------ forward rendering
// ForwardRender of the hash scene (NuiKinfuOpenCLHashScene.cpp:991-1012; forwardProject_kernel,
// findMissingPoints_kernel, genericRaycastMissingPoints_kernel, KinfuHashRaycast.cl:473-559,
// then estimate_normals_simple_kernel, normalEstimation.cl:770-822).  The previous reference
// maps' vertices land on the pixels they project to; only pixels nothing lands on whose
// expected range is not empty are raycast, listed in increasing order by a scan; normals are
// recomputed from the new vertex map.  Where several vertices land on one pixel the last in
// raster order wins (an atomic max of the source index: the reference's unordered stores
// made deterministic); colours are read from the previous map, not from the map being
// written (the reference copies them within one buffer).

// Where each previous vertex lands (mode 1: the reference's transform(p) * voxel; mode 2:
// the world point taken into the camera).  A coordinate in (-1, 0) truncates to pixel 0, as
// the reference's float-to-uint conversion does.
__global__ void __launch_bounds__(256) k_fwd_project(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.hash || !s.fwd || s.kind != kTrackFrame || s.ts->status != 0) return;
  const int W = s.W, H = s.H, n = W * H;
  const DevXform& m = s.ts->xf;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float3 p = xyz(s.vref[i]);
    if (isnan3(p)) continue;
    const float3 q = s.fwd == 2 ? xf_inverse(m, p) : mul3(xf_apply(m, p), s.voxel);
    const float u = q.x * s.cam.fx / q.z + s.cam.cx + 0.5f, v = q.y * s.cam.fy / q.z + s.cam.cy + 0.5f;
    if (!(u > -1.0f && v > -1.0f)) continue;
    const float tu = truncf(u), tv = truncf(v);
    if (!(tu < (float)W && tv < (float)H)) continue;
    atomicMax(s.fwd_owner + (int)tv * W + (int)tu, i + 1);
  }
}

__device__ __forceinline__ bool fwd_missing(const SessionDesc& s, int t, float landed_x) {
  const float2 mm = s.range[t];
  return isnan(landed_x) && mm.x < mm.y;
}

// Per pixel (1024 a block): the landed vertex (into nref, kept there until the commit) and
// colour, and the block's count of missing pixels.
__global__ void __launch_bounds__(1024) k_fwd_fill(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.hash || !s.fwd || s.kind != kTrackFrame || s.ts->status != 0) return;
  const int n = s.W * s.H;
  if ((int)blockIdx.x * 1024 >= n) return;
  const int t = blockIdx.x * 1024 + threadIdx.x;
  bool miss = false;
  if (t < n) {
    const int o = s.fwd_owner[t];
    const float4 v = o > 0 ? s.vref[o - 1] : make_float4(qnan(), qnan(), qnan(), 0.f);
    s.nref[t] = v;
    if (s.cmap) s.fwd_col[t] = o > 0 ? s.cmap[o - 1] : make_uchar4(0, 0, 0, 0);
    miss = fwd_missing(s, t, v.x);
  }
  const int c = __syncthreads_count(miss);
  if (threadIdx.x == 0) s.fwd_blk[blockIdx.x] = (unsigned)c;
}

// Exclusive scan of the per-block counts (one block per session); the total goes to hcount[11].
__global__ void __launch_bounds__(1024) k_fwd_scan(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.hash || !s.fwd || s.kind != kTrackFrame || s.ts->status != 0) return;
  const int nb = (s.W * s.H + 1023) / 1024;  // <= 1024 (images up to 1M pixels)
  __shared__ unsigned wsum[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned c = (int)threadIdx.x < nb ? s.fwd_blk[threadIdx.x] : 0u;
  unsigned incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    unsigned w = wsum[lane], wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    wsum[lane] = wi - w;
  }
  __syncthreads();
  const unsigned excl = wsum[warp] + incl - c;
  if ((int)threadIdx.x < nb) s.fwd_blk[threadIdx.x] = excl;
  if ((int)threadIdx.x == nb - 1) s.hcount[11] = (int)(excl + c);
}

// The new maps: landed vertices and colours (NaN / 0 where nothing landed), and the missing
// pixels listed in increasing order.
__global__ void __launch_bounds__(1024) k_fwd_commit(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.hash || !s.fwd || s.kind != kTrackFrame || s.ts->status != 0) return;
  const int n = s.W * s.H;
  if ((int)blockIdx.x * 1024 >= n) return;
  const int t = blockIdx.x * 1024 + threadIdx.x;
  bool miss = false;
  if (t < n) {
    const float4 v = s.nref[t];
    s.vref[t] = v;
    if (s.cmap) s.cmap[t] = s.fwd_col[t];
    miss = fwd_missing(s, t, v.x);
  }
  __shared__ unsigned wsum[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned b = __ballot_sync(0xffffffffu, miss);
  if (lane == 0) wsum[warp] = __popc(b);
  __syncthreads();
  unsigned before = 0;
  for (int w = 0; w < warp; ++w) before += wsum[w];
  if (miss) s.fwd_ids[s.fwd_blk[blockIdx.x] + before + __popc(b & ((1u << lane) - 1u))] = t;
}

// castRay of the listed pixels (genericRaycastMissingPoints_kernel): the march, its end
// waiting in nref for the refinement.
template <int HF>
__global__ void __launch_bounds__(128, 8) k_fwd_raycast(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.hash || !s.fwd || s.hfmt != HF || s.kind != kTrackFrame || s.ts->status != 0) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= s.hcount[11]) return;
  const int pid = s.fwd_ids[k];
  HashRead<HF> R{s, 0, 0, 0, -1};
  const float stepScale = s.mu * (1.0f / s.voxel) * 0.6f;
  float3 pr, dir;
  float total, totalMax, sdfv = 1.0f;
  hash_ray<HF>(s, pid, pr, total, totalMax, dir);
  hash_march<HF>(R, s, pr, total, totalMax, dir, stepScale, sdfv);
  s.nref[pid] = make_float4(pr.x, pr.y, pr.z, sdfv);
}

// The refinement and colour of the listed pixels (no normals: they follow from the map).
template <int HF>
__global__ void __launch_bounds__(256, 4) k_fwd_finish(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.hash || !s.fwd || s.hfmt != HF || s.kind != kTrackFrame || s.ts->status != 0) return;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= s.hcount[11]) return;
  const int pid = s.fwd_ids[k];
  const float4 e = s.nref[pid];
  HashRead<HF> R{s, 0, 0, 0, -1};
  const float stepScale = s.mu * (1.0f / s.voxel) * 0.6f;
  float3 ps, dir;
  float total, totalMax;
  hash_ray<HF>(s, pid, ps, total, totalMax, dir);
  hash_finish<HF, false>(R, s, pid, f3(e.x, e.y, e.z), dir, stepScale, e.w);
}

// Vertex2Normal (NuiKinfuOpenCLHashScene.cpp:940-983): estimate_normals_simple_kernel over the
// new world vertex map, depth threshold 0.3 m.
__global__ void __launch_bounds__(256) k_fwd_normals(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.hash || !s.fwd || s.kind != kTrackFrame || s.ts->status != 0) return;
  const int W = s.W, H = s.H;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W * H) return;
  const int x = i % W, y = i / W;
  const float thr = 0.3f;
  const float3 c = xyz(s.vref[i]);
  if (isnan3(c)) {
    s.nref[i] = make_float4(qnan(), qnan(), qnan(), 0.f);
    return;
  }
  auto pick = [&](bool ok, int j) {
    if (!ok) return c;
    const float3 q = xyz(s.vref[j]);
    if (isnan3(q) || fabsf(c.z - q.z) > thr) return c;
    return q;
  };
  const float3 l = pick(x > 0, i - 1), r = pick(x < W - 1, i + 1);
  const float3 u = pick(y > 0, i - W), d = pick(y < H - 1, i + W);
  s.nref[i] = w0(normalize3(cross3(sub3(r, l), sub3(d, u))));
}

template __global__ void k_fwd_raycast<0>(const SessionDesc*);
template __global__ void k_fwd_raycast<1>(const SessionDesc*);
template __global__ void k_fwd_finish<0>(const SessionDesc*);
template __global__ void k_fwd_finish<1>(const SessionDesc*);

// ------------------------------------------------------------------ global cache
// NuiKinfuOpenCLHashGlobalCache (NuiKinfuOpenCLHashGlobalCache.cpp:121-538) with its
// kernels (KinfuHashSwapping.cl:6-180).  The reference keeps the host store in host memory
// and moves blocks through a transfer buffer with blocking copies and host loops; here the
// store is pinned host memory mapped into the device, and the swap kernels read and write
// it directly over the bus, inside the tick.  Lists hold the flagged entries in index
// order, at most kTransferBlocks (SDF_TRANSFER_BLOCK_NUM) per operation; pops and pushes of
// the free list follow that order, as the reference's atomics do when run in order.

// After the visible list: re-allocation of swapped-out visible entries
// (reAllocateSwappedOutVoxelBlocks_kernel, :6-22) and the swap-in list.
__global__ void __launch_bounds__(kHashScanBlock) k_hash_swap_lists(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s) || !s.swapping) return;
  const unsigned n = (unsigned)(s.nb + s.ne);
  const unsigned b = blockIdx.x;
  if (b * kHashScanBlock >= n) return;
  const unsigned i = b * kHashScanBlock + threadIdx.x;
  bool fr, fi;
  unsigned tr, ti;
  const unsigned rr = block_rank(i, n, [&](unsigned k) { return s.vis[k] > 0 && entry_ptr(s, k) == -1; }, fr, tr);
  const unsigned ri = block_rank(i, n, [&](unsigned k) { return s.swap[k] == 1; }, fi, ti);
  if (fr) {
    const int vba = s.hcount[6] - (int)(s.blk[4 * b + 2] + rr);
    if (vba >= 0) reinterpret_cast<int*>(s.entries)[4 * i + 2] = s.alloc_list[vba];
  }
  if (fi) {
    const unsigned g = s.blk[4 * b + 3] + ri;
    if (g < (unsigned)kTransferBlocks) s.swap_in_ids[g] = (int)i;
  }
}

// After the integration: integrateOldIntoActiveData_kernel (:62-111).  One block per listed
// entry: its stored copy (zeros if it has none) is merged into the local block by weight.
template <int HF>
__global__ void __launch_bounds__(512) k_hash_swap_in(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s) || !s.swapping) return;
  const int nin = s.hcount[4];
  const int lid = threadIdx.x;
  for (int k = blockIdx.x; k < nin; k += gridDim.x) {
    const int id = s.swap_in_ids[k];
    const int ptr = entry_ptr(s, (unsigned)id);
    if (ptr < 0) continue;
    const int slot = s.store_slot[id];
    float oldF = 0.f, oldW = 0.f;
    uchar4 oc = make_uchar4(0, 0, 0, 0);
    if (slot >= 0) {
      const size_t si = (size_t)slot * 512 + lid;
      oldF = HVox<HF>::load(s.st_sdf, (unsigned)si);
      oldW = (float)s.st_w[si];
      if (s.st_rgb) oc = s.st_rgb[si];
    }
    const unsigned bi = (unsigned)ptr * 512u + (unsigned)lid;
    const float newW = (float)s.hw[bi], cw = oldW + newW;
    float newF = HVox<HF>::load(s.hsdf, bi);
    newF = oldW * oldF + newW * newF;
    newF /= cw;
    // both weights 0: 0 / 0, whose conversions give 0 (as on the reference's x86 host)
    HVox<HF>::store(s.hsdf, bi, isnan(newF) ? 0.f : newF);
    s.hw[bi] = (uint8_t)min((int)(uint8_t)(int)cw, s.max_w);
    if (s.hrgb) {
      const uchar4 lc = s.hrgb[bi];
      auto mix = [&](float o, float l) -> unsigned char {
        const float v = (oldW * o + newW * l) / cw;
        return isnan(v) ? (unsigned char)0 : (unsigned char)(int)fminf(fmaxf(v, 0.f), 255.f);
      };
      s.hrgb[bi] = make_uchar4(mix(oc.x, lc.x), mix(oc.y, lc.y), mix(oc.z, lc.z), lc.w);
    }
    if (lid == 0) s.swap[id] = 2;
  }
}

// The swap-out list (buildSwapOutList_kernel, :113-124), then a store slot for every listed
// entry that has none yet (an entry keeps its slot; a full store refuses the entry, which
// then stays in the device pool: -1 in the list).
__global__ void __launch_bounds__(kHashScanBlock) k_hash_swap_out_list(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s) || !s.swapping) return;
  const unsigned n = (unsigned)(s.nb + s.ne);
  const unsigned b = blockIdx.x;
  if (b * kHashScanBlock >= n) return;
  const unsigned i = b * kHashScanBlock + threadIdx.x;
  bool f;
  unsigned t;
  const unsigned r = block_rank(i, n, [&](unsigned k) { return swap_out_flag(s, k); }, f, t);
  if (!f) return;
  const unsigned g = s.blk[4 * b + 2] + r;
  if (g >= (unsigned)kTransferBlocks) return;
  int id = (int)i;
  if (s.store_slot[i] < 0) {
    const int slot = atomicAdd(&s.hcount[7], 1);
    if (slot < s.st_cap) {
      s.store_slot[i] = slot;
    } else {
      atomicAdd(&s.hcount[8], 1);
      id = -1;
    }
  }
  s.swap_out_ids[g] = id;
}

// moveActiveDataToTransferBuffer_kernel (:126-153): the local block goes to the entry's
// store slot and is cleared (sdf 0, weight 0, colour 0).
template <int HF>
__global__ void __launch_bounds__(512) k_hash_swap_out(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!hash_active(s) || !s.swapping) return;
  const int nout = s.hcount[5];
  const int lid = threadIdx.x;
  for (int k = blockIdx.x; k < nout; k += gridDim.x) {
    const int id = s.swap_out_ids[k];
    if (id < 0) continue;
    const int ptr = entry_ptr(s, (unsigned)id);
    const unsigned bi = (unsigned)ptr * 512u + (unsigned)lid;
    const size_t si = (size_t)s.store_slot[id] * 512 + lid;
    if (HF == 0)
      reinterpret_cast<short*>(s.st_sdf)[si] = reinterpret_cast<const short*>(s.hsdf)[bi];
    else
      reinterpret_cast<__half*>(s.st_sdf)[si] = reinterpret_cast<const __half*>(s.hsdf)[bi];
    s.st_w[si] = s.hw[bi];
    if (s.st_rgb) s.st_rgb[si] = s.hrgb ? s.hrgb[bi] : make_uchar4(0, 0, 0, 0);
    HVox<HF>::store(s.hsdf, bi, 0.f);
    s.hw[bi] = 0;
    if (s.hrgb) s.hrgb[bi] = make_uchar4(0, 0, 0, 0);
  }
}

// cleanVoxelMemory_kernel (:155-180): the swapped-out entries leave state 2 and push their
// blocks on the free list (atomic_inc in list order); one block per session.
__global__ void __launch_bounds__(1024) k_hash_swap_clean(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.x];
  if (!hash_active(s) || !s.swapping) return;
  __shared__ int base;
  __shared__ unsigned wsum[32];
  __shared__ unsigned carry;
  if (threadIdx.x == 0) {
    base = s.hcount[0];
    carry = 0;
  }
  __syncthreads();
  const int nout = s.hcount[5];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k0 = 0; k0 < nout; k0 += 1024) {
    const int k = k0 + (int)threadIdx.x;
    const int id = k < nout ? s.swap_out_ids[k] : -1;
    const bool f = id >= 0;
    const unsigned ballot = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wsum[warp] = __popc(ballot);
    __syncthreads();
    unsigned before = carry;
    for (int w = 0; w < warp; ++w) before += wsum[w];
    const unsigned rank = before + __popc(ballot & ((1u << lane) - 1u));
    if (f) {
      s.swap[id] = 0;
      const int vba = base + (int)rank;
      if (vba < s.np - 1) {
        s.alloc_list[vba + 1] = entry_ptr(s, (unsigned)id);
        reinterpret_cast<int*>(s.entries)[4 * id + 2] = -1;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned tot = 0;
      for (int w = 0; w < 32; ++w) tot += wsum[w];
      carry += tot;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) s.hcount[0] = base + (int)carry;
}

// fetchHashScene_kernel (KinfuHashVisualization.cl:5-52), launched as
// NuiKinfuOpenCLHashScene::Volume2CLVertices does (NuiKinfuOpenCLHashScene.cpp:1066-1180):
// a point at the centre of every weighted voxel of a visible block whose |sdf| is below
// truncScale (compared in the int16 scale of the reference's voxels), with the voxel's
// colour / 255 and alpha 1.  One block per visible entry, one thread per voxel; points are
// appended atomically (no fixed order), at most cap of them.
template <int HF>
__global__ void __launch_bounds__(512) k_hash_fetch(const SessionDesc* __restrict__ descs, float* xyz, float* rgba,
                                                    long long cap, unsigned long long* counter) {
  const SessionDesc& s = descs[0];
  const int nvis = s.hcount[2];
  const float lim = 32767.f * s.mu;
  const int i = threadIdx.x;
  for (int v = blockIdx.x; v < nvis; v += gridDim.x) {
    const int id = s.vis_ids[v];
    if (id < 0) continue;
    const HEntry en = load_entry(s.entries, (unsigned)id);
    if (en.ptr < 0) continue;
    const unsigned bi = (unsigned)en.ptr * 512u + (unsigned)i;
    if (s.hw[bi] == 0) continue;
    const float a = HF == 0 ? (float)abs((int)reinterpret_cast<const short*>(s.hsdf)[bi])
                            : fabsf(HVox<1>::load(s.hsdf, bi) * 32767.f);
    if (!(a < lim)) continue;
    const unsigned long long k = atomicAdd(counter, 1ull);
    if ((long long)k >= cap) continue;
    xyz[3 * k + 2] = ((float)(en.pos[2] * 8) + ((float)(i / 64) + 0.5f)) * s.voxel;
    xyz[3 * k + 1] = ((float)(en.pos[1] * 8) + ((float)((i % 64) / 8) + 0.5f)) * s.voxel;
    xyz[3 * k + 0] = ((float)(en.pos[0] * 8) + ((float)((i % 64) % 8) + 0.5f)) * s.voxel;
    const uchar4 c = s.hrgb ? s.hrgb[bi] : make_uchar4(0, 0, 0, 0);
    reinterpret_cast<float4*>(rgba)[k] = make_float4((float)c.x / 255.f, (float)c.y / 255.f, (float)c.z / 255.f, 1.f);
  }
}

template __global__ void k_hash_swap_in<0>(const SessionDesc*);
template __global__ void k_hash_swap_in<1>(const SessionDesc*);
template __global__ void k_hash_swap_out<0>(const SessionDesc*);
template __global__ void k_hash_swap_out<1>(const SessionDesc*);
template __global__ void k_hash_fetch<0>(const SessionDesc*, float*, float*, long long, unsigned long long*);
template __global__ void k_hash_fetch<1>(const SessionDesc*, float*, float*, long long, unsigned long long*);
template __global__ void k_hash_integrate<0>(const SessionDesc*);
template __global__ void k_hash_integrate<1>(const SessionDesc*);
template __global__ void k_hash_raycast<0>(const SessionDesc*, int);
template __global__ void k_hash_raycast<1>(const SessionDesc*, int);
template __global__ void k_hash_finish<0>(const SessionDesc*);
template __global__ void k_hash_finish<1>(const SessionDesc*);

}  // namespace nui

namespace nui {
// NuiKinfuVoxelBlockHash::reset (NuiKinfuVoxelBlockHash.cpp:78-213): every entry free,
// identity free lists, every voxel (sdf 0, weight 0, colour 0).
__global__ void k_hash_reset(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[0];
  const size_t ne = (size_t)s.nb + s.ne, nv = (size_t)s.np * 512;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t t0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (size_t i = t0; i < ne; i += stride) {
    HEntry e;
    e.pos[0] = e.pos[1] = e.pos[2] = 0;
    e.pad = 0;
    e.ptr = -2;
    e.offset = 0;
    store_entry(s.entries, (unsigned)i, e);
    s.alloc_type[i] = 0;
    s.vis[i] = 0;
    s.keys[i] = 0ull;
  }
  for (size_t i = t0; i < (size_t)s.np; i += stride) s.alloc_list[i] = (int)i;
  for (size_t i = t0; i < (size_t)s.ne; i += stride) s.excess_list[i] = (int)i;
  for (size_t i = t0; i < nv; i += stride) {
    if (s.hfmt == 0)
      reinterpret_cast<short*>(s.hsdf)[i] = 0;
    else
      reinterpret_cast<__half*>(s.hsdf)[i] = __float2half_rn(0.f);
    s.hw[i] = 0;
    if (s.hrgb) s.hrgb[i] = make_uchar4(0, 0, 0, 0);
  }
  if (s.swapping)
    for (size_t i = t0; i < ne; i += stride) {
      s.swap[i] = 0;
      s.store_slot[i] = -1;
    }
  if (t0 == 0) {
    s.hcount[0] = s.np - 1;
    s.hcount[1] = s.ne - 1;
    s.hcount[2] = 0;
    s.hcount[3] = 0;
    for (int k = 4; k < 16; ++k) s.hcount[k] = 0;
  }
}

// Pool voxels in the reference's AoS layout (short sdf, uchar rgb[3], uchar weight).
__global__ void k_hash_export_voxels(const SessionDesc* __restrict__ descs, uint8_t* out) {
  const SessionDesc& s = descs[0];
  const size_t nv = (size_t)s.np * 512;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += (size_t)gridDim.x * blockDim.x) {
    short v;
    if (s.hfmt == 0)
      v = reinterpret_cast<const short*>(s.hsdf)[i];
    else
      v = (short)__float2int_rz(__half2float(reinterpret_cast<const __half*>(s.hsdf)[i]) * 32767.0f);
    uint8_t* o = out + 6 * i;
    o[0] = (uint8_t)(v & 0xff);
    o[1] = (uint8_t)((unsigned short)v >> 8);
    const uchar4 c = s.hrgb ? s.hrgb[i] : make_uchar4(0, 0, 0, 0);
    o[2] = c.x;
    o[3] = c.y;
    o[4] = c.z;
    o[5] = s.hw[i];
  }
}
}  // namespace nui

// ------------------------------------------------------------------ marching cubes
// meshHashScene_kernel (KinfuHashVisualization.cl:88-271): the cubes of every visible
// block, emitted in visible-list order, voxels z-y-x inside a block (thread id = x + 8y +
// 64z), triangles in table order.  No weight test: the reference reads sdf alone.
namespace nui {
__constant__ uint64_t c_htri[256];
void hash_mc_upload_tables(cudaStream_t st, const uint64_t* table) {
  cudaMemcpyToSymbolAsync(c_htri, table, 256 * sizeof(uint64_t), 0, cudaMemcpyHostToDevice, st);
}

template <int HF>
__device__ __forceinline__ int hash_cube(HashRead<HF>& R, int vx, int vy, int vz, float* sv) {
  const int CX[8] = {0, 1, 1, 0, 0, 1, 1, 0}, CY[8] = {0, 0, 1, 1, 0, 0, 1, 1}, CZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};
  int cube = 0;
  for (int k = 0; k < 8; ++k) {
    const int bi = R.find(vx + CX[k], vy + CY[k], vz + CZ[k]);
    if (bi < 0) return -1;
    sv[k] = HVox<HF>::load(R.s.hsdf, (unsigned)bi);
    if (sv[k] < 0) cube |= 1 << k;
  }
  return cube;
}

template <int HF>
__global__ void __launch_bounds__(512) k_hash_mesh_count(const SessionDesc* __restrict__ descs, unsigned* cnt) {
  const SessionDesc& s = descs[0];
  const int nvis = s.hcount[2];
  __shared__ unsigned wsum[16];
  HashRead<HF> R{s, 0, 0, 0, -1};
  for (int k = blockIdx.x; k < nvis; k += gridDim.x) {
    const HEntry en = load_entry(s.entries, (unsigned)s.vis_ids[k]);
    unsigned n = 0;
    if (en.ptr >= 0) {
      const int lid = threadIdx.x;
      float sv[8];
      const int c = hash_cube<HF>(R, en.pos[0] * 8 + (lid & 7), en.pos[1] * 8 + ((lid >> 3) & 7),
                                  en.pos[2] * 8 + (lid >> 6), sv);
      if (c >= 0) n = 3u * (unsigned)(c_htri[c] >> 60);
    }
    n = __reduce_add_sync(0xffffffffu, n);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned t = 0;
      for (int w = 0; w < 16; ++w) t += wsum[w];
      cnt[k] = t;
    }
    __syncthreads();
  }
}

// In-place exclusive scan of n counts (u32 -> u64 offsets), total at off[n].
__global__ void __launch_bounds__(1024) k_hash_mesh_scan(const unsigned* cnt, unsigned long long* off, int n) {
  __shared__ unsigned long long wt[32];
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < n; base += 1024) {
    const int i = base + threadIdx.x;
    const unsigned long long v = i < n ? cnt[i] : 0ull;
    unsigned long long inc = v;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) wt[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      const unsigned long long w = wt[lane];
      unsigned long long wi = w;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long t = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane >= o) wi += t;
      }
      wt[lane] = wi - w;
    }
    __syncthreads();
    const unsigned long long ex = carry + wt[warp] + inc - v;
    __syncthreads();
    if (i < n) off[i] = ex;
    if (threadIdx.x == 1023) carry = ex + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) off[n] = carry;
}

__device__ __forceinline__ float3 sdf_interp3(float3 p1, float3 p2, float v1, float v2) {
  if (fabsf(0.0f - v1) < 0.00001f) return p1;
  if (fabsf(0.0f - v2) < 0.00001f) return p2;
  if (fabsf(v1 - v2) < 0.00001f) return p1;
  return add3(p1, mul3(sub3(p2, p1), (0.0f - v1) / (v2 - v1)));
}

template <int HF>
__global__ void __launch_bounds__(512) k_hash_mesh_emit(const SessionDesc* __restrict__ descs,
                                                        const unsigned long long* off, float* pos, float* col,
                                                        unsigned long long cap) {
  const SessionDesc& s = descs[0];
  const int nvis = s.hcount[2];
  __shared__ unsigned wsum[16];
  HashRead<HF> R{s, 0, 0, 0, -1};
  const int lid = threadIdx.x, lane = lid & 31, warp = lid >> 5;
  const int CX[8] = {0, 1, 1, 0, 0, 1, 1, 0}, CY[8] = {0, 0, 1, 1, 0, 0, 1, 1}, CZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};
  const int E0[12] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3}, E1[12] = {1, 2, 3, 0, 5, 6, 7, 4, 4, 5, 6, 7};
  for (int k = blockIdx.x; k < nvis; k += gridDim.x) {
    const HEntry en = load_entry(s.entries, (unsigned)s.vis_ids[k]);
    float sv[8];
    int c = -1;
    const int vx = en.pos[0] * 8 + (lid & 7), vy = en.pos[1] * 8 + ((lid >> 3) & 7), vz = en.pos[2] * 8 + (lid >> 6);
    if (en.ptr >= 0) c = hash_cube<HF>(R, vx, vy, vz, sv);
    const unsigned n = c >= 0 ? 3u * (unsigned)(c_htri[c] >> 60) : 0u;
    unsigned inc = n;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    unsigned before = 0;
    for (int w = 0; w < warp; ++w) before += wsum[w];
    __syncthreads();
    unsigned long long out = off[k] + before + inc - n;
    if (n == 0) continue;
    const uint64_t word = c_htri[c];
    float3 pt[8], cl[8];
    for (int q = 0; q < 8; ++q) {
      pt[q] = f3((float)(vx + CX[q]), (float)(vy + CY[q]), (float)(vz + CZ[q]));
      cl[q] = f3(0.f, 0.f, 0.f);
      if (col && s.hrgb) {
        const int bi = R.find(vx + CX[q], vy + CY[q], vz + CZ[q]);
        const uchar4 v = s.hrgb[bi];
        cl[q] = f3((float)v.x / 255.f, (float)v.y / 255.f, (float)v.z / 255.f);
      }
    }
    for (unsigned j = 0; j < n && out < cap; ++j, ++out) {
      const int e = (int)((word >> (4 * j)) & 0xF);
      const int a = E0[e], b = E1[e];
      if (pos) {
        const float3 p = mul3(sdf_interp3(pt[a], pt[b], sv[a], sv[b]), s.voxel);
        pos[3 * out] = p.x;
        pos[3 * out + 1] = p.y;
        pos[3 * out + 2] = p.z;
      }
      if (col) {
        const float3 cc = sdf_interp3(cl[a], cl[b], sv[a], sv[b]);
        reinterpret_cast<float4*>(col)[out] = make_float4(cc.x, cc.y, cc.z, 1.0f);
      }
    }
  }
}

template __global__ void k_hash_mesh_count<0>(const SessionDesc*, unsigned*);
template __global__ void k_hash_mesh_count<1>(const SessionDesc*, unsigned*);
template __global__ void k_hash_mesh_emit<0>(const SessionDesc*, const unsigned long long*, float*, float*,
                                             unsigned long long);
template __global__ void k_hash_mesh_emit<1>(const SessionDesc*, const unsigned long long*, float*, float*,
                                             unsigned long long);
}  // namespace nui
