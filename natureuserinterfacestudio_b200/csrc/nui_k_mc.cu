// Marching cubes over the dense volume (marchingCubeKernel, marchingCube.cl:100-256) with
// deterministic prefix-sum compaction (the role of NuiOpenCLPrefixSum, prefixSum.cl:10-232).
//
// Order: cubes are emitted in the order of the reference's own CPU extraction
// (NuiKinfuOpenCLScene::Volume2Mesh, NuiKinfuOpenCLScene.cpp:823-836): y outermost, then x,
// then z.  A block owns 128 consecutive x of one y row; each thread walks its (x, y)
// column over z, so the warp's loads of every z slice are contiguous, and the block's
// cubes form one contiguous run of that order.
//   k_mc_count  per-column vertex counts + per-block totals
//   k_mc_scan   exclusive scan of the block totals (one block, warp-shuffle scan)
//   k_mc_emit   per-thread exclusive scan inside the block (warp shuffles), then each
//               thread re-walks its column writing vertices at its offset.
// Per cube: skip if any corner has weight <= 0; case bit i = tsdf_i < 0; vertices on the
// table's edges by clamped linear interpolation (vertex_interp, marchingCube.cl:86-91);
// positions ((x + 0.5 - rx/2) c, (-y - 0.5 + ry/2) c, (z + 0.5) c) (getNodeCoo :81-84).
#include "nui_device.cuh"
#include "nui_mc_tables.h"

namespace nui {

constexpr int kMcThreads = 128;
__constant__ uint64_t c_tri[256];

void mc_upload_tables(cudaStream_t st) {
  cudaMemcpyToSymbolAsync(c_tri, NUI_MC_TRI_PACKED, sizeof(NUI_MC_TRI_PACKED), 0, cudaMemcpyHostToDevice, st);
}

template <int FMT>
__device__ __forceinline__ bool corner(const SessionDesc& s, int x, int y, int z, float& f) {
  if (s.occ && __ldg(s.occ + occ_index(s, x, y, z)) == 0) return false;  // brick never weighted
  int w;
  Voxel<FMT>::load(s, vox_index(s, x, y, z), f, w);
  return w > 0;
}

// Case index of cube (x, y, z); -1 when a corner has no weight.
template <int FMT>
__device__ __forceinline__ int cube_case(const SessionDesc& s, int x, int y, int z, float* f) {
  if (!corner<FMT>(s, x, y, z, f[0])) return -1;
  if (!corner<FMT>(s, x + 1, y, z, f[1])) return -1;
  if (!corner<FMT>(s, x + 1, y + 1, z, f[2])) return -1;
  if (!corner<FMT>(s, x, y + 1, z, f[3])) return -1;
  if (!corner<FMT>(s, x, y, z + 1, f[4])) return -1;
  if (!corner<FMT>(s, x + 1, y, z + 1, f[5])) return -1;
  if (!corner<FMT>(s, x + 1, y + 1, z + 1, f[6])) return -1;
  if (!corner<FMT>(s, x, y + 1, z + 1, f[7])) return -1;
  int c = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) c += (f[k] < 0) ? (1 << k) : 0;
  return c;
}

template <int FMT>
__global__ void __launch_bounds__(kMcThreads) k_mc_count(const SessionDesc* __restrict__ descs, unsigned int* colcount,
                                                         unsigned long long* blocktot, uint8_t* cases) {
  const SessionDesc& s = descs[0];
  const int rx = s.res[0], ry = s.res[1], rz = s.res[2];
  const int tilesX = (rx - 1 + kMcThreads - 1) / kMcThreads;
  const int y = blockIdx.x / tilesX, xt = blockIdx.x % tilesX;
  const int x = xt * kMcThreads + threadIdx.x;
  unsigned int n = 0;
  if (y < ry - 1 && x < rx - 1) {
    const size_t cbase = ((size_t)y * (rx - 1) + x) * (size_t)(rz - 1);
    for (int z = 0; z < rz - 1; ++z) {
      float f[8];
      const int c = cube_case<FMT>(s, x, y, z, f);
      if (cases) cases[cbase + z] = c < 0 ? 0 : (uint8_t)c;
      if (c > 0) n += 3u * (unsigned)(c_tri[c] >> 60);
    }
    colcount[(size_t)y * (rx - 1) + x] = n;
  }
  __shared__ unsigned long long wsum[kMcThreads / 32];
  unsigned long long v = n;
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int i = 0; i < kMcThreads / 32; ++i) t += wsum[i];
    blocktot[blockIdx.x] = t;
  }
}

// Exclusive scan of n block totals in place, total in out[n]; one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_mc_scan(unsigned long long* tot, int n) {
  __shared__ unsigned long long warp_tot[32];
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < n; base += 1024) {
    const int i = base + threadIdx.x;
    unsigned long long v = i < n ? tot[i] : 0ull;
    unsigned long long inc = v;
    for (int off = 1; off < 32; off <<= 1) {
      unsigned long long o = __shfl_up_sync(0xffffffffu, inc, off);
      if (lane >= off) inc += o;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      unsigned long long w = warp_tot[lane], wi = w;
      for (int off = 1; off < 32; off <<= 1) {
        unsigned long long o = __shfl_up_sync(0xffffffffu, wi, off);
        if (lane >= off) wi += o;
      }
      warp_tot[lane] = wi - w;  // exclusive prefix of the warp totals
    }
    __syncthreads();
    const unsigned long long excl = carry + warp_tot[warp] + inc - v;
    __syncthreads();
    if (i < n) tot[i] = excl;
    if (threadIdx.x == 1023) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) tot[n] = carry;
}

template <int FMT>
__global__ void __launch_bounds__(kMcThreads) k_mc_emit(const SessionDesc* __restrict__ descs,
                                                        const unsigned int* colcount,
                                                        const unsigned long long* blockoff, float* pos,
                                                        float* col, unsigned long long cap) {
  const SessionDesc& s = descs[0];
  const int rx = s.res[0], ry = s.res[1], rz = s.res[2];
  const int tilesX = (rx - 1 + kMcThreads - 1) / kMcThreads;
  const int y = blockIdx.x / tilesX, xt = blockIdx.x % tilesX;
  const int x = xt * kMcThreads + threadIdx.x;
  const bool live = y < ry - 1 && x < rx - 1;
  const unsigned int n = live ? colcount[(size_t)y * (rx - 1) + x] : 0u;
  // exclusive scan of the column counts over the block, in x order
  __shared__ unsigned long long wsum[kMcThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long inc = n;
  for (int off = 1; off < 32; off <<= 1) {
    unsigned long long o = __shfl_up_sync(0xffffffffu, inc, off);
    if (lane >= off) inc += o;
  }
  if (lane == 31) wsum[warp] = inc;
  __syncthreads();
  unsigned long long before = 0;
  for (int w = 0; w < warp; ++w) before += wsum[w];
  unsigned long long out = blockoff[blockIdx.x] + before + inc - n;
  if (!live || n == 0 || out >= cap) return;
  const float c0 = s.cell[0], c1 = s.cell[1], c2 = s.cell[2];
  const float hx = (float)(rx >> 1), hy = (float)(ry >> 1);
  const int E0[12] = {0, 1, 2, 3, 4, 5, 6, 7, 0, 1, 2, 3};
  const int E1[12] = {1, 2, 3, 0, 5, 6, 7, 4, 4, 5, 6, 7};
  const int CX[8] = {0, 1, 1, 0, 0, 1, 1, 0}, CY[8] = {0, 0, 1, 1, 0, 0, 1, 1}, CZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};
  for (int z = 0; z < rz - 1 && out < cap; ++z) {
    float f[8];
    const int c = cube_case<FMT>(s, x, y, z, f);
    if (c <= 0) continue;
    const uint64_t word = c_tri[c];
    const int nv = 3 * (int)(word >> 60);
    if (nv == 0) continue;
    for (int k = 0; k < nv && out < cap; ++k, ++out) {
      const int e = (int)((word >> (4 * k)) & 0xF);
      const int a = E0[e], b = E1[e];
      const float3 pa = f3(((float)(x + CX[a]) + 0.5f - hx) * c0, (-(float)(y + CY[a]) - 0.5f + hy) * c1,
                           ((float)(z + CZ[a]) + 0.5f) * c2);
      const float3 pb = f3(((float)(x + CX[b]) + 0.5f - hx) * c0, (-(float)(y + CY[b]) - 0.5f + hy) * c1,
                           ((float)(z + CZ[b]) + 0.5f) * c2);
      float t = (0.f - f[a]) / (f[b] - f[a] + 1e-15f);
      t = fminf(fmaxf(t, 0.0f), 1.0f);
      if (pos) {
        pos[3 * out] = pa.x + (pb.x - pa.x) * t;
        pos[3 * out + 1] = pa.y + (pb.y - pa.y) * t;
        pos[3 * out + 2] = pa.z + (pb.z - pa.z) * t;
      }
      if (col) {
        float4 cc = make_float4(0.f, 0.f, 0.f, 1.f);
        if (s.cvol) {
          const bool near_a = fabsf(f[a]) < fabsf(f[b]);
          const uchar4 v = s.cvol[vox_index(s, x + (near_a ? CX[a] : CX[b]), y + (near_a ? CY[a] : CY[b]),
                                            z + (near_a ? CZ[a] : CZ[b]))];
          cc = make_float4((float)v.z / 255.f, (float)v.y / 255.f, (float)v.x / 255.f, 1.f);
        }
        reinterpret_cast<float4*>(col)[out] = cc;
      }
    }
  }
}

#define NUI_MC_INST(F)                                                                                       \
  template __global__ void k_mc_count<F>(const SessionDesc*, unsigned int*, unsigned long long*, uint8_t*); \
  template __global__ void k_mc_emit<F>(const SessionDesc*, const unsigned int*, const unsigned long long*, \
                                        float*, float*, unsigned long long);
NUI_MC_INST(0)
NUI_MC_INST(1)
NUI_MC_INST(2)
NUI_MC_INST(3)

}  // namespace nui
