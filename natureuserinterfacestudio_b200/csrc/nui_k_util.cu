// Small utility kernels: per-session result publication and conversion between the
// session volume layout and the reference layout ((x + y*rx)*rz + z, short2).
#include "nui_device.cuh"

namespace nui {

// One thread per session: status, gate and pose of this tick into a packed array that
// the host reads back with one copy.
__global__ void k_publish(const SessionDesc* __restrict__ descs, int n, float* pose, int* status, int fam) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !pose || !status) return;
  const SessionDesc& s = descs[i];
  if (s.ts == nullptr || !in_family(s, fam)) return;
  const TrackState* ts = s.ts;
  const int o = s.slot;
  status[2 * o] = s.kind < 0 ? 0 : ts->status;
  status[2 * o + 1] = ts->integrate;
  for (int k = 0; k < 9; ++k) pose[14 * o + k] = ts->xf.R[k];
  for (int k = 0; k < 3; ++k) pose[14 * o + 9 + k] = ts->xf.t[k];
  pose[14 * o + 12] = ts->error;
  pose[14 * o + 13] = ts->count;
}

// Start of a tick: clear the per-frame counters of every active session, and the flag of a
// frame that lost tracking (the state stayed on the frame before it; this frame starts
// from a clean tracker even when it was launched before the loss was read back).
__global__ void k_tick_begin(const SessionDesc* __restrict__ descs, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SessionDesc& s = descs[i];
  if (s.kind < 0 || !s.ts) return;
  s.ts->status = 0;
  s.ts->dmax_bits = 0;
  s.ts->touched = 0ull;
  s.ts->ray_reads = s.ts->ray_samples = s.ts->ray_hits = s.ts->bricks = s.ts->tiles = 0ull;
  for (int l = 0; l < kMaxLevels; ++l) s.ts->icp_iters[l] = 0u;
  if (s.hcount) {
    s.hcount[kHashFailedBefore] = s.hcount[kHashFailed];
    s.hcount[kHashChainFaults] = 0;
  }
}

// End of a tick with voxel-hash sessions: a frame whose allocation ran out of pool blocks
// or excess slots (the reference's atomic_dec of an empty free list,
// KinfuHashScene.cl:155,171-172, silently drops the block) or met a corrupted excess chain
// reports NUI_ERR_HASH_FULL (4) unless tracking already failed.
__global__ void k_hash_health(const SessionDesc* __restrict__ descs, int n, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !status) return;
  const SessionDesc& s = descs[i];
  if (s.kind < 0 || !s.ts || !s.hcount) return;
  const int o = s.slot;
  if (status[2 * o] != 0) return;
  if (s.hcount[kHashFailed] > s.hcount[kHashFailedBefore] || s.hcount[kHashChainFaults] > 0) status[2 * o] = 4;
}

template <int FMT>
__global__ void k_export_ref(const SessionDesc* __restrict__ descs, short2* out, uchar4* cout) {
  const SessionDesc& s = descs[0];
  const int rx = s.res[0], ry = s.res[1], rz = s.res[2];
  const size_t n = (size_t)rx * ry * rz;
  // a shifting volume's voxel sits in the reference's buffer at its wrap
  const int wx = ref_wrap(s.ts->voff[0], rx), wy = ref_wrap(s.ts->voff[1], ry), wz = ref_wrap(s.ts->voff[2], rz);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % rx);
    const int y = (int)((i / rx) % ry);
    const int z = (int)(i / ((size_t)rx * ry));
    const size_t o = ((size_t)((x + wx) % rx) + (size_t)((y + wy) % ry) * rx) * rz + (z + wz) % rz;
    if (out) {
      if (FMT == 0) {
        out[o] = reinterpret_cast<const short2*>(s.vol)[i];
      } else {
        float F;
        int W;
        Voxel<FMT>::load(s, i, F, W);
        out[o] = make_short2((short)__float2int_rz(F * 32766.f), (short)W);
      }
    }
    if (cout && s.cvol) cout[o] = s.cvol[i];
  }
}

// Clears the occupancy bytes of a session (before an import or at reset).
__global__ void k_occ_clear(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[0];
  if (!s.occ) return;
  const size_t n = (size_t)((s.res[0] + 7) >> 3) * ((s.res[1] + 7) >> 3) * ((s.res[2] + 7) >> 3);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
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

template <int FMT>
__global__ void k_import_ref(const SessionDesc* __restrict__ descs, const short2* in) {
  const SessionDesc& s = descs[0];
  const int rx = s.res[0], ry = s.res[1], rz = s.res[2];
  const size_t n = (size_t)rx * ry * rz;
  const int wx = ref_wrap(s.ts->voff[0], rx), wy = ref_wrap(s.ts->voff[1], ry), wz = ref_wrap(s.ts->voff[2], rz);
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % rx);
    const int y = (int)((i / rx) % ry);
    const int z = (int)(i / ((size_t)rx * ry));
    const short2 v = in[((size_t)((x + wx) % rx) + (size_t)((y + wy) % ry) * rx) * rz + (z + wz) % rz];
    if (FMT == 0)
      reinterpret_cast<short2*>(s.vol)[i] = v;
    else
      Voxel<FMT>::store(s, i, (float)v.x / 32766.f, v.y);
    if (s.occ && v.y > 0) s.occ[occ_index(s, x, y, z)] = kBrickDirty;
  }
}

template __global__ void k_export_ref<0>(const SessionDesc*, short2*, uchar4*);
template __global__ void k_export_ref<1>(const SessionDesc*, short2*, uchar4*);
template __global__ void k_export_ref<2>(const SessionDesc*, short2*, uchar4*);
template __global__ void k_export_ref<3>(const SessionDesc*, short2*, uchar4*);
template __global__ void k_import_ref<0>(const SessionDesc*, const short2*);
template __global__ void k_import_ref<1>(const SessionDesc*, const short2*);
template __global__ void k_import_ref<2>(const SessionDesc*, const short2*);
template __global__ void k_import_ref<3>(const SessionDesc*, const short2*);

}  // namespace nui
