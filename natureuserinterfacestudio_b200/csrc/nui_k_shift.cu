// Shifting dense volume (NuiKinfuOpenCLShiftScene, NuiKinfuOpenCLShiftScene.cpp:76-362) and
// the point fetches of the dense scenes (fetchVolumeKernel / fetchShiftVolumeKernel,
// extract.cl:4-179).
//
// The reference keeps every voxel where it was written and reaches it through voxelWrap:
// voxel (x, y, z) of the volume lives at ((x + wx) % rx, (y + wy) % ry, (z + wz) % rz) of
// its buffer, and a shift clears the slab that leaves and moves the wrap.  Here the voxels
// stay in volume order: a shift rolls the volume in HBM by the shift, one axis at a time,
// each line through shared memory, and writes the cleared value where the slab that left
// comes back in.  Every voxel holds what the reference's holds, so integration, raycast,
// brick summaries and meshing run unchanged and no hot loop pays a modulo.  A shift moves
// each voxel once per shifted axis (a 512^3 FP16 + u8 volume: 0.8 GB of traffic, about
// 0.15 ms), at most once per frame and only after the camera has moved voxel_shift voxels.
//
// The kernels run in every tick that holds a shifting session; without a shift they return
// at once.  Grid-stride loops keep that cost to a few hundred blocks per launch.
#include "nui_device.cuh"

namespace nui {

constexpr int kShiftThreads = 256;
constexpr int kRollBytes = 32768;  // shared-memory tile of the rolls

__device__ __forceinline__ bool shifting(const SessionDesc& s, int axis) {
  return s.kind >= 0 && s.voxel_shift > 0 && s.fmt >= 0 && s.ts->shift[axis] != 0;
}

// One column of fetchShiftVolumeKernel (extract.cl:82-179) at work item (vx, vy), in the
// reference's buffer coordinates: its z loop runs from wrap.z and adds the wrap a second
// time in the index, and its offsets step by whole volumes, as written.  W is the wrap
// that maps the buffer to this volume's voxels (buffer position p holds voxel
// (p - W) mod r).  Points go to the cache through `counter`, at most cap of them.
template <int FMT>
__device__ void fetch_column(const SessionDesc& s, int vx, int vy, int range_z, const int* wrap, const int* voff,
                             const int* W, float* xyz, float* rgba, long long cap, unsigned long long* counter) {
  const int rx = s.res[0], ry = s.res[1], rz = s.res[2];
  const float half_x = (float)(rx >> 1), half_y = (float)(ry >> 1);
  const int lx = ((vx + wrap[0]) % rx - W[0] + rx) % rx;
  const int ly = ((vy + wrap[1]) % ry - W[1] + ry) % ry;
  int obx = (voff[0] / rx) * rx, oby = (voff[1] / ry) * ry;
  const int obz = (voff[2] / rz) * rz;
  if (voff[0] > 0) {
    if (vx < voff[0] % rx) obx += rx;
  } else if (vx > rx + voff[0] % rx) {
    obx -= rx;
  }
  if (voff[1] > 0) {
    if (vy < voff[1] % ry) oby += ry;
  } else if (vy > ry + voff[1] % ry) {
    oby -= ry;
  }
  const float px = ((float)(vx + obx) + 0.5f - half_x) * s.cell[0];
  const float py = (-(float)(vy + oby) - 0.5f + half_y) * s.cell[1];
  float tsdf = __int_as_float(0x7fc00000);
  const int zend = range_z + wrap[2];
  for (int vz = wrap[2]; vz < zend; ++vz) {
    const float prev = tsdf;
    const int lz = ((vz + wrap[2]) % rz - W[2] + rz) % rz;
    const size_t i = vox_index(s, lx, ly, lz);
    float F;
    int Wt;
    Voxel<FMT>::load(s, i, F, Wt);
    if (Wt <= 0) {
      tsdf = __int_as_float(0x7fc00000);
      continue;
    }
    int oz = obz;
    if (voff[2] > 0) {
      if (vz < voff[2] % rz) oz += rz;
    } else if (vz > rz + voff[2] % rz) {
      oz -= rz;
    }
    tsdf = F;
    const bool zero = tsdf == 0.f;
    if (!zero && !((prev < 0.f && tsdf > 0.f) || (prev > 0.f && tsdf < 0.f))) continue;
    float pz;
    float4 c = make_float4(0.f, 0.f, 0.f, 1.f);
    const uchar4 g = s.cvol ? s.cvol[i] : make_uchar4(0, 0, 0, 0);
    if (zero) {
      pz = ((float)(vz + oz) + 0.5f) * s.cell[2];
      if (s.cvol) c = make_float4((float)g.x / 255.f, (float)g.y / 255.f, (float)g.z / 255.f, 1.f);
    } else {
      const float ti = 1.f / fabsf(tsdf), tpi = 1.f / fabsf(prev);
      const float dp = (ti * (float)(vz + oz) + tpi * (float)(vz + oz - 1)) / (ti + tpi);
      pz = (dp + 0.5f) * s.cell[2];
      // the crossing case reads the colour bytes in reverse order (extract.cl:167-169)
      if (s.cvol) c = make_float4((float)g.z / 255.f, (float)g.y / 255.f, (float)g.x / 255.f, 1.f);
    }
    const unsigned long long k = atomicAdd(counter, 1ull);
    if ((long long)k < cap) {
      xyz[3 * k] = px;
      xyz[3 * k + 1] = py;
      xyz[3 * k + 2] = pz;
      reinterpret_cast<float4*>(rgba)[k] = c;
    }
  }
}

// fetchSlice of one axis's shift (NuiKinfuOpenCLShiftScene.cpp:117-233, 235-286): the slab
// of |shift| voxels about to leave, as the reference's buffer held it then (the axes
// before this one have moved, this one and those after it not yet), into the session's
// point cache.
template <int FMT>
__global__ void __launch_bounds__(kShiftThreads) k_shift_fetch(const SessionDesc* __restrict__ descs, int axis) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.fmt != FMT || !shifting(s, axis) || !s.pts_xyz) return;
  const TrackState* ts = s.ts;
  const int r[3] = {s.res[0], s.res[1], s.res[2]};
  const int tr = ts->shift[axis];
  int voff[3], W[3], wrap[3] = {0, 0, 0}, range[3] = {r[0], r[1], r[2]};
  for (int b = 0; b < 3; ++b) {
    voff[b] = ts->voff[b] - (b >= axis ? ts->shift[b] : 0);
    W[b] = ref_wrap(voff[b], r[b]) % r[b];
  }
  int off = voff[axis] + (tr < 0 ? tr : 0);
  off = off >= 0 ? off % r[axis] : r[axis] - (-off) % r[axis];
  wrap[axis] = off;
  range[axis] = abs(tr);
  const long n = (long)range[0] * range[1];
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    fetch_column<FMT>(s, (int)(i % range[0]), (int)(i / range[0]), range[2], wrap, voff, W, s.pts_xyz, s.pts_rgba,
                      s.pts_cap, &s.ts->points);
}

// Volume2CLVertices of the dense scenes (NuiKinfuOpenCLScene: fetchVolumeKernel;
// NuiKinfuOpenCLShiftScene.cpp:354-520: fetchShiftVolumeKernel with wrap 0 and the volume's
// offset): every column of the reference's buffer.  A fixed volume has offset 0, which
// makes the two kernels the same.
template <int FMT>
__global__ void __launch_bounds__(kShiftThreads) k_fetch_volume(const SessionDesc* __restrict__ descs, float* xyz,
                                                                 float* rgba, long long cap,
                                                                 unsigned long long* counter) {
  const SessionDesc& s = descs[0];
  const int r[3] = {s.res[0], s.res[1], s.res[2]};
  int voff[3], W[3];
  const int wrap[3] = {0, 0, 0};
  for (int b = 0; b < 3; ++b) {
    voff[b] = s.ts->voff[b];
    W[b] = ref_wrap(voff[b], r[b]) % r[b];
  }
  const long n = (long)r[0] * r[1];
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    fetch_column<FMT>(s, (int)(i % r[0]), (int)(i / r[0]), r[2], wrap, voff, W, xyz, rgba, cap, counter);
}

// The per-voxel array `which` (0: the format's storage, 1: the u8 weight plane of
// NUI_TSDF_F16_U8, 2: the colour volume) when its element is a T, with the value
// initializeVolume leaves in it (tsdfVolume.cl:192-211; 1.0 / weight 0 for the float
// formats, as k_volume_init writes).
template <typename T>
__device__ __forceinline__ bool roll_array(const SessionDesc& s, int which, T*& a, T& init) {
  unsigned long long bits = 0;
  size_t bytes = 0;
  if (which == 0) {
    a = reinterpret_cast<T*>(s.vol);
    switch (s.fmt) {
      case 0: bytes = 4, bits = 0x00007fffull; break;          // short2(32767, 0)
      case 1: bytes = 8, bits = 0x000000003f800000ull; break;  // float2(1, 0)
      case 2: bytes = 2, bits = 0x3c00ull; break;              // half 1
      default: bytes = 4, bits = 0x00003c00ull; break;         // half2(1, 0)
    }
  } else if (which == 1) {
    a = reinterpret_cast<T*>(s.wvol);
    bytes = 1;
  } else {
    a = reinterpret_cast<T*>(s.cvol);
    bytes = 4;
  }
  if (!a || bytes != sizeof(T)) return false;
  static_assert(sizeof(T) <= 8, "element of at most 8 bytes");
  memcpy(&init, &bits, sizeof(T));
  return true;
}

// One axis of a shift along x: v'[x] = v[x + tr] where 0 <= x + tr < rx, else the cleared
// value (the voxels of the slab the reference clears).  Lines of x are contiguous; a block
// stages several lines in shared memory, then writes them back moved.
template <typename T>
__global__ void __launch_bounds__(kShiftThreads) k_shift_roll_x(const SessionDesc* __restrict__ descs, int which) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!shifting(s, 0)) return;
  T* a;
  T init;
  if (!roll_array<T>(s, which, a, init)) return;
  constexpr int kElems = kRollBytes / (int)sizeof(T);
  __shared__ T line[kElems];
  const int rx = s.res[0], tr = s.ts->shift[0];
  const long nlines = (long)s.res[1] * s.res[2];
  const int per = kElems / rx;  // rx <= 1024: at least 4 lines
  for (long L0 = (long)blockIdx.x * per; L0 < nlines; L0 += (long)gridDim.x * per) {
    const int nl = (int)min((long)per, nlines - L0);
    T* base = a + (size_t)L0 * rx;
    for (int k = threadIdx.x; k < nl * rx; k += blockDim.x) line[k] = base[k];
    __syncthreads();
    for (int k = threadIdx.x; k < nl * rx; k += blockDim.x) {
      const int x = k % rx, src = x + tr;
      base[k] = (src >= 0 && src < rx) ? line[k - x + src] : init;
    }
    __syncthreads();
  }
}

// The same along y (axis 1) or z (axis 2): a block stages a tile of TX consecutive x by the
// whole axis for one position of the remaining axis (rows of TX elements are >= 32 bytes).
template <typename T>
__global__ void __launch_bounds__(kShiftThreads) k_shift_roll_yz(const SessionDesc* __restrict__ descs, int axis,
                                                                  int which) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!shifting(s, axis)) return;
  T* a;
  T init;
  if (!roll_array<T>(s, which, a, init)) return;
  constexpr int TX = 32 / (int)sizeof(T);  // 32-byte rows
  __shared__ T tile[kRollBytes / sizeof(T)];  // the whole axis: r * TX * sizeof(T) <= 1024 * 32
  const int rx = s.res[0], ry = s.res[1];
  const int r = s.res[axis], other = axis == 1 ? s.res[2] : s.res[1], tr = s.ts->shift[axis];
  const size_t si = axis == 1 ? (size_t)rx : (size_t)rx * ry;  // stride along the axis
  const size_t so = axis == 1 ? (size_t)rx * ry : (size_t)rx;  // stride along the other axis
  const int xtiles = (rx + TX - 1) / TX;
  const long groups = (long)xtiles * other;
  for (long g = blockIdx.x; g < groups; g += gridDim.x) {
    const int x0 = (int)(g % xtiles) * TX, o = (int)(g / xtiles);
    const int nx = min(TX, rx - x0);
    T* base = a + (size_t)x0 + so * (size_t)o;
    for (int k = threadIdx.x; k < r * TX; k += blockDim.x) {
      const int i = k / TX, dx = k % TX;
      if (dx < nx) tile[k] = base[(size_t)dx + si * i];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < r * TX; k += blockDim.x) {
      const int i = k / TX, dx = k % TX, src = i + tr;
      if (dx < nx) base[(size_t)dx + si * i] = (src >= 0 && src < r) ? tile[src * TX + dx] : init;
    }
    __syncthreads();
  }
}

// After a shift every brick's content moved: all are re-classified with the summaries
// that follow the integration.
__global__ void __launch_bounds__(kShiftThreads) k_shift_dirty(const SessionDesc* __restrict__ descs) {
  const SessionDesc& s = descs[blockIdx.y];
  if (!s.occ || !(shifting(s, 0) || shifting(s, 1) || shifting(s, 2))) return;
  const long nb = (long)((s.res[0] + 7) >> 3) * ((s.res[1] + 7) >> 3) * ((s.res[2] + 7) >> 3);
  for (long b = (long)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (long)gridDim.x * blockDim.x)
    s.occ[b] = kBrickDirty;
}

template __global__ void k_shift_fetch<0>(const SessionDesc*, int);
template __global__ void k_shift_fetch<1>(const SessionDesc*, int);
template __global__ void k_shift_fetch<2>(const SessionDesc*, int);
template __global__ void k_shift_fetch<3>(const SessionDesc*, int);
template __global__ void k_fetch_volume<0>(const SessionDesc*, float*, float*, long long, unsigned long long*);
template __global__ void k_fetch_volume<1>(const SessionDesc*, float*, float*, long long, unsigned long long*);
template __global__ void k_fetch_volume<2>(const SessionDesc*, float*, float*, long long, unsigned long long*);
template __global__ void k_fetch_volume<3>(const SessionDesc*, float*, float*, long long, unsigned long long*);
template __global__ void k_shift_roll_x<uint8_t>(const SessionDesc*, int);
template __global__ void k_shift_roll_x<uint16_t>(const SessionDesc*, int);
template __global__ void k_shift_roll_x<uint32_t>(const SessionDesc*, int);
template __global__ void k_shift_roll_x<unsigned long long>(const SessionDesc*, int);
template __global__ void k_shift_roll_yz<uint8_t>(const SessionDesc*, int, int);
template __global__ void k_shift_roll_yz<uint16_t>(const SessionDesc*, int, int);
template __global__ void k_shift_roll_yz<uint32_t>(const SessionDesc*, int, int);
template __global__ void k_shift_roll_yz<unsigned long long>(const SessionDesc*, int, int);

}  // namespace nui
