// Colour pyramid and gradients of the colour tracker (A8): the preprocessing of
// NuiKinfuOpenCLColorTracker::EstimatePose (NuiKinfuOpenCLColorTracker.cpp:580-606).
//
//   k_color_level  one level of the colour pyramid (half_sample_bgra_kernel,
//                  transformMaps.cl:106-146, radius 1 as the host passes it :159): the
//                  truncated integer mean of every channel over the 3 x 3 taps around
//                  (2x, 2y) of the level below, clamped to that image; alpha 255.
//   k_color_grad   x / y gradients of every level in one launch (bgra_gradient_kernel,
//                  transformMaps.cl:514-560): Sobel / 8 per colour channel in float,
//                  stored as the low byte of its truncation toward zero (a negative
//                  gradient wraps; the tracker reads the byte as a signed char), alpha
//                  255; border pixels (0, 0, 0, 0).  The reference kernel steps to the
//                  rows above and below by the image height and stores its result one
//                  row and one pixel past the centre; here rows are stepped by the width
//                  and the result is stored at the centre.
// Level 0 of the pyramid is the frame's BGRA buffer itself.  The tracker uses level 0 and
// its gradients; the whole pyramid is the kernel-level entry point's.
//   k_color_keep   the frame's colours become the next frame's model colours.
#include "nui_device.cuh"

namespace nui {

__device__ __forceinline__ const uchar4* color_level(const SessionDesc& s, int l) {
  return l == 0 ? reinterpret_cast<const uchar4*>(s.bgra) : s.cpyr[l];
}

__global__ void __launch_bounds__(256) k_color_level(const SessionDesc* __restrict__ descs, int l) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind != kTrackFrame || !(s.photo_w > 0.f) || !s.bgra || l >= s.levels || !s.cpyr[l]) return;
  const int dW = s.W >> l, dH = s.H >> l, sW = 2 * dW, sH = 2 * dH;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= dW * dH) return;
  const int x = i % dW, y = i / dW;
  const uchar4* __restrict__ src = color_level(s, l - 1);
  const int x0 = max(2 * x - 1, 0), x1 = min(2 * x + 2, sW), y0 = max(2 * y - 1, 0), y1 = min(2 * y + 2, sH);
  int b = 0, g = 0, r = 0, a = 0, n = 0;
  for (int cy = y0; cy < y1; ++cy)
    for (int cx = x0; cx < x1; ++cx) {
      const uchar4 v = __ldg(src + cy * sW + cx);
      b += v.x;
      g += v.y;
      r += v.z;
      a += v.w;
      ++n;
    }
  (void)a;
  s.cpyr[l][i] = make_uchar4((unsigned char)(b / n), (unsigned char)(g / n), (unsigned char)(r / n), 255);
}

__device__ __forceinline__ unsigned char grad_byte(float v) { return (unsigned char)(int)v; }

__global__ void __launch_bounds__(256) k_color_grad(const SessionDesc* __restrict__ descs, int fam) {
  const SessionDesc& s = descs[blockIdx.y];
  const int l = blockIdx.z;
  if (s.kind != kTrackFrame || !in_family(s, fam) || !(s.photo_w > 0.f) || !s.bgra || l >= s.levels || !s.cgx[l]) return;
  const int W = s.W >> l, H = s.H >> l;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W * H) return;
  const int x = i % W, y = i / W;
  if (!(x > 0 && x < W - 1 && y > 0 && y < H - 1)) {
    s.cgx[l][i] = make_uchar4(0, 0, 0, 0);
    s.cgy[l][i] = make_uchar4(0, 0, 0, 0);
    return;
  }
  const uchar4* __restrict__ c = color_level(s, l);
  const uchar4 s11 = __ldg(c + i - W - 1), s12 = __ldg(c + i - W), s13 = __ldg(c + i - W + 1);
  const uchar4 s21 = __ldg(c + i - 1), s23 = __ldg(c + i + 1);
  const uchar4 s31 = __ldg(c + i + W - 1), s32 = __ldg(c + i + W), s33 = __ldg(c + i + W + 1);
  auto sob_x = [](float a13, float a11, float a23, float a21, float a33, float a31) {
    return ((a13 - a11) + 2 * (a23 - a21) + (a33 - a31)) / 8.0f;
  };
  s.cgx[l][i] = make_uchar4(grad_byte(sob_x(s13.x, s11.x, s23.x, s21.x, s33.x, s31.x)),
                            grad_byte(sob_x(s13.y, s11.y, s23.y, s21.y, s33.y, s31.y)),
                            grad_byte(sob_x(s13.z, s11.z, s23.z, s21.z, s33.z, s31.z)), 255);
  // y: (s31 - s11) + 2 (s32 - s12) + (s33 - s13), the same form with the roles turned
  s.cgy[l][i] = make_uchar4(grad_byte(sob_x(s31.x, s11.x, s32.x, s12.x, s33.x, s13.x)),
                            grad_byte(sob_x(s31.y, s11.y, s32.y, s12.y, s33.y, s13.y)),
                            grad_byte(sob_x(s31.z, s11.z, s32.z, s12.z, s33.z, s13.z)), 255);
}

// Four pixels a thread (16-byte copies when both buffers allow them).
__global__ void __launch_bounds__(256) k_color_keep(const SessionDesc* __restrict__ descs, int fam) {
  const SessionDesc& s = descs[blockIdx.y];
  if (s.kind < 0 || !in_family(s, fam) || !(s.photo_w > 0.f) || !s.bgra || !s.cprev) return;
  const int n = s.W * s.H;
  const int i = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= n) return;
  const uchar4* src = reinterpret_cast<const uchar4*>(s.bgra);
  const bool vec = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(s.cprev)) & 15) == 0;
  if (vec && i + 3 < n) {
    reinterpret_cast<uint4*>(s.cprev)[i / 4] = __ldg(reinterpret_cast<const uint4*>(src) + i / 4);
  } else {
    for (int k = i; k < min(i + 4, n); ++k) s.cprev[k] = __ldg(src + k);
  }
}

}  // namespace nui
