// CPU ORACLE -- test infrastructure only.
//
// A plain C++17 restatement of the per-frame KinectFusion path of the reference
// (hustztz/NatureUserInterfaceStudio, OpenCL kernels under src/Kernels and their host
// drivers under src/SLAM/VisualOdometry).  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference arm of bench.py may load this library, and only as the
// checker or the timed CPU baseline; the product never calls it.
//
// Conventions fixed here (the reference leaves them implementation-defined):
//  * no floating-point contraction (built with -ffp-contract=off): every a*b+c is a
//    rounded multiply followed by a rounded add, as written in the OpenCL source;
//  * exp() of the bilateral filter is oracle_expf(): Cody-Waite range reduction with a
//    degree-7 Taylor polynomial, within 2 ulp of the exact value (OpenCL allows 3);
//  * fast_length(v) = sqrtf(dot(v,v)), dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z,
//    normalize / fast_normalize(v) = v / sqrtf(dot(v,v)), and a zero vector stays zero
//    (OpenCL 1.2 spec, 6.12.5);
//  * round() is half-away-from-zero (roundf), convert_int/short/uchar truncate.
//
// Volumes are kept in the reference layout: voxel (x,y,z) at ((x + y*resX)*resZ + z),
// stored as short2 (tsdf * 32766 truncated, weight)  [tsdfVolume.cl:71,104].
//
// Each function cites the reference file:line it restates.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <unordered_map>
#include <vector>

#include "../natureuserinterfacestudio_b200/csrc/nui_mc_tables.h"

#define ORC_API extern "C" __attribute__((visibility("default")))

namespace {

struct f3 {
  float x, y, z;
};
inline f3 mk(float x, float y, float z) { return f3{x, y, z}; }
inline f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline f3 operator*(float s, f3 a) { return mk(s * a.x, s * a.y, s * a.z); }
inline float dot3(f3 a, f3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline f3 cross3(f3 a, f3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline bool isnan3(f3 v) { return std::isnan(v.x) || std::isnan(v.y) || std::isnan(v.z); }
inline float length3(f3 v) { return std::sqrt(dot3(v, v)); }
inline f3 normalize3(f3 v) {
  if (v.x == 0.f && v.y == 0.f && v.z == 0.f) return v;
  float l = std::sqrt(dot3(v, v));
  return mk(v.x / l, v.y / l, v.z / l);
}
inline f3 ld3(const float* p, long i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
inline void st3(float* p, long i, f3 v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}
const float QNAN = std::numeric_limits<float>::quiet_NaN();

}  // namespace

// ---------------------------------------------------------------------------------
// Shared parameter blocks (same field meaning as gpu_def.h:5-34).
struct OrcCam {
  float fx, fy, fx_inv, fy_inv, cx, cy;
  uint32_t W, H;
  float dmin, dmax;
};
struct OrcXform {
  float R[9];      // row-major camera->world rotation
  float R_inv[9];  // its inverse (row-major)
  float t[3];      // camera position in world
};
struct OrcTsdf {
  float res[3], dim[3], cell[3], trunc;
};

// exp() used for OpenCL's exp(): x = k*ln2 + r (Cody-Waite split of ln2),
// exp(r) by Horner evaluation of the degree-7 Taylor polynomial, times 2^k; the reduction
// and the polynomial in fused multiply-adds (std::fma, exactly rounded like the device's).
ORC_API float oracle_expf(float x) {
  if (std::isnan(x)) return x;
  if (x > 88.5f) return std::numeric_limits<float>::infinity();
  if (x < -103.5f) return 0.f;
  const float kf = std::nearbyint(x * 1.44269504088896341f);
  float r = std::fma(-kf, 0.693145751953125f, x);
  r = std::fma(-kf, 1.42860682030941723e-6f, r);
  float p = 1.98412698412698413e-4f;
  p = std::fma(p, r, 1.38888888888888889e-3f);
  p = std::fma(p, r, 8.33333333333333333e-3f);
  p = std::fma(p, r, 4.16666666666666667e-2f);
  p = std::fma(p, r, 1.66666666666666667e-1f);
  p = std::fma(p, r, 0.5f);
  p = std::fma(p, r, 1.0f);
  p = std::fma(p, r, 1.0f);
  int k = (int)kf;
  // multiply by 2^k in two exact steps so that k down to -149 stays representable
  int k1 = k / 2, k2 = k - k1;
  float s1, s2;
  uint32_t b1 = (uint32_t)(k1 + 127) << 23, b2 = (uint32_t)(k2 + 127) << 23;
  std::memcpy(&s1, &b1, 4);
  std::memcpy(&s2, &b2, 4);
  return (p * s1) * s2;
}

// ---------------------------------------------------------------------------------
// A1  depth_passing_filter_kernel   filters.cl:9-23
ORC_API void orc_pass_filter(const uint16_t* raw, long n, float dmin, float dmax, float* out) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) {
    float dp = (float)raw[i] * 0.001f;
    out[i] = (dp > dmin && dp < dmax) ? dp : QNAN;
  }
}

// Gaussian spatial table built on the host   NuiKinfuOpenCLFrame.cpp:165-190
ORC_API void orc_gaussian_table(int radius, float sigma_space2_inv_half, float* table) {
  for (int i = 0; i < 2 * radius + 1; ++i) {
    int x = i - radius;
    table[i] = std::exp((float)(-(x * x)) * sigma_space2_inv_half);
  }
}

// A2  bilateral_filter_depth_kernel   bilateralFilter.cl:68-119
ORC_API void orc_bilateral(const float* in, int W, int H, const float* gauss, int radius,
                           float sigma_depth, float thr, float* out) {
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      float c = in[(long)y * W + x];
      if (std::isnan(c)) {
        out[(long)y * W + x] = QNAN;
        continue;
      }
      int x0 = std::max(x - radius, 0), x1 = std::min(x + radius + 1, W);
      int y0 = std::max(y - radius, 0), y1 = std::min(y + radius + 1, H);
      float sd = 0.f, sw = 0.f;
      for (int cy = y0; cy < y1; ++cy)
        for (int cx = x0; cx < x1; ++cx) {
          float nr = in[(long)cy * W + cx];
          if (std::isnan(nr)) continue;
          float diff = std::fabs(c - nr);
          if (nr > 0.f && diff < thr) {
            float d2 = diff * diff;
            float w = gauss[cx + radius - x] * gauss[cy + radius - y] * oracle_expf(-(d2 * sigma_depth));
            sd += nr * w;
            sw += w;
          }
        }
      out[(long)y * W + x] = sd / sw;
    }
}

// A3  half_sample_kernel   transformMaps.cl:44-88  (the `_isnan3(near)` on a scalar at
// :79 is read as isnan(near))
ORC_API void orc_half_sample(const float* src, int dW, int dH, int radius, float thr, float* dst) {
  const int sW = dW * 2, sH = dH * 2;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < dH; ++y)
    for (int x = 0; x < dW; ++x) {
      int sx = x * 2, sy = y * 2;
      float c = src[(long)sy * sW + sx];
      int x0 = std::max(sx - radius, 0), x1 = std::min(sx + radius + 1, sW);
      int y0 = std::max(sy - radius, 0), y1 = std::min(sy + radius + 1, sH);
      float s = 0.f;
      int n = 0;
      for (int cy = y0; cy < y1; ++cy)
        for (int cx = x0; cx < x1; ++cx) {
          float nr = src[(long)cy * sW + cx];
          if (!std::isnan(nr) && (std::isnan(c) || std::fabs(c - nr) < thr)) {
            s += nr;
            n += 1;
          }
        }
      dst[(long)y * dW + x] = n > 0 ? s / (float)n : QNAN;
    }
}

// A4  depth2vertex_kernel   transformMaps.cl:18-42
ORC_API void orc_depth2vertex(const float* d, int W, int H, const OrcCam* cam, int div, float* v) {
  const float fxi = (float)div * cam->fx_inv, fyi = (float)div * cam->fy_inv;
  const float cx = cam->cx / (float)div, cy = cam->cy / (float)div;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      long i = (long)y * W + x;
      float dp = d[i];
      f3 r = mk(QNAN, QNAN, QNAN);
      if (!std::isnan(dp)) r = dp * mk(((float)x - cx) * fxi, ((float)y - cy) * fyi, 1.0f);
      st3(v, i, r);
    }
}

// A5  estimate_normals_simple_kernel   normalEstimation.cl:770-822
ORC_API void orc_normals(const float* v, int W, int H, float thr, float* n) {
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      long i = (long)y * W + x;
      f3 c = ld3(v, i);
      if (isnan3(c)) {
        st3(n, i, mk(QNAN, QNAN, QNAN));
        continue;
      }
      auto pick = [&](bool ok, long j) {
        if (!ok) return c;
        f3 q = ld3(v, j);
        if (isnan3(q) || std::fabs(c.z - q.z) > thr) return c;
        return q;
      };
      f3 l = pick(x > 0, i - 1), r = pick(x < W - 1, i + 1);
      f3 u = pick(y > 0, i - W), dn = pick(y < H - 1, i + W);
      st3(n, i, normalize3(cross3(r - l, dn - u)));
    }
}

// A6  transform_maps_kernel   transformMaps.cl:91-127
ORC_API void orc_transform_maps(const float* v, const float* n, int W, int H, const OrcXform* m,
                                float* vo, float* no) {
  const f3 r0 = mk(m->R[0], m->R[1], m->R[2]), r1 = mk(m->R[3], m->R[4], m->R[5]),
           r2 = mk(m->R[6], m->R[7], m->R[8]), t = mk(m->t[0], m->t[1], m->t[2]);
  const long N = (long)W * H;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < N; ++i) {
    f3 a = ld3(v, i);
    if (isnan3(a)) {
      st3(vo, i, mk(QNAN, QNAN, QNAN));
      st3(no, i, mk(QNAN, QNAN, QNAN));
      continue;
    }
    st3(vo, i, mk(dot3(r0, a), dot3(r1, a), dot3(r2, a)) + t);
    f3 b = ld3(n, i);
    if (isnan3(b)) {
      st3(no, i, mk(QNAN, QNAN, QNAN));
      continue;
    }
    st3(no, i, mk(dot3(r0, b), dot3(r1, b), dot3(r2, b)));
  }
}

// A9  scaleDepthsKernel   tsdfVolume.cl:8-29 (in place)
ORC_API void orc_scale_depths(float* d, int W, int H, const OrcCam* cam) {
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      long i = (long)y * W + x;
      if (std::isnan(d[i])) continue;
      float xl = ((float)x - cam->cx) * cam->fx_inv;
      float yl = ((float)y - cam->cy) * cam->fy_inv;
      float lambda = std::sqrt(xl * xl + yl * yl + 1.f);
      d[i] = d[i] * lambda;
    }
}

// A11  initializeVolume   tsdfVolume.cl:192-211
ORC_API void orc_tsdf_init(int16_t* vol, uint8_t* cvol, long nvox) {
  for (long i = 0; i < nvox; ++i) {
    vol[2 * i] = 32767;
    vol[2 * i + 1] = 0;
  }
  if (cvol) std::memset(cvol, 0, (size_t)nvox * 4);
}

// A10  integrateTsdfVolumeKernel   tsdfVolume.cl:31-190 (normals = NULL as passed by
// NuiKinfuOpenCLScene.cpp:278).  `touched` receives the number of voxels
// read-modify-written.  wrap: the shifting volume's voxelWrap (tsdfVolume.cl:71,104; voxel
// (x, y, z) lives at ((x + wx) % rx, (y + wy) % ry, (z + wz) % rz)), NULL for none.
ORC_API void orc_tsdf_integrate_wrap(const float* depth, const uint8_t* bgra, const OrcCam* cam,
                                     const OrcXform* m, const OrcTsdf* p, int16_t* vol, uint8_t* cvol,
                                     int max_color_weight, long* touched, const int* wrap) {
  const int rx = (int)p->res[0], ry = (int)p->res[1], rz = (int)p->res[2];
  const int wx = wrap ? wrap[0] : 0, wy = wrap ? wrap[1] : 0, wz = wrap ? wrap[2] : 0;
  const int W = (int)cam->W, H = (int)cam->H;
  long cnt = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : cnt)
  for (int vy = 0; vy < ry; ++vy)
    for (int vx = 0; vx < rx; ++vx) {
      const float* Ri = m->R_inv;
      const float vgx = ((float)(vx - rx / 2) + 0.5f) * p->cell[0] - m->t[0];
      const float vgy = ((float)(vy - ry / 2) + 0.5f) * p->cell[1] - m->t[1];
      float vgz = (0.5f) * p->cell[2] - m->t[2];
      const float part = vgx * vgx + vgy * vgy;
      float v_x = (Ri[0] * vgx + Ri[1] * vgy + Ri[2] * vgz) * cam->fx;
      float v_y = (Ri[3] * vgx + Ri[4] * vgy + Ri[5] * vgz) * cam->fy;
      const float v_z = (Ri[6] * vgx + Ri[7] * vgy + Ri[8] * vgz);
      float zs = 0.f;
      const float tinv = 1.f / p->trunc;
      const float dx = Ri[2] * p->cell[2] * cam->fx;
      const float dy = Ri[5] * p->cell[2] * cam->fy;
      const long base = ((long)((vx + wx) % rx) + (long)((vy + wy) % ry) * rx) * rz;
      for (int vz = 0; vz < rz; ++vz, vgz += p->cell[2], zs += p->cell[2], v_x += dx, v_y += dy) {
        float inv_z = 1.0f / (v_z + Ri[8] * zs);
        if (inv_z < 0.f) continue;
        float ux = std::round(v_x * inv_z + cam->cx);
        float uy = std::round(v_y * inv_z + cam->cy);
        if (!(ux >= 0.f && uy >= 0.f && ux < (float)W && uy < (float)H)) continue;
        long cid = (long)uy * W + (long)ux;
        float Dp = depth[cid];
        float sdf = Dp - std::sqrt(vgz * vgz + part);
        if (std::isnan(Dp) || !(sdf >= -p->trunc)) continue;
        float tsdf = std::min(1.0f, sdf * tinv);
        long idx = base + (vz + wz) % rz;
        int16_t* vp = vol + 2 * idx;
        float F = (float)vp[0] / 32766.f;
        int Wt = vp[1];
        float tn = (F * (float)Wt + tsdf) / (float)(Wt + 1);
        int wn = std::min(Wt + 1, 128);
        vp[0] = (int16_t)(tn * 32766.f);
        vp[1] = (int16_t)wn;
        ++cnt;
        if (cvol && bgra && std::fabs(sdf) < p->trunc) {
          const uint8_t* nc = bgra + 4 * cid;
          if (nc[3] != 0) {
            uint8_t* vc = cvol + 4 * idx;
            float wr = 1.f;
            float nx = ((float)(vc[0] * vc[3]) + wr * (float)nc[0]) / ((float)vc[3] + wr);
            float ny = ((float)(vc[1] * vc[3]) + wr * (float)nc[1]) / ((float)vc[3] + wr);
            float nz = ((float)(vc[2] * vc[3]) + wr * (float)nc[2]) / ((float)vc[3] + wr);
            uint8_t wnew = (uint8_t)(vc[3] + 1);
            vc[0] = (uint8_t)std::min(std::max(nx, 0.f), 255.f);
            vc[1] = (uint8_t)std::min(std::max(ny, 0.f), 255.f);
            vc[2] = (uint8_t)std::min(std::max(nz, 0.f), 255.f);
            vc[3] = std::min((uint8_t)max_color_weight, wnew);
          }
        }
      }
    }
  if (touched) *touched = cnt;
}

ORC_API void orc_tsdf_integrate(const float* depth, const uint8_t* bgra, const OrcCam* cam,
                                const OrcXform* m, const OrcTsdf* p, int16_t* vol, uint8_t* cvol,
                                int max_color_weight, long* touched) {
  orc_tsdf_integrate_wrap(depth, bgra, cam, m, p, vol, cvol, max_color_weight, touched, nullptr);
}

// ---------------------------------------------------------------------------------
// A12  raycastKernel   raycast.cl:128-277 with interpolateTrilineary raycast.cl:36-120.
// The trilinear weights are reproduced as written: the x-neighbour voxel is weighted
// with the y fraction and vice versa (raycast.cl:78-119 vs the index steps at :71-101).
namespace {
struct RcVol {
  const int16_t* v;
  int rx, ry, rz;
  float cell[3];
  int w[3];  // voxelWrap (raycast.cl:62,184,201)
  // the reference's trilinear neighbour addressing (buffer strides from the wrapped first
  // voxel), for pinning only; false: each neighbour wrapped on its own
  bool strides = false;
  // TSDF values stored as floats (the FP16 serving formats, widened), one per voxel, in place
  // of the int16 values / 32766; the weights stay those of v.  nullptr: the int16 values
  const float* values = nullptr;
  long idx(int x, int y, int z) const {
    return ((long)((y + w[1]) % ry) * rx + (x + w[0]) % rx) * rz + (z + w[2]) % rz;
  }
  // neighbour (dx, dy, dz) in {0, 1}^3 of voxel (x, y, z)
  long nidx(int x, int y, int z, int dx, int dy, int dz) const {
    if (!strides) return idx(x + dx, y + dy, z + dz);
    return idx(x, y, z) + dz + (long)dx * rz + (long)dy * rx * rz;
  }
};
inline void voxel_of(f3 p, const float* cell, int& gx, int& gy, int& gz) {
  gx = (int)std::round(p.x / cell[0]);
  gy = (int)std::round(p.y / cell[1]);
  gz = (int)std::round(p.z / cell[2]);
}
inline bool tsdf_at(const RcVol& V, long idx, float& f) {
  if (idx < 0 || idx >= (long)V.rx * V.ry * V.rz) return false;  // strides past the buffer
  int16_t a = V.v[2 * idx], w = V.v[2 * idx + 1];
  f = V.values ? V.values[idx] : (float)a / 32766.f;
  return w > 0;
}
float trilinear(f3 p, const RcVol& V) {
  int gx, gy, gz;
  voxel_of(p, V.cell, gx, gy, gz);
  if (gx <= 0 || gx >= V.rx - 1) return QNAN;
  if (gy <= 0 || gy >= V.ry - 1) return QNAN;
  if (gz <= 0 || gz >= V.rz - 1) return QNAN;
  float vx = ((float)gx + 0.5f) * V.cell[0];
  float vy = ((float)gy + 0.5f) * V.cell[1];
  float vz = ((float)gz + 0.5f) * V.cell[2];
  gx = (p.x < vx) ? gx - 1 : gx;
  gy = (p.y < vy) ? gy - 1 : gy;
  gz = (p.z < vz) ? gz - 1 : gz;
  float a = (p.x - ((float)gx + 0.5f) * V.cell[0]) / V.cell[0];
  float b = (p.y - ((float)gy + 0.5f) * V.cell[1]) / V.cell[1];
  float c = (p.z - ((float)gz + 0.5f) * V.cell[2]) / V.cell[2];
  // names follow the reference: t_abc with a = y step, b = x step, c = z step
  float t000, t001, t011, t010, t110, t111, t101, t100;
  if (!tsdf_at(V, V.idx(gx, gy, gz), t000)) return QNAN;
  if (!tsdf_at(V, V.nidx(gx, gy, gz, 0, 0, 1), t001)) return QNAN;
  if (!tsdf_at(V, V.nidx(gx, gy, gz, 1, 0, 1), t011)) return QNAN;
  if (!tsdf_at(V, V.nidx(gx, gy, gz, 1, 0, 0), t010)) return QNAN;
  if (!tsdf_at(V, V.nidx(gx, gy, gz, 1, 1, 0), t110)) return QNAN;
  if (!tsdf_at(V, V.nidx(gx, gy, gz, 1, 1, 1), t111)) return QNAN;
  if (!tsdf_at(V, V.nidx(gx, gy, gz, 0, 1, 1), t101)) return QNAN;
  if (!tsdf_at(V, V.nidx(gx, gy, gz, 0, 1, 0), t100)) return QNAN;
  return t000 * (1 - a) * (1 - b) * (1 - c) + t001 * (1 - a) * (1 - b) * c +
         t010 * (1 - a) * b * (1 - c) + t011 * (1 - a) * b * c + t100 * a * (1 - b) * (1 - c) +
         t101 * a * (1 - b) * c + t110 * a * b * (1 - c) + t111 * a * b * c;
}
}  // namespace

// ref_strides: the trilinear reads reach their neighbours by the reference's buffer strides
// from the wrapped first voxel (raycast.cl:62-108), so that a read straddling the wrap seam
// takes voxels of the next buffer row as the reference does; used to pin the rest of this
// function against the reference.  0: each neighbour is the voxel's true neighbour.
namespace {
void raycast_impl(const int16_t* vol, const float* values, const uint8_t* cvol, const OrcTsdf* p, const OrcCam* cam,
                  const OrcXform* m, int W, int H, float* vmap, float* nmap, uint8_t* cmap, long* steps_out,
                  const int* wrap, int ref_strides) {
  RcVol V{vol, (int)p->res[0], (int)p->res[1], (int)p->res[2], {p->cell[0], p->cell[1], p->cell[2]},
          {wrap ? wrap[0] : 0, wrap ? wrap[1] : 0, wrap ? wrap[2] : 0}, ref_strides != 0, values};
  const f3 off = mk(p->dim[0] / 2.0f, p->dim[1] / 2.0f, 0.f);
  const f3 r0 = mk(m->R[0], m->R[1], m->R[2]), r1 = mk(m->R[3], m->R[4], m->R[5]),
           r2 = mk(m->R[6], m->R[7], m->R[8]), t = mk(m->t[0], m->t[1], m->t[2]);
  long steps_total = 0;
#pragma omp parallel for schedule(dynamic, 2) reduction(+ : steps_total)
  for (int py = 0; py < H; ++py)
    for (int px = 0; px < W; ++px) {
      long id = (long)py * W + px;
      st3(vmap, id, mk(QNAN, QNAN, QNAN));
      st3(nmap, id, mk(QNAN, QNAN, QNAN));
      if (cmap) std::memset(cmap + 4 * id, 0, 4);
      f3 start = t + off;
      f3 nx = mk(((float)px - cam->cx) * cam->fx_inv, ((float)py - cam->cy) * cam->fy_inv, 1.f);
      nx = mk(dot3(r0, nx), dot3(r1, nx), dot3(r2, nx)) + t;
      nx = nx + off;
      f3 dir = normalize3(nx - start);
      const float* D = p->dim;
      float txmin = (std::fabs(dir.x) < 1e-14) ? 0.f : (((dir.x > 0 ? 0.f : D[0]) - start.x) / dir.x);
      float tymin = (std::fabs(dir.y) < 1e-14) ? 0.f : (((dir.y > 0 ? 0.f : D[1]) - start.y) / dir.y);
      float tzmin = (std::fabs(dir.z) < 1e-14) ? 0.f : (((dir.z > 0 ? 0.f : D[2]) - start.z) / dir.z);
      float tmin = std::max(std::max(txmin, tymin), tzmin);
      float txmax = (std::fabs(dir.x) < 1e-14) ? 1e14f : (((dir.x > 0 ? D[0] : 0.f) - start.x) / dir.x);
      float tymax = (std::fabs(dir.y) < 1e-14) ? 1e14f : (((dir.y > 0 ? D[1] : 0.f) - start.y) / dir.y);
      float tzmax = (std::fabs(dir.z) < 1e-14) ? 1e14f : (((dir.z > 0 ? D[2] : 0.f) - start.z) / dir.z);
      float tmax = std::min(std::min(txmax, tymax), tzmax);
      tmin = std::max(tmin, 0.f);
      if (tmin >= tmax) continue;
      float tc = tmin;
      int gx, gy, gz;
      voxel_of(start + dir * tc, p->cell, gx, gy, gz);
      gx = std::max(0, std::min(gx, V.rx - 1));
      gy = std::max(0, std::min(gy, V.ry - 1));
      gz = std::max(0, std::min(gz, V.rz - 1));
      float tsdf = QNAN, f;
      if (tsdf_at(V, V.idx(gx, gy, gz), f)) tsdf = f;
      const float max_time = 3 * (D[0] + D[1] + D[2]);
      const float step = p->trunc * 0.8f;
      for (; tc < max_time; tc += step) {
        float prev = tsdf;
        voxel_of(start + dir * (tc + step), p->cell, gx, gy, gz);
        if (!(gx >= 0 && gy >= 0 && gz >= 0 && gx < V.rx && gy < V.ry && gz < V.rz)) break;
        ++steps_total;
        long idx = V.idx(gx, gy, gz);
        tsdf = tsdf_at(V, idx, f) ? f : QNAN;
        if (std::isnan(tsdf) || std::isnan(prev)) continue;
        if (prev < 0.f && tsdf > 0.f) break;
        if (prev >= 0.f && tsdf <= 0.f) {
          float Ftdt = trilinear(start + dir * (tc + step), V);
          if (std::isnan(Ftdt)) break;
          float Ft = trilinear(start + dir * tc, V);
          if (std::isnan(Ft)) break;
          float Ts = tc - step * Ft / (Ftdt - Ft);
          f3 vf = start + dir * Ts;
          st3(vmap, id, vf - off);
          if (cvol && cmap) std::memcpy(cmap + 4 * id, cvol + 4 * idx, 4);
          int hx, hy, hz;
          voxel_of(start + dir * tc, p->cell, hx, hy, hz);
          if (hx > 1 && hy > 1 && hz > 1 && hx < V.rx - 2 && hy < V.ry - 2 && hz < V.rz - 2) {
            f3 q, n;
            q = vf; q.x += p->cell[0]; float fx1 = trilinear(q, V);
            q = vf; q.x -= p->cell[0]; float fx2 = trilinear(q, V);
            n.x = fx1 - fx2;
            q = vf; q.y += p->cell[1]; float fy1 = trilinear(q, V);
            q = vf; q.y -= p->cell[1]; float fy2 = trilinear(q, V);
            n.y = fy1 - fy2;
            q = vf; q.z += p->cell[2]; float fz1 = trilinear(q, V);
            q = vf; q.z -= p->cell[2]; float fz2 = trilinear(q, V);
            n.z = fz1 - fz2;
            st3(nmap, id, normalize3(n));
          }
          break;
        }
      }
    }
  if (steps_out) *steps_out = steps_total;
}
}  // namespace

ORC_API void orc_raycast_wrap_mode(const int16_t* vol, const uint8_t* cvol, const OrcTsdf* p, const OrcCam* cam,
                                   const OrcXform* m, int W, int H, float* vmap, float* nmap, uint8_t* cmap,
                                   long* steps_out, const int* wrap, int ref_strides) {
  raycast_impl(vol, nullptr, cvol, p, cam, m, W, H, vmap, nmap, cmap, steps_out, wrap, ref_strides);
}

// The same raycast over TSDF values given as floats (one per voxel, reference layout) with
// the weights of vol: the reference's march and refinement applied to the values a
// half-precision volume stores.
ORC_API void orc_raycast_values(const int16_t* vol, const float* values, const OrcTsdf* p, const OrcCam* cam,
                                const OrcXform* m, int W, int H, float* vmap, float* nmap) {
  raycast_impl(vol, values, nullptr, p, cam, m, W, H, vmap, nmap, nullptr, nullptr, nullptr, 0);
}

ORC_API void orc_raycast_wrap(const int16_t* vol, const uint8_t* cvol, const OrcTsdf* p, const OrcCam* cam,
                              const OrcXform* m, int W, int H, float* vmap, float* nmap, uint8_t* cmap,
                              long* steps_out, const int* wrap) {
  orc_raycast_wrap_mode(vol, cvol, p, cam, m, W, H, vmap, nmap, cmap, steps_out, wrap, 0);
}

ORC_API void orc_raycast(const int16_t* vol, const uint8_t* cvol, const OrcTsdf* p,
                         const OrcCam* cam, const OrcXform* m, int W, int H, float* vmap,
                         float* nmap, uint8_t* cmap, long* steps_out) {
  orc_raycast_wrap(vol, cvol, p, cam, m, W, H, vmap, nmap, cmap, steps_out, nullptr);
}

// ---------------------------------------------------------------------------------
// Shifting dense volume (NuiKinfuOpenCLShiftScene, the eScene_ShiftingVolume scene of
// NuiSLAMController.cpp:55-62): a cyclic volume addressed through voxelWrap.

// initializeVolume over a slab (tsdfVolume.cl:192-211 as launched by clearSlice,
// NuiKinfuOpenCLShiftScene.cpp:76-115): voxels (x + off) of x in [0, range) per axis.
ORC_API void orc_tsdf_clear_slice(int16_t* vol, uint8_t* cvol, const OrcTsdf* p, const int* off,
                                  const int* range) {
  const int rx = (int)p->res[0], ry = (int)p->res[1], rz = (int)p->res[2];
  for (int y = 0; y < range[1]; ++y)
    for (int x = 0; x < range[0]; ++x)
      for (int z = 0; z < range[2]; ++z) {
        const long idx = ((long)((y + off[1]) % ry) * rx + (x + off[0]) % rx) * rz + (z + off[2]) % rz;
        vol[2 * idx] = 32767;
        vol[2 * idx + 1] = 0;
        if (cvol) std::memset(cvol + 4 * idx, 0, 4);
      }
}

// fetchShiftVolumeKernel (extract.cl:82-179): surface points of a slab, from each voxel
// whose tsdf is exactly 0 and between z-neighbours of opposite sign, with the kernel's
// own index arithmetic (its z loop adds voxelWrap.z twice, and its offsets step by whole
// volumes as written).  fetchVolumeKernel (extract.cl:4-79) is the case wrap = offset = 0.
// Points go to xyz (3 floats) / rgba (4 floats) up to cap; returns how many were found.
ORC_API long orc_fetch_points(const int16_t* vol, const uint8_t* cvol, const OrcTsdf* p, const int* range,
                              const int* wrap, const int* voff, float* xyz, float* rgba, long cap) {
  const int rx = (int)p->res[0], ry = (int)p->res[1], rz = (int)p->res[2];
  const float half_x = (float)(rx >> 1), half_y = (float)(ry >> 1);
  const float* cs = p->cell;
  long n = 0;
  auto emit = [&](float x, float y, float z, const float c[4]) {
    if (n < cap) {
      xyz[3 * n] = x;
      xyz[3 * n + 1] = y;
      xyz[3 * n + 2] = z;
      std::memcpy(rgba + 4 * n, c, 4 * sizeof(float));
    }
    ++n;
  };
  for (int vx = 0; vx < range[0]; ++vx)
    for (int vy = 0; vy < range[1]; ++vy) {
      const long vid = ((long)((vy + wrap[1]) % ry) * rx + (vx + wrap[0]) % rx) * rz;
      int ob[3] = {(voff[0] / rx) * rx, (voff[1] / ry) * ry, (voff[2] / rz) * rz};
      if (voff[0] > 0) {
        if (vx < voff[0] % rx) ob[0] += rx;
      } else if (vx > rx + voff[0] % rx) {
        ob[0] -= rx;
      }
      if (voff[1] > 0) {
        if (vy < voff[1] % ry) ob[1] += ry;
      } else if (vy > ry + voff[1] % ry) {
        ob[1] -= ry;
      }
      float tsdf = QNAN;
      const int zend = range[2] + wrap[2];
      for (int vz = wrap[2]; vz < zend; ++vz) {
        const float prev = tsdf;
        const long idx = vid + (vz + wrap[2]) % rz;
        const int16_t* v = vol + 2 * idx;
        if (v[1] <= 0) {
          tsdf = QNAN;
          continue;
        }
        int oz = ob[2];
        if (voff[2] > 0) {
          if (vz < voff[2] % rz) oz += rz;
        } else if (vz > rz + voff[2] % rz) {
          oz -= rz;
        }
        tsdf = (float)v[0] / 32766.f;
        if (tsdf == 0.f) {
          float c[4] = {0.f, 0.f, 0.f, 1.f};
          if (cvol) {
            const uint8_t* g = cvol + 4 * idx;
            c[0] = (float)g[0] / 255.f;
            c[1] = (float)g[1] / 255.f;
            c[2] = (float)g[2] / 255.f;
          }
          emit(((float)(vx + ob[0]) + 0.5f - half_x) * cs[0], (-(float)(vy + ob[1]) - 0.5f + half_y) * cs[1],
               ((float)(vz + oz) + 0.5f) * cs[2], c);
        } else if ((prev < 0.f && tsdf > 0.f) || (prev > 0.f && tsdf < 0.f)) {
          const float ti = 1.f / std::fabs(tsdf), tpi = 1.f / std::fabs(prev);
          const float dp = (ti * (float)(vz + oz) + tpi * (float)(vz + oz - 1)) / (ti + tpi);
          float c[4] = {0.f, 0.f, 0.f, 1.f};
          if (cvol) {  // the crossing case reads the colour bytes in reverse order
            const uint8_t* g = cvol + 4 * idx;
            c[0] = (float)g[2] / 255.f;
            c[1] = (float)g[1] / 255.f;
            c[2] = (float)g[0] / 255.f;
          }
          emit(((float)(vx + ob[0]) + 0.5f - half_x) * cs[0], (-(float)(vy + ob[1]) - 0.5f + half_y) * cs[1],
               (dp + 0.5f) * cs[2], c);
        }
      }
    }
  return n;
}

// ---------------------------------------------------------------------------------
// A7  icp_block_kernel + compute_sums (icp.cl:222-326): per-pixel rows, summed here in
// double, each product of the row's float values taken exactly (a double fused
// multiply-add) -- the reference rounds the products to float and sums in float; the
// sums agree within its float rounding.  `vcur` is the level's vertex map (w x h), `vref`/`nref` the full-size world
// reference maps (cam->W x cam->H), Rc/tc the current estimate (row-major), prev the
// previous camera transform.  sums[0..26] = upper triangle of [J|r]^T[J|r] by rows,
// sums[27] = sum r^2, sums[28] = count.
namespace {
inline f3 bilinear_holes(const float* src, float px, float py, int W, long N) {
  int ix = (int)std::floor(px), iy = (int)std::floor(py);
  float dx = px - (float)ix, dy = py - (float)iy;
  long ia = (long)ix + (long)iy * W, ib = (long)(ix + 1) + (long)iy * W;
  long ic = (long)ix + (long)(iy + 1) * W, id = (long)(ix + 1) + (long)(iy + 1) * W;
  // linear indices past the buffer end read as holes
  if (ia >= N || ib >= N || ic >= N || id >= N) return mk(QNAN, QNAN, QNAN);
  f3 a = ld3(src, ia), b = ld3(src, ib), c = ld3(src, ic), d = ld3(src, id);
  if (isnan3(a) || isnan3(b) || isnan3(c) || isnan3(d)) return mk(QNAN, QNAN, QNAN);
  f3 r;
  r.x = a.x * (1.0f - dx) * (1.0f - dy) + b.x * dx * (1.0f - dy) + c.x * (1.0f - dx) * dy + d.x * dx * dy;
  r.y = a.y * (1.0f - dx) * (1.0f - dy) + b.y * dx * (1.0f - dy) + c.y * (1.0f - dx) * dy + d.y * dx * dy;
  r.z = a.z * (1.0f - dx) * (1.0f - dy) + b.z * dx * (1.0f - dy) + c.z * (1.0f - dx) * dy + d.z * dx * dy;
  return r;
}
}  // namespace

ORC_API void orc_icp_rows(const float* vcur, int w, int h, const float* vref, const float* nref,
                          const OrcCam* cam, const float* Rc, const float* tc, const OrcXform* prev,
                          float dist_thr, float* rows /* nullable: w*h*29 floats */, double* sums) {
  const long n = (long)w * h;
  const long NR = (long)cam->W * cam->H;
  const long CH = 4096;  // fixed chunks: the sum does not depend on the thread count
  const long nch = (n + CH - 1) / CH;
  std::vector<double> part((size_t)std::max(nch, 1L) * 29, 0.0);
  const f3 q0 = mk(Rc[0], Rc[1], Rc[2]), q1 = mk(Rc[3], Rc[4], Rc[5]), q2 = mk(Rc[6], Rc[7], Rc[8]);
  const float* Ri = prev->R_inv;
  const f3 i0 = mk(Ri[0], Ri[1], Ri[2]), i1 = mk(Ri[3], Ri[4], Ri[5]), i2 = mk(Ri[6], Ri[7], Ri[8]);
  const f3 pt = mk(prev->t[0], prev->t[1], prev->t[2]), ct = mk(tc[0], tc[1], tc[2]);
#pragma omp parallel for schedule(dynamic, 1)
  for (long ch = 0; ch < nch; ++ch) {
    double* acc = part.data() + 29 * (size_t)ch;
    for (long i = ch * CH; i < std::min(n, (ch + 1) * CH); ++i) {
      float cr[29];
      bool ok = false;
      f3 v = ld3(vcur, i);
      if (!isnan3(v)) {
        f3 pv = mk(dot3(q0, v), dot3(q1, v), dot3(q2, v)) + ct;
        f3 q = pv - pt;
        f3 pp = mk(dot3(i0, q), dot3(i1, q), dot3(i2, q));
        float u = pp.x * cam->fx / pp.z + cam->cx;
        float vv = pp.y * cam->fy / pp.z + cam->cy;
        if (u >= 0.0f && u < (float)cam->W && vv >= 0.0f && vv < (float)cam->H) {
          f3 rn = bilinear_holes(nref, u, vv, (int)cam->W, NR);
          if (!isnan3(rn)) {
            f3 rv = bilinear_holes(vref, u, vv, (int)cam->W, NR);
            if (!isnan3(rv)) {
              f3 diff = rv - pv;
              float dist = length3(diff);
              if (dist < dist_thr) {
                f3 r0 = cross3(rn, pv);
                float c7[7] = {r0.x, r0.y, r0.z, rn.x, rn.y, rn.z, dot3(rn, diff)};
                int s = 0;
                for (int a = 0; a < 6; ++a)
                  for (int b = a; b < 7; ++b) cr[s++] = c7[a] * c7[b];
                cr[s++] = c7[6] * c7[6];
                cr[s++] = 1.0f;
                // the sums take each product exactly (FP64 fused multiply-add of the FP32
                // row values), not the FP32-rounded rows above
                s = 0;
                for (int a = 0; a < 6; ++a)
                  for (int b = a; b < 7; ++b, ++s) acc[s] = std::fma((double)c7[a], (double)c7[b], acc[s]);
                acc[27] = std::fma((double)c7[6], (double)c7[6], acc[27]);
                acc[28] += 1.0;
                ok = true;
              }
            }
          }
        }
      }
      if (!ok)
        for (int k = 0; k < 29; ++k) cr[k] = 0.f;
      if (rows)
        for (int k = 0; k < 29; ++k) rows[29 * i + k] = cr[k];
    }
  }
  for (int k = 0; k < 29; ++k) {
    double s = 0.0;
    for (long c = 0; c < nch; ++c) s += part[29 * (size_t)c + k];
    sums[k] = s;
  }
}

// ---------------------------------------------------------------------------------
// A8  colour ICP.
//
// Colour pyramid   half_sample_bgra_kernel  transformMaps.cl:106-146, radius 1 from the host
// (NuiKinfuOpenCLColorTracker.cpp:159-191): pixel (x, y) of the dW x dH level is the integer
// mean (truncated) of every channel over the taps of the (2r+1)^2 window around (2x, 2y) of
// the level below, clamped to that image; alpha 255.
ORC_API void orc_color_half_sample(const uint8_t* src, int dW, int dH, int radius, uint8_t* dst) {
  const int sW = dW * 2, sH = dH * 2;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < dH; ++y)
    for (int x = 0; x < dW; ++x) {
      const int sx = 2 * x, sy = 2 * y;
      const int x0 = std::max(sx - radius, 0), x1 = std::min(sx + radius + 1, sW);
      const int y0 = std::max(sy - radius, 0), y1 = std::min(sy + radius + 1, sH);
      int sum[4] = {0, 0, 0, 0}, n = 0;
      for (int cy = y0; cy < y1; ++cy)
        for (int cx = x0; cx < x1; ++cx) {
          for (int k = 0; k < 4; ++k) sum[k] += src[4 * ((long)cy * sW + cx) + k];
          ++n;
        }
      uint8_t* o = dst + 4 * ((long)y * dW + x);
      for (int k = 0; k < 3; ++k) o[k] = (uint8_t)(n > 0 ? sum[k] / n : 0);
      o[3] = 255;
    }
}

// BGRA gradients   bgra_gradient_kernel  transformMaps.cl:514-560: Sobel / 8 of each colour
// channel in float, stored as convert_uchar (the low byte of the truncation toward zero:
// a negative gradient wraps, and since |Sobel / 8| <= 127.5 reading the byte as a signed
// char gives the truncated gradient back); alpha 255; border pixels (0, 0, 0, 0).
// The reference steps to the rows above and below by the image height and stores one row
// and one pixel past the centre, which agree with the centre-stored Sobel only on square
// images and off by (1, 1); here rows are stepped by the width and stored at the centre.
ORC_API void orc_color_gradient(const uint8_t* c, int W, int H, uint8_t* gx, uint8_t* gy) {
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const long i = (long)y * W + x;
      if (!(x > 0 && x < W - 1 && y > 0 && y < H - 1)) {
        for (int k = 0; k < 4; ++k) gx[4 * i + k] = gy[4 * i + k] = 0;
        continue;
      }
      auto px = [&](int dx, int dy, int k) { return (float)c[4 * (i + dx + (long)dy * W) + k]; };
      for (int k = 0; k < 3; ++k) {
        float tx = (px(1, -1, k) - px(-1, -1, k)) + 2 * (px(1, 0, k) - px(-1, 0, k)) + (px(1, 1, k) - px(-1, 1, k));
        float ty = (px(-1, 1, k) - px(-1, -1, k)) + 2 * (px(0, 1, k) - px(0, -1, k)) + (px(1, 1, k) - px(1, -1, k));
        tx /= 8.0f;
        ty /= 8.0f;
        gx[4 * i + k] = (uint8_t)(int)tx;
        gy[4 * i + k] = (uint8_t)(int)ty;
      }
      gx[4 * i + 3] = gy[4 * i + 3] = 255;
    }
}

// Photometric rows   color_icp_block_kernel  colorIcp.cl:91-183, per model point i of the
// full-size model maps (world vertices mv, colours mc: the previous raycast), against the
// level-`level` colour image of the current frame and its gradients.
//
// ref_mode = 1 evaluates the kernel as written, for pinning: the point is moved by (R, t)
// as given, parameters are ordered (tx, ty, tz, rx, ry, rz) with rotations about the
// camera axes, gradients are read as unsigned bytes, colours unscaled, both colours must
// have alpha 255, and the 29 outputs are packed as the kernel packs them (per parameter
// p: d_p.d_q for q <= p, then d_p.diff; then |diff|, 1).
//
// ref_mode = 0 is the tracker's form: (R, t) is the camera-to-world estimate, so the
// point's camera coordinates are R^T (m - t); the parameters are those of the depth ICP
// step ((alpha, beta, gamma, tx, ty, tz) of R <- Rinc^-1 R, t <- Rinc^-1 t + tinc), whose
// derivatives of the camera point are R^T (e_k x m) and -R^T e_k; gradients are signed
// bytes; colours and gradients are scaled by 1/255; outputs are packed like the depth
// rows: the upper triangle of [D | -diff]^T [D | -diff] by rows (21 + 6), then |diff|^2
// and 1.  In both modes a model colour counts when its alpha is 255.
ORC_API void orc_color_rows(const float* mv, const uint8_t* mc, const OrcCam* cam, int level,
                            const uint8_t* pc, const uint8_t* pgx, const uint8_t* pgy, const float* R,
                            const float* t, int ref_mode, float* rows, double* sums) {
  const int W = (int)cam->W, H = (int)cam->H;
  const long n = (long)W * H;
  const int div = 1 << level;
  const float fx = cam->fx / (float)div, fy = cam->fy / (float)div;
  const float cx = cam->cx / (float)div, cy = cam->cy / (float)div;
  const int lw = W / div, lh = H / div;
  const long CH = 4096;
  const long nch = (n + CH - 1) / CH;
  std::vector<double> part((size_t)std::max(nch, 1L) * 29, 0.0);
  const float k255 = 1.0f / 255.0f;
#pragma omp parallel for schedule(dynamic, 1)
  for (long ch = 0; ch < nch; ++ch) {
    double* acc = part.data() + 29 * (size_t)ch;
    for (long i = ch * CH; i < std::min(n, (ch + 1) * CH); ++i) {
      float cr[29];
      for (int k = 0; k < 29; ++k) cr[k] = 0.f;
      bool ok = false;
      const f3 m = ld3(mv, i);
      const uint8_t* kc = mc + 4 * i;
      if (!isnan3(m) && kc[3] == 255) {
        f3 p;
        if (ref_mode) {
          p = mk(dot3(mk(R[0], R[1], R[2]), m), dot3(mk(R[3], R[4], R[5]), m), dot3(mk(R[6], R[7], R[8]), m)) +
              mk(t[0], t[1], t[2]);
        } else {
          const f3 d = m - mk(t[0], t[1], t[2]);
          p = mk(dot3(mk(R[0], R[3], R[6]), d), dot3(mk(R[1], R[4], R[7]), d), dot3(mk(R[2], R[5], R[8]), d));
        }
        const int u = (int)std::round(p.x * fx / p.z + cx), v = (int)std::round(p.y * fy / p.z + cy);
        if (u >= 0 && u < lw && v >= 0 && v < lh) {
          const long li = (long)v * lw + u;
          const uint8_t *co = pc + 4 * li, *gx = pgx + 4 * li, *gy = pgy + 4 * li;
          if (co[3] == 255 && gx[3] == 255 && gy[3] == 255) {
            f3 diff = mk((float)co[0] - (float)kc[0], (float)co[1] - (float)kc[1], (float)co[2] - (float)kc[2]);
            f3 g1, g2;
            if (ref_mode) {
              g1 = mk((float)gx[0], (float)gx[1], (float)gx[2]);
              g2 = mk((float)gy[0], (float)gy[1], (float)gy[2]);
            } else {
              diff = diff * k255;
              g1 = mk((float)(int8_t)gx[0], (float)(int8_t)gx[1], (float)(int8_t)gx[2]) * k255;
              g2 = mk((float)(int8_t)gy[0], (float)(int8_t)gy[1], (float)(int8_t)gy[2]) * k255;
            }
            f3 d[6];
            for (int k = 0; k < 6; ++k) {
              f3 dp;
              if (ref_mode) {
                switch (k) {
                  case 0: dp = mk(1.f, 0.f, 0.f); break;
                  case 1: dp = mk(0.f, 1.f, 0.f); break;
                  case 2: dp = mk(0.f, 0.f, 1.f); break;
                  case 3: dp = mk(0.f, -p.z, p.y); break;
                  case 4: dp = mk(p.z, 0.f, -p.x); break;
                  default: dp = mk(-p.y, p.x, 0.f); break;
                }
              } else {
                f3 w;  // e_k x m (rotations) or -e_k (translations), then R^T
                switch (k) {
                  case 0: w = mk(0.f, -m.z, m.y); break;
                  case 1: w = mk(m.z, 0.f, -m.x); break;
                  case 2: w = mk(-m.y, m.x, 0.f); break;
                  case 3: w = mk(-1.f, 0.f, 0.f); break;
                  case 4: w = mk(0.f, -1.f, 0.f); break;
                  default: w = mk(0.f, 0.f, -1.f); break;
                }
                dp = mk(dot3(mk(R[0], R[3], R[6]), w), dot3(mk(R[1], R[4], R[7]), w), dot3(mk(R[2], R[5], R[8]), w));
              }
              const float zz = p.z * p.z;
              const float jx = fx * ((p.z * dp.x - dp.z * p.x) / zz);
              const float jy = fy * ((p.z * dp.y - dp.z * p.y) / zz);
              d[k] = mk(jx * g1.x + jy * g2.x, jx * g1.y + jy * g2.y, jx * g1.z + jy * g2.z);
            }
            int s = 0;
            if (ref_mode) {
              for (int a = 0; a < 6; ++a) {
                for (int b = 0; b <= a; ++b) cr[s++] = dot3(d[a], d[b]);
                cr[s++] = dot3(d[a], diff);
              }
              cr[s++] = length3(diff);
            } else {
              const f3 nd = mk(-diff.x, -diff.y, -diff.z);
              for (int a = 0; a < 6; ++a) {
                for (int b = a; b < 6; ++b) cr[s++] = dot3(d[a], d[b]);
                cr[s++] = dot3(d[a], nd);
              }
              cr[s++] = dot3(diff, diff);
            }
            cr[s++] = 1.0f;
            ok = true;
          }
        }
      }
      if (rows)
        for (int k = 0; k < 29; ++k) rows[29 * i + k] = cr[k];
      if (ok)
        for (int k = 0; k < 29; ++k) acc[k] += (double)cr[k];
    }
  }
  for (int k = 0; k < 29; ++k) {
    double s = 0.0;
    for (long c = 0; c < nch; ++c) s += part[29 * (size_t)c + k];
    sums[k] = s;
  }
}

// ---------------------------------------------------------------------------------
// Small dense linear algebra for the ICP host step (Eigen in the reference; Eigen is not
// vendored, so these are textbook restatements: partial-pivot LU determinant and
// Cholesky LL^T solve, both in double).
namespace {
double det6(const double A_in[36]) {
  double A[36];
  std::memcpy(A, A_in, sizeof(A));
  double det = 1.0;
  for (int c = 0; c < 6; ++c) {
    int piv = c;
    for (int r = c + 1; r < 6; ++r)
      if (std::fabs(A[r * 6 + c]) > std::fabs(A[piv * 6 + c])) piv = r;
    if (A[piv * 6 + c] == 0.0) return 0.0;
    if (piv != c) {
      for (int k = 0; k < 6; ++k) std::swap(A[c * 6 + k], A[piv * 6 + k]);
      det = -det;
    }
    det *= A[c * 6 + c];
    for (int r = c + 1; r < 6; ++r) {
      double f = A[r * 6 + c] / A[c * 6 + c];
      for (int k = c; k < 6; ++k) A[r * 6 + k] -= f * A[c * 6 + k];
    }
  }
  return det;
}
bool llt_solve6(const double A[36], const double b[6], double x[6]) {
  double L[36] = {0};
  for (int j = 0; j < 6; ++j) {
    double s = A[j * 6 + j];
    for (int k = 0; k < j; ++k) s -= L[j * 6 + k] * L[j * 6 + k];
    if (!(s > 0.0)) return false;
    L[j * 6 + j] = std::sqrt(s);
    for (int i = j + 1; i < 6; ++i) {
      double t = A[i * 6 + j];
      for (int k = 0; k < j; ++k) t -= L[i * 6 + k] * L[j * 6 + k];
      L[i * 6 + j] = t / L[j * 6 + j];
    }
  }
  double y[6];
  for (int i = 0; i < 6; ++i) {
    double t = b[i];
    for (int k = 0; k < i; ++k) t -= L[i * 6 + k] * y[k];
    y[i] = t / L[i * 6 + i];
  }
  for (int i = 5; i >= 0; --i) {
    double t = y[i];
    for (int k = i + 1; k < 6; ++k) t -= L[k * 6 + i] * x[k];
    x[i] = t / L[i * 6 + i];
  }
  return true;
}
// Rz(g) * Ry(b) * Rx(a) (Eigen AngleAxis composition at NuiKinfuOpenCLDepthTracker.cpp:486)
void euler_zyx(double a, double b, double g, double R[9]) {
  double ca = std::cos(a), sa = std::sin(a), cb = std::cos(b), sb = std::sin(b), cg = std::cos(g),
         sg = std::sin(g);
  double Rz[9] = {cg, -sg, 0, sg, cg, 0, 0, 0, 1};
  double Ry[9] = {cb, 0, sb, 0, 1, 0, -sb, 0, cb};
  double Rx[9] = {1, 0, 0, 0, ca, -sa, 0, sa, ca};
  double T[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += Rz[i * 3 + k] * Ry[k * 3 + j];
      T[i * 3 + j] = s;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += T[i * 3 + k] * Rx[k * 3 + j];
      R[i * 3 + j] = s;
    }
}
}  // namespace

// 3x3 inverse by cofactors, double precision, rounded to float (NuiKinfuOpenCLCameraState.cpp:83)
ORC_API void orc_inverse3(const float* R, float* Ri) {
  double a[9];
  for (int i = 0; i < 9; ++i) a[i] = R[i];
  double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
  double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  double inv[9] = {c00, a[2] * a[7] - a[1] * a[8], a[1] * a[5] - a[2] * a[4],
                   c01, a[0] * a[8] - a[2] * a[6], a[2] * a[3] - a[0] * a[5],
                   c02, a[1] * a[6] - a[0] * a[7], a[0] * a[4] - a[1] * a[3]};
  for (int i = 0; i < 9; ++i) Ri[i] = (float)(inv[i] / det);
}

ORC_API void orc_make_xform(const float* R, const float* t, OrcXform* out) {
  std::memcpy(out->R, R, 9 * sizeof(float));
  orc_inverse3(R, out->R_inv);
  std::memcpy(out->t, t, 3 * sizeof(float));
}

struct OrcIcpStats {
  float error, count;
  int iterations;
  int status;  // 0 ok, 1 singular (tracking lost)
};

// Photometric term of the colour tracker (A8), used at the finest level: the world
// vertices of the previous raycast with the previous frame's colours (the raycast is
// rendered from the previous pose, so pixel i of both holds the same surface point), and
// the current frame's colour image and gradients; weight on its normal equations.
struct OrcColorIcp {
  const float* mv;      // model world vertices (W x H float3)
  const uint8_t* mc;    // model colours: the previous frame (W x H BGRA)
  const uint8_t* pyr;   // current frame (W x H BGRA)
  const uint8_t* gx;    // its x / y gradients (signed bytes)
  const uint8_t* gy;
  float weight;
};

// A7 host loop   NuiKinfuOpenCLDepthTracker.cpp:240-504.
// vlevels[l] is the level-l vertex map ((W>>l) x (H>>l)); iters[l] its iteration count.
// R/t: in = initial estimate, out = estimate.  Returns 0 on success, 1 on singular system.
// With `col` (nullable, weight > 0) every iteration of the finest level adds the
// photometric normal equations of orc_color_rows times the weight to the point-to-plane
// ones, and the weighted |diff|^2 sum to the residual sum; the accept/reject count stays
// the depth count.
// The 29 sums of one iteration at level lv for the estimate (R, t); user: the caller's state.
typedef void (*OrcIcpRowsFn)(void* user, int lv, const float* R, const float* t, double* sums29);
static int icp_host_loop(const float* const* vlevels, const int* iters, int levels, const float* vref,
                         const float* nref, const OrcCam* cam, const OrcXform* prev, float dist_thr, float* R,
                         float* t, OrcIcpStats* stats, const OrcColorIcp* col, OrcIcpRowsFn rows_fn, void* user);

ORC_API int orc_icp(const float* const* vlevels, const int* iters, int levels, const float* vref,
                    const float* nref, const OrcCam* cam, const OrcXform* prev, float dist_thr,
                    float* R, float* t, OrcIcpStats* stats, const OrcColorIcp* col) {
  return icp_host_loop(vlevels, iters, levels, vref, nref, cam, prev, dist_thr, R, t, stats, col, nullptr, nullptr);
}

// The same host loop with the per-iteration sums supplied by the caller (for example the
// reference's own icp_block_kernel + compute_sums run on the host).
ORC_API int orc_icp_with_rows(const int* iters, int levels, const OrcCam* cam, float* R, float* t,
                              OrcIcpStats* stats, OrcIcpRowsFn rows_fn, void* user) {
  return icp_host_loop(nullptr, iters, levels, nullptr, nullptr, cam, nullptr, 0.f, R, t, stats, nullptr, rows_fn,
                       user);
}

static int icp_host_loop(const float* const* vlevels, const int* iters, int levels, const float* vref,
                         const float* nref, const OrcCam* cam, const OrcXform* prev, float dist_thr, float* R,
                         float* t, OrcIcpStats* stats, const OrcColorIcp* col, OrcIcpRowsFn rows_fn, void* user) {
  size_t gsize = (size_t)cam->W * cam->H;  // kernelGlobalSize[0]; stale across levels
  float Rc[9], tc[3];
  std::memcpy(Rc, R, sizeof(Rc));
  std::memcpy(tc, t, sizeof(tc));
  float err = 0.f, cnt = 0.f;
  int total_iters = 0;
  for (int lv = levels - 1; lv >= 0; --lv) {
    const unsigned thr = (unsigned)((double)(gsize >> (2 * lv)) * 0.1);
    float lambda = 1.0f;
    float Rg[9], tg[3];
    std::memcpy(Rg, Rc, sizeof(Rg));
    std::memcpy(tg, tc, sizeof(tg));
    float errOld = 1e20f;
    double good[27] = {0};
    const int w = (int)cam->W >> lv, h = (int)cam->H >> lv;
    for (int it = 0; it < iters[lv]; ++it) {
      double sums[29];
      if (rows_fn)
        rows_fn(user, lv, Rc, tc, sums);
      else
        orc_icp_rows(vlevels[lv], w, h, vref, nref, cam, Rc, tc, prev, dist_thr, nullptr, sums);
      if (col && col->weight > 0.f && lv == 0) {
        double sc[29];
        orc_color_rows(col->mv, col->mc, cam, 0, col->pyr, col->gx, col->gy, Rc, tc, 0, nullptr, sc);
        for (int k = 0; k < 28; ++k) sums[k] += (double)col->weight * sc[k];
      }
      ++total_iters;
      gsize = (size_t)w * h;
      unsigned size = (unsigned)std::ceil((float)gsize / 128.f);
      unsigned nblocks = (unsigned)std::ceil((float)size / 128.f);
      gsize = (size_t)nblocks * 128;
      err = (float)sums[27];
      cnt = (float)sums[28];
      err = (cnt > 0.f) ? std::sqrt(err) / cnt : std::numeric_limits<float>::max();
      if (cnt < (float)thr || err > errOld) {
        lambda *= 10.0f;
        std::memcpy(Rc, Rg, sizeof(Rc));
        std::memcpy(tc, tg, sizeof(tc));
        if (it == 0) break;
      } else {
        lambda /= 10.0f;
        std::memcpy(Rg, Rc, sizeof(Rg));
        std::memcpy(tg, tc, sizeof(tg));
        errOld = err;
        for (int k = 0; k < 27; ++k) good[k] = sums[k];
      }
      double A[36], b[6];
      for (int i = 0, s = 0; i < 6; ++i) {
        for (int j = i; j < 7; ++j, ++s) {
          double v = good[s] / (double)cnt;
          if (j == 6)
            b[i] = v;
          else
            A[j * 6 + i] = A[i * 6 + j] = v;
        }
        A[i * 6 + i] *= (double)(1.0f + lambda);
      }
      double det = det6(A);
      if (std::fabs(det) < 1e-15 || std::isnan(det)) {
        if (stats) *stats = OrcIcpStats{err, cnt, total_iters, 1};
        return 1;
      }
      double x[6];
      if (!llt_solve6(A, b, x)) {
        if (stats) *stats = OrcIcpStats{err, cnt, total_iters, 1};
        return 1;
      }
      float al = (float)x[0], be = (float)x[1], ga = (float)x[2];
      if (al * al + be * be + ga * ga < 1e-6f) break;
      double Rinc[9];
      euler_zyx(al, be, ga, Rinc);
      // RincInv = Rinc^T ; t = RincInv t + tinc ; R = RincInv R
      double tn[3], Rn[9];
      for (int i = 0; i < 3; ++i) {
        double s = 0;
        for (int k = 0; k < 3; ++k) s += Rinc[k * 3 + i] * (double)tc[k];
        tn[i] = s + (double)(float)x[3 + i];
      }
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          double s = 0;
          for (int k = 0; k < 3; ++k) s += Rinc[k * 3 + i] * (double)Rc[k * 3 + j];
          Rn[i * 3 + j] = s;
        }
      for (int i = 0; i < 3; ++i) tc[i] = (float)tn[i];
      for (int i = 0; i < 9; ++i) Rc[i] = (float)Rn[i];
    }
  }
  std::memcpy(R, Rc, sizeof(Rc));
  std::memcpy(t, tc, sizeof(tc));
  if (stats) *stats = OrcIcpStats{err, cnt, total_iters, 0};
  return 0;
}

// ---------------------------------------------------------------------------------
// A13  marchingCubeKernel   marchingCube.cl:100-256, emitted in the order of the
// reference's own CPU extraction (y, then x, then z fastest; NuiKinfuOpenCLScene.cpp:823-836).
// Outputs: per-cube case index (nullable, (rx-1)*(ry-1)*(rz-1) bytes in that order, 0 for
// skipped cubes), vertex positions / colours up to `cap` vertices, the total vertex
// count (uncapped) and, if `cvol` is null, colours (0,0,0,1).
ORC_API long orc_marching_cubes(const int16_t* vol, const uint8_t* cvol, const OrcTsdf* p,
                                uint8_t* cases, float* pos, float* col, long cap) {
  const int rx = (int)p->res[0], ry = (int)p->res[1], rz = (int)p->res[2];
  const float hx = (float)(rx >> 1), hy = (float)(ry >> 1);
  const float* cs = p->cell;
  auto node = [&](int x, int y, int z) {
    return mk(((float)x + 0.5f - hx) * cs[0], (-(float)y - 0.5f + hy) * cs[1], ((float)z + 0.5f) * cs[2]);
  };
  auto vidx = [&](int x, int y, int z) { return ((long)y * rx + x) * rz + z; };
  long out = 0;
  long ci = 0;
  for (int y = 0; y < ry - 1; ++y)
    for (int x = 0; x < rx - 1; ++x)
      for (int z = 0; z < rz - 1; ++z, ++ci) {
        long id[8] = {vidx(x, y, z),         vidx(x + 1, y, z),         vidx(x + 1, y + 1, z),
                      vidx(x, y + 1, z),     vidx(x, y, z + 1),         vidx(x + 1, y, z + 1),
                      vidx(x + 1, y + 1, z + 1), vidx(x, y + 1, z + 1)};
        float f[8];
        bool ok = true;
        for (int k = 0; k < 8; ++k) {
          if (vol[2 * id[k] + 1] <= 0) {
            ok = false;
            break;
          }
          f[k] = (float)vol[2 * id[k]] / 32766.f;
        }
        if (cases) cases[ci] = 0;
        if (!ok) continue;
        int cube = 0;
        for (int k = 0; k < 8; ++k) cube += (f[k] < 0) ? (1 << k) : 0;
        if (cases) cases[ci] = (uint8_t)cube;
        uint64_t word = NUI_MC_TRI_PACKED[cube];
        int ntri = (int)(word >> 60);
        if (ntri == 0) continue;
        f3 v[8] = {node(x, y, z),         node(x + 1, y, z),         node(x + 1, y + 1, z),
                   node(x, y + 1, z),     node(x, y, z + 1),         node(x + 1, y, z + 1),
                   node(x + 1, y + 1, z + 1), node(x, y + 1, z + 1)};
        static const int E[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                     {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
        for (int k = 0; k < 3 * ntri; ++k, ++out) {
          int e = (int)((word >> (4 * k)) & 0xF);
          int a = E[e][0], b = E[e][1];
          float tt = (0.f - f[a]) / (f[b] - f[a] + 1e-15f);
          tt = std::min(std::max(tt, 0.0f), 1.0f);
          f3 q = v[a] + (v[b] - v[a]) * tt;
          if (out < cap) {
            if (pos) st3(pos, out, q);
            if (col) {
              float* c = col + 4 * out;
              if (cvol) {
                const uint8_t* cc = cvol + 4 * (std::fabs(f[a]) < std::fabs(f[b]) ? id[a] : id[b]);
                c[0] = (float)cc[2] / 255.f;
                c[1] = (float)cc[1] / 255.f;
                c[2] = (float)cc[0] / 255.f;
              } else {
                c[0] = c[1] = c[2] = 0.f;
              }
              c[3] = 1.f;
            }
          }
        }
      }
  return out;
}

// A14  exclusive scan of (flag > 0) + compaction of flagged ids in increasing order.
// NuiOpenCLPrefixSum.cpp:16-311 / prefixSum.cl:10-232 under their intended semantics
// (every flagged id written once; count = number of flags).
ORC_API long orc_scan_compact(const uint8_t* flags, long n, uint32_t* prefix, int32_t* ids) {
  long s = 0;
  for (long i = 0; i < n; ++i) {
    if (prefix) prefix[i] = (uint32_t)s;
    if (flags[i] > 0) {
      if (ids) ids[s] = (int32_t)i;
      ++s;
    }
  }
  return s;
}

// ---------------------------------------------------------------------------------
// A20  per-frame driver: NuiKinfuTrackingEngine::RunTracking (NuiKinfuTrackingEngine.cpp:68-142)
// over the dense scene (NuiKinfuOpenCLScene), the OpenCL frame / feedback frame and the
// depth tracker, with the integration gate of :115-127.
struct OrcEngineCfg {
  int W, H;
  float fx, fy, cx, cy, dmin, dmax;
  int res[3];
  float dim[3];
  float trunc_cfg;  // VolumeTrancDist; the scene uses max(cfg, 2.1 * cell)
  int color;        // colour volume on/off
  int max_color_weight;
  int levels;
  int iters[4];  // finest level first (NuiTrackerConfig::iterations)
  int filter_radius;
  float sigma_space2_inv_half, sigma_depth2_inv_half, depth_threshold, dist_threshold;
  float integration_threshold;
  int hash;  // 1: voxel-block hash scene (NuiKinfuOpenCLHashScene) instead of the dense volume
  float voxel, mu;
  int buckets, excess, pool, max_w;
  float photometric_weight;  // > 0 (with colour): the colour tracker's term joins ICP
  int voxel_shift;           // > 0: the shifting dense volume (NuiKinfuVolumeConfig::voxel_shift)
  float shift_basis[3];      // NuiKinfuVolumeConfig::translateBasis
  long point_cap;            // points kept of the slabs that leave the shifting volume
  int swapping;              // hash scene: the global cache (NuiHashingSDFConfig::m_bUseSwapping)
  int forward_render;        // hash scene: ForwardRender instead of the full raycast (m_bUseForwardRender)
};

struct OrcHash;
OrcHash* orc_hash_create_internal(int buckets, int excess, int pool, float voxel, float mu, int max_w,
                                  int swapping);
void orc_hash_destroy_internal(OrcHash* h);
void orc_hash_scene_integrate(OrcHash* h, const float* depth, const uint8_t* bgra, const OrcCam* cam,
                              const OrcXform* m, long* touched);
void orc_hash_scene_raycast(OrcHash* h, const OrcCam* cam, const OrcXform* m, float* vmap, float* nmap,
                            uint8_t* cmap);

struct OrcEngine {
  OrcEngineCfg c;
  OrcCam cam;
  OrcTsdf tp;
  OrcXform xf;
  float lastR[9], lastT[3];
  long frames = 0;
  std::vector<int16_t> vol;
  std::vector<uint8_t> cvol;
  std::vector<float> gauss, depth, filt, vref, nref, normals;
  std::vector<std::vector<float>> dl, vl;  // per-level depth / vertices
  OrcIcpStats last{};
  long touched = 0;
  OrcHash* hs = nullptr;
  // colour tracking: the previous frame's colours, the current frame's gradients
  std::vector<uint8_t> cprev, cgx, cgy;
  // shifting volume: m_voxel_offset and the point cache (NuiKinfuVertexCache)
  int voff[3] = {0, 0, 0};
  std::vector<float> pts_xyz, pts_rgba;
  long pts_n = 0;
};

ORC_API OrcEngine* orc_engine_create(const OrcEngineCfg* cfg) {
  OrcEngine* e = new OrcEngine();
  e->c = *cfg;
  const OrcEngineCfg& c = e->c;
  e->cam = OrcCam{c.fx, c.fy, 1 / c.fx, 1 / c.fy, c.cx, c.cy, (uint32_t)c.W, (uint32_t)c.H, c.dmin, c.dmax};
  for (int i = 0; i < 3; ++i) {
    e->tp.res[i] = (float)c.res[i];
    e->tp.dim[i] = c.dim[i];
    e->tp.cell[i] = c.dim[i] / (float)c.res[i];
  }
  e->tp.trunc = std::max(c.trunc_cfg, 2.1f * std::max(e->tp.cell[0], std::max(e->tp.cell[1], e->tp.cell[2])));
  if (c.hash) {
    e->hs = orc_hash_create_internal(c.buckets, c.excess, c.pool, c.voxel, c.mu, c.max_w, c.swapping);
  } else {
    long nvox = (long)c.res[0] * c.res[1] * c.res[2];
    e->vol.resize(2 * nvox);
    if (c.color) e->cvol.resize(4 * nvox);
    orc_tsdf_init(e->vol.data(), c.color ? e->cvol.data() : nullptr, nvox);
  }
  e->gauss.resize(2 * c.filter_radius + 1);
  orc_gaussian_table(c.filter_radius, c.sigma_space2_inv_half, e->gauss.data());
  long N = (long)c.W * c.H;
  e->depth.resize(N);
  e->filt.resize(N);
  e->vref.resize(3 * N);
  e->nref.resize(3 * N);
  e->normals.resize(3 * N);
  e->dl.resize(c.levels);
  e->vl.resize(c.levels);
  if (c.color && c.photometric_weight > 0.f) {
    e->cprev.assign(4 * N, 0);
    e->cgx.assign(4 * N, 0);
    e->cgy.assign(4 * N, 0);
  }
  for (int l = 0; l < c.levels; ++l) {
    long n = (long)(c.W >> l) * (c.H >> l);
    e->dl[l].resize(n);
    e->vl[l].resize(3 * n);
  }
  float I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, z[3] = {0, 0, 0};
  orc_make_xform(I, z, &e->xf);
  std::memcpy(e->lastR, I, sizeof(I));
  std::memcpy(e->lastT, z, sizeof(z));
  return e;
}

ORC_API void orc_engine_destroy(OrcEngine* e) {
  if (e->hs) orc_hash_destroy_internal(e->hs);
  delete e;
}

static double rel_angle(const float* Ra, const float* Rb) {
  // angle of Ra^-1 Rb (rodrigues2 norm, NuiMatrixUtilities.cpp:7-52)
  double tr = 0;
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) tr += (double)Ra[k * 3 + i] * (double)Rb[k * 3 + i];
  double cv = std::max(-1.0, std::min(1.0, (tr - 1.0) / 2.0));
  return std::acos(cv);
}

// NuiKinfuOpenCLShiftScene::getVoxelWrap (NuiKinfuOpenCLShiftScene.cpp:44-56)
static void engine_voxel_wrap(const OrcEngine* e, int* w) {
  for (int a = 0; a < 3; ++a) w[a] = e->voff[a] >= 0 ? e->voff[a] : e->c.res[a] - ((-e->voff[a]) % e->c.res[a]);
}

// The camera's global translation: local + getVoxelOffsetSize (:58-66); a fixed volume
// (offset 0) keeps the local translation.
static void engine_global_t(const OrcEngine* e, float* g) {
  for (int a = 0; a < 3; ++a) g[a] = e->voff[a] ? e->xf.t[a] + (float)e->voff[a] * e->tp.cell[a] : e->xf.t[a];
}

// fetchAndClearX/Y/Z (:235-286): the slab of |tr| voxels that leaves the volume goes to the
// point cache (fetchSlice, :117-233), is cleared (clearSlice, :76-115), and the offset moves.
static void engine_fetch_and_clear(OrcEngine* e, int a, int tr) {
  const OrcEngineCfg& c = e->c;
  int off = e->voff[a];
  if (tr < 0) off += tr;
  off = off >= 0 ? off % c.res[a] : c.res[a] - (-off) % c.res[a];
  int wrap[3] = {0, 0, 0}, range[3] = {c.res[0], c.res[1], c.res[2]};
  wrap[a] = off;
  range[a] = std::abs(tr);
  if (c.point_cap > 0) {
    const long room = std::max(0L, c.point_cap - e->pts_n);
    std::vector<float> xyz(3 * (size_t)room + 3), rgba(4 * (size_t)room + 4);
    const long n = orc_fetch_points(e->vol.data(), c.color ? e->cvol.data() : nullptr, &e->tp, range, wrap, e->voff,
                                    xyz.data(), rgba.data(), room);
    const long keep = std::min(n, room);
    e->pts_xyz.insert(e->pts_xyz.end(), xyz.begin(), xyz.begin() + 3 * keep);
    e->pts_rgba.insert(e->pts_rgba.end(), rgba.begin(), rgba.begin() + 4 * keep);
    e->pts_n += n;
  }
  orc_tsdf_clear_slice(e->vol.data(), c.color ? e->cvol.data() : nullptr, &e->tp, wrap, range);
  e->voff[a] += tr;
}

// shiftVolume (:288-351) on the camera's local translation, before the integration.
static void engine_shift_volume(OrcEngine* e) {
  const OrcEngineCfg& c = e->c;
  float st[3];
  int tr[3];
  for (int a = 0; a < 3; ++a) {
    st[a] = e->xf.t[a] - c.shift_basis[a];
    const int f = (int)std::floor(st[a] / e->tp.cell[a]);
    tr[a] = st[a] < 0 ? std::max(-c.voxel_shift, f) : std::min(c.voxel_shift, f);
  }
  for (int a = 0; a < 3; ++a)
    if (std::abs(tr[a]) >= c.voxel_shift) {
      engine_fetch_and_clear(e, a, tr[a]);
      st[a] -= (float)tr[a] * e->tp.cell[a];
    }
  float R[9], t[3];
  std::memcpy(R, e->xf.R, sizeof(R));
  for (int a = 0; a < 3; ++a) t[a] = st[a] + c.shift_basis[a];
  orc_make_xform(R, t, &e->xf);
}

// NuiKinfuScene::integrateVolume of the configured scene on the pass-filtered depth: the
// hash scene, the fixed volume, or the shifting volume (shift, then integrate through the
// wrap).
static void engine_integrate(OrcEngine* e, const uint8_t* col) {
  const OrcEngineCfg& c = e->c;
  if (e->hs) {
    orc_hash_scene_integrate(e->hs, e->depth.data(), col, &e->cam, &e->xf, &e->touched);
    return;
  }
  if (c.voxel_shift > 0) engine_shift_volume(e);
  int w[3];
  engine_voxel_wrap(e, w);
  orc_scale_depths(e->depth.data(), c.W, c.H, &e->cam);
  orc_tsdf_integrate_wrap(e->depth.data(), col, &e->cam, &e->xf, &e->tp, e->vol.data(),
                          c.color ? e->cvol.data() : nullptr, c.max_color_weight, &e->touched, w);
}

// NuiKinfuScene::raycastRender into the reference maps.
ORC_API long orc_hash_forward_render(OrcHash* h, const OrcCam* cam, const OrcXform* m, const float* vprev,
                                     const uint8_t* cprev, float* vmap, float* nmap, uint8_t* cmap, float* range_out,
                                     uint8_t* missing_out, int mode);
static void engine_raycast(OrcEngine* e) {
  const OrcEngineCfg& c = e->c;
  if (e->hs) {
    if (c.forward_render) {  // from the previous maps (a copy: the render rewrites vref)
      const std::vector<float> vprev = e->vref;
      orc_hash_forward_render(e->hs, &e->cam, &e->xf, vprev.data(), nullptr, e->vref.data(), e->nref.data(), nullptr,
                              nullptr, nullptr, c.forward_render);
    } else {
      orc_hash_scene_raycast(e->hs, &e->cam, &e->xf, e->vref.data(), e->nref.data(), nullptr);
    }
    return;
  }
  int w[3];
  engine_voxel_wrap(e, w);
  orc_raycast_wrap(e->vol.data(), c.color ? e->cvol.data() : nullptr, &e->tp, &e->cam, &e->xf, c.W, c.H,
                   e->vref.data(), e->nref.data(), nullptr, nullptr, w);
}

// Returns 0 on success, 1 when tracking is lost (singular ICP system).
ORC_API int orc_engine_frame(OrcEngine* e, const uint16_t* raw, const uint8_t* bgra) {
  const OrcEngineCfg& c = e->c;
  const int W = c.W, H = c.H;
  const long N = (long)W * H;
  e->touched = 0;  // voxels updated by this frame (0 when the gate skips the integration)
  orc_pass_filter(raw, N, c.dmin, c.dmax, e->depth.data());
  orc_bilateral(e->depth.data(), W, H, e->gauss.data(), c.filter_radius, c.sigma_depth2_inv_half,
                c.depth_threshold, e->dl[0].data());
  orc_depth2vertex(e->dl[0].data(), W, H, &e->cam, 1, e->vl[0].data());
  const uint8_t* col = c.color ? bgra : nullptr;
  // NuiKinfuScene::integrateVolume of the configured scene
  auto integrate = [&]() { engine_integrate(e, col); };
  const bool photometric = col && !e->cprev.empty();
  if (e->frames == 0) {
    orc_normals(e->vl[0].data(), W, H, c.depth_threshold, e->normals.data());
    orc_transform_maps(e->vl[0].data(), e->normals.data(), W, H, &e->xf, e->vref.data(), e->nref.data());
    integrate();
  } else {
    for (int l = 1; l < c.levels; ++l) {
      orc_half_sample(e->dl[l - 1].data(), W >> l, H >> l, 1, c.depth_threshold, e->dl[l].data());
      orc_depth2vertex(e->dl[l].data(), W >> l, H >> l, &e->cam, 1 << l, e->vl[l].data());
    }
    std::vector<const float*> lv(c.levels);
    for (int l = 0; l < c.levels; ++l) lv[l] = e->vl[l].data();
    float R[9], t[3];
    std::memcpy(R, e->xf.R, sizeof(R));
    std::memcpy(t, e->xf.t, sizeof(t));
    const float step = c.dist_threshold / (float)c.levels;
    const float dthr = c.dist_threshold + step;
    OrcColorIcp ci{};
    if (photometric) {  // NuiKinfuOpenCLColorTracker::GradientBuffers (:194-242), finest level
      orc_color_gradient(col, W, H, e->cgx.data(), e->cgy.data());
      ci = OrcColorIcp{e->vref.data(), e->cprev.data(), col, e->cgx.data(), e->cgy.data(), c.photometric_weight};
    }
    int st = orc_icp(lv.data(), c.iters, c.levels, e->vref.data(), e->nref.data(), &e->cam, &e->xf, dthr,
                     R, t, &e->last, photometric ? &ci : nullptr);
    if (st != 0) return 1;
    orc_make_xform(R, t, &e->xf);
    // the gate compares global translations (local + volume offset, NuiCameraPos.h:43);
    // lastT holds the global translation of the last integration
    double rn = rel_angle(e->xf.R, e->lastR);
    float g[3];
    engine_global_t(e, g);
    double tn = std::sqrt((double)(g[0] - e->lastT[0]) * (g[0] - e->lastT[0]) +
                          (double)(g[1] - e->lastT[1]) * (g[1] - e->lastT[1]) +
                          (double)(g[2] - e->lastT[2]) * (g[2] - e->lastT[2]));
    if ((float)((rn + tn) / 2) >= c.integration_threshold) {
      integrate();
      std::memcpy(e->lastR, e->xf.R, sizeof(e->lastR));
      engine_global_t(e, e->lastT);
    }
    engine_raycast(e);
  }
  if (photometric) std::memcpy(e->cprev.data(), col, 4 * N);  // the next frame's model colours
  e->frames += 1;
  return 0;
}

// A frame at a given camera pose: UpdateVertexBuffers, UpdateCameraTransform(R, t),
// integrateVolume and raycastRender of the configured scene, without tracking (the
// step-wise path of a caller that sets the pose itself).
ORC_API void orc_engine_integrate_at(OrcEngine* e, const uint16_t* raw, const uint8_t* bgra, const float* R,
                                     const float* t) {
  const OrcEngineCfg& c = e->c;
  orc_pass_filter(raw, (long)c.W * c.H, c.dmin, c.dmax, e->depth.data());
  orc_make_xform(R, t, &e->xf);
  engine_integrate(e, c.color ? bgra : nullptr);
  engine_raycast(e);
}

ORC_API void orc_engine_pose(const OrcEngine* e, float* R, float* t) {
  std::memcpy(R, e->xf.R, 9 * sizeof(float));
  std::memcpy(t, e->xf.t, 3 * sizeof(float));
}
ORC_API const int16_t* orc_engine_volume(const OrcEngine* e) { return e->vol.data(); }
ORC_API void orc_engine_shift_state(const OrcEngine* e, int* voff) { std::memcpy(voff, e->voff, sizeof(e->voff)); }
// Points of the slabs that left the shifting volume: copies up to cap, returns how many
// were found in all (more than cap were found when the cache overflowed).
ORC_API long orc_engine_points(const OrcEngine* e, float* xyz, float* rgba, long cap) {
  const long n = std::min(cap, (long)(e->pts_xyz.size() / 3));
  std::memcpy(xyz, e->pts_xyz.data(), sizeof(float) * 3 * n);
  std::memcpy(rgba, e->pts_rgba.data(), sizeof(float) * 4 * n);
  return e->pts_n;
}
ORC_API OrcHash* orc_engine_hash(const OrcEngine* e) { return e->hs; }
ORC_API const uint8_t* orc_engine_color_volume(const OrcEngine* e) {
  return e->cvol.empty() ? nullptr : e->cvol.data();
}
ORC_API const float* orc_engine_refmap(const OrcEngine* e, int which) {
  return which == 0 ? e->vref.data() : e->nref.data();
}
ORC_API void orc_engine_tsdf_params(const OrcEngine* e, OrcTsdf* out) { *out = e->tp; }
ORC_API void orc_engine_icp_stats(const OrcEngine* e, OrcIcpStats* out) { *out = e->last; }
ORC_API long orc_engine_touched(const OrcEngine* e) { return e->touched; }

// =================================================================================
// Voxel-block hashing (KinfuHashScene.cl, KinfuHashRaycast.cl, KinfuHashVisualization.cl,
// host NuiKinfuOpenCLHashScene.cpp / NuiKinfuVoxelBlockHash.cpp), with runtime table sizes.
// Races of the reference are given deterministic intended semantics:
//  * new blocks colliding in one bucket (or chain end) in one frame: the block coordinate
//    written last in pixel-raster / ray-step order wins (what the kernel gives when its
//    work-items run one after another, KinfuHashScene.cl:127-130);
//  * free blocks and excess slots are popped in increasing entry index
//    (KinfuHashScene.cl:138-194 run sequentially);
//  * the visible list is the increasing list of entries with visible type > 0
//    (intended meaning of compactifyValidPrefixSum_kernel, prefixSum.cl:222-232) over all
//    entries (the reference's scan covers only the first 2^20, NuiOpenCLPrefixSum.cpp:16-41);
//  * every voxel of the pool starts at (sdf 0, weight 0, colour 0) (reset_voxel_block_kernel,
//    KinfuHashScene.cl:5-20, clears only the first 2^20+511 voxels);
//  * the expected-range image is updated with atomic min / max
//    (project_minmax_depths_kernel, KinfuHashRaycast.cl:67-75, is a plain read-modify-write);
//    its `zRange.y = fmax(zRange.x, z)` (:49) is kept as written;
//  * castRay reads the voxel before checking the block index (KinfuHashRaycast.cl:193-195):
//    a missing block reads as sdf 1.
namespace {
struct HEntry {
  int16_t pos[3];
  int16_t pad;
  int32_t ptr;
  uint32_t offset;
};
}  // namespace

struct OrcHashCfg {
  int buckets, excess, pool;  // bucket count, excess list length, voxel blocks in the pool
  uint32_t mask;              // hash mask (buckets - 1 for power-of-two tables)
  float voxel, mu;            // virtualVoxelSize, truncScale
  int max_w;                  // integrationWeightMax
  int swapping;               // NuiHashingSDFConfig::m_bUseSwapping: the global cache
};

// A voxel block kept by the global cache (NuiKinfuOpenCLHashGlobalCache m_storedVoxelBlocks).
struct OrcStoredBlock {
  int16_t sdf[512];
  uint8_t w[512], rgb[512 * 3];
};

struct OrcHash {
  OrcHashCfg c;
  std::vector<uint8_t> swap;                     // per entry swap state (0, 1, 2)
  std::unordered_map<int, OrcStoredBlock> store;  // host copies by entry
  std::vector<HEntry> e;
  std::vector<int16_t> sdf;
  std::vector<uint8_t> w, rgb;
  std::vector<int> alloc_list, excess_list;
  int last_block, last_excess;
  std::vector<uint8_t> alloc_type, vis;
  std::vector<int16_t> coords;
  std::vector<int> vis_ids;
  std::vector<float> range;  // expected range image (2 floats per pixel)
  long failed_allocs = 0;
};

ORC_API void orc_hash_reset(OrcHash* h) {
  const long ne = (long)h->c.buckets + h->c.excess;
  for (long i = 0; i < ne; ++i) h->e[i] = HEntry{{0, 0, 0}, 0, -2, 0};
  std::fill(h->sdf.begin(), h->sdf.end(), 0);
  std::fill(h->w.begin(), h->w.end(), 0);
  std::fill(h->rgb.begin(), h->rgb.end(), 0);
  for (int i = 0; i < h->c.pool; ++i) h->alloc_list[i] = i;
  for (int i = 0; i < h->c.excess; ++i) h->excess_list[i] = i;
  h->last_block = h->c.pool - 1;
  h->last_excess = h->c.excess - 1;
  std::fill(h->alloc_type.begin(), h->alloc_type.end(), 0);
  std::fill(h->vis.begin(), h->vis.end(), 0);
  h->vis_ids.clear();
  h->failed_allocs = 0;
  std::fill(h->swap.begin(), h->swap.end(), 0);  // NuiKinfuOpenCLHashGlobalCache::reset
  h->store.clear();
}

ORC_API OrcHash* orc_hash_create(const OrcHashCfg* cfg) {
  OrcHash* h = new OrcHash();
  h->c = *cfg;
  const long ne = (long)cfg->buckets + cfg->excess;
  h->e.resize(ne);
  h->sdf.resize((size_t)cfg->pool * 512);
  h->w.resize((size_t)cfg->pool * 512);
  h->rgb.resize((size_t)cfg->pool * 512 * 3);
  h->alloc_list.resize(cfg->pool);
  h->excess_list.resize(cfg->excess);
  h->alloc_type.resize(ne);
  h->vis.resize(ne);
  h->coords.resize(3 * ne);
  h->swap.resize(ne);
  orc_hash_reset(h);
  return h;
}
ORC_API void orc_hash_destroy(OrcHash* h) { delete h; }

static inline uint32_t hash_index(const OrcHashCfg& c, int x, int y, int z) {
  return (((uint32_t)x * 73856093u) ^ ((uint32_t)y * 19349669u) ^ ((uint32_t)z * 83492791u)) & c.mask;
}

// Block-pool voxel index of virtual voxel v (findVoxelBlockIndex, KinfuHashRaycast.cl:78-111);
// -1 when its block is not allocated.
static long hash_find(const OrcHash* h, int vx, int vy, int vz) {
  int bx = vx < 0 ? vx - 7 : vx, by = vy < 0 ? vy - 7 : vy, bz = vz < 0 ? vz - 7 : vz;
  bx /= 8;
  by /= 8;
  bz /= 8;
  const int lin = (vx - 8 * bx) + 8 * (vy - 8 * by) + 64 * (vz - 8 * bz);
  const int16_t sx = (int16_t)bx, sy = (int16_t)by, sz = (int16_t)bz;
  uint32_t hi = hash_index(h->c, sx, sy, sz);
  for (;;) {
    const HEntry& en = h->e[hi];
    if (en.pos[0] == sx && en.pos[1] == sy && en.pos[2] == sz && en.ptr >= 0) return (long)en.ptr * 512 + lin;
    if (en.offset < 1) break;
    hi = (uint32_t)h->c.buckets + en.offset - 1;
  }
  return -1;
}

static inline f3 xf_apply(const OrcXform* m, f3 v) {
  return mk(dot3(mk(m->R[0], m->R[1], m->R[2]), v), dot3(mk(m->R[3], m->R[4], m->R[5]), v),
            dot3(mk(m->R[6], m->R[7], m->R[8]), v)) + mk(m->t[0], m->t[1], m->t[2]);
}
static inline f3 xf_inverse(const OrcXform* m, f3 v) {
  v = v - mk(m->t[0], m->t[1], m->t[2]);
  return mk(dot3(mk(m->R_inv[0], m->R_inv[1], m->R_inv[2]), v), dot3(mk(m->R_inv[3], m->R_inv[4], m->R_inv[5]), v),
            dot3(mk(m->R_inv[6], m->R_inv[7], m->R_inv[8]), v));
}
// kinectDepthToSkeleton (cameraUtils.cl:46-53)
static inline f3 depth_to_point(const OrcCam* cam, int ux, int uy, float d) {
  const float x = ((float)ux - cam->cx) / cam->fx, y = ((float)uy - cam->cy) / cam->fy;
  return mk(d * x, d * y, d);
}

// A16: ResetVisibleEntrys + ResetAllocType + buildHashAllocAndVisibleType +
// allocateVoxelBlocksList + buildVisibleList + compaction (AllocateSceneFromDepth,
// NuiKinfuOpenCLHashScene.cpp:404-424).  depth: pass-filtered z-depth (NaN invalid).
ORC_API long orc_hash_allocate(OrcHash* h, const float* depth, const OrcCam* cam, const OrcXform* m) {
  const OrcHashCfg& c = h->c;
  const long ne = (long)c.buckets + c.excess;
  for (int id : h->vis_ids) h->vis[id] = 3;
  std::fill(h->alloc_type.begin(), h->alloc_type.end(), 0);
  const float obs = 1.0f / (c.voxel * 8);
  const int W = (int)cam->W, H = (int)cam->H;
  for (int py = 0; py < H; ++py)
    for (int px = 0; px < W; ++px) {
      const float Dp = depth[(long)py * W + px];
      if (std::isnan(Dp)) continue;
      const f3 pc = depth_to_point(cam, px, py, Dp);
      const float norm = c.mu / length3(pc);
      f3 rmin = xf_apply(m, pc * (1.0f - norm)) * obs;
      const f3 rmax = xf_apply(m, pc * (1.0f + norm)) * obs;
      f3 rdir = rmax - rmin;
      const float rn = length3(rdir);
      const int steps = (int)std::ceil(2.0f * rn);
      const float dv = (float)(steps - 1);
      rdir = mk(rdir.x / dv, rdir.y / dv, rdir.z / dv);
      for (int i = 0; i < steps; ++i) {
        const int16_t bx = (int16_t)std::floor(rmin.x), by = (int16_t)std::floor(rmin.y), bz = (int16_t)std::floor(rmin.z);
        uint32_t hi = hash_index(c, bx, by, bz);
        HEntry en = h->e[hi];
        bool found = false;
        if (en.pos[0] == bx && en.pos[1] == by && en.pos[2] == bz && en.ptr >= -1) {
          h->vis[hi] = (en.ptr == -1) ? 2 : 1;
          found = true;
        }
        if (!found) {
          bool excess = false;
          if (en.ptr >= -1) {
            while (en.offset >= 1) {
              hi = (uint32_t)c.buckets + en.offset - 1;
              en = h->e[hi];
              if (en.pos[0] == bx && en.pos[1] == by && en.pos[2] == bz && en.ptr >= -1) {
                h->vis[hi] = (en.ptr == -1) ? 2 : 1;
                found = true;
                break;
              }
            }
            excess = true;
          }
          if (!found) {
            h->alloc_type[hi] = excess ? 2 : 1;
            h->vis[hi] = 1;
            h->coords[3 * hi] = bx;
            h->coords[3 * hi + 1] = by;
            h->coords[3 * hi + 2] = bz;
          }
        }
        rmin = rmin + rdir;
      }
    }
  for (long i = 0; i < ne; ++i) {
    const int t = h->alloc_type[i];
    if (t == 1) {
      const int vba = h->last_block--;
      if (vba >= 0) {
        HEntry en{{h->coords[3 * i], h->coords[3 * i + 1], h->coords[3 * i + 2]}, 0, h->alloc_list[vba], 0};
        h->e[i] = en;
      } else {
        ++h->failed_allocs;
      }
    } else if (t == 2) {
      const int vba = h->last_block--;
      const int exl = h->last_excess--;
      if (vba >= 0 && exl >= 0) {
        HEntry en{{h->coords[3 * i], h->coords[3 * i + 1], h->coords[3 * i + 2]}, 0, h->alloc_list[vba], 0};
        const int off = h->excess_list[exl];
        h->e[i].offset = (uint32_t)off + 1;
        h->e[(long)c.buckets + off] = en;
        h->vis[(long)c.buckets + off] = 1;
      } else {
        ++h->failed_allocs;
      }
    }
  }
  // buildVisibleList_kernel (KinfuHashScene.cl:262-285) with checkBlockVisibility (:196-260)
  const float factor = 8.0f * c.voxel;
  auto point_visible = [&](f3 p) {
    const f3 q = xf_inverse(m, p);
    if (isnan3(q)) return false;
    const int sx = (int)(q.x * cam->fx / q.z + cam->cx + 0.5f), sy = (int)(q.y * cam->fy / q.z + cam->cy + 0.5f);
    return sx >= 0 && sx < (int)cam->W && sy >= 0 && sy < (int)cam->H;
  };
  if (c.swapping) {
    // buildVisibleEnlargedList_kernel (KinfuHashScene.cl:358-385).  Its bounds are
    // lims = (-W/8, W + W/8, -H/8, H + H/8) as unsigned numbers (:306-311): the lower bound
    // wraps above the upper one, so checkBlockVisibilityEnlarged never passes and an entry
    // seen only at the previous frame drops out.  Every entry visible at the start of the
    // kernel, unless already merged (state 2), is marked for swap-in.
    const uint32_t lx = (uint32_t)(-(int64_t)cam->W) / 8u, ux = cam->W + cam->W / 8u;
    for (long i = 0; i < ne; ++i) {
      const uint8_t t = h->vis[i];
      if (t == 3 && !(lx < ux)) h->vis[i] = 0;
      if (t > 0 && h->swap[i] != 2) h->swap[i] = 1;
    }
  }
  for (long i = 0; i < ne && !c.swapping; ++i) {
    if (h->vis[i] != 3) continue;
    const HEntry& en = h->e[i];
    f3 p = mk((float)en.pos[0] * factor, (float)en.pos[1] * factor, (float)en.pos[2] * factor);
    bool v = point_visible(p);
    if (!v) { p.z += factor; v = point_visible(p); }
    if (!v) { p.y += factor; v = point_visible(p); }
    if (!v) { p.x += factor; v = point_visible(p); }
    if (!v) { p.z -= factor; v = point_visible(p); }
    if (!v) { p.y -= factor; v = point_visible(p); }
    if (!v) { p.x -= factor; p.y += factor; v = point_visible(p); }
    if (!v) { p.x += factor; p.y -= factor; p.z += factor; v = point_visible(p); }
    if (!v) h->vis[i] = 0;
  }
  h->vis_ids.clear();
  for (long i = 0; i < ne; ++i)
    if (h->vis[i] > 0) h->vis_ids.push_back((int)i);
  if (c.swapping) {
    // reAllocateSwappedOutVoxelBlocks_kernel (KinfuHashSwapping.cl:6-22): a visible entry
    // whose block was swapped out takes a free block, the pops in index order
    for (long i = 0; i < ne; ++i)
      if (h->vis[i] > 0 && h->e[i].ptr == -1) {
        const int vba = h->last_block--;
        if (vba >= 0) h->e[i].ptr = h->alloc_list[vba];
      }
  }
  return (long)h->vis_ids.size();
}

// NuiKinfuOpenCLHashGlobalCache::integrateGlobalIntoLocal + saveToGlobalMemory
// (NuiKinfuOpenCLHashGlobalCache.cpp:192-538), after the integration.  Lists are the
// flagged entries in index order (the prefix sums' intended meaning), at most
// SDF_TRANSFER_BLOCK_NUM = 4096 per operation.
ORC_API void orc_hash_swap(OrcHash* h) {
  const OrcHashCfg& c = h->c;
  const long ne = (long)c.buckets + c.excess;
  const int kTransfer = 4096;
  // swap-in: entries marked 1 merge their stored copy (zeros if none) into the local block
  // (integrateOldIntoActiveData_kernel, KinfuHashSwapping.cl:62-111)
  std::vector<int> need;
  for (long i = 0; i < ne && (int)need.size() < kTransfer; ++i)
    if (h->swap[i] == 1) need.push_back((int)i);
  static const OrcStoredBlock zero{};
  for (int id : need) {
    const int ptr = h->e[id].ptr;
    if (ptr < 0) continue;
    auto it = h->store.find(id);
    const OrcStoredBlock& sb = it != h->store.end() ? it->second : zero;
    for (int lid = 0; lid < 512; ++lid) {
      const long bi = (long)ptr * 512 + lid;
      const float oldF = (float)sb.sdf[lid] / 32767.0f, oldW = (float)sb.w[lid];
      float newF = (float)h->sdf[bi] / 32767.0f;
      const float newW = (float)h->w[bi], cw = oldW + newW;
      newF = oldW * oldF + newW * newF;
      newF /= cw;
      // both weights 0: 0 / 0; the conversions of the NaN give 0 (x86 and CUDA alike)
      h->sdf[bi] = std::isnan(newF) ? (int16_t)0 : (int16_t)(int)(newF * 32767.0f);
      h->w[bi] = (uint8_t)std::min((int)(uint8_t)(int)cw, c.max_w);
      for (int k = 0; k < 3; ++k) {
        const float v = (oldW * (float)sb.rgb[3 * lid + k] + newW * (float)h->rgb[3 * bi + k]) / cw;
        h->rgb[3 * bi + k] = std::isnan(v) ? (uint8_t)0 : (uint8_t)(int)std::min(std::max(v, 0.0f), 255.f);
      }
    }
    h->swap[id] = 2;
  }
  // swap-out: merged entries (2) that are not visible leave for the host; their blocks are
  // cleared and pushed back on the free list (buildSwapOutList_kernel,
  // moveActiveDataToTransferBuffer_kernel, cleanVoxelMemory_kernel, :113-180).  Block 0 is
  // never swapped out (the kernel tests ptr > 0).
  std::vector<int> out;
  for (long i = 0; i < ne && (int)out.size() < kTransfer; ++i)
    if (h->swap[i] == 2 && h->e[i].ptr > 0 && h->vis[i] == 0) out.push_back((int)i);
  for (int id : out) {
    const int ptr = h->e[id].ptr;
    OrcStoredBlock& sb = h->store[id];
    for (int lid = 0; lid < 512; ++lid) {
      const long bi = (long)ptr * 512 + lid;
      sb.sdf[lid] = h->sdf[bi];
      sb.w[lid] = h->w[bi];
      std::memcpy(&sb.rgb[3 * lid], &h->rgb[3 * bi], 3);
      h->sdf[bi] = 0;
      h->w[bi] = 0;
      std::memset(&h->rgb[3 * bi], 0, 3);
    }
  }
  for (int id : out) {
    h->swap[id] = 0;
    const int vba = h->last_block++ ;
    if (vba < c.pool - 1) {
      h->alloc_list[vba + 1] = h->e[id].ptr;
      h->e[id].ptr = -1;
    }
  }
}

ORC_API const uint8_t* orc_hash_swap_states(const OrcHash* h) { return h->swap.data(); }
// The stored copy of entry id: copies it out and returns 1, or returns 0 if there is none.
ORC_API int orc_hash_stored(const OrcHash* h, int id, int16_t* sdf, uint8_t* w, uint8_t* rgb) {
  auto it = h->store.find(id);
  if (it == h->store.end()) return 0;
  std::memcpy(sdf, it->second.sdf, sizeof(it->second.sdf));
  std::memcpy(w, it->second.w, sizeof(it->second.w));
  std::memcpy(rgb, it->second.rgb, sizeof(it->second.rgb));
  return 1;
}
ORC_API long orc_hash_stored_count(const OrcHash* h) { return (long)h->store.size(); }
// Entries with a stored copy, in increasing order; returns how many (up to cap written).
ORC_API long orc_hash_stored_ids(const OrcHash* h, int* ids, long cap) {
  std::vector<int> v;
  for (const auto& kv : h->store) v.push_back(kv.first);
  std::sort(v.begin(), v.end());
  for (long i = 0; i < (long)v.size() && i < cap; ++i) ids[i] = v[i];
  return (long)v.size();
}

// A17: integrateIntoScene_kernel (KinfuHashScene.cl:387-470) over the visible list.
ORC_API void orc_hash_integrate(OrcHash* h, const float* depth, const uint8_t* bgra, const OrcCam* cam,
                                const OrcXform* m, long* touched) {
  const OrcHashCfg& c = h->c;
  long cnt = 0;
  const long nvis = (long)h->vis_ids.size();
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : cnt)
  for (long k = 0; k < nvis; ++k) {
    const HEntry en = h->e[h->vis_ids[k]];
    if (en.ptr < 0) continue;
    for (int lid = 0; lid < 512; ++lid) {
      const long bid = (long)en.ptr * 512 + lid;
      if (c.max_w == h->w[bid]) continue;
      const int lx = (lid % 64) % 8, ly = (lid % 64) / 8, lz = lid / 64;
      const f3 pm = mk((float)(en.pos[0] * 8 + lx), (float)(en.pos[1] * 8 + ly), (float)(en.pos[2] * 8 + lz)) * c.voxel;
      const f3 pc = xf_inverse(m, pm);
      if (pc.z <= 0) continue;
      const int ix = (int)(pc.x * cam->fx / pc.z + cam->cx + 0.5f), iy = (int)(pc.y * cam->fy / pc.z + cam->cy + 0.5f);
      if (ix < 0 || ix >= (int)cam->W || iy < 0 || iy >= (int)cam->H) continue;
      const long sid = (long)iy * cam->W + ix;
      const float d = depth[sid];
      if (std::isnan(d)) continue;
      const float eta = d - pc.z;
      const float sdf = eta / c.mu;
      if (eta < -c.mu) continue;
      const float oldF = (float)h->sdf[bid] / 32767.0f, oldW = (float)h->w[bid];
      float newF = std::min(1.0f, sdf);
      const float newW = 1.0f, cw = oldW + newW;
      if (bgra && eta < c.mu && std::fabs(sdf) < 0.25f) {
        const uint8_t* col = bgra + 4 * sid;
        if (col[3] == 255) {
          uint8_t* vc = &h->rgb[3 * bid];
          const float r = (oldW * (float)vc[0] + newW * (float)col[2]) / cw;
          const float g = (oldW * (float)vc[1] + newW * (float)col[1]) / cw;
          const float b = (oldW * (float)vc[2] + newW * (float)col[0]) / cw;
          vc[0] = (uint8_t)std::min(std::max(r, 0.f), 255.f);
          vc[1] = (uint8_t)std::min(std::max(g, 0.f), 255.f);
          vc[2] = (uint8_t)std::min(std::max(b, 0.f), 255.f);
        }
      }
      newF = oldW * oldF + newW * newF;
      newF /= cw;
      h->sdf[bid] = (int16_t)(newF * 32767.0f);
      h->w[bid] = (uint8_t)std::min((int)(uint8_t)cw, c.max_w);
      ++cnt;
    }
  }
  if (touched) *touched = cnt;
}

// A18: CreateExpectedDepths (project_minmax_depths_kernel) + castRay, the plain raycast
// path of NuiKinfuOpenCLHashScene::raycastRender (forward rendering off).  Outputs world
// vertex / normal maps (3 floats per pixel), colour (4 bytes, nullable) and the range image.
static float hash_read_sdf(const OrcHash* h, int x, int y, int z) {
  const long bi = hash_find(h, x, y, z);
  return bi < 0 ? 1.0f : (float)h->sdf[bi] / 32767.0f;
}

// CreateExpectedDepths (project_minmax_depths_kernel, KinfuHashRaycast.cl:4-76) over the
// visible list: per pixel (min, max) camera depth of the visible blocks that cover it.
static void hash_expected_range(const OrcHash* h, const OrcCam* cam, const OrcXform* m, std::vector<float>& rg) {
  const OrcHashCfg& c = h->c;
  const int W = (int)cam->W, H = (int)cam->H;
  const long N = (long)W * H;
  rg.assign(2 * N, 0.f);
  for (long i = 0; i < N; ++i) {
    rg[2 * i] = 999999.9f;
    rg[2 * i + 1] = 0.05f;
  }
  for (int id : h->vis_ids) {
    const HEntry& en = h->e[id];
    if (en.ptr < 0) continue;
    int ulx = W, uly = H, lrx = 0, lry = 0;
    float zx = 999999.9f, zy = 0.05f;
    for (int corner = 0; corner < 8; ++corner) {
      const int cx = en.pos[0] + ((corner & 1) ? 1 : 0), cy = en.pos[1] + ((corner & 2) ? 1 : 0),
                cz = en.pos[2] + ((corner & 4) ? 1 : 0);
      f3 p = mk((float)(int16_t)cx, (float)(int16_t)cy, (float)(int16_t)cz) * 8.0f * c.voxel;
      p = xf_inverse(m, p);
      if (isnan3(p) || p.z < 1e-6) continue;
      const float u = p.x * cam->fx / p.z + cam->cx, v = p.y * cam->fy / p.z + cam->cy;
      ulx = std::min(ulx, (int)std::floor(u));
      lrx = std::max(lrx, (int)std::ceil(u));
      uly = std::min(uly, (int)std::floor(v));
      lry = std::max(lry, (int)std::ceil(v));
      zx = std::fmin(zx, p.z);
      zy = std::fmax(zx, p.z);
    }
    if (ulx < 0) ulx = 0;
    if (uly < 0) uly = 0;
    if (lrx >= W) lrx = W - 1;
    if (lry >= H) lry = H - 1;
    if (zx < 0.05f) zx = 0.05f;
    for (int by = uly; by <= lry; ++by)
      for (int bx = ulx; bx <= lrx; ++bx) {
        const long li = (long)by * W + bx;
        rg[2 * li] = std::fmin(rg[2 * li], zx);
        rg[2 * li + 1] = std::fmax(rg[2 * li + 1], zy);
      }
  }
}

// castRay (KinfuHashRaycast.cl:155-452) of pixel (px, py) over its expected range: writes the
// world vertex (and, when nmap is given, the normal) and the colour of the pixel.
static void hash_cast_ray(const OrcHash* h, const OrcCam* cam, const OrcXform* m, const float* rg, int px, int py,
                          float* vmap, float* nmap, uint8_t* cmap) {
  const OrcHashCfg& c = h->c;
  const int W = (int)cam->W;
  const float oov = 1.0f / c.voxel;
  const float stepScale = c.mu * oov * 0.6f;
  {
    {
      const long pid = (long)py * W + px;
      f3 ps = depth_to_point(cam, px, py, rg[2 * pid]);
      float total = length3(ps) * oov;
      ps = xf_apply(m, ps) * oov;
      f3 pe = depth_to_point(cam, px, py, rg[2 * pid + 1]);
      const float totalMax = length3(pe) * oov;
      pe = xf_apply(m, pe) * oov;
      float sdfv = 1.0f, stepLen;
      const f3 dir = normalize3(pe - ps);
      f3 pr = ps;
      while (total < totalMax) {
        const int vx = (int)std::round(pr.x), vy = (int)std::round(pr.y), vz = (int)std::round(pr.z);
        const long bi = hash_find(h, vx, vy, vz);
        if (bi < 0) {
          sdfv = 1.0f;
          stepLen = 8.0f;
        } else {
          sdfv = (float)h->sdf[bi] / 32767.0f;
          if (sdfv <= 0.1f && sdfv >= -0.5f) {
            // readInterpolatedVoxelSDF (KinfuHashRaycast.cl:124-153)
            const int ix = (int)std::floor(pr.x), iy = (int)std::floor(pr.y), iz = (int)std::floor(pr.z);
            const f3 cf = mk(pr.x - (float)ix, pr.y - (float)iy, pr.z - (float)iz);
            float v1 = hash_read_sdf(h, ix, iy, iz), v2 = hash_read_sdf(h, ix + 1, iy, iz);
            float r1 = (1.0f - cf.x) * v1 + cf.x * v2;
            v1 = hash_read_sdf(h, ix, iy + 1, iz);
            v2 = hash_read_sdf(h, ix + 1, iy + 1, iz);
            r1 = (1.0f - cf.y) * r1 + cf.y * ((1.0f - cf.x) * v1 + cf.x * v2);
            v1 = hash_read_sdf(h, ix, iy, iz + 1);
            v2 = hash_read_sdf(h, ix + 1, iy, iz + 1);
            float r2 = (1.0f - cf.x) * v1 + cf.x * v2;
            v1 = hash_read_sdf(h, ix, iy + 1, iz + 1);
            v2 = hash_read_sdf(h, ix + 1, iy + 1, iz + 1);
            r2 = (1.0f - cf.y) * r2 + cf.y * ((1.0f - cf.x) * v1 + cf.x * v2);
            sdfv = (1.0f - cf.z) * r1 + cf.z * r2;
          }
          if (sdfv <= 0.0f) break;
          stepLen = std::max(sdfv * stepScale, 1.0f);
        }
        pr = pr + dir * stepLen;
        total += stepLen;
      }
      f3 vout = mk(QNAN, QNAN, QNAN), nout = mk(QNAN, QNAN, QNAN);
      uint8_t col[4] = {0, 0, 0, 0};
      if (sdfv <= 0.0f) {
        stepLen = sdfv * stepScale;
        pr = pr + dir * stepLen;
        const int ix = (int)std::floor(pr.x), iy = (int)std::floor(pr.y), iz = (int)std::floor(pr.z);
        const f3 cf = mk(pr.x - (float)ix, pr.y - (float)iy, pr.z - (float)iz);
        const f3 nc = mk(1.0f - cf.x, 1.0f - cf.y, 1.0f - cf.z);
        static const int O[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}, {0, 0, 1}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}};
        float fb[8];
        float nearest = 1.0e20f;
        for (int k = 0; k < 8; ++k) {
          const long bi = hash_find(h, ix + O[k][0], iy + O[k][1], iz + O[k][2]);
          fb[k] = bi < 0 ? 1.0f : (float)h->sdf[bi] / 32767.0f;
          const f3 dd = mk(O[k][0] ? nc.x : cf.x, O[k][1] ? nc.y : cf.y, O[k][2] ? nc.z : cf.z);
          const float cd = length3(dd);
          if (cmap && bi >= 0 && (k == 0 || nearest > cd)) {
            nearest = cd;
            col[0] = h->rgb[3 * bi];
            col[1] = h->rgb[3 * bi + 1];
            col[2] = h->rgb[3 * bi + 2];
            col[3] = 255;
          }
        }
        // front = k 0..3 (x, y), back = k 4..7
        sdfv = fb[0] * nc.x * nc.y * nc.z + fb[1] * cf.x * nc.y * nc.z + fb[2] * nc.x * cf.y * nc.z +
               fb[3] * cf.x * cf.y * nc.z + fb[4] * nc.x * nc.y * cf.z + fb[5] * cf.x * nc.y * cf.z +
               fb[6] * nc.x * cf.y * cf.z + fb[7] * cf.x * cf.y * cf.z;
        stepLen = sdfv * stepScale;
        pr = pr + dir * stepLen;
        vout = pr * c.voxel;
        if (nmap) {
          auto rs = [&](int a, int b, int cc) { return hash_read_sdf(h, ix + a, iy + b, iz + cc); };
          float p1, p2, v1;
          f3 g;
          p1 = fb[0] * nc.y * nc.z + fb[2] * cf.y * nc.z + fb[4] * nc.y * cf.z + fb[6] * cf.y * cf.z;
          p2 = rs(-1, 0, 0) * nc.y * nc.z + rs(-1, 1, 0) * cf.y * nc.z + rs(-1, 0, 1) * nc.y * cf.z +
               rs(-1, 1, 1) * cf.y * cf.z;
          v1 = p1 * cf.x + p2 * nc.x;
          p1 = fb[1] * nc.y * nc.z + fb[3] * cf.y * nc.z + fb[5] * nc.y * cf.z + fb[7] * cf.y * cf.z;
          p2 = rs(2, 0, 0) * nc.y * nc.z + rs(2, 1, 0) * cf.y * nc.z + rs(2, 0, 1) * nc.y * cf.z +
               rs(2, 1, 1) * cf.y * cf.z;
          g.x = p1 * nc.x + p2 * cf.x - v1;
          p1 = fb[0] * nc.x * nc.z + fb[1] * cf.x * nc.z + fb[4] * nc.x * cf.z + fb[5] * cf.x * cf.z;
          p2 = rs(0, -1, 0) * nc.x * nc.z + rs(1, -1, 0) * cf.x * nc.z + rs(0, -1, 1) * nc.x * cf.z +
               rs(1, -1, 1) * cf.x * cf.z;
          v1 = p1 * cf.y + p2 * nc.y;
          p1 = fb[2] * nc.x * nc.z + fb[3] * cf.x * nc.z + fb[6] * nc.x * cf.z + fb[7] * cf.x * cf.z;
          p2 = rs(0, 2, 0) * nc.x * nc.z + rs(1, 2, 0) * cf.x * nc.z + rs(0, 2, 1) * nc.x * cf.z +
               rs(1, 2, 1) * cf.x * cf.z;
          g.y = p1 * nc.y + p2 * cf.y - v1;
          p1 = fb[0] * nc.x * nc.y + fb[1] * cf.x * nc.y + fb[2] * nc.x * cf.y + fb[3] * cf.x * cf.y;
          p2 = rs(0, 0, -1) * nc.x * nc.y + rs(1, 0, -1) * cf.x * nc.y + rs(0, 1, -1) * nc.x * cf.y +
               rs(1, 1, -1) * cf.x * cf.y;
          v1 = p1 * cf.z + p2 * nc.z;
          p1 = fb[4] * nc.x * nc.y + fb[5] * cf.x * nc.y + fb[6] * nc.x * cf.y + fb[7] * cf.x * cf.y;
          p2 = rs(0, 0, 2) * nc.x * nc.y + rs(1, 0, 2) * cf.x * nc.y + rs(0, 1, 2) * nc.x * cf.y +
               rs(1, 1, 2) * cf.x * cf.y;
          g.z = p1 * nc.z + p2 * cf.z - v1;
          nout = normalize3(g);
        }
      }
      st3(vmap, pid, vout);
      if (nmap) st3(nmap, pid, nout);
      if (cmap) std::memcpy(cmap + 4 * pid, col, 4);
    }
  }
}

// A18, forward rendering off (NuiKinfuOpenCLHashScene::Raycast, :659-736): every pixel.
ORC_API void orc_hash_raycast(OrcHash* h, const OrcCam* cam, const OrcXform* m, float* vmap, float* nmap,
                              uint8_t* cmap, float* range_out) {
  const int W = (int)cam->W, H = (int)cam->H;
  std::vector<float> rg;
  hash_expected_range(h, cam, m, rg);
  if (range_out) std::memcpy(range_out, rg.data(), sizeof(float) * 2 * (size_t)W * H);
#pragma omp parallel for schedule(dynamic, 4)
  for (int py = 0; py < H; ++py)
    for (int px = 0; px < W; ++px) hash_cast_ray(h, cam, m, rg.data(), px, py, vmap, nmap, cmap);
}

// A18 with forward rendering on, the reference's default for the hash scene
// (NuiSLAMController.cpp:47; NuiKinfuOpenCLHashScene::ForwardRender, :991-1012):
//  1. forwardProject_kernel (KinfuHashRaycast.cl:473-506): every valid vertex p of the
//     previous maps goes to pixel trunc(screen(transform(p) * voxel) + 0.5) -- transform is
//     the camera-to-world transform of the current pose, applied here to a world point, as
//     the reference writes it -- when that lies inside the image (a value in (-1, 0) truncates
//     to 0, as the reference's float-to-uint conversion does); it carries its vertex and
//     colour there.  Several vertices may land on one pixel: the last in raster order wins
//     (the reference's unordered stores; its in-place colour copy is read from the previous
//     colours here);
//  2. findMissingPoints_kernel (:508-528): a pixel is missing when nothing landed on it and
//     its expected range is not empty; other pixels take what landed (NaN if nothing);
//  3. genericRaycastMissingPoints_kernel (:530-559): castRay without normals for every
//     missing pixel, which a prefix-sum compaction lists in increasing order (the
//     reference's compaction sizes its scan down to a power of two and loses the first
//     index; every missing pixel is cast here);
//  4. Vertex2Normal (:940-983): estimate_normals_simple_kernel over the new vertices, depth
//     threshold 0.3 m.
// vprev / cprev: the previous world vertex map (3 floats a pixel) and colours (nullable);
// missing_out (nullable): 1 for the pixels that were cast.  Returns the missing count.
ORC_API long orc_hash_forward_render(OrcHash* h, const OrcCam* cam, const OrcXform* m, const float* vprev,
                                     const uint8_t* cprev, float* vmap, float* nmap, uint8_t* cmap, float* range_out,
                                     uint8_t* missing_out, int mode) {
  const OrcHashCfg& c = h->c;
  const int W = (int)cam->W, H = (int)cam->H;
  const long N = (long)W * H;
  std::vector<float> rg;
  hash_expected_range(h, cam, m, rg);
  if (range_out) std::memcpy(range_out, rg.data(), sizeof(float) * 2 * N);
  std::vector<long> owner(N, -1);
  for (long i = 0; i < N; ++i) {
    const f3 p = ld3(vprev, i);
    if (isnan3(p)) continue;
    // mode 1: the reference's expression; mode 2: the world point taken into the camera
    const f3 q = mode == 2 ? xf_inverse(m, p) : xf_apply(m, p) * c.voxel;
    const float u = q.x * cam->fx / q.z + cam->cx + 0.5f, v = q.y * cam->fy / q.z + cam->cy + 0.5f;
    if (!(u > -1.0f && v > -1.0f)) continue;
    const float tu = std::trunc(u), tv = std::trunc(v);
    if (!(tu < (float)W && tv < (float)H)) continue;
    owner[(long)tv * W + (long)tu] = i;
  }
  std::vector<uint8_t> missing(N, 0);
  long nmiss = 0;
  for (long t = 0; t < N; ++t) {
    const long o = owner[t];
    const bool empty_range = !(rg[2 * t] < rg[2 * t + 1]);
    if (o < 0 && !empty_range) {
      missing[t] = 1;
      ++nmiss;
      continue;
    }
    st3(vmap, t, o >= 0 ? ld3(vprev, o) : mk(QNAN, QNAN, QNAN));
    if (cmap) {
      if (o >= 0 && cprev) std::memcpy(cmap + 4 * t, cprev + 4 * o, 4);
      else std::memset(cmap + 4 * t, 0, 4);
    }
  }
#pragma omp parallel for schedule(dynamic, 4)
  for (int py = 0; py < H; ++py)
    for (int px = 0; px < W; ++px)
      if (missing[(long)py * W + px]) hash_cast_ray(h, cam, m, rg.data(), px, py, vmap, nullptr, cmap);
  orc_normals(vmap, W, H, 0.3f, nmap);
  if (missing_out) std::memcpy(missing_out, missing.data(), N);
  return nmiss;
}

// A19: meshHashScene_kernel (KinfuHashVisualization.cl:88-271) over the visible list, in
// visible-list order, voxels z-y-x within a block, triangles in table order.  Returns the
// vertex count (uncapped); positions / colours written up to cap vertices.
static inline f3 sdf_interp(f3 p1, f3 p2, float v1, float v2) {
  if (std::fabs(0.0f - v1) < 0.00001f) return p1;
  if (std::fabs(0.0f - v2) < 0.00001f) return p2;
  if (std::fabs(v1 - v2) < 0.00001f) return p1;
  return p1 + (p2 - p1) * ((0.0f - v1) / (v2 - v1));
}

// fetchHashScene_kernel (KinfuHashVisualization.cl:5-52) over the visible list, as
// NuiKinfuOpenCLHashScene::Volume2CLVertices launches it (NuiKinfuOpenCLHashScene.cpp:1066-1180):
// a point at the centre of every weighted voxel with |sdf| < 32767 * truncScale, in visible
// list and voxel order, with the voxel's colour / 255 (alpha 1).  Up to cap points; returns
// how many were found.
ORC_API long orc_hash_fetch_points(const OrcHash* h, float* xyz, float* rgba, long cap) {
  long out = 0;
  for (int id : h->vis_ids) {
    const HEntry& en = h->e[id];
    if (en.ptr < 0) continue;
    for (int i = 0; i < 512; ++i) {
      const long bi = (long)en.ptr * 512 + i;
      if (!(h->w[bi] > 0 && (float)std::abs((int)h->sdf[bi]) < 32767.f * h->c.mu)) continue;
      if (out < cap) {
        xyz[3 * out + 2] = ((float)(en.pos[2] * 8) + ((float)(i / 64) + 0.5f)) * h->c.voxel;
        xyz[3 * out + 1] = ((float)(en.pos[1] * 8) + ((float)((i % 64) / 8) + 0.5f)) * h->c.voxel;
        xyz[3 * out + 0] = ((float)(en.pos[0] * 8) + ((float)((i % 64) % 8) + 0.5f)) * h->c.voxel;
        rgba[4 * out + 0] = (float)h->rgb[3 * bi] / 255.f;
        rgba[4 * out + 1] = (float)h->rgb[3 * bi + 1] / 255.f;
        rgba[4 * out + 2] = (float)h->rgb[3 * bi + 2] / 255.f;
        rgba[4 * out + 3] = 1.0f;
      }
      ++out;
    }
  }
  return out;
}

ORC_API long orc_hash_mesh(const OrcHash* h, float* pos, float* col, long cap) {
  static const int CO[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  static const int E[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  long out = 0;
  for (int id : h->vis_ids) {
    const HEntry& en = h->e[id];
    if (en.ptr < 0) continue;
    const int gx = en.pos[0] * 8, gy = en.pos[1] * 8, gz = en.pos[2] * 8;
    for (int z = 0; z < 8; ++z)
      for (int y = 0; y < 8; ++y)
        for (int x = 0; x < 8; ++x) {
          float sv[8];
          f3 pt[8], cl[8];
          bool ok = true;
          for (int k = 0; k < 8 && ok; ++k) {
            const int vx = gx + x + CO[k][0], vy = gy + y + CO[k][1], vz = gz + z + CO[k][2];
            const long bi = hash_find(h, vx, vy, vz);
            if (bi < 0) {
              ok = false;
              break;
            }
            sv[k] = (float)h->sdf[bi] / 32767.0f;
            pt[k] = mk((float)vx, (float)vy, (float)vz);
            cl[k] = mk((float)h->rgb[3 * bi], (float)h->rgb[3 * bi + 1], (float)h->rgb[3 * bi + 2]);
            cl[k] = mk(cl[k].x / 255.f, cl[k].y / 255.f, cl[k].z / 255.f);
          }
          if (!ok) continue;
          int cube = 0;
          for (int k = 0; k < 8; ++k)
            if (sv[k] < 0) cube |= 1 << k;
          const uint64_t word = NUI_MC_TRI_PACKED[cube];
          const int ntri = (int)(word >> 60);
          if (ntri == 0) continue;
          for (int t = 0; t < ntri; ++t)
            for (int q = 0; q < 3; ++q, ++out) {
              const int e = (int)((word >> (4 * (3 * t + q))) & 0xF);
              if (out < cap) {
                const f3 p = sdf_interp(pt[E[e][0]], pt[E[e][1]], sv[E[e][0]], sv[E[e][1]]) * h->c.voxel;
                if (pos) st3(pos, out, p);
                if (col) {
                  const f3 cc = sdf_interp(cl[E[e][0]], cl[E[e][1]], sv[E[e][0]], sv[E[e][1]]);
                  col[4 * out] = cc.x;
                  col[4 * out + 1] = cc.y;
                  col[4 * out + 2] = cc.z;
                  col[4 * out + 3] = 1.0f;
                }
              }
            }
        }
  }
  return out;
}

// accessors for tests
ORC_API long orc_hash_visible(const OrcHash* h, int* ids, long cap) {
  const long n = (long)h->vis_ids.size();
  for (long i = 0; i < n && i < cap; ++i) ids[i] = h->vis_ids[i];
  return n;
}
ORC_API const void* orc_hash_entries(const OrcHash* h) { return h->e.data(); }
ORC_API const int16_t* orc_hash_sdf(const OrcHash* h) { return h->sdf.data(); }
ORC_API const uint8_t* orc_hash_weight(const OrcHash* h) { return h->w.data(); }
ORC_API const uint8_t* orc_hash_rgb(const OrcHash* h) { return h->rgb.data(); }
ORC_API void orc_hash_counters(const OrcHash* h, int* last_block, int* last_excess, long* failed) {
  *last_block = h->last_block;
  *last_excess = h->last_excess;
  *failed = h->failed_allocs;
}

// Engine glue for the hash scene (NuiKinfuOpenCLHashScene::integrateVolume, :533-583, and
// raycastRender with forward rendering off, :1014-1064).
OrcHash* orc_hash_create_internal(int buckets, int excess, int pool, float voxel, float mu, int max_w,
                                  int swapping) {
  OrcHashCfg c{buckets, excess, pool, (uint32_t)(buckets - 1), voxel, mu, max_w, swapping};
  return orc_hash_create(&c);
}
void orc_hash_destroy_internal(OrcHash* h) { orc_hash_destroy(h); }
void orc_hash_scene_integrate(OrcHash* h, const float* depth, const uint8_t* bgra, const OrcCam* cam,
                              const OrcXform* m, long* touched) {
  orc_hash_allocate(h, depth, cam, m);
  orc_hash_integrate(h, depth, bgra, cam, m, touched);
  if (h->c.swapping) orc_hash_swap(h);
}
void orc_hash_scene_raycast(OrcHash* h, const OrcCam* cam, const OrcXform* m, float* vmap, float* nmap,
                            uint8_t* cmap) {
  orc_hash_raycast(h, cam, m, vmap, nmap, cmap, nullptr);
}
