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
#include <limits>
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
// exp(r) by Horner evaluation of the degree-7 Taylor polynomial, times 2^k.
ORC_API float oracle_expf(float x) {
  if (std::isnan(x)) return x;
  if (x > 88.5f) return std::numeric_limits<float>::infinity();
  if (x < -103.5f) return 0.f;
  float kf = std::nearbyint(x * 1.44269504088896341f);
  float r = x - kf * 0.693145751953125f;
  r = r - kf * 1.42860682030941723e-6f;
  float p = 1.98412698412698413e-4f;
  p = p * r + 1.38888888888888889e-3f;
  p = p * r + 8.33333333333333333e-3f;
  p = p * r + 4.16666666666666667e-2f;
  p = p * r + 1.66666666666666667e-1f;
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
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

// A10  integrateTsdfVolumeKernel   tsdfVolume.cl:31-190 (voxelWrap = 0, normals = NULL as
// passed by NuiKinfuOpenCLScene.cpp:278).  `touched` receives the number of voxels
// read-modify-written.
ORC_API void orc_tsdf_integrate(const float* depth, const uint8_t* bgra, const OrcCam* cam,
                                const OrcXform* m, const OrcTsdf* p, int16_t* vol, uint8_t* cvol,
                                int max_color_weight, long* touched) {
  const int rx = (int)p->res[0], ry = (int)p->res[1], rz = (int)p->res[2];
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
      const long base = ((long)vx + (long)vy * rx) * rz;
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
        long idx = base + vz;
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

// ---------------------------------------------------------------------------------
// A12  raycastKernel   raycast.cl:128-277 with interpolateTrilineary raycast.cl:36-120.
// The trilinear weights are reproduced as written: the x-neighbour voxel is weighted
// with the y fraction and vice versa (raycast.cl:78-119 vs the index steps at :71-101).
namespace {
struct RcVol {
  const int16_t* v;
  int rx, ry, rz;
  float cell[3];
  long idx(int x, int y, int z) const { return ((long)y * rx + x) * rz + z; }
};
inline void voxel_of(f3 p, const float* cell, int& gx, int& gy, int& gz) {
  gx = (int)std::round(p.x / cell[0]);
  gy = (int)std::round(p.y / cell[1]);
  gz = (int)std::round(p.z / cell[2]);
}
inline bool tsdf_at(const RcVol& V, long idx, float& f) {
  int16_t a = V.v[2 * idx], w = V.v[2 * idx + 1];
  f = (float)a / 32766.f;
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
  if (!tsdf_at(V, V.idx(gx, gy, gz + 1), t001)) return QNAN;
  if (!tsdf_at(V, V.idx(gx + 1, gy, gz + 1), t011)) return QNAN;
  if (!tsdf_at(V, V.idx(gx + 1, gy, gz), t010)) return QNAN;
  if (!tsdf_at(V, V.idx(gx + 1, gy + 1, gz), t110)) return QNAN;
  if (!tsdf_at(V, V.idx(gx + 1, gy + 1, gz + 1), t111)) return QNAN;
  if (!tsdf_at(V, V.idx(gx, gy + 1, gz + 1), t101)) return QNAN;
  if (!tsdf_at(V, V.idx(gx, gy + 1, gz), t100)) return QNAN;
  return t000 * (1 - a) * (1 - b) * (1 - c) + t001 * (1 - a) * (1 - b) * c +
         t010 * (1 - a) * b * (1 - c) + t011 * (1 - a) * b * c + t100 * a * (1 - b) * (1 - c) +
         t101 * a * (1 - b) * c + t110 * a * b * (1 - c) + t111 * a * b * c;
}
}  // namespace

ORC_API void orc_raycast(const int16_t* vol, const uint8_t* cvol, const OrcTsdf* p,
                         const OrcCam* cam, const OrcXform* m, int W, int H, float* vmap,
                         float* nmap, uint8_t* cmap, long* steps_out) {
  RcVol V{vol, (int)p->res[0], (int)p->res[1], (int)p->res[2], {p->cell[0], p->cell[1], p->cell[2]}};
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

// ---------------------------------------------------------------------------------
// A7  icp_block_kernel + compute_sums (icp.cl:222-326): per-pixel rows, summed here in
// double.  `vcur` is the level's vertex map (w x h), `vref`/`nref` the full-size world
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

// A7 host loop   NuiKinfuOpenCLDepthTracker.cpp:240-504.
// vlevels[l] is the level-l vertex map ((W>>l) x (H>>l)); iters[l] its iteration count.
// R/t: in = initial estimate, out = estimate.  Returns 0 on success, 1 on singular system.
ORC_API int orc_icp(const float* const* vlevels, const int* iters, int levels, const float* vref,
                    const float* nref, const OrcCam* cam, const OrcXform* prev, float dist_thr,
                    float* R, float* t, OrcIcpStats* stats) {
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
      orc_icp_rows(vlevels[lv], w, h, vref, nref, cam, Rc, tc, prev, dist_thr, nullptr, sums);
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
};

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
  long nvox = (long)c.res[0] * c.res[1] * c.res[2];
  e->vol.resize(2 * nvox);
  if (c.color) e->cvol.resize(4 * nvox);
  orc_tsdf_init(e->vol.data(), c.color ? e->cvol.data() : nullptr, nvox);
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

ORC_API void orc_engine_destroy(OrcEngine* e) { delete e; }

static double rel_angle(const float* Ra, const float* Rb) {
  // angle of Ra^-1 Rb (rodrigues2 norm, NuiMatrixUtilities.cpp:7-52)
  double tr = 0;
  for (int i = 0; i < 3; ++i)
    for (int k = 0; k < 3; ++k) tr += (double)Ra[k * 3 + i] * (double)Rb[k * 3 + i];
  double cv = std::max(-1.0, std::min(1.0, (tr - 1.0) / 2.0));
  return std::acos(cv);
}

// Returns 0 on success, 1 when tracking is lost (singular ICP system).
ORC_API int orc_engine_frame(OrcEngine* e, const uint16_t* raw, const uint8_t* bgra) {
  const OrcEngineCfg& c = e->c;
  const int W = c.W, H = c.H;
  const long N = (long)W * H;
  orc_pass_filter(raw, N, c.dmin, c.dmax, e->depth.data());
  orc_bilateral(e->depth.data(), W, H, e->gauss.data(), c.filter_radius, c.sigma_depth2_inv_half,
                c.depth_threshold, e->dl[0].data());
  orc_depth2vertex(e->dl[0].data(), W, H, &e->cam, 1, e->vl[0].data());
  const uint8_t* col = c.color ? bgra : nullptr;
  if (e->frames == 0) {
    orc_normals(e->vl[0].data(), W, H, c.depth_threshold, e->normals.data());
    orc_transform_maps(e->vl[0].data(), e->normals.data(), W, H, &e->xf, e->vref.data(), e->nref.data());
    orc_scale_depths(e->depth.data(), W, H, &e->cam);
    orc_tsdf_integrate(e->depth.data(), col, &e->cam, &e->xf, &e->tp, e->vol.data(),
                       c.color ? e->cvol.data() : nullptr, c.max_color_weight, &e->touched);
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
    int st = orc_icp(lv.data(), c.iters, c.levels, e->vref.data(), e->nref.data(), &e->cam, &e->xf, dthr,
                     R, t, &e->last);
    if (st != 0) return 1;
    orc_make_xform(R, t, &e->xf);
    double rn = rel_angle(e->xf.R, e->lastR);
    double tn = std::sqrt((double)(e->xf.t[0] - e->lastT[0]) * (e->xf.t[0] - e->lastT[0]) +
                          (double)(e->xf.t[1] - e->lastT[1]) * (e->xf.t[1] - e->lastT[1]) +
                          (double)(e->xf.t[2] - e->lastT[2]) * (e->xf.t[2] - e->lastT[2]));
    if ((float)((rn + tn) / 2) >= c.integration_threshold) {
      orc_scale_depths(e->depth.data(), W, H, &e->cam);
      orc_tsdf_integrate(e->depth.data(), col, &e->cam, &e->xf, &e->tp, e->vol.data(),
                         c.color ? e->cvol.data() : nullptr, c.max_color_weight, &e->touched);
      std::memcpy(e->lastR, e->xf.R, sizeof(e->lastR));
      std::memcpy(e->lastT, e->xf.t, sizeof(e->lastT));
    }
    orc_raycast(e->vol.data(), c.color ? e->cvol.data() : nullptr, &e->tp, &e->cam, &e->xf, W, H,
                e->vref.data(), e->nref.data(), nullptr, nullptr);
  }
  e->frames += 1;
  return 0;
}

ORC_API void orc_engine_pose(const OrcEngine* e, float* R, float* t) {
  std::memcpy(R, e->xf.R, 9 * sizeof(float));
  std::memcpy(t, e->xf.t, 3 * sizeof(float));
}
ORC_API const int16_t* orc_engine_volume(const OrcEngine* e) { return e->vol.data(); }
ORC_API const uint8_t* orc_engine_color_volume(const OrcEngine* e) {
  return e->cvol.empty() ? nullptr : e->cvol.data();
}
ORC_API const float* orc_engine_refmap(const OrcEngine* e, int which) {
  return which == 0 ? e->vref.data() : e->nref.data();
}
ORC_API void orc_engine_tsdf_params(const OrcEngine* e, OrcTsdf* out) { *out = e->tp; }
ORC_API void orc_engine_icp_stats(const OrcEngine* e, OrcIcpStats* out) { *out = e->last; }
ORC_API long orc_engine_touched(const OrcEngine* e) { return e->touched; }
