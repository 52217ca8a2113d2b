// Seeded synthetic RGB-D input: analytic SDF scenes, camera trajectories, depth/colour
// rendering by sphere tracing, and the Kinect noise model
//   sigma(z) = 0.0012 + 0.0019 (z - 0.4)^2 m, 1 mm quantisation, 2% dropouts,
//   depth outside [0.4, 4.5] m -> 0.
// The reference reads recorded Kinect frames (NuiFrameLoader.cpp:26-92); this generator
// stands in for those recordings.  It is host code (OpenMP), shared by tests and bench.
//
// Frames: camera x right, y down, z forward; world = camera frame of frame 0.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "nui_synth.h"

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
inline double u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(splitmix64(seed)) {}
  double uni() {
    s = splitmix64(s);
    return u01(s);
  }
  double uni(double a, double b) { return a + (b - a) * uni(); }
  double gauss() {
    double a = std::max(uni(), 1e-300), b = uni();
    return std::sqrt(-2.0 * std::log(a)) * std::cos(6.283185307179586 * b);
  }
};

struct V3 {
  double x, y, z;
};
inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double len(V3 a) { return std::sqrt(dot(a, a)); }

enum PrimKind { P_PLANE = 0, P_SPHERE = 1, P_BOX = 2, P_CYL = 3, P_ROOM = 4 };
struct Prim {
  int kind;
  V3 c;    // centre / point on plane
  V3 h;    // half extents (box, room), normal (plane), (r, half-height, 0) cylinder
  double r;
};

}  // namespace

struct nui_synth_scene {
  int kind;
  uint64_t seed;
  std::vector<Prim> prims;
  double tex_scale;
};

namespace {

double prim_sdf(const Prim& p, V3 q) {
  switch (p.kind) {
    case P_PLANE:
      return dot(q - p.c, p.h);
    case P_SPHERE:
      return len(q - p.c) - p.r;
    case P_BOX: {
      V3 d = q - p.c;
      V3 a = v3(std::fabs(d.x) - p.h.x, std::fabs(d.y) - p.h.y, std::fabs(d.z) - p.h.z);
      V3 o = v3(std::max(a.x, 0.0), std::max(a.y, 0.0), std::max(a.z, 0.0));
      return len(o) + std::min(std::max(a.x, std::max(a.y, a.z)), 0.0);
    }
    case P_CYL: {  // axis along y
      V3 d = q - p.c;
      double rr = std::sqrt(d.x * d.x + d.z * d.z) - p.h.x;
      double hh = std::fabs(d.y) - p.h.y;
      double ox = std::max(rr, 0.0), oy = std::max(hh, 0.0);
      return std::sqrt(ox * ox + oy * oy) + std::min(std::max(rr, hh), 0.0);
    }
    case P_ROOM: {  // inside of a box: positive inside, walls at the box faces
      V3 d = q - p.c;
      return std::min(std::min(p.h.x - std::fabs(d.x), p.h.y - std::fabs(d.y)), p.h.z - std::fabs(d.z));
    }
  }
  return 1e9;
}

double scene_sdf(const nui_synth_scene& s, V3 q) {
  double d = 1e9;
  for (const Prim& p : s.prims) d = std::min(d, prim_sdf(p, q));
  return d;
}

// 3-D value noise on a hashed integer lattice, trilinear with smoothstep weights
double lattice(uint64_t seed, long x, long y, long z) {
  uint64_t h = splitmix64(seed ^ splitmix64((uint64_t)x * 0x8DA6B343ULL ^ splitmix64((uint64_t)y * 0xD8163841ULL ^
                                                                                      (uint64_t)z * 0xCB1AB31FULL)));
  return u01(h);
}
double value_noise(uint64_t seed, V3 p) {
  double fx = std::floor(p.x), fy = std::floor(p.y), fz = std::floor(p.z);
  long ix = (long)fx, iy = (long)fy, iz = (long)fz;
  double tx = p.x - fx, ty = p.y - fy, tz = p.z - fz;
  tx = tx * tx * (3 - 2 * tx);
  ty = ty * ty * (3 - 2 * ty);
  tz = tz * tz * (3 - 2 * tz);
  double c[2][2][2];
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b)
      for (int e = 0; e < 2; ++e) c[a][b][e] = lattice(seed, ix + a, iy + b, iz + e);
  double x00 = c[0][0][0] + (c[1][0][0] - c[0][0][0]) * tx, x10 = c[0][1][0] + (c[1][1][0] - c[0][1][0]) * tx;
  double x01 = c[0][0][1] + (c[1][0][1] - c[0][0][1]) * tx, x11 = c[0][1][1] + (c[1][1][1] - c[0][1][1]) * tx;
  double y0 = x00 + (x10 - x00) * ty, y1 = x01 + (x11 - x01) * ty;
  return y0 + (y1 - y0) * tz;
}

void rot_axis_angle(V3 axis, double ang, double R[9]) {
  double n = len(axis);
  if (n < 1e-15) {
    double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::memcpy(R, I, sizeof(I));
    return;
  }
  axis = axis * (1.0 / n);
  double c = std::cos(ang), s = std::sin(ang), C = 1 - c;
  double x = axis.x, y = axis.y, z = axis.z;
  double M[9] = {c + x * x * C,     x * y * C - z * s, x * z * C + y * s, y * x * C + z * s, c + y * y * C,
                 y * z * C - x * s, z * x * C - y * s, z * y * C + x * s, c + z * z * C};
  std::memcpy(R, M, sizeof(M));
}
void matmul3(const double A[9], const double B[9], double C[9]) {
  double T[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) T[i * 3 + j] = A[i * 3] * B[j] + A[i * 3 + 1] * B[3 + j] + A[i * 3 + 2] * B[6 + j];
  std::memcpy(C, T, sizeof(T));
}

}  // namespace

extern "C" {

NUI_SYNTH_API nui_synth_scene* nui_synth_scene_create(int kind, uint64_t seed, float extent) {
  nui_synth_scene* s = new nui_synth_scene();
  s->kind = kind;
  s->seed = seed;
  Rng rng(seed * 0x2545F4914F6CDD1DULL + 17);
  if (kind == NUI_SYNTH_TABLETOP) {
    // volume cube of side D spans x,y in [-D/2, D/2], z in [0, D]; objects around (0, 0, D/2)
    const double D = extent > 0 ? extent : 3.0;
    const double ground = 0.5;  // y down: the ground is 0.5 m below the camera height
    s->prims.push_back(Prim{P_PLANE, v3(0, ground, 0), v3(0, -1, 0), 0});
    const double zc = D / 2;
    for (int i = 0; i < 3; ++i) {
      double r = rng.uni(0.2, 0.5);
      double ang = 2.0943951 * i + rng.uni(-0.4, 0.4), rad = rng.uni(0.2, 0.6);
      s->prims.push_back(Prim{P_SPHERE, v3(rad * std::cos(ang), ground - r - rng.uni(0.0, 0.3), zc + rad * std::sin(ang)),
                              v3(0, 0, 0), r});
    }
    for (int i = 0; i < 2; ++i) {
      V3 h = v3(rng.uni(0.15, 0.35), rng.uni(0.15, 0.35), rng.uni(0.15, 0.35));
      double ang = 1.0471976 + 3.1415927 * i + rng.uni(-0.4, 0.4), rad = rng.uni(0.3, 0.7);
      s->prims.push_back(Prim{P_BOX, v3(rad * std::cos(ang), ground - h.y, zc + rad * std::sin(ang)), h, 0});
    }
    s->tex_scale = 12.0;
  } else {
    // room 8 x 3 x 6 m (x, y(down), z), camera start near the centre at eye height
    const V3 centre = v3(0, 0.3, 0);
    s->prims.push_back(Prim{P_ROOM, centre, v3(4.0, 1.5, 3.0), 0});
    for (int i = 0; i < 40; ++i) {
      int k = i % 3;
      double x = rng.uni(-3.5, 3.5), z = rng.uni(-2.6, 2.6);
      if (std::fabs(x) < 0.8 && std::fabs(z) < 0.8) x += (x < 0 ? -1.0 : 1.0);  // keep the start clear
      double floor_y = centre.y + 1.5;
      if (k == 0) {
        double r = rng.uni(0.1, 0.4);
        s->prims.push_back(Prim{P_SPHERE, v3(x, floor_y - r - rng.uni(0, 1.2), z), v3(0, 0, 0), r});
      } else if (k == 1) {
        V3 h = v3(rng.uni(0.1, 0.45), rng.uni(0.1, 0.6), rng.uni(0.1, 0.45));
        s->prims.push_back(Prim{P_BOX, v3(x, floor_y - h.y, z), h, 0});
      } else {
        double r = rng.uni(0.08, 0.3), hh = rng.uni(0.2, 1.0);
        s->prims.push_back(Prim{P_CYL, v3(x, floor_y - hh, z), v3(r, hh, 0), 0});
      }
    }
    s->tex_scale = 10.0;
  }
  return s;
}

NUI_SYNTH_API void nui_synth_scene_destroy(nui_synth_scene* s) { delete s; }

NUI_SYNTH_API float nui_synth_scene_sdf(const nui_synth_scene* s, float x, float y, float z) {
  return (float)scene_sdf(*s, v3(x, y, z));
}

NUI_SYNTH_API void nui_synth_scene_sdf_many(const nui_synth_scene* s, const float* xyz, long n, float* out) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) out[i] = (float)scene_sdf(*s, v3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
}

// Camera-to-world pose (R row-major, t = camera centre) of `frame` on the scene's path.
//  tabletop: orbit of radius `radius` around (0, 0, radius) starting at the origin looking
//            down +z, deg_per_frame per frame, seeded jitter (1 mm, 0.2 deg, 1 sigma).
//  room:     walk at 1.2 m/s (30 Hz) along a seeded smooth loop, yaw rate <= 60 deg/s.
NUI_SYNTH_API void nui_synth_trajectory(int kind, uint64_t seed, int frame, float radius, float deg_per_frame,
                                  float* R_out, float* t_out) {
  double R[9], t[3];
  if (kind == NUI_SYNTH_TABLETOP) {
    double th = (double)deg_per_frame * frame * 3.141592653589793 / 180.0;
    double r = radius;
    double Ry[9] = {std::cos(th), 0, std::sin(th), 0, 1, 0, -std::sin(th), 0, std::cos(th)};
    t[0] = -r * std::sin(th);
    t[1] = 0;
    t[2] = r - r * std::cos(th);
    std::memcpy(R, Ry, sizeof(R));
    if (frame > 0) {
      Rng rng(seed ^ splitmix64((uint64_t)frame + 0x51ED27ULL));
      for (int i = 0; i < 3; ++i) t[i] += 0.001 * rng.gauss();
      V3 ax = v3(rng.gauss(), rng.gauss(), rng.gauss());
      double ang = 0.2 * 3.141592653589793 / 180.0 * rng.gauss();
      double J[9];
      rot_axis_angle(ax, ang, J);
      matmul3(R, J, R);
    }
  } else {
    // smooth closed loop: superposition of seeded sinusoids; heading follows the path
    Rng rng(seed * 0x9E3779B97F4A7C15ULL + 3);
    double a1 = rng.uni(1.2, 2.0), a2 = rng.uni(0.6, 1.1), ph1 = rng.uni(0, 6.28), ph2 = rng.uni(0, 6.28);
    const double dt = 1.0 / 30.0, speed = 1.2;
    // arc-length parametrised by numerically integrating the curve speed
    auto curve = [&](double u, double& x, double& z) {
      x = a1 * std::sin(u + ph1) - a1 * std::sin(ph1) + 0.25 * std::sin(3 * u + ph2) - 0.25 * std::sin(ph2);
      z = a2 * std::sin(2 * u) + 0.2 * std::cos(2 * u + ph2) - 0.2 * std::cos(ph2);
    };
    double u = 0, sacc = 0, target = speed * dt * frame;
    double px, pz;
    curve(0, px, pz);
    const double du = 1e-3;
    while (sacc < target) {
      double nx, nz;
      curve(u + du, nx, nz);
      sacc += std::sqrt((nx - px) * (nx - px) + (nz - pz) * (nz - pz));
      px = nx;
      pz = nz;
      u += du;
    }
    double nx, nz;
    curve(u + 0.05, nx, nz);
    double heading = std::atan2(nx - px, nz - pz);  // rotation about y, 0 = +z
    // limit the turn so that the yaw rate stays below 60 deg/s: heading blended with a
    // slow seeded look-around
    heading = 0.6 * heading + 0.3 * std::sin(0.7 * frame * dt + ph1);
    double c = std::cos(heading), s = std::sin(heading);
    double Ry[9] = {c, 0, s, 0, 1, 0, -s, 0, c};
    std::memcpy(R, Ry, sizeof(R));
    t[0] = px;
    t[1] = 0.02 * std::sin(2 * 3.14159 * 1.8 * frame * dt);  // walking bob
    t[2] = pz;
  }
  for (int i = 0; i < 9; ++i) R_out[i] = (float)R[i];
  for (int i = 0; i < 3; ++i) t_out[i] = (float)t[i];
}

// Renders one frame: uint16 depth in mm (0 = no measurement) and optional BGRA8 colour.
NUI_SYNTH_API void nui_synth_render(const nui_synth_scene* s, const float* Rf, const float* tf, int W, int H, float fx,
                              float fy, float cx, float cy, uint64_t noise_seed, int frame, int add_noise,
                              uint16_t* depth_mm, uint8_t* bgra) {
  double R[9], t[3];
  for (int i = 0; i < 9; ++i) R[i] = Rf[i];
  for (int i = 0; i < 3; ++i) t[i] = tf[i];
  const uint64_t fseed = splitmix64(noise_seed ^ splitmix64((uint64_t)frame * 0x632BE59BD9B4E019ULL + 1));
#pragma omp parallel for schedule(dynamic, 4)
  for (int v = 0; v < H; ++v)
    for (int u = 0; u < W; ++u) {
      const long i = (long)v * W + u;
      V3 dc = v3((u - cx) / fx, (v - cy) / fy, 1.0);
      const double dl = len(dc);
      V3 d = v3(R[0] * dc.x + R[1] * dc.y + R[2] * dc.z, R[3] * dc.x + R[4] * dc.y + R[5] * dc.z,
                R[6] * dc.x + R[7] * dc.y + R[8] * dc.z) *
             (1.0 / dl);
      V3 o = v3(t[0], t[1], t[2]);
      double tt = 0.05, hit = -1;
      for (int k = 0; k < 256 && tt < 8.0; ++k) {
        double sd = scene_sdf(*s, o + d * tt);
        if (sd < 1e-5) {
          hit = tt;
          break;
        }
        tt += sd;
      }
      uint16_t out = 0;
      V3 P = v3(0, 0, 0);
      if (hit > 0) {
        // refine with a few secant-free bisection steps around the hit
        double a = std::max(0.0, hit - 1e-3), b = hit + 1e-3;
        for (int k = 0; k < 20; ++k) {
          double m = 0.5 * (a + b);
          if (scene_sdf(*s, o + d * m) > 0) a = m; else b = m;
        }
        hit = 0.5 * (a + b);
        P = o + d * hit;
        double z = hit / dl;  // z-depth
        if (add_noise) {
          uint64_t h = splitmix64(fseed ^ (uint64_t)i * 0x9E3779B97F4A7C15ULL);
          double g1 = std::max(u01(h), 1e-300), g2 = u01(splitmix64(h));
          double gn = std::sqrt(-2.0 * std::log(g1)) * std::cos(6.283185307179586 * g2);
          double sig = 0.0012 + 0.0019 * (z - 0.4) * (z - 0.4);
          z += sig * gn;
          double drop = u01(splitmix64(h ^ 0xD1B54A32D192ED03ULL));
          if (drop < 0.02) z = 0;
        }
        if (z >= 0.4 && z <= 4.5) out = (uint16_t)std::lround(z * 1000.0);
      }
      depth_mm[i] = out;
      if (bgra) {
        uint8_t* c = bgra + 4 * i;
        if (hit > 0) {
          V3 q = P * s->tex_scale;
          double n1 = value_noise(s->seed * 3 + 1, q), n2 = value_noise(s->seed * 3 + 2, q * 2.3);
          double n3 = value_noise(s->seed * 3 + 3, q * 0.7);
          c[0] = (uint8_t)std::min(255.0, 40 + 200 * (0.6 * n1 + 0.4 * n2));
          c[1] = (uint8_t)std::min(255.0, 40 + 200 * (0.5 * n2 + 0.5 * n3));
          c[2] = (uint8_t)std::min(255.0, 40 + 200 * (0.7 * n3 + 0.3 * n1));
          c[3] = 255;
        } else {
          c[0] = c[1] = c[2] = 0;
          c[3] = 0;
        }
      }
    }
}

}  // extern "C"
