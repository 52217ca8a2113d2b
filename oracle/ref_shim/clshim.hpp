// OpenCL C -> host C++ shim (test infrastructure).
//
// Lets the reference's own kernel sources (src/Kernels/*.cl) compile unmodified, after
// the mechanical rewrites done by build_ref.py (vector literals `(float3)(a,b,c)` ->
// `float3(a,b,c)`, multi-component swizzles `.xy` -> `.swz<0,1>()`, `__local` arrays
// inside kernels -> per-host-thread statics), and run on the CPU: one host thread
// executes one work-group at a time; work-items of a group that call barrier() run as
// cooperative user-level contexts that switch at each barrier.
//
// Semantics chosen where OpenCL leaves them to the implementation: no contraction
// (-ffp-contract=off), glibc expf/sqrtf/hypotf, fast_length = sqrt(dot),
// fast_normalize = normalize = v / sqrt(dot) with zero vectors returned unchanged,
// convert_<int type> truncates toward zero.
#pragma once
#include <math.h>
#include <float.h>
#include <stdint.h>
#include <string.h>
#include <ucontext.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

namespace clshim {

typedef unsigned char uchar;
typedef unsigned short ushort;
typedef unsigned int uint;
typedef unsigned long ulong;

// ------------------------------------------------------------------ vector types
template <class T, int N>
struct vec;

#define CLSHIM_VEC_COMMON(N_)                                                            \
  typedef T value_type;                                                                  \
  static const int size = N_;                                                            \
  T& operator[](int i) { return (&s0)[i]; }                                              \
  const T& operator[](int i) const { return (&s0)[i]; }                                  \
  template <int... I>                                                                    \
  vec<T, sizeof...(I)> swz() const {                                                     \
    vec<T, sizeof...(I)> r;                                                              \
    int k = 0;                                                                           \
    ((r[k++] = (*this)[I]), ...);                                                        \
    return r;                                                                            \
  }

template <class T>
struct vec<T, 2> {
  union {
    struct { T x, y; };
    struct { T s0, s1; };
  };
  CLSHIM_VEC_COMMON(2)
  vec() : x(), y() {}
  template <class A, typename std::enable_if<std::is_arithmetic<A>::value, int>::type = 0>
  vec(A a) : x((T)a), y((T)a) {}
  template <class A, class B>
  vec(A a, B b) : x((T)a), y((T)b) {}
};

template <class T>
struct vec<T, 3> {
  union {
    struct { T x, y, z, pad_; };
    struct { T s0, s1, s2, s3_; };
  };
  CLSHIM_VEC_COMMON(3)
  vec() : x(), y(), z(), pad_() {}
  template <class A, typename std::enable_if<std::is_arithmetic<A>::value, int>::type = 0>
  vec(A a) : x((T)a), y((T)a), z((T)a), pad_() {}
  template <class A, class B, class C>
  vec(A a, B b, C c) : x((T)a), y((T)b), z((T)c), pad_() {}
  template <class A>
  vec(vec<A, 2> ab, T c) : x((T)ab.x), y((T)ab.y), z(c), pad_() {}
  template <class A>
  vec(T a, vec<A, 2> bc) : x(a), y((T)bc.x), z((T)bc.y), pad_() {}
};

template <class T>
struct vec<T, 4> {
  union {
    struct { T x, y, z, w; };
    struct { T s0, s1, s2, s3; };
  };
  CLSHIM_VEC_COMMON(4)
  vec() : x(), y(), z(), w() {}
  template <class A, typename std::enable_if<std::is_arithmetic<A>::value, int>::type = 0>
  vec(A a) : x((T)a), y((T)a), z((T)a), w((T)a) {}
  template <class A, class C, class D>
  vec(vec<A, 2> ab, C c, D d) : x((T)ab.x), y((T)ab.y), z((T)c), w((T)d) {}
  template <class A, class B, class C, class D>
  vec(A a, B b, C c, D d) : x((T)a), y((T)b), z((T)c), w((T)d) {}
  template <class A, class D>
  vec(vec<A, 3> abc, D d) : x((T)abc.x), y((T)abc.y), z((T)abc.z), w((T)d) {}
};

template <class T>
struct vec<T, 8> {
  T s0, s1, s2, s3, s4, s5, s6, s7;
  CLSHIM_VEC_COMMON(8)
  vec() : s0(), s1(), s2(), s3(), s4(), s5(), s6(), s7() {}
  template <class A, typename std::enable_if<std::is_arithmetic<A>::value, int>::type = 0>
  vec(A a) { for (int i = 0; i < 8; ++i) (*this)[i] = (T)a; }
  template <class... A, typename std::enable_if<sizeof...(A) == 8, int>::type = 0>
  vec(A... a) {
    int k = 0;
    ((( *this)[k++] = (T)a), ...);
  }
  // (float8)(float3, float3, float2) style constructors are not used by the kernels
};

#define CLSHIM_DEFV(base, T)        \
  typedef vec<T, 2> base##2;        \
  typedef vec<T, 3> base##3;        \
  typedef vec<T, 4> base##4;        \
  typedef vec<T, 8> base##8;
CLSHIM_DEFV(float, float)
CLSHIM_DEFV(int, int)
CLSHIM_DEFV(uint, uint)
CLSHIM_DEFV(short, short)
CLSHIM_DEFV(ushort, ushort)
CLSHIM_DEFV(char, signed char)
CLSHIM_DEFV(uchar, uchar)

template <class T>
struct is_vec : std::false_type {};
template <class T, int N>
struct is_vec<vec<T, N>> : std::true_type {};

#define CLSHIM_BINOP(op)                                                                 \
  template <class T, int N>                                                              \
  vec<T, N> operator op(const vec<T, N>& a, const vec<T, N>& b) {                        \
    vec<T, N> r;                                                                         \
    for (int i = 0; i < N; ++i) r[i] = (T)(a[i] op b[i]);                                \
    return r;                                                                            \
  }                                                                                      \
  template <class T, int N, class S, typename std::enable_if<!is_vec<S>::value, int>::type = 0> \
  vec<T, N> operator op(const vec<T, N>& a, S b) {                                       \
    vec<T, N> r;                                                                         \
    for (int i = 0; i < N; ++i) r[i] = (T)(a[i] op (T)b);                                \
    return r;                                                                            \
  }                                                                                      \
  template <class T, int N, class S, typename std::enable_if<!is_vec<S>::value, int>::type = 0> \
  vec<T, N> operator op(S a, const vec<T, N>& b) {                                       \
    vec<T, N> r;                                                                         \
    for (int i = 0; i < N; ++i) r[i] = (T)((T)a op b[i]);                                \
    return r;                                                                            \
  }                                                                                      \
  template <class T, int N, class S>                                                     \
  vec<T, N>& operator op##=(vec<T, N>& a, const S& b) {                                  \
    a = a op b;                                                                          \
    return a;                                                                            \
  }
CLSHIM_BINOP(+)
CLSHIM_BINOP(-)
CLSHIM_BINOP(*)
CLSHIM_BINOP(/)
template <class T, int N>
vec<T, N> operator-(const vec<T, N>& a) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r[i] = -a[i];
  return r;
}

// ------------------------------------------------------------------ work-item state
struct WorkItem {
  size_t gid[3], lid[3], grp[3];
};
struct NDRange {
  int dims;
  size_t gsz[3], lsz[3];
};
extern thread_local WorkItem* cur_item;
extern thread_local const NDRange* cur_range;
inline size_t get_global_id(uint d) { return d < 3 ? cur_item->gid[d] : 0; }
inline size_t get_local_id(uint d) { return d < 3 ? cur_item->lid[d] : 0; }
inline size_t get_group_id(uint d) { return d < 3 ? cur_item->grp[d] : 0; }
inline size_t get_global_size(uint d) { return d < 3 ? cur_range->gsz[d] : 1; }
inline size_t get_local_size(uint d) { return d < 3 ? cur_range->lsz[d] : 1; }
inline size_t get_num_groups(uint d) { return d < 3 ? cur_range->gsz[d] / cur_range->lsz[d] : 1; }
void barrier_impl();
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
inline void barrier(int) { barrier_impl(); }
inline void mem_fence(int) {}

// ------------------------------------------------------------------ scalar builtins
inline int mul24(int a, int b) { return a * b; }
inline uint mul24(uint a, uint b) { return a * b; }
template <class A, class B>
inline auto min(A a, B b) -> typename std::common_type<A, B>::type {
  typedef typename std::common_type<A, B>::type C;
  return (C)b < (C)a ? (C)b : (C)a;
}
template <class A, class B>
inline auto max(A a, B b) -> typename std::common_type<A, B>::type {
  typedef typename std::common_type<A, B>::type C;
  return (C)a < (C)b ? (C)b : (C)a;
}
template <class T, int N>
inline vec<T, N> min(vec<T, N> a, vec<T, N> b) {
  for (int i = 0; i < N; ++i) a[i] = b[i] < a[i] ? b[i] : a[i];
  return a;
}
template <class T, int N>
inline vec<T, N> max(vec<T, N> a, vec<T, N> b) {
  for (int i = 0; i < N; ++i) a[i] = a[i] < b[i] ? b[i] : a[i];
  return a;
}
template <class A, class B, class C>
inline A clamp(A x, B lo, C hi) {
  return (A)min(max(x, (A)lo), (A)hi);
}
// sqrt/exp/floor/round/fabs/fmin/fmax/hypot/sin/cos/isnan on float resolve to the C++
// standard library float overloads (sqrtf, expf, ... semantics).
inline float rsqrt(float a) { return 1.0f / sqrtf(a); }
inline float sign(float a) { return std::isnan(a) ? 0.f : (a > 0.f ? 1.f : (a < 0.f ? -1.f : a)); }
template <class T, int N>
inline vec<T, N> fabs(vec<T, N> a) {
  for (int i = 0; i < N; ++i) a[i] = fabsf(a[i]);
  return a;
}
template <class T, int N>
inline vec<T, N> floor(vec<T, N> a) {
  for (int i = 0; i < N; ++i) a[i] = floorf(a[i]);
  return a;
}
template <class T, int N>
inline vec<T, N> sign(vec<T, N> a) {
  for (int i = 0; i < N; ++i) a[i] = sign(a[i]);
  return a;
}
inline float mix(float a, float b, float t) { return a + (b - a) * t; }
template <class T, int N>
inline vec<T, N> mix(vec<T, N> a, vec<T, N> b, T t) {
  return a + (b - a) * t;
}
template <int N>
inline float dot(vec<float, N> a, vec<float, N> b) {
  float s = a[0] * b[0];
  for (int i = 1; i < N; ++i) s = s + a[i] * b[i];
  return s;
}
inline float dot(float a, float b) { return a * b; }
inline float3 cross(float3 a, float3 b) {
  return float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <int N>
inline float length(vec<float, N> a) { return sqrtf(dot(a, a)); }
template <int N>
inline float fast_length(vec<float, N> a) { return sqrtf(dot(a, a)); }
template <int N>
inline vec<float, N> normalize(vec<float, N> a) {
  bool zero = true;
  for (int i = 0; i < N; ++i) zero = zero && a[i] == 0.f;
  if (zero) return a;
  float l = sqrtf(dot(a, a));
  for (int i = 0; i < N; ++i) a[i] = a[i] / l;
  return a;
}
template <int N>
inline vec<float, N> fast_normalize(vec<float, N> a) { return normalize(a); }
template <class T, int N>
inline int all(vec<T, N> a) {
  for (int i = 0; i < N; ++i)
    if (!a[i]) return 0;
  return 1;
}
template <class T, int N>
inline int any(vec<T, N> a) {
  for (int i = 0; i < N; ++i)
    if (a[i]) return 1;
  return 0;
}

// conversions: truncation toward zero for float -> integer
#define CLSHIM_CONV(name, T)                                                             \
  template <class S>                                                                     \
  inline T convert_##name(S s) { return (T)s; }                                          \
  template <class S, int N>                                                              \
  inline vec<T, N> convert_##name##N(vec<S, N> s) {                                      \
    vec<T, N> r;                                                                         \
    for (int i = 0; i < N; ++i) r[i] = (T)s[i];                                          \
    return r;                                                                            \
  }                                                                                      \
  template <class S>                                                                     \
  inline vec<T, 2> convert_##name##2(vec<S, 2> s) { return convert_##name##N(s); }       \
  template <class S>                                                                     \
  inline vec<T, 3> convert_##name##3(vec<S, 3> s) { return convert_##name##N(s); }       \
  template <class S>                                                                     \
  inline vec<T, 4> convert_##name##4(vec<S, 4> s) { return convert_##name##N(s); }
CLSHIM_CONV(float, float)
CLSHIM_CONV(int, int)
CLSHIM_CONV(uint, uint)
CLSHIM_CONV(short, short)
CLSHIM_CONV(ushort, ushort)
CLSHIM_CONV(uchar, uchar)
// float -> uchar: OpenCL leaves out-of-range values to the implementation; this shim keeps
// the low byte of the truncation toward zero (negative values wrap), as x86 hosts do.
inline uchar convert_uchar(float s) { return (uchar)(int)s; }
CLSHIM_CONV(char, signed char)

// ------------------------------------------------------------------ loads / stores
template <class T>
inline T vload(size_t i, const T* p) { return p[i]; }
template <class T>
inline void vstore(T v, size_t i, T* p) { p[i] = v; }
template <class T>
inline void vstore(double v, size_t i, T* p) { p[i] = (T)v; }
template <class T>
inline vec<T, 2> vload2(size_t i, const T* p) { return vec<T, 2>(p[2 * i], p[2 * i + 1]); }
template <class T>
inline vec<T, 3> vload3(size_t i, const T* p) { return vec<T, 3>(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
template <class T>
inline vec<T, 4> vload4(size_t i, const T* p) {
  return vec<T, 4>(p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]);
}
template <class T>
inline void vstore2(vec<T, 2> v, size_t i, T* p) { p[2 * i] = v.x; p[2 * i + 1] = v.y; }
template <class T>
inline void vstore3(vec<T, 3> v, size_t i, T* p) {
  p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z;
}
template <class T>
inline void vstore3(float s, size_t i, T* p) { p[3 * i] = p[3 * i + 1] = p[3 * i + 2] = (T)s; }
template <class T>
inline void vstore4(vec<T, 4> v, size_t i, T* p) {
  p[4 * i] = v.x; p[4 * i + 1] = v.y; p[4 * i + 2] = v.z; p[4 * i + 3] = v.w;
}
template <class T, class U>
inline void vstore4(vec<U, 4> v, size_t i, T* p) {
  p[4 * i] = (T)v.x; p[4 * i + 1] = (T)v.y; p[4 * i + 2] = (T)v.z; p[4 * i + 3] = (T)v.w;
}

// ------------------------------------------------------------------ atomics
template <class T>
inline T atomic_add(volatile T* p, T v) { return __atomic_fetch_add((T*)p, v, __ATOMIC_SEQ_CST); }
template <class T>
inline T atomic_inc(volatile T* p) { return __atomic_fetch_add((T*)p, (T)1, __ATOMIC_SEQ_CST); }
template <class T>
inline T atomic_dec(volatile T* p) { return __atomic_fetch_sub((T*)p, (T)1, __ATOMIC_SEQ_CST); }
template <class T>
inline T atomic_xchg(volatile T* p, T v) { return __atomic_exchange_n((T*)p, v, __ATOMIC_SEQ_CST); }
template <class T>
inline T atomic_cmpxchg(volatile T* p, T cmp, T v) {
  __atomic_compare_exchange_n((T*)p, &cmp, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
  return cmp;
}
template <class T>
inline T atom_cmpxchg(volatile T* p, T cmp, T v) { return atomic_cmpxchg(p, cmp, v); }
template <class T>
inline T atom_xchg(volatile T* p, T v) { return atomic_xchg(p, v); }

// image types appear only in GL-interop kernels, which are never launched here
struct image2d_t {};
inline void write_imagef(image2d_t, int2, float4) {}

}  // namespace clshim

#ifndef NAN
#define NAN (__builtin_nanf(""))
#endif
#define MAXFLOAT FLT_MAX
#define __kernel
#define kernel
#define __global
#define __constant const
#define __private
#define __read_only
#define __write_only
#define write_only
#define read_only
#define __local

// ------------------------------------------------------------------ launcher
#include <functional>
namespace clshim {
// Runs `body()` once per work-item of the NDRange.  Groups are spread over OpenMP host
// threads.  If `cooperative`, all items of a group run as user contexts that yield at
// barrier(); otherwise items run to completion one after another.
void run_ndrange_fn(int dims, const size_t* gsz, const size_t* lsz, bool cooperative,
                    const std::function<void()>& body);
}  // namespace clshim
