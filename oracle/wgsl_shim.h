// WGSL types and builtins in C++, for the translated reference shader
// functions of oracle/_ref (test infrastructure: only the pin test of the
// oracle uses it, never the product).
//
// The translation (oracle/wgsl_to_cpp.py) turns `vec3<f32>` into `vec3f`,
// `.xz` into `.xz()`, `u32(x)` into `wgsl_u32(x)` and so on; this header
// supplies those names with the semantics the oracle documents for the WGSL
// builtins: mix(a,b,t) = a*(1-t) + b*t, smoothstep per the WGSL spec,
// clamp = min(max(x, lo), hi), min/max as IEEE minimumNumber/maximumNumber,
// normalize(v) = v * (1/sqrt(dot(v,v))), saturating float -> integer
// conversion, and sin/cos/exp/pow from include/vxe/detmath.h.  With the same
// elementary functions on both sides, any difference between a translated
// reference function and the oracle's restatement of it is a difference in
// the restatement.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>

#include "vxe/detmath.h"

namespace wgsl {

using f32 = float;
using u32 = uint32_t;
using i32 = int32_t;

inline float wmin(float a, float b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a < b) return a;
  if (b < a) return b;
  return std::signbit(a) ? a : b;
}
inline float wmax(float a, float b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a > b) return a;
  if (b > a) return b;
  return std::signbit(a) ? b : a;
}
inline u32 wmin(u32 a, u32 b) { return a < b ? a : b; }
inline u32 wmax(u32 a, u32 b) { return a > b ? a : b; }
inline i32 wmin(i32 a, i32 b) { return a < b ? a : b; }
inline i32 wmax(i32 a, i32 b) { return a > b ? a : b; }

// Conversions with WGSL semantics (float -> integer saturates, NaN -> 0).
inline float wgsl_f32(float x) { return x; }
inline float wgsl_f32(u32 x) { return (float)x; }
inline float wgsl_f32(i32 x) { return (float)x; }
inline float wgsl_f32(bool x) { return x ? 1.0f : 0.0f; }
inline u32 wgsl_u32(float f) {
  if (f != f || f <= 0.0f) return 0u;
  if (f >= 4294967296.0f) return 0xFFFFFFFFu;
  return (u32)f;
}
inline u32 wgsl_u32(u32 x) { return x; }
inline u32 wgsl_u32(i32 x) { return (u32)x; }
inline u32 wgsl_u32(bool x) { return x ? 1u : 0u; }
inline i32 wgsl_i32(float f) {
  if (f != f) return 0;
  if (f >= 2147483648.0f) return INT32_MAX;
  if (f <= -2147483648.0f) return INT32_MIN;
  return (i32)f;
}
inline i32 wgsl_i32(i32 x) { return x; }
inline i32 wgsl_i32(u32 x) { return (i32)x; }
template <class T>
inline T wgsl_conv(float x) {
  if constexpr (std::is_same_v<T, float>) return x;
  else if constexpr (std::is_same_v<T, u32>) return wgsl_u32(x);
  else return wgsl_i32(x);
}
template <class T>
inline T wgsl_conv(u32 x) {
  if constexpr (std::is_same_v<T, float>) return (float)x;
  else return (T)x;
}
template <class T>
inline T wgsl_conv(i32 x) {
  if constexpr (std::is_same_v<T, float>) return (float)x;
  else return (T)x;
}

template <class T, int N>
struct vec {
  T v[N];
  T& operator[](int i) { return v[i]; }
  const T& operator[](int i) const { return v[i]; }
};

template <class T>
struct vec<T, 2> {
  T x, y;
  vec() : x(), y() {}
  explicit vec(T s) : x(s), y(s) {}
  vec(T a, T b) : x(a), y(b) {}
  template <class U>
  explicit vec(const vec<U, 2>& o) : x(wgsl_conv<T>(o.x)), y(wgsl_conv<T>(o.y)) {}
  T& operator[](int i) { return i == 0 ? x : y; }
  const T& operator[](int i) const { return i == 0 ? x : y; }
};

template <class T>
struct vec<T, 3> {
  T x, y, z;
  vec() : x(), y(), z() {}
  explicit vec(T s) : x(s), y(s), z(s) {}
  vec(T a, T b, T c) : x(a), y(b), z(c) {}
  vec(vec<T, 2> a, T c) : x(a.x), y(a.y), z(c) {}
  vec(T a, vec<T, 2> b) : x(a), y(b.x), z(b.y) {}
  template <class U>
  explicit vec(const vec<U, 3>& o) : x(wgsl_conv<T>(o.x)), y(wgsl_conv<T>(o.y)), z(wgsl_conv<T>(o.z)) {}
  vec<T, 2> xy() const { return {x, y}; }
  vec<T, 2> xz() const { return {x, z}; }
  vec<T, 3> xyz() const { return *this; }
  T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  const T& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

template <class T>
struct vec<T, 4> {
  T x, y, z, w;
  vec() : x(), y(), z(), w() {}
  explicit vec(T s) : x(s), y(s), z(s), w(s) {}
  vec(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
  vec(vec<T, 3> a, T d) : x(a.x), y(a.y), z(a.z), w(d) {}
  vec(vec<T, 2> a, T c, T d) : x(a.x), y(a.y), z(c), w(d) {}
  vec(vec<T, 2> a, vec<T, 2> b) : x(a.x), y(a.y), z(b.x), w(b.y) {}
  template <class U>
  explicit vec(const vec<U, 4>& o)
      : x(wgsl_conv<T>(o.x)), y(wgsl_conv<T>(o.y)), z(wgsl_conv<T>(o.z)), w(wgsl_conv<T>(o.w)) {}
  vec<T, 2> xy() const { return {x, y}; }
  vec<T, 2> xz() const { return {x, z}; }
  vec<T, 3> xyz() const { return {x, y, z}; }
  T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  const T& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};

using vec2f = vec<float, 2>;
using vec3f = vec<float, 3>;
using vec4f = vec<float, 4>;
using vec2i = vec<i32, 2>;
using vec3i = vec<i32, 3>;
using vec4i = vec<i32, 4>;
using vec2u = vec<u32, 2>;
using vec3u = vec<u32, 3>;
using vec4u = vec<u32, 4>;

// Component-wise application.
template <class T, int N, class F>
inline vec<T, N> cw(const vec<T, N>& a, F f) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r[i] = f(a[i]);
  return r;
}
template <class T, int N, class F>
inline vec<T, N> cw2(const vec<T, N>& a, const vec<T, N>& b, F f) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r[i] = f(a[i], b[i]);
  return r;
}

// Scalar operands of any arithmetic type convert to the vector's component
// type (WGSL's abstract literals take the type of the other operand).
#define WGSL_VEC_OP(op)                                                                      \
  template <class T, int N>                                                                  \
  inline vec<T, N> operator op(const vec<T, N>& a, const vec<T, N>& b) {                      \
    return cw2(a, b, [](T p, T q) { return p op q; });                                       \
  }                                                                                          \
  template <class T, int N, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>      \
  inline vec<T, N> operator op(const vec<T, N>& a, S s0) {                                   \
    const T s = (T)s0;                                                                       \
    return cw(a, [s](T p) { return p op s; });                                               \
  }                                                                                          \
  template <class T, int N, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>      \
  inline vec<T, N> operator op(S s0, const vec<T, N>& a) {                                   \
    const T s = (T)s0;                                                                       \
    return cw(a, [s](T p) { return s op p; });                                               \
  }                                                                                          \
  template <class T, int N>                                                                  \
  inline vec<T, N>& operator op##=(vec<T, N>& a, const vec<T, N>& b) { return a = a op b; }   \
  template <class T, int N, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>      \
  inline vec<T, N>& operator op##=(vec<T, N>& a, S s) { return a = a op s; }
WGSL_VEC_OP(+)
WGSL_VEC_OP(-)
WGSL_VEC_OP(*)
WGSL_VEC_OP(/)
#undef WGSL_VEC_OP

// Component-wise comparisons -> vec<bool, N>, reduced by all / any.
#define WGSL_VEC_CMP(op)                                                          \
  template <class T, int N>                                                       \
  inline vec<bool, N> operator op(const vec<T, N>& a, const vec<T, N>& b) {        \
    vec<bool, N> r;                                                               \
    for (int i = 0; i < N; ++i) r[i] = a[i] op b[i];                              \
    return r;                                                                     \
  }
WGSL_VEC_CMP(<)
WGSL_VEC_CMP(<=)
WGSL_VEC_CMP(>)
WGSL_VEC_CMP(>=)
WGSL_VEC_CMP(==)
WGSL_VEC_CMP(!=)
#undef WGSL_VEC_CMP
template <int N>
inline bool all(const vec<bool, N>& v) {
  for (int i = 0; i < N; ++i)
    if (!v[i]) return false;
  return true;
}
template <int N>
inline bool any(const vec<bool, N>& v) {
  for (int i = 0; i < N; ++i)
    if (v[i]) return true;
  return false;
}
inline bool all(bool b) { return b; }
inline bool any(bool b) { return b; }

// mat2x2<f32>: two columns; m * v sums column by column (c0 * v.x + c1 * v.y).
struct mat2x2f {
  vec2f c0, c1;
  mat2x2f(float a, float b, float c, float d) : c0(a, b), c1(c, d) {}
};
inline vec2f operator*(const mat2x2f& m, const vec2f& v) { return m.c0 * v.x + m.c1 * v.y; }

// mat3x3<f32>: three columns; m * v sums column by column.
struct mat3x3f {
  vec3f c[3];
  mat3x3f() = default;
  mat3x3f(vec3f a, vec3f b, vec3f d) : c{a, b, d} {}
  vec3f& operator[](int i) { return c[i]; }
  const vec3f& operator[](int i) const { return c[i]; }
};
inline vec3f operator*(const mat3x3f& m, const vec3f& v) { return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z; }

// mat4x4<f32>: four columns, laid out as the uniform buffer holds them.
struct mat4x4f {
  vec4f c[4];
};
inline vec4f operator*(const mat4x4f& m, const vec4f& v) {
  return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z + m.c[3] * v.w;
}

// texture_2d_array<f32> read with textureLoad (R32F layers of res x res
// texels, row-major): a texel outside the texture reads zero.
struct Tex2DArrayF {
  const float* p = nullptr;
  int32_t res = 0, layers = 0;
};
inline vec4f textureLoad(const Tex2DArrayF& t, vec<i32, 2> c, i32 layer, i32 /*mip*/) {
  if (!t.p || c.x < 0 || c.y < 0 || c.x >= t.res || c.y >= t.res || layer < 0 || layer >= t.layers)
    return vec4f(0.0f, 0.0f, 0.0f, 0.0f);
  return vec4f(t.p[((size_t)layer * t.res + (size_t)c.y) * t.res + (size_t)c.x], 0.0f, 0.0f, 1.0f);
}

// texture_2d<f32> and texture_storage_2d<rgba32float | r32float> over host
// images (w x h texels of `ch` floats, row-major).  Loads outside the image
// read zero, stores outside it are dropped.  textureSampleLevel samples the
// nearest texel with clamp-to-edge addressing, the reference's one sampler
// (nearest, clamp).
struct Tex2D {
  float* p = nullptr;
  int32_t w = 0, h = 0, ch = 4;
};
struct Sampler {};
inline vec4f tex_fetch(const Tex2D& t, i32 x, i32 y) {
  if (!t.p || x < 0 || y < 0 || x >= t.w || y >= t.h) return vec4f(0.0f, 0.0f, 0.0f, 0.0f);
  const float* q = t.p + ((size_t)y * t.w + (size_t)x) * t.ch;
  return t.ch == 4 ? vec4f(q[0], q[1], q[2], q[3]) : vec4f(q[0], 0.0f, 0.0f, 1.0f);
}
inline vec4f textureLoad(const Tex2D& t, vec<i32, 2> c, i32 /*mip*/) { return tex_fetch(t, c.x, c.y); }
inline vec4f textureLoad(const Tex2D& t, vec<u32, 2> c, i32 mip) { return textureLoad(t, vec<i32, 2>((i32)c.x, (i32)c.y), mip); }
inline void textureStore(Tex2D& t, vec<i32, 2> c, vec4f v) {
  if (!t.p || c.x < 0 || c.y < 0 || c.x >= t.w || c.y >= t.h) return;
  float* q = t.p + ((size_t)c.y * t.w + (size_t)c.x) * t.ch;
  q[0] = v.x;
  if (t.ch == 4) q[1] = v.y, q[2] = v.z, q[3] = v.w;
}
inline void textureStore(Tex2D& t, vec<u32, 2> c, vec4f v) { textureStore(t, vec<i32, 2>((i32)c.x, (i32)c.y), v); }
inline vec<u32, 2> textureDimensions(const Tex2D& t) { return vec<u32, 2>((u32)t.w, (u32)t.h); }
inline vec<u32, 2> textureDimensions(const Tex2D& t, i32 /*mip*/) { return textureDimensions(t); }
inline vec4f textureSampleLevel(const Tex2D& t, const Sampler&, vec2f uv, float /*lod*/) {
  const i32 x = wmin(wmax(wgsl_i32(std::floor(uv.x * (float)t.w)), (i32)0), (i32)(t.w - 1));
  const i32 y = wmin(wmax(wgsl_i32(std::floor(uv.y * (float)t.h)), (i32)0), (i32)(t.h - 1));
  return tex_fetch(t, x, y);
}

// A read-write storage buffer (array<T>): writes past the end are dropped.
template <class T>
struct RWBuf {
  T* p = nullptr;
  uint64_t n = 0;
  T sink{};
  T& operator[](uint64_t i) { return i < n ? p[i] : (sink = T{}); }
  T& operator[](uint32_t i) { return (*this)[(uint64_t)i]; }
  T& operator[](int32_t i) { return i >= 0 ? (*this)[(uint64_t)i] : (sink = T{}); }
};

// Workgroup atomics for a one-lane emulation of a workgroup (the tile's
// lane-0 work runs alone, so the barriers have nothing to wait for).
struct atomic_u32 {
  u32 v;
};
inline u32 atomicLoad(atomic_u32* a) { return a->v; }
inline void atomicStore(atomic_u32* a, u32 x) { a->v = x; }
inline u32 atomicAdd(atomic_u32* a, u32 x) {
  const u32 o = a->v;
  a->v = o + x;
  return o;
}
inline void workgroupBarrier() {}

// A read-only storage buffer (array<T>): an index past the end reads a zero
// record, as the oracle's checked reads do.
template <class T>
struct Buf {
  const T* p = nullptr;
  uint64_t n = 0;
  T operator[](uint64_t i) const { return i < n ? p[i] : T{}; }
  T operator[](int32_t i) const { return i >= 0 ? (*this)[(uint64_t)i] : T{}; }
  T operator[](uint32_t i) const { return (*this)[(uint64_t)i]; }
};

template <class T, int N>
inline vec<T, N> operator-(const vec<T, N>& a) {
  return cw(a, [](T p) { return -p; });
}

// Scalars (WGSL spellings).
inline float abs(float x) { return std::fabs(x); }
inline i32 abs(i32 x) { return x < 0 ? -x : x; }
inline float floor(float x) { return std::floor(x); }
inline float ceil(float x) { return std::ceil(x); }
inline float round(float x) { return std::nearbyint(x); }
inline float trunc(float x) { return std::trunc(x); }
inline float fract(float x) { return x - std::floor(x); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float inverseSqrt(float x) { return 1.0f / std::sqrt(x); }
inline float sin(float x) { return vxe_sinf(x); }
inline float cos(float x) { return vxe_cosf(x); }
inline float exp(float x) { return vxe_expf(x); }
inline float pow(float x, float y) { return vxe_powf(x, y); }
inline float min(float a, float b) { return wmin(a, b); }
inline float max(float a, float b) { return wmax(a, b); }
inline u32 min(u32 a, u32 b) { return wmin(a, b); }
inline u32 max(u32 a, u32 b) { return wmax(a, b); }
inline i32 min(i32 a, i32 b) { return wmin(a, b); }
inline i32 max(i32 a, i32 b) { return wmax(a, b); }
inline float clamp(float x, float lo, float hi) { return wmin(wmax(x, lo), hi); }
inline u32 clamp(u32 x, u32 lo, u32 hi) { return wmin(wmax(x, lo), hi); }
inline i32 clamp(i32 x, i32 lo, i32 hi) { return wmin(wmax(x, lo), hi); }
inline float mix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
inline float smoothstep(float e0, float e1, float x) {
  const float t = clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
inline float step(float edge, float x) { return x < edge ? 0.0f : 1.0f; }
inline float sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
inline float saturate(float x) { return clamp(x, 0.0f, 1.0f); }

// Vectors.
#define WGSL_VEC_FN1(name)                                                \
  template <class T, int N>                                               \
  inline vec<T, N> name(const vec<T, N>& a) {                             \
    return cw(a, [](T p) { return name(p); });                            \
  }
WGSL_VEC_FN1(abs)
WGSL_VEC_FN1(floor)
WGSL_VEC_FN1(ceil)
WGSL_VEC_FN1(round)
WGSL_VEC_FN1(trunc)
WGSL_VEC_FN1(fract)
WGSL_VEC_FN1(sqrt)
WGSL_VEC_FN1(sin)
WGSL_VEC_FN1(cos)
WGSL_VEC_FN1(exp)
WGSL_VEC_FN1(sign)
WGSL_VEC_FN1(saturate)
#undef WGSL_VEC_FN1

template <class T, int N>
inline vec<T, N> min(const vec<T, N>& a, const vec<T, N>& b) {
  return cw2(a, b, [](T p, T q) { return min(p, q); });
}
template <class T, int N>
inline vec<T, N> max(const vec<T, N>& a, const vec<T, N>& b) {
  return cw2(a, b, [](T p, T q) { return max(p, q); });
}
template <class T, int N>
inline vec<T, N> pow(const vec<T, N>& a, const vec<T, N>& b) {
  return cw2(a, b, [](T p, T q) { return pow(p, q); });
}
template <class T, int N>
inline vec<T, N> clamp(const vec<T, N>& x, const vec<T, N>& lo, const vec<T, N>& hi) {
  vec<T, N> r;
  for (int i = 0; i < N; ++i) r[i] = clamp(x[i], lo[i], hi[i]);
  return r;
}
template <class T, int N>
inline vec<T, N> clamp(const vec<T, N>& x, T lo, T hi) {
  return cw(x, [lo, hi](T p) { return clamp(p, lo, hi); });
}
template <int N>
inline vec<float, N> mix(const vec<float, N>& a, const vec<float, N>& b, float t) {
  vec<float, N> r;
  for (int i = 0; i < N; ++i) r[i] = mix(a[i], b[i], t);
  return r;
}
template <int N>
inline vec<float, N> mix(const vec<float, N>& a, const vec<float, N>& b, const vec<float, N>& t) {
  vec<float, N> r;
  for (int i = 0; i < N; ++i) r[i] = mix(a[i], b[i], t[i]);
  return r;
}
template <int N>
inline vec<float, N> smoothstep(float e0, float e1, const vec<float, N>& x) {
  return cw(x, [e0, e1](float p) { return smoothstep(e0, e1, p); });
}
template <int N>
inline vec<float, N> step(const vec<float, N>& e, const vec<float, N>& x) {
  return cw2(e, x, [](float p, float q) { return step(p, q); });
}
// dot sums left to right: ((a.x*b.x + a.y*b.y) + a.z*b.z) + a.w*b.w
template <class T, int N>
inline T dot(const vec<T, N>& a, const vec<T, N>& b) {
  T s = a[0] * b[0];
  for (int i = 1; i < N; ++i) s = s + a[i] * b[i];
  return s;
}
inline vec3f cross(const vec3f& a, const vec3f& b) {
  return vec3f(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <int N>
inline float length(const vec<float, N>& a) {
  return std::sqrt(dot(a, a));
}
template <int N>
inline vec<float, N> normalize(const vec<float, N>& a) {
  const float inv = 1.0f / std::sqrt(dot(a, a));
  return a * inv;
}
inline float length(float a) { return std::fabs(a); }

template <class T>
inline T wgsl_select(T f, T t, bool c) {
  return c ? t : f;
}

inline u32 countOneBits(u32 x) { return (u32)__builtin_popcount(x); }
inline u32 countLeadingZeros(u32 x) { return x == 0u ? 32u : (u32)__builtin_clz(x); }
inline u32 countTrailingZeros(u32 x) { return x == 0u ? 32u : (u32)__builtin_ctz(x); }
inline u32 firstLeadingBit(u32 x) { return x == 0u ? 0xFFFFFFFFu : 31u - (u32)__builtin_clz(x); }
inline u32 bitcast_u32(float f) {
  u32 u;
  std::memcpy(&u, &f, 4);
  return u;
}
inline u32 bitcast_u32(i32 i) { return (u32)i; }
inline i32 bitcast_i32(u32 u) { return (i32)u; }
inline i32 bitcast_i32(float f) {
  i32 i;
  std::memcpy(&i, &f, 4);
  return i;
}
inline float bitcast_f32(i32 i) {
  float f;
  std::memcpy(&f, &i, 4);
  return f;
}
inline float bitcast_f32(u32 u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

}  // namespace wgsl
