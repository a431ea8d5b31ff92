// wgsl_rt.h — CPU runtime for WGSL compute shaders translated to C++ by
// oracle/wgsl2cpp.py.  TEST INFRASTRUCTURE ONLY: it exists so the reference's
// own shader sources (splat_backward.wgsl, splat_step.wgsl, splat_adc.wgsl,
// bezier_backward.wgsl, bezier_step.wgsl, bezier_adc.wgsl) can be executed on
// the host and used as the ground truth that pins the oracle restatement.
//
// Semantics follow the WGSL specification for the subset those shaders use:
//   * vecN<T> with swizzles, matNxM column-major (m[c][r] = column c, row r);
//   * f32 arithmetic in IEEE single precision, no FMA contraction (the build
//     recipe passes -ffp-contract=off);
//   * f32 -> i32/u32 conversion truncates toward zero and saturates;
//   * atomics are plain read-modify-writes: invocations of one workgroup run as
//     cooperative fibers on ONE host thread, switching only at
//     workgroupBarrier(), so no two invocations ever run at the same time;
//   * workgroup memory is zeroed at the start of every workgroup.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <type_traits>
#include <ucontext.h>
#include <utility>
#include <vector>

namespace wgsl {

using f32 = float;
using u32 = uint32_t;
using i32 = int32_t;

template <class T, int N> struct vec;

// member swizzle used by translated code: v.sw__<0,1,2>()  <=>  WGSL v.xyz
#define WGSL_SWZ                                                            \
  template <int... I> vec<T, (int)sizeof...(I)> sw__() const {              \
    vec<T, (int)sizeof...(I)> o;                                            \
    int k = 0;                                                              \
    ((o[k++] = (*this)[I]), ...);                                           \
    return o;                                                               \
  }

template <class T> struct vec<T, 2> {
  union { T x; T r; };
  union { T y; T g; };
  T& operator[](u32 i) { return i == 0 ? x : y; }
  const T& operator[](u32 i) const { return i == 0 ? x : y; }
  WGSL_SWZ
};
template <class T> struct vec<T, 3> {
  union { T x; T r; };
  union { T y; T g; };
  union { T z; T b; };
  T& operator[](u32 i) { return i == 0 ? x : (i == 1 ? y : z); }
  const T& operator[](u32 i) const { return i == 0 ? x : (i == 1 ? y : z); }
  WGSL_SWZ
};
template <class T> struct vec<T, 4> {
  union { T x; T r; };
  union { T y; T g; };
  union { T z; T b; };
  union { T w; T a; };
  T& operator[](u32 i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  const T& operator[](u32 i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  WGSL_SWZ
};

template <class X> struct is_vec : std::false_type {};
template <class T, int N> struct is_vec<vec<T, N>> : std::true_type {};

// ---- construction: flatten scalars and vectors into components -------------
template <class T, int N, class A>
inline void vput(vec<T, N>& v, int& k, const A& a) {
  if constexpr (is_vec<A>::value) {
    for (int i = 0; i < (int)sizeof(A) / (int)sizeof(a.x); ++i) v[k++] = (T)a[i];
  } else {
    v[k++] = (T)a;
  }
}
template <class T, int N, class... A>
inline vec<T, N> mk(const A&... a) {
  vec<T, N> v;
  if constexpr (sizeof...(A) == 0) {
    for (int i = 0; i < N; ++i) v[i] = T(0);
  } else if constexpr (sizeof...(A) == 1 && !(is_vec<A>::value || ...)) {
    T s = (T)(a, ...);
    for (int i = 0; i < N; ++i) v[i] = s;
  } else {
    int k = 0;
    (vput(v, k, a), ...);
  }
  return v;
}

using vec2f = vec<f32, 2>;
using vec3f = vec<f32, 3>;
using vec4f = vec<f32, 4>;
using vec2u = vec<u32, 2>;
using vec3u = vec<u32, 3>;
using vec4u = vec<u32, 4>;
using vec2i = vec<i32, 2>;
using vec3i = vec<i32, 3>;
using vec4i = vec<i32, 4>;

template <class... A> inline vec2f vec2f_(const A&... a) { return mk<f32, 2>(a...); }
template <class... A> inline vec3f vec3f_(const A&... a) { return mk<f32, 3>(a...); }
template <class... A> inline vec4f vec4f_(const A&... a) { return mk<f32, 4>(a...); }
template <class... A> inline vec2u vec2u_(const A&... a) { return mk<u32, 2>(a...); }
template <class... A> inline vec3u vec3u_(const A&... a) { return mk<u32, 3>(a...); }
template <class... A> inline vec4u vec4u_(const A&... a) { return mk<u32, 4>(a...); }
template <class... A> inline vec2i vec2i_(const A&... a) { return mk<i32, 2>(a...); }
template <class... A> inline vec3i vec3i_(const A&... a) { return mk<i32, 3>(a...); }
template <class... A> inline vec4i vec4i_(const A&... a) { return mk<i32, 4>(a...); }

// swizzle read: v.sw<0,1,2>()  <=>  v.xyz
template <int... I, class T, int N>
inline vec<T, (int)sizeof...(I)> sw(const vec<T, N>& v) {
  vec<T, (int)sizeof...(I)> o;
  int k = 0;
  ((o[k++] = v[I]), ...);
  return o;
}

// ---- arithmetic -------------------------------------------------------------
#define WGSL_VOP(op)                                                               \
  template <class T, int N> inline vec<T, N> operator op(vec<T, N> a, const vec<T, N>& b) { \
    for (int i = 0; i < N; ++i) a[i] = a[i] op b[i];                               \
    return a;                                                                      \
  }                                                                                \
  template <class T, int N, class S, class = std::enable_if_t<std::is_arithmetic<S>::value>> \
  inline vec<T, N> operator op(vec<T, N> a, S s) {                                 \
    for (int i = 0; i < N; ++i) a[i] = a[i] op (T)s;                               \
    return a;                                                                      \
  }                                                                                \
  template <class T, int N, class S, class = std::enable_if_t<std::is_arithmetic<S>::value>> \
  inline vec<T, N> operator op(S s, vec<T, N> a) {                                 \
    for (int i = 0; i < N; ++i) a[i] = (T)s op a[i];                               \
    return a;                                                                      \
  }                                                                                \
  template <class T, int N, class R> inline vec<T, N>& operator op##=(vec<T, N>& a, const R& b) { \
    a = a op b;                                                                    \
    return a;                                                                      \
  }
WGSL_VOP(+)
WGSL_VOP(-)
WGSL_VOP(*)
WGSL_VOP(/)
#undef WGSL_VOP
template <class T, int N> inline vec<T, N> operator-(vec<T, N> a) {
  for (int i = 0; i < N; ++i) a[i] = -a[i];
  return a;
}

struct mat4x4f {
  vec4f c[4];
  vec4f& operator[](u32 i) { return c[i]; }
  const vec4f& operator[](u32 i) const { return c[i]; }
};
inline vec4f operator*(const mat4x4f& m, const vec4f& v) {
  // WGSL: M * v = sum_k column_k * v[k]
  vec4f o;
  for (int r = 0; r < 4; ++r) o[r] = m.c[0][r] * v[0] + m.c[1][r] * v[1] + m.c[2][r] * v[2] + m.c[3][r] * v[3];
  return o;
}

// ---- fixed-size arrays -------------------------------------------------------
template <class T, unsigned long long N> struct warray {
  T d[N];
  T& operator[](u32 i) { return d[i]; }
  const T& operator[](u32 i) const { return d[i]; }
};
template <class T, unsigned long long N, class... A>
inline warray<T, N> mkarr(const A&... a) {
  warray<T, N> r{};
  if constexpr (sizeof...(A) > 0) {
    T tmp[] = {(T)a...};
    for (unsigned long long i = 0; i < sizeof...(A); ++i) r.d[i] = tmp[i];
  }
  return r;
}

// ---- conversions ---------------------------------------------------------------
template <class A> inline f32 f32_(A a) { return (f32)a; }
inline i32 i32_(f32 a) {
  if (std::isnan(a)) return 0;
  if (a >= 2147483520.0f) return 2147483520;  // largest f32 below 2^31
  if (a <= -2147483648.0f) return INT32_MIN;
  return (i32)a;
}
inline i32 i32_(u32 a) { return (i32)a; }
inline i32 i32_(i32 a) { return a; }
inline u32 u32_(f32 a) {
  if (std::isnan(a) || a <= 0.0f) return 0u;
  if (a >= 4294967040.0f) return 4294967040u;
  return (u32)a;
}
inline u32 u32_(i32 a) { return (u32)a; }
inline u32 u32_(u32 a) { return a; }
inline bool bool_(bool a) { return a; }

// ---- builtins -------------------------------------------------------------------
template <class F, class T> inline auto select(const F& f, const T& t, bool c) -> F { return c ? (F)t : f; }
// component-wise comparison and selection
#define WGSL_VCMP(OP)                                                                             \
  template <class T, int N> inline vec<bool, N> operator OP(const vec<T, N>& a, const vec<T, N>& b) { \
    vec<bool, N> o;                                                                               \
    for (int i = 0; i < N; ++i) o[i] = a[i] OP b[i];                                              \
    return o;                                                                                     \
  }
WGSL_VCMP(>)
WGSL_VCMP(<)
WGSL_VCMP(>=)
WGSL_VCMP(<=)
#undef WGSL_VCMP
template <class T, int N> inline vec<T, N> select(const vec<T, N>& f, const vec<T, N>& t, const vec<bool, N>& c) {
  vec<T, N> o;
  for (int i = 0; i < N; ++i) o[i] = c[i] ? t[i] : f[i];
  return o;
}

inline f32 min(f32 a, f32 b) { return std::fmin(a, b); }
inline f32 max(f32 a, f32 b) { return std::fmax(a, b); }
inline u32 min(u32 a, u32 b) { return a < b ? a : b; }
inline u32 max(u32 a, u32 b) { return a > b ? a : b; }
inline i32 min(i32 a, i32 b) { return a < b ? a : b; }
inline i32 max(i32 a, i32 b) { return a > b ? a : b; }
template <class T, int N> inline vec<T, N> min(vec<T, N> a, const vec<T, N>& b) {
  for (int i = 0; i < N; ++i) a[i] = min(a[i], b[i]);
  return a;
}
template <class T, int N> inline vec<T, N> max(vec<T, N> a, const vec<T, N>& b) {
  for (int i = 0; i < N; ++i) a[i] = max(a[i], b[i]);
  return a;
}
inline f32 clamp(f32 e, f32 lo, f32 hi) { return min(max(e, lo), hi); }
inline u32 clamp(u32 e, u32 lo, u32 hi) { return min(max(e, lo), hi); }
inline i32 clamp(i32 e, i32 lo, i32 hi) { return min(max(e, lo), hi); }
template <class T, int N> inline vec<T, N> clamp(vec<T, N> e, const vec<T, N>& lo, const vec<T, N>& hi) {
  for (int i = 0; i < N; ++i) e[i] = clamp(e[i], lo[i], hi[i]);
  return e;
}
inline f32 abs(f32 a) { return std::fabs(a); }
inline f32 sqrt(f32 a) { return std::sqrt(a); }
inline f32 exp(f32 a) { return std::exp(a); }
inline f32 log(f32 a) { return std::log(a); }
inline f32 pow(f32 a, f32 b) { return std::pow(a, b); }
template <int N> inline vec<f32, N> pow(vec<f32, N> a, const vec<f32, N>& b) {
  for (int i = 0; i < N; ++i) a[i] = std::pow(a[i], b[i]);
  return a;
}
inline f32 sin(f32 a) { return std::sin(a); }
inline f32 cos(f32 a) { return std::cos(a); }
inline f32 floor(f32 a) { return std::floor(a); }
inline f32 fract(f32 a) { return a - std::floor(a); }
inline f32 step(f32 edge, f32 x) { return edge <= x ? 1.0f : 0.0f; }
inline f32 smoothstep(f32 lo, f32 hi, f32 x) {
  f32 t = clamp((x - lo) / (hi - lo), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
template <class T, int N> inline T dot(const vec<T, N>& a, const vec<T, N>& b) {
  T s = a[0] * b[0];
  for (int i = 1; i < N; ++i) s = s + a[i] * b[i];
  return s;
}
template <class T, int N> inline vec<T, N> abs(vec<T, N> a) {
  for (int i = 0; i < N; ++i) a[i] = abs(a[i]);
  return a;
}
inline f32 atan2(f32 y, f32 x) { return std::atan2(y, x); }
inline f32 asin(f32 a) { return std::asin(a); }
inline f32 acos(f32 a) { return std::acos(a); }
inline f32 atan(f32 a) { return std::atan(a); }
inline f32 tan(f32 a) { return std::tan(a); }
inline f32 sign(f32 a) { return a > 0.0f ? 1.0f : (a < 0.0f ? -1.0f : 0.0f); }
template <int N> inline vec<f32, N> normalize(const vec<f32, N>& a) { return a * (1.0f / std::sqrt(dot(a, a))); }
template <int N> inline vec<f32, N> reflect(const vec<f32, N>& e, const vec<f32, N>& n) {
  return e - 2.0f * dot(n, e) * n;
}
// bitcast<T>(x) between 32-bit scalar types
template <class T, class S> inline T bitcast(const S& s) {
  static_assert(sizeof(T) == sizeof(S), "bitcast between 32-bit scalars");
  T t;
  std::memcpy(&t, &s, sizeof t);
  return t;
}
inline vec3f cross(const vec3f& a, const vec3f& b) {
  vec3f o;
  o.x = a.y * b.z - a.z * b.y;
  o.y = a.z * b.x - a.x * b.z;
  o.z = a.x * b.y - a.y * b.x;
  return o;
}
template <int N> inline f32 length(const vec<f32, N>& a) { return std::sqrt(dot(a, a)); }
inline f32 length(f32 a) { return std::fabs(a); }
inline u32 countTrailingZeros(u32 v) { return v == 0 ? 32u : (u32)__builtin_ctz(v); }

// atomics: invocations never run concurrently (see header), so plain RMW.
inline i32 atomicAdd(i32* p, i32 v) { i32 o = *p; *p = (i32)((u32)o + (u32)v); return o; }
inline u32 atomicAdd(u32* p, u32 v) { u32 o = *p; *p = o + v; return o; }
inline u32 atomicOr(u32* p, u32 v) { u32 o = *p; *p = o | v; return o; }
inline i32 atomicExchange(i32* p, i32 v) { i32 o = *p; *p = v; return o; }
template <class T> inline T atomicLoad(T* p) { return *p; }
template <class T, class V> inline void atomicStore(T* p, V v) { *p = (T)v; }

// ---- textures (texture_2d<f32>, level 0 only) -------------------------------------
struct texture_2d {
  const float* rgba = nullptr;  // H*W*4 floats, row-major, y = 0 is the top row
  u32 w = 0, h = 0;
};
template <class C> inline vec4f textureLoad(const texture_2d& t, const C& c, int) {
  i32 x = (i32)c.x, y = (i32)c.y;
  vec4f o = mk<f32, 4>(0.0f);
  if (x < 0 || y < 0 || x >= (i32)t.w || y >= (i32)t.h) return o;
  const float* p = t.rgba + ((size_t)y * t.w + (size_t)x) * 4;
  o.x = p[0]; o.y = p[1]; o.z = p[2]; o.w = p[3];
  return o;
}
inline vec2u textureDimensions(const texture_2d& t) { vec2u o; o.x = t.w; o.y = t.h; return o; }
// texture_storage_2d<..., write>: textureStore keeps the float value handed to
// it (the format conversion, e.g. rgba8unorm, is applied by the caller)
struct texture_storage_2d {
  float* rgba = nullptr;  // H*W*4 floats
  u32 w = 0, h = 0;
};
template <class C> inline void textureStore(const texture_storage_2d& t, const C& c, const vec4f& v) {
  i32 x = (i32)c.x, y = (i32)c.y;
  if (x < 0 || y < 0 || x >= (i32)t.w || y >= (i32)t.h) return;
  float* p = t.rgba + ((size_t)y * t.w + (size_t)x) * 4;
  p[0] = v.x; p[1] = v.y; p[2] = v.z; p[3] = v.w;
}
inline vec2u textureDimensions(const texture_storage_2d& t) { vec2u o; o.x = t.w; o.y = t.h; return o; }

// runtime-sized array<T> bound to a storage buffer: indexes the buffer itself
template <class T> struct rtarray {
  T& operator[](u32 i) { return reinterpret_cast<T*>(this)[i]; }
  const T& operator[](u32 i) const { return reinterpret_cast<const T*>(this)[i]; }
};
// sampler + textureSampleLevel (level 0): WebGPU's filtering with nearest or
// linear magnification and the repeat / clamp-to-edge address modes; the
// bilinear weights are exact f32 fractions
enum { ADDRESS_CLAMP = 0, ADDRESS_REPEAT = 1 };
struct sampler {
  int linear = 1;
  int address_u = ADDRESS_CLAMP, address_v = ADDRESS_CLAMP;
};
inline i32 address_texel(i32 i, i32 n, int mode) {
  if (mode == ADDRESS_REPEAT) {
    i32 r = i % n;
    return r < 0 ? r + n : r;
  }
  return i < 0 ? 0 : (i >= n ? n - 1 : i);
}
inline f32 address_coord(f32 u, int mode) { return mode == ADDRESS_REPEAT ? u - std::floor(u) : u; }
inline vec4f texel(const texture_2d& t, i32 x, i32 y) {
  const float* p = t.rgba + ((size_t)y * t.w + (size_t)x) * 4;
  vec4f o;
  o.x = p[0]; o.y = p[1]; o.z = p[2]; o.w = p[3];
  return o;
}
inline vec4f textureSampleLevel(const texture_2d& t, const sampler& s, const vec2f& uv, f32) {
  const i32 w = (i32)t.w, h = (i32)t.h;
  const f32 u = address_coord(uv.x, s.address_u) * (f32)w, v = address_coord(uv.y, s.address_v) * (f32)h;
  if (!s.linear) {
    const i32 x = address_texel((i32)std::floor(u), w, s.address_u);
    const i32 y = address_texel((i32)std::floor(v), h, s.address_v);
    return texel(t, x, y);
  }
  const f32 fx = u - 0.5f, fy = v - 0.5f;
  const f32 x0f = std::floor(fx), y0f = std::floor(fy);
  const f32 ax = fx - x0f, ay = fy - y0f;
  const i32 x0 = address_texel((i32)x0f, w, s.address_u), x1 = address_texel((i32)x0f + 1, w, s.address_u);
  const i32 y0 = address_texel((i32)y0f, h, s.address_v), y1 = address_texel((i32)y0f + 1, h, s.address_v);
  const vec4f a = texel(t, x0, y0), b = texel(t, x1, y0), c = texel(t, x0, y1), d = texel(t, x1, y1);
  vec4f o;
  for (int i = 0; i < 4; ++i) {
    const f32 top = a[i] + (b[i] - a[i]) * ax, bot = c[i] + (d[i] - c[i]) * ax;
    o[i] = top + (bot - top) * ay;
  }
  return o;
}

// textureSample (implicit level of detail): the textures bound here have one
// level, so it samples level 0
inline vec4f textureSample(const texture_2d& t, const sampler& s, const vec2f& uv) {
  return textureSampleLevel(t, s, uv, 0.0f);
}

// ---- workgroup execution with fibers ------------------------------------------------
struct FiberPool {
  ucontext_t sched;
  std::vector<ucontext_t> ctx;
  std::vector<char*> stacks;
  std::vector<int> done;
  int cur = -1;
  size_t stack_bytes = 512 * 1024;
  ~FiberPool() { for (char* s : stacks) std::free(s); }
};
inline FiberPool& pool() { static FiberPool p; return p; }
inline void workgroupBarrier() {
  FiberPool& p = pool();
  swapcontext(&p.ctx[p.cur], &p.sched);
}
inline void storageBarrier() { workgroupBarrier(); }

using EntryFn = void (*)(vec3u gid, vec3u wid, vec3u lid, u32 lidx, vec3u nwg);
struct Launch {
  EntryFn fn;
  vec3u wid, wgsize, nwg;
};
inline Launch& launch() { static Launch l; return l; }
inline void fiber_main(int idx) {
  Launch& L = launch();
  u32 lx = (u32)idx % L.wgsize.x, ly = ((u32)idx / L.wgsize.x) % L.wgsize.y, lz = (u32)idx / (L.wgsize.x * L.wgsize.y);
  vec3u lid = mk<u32, 3>(lx, ly, lz);
  vec3u gid = mk<u32, 3>(L.wid.x * L.wgsize.x + lx, L.wid.y * L.wgsize.y + ly, L.wid.z * L.wgsize.z + lz);
  L.fn(gid, L.wid, lid, (u32)idx, L.nwg);
  pool().done[idx] = 1;
  // returning ends the fiber; uc_link brings control back to the scheduler
}
// Runs every invocation of workgroup `wid` to completion.
inline void run_workgroup(EntryFn fn, vec3u wid, vec3u wgsize, vec3u nwg) {
  FiberPool& p = pool();
  int n = (int)(wgsize.x * wgsize.y * wgsize.z);
  if ((int)p.ctx.size() < n) {
    p.ctx.resize(n);
    while ((int)p.stacks.size() < n) p.stacks.push_back((char*)std::malloc(p.stack_bytes));
  }
  p.done.assign(n, 0);
  Launch& L = launch();
  L.fn = fn; L.wid = wid; L.wgsize = wgsize; L.nwg = nwg;
  for (int i = 0; i < n; ++i) {
    getcontext(&p.ctx[i]);
    p.ctx[i].uc_stack.ss_sp = p.stacks[i];
    p.ctx[i].uc_stack.ss_size = p.stack_bytes;
    p.ctx[i].uc_link = &p.sched;
    makecontext(&p.ctx[i], (void (*)())fiber_main, 1, i);
  }
  bool any = true;
  while (any) {
    any = false;
    for (int i = 0; i < n; ++i) {
      if (p.done[i]) continue;
      p.cur = i;
      swapcontext(&p.sched, &p.ctx[i]);
      if (!p.done[i]) any = true;
    }
  }
}

}  // namespace wgsl
