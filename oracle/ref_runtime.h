// ref_runtime.h — the WGSL types and built-in functions, on the CPU, for the
// reference's own shader code translated to C++ by oracle/wgsl_translate.py.
//
// TEST INFRASTRUCTURE ONLY (with ref_harness.cpp): it runs the reference's
// shader source itself, so that the oracle's hand restatement can be checked
// against it.  Nothing in the product library includes it.
//
// Semantics follow the WGSL specification where it fixes them; where it
// leaves the rounding to the implementation, the choice is the one the
// oracle makes, so that a difference between the two runs can only come
// from the shader code:
//  * arithmetic: IEEE binary32, every operation rounded on its own (the
//    translation units are built with -ffp-contract=off);
//  * pow(x, 2.0) is x * x (what shader compilers emit; undefined for x < 0
//    in SPIR-V), any other pow is powf; exp, sin, cos, tan, atan: libm's
//    float functions; sqrt correctly rounded;
//  * dot and matrix products sum their terms from the first component up;
//    normalize(v) = v / length(v); reflect, refract, clamp, sign and the
//    float remainder (e1 - e2 * trunc(e1 / e2)) as the specification writes
//    them;
//  * float -> integer conversions truncate and saturate;
//  * ray queries are answered by a callback (ref_harness.cpp answers them with
//    the oracle's FP64 query, the part a Vulkan driver answers in the
//    reference); atomics are real (relaxed) atomics, so a dispatch may run
//    its invocations on several threads, in which order they land then
//    varies as on a GPU; run one after another they give the sequential
//    order.
#ifndef SRT_REF_RUNTIME_H
#define SRT_REF_RUNTIME_H

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>

namespace wgsl_rt {

// ------------------------------------------------------------ scalar conversions
inline float f32c(float x) { return x; }
template <class T>
inline float f32c(T x) { return (float)x; }
inline int32_t to_i32(float x) {
    if (!(x == x)) return 0;
    if (x >= 2147483520.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}
inline uint32_t to_u32(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967040.0f) return UINT32_MAX;
    return (uint32_t)x;
}
template <class D, class S>
inline D conv(S x) {
    if constexpr (std::is_same_v<D, int32_t> && std::is_floating_point_v<S>) return to_i32((float)x);
    else if constexpr (std::is_same_v<D, uint32_t> && std::is_floating_point_v<S>) return to_u32((float)x);
    else return (D)x;
}

// ------------------------------------------------------------ vectors
template <class T, int N>
struct vec;

template <class T>
struct vec<T, 2> {
    T x{}, y{};
    vec() = default;
    vec(T a, T b) : x(a), y(b) {}
    template <class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>
    explicit vec(S s) : x((T)s), y((T)s) {}
    template <class U>
    explicit vec(const vec<U, 2>& o) : x(conv<T>(o.x)), y(conv<T>(o.y)) {}
    T& operator[](uint32_t i) { return i == 0 ? x : y; }
    T operator[](uint32_t i) const { return i == 0 ? x : y; }
    template <int... I>
    vec<T, (int)sizeof...(I)> sw() const { return vec<T, (int)sizeof...(I)>((*this)[I]...); }
};
template <class T>
struct vec<T, 3> {
    T x{}, y{}, z{};
    vec() = default;
    vec(T a, T b, T c) : x(a), y(b), z(c) {}
    template <class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>
    explicit vec(S s) : x((T)s), y((T)s), z((T)s) {}
    vec(const vec<T, 2>& a, T c) : x(a.x), y(a.y), z(c) {}
    template <class U>
    explicit vec(const vec<U, 3>& o) : x(conv<T>(o.x)), y(conv<T>(o.y)), z(conv<T>(o.z)) {}
    T& operator[](uint32_t i) { return i == 0 ? x : (i == 1 ? y : z); }
    T operator[](uint32_t i) const { return i == 0 ? x : (i == 1 ? y : z); }
    template <int... I>
    vec<T, (int)sizeof...(I)> sw() const { return vec<T, (int)sizeof...(I)>((*this)[I]...); }
};
template <class T>
struct vec<T, 4> {
    T x{}, y{}, z{}, w{};
    vec() = default;
    vec(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    template <class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>
    explicit vec(S s) : x((T)s), y((T)s), z((T)s), w((T)s) {}
    vec(const vec<T, 3>& a, T d) : x(a.x), y(a.y), z(a.z), w(d) {}
    vec(const vec<T, 2>& a, T c, T d) : x(a.x), y(a.y), z(c), w(d) {}
    template <class U>
    explicit vec(const vec<U, 4>& o) : x(conv<T>(o.x)), y(conv<T>(o.y)), z(conv<T>(o.z)), w(conv<T>(o.w)) {}
    T& operator[](uint32_t i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    T operator[](uint32_t i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    template <int... I>
    vec<T, (int)sizeof...(I)> sw() const { return vec<T, (int)sizeof...(I)>((*this)[I]...); }
};

using vec2f = vec<float, 2>;
using vec3f = vec<float, 3>;
using vec4f = vec<float, 4>;
using vec2u = vec<uint32_t, 2>;
using vec3u = vec<uint32_t, 3>;
using vec4u = vec<uint32_t, 4>;
using vec2i = vec<int32_t, 2>;
using vec3i = vec<int32_t, 3>;
using vec4i = vec<int32_t, 4>;
static_assert(sizeof(vec3f) == 12 && sizeof(vec4f) == 16, "vector layout");

template <class T, int N, class F>
inline vec<T, N> map2(const vec<T, N>& a, const vec<T, N>& b, F f) {
    vec<T, N> r;
    for (uint32_t i = 0; i < (uint32_t)N; ++i) r[i] = f(a[i], b[i]);
    return r;
}
template <class T, int N, class F>
inline vec<T, N> map1(const vec<T, N>& a, F f) {
    vec<T, N> r;
    for (uint32_t i = 0; i < (uint32_t)N; ++i) r[i] = f(a[i]);
    return r;
}

#define WGSL_VEC_OP(OP)                                                                          \
    template <class T, int N>                                                                    \
    inline vec<T, N> operator OP(const vec<T, N>& a, const vec<T, N>& b) {                       \
        return map2(a, b, [](T p, T q) { return (T)(p OP q); });                                 \
    }                                                                                            \
    template <class T, int N, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>        \
    inline vec<T, N> operator OP(const vec<T, N>& a, S s) {                                      \
        const T t = (T)s;                                                                        \
        return map1(a, [t](T p) { return (T)(p OP t); });                                        \
    }                                                                                            \
    template <class T, int N, class S, class = std::enable_if_t<std::is_arithmetic_v<S>>>        \
    inline vec<T, N> operator OP(S s, const vec<T, N>& a) {                                      \
        const T t = (T)s;                                                                        \
        return map1(a, [t](T p) { return (T)(t OP p); });                                        \
    }                                                                                            \
    template <class T, int N, class R>                                                           \
    inline vec<T, N>& operator OP##=(vec<T, N>& a, const R& b) {                                 \
        a = a OP b;                                                                              \
        return a;                                                                                \
    }
WGSL_VEC_OP(+)
WGSL_VEC_OP(-)
WGSL_VEC_OP(*)
WGSL_VEC_OP(/)
#undef WGSL_VEC_OP

template <class T, int N>
inline vec<T, N> operator-(const vec<T, N>& a) {
    return map1(a, [](T p) { return (T)(-p); });
}

// float remainder: e1 - e2 * trunc(e1 / e2)
inline float frem(float a, float b) { return a - b * std::trunc(a / b); }
template <int N>
inline vec<float, N> operator%(const vec<float, N>& a, float b) {
    return map1(a, [b](float p) { return frem(p, b); });
}
template <int N>
inline vec<float, N> operator%(const vec<float, N>& a, const vec<float, N>& b) {
    return map2(a, b, [](float p, float q) { return frem(p, q); });
}

// ------------------------------------------------------------ matrices (column-major)
template <int C, int R>
struct mat {
    vec<float, R> c[C];
    mat() = default;
    template <class... V, class = std::enable_if_t<sizeof...(V) == (size_t)C>>
    mat(const V&... cols) : c{cols...} {}
    vec<float, R>& operator[](uint32_t i) { return c[i]; }
    const vec<float, R>& operator[](uint32_t i) const { return c[i]; }
};
using mat3x3f = mat<3, 3>;
using mat4x4f = mat<4, 4>;
using mat4x3f = mat<4, 3>;
static_assert(sizeof(mat4x4f) == 64, "matrix layout");

// M * v: component r = M[0][r] v[0] + M[1][r] v[1] + ..., summed from the first column
template <int C, int R>
inline vec<float, R> operator*(const mat<C, R>& m, const vec<float, C>& v) {
    vec<float, R> out;
    for (uint32_t r = 0; r < (uint32_t)R; ++r) {
        float s = m.c[0][r] * v[0];
        for (uint32_t k = 1; k < (uint32_t)C; ++k) s = s + m.c[k][r] * v[k];
        out[r] = s;
    }
    return out;
}
// v * M: component c = dot(v, M[c])
template <int C, int R>
inline vec<float, C> operator*(const vec<float, R>& v, const mat<C, R>& m) {
    vec<float, C> out;
    for (uint32_t k = 0; k < (uint32_t)C; ++k) {
        float s = v[0] * m.c[k][0];
        for (uint32_t r = 1; r < (uint32_t)R; ++r) s = s + v[r] * m.c[k][r];
        out[k] = s;
    }
    return out;
}
// A * B: column j = A * B[j]
template <int K, int R, int C>
inline mat<C, R> operator*(const mat<K, R>& a, const mat<C, K>& b) {
    mat<C, R> out;
    for (uint32_t j = 0; j < (uint32_t)C; ++j) out.c[j] = a * b.c[j];
    return out;
}

// ------------------------------------------------------------ fixed arrays
template <class T, int N>
struct warr {
    T a[N];
    T& operator[](uint32_t i) { return a[i]; }
    const T& operator[](uint32_t i) const { return a[i]; }
};

// ------------------------------------------------------------ storage buffers and atomics
[[noreturn]] inline void oob(const char* what, uint64_t i, uint64_t n) {
    std::fprintf(stderr, "ref_runtime: %s index %llu out of %llu\n", what, (unsigned long long)i,
                 (unsigned long long)n);
    std::abort();
}
template <class T>
struct StorageArray {
    T* p = nullptr;
    uint32_t n = 0;
    T& operator[](uint32_t i) const {
        if (i >= n) oob("storage", i, n);
        return p[i];
    }
};
template <class T>
struct Atomic {
    T v{};
};
template <class T>
inline uint32_t wb_arrayLength(const StorageArray<T>* a) { return a->n; }
template <class T>
inline T wb_atomicAdd(Atomic<T>* a, T x) { return __atomic_fetch_add(&a->v, x, __ATOMIC_RELAXED); }
template <class T>
inline T wb_atomicLoad(Atomic<T>* a) { return __atomic_load_n(&a->v, __ATOMIC_RELAXED); }
template <class T>
inline T wb_atomicExchange(Atomic<T>* a, T x) { return __atomic_exchange_n(&a->v, x, __ATOMIC_RELAXED); }

// ------------------------------------------------------------ textures
struct texture_storage_2d {
    uint32_t w = 0, h = 0;
    uint8_t* rgba8 = nullptr;  // rgba8unorm, row-major
};
inline vec2u wb_textureDimensions(const texture_storage_2d& t) { return vec2u(t.w, t.h); }
inline uint8_t unorm8(float c) {
    const float x = c < 0.0f ? 0.0f : (c > 1.0f ? 1.0f : c);  // NaN -> 0
    return (uint8_t)std::nearbyint(x * 255.0f);
}
inline void wb_textureStore(texture_storage_2d& t, vec2u p, vec4f c) {
    if (p.x >= t.w || p.y >= t.h) return;
    uint8_t* o = t.rgba8 + 4 * ((size_t)p.y * t.w + p.x);
    o[0] = unorm8(c.x);
    o[1] = unorm8(c.y);
    o[2] = unorm8(c.z);
    o[3] = unorm8(c.w);
}

// ------------------------------------------------------------ ray queries
struct RayDesc {
    uint32_t flags;
    uint32_t cull_mask;
    float tmin;
    float tmax;
    vec3f origin;
    vec3f dir;
};
struct RayIntersection {
    uint32_t kind{};  // 0 none, 1 triangle
    float t{};
    uint32_t instance_custom_data{};
    uint32_t instance_index{};
    uint32_t sbt_record_offset{};
    uint32_t geometry_index{};
    uint32_t primitive_index{};
    vec2f barycentrics{};
    bool front_face{};
    mat4x3f object_to_world{};
    mat4x3f world_to_object{};
};
constexpr uint32_t RAY_FLAG_TERMINATE_ON_FIRST_HIT = 0x4u;
struct acceleration_structure {
    void* ctx = nullptr;
    void (*trace)(void* ctx, const RayDesc& d, RayIntersection& out) = nullptr;
};
struct ray_query {
    acceleration_structure* as = nullptr;
    RayDesc desc{};
    RayIntersection committed{};
};
inline void wb_rayQueryInitialize(ray_query* q, acceleration_structure& as, RayDesc d) {
    q->as = &as;
    q->desc = d;
    q->committed = RayIntersection{};
}
inline bool wb_rayQueryProceed(ray_query* q) {
    q->as->trace(q->as->ctx, q->desc, q->committed);  // opaque geometry: no candidates to confirm
    return false;
}
inline RayIntersection wb_rayQueryGetCommittedIntersection(ray_query* q) { return q->committed; }

// ------------------------------------------------------------ built-in functions
template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
inline T wb_max(T a, T b) { return a < b ? b : a; }
template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
inline T wb_min(T a, T b) { return b < a ? b : a; }
template <class T, int N>
inline vec<T, N> wb_max(const vec<T, N>& a, const vec<T, N>& b) {
    return map2(a, b, [](T p, T q) { return wb_max(p, q); });
}
template <class T, int N>
inline vec<T, N> wb_min(const vec<T, N>& a, const vec<T, N>& b) {
    return map2(a, b, [](T p, T q) { return wb_min(p, q); });
}
inline float wb_clamp(float e, float lo, float hi) { return wb_min(wb_max(e, lo), hi); }
template <int N>
inline vec<float, N> wb_clamp(const vec<float, N>& e, const vec<float, N>& lo, const vec<float, N>& hi) {
    return wb_min(wb_max(e, lo), hi);
}
inline float wb_abs(float x) { return std::fabs(x); }
template <int N>
inline vec<float, N> wb_abs(const vec<float, N>& a) { return map1(a, [](float p) { return std::fabs(p); }); }
inline float wb_sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
inline float wb_sqrt(float x) { return std::sqrt(x); }
inline float wb_exp(float x) { return std::exp(x); }
inline float wb_cos(float x) { return std::cos(x); }
inline float wb_sin(float x) { return std::sin(x); }
inline float wb_tan(float x) { return std::tan(x); }
inline float wb_atan(float x) { return std::atan(x); }
inline float wb_floor(float x) { return std::floor(x); }
template <int N>
inline vec<float, N> wb_floor(const vec<float, N>& a) { return map1(a, [](float p) { return std::floor(p); }); }
inline float wb_pow(float x, float y) { return y == 2.0f ? x * x : std::pow(x, y); }
template <int N>
inline float wb_dot(const vec<float, N>& a, const vec<float, N>& b) {
    float s = a[0] * b[0];
    for (uint32_t i = 1; i < (uint32_t)N; ++i) s = s + a[i] * b[i];
    return s;
}
template <int N>
inline float wb_length(const vec<float, N>& a) { return std::sqrt(wb_dot(a, a)); }
template <int N>
inline vec<float, N> wb_normalize(const vec<float, N>& a) { return a / wb_length(a); }
inline vec3f wb_cross(const vec3f& a, const vec3f& b) {
    return vec3f(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// e1 - 2 * dot(e2, e1) * e2
inline vec3f wb_reflect(const vec3f& e1, const vec3f& e2) { return e1 - 2.0f * wb_dot(e2, e1) * e2; }
// k = 1 - e3^2 (1 - dot(e2, e1)^2); 0 if k < 0, else e3 e1 - (e3 dot(e2, e1) + sqrt(k)) e2
inline vec3f wb_refract(const vec3f& e1, const vec3f& e2, float e3) {
    const float d = wb_dot(e2, e1);
    const float k = 1.0f - e3 * e3 * (1.0f - d * d);
    if (k < 0.0f) return vec3f(0.0f);
    return e3 * e1 - (e3 * d + std::sqrt(k)) * e2;
}
template <class T>
inline T wb_select(const T& f, const T& t, bool c) { return c ? t : f; }

// ------------------------------------------------------------ scalar constructors
inline float f32(float x) { return x; }
inline float f32(uint32_t x) { return (float)x; }
inline float f32(int32_t x) { return (float)x; }
inline uint32_t u32(uint32_t x) { return x; }
inline uint32_t u32(int32_t x) { return (uint32_t)x; }
inline uint32_t u32(float x) { return to_u32(x); }
inline uint32_t u32(bool x) { return x ? 1u : 0u; }
inline int32_t i32(int32_t x) { return x; }
inline int32_t i32(uint32_t x) { return (int32_t)x; }
inline int32_t i32(float x) { return to_i32(x); }

}  // namespace wgsl_rt

#endif
