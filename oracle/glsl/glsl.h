// A GLSL 4.50 subset in C++, for running the reference's shader stages
// (shaders/cull.glsl, shaders/splat.glsl, shaders/gps.glsl,
// shaders/accum.glsl) on the CPU, one invocation at a time.
//
// TEST INFRASTRUCTURE ONLY: part of the oracle's checker; nothing in the
// product path includes or links it.
//
// What the shader source fixes is kept: every expression, its operand order
// and its float types.  What GLSL leaves to the implementation is defined
// here, each choice the one the oracle (gs_oracle.c) restates, so that a
// stage run through this header and the oracle can be compared bit for bit:
//   - float arithmetic is IEEE single precision, round to nearest even, no
//     contraction into FMA (compile with -ffp-contract=off);
//   - matrix-vector and matrix-matrix products sum their terms left to
//     right, column 0 first; dot() likewise;
//   - mix(x, y, a) = x * (1 - a) + y * a; clamp = min(max(x, lo), hi);
//     max(x, y) = x < y ? y : x and min(x, y) = y < x ? y : x (the
//     specification's definitions); fract(x) = x - floor(x);
//     normalize(v) = v / length(v), length(v) = sqrt(dot(v, v));
//     smoothstep by its specified Hermite formula;
//   - sqrt and division are correctly rounded; round() rounds half to even;
//   - exp, log and sin/cos are the oracle's deterministic functions
//     (oc_expf, oc_logf, oc_sincosf); exp2(x) = oc_expf(x * ln 2) and
//     log2(x) = oc_logf(x) * log2(e), as the oracle's display transform;
//     a stage's harness may declare another exp in the stage's namespace,
//     which hides this one;
//   - float to integer conversions truncate and saturate (NaN to 0), like
//     the GPU's cvt.rzi instructions;
//   - texture() with a non-filtering sampler returns the texel under the
//     coordinate (floor(uv * size), clamped to the edge).
#pragma once

#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>

extern "C" {
float oc_logf(float x);
float oc_expf(float x);
void oc_sincosf(float x, float* s, float* c);
float oc_half_to_float(uint16_t h);
}

namespace glsl {

typedef uint32_t uint;

// ---------------------------------------------------------------- conversions
inline uint u32_of(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint)x;
}
inline uint u32_of(int x) { return (uint)x; }
inline uint u32_of(uint x) { return x; }
inline uint u32_of(bool b) { return b ? 1u : 0u; }
uint u32_of(double) = delete;  // a double here means an unsuffixed literal slipped through

inline int i32_of(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return INT_MAX;
    if (x < -2147483648.0f) return INT_MIN;
    return (int)x;
}
inline int i32_of(int x) { return x; }
inline int i32_of(uint x) { return (int)x; }
inline int i32_of(bool b) { return b ? 1 : 0; }
int i32_of(double) = delete;

template <typename T> struct cv;
template <> struct cv<float> {
    static float of(float u) { return u; }
    static float of(int u) { return (float)u; }
    static float of(uint u) { return (float)u; }
};
template <> struct cv<int> {
    template <typename U> static int of(U u) { return i32_of(u); }
};
template <> struct cv<uint> {
    template <typename U> static uint of(U u) { return u32_of(u); }
};

// ------------------------------------------------------------------- swizzles
template <typename T> struct tvec2;
template <typename T> struct tvec3;
template <typename T> struct tvec4;
template <typename T, int K> struct vsel;
template <typename T> struct vsel<T, 2> { typedef tvec2<T> type; };
template <typename T> struct vsel<T, 3> { typedef tvec3<T> type; };
template <typename T> struct vsel<T, 4> { typedef tvec4<T> type; };

// A swizzle member of an N-component vector: reads build a vector of the
// selected components; writes (distinct components only) store them back.
template <typename T, int N, int... I> struct swz {
    T d[N];
    typedef typename vsel<T, (int)sizeof...(I)>::type V;
    operator V() const { return V(d[I]...); }
    swz& operator=(const V& v) {
        int k = 0;
        ((d[I] = v.d[k++]), ...);
        return *this;
    }
    swz& operator=(const swz& o) {
        const V t = o;
        return *this = t;
    }
};

// -------------------------------------------------------------------- vectors
template <typename T> struct tvec2 {
    union {
        T d[2];
        struct { T x, y; };
        struct { T r, g; };
        swz<T, 2, 0, 1> xy;
    };
    tvec2() : d{T(0), T(0)} {}
    explicit tvec2(T s) : d{s, s} {}
    tvec2(T a, T b) : d{a, b} {}
    tvec2(const tvec2& o) : d{o.d[0], o.d[1]} {}
    template <typename U> explicit tvec2(const tvec2<U>& o) : d{cv<T>::of(o.d[0]), cv<T>::of(o.d[1])} {}
    template <typename U> explicit tvec2(const tvec3<U>& o) : d{cv<T>::of(o.d[0]), cv<T>::of(o.d[1])} {}
    template <typename U> explicit tvec2(const tvec4<U>& o) : d{cv<T>::of(o.d[0]), cv<T>::of(o.d[1])} {}
    template <typename U, int N, int A, int B>
    explicit tvec2(const swz<U, N, A, B>& s) : d{cv<T>::of(s.d[A]), cv<T>::of(s.d[B])} {}
    tvec2& operator=(const tvec2& o) {
        d[0] = o.d[0];
        d[1] = o.d[1];
        return *this;
    }
    T& operator[](int i) { return d[i]; }
    T operator[](int i) const { return d[i]; }
};

template <typename T> struct tvec3 {
    union {
        T d[3];
        struct { T x, y, z; };
        struct { T r, g, b; };
        swz<T, 3, 0, 1> xy;
        swz<T, 3, 1, 2> yz;
        swz<T, 3, 0, 1, 2> xyz;
        swz<T, 3, 0, 1, 2> rgb;
        swz<T, 3, 1, 2, 0> yzx;
    };
    tvec3() : d{T(0), T(0), T(0)} {}
    explicit tvec3(T s) : d{s, s, s} {}
    tvec3(T a, T b, T c) : d{a, b, c} {}
    tvec3(const tvec2<T>& v, T c) : d{v.d[0], v.d[1], c} {}
    tvec3(T a, const tvec2<T>& v) : d{a, v.d[0], v.d[1]} {}
    tvec3(const tvec3& o) : d{o.d[0], o.d[1], o.d[2]} {}
    template <typename U>
    explicit tvec3(const tvec3<U>& o) : d{cv<T>::of(o.d[0]), cv<T>::of(o.d[1]), cv<T>::of(o.d[2])} {}
    template <typename U>
    explicit tvec3(const tvec4<U>& o) : d{cv<T>::of(o.d[0]), cv<T>::of(o.d[1]), cv<T>::of(o.d[2])} {}
    template <typename U, int N, int A, int B, int C>
    explicit tvec3(const swz<U, N, A, B, C>& s) : d{cv<T>::of(s.d[A]), cv<T>::of(s.d[B]), cv<T>::of(s.d[C])} {}
    tvec3& operator=(const tvec3& o) {
        d[0] = o.d[0];
        d[1] = o.d[1];
        d[2] = o.d[2];
        return *this;
    }
    T& operator[](int i) { return d[i]; }
    T operator[](int i) const { return d[i]; }
};

template <typename T> struct tvec4 {
    union {
        T d[4];
        struct { T x, y, z, w; };
        struct { T r, g, b, a; };
        swz<T, 4, 0, 1> xy;
        swz<T, 4, 2, 3> zw;
        swz<T, 4, 1, 2> yz;
        swz<T, 4, 0, 1, 2> xyz;
        swz<T, 4, 0, 1, 2> rgb;
    };
    tvec4() : d{T(0), T(0), T(0), T(0)} {}
    explicit tvec4(T s) : d{s, s, s, s} {}
    tvec4(T a, T b, T c, T e) : d{a, b, c, e} {}
    tvec4(const tvec3<T>& v, T e) : d{v.d[0], v.d[1], v.d[2], e} {}
    tvec4(const tvec2<T>& v, T c, T e) : d{v.d[0], v.d[1], c, e} {}
    tvec4(const tvec2<T>& v, const tvec2<T>& u) : d{v.d[0], v.d[1], u.d[0], u.d[1]} {}
    tvec4(const tvec4& o) : d{o.d[0], o.d[1], o.d[2], o.d[3]} {}
    template <typename U>
    explicit tvec4(const tvec4<U>& o)
        : d{cv<T>::of(o.d[0]), cv<T>::of(o.d[1]), cv<T>::of(o.d[2]), cv<T>::of(o.d[3])} {}
    tvec4& operator=(const tvec4& o) {
        std::memcpy(d, o.d, sizeof(d));
        return *this;
    }
    T& operator[](int i) { return d[i]; }
    T operator[](int i) const { return d[i]; }
};

typedef tvec2<float> vec2;
typedef tvec3<float> vec3;
typedef tvec4<float> vec4;
typedef tvec2<int> ivec2;
typedef tvec3<int> ivec3;
typedef tvec4<int> ivec4;
typedef tvec2<uint> uvec2;
typedef tvec3<uint> uvec3;
typedef tvec4<uint> uvec4;

// Component-wise operators, spelled out per type (non-template functions, so
// that swizzles convert to vectors in argument positions).
#define GLSL_VEC_ARITH(V, T, N)                                                                  \
    inline V operator+(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i]; return r; } \
    inline V operator-(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i]; return r; } \
    inline V operator*(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.d[i]; return r; } \
    inline V operator/(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] / b.d[i]; return r; } \
    inline V operator+(const V& a, T s) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + s; return r; }          \
    inline V operator-(const V& a, T s) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - s; return r; }          \
    inline V operator*(const V& a, T s) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * s; return r; }          \
    inline V operator/(const V& a, T s) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] / s; return r; }          \
    inline V operator+(T s, const V& a) { V r; for (int i = 0; i < N; ++i) r.d[i] = s + a.d[i]; return r; }          \
    inline V operator-(T s, const V& a) { V r; for (int i = 0; i < N; ++i) r.d[i] = s - a.d[i]; return r; }          \
    inline V operator*(T s, const V& a) { V r; for (int i = 0; i < N; ++i) r.d[i] = s * a.d[i]; return r; }          \
    inline V operator/(T s, const V& a) { V r; for (int i = 0; i < N; ++i) r.d[i] = s / a.d[i]; return r; }          \
    inline V operator-(const V& a) { V r; for (int i = 0; i < N; ++i) r.d[i] = -a.d[i]; return r; }                   \
    inline V& operator+=(V& a, const V& b) { return a = a + b; }                                                       \
    inline V& operator-=(V& a, const V& b) { return a = a - b; }                                                       \
    inline V& operator*=(V& a, const V& b) { return a = a * b; }                                                       \
    inline V& operator/=(V& a, const V& b) { return a = a / b; }                                                       \
    inline V& operator+=(V& a, T s) { return a = a + s; }                                                              \
    inline V& operator-=(V& a, T s) { return a = a - s; }                                                              \
    inline V& operator*=(V& a, T s) { return a = a * s; }                                                              \
    inline V& operator/=(V& a, T s) { return a = a / s; }

#define GLSL_VEC_BITS(V, T, N)                                                                                       \
    inline V operator^(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] ^ b.d[i]; return r; } \
    inline V operator|(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] | b.d[i]; return r; } \
    inline V operator&(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] & b.d[i]; return r; } \
    inline V operator>>(const V& a, T s) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] >> s; return r; }         \
    inline V operator<<(const V& a, T s) { V r; for (int i = 0; i < N; ++i) r.d[i] = a.d[i] << s; return r; }         \
    inline V& operator^=(V& a, const V& b) { return a = a ^ b; }                                                       \
    inline V& operator|=(V& a, const V& b) { return a = a | b; }                                                       \
    inline V& operator&=(V& a, const V& b) { return a = a & b; }

GLSL_VEC_ARITH(vec2, float, 2)
GLSL_VEC_ARITH(vec3, float, 3)
GLSL_VEC_ARITH(vec4, float, 4)
GLSL_VEC_ARITH(ivec2, int, 2)
GLSL_VEC_ARITH(ivec3, int, 3)
GLSL_VEC_ARITH(ivec4, int, 4)
GLSL_VEC_ARITH(uvec2, uint, 2)
GLSL_VEC_ARITH(uvec3, uint, 3)
GLSL_VEC_ARITH(uvec4, uint, 4)
GLSL_VEC_BITS(ivec2, int, 2)
GLSL_VEC_BITS(uvec2, uint, 2)
GLSL_VEC_BITS(uvec3, uint, 3)
GLSL_VEC_BITS(uvec4, uint, 4)
#undef GLSL_VEC_ARITH
#undef GLSL_VEC_BITS

// ------------------------------------------------------------------- matrices
// Column-major, m[c] is column c and m[c][r] its row r, as in GLSL.
struct mat4 {
    vec4 c[4];
    mat4() {}
    vec4& operator[](int i) { return c[i]; }
    const vec4& operator[](int i) const { return c[i]; }
};

struct mat3 {
    vec3 c[3];
    mat3() {}
    mat3(float a0, float a1, float a2, float a3, float a4, float a5, float a6, float a7, float a8)
        : c{vec3(a0, a1, a2), vec3(a3, a4, a5), vec3(a6, a7, a8)} {}
    mat3(const vec3& a, const vec3& b, const vec3& e) : c{a, b, e} {}
    explicit mat3(const mat4& m)
        : c{vec3(m.c[0].d[0], m.c[0].d[1], m.c[0].d[2]), vec3(m.c[1].d[0], m.c[1].d[1], m.c[1].d[2]),
            vec3(m.c[2].d[0], m.c[2].d[1], m.c[2].d[2])} {}
    vec3& operator[](int i) { return c[i]; }
    const vec3& operator[](int i) const { return c[i]; }
};

inline vec3 operator*(const mat3& m, const vec3& v) {
    vec3 r;
    for (int i = 0; i < 3; ++i) r.d[i] = (m.c[0].d[i] * v.d[0] + m.c[1].d[i] * v.d[1]) + m.c[2].d[i] * v.d[2];
    return r;
}
inline mat3 operator*(const mat3& a, const mat3& b) {
    mat3 r;
    for (int k = 0; k < 3; ++k) r.c[k] = a * b.c[k];
    return r;
}
inline mat3 operator-(const mat3& m) { return mat3(-m.c[0], -m.c[1], -m.c[2]); }
inline mat3 transpose(const mat3& m) {
    mat3 r;
    for (int c = 0; c < 3; ++c)
        for (int i = 0; i < 3; ++i) r.c[c].d[i] = m.c[i].d[c];
    return r;
}
inline vec4 operator*(const mat4& m, const vec4& v) {
    vec4 r;
    for (int i = 0; i < 4; ++i)
        r.d[i] = ((m.c[0].d[i] * v.d[0] + m.c[1].d[i] * v.d[1]) + m.c[2].d[i] * v.d[2]) + m.c[3].d[i] * v.d[3];
    return r;
}

// ------------------------------------------------------------------ built-ins
inline float min(float x, float y) { return y < x ? y : x; }
inline float max(float x, float y) { return x < y ? y : x; }
inline int min(int x, int y) { return y < x ? y : x; }
inline int max(int x, int y) { return x < y ? y : x; }
inline uint min(uint x, uint y) { return y < x ? y : x; }
inline uint max(uint x, uint y) { return x < y ? y : x; }
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline int clamp(int x, int lo, int hi) { return min(max(x, lo), hi); }
inline uint clamp(uint x, uint lo, uint hi) { return min(max(x, lo), hi); }
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
inline float abs(float x) { return std::fabs(x); }
inline float floor(float x) { return std::floor(x); }
inline float ceil(float x) { return std::ceil(x); }
inline float fract(float x) { return x - std::floor(x); }
inline float round(float x) { return std::rint(x); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float exp(float x) { return oc_expf(x); }
inline float log(float x) { return oc_logf(x); }
inline float exp2(float x) { return oc_expf(x * 0.6931471805599453f); }
inline float log2(float x) { return oc_logf(x) * 1.4426950216293335f; }
inline float sin(float x) {
    float s, c;
    oc_sincosf(x, &s, &c);
    return s;
}
inline float cos(float x) {
    float s, c;
    oc_sincosf(x, &s, &c);
    return c;
}
inline float step(float edge, float x) { return x < edge ? 0.0f : 1.0f; }
inline float smoothstep(float e0, float e1, float x) {
    const float t = clamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

#define GLSL_VEC_FN1(V, N, F)                                \
    inline V F(const V& a) {                                 \
        V r;                                                 \
        for (int i = 0; i < N; ++i) r.d[i] = F(a.d[i]);      \
        return r;                                            \
    }
#define GLSL_VEC_FNS(V, N)                                                                     \
    GLSL_VEC_FN1(V, N, floor) GLSL_VEC_FN1(V, N, ceil) GLSL_VEC_FN1(V, N, fract)               \
    GLSL_VEC_FN1(V, N, round) GLSL_VEC_FN1(V, N, abs) GLSL_VEC_FN1(V, N, sqrt)                 \
    GLSL_VEC_FN1(V, N, exp2) GLSL_VEC_FN1(V, N, log2)                                          \
    inline V min(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.d[i] = min(a.d[i], b.d[i]); return r; } \
    inline V max(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.d[i] = max(a.d[i], b.d[i]); return r; } \
    inline V min(const V& a, float s) { return min(a, V(s)); }                                \
    inline V max(const V& a, float s) { return max(a, V(s)); }                                \
    inline V clamp(const V& x, const V& lo, const V& hi) { return min(max(x, lo), hi); }      \
    inline V clamp(const V& x, float lo, float hi) { return min(max(x, V(lo)), V(hi)); }      \
    inline V mix(const V& x, const V& y, float a) { return x * (1.0f - a) + y * a; }          \
    inline V mix(const V& x, const V& y, const V& a) { return x * (1.0f - a) + y * a; }       \
    inline float dot(const V& a, const V& b) {                                                \
        float s = a.d[0] * b.d[0];                                                            \
        for (int i = 1; i < N; ++i) s = s + a.d[i] * b.d[i];                                  \
        return s;                                                                             \
    }                                                                                         \
    inline float length(const V& a) { return sqrt(dot(a, a)); }                               \
    inline float distance(const V& a, const V& b) { return length(a - b); }                   \
    inline V normalize(const V& a) { return a / length(a); }
GLSL_VEC_FNS(vec2, 2)
GLSL_VEC_FNS(vec3, 3)
GLSL_VEC_FNS(vec4, 4)
#undef GLSL_VEC_FNS
#undef GLSL_VEC_FN1

#define GLSL_IVEC_FNS(V, T, N)                                                                \
    inline V min(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.d[i] = min(a.d[i], b.d[i]); return r; } \
    inline V max(const V& a, const V& b) { V r; for (int i = 0; i < N; ++i) r.d[i] = max(a.d[i], b.d[i]); return r; } \
    inline V clamp(const V& x, const V& lo, const V& hi) { return min(max(x, lo), hi); }
GLSL_IVEC_FNS(ivec2, int, 2)
GLSL_IVEC_FNS(ivec3, int, 3)
GLSL_IVEC_FNS(uvec2, uint, 2)
#undef GLSL_IVEC_FNS

inline uint floatBitsToUint(float f) {
    uint u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float uintBitsToFloat(uint u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline int bitCount(uint v) { return __builtin_popcount(v); }
inline vec2 unpackHalf2x16(uint v) {
    return vec2(oc_half_to_float((uint16_t)(v & 0xFFFFu)), oc_half_to_float((uint16_t)(v >> 16)));
}

// Atomics: invocations run one after another, so each is a plain
// read-modify-write that returns the old value.
inline uint atomicAdd(uint& m, uint v) { const uint o = m; m = o + v; return o; }
inline uint atomicOr(uint& m, uint v) { const uint o = m; m = o | v; return o; }
inline uint atomicMin(uint& m, uint v) { const uint o = m; m = min(o, v); return o; }
inline uint atomicMax(uint& m, uint v) { const uint o = m; m = max(o, v); return o; }

// ------------------------------------------------------------------- textures
// A 2-D float texture: `channels` floats per texel, row y = 0 first (the
// bottom row in GL's window orientation).  A one-channel texture reads as
// (r, 0, 0, 1), as an R32F texture does.
struct texture2D {
    const float* data = nullptr;
    int width = 0, height = 0, channels = 4;
};
struct sampler {};
struct sampler2D {
    const texture2D* t;
    sampler2D(const texture2D& tex, const sampler&) : t(&tex) {}
};
inline ivec2 textureSize(const sampler2D& s, int) { return ivec2(s.t->width, s.t->height); }
inline vec4 texelFetch(const sampler2D& s, const ivec2& p, int) {
    const texture2D& t = *s.t;
    const float* q = t.data + ((size_t)p.y * (size_t)t.width + (size_t)p.x) * (size_t)t.channels;
    if (t.channels == 1) return vec4(q[0], 0.0f, 0.0f, 1.0f);
    return vec4(q[0], q[1], q[2], q[3]);
}
inline vec4 texture(const sampler2D& s, const vec2& uv) {
    const int x = clamp(i32_of(floor(uv.x * (float)s.t->width)), 0, s.t->width - 1);
    const int y = clamp(i32_of(floor(uv.y * (float)s.t->height)), 0, s.t->height - 1);
    return texelFetch(s, ivec2(x, y), 0);
}

}  // namespace glsl
