// shim.h -- the HLSL types and intrinsics the reference's shaders use, in C++.
//
// TEST INFRASTRUCTURE: with this header, the reference's own shader sources
// (rewritten only syntactically by oracle/hlsl2cpp.py) compile on the host
// into oracle/_ref/, which then checks the oracle's restatement.
//
// What HLSL leaves to the implementation is fixed here to the conventions the
// oracle and the CUDA kernels share: one IEEE single-precision rounding per
// operation and no fused multiply-add (build with -ffp-contract=off);
// dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z; cross is the textbook formula;
// normalize(v) = v * (1/sqrt(dot(v, v))); length(v) = sqrt(dot(v, v));
// min/max/clamp/saturate are fminf/fmaxf (a NaN operand yields the other);
// mul(M, v) sums each row's products left to right; sin/cos/acos are the
// project's own (oracle/own_math.h).  Matrices in buffers are the
// column-major glm layout the reference uploads (element (r, c) at
// m[c*4 + r]); float3x3 values are held by rows.
//
// Buffers are bounds-checked: an out-of-range read returns a zeroed element
// and sets ref_ub (thread-local), so a caller can tell which results passed
// through an access whose result the reference leaves undefined.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../own_math.h"

typedef uint32_t uint;

extern thread_local int ref_ub;

template <class T> struct V2;
template <class T> struct V3;
template <class T> struct V4;

// A read/write view of three components of a vector (.xyz, .rgb).
template <class T> struct Swz3 : V3<T> {
    T* p;
    Swz3(T* q) : V3<T>(q[0], q[1], q[2]), p(q) {}
    Swz3& operator=(const V3<T>& v)
    {
        p[0] = v.x; p[1] = v.y; p[2] = v.z;
        this->x = v.x; this->y = v.y; this->z = v.z;
        return *this;
    }
};
template <class T> struct Swz2 : V2<T> {
    T* p;
    Swz2(T* q) : V2<T>(q[0], q[1]), p(q) {}
    Swz2& operator=(const V2<T>& v)
    {
        p[0] = v.x; p[1] = v.y;
        this->x = v.x; this->y = v.y;
        return *this;
    }
};

#define SHIM_VEC_OPS(VT, N)                                                                             \
    friend VT operator+(const VT& a, const VT& b) { VT r; for (int i = 0; i < N; ++i) r[i] = a[i] + b[i]; return r; } \
    friend VT operator-(const VT& a, const VT& b) { VT r; for (int i = 0; i < N; ++i) r[i] = a[i] - b[i]; return r; } \
    friend VT operator*(const VT& a, const VT& b) { VT r; for (int i = 0; i < N; ++i) r[i] = a[i] * b[i]; return r; } \
    friend VT operator/(const VT& a, const VT& b) { VT r; for (int i = 0; i < N; ++i) r[i] = a[i] / b[i]; return r; } \
    friend VT operator+(const VT& a, T s) { VT r; for (int i = 0; i < N; ++i) r[i] = a[i] + s; return r; }        \
    friend VT operator-(const VT& a, T s) { VT r; for (int i = 0; i < N; ++i) r[i] = a[i] - s; return r; }        \
    friend VT operator*(const VT& a, T s) { VT r; for (int i = 0; i < N; ++i) r[i] = a[i] * s; return r; }        \
    friend VT operator/(const VT& a, T s) { VT r; for (int i = 0; i < N; ++i) r[i] = a[i] / s; return r; }        \
    friend VT operator+(T s, const VT& a) { VT r; for (int i = 0; i < N; ++i) r[i] = s + a[i]; return r; }        \
    friend VT operator-(T s, const VT& a) { VT r; for (int i = 0; i < N; ++i) r[i] = s - a[i]; return r; }        \
    friend VT operator*(T s, const VT& a) { VT r; for (int i = 0; i < N; ++i) r[i] = s * a[i]; return r; }        \
    friend VT operator/(T s, const VT& a) { VT r; for (int i = 0; i < N; ++i) r[i] = s / a[i]; return r; }        \
    friend VT operator-(const VT& a) { VT r; for (int i = 0; i < N; ++i) r[i] = -a[i]; return r; }                 \
    VT& operator+=(const VT& b) { for (int i = 0; i < N; ++i) (*this)[i] = (*this)[i] + b[i]; return *this; }     \
    VT& operator-=(const VT& b) { for (int i = 0; i < N; ++i) (*this)[i] = (*this)[i] - b[i]; return *this; }     \
    VT& operator*=(const VT& b) { for (int i = 0; i < N; ++i) (*this)[i] = (*this)[i] * b[i]; return *this; }     \
    VT& operator/=(const VT& b) { for (int i = 0; i < N; ++i) (*this)[i] = (*this)[i] / b[i]; return *this; }     \
    VT& operator*=(T s) { for (int i = 0; i < N; ++i) (*this)[i] = (*this)[i] * s; return *this; }               \
    VT& operator/=(T s) { for (int i = 0; i < N; ++i) (*this)[i] = (*this)[i] / s; return *this; }               \
    T& operator[](int i) { return (&x)[i]; }                                                                      \
    const T& operator[](int i) const { return (&x)[i]; }

#define SHIM_VEC_CMP(VT, BT, N)                                                                                   \
    friend BT operator<(const VT& a, const VT& b) { BT r; for (int i = 0; i < N; ++i) r[i] = a[i] < b[i]; return r; }   \
    friend BT operator>(const VT& a, const VT& b) { BT r; for (int i = 0; i < N; ++i) r[i] = a[i] > b[i]; return r; }   \
    friend BT operator<=(const VT& a, const VT& b) { BT r; for (int i = 0; i < N; ++i) r[i] = a[i] <= b[i]; return r; } \
    friend BT operator>=(const VT& a, const VT& b) { BT r; for (int i = 0; i < N; ++i) r[i] = a[i] >= b[i]; return r; }

template <class T> struct V2 {
    union { struct { T x, y; }; struct { T r, g; }; };
    V2() : x(T(0)), y(T(0)) {}
    V2(T s) : x(s), y(s) {}
    V2(T a, T b) : x(a), y(b) {}
    template <class U> V2(const V2<U>& o) : x(T(o.x)), y(T(o.y)) {}
    Swz2<T> xy() { return Swz2<T>(&x); }
    SHIM_VEC_OPS(V2, 2)
    SHIM_VEC_CMP(V2, V2<bool>, 2)
};

template <class T> struct V3 {
    union { struct { T x, y, z; }; struct { T r, g, b; }; };
    V3() : x(T(0)), y(T(0)), z(T(0)) {}
    V3(T s) : x(s), y(s), z(s) {}
    V3(T a, T b, T c) : x(a), y(b), z(c) {}
    V3(const V2<T>& v, T c) : x(v.x), y(v.y), z(c) {}
    template <class U> V3(const V3<U>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
    Swz2<T> xy() { return Swz2<T>(&x); }
    Swz3<T> xyz() { return Swz3<T>(&x); }
    Swz3<T> rgb() { return Swz3<T>(&x); }
    SHIM_VEC_OPS(V3, 3)
    SHIM_VEC_CMP(V3, V3<bool>, 3)
};

template <class T> struct V4 {
    union { struct { T x, y, z, w; }; struct { T r, g, b, a; }; };
    V4() : x(T(0)), y(T(0)), z(T(0)), w(T(0)) {}
    V4(T s) : x(s), y(s), z(s), w(s) {}
    V4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    V4(const V3<T>& v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
    V4(const V2<T>& v, T c, T d) : x(v.x), y(v.y), z(c), w(d) {}
    template <class U> V4(const V4<U>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)), w(T(o.w)) {}
    Swz2<T> xy() { return Swz2<T>(&x); }
    Swz3<T> xyz() { return Swz3<T>(&x); }
    Swz3<T> rgb() { return Swz3<T>(&x); }
    SHIM_VEC_OPS(V4, 4)
};

typedef V2<float> float2;
typedef V3<float> float3;
typedef V4<float> float4;
typedef V2<int> int2;
typedef V3<int> int3;
typedef V2<uint> uint2;
typedef V3<uint> uint3;
typedef V2<bool> bool2;
typedef V3<bool> bool3;

static_assert(sizeof(float3) == 12 && sizeof(float4) == 16 && sizeof(int2) == 8, "vector layout");

// mixed-type arithmetic the shaders use (HLSL promotes the integer vector to
// float, and a signed operand of a comparison with an unsigned one to
// unsigned)
inline float2 operator+(const uint2& a, float s) { return float2(float(a.x) + s, float(a.y) + s); }
inline bool2 operator>=(const uint2& a, const int2& b) { return bool2(a.x >= (uint)b.x, a.y >= (uint)b.y); }

// Row-held 3x3 matrix value (float3x3(a, b, c) has rows a, b, c).
struct float4x4;
struct float3x3 {
    float3 r0, r1, r2;
    float3x3() {}
    float3x3(const float3& a, const float3& b, const float3& c) : r0(a), r1(b), r2(c) {}
    explicit float3x3(const float4x4& m);
    float3& operator[](int i) { return i == 0 ? r0 : (i == 1 ? r1 : r2); }
    const float3& operator[](int i) const { return i == 0 ? r0 : (i == 1 ? r1 : r2); }
};

// 4x4 matrix in the buffer layout: column-major, element (r, c) at m[c*4 + r].
struct float4x4 {
    float m[16];
    float4x4() { memset(m, 0, sizeof(m)); }
    float at(int r, int c) const { return m[c * 4 + r]; }
};
static_assert(sizeof(float4x4) == 64, "matrix layout");

inline float3x3::float3x3(const float4x4& M)
    : r0(M.at(0, 0), M.at(0, 1), M.at(0, 2)), r1(M.at(1, 0), M.at(1, 1), M.at(1, 2)),
      r2(M.at(2, 0), M.at(2, 1), M.at(2, 2))
{
}

// ---- intrinsics ---------------------------------------------------------------
inline float hl_asfloat(uint u) { float f; memcpy(&f, &u, 4); return f; }
inline float hl_asfloat(int i) { float f; memcpy(&f, &i, 4); return f; }
inline int hl_asint(float f) { int i; memcpy(&i, &f, 4); return i; }
inline uint hl_asuint(float f) { uint u; memcpy(&u, &f, 4); return u; }

inline float hl_abs(float x) { return fabsf(x); }
inline int hl_abs(int x) { return x < 0 ? -x : x; }
inline float hl_sqrt(float x) { return sqrtf(x); }
inline float hl_min(float a, float b) { return fminf(a, b); }
inline float hl_max(float a, float b) { return fmaxf(a, b); }
inline int hl_min(int a, int b) { return a < b ? a : b; }
inline int hl_max(int a, int b) { return a > b ? a : b; }
inline float hl_clamp(float x, float a, float b) { return fminf(fmaxf(x, a), b); }
inline float hl_saturate(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
inline float hl_lerp(float a, float b, float t) { return a + t * (b - a); }
inline bool hl_isnan(float x) { return std::isnan(x); }
inline float hl_sin(float x) { return own_sinf(x); }
inline float hl_cos(float x) { return own_cosf(x); }
inline float hl_acos(float x) { return own_acosf(x); }
inline float hl_pow(float x, float y) { return powf(x, y); }
inline float hl_floor(float x) { return floorf(x); }

inline float3 hl_min(const float3& a, const float3& b) { return float3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
inline float3 hl_max(const float3& a, const float3& b) { return float3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
inline float3 hl_abs(const float3& a) { return float3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
inline float3 hl_saturate(const float3& a) { return float3(hl_saturate(a.x), hl_saturate(a.y), hl_saturate(a.z)); }
inline bool3 hl_isnan(const float3& a) { return bool3(std::isnan(a.x), std::isnan(a.y), std::isnan(a.z)); }
inline bool hl_any(const bool2& b) { return b.x || b.y; }
inline bool hl_any(const bool3& b) { return b.x || b.y || b.z; }
inline bool hl_all(const float3& v) { return v.x != 0.0f && v.y != 0.0f && v.z != 0.0f; }
inline bool hl_all(const bool2& b) { return b.x && b.y; }

inline float hl_dot(const float2& a, const float2& b) { return a.x * b.x + a.y * b.y; }
inline float hl_dot(const float3& a, const float3& b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline uint hl_dot(const uint2& a, const uint2& b) { return a.x * b.x + a.y * b.y; }
inline float3 hl_cross(const float3& a, const float3& b)
{
    return float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float hl_length(const float3& v) { return sqrtf(hl_dot(v, v)); }
inline float3 hl_normalize(const float3& v) { return v * (1.0f / sqrtf(hl_dot(v, v))); }

inline float4 hl_mul(const float4x4& M, const float4& v)
{
    float4 r;
    for (int i = 0; i < 4; ++i) r[i] = ((M.at(i, 0) * v.x + M.at(i, 1) * v.y) + M.at(i, 2) * v.z) + M.at(i, 3) * v.w;
    return r;
}
inline float3 hl_mul(const float3x3& M, const float3& v)
{
    float3 r;
    for (int i = 0; i < 3; ++i) r[i] = (M[i].x * v.x + M[i].y * v.y) + M[i].z * v.z;
    return r;
}
// row vector times matrix: r[c] = sum over rows k of v[k] * M[k][c]
inline float3 hl_mul(const float3& v, const float3x3& M)
{
    float3 r;
    for (int c = 0; c < 3; ++c) r[c] = (v.x * M[0][c] + v.y * M[1][c]) + v.z * M[2][c];
    return r;
}
inline float3x3 hl_transpose(const float3x3& M)
{
    return float3x3(float3(M[0].x, M[1].x, M[2].x), float3(M[0].y, M[1].y, M[2].y), float3(M[0].z, M[1].z, M[2].z));
}
template <class T> inline T hl_NonUniformResourceIndex(T i) { return i; }

// ---- resources ------------------------------------------------------------------
template <class T> struct StructuredBuffer {
    const T* p = nullptr;
    uint64_t n = 0;
    T operator[](uint64_t i) const
    {
        if (i >= n) {
            ref_ub = 1;
            return T{};
        }
        T v;
        memcpy(static_cast<void*>(&v), static_cast<const void*>(&p[i]), sizeof(T));
        return v;
    }
};
// A writable buffer over the window [base, base + n) of the logical index space.
template <class T> struct RWStructuredBuffer {
    T* p = nullptr;
    uint64_t base = 0, n = 0;
    T dummy{};
    T& operator[](uint64_t i)
    {
        if (i < base || i - base >= n) {
            ref_ub = 1;
            return dummy;
        }
        return p[i - base];
    }
};
template <class T> struct ConstantBuffer : T {};
struct SamplerState {};
// Image of RGBA32F texels, width x height, row-major.
template <class T> struct Texture2D {
    const T* p = nullptr;
    uint w = 0, h = 0;
    T operator[](const uint2& ij) const
    {
        if (ij.x >= w || ij.y >= h) {
            ref_ub = 1;
            return T{};
        }
        return p[(size_t)ij.y * w + ij.x];
    }
    // Linear filter with clamp-to-edge addressing (the upscale pass's sampler,
    // src/render/upscalepass.cpp:12-38): texel-space position uv * size - 0.5,
    // the four clamped neighbours, exact FP32 weights blended in a fixed order.
    // The hardware filter rounds its weights to a sub-texel precision of the
    // implementation's choosing; this is the convention the oracle and the
    // kernels share.
    T SampleLevel(const SamplerState&, const float2& uv, int) const
    {
        const float fx = uv.x * (float)w - 0.5f;
        const float fy = uv.y * (float)h - 0.5f;
        const float flx = floorf(fx), fly = floorf(fy);
        const float a = fx - flx, b = fy - fly;
        int x0 = (int)flx, y0 = (int)fly, x1 = x0 + 1, y1 = y0 + 1;
        const int mx = (int)w - 1, my = (int)h - 1;
        x0 = x0 < 0 ? 0 : (x0 > mx ? mx : x0);
        x1 = x1 < 0 ? 0 : (x1 > mx ? mx : x1);
        y0 = y0 < 0 ? 0 : (y0 > my ? my : y0);
        y1 = y1 < 0 ? 0 : (y1 > my ? my : y1);
        const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
        const T c00 = p[(size_t)y0 * w + x0], c10 = p[(size_t)y0 * w + x1];
        const T c01 = p[(size_t)y1 * w + x0], c11 = p[(size_t)y1 * w + x1];
        T o;
        for (int c = 0; c < 3; ++c) o[c] = ((c00[c] * w00 + c10[c] * w10) + c01[c] * w01) + c11[c] * w11;
        o[3] = c00[3];
        return o;
    }
    // The shaders on this path call Sample only from helpers they never use.
    T Sample(const SamplerState&, const float2&) const
    {
        ref_ub = 1;
        return T{};
    }
};
template <class T> struct RWTexture2D {
    T* p = nullptr;
    uint w = 0, h = 0;
    T dummy{};
    T& operator[](const uint2& ij)
    {
        if (ij.x >= w || ij.y >= h) {
            ref_ub = 1;
            return dummy;
        }
        return p[(size_t)ij.y * w + ij.x];
    }
};
template <class T> struct TextureCube {};
