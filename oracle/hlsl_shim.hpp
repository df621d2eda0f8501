// Just enough of HLSL's shader-model-4 vocabulary, in C++, to compile the reference's
// compute.hlsl on the CPU (test infrastructure: it builds the reference-side checker under
// oracle/_ref/, never the product).
//
// What it models, and how D3D11 defines it:
//   * float2/3/4 with .x/.y/.z/.w and .r/.g/.b/.a naming the same component, component-wise
//     arithmetic, scalar promotion, and the .rg/.rgb swizzles the shader uses (the build-time
//     transform turns `v.rg` into `v.rg_()`; `B.rg = ...` assigns through a proxy);
//   * int3 with HLSL's float->int conversion (truncation toward zero);
//   * Texture2D<T>::Load(int3): reads the shader-resource view bound to the texture's register
//     (several names share one register, as in the shader); a load outside the bound texture
//     returns zero, as D3D10+ specifies for out-of-range Load;
//   * intrinsics: min/max/abs/sqrt/pow/sin/cos/tanh/cosh/atan/normalize.  sqrt and the
//     arithmetic operators are IEEE single precision; the transcendentals are evaluated in double
//     and rounded once (the same convention as the oracle's FP32 build and the product's plain
//     form; HLSL leaves their precision to the driver).
// Floating literals are made single precision by the transform (HLSL literals are float).
#pragma once

#include <cmath>

namespace hlsl {

typedef unsigned int uint;

struct float2;
struct float3;
struct float4;

struct float2 {
    union { float x; float r; };
    union { float y; float g; };
    float2() : x(0.f), y(0.f) {}
    template <class A, class B>
    float2(A a, B b) : x(float(a)), y(float(b)) {}
    float2 rg_() const { return *this; }
};

struct float3 {
    union { float x; float r; };
    union { float y; float g; };
    union { float z; float b; };
    float3() : x(0.f), y(0.f), z(0.f) {}
    template <class A, class B, class C>
    float3(A a, B b, C c) : x(float(a)), y(float(b)), z(float(c)) {}
    float2 rg_() const { return float2(x, y); }
    float3 rgb_() const { return *this; }
};

struct float4 {
    union { float x; float r; };
    union { float y; float g; };
    union { float z; float b; };
    union { float w; float a; };
    float4() : x(0.f), y(0.f), z(0.f), w(0.f) {}
    template <class A, class B, class C, class D>
    float4(A a, B b, C c, D d) : x(float(a)), y(float(b)), z(float(c)), w(float(d)) {}
    // .rg as an l-value (B.rg = ...) or an r-value
    struct RG {
        float4& v;
        RG& operator=(const float2& s) { v.x = s.x; v.y = s.y; return *this; }
        operator float2() const { return float2(v.x, v.y); }
    };
    RG rg_() { return RG{*this}; }
    float2 rg_() const { return float2(x, y); }
    float3 rgb_() const { return float3(x, y, z); }
};

struct int3 {
    int x, y, z;
    int3() : x(0), y(0), z(0) {}
    template <class A, class B, class C>
    int3(A a, B b, C c) : x(int(a)), y(int(b)), z(int(c)) {}
};
inline int3 operator+(int3 a, int3 b) { return int3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline int3 operator*(int3 a, int k) { return int3(a.x * k, a.y * k, a.z * k); }

// ---- component-wise arithmetic ----------------------------------------------------------
#define HLSL_VEC_OPS(V, N, EXPR)                                                               \
    inline V operator+(V a, V b) { V o; for (int i = 0; i < N; ++i) (&o.x)[i] = (&a.x)[i] + (&b.x)[i]; return o; } \
    inline V operator-(V a, V b) { V o; for (int i = 0; i < N; ++i) (&o.x)[i] = (&a.x)[i] - (&b.x)[i]; return o; } \
    inline V operator*(V a, V b) { V o; for (int i = 0; i < N; ++i) (&o.x)[i] = (&a.x)[i] * (&b.x)[i]; return o; } \
    inline V operator/(V a, V b) { V o; for (int i = 0; i < N; ++i) (&o.x)[i] = (&a.x)[i] / (&b.x)[i]; return o; } \
    inline V operator*(V a, float s) { V o; for (int i = 0; i < N; ++i) (&o.x)[i] = (&a.x)[i] * s; return o; }      \
    inline V operator*(float s, V a) { V o; for (int i = 0; i < N; ++i) (&o.x)[i] = s * (&a.x)[i]; return o; }      \
    inline V operator/(V a, float s) { V o; for (int i = 0; i < N; ++i) (&o.x)[i] = (&a.x)[i] / s; return o; }      \
    inline V operator-(V a) { V o; for (int i = 0; i < N; ++i) (&o.x)[i] = -(&a.x)[i]; return o; }                   \
    inline V sqrt(V a) { V o; for (int i = 0; i < N; ++i) (&o.x)[i] = std::sqrt((&a.x)[i]); return o; }
HLSL_VEC_OPS(float2, 2, 0)
HLSL_VEC_OPS(float3, 3, 0)
HLSL_VEC_OPS(float4, 4, 0)
#undef HLSL_VEC_OPS

// ---- intrinsics -------------------------------------------------------------------------
// max/min follow std::max/std::min (the first argument unless the second compares greater /
// smaller), which is what the oracle uses; the two differ from D3D only for NaN and -0/+0.
inline float max(float a, float b) { return (a < b) ? b : a; }
inline float min(float a, float b) { return (b < a) ? b : a; }
inline float max(float a, int b) { return max(a, float(b)); }
inline float max(int a, float b) { return max(float(a), b); }
inline float min(float a, int b) { return min(a, float(b)); }
inline float min(int a, float b) { return min(float(a), b); }
inline float4 max(float4 a, float s) { return float4(max(a.x, s), max(a.y, s), max(a.z, s), max(a.w, s)); }
inline float4 max(float4 a, float4 b) { return float4(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z), max(a.w, b.w)); }
inline float abs(float a) { return std::fabs(a); }
inline float sqrt(float a) { return std::sqrt(a); }
inline float sin(float a) { return float(std::sin(double(a))); }
inline float cos(float a) { return float(std::cos(double(a))); }
inline float tanh(float a) { return float(std::tanh(double(a))); }
inline float cosh(float a) { return float(std::cosh(double(a))); }
inline float atan(float a) { return float(std::atan(double(a))); }
inline float pow(float a, float b) { return float(std::pow(double(a), double(b))); }
inline float pow(float a, int b) { return pow(a, float(b)); }
inline float3 normalize(float3 v) { return v / std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }

// ---- textures and the shader-resource slots --------------------------------------------
// One bound view: `comps` floats per texel (4 = RGBA32F, 3 = RGB32F), `w` x `h` texels.
struct SRV {
    const float* data = nullptr;
    int w = 0, h = 0, comps = 4;
};
SRV& srv_slot(int reg);  // defined by the driver

template <class T>
struct Texture2D {
    int reg;
    T Load(int3 i) const {
        const SRV& s = srv_slot(reg);
        float v[4] = {0.f, 0.f, 0.f, 0.f};
        if (s.data && i.x >= 0 && i.y >= 0 && i.x < s.w && i.y < s.h) {
            const float* p = s.data + (size_t(i.y) * s.w + i.x) * s.comps;
            for (int k = 0; k < s.comps && k < 4; ++k) v[k] = p[k];
        }
        return make(v, static_cast<T*>(nullptr));
    }
    static float4 make(const float* v, float4*) { return float4(v[0], v[1], v[2], v[3]); }
    static float3 make(const float* v, float3*) { return float3(v[0], v[1], v[2]); }
};

}  // namespace hlsl
