// Device restatements of the per-cell shader helpers of compute.hlsl (lines cited per
// function).  Operation order follows the shader expressions, so a translation unit compiled
// with -fmad=false reproduces IEEE single-precision results of the same expressions.
//
// Transcendentals: with CEL_EXACT_FP32 defined (the plain form) every single-precision
// transcendental is evaluated in double and rounded once to float — the correctly rounded
// value, which the FP32 transcription on the CPU computes the same way, so the two agree bit for
// bit.  Without it (fused forms) the CUDA single-precision functions are used.  All helpers
// have internal linkage because the two builds differ.
#pragma once

#include <cuda_runtime.h>

#include "celeris_internal.hpp"

namespace cel {
namespace {

#ifdef CEL_EXACT_FP32
__device__ __forceinline__ float t_sin(float x) { return float(sin(double(x))); }
__device__ __forceinline__ float t_cos(float x) { return float(cos(double(x))); }
__device__ __forceinline__ float t_tanh(float x) { return float(tanh(double(x))); }
__device__ __forceinline__ float t_atan(float x) { return float(atan(double(x))); }
__device__ __forceinline__ float t_cosh(float x) { return float(cosh(double(x))); }
__device__ __forceinline__ float t_pow(float x, float y) { return float(pow(double(x), double(y))); }
#else
__device__ __forceinline__ float t_sin(float x) { return sinf(x); }
__device__ __forceinline__ float t_cos(float x) { return cosf(x); }
__device__ __forceinline__ float t_tanh(float x) { return tanhf(x); }
__device__ __forceinline__ float t_atan(float x) { return atanf(x); }
__device__ __forceinline__ float t_cosh(float x) { return coshf(x); }
__device__ __forceinline__ float t_pow(float x, float y) { return powf(x, y); }
#endif

#define CEL_MIN_DEPTH 0.0001f  // compute.hlsl:1062
#define CEL_PI_F 3.14159274101257324f  // 4*atan(1.0f) in float (engine.cpp:89)

// MinMod (compute.hlsl:292-296)
__device__ __forceinline__ float minmod3(float a, float b, float c) {
    return (a > 0.f && b > 0.f && c > 0.f) ? fminf(fminf(a, b), c)
         : (a < 0.f && b < 0.f && c < 0.f) ? fmaxf(fmaxf(a, b), c) : 0.f;
}

// Reconstruct (compute.hlsl:298-315); sd is the breaking-indicator standard deviation.
__device__ __forceinline__ void reconstruct(float tt, float w, float c, float e, float& ow, float& oe) {
    const float z1 = tt * (c - w), z2 = e - w, z3 = tt * (e - c);
    const float g2 = 0.25f * minmod3(z1, z2, z3);
    oe = c + g2;
    ow = c - g2;
}
__device__ __forceinline__ void reconstruct_sd(float tt, float w, float c, float e, float& ow, float& oe, float& sd) {
    const float z1 = tt * (c - w), z2 = e - w, z3 = tt * (e - c);
    const float g2 = 0.25f * minmod3(z1, z2, z3);
    const float mu = 0.5f * (z1 + z2 + z3) / 3.0f;
    sd = sqrtf(((z1 - mu) * (z1 - mu) + (z2 - mu) * (z2 - mu) + (z3 - mu) * (z3 - mu)) / 3.0f);
    oe = c + g2;
    ow = c - g2;
}

// CorrectW (compute.hlsl:317-328)
__device__ __forceinline__ void correct_w(float Bw, float Be, float wbar, float& ww, float& we) {
    if (we < Be) { we = Be; ww = fmaxf(Bw, 2.f * wbar - Be); }
    else if (ww < Bw) { we = fmaxf(Be, 2.f * wbar - Bw); ww = Bw; }
}

// divide_by_h of CalcUV / CalcUV_Scalar (compute.hlsl:330-352)
__device__ __forceinline__ float div_by_h(float h, float eps) {
    const float h2 = h * h, h4 = h2 * h2;
    return 1.41421354f * h / sqrtf(h4 + fmaxf(h4, eps));
}

// NumericalFlux (compute.hlsl:363-370)
__device__ __forceinline__ float numflux(float ap, float am, float Fp, float Fm, float dU) {
    if (ap - am != 0.f) return (ap * Fm - am * Fp + ap * am * dU) / (ap - am);
    return 0.f;
}

// FrictionCalc (compute.hlsl:544-553)
__device__ __forceinline__ float friction_calc(float hu, float hv, float h, float friction, int manning, float g,
                                               float eps) {
    float f = friction;
    const float h4 = t_pow(h, 4.0f);
    const float dbh = 1.41421354f * h / sqrtf(h4 + fmaxf(h4, eps));
    if (manning == 1) f = g * friction * friction * t_pow(fabsf(dbh), 0.3333f);
    return f * sqrtf(hu * hu + hv * hv) * dbh * dbh;
}

// Source texel of a solid-wall ghost cell (compute.hlsl:985-1009).  The shaders mirror with
// `4 - tex_idx` and `reflect - tex_idx` (reflect = 2n+2, engine.cpp:1308-1309) where tex_idx is
// the interpolated pixel coordinate x + 0.5 (engine.cpp:579), and int3() truncates toward zero:
// the west/south ghosts read 3 - x, the east/north ghosts read 2n + 1 - x.  A source outside the
// texture reads zero.
__host__ __device__ __forceinline__ int solid_mirror(int c, int x) {
    return int(float(c) - (float(x) + 0.5f));
}
__host__ __device__ __forceinline__ void solid_source(int side, int x, int y, int nx, int ny, int& qx, int& qy) {
    qx = x; qy = y;
    if (side == 3) qx = solid_mirror(4, x);
    else if (side == 1) qx = solid_mirror(2 * nx + 2, x);
    else if (side == 2) qy = solid_mirror(4, y);
    else qy = solid_mirror(2 * ny + 2, y);
}

// SpongeFunction (compute.hlsl:1056-1059)
__device__ __forceinline__ float sponge_fn(float L, float x) {
    return 0.5f + 0.5f * t_cos(CEL_PI_F * fmaxf(L - x, 0.f) / L);
}

// sineWave with Eckart's wavenumber (compute.hlsl:1080-1101); t is float as in the reference.
__device__ __forceinline__ void sine_wave(float x, float y, float t, float d, float amp, float period,
                                          float th, float phase, float g, float& e, float& hu, float& hv) {
    const float omega = 2.f * CEL_PI_F / period;
    const float k = omega * omega / (g * sqrtf(t_tanh(omega * omega * d / g)));
    const float c = omega / k;
    const float kx = t_cos(th) * x * k;
    const float ky = t_sin(th) * y * k;
    e = amp * t_sin(omega * t - kx - ky + phase);
    hu = c * t_cos(th) * e;
    hv = c * t_sin(th) * e;
}

}  // namespace
}  // namespace cel
