// Fused, batched B200 form of the Celeris timestep path.
//
// One pass (predictor, corrector or Euler) of every domain in a batch is three kernels plus the
// boundary kernels, each launched once for all domains over a cross-domain work list:
//   k_march    : Pass1 (minmod reconstruction, positivity fix, desingularised velocities) +
//                Pass2 (Kurganov-Petrova central-upwind fluxes) + Pass3Predictor (flux
//                divergence, bed slope, friction, Madsen-Sorensen dispersion, F*/G*, AB3/AM4
//                combination) + white-water/inundation aux + the GetStats reduction, marching
//                down 126-column strips with a 6-row shared-memory ring.  It writes the new w
//                and, for hu and hv, the right-hand side of the implicit dispersive system in
//                increment form: M dhu = r, hu_new = hu_base + dhu.
//   k_rows / k_cols : the tridiagonal solves along x (one CTA per row) and y (one CTA per band
//                of 16 columns), a chunked Thomas elimination whose forward and backward sweeps
//                are first-order linear recurrences combined across chunks by a scan; the
//                time-invariant LU factors are precomputed per domain.
//   k_boundary : East, North, West, South strips in the reference's order (one launch each).
// The whole physical step (predictor + correctors) is captured once per buffer-rotation phase
// into CUDA graphs and replayed.
//
// CEL_FORM_MIXED additionally keeps a compensation (low) word for w, hu and hv and adds every
// increment with a two-sum, evaluates the wave-maker phase omega*t in FP64 from an FP64 clock,
// and reduces mass/energy in FP64.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "batch.hpp"
#include "device_math.cuh"
#include "engine_iface.hpp"
#include "scheme.hpp"

namespace cel {

namespace {

constexpr int TX = 32, TY = 16;
// column solver threads per CTA: CW columns x (NT/CW) chunks, NT 256 or 512 (a tuning choice; the
// chunk length is the solver's switch point from the parallel carry scan to serial sweeps).  1024
// threads at one CTA per SM (64 registers) measured slower on C4 than 512 at two: 10.07 with
// 32-column bands and 9.67 with 16, against 10.34 Gcell-steps/s; a CTA's barriers and carry scans
// then stall the whole SM.
constexpr int NTC_DEFAULT = 512;
// column solver CTAs per SM the build targets at 512 threads: 2 (64 registers, no spills); 1 lets
// the compiler take about 100 registers and run one CTA per SM, 3 spills (measured on C4: 8.9 / 10.3
// / 9.2 Gcell-steps/s).  256-thread CTAs target twice as many, at the same 64 registers.
#ifndef CEL_COLS_MIN_CTAS
#define CEL_COLS_MIN_CTAS 2
#endif
constexpr int cols_min_ctas(int nt) { return CEL_COLS_MIN_CTAS * 512 / nt; }
constexpr int STATS_N = 12;

// stats accumulator layout
// [0] sum h  [1] sum h(B+h/2)  [2] sum hu  [3] sum hv  [4] sum (hu u + hv v)  [5] sum h (every cell)
// [6] max u^2+v^2  [7] max h  [8] max cfl rate  [9] max (u^2+v^2)/h  [10] health flag
struct MemberDev {
    SimConsts c;
    int P;                  // plane pitch in floats
    float* base;            // first plane; plane k starts at base + k * plane
    unsigned long long plane;
    const CUtensorMap* tmaps;  // 2D row maps: state [buffer*3 + field], then BA, BX, BY
    float tan_thr;          // tan(dissipation threshold): atan(x) > thr  <=>  x > tan(thr)
    const float* dtp;       // this member's time step (device table, host-updatable)
    const float* ab;        // adaptive AB3 predictor: {k, A0, A1, A2, K0, K1, K2} (see k_choose_dt)
    float* S[3][3];         // state buffers [buffer][w, hu, hv]
    float* L[3][3];         // compensation words (mixed form)
    const float* BY;
    const float* BX;
    const float* BA;
    float* R[2];            // increment right-hand sides for hu, hv
    float4* HA[4];          // history slots: {dw/dt, dhu/dt, dhv/dt, F*}
    float* HB[4];           // history slots: G*
    float* AUX[2];          // {max inundated depth, breaking} as one float2 plane pair (AUX[0])
    const float* FX[3];     // x-systems: c', inv_den, m
    const float* FYF[3];    // y-systems: c', inv_den, m
    float* CORN;            // bathymetry at cell corners, (NX+1) x (NY+1) with pitch PC (the stencil rebuilds BA, BX, BY)
    float* FYB[3];          // the y factors band-major for the banded column solve: band b, row i, column c at
                            // (b * ny + i) * band width + c
    int PC;
    BoundaryDesc bd[4];     // N, E, S, W
    const float4* waves;
    const double* waves64;  // the same components in FP64, 4 per component (compensated form)
    const float* uts[4];    // (t, eta, hu, hv) tables, float
    const double* uts64[4]; // the same tables in FP64 (compensated form)
    int nuts[4];
    double dx64, dy64, g64; // grid spacing and gravity in FP64 (the compensated form's strip values)
    float* strip;           // two-phase strips: 3 floats per cell (6 with the low words)
    double* stats;
    double* stats_now;
    double* time64;
    float* time32;
};

struct PassArgs {
    int in, out, cur;
    int og, oog, scr, pred;
    int scheme;
    int stats;          // accumulate GetStats of the input state (first pass of a physical step)
    int friction;       // some member has a nonzero friction coefficient
    double* late_flag;  // set when a bounded TMA wait gave up
};

__device__ __forceinline__ void two_sum_add(float& hi, float& lo, float d) {
    // (hi + lo) + d with the rounding error of hi + d carried in lo (Knuth two-sum)
    const float s = hi + d;
    const float bp = s - hi;
    const float err = (hi - (s - bp)) + (d - bp);
    const float lo2 = lo + err;
    const float h2 = s + lo2;
    lo = lo2 - (h2 - s);
    hi = h2;
}

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

// Block reduction of the GetStats quantities of one cell per thread into the member's
// accumulators (FP64 sums, maxima via the ordering of non-negative doubles).
__device__ void stats_reduce(double* acc, bool cnt_block, bool cnt_all, float h, double h64, float B, float hu,
                             float hv, float u, float v, float q, float cc, float odx, float ody, bool bad,
                             double (*red)[STATS_N]) {
    double s[STATS_N];
    for (int k = 0; k < STATS_N; ++k) s[k] = 0.0;
    if (cnt_block) {
        s[0] = h; s[1] = double(h * (B + 0.5f * h)); s[2] = hu; s[3] = hv; s[4] = double(hu * u + hv * v);
        const float u2v2 = u * u + v * v;
        s[6] = u2v2; s[7] = h;
        s[8] = fmaxf((fabsf(u) + cc) * odx, (fabsf(v) + cc) * ody);
        s[9] = u2v2 * q;
    }
    if (cnt_all) s[5] = h64;
    s[10] = bad ? 1.0 : 0.0;
    for (int off = 16; off; off >>= 1)
        for (int k = 0; k < 11; ++k) {
            const double o = __shfl_down_sync(0xffffffffu, s[k], off);
            s[k] = (k >= 6) ? fmax(s[k], o) : s[k] + o;
        }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < 11; ++k) red[wid][k] = s[k];
    __syncthreads();
    if (threadIdx.x < 11) {
        const int k = threadIdx.x;
        const int nw = blockDim.x >> 5;
        double a = red[0][k];
        for (int w = 1; w < nw; ++w) a = (k >= 6) ? fmax(a, red[w][k]) : a + red[w][k];
        if (k < 6) { if (a != 0.0) atomicAdd(acc + k, a); }
        else atomic_max_nonneg(acc + k, a);
    }
}

// ---------------------------------------------------------------------------------------------
// k_march: Pass1 + Pass2 + Pass3 + aux + GetStats, marching down a strip of MO = 126 output
// columns for MH rows.  Thread i owns column x0 - 1 + i (128 threads: the 126 output columns
// plus one halo column each side for the faces the fluxes need).  State and bottom rows sit in
// a 6-row shared-memory ring (rows t-2 .. t+3 around the output row t); faces travel along y in
// registers (the north face of row t becomes the south side of the y flux), east/west faces and
// the x fluxes are exchanged through shared memory.  Two barriers per row.
// ---------------------------------------------------------------------------------------------
// CTAs per SM the stencil's register budget is sized for (65,536 / (128 x this) registers a thread)
#ifndef CEL_MARCH_MIN_CTAS
#define CEL_MARCH_MIN_CTAS 5
#endif
constexpr int MARCH_MIN_CTAS = CEL_MARCH_MIN_CTAS;
#ifndef CEL_MARCH2_MIN_CTAS
#define CEL_MARCH2_MIN_CTAS 3
#endif
constexpr int MARCH2_MIN_CTAS = CEL_MARCH2_MIN_CTAS;   // the paired-row stencil (49.6 KB smem, 166 registers)
constexpr int MW = 128;          // threads = columns with faces per row
constexpr int MO = MW - 2;       // output columns per strip
constexpr int MH_DEFAULT = 64;   // rows per strip unless tuned (each work item carries its height)
constexpr int RING = 7;          // state / bottom rows resident in shared memory (PREFETCH + 5)
constexpr int RBOX = 136;        // TMA box width in floats (covers columns x0-2 .. x0+127)
constexpr int RSTR = 160;        // ring row stride in floats (640 B, a multiple of 128 B)
constexpr int CBOX = RBOX + 4;   // corner-grid box: the RBOX cells' corners (one more), rounded to 16 B
constexpr unsigned ROW_BYTES = 6u * RBOX * 4u;
constexpr int PREFETCH = 2;      // rows requested ahead of the row being consumed

// ---- TMA and mbarrier helpers (inline PTX; single-CTA, no multicast) -----------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after a fixed number of polls and reports false (the caller flags the
// error and carries on with whatever the buffer holds, so no thread can hang on it).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity, int polls) {
    for (int k = 0; k < polls; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// After a wait gave up: before the CTA exits, wait (bounded) for the copies still in flight into its
// ring, i.e. on every slot for the phase of the last row requested into it.  Rows carry sequence
// numbers 0, 1, ... in request order; row q goes to slot q % ring and completes phase (q / ring) & 1.
__device__ __forceinline__ void drain_ring(unsigned long long* bars, int ring, unsigned requested) {
    for (int s = 0; s < ring; ++s) {
        if (requested <= unsigned(s)) continue;
        const unsigned q = unsigned(s) + unsigned(ring) * ((requested - 1u - unsigned(s)) / unsigned(ring));
        (void)mbar_wait_bounded(&bars[s], (q / unsigned(ring)) & 1u, 1 << 22);
    }
}
__device__ __forceinline__ void tma_row(float* dst, const CUtensorMap* map, int x, int y, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// ---- fast single-precision helpers of the fused forms (same formulas, fewer instructions) ----
__device__ __forceinline__ float div_by_h_fast(float h, float eps) {
    const float h2 = h * h, h4 = h2 * h2;
    return 1.41421354f * h * rsqrtf(h4 + fmaxf(h4, eps));
}
// Reciprocal of the Kurganov-Petrova denominator a+ - a- (> 0 where it is used): the hardware
// approximation r0 = __fdividef(1, x), refined by one Newton-Raphson iteration for f(r) = 1/r - x,
//   r1 = r0 + r0 (1 - x r0),
// with both steps as fused multiply-adds (Newton's method for the reciprocal, as in Markstein,
// "IA-64 and Elementary Functions", 2000, ch. 8).  The approximation alone errs with a small
// systematic bias; through the fluxes at an open boundary the compensated form's water volume
// picked it up as a steady drift from the FP64 oracle (6.5e-9 of the volume after 10,000 steps of
// the C1 flume, 3.2e-9 and 2.7e-9 on two C4 members).  Refined, the drift is gone (0.3e-9, 0.4e-9,
// 0.2e-9) at no measurable cost.  The refined values stay within one unit in the last place of the
// correctly rounded reciprocal (cel_selftest_reciprocal checks it on the device).
__device__ __forceinline__ float rcp_newton(float x) {
    const float r = __fdividef(1.0f, x);
    return fmaf(r, fmaf(-x, r, 1.0f), r);
}
// NumericalFlux for the three components of one face, sharing the reciprocal of a+ - a-
__device__ __forceinline__ void numflux3(float ap, float am, const float Fp[3], const float Fm[3], const float dU[3],
                                         float out[3]) {
    const float den = ap - am;
    const float inv = den != 0.f ? rcp_newton(den) : 0.f;
    const float apam = ap * am;
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = (ap * Fm[k] - am * Fp[k] + apam * dU[k]) * inv;
}
__device__ __forceinline__ float friction_fast(float hu, float hv, float h, float friction, int manning, float g,
                                              float eps) {
    if (friction == 0.f) return 0.f;   // both friction laws vanish with a zero coefficient
    const float h2 = h * h, h4 = h2 * h2;
    const float dbh = 1.41421354f * h * rsqrtf(h4 + fmaxf(h4, eps));
    float f = friction;
    if (manning == 1) f = g * friction * friction * exp2f(0.3333f * __log2f(fabsf(dbh)));
    return f * sqrtf(hu * hu + hv * hv) * dbh * dbh;
}

// face depths h, velocities u, v, and the face water levels w (h = w - face bottom)
struct Face { float hN, hE, hS, hW, uN, uE, uS, uW, vN, vE, vS, vW, wN, wE, wS, wW, msd; };

// MinMod (compute.hlsl:292-296) without branches: all three positive <=> their minimum is
// positive, all negative <=> their maximum is negative (identical results for finite inputs).
__device__ __forceinline__ float minmod3_fast(float a, float b, float c) {
    const float mn = fminf(fminf(a, b), c), mx = fmaxf(fmaxf(a, b), c);
    return mn > 0.f ? mn : (mx < 0.f ? mx : 0.f);
}
// Reconstruct with the breaking-indicator standard deviation, divisions by 3 as products
__device__ __forceinline__ void reconstruct_sd_fast(float tt, float w, float c, float e, float& ow, float& oe, float& sd) {
    const float z1 = tt * (c - w), z2 = e - w, z3 = tt * (e - c);
    const float g2 = 0.25f * minmod3_fast(z1, z2, z3);
    const float mu = (0.5f / 3.0f) * (z1 + z2 + z3);
    sd = sqrtf(((z1 - mu) * (z1 - mu) + (z2 - mu) * (z2 - mu) + (z3 - mu) * (z3 - mu)) * (1.0f / 3.0f));
    oe = c + g2;
    ow = c - g2;
}

// Kahan-compensated single-precision accumulator (statistics without per-cell FP64 work)
struct Kahan {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add(float x) {
        const float y = x - c;
        const float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return double(s) - double(c); }
};

// Ring layout: field f, slot s, column k at ring[f * FSTR + s * RSTR + k]; a "row base" is
// s * RSTR + (this thread's column), so every access is base + compile-time offset.
constexpr int FSTR = RING * RSTR;
constexpr int DSTR = RSTR;   // still-water depth ring: the ring's row stride, so one offset serves both

__device__ __forceinline__ void reconstruct_fast(float tt, float w, float c, float e, float& ow, float& oe) {
    const float z1 = tt * (c - w), z2 = e - w, z3 = tt * (e - c);
    const float g2 = 0.25f * minmod3_fast(z1, z2, z3);
    oe = c + g2;
    ow = c - g2;
}
// CorrectW (compute.hlsl:317-328) as selects
__device__ __forceinline__ void correct_w_fast(float Bw, float Be, float wbar, float& ww, float& we) {
    const bool c1 = we < Be, c2 = !c1 && (ww < Bw);
    const float nwe = c1 ? Be : (c2 ? fmaxf(Be, 2.f * wbar - Bw) : we);
    const float nww = c1 ? fmaxf(Bw, 2.f * wbar - Be) : (c2 ? Bw : ww);
    we = nwe;
    ww = nww;
}

// Pass1 at one cell: rows below / here / above given by their row bases.
__device__ __forceinline__ void faces_at(const float* __restrict__ ring, int bm, int b0, int bp, const SimConsts& c,
                                         Face& f) {
    const float* W = ring;
    const float* HU = ring + FSTR;
    const float* HV = ring + 2 * FSTR;
    const float* BXr = ring + 4 * FSTR;
    const float* BYr = ring + 5 * FSTR;
    const float wc = W[b0], wl = W[b0 - 1], wr = W[b0 + 1], wd = W[bm], wu = W[bp];
    const float BN = BYr[b0], BE = BXr[b0], BS = BYr[bm], BW = BXr[b0 - 1];
    float wN, wE, wS, wW, huN, huE, huS, huW, hvN, hvE, hvS, hvW, sd1, sd2;
    reconstruct_sd_fast(c.two_theta, wl, wc, wr, wW, wE, sd1);
    reconstruct_sd_fast(c.two_theta, wd, wc, wu, wS, wN, sd2);
    const float huc = HU[b0], hvc = HV[b0];
    reconstruct_fast(c.two_theta, HU[b0 - 1], huc, HU[b0 + 1], huW, huE);
    reconstruct_fast(c.two_theta, HU[bm], huc, HU[bp], huS, huN);
    reconstruct_fast(c.two_theta, HV[b0 - 1], hvc, HV[b0 + 1], hvW, hvE);
    reconstruct_fast(c.two_theta, HV[bm], hvc, HV[bp], hvS, hvN);
    correct_w_fast(BW, BE, wc, wW, wE);
    correct_w_fast(BS, BN, wc, wS, wN);
    f.hN = wN - BN; f.hE = wE - BE; f.hS = wS - BS; f.hW = wW - BW;
    f.wN = wN; f.wE = wE; f.wS = wS; f.wW = wW;
    float q;
    q = div_by_h_fast(f.hN, c.epsilon); f.uN = q * huN; f.vN = q * hvN;
    q = div_by_h_fast(f.hE, c.epsilon); f.uE = q * huE; f.vE = q * hvE;
    q = div_by_h_fast(f.hS, c.epsilon); f.uS = q * huS; f.vS = q * hvS;
    q = div_by_h_fast(f.hW, c.epsilon); f.uW = q * huW; f.vW = q * hvW;
    f.msd = fmaxf(sd1 * c.one_over_dx, sd2 * c.one_over_dy);
}

// KP07 flux through one face for the three equations, given the two face states (m: the side
// with the lower index, p: the other); `xdir` selects the velocity normal to the face.  Both
// sides of a face share its bottom, so the depth jump hp - hm equals the jump of the face water
// levels wp - wm; it is taken from those, which keep the bits of eta that a depth of several metres
// rounds away in single precision (at an open boundary that jump carries the mass exchange).
__device__ __forceinline__ void face_flux(float hm, float um, float vm, float wm, float hp, float up, float vp,
                                          float wp, float g, float hg, bool xdir, float out[3]) {
    const float cm = sqrtf(g * hm), cpp = sqrtf(g * hp);
    const float nm = xdir ? um : vm, np = xdir ? up : vp;
    const float ap = fmaxf(fmaxf(nm + cm, np + cpp), 0.f);
    const float am = fminf(fminf(nm - cm, np - cpp), 0.f);
    const float qp = hp * np, qm = hm * nm;          // normal mass fluxes
    float Fp[3], Fm[3], dU[3];
    Fp[0] = qp; Fm[0] = qm; dU[0] = wp - wm;
    if (xdir) {
        Fp[1] = hp * (up * up + hg * hp); Fm[1] = hm * (um * um + hg * hm); dU[1] = hp * up - hm * um;
        Fp[2] = qp * vp; Fm[2] = qm * vm; dU[2] = hp * vp - hm * vm;
    } else {
        Fp[1] = qp * up; Fm[1] = qm * um; dU[1] = hp * up - hm * um;
        Fp[2] = hp * (vp * vp + hg * hp); Fm[2] = hm * (vm * vm + hg * hm); dU[2] = hp * vp - hm * vm;
    }
    numflux3(ap, am, Fp, Fm, dU, out);
}

// ---------------------------------------------------------------------------------------------
// Plane layout of a member (offsets in planes of P x NY floats):
//   S: w, hu, hv for 3 buffers (9) | L: their low words (9, mixed form only) | BY BX BA | R0 R1 |
//   H[s], s = 0..3: HA = float4 {dw/dt, dhu/dt, dhv/dt, F*} (4 planes) and HB = G* (1 plane) |
//   AUX = float2 {max inundated depth, breaking} (2 planes) | FX (3) | FY (3)
// ---------------------------------------------------------------------------------------------
template <bool MIXED, bool ADAPT>
__global__ void __launch_bounds__(MW, MARCH_MIN_CTAS) k_march(const MemberDev* __restrict__ mems, const int4* __restrict__ tiles,
                                                 int ntiles, PassArgs pa) {
    __shared__ __align__(128) float ring[6 * FSTR];
    __shared__ float dring[RING * DSTR];  // still-water depth max(0, sea level - BA) of each ring row
    __shared__ __align__(8) unsigned long long bars[RING];
    __shared__ float fW[2][4][MW];       // [row parity][hW, uW, vW, wW][thread]: west faces for the x flux
    __shared__ float xb[3][MW];          // x flux at the thread's east face, this row
    constexpr int OFF = MIXED ? 18 : 9;
    constexpr int iR0 = OFF + 3, iH0 = OFF + 5, iAUX = OFF + 25;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int k = 0; k < RING; ++k) mbar_init(&bars[k], 1);
        mbar_fence_init();
    }
    __syncthreads();
    unsigned seq = 0;          // rows requested by this CTA so far (the same value in every thread)
    unsigned requested = 0;    // thread 0: sequence number of the last row it requested, plus one
    bool tma_late = false;
    const float* W = ring;
    const float* HU = ring + FSTR;
    const float* HV = ring + 2 * FSTR;
    const float* BAr = ring + 3 * FSTR;
    const float* BXr = ring + 4 * FSTR;
    const float* BYr = ring + 5 * FSTR;
    const bool stats = pa.stats != 0;
    const bool corr = pa.scheme == CEL_SCHEME_CORRECTOR;
    const bool euler = pa.scheme == CEL_SCHEME_EULER;

    for (int it = blockIdx.x; it < ntiles; it += gridDim.x) {
        const int4 tl = tiles[it];
        const MemberDev& M = mems[tl.x];
        const SimConsts c = M.c;
        const int P = M.P, nx = c.nx, ny = c.ny;
        float* __restrict__ B = M.base;
        const size_t PL = M.plane;
        const CUtensorMap* tm = M.tmaps;
        const int x0 = tl.y, y0 = tl.z, MH = tl.w;   // strip: columns x0 .. x0+MO-1, rows y0 .. y0+MH-1
        const int xs = (x0 - 2) & ~3;          // TMA box start, 16-byte aligned
        const int xc = x0 - 1 + tid;           // this thread's column
        const int rc0 = xc - xs;               // its ring column (1 .. 131)
        // Pass3 of the halo threads (0 and MW-1) runs on a clamped column and stores nothing; their
        // faces (needed by the neighbouring output columns) use the true column
        const int rc = max(rc0, 2);
        const int yend = min(y0 + MH, ny + 2);
        const int last_row = yend + 1;
        const bool out_col = tid >= 1 && tid <= MO && xc < nx + 2;
        const float dtm = *M.dtp;
        const float decay = t_pow(fabsf(c.whitewater_decay_rate), dtm);
        const float sl = c.sea_level;
        // per-plane bases of this pass
        const float4* __restrict__ HAo = reinterpret_cast<const float4*>(B + (iH0 + 5 * pa.og) * PL);
        const float4* __restrict__ HAoo = reinterpret_cast<const float4*>(B + (iH0 + 5 * pa.oog) * PL);
        const float4* __restrict__ HAp = reinterpret_cast<const float4*>(B + (iH0 + 5 * pa.pred) * PL);
        float4* __restrict__ HAs = reinterpret_cast<float4*>(B + (iH0 + 5 * pa.scr) * PL);
        const float* __restrict__ HBo = B + (iH0 + 5 * pa.og + 4) * PL;
        const float* __restrict__ HBoo = B + (iH0 + 5 * pa.oog + 4) * PL;
        const float* __restrict__ HBp = B + (iH0 + 5 * pa.pred + 4) * PL;
        float* __restrict__ HBs = B + (iH0 + 5 * pa.scr + 4) * PL;
        float* __restrict__ Wout = B + (3 * pa.out) * PL;
        const float* __restrict__ Wcur = B + (3 * pa.cur) * PL;
        float* __restrict__ R0 = B + iR0 * PL;
        float2* __restrict__ AUX = reinterpret_cast<float2*>(B + iAUX * PL);
        const float* __restrict__ Lbase = B + (9 + 3 * (corr ? pa.cur : pa.in)) * PL;
        float* __restrict__ Lout = B + (9 + 3 * pa.out) * PL;

        const unsigned seq0 = seq;
        auto issue = [&](int row, int sl_) {   // one thread: request the 6 fields of a row into slot sl_
            if (tma_late) return;                // a wait gave up: request nothing more
            requested = seq0 + unsigned(row - (y0 - 2)) + 1u;
            mbar_expect_tx(&bars[sl_], ROW_BYTES);
            float* dst = ring + sl_ * RSTR;
            tma_row(dst, tm + pa.in * 3 + 0, xs, row, &bars[sl_]);
            tma_row(dst + FSTR, tm + pa.in * 3 + 1, xs, row, &bars[sl_]);
            tma_row(dst + 2 * FSTR, tm + pa.in * 3 + 2, xs, row, &bars[sl_]);
            tma_row(dst + 3 * FSTR, tm + 9, xs, row, &bars[sl_]);
            tma_row(dst + 4 * FSTR, tm + 10, xs, row, &bars[sl_]);
            tma_row(dst + 5 * FSTR, tm + 11, xs, row, &bars[sl_]);
        };
        auto next_slot = [](int s) { return s + 1 == RING ? 0 : s + 1; };
        // still-water depth of a ring row: thread k covers ring column rc0(thread 0) - 1 + k, and
        // threads 0 and 1 also the two columns past the last thread (every column Pass3 reads)
        const int dcol = rc0 - 1;
        auto depth_row = [&](int off) {   // off = slot * RSTR
            const float* ba = BAr + off;
            float* dr = dring + off;
            dr[dcol] = fmaxf(0.f, sl - ba[dcol]);
            const int d2c = min(dcol + MW, RBOX - 1);
            if (tid < 2) dr[d2c] = fmaxf(0.f, sl - ba[d2c]);
        };

        Kahan acc[5];
        double mfull = 0.0;
        float mx[4] = {0.f, 0.f, 0.f, 0.f};
        bool bad = false;
        float nh = 0.f, nu = 0.f, nv = 0.f, nw = 0.f;   // north face of the previous row (this column)
        float eh = 0.f, eu = 0.f, ev = 0.f, ew = 0.f;   // east face of row t (this column), from the last step
        float ypv0 = 0.f, ypv1 = 0.f, ypv2 = 0.f; // y flux below the current row

        const int sA = int(seq0 % RING), sB = next_slot(sA), sC = next_slot(sB);  // rows y0-2, y0-1, y0

        __syncthreads();  // the previous strip is done with shared memory
        if (tid == 0) {
            fence_proxy_async();
            // rows y0-2 .. y0+PREFETCH-1 here; the loop requests row t+PREFETCH+2 at step t, so every
            // row is requested exactly once (one arrive per mbarrier phase)
            int sl_ = sA;
            for (int r = y0 - 2; r <= min(y0 + PREFETCH - 1, last_row); ++r) { issue(r, sl_); sl_ = next_slot(sl_); }
        }
        {   // the first step also reads rows y0-2 and y0-1
            const unsigned pA = (seq0 / RING) & 1u, pB = ((seq0 + 1) / RING) & 1u;
            if (!mbar_wait_bounded(&bars[sA], pA, tma_late ? 1 : (1 << 22))) tma_late = true;
            if (!mbar_wait_bounded(&bars[sB], pB, tma_late ? 1 : (1 << 22))) tma_late = true;
            depth_row(sA * RSTR);
            depth_row(sB * RSTR);
        }
        int s2p = sC;                                          // slot of row t+2 (mbarrier index)
        // ring-row offsets (slot * RSTR) of rows t-2 .. t+2, rotated as the window moves
        int o2m = sA * RSTR, o1m = sA * RSTR, o0 = sA * RSTR, o1p = sB * RSTR, o2p = sC * RSTR;
        unsigned par2p = ((seq0 + 2) / RING) & 1u;            // phase parity of row t+2
        int sReq = int((seq0 + unsigned(PREFETCH) + 2) % RING);  // slot of row t+PREFETCH+2
        size_t erow = size_t(y0 - 2) * P;                     // first cell of row t
        const int xl = min(xc, c.NX - 1);

        for (int t = y0 - 2; t < yend; ++t) {
            const bool p3 = t >= y0;                   // Pass3 runs on this row (uniform)
            const size_t e = erow + size_t(xc);        // this thread's cell of row t
            // loads use a column inside the row (the halo thread past the last column reads a
            // neighbour it never stores to)
            const size_t el = erow + size_t(xl);
            // per-cell inputs of Pass3 at (xc, t), requested before the face work
            float4 ho = make_float4(0.f, 0.f, 0.f, 0.f), hoo = ho, hp = ho;
            float go = 0.f, goo = 0.f, gp = 0.f, wcur = 0.f, wlo = 0.f;
            // aux texel of row t+1 owned by this strip (ghost texels x = 1 / y = 1 go with column /
            // row 2), read-modify-written after the faces of row t+1
            const int gy = t + 1;
            const int cxa = xc < 2 ? 2 : xc, cya = gy < 2 ? 2 : gy;
            const bool aux_ok = xc >= 1 && xc < nx + 2 && gy >= 1 && gy < ny + 2 && cxa >= x0 && cxa < x0 + MO &&
                                cya >= y0 && cya < y0 + MH;
            float2* a0 = AUX + (size_t(gy) * P + xc);
            float2 aux_old = make_float2(0.f, 0.f);
            if (aux_ok) aux_old = *a0;
            if (p3) {
                if (!euler) {
                    ho = __ldg(HAo + el); hoo = __ldg(HAoo + el);
                    go = __ldg(HBo + el); goo = __ldg(HBoo + el);
                    if (corr) { hp = __ldg(HAp + el); gp = __ldg(HBp + el); wcur = __ldg(Wcur + el); }
                }
                if (MIXED) wlo = __ldg(Lbase + el);
            }
            __syncthreads();  // (A) the previous row step is complete: its oldest ring slot is free
            if (tid == 0 && t + PREFETCH + 2 <= last_row) {
                fence_proxy_async();
                issue(t + PREFETCH + 2, sReq);
            }
            sReq = next_slot(sReq);
            if (!mbar_wait_bounded(&bars[s2p], par2p, tma_late ? 1 : (1 << 22))) tma_late = true;
            depth_row(o2p);
            const int bm = o0 + rc0, b0 = o1p + rc0, bp = o2p + rc0;  // rows t, t+1, t+2
            // ---- faces of row t+1 (Pass1), aux of that row, y flux between rows t and t+1 ----
            Face f;
            faces_at(ring, bm, b0, bp, c, f);
            const int par1 = (t + 1) & 1;
            fW[par1][0][tid] = f.hW; fW[par1][1][tid] = f.uW; fW[par1][2][tid] = f.vW; fW[par1][3][tid] = f.wW;
            if (aux_ok) {
                const float md = fmaxf((f.hN + f.hE + f.hS + f.hW) * 0.25f, aux_old.x);
                const float bw = (f.msd > M.tan_thr) ? 1.0f : aux_old.y;   // atan(msd) > threshold
                *a0 = make_float2(md, bw * decay);
            }
            const float g = c.g, hg = c.half_g;
            float yf[3];   // y flux at the north face of row t: north face of row t vs south face of row t+1
            face_flux(nh, nu, nv, nw, f.hS, f.uS, f.vS, f.wS, g, hg, false, yf);
            // ---- x flux at the east face of (xc, t): east face of row t (registers) vs west face of (xc+1, t)
            const int par = t & 1;
            {
                const int tn = min(tid + 1, MW - 1);
                float xo[3];
                face_flux(eh, eu, ev, ew, fW[par][0][tn], fW[par][1][tn], fW[par][2][tn], fW[par][3][tn], g, hg, true,
                          xo);
                xb[0][tid] = xo[0]; xb[1][tid] = xo[1]; xb[2][tid] = xo[2];
            }
            __syncthreads();  // (B)
            // ---- Pass3 at (xc, t) ----
            if (p3) {
                const int c0 = o0 + rc, cm = o1m + rc, cpp1 = o1p + rc;
                const int cmm = o2m + rc, cpp2 = o2p + rc;   // rows t, t-1, t+1, t-2, t+2
                const int d0 = c0;
                const float wc = W[c0], huc = HU[c0], hvc = HV[c0];
                const float BAh = BAr[c0], BXh = BXr[c0], BYh = BYr[c0];
                const float BXw = BXr[c0 - 1], BYs = BYr[cm];
                const float h = fmaxf(0.f, wc - BAh);
                const float dh = dring[d0], d2 = dh * dh, d3 = d2 * dh;
                const float dl = dring[d0 - 1], dr = dring[d0 + 1], dll = dring[d0 - 2], drr = dring[d0 + 2];
                const float ddn = dring[cm], du = dring[cpp1];
                const float ddd = dring[cmm], duu = dring[cpp2];
                // eta = w - sea level enters only through differences, where the sea level cancels
                const float e0 = wc, el_ = W[c0 - 1], er = W[c0 + 1], ed = W[cm], eu_ = W[cpp1];
                const float ell = W[c0 - 2], err = W[c0 + 2], edd = W[cmm], euu = W[cpp2];
                const float eul = W[cpp1 - 1], eur = W[cpp1 + 1], edl = W[cm - 1], edr = W[cm + 1];
                const float odx = c.one_over_dx, ody = c.one_over_dy;
                const float od2x = odx * odx, od3x = od2x * odx, od2y = ody * ody, od3y = od2y * ody;
                const float ddx = (-drr + 8 * dr - 8 * dl + dll) * odx * (1.0f / 12.0f);
                const float ddy = (-duu + 8 * du - 8 * ddn + ddd) * ody * (1.0f / 12.0f);
                const float exy = (0.25f * odx * ody * (eur - edr - eul + edl));
                const float exx = od2x * (er - 2 * e0 + el_);
                const float eyy = od2y * (eu_ - 2 * e0 + ed);
                const float Bg = c.Bcoef_g;
                const float P1x = Bg * (d3) * ((err - 2 * er + 2 * el_ - ell) * (0.5f * od3x) +
                                               (eur - eul - 2 * er + 2 * el_ + edr - edl) * (0.5f * odx * od2y));
                const float P2x = Bg * (d2) * (ddx * (2 * exx + eyy) + ddy * exy);
                const float P1y = Bg * (d3) * ((euu - 2 * eu_ + 2 * ed - edd) * (0.5f * od3y) +
                                               (eur + eul - 2 * eu_ + 2 * ed - edr - edl) * (0.5f * ody * od2x));
                const float P2y = Bg * (d2) * (ddy * (exx + 2 * eyy) + ddx * exy);
                const float fr = pa.friction ? friction_fast(huc, hvc, h, c.friction, c.is_manning, c.g, c.epsilon) : 0.f;
                const float s1 = -c.g_over_dx * h * (BXh - BXw) - huc * fr + (P1x + P2x);
                const float s2 = -c.g_over_dy * h * (BYh - BYs) - hvc * fr + (P1y + P2y);
                const int tw = max(tid - 1, 0);
                const float f0 = (xb[0][tw] - xb[0][tid]) * odx + (ypv0 - yf[0]) * ody;
                const float f1 = (xb[1][tw] - xb[1][tid]) * odx + (ypv1 - yf[1]) * ody + s1;
                const float f2 = (xb[2][tw] - xb[2][tid]) * odx + (ypv2 - yf[2]) * ody + s2;
                const float sixth = 1.0f / 6.0f;
                const float Fs = (sixth * dh * (ddx * ((ody * 0.5f) * (HV[cpp1] - HV[cm])) +
                                                (ddy * ((odx * 0.5f) * (HV[c0 + 1] - HV[c0 - 1])))));
                const float Gs = (sixth * dh * (ddx * ((ody * 0.5f) * (HU[cpp1] - HU[cm])) +
                                                (ddy * ((odx * 0.5f) * (HU[c0 + 1] - HU[c0 - 1])))));
                const float dt = dtm;
                float dw, rhu, rhv;
                float wbase = wc;
                if (euler) {
                    dw = dt * f0; rhu = dt * f1; rhv = dt * f2;
                } else if (!corr && ADAPT) {
                    // variable-step AB3 (compute.hlsl:766-780) with the member's coefficients
                    const float* q = M.ab;
                    const float kA = q[0], A0 = q[1], A1 = q[2], A2 = q[3], K0 = q[4], K1 = q[5], K2 = q[6];
                    dw = kA * (A0 * f0 + A1 * ho.x + A2 * hoo.x);
                    rhu = kA * (A0 * f1 + A1 * ho.y + A2 * hoo.y) + (K0 * Fs + K1 * ho.w + K2 * hoo.w);
                    rhv = kA * (A0 * f2 + A1 * ho.z + A2 * hoo.z) + (K0 * Gs + K1 * go + K2 * goo);
                } else if (!corr) {
                    const float k12 = dt * (1.0f / 12.0f);
                    dw = k12 * (23.0f * f0 - 16.0f * ho.x + 5.0f * hoo.x);
                    rhu = k12 * (23.0f * f1 - 16.0f * ho.y + 5.0f * hoo.y) + (2.0f * Fs - 3.0f * ho.w + hoo.w);
                    rhv = k12 * (23.0f * f2 - 16.0f * ho.z + 5.0f * hoo.z) + (2.0f * Gs - 3.0f * go + goo);
                } else {
                    const float k24 = dt * (1.0f / 24.0f);
                    dw = k24 * (9 * f0 + 19 * hp.x - 5 * ho.x + 1 * hoo.x);
                    rhu = k24 * (9 * f1 + 19 * hp.y - 5 * ho.y + 1 * hoo.y) + Fs - hp.w;
                    rhv = k24 * (9 * f2 + 19 * hp.z - 5 * ho.z + 1 * hoo.z) + Gs - gp;
                    wbase = wcur;
                }
                float wn = wbase, wl = wlo;
                if (MIXED) two_sum_add(wn, wl, dw);
                else wn = wbase + dw;
                if (out_col) {
                    Wout[e] = wn;
                    if (MIXED) Lout[e] = wl;
                    R0[e] = rhu;
                    R0[e + PL] = rhv;
                    HAs[e] = make_float4(f0, f1, f2, Fs);
                    HBs[e] = Gs;
                }
                if (stats) {   // GetStats (compute.hlsl:1319-1378) of the input state
                    const float q = div_by_h_fast(h, c.epsilon);
                    const float u = q * huc, v = q * hvc;
                    // cells outside the 4x4 blocks (and the halo threads) contribute zeros; selects,
                    // not products, so a halo value that is not finite cannot leak in
                    const bool blk = out_col && xc < 2 + 4 * (nx / 4) && t < 2 + 4 * (ny / 4);
                    const float u2v2 = u * u + v * v;
                    const float cc = sqrtf(c.g * h);
                    acc[0].add(blk ? h : 0.f); acc[1].add(blk ? h * (BAh + 0.5f * h) : 0.f);
                    acc[2].add(blk ? huc : 0.f); acc[3].add(blk ? hvc : 0.f);
                    acc[4].add(blk ? huc * u + hvc * v : 0.f);
                    mx[0] = fmaxf(mx[0], blk ? u2v2 : 0.f); mx[1] = fmaxf(mx[1], blk ? h : 0.f);
                    mx[2] = fmaxf(mx[2], blk ? fmaxf((fabsf(u) + cc) * odx, (fabsf(v) + cc) * ody) : 0.f);
                    mx[3] = fmaxf(mx[3], blk ? u2v2 * q : 0.f);
                    // volume in FP64 from the compensated state (w + its low word)
                    if (out_col) mfull += fmax(0.0, double(wc) - double(BAh) + (MIXED ? double(wlo) : 0.0));
                    bad = bad | (out_col & !(fabsf(wc) <= 3.0e38f && fabsf(huc) <= 3.0e38f && fabsf(hvc) <= 3.0e38f));
                }
            }
            ypv0 = yf[0]; ypv1 = yf[1]; ypv2 = yf[2];
            nh = f.hN; nu = f.uN; nv = f.vN; nw = f.wN;
            eh = f.hE; eu = f.uE; ev = f.vE; ew = f.wE;
            // advance the ring window: rows t-1 .. t+3 become t-2 .. t+2
            o2m = o1m; o1m = o0; o0 = o1p; o1p = o2p;
            o2p = (o2p + RSTR == RING * RSTR) ? 0 : o2p + RSTR;
            s2p = next_slot(s2p);
            if (s2p == 0) par2p ^= 1u;
            erow += size_t(P);
        }
        seq = seq0 + unsigned(last_row - (y0 - 2) + 1);
        // ---- zero the ghost ring of the output state next to this strip (engine.cpp:1007) ----
        const int NX = c.NX, NY = c.NY;
        const bool west = x0 == 2, east = x0 + MO >= nx + 2, south = y0 == 2, north = y0 + MH >= ny + 2;
        if (west || east || south || north) {
            const int cx0 = west ? 0 : x0, cx1 = east ? NX : x0 + MO;
            const int cy0 = south ? 0 : y0, cy1 = north ? NY : y0 + MH;
            const int w = cx1 - cx0;
            for (int k = tid; k < w * (cy1 - cy0); k += MW) {
                const int gx = cx0 + k % w, gy = cy0 + k / w;
                if (gx >= 2 && gx < nx + 2 && gy >= 2 && gy < ny + 2) continue;
                const size_t gi = size_t(gy) * P + gx;
                for (int q = 0; q < 3; ++q) {
                    Wout[gi + q * PL] = 0.f;
                    if (MIXED) Lout[gi + q * PL] = 0.f;
                }
            }
        }
        // ---- strip statistics -> member accumulators (statistics pass only) ----
        if (stats) {
            double sv[STATS_N];
            for (int k = 0; k < 5; ++k) sv[k] = acc[k].value();
            sv[5] = mfull;
            for (int k = 0; k < 4; ++k) sv[6 + k] = mx[k];
            sv[10] = bad ? 1.0 : 0.0;
            sv[11] = 0.0;
            for (int off = 16; off; off >>= 1)
                for (int k = 0; k < STATS_N - 1; ++k) {
                    const double o = __shfl_down_sync(0xffffffffu, sv[k], off);
                    sv[k] = (k >= 6) ? fmax(sv[k], o) : sv[k] + o;
                }
            // the reduction scratch reuses the ring: every row of this strip has been consumed and
            // the next strip requests rows only after its opening barrier
            double (*red)[STATS_N] = reinterpret_cast<double (*)[STATS_N]>(ring);
            const int lane = tid & 31, wid = tid >> 5;
            __syncthreads();
            if (lane == 0)
                for (int k = 0; k < STATS_N - 1; ++k) red[wid][k] = sv[k];
            __syncthreads();
            if (tid < STATS_N - 1) {
                double a = red[0][tid];
                for (int w = 1; w < MW / 32; ++w) a = (tid >= 6) ? fmax(a, red[w][tid]) : a + red[w][tid];
                if (tid < 6) { if (a != 0.0) atomicAdd(M.stats + tid, a); }
                else atomic_max_nonneg(M.stats + tid, a);
            }
        }
    }
    // a bounded TMA wait that gave up anywhere in this CTA marks the whole pass (the host reports
    // it as a CUDA error of the batch)
    if (__syncthreads_or(tma_late) && tid == 0) {
        drain_ring(bars, RING, requested);
        atomic_max_nonneg(pa.late_flag, 1.0);
    }
}

// ---------------------------------------------------------------------------------------------
// k_march2: the passes of k_march on two rows per step.  Every per-cell quantity is a pair
// (row t, row t+1) held in a float2, and arithmetic on pairs uses the paired single-precision
// instructions of sm_100 (__fadd2_rn, __fmul2_rn, __ffma2_rn): one instruction does the work of
// two cells.  The per-step bookkeeping (barriers, TMA requests, ring rotation, addressing) is paid
// once per two rows.  The faces run one step ahead of Pass3: step j computes the faces of rows
// t+2 and t+3 and uses those of rows t and t+1 from step j-1.  Ring: RING2 = 9 rows, the window
// t-2 .. t+4 plus the two rows requested one step ahead.
// ---------------------------------------------------------------------------------------------
// CTAs per SM the paired-row stencil is built for: 3 of 128 threads or 4 of 96 (12 warps either
// way, within the register file at up to 168 registers per thread)
constexpr int march2_min_ctas(int w) { return w == 128 ? MARCH2_MIN_CTAS : 4; }
constexpr int RING2 = 9;
constexpr int FSTR2 = RING2 * RSTR;
// the 9-row TMA ring of the paired-row stencil: fields w, hu, hv and the corner grid row above
// each cell row (the bottom BA, BX, BY is rebuilt from the corners)
constexpr size_t MARCH2_DYN_SMEM = sizeof(float) * 4 * FSTR2;
constexpr unsigned ROW_BYTES2 = (3u * RBOX + unsigned(CBOX)) * 4u;



typedef float2 f2;
__device__ __forceinline__ f2 P2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ f2 S2(float a) { return make_float2(a, a); }
__device__ __forceinline__ f2 add2(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 sub2(f2 a, f2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ f2 mul2(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 max2(f2 a, f2 b) { return P2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ f2 min2(f2 a, f2 b) { return P2(fminf(a.x, b.x), fminf(a.y, b.y)); }

__device__ __forceinline__ void recon2(f2 tt, f2 w, f2 c, f2 e, f2& ow, f2& oe) {
    const f2 z1 = mul2(tt, sub2(c, w)), z2 = sub2(e, w), z3 = mul2(tt, sub2(e, c));
    const f2 g2 = mul2(S2(0.25f), P2(minmod3_fast(z1.x, z2.x, z3.x), minmod3_fast(z1.y, z2.y, z3.y)));
    oe = add2(c, g2);
    ow = sub2(c, g2);
}
__device__ __forceinline__ void recon_sd2(f2 tt, f2 w, f2 c, f2 e, f2& ow, f2& oe, f2& sd) {
    const f2 z1 = mul2(tt, sub2(c, w)), z2 = sub2(e, w), z3 = mul2(tt, sub2(e, c));
    const f2 g2 = mul2(S2(0.25f), P2(minmod3_fast(z1.x, z2.x, z3.x), minmod3_fast(z1.y, z2.y, z3.y)));
    const f2 mu = mul2(S2(0.5f / 3.0f), add2(add2(z1, z2), z3));
    const f2 d1 = sub2(z1, mu), d2 = sub2(z2, mu), d3 = sub2(z3, mu);
    const f2 v = mul2(fma2(d1, d1, fma2(d2, d2, mul2(d3, d3))), S2(1.0f / 3.0f));
    sd = P2(sqrtf(v.x), sqrtf(v.y));
    oe = add2(c, g2);
    ow = sub2(c, g2);
}
__device__ __forceinline__ void correct_w2(f2 Bw, f2 Be, f2 wbar, f2& ww, f2& we) {
    float a = ww.x, b = we.x, c = ww.y, d = we.y;
    correct_w_fast(Bw.x, Be.x, wbar.x, a, b);
    correct_w_fast(Bw.y, Be.y, wbar.y, c, d);
    ww = P2(a, c);
    we = P2(b, d);
}
__device__ __forceinline__ f2 div_by_h2(f2 h, float eps) {
    const f2 h2 = mul2(h, h), h4 = mul2(h2, h2);
    const f2 t = add2(h4, max2(h4, S2(eps)));
    return mul2(mul2(S2(1.41421354f), h), P2(rsqrtf(t.x), rsqrtf(t.y)));
}

// The bottom of a pair of cells (rows r, r+1 of one column) from the corner grid, exactly as the
// host's prepare_bottom sums the corners (terrain_heightfield.cpp:213-297): BA = ((z00/4 + z10/4)
// + z01/4) + z11/4, BX = z10/2 + z11/2 (east edge), BY = z01/2 + z11/2 (north edge).  The
// products by powers of two are exact, so these sums round as the host's do with or without FMA
// contraction.  L0/R0: the left/right corners on the south edges of the two cells (corner rows
// r, r+1), L1/R1: on their north edges (corner rows r+1, r+2).
__device__ __forceinline__ f2 corner_mean2(f2 a, f2 b) { return fma2(S2(0.5f), b, mul2(S2(0.5f), a)); }
__device__ __forceinline__ f2 corner_mean4(f2 l0, f2 r0, f2 l1, f2 r1) {
    const f2 q = S2(0.25f);
    return fma2(q, r1, fma2(q, l1, fma2(q, r0, mul2(q, l0))));
}

struct Face2 { f2 hN, hE, hS, hW, uN, uE, uS, uW, vN, vE, vS, vW, wN, wE, wS, wW, msd; };
// what the next step needs of a pair's faces: north and east faces of both rows, south face of
// the second row (depth, velocities, water level)
struct Carry2 {
    f2 hN, uN, vN, wN, hE, uE, vE, wE;
    float hS1, uS1, vS1, wS1;
    __device__ __forceinline__ void set(const Face2& f) {
        hN = f.hN; uN = f.uN; vN = f.vN; wN = f.wN; hE = f.hE; uE = f.uE; vE = f.vE; wE = f.wE;
        hS1 = f.hS.y; uS1 = f.uS.y; vS1 = f.vS.y; wS1 = f.wS.y;
    }
};

// Pass1 on rows r and r+1 of one column: ring-row offsets of rows r-1, r, r+1, r+2 and the column.
__device__ __forceinline__ void faces_at2(const float* __restrict__ ring, int om1, int o0, int o1, int o2, int col,
                                          const SimConsts& c, Face2& f) {
    const float* W = ring;
    const float* HU = ring + FSTR2;
    const float* HV = ring + 2 * FSTR2;
    const float* Cr = ring + 3 * FSTR2;   // slot of row q holds corner row q+1
    const int a0 = o0 + col, a1 = o1 + col;
    const f2 tt = S2(c.two_theta);
    const f2 wc = P2(W[a0], W[a1]), wl = P2(W[a0 - 1], W[a1 - 1]), wr = P2(W[a0 + 1], W[a1 + 1]);
    const f2 wd = P2(W[om1 + col], W[a0]), wu = P2(W[a1], W[o2 + col]);
    // corners of cells (r, r+1): south edges in the slots of rows r-1, r; north edges in r, r+1
    const f2 L0 = P2(Cr[om1 + col], Cr[a0]), L1 = P2(Cr[a0], Cr[a1]);
    const f2 R0 = P2(Cr[om1 + col + 1], Cr[a0 + 1]), R1 = P2(Cr[a0 + 1], Cr[a1 + 1]);
    const f2 BN = corner_mean2(L1, R1), BE = corner_mean2(R0, R1);
    const f2 BS = corner_mean2(L0, R0), BW = corner_mean2(L0, L1);
    f2 wN, wE, wS, wW, huN, huE, huS, huW, hvN, hvE, hvS, hvW, sd1, sd2;
    recon_sd2(tt, wl, wc, wr, wW, wE, sd1);
    recon_sd2(tt, wd, wc, wu, wS, wN, sd2);
    const f2 huc = P2(HU[a0], HU[a1]), hvc = P2(HV[a0], HV[a1]);
    recon2(tt, P2(HU[a0 - 1], HU[a1 - 1]), huc, P2(HU[a0 + 1], HU[a1 + 1]), huW, huE);
    recon2(tt, P2(HU[om1 + col], HU[a0]), huc, P2(HU[a1], HU[o2 + col]), huS, huN);
    recon2(tt, P2(HV[a0 - 1], HV[a1 - 1]), hvc, P2(HV[a0 + 1], HV[a1 + 1]), hvW, hvE);
    recon2(tt, P2(HV[om1 + col], HV[a0]), hvc, P2(HV[a1], HV[o2 + col]), hvS, hvN);
    correct_w2(BW, BE, wc, wW, wE);
    correct_w2(BS, BN, wc, wS, wN);
    f.hN = sub2(wN, BN); f.hE = sub2(wE, BE); f.hS = sub2(wS, BS); f.hW = sub2(wW, BW);
    f.wN = wN; f.wE = wE; f.wS = wS; f.wW = wW;
    f2 q;
    q = div_by_h2(f.hN, c.epsilon); f.uN = mul2(q, huN); f.vN = mul2(q, hvN);
    q = div_by_h2(f.hE, c.epsilon); f.uE = mul2(q, huE); f.vE = mul2(q, hvE);
    q = div_by_h2(f.hS, c.epsilon); f.uS = mul2(q, huS); f.vS = mul2(q, hvS);
    q = div_by_h2(f.hW, c.epsilon); f.uW = mul2(q, huW); f.vW = mul2(q, hvW);
    f.msd = max2(mul2(sd1, S2(c.one_over_dx)), mul2(sd2, S2(c.one_over_dy)));
}

// KP07 fluxes through a pair of faces (m: lower-index side, p: the other); xdir selects the normal.
// The depth jump is taken from the face water levels, as in face_flux.
__device__ __forceinline__ void face_flux2(f2 hm, f2 um, f2 vm, f2 wm, f2 hp, f2 up, f2 vp, f2 wp, float g, float hg,
                                           bool xdir, f2 out[3]) {
    const f2 cm = P2(sqrtf(g * hm.x), sqrtf(g * hm.y)), cpp = P2(sqrtf(g * hp.x), sqrtf(g * hp.y));
    const f2 nm = xdir ? um : vm, np = xdir ? up : vp;
    const f2 ap = max2(max2(add2(nm, cm), add2(np, cpp)), S2(0.f));
    const f2 am = min2(min2(sub2(nm, cm), sub2(np, cpp)), S2(0.f));
    const f2 qp = mul2(hp, np), qm = mul2(hm, nm);
    const f2 hgv = S2(hg);
    f2 Fp[3], Fm[3], dU[3];
    Fp[0] = qp; Fm[0] = qm; dU[0] = sub2(wp, wm);
    if (xdir) {
        Fp[1] = mul2(hp, fma2(hgv, hp, mul2(up, up))); Fm[1] = mul2(hm, fma2(hgv, hm, mul2(um, um)));
        dU[1] = sub2(mul2(hp, up), mul2(hm, um));
        Fp[2] = mul2(qp, vp); Fm[2] = mul2(qm, vm); dU[2] = sub2(mul2(hp, vp), mul2(hm, vm));
    } else {
        Fp[1] = mul2(qp, up); Fm[1] = mul2(qm, um); dU[1] = sub2(mul2(hp, up), mul2(hm, um));
        Fp[2] = mul2(hp, fma2(hgv, hp, mul2(vp, vp))); Fm[2] = mul2(hm, fma2(hgv, hm, mul2(vm, vm)));
        dU[2] = sub2(mul2(hp, vp), mul2(hm, vm));
    }
    const f2 den = sub2(ap, am);
    const f2 inv = P2(den.x != 0.f ? rcp_newton(den.x) : 0.f, den.y != 0.f ? rcp_newton(den.y) : 0.f);
    const f2 apam = mul2(ap, am);
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = mul2(fma2(apam, dU[k], sub2(mul2(ap, Fm[k]), mul2(am, Fp[k]))), inv);
}

// Kahan accumulation of a pair of rows
struct Kahan2 {
    f2 s = make_float2(0.f, 0.f), c = make_float2(0.f, 0.f);
    __device__ __forceinline__ void add(f2 x) {
        const f2 y = sub2(x, c);
        const f2 t = add2(s, y);
        c = sub2(sub2(t, s), y);
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double(s.x) - double(c.x)) + (double(s.y) - double(c.y)); }
};

template <bool MIXED, bool ADAPT, int TW>
__global__ void __launch_bounds__(TW, march2_min_ctas(TW)) k_march2(const MemberDev* __restrict__ mems,
                                                               const int4* __restrict__ tiles, int ntiles, PassArgs pa) {
    extern __shared__ __align__(128) float ring[];   // 4 * FSTR2 floats: w, hu, hv, corner rows
    __shared__ float dring[RING2 * RSTR];   // still-water depth of each ring row (same stride as the ring)
    __shared__ __align__(8) unsigned long long bars[RING2];
    __shared__ float fW[2][2][4][TW];       // [step parity][row of the pair][hW, uW, vW, wW][thread]
    __shared__ float xb[2][3][TW];          // [row of the pair][component][thread]
    constexpr int OFF = MIXED ? 18 : 9;
    constexpr int iR0 = OFF + 3, iH0 = OFF + 5, iAUX = OFF + 25;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int k = 0; k < RING2; ++k) mbar_init(&bars[k], 1);
        mbar_fence_init();
    }
    __syncthreads();
    unsigned seq = 0;          // rows requested by this CTA so far (the same value in every thread)
    unsigned requested = 0;    // thread 0: sequence number of the last row it requested, plus one
    bool tma_late = false;
    const float* W = ring;
    const float* HU = ring + FSTR2;
    const float* HV = ring + 2 * FSTR2;
    const float* Cr = ring + 3 * FSTR2;   // slot of row q: corner row q+1
    const bool stats = pa.stats != 0;
    const bool corr = pa.scheme == CEL_SCHEME_CORRECTOR;
    const bool euler = pa.scheme == CEL_SCHEME_EULER;

    for (int it = blockIdx.x; it < ntiles; it += gridDim.x) {
        const int4 tl = tiles[it];
        const MemberDev& M = mems[tl.x];
        const SimConsts c = M.c;
        const int P = M.P, nx = c.nx, ny = c.ny, NYm1 = c.NY - 1;
        float* __restrict__ B = M.base;
        const size_t PL = M.plane;
        const CUtensorMap* tm = M.tmaps;
        const int x0 = tl.y, y0 = tl.z, MH = tl.w;
        const int xs = (x0 - 2) & ~3;          // TMA box start, 16-byte aligned
        const int xc = x0 - 1 + tid;           // this thread's column
        const int rc0 = xc - xs;               // its ring column (1 .. 131)
        const int rc = max(rc0, 2);            // Pass3 column (clamped for the halo thread 0)
        const int yend = min(y0 + MH, ny + 2);
        const int nsteps = (yend - y0 + 1) / 2;             // output row pairs of this strip
        const int last_row = y0 + 2 * (nsteps - 1) + 4;     // last row any step reads
        const bool out_col = tid >= 1 && tid <= (TW - 2) && xc < nx + 2;
        const int xl = min(xc, c.NX - 1);
        const float dtm = *M.dtp;
        const float decay = t_pow(fabsf(c.whitewater_decay_rate), dtm);
        const float sl = c.sea_level;
        const float4* __restrict__ HAo = reinterpret_cast<const float4*>(B + (iH0 + 5 * pa.og) * PL);
        const float4* __restrict__ HAoo = reinterpret_cast<const float4*>(B + (iH0 + 5 * pa.oog) * PL);
        const float4* __restrict__ HAp = reinterpret_cast<const float4*>(B + (iH0 + 5 * pa.pred) * PL);
        float4* __restrict__ HAs = reinterpret_cast<float4*>(B + (iH0 + 5 * pa.scr) * PL);
        const float* __restrict__ HBo = B + (iH0 + 5 * pa.og + 4) * PL;
        const float* __restrict__ HBoo = B + (iH0 + 5 * pa.oog + 4) * PL;
        const float* __restrict__ HBp = B + (iH0 + 5 * pa.pred + 4) * PL;
        float* __restrict__ HBs = B + (iH0 + 5 * pa.scr + 4) * PL;
        float* __restrict__ Wout = B + (3 * pa.out) * PL;
        const float* __restrict__ Wcur = B + (3 * pa.cur) * PL;
        float* __restrict__ R0 = B + iR0 * PL;
        float2* __restrict__ AUX = reinterpret_cast<float2*>(B + iAUX * PL);
        const float* __restrict__ Lbase = B + (9 + 3 * (corr ? pa.cur : pa.in)) * PL;
        float* __restrict__ Lout = B + (9 + 3 * pa.out) * PL;

        // row r of the strip has sequence number seq0 + (r - (y0 - 2)): slot seq % RING2, mbarrier
        // phase parity (seq / RING2) & 1
        const unsigned seq0 = seq;
        auto slot_of = [&](int r) { return int((seq0 + unsigned(r - (y0 - 2))) % RING2); };
        auto par_of = [&](int r) { return ((seq0 + unsigned(r - (y0 - 2))) / RING2) & 1u; };
        auto issue = [&](int row) {   // one thread: request a row's w, hu, hv and the corner row above it
            if (tma_late) return;       // a wait gave up: request nothing more
            requested = seq0 + unsigned(row - (y0 - 2)) + 1u;
            const int sl_ = slot_of(row);
            const int ry = min(row, NYm1);          // rows past the domain are never used; load the last
            mbar_expect_tx(&bars[sl_], ROW_BYTES2);
            float* dst = ring + sl_ * RSTR;
            tma_row(dst, tm + pa.in * 3 + 0, xs, ry, &bars[sl_]);
            tma_row(dst + FSTR2, tm + pa.in * 3 + 1, xs, ry, &bars[sl_]);
            tma_row(dst + 2 * FSTR2, tm + pa.in * 3 + 2, xs, ry, &bars[sl_]);
            tma_row(dst + 3 * FSTR2, tm + 12, xs, ry + 1, &bars[sl_]);   // corner rows 0 .. NY
        };
        auto wait_row = [&](int row) {
            if (!mbar_wait_bounded(&bars[slot_of(row)], par_of(row), tma_late ? 1 : (1 << 22))) tma_late = true;
        };
        // still-water depth of a ring row: thread k covers ring column rc0(thread 0) - 1 + k, and
        // threads 0 and 1 also the two columns past the last thread.  BA is rebuilt from the corner
        // rows in the slots of rows row-1 and row; the strip's first row (whose lower corner row is
        // not in the ring) reads BA from its plane (zero past the row, as the TMA fill would give).
        const int dcol = rc0 - 1;
        const int d2c = min(dcol + TW, RBOX - 1);
        auto depth_at = [&](int row, int k) {
            float ba;
            if (row == y0 - 2) {
                const int gx = xs + k;
                ba = gx < c.NX ? M.BA[size_t(row) * P + gx] : 0.f;
            } else {
                const float* lo = Cr + slot_of(row - 1) * RSTR;
                const float* up = Cr + slot_of(row) * RSTR;
                ba = fmaf(0.25f, up[k + 1], fmaf(0.25f, up[k], fmaf(0.25f, lo[k + 1], 0.25f * lo[k])));
            }
            return fmaxf(0.f, sl - ba);
        };
        auto depth_row = [&](int row) {
            float* dr = dring + slot_of(row) * RSTR;
            dr[dcol] = depth_at(row, dcol);
            if (tid < 2) dr[d2c] = depth_at(row, d2c);
        };

        Kahan2 acc[5];
        double mfull = 0.0;
        f2 mx[4] = {S2(0.f), S2(0.f), S2(0.f), S2(0.f)};
        bool bad = false;

        __syncthreads();  // the previous strip is done with shared memory
        if (tid == 0) {
            fence_proxy_async();
            for (int r = y0 - 2; r <= min(y0 + 2, last_row); ++r) issue(r);   // rows of the prologue and step -1
        }
        // prologue: faces of rows y0-2 and y0-1 (row y0-3's slot holds stale data: only row y0-2's
        // faces read it, and those are never used)
        wait_row(y0 - 2); wait_row(y0 - 1); wait_row(y0);
        depth_row(y0 - 2); depth_row(y0 - 1); depth_row(y0);
        Carry2 fp;   // faces of the previous step's rows (t, t+1 of the coming step)
        float ypv[3] = {0.f, 0.f, 0.f};   // y flux through the south face of row t (per component)
        {
        Face2 fq;
        faces_at2(ring, slot_of(y0 - 3) * RSTR, slot_of(y0 - 2) * RSTR, slot_of(y0 - 1) * RSTR, slot_of(y0) * RSTR,
                  rc0, c, fq);
        {
            const int pp = 1;   // parity of step -1
            fW[pp][0][0][tid] = fq.hW.x; fW[pp][0][1][tid] = fq.uW.x; fW[pp][0][2][tid] = fq.vW.x;
            fW[pp][1][0][tid] = fq.hW.y; fW[pp][1][1][tid] = fq.uW.y; fW[pp][1][2][tid] = fq.vW.y;
            fW[pp][0][3][tid] = fq.wW.x; fW[pp][1][3][tid] = fq.wW.y;
        }
        {   // aux of row y0-1 (the ghost row y = 1 belongs to the first strip)
            const int gy = y0 - 1;
            const int cxa = xc < 2 ? 2 : xc, cya = gy < 2 ? 2 : gy;
            if (xc >= 1 && xc < nx + 2 && gy >= 1 && cxa >= x0 && cxa < x0 + (TW - 2) && cya >= y0 && cya < y0 + MH) {
                float2* a = AUX + (size_t(gy) * P + xc);
                const float2 old = *a;
                const float md = (((fq.hN.y + fq.hE.y) + (fq.hS.y + fq.hW.y)) * 0.25f);
                const float bw = (fq.msd.y > M.tan_thr) ? 1.0f : old.y;
                *a = make_float2(fmaxf(md, old.x), bw * decay);
            }
        }
        fp.set(fq);
        }

        for (int j = -1; j < nsteps; ++j) {
            const int t = y0 + 2 * j;
            const bool p3 = j >= 0;
            const bool row1 = t + 1 < yend;                  // the second row of the pair exists
            const size_t e0 = size_t(t) * P + xc, e1 = e0 + P;
            const size_t l0 = size_t(t) * P + xl, l1 = l0 + P;
            // Pass3 inputs of rows t and t+1
            float4 ho0 = make_float4(0.f, 0.f, 0.f, 0.f), ho1 = ho0, hoo0 = ho0, hoo1 = ho0, hp0 = ho0, hp1 = ho0;
            f2 go = S2(0.f), goo = go, gp = go, wcur = go, wlo = go;
            if (p3) {
                if (!euler) {
                    ho0 = __ldg(HAo + l0); ho1 = __ldg(HAo + l1);
                    hoo0 = __ldg(HAoo + l0); hoo1 = __ldg(HAoo + l1);
                    go = P2(__ldg(HBo + l0), __ldg(HBo + l1));
                    goo = P2(__ldg(HBoo + l0), __ldg(HBoo + l1));
                    if (corr) {
                        hp0 = __ldg(HAp + l0); hp1 = __ldg(HAp + l1);
                        gp = P2(__ldg(HBp + l0), __ldg(HBp + l1));
                        wcur = P2(__ldg(Wcur + l0), __ldg(Wcur + l1));
                    }
                }
                if (MIXED) wlo = P2(__ldg(Lbase + l0), __ldg(Lbase + l1));
            }
            // aux texels of rows t+2 and t+3 owned by this strip, read-modify-written after their faces
            bool aux_ok[2];
            float2* ap[2];
            float2 aux_old[2];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int gy = t + 2 + k;
                const int cxa = xc < 2 ? 2 : xc, cya = gy < 2 ? 2 : gy;
                aux_ok[k] = xc >= 1 && xc < nx + 2 && gy >= 1 && gy < ny + 2 && cxa >= x0 && cxa < x0 + (TW - 2) &&
                            cya >= y0 && cya < y0 + MH;
                ap[k] = AUX + (size_t(min(gy, NYm1)) * P + xc);
                aux_old[k] = aux_ok[k] ? *ap[k] : make_float2(0.f, 0.f);
            }
            __syncthreads();  // (A) the previous step is complete: ring slots of rows t-4, t-3 are free
            if (tid == 0) {
                fence_proxy_async();
                if (t + 5 <= last_row) issue(t + 5);
                if (t + 6 <= last_row) issue(t + 6);
            }
            wait_row(t + 3);
            wait_row(t + 4);
            depth_row(t + 3);
            depth_row(t + 4);
            const int om2 = slot_of(t - 2) * RSTR, om1 = slot_of(t - 1) * RSTR, o0 = slot_of(t) * RSTR;
            const int o1 = slot_of(t + 1) * RSTR, o2 = slot_of(t + 2) * RSTR, o3 = slot_of(t + 3) * RSTR;
            const int o4 = slot_of(t + 4) * RSTR;
            // ---- faces of rows t+2, t+3 (Pass1), their aux, and the y fluxes of rows t, t+1 ----
            Face2 f;
            faces_at2(ring, o1, o2, o3, o4, rc0, c, f);
            const int npar = (j + 1) & 1, par = j & 1;
            fW[npar][0][0][tid] = f.hW.x; fW[npar][0][1][tid] = f.uW.x; fW[npar][0][2][tid] = f.vW.x;
            fW[npar][1][0][tid] = f.hW.y; fW[npar][1][1][tid] = f.uW.y; fW[npar][1][2][tid] = f.vW.y;
            fW[npar][0][3][tid] = f.wW.x; fW[npar][1][3][tid] = f.wW.y;
            {
                const f2 md = mul2(add2(add2(f.hN, f.hE), add2(f.hS, f.hW)), S2(0.25f));
                if (aux_ok[0]) {
                    const float bw = (f.msd.x > M.tan_thr) ? 1.0f : aux_old[0].y;   // atan(msd) > threshold
                    *ap[0] = make_float2(fmaxf(md.x, aux_old[0].x), bw * decay);
                }
                if (aux_ok[1]) {
                    const float bw = (f.msd.y > M.tan_thr) ? 1.0f : aux_old[1].y;
                    *ap[1] = make_float2(fmaxf(md.y, aux_old[1].x), bw * decay);
                }
            }
            const float g = c.g, hg = c.half_g;
            f2 yf[3];   // north faces of rows t, t+1: (N(t) vs S(t+1)), (N(t+1) vs S(t+2))
            face_flux2(fp.hN, fp.uN, fp.vN, fp.wN, P2(fp.hS1, f.hS.x), P2(fp.uS1, f.uS.x), P2(fp.vS1, f.vS.x),
                       P2(fp.wS1, f.wS.x), g, hg, false, yf);
            {   // x fluxes of rows t, t+1 at this thread's east face
                const int tn = min(tid + 1, TW - 1);
                f2 xo[3];
                face_flux2(fp.hE, fp.uE, fp.vE, fp.wE, P2(fW[par][0][0][tn], fW[par][1][0][tn]),
                           P2(fW[par][0][1][tn], fW[par][1][1][tn]), P2(fW[par][0][2][tn], fW[par][1][2][tn]),
                           P2(fW[par][0][3][tn], fW[par][1][3][tn]), g, hg, true, xo);
#pragma unroll
                for (int k = 0; k < 3; ++k) { xb[0][k][tid] = xo[k].x; xb[1][k][tid] = xo[k].y; }
            }
            __syncthreads();  // (B)
            // ---- Pass3 at (xc, t) and (xc, t+1) ----
            if (p3) {
                const int am2 = om2 + rc, am1 = om1 + rc, a0 = o0 + rc, a1 = o1 + rc, a2 = o2 + rc, a3 = o3 + rc;
                // rows t, t+1 as pairs; "d" = the row below, "u" = the row above
                const f2 wc = P2(W[a0], W[a1]);
                const f2 huc = P2(HU[a0], HU[a1]), hvc = P2(HV[a0], HV[a1]);
                // the bottom of cells (rc, t) and (rc, t+1) from the corner rows t .. t+2
                const f2 cL0 = P2(Cr[am1], Cr[a0]), cL1 = P2(Cr[a0], Cr[a1]);
                const f2 cR0 = P2(Cr[am1 + 1], Cr[a0 + 1]), cR1 = P2(Cr[a0 + 1], Cr[a1 + 1]);
                const f2 BAh = corner_mean4(cL0, cR0, cL1, cR1), BXh = corner_mean2(cR0, cR1);
                const f2 BYh = corner_mean2(cL1, cR1), BXw = corner_mean2(cL0, cL1), BYs = corner_mean2(cL0, cR0);
                const f2 h = max2(S2(0.f), sub2(wc, BAh));
                const f2 dh = P2(dring[a0], dring[a1]), d2 = mul2(dh, dh), d3 = mul2(d2, dh);
                const f2 dl = P2(dring[a0 - 1], dring[a1 - 1]), dr = P2(dring[a0 + 1], dring[a1 + 1]);
                const f2 dll = P2(dring[a0 - 2], dring[a1 - 2]), drr = P2(dring[a0 + 2], dring[a1 + 2]);
                const f2 ddn = P2(dring[am1], dring[a0]), du = P2(dring[a1], dring[a2]);
                const f2 ddd = P2(dring[am2], dring[am1]), duu = P2(dring[a2], dring[a3]);
                // eta = w - sea level enters only through differences, where the sea level cancels
                const f2 ec = wc, el_ = P2(W[a0 - 1], W[a1 - 1]), er = P2(W[a0 + 1], W[a1 + 1]);
                const f2 ed = P2(W[am1], W[a0]), eu_ = P2(W[a1], W[a2]);
                const f2 ell = P2(W[a0 - 2], W[a1 - 2]), err = P2(W[a0 + 2], W[a1 + 2]);
                const f2 edd = P2(W[am2], W[am1]), euu = P2(W[a2], W[a3]);
                const f2 eul = P2(W[a1 - 1], W[a2 - 1]), eur = P2(W[a1 + 1], W[a2 + 1]);
                const f2 edl = P2(W[am1 - 1], W[a0 - 1]), edr = P2(W[am1 + 1], W[a0 + 1]);
                const float odx = c.one_over_dx, ody = c.one_over_dy;
                const float od2x = odx * odx, od3x = od2x * odx, od2y = ody * ody, od3y = od2y * ody;
                const f2 two = S2(2.f), eight = S2(8.f);
                // (-r2 + 8 r1 - 8 l1 + l2) / 12 per unit length
                const f2 ddx = mul2(add2(sub2(fma2(eight, dr, P2(-drr.x, -drr.y)), mul2(eight, dl)), dll),
                                    S2(odx * (1.0f / 12.0f)));
                const f2 ddy = mul2(add2(sub2(fma2(eight, du, P2(-duu.x, -duu.y)), mul2(eight, ddn)), ddd),
                                    S2(ody * (1.0f / 12.0f)));
                const f2 exy = mul2(S2(0.25f * odx * ody), add2(sub2(sub2(eur, edr), eul), edl));
                const f2 exx = mul2(S2(od2x), add2(fma2(S2(-2.f), ec, er), el_));
                const f2 eyy = mul2(S2(od2y), add2(fma2(S2(-2.f), ec, eu_), ed));
                const f2 Bg = S2(c.Bcoef_g);
                const f2 P1x = mul2(mul2(Bg, d3),
                    fma2(sub2(fma2(two, el_, fma2(S2(-2.f), er, err)), ell), S2(0.5f * od3x),
                         mul2(sub2(add2(fma2(two, el_, fma2(S2(-2.f), er, sub2(eur, eul))), edr), edl),
                              S2(0.5f * odx * od2y))));
                const f2 P2x = mul2(mul2(Bg, d2), fma2(ddx, fma2(two, exx, eyy), mul2(ddy, exy)));
                const f2 P1y = mul2(mul2(Bg, d3),
                    fma2(sub2(fma2(two, ed, fma2(S2(-2.f), eu_, euu)), edd), S2(0.5f * od3y),
                         mul2(sub2(sub2(fma2(two, ed, fma2(S2(-2.f), eu_, add2(eur, eul))), edr), edl),
                              S2(0.5f * ody * od2x))));
                const f2 P2y = mul2(mul2(Bg, d2), fma2(ddy, fma2(two, eyy, exx), mul2(ddx, exy)));
                f2 fr = S2(0.f);
                if (pa.friction)
                    fr = P2(friction_fast(huc.x, hvc.x, h.x, c.friction, c.is_manning, c.g, c.epsilon),
                            friction_fast(huc.y, hvc.y, h.y, c.friction, c.is_manning, c.g, c.epsilon));
                const f2 s1 = add2(sub2(mul2(mul2(S2(-c.g_over_dx), h), sub2(BXh, BXw)), mul2(huc, fr)), add2(P1x, P2x));
                const f2 s2 = add2(sub2(mul2(mul2(S2(-c.g_over_dy), h), sub2(BYh, BYs)), mul2(hvc, fr)), add2(P1y, P2y));
                const int tw = max(tid - 1, 0);
                f2 fl[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    // x fluxes: west face (the neighbour's east face) minus east face; y fluxes: the
                    // south faces of rows t, t+1 are the north faces of rows t-1, t
                    const f2 xw = P2(xb[0][k][tw], xb[1][k][tw]), xh = P2(xb[0][k][tid], xb[1][k][tid]);
                    const f2 ys = P2(ypv[k], yf[k].x);
                    fl[k] = fma2(sub2(xw, xh), S2(odx), mul2(sub2(ys, yf[k]), S2(ody)));
                }
                const f2 f0 = fl[0], f1 = add2(fl[1], s1), f2v = add2(fl[2], s2);
                const f2 sixth = S2(1.0f / 6.0f);
                const f2 Fs = mul2(mul2(sixth, dh),
                                   fma2(ddx, mul2(S2(ody * 0.5f), sub2(P2(HV[a1], HV[a2]), P2(HV[am1], HV[a0]))),
                                        mul2(ddy, mul2(S2(odx * 0.5f), sub2(P2(HV[a0 + 1], HV[a1 + 1]), P2(HV[a0 - 1], HV[a1 - 1]))))));
                const f2 Gs = mul2(mul2(sixth, dh),
                                   fma2(ddx, mul2(S2(ody * 0.5f), sub2(P2(HU[a1], HU[a2]), P2(HU[am1], HU[a0]))),
                                        mul2(ddy, mul2(S2(odx * 0.5f), sub2(P2(HU[a0 + 1], HU[a1 + 1]), P2(HU[a0 - 1], HU[a1 - 1]))))));
                const f2 dt = S2(dtm);
                f2 dw, rhu, rhv;
                f2 wbase = wc;
                if (euler) {
                    dw = mul2(dt, f0); rhu = mul2(dt, f1); rhv = mul2(dt, f2v);
                } else if (!corr && ADAPT) {
                    // variable-step AB3 (compute.hlsl:766-780) with the member's coefficients
                    const float* q = M.ab;
                    const f2 kA = S2(q[0]), A0 = S2(q[1]), A1 = S2(q[2]), A2 = S2(q[3]);
                    const f2 K0 = S2(q[4]), K1 = S2(q[5]), K2 = S2(q[6]);
                    const f2 o_x = P2(ho0.x, ho1.x), o_y = P2(ho0.y, ho1.y), o_z = P2(ho0.z, ho1.z), o_w = P2(ho0.w, ho1.w);
                    const f2 q_x = P2(hoo0.x, hoo1.x), q_y = P2(hoo0.y, hoo1.y), q_z = P2(hoo0.z, hoo1.z), q_w = P2(hoo0.w, hoo1.w);
                    dw = mul2(kA, fma2(A2, q_x, fma2(A1, o_x, mul2(A0, f0))));
                    rhu = fma2(kA, fma2(A2, q_y, fma2(A1, o_y, mul2(A0, f1))), fma2(K2, q_w, fma2(K1, o_w, mul2(K0, Fs))));
                    rhv = fma2(kA, fma2(A2, q_z, fma2(A1, o_z, mul2(A0, f2v))), fma2(K2, goo, fma2(K1, go, mul2(K0, Gs))));
                } else if (!corr) {
                    const f2 k12 = S2(dtm * (1.0f / 12.0f));
                    const f2 o_x = P2(ho0.x, ho1.x), o_y = P2(ho0.y, ho1.y), o_z = P2(ho0.z, ho1.z), o_w = P2(ho0.w, ho1.w);
                    const f2 q_x = P2(hoo0.x, hoo1.x), q_y = P2(hoo0.y, hoo1.y), q_z = P2(hoo0.z, hoo1.z), q_w = P2(hoo0.w, hoo1.w);
                    const f2 c23 = S2(23.0f), c16 = S2(-16.0f), c5 = S2(5.0f);
                    dw = mul2(k12, fma2(c5, q_x, fma2(c16, o_x, mul2(c23, f0))));
                    rhu = fma2(k12, fma2(c5, q_y, fma2(c16, o_y, mul2(c23, f1))), add2(fma2(S2(-3.f), o_w, mul2(two, Fs)), q_w));
                    rhv = fma2(k12, fma2(c5, q_z, fma2(c16, o_z, mul2(c23, f2v))), add2(fma2(S2(-3.f), go, mul2(two, Gs)), goo));
                } else {
                    const f2 k24 = S2(dtm * (1.0f / 24.0f));
                    const f2 o_x = P2(ho0.x, ho1.x), o_y = P2(ho0.y, ho1.y), o_z = P2(ho0.z, ho1.z);
                    const f2 q_x = P2(hoo0.x, hoo1.x), q_y = P2(hoo0.y, hoo1.y), q_z = P2(hoo0.z, hoo1.z);
                    const f2 p_x = P2(hp0.x, hp1.x), p_y = P2(hp0.y, hp1.y), p_z = P2(hp0.z, hp1.z), p_w = P2(hp0.w, hp1.w);
                    const f2 c9 = S2(9.f), c19 = S2(19.f), c5 = S2(-5.f);
                    dw = mul2(k24, add2(fma2(c5, o_x, fma2(c19, p_x, mul2(c9, f0))), q_x));
                    rhu = add2(fma2(k24, add2(fma2(c5, o_y, fma2(c19, p_y, mul2(c9, f1))), q_y), Fs), P2(-p_w.x, -p_w.y));
                    rhv = add2(fma2(k24, add2(fma2(c5, o_z, fma2(c19, p_z, mul2(c9, f2v))), q_z), Gs), P2(-gp.x, -gp.y));
                    wbase = wcur;
                }
                f2 wn = wbase, wl = wlo;
                if (MIXED) {
                    float a = wn.x, b = wl.x, cc = wn.y, d = wl.y;
                    two_sum_add(a, b, dw.x);
                    two_sum_add(cc, d, dw.y);
                    wn = P2(a, cc); wl = P2(b, d);
                } else {
                    wn = add2(wbase, dw);
                }
                if (out_col) {
                    Wout[e0] = wn.x;
                    if (MIXED) Lout[e0] = wl.x;
                    R0[e0] = rhu.x;
                    R0[e0 + PL] = rhv.x;
                    HAs[e0] = make_float4(f0.x, f1.x, f2v.x, Fs.x);
                    HBs[e0] = Gs.x;
                    if (row1) {
                        Wout[e1] = wn.y;
                        if (MIXED) Lout[e1] = wl.y;
                        R0[e1] = rhu.y;
                        R0[e1 + PL] = rhv.y;
                        HAs[e1] = make_float4(f0.y, f1.y, f2v.y, Fs.y);
                        HBs[e1] = Gs.y;
                    }
                }
                if (stats) {   // GetStats (compute.hlsl:1319-1378) of the input state
                    const f2 q = div_by_h2(h, c.epsilon);
                    const f2 u = mul2(q, huc), v = mul2(q, hvc);
                    const bool in_cols = out_col && xc < 2 + 4 * (nx / 4);
                    const bool b0 = in_cols && t < 2 + 4 * (ny / 4), b1 = in_cols && row1 && t + 1 < 2 + 4 * (ny / 4);
                    const bool a0_ = out_col, a1_ = out_col && row1;
                    auto pick = [](bool k0, bool k1, f2 v_) { return P2(k0 ? v_.x : 0.f, k1 ? v_.y : 0.f); };
                    const f2 u2v2 = fma2(u, u, mul2(v, v));
                    const f2 cc = P2(sqrtf(c.g * h.x), sqrtf(c.g * h.y));
                    acc[0].add(pick(b0, b1, h));
                    acc[1].add(pick(b0, b1, mul2(h, fma2(S2(0.5f), h, BAh))));
                    acc[2].add(pick(b0, b1, huc));
                    acc[3].add(pick(b0, b1, hvc));
                    acc[4].add(pick(b0, b1, fma2(huc, u, mul2(hvc, v))));
                    mx[0] = max2(mx[0], pick(b0, b1, u2v2));
                    mx[1] = max2(mx[1], pick(b0, b1, h));
                    const f2 cx = mul2(add2(P2(fabsf(u.x), fabsf(u.y)), cc), S2(odx));
                    const f2 cy = mul2(add2(P2(fabsf(v.x), fabsf(v.y)), cc), S2(ody));
                    mx[2] = max2(mx[2], pick(b0, b1, max2(cx, cy)));
                    mx[3] = max2(mx[3], pick(b0, b1, mul2(u2v2, q)));
                    // volume in FP64 from the compensated state (w + its low word)
                    if (a0_) mfull += fmax(0.0, double(wc.x) - double(BAh.x) + (MIXED ? double(wlo.x) : 0.0));
                    if (a1_) mfull += fmax(0.0, double(wc.y) - double(BAh.y) + (MIXED ? double(wlo.y) : 0.0));
                    const bool nb0 = !(fabsf(wc.x) <= 3.0e38f && fabsf(huc.x) <= 3.0e38f && fabsf(hvc.x) <= 3.0e38f);
                    const bool nb1 = !(fabsf(wc.y) <= 3.0e38f && fabsf(huc.y) <= 3.0e38f && fabsf(hvc.y) <= 3.0e38f);
                    bad = bad | (a0_ & nb0) | (a1_ & nb1);
                }
            }
            // the y flux through the north face of row t+1 is the south flux of the next pair's first row
            ypv[0] = yf[0].y; ypv[1] = yf[1].y; ypv[2] = yf[2].y;
            fp.set(f);
        }
        seq = seq0 + unsigned(last_row - (y0 - 2) + 1);
        // ---- zero the ghost ring of the output state next to this strip (engine.cpp:1007) ----
        const int NX = c.NX, NY = c.NY;
        const bool west = x0 == 2, east = x0 + (TW - 2) >= nx + 2, south = y0 == 2, north = y0 + MH >= ny + 2;
        if (west || east || south || north) {
            const int cx0 = west ? 0 : x0, cx1 = east ? NX : x0 + (TW - 2);
            const int cy0 = south ? 0 : y0, cy1 = north ? NY : y0 + MH;
            const int w = cx1 - cx0;
            for (int k = tid; k < w * (cy1 - cy0); k += TW) {
                const int gx = cx0 + k % w, gy = cy0 + k / w;
                if (gx >= 2 && gx < nx + 2 && gy >= 2 && gy < ny + 2) continue;
                const size_t gi = size_t(gy) * P + gx;
                for (int q = 0; q < 3; ++q) {
                    Wout[gi + q * PL] = 0.f;
                    if (MIXED) Lout[gi + q * PL] = 0.f;
                }
            }
        }
        if (stats) {
            double sv[STATS_N];
            for (int k = 0; k < 5; ++k) sv[k] = acc[k].value();
            sv[5] = mfull;
            for (int k = 0; k < 4; ++k) sv[6 + k] = fmaxf(mx[k].x, mx[k].y);
            sv[10] = bad ? 1.0 : 0.0;
            sv[11] = 0.0;
            for (int off = 16; off; off >>= 1)
                for (int k = 0; k < STATS_N - 1; ++k) {
                    const double o = __shfl_down_sync(0xffffffffu, sv[k], off);
                    sv[k] = (k >= 6) ? fmax(sv[k], o) : sv[k] + o;
                }
            double (*red)[STATS_N] = reinterpret_cast<double (*)[STATS_N]>(ring);
            const int lane = tid & 31, wid = tid >> 5;
            __syncthreads();
            if (lane == 0)
                for (int k = 0; k < STATS_N - 1; ++k) red[wid][k] = sv[k];
            __syncthreads();
            if (tid < STATS_N - 1) {
                double a = red[0][tid];
                for (int w = 1; w < TW / 32; ++w) a = (tid >= 6) ? fmax(a, red[w][tid]) : a + red[w][tid];
                if (tid < 6) { if (a != 0.0) atomicAdd(M.stats + tid, a); }
                else atomic_max_nonneg(M.stats + tid, a);
            }
        }
    }
    if (__syncthreads_or(tma_late) && tid == 0) {
        drain_ring(bars, RING2, requested);
        atomic_max_nonneg(pa.late_flag, 1.0);
    }
}

// Stats of the current state only (resetTimestep on demand).
__global__ void __launch_bounds__(256) k_stats_only(const MemberDev* __restrict__ mems, const int4* __restrict__ tiles,
                                                    int ntiles, int buf) {
    __shared__ double red[256 / 32][STATS_N];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int4 tl = tiles[t];
        const MemberDev& M = mems[tl.x];
        const SimConsts c = M.c;
        for (int sub = 0; sub < (TX * TY) / 256; ++sub) {
            const int k = sub * 256 + threadIdx.x;
            const int gx = tl.y + k % TX, gy = tl.z + k / TX;
            const bool valid = gx < c.nx + 2 && gy < c.ny + 2;
            float h = 0, B = 0, hu = 0, hv = 0, u = 0, v = 0, q = 0, cc = 0;
            double h64 = 0.0;
            bool bad = false;
            if (valid) {
                const size_t gi = size_t(gy) * M.P + gx;
                const float w = M.S[buf][0][gi];
                hu = M.S[buf][1][gi]; hv = M.S[buf][2][gi]; B = M.BA[gi];
                h = fmaxf(0.f, w - B);
                // the volume total in FP64 from the compensated state where there is one (the FP32
                // difference w - B drops positive parts of eta below half an ulp of the depth)
                h64 = fmax(0.0, double(w) - double(B) + (M.L[buf][0] ? double(M.L[buf][0][gi]) : 0.0));
                q = div_by_h(h, c.epsilon);
                u = q * hu; v = q * hv;
                cc = sqrtf(c.g * h);
                bad = !isfinite(w) || !isfinite(hu) || !isfinite(hv);
            }
            const bool in_block = valid && gx < 2 + 4 * (c.nx / 4) && gy < 2 + 4 * (c.ny / 4);
            stats_reduce(M.stats_now, in_block, valid, h, h64, B, hu, hv, u, v, q, cc, c.one_over_dx, c.one_over_dy, bad,
                         red);
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Tridiagonal solves.  For one system with Thomas factors (c', inv, m):
//   forward   d'_i = inv_i r_i + m_i d'_{i-1}
//   backward  x_i  = d'_i - c'_i x_{i+1}
// Each thread runs both recurrences over a contiguous chunk with zero carry-in; the chunk
// transfer maps (product of multipliers, local end value) are combined by a scan and the
// chunk values are corrected with the running products.
// ---------------------------------------------------------------------------------------------
struct Affine { float a, b; };  // x -> b + a x

__device__ __forceinline__ Affine compose(const Affine& later, const Affine& earlier) {
    return Affine{later.a * earlier.a, later.b + later.a * earlier.b};
}



// Row (x) solves, one warp per row.  A row is swept in tiles of RT = 256 columns; lane j owns the
// RK = 8 consecutive columns tile*256 + 8j .. +7 (two float4 loads per array, 16-byte aligned
// since rows start on 128-byte boundaries).  Within a tile each lane runs the recurrence over its
// 8 columns from zero, the lanes' affine transfer maps are combined by a warp shuffle scan, and
// the tile's carry passes to the next tile.  Columns outside the interior [2, nx+2) are identity
// rows (m = c' = 0, right-hand side 0).  The forward values are kept in shared memory for the
// backward sweep, which walks the tiles in reverse with the mirrored scan and writes
// hu = hu_base + x (two-sum into the low word in the mixed form).
constexpr int RK = 8, RT = 32 * RK;

__device__ __forceinline__ Affine shfl_up_affine(const Affine& v, int off) {
    return Affine{__shfl_up_sync(0xffffffffu, v.a, off), __shfl_up_sync(0xffffffffu, v.b, off)};
}
__device__ __forceinline__ Affine shfl_down_affine(const Affine& v, int off) {
    return Affine{__shfl_down_sync(0xffffffffu, v.a, off), __shfl_down_sync(0xffffffffu, v.b, off)};
}
__device__ __forceinline__ void load8(const float* __restrict__ p, int c, int ncol, float v[RK]) {
    // columns c .. c+7 of a row; a float4 is loaded only when it starts inside [0, ncol) (then it
    // lies inside the row, whose pitch is a multiple of 32 and at least ncol + 2)
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 a = c < ncol ? __ldg(reinterpret_cast<const float4*>(p + c)) : z;
    const float4 b = c + 4 < ncol ? __ldg(reinterpret_cast<const float4*>(p + c + 4)) : z;
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}

template <bool MIXED>
__global__ void __launch_bounds__(256) k_rows(const MemberDev* __restrict__ mems, const int2* __restrict__ rows,
                                              int nrows, int rowbuf, PassArgs pa) {
    extern __shared__ float4 rsm4[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    float* __restrict__ ybuf = reinterpret_cast<float*>(rsm4) + size_t(wid) * rowbuf;
    const int base_buf = (pa.scheme == CEL_SCHEME_CORRECTOR) ? pa.cur : pa.in;
    for (int it = blockIdx.x * nw + wid; it < nrows; it += gridDim.x * nw) {
        const int2 rw = rows[it];
        const MemberDev& M = mems[rw.x];
        const int nx = M.c.nx;
        const size_t row = size_t(rw.y) * M.P;
        const int ncol = nx + 2;                       // columns [0, nx+2) are swept
        const int ntile = (ncol + RT - 1) / RT;
        const float* __restrict__ r = M.R[0] + row;
        const float* __restrict__ cpp = M.FX[0] + row;
        const float* __restrict__ inv = M.FX[1] + row;
        const float* __restrict__ mm = M.FX[2] + row;
        // ---- forward: y_i = inv_i r_i + m_i y_{i-1}; the next tile's loads are issued before the
        // current tile is computed ----
        float carry = 0.f;
        float rn[RK], in_[RK], mn[RK];
        load8(r, lane * RK, ncol, rn);
        load8(inv, lane * RK, ncol, in_);
        load8(mm, lane * RK, ncol, mn);
        for (int ti = 0; ti < ntile; ++ti) {
            const int c0 = ti * RT + lane * RK;
            float rv[RK], iv[RK], mv[RK], yv[RK];
#pragma unroll
            for (int k = 0; k < RK; ++k) { rv[k] = rn[k]; iv[k] = in_[k]; mv[k] = mn[k]; }
            if (ti + 1 < ntile) {
                load8(r, c0 + RT, ncol, rn);
                load8(inv, c0 + RT, ncol, in_);
                load8(mm, c0 + RT, ncol, mn);
            }
            float a = 1.f, b = 0.f;
#pragma unroll
            for (int k = 0; k < RK; ++k) {
                const bool ok = c0 + k >= 2 && c0 + k < ncol;
                const float m = ok ? mv[k] : 0.f;
                b = (ok ? iv[k] * rv[k] : 0.f) + m * b;
                a *= m;
                yv[k] = b;
                mv[k] = m;
            }
            Affine inc{a, b};
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const Affine o = shfl_up_affine(inc, off);
                if (lane >= off) inc = compose(inc, o);
            }
            const Affine before = shfl_up_affine(inc, 1);
            const float cin = lane > 0 ? before.b + before.a * carry : carry;
            float pref = 1.f;
#pragma unroll
            for (int k = 0; k < RK; ++k) {
                pref *= mv[k];
                yv[k] += pref * cin;
            }
            float4* yb = reinterpret_cast<float4*>(ybuf + c0);
            yb[0] = make_float4(yv[0], yv[1], yv[2], yv[3]);
            yb[1] = make_float4(yv[4], yv[5], yv[6], yv[7]);
            carry = __shfl_sync(0xffffffffu, inc.b + inc.a * carry, 31);
        }
        // ---- backward: x_i = y_i - c'_i x_{i+1}; hu = base + x (each lane reads back its own
        // chunks of the forward buffer, so no synchronisation is needed) ----
        float* __restrict__ ohi = M.S[pa.out][1] + row;
        const float* __restrict__ bhi = M.S[base_buf][1] + row;
        float* __restrict__ olo = MIXED ? M.L[pa.out][1] + row : nullptr;
        const float* __restrict__ blo = MIXED ? M.L[base_buf][1] + row : nullptr;
        float xcarry = 0.f;
        float cn_[RK], bhn[RK], bln[RK];
        {
            const int cl = (ntile - 1) * RT + lane * RK;
            load8(cpp, cl, ncol, cn_);
            load8(bhi, cl, ncol, bhn);
            if (MIXED) load8(blo, cl, ncol, bln);
        }
        for (int ti = ntile - 1; ti >= 0; --ti) {
            const int c0 = ti * RT + lane * RK;
            float cv[RK], yv[RK], bh[RK], bl[RK];
#pragma unroll
            for (int k = 0; k < RK; ++k) { cv[k] = cn_[k]; bh[k] = bhn[k]; bl[k] = MIXED ? bln[k] : 0.f; }
            if (ti > 0) {
                load8(cpp, c0 - RT, ncol, cn_);
                load8(bhi, c0 - RT, ncol, bhn);
                if (MIXED) load8(blo, c0 - RT, ncol, bln);
            }
            {
                const float4* yb = reinterpret_cast<const float4*>(ybuf + c0);
                const float4 p = yb[0], q = yb[1];
                yv[0] = p.x; yv[1] = p.y; yv[2] = p.z; yv[3] = p.w; yv[4] = q.x; yv[5] = q.y; yv[6] = q.z; yv[7] = q.w;
            }
            float z = 0.f, qa = 1.f;
#pragma unroll
            for (int k = RK - 1; k >= 0; --k) {
                const bool ok = c0 + k >= 2 && c0 + k < ncol;
                const float cn = ok ? -cv[k] : 0.f;
                z = yv[k] + cn * z;
                qa *= cn;
                yv[k] = z;
                cv[k] = cn;
            }
            Affine inc{qa, z};
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const Affine o = shfl_down_affine(inc, off);
                if (lane + off < 32) inc = compose(inc, o);
            }
            const Affine after = shfl_down_affine(inc, 1);
            const float cnext = lane < 31 ? after.b + after.a * xcarry : xcarry;
            float suf = 1.f;
#pragma unroll
            for (int k = RK - 1; k >= 0; --k) {
                suf *= cv[k];
                yv[k] += suf * cnext;
            }
            xcarry = __shfl_sync(0xffffffffu, inc.b + inc.a * xcarry, 0);
            float oh[RK], ol[RK];
#pragma unroll
            for (int k = 0; k < RK; ++k) {
                if (MIXED) {
                    float hi = bh[k], lo = bl[k];
                    two_sum_add(hi, lo, yv[k]);
                    oh[k] = hi; ol[k] = lo;
                } else {
                    oh[k] = bh[k] + yv[k];
                }
            }
            if (c0 >= 2 && c0 + RK <= ncol) {
                reinterpret_cast<float4*>(ohi + c0)[0] = make_float4(oh[0], oh[1], oh[2], oh[3]);
                reinterpret_cast<float4*>(ohi + c0)[1] = make_float4(oh[4], oh[5], oh[6], oh[7]);
                if (MIXED) {
                    reinterpret_cast<float4*>(olo + c0)[0] = make_float4(ol[0], ol[1], ol[2], ol[3]);
                    reinterpret_cast<float4*>(olo + c0)[1] = make_float4(ol[4], ol[5], ol[6], ol[7]);
                }
            } else {
#pragma unroll
                for (int k = 0; k < RK; ++k)
                    if (c0 + k >= 2 && c0 + k < ncol) {
                        ohi[c0 + k] = oh[k];
                        if (MIXED) olo[c0 + k] = ol[k];
                    }
            }
        }
    }
}

template <bool MIXED, int CW, int NT>
__global__ void __launch_bounds__(NT, cols_min_ctas(NT)) k_cols(const MemberDev* __restrict__ mems, const int2* __restrict__ bands,
                                              int nbands, PassArgs pa) {
    // Column (y) solves: a CTA takes a band of CW adjacent columns, thread (c, k) runs chunk k of
    // column c; CW consecutive threads read CW consecutive floats of one row.  Every loop over a
    // chunk's rows issues the loads of CU rows before using them, so each thread keeps several rows
    // of requests in flight (the recurrences themselves are serial).  Three walks over a chunk:
    //   1. down: the forward sweep from zero, y0_i (kept in shared memory), with the chunk's forward
    //      map y_end = A y_in + y0_end and, from the same values, its backward map in terms of the
    //      carry in: x_top = Q x_below + Z0 + Z1 y_in (Q = prod(-c'), Z0 = sum q_i y0_i,
    //      Z1 = sum q_i P_i with q_i = prod_{j<i}(-c'_j), P_i = prod_{j<=i} m_j, since
    //      y_i = y0_i + P_i y_in);
    //   then the carries into every chunk of the forward sweep and, right after, of the backward
    //   sweep, each by recursive doubling over the chunks of a column (warp shuffles), i.e. parallel
    //   reduction of the L and U sweeps down to chunks of ceil(ny / NCH) rows swept serially;
    //   2. down: y_i = y0_i + P_i y_in;
    //   3. up: x_i = y_i - c'_i x_{i+1} from the chunk's carry, hv = base + x.
    constexpr int NTC = NT;
    constexpr int NCH = NTC / CW;
    // carry scans: one warp per column; each of the first LN lanes holds G consecutive chunks
    constexpr int G = NCH >= 32 ? NCH / 32 : 1;
    constexpr int LN = NCH >= 32 ? 32 : NCH;
    static_assert(NCH % LN == 0, "carry scan layout");
    constexpr int CU = 8;
    extern __shared__ float cs[];
    __shared__ float carP[NCH][CW], carY[NCH][CW], carQ[NCH][CW], carZ0[NCH][CW], carZ1[NCH][CW];
    __shared__ float cin_f[NCH][CW], cin_b[NCH][CW];
    const int c = threadIdx.x % CW, k = threadIdx.x / CW;
    for (int it = blockIdx.x; it < nbands; it += gridDim.x) {
        const int2 bd = bands[it];
        const MemberDev& M = mems[bd.x];
        const int n = M.c.ny, P = M.P;
        const int gx = bd.y + c;
        const bool col_ok = gx >= 2 && gx < M.c.nx + 2;
        const int mc = (n + NCH - 1) / NCH;
        const int i0 = min(n, k * mc), i1 = min(n, i0 + mc);
        const float* __restrict__ r = M.R[1] + gx;
        // factors band-major: a chunk's rows of this band are contiguous (CW floats apart)
        const size_t fb = size_t(bd.y / CW) * n * CW + c;
        const float* __restrict__ cp = M.FYB[0] + fb;
        const float* __restrict__ inv = M.FYB[1] + fb;
        const float* __restrict__ mm = M.FYB[2] + fb;
        auto at = [&](int i) { return size_t(i + 2) * P; };   // row offset of system element i
        auto atf = [&](int i) { return size_t(i) * CW; };     // factor offset of system element i
        __syncthreads();
        float yv = 0.f, pa_ = 1.f, q = 1.f, z0 = 0.f, z1 = 0.f;
        if (col_ok)
            for (int i = i0; i < i1; i += CU) {
                float mv[CU], iv[CU], rv[CU], cv[CU];
#pragma unroll
                for (int u = 0; u < CU; ++u) {
                    const bool ok = i + u < i1;
                    mv[u] = ok ? __ldg(mm + atf(i + u)) : 0.f;
                    iv[u] = ok ? __ldg(inv + atf(i + u)) : 0.f;
                    rv[u] = ok ? __ldg(r + at(i + u)) : 0.f;
                    cv[u] = ok ? __ldg(cp + atf(i + u)) : 0.f;
                }
#pragma unroll
                for (int u = 0; u < CU; ++u)
                    if (i + u < i1) {
                        yv = iv[u] * rv[u] + mv[u] * yv;
                        pa_ *= mv[u];
                        z0 += q * yv;
                        z1 += q * pa_;
                        q *= -cv[u];
                        cs[(i + u) * CW + c] = yv;
                    }
            }
        carP[k][c] = pa_;
        carY[k][c] = yv;
        carQ[k][c] = q;
        carZ0[k][c] = z0;
        carZ1[k][c] = z1;
        __syncthreads();
        // forward carries into the chunks of each column: warp w < CW scans column w's chunk maps;
        // each chunk's backward map then follows from its carry
        for (int col = threadIdx.x >> 5; col < CW; col += NTC / 32) {   // warp-uniform loop
            const int qq = threadIdx.x & 31;
            Affine loc{1.f, 0.f};
            if (qq < LN) {
#pragma unroll
                for (int g = 0; g < G; ++g) loc = compose(Affine{carP[qq * G + g][col], carY[qq * G + g][col]}, loc);
            }
            Affine inc = loc;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const Affine o = Affine{__shfl_up_sync(0xffffffffu, inc.a, off), __shfl_up_sync(0xffffffffu, inc.b, off)};
                if (qq >= off) inc = compose(inc, o);
            }
            const float before = __shfl_up_sync(0xffffffffu, inc.b, 1);
            float cur = qq > 0 ? before : 0.f;
            Affine bl{1.f, 0.f};   // this lane's chunks' backward maps composed (x_below -> x_top)
            if (qq < LN) {
#pragma unroll
                for (int g = 0; g < G; ++g) {
                    const int kk = qq * G + g;
                    cin_f[kk][col] = cur;
                    const float zb = carZ0[kk][col] + carZ1[kk][col] * cur;
                    carZ0[kk][col] = zb;
                    cur = carY[kk][col] + carP[kk][col] * cur;
                }
#pragma unroll
                for (int g = G - 1; g >= 0; --g) {
                    const int kk = qq * G + g;
                    bl = compose(Affine{carQ[kk][col], carZ0[kk][col]}, bl);
                }
            }
            // backward carries: the mirrored scan from the bottom chunk up
            Affine binc = bl;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const Affine o = Affine{__shfl_down_sync(0xffffffffu, binc.a, off), __shfl_down_sync(0xffffffffu, binc.b, off)};
                if (qq + off < 32) binc = compose(binc, o);
            }
            const float after = __shfl_down_sync(0xffffffffu, binc.b, 1);
            float xb = qq < 31 ? after : 0.f;
            if (qq < LN) {
#pragma unroll
                for (int g = G - 1; g >= 0; --g) {
                    const int kk = qq * G + g;
                    cin_b[kk][col] = xb;
                    xb = carZ0[kk][col] + carQ[kk][col] * xb;
                }
            }
        }
        __syncthreads();
        if (col_ok) {
            // walk 2: the forward values with the carry in
            const float cin = cin_f[k][c];
            float pref = 1.f;
            for (int i = i0; i < i1; i += CU) {
                float mv[CU];
#pragma unroll
                for (int u = 0; u < CU; ++u) mv[u] = (i + u < i1) ? __ldg(mm + atf(i + u)) : 0.f;
#pragma unroll
                for (int u = 0; u < CU; ++u)
                    if (i + u < i1) {
                        pref *= mv[u];
                        cs[(i + u) * CW + c] += pref * cin;
                    }
            }
            // walk 3: the backward sweep from the carry below, hv = base + x
            float x = cin_b[k][c];
            const int out = pa.out, base = (pa.scheme == CEL_SCHEME_CORRECTOR) ? pa.cur : pa.in;
            const float* __restrict__ bhi = M.S[base][2] + gx;
            float* __restrict__ ohi = M.S[out][2] + gx;
            const float* __restrict__ blo = MIXED ? M.L[base][2] + gx : nullptr;
            float* __restrict__ olo = MIXED ? M.L[out][2] + gx : nullptr;
            for (int i = i1 - 1; i >= i0; i -= CU) {
                float cv[CU], bh[CU], bl[CU];
#pragma unroll
                for (int u = 0; u < CU; ++u) {
                    const bool ok = i - u >= i0;
                    cv[u] = ok ? __ldg(cp + atf(i - u)) : 0.f;
                    bh[u] = ok ? bhi[at(i - u)] : 0.f;
                    bl[u] = (MIXED && ok) ? blo[at(i - u)] : 0.f;
                }
#pragma unroll
                for (int u = 0; u < CU; ++u)
                    if (i - u >= i0) {
                        x = cs[(i - u) * CW + c] - cv[u] * x;
                        if (MIXED) {
                            float hi = bh[u], lo = bl[u];
                            two_sum_add(hi, lo, x);
                            ohi[at(i - u)] = hi;
                            olo[at(i - u)] = lo;
                        } else {
                            ohi[at(i - u)] = bh[u] + x;
                        }
                    }
            }
        }
    }
}

// Column (y) solves through tile-transposed shared memory: a CTA of 16 warps takes a band of 16
// columns and walks it in tiles of TT_ROWS rows.  The CTA loads a tile of every input it needs as
// 64-byte row pieces into shared memory laid out by column (a 4-float pad per column row), then
// warp w sweeps column w of the tile the way k_rows sweeps a row: lane j owns rows 4j .. 4j+3, read
// as one float4, runs the recurrence over them from zero, and the lanes' affine maps are joined by a
// warp-shuffle scan, with the tile's carry passed on to the next tile.  The forward values of the
// whole band stay in shared memory (16 x ny floats) for the backward walk, which loads c' and the
// base state per tile, sweeps up the same way, and writes hv = base + x back as row pieces.  Every
// input is read once; no walk re-reads a plane.
constexpr int TT_ROWS = 128, TT_CW = 16, TT_STR = TT_ROWS + 4;

template <bool MIXED>
__global__ void __launch_bounds__(512, 2) k_cols_tt(const MemberDev* __restrict__ mems, const int2* __restrict__ bands,
                                                    int nbands, PassArgs pa) {
    extern __shared__ __align__(16) float fwd[];          // [TT_CW][ny rounded to 4]: forward values by column
    __shared__ __align__(16) float stg[3][TT_CW][TT_STR];  // one tile of three inputs, by column
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int it = blockIdx.x; it < nbands; it += gridDim.x) {
        const int2 bd = bands[it];
        const MemberDev& M = mems[bd.x];
        const int n = M.c.ny, P = M.P, x0 = bd.y, nxe = M.c.nx + 2;
        const int ntile = (n + TT_ROWS - 1) / TT_ROWS;
        const int base = (pa.scheme == CEL_SCHEME_CORRECTOR) ? pa.cur : pa.in;
        float* __restrict__ yb = fwd + size_t(w) * ((n + 3) & ~3);   // 16-byte aligned columns
        // ---- forward: y_i = inv_i r_i + m_i y_{i-1} ----
        float carry = 0.f;
        for (int t = 0; t < ntile; ++t) {
            const int r0 = t * TT_ROWS;
            __syncthreads();   // the previous tile (or band) is done with the staging buffer
            for (int e = tid; e < TT_ROWS * TT_CW; e += 512) {
                const int rr = e / TT_CW, cc = e % TT_CW, i = r0 + rr, gx = x0 + cc;
                float m = 0.f, iv = 0.f, r = 0.f;
                if (i < n && gx >= 2 && gx < nxe) {
                    const size_t o = size_t(i + 2) * P + gx;
                    m = __ldg(M.FYF[2] + o); iv = __ldg(M.FYF[1] + o); r = __ldg(M.R[1] + o);
                }
                stg[0][cc][rr] = m; stg[1][cc][rr] = iv; stg[2][cc][rr] = r;
            }
            __syncthreads();
            const float4 m4 = *reinterpret_cast<const float4*>(&stg[0][w][4 * lane]);
            const float4 i4 = *reinterpret_cast<const float4*>(&stg[1][w][4 * lane]);
            const float4 r4 = *reinterpret_cast<const float4*>(&stg[2][w][4 * lane]);
            const float mv[4] = {m4.x, m4.y, m4.z, m4.w}, iv[4] = {i4.x, i4.y, i4.z, i4.w};
            const float rv[4] = {r4.x, r4.y, r4.z, r4.w};
            float yv[4], a = 1.f, b = 0.f;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                b = iv[k] * rv[k] + mv[k] * b;
                a *= mv[k];
                yv[k] = b;
            }
            Affine inc{a, b};
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const Affine o = shfl_up_affine(inc, off);
                if (lane >= off) inc = compose(inc, o);
            }
            const Affine before = shfl_up_affine(inc, 1);
            const float cin = lane > 0 ? before.b + before.a * carry : carry;
            float pref = 1.f;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                pref *= mv[k];
                yv[k] += pref * cin;
            }
            const int i0 = r0 + 4 * lane;
            if (i0 + 3 < n) {
                *reinterpret_cast<float4*>(yb + i0) = make_float4(yv[0], yv[1], yv[2], yv[3]);
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (i0 + k < n) yb[i0 + k] = yv[k];
            }
            carry = __shfl_sync(0xffffffffu, inc.b + inc.a * carry, 31);
        }
        // ---- backward: x_i = y_i - c'_i x_{i+1}; hv = base + x ----
        const float* __restrict__ bhi = M.S[base][2];
        float* __restrict__ ohi = M.S[pa.out][2];
        const float* __restrict__ blo = MIXED ? M.L[base][2] : nullptr;
        float* __restrict__ olo = MIXED ? M.L[pa.out][2] : nullptr;
        float xcarry = 0.f;
        for (int t = ntile - 1; t >= 0; --t) {
            const int r0 = t * TT_ROWS;
            __syncthreads();
            for (int e = tid; e < TT_ROWS * TT_CW; e += 512) {
                const int rr = e / TT_CW, cc = e % TT_CW, i = r0 + rr, gx = x0 + cc;
                float cp = 0.f, bh = 0.f, bl = 0.f;
                if (i < n && gx >= 2 && gx < nxe) {
                    const size_t o = size_t(i + 2) * P + gx;
                    cp = __ldg(M.FYF[0] + o); bh = bhi[o];
                    if (MIXED) bl = blo[o];
                }
                stg[0][cc][rr] = cp; stg[1][cc][rr] = bh; stg[2][cc][rr] = bl;
            }
            __syncthreads();
            const int i0 = r0 + 4 * lane;
            const float4 c4 = *reinterpret_cast<const float4*>(&stg[0][w][4 * lane]);
            float cv[4] = {c4.x, c4.y, c4.z, c4.w}, yv[4];
            if (i0 + 3 < n) {
                const float4 y4 = *reinterpret_cast<const float4*>(yb + i0);
                yv[0] = y4.x; yv[1] = y4.y; yv[2] = y4.z; yv[3] = y4.w;
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k) yv[k] = (i0 + k < n) ? yb[i0 + k] : 0.f;
            }
            float z = 0.f, qa = 1.f;
#pragma unroll
            for (int k = 3; k >= 0; --k) {
                const float cn = (i0 + k < n) ? -cv[k] : 0.f;
                z = yv[k] + cn * z;
                qa *= cn;
                yv[k] = z;
                cv[k] = cn;
            }
            Affine inc{qa, z};
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const Affine o = shfl_down_affine(inc, off);
                if (lane + off < 32) inc = compose(inc, o);
            }
            const Affine after = shfl_down_affine(inc, 1);
            const float cnext = lane < 31 ? after.b + after.a * xcarry : xcarry;
            float suf = 1.f;
#pragma unroll
            for (int k = 3; k >= 0; --k) {
                suf *= cv[k];
                yv[k] += suf * cnext;
            }
            xcarry = __shfl_sync(0xffffffffu, inc.b + inc.a * xcarry, 0);
            // lane j alone used its c' entries: overwrite them with x for the write-back
            *reinterpret_cast<float4*>(&stg[0][w][4 * lane]) = make_float4(yv[0], yv[1], yv[2], yv[3]);
            __syncthreads();
            for (int e = tid; e < TT_ROWS * TT_CW; e += 512) {
                const int rr = e / TT_CW, cc = e % TT_CW, i = r0 + rr, gx = x0 + cc;
                if (i < n && gx >= 2 && gx < nxe) {
                    const size_t o = size_t(i + 2) * P + gx;
                    const float x = stg[0][cc][rr];
                    if (MIXED) {
                        float hi = stg[1][cc][rr], lo = stg[2][cc][rr];
                        two_sum_add(hi, lo, x);
                        ohi[o] = hi;
                        olo[o] = lo;
                    } else {
                        ohi[o] = stg[1][cc][rr] + x;
                    }
                }
            }
        }
    }
}

// Column (y) solves, one thread per column: the thread runs the forward recurrence down its whole
// column and the backward one up it.  A warp covers 32 adjacent columns, so every row access is a
// coalesced 128-byte segment, and each thread issues the loads of CS rows before using them.  The
// forward values overwrite the right-hand side in place (the same thread reads them back in the
// backward sweep, mostly from L2), so the kernel needs no shared memory.
constexpr int CS = 16;

template <bool MIXED>
__global__ void __launch_bounds__(128) k_cols_serial(const MemberDev* __restrict__ mems, const int2* __restrict__ cols,
                                                     int ncols, PassArgs pa) {
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= ncols) return;
    const int2 cl = cols[it];
    if (cl.y < 0) return;   // padding that keeps each warp on 32 aligned columns
    const MemberDev& M = mems[cl.x];
    const int n = M.c.ny, P = M.P, gx = cl.y;
    float* __restrict__ rr = M.R[1] + gx;              // right-hand side, then the forward values
    const float* __restrict__ cp = M.FYF[0] + gx;
    const float* __restrict__ inv = M.FYF[1] + gx;
    const float* __restrict__ mm = M.FYF[2] + gx;
    auto at = [&](int i) { return size_t(i + 2) * P; };   // row offset of system element i
    float y = 0.f;
    for (int i = 0; i < n; i += CS) {
        float mv[CS], iv[CS], rv[CS];
#pragma unroll
        for (int u = 0; u < CS; ++u) {
            const bool ok = i + u < n;
            mv[u] = ok ? __ldg(mm + at(i + u)) : 0.f;
            iv[u] = ok ? __ldg(inv + at(i + u)) : 0.f;
            rv[u] = ok ? rr[at(i + u)] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < CS; ++u)
            if (i + u < n) {
                y = iv[u] * rv[u] + mv[u] * y;
                rr[at(i + u)] = y;
            }
    }
    const int base = (pa.scheme == CEL_SCHEME_CORRECTOR) ? pa.cur : pa.in;
    const float* __restrict__ bhi = M.S[base][2] + gx;
    float* __restrict__ ohi = M.S[pa.out][2] + gx;
    const float* __restrict__ blo = MIXED ? M.L[base][2] + gx : nullptr;
    float* __restrict__ olo = MIXED ? M.L[pa.out][2] + gx : nullptr;
    float x = 0.f;
    for (int i = n - 1; i >= 0; i -= CS) {
        float cv[CS], yv[CS], bh[CS], bl[CS];
#pragma unroll
        for (int u = 0; u < CS; ++u) {
            const bool ok = i - u >= 0;
            cv[u] = ok ? __ldg(cp + at(i - u)) : 0.f;
            yv[u] = ok ? rr[at(i - u)] : 0.f;
            bh[u] = ok ? bhi[at(i - u)] : 0.f;
            bl[u] = (MIXED && ok) ? blo[at(i - u)] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < CS; ++u)
            if (i - u >= 0) {
                x = yv[u] - cv[u] * x;
                if (MIXED) {
                    float hi = bh[u], lo = bl[u];
                    two_sum_add(hi, lo, x);
                    ohi[at(i - u)] = hi;
                    olo[at(i - u)] = lo;
                } else {
                    ohi[at(i - u)] = bh[u] + x;
                }
            }
    }
}

// Column (y) solves by thread-block clusters, every input read once and held in registers.  A
// cluster of CL CTAs takes a band of 32 adjacent columns and splits its height into CL x CKC chunks
// of at most CMC rows: warp k of the CTA of cluster rank r owns chunk r*CKC + k, lane j the column
// x0 + j, so every load is a 128-byte row piece and a warp keeps 16 rows of its chunk in flight for
// each array.  Per chunk the thread computes, from its registers:
//   forward map   y_end = A y_in + b                      (A = prod m, b = chunk sweep from 0)
//   backward map  x_top = Q x_below + Z0 + Z1 y_in        (Q = prod(-c'); Z0, Z1 from the zero-start
//                 forward values y0_i and the running products P_i, since y_i = y0_i + P_i y_in)
// so one exchange fixes every chunk's carry into the forward sweep, and a second one the carry from
// below into the backward sweep.  The chunk maps are joined inside a CTA through shared memory and
// across the cluster through distributed shared memory: each CTA pushes its aggregate into the
// CTAs that need it (lower ranks' forward aggregates to higher ranks, higher ranks' backward
// aggregates to lower ranks) between hardware cluster barriers.  Then each thread finishes its chunk
// in registers (y_i = y0_i + P_i y_in, x_i = y_i - c'_i x_{i+1}, hv = base + x) and stores it.
// Bytes per cell: m, inv, r, c', base (and its low word) in, hv (and its low word) out, each once.
// The host guarantees ceil(ny / (CL*CKC)) <= CMC for every member of the launch.
constexpr int CKC = 8, CMC = 16, CL_MAX = 16;

__device__ __forceinline__ void cluster_arrive_relaxed() { asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }
__device__ __forceinline__ unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_size() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;\n" : "=r"(r));
    return r;
}
// stores v into the shared-memory variable at `local` of the cluster's CTA `rank`
__device__ __forceinline__ void dsmem_store(float* local, unsigned rank, float v) {
    const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(local));
    unsigned ra;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(ra) : "r"(a), "r"(rank));
    asm volatile("st.shared::cluster.f32 [%0], %1;\n" ::"r"(ra), "f"(v) : "memory");
}

template <bool MIXED>
__global__ void __launch_bounds__(256, 2) k_cols_cluster(const MemberDev* __restrict__ mems,
                                                         const int2* __restrict__ bands, PassArgs pa) {
    __shared__ float sA[CKC][32], sB[CKC][32], sQ[CKC][32], sZ0[CKC][32], sZ1[CKC][32];
    __shared__ float cinK[CKC][32], xK[CKC][32];
    __shared__ float aggF[CL_MAX][2][32];   // [source rank][A, b][column]: pushed by lower ranks
    __shared__ float aggB[CL_MAX][2][32];   // [source rank][Q, Z][column]: pushed by higher ranks
    // every CTA of the cluster must have started before another one stores into its shared memory:
    // arrive now, wait just before the first remote store
    cluster_arrive_relaxed();
    const unsigned CL = cluster_size(), rank = cluster_rank();
    const int lane = threadIdx.x & 31, k = threadIdx.x >> 5;
    const int2 bd = bands[blockIdx.x / CL];
    const MemberDev& M = mems[bd.x];
    const int n = M.c.ny, P = M.P;
    const int gx = bd.y + lane;
    const bool col_ok = gx >= 2 && gx < M.c.nx + 2;
    const int nch = int(CL) * CKC;
    const int mc = (n + nch - 1) / nch;
    const int i0 = min(n, (int(rank) * CKC + k) * mc);
    const int cnt = min(n, i0 + mc) - i0;           // rows of this warp's chunk (warp-uniform, may be 0)
    const size_t o0 = size_t(i0 + 2) * P + gx;      // system element i lies in row i + 2
    const int base = (pa.scheme == CEL_SCHEME_CORRECTOR) ? pa.cur : pa.in;

    float mv[CMC], yv[CMC], cv[CMC];
    {
        float iv[CMC];
#pragma unroll
        for (int u = 0; u < CMC; ++u) {
            const bool ok = col_ok && u < cnt;
            const size_t o = o0 + size_t(u) * P;
            mv[u] = ok ? __ldg(M.FYF[2] + o) : 0.f;
            iv[u] = ok ? __ldg(M.FYF[1] + o) : 0.f;
            yv[u] = ok ? __ldg(M.R[1] + o) : 0.f;
            cv[u] = ok ? __ldg(M.FYF[0] + o) : 0.f;
        }
        // forward sweep of the chunk from zero (y0), its map, and the backward partials
        float y = 0.f, A = 1.f, Q = 1.f, Z0 = 0.f, Z1 = 0.f;
#pragma unroll
        for (int u = 0; u < CMC; ++u)
            if (u < cnt) {
                y = iv[u] * yv[u] + mv[u] * y;
                yv[u] = y;
                A *= mv[u];
                Z0 += Q * y;
                Z1 += Q * A;
                Q *= -cv[u];
            }
        sA[k][lane] = A; sB[k][lane] = y; sQ[k][lane] = Q; sZ0[k][lane] = Z0; sZ1[k][lane] = Z1;
    }
    // the base state of the chunk: loaded now so that the loads overlap the exchanges
    float bh[CMC], bl[CMC];
#pragma unroll
    for (int u = 0; u < CMC; ++u) {
        const bool ok = col_ok && u < cnt;
        const size_t o = o0 + size_t(u) * P;
        bh[u] = ok ? M.S[base][2][o] : 0.f;
        bl[u] = (MIXED && ok) ? M.L[base][2][o] : 0.f;
    }
    __syncthreads();
    cluster_wait();   // (every CTA of the cluster has started)
    if (k == 0) {
        // this CTA's forward aggregate, pushed to the higher ranks
        float A = 1.f, b = 0.f;
        for (int q = 0; q < CKC; ++q) { b = sB[q][lane] + sA[q][lane] * b; A *= sA[q][lane]; }
        for (unsigned r = rank + 1; r < CL; ++r) {
            dsmem_store(&aggF[rank][0][lane], r, A);
            dsmem_store(&aggF[rank][1][lane], r, b);
        }
    }
    cluster_arrive();
    cluster_wait();
    if (k == 0) {
        // carry into this CTA's first row from the ranks above, then into each chunk
        float cur = 0.f;
        for (unsigned r = 0; r < rank; ++r) cur = aggF[r][1][lane] + aggF[r][0][lane] * cur;
        for (int q = 0; q < CKC; ++q) {
            cinK[q][lane] = cur;
            sZ0[q][lane] += sZ1[q][lane] * cur;   // the chunk's backward map: x_top = Q x_below + Z
            cur = sB[q][lane] + sA[q][lane] * cur;
        }
        float Qa = 1.f, Za = 0.f;
        for (int q = CKC - 1; q >= 0; --q) {
            Za = sZ0[q][lane] + sQ[q][lane] * Za;
            Qa *= sQ[q][lane];
        }
        for (unsigned r = 0; r < rank; ++r) {
            dsmem_store(&aggB[rank][0][lane], r, Qa);
            dsmem_store(&aggB[rank][1][lane], r, Za);
        }
    }
    cluster_arrive();
    cluster_wait();
    if (k == 0) {
        // carry from below into this CTA's last row from the ranks below it, then into each chunk
        float cur = 0.f;
        for (unsigned r = CL - 1; r > rank; --r) cur = aggB[r][1][lane] + aggB[r][0][lane] * cur;
        for (int q = CKC - 1; q >= 0; --q) {
            xK[q][lane] = cur;
            cur = sZ0[q][lane] + sQ[q][lane] * cur;
        }
    }
    __syncthreads();
    if (!col_ok || cnt <= 0) return;
    const float cin = cinK[k][lane];
    float Pr = 1.f;
#pragma unroll
    for (int u = 0; u < CMC; ++u)
        if (u < cnt) {
            Pr *= mv[u];
            yv[u] += Pr * cin;
        }
    float x = xK[k][lane];
    float* __restrict__ ohi = M.S[pa.out][2];
    float* __restrict__ olo = MIXED ? M.L[pa.out][2] : nullptr;
#pragma unroll
    for (int u = CMC - 1; u >= 0; --u)
        if (u < cnt) {
            x = yv[u] - cv[u] * x;
            const size_t o = o0 + size_t(u) * P;
            if (MIXED) {
                float hi = bh[u], lo = bl[u];
                two_sum_add(hi, lo, x);
                ohi[o] = hi;
                olo[o] = lo;
            } else {
                ohi[o] = bh[u] + x;
            }
        }
}

// ---------------------------------------------------------------------------------------------
// Boundary strips (compute.hlsl:985-1309), one side per launch over every member.
// work item: {member, first strip cell}; 256 strip cells per item, BND_CELLS for a sponge strip
// (its threads take BND_CPT cells each and issue all their loads before the first store), and
// BND_IRR_CELLS for an irregular wave-maker strip (one cell per warp, its components spread over
// the lanes).  The narrow strips of the other kinds keep one cell per thread, so they still spread
// over the SMs.
// phase 0: compute and write in place; 1: compute into the member's scratch; 2: copy back.
// The compensated form evaluates the sine, irregular and time-series values in FP64 and applies the
// sponge's factor to the full compensated value in FP64; it stores the results as a float pair
// (value + low word), so the strips keep the state's precision.
// ---------------------------------------------------------------------------------------------
constexpr double CEL_PI_D = 3.14159265358979323846;
constexpr double CEL_MIN_DEPTH_D = 0.0001;   // compute.hlsl:1062

// v as a float pair: hi = v rounded, lo = the rest rounded
__device__ __forceinline__ void split_hl(double v, float& hi, float& lo) {
    hi = float(v);
    lo = float(v - double(hi));
}

// sineWave with Eckart's wavenumber (compute.hlsl:1080-1101) in FP64
__device__ __forceinline__ void sine_wave_d(double x, double y, double t, double d, double amp, double period, double th,
                                            double phase, double g, double& e, double& hu, double& hv) {
    const double omega = 2.0 * CEL_PI_D / period;
    const double k = omega * omega / (g * sqrt(tanh(omega * omega * d / g)));
    const double c = omega / k;
    double sth, cth;
    sincos(th, &sth, &cth);
    e = amp * sin(omega * t - cth * x * k - sth * y * k + phase);
    hu = c * cth * e;
    hv = c * sth * e;
}

// The same pairwise tree restricted to the aligned power-of-two range of components [m0, m1),
// continuing from `carry`, the sum of the aligned range of carry_size components just before m0
// (carry_size 0: none).  Padding components (m >= nreal) are blocks of sea level in eta and 0 in
// hu, hv; every block sum is an exact power-of-two multiple of the sea level, so any grouping of
// them rounds identically.
__device__ float3 irregular_range(const BoundaryDesc& b, const float4* waves, float xx, float yy, float t, float dh,
                                  float g, int nreal, int m0, int m1, float3 carry, int carry_size) {
    float3 stk[17];
    int sz[17];
    int top = 0;
    if (carry_size > 0) { stk[0] = carry; sz[0] = carry_size; top = 1; }
    int m = m0;
    while (m < m1) {
        float3 v;
        int s;
        if (m < nreal) {
            float e, hu, hv;
            const float4 wv = waves[b.wave_offset + m];
            sine_wave(xx, yy, t, dh, wv.x, wv.y, wv.z, wv.w, g, e, hu, hv);
            v = make_float3(e + b.sea_level, hu, hv);
            s = 1;
        } else {
            s = (m == 0) ? m1 : (m & -m);
            while (m + s > m1) s >>= 1;
            v = make_float3(float(s) * b.sea_level, 0.f, 0.f);
        }
        m += s;
        stk[top] = v;
        sz[top] = s;
        ++top;
        while (top >= 2 && sz[top - 1] == sz[top - 2]) {
            const float3 r = stk[top - 1], l = stk[top - 2];
            stk[top - 2] = make_float3(l.x + r.x, l.y + r.y, l.z + r.z);
            sz[top - 2] *= 2;
            --top;
        }
    }
    return stk[0];
}

// The irregular wave-maker value (compute.hlsl:1196-1212: the components' sineWave values summed
// over a balanced pairwise tree of nleaf leaves, the first n_waves real, the rest sea level) with
// the work spread over a warp (all 32 lanes call it; lane 0's result is the sum).  The real
// components lie in [0, R), R the smallest power of two >= their count: the lanes take equal
// aligned parts of it, a pairwise shuffle tree joins the parts in the same tree shape, and the
// padding up to nleaf follows on top, so the result is bit-identical to the sequential tree.
__device__ float3 irregular_warp(const BoundaryDesc& b, const float4* waves, float xx, float yy, float t, float dh,
                                 float g, int lane) {
    const float3 zero = make_float3(0.f, 0.f, 0.f);
    const int nreal = (dh > CEL_MIN_DEPTH) ? min(b.n_waves, b.nleaf) : 0;
    if (nreal == 0) return irregular_range(b, waves, xx, yy, t, dh, g, 0, 0, b.nleaf, zero, 0);
    int R = 1;
    while (R < nreal) R <<= 1;
    const int A = min(32, R), per = R / A;
    float3 v = zero;
    if (lane < A) v = irregular_range(b, waves, xx, yy, t, dh, g, nreal, lane * per, (lane + 1) * per, zero, 0);
    for (int off = 1; off < A; off <<= 1) {   // A is the same on every lane
        const float ox = __shfl_down_sync(0xffffffffu, v.x, off);
        const float oy = __shfl_down_sync(0xffffffffu, v.y, off);
        const float oz = __shfl_down_sync(0xffffffffu, v.z, off);
        if ((lane & (2 * off - 1)) == 0) v = make_float3(v.x + ox, v.y + oy, v.z + oz);
    }
    if (R < b.nleaf) v = irregular_range(b, waves, xx, yy, t, dh, g, nreal, R, b.nleaf, v, R);
    return v;
}

// The irregular wave-maker value in FP64 (compensated form): the nleaf leaves sum to
// sum_i (e_i + sea level) + (nleaf - n) sea level = sum_i e_i + nleaf sea level.  Lanes take the
// components lane, lane + 32, ...; a shuffle tree joins them; every lane gets the sums.
__device__ void irregular_warp_d(const BoundaryDesc& b, const double* waves, double xx, double yy, double t,
                                 double dh, double g, int lane, double out[3]) {
    const int nreal = (dh > CEL_MIN_DEPTH_D) ? min(b.n_waves, b.nleaf) : 0;
    double e = 0.0, u = 0.0, v = 0.0;
    for (int m = lane; m < nreal; m += 32) {
        const double* wv = waves + 4 * size_t(b.wave_offset + m);
        double ei, ui, vi;
        sine_wave_d(xx, yy, t, dh, wv[0], wv[1], wv[2], wv[3], g, ei, ui, vi);
        e += ei; u += ui; v += vi;
    }
    for (int off = 16; off; off >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, off);
        u += __shfl_xor_sync(0xffffffffu, u, off);
        v += __shfl_xor_sync(0xffffffffu, v, off);
    }
    out[0] = e + double(b.nleaf) * b.sea_level64;
    out[1] = u;
    out[2] = v;
}

// timeSeriesHelper (engine.cpp:1882-1904) for a table sorted by time: the first row at or after t
// (from row 1 on), linear interpolation from the row before; zero past the end.
template <typename T>
__device__ void uts_lookup(const T* tab, int n, T t, T out[3]) {
    out[0] = out[1] = out[2] = T(0);
    int lo = 1, hi = n;  // first index in [1, n) with tab.t >= t, or n
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (tab[4 * mid] < t) lo = mid + 1; else hi = mid;
    }
    if (lo >= n) return;
    const T t0 = tab[4 * (lo - 1)], t1 = tab[4 * lo];
    const T m = (t - t0) / (t1 - t0);
    for (int q = 0; q < 3; ++q) {
        const T v0 = tab[4 * (lo - 1) + q + 1], v1 = tab[4 * lo + q + 1];
        out[q] = v0 + (v1 - v0) * m;
    }
}

// Sponge length and distance of strip texel (x, y) on `side` (compute.hlsl:1011-1060)
template <typename T>
__device__ __forceinline__ void sponge_geometry(int side, int x, int y, int NX, int NY, int width, T dx, T dy, T& L,
                                                T& dist) {
    if (side == 3) { L = T(width) * dx; dist = T(x) * dx; }
    else if (side == 1) { L = T(width) * dx; dist = T(NX - x) * dx; }
    else if (side == 2) { L = T(width) * dy; dist = T(y) * dy; }
    else { L = T(width) * dy; dist = T(NY - y) * dy; }
}

// The sponge's damping factor at one texel (compute.hlsl:1011-1060): SpongeFunction(L, d) /
// SpongeFunction(L, d + sqrt(g h) dt) with SpongeFunction(L, x) = 0.5 + 0.5 cos(pi max(L - x, 0) / L).
// The fused forms evaluate the same function as sin^2(pi min(x, L) / (2 L)), which it equals: near
// x = 0 the cosine form cancels to zero in single precision, and at the strip's outermost texel over
// dry ground (depth clamped to 1e-4 m, so the shifted distance is under a millimetre) both sponge
// values round to 0 and their ratio is 0/0.  The compensated form applies the factor to the full
// (hi, lo) value in FP64.
__device__ __forceinline__ float sponge_sin2(float L, float x) {
    const float s = sinf((0.5f * CEL_PI_F) * (fminf(x, L) / L));
    return s * s;
}
__device__ __forceinline__ float sponge_gamma(const MemberDev& M, const BoundaryDesc& b, int side, int x, int y,
                                              float ba) {
    float L, dist;
    sponge_geometry(side, x, y, M.c.NX, M.c.NY, b.width, M.c.dx, M.c.dy, L, dist);
    const float dh = fmaxf(CEL_MIN_DEPTH, b.sea_level - ba);
    return sponge_sin2(L, dist) / sponge_sin2(L, dist + sqrtf(M.c.g * dh) * (*M.dtp));
}

// The sponged texel (hi, lo) pairs in place: eta scaled about the sea level, hu and hv scaled
__device__ __forceinline__ void sponge_apply_d(double gam, double sl, float& w, float& lw, float& u, float& lu, float& v,
                                               float& lv) {
    split_hl(gam * ((double(w) + double(lw)) - sl) + sl, w, lw);
    split_hl(gam * (double(u) + double(lu)), u, lu);
    split_hl(gam * (double(v) + double(lv)), v, lv);
}

constexpr int BND_CPT = 4;
constexpr int BND_CELLS = 256 * BND_CPT;
constexpr int BND_IRR_CELLS = 256 / 32;   // irregular wave-maker strips: one cell per warp

__host__ __device__ __forceinline__ int boundary_item_cells(int type) {
    return type == CEL_BC_SPONGE ? BND_CELLS : type == CEL_BC_IRREGULAR ? BND_IRR_CELLS : 256;
}

template <bool MIXED>
__global__ void __launch_bounds__(256, 2) k_boundary(const MemberDev* __restrict__ mems, const int2* __restrict__ items,
                                                  int nitems, int side, int phase, int out) {
    constexpr int SS = MIXED ? 6 : 3;   // strip floats per cell: w, hu, hv (+ their low words)
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 wi = items[it];
        const MemberDev& M = mems[wi.x];
        const SimConsts c = M.c;
        const BoundaryDesc& b = M.bd[side];
        const int NX = c.NX, NY = c.NY, P = M.P;
        int x0, y0, sw, sh;
        if (side == 0) { x0 = 0; sw = NX; y0 = NY - b.width; sh = b.width; }
        else if (side == 1) { x0 = NX - b.width; sw = b.width; y0 = 0; sh = NY; }
        else if (side == 2) { x0 = 0; sw = NX; y0 = 0; sh = b.width; }
        else { x0 = 0; sw = b.width; y0 = 0; sh = NY; }
        if (x0 < 0) { sw += x0; x0 = 0; }
        if (y0 < 0) { sh += y0; y0 = 0; }
        sw = min(sw, NX - x0); sh = min(sh, NY - y0);
        float* W = M.S[out][0];
        float* HU = M.S[out][1];
        float* HV = M.S[out][2];
        float* LW = MIXED ? M.L[out][0] : nullptr;
        float* LU = MIXED ? M.L[out][1] : nullptr;
        float* LV = MIXED ? M.L[out][2] : nullptr;
        const int cend = min(sw * sh, wi.y + boundary_item_cells(b.type));   // this item's cells end here
        if (b.type == CEL_BC_SPONGE && phase == 0) {
            // Pointwise: the loads of all the thread's cells are issued before the first store.
            const float sl = b.sea_level;
            size_t gi[BND_CPT];
            int cx[BND_CPT], cy[BND_CPT];
            float vw[BND_CPT], vu[BND_CPT], vv[BND_CPT], ba[BND_CPT];
            float l0[BND_CPT], l1[BND_CPT], l2[BND_CPT];
            bool ok[BND_CPT];
#pragma unroll
            for (int k = 0; k < BND_CPT; ++k) {
                const int cell = wi.y + k * 256 + threadIdx.x;
                ok[k] = cell < cend;
                cx[k] = x0 + cell % sw; cy[k] = y0 + cell / sw;
                gi[k] = size_t(cy[k]) * P + cx[k];
                vw[k] = vu[k] = vv[k] = ba[k] = l0[k] = l1[k] = l2[k] = 0.f;
                if (ok[k]) {
                    vw[k] = W[gi[k]]; vu[k] = HU[gi[k]]; vv[k] = HV[gi[k]]; ba[k] = M.BA[gi[k]];
                    if (MIXED) { l0[k] = LW[gi[k]]; l1[k] = LU[gi[k]]; l2[k] = LV[gi[k]]; }
                }
            }
#pragma unroll
            for (int k = 0; k < BND_CPT; ++k) {
                if (!ok[k]) continue;
                const float gam = sponge_gamma(M, b, side, cx[k], cy[k], ba[k]);
                if (MIXED) {
                    sponge_apply_d(gam, b.sea_level64, vw[k], l0[k], vu[k], l1[k], vv[k], l2[k]);
                    W[gi[k]] = vw[k]; HU[gi[k]] = vu[k]; HV[gi[k]] = vv[k];
                    LW[gi[k]] = l0[k]; LU[gi[k]] = l1[k]; LV[gi[k]] = l2[k];
                } else {
                    W[gi[k]] = gam * (vw[k] - sl) + sl;
                    HU[gi[k]] = gam * vu[k];
                    HV[gi[k]] = gam * vv[k];
                }
            }
            continue;
        }
        if (b.type == CEL_BC_IRREGULAR && phase != 2) {
            // one cell per warp, its components spread over the lanes (BND_IRR_CELLS per item)
            const int lane = threadIdx.x & 31;
            const int cell = wi.y + (threadIdx.x >> 5);
            if (cell >= cend) continue;   // warp-uniform
            const int x = x0 + cell % sw, y = y0 + cell / sw;
            const size_t gi = size_t(y) * P + x;
            const bool colwise = (side == 1 || side == 3);
            const int along = colwise ? y : x;
            const int lim = colwise ? c.ny : c.nx;
            float o[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};   // w, hu, hv, then their low words
            if (along >= 2 && along < lim + 2) {
                if (MIXED) {
                    const double dh = fmax(0.0, b.sea_level64 - double(M.BA[gi]));
                    const double xx = (side == 1) ? double(x - NX) * M.dx64 : double(x) * M.dx64;
                    const double yy = (side == 0) ? double(y - NY) * M.dy64 : double(y) * M.dy64;
                    double r[3];
                    irregular_warp_d(b, M.waves64, xx, yy, *M.time64, dh, M.g64, lane, r);
                    for (int q = 0; q < 3; ++q) split_hl(r[q], o[q], o[3 + q]);
                } else {
                    const float dh = fmaxf(0.f, b.sea_level - M.BA[gi]);
                    const float xx = (side == 1) ? float(x - NX) * c.dx : float(x) * c.dx;
                    const float yy = (side == 0) ? float(y - NY) * c.dy : float(y) * c.dy;
                    const float3 r = irregular_warp(b, M.waves, xx, yy, *M.time32, dh, c.g, lane);
                    o[0] = r.x; o[1] = r.y; o[2] = r.z;
                }
            }
            if (lane == 0) {
                if (phase == 1) {
                    for (int q = 0; q < SS; ++q) M.strip[SS * cell + q] = o[q];
                } else {
                    W[gi] = o[0]; HU[gi] = o[1]; HV[gi] = o[2];
                    if (MIXED) { LW[gi] = o[3]; LU[gi] = o[4]; LV[gi] = o[5]; }
                }
            }
            continue;
        }
        const int cpt = (b.type == CEL_BC_SPONGE) ? BND_CPT : 1;
        for (int k = 0; k < cpt; ++k) {
            const int cell = wi.y + k * 256 + threadIdx.x;
            if (cell >= cend) break;   // cells ascend with k
            const int x = x0 + cell % sw, y = y0 + cell / sw;
            const size_t gi = size_t(y) * P + x;
            if (phase == 2) {
                W[gi] = M.strip[SS * cell]; HU[gi] = M.strip[SS * cell + 1]; HV[gi] = M.strip[SS * cell + 2];
                if (MIXED) { LW[gi] = M.strip[SS * cell + 3]; LU[gi] = M.strip[SS * cell + 4]; LV[gi] = M.strip[SS * cell + 5]; }
                continue;
            }
            float ow = 0.f, ou = 0.f, ov = 0.f;
            float lw = 0.f, lu = 0.f, lv = 0.f;
            const float sl = b.sea_level;
            if (b.type == CEL_BC_SOLID) {
                int qx, qy;
                solid_source(side, x, y, c.nx, c.ny, qx, qy);
                float sw_ = 0.f, su = 0.f, sv = 0.f, lw_ = 0.f, lu_ = 0.f, lv_ = 0.f;
                if (qx >= 0 && qy >= 0 && qx < NX && qy < NY) {
                    const size_t qi = size_t(qy) * P + qx;
                    sw_ = W[qi]; su = HU[qi]; sv = HV[qi];
                    if (MIXED) { lw_ = LW[qi]; lu_ = LU[qi]; lv_ = LV[qi]; }
                }
                ow = sw_; lw = lw_;
                ou = (side == 1 || side == 3) ? -su : su; lu = (side == 1 || side == 3) ? -lu_ : lu_;
                ov = (side == 0 || side == 2) ? -sv : sv; lv = (side == 0 || side == 2) ? -lv_ : lv_;
            } else if (b.type == CEL_BC_SPONGE) {
                ow = W[gi]; ou = HU[gi]; ov = HV[gi];
                const float gam = sponge_gamma(M, b, side, x, y, M.BA[gi]);
                if (MIXED) {
                    lw = LW[gi]; lu = LU[gi]; lv = LV[gi];
                    sponge_apply_d(gam, b.sea_level64, ow, lw, ou, lu, ov, lv);
                } else {
                    ow = gam * (ow - sl) + sl;
                    ou = gam * ou;
                    ov = gam * ov;
                }
            } else if (b.type == CEL_BC_SINEWAVE) {
                if (MIXED) {
                    const double dh = fmax(0.0, b.sea_level64 - double(M.BA[gi]));
                    const double xx = (side == 1) ? double(x - NX) * M.dx64 : double(x) * M.dx64;
                    const double yy = (side == 0) ? double(y - NY) * M.dy64 : double(y) * M.dy64;
                    double e = 0.0, hu = 0.0, hv = 0.0;
                    if (dh > CEL_MIN_DEPTH_D)
                        sine_wave_d(xx, yy, *M.time64, dh, b.amplitude64, b.period64, b.theta64, 0.0, M.g64, e, hu, hv);
                    split_hl(e + b.sea_level64, ow, lw);
                    split_hl(hu, ou, lu);
                    split_hl(hv, ov, lv);
                } else {
                    const float dh = fmaxf(0.f, sl - M.BA[gi]);
                    const float xx = (side == 1) ? float(x - NX) * c.dx : float(x) * c.dx;
                    const float yy = (side == 0) ? float(y - NY) * c.dy : float(y) * c.dy;
                    float e = 0.f, hu = 0.f, hv = 0.f;
                    if (dh > CEL_MIN_DEPTH) sine_wave(xx, yy, *M.time32, dh, b.amplitude, b.period, b.theta, 0.f, c.g, e, hu, hv);
                    ow = e + sl; ou = hu; ov = hv;
                }
            } else if (b.type == CEL_BC_UTS) {
                if (MIXED) {
                    double v[3];
                    uts_lookup<double>(M.uts64[side], M.nuts[side], *M.time64, v);
                    split_hl(v[0] + b.sea_level64, ow, lw);
                    split_hl(v[1], ou, lu);
                    split_hl(v[2], ov, lv);
                } else {
                    float v[3];
                    uts_lookup<float>(M.uts[side], M.nuts[side], *M.time32, v);
                    ow = v[0] + sl; ou = v[1]; ov = v[2];
                }
            }
            if (phase == 1) {
                M.strip[SS * cell] = ow; M.strip[SS * cell + 1] = ou; M.strip[SS * cell + 2] = ov;
                if (MIXED) { M.strip[SS * cell + 3] = lw; M.strip[SS * cell + 4] = lu; M.strip[SS * cell + 5] = lv; }
            } else {
                W[gi] = ow; HU[gi] = ou; HV[gi] = ov;
                if (MIXED) { LW[gi] = lw; LU[gi] = lu; LV[gi] = lv; }
            }
        }
    }
}

// AddSolitaryWave (compute.hlsl:949-976) on member i's state buffer `buf`: every texel of
// [1, nx+3) x [1, ny+3) adds the sech^2 wave of its own water depth (the draw region of
// engine.cpp:2154-2219).  Each texel reads only itself, so the update runs in place; the
// transcendentals run in double.
template <bool MIXED>
__global__ void k_add_solitary(const MemberDev* __restrict__ mems, int i, int buf, float H, float th, float xc, float yc) {
    const MemberDev& M = mems[i];
    const SimConsts& c = M.c;
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (x >= c.nx + 3 || y >= c.ny + 3) return;
    const size_t gi = size_t(y) * M.P + x;
    float* W = M.S[buf][0];
    float* HU = M.S[buf][1];
    float* HV = M.S[buf][2];
    const double w = double(W[gi]) + (MIXED ? double(M.L[buf][0][gi]) : 0.0);
    const double depth = fmax(w - double(M.BA[gi]), 0.0);
    const double K = sqrt(0.75 * fabs(double(H)) / (depth * depth * depth));
    const double C = sqrt(double(c.g) * (double(H) + depth));
    const double ch = cosh(K * ((double(x) * c.dx - xc) * cos(double(th)) + (double(y) * c.dy - yc) * sin(double(th))));
    const double e = double(H) / (ch * ch);
    const float de = float(e), du = float(C * cos(double(th)) * e), dv = float(C * sin(double(th)) * e);
    if (MIXED) {
        float hi = W[gi], lo = M.L[buf][0][gi];
        two_sum_add(hi, lo, de); W[gi] = hi; M.L[buf][0][gi] = lo;
        hi = HU[gi]; lo = M.L[buf][1][gi];
        two_sum_add(hi, lo, du); HU[gi] = hi; M.L[buf][1][gi] = lo;
        hi = HV[gi]; lo = M.L[buf][2][gi];
        two_sum_add(hi, lo, dv); HV[gi] = hi; M.L[buf][2][gi] = lo;
    } else {
        W[gi] += de; HU[gi] += du; HV[gi] += dv;
    }
}

// Per-member time-step controller of an adaptive batch: resetTimestep's dt logic
// (engine.cpp:1698-1726) kept on the device, so a physical step needs no host readback and can
// be replayed from a CUDA graph.  Single precision with IEEE-rounded operations, as the reference's
// float arithmetic.
struct DtCtl {
    float dt, dt_old, dt_old_old;   // this pass, and the two previous steps (engine.hpp:300-301)
    float target_cfl;               // "target cfl": timestep x the first positive CFL rate
    int target_set, initialized;
    float base, min_ratio, alpha;   // timestep, min_timestep_ratio, exponentialMovingAverageAlpha
    float dt_first;                 // dt of the first pass of the most recent step
    float ab[7];                    // variable-step AB3 coefficients of the latest adaptive predictor
};

// std::max(a, b): a unless a < b (NaN in a stays)
__device__ __forceinline__ float std_max(float a, float b) { return (a < b) ? b : a; }

// AdamsBashforthCoef and the three second-order derivative stencils (compute.hlsl:560-605),
// folded into one coefficient per history level: the predictor computes
//   w  += k (A0 f + A1 f_old + A2 f_oldold)
//   hu  = (A hu_W + B hu + C hu_E) + k (A0 f + ...) + (K0 F* + K1 F*_old + K2 F*_oldold)
// where K_j = k * sum_m coef_m * D_m,j and D_m,j is the weight of level j in derivative m
// (backward at t_n, central at t_n-1, forward at t_n-2).  With equal steps this gives
// k = dt/6, A = (11.5, -8, 2.5) and K = (2, -3, 1): the fixed-step AB3 of the predictor.
__device__ void ab3_coefficients(float dt, float d1, float d2, float* ab) {
    const float r = __fdiv_rn(dt, d1);
    const float s12 = __fadd_rn(d1, d2);
    const float c0 = __fadd_rn(__fmul_rn(r, __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(2.f, dt), __fmul_rn(6.f, d1)), __fmul_rn(3.f, d2)), s12)), 6.f);
    const float c1 = -__fmul_rn(r, __fdiv_rn(__fadd_rn(__fadd_rn(__fmul_rn(2.f, dt), __fmul_rn(3.f, d1)), __fmul_rn(3.f, d2)), d2));
    const float c2 = __fmul_rn(__fdiv_rn(dt, d2), __fdiv_rn(__fadd_rn(__fmul_rn(2.f, dt), __fmul_rn(3.f, d1)), s12));
    const float p1 = __fmul_rn(d1, s12), p2 = __fmul_rn(d2, s12), p12 = __fmul_rn(d1, d2);
    // rows: backward, central, forward; columns: levels n, n-1, n-2
    const float D[3][3] = {
        {__fdiv_rn(__fadd_rn(__fmul_rn(2.f, d1), d2), p1), -__fdiv_rn(s12, p12), __fdiv_rn(d1, p2)},
        {__fdiv_rn(d2, p1), __fdiv_rn(__fsub_rn(d1, d2), p12), -__fdiv_rn(d1, p2)},
        {-__fdiv_rn(d2, p1), __fdiv_rn(s12, p12), -__fdiv_rn(__fadd_rn(d1, __fmul_rn(2.f, d2)), p2)}};
    const float k = __fdiv_rn(dt, 6.f);
    ab[0] = k; ab[1] = c0; ab[2] = c1; ab[3] = c2;
    for (int j = 0; j < 3; ++j)
        ab[4 + j] = __fmul_rn(k, __fadd_rn(__fadd_rn(__fmul_rn(c0, D[0][j]), __fmul_rn(c1, D[1][j])), __fmul_rn(c2, D[2][j])));
}

// Max CFL rate max((|u| + c)/dx, (|v| + c)/dy) of each member's current state over the cells of
// its 4x4 blocks (the GetStats region, compute.hlsl:1319-1378), as non-negative float bits.
// Each CTA takes a contiguous range of tiles (consecutive tiles mostly belong to one member), keeps
// the maximum in registers and publishes it with one atomic per warp when the member changes or
// the range ends: a few thousand atomics instead of one per warp per tile on 64 words.
__global__ void __launch_bounds__(256) k_cfl(const MemberDev* __restrict__ mems, const int4* __restrict__ tiles,
                                             int ntiles, int buf, unsigned int* __restrict__ out) {
    const int per = (ntiles + gridDim.x - 1) / gridDim.x;
    const int t_begin = blockIdx.x * per, t_end = min(ntiles, t_begin + per);
    int cur = -1;
    float m = 0.f;
    auto flush = [&]() {   // warp-uniform: every lane has the same `cur`
        float v = m;
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0 && cur >= 0 && v > 0.f) atomicMax(out + cur, __float_as_uint(v));
        m = 0.f;
    };
    for (int t = t_begin; t < t_end; ++t) {
        const int4 tl = tiles[t];
        if (tl.x != cur) { flush(); cur = tl.x; }
        const MemberDev& M = mems[tl.x];
        const SimConsts& c = M.c;
#pragma unroll
        for (int r = 0; r < (TX * TY) / 256; ++r) {
            const int k = r * 256 + threadIdx.x;
            const int gx = tl.y + k % TX, gy = tl.z + k / TX;
            if (gx < 2 + 4 * (c.nx / 4) && gy < 2 + 4 * (c.ny / 4)) {
                const size_t gi = size_t(gy) * M.P + gx;
                const float h = fmaxf(0.f, M.S[buf][0][gi] - M.BA[gi]);
                const float q = div_by_h_fast(h, c.epsilon);
                const float cc = sqrtf(c.g * h);
                m = fmaxf(m, fmaxf((fabsf(q * M.S[buf][1][gi]) + cc) * c.one_over_dx,
                                   (fabsf(q * M.S[buf][2][gi]) + cc) * c.one_over_dy));
            }
        }
    }
    flush();
}

// resetTimestep's dt choice for every member before a pass (engine.cpp:1698-1726): the target
// CFL is set from the first positive CFL rate seen; adaptive predictors take
// max(target / cfl, timestep * min ratio), smoothed by the moving average when it grows; every
// other pass runs with the uniform time step.  cfl may be null (no reduction before this pass).
__global__ void k_choose_dt(DtCtl* __restrict__ ctl, float* __restrict__ dt_table, const unsigned int* __restrict__ cfl,
                            int n, int scheme, int first_of_step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    DtCtl& C = ctl[i];
    float rate = cfl ? __uint_as_float(cfl[i]) : 0.f;
    if (rate > 0.f && !C.target_set) { C.target_cfl = __fmul_rn(C.base, rate); C.target_set = 1; }
    if (!C.initialized) {
        C.dt = C.base;
        C.dt_old_old = C.dt;
        C.dt_old = C.dt;
        C.initialized = 1;
    }
    if (scheme == CEL_SCHEME_PREDICTOR_ADAPTIVE) {
        const float tgt = std_max(__fdiv_rn(C.target_cfl, rate), __fmul_rn(C.base, C.min_ratio));
        C.dt = tgt > C.dt_old ? __fadd_rn(__fmul_rn(C.alpha, tgt), __fmul_rn(__fsub_rn(1.f, C.alpha), C.dt_old)) : tgt;
        ab3_coefficients(C.dt, C.dt_old, C.dt_old_old, C.ab);
    } else {
        C.dt = C.base;
    }
    if (first_of_step) C.dt_first = C.dt;
    dt_table[i] = C.dt;
}

// End of a physical step: advance the clocks by the dt of the step's last pass and, in adaptive
// batches, shift the controller's dt queue (engine.cpp:1507-1518).
// The band-major copy of a member's y factors for band width cw (k_cols reads it).
__global__ void k_band_major(const MemberDev* __restrict__ mems, int mi, int cw) {
    const MemberDev& M = mems[mi];
    const int n = M.c.ny, NX = M.c.NX, nb = (M.c.nx + 2 + cw - 1) / cw;
    const size_t total = size_t(nb) * n * cw;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
        const int c = int(e % cw), i = int((e / cw) % n), b = int(e / (size_t(cw) * n));
        const int x = b * cw + c;
        const size_t o = size_t(i + 2) * M.P + x;
        for (int q = 0; q < 3; ++q) M.FYB[q][e] = x < NX ? M.FYF[q][o] : 0.f;
    }
}

// rcp_newton over a caller's inputs (the device self-test behind cel_selftest_reciprocal)
__global__ void k_rcp_selftest(const float* __restrict__ x, float* __restrict__ out, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = rcp_newton(x[i]);
}

__global__ void k_advance_time(const MemberDev* __restrict__ mems, DtCtl* __restrict__ ctl, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const MemberDev& M = mems[i];
    *M.time64 += double(*M.dtp);
    *M.time32 += *M.dtp;
    if (ctl) {
        ctl[i].dt_old_old = ctl[i].dt_old;
        ctl[i].dt_old = ctl[i].dt;
    }
}

// Final Pass1 aux update of the current state (txAuxiliary2 -> reported txAuxiliary1 values are
// what the device keeps; this kernel is not needed for them).
}  // namespace

// ---------------------------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------------------------
struct Member {
    cel_params p{};
    HostSetup hs;
    int P = 0;
    size_t plane = 0;
    std::vector<float> uts_host[4];
};

struct Idx {
    int sin = 0, cur = 0;
    int og = 0, oog = 1, scr = 2, spare = 3, pred = 3;
    bool operator==(const Idx& o) const {
        return sin == o.sin && cur == o.cur && og == o.og && oog == o.oog && scr == o.scr && spare == o.spare;
    }
};

}  // namespace cel

struct cel_lane {
    int form = CEL_FORM_FUSED;
    bool mixed = false;
    std::vector<cel::Member> mem;
    std::vector<cel::MemberDev> hdev;
    cel::MemberDev* ddev = nullptr;
    std::vector<void*> allocs;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaStream_t side = nullptr;       // second stream: the column solve runs beside the row solve
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cel::KernelTimer tm;
    cel::Scheme sch;      // shared pass sequence (all members use the same correction count)
    cel::Idx ix;
    int4* tiles = nullptr; int ntiles = 0;      // 32x16 tiles (statistics on demand)
    int4* mtiles = nullptr; int nmtiles = 0;    // marching strips of the fused stencil
    int2* rows = nullptr; int nrows = 0;
    int2* bands = nullptr; int nbands = 0;
    int2* bitems[4] = {nullptr, nullptr, nullptr, nullptr};
    int nbitems[4] = {0, 0, 0, 0};
    bool two_phase[4] = {false, false, false, false};
    double* stats_all = nullptr;       // members * STATS_N, gathered by the first pass of each step
    double* stats_now_all = nullptr;   // members * STATS_N, on-demand statistics of the current state
    double* late_flag = nullptr;       // a bounded TMA wait gave up (sticky)
    // readback block: late_flag | clock64 (n) | stats_all (n x STATS_N) | stats_now_all, so that
    // the statistics of a step, the clocks and the flag come back in one copy
    double* clock64 = nullptr;         // per-member FP64 clocks
    float* clock32 = nullptr;          // per-member FP32 clocks
    double* rb_host = nullptr;         // pinned host copy of the readback block
    bool step_stats_valid = false;     // stats_all describes the start of the most recent step
    std::vector<float> step_dt;        // the time step each member took in its most recent step
    bool any_friction = false;
    float* dt_table = nullptr;         // per-member time step on the device
    float* dt_host = nullptr;          // pinned mirror of dt_table
    cudaEvent_t dt_copied = nullptr;   // recorded after each upload of dt_host
    bool adaptive = false;              // adaptive time steps: dt chosen per member on the device
    cel::DtCtl* ctl = nullptr;          // per-member dt controllers (adaptive batches)
    std::vector<cel::DtCtl> ctl_host;   // their read-back copy (statistics)
    unsigned int* cfl_now = nullptr;    // per-member max CFL rate of the current state (float bits)
    bool dt_started = false;            // the controllers have made their first choice
    size_t smem_rows = 0, smem_cols = 0;
    int rowbuf = 0, rows_threads = 256;   // row solver: floats of forward values per warp, threads per CTA
    int grid_stencil = 0, grid_rows = 0, grid_cols = 0;
    int sms = 148;
    bool use_graph = false;
    std::vector<cudaGraphExec_t> graphs;
    std::vector<cel::Idx> graph_idx;   // index state at the start of each captured step
    int graph_pos = 0;
    long long cells = 0;
    int cw = 16;                        // column solver band width (columns per CTA)
    int cnt = 512;                      // column solver threads per CTA (chunks per column = cnt / cw)
    int col_cl = 0;                     // cluster column solver: CTAs per cluster (0: not in use)
    bool col_tt = false;                // tile-transposed column solver (band width 16, "1 chunk")
    int mh = cel::MH_DEFAULT;           // stencil strip height (rows per CTA work item)
    int rows_per_step = 1;              // stencil rows per thread step: 1 (k_march) or 2 (k_march2)
    int mw = 128;                       // stencil CTA width in threads (k_march2: 128 or 96)
    int max_nx = 0, max_ny = 0;
    bool any_log = false;               // some member has <logData> doLog set
    const float* elapsed_src = nullptr; // engine handles: the elapsed time of their latest resetTimestep
    std::chrono::steady_clock::time_point created = std::chrono::steady_clock::now();
};

namespace cel {

namespace {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link needed)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }
    return fn;
}

// Row map of one NX x NY plane with pitch P floats: boxes of RBOX x 1 floats; reads outside
// the plane return zero, like the reference's out-of-range texture loads.
int encode_row_map(CUtensorMap* m, const float* plane, int NX, int NY, int P, std::string& err, int box_w = RBOX) {
    auto enc = tensor_map_encoder();
    if (!enc) { err = "cuTensorMapEncodeTiled unavailable"; return CEL_ERR_CUDA; }
    cuuint64_t dims[2] = {cuuint64_t(NX), cuuint64_t(NY)};
    cuuint64_t strides[1] = {cuuint64_t(P) * sizeof(float)};
    cuuint32_t box[2] = {cuuint32_t(box_w), 1u};
    cuuint32_t estr[2] = {1u, 1u};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(plane), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) { err = "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")"; return CEL_ERR_CUDA; }
    return CEL_OK;
}

int dalloc(cel_lane* b, void** ptr, size_t bytes, std::string& err) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) { err = std::string("cudaMalloc: ") + cudaGetErrorString(e); return CEL_ERR_CUDA; }
    e = cudaMemset(q, 0, bytes);
    if (e != cudaSuccess) { err = std::string("cudaMemset: ") + cudaGetErrorString(e); return CEL_ERR_CUDA; }
    b->allocs.push_back(q);
    *ptr = q;
    return CEL_OK;
}

#define B_TRY(expr)                                                                     \
    do {                                                                                \
        cudaError_t _e = (expr);                                                        \
        if (_e != cudaSuccess) { err = std::string(#expr) + ": " + cudaGetErrorString(_e); return CEL_ERR_CUDA; } \
    } while (0)

// Uploads the member's corner grid (HostSetup::corners) into its pitched corner plane: on the legacy
// stream and synchronously when `stream` is null (set-up), else ordered on `stream` from `keep`,
// which the caller holds until the stream has passed the copy.
int upload_corners(const Member& m, const MemberDev& d, cudaStream_t stream, std::string& err,
                   std::vector<float>* keep = nullptr) {
    const int NX = m.hs.NX, NY = m.hs.NY;
    std::vector<float> local;
    std::vector<float>& pl = keep ? *keep : local;
    pl.assign(size_t(d.PC) * (NY + 1), 0.f);
    for (int y = 0; y <= NY; ++y)
        std::memcpy(&pl[size_t(y) * d.PC], &m.hs.corners[size_t(y) * (NX + 1)], sizeof(float) * (NX + 1));
    const cudaError_t e = stream ? cudaMemcpyAsync(d.CORN, pl.data(), pl.size() * sizeof(float), cudaMemcpyHostToDevice, stream)
                                 : cudaMemcpy(d.CORN, pl.data(), pl.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { err = std::string("corner upload: ") + cudaGetErrorString(e); return CEL_ERR_CUDA; }
    return CEL_OK;
}

// Uploads a member's state (RGBA texels); `lo3`, when given, holds the mixed form's low words
// (3 per texel), else they start at zero.
int upload_state(cel_lane* b, int i, const float* rgba, std::string& err, const float* lo3 = nullptr) {
    b->step_stats_valid = false;
    Member& m = b->mem[i];
    const MemberDev& d = b->hdev[i];
    const int NX = m.hs.NX, NY = m.hs.NY;
    std::vector<float> pl[3], lp[3];
    for (int q = 0; q < 3; ++q) { pl[q].assign(m.plane, 0.f); lp[q].assign(lo3 ? m.plane : 0, 0.f); }
    for (int y = 0; y < NY; ++y)
        for (int x = 0; x < NX; ++x)
            for (int q = 0; q < 3; ++q) {
                pl[q][size_t(y) * m.P + x] = rgba[(size_t(y) * NX + x) * 4 + q];
                if (lo3) lp[q][size_t(y) * m.P + x] = lo3[(size_t(y) * NX + x) * 3 + q];
            }
    for (int q = 0; q < 3; ++q) {
        B_TRY(cudaMemcpyAsync(d.S[b->ix.sin][q], pl[q].data(), m.plane * sizeof(float), cudaMemcpyHostToDevice, b->stream));
        if (b->mixed) {
            if (lo3) B_TRY(cudaMemcpyAsync(d.L[b->ix.sin][q], lp[q].data(), m.plane * sizeof(float), cudaMemcpyHostToDevice, b->stream));
            else B_TRY(cudaMemsetAsync(d.L[b->ix.sin][q], 0, m.plane * sizeof(float), b->stream));
        }
    }
    B_TRY(cudaStreamSynchronize(b->stream));
    return CEL_OK;
}

using ColsKernel = void (*)(const MemberDev*, const int2*, int, PassArgs);
template <int NT>
ColsKernel cols_kernel_nt(bool mixed, int cw) {
    if (cw == 32) return mixed ? k_cols<true, 32, NT> : k_cols<false, 32, NT>;
    if (cw == 16) return mixed ? k_cols<true, 16, NT> : k_cols<false, 16, NT>;
    return mixed ? k_cols<true, 8, NT> : k_cols<false, 8, NT>;
}
ColsKernel cols_kernel(bool mixed, int cw, int nt) {
    return nt == 256 ? cols_kernel_nt<256>(mixed, cw) : cols_kernel_nt<512>(mixed, cw);
}

using March2Kernel = void (*)(const MemberDev*, const int4*, int, PassArgs);
March2Kernel march2_kernel(bool mixed, bool adapt, int w) {
    if (w == 96)
        return mixed ? (adapt ? k_march2<true, true, 96> : k_march2<true, false, 96>)
                     : (adapt ? k_march2<false, true, 96> : k_march2<false, false, 96>);
    return mixed ? (adapt ? k_march2<true, true, 128> : k_march2<true, false, 128>)
                 : (adapt ? k_march2<false, true, 128> : k_march2<false, false, 128>);
}

int launch_pass(cel_lane* b, const PassArgs& pa, std::string& err) {
    // the launch checks below read the runtime's last-error state: drop what calls outside this pass
    // left there (they reported it, or ignored it, where they happened)
    (void)cudaGetLastError();
    const size_t nm = b->mem.size();
    if (pa.stats) B_TRY(cudaMemsetAsync(b->stats_all, 0, nm * STATS_N * sizeof(double), b->stream));
    {
        TimedLaunch t(&b->tm, b->stream, "fused_stencil");
        const bool ad = pa.scheme == CEL_SCHEME_PREDICTOR_ADAPTIVE;
        if (b->rows_per_step == 2) {
            march2_kernel(b->mixed, ad, b->mw)<<<b->grid_stencil, b->mw, MARCH2_DYN_SMEM, b->stream>>>(
                b->ddev, b->mtiles, b->nmtiles, pa);
        } else {
            auto* k = b->mixed ? (ad ? k_march<true, true> : k_march<true, false>)
                               : (ad ? k_march<false, true> : k_march<false, false>);
            k<<<b->grid_stencil, MW, 0, b->stream>>>(b->ddev, b->mtiles, b->nmtiles, pa);
        }
    }
    // the row (x) and column (y) solves are independent: fork the column solve onto the side
    // stream and join before the boundaries (a fork/join pair inside the captured graph)
    B_TRY(cudaEventRecord(b->ev_fork, b->stream));
    B_TRY(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
    {
        TimedLaunch t(&b->tm, b->side, "tridiag_cols");
        if (b->cw == 1) {
            if (b->mixed) k_cols_serial<true><<<b->grid_cols, 128, 0, b->side>>>(b->ddev, b->bands, b->nbands, pa);
            else k_cols_serial<false><<<b->grid_cols, 128, 0, b->side>>>(b->ddev, b->bands, b->nbands, pa);
        } else if (b->col_tt) {
            if (b->mixed) k_cols_tt<true><<<b->grid_cols, 512, b->smem_cols, b->side>>>(b->ddev, b->bands, b->nbands, pa);
            else k_cols_tt<false><<<b->grid_cols, 512, b->smem_cols, b->side>>>(b->ddev, b->bands, b->nbands, pa);
        } else if (b->col_cl > 0) {
            // one cluster of col_cl CTAs per 32-column band
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(unsigned(b->nbands) * unsigned(b->col_cl));
            cfg.blockDim = dim3(256);
            cfg.dynamicSmemBytes = 0;
            cfg.stream = b->side;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = unsigned(b->col_cl);
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            const MemberDev* md = b->ddev;
            const int2* bl = b->bands;
            B_TRY(cudaLaunchKernelEx(&cfg, b->mixed ? k_cols_cluster<true> : k_cols_cluster<false>, md, bl, pa));
        } else {
            auto* kc = cols_kernel(b->mixed, b->cw, b->cnt);
            kc<<<b->grid_cols, b->cnt, b->smem_cols, b->side>>>(b->ddev, b->bands, b->nbands, pa);
        }
    }
    {
        TimedLaunch t(&b->tm, b->stream, "tridiag_rows");
        if (b->mixed)
            k_rows<true><<<b->grid_rows, b->rows_threads, b->smem_rows, b->stream>>>(b->ddev, b->rows, b->nrows,
                                                                                    b->rowbuf, pa);
        else
            k_rows<false><<<b->grid_rows, b->rows_threads, b->smem_rows, b->stream>>>(b->ddev, b->rows, b->nrows,
                                                                                     b->rowbuf, pa);
    }
    B_TRY(cudaEventRecord(b->ev_join, b->side));
    B_TRY(cudaStreamWaitEvent(b->stream, b->ev_join, 0));
    for (int side : {1, 0, 3, 2}) {
        if (b->nbitems[side] == 0) continue;
        const int g = std::min(b->nbitems[side], b->sms * 8);
        TimedLaunch t(&b->tm, b->stream, "boundary");
        if (b->two_phase[side]) {
            if (b->mixed) {
                k_boundary<true><<<g, 256, 0, b->stream>>>(b->ddev, b->bitems[side], b->nbitems[side], side, 1, pa.out);
                k_boundary<true><<<g, 256, 0, b->stream>>>(b->ddev, b->bitems[side], b->nbitems[side], side, 2, pa.out);
            } else {
                k_boundary<false><<<g, 256, 0, b->stream>>>(b->ddev, b->bitems[side], b->nbitems[side], side, 1, pa.out);
                k_boundary<false><<<g, 256, 0, b->stream>>>(b->ddev, b->bitems[side], b->nbitems[side], side, 2, pa.out);
            }
        } else {
            if (b->mixed) k_boundary<true><<<g, 256, 0, b->stream>>>(b->ddev, b->bitems[side], b->nbitems[side], side, 0, pa.out);
            else k_boundary<false><<<g, 256, 0, b->stream>>>(b->ddev, b->bitems[side], b->nbitems[side], side, 0, pa.out);
        }
    }
    B_TRY(cudaGetLastError());
    return CEL_OK;
}

// <logData> output after a physical step (engine.cpp:1488-1493): each member whose step count is a
// multiple of its logStep writes the state after the step with the time at the step's start, here
// the member's FP64 clock minus the step's dt, rounded to float.
int log_after_step(cel_lane* b, std::string& err) {
    if (!b->any_log) return CEL_OK;
    const int count = b->sch.last_count;
    for (size_t i = 0; i < b->mem.size(); ++i) {
        const Member& m = b->mem[i];
        const cel_log& lg = m.p.log;
        if (!lg.do_log || count % lg.log_step != 0) continue;
        std::vector<float> host(size_t(m.hs.NX) * m.hs.NY * 4);
        if (int e = lane_get_state(b, int(i), host.data(), err)) return e;
        double t_end = 0;
        float last_dt = b->step_dt[i];   // the dt the clock advanced by at the end of the step
        B_TRY(cudaMemcpyAsync(&t_end, b->hdev[i].time64, sizeof(double), cudaMemcpyDeviceToHost, b->stream));
        if (b->adaptive) B_TRY(cudaMemcpyAsync(&last_dt, b->dt_table + i, sizeof(float), cudaMemcpyDeviceToHost, b->stream));
        B_TRY(cudaStreamSynchronize(b->stream));
        const float t0 = float(t_end - double(last_dt));
        const float elapsed = b->elapsed_src ? *b->elapsed_src
                                             : std::chrono::duration<float>(std::chrono::steady_clock::now() - b->created).count();
        if (int e = log_dump(lg, host.data(), m.hs.nx, m.hs.ny, t0, elapsed, err)) return e;
    }
    return CEL_OK;
}

// Adaptive batches: the CFL rate of every member's current state (before the first pass and
// before each adaptive predictor), then each member's dt for this pass.
int choose_dt_device(cel_lane* b, bool first_of_step, std::string& err) {
    const int n = int(b->mem.size());
    const int scheme = b->sch.time_scheme;
    const bool need_cfl = !b->dt_started || scheme == CEL_SCHEME_PREDICTOR_ADAPTIVE;
    if (need_cfl) {
        B_TRY(cudaMemsetAsync(b->cfl_now, 0, n * sizeof(unsigned int), b->stream));
        TimedLaunch t(&b->tm, b->stream, "cfl");
        k_cfl<<<std::min(b->ntiles, b->sms * 8), 256, 0, b->stream>>>(b->ddev, b->tiles, b->ntiles, b->ix.sin, b->cfl_now);
    }
    k_choose_dt<<<(n + 127) / 128, 128, 0, b->stream>>>(b->ctl, b->dt_table, need_cfl ? b->cfl_now : nullptr, n, scheme,
                                                        first_of_step ? 1 : 0);
    B_TRY(cudaGetLastError());
    b->dt_started = true;
    return CEL_OK;
}

// One pass with the host state machine; updates the buffer indices.
int run_pass(cel_lane* b, bool first_of_step, std::string& err) {
    Scheme& s = b->sch;
    Idx& ix = b->ix;
    if (b->adaptive) {
        if (int e = choose_dt_device(b, first_of_step, err)) return e;
        s.initialized = true;
    } else {
        s.choose_dt(0.f);
    }
    PassArgs pa{};
    pa.scheme = s.time_scheme;
    pa.in = ix.sin;
    if (s.time_scheme == CEL_SCHEME_CORRECTOR) {
        pa.cur = ix.cur;
        pa.out = 3 - pa.in - pa.cur;
    } else {
        ix.cur = ix.sin;
        pa.cur = ix.cur;
        pa.out = (ix.sin + 1) % 3;
    }
    pa.og = ix.og; pa.oog = ix.oog; pa.scr = ix.scr; pa.pred = ix.pred;
    pa.stats = first_of_step ? 1 : 0;
    pa.friction = b->any_friction ? 1 : 0;
    pa.late_flag = b->late_flag;
    if (int e = launch_pass(b, pa, err)) return e;
    if (first_of_step) {
        b->step_stats_valid = true;
        b->step_dt.assign(b->dt_host, b->dt_host + b->mem.size());
    }
    const bool was_pred = s.is_predictor();
    const bool book = s.after_pass();
    if (book) {
        const int o = ix.og, oo = ix.oog, sc = ix.scr;
        ix.og = sc; ix.oog = o; ix.scr = oo;
        k_advance_time<<<(int(b->mem.size()) + 127) / 128, 128, 0, b->stream>>>(b->ddev, b->ctl, int(b->mem.size()));
        B_TRY(cudaGetLastError());
    } else if (was_pred) {
        ix.pred = ix.scr;
        std::swap(ix.scr, ix.spare);
    }
    ix.sin = pa.out;
    if (book) return log_after_step(b, err);
    return CEL_OK;
}

int run_physical_step(cel_lane* b, std::string& err) {
    if (int e = run_pass(b, true, err)) return e;
    while (b->sch.time_scheme == CEL_SCHEME_CORRECTOR)
        if (int e = run_pass(b, false, err)) return e;
    return CEL_OK;
}

void free_graphs(cel_lane* b) {
    for (cudaGraphExec_t g : b->graphs) cudaGraphExecDestroy(g);
    b->graphs.clear();
    b->graph_idx.clear();
    b->graph_pos = 0;
}

// Captures one graph per physical step until the buffer-rotation state repeats.
int build_graphs(cel_lane* b, std::string& err) {
    free_graphs(b);
    Scheme s0 = b->sch;
    Idx i0 = b->ix;
    std::vector<Idx> starts;
    for (int k = 0; k < 24; ++k) {
        starts.push_back(b->ix);
        cudaGraph_t g = nullptr;
        B_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        // no timers and no log writes (host readbacks) inside a capture; replays log after each step
        const bool tm_on = b->tm.enabled, log_on = b->any_log;
        b->tm.enabled = false;
        b->any_log = false;
        int st = run_physical_step(b, err);
        b->tm.enabled = tm_on;
        b->any_log = log_on;
        cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (st) { if (g) cudaGraphDestroy(g); return st; }
        if (ce != cudaSuccess) { err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce); return CEL_ERR_CUDA; }
        cudaGraphExec_t ge = nullptr;
        ce = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) { err = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ce); return CEL_ERR_CUDA; }
        b->graphs.push_back(ge);
        if (b->ix == starts[0]) break;
    }
    b->graph_idx = starts;
    b->sch = s0;
    b->ix = i0;
    b->graph_pos = 0;
    return CEL_OK;
}

}  // namespace

void byte_model(int form, int N, double& stencil, double& step) {
    // Algorithmic HBM bytes per interior cell (compulsory traffic of this design), for the
    // paired-row stencil (k_march2), which rebuilds the bottom from the corner grid:
    //  stencil, predictor: read state 12 + corner grid 4 + history 40 + aux 8;
    //                      write w 4 + rhs 8 + history 20 + aux 8  -> 104
    //  stencil, corrector: + predicted history 20 + CURRENT_STATE w 4  -> 128
    //  (the one-row stencil k_march reads BA, BX and BY: 8 more in each pass)
    //  tridiagonal (x and y): read rhs 8 + factors 24 + base 8, write 8 -> 48
    //  mixed form: + compensation words: stencil w lo read/write 8, solves hu/hv lo 16 -> +24
    const double comp = (form == CEL_FORM_MIXED) ? 1.0 : 0.0;
    const double st_pred = 104 + 8 * comp, st_corr = 128 + 8 * comp;
    const double tri = 48 + 16 * comp;
    stencil = st_pred;
    step = (st_pred + tri) + N * (st_corr + tri);
}

// (Re)builds the stencil strips (height mh) and the column bands (width cw) of a batch, sizes the
// column solver's shared memory and grids, and drops captured graphs (they hold the old lists).
// Lets `kernel` take as much dynamic shared memory as the device allows beside its static shared
// memory.  The limit is an attribute of the function for the whole process, so setting it to one
// batch's need would refuse the larger launches of another live batch; the launches themselves
// still request only what their batch needs (occupancy follows the request, not the limit).
cudaError_t allow_max_dynamic_smem(const void* kernel) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kernel);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - int(fa.sharedSizeBytes));
    return e;
}

int configure_work(cel_lane* b, int cw, int mh, int rps, int mw, int nt, std::string& err) {
    // 32-column bands with 32, 64 or 128 chunks per column (nt = chunks x 32 = 1024, 2048, 4096):
    // the cluster solver, 8 chunks per CTA and nt / 256 CTAs per cluster
    const int cl = (cw == 32 && (nt == 1024 || nt == 2048 || nt == 4096)) ? nt / 256 : 0;
    // 16-column bands with "1 chunk per column" (nt = 16): the tile-transposed solver
    const bool tt = (cw == 16 && nt == 16);
    if (nt != 256 && nt != 512 && cl == 0 && !tt) {
        err = "column solver chunks x band width must be 256 or 512 threads (or 32 columns x 32, 64 or 128 chunks)";
        return CEL_ERR_ARG;
    }
    if (cl > 0 && b->max_ny > cl * CKC * CMC) {
        err = "column band too tall for the cluster solver (" + std::to_string(cl * CKC * CMC) + " rows at most with " +
              std::to_string(cl * CKC) + " chunks per column)";
        return CEL_ERR_ARG;
    }
    if (cl > 0) {
        for (auto* kk : {k_cols_cluster<true>, k_cols_cluster<false>}) {
            if (cl > 8) B_TRY(cudaFuncSetAttribute(reinterpret_cast<const void*>(kk),
                                                   cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(unsigned(cl));
            cfg.blockDim = dim3(256);
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = unsigned(cl);
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int nc = 0;
            B_TRY(cudaOccupancyMaxActiveClusters(&nc, reinterpret_cast<const void*>(kk), &cfg));
            if (nc < 1) { err = "the device cannot place a cluster of " + std::to_string(cl) + " column-solver CTAs"; return CEL_ERR_ARG; }
        }
    }
    if (rps != 1 && rps != 2) { err = "stencil rows per step must be 1 or 2"; return CEL_ERR_ARG; }
    if (mw != 128 && mw != 96) { err = "stencil width must be 128 or 96 threads"; return CEL_ERR_ARG; }
    if (rps == 1) mw = MW;   // the one-row stencil has one width
    b->rows_per_step = rps;
    const int mo = mw - 2;   // output columns per strip
    if (cw != 1 && cw != 8 && cw != 16 && cw != 32) { err = "column band width must be 1, 8, 16 or 32"; return CEL_ERR_ARG; }
    if (mh < 8 || mh > 1024) { err = "strip height must be in [8, 1024]"; return CEL_ERR_ARG; }
    const size_t smem_cols = tt ? sizeof(float) * size_t(TT_CW) * size_t((b->max_ny + 3) & ~3)
                             : (cw == 1 || cl > 0) ? 0 : sizeof(float) * size_t(b->max_ny) * cw;
    if (smem_cols + COLS_STATIC_SMEM > 227 * 1024) { err = "column band too wide for the tallest member (shared memory)"; return CEL_ERR_ARG; }
    std::vector<int4> mt;
    std::vector<int2> bd;
    for (int i = 0; i < int(b->mem.size()); ++i) {
        const HostSetup& hs = b->mem[i].hs;
        for (int y0 = 2; y0 < hs.ny + 2; y0 += mh)
            for (int x0 = 2; x0 < hs.nx + 2; x0 += mo) mt.push_back(make_int4(i, x0, y0, mh));
        if (cw == 1) {
            // one entry per column; columns 0, 1 and past nx+1 are padding (-1) so that each warp
            // covers 32 columns starting on a 128-byte boundary
            const int w = (hs.nx + 2 + 31) / 32 * 32;
            for (int x = 0; x < w; ++x) bd.push_back(make_int2(i, (x >= 2 && x < hs.nx + 2) ? x : -1));
        } else {
            // bands start on multiples of the band width so column loads are sector aligned
            for (int x0 = 0; x0 < hs.nx + 2; x0 += cw) bd.push_back(make_int2(i, x0));
        }
    }
    free_graphs(b);
    B_TRY(cudaStreamSynchronize(b->stream));
    B_TRY(cudaStreamSynchronize(b->side));
    for (void* p : {static_cast<void*>(b->mtiles), static_cast<void*>(b->bands)})
        if (p) { cudaFree(p); b->allocs.erase(std::remove(b->allocs.begin(), b->allocs.end(), p), b->allocs.end()); }
    b->mtiles = nullptr;
    b->bands = nullptr;
    void* p = nullptr;
    if (dalloc(b, &p, mt.size() * sizeof(int4), err)) return CEL_ERR_CUDA;
    b->mtiles = static_cast<int4*>(p);
    if (dalloc(b, &p, bd.size() * sizeof(int2), err)) return CEL_ERR_CUDA;
    b->bands = static_cast<int2*>(p);
    // the allocations' zeroing ran on the legacy stream: finish it before the batch stream writes
    B_TRY(cudaDeviceSynchronize());
    // on the batch stream (non-blocking: it would not wait for legacy-stream copies)
    B_TRY(cudaMemcpyAsync(b->mtiles, mt.data(), mt.size() * sizeof(int4), cudaMemcpyHostToDevice, b->stream));
    B_TRY(cudaMemcpyAsync(b->bands, bd.data(), bd.size() * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
    B_TRY(cudaStreamSynchronize(b->stream));
    b->nmtiles = int(mt.size());
    b->nbands = int(bd.size());
    b->cw = cw;
    b->cnt = nt;
    b->mh = mh;
    b->mw = mw;
    b->smem_cols = smem_cols;
    b->col_cl = cl;
    b->col_tt = tt;
    if (cw == 8 || cw == 16 || cw == 32) {
        for (int i = 0; i < int(b->mem.size()); ++i) k_band_major<<<b->sms * 4, 256, 0, b->stream>>>(b->ddev, i, cw);
        B_TRY(cudaGetLastError());
        B_TRY(cudaStreamSynchronize(b->stream));
    }
    int occ = 1;
    if (cw == 1) {
        b->grid_cols = (b->nbands + 127) / 128;
    } else if (tt) {
        for (auto* kk : {k_cols_tt<true>, k_cols_tt<false>}) B_TRY(allow_max_dynamic_smem(reinterpret_cast<const void*>(kk)));
        B_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, b->mixed ? k_cols_tt<true> : k_cols_tt<false>, 512,
                                                            smem_cols));
        if (occ < 1) { err = "column band too tall for the tile-transposed solver (shared memory)"; return CEL_ERR_ARG; }
        b->grid_cols = std::max(1, std::min(b->nbands, b->sms * occ * 4));
    } else if (cl > 0) {
        b->grid_cols = b->nbands * cl;
    } else {
        ColsKernel kc = cols_kernel(b->mixed, cw, nt);
        B_TRY(allow_max_dynamic_smem(reinterpret_cast<const void*>(kc)));
        B_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kc, nt, smem_cols));
        b->grid_cols = std::max(1, std::min(b->nbands, b->sms * std::max(occ, 1) * 4));
    }
    // both variants of the stencil (fixed and adaptive predictor) run on the same grid
    if (b->rows_per_step == 2) {
        occ = 1 << 20;
        for (auto* k2 : {march2_kernel(b->mixed, false, mw), march2_kernel(b->mixed, true, mw)}) {
            int o = 0;
            B_TRY(allow_max_dynamic_smem(reinterpret_cast<const void*>(k2)));
            B_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k2, mw, MARCH2_DYN_SMEM));
            occ = std::min(occ, o);
        }
    } else {
        occ = 1 << 20;
        for (auto* k1 : {b->mixed ? k_march<true, false> : k_march<false, false>,
                         b->mixed ? k_march<true, true> : k_march<false, true>}) {
            int o = 0;
            B_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k1, MW, 0));
            occ = std::min(occ, o);
        }
    }
    b->grid_stencil = std::max(1, std::min(b->nmtiles, b->sms * std::max(occ, 1)));
    return CEL_OK;
}

cel_lane* lane_create(int n, const cel_params* const* params, const float* const* bathy, const int* bnx,
                        const int* bny, int form, std::string& err) {
    std::unique_ptr<cel_lane> b(new cel_lane());
    b->form = form;
    b->mixed = (form == CEL_FORM_MIXED);
    const int N0 = params[0]->correction_steps;
    for (int i = 0; i < n; ++i) {
        if (params[i]->correction_steps != N0) { err = "batch members must share correctionStepsNum"; return nullptr; }
        if ((params[i]->adaptive != 0) != (params[0]->adaptive != 0)) {
            err = "batch members must share the adaptive time-step setting";
            return nullptr;
        }
        if (params[i]->ny > 6900) { err = "fused form supports ny <= 6900 (column band in shared memory)"; return nullptr; }
        if (params[i]->nx > 16000) { err = "fused form supports nx <= 16000 (row in shared memory)"; return nullptr; }
        if (log_validate(params[i]->log, params[i]->nx, params[i]->ny, err)) {
            err = "member " + std::to_string(i) + ": " + err;
            return nullptr;
        }
        if (params[i]->log.do_log) b->any_log = true;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { err = "no CUDA device"; return nullptr; }
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        err = "stream creation failed";
        return nullptr;
    }
    b->own_stream = true;
    b->mem.resize(n);
    b->hdev.resize(n);
    std::vector<float4> waves;
    std::vector<double> waves64;
    {
        void* p = nullptr;
        const size_t nd = 1 + size_t(n) + 2 * size_t(n) * STATS_N;
        if (dalloc(b.get(), &p, nd * sizeof(double) + size_t(n) * sizeof(float), err)) return nullptr;
        double* blk = static_cast<double*>(p);
        b->late_flag = blk;
        b->clock64 = blk + 1;
        b->stats_all = blk + 1 + n;
        b->stats_now_all = blk + 1 + n + size_t(n) * STATS_N;
        b->clock32 = reinterpret_cast<float*>(blk + nd);
        if (cudaMallocHost(&p, nd * sizeof(double)) != cudaSuccess) { err = "cudaMallocHost failed"; return nullptr; }
        b->rb_host = static_cast<double*>(p);
        if (dalloc(b.get(), &p, size_t(n) * sizeof(float), err)) return nullptr;
        b->dt_table = static_cast<float*>(p);
        if (cudaMallocHost(&p, size_t(n) * sizeof(float)) != cudaSuccess) { err = "cudaMallocHost failed"; return nullptr; }
        b->dt_host = static_cast<float*>(p);
        b->adaptive = params[0]->adaptive != 0;
        if (b->adaptive) {
            if (dalloc(b.get(), &p, size_t(n) * sizeof(DtCtl), err)) return nullptr;
            b->ctl = static_cast<DtCtl*>(p);
            if (dalloc(b.get(), &p, size_t(n) * sizeof(unsigned int), err)) return nullptr;
            b->cfl_now = static_cast<unsigned int*>(p);
            std::vector<DtCtl> c0(n);
            for (int i = 0; i < n; ++i) {
                std::memset(&c0[i], 0, sizeof(DtCtl));
                c0[i].base = float(params[i]->timestep);
                c0[i].min_ratio = float(params[i]->min_timestep_ratio);
                c0[i].alpha = float(params[i]->ema_alpha);
            }
            cudaMemcpy(b->ctl, c0.data(), n * sizeof(DtCtl), cudaMemcpyHostToDevice);
        }
    }
    std::vector<int4> tiles;
    std::vector<int2> rows, bitems[4];
    int max_nx = 0, max_ny = 0;
    for (int i = 0; i < n; ++i) {
        Member& m = b->mem[i];
        m.p = *params[i];
        if (m.p.friction != 0.0) b->any_friction = true;
        if (make_setup(m.p, bathy[i], bnx[i], bny[i], m.hs, err)) return nullptr;
        // the fused solver needs only the level-0 systems
        m.hs.ABCx.resize(1);
        m.hs.ABCy.resize(1);
        const int NX = m.hs.NX, NY = m.hs.NY;
        m.P = (NX + 31) / 32 * 32;
        m.plane = size_t(m.P) * NY;
        b->cells += (long long)m.hs.nx * m.hs.ny;
        max_nx = std::max(max_nx, m.hs.nx);
        max_ny = std::max(max_ny, m.hs.ny);
        MemberDev& d = b->hdev[i];
        std::memset(&d, 0, sizeof(d));
        d.c = make_consts(m.p, m.hs, m.P);
        d.P = m.P;
        d.dx64 = m.p.width / double(m.hs.nx - 1);
        d.dy64 = m.p.length / double(m.hs.ny - 1);
        d.g64 = m.p.gravity;
        b->dt_host[i] = float(m.p.timestep);
        d.dtp = b->dt_table + i;
        d.ab = b->ctl ? b->ctl[i].ab : nullptr;
        // planes: state 9 (+9 lo), bottom 3, rhs 2, history 12 + 8, aux 2, factors 6
        const int nplanes = 9 + (b->mixed ? 9 : 0) + 3 + 2 + 12 + 8 + 2 + 6;
        void* base = nullptr;
        if (dalloc(b.get(), &base, m.plane * nplanes * sizeof(float), err)) return nullptr;
        float* q = static_cast<float*>(base);
        d.base = q;
        d.plane = m.plane;
        {   // tan of the breaking threshold (atan is monotonic on (-pi/2, pi/2))
            const double th = m.p.dissipation_threshold;
            d.tan_thr = th >= M_PI / 2 ? INFINITY : th <= -M_PI / 2 ? -INFINITY : float(std::tan(th));
        }
        auto next = [&]() { float* r = q; q += m.plane; return r; };
        for (int s = 0; s < 3; ++s) for (int k = 0; k < 3; ++k) d.S[s][k] = next();
        if (b->mixed) for (int s = 0; s < 3; ++s) for (int k = 0; k < 3; ++k) d.L[s][k] = next();
        float* by = next(); float* bx = next(); float* ba = next();
        d.BY = by; d.BX = bx; d.BA = ba;
        d.R[0] = next(); d.R[1] = next();
        // history slots: HA (float4 {dw/dt, dhu/dt, dhv/dt, F*}, 4 planes) and HB (G*, 1 plane)
        for (int s = 0; s < 4; ++s) {
            d.HA[s] = reinterpret_cast<float4*>(q); q += 4 * m.plane;
            d.HB[s] = next();
        }
        d.AUX[0] = next(); d.AUX[1] = next();   // one float2 plane pair
        float* fx[3]; float* fy[3];
        for (int k = 0; k < 3; ++k) fx[k] = next();
        for (int k = 0; k < 3; ++k) fy[k] = next();
        for (int k = 0; k < 3; ++k) { d.FX[k] = fx[k]; d.FYF[k] = fy[k]; }
        {   // band-major y factors, sized for the widest band (32 columns)
            const size_t nbm = size_t((m.hs.nx + 2 + 31) / 32) * 32 * m.hs.ny;
            void* fp_ = nullptr;
            if (dalloc(b.get(), &fp_, 3 * nbm * sizeof(float), err)) return nullptr;
            for (int k = 0; k < 3; ++k) d.FYB[k] = static_cast<float*>(fp_) + k * nbm;
        }
        {   // TMA row maps: the three state buffers (w, hu, hv), then BA, BX, BY
            std::vector<CUtensorMap> maps(13);
            for (int sb = 0; sb < 3; ++sb)
                for (int k = 0; k < 3; ++k)
                    if (encode_row_map(&maps[sb * 3 + k], d.S[sb][k], NX, NY, m.P, err)) return nullptr;
            if (encode_row_map(&maps[9], ba, NX, NY, m.P, err) || encode_row_map(&maps[10], bx, NX, NY, m.P, err) ||
                encode_row_map(&maps[11], by, NX, NY, m.P, err))
                return nullptr;
            // the corner grid: rows of CBOX floats, so that a ring row's RBOX cells have both corners
            d.PC = (NX + 1 + 31) / 32 * 32;
            void* cp_ = nullptr;
            if (dalloc(b.get(), &cp_, sizeof(float) * size_t(d.PC) * (NY + 1), err)) return nullptr;
            d.CORN = static_cast<float*>(cp_);
            if (encode_row_map(&maps[12], d.CORN, NX + 1, NY + 1, d.PC, err, CBOX)) return nullptr;
            void* mp = nullptr;
            if (dalloc(b.get(), &mp, sizeof(CUtensorMap) * 13, err)) return nullptr;
            if (cudaMemcpy(mp, maps.data(), sizeof(CUtensorMap) * 13, cudaMemcpyHostToDevice) != cudaSuccess) {
                err = "tensor map upload failed";
                return nullptr;
            }
            d.tmaps = static_cast<const CUtensorMap*>(mp);
        }
        d.stats = b->stats_all + size_t(i) * STATS_N;
        d.stats_now = b->stats_now_all + size_t(i) * STATS_N;
        d.time64 = b->clock64 + i;
        d.time32 = b->clock32 + i;
        // upload planes (pitched)
        auto put = [&](float* dst, const std::vector<float>& src) -> int {
            std::vector<float> pl(m.plane, 0.f);
            for (int y = 0; y < NY; ++y) std::memcpy(&pl[size_t(y) * m.P], &src[size_t(y) * NX], NX * sizeof(float));
            cudaError_t e = cudaMemcpy(dst, pl.data(), m.plane * sizeof(float), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) { err = cudaGetErrorString(e); return CEL_ERR_CUDA; }
            return CEL_OK;
        };
        if (put(by, m.hs.BY) || put(bx, m.hs.BX) || put(ba, m.hs.BA)) return nullptr;
        if (upload_corners(m, d, nullptr, err)) return nullptr;
        {
            std::vector<float> cpv, inv, mv;
            thomas_factors_x(m.hs, cpv, inv, mv);
            if (put(fx[0], cpv) || put(fx[1], inv) || put(fx[2], mv)) return nullptr;
            thomas_factors_y(m.hs, cpv, inv, mv);
            if (put(fy[0], cpv) || put(fy[1], inv) || put(fy[2], mv)) return nullptr;
        }
        // boundaries
        const cel_boundary* sides[4] = {&m.p.north, &m.p.east, &m.p.south, &m.p.west};
        for (int s = 0; s < 4; ++s) {
            const cel_boundary& bb = *sides[s];
            BoundaryDesc& bd = d.bd[s];
            bd.type = bb.type; bd.width = bb.width;
            bd.sea_level = float(bb.sea_level); bd.amplitude = float(bb.amplitude);
            bd.period = float(bb.period); bd.theta = float(bb.theta);
            bd.sea_level64 = bb.sea_level; bd.amplitude64 = bb.amplitude;
            bd.period64 = bb.period; bd.theta64 = bb.theta;
            bd.n_waves = bb.type == CEL_BC_IRREGULAR ? bb.n_waves : 0;
            const int Kn = (s == 0 || s == 2) ? m.hs.Ky : m.hs.Kx;
            bd.nleaf = 1 << (Kn - 1);
            bd.wave_offset = int(waves.size());
            for (int k = 0; k < bd.n_waves; ++k) {
                waves.push_back(make_float4(float(bb.waves[k][0]), float(bb.waves[k][1]), float(bb.waves[k][2]),
                                            float(bb.waves[k][3])));
                for (int q = 0; q < 4; ++q) waves64.push_back(bb.waves[k][q]);
            }
            if (bb.type == CEL_BC_UTS) {
                m.uts_host[s].resize(size_t(bb.n_uts) * 4);
                for (int k = 0; k < 4 * bb.n_uts; ++k) m.uts_host[s][k] = float(bb.uts[k]);
                void* up = nullptr;
                if (dalloc(b.get(), &up, m.uts_host[s].size() * sizeof(float), err)) return nullptr;
                cudaMemcpy(up, m.uts_host[s].data(), m.uts_host[s].size() * sizeof(float), cudaMemcpyHostToDevice);
                d.uts[s] = static_cast<float*>(up);
                if (dalloc(b.get(), &up, size_t(bb.n_uts) * 4 * sizeof(double), err)) return nullptr;
                cudaMemcpy(up, bb.uts, size_t(bb.n_uts) * 4 * sizeof(double), cudaMemcpyHostToDevice);
                d.uts64[s] = static_cast<double*>(up);
                d.nuts[s] = bb.n_uts;
            }
            const int cellsn = (s == 0 || s == 2) ? NX * std::min(bb.width, NY) : std::min(bb.width, NX) * NY;
            for (int c0 = 0; c0 < cellsn; c0 += boundary_item_cells(bb.type)) bitems[s].push_back(make_int2(i, c0));
            // a solid strip wider than 2 reads ghost cells of its own strip: compute, then write
            if (bb.type == CEL_BC_SOLID && bb.width >= 3) b->two_phase[s] = true;
        }
        {
            size_t strip = 0;
            for (int s = 0; s < 4; ++s) {
                const int w = sides[s]->width;
                strip = std::max(strip, size_t((s == 0 || s == 2) ? NX * std::min(w, NY) : std::min(w, NX) * NY));
            }
            void* sp = nullptr;
            const size_t per_cell = b->mixed ? 6 : 3;   // w, hu, hv (+ their low words)
            if (dalloc(b.get(), &sp, std::max<size_t>(strip, 1) * per_cell * sizeof(float), err)) return nullptr;
            d.strip = static_cast<float*>(sp);
        }
        // work lists
        for (int y0 = 2; y0 < m.hs.ny + 2; y0 += TY)
            for (int x0 = 2; x0 < m.hs.nx + 2; x0 += TX) tiles.push_back(make_int4(i, x0, y0, 0));
        for (int y = 2; y < m.hs.ny + 2; ++y) rows.push_back(make_int2(i, y));
    }
    b->max_nx = max_nx;
    b->max_ny = max_ny;
    {
        void* wp = nullptr;
        if (waves.empty()) waves.push_back(make_float4(0, 0, 0, 0));
        if (dalloc(b.get(), &wp, waves.size() * sizeof(float4), err)) return nullptr;
        cudaMemcpy(wp, waves.data(), waves.size() * sizeof(float4), cudaMemcpyHostToDevice);
        for (auto& d : b->hdev) d.waves = static_cast<float4*>(wp);
        if (waves64.empty()) waves64.assign(4, 0.0);
        if (dalloc(b.get(), &wp, waves64.size() * sizeof(double), err)) return nullptr;
        cudaMemcpy(wp, waves64.data(), waves64.size() * sizeof(double), cudaMemcpyHostToDevice);
        for (auto& d : b->hdev) d.waves64 = static_cast<double*>(wp);
    }
    // Sort tiles and lines so that large domains are scheduled first (load balance).
    auto upload_list = [&](auto& v, auto** dst, int& cnt) -> int {
        cnt = int(v.size());
        void* p = nullptr;
        if (dalloc(b.get(), &p, std::max<size_t>(v.size(), 1) * sizeof(v[0]), err)) return CEL_ERR_CUDA;
        if (!v.empty()) cudaMemcpy(p, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice);
        *dst = static_cast<std::remove_reference_t<decltype(**dst)>*>(p);
        return CEL_OK;
    };
    if (upload_list(tiles, &b->tiles, b->ntiles) || upload_list(rows, &b->rows, b->nrows)) return nullptr;
    for (int s = 0; s < 4; ++s)
        if (upload_list(bitems[s], &b->bitems[s], b->nbitems[s])) return nullptr;
    {
        void* p = nullptr;
        if (dalloc(b.get(), &p, sizeof(MemberDev) * n, err)) return nullptr;
        b->ddev = static_cast<MemberDev*>(p);
        cudaMemcpy(b->ddev, b->hdev.data(), sizeof(MemberDev) * n, cudaMemcpyHostToDevice);
    }
    // row solver: one warp per row, each with a buffer of the row's forward values (whole tiles)
    b->rowbuf = (max_nx + 2 + RT - 1) / RT * RT;
    {
        const size_t per_warp = sizeof(float) * size_t(b->rowbuf);
        const int warps = int(std::min<size_t>(8, (200 * 1024) / per_warp));
        if (warps < 1) { err = "domain too large for the fused solver"; return nullptr; }
        b->rows_threads = 32 * warps;
        b->smem_rows = per_warp * warps;
    }
    for (const void* kr : {reinterpret_cast<const void*>(k_rows<false>), reinterpret_cast<const void*>(k_rows<true>)})
        if (allow_max_dynamic_smem(kr) != cudaSuccess) { err = "cannot raise the row solver's shared-memory limit"; return nullptr; }
    {
        int occ = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rows<true>, b->rows_threads, b->smem_rows);
        const int wpc = b->rows_threads / 32;
        b->grid_rows = std::max(1, std::min((b->nrows + wpc - 1) / wpc, b->sms * std::max(occ, 1)));
    }
    {   // column bands of 16 columns (8 for tall domains: shared-memory capacity), strips of 64 rows
        const int cw = (size_t(max_ny) * 16 * sizeof(float) + COLS_STATIC_SMEM <= 227 * 1024) ? 16 : 8;
        if (configure_work(b.get(), cw, MH_DEFAULT, 1, MW, NTC_DEFAULT, err)) return nullptr;
    }
    b->sch.reset(*params[0]);
    cudaMemcpy(b->dt_table, b->dt_host, sizeof(float) * n, cudaMemcpyHostToDevice);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { err = std::string("batch setup: ") + cudaGetErrorString(e); return nullptr; }
    // initial condition
    for (int i = 0; i < n; ++i) {
        const HostSetup& hs = b->mem[i].hs;
        const size_t nt = size_t(hs.NX) * hs.NY;
        std::vector<float> rgba(nt * 4, 0.f), lo;
        if (b->mixed) {
            // the compensated form starts from the double-precision initial condition: hi + lo
            lo.assign(nt * 3, 0.f);
            for (size_t k = 0; k < nt; ++k)
                for (int q = 0; q < 3; ++q) {
                    const double v = hs.ic64[3 * k + q];
                    const float hi = float(v);
                    rgba[4 * k + q] = hi;
                    lo[3 * k + q] = float(v - double(hi));
                }
        } else {
            for (size_t k = 0; k < nt; ++k) {
                rgba[4 * k] = hs.ic[3 * k]; rgba[4 * k + 1] = hs.ic[3 * k + 1]; rgba[4 * k + 2] = hs.ic[3 * k + 2];
            }
        }
        if (upload_state(b.get(), i, rgba.data(), err, lo.empty() ? nullptr : lo.data())) return nullptr;
    }
    // The set-up copies and memsets above ran on the legacy stream, which the batch's non-blocking
    // streams do not wait for (and a pageable upload may return before its DMA lands): finish them.
    if (cudaDeviceSynchronize() != cudaSuccess) { err = "batch setup: device synchronisation failed"; return nullptr; }
    return b.release();
}

void lane_destroy(cel_lane* b) {
    if (!b) return;
    free_graphs(b);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->side) cudaStreamSynchronize(b->side);
    for (void* a : b->allocs) cudaFree(a);
    if (b->dt_host) cudaFreeHost(b->dt_host);
    if (b->rb_host) cudaFreeHost(b->rb_host);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->dt_copied) cudaEventDestroy(b->dt_copied);
    delete b;
    (void)cudaGetLastError();   // teardown has no caller to report to; leave no stale error behind
}

int lane_set_stream(cel_lane* b, cudaStream_t s, std::string& err) {
    B_TRY(cudaStreamSynchronize(b->stream));
    free_graphs(b);
    if (b->own_stream) cudaStreamDestroy(b->stream);
    b->own_stream = (s == nullptr);
    if (b->own_stream) B_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    else b->stream = s;
    return CEL_OK;
}

int lane_step(cel_lane* b, int nsteps, std::string& err) {
    for (int k = 0; k < nsteps; ++k) {
        const bool bootstrap = b->sch.timestep_count < 3;
        if (b->use_graph && !bootstrap) {
            if (b->graphs.empty()) { if (int e = build_graphs(b, err)) return e; }
            // keep the host state machine and indices in step with the replayed graph
            if (!(b->ix == b->graph_idx[b->graph_pos])) { if (int e = build_graphs(b, err)) return e; }
            B_TRY(cudaGraphLaunch(b->graphs[b->graph_pos], b->stream));
            // advance host bookkeeping exactly like run_physical_step without launching
            Scheme& s = b->sch;
            Idx& ix = b->ix;
            do {
                if (!b->adaptive) s.choose_dt(0.f);
                const int in = ix.sin;
                int out;
                if (s.time_scheme == CEL_SCHEME_CORRECTOR) out = 3 - in - ix.cur;
                else { ix.cur = ix.sin; out = (ix.sin + 1) % 3; }
                const bool was_pred = s.is_predictor();
                const bool book = s.after_pass();
                if (book) { const int o = ix.og, oo = ix.oog, sc = ix.scr; ix.og = sc; ix.oog = o; ix.scr = oo; }
                else if (was_pred) { ix.pred = ix.scr; std::swap(ix.scr, ix.spare); }
                ix.sin = out;
            } while (s.time_scheme == CEL_SCHEME_CORRECTOR);
            b->graph_pos = (b->graph_pos + 1) % int(b->graphs.size());
            b->step_stats_valid = true;
            b->step_dt.assign(b->dt_host, b->dt_host + b->mem.size());
            if (int e = log_after_step(b, err)) return e;
        } else {
            if (int e = run_physical_step(b, err)) return e;
        }
    }
    return CEL_OK;
}

int lane_stats(cel_lane* b, cel_stats* out, bool current, std::string& err) {
    if (int e = lane_stats_enqueue(b, current, err)) return e;
    return lane_stats_finish(b, out, current, err);
}

// The statistics pass (when the step's own totals do not describe the current state) and the
// read-back copies, on the lane's stream; lane_stats_finish waits for them.
int lane_stats_enqueue(cel_lane* b, bool current, std::string& err) {
    const size_t n = b->mem.size();
    const bool at_step = !current && b->step_stats_valid;
    if (!at_step) {
        B_TRY(cudaMemsetAsync(b->stats_now_all, 0, n * STATS_N * sizeof(double), b->stream));
        k_stats_only<<<std::min(b->ntiles, b->sms * 8), 256, 0, b->stream>>>(b->ddev, b->tiles, b->ntiles, b->ix.sin);
        B_TRY(cudaGetLastError());
    }
    // flag, clocks and the step's statistics are contiguous: one copy into pinned memory
    double* h = b->rb_host;
    const size_t head = 1 + n;
    if (at_step) {
        B_TRY(cudaMemcpyAsync(h, b->late_flag, (head + n * STATS_N) * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    } else {
        B_TRY(cudaMemcpyAsync(h, b->late_flag, head * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
        B_TRY(cudaMemcpyAsync(h + head, b->stats_now_all, n * STATS_N * sizeof(double), cudaMemcpyDeviceToHost,
                              b->stream));
    }
    b->ctl_host.resize(b->adaptive ? n : 0);
    if (b->adaptive)
        B_TRY(cudaMemcpyAsync(b->ctl_host.data(), b->ctl, n * sizeof(DtCtl), cudaMemcpyDeviceToHost, b->stream));
    return CEL_OK;
}

int lane_stats_finish(cel_lane* b, cel_stats* out, bool current, std::string& err) {
    const size_t n = b->mem.size();
    const bool at_step = !current && b->step_stats_valid;
    const double* h = b->rb_host;
    const size_t head = 1 + n;
    const std::vector<DtCtl>& ctl = b->ctl_host;
    B_TRY(cudaStreamSynchronize(b->stream));
    const double late = h[0];
    const double* t64 = h + 1;
    const double* v = h + head;
    for (size_t i = 0; i < n; ++i) {
        const double* s = &v[i * STATS_N];
        const Member& m = b->mem[i];
        const double DENSITY = 1000;
        const double AREA = double(float(m.p.width) / float(m.hs.nx - 1) * float(m.p.length) / float(m.hs.ny - 1));
        const double g = m.p.gravity;
        cel_stats& o = out[i];
        std::memset(&o, 0, sizeof(o));
        o.mass = s[0] * DENSITY * AREA;
        o.potential_energy = s[1] * g * DENSITY * AREA;
        o.x_momentum = s[2] * DENSITY * AREA;
        o.y_momentum = s[3] * DENSITY * AREA;
        o.kinetic_energy = s[4] * 0.5 * DENSITY * AREA;
        o.total_energy = o.kinetic_energy + o.potential_energy;
        o.mass_full = s[5];
        o.max_speed = std::sqrt(s[6]);
        o.max_depth = s[7];
        o.cfl_rate = s[8];
        o.max_froude = std::sqrt(s[9] / g);
        o.health = s[10] != 0 ? CEL_ERR_NUMERIC : 0;
        // a bounded TMA wait that gave up (should never happen) is a CUDA error of the batch
        if (late != 0) o.health = CEL_ERR_CUDA;
        // adaptive members: the dt of the step's first pass; the clock advanced by the last pass's dt
        // (before an adaptive batch's first pass its controllers have chosen nothing: the uniform step)
        o.timestep = (b->adaptive && b->dt_started) ? double(ctl[i].dt_first) : double(b->dt_host[i]);
        o.cfl_number = o.cfl_rate * o.timestep;
        const double last_dt = (b->adaptive && b->dt_started) ? double(ctl[i].dt) : double(b->step_dt.empty() ? 0.f : b->step_dt[i]);
        o.total_time = at_step ? t64[i] - last_dt : t64[i];
        o.time_scheme = b->sch.time_scheme;
    }
    return CEL_OK;
}

// The state as two float textures whose sum is the compensated value: hi = the stored state, lo =
// its low words (zero in the FP32 forms).  Either pointer may be null.
int lane_get_state_parts(cel_lane* b, int i, float* hi_rgba, float* lo_rgba, std::string& err) {
    if (i < 0 || i >= int(b->mem.size())) { err = "member index out of range"; return CEL_ERR_ARG; }
    Member& m = b->mem[i];
    const MemberDev& d = b->hdev[i];
    const int NX = m.hs.NX, NY = m.hs.NY;
    std::vector<float> pl[3], lo[3];
    for (int q = 0; q < 3; ++q) {
        pl[q].resize(m.plane);
        lo[q].assign(m.plane, 0.f);
        B_TRY(cudaMemcpyAsync(pl[q].data(), d.S[b->ix.sin][q], m.plane * sizeof(float), cudaMemcpyDeviceToHost, b->stream));
        if (b->mixed)
            B_TRY(cudaMemcpyAsync(lo[q].data(), d.L[b->ix.sin][q], m.plane * sizeof(float), cudaMemcpyDeviceToHost, b->stream));
    }
    B_TRY(cudaStreamSynchronize(b->stream));
    for (int y = 0; y < NY; ++y)
        for (int x = 0; x < NX; ++x) {
            const size_t k = size_t(y) * m.P + x, o = (size_t(y) * NX + x) * 4;
            for (int q = 0; q < 3; ++q) {
                if (hi_rgba) hi_rgba[o + q] = pl[q][k];
                if (lo_rgba) lo_rgba[o + q] = lo[q][k];
            }
            if (hi_rgba) hi_rgba[o + 3] = 0.f;
            if (lo_rgba) lo_rgba[o + 3] = 0.f;
        }
    return CEL_OK;
}

int lane_get_state(cel_lane* b, int i, float* rgba, std::string& err) {
    if (i < 0 || i >= int(b->mem.size())) { err = "member index out of range"; return CEL_ERR_ARG; }
    Member& m = b->mem[i];
    const MemberDev& d = b->hdev[i];
    const int NX = m.hs.NX, NY = m.hs.NY;
    std::vector<float> pl[3], lo[3];
    for (int q = 0; q < 3; ++q) {
        pl[q].resize(m.plane);
        B_TRY(cudaMemcpyAsync(pl[q].data(), d.S[b->ix.sin][q], m.plane * sizeof(float), cudaMemcpyDeviceToHost, b->stream));
        if (b->mixed) {
            lo[q].resize(m.plane);
            B_TRY(cudaMemcpyAsync(lo[q].data(), d.L[b->ix.sin][q], m.plane * sizeof(float), cudaMemcpyDeviceToHost, b->stream));
        }
    }
    B_TRY(cudaStreamSynchronize(b->stream));
    for (int y = 0; y < NY; ++y)
        for (int x = 0; x < NX; ++x) {
            const size_t k = size_t(y) * m.P + x;
            float* o = rgba + (size_t(y) * NX + x) * 4;
            for (int q = 0; q < 3; ++q) o[q] = b->mixed ? float(double(pl[q][k]) + double(lo[q][k])) : pl[q][k];
            o[3] = 0.f;
        }
    return CEL_OK;
}

int lane_set_state(cel_lane* b, int i, const float* rgba, std::string& err) {
    if (i < 0 || i >= int(b->mem.size())) { err = "member index out of range"; return CEL_ERR_ARG; }
    return upload_state(b, i, rgba, err);
}

// newTerrainSettings for member i (engine.cpp:3313-3379): every texel keeps its water depth
// (w - BA_old + BA_new; in double on the compensated state of the mixed form), the bottom planes
// are resampled from the new grid, the aux planes are cleared; the Thomas factors stay those of
// the old bottom, as the reference keeps its coefficient textures until a remesh.
int lane_set_bathymetry(cel_lane* b, int i, const float* z, int bnx, int bny, std::string& err) {
    if (i < 0 || i >= int(b->mem.size())) { err = "member index out of range"; return CEL_ERR_ARG; }
    if (!z || bnx < 2 || bny < 2) { err = "bathymetry grid needs at least 2 x 2 values"; return CEL_ERR_ARG; }
    Member& m = b->mem[i];
    MemberDev& d = b->hdev[i];
    const int NX = m.hs.NX, NY = m.hs.NY, sin = b->ix.sin;
    std::vector<float> hi(m.plane), lo(b->mixed ? m.plane : 0);
    B_TRY(cudaMemcpyAsync(hi.data(), d.S[sin][0], m.plane * sizeof(float), cudaMemcpyDeviceToHost, b->stream));
    if (b->mixed)
        B_TRY(cudaMemcpyAsync(lo.data(), d.L[sin][0], m.plane * sizeof(float), cudaMemcpyDeviceToHost, b->stream));
    B_TRY(cudaStreamSynchronize(b->stream));
    const std::vector<float> ba_old = m.hs.BA;
    prepare_bottom(z, bnx, bny, m.hs.nx, m.hs.ny, float(m.p.width), float(m.p.length), m.hs);
    std::vector<float> by(m.plane, 0.f), bx(m.plane, 0.f), ba(m.plane, 0.f);
    for (int y = 0; y < NY; ++y)
        for (int x = 0; x < NX; ++x) {
            const size_t k = size_t(y) * NX + x, e = size_t(y) * m.P + x;
            by[e] = m.hs.BY[k]; bx[e] = m.hs.BX[k]; ba[e] = m.hs.BA[k];
            if (b->mixed) {
                const double w = (double(hi[e]) + double(lo[e])) - double(ba_old[k]) + double(m.hs.BA[k]);
                hi[e] = float(w);
                lo[e] = float(w - double(hi[e]));
            } else {
                hi[e] = (hi[e] - ba_old[k]) + m.hs.BA[k];
            }
        }
    // ordered on the batch stream, and complete before the host buffers go out of scope
    const size_t pb = m.plane * sizeof(float);
    B_TRY(cudaMemcpyAsync(const_cast<float*>(d.BY), by.data(), pb, cudaMemcpyHostToDevice, b->stream));
    B_TRY(cudaMemcpyAsync(const_cast<float*>(d.BX), bx.data(), pb, cudaMemcpyHostToDevice, b->stream));
    B_TRY(cudaMemcpyAsync(const_cast<float*>(d.BA), ba.data(), pb, cudaMemcpyHostToDevice, b->stream));
    std::vector<float> corners;
    if (int e = upload_corners(m, d, b->stream, err, &corners)) return e;
    B_TRY(cudaMemcpyAsync(d.S[sin][0], hi.data(), pb, cudaMemcpyHostToDevice, b->stream));
    if (b->mixed) B_TRY(cudaMemcpyAsync(d.L[sin][0], lo.data(), pb, cudaMemcpyHostToDevice, b->stream));
    B_TRY(cudaMemsetAsync(d.AUX[0], 0, 2 * pb, b->stream));
    B_TRY(cudaStreamSynchronize(b->stream));
    b->step_stats_valid = false;   // the gathered totals describe the state before the change
    return CEL_OK;
}

// addSolitaryWave (engine.cpp:2154-2219) on member i; theta in degrees
int lane_add_solitary_wave(cel_lane* b, int i, double H, double theta_deg, double xc, double yc, std::string& err) {
    if (i < 0 || i >= int(b->mem.size())) { err = "member index out of range"; return CEL_ERR_ARG; }
    const HostSetup& hs = b->mem[i].hs;
    const float th = float(theta_deg) * 3.14159274101257324f / 180.0f;
    const dim3 blk(32, 8), grd((hs.nx + 2 + 31) / 32, (hs.ny + 2 + 7) / 8);
    if (b->mixed)
        k_add_solitary<true><<<grd, blk, 0, b->stream>>>(b->ddev, i, b->ix.sin, float(H), th, float(xc), float(yc));
    else
        k_add_solitary<false><<<grd, blk, 0, b->stream>>>(b->ddev, i, b->ix.sin, float(H), th, float(xc), float(yc));
    B_TRY(cudaGetLastError());
    B_TRY(cudaStreamSynchronize(b->stream));
    b->step_stats_valid = false;
    return CEL_OK;
}

int lane_get_aux(cel_lane* b, int i, float* rgba, std::string& err) {
    if (i < 0 || i >= int(b->mem.size())) { err = "member index out of range"; return CEL_ERR_ARG; }
    Member& m = b->mem[i];
    const MemberDev& d = b->hdev[i];
    // AUX is one float2 plane pair: {max inundated depth, breaking indicator} per texel
    std::vector<float> a(2 * m.plane);
    B_TRY(cudaMemcpyAsync(a.data(), d.AUX[0], 2 * m.plane * sizeof(float), cudaMemcpyDeviceToHost, b->stream));
    B_TRY(cudaStreamSynchronize(b->stream));
    const int NX = m.hs.NX, NY = m.hs.NY;
    for (int y = 0; y < NY; ++y)
        for (int x = 0; x < NX; ++x) {
            float* o = rgba + (size_t(y) * NX + x) * 4;
            const size_t k = 2 * (size_t(y) * m.P + x);
            o[0] = a[k]; o[1] = 0.f; o[2] = 0.f; o[3] = a[k + 1];
        }
    return CEL_OK;
}

int lane_use_graph(cel_lane* b, bool enable, std::string& err) {
    (void)err;
    if (!enable) free_graphs(b);
    b->use_graph = enable;
    return CEL_OK;
}

long long lane_cells(const cel_lane* b) { return b->cells; }

int lane_set_timestep(cel_lane* b, const float* dt, std::string& err) {
    if (b->adaptive) { err = "an adaptive batch chooses its time steps on the device"; return CEL_ERR_STATE; }
    // the uniform time step of each member (the reference's "uniform time step" setting,
    // uploaded with the constant buffers before every pass, engine.cpp:1728-1750)
    for (size_t i = 0; i < b->mem.size(); ++i)
        if (!(dt[i] > 0.f)) { err = "time steps must be > 0"; return CEL_ERR_ARG; }
    // the previous upload reads the same pinned buffer: let it finish before the buffer changes
    if (!b->dt_copied) B_TRY(cudaEventCreateWithFlags(&b->dt_copied, cudaEventDisableTiming));
    B_TRY(cudaEventSynchronize(b->dt_copied));
    for (size_t i = 0; i < b->mem.size(); ++i) b->dt_host[i] = dt[i];
    B_TRY(cudaMemcpyAsync(b->dt_table, b->dt_host, sizeof(float) * b->mem.size(), cudaMemcpyHostToDevice, b->stream));
    B_TRY(cudaEventRecord(b->dt_copied, b->stream));
    return CEL_OK;
}

int lane_set_tuning(cel_lane* b, int tx, int ty, int pcr, std::string& err) {
    // pcr: chunks per column of the column solver (the carry scan joins that many chunks; each is
    // swept serially), so the CTA has pcr x band width threads; 0 keeps the threads per CTA
    const int cw = tx > 0 ? tx : b->cw;
    const int nt = (pcr > 0 && cw > 1) ? pcr * cw : b->cnt;
    return configure_work(b, cw, ty > 0 ? ty : b->mh, b->rows_per_step, b->mw, nt, err);
}

int lane_get_tuning(const cel_lane* b, int* tx, int* ty, int* rps) {
    if (tx) *tx = b->cw;
    if (ty) *ty = b->mh;
    if (rps) *rps = b->rows_per_step;
    return CEL_OK;
}

int lane_col_chunks(const cel_lane* b) { return b->cw > 1 ? b->cnt / b->cw : 1; }

int lane_set_stencil_rows(cel_lane* b, int rps, std::string& err) {
    return configure_work(b, b->cw, b->mh, rps, rps == 2 ? b->mw : MW, b->cnt, err);
}

int lane_set_stencil_width(cel_lane* b, int threads, std::string& err) {
    if (b->rows_per_step != 2 && threads != MW) {
        err = "the one-row stencil runs 128-thread strips; select two rows per step first";
        return CEL_ERR_ARG;
    }
    return configure_work(b, b->cw, b->mh, b->rows_per_step, threads, b->cnt, err);
}

int lane_stencil_width(const cel_lane* b) { return b->mw; }

cudaStream_t lane_stream(const cel_lane* b) { return b->stream; }
int lane_members(const cel_lane* b) { return int(b->mem.size()); }
int lane_max_ny(const cel_lane* b) { return b->max_ny; }
int lane_configure(cel_lane* b, int cw, int mh, int rps, int mw, int nt, std::string& err) {
    return configure_work(b, cw, mh, rps, mw, nt, err);
}
int lane_col_threads(const cel_lane* b) { return b->cnt; }

KernelTimer* lane_timer(cel_lane* b) { return &b->tm; }

int lane_launches_per_step(const cel_lane* b) {
    int per_pass = 3;  // stencil, row solve, column solve
    for (int s = 0; s < 4; ++s)
        if (b->nbitems[s] > 0) per_pass += b->two_phase[s] ? 2 : 1;
    // adaptive batches add the dt choice before every pass and the CFL reduction before the predictor
    if (b->adaptive) per_pass += 1;
    return (1 + b->sch.N) * per_pass + 1 + (b->adaptive ? 1 : 0);  // + the clock advance
}

// ---- single-domain fused engine (a batch of one) behind the engine interface ---------------
namespace {

class FusedEngine : public EngineIface {
public:
    cel_lane* b = nullptr;
    cel_params p{};
    std::vector<float> bathy;
    int bnx = 0, bny = 0, form = CEL_FORM_FUSED;
    ~FusedEngine() override { lane_destroy(b); }
    int make() {
        const cel_params* pp = &p;
        const float* bz = bathy.empty() ? nullptr : bathy.data();
        std::vector<float> tmp;
        if (!bz) {
            if (int st = read_cbf(p.bathymetry_path, &tmp, bnx, bny, err)) return st;
            bz = tmp.data();
        }
        b = lane_create(1, &pp, &bz, &bnx, &bny, form, err);
        if (b) b->elapsed_src = &log_elapsed;
        return b ? CEL_OK : CEL_ERR_ARG;
    }
    int remesh() override {
        lane_destroy(b);
        b = nullptr;
        return make();
    }
    int set_state(const float* rgba) override { return lane_set_state(b, 0, rgba, err); }
    int get_state(float* rgba) override { return lane_get_state(b, 0, rgba, err); }
    int get_bottom(float* b3) override {
        const HostSetup& hs = b->mem[0].hs;
        for (size_t i = 0; i < hs.BA.size(); ++i) { b3[3 * i] = hs.BY[i]; b3[3 * i + 1] = hs.BX[i]; b3[3 * i + 2] = hs.BA[i]; }
        return CEL_OK;
    }
    int get_aux(float* rgba) override { return lane_get_aux(b, 0, rgba, err); }
    int reset_timestep(float, float, cel_stats* out) override {
        if (!b->adaptive) b->sch.choose_dt(0.f);
        if (!out) return CEL_OK;
        return lane_stats(b, out, true, err);
    }
    int timestep() override { return run_pass(b, b->sch.time_scheme != CEL_SCHEME_CORRECTOR, err); }
    int timesteps(int n) override {
        for (int i = 0; i < n; ++i)
            if (int e = run_pass(b, b->sch.time_scheme != CEL_SCHEME_CORRECTOR, err)) return e;
        return CEL_OK;
    }
    int physical_steps(int n) override { return lane_step(b, n, err); }
    int get_stats(cel_stats* out) override { return lane_stats(b, out, true, err); }
    int add_solitary_wave(double Hh, double theta_deg, double xc, double yc) override {
        return lane_add_solitary_wave(b, 0, Hh, theta_deg, xc, yc, err);
    }
    // the block's depth sum is taken from the current state, in GetStats' order (compute.hlsl:1331-1345)
    int water_height(float x, float y, float* out) override {
        const HostSetup& hs = b->mem[0].hs;
        const float W = float(p.width), L = float(p.length);
        if (hs.nx < 4 || hs.ny < 4) { err = "getWaterHeight needs at least one 4x4 block"; return CEL_ERR_STATE; }
        std::vector<float> st(size_t(hs.NX) * hs.NY * 4);
        if (int e = lane_get_state(b, 0, st.data(), err)) return e;
        int ix = 0, iy = 0;
        water_height_block(hs.nx, hs.ny, W, L, x, y, ix, iy);
        float sum_h = 0.f;
        for (int j = 2; j < 6; ++j)
            for (int i = 2; i < 6; ++i) {
                const size_t k = size_t(iy * 4 + j) * hs.NX + ix * 4 + i;
                sum_h += std::max(0.f, st[4 * k] - hs.BA[k]);
            }
        *out = terrain_height(hs, W, L, x, y) + sum_h / 16.0f;
        return CEL_OK;
    }
    int set_bathymetry(const float* z, int gx, int gy) override {
        if (int st = lane_set_bathymetry(b, 0, z, gx, gy, err)) return st;
        bathy.assign(z, z + size_t(gx) * gy);   // a remesh starts over from the new grid
        bnx = gx;
        bny = gy;
        return CEL_OK;
    }
    int set_stream(cudaStream_t s) override { return lane_set_stream(b, s, err); }
    int synchronize() override {
        cudaError_t e = cudaStreamSynchronize(b->stream);
        if (e != cudaSuccess) { err = cudaGetErrorString(e); return CEL_ERR_CUDA; }
        return CEL_OK;
    }
    int set_tuning(int tx, int ty, int pcr) override { return lane_set_tuning(b, tx, ty, pcr, err); }
    KernelTimer* timer() override { return &b->tm; }
    int nx() const override { return p.nx; }
    int ny() const override { return p.ny; }
};

}  // namespace

EngineIface* make_fused_engine(const cel_params& p, const float* bathy, int bnx, int bny, int form, std::string& err) {
    auto* e = new FusedEngine();
    e->p = p;
    e->form = form;
    e->bnx = bnx;
    e->bny = bny;
    if (bathy) e->bathy.assign(bathy, bathy + size_t(bnx) * bny);
    if (int st = e->make()) {
        err = e->err;
        delete e;
        (void)st;
        return nullptr;
    }
    return e;
}

int selftest_reciprocal(const float* x, float* out, int n, std::string& err) {
    if (n < 0 || (n > 0 && (!x || !out))) { err = "selftest_reciprocal: bad arguments"; return CEL_ERR_ARG; }
    if (n == 0) return CEL_OK;
    float* d = nullptr;
    B_TRY(cudaMalloc(&d, 2 * sizeof(float) * size_t(n)));
    cudaError_t e = cudaMemcpy(d, x, sizeof(float) * size_t(n), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_rcp_selftest<<<std::min((n + 255) / 256, 4096), 256>>>(d, d + n, n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d + n, sizeof(float) * size_t(n), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) { err = std::string("selftest_reciprocal: ") + cudaGetErrorString(e); return CEL_ERR_CUDA; }
    return CEL_OK;
}

}  // namespace cel
