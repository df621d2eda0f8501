// Plain FP32 form: one CUDA kernel per reference pass and one per cyclic-reduction level,
// over float4 "textures" with the reference's ghost layout.  This is the straightforward GPU
// restatement of timestep()/resetTimestep() (engine.cpp:849-1756) and of the compute.hlsl
// pixel shaders; it is compiled with -fmad=false so its arithmetic follows the FP32
// transcription operation by operation.  One domain per launch set.
#define CEL_EXACT_FP32 1
#include <cuda_runtime.h>

#include <mutex>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "device_math.cuh"
#include "engine_iface.hpp"
#include "scheme.hpp"

namespace cel {

namespace {

constexpr int BX2 = 32, BY2 = 8;

inline dim3 grid2(int w, int h) { return dim3((w + BX2 - 1) / BX2, (h + BY2 - 1) / BY2); }

// ---- Pass1 (compute.hlsl:380-458): faces h,u,v {N,E,S,W}; aux; region [1,nx+3)x[1,ny+3) ----
__global__ void k_pass1(const float4* __restrict__ st, const float4* __restrict__ bot,
                        const float4* __restrict__ aux1, float4* __restrict__ H, float4* __restrict__ U,
                        float4* __restrict__ V, float4* __restrict__ aux2, SimConsts c) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (x >= c.nx + 3 || y >= c.ny + 3) return;
    const int NX = c.NX;
    const size_t i = size_t(y) * NX + x;
    const float4 cc = st[i], s = st[i - NX], n = st[i + NX], w = st[i - 1], e = st[i + 1];
    const float BN = bot[i].x, BE = bot[i].y, BS = bot[i - NX].x, BW = bot[i - 1].y;
    float wN, wE, wS, wW, huN, huE, huS, huW, hvN, hvE, hvS, hvW, sd, msd;
    reconstruct_sd(c.two_theta, w.x, cc.x, e.x, wW, wE, sd);
    msd = sd * c.one_over_dx;
    reconstruct_sd(c.two_theta, s.x, cc.x, n.x, wS, wN, sd);
    msd = t_atan(fmaxf(msd, sd * c.one_over_dy));
    reconstruct(c.two_theta, w.y, cc.y, e.y, huW, huE);
    reconstruct(c.two_theta, s.y, cc.y, n.y, huS, huN);
    reconstruct(c.two_theta, w.z, cc.z, e.z, hvW, hvE);
    reconstruct(c.two_theta, s.z, cc.z, n.z, hvS, hvN);
    correct_w(BW, BE, cc.x, wW, wE);
    correct_w(BS, BN, cc.x, wS, wN);
    const float4 h = make_float4(wN - BN, wE - BE, wS - BS, wW - BW);
    float4 u, v;
    float q;
    q = div_by_h(h.x, c.epsilon); u.x = q * huN; v.x = q * hvN;
    q = div_by_h(h.y, c.epsilon); u.y = q * huE; v.y = q * hvE;
    q = div_by_h(h.z, c.epsilon); u.z = q * huS; v.z = q * hvS;
    q = div_by_h(h.w, c.epsilon); u.w = q * huW; v.w = q * hvW;
    H[i] = h; U[i] = u; V[i] = v;
    const float4 a1 = aux1[i];
    const float mid = fmaxf((h.x + h.y + h.z + h.w) / 4.0f, a1.x);
    float bw = a1.w;
    if (msd > c.dissipation_threshold) bw = 1.0f;
    aux2[i] = make_float4(mid, 0.f, msd, bw);
}

// ---- Pass2 (compute.hlsl:470-542): KP fluxes at east / north faces; region [1,nx+2)x[1,ny+2) --
__global__ void k_pass2(const float4* __restrict__ H, const float4* __restrict__ U, const float4* __restrict__ V,
                        const float4* __restrict__ aux2, float4* __restrict__ XF, float4* __restrict__ YF,
                        float4* __restrict__ aux1, SimConsts c, float dt) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (x >= c.nx + 2 || y >= c.ny + 2) return;
    const int NX = c.NX;
    const size_t i = size_t(y) * NX + x;
    const float4 hc = H[i], uc = U[i], vc = V[i];
    const float hN = hc.x, hE = hc.y, uN = uc.x, uE = uc.y, vN = vc.x, vE = vc.y;
    const float hWe = H[i + 1].w, hSn = H[i + NX].z;
    const float uWe = U[i + 1].w, uSn = U[i + NX].z;
    const float vWe = V[i + 1].w, vSn = V[i + NX].z;
    const float g = c.g, hg = c.half_g;
    const float cN = sqrtf(g * hN), cE = sqrtf(g * hE), cW = sqrtf(g * hWe), cS = sqrtf(g * hSn);
    const float ap = fmaxf(fmaxf(uE + cE, uWe + cW), 0.f);
    const float am = fminf(fminf(uE - cE, uWe - cW), 0.f);
    const float bp = fmaxf(fmaxf(vN + cN, vSn + cS), 0.f);
    const float bm = fminf(fminf(vN - cN, vSn - cS), 0.f);
    float4 xf, yf;
    xf.x = numflux(ap, am, hWe * uWe, hE * uE, hWe - hE);
    xf.y = numflux(ap, am, hWe * (uWe * uWe + hg * hWe), hE * (uE * uE + hg * hE), hWe * uWe - hE * uE);
    xf.z = numflux(ap, am, hWe * uWe * vWe, hE * uE * vE, hWe * vWe - hE * vE);
    xf.w = 0.f;
    yf.x = numflux(bp, bm, hSn * vSn, hN * vN, hSn - hN);
    yf.y = numflux(bp, bm, hSn * uSn * vSn, hN * uN * vN, hSn * uSn - hN * uN);
    yf.z = numflux(bp, bm, hSn * (vSn * vSn + hg * hSn), hN * (vN * vN + hg * hN), hSn * vSn - hN * vN);
    yf.w = 0.f;
    XF[i] = xf; YF[i] = yf;
    const float4 a2 = aux2[i];
    aux1[i] = make_float4(a2.x, 0.f, a2.z, a2.w * t_pow(fabsf(c.whitewater_decay_rate), dt));
}

struct Pass3Args {
    const float4* st; const float4* bot; const float4* XF; const float4* YF;
    const float4* ABCx; const float4* ABCy;
    const float4* og; const float4* oog; const float4* ofg; const float4* oofg;
    const float4* cur; const float4* pred; const float4* fgpred;
    float4* out; float4* sgrad; float4* sfg;
    float dt, dt_old, dt_old_old;
    int scheme;
};

// AdamsBashforthCoef (compute.hlsl:560-566)
__device__ __forceinline__ void ab_coef(float a, float b, float cc, float o[3]) {
    o[0] = (a / b) * ((2 * a + 6 * b + 3 * cc) / (b + cc)) + 6;
    o[1] = -(a / b) * ((2 * a + 3 * b + 3 * cc) / (cc));
    o[2] = (a / cc) * ((2 * a + 3 * b) / (b + cc));
}
// SecondOrderDerivatives (compute.hlsl:569-605)
__device__ __forceinline__ void second_order(float yn, float y1, float y2, float b, float cc, float o[3]) {
    float r = (2 * b + cc) / (b * (b + cc)), g = -(b + cc) / (b * cc), bb = (b) / (cc * (b + cc));
    o[0] = r * yn + g * y1 + bb * y2;
    r = (cc) / (b * (b + cc)); g = (b - cc) / (b * cc); bb = -(b) / (cc * (b + cc));
    o[1] = r * yn + g * y1 + bb * y2;
    r = -(cc) / (b * (b + cc)); g = (b + cc) / (b * cc); bb = -(b + 2 * cc) / (cc * (b + cc));
    o[2] = r * yn + g * y1 + bb * y2;
}

// ---- Pass3Predictor (compute.hlsl:616-812): RHS, time scheme; interior [2,nx+2)x[2,ny+2) -----
__global__ void k_pass3(Pass3Args a, SimConsts c) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + 2;
    if (x >= c.nx + 2 || y >= c.ny + 2) return;
    const int NX = c.NX;
    const size_t i = size_t(y) * NX + x;
    const float4* st = a.st;
    const float4* bot = a.bot;
    const float BYh = bot[i].x, BXh = bot[i].y, BAh = bot[i].z;
    const float BXw = bot[i - 1].y, BYs = bot[i - NX].x;
    const float4 cc = st[i], r = st[i + 1], l = st[i - 1], u = st[i + NX], d = st[i - NX];
    const float4 cx = a.ABCx[i], cy = a.ABCy[i];
    const float sl = c.sea_level;
    const float h = fmaxf(0.f, cc.x - BAh);
    const float dh = fmaxf(0.f, sl - BAh), d2 = dh * dh, d3 = d2 * dh;
    const float dl = fmaxf(0.f, sl - bot[i - 1].z), dr = fmaxf(0.f, sl - bot[i + 1].z);
    const float ddn = fmaxf(0.f, sl - bot[i - NX].z), du = fmaxf(0.f, sl - bot[i + NX].z);
    const float dll = fmaxf(0.f, sl - bot[i - 2].z), drr = fmaxf(0.f, sl - bot[i + 2].z);
    const float ddd = fmaxf(0.f, sl - bot[i - 2 * NX].z), duu = fmaxf(0.f, sl - bot[i + 2 * NX].z);
    const float e0 = cc.x - sl;
    const float el = l.x - sl, er = r.x - sl, ed = d.x - sl, eu = u.x - sl;
    const float ell = st[i - 2].x - sl, err = st[i + 2].x - sl;
    const float edd = st[i - 2 * NX].x - sl, euu = st[i + 2 * NX].x - sl;
    const float eul = st[i + NX - 1].x - sl, eur = st[i + NX + 1].x - sl;
    const float edl = st[i - NX - 1].x - sl, edr = st[i - NX + 1].x - sl;
    const float4 xh = a.XF[i], xw = a.XF[i - 1], yh = a.YF[i], ys = a.YF[i - NX];
    const float odx = c.one_over_dx, ody = c.one_over_dy;
    const float od2x = odx * odx, od3x = od2x * odx, od2y = ody * ody, od3y = od2y * ody;
    const float ddx = (-drr + 8 * dr - 8 * dl + dll) * odx / 12.0f;
    const float ddy = (-duu + 8 * du - 8 * ddn + ddd) * ody / 12.0f;
    const float exy = (0.25f * odx * ody * (eur - edr - eul + edl));
    const float exx = od2x * (er - 2 * e0 + el);
    const float eyy = od2y * (eu - 2 * e0 + ed);
    const float Bg = c.Bcoef_g;
    const float P1x = Bg * (d3) * ((err - 2 * er + 2 * el - ell) * (0.5f * od3x) +
                                   (eur - eul - 2 * er + 2 * el + edr - edl) * (0.5f * odx * od2y));
    const float P2x = Bg * (d2) * (ddx * (2 * exx + eyy) + ddy * exy);
    const float P1y = Bg * (d3) * ((euu - 2 * eu + 2 * ed - edd) * (0.5f * od3y) +
                                   (eur + eul - 2 * eu + 2 * ed - edr - edl) * (0.5f * ody * od2x));
    const float P2y = Bg * (d2) * (ddy * (exx + 2 * eyy) + ddx * exy);
    const float fr = friction_calc(cc.y, cc.z, h, c.friction, c.is_manning, c.g, c.epsilon);
    const float s1 = -c.g_over_dx * h * (BXh - BXw) - cc.y * fr + (P1x + P2x);
    const float s2 = -c.g_over_dy * h * (BYh - BYs) - cc.z * fr + (P1y + P2y);
    const float f0 = (xw.x - xh.x) * odx + (ys.x - yh.x) * ody + 0.f;
    const float f1 = (xw.y - xh.y) * odx + (ys.y - yh.y) * ody + s1;
    const float f2 = (xw.z - xh.z) * odx + (ys.z - yh.z) * ody + s2;
    const float sixth = 1.0f / 6.0f;
    const float Fs = (sixth * dh * (ddx * ((ody / 2.0f) * (u.z - d.z)) + (ddy * ((odx / 2.0f) * (r.z - l.z)))));
    const float Gs = (sixth * dh * (ddx * ((ody / 2.0f) * (u.y - d.y)) + (ddy * ((odx / 2.0f) * (r.y - l.y)))));
    const float dt = a.dt;
    float wO = 0.f, huO = 0.f, hvO = 0.f;
    if (a.scheme == CEL_SCHEME_EULER) {
        wO = cc.x + dt * f0;
        huO = cx.x * l.y + cx.y * cc.y + cx.z * r.y + dt * f1;
        hvO = cy.x * d.z + cy.y * cc.z + cy.z * u.z + dt * f2;
    } else {
        const float4 o = a.og[i], oo = a.oog[i], fo = a.ofg[i], foo = a.oofg[i];
        if (a.scheme == CEL_SCHEME_PREDICTOR) {
            wO = cc.x + dt / 12.0f * (23.0f * f0 - 16.0f * o.x + 5.0f * oo.x);
            huO = cx.x * l.y + cx.y * cc.y + cx.z * r.y + dt / 12.0f * (23.0f * f1 - 16.0f * o.y + 5.0f * oo.y) +
                  (2.0f * Fs - 3.0f * fo.x + foo.x);
            hvO = cy.x * d.z + cy.y * cc.z + cy.z * u.z + dt / 12.0f * (23.0f * f2 - 16.0f * o.z + 5.0f * oo.z) +
                  (2.0f * Gs - 3.0f * fo.y + foo.y);
        } else if (a.scheme == CEL_SCHEME_PREDICTOR_ADAPTIVE) {
            float cf[3], dF[3], dG[3];
            ab_coef(dt, a.dt_old, a.dt_old_old, cf);
            second_order(Fs, fo.x, foo.x, a.dt_old, a.dt_old_old, dF);
            second_order(Gs, fo.y, foo.y, a.dt_old, a.dt_old_old, dG);
            wO = cc.x + dt / 6.0f * (cf[0] * f0 + cf[1] * o.x + cf[2] * oo.x);
            huO = cx.x * l.y + cx.y * cc.y + cx.z * r.y + dt / 6.0f * (cf[0] * f1 + cf[1] * o.y + cf[2] * oo.y) +
                  dt / 6.0f * (cf[0] * dF[0] + cf[1] * dF[1] + cf[2] * dF[2]);
            hvO = cy.x * d.z + cy.y * cc.z + cy.z * u.z + dt / 6.0f * (cf[0] * f2 + cf[1] * o.z + cf[2] * oo.z) +
                  dt / 6.0f * (cf[0] * dG[0] + cf[1] * dG[1] + cf[2] * dG[2]);
        } else {  // corrector
            const float4 qc = a.cur[i], qr = a.cur[i + 1], ql = a.cur[i - 1], qu = a.cur[i + NX], qd = a.cur[i - NX];
            const float4 pr = a.pred[i], fp = a.fgpred[i];
            wO = qc.x + dt / 24.0f * (9 * f0 + 19 * pr.x - 5 * o.x + 1 * oo.x);
            huO = cx.x * ql.y + cx.y * qc.y + cx.z * qr.y + dt / 24.0f * (9 * f1 + 19 * pr.y - 5 * o.y + 1 * oo.y) + Fs -
                  fp.x;
            hvO = cy.x * qd.z + cy.y * qc.z + cy.z * qu.z + dt / 24.0f * (9 * f2 + 19 * pr.z - 5 * o.z + 1 * oo.z) + Gs -
                  fp.y;
        }
    }
    a.out[i] = make_float4(wO, huO, hvO, 0.f);
    a.sgrad[i] = make_float4(f0, f1, f2, 0.f);
    a.sfg[i] = make_float4(Fs, Gs, 0.f, 0.f);
}

// ---- Cyclic reduction, one level per launch (compute.hlsl:835-947) ------------------------
// D arrays: element (x, y) at base[y*pitch + x*stride] (the level-0 RHS is a channel of the
// float4 state; reduced levels are plain float planes).
__global__ void k_cr_reduce_x(const float* __restrict__ Dp, int dps, int dpp, const float4* __restrict__ Ap, int app,
                              float* __restrict__ Dk, int dkp, int len_k, int ny) {
    const int x2 = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + 2;
    if (x2 >= len_k + 2 || y >= ny + 2) return;
    const int x1 = (x2 - 2) * 2 + 3;
    const float* row = Dp + size_t(y) * dpp;
    const float4* ar = Ap + size_t(y) * app;
    const float k1 = ar[x1].x / ar[x1 - 1].y, k2 = ar[x1].z / ar[x1 + 1].y;
    Dk[size_t(y) * dkp + x2] = row[x1 * dps] - row[(x1 - 1) * dps] * k1 - row[(x1 + 1) * dps] * k2;
}

__global__ void k_cr_subst_x(const float* __restrict__ Dk, int dks, int dkp, const float4* __restrict__ Ak, int akp,
                             const float* __restrict__ Xn, int xnp, float* __restrict__ Xk, int xkp, int len_k, int ny) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + 2;
    if (x >= len_k + 2 || y >= ny + 2) return;
    float o;
    const float* xn = Xn ? Xn + size_t(y) * xnp : nullptr;
    if (x % 2 == 1) {
        o = xn ? xn[x / 2 + 1] : 0.f;
    } else {
        const float4 a = Ak[size_t(y) * akp + x];
        const float x1 = xn ? xn[x / 2] : 0.f, x2 = xn ? xn[x / 2 + 1] : 0.f;
        o = (Dk[size_t(y) * dkp + size_t(x) * dks] - a.x * x1 - a.z * x2) / a.y;
    }
    Xk[size_t(y) * xkp + x] = o;
}

__global__ void k_cr_reduce_y(const float* __restrict__ Dp, int dps, int dpp, const float4* __restrict__ Ap, int NX,
                              float* __restrict__ Dk, int len_k, int nx) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int y2 = blockIdx.y * blockDim.y + threadIdx.y + 2;
    if (x >= nx + 2 || y2 >= len_k + 2) return;
    const int y1 = (y2 - 2) * 2 + 3;
    const float4 a0 = Ap[size_t(y1) * NX + x];
    const float k1 = a0.x / Ap[size_t(y1 - 1) * NX + x].y, k2 = a0.z / Ap[size_t(y1 + 1) * NX + x].y;
    const float dIn = Dp[size_t(y1) * dpp + size_t(x) * dps];
    const float dL = Dp[size_t(y1 - 1) * dpp + size_t(x) * dps];
    const float dR = Dp[size_t(y1 + 1) * dpp + size_t(x) * dps];
    Dk[size_t(y2) * NX + x] = dIn - dL * k1 - dR * k2;
}

__global__ void k_cr_subst_y(const float* __restrict__ Dk, int dks, int dkp, const float4* __restrict__ Ak, int NX,
                             const float* __restrict__ Xn, float* __restrict__ Xk, int len_k, int nx) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + 2;
    if (x >= nx + 2 || y >= len_k + 2) return;
    float o;
    if (y % 2 == 1) {
        o = Xn ? Xn[size_t(y / 2 + 1) * NX + x] : 0.f;
    } else {
        const float4 a = Ak[size_t(y) * NX + x];
        const float x1 = Xn ? Xn[size_t(y / 2) * NX + x] : 0.f, x2 = Xn ? Xn[size_t(y / 2 + 1) * NX + x] : 0.f;
        o = (Dk[size_t(y) * dkp + size_t(x) * dks] - a.x * x1 - a.z * x2) / a.y;
    }
    Xk[size_t(y) * NX + x] = o;
}

// CopyFromXxAndXy (compute.hlsl:814-823) over the interior
__global__ void k_copy_from(float4* __restrict__ st, const float* __restrict__ Xx, const float* __restrict__ Xy,
                            SimConsts c) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 2;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + 2;
    if (x >= c.nx + 2 || y >= c.ny + 2) return;
    const size_t i = size_t(y) * c.NX + x;
    float4 s = st[i];
    s.y = Xx[i];
    s.z = Xy[i];
    s.w = 0.f;
    st[i] = s;
}

// ---- Boundaries (compute.hlsl:985-1309) --------------------------------------------------
struct BArgs {
    int side;  // 0 = N, 1 = E, 2 = S, 3 = W
    int type, width;
    float sea_level, amp, period, theta;
    float uts_eta, uts_hu, uts_hv;
    int n_waves, nleaf;
    const float4* waves;
    float t, dt;
    int x0, y0, sw, sh;
};

// Pairwise tree sum of the irregular-wave components over 2^(K-1) leaves
// (ColumnSumReduce / RowSumReduce, compute.hlsl:1196-1212): a binary-counter stack gives the
// balanced-tree association; runs of constant components (sea level, 0, 0) are pushed as whole
// aligned subtrees.
__device__ float3 irregular_sum(const BArgs& b, float xx, float yy, float dh, float g) {
    float3 stk[17];
    int sz[17];
    int top = 0;
    const bool wet = dh > CEL_MIN_DEPTH;
    const int nreal = wet ? min(b.n_waves, b.nleaf) : 0;
    int m = 0;
    while (m < b.nleaf) {
        float3 v;
        int s;
        if (m < nreal) {
            float e, hu, hv;
            const float4 wv = b.waves[m];
            sine_wave(xx, yy, b.t, dh, wv.x, wv.y, wv.z, wv.w, g, e, hu, hv);
            v = make_float3(e + b.sea_level, hu, hv);
            s = 1;
        } else {
            s = (m == 0) ? b.nleaf : (m & -m);
            while (m + s > b.nleaf) s >>= 1;
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

__global__ void k_boundary(const float4* __restrict__ st, const float4* __restrict__ bot, float4* __restrict__ strip,
                           BArgs b, SimConsts c) {
    const int sx = blockIdx.x * blockDim.x + threadIdx.x;
    const int sy = blockIdx.y * blockDim.y + threadIdx.y;
    if (sx >= b.sw || sy >= b.sh) return;
    const int x = b.x0 + sx, y = b.y0 + sy;
    const int NX = c.NX, NY = c.NY;
    const size_t i = size_t(y) * NX + x;
    float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
    const float sl = b.sea_level;
    if (b.type == CEL_BC_SOLID) {
        int qx, qy;
        solid_source(b.side, x, y, c.nx, c.ny, qx, qy);
        float4 s = make_float4(0.f, 0.f, 0.f, 0.f);  // out-of-range texture loads read zero
        if (qx >= 0 && qy >= 0 && qx < NX && qy < NY) s = st[size_t(qy) * NX + qx];
        o.x = s.x;
        o.y = (b.side == 1 || b.side == 3) ? -s.y : s.y;
        o.z = (b.side == 0 || b.side == 2) ? -s.z : s.z;
    } else if (b.type == CEL_BC_SPONGE) {
        const float dh = fmaxf(CEL_MIN_DEPTH, sl - bot[i].z);
        float L, dist;
        if (b.side == 3) { L = float(b.width) * c.dx; dist = float(x) * c.dx; }
        else if (b.side == 1) { L = float(b.width) * c.dx; dist = float(NX - x) * c.dx; }
        else if (b.side == 2) { L = float(b.width) * c.dy; dist = float(y) * c.dy; }
        else { L = float(b.width) * c.dy; dist = float(NY - y) * c.dy; }
        const float gam = sponge_fn(L, dist) / sponge_fn(L, dist + sqrtf(c.g * dh) * b.dt);
        const float4 s = st[i];
        o.x = gam * (s.x - sl) + sl;
        o.y = gam * s.y;
        o.z = gam * s.z;
    } else if (b.type == CEL_BC_SINEWAVE) {
        const float dh = fmaxf(0.f, sl - bot[i].z);
        const float xx = (b.side == 1) ? float(x - NX) * c.dx : float(x) * c.dx;
        const float yy = (b.side == 0) ? float(y - NY) * c.dy : float(y) * c.dy;
        float e = 0.f, hu = 0.f, hv = 0.f;
        if (dh > CEL_MIN_DEPTH) sine_wave(xx, yy, b.t, dh, b.amp, b.period, b.theta, 0.f, c.g, e, hu, hv);
        o.x = e + sl; o.y = hu; o.z = hv;
    } else if (b.type == CEL_BC_UTS) {
        o.x = b.uts_eta + sl; o.y = b.uts_hu; o.z = b.uts_hv;
    } else {  // irregular waves: one component per texel along the side, tree-summed
        const bool colwise = (b.side == 1 || b.side == 3);
        const int along = colwise ? y : x;
        const int lim = colwise ? c.ny : c.nx;
        if (along >= 2 && along < lim + 2) {
            const float dh = fmaxf(0.f, sl - bot[i].z);
            const float xx = (b.side == 1) ? float(x - NX) * c.dx : float(x) * c.dx;
            const float yy = (b.side == 0) ? float(y - NY) * c.dy : float(y) * c.dy;
            const float3 r = irregular_sum(b, xx, yy, dh, c.g);
            o.x = r.x; o.y = r.y; o.z = r.z;
        }
    }
    strip[size_t(sy) * b.sw + sx] = o;
}

__global__ void k_strip_copy(float4* __restrict__ st, const float4* __restrict__ strip, int x0, int y0, int sw, int sh,
                             int NX) {
    const int sx = blockIdx.x * blockDim.x + threadIdx.x;
    const int sy = blockIdx.y * blockDim.y + threadIdx.y;
    if (sx >= sw || sy >= sh) return;
    st[size_t(y0 + sy) * NX + x0 + sx] = strip[size_t(sy) * sw + sx];
}

// ---- GetStats (compute.hlsl:1319-1378) per 4x4 block, then an FP64 reduction -------------
__global__ void k_getstats(const float4* __restrict__ st, const float4* __restrict__ bot, float* __restrict__ blocks,
                           SimConsts c) {
    const int bx = blockIdx.x * blockDim.x + threadIdx.x;
    const int by = blockIdx.y * blockDim.y + threadIdx.y;
    const int nbx = c.nx / 4, nby = c.ny / 4;
    if (bx >= nbx || by >= nby) return;
    float sh = 0, sb = 0, shu = 0, shv = 0, sk = 0, mu = 0, mh = 0, mc = 0, mf = 0;
    for (int j = 2; j < 6; ++j)
        for (int ii = 2; ii < 6; ++ii) {
            const size_t i = size_t(by * 4 + j) * c.NX + bx * 4 + ii;
            const float4 s = st[i];
            const float B = bot[i].z;
            const float h = fmaxf(0.f, s.x - B);
            const float cc = sqrtf(c.g * h);
            const float q = div_by_h(h, c.epsilon);
            const float u = q * s.y, v = q * s.z;
            sh += h; sb += h * (B + 0.5f * h); shu += s.y; shv += s.z;
            sk += (s.y * u + s.z * v);
            const float u2v2 = u * u + v * v;
            mu = fmaxf(mu, u2v2); mh = fmaxf(mh, h);
            mc = fmaxf(mc, (fabsf(u) + cc) * c.one_over_dx);
            mc = fmaxf(mc, (fabsf(v) + cc) * c.one_over_dy);
            mf = fmaxf(mf, u2v2 * q);
        }
    float* o = blocks + (size_t(by) * nbx + bx) * 9;
    o[0] = sh; o[1] = sb; o[2] = shu; o[3] = shv; o[4] = sk; o[5] = mu; o[6] = mh; o[7] = mc; o[8] = mf;
}

// One CTA: FP64 sums / maxima of the block partials, plus the FP64 sum of h over every interior
// cell (out[9]).  out[10] = 1 if any state value is non-finite (health flag).
__global__ void k_reduce_stats(const float* __restrict__ blocks, int nb, const float4* __restrict__ st,
                               const float4* __restrict__ bot, SimConsts c, double* __restrict__ out) {
    __shared__ double sm[10][32];
    __shared__ int bad_s;
    double v[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    int bad = 0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        const float* b = blocks + size_t(k) * 9;
        for (int q = 0; q < 5; ++q) v[q] += double(b[q]);
        for (int q = 5; q < 9; ++q) v[q] = fmax(v[q], double(b[q]));
    }
    const int n = c.nx * c.ny;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int x = k % c.nx + 2, y = k / c.nx + 2;
        const size_t i = size_t(y) * c.NX + x;
        const float4 s = st[i];
        if (!isfinite(s.x) || !isfinite(s.y) || !isfinite(s.z)) bad = 1;
        v[9] += fmax(0.0, double(s.x) - double(bot[i].z));
    }
    if (threadIdx.x == 0) bad_s = 0;
    __syncthreads();
    if (bad) bad_s = 1;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int q = 0; q < 10; ++q) {
        double x = v[q];
        for (int off = 16; off; off >>= 1) {
            const double y = __shfl_down_sync(0xffffffffu, x, off);
            x = (q >= 5 && q < 9) ? fmax(x, y) : x + y;
        }
        if (lane == 0) sm[q][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = blockDim.x >> 5;
        for (int q = 0; q < 10; ++q) {
            double x = lane < nw ? sm[q][lane] : 0.0;
            for (int off = 16; off; off >>= 1) {
                const double y = __shfl_down_sync(0xffffffffu, x, off);
                x = (q >= 5 && q < 9) ? fmax(x, y) : x + y;
            }
            if (lane == 0) out[q] = x;
        }
        if (lane == 0) out[10] = bad_s ? 1.0 : 0.0;
    }
}

// AddSolitaryWave (compute.hlsl:949-976) over [1,nx+3)x[1,ny+3), reading a copy of the state
__global__ void k_add_solitary(const float4* __restrict__ copy, const float4* __restrict__ bot, float4* __restrict__ st,
                               SimConsts c, float H, float th, float xc, float yc) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (x >= c.nx + 3 || y >= c.ny + 3) return;
    const size_t i = size_t(y) * c.NX + x;
    const float4 s = copy[i];
    const float depth = fmaxf(s.x - bot[i].z, 0.f);
    const float K = sqrtf(0.75f * fabsf(H) / t_pow(depth, 3.0f));
    const float C = sqrtf(c.g * (H + depth));
    const float ch = t_cosh(K * ((float(x) * c.dx - xc) * t_cos(th) + (float(y) * c.dy - yc) * t_sin(th)));
    const float e = H * 1.0f / t_pow(ch, 2.0f);
    st[i] = make_float4(s.x + e, s.y + C * t_cos(th) * e, s.z + C * t_sin(th) * e, 0.f);
}

// ---------------------------------------------------------------------------------------------
class PlainEngine : public EngineIface {
public:
    cel_params p{};
    HostSetup hs;
    SimConsts c{};
    Scheme sch;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    KernelTimer tm;
    size_t ntex = 0;
    // device textures
    float4 *st[2] = {nullptr, nullptr}, *H = nullptr, *U = nullptr, *V = nullptr, *XF = nullptr, *YF = nullptr;
    float4 *AUX1 = nullptr, *AUX2 = nullptr, *CUR = nullptr, *PRED = nullptr, *FGPRED = nullptr, *BOT = nullptr;
    float4 *GRAD[3] = {nullptr, nullptr, nullptr}, *FG[3] = {nullptr, nullptr, nullptr}, *STRIP = nullptr;
    float4* WAVES = nullptr;
    std::vector<float4*> ABCx, ABCy;
    std::vector<float*> Dx, Xx, Dy, Xy;
    float* blocks = nullptr;
    double* dstats = nullptr;
    std::vector<void*> allocs;
    int wave_off[4] = {0, 0, 0, 0};
    int sim_idx = 0, old_i = 0, oldold_i = 1, scratch_i = 2;
    int uts_iter[4] = {1, 1, 1, 1};
    bool bootstrap_needed = true;
    std::vector<float> terrain;   // bathymetry grid given by set_bathymetry (used by remesh)
    int terrain_nx = 0, terrain_ny = 0;
    // stats bookkeeping for the latest device-side GetStats
    int last_stats_scheme = 0;
    float last_stats_dt = 0, last_stats_time = 0;

    ~PlainEngine() override {
        for (void* a : allocs) cudaFree(a);
        for (cel_boundary* b : {&p.west, &p.east, &p.south, &p.north})
            if (b->uts) std::free(b->uts);
        if (own_stream && stream) cudaStreamDestroy(stream);
        (void)cudaGetLastError();   // teardown has no caller to report to; leave no stale error behind
    }

    template <typename T>
    int dalloc(T*& ptr, size_t count) {
        void* q = nullptr;
        CEL_CUDA_TRY(cudaMalloc(&q, count * sizeof(T)));
        CEL_CUDA_TRY(cudaMemset(q, 0, count * sizeof(T)));
        allocs.push_back(q);
        ptr = static_cast<T*>(q);
        return CEL_OK;
    }

    int init(const cel_params& prm, const float* bathy, int bnx, int bny) {
        p = prm;
        for (cel_boundary* b : {&p.west, &p.east, &p.south, &p.north})
            if (b->type != CEL_BC_UTS) { b->uts = nullptr; b->n_uts = 0; }
        if (int st = log_validate(p.log, p.nx, p.ny, err)) return st;
        int st0 = make_setup(p, bathy, bnx, bny, hs, err);
        if (st0) return st0;
        int dev = 0;
        CEL_CUDA_TRY(cudaGetDevice(&dev));
        CEL_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        own_stream = true;
        c = make_consts(p, hs, hs.NX);
        ntex = size_t(hs.NX) * hs.NY;
        for (float4** t : {&st[0], &st[1], &H, &U, &V, &XF, &YF, &AUX1, &AUX2, &CUR, &PRED, &FGPRED, &BOT, &STRIP})
            if (int e = dalloc(*t, ntex)) return e;
        for (int k = 0; k < 3; ++k) {
            if (int e = dalloc(GRAD[k], ntex)) return e;
            if (int e = dalloc(FG[k], ntex)) return e;
        }
        ABCx.assign(hs.Kx, nullptr); Dx.assign(hs.Kx, nullptr); Xx.assign(hs.Kx, nullptr);
        ABCy.assign(hs.Ky, nullptr); Dy.assign(hs.Ky, nullptr); Xy.assign(hs.Ky, nullptr);
        for (int k = 0; k < hs.Kx; ++k) {
            const size_t n = size_t(hs.lenx[k] + 4) * hs.NY;
            if (int e = dalloc(ABCx[k], n)) return e;
            if (int e = dalloc(Dx[k], n)) return e;
            if (int e = dalloc(Xx[k], k == 0 ? ntex : n)) return e;
            CEL_CUDA_TRY(cudaMemcpy(ABCx[k], hs.ABCx[k].data(), n * sizeof(float4), cudaMemcpyHostToDevice));
        }
        for (int k = 0; k < hs.Ky; ++k) {
            const size_t n = size_t(hs.NX) * (hs.leny[k] + 4);
            if (int e = dalloc(ABCy[k], n)) return e;
            if (int e = dalloc(Dy[k], n)) return e;
            if (int e = dalloc(Xy[k], k == 0 ? ntex : n)) return e;
            CEL_CUDA_TRY(cudaMemcpy(ABCy[k], hs.ABCy[k].data(), n * sizeof(float4), cudaMemcpyHostToDevice));
        }
        {
            std::vector<float4> b(ntex);
            for (size_t i = 0; i < ntex; ++i) b[i] = make_float4(hs.BY[i], hs.BX[i], hs.BA[i], 0.f);
            CEL_CUDA_TRY(cudaMemcpy(BOT, b.data(), ntex * sizeof(float4), cudaMemcpyHostToDevice));
        }
        {   // irregular-wave component table: sides N, E, S, W back to back
            std::vector<float4> wv;
            const cel_boundary* sides[4] = {&p.north, &p.east, &p.south, &p.west};
            for (int s = 0; s < 4; ++s) {
                wave_off[s] = int(wv.size());
                if (sides[s]->type == CEL_BC_IRREGULAR)
                    for (int k = 0; k < sides[s]->n_waves; ++k)
                        wv.push_back(make_float4(float(sides[s]->waves[k][0]), float(sides[s]->waves[k][1]),
                                                 float(sides[s]->waves[k][2]), float(sides[s]->waves[k][3])));
            }
            if (wv.empty()) wv.push_back(make_float4(0, 0, 0, 0));
            if (int e = dalloc(WAVES, wv.size())) return e;
            CEL_CUDA_TRY(cudaMemcpy(WAVES, wv.data(), wv.size() * sizeof(float4), cudaMemcpyHostToDevice));
            // UTS tables stay on the host (timeSeriesHelper interpolates on the host)
            for (cel_boundary* b : {&p.west, &p.east, &p.south, &p.north}) {
                if (b->type == CEL_BC_UTS && b->n_uts > 0) {
                    double* copy = static_cast<double*>(std::malloc(sizeof(double) * 4 * b->n_uts));
                    std::memcpy(copy, b->uts, sizeof(double) * 4 * b->n_uts);
                    b->uts = copy;
                }
            }
        }
        const int nb = std::max(1, (hs.nx / 4) * (hs.ny / 4));
        if (int e = dalloc(blocks, size_t(nb) * 9)) return e;
        if (int e = dalloc(dstats, 16)) return e;
        // the set-up copies and memsets above ran on the legacy stream, which the engine's
        // non-blocking stream does not wait for: finish them
        CEL_CUDA_TRY(cudaDeviceSynchronize());
        return remesh();
    }

    int remesh() override {
        if (!terrain.empty()) {   // the bathymetry changed since creation: rebuild from the new grid
            HostSetup fresh;
            if (int st0 = make_setup(p, terrain.data(), terrain_nx, terrain_ny, fresh, err)) return st0;
            hs = fresh;
            // on the engine's stream, finished before the host copies go out of scope
            for (int k = 0; k < hs.Kx; ++k)
                CEL_CUDA_TRY(cudaMemcpyAsync(ABCx[k], hs.ABCx[k].data(), size_t(hs.lenx[k] + 4) * hs.NY * sizeof(float4),
                                             cudaMemcpyHostToDevice, stream));
            for (int k = 0; k < hs.Ky; ++k)
                CEL_CUDA_TRY(cudaMemcpyAsync(ABCy[k], hs.ABCy[k].data(), size_t(hs.NX) * (hs.leny[k] + 4) * sizeof(float4),
                                             cudaMemcpyHostToDevice, stream));
            std::vector<float4> b(ntex);
            for (size_t i = 0; i < ntex; ++i) b[i] = make_float4(hs.BY[i], hs.BX[i], hs.BA[i], 0.f);
            CEL_CUDA_TRY(cudaMemcpyAsync(BOT, b.data(), ntex * sizeof(float4), cudaMemcpyHostToDevice, stream));
            CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        }
        std::vector<float4> s(ntex);
        for (size_t i = 0; i < ntex; ++i) s[i] = make_float4(hs.ic[3 * i], hs.ic[3 * i + 1], hs.ic[3 * i + 2], 0.f);
        CEL_CUDA_TRY(cudaMemcpyAsync(st[0], s.data(), ntex * sizeof(float4), cudaMemcpyHostToDevice, stream));
        CEL_CUDA_TRY(cudaMemcpyAsync(st[1], s.data(), ntex * sizeof(float4), cudaMemcpyHostToDevice, stream));
        for (float4* t : {H, U, V, XF, YF, AUX1, AUX2, CUR, PRED, FGPRED, GRAD[0], GRAD[1], GRAD[2], FG[0], FG[1], FG[2]})
            CEL_CUDA_TRY(cudaMemsetAsync(t, 0, ntex * sizeof(float4), stream));
        CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        sch.reset(p);
        sim_idx = 0; old_i = 0; oldold_i = 1; scratch_i = 2;
        for (int& u : uts_iter) u = 1;
        bootstrap_needed = true;
        return CEL_OK;
    }

    void uts_value(const cel_boundary& b, int side, float t, float out[3]) {
        // timeSeriesHelper (engine.cpp:1882-1904), with float arithmetic
        out[0] = out[1] = out[2] = 0.f;
        const int n = b.n_uts;
        int& it = uts_iter[side];
        while (it < n && float(b.uts[4 * it]) < t) ++it;
        if (it >= n) return;
        const float t0 = float(b.uts[4 * (it - 1)]), t1 = float(b.uts[4 * it]);
        const float m = (t - t0) / (t1 - t0);
        for (int q = 0; q < 3; ++q) {
            const float v0 = float(b.uts[4 * (it - 1) + q + 1]), v1 = float(b.uts[4 * it + q + 1]);
            out[q] = v0 + (v1 - v0) * m;
        }
    }

    int boundary_side(float4* stt, int side) {
        const cel_boundary& b = side == 0 ? p.north : side == 1 ? p.east : side == 2 ? p.south : p.west;
        const int NX = hs.NX, NY = hs.NY;
        int x0, x1, y0, y1;
        if (side == 0) { x0 = 0; x1 = NX; y0 = NY - b.width; y1 = NY; }
        else if (side == 1) { x0 = NX - b.width; x1 = NX; y0 = 0; y1 = NY; }
        else if (side == 2) { x0 = 0; x1 = NX; y0 = 0; y1 = b.width; }
        else { x0 = 0; x1 = b.width; y0 = 0; y1 = NY; }
        x0 = std::max(x0, 0); y0 = std::max(y0, 0); x1 = std::min(x1, NX); y1 = std::min(y1, NY);
        if (x1 <= x0 || y1 <= y0) return CEL_OK;
        BArgs a{};
        a.side = side; a.type = b.type; a.width = b.width;
        a.sea_level = float(b.sea_level); a.amp = float(b.amplitude); a.period = float(b.period);
        a.theta = float(b.theta);
        a.n_waves = b.type == CEL_BC_IRREGULAR ? b.n_waves : 0;
        const int Kn = (side == 0 || side == 2) ? hs.Ky : hs.Kx;
        a.nleaf = 1 << (Kn - 1);
        a.waves = WAVES + wave_off[side];
        a.t = sch.total_time;
        a.dt = sch.dt;
        if (b.type == CEL_BC_UTS) {
            float v[3];
            uts_value(b, side, sch.total_time, v);
            a.uts_eta = v[0]; a.uts_hu = v[1]; a.uts_hv = v[2];
        }
        a.x0 = x0; a.y0 = y0; a.sw = x1 - x0; a.sh = y1 - y0;
        {
            TimedLaunch tl(&tm, stream, "plain_boundary");
            k_boundary<<<grid2(a.sw, a.sh), dim3(BX2, BY2), 0, stream>>>(stt, BOT, STRIP, a, c);
        }
        {
            TimedLaunch tl(&tm, stream, "plain_strip_copy");
            k_strip_copy<<<grid2(a.sw, a.sh), dim3(BX2, BY2), 0, stream>>>(stt, STRIP, x0, y0, a.sw, a.sh, NX);
        }
        return CEL_OK;
    }

    int run_stats_kernels() {
        (void)cudaGetLastError();
        const float4* s = st[sim_idx];
        const int nbx = hs.nx / 4, nby = hs.ny / 4;
        if (nbx > 0 && nby > 0) {
            TimedLaunch tl(&tm, stream, "plain_getstats");
            k_getstats<<<grid2(nbx, nby), dim3(BX2, BY2), 0, stream>>>(s, BOT, blocks, c);
        }
        {
            TimedLaunch tl(&tm, stream, "plain_reduce_stats");
            k_reduce_stats<<<1, 1024, 0, stream>>>(blocks, nbx * nby, s, BOT, c, dstats);
        }
        CEL_CUDA_TRY(cudaGetLastError());
        return CEL_OK;
    }

    void finish_stats(const double* v, float cfl_used, cel_stats* o) {
        const double DENSITY = 1000;
        const double AREA = double(float(p.width) / float(hs.nx - 1) * float(p.length) / float(hs.ny - 1));
        const double g = double(c.g);
        o->mass = v[0] * DENSITY * AREA;
        o->potential_energy = v[1] * g * DENSITY * AREA;
        o->x_momentum = v[2] * DENSITY * AREA;
        o->y_momentum = v[3] * DENSITY * AREA;
        o->kinetic_energy = v[4] * 0.5 * DENSITY * AREA;
        o->total_energy = o->kinetic_energy + o->potential_energy;
        o->max_speed = std::sqrt(v[5]);
        o->max_depth = v[6];
        o->max_froude = std::sqrt(v[8] / g);
        o->cfl_rate = double(cfl_used);
        o->mass_full = v[9];
        o->health = v[10] != 0 ? CEL_ERR_NUMERIC : 0;
    }

    // resetTimestep: GetStats on the current state, then dt (engine.cpp:1536-1756)
    int reset_timestep(float, float, cel_stats* out) override {
        if (int e = run_stats_kernels()) return e;
        double v[16];
        CEL_CUDA_TRY(cudaMemcpyAsync(v, dstats, sizeof(double) * 11, cudaMemcpyDeviceToHost, stream));
        CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        const float cfl = sch.choose_dt(float(v[7]));
        if (out) {
            finish_stats(v, cfl, out);
            out->cfl_number = double(cfl * sch.dt);
            out->timestep = double(sch.dt);
            out->total_time = double(sch.total_time);
            out->time_scheme = sch.time_scheme;
        }
        last_stats_scheme = sch.time_scheme;
        last_stats_dt = sch.dt;
        last_stats_time = sch.total_time;
        return CEL_OK;
    }

    // resetTimestep without a host readback (fixed dt); adaptive dt needs the CFL on the host.
    int reset_timestep_device() {
        if (sch.adaptive) return reset_timestep(0.f, 0.f, nullptr);
        if (int e = run_stats_kernels()) return e;
        sch.choose_dt(0.f);
        last_stats_scheme = sch.time_scheme;
        last_stats_dt = sch.dt;
        last_stats_time = sch.total_time;
        return CEL_OK;
    }

    int get_stats(cel_stats* out) override {
        double v[16];
        CEL_CUDA_TRY(cudaMemcpyAsync(v, dstats, sizeof(double) * 11, cudaMemcpyDeviceToHost, stream));
        CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        finish_stats(v, float(v[7]), out);
        out->cfl_number = v[7] * double(last_stats_dt);
        out->timestep = double(last_stats_dt);
        out->total_time = double(last_stats_time);
        out->time_scheme = last_stats_scheme;
        return CEL_OK;
    }

    // timestep() (engine.cpp:849-1522): one pass
    int timestep() override {
        (void)cudaGetLastError();   // the launch checks below must see only this pass's launches
        if (!sch.initialized) { if (int e = reset_timestep(0.f, 0.f, nullptr)) return e; }
        const dim3 blk(BX2, BY2);
        float4* old_state = st[sim_idx];
        float4* new_state = st[1 - sim_idx];
        if (bootstrap_needed) {
            TimedLaunch tl(&tm, stream, "plain_pass1");
            k_pass1<<<grid2(hs.nx + 2, hs.ny + 2), blk, 0, stream>>>(old_state, BOT, AUX1, H, U, V, AUX2, c);
            bootstrap_needed = false;
        }
        CEL_CUDA_TRY(cudaMemsetAsync(XF, 0, ntex * sizeof(float4), stream));
        CEL_CUDA_TRY(cudaMemsetAsync(YF, 0, ntex * sizeof(float4), stream));
        {
            TimedLaunch tl(&tm, stream, "plain_pass2");
            k_pass2<<<grid2(hs.nx + 1, hs.ny + 1), blk, 0, stream>>>(H, U, V, AUX2, XF, YF, AUX1, c, sch.dt);
        }
        CEL_CUDA_TRY(cudaMemsetAsync(new_state, 0, ntex * sizeof(float4), stream));
        Pass3Args a{};
        a.st = old_state; a.bot = BOT; a.XF = XF; a.YF = YF; a.ABCx = ABCx[0]; a.ABCy = ABCy[0];
        a.og = GRAD[old_i]; a.oog = GRAD[oldold_i]; a.ofg = FG[old_i]; a.oofg = FG[oldold_i];
        a.cur = CUR; a.pred = PRED; a.fgpred = FGPRED;
        a.out = new_state; a.sgrad = GRAD[scratch_i]; a.sfg = FG[scratch_i];
        a.dt = sch.dt; a.dt_old = sch.dt_old; a.dt_old_old = sch.dt_old_old;
        a.scheme = sch.time_scheme;
        {
            TimedLaunch tl(&tm, stream, "plain_pass3");
            k_pass3<<<grid2(hs.nx, hs.ny), blk, 0, stream>>>(a, c);
        }
        if (sch.is_predictor()) {  // engine.cpp:1050-1058
            CEL_CUDA_TRY(cudaMemcpyAsync(PRED, GRAD[scratch_i], ntex * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
            CEL_CUDA_TRY(cudaMemcpyAsync(FGPRED, FG[scratch_i], ntex * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
            CEL_CUDA_TRY(cudaMemcpyAsync(CUR, old_state, ntex * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
        }
        // cyclic reduction in x then y, then back substitution (engine.cpp:1060-1217)
        const float* rhs_x = reinterpret_cast<const float*>(new_state) + 1;
        const float* rhs_y = reinterpret_cast<const float*>(new_state) + 2;
        for (int k = 1; k < hs.Kx; ++k) {
            const bool l0 = (k == 1);
            TimedLaunch tl(&tm, stream, "plain_cr_reduce_x");
            k_cr_reduce_x<<<grid2(hs.lenx[k], hs.ny), blk, 0, stream>>>(
                l0 ? rhs_x : Dx[k - 1], l0 ? 4 : 1, l0 ? hs.NX * 4 : hs.lenx[k - 1] + 4, ABCx[k - 1],
                l0 ? hs.NX : hs.lenx[k - 1] + 4, Dx[k], hs.lenx[k] + 4, hs.lenx[k], hs.ny);
        }
        for (int k = 1; k < hs.Ky; ++k) {
            const bool l0 = (k == 1);
            TimedLaunch tl(&tm, stream, "plain_cr_reduce_y");
            k_cr_reduce_y<<<grid2(hs.nx, hs.leny[k]), blk, 0, stream>>>(
                l0 ? rhs_y : Dy[k - 1], l0 ? 4 : 1, l0 ? hs.NX * 4 : hs.NX, ABCy[k - 1], hs.NX, Dy[k], hs.leny[k], hs.nx);
        }
        for (int k = hs.Kx - 1; k >= 0; --k) {
            const bool l0 = (k == 0);
            TimedLaunch tl(&tm, stream, "plain_cr_subst_x");
            k_cr_subst_x<<<grid2(hs.lenx[k], hs.ny), blk, 0, stream>>>(
                l0 ? rhs_x : Dx[k], l0 ? 4 : 1, l0 ? hs.NX * 4 : hs.lenx[k] + 4, ABCx[k], l0 ? hs.NX : hs.lenx[k] + 4,
                k + 1 < hs.Kx ? Xx[k + 1] : nullptr, k + 1 < hs.Kx ? hs.lenx[k + 1] + 4 : 0, Xx[k],
                l0 ? hs.NX : hs.lenx[k] + 4, hs.lenx[k], hs.ny);
        }
        for (int k = hs.Ky - 1; k >= 0; --k) {
            const bool l0 = (k == 0);
            TimedLaunch tl(&tm, stream, "plain_cr_subst_y");
            k_cr_subst_y<<<grid2(hs.nx, hs.leny[k]), blk, 0, stream>>>(
                l0 ? rhs_y : Dy[k], l0 ? 4 : 1, l0 ? hs.NX * 4 : hs.NX, ABCy[k], hs.NX,
                k + 1 < hs.Ky ? Xy[k + 1] : nullptr, Xy[k], hs.leny[k], hs.nx);
        }
        {
            TimedLaunch tl(&tm, stream, "plain_copy_from");
            k_copy_from<<<grid2(hs.nx, hs.ny), blk, 0, stream>>>(new_state, Xx[0], Xy[0], c);
        }
        // boundaries East, North, West, South (engine.cpp:1342-1438)
        for (int side : {1, 0, 3, 2})
            if (int e = boundary_side(new_state, side)) return e;
        {
            TimedLaunch tl(&tm, stream, "plain_pass1");
            k_pass1<<<grid2(hs.nx + 2, hs.ny + 2), blk, 0, stream>>>(new_state, BOT, AUX1, H, U, V, AUX2, c);
        }
        CEL_CUDA_TRY(cudaGetLastError());
        const bool book = sch.after_pass();
        if (book) {
            const int o = old_i, oo = oldold_i, s = scratch_i;
            old_i = s; oldold_i = o; scratch_i = oo;
        }
        sim_idx = 1 - sim_idx;
        if (book && p.log.do_log && sch.last_count % p.log.log_step == 0) {
            // st_DumpToFile of the new state, with the time at the start of the step (engine.cpp:1488-1493)
            std::vector<float> host(ntex * 4);
            if (int e = get_state(host.data())) return e;
            if (int e = log_dump(p.log, host.data(), hs.nx, hs.ny, sch.last_start_time, log_elapsed, err)) return e;
        }
        return CEL_OK;
    }

    int timesteps(int n) override {
        for (int i = 0; i < n; ++i) {
            if (int e = reset_timestep_device()) return e;
            if (int e = timestep()) return e;
        }
        return CEL_OK;
    }

    int physical_steps(int n) override {
        for (int i = 0; i < n; ++i) {
            if (int e = reset_timestep_device()) return e;
            if (int e = timestep()) return e;
            while (sch.time_scheme == CEL_SCHEME_CORRECTOR) {
                if (int e = reset_timestep_device()) return e;
                if (int e = timestep()) return e;
            }
        }
        return CEL_OK;
    }

    int set_state(const float* rgba) override {
        CEL_CUDA_TRY(cudaMemcpyAsync(st[sim_idx], rgba, ntex * sizeof(float4), cudaMemcpyHostToDevice, stream));
        CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        bootstrap_needed = true;
        return CEL_OK;
    }
    int get_state(float* rgba) override {
        CEL_CUDA_TRY(cudaMemcpyAsync(rgba, st[sim_idx], ntex * sizeof(float4), cudaMemcpyDeviceToHost, stream));
        CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        return CEL_OK;
    }
    int get_bottom(float* b3) override {
        for (size_t i = 0; i < ntex; ++i) { b3[3 * i] = hs.BY[i]; b3[3 * i + 1] = hs.BX[i]; b3[3 * i + 2] = hs.BA[i]; }
        return CEL_OK;
    }
    int get_aux(float* rgba) override {
        CEL_CUDA_TRY(cudaMemcpyAsync(rgba, AUX1, ntex * sizeof(float4), cudaMemcpyDeviceToHost, stream));
        CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        return CEL_OK;
    }
    // newTerrainSettings -> fillTerrainTexture (engine.cpp:3313-3379): keep every texel's water depth
    // (w - BA_old + BA_new, in float as there), resample the bottom, clear both aux textures and
    // re-bootstrap.  The tridiagonal coefficients stay those of the old bottom until cel_remesh,
    // which rebuilds everything from the new grid (remesh re-creates the coefficient textures).
    int set_bathymetry(const float* z, int bnx, int bny) override {
        std::vector<float> host(ntex * 4);
        if (int e = get_state(host.data())) return e;
        for (size_t k = 0; k < ntex; ++k) host[4 * k] -= hs.BA[k];
        prepare_bottom(z, bnx, bny, hs.nx, hs.ny, float(p.width), float(p.length), hs);
        for (size_t k = 0; k < ntex; ++k) host[4 * k] += hs.BA[k];
        std::vector<float4> b(ntex);
        for (size_t i = 0; i < ntex; ++i) b[i] = make_float4(hs.BY[i], hs.BX[i], hs.BA[i], 0.f);
        CEL_CUDA_TRY(cudaMemcpyAsync(BOT, b.data(), ntex * sizeof(float4), cudaMemcpyHostToDevice, stream));
        CEL_CUDA_TRY(cudaMemcpyAsync(st[sim_idx], host.data(), ntex * sizeof(float4), cudaMemcpyHostToDevice, stream));
        CEL_CUDA_TRY(cudaMemsetAsync(AUX1, 0, ntex * sizeof(float4), stream));
        CEL_CUDA_TRY(cudaMemsetAsync(AUX2, 0, ntex * sizeof(float4), stream));
        CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        terrain.assign(z, z + size_t(bnx) * bny);
        terrain_nx = bnx;
        terrain_ny = bny;
        bootstrap_needed = true;
        return CEL_OK;
    }

    // the block sum of h comes from the latest GetStats (the state of the latest resetTimestep),
    // as the reference reads its GetStats staging texture
    int water_height(float x, float y, float* out) override {
        const float W = float(p.width), L = float(p.length);
        if (hs.nx < 4 || hs.ny < 4) { err = "getWaterHeight needs at least one 4x4 block"; return CEL_ERR_STATE; }
        if (!sch.initialized) { if (int e = reset_timestep(0.f, 0.f, nullptr)) return e; }
        int ix = 0, iy = 0;
        water_height_block(hs.nx, hs.ny, W, L, x, y, ix, iy);
        float sum_h = 0.f;
        CEL_CUDA_TRY(cudaMemcpyAsync(&sum_h, blocks + (size_t(iy) * (hs.nx / 4) + ix) * 9, sizeof(float),
                                     cudaMemcpyDeviceToHost, stream));
        CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        *out = terrain_height(hs, W, L, x, y) + sum_h / 16.0f;
        return CEL_OK;
    }

    int add_solitary_wave(double Hh, double theta_deg, double xc, double yc) override {
        // the state texture is updated in place from a copy; faces are not rebuilt
        // (engine.cpp:2154-2219 leaves bootstrap_needed unchanged)
        float4* s = st[sim_idx];
        CEL_CUDA_TRY(cudaMemcpyAsync(STRIP, s, ntex * sizeof(float4), cudaMemcpyDeviceToDevice, stream));
        const float th = float(theta_deg) * CEL_PI_HOST / 180.0f;
        k_add_solitary<<<grid2(hs.nx + 2, hs.ny + 2), dim3(BX2, BY2), 0, stream>>>(STRIP, BOT, s, c, float(Hh), th,
                                                                                   float(xc), float(yc));
        CEL_CUDA_TRY(cudaGetLastError());
        CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        return CEL_OK;
    }
    static constexpr float CEL_PI_HOST = 3.14159274101257324f;
    int set_stream(cudaStream_t s) override {
        CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        if (own_stream) cudaStreamDestroy(stream);
        own_stream = (s == nullptr);
        if (own_stream) CEL_CUDA_TRY(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        else stream = s;
        return CEL_OK;
    }
    int synchronize() override {
        CEL_CUDA_TRY(cudaStreamSynchronize(stream));
        return CEL_OK;
    }
    int set_tuning(int, int, int) override { return CEL_OK; }
    KernelTimer* timer() override { return &tm; }
    int nx() const override { return hs.nx; }
    int ny() const override { return hs.ny; }
};

}  // namespace

EngineIface* make_plain_engine(const cel_params& p, const float* bathy, int bnx, int bny, std::string& err) {
    auto* e = new PlainEngine();
    if (int s = e->init(p, bathy, bnx, bny)) {
        err = e->err;
        delete e;
        (void)s;
        return nullptr;
    }
    return e;
}

}  // namespace cel

// ---------------------------------------------------------------------------------------------
// Allocation-free statistics entry point.
//
// Some callers of this library must not allocate device memory at the moment they ask for the
// domain statistics: frame loops where the device-wide synchronisation of cudaMalloc / cudaFree
// would stall every other stream, and host applications whose device memory is entirely handed out
// by their own allocator.  cel_stats_noalloc computes the GetStats reduction and the FP64 volume of
// a state that the caller already keeps in device memory, using only the fixed scratch array below:
// the 4x4 block partials, the volume partials and the FP64 totals.  The array is reserved on every
// GPU that loads the library and stays there until the process exits.  All calls share it, so two
// calls whose work overlaps on the GPU (on different streams, or from different threads) race; run
// them one after another.
// ---------------------------------------------------------------------------------------------
namespace cel {
namespace {

constexpr int NOALLOC_MAX_BLOCKS = 65536;                  // 4x4 blocks: up to 1,048,576 cells
constexpr int NOALLOC_VOL_CTAS = 1184;                     // volume partials: 8 CTAs per SM of a B200
// block partials (9 floats each) | volume partials (2 doubles per CTA) | 16 doubles of totals
constexpr int NOALLOC_FLOATS = NOALLOC_MAX_BLOCKS * 9 + NOALLOC_VOL_CTAS * 4 + 32;
static __device__ __align__(256) float g_noalloc_scratch[NOALLOC_FLOATS];

// GetStats (compute.hlsl:1319-1378) reading the bottom in the public {BY, BX, BA} layout.
__global__ void k_getstats_b3(const float4* __restrict__ st, const float* __restrict__ b3, float* __restrict__ blocks,
                              SimConsts c) {
    const int bx = blockIdx.x * blockDim.x + threadIdx.x;
    const int by = blockIdx.y * blockDim.y + threadIdx.y;
    const int nbx = c.nx / 4, nby = c.ny / 4;
    if (bx >= nbx || by >= nby) return;
    float sh = 0, sb = 0, shu = 0, shv = 0, sk = 0, mu = 0, mh = 0, mc = 0, mf = 0;
    for (int j = 2; j < 6; ++j)
        for (int ii = 2; ii < 6; ++ii) {
            const size_t i = size_t(by * 4 + j) * c.NX + bx * 4 + ii;
            const float4 s = st[i];
            const float B = b3[3 * i + 2];
            const float h = fmaxf(0.f, s.x - B);
            const float cc = sqrtf(c.g * h);
            const float q = div_by_h(h, c.epsilon);
            const float u = q * s.y, v = q * s.z;
            sh += h; sb += h * (B + 0.5f * h); shu += s.y; shv += s.z;
            sk += (s.y * u + s.z * v);
            const float u2v2 = u * u + v * v;
            mu = fmaxf(mu, u2v2); mh = fmaxf(mh, h);
            mc = fmaxf(mc, (fabsf(u) + cc) * c.one_over_dx);
            mc = fmaxf(mc, (fabsf(v) + cc) * c.one_over_dy);
            mf = fmaxf(mf, u2v2 * q);
        }
    float* o = blocks + (size_t(by) * nbx + bx) * 9;
    o[0] = sh; o[1] = sb; o[2] = shu; o[3] = shv; o[4] = sk; o[5] = mu; o[6] = mh; o[7] = mc; o[8] = mf;
}

// FP64 volume of the interior cells (and the non-finite flag), one partial per CTA: CTA k sums a
// fixed interleaved share of the cells, so the totals do not depend on scheduling.
__global__ void __launch_bounds__(256) k_volume_b3(const float4* __restrict__ st, const float* __restrict__ b3,
                                                   SimConsts c, double* __restrict__ part) {
    __shared__ double sv[8];
    __shared__ int sb;
    if (threadIdx.x == 0) sb = 0;
    __syncthreads();
    double v = 0.0;
    int bad = 0;
    const int n = c.nx * c.ny;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const size_t i = size_t(k / c.nx + 2) * c.NX + (k % c.nx + 2);
        const float4 s = st[i];
        if (!isfinite(s.x) || !isfinite(s.y) || !isfinite(s.z)) bad = 1;
        v += fmax(0.0, double(s.x) - double(b3[3 * i + 2]));
    }
    for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) sv[threadIdx.x >> 5] = v;
    if (bad) sb = 1;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += sv[w];
        part[2 * blockIdx.x] = t;
        part[2 * blockIdx.x + 1] = sb ? 1.0 : 0.0;
    }
}

// One CTA: FP64 totals of the block partials and the volume partials; every output word is
// written on every call.
__global__ void k_reduce_b3(const float* __restrict__ blocks, int nb, const double* __restrict__ vol, int nvol,
                            double* __restrict__ out) {
    __shared__ double sm[10][32];
    __shared__ int bad_s;
    double v[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    int bad = 0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        const float* b = blocks + size_t(k) * 9;
        for (int q = 0; q < 5; ++q) v[q] += double(b[q]);
        for (int q = 5; q < 9; ++q) v[q] = fmax(v[q], double(b[q]));
    }
    for (int k = threadIdx.x; k < nvol; k += blockDim.x) {
        v[9] += vol[2 * k];
        if (vol[2 * k + 1] != 0.0) bad = 1;
    }
    if (threadIdx.x == 0) bad_s = 0;
    __syncthreads();
    if (bad) bad_s = 1;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int q = 0; q < 10; ++q) {
        double x = v[q];
        for (int off = 16; off; off >>= 1) {
            const double y = __shfl_down_sync(0xffffffffu, x, off);
            x = (q >= 5 && q < 9) ? fmax(x, y) : x + y;
        }
        if (lane == 0) sm[q][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = blockDim.x >> 5;
        for (int q = 0; q < 10; ++q) {
            double x = lane < nw ? sm[q][lane] : 0.0;
            for (int off = 16; off; off >>= 1) {
                const double y = __shfl_down_sync(0xffffffffu, x, off);
                x = (q >= 5 && q < 9) ? fmax(x, y) : x + y;
            }
            if (lane == 0) out[q] = x;
        }
        if (lane == 0) out[10] = bad_s ? 1.0 : 0.0;
    }
}

// Device address of the scratch array, looked up once per device (with that device current).
constexpr int NOALLOC_MAX_DEVICES = 64;
float* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};   // guarded by g_noalloc_mutex
std::mutex g_noalloc_mutex;

}  // namespace

}  // namespace cel

extern "C" int cel_stats_noalloc(const float* d_state_rgba, const float* d_bottom_b3, const cel_params* p,
                                 void* cuda_stream, cel_stats* out) {
    using namespace cel;
    if (!d_state_rgba || !d_bottom_b3 || !p || !out) { set_error("null argument"); return CEL_ERR_ARG; }
    if (p->nx < 4 || p->ny < 4) { set_error("cel_stats_noalloc: nx and ny must be >= 4"); return CEL_ERR_ARG; }
    const long long nb = (long long)(p->nx / 4) * (p->ny / 4);
    if (nb > NOALLOC_MAX_BLOCKS) {
        set_error("cel_stats_noalloc: domain has " + std::to_string(nb) + " 4x4 blocks; the fixed scratch holds " +
                  std::to_string(NOALLOC_MAX_BLOCKS) + " (at most 1,048,576 interior cells)");
        return CEL_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { set_error(std::string("cel_stats_noalloc: ") + cudaGetErrorString(e)); return CEL_ERR_CUDA; }
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) { set_error("cel_stats_noalloc: device index out of range"); return CEL_ERR_ARG; }
    float* blocks = nullptr;
    {
        // the array's device address on this device, resolved by the first call here (with the
        // device current) under a lock, so that concurrent first calls do not race
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_ptr[dev]) {
            float* ptr = nullptr;
            e = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_noalloc_scratch);
            if (e != cudaSuccess || !ptr) {
                set_error(std::string("cel_stats_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
                return CEL_ERR_CUDA;
            }
            g_noalloc_ptr[dev] = ptr;
        }
        blocks = g_noalloc_ptr[dev];
    }
    // volume partials after the block partials (byte offset 65,536 x 36, a multiple of 256), totals last
    double* vol = reinterpret_cast<double*>(blocks + size_t(NOALLOC_MAX_BLOCKS) * 9);
    double* totals = vol + 2 * NOALLOC_VOL_CTAS;
    HostSetup hs;
    hs.nx = p->nx; hs.ny = p->ny; hs.NX = p->nx + 4; hs.NY = p->ny + 4;
    hs.dx = float(p->width) / float(p->nx - 1);
    hs.dy = float(p->length) / float(p->ny - 1);
    {
        const float m = std::max(hs.dx, hs.dy);
        hs.eps = std::min(float(p->epsilon), m * m * m * m);
    }
    const SimConsts c = make_consts(*p, hs, hs.NX);
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    const float4* st = reinterpret_cast<const float4*>(d_state_rgba);
    const int nbx = p->nx / 4, nby = p->ny / 4;
    k_getstats_b3<<<grid2(nbx, nby), dim3(BX2, BY2), 0, s>>>(st, d_bottom_b3, blocks, c);
    const int nvol = int(std::min<long long>(NOALLOC_VOL_CTAS, (p->nx * (long long)p->ny + 255) / 256));
    k_volume_b3<<<nvol, 256, 0, s>>>(st, d_bottom_b3, c, vol);
    k_reduce_b3<<<1, 1024, 0, s>>>(blocks, int(nb), vol, nvol, totals);
    e = cudaGetLastError();
    if (e != cudaSuccess) { set_error(std::string("cel_stats_noalloc: ") + cudaGetErrorString(e)); return CEL_ERR_CUDA; }
    double v[11];
    e = cudaMemcpyAsync(v, totals, sizeof(v), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { set_error(std::string("cel_stats_noalloc: ") + cudaGetErrorString(e)); return CEL_ERR_CUDA; }
    const double DENSITY = 1000;
    const double AREA = double(float(p->width) / float(p->nx - 1) * float(p->length) / float(p->ny - 1));
    const double g = double(c.g);
    std::memset(out, 0, sizeof(*out));
    out->mass = v[0] * DENSITY * AREA;
    out->potential_energy = v[1] * g * DENSITY * AREA;
    out->x_momentum = v[2] * DENSITY * AREA;
    out->y_momentum = v[3] * DENSITY * AREA;
    out->kinetic_energy = v[4] * 0.5 * DENSITY * AREA;
    out->total_energy = out->kinetic_energy + out->potential_energy;
    out->max_speed = std::sqrt(v[5]);
    out->max_depth = v[6];
    out->cfl_rate = v[7];
    out->max_froude = std::sqrt(v[8] / g);
    out->mass_full = v[9];
    out->health = v[10] != 0 ? CEL_ERR_NUMERIC : 0;
    out->timestep = p->timestep;
    out->cfl_number = out->cfl_rate * double(float(p->timestep));
    return CEL_OK;
}
