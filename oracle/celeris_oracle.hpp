// CPU oracle for the Celeris Boussinesq timestep path — TEST INFRASTRUCTURE ONLY.
//
// This header restates, line by line, the reference's per-timestep path:
//   * msvc/Release/shaders/compute.hlsl  (Pass1/Pass2/Pass3Predictor, CR reduce/substitute,
//     CopyFromXxAndXy, boundary shaders, GetStats, AddSolitaryWave)
//   * engine.cpp  (timestep() pass order, zeroing copies, E->N->W->S boundary order,
//     scheme state machine and history rotation, resetTimestep() stats and dt,
//     createTridiagonalCoefTextures(), createSimTextures() initial condition)
//   * terrain_heightfield.cpp (bathymetry bilinear sampling and BY/BX/BA staggering)
// It is templated on the arithmetic type: Real = double is the correctness oracle,
// Real = float (OpenMP) is the CPU FP32 transcription used as the CPU baseline.
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg may use this code; the
// product library (celeris_b200/) never links or calls it.
//
// Parity pinning: the reference ships no golden vectors.  This restatement is pinned by
// (i) the reference's own terrain_heightfield.cpp compiled in place (oracle/ref_build.py),
// (ii) the reference's own compute.hlsl passes compiled as C++ in place and stepped through
// the same orchestration (oracle/ref_build.py -> oracle/_ref), and (iii) analytic
// known-answer tests (lake at rest, solitary-wave celerity, tridiagonal vs dense solve).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------------------------------
// Parameters (the fields readInputCML fills, main.cpp:500-913, settings.hpp:306-438)
// ---------------------------------------------------------------------------------------
enum BoundaryType { B_SOLID = 0, B_SPONGE = 1, B_SINEWAVE = 2, B_IRREGULAR = 3, B_UTS = 4 };
enum TimeScheme { EULER = 0, PREDICTOR = 1, CORRECTOR = 2, PREDICTOR_ADAPTIVE = 3 };  // settings.hpp:298

struct Boundary {
    int type = B_SOLID;      // BoundarySetting() default "Solid", width 2 (settings.hpp:166)
    int width = 2;
    double sea_level = 0;
    double amplitude = 0, period = 0, theta = 0;      // sine wave; theta in radians
    std::vector<std::array<double, 4>> waves;          // irregular: amplitude, period, theta, phase
    std::vector<std::array<double, 4>> uts;            // uniform time series: t, eta, hu, hv
};

struct Soliton { double H, theta, xc, yc, length; };  // theta in radians (main.cpp:651)

struct Params {
    int nx = 100, ny = 100;
    double width = 100, length = 100, swl = 0;        // InitSetting() defaults (settings.hpp:386-411)
    bool boussinesq = true;
    double epsilon = 5e-8, theta = 2;
    int correction_steps = 0;
    double timestep = 1e-4;
    bool adaptive = false;
    double ema_alpha = 0.5, min_timestep_ratio = 0.05;
    bool manning = false;
    double friction = 0;
    double gravity = 9.81;                            // gui_manager.cpp:106
    double dissipation_threshold = 0.25;              // SurfaceShadingSetting() (settings.hpp:223)
    double whitewater_decay = 0.25;
    Boundary west, east, south, north;
    std::vector<Soliton> solitons;
};

struct Stats {
    // resetTimestep() outputs (engine.cpp:1685-1746)
    double mass, x_momentum, y_momentum, kinetic_energy, potential_energy, total_energy;
    double max_speed, max_depth, max_froude, cfl_rate, cfl_number, timestep, total_time;
    // Full-interior double sum of h (every interior cell, not only the 4x4 blocks)
    double mass_full;
};

// ---------------------------------------------------------------------------------------
// Bathymetry prep: terrain_heightfield.cpp:213-311.  Always evaluated in float, exactly as
// the reference does, so every form (FP64 oracle, FP32 forms, GPU) starts from the same
// staggered bottom.  Output planes are (nx+4)*(ny+4), row-major y*(nx+4)+x.
// ---------------------------------------------------------------------------------------
inline float bathy_sample(const std::vector<float>& z, int bnx, int bny, float W, float L, float x, float y) {
    // getBathymetry (terrain_heightfield.cpp:213-242)
    x = (x + W / 2) / W * (bnx - 1);
    y = y / L * (bny - 1);
    if (x < 0) x = 0;
    if (x > bnx - 1) x = float(bnx - 1);
    if (y < 0) y = 0;
    if (y > bny - 1) y = float(bny - 1);
    const int xdown = int(std::floor(x)), xup = int(std::ceil(x));
    const int ydown = int(std::floor(y)), yup = int(std::ceil(y));
    const float xf = x - xdown, yf = y - ydown;
    auto lerp = [](float t, float a, float b) { return a + t * (b - a); };
    const float d0 = lerp(xf, z[size_t(ydown) * bnx + xdown], z[size_t(ydown) * bnx + xup]);
    const float d1 = lerp(xf, z[size_t(yup) * bnx + xdown], z[size_t(yup) * bnx + xup]);
    return lerp(yf, d0, d1);
}

inline void prepare_bottom(const std::vector<float>& z, int bnx, int bny, int nx, int ny, float W, float L,
                           std::vector<float>& BY, std::vector<float>& BX, std::vector<float>& BA) {
    // UpdateTerrainHeightfield (terrain_heightfield.cpp:244-297): corner samples at (i-2.5, j-2.5)
    // and the same accumulation order (so float results are identical).
    const int pitch = nx + 4;
    BY.assign(size_t(pitch) * (ny + 4), 0.f);
    BX.assign(size_t(pitch) * (ny + 4), 0.f);
    BA.assign(size_t(pitch) * (ny + 4), 0.f);
    for (int j = 0; j < ny + 5; ++j) {
        const float y = (float(j) - 2.5f) / float(ny - 1) * L;
        for (int i = 0; i < nx + 5; ++i) {
            const float x = (float(i) - 2.5f) / float(nx - 1) * W - (W / 2);
            const float zz = bathy_sample(z, bnx, bny, W, L, x, y);
            if (i < nx + 4) {
                if (j < ny + 4) BA[size_t(j) * pitch + i] = 0.25f * zz;
                if (j > 0) {
                    BA[size_t(j - 1) * pitch + i] += 0.25f * zz;
                    BY[size_t(j - 1) * pitch + i] = 0.5f * zz;
                }
            }
            if (i > 0) {
                if (j < ny + 4) {
                    BA[size_t(j) * pitch + i - 1] += 0.25f * zz;
                    BX[size_t(j) * pitch + i - 1] = 0.5f * zz;
                }
                if (j > 0) {
                    BA[size_t(j - 1) * pitch + i - 1] += 0.25f * zz;
                    BX[size_t(j - 1) * pitch + i - 1] += 0.5f * zz;
                    BY[size_t(j - 1) * pitch + i - 1] += 0.5f * zz;
                }
            }
        }
    }
}

inline int count_of_matrices(int n) {  // st_getCountOfMatrices (engine.cpp:741-748)
    int c = 1;
    while (n > 1) { n /= 2; ++c; }
    return c;
}

// Transcendentals: in the float build each one is evaluated in double and rounded once to
// float (the correctly rounded value); the plain GPU form computes them the same way, so the two
// FP32 paths agree bit for bit.  (The reference's HLSL intrinsics are approximate GPU
// instructions; no CPU restatement can reproduce them exactly.)
template <typename R> inline R t_sin(R x) { return std::sin(x); }
template <typename R> inline R t_cos(R x) { return std::cos(x); }
template <typename R> inline R t_tanh(R x) { return std::tanh(x); }
template <typename R> inline R t_atan(R x) { return std::atan(x); }
template <typename R> inline R t_cosh(R x) { return std::cosh(x); }
template <typename R> inline R t_pow(R x, R y) { return std::pow(x, y); }
template <> inline float t_sin<float>(float x) { return float(std::sin(double(x))); }
template <> inline float t_cos<float>(float x) { return float(std::cos(double(x))); }
template <> inline float t_tanh<float>(float x) { return float(std::tanh(double(x))); }
template <> inline float t_atan<float>(float x) { return float(std::atan(double(x))); }
template <> inline float t_cosh<float>(float x) { return float(std::cosh(double(x))); }
template <> inline float t_pow<float>(float x, float y) { return float(std::pow(double(x), double(y))); }

// ---------------------------------------------------------------------------------------
// The engine (templated on the arithmetic type)
// ---------------------------------------------------------------------------------------
template <typename R>
struct V4 { R r = 0, g = 0, b = 0, a = 0; };

template <typename R>
class Engine {
public:
    using T4 = V4<R>;
    Params p;
    int nx = 0, ny = 0, NX = 0, NY = 0;
    R dx = 0, dy = 0, eps = 0, PI_ = 0;
    std::vector<R> BY, BX, BA;

    // Texture mirror of engine.hpp:198-216 (ghost-padded NX*NY, row-major)
    std::vector<T4> state[2], H, U, V, xflux, yflux, aux1, aux2, cur;
    std::vector<T4> grad[3], pred, fg[3], fgpred;
    // Cyclic-reduction level textures (engine.cpp:2612-2887, 3070-3230)
    std::vector<std::vector<T4>> ABCx, D1x, D1xc, ABCy, D1y, D1yc;
    int Kx = 0, Ky = 0;
    std::vector<int> lenx, leny;

    int sim_idx = 0, old_i = 0, oldold_i = 1, scratch_i = 2;
    int fg_old_i = 0, fg_oldold_i = 1, fg_scratch_i = 2;
    bool bootstrap_needed = true;
    int time_scheme = EULER, timestep_count = 1, correction_steps_count = 0;
    R current_timestep = 0, old_timestep = 0, old_old_timestep = 0, total_time = 0;
    bool initialized_timesteps = false, target_cfl_set = false;
    double target_cfl = 0;
    int uts_iter[4] = {1, 1, 1, 1};
    int passes = 0;

    static constexpr double MIN_DEPTH = 0.0001;  // compute.hlsl:1062

    size_t at(int x, int y) const { return size_t(y) * NX + x; }

    // ---- setup ---------------------------------------------------------------------------
    void init(const Params& prm, const std::vector<float>& zgrid, int bnx, int bny,
              const std::vector<float>* hot = nullptr) {
        p = prm;
        nx = p.nx; ny = p.ny; NX = nx + 4; NY = ny + 4;
        const float Wf = float(p.width), Lf = float(p.length);
        std::vector<float> by, bx, ba;
        prepare_bottom(zgrid, bnx, bny, nx, ny, Wf, Lf, by, bx, ba);
        BY.assign(by.begin(), by.end()); BX.assign(bx.begin(), bx.end()); BA.assign(ba.begin(), ba.end());
        dx = R(p.width) / R(nx - 1);
        dy = R(p.length) / R(ny - 1);
        // CalcEpsilon (engine.cpp:290-299)
        {
            R mx = std::max(dx, dy);
            R p4 = mx * mx * mx * mx;
            eps = std::min(R(p.epsilon), p4);
        }
        PI_ = std::is_same<R, float>::value ? R(4.0f * std::atan(1.0f)) : R(3.14159265358979323846);
        const size_t n = size_t(NX) * NY;
        for (auto* t : {&state[0], &state[1], &H, &U, &V, &xflux, &yflux, &aux1, &aux2, &cur, &pred, &fgpred})
            t->assign(n, T4());
        for (int k = 0; k < 3; ++k) { grad[k].assign(n, T4()); fg[k].assign(n, T4()); }
        build_coefficients();
        initial_condition(hot);
        sim_idx = 0; old_i = 0; oldold_i = 1; scratch_i = 2;
        fg_old_i = 0; fg_oldold_i = 1; fg_scratch_i = 2;
        bootstrap_needed = true;
        time_scheme = EULER; timestep_count = 1; correction_steps_count = p.correction_steps;
        total_time = 0; initialized_timesteps = false; target_cfl_set = false;
        current_timestep = old_timestep = old_old_timestep = 0;
        for (int& u : uts_iter) u = 1;
        passes = 0;
        // Adaptive target CFL: readBathymetry sets it (terrain_heightfield.cpp:203-207), then
        // resetTimestep replaces it with dt*cfl on the first call (engine.cpp:1700-1703).
        target_cfl = 0;
    }

    R sea_level_for_coefs() const { return p.boussinesq ? R(p.swl) : R(-9999); }

    // createTridiagonalCoefTextures (engine.cpp:2612-2887)
    void build_coefficients() {
        const R BCOEF = std::is_same<R, float>::value ? R(1 / 15.0f) : R(1.0 / 15.0);
        const R THIRD = std::is_same<R, float>::value ? R(1 / 3.0f) : R(1.0 / 3.0);
        const R dx2 = dx * dx, dy2 = dy * dy;
        const R sl = sea_level_for_coefs();
        Kx = count_of_matrices(nx); Ky = count_of_matrices(ny);
        lenx.resize(Kx); leny.resize(Ky);
        { int L = nx; for (int k = 0; k < Kx; ++k) { lenx[k] = L; L /= 2; } }
        { int L = ny; for (int k = 0; k < Ky; ++k) { leny[k] = L; L /= 2; } }
        ABCx.assign(Kx, {}); D1x.assign(Kx, {}); D1xc.assign(Kx, {});
        ABCy.assign(Ky, {}); D1y.assign(Ky, {}); D1yc.assign(Ky, {});
        for (int k = 0; k < Kx; ++k) {
            const size_t n = size_t(lenx[k] + 4) * NY;
            ABCx[k].assign(n, T4()); D1x[k].assign(n, T4()); D1xc[k].assign(n, T4());
        }
        for (int k = 0; k < Ky; ++k) {
            const size_t n = size_t(NX) * (leny[k] + 4);
            ABCy[k].assign(n, T4()); D1y[k].assign(n, T4()); D1yc[k].assign(n, T4());
        }
        auto dat = [&](int x, int y) { return std::max(R(0), sl - BA[at(x, y)]); };
        // x, level 0
        {
            const int W0 = NX;
            for (int i = 0; i < NY; ++i) {
                const int ii = std::max(2, std::min(ny + 1, i));
                for (int j = 0; j < NX; ++j) {
                    T4& c = ABCx[0][size_t(i) * W0 + j];
                    if (j <= 1 || j >= NX - 2) { c.r = 0; c.g = 1; c.b = 0; continue; }
                    const int jj = std::max(2, std::min(nx + 1, j));
                    const R d = dat(jj, ii), drr = dat(jj + 2, ii), dr = dat(jj + 1, ii);
                    const R dl = dat(jj - 1, ii), dll = dat(jj - 2, ii);
                    const R K1 = (BCOEF + THIRD) * (d * d / dx2);
                    const R K2 = (d / dx2) * (-drr + 8 * dr - 8 * dl + dll);
                    c.r = -K1 + K2 / R(72);
                    if (j == 2) c.r = 0;
                    c.g = 1 + 2 * K1;
                    c.b = -(K1 + K2 / R(72));
                    if (j == NX - 3) c.b = 0;
                }
            }
        }
        // x, levels k >= 1 (CR-reduced coefficients)
        for (int k = 1; k < Kx; ++k) {
            const int Wp = lenx[k - 1] + 4, Wk = lenx[k] + 4;
            for (int i = 0; i < NY; ++i) {
                for (int j = 0; j < Wk; ++j) {
                    T4& c = ABCx[k][size_t(i) * Wk + j];
                    if (j <= 1 || j >= Wk - 2) { c.r = 0; c.g = 1; c.b = 0; continue; }
                    const int pj = (j - 2) * 2 + 3;  // odd row of the previous level
                    const T4& pm = ABCx[k - 1][size_t(i) * Wp + pj - 1];
                    const T4& p0 = ABCx[k - 1][size_t(i) * Wp + pj];
                    const T4& pp = ABCx[k - 1][size_t(i) * Wp + pj + 1];
                    const R k1 = p0.r / pm.g, k2 = p0.b / pp.g;
                    c.r = -pm.r * k1;
                    c.g = p0.g - pm.b * k1 - pp.r * k2;
                    c.b = -pp.b * k2;
                }
            }
        }
        // y, level 0
        {
            for (int i = 0; i < NY; ++i) {
                const int ii = std::max(2, std::min(ny + 1, i));
                for (int j = 0; j < NX; ++j) {
                    T4& c = ABCy[0][size_t(i) * NX + j];
                    if (i <= 1 || i >= NY - 2) { c.r = 0; c.g = 1; c.b = 0; continue; }
                    const int jj = std::max(2, std::min(nx + 1, j));
                    const R d = dat(jj, ii), duu = dat(jj, ii + 2), du = dat(jj, ii + 1);
                    const R dd = dat(jj, ii - 1), ddd = dat(jj, ii - 2);
                    const R K1 = (BCOEF + THIRD) * (d * d / dy2);
                    const R K2 = (d / dy2) * (-duu + 8 * du - 8 * dd + ddd);
                    c.r = -K1 + K2 / R(72);
                    if (i == 2) c.r = 0;
                    c.g = 1 + 2 * K1;
                    c.b = -(K1 + K2 / R(72));
                    if (i == NY - 3) c.b = 0;
                }
            }
        }
        for (int k = 1; k < Ky; ++k) {
            const int Hk = leny[k] + 4;
            for (int i = 0; i < Hk; ++i) {
                for (int j = 0; j < NX; ++j) {
                    T4& c = ABCy[k][size_t(i) * NX + j];
                    if (i <= 1 || i >= Hk - 2) { c.r = 0; c.g = 1; c.b = 0; continue; }
                    const int pi = (i - 1) * 2 + 1;
                    const T4& pm = ABCy[k - 1][size_t(pi - 1) * NX + j];
                    const T4& p0 = ABCy[k - 1][size_t(pi) * NX + j];
                    const T4& pp = ABCy[k - 1][size_t(pi + 1) * NX + j];
                    const R k1 = p0.r / pm.g, k2 = p0.b / pp.g;
                    c.r = -pm.r * k1;
                    c.g = p0.g - pm.b * k1 - pp.r * k2;
                    c.b = -pp.b * k2;
                }
            }
        }
    }

    // host solitaryWave (engine.cpp:103-112)
    void solitary_host(R depth, R Hh, R th, R x0, R y0, R x, R y, R& eta, R& hu, R& hv) const {
        const R K = std::sqrt(R(0.75) * std::abs(Hh) / (depth * depth * depth));
        const R C = std::sqrt(R(p.gravity) * (Hh + depth));
        const R ch = std::cosh(K * ((x - x0) * std::cos(th) + (y - y0) * std::sin(th)));
        const R te = Hh * R(1) / (ch * ch);
        eta = te; hu = C * std::cos(th) * te; hv = C * std::sin(th) * te;
    }

    // createSimTextures initial condition (engine.cpp:2940-3016)
    void initial_condition(const std::vector<float>* hot) {
        const R swl = R(p.swl);
        for (int j = 0; j < NY; ++j)
            for (int i = 0; i < NX; ++i) {
                const int ii = std::max(2, std::min(nx + 1, i));
                const int jj = std::max(2, std::min(ny + 1, j));
                const R B = BA[at(ii, jj)];
                const R depth = std::max(R(0), swl - B);
                R w, hu, hv;
                if (hot) {
                    const size_t k = (size_t(j) * NX + i) * 3;
                    w = R((*hot)[k]); hu = R((*hot)[k + 1]); hv = R((*hot)[k + 2]);
                } else {
                    w = std::max(swl, B); hu = 0; hv = 0;
                }
                for (const Soliton& s : p.solitons) {
                    if (s.H == 0) continue;
                    // Dry cell: the sech^2 profile's limit is 0 there; the reference evaluates
                    // 0 * sqrt(0/0) = NaN for a zero-height taper and at the crest line.
                    if (depth == 0) continue;
                    const R th = R(s.theta);
                    const R vd = std::abs(std::sin(th) * (dx * R(i) - R(s.xc))) +
                                 std::abs(std::cos(th) * (dy * R(j) - R(s.yc)));
                    R e, u, v;
                    if (vd > R(s.length) / 2) {
                        R tH = 0;
                        const R sm = PI_ / std::sqrt(R(0.75) * R(s.H) / (depth * depth * depth));
                        if (vd - R(s.length) / 2 < sm)
                            tH = R(s.H) * (R(0.5) * std::cos(PI_ / sm * (vd - R(s.length) / 2)) + R(0.5));
                        solitary_host(depth, tH, th, R(s.xc), R(s.yc), dx * R(i), dy * R(j), e, u, v);
                    } else {
                        solitary_host(depth, R(s.H), th, R(s.xc), R(s.yc), dx * R(i), dy * R(j), e, u, v);
                    }
                    w += e; hu += u; hv += v;
                }
                T4 s; s.r = w; s.g = hu; s.b = hv; s.a = 0;
                state[0][at(i, j)] = s;
                state[1][at(i, j)] = s;
            }
    }

    // ---- shader helpers (compute.hlsl:292-370) --------------------------------------------
    R two_theta() const { return R(2) * R(p.theta); }
    static R minmod(R a, R b, R c) {
        return (a > 0 && b > 0 && c > 0) ? std::min(std::min(a, b), c)
             : (a < 0 && b < 0 && c < 0) ? std::max(std::max(a, b), c) : R(0);
    }
    void reconstruct(R west, R here, R east, R& ow, R& oe, R& sd) const {
        const R tt = two_theta();
        const R z1 = tt * (here - west), z2 = east - west, z3 = tt * (east - here);
        const R g2 = R(0.25) * minmod(z1, z2, z3);
        const R mu = R(0.5) * (z1 + z2 + z3) / R(3);
        sd = std::sqrt(((z1 - mu) * (z1 - mu) + (z2 - mu) * (z2 - mu) + (z3 - mu) * (z3 - mu)) / R(3));
        oe = here + g2;
        ow = here - g2;
    }
    static void correct_w(R Bw, R Be, R wbar, R& ww, R& we) {
        if (we < Be) { we = Be; ww = std::max(Bw, 2 * wbar - Be); }
        else if (ww < Bw) { we = std::max(Be, 2 * wbar - Bw); ww = Bw; }
    }
    R div_by_h(R h) const {
        const R h2 = h * h, h4 = h2 * h2;
        return std::sqrt(R(2)) * h / std::sqrt(h4 + std::max(h4, eps));
    }
    static R numflux(R ap, R am, R Fp, R Fm, R dU) {
        if (ap - am != 0) return (ap * Fm - am * Fp + ap * am * dU) / (ap - am);
        return 0;
    }
    R dt_() const { return current_timestep; }
    // initSetting.timestep is a float (settings.hpp:318): every build, FP64 included, steps with
    // the single-precision value of the configured time step
    R dt_setting() const { return R(float(p.timestep)); }
    R g_() const { return R(p.gravity); }

    // ---- Pass1 (compute.hlsl:380-458), region [1,nx+3) x [1,ny+3) -------------------------
    virtual ~Engine() = default;

    virtual void pass1(const std::vector<T4>& st) {
        const R odx = R(1) / dx, ody = R(1) / dy;
        const R thr = R(p.dissipation_threshold);
#pragma omp parallel for schedule(static)
        for (int y = 1; y < ny + 3; ++y)
            for (int x = 1; x < nx + 3; ++x) {
                const T4 c = st[at(x, y)], s = st[at(x, y - 1)], n = st[at(x, y + 1)];
                const T4 w_ = st[at(x - 1, y)], e = st[at(x + 1, y)];
                const R BN = BY[at(x, y)], BE = BX[at(x, y)], BS = BY[at(x, y - 1)], BW = BX[at(x - 1, y)];
                R wN, wE, wS, wW, huN, huE, huS, huW, hvN, hvE, hvS, hvW, sd, msd;
                reconstruct(w_.r, c.r, e.r, wW, wE, sd);
                msd = sd * odx;
                reconstruct(s.r, c.r, n.r, wS, wN, sd);
                msd = t_atan(std::max(msd, sd * ody));
                reconstruct(w_.g, c.g, e.g, huW, huE, sd);
                reconstruct(s.g, c.g, n.g, huS, huN, sd);
                reconstruct(w_.b, c.b, e.b, hvW, hvE, sd);
                reconstruct(s.b, c.b, n.b, hvS, hvN, sd);
                correct_w(BW, BE, c.r, wW, wE);
                correct_w(BS, BN, c.r, wS, wN);
                T4 h; h.r = wN - BN; h.g = wE - BE; h.b = wS - BS; h.a = wW - BW;
                T4 u, v;
                { R q = div_by_h(h.r); u.r = q * huN; v.r = q * hvN; }
                { R q = div_by_h(h.g); u.g = q * huE; v.g = q * hvE; }
                { R q = div_by_h(h.b); u.b = q * huS; v.b = q * hvS; }
                { R q = div_by_h(h.a); u.a = q * huW; v.a = q * hvW; }
                H[at(x, y)] = h; U[at(x, y)] = u; V[at(x, y)] = v;
                const T4 a1 = aux1[at(x, y)];
                const R mid = std::max((h.r + h.g + h.b + h.a) / R(4), a1.r);
                R bw = a1.a;
                if (msd > thr) bw = R(1);
                T4 a2; a2.r = mid; a2.g = 0; a2.b = msd; a2.a = bw;
                aux2[at(x, y)] = a2;
            }
    }

    // ---- Pass2 (compute.hlsl:470-542), region [1,nx+2) x [1,ny+2) -------------------------
    virtual void pass2() {
        const R g = g_(), half_g = R(0.5) * g;
        const R decay = R(1) / (R(1) + R(2) * R(p.whitewater_decay));
        const R decay_dt = t_pow(std::abs(decay), dt_());
        std::fill(xflux.begin(), xflux.end(), T4());
        std::fill(yflux.begin(), yflux.end(), T4());
#pragma omp parallel for schedule(static)
        for (int y = 1; y < ny + 2; ++y)
            for (int x = 1; x < nx + 2; ++x) {
                const T4 hc = H[at(x, y)], uc = U[at(x, y)], vc = V[at(x, y)];
                const R hN = hc.r, hE = hc.g, uN = uc.r, uE = uc.g, vN = vc.r, vE = vc.g;
                const R hWe = H[at(x + 1, y)].a, hSn = H[at(x, y + 1)].b;
                const R uWe = U[at(x + 1, y)].a, uSn = U[at(x, y + 1)].b;
                const R vWe = V[at(x + 1, y)].a, vSn = V[at(x, y + 1)].b;
                const R cN = std::sqrt(g * hN), cE = std::sqrt(g * hE);
                const R cW = std::sqrt(g * hWe), cS = std::sqrt(g * hSn);
                const R ap = std::max(std::max(uE + cE, uWe + cW), R(0));
                const R am = std::min(std::min(uE - cE, uWe - cW), R(0));
                const R bp = std::max(std::max(vN + cN, vSn + cS), R(0));
                const R bm = std::min(std::min(vN - cN, vSn - cS), R(0));
                T4 xf, yf;
                xf.r = numflux(ap, am, hWe * uWe, hE * uE, hWe - hE);
                xf.g = numflux(ap, am, hWe * (uWe * uWe + half_g * hWe), hE * (uE * uE + half_g * hE),
                               hWe * uWe - hE * uE);
                xf.b = numflux(ap, am, hWe * uWe * vWe, hE * uE * vE, hWe * vWe - hE * vE);
                yf.r = numflux(bp, bm, hSn * vSn, hN * vN, hSn - hN);
                yf.g = numflux(bp, bm, hSn * uSn * vSn, hN * uN * vN, hSn * uSn - hN * uN);
                yf.b = numflux(bp, bm, hSn * (vSn * vSn + half_g * hSn), hN * (vN * vN + half_g * hN),
                               hSn * vSn - hN * vN);
                xflux[at(x, y)] = xf; yflux[at(x, y)] = yf;
                const T4 a2 = aux2[at(x, y)];
                T4 a1; a1.r = a2.r; a1.g = 0; a1.b = a2.b; a1.a = a2.a * decay_dt;
                aux1[at(x, y)] = a1;
            }
    }

    R friction_calc(R hu, R hv, R h) const {  // compute.hlsl:544-553
        R f = R(p.friction);
        const R h4 = t_pow(h, R(4));
        const R dbh = std::sqrt(R(2)) * h / std::sqrt(h4 + std::max(h4, eps));
        if (p.manning) {
            const R expo = std::is_same<R, float>::value ? R(0.3333f) : R(0.3333);
            f = g_() * R(p.friction) * R(p.friction) * t_pow(std::abs(dbh), expo);
        }
        return f * std::sqrt(hu * hu + hv * hv) * dbh * dbh;
    }

    // AdamsBashforthCoef and SecondOrder* (compute.hlsl:560-605)
    static void ab_coef(R a, R b, R c, R out[3]) {
        out[0] = (a / b) * ((2 * a + 6 * b + 3 * c) / (b + c)) + 6;
        out[1] = -(a / b) * ((2 * a + 3 * b + 3 * c) / (c));
        out[2] = (a / c) * ((2 * a + 3 * b) / (b + c));
    }
    static void second_order(R yn, R y1, R y2, R /*a*/, R b, R c, R out[3]) {
        R cr = (2 * b + c) / (b * (b + c)), cg = -(b + c) / (b * c), cb = (b) / (c * (b + c));
        out[0] = cr * yn + cg * y1 + cb * y2;
        cr = (c) / (b * (b + c)); cg = (b - c) / (b * c); cb = -(b) / (c * (b + c));
        out[1] = cr * yn + cg * y1 + cb * y2;
        cr = -(c) / (b * (b + c)); cg = (b + c) / (b * c); cb = -(b + 2 * c) / (c * (b + c));
        out[2] = cr * yn + cg * y1 + cb * y2;
    }

    // ---- Pass3Predictor (compute.hlsl:616-812), region [2,nx+2) x [2,ny+2) ----------------
    virtual void pass3(const std::vector<T4>& st, std::vector<T4>& out, std::vector<T4>& sgrad, std::vector<T4>& sfg) {
        const R g = g_();
        const R odx = R(1) / dx, ody = R(1) / dy;
        const R gdx = g / dx, gdy = g / dy;
        const R Bg = (std::is_same<R, float>::value ? R(1 / 15.0f) : R(1.0 / 15.0)) * g;
        const R sl = R(p.swl);
        const R dt = dt_(), dto = old_timestep, dtoo = old_old_timestep;
        const int ts = time_scheme;
        const std::vector<T4>& og = grad[old_i];
        const std::vector<T4>& oog = grad[oldold_i];
        const std::vector<T4>& ofg = fg[fg_old_i];
        const std::vector<T4>& oofg = fg[fg_oldold_i];
        std::fill(out.begin(), out.end(), T4());  // engine.cpp:1007 (reset new state to zero)
        const std::vector<T4>& A0 = ABCx[0];
        const std::vector<T4>& C0 = ABCy[0];
#pragma omp parallel for schedule(static)
        for (int y = 2; y < ny + 2; ++y)
            for (int x = 2; x < nx + 2; ++x) {
                const R BYh = BY[at(x, y)], BXh = BX[at(x, y)], BAh = BA[at(x, y)];
                const R BXw = BX[at(x - 1, y)], BYs = BY[at(x, y - 1)];
                const T4 c = st[at(x, y)], r = st[at(x + 1, y)], l = st[at(x - 1, y)];
                const T4 u = st[at(x, y + 1)], d = st[at(x, y - 1)];
                const T4 cx = A0[at(x, y)], cy = C0[at(x, y)];
                const R h = std::max(R(0), c.r - BAh);
                auto dep = [&](int xx, int yy) { return std::max(R(0), sl - BA[at(xx, yy)]); };
                const R dh = dep(x, y), d2 = dh * dh, d3 = d2 * dh;
                const R dl = dep(x - 1, y), dr = dep(x + 1, y), ddn = dep(x, y - 1), du = dep(x, y + 1);
                const R dll = dep(x - 2, y), drr = dep(x + 2, y), ddd = dep(x, y - 2), duu = dep(x, y + 2);
                auto eta = [&](int xx, int yy) { return st[at(xx, yy)].r - sl; };
                const R e0 = c.r - sl;
                const R el = eta(x - 1, y), er = eta(x + 1, y), ed = eta(x, y - 1), eu = eta(x, y + 1);
                const R ell = eta(x - 2, y), err = eta(x + 2, y), edd = eta(x, y - 2), euu = eta(x, y + 2);
                const R eul = eta(x - 1, y + 1), eur = eta(x + 1, y + 1), edl = eta(x - 1, y - 1), edr = eta(x + 1, y - 1);
                const T4 xh = xflux[at(x, y)], xw = xflux[at(x - 1, y)];
                const T4 yh = yflux[at(x, y)], ys = yflux[at(x, y - 1)];
                const R od2x = odx * odx, od3x = od2x * odx, od2y = ody * ody, od3y = od2y * ody;
                const R ddx = (-drr + 8 * dr - 8 * dl + dll) * odx / R(12);
                const R ddy = (-duu + 8 * du - 8 * ddn + ddd) * ody / R(12);
                const R exy = (R(0.25) * odx * ody * (eur - edr - eul + edl));
                const R exx = od2x * (er - 2 * e0 + el);
                const R eyy = od2y * (eu - 2 * e0 + ed);
                const R P1x = Bg * (d3) * ((err - 2 * er + 2 * el - ell) * (R(0.5) * od3x)
                                + (eur - eul - 2 * er + 2 * el + edr - edl) * (R(0.5) * odx * od2y));
                const R P2x = Bg * (d2) * (ddx * (2 * exx + eyy) + ddy * exy);
                const R P1y = Bg * (d3) * ((euu - 2 * eu + 2 * ed - edd) * (R(0.5) * od3y)
                                + (eur + eul - 2 * eu + 2 * ed - edr - edl) * (R(0.5) * ody * od2x));
                const R P2y = Bg * (d2) * (ddy * (exx + 2 * eyy) + ddx * exy);
                const R fr = friction_calc(c.g, c.b, h);
                const R s1 = -gdx * h * (BXh - BXw) - c.g * fr + (P1x + P2x);
                const R s2 = -gdy * h * (BYh - BYs) - c.b * fr + (P1y + P2y);
                R f0 = (xw.r - xh.r) * odx + (ys.r - yh.r) * ody + R(0);
                R f1 = (xw.g - xh.g) * odx + (ys.g - yh.g) * ody + s1;
                R f2 = (xw.b - xh.b) * odx + (ys.b - yh.b) * ody + s2;
                const R sixth = std::is_same<R, float>::value ? R(1.0f / 6.0f) : R(1.0 / 6.0);
                const R Fs = (sixth * dh * (ddx * ((ody / R(2)) * (u.b - d.b)) + (ddy * ((odx / R(2)) * (r.b - l.b)))));
                const R Gs = (sixth * dh * (ddx * ((ody / R(2)) * (u.g - d.g)) + (ddy * ((odx / R(2)) * (r.g - l.g)))));
                R wO = 0, huO = 0, hvO = 0;
                if (ts == EULER) {
                    wO = c.r + dt * f0;
                    huO = cx.r * l.g + cx.g * c.g + cx.b * r.g + dt * f1;
                    hvO = cy.r * d.b + cy.g * c.b + cy.b * u.b + dt * f2;
                } else {
                    const T4 o = og[at(x, y)], oo = oog[at(x, y)];
                    const T4 fo = ofg[at(x, y)], foo = oofg[at(x, y)];
                    if (ts == PREDICTOR) {
                        wO = c.r + dt / R(12) * (R(23) * f0 - R(16) * o.r + R(5) * oo.r);
                        huO = cx.r * l.g + cx.g * c.g + cx.b * r.g +
                              dt / R(12) * (R(23) * f1 - R(16) * o.g + R(5) * oo.g) +
                              (R(2) * Fs - R(3) * fo.r + foo.r);
                        hvO = cy.r * d.b + cy.g * c.b + cy.b * u.b +
                              dt / R(12) * (R(23) * f2 - R(16) * o.b + R(5) * oo.b) +
                              (R(2) * Gs - R(3) * fo.g + foo.g);
                    } else if (ts == PREDICTOR_ADAPTIVE) {
                        R cf[3], dF[3], dG[3];
                        ab_coef(dt, dto, dtoo, cf);
                        second_order(Fs, fo.r, foo.r, dt, dto, dtoo, dF);
                        second_order(Gs, fo.g, foo.g, dt, dto, dtoo, dG);
                        wO = c.r + dt / R(6) * (cf[0] * f0 + cf[1] * o.r + cf[2] * oo.r);
                        huO = cx.r * l.g + cx.g * c.g + cx.b * r.g +
                              dt / R(6) * (cf[0] * f1 + cf[1] * o.g + cf[2] * oo.g) +
                              dt / R(6) * (cf[0] * dF[0] + cf[1] * dF[1] + cf[2] * dF[2]);
                        hvO = cy.r * d.b + cy.g * c.b + cy.b * u.b +
                              dt / R(6) * (cf[0] * f2 + cf[1] * o.b + cf[2] * oo.b) +
                              dt / R(6) * (cf[0] * dG[0] + cf[1] * dG[1] + cf[2] * dG[2]);
                    } else {  // CORRECTOR
                        const T4 cc = cur[at(x, y)], cr = cur[at(x + 1, y)], cl = cur[at(x - 1, y)];
                        const T4 cu = cur[at(x, y + 1)], cd = cur[at(x, y - 1)];
                        const T4 pr = pred[at(x, y)], fp = fgpred[at(x, y)];
                        wO = cc.r + dt / R(24) * (9 * f0 + 19 * pr.r - 5 * o.r + 1 * oo.r);
                        huO = cx.r * cl.g + cx.g * cc.g + cx.b * cr.g +
                              dt / R(24) * (9 * f1 + 19 * pr.g - 5 * o.g + 1 * oo.g) + Fs - fp.r;
                        hvO = cy.r * cd.b + cy.g * cc.b + cy.b * cu.b +
                              dt / R(24) * (9 * f2 + 19 * pr.b - 5 * o.b + 1 * oo.b) + Gs - fp.g;
                    }
                }
                T4 ns; ns.r = wO; ns.g = huO; ns.b = hvO; ns.a = 0;
                out[at(x, y)] = ns;
                T4 gd; gd.r = f0; gd.g = f1; gd.b = f2; gd.a = 0;
                sgrad[at(x, y)] = gd;
                T4 fgv; fgv.r = Fs; fgv.g = Gs;
                sfg[at(x, y)] = fgv;
            }
    }

    // ---- Cyclic reduction (compute.hlsl:835-947, engine.cpp:1060-1217) --------------------
    virtual void cr_solve_x(const std::vector<T4>& rhs) {
        // reduce: D1x[k] from level k-1 (level-0 RHS is the new-state texture .g)
        for (int k = 1; k < Kx; ++k) {
            const int Wp = (k == 1) ? NX : lenx[k - 1] + 4, Wk = lenx[k] + 4;
            const std::vector<T4>& Dp = (k == 1) ? rhs : D1x[k - 1];
            const std::vector<T4>& Ap = ABCx[k - 1];
            std::vector<T4>& Dk = D1x[k];
#pragma omp parallel for schedule(static)
            for (int y = 2; y < ny + 2; ++y)
                for (int x2 = 2; x2 < lenx[k] + 2; ++x2) {
                    const int x1 = (x2 - 2) * 2 + 2 + 1;
                    const R dIn = Dp[size_t(y) * Wp + x1].g, dL = Dp[size_t(y) * Wp + x1 - 1].g;
                    const R dR = Dp[size_t(y) * Wp + x1 + 1].g;
                    const R aIn = Ap[size_t(y) * Wp + x1].r, cIn = Ap[size_t(y) * Wp + x1].b;
                    const R bL = Ap[size_t(y) * Wp + x1 - 1].g, bR = Ap[size_t(y) * Wp + x1 + 1].g;
                    const R k1 = aIn / bL, k2 = cIn / bR;
                    T4 o; o.g = dIn - dL * k1 - dR * k2;
                    Dk[size_t(y) * Wk + x2] = o;
                }
        }
        // substitute, from the coarsest level down (the coarsest reads a null texture = 0)
        for (int k = Kx - 1; k >= 0; --k) {
            const int Wk = (k == 0) ? NX : lenx[k] + 4;
            const int Wn = (k + 1 < Kx) ? lenx[k + 1] + 4 : 0;
            const std::vector<T4>& Dk = (k == 0) ? rhs : D1x[k];
            const std::vector<T4>& Ak = ABCx[k];
            std::vector<T4>& Xk = D1xc[k];
            const std::vector<T4>* Xn = (k + 1 < Kx) ? &D1xc[k + 1] : nullptr;
            const int Wa = lenx[k] + 4;
#pragma omp parallel for schedule(static)
            for (int y = 2; y < ny + 2; ++y)
                for (int x = 2; x < lenx[k] + 2; ++x) {
                    T4 o;
                    auto xn = [&](int xx) { return Xn ? (*Xn)[size_t(y) * Wn + xx].g : R(0); };
                    if (x % 2 == 1) {
                        o.g = xn(x / 2 + 1);
                    } else {
                        const R dIn = Dk[size_t(y) * Wk + x].g;
                        const T4 a = Ak[size_t(y) * Wa + x];
                        o.g = (dIn - a.r * xn(x / 2) - a.b * xn(x / 2 + 1)) / a.g;
                    }
                    Xk[size_t(y) * Wa + x] = o;
                }
        }
    }
    virtual void cr_solve_y(const std::vector<T4>& rhs) {
        for (int k = 1; k < Ky; ++k) {
            const std::vector<T4>& Dp = (k == 1) ? rhs : D1y[k - 1];
            const std::vector<T4>& Ap = ABCy[k - 1];
            std::vector<T4>& Dk = D1y[k];
#pragma omp parallel for schedule(static)
            for (int y2 = 2; y2 < leny[k] + 2; ++y2)
                for (int x = 2; x < nx + 2; ++x) {
                    const int y1 = (y2 - 2) * 2 + 2 + 1;
                    const R dIn = Dp[size_t(y1) * NX + x].b, dL = Dp[size_t(y1 - 1) * NX + x].b;
                    const R dR = Dp[size_t(y1 + 1) * NX + x].b;
                    const R aIn = Ap[size_t(y1) * NX + x].r, cIn = Ap[size_t(y1) * NX + x].b;
                    const R bL = Ap[size_t(y1 - 1) * NX + x].g, bR = Ap[size_t(y1 + 1) * NX + x].g;
                    const R k1 = aIn / bL, k2 = cIn / bR;
                    T4 o; o.b = dIn - dL * k1 - dR * k2;
                    Dk[size_t(y2) * NX + x] = o;
                }
        }
        for (int k = Ky - 1; k >= 0; --k) {
            const std::vector<T4>& Dk = (k == 0) ? rhs : D1y[k];
            const std::vector<T4>& Ak = ABCy[k];
            std::vector<T4>& Xk = D1yc[k];
            const std::vector<T4>* Xn = (k + 1 < Ky) ? &D1yc[k + 1] : nullptr;
#pragma omp parallel for schedule(static)
            for (int y = 2; y < leny[k] + 2; ++y)
                for (int x = 2; x < nx + 2; ++x) {
                    T4 o;
                    auto xn = [&](int yy) { return Xn ? (*Xn)[size_t(yy) * NX + x].b : R(0); };
                    if (y % 2 == 1) {
                        o.b = xn(y / 2 + 1);
                    } else {
                        const R dIn = Dk[size_t(y) * NX + x].b;
                        const T4 a = Ak[size_t(y) * NX + x];
                        o.b = (dIn - a.r * xn(y / 2) - a.b * xn(y / 2 + 1)) / a.g;
                    }
                    Xk[size_t(y) * NX + x] = o;
                }
        }
    }

    // ---- Boundaries (compute.hlsl:985-1309, engine.cpp:1236-1438) ---------------------------
    R sponge_fn(R L, R x) const { return R(0.5) + R(0.5) * t_cos(PI_ * std::max(L - x, R(0)) / L); }
    void sine_wave(R x, R y, R t, R d, R amp, R period, R th, R phase, R out[3]) const {
        const R omega = 2 * PI_ / period;
        const R k = omega * omega / (g_() * std::sqrt(t_tanh(omega * omega * d / g_())));
        const R c = omega / k;
        const R kx = t_cos(th) * x * k;
        const R ky = t_sin(th) * y * k;
        const R e = amp * t_sin(omega * t - kx - ky + phase);
        out[0] = e; out[1] = c * t_cos(th) * e; out[2] = c * t_sin(th) * e;
    }
    static bool inb(int x, int y, int NXX, int NYY) { return x >= 0 && y >= 0 && x < NXX && y < NYY; }

    // timeSeriesHelper (engine.cpp:1882-1904)
    void uts_value(const Boundary& b, int side, R t, R out[3]) {
        out[0] = out[1] = out[2] = 0;
        const int n = int(b.uts.size());
        int& it = uts_iter[side];
        while (it < n && R(b.uts[it][0]) < t) ++it;
        if (it >= n) return;
        const R t0 = R(b.uts[it - 1][0]), t1 = R(b.uts[it][0]);
        const R m = (t - t0) / (t1 - t0);
        for (int q = 0; q < 3; ++q) {
            const R v0 = R(b.uts[it - 1][q + 1]), v1 = R(b.uts[it][q + 1]);
            out[q] = v0 + (v1 - v0) * m;
        }
    }

    T4 tree_sum(const Boundary& b, R xx, R yy, R t, R dh, R sl, int nw, int lo, int size) const {
        T4 o;
        if (lo >= nw || !(dh > R(MIN_DEPTH))) { o.r = R(size) * sl; return o; }
        if (size == 1) {
            R res[3] = {0, 0, 0};
            sine_wave(xx, yy, t, dh, R(b.waves[lo][0]), R(b.waves[lo][1]), R(b.waves[lo][2]), R(b.waves[lo][3]), res);
            o.r = res[0] + sl; o.g = res[1]; o.b = res[2];
            return o;
        }
        const T4 a = tree_sum(b, xx, yy, t, dh, sl, nw, lo, size / 2);
        const T4 c = tree_sum(b, xx, yy, t, dh, sl, nw, lo + size / 2, size / 2);
        o.r = a.r + c.r; o.g = a.g + c.g; o.b = a.b + c.b;
        return o;
    }

    // One side: 0=N,1=E,2=S,3=W (engine.cpp:1339 naming).  Computes the strip from the state
    // as it is before this side (render-to-scratch), then writes the strip back.
    virtual void boundary_side(std::vector<T4>& st, int side) {
        const Boundary& b = side == 0 ? p.north : side == 1 ? p.east : side == 2 ? p.south : p.west;
        int x0, x1, y0, y1;
        if (side == 0) { x0 = 0; x1 = NX; y0 = NY - b.width; y1 = NY; }
        else if (side == 1) { x0 = NX - b.width; x1 = NX; y0 = 0; y1 = NY; }
        else if (side == 2) { x0 = 0; x1 = NX; y0 = 0; y1 = b.width; }
        else { x0 = 0; x1 = b.width; y0 = 0; y1 = NY; }
        x0 = std::max(x0, 0); y0 = std::max(y0, 0); x1 = std::min(x1, NX); y1 = std::min(y1, NY);
        if (x1 <= x0 || y1 <= y0) return;
        std::vector<T4> strip(size_t(x1 - x0) * (y1 - y0));
        const R sl = R(b.sea_level), g = g_(), dt = current_timestep, t = total_time;
        R utsv[3] = {0, 0, 0};
        if (b.type == B_UTS) {
            static const int uts_side_of[4] = {0, 1, 2, 3};
            uts_value(b, uts_side_of[side], t, utsv);
        }
        const int Kn = (side == 0 || side == 2) ? Ky : Kx;
        const int nleaf = 1 << (Kn - 1);
        for (int y = y0; y < y1; ++y)
            for (int x = x0; x < x1; ++x) {
                T4 o;
                if (b.type == B_SOLID) {
                    // compute.hlsl:985-1009: `4 - tex_idx` / `reflect - tex_idx` (reflect = 2n+2,
                    // engine.cpp:1308) with tex_idx = x + 0.5 at the pixel centre (engine.cpp:579),
                    // truncated toward zero by int3(): west/south read 3 - x, east/north 2n + 1 - x.
                    auto mirror = [](int c, int q) { return int(float(c) - (float(q) + 0.5f)); };
                    int sx = x, sy = y;
                    if (side == 3) sx = mirror(4, x);
                    else if (side == 1) sx = mirror(2 * nx + 2, x);
                    else if (side == 2) sy = mirror(4, y);
                    else sy = mirror(2 * ny + 2, y);
                    T4 s;
                    if (inb(sx, sy, NX, NY)) s = st[at(sx, sy)];
                    o.r = s.r;
                    o.g = (side == 1 || side == 3) ? -s.g : s.g;
                    o.b = (side == 0 || side == 2) ? -s.b : s.b;
                } else if (b.type == B_SPONGE) {
                    const R dh = std::max(R(MIN_DEPTH), sl - BA[at(x, y)]);
                    R L, dist;
                    if (side == 3) { L = R(b.width) * dx; dist = R(x) * dx; }
                    else if (side == 1) { L = R(b.width) * dx; dist = R(NX - x) * dx; }
                    else if (side == 2) { L = R(b.width) * dy; dist = R(y) * dy; }
                    else { L = R(b.width) * dy; dist = R(NY - y) * dy; }
                    const R gam = sponge_fn(L, dist) / sponge_fn(L, dist + std::sqrt(g * dh) * dt);
                    const T4 s = st[at(x, y)];
                    o.r = gam * (s.r - sl) + sl; o.g = gam * s.g; o.b = gam * s.b;
                } else if (b.type == B_SINEWAVE) {
                    const R dh = std::max(R(0), sl - BA[at(x, y)]);
                    R xx = R(x) * dx, yy = R(y) * dy;
                    if (side == 1) xx = R(x - NX) * dx;
                    if (side == 0) yy = R(y - NY) * dy;
                    R res[3] = {0, 0, 0};
                    if (dh > R(MIN_DEPTH)) sine_wave(xx, yy, t, dh, R(b.amplitude), R(b.period), R(b.theta), 0, res);
                    o.r = res[0] + sl; o.g = res[1]; o.b = res[2];
                } else if (b.type == B_UTS) {
                    o.r = utsv[0] + sl; o.g = utsv[1]; o.b = utsv[2];
                } else {  // B_IRREGULAR: one component per texel, pairwise tree sum
                    const bool colwise = (side == 1 || side == 3);
                    const int along = colwise ? y : x;
                    const int lim = colwise ? ny : nx;
                    if (along < 2 || along >= lim + 2) { o = T4(); }
                    else {
                        const R dh = std::max(R(0), sl - BA[at(x, y)]);
                        R xx = R(x) * dx, yy = R(y) * dy;
                        if (side == 1) xx = R(x - NX) * dx;
                        if (side == 0) yy = R(y - NY) * dy;
                        const int nw = int(b.waves.size());
                        // Balanced pairwise tree over 2^(K-1) components (ColumnSumReduce /
                        // RowSumReduce, compute.hlsl:1196-1212).  Subtrees made only of the
                        // constant component (sea level, 0, 0) sum exactly to size*sea level.
                        T4 tot = tree_sum(b, xx, yy, t, dh, sl, nw, 0, nleaf);
                        o.r = tot.r; o.g = tot.g; o.b = tot.b;
                    }
                }
                o.a = 0;
                strip[size_t(y - y0) * (x1 - x0) + (x - x0)] = o;
            }
        for (int y = y0; y < y1; ++y)
            for (int x = x0; x < x1; ++x) st[at(x, y)] = strip[size_t(y - y0) * (x1 - x0) + (x - x0)];
    }

    // ---- GetStats (compute.hlsl:1319-1378): one 4x4 block --------------------------------
    // o = {sum h, sum h(B+h/2), sum hu, sum hv, sum (hu u + hv v), max u^2+v^2, max h, max cfl,
    //      max (u^2+v^2)/h}
    virtual void stats_block(const std::vector<T4>& st, int bx, int by, R o[9]) const {
        const R g = g_(), odx = R(1) / dx, ody = R(1) / dy;
        R sh = 0, sb = 0, shu = 0, shv = 0, sk = 0, mu = 0, mh = 0, mc = 0, mf2 = 0;
        for (int j = 2; j < 6; ++j)
            for (int i = 2; i < 6; ++i) {
                const int x = bx * 4 + i, y = by * 4 + j;
                const T4 s = st[at(x, y)];
                const R B = BA[at(x, y)];
                const R h = std::max(R(0), s.r - B);
                const R c = std::sqrt(g * h);
                const R q = div_by_h(h);
                const R u = q * s.g, v = q * s.b;
                sh += h; sb += h * (B + R(0.5) * h); shu += s.g; shv += s.b;
                sk += (s.g * u + s.b * v);
                const R u2v2 = u * u + v * v;
                mu = std::max(mu, u2v2); mh = std::max(mh, h);
                mc = std::max(mc, (std::abs(u) + c) * odx);
                mc = std::max(mc, (std::abs(v) + c) * ody);
                mf2 = std::max(mf2, u2v2 * q);
            }
        o[0] = sh; o[1] = sb; o[2] = shu; o[3] = shv; o[4] = sk; o[5] = mu; o[6] = mh; o[7] = mc; o[8] = mf2;
    }

    // ---- resetTimestep (engine.cpp:1536-1756) ----------------------------------------------
    Stats reset_timestep() {
        const std::vector<T4>& st = state[sim_idx];
        const R g = g_();
        R mass = 0, xm = 0, ym = 0, ke = 0, pe = 0, ms = 0, md = 0, cfl = 0, mf = 0;
        for (int by = 0; by < ny / 4; ++by)
            for (int bx = 0; bx < nx / 4; ++bx) {
                R o[9];
                stats_block(st, bx, by, o);
                mass += o[0]; pe += o[1]; xm += o[2]; ym += o[3]; ke += o[4];
                ms = std::max(ms, o[5]); md = std::max(md, o[6]); cfl = std::max(cfl, o[7]); mf = std::max(mf, o[8]);
            }
        const R DENSITY = 1000;
        const R AREA = R(p.width) / R(nx - 1) * R(p.length) / R(ny - 1);
        mass *= DENSITY * AREA; xm *= DENSITY * AREA; ym *= DENSITY * AREA;
        ke *= R(0.5) * DENSITY * AREA; pe *= g * DENSITY * AREA;
        ms = std::sqrt(ms); mf /= g; mf = std::sqrt(mf);
        if (cfl > 0 && !target_cfl_set && p.adaptive) { target_cfl = double(dt_setting() * cfl); target_cfl_set = true; }
        if (!initialized_timesteps) {
            current_timestep = dt_setting();
            if (p.adaptive && !target_cfl_set) target_cfl = 0;
            cfl = (p.adaptive ? R(target_cfl) : R(0)) / current_timestep;
            old_old_timestep = current_timestep; old_timestep = current_timestep;
            initialized_timesteps = true;
        }
        if (time_scheme == PREDICTOR_ADAPTIVE) {
            const R tgt = std::max(R(target_cfl) / cfl, dt_setting() * R(float(p.min_timestep_ratio)));
            current_timestep = tgt > old_timestep ? R(p.ema_alpha) * tgt + (1 - R(p.ema_alpha)) * old_timestep : tgt;
        } else {
            current_timestep = dt_setting();
        }
        Stats out{};
        out.mass = double(mass); out.x_momentum = double(xm); out.y_momentum = double(ym);
        out.kinetic_energy = double(ke); out.potential_energy = double(pe); out.total_energy = double(ke + pe);
        out.max_speed = double(ms); out.max_depth = double(md); out.max_froude = double(mf);
        out.cfl_rate = double(cfl); out.cfl_number = double(cfl * current_timestep);
        out.timestep = double(current_timestep); out.total_time = double(total_time);
        double mfull = 0;
        for (int y = 2; y < ny + 2; ++y)
            for (int x = 2; x < nx + 2; ++x) mfull += std::max(0.0, double(st[at(x, y)].r) - double(BA[at(x, y)]));
        out.mass_full = mfull;
        return out;
    }

    // CopyFromXxAndXy (compute.hlsl:814-823) over the interior (engine.cpp:1219-1233)
    virtual void copy_from(std::vector<T4>& new_state) {
        for (int y = 2; y < ny + 2; ++y)
            for (int x = 2; x < nx + 2; ++x) {
                T4& s = new_state[at(x, y)];
                s.g = D1xc[0][at(x, y)].g;
                s.b = D1yc[0][at(x, y)].b;
                s.a = 0;
            }
    }

    // ---- timestep() (engine.cpp:849-1522): one pass ------------------------------------------
    void timestep() {
        std::vector<T4>& old_state = state[sim_idx];
        std::vector<T4>& new_state = state[1 - sim_idx];
        if (bootstrap_needed) { pass1(old_state); bootstrap_needed = false; }
        pass2();
        pass3(old_state, new_state, grad[scratch_i], fg[fg_scratch_i]);
        if (time_scheme == PREDICTOR || time_scheme == PREDICTOR_ADAPTIVE) {
            pred = grad[scratch_i];
            fgpred = fg[fg_scratch_i];
            cur = old_state;
        }
        cr_solve_x(new_state);
        cr_solve_y(new_state);
        copy_from(new_state);
        // Boundaries in the order East, North, West, South (engine.cpp:1342-1438)
        boundary_side(new_state, 1);
        boundary_side(new_state, 0);
        boundary_side(new_state, 3);
        boundary_side(new_state, 2);
        pass1(new_state);
        // Scheme switching and bookkeeping (engine.cpp:1476-1521)
        if (timestep_count >= 2) {
            if (correction_steps_count == p.correction_steps) {
                time_scheme = p.adaptive ? PREDICTOR_ADAPTIVE : PREDICTOR;
                correction_steps_count = 0;
            } else {
                time_scheme = CORRECTOR;
                correction_steps_count++;
            }
        }
        if (time_scheme == PREDICTOR || time_scheme == PREDICTOR_ADAPTIVE || time_scheme == EULER) {
            timestep_count++;
            // old <- scratch, old_old <- old, scratch <- old_old
            int o = old_i, oo = oldold_i, s = scratch_i;
            old_i = s; oldold_i = o; scratch_i = oo;
            o = fg_old_i; oo = fg_oldold_i; s = fg_scratch_i;
            fg_old_i = s; fg_oldold_i = o; fg_scratch_i = oo;
            old_old_timestep = old_timestep;
            old_timestep = current_timestep;
            total_time += current_timestep;
        }
        sim_idx = 1 - sim_idx;
        ++passes;
    }

    // One "physical" step = resetTimestep + timestep for the predictor (or Euler) pass and
    // for each corrector pass that follows it (main.cpp:383-430 with one step per frame).
    Stats physical_step() {
        Stats s = reset_timestep();
        timestep();
        while (time_scheme == CORRECTOR) { s = reset_timestep(); timestep(); }
        return s;
    }

    // newTerrainSettings -> fillTerrainTexture (engine.cpp:820-823, 3313-3379): the water depth of
    // every texel is kept (w - BA_old, then + BA_new), the bottom is sampled from the new grid,
    // both aux textures are reset (copied from a tridiagonal scratch level the engine never writes,
    // i.e. cleared), and the next pass re-bootstraps.  The tridiagonal coefficients are not rebuilt.
    virtual void new_terrain(const std::vector<float>& zgrid, int bnx, int bny) {
        std::vector<T4>& st = state[sim_idx];
        for (size_t k = 0; k < st.size(); ++k) st[k].r -= BA[k];
        std::vector<float> by, bx, ba;
        prepare_bottom(zgrid, bnx, bny, nx, ny, float(p.width), float(p.length), by, bx, ba);
        BY.assign(by.begin(), by.end()); BX.assign(bx.begin(), bx.end()); BA.assign(ba.begin(), ba.end());
        for (auto* t : {&aux1, &aux2}) t->assign(t->size(), T4());
        for (size_t k = 0; k < st.size(); ++k) st[k].r += BA[k];
        bootstrap_needed = true;
    }

    // AddSolitaryWave (compute.hlsl:949-976, engine.cpp:2154-2219); theta in degrees
    virtual void add_solitary_wave(double Hh, double theta_deg, double xc, double yc) {
        std::vector<T4>& st = state[sim_idx];
        const std::vector<T4> copy = st;
        const R th = R(theta_deg) * PI_ / R(180);
        for (int y = 1; y < ny + 3; ++y)
            for (int x = 1; x < nx + 3; ++x) {
                const T4 c = copy[at(x, y)];
                const R depth = std::max(c.r - BA[at(x, y)], R(0));
                const R K = std::sqrt(R(0.75) * std::abs(R(Hh)) / t_pow(depth, R(3)));
                const R C = std::sqrt(g_() * (R(Hh) + depth));
                const R ch = t_cosh(K * ((R(x) * dx - R(xc)) * t_cos(th) + (R(y) * dy - R(yc)) * t_sin(th)));
                const R e = R(Hh) * R(1) / t_pow(ch, R(2));
                T4 o = c; o.r = c.r + e; o.g = c.g + C * t_cos(th) * e; o.b = c.b + C * t_sin(th) * e; o.a = 0;
                st[at(x, y)] = o;
            }
    }
};

}  // namespace oracle
