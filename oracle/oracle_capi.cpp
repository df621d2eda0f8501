// C entry points of the CPU oracle (test infrastructure only).  Compiled twice:
// -DORACLE_REAL=double -> liboracle_f64.so (the correctness oracle) and
// -DORACLE_REAL=float -fopenmp -> liboracle_f32.so (the FP32 transcription / CPU baseline).
// Parameters arrive as the product's public `cel_params` struct so a test hands the very same
// value to the oracle and to the CUDA library.
#include "celeris_oracle.hpp"

#include "../include/celeris_b200.h"

#include <chrono>
#ifdef _OPENMP
#include <omp.h>
#endif
#include <cstdio>
#include <memory>

#ifndef ORACLE_REAL
#define ORACLE_REAL double
#endif

using Real = ORACLE_REAL;
#ifdef ORACLE_REF_SHADER
// The reference's shader code driven by the oracle's schedule (built by ref_build.py).
#include "ref_engine.hpp"
using Eng = refshader::RefEngine;
#else
using Eng = oracle::Engine<Real>;
#endif

namespace {

oracle::Boundary conv_boundary(const cel_boundary& b) {
    oracle::Boundary o;
    o.type = b.type;
    o.width = b.width;
    o.sea_level = b.sea_level;
    o.amplitude = b.amplitude;
    o.period = b.period;
    o.theta = b.theta;
    for (int i = 0; i < b.n_waves && i < CEL_MAX_WAVES; ++i)
        o.waves.push_back({b.waves[i][0], b.waves[i][1], b.waves[i][2], b.waves[i][3]});
    for (int i = 0; i < b.n_uts; ++i)
        o.uts.push_back({b.uts[4 * i], b.uts[4 * i + 1], b.uts[4 * i + 2], b.uts[4 * i + 3]});
    return o;
}

oracle::Params conv_params(const cel_params& c) {
    oracle::Params p;
    p.nx = c.nx; p.ny = c.ny;
    p.width = c.width; p.length = c.length; p.swl = c.still_water_elevation;
    p.boussinesq = c.boussinesq != 0;
    p.epsilon = c.epsilon; p.theta = c.theta;
    p.correction_steps = c.correction_steps;
    p.timestep = c.timestep;
    p.adaptive = c.adaptive != 0;
    p.ema_alpha = c.ema_alpha; p.min_timestep_ratio = c.min_timestep_ratio;
    p.manning = c.manning != 0; p.friction = c.friction;
    p.gravity = c.gravity;
    p.dissipation_threshold = c.dissipation_threshold;
    p.whitewater_decay = c.whitewater_decay;
    p.west = conv_boundary(c.west); p.east = conv_boundary(c.east);
    p.south = conv_boundary(c.south); p.north = conv_boundary(c.north);
    for (int i = 0; i < c.n_solitons && i < CEL_MAX_SOLITONS; ++i)
        p.solitons.push_back({c.solitons[i].H, c.solitons[i].theta, c.solitons[i].xc, c.solitons[i].yc,
                              c.solitons[i].length});
    return p;
}

void to_stats(const oracle::Stats& s, const Eng& e, cel_stats* o) {
    if (!o) return;
    o->mass = s.mass; o->x_momentum = s.x_momentum; o->y_momentum = s.y_momentum;
    o->kinetic_energy = s.kinetic_energy; o->potential_energy = s.potential_energy;
    o->total_energy = s.total_energy; o->max_speed = s.max_speed; o->max_depth = s.max_depth;
    o->max_froude = s.max_froude; o->cfl_rate = s.cfl_rate; o->cfl_number = s.cfl_number;
    o->timestep = s.timestep; o->total_time = s.total_time; o->mass_full = s.mass_full;
    o->time_scheme = e.time_scheme; o->health = 0;
}

}  // namespace

extern "C" {

void* orc_create(const cel_params* p, const float* bathy, int bnx, int bny, const float* hot_w_hu_hv) {
    auto* e = new Eng();
    std::vector<float> z(bathy, bathy + size_t(bnx) * bny);
    oracle::Params prm = conv_params(*p);
    if (hot_w_hu_hv) {
        std::vector<float> hot(hot_w_hu_hv, hot_w_hu_hv + size_t(p->nx + 4) * (p->ny + 4) * 3);
        e->init(prm, z, bnx, bny, &hot);
    } else {
        e->init(prm, z, bnx, bny, nullptr);
    }
    return e;
}

void orc_destroy(void* h) { delete static_cast<Eng*>(h); }

int orc_real_bytes(void) { return int(sizeof(Real)); }

void orc_reset_timestep(void* h, cel_stats* out) {
    Eng* e = static_cast<Eng*>(h);
    oracle::Stats s = e->reset_timestep();
    to_stats(s, *e, out);
}

void orc_timestep(void* h) { static_cast<Eng*>(h)->timestep(); }

// n passes, each preceded by resetTimestep (main.cpp:383-430).  Returns the last stats.
void orc_timesteps(void* h, int n, cel_stats* out) {
    Eng* e = static_cast<Eng*>(h);
    oracle::Stats s{};
    for (int i = 0; i < n; ++i) { s = e->reset_timestep(); e->timestep(); }
    to_stats(s, *e, out);
}

// n physical steps; returns the stats taken before the last step's first pass.
void orc_physical_steps(void* h, int n, cel_stats* out) {
    Eng* e = static_cast<Eng*>(h);
    oracle::Stats s{};
    for (int i = 0; i < n; ++i) s = e->physical_step();
    to_stats(s, *e, out);
}

// State texture (w, hu, hv, a) of the current state as double, (nx+4)*(ny+4)*4.
void orc_get_state(void* h, double* out) {
    Eng* e = static_cast<Eng*>(h);
    const auto& st = e->state[e->sim_idx];
    for (size_t i = 0; i < st.size(); ++i) {
        out[4 * i] = double(st[i].r); out[4 * i + 1] = double(st[i].g);
        out[4 * i + 2] = double(st[i].b); out[4 * i + 3] = double(st[i].a);
    }
}

void orc_set_state(void* h, const double* in) {
    Eng* e = static_cast<Eng*>(h);
    auto& st = e->state[e->sim_idx];
    for (size_t i = 0; i < st.size(); ++i) {
        st[i].r = Real(in[4 * i]); st[i].g = Real(in[4 * i + 1]);
        st[i].b = Real(in[4 * i + 2]); st[i].a = Real(in[4 * i + 3]);
    }
    e->bootstrap_needed = true;
}

// txAuxiliary1 (maxdepth, 0, max_sd2, breaking), (nx+4)*(ny+4)*4
void orc_get_aux(void* h, double* out) {
    Eng* e = static_cast<Eng*>(h);
    for (size_t i = 0; i < e->aux1.size(); ++i) {
        out[4 * i] = double(e->aux1[i].r); out[4 * i + 1] = double(e->aux1[i].g);
        out[4 * i + 2] = double(e->aux1[i].b); out[4 * i + 3] = double(e->aux1[i].a);
    }
}

void orc_get_bottom(void* h, double* out) {
    Eng* e = static_cast<Eng*>(h);
    for (size_t i = 0; i < e->BA.size(); ++i) {
        out[3 * i] = double(e->BY[i]); out[3 * i + 1] = double(e->BX[i]); out[3 * i + 2] = double(e->BA[i]);
    }
}

// Level-0 tridiagonal coefficients {A,B,C} for x and y, (nx+4)*(ny+4)*3 each
void orc_get_coefs(void* h, double* ax, double* ay) {
    Eng* e = static_cast<Eng*>(h);
    for (size_t i = 0; i < e->ABCx[0].size(); ++i) {
        ax[3 * i] = double(e->ABCx[0][i].r); ax[3 * i + 1] = double(e->ABCx[0][i].g); ax[3 * i + 2] = double(e->ABCx[0][i].b);
        ay[3 * i] = double(e->ABCy[0][i].r); ay[3 * i + 1] = double(e->ABCy[0][i].g); ay[3 * i + 2] = double(e->ABCy[0][i].b);
    }
}

int orc_time_scheme(void* h) { return static_cast<Eng*>(h)->time_scheme; }
double orc_total_time(void* h) { return double(static_cast<Eng*>(h)->total_time); }
int orc_passes(void* h) { return static_cast<Eng*>(h)->passes; }

// The next pass recomputes the Pass1 faces from the current state (what the fused forms, which keep
// no Pass1 textures, do after any change of state).
void orc_rebootstrap(void* h) { static_cast<Eng*>(h)->bootstrap_needed = true; }

void orc_new_terrain(void* h, const float* bathy, int bnx, int bny) {
    static_cast<Eng*>(h)->new_terrain(std::vector<float>(bathy, bathy + size_t(bnx) * bny), bnx, bny);
}

void orc_add_solitary_wave(void* h, double H, double theta_deg, double xc, double yc) {
    static_cast<Eng*>(h)->add_solitary_wave(H, theta_deg, xc, yc);
}

// Solve one tridiagonal row with the engine's CR path on a synthetic system (tests).
// a,b,c,d: n entries each; x: n outputs.  Uses the same level recursion as cr_solve_x.
void orc_cr_solve(int n, const double* a, const double* b, const double* c, const double* d, double* x) {
    // Build a minimal engine-like structure: one row, texture widths len_k + 4.
    std::vector<int> len;
    int L = n;
    const int K = oracle::count_of_matrices(n);
    for (int k = 0; k < K; ++k) { len.push_back(L); L /= 2; }
    std::vector<std::vector<Real>> A(K), B(K), C(K), D(K), X(K);
    for (int k = 0; k < K; ++k) {
        A[k].assign(len[k] + 4, 0); B[k].assign(len[k] + 4, 1); C[k].assign(len[k] + 4, 0);
        D[k].assign(len[k] + 4, 0); X[k].assign(len[k] + 4, 0);
    }
    for (int i = 0; i < n; ++i) { A[0][i + 2] = Real(a[i]); B[0][i + 2] = Real(b[i]); C[0][i + 2] = Real(c[i]); D[0][i + 2] = Real(d[i]); }
    A[0][2] = 0; C[0][n + 1] = 0;
    for (int k = 1; k < K; ++k)
        for (int j = 2; j < len[k] + 2; ++j) {
            const int pj = (j - 2) * 2 + 3;
            const Real k1 = A[k - 1][pj] / B[k - 1][pj - 1], k2 = C[k - 1][pj] / B[k - 1][pj + 1];
            A[k][j] = -A[k - 1][pj - 1] * k1;
            B[k][j] = B[k - 1][pj] - C[k - 1][pj - 1] * k1 - A[k - 1][pj + 1] * k2;
            C[k][j] = -C[k - 1][pj + 1] * k2;
            D[k][j] = D[k - 1][pj] - D[k - 1][pj - 1] * k1 - D[k - 1][pj + 1] * k2;
        }
    for (int k = K - 1; k >= 0; --k)
        for (int j = 2; j < len[k] + 2; ++j) {
            auto xn = [&](int q) { return (k + 1 < K) ? X[k + 1][q] : Real(0); };
            if (j % 2 == 1) X[k][j] = xn(j / 2 + 1);
            else X[k][j] = (D[k][j] - A[k][j] * xn(j / 2) - C[k][j] * xn(j / 2 + 1)) / B[k][j];
        }
    for (int i = 0; i < n; ++i) x[i] = double(X[0][i + 2]);
}

// Wall-clock timing of n physical steps (CPU baseline); returns seconds.
double orc_time_physical_steps(void* h, int n) {
    Eng* e = static_cast<Eng*>(h);
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < n; ++i) e->physical_step();
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
