// Irregular-wave components from a directional spectrum: the reference's generateSpectrumWaves
// (engine.cpp:3559-3776), host side.
//
// The reference builds a JONSWAP-shaped frequency spectrum (the TMA depth factor is computed
// but, as there, not applied), spreads it over directions with a cos^(2s) function whose
// spreading s depends on f/f_peak, normalises each frequency's directional weights, truncates the
// frequencies below 5 % of the peak of one direction column, and turns every (f, theta) cell
// into one sine component with amplitude sqrt(2 E dF) and a random phase.  This restatement
// keeps its grids, constants (pi as 3.1415) and index choices so that the same inputs give the
// same components, with two deliberate changes:
//   * phases come from a seeded generator (splitmix64) instead of srand(time(0)) / rand(), so a
//     run can be reproduced; they keep the reference's quantisation (r % 10000) / 10000 * 2 pi;
//   * log-gamma is std::lgamma (the reference uses boost::math::lgamma<float>).
// The arithmetic runs in double and is rounded to float wherever the reference stores a float.
#include "celeris_internal.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <string>
#include <vector>

namespace cel {

namespace {

uint64_t splitmix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

constexpr float kPi = 3.1415f;   // the generator's value of pi (engine.cpp:3597-3769)

}  // namespace

int spectrum_waves(const cel_spectrum& in, double gravity, unsigned long long seed, cel_boundary* b, const char* path,
                   std::string& err) {
    const float Hs_in = float(in.significant_waveheight), Tp = float(in.peak_period);
    const float theta_p = float(in.mean_theta), h = float(in.depth_at_source), g = float(gravity);
    if (h == 0.f || Tp == 0.f || Hs_in == 0.f) {
        err = "spectrum needs a nonzero significant wave height, peak period and source depth";
        return CEL_ERR_ARG;
    }
    const float gamma_s = 3.3f, spread_o = 50.0f, del_f0 = 0.005f, del_t = 5.0f, trunc = 0.05f;
    const float f_peak = 1.0f / Tp;
    const float Hs = std::min(Hs_in, h * 0.5f);   // at most half the source depth
    const float beta = float(0.0624 / (0.23 + 0.033 * double(gamma_s) - 0.185 / (1.9 + double(gamma_s))));

    // frequency grid f_peak +- 5 dF (float accumulation, as the reference's loop)
    std::vector<float> f;
    const float f_end = f_peak + 5 * del_f0;
    for (float v = std::max(del_f0, f_peak - 5 * del_f0); v <= f_end; v += del_f0) f.push_back(v);
    // direction grid mean +- 20 degrees in 5-degree steps
    std::vector<float> th;
    const float th_end = 20 + theta_p;
    for (float v = -20 + theta_p; v <= th_end; v += del_t) th.push_back(v);
    const size_t nf = f.size(), nt = th.size();
    if (nf < 3 || nt == 0) { err = "spectrum frequency grid has fewer than 3 entries"; return CEL_ERR_ARG; }

    // frequency spectrum (engine.cpp:3596-3618); the TMA factor phiK is not applied there either
    (void)g;
    std::vector<float> E(nf);
    for (size_t i = 0; i < nf; ++i) {
        const double fi = f[i], frat = double(f[i] / f_peak);
        const double sigma = f[i] <= f_peak ? 0.07 : 0.09;
        const double fr4 = frat * frat * frat * frat;
        E[i] = float(double(beta) * Hs * Hs / (fi * fr4) * std::exp(-1.25 / fr4) *
                     std::pow(double(gamma_s), std::exp(-(frat - 1.0) * (frat - 1.0) / (2.0 * sigma * sigma))));
    }
    // directional spreading (engine.cpp:3630-3648), each row normalised (3650-3659)
    std::vector<std::vector<float>> ED(nf, std::vector<float>(nt));
    for (size_t i = 0; i < nf; ++i) {
        const double frat = double(f[i] / f_peak);
        const double s = frat < 1.0 ? spread_o * std::pow(frat, 5.0) : spread_o * std::pow(frat, -2.5);
        const double beta_s = std::pow(2.0, 2 * s - 1) / kPi * std::exp(2 * std::lgamma(s + 1) - std::lgamma(2 * s + 1));
        float sum = 0.f;
        for (size_t j = 0; j < nt; ++j) {
            const double a = 0.5 * (double(th[j] - theta_p) * kPi / 180.0);
            ED[i][j] = float(beta_s * std::pow(std::cos(a), 2 * s));
            sum += ED[i][j];
        }
        for (size_t j = 0; j < nt; ++j) ED[i][j] = E[i] * (ED[i][j] / sum);
    }
    // total energy; the first frequency's width is taken from the 2nd and 3rd (engine.cpp:3672-3684)
    float Hmo = 0.f;
    for (size_t i = 0; i < nf; ++i) {
        const float dfi = i == 0 ? f[2] - f[1] : i == nf - 1 ? f[nf - 1] - f[nf - 2]
                                                           : (f[i + 1] - f[i]) / 2.0f + (f[i] - f[i - 1]) / 2.0f;
        for (size_t j = 0; j < nt; ++j) Hmo += ED[i][j] * dfi;
    }
    if (!(Hmo > 0.f)) { err = "spectrum has no energy"; return CEL_ERR_ARG; }
    // truncation at 5 % of the maximum of direction column floor(nt/2 + 0.5) (engine.cpp:3697-3723);
    // for the 9 directions this is column 5, one step past the mean direction
    const size_t jc = size_t(std::floor(double(nt) / 2.0 + 0.5));
    float max_E = ED[0][jc];
    for (size_t i = 0; i < nf; ++i) max_E = std::max(max_E, ED[i][jc]);
    const float min_E = trunc * max_E;
    std::vector<size_t> keep;
    for (size_t i = 0; i < nf; ++i)
        if (ED[i][jc] > min_E) keep.push_back(i);
    const size_t count = keep.size();
    if (count * nt > size_t(CEL_MAX_WAVES)) { err = "spectrum gives more components than a boundary holds"; return CEL_ERR_ARG; }
    // components (engine.cpp:3752-3772): the frequency width of kept entry k is taken at grid
    // position k of the full grid, as the reference indexes it
    uint64_t rng = seed;
    int n = 0;
    for (size_t k = 0; k < count; ++k) {
        const float dfk = k == 0 ? f[1] - f[0] : k == count - 1 ? f[count - 1] - f[count - 2]
                                                                : (f[k + 1] - f[k]) / 2.0f + (f[k] - f[k - 1]) / 2.0f;
        const size_t i = keep[k];
        for (size_t j = 0; j < nt; ++j) {
            const float amp = std::sqrt(2 * ED[i][j] * dfk);
            const float period = 1 / f[i];
            const float theta = float(double(th[j]) * 3.1415 / 180.0f);
            const float r = float(splitmix64(rng) % 10000) / 10000.0f;
            const float phase = float(double(r * 2) * 3.1415);
            b->waves[n][0] = amp;
            b->waves[n][1] = period;
            b->waves[n][2] = theta;
            b->waves[n][3] = phase;
            ++n;
        }
    }
    b->n_waves = n;
    if (path) {
        std::ofstream o(path, std::ios::out | std::ios::trunc);
        if (!o) { err = std::string("cannot open ") + path + " for writing"; return CEL_ERR_IO; }
        o << "[Hs] " << Hs_in << "\n" << "[Tp] " << Tp << "\n" << "[Theta_p] " << theta_p << "\n"
          << "[h_source] " << h << "\n" << "\n\n"
          << "# This file contains the sinewaves generated for the spectrum given above." << "\n\n"
          << "[NumberOfWaves] " << n << "\n" << "\n\n" << "====================================" << "\n";
        for (int k = 0; k < n; ++k)
            o << float(b->waves[k][0]) << "\t" << float(b->waves[k][1]) << "\t" << float(b->waves[k][2]) << "\t"
              << float(b->waves[k][3]) << "\n";
        if (!o) { err = std::string("write failed: ") + path; return CEL_ERR_IO; }
    }
    return CEL_OK;
}

}  // namespace cel
