// Once-per-remesh host work: staggered bottom, tridiagonal coefficients (all CR levels),
// initial condition, and Thomas factors for the fused solver.  This is the host-side part of
// the reference's remesh() (engine.cpp:726-737): UpdateTerrainHeightfield
// (terrain_heightfield.cpp:244-297), createTridiagonalCoefTextures (engine.cpp:2612-2887) and
// createSimTextures (engine.cpp:2890-3016).  Bottom and coefficients are computed in float
// with the reference's operation order, so every form starts from the reference's values.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "celeris_internal.hpp"

namespace cel {

int count_of_matrices(int n) {  // st_getCountOfMatrices (engine.cpp:741-748)
    int c = 1;
    while (n > 1) { n /= 2; ++c; }
    return c;
}

namespace {

float sample(const float* z, int bnx, int bny, float W, float L, float x, float y) {
    // getBathymetry (terrain_heightfield.cpp:213-242): grid spans x in [-W/2, W/2], y in [0, L]
    x = (x + W / 2) / W * (bnx - 1);
    y = y / L * (bny - 1);
    x = x < 0 ? 0.f : x;
    x = x > bnx - 1 ? float(bnx - 1) : x;
    y = y < 0 ? 0.f : y;
    y = y > bny - 1 ? float(bny - 1) : y;
    const int x0 = int(std::floor(x)), x1 = int(std::ceil(x));
    const int y0 = int(std::floor(y)), y1 = int(std::ceil(y));
    const float fx = x - x0, fy = y - y0;
    const float* r0 = z + size_t(y0) * bnx;
    const float* r1 = z + size_t(y1) * bnx;
    const float lo = r0[x0] + fx * (r0[x1] - r0[x0]);
    const float hi = r1[x0] + fx * (r1[x1] - r1[x0]);
    return lo + fy * (hi - lo);
}

}  // namespace

float terrain_height(const HostSetup& s, float W, float L, float x, float y) {
    const int width = s.nx, height = s.ny;
    x = (x + W / 2) / W * float(width - 1);
    y = y / L * float(height - 1);
    x = x < 0 ? 0.f : (x > float(width - 1) ? float(width - 1) : x);
    y = y < 0 ? 0.f : (y > float(height - 1) ? float(height - 1) : y);
    x += 2;
    y += 2;
    const int xd = int(std::floor(x)), xu = int(std::ceil(x)), yd = int(std::floor(y)), yu = int(std::ceil(y));
    const float xf = x - float(xd), yf = y - float(yd);
    const int pitch = width + 4;
    auto B = [&](int xx, int yy) { return s.BA[size_t(yy) * pitch + xx]; };
    auto lerp = [](float t, float dn, float up) { return dn + t * (up - dn); };
    return lerp(yf, lerp(xf, B(xd, yd), B(xu, yd)), lerp(xf, B(xd, yu), B(xu, yu)));
}

void water_height_block(int nx, int ny, float W, float L, float x, float y, int& ix, int& iy) {
    const float tx = (x + W / 2) / W, ty = y / L;
    ix = int(tx * float(nx / 4));
    iy = int(ty * float(ny / 4));
    ix = ix < 0 ? 0 : (ix > nx / 4 - 1 ? nx / 4 - 1 : ix);
    iy = iy < 0 ? 0 : (iy > ny / 4 - 1 ? ny / 4 - 1 : iy);
}

void prepare_bottom(const float* z, int bnx, int bny, int nx, int ny, float W, float L, HostSetup& s) {
    const int NX = nx + 4, NY = ny + 4;
    s.corners.assign(size_t(NX + 1) * (NY + 1), 0.f);
    for (int j = 0; j <= NY; ++j) {
        const float y = (float(j) - 2.5f) / float(ny - 1) * L;
        for (int i = 0; i <= NX; ++i) {
            const float x = (float(i) - 2.5f) / float(nx - 1) * W - (W / 2);
            s.corners[size_t(j) * (NX + 1) + i] = sample(z, bnx, bny, W, L, x, y);
        }
    }
    // Each texel's BA is the mean of its four corners and BX / BY the means of its east / north
    // corner pairs, summed in the order the reference's corner loop visits them.
    s.BY.assign(size_t(NX) * NY, 0.f);
    s.BX.assign(size_t(NX) * NY, 0.f);
    s.BA.assign(size_t(NX) * NY, 0.f);
    const int cp = NX + 1;
    for (int j = 0; j < NY; ++j)
        for (int i = 0; i < NX; ++i) {
            const float z00 = s.corners[size_t(j) * cp + i], z10 = s.corners[size_t(j) * cp + i + 1];
            const float z01 = s.corners[size_t(j + 1) * cp + i], z11 = s.corners[size_t(j + 1) * cp + i + 1];
            float ba = 0.25f * z00;
            ba += 0.25f * z10;
            ba += 0.25f * z01;
            ba += 0.25f * z11;
            float bx = 0.5f * z10;
            bx += 0.5f * z11;
            float by = 0.5f * z01;
            by += 0.5f * z11;
            s.BA[size_t(j) * NX + i] = ba;
            s.BX[size_t(j) * NX + i] = bx;
            s.BY[size_t(j) * NX + i] = by;
        }
}

void build_cr_levels(const cel_params& p, HostSetup& s) {
    const int nx = s.nx, ny = s.ny, NX = s.NX, NY = s.NY;
    const float BCOEF = 1 / 15.0f;
    const float dx2 = s.dx * s.dx, dy2 = s.dy * s.dy;
    const float sl = p.boussinesq ? float(p.still_water_elevation) : -9999.f;
    auto depth = [&](int x, int y) { return std::max(0.0f, sl - s.BA[size_t(y) * NX + x]); };
    s.Kx = count_of_matrices(nx);
    s.Ky = count_of_matrices(ny);
    s.lenx.assign(s.Kx, 0);
    s.leny.assign(s.Ky, 0);
    for (int k = 0, L = nx; k < s.Kx; ++k, L /= 2) s.lenx[k] = L;
    for (int k = 0, L = ny; k < s.Ky; ++k, L /= 2) s.leny[k] = L;
    const Float4 unit = {0.f, 1.f, 0.f, 0.f};
    s.ABCx.assign(s.Kx, {});
    s.ABCy.assign(s.Ky, {});
    // x direction, level 0: one system per row over the interior columns
    s.ABCx[0].assign(size_t(NX) * NY, unit);
    for (int y = 0; y < NY; ++y) {
        const int yy = std::max(2, std::min(ny + 1, y));
        for (int x = 2; x <= NX - 3; ++x) {
            const float d = depth(x, yy);
            const float K1 = (BCOEF + 1 / 3.0f) * (d * d / dx2);
            const float K2 = (d / dx2) * (-depth(x + 2, yy) + 8 * depth(x + 1, yy) - 8 * depth(x - 1, yy) + depth(x - 2, yy));
            Float4& c = s.ABCx[0][size_t(y) * NX + x];
            c.x = (x == 2) ? 0.f : -K1 + K2 / 72.0f;
            c.y = 1 + 2 * K1;
            c.z = (x == NX - 3) ? 0.f : -(K1 + K2 / 72.0f);
        }
    }
    // y direction, level 0: one system per column over the interior rows
    s.ABCy[0].assign(size_t(NX) * NY, unit);
    for (int y = 2; y <= NY - 3; ++y)
        for (int x = 0; x < NX; ++x) {
            const int xx = std::max(2, std::min(nx + 1, x));
            const float d = depth(xx, y);
            const float K1 = (BCOEF + 1 / 3.0f) * (d * d / dy2);
            const float K2 = (d / dy2) * (-depth(xx, y + 2) + 8 * depth(xx, y + 1) - 8 * depth(xx, y - 1) + depth(xx, y - 2));
            Float4& c = s.ABCy[0][size_t(y) * NX + x];
            c.x = (y == 2) ? 0.f : -K1 + K2 / 72.0f;
            c.y = 1 + 2 * K1;
            c.z = (y == NY - 3) ? 0.f : -(K1 + K2 / 72.0f);
        }
    // Reduced levels: equation m' of level k is odd equation 2m'+1 of level k-1 with its
    // neighbours eliminated.
    auto reduce = [](const Float4& lo, const Float4& mid, const Float4& hi) {
        const float k1 = mid.x / lo.y, k2 = mid.z / hi.y;
        Float4 o;
        o.x = -lo.x * k1;
        o.y = mid.y - lo.z * k1 - hi.x * k2;
        o.z = -hi.z * k2;
        o.w = 0.f;
        return o;
    };
    for (int k = 1; k < s.Kx; ++k) {
        const int Wp = s.lenx[k - 1] + 4, Wk = s.lenx[k] + 4;
        s.ABCx[k].assign(size_t(Wk) * NY, unit);
        for (int y = 0; y < NY; ++y)
            for (int x = 2; x < Wk - 2; ++x) {
                const int q = (x - 2) * 2 + 3;
                const Float4* row = &s.ABCx[k - 1][size_t(y) * Wp];
                s.ABCx[k][size_t(y) * Wk + x] = reduce(row[q - 1], row[q], row[q + 1]);
            }
    }
    for (int k = 1; k < s.Ky; ++k) {
        const int Hk = s.leny[k] + 4;
        s.ABCy[k].assign(size_t(NX) * Hk, unit);
        for (int y = 2; y < Hk - 2; ++y) {
            const int q = (y - 2) * 2 + 3;
            for (int x = 0; x < NX; ++x)
                s.ABCy[k][size_t(y) * NX + x] = reduce(s.ABCy[k - 1][size_t(q - 1) * NX + x],
                                                       s.ABCy[k - 1][size_t(q) * NX + x],
                                                       s.ABCy[k - 1][size_t(q + 1) * NX + x]);
        }
    }
}

void initial_condition(const cel_params& p, const std::vector<float>* hot, HostSetup& s) {
    const int nx = s.nx, ny = s.ny, NX = s.NX, NY = s.NY;
    const float swl = float(p.still_water_elevation);
    const float g = float(p.gravity);
    const float PI = 4.0f * std::atan(1.0f);
    s.ic.assign(size_t(NX) * NY * 3, 0.f);
    for (int j = 0; j < NY; ++j)
        for (int i = 0; i < NX; ++i) {
            const int ii = std::max(2, std::min(nx + 1, i)), jj = std::max(2, std::min(ny + 1, j));
            const float B = s.BA[size_t(jj) * NX + ii];
            const float depth = std::max(0.0f, swl - B);
            float w, hu, hv;
            const size_t k = (size_t(j) * NX + i) * 3;
            if (hot) { w = (*hot)[k]; hu = (*hot)[k + 1]; hv = (*hot)[k + 2]; }
            else { w = std::max(swl, B); hu = 0; hv = 0; }
            for (int q = 0; q < p.n_solitons; ++q) {
                const cel_soliton& sw = p.solitons[q];
                if (sw.H == 0) continue;
                // Over a dry cell the sech^2 profile tends to 0; the reference's formula gives
                // 0 * sqrt(0/0) = NaN there for a zero-height taper, so the term is skipped.
                if (depth == 0) continue;
                const float th = float(sw.theta), H = float(sw.H), xc = float(sw.xc), yc = float(sw.yc);
                const float len = float(sw.length);
                const float xs = s.dx * float(i), ys = s.dy * float(j);
                const float dist = std::fabs(std::sin(th) * (xs - xc)) + std::fabs(std::cos(th) * (ys - yc));
                float Hq = H;
                if (dist > len / 2.0f) {
                    // cosine taper beyond a finite crest (engine.cpp:2972-3003)
                    const float smooth = PI / std::sqrt(0.75f * H / (depth * depth * depth));
                    Hq = (dist - len / 2.0f < smooth) ? H * (0.5f * std::cos(PI / smooth * (dist - len / 2.0f)) + 0.5f) : 0.f;
                }
                const float K = std::sqrt(0.75f * std::fabs(Hq) / (depth * depth * depth));
                const float C = std::sqrt(g * (Hq + depth));
                const float ch = std::cosh(K * ((xs - xc) * std::cos(th) + (ys - yc) * std::sin(th)));
                const float eta = Hq * 1.0f / (ch * ch);
                w += eta;
                hu += C * std::cos(th) * eta;
                hv += C * std::sin(th) * eta;
            }
            s.ic[k] = w; s.ic[k + 1] = hu; s.ic[k + 2] = hv;
        }
    // The same initial condition evaluated in double precision: the mixed form starts from it as
    // a (high, low) pair of floats, so its first state is the double-precision one to ~1e-15.
    const double swl64 = p.still_water_elevation, g64 = p.gravity, PI64 = 3.14159265358979323846;
    const double dx64 = p.width / double(nx - 1), dy64 = p.length / double(ny - 1);
    s.ic64.assign(size_t(NX) * NY * 3, 0.0);
    for (int j = 0; j < NY; ++j)
        for (int i = 0; i < NX; ++i) {
            const int ii = std::max(2, std::min(nx + 1, i)), jj = std::max(2, std::min(ny + 1, j));
            const double B = s.BA[size_t(jj) * NX + ii];
            const double depth = std::max(0.0, swl64 - B);
            const size_t k = (size_t(j) * NX + i) * 3;
            double w, hu, hv;
            if (hot) { w = (*hot)[k]; hu = (*hot)[k + 1]; hv = (*hot)[k + 2]; }
            else { w = std::max(swl64, B); hu = 0; hv = 0; }
            for (int q = 0; q < p.n_solitons; ++q) {
                const cel_soliton& sw = p.solitons[q];
                if (sw.H == 0 || depth == 0) continue;
                const double th = sw.theta, x = dx64 * i, y = dy64 * j;
                const double dist = std::fabs(std::sin(th) * (x - sw.xc)) + std::fabs(std::cos(th) * (y - sw.yc));
                double Hq = sw.H;
                if (dist > sw.length / 2) {
                    const double smooth = PI64 / std::sqrt(0.75 * sw.H / (depth * depth * depth));
                    Hq = (dist - sw.length / 2 < smooth) ? sw.H * (0.5 * std::cos(PI64 / smooth * (dist - sw.length / 2)) + 0.5)
                                                         : 0.0;
                }
                const double K = std::sqrt(0.75 * std::fabs(Hq) / (depth * depth * depth));
                const double C = std::sqrt(g64 * (Hq + depth));
                const double ch = std::cosh(K * ((x - sw.xc) * std::cos(th) + (y - sw.yc) * std::sin(th)));
                const double eta = Hq / (ch * ch);
                w += eta;
                hu += C * std::cos(th) * eta;
                hv += C * std::sin(th) * eta;
            }
            s.ic64[k] = w; s.ic64[k + 1] = hu; s.ic64[k + 2] = hv;
        }
}

int make_setup(const cel_params& p, const float* bathy, int bnx, int bny, HostSetup& s, std::string& err) {
    if (p.nx < 2 || p.ny < 2) { err = "nx and ny must be >= 2"; return CEL_ERR_ARG; }
    if (p.nx > 32768 || p.ny > 32768) { err = "nx and ny must be <= 32768 (15 CR levels)"; return CEL_ERR_ARG; }
    if (!(p.width > 0) || !(p.length > 0)) { err = "width and length must be > 0"; return CEL_ERR_ARG; }
    for (const cel_boundary* b : {&p.west, &p.east, &p.south, &p.north}) {
        if (b->type < 0 || b->type > 4) { err = "unknown boundary type"; return CEL_ERR_ARG; }
        if (b->width < 0) { err = "negative boundary width"; return CEL_ERR_ARG; }
        if (b->type == CEL_BC_UTS && b->n_uts < 2) { err = "UniformTimeSeries boundary needs >= 2 rows"; return CEL_ERR_ARG; }
        if (b->type == CEL_BC_IRREGULAR && (b->n_waves < 0 || b->n_waves > CEL_MAX_WAVES)) { err = "bad n_waves"; return CEL_ERR_ARG; }
        if (b->type == CEL_BC_SINEWAVE && !(b->period > 0)) { err = "SineWave period must be > 0"; return CEL_ERR_ARG; }
    }
    s.nx = p.nx; s.ny = p.ny; s.NX = p.nx + 4; s.NY = p.ny + 4;
    std::vector<float> zf;
    if (!bathy) {
        const int st = read_cbf(p.bathymetry_path, &zf, bnx, bny, err);
        if (st) return st;
        bathy = zf.data();
    }
    if (bnx < 2 || bny < 2) { err = "bathymetry grid must be at least 2x2"; return CEL_ERR_ARG; }
    const float W = float(p.width), L = float(p.length);
    prepare_bottom(bathy, bnx, bny, p.nx, p.ny, W, L, s);
    s.dx = W / float(p.nx - 1);
    s.dy = L / float(p.ny - 1);
    {   // CalcEpsilon (engine.cpp:290-299)
        const float m = std::max(s.dx, s.dy);
        s.eps = std::min(float(p.epsilon), m * m * m * m);
    }
    build_cr_levels(p, s);
    std::vector<float> hot;
    if (p.hotstart_path[0]) {
        const int st = read_hotstart(p.hotstart_path, p.nx, p.ny, hot, err);
        if (st) return st;
    }
    initial_condition(p, p.hotstart_path[0] ? &hot : nullptr, s);
    return CEL_OK;
}

// Thomas factorisation of each level-0 system: for x in the system,
//   den_i = b_i - a_i * c'_{i-1},  c'_i = c_i / den_i,  inv_i = 1 / den_i,  m_i = -a_i * inv_i
// so that forward elimination is d'_i = inv_i * d_i + m_i * d'_{i-1} and back substitution is
// x_i = d'_i - c'_i x_{i+1}.  Computed in double, stored in float.
void thomas_factors_x(const HostSetup& s, std::vector<float>& cp, std::vector<float>& inv, std::vector<float>& m) {
    const size_t n = size_t(s.NX) * s.NY;
    cp.assign(n, 0.f); inv.assign(n, 0.f); m.assign(n, 0.f);
    for (int y = 2; y < s.ny + 2; ++y) {
        double cprev = 0;
        for (int x = 2; x < s.nx + 2; ++x) {
            const Float4& c = s.ABCx[0][size_t(y) * s.NX + x];
            const double den = double(c.y) - double(c.x) * cprev;
            const double iv = 1.0 / den;
            cprev = double(c.z) * iv;
            cp[size_t(y) * s.NX + x] = float(cprev);
            inv[size_t(y) * s.NX + x] = float(iv);
            m[size_t(y) * s.NX + x] = float(-double(c.x) * iv);
        }
    }
}

void thomas_factors_y(const HostSetup& s, std::vector<float>& cp, std::vector<float>& inv, std::vector<float>& m) {
    const size_t n = size_t(s.NX) * s.NY;
    cp.assign(n, 0.f); inv.assign(n, 0.f); m.assign(n, 0.f);
    for (int x = 2; x < s.nx + 2; ++x) {
        double cprev = 0;
        for (int y = 2; y < s.ny + 2; ++y) {
            const Float4& c = s.ABCy[0][size_t(y) * s.NX + x];
            const double den = double(c.y) - double(c.x) * cprev;
            const double iv = 1.0 / den;
            cprev = double(c.z) * iv;
            cp[size_t(y) * s.NX + x] = float(cprev);
            inv[size_t(y) * s.NX + x] = float(iv);
            m[size_t(y) * s.NX + x] = float(-double(c.x) * iv);
        }
    }
}

SimConsts make_consts(const cel_params& p, const HostSetup& s, int pitch) {
    SimConsts c{};
    c.nx = s.nx; c.ny = s.ny; c.NX = s.NX; c.NY = s.NY; c.pitch = pitch;
    const float g = float(p.gravity);
    // fillConstantBuffers (engine.cpp:4099-4136)
    c.two_theta = 2 * float(p.theta);
    c.g = g;
    c.half_g = 0.5f * g;
    c.Bcoef_g = (1 / 15.0f) * g;
    c.g_over_dx = g / s.dx;
    c.g_over_dy = g / s.dy;
    c.one_over_dx = 1.0f / s.dx;
    c.one_over_dy = 1.0f / s.dy;
    c.dx = s.dx;
    c.dy = s.dy;
    c.epsilon = s.eps;
    c.friction = float(p.friction);
    c.is_manning = p.manning ? 1 : 0;
    c.sea_level = float(p.still_water_elevation);
    c.dissipation_threshold = float(p.dissipation_threshold);
    c.whitewater_decay_rate = 1.0f / (1 + 2 * float(p.whitewater_decay));
    return c;
}

}  // namespace cel
