// The reference's own shader code driven on the CPU (test infrastructure only).
//
// RefEngine is the FP32 oracle engine with every per-texel computation replaced by a call into
// the reference's compute.hlsl entry points, compiled as C++ (hlsl_shim.hpp plus the transform
// in ref_build.py, which writes oracle/_ref/compute_hlsl.inc).  The host-side schedule --
// which pass runs when, render regions, zeroing copies, history rotation, boundary order -- is
// the oracle's restatement of engine.cpp; each draw binds the textures and constant-buffer
// values that engine.cpp binds for it and invokes the pixel shader once per texel of the draw's
// region with tex_idx = (x + 0.5, y + 0.5), the pixel-centre coordinate the reference's vertex
// buffers produce (engine.cpp:573-593).  Comparing RefEngine with the oracle's FP32 build on
// the same inputs pins the oracle's restatement of the shader arithmetic to the reference's
// source.
#pragma once

#include <cstring>
#include <vector>

#include "hlsl_shim.hpp"

namespace hlsl {
#include "compute_hlsl.inc"

SRV& srv_slot(int reg) {
    static SRV slots[16];
    return slots[reg];
}
}  // namespace hlsl

#include "celeris_oracle.hpp"

namespace refshader {

using T4 = oracle::V4<float>;

inline T4 t4(const hlsl::float4& v) {
    T4 o; o.r = v.x; o.g = v.y; o.b = v.z; o.a = v.w;
    return o;
}

class RefEngine : public oracle::Engine<float> {
public:
    using Base = oracle::Engine<float>;
    std::vector<float> bottom3;  // RGB32F bottom texture {BY, BX, BA} (terrain_heightfield.hpp:50-52)

    // ---- binding helpers ----------------------------------------------------------------
    static void bind(int reg, const std::vector<T4>& t, int w, int h) {
        hlsl::SRV& s = hlsl::srv_slot(reg);
        s.data = reinterpret_cast<const float*>(t.data());
        s.w = w; s.h = h; s.comps = 4;
    }
    static void unbind_all() {
        for (int r = 0; r < 16; ++r) hlsl::srv_slot(r) = hlsl::SRV();
    }
    void bind_bottom(int reg) {
        if (bottom3.size() != size_t(NX) * NY * 3) {
            bottom3.resize(size_t(NX) * NY * 3);
            for (size_t i = 0; i < size_t(NX) * NY; ++i) {
                bottom3[3 * i] = BY[i]; bottom3[3 * i + 1] = BX[i]; bottom3[3 * i + 2] = BA[i];
            }
        }
        hlsl::SRV& s = hlsl::srv_slot(reg);
        s.data = bottom3.data(); s.w = NX; s.h = NY; s.comps = 3;
    }
    static hlsl::VS_OUTPUT pixel(int x, int y) {
        hlsl::VS_OUTPUT in;
        in.tex_idx = hlsl::float2(float(x) + 0.5f, float(y) + 0.5f);
        return in;
    }

    // SimConstBuffer as engine.cpp:4099-4136 fills it
    void set_sim_consts() {
        using namespace hlsl::cb_SimConstBuffer;
        const float theta = float(p.theta), g_ = float(p.gravity);
        TWO_THETA = 2 * theta;
        two_over_nx_plus_four = 2.0f / float(nx + 4);
        two_over_ny_plus_four = 2.0f / float(ny + 4);
        g = g_;
        half_g = 0.5f * g_;
        Bcoef_g = (1 / 15.0f) * g_;
        g_over_dx = g_ / dx;
        g_over_dy = g_ / dy;
        one_over_dx = 1.0f / dx;
        one_over_dy = 1.0f / dy;
        dt = current_timestep;
        dt_old = old_timestep;
        dt_old_old = old_old_timestep;
        epsilon = eps;
        hlsl::cb_SimConstBuffer::nx = Base::nx;
        hlsl::cb_SimConstBuffer::ny = Base::ny;
        friction = float(p.friction);
        isManning = p.manning ? 1 : 0;
        seaLevel = float(p.swl);
        dissipation_threshold = float(p.dissipation_threshold);
        whiteWaterDecayRate = 1.0f / (1 + 2 * float(p.whitewater_decay));
    }

    // ---- Pass1: region [1, nx+3) x [1, ny+3) (engine.cpp:2532) -------------------------
    // the bound bottom texture is rebuilt from the new BY/BX/BA (UpdateSubresource, engine.cpp:3349-3354)
    void new_terrain(const std::vector<float>& zgrid, int bnx, int bny) override {
        oracle::Engine<float>::new_terrain(zgrid, bnx, bny);
        bottom3.clear();
    }

    void pass1(const std::vector<T4>& st) override {
        set_sim_consts();
        unbind_all();
        bind(0, st, NX, NY); bind_bottom(1); bind(3, aux1, NX, NY);
        for (int y = 1; y < ny + 3; ++y)
            for (int x = 1; x < nx + 3; ++x) {
                const hlsl::PASS_1_OUTPUT o = hlsl::Pass1(pixel(x, y));
                H[at(x, y)] = t4(o.h); U[at(x, y)] = t4(o.u); V[at(x, y)] = t4(o.v);
                aux2[at(x, y)] = t4(o.aux);
            }
        unbind_all();
    }

    // ---- Pass2: region [1, nx+2) x [1, ny+2), flux targets cleared first ----------------
    void pass2() override {
        set_sim_consts();
        std::fill(xflux.begin(), xflux.end(), T4());
        std::fill(yflux.begin(), yflux.end(), T4());
        unbind_all();
        bind(0, H, NX, NY); bind(1, U, NX, NY); bind(2, V, NX, NY); bind(4, aux2, NX, NY);
        for (int y = 1; y < ny + 2; ++y)
            for (int x = 1; x < nx + 2; ++x) {
                const hlsl::PASS_2_OUTPUT o = hlsl::Pass2(pixel(x, y));
                xflux[at(x, y)] = t4(o.xflux); yflux[at(x, y)] = t4(o.yflux); aux1[at(x, y)] = t4(o.auxiliary);
            }
        unbind_all();
    }

    // ---- Pass3Predictor: region [2, nx+2) x [2, ny+2), new state cleared first ----------
    void pass3(const std::vector<T4>& st, std::vector<T4>& out, std::vector<T4>& sgrad, std::vector<T4>& sfg) override {
        set_sim_consts();
        hlsl::cb_TimeIntegrationBuffer::timeScheme = time_scheme;
        std::fill(out.begin(), out.end(), T4());
        unbind_all();
        bind(0, st, NX, NY); bind_bottom(1);
        bind(2, xflux, NX, NY); bind(3, yflux, NX, NY);
        bind(4, grad[old_i], NX, NY); bind(5, grad[oldold_i], NX, NY);
        bind(6, ABCx[0], NX, NY); bind(7, ABCy[0], NX, NY);
        bind(8, fg[fg_old_i], NX, NY); bind(9, fg[fg_oldold_i], NX, NY);
        bind(10, pred, NX, NY); bind(11, fgpred, NX, NY); bind(12, cur, NX, NY);
        for (int y = 2; y < ny + 2; ++y)
            for (int x = 2; x < nx + 2; ++x) {
                const hlsl::PASS_3_OUTPUT o = hlsl::Pass3Predictor(pixel(x, y));
                out[at(x, y)] = t4(o.newState); sgrad[at(x, y)] = t4(o.dU_by_dt); sfg[at(x, y)] = t4(o.F_G_star);
            }
        unbind_all();
    }

    // ---- cyclic reduction in x (engine.cpp:1060-1217): reduce levels 1.., substitute down
    void cr_solve_x(const std::vector<T4>& rhs) override {
        set_sim_consts();
        for (int k = 1; k < Kx; ++k) {
            unbind_all();
            const int Wp = (k == 1) ? NX : lenx[k - 1] + 4;
            bind(1, (k == 1) ? rhs : D1x[k - 1], Wp, NY);   // D1x (t1)
            bind(6, ABCx[k - 1], lenx[k - 1] + 4, NY);      // coefMatx (t6)
            const int Wk = lenx[k] + 4;
            for (int y = 2; y < ny + 2; ++y)
                for (int x = 2; x < lenx[k] + 2; ++x)
                    D1x[k][size_t(y) * Wk + x] = t4(hlsl::CyclicReduceDx(pixel(x, y)));
        }
        for (int k = Kx - 1; k >= 0; --k) {
            unbind_all();
            const int Wk = lenx[k] + 4;
            bind(1, (k == 0) ? rhs : D1x[k], (k == 0) ? NX : Wk, NY);
            bind(6, ABCx[k], Wk, NY);
            if (k + 1 < Kx) bind(2, D1xc[k + 1], lenx[k + 1] + 4, NY);  // Xx (t2); the coarsest reads nothing
            for (int y = 2; y < ny + 2; ++y)
                for (int x = 2; x < lenx[k] + 2; ++x)
                    D1xc[k][size_t(y) * Wk + x] = t4(hlsl::CyclicSubstituteXx(pixel(x, y)));
        }
        unbind_all();
    }

    void cr_solve_y(const std::vector<T4>& rhs) override {
        set_sim_consts();
        for (int k = 1; k < Ky; ++k) {
            unbind_all();
            const int Hp = (k == 1) ? NY : leny[k - 1] + 4;
            bind(1, (k == 1) ? rhs : D1y[k - 1], NX, Hp);   // D1y (t1)
            bind(7, ABCy[k - 1], NX, leny[k - 1] + 4);      // coefMaty (t7)
            for (int y = 2; y < leny[k] + 2; ++y)
                for (int x = 2; x < nx + 2; ++x)
                    D1y[k][size_t(y) * NX + x] = t4(hlsl::CyclicReduceDy(pixel(x, y)));
        }
        for (int k = Ky - 1; k >= 0; --k) {
            unbind_all();
            const int Hk = leny[k] + 4;
            bind(1, (k == 0) ? rhs : D1y[k], NX, (k == 0) ? NY : Hk);
            bind(7, ABCy[k], NX, Hk);
            if (k + 1 < Ky) bind(3, D1yc[k + 1], NX, leny[k + 1] + 4);  // Xy (t3)
            for (int y = 2; y < leny[k] + 2; ++y)
                for (int x = 2; x < nx + 2; ++x)
                    D1yc[k][size_t(y) * NX + x] = t4(hlsl::CyclicSubstituteXy(pixel(x, y)));
        }
        unbind_all();
    }

    // ---- CopyFromXxAndXy over the interior (engine.cpp:1219-1233) -----------------------
    void copy_from(std::vector<T4>& new_state) override {
        unbind_all();
        const std::vector<T4> src = new_state;  // txState (t0) is the pass's new state
        bind(0, src, NX, NY);
        bind(2, D1xc[0], NX, NY);
        bind(3, D1yc[0], NX, NY);
        for (int y = 2; y < ny + 2; ++y)
            for (int x = 2; x < nx + 2; ++x) new_state[at(x, y)] = t4(hlsl::CopyFromXxAndXy(pixel(x, y)));
        unbind_all();
    }

    // ---- boundaries (engine.cpp:1236-1438, 1811-2151) -------------------------------------
    void set_boundary_consts() {
        namespace cb = hlsl::cb_BoundaryConstBuffer;
        cb::PI = PI_;
        cb::boundary_epsilon = eps;
        cb::boundary_nx = NX; cb::boundary_ny = NY;
        cb::dx = Base::dx; cb::dy = Base::dy;
        cb::reflect_x = 2 * nx + 2; cb::reflect_y = 2 * ny + 2;
        cb::northBoundaryWidth = p.north.width; cb::eastBoundaryWidth = p.east.width;
        cb::westBoundaryWidth = p.west.width; cb::southBoundaryWidth = p.south.width;
        cb::northSeaLevel = float(p.north.sea_level); cb::eastSeaLevel = float(p.east.sea_level);
        cb::westSeaLevel = float(p.west.sea_level); cb::southSeaLevel = float(p.south.sea_level);
        const oracle::Boundary* sides[4] = {&p.north, &p.east, &p.south, &p.west};
        float* amp[4] = {&cb::northAmplitude_or_eta, &cb::eastAmplitude_or_eta, &cb::southAmplitude_or_eta,
                         &cb::westAmplitude_or_eta};
        float* per[4] = {&cb::northPeriod_or_hu, &cb::eastPeriod_or_hu, &cb::southPeriod_or_hu, &cb::westPeriod_or_hu};
        float* th[4] = {&cb::northTheta_or_hv, &cb::eastTheta_or_hv, &cb::southTheta_or_hv, &cb::westTheta_or_hv};
        for (int s = 0; s < 4; ++s) {
            const oracle::Boundary& b = *sides[s];
            if (b.type == oracle::B_UTS) {
                float v[3] = {0, 0, 0};
                uts_value(b, s, total_time, v);
                *amp[s] = v[0]; *per[s] = v[1]; *th[s] = v[2];
            } else {
                *amp[s] = float(b.amplitude); *per[s] = float(b.period); *th[s] = float(b.theta);
            }
        }
        cb::boundary_g = float(p.gravity);
        cb::boundary_dt = current_timestep;
        cb::total_time = total_time;
    }

    // the pixel shader of one side for a non-irregular boundary type
    hlsl::float4 side_shader(int side, int type, int x, int y) {
        const hlsl::VS_OUTPUT in = pixel(x, y);
        switch (side) {
            case 0:
                if (type == oracle::B_SOLID) return hlsl::NorthBoundarySolid(in);
                if (type == oracle::B_SPONGE) return hlsl::NorthBoundarySponge(in);
                if (type == oracle::B_SINEWAVE) return hlsl::NorthBoundarySineWave(in);
                return hlsl::NorthBoundaryUniformTimeSeries(in);
            case 1:
                if (type == oracle::B_SOLID) return hlsl::EastBoundarySolid(in);
                if (type == oracle::B_SPONGE) return hlsl::EastBoundarySponge(in);
                if (type == oracle::B_SINEWAVE) return hlsl::EastBoundarySineWave(in);
                return hlsl::EastBoundaryUniformTimeSeries(in);
            case 2:
                if (type == oracle::B_SOLID) return hlsl::SouthBoundarySolid(in);
                if (type == oracle::B_SPONGE) return hlsl::SouthBoundarySponge(in);
                if (type == oracle::B_SINEWAVE) return hlsl::SouthBoundarySineWave(in);
                return hlsl::SouthBoundaryUniformTimeSeries(in);
            default:
                if (type == oracle::B_SOLID) return hlsl::WestBoundarySolid(in);
                if (type == oracle::B_SPONGE) return hlsl::WestBoundarySponge(in);
                if (type == oracle::B_SINEWAVE) return hlsl::WestBoundarySineWave(in);
                return hlsl::WestBoundaryUniformTimeSeries(in);
        }
    }

    // Irregular waves along one side (engine.cpp:1811-1880 and its three siblings): for each
    // strip column (row), one component per texel of the level-0 region, then pairwise sums
    // down the cyclic-reduction levels, then the surviving column (row) copied into the state.
    void irregular_side(std::vector<T4>& st, int side) {
        namespace ic = hlsl::cb_IrregularWavesConstBuffer;
        namespace rc = hlsl::cb_IrregularWavesColumnRowConstBuffer;
        const oracle::Boundary* bs[4] = {&p.north, &p.east, &p.south, &p.west};
        hlsl::float4* tables[4] = {ic::irregularWavesNorth, ic::irregularWavesEast, ic::irregularWavesSouth,
                                   ic::irregularWavesWest};
        int* counts[4] = {&ic::numberOfWavesNorth, &ic::numberOfWavesEast, &ic::numberOfWavesSouth,
                          &ic::numberOfWavesWest};
        for (int s = 0; s < 4; ++s) {
            const oracle::Boundary& b = *bs[s];
            *counts[s] = int(b.waves.size());
            for (size_t k = 0; k < b.waves.size() && k < 1000; ++k)
                tables[s][k] = hlsl::float4(float(b.waves[k][0]), float(b.waves[k][1]), float(b.waves[k][2]),
                                            float(b.waves[k][3]));
        }
        const oracle::Boundary& b = *bs[side];
        const bool colwise = (side == 1 || side == 3);
        const int K = colwise ? Kx : Ky;
        const std::vector<int>& len = colwise ? lenx : leny;
        int lo, hi;
        if (side == 3) { lo = 0; hi = b.width; }
        else if (side == 1) { lo = NX - b.width; hi = NX; }
        else if (side == 2) { lo = 0; hi = b.width; }
        else { lo = NY - b.width; hi = NY; }
        std::vector<std::vector<T4>> lev(K);
        for (int k = 0; k < K; ++k)
            lev[k].assign(colwise ? size_t(len[k] + 4) * NY : size_t(NX) * (len[k] + 4), T4());
        for (int line = lo; line < hi; ++line) {
            rc::columnNumber = colwise ? line : 0;
            rc::rowNumber = colwise ? 0 : line;
            // level 0 (the cleared scratch texture, NX x NY), region [2, nx+2) x [2, ny+2)
            std::vector<T4> scratch(size_t(NX) * NY, T4());
            unbind_all();
            bind_bottom(1);
            for (int y = 2; y < ny + 2; ++y)
                for (int x = 2; x < nx + 2; ++x) {
                    const hlsl::VS_OUTPUT in = pixel(x, y);
                    hlsl::float4 o;
                    if (side == 3) o = hlsl::WestBoundaryIrregularWaves(in);
                    else if (side == 1) o = hlsl::EastBoundaryIrregularWaves(in);
                    else if (side == 2) o = hlsl::SouthBoundaryIrregularWaves(in);
                    else o = hlsl::NorthBoundaryIrregularWaves(in);
                    scratch[at(x, y)] = t4(o);
                }
            for (int k = 1; k < K; ++k) {
                unbind_all();
                if (colwise) {
                    bind(0, k == 1 ? scratch : lev[k - 1], k == 1 ? NX : len[k - 1] + 4, NY);
                    const int Wk = len[k] + 4;
                    for (int y = 2; y < ny + 2; ++y)
                        for (int x = 2; x < len[k] + 2; ++x)
                            lev[k][size_t(y) * Wk + x] = t4(hlsl::ColumnSumReduce(pixel(x, y)));
                } else {
                    bind(0, k == 1 ? scratch : lev[k - 1], NX, k == 1 ? NY : len[k - 1] + 4);
                    for (int y = 2; y < len[k] + 2; ++y)
                        for (int x = 2; x < nx + 2; ++x)
                            lev[k][size_t(y) * NX + x] = t4(hlsl::RowSumReduce(pixel(x, y)));
                }
            }
            const std::vector<T4>& last = K > 1 ? lev[K - 1] : scratch;
            const int Wl = K > 1 ? (colwise ? len[K - 1] + 4 : NX) : NX;
            if (colwise)
                for (int y = 0; y < NY; ++y) st[at(line, y)] = last[size_t(y) * Wl + 2];
            else
                for (int x = 0; x < NX; ++x) st[at(x, line)] = last[size_t(2) * Wl + x];
        }
        unbind_all();
    }

    void boundary_side(std::vector<T4>& st, int side) override {
        set_boundary_consts();
        const oracle::Boundary& b = side == 0 ? p.north : side == 1 ? p.east : side == 2 ? p.south : p.west;
        if (b.type == oracle::B_IRREGULAR) { irregular_side(st, side); return; }
        int x0, x1, y0, y1;
        if (side == 0) { x0 = 0; x1 = NX; y0 = NY - b.width; y1 = NY; }
        else if (side == 1) { x0 = NX - b.width; x1 = NX; y0 = 0; y1 = NY; }
        else if (side == 2) { x0 = 0; x1 = NX; y0 = 0; y1 = b.width; }
        else { x0 = 0; x1 = b.width; y0 = 0; y1 = NY; }
        x0 = std::max(x0, 0); y0 = std::max(y0, 0); x1 = std::min(x1, NX); y1 = std::min(y1, NY);
        if (x1 <= x0 || y1 <= y0) return;
        // render into the scratch texture from the current state, then copy the strip back
        unbind_all();
        bind(0, st, NX, NY); bind_bottom(1);
        std::vector<T4> strip(size_t(x1 - x0) * (y1 - y0));
        for (int y = y0; y < y1; ++y)
            for (int x = x0; x < x1; ++x) strip[size_t(y - y0) * (x1 - x0) + (x - x0)] = t4(side_shader(side, b.type, x, y));
        unbind_all();
        for (int y = y0; y < y1; ++y)
            for (int x = x0; x < x1; ++x) st[at(x, y)] = strip[size_t(y - y0) * (x1 - x0) + (x - x0)];
    }

    // ---- GetStats: pixel (bx, by) covers the 4x4 block at (4bx+2, 4by+2) ---------------
    void stats_block(const std::vector<T4>& st, int bx, int by, float o[9]) const override {
        const_cast<RefEngine*>(this)->set_sim_consts();
        unbind_all();
        bind(0, st, NX, NY);
        const_cast<RefEngine*>(this)->bind_bottom(1);
        const hlsl::GET_STATS_OUTPUT r = hlsl::GetStats(pixel(bx, by));
        unbind_all();
        o[0] = r.target0.x; o[1] = r.target0.y; o[2] = r.target0.z; o[3] = r.target0.w;
        o[4] = r.target1.x; o[5] = r.target1.y; o[6] = r.target1.z; o[7] = r.target1.w;
        o[8] = r.target2;
    }

    // ---- AddSolitaryWave over [1, nx+3) x [1, ny+3) (engine.cpp:2154-2219) -----------------
    void add_solitary_wave(double Hh, double theta_deg, double xc, double yc) override {
        namespace sw = hlsl::cb_SolitaryWave;
        sw::sw_g = float(p.gravity);
        sw::sw_dx = dx; sw::sw_dy = dy;
        sw::sw_param_H = float(Hh);
        sw::sw_x_zero = float(xc); sw::sw_y_zero = float(yc);
        sw::sw_theta = float(theta_deg) * PI_ / 180.0f;
        std::vector<T4>& st = state[sim_idx];
        const std::vector<T4> copy = st;
        unbind_all();
        bind(0, copy, NX, NY); bind_bottom(1);
        for (int y = 1; y < ny + 3; ++y)
            for (int x = 1; x < nx + 3; ++x) st[at(x, y)] = t4(hlsl::AddSolitaryWave(pixel(x, y)).newState);
        unbind_all();
    }
};

}  // namespace refshader
