// Internal declarations shared by the host setup, the CUDA engines and the C ABI.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/celeris_b200.h"

namespace cel {

// ---- settings boundary (params.cpp) --------------------------------------------------------
void params_default(cel_params* p);
int params_from_cml(const char* path, cel_params* out, std::string& err);
void params_release(cel_params* p);
int read_irregular(const std::string& path, cel_boundary* b, std::string& err);
int read_uts(const std::string& path, cel_boundary* b, std::string& err);
int read_cbf(const std::string& path, std::vector<float>* z, int& bnx, int& bny, std::string& err);
int read_hotstart(const std::string& path, int nx, int ny, std::vector<float>& whuhv, std::string& err);

// ---- irregular-wave spectrum (spectrum.cpp) --------------------------------------------------
int spectrum_waves(const cel_spectrum& in, double gravity, unsigned long long seed, cel_boundary* b, const char* path,
                   std::string& err);

// ---- file output (logio.cpp) ------------------------------------------------------------------
int log_validate(const cel_log& lg, int nx, int ny, std::string& err);
int log_dump(const cel_log& lg, const float* rgba, int nx, int ny, float total_time, float elapsed, std::string& err);
int write_inundation(const cel_log& lg, const float* aux, int nx, int ny, const char* path, std::string& err);
int write_bathymetry(const cel_log& lg, const float* b3, int nx, int ny, const char* path, std::string& err);
int write_hotstart(const float* rgba, int nx, int ny, const char* path, std::string& err);

// ---- host setup (setup.cpp): the once-per-remesh host work of the reference ----------------
struct Float4 { float x, y, z, w; };

struct HostSetup {
    int nx = 0, ny = 0, NX = 0, NY = 0;
    float dx = 0, dy = 0, eps = 0;
    std::vector<float> BY, BX, BA;          // staggered bottom, NX*NY each
    std::vector<float> corners;             // bathymetry sampled at cell corners, (NX+1)*(NY+1)
    std::vector<float> ic;                  // initial (w, hu, hv) per texel, NX*NY*3
    std::vector<double> ic64;               // the same in double precision (for the compensated form)
    // Cyclic-reduction coefficient levels, {A, B, C, 0} per texel (engine.cpp:2612-2887)
    int Kx = 0, Ky = 0;
    std::vector<int> lenx, leny;
    std::vector<std::vector<Float4>> ABCx, ABCy;
};

int count_of_matrices(int n);
// GetTerrainHeight (terrain_heightfield.cpp:313-351): bilinear in float of the cell-centre bottom
// BA (the terrain heightfield's B) at world point (x, y), x in [-W/2, W/2], y in [0, L], clamped.
float terrain_height(const HostSetup& s, float W, float L, float x, float y);
// getWaterHeight's 4x4 block (engine.cpp:5001-5006): the GetStats block of world point (x, y),
// clamped to the block array (the reference reads past it at x = W/2 or y = L).
void water_height_block(int nx, int ny, float W, float L, float x, float y, int& ix, int& iy);
// terrain_heightfield.cpp:213-297 (bilinear sampling, corner averaging), in float
void prepare_bottom(const float* z, int bnx, int bny, int nx, int ny, float W, float L, HostSetup& s);
// engine.cpp:2612-2887
void build_cr_levels(const cel_params& p, HostSetup& s);
// engine.cpp:2940-3016 (+ hot start)
void initial_condition(const cel_params& p, const std::vector<float>* hot, HostSetup& s);
int make_setup(const cel_params& p, const float* bathy, int bnx, int bny, HostSetup& s, std::string& err);

// Thomas factors of the level-0 tridiagonal systems for the fused solver, per direction:
// for each interior cell, {cprime, inv_den, m = -a*inv_den} (see fused kernels).
void thomas_factors_x(const HostSetup& s, std::vector<float>& cprime, std::vector<float>& inv, std::vector<float>& m);
void thomas_factors_y(const HostSetup& s, std::vector<float>& cprime, std::vector<float>& inv, std::vector<float>& m);

// ---- constants shared by kernels ------------------------------------------------------------
// SimConstBuffer (compute.hlsl:65-94) + BoundaryConstBuffer fields (compute.hlsl:118-145)
struct SimConsts {
    int nx, ny, NX, NY, pitch;
    float two_theta, g, half_g, Bcoef_g, g_over_dx, g_over_dy, one_over_dx, one_over_dy;
    float dx, dy;
    float epsilon, friction, sea_level;
    int is_manning;
    float dissipation_threshold, whitewater_decay_rate;
};

struct BoundaryDesc {
    int type, width;
    float sea_level, amplitude, period, theta;
    int n_waves;
    int nleaf;          // 2^(K-1): components summed by the reference's pairwise tree
    int wave_offset;    // into the engine's device wave table (float4 per component)
    // the same settings unrounded, for the compensated form's FP64 strip values
    double sea_level64, amplitude64, period64, theta64;
};

SimConsts make_consts(const cel_params& p, const HostSetup& s, int pitch);

// ---- thread-local error message for the C ABI -----------------------------------------------
void set_error(const std::string& msg);
const char* last_error();

}  // namespace cel
