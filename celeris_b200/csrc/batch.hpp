// Batched fused engine (many domains per launch) — host interface used by the C ABI.
//
// A batch (`cel_batch`, lanes.cpp) splits its members into lanes.  A lane (`cel_lane`, fused.cu)
// is one set of members advanced by one launch per kernel phase on its own stream, replayed from
// its own CUDA graphs.  Lanes run side by side, so one lane's small launches (boundary strips,
// the clock) and kernel tails overlap another lane's stencil.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "celeris_internal.hpp"
#include "engine_iface.hpp"

struct cel_lane;
struct cel_batch;

namespace cel {

// Room the banded column solver leaves beside its forward values (max_ny x band width floats of
// dynamic shared memory) for its static shared memory: the chunks' transfer maps and carries.
constexpr size_t COLS_STATIC_SMEM = 16384;

// ---- one lane (fused.cu) ----------------------------------------------------------------------
cel_lane* lane_create(int n, const cel_params* const* params, const float* const* bathy, const int* bnx,
                      const int* bny, int form, std::string& err);
void lane_destroy(cel_lane* b);
int lane_set_stream(cel_lane* b, cudaStream_t s, std::string& err);
cudaStream_t lane_stream(const cel_lane* b);
int lane_members(const cel_lane* b);
int lane_max_ny(const cel_lane* b);
int lane_step(cel_lane* b, int nsteps, std::string& err);
int lane_stats(cel_lane* b, cel_stats* out, bool current, std::string& err);
// lane_stats in two halves: enqueue the statistics pass and the read-back copies; then wait and convert
int lane_stats_enqueue(cel_lane* b, bool current, std::string& err);
int lane_stats_finish(cel_lane* b, cel_stats* out, bool current, std::string& err);
int lane_get_state(cel_lane* b, int i, float* rgba, std::string& err);
int lane_get_state_parts(cel_lane* b, int i, float* hi_rgba, float* lo_rgba, std::string& err);
int lane_set_state(cel_lane* b, int i, const float* rgba, std::string& err);
int lane_get_aux(cel_lane* b, int i, float* rgba, std::string& err);
int lane_set_bathymetry(cel_lane* b, int i, const float* z, int bnx, int bny, std::string& err);
int lane_add_solitary_wave(cel_lane* b, int i, double H, double theta_deg, double xc, double yc, std::string& err);
int lane_use_graph(cel_lane* b, bool enable, std::string& err);
long long lane_cells(const cel_lane* b);
int lane_set_timestep(cel_lane* b, const float* dt, std::string& err);
int lane_set_tuning(cel_lane* b, int tx, int ty, int pcr, std::string& err);
int lane_get_tuning(const cel_lane* b, int* tx, int* ty, int* rps);
int lane_set_stencil_rows(cel_lane* b, int rps, std::string& err);
int lane_set_stencil_width(cel_lane* b, int threads, std::string& err);
int lane_stencil_width(const cel_lane* b);
// column band width, strip height, stencil rows per step, stencil width, column solver threads in one call
int lane_configure(cel_lane* b, int cw, int mh, int rps, int mw, int nt, std::string& err);
int lane_col_threads(const cel_lane* b);
int lane_col_chunks(const cel_lane* b);   // chunks per column of the column solver (1: serial columns)
KernelTimer* lane_timer(cel_lane* b);
int lane_launches_per_step(const cel_lane* b);
void byte_model(int form, int correction_steps, double& stencil_bytes, double& step_bytes);
// the fused forms' flux reciprocal (rcp_newton) over n host values, run on the current device
int selftest_reciprocal(const float* x, float* out, int n, std::string& err);

// ---- a batch of lanes (lanes.cpp); member indices are the caller's ------------------------------
// lanes <= 0 picks the default: 2 lanes for 2 or more members, else 1.
cel_batch* batch_create(int n, const cel_params* const* params, const float* const* bathy, const int* bnx,
                        const int* bny, int form, int lanes, std::string& err);
void batch_destroy(cel_batch* b);
int batch_lanes(const cel_batch* b);
int batch_set_stream(cel_batch* b, cudaStream_t s, std::string& err);
int batch_step(cel_batch* b, int nsteps, std::string& err);
int batch_stats(cel_batch* b, cel_stats* out, bool current, std::string& err);
int batch_get_state(cel_batch* b, int i, float* rgba, std::string& err);
int batch_get_state_parts(cel_batch* b, int i, float* hi_rgba, float* lo_rgba, std::string& err);
int batch_set_state(cel_batch* b, int i, const float* rgba, std::string& err);
int batch_get_aux(cel_batch* b, int i, float* rgba, std::string& err);
int batch_set_bathymetry(cel_batch* b, int i, const float* z, int bnx, int bny, std::string& err);
int batch_add_solitary_wave(cel_batch* b, int i, double H, double theta_deg, double xc, double yc, std::string& err);
int batch_use_graph(cel_batch* b, bool enable, std::string& err);
long long batch_cells(const cel_batch* b);
int batch_set_timestep(cel_batch* b, const float* dt, std::string& err);
int batch_set_tuning(cel_batch* b, int tx, int ty, int pcr, std::string& err);
int batch_get_tuning(const cel_batch* b, int* tx, int* ty, int* rps);
int batch_col_chunks(const cel_batch* b);
int batch_set_stencil_rows(cel_batch* b, int rps, std::string& err);
int batch_set_stencil_width(cel_batch* b, int threads, std::string& err);
int batch_stencil_width(const cel_batch* b);
int batch_autotune(cel_batch* b, int steps, int* tx, int* ty, double* best_ms, std::string& err);
void batch_kernel_timing(cel_batch* b, bool enable);
// per-kernel totals summed over the lanes (synchronizes the pending timer events)
std::vector<KernelTimer::Rec> batch_kernel_records(cel_batch* b);
int batch_launches_per_step(const cel_batch* b);

}  // namespace cel
