// Batched fused engine (many domains per launch) — host interface used by the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "celeris_internal.hpp"
#include "engine_iface.hpp"

struct cel_batch;

namespace cel {

cel_batch* batch_create(int n, const cel_params* const* params, const float* const* bathy, const int* bnx,
                        const int* bny, int form, std::string& err);
void batch_destroy(cel_batch* b);
int batch_set_stream(cel_batch* b, cudaStream_t s, std::string& err);
int batch_step(cel_batch* b, int nsteps, std::string& err);
int batch_stats(cel_batch* b, cel_stats* out, bool current, std::string& err);
int batch_get_state(cel_batch* b, int i, float* rgba, std::string& err);
int batch_set_state(cel_batch* b, int i, const float* rgba, std::string& err);
int batch_get_aux(cel_batch* b, int i, float* rgba, std::string& err);
int batch_set_bathymetry(cel_batch* b, int i, const float* z, int bnx, int bny, std::string& err);
int batch_add_solitary_wave(cel_batch* b, int i, double H, double theta_deg, double xc, double yc, std::string& err);
int batch_use_graph(cel_batch* b, bool enable, std::string& err);
long long batch_cells(const cel_batch* b);
int batch_set_timestep(cel_batch* b, const float* dt, std::string& err);
int batch_set_tuning(cel_batch* b, int tx, int ty, int pcr, std::string& err);
int batch_get_tuning(const cel_batch* b, int* tx, int* ty, int* rps);
int batch_set_stencil_rows(cel_batch* b, int rps, std::string& err);
int batch_set_stencil_width(cel_batch* b, int threads, std::string& err);
int batch_stencil_width(const cel_batch* b);
int batch_autotune(cel_batch* b, int steps, int* tx, int* ty, double* best_ms, std::string& err);
KernelTimer* batch_timer(cel_batch* b);
int batch_launches_per_step(const cel_batch* b);
void byte_model(int form, int correction_steps, double& stencil_bytes, double& step_bytes);

}  // namespace cel
