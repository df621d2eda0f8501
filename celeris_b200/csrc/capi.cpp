// The C ABI (include/celeris_b200.h): status codes in, no exceptions out.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "batch.hpp"
#include "celeris_internal.hpp"
#include "engine_iface.hpp"

namespace cel {

namespace {
thread_local std::string g_err;
}

void set_error(const std::string& msg) { g_err = msg; }
const char* last_error() { return g_err.c_str(); }

cudaEvent_t KernelTimer::get_event() {
    if (!pool.empty()) {
        cudaEvent_t e = pool.back();
        pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void KernelTimer::begin(cudaStream_t s, const char* name, cudaEvent_t& ev0, int& idx) {
    idx = -1;
    for (size_t k = 0; k < recs.size(); ++k)
        if (recs[k].name == name) { idx = int(k); break; }
    if (idx < 0) {
        recs.push_back({name, 0.0, 0});
        idx = int(recs.size() - 1);
    }
    ev0 = get_event();
    cudaEventRecord(ev0, s);
}

void KernelTimer::end(cudaStream_t s, int idx, cudaEvent_t ev0) {
    cudaEvent_t e1 = get_event();
    cudaEventRecord(e1, s);
    pending.push_back({idx, {ev0, e1}});
    if (pending.size() > 4096) collect();
}

void KernelTimer::collect() {
    for (auto& pnd : pending) {
        cudaEventSynchronize(pnd.second.second);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, pnd.second.first, pnd.second.second);
        recs[pnd.first].ms += ms;
        recs[pnd.first].n += 1;
        pool.push_back(pnd.second.first);
        pool.push_back(pnd.second.second);
    }
    pending.clear();
}

KernelTimer::~KernelTimer() {
    for (auto& pnd : pending) { cudaEventDestroy(pnd.second.first); cudaEventDestroy(pnd.second.second); }
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
}

}  // namespace cel

struct cel_engine {
    cel::EngineIface* impl = nullptr;
};

using cel::set_error;

#define CEL_GUARD_BEGIN try {
#define CEL_GUARD_END                                               \
    }                                                               \
    catch (const std::exception& ex) {                              \
        set_error(std::string("internal error: ") + ex.what());     \
        return CEL_ERR_STATE;                                       \
    }                                                               \
    catch (...) {                                                   \
        set_error("internal error");                                \
        return CEL_ERR_STATE;                                       \
    }

static int ret(cel::EngineIface* e, int st) {
    if (st != CEL_OK) set_error(e->err);
    return st;
}

static int need_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_error(std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "0 devices"));
        return CEL_ERR_CUDA;
    }
    return CEL_OK;
}

extern "C" {

const char* cel_last_error(void) { return cel::last_error(); }
const char* cel_version(void) { return "celeris_b200 1.0 (sm_100a)"; }

int cel_params_default(cel_params* p) {
    if (!p) { set_error("null params"); return CEL_ERR_ARG; }
    cel::params_default(p);
    return CEL_OK;
}

int cel_params_from_cml(const char* path, cel_params* out) {
    if (!path || !out) { set_error("null argument"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN
    std::string err;
    const int st = cel::params_from_cml(path, out, err);
    if (st) set_error(err);
    return st;
    CEL_GUARD_END
}

int cel_read_irregular_waves(const char* path, cel_boundary* b) {
    if (!path || !b) { set_error("null argument"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN
    std::string err;
    const int st = cel::read_irregular(path, b, err);
    if (st) set_error(err);
    return st;
    CEL_GUARD_END
}

int cel_read_uts(const char* path, cel_boundary* b) {
    if (!path || !b) { set_error("null argument"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN
    std::string err;
    const int st = cel::read_uts(path, b, err);
    if (st) set_error(err);
    return st;
    CEL_GUARD_END
}

void cel_params_release(cel_params* p) {
    if (p) cel::params_release(p);
}

size_t cel_params_size(void) { return sizeof(cel_params); }

int cel_spectrum_waves(const cel_spectrum* s, double gravity, unsigned long long seed, cel_boundary* b, const char* path) {
    if (!s || !b) { set_error("null argument"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN
    std::string err;
    const int st = cel::spectrum_waves(*s, gravity, seed, b, path, err);
    if (st) set_error(err);
    return st;
    CEL_GUARD_END
}

int cel_log_dump(const cel_params* p, const float* rgba, float total_time, float elapsed) {
    if (!p || !rgba) { set_error("null argument"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN
    std::string err;
    const int st = cel::log_dump(p->log, rgba, p->nx, p->ny, total_time, elapsed, err);
    if (st) set_error(err);
    return st;
    CEL_GUARD_END
}

int cel_write_inundation(const cel_params* p, const float* aux_rgba, const char* path) {
    if (!p || !aux_rgba) { set_error("null argument"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN
    std::string err;
    const int st = cel::write_inundation(p->log, aux_rgba, p->nx, p->ny, path, err);
    if (st) set_error(err);
    return st;
    CEL_GUARD_END
}

int cel_write_bathymetry(const cel_params* p, const float* bottom_b3, const char* path) {
    if (!p || !bottom_b3) { set_error("null argument"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN
    std::string err;
    const int st = cel::write_bathymetry(p->log, bottom_b3, p->nx, p->ny, path, err);
    if (st) set_error(err);
    return st;
    CEL_GUARD_END
}

int cel_write_hotstart(const cel_params* p, const float* rgba, const char* path) {
    if (!p || !rgba || !path) { set_error("null argument"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN
    std::string err;
    const int st = cel::write_hotstart(rgba, p->nx, p->ny, path, err);
    if (st) set_error(err);
    return st;
    CEL_GUARD_END
}

int cel_read_cbf(const char* path, float* z, size_t capacity, int* bnx, int* bny) {
    if (!path || !bnx || !bny) { set_error("null argument"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN
    std::string err;
    std::vector<float> v;
    int nx = 0, ny = 0;
    int st = cel::read_cbf(path, z ? &v : nullptr, nx, ny, err);
    if (st) { set_error(err); return st; }
    *bnx = nx; *bny = ny;
    if (z) {
        if (capacity < v.size()) { set_error("capacity smaller than nx*ny"); return CEL_ERR_ARG; }
        std::memcpy(z, v.data(), v.size() * sizeof(float));
    }
    return CEL_OK;
    CEL_GUARD_END
}

int cel_create(const cel_params* p, const float* bathy, int bnx, int bny, int form, cel_engine** out) {
    if (!p || !out) { set_error("null argument"); return CEL_ERR_ARG; }
    if (form < CEL_FORM_PLAIN || form > CEL_FORM_MIXED) { set_error("unknown form"); return CEL_ERR_ARG; }
    if (int st = need_device()) return st;
    CEL_GUARD_BEGIN
    std::string err;
    cel::EngineIface* e = (form == CEL_FORM_PLAIN) ? cel::make_plain_engine(*p, bathy, bnx, bny, err)
                                                   : cel::make_fused_engine(*p, bathy, bnx, bny, form, err);
    if (!e) { set_error(err); return err.find("cuda") != std::string::npos || err.find("CUDA") != std::string::npos ? CEL_ERR_CUDA : CEL_ERR_ARG; }
    auto* h = new cel_engine();
    h->impl = e;
    *out = h;
    return CEL_OK;
    CEL_GUARD_END
}

int cel_destroy(cel_engine* h) {
    if (!h) return CEL_OK;
    delete h->impl;
    delete h;
    return CEL_OK;
}

#define ENG(h)                                                  \
    if (!h || !h->impl) { set_error("null engine"); return CEL_ERR_ARG; } \
    cel::EngineIface* e = h->impl;

int cel_remesh(cel_engine* h) { ENG(h); CEL_GUARD_BEGIN return ret(e, e->remesh()); CEL_GUARD_END }
int cel_set_stream(cel_engine* h, void* s) { ENG(h); CEL_GUARD_BEGIN return ret(e, e->set_stream(static_cast<cudaStream_t>(s))); CEL_GUARD_END }
int cel_get_dims(const cel_engine* h, int* nx, int* ny) {
    if (!h || !h->impl || !nx || !ny) { set_error("null argument"); return CEL_ERR_ARG; }
    *nx = h->impl->nx(); *ny = h->impl->ny();
    return CEL_OK;
}
int cel_set_state(cel_engine* h, const float* rgba) {
    ENG(h);
    if (!rgba) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN return ret(e, e->set_state(rgba)); CEL_GUARD_END
}
int cel_get_state(cel_engine* h, float* rgba) {
    ENG(h);
    if (!rgba) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN return ret(e, e->get_state(rgba)); CEL_GUARD_END
}
int cel_get_bottom(cel_engine* h, float* b) {
    ENG(h);
    if (!b) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN return ret(e, e->get_bottom(b)); CEL_GUARD_END
}
int cel_get_aux(cel_engine* h, float* rgba) {
    ENG(h);
    if (!rgba) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN return ret(e, e->get_aux(rgba)); CEL_GUARD_END
}
int cel_reset_timestep(cel_engine* h, float rdt, float el, cel_stats* out) {
    ENG(h);
    e->log_elapsed = el;
    CEL_GUARD_BEGIN return ret(e, e->reset_timestep(rdt, el, out)); CEL_GUARD_END
}
int cel_timestep(cel_engine* h) { ENG(h); CEL_GUARD_BEGIN return ret(e, e->timestep()); CEL_GUARD_END }
int cel_timesteps(cel_engine* h, int n) {
    ENG(h);
    if (n < 0) { set_error("negative step count"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN return ret(e, e->timesteps(n)); CEL_GUARD_END
}
int cel_physical_steps(cel_engine* h, int n) {
    ENG(h);
    if (n < 0) { set_error("negative step count"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN return ret(e, e->physical_steps(n)); CEL_GUARD_END
}
int cel_get_stats(cel_engine* h, cel_stats* out) {
    ENG(h);
    if (!out) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN return ret(e, e->get_stats(out)); CEL_GUARD_END
}
int cel_add_solitary_wave(cel_engine* h, double H, double th, double xc, double yc) {
    ENG(h);
    CEL_GUARD_BEGIN return ret(e, e->add_solitary_wave(H, th, xc, yc)); CEL_GUARD_END
}
int cel_get_water_height(cel_engine* h, float x, float y, float* out) {
    // getWaterHeight (engine.cpp:4994-5012) at a world point (x in [-W/2, W/2], y in [0, L])
    ENG(h);
    if (!out) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN return ret(e, e->water_height(x, y, out)); CEL_GUARD_END
}
int cel_set_bathymetry(cel_engine* h, const float* bathy, int bnx, int bny) {
    ENG(h);
    if (!bathy || bnx < 2 || bny < 2) { set_error("bathymetry grid needs at least 2 x 2 values"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN return ret(e, e->set_bathymetry(bathy, bnx, bny)); CEL_GUARD_END
}
int cel_synchronize(cel_engine* h) { ENG(h); CEL_GUARD_BEGIN return ret(e, e->synchronize()); CEL_GUARD_END }
int cel_set_tuning(cel_engine* h, int tx, int ty, int pcr) {
    ENG(h);
    CEL_GUARD_BEGIN return ret(e, e->set_tuning(tx, ty, pcr)); CEL_GUARD_END
}
int cel_engine_kernel_timing(cel_engine* h, int enable) {
    ENG(h);
    e->timer()->enabled = enable != 0;
    return CEL_OK;
}

// ---- batches -------------------------------------------------------------------------------
int cel_batch_create(int n, const cel_params* const* params, const float* const* bathy, const int* bnx,
                     const int* bny, int form, cel_batch** out) {
    return cel_batch_create_lanes(n, params, bathy, bnx, bny, form, 0, out);
}

int cel_batch_create_lanes(int n, const cel_params* const* params, const float* const* bathy, const int* bnx,
                           const int* bny, int form, int lanes, cel_batch** out) {
    if (n <= 0 || !params || !out || !bathy || !bnx || !bny) { set_error("bad batch arguments"); return CEL_ERR_ARG; }
    if (lanes < 0) { set_error("lanes must be >= 0 (0 = the default)"); return CEL_ERR_ARG; }
    for (int i = 0; i < n; ++i)
        if (!params[i]) { set_error("null member parameters"); return CEL_ERR_ARG; }
    if (form != CEL_FORM_FUSED && form != CEL_FORM_MIXED) { set_error("batches use CEL_FORM_FUSED or CEL_FORM_MIXED"); return CEL_ERR_ARG; }
    if (int st = need_device()) return st;
    CEL_GUARD_BEGIN
    std::string err;
    cel_batch* b = cel::batch_create(n, params, bathy, bnx, bny, form, lanes, err);
    if (!b) { set_error(err); return CEL_ERR_ARG; }
    *out = b;
    return CEL_OK;
    CEL_GUARD_END
}

#define BAT(b) if (!b) { set_error("null batch"); return CEL_ERR_ARG; }
#define BRET(expr) do { std::string err; int st = (expr); if (st) set_error(err); return st; } while (0)

int cel_batch_destroy(cel_batch* b) { cel::batch_destroy(b); return CEL_OK; }
int cel_batch_set_stream(cel_batch* b, void* s) { BAT(b); CEL_GUARD_BEGIN BRET(cel::batch_set_stream(b, static_cast<cudaStream_t>(s), err)); CEL_GUARD_END }
int cel_batch_step(cel_batch* b, int n) {
    BAT(b);
    if (n < 0) { set_error("negative step count"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN BRET(cel::batch_step(b, n, err)); CEL_GUARD_END
}
int cel_batch_stats(cel_batch* b, cel_stats* out) {
    BAT(b);
    if (!out) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN BRET(cel::batch_stats(b, out, false, err)); CEL_GUARD_END
}
int cel_batch_stats_current(cel_batch* b, cel_stats* out) {
    BAT(b);
    if (!out) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN BRET(cel::batch_stats(b, out, true, err)); CEL_GUARD_END
}
int cel_batch_get_state(cel_batch* b, int i, float* rgba) {
    BAT(b);
    if (!rgba) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN BRET(cel::batch_get_state(b, i, rgba, err)); CEL_GUARD_END
}
int cel_batch_get_state_parts(cel_batch* b, int i, float* hi_rgba, float* lo_rgba) {
    BAT(b);
    if (!hi_rgba && !lo_rgba) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN BRET(cel::batch_get_state_parts(b, i, hi_rgba, lo_rgba, err)); CEL_GUARD_END
}
int cel_batch_set_state(cel_batch* b, int i, const float* rgba) {
    BAT(b);
    if (!rgba) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN BRET(cel::batch_set_state(b, i, rgba, err)); CEL_GUARD_END
}
int cel_batch_add_solitary_wave(cel_batch* b, int i, double H, double th, double xc, double yc) {
    BAT(b);
    CEL_GUARD_BEGIN BRET(cel::batch_add_solitary_wave(b, i, H, th, xc, yc, err)); CEL_GUARD_END
}
int cel_batch_set_bathymetry(cel_batch* b, int i, const float* bathy, int bnx, int bny) {
    BAT(b);
    CEL_GUARD_BEGIN BRET(cel::batch_set_bathymetry(b, i, bathy, bnx, bny, err)); CEL_GUARD_END
}
int cel_batch_get_aux(cel_batch* b, int i, float* rgba) {
    BAT(b);
    if (!rgba) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN BRET(cel::batch_get_aux(b, i, rgba, err)); CEL_GUARD_END
}
int cel_batch_use_graph(cel_batch* b, int enable) { BAT(b); CEL_GUARD_BEGIN BRET(cel::batch_use_graph(b, enable != 0, err)); CEL_GUARD_END }
long long cel_batch_cells(const cel_batch* b) { return b ? cel::batch_cells(b) : 0; }
int cel_batch_launches_per_step(const cel_batch* b) { return b ? cel::batch_launches_per_step(b) : 0; }
int cel_batch_set_timestep(cel_batch* b, const float* dt) {
    BAT(b);
    if (!dt) { set_error("null buffer"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN BRET(cel::batch_set_timestep(b, dt, err)); CEL_GUARD_END
}
int cel_batch_set_tuning(cel_batch* b, int tx, int ty, int pcr) {
    BAT(b);
    CEL_GUARD_BEGIN BRET(cel::batch_set_tuning(b, tx, ty, pcr, err)); CEL_GUARD_END
}
int cel_batch_get_tuning(const cel_batch* b, int* tx, int* ty, int* rows_per_step) {
    if (!b) { set_error("null batch"); return CEL_ERR_ARG; }
    return cel::batch_get_tuning(b, tx, ty, rows_per_step);
}
int cel_batch_col_chunks(const cel_batch* b) { return b ? cel::batch_col_chunks(b) : 0; }
int cel_batch_set_stencil_width(cel_batch* b, int threads) {
    BAT(b);
    CEL_GUARD_BEGIN BRET(cel::batch_set_stencil_width(b, threads, err)); CEL_GUARD_END
}
int cel_batch_stencil_width(const cel_batch* b) { return b ? cel::batch_stencil_width(b) : 0; }
int cel_batch_set_stencil_rows(cel_batch* b, int rows_per_step) {
    BAT(b);
    CEL_GUARD_BEGIN BRET(cel::batch_set_stencil_rows(b, rows_per_step, err)); CEL_GUARD_END
}
int cel_batch_autotune(cel_batch* b, int steps, int* tx, int* ty, double* ms) {
    BAT(b);
    CEL_GUARD_BEGIN BRET(cel::batch_autotune(b, steps, tx, ty, ms, err)); CEL_GUARD_END
}
int cel_batch_kernel_timing(cel_batch* b, int enable) {
    BAT(b);
    cel::batch_kernel_timing(b, enable != 0);
    return CEL_OK;
}

int cel_batch_lanes(const cel_batch* b) { return b ? cel::batch_lanes(b) : 0; }

int cel_kernel_times(void* handle, int is_batch, char (*names)[64], double* total_ms, long long* launches, int cap,
                     int* n) {
    if (!handle || !n) { set_error("null argument"); return CEL_ERR_ARG; }
    CEL_GUARD_BEGIN
    std::vector<cel::KernelTimer::Rec> recs;
    if (is_batch) {
        recs = cel::batch_kernel_records(static_cast<cel_batch*>(handle));
    } else {
        cel::KernelTimer* t = static_cast<cel_engine*>(handle)->impl->timer();
        t->collect();
        recs = t->recs;
    }
    int k = 0;
    for (const auto& r : recs) {
        if (k >= cap) break;
        if (names) std::snprintf(names[k], 64, "%s", r.name.c_str());
        if (total_ms) total_ms[k] = r.ms;
        if (launches) launches[k] = r.n;
        ++k;
    }
    *n = k;
    return CEL_OK;
    CEL_GUARD_END
}

int cel_selftest_reciprocal(const float* x, float* out, int n) {
    CEL_GUARD_BEGIN
    std::string err;
    const int st = cel::selftest_reciprocal(x, out, n, err);
    if (st) set_error(err);
    return st;
    CEL_GUARD_END
}

int cel_byte_model(int form, int correction_steps, double* stencil, double* step) {
    double s = 0, t = 0;
    cel::byte_model(form, correction_steps, s, t);
    if (stencil) *stencil = s;
    if (step) *step = t;
    return CEL_OK;
}

}  // extern "C"
