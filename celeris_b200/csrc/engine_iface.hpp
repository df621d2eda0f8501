// Abstract single-domain engine behind the C ABI handle (`cel_engine`), so the plain form and
// the fused forms present the same ShallowWaterEngine-shaped interface.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "celeris_internal.hpp"

namespace cel {

struct KernelTimer {
    bool enabled = false;
    struct Rec { std::string name; double ms = 0; long long n = 0; };
    std::vector<Rec> recs;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t get_event();
    void begin(cudaStream_t s, const char* name, cudaEvent_t& ev0, int& idx);
    void end(cudaStream_t s, int idx, cudaEvent_t ev0);
    void collect();  // synchronizes pending events and accumulates
    ~KernelTimer();
};

// Scoped timing of one launch (no-op unless enabled).
struct TimedLaunch {
    KernelTimer* t; cudaStream_t s; cudaEvent_t e0 = nullptr; int idx = -1;
    TimedLaunch(KernelTimer* tt, cudaStream_t ss, const char* name) : t(tt), s(ss) {
        if (t && t->enabled) t->begin(s, name, e0, idx);
    }
    ~TimedLaunch() { if (t && t->enabled) t->end(s, idx, e0); }
};

class EngineIface {
public:
    virtual ~EngineIface() {}
    virtual int remesh() = 0;
    virtual int set_state(const float* rgba) = 0;
    virtual int get_state(float* rgba) = 0;
    virtual int get_bottom(float* b3) = 0;
    virtual int get_aux(float* rgba) = 0;
    virtual int reset_timestep(float realworld_dt, float elapsed, cel_stats* out) = 0;
    virtual int timestep() = 0;
    virtual int timesteps(int n) = 0;
    virtual int physical_steps(int n) = 0;
    virtual int get_stats(cel_stats* out) = 0;
    virtual int add_solitary_wave(double H, double theta_deg, double xc, double yc) = 0;
    // newTerrainSettings (engine.cpp:820-823, 3313-3379) with a new bathymetry grid
    virtual int set_bathymetry(const float* z, int bnx, int bny) = 0;
    // getWaterHeight (engine.cpp:4994-5012): terrain height at (x, y) plus the mean depth of the
    // GetStats 4x4 block holding the point
    virtual int water_height(float x, float y, float* out) = 0;
    virtual int set_stream(cudaStream_t s) = 0;
    virtual int synchronize() = 0;
    virtual int set_tuning(int tx, int ty, int pcr) = 0;
    virtual KernelTimer* timer() = 0;
    virtual int nx() const = 0;
    virtual int ny() const = 0;
    std::string err;
    float log_elapsed = 0.f;   // `elapsed` of the latest cel_reset_timestep (the log's elapsed time)
};

EngineIface* make_plain_engine(const cel_params& p, const float* bathy, int bnx, int bny, std::string& err);
EngineIface* make_fused_engine(const cel_params& p, const float* bathy, int bnx, int bny, int form, std::string& err);

#define CEL_CUDA_TRY(expr)                                                              \
    do {                                                                                \
        cudaError_t _e = (expr);                                                        \
        if (_e != cudaSuccess) {                                                        \
            err = std::string(#expr) + ": " + cudaGetErrorString(_e);                   \
            return CEL_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)

}  // namespace cel
