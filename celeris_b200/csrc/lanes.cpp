// A batch as a set of lanes.
//
// The members are split into lanes of about equal interior cell counts; each lane is a complete
// batched engine (fused.cu) with its own stream, work lists and CUDA graphs.  Lane 0 runs on the
// batch's stream (the caller's, once set); every other lane has its own non-blocking stream that
// waits for the batch stream at the start of each call (a fork) and that the batch stream waits
// for at its end (a join), so to the caller a batch behaves as one stream-ordered object.  A step
// launches the lanes' graphs in turn, one physical step at a time, and the GPU runs them side by
// side: one lane's boundary strips, clock advance and kernel tails, which leave most SMs idle,
// overlap another lane's stencil.  Every member's arithmetic is the same in any lane, so the
// results do not depend on the split.
#include <algorithm>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "batch.hpp"

struct cel_batch {
    std::vector<cel_lane*> lanes;
    std::vector<std::vector<int>> members;   // lane -> the caller's member indices, ascending
    std::vector<int> lane_of, slot_of;        // member -> lane, index within the lane
    bool timing = false;                      // kernel timing: lanes run one after another
    cudaEvent_t ev_fork = nullptr;
    std::vector<cudaEvent_t> ev_lane;         // one per lane: joins and the chain of timed steps

    ~cel_batch() {
        for (cel_lane* l : lanes) cel::lane_destroy(l);
        if (ev_fork) cudaEventDestroy(ev_fork);
        for (cudaEvent_t e : ev_lane)
            if (e) cudaEventDestroy(e);
        (void)cudaGetLastError();
    }
};

namespace cel {

namespace {

#define G_TRY(expr)                                                                     \
    do {                                                                                \
        cudaError_t _e = (expr);                                                        \
        if (_e != cudaSuccess) { err = std::string(#expr) + ": " + cudaGetErrorString(_e); return CEL_ERR_CUDA; } \
    } while (0)

cudaStream_t batch_stream(const cel_batch* g) { return lane_stream(g->lanes[0]); }

// lanes 1.. wait for the work the batch stream holds so far
int fork_lanes(cel_batch* g, std::string& err) {
    if (g->lanes.size() < 2) return CEL_OK;
    G_TRY(cudaEventRecord(g->ev_fork, batch_stream(g)));
    for (size_t l = 1; l < g->lanes.size(); ++l) G_TRY(cudaStreamWaitEvent(lane_stream(g->lanes[l]), g->ev_fork, 0));
    return CEL_OK;
}

// the batch stream waits for the work of lanes 1..
int join_lanes(cel_batch* g, std::string& err) {
    for (size_t l = 1; l < g->lanes.size(); ++l) {
        G_TRY(cudaEventRecord(g->ev_lane[l], lane_stream(g->lanes[l])));
        G_TRY(cudaStreamWaitEvent(batch_stream(g), g->ev_lane[l], 0));
    }
    return CEL_OK;
}

// f(lane) for every lane, between a fork and a join
template <class F>
int each(cel_batch* g, std::string& err, F f) {
    if (int e = fork_lanes(g, err)) return e;
    int rc = CEL_OK;
    for (cel_lane* l : g->lanes)
        if ((rc = f(l))) break;
    std::string jerr;
    const int rj = join_lanes(g, jerr);
    if (!rc && rj) err = jerr;
    return rc ? rc : rj;
}

int check_member(const cel_batch* g, int i, std::string& err) {
    if (i < 0 || i >= int(g->lane_of.size())) { err = "member index out of range"; return CEL_ERR_ARG; }
    return CEL_OK;
}

// f(lane, index within the lane) for member i
template <class F>
int on_member(cel_batch* g, int i, std::string& err, F f) {
    if (int e = check_member(g, i, err)) return e;
    if (int e = fork_lanes(g, err)) return e;
    const int rc = f(g->lanes[g->lane_of[i]], g->slot_of[i]);
    std::string jerr;
    const int rj = join_lanes(g, jerr);
    if (!rc && rj) err = jerr;
    return rc ? rc : rj;
}

}  // namespace

cel_batch* batch_create(int n, const cel_params* const* params, const float* const* bathy, const int* bnx,
                        const int* bny, int form, int lanes, std::string& err) {
    if (n <= 0) { err = "a batch needs at least one member"; return nullptr; }
    // the lanes step together, so the whole batch shares one pass sequence (whatever the split)
    for (int i = 1; i < n; ++i) {
        if (params[i]->correction_steps != params[0]->correction_steps) {
            err = "batch members must share correctionStepsNum";
            return nullptr;
        }
        if ((params[i]->adaptive != 0) != (params[0]->adaptive != 0)) {
            err = "batch members must share the adaptive time-step setting";
            return nullptr;
        }
    }
    int L = lanes > 0 ? lanes : (n >= 2 ? 2 : 1);
    L = std::min(L, n);
    auto g = std::make_unique<cel_batch>();
    // largest members first, each onto the lane with the fewest cells so far
    std::vector<long long> cells(n);
    for (int i = 0; i < n; ++i) cells[i] = (long long)params[i]->nx * params[i]->ny;
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cells[a] > cells[b]; });
    std::vector<long long> load(L, 0);
    g->members.assign(L, {});
    for (int i : order) {
        const int l = int(std::min_element(load.begin(), load.end()) - load.begin());
        g->members[l].push_back(i);
        load[l] += cells[i];
    }
    g->lane_of.assign(n, 0);
    g->slot_of.assign(n, 0);
    for (int l = 0; l < L; ++l) {
        std::vector<int>& ms = g->members[l];
        std::sort(ms.begin(), ms.end());
        std::vector<const cel_params*> p;
        std::vector<const float*> z;
        std::vector<int> bx, by;
        for (size_t k = 0; k < ms.size(); ++k) {
            g->lane_of[ms[k]] = l;
            g->slot_of[ms[k]] = int(k);
            p.push_back(params[ms[k]]);
            z.push_back(bathy[ms[k]]);
            bx.push_back(bnx[ms[k]]);
            by.push_back(bny[ms[k]]);
        }
        cel_lane* ln = lane_create(int(ms.size()), p.data(), z.data(), bx.data(), by.data(), form, err);
        if (!ln) return nullptr;   // the lanes made so far go with g
        g->lanes.push_back(ln);
    }
    if (L > 1) {
        if (cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming) != cudaSuccess) {
            err = "cudaEventCreate failed";
            return nullptr;
        }
        g->ev_lane.assign(L, nullptr);
        for (cudaEvent_t& e : g->ev_lane)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
                err = "cudaEventCreate failed";
                return nullptr;
            }
    }
    return g.release();
}

void batch_destroy(cel_batch* b) { delete b; }

int batch_lanes(const cel_batch* b) { return int(b->lanes.size()); }

int batch_set_stream(cel_batch* b, cudaStream_t s, std::string& err) {
    // lanes 1.. finish what they hold, then order themselves against the new batch stream
    for (size_t l = 1; l < b->lanes.size(); ++l) G_TRY(cudaStreamSynchronize(lane_stream(b->lanes[l])));
    return lane_set_stream(b->lanes[0], s, err);
}

int batch_step(cel_batch* b, int nsteps, std::string& err) {
    if (nsteps < 0) { err = "negative step count"; return CEL_ERR_ARG; }
    if (int e = fork_lanes(b, err)) return e;
    const size_t L = b->lanes.size();
    if (b->timing && L > 1) {
        // kernel timing: each lane takes all its steps after the previous lane has finished, so
        // that every launch's event-timed span covers that launch alone
        for (size_t l = 0; l < L; ++l) {
            if (l > 0) {
                G_TRY(cudaEventRecord(b->ev_lane[l - 1], lane_stream(b->lanes[l - 1])));
                G_TRY(cudaStreamWaitEvent(lane_stream(b->lanes[l]), b->ev_lane[l - 1], 0));
            }
            if (int e = lane_step(b->lanes[l], nsteps, err)) return e;
        }
    } else {
        for (int k = 0; k < nsteps; ++k)
            for (cel_lane* l : b->lanes)
                if (int e = lane_step(l, 1, err)) return e;
    }
    return join_lanes(b, err);
}

int batch_stats(cel_batch* b, cel_stats* out, bool current, std::string& err) {
    // every lane's read-back is queued before the first wait, so the copies overlap.  No fork or
    // join: the statistics read only what the lanes' own streams wrote, and the call returns after
    // everything it read has arrived.
    for (cel_lane* ln : b->lanes)
        if (int e = lane_stats_enqueue(ln, current, err)) return e;
    std::vector<cel_stats> tmp;
    for (size_t l = 0; l < b->lanes.size(); ++l) {
        const std::vector<int>& ms = b->members[l];
        tmp.resize(ms.size());
        if (int e = lane_stats_finish(b->lanes[l], tmp.data(), current, err)) return e;
        for (size_t k = 0; k < ms.size(); ++k) out[ms[k]] = tmp[k];
    }
    return CEL_OK;
}

int batch_get_state(cel_batch* b, int i, float* rgba, std::string& err) {
    return on_member(b, i, err, [&](cel_lane* l, int k) { return lane_get_state(l, k, rgba, err); });
}

int batch_get_state_parts(cel_batch* b, int i, float* hi_rgba, float* lo_rgba, std::string& err) {
    return on_member(b, i, err, [&](cel_lane* l, int k) { return lane_get_state_parts(l, k, hi_rgba, lo_rgba, err); });
}

int batch_set_state(cel_batch* b, int i, const float* rgba, std::string& err) {
    return on_member(b, i, err, [&](cel_lane* l, int k) { return lane_set_state(l, k, rgba, err); });
}

int batch_get_aux(cel_batch* b, int i, float* rgba, std::string& err) {
    return on_member(b, i, err, [&](cel_lane* l, int k) { return lane_get_aux(l, k, rgba, err); });
}

int batch_set_bathymetry(cel_batch* b, int i, const float* z, int bnx, int bny, std::string& err) {
    return on_member(b, i, err, [&](cel_lane* l, int k) { return lane_set_bathymetry(l, k, z, bnx, bny, err); });
}

int batch_add_solitary_wave(cel_batch* b, int i, double H, double theta_deg, double xc, double yc, std::string& err) {
    return on_member(b, i, err,
                     [&](cel_lane* l, int k) { return lane_add_solitary_wave(l, k, H, theta_deg, xc, yc, err); });
}

int batch_use_graph(cel_batch* b, bool enable, std::string& err) {
    for (cel_lane* l : b->lanes)
        if (int e = lane_use_graph(l, enable, err)) return e;
    return CEL_OK;
}

long long batch_cells(const cel_batch* b) {
    long long c = 0;
    for (const cel_lane* l : b->lanes) c += lane_cells(l);
    return c;
}

int batch_set_timestep(cel_batch* b, const float* dt, std::string& err) {
    // No fork or join: each lane copies the host values into its pinned buffer and uploads them on
    // its own stream, ahead of its next step.  Every value is checked first, so that a refused
    // call changes no lane.
    for (size_t i = 0; i < b->lane_of.size(); ++i)
        if (!(dt[i] > 0.f)) { err = "time steps must be > 0"; return CEL_ERR_ARG; }
    std::vector<float> part;
    for (size_t l = 0; l < b->lanes.size(); ++l) {
        const std::vector<int>& ms = b->members[l];
        part.resize(ms.size());
        for (size_t k = 0; k < ms.size(); ++k) part[k] = dt[ms[k]];
        if (int e = lane_set_timestep(b->lanes[l], part.data(), err)) return e;
    }
    return CEL_OK;
}

int batch_set_tuning(cel_batch* b, int tx, int ty, int pcr, std::string& err) {
    return each(b, err, [&](cel_lane* l) { return lane_set_tuning(l, tx, ty, pcr, err); });
}

int batch_get_tuning(const cel_batch* b, int* tx, int* ty, int* rps) { return lane_get_tuning(b->lanes[0], tx, ty, rps); }

int batch_set_stencil_rows(cel_batch* b, int rps, std::string& err) {
    return each(b, err, [&](cel_lane* l) { return lane_set_stencil_rows(l, rps, err); });
}

int batch_set_stencil_width(cel_batch* b, int threads, std::string& err) {
    return each(b, err, [&](cel_lane* l) { return lane_set_stencil_width(l, threads, err); });
}

int batch_stencil_width(const cel_batch* b) { return lane_stencil_width(b->lanes[0]); }

// Times `steps` physical steps of the whole batch (all lanes side by side) for each candidate, in
// the launch mode the batch is set to, two rounds in turn, and keeps the fastest by its better
// round.  The stencil and the solvers are separate kernels, so the search runs in two stages: the
// stencil (rows per step and width x strip height) with the default solvers, then the column solver
// (band width x chunks per column, i.e. the switch point from the carry scan to serial sweeps, and
// the cluster solver where the tallest member fits its chunks) with the chosen stencil.  Every lane takes the same candidate and the same steps, so the members stay
// in step with one another.
int batch_autotune(cel_batch* b, int steps, int* tx, int* ty, double* best_ms, std::string& err) {
    if (steps < 1) { err = "autotune needs at least one step per candidate"; return CEL_ERR_ARG; }
    int max_ny = 0;
    for (const cel_lane* l : b->lanes) max_ny = std::max(max_ny, lane_max_ny(l));
    struct Cand { int cw, mh, rps, mw, nt; };
    auto configure = [&](const Cand& c) {
        return each(b, err, [&](cel_lane* l) { return lane_configure(l, c.cw, c.mh, c.rps, c.mw, c.nt, err); });
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    G_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        err = "cudaEventCreate failed";
        return CEL_ERR_CUDA;
    }
    const cudaStream_t s = batch_stream(b);
    int rc = CEL_OK;
    // times every candidate (two rounds) and returns the index of the fastest, or -1 on error
    auto search = [&](const std::vector<Cand>& cand, double& best_out) -> int {
        std::vector<double> best(cand.size(), 1e300);
        for (int round = 0; round < 2 && !rc; ++round)
            for (size_t k = 0; k < cand.size() && !rc; ++k) {
                if ((rc = configure(cand[k]))) break;
                if ((rc = batch_step(b, 2, err))) break;   // warm-up (captures the graphs in graph mode)
                cudaEventRecord(e0, s);
                if ((rc = batch_step(b, steps, err))) break;
                cudaEventRecord(e1, s);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                best[k] = std::min(best[k], double(ms) / steps);
            }
        if (rc) return -1;
        const size_t kb = size_t(std::min_element(best.begin(), best.end()) - best.begin());
        best_out = best[kb];
        return int(kb);
    };
    const bool cw16_fits = sizeof(float) * size_t(max_ny) * 16 + COLS_STATIC_SMEM <= 227 * 1024;
    const int cw0 = cw16_fits ? 16 : 8;
    std::vector<Cand> stencil;
    const int variants[3][2] = {{1, 128}, {2, 128}, {2, 96}};   // stencil rows per step, stencil width
    for (const auto& v : variants)
        for (int mh : {32, 64, 128}) stencil.push_back({cw0, mh, v[0], v[1], 512});
    double ms = 0.0;
    const int ks = search(stencil, ms);
    std::vector<Cand> solver;
    if (ks >= 0) {
        const Cand st = stencil[size_t(ks)];
        solver.push_back({1, st.mh, st.rps, st.mw, 512});
        for (int cw : {8, 16, 32})
            if (sizeof(float) * size_t(max_ny) * cw + COLS_STATIC_SMEM <= 227 * 1024)
                for (int nt : {256, 512}) solver.push_back({cw, st.mh, st.rps, st.mw, nt});
        // the cluster solver (32-column bands, 32 or 64 chunks per column of at most 16 rows each,
        // clusters of 4 or 8 CTAs)
        for (int nt : {1024, 2048})
            if (max_ny <= nt / 2) solver.push_back({32, st.mh, st.rps, st.mw, nt});
        // the tile-transposed solver (16-column bands, the band's forward values in shared memory)
        if (sizeof(float) * 16 * size_t((max_ny + 3) & ~3) + 27 * 1024 <= 227 * 1024)
            solver.push_back({16, st.mh, st.rps, st.mw, 16});
    }
    const int kb = ks >= 0 ? search(solver, ms) : -1;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if ((rc = configure(solver[size_t(kb)]))) return rc;
    if (tx) *tx = solver[size_t(kb)].cw;
    if (ty) *ty = solver[size_t(kb)].mh;
    if (best_ms) *best_ms = ms;
    return CEL_OK;
}

int batch_col_chunks(const cel_batch* b) { return lane_col_chunks(b->lanes[0]); }

void batch_kernel_timing(cel_batch* b, bool enable) {
    b->timing = enable;
    for (cel_lane* l : b->lanes) lane_timer(l)->enabled = enable;
}

std::vector<KernelTimer::Rec> batch_kernel_records(cel_batch* b) {
    std::vector<KernelTimer::Rec> out;
    for (cel_lane* l : b->lanes) {
        KernelTimer* t = lane_timer(l);
        t->collect();
        for (const KernelTimer::Rec& r : t->recs) {
            auto it = std::find_if(out.begin(), out.end(), [&](const KernelTimer::Rec& o) { return o.name == r.name; });
            if (it == out.end()) out.push_back(r);
            else { it->ms += r.ms; it->n += r.n; }
        }
    }
    return out;
}

int batch_launches_per_step(const cel_batch* b) {
    int n = 0;
    for (const cel_lane* l : b->lanes) n += lane_launches_per_step(l);
    return n;
}

}  // namespace cel
