// Host-side time-scheme state machine of the reference (engine.cpp:1476-1521, initial values
// engine.cpp:3254-3269) and the resetTimestep dt logic (engine.cpp:1700-1729), shared by all
// forms so that every form runs the same pass sequence:
//   passes 1-2 Euler; then an AB3 predictor followed by N AM4 correctors; history rotation,
//   the dt queue shift and total_time += dt happen only after the last pass of a step.
#pragma once

#include <algorithm>

#include "celeris_internal.hpp"

namespace cel {

struct Scheme {
    int N = 0;                   // correctionStepsNum
    bool adaptive = false;
    int time_scheme = CEL_SCHEME_EULER;
    int timestep_count = 1;
    int correction_steps_count = 0;
    float dt = 0, dt_old = 0, dt_old_old = 0;
    float total_time = 0;        // float, as the reference (engine.hpp:302)
    int last_count = 0;          // timestep_count tested by the reference's log dump (engine.cpp:1491)
    float last_start_time = 0;   // total_time before the latest step's dt was added
    double total_time_d = 0;     // FP64 copy (the mixed form's wave-maker phase)
    bool initialized = false, target_cfl_set = false;
    float target_cfl = 0;
    float base_dt = 0, min_ratio = 0.05f, ema_alpha = 0.5f;

    void reset(const cel_params& p) {
        N = p.correction_steps;
        adaptive = p.adaptive != 0;
        time_scheme = CEL_SCHEME_EULER;
        timestep_count = 1;
        correction_steps_count = N;
        dt = dt_old = dt_old_old = 0;
        total_time = 0;
        total_time_d = 0;
        last_count = 0;
        last_start_time = 0;
        initialized = false;
        target_cfl_set = false;
        target_cfl = 0;
        base_dt = float(p.timestep);
        min_ratio = float(p.min_timestep_ratio);
        ema_alpha = float(p.ema_alpha);
    }
    // resetTimestep's dt selection; cfl is the max CFL rate of the current state.
    float choose_dt(float cfl) {
        if (cfl > 0 && !target_cfl_set && adaptive) { target_cfl = base_dt * cfl; target_cfl_set = true; }
        if (!initialized) {
            dt = base_dt;
            cfl = (adaptive ? target_cfl : 0.f) / dt;
            dt_old_old = dt;
            dt_old = dt;
            initialized = true;
        }
        if (time_scheme == CEL_SCHEME_PREDICTOR_ADAPTIVE) {
            const float tgt = std::max(target_cfl / cfl, base_dt * min_ratio);
            dt = tgt > dt_old ? ema_alpha * tgt + (1 - ema_alpha) * dt_old : tgt;
        } else {
            dt = base_dt;
        }
        return cfl;
    }
    bool is_predictor() const {
        return time_scheme == CEL_SCHEME_PREDICTOR || time_scheme == CEL_SCHEME_PREDICTOR_ADAPTIVE;
    }
    // Called after a pass; returns true when the bookkeeping (history rotation, dt queue
    // shift, time advance) ran.
    bool after_pass() {
        if (timestep_count >= 2) {
            if (correction_steps_count == N) {
                time_scheme = adaptive ? CEL_SCHEME_PREDICTOR_ADAPTIVE : CEL_SCHEME_PREDICTOR;
                correction_steps_count = 0;
            } else {
                time_scheme = CEL_SCHEME_CORRECTOR;
                correction_steps_count++;
            }
        }
        if (time_scheme != CEL_SCHEME_CORRECTOR) {
            last_count = timestep_count;
            last_start_time = total_time;
            timestep_count++;
            dt_old_old = dt_old;
            dt_old = dt;
            total_time += dt;
            total_time_d += double(dt);
            return true;
        }
        return false;
    }
};

}  // namespace cel
