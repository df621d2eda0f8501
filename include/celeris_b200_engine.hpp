// Drop-in for the compute half of the reference's ShallowWaterEngine (engine.hpp:58-312), on top
// of the C ABI in celeris_b200.h.  The reference's main loop keeps its calls: remesh, resetTimestep,
// timestep, afterTimestep, newTerrainSettings, getWaterHeight, addSolitaryWave.  Errors come back
// from the library as status codes and are turned into C++ exceptions here, as the reference's own
// engine reports them.  Header only; link with -lceleris_b200.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "celeris_b200.h"

class CelerisB200Engine {
public:
    // engine.cpp:709-724 reads initSetting / g_settings; here the same values come from the .cml
    // (readInputCML, main.cpp:500-913).  form: CEL_FORM_PLAIN, CEL_FORM_FUSED or CEL_FORM_MIXED.
    CelerisB200Engine(const std::string& cml_path, const std::vector<float>& bathy, int bnx, int bny,
                      int form = CEL_FORM_MIXED) {
        check(cel_params_from_cml(cml_path.c_str(), &p_));
        const int st = cel_create(&p_, bathy.empty() ? nullptr : bathy.data(), bnx, bny, form, &h_);
        if (st != CEL_OK) {
            const std::string msg = cel_last_error();
            cel_params_release(&p_);
            throw std::runtime_error(msg);
        }
    }
    ~CelerisB200Engine() {
        cel_destroy(h_);
        cel_params_release(&p_);
    }
    CelerisB200Engine(const CelerisB200Engine&) = delete;
    CelerisB200Engine& operator=(const CelerisB200Engine&) = delete;

    void remesh() { check(cel_remesh(h_)); }                                        // engine.hpp:64
    cel_stats resetTimestep(float realworld_dt, float elapsed) {                    // engine.hpp:81
        cel_stats s;
        check(cel_reset_timestep(h_, realworld_dt, elapsed, &s));
        return s;
    }
    void timestep() { check(cel_timestep(h_)); }                                    // engine.hpp:73
    // engine.cpp:1523-1535: the GUI's "save" flags write the inundation map and the bathymetry
    void afterTimestep(bool& saveInundation, bool& saveBathymetry) {                // engine.hpp:76
        int nx, ny;
        check(cel_get_dims(h_, &nx, &ny));
        std::vector<float> buf(size_t(nx + 4) * (ny + 4) * 4);
        if (saveInundation) {   // <logPath>/<Y-M-D H-M-S>-inundation.txt, as dumpInundationToFile
            check(cel_get_aux(h_, buf.data()));
            check(cel_write_inundation(&p_, buf.data(), nullptr));
            saveInundation = false;
        }
        if (saveBathymetry) {   // <logPath>/<Y-M-D H-M-S>.cbf, as dumpBathymetryToFile
            check(cel_get_bottom(h_, buf.data()));
            check(cel_write_bathymetry(&p_, buf.data(), nullptr));
            saveBathymetry = false;
        }
    }
    void newTerrainSettings(const std::vector<float>& bathy, int bnx, int bny) {     // engine.hpp:63
        check(cel_set_bathymetry(h_, bathy.data(), bnx, bny));                      // depth kept, aux cleared
    }
    float getWaterHeight(float x, float y) {                                        // engine.hpp:93
        float eta = 0;
        check(cel_get_water_height(h_, x, y, &eta));
        return eta;
    }
    void addSolitaryWave(float H, float theta, float xc, float yc) {                 // engine.cpp:2154-2219
        check(cel_add_solitary_wave(h_, H, theta, xc, yc));
    }
    // The renderer's txState: RGBA32F, (nx+4) x (ny+4), {w, hu, hv, 0}; copy into a staging texture
    void readState(std::vector<float>& rgba) {
        int nx, ny;
        check(cel_get_dims(h_, &nx, &ny));
        rgba.resize(size_t(nx + 4) * (ny + 4) * 4);
        check(cel_get_state(h_, rgba.data()));
    }
    const cel_params& params() const { return p_; }

private:
    static void check(int st) {
        if (st != CEL_OK) throw std::runtime_error(cel_last_error());
    }
    cel_params p_{};
    cel_engine* h_ = nullptr;
};
