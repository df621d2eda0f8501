// C entry point over the reference's own bathymetry code (terrain_heightfield.cpp and
// settings.cpp, compiled unchanged by ref_build.py).  Test infrastructure only: it lets the tests
// compare the product's .cbf reader and bottom sampling with the reference's.
#include <cstring>
#include <string>

#include "settings.hpp"
#include "terrain_heightfield.hpp"

// main.cpp:74-75 owns the settings object; this stands in for it.
InitSetting* p_initSetting = new InitSetting();
InitSetting& initSetting = *p_initSetting;

extern "C" int ref_bottom(const char* cbf_path, int nx, int ny, double width, double length, double swl,
                          double gravity, float* out_by_bx_ba) {
    initSetting.bathymetryFileName = cbf_path;
    initSetting.rereadBathy = true;
    initSetting.stillWaterElevation = float(swl);
    SetSetting("mesh_size_x", float(nx));
    SetSetting("mesh_size_y", float(ny));
    SetSetting("valley_width", float(width));
    SetSetting("valley_length", float(length));
    SetSetting("gravity", float(gravity));
    UpdateTerrainHeightfield();
    const size_t n = size_t(nx + 4) * (ny + 4);
    for (size_t i = 0; i < n; ++i) {
        out_by_bx_ba[3 * i] = g_bottom[i].BY;
        out_by_bx_ba[3 * i + 1] = g_bottom[i].BX;
        out_by_bx_ba[3 * i + 2] = g_bottom[i].BA;
    }
    return 0;
}

extern "C" float ref_terrain_height(float x, float y) { return GetTerrainHeight(x, y); }
