// C entry point over the reference's own spectrum wave-maker, ShallowWaterEngine::
// generateSpectrumWaves (engine.cpp:3559-3776), extracted from engine.cpp by ref_build.py into
// spectrum_ref.inc.  Test infrastructure only.  engine.cpp does not build here (Direct3D 11,
// Windows, Boost), so the extraction turns the member function into a free function and gives it
// what it reads from the engine's world:
//   GetSetting("gravity")       -> ref_gravity (settings.cpp's table value, set per call)
//   boost::math::lgamma<float>  -> ref_lgammaf, i.e. std::lgamma on a float
//   initSetting.logPath         -> ref_log_path (the folder the component file goes to)
//   srand(time(0))              -> srand(ref_seed), so that rand()'s phase sequence is repeatable
// Everything else, the arithmetic and the file it writes included, is the reference's text.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "settings.hpp"

static float ref_gravity = 9.81f;
static std::string ref_log_path = ".";
static unsigned ref_seed = 1;
static float ref_lgammaf(float x) { return std::lgamma(x); }

#include "spectrum_ref.inc"

// Runs the reference's generator for one setting; writes the component file into `dir` and copies
// its path into out_path (cap bytes).  Returns 0, or 1 when the reference returned "NA" (a zero
// input), 2 when out_path is too small.
extern "C" int ref_spectrum_file(double hs, double tp, double mean_theta_deg, double depth, double gravity,
                                 unsigned seed, const char* dir, char* out_path, int cap) {
    IrregularWaveSpectrumSetting s;
    s.useSpectrum = true;
    s.significant_waveheight = float(hs);
    s.peak_period = float(tp);
    s.mean_theta = float(mean_theta_deg);
    s.depth_at_source = float(depth);
    ref_gravity = float(gravity);
    ref_log_path = dir;
    ref_seed = seed;
    const std::string f = ref_generateSpectrumWaves(s, "West");
    if (f == "NA") return 1;
    if (int(f.size()) + 1 > cap) return 2;
    std::memcpy(out_path, f.c_str(), f.size() + 1);
    return 0;
}
