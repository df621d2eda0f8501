// File output of the engine: the <logData> time series (time axis, ranges, gauges), the
// maximum-inundation map, the bathymetry grid and hot-start files, in the reference's text
// formats.  Host code only: callers hand in host copies of the texture-layout arrays.
//
// Formats follow the reference's writers:
//   st_DumpToFile         engine.cpp:628-675   time axis, elapsed time, ranges, gauges
//   dumpInundationToFile  engine.cpp:781-817   "[nx]/[ny]" header, max depth per texel
//   dumpBathymetryToFile  engine.cpp:750-779   .cbf text grid of the interior bottom
//   hot-start reader      engine.cpp:2943-2966 "i j w hu hv a" per texel, j outer
// Numbers go through std::ostream with its default format (6 significant digits, %g style),
// as the reference's ofstream writes them; hot-start files use 9 significant digits instead so
// that every float reads back exactly.
#include "celeris_internal.hpp"

#include <ctime>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>

namespace cel {

namespace {

// "<year>-<month>-<day> <hour>-<min>-<sec>" in local time, without zero padding
// (engine.cpp:757-760, 789-792).
std::string stamp() {
    const std::time_t now = std::time(nullptr);
    std::tm t{};
    localtime_r(&now, &t);
    std::ostringstream s;
    s << t.tm_year + 1900 << "-" << t.tm_mon + 1 << "-" << t.tm_mday << " " << t.tm_hour << "-" << t.tm_min << "-"
      << t.tm_sec;
    return s.str();
}

// Opens a file for appending (the reference opens every log file with ios::app).
bool open_append(std::ofstream& f, const std::string& path, std::string& err) {
    f.open(path.c_str(), std::ios::out | std::ios::app);
    if (!f) { err = "cannot open " + path + " for writing"; return false; }
    return true;
}

// One texel as a log line: "i\tj\tw\thu\thv\ta\n".
void texel_line(std::ostream& o, const float* rgba, int NX, int i, int j) {
    const float* t = rgba + (size_t(j) * NX + i) * 4;
    o << i << "\t" << j << "\t" << t[0] << "\t" << t[1] << "\t" << t[2] << "\t" << t[3] << "\n";
}

}  // namespace

int log_validate(const cel_log& lg, int nx, int ny, std::string& err) {
    if (!lg.do_log) return CEL_OK;
    if (lg.log_step < 1) { err = "logData logStep must be >= 1"; return CEL_ERR_ARG; }
    const int xmax = nx + 3, ymax = ny + 3;
    auto inside = [&](int x, int y) { return x >= 0 && y >= 0 && x <= xmax && y <= ymax; };
    for (int r = 0; r < lg.n_ranges; ++r) {
        const cel_log_range& R = lg.ranges[r];
        if (R.x0 > R.x1 || R.y0 > R.y1) continue;  // writes nothing, as the reference's loops
        if (!inside(R.x0, R.y0) || !inside(R.x1, R.y1)) {
            err = "log range '" + std::string(R.name) + "' reaches outside the " + std::to_string(xmax + 1) + "x" +
                  std::to_string(ymax + 1) + " texture";
            return CEL_ERR_ARG;
        }
    }
    for (int g = 0; g < lg.n_gauges; ++g)
        if (!inside(lg.gauges[g][0], lg.gauges[g][1])) {
            err = "gauge " + std::to_string(g) + " (" + std::to_string(lg.gauges[g][0]) + "," +
                  std::to_string(lg.gauges[g][1]) + ") lies outside the texture";
            return CEL_ERR_ARG;
        }
    return CEL_OK;
}

int log_dump(const cel_log& lg, const float* rgba, int nx, int ny, float total_time, float elapsed, std::string& err) {
    if (int st = log_validate(lg, nx, ny, err)) return st;
    const std::string dir = std::string(lg.path) + "/";
    const int NX = nx + 4;
    {
        std::ofstream f;
        if (!open_append(f, dir + lg.time_axis_name + ".txt", err)) return CEL_ERR_IO;
        f << total_time << "\n";
    }
    {
        std::ofstream f;
        if (!open_append(f, dir + lg.time_axis_name + "-elapsed.txt", err)) return CEL_ERR_IO;
        f << elapsed << "\n";
    }
    for (int r = 0; r < lg.n_ranges; ++r) {
        const cel_log_range& R = lg.ranges[r];
        std::ofstream f;
        if (!open_append(f, dir + R.name + ".txt", err)) return CEL_ERR_IO;
        for (int j = R.y0; j <= R.y1; ++j)
            for (int i = R.x0; i <= R.x1; ++i) texel_line(f, rgba, NX, i, j);
        if (!f) { err = std::string("write failed: ") + R.name; return CEL_ERR_IO; }
    }
    // the gauges file is opened (and so created) on every dump, gauges or not (engine.cpp:663-667)
    std::ofstream f;
    if (!open_append(f, dir + lg.gauges_name + ".txt", err)) return CEL_ERR_IO;
    for (int g = 0; g < lg.n_gauges; ++g) texel_line(f, rgba, NX, lg.gauges[g][0], lg.gauges[g][1]);
    if (!f) { err = "write failed: gauges"; return CEL_ERR_IO; }
    return CEL_OK;
}

int write_inundation(const cel_log& lg, const float* aux, int nx, int ny, const char* path, std::string& err) {
    const std::string name = path ? std::string(path) : std::string(lg.path) + "/" + stamp() + "-inundation.txt";
    std::ofstream f;
    if (!open_append(f, name, err)) return CEL_ERR_IO;
    f << "[nx] " << nx << "\n" << "[ny] " << ny << "\n" << "\n\n"
      << "# This file contains the maximum depth of inundation on each point, in meters." << "\n\n"
      << "====================================" << "\n";
    const int NX = nx + 4;
    for (int j = 2; j < ny + 2; ++j) {
        for (int i = 2; i <= nx + 2; ++i) f << aux[(size_t(j) * NX + i) * 4] << "\t";
        f << "\n";
    }
    if (!f) { err = "write failed: " + name; return CEL_ERR_IO; }
    return CEL_OK;
}

int write_bathymetry(const cel_log& lg, const float* b3, int nx, int ny, const char* path, std::string& err) {
    const std::string name = path ? std::string(path) : std::string(lg.path) + "/" + stamp() + ".cbf";
    std::ofstream f;
    if (!open_append(f, name, err)) return CEL_ERR_IO;
    f << "[nx] " << nx << "\n" << "[ny] " << ny << "\n" << "\n\n" << "====================================" << "\n";
    const int NX = nx + 4;
    for (int j = 2; j < ny + 2; ++j) {
        for (int i = 2; i < nx + 2; ++i) f << b3[(size_t(j) * NX + i) * 3 + 2] << "\t";
        f << "\n";
    }
    if (!f) { err = "write failed: " + name; return CEL_ERR_IO; }
    return CEL_OK;
}

int write_hotstart(const float* rgba, int nx, int ny, const char* path, std::string& err) {
    // truncates: a hot-start file describes one state
    std::ofstream f(path, std::ios::out | std::ios::trunc);
    if (!f) { err = std::string("cannot open ") + path + " for writing"; return CEL_ERR_IO; }
    f.precision(std::numeric_limits<float>::max_digits10);
    const int NX = nx + 4;
    for (int j = 0; j < ny + 4; ++j)
        for (int i = 0; i < NX; ++i) {
            const float* t = rgba + (size_t(j) * NX + i) * 4;
            f << i << " " << j << " " << t[0] << " " << t[1] << " " << t[2] << " " << t[3] << "\n";
        }
    if (!f) { err = std::string("write failed: ") + path; return CEL_ERR_IO; }
    return CEL_OK;
}

}  // namespace cel
