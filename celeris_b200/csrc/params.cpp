// Settings boundary: `.cml` simulation parameters, `.cbf` bathymetry, irregular-wave and
// uniform-time-series files.
//
// Mirrors readInputCML (reference main.cpp:500-913) field by field, but with a small lenient
// XML reader of this project's own: it accepts unquoted attribute values (`a = 5e-12`),
// comments, processing instructions and repeated elements, which is what the reference's
// TinyXML 2.6.2 accepts for the shipped examples.
#include "celeris_internal.hpp"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace cel {

namespace {

struct XNode {
    std::string name;
    std::map<std::string, std::string> attrs;
    std::string text;
    std::vector<XNode> kids;
    const XNode* child(const char* n) const {
        for (const XNode& k : kids)
            if (k.name == n) return &k;
        return nullptr;
    }
    bool attr(const char* n, std::string& out) const {
        auto it = attrs.find(n);
        if (it == attrs.end()) return false;
        out = it->second;
        return true;
    }
};

class XParser {
public:
    explicit XParser(const std::string& s) : s_(s) {}
    bool parse(XNode& root, std::string& err) {
        skip_misc();
        if (!parse_element(root)) { err = err_.empty() ? "malformed XML" : err_; return false; }
        return true;
    }

private:
    const std::string& s_;
    size_t i_ = 0;
    std::string err_;
    bool eof() const { return i_ >= s_.size(); }
    void ws() { while (!eof() && std::isspace(static_cast<unsigned char>(s_[i_]))) ++i_; }
    bool starts(const char* t) const { return s_.compare(i_, std::strlen(t), t) == 0; }
    void skip_misc() {
        for (;;) {
            ws();
            if (starts("<?")) { size_t e = s_.find("?>", i_); i_ = e == std::string::npos ? s_.size() : e + 2; }
            else if (starts("<!--")) { size_t e = s_.find("-->", i_); i_ = e == std::string::npos ? s_.size() : e + 3; }
            else if (starts("<!")) { size_t e = s_.find('>', i_); i_ = e == std::string::npos ? s_.size() : e + 1; }
            else break;
        }
    }
    std::string name() {
        size_t b = i_;
        while (!eof() && (std::isalnum(static_cast<unsigned char>(s_[i_])) || s_[i_] == '_' || s_[i_] == '-' ||
                          s_[i_] == ':' || s_[i_] == '.'))
            ++i_;
        return s_.substr(b, i_ - b);
    }
    bool parse_element(XNode& n) {
        if (eof() || s_[i_] != '<') { err_ = "expected '<'"; return false; }
        ++i_;
        n.name = name();
        if (n.name.empty()) { err_ = "empty element name"; return false; }
        for (;;) {
            ws();
            if (eof()) { err_ = "unterminated tag <" + n.name; return false; }
            if (starts("/>")) { i_ += 2; return true; }
            if (s_[i_] == '>') { ++i_; break; }
            std::string an = name();
            if (an.empty()) { err_ = "bad attribute in <" + n.name; return false; }
            ws();
            if (eof() || s_[i_] != '=') { err_ = "attribute without '=' in <" + n.name; return false; }
            ++i_;
            ws();
            std::string v;
            if (!eof() && (s_[i_] == '"' || s_[i_] == '\'')) {
                const char q = s_[i_++];
                size_t e = s_.find(q, i_);
                if (e == std::string::npos) { err_ = "unterminated attribute"; return false; }
                v = s_.substr(i_, e - i_);
                i_ = e + 1;
            } else {  // unquoted value: up to whitespace, '>' or "/>"
                size_t b = i_;
                while (!eof() && !std::isspace(static_cast<unsigned char>(s_[i_])) && s_[i_] != '>' &&
                       !starts("/>"))
                    ++i_;
                v = s_.substr(b, i_ - b);
            }
            n.attrs[an] = v;
        }
        // content
        for (;;) {
            if (eof()) { err_ = "unterminated element <" + n.name; return false; }
            if (starts("<!--")) { size_t e = s_.find("-->", i_); i_ = e == std::string::npos ? s_.size() : e + 3; continue; }
            if (starts("</")) {
                i_ += 2;
                std::string en = name();
                ws();
                if (eof() || s_[i_] != '>' || en != n.name) { err_ = "mismatched </" + en + "> for <" + n.name + ">"; return false; }
                ++i_;
                return true;
            }
            if (s_[i_] == '<') {
                XNode k;
                if (!parse_element(k)) return false;
                n.kids.push_back(std::move(k));
                continue;
            }
            size_t e = s_.find('<', i_);
            if (e == std::string::npos) e = s_.size();
            n.text += s_.substr(i_, e - i_);
            i_ = e;
        }
    }
};

std::string trim(const std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace(static_cast<unsigned char>(s[b]))) ++b;
    while (e > b && std::isspace(static_cast<unsigned char>(s[e - 1]))) --e;
    return s.substr(b, e - b);
}

bool to_d(const XNode& n, const char* a, double& out) {
    std::string v;
    if (!n.attr(a, v)) return false;
    char* end = nullptr;
    double d = std::strtod(v.c_str(), &end);
    if (end == v.c_str()) return false;
    out = d;
    return true;
}

bool to_i(const XNode& n, const char* a, int& out) {
    double d;
    if (!to_d(n, a, d)) return false;
    out = int(d);
    return true;
}

bool to_b(const XNode& n, const char* a, bool& out) {
    std::string v;
    if (!n.attr(a, v)) return false;
    if (v == "true" || v == "1" || v == "True" || v == "TRUE") { out = true; return true; }
    if (v == "false" || v == "0" || v == "False" || v == "FALSE") { out = false; return true; }
    return false;
}

std::string dir_of(const std::string& p) {
    size_t k = p.find_last_of("/\\");
    return k == std::string::npos ? std::string(".") : p.substr(0, k);
}

std::string resolve(const std::string& base, const std::string& f) {
    std::string t = trim(f);
    if (t.empty()) return t;
    if (t[0] == '/') return t;
    return dir_of(base) + "/" + t;
}

void copy_str(char* dst, size_t cap, const std::string& s) {
    std::snprintf(dst, cap, "%s", s.c_str());
}

int bc_type(const std::string& t) {
    if (t == "Solid") return CEL_BC_SOLID;
    if (t == "Sponge") return CEL_BC_SPONGE;
    if (t == "SineWave") return CEL_BC_SINEWAVE;
    if (t == "IrregularWaves") return CEL_BC_IRREGULAR;
    if (t == "UniformTimeSeries") return CEL_BC_UTS;
    return -1;
}

// decodeLine / decodeLine2 (terrain_heightfield.cpp:85-127, engine.cpp:3476-3510):
// "[tag] value" header lines.
bool decode_tag(const std::string& line, std::string& tag, std::string& value) {
    size_t i = 0;
    while (i < line.size() && (line[i] == ' ' || line[i] == '\t')) ++i;
    if (i >= line.size() || line[i] != '[') return false;
    size_t e = line.find(']', i);
    if (e == std::string::npos) return false;
    tag = line.substr(i, e - i + 1);
    size_t v = e + 1;
    while (v < line.size() && line[v] == ' ') ++v;
    value = line.substr(v);
    return true;
}

}  // namespace

void params_default(cel_params* p) {
    std::memset(p, 0, sizeof(*p));
    p->nx = 100; p->ny = 100;
    p->width = 100; p->length = 100;
    p->still_water_elevation = 0;
    p->boussinesq = 1;
    p->epsilon = 5e-8;
    p->theta = 2;
    p->correction_steps = 0;
    p->timestep = 0.0001;
    p->adaptive = 0;
    p->ema_alpha = 0.5;
    p->min_timestep_ratio = 0.05;
    p->manning = 0;
    p->friction = 0;
    p->gravity = 9.81;
    p->dissipation_threshold = 0.25;
    p->whitewater_decay = 0.25;
    for (cel_boundary* b : {&p->west, &p->east, &p->south, &p->north}) {
        b->type = CEL_BC_SOLID;
        b->width = 2;
    }
    // logging defaults (settings.hpp:389, 423-433)
    p->log.log_step = 100;
    copy_str(p->log.path, sizeof(p->log.path), "NA");
    copy_str(p->log.time_axis_name, sizeof(p->log.time_axis_name), "time_axis");
    copy_str(p->log.gauges_name, sizeof(p->log.gauges_name), "gauges");
}

int read_irregular(const std::string& path, cel_boundary* b, std::string& err) {
    // getNumberOfWavesFromFileStream + component rows (engine.cpp:3512-3551)
    std::ifstream in(path.c_str());
    if (!in) { err = "cannot open irregular-wave file " + path; return CEL_ERR_IO; }
    std::string line;
    int n = -1;
    while (std::getline(in, line)) {
        if (!line.empty() && line[0] == '=') break;
        if (line.empty() || line[0] == '#') continue;
        std::string tag, value;
        if (decode_tag(line, tag, value) && tag == "[NumberOfWaves]" && !trim(value).empty())
            n = std::min(CEL_MAX_WAVES, std::atoi(value.c_str()));
    }
    if (n < 0) { err = "irregular-wave file without [NumberOfWaves]: " + path; return CEL_ERR_IO; }
    int count = 0;
    for (; count < n; ++count) {
        double a, t, th, ph;
        if (!(in >> a >> t >> th >> ph)) break;
        b->waves[count][0] = a; b->waves[count][1] = t; b->waves[count][2] = th; b->waves[count][3] = ph;
    }
    if (count < n) { err = "irregular-wave file has fewer rows than [NumberOfWaves]: " + path; return CEL_ERR_IO; }
    b->n_waves = n;
    return CEL_OK;
}

int read_uts(const std::string& path, cel_boundary* b, std::string& err) {
    // skipCommentsInFileStream + rows of (t, eta, hu, hv) (engine.cpp:3863-3874)
    std::ifstream in(path.c_str());
    if (!in) { err = "cannot open time-series file " + path; return CEL_ERR_IO; }
    std::string line;
    while (std::getline(in, line))
        if (!line.empty() && line[0] == '=') break;
    std::vector<double> rows;
    double t, e, u, v;
    while (in >> t >> e >> u >> v) { rows.push_back(t); rows.push_back(e); rows.push_back(u); rows.push_back(v); }
    if (rows.size() < 8) { err = "time-series file needs at least two rows: " + path; return CEL_ERR_IO; }
    if (b->uts) std::free(b->uts);
    b->uts = static_cast<double*>(std::malloc(rows.size() * sizeof(double)));
    std::memcpy(b->uts, rows.data(), rows.size() * sizeof(double));
    b->n_uts = int(rows.size() / 4);
    return CEL_OK;
}

// <logData doLog logStep> with <logPath>, <timeAxis filename>, <range filename> (bottomLeft /
// topRight x, y) and <gauges filename>x,y,x,y,...</gauges> children (main.cpp:825-887).
static int read_log_data(const XNode& e, const std::string& cml, cel_log& lg, std::string& err) {
    bool on = false;
    if (to_b(e, "doLog", on)) lg.do_log = on ? 1 : 0;
    to_i(e, "logStep", lg.log_step);
    for (const XNode& k : e.kids) {
        std::string fname;
        if (k.name == "logPath") {
            // relative paths are taken from the .cml folder; an empty one means that folder
            const std::string t = trim(k.text);
            copy_str(lg.path, sizeof(lg.path), t.empty() ? dir_of(cml) : resolve(cml, t));
        } else if (k.name == "timeAxis") {
            k.attr("filename", fname);
            copy_str(lg.time_axis_name, sizeof(lg.time_axis_name), fname);
        } else if (k.name == "range") {
            if (lg.n_ranges >= CEL_MAX_LOG_RANGES) { err = "more than 100 log ranges"; return CEL_ERR_IO; }
            const XNode* bl = k.child("bottomLeft");
            const XNode* tr = k.child("topRight");
            if (!bl || !tr) { err = "log range without bottomLeft/topRight"; return CEL_ERR_IO; }
            cel_log_range& R = lg.ranges[lg.n_ranges++];
            k.attr("filename", fname);
            copy_str(R.name, sizeof(R.name), fname);
            to_i(*bl, "x", R.x0);
            to_i(*bl, "y", R.y0);
            to_i(*tr, "x", R.x1);
            to_i(*tr, "y", R.y1);
        } else if (k.name == "gauges") {
            k.attr("filename", fname);
            copy_str(lg.gauges_name, sizeof(lg.gauges_name), fname);
            // Pairs are read as `>> x >> sep >> y >> sep` until the stream fails, and the pair of
            // the failing round is kept too (main.cpp:866-876): "1,2,3,4" gives two gauges and a
            // trailing comma repeats the last one.  A text without any number gives none.
            std::istringstream in(k.text);
            int x = 0, y = 0, rounds = 0;
            char sep = 0;
            while (in) {
                in >> x;
                const bool got_x = bool(in);
                in >> sep >> y >> sep;
                if (!got_x && rounds == 0) break;
                if (lg.n_gauges >= CEL_MAX_GAUGES) { err = "more than 1000 gauges"; return CEL_ERR_IO; }
                lg.gauges[lg.n_gauges][0] = x;
                lg.gauges[lg.n_gauges][1] = y;
                lg.n_gauges++;
                ++rounds;
            }
        }
    }
    return CEL_OK;
}

int params_from_cml(const char* path, cel_params* out, std::string& err) {
    params_default(out);
    std::ifstream in(path, std::ios::binary);
    if (!in) { err = std::string("cannot open ") + path; return CEL_ERR_IO; }
    std::stringstream ss;
    ss << in.rdbuf();
    const std::string text = ss.str();
    XNode root;
    XParser xp(text);
    if (!xp.parse(root, err)) { err = std::string(path) + ": " + err; return CEL_ERR_IO; }
    const std::string cml = path;
    for (const XNode& e : root.kids) {
        const std::string& n = e.name;
        if (n == "fieldDimensions") {
            to_d(e, "length", out->length);
            to_d(e, "width", out->width);
            to_d(e, "stillWaterElevation", out->still_water_elevation);
        } else if (n == "name") {
            copy_str(out->project_name, sizeof(out->project_name), trim(e.text));
        } else if (n == "model") {
            std::string mt;
            e.attr("type", mt);
            out->boussinesq = (mt == "NLSW") ? 0 : 1;
            if (const XNode* pr = e.child("parameters")) {
                to_d(*pr, "epsilon", out->epsilon);
                to_d(*pr, "Theta", out->theta);
                to_i(*pr, "correctionStepsNum", out->correction_steps);
                to_d(*pr, "timestep", out->timestep);
                bool ad = false;
                to_b(*pr, "adaptive", ad);
                out->adaptive = ad ? 1 : 0;
                to_d(*pr, "exponentialMovingAverageAlpha", out->ema_alpha);
            }
            if (const XNode* fr = e.child("friction")) {
                std::string ft;
                fr->attr("type", ft);
                out->manning = (ft == "Manning") ? 1 : 0;
                to_d(*fr, "coef", out->friction);
            }
        } else if (n == "gridSize") {
            to_i(e, "nx", out->nx);
            to_i(e, "ny", out->ny);
        } else if (n == "bathymetryFilePath") {
            copy_str(out->bathymetry_path, sizeof(out->bathymetry_path), resolve(cml, e.text));
        } else if (n == "hotStartFilePath") {
            std::string t = trim(e.text);
            if (!t.empty() && t != "N/A" && t != "NA")
                copy_str(out->hotstart_path, sizeof(out->hotstart_path), resolve(cml, t));
        } else if (n == "solitaryWave") {
            if (out->n_solitons < CEL_MAX_SOLITONS) {
                cel_soliton& s = out->solitons[out->n_solitons];
                double deg = 0;
                to_d(e, "H", s.H);
                to_d(e, "theta", deg);
                to_d(e, "xc", s.xc);
                to_d(e, "yc", s.yc);
                s.length = 1e30;  // no attribute: infinitely long crest (main.cpp:647-649)
                to_d(e, "length", s.length);
                s.theta = M_PI / 180.0 * deg;
                out->n_solitons++;
            }
        } else if (n == "westBoundary" || n == "eastBoundary" || n == "northBoundary" || n == "southBoundary") {
            cel_boundary* b = n[0] == 'w' ? &out->west : n[0] == 'e' ? &out->east : n[0] == 'n' ? &out->north : &out->south;
            std::string t;
            e.attr("type", t);
            const int ty = bc_type(t);
            if (ty < 0) { err = "unknown boundary type '" + t + "' in " + n; return CEL_ERR_IO; }
            b->type = ty;
            to_d(e, "seaLevel", b->sea_level);
            double w = b->width;
            if (to_d(e, "widthNum", w)) b->width = int(w);
            if (ty == CEL_BC_SINEWAVE) {
                if (const XNode* sw = e.child("sineWave")) {
                    double deg = 0;
                    to_d(*sw, "amplitude", b->amplitude);
                    to_d(*sw, "period", b->period);
                    to_d(*sw, "theta", deg);
                    b->theta = M_PI / 180.0 * deg;
                }
            } else if (ty == CEL_BC_IRREGULAR || ty == CEL_BC_UTS) {
                const XNode* fp = e.child("filePath");
                if (!fp) { err = n + " needs a <filePath>"; return CEL_ERR_IO; }
                const std::string f = resolve(cml, fp->text);
                const int st = ty == CEL_BC_IRREGULAR ? read_irregular(f, b, err) : read_uts(f, b, err);
                if (st != CEL_OK) return st;
            }
        } else if (n == "logData") {
            if (int st = read_log_data(e, cml, out->log, err)) return st;
        } else if (n == "graphics") {
            if (const XNode* ss2 = e.child("surfaceShading"))
                if (const XNode* di = ss2->child("dissipationIntensity")) {
                    // readGraphicsInput_helper (main.cpp:965-977): element defaults .25 / .1
                    out->dissipation_threshold = 0.25;
                    out->whitewater_decay = 0.1;
                    to_d(*di, "threshold", out->dissipation_threshold);
                    to_d(*di, "decay", out->whitewater_decay);
                }
        }
    }
    if (out->nx < 2 || out->ny < 2) { err = "gridSize nx and ny must be >= 2"; return CEL_ERR_ARG; }
    return CEL_OK;
}

void params_release(cel_params* p) {
    for (cel_boundary* b : {&p->west, &p->east, &p->south, &p->north}) {
        if (b->uts) std::free(b->uts);
        b->uts = nullptr;
        b->n_uts = 0;
    }
}

int read_cbf(const std::string& path, std::vector<float>* z, int& bnx, int& bny, std::string& err) {
    // readBathymetry (terrain_heightfield.cpp:136-209)
    std::ifstream in(path.c_str());
    if (!in) { err = "cannot open bathymetry file " + path; return CEL_ERR_IO; }
    std::string line;
    bnx = bny = 0;
    while (std::getline(in, line)) {
        if (!line.empty() && line[0] == '=') break;
        std::string tag, value;
        if (decode_tag(line, tag, value) && !trim(value).empty()) {
            if (tag == "[nx]") bnx = std::atoi(value.c_str());
            else if (tag == "[ny]") bny = std::atoi(value.c_str());
        }
    }
    if (bnx < 2 || bny < 2) { err = "bathymetry file without a valid [nx]/[ny] header: " + path; return CEL_ERR_IO; }
    if (!z) return CEL_OK;
    z->assign(size_t(bnx) * bny, 0.f);
    size_t k = 0;
    for (; k < z->size(); ++k) {
        float v;
        if (!(in >> v)) break;
        (*z)[k] = v;
    }
    if (k < z->size()) { err = "bathymetry file has fewer values than nx*ny: " + path; return CEL_ERR_IO; }
    return CEL_OK;
}

int read_hotstart(const std::string& path, int nx, int ny, std::vector<float>& whuhv, std::string& err) {
    // Hot start: rows of "i j w hu hv alpha" over (nx+4)(ny+4) texels (engine.cpp:2943-2966)
    std::ifstream in(path.c_str());
    if (!in) { err = "cannot open hot-start file " + path; return CEL_ERR_IO; }
    const size_t n = size_t(nx + 4) * (ny + 4);
    whuhv.assign(n * 3, 0.f);
    for (size_t k = 0; k < n; ++k) {
        int i, j;
        float w, hu, hv, a;
        if (!(in >> i >> j >> w >> hu >> hv >> a)) { err = "hot-start file is short: " + path; return CEL_ERR_IO; }
        whuhv[3 * k] = w; whuhv[3 * k + 1] = hu; whuhv[3 * k + 2] = hv;
    }
    return CEL_OK;
}

}  // namespace cel
