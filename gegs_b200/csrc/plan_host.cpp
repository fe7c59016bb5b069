// C++ host side of the drop-in path (include/gegs_plan.h): the reference's
// input files read into gegs_physics / gegs_scene, and the dose file written.
//
// The text parsers follow the reference's C++ stream reads (`infile >> value
// >> ch` reads a number and the one separator character after it;
// `ignore(n, '\n')` drops the rest of a line), and every number is computed
// with the arithmetic of the package's Python reader (gegs_b200/plan.py,
// io_formats.py, geometry.py), so both produce the same scene bit for bit.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/gegs_plan.h"

namespace fs = std::filesystem;

namespace {

struct PlanError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// ---- text ------------------------------------------------------------------
bool py_space(unsigned char c)
{
    return c == ' ' || (c >= 9 && c <= 13) || (c >= 28 && c <= 31) || c == 0x85 || c == 0xA0;
}

std::string strip(const std::string &s)
{
    size_t a = 0, b = s.size();
    while (a < b && py_space((unsigned char)s[a])) a++;
    while (b > a && py_space((unsigned char)s[b - 1])) b--;
    return s.substr(a, b - a);
}

std::string lower(std::string s)
{
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

std::vector<std::string> split_ws(const std::string &s)
{
    std::vector<std::string> out;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && py_space((unsigned char)s[i])) i++;
        size_t j = i;
        while (j < s.size() && !py_space((unsigned char)s[j])) j++;
        if (j > i) out.push_back(s.substr(i, j - i));
        i = j;
    }
    return out;
}

std::string read_text(const fs::path &p)
{
    std::ifstream f(p, std::ios::binary);
    if (!f) throw PlanError(p.string() + ": cannot open");
    std::stringstream ss;
    ss << f.rdbuf();
    std::string s = ss.str(), out;
    out.reserve(s.size());
    for (size_t i = 0; i < s.size(); i++) {          // "\r\n" -> "\n"
        if (s[i] == '\r' && i + 1 < s.size() && s[i + 1] == '\n') continue;
        out += s[i];
    }
    return out;
}

// A number as the reference reads it: into a float (`stream >> float`,
// scanf's %f), rounded once from the decimal.
float to_float(const std::string &t, const std::string &what)
{
    const char *b = t.c_str();
    char *e = nullptr;
    errno = 0;
    float v = std::strtof(b, &e);
    if (e == b || *e != '\0') throw PlanError("could not parse " + what + " '" + t + "'");
    return v;
}

// The subset of std::istream the reference's parsers use (see the header note).
struct Stream {
    std::string s;
    size_t i = 0;
    explicit Stream(std::string t) : s(std::move(t)) {}
    bool eof() const { return i >= s.size(); }
    std::string getline()
    {
        size_t j = s.find('\n', i);
        std::string line;
        if (j == std::string::npos) { line = s.substr(i); i = s.size(); }
        else { line = s.substr(i, j - i); i = j + 1; }
        return line;
    }
    void ignore(size_t n = 100, char delim = '\n')
    {
        size_t end = std::min(s.size(), i + n);
        size_t j = s.find(delim, i);
        i = (j == std::string::npos || j >= end) ? end : j + 1;
    }
    void skip_ws() { while (i < s.size() && py_space((unsigned char)s[i])) i++; }
    // [+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?
    std::string token()
    {
        skip_ws();
        size_t j = i;
        auto digit = [&](size_t k) { return k < s.size() && s[k] >= '0' && s[k] <= '9'; };
        if (j < s.size() && (s[j] == '+' || s[j] == '-')) j++;
        size_t m = j;
        if (digit(m)) {
            while (digit(m)) m++;
            if (m < s.size() && s[m] == '.') { m++; while (digit(m)) m++; }
        } else if (m < s.size() && s[m] == '.' && digit(m + 1)) {
            m++;
            while (digit(m)) m++;
        } else {
            throw PlanError("expected a number at offset " + std::to_string(i) + ": '" + s.substr(i, 30) + "'");
        }
        if (m < s.size() && (s[m] == 'e' || s[m] == 'E')) {
            size_t q = m + 1;
            if (q < s.size() && (s[q] == '+' || s[q] == '-')) q++;
            if (digit(q)) { while (digit(q)) q++; m = q; }
        }
        std::string t = s.substr(i, m - i);
        i = m;
        return t;
    }
    float num() { return to_float(token(), "number"); }
    long long num_int()
    {
        std::string t = token();
        if (t.find_first_of(".eE") != std::string::npos) return (long long)std::strtod(t.c_str(), nullptr);
        return std::stoll(t);
    }
    void chr() { skip_ws(); i++; }
    float num_sep() { float v = num(); chr(); return v; }
    long long num_sep_int() { long long v = num_int(); chr(); return v; }
    bool find_line_starting(const std::string &title)
    {
        while (!eof())
            if (getline().rfind(title, 0) == 0) return true;
        return false;
    }
};

// ---- INI (the profile-API rules: case-insensitive sections and keys) ------
using Ini = std::map<std::string, std::map<std::string, std::string>>;

Ini read_ini(const fs::path &p)
{
    Ini ini;
    std::string text = read_text(p);
    std::map<std::string, std::string> *cur = nullptr;
    std::stringstream ss(text);
    std::string raw;
    while (std::getline(ss, raw)) {
        std::string line = strip(raw);
        if (line.empty() || line[0] == ';' || line[0] == '#') continue;
        if (line.size() >= 3 && line.front() == '[' && line.back() == ']') {
            cur = &ini[lower(strip(line.substr(1, line.size() - 2)))];
            continue;
        }
        size_t eq = line.find('=');
        if (eq == std::string::npos || !cur) continue;
        std::string k = lower(strip(line.substr(0, eq))), v = strip(line.substr(eq + 1));
        if (v.size() >= 2 && v.front() == v.back() && (v.front() == '"' || v.front() == '\'')) v = v.substr(1, v.size() - 2);
        (*cur)[k] = v;
    }
    return ini;
}

const std::string *ini_get(const Ini &ini, const std::string &sec, const std::string &key)
{
    auto s = ini.find(lower(sec));
    if (s == ini.end()) return nullptr;
    auto k = s->second.find(lower(key));
    return k == s->second.end() ? nullptr : &k->second;
}

std::string ini_req(const Ini &ini, const std::string &sec, const std::string &key)
{
    const std::string *v = ini_get(ini, sec, key);
    if (!v) throw PlanError("property \"" + key + "\" is not specified in the section \"" + sec + "\"");
    return *v;
}

std::string ini_opt(const Ini &ini, const std::string &sec, const std::string &key, const std::string &dflt)
{
    const std::string *v = ini_get(ini, sec, key);
    return v ? *v : dflt;
}

bool ini_on(const Ini &ini, const std::string &sec, const std::string &key)
{
    const std::string *v = ini_get(ini, sec, key);
    if (!v) return false;
    std::string t = lower(strip(*v));
    return t == "on" || t == "yes" || t == "true" || t == "1";
}

std::vector<double> floats(const std::string &v, size_t n, const std::string &what)
{
    std::vector<double> out;
    for (const auto &t : split_ws(v)) out.push_back(to_float(t, what));
    if (out.size() < n) throw PlanError(what + " needs " + std::to_string(n) + " numbers, got '" + v + "'");
    out.resize(n);
    return out;
}

fs::path data_path(const fs::path &base, std::string rel)
{
    std::replace(rel.begin(), rel.end(), '\\', '/');
    fs::path p(rel);
    return p.is_absolute() ? p : (base / p).lexically_normal();
}

// ---- egsphant (init.cu:1164-1275) -------------------------------------------
struct Phantom {
    std::vector<std::string> media;
    int nx = 0, ny = 0, nz = 0;
    std::vector<float> xb, yb, zb, density;
    std::vector<uint16_t> med;
};

Phantom read_egsphant(const fs::path &path)
{
    const std::string text = read_text(path), name = path.string();
    std::vector<std::string> lines;
    {
        size_t a = 0;
        for (;;) {
            size_t b = text.find('\n', a);
            if (b == std::string::npos) { lines.push_back(text.substr(a)); break; }
            lines.push_back(text.substr(a, b - a));
            a = b + 1;
        }
    }
    Phantom ph;
    size_t k = 0;
    auto tok0 = split_ws(lines.at(k++));
    if (tok0.empty()) throw PlanError(name + ": no medium count");
    const int nmed = std::stoi(tok0[0]);
    for (int i = 0; i < nmed; i++) {
        std::string m = strip(lines.at(k++));
        if (m.empty()) throw PlanError(name + ": medium name " + std::to_string(i) + " is empty");
        ph.media.push_back(m);
    }
    k++;                                                   // ESTEPE line
    {
        auto t = k < lines.size() ? split_ws(lines[k]) : std::vector<std::string>{};
        if (t.size() < 3) throw PlanError(name + ": line " + std::to_string(k + 1) + " must hold the three voxel counts nx ny nz");
        try { ph.nx = std::stoi(t[0]); ph.ny = std::stoi(t[1]); ph.nz = std::stoi(t[2]); }
        catch (...) { throw PlanError(name + ": line " + std::to_string(k + 1) + " must hold the three voxel counts nx ny nz"); }
        if (std::min({ph.nx, ph.ny, ph.nz}) < 1) throw PlanError(name + ": voxel counts must be positive");
        k++;
    }
    std::string rest_text;
    for (size_t j = k; j < lines.size(); j++) { rest_text += lines[j]; if (j + 1 < lines.size()) rest_text += '\n'; }
    Stream r(rest_text);
    for (int i = 0; i <= ph.nx; i++) ph.xb.push_back((float)r.num());
    for (int i = 0; i <= ph.ny; i++) ph.yb.push_back((float)r.num());
    for (int i = 0; i <= ph.nz; i++) ph.zb.push_back((float)r.num());
    r.ignore((size_t)1 << 30, '\n');
    const size_t nvox = (size_t)ph.nx * ph.ny * ph.nz;
    ph.med.resize(nvox);
    for (int z = 0; z < ph.nz; z++)
        for (int y = 0; y < ph.ny; y++) {
            std::string row = strip(r.getline());
            while (row.empty() && !r.eof()) row = strip(r.getline());
            if ((int)row.size() < ph.nx) throw PlanError(name + ": medium row (y=" + std::to_string(y) + ", z=" + std::to_string(z) + ") is short");
            const size_t base = (size_t)z * ph.nx * ph.ny + (size_t)y * ph.nx;
            for (int x = 0; x < ph.nx; x++) {
                int v = (int)(unsigned char)row[x] - '0';
                if (v < 1 || v > nmed) throw PlanError(name + ": medium number outside 1.." + std::to_string(nmed));
                ph.med[base + x] = (uint16_t)(v - 1);
            }
        }
    auto d = split_ws(r.s.substr(r.i));
    if (d.size() < nvox) throw PlanError(name + ": " + std::to_string(d.size()) + " densities for " + std::to_string(nvox) + " voxels");
    ph.density.resize(nvox);
    for (size_t v = 0; v < nvox; v++) ph.density[v] = to_float(d[v], "density");
    return ph;
}

// ---- egsphsp1 (read_egsphsp.cpp:44-232) --------------------------------------
uint32_t bswap32(uint32_t x) { return (x >> 24) | ((x >> 8) & 0xFF00u) | ((x << 8) & 0xFF0000u) | (x << 24); }

void read_egsphsp1(const fs::path &path, std::vector<gegs_phsp_record> &out)
{
    const std::string name = path.string();
    std::ifstream f(path, std::ios::binary);
    if (!f) throw PlanError(name + ": cannot open");
    f.seekg(0, std::ios::end);
    const uint64_t size = (uint64_t)f.tellg();
    f.seekg(0);
    unsigned char head[32] = {};
    f.read((char *)head, 32);
    const std::string mode((const char *)head, 5);
    if (mode != "MODE0" && mode != "MODE2") throw PlanError(name + ": unknown phase-space mode '" + mode + "'");
    int32_t n_le;
    std::memcpy(&n_le, head + 5, 4);
    bool big = false;
    int64_t n = n_le;
    const int64_t held28 = (int64_t)(size / 28);
    if (n < 0 || n > held28) {
        const int32_t n_be = (int32_t)bswap32((uint32_t)n_le);
        if (n_be >= 0 && n_be <= held28) { big = true; n = n_be; }
        else if (n < 0) throw PlanError(name + ": negative particle count in the header");
    }
    const uint64_t reclen = mode == "MODE0" ? 28 : 32;
    const int64_t held = (int64_t)(size / reclen) - 1;
    if (n > held) throw PlanError(name + ": the header announces " + std::to_string(n) + " particles but the file holds " + std::to_string(std::max<int64_t>(held, 0)) + " records (truncated)");
    std::vector<unsigned char> buf((size_t)(reclen * (uint64_t)n));
    f.seekg((std::streamoff)reclen);
    f.read((char *)buf.data(), (std::streamsize)buf.size());
    const size_t first = out.size();
    out.resize(first + (size_t)n);
    for (int64_t k = 0; k < n; k++) {
        uint32_t w[7];
        std::memcpy(w, buf.data() + (size_t)k * reclen, 28);
        if (big) for (auto &x : w) x = bswap32(x);
        gegs_phsp_record &r = out[first + (size_t)k];
        std::memcpy(&r, w, 28);
    }
}

// ---- egsinp component modules (init.cu:345-689) -----------------------------
// Every number is read into a float, as the reference reads it (`infile >> float`).
struct Leaf {
    float wl, wt, wg, wtip, wts, wbs, ztip, zl, zt, zg, zth, zbh, holepos, zts, zbs;
};

struct DynVMLC {
    float rmax, zmin, zthick, x_start, air_gap, rad_end;
    Leaf full, target, iso;
    long long n_full, n_half;
    std::vector<std::tuple<float, float, long long>> open;
    std::string media;
};

struct SecJaws {
    float rmax, zminy, zmaxy, zminx, zmaxx;
    std::string media;
};

const char *kDynvmlcTitle = "*********** start of CM DYNVMLC";
const char *kSecjawsTitle = "*********** start of CM JAWS with identifier SECJAWS";

Leaf read_leaf(Stream &r, bool target_order)
{
    Leaf L{};
    L.wl = r.num_sep(); L.wt = r.num_sep(); L.wg = r.num_sep(); L.wtip = r.num_sep(); L.wts = r.num_sep();
    L.wbs = r.num_sep();
    if (!target_order) {
        L.ztip = r.num_sep(); L.zl = r.num_sep(); L.zt = r.num_sep(); L.zg = r.num_sep(); L.zth = r.num_sep();
        L.zbh = r.num_sep(); L.holepos = r.num_sep(); L.zts = r.num_sep(); L.zbs = r.num_sep();
    } else {
        L.zts = r.num_sep(); L.zbs = r.num_sep(); L.zth = r.num_sep(); L.zbh = r.num_sep(); L.holepos = r.num_sep();
        L.zt = r.num_sep(); L.zg = r.num_sep(); L.zl = r.num_sep(); L.ztip = r.num_sep();
    }
    return L;
}

DynVMLC read_dynvmlc(const fs::path &path)
{
    Stream r(read_text(path));
    if (!r.find_line_starting(kDynvmlcTitle)) throw PlanError(path.string() + ": no CM DYNVMLC block");
    DynVMLC m{};
    m.rmax = r.num_sep(); r.ignore();
    r.ignore(); r.ignore();
    m.zmin = r.num_sep(); r.ignore();
    m.zthick = r.num_sep(); r.ignore();
    m.full = read_leaf(r, false);
    m.target = read_leaf(r, true);
    m.iso = read_leaf(r, false);
    m.n_full = r.num_sep_int(); r.ignore();
    m.n_half = r.num_sep_int(); r.ignore();
    r.ignore();
    m.x_start = r.num_sep(); r.ignore();
    m.air_gap = r.num_sep(); r.ignore();
    r.ignore();
    m.rad_end = r.num_sep(); r.ignore();
    r.ignore();
    long long total = 0;
    while (total < 60) {
        float neg = r.num_sep(), pos = r.num_sep();
        long long num = r.num_int();
        m.open.emplace_back(neg, pos, num);
        total += num;
        if (num <= 0) throw PlanError(path.string() + ": leaf-opening row with NUM <= 0");
    }
    r.ignore();
    for (int k = 0; k < 3; k++) r.ignore();
    m.media = strip(r.getline());
    if (m.media.empty()) m.media = "W700ICRU";
    return m;
}

SecJaws read_secjaws(const fs::path &path)
{
    Stream r(read_text(path));
    if (!r.find_line_starting(kSecjawsTitle)) throw PlanError(path.string() + ": no CM JAWS SECJAWS block");
    SecJaws j{};
    j.rmax = r.num_sep(); r.ignore();
    for (int k = 0; k < 3; k++) r.ignore();
    j.zminy = r.num_sep(); j.zmaxy = r.num_sep(); r.ignore();
    r.ignore();
    j.zminx = r.num_sep(); j.zmaxx = r.num_sep(); r.ignore();
    r.ignore();
    r.ignore();
    j.media = strip(r.getline());
    return j;
}

// 14 (x, z) vertices of a leaf type, in float (read_egsinp.h:37-88)
void leaf_vertices(const Leaf &L, int kind, float zmin, float zthick, float v[14][2])
{
    const float wl = L.wl, wt = L.wt, wg = L.wg, wtip = L.wtip, wts = L.wts, wbs = L.wbs, zmax = zmin + zthick;
    if (kind == 0) {
        const float t[14][2] = {{0, L.ztip}, {wtip, L.ztip}, {wtip, L.zl}, {wt + wl - wg, L.zl}, {wt + wl - wg, L.zg},
                                {wt + wl, L.zg}, {wt + wl, zmax}, {wt + wts - wbs, zmax}, {wt + wts - wbs, L.zbs},
                                {wt + wts, L.zbs}, {wt + wts, L.zts}, {wt, L.zts}, {wt, L.zt}, {0, L.zt}};
        std::memcpy(v, t, sizeof t);
    } else if (kind == 1) {
        const float t[14][2] = {{0, zmin}, {wt + wl - wbs + wts, zmin}, {wt + wl - wbs + wts, L.zts},
                                {wt + wl - wbs, L.zts}, {wt + wl - wbs, L.zbs}, {wt + wl, L.zbs}, {wt + wl, L.zg},
                                {wt + wl - wg, L.zg}, {wt + wl - wg, L.ztip}, {wt + wl - wg - wtip, L.ztip},
                                {wt + wl - wg - wtip, L.zl}, {wt, L.zl}, {wt, L.zt}, {0, L.zt}};
        std::memcpy(v, t, sizeof t);
    } else {
        const float t[14][2] = {{0, L.zt}, {wt, L.zt}, {wt, L.ztip}, {wt + wtip, L.ztip}, {wt + wtip, L.zl},
                                {wt + wl - wg, L.zl}, {wt + wl - wg, L.zg}, {wt + wl, L.zg}, {wt + wl, zmax},
                                {wts - wbs, zmax}, {wts - wbs, L.zbs}, {wts, L.zbs}, {wts, L.zts}, {0, L.zts}};
        std::memcpy(v, t, sizeof t);
    }
}

// The reference's leaf-end outline of bank A (leaf_end, init.cu:266-280),
// bottom to top; the first and last depth are -/+ half the leaf thickness.
const float kLeafEndX[15] = {-0.86708f, -0.64016f, -0.44640f, -0.28667f, -0.16167f, -0.07199f, -0.01802f, 0.0f,
                             -0.01802f, -0.07199f, -0.16167f, -0.28667f, -0.44640f, -0.64016f, -0.86708f};
const float kLeafEndY[15] = {0.0f, -2.92273f, -2.45316f, -1.97406f, -1.48729f, -0.99475f, -0.49834f, 0.0f,
                             0.49834f, 0.99475f, 1.48729f, 1.97406f, 2.45316f, 2.92273f, 0.0f};

// crossXZ, boundaries and constants of the MLC in float (read_egsinp,
// init.cu:451-561), and the leaf-end outline (leaf_end, init.cu:256-343).
// Entries the reference leaves unset (the 16th vertex of most leaves) are 0.
void build_mlc(const DynVMLC &m, gegs_scene &S, float cross_yz[34][2])
{
    std::memset(S.crossXZ, 0, sizeof S.crossXZ);
    const float zmin = m.zmin, zthick = m.zthick, air_gap = m.air_gap;
    float vf[14][2], vt[14][2], vi[14][2];
    leaf_vertices(m.full, 0, zmin, zthick, vf);
    leaf_vertices(m.target, 1, zmin, zthick, vt);
    leaf_vertices(m.iso, 2, zmin, zthick, vi);
    float X = m.x_start;
    int i = 0;
    auto put = [&](int i, float X, const float v[14][2]) {
        for (int k = 0; k < 14; k++) {
            S.crossXZ[i * 16 + k][0] = (X + v[k][0]) / zmin * v[k][1];
            S.crossXZ[i * 16 + k][1] = v[k][1];
        }
    };
    for (long long k = 0; k < m.n_full; k++) { put(i, X, vf); X = X + m.full.wl + air_gap; i++; }
    const float x_mid_1 = X;
    for (long long k = 0; k < m.n_half / 2; k++) {
        put(i, X, vt); X = X + m.target.wl + air_gap; i++;
        put(i, X, vi); X = X + m.iso.wl + air_gap; i++;
    }
    const float x_mid_2 = X;
    for (long long k = 0; k < m.n_full; k++) { put(i, X, vf); X = X + m.full.wl + air_gap; i++; }
    const float x_end = X - air_gap + m.full.wg;
    int kk = 0;
    for (const auto &row : m.open)
        for (long long q = 0; q < std::get<2>(row); q++, kk++)
            if (kk < 60) { S.crossXZ[14 + kk * 16][0] = std::get<0>(row); S.crossXZ[14 + kk * 16][1] = std::get<1>(row); }
    S.crossXZ[15][0] = zmin; S.crossXZ[15][1] = zthick;
    S.crossXZ[31][0] = m.x_start; S.crossXZ[31][1] = x_end;
    S.crossXZ[47][0] = x_mid_1; S.crossXZ[47][1] = x_mid_2;
    S.crossXZ[63][1] = air_gap;
    S.crossXZ[79][0] = m.full.wl; S.crossXZ[79][1] = m.target.wl;
    S.crossXZ[95][0] = m.iso.wl; S.crossXZ[95][1] = m.full.wt;
    S.crossXZ[111][0] = m.rmax;
    const float ztop = zthick + zmin;
    const float bxz[4][2] = {{m.x_start / zmin * (zmin + zthick), ztop}, {m.x_start, zmin}, {x_end, zmin},
                             {x_end / zmin * (zmin + zthick), ztop}};
    const float byz[4][2] = {{-m.rmax, ztop}, {-m.rmax, zmin}, {m.rmax, zmin}, {m.rmax, ztop}};
    std::memcpy(S.boundaryXZ, bxz, sizeof bxz);
    std::memcpy(S.boundaryYZ, byz, sizeof byz);
    S.mlc_rmax = m.rmax; S.mlc_zmin = zmin; S.mlc_zthick = zthick;
    S.mlc_x_start = m.x_start; S.mlc_x_end = x_end; S.mlc_x_mid_1 = x_mid_1;
    S.mlc_x_mid_2 = x_mid_2; S.mlc_air_gap = air_gap; S.mlc_wl_full = m.full.wl;
    S.mlc_wl_target = m.target.wl; S.mlc_wl_isocenter = m.iso.wl; S.mlc_wt = m.full.wt;
    const float zc = zthick / 2;
    float n[30][2];
    for (int k = 0; k < 15; k++) {
        const float y = k == 0 ? -zc : (k == 14 ? zc : kLeafEndY[k]);
        n[k][0] = kLeafEndX[k]; n[k][1] = y;                       // bank A
        n[29 - k][0] = std::fabs(kLeafEndX[k]); n[29 - k][1] = y;  // bank B, its mirror
    }
    cross_yz[0][0] = -m.rmax; cross_yz[0][1] = zthick + zmin;
    cross_yz[1][0] = -m.rmax; cross_yz[1][1] = zmin;
    for (int k = 0; k < 30; k++) { cross_yz[2 + k][0] = n[k][0]; cross_yz[2 + k][1] = n[k][1] + zc + zmin; }
    cross_yz[32][0] = m.rmax; cross_yz[32][1] = zmin;
    cross_yz[33][0] = m.rmax; cross_yz[33][1] = zthick + zmin;
}

// per-field jaw polygons in float (setup_secjaws, init.cu:1504-1592)
void secjaws_polygons(const SecJaws &j, float x1, float x2, float y1, float y2, float sid, gegs_field &F)
{
    const float h = 0.5f;
    const float bminy[4][2] = {{x1 * j.zminy / sid - h, y1 * j.zminy / sid - h}, {x2 * j.zminy / sid + h, y1 * j.zminy / sid - h},
                               {x2 * j.zminy / sid + h, y2 * j.zminy / sid + h}, {x1 * j.zminy / sid - h, y2 * j.zminy / sid + h}};
    const float bminx[4][2] = {{x1 * j.zminx / sid - h, y1 * j.zminx / sid - h}, {x2 * j.zminx / sid + h, y1 * j.zminx / sid - h},
                               {x2 * j.zminx / sid + h, y2 * j.zminx / sid + h}, {x1 * j.zminx / sid - h, y2 * j.zminx / sid + h}};
    const float bmaxy[4][2] = {{-j.rmax, j.zminy}, {j.rmax, j.zminy}, {j.rmax, j.zmaxy}, {-j.rmax, j.zmaxy}};
    const float bmaxx[4][2] = {{-j.rmax, j.zminx}, {j.rmax, j.zminx}, {j.rmax, j.zmaxx}, {-j.rmax, j.zmaxx}};
    const float gy[8][2] = {{-j.rmax, j.zmaxy}, {-j.rmax, j.zminy}, {y1 * j.zminy / sid, j.zminy}, {y1 * j.zmaxy / sid, j.zmaxy},
                            {y2 * j.zmaxy / sid, j.zmaxy}, {y2 * j.zminy / sid, j.zminy}, {j.rmax, j.zminy}, {j.rmax, j.zmaxy}};
    const float gx[8][2] = {{-j.rmax, j.zmaxx}, {-j.rmax, j.zminx}, {x1 * j.zminx / sid, j.zminx}, {x1 * j.zmaxx / sid, j.zmaxx},
                            {x2 * j.zmaxx / sid, j.zmaxx}, {x2 * j.zminx / sid, j.zminx}, {j.rmax, j.zminx}, {j.rmax, j.zmaxx}};
    std::memcpy(F.boundMinY, bminy, sizeof bminy);
    std::memcpy(F.boundMinX, bminx, sizeof bminx);
    std::memcpy(F.boundMaxY, bmaxy, sizeof bmaxy);
    std::memcpy(F.boundMaxX, bmaxx, sizeof bmaxx);
    std::memcpy(F.jawsGeomY, gy, sizeof gy);
    std::memcpy(F.jawsGeomX, gx, sizeof gx);
}

// per-field leaf-end polygons in float (init_leaf_pos, init.cu:1594-1662):
// pair j is moved by POS = pos[j] and NEG = -pos[j+60] (the reference's bank
// swap); a pair whose positions do not add up to more than 0 keeps the outline
void leaf_endnodes(const float cross_yz[34][2], const float pos[120], float zmin, float zthick, float sid, gegs_field &F)
{
    const float zc = zmin + zthick / 2;
    for (int j = 0; j < 60; j++) {
        for (int k = 0; k < 34; k++) { F.endnode[j][k][0] = cross_yz[k][0]; F.endnode[j][k][1] = cross_yz[k][1]; }
        if (pos[j] + pos[j + 60] > 0.0f) {
            const float POS = pos[j], NEG = -pos[j + 60];
            for (int k = 2; k < 17; k++) F.endnode[j][k][0] = cross_yz[k][0] + NEG * zc / sid;
            for (int k = 17; k < 32; k++) F.endnode[j][k][0] = cross_yz[k][0] + POS * zc / sid;
        }
    }
}

}  // namespace

// ---- the plan -----------------------------------------------------------------
struct gegs_plan {
    gegs_physics physics{};
    gegs_scene scene{};
    std::vector<gegs_field> fields;
    std::vector<float> xb, yb, zb, rhof, density;
    std::vector<uint16_t> med;
    std::vector<gegs_phsp_record> phsp;
    std::vector<double> output_factor;
    uint64_t histories = 0;
    double dose_unit = 1.6e-8;
    std::string output_base;
};

namespace {

void read_physics_file(const fs::path &path, const std::vector<std::string> &media, gegs_physics &P)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) throw PlanError(path.string() + ": cannot open the physics file");
    char magic[8];
    uint32_t size = 0, nmed = 0;
    f.read(magic, 8);
    f.read((char *)&size, 4);
    f.read((char *)&nmed, 4);
    if (!f || std::memcmp(magic, "GEGSPHY1", 8) != 0) throw PlanError(path.string() + ": not a GEGSPHY1 physics file");
    if (size != sizeof(gegs_physics)) throw PlanError(path.string() + ": physics block of another layout");
    std::vector<std::string> names;
    for (uint32_t k = 0; k < nmed; k++) {
        char nm[33] = {};
        f.read(nm, 32);
        names.emplace_back(nm);
    }
    if (names != media) {
        std::string want, got;
        for (const auto &m : media) want += m + " ";
        for (const auto &m : names) got += m + " ";
        throw PlanError(path.string() + ": physics for media [" + got + "], the plan needs [" + want +
                        "] (write it with --write-physics)");
    }
    f.read((char *)&P, sizeof P);
    if (!f) throw PlanError(path.string() + ": truncated physics block");
    char msg[192];
    if (gegs_check_physics(&P, msg, sizeof msg) != GEGS_OK) throw PlanError(path.string() + ": " + msg);
}

void load(gegs_plan &pl, const fs::path &ini_path_in, const fs::path &physics_path, uint64_t max_hist)
{
    const fs::path ini_path = fs::absolute(ini_path_in).lexically_normal();
    const Ini ini = read_ini(ini_path);
    const fs::path here = ini_path.parent_path();
    const std::string prefix = ini_req(ini, "General", "output prefix");
    const fs::path outdir = data_path(here, ini_req(ini, "General", "output directory"));
    const float hpm = floats(ini_req(ini, "General", "histories"), 1, "histories")[0];
    const fs::path data_dir = data_path(here, ini_req(ini, "Data", "data directory"));
    auto data = [&](const std::string &n) { return data_path(data_dir, n); };
    const std::string default_medium = ini_opt(ini, "Data", "default medium", "AIR700ICRU");
    const fs::path egsinp = data(ini_req(ini, "Data", "egsinp file"));
    const bool secjaws_on = ini_on(ini, "SecJaws", "module SecJaws"), mlc_on = ini_on(ini, "MLC", "module MLC");
    if (ini_on(ini, "Block", "module Block")) throw PlanError("the Block module is not supported by this transport path");
    if (ini_on(ini, "Wedge", "module Wedge")) throw PlanError("the Wedge module is not supported by this transport path");
    if (ini_on(ini, "CTcreate", "use ctcreate"))
        throw PlanError("building the phantom from DICOM (use ctcreate = Yes) is not supported; give an egsphant file");

    Phantom ph = read_egsphant(data(ini_req(ini, "Phantom", "egsphant file")));
    const bool change_xyz = lower(strip(ini_opt(ini, "Phantom", "change coordinate", "Yes"))) != "no";
    const auto iso = floats(ini_req(ini, "Phantom", "isocenter location"), 3, "isocenter location");
    const float sid = floats(ini_req(ini, "Phantom", "source to isocenter"), 1, "source to isocenter")[0];

    SecJaws jaws{};
    DynVMLC mlc{};
    if (secjaws_on) jaws = read_secjaws(data(ini_opt(ini, "SecJaws", "secjaws file", "VarianMLC.egsinp")));
    if (mlc_on) mlc = read_dynvmlc(egsinp);
    std::vector<std::string> media = ph.media;
    const std::vector<std::string> other = {default_medium, secjaws_on ? jaws.media : default_medium,
                                            mlc_on ? mlc.media : default_medium, default_medium, default_medium};
    for (const auto &n : other)
        if (std::find(media.begin(), media.end(), n) == media.end()) media.push_back(n);
    if (media.size() > GEGS_MXMED) throw PlanError("more than GEGS_MXMED media");
    read_physics_file(physics_path, media, pl.physics);

    // phantom regions (init.cu:909-1052): density ratio to the medium's standard density
    gegs_scene &S = pl.scene;
    pl.xb = ph.xb; pl.yb = ph.yb; pl.zb = ph.zb;
    pl.med = ph.med;
    pl.density = ph.density;
    const size_t nvox = ph.med.size();
    pl.rhof.resize(nvox);
    for (size_t v = 0; v < nvox; v++) {
        const float d = ph.density[v];
        pl.rhof[v] = d == 0.0f ? 1.0f : d / pl.physics.rho[ph.med[v]];
    }
    S.nx = ph.nx; S.ny = ph.ny; S.nz = ph.nz;
    S.x_bounds = pl.xb.data(); S.y_bounds = pl.yb.data(); S.z_bounds = pl.zb.data();
    S.voxel_med = pl.med.data();
    S.voxel_rhof = pl.rhof.data();
    for (int k = 0; k < 5; k++) S.other_med[k] = (int32_t)(std::find(media.begin(), media.end(), other[k]) - media.begin());
    S.region_flags = GEGS_F_RAYLEIGH | GEGS_F_BOUND_COMPTON | GEGS_F_ATOMIC_RELAXATION | GEGS_F_PHOTO_ANGULAR;
    S.change_xyz = change_xyz ? 1 : 0;
    S.source_to_isocenter = sid;
    for (int k = 0; k < 3; k++) S.iso[k] = (float)iso[k];
    // module order (CUDA_EGS.cu:1277-1305)
    int8_t order[8] = {0};
    int nxt = GEGS_M_PHANTOM;
    if (mlc_on) { order[GEGS_M_VARMLC] = (int8_t)nxt; nxt = GEGS_M_VARMLC; }
    if (secjaws_on) { order[GEGS_M_SECJAWX] = (int8_t)nxt; order[GEGS_M_SECJAWY] = GEGS_M_SECJAWX; nxt = GEGS_M_SECJAWY; }
    order[0] = (int8_t)nxt;
    std::memcpy(S.module_order, order, 8);
    float cross_yz[34][2] = {};
    if (mlc_on) build_mlc(mlc, S, cross_yz);

    // phase space
    const long long nfiles = (long long)floats(ini_opt(ini, "Phase space", "phsp file number", "1"), 1, "phsp file number")[0];
    const std::string base = data(ini_req(ini, "Phase space", "phase space file")).string();
    if (nfiles <= 1) read_egsphsp1(base + ".egsphsp1", pl.phsp);
    else for (long long k = 0; k < nfiles; k++) read_egsphsp1(base + "_p" + std::to_string(k) + ".egsphsp1", pl.phsp);
    S.z_phsp = (float)floats(ini_req(ini, "Phase space", "z position"), 1, "z position")[0];
    if (pl.phsp.empty()) throw PlanError("the phase space holds no particles");

    // fields (read_mlcinfo / read_mlcinp, init.cu:1377-1500)
    struct FieldInfo { float angle, x1, x2, y1, y2; long long mu; std::string mlcinp; };
    std::vector<FieldInfo> finfo;
    const std::string *mlcinfo = ini_get(ini, "MLC", "mlcinfo file");
    if (mlc_on && !mlcinfo) throw PlanError("property \"mlcinfo file\" is not specified in the section \"MLC\"");
    if (mlcinfo) {
        Stream r(read_text(data(*mlcinfo)));
        r.ignore();
        const long long n = r.num_int();
        r.ignore();
        for (long long k = 0; k < std::min<long long>(n, 64); k++) {
            if (r.eof()) break;
            FieldInfo f{};
            r.num_sep_int();
            f.angle = r.num_sep(); f.x1 = r.num_sep(); f.x2 = r.num_sep(); f.y1 = r.num_sep(); f.y2 = r.num_sep();
            f.mu = r.num_sep_int();
            f.mlcinp = strip(r.getline());
            finfo.push_back(f);
        }
    } else {
        finfo.push_back(FieldInfo{0.0f, -20.0f, 20.0f, -20.0f, 20.0f, 1, ""});
    }
    if (finfo.empty()) throw PlanError("the mlcinfo file lists no fields");
    if ((int)finfo.size() > GEGS_MAX_FIELDS) throw PlanError("more fields than GEGS_MAX_FIELDS");
    // output factors: interpolation in sqrt(field area), in float (read_mlcinp,
    // init.cu:1449-1458); a field size outside the table leaves the reference's
    // factor unset, 0 in its zero-initialised field array
    pl.output_factor.assign(finfo.size(), 1.0);
    if (ini_on(ini, "Output factor", "use output factor")) {
        Stream r(read_text(data(ini_req(ini, "Output factor", "output factor file"))));
        r.ignore();
        const long long n = r.num_int();
        r.ignore();
        std::vector<std::pair<float, float>> tab;
        for (long long k = 0; k < n; k++) { float a = r.num(), b = r.num(); r.ignore(); tab.emplace_back(a, b); }
        for (size_t i = 0; i < finfo.size(); i++) {
            const FieldInfo &f = finfo[i];
            const float size = std::sqrt((f.x2 - f.x1) * (f.y2 - f.y1));
            pl.output_factor[i] = 0.0;
            for (size_t j = 0; j + 1 < tab.size(); j++)
                if (tab[j].first < size && size <= tab[j + 1].first) {
                    pl.output_factor[i] = (double)(tab[j].second + (size - tab[j].first) * (tab[j + 1].second - tab[j].second)
                                                                       / (tab[j + 1].first - tab[j].first));
                    break;
                }
        }
    }
    pl.fields.assign(finfo.size(), gegs_field{});
    uint64_t h = 0;
    for (size_t i = 0; i < finfo.size(); i++) {
        const FieldInfo &f = finfo[i];
        gegs_field &F = pl.fields[i];
        uint64_t n = (uint64_t)(f.mu * (long long)hpm);
        if (max_hist > 0) n = std::min(n, max_hist);
        const uint64_t nrep = n > 0 ? (n - 1) / pl.phsp.size() : 0;
        if (nrep > 255) throw PlanError("more than 256 uses of each phase-space particle; add phase-space particles");
        // gantry cos/sin as the reference uploads them (CUDA_EGS.cu:420-422): the
        // angle times 3.1415926 / 180 in double, stored as a float; cos and sin
        // of that float, correctly rounded
        const float a = (float)((double)f.angle * 3.1415926 / 180);
        F.cos_angle = (float)std::cos((double)a);
        F.sin_angle = (float)std::sin((double)a);
        F.hist_begin = h; F.hist_end = h + n;
        F.nrepeat = (int32_t)nrep;
        if (secjaws_on) secjaws_polygons(jaws, f.x1, f.x2, f.y1, f.y2, sid, F);
        if (mlc_on) {
            float pos[120];
            Stream r(read_text(data(f.mlcinp)));
            for (int k = 0; k < 14; k++) r.ignore();
            for (int j = 0; j < 120; j++) { r.ignore(10, '\n'); pos[j] = (float)r.num(); r.ignore(); }
            leaf_endnodes(cross_yz, pos, mlc.zmin, mlc.zthick, sid, F);
        }
        h += n;
    }
    pl.histories = h;
    S.nfields = (int32_t)pl.fields.size();
    S.fields = pl.fields.data();
    S.phsp = pl.phsp.data();
    S.nphsp = pl.phsp.size();
    S.hownear_region_offset = 5;
    S.seed = 0x6E65;
    pl.dose_unit = 1.6e-8f;                              // a float (CUDA_EGS.h:536)
    if (ini_on(ini, "Calibration", "dose calibration")) {
        const float hpc = floats(ini_req(ini, "Calibration", "histories per cGy"), 1, "histories per cGy")[0];
        pl.dose_unit = 1.6e-8f * hpc / hpm;              // in float (CUDA_EGS.cu:1478)
    }
    pl.output_base = (outdir / prefix).string();
}

gegs_status fail(char *msg, size_t len, const std::string &text)
{
    if (msg && len) std::snprintf(msg, len, "%s", text.c_str());
    return GEGS_ERR_ARG;
}

}  // namespace

extern "C" {

gegs_status gegs_plan_load(const char *ini_path, const char *physics_path, uint64_t max_histories_per_field,
                           gegs_plan **out, char *msg, size_t msg_len)
{
    if (!out) return fail(msg, msg_len, "gegs_plan_load: out is NULL");
    *out = nullptr;
    if (!ini_path || !physics_path) return fail(msg, msg_len, "gegs_plan_load: a path is NULL");
    gegs_plan *p = new gegs_plan();
    try {
        load(*p, ini_path, physics_path, max_histories_per_field);
    } catch (const std::exception &ex) {
        delete p;
        return fail(msg, msg_len, ex.what());
    }
    if (msg && msg_len) msg[0] = '\0';
    *out = p;
    return GEGS_OK;
}

void gegs_plan_free(gegs_plan *p) { delete p; }
const gegs_physics *gegs_plan_physics(const gegs_plan *p) { return p ? &p->physics : nullptr; }
const gegs_scene *gegs_plan_scene(const gegs_plan *p) { return p ? &p->scene : nullptr; }
uint64_t gegs_plan_histories(const gegs_plan *p) { return p ? p->histories : 0; }
uint64_t gegs_plan_nvox(const gegs_plan *p) { return p ? (uint64_t)p->med.size() : 0; }
double gegs_plan_dose_unit(const gegs_plan *p) { return p ? p->dose_unit : 0.0; }
int32_t gegs_plan_nfields(const gegs_plan *p) { return p ? (int32_t)p->fields.size() : 0; }

double gegs_plan_output_factor(const gegs_plan *p, int32_t field)
{
    if (!p || field < 0 || field >= (int32_t)p->output_factor.size()) return 0.0;
    return p->output_factor[(size_t)field];
}

gegs_status gegs_plan_voxel_mass(const gegs_plan *p, float *mass, uint64_t nvox)
{
    if (!p || !mass || nvox != p->med.size()) return GEGS_ERR_ARG;
    const int nx = p->scene.nx, ny = p->scene.ny, nz = p->scene.nz;
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                // (dx * dy) * dz in float, made positive, times the density (init.cu:1256-1271)
                float vol = (p->xb[x + 1] - p->xb[x]) * (p->yb[y + 1] - p->yb[y]) * (p->zb[z + 1] - p->zb[z]);
                if (vol < 0) vol = -vol;
                const size_t v = ((size_t)z * ny + y) * nx + x;
                const float m = vol * p->density[v];
                mass[v] = m == 0.0f ? 1.0f : m;
            }
    return GEGS_OK;
}

gegs_status gegs_plan_dose(const gegs_plan *p, const int64_t *tally, float *dose, uint64_t nvox)
{
    if (!p || !tally || !dose || nvox != p->med.size()) return GEGS_ERR_ARG;
    std::vector<float> mass(nvox);
    gegs_plan_voxel_mass(p, mass.data(), nvox);
    const float unit = (float)p->dose_unit;
    // (float)E / mass * dose_unit in float, E the energy in MeV (write_dose, output.c:887-891)
    for (uint64_t v = 0; v < nvox; v++) dose[v] = (float)((double)tally[v] * 9.313225746154785e-10) / mass[v] * unit;
    return GEGS_OK;
}

gegs_status gegs_plan_write_dose(const gegs_plan *p, const float *dose, uint64_t nvox, char *path, size_t path_len)
{
    if (!p || !dose || nvox != p->med.size()) return GEGS_ERR_ARG;
    char tail[64];
    std::snprintf(tail, sizeof tail, "_DoseResults_%03dx%03dx%03d.bin", p->scene.nx, p->scene.ny, p->scene.nz);
    const std::string name = p->output_base + tail;
    std::error_code ec;
    fs::create_directories(fs::path(name).parent_path(), ec);
    FILE *f = std::fopen(name.c_str(), "wb");
    if (!f) return GEGS_ERR_ARG;
    const size_t w = std::fwrite(dose, sizeof(float), (size_t)nvox, f);
    std::fclose(f);
    if (w != nvox) return GEGS_ERR_ARG;
    if (path && path_len) std::snprintf(path, path_len, "%s", name.c_str());
    return GEGS_OK;
}

}  // extern "C"
