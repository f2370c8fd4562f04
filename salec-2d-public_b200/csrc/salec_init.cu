// Standalone initialisation: input deck -> device-resident simulation.
//
// Restates the reference's start-up sequence (src/salec2d.c:45-105) on the host: deck
// parsing, run parameters and material records (src/sale2d_back.c:64-402), EOS tables
// (src/eos/eos_state.c:463-526, 635-662, src/eos/aneos_sieden.c:11-73, 196-262), mesh
// geometry (src/construct.c:11-594 with the quadratures of src/geometry/interpolate.c and
// src/geometry/interpolate_2d9.c), the hydrostatic target profile and the material
// distribution (src/target_profile.c:86-343, 572-1195). The fields are produced in the
// reference's layout, uploaded through the same path as salec_gpu_set_field, and the last
// steps (first EOS call, ghost fills, PML reference state, vertex velocities) run on the
// device with the step kernels. Arithmetic keeps the reference's operation order, so with
// the same glibc the initial state is the reference's to the last bit.
#include "../../include/salec_gpu.h"
#include "salec_deck.h"
#include "salec_device.cuh"
#include "salec_kernels.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

namespace salec {

// ================================================================== deck reader
namespace {

std::string lower(std::string s)
{
    for (auto &ch : s) ch = (char)tolower((unsigned char)ch);
    return s;
}

std::string trim_ref(const std::string &s)
{
    // rtrim whitespace; ltrim whitespace and '.' (src/io/InputParser.c:7-47)
    size_t e = s.size();
    while (e > 0 && isspace((unsigned char)s[e - 1])) --e;
    size_t b = 0;
    while (b < e && (isspace((unsigned char)s[b]) || s[b] == '.')) ++b;
    return s.substr(b, e - b);
}

// First run of characters outside `delim` after skipping leading delimiters; returns the
// index just past the run and any delimiters that follow it (Strok).
size_t take_token(const std::string &s, size_t from, const char *delim, std::string &tok)
{
    auto is_d = [&](char ch) { return strchr(delim, ch) != nullptr && ch != 0; };
    size_t p = from;
    tok.clear();
    while (p < s.size() && is_d(s[p])) ++p;
    while (p < s.size() && !is_d(s[p])) tok.push_back(s[p++]);
    while (p < s.size() && is_d(s[p])) ++p;
    return p;
}

// element k of "[a, b, c]"; returns false if the value is not a list
bool list_elem(const std::string &v, int k, std::string &out)
{
    out.clear();
    if (v.size() < 2 || v.front() != '[' || v.back() != ']') return false;
    int idx = 0;
    for (size_t i = 1; i + 1 < v.size(); ++i) {
        if (v[i] == ',') { ++idx; continue; }
        if (idx > k) break;
        if (idx == k) out.push_back(v[i]);
    }
    return true;
}

} // namespace

bool Deck::load(const std::string &path, bool eos_file, std::string &err)
{
    std::ifstream in(path);
    if (!in) { err = "cannot open " + path; return false; }
    std::string line, field = "mesh";
    const char *sub = eos_file ? "/#*\"" : "#*\"";
    while (std::getline(in, line)) {
        line = trim_ref(line);
        if (line.empty()) continue;
        if (strchr("\"#/-*", line[0])) continue;
        if (line.front() == '[' && line.back() == ']') { field = line.substr(1, line.size() - 2); continue; }
        std::string key, val;
        size_t r = take_token(line, 0, "= ", key);
        take_token(line, r, sub, val);
        if (key.empty() || val.empty()) continue;
        std::string full = key.find('.') == std::string::npos ? field + "." + key : key;
        kv_[lower(trim_ref(full))] = trim_ref(val);
    }
    return true;
}

const std::string *Deck::find(const std::string &key) const
{
    auto it = kv_.find(lower(key));
    return it == kv_.end() ? nullptr : &it->second;
}

bool Deck::has(const std::string &key) const { return find(key) != nullptr; }

std::string Deck::str(const std::string &key, const std::string &def) const
{
    const std::string *v = find(key);
    return v ? *v : def;
}

double Deck::num(const std::string &key, const std::string &def) const
{
    const std::string *v = find(key);
    return strtod((v ? *v : def).c_str(), nullptr);
}

int Deck::integer(const std::string &key, const std::string &def) const
{
    const std::string *v = find(key);
    return (int)strtol((v ? *v : def).c_str(), nullptr, 10);
}

double Deck::num_k(const std::string &key, int k, const std::string &def) const
{
    const std::string *v = find(key);
    if (!v) return strtod(def.c_str(), nullptr);
    std::string e;
    if (!list_elem(*v, k, e)) return k == 0 ? strtod(v->c_str(), nullptr) : strtod(def.c_str(), nullptr);
    return e.empty() ? strtod(def.c_str(), nullptr) : strtod(e.c_str(), nullptr);
}

int Deck::integer_k(const std::string &key, int k, const std::string &def) const
{
    const std::string *v = find(key);
    if (!v) return (int)strtod(def.c_str(), nullptr);
    std::string e;
    if (!list_elem(*v, k, e)) return k == 0 ? (int)strtol(v->c_str(), nullptr, 10) : (int)strtol(def.c_str(), nullptr, 10);
    return e.empty() ? (int)strtol(def.c_str(), nullptr, 10) : (int)strtol(e.c_str(), nullptr, 10);
}

std::string Deck::str_k(const std::string &key, int k, const std::string &def) const
{
    const std::string *v = find(key);
    if (!v) return def;
    std::string e;
    if (!list_elem(*v, k, e)) return k == 0 ? *v : def;
    e = trim_ref(e);
    return e.empty() ? def : e;
}

// ================================================================== init state
namespace {

enum EosKind { K_ANEOS = 0, K_TILL = 1, K_SIEDEN = 2, K_UNKNOWN = 3 };

struct Table {
    int ntem = 0, nden = 0;
    double Pnorm = 0, Tnorm = 0, Dnorm = 0;
    std::vector<double> xtem, yden, data;   // data[(iT*nden + iD)*3 + c]
    double D(int it, int id, int c) const { return data[((size_t)it * nden + id) * 3 + c]; }
};

struct Mat {
    EosKind kind = K_UNKNOWN;
    salec_material_desc d{};
    std::string yfunc, tfunc, dsdf, porfunc;
    double den0 = 0, c_heat = 0, thermexp = 0;
    std::vector<double> cold_x, cold_y;    // Tillotson cold curve
    Table tab;
};

struct TargetInfo {
    int n_layer = 1, sphere = 0;
    int material[10] = {0};
    double depth[10] = {0};
    int n_profile = 3001;
    double max_depth = 1.0, r_planet = 0, center[2] = {0, 0};
    int tem_type = 0;   // 0 const, 1 conductive, 2 convective, 3 lunar
    double surf_tem = 293, surf_dtdz = 0, surf_pre = 1e-5, surf_gravity = -1.63, t_lith = -1, d_lith = -1;
    double d_mantle = -1, t_mantle = -1;
};

struct Addition {
    int material = 0, type = 0;   // 0 sphere, 1 cube
    double par[12] = {0};
};

struct Setup {
    int npgx = 1, npgy = 1, nx = 0, ny = 0, nmat = 0;
    double dx = 1, dy = 1, oy = 0.7, ox = 0;
    double x_ext = -1, y_ext = -1;
    int nx_ext[2] = {0, 0}, ny_ext[2] = {0, 0};
    double avis1, avis2, anc, anc_depth, anc_width;
    std::string anc_pattern;
    double ejecta_threshold, ejecta_resistance, ejecta_friction, density_cutoff, velocity_max, velocity_min,
        acceleration_min;
    int partpres = 0, damp_type = 5, damp_x = 0, damp_y = 0, damp_x_left = 0, damp_y_top = 0, tracer_strip = 2;
    double lambda_x = 10, lambda_y = 10, damp_t = -1;
    double gravity[2] = {0, -1.62};
    int go[4] = {0, 0, 0, 0};
    int tensile_failure = 0, tracer_lubrication = 0;
    double tracer_lub_y0 = 0, tracer_lub_frac = 0;
    int tracer_lub_gy0 = 0, tracer_lub_gy1 = 0;   // rows of lubricating tracers (set with the mesh)
    // cycle
    double time0 = 0, time1 = 100, max_dt = 1, dt0 = 0;
    // projectile
    int p_mat = -1;
    double p_radius = 1, p_center[2] = {0, 300}, p_vel[2] = {0, -1000}, p_dam = 1, p_pre = 1, p_tem = 293;
    TargetInfo tinfo;
    std::vector<Addition> additions;
    std::vector<Mat> mats;
    // derived
    double alpha_damp_x = 0, alpha_damp_y = 0;
    int porosity_model = 0, acoustic_fluid = 0;
};

// ---------------------------------------------------------------- EOS on the host
double till_eos_interp_tp(const Mat &m, double tem, double pre, int id)
{
    // TillEOSInterpolateTP (src/eos/eos_state.c:528-579)
    const double *t = m.d.till;
    const double thermal = (tem - t[11]) * t[1];
    int di = 0, dj = (int)m.cold_x.size() - 1;
    while (di + 1 < dj) {
        int dm = (di + dj) / 2;
        double p, c;
        till_pressure(t, m.cold_y[dm] + thermal, m.cold_x[dm], p, c);
        if (p > pre) dj = dm; else di = dm;
    }
    double lo = m.cold_x[di], hi = m.cold_x[dj], mid = 0, e = 0, p = 0, c = 0;
    for (int k = 0; k < 50; ++k) {
        double err = (hi - lo) / hi;
        mid = (lo + hi) / 2.0;
        if (err < 1e-12) break;
        double dxl = (m.cold_x[dj] - mid) / t[12];
        double dxr = 1.0 - dxl;
        e = dxl * m.cold_y[di] + dxr * m.cold_y[dj] + thermal;
        till_pressure(t, e, mid, p, c);
        if (p > pre) hi = mid; else lo = mid;
    }
    if (id == -1) return mid;
    if (id == 0) return e * mid;
    if (id == 1) return pre;
    return c;
}

int vec_cmp4(const double *x, double y)
{
    int r = 0;
    for (int k = 0; k < 4; ++k)
        if (x[k] > y) r++;
    return r;
}

int abilinear(const double *x, const double *y, double *xl)
{
    // inverse bilinear map of a quadrilateral (src/geometry/linear.c:220-297)
    static const double bf[4][5] = {{1.0, -1.0, 1.0, -1.0, 0.0}, {-1.0, 1.0, 1.0, -1.0, 0.0},
                                    {-1.0, -1.0, 1.0, 1.0, 0.0}, {1.0, 1.0, 1.0, 1.0, -4.0}};
    double a[4] = {0.}, b[4] = {0.};
    for (int k = 0; k < 4; ++k)
        for (int j = 0; j < 5; ++j) {
            a[k] += bf[k][j] * x[j];
            b[k] += bf[k][j] * y[j];
        }
    double tA = -a[0] * b[2] + a[2] * b[0];
    double tB = -a[0] * b[3] + a[3] * b[0] - a[1] * b[2] + a[2] * b[1];
    double tC = -a[1] * b[3] + a[3] * b[1];
    double tD = tB * tB - 4.0 * tA * tC;
    double xt[4] = {0.0, 0.0, 0.0, 0.0};
    int ret = 0;
    if (tD < 0.) {
        ret = 0;
    } else if (fabs(tD) < 1e-24) {
        xt[1] = -tB / (2. * tA);
        xt[0] = -1.0 * (a[2] * xt[1] + a[3]) / (a[0] * xt[1] + a[1]);
        ret = 1;
        if (fabs(xt[0]) > 1.0 || fabs(xt[1]) > 1.0) { xt[0] = 0.0; xt[1] = 0.0; ret--; }
    } else {
        xt[1] = (-tB + sqrt(tD)) / (2. * tA);
        xt[0] = -1.0 * (a[2] * xt[1] + a[3]) / (a[0] * xt[1] + a[1]);
        xt[3] = (-tB - sqrt(tD)) / (2. * tA);
        xt[2] = -1.0 * (a[2] * xt[3] + a[3]) / (a[0] * xt[3] + a[1]);
        ret = 2;
        if (fabs(xt[0]) > 1.0 || fabs(xt[1]) > 1.0) { xt[0] = 0.0; xt[1] = 0.0; ret--; }
        if (fabs(xt[2]) > 1.0 || fabs(xt[3]) > 1.0) { xt[2] = 0.; xt[3] = 0.; ret--; }
    }
    if ((fabs(xt[2]) + fabs(xt[3])) > (fabs(xt[1]) + fabs(xt[0]))) { xl[0] = xt[2]; xl[1] = xt[3]; }
    else { xl[0] = xt[0]; xl[1] = xt[1]; }
    return ret;
}

// First (energy row, density column) cell, in row order, whose corner temperatures and
// pressures bracket (tem, pre) and whose bilinear inverse has a root in the cell: the
// search of ANEOSSieDenInterpolateTP (src/eos/aneos_sieden.c:124-194), with the bracket
// test on per-cell minima and maxima (equivalent to its corner counts) to skip cells fast.
bool sieden_locate(const Table &t, double tem, double pre, int &ti, int &di, double *xl)
{
    xl[0] = xl[1] = 0.;
    for (ti = 0; ti < t.ntem - 1; ++ti) {
        for (di = 0; di < t.nden - 1; ++di) {
            const double p4[4] = {t.D(ti, di, 1), t.D(ti + 1, di, 1), t.D(ti + 1, di + 1, 1), t.D(ti, di + 1, 1)};
            int pc = vec_cmp4(p4, pre);
            if (pc <= 0 || pc >= 4) continue;
            const double t4[4] = {t.D(ti, di, 0), t.D(ti + 1, di, 0), t.D(ti + 1, di + 1, 0), t.D(ti, di + 1, 0)};
            int tc = vec_cmp4(t4, tem);
            if (tc <= 0 || tc >= 4) continue;
            const double pin[5] = {p4[0], p4[1], p4[2], p4[3], pre};
            const double tin[5] = {t4[0], t4[1], t4[2], t4[3], tem};
            if (abilinear(tin, pin, xl) != 0) return true;
        }
    }
    return false;
}

double sieden_interp_tp(const Mat &m, double tem, double pre, int id)
{
    const Table &t = m.tab;
    int ti = 0, di = 0;
    double xl[2];
    sieden_locate(t, tem, pre, ti, di, xl);
    xl[0] = (xl[0] + 1.0) / 2.0;
    xl[1] = (xl[1] + 1.0) / 2.0;
    if (id == 0) {
        double r = t.xtem[ti] * (1.0 - xl[0]) + t.xtem[ti + 1] * xl[0];
        return r * (t.yden[di] * (1.0 - xl[1]) + t.yden[di + 1] * xl[1]);
    }
    if (id == -1) return t.yden[di] * (1.0 - xl[1]) + t.yden[di + 1] * xl[1];
    return 0.0;
}

double aneos_interp_tp(const Mat &m, double tem, double pre, int id)
{
    // ANEOSInterpolateTP (src/eos/eos_state.c:206-256)
    const Table &t = m.tab;
    int ti = 0, tj = t.ntem;
    while (ti + 1 < tj) {
        int tm = (ti + tj) / 2;
        if (t.xtem[tm] > tem) tj = tm; else ti = tm;
    }
    double txr = (tem - t.xtem[ti]) / (t.xtem[tj] - t.xtem[ti]);
    double txl = 1.0 - txr;
    int di = 0, dj = t.nden - 1;
    double irp = t.D(ti, di, 1) * txl + t.D(tj, di, 1) * txr;
    double jrp = t.D(ti, dj, 1) * txl + t.D(tj, dj, 1) * txr;
    while (di + 1 < dj) {
        int dm = (di + dj) / 2;
        double mrp = t.D(ti, dm, 1) * txl + t.D(tj, dm, 1) * txr;
        if (mrp > pre) { dj = dm; jrp = mrp; } else { di = dm; irp = mrp; }
    }
    double dxr = (pre - irp) / (jrp - irp);
    dxr = wind(dxr, 0.0, 1.0);
    double dxl = 1.0 - dxr;
    if (id == -1) return t.yden[di] * dxl + t.yden[dj] * dxr;
    return (t.D(ti, di, id) * dxl + t.D(ti, dj, id) * dxr) * txl + (t.D(tj, di, id) * dxl + t.D(tj, dj, id) * dxr) * txr;
}

double eos_interp_tp(const Mat &m, double tem, double pre, int id)
{
    if (m.kind == K_TILL) return till_eos_interp_tp(m, tem, pre, id);
    if (m.kind == K_SIEDEN) return sieden_interp_tp(m, tem, pre, id);
    return aneos_interp_tp(m, tem, pre, id);
}

void till_cold_curve(Mat &m)
{
    // TillColdEnergy (src/eos/eos_state.c:463-517): classic RK4 of dE/drho = p/rho^2
    double *t = m.d.till;
    const double ref = t[0], maxd = t[0] * 10.0;
    const int n = (int)m.cold_x.size();
    double step = maxd / (n - 1);
    for (int k = 0; k < n; ++k) { m.cold_x[k] = k * step; m.cold_y[k] = 0.0; }
    const int im = (int)(floor(ref / maxd * n));
    m.cold_x[im] = t[0];
    m.cold_y[im] = 0.0;
    auto dedr = [&](double e, double r) {
        double p, c;
        till_pressure(t, e, r, p, c);
        return p / (r * r);
    };
    for (int k = im + 1; k < n; ++k) {
        step = m.cold_x[k] - m.cold_x[k - 1];
        double e0 = m.cold_y[k - 1], r0 = m.cold_x[k - 1];
        double k1 = dedr(e0, r0);
        double k2 = dedr(e0 + 0.50 * k1 * step, r0 + 0.50 * step);
        double k3 = dedr(e0 + 0.50 * k2 * step, r0 + 0.50 * step);
        double k4 = dedr(e0 + k3 * step, r0 + step);
        m.cold_y[k] = e0 + (k1 + 2.0 * k2 + 2.0 * k3 + k4) * step / 6.0;
    }
    for (int k = im - 1; k >= 1; --k) {
        step = m.cold_x[k] - m.cold_x[k + 1];
        double e0 = m.cold_y[k + 1], r0 = m.cold_x[k + 1];
        double k1 = dedr(e0, r0);
        double k2 = dedr(e0 + 0.50 * k1 * step, r0 + 0.50 * step);
        double k3 = dedr(e0 + 0.50 * k2 * step, r0 + 0.50 * step);
        double k4 = dedr(e0 + k3 * step, r0 + step);
        m.cold_y[k] = e0 + (k1 + 2.0 * k2 + 2.0 * k3 + k4) * step / 6.0;
    }
    m.cold_y[0] = m.cold_y[1];
    t[12] = maxd / (n - 1);
}

// bilinear shape-function derivatives in the reference's corner order lb, rb, ru, lu
inline double ipb(int k, double x0, double x1)
{
    switch (k) {
    case 0: return 0.25 * (1 - x0) * (1 - x1);
    case 1: return 0.25 * (1 + x0) * (1 - x1);
    case 2: return 0.25 * (1 + x0) * (1 + x1);
    default: return 0.25 * (1 - x0) * (1 + x1);
    }
}
inline double ipb_d(int k, int dim, double x0, double x1)
{
    switch (k) {
    case 0: return dim == 0 ? -0.25 * (1 - x1) : -0.25 * (1 - x0);
    case 1: return dim == 0 ? 0.25 * (1 - x1) : -0.25 * (1 + x0);
    case 2: return dim == 0 ? 0.25 * (1 + x1) : 0.25 * (1 + x0);
    default: return dim == 0 ? -0.25 * (1 + x1) : 0.25 * (1 - x0);
    }
}

bool load_tables(Setup &S, const std::string &eosdir, const Deck &deck, std::string &err)
{
    for (int m = 1; m < S.nmat; ++m) {
        Mat &M = S.mats[m];
        std::string name = deck.str_k("material.name", m, "vacuum_");
        std::string post = lower(deck.str_k("material.postfix", m, "null"));
        std::string path;
        if (post == "aneos") { M.kind = K_ANEOS; path = eosdir + "/" + name + ".aneos"; }
        else if (post == "tillotson") { M.kind = K_TILL; path = eosdir + "/" + name + ".tillotson"; }
        else if (post == "aneos.sd") { M.kind = K_SIEDEN; path = eosdir + "/" + name + ".aneos.sd"; }
        else if (post == "aneos.td") { M.kind = K_ANEOS; path = eosdir + "/" + name + ".aneos.td"; }
        else { err = "unknown EOS type for material " + name; return false; }
        salec_material_desc &d = M.d;
        if (M.kind == K_TILL) {
            Deck e;
            if (!e.load(path, true, err)) return false;
            double *t = d.till;
            t[0] = e.num("Tillostson.Rho0", "2.7e3"); t[1] = e.num("ColdEnergy.Cv", "8.96e2");
            t[2] = e.num("Tillostson.BulkA", "7.52e10"); t[3] = e.num("Tillostson.BulkB", "6.50e10");
            t[4] = e.num("Tillostson.E0", "5.0e6"); t[5] = e.num("Tillostson.Ta", "0.50");
            t[6] = e.num("Tillostson.Tb", "1.63"); t[7] = e.num("Tillostson.Alpha", "5.0");
            t[8] = e.num("Tillostson.Beta", "5.0"); t[9] = e.num("Tillostson.Eiv", "3.00e6");
            t[10] = e.num("Tillostson.Ecv", "1.39e7"); t[11] = e.num("ColdEnergy.Tref", "293.0");
            int n = e.integer("ColdEnergy.RhoStep", "1501");
            M.cold_x.assign(n, 0.0);
            M.cold_y.assign(n, 0.0);
            till_cold_curve(M);
            // TillInitStateRef (src/eos/eos_state.c:581-593)
            d.MeltDen = 0.85 * t[0];
            double gasmin = 1.0e-4 * t[0];
            d.VaporDen = gasmin * 10.0;
            M.c_heat = t[1];
            M.thermexp = t[1] * (t[6] + t[5]) / (t[2] / t[0]);
            M.den0 = t[0];
            d.gamfrac = (t[6] + t[5]) / (t[2] / t[0]);
        } else {
            FILE *fp = fopen(path.c_str(), "r");
            if (!fp) { err = "cannot open " + path; return false; }
            Table &T = M.tab;
            char buf[1024];
            for (int k = 0; k < 3; ++k)
                if (!fgets(buf, sizeof(buf), fp)) { fclose(fp); err = "short table " + path; return false; }
            bool ok = true;
            if (M.kind == K_SIEDEN) {
                // LoadANEOSSieDen layout (src/eos/aneos_sieden.c:11-73)
                ok = fscanf(fp, "%d %d", &T.nden, &T.ntem) == 2 && fscanf(fp, "%le %le", &T.Pnorm, &T.Tnorm) == 2;
                T.xtem.resize(ok ? T.ntem : 0);
                T.yden.resize(ok ? T.nden : 0);
                T.data.assign(ok ? (size_t)T.ntem * T.nden * 3 : 0, 0.0);
                for (int i = 0; ok && i < T.ntem; ++i) ok = fscanf(fp, "%le", &T.xtem[i]) == 1;
                for (int i = 0; ok && i < T.nden; ++i) ok = fscanf(fp, "%le", &T.yden[i]) == 1;
                for (int j = 0; ok && j < T.nden; ++j)
                    for (int i = 0; ok && i < T.ntem; ++i) {
                        double *q = &T.data[((size_t)i * T.nden + j) * 3];
                        ok = fscanf(fp, "%le %le %le", q, q + 1, q + 2) == 3;
                    }
            } else {
                // LoadANEOS layout (src/eos/eos_state.c:94-146); energies stored as energy*density
                ok = fscanf(fp, "%d %d", &T.ntem, &T.nden) == 2 &&
                     fscanf(fp, "%le %le %le", &T.Tnorm, &T.Dnorm, &T.Pnorm) == 3;
                T.xtem.resize(ok ? T.ntem : 0);
                T.yden.resize(ok ? T.nden : 0);
                T.data.assign(ok ? (size_t)T.ntem * T.nden * 3 : 0, 0.0);
                for (int i = 0; ok && i < T.ntem; ++i) ok = fscanf(fp, "%le", &T.xtem[i]) == 1;
                for (int i = 0; ok && i < T.ntem; ++i)
                    for (int j = 0; ok && j < T.nden; ++j) {
                        double *q = &T.data[((size_t)i * T.nden + j) * 3];
                        ok = fscanf(fp, "%le %le %le", q, q + 1, q + 2) == 3;
                    }
                for (int i = 0; ok && i < T.nden; ++i) ok = fscanf(fp, "%le", &T.yden[i]) == 1;
                for (int i = 0; ok && i < T.ntem; ++i)
                    for (int j = 0; j < T.nden; ++j) T.data[((size_t)i * T.nden + j) * 3] *= T.yden[j];
            }
            fclose(fp);
            if (!ok || T.ntem < 2 || T.nden < 2) { err = "malformed table " + path; return false; }
            if (M.kind == K_SIEDEN) {
                // ANEOSSieDenInitStateRef (src/eos/aneos_sieden.c:196-262)
                int ti = 0, di = 0;
                double xl[2];
                sieden_locate(T, T.Tnorm, T.Pnorm, ti, di, xl);
                int tj = ti + 1, dj = di + 1;
                if (ti >= T.ntem - 1) { ti = T.ntem - 2; tj = ti + 1; }
                if (di >= T.nden - 1) { di = T.nden - 2; dj = di + 1; }
                T.Dnorm = T.yden[di] * (1.0 - xl[1]) / 2.0 + T.yden[dj] * (1.0 + xl[1]) / 2.0;
                // the reference's sound speed keeps only the first two corner terms
                double cs = T.D(ti, di, 2) * ipb(0, xl[0], xl[1]) + T.D(ti + 1, di, 2) * ipb(1, xl[0], xl[1]);
                d.MeltDen = 0.85 * T.Dnorm;
                d.VaporDen = 0.04 * T.Dnorm;
                double dpde = ipb_d(0, 0, xl[0], xl[1]) * T.D(ti, di, 1) + ipb_d(1, 0, xl[0], xl[1]) * T.D(tj, di, 1)
                            + ipb_d(2, 0, xl[0], xl[1]) * T.D(tj, dj, 1) + ipb_d(3, 0, xl[0], xl[1]) * T.D(ti, dj, 1);
                double dtde = ipb_d(0, 0, xl[0], xl[1]) * T.D(ti, di, 0) + ipb_d(1, 0, xl[0], xl[1]) * T.D(tj, di, 0)
                            + ipb_d(2, 0, xl[0], xl[1]) * T.D(tj, dj, 0) + ipb_d(3, 0, xl[0], xl[1]) * T.D(ti, dj, 0);
                dpde *= 2.0 / (T.xtem[tj] - T.xtem[ti]);
                dtde *= 2.0 / (T.xtem[tj] - T.xtem[ti]);
                M.den0 = T.Dnorm;
                M.thermexp = (dpde / dtde) / (cs * cs * T.Dnorm);
                M.c_heat = 1.0 / dtde;
                d.gamfrac = M.thermexp / M.c_heat;
            } else {
                // ANEOSInitStateRef (src/eos/eos_state.c:148-204)
                int ti = 0, tj = T.ntem;
                while (ti + 1 < tj) {
                    int tm = (ti + tj) / 2;
                    if (T.xtem[tm] > T.Tnorm) tj = tm; else ti = tm;
                }
                double txr = (T.Tnorm - T.xtem[ti]) / (T.xtem[tj] - T.xtem[ti]);
                double txl = 1.0 - txr;
                int di = 0, dj = T.nden - 1;
                double irp = T.D(ti, di, 1) * txl + T.D(tj, di, 1) * txr;
                double jrp = T.D(ti, dj, 1) * txl + T.D(tj, dj, 1) * txr;
                while (di + 1 < dj) {
                    int dm = (di + dj) / 2;
                    double mrp = T.D(ti, dm, 1) * txl + T.D(tj, dm, 1) * txr;
                    if (mrp > T.Pnorm) { dj = dm; jrp = mrp; } else { di = dm; irp = mrp; }
                }
                double dxr = (T.Pnorm - irp) / (jrp - irp);
                double dxl = 1.0 - dxr;
                T.Dnorm = T.yden[di] * dxl + T.yden[dj] * dxr;
                d.MeltDen = 0.85 * T.Dnorm;
                d.VaporDen = 0.04 * T.Dnorm;
                double l0 = txr * 2.0 - 1.0, l1 = dxr * 2.0 - 1.0;
                double dpdt = ipb_d(0, 0, l0, l1) * T.D(ti, di, 1) + ipb_d(1, 0, l0, l1) * T.D(tj, di, 1)
                            + ipb_d(2, 0, l0, l1) * T.D(tj, dj, 1) + ipb_d(3, 0, l0, l1) * T.D(ti, dj, 1);
                dpdt *= 2.0 / (T.xtem[tj] - T.xtem[ti]);
                double cs = (T.D(ti, di, 2) * dxl + T.D(ti, dj, 2) * dxr) * txl + (T.D(tj, di, 2) * dxl + T.D(tj, dj, 2) * dxr) * txr;
                M.thermexp = dpdt / (cs * cs * T.Dnorm);
                double dedt = ipb_d(0, 0, l0, l1) * T.D(ti, di, 0) / T.yden[di] + ipb_d(3, 0, l0, l1) * T.D(ti, dj, 0) / T.yden[dj]
                            + ipb_d(1, 0, l0, l1) * T.D(tj, di, 0) / T.yden[di] + ipb_d(2, 0, l0, l1) * T.D(tj, dj, 0) / T.yden[dj];
                dedt *= 2.0 / (T.xtem[tj] - T.xtem[ti]);
                M.c_heat = dedt;
                M.den0 = T.Dnorm;
                d.gamfrac = M.thermexp / M.c_heat;
            }
        }
    }
    return true;
}

int func_of(const std::string &name)
{
    return salec_gpu_func_index(name.c_str());
}

bool load_setup(Setup &S, const Deck &D, const std::string &eosdir, std::string &err)
{
    // cycle (src/sale2d.c:6-64)
    S.time0 = D.num("cycle.time0", "0.0");
    S.time1 = D.num("cycle.time1", "100.0");
    S.max_dt = D.num("cycle.maxdt", "1.0");
    S.dt0 = D.num("cycle.dt0", "0.0");
    // mesh and numerics (src/sale2d_back.c:64-247)
    S.npgx = D.integer("processor.npgx", "2");
    S.npgy = D.integer("processor.npgy", "2");
    S.dx = D.num("mesh.dx", "1.");
    S.dy = D.num("mesh.dy", "1.");
    S.oy = D.num("mesh.oy", "0.7");
    S.ox = D.num("mesh.ox", "0.0");
    S.nx = D.integer("mesh.npx", "32");
    S.ny = D.integer("mesh.npy", "32");
    if (lower(D.str("mesh.ext", "off")) != "off") {
        S.x_ext = D.num_k("mesh.ex", 0, "1.05");
        S.nx_ext[0] = D.integer_k("mesh.ex", 1, "0");
        S.nx_ext[1] = D.integer_k("mesh.ex", 2, "0");
        S.y_ext = D.num_k("mesh.ey", 0, "1.05");
        S.ny_ext[0] = D.integer_k("mesh.ey", 1, "0");
        S.ny_ext[1] = D.integer_k("mesh.ey", 2, "0");
    }
    S.avis2 = D.num("numerical.AVISQ", "1.2");
    S.avis1 = D.num("numerical.AVISL", "0.5");
    S.anc = D.num("numerical.ANC", "0.1");
    S.anc_depth = D.num("numerical.ANCD", "2.");
    S.anc_width = D.num("numerical.ANCW", "3.");
    S.anc_pattern = D.str("numerical.ANCPAT", "pml");
    S.ejecta_threshold = D.num("ejecta.threshold", "2.");
    S.ejecta_resistance = D.num("ejecta.resistance", "-1.0");
    S.ejecta_friction = D.num("ejecta.friction", "0.0");
    S.density_cutoff = D.num("numerical.MinDensity", "1.0e-2");
    S.velocity_max = D.num("numerical.MaxVelocity", "-1.63");
    S.velocity_min = D.num("numerical.MinVelocity", "-1e-8");
    S.acceleration_min = D.num("numerical.MinAcceleration", "-1e-3");
    S.partpres = D.integer("numerical.partpres", "0");
    std::string damp = lower(D.str("numerical.damping", "off"));
    S.damp_x = D.integer("numerical.DampX", "0");
    S.damp_y = D.integer("numerical.DampY", "0");
    S.lambda_x = D.num("numerical.LambdaX", "10");
    S.lambda_y = D.num("numerical.LambdaY", "10");
    S.damp_t = D.num("numerical.damp_time", "-1.0");
    if (S.damp_t < 0.) S.damp_t = D.num("cycle.time1", "100.0");
    S.damp_x_left = D.integer("numerical.DampX_Left", "0");
    S.damp_y_top = D.integer("numerical.DampY_Right", "0");
    if (damp == "on" || damp == "pml") S.damp_type = 0;
    else if (damp == "pml2") S.damp_type = 1;
    else if (damp == "pml3") S.damp_type = 2;
    else if (damp == "sbc") {
        S.damp_type = 3;
        S.lambda_x = wind(S.lambda_x, 0.0, 0.5);
        S.lambda_y = wind(S.lambda_y, 0.0, 0.5);
    } else if (damp == "ctlg" || damp == "rock") S.damp_type = 4;
    else {
        S.damp_type = 5;
        S.damp_x = S.damp_y = 0;
        S.lambda_x = S.lambda_y = 0.;
        S.damp_t = -1.0;
        S.damp_x_left = S.damp_y_top = 0;
    }
    S.nmat = D.integer("material.nm", "2");
    if (S.nmat < 2 || S.nmat > SALEC_MAXMAT) { err = "material.nm must be in [2, 10]"; return false; }
    S.gravity[1] = D.num_k("condition.gravity", 1, "-1.62");
    S.gravity[0] = D.num_k("condition.gravity", 0, "0.0");
    std::string gb[4] = {D.str("boundary.left", "freeslip"), D.str("boundary.right", "outflow"),
                         D.str("boundary.bottom", "freeslip"), D.str("boundary.top", "outflow")};
    for (int k = 0; k < 4; ++k) {
        std::string b = lower(gb[k]);
        if (b == "outflow") S.go[k] = 0;          // ght_outflow
        else if (b == "fixed") S.go[k] = 2;       // ght_fixed
        else if (b == "freeslip") S.go[k] = (k < 2) ? 9 : 7;   // reverse_vel_x / reverse_vel_y
        else S.go[k] = 3;                         // ght_zero
    }
    if (S.ox < 1e-6) S.go[0] = 5;                 // ght_mirror on the axis
    S.tracer_strip = D.integer("numerical.tarcer_strip", "2");
    S.tensile_failure = D.integer("numerical.tensile_failure", "0");
    S.tracer_lubrication = D.integer("tracer.lubrication", "0");
    S.tracer_lub_y0 = D.num("tracer.lub_y0", "0.");
    S.tracer_lub_frac = D.num("tracer.lub_frac", "0.");

    // materials (src/sale2d_back.c:250-402)
    S.mats.assign(S.nmat, Mat());
    for (int m = 1; m < S.nmat; ++m) {
        salec_material_desc &r = S.mats[m].d;
        double nu = D.num_k("material.poisson", m, "0.25");
        r.GaCoef = 1.5 * (1.0 - 2.0 * nu) / (1.0 + nu);
        r.Yint0 = D.num_k("material.yint0", m, "1.0");
        r.Yfricint = D.num_k("material.yintfri", m, "1.0");
        r.Ylimint = D.num_k("material.yintlim", m, "2.50e9");
        r.Ydam0 = D.num_k("material.ydam0", m, "1.0");
        r.Yfricdam = D.num_k("material.ydamfri", m, "1.0");
        r.Ylimdam = D.num_k("material.ydamlim", m, "2.50e9");
        S.mats[m].yfunc = D.str_k("material.yshear", m, "SimpleRock");
        r.Yten0 = D.num_k("material.yten0", m, "3.0e8");
        S.mats[m].tfunc = D.str_k("material.ytens", m, "SimpleTensile");
        r.IvanA = D.num_k("material.IvanA", m, "1.0e-4");
        r.IvanB = D.num_k("material.IvanB", m, "1.0e-11");
        r.IvanC = D.num_k("material.IvanC", m, "3.0e8");
        r.Pbd = D.num_k("material.Pbd", m, "2.7e9");
        r.Pbp = D.num_k("material.Pbp", m, "4.1e9");
        S.mats[m].dsdf = D.str_k("material.damage", m, "SimpleShear");
        r.JCA = D.num_k("material.JcA", m, "4.90e7");
        r.JCB = D.num_k("material.JcB", m, "1.57e8");
        r.JCN = D.num_k("material.JcN", m, "1.67e-1");
        r.JCC = D.num_k("material.JcC", m, "1.60e-2");
        r.JCM = D.num_k("material.JcM", m, "1.70");
        r.JCTREF = D.num_k("material.JcTref", m, "8.00e2");
        double jcminp = D.num_k("material.JcminP", m, "-2.44e9");
        r.JCMaxPlastic = D.num_k("material.JCMaxPlastic", m, "10.0");
        const std::string &yf = S.mats[m].yfunc;
        std::string ylow = lower(yf);
        if (ylow == "johnsoncook2" || ylow == "johnsoncook1" || ylow == "vonmises1" || ylow == "vonmises2") {
            r.minPdam = jcminp;
            r.minPint = jcminp;
        } else if (yf.find("Rock") != std::string::npos || ylow == "icestrength") {
            r.minPint = r.Yint0 / r.Yfricint * (r.Yint0 / r.Ylimint - 1.0);
            r.minPdam = -1.0 * r.Ydam0 / r.Yfricdam;
        } else {
            r.minPdam = 0.;
            r.minPint = 0.;
        }
        r.Asimon = 1.0 / D.num_k("material.SimonA", m, "6.00e9");
        r.Csimon = 1.0 / D.num_k("material.SimonC", m, "3.00");
        r.Tmelt0 = D.num_k("material.SimonT0", m, "933.0");
        r.Tfrac = D.num_k("material.OhnakaXi", m, "1.2");
        r.Tdelta = D.num_k("material.Tdelta", m, "0.0");
        r.PolyLiq = D.integer_k("material.PolyLiq", m, "0");
        r.Tlidc1 = D.num_k("material.Tlidc1", m, "0.0");
        r.Tlidc2 = D.num_k("material.Tlidc2", m, "0.0");
        r.Tlidc3 = D.num_k("material.Tlidc3", m, "0.0");
        r.PolySol = D.integer_k("material.PolySol", m, "0");
        r.Tsolc1 = D.num_k("material.Tsolc1", m, "0.0");
        r.Tsolc2 = D.num_k("material.Tsolc2", m, "0.0");
        r.Tsolc3 = D.num_k("material.Tsolc3", m, "0.0");
        double block = D.num_k("material.BlockSize", m, "-1.0");
        if (block < 0.) block = D.num("projectile.radiu", "1.0");
        double geta = D.num_k("material.GammaEta", m, "8.0e-3");
        double gbeta = D.num_k("material.GammaBeta", m, "1.15e2");
        r.Toff = D.num_k("material.Toff", m, "16.0");
        r.Cvib = D.num_k("material.Cvib", m, "0.1");
        r.VibMax = D.num_k("material.VibMax", m, "200.0");
        r.Pvlim = D.num_k("material.Pvlim", m, "2.50e10");
        r.Acvis = geta * block * 5000.0;
        r.Tdamp = gbeta * block / 5000.0;
        r.melt_viscosity = D.num_k("material.viscosityM", m, "0.0");
        S.mats[m].porfunc = D.str_k("material.Porosity", m, "None");
        std::string pl = lower(S.mats[m].porfunc);
        if (pl == "wunnemann") {
            r.alpha0 = D.num_k("material.alpha0", m, "1.0");
            r.alphax = D.num_k("material.alphax", m, "1.0");
            r.epse0 = D.num_k("material.epse0", m, "-1.0e-5");
            r.kappa = D.num_k("material.kappa", m, "0.98");
            r.chi = D.num_k("material.chi", m, "1.0");
            r.avel = D.num_k("material.avel", m, "1e-4");
            r.alphamax = r.alpha0;
            r.epsex = r.epse0 + log(r.alphax / r.alpha0) / r.kappa;
            r.epsec = r.epsex + 2.0 * (1.0 - r.alphax) / (r.kappa * r.alphax);
            if (r.epsex < r.epsec) r.epsec = r.epsex;
            r.alphae = r.alpha0 * (1.0 + (1.0 - r.chi * r.chi) * r.epse0);
            r.alphamax2 = r.alpha0;
        } else if (pl == "none") {
            r.alpha0 = 1.0; r.epse0 = 0.; r.kappa = 0.; r.chi = 0.; r.alphax = 1.0; r.alphamax = 1.0;
            // the reference leaves alphamax2 unset for non-porous materials; 1 keeps the
            // distension clamp of porous runs at its non-porous value
            r.alphamax2 = 1.0;
        } else {
            err = "undefined porosity model " + S.mats[m].porfunc;
            return false;
        }
        for (const std::string *fn : {&S.mats[m].yfunc, &S.mats[m].tfunc, &S.mats[m].dsdf, &S.mats[m].porfunc}) {
            int id = func_of(*fn);
            if (id <= 0) {
                // str2func rejects unknown names and index 0 (SimpleRock), src/strength.c:577-599
                err = "undefined function " + *fn + " (the reference exits on it)";
                return false;
            }
        }
        r.yfunc = func_of(S.mats[m].yfunc);
        r.tfunc = func_of(S.mats[m].tfunc);
        r.dsdf = func_of(S.mats[m].dsdf);
        r.porfunc = func_of(S.mats[m].porfunc);
    }

    // target (src/target_profile.c:345-484)
    TargetInfo &T = S.tinfo;
    T.n_layer = D.integer("target.number", "1");
    std::string ttype = lower(D.str("target.type", "plane"));
    if (ttype == "plane") T.sphere = 0;
    else if (ttype == "sphere") {
        T.sphere = 1;
        T.r_planet = D.num("target.r_planet", "1738.0e3");
        T.center[1] = -T.r_planet;
        T.center[0] = 0.0;
    } else { err = "unknown target type " + ttype; return false; }
    std::vector<std::string> names(S.nmat);
    for (int m = 0; m < S.nmat; ++m) names[m] = D.str_k("material.name", m, "vacuum_");
    auto mat_id = [&](const std::string &n) {
        for (int m = 0; m < S.nmat; ++m)
            if (lower(names[m]) == lower(n)) return m;
        return -1;
    };
    if (T.n_layer < 1 || T.n_layer > 10) { err = "target.number must be in [1, 10]"; return false; }
    for (int l = 0; l < T.n_layer; ++l) {
        T.depth[l] = D.num_k("target.depth", l, "1.");
        T.material[l] = mat_id(D.str_k("target.material", l, "unknown"));
        if (T.material[l] < 0) { err = "unknown target layer material"; return false; }
    }
    T.max_depth = D.num("target.max_depth", "1.");
    if (T.sphere) T.max_depth = T.r_planet;
    std::string tem = lower(D.str_k("target.temperature", 0, "const"));
    T.surf_pre = D.num("target.surf_pressure", "1.0e-5");
    if (tem == "const" || tem == "surface" || tem == "conductive") {
        T.tem_type = tem == "conductive" ? 1 : 0;
        T.surf_tem = tem == "surface" ? -1.0 : D.num("target.surf_temperature", "-1.0");
        if (T.surf_tem < 0.) T.surf_tem = D.num_k("target.temperature", 1, "293.0");
        if (T.tem_type == 1) T.surf_dtdz = D.num("target.surf_dtdz", "0.0");
        if (T.tem_type == 1 && !T.sphere) T.r_planet = D.num("target.r_planet", "0.0");
    } else {
        err = "target temperature profile '" + tem + "' is not supported by the deck initialiser";
        return false;
    }

    // projectile (src/sale2d_back.c:29-62)
    S.p_mat = mat_id(D.str("projectile.material", "unknown"));
    if (S.p_mat < 0) { err = "cannot get material id of the projectile"; return false; }
    S.p_radius = D.num("projectile.radiu", "1.0");
    S.p_center[0] = D.num_k("projectile.center", 0, "0.0");
    S.p_center[1] = D.num_k("projectile.center", 1, "300.0");
    S.p_vel[0] = D.num_k("projectile.velocity", 0, "0.0");
    S.p_vel[1] = D.num_k("projectile.velocity", 1, "-1000.0");
    S.p_dam = D.num_k("projectile.damage", 1, "1.0");
    S.p_pre = D.num_k("projectile.pressure", 1, "1.0");
    S.p_tem = D.num_k("projectile.temperature", 1, "293.0");

    // additions (src/target_profile.c:486-570)
    int nobj = D.integer("addition.nobject", "0");
    for (int k = 0; k < nobj; ++k) {
        Addition a;
        a.material = mat_id(D.str_k("addition.material", k, "unknown"));
        if (a.material < 0) { err = "unknown addition material"; return false; }
        std::string ty = lower(D.str_k("addition.type", k, "unknown"));
        std::string par = "addition." + D.str_k("addition.parameter", k, "unknown");
        if (!D.has(par)) { err = "cannot find parameter " + par; return false; }
        if (ty == "cube") { a.type = 1; for (int j = 0; j < 12; ++j) a.par[j] = D.num_k(par, j, "-1"); }
        else if (ty == "sphere") { a.type = 0; for (int j = 0; j < 9; ++j) a.par[j] = D.num_k(par, j, "-1"); }
        else { err = "unknown addition type " + ty; return false; }
        S.additions.push_back(a);
    }
    if (!load_tables(S, eosdir, D, err)) return false;
    // init_sale_mat flags (src/sale2d.c:496-513)
    for (int m = 1; m < S.nmat; ++m) {
        if (S.mats[m].d.Toff > 0.0) S.acoustic_fluid = 1;
        if (lower(S.mats[m].porfunc) != "none") S.porosity_model++;
        S.mats[m].d.eos_type = S.mats[m].kind;
    }
    return true;
}

// ---------------------------------------------------------------- grid spacing
double Sk(int k, double ext) { return ext * (pow(ext, k) - 1.0) / (ext - 1.0); }

double spacing2(int k, double ext, int eL, int eR, int dL, int dR, int N)
{
    // Spacing2 (src/construct.c:396-412)
    double Xk = 0.;
    if (k < dL) Xk = pow(ext, eL) * k;
    else if (k < dL + eL) Xk = Sk(eL, ext) - Sk(dL + eL - k, ext) + pow(ext, eL) * dL;
    else if (k < N - (dR + eR)) Xk = Sk(eL, ext) + pow(ext, eL) * dL + (k - (dL + eL));
    else if (k < N - dR) Xk = Sk(eL, ext) + pow(ext, eL) * dL + (N - (dL + eL) - (dR + eR)) + Sk(k - (N - dR - eR), ext);
    else Xk = Sk(eL, ext) + pow(ext, eL) * dL + (N - (dL + eL) - (dR + eR)) + Sk(eR, ext) + pow(ext, eR) * (k - (N - dR));
    return Xk;
}

double hanning(double x) { return 0.5 * (1.0 - cos(2.0 * M_PI * x)); }

// ---------------------------------------------------------------- element quadratures
const double kBETA = 0.57735026918962576451;
const double kGP[4][2] = {{-kBETA, -kBETA}, {-kBETA, kBETA}, {kBETA, -kBETA}, {kBETA, kBETA}};

double interp4(const double *v, const double *xl)
{
    double r = 0;
    for (int k = 0; k < 4; ++k) r += ipb(k, xl[0], xl[1]) * v[k];
    return r;
}

double jacobi4(const double *X, const double *xl)
{
    // X: 4 corners (x, y) interleaved
    double J[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; ++k) J[0] += ipb_d(k, 0, xl[0], xl[1]) * X[2 * k];
    for (int k = 0; k < 4; ++k) J[1] += ipb_d(k, 1, xl[0], xl[1]) * X[2 * k];
    for (int k = 0; k < 4; ++k) J[2] += ipb_d(k, 0, xl[0], xl[1]) * X[2 * k + 1];
    for (int k = 0; k < 4; ++k) J[3] += ipb_d(k, 1, xl[0], xl[1]) * X[2 * k + 1];
    return J[0] * J[3] - J[1] * J[2];
}

double integrate(const double *X, const double *Y)
{
    double r = 0;
    for (int j = 0; j < 4; ++j) r += 1.0 * interp4(Y, kGP[j]) * jacobi4(X, kGP[j]);
    return r;
}

double integrate_cyl(const double *X, const double *Y)
{
    double r = 0;
    for (int j = 0; j < 4; ++j) {
        const double xs[4] = {X[0], X[2], X[4], X[6]};
        double lr = fabs(interp4(xs, kGP[j]));
        r += 1.0 * interp4(Y, kGP[j]) * jacobi4(X, kGP[j]) * lr;
    }
    return r;
}

double integrate_cyl_fdx(const double *X, const double *F, int dim)
{
    double lf[8];
    memcpy(lf, X, sizeof(lf));
    for (int k = 0; k < 4; ++k) lf[2 * k + dim] = F[k];
    double r = 0;
    for (int j = 0; j < 4; ++j) {
        const double xs[4] = {X[0], X[2], X[4], X[6]};
        double lr = interp4(xs, kGP[j]);
        r += 1.0 * jacobi4(lf, kGP[j]) * fabs(lr);
    }
    return r;
}

void cross_line(const double *a, const double *b, double *s)
{
    double r0 = (b[0] + a[0]) / 2.0;
    r0 = fabs(r0);
    s[0] = -1.0 * (b[1] - a[1]) * r0;
    s[1] = (b[0] - a[0]) * r0;
}

// generate2dcyl_suf_and_vol, generate2dcyl_grad, generate2d_center (src/construct.c:480-582)
void cell_geometry(const double *pos, double *suf, double *subvol, double *vol, double *grad, double *center)
{
    static const double lxl[4][4][2] = {{{-1.0, -1.0}, {0.0, -1.0}, {0.0, 0.0}, {-1.0, 0.0}},
                                        {{0.0, -1.0}, {1.0, -1.0}, {1.0, 0.0}, {0.0, 0.0}},
                                        {{0.0, 0.0}, {1.0, 0.0}, {1.0, 1.0}, {0.0, 1.0}},
                                        {{-1.0, 0.0}, {0.0, 0.0}, {0.0, 1.0}, {-1.0, 1.0}}};
    const double ones[4] = {1., 1., 1., 1.};
    const double xs[4] = {pos[0], pos[2], pos[4], pos[6]}, ys[4] = {pos[1], pos[3], pos[5], pos[7]};
    double sv[4], rv[4];
    const double sign_er = pos[0] + pos[2] + pos[4] + pos[6];
    for (int k = 0; k < 4; ++k) {
        double g[8];
        for (int j = 0; j < 4; ++j) { g[2 * j] = interp4(xs, lxl[k][j]); g[2 * j + 1] = interp4(ys, lxl[k][j]); }
        rv[k] = integrate_cyl(g, ones);
        sv[k] = integrate(g, ones);
        if (sign_er < 0.0) sv[k] *= -1.0;
        // rotate the sub-quadrilateral k+1 times, then the surface of its first two edges
        for (int r = 0; r < k + 1; ++r) {
            double t[8];
            for (int q = 0; q < 4; ++q) { t[2 * q] = g[2 * ((q + 1) % 4)]; t[2 * q + 1] = g[2 * ((q + 1) % 4) + 1]; }
            memcpy(g, t, sizeof(t));
        }
        double p[2] = {0., 0.}, tl[2];
        for (int q = 1; q < 3; ++q) {
            cross_line(g + 2 * (q - 1), g + 2 * q, tl);
            p[0] += 1.0 * tl[0];
            p[1] += 1.0 * tl[1];
        }
        suf[2 * k] = p[0];
        suf[2 * k + 1] = p[1];
    }
    for (int k = 0; k < 4; ++k) rv[k] = fabs(rv[k]);
    vol[0] = fabs(rv[0]) + fabs(rv[1]) + fabs(rv[2]) + fabs(rv[3]);
    for (int k = 0; k < 4; ++k) { subvol[k] = sv[k]; subvol[4 + k] = rv[k]; }
    const double tv = integrate_cyl(pos, ones);
    for (int j = 0; j < 4; ++j) {
        double e[4] = {0, 0, 0, 0};
        e[j] = 1.;
        for (int k = 0; k < 2; ++k) grad[4 * k + j] = integrate_cyl_fdx(pos, e, k);
    }
    for (int j = 0; j < 4; ++j) {
        double e[4] = {0, 0, 0, 0};
        e[j] = 1.;
        grad[8 + j] = integrate(pos, e);
        if (sign_er < 0.) grad[8 + j] *= -1.0;
    }
    const double s = 1.0 / tv;
    for (int k = 0; k < 12; ++k) grad[k] *= s;
    for (int k = 0; k < 4; ++k) center[k] = 0.;
    for (int k = 0; k < 4; ++k) { center[0] += 0.25 * pos[2 * k]; center[1] += 0.25 * pos[2 * k + 1]; }
    for (int k = 0; k < 4; ++k)
        for (int j = 0; j < 4; ++j) {
            center[2] = dmax(fabs(pos[2 * k] - pos[2 * j]), center[2]);
            center[3] = dmax(fabs(pos[2 * k + 1] - pos[2 * j + 1]), center[3]);
        }
}

// ---------------------------------------------------------------- nine-point Laplacian
// Laplace2d9 of src/geometry/interpolate_2d9.c:398-424 over a biquadratic nine-node element.
const double kXL9[9][2] = {{-1., -1.}, {0., -1.}, {1., -1.}, {-1., 0.}, {0., 0.}, {1., 0.}, {-1., 1.}, {0., 1.}, {1., 1.}};
const int kXLI9[9][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {3, 4, 5}, {4, 5, 3}, {5, 3, 4}, {6, 7, 8}, {7, 8, 6}, {8, 6, 7}};
const int kXLJ9[9][3] = {{0, 3, 6}, {1, 4, 7}, {2, 5, 8}, {3, 0, 6}, {4, 7, 1}, {5, 8, 2}, {6, 0, 3}, {7, 1, 4}, {8, 2, 5}};
inline double lag(double x, double x0, double x1) { return (x - x1) / (x0 - x1); }
inline double lag_x(double, double x0, double x1) { return 1.0 / (x0 - x1); }

// derivatives of shape function k: d = 0 value, 1 d/dxi, 2 d/deta, 3 d2/dxi2, 4 d2/dxideta, 5 d2/deta2
double shape9(int k, int d, const double *x)
{
    const double xi = x[0], eta = x[1];
    const int i0 = kXLI9[k][0], i1 = kXLI9[k][1], i2 = kXLI9[k][2];
    const int j0 = kXLJ9[k][0], j1 = kXLJ9[k][1], j2 = kXLJ9[k][2];
    const double a0 = kXL9[i0][0], a1 = kXL9[i1][0], a2 = kXL9[i2][0];
    const double b0 = kXL9[j0][1], b1 = kXL9[j1][1], b2 = kXL9[j2][1];
    switch (d) {
    case 0: {
        double xf = lag(xi, a0, a1) * lag(xi, a0, a2);
        double yf = lag(eta, b0, b1) * lag(eta, b0, b2);
        return xf * yf;
    }
    case 1: {
        double xf_x = lag_x(xi, a0, a1) * lag(xi, a0, a2) + lag(xi, a0, a1) * lag_x(xi, a0, a2);
        double yf = lag(eta, b0, b1) * lag(eta, b0, b2);
        return xf_x * yf;
    }
    case 2: {
        double xf = lag(xi, a0, a1) * lag(xi, a0, a2);
        double yf_x = lag_x(eta, b0, b1) * lag(eta, b0, b2) + lag(eta, b0, b1) * lag_x(eta, b0, b2);
        return xf * yf_x;
    }
    default: {
        double x2f_xx = 2.0 * lag_x(eta, b0, b1) * lag_x(eta, b0, b2);
        double x1f_xx = 2.0 * lag_x(xi, a0, a1) * lag_x(xi, a0, a2);
        double x1f_x = lag_x(xi, a0, a1) * lag(xi, a0, a2) + lag(xi, a0, a1) * lag_x(xi, a0, a2);
        double x2f_x = lag_x(eta, b0, b1) * lag(eta, b0, b2) + lag(eta, b0, b1) * lag_x(eta, b0, b2);
        double x2f = lag(eta, b0, b1) * lag(eta, b0, b2);
        double x1f = lag(xi, a0, a1) * lag(xi, a0, a2);
        if (d == 3) return x1f_xx * x2f;
        if (d == 5) return x1f * x2f_xx;
        return x1f_x * x2f_x;
    }
    }
}

// Shape-function values at the nine (gamma-scaled) Gauss points depend on nothing else, so
// they are tabulated once; the products below use them exactly as evaluated on the fly.
struct Shape9Table {
    double gamma = -1.0;
    double w[9];
    double v[9][9][6];   // [gauss point][node][derivative]
};

const Shape9Table &shape9_table(double gamma)
{
    static Shape9Table t;
    static std::once_flag once;
    std::call_once(once, [&] {
        const double s35 = 0.77459666924148337703585307995648;
        const double gp[9][2] = {{-s35, -s35}, {-s35, 0.}, {-s35, s35}, {0., -s35}, {0., 0.}, {0., s35},
                                 {s35, -s35}, {s35, 0.}, {s35, s35}};
        const double gw[9] = {(5.0 / 9.0) * (5.0 / 9.0), (5.0 / 9.0) * (8.0 / 9.0), (5.0 / 9.0) * (5.0 / 9.0),
                              (8.0 / 9.0) * (5.0 / 9.0), (8.0 / 9.0) * (8.0 / 9.0), (8.0 / 9.0) * (5.0 / 9.0),
                              (5.0 / 9.0) * (5.0 / 9.0), (5.0 / 9.0) * (8.0 / 9.0), (5.0 / 9.0) * (5.0 / 9.0)};
        t.gamma = gamma;
        for (int g = 0; g < 9; ++g) {
            t.w[g] = gw[g];
            const double xl[2] = {gp[g][0] * gamma, gp[g][1] * gamma};
            for (int k = 0; k < 9; ++k)
                for (int d = 0; d < 6; ++d) t.v[g][k][d] = shape9(k, d, xl);
        }
    });
    return t;
}

double laplace9(const double *X, const double *Y, double gamma)
{
    const Shape9Table &T = shape9_table(gamma);
    double val = 0., area = 0.;
    for (int g = 0; g < 9; ++g) {
        double J[4] = {0., 0., 0., 0.};
        for (int k = 0; k < 9; ++k) J[0] += T.v[g][k][1] * X[2 * k];
        for (int k = 0; k < 9; ++k) J[1] += T.v[g][k][2] * X[2 * k];
        for (int k = 0; k < 9; ++k) J[2] += T.v[g][k][1] * X[2 * k + 1];
        for (int k = 0; k < 9; ++k) J[3] += T.v[g][k][2] * X[2 * k + 1];
        const double det = J[0] * J[3] - J[1] * J[2];
        double inv[4];
        inv[0] = J[3] / det;
        inv[3] = J[0] / det;
        inv[1] = -J[2] / det;
        inv[2] = -J[1] / det;
        double y11 = 0., y12 = 0., y22 = 0.;
        for (int q = 0; q < 9; ++q) y11 += T.v[g][q][3] * Y[q];
        for (int q = 0; q < 9; ++q) y12 += T.v[g][q][4] * Y[q];
        for (int q = 0; q < 9; ++q) y22 += T.v[g][q][5] * Y[q];
        const double dxx = y11 * inv[0] * inv[0] + 2.0 * y12 * inv[0] * inv[2] + y22 * inv[2] * inv[2];
        const double dyy = y11 * inv[1] * inv[1] + 2.0 * y12 * inv[1] * inv[3] + y22 * inv[3] * inv[3];
        val += (gamma * gamma) * T.w[g] * (dxx + dyy) * det;
        area += (gamma * gamma) * T.w[g] * 1.0 * det;
    }
    return val / area;
}

void parallel_rows(int n, const std::function<void(int, int)> &fn)
{
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 64) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t) {
        int a = (int)((long long)n * t / nt), b = (int)((long long)n * (t + 1) / nt);
        th.emplace_back(fn, a, b);
    }
    for (auto &x : th) x.join();
}

} // namespace

// ================================================================== build the state
// Host arrays in the reference's layout (x-fastest points, components innermost).
struct HostState {
    int enx, eny, vnx, vny, nmat;
    std::map<std::string, std::vector<double>> f;
    std::vector<double> &get(const std::string &n, size_t size)
    {
        auto &v = f[n];
        if (v.size() != size) v.assign(size, 0.0);
        return v;
    }
};

int build_host_state(const Setup &S0, Setup &S, HostState &H, std::vector<double> &tracer_rows, std::string &err)
{
    S = S0;
    const int pad = 2;
    const int nx = S.npgx * S.nx, ny = S.npgy * S.ny;   // one domain for the whole process grid
    H.enx = nx + 2 * pad; H.eny = ny + 2 * pad; H.vnx = nx + 2 * pad + 1; H.vny = ny + 2 * pad + 1;
    H.nmat = S.nmat;
    const int enx = H.enx, eny = H.eny, vnx = H.vnx, vny = H.vny, nmat = S.nmat;
    const size_t NE = (size_t)enx * eny, NV = (size_t)vnx * vny;

    // ---------------- vertex positions (src/construct.c:11-80)
    const int ncy = ny + 2 * pad, ncx = nx + 2 * pad;
    const int YeL = S.ny_ext[0], YeR = S.ny_ext[1], XeL = S.nx_ext[0], XeR = S.nx_ext[1];
    const double Yext = S.y_ext, Xext = S.x_ext;
    const int XdR = S.damp_x, XdL = S.damp_x_left, YdL = S.damp_y, YdR = S.damp_y_top;
    auto SY = [&](int k) { return spacing2(k, Yext, YeL, YeR, YdL, YdR, ncy); };
    auto SX = [&](int k) { return spacing2(k, Xext, XeL, XeR, XdL, XdR, ncx); };
    const double Ly = SY(ny + pad) - SY(pad);
    int y0i;
    for (y0i = 0; y0i < ncy + 1; ++y0i)
        if (SY(y0i + pad) >= Ly * S.oy) break;
    const double y0 = -SY(y0i + pad) * S.dy;
    const double Lx = SX(nx + pad) - SX(pad);
    int x0i;
    for (x0i = 0; x0i < ncx + 1; ++x0i)
        if (SX(x0i) >= Lx * S.ox) break;
    const double x0 = -SX(x0i + pad) * S.dx;
    // rows of the lubricating tracer layer: from tracer.lubrication cells below the surface up to
    // the surface (src/construct.c:75-91)
    if (S.tracer_lubrication >= 1) {
        S.tracer_lub_gy0 = 0;
        S.tracer_lub_gy1 = ncy;
        int j = 0;
        for (; j < ncy + 1; ++j) {
            const double tmpy = SY(j) * S.dy + y0;
            S.tracer_lub_gy0 = j;
            if (tmpy >= S.tracer_lubrication * S.dy * (-1.0)) break;
        }
        for (; j < ncy + 1; ++j) {
            const double tmpy = SY(j) * S.dy + y0;
            S.tracer_lub_gy1 = j;
            if (tmpy >= 0.0) break;
        }
    }
    std::vector<double> &vpos = H.get("v_pos", NV * 2);
    for (int j = 0; j < vny; ++j)
        for (int i = 0; i < vnx; ++i) {
            vpos[2 * ((size_t)i + (size_t)vnx * j)] = SX(i) * S.dx + x0;
            vpos[2 * ((size_t)i + (size_t)vnx * j) + 1] = SY(j) * S.dy + y0;
        }

    // ---------------- cell geometry and damping coefficients (src/construct.c:82-216)
    std::vector<double> &epos = H.get("e_pos", NE * 4), &evol = H.get("e_vol", NE), &esuf = H.get("e_suf", NE * 8);
    std::vector<double> &egrad = H.get("e_grad", NE * 12), &esub = H.get("e_subvol", NE * 8);
    std::vector<double> &esig = H.get("e_sigma", NE * 2);
    const double dly = spacing2(S.damp_y, Yext, YeL, YeR, YdL, YdR, ncy) * S.dy;
    const double dlx = spacing2(ncx, Xext, XeL, XeR, XdL, XdR, ncx) * S.dx - spacing2(ncx - S.damp_x, Xext, XeL, XeR, XdL, XdR, ncx) * S.dx;
    const double csd = 5.0e3, pml_b = 2.3;
    parallel_rows(eny, [&](int ja, int jb) {
        for (int j = ja; j < jb; ++j)
            for (int i = 0; i < enx; ++i) {
                const size_t e = (size_t)i + (size_t)enx * j;
                const size_t v[4] = {(size_t)i + (size_t)vnx * j, (size_t)i + 1 + (size_t)vnx * j,
                                     (size_t)i + 1 + (size_t)vnx * (j + 1), (size_t)i + (size_t)vnx * (j + 1)};
                double pos[8];
                for (int k = 0; k < 4; ++k) { pos[2 * k] = vpos[2 * v[k]]; pos[2 * k + 1] = vpos[2 * v[k] + 1]; }
                cell_geometry(pos, &esuf[8 * e], &esub[8 * e], &evol[e], &egrad[12 * e], &epos[4 * e]);
                double *sg = &esig[2 * e];
                const double dy_ = epos[4 * e + 1] - y0;
                const double dx_ = spacing2(ncx, Xext, XeL, XeR, XdL, XdR, ncx) * S.dx - (epos[4 * e] - x0);
                switch (S.damp_type) {
                case 0: case 1: case 2:
                    sg[1] = sg[0] = 0.;
                    if (dy_ <= dly) sg[1] = pow(1.0 - dy_ / dly, 2.0) / (2.0 * dly) * (3.0 * csd) * S.lambda_y;
                    if (dx_ <= dlx) sg[0] = pow(1.0 - dx_ / dlx, 2.0) / (2.0 * dlx) * (3.0 * csd) * S.lambda_x;
                    break;
                case 3:
                    sg[1] = sg[0] = 1.0;
                    if (dy_ <= dly) sg[1] = hanning(0.5 * ((1.0 - S.lambda_y) * dy_ / dly + S.lambda_y));
                    if (dx_ <= dlx) sg[0] = hanning(0.5 * ((1.0 - S.lambda_x) * dx_ / dlx + S.lambda_x));
                    sg[0] = dmin(sg[0], sg[1]);
                    break;
                default:
                    sg[0] = sg[1] = 0.;
                    if (dy_ <= dly) sg[1] = 1.0;
                    if (dx_ <= dlx) sg[0] = 1.0;
                    break;
                }
            }
    });
    if (S.damp_type <= 2) {
        S.alpha_damp_x = (csd * 2.0) / dlx * pml_b;
        S.alpha_damp_y = (csd * 2.0) / dly * pml_b;
    }

    // ---------------- vertex volumes, surfaces, Laplacian (src/construct.c:218-300)
    const std::string anc_pat = lower(S.anc_pattern);
    auto need_laplacian = [&](int i, int j) {
        if (S.tinfo.sphere || anc_pat == "none") return false;
        if (anc_pat == "pml")
            return (S.damp_y >= 1 && j <= 2 * S.damp_y) || (S.damp_x >= 1 && i >= vnx - 2 * S.damp_x);
        return true;
    };
    std::vector<double> &vvol = H.get("v_vol", NV * 5), &vsub = H.get("v_subvol", NV * 4);
    std::vector<double> &vsuf = H.get("v_suf", NV * 8), &vlap = H.get("v_laplace", NV * 9);
    parallel_rows(vny, [&](int ja, int jb) {
        for (int j = ja; j < jb; ++j)
            for (int i = 0; i < vnx; ++i) {
                if (i < 1 || i > vnx - 2 || j < 1 || j > vny - 2) continue;
                const size_t p = (size_t)i + (size_t)vnx * j;
                const size_t c[4] = {(size_t)(i - 1) + (size_t)enx * (j - 1), (size_t)i + (size_t)enx * (j - 1),
                                     (size_t)i + (size_t)enx * j, (size_t)(i - 1) + (size_t)enx * j};
                const int off[4] = {2, 3, 0, 1};
                vvol[5 * p] = 0.;
                for (int k = 0; k < 4; ++k) {
                    vvol[5 * p] += esub[8 * c[k] + 4 + off[k]];
                    vsub[4 * p + k] = esub[8 * c[k] + off[k]];
                    vvol[5 * p + k + 1] = esub[8 * c[k] + off[k] + 4];
                    vsuf[8 * p + 2 * k] = esuf[8 * c[k] + off[k] * 2];
                    vsuf[8 * p + 2 * k + 1] = esuf[8 * c[k] + off[k] * 2 + 1];
                }
                // the weights are tapered to zero outside the ANC band right after this loop,
                // so they are only evaluated where the taper can be non-zero
                if (!need_laplacian(i, j)) continue;
                double X[18];
                int q = 0;
                for (int dj = -1; dj <= 1; ++dj)
                    for (int di = -1; di <= 1; ++di, ++q) {
                        const size_t n = (size_t)(i + di) + (size_t)vnx * (j + dj);
                        X[2 * q] = vpos[2 * n];
                        X[2 * q + 1] = vpos[2 * n + 1];
                    }
                for (int k = 0; k < 9; ++k) {
                    double Y[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                    Y[k] = 1.;
                    vlap[9 * p + k] = laplace9(X, Y, 0.5);
                }
            }
    });

    // ---------------- face normals (src/construct.c:302-357)
    std::vector<double> &bxn = H.get("bx_normal", (size_t)vnx * eny * 2), &byn = H.get("by_normal", (size_t)enx * vny * 2);
    auto norm2 = [](double *x) {
        double len = 0.;
        len += x[0] * x[0];
        len += x[1] * x[1];
        len = sqrt(len);
        for (int k = 0; k < 2; ++k) { x[k] /= len; if (std::isnan(x[k])) x[k] = 1.0; }
    };
    for (int j = 0; j < eny; ++j)
        for (int i = 0; i < vnx; ++i) {
            int xd = std::min(i, vnx - 1 - i), yd = std::min(j, eny - 1 - j);
            if (xd <= 0 || yd <= 0) continue;
            double *n = &bxn[2 * ((size_t)i + (size_t)vnx * j)];
            const double *u = &epos[4 * ((size_t)i + (size_t)enx * j)], *b = &epos[4 * ((size_t)(i - 1) + (size_t)enx * j)];
            n[0] = 1.0 * u[0] + -1.0 * b[0];
            n[1] = 1.0 * u[1] + -1.0 * b[1];
            norm2(n);
        }
    for (int j = 0; j < vny; ++j)
        for (int i = 0; i < enx; ++i) {
            int xd = std::min(i, enx - 1 - i), yd = std::min(j, vny - 1 - j);
            if (xd <= 0 || yd <= 0) continue;
            double *n = &byn[2 * ((size_t)i + (size_t)enx * j)];
            const double *r = &epos[4 * ((size_t)i + (size_t)enx * j)], *l = &epos[4 * ((size_t)i + (size_t)enx * (j - 1))];
            n[0] = 1.0 * r[0] + -1.0 * l[0];
            n[1] = 1.0 * r[1] + -1.0 * l[1];
            norm2(n);
        }

    // ---------------- target profile (src/target_profile.c:86-343, 1161-1195)
    const TargetInfo &T = S.tinfo;
    const double dz = dmin(S.dy * 0.5, T.max_depth / T.n_profile);
    const int n = (int)ceil(T.max_depth / dz);
    std::vector<double> pre(n), rad(n), den(n), tem(n), gra(n), dam(n), eng(n);
    std::vector<int> mat(n);
    {
        int cur = n - 1;
        for (int l = 0; l < T.n_layer; ++l) {
            int iv = (int)floor(T.depth[l] / dz);
            for (int j = 0; j < iv && cur > 0; ++j) mat[cur--] = T.material[l];
        }
        for (; cur >= 0; --cur) mat[cur] = T.material[T.n_layer - 1];
    }
    for (int k = 0; k < n; ++k) {
        pre[k] = T.surf_pre;
        den[k] = S.mats[mat[k]].den0;
        rad[k] = (T.sphere ? T.r_planet : T.max_depth) * k / (n - 1);
    }
    if (T.tem_type == 0) {
        for (int k = 0; k < n; ++k) tem[k] = T.surf_tem;
    } else {
        for (int k = n - 1; k >= 0; --k) {
            double depth = rad[n - 1] - rad[k];
            if (n == k + 1) { tem[k] = T.surf_tem; continue; }
            double g = T.surf_dtdz * (1.0 + depth / T.r_planet);
            tem[k] = tem[k + 1] + (g) * (rad[k + 1] - rad[k]);
        }
    }
    for (int k = 0; k < n; ++k) { gra[k] = S.gravity[1]; dam[k] = 0.; }
    auto integrate_gravity = [&]() {
        if (T.sphere) {
            gra[0] = 0.0;
            for (int k = 1; k < n; ++k)
                gra[k] = gra[k - 1] - 4.0 * M_PI * 6.674e-11 * (den[k] + den[k - 1]) * (rad[k] + rad[k - 1]) *
                                          (rad[k] + rad[k - 1]) / 8.0 * (rad[k] - rad[k - 1]);
            for (int k = 1; k < n; ++k) gra[k] = gra[k] / (rad[k] * rad[k]);
            for (int k = n - 2; k >= 0; --k)
                pre[k] = pre[k + 1] + (den[k] + den[k + 1]) * (gra[k] + gra[k + 1]) * (rad[k] - rad[k + 1]) / 4.0;
        } else {
            for (int k = n - 2; k >= 0; --k) {
                double drg = 0.25 * (den[k + 1] + den[k]) * (gra[k] + gra[k + 1]);
                pre[k] = pre[k + 1] + drg * (rad[k] - rad[k + 1]);
            }
        }
    };
    auto solidus = [&](double p, const salec_material_desc &s) {
        double sol = s.Tmelt0 * pow(s.Asimon * p + 1.0, s.Csimon);
        if (s.PolySol > 0) {
            double pg = p * 1.0e-9;
            sol = s.Tsolc1 + s.Tsolc2 * pg + s.Tsolc3 * pg * pg;
        }
        return sol;
    };
    // The reference runs 2000 fixed-point iterations. Each iteration is a function of the density
    // and temperature it starts from (pressure and gravity are integrated from them first), so once
    // an iteration starts from exactly the bits the previous one started from, every remaining
    // iteration reproduces them: stopping there gives the state of all 2000, bit for bit. The
    // profiles reach that point after a few iterations.
    std::vector<double> last_den, last_tem;
    for (int it = 0; it < 2000; ++it) {
        if (it > 0 && memcmp(last_den.data(), den.data(), sizeof(double) * n) == 0 &&
            memcmp(last_tem.data(), tem.data(), sizeof(double) * n) == 0)
            break;
        last_den = den;
        last_tem = tem;
        integrate_gravity();
        parallel_rows(n, [&](int a, int b) {
            for (int k = a; k < b; ++k) {
                const Mat &M = S.mats[mat[k]];
                const double mt = solidus(pre[k], M.d);
                const double lt = dmin(tem[k], mt);
                const double pt = M.d.alpha0;
                tem[k] = lt;
                eng[k] = eos_interp_tp(M, lt, pre[k] * pt, 0) / pt;
                den[k] = eos_interp_tp(M, lt, pre[k] * pt, -1) / pt;
            }
        });
    }
    integrate_gravity();

    // ---------------- material distribution (src/target_profile.c:588-834, 996-1158)
    std::vector<double> &evof = H.get("m_vof", NE * nmat), &mden = H.get("m_den", NE * nmat), &meng = H.get("m_eng", NE * nmat);
    std::vector<double> &mpty = H.get("m_pty", NE * nmat), &epre = H.get("e_pre", NE), &etem = H.get("e_tem", NE);
    std::vector<double> &edam = H.get("e_dam", NE), &ewpt = H.get("e_wpt", NE * 4), &evel = H.get("e_vel", NE * 2);
    std::vector<double> &ecvs = H.get("e_cvs", NE);
    H.get("e_tps", NE);
    H.get("e_vib", NE);
    const Mat &PM = S.mats[S.p_mat];
    const double ppty = PM.d.alpha0;
    const double p_den = eos_interp_tp(PM, S.p_tem, S.p_pre * ppty, -1) / ppty;
    const double p_eng = eos_interp_tp(PM, S.p_tem, S.p_pre * ppty, 0) / ppty;
    for (size_t e = 0; e < NE; ++e) {
        const double *ep = &epos[4 * e];
        double *vf = &evof[nmat * e], *md = &mden[nmat * e], *me = &meng[nmat * e], *mp = &mpty[nmat * e];
        evel[2 * e] = evel[2 * e + 1] = 0.;
        for (int m = 0; m < nmat; ++m) mp[m] = 1.0;
        ecvs[e] = 0.;
        double d2 = 0.;
        d2 += (ep[0] - S.p_center[0]) * (ep[0] - S.p_center[0]);
        d2 += (ep[1] - S.p_center[1]) * (ep[1] - S.p_center[1]);
        const double pdis = sqrt(d2);
        double pl = 0.;
        if (T.sphere) {
            double q = 0.;
            q += (ep[0] - T.center[0]) * (ep[0] - T.center[0]);
            q += (ep[1] - T.center[1]) * (ep[1] - T.center[1]);
            pl = sqrt(q);
        }
        if (pdis <= S.p_radius) {
            for (int m = 0; m < nmat; ++m) { vf[m] = 0.; md[m] = 0.; me[m] = 0.; }
            vf[S.p_mat] = 1.0;
            epre[e] = S.p_pre; etem[e] = S.p_tem; edam[e] = S.p_dam;
            md[S.p_mat] = p_den;
            me[S.p_mat] = p_eng;
            evel[2 * e] = S.p_vel[0];
            evel[2 * e + 1] = S.p_vel[1];
            for (int k = 0; k < 4; ++k) ewpt[4 * e + k] = -0.25;
            mp[S.p_mat] = ppty;
        } else if ((!T.sphere && ep[1] <= 0.) || (T.sphere && pl <= T.r_planet)) {
            int li;
            if (!T.sphere) {
                li = (int)floor(fabs(ep[1]) / T.max_depth * (n - 1)) + 1;
                li = n - 1 - li;
            } else {
                li = (int)floor(pl / dz);
            }
            li = std::min(li, n - 1);
            li = std::max(li, 0);
            const int lid = mat[li];
            for (int m = 0; m < nmat; ++m) { vf[m] = 0.; md[m] = 0.; me[m] = 0.; }
            epre[e] = pre[li]; etem[e] = tem[li]; edam[e] = dam[li];
            vf[lid] = 1.0;
            md[lid] = den[li];
            me[lid] = eng[li];
            mp[lid] = S.mats[lid].d.alpha0;
            for (int k = 0; k < 4; ++k) ewpt[4 * e + k] = -0.25;
        } else {
            for (int m = 0; m < nmat; ++m) vf[m] = 0.;
            vf[0] = 1.0;
            for (int k = 0; k < 4; ++k) ewpt[4 * e + k] = 1.0;
        }
        for (const Addition &a : S.additions) {
            double tm, pr, dm, pt, v0, v1;
            if (a.type == 1) {
                const double lbp[2] = {a.par[0], a.par[1]}, xa[2] = {a.par[2], a.par[3]}, ya[2] = {a.par[4], a.par[5]};
                v0 = a.par[6]; v1 = a.par[7]; tm = a.par[8]; pr = a.par[9]; dm = a.par[10]; pt = a.par[11];
                const double xx[2] = {1.0 * ep[0] + -1.0 * lbp[0], 1.0 * ep[1] + -1.0 * lbp[1]};
                double lxa = sqrt(0. + xa[0] * xa[0] + xa[1] * xa[1]);
                double lya = sqrt(0. + ya[0] * ya[0] + ya[1] * ya[1]);
                double xl = (0. + xx[0] * xa[0] + xx[1] * xa[1]) / lxa / lxa;
                double yl = (0. + xx[0] * ya[0] + xx[1] * ya[1]) / lya / lya;
                if (xl * (1 - xl) < 0 || yl * (1 - yl) < 0) continue;
            } else {
                v0 = a.par[3]; v1 = a.par[4]; tm = a.par[5]; pr = a.par[6]; dm = a.par[7]; pt = a.par[8];
                double q = 0.;
                q += (a.par[0] - ep[0]) * (a.par[0] - ep[0]);
                q += (a.par[1] - ep[1]) * (a.par[1] - ep[1]);
                if (sqrt(q) > a.par[2]) continue;
            }
            tm = tm >= 0 ? tm : etem[e];
            pr = pr >= 0 ? pr : epre[e];
            pt = pt >= 0 ? pt : mp[a.material];
            dm = dm >= 0 ? dm : edam[e];
            for (int m = 0; m < nmat; ++m) { vf[m] = 0.; md[m] = 0.; me[m] = 0.; }
            if (a.material == 0) {
                vf[0] = 1.0;
                for (int k = 0; k < 4; ++k) ewpt[4 * e + k] = 1.0;
            } else {
                epre[e] = pr; etem[e] = tm; edam[e] = dm;
                vf[a.material] = 1.0;
                const Mat &AM = S.mats[a.material];
                md[a.material] = eos_interp_tp(AM, tm, pr, -1) / pt;
                me[a.material] = eos_interp_tp(AM, tm, pr, 0) / pt;
                mp[a.material] = pt;
                for (int k = 0; k < 4; ++k) ewpt[4 * e + k] = -0.25;
                evel[2 * e] = v0;
                evel[2 * e + 1] = v1;
            }
        }
    }

    // gravity body force and the ANC taper of the Laplacian weights
    std::vector<double> &vbf = H.get("v_bf", NV * 2);
    std::string pat = lower(S.anc_pattern);
    for (int j = 0; j < vny; ++j)
        for (int i = 0; i < vnx; ++i) {
            const size_t p = (size_t)i + (size_t)vnx * j;
            double *bf = &vbf[2 * p];
            if (T.sphere) {
                const double *vp = &vpos[2 * p];
                double q = 0.;
                q += (vp[0] - T.center[0]) * (vp[0] - T.center[0]);
                q += (vp[1] - T.center[1]) * (vp[1] - T.center[1]);
                const double pdis = sqrt(q);
                double g[2] = {1.0 * vp[0] + -1.0 * T.center[0], 1.0 * vp[1] + -1.0 * T.center[1]};
                norm2(g);
                int li = (int)floor(pdis / dz);
                li = std::min(li, n - 1);
                li = std::max(li, 0);
                bf[0] = gra[li] * g[0];
                bf[1] = gra[li] * g[1];
                if (pdis >= T.r_planet) {
                    const double s = (T.r_planet / pdis) * (T.r_planet / pdis);
                    bf[0] *= s;
                    bf[1] *= s;
                }
                for (int k = 0; k < 9; ++k) vlap[9 * p + k] *= 0.;
                continue;
            }
            bf[0] = S.gravity[0];
            bf[1] = S.gravity[1];
            if (j <= pad) bf[1] = 0.;
            double red = 0.;
            if (pat == "pml") {
                if (S.damp_y >= 1 && j <= 2 * S.damp_y) {
                    double lx = 0.5 * j / S.damp_y;
                    red = 2.0 * dmax(red, 2.0 * hanning(0.5 * (1.0 - lx)));
                }
                if (S.damp_x >= 1 && i >= vnx - 2 * S.damp_x) {
                    double lx = 0.5 * (vnx - 2 * S.damp_x - i) / S.damp_x;
                    red = 2.0 * dmax(red, 2.0 * hanning(0.5 * lx));
                }
            } else if (pat == "uniform") {
                red = 1.0;
            } else if (pat == "none") {
                red = 0.;
            } else {
                err = "ANC pattern '" + S.anc_pattern + "' is not supported by the deck initialiser";
                return SALEC_ERR_UNSUPPORTED;
            }
            for (int k = 0; k < 9; ++k) vlap[9 * p + k] *= red;
        }

    // tracer seeds: cell index and global id of every strip-th interior cell (the velocity,
    // which needs the vertex field, is filled in after the device init)
    tracer_rows.clear();
    const int strip = S.tracer_strip < 0 ? -S.tracer_strip : S.tracer_strip;
    for (int j = 0; j < eny; ++j)
        for (int i = 0; i < enx; ++i) {
            if (i < 2 || i > enx - 3 || j < 2 || j > eny - 3) continue;
            if (i % strip != 0 || j % strip != 0) continue;
            const size_t e = (size_t)i + (size_t)enx * j;
            int mid = 0;
            for (int m = 1; m < nmat; ++m)
                if (evof[nmat * e + mid] < evof[nmat * e + m]) mid = m;
            if (mid == 0) continue;
            const double row[12] = {epos[4 * e], epos[4 * e + 1], 0., 0., 0., 0., (double)i, (double)j,
                                    (double)(i + enx * j), (double)mid, (double)i, (double)j};
            tracer_rows.insert(tracer_rows.end(), row, row + 12);
        }
    return SALEC_OK;
}

} // namespace salec

// ================================================================== device finish + C ABI
// implemented in salec_runtime.cu
int salec_internal_finish_init(salec_gpu *h, double damp_time_in, double *damp_time_out);
int salec_internal_fail(int code, const char *msg);

extern "C" int salec_gpu_create_from_deck(const char *deck_path, const char *eos_dir, salec_gpu **out)
{
    return salec_gpu_create_from_deck_ex(deck_path, eos_dir, SALEC_PRECISION_FP64, out);
}

extern "C" int salec_gpu_create_from_deck_ex(const char *deck_path, const char *eos_dir, int precision,
                                             salec_gpu **out)
{
    using namespace salec;
    if (!deck_path || !eos_dir || !out) return salec_internal_fail(SALEC_ERR_ARG, "null argument");
    *out = nullptr;
    std::string err;
    Deck D;
    if (!D.load(deck_path, false, err)) return salec_internal_fail(SALEC_ERR_ARG, err.c_str());
    Setup S0, S;
    if (!load_setup(S0, D, eos_dir, err)) return salec_internal_fail(SALEC_ERR_ARG, err.c_str());
    HostState H;
    std::vector<double> tracer_rows;
    int rc = build_host_state(S0, S, H, tracer_rows, err);
    if (rc) return salec_internal_fail(rc, err.c_str());

    salec_run_desc run{};
    run.precision = precision;
    run.nx = S.npgx * S.nx;
    run.ny = S.npgy * S.ny;
    run.nmat = S.nmat;
    run.damp_type = S.damp_type;
    for (int k = 0; k < 4; ++k) run.go[k] = S.go[k];
    run.partpres = S.partpres;
    run.porosity_model = S.porosity_model;
    run.acoustic_fluid = S.acoustic_fluid;
    run.tensile_failure = S.tensile_failure;
    run.tracer_lubrication = S.tracer_lubrication;
    run.avis1 = S.avis1; run.avis2 = S.avis2; run.anc = S.anc;
    run.density_cutoff = S.density_cutoff;
    // velocity limits relative to the impact speed or gravity when negative (src/sale2d.c:456-483)
    const double pv = sqrt(0. + S.p_vel[0] * S.p_vel[0] + S.p_vel[1] * S.p_vel[1]);
    const double gv = sqrt(0. + S.gravity[0] * S.gravity[0] + S.gravity[1] * S.gravity[1]);
    run.velocity_max = S.velocity_max > 0. ? S.velocity_max : fabs(S.velocity_max) * pv;
    run.velocity_min = S.velocity_min > 0. ? S.velocity_min : fabs(S.velocity_min) * pv;
    run.acceleration_min = S.acceleration_min > 0. ? S.acceleration_min : fabs(S.acceleration_min) * gv;
    run.alpha_damp_x = S.alpha_damp_x;
    run.alpha_damp_y = S.alpha_damp_y;
    run.damp_time = S.damp_t;
    run.threshold_z = S.ejecta_threshold * S.p_radius;
    run.flow_resistance = S.ejecta_resistance;
    run.flow_friction = S.ejecta_friction;
    run.tracer_lub_y0 = S.tracer_lub_y0;
    run.tracer_lub_gy0 = S.tracer_lub_gy0;
    run.tracer_lub_gy1 = S.tracer_lub_gy1;
    run.tracer_lub_frac = S.tracer_lub_frac;
    run.max_dt = S.max_dt;
    run.dt = S.dt0;
    run.time = S.time0;
    run.i_step = 0;
    std::vector<salec_material_desc> mats(S.nmat);
    for (int m = 1; m < S.nmat; ++m) {
        salec_material_desc d = S.mats[m].d;
        d.eos_type = S.mats[m].kind;
        if (S.mats[m].kind == 1) {
            d.cold_n = (int)S.mats[m].cold_y.size();
            d.cold_xden = S.mats[m].cold_x.data();
            d.cold_yeng = S.mats[m].cold_y.data();
        } else {
            d.ntem = S.mats[m].tab.ntem;
            d.nden = S.mats[m].tab.nden;
            d.xtem = S.mats[m].tab.xtem.data();
            d.yden = S.mats[m].tab.yden.data();
            d.data = S.mats[m].tab.data.data();
        }
        mats[m] = d;
    }
    salec_gpu *h = nullptr;
    rc = salec_gpu_create(&run, mats.data(), &h);
    if (rc) return rc;
    // The device pool starts zeroed (salec_gpu_create), so a field whose every value has the
    // bits of +0.0 needs no upload. The scan runs on this thread, while uploads of concurrent
    // initialisations serialise in the driver. Fields whose upload also builds device tables
    // (geometry rows, the Laplacian mask) always go through salec_gpu_set_field.
    auto all_plus_zero = [](const std::vector<double> &v) {
        const unsigned long long *w = reinterpret_cast<const unsigned long long *>(v.data());
        for (size_t k = 0; k < v.size(); k += 4096) {   // blocks of 32 KiB, early exit
            const size_t e = std::min(v.size(), k + 4096);
            unsigned long long acc = 0;
            for (size_t j = k; j < e; ++j) acc |= w[j];
            if (acc) return false;
        }
        return true;
    };
    static const char *const kTableFields[] = {"v_vol", "v_subvol", "v_suf", "e_grad", "e_vol", "v_laplace"};
    for (auto &kv : H.f) {
        int fid = salec_gpu_field_index(kv.first.c_str());
        if (fid < 0) continue;
        bool tables = false;
        for (const char *n : kTableFields) tables = tables || kv.first == n;
        if (!tables && all_plus_zero(kv.second)) {
            std::vector<double>().swap(kv.second);
            continue;
        }
        rc = salec_gpu_set_field(h, fid, kv.second.data(), (long long)kv.second.size());
        if (rc) { salec_gpu_destroy(h); return rc; }
        std::vector<double>().swap(kv.second);
    }
    double damp_time = 0.;
    rc = salec_internal_finish_init(h, run.damp_time, &damp_time);
    if (rc) { salec_gpu_destroy(h); return rc; }
    // tracer velocity: mean of the four vertex velocities (Interpolate2d_k at the cell centre)
    if (!tracer_rows.empty()) {
        int nx_, ny_, nc_;
        const int fv = salec_gpu_field_index("v_vel");
        salec_gpu_field_shape(h, fv, &nx_, &ny_, &nc_);
        std::vector<double> vv((size_t)nx_ * ny_ * nc_);
        rc = salec_gpu_get_field(h, fv, vv.data(), (long long)vv.size());
        if (rc) { salec_gpu_destroy(h); return rc; }
        const size_t nt = tracer_rows.size() / 12;
        for (size_t t = 0; t < nt; ++t) {
            double *r = &tracer_rows[12 * t];
            const int i = (int)r[10], j = (int)r[11];
            const size_t v[4] = {(size_t)i + (size_t)nx_ * j, (size_t)i + 1 + (size_t)nx_ * j,
                                 (size_t)i + 1 + (size_t)nx_ * (j + 1), (size_t)i + (size_t)nx_ * (j + 1)};
            for (int c = 0; c < 2; ++c) {
                double s = 0;
                for (int k = 0; k < 4; ++k) s += salec::ipb(k, 0., 0.) * vv[2 * v[k] + c];
                r[2 + c] = s;
            }
        }
        rc = salec_gpu_set_tracers(h, (int)nt, tracer_rows.data());
        if (rc) { salec_gpu_destroy(h); return rc; }
    }
    *out = h;
    return SALEC_OK;
}
