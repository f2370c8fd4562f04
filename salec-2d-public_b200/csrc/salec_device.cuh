// Device-side data model of the B200 mesh update: dimensions, field planes, run parameters,
// material records and the pointwise physics (equations of state, strength, damage and
// porosity functions) that the step kernels call.
//
// Layout: every scalar component of every field is its own plane of P x R doubles, row-major
// with x fastest (the reference's point order, src/mpi_vec/mpi_vec.h:372-376), so a warp
// touching 32 consecutive x points of one component issues one 256-byte transaction.
// Cells, vertices and faces share the pitch P and the plane stride PL, so the four vertices
// of cell (i, j) are the points i + P*j, i+1 + P*j, i+1 + P*(j+1) and i + P*(j+1) of any
// vertex plane.
//
// Arithmetic follows the reference's expression order term by term (no reassociation; the
// library is compiled with --fmad=false) so that the FP64 form reproduces the reference's
// rounding wherever the math library allows.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#define SALEC_MAXMAT 10
#define SALEC_TOLVOF 1.0e-6
#define SALEC_TOLRHO 1.0e-4
#define SALEC_TOLQPRE 1e-4
#define SALEC_DTF 0.2
#define SALEC_CISSAMK1 1.0

namespace salec {

struct Dims {
    int P, R;            // pitch (points per row) and rows of every plane
    long long PL;        // plane stride in doubles
    int enx, eny;        // cells including the two-cell pad
    int vnx, vny;        // vertices including the pad
    int nmat, phi;       // materials (with vacuum) and doubles per face flux record
};

// Per-material parameters; the reference's state_reference (src/eos/eos_state.h:43-151)
// restricted to what the step reads, plus the EOS table on the device.
struct DevMat {
    int eos_type, yfunc, tfunc, dsdf, porfunc, PolyLiq, PolySol, pad_;
    double VaporDen, MeltDen, GaCoef;
    double Yint0, Yfricint, Ylimint, Ydam0, Yfricdam, Ylimdam, Yten0;
    double IvanA, IvanB, IvanC, Pbd, Pbp, minPint, minPdam;
    double JCA, JCB, JCN, JCC, JCM, JCTREF, JCMaxPlastic;
    double Asimon, Csimon, Tmelt0, Tfrac, Tdelta;
    double Tlidc1, Tlidc2, Tlidc3, Tsolc1, Tsolc2, Tsolc3;
    double Toff, Cvib, VibMax, Tdamp, Pvlim, Acvis;
    double alpha0, alphax, epse0, chi, kappa, avel, epsec, epsex, alphamax, alphamax2, alphae;
    double gamfrac, melt_viscosity;
    // Tillotson: rho0, Cv, A, B, E0, a, b, alpha, beta, Eiv, Ecv, Tref, StepDen
    double tl[13];
    int cold_n, ntem, nden, pad2_;
    const double *cold_yeng;   // cold energy on the uniform density grid k*StepDen
    const double *xtem, *yden; // tabulated axes
    const double *data;        // [ntem][nden][3]
    // bucket guesses of the axis searches (axis_search); null where an axis is not monotone
    const int *xtem_bkt, *yden_bkt;
    double xtem_b0, xtem_binv, yden_b0, yden_binv;
    int xtem_nb, yden_nb;
};

// Run parameters fixed for the whole run (sale2d_var / mesh2d_info members).
struct RunParams {
    int damp_type, partpres, porosity_model, acoustic_fluid, tensile_failure;
    int tracer_lubrication, tracer_lub_gy0, tracer_lub_gy1;
    double avis1, avis2, anc;
    double density_cutoff, velocity_max, velocity_min, acceleration_min;
    double alpha_damp_x, alpha_damp_y, damp_time;
    double threshold_z, flow_resistance, flow_friction;
    double tracer_lub_y0, tracer_lub_frac;
    double max_dt;
};

// Scalars that evolve on the device, so that a step needs no host round trip.
struct Scal {
    double dt;                    // time step of the current cycle (final after the dt phase)
    double time;                  // simulated time at the start of the cycle
    unsigned long long dt_acc;    // ordered-bits MIN accumulator of the CFL candidates
    long long i_step;
    unsigned long long nan_count; // used by salec_gpu_check
    unsigned long long aux;       // ordered-bits MAX accumulator used at initialisation
    // NaN CFL candidates, kept as the reference's sequential MIN keeps them: the largest
    // traversal index (j * enx + i) of a cell whose candidate is NaN (-1: none), the MIN of the
    // candidates after it and the count of finished blocks of that recount
    long long dt_nan_last;
    unsigned long long dt_tail;
    unsigned int dt_tail_blocks, pad_;
};

// Device planes of every field. R is the storage type of the "relaxed" fields: double in the
// plain FP64 form, float in the mixed form. The fields that carry volume-fraction advection,
// mass and energy conservation and the mesh positions stay FP64 in both forms (m_vof, m_den,
// m_eng, v_pos, e_pos, e_vol, the face records bx_phi/by_phi and the surface profile), and so
// do the porosity state (distension m_pty and cold volume strain e_cvs): the compaction law is
// evaluated next to its thresholds (alpha0, epse0), where FP32 rounding of the distension
// moves it across them.
// Every member is a pointer, so all instances share one layout.
template <class R>
struct FieldsT {
    // vertices
    R *v_vel, *v_bf, *v_acc, *v_dis;
    double *v_pos;
    R *v_vof, *v_mass, *v_vol, *v_subvol, *v_laplace, *v_suf, *v_alpha, *v_beta;
    // cells
    R *e_vel, *e_div_vel, *e_grad_vel, *e_ste, *e_mu, *e_dvel, *e_pre, *e_tem, *e_den, *e_eng, *e_csd, *e_dam;
    double *e_cvs, *m_vof, *m_den, *m_eng, *m_pty;
    R *e_wpt;
    double *e_pos, *e_vol;
    R *e_suf, *e_grad, *e_subvol, *e_q, *e_strength, *e_cnd, *e_tps, *e_ste2s, *e_sta2s, *e_alpha, *e_beta,
        *e_sigma, *e_dampref, *e_vib, *e_ejt;
    // faces and columns
    double *bx_phi, *by_phi;
    R *bx_normal, *by_normal;
    double *y_profile;
};
using Fields = FieldsT<double>;
static_assert(sizeof(FieldsT<float>) == sizeof(FieldsT<double>), "field tables share one layout");

// Lagrangian tracers as structure-of-arrays in the reference's list order
// (tracer_t of src/mpi_vec/linked_list.h:17-27 plus the cell index and a live flag).
struct Tracers {
    double *x, *y, *vx, *vy, *rec_pre, *rec_tem;
    float *mpre, *mtem;
    int *gx, *gy, *tag, *matid, *cx, *cy, *alive;
    int n;
};

// A geometry field read through a table of its distinct rows: mesh row j holds the values of
// table row row[j] (the identity map over the field's own planes when the rows do not repeat).
// The values read are the field's own values; only their location differs.
template <class T>
struct GeoTab {
    const T *tab;      // component-0 plane of the table
    const int *row;    // table row of every mesh row
    long long plane;   // elements between components
};

template <class R>
struct CtxT {
    using real = R;
    Dims d;
    FieldsT<R> f;
    RunParams rp;
    const DevMat *mat;
    Scal *scal;
    Tracers tr;
    // one bit per vertex (rows of P/32 words): set where any nine-point Laplacian weight is non-zero
    const unsigned *lap_mask;
    GeoTab<R> g_v_vol, g_v_subvol, g_v_suf, g_e_grad;
    GeoTab<double> g_e_vol;
};
using Ctx = CtxT<double>;

// ------------------------------------------------------------------ small helpers
__host__ __device__ __forceinline__ double dmin(double a, double b) { return a < b ? a : b; }   // MIN / Min
__host__ __device__ __forceinline__ double dmax(double a, double b) { return a > b ? a : b; }   // MAX / Max
__host__ __device__ __forceinline__ double wind(double x, double lo, double hi)
{
    return x < lo ? lo : (x > hi ? hi : x);
}
__host__ __device__ __forceinline__ double sqrt_trunc(double x) { return x < 1.0e-2 ? -sqrt(fabs(x)) : sqrt(x); }

// Order-preserving map of doubles to unsigned integers (for atomic MIN of doubles).
__host__ __device__ __forceinline__ unsigned long long ord_encode(double v)
{
#ifdef __CUDA_ARCH__
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
#else
    unsigned long long b;
    memcpy(&b, &v, 8);
#endif
    return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}
__host__ __device__ __forceinline__ double ord_decode(unsigned long long u)
{
    unsigned long long b = (u & 0x8000000000000000ULL) ? (u & 0x7FFFFFFFFFFFFFFFULL) : ~u;
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double v;
    memcpy(&v, &b, 8);
    return v;
#endif
}

// Second invariant of a (rr, rz, zz, theta) tensor: geometry/linear.c:188-194.
__device__ __forceinline__ double second_inv(double xx, double xy, double yy, double th)
{
    return ((xx - yy) * (xx - yy) + (yy - th) * (yy - th) + (th - xx) * (th - xx)) / 6.0 + xy * xy;
}

// Interval search of geometry/linear.c:196-218: leftmost/rightmost interval outside the range.
__host__ __device__ __forceinline__ int bisearch(double x, const double *xs, int n)
{
    int lo = 0, hi = n - 1;
    if (x < xs[lo]) return lo;
    if (x >= xs[hi]) return hi - 1;
    while (lo + 1 < hi) {
        int mid = (lo + hi) / 2;
        if (xs[mid] > x) hi = mid; else lo = mid;
    }
    return lo;
}

// bisearch over a non-decreasing axis, started from a bucket guess. For x in [xs[0], xs[n-1])
// the bisection ends at the unique k with xs[k] <= x < xs[k+1] (its loop keeps xs[lo] <= x <
// xs[hi]); the guess bkt[(x - b0) * binv] is moved by the same comparisons until it satisfies
// both, so the index is the bisection's whatever the rounding of the bucket number. Below,
// above and NaN take the bisection's own exits (0, n-2, n-2). Typically two dependent loads
// instead of log2(n).
__host__ __device__ __forceinline__ int axis_search(double x, const double *xs, int n, const int *bkt, int nb, double b0,
                                           double binv)
{
    if (!bkt) return bisearch(x, xs, n);
    if (x < xs[0]) return 0;
    if (!(x < xs[n - 1])) return n - 2;
    int b = (int)((x - b0) * binv);
    b = b < 0 ? 0 : (b >= nb ? nb - 1 : b);
    int g = bkt[b];
    while (g < n - 2 && xs[g + 1] <= x) ++g;
    while (g > 0 && xs[g] > x) --g;
    return g;
}

// Bucket guesses for axis_search over xs[0..n-1]: 2n uniform buckets over [xs[0], xs[n-1]);
// bucket b holds the largest k <= n-2 with xs[k] <= xs[0] + b * width. No table (false) for an
// axis that is not non-decreasing and finite: the device then bisects.
inline bool build_axis_buckets(const double *xs, int n, std::vector<int> &bkt, double &b0, double &binv)
{
    if (n < 3) return false;
    for (int k = 0; k < n; ++k)
        if (!std::isfinite(xs[k]) || (k && !(xs[k] >= xs[k - 1]))) return false;
    const double span = xs[n - 1] - xs[0];
    const int nb = 2 * n;
    if (!(span > 0.0) || !std::isfinite(nb / span)) return false;
    b0 = xs[0];
    binv = nb / span;
    bkt.resize(nb);
    int k = 0;
    for (int b = 0; b < nb; ++b) {
        const double edge = xs[0] + b * (span / nb);
        while (k < n - 2 && xs[k + 1] <= edge) ++k;
        bkt[b] = k;
    }
    return true;
}

// ------------------------------------------------------------------ Tillotson EOS
// Tillotson (1962) as evaluated in src/eos/eos_state.c:322-438 (TillCold, TillHot, TillTran,
// TillPres); t = {rho0, Cv, A, B, E0, a, b, alpha, beta, Eiv, Ecv, Tref, StepDen}.
__host__ __device__ __forceinline__ void till_pressure(const double *t, double E, double rho, double &pres, double &cs)
{
    const double rho0 = t[0], A = t[2], B = t[3], E0 = t[4], a = t[5], b = t[6];
    const double al = t[7], be = t[8], Eiv = t[9], Ecv = t[10];
    const double eta = rho / rho0;
    const double mu = eta - 1.0;
    const double phi0 = E / (E0 * eta * eta);
    const double phi1 = 1.0 / (phi0 + 1.0);
    if ((rho >= rho0) || (E < Eiv)) {
        // compressed or cold
        double Bx = eta < 1.0 ? A : B;
        pres = (a + b * phi1) * E * rho + A * mu + Bx * mu * mu;
        double c1 = (1.0 / rho0) * (A + 2.0 * Bx * mu) + E * (a + b * phi1 * (3.0 - 2.0 * phi1));
        double c2 = (a + b * phi1 * phi1) * pres / rho;
        cs = sqrt_trunc(c1 + c2);
    } else {
        const double xi = rho0 / rho - 1.0;
        double ea = 0.0, eb = 0.0;
        if (al * xi * xi < 100.0) ea = exp(-1.0 * al * xi * xi);
        if (be * xi < 100.0) eb = exp(-1.0 * be * xi);
        const double ph = a * rho * E + (b * E * rho * phi1 + A * mu * eb) * ea;
        if (E > Ecv) {
            // expanded and hot
            pres = ph;
            double c1 = a * E + b * E * phi1 * (3.0 + 2.0 * al * xi / eta - 2.0 * phi1) * ea
                      + A / rho0 * (1.0 - (xi / eta) * (be + 2.0 * al * xi)) * ea * eb;
            double c2 = (a + b * phi1 * phi1 * ea) * pres / rho;
            cs = sqrt_trunc(c1 + c2);
        } else {
            // linear blend of the two branches between Eiv and Ecv
            const double dT = Ecv - Eiv, dEr = E - Eiv, dEl = Ecv - E;
            double Bx = eta < 1.0 ? A : B;
            const double pc = (a + b * phi1) * E * rho + A * mu + Bx * mu * mu;
            pres = (dEl * pc + dEr * ph) / dT;
            double cc1 = (1.0 / rho0) * (A + 2.0 * Bx * mu) + E * (a + b * phi1 * (3.0 - 2.0 * phi1));
            double cc2 = (a + b * phi1 * phi1) * pres / rho;
            double ch1 = a * E + b * E * phi1 * (3.0 + 2.0 * al * xi / eta - 2.0 * phi1) * ea
                       + A / rho0 * (1.0 - (xi / eta) * (be + 2.0 * al * xi)) * ea * eb;
            double ch2 = (a + b * phi1 * phi1 * ea) * pres / rho;
            double c2c = cc1 + cc2;
            double c2h = ch1 + ch2;
            double s1 = (dEl * c2c + dEr * c2h) / dT;
            double s2 = (ph - pc) / dT * pres / (rho * rho);
            cs = sqrt_trunc(s1 + s2);
        }
    }
    if (pres <= 1.0e-2) cs = sqrt_trunc(A / rho0);
}

// Temperature from the cold-energy curve sampled at k*StepDen (src/eos/eos_state.c:519-526).
__device__ __forceinline__ double till_temperature(const DevMat &m, double E, double rho)
{
    const double *t = m.tl;
    const double step = t[12];
    int dl = (int)(wind(floor(rho / step), 0, m.cold_n - 2));
    double dxl = dl + 1.0 - rho / step;
    double dxr = 1.0 - dxl;
    double ecold = dxl * m.cold_yeng[dl] + dxr * m.cold_yeng[dl + 1];
    return dmax((E - ecold) / t[1] + t[11], 0.0);
}

// Bilinear table lookup over (density, specific energy): src/eos/aneos_sieden.c:264-290.
__device__ __forceinline__ void sieden_state(const DevMat &m, double den, double eng, double &tem, double &pre, double &csd)
{
    const double tden = den;
    const double teng = eng / den;
    const int di = axis_search(tden, m.yden, m.nden, m.yden_bkt, m.yden_nb, m.yden_b0, m.yden_binv), dj = di + 1;
    const int ti = axis_search(teng, m.xtem, m.ntem, m.xtem_bkt, m.xtem_nb, m.xtem_b0, m.xtem_binv), tj = ti + 1;
    const double dxr = (tden - m.yden[di]) / (m.yden[dj] - m.yden[di]);
    const double dxl = wind(1.0 - dxr, 0.0, 1.0);
    const double exr = (teng - m.xtem[ti]) / (m.xtem[tj] - m.xtem[ti]);
    const double exl = wind(1.0 - exr, 0., 1.0);
    const double *a = m.data + ((size_t)ti * m.nden + di) * 3;
    const double *b = m.data + ((size_t)ti * m.nden + dj) * 3;
    const double *c = m.data + ((size_t)tj * m.nden + di) * 3;
    const double *d = m.data + ((size_t)tj * m.nden + dj) * 3;
    tem = (a[0] * dxl + b[0] * dxr) * exl + (c[0] * dxl + d[0] * dxr) * exr;
    pre = (a[1] * dxl + b[1] * dxr) * exl + (c[1] * dxl + d[1] * dxr) * exr;
    csd = (a[2] * dxl + b[2] * dxr) * exl + (c[2] * dxl + d[2] * dxr) * exr;
}

// Temperature-density table with energy rows searched per density: src/eos/eos_state.c:793-841.
__device__ __forceinline__ void aneos_td_state(const DevMat &m, double den, double eng, double &tem, double &pre, double &csd)
{
    // on a monotone axis the bracketing loop of eos_state.c ends where axis_search does: 0 below
    // the axis, n-2 above it and for NaN, else the k with yden[k] <= den < yden[k+1]
    int di = 0, dj = m.nden - 1;
    if (m.yden_bkt) {
        di = axis_search(den, m.yden, m.nden, m.yden_bkt, m.yden_nb, m.yden_b0, m.yden_binv);
        dj = di + 1;
    } else {
        while (di + 1 < dj) {
            int dm = (di + dj) / 2;
            if (m.yden[dm] > den) dj = dm; else di = dm;
        }
    }
    double dxr = (den - m.yden[di]) / (m.yden[dj] - m.yden[di]);
    dxr = wind(dxr, 0.0, 1.0);
    const double dxl = 1.0 - dxr;
    auto D = [&](int it, int id, int c) { return m.data[((size_t)it * m.nden + id) * 3 + c]; };
    int ti = 0, tj = m.ntem - 1;
    double ire = D(ti, di, 0) * dxl + D(ti, dj, 0) * dxr;
    double jre = D(tj, di, 0) * dxl + D(tj, dj, 0) * dxr;
    while (ti + 1 < tj) {
        int tm = (ti + tj) / 2;
        double mre = D(tm, di, 0) * dxl + D(tm, dj, 0) * dxr;
        if (mre > eng) { tj = tm; jre = mre; } else { ti = tm; ire = mre; }
    }
    double txr = (eng - ire) / (jre - ire);
    txr = wind(txr, 0.0, 1.0);
    const double txl = 1.0 - txr;
    tem = m.xtem[ti] * txl + m.xtem[tj] * txr;
    pre = (D(ti, di, 1) * dxl + D(ti, dj, 1) * dxr) * txl + (D(tj, di, 1) * dxl + D(tj, dj, 1) * dxr) * txr;
    csd = (D(ti, di, 2) * dxl + D(ti, dj, 2) * dxr) * txl + (D(tj, di, 2) * dxl + D(tj, dj, 2) * dxr) * txr;
}

// calculate_state_correct with CAP_MINPRESSURE (src/eos/eos_state.c:747-791): porosity-scaled
// state, porous sound speed, pressure floor.
__device__ __forceinline__ void material_state(const DevMat &m, double den, double eng, double plim, double pty,
                                               double &tem, double &pre, double &csd)
{
    double t = 0., p = 0., c = 0.;
    const double d = den * pty, e = eng * pty;
    if (m.eos_type == 1) {
        const double ein = e / d;
        t = till_temperature(m, ein, d);
        till_pressure(m.tl, ein, d, p, c);
    } else if (m.eos_type == 2) {
        sieden_state(m, d, e, t, p, c);
    } else {
        aneos_td_state(m, d, e, t, p, c);
    }
    p = p / pty;
    if (pty > 1.0) c *= (1.0 + (m.chi - 1.0) * fmax(0.0, fmin(1.0, (pty - 1.0) / (m.alpha0 - 1.0))));
    if (p < plim) p = dmax(p, plim);
    tem = t; pre = p; csd = c;
}

// ------------------------------------------------------------------ strength model pieces
// Published forms as written in src/strength.c:505-570.
__device__ __forceinline__ double y_lundborg(double p, double y0, double fric, double ylim)
{
    return y0 + p * fric / (1 + p * fric / (ylim - y0));
}
__device__ __forceinline__ double y_drucker(double p, double y0, double fric, double ylim)
{
    return dmin(y0 + fric * p, ylim);
}
__device__ __forceinline__ double simon_melt(double pre, const DevMat &s)
{
    double sol = s.Tmelt0 * pow(s.Asimon * pre + 1.0, s.Csimon);
    if (s.PolyLiq <= 0 && s.PolySol <= 0) return sol;
    if (s.PolySol > 0) {
        double pg = pre * 1.0e-9;
        sol = s.Tsolc1 + s.Tsolc2 * pg + s.Tsolc3 * pg * pg;
    }
    double pg = pre * 1.0e-9;
    double liq = s.Tlidc1 + s.Tlidc2 * pg + s.Tlidc3 * pg * pg;
    return dmax(sol, liq);
}
__device__ __forceinline__ double ohnaka_soft(double tem, const DevMat &s, double tmelt)
{
    return tanh(((tmelt + s.Tdelta) / tem - 1.0) * s.Tfrac);
}
__device__ __forceinline__ double jnck_soft(double tem, double pre, const DevMat &s)
{
    double tm = simon_melt(pre, s);
    double mf = (tem - s.JCTREF) / (tm - s.JCTREF);
    mf = wind(mf, 0.0, 1.0);
    return wind(1.0 - pow(mf, s.JCM), 0.0, 1.0);
}
__device__ __forceinline__ double ice_melt(double p)
{
    // piecewise ice melting curve with a Simon-type high-pressure branch (src/strength.c:725-754)
    const double p0 = 0.0, p1 = 0.2e9, p2 = 0.34e9, p3 = 0.61e9, p4 = 2.17e9;
    const double t0 = 273.0, t1 = 252.0, t2 = 257.0, t3 = 274.0, t4 = 354.8;
    if (p <= p1) return t0 + (t1 - t0) * (p - p0) / (p1 - p0);
    else if (p > p1 && p <= p2) return t1 + (t2 - t1) * (p - p1) / (p2 - p1);
    else if (p > p2 && p <= p3) return t2 + (t3 - t2) * (p - p2) / (p3 - p2);
    else if (p > p3 && p <= p4) return t3 + (t4 - t3) * (p - p3) / (p4 - p3);
    return t4 * pow(((p - p4) / 1.253e9) + 1, 1.0 / 3.0);
}

// The registry of src/strength.c:860-875 as one dispatcher. pa = {pressure, damage, plastic
// strain, strain rate, temperature, ...} (porosity uses its own six arguments); passed by value
// so that no caller keeps an array in local memory.
static __device__ __noinline__ double strength_fn(int id, double p0, double p1, double p2, double p3, double p4,
                                                  double p5, const DevMat &s)
{
    const double pa[6] = {p0, p1, p2, p3, p4, p5};
    const double BETA = 0.57735026918962576451;   // JohnsonCook factor as in interpolate_fn.h
    switch (id) {
    case 0: { // SimpleRock (never selectable in the reference: str2func rejects index 0)
        double yint = y_lundborg(pa[0], s.Yint0, s.Yfricint, s.Ylimint);
        double ydam = y_drucker(pa[0], s.Ydam0, s.Yfricdam, s.Ylimdam);
        ydam = dmin(yint, ydam);
        return ydam * pa[1] + yint * (1.0 - pa[1]);
    }
    case 1: case 7: // SimpleShear / Ivanov damage increment
        return 1.0 / dmax(s.IvanA, s.IvanB * (pa[0] - s.IvanC));
    case 2: case 3: { // JohnsonCook1 / JohnsonCook2
        double ps = wind(pa[2], 0.0, s.JCMaxPlastic);
        double y1 = s.JCA + s.JCB * pow(ps, s.JCN);
        double y2 = 1.0;
        if (pa[3] > 1.0 && s.JCC > 0.0) y2 = 1.0 + s.JCC * log(pa[3]);
        if (id == 3) return y1 * y2 * jnck_soft(pa[4], pa[0], s) * BETA;
        return y1 * y2 * BETA;
    }
    case 4: { // RockStrengthT
        double pre = pa[0], dam = pa[1];
        double dps = pa[3], temp = pa[4];
        double yint = y_lundborg(pre, s.Yint0, s.Yfricint, s.Ylimint);
        double ydam = y_drucker(pre, s.Ydam0, s.Yfricdam, s.Ylimdam);
        ydam = dmin(yint, ydam);
        double tm = simon_melt(pre, s);
        double soft = ohnaka_soft(temp, s, tm);
        soft = wind(soft, 0.0, 1.0);
        double ymed = (ydam * dam + yint * (1.0 - dam)) * soft;
        double yvis = dps * s.melt_viscosity * (1.0 - soft);
        return dmax(ymed, yvis);
    }
    case 5: { // IceStrength
        double pre = pa[0], dam = pa[1], temp = pa[4];
        double yint = y_lundborg(pre, s.Yint0, s.Yfricint, s.Ylimint);
        double ydam = y_lundborg(pre, s.Ydam0, s.Yfricdam, s.Ylimdam);
        ydam = dmin(yint, ydam);
        double tm = ice_melt(pre);
        double soft = ohnaka_soft(temp, s, tm);
        soft = wind(soft, 0.0, 1.0);
        return (ydam * dam + yint * (1.0 - dam)) * soft;
    }
    case 6: { // Collins damage increment
        double pre = pa[0], inc;
        if (pre < s.Pbd) inc = dmax(0.01, 0.01 + 0.04 * pre / s.Pbd);
        else if (pre < s.Pbp) inc = 0.05 + 0.05 * (pre - s.Pbd) / (s.Pbp - s.Pbd);
        else inc = 0.1 + 0.5 * (pre - s.Pbp) / s.Pbp;
        return 1.0 / inc;
    }
    case 8: { // SimpleTensile
        double tm = simon_melt(pa[0], s);
        double soft = ohnaka_soft(pa[4], s, tm);
        soft = wind(soft, 0.0, 1.0);
        return s.Yten0 * (1.0 - pa[1]) * soft;
    }
    case 11: { // VonMises1
        double yint = s.Yint0, ydam = dmin(yint, s.Ydam0);
        return ydam * pa[1] + yint * (1.0 - pa[1]);
    }
    case 12: { // VonMises2
        double yint = s.Yint0, ydam = dmin(yint, s.Ydam0);
        double tm = simon_melt(pa[0], s);
        double soft = wind(ohnaka_soft(pa[4], s, tm), 0.0, 1.0);
        return (ydam * pa[1] + yint * (1.0 - pa[1])) * soft;
    }
    case 10: { // Wunnemann et al. (2006) epsilon-alpha porosity rate (src/strength.c:801-854)
        double pty = pa[0], cvs = pa[1], pre = pa[2], dcvs = pa[3], evx = pa[4], evy = pa[5];
        if (pty <= 1.0 || pty > s.alphamax || pre <= 0.) return 0.;
        double v2 = evx * evx + evy * evy;
        if (v2 <= s.avel * s.avel) return 0.;
        double cvs_c;
        if (pty > s.alphae) cvs_c = s.epse0;
        else if (pty > s.alphax) cvs_c = s.epse0 + log(pty / s.alphae) / s.kappa;
        else cvs_c = s.epsec - sqrt((pty - 1.0) / (s.alphax - 1.0)) * (s.epsec - s.epsex);
        double ratio = 1.0 + (s.chi - 1.0) * fmax(0.0, fmin(1.0, (pty - 1.0) / (s.alphamax - 1.0)));
        double dade = pty * (1.0 - ratio * ratio);
        if (dcvs < 0. && cvs < cvs_c) {
            if (pty > s.alphax) dade = s.kappa * pty;
            else dade = sqrt((pty - 1.) / (s.alphax - 1.0)) * s.kappa * s.alphax;
        } else {
            dade = pty * (1.0 - ratio * ratio);
        }
        return dade * dcvs;
    }
    case 9:
    default:
        return 0.0;
    }
}

} // namespace salec
