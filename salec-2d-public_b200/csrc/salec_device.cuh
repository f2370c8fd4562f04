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
    const float *data_f;       // the same table rounded to float (mixed form: FP32 interpolation)
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
    // prescribed time steps (null: none): cycle i_step = dt_sched_i0 + k takes dt_sched[k] for
    // 0 <= k < dt_sched_n instead of the CFL reduction
    const double *dt_sched;
    long long dt_sched_i0;
    int dt_sched_n;
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
// The same on the arithmetic type A of a sweep: double in the plain form, float where the mixed
// form computes in FP32 (stress, strength, viscosity, stress divergence, table interpolation).
// With A = double every operation is the FP64 form's.
template <class A> __host__ __device__ __forceinline__ A amin(A a, A b) { return a < b ? a : b; }
template <class A> __host__ __device__ __forceinline__ A amax(A a, A b) { return a > b ? a : b; }
template <class A> __host__ __device__ __forceinline__ A awind(A x, A lo, A hi) { return x < lo ? lo : (x > hi ? hi : x); }
template <class A> __host__ __device__ __forceinline__ A asqrt_trunc(A x) { return x < 1.0e-2 ? -sqrt(fabs(x)) : sqrt(x); }
// the value of a scalar (the dual numbers of salec_dual.cuh overload it)
__host__ __device__ __forceinline__ double val(double x) { return x; }

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
template <class A>
__host__ __device__ __forceinline__ A second_inv(A xx, A xy, A yy, A th)
{
    return ((xx - yy) * (xx - yy) + (yy - th) * (yy - th) + (th - xx) * (th - xx)) / A(6.0) + xy * xy;
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
// TillPres); t = {rho0, Cv, A, B, E0, a, b, alpha, beta, Eiv, Ecv, Tref, StepDen}. T is double in
// the step and a dual number in the adjoint (its local derivatives).
template <class T>
__host__ __device__ __forceinline__ void till_pressure(const double *t, T E, T rho, T &pres, T &cs)
{
    const double rho0 = t[0], A = t[2], B = t[3], E0 = t[4], a = t[5], b = t[6];
    const double al = t[7], be = t[8], Eiv = t[9], Ecv = t[10];
    const T eta = rho / rho0;
    const T mu = eta - 1.0;
    const T phi0 = E / (E0 * eta * eta);
    const T phi1 = 1.0 / (phi0 + 1.0);
    if ((rho >= rho0) || (E < Eiv)) {
        // compressed or cold
        double Bx = eta < 1.0 ? A : B;
        pres = (a + b * phi1) * E * rho + A * mu + Bx * mu * mu;
        T c1 = (1.0 / rho0) * (A + 2.0 * Bx * mu) + E * (a + b * phi1 * (3.0 - 2.0 * phi1));
        T c2 = (a + b * phi1 * phi1) * pres / rho;
        cs = asqrt_trunc(c1 + c2);
    } else {
        const T xi = rho0 / rho - 1.0;
        T ea = T(0.0), eb = T(0.0);
        if (al * xi * xi < 100.0) ea = exp(-1.0 * al * xi * xi);
        if (be * xi < 100.0) eb = exp(-1.0 * be * xi);
        const T ph = a * rho * E + (b * E * rho * phi1 + A * mu * eb) * ea;
        if (E > Ecv) {
            // expanded and hot
            pres = ph;
            T c1 = a * E + b * E * phi1 * (3.0 + 2.0 * al * xi / eta - 2.0 * phi1) * ea
                 + A / rho0 * (1.0 - (xi / eta) * (be + 2.0 * al * xi)) * ea * eb;
            T c2 = (a + b * phi1 * phi1 * ea) * pres / rho;
            cs = asqrt_trunc(c1 + c2);
        } else {
            // linear blend of the two branches between Eiv and Ecv
            const double dT = Ecv - Eiv;
            const T dEr = E - Eiv, dEl = Ecv - E;
            double Bx = eta < 1.0 ? A : B;
            const T pc = (a + b * phi1) * E * rho + A * mu + Bx * mu * mu;
            pres = (dEl * pc + dEr * ph) / dT;
            T cc1 = (1.0 / rho0) * (A + 2.0 * Bx * mu) + E * (a + b * phi1 * (3.0 - 2.0 * phi1));
            T cc2 = (a + b * phi1 * phi1) * pres / rho;
            T ch1 = a * E + b * E * phi1 * (3.0 + 2.0 * al * xi / eta - 2.0 * phi1) * ea
                  + A / rho0 * (1.0 - (xi / eta) * (be + 2.0 * al * xi)) * ea * eb;
            T ch2 = (a + b * phi1 * phi1 * ea) * pres / rho;
            T c2c = cc1 + cc2;
            T c2h = ch1 + ch2;
            T s1 = (dEl * c2c + dEr * c2h) / dT;
            T s2 = (ph - pc) / dT * pres / (rho * rho);
            cs = asqrt_trunc(s1 + s2);
        }
    }
    if (pres <= 1.0e-2) cs = T(asqrt_trunc(A / rho0));
}

// Temperature from the cold-energy curve sampled at k*StepDen (src/eos/eos_state.c:519-526).
template <class T>
__device__ __forceinline__ T till_temperature(const DevMat &m, T E, T rho)
{
    const double *t = m.tl;
    const double step = t[12];
    int dl = (int)(wind(floor(val(rho) / step), 0, m.cold_n - 2));
    T dxl = dl + 1.0 - rho / step;
    T dxr = 1.0 - dxl;
    T ecold = dxl * m.cold_yeng[dl] + dxr * m.cold_yeng[dl + 1];
    return amax((E - ecold) / t[1] + t[11], T(0.0));
}

// Table value k of a tabulated material on the arithmetic type: the FP64 table, or its float copy.
template <class A>
__device__ __forceinline__ A tab_at(const DevMat &m, size_t k)
{
    if constexpr (sizeof(A) == sizeof(float)) return m.data_f[k];
    else return m.data[k];
}

// Bilinear table lookup over (density, specific energy): src/eos/aneos_sieden.c:264-290. The axis
// searches and the interpolation weights are FP64 (the weights' differences cancel); the blend of
// the table values runs on A.
template <class A>
__device__ __forceinline__ void sieden_state(const DevMat &m, double den, double eng, A &tem, A &pre, A &csd)
{
    const double tden = den;
    const double teng = eng / den;
    const int di = axis_search(tden, m.yden, m.nden, m.yden_bkt, m.yden_nb, m.yden_b0, m.yden_binv), dj = di + 1;
    const int ti = axis_search(teng, m.xtem, m.ntem, m.xtem_bkt, m.xtem_nb, m.xtem_b0, m.xtem_binv), tj = ti + 1;
    const double dxr = (tden - m.yden[di]) / (m.yden[dj] - m.yden[di]);
    const double dxl = wind(1.0 - dxr, 0.0, 1.0);
    const double exr = (teng - m.xtem[ti]) / (m.xtem[tj] - m.xtem[ti]);
    const double exl = wind(1.0 - exr, 0., 1.0);
    const A wr = A(dxr), wl = A(dxl), er = A(exr), el = A(exl);
    const size_t a = ((size_t)ti * m.nden + di) * 3;
    const size_t b = ((size_t)ti * m.nden + dj) * 3;
    const size_t c = ((size_t)tj * m.nden + di) * 3;
    const size_t d = ((size_t)tj * m.nden + dj) * 3;
    tem = (tab_at<A>(m, a) * wl + tab_at<A>(m, b) * wr) * el + (tab_at<A>(m, c) * wl + tab_at<A>(m, d) * wr) * er;
    pre = (tab_at<A>(m, a + 1) * wl + tab_at<A>(m, b + 1) * wr) * el +
          (tab_at<A>(m, c + 1) * wl + tab_at<A>(m, d + 1) * wr) * er;
    csd = (tab_at<A>(m, a + 2) * wl + tab_at<A>(m, b + 2) * wr) * el +
          (tab_at<A>(m, c + 2) * wl + tab_at<A>(m, d + 2) * wr) * er;
}

// Temperature-density table with energy rows searched per density: src/eos/eos_state.c:793-841.
// The searches and weights are FP64; the blend of pressure and sound speed runs on A.
template <class A>
__device__ __forceinline__ void aneos_td_state(const DevMat &m, double den, double eng, A &tem, A &pre, A &csd)
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
    auto DA = [&](int it, int id, int c) { return tab_at<A>(m, ((size_t)it * m.nden + id) * 3 + c); };
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
    tem = A(m.xtem[ti] * txl + m.xtem[tj] * txr);
    const A wl = A(dxl), wr = A(dxr), ul = A(txl), ur = A(txr);
    pre = (DA(ti, di, 1) * wl + DA(ti, dj, 1) * wr) * ul + (DA(tj, di, 1) * wl + DA(tj, dj, 1) * wr) * ur;
    csd = (DA(ti, di, 2) * wl + DA(ti, dj, 2) * wr) * ul + (DA(tj, di, 2) * wl + DA(tj, dj, 2) * wr) * ur;
}

// calculate_state_correct with CAP_MINPRESSURE (src/eos/eos_state.c:747-791): porosity-scaled
// state, porous sound speed, pressure floor. The Tillotson form is evaluated in FP64 (its
// compression mu = rho/rho0 - 1 cancels); the tabulated forms interpolate on A.
template <class A>
__device__ __forceinline__ void material_state(const DevMat &m, double den, double eng, double plim, double pty,
                                               A &tem, A &pre, A &csd)
{
    A t = A(0.), p = A(0.), c = A(0.);
    const double d = den * pty, e = eng * pty;
    if (m.eos_type == 1) {
        const double ein = e / d;
        double pd, cd;
        t = A(till_temperature(m, ein, d));
        till_pressure(m.tl, ein, d, pd, cd);
        p = A(pd);
        c = A(cd);
    } else if (m.eos_type == 2) {
        sieden_state<A>(m, d, e, t, p, c);
    } else {
        aneos_td_state<A>(m, d, e, t, p, c);
    }
    p = p / A(pty);
    if (pty > 1.0) c *= A(1.0 + (m.chi - 1.0) * fmax(0.0, fmin(1.0, (pty - 1.0) / (m.alpha0 - 1.0))));
    if (p < A(plim)) p = amax(p, A(plim));
    tem = t; pre = p; csd = c;
}

// ------------------------------------------------------------------ flux geometry
// Pieces of calculate_flux_mixed (src/advect.c:861-1136), templates on the scalar type (double
// in the step, a dual number in the adjoint).
template <class T>
__host__ __device__ __forceinline__ T swept_volume(double xa, double ya, double xb, double yb, T dxa, T dya, T dxb, T dyb)
{
    // get_flux_volcyl (src/advect.c:1347-1354)
    const T x1 = -1.0 * dxa, y1 = -1.0 * dya, x2 = -1.0 * dxb, y2 = -1.0 * dyb;
    const T vol = x1 * (ya - yb - y2) + x2 * (ya - yb + y1) + (y1 + y2) * (xb - xa);
    return vol * fabs(2.0 * xa + 2.0 * xb + x1 + x2) / 8.0;
}

template <class T>
__host__ __device__ __forceinline__ T face_ratio(T p1, T p2)
{
    // geometric_flux_ratio (src/advect.c:1312-1330)
    T a = p1, b = p2;
    if (b > a) { a = p2; b = p1; }
    if (b >= 0.0) return T(1.0);
    if (a <= 0.0) return T(0.0);
    return a / (a + fabs(b));
}

template <class T>
__host__ __device__ __forceinline__ T cut_length(T vf, T a, T b)
{
    // cut_length / cut_length_l / cut_length_s (src/advect.c:1356-1407)
    if (a < b) { T t = a; a = b; b = t; }
    if (1.0e-5 * a > b) {
        T d;
        if (vf <= 0.0) d = T(0.0);
        else if (vf <= 1.0) d = vf * a;
        else d = a;
        return d + b;
    }
    const T crf1 = 0.5 * b / a;
    if (vf <= crf1) return sqrt(2.0 * a * b * vf);
    if (vf <= 1.0 - crf1) return 0.5 * b + a * vf;
    if (vf <= 1.0) return a + b - sqrt(2.0 * a * b * (1.0 - vf));
    return a + b;
}

template <class T>
__host__ __device__ __forceinline__ void normalise2(T &x, T &y)
{
    // vec_norm (src/geometry/linear.c:132-146)
    T len = T(0.);
    len += x * x;
    len += y * y;
    len = sqrt(len);
    x /= len;
    if (isnan(val(x))) x = T(1.0);
    y /= len;
    if (isnan(val(y))) y = T(1.0);
}

__device__ __forceinline__ double mstacs(double nd, double gf, double cr)
{
    // vofMSTACS (src/advect.c:1259-1274)
    double cds, st;
    if (cr < 1.0 / 3.0) cds = dmin(nd / cr, 1.0);
    else cds = dmin(3.0 * nd, 1.0);
    if (nd < 1.0 / 5.0) st = 3.0 * nd;
    else if (nd < 1.0 / 2.0) st = (1.0 + nd) / 2.0;
    else st = dmin((6.0 * nd + 3.0) / 8.0, 1.0);
    return gf * cds + (1.0 - gf) * st;
}

__device__ __forceinline__ double algebraic_ratio(double vu, double vd, double va, double cr, double nx, double ny,
                                                  double gx, double gy)
{
    // algebraic_flux_ratio (src/advect.c:1226-1253)
    const double tmp = va - vu;
    const double nd = (vd - vu) / tmp;
    if (fabs(tmp) < SALEC_TOLVOF) return vd;
    if (nd < SALEC_TOLVOF || nd > 1.0 - SALEC_TOLVOF) return vd;
    double dot = 0.; dot += gx * nx; dot += gy * ny;
    double len = 0.; len += gx * gx; len += gy * gy;
    double cost = dot / sqrt(len);
    cost = cost * cost;
    const double gf = dmin(SALEC_CISSAMK1 * cost * cost, 1.0);
    return vu + mstacs(nd, gf, cr) * (va - vu);
}

// ------------------------------------------------------------------ strength model pieces
// Published forms as written in src/strength.c:505-570, on the arithmetic type A.
template <class A>
__host__ __device__ __forceinline__ A y_lundborg(A p, A y0, A fric, A ylim)
{
    return y0 + p * fric / (A(1) + p * fric / (ylim - y0));
}
template <class A>
__host__ __device__ __forceinline__ A y_drucker(A p, A y0, A fric, A ylim)
{
    return amin(y0 + fric * p, ylim);
}
template <class A>
__host__ __device__ __forceinline__ A simon_melt(A pre, const DevMat &s)
{
    A sol = A(s.Tmelt0) * pow(A(s.Asimon) * pre + A(1.0), A(s.Csimon));
    if (s.PolyLiq <= 0 && s.PolySol <= 0) return sol;
    if (s.PolySol > 0) {
        A pg = pre * A(1.0e-9);
        sol = A(s.Tsolc1) + A(s.Tsolc2) * pg + A(s.Tsolc3) * pg * pg;
    }
    A pg = pre * A(1.0e-9);
    A liq = A(s.Tlidc1) + A(s.Tlidc2) * pg + A(s.Tlidc3) * pg * pg;
    return amax(sol, liq);
}
template <class A>
__host__ __device__ __forceinline__ A ohnaka_soft(A tem, const DevMat &s, A tmelt)
{
    return tanh(((tmelt + A(s.Tdelta)) / tem - A(1.0)) * A(s.Tfrac));
}
template <class A>
__device__ __forceinline__ A jnck_soft(A tem, A pre, const DevMat &s)
{
    A tm = simon_melt<A>(pre, s);
    A mf = (tem - A(s.JCTREF)) / (tm - A(s.JCTREF));
    mf = awind(mf, A(0.0), A(1.0));
    return awind(A(1.0) - pow(mf, A(s.JCM)), A(0.0), A(1.0));
}
template <class A>
__device__ __forceinline__ A ice_melt(A p)
{
    // piecewise ice melting curve with a Simon-type high-pressure branch (src/strength.c:725-754)
    const A p0 = A(0.0), p1 = A(0.2e9), p2 = A(0.34e9), p3 = A(0.61e9), p4 = A(2.17e9);
    const A t0 = A(273.0), t1 = A(252.0), t2 = A(257.0), t3 = A(274.0), t4 = A(354.8);
    if (p <= p1) return t0 + (t1 - t0) * (p - p0) / (p1 - p0);
    else if (p > p1 && p <= p2) return t1 + (t2 - t1) * (p - p1) / (p2 - p1);
    else if (p > p2 && p <= p3) return t2 + (t3 - t2) * (p - p2) / (p3 - p2);
    else if (p > p3 && p <= p4) return t3 + (t4 - t3) * (p - p3) / (p4 - p3);
    return t4 * pow(((p - p4) / A(1.253e9)) + A(1), A(1.0 / 3.0));
}

// RockStrengthT (src/strength.c:697-722) with its cohesions, frictions and limits as arguments, so
// that the adjoint can differentiate with respect to them.
template <class A>
__host__ __device__ __forceinline__ A rock_strength_t(A pre, A dam, A dps, A temp, A yint0, A fint, A ylimint, A ydam0, A fdam,
                                             A ylimdam, const DevMat &s)
{
    A yint = y_lundborg<A>(pre, yint0, fint, ylimint);
    A ydam = y_drucker<A>(pre, ydam0, fdam, ylimdam);
    ydam = amin(yint, ydam);
    A tm = simon_melt<A>(pre, s);
    A soft = ohnaka_soft<A>(temp, s, tm);
    soft = awind(soft, A(0.0), A(1.0));
    A ymed = (ydam * dam + yint * (A(1.0) - dam)) * soft;
    A yvis = dps * A(s.melt_viscosity) * (A(1.0) - soft);
    return amax(ymed, yvis);
}

// The registry of src/strength.c:860-875 as one dispatcher, on the arithmetic type A. pa =
// {pressure, damage, plastic strain, strain rate, temperature, ...} (porosity uses its own six
// arguments); passed by value so that no caller keeps an array in local memory.
template <class A>
static __device__ __noinline__ A strength_fn(int id, A p0, A p1, A p2, A p3, A p4, A p5, const DevMat &s)
{
    const A pa[6] = {p0, p1, p2, p3, p4, p5};
    const A BETA = A(0.57735026918962576451);   // JohnsonCook factor as in interpolate_fn.h
    switch (id) {
    case 0: { // SimpleRock (never selectable in the reference: str2func rejects index 0)
        A yint = y_lundborg<A>(pa[0], A(s.Yint0), A(s.Yfricint), A(s.Ylimint));
        A ydam = y_drucker<A>(pa[0], A(s.Ydam0), A(s.Yfricdam), A(s.Ylimdam));
        ydam = amin(yint, ydam);
        return ydam * pa[1] + yint * (A(1.0) - pa[1]);
    }
    case 1: case 7: // SimpleShear / Ivanov damage increment
        return A(1.0) / amax(A(s.IvanA), A(s.IvanB) * (pa[0] - A(s.IvanC)));
    case 2: case 3: { // JohnsonCook1 / JohnsonCook2
        A ps = awind(pa[2], A(0.0), A(s.JCMaxPlastic));
        A y1 = A(s.JCA) + A(s.JCB) * pow(ps, A(s.JCN));
        A y2 = A(1.0);
        if (pa[3] > A(1.0) && s.JCC > 0.0) y2 = A(1.0) + A(s.JCC) * log(pa[3]);
        if (id == 3) return y1 * y2 * jnck_soft<A>(pa[4], pa[0], s) * BETA;
        return y1 * y2 * BETA;
    }
    case 4: // RockStrengthT
        return rock_strength_t<A>(pa[0], pa[1], pa[3], pa[4], A(s.Yint0), A(s.Yfricint), A(s.Ylimint), A(s.Ydam0),
                                  A(s.Yfricdam), A(s.Ylimdam), s);
    case 5: { // IceStrength
        A pre = pa[0], dam = pa[1], temp = pa[4];
        A yint = y_lundborg<A>(pre, A(s.Yint0), A(s.Yfricint), A(s.Ylimint));
        A ydam = y_lundborg<A>(pre, A(s.Ydam0), A(s.Yfricdam), A(s.Ylimdam));
        ydam = amin(yint, ydam);
        A tm = ice_melt<A>(pre);
        A soft = ohnaka_soft<A>(temp, s, tm);
        soft = awind(soft, A(0.0), A(1.0));
        return (ydam * dam + yint * (A(1.0) - dam)) * soft;
    }
    case 6: { // Collins damage increment
        A pre = pa[0], inc;
        if (pre < A(s.Pbd)) inc = amax(A(0.01), A(0.01) + A(0.04) * pre / A(s.Pbd));
        else if (pre < A(s.Pbp)) inc = A(0.05) + A(0.05) * (pre - A(s.Pbd)) / (A(s.Pbp) - A(s.Pbd));
        else inc = A(0.1) + A(0.5) * (pre - A(s.Pbp)) / A(s.Pbp);
        return A(1.0) / inc;
    }
    case 8: { // SimpleTensile
        A tm = simon_melt<A>(pa[0], s);
        A soft = ohnaka_soft<A>(pa[4], s, tm);
        soft = awind(soft, A(0.0), A(1.0));
        return A(s.Yten0) * (A(1.0) - pa[1]) * soft;
    }
    case 11: { // VonMises1
        A yint = A(s.Yint0), ydam = amin(yint, A(s.Ydam0));
        return ydam * pa[1] + yint * (A(1.0) - pa[1]);
    }
    case 12: { // VonMises2
        A yint = A(s.Yint0), ydam = amin(yint, A(s.Ydam0));
        A tm = simon_melt<A>(pa[0], s);
        A soft = awind(ohnaka_soft<A>(pa[4], s, tm), A(0.0), A(1.0));
        return (ydam * pa[1] + yint * (A(1.0) - pa[1])) * soft;
    }
    case 10: { // Wunnemann et al. (2006) epsilon-alpha porosity rate (src/strength.c:801-854)
        A pty = pa[0], cvs = pa[1], pre = pa[2], dcvs = pa[3], evx = pa[4], evy = pa[5];
        if (pty <= A(1.0) || pty > A(s.alphamax) || pre <= A(0.)) return A(0.);
        A v2 = evx * evx + evy * evy;
        if (v2 <= A(s.avel) * A(s.avel)) return A(0.);
        A cvs_c;
        if (pty > A(s.alphae)) cvs_c = A(s.epse0);
        else if (pty > A(s.alphax)) cvs_c = A(s.epse0) + log(pty / A(s.alphae)) / A(s.kappa);
        else cvs_c = A(s.epsec) - sqrt((pty - A(1.0)) / (A(s.alphax) - A(1.0))) * (A(s.epsec) - A(s.epsex));
        A ratio = A(1.0) + (A(s.chi) - A(1.0)) * fmax(A(0.0), fmin(A(1.0), (pty - A(1.0)) / (A(s.alphamax) - A(1.0))));
        A dade = pty * (A(1.0) - ratio * ratio);
        if (dcvs < A(0.) && cvs < cvs_c) {
            if (pty > A(s.alphax)) dade = A(s.kappa) * pty;
            else dade = sqrt((pty - A(1.)) / (A(s.alphax) - A(1.0))) * A(s.kappa) * A(s.alphax);
        } else {
            dade = pty * (A(1.0) - ratio * ratio);
        }
        return dade * dcvs;
    }
    case 9:
    default:
        return A(0.0);
    }
}

} // namespace salec
