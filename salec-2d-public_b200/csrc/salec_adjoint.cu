// Reverse (adjoint) sweeps of the mesh update, FP64.
//
// Each kernel reverses one forward sweep of salec_step.cu for the configuration the adjoint
// supports (one material beside vacuum, Tillotson EOS, RockStrengthT yield with Ivanov or
// SimpleShear damage, no damping layers, porosity, acoustic fluidisation, tensile failure,
// tracer lubrication or ejecta drag): given the forward state before the sweep (a.c) and the
// adjoints of the sweep's outputs (in a.b), it adds the adjoints of the sweep's inputs and
// clears those of the outputs it overwrote. A thread recomputes its point's forward values,
// branch by branch as the forward sweep took them, and applies the transposed local
// derivatives; adjoints of inputs at neighbouring points are added with atomics (the
// transpose of a gather is a scatter). The long scalar formulas get their local derivatives
// from forward-mode dual numbers (salec_dual.cuh) run over the step's own templated code.
//
// Discrete quantities carry no adjoint: void-corner counts, material flags, the cut-line
// corner distances e_wpt, the surface profile y_profile and the time step, which is frozen at
// the forward run's value (the derivatives are those of the step at the recorded dt). Fields
// that influence no other field in the supported configuration (plastic strain, vibration
// energy, ejecta fraction, cold volume strain, strain-rate and strength records) are left out.
#include "salec_adjoint.h"
#include "salec_dual.cuh"

namespace salec {

#define KIDX(i, j) ((long long)(i) + (long long)c.d.P * (long long)(j))
#define PLN(ptr, comp) ((ptr) + (long long)(comp) * c.d.PL)
#define GEO(g, comp) ((g).tab[(long long)(comp) * (g).plane + i + (long long)c.d.P * (g).row[j]])

namespace {

__device__ __forceinline__ bool a_cell_interior(const Ctx &c, int i, int j)
{
    return i >= 2 && i <= c.d.enx - 3 && j >= 2 && j <= c.d.eny - 3;
}
__device__ __forceinline__ bool a_vert_active(const Ctx &c, int i, int j)
{
    return i >= 1 && i <= c.d.vnx - 2 && j >= 1 && j <= c.d.vny - 2;
}
__device__ __forceinline__ bool a_vert_pad(const Ctx &c, int i, int j)
{
    int xd = min(i, c.d.vnx - 1 - i), yd = min(j, c.d.vny - 1 - j);
    return xd <= 1 || yd <= 1;
}

__device__ __forceinline__ void add(double *p, double v)
{
    if (v != 0.0) atomicAdd(p, v);
}

// warp-summed atomic add of a per-thread parameter gradient
__device__ __forceinline__ void add_theta(double *t, double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(t, v);
}

// derivative of sqrt(second_inv(x)) with respect to the four components, times g
__device__ __forceinline__ void second_inv_sqrt_adj(const double x[4], double root, double g, double out[4])
{
    if (!(root > 0.0)) { out[0] = out[1] = out[2] = out[3] = 0.0; return; }
    const double h = g / (2.0 * root);
    out[0] = h * (2.0 * x[0] - x[2] - x[3]) / 3.0;
    out[1] = h * 2.0 * x[1];
    out[2] = h * (2.0 * x[2] - x[0] - x[3]) / 3.0;
    out[3] = h * (2.0 * x[3] - x[2] - x[0]) / 3.0;
}

// ---------------------------------------------------------------- phase 1: vertex momentum
// update_v_vof + update_v_vel_inc (src/sale2d.c:751-791, 930-1049)
__global__ void ka_vertex_momentum(const AdjCtx a)
{
    const Ctx &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!a_vert_active(c, i, j)) return;
    const long long cl[4] = {KIDX(i - 1, j - 1), KIDX(i, j - 1), KIDX(i, j), KIDX(i - 1, j)};
    const long long p = KIDX(i, j);
    // vertex volume fractions: v_vof[m] = sum 0.25 m_vof[m]
    for (int m = 0; m < c.d.nmat; ++m) {
        const double g = PLN(a.b.v_vof, m)[p];
        if (g != 0.0)
            for (int k = 0; k < 4; ++k) add(PLN(a.b.m_vof, m) + cl[k], 0.25 * g);
        PLN(a.b.v_vof, m)[p] = 0.0;
    }
    // momentum: recompute the forward values
    const double old_x = c.f.v_vel[p], old_y = PLN(c.f.v_vel, 1)[p];
    const double m0 = c.f.v_mass[p];
    double inc_x = 0., inc_y = 0., vvol = 0., vmass = 0.;
    double lvk[4], rhok[4];
    bool use[4];
    for (int k = 0; k < 4; ++k) {
        const double rho = c.f.e_den[cl[k]];
        use[k] = !(rho < SALEC_TOLRHO);
        rhok[k] = rho;
        lvk[k] = GEO(c.g_v_vol, k + 1);
        if (!use[k]) continue;
        const double lv = lvk[k];
        vvol += lv;
        vmass += rho * lv;
        const double w = rho * lv;
        inc_x += w * c.f.e_dvel[cl[k]];
        inc_y += w * PLN(c.f.e_dvel, 1)[cl[k]];
    }
    const bool massive = vmass > SALEC_TOLRHO * vvol;
    double nx_ = 0., ny_ = 0., pa = 0., pb = 0.;
    if (massive) {
        pa = 1.0 / vmass;
        pb = m0 / vmass;
        nx_ = pa * inc_x + pb * old_x;
        ny_ = pa * inc_y + pb * old_y;
    }
    double vn = 0.;
    vn += nx_ * nx_;
    vn += ny_ * ny_;
    vn = sqrt(vn);
    double gx = a.b.v_vel[p], gy = PLN(a.b.v_vel, 1)[p];
    const double gm = a.b.v_mass[p];
    // |v| clamp and cut-off (on the norm before the clamp)
    if (vn < c.rp.velocity_min * 1) {
        gx = gy = 0.;
    } else if (vn > c.rp.velocity_max) {
        const double s = c.rp.velocity_max / vn;
        const double d = (gx * nx_ + gy * ny_) / (vn * vn);
        gx = s * (gx - nx_ * d);
        gy = s * (gy - ny_ * d);
    }
    double g_oldx = 0., g_oldy = 0., g_m0 = 0., g_incx = 0., g_incy = 0., g_vmass = 0.;
    if (massive) {
        g_incx = gx * pa;
        g_incy = gy * pa;
        g_oldx = gx * pb;
        g_oldy = gy * pb;
        g_m0 = (gx * old_x + gy * old_y) / vmass;
        g_vmass = -(gx * nx_ + gy * ny_) / vmass + gm;
    }
    for (int k = 0; k < 4; ++k) {
        if (!use[k]) continue;
        const double lv = lvk[k], w = rhok[k] * lv;
        const double dvx = c.f.e_dvel[cl[k]], dvy = PLN(c.f.e_dvel, 1)[cl[k]];
        const double gw = g_incx * dvx + g_incy * dvy;
        add(a.b.e_dvel + cl[k], g_incx * w);
        add(PLN(a.b.e_dvel, 1) + cl[k], g_incy * w);
        add(a.b.e_den + cl[k], g_vmass * lv + gw * lv);
    }
    a.b.v_vel[p] = g_oldx;
    PLN(a.b.v_vel, 1)[p] = g_oldy;
    a.b.v_mass[p] = g_m0;
    PLN(a.b.v_mass, 1)[p] = 0.0;
}

// ---------------------------------------------------------------- phase 3: cell velocity
// update_e_vel (src/sale2d.c:838-928)
__global__ void ka_cell_velocity(const AdjCtx a)
{
    const Ctx &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!a_cell_interior(c, i, j)) return;
    const long long p = KIDX(i, j);
    const double gx = a.b.e_vel[p], gy = PLN(a.b.e_vel, 1)[p];
    a.b.e_vel[p] = 0.0;
    PLN(a.b.e_vel, 1)[p] = 0.0;
    if (gx == 0.0 && gy == 0.0) return;
    const long long vl[4] = {KIDX(i, j), KIDX(i + 1, j), KIDX(i + 1, j + 1), KIDX(i, j + 1)};
    const double rho = c.f.e_den[p];
    if (rho < SALEC_TOLRHO) return;
    int vac = 0;
    double wpt[4];
    for (int k = 0; k < 4; ++k) {
        wpt[k] = PLN(c.f.e_wpt, k)[p];
        const double nvoid = PLN(c.f.v_mass, 1)[vl[k]];
        if (nvoid >= 4.0 || (nvoid >= 3.0 && wpt[k] < 0.)) vac++;
    }
    if (vac == 4) return;
    double ex = 0., ey = 0., sm = 0.;
    for (int k = 0; k < 4; ++k) {
        if (wpt[k] > 0.0) continue;
        const double mk = c.f.v_mass[vl[k]];
        ex += mk * c.f.v_vel[vl[k]];
        ey += mk * PLN(c.f.v_vel, 1)[vl[k]];
        sm += mk;
    }
    if (!(sm > 0.)) return;
    const double s = 1.0 / sm;
    ex *= s;
    ey *= s;
    for (int k = 0; k < 4; ++k) {
        if (wpt[k] > 0.0) continue;
        const double mk = c.f.v_mass[vl[k]];
        const double vx = c.f.v_vel[vl[k]], vy = PLN(c.f.v_vel, 1)[vl[k]];
        add(a.b.v_vel + vl[k], gx * mk * s);
        add(PLN(a.b.v_vel, 1) + vl[k], gy * mk * s);
        add(a.b.v_mass + vl[k], (gx * (vx - ex) + gy * (vy - ey)) * s);
    }
}

// ---------------------------------------------------------------- phase 4: void vertices
// check_v_vel (src/sale2d.c:1051-1142)
__global__ void ka_void_vertices(const AdjCtx a)
{
    const Ctx &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!a_vert_active(c, i, j)) return;
    const long long cl[4] = {KIDX(i - 1, j - 1), KIDX(i, j - 1), KIDX(i, j), KIDX(i - 1, j)};
    const int corner[4] = {2, 3, 0, 1};
    int void_cell = 0, void_corner = 0;
    for (int k = 0; k < 4; ++k) {
        if (c.f.e_den[cl[k]] < SALEC_TOLRHO) void_cell++;
        if (PLN(c.f.e_wpt, corner[k])[cl[k]] > 0.) void_corner++;
    }
    if (void_cell >= 4 || void_corner < 4) return;
    const long long p = KIDX(i, j);
    const double gx = a.b.v_vel[p], gy = PLN(a.b.v_vel, 1)[p];
    a.b.v_vel[p] = 0.0;
    PLN(a.b.v_vel, 1)[p] = 0.0;
    double ax = 0., ay = 0., ad = 0.;
    for (int k = 0; k < 4; ++k) {
        const double rho = c.f.e_den[cl[k]];
        if (rho < SALEC_TOLRHO) continue;
        ad += rho;
        ax += rho * c.f.e_vel[cl[k]];
        ay += rho * PLN(c.f.e_vel, 1)[cl[k]];
    }
    const double s = 1.0 / ad;
    const double vx = s * ax, vy = s * ay;
    for (int k = 0; k < 4; ++k) {
        const double rho = c.f.e_den[cl[k]];
        if (rho < SALEC_TOLRHO) continue;
        const double ex = c.f.e_vel[cl[k]], ey = PLN(c.f.e_vel, 1)[cl[k]];
        add(a.b.e_vel + cl[k], gx * rho * s);
        add(PLN(a.b.e_vel, 1) + cl[k], gy * rho * s);
        add(a.b.e_den + cl[k], (gx * (ex - vx) + gy * (ey - vy)) * s);
    }
}

// ---------------------------------------------------------------- phase 5: gradient, viscosity
// update_e_gradvel with the artificial viscosity (src/sale2d.c:1144-1236)
__device__ __forceinline__ void gradient_adj(const AdjCtx &a, int i, int j, double corner[8])
{
    const Ctx &c = a.c;
    const long long p = KIDX(i, j);
    double gd[5];
    for (int k = 0; k < 5; ++k) { gd[k] = PLN(a.b.e_grad_vel, k)[p]; PLN(a.b.e_grad_vel, k)[p] = 0.0; }
    double gdiv = a.b.e_div_vel[p];
    a.b.e_div_vel[p] = 0.0;
    const double gq = a.b.e_q[p];
    a.b.e_q[p] = 0.0;
    const long long vl[4] = {KIDX(i, j), KIDX(i + 1, j), KIDX(i + 1, j + 1), KIDX(i, j + 1)};
    double vx[4], vy[4], g[12];
    for (int k = 0; k < 4; ++k) { vx[k] = c.f.v_vel[vl[k]]; vy[k] = PLN(c.f.v_vel, 1)[vl[k]]; }
    for (int k = 0; k < 12; ++k) g[k] = GEO(c.g_e_grad, k);
    if (gq != 0.0) {
        double d0 = 0., d3 = 0., d4 = 0.;
        for (int k = 0; k < 4; ++k) d0 += g[k] * vx[k];
        for (int k = 0; k < 4; ++k) d3 += g[4 + k] * vy[k];
        for (int k = 0; k < 4; ++k) d4 += g[8 + k] * vx[k];
        const double div = d0 + d3 + d4;
        // a divergence that is zero to within the rounding of its terms (a body at rest or in
        // uniform motion) sits on the kink of the viscosity, min(0, div) below the TOLQPRE cut:
        // the derivative there is the average of the two sides, -rho ql / 2 and 0
        double dterms = 0.;
        for (int k = 0; k < 4; ++k) dterms += fabs(g[k] * vx[k]) + fabs(g[4 + k] * vy[k]) + fabs(g[8 + k] * vx[k]);
        const bool on_kink = fabs(div) <= 1e-12 * dterms;
        const double vof0 = c.f.m_vof[p];
        if (!(vof0 > SALEC_TOLVOF || c.f.e_pre[p] <= 0.0)) {
            double area = GEO(c.g_e_vol, 0) / c.f.e_pos[p];
            area = fabs(area);
            const double csd = c.f.e_csd[p], rho = c.f.e_den[p];
            const double ql = c.rp.avis1 * csd * sqrt(area);
            const double qq = c.rp.avis2 * div * area;
            const double q = dmin(0., div) * rho * (qq - ql);
            if (on_kink) {
                gdiv += gq * (-0.5 * rho * ql);
            } else if (!(q < SALEC_TOLQPRE) && div < 0.) {
                gdiv += gq * (rho * (qq - ql) + div * rho * c.rp.avis2 * area);
                a.b.e_den[p] += gq * div * (qq - ql);
                a.b.e_csd[p] += gq * (-div * rho * c.rp.avis1 * sqrt(area));
            }
        }
    }
    gd[0] += gdiv;
    gd[3] += gdiv;
    gd[4] += gdiv;
    for (int k = 0; k < 4; ++k) {
        corner[2 * k] = g[k] * gd[0] + g[4 + k] * gd[1] + g[8 + k] * gd[4];
        corner[2 * k + 1] = g[k] * gd[2] + g[4 + k] * gd[3];
    }
}

// the vertex-velocity adjoints go to the corner scratch of the cell (planes 2k, 2k+1 for corner
// k); ka_corner_sum adds them up per vertex, without atomics
__global__ void ka_gradient(const AdjCtx a)
{
    const Ctx &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.d.enx || j >= c.d.eny) return;
    double corner[8] = {0., 0., 0., 0., 0., 0., 0., 0.};
    if (a_cell_interior(c, i, j)) gradient_adj(a, i, j, corner);
    const long long p = KIDX(i, j);
#pragma unroll
    for (int q = 0; q < 8; ++q) a.scr[q * c.d.PL + p] = corner[q];
}

// vertex (I, J) is corner 0 of cell (I, J), 1 of (I-1, J), 2 of (I-1, J-1), 3 of (I, J-1): the
// sum of their corner scratch (planes first + 2k + comp) is added to dst's two components
__global__ void ka_corner_sum(const AdjCtx a, double *dst, int first)
{
    const Ctx &c = a.c;
    const int I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y;
    if (I >= c.d.vnx || J >= c.d.vny) return;
    const long long PL = c.d.PL;
    const bool in_x = I < c.d.enx, in_y = J < c.d.eny, lo_x = I >= 1, lo_y = J >= 1;
#pragma unroll
    for (int comp = 0; comp < 2; ++comp) {
        const double *s = a.scr + (long long)(first + comp) * PL;
        double v = 0.;
        if (in_x && in_y) v += s[KIDX(I, J)];
        if (lo_x && in_y) v += s[2 * PL + KIDX(I - 1, J)];
        if (lo_x && lo_y) v += s[4 * PL + KIDX(I - 1, J - 1)];
        if (in_x && lo_y) v += s[6 * PL + KIDX(I, J - 1)];
        if (v != 0.0) dst[comp * PL + KIDX(I, J)] += v;
    }
}

// ---------------------------------------------------------------- phase 7: stress, strength, damage
// update_e_stress (src/strength.c:7-349) with RockStrengthT (:697-722) and Ivanov damage
// (:470-503); theta: d/d Yint0, Yfricint, Ydam0, Yfricdam
__global__ void ka_stress(const AdjCtx a)
{
    const Ctx &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    double th[4] = {0., 0., 0., 0.};
    if (a_cell_interior(c, i, j)) {
        const long long p = KIDX(i, j);
        const double dt = c.scal->dt;
        const double vof0 = c.f.m_vof[p];
        if (vof0 > SALEC_TOLVOF) {
            for (int q = 0; q < 4; ++q) PLN(a.b.e_ste, q)[p] = 0.0;
            a.b.e_ste2s[p] = 0.0;
        } else {
            const double vm = PLN(c.f.m_vof, 1)[p];
            const bool vm_on = !(vm < SALEC_TOLVOF);
            const DevMat &s = c.mat[1];
            const double rho = c.f.e_den[p];
            const double vapor_ref = vm_on ? vm * s.VaporDen : 0.0, melt_ref = vm_on ? vm * s.MeltDen : 0.0;
            if (rho <= vapor_ref || rho <= melt_ref) {
                // vapour or melt: stress, its invariant and the damage are set, not updated
                for (int q = 0; q < 4; ++q) PLN(a.b.e_ste, q)[p] = 0.0;
                a.b.e_ste2s[p] = 0.0;
                a.b.e_dam[p] = 0.0;
            } else {
                const double s_in[4] = {c.f.e_ste[p], PLN(c.f.e_ste, 1)[p], PLN(c.f.e_ste, 2)[p], PLN(c.f.e_ste, 3)[p]};
                const double ste2s_old = c.f.e_ste2s[p];
                const double dam_in = c.f.e_dam[p];
                const double g0 = c.f.e_grad_vel[p], g1 = PLN(c.f.e_grad_vel, 1)[p], g2 = PLN(c.f.e_grad_vel, 2)[p],
                             g3 = PLN(c.f.e_grad_vel, 3)[p], g4 = PLN(c.f.e_grad_vel, 4)[p];
                const double mu = c.f.e_mu[p], pre = c.f.e_pre[p], tem = c.f.e_tem[p];
                // forward, as k_stress computes it
                double e[4] = {g0, 0.5 * g1 + 0.5 * g2, g3, g4};
                const double tr = e[0] + e[2] + e[3];
                e[0] -= tr / 3.0;
                e[2] -= tr / 3.0;
                e[3] -= tr / 3.0;
                double sin2o_raw = (g2 - g1) * dt;
                const double sn = wind(sin2o_raw, -1., 1.);
                const double rt = sqrt(1.0 - sn * sn);
                const double cs = rt - 1.0;
                const double ss2 = (s_in[0] - s_in[2]) / 2.0;
                double se[4];
                se[0] = s_in[0] + 1.0 * (ss2 * cs + s_in[1] * sn);
                se[1] = s_in[1] + 1.0 * (s_in[1] * cs - ss2 * sn);
                se[2] = s_in[2] + 1.0 * (-ss2 * cs - s_in[1] * sn);
                se[3] = s_in[3] + 1.0 * 0.0;
                const double k2 = 2.0 * mu * dt;
                for (int q = 0; q < 4; ++q) se[q] += k2 * e[q];
                const double ste2s_e = sqrt(second_inv(se[0], se[1], se[2], se[3]));
                const double sta2s_e = sqrt(second_inv(e[0], e[1], e[2], e[3]));
                // yield strength on dual numbers: pre, dam, strain rate, temperature, Yint0, Yfricint,
                // Ydam0, Yfricdam
                using D = Dual<8>;
                const D my = rock_strength_t<D>(D::seed(pre, 0), D::seed(dam_in, 1), D::seed(sta2s_e, 2), D::seed(tem, 3),
                                                D::seed(s.Yint0, 4), D::seed(s.Yfricint, 5), D(s.Ylimint),
                                                D::seed(s.Ydam0, 6), D::seed(s.Yfricdam, 7), D(s.Ylimdam), s);
                const double shear = vm_on ? vm * dmax(my.v, 0.0) : 0.0;
                const bool yield = shear < ste2s_e;
                double gs_out[4];
                for (int q = 0; q < 4; ++q) gs_out[q] = PLN(a.b.e_ste, q)[p];
                const double gss = a.b.e_ste2s[p], gdam = a.b.e_dam[p];
                double gs_e[4], gste2s_e = 0., gsta2s_e = 0., gshear = 0., gvm = 0., gpre = 0., gdam_in = 0., gtem = 0.;
                double gste2s_old = 0.;
                if (yield) {
                    double M = (ste2s_e - ste2s_old) / (ste2s_e - shear);
                    const bool Mr = !(0.5 > M);
                    M = dmax(0.5, M);
                    const double sta2s_c = sta2s_e / M;
                    const double sfac = shear / ste2s_e;
                    const DevMat &sd = s;
                    const double ivb = sd.IvanB * (pre - sd.IvanC);
                    const double inc = 1.0 / dmax(sd.IvanA, ivb);
                    const double dsd = vm * inc;
                    const double x = dam_in + sta2s_c * dsd * dt;
                    const double gx = (x >= 0.0 && x <= 1.0) ? gdam : 0.0;
                    gdam_in += gx;
                    const double gsta2s_c = gx * dsd * dt;
                    const double gdsd = gx * sta2s_c * dt;
                    gvm += gdsd * inc;
                    if (ivb > sd.IvanA) gpre += gdsd * vm * (-sd.IvanB / (ivb * ivb));
                    double gsfac = 0.;
                    for (int q = 0; q < 4; ++q) { gsfac += gs_out[q] * se[q]; gs_e[q] = gs_out[q] * sfac; }
                    gshear += gss;
                    gshear += gsfac / ste2s_e;
                    gste2s_e += -gsfac * shear / (ste2s_e * ste2s_e);
                    gsta2s_e += gsta2s_c / M;
                    const double gM = -gsta2s_c * sta2s_e / (M * M);
                    if (Mr) {
                        const double den = ste2s_e - shear;
                        gste2s_e += gM * (ste2s_old - shear) / (den * den);
                        gste2s_old = -gM / den;
                        gshear += gM * (ste2s_e - ste2s_old) / (den * den);
                    }
                } else {
                    for (int q = 0; q < 4; ++q) gs_e[q] = gs_out[q];
                    gste2s_e = gss;
                    gdam_in += gdam;
                }
                // shear = vm * max(my, 0), my on dual numbers
                if (vm_on && my.v > 0.0 && gshear != 0.0) {
                    gvm += gshear * my.v;
                    const double gmy = gshear * vm;
                    gpre += gmy * my.d[0];
                    gdam_in += gmy * my.d[1];
                    gsta2s_e += gmy * my.d[2];
                    gtem += gmy * my.d[3];
                    th[0] += gmy * my.d[4];
                    th[1] += gmy * my.d[5];
                    th[2] += gmy * my.d[6];
                    th[3] += gmy * my.d[7];
                }
                // invariants
                double t4[4];
                second_inv_sqrt_adj(se, ste2s_e, gste2s_e, t4);
                for (int q = 0; q < 4; ++q) gs_e[q] += t4[q];
                double ge[4];
                second_inv_sqrt_adj(e, sta2s_e, gsta2s_e, ge);
                // se = s_rot + k2 e
                double gk2 = 0.;
                for (int q = 0; q < 4; ++q) { gk2 += gs_e[q] * e[q]; ge[q] += gs_e[q] * k2; }
                const double gmu = gk2 * 2.0 * dt;
                // Wilkins rotation
                const double gss2 = gs_e[0] * cs - gs_e[1] * sn - gs_e[2] * cs;
                double gs_in[4];
                gs_in[1] = gs_e[1] + gs_e[0] * sn + gs_e[1] * cs - gs_e[2] * sn;
                gs_in[0] = gs_e[0] + 0.5 * gss2;
                gs_in[2] = gs_e[2] - 0.5 * gss2;
                gs_in[3] = gs_e[3];
                const double gcs = gs_e[0] * ss2 + gs_e[1] * s_in[1] - gs_e[2] * ss2;
                double gsn = gs_e[0] * s_in[1] - gs_e[1] * ss2 - gs_e[2] * s_in[1];
                if (rt > 0.0) gsn += gcs * (-sn / rt);
                double gg[5] = {0., 0., 0., 0., 0.};
                if (sin2o_raw > -1.0 && sin2o_raw < 1.0) { gg[2] += gsn * dt; gg[1] -= gsn * dt; }
                // deviatoric strain rate
                const double ges = ge[0] + ge[2] + ge[3];
                gg[0] += ge[0] - ges / 3.0;
                gg[3] += ge[2] - ges / 3.0;
                gg[4] += ge[3] - ges / 3.0;
                gg[1] += 0.5 * ge[1];
                gg[2] += 0.5 * ge[1];
                for (int q = 0; q < 4; ++q) PLN(a.b.e_ste, q)[p] = gs_in[q];
                a.b.e_ste2s[p] = gste2s_old;
                a.b.e_dam[p] = gdam_in;
                for (int k = 0; k < 5; ++k) PLN(a.b.e_grad_vel, k)[p] += gg[k];
                a.b.e_mu[p] += gmu;
                a.b.e_pre[p] += gpre;
                a.b.e_tem[p] += gtem;
                PLN(a.b.m_vof, 1)[p] += gvm;
            }
        }
    }
    for (int k = 0; k < 4; ++k) add_theta(a.theta + k, th[k]);
}

// ---------------------------------------------------------------- phase 8: vertex acceleration
// calculate_acc_default (src/velocity.c:9-156)
__global__ void ka_acceleration(const AdjCtx a)
{
    const Ctx &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!a_vert_active(c, i, j)) return;
    const long long p = KIDX(i, j);
    double gax = a.b.v_acc[p], gay = PLN(a.b.v_acc, 1)[p];
    a.b.v_acc[p] = 0.0;
    PLN(a.b.v_acc, 1)[p] = 0.0;
    if (gax == 0.0 && gay == 0.0) return;
    const long long cl[4] = {KIDX(i - 1, j - 1), KIDX(i, j - 1), KIDX(i, j), KIDX(i - 1, j)};
    double ax = 0., ay = 0., vmass = 0., vvol = 0.;
    double sub[4];
    for (int k = 0; k < 4; ++k) sub[k] = GEO(c.g_v_subvol, k);
    for (int k = 0; k < 4; ++k) {
        const long long e = cl[k];
        const double sfx = GEO(c.g_v_suf, 2 * k), sfy = GEO(c.g_v_suf, 2 * k + 1);
        const double lp = c.f.e_pre[e] + c.f.e_q[e];
        const double sxx = c.f.e_ste[e], sxz = PLN(c.f.e_ste, 1)[e], szz = PLN(c.f.e_ste, 2)[e],
                     sth = PLN(c.f.e_ste, 3)[e];
        double fpx = 0., fpy = 0.;
        fpx += lp * sfx;
        fpy += lp * sfy;
        fpx += sub[k] * lp;
        double fsx = 0., fsy = 0.;
        fsx += sfx * sxx; fsx += sfy * sxz;
        fsy += sfx * sxz; fsy += sfy * szz;
        fsx += sub[k] * sth;
        ax += -1.0 * fsx; ay += -1.0 * fsy;
        ax += 1.0 * fpx; ay += 1.0 * fpy;
        const double lv = GEO(c.g_v_vol, 1 + k);
        vmass += lv * c.f.e_den[e];
        vvol += lv;
    }
    double ancx = 0., ancy = 0., lvx = 0., lvy = 0., sc = 0.;
    const bool lap = (c.lap_mask[(long long)j * (c.d.P >> 5) + (i >> 5)] >> (i & 31)) & 1u;
    bool anc_on = !a_vert_pad(c, i, j) && lap;
    if (anc_on) {
        int k = 0;
        for (int dj = -1; dj <= 1; ++dj)
            for (int di = -1; di <= 1; ++di, ++k) {
                const long long q = KIDX(i + di, j + dj);
                const double w = PLN(c.f.v_laplace, k)[p];
                lvx += w * c.f.v_vel[q];
                lvy += w * PLN(c.f.v_vel, 1)[q];
            }
        sc = 5.0e3 * sqrt(fabs(sub[0]) + fabs(sub[2]));
        ancx = sc * lvx;
        ancy = sc * lvy;
    }
    if (PLN(c.f.v_mass, 1)[p] >= 1.) { ancx = 0.; ancy = 0.; anc_on = false; }
    if (!(vmass > SALEC_TOLRHO * vvol)) return;   // the acceleration is set to zero there
    const double s = 1.0 / vmass;
    double fx = ax * s + 1.0 * c.f.v_bf[p] + c.rp.anc * ancx;
    double fy = ay * s + 1.0 * PLN(c.f.v_bf, 1)[p] + c.rp.anc * ancy;
    if (fabs(fx) < c.rp.acceleration_min * 1) gax = 0.;
    if (fabs(fy) < c.rp.acceleration_min * 1) gay = 0.;
    const double gFx = gax * s, gFy = gay * s;
    const double gvmass = -(gax * ax + gay * ay) * s * s;
    if (anc_on) {
        const double glx = gax * c.rp.anc * sc, gly = gay * c.rp.anc * sc;
        int k = 0;
        for (int dj = -1; dj <= 1; ++dj)
            for (int di = -1; di <= 1; ++di, ++k) {
                const long long q = KIDX(i + di, j + dj);
                const double w = PLN(c.f.v_laplace, k)[p];
                add(a.b.v_vel + q, glx * w);
                add(PLN(a.b.v_vel, 1) + q, gly * w);
            }
    }
    for (int k = 0; k < 4; ++k) {
        const long long e = cl[k];
        const double sfx = GEO(c.g_v_suf, 2 * k), sfy = GEO(c.g_v_suf, 2 * k + 1);
        const double glp = gFx * (sfx + sub[k]) + gFy * sfy;
        add(a.b.e_pre + e, glp);
        add(a.b.e_q + e, glp);
        add(a.b.e_ste + e, -gFx * sfx);
        add(PLN(a.b.e_ste, 1) + e, -gFx * sfy - gFy * sfx);
        add(PLN(a.b.e_ste, 2) + e, -gFy * sfy);
        add(PLN(a.b.e_ste, 3) + e, -gFx * sub[k]);
        add(a.b.e_den + e, gvmass * GEO(c.g_v_vol, 1 + k));
    }
}

// ---------------------------------------------------------------- phase 9: vertex displacement
// calculate_v_dis (src/sale2d.c:1238-1268)
__global__ void ka_displacement(const AdjCtx a)
{
    const Ctx &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!a_vert_active(c, i, j)) return;
    const long long p = KIDX(i, j);
    const double dt = c.scal->dt, hdt2 = 0.5 * dt * dt;
    for (int k = 0; k < 2; ++k) {
        const double gdis = PLN(a.b.v_dis, k)[p], gvel = PLN(a.b.v_vel, k)[p];
        PLN(a.b.v_vel, k)[p] = gvel + dt * gdis;
        PLN(a.b.v_acc, k)[p] += dt * gvel + hdt2 * gdis;
        PLN(a.b.v_dis, k)[p] = 0.0;
    }
}

// ---------------------------------------------------------------- phase 10: internal energy
// update_energy (src/sale2d.c:564-712)
__global__ void ka_energy(const AdjCtx a)
{
    const Ctx &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!a_cell_interior(c, i, j)) return;
    const long long p = KIDX(i, j);
    if (c.f.m_vof[p] > SALEC_TOLVOF || c.f.e_den[p] < SALEC_TOLRHO) return;
    const double vm = PLN(c.f.m_vof, 1)[p], rm = PLN(c.f.m_den, 1)[p], em = PLN(c.f.m_eng, 1)[p];
    const double ge = PLN(a.b.m_eng, 1)[p];
    if (vm <= SALEC_TOLVOF || rm <= SALEC_TOLRHO) { PLN(a.b.m_eng, 1)[p] = 0.0; return; }
    const double dt = c.scal->dt;
    const double pre = c.f.e_pre[p], q = c.f.e_q[p], div = c.f.e_div_vel[p];
    double g[5], s[4];
    for (int k = 0; k < 5; ++k) g[k] = PLN(c.f.e_grad_vel, k)[p];
    for (int k = 0; k < 4; ++k) s[k] = PLN(c.f.e_ste, k)[p];
    const double lp = pre + q;
    const double dE_pre = -lp * div;
    const double dE_ste = s[0] * g[0] + s[1] * (g[1] + g[2]) + s[2] * g[3] + s[3] * g[4];
    const double x = em + (dE_pre + dE_ste) * dt * 1.0;
    if (0. > x) { PLN(a.b.m_eng, 1)[p] = 0.0; return; }
    const double gd = ge * dt;
    a.b.e_pre[p] += -gd * div;
    a.b.e_q[p] += -gd * div;
    a.b.e_div_vel[p] += -gd * lp;
    PLN(a.b.e_ste, 0)[p] += gd * g[0];
    PLN(a.b.e_ste, 1)[p] += gd * (g[1] + g[2]);
    PLN(a.b.e_ste, 2)[p] += gd * g[3];
    PLN(a.b.e_ste, 3)[p] += gd * g[4];
    PLN(a.b.e_grad_vel, 0)[p] += gd * s[0];
    PLN(a.b.e_grad_vel, 1)[p] += gd * s[1];
    PLN(a.b.e_grad_vel, 2)[p] += gd * s[1];
    PLN(a.b.e_grad_vel, 3)[p] += gd * s[2];
    PLN(a.b.e_grad_vel, 4)[p] += gd * s[3];
}

// ---------------------------------------------------------------- phase 12: face fluxes
// calculate_flux_mixed (src/advect.c:861-1223), interior and pad cells alike
__device__ __forceinline__ void swept_volume_adj(double xa, double ya, double xb, double yb, double dxa, double dya,
                                                 double dxb, double dyb, double g, double out[4])
{
    using D = Dual<4>;
    const D v = swept_volume<D>(xa, ya, xb, yb, D::seed(dxa, 0), D::seed(dya, 1), D::seed(dxb, 2), D::seed(dyb, 3));
    for (int k = 0; k < 4; ++k) out[k] = g * v.d[k];
}

// corner[2k + comp]: adjoint of v_dis at corner k; corner[8 + 2k + m]: adjoint of v_vof[m] there.
// CUT selects the cells with a cut line (primary fraction below 1 - TOLVOF); the others take the
// light instance, which holds none of the cut line's registers.
template <bool CUT>
__device__ __forceinline__ void flux_adj(const AdjCtx &a, int i, int j, double corner[16])
{
    const Ctx &c = a.c;
    const long long p = KIDX(i, j);
    double vof[2] = {c.f.m_vof[p], PLN(c.f.m_vof, 1)[p]};
    int prim = 0;
    double vprim = vof[0];
    if (vof[0] < SALEC_TOLVOF && vof[1] > vprim) { prim = 1; vprim = vof[1]; }
    const bool full = vprim > 1.0 - SALEC_TOLVOF;
    if (full == CUT) return;
    const long long vl[4] = {KIDX(i, j), KIDX(i + 1, j), KIDX(i + 1, j + 1), KIDX(i, j + 1)};
    double px[4], py[4], dx[4], dy[4];
    for (int k = 0; k < 4; ++k) {
        px[k] = c.f.v_pos[vl[k]]; py[k] = PLN(c.f.v_pos, 1)[vl[k]];
        dx[k] = c.f.v_dis[vl[k]]; dy[k] = PLN(c.f.v_dis, 1)[vl[k]];
    }
    // faces l, b, r, u with their vertex pairs (a, b) as in k_flux
    const int fa[4] = {0, 1, 2, 3}, fb[4] = {3, 0, 1, 2};
    double vol[4];
    for (int k = 0; k < 4; ++k)
        vol[k] = swept_volume(px[fa[k]], py[fa[k]], px[fb[k]], py[fb[k]], dx[fa[k]], dy[fa[k]], dx[fb[k]], dy[fb[k]]);
    double *bface[4] = {a.b.bx_phi + KIDX(i, j), a.b.by_phi + KIDX(i, j), a.b.bx_phi + KIDX(i + 1, j),
                        a.b.by_phi + KIDX(i, j + 1)};
    const long long PL = c.d.PL;
    const int nmat = 2;
    // adjoints of the records this cell writes (donor faces); the copied state members go to
    // the cell's own state
    // adjoints of the material volumes of the records this cell writes (donor faces), by material;
    // the copied state members go to the cell's own state
    double g0[4] = {0., 0., 0., 0.}, g1[4] = {0., 0., 0., 0.};
    bool any = false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (vol[k] <= 0.) {
            double *f = bface[k];
            g0[k] = f[0];
            g1[k] = f[PL];
            f[0] = 0.0;
            f[PL] = 0.0;
            if (vol[k] < 0.) {
#pragma unroll
                for (int m = 0; m < nmat; ++m) {
                    const double gr = f[(m + nmat) * PL], gen = f[(m + 2 * nmat) * PL];
                    f[(m + nmat) * PL] = 0.0;
                    f[(m + 2 * nmat) * PL] = 0.0;
                    if (gr != 0.0) PLN(a.b.m_den, m)[p] += gr;
                    if (gen != 0.0) PLN(a.b.m_eng, m)[p] += gen;
                }
                const int b = 3 * nmat;
                a.b.e_vel[p] += f[(b + 0) * PL];
                PLN(a.b.e_vel, 1)[p] += f[(b + 1) * PL];
#pragma unroll
                for (int q = 0; q < 4; ++q) PLN(a.b.e_ste, q)[p] += f[(b + 2 + q) * PL];
                a.b.e_dam[p] += f[(b + 6) * PL];
#pragma unroll
                for (int q = 0; q < 10; ++q) f[(b + q) * PL] = 0.0;
                any = true;
            }
        }
    }
    if (!any) return;
    // forward flux of this cell; the arrays are kept per role (primary P, other O) so that no
    // local array is indexed by the run-time material number
    const double evol = c.f.e_vol[p];
    const bool p1 = prim == 1;
    const int other = 1 - prim;
    const double vother = p1 ? vof[0] : vof[1];
    const double sg[4] = {1.0, 1.0, -1.0, -1.0};
    double mv[4], gP[4], gO[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        mv[k] = dmin(vol[k], 0.0);
        gP[k] = p1 ? g1[k] : g0[k];
        gO[k] = p1 ? g0[k] : g1[k];
    }
    double fP[4], fO[4], fpv[4] = {1., 1., 1., 1.}, fnp[4] = {0., 0., 0., 0.};
    Dual<5> fpd[4];
    bool fnp_ratio[4] = {false, false, false, false};
    if (!CUT) {
#pragma unroll
        for (int k = 0; k < 4; ++k) { fP[k] = sg[k] * mv[k]; fO[k] = 0.0; }
    } else {
        // cut line of the primary material on dual numbers over its four vertex fractions and its
        // cell fraction
        using D = Dual<5>;
        const double *vvp = PLN(c.f.v_vof, prim);
        D vq[4];
        for (int k = 0; k < 4; ++k) vq[k] = D::seed(vvp[vl[k]], k);
        const D vpd = D::seed(vprim, 4);
        double grd[8];
        for (int k = 0; k < 8; ++k) grd[k] = GEO(c.g_e_grad, k);
        D gx(0.), gy(0.);
        for (int k = 0; k < 4; ++k) gx += vq[k] * grd[k];
        for (int k = 0; k < 4; ++k) gy += vq[k] * grd[4 + k];
        normalise2(gx, gy);
        // a cut line parallel to a mesh line up to the rounding of the fraction gradient (a
        // component of about 1e-16) sits on the kinks of |n| and of the corner maximum, which a
        // perturbation of the fractions crosses: it is put on them, so that the derivatives are
        // the averages of both sides
        snap_zero(gx, 1e-12);
        snap_zero(gy, 1e-12);
        D ca = PLN(c.f.e_pos, 2)[p] * fabs(gx);
        D cb = PLN(c.f.e_pos, 3)[p] * fabs(gy);
        if (ca < cb) { D t = ca; ca = cb; cb = t; }
        const D dstar = cut_length(vpd, ca, cb);
        D lw[4];
        for (int k = 0; k < 4; ++k) { D s(0.); s += gx * px[k]; s += gy * py[k]; lw[k] = s; }
        // dmax(dmax(l0, l1), dmax(l2, l3)) as the step forms it; ties (a horizontal or vertical cut
        // line has two equal corners), to rounding, take the average of the one-sided derivatives
        double lmax = 0.;
        for (int k = 0; k < 4; ++k) lmax = dmax(lmax, fabs(lw[k].v));
        const double ltol = 1e-12 * lmax;
        const D mw = fmax_near(fmax_near(lw[0], lw[1], ltol), fmax_near(lw[2], lw[3], ltol), ltol);
        for (int k = 0; k < 4; ++k) lw[k] = lw[k] - mw + dstar;
        fpd[0] = face_ratio(lw[3], lw[0]);
        fpd[2] = face_ratio(lw[2], lw[1]);
        fpd[1] = face_ratio(lw[0], lw[1]);
        fpd[3] = face_ratio(lw[3], lw[2]);
        for (int k = 0; k < 4; ++k) fpv[k] = fpd[k].v;
        // fractions of the other material: with one material beside vacuum, the MSTACS
        // fraction divided by its own sum is 1 where that sum exceeds TOLVOF, else the content
        // ratio
        if (!p1) {
            double cr = dmin(vol[0], 0.0) + dmin(vol[2], 0) + dmin(vol[1], 0) + dmin(vol[3], 0);
            cr = fabs(cr) / evol;
            const double *vvo = PLN(c.f.v_vof, other);
            double ngx = 0., ngy = 0.;
            for (int k = 0; k < 4; ++k) ngx += vvo[vl[k]] * grd[k];
            for (int k = 0; k < 4; ++k) ngy += vvo[vl[k]] * grd[4 + k];
            normalise2(ngx, ngy);
            long long nb[4] = {KIDX(i - 1, j), KIDX(i, j - 1), KIDX(i + 1, j), KIDX(i, j + 1)};
            if (i - 1 < 0) nb[0] = p;
            if (j - 1 < 0) nb[1] = p;
            if (i + 1 >= c.d.enx) nb[2] = p;
            if (j + 1 >= c.d.eny) nb[3] = p;
            const long long fbn[4] = {KIDX(i, j), KIDX(i, j), KIDX(i + 1, j), KIDX(i, j + 1)};
            double fnx[4], fny[4];
            fnx[0] = c.f.bx_normal[fbn[0]]; fny[0] = PLN(c.f.bx_normal, 1)[fbn[0]];
            fnx[2] = c.f.bx_normal[fbn[2]]; fny[2] = PLN(c.f.bx_normal, 1)[fbn[2]];
            fnx[1] = c.f.by_normal[fbn[1]]; fny[1] = PLN(c.f.by_normal, 1)[fbn[1]];
            fnx[3] = c.f.by_normal[fbn[3]]; fny[3] = PLN(c.f.by_normal, 1)[fbn[3]];
            const double *ev = PLN(c.f.m_vof, other);
            const double up[4] = {ev[nb[0]], ev[nb[1]], ev[nb[2]], ev[nb[3]]};
            const double ac[4] = {up[2], up[3], up[0], up[1]};
            for (int k = 0; k < 4; ++k) {
                const double ar = algebraic_ratio(up[k], vother, ac[k], cr, fnx[k], fny[k], ngx, ngy);
                if (ar > SALEC_TOLVOF) fnp[k] = ar / ar;
                else { fnp[k] = vother / (1.0 - vprim); fnp_ratio[k] = true; }
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            fP[k] = sg[k] * mv[k] * fpv[k];
            fO[k] = sg[k] * mv[k] * (1.0 - fpv[k]) * fnp[k];
        }
    }
    // the content cap of material 1
    double gvP = 0., gvO = 0.;
    {
        double F1[4], G1[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) { F1[k] = p1 ? fP[k] : fO[k]; G1[k] = p1 ? gP[k] : gO[k]; }
        double d = 0.;
        d += F1[0] * 1.0; d += F1[1] * 1.0; d += F1[2] * -1.0; d += F1[3] * -1.0;
        const double out = -1.0 * d;
        if (out > vof[1] * evol) {
            const double s = vof[1] * evol / out;
            double G = 0.;
#pragma unroll
            for (int k = 0; k < 4; ++k) G += G1[k] * F1[k];
            const double gout = -G * s / out;
            const double dout[4] = {-1.0, -1.0, 1.0, 1.0};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const double gk = G1[k] * s + gout * dout[k];
                if (p1) gP[k] = gk;
                else gO[k] = gk;
            }
            if (p1) gvP += G * evol / out;
            else gvO += G * evol / out;
        }
    }
    // back through the flux formulas to the swept volumes and the cut line
    double gvol[4] = {0., 0., 0., 0.};
    if (!CUT) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (vol[k] < 0.) gvol[k] += gP[k] * sg[k];
    } else {
        double gfp[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double gmv = sg[k] * (gP[k] * fpv[k] + gO[k] * (1.0 - fpv[k]) * fnp[k]);
            if (vol[k] < 0.) gvol[k] += gmv;
            gfp[k] = sg[k] * mv[k] * (gP[k] - gO[k] * fnp[k]);
            if (!p1 && fnp_ratio[k]) {
                const double gfn = sg[k] * mv[k] * (1.0 - fpv[k]) * gO[k];
                gvO += gfn / (1.0 - vprim);
                gvP += gfn * vother / ((1.0 - vprim) * (1.0 - vprim));
            }
        }
        double gvq[5] = {0., 0., 0., 0., 0.};
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int q = 0; q < 5; ++q) gvq[q] += gfp[k] * fpd[k].d[q];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (prim == 0) corner[8 + 2 * k] = gvq[k];
            else corner[9 + 2 * k] = gvq[k];
        }
        gvP += gvq[4];
    }
    {
        const double gv0 = p1 ? gvO : gvP, gv1 = p1 ? gvP : gvO;
        if (gv0 != 0.0) a.b.m_vof[p] += gv0;
        if (gv1 != 0.0) PLN(a.b.m_vof, 1)[p] += gv1;
    }
    double gd[4][2] = {{0., 0.}, {0., 0.}, {0., 0.}, {0., 0.}};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (gvol[k] == 0.0) continue;
        double o[4];
        swept_volume_adj(px[fa[k]], py[fa[k]], px[fb[k]], py[fb[k]], dx[fa[k]], dy[fa[k]], dx[fb[k]], dy[fb[k]],
                         gvol[k], o);
        gd[fa[k]][0] += o[0]; gd[fa[k]][1] += o[1];
        gd[fb[k]][0] += o[2]; gd[fb[k]][1] += o[3];
    }
    for (int k = 0; k < 4; ++k) {
        corner[2 * k] = gd[k][0];
        corner[2 * k + 1] = gd[k][1];
    }
}

// the light instance writes every cell's corner scratch (zeros for cut cells), the cut instance
// then overwrites the cut cells'
template <bool CUT>
__global__ void __launch_bounds__(128, CUT ? 1 : 5) ka_flux(const AdjCtx a)
{
    const Ctx &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.d.enx || j >= c.d.eny) return;
    const long long p = KIDX(i, j);
    if (CUT) {
        const double v0 = c.f.m_vof[p], v1 = PLN(c.f.m_vof, 1)[p];
        const double vprim = (v0 < SALEC_TOLVOF && v1 > v0) ? v1 : v0;
        if (vprim > 1.0 - SALEC_TOLVOF) return;
    }
    double corner[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) corner[q] = 0.;
    flux_adj<CUT>(a, i, j, corner);
#pragma unroll
    for (int q = 0; q < 16; ++q) a.scr[q * c.d.PL + p] = corner[q];
}

// ---------------------------------------------------------------- phase 14: remap and EOS
// advect_flux_default (src/advect.c:26-302) and update_state (src/sale2d.c:1635-1742)
__global__ void ka_remap_state(const AdjCtx a)
{
    const Ctx &c = a.c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    double th[4] = {0., 0., 0., 0.};
    if (a_cell_interior(c, i, j)) {
        const long long p = KIDX(i, j);
        const long long PL = c.d.PL;
        const int nmat = 2, b = 6;
        const double *face[4] = {c.f.bx_phi + KIDX(i, j), c.f.by_phi + KIDX(i, j), c.f.bx_phi + KIDX(i + 1, j),
                                 c.f.by_phi + KIDX(i, j + 1)};
        double *bface[4] = {a.b.bx_phi + KIDX(i, j), a.b.by_phi + KIDX(i, j), a.b.bx_phi + KIDX(i + 1, j),
                            a.b.by_phi + KIDX(i, j + 1)};
        const double dir[4] = {1.0, 1.0, -1.0, -1.0};
        double vof[2], rho[2], eng[2];
        for (int m = 0; m < nmat; ++m) {
            vof[m] = PLN(c.f.m_vof, m)[p];
            rho[m] = PLN(c.f.m_den, m)[p];
            eng[m] = PLN(c.f.m_eng, m)[p];
        }
        const double evol = c.f.e_vol[p];
        const double eden0 = c.f.e_den[p];
        double st0[4];
        for (int q = 0; q < 4; ++q) st0[q] = PLN(c.f.e_ste, q)[p];
        const double dam0 = c.f.e_dam[p];
        // forward remap
        double dphi[16];
        for (int q = 0; q < 16; ++q) dphi[q] = 0.;
        for (int k = 0; k < 4; ++k) {
            const double *f = face[k];
            for (int m = 0; m < nmat; ++m) {
                const double mvk = dir[k] * f[m * PL];
                if (mvk == 0.0) continue;
                const double rho_f = f[(m + nmat) * PL];
                dphi[m] += mvk;
                dphi[m + nmat] += mvk * rho_f;
                dphi[m + 2 * nmat] += mvk * f[(m + 2 * nmat) * PL];
                const double fm = mvk * rho_f;
                for (int q = 0; q < 10; ++q) dphi[b + q] += fm * f[(b + q) * PL];
            }
        }
        double emass0 = evol * eden0;
        double sphi[16];
        for (int m = 0; m < nmat; ++m) {
            sphi[m] = (0.0 + vof[m] * evol) + 1.0 * dphi[m];
            sphi[m + nmat] = (0.0 + vof[m] * evol * rho[m]) + 1.0 * dphi[m + nmat];
            sphi[m + 2 * nmat] = (0.0 + vof[m] * evol * eng[m]) + 1.0 * dphi[m + 2 * nmat];
        }
        sphi[b] = 0.0 + 1.0 * dphi[b];
        sphi[b + 1] = 0.0 + 1.0 * dphi[b + 1];
        for (int q = 0; q < 4; ++q) sphi[b + 2 + q] = (0.0 + emass0 * st0[q]) + 1.0 * dphi[b + 2 + q];
        sphi[b + 6] = emass0 * dam0 + 1.0 * dphi[b + 6];
        bool clampm[2] = {false, false};
        double zeta = 0.0, emass = 0.;
        for (int m = 0; m < nmat; ++m) {
            if (sphi[m] < 0.) { sphi[m] = 0.; sphi[m + nmat] = 0.; clampm[m] = true; }
            if (m == 0) continue;
            zeta += sphi[m];
            emass += sphi[m + nmat];
        }
        int vbranch;
        double nvof[2];
        if (zeta > evol * (1.0 - SALEC_TOLVOF) || (zeta > 0. && sphi[0] < evol * SALEC_TOLVOF)) {
            vbranch = 0;
            const double sc = 1.0 / zeta;
            nvof[1] = sc * sphi[1];
            nvof[0] = 0.0;
        } else if (zeta < evol * SALEC_TOLVOF) {
            vbranch = 1;
            nvof[1] = 0.;
            nvof[0] = 1.0;
        } else {
            vbranch = 2;
            const double sc = 1.0 / evol;
            nvof[0] = sc * (evol - zeta);
            nvof[1] = sc * sphi[1];
        }
        bool killed = false;
        double nrho1 = 0., neng1 = 0.;
        if (nvof[1] < SALEC_TOLVOF || sphi[1 + nmat] < SALEC_TOLRHO * SALEC_TOLVOF * evol) {
            killed = true;
            nvof[1] = 0.;
        } else {
            neng1 = sphi[1 + 2 * nmat] / (nvof[1] * evol);
            nrho1 = sphi[1 + nmat] / (nvof[1] * evol);
        }
        const bool massive = emass > SALEC_TOLRHO * evol;
        double dv[2] = {0., 0.}, st[4] = {0., 0., 0., 0.}, damr = 0.;
        if (massive) {
            const double sc = 1.0 / emass;
            dv[0] = sc * sphi[b];
            dv[1] = sc * sphi[b + 1];
            for (int q = 0; q < 4; ++q) st[q] = sc * sphi[b + 2 + q];
            damr = sphi[b + 6] / emass;
        }
        const double eden_r = emass / evol;
        const double dam = wind(damr, 0.0, 1.0);
        const bool vacuum = eden_r < c.rp.density_cutoff || eden_r < 10.0 * c.rp.density_cutoff * (1.0 - nvof[0]);
        // adjoints of the outputs
        double gvof[2], grho[2], geng[2], gdv[2], gst[4], gdam;
        for (int m = 0; m < nmat; ++m) {
            gvof[m] = PLN(a.b.m_vof, m)[p];
            grho[m] = PLN(a.b.m_den, m)[p];
            geng[m] = PLN(a.b.m_eng, m)[p];
        }
        for (int q = 0; q < 2; ++q) gdv[q] = PLN(a.b.e_dvel, q)[p];
        for (int q = 0; q < 4; ++q) gst[q] = PLN(a.b.e_ste, q)[p];
        gdam = a.b.e_dam[p];
        const double gepre = a.b.e_pre[p], gecsd = a.b.e_csd[p], getem = a.b.e_tem[p], geden = a.b.e_den[p],
                     gemu = a.b.e_mu[p];
        // input adjoints of this cell
        double ivof[2] = {0., 0.}, irho[2] = {0., 0.}, ieng[2] = {0., 0.}, ist[4] = {0., 0., 0., 0.}, idam = 0.,
               ieden = 0.;
        if (!vacuum) {
            // m = 0 (vacuum material): density and energy pass through unchanged
            irho[0] = grho[0];
            ieng[0] = geng[0];
            // EOS of material 1 on the remapped state
            const double vm = nvof[1], r1 = nrho1, e1 = neng1;
            const bool override_ = nvof[0] > SALEC_TOLVOF;
            if (!(vm < SALEC_TOLVOF)) {
                const DevMat &ms = c.mat[1];
                const double plim = (1.0 - dam) * ms.minPint + dam * ms.minPdam;
                using D = Dual<3>;
                const D dd = D::seed(r1, 0), de = D::seed(e1, 1), dl = D::seed(plim, 2);
                const D ein = de / dd;
                const D t = till_temperature<D>(ms, ein, dd);
                D pp, cc;
                till_pressure<D>(ms.tl, ein, dd, pp, cc);
                if (pp < dl) pp = fmax(pp, dl);
                double gp = 0., gc = 0., gt = getem * vm;
                gvof[1] += getem * t.v;
                gvof[1] += geden * r1;
                grho[1] += geden * vm;
                if (!override_) {
                    gvof[1] += gepre * pp.v;
                    gp = gepre * vm;
                    const double cm = dmax(1.0, cc.v);
                    const double ecs = vm / cm;
                    if (ecs > 0.) {
                        const double gsum = -gecsd / (ecs * ecs);
                        gvof[1] += gsum / cm;
                        if (cc.v > 1.0) gc += gsum * (-vm / (cc.v * cc.v));
                    }
                    const double X = r1 * cc.v * cc.v * ms.GaCoef;
                    const double Xm = dmax(1.0, X);
                    const double emus = vm / Xm;
                    if (emus > 0.) {
                        const double gsum = -gemu / (emus * emus);
                        gvof[1] += gsum / Xm;
                        if (X > 1.0) {
                            const double gX = gsum * (-vm / (X * X));
                            grho[1] += gX * cc.v * cc.v * ms.GaCoef;
                            gc += gX * 2.0 * r1 * cc.v * ms.GaCoef;
                        }
                    }
                }
                grho[1] += gt * t.d[0] + gp * pp.d[0] + gc * cc.d[0];
                geng[1] += gt * t.d[1] + gp * pp.d[1] + gc * cc.d[1];
                const double gplim = gp * pp.d[2];
                if (gplim != 0.0) {
                    gdam += gplim * (ms.minPdam - ms.minPint);
                    const double gpi = gplim * (1.0 - dam), gpd = gplim * dam;
                    th[0] += gpi * (2.0 * ms.Yint0 / ms.Ylimint - 1.0) / ms.Yfricint;
                    th[1] += gpi * (-(ms.Yint0 / (ms.Yfricint * ms.Yfricint)) * (ms.Yint0 / ms.Ylimint - 1.0));
                    th[2] += gpd * (-1.0 / ms.Yfricdam);
                    th[3] += gpd * (ms.Ydam0 / (ms.Yfricdam * ms.Yfricdam));
                }
            } else {
                gvof[1] += geden * r1;   // e_den = vof * rho with the density of a killed material, 0
            }
            // back through the remap
            double gs[16];
            for (int q = 0; q < 16; ++q) gs[q] = 0.;
            const double gdamr = (damr >= 0.0 && damr <= 1.0) ? gdam : 0.0;
            double gemass = 0.;
            if (massive) {
                gs[b] += gdv[0] / emass;
                gs[b + 1] += gdv[1] / emass;
                for (int q = 0; q < 4; ++q) gs[b + 2 + q] += gst[q] / emass;
                gs[b + 6] += gdamr / emass;
                gemass = -(gdv[0] * dv[0] + gdv[1] * dv[1] + gst[0] * st[0] + gst[1] * st[1] + gst[2] * st[2] +
                           gst[3] * st[3] + gdamr * damr) / emass;
            }
            double gzeta = 0.;
            double gnv1 = gvof[1], gnv0 = gvof[0];
            if (!killed) {
                gs[1 + 2 * nmat] += geng[1] / (nvof[1] * evol);
                gs[1 + nmat] += grho[1] / (nvof[1] * evol);
                gnv1 += -(geng[1] * neng1 + grho[1] * nrho1) / nvof[1];
            } else {
                gnv1 = 0.;
            }
            if (vbranch == 0) {
                gs[1] += gnv1 / zeta;
                gzeta += -gnv1 * nvof[1] / zeta;
            } else if (vbranch == 2) {
                gs[1] += gnv1 / evol;
                gzeta += -gnv0 / evol;
            }
            gs[1] += gzeta;
            gs[1 + nmat] += gemass;
            for (int m = 0; m < nmat; ++m)
                if (clampm[m]) { gs[m] = 0.; gs[m + nmat] = 0.; }
            gs[0] = 0.;   // the vacuum volume enters only the branch tests
            gs[nmat] = 0.;
            gs[2 * nmat] = 0.;
            // sphi from the cell's content and the face fluxes
            for (int m = 0; m < nmat; ++m) {
                ivof[m] += gs[m] * evol + gs[m + nmat] * evol * rho[m] + gs[m + 2 * nmat] * evol * eng[m];
                irho[m] += gs[m + nmat] * vof[m] * evol;
                ieng[m] += gs[m + 2 * nmat] * vof[m] * evol;
            }
            double gem0 = 0.;
            for (int q = 0; q < 4; ++q) { gem0 += gs[b + 2 + q] * st0[q]; ist[q] = gs[b + 2 + q] * emass0; }
            gem0 += gs[b + 6] * dam0;
            idam = gs[b + 6] * emass0;
            ieden = gem0 * evol;
            for (int k = 0; k < 4; ++k) {
                const double *f = face[k];
                double *bf = bface[k];
                for (int m = 0; m < nmat; ++m) {
                    const double mvk = dir[k] * f[m * PL];
                    if (mvk == 0.0) continue;
                    const double rho_f = f[(m + nmat) * PL], eng_f = f[(m + 2 * nmat) * PL];
                    double gmv = gs[m] + gs[m + nmat] * rho_f + gs[m + 2 * nmat] * eng_f;
                    double grf = gs[m + nmat] * mvk;
                    add(bf + (m + 2 * nmat) * PL, gs[m + 2 * nmat] * mvk);
                    const double fm = mvk * rho_f;
                    double gfm = 0.;
                    for (int q = 0; q < 7; ++q) {
                        gfm += gs[b + q] * f[(b + q) * PL];
                        add(bf + (b + q) * PL, gs[b + q] * fm);
                    }
                    gmv += gfm * rho_f;
                    grf += gfm * mvk;
                    add(bf + (m + nmat) * PL, grf);
                    add(bf + m * PL, gmv * dir[k]);
                }
            }
        }
        for (int m = 0; m < nmat; ++m) {
            PLN(a.b.m_vof, m)[p] = ivof[m];
            PLN(a.b.m_den, m)[p] = irho[m];
            PLN(a.b.m_eng, m)[p] = ieng[m];
        }
        a.b.e_dvel[p] = 0.0;
        PLN(a.b.e_dvel, 1)[p] = 0.0;
        for (int q = 0; q < 4; ++q) PLN(a.b.e_ste, q)[p] = ist[q];
        a.b.e_dam[p] = idam;
        a.b.e_den[p] = ieden;
        a.b.e_pre[p] = 0.0;
        a.b.e_csd[p] = 0.0;
        a.b.e_tem[p] = 0.0;
        a.b.e_mu[p] = 0.0;
    }
    for (int k = 0; k < 4; ++k) add_theta(a.theta + k, th[k]);
}

// ---------------------------------------------------------------- gathers
__device__ __forceinline__ double op_deriv(unsigned op, double src)
{
    switch (op) {
    case 0: return 1.0;
    case 1: return -1.0;
    case 2: return src < 0.0 ? -1.0 : 1.0;
    case 3: return src < 0.0 ? 1.0 : -1.0;
    default: return 0.0;
    }
}

struct AdjGatherArgs {
    GatherBatch g;
    int estart[SALEC_MAX_GATHER_FIELDS + 1];   // entry offsets per field
    double *adj[SALEC_MAX_GATHER_FIELDS];      // adjoint planes of each field
};

__device__ __forceinline__ void locate(const AdjGatherArgs &A, int t, int &f, int &e)
{
    f = 0;
    while (f + 1 < A.g.nfield && t >= A.estart[f + 1]) ++f;
    e = t - A.estart[f];
}

// stage 0: read the adjoints of every destination; 1: clear them; 2: add them to the sources
__global__ void ka_gather(AdjGatherArgs A, int stage, double *scratch)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.estart[A.g.nfield]) return;
    int f, e;
    locate(A, t, f, e);
    const GatherField &gf = A.g.field[f];
    const double *fwd = static_cast<const double *>(gf.base);
    double *adj = A.adj[f];
    const int d = gf.dst[e], s = gf.src[e];
    const unsigned ops = gf.ops[e];
    for (int comp = 0; comp < gf.ncomp; ++comp) {
        const long long off = (long long)comp * gf.plane;
        double &slot = scratch[(long long)t * gf.ncomp_max + comp];
        if (stage == 0) slot = adj[off + d];
        else if (stage == 1) adj[off + d] = 0.0;
        else {
            const double gv = slot * op_deriv((ops >> (3 * comp)) & 7u, fwd[off + s]);
            if (gv != 0.0) atomicAdd(adj + off + s, gv);
        }
    }
}

// The forward gather's semantics are parallel: every destination takes op(source) of the values
// before the gather. Where no reading entry's source is a destination, entries are independent:
// one thread moves its destination's adjoint to its source (atomically: sources are shared).
// Where sources include destinations, the map comes as connected components of the
// destination/source relation, one per thread, disjoint in their points: the thread reads all
// destination adjoints of its component, clears them, then adds to the sources, without atomics.
__global__ void ka_gather_fused(AdjGatherArgs A)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.g.total) return;
    int f = 0;
    while (f + 1 < A.g.nfield && t >= A.g.start[f + 1]) ++f;
    const GatherField &gf = A.g.field[f];
    const int k = t - A.g.start[f];
    const double *fwd = static_cast<const double *>(gf.base);
    double *adj = A.adj[f];
    if (gf.cstart) {
        const int a = gf.cstart[k], b = gf.cstart[k + 1];
        for (int comp = 0; comp < gf.ncomp; ++comp) {
            const long long off = (long long)comp * gf.plane;
            double g[SALEC_GATHER_MAX_COMPONENT];
#pragma unroll
            for (int e = 0; e < SALEC_GATHER_MAX_COMPONENT; ++e)
                if (a + e < b) g[e] = adj[off + gf.dst[a + e]];
#pragma unroll
            for (int e = 0; e < SALEC_GATHER_MAX_COMPONENT; ++e)
                if (a + e < b) adj[off + gf.dst[a + e]] = 0.0;
#pragma unroll
            for (int e = 0; e < SALEC_GATHER_MAX_COMPONENT; ++e)
                if (a + e < b) {
                    const int src = gf.src[a + e];
                    const double gv = g[e] * op_deriv((gf.ops[a + e] >> (3 * comp)) & 7u, fwd[off + src]);
                    if (gv != 0.0) adj[off + src] += gv;
                }
        }
    } else {
        const int d = gf.dst[k], src = gf.src[k];
        const unsigned ops = gf.ops[k];
        for (int comp = 0; comp < gf.ncomp; ++comp) {
            const long long off = (long long)comp * gf.plane;
            const double g = adj[off + d];
            adj[off + d] = 0.0;
            const double gv = g * op_deriv((ops >> (3 * comp)) & 7u, fwd[off + src]);
            if (gv != 0.0) atomicAdd(adj + off + src, gv);
        }
    }
}

// ---------------------------------------------------------------- surface-profile misfit
// per interior column: h = sum over interior rows of (1 - m_vof[0]) * e_pos[3]
__global__ void ka_profile_height(const Ctx c, double *h)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 2 || i > c.d.enx - 3) return;
    double s = 0.;
    for (int j = 2; j <= c.d.eny - 3; ++j) {
        const long long p = KIDX(i, j);
        s += (1.0 - c.f.m_vof[p]) * PLN(c.f.e_pos, 3)[p];
    }
    h[i - 2] = s;
}

__global__ void ka_profile_seed(const Ctx c, const Fields b, const double *h, const double *target, const double *w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i < 2 || i > c.d.enx - 3 || j < 2 || j > c.d.eny - 3) return;
    const int col = i - 2;
    const double r = h[col] - target[col];
    const long long p = KIDX(i, j);
    b.m_vof[p] += -w[col] * r * PLN(c.f.e_pos, 3)[p];
}

// J = 0.5 sum_i w_i r_i^2 in a fixed order (one block: strided partial sums, then a tree), so
// that the misfit is the same bits on every run
__global__ void ka_profile_sum(const double *h, const double *target, const double *w, int ncols, double *J)
{
    __shared__ double part[256];
    double s = 0.;
    for (int col = threadIdx.x; col < ncols; col += 256) {
        const double r = h[col] - target[col];
        s += 0.5 * w[col] * r * r;
    }
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *J = part[0];
}

__global__ void __launch_bounds__(256, 4) ka_list_copy(const CopySeg *segs, char *base, const long long *slot,
                                                       unsigned long long stride, int save)
{
    // blockIdx.y: the field; the x-blocks stride over its 16-byte words (a field is below 2^31
    // words), four in flight per thread
    char *rec = base + (slot ? (unsigned long long)*slot * stride : 0ULL);
    const CopySeg g = segs[blockIdx.y];
    char *dst = save ? rec + g.off : g.field;
    const char *src = save ? g.field : rec + g.off;
    const unsigned n16 = (unsigned)(g.bytes >> 4);
    const unsigned nt = gridDim.x * blockDim.x;
    uint4 *d4 = reinterpret_cast<uint4 *>(dst);
    const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
    unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
    for (; q + 3 * nt < n16; q += 4 * nt) {
        const uint4 a0 = s4[q], a1 = s4[q + nt], a2 = s4[q + 2 * nt], a3 = s4[q + 3 * nt];
        d4[q] = a0;
        d4[q + nt] = a1;
        d4[q + 2 * nt] = a2;
        d4[q + 3 * nt] = a3;
    }
    for (; q < n16; q += nt) d4[q] = s4[q];
    if (blockIdx.x == 0)
        for (unsigned b = (n16 << 4) + threadIdx.x; b < g.bytes; b += blockDim.x) dst[b] = src[b];
}

__global__ void ka_slot(long long *slot, long long v, int add)
{
    if (threadIdx.x == 0) *slot = add ? *slot + v : v;
}

} // namespace

void launch_list_copy(const CopySeg *segs, int nseg, unsigned long long max_bytes, char *base, const long long *slot,
                      unsigned long long stride, bool save, cudaStream_t s)
{
    // about four 16-byte words per thread of the largest field, at most 8 blocks per SM in all
    const unsigned long long words = (max_bytes + 15) >> 4;
    unsigned long long bx = (words + 4 * 256 - 1) / (4 * 256);
    const unsigned long long cap = (unsigned long long)(8 * 148 + nseg - 1) / nseg;
    if (bx > cap) bx = cap;
    if (bx < 1) bx = 1;
    ka_list_copy<<<dim3((unsigned)bx, (unsigned)nseg), 256, 0, s>>>(segs, base, slot, stride, save ? 1 : 0);
}

void launch_slot_set(long long *slot, long long value, cudaStream_t s) { ka_slot<<<1, 32, 0, s>>>(slot, value, 0); }

void launch_slot_add(long long *slot, long long delta, cudaStream_t s) { ka_slot<<<1, 32, 0, s>>>(slot, delta, 1); }

void launch_adjoint_kernel(AdjKernel k, const AdjCtx &a, cudaStream_t s)
{
    const dim3 blk(32, 4);
    const dim3 g((a.c.d.enx + blk.x - 1) / blk.x, (a.c.d.eny + blk.y - 1) / blk.y);
    const dim3 gv((a.c.d.vnx + blk.x - 1) / blk.x, (a.c.d.vny + blk.y - 1) / blk.y);
    switch (k) {
    case AK_VERTEX_MOMENTUM: ka_vertex_momentum<<<gv, blk, 0, s>>>(a); break;
    case AK_CELL_VELOCITY: ka_cell_velocity<<<g, blk, 0, s>>>(a); break;
    case AK_VOID_VERTICES: ka_void_vertices<<<gv, blk, 0, s>>>(a); break;
    case AK_GRADIENT:
        ka_gradient<<<g, blk, 0, s>>>(a);
        ka_corner_sum<<<gv, blk, 0, s>>>(a, a.b.v_vel, 0);
        break;
    case AK_STRESS: ka_stress<<<g, blk, 0, s>>>(a); break;
    case AK_ACCELERATION: ka_acceleration<<<gv, blk, 0, s>>>(a); break;
    case AK_DISPLACEMENT: ka_displacement<<<gv, blk, 0, s>>>(a); break;
    case AK_ENERGY: ka_energy<<<g, blk, 0, s>>>(a); break;
    case AK_FLUX:
        ka_flux<false><<<g, blk, 0, s>>>(a);
        ka_flux<true><<<g, blk, 0, s>>>(a);
        ka_corner_sum<<<gv, blk, 0, s>>>(a, a.b.v_dis, 0);
        ka_corner_sum<<<gv, blk, 0, s>>>(a, a.b.v_vof, 8);
        break;
    case AK_REMAP_STATE: ka_remap_state<<<g, blk, 0, s>>>(a); break;
    }
}

void launch_adjoint_gather(const GatherBatch &g, const int *entries, const void *const *adj_base, double *scratch,
                           bool two_pass, cudaStream_t s)
{
    AdjGatherArgs A;
    A.g = g;
    A.estart[0] = 0;
    for (int f = 0; f < g.nfield; ++f) {
        A.estart[f + 1] = A.estart[f] + entries[f];
        A.adj[f] = static_cast<double *>(const_cast<void *>(adj_base[f]));
    }
    const int n = A.estart[g.nfield];
    if (n == 0) return;
    const int tb = 256;
    if (!two_pass) {
        ka_gather_fused<<<(g.total + tb - 1) / tb, tb, 0, s>>>(A);
        return;
    }
    const int nb = (n + tb - 1) / tb;
    for (int stage = 0; stage < 3; ++stage) ka_gather<<<nb, tb, 0, s>>>(A, stage, scratch);
}

void launch_profile_misfit(const Ctx &c, const Fields &b, const double *target, const double *weight, double *J,
                           double *h, cudaStream_t s)
{
    ka_profile_height<<<(c.d.enx + 127) / 128, 128, 0, s>>>(c, h);
    const dim3 blk(32, 4);
    const dim3 g((c.d.enx + blk.x - 1) / blk.x, (c.d.eny + blk.y - 1) / blk.y);
    ka_profile_seed<<<g, blk, 0, s>>>(c, b, h, target, weight);
    ka_profile_sum<<<1, 256, 0, s>>>(h, target, weight, c.d.enx - 4, J);
}

} // namespace salec
