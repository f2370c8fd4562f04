// Step kernels of the B200 mesh update (FP64 form).
//
// One kernel per sweep group of the reference's time loop (src/salec2d.c:115-272); each
// thread owns one cell or one vertex, which is exactly the reference's Jacobi structure:
// every sweep writes only its own point (or, in the flux sweep, only the faces on which its
// own cell is the upwind donor). Cross-point boundary fills (ghost cells and restricted
// vertices) are separate gather passes, see salec_ghost.cpp.
//
// Point sections (src/mpi_vec/mpi_vec.c:111-230, one rank):
//   cells:    interior = 2 <= i <= enx-3 and 2 <= j <= eny-3 (internal|send); the rest is pad.
//   vertices: active = 1 <= i <= vnx-2 and 1 <= j <= vny-2 (update|internal); the outer ring is
//             never updated; "pad_section" = x or y distance to the outer ring <= 1.
#include "salec_device.cuh"
#include "salec_kernels.h"

namespace salec {

#define KIDX(i, j) ((long long)(i) + (long long)c.d.P * (long long)(j))
#define PLN(ptr, comp) ((ptr) + (long long)(comp) * c.d.PL)
// component comp of a row-tabled geometry field at the thread's own point (i, j)
#define GEO(g, comp) ((g).tab[(long long)(comp) * (g).plane + i + (long long)c.d.P * (g).row[j]])

// Register budget per thread of the heavy sweeps: SALEC_REGS_<K> > 0 caps the allocator at that
// many registers (__maxnreg__), trading a few spilled values that stay in L1 for more resident
// warps to hide the dependent loads; 0 leaves the allocator's own choice under the default
// bounds (256-thread blocks where a kernel declares them, else the 1024-thread default). The
// defaults are the fastest budgets measured on B200 for the 2048x2048 impact in FP64 (registers
// are granted per warp in units of 256, so only multiples of 8 differ); the budgets change
// which values live in registers, never the arithmetic.
#ifndef SALEC_REGS_STRESS
#define SALEC_REGS_STRESS 56
#endif
#ifndef SALEC_REGS_FLUX
#define SALEC_REGS_FLUX 80
#endif
#ifndef SALEC_REGS_REMAP
#define SALEC_REGS_REMAP 96
#endif
#ifndef SALEC_REGS_ACCEL
#define SALEC_REGS_ACCEL 40
#endif
#ifndef SALEC_REGS_VOFMOM
#define SALEC_REGS_VOFMOM 32
#endif
#ifndef SALEC_REGS_GRAD
#define SALEC_REGS_GRAD 40
#endif
#ifndef SALEC_REGS_ENERGY
#define SALEC_REGS_ENERGY 40
#endif
// budgets of the mixed form's instances (relaxed fields stored as float), SALEC_REGS_<K>_F:
// the FP64 budgets by default. Remap 88, acceleration 56 and energy 32 make the 2048x2048 mixed
// cycle 1.8% faster but an ensemble of small meshes in 32x4 blocks 4% slower, so a build for
// large single meshes may set them.
#ifndef SALEC_REGS_STRESS_F
#define SALEC_REGS_STRESS_F SALEC_REGS_STRESS
#endif
// the stress sweep with the energy update fused (the cycle graph's form): 72 measured best
// against 56, 64, 80 and 96 (1.2695, 1.2639, 1.2572, 1.2825, 1.2946 ms per cycle at 2048²)
#ifndef SALEC_REGS_STRESS_EN
#define SALEC_REGS_STRESS_EN 72
#endif
#ifndef SALEC_REGS_STRESS_EN_F
#define SALEC_REGS_STRESS_EN_F SALEC_REGS_STRESS_EN
#endif
#ifndef SALEC_REGS_FLUX_F
#define SALEC_REGS_FLUX_F SALEC_REGS_FLUX
#endif
#ifndef SALEC_REGS_REMAP_F
#define SALEC_REGS_REMAP_F SALEC_REGS_REMAP
#endif
#ifndef SALEC_REGS_ENERGY_F
#define SALEC_REGS_ENERGY_F SALEC_REGS_ENERGY
#endif
#ifndef SALEC_REGS_ACCEL_F
#define SALEC_REGS_ACCEL_F SALEC_REGS_ACCEL
#endif
#ifndef SALEC_REGS_VOFMOM_F
#define SALEC_REGS_VOFMOM_F SALEC_REGS_VOFMOM
#endif
#ifndef SALEC_REGS_GRAD_F
#define SALEC_REGS_GRAD_F SALEC_REGS_GRAD
#endif
#if SALEC_REGS_STRESS > 0
#define SALEC_BOUNDS_STRESS                                                                              \
    __maxnreg__((EN ? (sizeof(R) == 4 ? SALEC_REGS_STRESS_EN_F : SALEC_REGS_STRESS_EN)                  \
                    : (sizeof(R) == 4 ? SALEC_REGS_STRESS_F : SALEC_REGS_STRESS)))
#else
#define SALEC_BOUNDS_STRESS __launch_bounds__(256)
#endif
#if SALEC_REGS_FLUX > 0
#define SALEC_BOUNDS_FLUX __maxnreg__((sizeof(R) == 4 ? SALEC_REGS_FLUX_F : SALEC_REGS_FLUX))
#else
#define SALEC_BOUNDS_FLUX __launch_bounds__(256)
#endif
#if SALEC_REGS_REMAP > 0
#define SALEC_BOUNDS_REMAP __maxnreg__((sizeof(R) == 4 ? SALEC_REGS_REMAP_F : SALEC_REGS_REMAP))
#else
#define SALEC_BOUNDS_REMAP __launch_bounds__(256)
#endif
#if SALEC_REGS_ENERGY > 0
#define SALEC_BOUNDS_ENERGY __maxnreg__((sizeof(R) == 4 ? SALEC_REGS_ENERGY_F : SALEC_REGS_ENERGY))
#else
#define SALEC_BOUNDS_ENERGY __launch_bounds__(256)
#endif
#if SALEC_REGS_ACCEL > 0
#define SALEC_BOUNDS_ACCEL __maxnreg__((sizeof(R) == 4 ? SALEC_REGS_ACCEL_F : SALEC_REGS_ACCEL))
#else
#define SALEC_BOUNDS_ACCEL
#endif
#if SALEC_REGS_VOFMOM > 0
#define SALEC_BOUNDS_VOFMOM __maxnreg__((sizeof(R) == 4 ? SALEC_REGS_VOFMOM_F : SALEC_REGS_VOFMOM))
#else
#define SALEC_BOUNDS_VOFMOM
#endif
#if SALEC_REGS_GRAD > 0
#define SALEC_BOUNDS_GRAD __maxnreg__((sizeof(R) == 4 ? SALEC_REGS_GRAD_F : SALEC_REGS_GRAD))
#else
#define SALEC_BOUNDS_GRAD
#endif

template <class C>
__device__ __forceinline__ bool cell_interior(const C &c, int i, int j)
{
    return i >= 2 && i <= c.d.enx - 3 && j >= 2 && j <= c.d.eny - 3;
}
template <class C>
__device__ __forceinline__ bool vert_active(const C &c, int i, int j)
{
    return i >= 1 && i <= c.d.vnx - 2 && j >= 1 && j <= c.d.vny - 2;
}
template <class C>
__device__ __forceinline__ bool vert_pad(const C &c, int i, int j)
{
    int xd = min(i, c.d.vnx - 1 - i), yd = min(j, c.d.vny - 1 - j);
    return xd <= 1 || yd <= 1;
}
template <class C>
__device__ __forceinline__ double step_dt(const C &c)
{
    // Min(max_dt, CFL reduction) as in src/salec2d.c:167
    double r = ord_decode(c.scal->dt_acc);
    return dmin(c.rp.max_dt, r);
}

// CFL candidate of an interior cell that is not pure vacuum: calculate_dt (src/sale2d.c:1999-2002),
// DTF * MIN(dt_r, dt_z) with MIN's own NaN behaviour (a NaN first argument yields the second)
template <class C>
__device__ __forceinline__ double cfl_candidate(const C &c, long long p, double csd)
{
    const double dt_r = 1.0 * PLN(c.f.e_pos, 2)[p] / (fabs(c.f.e_vel[p]) + csd);
    const double dt_z = 1.0 * PLN(c.f.e_pos, 3)[p] / (fabs(PLN(c.f.e_vel, 1)[p]) + csd);
    return SALEC_DTF * dmin(dt_r, dt_z);
}

// ============================================================ phase 0: surface profile
// trace_profile (src/ejecta.c:8-63): per column, MIN of cell-centre y over cells whose vacuum
// fraction exceeds 0.1; cells above the ejecta threshold with no vacuum get e_ejt = 1.
template <class R>
__global__ void k_profile_reset(const CtxT<R> c)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < c.d.enx) c.f.y_profile[i] = __longlong_as_double((long long)ord_encode(c.rp.threshold_z * 2.0));
}

template <class R>
__global__ void k_trace_profile(const CtxT<R> c)
{
    __shared__ unsigned long long smin[8][32];
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j0 = blockIdx.y * 64 + threadIdx.y;
    unsigned long long best = ~0ULL;
    if (i < c.d.enx) {
        // the thread's 8 rows are loaded before any is used, so that all 16 loads are in flight
        // together; the MIN is order-independent
        const int jend = min(c.d.eny, (int)blockIdx.y * 64 + 64);
        double v0[8], y[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int j = j0 + 8 * k;
            v0[k] = 0.0; y[k] = 0.0;
            if (j < jend) {
                const long long p = KIDX(i, j);
                v0[k] = c.f.m_vof[p];
                y[k] = PLN(c.f.e_pos, 1)[p];
            }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int j = j0 + 8 * k;
            if (j >= jend) continue;
            if (v0[k] > 0.1) best = min(best, ord_encode(y[k]));
            if (y[k] > c.rp.threshold_z && v0[k] < SALEC_TOLVOF) c.f.e_ejt[KIDX(i, j)] = 1.0;
        }
    }
    smin[threadIdx.y][threadIdx.x] = best;
    __syncthreads();
    if (threadIdx.y == 0 && i < c.d.enx) {
        for (int k = 1; k < 8; ++k) best = min(best, smin[k][threadIdx.x]);
        if (best != ~0ULL) atomicMin((unsigned long long *)&c.f.y_profile[i], best);
    }
}

template <class R>
__global__ void k_profile_decode(const CtxT<R> c)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < c.d.enx) {
        unsigned long long u = (unsigned long long)__double_as_longlong(c.f.y_profile[i]);
        c.f.y_profile[i] = ord_decode(u);
    }
}

// ============================================================ phase 1: vertex volume fractions
// update_v_vof (src/sale2d.c:751-791): mean of the four surrounding cells.
template <class C>
__device__ __forceinline__ void vertex_vof(const C &c, int i, int j)
{
    const long long cl[4] = {KIDX(i - 1, j - 1), KIDX(i, j - 1), KIDX(i, j), KIDX(i - 1, j)};
    const long long p = KIDX(i, j);
    for (int m = 0; m < c.d.nmat; ++m) {
        const double *ev = PLN(c.f.m_vof, m);
        double s = 0.0;
        for (int k = 0; k < 4; ++k) s += 0.25 * ev[cl[k]];
        PLN(c.f.v_vof, m)[p] = s;
    }
}

// ============================================================ phase 2: vertex momentum
// update_v_vel_inc (src/sale2d.c:930-1049): add the advected momentum increments of the
// four cells, weighted by density and corner sub-volume; clamp |v|; count void corners.
template <class C>
__device__ __forceinline__ void vertex_momentum(const C &c, int i, int j)
{
    const long long cl[4] = {KIDX(i - 1, j - 1), KIDX(i, j - 1), KIDX(i, j), KIDX(i - 1, j)};
    const int corner[4] = {2, 3, 0, 1};
    const long long p = KIDX(i, j);
    auto *vx = c.f.v_vel, *vy = PLN(c.f.v_vel, 1);
    auto *m0 = c.f.v_mass, *m1 = PLN(c.f.v_mass, 1);
    const double old_x = vx[p], old_y = vy[p];
    double inc_x = 0., inc_y = 0., vvol = 0., vmass = 0.;
    int void_corner = 0;
    for (int k = 0; k < 4; ++k) {
        if (PLN(c.f.e_wpt, corner[k])[cl[k]] > 0.) void_corner++;
        const double rho = c.f.e_den[cl[k]];
        if (rho < SALEC_TOLRHO) continue;
        const double lv = GEO(c.g_v_vol, k + 1);
        vvol += lv;
        vmass += rho * lv;
        const double w = rho * lv;
        inc_x += w * c.f.e_dvel[cl[k]];
        inc_y += w * PLN(c.f.e_dvel, 1)[cl[k]];
    }
    double nx_, ny_;
    if (vmass > SALEC_TOLRHO * vvol) {
        const double pa = 1.0 / vmass, pb = m0[p] / vmass;
        nx_ = pa * inc_x + pb * old_x;
        ny_ = pa * inc_y + pb * old_y;
        m0[p] = vmass;
    } else {
        m0[p] = 0.;
        nx_ = 0.; ny_ = 0.;
    }
    m1[p] = 1.0 * void_corner;
    double vn = 0.;
    vn += nx_ * nx_;
    vn += ny_ * ny_;
    vn = sqrt(vn);
    if (vn > c.rp.velocity_max) {
        const double s = c.rp.velocity_max / vn;
        nx_ *= s; ny_ *= s;
    }
    if (vn < c.rp.velocity_min * 1) { nx_ = 0.; ny_ = 0.; }
    vx[p] = nx_; vy[p] = ny_;
}

// Phases 1 and 2 in one vertex sweep: both read only cell fields that no vertex sweep writes,
// so one thread per vertex does both (the m_vof and e_dvel/e_den ghost fills run first).
template <class R>
__global__ void SALEC_BOUNDS_VOFMOM k_vertex_vof_momentum(const CtxT<R> c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!vert_active(c, i, j)) return;
    vertex_vof(c, i, j);
    vertex_momentum(c, i, j);
}

// ============================================================ phase 3: cell velocity
// update_e_vel (src/sale2d.c:838-928): mass-weighted mean over the solid corner vertices.
template <class R>
__global__ void k_cell_velocity(const CtxT<R> c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!cell_interior(c, i, j)) return;
    const long long p = KIDX(i, j);
    const long long vl[4] = {KIDX(i, j), KIDX(i + 1, j), KIDX(i + 1, j + 1), KIDX(i, j + 1)};
    double ex = 0., ey = 0.;
    const double rho = c.f.e_den[p];
    if (!(rho < SALEC_TOLRHO)) {
        int vac = 0;
        double wpt[4];
        for (int k = 0; k < 4; ++k) {
            wpt[k] = PLN(c.f.e_wpt, k)[p];
            const double nvoid = PLN(c.f.v_mass, 1)[vl[k]];
            if (nvoid >= 4.0 || (nvoid >= 3.0 && wpt[k] < 0.)) vac++;
        }
        if (vac != 4) {
            double sm = 0.;
            for (int k = 0; k < 4; ++k) {
                if (wpt[k] > 0.0 || rho < SALEC_TOLRHO) continue;
                const double mk = c.f.v_mass[vl[k]];
                ex += mk * c.f.v_vel[vl[k]];
                ey += mk * PLN(c.f.v_vel, 1)[vl[k]];
                sm += mk;
            }
            if (sm > 0.) {
                const double s = 1.0 / sm;
                ex *= s; ey *= s;
            } else {
                ex = 0.; ey = 0.;
            }
        }
    }
    c.f.e_vel[p] = ex;
    PLN(c.f.e_vel, 1)[p] = ey;
}

// ============================================================ phase 4: void vertices
// check_v_vel (src/sale2d.c:1051-1142): a vertex whose four corners are all void takes the
// density-weighted velocity of its non-empty cells.
template <class R>
__global__ void k_void_vertices(const CtxT<R> c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!vert_active(c, i, j)) return;
    const long long cl[4] = {KIDX(i - 1, j - 1), KIDX(i, j - 1), KIDX(i, j), KIDX(i - 1, j)};
    const int corner[4] = {2, 3, 0, 1};
    int void_cell = 0, void_corner = 0;
    for (int k = 0; k < 4; ++k) {
        if (c.f.e_den[cl[k]] < SALEC_TOLRHO) void_cell++;
        if (PLN(c.f.e_wpt, corner[k])[cl[k]] > 0.) void_corner++;
    }
    if (void_cell >= 4 || void_corner < 4) return;
    double ax = 0., ay = 0., ad = 0.;
    for (int k = 0; k < 4; ++k) {
        const double rho = c.f.e_den[cl[k]];
        if (rho < SALEC_TOLRHO) continue;
        ad += rho;
        ax += rho * c.f.e_vel[cl[k]];
        ay += rho * PLN(c.f.e_vel, 1)[cl[k]];
    }
    const double s = 1.0 / ad;
    const long long p = KIDX(i, j);
    c.f.v_vel[p] = s * ax;
    PLN(c.f.v_vel, 1)[p] = s * ay;
}

// ============================================================ phase 5 (+6): velocity gradient,
// artificial viscosity and the CFL candidate of every interior cell.
// update_e_gradvel (src/sale2d.c:1144-1236) and calculate_dt (src/sale2d.c:1959-2016).
template <class R>
__global__ void SALEC_BOUNDS_GRAD k_gradient_viscosity_cfl(const CtxT<R> c)
{
    using A = R;   // arithmetic of the gradient and the viscosity: FP64, or FP32 in the mixed form
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    unsigned long long cand = ~0ULL;
    if (cell_interior(c, i, j)) {
        const long long p = KIDX(i, j);
        const long long vl[4] = {KIDX(i, j), KIDX(i + 1, j), KIDX(i + 1, j + 1), KIDX(i, j + 1)};
        A vx[4], vy[4];
        for (int k = 0; k < 4; ++k) { vx[k] = c.f.v_vel[vl[k]]; vy[k] = PLN(c.f.v_vel, 1)[vl[k]]; }
        A g[12];
        for (int k = 0; k < 12; ++k) g[k] = GEO(c.g_e_grad, k);
        A d0 = A(0.), d1 = A(0.), d2 = A(0.), d3 = A(0.), d4 = A(0.);
        for (int k = 0; k < 4; ++k) d0 += g[k] * vx[k];        // dv_r/dr
        for (int k = 0; k < 4; ++k) d2 += g[k] * vy[k];        // dv_z/dr
        for (int k = 0; k < 4; ++k) d1 += g[4 + k] * vx[k];    // dv_r/dz
        for (int k = 0; k < 4; ++k) d3 += g[4 + k] * vy[k];    // dv_z/dz
        for (int k = 0; k < 4; ++k) d4 += g[8 + k] * vx[k];    // v_r/r
        PLN(c.f.e_grad_vel, 0)[p] = d0;
        PLN(c.f.e_grad_vel, 1)[p] = d1;
        PLN(c.f.e_grad_vel, 2)[p] = d2;
        PLN(c.f.e_grad_vel, 3)[p] = d3;
        PLN(c.f.e_grad_vel, 4)[p] = d4;
        const A div = d0 + d3 + d4;
        c.f.e_div_vel[p] = div;
        const double vof0 = c.f.m_vof[p];
        const A csd = c.f.e_csd[p];
        A q;
        if (vof0 > SALEC_TOLVOF || c.f.e_pre[p] <= A(0.0)) {
            q = A(0.);
        } else {
            double aread = GEO(c.g_e_vol, 0) / c.f.e_pos[p];
            const A area = A(fabs(aread));
            const A ql = A(c.rp.avis1) * csd * sqrt(area);
            const A qq = A(c.rp.avis2) * div * area;
            q = amin(A(0.), div) * A(c.f.e_den[p]) * (qq - ql);
            if (q < A(SALEC_TOLQPRE)) q = A(0.);
        }
        c.f.e_q[p] = q;
        // CFL candidate over cells that are not pure vacuum, in FP64; a NaN candidate is recorded
        // by its position in the reference's traversal order instead (see k_finalize_dt)
        if (!(vof0 > 1.0 - SALEC_TOLVOF)) {
            const double dt_rz = cfl_candidate(c, p, (double)csd);
            if (dt_rz == dt_rz) cand = ord_encode(dt_rz);
            else atomicMax(&c.scal->dt_nan_last, (long long)j * c.d.enx + i);
        }
    }
    // block MIN, one atomic per block
    for (int o = 16; o > 0; o >>= 1) cand = min(cand, __shfl_xor_sync(0xffffffffu, cand, o));
    __shared__ unsigned long long wmin[32];
    const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
    const int warp = (threadIdx.y * blockDim.x + threadIdx.x) >> 5;
    if (lane == 0) wmin[warp] = cand;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x * blockDim.y + 31) >> 5;
        unsigned long long v = lane < nw ? wmin[lane] : ~0ULL;
        for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0 && v != ~0ULL) atomicMin(&c.scal->dt_acc, v);
    }
}

// phase 6: dt of this cycle: a prescribed time step where the handle has a schedule for this
// cycle (salec_gpu_set_dt_schedule), else the CFL reduction. The reference folds the candidates in traversal order (j outer, i
// inner) with MIN(a, b) = a < b ? a : b (src/mpi_vec/mpi_vec_types.h:262), starting from
// 1.1 * dt_prev: a NaN candidate makes the running value NaN, and the next candidate replaces
// it. So with no NaN the result is the order-free MIN of the gradient sweep; otherwise it is
// the MIN of the candidates after the last NaN (NaN when the NaN came last). That recount
// runs here, over the whole grid, only when the gradient sweep saw a NaN; otherwise one thread
// finishes the cycle's dt. The last block of a recount resets its accumulators.
#define SALEC_FINALIZE_THREADS 256
template <class R>
__global__ void __launch_bounds__(SALEC_FINALIZE_THREADS) k_finalize_dt(const CtxT<R> c)
{
    if (c.dt_sched) {
        const long long k = c.scal->i_step - c.dt_sched_i0;
        if (k >= 0 && k < c.dt_sched_n) {
            if (threadIdx.x == 0 && blockIdx.x == 0) c.scal->dt = c.dt_sched[k];
            return;
        }
    }
    const long long last = c.scal->dt_nan_last;
    if (last < 0) {
        if (threadIdx.x == 0 && blockIdx.x == 0) c.scal->dt = step_dt(c);
        return;
    }
    const int nx = c.d.enx - 4;
    const long long n = (long long)nx * (c.d.eny - 4);
    unsigned long long best = ~0ULL;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % nx) + 2, j = (int)(t / nx) + 2;
        if ((long long)j * c.d.enx + i <= last) continue;
        const long long p = KIDX(i, j);
        if (c.f.m_vof[p] > 1.0 - SALEC_TOLVOF) continue;
        best = min(best, ord_encode(cfl_candidate(c, p, (double)c.f.e_csd[p])));
    }
    __shared__ unsigned long long wmin[SALEC_FINALIZE_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < SALEC_FINALIZE_THREADS / 32; ++w) best = min(best, wmin[w]);
        if (best != ~0ULL) atomicMin(&c.scal->dt_tail, best);
        __threadfence();
        if (atomicAdd(&c.scal->dt_tail_blocks, 1u) == gridDim.x - 1) {
            __threadfence();
            const unsigned long long tail = atomicMin(&c.scal->dt_tail, ~0ULL);
            const double r = tail == ~0ULL ? __longlong_as_double(0x7ff8000000000000LL) : ord_decode(tail);
            c.scal->dt = dmin(c.rp.max_dt, r);
            c.scal->dt_tail = ~0ULL;
            c.scal->dt_tail_blocks = 0u;
        }
    }
}

// ============================================================ phase 7: vibration, stress, damage
// block_vibration (src/strength.c:625-695) and update_e_stress (src/strength.c:7-349).
template <class R, int NM, bool POR>
__device__ __forceinline__ void energy_cell(const CtxT<R> &c, long long p, double s0, double s1, double s2, double s3,
                                            double g0, double g1, double g2, double g3, double g4, double pre);

// EN: the energy update of phase 10 follows in the same thread (the cycle graph's form). It reads
// the cell's new stress, its velocity gradient, pressure and viscosity, which phases 8 and 9 do
// not change for an interior cell, and writes m_eng, m_pty and e_cvs, which they do not read, so
// it computes what the separate sweep computes after them.
template <class R, int NM, bool POR, bool EN = false>
__global__ void SALEC_BOUNDS_STRESS k_stress(const CtxT<R> c)
{
    using A = R;   // arithmetic of stress, strength and damage: FP64, or FP32 in the mixed form
    constexpr int MM = NM > 0 ? NM : SALEC_MAXMAT;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!cell_interior(c, i, j)) return;
    const long long p = KIDX(i, j);
    const int nmat = NM > 0 ? NM : c.d.nmat;
    const A dt = A(c.scal->dt);
    const double vof0 = c.f.m_vof[p];
    A dam = c.f.e_dam[p];

    // --- acoustic fluidisation (block model)
    if (c.rp.acoustic_fluid) {
        A vib = c.f.e_vib[p];
        if (vof0 > SALEC_TOLVOF || dam < A(0.5)) {
            vib = A(0.);
        } else {
            A tdec = A(-1.0), cvib = A(0.0), toff = A(-1.0), vmax = A(0.0), pvl = A(0.0);
            for (int m = 1; m < nmat; ++m) {
                if (PLN(c.f.m_vof, m)[p] < SALEC_TOLVOF) continue;
                const DevMat &s = c.mat[m];
                tdec = amax(A(s.Tdamp), tdec);
                cvib = amax(A(s.Cvib), cvib);
                toff = amax(A(s.Toff), toff);
                vmax = amax(A(s.VibMax), vmax);
                pvl = amax(A(s.Pvlim), pvl);
            }
            if (tdec <= A(0.) || toff <= A(0.)) {
                vib = A(0.);
            } else {
                const A evx = c.f.e_vel[p], evy = PLN(c.f.e_vel, 1)[p];
                A len = A(0.);
                len += evx * evx;
                len += evy * evy;
                const A nv = cvib * sqrt(len);
                const A nv2 = nv * nv;
                const A t = A(c.scal->time);
                if ((t <= toff) && (nv2 >= vib) && (nv >= A(1.0)) && (c.f.e_q[p] > A(0.)))
                    vib = amin(nv2, vmax * vmax);
                else
                    vib = amax(vib * (A(1.0) - A(2.0) * dt / tdec + A(2.0) * (dt / tdec) * (dt / tdec)), A(0.0));
            }
        }
        c.f.e_vib[p] = vib;
    }

    // --- stress update
    if (vof0 > SALEC_TOLVOF) {
        c.f.e_ste[p] = 0.; PLN(c.f.e_ste, 1)[p] = 0.; PLN(c.f.e_ste, 2)[p] = 0.; PLN(c.f.e_ste, 3)[p] = 0.;
        c.f.e_ste2s[p] = 0.; c.f.e_sta2s[p] = 0.; c.f.e_strength[p] = 0.;
        return;
    }
    // every input of a full cell, issued in one batch
    A s0 = c.f.e_ste[p], s1 = PLN(c.f.e_ste, 1)[p], s2 = PLN(c.f.e_ste, 2)[p], s3 = PLN(c.f.e_ste, 3)[p];
    A ste2s = c.f.e_ste2s[p], sta2s = c.f.e_sta2s[p], tps = c.f.e_tps[p], strength = c.f.e_strength[p];
    A vmat[MM], ptm[MM];
    #pragma unroll
    for (int m = 1; m < nmat; ++m) {
        vmat[m] = A(PLN(c.f.m_vof, m)[p]);
        ptm[m] = POR ? A(PLN(c.f.m_pty, m)[p]) : A(1.0);
    }
    const A rho = c.f.e_den[p];
    const A g0 = c.f.e_grad_vel[p], g1 = PLN(c.f.e_grad_vel, 1)[p], g2 = PLN(c.f.e_grad_vel, 2)[p],
            g3 = PLN(c.f.e_grad_vel, 3)[p], g4 = PLN(c.f.e_grad_vel, 4)[p];
    const A mu = c.f.e_mu[p];
    const A pre = c.f.e_pre[p], tem = c.f.e_tem[p], csd = c.f.e_csd[p];
    A vapor_ref = A(0.), melt_ref = A(0.);
    #pragma unroll
    for (int m = 1; m < nmat; ++m) {
        const A vm = vmat[m];
        if (PLN(c.f.m_vof, m)[p] < SALEC_TOLVOF) continue;
        vapor_ref += vm * A(c.mat[m].VaporDen);
        melt_ref += vm * A(c.mat[m].MeltDen);
    }
    A porosity = A(0.0);
    if (POR) {
        A mv = A(0.0);
        #pragma unroll
        for (int m = 1; m < nmat; ++m) {
            const A vm = vmat[m];
            if (PLN(c.f.m_vof, m)[p] < SALEC_TOLVOF) continue;
            porosity += vm * ptm[m];
            mv += vm;
        }
        porosity /= mv;
    } else {
        porosity = A(1.0);
    }
    porosity = amax(porosity, A(1.0));
    vapor_ref /= porosity;
    melt_ref /= porosity;

    const A ste2s_old = ste2s;
    int state; // 0 solid, 1 melt, 2 vapour
    if (rho <= vapor_ref) {
        state = 2;
        s0 = s1 = s2 = s3 = A(0.);
        ste2s = A(0.);
        tps = A(0.);
        dam = A(0.);
        strength = A(0.);
    } else {
        A e0 = g0, e1 = A(0.5) * g1 + A(0.5) * g2, e2 = g3, e3 = g4;
        const A tr = e0 + e2 + e3;
        e0 -= tr / A(3.0);
        e2 -= tr / A(3.0);
        e3 -= tr / A(3.0);
        if (rho <= melt_ref) {
            state = 1;
            s0 = s1 = s2 = s3 = A(0.);
            ste2s = A(0.);
            sta2s = sqrt(second_inv(e0, e1, e2, e3));
            tps = amin(tps + sta2s * dt, A(10.));
            dam = A(1.);
            strength = A(0.);
        } else {
            state = 0;
            // Wilkins rotation
            A sin2o = (g2 - g1) * dt;
            sin2o = awind(sin2o, A(-1.), A(1.));
            const A cos2o1 = sqrt(A(1.0) - sin2o * sin2o) - A(1.0);
            const A ss2 = (s0 - s2) / A(2.0);
            const A r0 = ss2 * cos2o1 + s1 * sin2o;
            const A r1 = s1 * cos2o1 - ss2 * sin2o;
            const A r2 = -ss2 * cos2o1 - s1 * sin2o;
            s0 += A(1.0) * r0; s1 += A(1.0) * r1; s2 += A(1.0) * r2; s3 += A(1.0) * A(0.0);
            const A k2 = A(2.0) * mu * dt;
            s0 += k2 * e0; s1 += k2 * e1; s2 += k2 * e2; s3 += k2 * e3;
            ste2s = sqrt(second_inv(s0, s1, s2, s3));
            sta2s = sqrt(second_inv(e0, e1, e2, e3));
        }
    }

    if (state == 2) {
        dam = A(0.);
    } else if (state == 1) {
        dam = A(1.0);
    } else {
        A shear = A(0.0), tensile = A(0.);
        #pragma unroll
        for (int m = 1; m < nmat; ++m) {
            const A vm = vmat[m];
            if (PLN(c.f.m_vof, m)[p] < SALEC_TOLVOF) continue;
            const DevMat &s = c.mat[m];
            A my = strength_fn<A>(s.yfunc, pre, dam, tps, sta2s, tem, A(0.), s);
            if (c.rp.acoustic_fluid && pre >= A(0.)) {
                const A vibp = amin(rho * csd * sqrt(A(c.f.e_vib[p])), pre);
                const A tm = simon_melt<A>(pre, s);
                A soft = ohnaka_soft<A>(tem, s, tm);
                soft = awind(soft, A(0.0), A(1.0));
                const A lp = pre - vibp * dam * dam * sqrt(soft);
                const A myv = strength_fn<A>(s.yfunc, lp, dam, tps, sta2s, tem, A(0.), s) + rho * A(s.Acvis) * sta2s;
                my = amin(myv, my);
            }
            shear += vm * amax(my, A(0.0));
            if (c.rp.tensile_failure) tensile += vm * strength_fn<A>(s.tfunc, pre, dam, tps, sta2s, tem, A(0.), s);
        }
        if (c.rp.tracer_lubrication >= 1 && c.f.e_cnd[p] >= A(1.0)) {
            const A lub = amin(pre * A(c.rp.tracer_lub_frac) + A(c.rp.tracer_lub_y0), A(0.0));
            shear = amin(shear, lub);
        }
        strength = shear;
        if (shear < ste2s) {
            sta2s = sta2s / amax(A(0.5), (ste2s - ste2s_old) / (ste2s - shear));
            const A sfac = shear / ste2s;
            s0 *= sfac; s1 *= sfac; s2 *= sfac; s3 *= sfac;
            ste2s = shear;
            A dsd = A(0.);
            #pragma unroll
            for (int m = 1; m < nmat; ++m) {
                const DevMat &s = c.mat[m];
                dsd += vmat[m] * strength_fn<A>(s.dsdf, pre, dam, A(0.), A(0.), A(0.), A(0.), s);
            }
            dam = awind(dam + sta2s * dsd * dt, A(0.0), A(1.0));
            tps = amin(tps + sta2s * dt, A(10.));
        }
        if (c.rp.tensile_failure) {
            const A sxx = s0, szz = s2, sxz = s1, sth = s3;
            const A ts = sqrt(sxz * sxz + A(0.25) * (sxx - szz) * (sxx - szz));
            A tmax = amax(A(0.5) * (sxx + szz) - ts, A(0.5) * (sxx + szz) + ts);
            tmax = amax(tmax, sth);
            if ((tmax - pre) > tensile) {
                // the reference divides by Min(e_pos[1], e_pos[2]) (centre y and scale x)
                const A dinc = A(0.4) * csd / A(dmin(PLN(c.f.e_pos, 1)[p], PLN(c.f.e_pos, 2)[p]));
                const A dold = dam;
                A third = pow(dold, A(1.0 / 3.));
                third += dinc;
                dam = awind(pow(third, A(3.0)), A(0.), A(1.));
                const A sfac = dold < A(0.98) ? (A(1.0) - dam) / (A(1.0) - dold) : A(0.0);
                s0 *= sfac; s1 *= sfac; s2 *= sfac; s3 *= sfac;
                ste2s *= sfac;
            }
        }
    }
    c.f.e_ste[p] = s0; PLN(c.f.e_ste, 1)[p] = s1; PLN(c.f.e_ste, 2)[p] = s2; PLN(c.f.e_ste, 3)[p] = s3;
    c.f.e_ste2s[p] = ste2s;
    c.f.e_sta2s[p] = sta2s;
    c.f.e_tps[p] = tps;
    c.f.e_dam[p] = dam;
    c.f.e_strength[p] = strength;
    if (EN && !(rho < SALEC_TOLRHO))
        energy_cell<R, NM, POR>(c, p, R(s0), R(s1), R(s2), R(s3), g0, g1, g2, g3, g4, pre);
}

// ============================================================ phase 8: vertex acceleration
// calculate_acc_default / calculate_acc_pml (src/velocity.c:9-340): surface integral of
// pressure + viscosity and deviatoric stress, hoop term, gravity and the nine-point
// Laplacian damping (ANC); the PML form also integrates the auxiliary v_alpha.
template <class R>
__global__ void SALEC_BOUNDS_ACCEL k_vertex_acceleration(const CtxT<R> c)
{
    using A = R;   // arithmetic of the stress divergence: FP64, or FP32 in the mixed form
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!vert_active(c, i, j)) return;
    const long long p = KIDX(i, j);
    const long long cl[4] = {KIDX(i - 1, j - 1), KIDX(i, j - 1), KIDX(i, j), KIDX(i - 1, j)};
    const bool pml = (c.rp.damp_type == 1 || c.rp.damp_type == 2);
    const A dt = A(c.scal->dt);
    A ax = A(0.), ay = A(0.), vmass = A(0.), vvol = A(0.);
    A sub[4];
    for (int k = 0; k < 4; ++k) sub[k] = GEO(c.g_v_subvol, k);
    A sigx = A(0.), sigy = A(0.);
    A alx = A(0.), aly = A(0.);
    if (pml) {
        for (int k = 0; k < 4; ++k) {
            sigx += A(0.25) * A(c.f.e_sigma[cl[k]]);
            sigy += A(0.25) * A(PLN(c.f.e_sigma, 1)[cl[k]]);
        }
        alx = c.f.v_alpha[p];
        aly = PLN(c.f.v_alpha, 1)[p];
    }
    const bool damped = pml && (sigx > A(0.) || sigy > A(0.));
    for (int k = 0; k < 4; ++k) {
        const long long e = cl[k];
        const A sfx = GEO(c.g_v_suf, 2 * k), sfy = GEO(c.g_v_suf, 2 * k + 1);
        const A lp = A(c.f.e_pre[e]) + A(c.f.e_q[e]);
        const A ste0 = c.f.e_ste[e], ste1 = PLN(c.f.e_ste, 1)[e], ste2 = PLN(c.f.e_ste, 2)[e],
                ste3 = PLN(c.f.e_ste, 3)[e];
        if (!pml) {
            A fpx = A(0.), fpy = A(0.);
            fpx += lp * sfx;
            fpy += lp * sfy;
            fpx += sub[k] * lp;
            const A sxx = ste0, szz = ste2, sxz = ste1, sth = ste3;
            A fsx = A(0.), fsy = A(0.);
            fsx += sfx * sxx; fsx += sfy * sxz;
            fsy += sfx * sxz; fsy += sfy * szz;
            fsx += sub[k] * sth;
            ax += A(-1.0) * fsx; ay += A(-1.0) * fsy;
            ax += A(1.0) * fpx; ay += A(1.0) * fpy;
        } else {
            const A lpr = PLN(c.f.e_dampref, 2)[e];
            A sxx = ste0 - lp, szz = ste2 - lp, sxz = ste1, sth = ste3 - lp;
            A fsx = A(0.), fsy = A(0.);
            fsx += sfx * sxx; fsx += sfy * sxz;
            fsy += sfx * sxz; fsy += sfy * szz;
            fsx += sub[k] * sth;
            ax += A(-1.0) * fsx; ay += A(-1.0) * fsy;
            if (damped) {
                sxx += lpr; szz += lpr; sth += lpr;
                A t0 = A(0.); t0 += sfx * (sigy * sxx); t0 += sfy * (sigx * sxz);
                alx += t0 * dt;
                A t1 = A(0.); t1 += sfx * (sigy * sxz); t1 += sfy * (sigx * szz);
                aly += t1 * dt;
                alx += (sigx + sigy) * sub[k] * sth * dt;
            }
        }
        const A lv = GEO(c.g_v_vol, 1 + k);
        vmass += lv * A(c.f.e_den[e]);
        vvol += lv;
    }
    if (damped) {
        alx -= A(c.rp.alpha_damp_x) * alx * dt;
        aly -= A(c.rp.alpha_damp_y) * aly * dt;
        ax += A(-1.0) * alx; ay += A(-1.0) * aly;
    }
    if (pml) { c.f.v_alpha[p] = alx; PLN(c.f.v_alpha, 1)[p] = aly; }

    A ancx = A(0.), ancy = A(0.);
    // where all nine weights are zero (outside the ANC band) the stencil sums to +0 and the term
    // is +0: the weights are not read there
    const bool lap = (c.lap_mask[(long long)j * (c.d.P >> 5) + (i >> 5)] >> (i & 31)) & 1u;
    if (!vert_pad(c, i, j) && lap) {
        A lvx = A(0.), lvy = A(0.);
        int k = 0;
        for (int dj = -1; dj <= 1; ++dj)
            for (int di = -1; di <= 1; ++di, ++k) {
                const long long q = KIDX(i + di, j + dj);
                const A w = PLN(c.f.v_laplace, k)[p];
                lvx += w * A(c.f.v_vel[q]);
                lvy += w * A(PLN(c.f.v_vel, 1)[q]);
            }
        const A sc = A(5.0e3) * sqrt(fabs(sub[0]) + fabs(sub[2]));
        ancx = sc * lvx;
        ancy = sc * lvy;
    }
    if (PLN(c.f.v_mass, 1)[p] >= A(1.)) { ancx = A(0.); ancy = A(0.); }
    if (vmass > A(SALEC_TOLRHO) * vvol) {
        const A s = A(1.0) / vmass;
        ax *= s; ay *= s;
        ax += A(1.0) * A(c.f.v_bf[p]); ay += A(1.0) * A(PLN(c.f.v_bf, 1)[p]);
        ax += A(c.rp.anc) * ancx; ay += A(c.rp.anc) * ancy;
    } else if (pml) {
        ax = c.f.v_bf[p]; ay = PLN(c.f.v_bf, 1)[p];
    } else {
        ax = A(0.); ay = A(0.);
    }
    if (fabs(ax) < A(c.rp.acceleration_min * 1)) ax = A(0.);
    if (fabs(ay) < A(c.rp.acceleration_min * 1)) ay = A(0.);
    c.f.v_acc[p] = ax;
    PLN(c.f.v_acc, 1)[p] = ay;
}

// ============================================================ phase 9: vertex displacement
// calculate_v_dis (src/sale2d.c:1238-1268).
template <class R>
__global__ void k_vertex_displacement(const CtxT<R> c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!vert_active(c, i, j)) return;
    const long long p = KIDX(i, j);
    const double dt = c.scal->dt;
    const double hdt2 = 0.5 * dt * dt;
    for (int k = 0; k < 2; ++k) {
        const double v = PLN(c.f.v_vel, k)[p], a = PLN(c.f.v_acc, k)[p];
        PLN(c.f.v_dis, k)[p] = dt * v + hdt2 * a;
        PLN(c.f.v_vel, k)[p] = v + dt * a;
    }
}

// ============================================================ phase 10: internal energy
// update_energy (src/sale2d.c:564-712) with the Wunnemann porosity update. After the vacuum
// test, every input of the cell is loaded in one batch (no load waits on another).
// The energy update of one interior cell p that is not vacuum, from the cell's new stress (s),
// its velocity gradient (g) and pressure as stored (widened from R to FP64).
template <class R, int NM, bool POR>
__device__ __forceinline__ void energy_cell(const CtxT<R> &c, long long p, double s0, double s1, double s2, double s3,
                                            double g0, double g1, double g2, double g3, double g4, double pre)
{
    constexpr int MM = NM > 0 ? NM : SALEC_MAXMAT;
    const int nmat = NM > 0 ? NM : c.d.nmat;
    double vm[MM], rm[MM], em[MM], pt[MM];
    #pragma unroll
    for (int m = 1; m < nmat; ++m) {
        vm[m] = PLN(c.f.m_vof, m)[p];
        rm[m] = PLN(c.f.m_den, m)[p];
        em[m] = PLN(c.f.m_eng, m)[p];
        pt[m] = POR ? PLN(c.f.m_pty, m)[p] : 1.0;
    }
    const double dt = c.scal->dt;
    const double q = c.f.e_q[p];
    const double div = c.f.e_div_vel[p];
    const double cvs_old = c.f.e_cvs[p];
    double sig = 0., ev0 = 0., ev1 = 0.;
    if (POR) {
        sig = c.f.e_sigma[p] + PLN(c.f.e_sigma, 1)[p];
        ev0 = c.f.e_vel[p];
        ev1 = PLN(c.f.e_vel, 1)[p];
    }
    const double lp = pre + q;
    const double dE_pre = -lp * div;
    const double dE_ste = s0 * g0 + s1 * (g1 + g2) + s2 * g3 + s3 * g4;
    double gam = 0.;
    #pragma unroll
    for (int m = 1; m < nmat; ++m)
        if (vm[m] > SALEC_TOLVOF) gam += vm[m] * c.mat[m].gamfrac / rm[m];
    const double dcvs = div - gam * (dE_pre + dE_ste);
    const double cvs = POR ? cvs_old : 0.0;
    #pragma unroll
    for (int m = 1; m < nmat; ++m) {
        if (vm[m] <= SALEC_TOLVOF || rm[m] <= SALEC_TOLRHO) {
            em[m] = 0.;
            if (POR) pt[m] = 1.;
        } else {
            const double fac = 1.0;
            em[m] = dmax(0., em[m] + (dE_pre + dE_ste) * dt * fac);
            if (POR) {
                double dpty = 0.;
                if (sig <= 0.) dpty = strength_fn(c.mat[m].porfunc, pt[m], cvs, pre, dcvs, ev0, ev1, c.mat[m]);
                pt[m] += dpty * dt;
                pt[m] = wind(pt[m], 1.0, c.mat[m].alphamax2);
            }
        }
        PLN(c.f.m_eng, m)[p] = em[m];
        if (POR) PLN(c.f.m_pty, m)[p] = pt[m];
    }
    // the reference updates e_cvs for every non-vacuum cell, with or without porosity
    c.f.e_cvs[p] = wind(cvs_old + dcvs * dt, -10.0, 10.0);
}

template <class R, int NM, bool POR>
__global__ void SALEC_BOUNDS_ENERGY k_energy(const CtxT<R> c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!cell_interior(c, i, j)) return;
    const long long p = KIDX(i, j);
    if (c.f.m_vof[p] > SALEC_TOLVOF || c.f.e_den[p] < SALEC_TOLRHO) return;
    energy_cell<R, NM, POR>(c, p, c.f.e_ste[p], PLN(c.f.e_ste, 1)[p], PLN(c.f.e_ste, 2)[p], PLN(c.f.e_ste, 3)[p],
                            c.f.e_grad_vel[p], PLN(c.f.e_grad_vel, 1)[p], PLN(c.f.e_grad_vel, 2)[p],
                            PLN(c.f.e_grad_vel, 3)[p], PLN(c.f.e_grad_vel, 4)[p], c.f.e_pre[p]);
}

// ============================================================ phase 11: tracers
// fl_update_node (src/tracer.c:52-175): bilinear interpolation of the vertex displacement
// (or, in cells with vacuum, ballistic motion under the interpolated vertex acceleration),
// ejecta tagging, peak pressure/temperature, and the cell index walk; a tracer that leaves
// the interior cells is deleted.
__device__ __forceinline__ double bilinear4(const double *v, double xi, double eta)
{
    // shape functions of the reference's IpB order: lb, rb, ru, lu (src/geometry/interpolate_fn.c:249)
    double r = 0;
    r += 0.25 * (1 - xi) * (1 - eta) * v[0];
    r += 0.25 * (1 + xi) * (1 - eta) * v[1];
    r += 0.25 * (1 + xi) * (1 + eta) * v[2];
    r += 0.25 * (1 - xi) * (1 + eta) * v[3];
    return r;
}

template <class R>
__global__ void k_tracers(const CtxT<R> c)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const Tracers &T = c.tr;
    if (t >= T.n || !T.alive[t]) return;
    const int k = T.cx[t], j = T.cy[t];
    const double dt = c.scal->dt;
    const long long vl[4] = {KIDX(k, j), KIDX(k + 1, j), KIDX(k + 1, j + 1), KIDX(k, j + 1)};
    // vertex coordinate lines of the reference's tracer list (v_pos along row 1 and column 1)
    const double vxk = c.f.v_pos[KIDX(k, 1)], vxk1 = c.f.v_pos[KIDX(k + 1, 1)];
    const double vyj = PLN(c.f.v_pos, 1)[KIDX(1, j)], vyj1 = PLN(c.f.v_pos, 1)[KIDX(1, j + 1)];
    double px = T.x[t], py = T.y[t];
    double rx = 1.0 * px + -1.0 * c.f.v_pos[vl[0]];
    double ry = 1.0 * py + -1.0 * PLN(c.f.v_pos, 1)[vl[0]];
    rx = rx / (vxk1 - vxk) * 2.0 - 1.0;
    ry = ry / (vyj1 - vyj) * 2.0 - 1.0;
    double q[4];
    if (c.f.m_vof[KIDX(k, j)] > SALEC_TOLVOF) {
        for (int a = 0; a < 4; ++a) q[a] = c.f.v_acc[vl[a]];
        const double bx = bilinear4(q, rx, ry);
        for (int a = 0; a < 4; ++a) q[a] = PLN(c.f.v_acc, 1)[vl[a]];
        const double by = bilinear4(q, rx, ry);
        const double hdt2 = 0.5 * dt * dt;
        const double dx = dt * T.vx[t] + hdt2 * bx;
        const double dy = dt * T.vy[t] + hdt2 * by;
        T.vx[t] += dt * bx;
        T.vy[t] += dt * by;
        px += 1.0 * dx;
        py += 1.0 * dy;
    } else {
        for (int a = 0; a < 4; ++a) q[a] = c.f.v_dis[vl[a]];
        const double dx = bilinear4(q, rx, ry);
        for (int a = 0; a < 4; ++a) q[a] = PLN(c.f.v_dis, 1)[vl[a]];
        const double dy = bilinear4(q, rx, ry);
        for (int a = 0; a < 4; ++a) q[a] = c.f.v_vel[vl[a]];
        const double ux = bilinear4(q, rx, ry);
        for (int a = 0; a < 4; ++a) q[a] = PLN(c.f.v_vel, 1)[vl[a]];
        const double uy = bilinear4(q, rx, ry);
        px += 1.0 * dx;
        py += 1.0 * dy;
        T.vx[t] = 1.0 * ux;
        T.vy[t] = 1.0 * uy;
    }
    T.x[t] = px;
    T.y[t] = py;
    if (T.matid[t] > 0 && py > c.rp.threshold_z) T.matid[t] = -T.matid[t];
    const long long e = KIDX(k, j);
    const double pre = c.f.e_pre[e], tem = c.f.e_tem[e];
    T.mpre[t] = (float)((double)T.mpre[t] > pre ? (double)T.mpre[t] : pre);
    T.mtem[t] = (float)((double)T.mtem[t] > tem ? (double)T.mtem[t] : tem);
    T.rec_pre[t] = pre;
    T.rec_tem[t] = tem;
    // GET_OFFSET2 walk of the cell index, then the interior test of fl_node_nei
    const int ox = px < vxk ? -1 : ((px < vxk1 && px >= vxk) ? 0 : 1);
    const int oy = py < vyj ? -1 : ((py < vyj1 && py >= vyj) ? 0 : 1);
    const int nk = k + ox, nj = j + oy;
    T.cx[t] = nk;
    T.cy[t] = nj;
    if (!(nk >= 2 && nk <= c.d.enx - 3 && nj >= 2 && nj <= c.d.eny - 3)) T.alive[t] = 0;
}

// ============================================================ phase 13: strength condition
// update_strength_condition (src/strength.c:351-376): e_cnd (cleared before the launch) counts
// the live tracers of the lubricating rows gy0 <= gy < gy1 in every cell. The counts are small
// integers, so the order of the atomic additions does not change them.
template <class R>
__global__ void k_strength_condition(const CtxT<R> c)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const Tracers &T = c.tr;
    if (t >= T.n || !T.alive[t]) return;
    const int gy = T.gy[t];
    if (gy < c.rp.tracer_lub_gy1 && gy >= c.rp.tracer_lub_gy0)
        atomicAdd(c.f.e_cnd + KIDX(T.cx[t], T.cy[t]), (R)1.0);
}

// ============================================================ phase 12: face flux volumes
// calculate_flux_mixed (src/advect.c:861-1136) with _calculate_flux_set_bphi (:1138-1223):
// swept face volumes, geometric cut-line reconstruction of the primary material, algebraic
// (MSTACS) fractions of the others, and the upwind state written on each outflow face.
// A face with zero swept volume gets zero material volumes, which stands in for the
// reference's clean_flux (src/advect.c:597-626): the other members of such a record are only
// ever multiplied by those zero volumes.
// Upwind record of one face of cell p (_calculate_flux_set_bphi, src/advect.c:1138-1223): the
// face is written by the cell it flows out of; a face with zero swept volume gets zero material
// volumes (see k_flux).
template <class R, int NM, bool POR, int MM>
__device__ __forceinline__ void store_face(const CtxT<R> &c, double *f, double vol, const double (&flux)[MM][4], int k,
                                           long long p, int nmat)
{
    if (vol > 0.) return;
    const long long PL = c.d.PL;
    if (vol == 0.) {
#pragma unroll
        for (int m = 0; m < nmat; ++m) f[m * PL] = 0.0;
        return;
    }
#pragma unroll
    for (int m = 0; m < nmat; ++m) {
        f[m * PL] = flux[m][k];
        f[(m + nmat) * PL] = PLN(c.f.m_den, m)[p];
        f[(m + 2 * nmat) * PL] = PLN(c.f.m_eng, m)[p];
    }
    const int b = 3 * nmat;
    f[(b + 0) * PL] = c.f.e_vel[p];
    f[(b + 1) * PL] = PLN(c.f.e_vel, 1)[p];
#pragma unroll
    for (int q = 0; q < 4; ++q) f[(b + 2 + q) * PL] = 1.0 * PLN(c.f.e_ste, q)[p];
    f[(b + 6) * PL] = 1.0 * c.f.e_dam[p];
    f[(b + 7) * PL] = 1.0 * c.f.e_tps[p];
    f[(b + 8) * PL] = 1.0 * c.f.e_vib[p];
    f[(b + 9) * PL] = 1.0 * c.f.e_ejt[p];
    if (POR) {
        f[(b + 10) * PL] = 1.0 * c.f.e_cvs[p];
#pragma unroll
        for (int m = 0; m < nmat; ++m) f[(b + 11 + m) * PL] = PLN(c.f.m_pty, m)[p];
    }
}

// Cell t of the two-cell pad ring, t < 4 enx + 4 (eny - 4): the two bottom rows, the two top
// rows, then the four pad cells of each row between them (needs enx, eny >= 5).
__device__ __forceinline__ void pad_ring_cell(int t, int enx, int eny, int &i, int &j)
{
    if (t < 2 * enx) {
        j = t / enx; i = t - j * enx;
    } else if (t < 4 * enx) {
        const int u = t - 2 * enx, r = u / enx;
        j = eny - 2 + r; i = u - r * enx;
    } else {
        const int u = t - 4 * enx, r = u >> 2, k = u & 3;
        j = 2 + r; i = k < 2 ? k : enx - 4 + k;
    }
}

// pass 0: interior cells; pass 1: pad cells (after the ghost fills of m_den, m_eng, ...), over
// the whole grid; pass 2: the same pad cells, one thread each (1-D grid over the pad ring);
// pass 3: every cell, after the ghost fills. No cell's flux reads a ghost member the fills write
// except the pad cells' own, and no flux writes what the fills read, so pass 3 computes what
// passes 0 and 2 around the fills compute, in one launch whose pad cells hide in the interior's
// waves.
template <class R, int NM, bool POR>
__global__ void SALEC_BOUNDS_FLUX k_flux(const CtxT<R> c, int pass)
{
    int i, j;
    if (pass == 2) {
        const int t = (blockIdx.x * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
        if (t >= 4 * c.d.enx + 4 * (c.d.eny - 4)) return;
        pad_ring_cell(t, c.d.enx, c.d.eny, i, j);
    } else {
        i = blockIdx.x * blockDim.x + threadIdx.x;
        j = blockIdx.y * blockDim.y + threadIdx.y;
        if (i >= c.d.enx || j >= c.d.eny) return;
        if (pass != 3 && (pass == 0) != cell_interior(c, i, j)) return;
    }
    constexpr int MM = NM > 0 ? NM : SALEC_MAXMAT;
    const int nmat = NM > 0 ? NM : c.d.nmat;
    const long long p = KIDX(i, j);
    const long long vl[4] = {KIDX(i, j), KIDX(i + 1, j), KIDX(i + 1, j + 1), KIDX(i, j + 1)};
    double px[4], py[4], dx[4], dy[4];
    #pragma unroll
    for (int k = 0; k < 4; ++k) {
        px[k] = c.f.v_pos[vl[k]]; py[k] = PLN(c.f.v_pos, 1)[vl[k]];
        dx[k] = c.f.v_dis[vl[k]]; dy[k] = PLN(c.f.v_dis, 1)[vl[k]];
    }
    const double lv = swept_volume(px[0], py[0], px[3], py[3], dx[0], dy[0], dx[3], dy[3]);
    const double rv = swept_volume(px[2], py[2], px[1], py[1], dx[2], dy[2], dx[1], dy[1]);
    const double bv = swept_volume(px[1], py[1], px[0], py[0], dx[1], dy[1], dx[0], dy[0]);
    const double uv = swept_volume(px[3], py[3], px[2], py[2], dx[3], dy[3], dx[2], dy[2]);
    double vof[MM];
    #pragma unroll
    for (int m = 0; m < nmat; ++m) vof[m] = PLN(c.f.m_vof, m)[p];
    const double evol = c.f.e_vol[p];
    double flux[MM][4];
    #pragma unroll
    for (int m = 0; m < nmat; ++m) flux[m][0] = flux[m][1] = flux[m][2] = flux[m][3] = 0.;

    // primary material: vacuum, or the largest fraction when the cell holds no vacuum; selected
    // with compare loops so that the per-material arrays stay in registers
    int prim = 0;
    double vprim = vof[0];
    if (vof[0] < SALEC_TOLVOF) {
#pragma unroll
        for (int m = 1; m < nmat; ++m)
            if (vof[m] > vprim) { prim = m; vprim = vof[m]; }
    }

    double wpt[4];
    if (vprim > 1.0 - SALEC_TOLVOF) {
#pragma unroll
        for (int m = 0; m < nmat; ++m)
            if (m == prim) {
                flux[m][0] = dmin(lv, 0);
                flux[m][2] = -1.0 * dmin(rv, 0);
                flux[m][1] = dmin(bv, 0);
                flux[m][3] = -1.0 * dmin(uv, 0);
            }
        const double w = prim == 0 ? 1.0 : -0.25;
        wpt[0] = wpt[1] = wpt[2] = wpt[3] = w;
    } else {
        double grd[12];
        #pragma unroll
        for (int k = 0; k < 8; ++k) grd[k] = GEO(c.g_e_grad, k);
        double gx = 0., gy = 0.;
        {
            const auto *vv = PLN(c.f.v_vof, prim);
            double vq[4];
            #pragma unroll
            for (int k = 0; k < 4; ++k) vq[k] = vv[vl[k]];
            #pragma unroll
            for (int k = 0; k < 4; ++k) gx += vq[k] * grd[k];
            #pragma unroll
            for (int k = 0; k < 4; ++k) gy += vq[k] * grd[4 + k];
        }
        normalise2(gx, gy);
        double ca = PLN(c.f.e_pos, 2)[p] * fabs(gx);
        double cb = PLN(c.f.e_pos, 3)[p] * fabs(gy);
        if (ca < cb) { double t = ca; ca = cb; cb = t; }
        const double dstar = cut_length(vprim, ca, cb);
        double lw[4];
        #pragma unroll
        for (int k = 0; k < 4; ++k) { double s = 0.; s += gx * px[k]; s += gy * py[k]; lw[k] = s; }
        const double mw = dmax(dmax(lw[0], lw[1]), dmax(lw[2], lw[3]));
        #pragma unroll
        for (int k = 0; k < 4; ++k) lw[k] = lw[k] - mw + dstar;
        if (prim == 0) { for (int k = 0; k < 4; ++k) wpt[k] = lw[k]; }
        else wpt[0] = wpt[1] = wpt[2] = wpt[3] = -0.25;
        double fp[4];
        fp[0] = face_ratio(lw[3], lw[0]);
        fp[2] = face_ratio(lw[2], lw[1]);
        fp[1] = face_ratio(lw[0], lw[1]);
        fp[3] = face_ratio(lw[3], lw[2]);
        double cr = dmin(lv, 0.0) + dmin(rv, 0) + dmin(bv, 0) + dmin(uv, 0);
        cr = fabs(cr) / evol;
        // neighbours l, b, r, u (the cell itself where the neighbour is off the mesh)
        long long nb[4] = {KIDX(i - 1, j), KIDX(i, j - 1), KIDX(i + 1, j), KIDX(i, j + 1)};
        if (i - 1 < 0) nb[0] = p;
        if (j - 1 < 0) nb[1] = p;
        if (i + 1 >= c.d.enx) nb[2] = p;
        if (j + 1 >= c.d.eny) nb[3] = p;
        // face normals l, b, r, u
        const long long fb[4] = {KIDX(i, j), KIDX(i, j), KIDX(i + 1, j), KIDX(i, j + 1)};
        double fnx[4], fny[4];
        fnx[0] = c.f.bx_normal[fb[0]]; fny[0] = PLN(c.f.bx_normal, 1)[fb[0]];
        fnx[2] = c.f.bx_normal[fb[2]]; fny[2] = PLN(c.f.bx_normal, 1)[fb[2]];
        fnx[1] = c.f.by_normal[fb[1]]; fny[1] = PLN(c.f.by_normal, 1)[fb[1]];
        fnx[3] = c.f.by_normal[fb[3]]; fny[3] = PLN(c.f.by_normal, 1)[fb[3]];
        double fnp[MM][4];
        double snp[4] = {0., 0., 0., 0.};
        #pragma unroll
        for (int m = 0; m < nmat; ++m) fnp[m][0] = fnp[m][1] = fnp[m][2] = fnp[m][3] = 0.;
        #pragma unroll
        for (int m = 1; m < nmat; ++m) {
            if (m == prim) continue;
            const auto *vv = PLN(c.f.v_vof, m);
            double vq[4];
            #pragma unroll
            for (int k = 0; k < 4; ++k) vq[k] = vv[vl[k]];
            double ngx = 0., ngy = 0.;
            #pragma unroll
            for (int k = 0; k < 4; ++k) ngx += vq[k] * grd[k];
            #pragma unroll
            for (int k = 0; k < 4; ++k) ngy += vq[k] * grd[4 + k];
            normalise2(ngx, ngy);
            const double *ev = PLN(c.f.m_vof, m);
            const double up[4] = {ev[nb[0]], ev[nb[1]], ev[nb[2]], ev[nb[3]]};
            const double ac[4] = {up[2], up[3], up[0], up[1]};
            #pragma unroll
            for (int k = 0; k < 4; ++k) {
                fnp[m][k] = algebraic_ratio(up[k], vof[m], ac[k], cr, fnx[k], fny[k], ngx, ngy);
                snp[k] += fnp[m][k];
            }
        }
        #pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (snp[k] > SALEC_TOLVOF) {
                #pragma unroll
                for (int m = 1; m < nmat; ++m) fnp[m][k] = fnp[m][k] / snp[k];
            } else {
                #pragma unroll
                for (int m = 1; m < nmat; ++m) fnp[m][k] = vof[m] / (1.0 - vprim);
            }
        }
        #pragma unroll
        for (int m = 0; m < nmat; ++m) {
            if (m == prim) {
                flux[m][0] = dmin(lv, 0.0) * fp[0];
                flux[m][2] = -1.0 * dmin(rv, 0.0) * fp[2];
                flux[m][1] = dmin(bv, 0.0) * fp[1];
                flux[m][3] = -1.0 * dmin(uv, 0.0) * fp[3];
            } else {
                flux[m][0] = dmin(lv, 0.0) * (1.0 - fp[0]) * fnp[m][0];
                flux[m][2] = -1.0 * dmin(rv, 0.0) * (1.0 - fp[2]) * fnp[m][2];
                flux[m][1] = dmin(bv, 0.0) * (1.0 - fp[1]) * fnp[m][1];
                flux[m][3] = -1.0 * dmin(uv, 0.0) * (1.0 - fp[3]) * fnp[m][3];
            }
        }
    }
    #pragma unroll
    for (int k = 0; k < 4; ++k) PLN(c.f.e_wpt, k)[p] = wpt[k];

    // cap the out-flux of each material by its content
    #pragma unroll
    for (int m = 1; m < nmat; ++m) {
        double d = 0.;
        d += flux[m][0] * 1.0; d += flux[m][1] * 1.0; d += flux[m][2] * -1.0; d += flux[m][3] * -1.0;
        const double out = -1.0 * d;
        if (out > vof[m] * evol) {
            const double s = vof[m] * evol / out;
            #pragma unroll
            for (int k = 0; k < 4; ++k) flux[m][k] *= s;
        }
    }

    // faces l, b, r, u
    store_face<R, NM, POR>(c, c.f.bx_phi + KIDX(i, j), lv, flux, 0, p, nmat);
    store_face<R, NM, POR>(c, c.f.by_phi + KIDX(i, j), bv, flux, 1, p, nmat);
    store_face<R, NM, POR>(c, c.f.bx_phi + KIDX(i + 1, j), rv, flux, 2, p, nmat);
    store_face<R, NM, POR>(c, c.f.by_phi + KIDX(i, j + 1), uv, flux, 3, p, nmat);
}

// ============================================================ phase 14: remap + damping + EOS
// advect_flux_default (src/advect.c:26-302), damp_on_cell (src/velocity.c:356-767),
// ejecta_flow (src/ejecta.c:65-133) and update_state (src/sale2d.c:1635-1742), fused per cell:
// the damping reads only its own cell, and the EOS reads the damped material state.
// The cell's state travels through remap, damping, ejecta drag and EOS in registers: each
// member is loaded once and stored once per step.
template <int NM, bool POR>
struct CellState {
    static constexpr int MM = NM > 0 ? NM : SALEC_MAXMAT;
    double vof[MM], rho[MM], eng[MM], pty[MM];
    double dvx, dvy, st[4], dam, tps, vib, ejt, cvs, eden;
};

template <class R, int NM, bool POR>
__device__ __forceinline__ void load_cell(const CtxT<R> &c, long long p, CellState<NM, POR> &s)
{
    const int nmat = NM > 0 ? NM : c.d.nmat;
    #pragma unroll
    for (int m = 0; m < nmat; ++m) {
        s.vof[m] = PLN(c.f.m_vof, m)[p];
        s.rho[m] = PLN(c.f.m_den, m)[p];
        s.eng[m] = PLN(c.f.m_eng, m)[p];
        s.pty[m] = POR ? PLN(c.f.m_pty, m)[p] : 1.0;
    }
    s.dvx = c.f.e_dvel[p];
    s.dvy = PLN(c.f.e_dvel, 1)[p];
    #pragma unroll
    for (int q = 0; q < 4; ++q) s.st[q] = PLN(c.f.e_ste, q)[p];
    s.dam = c.f.e_dam[p];
    s.tps = c.f.e_tps[p];
    s.vib = c.f.e_vib[p];
    s.ejt = c.f.e_ejt[p];
    s.cvs = POR ? c.f.e_cvs[p] : 0.0;
    s.eden = c.f.e_den[p];
}

template <class R, int NM, bool POR>
__device__ __forceinline__ void store_cell(const CtxT<R> &c, long long p, const CellState<NM, POR> &s, bool den)
{
    const int nmat = NM > 0 ? NM : c.d.nmat;
    #pragma unroll
    for (int m = 0; m < nmat; ++m) {
        PLN(c.f.m_vof, m)[p] = s.vof[m];
        PLN(c.f.m_den, m)[p] = s.rho[m];
        PLN(c.f.m_eng, m)[p] = s.eng[m];
        if (POR) PLN(c.f.m_pty, m)[p] = s.pty[m];
    }
    c.f.e_dvel[p] = s.dvx;
    PLN(c.f.e_dvel, 1)[p] = s.dvy;
    #pragma unroll
    for (int q = 0; q < 4; ++q) PLN(c.f.e_ste, q)[p] = s.st[q];
    c.f.e_dam[p] = s.dam;
    c.f.e_tps[p] = s.tps;
    c.f.e_vib[p] = s.vib;
    c.f.e_ejt[p] = s.ejt;
    if (POR) c.f.e_cvs[p] = s.cvs;
    if (den) c.f.e_den[p] = s.eden;
}

// advect_flux_default (src/advect.c:26-302) for one interior cell, into registers. The loads
// that do not depend on the flow (the cell's own state and the material volumes of its four
// faces) are all issued before the first dependent one.
template <class R, int NM, bool POR, bool P3>
__device__ __forceinline__ void remap_cell(const CtxT<R> &c, int i, int j, long long p, CellState<NM, POR> &s)
{
    constexpr int MM = CellState<NM, POR>::MM;
    const int nmat = NM > 0 ? NM : c.d.nmat;
    const int phi = 3 * nmat + 10 + (POR ? nmat + 1 : 0);
    const long long PL = c.d.PL;
    constexpr bool por = POR;
    const double *face[4] = {c.f.bx_phi + KIDX(i, j), c.f.by_phi + KIDX(i, j), c.f.bx_phi + KIDX(i + 1, j),
                             c.f.by_phi + KIDX(i, j + 1)};
    const double dir[4] = {1.0, 1.0, -1.0, -1.0};
    double fv[4][MM];
    #pragma unroll
    for (int k = 0; k < 4; ++k)
        #pragma unroll
        for (int m = 0; m < nmat; ++m) fv[k][m] = face[k][m * PL];
    double vof[MM], rho[MM], eng[MM], pty[MM];
    #pragma unroll
    for (int m = 0; m < nmat; ++m) {
        vof[m] = PLN(c.f.m_vof, m)[p];
        rho[m] = PLN(c.f.m_den, m)[p];
        eng[m] = PLN(c.f.m_eng, m)[p];
        pty[m] = por ? PLN(c.f.m_pty, m)[p] : 1.0;
    }
    const double evol = c.f.e_vol[p];
    const double eden0 = c.f.e_den[p];
    double st0[4];
    #pragma unroll
    for (int q = 0; q < 4; ++q) st0[q] = PLN(c.f.e_ste, q)[p];
    const double dam0 = c.f.e_dam[p], tps0 = c.f.e_tps[p], vib0 = c.f.e_vib[p], ejt0 = c.f.e_ejt[p];
    const double cvs0 = por ? c.f.e_cvs[p] : 0.0;

    // advect_flux_pml3 (src/advect.c:304-594) differs from the default remap in the PML
    // auxiliaries e_beta (fluxes of mass, energy and momentum weighted by the layer's sigma,
    // accumulated here and damped below), in its clamps and low-density test, and in leaving the
    // porosity state alone
    constexpr bool p3 = P3;   // damping = pml3
    double sgx = 0., sgy = 0., eb0 = 0., eb1 = 0., eb2 = 0., eb3 = 0.;
    if (p3) {
        sgx = c.f.e_sigma[p];
        sgy = PLN(c.f.e_sigma, 1)[p];
        eb0 = c.f.e_beta[p];
        eb1 = PLN(c.f.e_beta, 1)[p];
        eb2 = PLN(c.f.e_beta, 2)[p];
        eb3 = PLN(c.f.e_beta, 3)[p];
    }
    const bool p3_layer = p3 && (sgx > 0. || sgy > 0.);
    const double para[4] = {-sgy, -sgx, -sgy, -sgx};   // faces l, b, r, u

    double dphi[4 * MM + 11];
    #pragma unroll
    for (int q = 0; q < phi; ++q) dphi[q] = 0.;
    const int b = 3 * nmat;
    #pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double *f = face[k];
        #pragma unroll
        for (int m = 0; m < nmat; ++m) {
            const double mv = dir[k] * fv[k][m];
            if (mv == 0.0) continue;   // adds only signed zeros to dphi and e_beta (see k_flux)
            const double rho_f = f[(m + nmat) * PL];
            dphi[m] += mv;
            dphi[m + nmat] += mv * rho_f;
            dphi[m + 2 * nmat] += mv * f[(m + 2 * nmat) * PL];
            const double fm = mv * rho_f;
            #pragma unroll
            for (int q = 0; q < 10; ++q) dphi[b + q] += fm * f[(b + q) * PL];
            if (por && !p3) {
                dphi[b + 10] += (f[(b + 10) * PL]) * (mv * rho_f);
                dphi[m + b + 11] += (f[(m + b + 11) * PL]) * (mv * rho_f);
            }
            if (p3_layer) {
                eb0 += mv * rho_f * para[k];
                eb1 += mv * f[(m + 2 * nmat) * PL] * para[k];
                eb2 += mv * rho_f * para[k] * f[b * PL];
                eb3 += mv * rho_f * para[k] * f[(b + 1) * PL];
            }
        }
    }
    // sphi = cell content + face fluxes, accumulated in place in dphi (the content of each
    // member is formed as 0 + term, then the flux sum is added, as in the reference)
    double emass = evol * eden0;
    double *sphi = dphi;
    #pragma unroll
    for (int m = 0; m < nmat; ++m) {
        sphi[m] = (0.0 + vof[m] * evol) + 1.0 * dphi[m];
        sphi[m + nmat] = (0.0 + vof[m] * evol * rho[m]) + 1.0 * dphi[m + nmat];
        sphi[m + 2 * nmat] = (0.0 + vof[m] * evol * eng[m]) + 1.0 * dphi[m + 2 * nmat];
    }
    sphi[b] = 0.0 + 1.0 * dphi[b];
    sphi[b + 1] = 0.0 + 1.0 * dphi[b + 1];
    #pragma unroll
    for (int q = 0; q < 4; ++q) sphi[b + 2 + q] = (0.0 + emass * st0[q]) + 1.0 * dphi[b + 2 + q];
    sphi[b + 6] = emass * dam0 + 1.0 * dphi[b + 6];
    sphi[b + 7] = emass * tps0 + 1.0 * dphi[b + 7];
    sphi[b + 8] = emass * vib0 + 1.0 * dphi[b + 8];
    sphi[b + 9] = emass * ejt0 + 1.0 * dphi[b + 9];
    if (por && !p3) {
        sphi[b + 10] = emass * cvs0 + 1.0 * dphi[b + 10];
        #pragma unroll
        for (int m = 0; m < nmat; ++m) sphi[b + 11 + m] = vof[m] * evol * rho[m] * pty[m] + 1.0 * dphi[b + 11 + m];
    }
    if (p3 && sgx + sgy > 0.) {
        const double adxy = c.rp.alpha_damp_x + c.rp.alpha_damp_y;
        const double dt = c.scal->dt;
        eb0 += -1.0 * adxy * eb0 * dt;
        eb1 += -1.0 * adxy * eb1 * dt;
        eb2 += -1.0 * adxy * eb2 * dt;
        eb3 += -1.0 * adxy * eb3 * dt;
        if (sphi[0] < SALEC_TOLVOF) {
            sphi[b] += eb2 * dt;
            sphi[b + 1] += eb3 * dt;
        }
        int mf = -1;   // first material (from 1) with a positive volume
        #pragma unroll
        for (int m = (NM > 0 ? NM : SALEC_MAXMAT) - 1; m >= 1; --m)
            if (m < nmat && sphi[m] > SALEC_TOLVOF) mf = m;
        #pragma unroll
        for (int m = 1; m < nmat; ++m)
            if (m == mf) {
                sphi[m + nmat] += eb0 * dt;
                sphi[m + 2 * nmat] += eb1 * dt;
            }
    }
    if (p3_layer) {
        c.f.e_beta[p] = eb0;
        PLN(c.f.e_beta, 1)[p] = eb1;
        PLN(c.f.e_beta, 2)[p] = eb2;
        PLN(c.f.e_beta, 3)[p] = eb3;
    }
    double zeta = 0.0;
    emass = 0.;
    #pragma unroll
    for (int m = 0; m < nmat; ++m) {
        if (sphi[m] < 0. || (p3 && sphi[m + nmat] < 0.)) { sphi[m] = 0.; sphi[m + nmat] = 0.; }
        if (m == 0) continue;
        zeta += sphi[m];
        emass += sphi[m + nmat];
    }
    if (zeta > evol * (1.0 - SALEC_TOLVOF) || (zeta > 0. && sphi[0] < evol * SALEC_TOLVOF)) {
        const double sc = 1.0 / zeta;
        #pragma unroll
        for (int m = 0; m < nmat; ++m) vof[m] = sc * sphi[m];
        vof[0] = 0.0;
    } else if (zeta < evol * SALEC_TOLVOF) {
        #pragma unroll
        for (int m = 0; m < nmat; ++m) vof[m] = 0.;
        vof[0] = 1.0;
    } else if (c.rp.partpres) {
        const double sc = 1.0 / (zeta + sphi[0]);
        #pragma unroll
        for (int m = 0; m < nmat; ++m) vof[m] = sc * sphi[m];
    } else {
        sphi[0] = evol - zeta;
        const double sc = 1.0 / evol;
        #pragma unroll
        for (int m = 0; m < nmat; ++m) vof[m] = sc * sphi[m];
    }
    #pragma unroll
    for (int m = 1; m < nmat; ++m) {
        if (vof[m] < SALEC_TOLVOF || (!p3 && sphi[m + nmat] < SALEC_TOLRHO * SALEC_TOLVOF * evol)) {
            eng[m] = 0.0; rho[m] = 0.0; vof[m] = 0.0;
            if (por && !p3) pty[m] = 1.0;
        } else {
            eng[m] = sphi[m + 2 * nmat] / (vof[m] * evol);
            rho[m] = sphi[m + nmat] / (vof[m] * evol);
            if (por && !p3) pty[m] = sphi[b + 11 + m] / sphi[m + nmat];
        }
    }
    double dvx, dvy, st[4], dam, tps, vib, ejt, cvs = cvs0;
    if (emass > SALEC_TOLRHO * evol) {
        const double sc = 1.0 / emass;
        dvx = sc * sphi[b]; dvy = sc * sphi[b + 1];
        #pragma unroll
        for (int q = 0; q < 4; ++q) st[q] = sc * sphi[b + 2 + q];
        dam = sphi[b + 6] / emass;
        tps = sphi[b + 7] / emass;
        vib = sphi[b + 8] / emass;
        ejt = sphi[b + 9] / emass;
        if (por && !p3) cvs = sphi[b + 10] / emass;
    } else {
        dvx = dvy = 0.;
        st[0] = st[1] = st[2] = st[3] = 0.;
        dam = tps = vib = ejt = 0.;
        if (por && !p3) cvs = 0.;
    }
    double eden = emass / evol;
    tps = wind(tps, 0.0, 10.0);
    dam = wind(dam, 0.0, 1.0);
    ejt = wind(ejt, 0.0, 1.0);
    if (por && !p3)
        #pragma unroll
        for (int m = 1; m < nmat; ++m) pty[m] = wind(pty[m], 1.0, c.mat[m].alphamax2);
    if (eden < c.rp.density_cutoff || (!p3 && eden < 10.0 * c.rp.density_cutoff * (1.0 - vof[0]))) {
        #pragma unroll
        for (int m = 0; m < nmat; ++m) { vof[m] = 0.; rho[m] = 0.; eng[m] = 0.; }
        vof[0] = 1.0;
        dvx = dvy = 0.;
        st[0] = st[1] = st[2] = st[3] = 0.;
        dam = tps = vib = ejt = 0.;
        if (por && !p3) {
            cvs = 0.;
            #pragma unroll
            for (int m = 1; m < nmat; ++m) pty[m] = 1.0;
        }
    }
    #pragma unroll
    for (int m = 0; m < nmat; ++m) { s.vof[m] = vof[m]; s.rho[m] = rho[m]; s.eng[m] = eng[m]; s.pty[m] = pty[m]; }
    s.dvx = dvx; s.dvy = dvy;
    #pragma unroll
    for (int q = 0; q < 4; ++q) s.st[q] = st[q];
    s.dam = dam; s.tps = tps; s.vib = vib; s.ejt = ejt; s.cvs = cvs; s.eden = eden;
}

// The lowest material index whose volume fraction is at least (strict: above) 1 - TOLVOF, or
// -1: the material the damping of a full cell acts on.
template <int NM, bool POR>
__device__ __forceinline__ int first_material(const CellState<NM, POR> &s, int nmat, bool strict)
{
    int mf = -1;
    #pragma unroll
    for (int m = (NM > 0 ? NM : SALEC_MAXMAT) - 1; m >= 1; --m) {
        if (m >= nmat) continue;
        const bool full = strict ? s.vof[m] > 1.0 - SALEC_TOLVOF : s.vof[m] >= 1.0 - SALEC_TOLVOF;
        if (full) mf = m;
    }
    return mf;
}

// damp_on_cell (src/velocity.c:356-767) on the register state; the auxiliary e_alpha is read
// and written here. Returns whether the cell's state changed.
template <class R, int NM, bool POR>
__device__ __forceinline__ bool damp_cell(const CtxT<R> &c, long long p, double dt, CellState<NM, POR> &s)
{
    const int nmat = NM > 0 ? NM : c.d.nmat;
    const int ty = c.rp.damp_type;
    if (ty == 4 || ty == 5) return false;
    if (s.vof[0] > SALEC_TOLVOF) return false;
    const double sx = c.f.e_sigma[p], sy = PLN(c.f.e_sigma, 1)[p];
    const double d0 = c.f.e_dampref[p], d1 = PLN(c.f.e_dampref, 1)[p];
    constexpr bool por = POR;
    if (ty == 0) {
        // damp_on_cell_pml (src/velocity.c:378-467)
        double ax = c.f.e_alpha[p], ay = PLN(c.f.e_alpha, 1)[p];
        const double pre = c.f.e_pre[p];
        if (sy > 0.0) {
            ay += (sy * PLN(c.f.e_grad_vel, 0)[p] + sy * PLN(c.f.e_grad_vel, 4)[p] - c.rp.alpha_damp_y * ay) * dt;
            s.dvy += -1.0 * sy * PLN(c.f.e_vel, 1)[p] * dt;
            const int mf = first_material(s, nmat, false);
            #pragma unroll
            for (int m = 1; m < nmat; ++m) {
                if (m != mf) continue;
                const double pt = por ? s.pty[m] : 1.0;
                const double rd = (-sy * (s.rho[m] - d0) - d0 * ay) * dt;
                const double ed = (-sy * (s.eng[m] - d1) - pre * ay) * dt;
                s.rho[m] += rd / pt;
                s.eng[m] += ed / pt;
            }
        }
        if (sx > 0.0) {
            ax += (sx * PLN(c.f.e_grad_vel, 3)[p] + sx * PLN(c.f.e_grad_vel, 4)[p] - c.rp.alpha_damp_x * ax) * dt;
            s.dvx += -1.0 * sx * c.f.e_vel[p] * dt;
            const int mf = first_material(s, nmat, true);
            #pragma unroll
            for (int m = 1; m < nmat; ++m) {
                if (m != mf) continue;
                const double pt = por ? s.pty[m] : 1.0;
                const double rd = (-sx * (s.rho[m] - d0) - d0 * (ax + ay)) * dt;
                const double ed = (-sx * (s.eng[m] - d1) - pre * (ax + ay)) * dt;
                s.rho[m] += rd / pt;
                s.eng[m] += ed / pt;
            }
        }
        c.f.e_alpha[p] = ax;
        PLN(c.f.e_alpha, 1)[p] = ay;
        return sx > 0.0 || sy > 0.0;
    } else if (ty == 1 || ty == 2) {
        // damp_on_cell_pml2 / _pml3 (src/velocity.c:471-654)
        if (!(sy > 0.0 || sx > 0.0)) return false;
        const double ss = sx + sy;
        s.dvx += -1.0 * ss * c.f.e_vel[p] * dt;
        s.dvy += -1.0 * ss * PLN(c.f.e_vel, 1)[p] * dt;
        double ax = c.f.e_alpha[p], ay = PLN(c.f.e_alpha, 1)[p];
        const double g0 = PLN(c.f.e_grad_vel, 0)[p], g1 = PLN(c.f.e_grad_vel, 1)[p], g2 = PLN(c.f.e_grad_vel, 2)[p],
                     g3 = PLN(c.f.e_grad_vel, 3)[p], g4 = PLN(c.f.e_grad_vel, 4)[p];
        const double adx = c.rp.alpha_damp_x, ady = c.rp.alpha_damp_y;
        ax += (sy * g0 + sy * g4 - ady * ax) * dt + (sx * g3 + sx * g4 - adx * ax) * dt;
        const double lp = c.f.e_pre[p] + c.f.e_q[p] - PLN(c.f.e_dampref, 2)[p];
        const double t0 = s.st[0], t1 = s.st[1], t2 = s.st[2], t3 = s.st[3];
        const double sd = (t0 - lp) * sy * g0 + t1 * (sy * g1 + sx * g2) + (t2 - lp) * sx * g3 + (sy + sx) * t3 * g4;
        ay += -1.0 * sd * dt - 1.0 * (adx + ady) * ay * dt;
        c.f.e_alpha[p] = ax;
        PLN(c.f.e_alpha, 1)[p] = ay;
        const int mf = first_material(s, nmat, false);
        #pragma unroll
        for (int m = 1; m < nmat; ++m) {
            if (m != mf) continue;
            if (ty == 1) {
                const double pt = por ? s.pty[m] : 1.0;
                const double rd = (-(sx + sy) * (s.rho[m] - d0) - d0 * ax) * dt;
                const double ed = (-(sx + sy) * (s.eng[m] - d1) - ay) * dt;
                s.rho[m] += rd / pt;
                s.eng[m] += ed / pt;
            } else {
                const double rd = (-(sx + sy) * (s.rho[m] - d0)) * dt;
                const double ed = (-(sx + sy) * (s.eng[m] - d1) - ay) * dt;
                s.rho[m] += rd;
                s.eng[m] += ed;
            }
        }
        return true;
    } else if (ty == 3) {
        // damp_on_cell_sbc (src/velocity.c:658-767); "+=" in y and "=" in x as in the reference
        bool changed = false;
        if (sy < 1.0) {
            #pragma unroll
            for (int m = 1; m < nmat; ++m) {
                if (s.vof[m] < SALEC_TOLVOF) continue;
                const double dd = s.rho[m] - d0, de = s.eng[m] - d1;
                s.rho[m] += dd * sy + d0;
                s.eng[m] += de * sy + d1;
                changed = true;
            }
        }
        if (sx < 1.0) {
            #pragma unroll
            for (int m = 1; m < nmat; ++m) {
                if (s.vof[m] < SALEC_TOLVOF) continue;
                const double dd = s.rho[m] - d0, de = s.eng[m] - d1;
                s.rho[m] = dd * sx + d0;
                s.eng[m] = de * sx * sx + d1;
                changed = true;
            }
        }
        return changed;
    }
    return false;
}

// ejecta_flow (src/ejecta.c:65-133); launched only when resistance or friction is positive
template <class R, int NM, bool POR>
__device__ __forceinline__ void ejecta_drag_cell(const CtxT<R> &c, int i, int j, long long p, double dt,
                                                 CellState<NM, POR> &s)
{
    const double ey = PLN(c.f.e_pos, 1)[p];
    const double gy = 0.5 * PLN(c.f.v_bf, 1)[KIDX(i - 1, j - 1)] + 0.5 * PLN(c.f.v_bf, 1)[KIDX(i, j - 1)];
    double gyy = 0.;
    gyy += gy;
    if (ey <= c.f.y_profile[i] && s.ejt > 0.1) {
        if (c.rp.flow_resistance > 0.) {
            s.dvx += -c.rp.flow_resistance * dt * c.f.e_vel[p];
            s.dvy += -c.rp.flow_resistance * dt * PLN(c.f.e_vel, 1)[p];
        }
        if (c.rp.flow_friction > 0.) {
            #pragma unroll
            for (int q = 0; q < 4; ++q) s.st[q] = 0.;
            if (c.f.e_vel[p] >= 0.) s.dvx += -1.0 * c.rp.flow_friction * fabs(gyy) * dt;
            else s.dvx += 1.0 * c.rp.flow_friction * fabs(gyy) * dt;
        }
    }
}

// update_state (src/sale2d.c:1635-1742) from the register state
template <class R, int NM, bool POR>
__device__ __forceinline__ void state_cell(const CtxT<R> &c, long long p, const CellState<NM, POR> &s)
{
    constexpr int MM = CellState<NM, POR>::MM;
    using A = R;   // arithmetic of the table interpolation and the mixture rules: FP64, or FP32 in the mixed form
    const int nmat = NM > 0 ? NM : c.d.nmat;
    constexpr bool por = POR;
    const double dam = s.dam;
    A mpre[MM], mcsd[MM], mtem[MM];
    A epre = A(0.0), ecsd = A(0.0), etem = A(0.0), eden = A(0.0), emu = A(0.0);
    #pragma unroll
    for (int m = 1; m < nmat; ++m) {
        const double vm = s.vof[m];
        if (vm < SALEC_TOLVOF) {
            mpre[m] = A(0.); mcsd[m] = A(1.); mtem[m] = A(0.);
        } else {
            const DevMat &ms = c.mat[m];
            const double plim = (1.0 - dam) * ms.minPint + dam * ms.minPdam;
            const double pt = por ? s.pty[m] : 1.0;
            material_state<A>(ms, s.rho[m], s.eng[m], plim, pt, mtem[m], mpre[m], mcsd[m]);
        }
    }
    #pragma unroll
    for (int m = 1; m < nmat; ++m) {
        const A vm = A(s.vof[m]);
        const A rm = A(s.rho[m]);
        epre += vm * mpre[m];
        ecsd += vm / amax(A(1.0), mcsd[m]);
        etem += vm * mtem[m];
        eden += vm * rm;
        emu += vm / amax(A(1.0), rm * mcsd[m] * mcsd[m] * A(c.mat[m].GaCoef));
    }
    if (emu > A(0.)) emu = A(1.0) / emu;
    if (ecsd > A(0.)) ecsd = A(1.0) / ecsd;
    const double v0 = s.vof[0];
    if ((c.rp.partpres == 0 && v0 > SALEC_TOLVOF) || (c.rp.partpres == 1 && v0 > 1.0 - SALEC_TOLVOF)) {
        epre = A(0.);
        ecsd = A(1.0);
        emu = A(0.);
    } else if (c.rp.partpres == 1) {
        ecsd = ecsd * A(1.0 - v0);
        etem = etem / A(1.0 - v0);
        emu = emu * A(1.0 - v0);
    }
    c.f.e_pre[p] = epre;
    c.f.e_csd[p] = ecsd;
    c.f.e_tem[p] = etem;
    c.f.e_den[p] = eden;
    c.f.e_mu[p] = emu;
}

// One thread per cell: remap (interior), damping (every cell, while t < damp_time), ejecta
// drag and EOS (interior). The cell's state is stored once, after damping and drag.
template <class R, int NM, bool POR, bool P3>
__global__ void SALEC_BOUNDS_REMAP k_remap_damp_state(const CtxT<R> c, int do_remap, int do_damp, int do_ejecta, int do_state)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= c.d.enx || j >= c.d.eny) return;
    const long long p = KIDX(i, j);
    const bool interior = cell_interior(c, i, j);
    const double dt = c.scal->dt;
    const bool remap = do_remap && interior;
    const bool damp = do_damp && c.rp.damp_time > c.scal->time && c.rp.damp_type != 4 && c.rp.damp_type != 5;
    const bool ejecta = do_ejecta && interior;
    const bool state = do_state && interior;
    if (!(remap || damp || ejecta || state)) return;
    CellState<NM, POR> s;
    if (remap) remap_cell<R, NM, POR, P3>(c, i, j, p, s);
    else load_cell<R, NM, POR>(c, p, s);
    bool dirty = remap;
    if (damp) dirty |= damp_cell<R, NM, POR>(c, p, dt, s);
    if (ejecta) {
        ejecta_drag_cell<R, NM, POR>(c, i, j, p, dt, s);
        dirty = true;
    }
    if (dirty) store_cell<R, NM, POR>(c, p, s, !state);   // the EOS pass writes e_den itself
    if (state) state_cell<R, NM, POR>(c, p, s);
}

// ============================================================ phase 15: cycle control
// update_cycle_control (src/sale2d.c:71-136): advance time and step counter; seed the next
// CFL reduction with 1.1 * dt (src/sale2d.c:1961).
template <class R>
__global__ void k_cycle(const CtxT<R> c)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        Scal *s = c.scal;
        s->time += s->dt;
        s->i_step += 1;
        s->dt_acc = ord_encode(1.1 * s->dt);
        s->dt_nan_last = -1;
    }
}

// ============================================================ initialisation sweeps
// record_avg_value (src/sale2d.c:1562-1627): reference state of the damping layers and the
// latest arrival time of the impact wave at a damped cell (MAX over cells).
template <class R>
__global__ void k_record_reference_state(const CtxT<R> c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    unsigned long long cand = 0ULL;
    if (i < c.d.enx && j < c.d.eny) {
        const long long p = KIDX(i, j);
        PLN(c.f.e_dampref, 0)[p] = c.f.e_den[p];
        const double x = c.f.e_pos[p], y = PLN(c.f.e_pos, 1)[p];
        double len = 0.;
        len += x * x;
        len += y * y;
        len = sqrt(len);
        const double csd = c.f.e_csd[p];
        if ((c.f.e_sigma[p] > 0. || PLN(c.f.e_sigma, 1)[p] > 0.) && csd > 2.0) cand = ord_encode(len / csd);
        double s = 0.0;
        for (int m = 1; m < c.d.nmat; ++m) s += PLN(c.f.m_vof, m)[p] * PLN(c.f.m_eng, m)[p];
        PLN(c.f.e_dampref, 1)[p] = s;
        PLN(c.f.e_dampref, 2)[p] = c.f.e_pre[p];
    }
    for (int o = 16; o > 0; o >>= 1) cand = max(cand, __shfl_xor_sync(0xffffffffu, cand, o));
    if (((threadIdx.y * blockDim.x + threadIdx.x) & 31) == 0 && cand) atomicMax(&c.scal->aux, cand);
}

// init_v_field (src/sale2d.c:1897-1957): vertex velocity and mass from the cell velocities.
template <class R>
__global__ void k_init_vertex_velocity(const CtxT<R> c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    if (!vert_active(c, i, j)) return;
    const long long p = KIDX(i, j);
    const long long cl[4] = {KIDX(i - 1, j - 1), KIDX(i, j - 1), KIDX(i, j), KIDX(i - 1, j)};
    double vx = 0., vy = 0., em = 0., ev = 0.;
    for (int k = 0; k < 4; ++k) {
        const double lv = PLN(c.f.v_vol, k + 1)[p];
        const double w = c.f.e_den[cl[k]] * lv;
        vx += w * c.f.e_vel[cl[k]];
        vy += w * PLN(c.f.e_vel, 1)[cl[k]];
        em += c.f.e_den[cl[k]] * lv;
        ev += lv;
    }
    if (em > SALEC_TOLRHO * ev) {
        const double s = 1.0 / em;
        vx *= s; vy *= s;
        c.f.v_mass[p] = em;
        PLN(c.f.v_mass, 1)[p] = ev;
    } else {
        vx = vy = 0.;
        c.f.v_mass[p] = 0.;
        PLN(c.f.v_mass, 1)[p] = 0.;
    }
    c.f.v_vel[p] = vx;
    PLN(c.f.v_vel, 1)[p] = vy;
}

// Bit mask of the vertices with a non-zero nine-point Laplacian weight; one warp per 32
// consecutive vertices of a row (the grid spans the padded pitch, so warps are whole).
template <class R>
__global__ void k_laplace_mask(const CtxT<R> c, unsigned *mask)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    bool nz = false;
    if (i < c.d.vnx && j < c.d.vny) {
        const long long p = KIDX(i, j);
        for (int k = 0; k < 9; ++k) nz = nz || PLN(c.f.v_laplace, k)[p] != (R)0;
    }
    const unsigned word = __ballot_sync(0xffffffffu, nz);
    if ((threadIdx.x & 31) == 0 && j < c.d.vny) mask[(long long)j * (c.d.P >> 5) + (i >> 5)] = word;
}

// ============================================================ boundary gathers
// Apply a precomputed gather map (built on the host from the reference's ghost and
// restriction tables): dst[k] = op_c(src[k]) per component c. In-place when no source is also
// a destination; otherwise gathered through scratch in two passes.
__device__ __forceinline__ double apply_op(unsigned op, double v)
{
    switch (op) {
    case 0: return v;
    case 1: return -1.0 * v;
    case 2: return fabs(v);
    case 3: return -fabs(v);
    default: return 0.0;
    }
}

template <class T>
__device__ __forceinline__ void gather_one(const GatherField &gf, int mode, long long d, long long s, unsigned ops,
                                           double *scratch, long long row)
{
    T *base = static_cast<T *>(gf.base);
    for (int comp = 0; comp < gf.ncomp; ++comp) {
        T *plane = base + (long long)comp * gf.plane;
        const unsigned op = (ops >> (3 * comp)) & 7u;
        if (mode == 0) {
            plane[d] = (T)apply_op(op, (double)plane[s]);
        } else if (mode == 1) {
            scratch[row * gf.ncomp_max + comp] = apply_op(op, (double)plane[s]);
        } else {
            plane[d] = (T)scratch[row * gf.ncomp_max + comp];
        }
    }
}

// One component of a map whose sources include destinations: per plane, every source of the
// component is read before any destination is written, which is what the two passes through
// scratch do for the whole map (the component's points are touched by no other thread, and
// planes are disjoint).
template <class T>
__device__ __forceinline__ void gather_component(const GatherField &gf, int a, int b)
{
    T *base = static_cast<T *>(gf.base);
    // fixed-length predicated loops: every load of the component is issued before the first
    // one is needed
    int src[SALEC_GATHER_MAX_COMPONENT], dst[SALEC_GATHER_MAX_COMPONENT];
    unsigned ops[SALEC_GATHER_MAX_COMPONENT];
#pragma unroll
    for (int e = 0; e < SALEC_GATHER_MAX_COMPONENT; ++e)
        if (a + e < b) { src[e] = gf.src[a + e]; dst[e] = gf.dst[a + e]; ops[e] = gf.ops[a + e]; }
    for (int comp = 0; comp < gf.ncomp; ++comp) {
        T *plane = base + (long long)comp * gf.plane;
        double v[SALEC_GATHER_MAX_COMPONENT];
#pragma unroll
        for (int e = 0; e < SALEC_GATHER_MAX_COMPONENT; ++e)
            if (a + e < b) v[e] = apply_op((ops[e] >> (3 * comp)) & 7u, (double)plane[src[e]]);
#pragma unroll
        for (int e = 0; e < SALEC_GATHER_MAX_COMPONENT; ++e)
            if (a + e < b) plane[dst[e]] = (T)v[e];
    }
}

__global__ void k_gather(GatherBatch g, int mode, double *scratch)
{
    // mode 0: in place, one entry (or one component, where the field has them) per thread;
    // 1: gather into scratch; 2: scatter from scratch
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.total) return;
    int f = 0;
    while (f + 1 < g.nfield && t >= g.start[f + 1]) ++f;
    const GatherField &gf = g.field[f];
    const int k = t - g.start[f];
    if (mode == 0 && gf.cstart) {
        if (gf.f32) gather_component<float>(gf, gf.cstart[k], gf.cstart[k + 1]);
        else gather_component<double>(gf, gf.cstart[k], gf.cstart[k + 1]);
        return;
    }
    if (gf.f32) gather_one<float>(gf, mode, gf.dst[k], gf.src[k], gf.ops[k], scratch, t);
    else gather_one<double>(gf, mode, gf.dst[k], gf.src[k], gf.ops[k], scratch, t);
}

// ============================================================ layout conversion
// Reference AoS block of doubles (points x-fastest, components innermost) <-> planes of T.
template <class T>
__global__ void k_aos_to_planes(const double *aos, T *base, long long plane, int P, int nx, int ny, int nc)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)nx * ny;
    if (t >= n) return;
    const int i = (int)(t % nx), j = (int)(t / nx);
    for (int k = 0; k < nc; ++k) base[(long long)k * plane + i + (long long)P * j] = (T)aos[t * nc + k];
}

template <class T>
__global__ void k_planes_to_aos(const T *base, double *aos, long long plane, int P, int nx, int ny, int nc)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)nx * ny;
    if (t >= n) return;
    const int i = (int)(t % nx), j = (int)(t / nx);
    for (int k = 0; k < nc; ++k) aos[t * nc + k] = (double)base[(long long)k * plane + i + (long long)P * j];
}

template <class T>
__global__ void k_count_nonfinite(const T *base, long long n, unsigned long long *out)
{
    unsigned long long bad = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        if (!isfinite(base[t])) ++bad;
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(0xffffffffu, bad, o);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(out, bad);
}

void launch_aos_to_planes(const double *aos, void *base, bool f32, long long plane, int P, int nx, int ny, int nc,
                          cudaStream_t s)
{
    const int tb = 256;
    const int nb = (int)(((long long)nx * ny + tb - 1) / tb);
    if (f32) k_aos_to_planes<float><<<nb, tb, 0, s>>>(aos, static_cast<float *>(base), plane, P, nx, ny, nc);
    else k_aos_to_planes<double><<<nb, tb, 0, s>>>(aos, static_cast<double *>(base), plane, P, nx, ny, nc);
}

void launch_planes_to_aos(const void *base, bool f32, double *aos, long long plane, int P, int nx, int ny, int nc,
                          cudaStream_t s)
{
    const int tb = 256;
    const int nb = (int)(((long long)nx * ny + tb - 1) / tb);
    if (f32) k_planes_to_aos<float><<<nb, tb, 0, s>>>(static_cast<const float *>(base), aos, plane, P, nx, ny, nc);
    else k_planes_to_aos<double><<<nb, tb, 0, s>>>(static_cast<const double *>(base), aos, plane, P, nx, ny, nc);
}

void launch_count_nonfinite(const void *base, bool f32, long long n, unsigned long long *out, cudaStream_t s)
{
    if (f32) k_count_nonfinite<float><<<592, 256, 0, s>>>(static_cast<const float *>(base), n, out);
    else k_count_nonfinite<double><<<592, 256, 0, s>>>(static_cast<const double *>(base), n, out);
}

// ============================================================ launchers
// The material count and the porosity switch are template parameters of the flux, remap,
// energy and stress kernels, so that their per-material arrays unroll into registers for the
// common material counts; other counts use the generic instance.
#define SALEC_NM_DISPATCH(KERNEL, ...)                                                                         \
    do {                                                                                                       \
        const bool por_ = c.rp.porosity_model != 0;                                                            \
        switch (c.d.nmat) {                                                                                    \
        case 2: if (por_) KERNEL<R, 2, true><<<g, b, 0, s>>>(__VA_ARGS__); else KERNEL<R, 2, false><<<g, b, 0, s>>>(__VA_ARGS__); break; \
        case 3: if (por_) KERNEL<R, 3, true><<<g, b, 0, s>>>(__VA_ARGS__); else KERNEL<R, 3, false><<<g, b, 0, s>>>(__VA_ARGS__); break; \
        case 4: if (por_) KERNEL<R, 4, true><<<g, b, 0, s>>>(__VA_ARGS__); else KERNEL<R, 4, false><<<g, b, 0, s>>>(__VA_ARGS__); break; \
        case 5: if (por_) KERNEL<R, 5, true><<<g, b, 0, s>>>(__VA_ARGS__); else KERNEL<R, 5, false><<<g, b, 0, s>>>(__VA_ARGS__); break; \
        default: if (por_) KERNEL<R, 0, true><<<g, b, 0, s>>>(__VA_ARGS__); else KERNEL<R, 0, false><<<g, b, 0, s>>>(__VA_ARGS__); break; \
        }                                                                                                      \
    } while (0)

#define SALEC_NM_DISPATCH_P3(KERNEL, X, ...)                                                                   \
    do {                                                                                                       \
        const bool por_ = c.rp.porosity_model != 0;                                                            \
        switch (c.d.nmat) {                                                                                    \
        case 2: if (por_) KERNEL<R, 2, true, X><<<g, b, 0, s>>>(__VA_ARGS__); else KERNEL<R, 2, false, X><<<g, b, 0, s>>>(__VA_ARGS__); break; \
        case 3: if (por_) KERNEL<R, 3, true, X><<<g, b, 0, s>>>(__VA_ARGS__); else KERNEL<R, 3, false, X><<<g, b, 0, s>>>(__VA_ARGS__); break; \
        case 4: if (por_) KERNEL<R, 4, true, X><<<g, b, 0, s>>>(__VA_ARGS__); else KERNEL<R, 4, false, X><<<g, b, 0, s>>>(__VA_ARGS__); break; \
        case 5: if (por_) KERNEL<R, 5, true, X><<<g, b, 0, s>>>(__VA_ARGS__); else KERNEL<R, 5, false, X><<<g, b, 0, s>>>(__VA_ARGS__); break; \
        default: if (por_) KERNEL<R, 0, true, X><<<g, b, 0, s>>>(__VA_ARGS__); else KERNEL<R, 0, false, X><<<g, b, 0, s>>>(__VA_ARGS__); break; \
        }                                                                                                      \
    } while (0)

template <class R>
void launch_step_kernel(StepKernel k, const CtxT<R> &c, cudaStream_t s, dim3 b, int a0, int a1, int a2, int a3)
{
    const dim3 b8(32, 8);
    const dim3 g((c.d.enx + b.x - 1) / b.x, (c.d.eny + b.y - 1) / b.y);   // cells (and faces)
    const dim3 gv((c.d.vnx + b.x - 1) / b.x, (c.d.vny + b.y - 1) / b.y);  // vertices
    const int ncol = (c.d.enx + 255) / 256;
    switch (k) {
    case SK_PROFILE_RESET: k_profile_reset<R><<<ncol, 256, 0, s>>>(c); break;
    case SK_TRACE_PROFILE: k_trace_profile<R><<<dim3((c.d.enx + 31) / 32, (c.d.eny + 63) / 64), b8, 0, s>>>(c); break;
    case SK_PROFILE_DECODE: k_profile_decode<R><<<ncol, 256, 0, s>>>(c); break;
    case SK_VERTEX_VOF_MOMENTUM: k_vertex_vof_momentum<R><<<gv, b, 0, s>>>(c); break;
    case SK_CELL_VELOCITY: k_cell_velocity<R><<<g, b, 0, s>>>(c); break;
    case SK_VOID_VERTICES: k_void_vertices<R><<<gv, b, 0, s>>>(c); break;
    case SK_GRADIENT: k_gradient_viscosity_cfl<R><<<g, b, 0, s>>>(c); break;
    case SK_FINALIZE_DT: k_finalize_dt<R><<<148, SALEC_FINALIZE_THREADS, 0, s>>>(c); break;
    case SK_STRESS: SALEC_NM_DISPATCH(k_stress, c); break;
    case SK_STRESS_ENERGY: SALEC_NM_DISPATCH_P3(k_stress, true, c); break;
    case SK_ACCELERATION: k_vertex_acceleration<R><<<gv, b, 0, s>>>(c); break;
    case SK_DISPLACEMENT: k_vertex_displacement<R><<<gv, b, 0, s>>>(c); break;
    case SK_ENERGY: SALEC_NM_DISPATCH(k_energy, c); break;
    case SK_TRACERS:
        if (c.tr.n > 0) k_tracers<R><<<(c.tr.n + 127) / 128, 128, 0, s>>>(c);
        break;
    case SK_FLUX:
        if (a0 == 2) {   // pad ring, 1-D
            const long long ring = 4LL * c.d.enx + 4LL * (c.d.eny - 4);
            const dim3 g((unsigned)((ring + b.x * b.y - 1) / (b.x * b.y)));
            SALEC_NM_DISPATCH(k_flux, c, a0);
        } else {
            SALEC_NM_DISPATCH(k_flux, c, a0);
        }
        break;
    case SK_REMAP_DAMP_STATE:
        // the pml3 remap is its own instance so that its extra state costs the others no registers
        if (c.rp.damp_type == 2) SALEC_NM_DISPATCH_P3(k_remap_damp_state, true, c, a0, a1, a2, a3);
        else SALEC_NM_DISPATCH_P3(k_remap_damp_state, false, c, a0, a1, a2, a3);
        break;
    case SK_LAPLACE_MASK:
        k_laplace_mask<R><<<dim3(c.d.P / 32, (c.d.vny + 7) / 8), b8, 0, s>>>(c, const_cast<unsigned *>(c.lap_mask));
        break;
    case SK_STRENGTH_CONDITION:
        if (c.tr.n > 0) k_strength_condition<R><<<(c.tr.n + 127) / 128, 128, 0, s>>>(c);
        break;
    case SK_CYCLE: k_cycle<R><<<1, 32, 0, s>>>(c); break;
    case SK_RECORD_REFERENCE: k_record_reference_state<R><<<g, b, 0, s>>>(c); break;
    case SK_INIT_VERTEX_VELOCITY: k_init_vertex_velocity<R><<<gv, b, 0, s>>>(c); break;
    }
}

template void launch_step_kernel<double>(StepKernel, const CtxT<double> &, cudaStream_t, dim3, int, int, int, int);
template void launch_step_kernel<float>(StepKernel, const CtxT<float> &, cudaStream_t, dim3, int, int, int, int);

} // namespace salec
