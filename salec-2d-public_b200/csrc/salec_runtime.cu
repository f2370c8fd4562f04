// Host runtime of the B200 mesh update: device memory of one simulation, upload/download in
// the reference's layout, the launch sequence of one cycle, and the C ABI of salec_gpu.h.
#include "../../include/salec_gpu.h"
#include "salec_device.cuh"
#include "salec_kernels.h"
#include "salec_adjoint.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cctype>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

using namespace salec;

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

static int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

#define CUDA_TRY(expr)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(SALEC_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------ field table
namespace {

enum Loc { L_CELL, L_VERT, L_BX, L_BY, L_COL };
enum NC { NC_FIX, NC_MAT, NC_PHI };

struct FieldInfo {
    const char *name;
    Loc loc;
    NC nck;
    int n;
    size_t off;   // offset of the pointer inside salec::Fields
};

#define F_(name, loc, nck, n) {#name, loc, nck, n, offsetof(Fields, name)}
const FieldInfo kFields[] = {
    F_(v_vel, L_VERT, NC_FIX, 2), F_(v_bf, L_VERT, NC_FIX, 2), F_(v_acc, L_VERT, NC_FIX, 2),
    F_(v_dis, L_VERT, NC_FIX, 2), F_(v_pos, L_VERT, NC_FIX, 2), F_(v_vof, L_VERT, NC_MAT, 1),
    F_(v_mass, L_VERT, NC_FIX, 2), F_(v_vol, L_VERT, NC_FIX, 5), F_(v_subvol, L_VERT, NC_FIX, 4),
    F_(v_laplace, L_VERT, NC_FIX, 9), F_(v_suf, L_VERT, NC_FIX, 8), F_(v_alpha, L_VERT, NC_FIX, 2),
    F_(v_beta, L_VERT, NC_FIX, 2),
    F_(e_vel, L_CELL, NC_FIX, 2), F_(e_div_vel, L_CELL, NC_FIX, 1), F_(e_grad_vel, L_CELL, NC_FIX, 5),
    F_(e_ste, L_CELL, NC_FIX, 4), F_(e_mu, L_CELL, NC_FIX, 1), F_(e_dvel, L_CELL, NC_FIX, 2),
    F_(e_pre, L_CELL, NC_FIX, 1), F_(e_tem, L_CELL, NC_FIX, 1), F_(e_den, L_CELL, NC_FIX, 1),
    F_(e_eng, L_CELL, NC_FIX, 1), F_(e_csd, L_CELL, NC_FIX, 1), F_(e_dam, L_CELL, NC_FIX, 1),
    F_(e_cvs, L_CELL, NC_FIX, 1), F_(m_vof, L_CELL, NC_MAT, 1), F_(m_den, L_CELL, NC_MAT, 1),
    F_(m_eng, L_CELL, NC_MAT, 1), F_(m_pty, L_CELL, NC_MAT, 1), F_(e_wpt, L_CELL, NC_FIX, 4),
    F_(e_pos, L_CELL, NC_FIX, 4), F_(e_vol, L_CELL, NC_FIX, 1), F_(e_suf, L_CELL, NC_FIX, 8),
    F_(e_grad, L_CELL, NC_FIX, 12), F_(e_subvol, L_CELL, NC_FIX, 8), F_(e_q, L_CELL, NC_FIX, 1),
    F_(e_strength, L_CELL, NC_FIX, 1), F_(e_cnd, L_CELL, NC_FIX, 1), F_(e_tps, L_CELL, NC_FIX, 1),
    F_(e_ste2s, L_CELL, NC_FIX, 1), F_(e_sta2s, L_CELL, NC_FIX, 1), F_(e_alpha, L_CELL, NC_FIX, 2),
    F_(e_beta, L_CELL, NC_FIX, 4), F_(e_sigma, L_CELL, NC_FIX, 2), F_(e_dampref, L_CELL, NC_FIX, 3),
    F_(e_vib, L_CELL, NC_FIX, 1), F_(e_ejt, L_CELL, NC_FIX, 1),
    F_(bx_phi, L_BX, NC_PHI, 1), F_(by_phi, L_BY, NC_PHI, 1), F_(bx_normal, L_BX, NC_FIX, 2),
    F_(by_normal, L_BY, NC_FIX, 2), F_(y_profile, L_COL, NC_FIX, 1),
};
#undef F_
constexpr int kNumFields = sizeof(kFields) / sizeof(kFields[0]);

// Fields kept FP64 in the mixed form (FieldsT in salec_device.cuh).
bool field_exact(int k)
{
    static const char *exact[] = {"v_pos", "m_vof", "m_den", "m_eng", "m_pty", "e_cvs", "e_pos", "e_vol",
                                  "bx_phi", "by_phi", "y_profile"};
    for (const char *e : exact)
        if (strcmp(kFields[k].name, e) == 0) return true;
    return false;
}

int field_by_name(const char *n)
{
    if (!n) return -1;
    for (int k = 0; k < kNumFields; ++k)
        if (strcmp(kFields[k].name, n) == 0) return k;
    // the reference's e_vof is the same array as m_vof (src/sale2d.c:333)
    if (strcmp(n, "e_vof") == 0) return field_by_name("m_vof");
    return -1;
}

const char *kFuncNames[] = {"SimpleRock", "SimpleShear", "JohnsonCook1", "JohnsonCook2", "RockStrengthT",
                            "IceStrength", "Collins", "Ivanov", "SimpleTensile", "None", "Wunnemann",
                            "VonMises1", "VonMises2"};

struct Gather {
    GatherBatch batch{};
    bool two_pass = false;
    int ncomp_max = 0;
    int entries[SALEC_MAX_GATHER_FIELDS] = {0};   // map entries per field (the adjoint walks entries)
};

} // namespace

void salec_internal_output_release(void *&writer);   // salec_output.cu

struct salec_gpu {
    Dims d{};
    RunParams rp{};
    int go[4] = {0, 0, 0, 0};
    cudaStream_t stream = nullptr;
    char *pool = nullptr;
    size_t pool_bytes = 0;
    int mixed = 0;              // 1: relaxed fields stored as float (mixed form)
    Fields f{};
    DevMat *mat = nullptr;
    std::vector<void *> owned;   // device allocations besides the pool
    // small device arrays of create (gather maps, EOS tables and their axis buckets): collected
    // on the host by upload_vec and sent in one allocation and one copy by flush_uploads, so
    // that creating a handle makes a few driver calls instead of one pair per array
    std::vector<char> up_host;
    std::vector<std::function<void(const char *)>> up_fix;
    Scal *scal = nullptr;
    Scal *scal_host = nullptr;   // pinned mirror
    double *scratch = nullptr;   // gather scratch
    size_t scratch_doubles = 0;
    double *staging = nullptr;   // AoS staging for field transfer
    size_t staging_doubles = 0;
    Gather g_mvof, g_dvel_den, g_evel, g_pre_ste_q, g_flux_state, r_vel, r_acc, r_dis, g_init;
    Tracers tr{};
    void *tr_block = nullptr;   // one allocation holding every tracer array
    size_t tr_bytes = 0;
    unsigned *lap_mask = nullptr;   // vertices with a non-zero Laplacian weight (1 bit each)
    // geometry fields read through tables of their distinct rows: v_vol, v_subvol, v_suf,
    // e_grad, e_vol (tab and row are owned when compact)
    struct GeoSlot {
        void *tab = nullptr;
        int *row = nullptr;
        long long plane = 0;
        bool compact = false;
    } geo[5];
    int *row_identity = nullptr;
    salec_run_desc run{};       // the description the handle was created from
    // optional per-phase timing with CUDA events on the handle's stream
    int profiling = 0;
    std::vector<cudaEvent_t> ev_a, ev_b;
    std::vector<int> ev_phase;
    size_t ev_used = 0;
    long long launches = 0;     // kernels launched by this handle
    dim3 blk[SK_COUNT];         // block shape of each 2-D sweep (salec_gpu_autotune picks them)
    // one full cycle captured as a CUDA graph (kernel arguments hold the run parameters and the
    // tracer arrays, so changing either drops the graph)
    cudaGraphExec_t cycle_graph = nullptr;
    long long cycle_graph_launches = 0;
    // in the captured cycle the tracer sweep runs on a side stream beside the flux sweep (it
    // reads nothing the flux writes and writes only tracer arrays); joined before phase 13
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // pipelined read-back (salec_gpu_step_report_async): per slot a pinned copy of the scalars,
    // its completion event and whether it is in flight
    Scal *report_scal[2] = {nullptr, nullptr};
    cudaEvent_t report_ev[2] = {nullptr, nullptr};
    bool report_pending[2] = {false, false};
    bool fork_tracers = false;
    void *output = nullptr;     // output writer state (salec_output.cu)
    void *conserve = nullptr;   // scratch of the conservation sums (salec_conserve.cu)
    // prescribed time steps (salec_gpu_set_dt_schedule)
    double *dt_sched = nullptr;
    long long dt_sched_i0 = 0;
    int dt_sched_n = 0;
    struct AdjointState *adj = nullptr;   // adjoint buffers (salec_gpu_adjoint_*)

    template <class R>
    CtxT<R> ctx_t() const
    {
        CtxT<R> c;
        c.d = d;
        memcpy(&c.f, &f, sizeof(c.f));   // same pointers; relaxed ones address floats in the mixed form
        c.rp = rp;
        c.mat = mat;
        c.scal = scal;
        c.tr = tr;
        c.lap_mask = lap_mask;
        c.g_v_vol = {static_cast<const R *>(geo[0].tab), geo[0].row, geo[0].plane};
        c.g_v_subvol = {static_cast<const R *>(geo[1].tab), geo[1].row, geo[1].plane};
        c.g_v_suf = {static_cast<const R *>(geo[2].tab), geo[2].row, geo[2].plane};
        c.g_e_grad = {static_cast<const R *>(geo[3].tab), geo[3].row, geo[3].plane};
        c.g_e_vol = {static_cast<const double *>(geo[4].tab), geo[4].row, geo[4].plane};
        c.dt_sched = dt_sched;
        c.dt_sched_i0 = dt_sched_i0;
        c.dt_sched_n = dt_sched_n;
        return c;
    }
    Ctx ctx() const { return ctx_t<double>(); }
};

namespace {

int field_ncomp(const salec_gpu *h, int k)
{
    const FieldInfo &fi = kFields[k];
    if (fi.nck == NC_MAT) return h->d.nmat * fi.n;
    if (fi.nck == NC_PHI) return h->d.phi;
    return fi.n;
}

void field_points(const salec_gpu *h, int k, int &nx, int &ny)
{
    switch (kFields[k].loc) {
    case L_CELL: nx = h->d.enx; ny = h->d.eny; break;
    case L_VERT: nx = h->d.vnx; ny = h->d.vny; break;
    case L_BX: nx = h->d.vnx; ny = h->d.eny; break;
    case L_BY: nx = h->d.enx; ny = h->d.vny; break;
    default: nx = h->d.enx; ny = 1; break;
    }
}

bool field_f32(const salec_gpu *h, int k) { return h->mixed && !field_exact(k); }
size_t field_elem(const salec_gpu *h, int k) { return field_f32(h, k) ? sizeof(float) : sizeof(double); }

double *&field_ptr(salec_gpu *h, int k)
{
    return *reinterpret_cast<double **>(reinterpret_cast<char *>(&h->f) + kFields[k].off);
}

// Queue a host array for the device: *out receives its device address at the next
// flush_uploads (null until then, and for an empty array).
template <typename T>
int upload_vec(salec_gpu *h, const std::vector<T> &v, const T **out)
{
    *out = nullptr;
    if (v.empty()) return SALEC_OK;
    const size_t off = (h->up_host.size() + 255) & ~(size_t)255;
    h->up_host.resize(off + v.size() * sizeof(T));
    memcpy(h->up_host.data() + off, v.data(), v.size() * sizeof(T));
    h->up_fix.push_back([out, off](const char *base) { *out = reinterpret_cast<const T *>(base + off); });
    return SALEC_OK;
}

// One device allocation for every queued array, one copy, then the addresses.
int flush_uploads(salec_gpu *h)
{
    if (h->up_fix.empty()) return SALEC_OK;
    void *p = nullptr;
    CUDA_TRY(cudaMalloc(&p, h->up_host.size()));
    h->owned.push_back(p);
    CUDA_TRY(cudaMemcpyAsync(p, h->up_host.data(), h->up_host.size(), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (auto &fix : h->up_fix) fix(static_cast<const char *>(p));
    std::vector<char>().swap(h->up_host);
    h->up_fix.clear();
    return SALEC_OK;
}

int upload_axis(salec_gpu *h, const double *xs, int n, const int **bkt, int *nb, double *b0, double *binv)
{
    std::vector<int> v;
    *bkt = nullptr;
    *nb = 0;
    if (!build_axis_buckets(xs, n, v, *b0, *binv)) return SALEC_OK;
    *nb = (int)v.size();
    return upload_vec(h, v, bkt);
}

int make_gather(salec_gpu *h, Gather &g, const std::vector<std::pair<int, GatherMap>> &maps)
{
    g = Gather();
    g.batch.nfield = (int)maps.size();
    int total = 0;
    for (size_t k = 0; k < maps.size(); ++k) g.ncomp_max = std::max(g.ncomp_max, field_ncomp(h, maps[k].first));
    // maps whose sources include destinations run as components in the same single launch;
    // only when a component is too large does the batch fall back to two passes through scratch
    std::vector<GatherMap> grouped(maps.size());
    std::vector<std::vector<int>> cstart(maps.size());
    for (size_t k = 0; k < maps.size() && !g.two_pass; ++k)
        if (maps[k].second.needs_scratch && !group_gather_components(maps[k].second, grouped[k], cstart[k]))
            g.two_pass = true;
    for (size_t k = 0; k < maps.size(); ++k) {
        const int fid = maps[k].first;
        const bool comp = !g.two_pass && maps[k].second.needs_scratch;
        const GatherMap &m = comp ? grouped[k] : maps[k].second;
        GatherField &gf = g.batch.field[k];
        gf.base = field_ptr(h, fid);
        gf.f32 = field_f32(h, fid) ? 1 : 0;
        gf.plane = h->d.PL;
        gf.ncomp = field_ncomp(h, fid);
        gf.ncomp_max = g.ncomp_max;
        gf.cstart = nullptr;
        int rc = upload_vec(h, m.dst, &gf.dst);
        if (rc) return rc;
        rc = upload_vec(h, m.src, &gf.src);
        if (rc) return rc;
        rc = upload_vec(h, m.ops, &gf.ops);
        if (rc) return rc;
        if (comp && (rc = upload_vec(h, cstart[k], &gf.cstart))) return rc;
        g.batch.start[k] = total;
        g.entries[k] = (int)m.dst.size();
        total += comp ? (int)cstart[k].size() - 1 : (int)m.dst.size();
    }
    g.batch.start[maps.size()] = total;
    g.batch.total = total;
    if (g.two_pass) h->scratch_doubles = std::max(h->scratch_doubles, (size_t)total * g.ncomp_max);
    return SALEC_OK;
}

int run_gather(salec_gpu *h, const Gather &g)
{
    if (g.batch.total == 0) return SALEC_OK;
    const int tb = 256, nb = (g.batch.total + tb - 1) / tb;
    h->launches += g.two_pass ? 2 : 1;
    if (!g.two_pass) {
        k_gather<<<nb, tb, 0, h->stream>>>(g.batch, 0, nullptr);
    } else {
        k_gather<<<nb, tb, 0, h->stream>>>(g.batch, 1, h->scratch);
        k_gather<<<nb, tb, 0, h->stream>>>(g.batch, 2, h->scratch);
    }
    CUDA_TRY(cudaGetLastError());
    return SALEC_OK;
}

// fused: the cycle graph's form, in which the stress sweep of phase 7 also does the energy
// update and phase 10 launches nothing; phase-by-phase callers and the adjoint use the
// separate sweeps, which compute the same bits
template <class R>
int run_phase_t(salec_gpu *h, int ph, bool fused)
{
    const CtxT<R> c = h->ctx_t<R>();
    cudaStream_t s = h->stream;
    int rc = SALEC_OK;
    static const int kLaunches[16] = {3, 1, 0, 1, 1, 1, 1, 1, 1, 1, 1, 0, 1, 0, 1, 1};
    h->launches += kLaunches[ph] + (ph == 11 && h->tr.n > 0 ? 1 : 0) - (fused && ph == 10 ? 1 : 0);
    switch (ph) {
    case 0:
        launch_step_kernel(SK_PROFILE_RESET, c, s, h->blk[SK_PROFILE_RESET]);
        launch_step_kernel(SK_TRACE_PROFILE, c, s, h->blk[SK_TRACE_PROFILE]);
        launch_step_kernel(SK_PROFILE_DECODE, c, s, h->blk[SK_PROFILE_DECODE]);
        break;
    case 1:   // vertex volume fractions and vertex momentum in one sweep (phase 2 is empty)
        rc = run_gather(h, h->g_mvof);
        if (!rc) rc = run_gather(h, h->g_dvel_den);
        launch_step_kernel(SK_VERTEX_VOF_MOMENTUM, c, s, h->blk[SK_VERTEX_VOF_MOMENTUM]);
        if (!rc) rc = run_gather(h, h->r_vel);
        break;
    case 2: break;
    case 3:
        launch_step_kernel(SK_CELL_VELOCITY, c, s, h->blk[SK_CELL_VELOCITY]);
        rc = run_gather(h, h->g_evel);
        break;
    case 4: launch_step_kernel(SK_VOID_VERTICES, c, s, h->blk[SK_VOID_VERTICES]); break;
    case 5: launch_step_kernel(SK_GRADIENT, c, s, h->blk[SK_GRADIENT]); break;
    case 6: launch_step_kernel(SK_FINALIZE_DT, c, s, h->blk[SK_FINALIZE_DT]); break;
    case 7: launch_step_kernel(fused ? SK_STRESS_ENERGY : SK_STRESS, c, s, h->blk[SK_STRESS]); break;
    case 8:
        rc = run_gather(h, h->g_pre_ste_q);
        launch_step_kernel(SK_ACCELERATION, c, s, h->blk[SK_ACCELERATION]);
        if (!rc) rc = run_gather(h, h->r_acc);
        break;
    case 9:
        launch_step_kernel(SK_DISPLACEMENT, c, s, h->blk[SK_DISPLACEMENT]);
        rc = run_gather(h, h->r_dis);
        break;
    case 10:
        if (!fused) launch_step_kernel(SK_ENERGY, c, s, h->blk[SK_ENERGY]);
        break;
    case 11:
        if (h->fork_tracers && h->tr.n > 0) {
            CUDA_TRY(cudaEventRecord(h->ev_fork, s));
            CUDA_TRY(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
            launch_step_kernel(SK_TRACERS, c, h->side, h->blk[SK_TRACERS]);
            CUDA_TRY(cudaEventRecord(h->ev_join, h->side));
        } else {
            launch_step_kernel(SK_TRACERS, c, s, h->blk[SK_TRACERS]);
        }
        break;
    case 12:   // ghost fills of the donor state, then the fluxes of every cell in one launch
        rc = run_gather(h, h->g_flux_state);
        launch_step_kernel(SK_FLUX, c, s, h->blk[SK_FLUX], 3);
        break;
    case 13:   // strength condition: count the lubricating tracers of every cell in e_cnd
        if (h->fork_tracers && h->tr.n > 0) CUDA_TRY(cudaStreamWaitEvent(s, h->ev_join, 0));
        if (h->rp.tracer_lubrication > 0) {
            const int fid = field_by_name("e_cnd");
            CUDA_TRY(cudaMemsetAsync(field_ptr(h, fid), 0, (size_t)h->d.PL * field_elem(h, fid), s));
            launch_step_kernel(SK_STRENGTH_CONDITION, c, s, h->blk[SK_STRENGTH_CONDITION]);
            if (h->tr.n > 0) h->launches += 1;
        }
        break;
    case 14: {
        const int ejecta = (h->rp.flow_resistance > 0. || h->rp.flow_friction > 0.) ? 1 : 0;
        launch_step_kernel(SK_REMAP_DAMP_STATE, c, s, h->blk[SK_REMAP_DAMP_STATE], 1, 1, ejecta, 1);
        break;
    }
    case 15: launch_step_kernel(SK_CYCLE, c, s, h->blk[SK_CYCLE]); break;
    default: return fail(SALEC_ERR_ARG, "phase out of range");
    }
    if (rc) return rc;
    CUDA_TRY(cudaGetLastError());
    return SALEC_OK;
}

int run_phase(salec_gpu *h, int ph, bool fused = false)
{
    return h->mixed ? run_phase_t<float>(h, ph, fused) : run_phase_t<double>(h, ph, fused);
}

int build_gathers(salec_gpu *h)
{
    const Dims &d = h->d;
    auto gm = [&](const char *name, GhostPattern pat) {
        int fid = field_by_name(name);
        return std::make_pair(fid, build_ghost_map(d.enx, d.eny, d.P, field_ncomp(h, fid), h->go, pat));
    };
    auto rm = [&](const char *name) {
        int fid = field_by_name(name);
        return std::make_pair(fid, build_restrict_map(d.vnx, d.vny, d.P, field_ncomp(h, fid), h->go));
    };
    int rc;
    if ((rc = make_gather(h, h->g_mvof, {gm("m_vof", GP_ALWAYS_COPY)}))) return rc;
    if ((rc = make_gather(h, h->g_dvel_den, {gm("e_dvel", GP_VELOCITY_INC), gm("e_den", GP_DENSITY)}))) return rc;
    if ((rc = make_gather(h, h->g_evel, {gm("e_vel", GP_VELOCITY)}))) return rc;
    if ((rc = make_gather(h, h->g_pre_ste_q,
                          {gm("e_pre", GP_ALWAYS_COPY), gm("e_ste", GP_STRESS), gm("e_q", GP_ALWAYS_COPY)})))
        return rc;
    std::vector<std::pair<int, GatherMap>> fs = {gm("m_den", GP_DENSITY), gm("e_vib", GP_ALWAYS_COPY),
                                                 gm("m_eng", GP_DENSITY)};
    if (h->rp.porosity_model) {
        fs.push_back(gm("m_pty", GP_ALWAYS_COPY));
        fs.push_back(gm("e_cvs", GP_ALWAYS_COPY));
    }
    if ((rc = make_gather(h, h->g_flux_state, fs))) return rc;
    if ((rc = make_gather(h, h->g_init,
                          {gm("e_den", GP_DENSITY), gm("e_pre", GP_ALWAYS_COPY), gm("e_ste", GP_STRESS),
                           gm("m_eng", GP_DENSITY), gm("m_pty", GP_ALWAYS_COPY), gm("e_cvs", GP_ALWAYS_COPY)})))
        return rc;
    if ((rc = make_gather(h, h->r_vel, {rm("v_vel")}))) return rc;
    if ((rc = make_gather(h, h->r_acc, {rm("v_acc")}))) return rc;
    if ((rc = make_gather(h, h->r_dis, {rm("v_dis")}))) return rc;
    if (h->scratch_doubles) {
        void *p = nullptr;
        CUDA_TRY(cudaMalloc(&p, h->scratch_doubles * sizeof(double)));
        h->owned.push_back(p);
        h->scratch = static_cast<double *>(p);
    }
    return SALEC_OK;
}

int upload_material(salec_gpu *h, const salec_material_desc &m, DevMat &dm)
{
    memset(&dm, 0, sizeof(dm));
    dm.eos_type = m.eos_type;
    dm.yfunc = m.yfunc; dm.tfunc = m.tfunc; dm.dsdf = m.dsdf; dm.porfunc = m.porfunc;
    dm.PolyLiq = m.PolyLiq; dm.PolySol = m.PolySol;
#define CP(x) dm.x = m.x
    CP(VaporDen); CP(MeltDen); CP(GaCoef); CP(Yint0); CP(Yfricint); CP(Ylimint); CP(Ydam0); CP(Yfricdam);
    CP(Ylimdam); CP(Yten0); CP(IvanA); CP(IvanB); CP(IvanC); CP(Pbd); CP(Pbp); CP(minPint); CP(minPdam);
    CP(JCA); CP(JCB); CP(JCN); CP(JCC); CP(JCM); CP(JCTREF); CP(JCMaxPlastic); CP(Asimon); CP(Csimon);
    CP(Tmelt0); CP(Tfrac); CP(Tdelta); CP(Tlidc1); CP(Tlidc2); CP(Tlidc3); CP(Tsolc1); CP(Tsolc2);
    CP(Tsolc3); CP(Toff); CP(Cvib); CP(VibMax); CP(Tdamp); CP(Pvlim); CP(Acvis); CP(alpha0); CP(alphax);
    CP(epse0); CP(chi); CP(kappa); CP(avel); CP(epsec); CP(epsex); CP(alphamax); CP(alphamax2); CP(alphae);
    CP(gamfrac); CP(melt_viscosity);
#undef CP
    for (int k = 0; k < 13; ++k) dm.tl[k] = m.till[k];
    int rc;
    if (m.eos_type == SALEC_EOS_TILLOTSON) {
        if (m.cold_n < 2 || !m.cold_yeng) return fail(SALEC_ERR_ARG, "Tillotson material without cold-energy curve");
        dm.cold_n = m.cold_n;
        std::vector<double> y(m.cold_yeng, m.cold_yeng + m.cold_n);
        if ((rc = upload_vec(h, y, &dm.cold_yeng))) return rc;
    } else if (m.eos_type == SALEC_EOS_ANEOS || m.eos_type == SALEC_EOS_ANEOS_SIEDEN) {
        if (m.ntem < 2 || m.nden < 2 || !m.xtem || !m.yden || !m.data) return fail(SALEC_ERR_ARG, "table EOS without table");
        dm.ntem = m.ntem;
        dm.nden = m.nden;
        std::vector<double> x(m.xtem, m.xtem + m.ntem), y(m.yden, m.yden + m.nden);
        std::vector<double> t(m.data, m.data + (size_t)m.ntem * m.nden * 3);
        if ((rc = upload_vec(h, x, &dm.xtem))) return rc;
        if ((rc = upload_vec(h, y, &dm.yden))) return rc;
        if ((rc = upload_vec(h, t, &dm.data))) return rc;
        if (h->mixed) {   // the mixed form interpolates the table in FP32
            std::vector<float> tf(t.begin(), t.end());
            if ((rc = upload_vec(h, tf, &dm.data_f))) return rc;
        }
        if ((rc = upload_axis(h, x.data(), m.ntem, &dm.xtem_bkt, &dm.xtem_nb, &dm.xtem_b0, &dm.xtem_binv))) return rc;
        if ((rc = upload_axis(h, y.data(), m.nden, &dm.yden_bkt, &dm.yden_nb, &dm.yden_b0, &dm.yden_binv))) return rc;
    } else {
        return fail(SALEC_ERR_ARG, "unknown EOS type");
    }
    return SALEC_OK;
}

const char *const kGeoFields[5] = {"v_vol", "v_subvol", "v_suf", "e_grad", "e_vol"};
constexpr int kGeoMaxRows = 512;   // more distinct rows than this: read the field's own planes

// Row hashing for the geometry tables. Each row of an AoS field (row_doubles words) is
// reduced to two 64-bit sums of a position-keyed splitmix64 finaliser of its words; the sums
// commute, so a block reduces a row in any order and the result is deterministic. Rows that
// hash alike are then compared word for word, so a collision costs a fallback, never a wrong
// table.
__device__ __forceinline__ unsigned long long geo_mix(unsigned long long z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__global__ void __launch_bounds__(256) k_geo_row_hash(const unsigned long long *__restrict__ src, long long row_words,
                                                      unsigned long long *__restrict__ out)
{
    const unsigned long long *r = src + (long long)blockIdx.x * row_words;
    unsigned long long a = 0, b = 0;
    for (long long k = threadIdx.x; k < row_words; k += blockDim.x) {
        const unsigned long long w = r[k];
        a += geo_mix(w + 0x9E3779B97F4A7C15ULL * (unsigned long long)(k + 1));
        b += geo_mix((w ^ 0xD6E8FEB86659FD93ULL) + 0xC2B2AE3D27D4EB4FULL * (unsigned long long)(k + 7));
    }
    for (int o = 16; o; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    __shared__ unsigned long long sa[8], sb[8];
    if ((threadIdx.x & 31) == 0) { sa[threadIdx.x >> 5] = a; sb[threadIdx.x >> 5] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { a += sa[w]; b += sb[w]; }
        out[2 * blockIdx.x] = a;
        out[2 * blockIdx.x + 1] = b;
    }
}

// Row j against its representative row rep[j]: any differing word sets *diff.
__global__ void __launch_bounds__(256) k_geo_row_verify(const unsigned long long *__restrict__ src, long long row_words,
                                                        const int *__restrict__ rep, unsigned *__restrict__ diff)
{
    const int j = blockIdx.x, q = rep[j];
    if (q == j) return;
    const unsigned long long *r = src + (long long)j * row_words, *t = src + (long long)q * row_words;
    bool bad = false;
    for (long long k = threadIdx.x; k < row_words; k += blockDim.x) bad |= r[k] != t[k];
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(diff, 1u);
}

// Distinct rows uniq[u] of src gathered into consecutive rows of dst.
__global__ void __launch_bounds__(256) k_geo_row_gather(const unsigned long long *__restrict__ src, long long row_words,
                                                        const int *__restrict__ uniq, unsigned long long *__restrict__ dst)
{
    const unsigned long long *r = src + (long long)uniq[blockIdx.x] * row_words;
    unsigned long long *d = dst + (long long)blockIdx.x * row_words;
    for (long long k = threadIdx.x; k < row_words; k += blockDim.x) d[k] = r[k];
}

// Table of the distinct rows of an uploaded geometry field, built from the AoS copy of the
// field in the staging buffer (nx x ny points of nc components); mesh rows that repeat bit for
// bit share one table row. The staging buffer is read in stream order after the upload.
int build_geo_table(salec_gpu *h, int slot, int fid, int nx, int ny, int nc)
{
    auto &g = h->geo[slot];
    const long long row_words = (long long)nx * nc;
    if (g.compact) { cudaFree(g.tab); cudaFree(g.row); }
    g = salec_gpu::GeoSlot();
    if (h->cycle_graph) { cudaGraphExecDestroy(h->cycle_graph); h->cycle_graph = nullptr; }
    const auto *src = reinterpret_cast<const unsigned long long *>(h->staging);

    // temporaries are stream-ordered (cudaMallocAsync / cudaFreeAsync): freeing them does not
    // synchronise the device, which would stall every other handle's work
    unsigned long long *d_hash = nullptr;
    CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&d_hash), sizeof(unsigned long long) * 2 * ny, h->stream));
    k_geo_row_hash<<<ny, 256, 0, h->stream>>>(src, row_words, d_hash);
    cudaError_t e = cudaGetLastError();
    std::vector<unsigned long long> hashes(2 * (size_t)ny);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hashes.data(), d_hash, sizeof(unsigned long long) * 2 * ny, cudaMemcpyDeviceToHost,
                            h->stream);
    cudaFreeAsync(d_hash, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    CUDA_TRY(e);

    // rows grouped in order of first appearance by their 128-bit hash
    struct Key {
        unsigned long long a, b;
        bool operator==(const Key &o) const { return a == o.a && b == o.b; }
    };
    struct KeyHash {
        size_t operator()(const Key &k) const { return (size_t)(k.a ^ (k.b * 0x9E3779B97F4A7C15ULL)); }
    };
    std::unordered_map<Key, int, KeyHash> first;
    std::vector<int> rowmap(h->d.R, 0), rep(ny), uniq;
    for (int j = 0; j < ny; ++j) {
        const Key k{hashes[2 * (size_t)j], hashes[2 * (size_t)j + 1]};
        auto it = first.find(k);
        int u;
        if (it == first.end()) {
            u = (int)uniq.size();
            uniq.push_back(j);
            first.emplace(k, u);
        } else {
            u = it->second;
        }
        rowmap[j] = u;
        rep[j] = uniq[u];
    }
    const int U = (int)uniq.size();
    auto full_planes = [&]() {
        g = salec_gpu::GeoSlot();
        g.tab = field_ptr(h, fid);
        g.row = h->row_identity;
        g.plane = h->d.PL;
    };
    if (U > kGeoMaxRows || U >= ny) {
        full_planes();
        return SALEC_OK;
    }

    const bool f32 = field_f32(h, fid);
    const long long plane = (((long long)U * h->d.P + 31) / 32) * 32;
    int *d_idx = nullptr;                   // rep[ny] then uniq[U]
    unsigned *d_diff = nullptr;
    unsigned long long *d_rows = nullptr;   // the U distinct rows, AoS
    auto release_tmp = [&]() {
        if (d_idx) cudaFreeAsync(d_idx, h->stream);
        if (d_diff) cudaFreeAsync(d_diff, h->stream);
        if (d_rows) cudaFreeAsync(d_rows, h->stream);
    };
    e = cudaMallocAsync(reinterpret_cast<void **>(&d_idx), sizeof(int) * ((size_t)ny + U), h->stream);
    if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void **>(&d_diff), sizeof(unsigned), h->stream);
    if (e == cudaSuccess)
        e = cudaMallocAsync(reinterpret_cast<void **>(&d_rows), sizeof(unsigned long long) * (size_t)U * row_words,
                            h->stream);
    if (e == cudaSuccess) e = cudaMalloc(&g.tab, (size_t)nc * plane * field_elem(h, fid));
    if (e == cudaSuccess) e = cudaMalloc(&g.row, sizeof(int) * h->d.R);
    g.compact = true;
    g.plane = plane;
    unsigned diff = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_idx, rep.data(), sizeof(int) * ny, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_idx + ny, uniq.data(), sizeof(int) * U, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_diff, 0, sizeof(unsigned), h->stream);
    if (e == cudaSuccess) {
        k_geo_row_verify<<<ny, 256, 0, h->stream>>>(src, row_words, d_idx, d_diff);
        k_geo_row_gather<<<U, 256, 0, h->stream>>>(src, row_words, d_idx + ny, d_rows);
        launch_aos_to_planes(reinterpret_cast<const double *>(d_rows), g.tab, f32, plane, h->d.P, nx, U, nc,
                             h->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g.row, rowmap.data(), sizeof(int) * h->d.R, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&diff, d_diff, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    release_tmp();
    if (e != cudaSuccess || diff) {
        cudaFree(g.tab);
        cudaFree(g.row);
        full_planes();
    }
    CUDA_TRY(e);
    return SALEC_OK;
}

// AoS staging buffer of at least `need` doubles (stream-ordered: no device-wide synchronisation)
int ensure_staging(salec_gpu *h, size_t need)
{
    if (need <= h->staging_doubles) return SALEC_OK;
    if (h->staging) CUDA_TRY(cudaFreeAsync(h->staging, h->stream));
    h->staging = nullptr;
    h->staging_doubles = 0;
    CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&h->staging), need * sizeof(double), h->stream));
    h->staging_doubles = need;
    return SALEC_OK;
}

int transfer(salec_gpu *h, int fid, double *host, long long n, bool to_device)
{
    if (fid < 0 || fid >= kNumFields) return fail(SALEC_ERR_ARG, "unknown field");
    int nx, ny;
    field_points(h, fid, nx, ny);
    const int nc = field_ncomp(h, fid);
    const long long need = (long long)nx * ny * nc;
    if (n != need) return fail(SALEC_ERR_ARG, std::string("field ") + kFields[fid].name + ": expected " +
                                                  std::to_string(need) + " doubles, got " + std::to_string(n));
    if (int rc = ensure_staging(h, (size_t)need)) return rc;
    void *base = field_ptr(h, fid);
    const bool f32 = field_f32(h, fid);
    const long long plane = kFields[fid].loc == L_COL ? 0 : h->d.PL;
    if (to_device) {
        CUDA_TRY(cudaMemcpyAsync(h->staging, host, need * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        launch_aos_to_planes(h->staging, base, f32, plane, h->d.P, nx, ny, nc, h->stream);
        CUDA_TRY(cudaGetLastError());
        for (int k = 0; k < 5; ++k)
            if (!strcmp(kFields[fid].name, kGeoFields[k])) {
                int rc = build_geo_table(h, k, fid, nx, ny, nc);
                if (rc) return rc;
            }
        if (!strcmp(kFields[fid].name, "v_laplace")) {
            if (h->mixed) launch_step_kernel(SK_LAPLACE_MASK, h->ctx_t<float>(), h->stream, h->blk[SK_LAPLACE_MASK]);
            else launch_step_kernel(SK_LAPLACE_MASK, h->ctx_t<double>(), h->stream, h->blk[SK_LAPLACE_MASK]);
            CUDA_TRY(cudaGetLastError());
        }
        CUDA_TRY(cudaStreamSynchronize(h->stream));
    } else {
        launch_planes_to_aos(base, f32, h->staging, plane, h->d.P, nx, ny, nc, h->stream);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(host, h->staging, need * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
    return SALEC_OK;
}

void adjoint_release(salec_gpu *h);
void adjoint_drop_graphs(salec_gpu *h);

void release(salec_gpu *h)
{
    if (!h) return;
    salec_internal_output_release(h->output);
    if (h->conserve) cudaFree(h->conserve);
    if (h->dt_sched) cudaFree(h->dt_sched);
    adjoint_release(h);
    for (void *p : h->owned) cudaFree(p);
    if (h->pool) cudaFree(h->pool);
    if (h->staging) cudaFree(h->staging);
    if (h->scal) cudaFree(h->scal);
    if (h->scal_host) cudaFreeHost(h->scal_host);
    if (h->mat) cudaFree(h->mat);
    if (h->tr_block) cudaFree(h->tr_block);
    if (h->lap_mask) cudaFree(h->lap_mask);
    for (auto &g : h->geo)
        if (g.compact) { cudaFree(g.tab); cudaFree(g.row); }
    if (h->row_identity) cudaFree(h->row_identity);
    if (h->cycle_graph) cudaGraphExecDestroy(h->cycle_graph);
    for (auto e : h->ev_a) cudaEventDestroy(e);
    for (auto e : h->ev_b) cudaEventDestroy(e);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    for (int k = 0; k < 2; ++k) {
        if (h->report_scal[k]) cudaFreeHost(h->report_scal[k]);
        if (h->report_ev[k]) cudaEventDestroy(h->report_ev[k]);
    }
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

template <class R>
int finish_init_t(salec_gpu *h, double damp_time_in, double *damp_time_out)
{
    const CtxT<R> c = h->ctx_t<R>();
    launch_step_kernel(SK_REMAP_DAMP_STATE, c, h->stream, h->blk[SK_REMAP_DAMP_STATE], 0, 0, 0, 1);
    int rc = run_gather(h, h->g_init);
    if (rc) return rc;
    CUDA_TRY(cudaMemsetAsync(&h->scal->aux, 0, sizeof(unsigned long long), h->stream));
    launch_step_kernel(SK_RECORD_REFERENCE, c, h->stream, h->blk[SK_RECORD_REFERENCE]);
    CUDA_TRY(cudaGetLastError());
    unsigned long long mx = 0;
    CUDA_TRY(cudaMemcpyAsync(&h->scal_host->aux, &h->scal->aux, sizeof(mx), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    mx = h->scal_host->aux;
    const double local = mx ? ord_decode(mx) : 0.0;
    const double dt2 = local * 2.0;
    h->rp.damp_time = dmax(dt2, damp_time_in);
    if (damp_time_out) *damp_time_out = h->rp.damp_time;
    launch_step_kernel(SK_INIT_VERTEX_VELOCITY, h->ctx_t<R>(), h->stream, h->blk[SK_INIT_VERTEX_VELOCITY]);
    CUDA_TRY(cudaGetLastError());
    for (const char *nm : {"e_vel", "e_ste", "e_dvel"}) {
        int fid = field_by_name(nm);
        CUDA_TRY(cudaMemsetAsync(field_ptr(h, fid), 0, (size_t)field_ncomp(h, fid) * h->d.PL * field_elem(h, fid),
                                 h->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SALEC_OK;
}

} // namespace

// Last start-up steps on the device (src/salec2d.c:76-94): first EOS call, ghost fills,
// damping reference state and arrival time, vertex velocities, cleared cell velocities.
int salec_internal_finish_init(salec_gpu *h, double damp_time_in, double *damp_time_out)
{
    return h->mixed ? finish_init_t<float>(h, damp_time_in, damp_time_out)
                    : finish_init_t<double>(h, damp_time_in, damp_time_out);
}

int salec_internal_fail(int code, const char *msg) { return fail(code, msg ? msg : "error"); }

// Views of the handle for the output writer (salec_output.cu).
int salec_internal_field_view(salec_gpu *h, const char *name, const void **base, int *f32, long long *plane,
                              int *pitch, int *nx, int *ny, int *nc)
{
    const int fid = field_by_name(name);
    if (fid < 0) return fail(SALEC_ERR_ARG, std::string("unknown field ") + name);
    field_points(h, fid, *nx, *ny);
    *nc = field_ncomp(h, fid);
    *base = field_ptr(h, fid);
    *f32 = field_f32(h, fid) ? 1 : 0;
    *plane = kFields[fid].loc == L_COL ? 0 : h->d.PL;
    *pitch = h->d.P;
    return SALEC_OK;
}
cudaStream_t salec_internal_stream(salec_gpu *h) { return h->stream; }
Tracers salec_internal_tracers(salec_gpu *h) { return h->tr; }
Dims salec_internal_dims(salec_gpu *h) { return h->d; }
void salec_internal_add_launches(salec_gpu *h, int n) { h->launches += n; }
void *&salec_internal_output_slot(salec_gpu *h) { return h->output; }
void *&salec_internal_conserve_slot(salec_gpu *h) { return h->conserve; }

// ================================================================== C ABI
extern "C" {

const char *salec_gpu_last_error(void) { return g_last_error.c_str(); }

int salec_gpu_func_index(const char *name)
{
    if (!name) return -1;
    for (int k = 0; k < (int)(sizeof(kFuncNames) / sizeof(kFuncNames[0])); ++k) {
        const char *a = kFuncNames[k], *b = name;
        while (*a && *b && tolower((unsigned char)*a) == tolower((unsigned char)*b)) { ++a; ++b; }
        if (*a == 0 && *b == 0) return k;
    }
    return -1;
}

int salec_gpu_field_index(const char *name) { return field_by_name(name); }

int salec_boundary_map(int kind, int pattern, int nx, int ny, int ncomp, const int go[4], int *n, int *dst,
                       int *src, unsigned *ops)
{
    if (!go || !n || nx < 8 || ny < 8 || ncomp < 1 || ncomp > 10 || pattern < 0 || pattern > 5)
        return fail(SALEC_ERR_ARG, "bad boundary map request");
    GatherMap m;
    if (kind == 0) m = build_ghost_map(nx, ny, nx, ncomp, go, (GhostPattern)pattern);
    else if (kind == 1) m = build_restrict_map(nx, ny, nx, ncomp, go);
    else return fail(SALEC_ERR_ARG, "kind must be 0 (ghost) or 1 (restrict)");
    const int cnt = (int)m.dst.size();
    if (dst && src && ops) {
        if (*n < cnt) { *n = cnt; return fail(SALEC_ERR_ARG, "map buffer too small"); }
        for (int k = 0; k < cnt; ++k) { dst[k] = m.dst[k]; src[k] = m.src[k]; ops[k] = m.ops[k]; }
    }
    *n = cnt;
    return SALEC_OK;
}

int salec_gpu_get_run(const salec_gpu *h, salec_run_desc *out)
{
    if (!h || !out) return fail(SALEC_ERR_ARG, "null argument");
    *out = h->run;
    out->damp_time = h->rp.damp_time;
    return SALEC_OK;
}

int salec_gpu_create(const salec_run_desc *run, const salec_material_desc *mats, salec_gpu **out)
{
    if (!run || !mats || !out) return fail(SALEC_ERR_ARG, "null argument");
    *out = nullptr;
    if (run->nx < 4 || run->ny < 4) return fail(SALEC_ERR_ARG, "mesh must have at least 4x4 cells");
    if (run->nmat < 2 || run->nmat > SALEC_MAXMAT) return fail(SALEC_ERR_ARG, "nmat must be in [2, 10]");
    if (run->damp_type < 0 || run->damp_type > 5) return fail(SALEC_ERR_ARG, "unknown damping type");
    if (run->precision != SALEC_PRECISION_FP64 && run->precision != SALEC_PRECISION_MIXED)
        return fail(SALEC_ERR_ARG, "precision must be SALEC_PRECISION_FP64 or SALEC_PRECISION_MIXED");
    salec_gpu *h = new salec_gpu();
    for (int k = 0; k < SK_COUNT; ++k) h->blk[k] = dim3(32, 4);
    Dims &d = h->d;
    d.nmat = run->nmat;
    d.enx = run->nx + 4;
    d.eny = run->ny + 4;
    d.vnx = run->nx + 5;
    d.vny = run->ny + 5;
    d.phi = 3 * d.nmat + 10 + (run->porosity_model ? d.nmat + 1 : 0);
    d.P = ((d.vnx + 31) / 32) * 32;
    d.R = d.vny;
    d.PL = (((long long)d.P * d.R + 31) / 32) * 32;
    for (int k = 0; k < 4; ++k) h->go[k] = run->go[k];
    h->run = *run;
    RunParams &rp = h->rp;
    rp.damp_type = run->damp_type; rp.partpres = run->partpres; rp.porosity_model = run->porosity_model;
    rp.acoustic_fluid = run->acoustic_fluid; rp.tensile_failure = run->tensile_failure;
    rp.tracer_lubrication = run->tracer_lubrication;
    rp.tracer_lub_gy0 = run->tracer_lub_gy0;
    rp.tracer_lub_gy1 = run->tracer_lub_gy1;
    rp.avis1 = run->avis1; rp.avis2 = run->avis2; rp.anc = run->anc;
    rp.density_cutoff = run->density_cutoff; rp.velocity_max = run->velocity_max;
    rp.velocity_min = run->velocity_min; rp.acceleration_min = run->acceleration_min;
    rp.alpha_damp_x = run->alpha_damp_x; rp.alpha_damp_y = run->alpha_damp_y; rp.damp_time = run->damp_time;
    rp.threshold_z = run->threshold_z; rp.flow_resistance = run->flow_resistance;
    rp.flow_friction = run->flow_friction; rp.tracer_lub_y0 = run->tracer_lub_y0;
    rp.tracer_lub_frac = run->tracer_lub_frac; rp.max_dt = run->max_dt;

    auto bail = [&](int rc) { release(h); return rc; };
    if (cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(SALEC_ERR_CUDA, "side stream or events"));
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(SALEC_ERR_CUDA, "cudaStreamCreate failed"));

    // one pool, every component plane 128-byte aligned (PL is a multiple of 32 elements)
    h->mixed = run->precision == SALEC_PRECISION_MIXED ? 1 : 0;
    const size_t col = (((size_t)d.enx + 31) / 32) * 32;
    size_t bytes = 0;
    for (int k = 0; k < kNumFields; ++k)
        bytes += kFields[k].loc == L_COL ? col * sizeof(double) : (size_t)field_ncomp(h, k) * d.PL * field_elem(h, k);
    h->pool_bytes = bytes;
    if (cudaMalloc(&h->pool, h->pool_bytes) != cudaSuccess)
        return bail(fail(SALEC_ERR_ALLOC, "device pool of " + std::to_string(h->pool_bytes) + " bytes"));
    if (cudaMemsetAsync(h->pool, 0, h->pool_bytes, h->stream) != cudaSuccess)
        return bail(fail(SALEC_ERR_CUDA, "pool memset failed"));
    size_t off = 0;
    for (int k = 0; k < kNumFields; ++k) {
        field_ptr(h, k) = reinterpret_cast<double *>(h->pool + off);
        off += kFields[k].loc == L_COL ? col * sizeof(double) : (size_t)field_ncomp(h, k) * d.PL * field_elem(h, k);
    }

    {
        const size_t words = (size_t)(d.P / 32) * d.R;
        if (cudaMalloc(&h->lap_mask, words * sizeof(unsigned)) != cudaSuccess)
            return bail(fail(SALEC_ERR_ALLOC, "Laplacian mask"));
        if (cudaMemsetAsync(h->lap_mask, 0, words * sizeof(unsigned), h->stream) != cudaSuccess)
            return bail(fail(SALEC_ERR_CUDA, "Laplacian mask memset"));
    }
    {
        std::vector<int> ident(d.R);
        for (int j = 0; j < d.R; ++j) ident[j] = j;
        if (cudaMalloc(&h->row_identity, sizeof(int) * d.R) != cudaSuccess)
            return bail(fail(SALEC_ERR_ALLOC, "row map"));
        if (cudaMemcpy(h->row_identity, ident.data(), sizeof(int) * d.R, cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(fail(SALEC_ERR_CUDA, "row map upload"));
        for (int k = 0; k < 5; ++k) {
            h->geo[k].tab = field_ptr(h, field_by_name(kGeoFields[k]));
            h->geo[k].row = h->row_identity;
            h->geo[k].plane = d.PL;
        }
    }

    std::vector<DevMat> dms(d.nmat);
    memset(dms.data(), 0, sizeof(DevMat) * d.nmat);
    for (int m = 1; m < d.nmat; ++m) {
        int rc = upload_material(h, mats[m], dms[m]);
        if (rc) return bail(rc);
    }
    if (int rc = flush_uploads(h)) return bail(rc);
    if (cudaMalloc(&h->mat, sizeof(DevMat) * d.nmat) != cudaSuccess) return bail(fail(SALEC_ERR_ALLOC, "materials"));
    if (cudaMemcpy(h->mat, dms.data(), sizeof(DevMat) * d.nmat, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(SALEC_ERR_CUDA, "material upload"));

    if (cudaMalloc(&h->scal, sizeof(Scal)) != cudaSuccess) return bail(fail(SALEC_ERR_ALLOC, "scalars"));
    if (cudaMallocHost(&h->scal_host, sizeof(Scal)) != cudaSuccess) return bail(fail(SALEC_ERR_ALLOC, "scalars"));
    Scal s0{};
    s0.dt = run->dt;
    s0.time = run->time;
    s0.i_step = run->i_step;
    s0.dt_acc = ord_encode(1.1 * run->dt);
    s0.dt_nan_last = -1;
    s0.dt_tail = ~0ULL;
    if (cudaMemcpy(h->scal, &s0, sizeof(Scal), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(SALEC_ERR_CUDA, "scalar upload"));

    int rc = build_gathers(h);
    if (rc) return bail(rc);
    if ((rc = flush_uploads(h))) return bail(rc);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(fail(SALEC_ERR_CUDA, "create sync"));
    *out = h;
    return SALEC_OK;
}

int salec_gpu_destroy(salec_gpu *h)
{
    if (!h) return fail(SALEC_ERR_ARG, "null handle");
    cudaStreamSynchronize(h->stream);
    release(h);
    return SALEC_OK;
}

int salec_gpu_field_shape(const salec_gpu *h, int field, int *nx, int *ny, int *ncomp)
{
    if (!h || field < 0 || field >= kNumFields) return fail(SALEC_ERR_ARG, "bad handle or field");
    int a, b;
    field_points(h, field, a, b);
    if (nx) *nx = a;
    if (ny) *ny = b;
    if (ncomp) *ncomp = field_ncomp(h, field);
    return SALEC_OK;
}

int salec_gpu_set_field(salec_gpu *h, int field, const double *host, long long n)
{
    if (!h || !host) return fail(SALEC_ERR_ARG, "null argument");
    return transfer(h, field, const_cast<double *>(host), n, true);
}

int salec_gpu_get_field(salec_gpu *h, int field, double *host, long long n)
{
    if (!h || !host) return fail(SALEC_ERR_ARG, "null argument");
    return transfer(h, field, host, n, false);
}

int salec_gpu_phases(salec_gpu *h, int first, int last)
{
    if (!h) return fail(SALEC_ERR_ARG, "null handle");
    if (first < 0 || last > 15 || first > last) return fail(SALEC_ERR_ARG, "phase range must lie in [0, 15]");
    for (int p = first; p <= last; ++p) {
        if (h->profiling) {
            if (h->ev_used == h->ev_a.size()) {
                cudaEvent_t a, b;
                CUDA_TRY(cudaEventCreate(&a));
                CUDA_TRY(cudaEventCreate(&b));
                h->ev_a.push_back(a);
                h->ev_b.push_back(b);
                h->ev_phase.push_back(0);
            }
            const size_t k = h->ev_used++;
            h->ev_phase[k] = p;
            CUDA_TRY(cudaEventRecord(h->ev_a[k], h->stream));
            int rc = run_phase(h, p);
            if (rc) return rc;
            CUDA_TRY(cudaEventRecord(h->ev_b[k], h->stream));
        } else {
            int rc = run_phase(h, p);
            if (rc) return rc;
        }
    }
    return SALEC_OK;
}

namespace {

void drop_cycle_graph(salec_gpu *h)
{
    if (h->cycle_graph) cudaGraphExecDestroy(h->cycle_graph);
    h->cycle_graph = nullptr;
    adjoint_drop_graphs(h);
}

// Capture phases 0-15 of one cycle on the handle's stream into a graph; on any failure the
// cycle is simply launched kernel by kernel.
void capture_cycle_graph(salec_gpu *h)
{
    cudaGraph_t g = nullptr;
    const long long before = h->launches;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    int rc = SALEC_OK;
    h->fork_tracers = true;
    for (int p = 0; p <= 15 && rc == SALEC_OK; ++p) rc = run_phase(h, p, true);
    h->fork_tracers = false;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->launches = before;
    if (rc != SALEC_OK || e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return;
    }
    cudaGraphExec_t exec = nullptr;
    if (cudaGraphInstantiate(&exec, g, 0) == cudaSuccess) {
        h->cycle_graph = exec;
        size_t n = 0;
        cudaGraphGetNodes(g, nullptr, &n);
        std::vector<cudaGraphNode_t> nodes(n);
        long long kernels = 0;
        if (n && cudaGraphGetNodes(g, nodes.data(), &n) == cudaSuccess)
            for (size_t k = 0; k < n; ++k) {
                cudaGraphNodeType ty;
                if (cudaGraphNodeGetType(nodes[k], &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel) ++kernels;
            }
        h->cycle_graph_launches = kernels;
    }
    cudaGraphDestroy(g);
    cudaGetLastError();
}

} // namespace

int salec_gpu_step(salec_gpu *h, int nsteps)
{
    if (!h) return fail(SALEC_ERR_ARG, "null handle");
    if (nsteps < 0) return fail(SALEC_ERR_ARG, "negative step count");
    if (!h->profiling && nsteps > 0 && !h->cycle_graph) capture_cycle_graph(h);
    for (int k = 0; k < nsteps; ++k) {
        if (!h->profiling && h->cycle_graph) {
            CUDA_TRY(cudaGraphLaunch(h->cycle_graph, h->stream));
            h->launches += h->cycle_graph_launches;
        } else {
            int rc = salec_gpu_phases(h, 0, 15);
            if (rc) return rc;
        }
    }
    return SALEC_OK;
}

int salec_gpu_step_report(salec_gpu *h, int nsteps, double *dt, double *time, double *profile, long long profile_n)
{
    if (!h) return fail(SALEC_ERR_ARG, "null handle");
    const int fid = field_by_name("y_profile");
    int nx = 0, ny = 0;
    field_points(h, fid, nx, ny);
    const long long need = (long long)nx * ny * field_ncomp(h, fid);
    if (profile && profile_n != need)
        return fail(SALEC_ERR_ARG, "y_profile: expected " + std::to_string(need) + " doubles, got " +
                                       std::to_string(profile_n));
    if (profile) {
        if (int rc = ensure_staging(h, (size_t)need)) return rc;
    }
    if (int rc = salec_gpu_step(h, nsteps)) return rc;
    // both read-backs queue behind the cycles; one synchronisation for all of them
    CUDA_TRY(cudaMemcpyAsync(h->scal_host, h->scal, sizeof(Scal), cudaMemcpyDeviceToHost, h->stream));
    if (profile) {
        const long long plane = kFields[fid].loc == L_COL ? 0 : h->d.PL;
        launch_planes_to_aos(field_ptr(h, fid), field_f32(h, fid), h->staging, plane, h->d.P, nx, ny,
                             field_ncomp(h, fid), h->stream);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(profile, h->staging, need * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (dt) *dt = h->scal_host->dt;
    if (time) *time = h->scal_host->time;
    return SALEC_OK;
}

int salec_gpu_step_report_async(salec_gpu *h, int nsteps, double *profile, long long profile_n, int slot)
{
    if (!h) return fail(SALEC_ERR_ARG, "null handle");
    if (slot < 0 || slot > 1) return fail(SALEC_ERR_ARG, "report slot must be 0 or 1");
    if (h->report_pending[slot]) return fail(SALEC_ERR_STATE, "report slot still in flight: wait for it first");
    const int fid = field_by_name("y_profile");
    int nx = 0, ny = 0;
    field_points(h, fid, nx, ny);
    const long long need = (long long)nx * ny * field_ncomp(h, fid);
    if (profile && profile_n != need)
        return fail(SALEC_ERR_ARG, "y_profile: expected " + std::to_string(need) + " doubles, got " +
                                       std::to_string(profile_n));
    if (profile) {
        if (int rc = ensure_staging(h, (size_t)need)) return rc;
    }
    if (!h->report_scal[slot]) {
        CUDA_TRY(cudaMallocHost(reinterpret_cast<void **>(&h->report_scal[slot]), sizeof(Scal)));
        CUDA_TRY(cudaEventCreateWithFlags(&h->report_ev[slot], cudaEventDisableTiming));
    }
    if (int rc = salec_gpu_step(h, nsteps)) return rc;
    // the copies queue behind the cycles; the staging buffer is reused in stream order
    CUDA_TRY(cudaMemcpyAsync(h->report_scal[slot], h->scal, sizeof(Scal), cudaMemcpyDeviceToHost, h->stream));
    if (profile) {
        const long long plane = kFields[fid].loc == L_COL ? 0 : h->d.PL;
        launch_planes_to_aos(field_ptr(h, fid), field_f32(h, fid), h->staging, plane, h->d.P, nx, ny,
                             field_ncomp(h, fid), h->stream);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(profile, h->staging, need * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    CUDA_TRY(cudaEventRecord(h->report_ev[slot], h->stream));
    h->report_pending[slot] = true;
    return SALEC_OK;
}

int salec_gpu_report_wait(salec_gpu *h, int slot, double *dt, double *time)
{
    if (!h) return fail(SALEC_ERR_ARG, "null handle");
    if (slot < 0 || slot > 1) return fail(SALEC_ERR_ARG, "report slot must be 0 or 1");
    if (!h->report_pending[slot]) return fail(SALEC_ERR_STATE, "report slot not queued");
    h->report_pending[slot] = false;
    CUDA_TRY(cudaEventSynchronize(h->report_ev[slot]));
    if (dt) *dt = h->report_scal[slot]->dt;
    if (time) *time = h->report_scal[slot]->time;
    return SALEC_OK;
}

int salec_gpu_step_many(salec_gpu *const *handles, int n, int nsteps, int chunk)
{
    if (!handles || n < 0 || nsteps < 0) return fail(SALEC_ERR_ARG, "bad argument");
    for (int k = 0; k < n; ++k)
        if (!handles[k]) return fail(SALEC_ERR_ARG, "null handle in the ensemble");
    if (chunk <= 0) chunk = 16;
    // round-robin: every member gets `chunk` cycles queued on its own stream before the next
    // member's turn, so the members' kernels overlap on the device
    for (int done = 0; done < nsteps; done += chunk) {
        const int k_steps = std::min(chunk, nsteps - done);
        for (int k = 0; k < n; ++k) {
            int rc = salec_gpu_step(handles[k], k_steps);
            if (rc) return rc;
        }
    }
    return SALEC_OK;
}

int salec_gpu_stream(salec_gpu *h, void **stream)
{
    if (!h || !stream) return fail(SALEC_ERR_ARG, "null argument");
    *stream = (void *)h->stream;
    return SALEC_OK;
}

int salec_gpu_profile(salec_gpu *h, int enable)
{
    if (!h) return fail(SALEC_ERR_ARG, "null handle");
    h->profiling = enable ? 1 : 0;
    h->ev_used = 0;
    return SALEC_OK;
}

int salec_gpu_phase_times(salec_gpu *h, double *ms, long long *count)
{
    if (!h || !ms || !count) return fail(SALEC_ERR_ARG, "null argument");
    for (int p = 0; p < 16; ++p) { ms[p] = 0.0; count[p] = 0; }
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (size_t k = 0; k < h->ev_used; ++k) {
        float t = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&t, h->ev_a[k], h->ev_b[k]));
        ms[h->ev_phase[k]] += t;
        count[h->ev_phase[k]] += 1;
    }
    h->ev_used = 0;
    return SALEC_OK;
}

namespace {
// the 2-D sweep of each phase whose block shape is tunable
const int kTunedPhase[] = {1, 3, 4, 5, 7, 8, 9, 10, 12, 14};
const StepKernel kTunedKernel[] = {SK_VERTEX_VOF_MOMENTUM, SK_CELL_VELOCITY, SK_VOID_VERTICES, SK_GRADIENT,
                                   SK_STRESS, SK_ACCELERATION, SK_DISPLACEMENT, SK_ENERGY, SK_FLUX,
                                   SK_REMAP_DAMP_STATE};
constexpr int kNumTuned = sizeof(kTunedPhase) / sizeof(kTunedPhase[0]);
}   // namespace

int salec_gpu_set_block_shapes(salec_gpu *h, const int *shapes, int n)
{
    if (!h || (n > 0 && !shapes) || n < 0) return fail(SALEC_ERR_ARG, "bad argument");
    for (int k = 0; k < n; ++k) {
        const int p = shapes[3 * k], bx = shapes[3 * k + 1], by = shapes[3 * k + 2];
        int t = 0;
        while (t < kNumTuned && kTunedPhase[t] != p) ++t;
        if (t == kNumTuned) return fail(SALEC_ERR_ARG, "phase " + std::to_string(p) + " has no tunable block shape");
        if (bx < 32 || bx % 32 || by < 1 || bx * by > 256)
            return fail(SALEC_ERR_ARG, "block shape " + std::to_string(bx) + "x" + std::to_string(by) +
                                           ": x must be a multiple of 32 and x*y at most 256");
    }
    for (int k = 0; k < n; ++k) {
        int t = 0;
        while (kTunedPhase[t] != shapes[3 * k]) ++t;
        h->blk[kTunedKernel[t]] = dim3(shapes[3 * k + 1], shapes[3 * k + 2]);
    }
    if (h->cycle_graph) { cudaGraphExecDestroy(h->cycle_graph); h->cycle_graph = nullptr; }
    return SALEC_OK;
}

int salec_gpu_autotune(salec_gpu *h, int cycles, int *shapes)
{
    if (!h || cycles < 1) return fail(SALEC_ERR_ARG, "bad argument");
    static const dim3 cand[] = {dim3(32, 4), dim3(32, 8), dim3(64, 2), dim3(32, 2), dim3(64, 4), dim3(128, 1),
                                dim3(32, 1), dim3(64, 1)};
    constexpr int ncand = sizeof(cand) / sizeof(cand[0]);
    const int *tuned_phase = kTunedPhase;
    const StepKernel *tuned_kernel = kTunedKernel;
    constexpr int ntuned = kNumTuned;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    // snapshot of everything the cycles change: the field pool, the scalars and the tracers
    void *snap = nullptr, *snap_tr = nullptr;
    Scal scal_host{};
    CUDA_TRY(cudaMemcpy(&scal_host, h->scal, sizeof(Scal), cudaMemcpyDeviceToHost));
    if (cudaMalloc(&snap, h->pool_bytes) != cudaSuccess) return fail(SALEC_ERR_ALLOC, "autotune snapshot");
    if (h->tr_bytes && cudaMalloc(&snap_tr, h->tr_bytes) != cudaSuccess) {
        cudaFree(snap);
        return fail(SALEC_ERR_ALLOC, "autotune snapshot");
    }
    auto restore = [&]() -> int {
        CUDA_TRY(cudaMemcpyAsync(h->pool, snap, h->pool_bytes, cudaMemcpyDeviceToDevice, h->stream));
        if (snap_tr) CUDA_TRY(cudaMemcpyAsync(h->tr_block, snap_tr, h->tr_bytes, cudaMemcpyDeviceToDevice, h->stream));
        CUDA_TRY(cudaMemcpyAsync(h->scal, &scal_host, sizeof(Scal), cudaMemcpyHostToDevice, h->stream));
        CUDA_TRY(cudaStreamSynchronize(h->stream));
        return SALEC_OK;
    };
    int rc = SALEC_OK;
    if (cudaMemcpyAsync(snap, h->pool, h->pool_bytes, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess ||
        (snap_tr && cudaMemcpyAsync(snap_tr, h->tr_block, h->tr_bytes, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess))
        rc = fail(SALEC_ERR_CUDA, "autotune snapshot copy");
    std::vector<double> best_ms(ntuned, 1e300);
    std::vector<int> best(ntuned, 0);
    const int was_profiling = h->profiling;
    for (int ci = 0; ci < ncand && rc == SALEC_OK; ++ci) {
        for (int t = 0; t < ntuned; ++t) h->blk[tuned_kernel[t]] = cand[ci];
        if ((rc = restore())) break;
        h->profiling = 1;
        h->ev_used = 0;
        for (int cy = 0; cy < cycles + 1 && rc == SALEC_OK; ++cy) {
            if (cy == 1) h->ev_used = 0;   // the first cycle warms up
            rc = salec_gpu_phases(h, 0, 15);
        }
        if (rc) break;
        double ms[16];
        long long cnt[16];
        if ((rc = salec_gpu_phase_times(h, ms, cnt))) break;
        for (int t = 0; t < ntuned; ++t) {
            const int p = tuned_phase[t];
            const double m = cnt[p] ? ms[p] / cnt[p] : 1e300;
            if (m < best_ms[t]) { best_ms[t] = m; best[t] = ci; }
        }
    }
    h->profiling = was_profiling;
    h->ev_used = 0;
    for (int t = 0; t < ntuned; ++t) h->blk[tuned_kernel[t]] = cand[best[t]];
    const int rc2 = restore();
    cudaFree(snap);
    if (snap_tr) cudaFree(snap_tr);
    if (h->cycle_graph) { cudaGraphExecDestroy(h->cycle_graph); h->cycle_graph = nullptr; }
    if (rc) return rc;
    if (rc2) return rc2;
    if (shapes)
        for (int t = 0; t < ntuned; ++t) {
            shapes[3 * t] = tuned_phase[t];
            shapes[3 * t + 1] = (int)cand[best[t]].x;
            shapes[3 * t + 2] = (int)cand[best[t]].y;
        }
    return SALEC_OK;
}

int salec_gpu_sync(salec_gpu *h)
{
    if (!h) return fail(SALEC_ERR_ARG, "null handle");
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SALEC_OK;
}

int salec_gpu_get_scalar(salec_gpu *h, const char *name, double *value)
{
    if (!h || !name || !value) return fail(SALEC_ERR_ARG, "null argument");
    CUDA_TRY(cudaMemcpyAsync(h->scal_host, h->scal, sizeof(Scal), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    const Scal &s = *h->scal_host;
    if (!strcmp(name, "dt")) *value = s.dt;
    else if (!strcmp(name, "time")) *value = s.time;
    else if (!strcmp(name, "i_step")) *value = (double)s.i_step;
    else if (!strcmp(name, "dt_candidate")) *value = ord_decode(s.dt_acc);
    else if (!strcmp(name, "damp_time")) *value = h->rp.damp_time;
    else if (!strcmp(name, "max_dt")) *value = h->rp.max_dt;
    else if (!strcmp(name, "launches")) *value = (double)h->launches;
    else return fail(SALEC_ERR_ARG, std::string("unknown scalar ") + name);
    return SALEC_OK;
}

int salec_gpu_set_scalar(salec_gpu *h, const char *name, double value)
{
    if (!h || !name) return fail(SALEC_ERR_ARG, "null argument");
    if (!strcmp(name, "damp_time")) { h->rp.damp_time = value; drop_cycle_graph(h); return SALEC_OK; }
    if (!strcmp(name, "max_dt")) { h->rp.max_dt = value; drop_cycle_graph(h); return SALEC_OK; }
    CUDA_TRY(cudaMemcpyAsync(h->scal_host, h->scal, sizeof(Scal), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    Scal s = *h->scal_host;
    if (!strcmp(name, "dt")) { s.dt = value; s.dt_acc = ord_encode(1.1 * value); s.dt_nan_last = -1; }
    else if (!strcmp(name, "time")) s.time = value;
    else if (!strcmp(name, "i_step")) s.i_step = (long long)value;
    else return fail(SALEC_ERR_ARG, std::string("unknown scalar ") + name);
    *h->scal_host = s;
    CUDA_TRY(cudaMemcpyAsync(h->scal, h->scal_host, sizeof(Scal), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SALEC_OK;
}

int salec_gpu_set_tracers(salec_gpu *h, int n, const double *rows)
{
    if (!h || n < 0 || (n > 0 && !rows)) return fail(SALEC_ERR_ARG, "bad argument");
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    drop_cycle_graph(h);
    if (h->tr_block) cudaFree(h->tr_block);
    h->tr_block = nullptr;
    h->tr = Tracers();
    if (n == 0) return SALEC_OK;
    const size_t nd = 6, nf = 2, ni = 7;
    auto rounded = [](size_t sz) { return ((sz + 255) / 256) * 256; };
    const size_t bytes = nd * rounded((size_t)n * 8) + (nf + ni) * rounded((size_t)n * 4);
    CUDA_TRY(cudaMalloc(&h->tr_block, bytes));
    h->tr_bytes = bytes;
    char *p = static_cast<char *>(h->tr_block);
    char *const end = p + bytes;
    auto take = [&](size_t sz) { char *q = p; p += rounded(sz); return q; };
    Tracers &T = h->tr;
    T.n = n;
    std::vector<double> d(nd * (size_t)n);
    std::vector<float> f(nf * (size_t)n);
    std::vector<int> iv(ni * (size_t)n);
    for (int t = 0; t < n; ++t) {
        const double *r = rows + 12 * (size_t)t;
        d[0 * (size_t)n + t] = r[0]; d[1 * (size_t)n + t] = r[1];
        d[2 * (size_t)n + t] = r[2]; d[3 * (size_t)n + t] = r[3];
        d[4 * (size_t)n + t] = 0.0; d[5 * (size_t)n + t] = 0.0;
        f[0 * (size_t)n + t] = (float)r[4]; f[1 * (size_t)n + t] = (float)r[5];
        for (int q = 0; q < 6; ++q) iv[q * (size_t)n + t] = (int)r[6 + q];
        iv[6 * (size_t)n + t] = 1;
    }
    double **dp[6] = {&T.x, &T.y, &T.vx, &T.vy, &T.rec_pre, &T.rec_tem};
    for (int q = 0; q < 6; ++q) {
        *dp[q] = reinterpret_cast<double *>(take((size_t)n * 8));
        CUDA_TRY(cudaMemcpy(*dp[q], d.data() + q * (size_t)n, (size_t)n * 8, cudaMemcpyHostToDevice));
    }
    float **fp[2] = {&T.mpre, &T.mtem};
    for (int q = 0; q < 2; ++q) {
        *fp[q] = reinterpret_cast<float *>(take((size_t)n * 4));
        CUDA_TRY(cudaMemcpy(*fp[q], f.data() + q * (size_t)n, (size_t)n * 4, cudaMemcpyHostToDevice));
    }
    int **ip[7] = {&T.gx, &T.gy, &T.tag, &T.matid, &T.cx, &T.cy, &T.alive};
    for (int q = 0; q < 7; ++q) {
        *ip[q] = reinterpret_cast<int *>(take((size_t)n * 4));
        CUDA_TRY(cudaMemcpy(*ip[q], iv.data() + q * (size_t)n, (size_t)n * 4, cudaMemcpyHostToDevice));
    }
    if (p > end) return fail(SALEC_ERR_STATE, "tracer block layout overflow");
    return SALEC_OK;
}

int salec_gpu_get_tracers(salec_gpu *h, double *rows, int *n)
{
    if (!h || !n) return fail(SALEC_ERR_ARG, "bad argument");
    const Tracers &T = h->tr;
    const size_t m = (size_t)T.n;
    std::vector<double> d(6 * m);
    std::vector<float> f(2 * m);
    std::vector<int> iv(7 * m);
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (m) {
        const double *dp[6] = {T.x, T.y, T.vx, T.vy, T.rec_pre, T.rec_tem};
        for (int q = 0; q < 6; ++q) CUDA_TRY(cudaMemcpy(d.data() + q * m, dp[q], m * 8, cudaMemcpyDeviceToHost));
        const float *fp[2] = {T.mpre, T.mtem};
        for (int q = 0; q < 2; ++q) CUDA_TRY(cudaMemcpy(f.data() + q * m, fp[q], m * 4, cudaMemcpyDeviceToHost));
        const int *ip[7] = {T.gx, T.gy, T.tag, T.matid, T.cx, T.cy, T.alive};
        for (int q = 0; q < 7; ++q) CUDA_TRY(cudaMemcpy(iv.data() + q * m, ip[q], m * 4, cudaMemcpyDeviceToHost));
    }
    int live = 0;
    for (size_t t = 0; t < m; ++t)
        if (iv[6 * m + t]) ++live;
    if (!rows) { *n = live; return SALEC_OK; }
    if (*n < live) { int cap = *n; *n = live; return fail(SALEC_ERR_ARG, "tracer buffer holds " + std::to_string(cap) + " rows, need " + std::to_string(live)); }
    int o = 0;
    for (size_t t = 0; t < m; ++t) {
        if (!iv[6 * m + t]) continue;
        double *r = rows + 12 * (size_t)o++;
        r[0] = d[0 * m + t]; r[1] = d[1 * m + t]; r[2] = d[2 * m + t]; r[3] = d[3 * m + t];
        r[4] = f[0 * m + t]; r[5] = f[1 * m + t];
        for (int q = 0; q < 6; ++q) r[6 + q] = iv[q * m + t];
    }
    *n = live;
    return SALEC_OK;
}

int salec_gpu_check(salec_gpu *h, long long *n_bad)
{
    if (!h) return fail(SALEC_ERR_ARG, "null handle");
    unsigned long long *cnt = &h->scal->nan_count;
    CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), h->stream));
    const char *names[] = {"v_vel", "v_acc", "v_dis", "e_vel", "e_ste", "e_dvel", "e_pre", "e_den", "e_csd",
                           "m_vof", "m_den", "m_eng"};
    for (const char *nm : names) {
        int fid = field_by_name(nm);
        const long long n = (long long)field_ncomp(h, fid) * h->d.PL;
        launch_count_nonfinite(field_ptr(h, fid), field_f32(h, fid), n, cnt, h->stream);
    }
    CUDA_TRY(cudaGetLastError());
    unsigned long long bad = 0;
    CUDA_TRY(cudaMemcpyAsync(&h->scal_host->nan_count, cnt, sizeof(bad), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    bad = h->scal_host->nan_count;
    if (n_bad) *n_bad = (long long)bad;
    return bad ? fail(SALEC_ERR_NUMERIC, std::to_string(bad) + " non-finite values") : SALEC_OK;
}

} // extern "C"

// ================================================================== adjoint of a window of cycles
// The reverse sweeps live in salec_adjoint.cu; this part keeps their buffers, replays the forward
// cycles with an undo log, and runs the sweeps in reverse order.
struct AdjointState {
    char *pool = nullptr;          // adjoint planes, laid out as the field pool
    Fields b{};
    double *theta = nullptr;       // d/d Yint0, Yfricint, Ydam0, Yfricdam of material 1
    double *gscratch = nullptr;    // reverse-gather scratch
    double *cscr = nullptr;        // per-cell corner scratch of the reverse sweeps (16 planes)
    size_t gscratch_doubles = 0;
    char *tmp = nullptr;           // forward fields of a phase kept while it is reversed
    size_t tmp_bytes = 0;
    char *ckpt = nullptr;          // checkpoints of the window (segment starts, then the end)
    size_t ckpt_bytes = 0;
    char *undo = nullptr;          // undo logs of one segment's cycles
    size_t undo_bytes = 0;
    double *mis = nullptr;         // misfit: J, column heights, target, weights
    size_t mis_doubles = 0;
    struct ListCopy {
        CopySeg *dev = nullptr;
        int n = 0;
        unsigned long long max_bytes = 0;
    };
    std::map<std::string, ListCopy> lists;   // device tables of the field lists copied to logs
    long long *slot = nullptr;     // undo-log record of the cycle being replayed or reversed
    cudaGraphExec_t replay = nullptr, reverse = nullptr;   // one replayed / one reversed cycle
    const char *graph_undo = nullptr;   // undo buffer and record size the graphs were captured for
    size_t graph_ub = 0;
};

namespace {

// fields a cycle writes and later cycles or sweeps read (state of a checkpoint); the face
// records and the pure transients are rewritten before they are read
const char *const kAdjSnapshot[] = {"e_ejt", "m_vof", "e_dvel", "e_den", "v_vof", "v_vel", "v_mass", "e_vel",
                                    "e_grad_vel", "e_div_vel", "e_q", "e_ste", "e_ste2s", "e_sta2s", "e_tps", "e_dam",
                                    "e_strength", "e_vib", "e_pre", "v_acc", "v_alpha", "v_dis", "m_eng", "e_cvs",
                                    "m_pty", "e_wpt", "m_den", "e_cnd", "e_csd", "e_tem", "e_mu", "e_alpha", "e_beta",
                                    "y_profile"};
// fields each phase writes that a reverse sweep or a recipe of the reverse reads (its undo log),
// face records excepted: every face is rewritten by its donor cell in phase 12 before phase 14
// reads it. Fields the adjoint's configuration leaves unused (porosity, damping auxiliaries,
// vibration, ejecta times, lubrication counts, the surface profile) or that only the forward
// reads (the strength, the plastic strain and its invariant, the vertex damping factor) are not
// logged: the checkpoints carry them for the replays
const std::vector<const char *> kAdjWrites[16] = {
    {},
    {"m_vof", "e_dvel", "e_den", "v_vof", "v_vel", "v_mass"},
    {},
    {"e_vel"},
    {"v_vel"},
    {"e_grad_vel", "e_div_vel", "e_q"},
    {},
    {"e_ste", "e_ste2s", "e_dam"},
    {"e_pre", "e_ste", "e_q", "v_acc"},
    {"v_dis", "v_vel"},
    {"m_eng"},
    {},
    {"e_wpt", "m_den", "m_eng"},
    {},
    {"m_vof", "m_den", "m_eng", "e_dvel", "e_ste", "e_dam", "e_den", "e_pre", "e_csd", "e_tem", "e_mu"},
    {},
};


size_t field_bytes(const salec_gpu *h, int k)
{
    const size_t col = (((size_t)h->d.enx + 31) / 32) * 32;
    return kFields[k].loc == L_COL ? col * sizeof(double) : (size_t)field_ncomp(h, k) * h->d.PL * field_elem(h, k);
}

template <class List>
size_t list_bytes(const salec_gpu *h, const List &names)
{
    size_t b = sizeof(Scal);
    for (const char *n : names) b += field_bytes(h, field_by_name(n));
    return (b + 255) & ~(size_t)255;
}

// fields whose ghost cells the reverse recipes fill again (the gathers inside phases 1, 8 and 12
// run before the sweep they feed), kept aside and put back afterwards
const std::vector<const char *> kKeep12 = {"m_den", "e_vib", "m_eng"};
const std::vector<const char *> kKeep8 = {"e_pre", "e_ste", "e_q"};
const std::vector<const char *> kKeep1 = {"m_vof", "e_dvel", "e_den"};

// Device table of a field list: the fields in order, then the scalar block, at the offsets of
// list_bytes' record layout. Built outside stream capture (adjoint_tables builds every list).
const AdjointState::ListCopy *list_table(salec_gpu *h, const std::vector<const char *> &names)
{
    AdjointState *st = h->adj;
    std::string key;
    for (const char *n : names) { key += n; key += ','; }
    auto it = st->lists.find(key);
    if (it != st->lists.end()) return &it->second;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return nullptr;
    std::vector<CopySeg> segs;
    unsigned long long off = 0;
    for (const char *n : names) {
        const int k = field_by_name(n);
        const size_t nb = field_bytes(h, k);
        segs.push_back({reinterpret_cast<char *>(field_ptr(h, k)), off, nb});
        off += nb;
    }
    segs.push_back({reinterpret_cast<char *>(h->scal), off, sizeof(Scal)});
    AdjointState::ListCopy L;
    if (cudaMalloc(reinterpret_cast<void **>(&L.dev), segs.size() * sizeof(CopySeg)) != cudaSuccess) return nullptr;
    if (cudaMemcpy(L.dev, segs.data(), segs.size() * sizeof(CopySeg), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(L.dev);
        return nullptr;
    }
    L.n = (int)segs.size();
    for (const CopySeg &g : segs) L.max_bytes = std::max(L.max_bytes, g.bytes);
    return &(st->lists[key] = L);
}

// device table of explicit segments under a key (built outside stream capture)
const AdjointState::ListCopy *seg_table(salec_gpu *h, const std::string &key, const std::vector<CopySeg> &segs)
{
    AdjointState *st = h->adj;
    auto it = st->lists.find(key);
    if (it != st->lists.end()) return &it->second;
    AdjointState::ListCopy L;
    if (cudaMalloc(reinterpret_cast<void **>(&L.dev), segs.size() * sizeof(CopySeg)) != cudaSuccess) return nullptr;
    if (cudaMemcpy(L.dev, segs.data(), segs.size() * sizeof(CopySeg), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(L.dev);
        return nullptr;
    }
    L.n = (int)segs.size();
    for (const CopySeg &g : segs) L.max_bytes = std::max(L.max_bytes, g.bytes);
    return &(st->lists[key] = L);
}

// copy the listed fields and the scalar block to (save) or from (restore) the record at buf, or,
// with slot, at buf + *slot * stride
int copy_list(salec_gpu *h, const std::vector<const char *> &names, char *buf, bool save, const long long *slot = nullptr,
              size_t stride = 0)
{
    const AdjointState::ListCopy *L = list_table(h, names);
    if (!L) return fail(SALEC_ERR_CUDA, "adjoint: list table unavailable");
    launch_list_copy(L->dev, L->n, L->max_bytes, buf, slot, stride, save, h->stream);
    CUDA_TRY(cudaGetLastError());
    return SALEC_OK;
}

void adjoint_drop_graphs(salec_gpu *h)
{
    AdjointState *st = h->adj;
    if (!st) return;
    if (st->replay) cudaGraphExecDestroy(st->replay);
    if (st->reverse) cudaGraphExecDestroy(st->reverse);
    st->replay = st->reverse = nullptr;
    st->graph_undo = nullptr;
}

void adjoint_release(salec_gpu *h)
{
    AdjointState *st = h->adj;
    if (!st) return;
    adjoint_drop_graphs(h);
    for (auto &kv : st->lists) cudaFree(kv.second.dev);
    cudaFree(st->slot);
    cudaFree(st->pool);
    cudaFree(st->theta);
    cudaFree(st->gscratch);
    cudaFree(st->cscr);
    cudaFree(st->tmp);
    cudaFree(st->ckpt);
    cudaFree(st->undo);
    cudaFree(st->mis);
    delete st;
    h->adj = nullptr;
}

const char *adjoint_unsupported(const salec_gpu *h, const DevMat &m1)
{
    if (h->mixed) return "the adjoint runs on the plain FP64 form";
    if (h->d.nmat != 2) return "the adjoint supports one material beside vacuum";
    if (h->rp.damp_type != 5) return "the adjoint supports damping = none";
    if (h->rp.porosity_model || h->rp.acoustic_fluid || h->rp.tensile_failure || h->rp.tracer_lubrication > 0)
        return "the adjoint supports no porosity, acoustic fluidisation, tensile failure or tracer lubrication";
    if (h->rp.flow_resistance > 0. || h->rp.flow_friction > 0.) return "the adjoint supports no ejecta drag";
    if (h->rp.partpres) return "the adjoint supports partpres = 0";
    if (m1.eos_type != SALEC_EOS_TILLOTSON) return "the adjoint supports a Tillotson material";
    if (m1.yfunc != SALEC_FN_ROCK_STRENGTH_T) return "the adjoint supports the RockStrengthT yield model";
    if (m1.dsdf != SALEC_FN_IVANOV && m1.dsdf != SALEC_FN_SIMPLE_SHEAR) return "the adjoint supports Ivanov damage";
    if (m1.PolyLiq > 0 || m1.PolySol > 0) return "the adjoint supports the Simon melting curve only";
    return nullptr;
}

int adjoint_ensure(salec_gpu *h)
{
    if (!h->adj) h->adj = new AdjointState();
    AdjointState *st = h->adj;
    if (!st->pool) {
        CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&st->pool), h->pool_bytes));
        CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&st->theta), 4 * sizeof(double)));
        for (int k = 0; k < kNumFields; ++k) {
            const size_t off = reinterpret_cast<char *>(field_ptr(h, k)) - h->pool;
            *reinterpret_cast<double **>(reinterpret_cast<char *>(&st->b) + kFields[k].off) =
                reinterpret_cast<double *>(st->pool + off);
        }
        size_t gs = 0;
        for (const Gather *g : {&h->g_mvof, &h->g_dvel_den, &h->g_evel, &h->g_pre_ste_q, &h->g_flux_state, &h->r_vel,
                                &h->r_acc, &h->r_dis}) {
            size_t e = 0;
            for (int f = 0; f < g->batch.nfield; ++f) e += g->entries[f];
            gs = std::max(gs, e * (size_t)std::max(g->ncomp_max, 1));
        }
        st->gscratch_doubles = std::max<size_t>(gs, 1);
        CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&st->gscratch), st->gscratch_doubles * sizeof(double)));
        size_t tb = 0;
        for (int p = 0; p < 16; ++p) tb = std::max(tb, list_bytes(h, kAdjWrites[p]));
        for (const auto *l : {&kKeep12, &kKeep8, &kKeep1}) tb = std::max(tb, list_bytes(h, *l));
        st->tmp_bytes = tb;
        CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&st->tmp), tb));
        CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&st->slot), sizeof(long long)));
        CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&st->cscr), 16 * (size_t)h->d.PL * sizeof(double)));
        // every list table, so that the graphs can be captured
        const std::vector<const char *> snap(std::begin(kAdjSnapshot), std::end(kAdjSnapshot));
        std::vector<const std::vector<const char *> *> all = {&snap, &kKeep12, &kKeep8, &kKeep1};
        for (int p = 0; p < 16; ++p) all.push_back(&kAdjWrites[p]);
        for (const auto *l : all)
            if (!list_table(h, *l)) return fail(SALEC_ERR_CUDA, "adjoint: list table");
    }
    return SALEC_OK;
}

int adjoint_zero(salec_gpu *h)
{
    CUDA_TRY(cudaMemsetAsync(h->adj->pool, 0, h->pool_bytes, h->stream));
    CUDA_TRY(cudaMemsetAsync(h->adj->theta, 0, 4 * sizeof(double), h->stream));
    return SALEC_OK;
}

int adjoint_gather(salec_gpu *h, const Gather &g)
{
    if (g.batch.total == 0) return SALEC_OK;
    const void *adj[SALEC_MAX_GATHER_FIELDS];
    for (int f = 0; f < g.batch.nfield; ++f)
        adj[f] = h->adj->pool + (static_cast<char *>(g.batch.field[f].base) - h->pool);
    launch_adjoint_gather(g.batch, g.entries, adj, h->adj->gscratch, g.two_pass, h->stream);
    CUDA_TRY(cudaGetLastError());
    return SALEC_OK;
}

// Reverse of phase p with the current field pool as the state before phase p (left so on return).
int adjoint_phase(salec_gpu *h, int p)
{
    AdjointState *st = h->adj;
    AdjCtx a;
    a.c = h->ctx();
    a.b = st->b;
    a.theta = st->theta;
    a.scr = st->cscr;
    cudaStream_t s = h->stream;
    auto keep = [&](const std::vector<const char *> &names, bool save) { return copy_list(h, names, st->tmp, save); };
    int rc = SALEC_OK;
    switch (p) {
    case 14: launch_adjoint_kernel(AK_REMAP_STATE, a, s); break;
    case 12:
        if ((rc = keep(kKeep12, true))) return rc;
        if ((rc = run_gather(h, h->g_flux_state))) return rc;
        launch_adjoint_kernel(AK_FLUX, a, s);
        if ((rc = keep(kKeep12, false))) return rc;
        if ((rc = adjoint_gather(h, h->g_flux_state))) return rc;
        break;
    case 10: launch_adjoint_kernel(AK_ENERGY, a, s); break;
    // The reverse of a gather needs the forward values only for the ops whose derivative depends
    // on them (|x|, in the velocity-increment ghosts of phase 1, whose sources are interior and
    // unchanged by the gather); the restrictions and the other ghost patterns copy, negate or
    // zero. So no recipe re-runs a sweep to obtain the values a later gather reads.
    case 9:
        if ((rc = adjoint_gather(h, h->r_dis))) return rc;
        launch_adjoint_kernel(AK_DISPLACEMENT, a, s);
        break;
    case 8:
        if ((rc = keep(kKeep8, true))) return rc;
        if ((rc = run_gather(h, h->g_pre_ste_q))) return rc;
        if ((rc = adjoint_gather(h, h->r_acc))) return rc;
        launch_adjoint_kernel(AK_ACCELERATION, a, s);
        if ((rc = keep(kKeep8, false))) return rc;
        if ((rc = adjoint_gather(h, h->g_pre_ste_q))) return rc;
        break;
    case 7: launch_adjoint_kernel(AK_STRESS, a, s); break;
    case 5: launch_adjoint_kernel(AK_GRADIENT, a, s); break;
    case 4: launch_adjoint_kernel(AK_VOID_VERTICES, a, s); break;
    case 3:
        if ((rc = adjoint_gather(h, h->g_evel))) return rc;
        launch_adjoint_kernel(AK_CELL_VELOCITY, a, s);
        break;
    case 1: {
        // the sweep reads the cell fields' ghosts as the gathers fill them
        if ((rc = keep(kKeep1, true))) return rc;
        if ((rc = run_gather(h, h->g_mvof))) return rc;
        if ((rc = run_gather(h, h->g_dvel_den))) return rc;
        if ((rc = adjoint_gather(h, h->r_vel))) return rc;
        launch_adjoint_kernel(AK_VERTEX_MOMENTUM, a, s);
        if ((rc = keep(kKeep1, false))) return rc;
        if ((rc = adjoint_gather(h, h->g_dvel_den))) return rc;
        if ((rc = adjoint_gather(h, h->g_mvof))) return rc;
        break;
    }
    default: break;   // phases 0, 2, 6, 11, 13 and 15 write nothing an adjoint flows through
    }
    CUDA_TRY(cudaGetLastError());
    return SALEC_OK;
}

int adjoint_transfer(salec_gpu *h, int fid, double *host, long long n, bool to_device)
{
    double *&slot = field_ptr(h, fid);
    double *saved = slot;
    slot = reinterpret_cast<double *>(h->adj->pool + (reinterpret_cast<char *>(saved) - h->pool));
    int rc = SALEC_OK;
    // the conversion only; the geometry tables and the Laplacian mask of the forward fields stay
    int nx, ny;
    field_points(h, fid, nx, ny);
    const int nc = field_ncomp(h, fid);
    const long long need = (long long)nx * ny * nc;
    if (n != need) rc = fail(SALEC_ERR_ARG, std::string("adjoint field ") + kFields[fid].name + ": expected " +
                                                 std::to_string(need) + " doubles");
    else if ((rc = ensure_staging(h, (size_t)need)) == SALEC_OK) {
        const long long plane = kFields[fid].loc == L_COL ? 0 : h->d.PL;
        cudaError_t e;
        if (to_device) {
            e = cudaMemcpyAsync(h->staging, host, need * sizeof(double), cudaMemcpyHostToDevice, h->stream);
            if (e == cudaSuccess) launch_aos_to_planes(h->staging, slot, false, plane, h->d.P, nx, ny, nc, h->stream);
        } else {
            launch_planes_to_aos(slot, false, h->staging, plane, h->d.P, nx, ny, nc, h->stream);
            e = cudaMemcpyAsync(host, h->staging, need * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) rc = fail(SALEC_ERR_CUDA, std::string("adjoint transfer: ") + cudaGetErrorString(e));
    }
    slot = saved;
    return rc;
}

// Capture `body` on the handle's stream into an executable graph.
int capture_graph(salec_gpu *h, const std::function<int()> &body, cudaGraphExec_t *exec)
{
    const long long before = h->launches;
    CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = body();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->launches = before;
    if (rc != SALEC_OK || e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc != SALEC_OK ? rc : fail(SALEC_ERR_CUDA, std::string("adjoint graph capture: ") + cudaGetErrorString(e));
    }
    const cudaError_t ei = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) return fail(SALEC_ERR_CUDA, std::string("adjoint graph: ") + cudaGetErrorString(ei));
    return SALEC_OK;
}

// The two graphs of the window: one cycle replayed with its undo log written to record *slot,
// and one cycle reversed from record *slot; each moves *slot on by one. The face flux records
// that the reverse of phase 14 reads are not logged: phase 12 is run again on the state before
// phase 14, which holds phase 12's inputs unchanged (phase 13 writes only lubrication counts,
// which the adjoint's configuration leaves off), and rewrites the same records.
int adjoint_graphs(salec_gpu *h, size_t ub, const std::vector<size_t> &uoff)
{
    AdjointState *st = h->adj;
    if (st->replay && st->reverse && st->graph_undo == st->undo && st->graph_ub == ub) return SALEC_OK;
    adjoint_drop_graphs(h);
    cudaStream_t s = h->stream;
    // The undo log of phase p holds its fields and the scalars as they were before phase p. A
    // field keeps that value from its previous writer in the cycle (or the cycle's start) up to
    // phase p, so it is saved right after that writer; the scalars change in phases 5 (CFL
    // candidates), 6 (dt) and 15. The saves of a cycle so fall into a few groups, one copy each.
    std::vector<std::vector<CopySeg>> groups(17);   // groups[q + 1]: saved after phase q
    for (int p = 0; p < 16; ++p) {
        if (kAdjWrites[p].empty()) continue;
        unsigned long long off = uoff[p];
        for (const char *n : kAdjWrites[p]) {
            int q = -1;
            for (int r = p - 1; r >= 0 && q < 0; --r)
                for (const char *m : kAdjWrites[r])
                    if (!strcmp(m, n)) { q = r; break; }
            const int k = field_by_name(n);
            const size_t nb = field_bytes(h, k);
            groups[q + 1].push_back({reinterpret_cast<char *>(field_ptr(h, k)), off, nb});
            off += nb;
        }
        const int qs = p > 6 ? 6 : (p > 5 ? 5 : -1);
        groups[qs + 1].push_back({reinterpret_cast<char *>(h->scal), off, sizeof(Scal)});
    }
    std::vector<const AdjointState::ListCopy *> gtab(17, nullptr);
    for (int g = 0; g < 17; ++g)
        if (!groups[g].empty() &&
            !(gtab[g] = seg_table(h, "save group " + std::to_string(g) + " of " + std::to_string(ub), groups[g])))
            return fail(SALEC_ERR_CUDA, "adjoint: save table");
    int rc = capture_graph(h, [&]() -> int {
        for (int p = 0; p <= 15; ++p) {
            if (const AdjointState::ListCopy *L = gtab[p]) {
                launch_list_copy(L->dev, L->n, L->max_bytes, st->undo, st->slot, ub, true, s);
                CUDA_TRY(cudaGetLastError());
            }
            // the cycle graph's form: the energy update inside phase 7. The logs are the same:
            // m_eng is saved at the cycle's start for phase 10 and after phase 10 for phase 12,
            // and phases 8 and 9 leave it alone
            if (int r = run_phase(h, p, true)) return r;
        }
        launch_slot_add(st->slot, 1, s);
        return SALEC_OK;
    }, &st->replay);
    if (rc) return rc;
    rc = capture_graph(h, [&]() -> int {
        for (int p = 15; p >= 0; --p) {
            // a phase without a log changes neither a logged field nor (phases 0, 2, 11, 13) the
            // scalars; the scalars phases 6 and 15 change are set back by the next log restored
            if (!kAdjWrites[p].empty())
                if (int r = copy_list(h, kAdjWrites[p], st->undo + uoff[p], false, st->slot, ub)) return r;
            if (p == 14)
                if (int r = run_phase(h, 12)) return r;
            if (int r = adjoint_phase(h, p)) return r;
        }
        launch_slot_add(st->slot, -1, s);
        return SALEC_OK;
    }, &st->reverse);
    if (rc) {
        adjoint_drop_graphs(h);
        return rc;
    }
    st->graph_undo = st->undo;
    st->graph_ub = ub;
    return SALEC_OK;
}

int adjoint_check(salec_gpu *h)
{
    DevMat m1;
    if (cudaMemcpy(&m1, h->mat + 1, sizeof(DevMat), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(SALEC_ERR_CUDA, "material read-back");
    if (const char *why = adjoint_unsupported(h, m1)) return fail(SALEC_ERR_UNSUPPORTED, why);
    return adjoint_ensure(h);
}

} // namespace

extern "C" {

int salec_gpu_set_dt_schedule(salec_gpu *h, const double *dts, int n)
{
    if (!h || n < 0 || (n > 0 && !dts)) return fail(SALEC_ERR_ARG, "bad argument");
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (h->dt_sched) CUDA_TRY(cudaFree(h->dt_sched));
    h->dt_sched = nullptr;
    h->dt_sched_n = 0;
    if (n > 0) {
        CUDA_TRY(cudaMemcpy(&h->scal_host->i_step, &h->scal->i_step, sizeof(long long), cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&h->dt_sched), n * sizeof(double)));
        CUDA_TRY(cudaMemcpy(h->dt_sched, dts, n * sizeof(double), cudaMemcpyHostToDevice));
        h->dt_sched_i0 = h->scal_host->i_step;
        h->dt_sched_n = n;
    }
    drop_cycle_graph(h);
    return SALEC_OK;
}

int salec_gpu_adjoint_reset(salec_gpu *h)
{
    if (!h) return fail(SALEC_ERR_ARG, "null handle");
    if (int rc = adjoint_check(h)) return rc;
    if (int rc = adjoint_zero(h)) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SALEC_OK;
}

int salec_gpu_adjoint_set_field(salec_gpu *h, int field, const double *host, long long n)
{
    if (!h || !host || !h->adj || !h->adj->pool) return fail(SALEC_ERR_STATE, "call salec_gpu_adjoint_reset first");
    if (field < 0 || field >= kNumFields) return fail(SALEC_ERR_ARG, "unknown field");
    return adjoint_transfer(h, field, const_cast<double *>(host), n, true);
}

int salec_gpu_adjoint_get_field(salec_gpu *h, int field, double *host, long long n)
{
    if (!h || !host || !h->adj || !h->adj->pool) return fail(SALEC_ERR_STATE, "call salec_gpu_adjoint_reset first");
    if (field < 0 || field >= kNumFields) return fail(SALEC_ERR_ARG, "unknown field");
    return adjoint_transfer(h, field, host, n, false);
}

int salec_gpu_adjoint_phase(salec_gpu *h, int phase)
{
    if (!h || !h->adj || !h->adj->pool) return fail(SALEC_ERR_STATE, "call salec_gpu_adjoint_reset first");
    if (phase < 0 || phase > 15) return fail(SALEC_ERR_ARG, "phase out of range");
    if (int rc = adjoint_phase(h, phase)) return rc;
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SALEC_OK;
}

int salec_gpu_adjoint_params(salec_gpu *h, double *theta)
{
    if (!h || !theta || !h->adj || !h->adj->pool) return fail(SALEC_ERR_STATE, "call salec_gpu_adjoint_reset first");
    CUDA_TRY(cudaMemcpyAsync(theta, h->adj->theta, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return SALEC_OK;
}

int salec_gpu_adjoint_window(salec_gpu *h, int nsteps, int every, const double *target, const double *weight,
                             int ncols, double *grad_density, long long n_density, salec_adjoint_result *out)
{
    if (!h || nsteps < 1 || every < 1 || !target || !out) return fail(SALEC_ERR_ARG, "bad argument");
    if (ncols != h->d.enx - 4) return fail(SALEC_ERR_ARG, "target and weights need one value per interior column");
    if (grad_density && n_density != (long long)h->d.enx * h->d.eny)
        return fail(SALEC_ERR_ARG, "grad_density needs (nx+4)*(ny+4) doubles");
    if (int rc = adjoint_check(h)) return rc;
    AdjointState *st = h->adj;
    cudaStream_t s = h->stream;
    const int nseg = (nsteps + every - 1) / every;
    const std::vector<const char *> snap(std::begin(kAdjSnapshot), std::end(kAdjSnapshot));
    const size_t sb = list_bytes(h, snap);
    size_t ub = 0;
    std::vector<size_t> uoff(16);
    for (int p = 0; p < 16; ++p) { uoff[p] = ub; ub += list_bytes(h, kAdjWrites[p]); }
    // buffers: nseg + 1 checkpoints (the last is the window's end), `every` undo logs
    const size_t need_ck = sb * (nseg + 1), need_ud = ub * every;
    if (st->ckpt_bytes < need_ck) {
        cudaFree(st->ckpt);
        st->ckpt = nullptr;
        st->ckpt_bytes = 0;
        CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&st->ckpt), need_ck));
        st->ckpt_bytes = need_ck;
    }
    if (st->undo_bytes < need_ud) {
        cudaFree(st->undo);
        st->undo = nullptr;
        st->undo_bytes = 0;
        CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&st->undo), need_ud));
        st->undo_bytes = need_ud;
    }
    const size_t md = 1 + 3 * (size_t)ncols;
    if (st->mis_doubles < md) {
        cudaFree(st->mis);
        st->mis = nullptr;
        CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&st->mis), md * sizeof(double)));
        st->mis_doubles = md;
    }
    if (int rc = adjoint_graphs(h, ub, uoff)) return rc;
    // forward window, with a checkpoint at every segment start; the last segment writes its undo
    // logs on the way, so that it is reversed without a replay
    for (int sgm = 0; sgm < nseg; ++sgm) {
        if (int rc = copy_list(h, snap, st->ckpt + sb * sgm, true)) return rc;
        const int n = std::min(every, nsteps - sgm * every);
        if (sgm < nseg - 1) {
            if (int rc = salec_gpu_step(h, n)) return rc;
        } else {
            launch_slot_set(st->slot, 0, s);
            for (int k = 0; k < n; ++k) CUDA_TRY(cudaGraphLaunch(st->replay, s));
        }
    }
    if (int rc = copy_list(h, snap, st->ckpt + sb * nseg, true)) return rc;
    // the tracers are not part of the differentiated state: the replays move them, so the end's
    // are kept and put back
    std::vector<char> tr_end(h->tr_bytes);
    if (h->tr_bytes) {
        CUDA_TRY(cudaStreamSynchronize(s));
        CUDA_TRY(cudaMemcpy(tr_end.data(), h->tr_block, h->tr_bytes, cudaMemcpyDeviceToHost));
    }
    // misfit of the final surface profile and the seed of the reverse sweep
    if (int rc = adjoint_zero(h)) return rc;
    std::vector<double> w(ncols, 1.0);
    if (weight) w.assign(weight, weight + ncols);
    CUDA_TRY(cudaMemsetAsync(st->mis, 0, sizeof(double), s));
    CUDA_TRY(cudaMemcpyAsync(st->mis + 1 + ncols, target, ncols * sizeof(double), cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(st->mis + 1 + 2 * ncols, w.data(), ncols * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_profile_misfit(h->ctx(), st->b, st->mis + 1 + ncols, st->mis + 1 + 2 * ncols, st->mis, st->mis + 1, s);
    CUDA_TRY(cudaGetLastError());
    double J = 0.;
    CUDA_TRY(cudaMemcpyAsync(&J, st->mis, sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    // reverse: per segment, replay its cycles from the checkpoint with undo logs, then walk back
    for (int sgm = nseg - 1; sgm >= 0; --sgm) {
        const int n = std::min(every, nsteps - sgm * every);
        if (sgm < nseg - 1) {
            if (int rc = copy_list(h, snap, st->ckpt + sb * sgm, false)) return rc;
            launch_slot_set(st->slot, 0, s);
            for (int k = 0; k < n; ++k) CUDA_TRY(cudaGraphLaunch(st->replay, s));
        }
        launch_slot_set(st->slot, n - 1, s);
        for (int k = 0; k < n; ++k) CUDA_TRY(cudaGraphLaunch(st->reverse, s));
    }
    // the pool now holds the window's start and the adjoint planes its sensitivities
    out->misfit = J;
    CUDA_TRY(cudaMemcpyAsync(out->d_params, st->theta, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    {
        const int fv = field_by_name("v_vel");
        int nx, ny;
        field_points(h, fv, nx, ny);
        const long long nv = (long long)nx * ny * 2;
        std::vector<double> v(nv), bv(nv);
        if (int rc = transfer(h, fv, v.data(), nv, false)) return rc;
        if (int rc = adjoint_transfer(h, fv, bv.data(), nv, false)) return rc;
        double sv = 0.;
        for (long long q = 0; q < nv; ++q) sv += bv[q] * v[q];
        out->d_velocity_scale = sv;
    }
    if (grad_density) {
        const int fm = field_by_name("m_den"), fe = field_by_name("e_den");
        const long long nc = (long long)h->d.enx * h->d.eny;
        std::vector<double> md2(nc * 2), bm(nc * 2), ed(nc), be(nc);
        if (int rc = transfer(h, fm, md2.data(), nc * 2, false)) return rc;
        if (int rc = adjoint_transfer(h, fm, bm.data(), nc * 2, false)) return rc;
        if (int rc = transfer(h, fe, ed.data(), nc, false)) return rc;
        if (int rc = adjoint_transfer(h, fe, be.data(), nc, false)) return rc;
        for (long long q = 0; q < nc; ++q) {
            const double g = bm[2 * q] * md2[2 * q] + bm[2 * q + 1] * md2[2 * q + 1] + be[q] * ed[q];
            grad_density[q] = ed[q] > 0.0 ? g / ed[q] : 0.0;
        }
    }
    // leave the simulation at the end of the window
    if (int rc = copy_list(h, snap, st->ckpt + sb * nseg, false)) return rc;
    if (h->tr_bytes) CUDA_TRY(cudaMemcpy(h->tr_block, tr_end.data(), h->tr_bytes, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaStreamSynchronize(s));
    return SALEC_OK;
}

} // extern "C"
