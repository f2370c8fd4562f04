/*
 * Oracle driver for the compiled reference SALEc2d (TEST INFRASTRUCTURE ONLY).
 *
 * This file is linked with the unmodified reference sources (built in place from the
 * reference tree by oracle/Makefile, output in oracle/_ref/) and the one-rank MPI shim.
 * It re-runs the reference's own initialisation sequence and per-step loop body from
 * src/salec2d.c:45-105 and :115-272, split into numbered phases so that a test can stop
 * between any two sweeps and compare the state with the GPU path. It never runs inside the
 * product: only tests/, __graft_entry__.smoke() and bench.py's CPU legs load it.
 *
 * Phases of one step (reference line numbers in src/salec2d.c):
 *   0  trace_profile + column MIN of y_profile                       :118-121
 *   1  update_v_vof (internal), ghost m_vof, update_v_vof (update)   :127-139
 *   2  update_v_vel_inc (both halves around the e_dvel/e_den ghosts),
 *      vertex restriction of v_vel                                   :135,147-151
 *   3  update_e_vel + ghost e_vel                                    :154-157
 *   4  check_v_vel                                                   :158
 *   5  update_e_gradvel (+ artificial viscosity)                     :162-163
 *   6  calculate_dt + MIN all-reduce                                 :167-168
 *   7  block_vibration + update_e_stress                             :174-179
 *   8  calculate_acc (both halves around the e_pre/e_ste/e_q ghosts),
 *      vertex restriction of v_acc                                   :186-191
 *   9  calculate_v_dis + restriction of v_dis                        :194-199
 *  10  update_energy                                                 :200-203
 *  11  tracer update                                                 :209-214
 *  12  clean_flux, calculate_flux (cells), ghosts, calculate_flux (pad) :220-235
 *  13  update_strength_condition                                     :238-239
 *  14  advect_flux, damp_on_cell, ejecta_flow, update_state          :254-259
 *  15  update_cycle_control + v_vel sync                             :264-271
 * The output point (:241-245) sits between phases 13 and 14 and is exposed separately.
 */
#include "sale2d.h"
#include "strength.h"
#include "ejecta.h"
#include "target_profile.h"
#include "write_vtk.h"

#include <errno.h>
#include <sys/stat.h>

#define ORACLE_NPHASE 16

static sale2d_var g_sale;
static mesh2d_info g_minfo;
static cycle_control g_ccl;
static InputFile *g_ifp = NULL;
static int g_stage = 0; /* 0 none, 1 begun, 2 material set, 3 ready */

static void ensure_dir(const char *path)
{
    if (mkdir(path, 0755) != 0 && errno != EEXIST) fprintf(stderr, "oracle: cannot create %s\n", path);
}

/* Mirror of src/salec2d.c:45-58 (deck, cycle control, mesh info, EOS, fields, ghosts, geometry). */
int ref_init_begin(const char *deck, const char *eosdir, const char *workdir)
{
    static int mpi_up = 0;
    if (!mpi_up) { MPI_Init(NULL, NULL); mpi_up = 1; }
    if (workdir && workdir[0]) {
        ensure_dir(workdir);
        if (chdir(workdir) != 0) return -1;
    }
    ensure_dir("./vts"); ensure_dir("./vtp"); ensure_dir("./txt"); ensure_dir("./post");

    memset(&g_sale, 0, sizeof(g_sale));
    memset(&g_minfo, 0, sizeof(g_minfo));
    memset(&g_ccl, 0, sizeof(g_ccl));

    g_ifp = OpenInputFile(deck);
    init_cycle_control(g_ifp, &g_ccl);
    load_mesh_info(g_ifp, &g_minfo, eosdir);
    init_sale_mat(&g_sale, &g_minfo);
    select_strength_model(&g_sale);
    init_sale2d_var(&g_sale, &g_minfo);
    /*
     * The reference allocates every field with malloc (src/mpi_vec/mpi_vec.c:680-683, :763, :797)
     * and never writes many points (outer vertex ring, m_den/m_eng of vacuum cells, e_ejt below
     * the ejecta threshold, ...). On the meshes it is run on, those blocks come from fresh zeroed
     * pages; on small test meshes malloc reuses dirty heap memory. Zero every field here so that
     * small meshes see the same all-zero start as large ones (the fields are contiguous,
     * src/sale2d.c:218-219, as clean_sale_var also assumes at :420-426).
     */
    for (int k = 0; k < g_sale.fv_counter; ++k) {
        field_var *fv = g_sale.v_vel + k;
        if (fv->data) memset(fv->data, 0, (size_t)fv->data_size * fv->bytes_per_unit);
    }
    /*
     * A material without a porosity model (material.Porosity = None) never gets
     * state_reference.alphamax2 (src/sale2d_back.c:369-395 sets it for Wunnemann only), yet a
     * run with any porous material clamps the distension of every material to [1, alphamax2]
     * (src/advect.c:272-277, src/sale2d.c:700-706). The clamp then reads heap garbage: a value
     * >= 1 leaves the distension at 1, anything else writes the garbage into m_pty (and a NaN
     * density later faults in TillTemp, src/eos/eos_state.c:521-524). Pin it to 1, the value
     * that keeps a non-porous material at distension 1; the library's initialiser does the same.
     */
    for (int m = 1; m < g_sale.nmat; ++m) {
        state_reference *r = g_sale.etb[m].ref;
        if (r && strcasecmp(r->porosityfunc, "None") == 0) r->alphamax2 = 1.0;
    }
    init_sale2d_other(&g_sale, g_ifp);
    init_sale2d_ghost(&g_sale, &g_minfo);
    CloseInputFile(g_ifp);
    g_ifp = NULL;
    init_mesh_pos(&g_sale, &g_minfo);
    g_stage = 1;
    return 0;
}

/* src/salec2d.c:74 */
int ref_init_material(void)
{
    if (g_stage != 1) return -1;
    init_material_distribution(&g_minfo, &g_sale);
    g_stage = 2;
    return 0;
}

/*
 * The reference builds every tracer from a stack variable whose peak pressure and temperature
 * (mpre, mtem) it never sets (fl_data tmp_data, src/tracer.c:405-445): they start at whatever
 * the stack held, and every peak recorded later is a MAX with that value, so two processes
 * differ. Both start at 0 here, as the library's deck initialiser starts them.
 */
static void pin_tracer_peaks(sale2d_var *s)
{
    field_list_iterator it;
    field_list_node *node;
    fl_iterator_init(&it, s->tracer_list, field_list_head);
    while ((node = fl_iterator_next(&it)) != NULL) {
        node->data.mpre = 0.0f;
        node->data.mtem = 0.0f;
    }
}

/* Mirror of src/salec2d.c:76-105: first EOS call, ghost fills, PML reference state, vertex velocity, tracers. */
int ref_init_finish(void)
{
    if (g_stage != 2) return -1;
    update_state(&g_sale, internal_section | send_section);
    sync_start(g_sale.e_den);
    sync_complete(g_sale.e_den);
    flush_ght(g_sale.e_pre);
    flush_ght(g_sale.e_ste);
    flush_ght(g_sale.m_eng);
    flush_ght(g_sale.m_pty);
    flush_ght(g_sale.e_cvs);

    double local_damp_time = record_avg_value(&g_sale);
    MPI_Allreduce(&local_damp_time, &(g_minfo.damp_t), 1, MPI_DOUBLE, MPI_MAX, g_sale.e_pre->comm);
    g_minfo.damp_t *= 2.0;
    g_sale.damp_time = Max(g_minfo.damp_t, g_sale.damp_time);

    init_v_field(&g_sale);
    clean_fv(g_sale.e_vel);
    clean_fv(g_sale.e_ste);
    clean_fv(g_sale.e_dvel);

    g_ccl.out_vts = 1;
    g_ccl.k_out_step = 1;
    init_sale2d_tracer(&g_sale, &g_minfo);
    pin_tracer_peaks(&g_sale);
    export_init_tracers(&g_sale, &g_minfo);
    g_stage = 3;
    return 0;
}

/*
 * Adopt a complete initial state set by the caller (every field through ref_set_field after
 * ref_init_begin) instead of running the reference's material set-up: records the damping
 * time, builds the tracer list from the adopted fields (init_sale2d_tracer,
 * src/sale2d.c:2081-2091) and makes the step loop available. Used to time the reference's
 * step on exactly the state another implementation starts from.
 */
int ref_init_adopt(double damp_time)
{
    if (g_stage != 1) return -1;
    g_sale.damp_time = damp_time;
    g_ccl.out_vts = 1;
    g_ccl.k_out_step = 1;
    init_sale2d_tracer(&g_sale, &g_minfo);
    pin_tracer_peaks(&g_sale);
    g_stage = 3;
    return 0;
}

int ref_init(const char *deck, const char *eosdir, const char *workdir)
{
    int rc = ref_init_begin(deck, eosdir, workdir);
    if (rc) return rc;
    rc = ref_init_material();
    if (rc) return rc;
    return ref_init_finish();
}

int ref_phase(int p)
{
    sale2d_var *s = &g_sale;
    cycle_control *c = &g_ccl;
    if (g_stage != 3) return -1;
    switch (p) {
    case 0:
        trace_profile(s);
        sync_index_start(s->y_profile, MPI_MIN);
        sync_start(s->e_ejt);
        break;
    case 1:
        sync_start(s->m_vof); sync_start(s->m_den); sync_start(s->e_dvel);
        sync_start(s->e_den); sync_start(s->e_wpt); sync_start(s->e_pre);
        update_v_vof(s, internal_section);
        update_v_vel_inc(s, internal_section);
        sync_complete(s->m_vof);
        update_v_vof(s, update_section);
        break;
    case 2:
        sync_complete(s->e_dvel);
        sync_complete(s->e_den);
        sync_complete(s->e_wpt);
        update_v_vel_inc(s, update_section);
        sync_restrict_vertexes(s->v_vel);
        break;
    case 3:
        update_e_vel(s, send_section);
        sync_start(s->e_vel);
        update_e_vel(s, internal_section);
        sync_complete(s->e_vel);
        break;
    case 4:
        check_v_vel(s, update_section | internal_section);
        break;
    case 5:
        update_e_gradvel(s, internal_section | send_section);
        sync_start(s->e_q);
        break;
    case 6:
        c->local_dt = Min(c->max_dt, calculate_dt(s, c->dt));
        MPI_Allreduce(&(c->local_dt), &(c->dt), 1, MPI_DOUBLE, MPI_MIN, s->e_pre->comm);
        break;
    case 7:
        block_vibration(s, internal_section | send_section, c->dt, c->step_time);
        update_e_stress(s, internal_section | send_section, c->dt);
        sync_start(s->e_tps); sync_start(s->e_dam); sync_start(s->e_vib); sync_start(s->e_ste);
        break;
    case 8:
        calculate_acc(g_minfo.damp_type, s, internal_section, c->dt);
        sync_complete(s->e_pre);
        sync_complete(s->e_ste);
        sync_complete(s->e_q);
        calculate_acc(g_minfo.damp_type, s, update_section, c->dt);
        sync_restrict_vertexes(s->v_acc);
        break;
    case 9:
        calculate_v_dis(s, update_section | internal_section, c->dt);
        sync_start(s->v_vel);
        sync_restrict_vertexes(s->v_dis);
        break;
    case 10:
        update_energy(s, internal_section | send_section, c->dt);
        sync_start(s->m_eng);
        if (s->porosity_model) sync_start(s->m_pty);
        if (s->porosity_model) sync_start(s->e_cvs);
        break;
    case 11:
        fl_tracer_update(s->tracer_list, c->dt);
        fl_sync_info_start(s->tracer_list);
        fl_sync_info_complete(s->tracer_list);
        fl_sync_node_start(s->tracer_list);
        break;
    case 12:
        clean_flux(s);
        calculate_flux(s, internal_section | send_section);
        sync_complete(s->m_den);
        sync_complete(s->e_tps);
        sync_complete(s->e_dam);
        sync_complete(s->e_vib);
        sync_complete(s->m_eng);
        if (s->porosity_model) sync_complete(s->m_pty);
        if (s->porosity_model) sync_complete(s->e_cvs);
        sync_complete(s->e_ejt);
        sync_index_complete(s->y_profile);
        calculate_flux(s, receive_section);
        break;
    case 13:
        fl_sync_node_complete(s->tracer_list);
        update_strength_condition(s);
        break;
    case 14:
        advect_flux(g_minfo.damp_type, s, internal_section | send_section, c->dt);
        damp_on_cell(g_minfo.damp_type, s, c->dt, c->step_time);
        ejecta_flow(s, internal_section | send_section, c->dt);
        update_state(s, internal_section | send_section);
        break;
    case 15:
        update_cycle_control(c, stdout);
        sync_complete(s->v_vel);
        break;
    default:
        return -2;
    }
    return 0;
}

int ref_phases(int first, int last)
{
    for (int p = first; p <= last; ++p) {
        int rc = ref_phase(p);
        if (rc) return rc;
    }
    return 0;
}

/* One full loop iteration without the output point. */
int ref_step(void) { return ref_phases(0, ORACLE_NPHASE - 1); }

int ref_run(int nsteps)
{
    for (int k = 0; k < nsteps; ++k) {
        int rc = ref_step();
        if (rc) return rc;
    }
    return 0;
}

/* Output point of src/salec2d.c:241-245 with the reference's own VTS/VTP writers. */
int ref_write_output(void)
{
    if (g_stage != 3) return -1;
    sale2d_write_vtk(&g_sale, &g_minfo, &g_ccl);
    sale2d_write_vtp(&g_sale, &g_minfo, &g_ccl);
    return 0;
}

/* ----------------------------------------------------------------- field access */

static field_var *field_by_name(const char *n)
{
    sale2d_var *s = &g_sale;
    struct { const char *name; field_var *fv; } tab[] = {
        {"v_vel", s->v_vel}, {"v_bf", s->v_bf}, {"v_acc", s->v_acc}, {"e_vel", s->e_vel},
        {"v_dis", s->v_dis}, {"e_div_vel", s->e_div_vel}, {"e_grad_vel", s->e_grad_vel},
        {"e_ste", s->e_ste}, {"e_mu", s->e_mu}, {"e_dvel", s->e_dvel}, {"e_pre", s->e_pre},
        {"e_tem", s->e_tem}, {"e_den", s->e_den}, {"e_eng", s->e_eng}, {"e_csd", s->e_csd},
        {"e_dam", s->e_dam}, {"e_cvs", s->e_cvs}, {"m_vof", s->m_vof}, {"m_den", s->m_den},
        {"m_eng", s->m_eng}, {"m_pty", s->m_pty}, {"e_wpt", s->e_wpt}, {"v_pos", s->v_pos},
        {"e_pos", s->e_pos}, {"e_vol", s->e_vol}, {"e_suf", s->e_suf}, {"e_grad", s->e_grad},
        {"e_subvol", s->e_subvol}, {"bx_phi", s->bx_phi}, {"by_phi", s->by_phi},
        {"bx_normal", s->bx_normal}, {"by_normal", s->by_normal}, {"v_vof", s->v_vof},
        {"v_mass", s->v_mass}, {"e_q", s->e_q}, {"e_strength", s->e_strength}, {"e_cnd", s->e_cnd},
        {"e_tps", s->e_tps}, {"e_ste2s", s->e_ste2s}, {"e_sta2s", s->e_sta2s}, {"v_vol", s->v_vol},
        {"v_subvol", s->v_subvol}, {"v_laplace", s->v_laplace}, {"v_suf", s->v_suf},
        {"e_alpha", s->e_alpha}, {"e_beta", s->e_beta}, {"e_sigma", s->e_sigma},
        {"v_alpha", s->v_alpha}, {"v_beta", s->v_beta}, {"e_dampref", s->e_dampref},
        {"e_vib", s->e_vib}, {"e_ejt", s->e_ejt}, {"y_profile", s->y_profile},
    };
    for (size_t k = 0; k < sizeof(tab) / sizeof(tab[0]); ++k)
        if (strcmp(tab[k].name, n) == 0) return tab[k].fv;
    return NULL;
}

/* dims[0] = points in x, dims[1] = points in y (1 for y_profile), dims[2] = doubles per point */
int ref_field_dims(const char *name, int *dims)
{
    field_var *fv = field_by_name(name);
    if (!fv || g_stage < 1) return -1;
    if (fv == g_sale.y_profile) {
        dims[0] = (int)fv->data_size; dims[1] = 1;
    } else {
        proc_info_2d *p = (proc_info_2d *)fv->proc_self;
        dims[0] = p->nx; dims[1] = p->ny;
    }
    dims[2] = (int)(fv->bytes_per_unit / sizeof(double));
    return 0;
}

int ref_get_field(const char *name, double *out)
{
    field_var *fv = field_by_name(name);
    if (!fv || g_stage < 1) return -1;
    memcpy(out, fv->data, (size_t)fv->data_size * fv->bytes_per_unit);
    return 0;
}

int ref_set_field(const char *name, const double *in)
{
    field_var *fv = field_by_name(name);
    if (!fv || g_stage < 1) return -1;
    memcpy(fv->data, in, (size_t)fv->data_size * fv->bytes_per_unit);
    return 0;
}

/* The reference's own boundary passes on one field: ghost fill (flush_ght,
 * src/mpi_vec/mpi_vec_ght.c:736-752) or vertex restriction (sync_restrict_vertexes, :723-734). */
int ref_ghost_fill(const char *name)
{
    field_var *fv = field_by_name(name);
    if (!fv || g_stage < 1) return -1;
    flush_ght(fv);
    return 0;
}

int ref_restrict(const char *name)
{
    field_var *fv = field_by_name(name);
    if (!fv || g_stage < 1) return -1;
    sync_restrict_vertexes(fv);
    return 0;
}

/* ----------------------------------------------------------------- scalars */

int ref_get_scalar(const char *n, double *v)
{
    sale2d_var *s = &g_sale;
    mesh2d_info *m = &g_minfo;
    cycle_control *c = &g_ccl;
#define S(name, expr) if (strcmp(n, name) == 0) { *v = (double)(expr); return 0; }
    S("dt", c->dt) S("local_dt", c->local_dt) S("max_dt", c->max_dt) S("time", c->step_time)
    S("i_step", c->i_step) S("max_step", c->max_step) S("end_time", c->end_time)
    S("cycle_continue", c->cycle_continue) S("out_vts", c->out_vts)
    S("nx", m->nx) S("ny", m->ny) S("nmat", s->nmat) S("phi_length", s->phi_length)
    S("avis1", s->avis1) S("avis2", s->avis2) S("anc", s->anc) S("damp_time", s->damp_time)
    S("density_cutoff", s->density_cutoff) S("velocity_max", s->velocity_max)
    S("velocity_min", s->velocity_min) S("acceleration_min", s->acceleration_min)
    S("partpres", s->partpres) S("acoustic_fluid", s->acoustic_fluid)
    S("porosity_model", s->porosity_model) S("tensile_failure", s->tensile_failure)
    S("alpha_damp_x", s->alpha_damp_x) S("alpha_damp_y", s->alpha_damp_y)
    S("threshold_z", s->threshold_z) S("flow_resistance", s->flow_resistance)
    S("flow_friction", s->flow_friction) S("damp_type", m->damp_type)
    S("tracer_lubrication", s->tracer_lubrication) S("tracer_lub_y0", s->tracer_lub_y0)
    S("tracer_lub_frac", s->tracer_lub_frac) S("tracer_lub_gy0", s->tracer_lub_gy0)
    S("tracer_lub_gy1", s->tracer_lub_gy1) S("tracer_strip", m->tracer_strip)
    S("go_left", m->go_list[0]) S("go_right", m->go_list[1])
    S("go_bottom", m->go_list[2]) S("go_top", m->go_list[3])
#undef S
    return -1;
}

int ref_set_scalar(const char *n, double v)
{
    cycle_control *c = &g_ccl;
    if (strcmp(n, "dt") == 0) { c->dt = v; return 0; }
    if (strcmp(n, "time") == 0) { c->step_time = v; return 0; }
    if (strcmp(n, "damp_time") == 0) { g_sale.damp_time = v; return 0; }
    return -1;
}

/* Per-material parameters of the reference's state_reference (src/eos/eos_state.h:43-151). */
int ref_get_material(int matid, const char *n, double *v)
{
    if (matid < 1 || matid >= g_sale.nmat) return -1;
    state_reference *r = g_sale.etb[matid].ref;
#define S(name) if (strcmp(n, #name) == 0) { *v = (double)(r->name); return 0; }
    S(VaporDen) S(MeltDen) S(GaCoef) S(Yint0) S(Yfricint) S(Ylimint) S(Ydam0) S(Yfricdam) S(Ylimdam)
    S(Yten0) S(IvanA) S(IvanB) S(IvanC) S(Pbd) S(Pbp) S(minPint) S(minPdam) S(JCA) S(JCB) S(JCN) S(JCC)
    S(JCM) S(JCTREF) S(JCMaxPlastic) S(JCMinP) S(Asimon) S(Csimon) S(Tmelt0) S(Tfrac) S(Tdelta)
    S(PolyLiq) S(Tlidc1) S(Tlidc2) S(Tlidc3) S(PolySol) S(Tsolc1) S(Tsolc2) S(Tsolc3) S(Toff) S(Cvib)
    S(VibMax) S(Tdamp) S(Pvlim) S(Acvis) S(alpha0) S(alphax) S(epse0) S(chi) S(kappa) S(avel) S(epsec)
    S(epsex) S(alphamax) S(alphamax2) S(alphae) S(gamfrac) S(csd0) S(den0) S(melt_viscosity)
#undef S
    return -1;
}

/* Names of the strength/damage/tensile/porosity functions chosen per material. */
int ref_get_material_str(int matid, const char *n, char *out, int len)
{
    if (matid < 1 || matid >= g_sale.nmat || len <= 0) return -1;
    state_reference *r = g_sale.etb[matid].ref;
    const char *src = NULL;
    if (strcmp(n, "yfunc") == 0) src = r->yfunc;
    else if (strcmp(n, "dSDf") == 0) src = r->dSDf;
    else if (strcmp(n, "tfunc") == 0) src = r->tfunc;
    else if (strcmp(n, "porosityfunc") == 0) src = r->porosityfunc;
    if (!src) return -1;
    snprintf(out, (size_t)len, "%s", src);
    return 0;
}

/* EOS kind per material: 0 ANEOS (T-rho), 1 Tillotson, 2 ANEOS SieDen, 3 unknown. */
int ref_eos_type(int matid)
{
    if (matid < 1 || matid >= g_sale.nmat) return -1;
    return (int)g_sale.etb[matid].type;
}

/* Tillotson constants p[0..11] and the cold-energy curve (src/eos/eos_state.c:463-517). */
int ref_get_tillotson(int matid, double *p, double *xden, double *yeng, int *nden)
{
    if (ref_eos_type(matid) != Tillotson) return -1;
    tillotson_table *t = (tillotson_table *)g_sale.etb[matid].table;
    if (p) {
        p[0] = t->TLRho0; p[1] = t->TLCv; p[2] = t->TLA; p[3] = t->TLB; p[4] = t->TLE0; p[5] = t->TLa;
        p[6] = t->TLb; p[7] = t->TLAlpha; p[8] = t->TLBeta; p[9] = t->TLEiv; p[10] = t->TLEcv;
        p[11] = t->TLTref; p[12] = t->StepDen;
    }
    if (nden) *nden = t->nDen;
    if (xden) memcpy(xden, t->xDen, sizeof(double) * (size_t)t->nDen);
    if (yeng) memcpy(yeng, t->yEng, sizeof(double) * (size_t)t->nDen);
    return 0;
}

/* Tabulated tables (both ANEOS kinds): axes and Data[iT][iD][0..2] flattened as [iT][iD][3]. */
int ref_get_table(int matid, int *ntem, int *nden, double *xtem, double *yden, double *data)
{
    int ty = ref_eos_type(matid);
    if (ty != ANEOS && ty != ANEOSSieDen) return -1;
    aneos_table *t = (aneos_table *)g_sale.etb[matid].table;
    *ntem = t->nTem;
    *nden = t->nDen;
    if (xtem) memcpy(xtem, t->xTem, sizeof(double) * (size_t)t->nTem);
    if (yden) memcpy(yden, t->yDen, sizeof(double) * (size_t)t->nDen);
    if (data)
        for (int i = 0; i < t->nTem; ++i)
            for (int j = 0; j < t->nDen; ++j)
                for (int c = 0; c < 3; ++c) data[((size_t)i * t->nDen + j) * 3 + c] = t->Data[i][j][c];
    return 0;
}

/* Direct EOS evaluation through the reference, for known-answer tests. */
int ref_eos_state(int matid, double den, double eng, double plim, double pty, double *out3)
{
    if (matid < 1 || matid >= g_sale.nmat) return -1;
    double tem = 0, pre = 0, csd = 0, pty_l = pty;
    calculate_state_correct(g_sale.etb + matid, den, eng, plim, &tem, &pre, &csd, &pty_l);
    out3[0] = tem; out3[1] = pre; out3[2] = csd;
    return 0;
}

/* ----------------------------------------------------------------- tracers */

int ref_tracer_count(void)
{
    if (g_stage != 3) return -1;
    int n = 0;
    field_list_iterator it;
    fl_iterator_init(&it, g_sale.tracer_list, field_list_head);
    field_list_node *node;
    while ((node = fl_iterator_next(&it)) != NULL)
        if (node->state != field_list_deleted) ++n;
    return n;
}

/* Per live tracer, in list order: x, y, vx, vy, mpre, mtem, gx, gy, tag, matid, cell_x, cell_y */
int ref_get_tracers(double *out)
{
    if (g_stage != 3) return -1;
    int n = 0;
    field_list_iterator it;
    fl_iterator_init(&it, g_sale.tracer_list, field_list_head);
    field_list_node *node;
    while ((node = fl_iterator_next(&it)) != NULL) {
        if (node->state == field_list_deleted) continue;
        double *o = out + 12 * (size_t)n;
        o[0] = node->data.position[0]; o[1] = node->data.position[1];
        o[2] = node->data.velocity[0]; o[3] = node->data.velocity[1];
        o[4] = node->data.mpre; o[5] = node->data.mtem;
        o[6] = node->data.gx; o[7] = node->data.gy; o[8] = node->data.tag; o[9] = node->data.matid;
        o[10] = node->id.x; o[11] = node->id.y;
        ++n;
    }
    return n;
}
