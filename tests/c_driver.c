/*
 * Reference-side host driver of the B200 library, compiled against the reference's own headers
 * and sources (recipe: oracle/Makefile, target salec_c_driver).
 *
 * This is the integration a maintainer adds to the reference's main (src/salec2d.c): the
 * start-up of src/salec2d.c:45-105 runs unchanged on the reference's sale2d_var, mesh2d_info and
 * cycle_control; then every run-wide parameter (salec_run_desc), every material's
 * state_reference and EOS table (salec_material_desc), every field of sale2d_var and the tracer
 * list are handed to the library through include/salec_gpu.h, and the loop body of
 * src/salec2d.c:115-272 becomes salec_gpu_step_report. At the end the driver writes the
 * reference's output files of the next cycle's output point through salec_gpu_write_output and
 * the final fields as raw doubles, so that a test can compare them with the reference's own run.
 *
 * Usage: salec_c_driver deck.inp eos_dir work_dir nsteps
 * Writes into work_dir: vts/, vtp/ (the output files) and gpu_fields.bin (dt, time, then
 * e_den, e_pre, m_eng, m_vof, v_vel, e_ste, e_dam in the reference's layout). Exit code 0 on
 * success; a library error prints its salec_gpu_last_error message and exits 2.
 */
#include "sale2d.h"
#include "strength.h"
#include "ejecta.h"
#include "target_profile.h"
#include "write_vtk.h"

#include "salec_gpu.h"

#include <errno.h>
#include <sys/stat.h>
#include <unistd.h>

#define CHECK(call)                                                                        \
    do {                                                                                   \
        int rc_ = (call);                                                                  \
        if (rc_ != SALEC_OK) {                                                             \
            fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, salec_gpu_last_error());   \
            return 2;                                                                      \
        }                                                                                  \
    } while (0)

/* the reference's field_var of a library field name */
static field_var *field_of(sale2d_var *s, const char *n)
{
    struct { const char *name; field_var *fv; } tab[] = {
        {"v_vel", s->v_vel}, {"v_bf", s->v_bf}, {"v_acc", s->v_acc}, {"v_dis", s->v_dis}, {"v_pos", s->v_pos},
        {"v_vof", s->v_vof}, {"v_mass", s->v_mass}, {"v_vol", s->v_vol}, {"v_subvol", s->v_subvol},
        {"v_laplace", s->v_laplace}, {"v_suf", s->v_suf}, {"v_alpha", s->v_alpha}, {"e_vel", s->e_vel},
        {"e_div_vel", s->e_div_vel}, {"e_grad_vel", s->e_grad_vel}, {"e_ste", s->e_ste}, {"e_mu", s->e_mu},
        {"e_dvel", s->e_dvel}, {"e_pre", s->e_pre}, {"e_tem", s->e_tem}, {"e_den", s->e_den}, {"e_csd", s->e_csd},
        {"e_dam", s->e_dam}, {"e_cvs", s->e_cvs}, {"m_vof", s->m_vof}, {"m_den", s->m_den}, {"m_eng", s->m_eng},
        {"m_pty", s->m_pty}, {"e_wpt", s->e_wpt}, {"e_pos", s->e_pos}, {"e_vol", s->e_vol}, {"e_grad", s->e_grad},
        {"e_q", s->e_q}, {"e_strength", s->e_strength}, {"e_cnd", s->e_cnd}, {"e_tps", s->e_tps},
        {"e_ste2s", s->e_ste2s}, {"e_sta2s", s->e_sta2s}, {"e_alpha", s->e_alpha}, {"e_beta", s->e_beta},
        {"e_sigma", s->e_sigma}, {"e_dampref", s->e_dampref}, {"e_vib", s->e_vib}, {"e_ejt", s->e_ejt},
        {"bx_phi", s->bx_phi}, {"by_phi", s->by_phi}, {"bx_normal", s->bx_normal}, {"by_normal", s->by_normal},
        {"y_profile", s->y_profile},
    };
    for (size_t k = 0; k < sizeof(tab) / sizeof(tab[0]); ++k)
        if (strcmp(tab[k].name, n) == 0) return tab[k].fv;
    return NULL;
}

static const char *const kUpload[] = {
    "v_vel", "v_bf", "v_acc", "v_dis", "v_pos", "v_vof", "v_mass", "v_vol", "v_subvol", "v_laplace", "v_suf",
    "v_alpha", "e_vel", "e_div_vel", "e_grad_vel", "e_ste", "e_mu", "e_dvel", "e_pre", "e_tem", "e_den", "e_csd",
    "e_dam", "e_cvs", "m_vof", "m_den", "m_eng", "m_pty", "e_wpt", "e_pos", "e_vol", "e_grad", "e_q",
    "e_strength", "e_cnd", "e_tps", "e_ste2s", "e_sta2s", "e_alpha", "e_beta", "e_sigma", "e_dampref", "e_vib",
    "e_ejt", "bx_phi", "by_phi", "bx_normal", "by_normal", "y_profile",
};

static const char *const kResult[] = {"e_den", "e_pre", "m_eng", "m_vof", "v_vel", "e_ste", "e_dam"};

static long long field_doubles(const field_var *fv) { return (long long)fv->data_size * (fv->bytes_per_unit / sizeof(double)); }

static void ensure_dir(const char *path)
{
    if (mkdir(path, 0755) != 0 && errno != EEXIST) fprintf(stderr, "cannot create %s\n", path);
}

/* the run-wide parameters as the reference holds them after its start-up */
static void fill_run(const sale2d_var *s, const mesh2d_info *m, const cycle_control *c, salec_run_desc *r)
{
    memset(r, 0, sizeof(*r));
    r->nx = m->nx;
    r->ny = m->ny;
    r->nmat = s->nmat;
    r->damp_type = (int)m->damp_type;
    for (int k = 0; k < 4; ++k) r->go[k] = (int)m->go_list[k];
    r->partpres = s->partpres;
    r->porosity_model = s->porosity_model;
    r->acoustic_fluid = s->acoustic_fluid;
    r->tensile_failure = s->tensile_failure;
    r->tracer_lubrication = s->tracer_lubrication;
    r->tracer_lub_gy0 = s->tracer_lub_gy0;
    r->tracer_lub_gy1 = s->tracer_lub_gy1;
    r->avis1 = s->avis1;
    r->avis2 = s->avis2;
    r->anc = s->anc;
    r->density_cutoff = s->density_cutoff;
    r->velocity_max = s->velocity_max;
    r->velocity_min = s->velocity_min;
    r->acceleration_min = s->acceleration_min;
    r->alpha_damp_x = s->alpha_damp_x;
    r->alpha_damp_y = s->alpha_damp_y;
    r->damp_time = s->damp_time;
    r->threshold_z = s->threshold_z;
    r->flow_resistance = s->flow_resistance;
    r->flow_friction = s->flow_friction;
    r->tracer_lub_y0 = s->tracer_lub_y0;
    r->tracer_lub_frac = s->tracer_lub_frac;
    r->max_dt = c->max_dt;
    r->dt = c->dt;
    r->time = c->step_time;
    r->i_step = c->i_step;
    r->precision = SALEC_PRECISION_FP64;
}

/* one material's state_reference and EOS table; table arrays are allocated here, freed by the caller */
static int fill_material(sale2d_var *s, int m, salec_material_desc *d)
{
    memset(d, 0, sizeof(*d));
    const state_reference *r = s->etb[m].ref;
    d->eos_type = (int)s->etb[m].type;
    d->yfunc = salec_gpu_func_index(r->yfunc);
    d->tfunc = salec_gpu_func_index(r->tfunc);
    d->dsdf = salec_gpu_func_index(r->dSDf);
    d->porfunc = salec_gpu_func_index(r->porosityfunc);
    d->VaporDen = r->VaporDen; d->MeltDen = r->MeltDen; d->GaCoef = r->GaCoef;
    d->Yint0 = r->Yint0; d->Yfricint = r->Yfricint; d->Ylimint = r->Ylimint;
    d->Ydam0 = r->Ydam0; d->Yfricdam = r->Yfricdam; d->Ylimdam = r->Ylimdam; d->Yten0 = r->Yten0;
    d->IvanA = r->IvanA; d->IvanB = r->IvanB; d->IvanC = r->IvanC; d->Pbd = r->Pbd; d->Pbp = r->Pbp;
    d->minPint = r->minPint; d->minPdam = r->minPdam;
    d->JCA = r->JCA; d->JCB = r->JCB; d->JCN = r->JCN; d->JCC = r->JCC; d->JCM = r->JCM; d->JCTREF = r->JCTREF;
    d->JCMaxPlastic = r->JCMaxPlastic;
    d->Asimon = r->Asimon; d->Csimon = r->Csimon; d->Tmelt0 = r->Tmelt0; d->Tfrac = r->Tfrac; d->Tdelta = r->Tdelta;
    d->PolyLiq = (int)r->PolyLiq; d->PolySol = (int)r->PolySol;
    d->Tlidc1 = r->Tlidc1; d->Tlidc2 = r->Tlidc2; d->Tlidc3 = r->Tlidc3;
    d->Tsolc1 = r->Tsolc1; d->Tsolc2 = r->Tsolc2; d->Tsolc3 = r->Tsolc3;
    d->Toff = r->Toff; d->Cvib = r->Cvib; d->VibMax = r->VibMax; d->Tdamp = r->Tdamp; d->Pvlim = r->Pvlim;
    d->Acvis = r->Acvis;
    d->alpha0 = r->alpha0; d->alphax = r->alphax; d->epse0 = r->epse0; d->chi = r->chi; d->kappa = r->kappa;
    d->avel = r->avel; d->epsec = r->epsec; d->epsex = r->epsex; d->alphamax = r->alphamax;
    d->alphamax2 = r->alphamax2; d->alphae = r->alphae; d->gamfrac = r->gamfrac;
    d->melt_viscosity = r->melt_viscosity;
    if (s->etb[m].type == Tillotson) {
        const tillotson_table *t = (const tillotson_table *)s->etb[m].table;
        const double p[13] = {t->TLRho0, t->TLCv, t->TLA, t->TLB, t->TLE0, t->TLa, t->TLb,
                              t->TLAlpha, t->TLBeta, t->TLEiv, t->TLEcv, t->TLTref, t->StepDen};
        memcpy(d->till, p, sizeof(p));
        d->cold_n = t->nDen;
        d->cold_xden = t->xDen;
        d->cold_yeng = t->yEng;
    } else if (s->etb[m].type == ANEOS || s->etb[m].type == ANEOSSieDen) {
        const aneos_table *t = (const aneos_table *)s->etb[m].table;
        d->ntem = t->nTem;
        d->nden = t->nDen;
        d->xtem = t->xTem;
        d->yden = t->yDen;
        double *data = (double *)malloc(sizeof(double) * (size_t)t->nTem * t->nDen * 3);
        if (!data) return -1;
        for (int i = 0; i < t->nTem; ++i)
            for (int j = 0; j < t->nDen; ++j)
                for (int k = 0; k < 3; ++k) data[((size_t)i * t->nDen + j) * 3 + k] = t->Data[i][j][k];
        d->data = data;
    }
    return 0;
}

/* the reference's tracer list as rows of 12 doubles (x, y, vx, vy, mpre, mtem, gx, gy, tag, matid, cell) */
static double *tracer_rows(sale2d_var *s, int *n)
{
    int count = 0;
    field_list_iterator it;
    field_list_node *node;
    fl_iterator_init(&it, s->tracer_list, field_list_head);
    while ((node = fl_iterator_next(&it)) != NULL)
        if (node->state != field_list_deleted) ++count;
    double *rows = (double *)calloc((size_t)(count > 0 ? count : 1) * 12, sizeof(double));
    int k = 0;
    fl_iterator_init(&it, s->tracer_list, field_list_head);
    while ((node = fl_iterator_next(&it)) != NULL) {
        if (node->state == field_list_deleted) continue;
        double *o = rows + 12 * (size_t)k++;
        o[0] = node->data.position[0]; o[1] = node->data.position[1];
        o[2] = node->data.velocity[0]; o[3] = node->data.velocity[1];
        o[4] = node->data.mpre; o[5] = node->data.mtem;
        o[6] = node->data.gx; o[7] = node->data.gy; o[8] = node->data.tag; o[9] = node->data.matid;
        o[10] = node->id.x; o[11] = node->id.y;
    }
    *n = count;
    return rows;
}

int main(int argc, char **argv)
{
    if (argc != 5) {
        fprintf(stderr, "usage: %s deck.inp eos_dir work_dir nsteps\n", argv[0]);
        return 1;
    }
    const char *inpfile = argv[1], *eospath = argv[2], *work = argv[3];
    const int nsteps = atoi(argv[4]);
    MPI_Init(&argc, &argv);
    ensure_dir(work);
    if (chdir(work) != 0) return 1;
    ensure_dir("./vts"); ensure_dir("./vtp"); ensure_dir("./txt"); ensure_dir("./post");

    sale2d_var sale2d;
    mesh2d_info minfo;
    cycle_control ccl;
    memset(&sale2d, 0, sizeof(sale2d));
    memset(&minfo, 0, sizeof(minfo));
    memset(&ccl, 0, sizeof(ccl));

    /* ---- the reference's start-up (src/salec2d.c:45-105) */
    InputFile *ifp = OpenInputFile(inpfile);
    init_cycle_control(ifp, &ccl);
    load_mesh_info(ifp, &minfo, (char *)eospath);
    init_sale_mat(&sale2d, &minfo);
    select_strength_model(&sale2d);
    init_sale2d_var(&sale2d, &minfo);
    /* the fields start from zeroed memory, as the large blocks malloc hands the reference do */
    for (int k = 0; k < sale2d.fv_counter; ++k) {
        field_var *fv = sale2d.v_vel + k;
        if (fv->data) memset(fv->data, 0, (size_t)fv->data_size * fv->bytes_per_unit);
    }
    init_sale2d_other(&sale2d, ifp);
    init_sale2d_ghost(&sale2d, &minfo);
    CloseInputFile(ifp);
    init_mesh_pos(&sale2d, &minfo);
    init_material_distribution(&minfo, &sale2d);
    update_state(&sale2d, internal_section | send_section);
    sync_start(sale2d.e_den);
    sync_complete(sale2d.e_den);
    flush_ght(sale2d.e_pre);
    flush_ght(sale2d.e_ste);
    flush_ght(sale2d.m_eng);
    flush_ght(sale2d.m_pty);
    flush_ght(sale2d.e_cvs);
    double local_damp_time = record_avg_value(&sale2d);
    MPI_Allreduce(&(local_damp_time), &(minfo.damp_t), 1, MPI_DOUBLE, MPI_MAX, sale2d.e_pre->comm);
    minfo.damp_t *= 2.0;
    sale2d.damp_time = Max(minfo.damp_t, sale2d.damp_time);
    init_v_field(&sale2d);
    clean_fv(sale2d.e_vel);
    clean_fv(sale2d.e_ste);
    clean_fv(sale2d.e_dvel);
    ccl.out_vts = 1;
    ccl.k_out_step = 1;
    init_sale2d_tracer(&sale2d, &minfo);
    /* the reference builds every tracer from a stack variable whose peak pressure and temperature
       it never sets (src/tracer.c:405-445); they start at 0, as in the library's own initialiser */
    {
        field_list_iterator it;
        field_list_node *node;
        fl_iterator_init(&it, sale2d.tracer_list, field_list_head);
        while ((node = fl_iterator_next(&it)) != NULL) {
            node->data.mpre = 0.0f;
            node->data.mtem = 0.0f;
        }
    }

    /* ---- hand-off to the device */
    salec_run_desc run;
    fill_run(&sale2d, &minfo, &ccl, &run);
    salec_material_desc *mats = (salec_material_desc *)calloc((size_t)sale2d.nmat, sizeof(salec_material_desc));
    for (int m = 1; m < sale2d.nmat; ++m)
        if (fill_material(&sale2d, m, mats + m) != 0) return 1;
    salec_gpu *h = NULL;
    CHECK(salec_gpu_create(&run, mats, &h));
    for (int m = 1; m < sale2d.nmat; ++m) free((void *)mats[m].data);
    free(mats);
    for (size_t k = 0; k < sizeof(kUpload) / sizeof(kUpload[0]); ++k) {
        field_var *fv = field_of(&sale2d, kUpload[k]);
        CHECK(salec_gpu_set_field(h, salec_gpu_field_index(kUpload[k]), (const double *)fv->data, field_doubles(fv)));
    }
    int ntr = 0;
    double *rows = tracer_rows(&sale2d, &ntr);
    CHECK(salec_gpu_set_tracers(h, ntr, rows));
    free(rows);

    /* ---- the time loop: one library call per cycle */
    double dt = 0., t = 0.;
    for (int k = 0; k < nsteps; ++k) CHECK(salec_gpu_step_report(h, 1, &dt, &t, NULL, 0));

    /* ---- the final fields in the reference's layout, into the reference's own arrays */
    FILE *fp = fopen("gpu_fields.bin", "wb");
    if (!fp) return 1;
    fwrite(&dt, sizeof(double), 1, fp);
    fwrite(&t, sizeof(double), 1, fp);
    for (size_t k = 0; k < sizeof(kResult) / sizeof(kResult[0]); ++k) {
        field_var *fv = field_of(&sale2d, kResult[k]);
        CHECK(salec_gpu_get_field(h, salec_gpu_field_index(kResult[k]), (double *)fv->data, field_doubles(fv)));
        fwrite(fv->data, sizeof(double), (size_t)field_doubles(fv), fp);
    }
    fclose(fp);

    /* ---- the next cycle's output point (src/salec2d.c:241-245) through the library's writer */
    CHECK(salec_gpu_phases(h, 0, 13));
    CHECK(salec_gpu_write_output(h, ".", minfo.prefix, 0, ccl.k_out_step - 1, SALEC_OUT_WAIT));
    CHECK(salec_gpu_destroy(h));
    MPI_Finalize();
    return 0;
}
