/*
 * salec_gpu.h - C ABI of the B200 (sm_100a) per-timestep mesh update of SALEc2d.
 *
 * The reference has no plugin or FFI layer: its step is a sequence of
 * `void f(sale2d_var *, node_type, double dt)` sweeps called from the time loop in
 * src/salec2d.c:115-272 (declarations in src/sale2d.h:397-466, src/strength.h:11-35,
 * src/ejecta.h:35-36, src/tracer.h:16-24). These entry points replace that loop body:
 * a host driver keeps the reference's own initialisation (deck parser, EOS loaders,
 * target profile, geometry) and output writers, uploads the initialised fields once,
 * calls salec_gpu_step() per cycle, and downloads fields at output cycles.
 *
 * Conventions (kept from the reference's interface):
 *   - field data crosses the boundary in the reference's own memory layout: one block per
 *     field, points with the x index fastest (src/mpi_vec/mpi_vec.h:372-376), and the
 *     components of one point contiguous, exactly the bytes of field_var.data;
 *   - point counts include the two-cell pad: cells (nx+4) x (ny+4), vertices (nx+5) x (ny+5),
 *     x faces (nx+5) x (ny+4), y faces (nx+4) x (ny+5) (src/sale2d_back.c:169-175);
 *   - the caller owns every host buffer; the library owns every device buffer.
 * Unlike the reference (which calls exit(0) on errors, e.g. src/sale2d_back.c:49-51), every
 * entry point returns SALEC_OK or a negative salec_status and never terminates the process.
 * One handle is used by one host thread at a time; all its work runs on one CUDA stream.
 */
#ifndef SALEC_GPU_H
#define SALEC_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct salec_gpu salec_gpu;

enum salec_status {
    SALEC_OK = 0,
    SALEC_ERR_ARG = -1,         /* invalid argument, unknown name or size mismatch */
    SALEC_ERR_CUDA = -2,        /* a CUDA runtime call failed; see salec_gpu_last_error() */
    SALEC_ERR_ALLOC = -3,       /* device or host allocation failed */
    SALEC_ERR_STATE = -4,       /* call not valid in the handle's current state */
    SALEC_ERR_UNSUPPORTED = -5, /* option the reference supports but this build does not */
    SALEC_ERR_NUMERIC = -6      /* non-finite values detected by salec_gpu_check() */
};

/* Equation-of-state kinds, numbered as the reference's eos_type (src/eos/eos_state.h:222-228). */
enum salec_eos_kind { SALEC_EOS_ANEOS = 0, SALEC_EOS_TILLOTSON = 1, SALEC_EOS_ANEOS_SIEDEN = 2 };

/* Damping layer kinds, numbered as the reference's damp_type_t (src/sale2d.h:252-260). */
enum salec_damp_kind { SALEC_DAMP_PML = 0, SALEC_DAMP_PML2 = 1, SALEC_DAMP_PML3 = 2,
                       SALEC_DAMP_SBC = 3, SALEC_DAMP_CTLG = 4, SALEC_DAMP_NONE = 5 };

/* Strength, damage, tensile and porosity functions, in the order of the reference's
 * registry str_func_list (src/strength.c:860-875); the name lookup is salec_gpu_func_index(). */
enum salec_func {
    SALEC_FN_SIMPLE_ROCK = 0, SALEC_FN_SIMPLE_SHEAR = 1, SALEC_FN_JOHNSON_COOK1 = 2,
    SALEC_FN_JOHNSON_COOK2 = 3, SALEC_FN_ROCK_STRENGTH_T = 4, SALEC_FN_ICE_STRENGTH = 5,
    SALEC_FN_COLLINS = 6, SALEC_FN_IVANOV = 7, SALEC_FN_SIMPLE_TENSILE = 8, SALEC_FN_NONE = 9,
    SALEC_FN_WUNNEMANN = 10, SALEC_FN_VON_MISES1 = 11, SALEC_FN_VON_MISES2 = 12
};

/*
 * Run-wide parameters. Each field is the value the reference holds after initialisation,
 * in sale2d_var (src/sale2d.h:34-174), mesh2d_info (:319-386) or cycle_control (:176-208).
 * go[4] are the ghost options of the left, right, bottom and top boundaries after
 * boundary_str2opt and the Ox < 1e-6 mirror rule (src/sale2d_back.c:230-238, :405-428),
 * numbered as the reference's ght_opt (src/mpi_vec/mpi_vec_types.h:74-95).
 */
typedef struct salec_run_desc {
    int nx, ny;                 /* interior cells (mesh.npx, mesh.npy) of the single domain */
    int nmat;                   /* materials including vacuum (material.nm) */
    int damp_type;              /* salec_damp_kind */
    int go[4];
    int partpres, porosity_model, acoustic_fluid, tensile_failure;
    int tracer_lubrication, tracer_lub_gy0, tracer_lub_gy1;
    double avis1, avis2, anc;
    double density_cutoff, velocity_max, velocity_min, acceleration_min;
    double alpha_damp_x, alpha_damp_y, damp_time;
    double threshold_z, flow_resistance, flow_friction;
    double tracer_lub_y0, tracer_lub_frac;
    double max_dt, dt, time;    /* cycle.maxdt, current dt and simulated time */
    int i_step;
    /* Storage precision of the device mesh (no counterpart in the reference, which is FP64):
     * SALEC_PRECISION_FP64 (0, the plain form, bit-parity with the reference) or
     * SALEC_PRECISION_MIXED (1): the fields of stress, strain rate, viscosity, EOS outputs,
     * velocities, accelerations, damping and geometry weights are stored as FP32 and computed in
     * FP64 registers; volume fractions, material densities and energies, the porosity state,
     * positions, cell volumes and the face flux records (volume-fraction advection, mass and
     * energy conservation) stay FP64. Zero-initialised descriptions select FP64. */
    int precision;
} salec_run_desc;

enum salec_precision { SALEC_PRECISION_FP64 = 0, SALEC_PRECISION_MIXED = 1 };

/*
 * One material (index >= 1; index 0 is vacuum and is ignored): the reference's
 * state_reference (src/eos/eos_state.h:43-151) plus its EOS table. Table arrays are read
 * during salec_gpu_create() only.
 */
typedef struct salec_material_desc {
    int eos_type;               /* salec_eos_kind */
    int yfunc, tfunc, dsdf, porfunc;   /* salec_func for shear strength, tensile strength,
                                          damage increment and porosity increment */
    double VaporDen, MeltDen, GaCoef;
    double Yint0, Yfricint, Ylimint, Ydam0, Yfricdam, Ylimdam, Yten0;
    double IvanA, IvanB, IvanC, Pbd, Pbp, minPint, minPdam;
    double JCA, JCB, JCN, JCC, JCM, JCTREF, JCMaxPlastic;
    double Asimon, Csimon, Tmelt0, Tfrac, Tdelta;
    int PolyLiq, PolySol;
    double Tlidc1, Tlidc2, Tlidc3, Tsolc1, Tsolc2, Tsolc3;
    double Toff, Cvib, VibMax, Tdamp, Pvlim, Acvis;
    double alpha0, alphax, epse0, chi, kappa, avel, epsec, epsex, alphamax, alphamax2, alphae;
    double gamfrac, melt_viscosity;
    /* Tillotson: Rho0, Cv, A, B, E0, a, b, Alpha, Beta, Eiv, Ecv, Tref, StepDen
       (src/eos/eos_state.h:168-186) and the cold-energy curve of TillColdEnergy. */
    double till[13];
    int cold_n;
    const double *cold_xden, *cold_yeng;
    /* Tabulated kinds: axes and Data[iT][iD][0..2] flattened as [ntem][nden][3]. */
    int ntem, nden;
    const double *xtem, *yden, *data;
} salec_material_desc;

/* Create a handle on the current CUDA device. mats has nmat entries (entry 0 unused). */
int salec_gpu_create(const salec_run_desc *run, const salec_material_desc *mats, salec_gpu **out);
int salec_gpu_destroy(salec_gpu *h);

/*
 * Create a handle directly from a reference input deck (.inp) and the folder holding its EOS
 * files (the reference's `salec2d deck.inp eos_dir`), without the reference's host code: the
 * start-up of src/salec2d.c:45-105 (deck, materials, EOS tables, geometry, hydrostatic target
 * profile, material distribution, first EOS call, damping reference state, vertex velocities,
 * tracers) is restated by the library. A deck for an npgx x npgy process grid is run as one
 * domain of (npgx*npx) x (npgy*npy) cells.
 */
int salec_gpu_create_from_deck(const char *deck_path, const char *eos_dir, salec_gpu **out);
/* The same with a storage precision (salec_precision) for the device mesh. */
int salec_gpu_create_from_deck_ex(const char *deck_path, const char *eos_dir, int precision, salec_gpu **out);
/* The run description of a handle (for a deck-created handle: the values derived from the deck). */
int salec_gpu_get_run(const salec_gpu *h, salec_run_desc *out);

/* Field names are the reference's member names of sale2d_var (e.g. "m_vof", "v_vel",
 * "bx_phi", "y_profile"). Returns the field index or -1. */
int salec_gpu_field_index(const char *name);
/* Points in x and y and doubles per point of a field in the reference's layout. */
int salec_gpu_field_shape(const salec_gpu *h, int field, int *nx, int *ny, int *ncomp);
/* Copy a whole field from / to a host buffer of n doubles in the reference's layout. */
int salec_gpu_set_field(salec_gpu *h, int field, const double *host, long long n);
int salec_gpu_get_field(salec_gpu *h, int field, double *host, long long n);

/* Advance nsteps full cycles: the loop body of src/salec2d.c:115-272 without the output point. */
int salec_gpu_step(salec_gpu *h, int nsteps);
/* salec_gpu_step, then the per-cycle quantities of the reference's loop: dt and the simulated
 * time (the MIN-reduced ccl.dt and ccl.step_time, src/salec2d.c:167-168; either pointer may be
 * NULL) and, when profile is not NULL, the surface profile y_profile (the MIN-reduced
 * sale2d.y_profile, src/salec2d.c:120, 232; profile_n doubles, its field shape). The read-backs are queued
 * behind the cycles and the call synchronises once, where salec_gpu_get_scalar and
 * salec_gpu_get_field would synchronise once each. Results equal those calls'. */
int salec_gpu_step_report(salec_gpu *h, int nsteps, double *dt, double *time, double *profile, long long profile_n);
/* The same, pipelined: queue nsteps cycles and the read-back of dt, time and (when profile is not
 * NULL) the surface profile into report slot `slot` (0 or 1), and return without waiting.
 * salec_gpu_report_wait(h, slot, &dt, &time) then waits for that slot's read-back and gives dt
 * and time. A host loop can so queue cycle k+1 before it waits for cycle k's results, and the
 * device does not idle while the host wakes up. profile should be page-locked memory
 * (cudaHostAlloc) for the copy to overlap; it is written when the slot's wait returns. A slot
 * must be waited for before it is queued again. */
int salec_gpu_step_report_async(salec_gpu *h, int nsteps, double *profile, long long profile_n, int slot);
int salec_gpu_report_wait(salec_gpu *h, int slot, double *dt, double *time);
/* Advance an ensemble of independent simulations (each handle a different deck or mesh size)
 * by nsteps cycles each. Cycles are queued round-robin, chunk cycles per member at a time, each
 * member on its own stream, so the kernels of small meshes run side by side on the device.
 * Every member computes exactly what salec_gpu_step() alone would. The call returns once the
 * work is queued; salec_gpu_sync() on a member waits for it. chunk <= 0 selects 16. */
int salec_gpu_step_many(salec_gpu *const *handles, int n, int nsteps, int chunk);
/* Run phases first..last of one cycle, for stepwise checks and timing. Phases follow the
 * reference's loop body (src/salec2d.c): 0 surface profile, 1 vertex volume fractions and
 * vertex momentum + restriction (one vertex sweep), 2 empty (the reference's second half of
 * the vertex momentum update is done in 1), 3 cell velocity + ghosts, 4 void vertices, 5 velocity
 * gradient, viscosity and CFL candidates, 6 time step, 7 vibration/stress/damage, 8 vertex
 * acceleration (+ ghosts, restriction), 9 vertex displacement + restriction, 10 internal
 * energy, 11 tracers, 12 face fluxes (+ ghosts), 13 strength condition, 14 remap, damping,
 * ejecta drag and EOS, 15 cycle control. */
int salec_gpu_phases(salec_gpu *h, int first, int last);
/* Pick the block shape of every 2-D sweep for this handle's mesh: each candidate shape is
 * timed per phase over `cycles` cycles (after one warm-up cycle) from a device snapshot of the
 * state, the fastest is kept per sweep, and the snapshot is restored, so the simulation is left
 * exactly where it was. The shape changes no result (one thread per point, exact reductions).
 * Takes a device copy of the field pool for its duration. If shapes is not NULL it receives 10
 * triples (phase, block x, block y). No counterpart in the reference. */
int salec_gpu_autotune(salec_gpu *h, int cycles, int *shapes);
/* Set the block shapes of the tunable 2-D sweeps from n triples (phase, block x, block y), as
 * salec_gpu_autotune returns them, e.g. to reuse one member's tuning for others of the same
 * mesh. Block x must be a multiple of 32 and x*y at most 256; any invalid triple rejects the
 * whole call (SALEC_ERR_ARG) with no shape changed. No counterpart in the reference. */
int salec_gpu_set_block_shapes(salec_gpu *h, const int *shapes, int n);
/* Block until the handle's stream is idle. */
int salec_gpu_sync(salec_gpu *h);
/* The CUDA stream (cudaStream_t) all work of the handle is queued on. */
int salec_gpu_stream(salec_gpu *h, void **stream);
/* Per-phase device timing: when enabled, every phase run is bracketed by CUDA events on the
 * handle's stream; salec_gpu_phase_times() waits for the stream and returns, per phase 0..15,
 * the summed milliseconds and the number of runs since the last call (or since enabling). */
int salec_gpu_profile(salec_gpu *h, int enable);
int salec_gpu_phase_times(salec_gpu *h, double *ms, long long *count);

/* Scalars: "dt", "time", "i_step", "damp_time", "max_dt". */
int salec_gpu_get_scalar(salec_gpu *h, const char *name, double *value);
int salec_gpu_set_scalar(salec_gpu *h, const char *name, double value);

/* Lagrangian tracers (src/tracer.c:52-175, list built by fl_tracer_init :380-450). Rows of 12
 * doubles per tracer: x, y, vx, vy, mpre, mtem, gx, gy, tag, matid, cell_x, cell_y (cell_x/y is
 * the reference's node->id). set replaces the tracer list; get returns the live tracers in
 * list order, *n is in/out (row capacity in, live count out); rows == NULL only counts. */
int salec_gpu_set_tracers(salec_gpu *h, int n, const double *rows);
int salec_gpu_get_tracers(salec_gpu *h, double *rows, int *n);

/*
 * Conservation sums of the current state, in FP64 with compensated (Neumaier) summation, also in
 * the mixed form. No counterpart in the reference; the quantities are those its conservative remap
 * and momentum update carry. out[0] total mass (sum over interior cells and materials of
 * m_vof * e_vol * m_den), out[1] and out[2] r and z momentum (sum over active vertices of
 * v_mass[0] * v_vel), out[3] internal energy (m_vof * e_vol * m_eng), out[4] kinetic energy
 * (0.5 * v_mass[0] * |v_vel|^2), out[4 + m] the mass of material m = 1 .. nmat-1; n >= 4 + nmat.
 * Synchronises the handle's stream.
 */
int salec_gpu_conservation(salec_gpu *h, double *out, int n);

/* Count non-finite values in the evolving cell and vertex fields; SALEC_ERR_NUMERIC if any. */
int salec_gpu_check(salec_gpu *h, long long *n_bad);

/*
 * Output files of the current state, byte for byte those the reference writes for one rank
 * (compiled with OUTPUT_GHT, as its CMakeLists does):
 *   <dir>/vts/<prefix>.proc<rank>.<out_step>.vts          sale2d_write_vtk (src/write_vtk.c:189-298)
 *   <dir>/vtp/<prefix>.tracer.proc<rank>.<out_step>.vtp   sale2d_write_vtp (src/write_vtk.c:354-480)
 *   <dir>/txt/<prefix>.tracer.proc<rank>.<out_step>.txt   with SALEC_OUT_TRACER_TXT (:482-498)
 * (rank and out_step printed %04d; out_step is the reference's k_out_step - 1). The reference
 * writes in the middle of a cycle, after the flux and before the remap: run phases 0-13, call
 * this, then phases 14-15. The device packs the arrays (FP64 -> FP32) and copies them to
 * pinned host memory on the handle's stream; compression and file writing then run on host
 * threads while the device continues. Without SALEC_OUT_WAIT the call returns once that work
 * is queued; the next output call, salec_gpu_output_wait() or salec_gpu_destroy() waits for it
 * and reports its errors.
 */
#define SALEC_OUT_WAIT 1
#define SALEC_OUT_TRACER_TXT 2
int salec_gpu_write_output(salec_gpu *h, const char *dir, const char *prefix, int rank, int out_step, int flags);
int salec_gpu_output_wait(salec_gpu *h);

/*
 * Boundary tables compiled to gather maps (host only, no device needed). The reference fills
 * ghost cells and restricts boundary vertices by walking a table point by point
 * (src/mpi_vec/mpi_vec_ght.c:279-357 and :657-696); the map gives, for each point the walk
 * writes, the original point its final value comes from and a per-component transform
 * (3 bits per component: 0 copy, 1 negate, 2 abs, 3 -abs, 4 +0, 5 -0).
 * kind 0: ghost table of a cell field with pattern (0 always-copy, 1 normal, 2 velocity
 * increment, 3 velocity, 4 stress, 5 density); kind 1: vertex restriction table.
 * nx, ny: points of the field in x and y; points are indexed x-fastest. *n is in/out
 * (capacity in, entries out); dst/src/ops may be NULL to query the count.
 */
int salec_boundary_map(int kind, int pattern, int nx, int ny, int ncomp, const int go[4], int *n, int *dst,
                       int *src, unsigned *ops);

/*
 * CFL time step of one cycle without allocating device memory. No counterpart in the
 * reference: it computes what calculate_dt (src/sale2d.c:1959-2016) and the Min with max_dt
 * (src/salec2d.c:167) give, for callers that cannot call cudaMalloc while they run their time
 * loop - a host code whose device memory belongs to its own pool allocator, or one that must
 * not take cudaMalloc's device-wide synchronisation inside a cycle.
 * Inputs are caller-owned device planes of (nx+4) x (ny+4) doubles in the reference's cell
 * order (x fastest, two-cell pad, row pitch exactly nx+4 with no padding between rows): cell
 * velocity r and z, sound speed, cell scales r and z (e_pos components 2 and 3) and the vacuum
 * volume fraction. The library's own device planes are not accepted: they have a padded pitch,
 * and in the mixed form (SALEC_PRECISION_MIXED) the velocity and sound speed are float planes.
 * dt_out is one device double; stream is a cudaStream_t (NULL: the default stream); the work is
 * enqueued, not waited for.
 * Scratch: fixed arrays in the library's device image (64 KiB of partial minima and 8 KiB of
 * flags), held on every device that loads the library until the process exits; they limit a
 * call to 8192 * 4096 = 33554432 interior cells (larger meshes return SALEC_ERR_ARG). Every
 * call looks the arrays' addresses up with the caller's device current; the first call on a
 * device also loads the library's device code there and should come before any stream capture.
 * All calls share the arrays, so calls that overlap on the GPU race and must be ordered by the
 * caller; each call rewrites every entry it reads, so nothing needs clearing between calls.
 * NaN candidates follow the reference's sequential MIN (src/mpi_vec/mpi_vec_types.h:262, folded
 * in traversal order from 1.1 * dt_prev), as salec_gpu_step does: the result is the MIN of the
 * candidates after the last NaN, or NaN when the NaN is the last candidate.
 */
int salec_cfl_dt_noalloc(int nx, int ny, const double *vel_r, const double *vel_z, const double *csd,
                         const double *scale_r, const double *scale_z, const double *vof_vacuum,
                         double dt_prev, double max_dt, double *dt_out, void *stream);

/*
 * Prescribed time steps: cycles i0 .. i0+n-1, where i0 is the handle's current cycle count, take
 * dts[k] instead of the CFL reduction of src/sale2d.c:1959-2016 (n = 0 removes the schedule).
 * No counterpart in the reference; it replays a recorded dt sequence, e.g. for finite-difference
 * checks of the adjoint, which differentiates at frozen time steps.
 */
int salec_gpu_set_dt_schedule(salec_gpu *h, const double *dts, int n);

/*
 * Adjoint (reverse-mode derivatives) of the mesh update. No counterpart in the reference.
 * Supported configuration: the plain FP64 form, one material beside vacuum with a Tillotson EOS,
 * RockStrengthT yield (src/strength.c:697-722) with Ivanov or SimpleShear damage, damping = none,
 * no porosity, acoustic fluidisation, tensile failure, tracer lubrication or ejecta drag, and
 * partpres = 0; other handles return SALEC_ERR_UNSUPPORTED. Derivatives are those of the step at
 * frozen time steps (the dt of each cycle as the forward run computed it); discrete quantities
 * (void-corner counts, material flags, cut-line corner distances, the surface profile y_profile)
 * carry none. Adjoint fields share the layout and names of the forward fields.
 *
 * The building blocks: salec_gpu_adjoint_reset allocates (once) and zeroes the adjoint planes and
 * the parameter gradients; salec_gpu_adjoint_set_field / _get_field move an adjoint field in the
 * reference's layout; salec_gpu_adjoint_phase(h, p) applies the reverse of phase p (the phases of
 * salec_gpu_phases) with the handle's current state taken as the state before that phase: the
 * adjoints of p's outputs become those of its inputs. salec_gpu_adjoint_params reads the
 * accumulated d/d Yint0, Yfricint, Ydam0, Yfricdam of material 1 (RockStrengthT's cohesions and
 * frictions, through the yield strength and the EOS pressure floor minPint/minPdam).
 */
int salec_gpu_adjoint_reset(salec_gpu *h);
int salec_gpu_adjoint_set_field(salec_gpu *h, int field, const double *host, long long n);
int salec_gpu_adjoint_get_field(salec_gpu *h, int field, double *host, long long n);
int salec_gpu_adjoint_phase(salec_gpu *h, int phase);
int salec_gpu_adjoint_params(salec_gpu *h, double *theta4);

typedef struct salec_adjoint_result {
    double misfit;            /* J = 0.5 * sum_i w_i (h_i - target_i)^2 at the window's end */
    double d_params[4];       /* dJ/d Yint0, Yfricint, Ydam0, Yfricdam of material 1 */
    double d_velocity_scale;  /* dJ/d lambda for the window's initial vertex velocities scaled by
                                 lambda at lambda = 1 (the impactor speed U: dJ/dU = this / U) */
} salec_adjoint_result;

/*
 * Adjoint of a window of nsteps cycles from the current state, checkpointed every `every` cycles:
 * the window runs forward saving a checkpoint at each segment start; the misfit of the final
 * surface-height profile is formed, h_i = sum over interior rows j of (1 - m_vof[0]) * e_pos[3]
 * (the material column height of interior column i, a smooth stand-in for the vacuum-based
 * y_profile), J = 0.5 * sum_i w_i (h_i - target_i)^2 with target and w (NULL: all 1) given per
 * interior column (ncols = nx); then each segment is replayed from its checkpoint with an undo log
 * of every phase, and the reverse phases run back to the window's start. Results: *out, the
 * adjoint fields of the window's start (salec_gpu_adjoint_get_field) and, when grad_density is not
 * NULL ((nx+4)*(ny+4) doubles, the cell layout), dJ/drho of every cell for a change of its initial
 * density that scales its material densities and its cell density together. The handle is left at
 * the window's end.
 */
int salec_gpu_adjoint_window(salec_gpu *h, int nsteps, int every, const double *target, const double *weight,
                             int ncols, double *grad_density, long long n_density, salec_adjoint_result *out);

/* Strength/damage/porosity function index for a reference name (case-insensitive), or -1. */
int salec_gpu_func_index(const char *name);
/* Message of the last error on this thread. */
const char *salec_gpu_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
