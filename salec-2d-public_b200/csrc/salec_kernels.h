// Kernel entry points and the gather-map types shared by the host runtime and the kernels.
#pragma once
#include <cstdint>
#include <vector>

namespace salec {

struct Ctx;

#define SALEC_MAX_GATHER_FIELDS 8

// Boundary fills as gathers: for entry k, dst[k] <- op_c(src[k]) for each component c, where
// op_c is 3 bits of ops[k]: 0 copy, 1 negate, 2 abs, 3 -abs, 4 +0.0, 5 -0.0.
struct GatherField {
    double *base;          // component-0 plane of the field
    long long plane;       // plane stride
    int ncomp, ncomp_max;  // components of this field; max over the batch (scratch stride)
    const int *dst, *src;
    const unsigned *ops;
};

struct GatherBatch {
    GatherField field[SALEC_MAX_GATHER_FIELDS];
    int start[SALEC_MAX_GATHER_FIELDS + 1];
    int nfield, total;
};

// Host-side gather map of one field: entries in increasing destination order.
struct GatherMap {
    std::vector<int> dst, src;
    std::vector<unsigned> ops;
    bool needs_scratch = false;   // some source is also a destination
};

// Ghost patterns of the reference (src/mpi_vec/mpi_vec_ght.c:156-277).
enum GhostPattern { GP_ALWAYS_COPY = 0, GP_NORMAL = 1, GP_VELOCITY_INC = 2, GP_VELOCITY = 3, GP_STRESS = 4,
                    GP_DENSITY = 5 };

// Build the gather map of the ghost-cell table of a cell field (enx x eny points, pitch P).
GatherMap build_ghost_map(int enx, int eny, int P, int ncomp, const int go[4], GhostPattern pat);
// Build the gather map of the vertex restriction table (vnx x vny points, pitch P).
GatherMap build_restrict_map(int vnx, int vny, int P, int ncomp, const int go[4]);

#ifdef __CUDACC__
// kernels (salec_step.cu)
__global__ void k_profile_reset(const Ctx c);
__global__ void k_trace_profile(const Ctx c);
__global__ void k_profile_decode(const Ctx c);
__global__ void k_vertex_vof_momentum(const Ctx c);
__global__ void k_cell_velocity(const Ctx c);
__global__ void k_void_vertices(const Ctx c);
__global__ void k_gradient_viscosity_cfl(const Ctx c);
__global__ void k_finalize_dt(const Ctx c);
__global__ void k_vertex_acceleration(const Ctx c);
__global__ void k_vertex_displacement(const Ctx c);
__global__ void k_tracers(const Ctx c);
__global__ void k_cycle(const Ctx c);
__global__ void k_record_reference_state(const Ctx c);
__global__ void k_init_vertex_velocity(const Ctx c);
__global__ void k_gather(GatherBatch g, int mode, double *scratch);
__global__ void k_aos_to_planes(const double *aos, double *base, long long plane, int P, int nx, int ny, int nc);
__global__ void k_planes_to_aos(const double *base, double *aos, long long plane, int P, int nx, int ny, int nc);
__global__ void k_count_nonfinite(const double *base, long long n, unsigned long long *out);
void launch_stress(const Ctx &c, dim3 g, dim3 b, cudaStream_t s);
void launch_energy(const Ctx &c, dim3 g, dim3 b, cudaStream_t s);
void launch_flux(const Ctx &c, int pass, dim3 g, dim3 b, cudaStream_t s);
void launch_remap_damp_state(const Ctx &c, int do_remap, int do_damp, int do_ejecta, int do_state, dim3 g, dim3 b,
                             cudaStream_t s);
#endif

} // namespace salec
