// Kernel entry points and the gather-map types shared by the host runtime and the kernels.
#pragma once
#include <cstdint>
#include <vector>

namespace salec {

template <class R>
struct CtxT;   // salec_device.cuh

#define SALEC_MAX_GATHER_FIELDS 8

// Boundary fills as gathers: for entry k, dst[k] <- op_c(src[k]) for each component c, where
// op_c is 3 bits of ops[k]: 0 copy, 1 negate, 2 abs, 3 -abs, 4 +0.0, 5 -0.0.
struct GatherField {
    void *base;            // component-0 plane of the field (double, or float when f32)
    long long plane;       // plane stride in elements
    int ncomp, ncomp_max;  // components of this field; max over the batch (scratch stride)
    int f32;               // the field is stored as float
    const int *dst, *src;
    const unsigned *ops;
    // null: one work item per entry. Otherwise entries are grouped into components (no point of
    // a component is read or written by another) and work item w covers entries
    // [cstart[w], cstart[w+1]), at most SALEC_GATHER_MAX_COMPONENT of them
    const int *cstart;
};

constexpr int SALEC_GATHER_MAX_COMPONENT = 16;

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

// Entries of a map whose sources include destinations, grouped into connected components of the
// read/write relation; false when a component exceeds SALEC_GATHER_MAX_COMPONENT entries.
bool group_gather_components(const GatherMap &m, GatherMap &out, std::vector<int> &cstart);

// Step kernels of salec_step.cu, launched over their own grids by launch_step_kernel; R is
// the storage type of the relaxed fields (double: plain FP64 form, float: mixed form).
enum StepKernel {
    SK_PROFILE_RESET, SK_TRACE_PROFILE, SK_PROFILE_DECODE, SK_VERTEX_VOF_MOMENTUM, SK_CELL_VELOCITY,
    SK_VOID_VERTICES, SK_GRADIENT, SK_FINALIZE_DT, SK_STRESS, SK_ACCELERATION, SK_DISPLACEMENT, SK_ENERGY,
    SK_TRACERS, SK_FLUX, SK_REMAP_DAMP_STATE, SK_CYCLE, SK_RECORD_REFERENCE, SK_INIT_VERTEX_VELOCITY,
    SK_STRENGTH_CONDITION, SK_LAPLACE_MASK, SK_STRESS_ENERGY, SK_COUNT
};

#ifdef __CUDACC__
// flux: a0 = pass (0 interior, 1 pad); remap: a0..a3 = remap, damping, ejecta drag, EOS switches
// blk is the block shape of the 2-D sweeps (cells, faces, vertices); the surface profile, the
// Laplacian mask, the tracer and the single-thread kernels use their own fixed shapes.
template <class R>
void launch_step_kernel(StepKernel k, const CtxT<R> &c, cudaStream_t s, dim3 blk, int a0 = 0, int a1 = 0,
                        int a2 = 0, int a3 = 0);
__global__ void k_gather(GatherBatch g, int mode, double *scratch);
void launch_aos_to_planes(const double *aos, void *base, bool f32, long long plane, int P, int nx, int ny, int nc,
                          cudaStream_t s);
void launch_planes_to_aos(const void *base, bool f32, double *aos, long long plane, int P, int nx, int ny, int nc,
                          cudaStream_t s);
void launch_count_nonfinite(const void *base, bool f32, long long n, unsigned long long *out, cudaStream_t s);
#endif

} // namespace salec
