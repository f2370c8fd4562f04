// Reverse (adjoint) sweeps of the mesh update, shared by the host driver (salec_runtime.cu) and
// the kernels (salec_adjoint.cu).
#pragma once
#include "salec_device.cuh"
#include "salec_kernels.h"

namespace salec {

// Forward state before the sweep (c), adjoint planes in the same layout (b), the step's time
// step, and the accumulators of the parameter gradients: theta[0] d/d cohesion (Yint0 = Ydam0),
// theta[1] d/d friction (Yfricint = Yfricdam).
struct AdjCtx {
    Ctx c;
    Fields b;
    double dt;
    double *theta;
};

// Reverse sweeps, numbered by the forward phase whose kernel they reverse.
enum AdjKernel { AK_VERTEX_MOMENTUM, AK_CELL_VELOCITY, AK_VOID_VERTICES, AK_GRADIENT, AK_STRESS, AK_ACCELERATION,
                 AK_DISPLACEMENT, AK_ENERGY, AK_FLUX, AK_REMAP_STATE };

#ifdef __CUDACC__
void launch_adjoint_kernel(AdjKernel k, const AdjCtx &a, cudaStream_t s);
// Reverse of a gather batch applied to the adjoint planes: for every entry dst <- op(src) the
// adjoint of dst moves to src (times op's derivative at the forward value of src, read from
// fwd_base), and dst's adjoint is cleared. entries[f] is the entry count of field f;
// scratch holds sum(entries) * ncomp_max doubles.
void launch_adjoint_gather(const GatherBatch &g, const int *entries, const void *const *adj_base,
                           double *scratch, cudaStream_t s);
// Seed of the surface-profile misfit: per interior column i, h_i = sum_j (1 - m_vof[0]) * e_pos[3]
// over the interior rows; J = 0.5 * sum_i w_i (h_i - target_i)^2 (target and weights per
// interior column); the adjoint of m_vof[0] receives -w_i (h_i - target_i) e_pos[3] and
// *J (one double on the device) the misfit.
void launch_profile_misfit(const Ctx &c, const Fields &b, const double *target, const double *weight, double *J,
                           double *h, cudaStream_t s);
#endif

} // namespace salec
