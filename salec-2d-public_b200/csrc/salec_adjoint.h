// Reverse (adjoint) sweeps of the mesh update, shared by the host driver (salec_runtime.cu) and
// the kernels (salec_adjoint.cu).
#pragma once
#include "salec_device.cuh"
#include "salec_kernels.h"

namespace salec {

// Forward state before the sweep (c; its scalar block holds the cycle's time step), adjoint
// planes in the same layout (b), and the accumulators of the parameter gradients: d/d Yint0,
// Yfricint, Ydam0, Yfricdam of material 1.
struct AdjCtx {
    Ctx c;
    Fields b;
    double *theta;
    double *scr;   // per-cell corner scratch, 16 planes of the pool's plane stride
};

// One field of a list copy: its bytes at `field` and their place `off` in a log record.
struct CopySeg {
    char *field;
    unsigned long long off, bytes;
};

// Reverse sweeps, numbered by the forward phase whose kernel they reverse.
enum AdjKernel { AK_VERTEX_MOMENTUM, AK_CELL_VELOCITY, AK_VOID_VERTICES, AK_GRADIENT, AK_STRESS, AK_ACCELERATION,
                 AK_DISPLACEMENT, AK_ENERGY, AK_FLUX, AK_REMAP_STATE };

#ifdef __CUDACC__
void launch_adjoint_kernel(AdjKernel k, const AdjCtx &a, cudaStream_t s);
// Reverse of a gather batch applied to the adjoint planes: for every entry dst <- op(src) the
// adjoint of dst moves to src (times op's derivative at the forward value of src, read from
// fwd_base), and dst's adjoint is cleared. entries[f] is the entry count of field f; a batch
// the forward runs in one pass is reversed in one launch, a two-pass batch in three stages
// through scratch (sum(entries) * ncomp_max doubles).
void launch_adjoint_gather(const GatherBatch &g, const int *entries, const void *const *adj_base,
                           double *scratch, bool two_pass, cudaStream_t s);
// Seed of the surface-profile misfit: per interior column i, h_i = sum_j (1 - m_vof[0]) * e_pos[3]
// over the interior rows; J = 0.5 * sum_i w_i (h_i - target_i)^2 (target and weights per
// interior column); the adjoint of m_vof[0] receives -w_i (h_i - target_i) e_pos[3] and
// *J (one double on the device) the misfit.
// Copies a list of fields into (save) or out of a log record at base + slot * stride (slot read on
// the device, so that one captured graph walks the records of a segment; a null slot is record
// 0). Fields and record offsets are 16-byte aligned.
void launch_list_copy(const CopySeg *segs, int nseg, unsigned long long max_bytes, char *base, const long long *slot,
                      unsigned long long stride, bool save, cudaStream_t s);
// *slot = value, or *slot += delta
void launch_slot_set(long long *slot, long long value, cudaStream_t s);
void launch_slot_add(long long *slot, long long delta, cudaStream_t s);
void launch_profile_misfit(const Ctx &c, const Fields &b, const double *target, const double *weight, double *J,
                           double *h, cudaStream_t s);
#endif

} // namespace salec
