// CFL time step without any device allocation (salec_cfl_dt_noalloc in include/salec_gpu.h).
//
// For callers that cannot allocate device memory while they run the time step: a host code
// that gives all device memory to its own pool (a framework's caching allocator, or the
// reference-side driver once it has mapped its fields), or that must not pay cudaMalloc's
// device-wide synchronisation inside a per-cycle loop. The two-stage MIN reduction of
// calculate_dt (src/sale2d.c:1959-2016) keeps its per-block partial results in a file-scope
// device array instead of an allocation.
//
// Facts a caller must know:
//  - the scratch arrays hold SALEC_CFL_MAX_PARTIALS partial minima (64 KiB) and as many one-byte
//    NaN flags (8 KiB) on every device that loads the library, for the life of the process;
//  - one partial covers SALEC_CFL_CELLS_PER_BLOCK interior cells, so a call accepts at most
//    SALEC_CFL_MAX_PARTIALS * SALEC_CFL_CELLS_PER_BLOCK cells and rejects larger meshes;
//  - every call looks up the array's device address (cudaGetSymbolAddress) with the caller's
//    device current, so the address always belongs to the context the kernels run in (also
//    after a cudaDeviceReset, or under a context the caller made current itself). The lookup
//    is a host-side table access; the first one on a device also loads the library's device
//    code there, so make the first call on a device before any stream capture begins;
//  - every call shares the array: calls whose kernels overlap on the GPU (different streams,
//    no ordering between them) race on it and must be serialised by the caller. Each call
//    overwrites every partial it reads, so nothing has to be cleared between calls;
//  - NaN candidates (from a NaN velocity or sound speed) are treated as the reference's
//    sequential MIN treats them (src/mpi_vec/mpi_vec_types.h:262, folded in traversal order
//    from 1.1 * dt_prev): the result is the MIN of the candidates after the last NaN, or NaN
//    when the NaN is the last candidate, as in the step's own CFL phase. Blocks cover
//    consecutive runs of the traversal order, so each block records whether it saw a NaN and
//    the MIN of its candidates after its own last NaN, and the final stage starts from the last
//    block with a NaN.
#include "../../include/salec_gpu.h"
#include "salec_device.cuh"

#include <cuda_runtime.h>

#include <string>

#define SALEC_CFL_THREADS 256
#define SALEC_CFL_CELLS_PER_THREAD 16
#define SALEC_CFL_CELLS_PER_BLOCK (SALEC_CFL_THREADS * SALEC_CFL_CELLS_PER_THREAD)
#define SALEC_CFL_MAX_PARTIALS 8192

int salec_internal_fail(int code, const char *msg);

namespace {

static __device__ __align__(256) unsigned long long g_cfl_partials[SALEC_CFL_MAX_PARTIALS];
static __device__ __align__(256) unsigned char g_cfl_nanflag[SALEC_CFL_MAX_PARTIALS];

__device__ __forceinline__ unsigned long long block_min(unsigned long long v)
{
    __shared__ unsigned long long wmin[SALEC_CFL_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < SALEC_CFL_THREADS / 32 ? wmin[threadIdx.x] : ~0ULL;
        for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

__device__ __forceinline__ long long block_max(long long v)
{
    __shared__ long long wmax[SALEC_CFL_THREADS / 32];
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < SALEC_CFL_THREADS / 32 ? wmax[threadIdx.x] : -1LL;
        for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

// CFL candidate of interior cell t (row-major over the interior, the reference's traversal
// order), or false for a pure-vacuum cell: calculate_dt (src/sale2d.c:1999-2002)
__device__ __forceinline__ bool cfl_cell(long long t, int nx, const double *vr, const double *vz, const double *csd,
                                         const double *sr, const double *sz, const double *vof0, double &cand)
{
    const int pitch = nx + 4;
    const int i = (int)(t % nx) + 2, j = (int)(t / nx) + 2;
    const long long p = i + (long long)pitch * j;
    if (vof0[p] > 1.0 - SALEC_TOLVOF) return false;
    const double c = csd[p];
    const double dt_r = 1.0 * sr[p] / (fabs(vr[p]) + c);
    const double dt_z = 1.0 * sz[p] / (fabs(vz[p]) + c);
    cand = SALEC_DTF * salec::dmin(dt_r, dt_z);
    return true;
}

// stage 1: per block, whether it saw a NaN candidate, and the MIN of its candidates after its
// last NaN (all of them when it saw none)
__global__ void __launch_bounds__(SALEC_CFL_THREADS)
k_cfl_partials(int nx, int ny, const double *vr, const double *vz, const double *csd, const double *sr,
               const double *sz, const double *vof0, unsigned long long *partials, unsigned char *nanflag)
{
    const long long ncell = (long long)nx * ny;
    const long long t0 = (long long)blockIdx.x * SALEC_CFL_CELLS_PER_BLOCK;
    unsigned long long best = ~0ULL;
    long long last_nan = -1;
    for (int k = 0; k < SALEC_CFL_CELLS_PER_THREAD; ++k) {
        const long long t = t0 + (long long)k * SALEC_CFL_THREADS + threadIdx.x;
        if (t >= ncell) break;
        double cand;
        if (!cfl_cell(t, nx, vr, vz, csd, sr, sz, vof0, cand)) continue;
        if (cand == cand) best = min(best, salec::ord_encode(cand));
        else last_nan = t;
    }
    last_nan = block_max(last_nan);
    __shared__ long long s_last;
    if (threadIdx.x == 0) s_last = last_nan;
    __syncthreads();
    last_nan = s_last;
    if (last_nan >= 0) {   // rare: recount the candidates after the block's last NaN
        best = ~0ULL;
        for (int k = 0; k < SALEC_CFL_CELLS_PER_THREAD; ++k) {
            const long long t = t0 + (long long)k * SALEC_CFL_THREADS + threadIdx.x;
            if (t >= ncell) break;
            double cand;
            if (t > last_nan && cfl_cell(t, nx, vr, vz, csd, sr, sz, vof0, cand)) best = min(best, salec::ord_encode(cand));
        }
    }
    __syncthreads();
    best = block_min(best);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = best;
        nanflag[blockIdx.x] = last_nan >= 0 ? 1 : 0;
    }
}

// stage 2: the MIN from the last block with a NaN on (from 1.1 * dt_prev and every block when
// there is none), NaN when nothing follows the last NaN; then Min(max_dt, .)
__global__ void __launch_bounds__(SALEC_CFL_THREADS)
k_cfl_final(int nblocks, double dt_prev, double max_dt, const unsigned long long *partials,
            const unsigned char *nanflag, double *dt_out)
{
    long long lastb = -1;
    for (int b = threadIdx.x; b < nblocks; b += SALEC_CFL_THREADS)
        if (nanflag[b]) lastb = b;
    lastb = block_max(lastb);
    __shared__ long long s_lastb;
    if (threadIdx.x == 0) s_lastb = lastb;
    __syncthreads();
    lastb = s_lastb;
    unsigned long long best = (threadIdx.x == 0 && lastb < 0) ? salec::ord_encode(1.1 * dt_prev) : ~0ULL;
    for (int b = threadIdx.x; b < nblocks; b += SALEC_CFL_THREADS)
        if (b >= lastb) best = min(best, partials[b]);
    __syncthreads();
    best = block_min(best);
    if (threadIdx.x == 0) {
        const double r = best == ~0ULL ? __longlong_as_double(0x7ff8000000000000LL) : salec::ord_decode(best);
        *dt_out = salec::dmin(max_dt, r);
    }
}

} // namespace

extern "C" int salec_cfl_dt_noalloc(int nx, int ny, const double *vel_r, const double *vel_z, const double *csd,
                                    const double *scale_r, const double *scale_z, const double *vof_vacuum,
                                    double dt_prev, double max_dt, double *dt_out, void *stream)
{
    if (nx < 1 || ny < 1 || !vel_r || !vel_z || !csd || !scale_r || !scale_z || !vof_vacuum || !dt_out)
        return salec_internal_fail(SALEC_ERR_ARG, "salec_cfl_dt_noalloc: empty mesh or null pointer");
    const long long ncell = (long long)nx * ny;
    const long long limit = (long long)SALEC_CFL_MAX_PARTIALS * SALEC_CFL_CELLS_PER_BLOCK;
    if (ncell > limit)
        return salec_internal_fail(SALEC_ERR_ARG, ("salec_cfl_dt_noalloc: " + std::to_string(ncell) +
                                                   " interior cells exceed its limit of " + std::to_string(limit))
                                                      .c_str());
    // the scratch array's address in the current device's context; the host-side name
    // g_cfl_partials is a stand-in that no kernel may be given
    void *addr = nullptr, *flag_addr = nullptr;
    cudaError_t le = cudaGetSymbolAddress(&addr, g_cfl_partials);
    if (le == cudaSuccess) le = cudaGetSymbolAddress(&flag_addr, g_cfl_nanflag);
    if (le != cudaSuccess || !addr || !flag_addr)
        return salec_internal_fail(SALEC_ERR_CUDA, (std::string("salec_cfl_dt_noalloc: cudaGetSymbolAddress: ") +
                                                    cudaGetErrorString(le)).c_str());
    unsigned long long *partials = static_cast<unsigned long long *>(addr);
    unsigned char *nanflag = static_cast<unsigned char *>(flag_addr);
    const int nblocks = (int)((ncell + SALEC_CFL_CELLS_PER_BLOCK - 1) / SALEC_CFL_CELLS_PER_BLOCK);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_cfl_partials<<<nblocks, SALEC_CFL_THREADS, 0, s>>>(nx, ny, vel_r, vel_z, csd, scale_r, scale_z, vof_vacuum,
                                                       partials, nanflag);
    k_cfl_final<<<1, SALEC_CFL_THREADS, 0, s>>>(nblocks, dt_prev, max_dt, partials, nanflag, dt_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return salec_internal_fail(SALEC_ERR_CUDA, (std::string("salec_cfl_dt_noalloc: launch: ") + cudaGetErrorString(e)).c_str());
    return SALEC_OK;
}
