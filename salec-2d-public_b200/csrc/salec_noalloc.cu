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
//  - the scratch array holds SALEC_CFL_MAX_PARTIALS partial minima (64 KiB) on every device that
//    loads the library, for the life of the process;
//  - one partial covers SALEC_CFL_CELLS_PER_BLOCK interior cells, so a call accepts at most
//    SALEC_CFL_MAX_PARTIALS * SALEC_CFL_CELLS_PER_BLOCK cells and rejects larger meshes;
//  - the first call on a device looks up the array's device address (cudaGetSymbolAddress) with
//    that device current; make that first call before any stream capture begins;
//  - every call shares the array: calls whose kernels overlap on the GPU (different streams,
//    no ordering between them) race on it and must be serialised by the caller. Each call
//    overwrites every partial it reads, so nothing has to be cleared between calls.
#include "../../include/salec_gpu.h"
#include "salec_device.cuh"

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#define SALEC_CFL_THREADS 256
#define SALEC_CFL_CELLS_PER_THREAD 16
#define SALEC_CFL_CELLS_PER_BLOCK (SALEC_CFL_THREADS * SALEC_CFL_CELLS_PER_THREAD)
#define SALEC_CFL_MAX_PARTIALS 8192
#define SALEC_CFL_MAX_DEVICES 64

int salec_internal_fail(int code, const char *msg);

namespace {

static __device__ __align__(256) unsigned long long g_cfl_partials[SALEC_CFL_MAX_PARTIALS];

std::mutex g_cfl_mutex;
unsigned long long *g_cfl_addr[SALEC_CFL_MAX_DEVICES] = {nullptr};

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

// stage 1: one partial MIN per block over its range of interior cells
__global__ void __launch_bounds__(SALEC_CFL_THREADS)
k_cfl_partials(int nx, int ny, const double *vr, const double *vz, const double *csd, const double *sr,
               const double *sz, const double *vof0, unsigned long long *partials)
{
    const long long ncell = (long long)nx * ny;
    const int pitch = nx + 4;
    unsigned long long best = ~0ULL;
    for (int k = 0; k < SALEC_CFL_CELLS_PER_THREAD; ++k) {
        const long long t = (long long)blockIdx.x * SALEC_CFL_CELLS_PER_BLOCK + (long long)k * SALEC_CFL_THREADS + threadIdx.x;
        if (t >= ncell) break;
        const int i = (int)(t % nx) + 2, j = (int)(t / nx) + 2;
        const long long p = i + (long long)pitch * j;
        if (vof0[p] > 1.0 - SALEC_TOLVOF) continue;
        const double c = csd[p];
        const double dt_r = 1.0 * sr[p] / (fabs(vr[p]) + c);
        const double dt_z = 1.0 * sz[p] / (fabs(vz[p]) + c);
        best = min(best, salec::ord_encode(SALEC_DTF * salec::dmin(dt_r, dt_z)));
    }
    best = block_min(best);
    if (threadIdx.x == 0) partials[blockIdx.x] = best;
}

// stage 2: MIN of the partials and of 1.1 * dt_prev, then Min(max_dt, .)
__global__ void __launch_bounds__(SALEC_CFL_THREADS)
k_cfl_final(int nblocks, double dt_prev, double max_dt, const unsigned long long *partials, double *dt_out)
{
    unsigned long long best = threadIdx.x == 0 ? salec::ord_encode(1.1 * dt_prev) : ~0ULL;
    for (int b = threadIdx.x; b < nblocks; b += SALEC_CFL_THREADS) best = min(best, partials[b]);
    best = block_min(best);
    if (threadIdx.x == 0) *dt_out = salec::dmin(max_dt, salec::ord_decode(best));
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
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= SALEC_CFL_MAX_DEVICES)
        return salec_internal_fail(SALEC_ERR_CUDA, "salec_cfl_dt_noalloc: no usable current device");
    unsigned long long *partials = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_cfl_mutex);
        if (!g_cfl_addr[dev]) {
            void *addr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&addr, g_cfl_partials);
            if (e != cudaSuccess)
                return salec_internal_fail(SALEC_ERR_CUDA, (std::string("salec_cfl_dt_noalloc: cudaGetSymbolAddress: ") +
                                                            cudaGetErrorString(e)).c_str());
            g_cfl_addr[dev] = static_cast<unsigned long long *>(addr);
        }
        partials = g_cfl_addr[dev];
    }
    const int nblocks = (int)((ncell + SALEC_CFL_CELLS_PER_BLOCK - 1) / SALEC_CFL_CELLS_PER_BLOCK);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    k_cfl_partials<<<nblocks, SALEC_CFL_THREADS, 0, s>>>(nx, ny, vel_r, vel_z, csd, scale_r, scale_z, vof_vacuum,
                                                       partials);
    k_cfl_final<<<1, SALEC_CFL_THREADS, 0, s>>>(nblocks, dt_prev, max_dt, partials, dt_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return salec_internal_fail(SALEC_ERR_CUDA, (std::string("salec_cfl_dt_noalloc: launch: ") + cudaGetErrorString(e)).c_str());
    return SALEC_OK;
}
