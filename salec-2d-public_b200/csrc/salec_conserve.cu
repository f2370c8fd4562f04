// Conservation sums of a simulation's state (salec_gpu_conservation in include/salec_gpu.h).
//
// The reference has no such reduction; the quantities are the ones its conservative remap
// (src/advect.c:26-302) and momentum update (src/sale2d.c:930-1049) carry:
//   mass of material m      sum over interior cells of m_vof[m] * e_vol * m_den[m]
//   internal energy         sum over interior cells and materials of m_vof[m] * e_vol * m_eng[m]
//                           (m_eng is energy per volume of material)
//   momentum (r, z)         sum over active vertices of v_mass[0] * v_vel
//   kinetic energy          sum over active vertices of 0.5 * v_mass[0] * |v_vel|^2
// Every product is formed in FP64 (also in the mixed form, whose velocities and vertex masses are
// stored as float) and summed with Neumaier's compensated summation: each thread keeps a running
// sum and a running compensation over its grid-stride points; pairs are merged across the warp,
// the block and the grid by adding the other sum with the same compensated step and the other
// compensation plainly. The result is sum + compensation, within a few ulps of the exact sum for
// the sizes this library runs (the compensation's own rounding is second order).
#include "../../include/salec_gpu.h"
#include "salec_device.cuh"
#include "salec_kernels.h"

#include <cuda_runtime.h>

#include <string>

using namespace salec;

int salec_internal_fail(int code, const char *msg);
int salec_internal_field_view(salec_gpu *h, const char *name, const void **base, int *f32, long long *plane,
                              int *pitch, int *nx, int *ny, int *nc);
cudaStream_t salec_internal_stream(salec_gpu *h);
Dims salec_internal_dims(salec_gpu *h);
void salec_internal_add_launches(salec_gpu *h, int n);
void *&salec_internal_conserve_slot(salec_gpu *h);

namespace {

constexpr int kThreads = 256;
constexpr int kBlocks = 296;                   // two per SM of a B200
constexpr int kQ = 5 + SALEC_MAXMAT - 1;       // total mass, momentum r, z, internal, kinetic, mass per material

__device__ __forceinline__ void comp_add(double &s, double &c, double x)
{
    // Neumaier's step: the rounding error of s + x, recovered exactly, goes into c
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

__device__ __forceinline__ void comp_merge(double &s, double &c, double s2, double c2)
{
    comp_add(s, c, s2);
    c += c2;
}

struct Planes {
    const double *m_vof, *m_den, *m_eng, *e_vol;
    const void *v_vel, *v_mass;
    int f32;            // v_vel and v_mass are float planes (mixed form)
    long long PL;
    int P, enx, eny, vnx, vny, nmat;
};

template <class R>
__device__ __forceinline__ void vertex_terms(const Planes &q, long long p, double &mv, double &vx, double &vy)
{
    const R *vel = static_cast<const R *>(q.v_vel);
    const R *mass = static_cast<const R *>(q.v_mass);
    mv = (double)mass[p];
    vx = (double)vel[p];
    vy = (double)vel[p + q.PL];
}

__global__ void __launch_bounds__(kThreads) k_conserve_partial(Planes q, double *partials)
{
    double s[kQ], c[kQ];
#pragma unroll
    for (int k = 0; k < kQ; ++k) { s[k] = 0.0; c[k] = 0.0; }
    const long long stride = (long long)gridDim.x * blockDim.x;
    const int inx = q.enx - 4;
    const long long ncell = (long long)inx * (q.eny - 4);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < ncell; t += stride) {
        const int i = (int)(t % inx) + 2, j = (int)(t / inx) + 2;
        const long long p = i + (long long)q.P * j;
        const double vol = q.e_vol[p];
#pragma unroll
        for (int m = 1; m < SALEC_MAXMAT; ++m) {
            if (m >= q.nmat) break;
            const double vf = q.m_vof[p + m * q.PL] * vol;
            const double mass = vf * q.m_den[p + m * q.PL];
            comp_add(s[0], c[0], mass);
            comp_add(s[4 + m], c[4 + m], mass);
            comp_add(s[3], c[3], vf * q.m_eng[p + m * q.PL]);
        }
    }
    const int anx = q.vnx - 2;
    const long long nvert = (long long)anx * (q.vny - 2);
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nvert; t += stride) {
        const int i = (int)(t % anx) + 1, j = (int)(t / anx) + 1;
        const long long p = i + (long long)q.P * j;
        double mv, vx, vy;
        if (q.f32) vertex_terms<float>(q, p, mv, vx, vy);
        else vertex_terms<double>(q, p, mv, vx, vy);
        comp_add(s[1], c[1], mv * vx);
        comp_add(s[2], c[2], mv * vy);
        comp_add(s[4], c[4], 0.5 * mv * (vx * vx + vy * vy));
    }
    // warp, then block
    __shared__ double ws[kThreads / 32][kQ], wc[kThreads / 32][kQ];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kQ; ++k) {
        for (int o = 16; o > 0; o >>= 1) {
            const double s2 = __shfl_xor_sync(0xffffffffu, s[k], o);
            const double c2 = __shfl_xor_sync(0xffffffffu, c[k], o);
            comp_merge(s[k], c[k], s2, c2);
        }
        if (lane == 0) { ws[warp][k] = s[k]; wc[warp][k] = c[k]; }
    }
    __syncthreads();
    if (threadIdx.x < kQ) {
        const int k = threadIdx.x;
        double bs = ws[0][k], bc = wc[0][k];
        for (int w = 1; w < kThreads / 32; ++w) comp_merge(bs, bc, ws[w][k], wc[w][k]);
        partials[(blockIdx.x * kQ + k) * 2] = bs;
        partials[(blockIdx.x * kQ + k) * 2 + 1] = bc;
    }
}

// one thread per quantity, over the blocks in order
__global__ void k_conserve_final(int nblocks, const double *partials, double *out)
{
    const int k = threadIdx.x;
    if (k >= kQ) return;
    double s = 0.0, c = 0.0;
    for (int b = 0; b < nblocks; ++b) comp_merge(s, c, partials[(b * kQ + k) * 2], partials[(b * kQ + k) * 2 + 1]);
    out[k] = s + c;
}

} // namespace

extern "C" int salec_gpu_conservation(salec_gpu *h, double *out, int n)
{
    if (!h || !out) return salec_internal_fail(SALEC_ERR_ARG, "salec_gpu_conservation: null argument");
    const Dims d = salec_internal_dims(h);
    const int need = 5 + (d.nmat - 1);
    if (n < need)
        return salec_internal_fail(SALEC_ERR_ARG, ("salec_gpu_conservation: needs " + std::to_string(need) +
                                                   " doubles, got " + std::to_string(n)).c_str());
    Planes q{};
    const void *base;
    int f32, pitch, nx, ny, nc;
    long long plane;
    int rc = 0;
    rc |= salec_internal_field_view(h, "m_vof", &base, &f32, &plane, &pitch, &nx, &ny, &nc);
    q.m_vof = static_cast<const double *>(base);
    rc |= salec_internal_field_view(h, "m_den", &base, &f32, &plane, &pitch, &nx, &ny, &nc);
    q.m_den = static_cast<const double *>(base);
    rc |= salec_internal_field_view(h, "m_eng", &base, &f32, &plane, &pitch, &nx, &ny, &nc);
    q.m_eng = static_cast<const double *>(base);
    rc |= salec_internal_field_view(h, "e_vol", &base, &f32, &plane, &pitch, &nx, &ny, &nc);
    q.e_vol = static_cast<const double *>(base);
    rc |= salec_internal_field_view(h, "v_mass", &base, &f32, &plane, &pitch, &nx, &ny, &nc);
    q.v_mass = base;
    rc |= salec_internal_field_view(h, "v_vel", &base, &f32, &plane, &pitch, &nx, &ny, &nc);
    q.v_vel = base;
    if (rc) return salec_internal_fail(SALEC_ERR_STATE, "salec_gpu_conservation: field view");
    q.f32 = f32;
    q.PL = d.PL;
    q.P = d.P;
    q.enx = d.enx; q.eny = d.eny; q.vnx = d.vnx; q.vny = d.vny;
    q.nmat = d.nmat;
    cudaStream_t s = salec_internal_stream(h);
    void *&slot = salec_internal_conserve_slot(h);
    if (!slot) {
        // block partials (kBlocks x kQ pairs) and the kQ results, kept for the handle's lifetime
        if (cudaMalloc(&slot, sizeof(double) * (2 * kBlocks * kQ + kQ)) != cudaSuccess)
            return salec_internal_fail(SALEC_ERR_ALLOC, "salec_gpu_conservation: scratch");
    }
    double *partials = static_cast<double *>(slot);
    double *res = partials + 2 * kBlocks * kQ;
    k_conserve_partial<<<kBlocks, kThreads, 0, s>>>(q, partials);
    k_conserve_final<<<1, 32, 0, s>>>(kBlocks, partials, res);
    salec_internal_add_launches(h, 2);
    double host[kQ];
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, res, sizeof(host), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return salec_internal_fail(SALEC_ERR_CUDA, (std::string("salec_gpu_conservation: ") + cudaGetErrorString(e)).c_str());
    for (int k = 0; k < need; ++k) out[k] = host[k];
    return SALEC_OK;
}
