// Output files of a cycle, byte-identical to the reference's writers:
//   <dir>/vts/<prefix>.proc<rank>.<step>.vts         sale2d_write_vtk (src/write_vtk.c:189-298)
//   <dir>/vtp/<prefix>.tracer.proc<rank>.<step>.vtp  sale2d_write_vtp (src/write_vtk.c:354-480)
//   <dir>/txt/<prefix>.tracer.proc<rank>.<step>.txt  its text export (src/write_vtk.c:482-498)
// Each data array is FP32, zlib-compressed and base64-encoded with the VTK header of four
// int32 (1, raw bytes, raw bytes, compressed bytes), as src/io/output.c:117-392 writes it.
//
// The device packs every array (FP64 planes -> FP32 in the reference's point order, tracer
// compaction data) into one staging buffer and copies it to pinned host memory on the
// simulation's stream, so the snapshot is ordered with the cycle's kernels. A host worker
// thread then compresses the arrays in parallel and writes the files while the device goes
// on with the next cycles; the next output call, salec_gpu_output_wait() or
// salec_gpu_destroy() joins it.
#include "../../include/salec_gpu.h"
#include "salec_device.cuh"

#include <cuda_runtime.h>
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <vector>

using namespace salec;

struct salec_gpu;
int salec_internal_fail(int code, const char *msg);
int salec_internal_field_view(salec_gpu *h, const char *name, const void **base, int *f32, long long *plane,
                              int *pitch, int *nx, int *ny, int *nc);
cudaStream_t salec_internal_stream(salec_gpu *h);
Tracers salec_internal_tracers(salec_gpu *h);
Dims salec_internal_dims(salec_gpu *h);
void salec_internal_add_launches(salec_gpu *h, int n);
void *&salec_internal_output_slot(salec_gpu *h);

namespace {

constexpr int kMaxSeg = 32;
constexpr int kTracerCols = 14;   // matid tag gx gy vx vy den tem pre mpre mtem x y z

struct PackSeg {
    const void *base;  // double planes, or float planes when f32
    long long plane;   // doubles between components
    long long out;     // first float of this array in the staging buffer
    long long start;   // first point of this segment in the batch
    int pitch, nx, ny, nc, oc;   // oc = output components per point (3 for coordinates)
    int f32;
};

struct PackBatch {
    PackSeg seg[kMaxSeg];
    int nseg;
    long long total;   // points over all segments
};

// FP64 planes -> FP32 arrays, points x-fastest, components innermost (as field_var.data).
__global__ void k_pack_points(PackBatch b, float *out)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < b.total; t += stride) {
        int s = 0;
        while (s + 1 < b.nseg && t >= b.seg[s + 1].start) ++s;
        const PackSeg &g = b.seg[s];
        const long long q = t - g.start;
        const int x = (int)(q % g.nx), y = (int)(q / g.nx);
        const long long src = x + (long long)g.pitch * y;
        float *o = out + g.out + q * g.oc;
        if (g.f32) {
            const float *b = static_cast<const float *>(g.base);
            for (int c = 0; c < g.nc; ++c) o[c] = b[c * g.plane + src];
        } else {
            const double *b = static_cast<const double *>(g.base);
            for (int c = 0; c < g.nc; ++c) o[c] = __double2float_rn(b[c * g.plane + src]);
        }
        for (int c = g.nc; c < g.oc; ++c) o[c] = 0.0f;
    }
}

// One row of the tracer export per tracer slot; slots of deleted tracers get live = 0.
__device__ __forceinline__ float value_f32(const void *base, int f32, long long k)
{
    return f32 ? static_cast<const float *>(base)[k] : __double2float_rn(static_cast<const double *>(base)[k]);
}

__global__ void k_pack_tracers(Tracers T, const void *e_den, const void *e_tem, const void *e_pre, int f32, int pitch,
                               float *rows, int *live)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T.n) return;
    live[t] = T.alive[t] ? 1 : 0;
    float *r = rows + (long long)t * kTracerCols;
    const long long cell = T.cx[t] + (long long)pitch * T.cy[t];
    r[0] = 1.0f * T.matid[t];
    r[1] = 1.0f * T.tag[t];
    r[2] = 1.0f * T.gx[t];
    r[3] = 1.0f * T.gy[t];
    r[4] = __double2float_rn(T.vx[t]);
    r[5] = __double2float_rn(T.vy[t]);
    r[6] = T.alive[t] ? value_f32(e_den, f32, cell) : 0.0f;
    r[7] = T.alive[t] ? value_f32(e_tem, f32, cell) : 0.0f;
    r[8] = T.alive[t] ? value_f32(e_pre, f32, cell) : 0.0f;
    r[9] = T.mpre[t];
    r[10] = T.mtem[t];
    r[11] = __double2float_rn(T.x[t]);
    r[12] = __double2float_rn(T.y[t]);
    r[13] = 0.0f;
}

// ------------------------------------------------------------------ encoders (host)
// zlib stream fed in 16 KiB pieces with Z_NO_FLUSH and the last piece with Z_FINISH, at the
// default level: the same deflate input sequence as the reference's zlibcompress.
bool deflate_like_reference(const unsigned char *in, size_t n, std::vector<unsigned char> &out)
{
    const size_t piece = 16384;
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    if (deflateInit(&zs, Z_DEFAULT_COMPRESSION) != Z_OK) return false;
    out.clear();
    out.reserve(n / 2 + 64);
    unsigned char buf[16384];
    size_t pos = 0;
    int flush;
    do {
        const size_t take = std::min(piece, n - pos);
        zs.next_in = const_cast<unsigned char *>(in + pos);
        zs.avail_in = (uInt)take;
        pos += take;
        flush = pos == n ? Z_FINISH : Z_NO_FLUSH;
        do {
            zs.next_out = buf;
            zs.avail_out = sizeof(buf);
            if (deflate(&zs, flush) == Z_STREAM_ERROR) { deflateEnd(&zs); return false; }
            out.insert(out.end(), buf, buf + (sizeof(buf) - zs.avail_out));
        } while (zs.avail_out == 0);
    } while (flush != Z_FINISH);
    deflateEnd(&zs);
    return true;
}

void base64_append(const unsigned char *in, size_t n, std::string &s)
{
    static const char al[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    for (size_t i = 0; i < n; i += 3) {
        const unsigned a = in[i], b = i + 1 < n ? in[i + 1] : 0, c = i + 2 < n ? in[i + 2] : 0;
        s.push_back(al[a >> 2]);
        s.push_back(al[((a & 3) << 4) | (b >> 4)]);
        s.push_back(i + 1 < n ? al[((b & 15) << 2) | (c >> 6)] : '=');
        s.push_back(i + 2 < n ? al[c & 63] : '=');
    }
}

// One <DataArray> element of FP32 values in the reference's binary form.
bool data_array(const char *name, int ncomp, const float *v, size_t n, std::string &s)
{
    char head[256];
    snprintf(head, sizeof(head), "        <DataArray type=\"Float32\" Name=\"%s\" NumberOfComponents=\"%d\" format=\"binary\">\n",
             name, ncomp);
    s += head;
    const size_t raw = n * sizeof(float);
    std::vector<unsigned char> z;
    if (!deflate_like_reference(reinterpret_cast<const unsigned char *>(v), raw, z)) return false;
    int32_t hdr[4] = {1, (int32_t)raw, (int32_t)raw, (int32_t)z.size()};
    base64_append(reinterpret_cast<const unsigned char *>(hdr), sizeof(hdr), s);
    base64_append(z.data(), z.size(), s);
    s += "\n        </DataArray>\n";
    return true;
}

bool make_dir(const std::string &p)
{
    return mkdir(p.c_str(), 0755) == 0 || errno == EEXIST;
}

struct ArrayOut {
    std::string name;
    int ncomp;
    long long off, n;   // floats in the staging buffer
    int section;        // 0 point data, 1 cell data, 2 coordinates
};

struct Writer {
    std::thread worker;
    bool running = false;
    std::string error;
    float *dev = nullptr;
    size_t dev_floats = 0;
    float *host = nullptr;   // pinned
    size_t host_floats = 0;
    int *dev_live = nullptr, *host_live = nullptr;
    size_t live_n = 0, host_live_n = 0;
    cudaEvent_t done = nullptr;

    void join()
    {
        if (running) {
            worker.join();
            running = false;
        }
    }
    ~Writer()
    {
        join();
        if (dev) cudaFree(dev);
        if (host) cudaFreeHost(host);
        if (dev_live) cudaFree(dev_live);
        if (host_live) cudaFreeHost(host_live);
        if (done) cudaEventDestroy(done);
    }
};

struct Job {
    std::string dir, prefix;
    int rank, step, txt, nx, ny, vnx, vny;
    std::vector<ArrayOut> arrays;
    long long tracer_off;   // first float of the tracer rows
    int ntr;
    int device;
};

// Encode the arrays of the job in parallel; fills text[k] for arrays[k].
bool encode_all(const Job &J, const float *host, std::vector<std::string> &text)
{
    text.assign(J.arrays.size(), std::string());
    std::atomic<size_t> next{0};
    std::atomic<bool> ok{true};
    auto work = [&]() {
        for (size_t k = next++; k < J.arrays.size(); k = next++) {
            const ArrayOut &a = J.arrays[k];
            if (!data_array(a.name.c_str(), a.ncomp, host + a.off, (size_t)a.n, text[k])) ok = false;
        }
    };
    unsigned nt = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), (unsigned)J.arrays.size()));
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    return ok;
}

bool write_file(const std::string &path, const std::string &body, std::string &err)
{
    FILE *fp = fopen(path.c_str(), "w");
    if (!fp) { err = "cannot create " + path; return false; }
    const bool ok = fwrite(body.data(), 1, body.size(), fp) == body.size();
    if (fclose(fp) != 0 || !ok) { err = "cannot write " + path; return false; }
    return true;
}

void run_job(Writer *W, Job J)
{
    cudaSetDevice(J.device);
    if (cudaEventSynchronize(W->done) != cudaSuccess) { W->error = "output copy failed"; return; }
    const float *host = W->host;
    char name[512];

    // ---- structured grid
    std::vector<std::string> text;
    const std::vector<ArrayOut> &grid = J.arrays;
    if (!encode_all(J, host, text)) { W->error = "zlib compression failed"; return; }
    std::string s;
    char head[1024];
    // OUTPUT_GHT extents of a single rank: the first rank starts at 0, and the "last rank" branch of
    // the reference is an else-if that a single rank never reaches (src/write_vtk.c:211-236)
    snprintf(head, sizeof(head),
             "<?xml version=\"1.0\"?>\n"
             "<VTKFile type=\"StructuredGrid\" version=\"0.1\" compressor=\"vtkZLibDataCompressor\" byte_order=\"LittleEndian\">\n"
             "  <StructuredGrid WholeExtent=\"%d %d %d %d 0 0\">\n"
             "    <Piece Extent=\"%d %d %d %d 0 0\">\n",
             0, J.nx + 2, 0, J.ny + 2, 0, J.vnx - 1, 0, J.vny - 1);
    s += head;
    s += "      <PointData>\n";
    for (size_t k = 0; k < grid.size(); ++k) if (grid[k].section == 0) s += text[k];
    s += "      </PointData>\n      <CellData>\n";
    for (size_t k = 0; k < grid.size(); ++k) if (grid[k].section == 1) s += text[k];
    s += "      </CellData>\n      <Points>\n";
    for (size_t k = 0; k < grid.size(); ++k) if (grid[k].section == 2) s += text[k];
    s += "      </Points>\n    </Piece>\n  </StructuredGrid>\n</VTKFile>\n";
    make_dir(J.dir);
    make_dir(J.dir + "/vts");
    snprintf(name, sizeof(name), "%s/vts/%s.proc%04d.%04d.vts", J.dir.c_str(), J.prefix.c_str(), J.rank, J.step);
    if (!write_file(name, s, W->error)) return;

    // ---- tracers: live rows in slot order (the reference's list order)
    const float *rows = host + J.tracer_off;
    int nlive = 0;
    for (int t = 0; t < J.ntr; ++t) nlive += W->host_live[t];
    const bool dummy = nlive == 0;
    const int np = dummy ? 1 : nlive;
    std::vector<float> mat(np), tag(np), gx(np), gy(np), vel(2 * np), den(np), tem(np), pre(np), mpre(np),
        mtem(np), pos(3 * np);
    if (dummy) {
        mat[0] = tag[0] = gx[0] = gy[0] = -1.0f;
        vel[0] = vel[1] = den[0] = tem[0] = pre[0] = mpre[0] = mtem[0] = 0.0f;
        pos[0] = pos[1] = pos[2] = 0.0f;
    } else {
        int k = 0;
        for (int t = 0; t < J.ntr; ++t) {
            if (!W->host_live[t]) continue;
            const float *r = rows + (long long)t * kTracerCols;
            mat[k] = r[0]; tag[k] = r[1]; gx[k] = r[2]; gy[k] = r[3];
            vel[2 * k] = r[4]; vel[2 * k + 1] = r[5];
            den[k] = r[6]; tem[k] = r[7]; pre[k] = r[8]; mpre[k] = r[9]; mtem[k] = r[10];
            pos[3 * k] = r[11]; pos[3 * k + 1] = r[12]; pos[3 * k + 2] = r[13];
            ++k;
        }
    }
    std::string v;
    snprintf(head, sizeof(head),
             "<?xml version=\"1.0\"?>\n"
             "<VTKFile type=\"PolyData\" version=\"1.0\" compressor=\"vtkZLibDataCompressor\" byte_order=\"LittleEndian\">\n"
             "  <PolyData>\n"
             "    <Piece NumberOfPoints=\"%d\" NumberOfVerts=\"0\" NumberOfLines=\"0\" NumberOfStrips=\"0\" NumberOfPolys=\"0\">\n",
             np);
    v += head;
    v += "      <PointData>\n";
    bool ok = data_array("matid", 1, mat.data(), np, v) && data_array("tag", 1, tag.data(), np, v) &&
              data_array("gx", 1, gx.data(), np, v) && data_array("gy", 1, gy.data(), np, v) &&
              data_array("vel", 2, vel.data(), 2 * (size_t)np, v) && data_array("den", 1, den.data(), np, v) &&
              data_array("tem", 1, tem.data(), np, v) && data_array("pre", 1, pre.data(), np, v) &&
              data_array("mpre", 1, mpre.data(), np, v) && data_array("mtem", 1, mtem.data(), np, v);
    v += "      </PointData>\n      <Points>\n";
    ok = ok && data_array("coordinate", 3, pos.data(), 3 * (size_t)np, v);
    v += "      </Points>\n    </Piece>\n  </PolyData>\n</VTKFile>\n";
    if (!ok) { W->error = "zlib compression failed"; return; }
    make_dir(J.dir + "/vtp");
    snprintf(name, sizeof(name), "%s/vtp/%s.tracer.proc%04d.%04d.vtp", J.dir.c_str(), J.prefix.c_str(), J.rank, J.step);
    if (!write_file(name, v, W->error)) return;

    if (J.txt) {
        std::string t;
        char line[512];
        snprintf(line, sizeof(line), "   %d\n", np - (dummy ? 1 : 0));
        t += line;
        for (int k = 0; k < np; ++k) {
            snprintf(line, sizeof(line),
                     "%10f, %5f, %5f, %5f, %10.5e, %10.5e, %10.5e, %10.5e, %10.5e, %10.5e, %10.5e, %10.5e\n",
                     tag[k], mat[k], gx[k], gy[k], pos[3 * k], pos[3 * k + 1], vel[2 * k], vel[2 * k + 1], mpre[k],
                     mtem[k], pre[k], tem[k]);
            t += line;
        }
        make_dir(J.dir + "/txt");
        snprintf(name, sizeof(name), "%s/txt/%s.tracer.proc%04d.%04d.txt", J.dir.c_str(), J.prefix.c_str(), J.rank,
                 J.step);
        if (!write_file(name, t, W->error)) return;
    }
}

int finish(Writer *W)
{
    W->join();
    if (!W->error.empty()) {
        std::string e = W->error;
        W->error.clear();
        return salec_internal_fail(SALEC_ERR_STATE, ("output writer: " + e).c_str());
    }
    return SALEC_OK;
}

template <typename T>
int ensure(T *&p, size_t &have, size_t need, bool pinned)
{
    if (need <= have) return 0;
    if (p) { if (pinned) cudaFreeHost(p); else cudaFree(p); }
    p = nullptr;
    have = 0;
    cudaError_t e = pinned ? cudaMallocHost((void **)&p, need * sizeof(T)) : cudaMalloc((void **)&p, need * sizeof(T));
    if (e != cudaSuccess) return -1;
    have = need;
    return 0;
}

} // namespace

void salec_internal_output_release(void *&writer)
{
    delete static_cast<Writer *>(writer);
    writer = nullptr;
}

extern "C" int salec_gpu_write_output(salec_gpu *h, const char *dir, const char *prefix, int rank, int out_step,
                                      int flags)
{
    if (!h || !dir || !prefix || rank < 0 || out_step < 0)
        return salec_internal_fail(SALEC_ERR_ARG, "salec_gpu_write_output: null or negative argument");
    void *&slot = salec_internal_output_slot(h);
    if (!slot) slot = new Writer();
    Writer *W = static_cast<Writer *>(slot);
    int rc = finish(W);   // the previous output must be on disk before its buffers are reused
    if (rc) return rc;

    const Dims d = salec_internal_dims(h);
    Job J;
    J.dir = dir;
    J.prefix = prefix;
    J.rank = rank;
    J.step = out_step;
    J.txt = (flags & SALEC_OUT_TRACER_TXT) != 0;
    J.nx = d.enx - 4;
    J.ny = d.eny - 4;
    J.vnx = d.vnx;
    J.vny = d.vny;
    cudaGetDevice(&J.device);

    // arrays of sale2d_write_vtk in file order; e_vof is m_vof and e_eng is m_eng there
    struct Item { const char *out, *field; int section; };
    static const Item items[] = {
        {"v_vel", "v_vel", 0}, {"v_acc", "v_acc", 0}, {"v_gra", "v_bf", 0}, {"v_vof", "v_vof", 0},
        {"e_den", "e_den", 1}, {"e_pre", "e_pre", 1}, {"e_wpt", "e_wpt", 1}, {"e_vof", "m_vof", 1},
        {"e_csd", "e_csd", 1}, {"e_dam", "e_dam", 1}, {"e_tps", "e_tps", 1}, {"e_q", "e_q", 1},
        {"e_tem", "e_tem", 1}, {"e_eng", "m_eng", 1}, {"m_den", "m_den", 1}, {"e_ste2s", "e_ste2s", 1},
        {"e_sta2s", "e_sta2s", 1}, {"e_ste", "e_ste", 1}, {"e_strength", "e_strength", 1}, {"e_vib", "e_vib", 1},
        {"e_ejt", "e_ejt", 1}, {"e_cvs", "e_cvs", 1}, {"m_pty", "m_pty", 1}, {"coordinate", "v_pos", 2},
    };
    PackBatch b{};
    long long off = 0, pts = 0;
    for (const Item &it : items) {
        PackSeg &g = b.seg[b.nseg++];
        int nx, ny, nc;
        if ((rc = salec_internal_field_view(h, it.field, &g.base, &g.f32, &g.plane, &g.pitch, &nx, &ny, &nc)))
            return rc;
        g.nx = nx; g.ny = ny; g.nc = nc;
        g.oc = it.section == 2 ? 3 : nc;
        g.out = off;
        g.start = pts;
        ArrayOut a;
        a.name = it.out;
        a.ncomp = g.oc;
        a.off = off;
        a.n = (long long)nx * ny * g.oc;
        a.section = it.section;
        J.arrays.push_back(a);
        off += a.n;
        pts += (long long)nx * ny;
    }
    b.total = pts;
    const Tracers T = salec_internal_tracers(h);
    J.ntr = T.n;
    J.tracer_off = off;
    const size_t floats = (size_t)off + (size_t)T.n * kTracerCols;
    if (ensure(W->dev, W->dev_floats, floats, false) || ensure(W->host, W->host_floats, floats, true) ||
        ensure(W->dev_live, W->live_n, (size_t)std::max(T.n, 1), false) ||
        ensure(W->host_live, W->host_live_n, (size_t)std::max(T.n, 1), true))
        return salec_internal_fail(SALEC_ERR_ALLOC, "salec_gpu_write_output: staging allocation failed");
    if (!W->done && cudaEventCreateWithFlags(&W->done, cudaEventDisableTiming) != cudaSuccess)
        return salec_internal_fail(SALEC_ERR_CUDA, "salec_gpu_write_output: event creation failed");

    cudaStream_t s = salec_internal_stream(h);
    const int tb = 256;
    const int nb = (int)std::min<long long>((pts + tb - 1) / tb, 148LL * 16);
    k_pack_points<<<nb, tb, 0, s>>>(b, W->dev);
    int launches = 1;
    if (T.n > 0) {
        const void *den, *tem, *pre;
        long long pl;
        int pitch, nx, ny, nc, f32;
        salec_internal_field_view(h, "e_den", &den, &f32, &pl, &pitch, &nx, &ny, &nc);
        salec_internal_field_view(h, "e_tem", &tem, &f32, &pl, &pitch, &nx, &ny, &nc);
        salec_internal_field_view(h, "e_pre", &pre, &f32, &pl, &pitch, &nx, &ny, &nc);
        k_pack_tracers<<<(T.n + 127) / 128, 128, 0, s>>>(T, den, tem, pre, f32, pitch, W->dev + J.tracer_off,
                                                          W->dev_live);
        ++launches;
    }
    salec_internal_add_launches(h, launches);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(W->host, W->dev, floats * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && T.n > 0)
        e = cudaMemcpyAsync(W->host_live, W->dev_live, (size_t)T.n * sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaEventRecord(W->done, s);
    if (e != cudaSuccess)
        return salec_internal_fail(SALEC_ERR_CUDA, (std::string("salec_gpu_write_output: ") + cudaGetErrorString(e)).c_str());
    W->worker = std::thread(run_job, W, std::move(J));
    W->running = true;
    if (flags & SALEC_OUT_WAIT) return finish(W);
    return SALEC_OK;
}

extern "C" int salec_gpu_output_wait(salec_gpu *h)
{
    if (!h) return salec_internal_fail(SALEC_ERR_ARG, "null handle");
    void *&slot = salec_internal_output_slot(h);
    if (!slot) return SALEC_OK;
    return finish(static_cast<Writer *>(slot));
}
