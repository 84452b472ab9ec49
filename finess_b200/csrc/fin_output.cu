// Frame files and conservation totals from device state: the formats of the
// reference's lib/2d/Output.cpp (q%04d.dat, a%04d.dat), ConSoln.cpp
// (conservation.dat) and their reader for a restart.
//
// The reference writes a frame with iostreams on the host thread that runs
// the solver, one value at a time, after the whole state is on the host.
// Here the state's interior is reordered on the device into the files'
// order, copied to pinned host memory on a side stream while the solver's
// stream goes on with the next steps, and formatted by several host threads
// into fixed 25-byte lines ("%24.16e\n", the same C library conversion that
// libstdc++'s num_put uses for setprecision(16) << scientific with setw(24)).
#include "fin_output.h"
#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "finess_b200.h"

namespace fin {
namespace io {

namespace {

// out[c][j][i] = q[c*plane + i*my + j] over the interior: 32 x 32 tiles
// through shared memory so both sides are coalesced.
__global__ void k_frame_order(const double* __restrict__ q, size_t plane, int mx, int my, double* __restrict__ out)
{
    __shared__ double tile[32][33];
    const int c = blockIdx.z;
    const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
    const double* qc = q + size_t(c) * plane;
    double* oc = out + size_t(c) * mx * my;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, j = j0 + threadIdx.x;
        if (i < mx && j < my) tile[r][threadIdx.x] = qc[size_t(i) * my + j];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int j = j0 + r, i = i0 + threadIdx.x;
        if (i < mx && j < my) oc[size_t(j) * mx + i] = tile[threadIdx.x][r];
    }
}

// The inverse: q[c*plane + i*my + j] = in[c][j][i].
__global__ void k_frame_unorder(const double* __restrict__ in, size_t plane, int mx, int my, double* __restrict__ q)
{
    __shared__ double tile[32][33];
    const int c = blockIdx.z;
    const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
    const double* ic = in + size_t(c) * mx * my;
    double* qc = q + size_t(c) * plane;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int j = j0 + r, i = i0 + threadIdx.x;
        if (i < mx && j < my) tile[r][threadIdx.x] = ic[size_t(j) * mx + i];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, j = j0 + threadIdx.x;
        if (i < mx && j < my) qc[size_t(i) * my + j] = tile[threadIdx.x][r];
    }
}

// Neumaier's compensated sum: (s, c) += x.
__device__ __forceinline__ void neumaier(double& s, double& c, double x)
{
    const double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

// Per (component, chunk): compensated sum of dxdy * q over the chunk's cells
// (a fixed partition), reduced across the CTA in a fixed tree order.
__global__ void __launch_bounds__(256) k_totals_partial(const double* __restrict__ q, size_t plane, size_t n,
                                                        double dxdy, double* __restrict__ part)
{
    __shared__ double ss[256], sc[256];
    const int c = blockIdx.y, k = blockIdx.x;
    const size_t b = n * k / NCHUNK, e = n * (k + 1) / NCHUNK;
    const double* qc = q + size_t(c) * plane;
    double s = 0.0, cc = 0.0;
    for (size_t g = b + threadIdx.x; g < e; g += 256) neumaier(s, cc, dxdy * qc[g]);
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = cc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            double a = ss[threadIdx.x], ac = sc[threadIdx.x] + sc[threadIdx.x + o];
            neumaier(a, ac, ss[threadIdx.x + o]);
            ss[threadIdx.x] = a;
            sc[threadIdx.x] = ac;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * (size_t(c) * NCHUNK + k)] = ss[0];
        part[2 * (size_t(c) * NCHUNK + k) + 1] = sc[0];
    }
}

// One thread per component: the chunks' pairs in order.
__global__ void k_totals_final(const double* __restrict__ part, int ncomp, double* __restrict__ out)
{
    const int c = threadIdx.x;
    if (c >= ncomp) return;
    double s = 0.0, cc = 0.0;
    for (int k = 0; k < NCHUNK; k++) {
        neumaier(s, cc, part[2 * (size_t(c) * NCHUNK + k)]);
        cc += part[2 * (size_t(c) * NCHUNK + k) + 1];
    }
    out[c] = s + cc;
}

inline void format_one(double v, char* dst)
{
    char b[40];
    std::snprintf(b, sizeof(b), "%24.16e\n", v);
    std::memcpy(dst, b, RECORD);
}

template <class F>
void parallel_for(size_t n, int nthreads, F&& f)
{
    const int nt = std::max(1, std::min<int>(nthreads, int((n + 65535) / 65536)));
    if (nt == 1) {
        f(size_t(0), n);
        return;
    }
    std::vector<std::thread> ts;
    for (int t = 0; t < nt; t++) {
        const size_t b = n * t / nt, e = n * (t + 1) / nt;
        ts.emplace_back([&f, b, e] { f(b, e); });
    }
    for (std::thread& t : ts) t.join();
}

int host_threads()
{
    const unsigned h = std::thread::hardware_concurrency();
    return int(std::min(16u, std::max(1u, h)));
}

// Header line and n values to path, formatted in chunks.
int write_frame_file(const std::string& path, double t, const double* v, size_t n, std::string* err)
{
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) {
        *err = "cannot open " + path + ": " + std::strerror(errno);
        return FIN_ERR_ARG;
    }
    char head[RECORD + 1];
    format_one(t, head);
    bool ok = std::fwrite(head, 1, RECORD, f) == size_t(RECORD);
    const size_t chunk = size_t(1) << 22;   // 4M values, 100 MB of text per pass
    std::vector<char> buf(std::min(n, chunk) * RECORD + 1);
    for (size_t b = 0; b < n && ok; b += chunk) {
        const size_t m = std::min(chunk, n - b);
        format_records(v + b, m, buf.data(), host_threads());
        ok = std::fwrite(buf.data(), 1, m * RECORD, f) == m * RECORD;
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        *err = "write failed: " + path;
        return FIN_ERR_ARG;
    }
    return FIN_OK;
}

}  // namespace

void format_records(const double* v, size_t n, char* out, int nthreads)
{
    parallel_for(n, nthreads, [&](size_t b, size_t e) {
        for (size_t k = b; k < e; k++) format_one(v[k], out + k * RECORD);
    });
    out[n * RECORD] = '\0';
}

bool parse_records(const char* text, size_t len, double* v, size_t n, int nthreads)
{
    bool fixed = len >= n * RECORD;
    for (size_t k = 0; fixed && k < n; k += std::max<size_t>(1, n / 64)) fixed = text[k * RECORD + RECORD - 1] == '\n';
    if (fixed && n > 0) fixed = text[(n - 1) * RECORD + RECORD - 1] == '\n';
    if (fixed) {
        std::atomic<bool> ok(true);
        parallel_for(n, nthreads, [&](size_t b, size_t e) {
            char field[RECORD];
            for (size_t k = b; k < e; k++) {
                std::memcpy(field, text + k * RECORD, RECORD - 1);
                field[RECORD - 1] = '\0';
                char* end = nullptr;
                v[k] = std::strtod(field, &end);
                if (end == field) {
                    ok.store(false);
                    return;
                }
            }
        });
        if (ok.load()) return true;
    }
    // general layout: whitespace-separated numbers
    std::string s(text, len);
    const char* p = s.c_str();
    for (size_t k = 0; k < n; k++) {
        char* end = nullptr;
        v[k] = std::strtod(p, &end);
        if (end == p) return false;
        p = end;
    }
    return true;
}

FrameWriter::~FrameWriter()
{
    wait();
    if (d_stage_) cudaFree(d_stage_);
    if (h_stage_) cudaFreeHost(h_stage_);
    if (ready_) cudaEventDestroy(ready_);
    if (copied_) cudaEventDestroy(copied_);
    if (side_) cudaStreamDestroy(side_);
}

int FrameWriter::ensure(size_t n)
{
    cudaError_t e;
    if (!side_ && (e = cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking)) != cudaSuccess) {
        err_ = std::string("stream: ") + cudaGetErrorString(e);
        return FIN_ERR_CUDA;
    }
    if (!ready_ && (e = cudaEventCreateWithFlags(&ready_, cudaEventDisableTiming)) != cudaSuccess) {
        err_ = std::string("event: ") + cudaGetErrorString(e);
        return FIN_ERR_CUDA;
    }
    if (!copied_ && (e = cudaEventCreateWithFlags(&copied_, cudaEventDisableTiming)) != cudaSuccess) {
        err_ = std::string("event: ") + cudaGetErrorString(e);
        return FIN_ERR_CUDA;
    }
    if (n <= cap_) return FIN_OK;
    if (d_stage_) cudaFree(d_stage_);
    if (h_stage_) cudaFreeHost(h_stage_);
    d_stage_ = nullptr;
    h_stage_ = nullptr;
    cap_ = 0;
    if ((e = cudaMalloc(&d_stage_, n * sizeof(double))) != cudaSuccess ||
        (e = cudaMallocHost(&h_stage_, n * sizeof(double))) != cudaSuccess) {
        err_ = std::string("frame staging: ") + cudaGetErrorString(e);
        return FIN_ERR_CUDA;
    }
    cap_ = n;
    return FIN_OK;
}

int FrameWriter::start(cudaStream_t stream, const double* q, int ncomp, const double* aux, int naux, size_t plane,
                       int mx, int my, double t, const std::string& qpath, const std::string& apath)
{
    int rc = wait();
    if (rc) return rc;
    const size_t per = size_t(mx) * my;
    if ((rc = ensure(per * size_t(ncomp + naux) + 1))) return rc;
    const dim3 blk(32, 8);
    cudaError_t e = cudaSuccess;
    if (ncomp > 0) {
        k_frame_order<<<dim3((my + 31) / 32, (mx + 31) / 32, ncomp), blk, 0, stream>>>(q, plane, mx, my, d_stage_);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && naux > 0) {
        if (aux) {
            k_frame_order<<<dim3((my + 31) / 32, (mx + 31) / 32, naux), blk, 0, stream>>>(aux, plane, mx, my,
                                                                                         d_stage_ + per * ncomp);
            e = cudaGetLastError();
        } else {   // no aux planes held: zeros
            e = cudaMemsetAsync(d_stage_ + per * ncomp, 0, per * naux * sizeof(double), stream);
        }
    }
    if (e == cudaSuccess) e = cudaEventRecord(ready_, stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(side_, ready_, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_stage_, d_stage_, per * size_t(ncomp + naux) * sizeof(double), cudaMemcpyDeviceToHost,
                            side_);
    if (e == cudaSuccess) e = cudaEventRecord(copied_, side_);
    if (e != cudaSuccess) {
        err_ = std::string("frame copy: ") + cudaGetErrorString(e);
        return FIN_ERR_CUDA;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    status_ = FIN_OK;
    err_.clear();
    const double* hq = h_stage_;
    const double* ha = h_stage_ + per * ncomp;
    cudaEvent_t copied = copied_;
    worker_ = std::thread([this, dev, copied, hq, ha, per, ncomp, naux, t, qpath, apath] {
        cudaSetDevice(dev);
        const cudaError_t w = cudaEventSynchronize(copied);
        if (w != cudaSuccess) {
            err_ = std::string("frame copy: ") + cudaGetErrorString(w);
            status_ = FIN_ERR_CUDA;
            return;
        }
        std::string m;
        int r = write_frame_file(qpath, t, hq, per * ncomp, &m);
        if (!r) r = write_frame_file(apath, t, ha, per * naux, &m);
        if (r) {
            err_ = m;
            status_ = r;
        }
    });
    return FIN_OK;
}

int FrameWriter::wait()
{
    if (worker_.joinable()) worker_.join();
    const int rc = status_;
    status_ = FIN_OK;
    return rc;
}

int append_conservation(const std::string& path, double t, const double* totals, int ncomp)
{
    FILE* f = std::fopen(path.c_str(), t == 0 ? "w" : "a");
    if (!f) return FIN_ERR_ARG;
    std::fprintf(f, "%24.16e ", t);
    for (int m = 0; m < ncomp; m++) {
        const double v = std::fabs(totals[m]) < 1.0e-99 ? 0.0 : totals[m];
        std::fprintf(f, "%24.16e ", v);
    }
    std::fprintf(f, "\n");
    return std::fclose(f) == 0 ? FIN_OK : FIN_ERR_ARG;
}

void launch_totals(cudaStream_t stream, const double* q, int ncomp, size_t plane, size_t n, double dxdy,
                   double* d_scratch, double* d_out)
{
    k_totals_partial<<<dim3(NCHUNK, ncomp), 256, 0, stream>>>(q, plane, n, dxdy, d_scratch);
    k_totals_final<<<1, 32, 0, stream>>>(d_scratch, ncomp, d_out);
}

int read_frame(const std::string& path, cudaStream_t stream, double* q, int ncomp, size_t plane, int mx, int my,
               double* d_stage, double* t, std::string* err)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        *err = "cannot open " + path + ": " + std::strerror(errno);
        return FIN_ERR_ARG;
    }
    std::fseek(f, 0, SEEK_END);
    const long len = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<char> text(size_t(std::max(0L, len)) + 1);
    const size_t got = std::fread(text.data(), 1, size_t(std::max(0L, len)), f);
    std::fclose(f);
    text[got] = '\0';
    char* end = nullptr;
    const double tt = std::strtod(text.data(), &end);
    if (end == text.data()) {
        *err = path + ": no time on the first line";
        return FIN_ERR_ARG;
    }
    const char* nl = std::strchr(end, '\n');
    const char* body = nl ? nl + 1 : end;
    const size_t n = size_t(mx) * my * ncomp;
    std::vector<double> h(n);
    if (!parse_records(body, got - size_t(body - text.data()), h.data(), n, host_threads())) {
        *err = path + ": fewer values than the grid holds";
        return FIN_ERR_ARG;
    }
    cudaError_t e = cudaMemcpyAsync(d_stage, h.data(), n * sizeof(double), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        k_frame_unorder<<<dim3((mx + 31) / 32, (my + 31) / 32, ncomp), dim3(32, 8), 0, stream>>>(d_stage, plane, mx,
                                                                                               my, q);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        *err = std::string("frame upload: ") + cudaGetErrorString(e);
        return FIN_ERR_CUDA;
    }
    *t = tt;
    return FIN_OK;
}

}  // namespace io
}  // namespace fin
