// Snapshots, restart and the energy-split diagnostic of a context's
// instances (include/rh3t.h rh3t_snapshot, rh3t_snapshot_wait, rh3t_restart,
// rh3t_energy_split).
//
// RH3TBIN1 (io.rs:1-24, the format of the reference's Python tooling):
// header  [8]u8 "RH3TBIN1" | u32 version 1 | u32 nvar 8 | u64 nx | u64 ny |
//         f64 time, little endian (40 bytes);
// payload nx*ny records of 8 f64 (x, y, rho, mom_x, mom_y, ee, ei, er),
//         j-major / i-fastest; the six state values are NaN at non-fluid
//         nodes (io.rs:58-73).
// A snapshot is packed on the device into that payload order, copied to
// pinned host memory on the context's stream, and written by a host thread
// to `path`.tmp, then renamed to `path` (io.rs:93-99), so the solver stream
// never waits on the file system.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "context.h"

using namespace rh3t;

namespace {

constexpr char kMagic[8] = {'R', 'H', '3', 'T', 'B', 'I', 'N', '1'};
constexpr uint32_t kVersion = 1, kNvar = 8;
constexpr int kHeaderBytes = 40;

// staging: [time, pad] + nx*ny*8 payload doubles
__global__ void k_pack_snapshot(const Inst* __restrict__ insts, int k, double x0, double y0,
                                double* __restrict__ out) {
    const Inst& I = insts[k];
    const long long n = (long long)I.nx * I.ny;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) { out[0] = I.sc->t_after; out[1] = 0.0; }
    if (t >= n) return;
    const int j = (int)(t / I.nx), i = (int)(t - (long long)j * I.nx); // j-major, i fastest
    const long long node = node_of(I, i, j);
    double* r = out + 2 + 8 * t;
    // GridInfo::x / y (field1.rs:6-15) without contraction
    r[0] = __dadd_rn(x0, __dmul_rn((double)i, I.dx));
    r[1] = __dadd_rn(y0, __dmul_rn((double)j, I.dy));
    const bool fl = I.mask[node] != 0;
    const double qnan = __longlong_as_double(0x7ff8000000000000ll); // Rust f64::NAN
#pragma unroll
    for (int c = 0; c < 6; ++c) r[2 + c] = fl ? I.U[c * I.plane + node] : qnan;
}

// energy split (py_utils/energy_split.py): per block, over fluid nodes in
// j-major order: max, sum and sum of squares of |ee - ei|, |ee - er|,
// |ei - er|; part[9 * block + q]
constexpr int ES_THREADS = 256;
__global__ void __launch_bounds__(ES_THREADS) k_energy_split(const Inst* __restrict__ insts, int k,
                                                             double* __restrict__ part, long long* __restrict__ cnt) {
    __shared__ double red[ES_THREADS / 32][9];
    __shared__ long long rc[ES_THREADS / 32];
    const Inst& I = insts[k];
    const long long n = (long long)I.nx * I.ny;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    long long valid = 0;
    if (t < n) {
        const int j = (int)(t / I.nx), i = (int)(t - (long long)j * I.nx);
        const long long node = node_of(I, i, j);
        if (I.mask[node]) {
            const double ee = I.U[3 * I.plane + node], ei = I.U[4 * I.plane + node], er = I.U[5 * I.plane + node];
            const double d[3] = {fabs(ee - ei), fabs(ee - er), fabs(ei - er)};
            for (int q = 0; q < 3; ++q) { v[q] = d[q]; v[3 + q] = d[q]; v[6 + q] = d[q] * d[q]; }
            valid = 1;
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 9; ++q)
        for (int o = 16; o > 0; o >>= 1) {
            const double x = __shfl_xor_sync(0xffffffffu, v[q], o);
            v[q] = q < 3 ? fmax(v[q], x) : v[q] + x;
        }
    for (int o = 16; o > 0; o >>= 1) valid += __shfl_xor_sync(0xffffffffu, valid, o);
    if (lane == 0) {
        for (int q = 0; q < 9; ++q) red[w][q] = v[q];
        rc[w] = valid;
    }
    __syncthreads();
    if (threadIdx.x < 9) {
        const int q = threadIdx.x;
        double a = red[0][q];
        for (int ww = 1; ww < ES_THREADS / 32; ++ww) a = q < 3 ? fmax(a, red[ww][q]) : a + red[ww][q];
        part[9 * blockIdx.x + q] = a;
    }
    if (threadIdx.x == 0) {
        long long s = 0;
        for (int ww = 0; ww < ES_THREADS / 32; ++ww) s += rc[ww];
        cnt[blockIdx.x] = s;
    }
}

// first fluid node (j-major) where |ee - er| equals the maximum
__global__ void k_energy_argmax(const Inst* __restrict__ insts, int k, double dmax,
                                unsigned long long* __restrict__ arg) {
    const Inst& I = insts[k];
    const long long n = (long long)I.nx * I.ny;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int j = (int)(t / I.nx), i = (int)(t - (long long)j * I.nx);
    const long long node = node_of(I, i, j);
    if (!I.mask[node]) return;
    if (fabs(I.U[3 * I.plane + node] - I.U[5 * I.plane + node]) == dmax) atomicMin(arg, (unsigned long long)t);
}

struct Writer {
    std::thread th;
    int status = RH3T_OK;
    std::string err;
};

int write_file(const std::string& path, const double* staging, long long nx, long long ny, std::string& err) {
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) { err = "cannot create " + tmp; return RH3T_ERR_INVALID_ARGUMENT; }
    unsigned char h[kHeaderBytes];
    const uint64_t unx = (uint64_t)nx, uny = (uint64_t)ny;
    const double time = staging[0];
    std::memcpy(h, kMagic, 8);
    std::memcpy(h + 8, &kVersion, 4);
    std::memcpy(h + 12, &kNvar, 4);
    std::memcpy(h + 16, &unx, 8);
    std::memcpy(h + 24, &uny, 8);
    std::memcpy(h + 32, &time, 8);
    const size_t nb = (size_t)nx * ny * 8;
    bool ok = std::fwrite(h, 1, kHeaderBytes, f) == (size_t)kHeaderBytes &&
              std::fwrite(staging + 2, sizeof(double), nb, f) == nb;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) { err = "short write to " + tmp; std::remove(tmp.c_str()); return RH3T_ERR_INVALID_ARGUMENT; }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) { err = "cannot rename " + tmp; return RH3T_ERR_INVALID_ARGUMENT; }
    return RH3T_OK;
}

} // namespace

// per-context snapshot state (context.h keeps an opaque pointer)
struct rh3t_io {
    double* d_stage = nullptr;
    double* h_stage = nullptr; // pinned
    size_t cap = 0;            // doubles
    cudaEvent_t done = nullptr;
    Writer w;
    double* d_part = nullptr;
    long long* d_cnt = nullptr;
    unsigned long long* d_arg = nullptr;
    size_t part_cap = 0;
};

namespace rh3t {
void io_free(rh3t_ctx* c) {
    rh3t_io* io = c->io;
    if (!io) return;
    if (io->w.th.joinable()) io->w.th.join();
    if (io->d_stage) cudaFree(io->d_stage);
    if (io->h_stage) cudaFreeHost(io->h_stage);
    if (io->done) cudaEventDestroy(io->done);
    if (io->d_part) cudaFree(io->d_part);
    if (io->d_cnt) cudaFree(io->d_cnt);
    if (io->d_arg) cudaFree(io->d_arg);
    delete io;
    c->io = nullptr;
}
} // namespace rh3t

namespace {
rh3t_io* io_of(rh3t_ctx* c) {
    if (!c->io) c->io = new rh3t_io();
    return c->io;
}

int join_writer(rh3t_ctx* c) {
    rh3t_io* io = io_of(c);
    if (io->w.th.joinable()) io->w.th.join();
    const int st = io->w.status;
    io->w.status = RH3T_OK;
    if (st) return set_error(c, st, io->w.err.c_str());
    return RH3T_OK;
}
} // namespace

extern "C" int rh3t_snapshot(rh3t_ctx* c, int32_t k, const char* path) {
    if (!c || !path || k < 0 || k >= c->n_inst) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    if (int rc = join_writer(c)) return rc; // the staging buffers are reused
    rh3t_io* io = io_of(c);
    const HostInst& H = c->hi[k];
    const size_t need = 2 + (size_t)H.nx * H.ny * 8;
    if (io->cap < need) {
        if (io->d_stage) cudaFree(io->d_stage);
        if (io->h_stage) cudaFreeHost(io->h_stage);
        io->d_stage = nullptr;
        io->h_stage = nullptr;
        io->cap = 0;
        CK(c, cudaMalloc(&io->d_stage, need * sizeof(double)));
        CK(c, cudaMallocHost(&io->h_stage, need * sizeof(double)));
        io->cap = need;
    }
    if (!io->done) CK(c, cudaEventCreateWithFlags(&io->done, cudaEventDisableTiming));
    const long long n = (long long)H.nx * H.ny;
    k_pack_snapshot<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->d_inst, k, H.grid.x0, H.grid.y0,
                                                                      io->d_stage);
    c->launches += 1;
    CK(c, cudaGetLastError());
    CK(c, cudaMemcpyAsync(io->h_stage, io->d_stage, need * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaEventRecord(io->done, c->stream));
    const std::string p(path);
    const long long nx = H.nx, ny = H.ny;
    io->w.status = RH3T_OK;
    io->w.err.clear();
    io->w.th = std::thread([io, p, nx, ny]() {
        if (cudaEventSynchronize(io->done) != cudaSuccess) {
            io->w.status = RH3T_ERR_CUDA;
            io->w.err = "snapshot copy failed";
            return;
        }
        io->w.status = write_file(p, io->h_stage, nx, ny, io->w.err);
    });
    return RH3T_OK;
}

extern "C" int rh3t_snapshot_wait(rh3t_ctx* c) {
    if (!c) return RH3T_ERR_INVALID_ARGUMENT;
    return join_writer(c);
}

extern "C" int rh3t_restart(rh3t_ctx* c, int32_t k, const char* path) {
    if (!c || !path || k < 0 || k >= c->n_inst) return RH3T_ERR_INVALID_ARGUMENT;
    const HostInst& H = c->hi[k];
    FILE* f = std::fopen(path, "rb");
    if (!f) return set_error(c, RH3T_ERR_INVALID_ARGUMENT, (std::string("cannot open restart file ") + path).c_str());
    unsigned char h[kHeaderBytes];
    if (std::fread(h, 1, kHeaderBytes, f) != (size_t)kHeaderBytes) {
        std::fclose(f);
        return set_error(c, RH3T_ERR_INVALID_ARGUMENT, "restart file shorter than its header");
    }
    uint32_t ver, nvar;
    uint64_t nx, ny;
    double time;
    std::memcpy(&ver, h + 8, 4);
    std::memcpy(&nvar, h + 12, 4);
    std::memcpy(&nx, h + 16, 8);
    std::memcpy(&ny, h + 24, 8);
    std::memcpy(&time, h + 32, 8);
    const char* bad = std::memcmp(h, kMagic, 8) != 0 ? "restart file: bad magic (not RH3TBIN1)"
                      : ver != kVersion               ? "restart file: unsupported version"
                      : nvar != kNvar                 ? "restart file: nvar is not 8"
                      : (nx != (uint64_t)H.nx || ny != (uint64_t)H.ny) ? "restart grid mismatch"
                                                                       : nullptr;
    if (bad) { std::fclose(f); return set_error(c, RH3T_ERR_INVALID_ARGUMENT, bad); }
    std::vector<double> rec((size_t)nx * ny * 8);
    const bool ok = std::fread(rec.data(), sizeof(double), rec.size(), f) == rec.size();
    std::fclose(f);
    if (!ok) return set_error(c, RH3T_ERR_INVALID_ARGUMENT, "restart file: truncated payload");
    // io.rs:113-121: fluid nodes take the record (and must be finite); the
    // value array is in the reference's i*ny + j order
    std::vector<double> value((size_t)nx * ny * 6, 0.0);
    for (uint64_t j = 0; j < ny; ++j)
        for (uint64_t i = 0; i < nx; ++i) {
            const size_t l = (size_t)i * ny + j;
            if (!H.fluid[l]) continue;
            const double* a = rec.data() + 8 * ((size_t)j * nx + i);
            for (int q = 0; q < 6; ++q) {
                if (!std::isfinite(a[2 + q])) {
                    char msg[160];
                    std::snprintf(msg, sizeof(msg), "non-finite restart state at (%llu, %llu)",
                                  (unsigned long long)i, (unsigned long long)j);
                    return set_error(c, RH3T_ERR_INVALID_ARGUMENT, msg);
                }
                value[6 * l + q] = a[2 + q];
            }
        }
    return rh3t_upload_instance(c, k, value.data(), time);
}

extern "C" int rh3t_energy_split(rh3t_ctx* c, int32_t k, double* out) {
    if (!c || !out || k < 0 || k >= c->n_inst) return RH3T_ERR_INVALID_ARGUMENT;
    CK(c, cudaSetDevice(c->device));
    rh3t_io* io = io_of(c);
    const HostInst& H = c->hi[k];
    const long long n = (long long)H.nx * H.ny;
    const unsigned nb = (unsigned)((n + ES_THREADS - 1) / ES_THREADS);
    if (io->part_cap < nb) {
        if (io->d_part) cudaFree(io->d_part);
        if (io->d_cnt) cudaFree(io->d_cnt);
        io->d_part = nullptr;
        io->d_cnt = nullptr;
        io->part_cap = 0;
        CK(c, cudaMalloc(&io->d_part, (size_t)nb * 9 * sizeof(double)));
        CK(c, cudaMalloc(&io->d_cnt, (size_t)nb * sizeof(long long)));
        io->part_cap = nb;
    }
    if (!io->d_arg) CK(c, cudaMalloc(&io->d_arg, sizeof(unsigned long long)));
    k_energy_split<<<nb, ES_THREADS, 0, c->stream>>>(c->d_inst, k, io->d_part, io->d_cnt);
    CK(c, cudaGetLastError());
    std::vector<double> part((size_t)nb * 9);
    std::vector<long long> cnt(nb);
    CK(c, cudaMemcpyAsync(part.data(), io->d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaMemcpyAsync(cnt.data(), io->d_cnt, cnt.size() * sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    double mx[3] = {0, 0, 0}, sm[3] = {0, 0, 0}, sq[3] = {0, 0, 0};
    long long valid = 0;
    for (unsigned b = 0; b < nb; ++b) { // blocks in order: a deterministic sum
        for (int q = 0; q < 3; ++q) {
            mx[q] = std::fmax(mx[q], part[9 * b + q]);
            sm[q] += part[9 * b + 3 + q];
            sq[q] += part[9 * b + 6 + q];
        }
        valid += cnt[b];
    }
    if (valid == 0) return set_error(c, RH3T_ERR_INVALID_ARGUMENT, "energy split: no fluid node");
    const unsigned long long none = ~0ull;
    CK(c, cudaMemcpyAsync(io->d_arg, &none, sizeof(none), cudaMemcpyHostToDevice, c->stream));
    k_energy_argmax<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->d_inst, k, mx[1], io->d_arg);
    c->launches += 2;
    unsigned long long arg = none;
    CK(c, cudaMemcpyAsync(&arg, io->d_arg, sizeof(arg), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    const long long j = (long long)(arg / (unsigned long long)H.nx), i = (long long)(arg % (unsigned long long)H.nx);
    for (int q = 0; q < 3; ++q) {
        out[q] = mx[q];
        out[3 + q] = sm[q] / (double)valid;
        out[6 + q] = std::sqrt(sq[q] / (double)valid);
    }
    out[9] = H.grid.x0 + (double)i * H.grid.dx;
    out[10] = H.grid.y0 + (double)j * H.grid.dy;
    out[11] = (double)valid;
    return RH3T_OK;
}
