// GPU build of the least-squares tables of the Wall / Outflow / FarField
// ghosts (bc1.rs:108-188 precompute_ghost_bc): per ghost and order r = 0..4
// the matrix A of the (r+1)^2 E_r nodes in the ghost's (normal, tangential)
// frame, its pseudo-inverse P (bc1.rs:162-165, singular values <= 1e-12
// dropped), S_r = P^T M_r P (bc1.rs:169-175) and the derivative rows w_r
// (bc1.rs:89-101, 176-186).
//
// One warp per ghost. The pseudo-inverse is the host builder's one-sided
// Jacobi SVD (ghostgrid.cpp pinv) with the same rotation order, the same
// stopping rule and every sum taken in the same order: each lane owns one
// row of A (and of V), the column sums are formed by every lane from shared
// memory in row order, and all arithmetic goes through the round-to-nearest
// intrinsics, so nothing is contracted into an FMA. The tables are therefore
// bit-identical to the host build's, in both library builds.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "host/lsbuild.h"

namespace rh3t {

namespace {

constexpr int LS_WARPS = 8;
constexpr long long LS_CHUNK = 65536; // ghosts per launch (630 MB of tables)

struct LsWarp {
    double U[25 * 15]; // rows of A, then of A V; later T = P^T M (row a, col c)
    double V[15 * 15];
};

__constant__ int kLsSt[5] = {0, 1, 5, 14, 30};
__constant__ int kLsS[5] = {0, 1, 17, 98, 354};
__constant__ int kLsW[5] = {0, 1, 9, 36, 100};
__constant__ int kLsM[5] = {0, 0, 9, 45, 145};

// compiler-rt __powidf2 (Rust f64::powi), as ghostgrid.cpp ipow
__device__ __forceinline__ double ipow_rn(double a, int b) {
    double r = 1.0;
    for (;;) {
        if (b & 1) r = __dmul_rn(r, a);
        b /= 2;
        if (b == 0) break;
        a = __dmul_rn(a, a);
    }
    return r;
}

template <int R>
__device__ void ls_order(const LsGrid& G, const LsJob& J, const uint32_t* __restrict__ st, double* __restrict__ S,
                         double* __restrict__ W, LsWarp& sh, int lane) {
    constexpr int M = (R + 1) * (R + 1), N = (R + 1) * (R + 2) / 2;
    double* U = sh.U;
    double* V = sh.V;
    // A: node a in the (n, t) frame, monomials n^i t^(tot - i) (bc1.rs:120-160)
    if (lane < M) {
        const uint32_t l = st[lane];
        const long long i = (long long)l / G.ny, j = (long long)l % G.ny;
        const double X = __dadd_rn(G.x0, __dmul_rn((double)i, G.dx));
        const double Y = __dadd_rn(G.y0, __dmul_rn((double)j, G.dy));
        const double dx = __dsub_rn(X, J.p0x), dy = __dsub_rn(Y, J.p0y);
        const double nor = __dadd_rn(__dmul_rn(J.nx, dx), __dmul_rn(J.ny, dy));
        const double tan = __dadd_rn(__dmul_rn(-dx, J.ny), __dmul_rn(dy, J.nx));
        int col = 0;
#pragma unroll
        for (int t = 0; t <= R; ++t)
#pragma unroll
            for (int i2 = 0; i2 <= t; ++i2) U[lane * N + col++] = __dmul_rn(ipow_rn(nor, i2), ipow_rn(tan, t - i2));
    }
    if (lane < N)
#pragma unroll
        for (int k = 0; k < N; ++k) V[lane * N + k] = lane == k ? 1.0 : 0.0;
    __syncwarp();
    // one-sided Jacobi: cyclic (p, q) order, at most 80 sweeps
    for (int sweep = 0; sweep < 80; ++sweep) {
        double off = 0.0;
#pragma unroll 1
        for (int p = 0; p < N - 1; ++p)
#pragma unroll 1
            for (int q = p + 1; q < N; ++q) {
                double al = 0.0, be = 0.0, ga = 0.0;
#pragma unroll
                for (int i = 0; i < M; ++i) {
                    const double up = U[i * N + p], uq = U[i * N + q];
                    al = __dadd_rn(al, __dmul_rn(up, up));
                    be = __dadd_rn(be, __dmul_rn(uq, uq));
                    ga = __dadd_rn(ga, __dmul_rn(up, uq));
                }
                // every lane holds the same sums: the branches are warp-uniform
                if (ga == 0.0) continue;
                const double rel = __ddiv_rn(fabs(ga), __dsqrt_rn(__dmul_rn(al, be)));
                off = fmax(off, rel);
                if (rel < 1e-17) continue;
                const double zeta = __ddiv_rn(__dsub_rn(be, al), __dmul_rn(2.0, ga));
                const double t = __ddiv_rn(zeta >= 0 ? 1.0 : -1.0,
                                           __dadd_rn(fabs(zeta), __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(zeta, zeta)))));
                const double c = __ddiv_rn(1.0, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(t, t))));
                const double s = __dmul_rn(c, t);
                if (lane < M) {
                    const double up = U[lane * N + p], uq = U[lane * N + q];
                    U[lane * N + p] = __dsub_rn(__dmul_rn(c, up), __dmul_rn(s, uq));
                    U[lane * N + q] = __dadd_rn(__dmul_rn(s, up), __dmul_rn(c, uq));
                }
                if (lane < N) {
                    const double vp = V[lane * N + p], vq = V[lane * N + q];
                    V[lane * N + p] = __dsub_rn(__dmul_rn(c, vp), __dmul_rn(s, vq));
                    V[lane * N + q] = __dadd_rn(__dmul_rn(s, vp), __dmul_rn(c, vq));
                }
                __syncwarp();
            }
        if (off < 1e-16) break;
    }
    // P = V diag(1 / sigma^2) (A V)^T, column a of P on lane a
    double Pc[N];
#pragma unroll
    for (int k = 0; k < N; ++k) Pc[k] = 0.0;
#pragma unroll 1
    for (int j = 0; j < N; ++j) {
        double sig = 0.0;
#pragma unroll
        for (int i = 0; i < M; ++i) sig = __dadd_rn(sig, __dmul_rn(U[i * N + j], U[i * N + j]));
        sig = __dsqrt_rn(sig);
        if (!(sig > 1.0e-12)) continue;
        if (lane < M) {
            const double sc = __ddiv_rn(__ddiv_rn(U[lane * N + j], sig), sig);
#pragma unroll
            for (int k = 0; k < N; ++k) Pc[k] = __dadd_rn(Pc[k], __dmul_rn(V[k * N + j], sc));
        }
    }
    __syncwarp();
    if (R == 0) {
        if (lane == 0) S[0] = G.s0; // bc1.rs:167-168
    } else {
        // T = P^T M_r (row a on lane a, into U), then S = T P (column b on lane b)
        const double* __restrict__ Mr = G.M + kLsM[R];
        if (lane < M) {
#pragma unroll 1
            for (int cc = 0; cc < N; ++cc) {
                double acc = 0.0;
#pragma unroll
                for (int kk = 0; kk < N; ++kk) acc = __dadd_rn(acc, __dmul_rn(Pc[kk], Mr[kk * N + cc]));
                U[lane * N + cc] = acc;
            }
        }
        __syncwarp();
        if (lane < M) {
#pragma unroll 1
            for (int a = 0; a < M; ++a) {
                double acc = 0.0;
#pragma unroll
                for (int kk = 0; kk < N; ++kk) acc = __dadd_rn(acc, __dmul_rn(U[a * N + kk], Pc[kk]));
                S[a * M + lane] = acc;
            }
        }
    }
    // w_r: row k is k! times the pure-normal coefficient row n^k of P
    if (lane < M) {
        double kf = 1.0;
#pragma unroll
        for (int kk = 0; kk <= R; ++kk) {
            if (kk > 0) kf = __dmul_rn(kf, (double)kk);
            W[kk * M + lane] = __dmul_rn(kf, Pc[kk * (kk + 1) / 2 + kk]);
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(LS_WARPS * 32) k_ls_tables(const LsGrid* __restrict__ grids,
                                                             const LsJob* __restrict__ jobs,
                                                             const uint32_t* __restrict__ st, long long n,
                                                             double* __restrict__ s, double* __restrict__ w) {
    __shared__ LsWarp sh[LS_WARPS];
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    for (long long g = (long long)blockIdx.x * LS_WARPS + wi; g < n; g += (long long)gridDim.x * LS_WARPS) {
        const LsJob J = jobs[g];
        const LsGrid& G = grids[J.grid];
        const uint32_t* sg = st + (size_t)LS_STENCIL * g;
        double* so = s + (size_t)LS_S * g;
        double* wo = w + (size_t)LS_W * g;
        ls_order<0>(G, J, sg + kLsSt[0], so + kLsS[0], wo + kLsW[0], sh[wi], lane);
        ls_order<1>(G, J, sg + kLsSt[1], so + kLsS[1], wo + kLsW[1], sh[wi], lane);
        ls_order<2>(G, J, sg + kLsSt[2], so + kLsS[2], wo + kLsW[2], sh[wi], lane);
        ls_order<3>(G, J, sg + kLsSt[3], so + kLsS[3], wo + kLsW[3], sh[wi], lane);
        ls_order<4>(G, J, sg + kLsSt[4], so + kLsS[4], wo + kLsW[4], sh[wi], lane);
    }
}

struct DevBufs {
    LsGrid* grids = nullptr;
    LsJob* jobs = nullptr;
    uint32_t* st = nullptr;
    double *s = nullptr, *w = nullptr;
    ~DevBufs() {
        void* p[] = {grids, jobs, st, s, w};
        for (void* q : p)
            if (q) cudaFree(q);
    }
};

int fail(cudaError_t e, const char* where, char* err, int err_len) {
    if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s: %s", where, cudaGetErrorString(e));
    return (int)e;
}

} // namespace

int ls_tables_device(int device, int n_grids, const LsGrid* grids, long long n_jobs, const LsJob* jobs,
                     const uint32_t* stencils, double* const* s_out, double* const* w_out, char* err, int err_len) {
    if (n_jobs <= 0) return 0;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e, "cudaSetDevice", err, err_len);
    const long long chunk = std::min(n_jobs, LS_CHUNK);
    DevBufs B;
#define LS_CK(call)                                            \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return fail(_e, #call, err, err_len); \
    } while (0)
    LS_CK(cudaMalloc(&B.grids, sizeof(LsGrid) * (size_t)n_grids));
    LS_CK(cudaMalloc(&B.jobs, sizeof(LsJob) * (size_t)chunk));
    LS_CK(cudaMalloc(&B.st, sizeof(uint32_t) * LS_STENCIL * (size_t)chunk));
    LS_CK(cudaMalloc(&B.s, sizeof(double) * LS_S * (size_t)chunk));
    LS_CK(cudaMalloc(&B.w, sizeof(double) * LS_W * (size_t)chunk));
    LS_CK(cudaMemcpy(B.grids, grids, sizeof(LsGrid) * (size_t)n_grids, cudaMemcpyHostToDevice));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    for (long long c0 = 0; c0 < n_jobs; c0 += chunk) {
        const long long c1 = std::min(n_jobs, c0 + chunk), nc = c1 - c0;
        LS_CK(cudaMemcpy(B.jobs, jobs + c0, sizeof(LsJob) * (size_t)nc, cudaMemcpyHostToDevice));
        LS_CK(cudaMemcpy(B.st, stencils + (size_t)LS_STENCIL * c0, sizeof(uint32_t) * LS_STENCIL * (size_t)nc,
                         cudaMemcpyHostToDevice));
        const long long blocks = std::min((nc + LS_WARPS - 1) / LS_WARPS, (long long)sms * 16);
        k_ls_tables<<<(unsigned)blocks, LS_WARPS * 32>>>(B.grids, B.jobs, B.st, nc, B.s, B.w);
        LS_CK(cudaGetLastError());
        LS_CK(cudaDeviceSynchronize());
        // runs of consecutive slots of one grid go back with one copy each
        for (long long a = c0; a < c1;) {
            long long b = a + 1;
            while (b < c1 && jobs[b].grid == jobs[a].grid && jobs[b].slot == jobs[b - 1].slot + 1) ++b;
            const LsJob& J = jobs[a];
            LS_CK(cudaMemcpy(s_out[J.grid] + (size_t)LS_S * J.slot, B.s + (size_t)LS_S * (a - c0),
                             sizeof(double) * LS_S * (size_t)(b - a), cudaMemcpyDeviceToHost));
            LS_CK(cudaMemcpy(w_out[J.grid] + (size_t)LS_W * J.slot, B.w + (size_t)LS_W * (a - c0),
                             sizeof(double) * LS_W * (size_t)(b - a), cudaMemcpyDeviceToHost));
            a = b;
        }
    }
#undef LS_CK
    return 0;
}

} // namespace rh3t
