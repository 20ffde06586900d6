// rh3t device kernels (sm_100a, FP64): the dt reduction, layout transfers and
// diagnostics. One launch of each kernel covers all instances of a context or
// batch: cell and face kernels walk a list of tiles, the ghost kernel a list
// of ghost records, so the plain solver is simply a batch of one.
//
// Per step: k_dt (main.rs:375-408, dt.rs), then per RK stage k_ghosts
// (ghosts.cu) -> k_flux (flux.cu) -> k_rhs_stage (rhs.cu). dt, stage times
// and RK coefficients never leave the device.
#include "common.cuh"
#include "kernels.cuh"
#include "physics.cuh"

namespace rh3t {

// ------------------------------------------------------------------ dt
// Orderable 64-bit key of a double (total order, NaN excluded by the caller).
__device__ __forceinline__ unsigned long long dkey(double x) {
    unsigned long long b = (unsigned long long)__double_as_longlong(x);
    return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
    unsigned long long b = (k & 0x8000000000000000ull) ? (k & ~0x8000000000000000ull) : ~k;
    return __longlong_as_double((long long)b);
}

// mode 0: dt_cfl only; mode 1: start of a step (dt = cfl_factor * dt_cfl,
// clipped to t_final, stage times and coefficients, main.rs:460-464).
__device__ void finalize_step(const Inst& I, double dt_cfl, int mode) {
    DevScalars& sc = *I.sc;
    if (mode == 1) {
        sc.step = sc.steps_started;
        sc.steps_started += 1;
        double t = sc.t_after;
        double dt = sc.cfl_factor * dt_cfl;
        if (t + dt > sc.t_final) dt = sc.t_final - t;
        if (!(dt > 0.0)) report(I, 0, 9, 0u);
        sc.t = t;
        sc.dt = dt;
        sc.t_stage[0] = t;
        sc.t_stage[1] = t + dt;
        sc.t_stage[2] = t + 0.5 * dt;
        sc.t_after = t + dt;
        sc.coef[0] = dt;
        sc.coef[1] = dt / 4.0;
        sc.coef[2] = 2.0 * dt / 3.0;
    }
}

__global__ void __launch_bounds__(128) k_dt(const Inst* __restrict__ insts, const Tile* __restrict__ tiles, int nt,
                                            int mode) {
    __shared__ double red[4];
    __shared__ bool last;
    if (blockIdx.x >= nt) return;
    const Tile t = tiles[blockIdx.x];
    const Inst& I = insts[t.inst];
    const int i = t.i, j = t.j0 + threadIdx.x;
    double m = INFINITY;
    if (j < I.ny) {
        const long long n = node_of(I, i, j);
        if (I.mask[n]) {
            double s[6];
            load6(I.U, I.plane, n, s);
            double d = local_dt(s, I.dx, I.dy, I.P);
            m = fmin(m, d);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double bm = fmin(fmin(red[0], red[1]), fmin(red[2], red[3]));
        if (!isnan(bm)) atomicMin(&I.sc->dt_cfl_bits, dkey(bm));
        __threadfence();
        unsigned int done = atomicAdd(&I.sc->counter, 1u);
        last = done == (unsigned)I.n_tiles_dt - 1u;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        unsigned long long k = atomicAdd(&I.sc->dt_cfl_bits, 0ull);
        double dt_cfl = dkey_inv(k);
        I.sc->dt_cfl_bits = dkey(INFINITY);
        I.sc->counter = 0u;
        I.sc->dt_cfl = dt_cfl;
        finalize_step(I, dt_cfl, mode);
    }
}

// A step with a caller-given dt (rk3_ssp(dt), main.rs:351-373), instances
// insts[0, n_inst)
__global__ void k_set_dt(const Inst* __restrict__ insts, int n_inst, double dt) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_inst) return;
    DevScalars& sc = *insts[k].sc;
    sc.step = sc.steps_started;
    sc.steps_started += 1;
    double t = sc.t_after;
    sc.t = t;
    sc.dt = dt;
    sc.t_stage[0] = t;
    sc.t_stage[1] = t + dt;
    sc.t_stage[2] = t + 0.5 * dt;
    sc.t_after = t + dt;
    sc.coef[0] = dt;
    sc.coef[1] = dt / 4.0;
    sc.coef[2] = 2.0 * dt / 3.0;
}

// ------------------------------------------------------------------ layout
// AoS (6 doubles per cell, i*ny+j, instance k at aos + 6*cell_off) <-> padded
// SoA planes of buffer U, fluid cells only. blockIdx.y = instance - k0.
__global__ void k_scatter(const Inst* __restrict__ insts, int k0, const double* __restrict__ aos,
                          const double* __restrict__ times) {
    const int k = k0 + blockIdx.y;
    const Inst& I = insts[k];
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l == 0) {
        I.sc->t_after = times[k];
        I.sc->t = times[k];
    }
    if (l >= (long long)I.nx * I.ny) return;
    int i = (int)(l / I.ny), j = (int)(l % I.ny);
    long long n = node_of(I, i, j);
    if (!I.mask[n]) return;
    const double* a = aos + 6 * (I.cell_off + l);
#pragma unroll
    for (int c = 0; c < 6; ++c) I.U[c * I.plane + n] = a[c];
}

__global__ void k_gather(const Inst* __restrict__ insts, int k0, double* __restrict__ aos) {
    const Inst& I = insts[k0 + blockIdx.y];
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= (long long)I.nx * I.ny) return;
    int i = (int)(l / I.ny), j = (int)(l % I.ny);
    long long n = node_of(I, i, j);
    bool f = I.mask[n] != 0;
    double* a = aos + 6 * (I.cell_off + l);
#pragma unroll
    for (int c = 0; c < 6; ++c) a[c] = f ? I.U[c * I.plane + n] : 0.0;
}

// cfl_factor / t_final of instances [k0, k0 + n)
__global__ void k_set_step(const Inst* __restrict__ insts, int k0, int n, double cfl, double t_final) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    DevScalars& sc = *insts[k0 + k].sc;
    sc.cfl_factor = cfl;
    sc.t_final = t_final;
}

// planes (6 x nx*ny) -> AoS, for rh3t_l's rhs
__global__ void k_planes_to_aos(const double* __restrict__ planes, long long n, double* __restrict__ aos) {
    long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n) return;
#pragma unroll
    for (int c = 0; c < 6; ++c) aos[l * 6 + c] = planes[c * n + l];
}

// ghost values of stage buffer U -> (n_ghosts x 6)
__global__ void k_ghost_values(const Inst* __restrict__ insts, const GhostRec* __restrict__ recs, int n,
                               double* __restrict__ out) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const GhostRec R = recs[g];
    const Inst& I = insts[R.inst];
#pragma unroll
    for (int c = 0; c < 6; ++c) out[(long long)g * 6 + c] = I.U[c * I.plane + R.node];
}

// ------------------------------------------------------------------ FP64 peak probe
// 8 independent FMA chains per thread, values kept in [0.5, 2].
__global__ void __launch_bounds__(256) k_dfma(double* out, int iters, double b, double c) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = 1.0 + 1e-3 * (threadIdx.x + k);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.678) out[blockIdx.x] = s; // never true; keeps the loop live
}

// ------------------------------------------------------------------ math check
// out[3k] = x^(1/4), out[3k+1] = x^10, out[3k+2] = x^q with the device
// routines used by the solver (diagnostic entry rh3t_math_check).
__global__ void k_math_check(const double* __restrict__ x, int n, double q, double* __restrict__ out) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    out[3 * k] = cr_pow_quarter(x[k]);
    out[3 * k + 1] = cr_powi(x[k], 10);
    out[3 * k + 2] = pow_q(x[k], q);
}

// ------------------------------------------------------------------ host launchers
void launch_math_check(cudaStream_t s, const double* x, int n, double q, double* out) {
    k_math_check<<<(n + 127) / 128, 128, 0, s>>>(x, n, q, out);
}
void launch_dfma(cudaStream_t s, int blocks, double* out, int iters) {
    k_dfma<<<blocks, 256, 0, s>>>(out, iters, 0.9999999, 1e-7);
}

void launch_dt(cudaStream_t s, const Inst* insts, const Tile* tc, int nt, int mode) {
    if (nt <= 0) return;
    k_dt<<<nt, 128, 0, s>>>(insts, tc, nt, mode);
}
void launch_set_dt(cudaStream_t s, const Inst* insts, int n_inst, double dt) {
    k_set_dt<<<(n_inst + 127) / 128, 128, 0, s>>>(insts, n_inst, dt);
}
void launch_scatter(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, const double* aos,
                    const double* times) {
    if (n <= 0) return;
    k_scatter<<<dim3((unsigned)((max_cells + 255) / 256), (unsigned)n), 256, 0, s>>>(insts, k0, aos, times);
}
void launch_gather(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, double* aos) {
    if (n <= 0) return;
    k_gather<<<dim3((unsigned)((max_cells + 255) / 256), (unsigned)n), 256, 0, s>>>(insts, k0, aos);
}
void launch_set_step(cudaStream_t s, const Inst* insts, int k0, int n, double cfl, double t_final) {
    if (n <= 0) return;
    k_set_step<<<(n + 127) / 128, 128, 0, s>>>(insts, k0, n, cfl, t_final);
}
void launch_planes_to_aos(cudaStream_t s, const double* planes, long long n, double* aos) {
    k_planes_to_aos<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(planes, n, aos);
}
void launch_ghost_values(cudaStream_t s, const Inst* insts, const GhostRec* recs, int n, double* out) {
    if (n <= 0) return;
    k_ghost_values<<<(n + 127) / 128, 128, 0, s>>>(insts, recs, n, out);
}

} // namespace rh3t
