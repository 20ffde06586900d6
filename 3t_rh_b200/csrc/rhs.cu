// Cell right-hand side fused with the SSP-RK3 stage update (main.rs:251-349):
// flux differences, the non-conservative x/y terms (noncon.rs:288-332), the
// exchange source (source.rs:7-21) and the diffusion differences, then
// u' = a u + b v + c dt rhs with the admissibility check (main.rs:22-33).
//
// A block covers TI x TJ = 256 cells (shape chosen per tile). The pressures and the transport
// velocities of the nodes within reach of the 9-point non-conservative
// stencils (the tile plus a 4-node halo, corners excluded) are computed once
// into shared memory; the reference's access-table gathers (main.rs:276-277)
// evaluate them once per use, 17 times per node.
//
// mode 0 writes the rhs (6 planes of nx*ny, i*ny+j, instance k at
// rhs_out + 6*cell_off) for l(); mode 1 applies the stage update of `stage`;
// mode 2 does both, the rhs into padded planes at rhs_out + aoff (the
// adjoint's record of the forward stages).
#include "common.cuh"
#include "kernels.cuh"
#include "physics.cuh"

namespace rh3t {

#ifdef RH3T_EXACT
constexpr bool kExactR = true;
#else
constexpr bool kExactR = false;
#endif

// divisors shared by every cell of an instance: 60 dx, dx, 60 dy, dy
// (noncon.rs:26-44, 315-331), 6 cve, 6 cvi, a_rad (state.rs:245-276)
constexpr int RHS_NR = 7;
__device__ __forceinline__ double rhs_divisor(const Inst& I, int k) {
    switch (k) {
    case 0: return 60.0 * I.dx;
    case 1: return I.dx;
    case 2: return 60.0 * I.dy;
    case 3: return I.dy;
    case 4: return 6.0 * I.P.cve;
    case 5: return 6.0 * I.P.cvi;
    default: return I.P.a_rad;
    }
}
__device__ __forceinline__ Recip rhs_recip(const Inst& I, const double* sR, int k) {
    return recip_of(rhs_divisor(I, k), sR[k]);
}

__global__ void __launch_bounds__(RHS_THREADS, 2) k_rhs_stage(const Inst* __restrict__ insts, const Tile* __restrict__ tiles,
                                                   int nt, int stage, int mode, double* __restrict__ rhs_out) {
    __shared__ double sP[5][RHS_NPT]; // pe, pi, pr, u, v
    __shared__ double sR[RHS_NR];      // reciprocals of the instance's divisors (rhs_divisor)
    if (blockIdx.x >= nt) return;
    const Tile t = tiles[blockIdx.x];
    const Inst& I = insts[t.inst];
    if (has_error(I)) return;
    const DevParams& P = I.P;
    const long long plane = I.plane;
    const double* __restrict__ src = stage_src(I, stage);
    const int nx = I.nx, ny = I.ny;
    const int TJ = 1 << t.lg, TI = RHS_THREADS >> t.lg;
    const int HJ = TJ + 8, NPT = (TI + 8) * HJ;
    if (threadIdx.x < RHS_NR) sR[threadIdx.x] = __ddiv_rn(1.0, rhs_divisor(I, threadIdx.x));
    // ---- stage node primitives (tile + 4-node cross halo)
    for (int p = threadIdx.x; p < NPT; p += blockDim.x) {
        const int hi = p / HJ, hj = p - hi * HJ;
        const bool corner = (hi < 4 || hi >= TI + 4) && (hj < 4 || hj >= TJ + 4);
        const int i = t.i - 4 + hi, j = t.j0 - 4 + hj;
        if (corner || i < -RH3T_PAD || i >= nx + RH3T_PAD || j < -RH3T_PAD || j >= ny + RH3T_PAD) continue;
        double s[6];
        load6(src, plane, node_of(I, i, j), s);
        Prim d = kExactR ? prim_from_state(s, P) : fastm::prim(s, P);
        sP[0][p] = d.pe; sP[1][p] = d.pi; sP[2][p] = d.pr; sP[3][p] = d.u; sP[4][p] = d.v;
    }
    __syncthreads();
    const int ti = threadIdx.x >> t.lg, tj = threadIdx.x & (TJ - 1);
    const int i = t.i + ti, j = t.j0 + tj;
    if (i >= nx || j >= ny) return;
    const long long n = node_of(I, i, j);
    if (!I.mask[n]) return;
    const double dx = I.dx, dy = I.dy;
    const long long fpx = (long long)(nx + 1) * ny, fix = (long long)i * ny + j;
    const long long fpy = (long long)nx * (ny + 1), fiy = (long long)i * (ny + 1) + j;
    double rhs[6];
    const double sx = 1.0 / dx, sy = 1.0 / dy;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        const double fl = I.fx[c * fpx + fix], fr = I.fx[c * fpx + fix + ny];
        const double fb = I.fy[c * fpy + fiy], ft = I.fy[c * fpy + fiy + 1];
        rhs[c] = -(fr - fl) * sx + -(ft - fb) * sy;
    }
    double pe[9], pi[9], pr[9], vel[9], ncx[3], ncy[3];
    const int hc = (ti + 4) * HJ + (tj + 4);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int p = hc + (q - 4) * HJ;
        pe[q] = sP[0][p]; pi[q] = sP[1][p]; pr[q] = sP[2][p]; vel[q] = sP[3][p];
    }
    if (kExactR) noncon9(pe, pi, pr, vel, rhs_recip(I, sR, 0), rhs_recip(I, sR, 1), ncx);
    else fastm::noncon9(pe, pi, pr, vel, 1.0 / (60.0 * dx), 1.0 / dx, ncx);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int p = hc + (q - 4);
        pe[q] = sP[0][p]; pi[q] = sP[1][p]; pr[q] = sP[2][p]; vel[q] = sP[4][p];
    }
    if (kExactR) noncon9(pe, pi, pr, vel, rhs_recip(I, sR, 2), rhs_recip(I, sR, 3), ncy);
    else fastm::noncon9(pe, pi, pr, vel, 1.0 / (60.0 * dy), 1.0 / dy, ncy);
#pragma unroll
    for (int k = 0; k < 3; ++k) rhs[3 + k] = rhs[3 + k] + ncx[k] + ncy[k];
    if (I.source) {
        double s[6];
        load6(src, plane, n, s);
        double te, ti_, tr;
        temps_from_state(s, P, rhs_recip(I, sR, 4), rhs_recip(I, sR, 5), rhs_recip(I, sR, 6), te, ti_, tr);
        const double so[3] = {-P.omega_ei * (te - ti_) - P.omega_er * (pow4d(te) - pow4d(tr)),
                              P.omega_ei * (te - ti_), P.omega_er * (pow4d(te) - pow4d(tr))};
#pragma unroll
        for (int k = 0; k < 3; ++k) rhs[3 + k] = rhs[3 + k] + so[k];
    }
    if (I.diffusion) {
        const double cx = -1.0 / (dx * dx), cy = -1.0 / (dy * dy);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double a = I.dfx[k * fpx + fix], b = I.dfx[k * fpx + fix + ny];
            const double c2 = I.dfy[k * fpy + fiy], d2 = I.dfy[k * fpy + fiy + 1];
            rhs[3 + k] = rhs[3 + k] + ((-(b - a) * cx) + (-(d2 - c2) * cy));
        }
    }
    if (mode == 0) {
        const long long ln = (long long)i * ny + j, lp = (long long)nx * ny;
        double* __restrict__ ro = rhs_out + 6 * I.cell_off;
#pragma unroll
        for (int c = 0; c < 6; ++c) ro[c * lp + ln] = rhs[c];
        return;
    }
    if (mode == 2) {
        double* __restrict__ ro = rhs_out + I.aoff;
#pragma unroll
        for (int c = 0; c < 6; ++c) ro[c * plane + n] = rhs[c];
    }
    const DevScalars& sc = *I.sc;
    double v[6];
    if (stage == 0) {
        const double coef = sc.coef[0];
#pragma unroll
        for (int c = 0; c < 6; ++c) v[c] = I.U[c * plane + n] + rhs[c] * coef;
#pragma unroll
        for (int c = 0; c < 6; ++c) I.A[c * plane + n] = v[c];
    } else if (stage == 1) {
        const double coef = sc.coef[1];
#pragma unroll
        for (int c = 0; c < 6; ++c) v[c] = I.U[c * plane + n] * 0.75 + I.A[c * plane + n] * 0.25 + rhs[c] * coef;
#pragma unroll
        for (int c = 0; c < 6; ++c) I.B[c * plane + n] = v[c];
    } else {
        const double coef = sc.coef[2];
        const double wb = 1.0 / 3.0, wa = 2.0 / 3.0;
#pragma unroll
        for (int c = 0; c < 6; ++c) v[c] = I.U[c * plane + n] * wb + I.B[c * plane + n] * wa + rhs[c] * coef;
#pragma unroll
        for (int c = 0; c < 6; ++c) I.U[c * plane + n] = v[c];
    }
    bool ok = isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]) && isfinite(v[3]) && isfinite(v[4]) &&
              isfinite(v[5]) && v[0] > 0.0;
    if (ok) { // main.rs:24-33, the five quotients by rho through one reciprocal (the same IEEE quotients)
        const Recip r0 = recip(v[0]);
        const double ux = div_rn(v[1], r0), uy = div_rn(v[2], r0);
        const double k = div6_rn(ux * ux + uy * uy);
        ok = !(div_rn(v[3], r0) - k <= 0.0 || div_rn(v[4], r0) - k <= 0.0 || div_rn(v[5], r0) - k <= 0.0);
    }
    if (!ok) report(I, 2 + 2 * stage, 1, (unsigned)((long long)i * ny + j));
}

void launch_rhs_stage(cudaStream_t s, const Inst* insts, const Tile* tc, int nt, int stage, int mode, double* rhs) {
    if (nt <= 0) return;
    k_rhs_stage<<<nt, RHS_THREADS, 0, s>>>(insts, tc, nt, stage, mode, rhs);
}

} // namespace rh3t
