// Ghost-node update of one RK stage (ghost.rs:199-268 update_values_parallel,
// bc1.rs:609-928 set_ghost_point_value with precomputed GhostBC data), in
// two launches.
//
// k_ghost_prep, one thread per ghost:
//   - heavy ghosts (Wall / Outflow / FarField): L, R and lambda at the
//     nearest fluid node, rotated to the (normal, tangential) frame
//     (bc1.rs:294-312); every thread runs the same six rows, so no lane waits
//     on another's branch. The 80 doubles of a ghost go through shared
//     memory and are stored into its record by whole warps (coalesced);
//   - cheap ghosts (ReflectiveWall, ZerothOrder, Periodic, Constant,
//     TimeDependent), six threads each, complete.
// k_ghosts, heavy ghosts on persistent warps, one ghost at a time per warp.
// A ghost's record (S_r, w, d, the E_r stencil and this stage's L, R,
// lambda; 10.5 KB) arrives in shared memory by one bulk copy (cp.async.bulk,
// completion on an mbarrier). One record buffer per warp: L, R and lambda
// are copied out of it first, and once step 3 has read S_r and w (and d is
// in registers) the next ghost's copy is issued into the same buffer, so the
// table stream overlaps steps 4-6, and 12 warps fit on an SM.
// Per ghost:
//   1. the E_r stencil states (E_0..E_4, 55 nodes, two per lane) were
//      gathered while the ghost before was processed; the fetches for the
//      next ghost are spread over the steps so that none waits on another;
//   2. lanes spread over the 55 stencil nodes: rotate the momentum and
//      project on the six characteristic fields (bc1.rs:209-219);
//   3. the 70 dot products with the stencil data, all six fields at once,
//      in three slots of 25, 16 and 4 terms (a fixed per-lane schedule):
//      the 55 rows of S_0..S_4, each stored as its beta term
//      d_c,a (S_r d_c)_a, and the 15 rows w_{r,k}, V^(k)_{c,r} = w_{r,k} . d_c
//      (bc1.rs:221-244); S_r is stored transposed so the lanes of one order
//      read consecutive words;
//   4. lanes (c, r): beta_{c,r} = the sum of its row terms in order and
//      alpha = d_r / (eps + beta)^q;
//   5. lanes (k, c): V^(k)_c = sum_r alpha_r / sum(alpha) V_r (bc1.rs:247-252);
//   6. FarField rows, R products and the Taylor sum on lanes (bc1.rs:829-923);
//      Wall (two 6x6 LU solves) and Outflow (LODI) on lane 0 (bc1.rs:691-828).
// The per-k loop of the reference (bc1.rs:673-675) recomputes steps 2-4
// unchanged; they are done once. Every sum keeps the reference's order, so
// the no-contraction build reproduces the reference's values.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "physics.cuh"
#include "ghost_rows.cuh"
#include "mbar.cuh"

namespace rh3t {

#ifdef RH3T_EXACT
constexpr bool kExactG = true;
#else
constexpr bool kExactG = false;
#endif

constexpr int GH_WARPS = 4;
constexpr int GH_BLOCKS_PER_SM = 3;
constexpr int GH_PREP_THREADS = 64; // 41.6 KB of staging per block: 5 blocks per SM
__constant__ int kStOff[6] = {0, 1, 5, 14, 30, 55};
__constant__ int kSOff[6] = {0, 1, 17, 98, 354, 979};
__constant__ int kWOff[6] = {0, 1, 9, 36, 100, 225};

struct GhostWarp {
    double rec[1][GH_REC]; // the heavy record (the next one is copied in during step 5)
    double LR[80];         // this ghost's L, R, lambda (copied out of the record)
    double D[56][6];       // characteristic data d_c at stencil node a, row d_row(a)
    double ACC[56][6];     // d_c,a (S_r d_c)_a at stencil row a; later u[5][6] and vinf[6]
    double alpha[6][5];
    double V[6][15];       // [c][r (r + 1) / 2 + k], k <= r
    double v[5][6];        // V^(k)_c
    GhostRec cur;          // this ghost's GhostRec (copied in while the ghost before it ran)
    unsigned long long bar[2];
};
static_assert(sizeof(GhostWarp) % 16 == 0, "records stay 16-byte aligned");
constexpr int GH_SMEM = GH_WARPS * (int)sizeof(GhostWarp);
constexpr int GH_LR_R = GH_R - GH_L, GH_LR_LAM = GH_LAM - GH_L;

// ---------------------------------------------------------------- bulk copy
// one thread: expect `bytes` on bar, then copy global -> shared (16-byte
// aligned addresses, bytes a multiple of 16). The buffer is reused: the
// proxy fence orders the warp's earlier reads of it (generic proxy, made
// visible to this thread by the __syncwarp before every call) before the
// copy's writes (async proxy).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// bc1.rs:467-469 solve6 with LAPACK getrf/getrs semantics
__device__ bool solve6(double A[6][6], double b[6]) {
    int piv[6];
    for (int j = 0; j < 6; ++j) {
        int p = j;
        double mx = fabs(A[j][j]);
        for (int i = j + 1; i < 6; ++i)
            if (fabs(A[i][j]) > mx) { mx = fabs(A[i][j]); p = i; }
        piv[j] = p;
        if (A[p][j] == 0.0) return false;
        if (p != j)
            for (int k = 0; k < 6; ++k) { double t = A[j][k]; A[j][k] = A[p][k]; A[p][k] = t; }
        double rcp = 1.0 / A[j][j];
        for (int i = j + 1; i < 6; ++i) A[i][j] *= rcp;
        for (int k = j + 1; k < 6; ++k)
            for (int i = j + 1; i < 6; ++i) A[i][k] -= A[i][j] * A[j][k];
    }
    for (int j = 0; j < 6; ++j)
        if (piv[j] != j) { double t = b[j]; b[j] = b[piv[j]]; b[piv[j]] = t; }
    for (int k = 0; k < 6; ++k)
        for (int i = k + 1; i < 6; ++i) b[i] -= b[k] * A[i][k];
    for (int k = 5; k >= 0; --k) {
        b[k] /= A[k][k];
        for (int i = 0; i < k; ++i) b[i] -= b[k] * A[i][k];
    }
    return true;
}

// out[i] = sum_j R[i][j] x[j] with R stored by column (Rc[6 j + i])
__device__ __forceinline__ void r_times(const double* Rc, const double x[6], double* out) {
    for (int i = 0; i < 6; ++i) {
        double acc = 0.0;
        for (int j = 0; j < 6; ++j) acc += Rc[6 * j + i] * x[j];
        out[i] = acc;
    }
}

// Wall (bc1.rs:691-756) and Outflow (bc1.rs:760-828) rows on one lane;
// fills u[5][6]. Returns false when an ILW system is singular.
__device__ __noinline__ bool serial_tail(const Inst& I, const GhostRec& Rg, const double* LR,
                                         const double (*v)[6], double (*u)[6]) {
    const DevParams& P = I.P;
    const double* L = LR;
    const double* Rc = LR + GH_LR_R;
    if (Rg.kind == BC_WALL) {
        double A0[6][6], rhs0[6];
        for (int i = 0; i < 6; ++i)
            for (int k = 0; k < 6; ++k) A0[i][k] = L[6 * i + k];
        for (int k = 0; k < 6; ++k) A0[0][k] = k == 1 ? 1.0 : 0.0;
        for (int k = 0; k < 6; ++k) rhs0[k] = v[0][k];
        rhs0[0] = 0.0;
        if (!solve6(A0, rhs0)) return false;
        for (int k = 0; k < 6; ++k) u[0][k] = rhs0[k];
        const double gi = P.gamma_i - 1.0, ge = P.gamma_e - 1.0, gr = P.gamma_r - 1.0;
        const double gt = gi + ge + gr;
        const double u1 = u[0][0], u3 = u[0][2];
        double row1[6] = {-gt * sqd(u3) / (6.0 * sqd(u1)), 0.0, gt * u3 / (6.0 * u1), -ge, -gi, -gr};
        double A1[6][6], rhs1[6];
        for (int i = 0; i < 6; ++i)
            for (int k = 0; k < 6; ++k) A1[i][k] = L[6 * i + k];
        for (int k = 0; k < 6; ++k) A1[0][k] = row1[k];
        for (int k = 0; k < 6; ++k) rhs1[k] = v[1][k];
        rhs1[0] = 0.0;
        if (!solve6(A1, rhs1)) return false;
        for (int k = 0; k < 6; ++k) u[1][k] = rhs1[k];
        for (int k = 2; k <= 4; ++k) r_times(Rc, v[k], u[k]);
        return true;
    }
    // Outflow
    const DevBC& bc = I.bcs[Rg.bc];
    r_times(Rc, v[0], u[0]);
    const double rho0 = u[0][0];
    const double un0 = u[0][1] / rho0, ut0 = u[0][2] / rho0;
    const double w2 = un0 * un0 + ut0 * ut0;
    const double ee1 = u[0][3] / rho0 - w2 / 6.0, ei1 = u[0][4] / rho0 - w2 / 6.0, er1 = u[0][5] / rho0 - w2 / 6.0;
    const double ge = P.gamma_e - 1.0, gi = P.gamma_i - 1.0, gr = P.gamma_r - 1.0;
    const double p0 = rho0 * (ge * ee1 + gi * ei1 + gr * er1);
    const double a2 = P.gamma_e * ge * ee1 + P.gamma_i * gi * ei1 + P.gamma_r * gr * er1;
    const double a = sqrt(a2);
    const double lambda1 = un0 - a;
    double rhs1[6];
    for (int k = 0; k < 6; ++k) rhs1[k] = v[1][k];
    if (lambda1 < 0.0) {
        const double m_local = fabs(un0 / a);
        const double l1 = bc.sigma * (1.0 - sqd(m_local)) * a / bc.l_domain * (p0 - bc.p_inf);
        rhs1[0] = l1 / lambda1;
    }
    r_times(Rc, rhs1, u[1]);
    for (int k = 2; k <= 4; ++k) r_times(Rc, v[k], u[k]);
    return true;
}

// ---------------------------------------------------------------- preparation
__device__ void cheap_ghost(const Inst& I, const GhostRec& Rg, int c, int stage) {
    double* buf = const_cast<double*>(stage_src(I, stage));
    const long long plane = I.plane;
    const DevBC& bc = I.bcs[Rg.bc];
    double val;
    if (Rg.kind == BC_CONSTANT) {
        val = bc.state[c]; // bc1.rs:631-633
    } else if (Rg.kind == BC_TIME_DEPENDENT) {
        const double xs = bc.td_x0 + bc.td_speed * I.sc->t_stage[stage]; // bc1.rs:634-636, init.rs:61-65
        val = Rg.p0x <= xs ? bc.td_left[c] : bc.td_right[c];
    } else if (Rg.kind == BC_REFLECTIVE_WALL) {
        double s[6]; // bc1.rs:930-1037
        load6(buf, plane, Rg.src, s);
        const double mom_n = s[1] * Rg.nx + s[2] * Rg.ny;
        val = c == 1 ? s[1] - 2.0 * mom_n * Rg.nx : (c == 2 ? s[2] - 2.0 * mom_n * Rg.ny : s[c]);
    } else {
        val = buf[c * plane + Rg.src]; // ZerothOrder bc1.rs:471-545, Periodic bc1.rs:547-607
    }
    if (!isfinite(val)) report(I, 1 + 2 * stage, 2, (unsigned)Rg.gid);
    buf[c * plane + Rg.node] = val;
}

// ---------------------------------------------------------------- heavy ghosts
// L, R and lambda at the nearest fluid node of heavy ghost Rg in its
// (normal, tangential) frame (bc1.rs:294-312): LR[6c + k] = L[c][k],
// LR[36 + 6c + i] = R[i][c], LR[72 + c] = lambda_c
__device__ __forceinline__ void local_lr(const Inst& I, const GhostRec& Rg, const double* __restrict__ buf,
                                         double* LR, int stride) {
    const DevParams& P = I.P;
    double s[6];
    load6(buf, I.plane, Rg.src, s);
    const double mom_n = s[1] * Rg.nx + s[2] * Rg.ny;
    const double mom_t = -s[1] * Rg.ny + s[2] * Rg.nx;
    const double q6[6] = {s[0], mom_n, mom_t, s[3], s[4], s[5]};
    const Prim d1 = prim_from_state(q6, P);
    const Roe q = roe_average(q6[0], d1, q6[0], d1, P);
    for (int row = 0; row < 6; ++row) {
        double Lr[6], Rc[6], lam;
        l_row<0>(row, q, P, Lr);
        r_col<0>(row, q, P, Rc, lam);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            LR[(6 * row + k) * stride] = Lr[k];
            LR[(GH_LR_R + 6 * row + k) * stride] = Rc[k];
        }
        LR[(GH_LR_LAM + row) * stride] = lam;
    }
}

// blocks [0, nbp): L, R, lambda of one heavy ghost per thread, staged in
// shared memory ([value][thread], stride GH_PREP_THREADS + 1) and stored by
// whole warps into the records; blocks [nbp, ...): cheap ghosts
constexpr int GH_PREP_SMEM = GH_LR * (GH_PREP_THREADS + 1) * (int)sizeof(double);
__global__ void __launch_bounds__(GH_PREP_THREADS) k_ghost_prep(const Inst* __restrict__ insts,
                                                               const GhostRec* __restrict__ heavy, int nh,
                                                               const GhostRec* __restrict__ cheap, int nc,
                                                               double* __restrict__ hrec, int stage, int nbp) {
    extern __shared__ __align__(16) double prep_smem[];
    if ((int)blockIdx.x < nbp) {
        constexpr int ST = GH_PREP_THREADS + 1;
        const int g0 = blockIdx.x * GH_PREP_THREADS, g = g0 + threadIdx.x;
        if (g < nh) {
            const GhostRec Rg = heavy[g];
            const Inst& I = insts[Rg.inst];
            if (!has_error(I)) local_lr(I, Rg, stage_src(I, stage), prep_smem + threadIdx.x, ST);
        }
        __syncthreads();
        // warp w stores the 80 values of ghosts g0 + 32 w .. g0 + 32 w + 31
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        for (int j = 0; j < 32; ++j) {
            const int t = 32 * w + j, gj = g0 + t;
            if (gj >= nh) break;
            double* r = hrec + (size_t)__ldg(&heavy[gj].heavy) * GH_REC + GH_L;
            for (int e = lane; e < GH_LR; e += 32) r[e] = prep_smem[e * ST + t];
        }
    } else {
        const int t = (blockIdx.x - nbp) * GH_PREP_THREADS + threadIdx.x;
        const int g = t / 6, c = t - 6 * (t / 6);
        if (g >= nc) return;
        const GhostRec Rg = cheap[g];
        const Inst& I = insts[Rg.inst];
        if (has_error(I)) return;
        cheap_ghost(I, Rg, c, stage);
    }
}

// characteristic data of stencil node a from its state (bc1.rs:209-219)
__device__ __forceinline__ void project_node(GhostWarp& G, const double* __restrict__ L, const double s[6],
                                             double nx, double ny, int a) {
    const double mn = s[1] * nx + s[2] * ny;
    const double mt = -s[1] * ny + s[2] * nx;
    const double u6[6] = {s[0], mn, mt, s[3], s[4], s[5]};
    double d[6];
#pragma unroll
    for (int c = 0; c < 6; ++c)
        d[c] = L[6 * c + 0] * u6[0] + L[6 * c + 1] * u6[1] + L[6 * c + 2] * u6[2] + L[6 * c + 3] * u6[3] +
               L[6 * c + 4] * u6[4] + L[6 * c + 5] * u6[5];
    store_d6(G.D[d_row(a)], d);
}

// source of a step-3 row: S_r transposed in the record (stride m, so the
// lanes of one order read consecutive words), or w_{r,k} (stride 1)
__device__ __forceinline__ const double* row_src(const double* __restrict__ rec, unsigned code, int m, int& stride) {
    const bool wr = (code >> 8) != 0;
    const int r = (int)((code >> 5) & 7u), ix = (int)(code & 31u);
    stride = wr ? 1 : m;
    return wr ? rec + GH_W + kWOff[r] + ix * m : rec + GH_S + kSOff[r] + ix;
}

// an S row stores d_c,a (S_r d_c)_a, the term of beta_{c,r}; a w row stores
// V^(k)_{c,r} = w_{r,k} . d_c
__device__ __forceinline__ void row_out(GhostWarp& G, unsigned code, const double acc[6]) {
    const int r = (int)((code >> 5) & 7u), ix = (int)(code & 31u);
    if ((code >> 8) != 0) {
#pragma unroll
        for (int c = 0; c < 6; ++c) G.V[c][r * (r + 1) / 2 + ix] = acc[c];
    } else {
        double d[6], p[6];
        load_d6(G.D[kDOff[r] + ix], d);
#pragma unroll
        for (int c = 0; c < 6; ++c) p[c] = d[c] * acc[c];
        store_d6(G.ACC[kStOff[r] + ix], p);
    }
}

// two rows of one order for all six fields c, each summed over b in order
// (bc1.rs:224-236)
__device__ __forceinline__ void dot_pair(GhostWarp& G, const double* __restrict__ rec, unsigned codes) {
    if (codes == kPairNone) return;
    const unsigned c1 = codes & 0xffffu, c2 = codes >> 16;
    const int r = (int)((c1 >> 5) & 7u);
    const int m = (r + 1) * (r + 1);
    const double(*__restrict__ D)[6] = G.D + kDOff[r];
    int st1, st2;
    const double* __restrict__ p1 = row_src(rec, c1, m, st1);
    const double* __restrict__ p2 = row_src(rec, c2, m, st2);
    double a1[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, a2[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
    for (int b = 0; b < m; ++b) {
        const double x1 = p1[b * st1], x2 = p2[b * st2];
        double d[6];
        load_d6(D[b], d);
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            a1[c] += x1 * d[c];
            a2[c] += x2 * d[c];
        }
    }
    row_out(G, c1, a1);
    row_out(G, c2, a2);
}

// Fetches for the warp's next ghost (record slot n_heavy, -1 for none, and
// instance n_inst, loaded before this ghost's wait) are spread over the steps
// so that no load waits on the one before it: its stencil indices and state
// buffer after step 3, its stencil states (n0, n1) and its instance's error
// flag (n_skip) after step 4, its record once step 3 has read this one.
__device__ __forceinline__ void heavy_ghost(const Inst* __restrict__ insts, const Inst& I, const GhostRec& Rg,
                                            GhostWarp& G, const double* __restrict__ rec,
                                            const double* __restrict__ hrec, int lane, int stage,
                                            unsigned slot_a, unsigned slot_b, double dr, const double s0[6],
                                            const double s1[6], int n_heavy, int n_inst, double n0[6],
                                            double n1[6], bool& n_skip) {
    const DevParams& P = I.P;
    double* buf = const_cast<double*>(stage_src(I, stage));
    const long long plane = I.plane;
    const double nx = Rg.nx, ny = Rg.ny;
    const double* L = G.LR;
    const double* Rc = G.LR + GH_LR_R;
    const double* lam = G.LR + GH_LR_LAM;
    // 2. characteristic data of the 55 stencil nodes
    project_node(G, L, s0, nx, ny, lane);
    if (lane + 32 < 55) project_node(G, L, s1, nx, ny, lane + 32);
    __syncwarp();
    // 3. the 70 rows: d_c,a (S_r d_c)_a and V^(k)_{c,r}
    dot_pair(G, rec, slot_a);
    dot_pair(G, rec, slot_b);
    // the next ghost's stencil indices, state buffer and error flag address
    int st0 = 0, st1 = 0;
    const double* nbuf = nullptr;
    long long nplane = 0;
    const DevError* nerr = nullptr;
    if (n_heavy >= 0) {
        const int32_t* st = reinterpret_cast<const int32_t*>(hrec + (size_t)n_heavy * GH_REC + GH_ST);
        st0 = __ldg(&st[lane]);
        if (lane + 32 < 55) st1 = __ldg(&st[lane + 32]);
        nbuf = stage_src(insts[n_inst], stage);
        nplane = insts[n_inst].plane;
        nerr = insts[n_inst].err;
    }
    __syncwarp();
    // the record is not read below: bring in the next ghost's
    if (lane == 0 && n_heavy >= 0) bulk_load(G.rec[0], hrec + (size_t)n_heavy * GH_REC, GH_REC * 8, &G.bar[0]);
    // 4. lanes (c, r): beta_{c,r} = sum_a d_a (S d)_a in order, alpha = d_r / (eps + beta)^q
    if (lane < 30) {
        const int c = lane / 5, r = lane - 5 * (lane / 5);
        const int m = (r + 1) * (r + 1), off = kStOff[r];
        double beta = 0.0;
#pragma unroll 5
        for (int a = 0; a < m; ++a) beta += G.ACC[off + a][c];
        const double x = P.eps + beta;
        double xq;
        if (!kExactG && P.weno_q == 10.0) { // four products (within a few ulp) in the FMA build
            const double x2 = x * x, x4 = x2 * x2, x8 = x4 * x4;
            xq = x8 * x2;
        } else {
            xq = pow_q(x, P.weno_q); // correctly rounded, as the reference's powf
        }
        G.alpha[c][r] = dr / xq;
    }
    // the next ghost's stencil states (used in its step 2) and error flag
    if (n_heavy >= 0) {
        load6(nbuf, nplane, st0, n0);
        if (lane + 32 < 55) load6(nbuf, nplane, st1, n1);
        n_skip = nerr->key != ~0ull;
    }
    __syncwarp();
    // 5. nonlinear weights (bc1.rs:247-252); V^(k)_r = 0 for k > r
    if (lane < 30) {
        const int k = lane / 6, c = lane - 6 * (lane / 6);
        double asum = 0.0;
        for (int r = 0; r < 5; ++r) asum += G.alpha[c][r];
        const Recip ra = recip(asum); // five quotients by one divisor (IEEE results, divrn.cuh)
        double res = 0.0;
        for (int r = 0; r < 5; ++r)
            res += div_rn(G.alpha[c][r], ra) * (k <= r ? G.V[c][r * (r + 1) / 2 + k] : 0.0);
        G.v[k][c] = res;
    }
    __syncwarp();
    // 6. BC rows, R products, Taylor expansion (bc1.rs:690-924)
    double (*u)[6] = reinterpret_cast<double (*)[6]>(&G.ACC[0][0]); // ACC is dead here
    double* vinf = &G.ACC[5][0];
    bool ok = true;
    if (Rg.kind == BC_FAR_FIELD) {
        const DevBC& bc = I.bcs[Rg.bc];
        if (lane < 6) {
            const double* ui = bc.state;
            const double uinf[6] = {ui[0], ui[1] * nx + ui[2] * ny, -ui[1] * ny + ui[2] * nx, ui[3], ui[4], ui[5]};
            double acc = 0.0;
            for (int j = 0; j < 6; ++j) acc += L[6 * lane + j] * uinf[j];
            vinf[lane] = acc;
        }
        __syncwarp();
        if (lane < 30) {
            const int k = lane / 6, i = lane - 6 * (lane / 6);
            double acc = 0.0;
            for (int m2 = 0; m2 < 6; ++m2) {
                const double x = lam[m2] < 0.0 ? (k == 0 ? vinf[m2] : 0.0) : G.v[k][m2];
                acc += Rc[6 * m2 + i] * x;
            }
            u[k][i] = acc;
        }
    } else if (lane == 0) {
        ok = serial_tail(I, Rg, G.LR, G.v, u);
    }
    __syncwarp();
    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    if (!ok) {
        if (lane == 0) report(I, 1 + 2 * stage, 3, (unsigned)Rg.gid);
        return;
    }
    double g = 0.0;
    if (lane < 6) {
        g = u[0][lane];
        double coef = 1.0;
        for (int k = 1; k <= 4; ++k) {
            coef *= Rg.dist / (double)k;
            g = g + coef * u[k][lane];
        }
    }
    const double mn = __shfl_sync(0xffffffffu, g, 1), mt = __shfl_sync(0xffffffffu, g, 2);
    if (lane < 6) {
        const double out = lane == 1 ? mn * nx - mt * ny : (lane == 2 ? mn * ny + mt * nx : g);
        buf[lane * plane + Rg.node] = out;
        if (!isfinite(out)) report(I, 1 + 2 * stage, 2, (unsigned)Rg.gid);
    }
}

// stencil states of ghost g (lane a and a + 32), from the record in global memory
__device__ __forceinline__ void gather_stencil(const Inst& I, const double* __restrict__ grec, int lane, int stage,
                                               double s0[6], double s1[6]) {
    const int32_t* st = reinterpret_cast<const int32_t*>(grec + GH_ST);
    const double* buf = stage_src(I, stage);
    load6(buf, I.plane, st[lane], s0);
    if (lane + 32 < 55) load6(buf, I.plane, st[lane + 32], s1);
}

// warps take the heavy ghosts in turn (record of the next one in flight; the
// next ghost's GhostRec is loaded at the start of a ghost and kept in shared
// memory, so a ghost starts without a dependent global load: 4.5% faster)
__global__ void __launch_bounds__(GH_WARPS * 32, GH_BLOCKS_PER_SM) k_ghosts(const Inst* __restrict__ insts,
                                                         const GhostRec* __restrict__ heavy, int nh,
                                                         const double* __restrict__ hrec, int stage) {
    extern __shared__ __align__(128) unsigned char gh_smem[];
    const int lane = threadIdx.x & 31;
    GhostWarp& G = reinterpret_cast<GhostWarp*>(gh_smem)[threadIdx.x >> 5];
    const int stride = gridDim.x * GH_WARPS;
    int g = blockIdx.x * GH_WARPS + (threadIdx.x >> 5);
    if (g < nh) { // warp-uniform
        const unsigned slot_a = kSlotA[lane], slot_b = kSlotB[lane];
        if (lane == 0) {
            mbar_init(&G.bar[0], 1);
            mbar_fence_init();
            bulk_load(G.rec[0], hrec + (size_t)heavy[g].heavy * GH_REC, GH_REC * 8, &G.bar[0]);
        }
        __syncwarp();
        // stencil states of the warp's first ghost; later ones are gathered
        // while the ghost before them is processed
        constexpr int kRecWords = (int)(sizeof(GhostRec) / 8);
        static_assert(sizeof(GhostRec) % 8 == 0 && kRecWords <= 32, "GhostRec copied as words by one warp");
        double s0[6], s1[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        bool skip;
        {
            const GhostRec& R0 = heavy[g];
            gather_stencil(insts[R0.inst], hrec + (size_t)R0.heavy * GH_REC, lane, stage, s0, s1);
            skip = has_error(insts[R0.inst]);
            if (lane < kRecWords)
                reinterpret_cast<unsigned long long*>(&G.cur)[lane] =
                    __ldg(reinterpret_cast<const unsigned long long*>(&heavy[g]) + lane);
        }
        for (int it = 0; g < nh; ++it, g += stride) {
            const int gn = g + stride;
            int n_heavy = -1, n_inst = 0;
            unsigned long long nword = 0;
            if (gn < nh) {
                n_heavy = __ldg(&heavy[gn].heavy);
                n_inst = __ldg(&heavy[gn].inst);
                if (lane < kRecWords) nword = __ldg(reinterpret_cast<const unsigned long long*>(&heavy[gn]) + lane);
            }
            __syncwarp();
            const GhostRec Rg = G.cur; // loaded while the ghost before ran (no dependent global load here)
            const Inst& I = insts[Rg.inst];
            bool n_skip = false;
            double n0[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, n1[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            const bool ok = __all_sync(0xffffffffu, mbar_wait(&G.bar[0], (uint32_t)(it & 1)));
            if (!ok) {
                if (lane == 0) report(I, 1 + 2 * stage, MBAR_TIMEOUT_CODE, (unsigned)Rg.gid);
                return;
            }
            for (int e = lane; e < GH_LR; e += 32) G.LR[e] = G.rec[0][GH_L + e];
            // d_r of lane (c, r), read here with L/R: every read of the record
            // is then long complete when the next ghost's copy overwrites it
            const double dr = lane < 30 ? G.rec[0][GH_D + lane - 5 * (lane / 5)] : 0.0;
            __syncwarp();
            if (!skip) {
                heavy_ghost(insts, I, Rg, G, G.rec[0], hrec, lane, stage, slot_a, slot_b, dr, s0, s1, n_heavy,
                            n_inst, n0, n1, n_skip);
            } else if (n_heavy >= 0) {
                if (lane == 0) bulk_load(G.rec[0], hrec + (size_t)n_heavy * GH_REC, GH_REC * 8, &G.bar[0]);
                gather_stencil(insts[n_inst], hrec + (size_t)n_heavy * GH_REC, lane, stage, n0, n1);
                n_skip = has_error(insts[n_inst]);
            }
            __syncwarp();
            if (lane < kRecWords) reinterpret_cast<unsigned long long*>(&G.cur)[lane] = nword;
            skip = n_skip;
#pragma unroll
            for (int q = 0; q < 6; ++q) { s0[q] = n0[q]; s1[q] = n1[q]; }
        }
    }
}

void launch_ghosts(cudaStream_t s, const Inst* insts, const GhostRec* heavy, int nh, const GhostRec* cheap, int nc,
                   double* hrec, int stage) {
    if (nh + nc <= 0) return;
    static int sm_count[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (sm_count[dev] == 0) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(k_ghosts, cudaFuncAttributeMaxDynamicSharedMemorySize, GH_SMEM);
        cudaFuncSetAttribute(k_ghost_prep, cudaFuncAttributeMaxDynamicSharedMemorySize, GH_PREP_SMEM);
        sm_count[dev] = n > 0 ? n : 1;
    }
    const int nbp = (nh + GH_PREP_THREADS - 1) / GH_PREP_THREADS;
    const int nbc = (nc * 6 + GH_PREP_THREADS - 1) / GH_PREP_THREADS;
    k_ghost_prep<<<nbp + nbc, GH_PREP_THREADS, GH_PREP_SMEM, s>>>(insts, heavy, nh, cheap, nc, hrec, stage, nbp);
    if (nh > 0) {
        const int nbh = std::min((nh + GH_WARPS - 1) / GH_WARPS, GH_BLOCKS_PER_SM * sm_count[dev]);
        k_ghosts<<<nbh, GH_WARPS * 32, GH_SMEM, s>>>(insts, heavy, nh, hrec, stage);
    }
}

int ghost_launches(int nh, int nc) { return (nh + nc > 0 ? 1 : 0) + (nh > 0 ? 1 : 0); }

// one warp: the ghost update's bounded wait on a fresh mbarrier whose phase
// completes (arrive: one arrival, no bytes expected) or never does; out[0] =
// 1 when the wait gave up
__global__ void k_wait_check(int arrive, int* out) {
    __shared__ unsigned long long bar;
    const int lane = threadIdx.x & 31;
    if (lane == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
        if (arrive)
            mbar_arrive(&bar);
    }
    __syncwarp();
    const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar, 0u));
    if (lane == 0) out[0] = ok ? 0 : 1;
}

} // namespace rh3t

extern "C" int rh3t_wait_check(int32_t device, int32_t arrive, int32_t* timed_out) {
    if (!timed_out) return 7; // RH3T_ERR_INVALID_ARGUMENT
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return 10; // RH3T_ERR_NO_DEVICE
    if (cudaSetDevice(device) != cudaSuccess) return 8;
    int* d = nullptr;
    if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) return 8;
    int h = -1;
    rh3t::k_wait_check<<<1, 32>>>(arrive ? 1 : 0, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return 8; // RH3T_ERR_CUDA
    *timed_out = h;
    return 0;
}
