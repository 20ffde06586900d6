// Interface fluxes (main.rs:165-246: weno.rs:685-802 reconstruction_fast per
// x and y face, plus diffusion.rs:27-50 when diffusion is on).
//
// A block of 6 warps covers 64 faces (a TI x TJ tile, shape chosen per tile)
// in three phases:
//   1. staging: the tile's stencil points (x faces: (TI + 5) x TJ points,
//      y faces: TI x (TJ + 5)) with their primitives and physical flux go to
//      shared memory once (the reference evaluates them once per face, six
//      times per point); then each face's Roe state, from the staged
//      primitives of its points 3 and 2, and its activity flag;
//   2. characteristic pass: a warp takes one characteristic field c for
//      32 faces (one per lane) at a time, two (field, half) pairs per warp,
//      so the row of L, the projections and the two WENO5 reconstructions
//      of f+ and f- are warp-uniform code; g_c goes to shared memory;
//   3. output pass: likewise one component k for 32 faces at a time,
//      returning (R g)_k = sum_c R[k][c] g_c in the reference's summation
//      order (weno.rs:793, 834-843), plus the diffusion flux for k >= 3.
// Point data sit in shared memory as component pairs (double2), so a lane
// reads a point's state and flux with six 16-byte loads.
//
// RH3T_EXACT selects the reference's expressions; otherwise the fastm forms
// (shared reciprocals, one division per WENO5) are used.
#include "common.cuh"
#include "kernels.cuh"
#include "physics.cuh"

namespace rh3t {

#ifdef RH3T_EXACT
constexpr bool kExact = true;
#else
constexpr bool kExact = false;
#endif

// Roe state: u v w2 ee ei er cs2 cs he hi hr b den, then the reciprocals
// the L rows divide by: FMA build 1/cs2, 1/b; no-contraction build RN(1/d)
// of d = den, b, 6 cs2, 3 cs2, gt cs2 (their quotients stay the IEEE ones)
constexpr int NQ = 18;

struct FluxShared {
    double2 U[3][FLUX_NPT]; // (rho, mx), (my, ee), (ei, er)
    double2 F[3][FLUX_NPT];
    double T[3][FLUX_NPT];
    double PR[5][FLUX_NPT]; // u, v, e_e, e_i, e_r of each point (the face Roe averages reuse them)
    double Q[NQ][FLUX_FACES];
    double G[6][FLUX_FACES];
    int act[FLUX_FACES];
};

// face f of the tile -> face (i, j), first stencil point p0 and point stride
template <int DIR>
__device__ __forceinline__ void face_index(const Tile& t, int f, int& i, int& j, int& p0, int& ps) {
    const int r = f >> t.lg, cc = f & ((1 << t.lg) - 1);
    i = t.i + r;
    j = t.j0 + cc;
    if (DIR == 0) { p0 = f; ps = 1 << t.lg; }
    else { p0 = r * ((1 << t.lg) + 5) + cc; ps = 1; }
}

__device__ __forceinline__ void load_q(const FluxShared& S, int f, Roe& q, double& ics2, double& ib) {
    q.u = S.Q[0][f]; q.v = S.Q[1][f]; q.w2 = S.Q[2][f]; q.ee = S.Q[3][f]; q.ei = S.Q[4][f];
    q.er = S.Q[5][f]; q.cs2 = S.Q[6][f]; q.cs = S.Q[7][f]; q.he = S.Q[8][f]; q.hi = S.Q[9][f];
    q.hr = S.Q[10][f]; q.b = S.Q[11][f]; q.den = S.Q[12][f];
    ics2 = S.Q[13][f]; ib = S.Q[14][f];
}

template <int DIR>
__device__ __forceinline__ double char_flux(const FluxShared& S, const DevParams& P, const Recip& rgt, int c, int f,
                                            int p0, int ps) {
    Roe q;
    double ics2, ib;
    load_q(S, f, q, ics2, ib);
    double Lc[6];
    if (kExact) {
        RoeDiv rd;
        const double gt = (P.gamma_i - 1.0) + (P.gamma_e - 1.0) + (P.gamma_r - 1.0);
        rd.den = recip_of(q.den, S.Q[13][f]);
        rd.b = recip_of(q.b, S.Q[14][f]);
        rd.c6 = recip_of(6.0 * q.cs2, S.Q[15][f]);
        rd.c3 = recip_of(3.0 * q.cs2, S.Q[16][f]);
        rd.cg = recip_of(gt * q.cs2, S.Q[17][f]);
        rd.gt = rgt;
        l_row<DIR>(c, q, rd, P, Lc);
    } else {
        fastm::l_row<DIR>(c, q, ics2, ib, P, Lc);
    }
    const double vel = DIR == 0 ? q.u : q.v;
    const double lam = c == 0 ? vel - q.cs : (c == 5 ? vel + q.cs : vel);
    const double a = fabs(lam);
    double fp[6], fm[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const int p = p0 + k * ps;
        const double2 u01 = S.U[0][p], u23 = S.U[1][p], u45 = S.U[2][p];
        const double2 f01 = S.F[0][p], f23 = S.F[1][p], f45 = S.F[2][p];
        const double cf = Lc[0] * f01.x + Lc[1] * f01.y + Lc[2] * f23.x + Lc[3] * f23.y + Lc[4] * f45.x +
                          Lc[5] * f45.y;
        const double cs = Lc[0] * u01.x + Lc[1] * u01.y + Lc[2] * u23.x + Lc[3] * u23.y + Lc[4] * u45.x +
                          Lc[5] * u45.y;
        fp[k] = 0.5 * (cf + a * cs);
        fm[k] = 0.5 * (cf - a * cs);
    }
    if (!kExact)
        return fastm::weno5(fp[0], fp[1], fp[2], fp[3], fp[4], P.eps) +
               fastm::weno5(fm[5], fm[4], fm[3], fm[2], fm[1], P.eps);
    // no-contraction build: the two reconstructions as a two-pass loop over
    // one inlined WENO5 (one copy of its code, no call: the out-of-line
    // version spilled registers around each of its calls and ran 3% slower)
    double r0 = 0.0, r1 = 0.0;
#pragma unroll 1
    for (int s = 0; s < 2; ++s) {
        const bool m = s != 0;
        const double w = weno5(m ? fm[5] : fp[0], m ? fm[4] : fp[1], m ? fm[3] : fp[2], m ? fm[2] : fp[3],
                               m ? fm[1] : fp[4], P.eps);
        if (m) r1 = w;
        else r0 = w;
    }
    return r0 + r1;
}

// The diffusion terms (off in most runs) are out of line: their code stays
// out of the instruction cache of runs without diffusion.
// diffusion.rs:27-50: component 3 <- Te, 4 <- Ti, 5 <- Tr^4 (m3 = 0, 1, 2)
static __device__ __noinline__ void diffusion_out(const FluxShared& S, const DevParams& P, int m3, int p0, int ps,
                                                  double* out) {
    double v[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        const double x = S.T[m3][p0 + m * ps];
        v[m] = m3 == 2 ? pow4d(x) : x;
    }
    const double kap = m3 == 0 ? P.kappa_e : (m3 == 1 ? P.kappa_i : P.kappa_r);
    const double term = kap * (2.0 * v[5] - 25.0 * v[4] + 245.0 * v[3] - 245.0 * v[2] + 25.0 * v[1] - 2.0 * v[0]);
    *out = term / 180.0;
}

// temperatures of staged point p (its state was written to S.U by this thread)
static __device__ __noinline__ void stage_temps(FluxShared& S, int p, const DevParams& P) {
    const double s[6] = {S.U[0][p].x, S.U[0][p].y, S.U[1][p].x, S.U[1][p].y, S.U[2][p].x, S.U[2][p].y};
    double te, ti, tr;
    temps_from_state(s, P, te, ti, tr);
    S.T[0][p] = te; S.T[1][p] = ti; S.T[2][p] = tr;
}

template <int DIR>
__device__ __forceinline__ void face_out(const Inst& I, const FluxShared& S, const Tile& t, int k, int f) {
    const DevParams& P = I.P;
    const int nx = I.nx, ny = I.ny;
    int i, j, p0, ps;
    face_index<DIR>(t, f, i, j, p0, ps);
    Roe q;
    double ics2, ib;
    load_q(S, f, q, ics2, ib);
    double Rr[6], lam_unused;
    r_row<DIR>(k, q, P, Rr, lam_unused);
    const double out = Rr[0] * S.G[0][f] + Rr[1] * S.G[1][f] + Rr[2] * S.G[2][f] + Rr[3] * S.G[3][f] +
                       Rr[4] * S.G[4][f] + Rr[5] * S.G[5][f];
    long long fplane, fidx;
    double *fo, *dfo;
    if (DIR == 0) { fplane = (long long)(nx + 1) * ny; fidx = (long long)i * ny + j; fo = I.fx; dfo = I.dfx; }
    else { fplane = (long long)nx * (ny + 1); fidx = (long long)i * (ny + 1) + j; fo = I.fy; dfo = I.dfy; }
    fo[k * fplane + fidx] = out;
    if (I.diffusion && k >= 3) diffusion_out(S, P, k - 3, p0, ps, dfo + (k - 3) * fplane + fidx);
}

template <int DIR>
__device__ __forceinline__ void flux_tile(const Inst& I, const Tile& t, int stage, FluxShared& S) {
    const DevParams& P = I.P;
    const double* __restrict__ buf = stage_src(I, stage);
    const long long plane = I.plane;
    const int nx = I.nx, ny = I.ny;
    const int cols = 1 << t.lg, rows = FLUX_FACES >> t.lg;
    const int np = DIR == 0 ? (rows + 5) * cols : rows * (cols + 5);
    const bool diff = I.diffusion != 0;
    // ---- 1. staging: points (state, primitives, physical flux), then faces
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        int pi, pj;
        if (DIR == 0) { pi = t.i - 3 + (p >> t.lg); pj = t.j0 + (p & (cols - 1)); }
        else { const int r = p / (cols + 5); pi = t.i + r; pj = t.j0 - 3 + (p - r * (cols + 5)); }
        double s[6] = {1.0, 0.0, 0.0, 1.0, 1.0, 1.0};
        if (pi >= -RH3T_PAD && pi < nx + RH3T_PAD && pj >= -RH3T_PAD && pj < ny + RH3T_PAD)
            load6(buf, plane, node_of(I, pi, pj), s);
        Prim d = kExact ? prim_from_state(s, P) : fastm::prim(s, P);
        double f[6];
        phys_flux<DIR>(s, d, f);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            S.U[k][p] = make_double2(s[2 * k], s[2 * k + 1]);
            S.F[k][p] = make_double2(f[2 * k], f[2 * k + 1]);
        }
        S.PR[0][p] = d.u; S.PR[1][p] = d.v; S.PR[2][p] = d.e_e; S.PR[3][p] = d.e_i; S.PR[4][p] = d.e_r;
        if (diff) stage_temps(S, p, P);
    }
    __syncthreads();
    for (int f = threadIdx.x; f < FLUX_FACES; f += blockDim.x) {
        int i, j, p0, ps;
        face_index<DIR>(t, f, i, j, p0, ps);
        bool valid = DIR == 0 ? (i <= nx && j < ny) : (i < nx && j <= ny);
        if (valid) {
            const uint8_t m0 = I.mask[node_of(I, i, j)];
            const uint8_t m1 = DIR == 0 ? I.mask[node_of(I, i - 1, j)] : I.mask[node_of(I, i, j - 1)];
            valid = (m0 | m1) != 0;
        }
        S.act[f] = valid ? 1 : 0;
        if (!valid) continue;
        // points[3] and points[2] of the face: the staged states and primitives
        // (the same functions of the same states as a fresh evaluation)
        const int p3 = p0 + 3 * ps, p2 = p0 + 2 * ps;
        Prim d3, d2;
        d3.u = S.PR[0][p3]; d3.v = S.PR[1][p3]; d3.e_e = S.PR[2][p3]; d3.e_i = S.PR[3][p3]; d3.e_r = S.PR[4][p3];
        d2.u = S.PR[0][p2]; d2.v = S.PR[1][p2]; d2.e_e = S.PR[2][p2]; d2.e_i = S.PR[3][p2]; d2.e_r = S.PR[4][p2];
        const double rho3 = S.U[0][p3].x, rho2 = S.U[0][p2].x;
        Roe q;
        if (kExact) {
            q = roe_average(rho3, d3, rho2, d2, P);
        } else {
            const double a6[6] = {sqrt(rho3), d3.u, d3.v, d3.e_e, d3.e_i, d3.e_r};
            const double b6[6] = {sqrt(rho2), d2.u, d2.v, d2.e_e, d2.e_i, d2.e_r};
            q = fastm::roe(a6, b6, P);
        }
        double qv[NQ] = {q.u, q.v, q.w2, q.ee, q.ei, q.er, q.cs2, q.cs, q.he, q.hi, q.hr, q.b, q.den,
                         0.0, 0.0, 0.0, 0.0, 0.0};
        if (kExact) {
            const RoeDiv rd = roe_div(q, P);
            qv[13] = rd.den.y; qv[14] = rd.b.y; qv[15] = rd.c6.y; qv[16] = rd.c3.y; qv[17] = rd.cg.y;
        } else {
            qv[13] = 1.0 / q.cs2;
            qv[14] = 1.0 / q.b;
        }
#pragma unroll
        for (int k = 0; k < NQ; ++k) S.Q[k][f] = qv[k];
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // Each warp takes one heavy and one light half in both passes, so the
    // six warps reach the barrier (and the block's end) together: the energy
    // fields' L rows hold most of a face's divisions (x faces: fields 1-3,
    // 0 and 5 acoustic, 4 transverse; y faces: 2-4, 0 and 5, 1), and so do
    // the energy components' R rows (3-5). Field of warp w for faces 0..31
    // and 32..63, one hex digit per warp:
    constexpr unsigned kC0 = DIR == 0 ? 0x450321u : 0x150432u;
    constexpr unsigned kC1 = DIR == 0 ? 0x321450u : 0x432150u;
    Recip rgt = {1.0, 1.0, false};
    if (kExact) rgt = recip((P.gamma_i - 1.0) + (P.gamma_e - 1.0) + (P.gamma_r - 1.0));
    // ---- 2. characteristic pass: field c of faces lane and lane + 32 (a
    // loop, not unrolled: one copy of the pass's code keeps the kernel
    // within the instruction cache)
#pragma unroll 1
    for (int h = 0; h < FLUX_FACES / 32; ++h) {
        const int f = lane + 32 * h;
        const int c = (int)(((h ? kC1 : kC0) >> (4 * w)) & 15u); // warp-uniform
        if (S.act[f]) {
            int i, j, p0, ps;
            face_index<DIR>(t, f, i, j, p0, ps);
            S.G[c][f] = char_flux<DIR>(S, P, rgt, c, f, p0, ps);
        }
    }
    __syncthreads();
    // ---- 3. output pass: component k of faces lane and lane + 32
#pragma unroll 1
    for (int h = 0; h < FLUX_FACES / 32; ++h) {
        const int f = lane + 32 * h;
        const int k = h ? (w + 3) % 6 : w;
        if (S.act[f]) face_out<DIR>(I, S, t, k, f);
    }
}

// FMA build: 64 registers, 5 blocks (30 warps) per SM instead of 4 at the
// uncapped 76. No-contraction build: 80 registers, 4 blocks (its divisions
// by shared reciprocals keep more values live; at 64 it spills).
#ifndef FLUX_MIN_BLOCKS_EXACT
#define FLUX_MIN_BLOCKS_EXACT 4
#endif
constexpr int FLUX_MIN_BLOCKS = kExact ? FLUX_MIN_BLOCKS_EXACT : 5;
// x faces and y faces in two launches: each kernel holds one direction's
// code, half of what an instruction cache shared by both would need
template <int DIR>
__global__ void __launch_bounds__(FLUX_THREADS, FLUX_MIN_BLOCKS) k_flux(const Inst* __restrict__ insts,
                                                                     const Tile* __restrict__ tiles, int stage) {
    __shared__ FluxShared S;
    const Tile t = tiles[blockIdx.x];
    const Inst& I = insts[t.inst];
    if (has_error(I)) return;
    flux_tile<DIR>(I, t, stage, S);
}

void launch_flux(cudaStream_t s, const Inst* insts, const Tile* tx, int ntx, const Tile* ty, int nty, int stage) {
    if (ntx > 0) k_flux<0><<<ntx, FLUX_THREADS, 0, s>>>(insts, tx, stage);
    if (nty > 0) k_flux<1><<<nty, FLUX_THREADS, 0, s>>>(insts, ty, stage);
}

int flux_launches(int ntx, int nty) { return (ntx > 0 ? 1 : 0) + (nty > 0 ? 1 : 0); }

} // namespace rh3t
