// Adjoint (vector-Jacobian products) of the semi-discrete operator l() and of
// the SSP-RK3 step (main.rs:135-373), hand-written per kernel of the forward
// path. No reference counterpart: the reference has no derivative code.
//
// vjp of l at a stage state X (ghost nodes of X set by the forward ghost
// update) for a cotangent rbar on the fluid cells, accumulated into Ubar:
//   k_adj_faces  x and y faces: the face flux cotangent from rbar, then the
//                reverse of weno.rs:685-802 (R g, WENO5 weights, Lax-Friedrichs
//                split, L projections, the Roe average of points 2 and 3, the
//                six physical fluxes) and of diffusion.rs:27-50 -> node
//                cotangents W (fluid and ghost nodes, atomic adds);
//   k_adj_cells  fluid cells: reverse of noncon.rs:288-332 (both directions)
//                and source.rs:7-21 -> W, and the exchange-coefficient
//                cotangents;
//   k_adj_ghosts heavy ghosts (FarField): reverse of bc1.rs:193-255 and
//                829-924 (Taylor sum, R products, incoming-characteristic
//                rows, nonlinear weights, smoothness indicators, the
//                characteristic projection, L and R of the nearest node)
//                from W at the ghost node -> Ubar at the stencil nodes and the
//                nearest node, and the FarField-state cotangent; cheap ghosts
//                (ReflectiveWall, ZerothOrder, Periodic) -> Ubar at the source;
//   k_adj_fluid  Ubar += W on fluid nodes.
// The eigenvector matrices of a face enter through its five Roe-averaged
// scalars (u, v, e_e, e_i, e_r); their partial derivatives come from
// evaluating the same builders (physics.cuh l_row, r_col) over dual numbers
// with five tangents (dual.cuh). Everything else is differentiated by hand.
// Kinks follow the values: d|x|/dx = +1 at 0, max/min pass the derivative to
// the first argument on ties, a FarField row switches on lambda < 0.
#include <algorithm>

#include "common.cuh"
#include "dual.cuh"
#include "kernels.cuh"
#include "physics.cuh"

namespace rh3t {

using D5 = DualN<5>;
using D8 = DualN<8>;

// Roe state from the five averaged scalars (the rest of roe_average)
template <class T>
__device__ __forceinline__ RoeT<T> roe_from_base(T u, T v, T ee, T ei, T er, const DevParams& P) {
    RoeT<T> q;
    q.u = u; q.v = v;
    q.w2 = sqd(u) + sqd(v);
    q.ee = ee; q.ei = ei; q.er = er;
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    q.cs2 = GE * ge * ee + GI * gi * ei + GR * gr * er;
    q.cs = sqrt(q.cs2);
    q.he = 6.0 * gi * gr * (GI * ei - GR * er) + GE * gt * ee * q.w2;
    q.hi = 6.0 * ge * gr * (GR * er - GE * ee) + GI * gt * ei * q.w2;
    q.hr = 6.0 * ge * gi * (GE * ee - GI * ei) + GR * gt * er * q.w2;
    q.b = gt * (36.0 * ge * gi * gr + gt * sqd(q.w2)) * q.cs2;
    q.den = 12.0 * q.cs2;
    return q;
}

// ---------------------------------------------------------------- pointwise vjps
// state.rs:245-276 primitives: cotangents of (u, v, e_e, e_i, e_r, p_e, p_i,
// p_r) -> state cotangent (added to sb)
__device__ __forceinline__ void prim_vjp(const double s[6], const DevParams& P, double bu, double bv, double bee,
                                         double bei, double ber, double bpe, double bpi, double bpr, double sb[6]) {
    const double rho = s[0], u = s[1] / rho, v = s[2] / rho;
    const double w2 = u * u + v * v;
    const double ge = P.gamma_e - 1.0, gi = P.gamma_i - 1.0, gr = P.gamma_r - 1.0;
    const double gp = ge * bpe + gi * bpi + gr * bpr;
    const double bw2 = -(bee + bei + ber) / 6.0 - gp * rho / 6.0;
    double brho = -(s[3] * bee + s[4] * bei + s[5] * ber) / (rho * rho) - gp * w2 / 6.0;
    const double bu2 = bu + 2.0 * u * bw2, bv2 = bv + 2.0 * v * bw2;
    brho -= (bu2 * u + bv2 * v) / rho;
    sb[0] += brho;
    sb[1] += bu2 / rho;
    sb[2] += bv2 / rho;
    sb[3] += bee / rho + ge * bpe;
    sb[4] += bei / rho + gi * bpi;
    sb[5] += ber / rho + gr * bpr;
}

// state.rs:118-135 temperatures: cotangents of (te, ti, tr) -> sb
__device__ __forceinline__ void temps_vjp(const double s[6], const DevParams& P, double bte, double bti, double btr,
                                          double sb[6]) {
    const double rho = s[0], u = s[1] / rho, v = s[2] / rho;
    const double w2 = u * u + v * v;
    double te, ti, tr;
    temps_from_state(s, P, te, ti, tr);
    const double er_term = s[5] / rho - w2 / 6.0;
    const double X = er_term * rho / P.a_rad;
    const double bX = btr * 0.25 * tr / X;
    // te = E_e / (rho cve) - w2 / (6 cve), ti likewise, X = (E_r / rho - w2 / 6) rho / a
    double brho = -s[3] * bte / (rho * rho * P.cve) - s[4] * bti / (rho * rho * P.cvi) - bX * (w2 / 6.0) / P.a_rad;
    const double bw2 = -bte / (6.0 * P.cve) - bti / (6.0 * P.cvi) - bX * rho / (6.0 * P.a_rad);
    const double bu = 2.0 * u * bw2, bv = 2.0 * v * bw2;
    brho -= (bu * u + bv * v) / rho;
    sb[0] += brho;
    sb[1] += bu / rho;
    sb[2] += bv / rho;
    sb[3] += bte / (rho * P.cve);
    sb[4] += bti / (rho * P.cvi);
    sb[5] += bX / P.a_rad;
}

// state.rs:56-85 physical flux: fb (6) -> sb
template <int DIR>
__device__ __forceinline__ void flux_vjp(const double s[6], const Prim& d, const DevParams& P, const double fb[6],
                                         double sb[6]) {
    const double rho = s[0], u = d.u, v = d.v;
    double brho, bu, bv, bp[3], bE[3];
    if (DIR == 0) {
        brho = fb[0] * u + fb[1] * u * u + fb[2] * u * v;
        bu = fb[0] * rho + fb[1] * 2.0 * rho * u + fb[2] * rho * v + fb[3] * (s[3] + d.pe) + fb[4] * (s[4] + d.pi) +
             fb[5] * (s[5] + d.pr);
        bv = fb[2] * rho * u;
        for (int a = 0; a < 3; ++a) { bp[a] = fb[1] + fb[3 + a] * u; bE[a] = fb[3 + a] * u; }
    } else {
        brho = fb[0] * v + fb[1] * u * v + fb[2] * v * v;
        bv = fb[0] * rho + fb[1] * rho * u + fb[2] * 2.0 * rho * v + fb[3] * (s[3] + d.pe) + fb[4] * (s[4] + d.pi) +
             fb[5] * (s[5] + d.pr);
        bu = fb[1] * rho * v;
        for (int a = 0; a < 3; ++a) { bp[a] = fb[2] + fb[3 + a] * v; bE[a] = fb[3 + a] * v; }
    }
    sb[0] += brho;
    sb[3] += bE[0]; sb[4] += bE[1]; sb[5] += bE[2];
    prim_vjp(s, P, bu, bv, 0.0, 0.0, 0.0, bp[0], bp[1], bp[2], sb);
}

// weno.rs:847-886 WENO5: cotangent gb of the result -> ub[5] (added)
__device__ __forceinline__ void weno5_vjp(const double x[5], double eps, double gb, double ub[5]) {
    const double t0 = x[0] - 2.0 * x[1] + x[2], r0 = x[0] - 4.0 * x[1] + 3.0 * x[2];
    const double t1 = x[1] - 2.0 * x[2] + x[3], r1 = x[1] - x[3];
    const double t2 = x[2] - 2.0 * x[3] + x[4], r2 = 3.0 * x[2] - 4.0 * x[3] + x[4];
    const double b0 = 13.0 / 12.0 * t0 * t0 + 0.25 * r0 * r0;
    const double b1 = 13.0 / 12.0 * t1 * t1 + 0.25 * r1 * r1;
    const double b2 = 13.0 / 12.0 * t2 * t2 + 0.25 * r2 * r2;
    const double a0 = 0.1 / sqd(eps + b0), a1 = 0.6 / sqd(eps + b1), a2 = 0.3 / sqd(eps + b2);
    const double S = a0 + a1 + a2;
    const double w0 = a0 / S, w1 = a1 / S, w2 = a2 / S;
    const double p0 = x[0] / 3.0 - 7.0 / 6.0 * x[1] + 11.0 / 6.0 * x[2];
    const double p1 = -x[1] / 6.0 + 5.0 / 6.0 * x[2] + x[3] / 3.0;
    const double p2 = x[2] / 3.0 + 5.0 / 6.0 * x[3] - x[4] / 6.0;
    const double pb0 = w0 * gb, pb1 = w1 * gb, pb2 = w2 * gb;
    const double wb0 = p0 * gb, wb1 = p1 * gb, wb2 = p2 * gb;
    const double m = w0 * wb0 + w1 * wb1 + w2 * wb2;
    const double ab0 = (wb0 - m) / S, ab1 = (wb1 - m) / S, ab2 = (wb2 - m) / S;
    const double bb0 = -2.0 * ab0 * a0 / (eps + b0), bb1 = -2.0 * ab1 * a1 / (eps + b1),
                 bb2 = -2.0 * ab2 * a2 / (eps + b2);
    ub[0] += pb0 / 3.0;
    ub[1] += -7.0 / 6.0 * pb0 - pb1 / 6.0;
    ub[2] += 11.0 / 6.0 * pb0 + 5.0 / 6.0 * pb1 + pb2 / 3.0;
    ub[3] += pb1 / 3.0 + 5.0 / 6.0 * pb2;
    ub[4] += -pb2 / 6.0;
    const double c0 = 13.0 / 6.0 * t0 * bb0, d0 = 0.5 * r0 * bb0;
    ub[0] += c0 + d0; ub[1] += -2.0 * c0 - 4.0 * d0; ub[2] += c0 + 3.0 * d0;
    const double c1 = 13.0 / 6.0 * t1 * bb1, d1 = 0.5 * r1 * bb1;
    ub[1] += c1 + d1; ub[2] += -2.0 * c1; ub[3] += c1 - d1;
    const double c2 = 13.0 / 6.0 * t2 * bb2, d2 = 0.5 * r2 * bb2;
    ub[2] += c2 + 3.0 * d2; ub[3] += -2.0 * c2 - 4.0 * d2; ub[4] += c2 + d2;
}

// Roe base cotangents (u, v, e_e, e_i, e_r) -> state cotangents of the two
// points (sa: points[3] / state1, sb: points[2] / state2), added
__device__ __forceinline__ void roe_vjp(const double sa[6], const double sb_[6], const DevParams& P,
                                        const double bb[5], double ga[6], double gb[6]) {
    const Prim da = prim_from_state(sa, P), db = prim_from_state(sb_, P);
    const double ra = sqrt(sa[0]), rb = sqrt(sb_[0]), rs = ra + rb;
    const double xa[5] = {da.u, da.v, da.e_e, da.e_i, da.e_r}, xb[5] = {db.u, db.v, db.e_e, db.e_i, db.e_r};
    double bra = 0.0, brb = 0.0, pa[5], pb[5];
    for (int k = 0; k < 5; ++k) {
        const double base = (xa[k] * ra + xb[k] * rb) / rs;
        pa[k] = bb[k] * ra / rs;
        pb[k] = bb[k] * rb / rs;
        bra += bb[k] * (xa[k] - base) / rs;
        brb += bb[k] * (xb[k] - base) / rs;
    }
    ga[0] += bra / (2.0 * ra);
    gb[0] += brb / (2.0 * rb);
    prim_vjp(sa, P, pa[0], pa[1], pa[2], pa[3], pa[4], 0.0, 0.0, 0.0, ga);
    prim_vjp(sb_, P, pb[0], pb[1], pb[2], pb[3], pb[4], 0.0, 0.0, 0.0, gb);
}

// Roe base cotangent of (L row c, R column c, lambda_c) cotangents
template <int DIR>
__device__ __forceinline__ void lr_base_vjp(int c, const double base[5], const DevParams& P, const double Lb[6],
                                            const double Rb[6], double lamb, double bb[5]) {
    const RoeT<D5> q = roe_from_base(D5::var(base[0], 0), D5::var(base[1], 1), D5::var(base[2], 2),
                                     D5::var(base[3], 3), D5::var(base[4], 4), P);
    D5 L[6], R[6], lam;
    l_row<DIR>(c, q, P, L);
    r_col<DIR>(c, q, P, R, lam);
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        double acc = lamb * lam.d[m];
#pragma unroll
        for (int j = 0; j < 6; ++j) acc += Lb[j] * L[j].d[m] + Rb[j] * R[j].d[m];
        bb[m] += acc;
    }
}

__device__ __forceinline__ void atomic_add6(double* W, long long plane, long long n, const double v[6]) {
#pragma unroll
    for (int c = 0; c < 6; ++c)
        if (v[c] != 0.0) atomicAdd(&W[c * plane + n], v[c]);
}

// ---------------------------------------------------------------- faces
// rbar: cell cotangent planes (padded, zero off the fluid); W: node cotangents
template <int DIR>
__device__ void face_vjp(const Inst& I, const double* __restrict__ X, const double* __restrict__ rbar,
                         double* __restrict__ W, int i, int j) {
    const DevParams& P = I.P;
    const long long plane = I.plane;
    const int nx = I.nx, ny = I.ny;
    // activity (main.rs:165-246): a face with a fluid cell on either side
    const long long n3 = node_of(I, i, j), n2 = DIR == 0 ? node_of(I, i - 1, j) : node_of(I, i, j - 1);
    if (!(I.mask[n3] | I.mask[n2])) return;
    const double sc = DIR == 0 ? 1.0 / I.dx : 1.0 / I.dy;
    double Fb[6];
    const bool in3 = DIR == 0 ? (i < nx) : (j < ny);
    const bool in2 = DIR == 0 ? (i >= 1) : (j >= 1);
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        const double r3 = in3 && I.mask[n3] ? rbar[c * plane + n3] : 0.0;
        const double r2 = in2 && I.mask[n2] ? rbar[c * plane + n2] : 0.0;
        Fb[c] = (r3 - r2) * sc;
    }
    // stencil points i-3..i+2 (x) / j-3..j+2 (y)
    double s[6][6];
    long long nd[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        nd[k] = DIR == 0 ? node_of(I, i - 3 + k, j) : node_of(I, i, j - 3 + k);
        load6(X, plane, nd[k], s[k]);
    }
    Prim d[6];
    double F[6][6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        d[k] = prim_from_state(s[k], P);
        phys_flux<DIR>(s[k], d[k], F[k]);
    }
    const Roe q = roe_average(s[3][0], d[3], s[2][0], d[2], P);
    const double base[5] = {q.u, q.v, q.ee, q.ei, q.er};
    double sbar[6][6], Fbar[6][6], bb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
        for (int m = 0; m < 6; ++m) { sbar[k][m] = 0.0; Fbar[k][m] = 0.0; }
    // g_c for R-bar needs all six reconstructions first
    double g[6];
    for (int c = 0; c < 6; ++c) {
        double Lc[6];
        l_row<DIR>(c, q, P, Lc);
        const double vel = DIR == 0 ? q.u : q.v;
        const double lam = c == 0 ? vel - q.cs : (c == 5 ? vel + q.cs : vel);
        const double a = fabs(lam);
        double fp[6], fm[6];
        for (int k = 0; k < 6; ++k) {
            double cf = 0.0, cs = 0.0;
            for (int m = 0; m < 6; ++m) { cf += Lc[m] * F[k][m]; cs += Lc[m] * s[k][m]; }
            fp[k] = 0.5 * (cf + a * cs);
            fm[k] = 0.5 * (cf - a * cs);
        }
        g[c] = weno5(fp[0], fp[1], fp[2], fp[3], fp[4], P.eps) + weno5(fm[5], fm[4], fm[3], fm[2], fm[1], P.eps);
    }
    for (int c = 0; c < 6; ++c) {
        double Lc[6], Rc[6], lam;
        l_row<DIR>(c, q, P, Lc);
        r_col<DIR>(c, q, P, Rc, lam);
        // F_i = sum_c R_ic g_c
        double gb = 0.0, Rb[6];
        for (int i2 = 0; i2 < 6; ++i2) { gb += Rc[i2] * Fb[i2]; Rb[i2] = Fb[i2] * g[c]; }
        const double a = fabs(lam);
        double w[6], f[6], fp[6], fm[6];
        for (int k = 0; k < 6; ++k) {
            double cf = 0.0, cs = 0.0;
            for (int m = 0; m < 6; ++m) { cf += Lc[m] * F[k][m]; cs += Lc[m] * s[k][m]; }
            f[k] = cf; w[k] = cs;
            fp[k] = 0.5 * (cf + a * cs);
            fm[k] = 0.5 * (cf - a * cs);
        }
        double fpb[6] = {0, 0, 0, 0, 0, 0}, fmb[6] = {0, 0, 0, 0, 0, 0};
        weno5_vjp(fp, P.eps, gb, fpb);
        {
            const double xm[5] = {fm[5], fm[4], fm[3], fm[2], fm[1]};
            double ubm[5] = {0, 0, 0, 0, 0};
            weno5_vjp(xm, P.eps, gb, ubm);
            fmb[5] += ubm[0]; fmb[4] += ubm[1]; fmb[3] += ubm[2]; fmb[2] += ubm[3]; fmb[1] += ubm[4];
        }
        double ab = 0.0, Lb[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 6; ++k) {
            const double fbk = 0.5 * (fpb[k] + fmb[k]);
            const double wbk = 0.5 * a * (fpb[k] - fmb[k]);
            ab += 0.5 * w[k] * (fpb[k] - fmb[k]);
            for (int m = 0; m < 6; ++m) {
                Lb[m] += wbk * s[k][m] + fbk * F[k][m];
                sbar[k][m] += wbk * Lc[m];
                Fbar[k][m] += fbk * Lc[m];
            }
        }
        const double lamb = lam < 0.0 ? -ab : ab;
        lr_base_vjp<DIR>(c, base, P, Lb, Rb, lamb, bb);
    }
    // Roe average of points 3 and 2
    roe_vjp(s[3], s[2], P, bb, sbar[3], sbar[2]);
    // physical fluxes
#pragma unroll
    for (int k = 0; k < 6; ++k) flux_vjp<DIR>(s[k], d[k], P, Fbar[k], sbar[k]);
    // diffusion.rs:27-50: rhs += -(b - a) cx per face pair, cx = -1 / ds^2
    if (I.diffusion) {
        const double cx = DIR == 0 ? -1.0 / (I.dx * I.dx) : -1.0 / (I.dy * I.dy);
        double Db[3];
        for (int m3 = 0; m3 < 3; ++m3) {
            const double r3 = in3 && I.mask[n3] ? rbar[(3 + m3) * plane + n3] : 0.0;
            const double r2 = in2 && I.mask[n2] ? rbar[(3 + m3) * plane + n2] : 0.0;
            Db[m3] = (r3 - r2) * cx;
        }
        const double cf[6] = {-2.0, 25.0, -245.0, 245.0, -25.0, 2.0};
        const double kap[3] = {P.kappa_e, P.kappa_i, P.kappa_r};
        for (int k = 0; k < 6; ++k) {
            double te, ti, tr;
            temps_from_state(s[k], P, te, ti, tr);
            const double bte = Db[0] * kap[0] * cf[k] / 180.0;
            const double bti = Db[1] * kap[1] * cf[k] / 180.0;
            const double btr = Db[2] * kap[2] * cf[k] / 180.0 * 4.0 * tr * tr * tr;
            temps_vjp(s[k], P, bte, bti, btr, sbar[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) atomic_add6(W, plane, nd[k], sbar[k]);
}

// X, rbar, W: batch-wide plane sets (instance k's 6 padded planes at I.aoff)
__global__ void __launch_bounds__(128) k_adj_faces(const Inst* __restrict__ insts, int k0,
                                                   const double* __restrict__ X, const double* __restrict__ rbar,
                                                   double* __restrict__ W, int dir) {
    const Inst& I = insts[k0 + blockIdx.y];
    if (has_error(I)) return;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (dir == 0) {
        if (t >= (long long)(I.nx + 1) * I.ny) return;
        const int i = (int)(t / I.ny), j = (int)(t % I.ny);
        face_vjp<0>(I, X + I.aoff, rbar + I.aoff, W + I.aoff, i, j);
    } else {
        if (t >= (long long)I.nx * (I.ny + 1)) return;
        const int i = (int)(t / (I.ny + 1)), j = (int)(t % (I.ny + 1));
        face_vjp<1>(I, X + I.aoff, rbar + I.aoff, W + I.aoff, i, j);
    }
}

// ---------------------------------------------------------------- cells
// noncon.rs:288-332 reverse: ob (3) -> cotangents of pe, pi, pr, vel at 9 points
__device__ __forceinline__ void noncon9_vjp(const double pe[9], const double pi[9], const double pr[9],
                                            const double vel[9], double ds, const double ob[3], double pe_b[9],
                                            double pi_b[9], double pr_b[9], double vel_b[9]) {
    const double v = vel[4];
    const double dpe = d6(pe[1], pe[2], pe[3], pe[5], pe[6], pe[7], ds);
    const double dpi = d6(pi[1], pi[2], pi[3], pi[5], pi[6], pi[7], ds);
    const double dpr = d6(pr[1], pr[2], pr[3], pr[5], pr[6], pr[7], ds);
    const double der[3] = {2.0 * dpe - dpi - dpr, 2.0 * dpi - dpe - dpr, 2.0 * dpr - dpe - dpi};
    double n[3][9];
    for (int k = 0; k < 9; ++k) {
        n[0][k] = 2.0 * pe[k] - pi[k] - pr[k];
        n[1][k] = 2.0 * pi[k] - pe[k] - pr[k];
        n[2][k] = 2.0 * pr[k] - pe[k] - pi[k];
    }
    const double jm[3] = {jump8(n[0]), jump8(n[1]), jump8(n[2])};
    const double jp[3] = {jump8(n[0] + 1), jump8(n[1] + 1), jump8(n[2] + 1)};
    const double xl = fmax(v, vel[3]), xr = fmin(v, vel[5]);
    const double cl = fmax(xl, 0.0) / 3.0, cr = fmin(xr, 0.0) / 3.0;
    for (int k = 0; k < 9; ++k) { pe_b[k] = 0.0; pi_b[k] = 0.0; pr_b[k] = 0.0; vel_b[k] = 0.0; }
    double clb = 0.0, crb = 0.0, derb[3], jmb[3], jpb[3];
    for (int a = 0; a < 3; ++a) {
        vel_b[4] += ob[a] * der[a] / 3.0;
        derb[a] = ob[a] * v / 3.0;
        clb += ob[a] * jm[a] / ds;
        crb += ob[a] * jp[a] / ds;
        jmb[a] = ob[a] * cl / ds;
        jpb[a] = ob[a] * cr / ds;
    }
    if (xl >= 0.0) { // fmax(xl, 0) takes xl
        if (v >= vel[3]) vel_b[4] += clb / 3.0;
        else vel_b[3] += clb / 3.0;
    }
    if (xr <= 0.0) {
        if (v <= vel[5]) vel_b[4] += crb / 3.0;
        else vel_b[5] += crb / 3.0;
    }
    // jump8(a) = q(a7..a1) - q(a0..a6) with q the 7-point pulse (noncon.rs:49-57)
    const double qc[7] = {-0.00714285714285723, 0.0595238095238118, -0.240476190476197, 0.759523809523819,
                          0.509523809523803, -0.0904761904761891, 0.00952380952380977};
    double nb[3][9];
    for (int a = 0; a < 3; ++a) {
        for (int k = 0; k < 9; ++k) nb[a][k] = 0.0;
        for (int w = 0; w < 2; ++w) {
            const int o = w; // window start
            const double jb = w == 0 ? jmb[a] : jpb[a];
            for (int t = 0; t < 7; ++t) {
                nb[a][o + 7 - t] += qc[t] * jb; // q(a7, a6, ..., a1)
                nb[a][o + t] -= qc[t] * jb;     // q(a0, ..., a6)
            }
        }
    }
    // der = M dp with M symmetric [[2,-1,-1],[-1,2,-1],[-1,-1,2]]
    const double dpb[3] = {2.0 * derb[0] - derb[1] - derb[2], 2.0 * derb[1] - derb[0] - derb[2],
                           2.0 * derb[2] - derb[0] - derb[1]};
    const double c6 = 1.0 / (60.0 * ds);
    const double w6[7] = {-1.0, 9.0, -45.0, 0.0, 45.0, -9.0, 1.0}; // points 1..7
    for (int t = 0; t < 7; ++t) {
        pe_b[1 + t] += w6[t] * c6 * dpb[0];
        pi_b[1 + t] += w6[t] * c6 * dpb[1];
        pr_b[1 + t] += w6[t] * c6 * dpb[2];
    }
    for (int k = 0; k < 9; ++k) {
        pe_b[k] += 2.0 * nb[0][k] - nb[1][k] - nb[2][k];
        pi_b[k] += 2.0 * nb[1][k] - nb[0][k] - nb[2][k];
        pr_b[k] += 2.0 * nb[2][k] - nb[0][k] - nb[1][k];
    }
}

// pbar: per-instance parameter cotangents [u_inf (6), omega_ei, omega_er]
__global__ void __launch_bounds__(128) k_adj_cells(const Inst* __restrict__ insts, int k0,
                                                   const double* __restrict__ Xb, const double* __restrict__ rbarb,
                                                   double* __restrict__ Wb, double* __restrict__ pbar) {
    const int kk = k0 + blockIdx.y;
    const Inst& I = insts[kk];
    if (has_error(I)) return;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)I.nx * I.ny) return;
    const int i = (int)(t / I.ny), j = (int)(t % I.ny);
    const long long n = node_of(I, i, j);
    if (!I.mask[n]) return;
    const DevParams& P = I.P;
    const long long plane = I.plane;
    const double* X = Xb + I.aoff;
    const double* rb = rbarb + I.aoff;
    double* W = Wb + I.aoff;
    const double ob[3] = {rb[3 * plane + n], rb[4 * plane + n], rb[5 * plane + n]};
    for (int dir = 0; dir < 2; ++dir) {
        double pe[9], pi[9], pr[9], vel[9], s9[9][6];
        for (int q = 0; q < 9; ++q) {
            const long long m = dir == 0 ? node_of(I, i - 4 + q, j) : node_of(I, i, j - 4 + q);
            load6(X, plane, m, s9[q]);
            const Prim d = prim_from_state(s9[q], P);
            pe[q] = d.pe; pi[q] = d.pi; pr[q] = d.pr; vel[q] = dir == 0 ? d.u : d.v;
        }
        double peb[9], pib[9], prb[9], velb[9];
        noncon9_vjp(pe, pi, pr, vel, dir == 0 ? I.dx : I.dy, ob, peb, pib, prb, velb);
        for (int q = 0; q < 9; ++q) {
            double sb[6] = {0, 0, 0, 0, 0, 0};
            prim_vjp(s9[q], P, dir == 0 ? velb[q] : 0.0, dir == 0 ? 0.0 : velb[q], 0.0, 0.0, 0.0, peb[q], pib[q],
                     prb[q], sb);
            const long long m = dir == 0 ? node_of(I, i - 4 + q, j) : node_of(I, i, j - 4 + q);
            atomic_add6(W, plane, m, sb);
        }
    }
    if (I.source) { // source.rs:7-21
        double s[6];
        load6(X, plane, n, s);
        double te, ti, tr;
        temps_from_state(s, P, te, ti, tr);
        const double oei = P.omega_ei, oer = P.omega_er;
        const double te3 = te * te * te, tr3 = tr * tr * tr;
        const double bte = -oei * ob[0] - oer * 4.0 * te3 * ob[0] + oei * ob[1] + oer * 4.0 * te3 * ob[2];
        const double bti = oei * ob[0] - oei * ob[1];
        const double btr = oer * 4.0 * tr3 * ob[0] - oer * 4.0 * tr3 * ob[2];
        double sb[6] = {0, 0, 0, 0, 0, 0};
        temps_vjp(s, P, bte, bti, btr, sb);
        atomic_add6(W, plane, n, sb);
        const double x4 = pow4d(te) - pow4d(tr);
        atomicAdd(&pbar[8 * kk + 6], -(te - ti) * ob[0] + (te - ti) * ob[1]);
        atomicAdd(&pbar[8 * kk + 7], -x4 * ob[0] + x4 * ob[2]);
    }
}

// ---------------------------------------------------------------- ghosts
constexpr int AG_WARPS = 3;
__constant__ int kAStOff[6] = {0, 1, 5, 14, 30, 55};
__constant__ int kASOff[6] = {0, 1, 17, 98, 354, 979};
__constant__ int kAWOff[6] = {0, 1, 9, 36, 100, 225};

struct AdjGhostWarp {
    double L[36], R[36], lam[6];             // L[6c + j]; R column c at R[6c + i]
    double D[6][56], ACC[6][56], STD[6][56]; // STD becomes D-bar in place
    double bb[6][5];
    double alpha[6][5], beta[6][5], V[6][5][5];
    double v[5][6], x[5][6], ub[5][6], xb[5][6], vinf[6], vinfb[6];
    double Lb[6][6], Rb[6][6];
    double vb[5][6];
};

__device__ __forceinline__ int aorder(int a) { return a < 1 ? 0 : (a < 5 ? 1 : (a < 14 ? 2 : (a < 30 ? 3 : 4))); }

// one heavy (FarField) ghost per warp; gb from W at the ghost node
__device__ void ghost_vjp_warp(const Inst& I, const GhostRec& Rg, const double* __restrict__ rec,
                               const double* __restrict__ X, const double* __restrict__ W, double* __restrict__ Ub,
                               double* __restrict__ pbar_k, AdjGhostWarp& G, int lane) {
    const DevParams& P = I.P;
    const long long plane = I.plane;
    const double nx = Rg.nx, ny = Rg.ny;
    // L, R, lambda at the nearest node of X (bc1.rs:294-312)
    if (lane < 6) {
        double s[6];
        load6(X, plane, Rg.src, s);
        const double q6[6] = {s[0], s[1] * nx + s[2] * ny, -s[1] * ny + s[2] * nx, s[3], s[4], s[5]};
        const Prim d1 = prim_from_state(q6, P);
        const Roe q = roe_average(q6[0], d1, q6[0], d1, P);
        double Lr[6], Rcol[6], lm;
        l_row<0>(lane, q, P, Lr);
        r_col<0>(lane, q, P, Rcol, lm);
        for (int k = 0; k < 6; ++k) { G.L[6 * lane + k] = Lr[k]; G.R[6 * lane + k] = Rcol[k]; }
        G.lam[lane] = lm;
    }
    __syncwarp();
    const double* L = G.L;    // L[c][j] = L[6c + j]
    const double* Rc = G.R;   // R[i][c] = Rc[6c + i]
    const double* lam = G.lam;
    const int32_t* st = reinterpret_cast<const int32_t*>(rec + GH_ST);
    const double* S = rec + GH_S;   // transposed per order: S_r[a][b] = S[off + b m + a]
    // ---- forward: D, ACC = S d, STD = S^T d, beta, alpha, V, v
    for (int a = lane; a < 55; a += 32) {
        double s[6];
        load6(X, plane, st[a], s);
        const double u6[6] = {s[0], s[1] * nx + s[2] * ny, -s[1] * ny + s[2] * nx, s[3], s[4], s[5]};
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0;
            for (int q = 0; q < 6; ++q) acc += L[6 * c + q] * u6[q];
            G.D[c][a] = acc;
        }
    }
    __syncwarp();
    for (int a = lane; a < 55; a += 32) {
        const int r = aorder(a), m = (r + 1) * (r + 1), off = kAStOff[r], ar = a - off;
        const double* Sr = S + kASOff[r];
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0, acct = 0.0;
            for (int b = 0; b < m; ++b) {
                acc += Sr[b * m + ar] * G.D[c][off + b];  // (S d)_a
                acct += Sr[ar * m + b] * G.D[c][off + b]; // (S^T d)_a
            }
            G.ACC[c][a] = acc;
            G.STD[c][a] = acct;
        }
    }
    __syncwarp();
    if (lane < 30) {
        const int c = lane / 5, r = lane - 5 * (lane / 5);
        const int m = (r + 1) * (r + 1), off = kAStOff[r];
        double beta = 0.0;
        for (int a = 0; a < m; ++a) beta += G.D[c][off + a] * G.ACC[c][off + a];
        G.beta[c][r] = beta;
        G.alpha[c][r] = rec[GH_D + r] / pow_q(P.eps + beta, P.weno_q);
        for (int k = 0; k < 5; ++k) {
            double v = 0.0;
            if (k <= r) {
                const double* w = rec + GH_W + kAWOff[r] + k * m;
                for (int a = 0; a < m; ++a) v += w[a] * G.D[c][off + a];
            }
            G.V[c][r][k] = v;
        }
    }
    __syncwarp();
    if (lane < 30) {
        const int k = lane / 6, c = lane - 6 * (lane / 6);
        double asum = 0.0;
        for (int r = 0; r < 5; ++r) asum += G.alpha[c][r];
        double res = 0.0;
        for (int r = 0; r < 5; ++r) res += (G.alpha[c][r] / asum) * G.V[c][r][k];
        G.v[k][c] = res;
    }
    __syncwarp();
    const DevBC& bc = I.bcs[Rg.bc];
    const double* ui = bc.state;
    const double uinf[6] = {ui[0], ui[1] * nx + ui[2] * ny, -ui[1] * ny + ui[2] * nx, ui[3], ui[4], ui[5]};
    if (lane < 6) {
        double acc = 0.0;
        for (int q = 0; q < 6; ++q) acc += L[6 * lane + q] * uinf[q];
        G.vinf[lane] = acc;
    }
    __syncwarp();
    if (lane < 30) {
        const int k = lane / 6, m2 = lane - 6 * (lane / 6);
        G.x[k][m2] = lam[m2] < 0.0 ? (k == 0 ? G.vinf[m2] : 0.0) : G.v[k][m2];
    }
    // ---- reverse: rotation back and Taylor sum
    const long long gn = Rg.node;
    if (lane == 0) {
        const double o[6] = {W[gn], W[plane + gn], W[2 * plane + gn], W[3 * plane + gn], W[4 * plane + gn],
                             W[5 * plane + gn]};
        // out1 = mn nx - mt ny, out2 = mn ny + mt nx
        const double gb[6] = {o[0], o[1] * nx + o[2] * ny, -o[1] * ny + o[2] * nx, o[3], o[4], o[5]};
        double coef = 1.0;
        for (int k = 0; k < 5; ++k) {
            if (k > 0) coef *= Rg.dist / (double)k;
            for (int c = 0; c < 6; ++c) G.ub[k][c] = coef * gb[c];
        }
    }
    __syncwarp();
    // u_k = R x_k: xb_k = R^T ub_k, Rb += ub_k x_k^T
    if (lane < 30) {
        const int k = lane / 6, m2 = lane - 6 * (lane / 6);
        double acc = 0.0;
        for (int i = 0; i < 6; ++i) acc += Rc[6 * m2 + i] * G.ub[k][i];
        G.xb[k][m2] = acc;
    }
    for (int e = lane; e < 36; e += 32) {
        const int i = e / 6, m2 = e - 6 * (e / 6);
        double acc = 0.0;
        for (int k = 0; k < 5; ++k) acc += G.ub[k][i] * G.x[k][m2];
        G.Rb[m2][i] = acc; // cotangent of R column m2, row i
    }
    __syncwarp();
    if (lane < 30) {
        const int k = lane / 6, m2 = lane - 6 * (lane / 6);
        G.vb[k][m2] = lam[m2] < 0.0 ? 0.0 : G.xb[k][m2];
    }
    if (lane < 6) G.vinfb[lane] = lam[lane] < 0.0 ? G.xb[0][lane] : 0.0;
    __syncwarp();
    // vinf = L uinf: Lb += vinfb uinf^T; uinf cotangent -> FarField state
    for (int e = lane; e < 36; e += 32) {
        const int c = e / 6, q = e - 6 * (e / 6);
        G.Lb[c][q] = G.vinfb[c] * uinf[q];
    }
    if (lane < 6) {
        double acc = 0.0;
        for (int c = 0; c < 6; ++c) acc += L[6 * c + lane] * G.vinfb[c];
        G.ub[0][lane] = acc; // reuse: rotated u_inf cotangent
    }
    __syncwarp();
    if (lane == 0) {
        const double* b = G.ub[0];
        const double bu[6] = {b[0], b[1] * nx - b[2] * ny, b[1] * ny + b[2] * nx, b[3], b[4], b[5]};
        for (int c = 0; c < 6; ++c) atomicAdd(&pbar_k[c], bu[c]);
    }
    // v[k][c] = sum_r (alpha_r / sum) V_r^k -> V-bar, alpha-bar -> beta-bar
    if (lane < 6) {
        const int c = lane;
        double asum = 0.0;
        for (int r = 0; r < 5; ++r) asum += G.alpha[c][r];
        double om[5], omb[5], m = 0.0;
        for (int r = 0; r < 5; ++r) {
            om[r] = G.alpha[c][r] / asum;
            omb[r] = 0.0;
            for (int k = 0; k < 5; ++k) omb[r] += G.V[c][r][k] * G.vb[k][c];
            m += om[r] * omb[r];
        }
        for (int r = 0; r < 5; ++r) {
            const double ab = (omb[r] - m) / asum;
            // alpha = d (eps + beta)^-q
            G.beta[c][r] = -P.weno_q * ab * G.alpha[c][r] / (P.eps + G.beta[c][r]); // now beta-bar
            for (int k = 0; k < 5; ++k) G.V[c][r][k] = om[r] * G.vb[k][c];          // now V-bar
        }
    }
    __syncwarp();
    // D-bar over the 55 nodes: beta = d^T S d, V = w . d
    for (int a = lane; a < 55; a += 32) {
        const int r = aorder(a), m = (r + 1) * (r + 1), off = kAStOff[r], ar = a - off;
        for (int c = 0; c < 6; ++c) {
            double acc = G.beta[c][r] * (G.ACC[c][a] + G.STD[c][a]);
            for (int k = 0; k <= r; ++k) acc += G.V[c][r][k] * rec[GH_W + kAWOff[r] + k * m + ar];
            G.STD[c][a] = acc; // D-bar
        }
    }
    __syncwarp();
    // D = L rot(u_a): Lb += DB rot(u_a)^T, rot(u_a)-bar = L^T DB
    for (int e = lane; e < 36; e += 32) {
        const int c = e / 6, q = e - 6 * (e / 6);
        double acc = 0.0;
        for (int a = 0; a < 55; ++a) {
            const long long na = st[a];
            const double s1 = X[plane + na], s2 = X[2 * plane + na];
            const double uq = q == 0 ? X[na]
                              : q == 1 ? s1 * nx + s2 * ny
                              : q == 2 ? -s1 * ny + s2 * nx
                                       : X[q * plane + na];
            acc += G.STD[c][a] * uq;
        }
        G.Lb[c][q] += acc;
    }
    for (int a = lane; a < 55; a += 32) {
        double ur[6];
        for (int q = 0; q < 6; ++q) {
            double acc = 0.0;
            for (int c = 0; c < 6; ++c) acc += L[6 * c + q] * G.STD[c][a];
            ur[q] = acc;
        }
        const double sb[6] = {ur[0], ur[1] * nx - ur[2] * ny, ur[1] * ny + ur[2] * nx, ur[3], ur[4], ur[5]};
        atomic_add6(Ub, plane, st[a], sb);
    }
    __syncwarp();
    // L, R of the nearest node: Roe base of two equal rotated states
    if (lane < 6) {
        double s[6];
        load6(X, plane, Rg.src, s);
        const double q6[6] = {s[0], s[1] * nx + s[2] * ny, -s[1] * ny + s[2] * nx, s[3], s[4], s[5]};
        const Prim d1 = prim_from_state(q6, P);
        const Roe q = roe_average(q6[0], d1, q6[0], d1, P);
        const double base[5] = {q.u, q.v, q.ee, q.ei, q.er};
        double bb[5] = {0, 0, 0, 0, 0};
        lr_base_vjp<0>(lane, base, P, G.Lb[lane], G.Rb[lane], 0.0, bb);
        for (int m = 0; m < 5; ++m) G.bb[lane][m] = bb[m];
    }
    __syncwarp();
    if (lane == 0) {
        double s[6];
        load6(X, plane, Rg.src, s);
        const double q6[6] = {s[0], s[1] * nx + s[2] * ny, -s[1] * ny + s[2] * nx, s[3], s[4], s[5]};
        double bb[5];
        for (int m = 0; m < 5; ++m) {
            double acc = 0.0;
            for (int c = 0; c < 6; ++c) acc += G.bb[c][m];
            bb[m] = acc;
        }
        {
            double ga[6] = {0, 0, 0, 0, 0, 0}, gb2[6] = {0, 0, 0, 0, 0, 0};
            roe_vjp(q6, q6, P, bb, ga, gb2);
            double gr[6];
            for (int c = 0; c < 6; ++c) gr[c] = ga[c] + gb2[c];
            const double sb[6] = {gr[0], gr[1] * nx - gr[2] * ny, gr[1] * ny + gr[2] * nx, gr[3], gr[4], gr[5]};
            atomic_add6(Ub, plane, Rg.src, sb);
        }
    }
}

__global__ void __launch_bounds__(AG_WARPS * 32) k_adj_ghosts(const Inst* __restrict__ insts,
                                                             const GhostRec* __restrict__ heavy, int nh,
                                                             const GhostRec* __restrict__ cheap, int nc,
                                                             const double* __restrict__ hrec,
                                                             const double* __restrict__ Xb,
                                                             const double* __restrict__ Wb,
                                                             double* __restrict__ Ubb, double* __restrict__ pbar,
                                                             int nbh) {
    __shared__ AdjGhostWarp G[AG_WARPS];
    const int lane = threadIdx.x & 31;
    if ((int)blockIdx.x < nbh) {
        const int g = blockIdx.x * AG_WARPS + (threadIdx.x >> 5);
        if (g >= nh) return;
        const GhostRec Rg = heavy[g];
        const Inst& I = insts[Rg.inst];
        if (has_error(I) || Rg.kind != BC_FAR_FIELD) return;
        ghost_vjp_warp(I, Rg, hrec + (size_t)Rg.heavy * GH_REC, Xb + I.aoff, Wb + I.aoff, Ubb + I.aoff,
                       pbar + 8 * Rg.inst, G[threadIdx.x >> 5], lane);
    } else {
        const int g = (blockIdx.x - nbh) * (AG_WARPS * 32) + threadIdx.x;
        if (g >= nc) return;
        const GhostRec Rg = cheap[g];
        const Inst& I = insts[Rg.inst];
        if (has_error(I)) return;
        const long long plane = I.plane;
        const double* W = Wb + I.aoff;
        double gb[6];
        for (int c = 0; c < 6; ++c) gb[c] = W[c * plane + Rg.node];
        double sb[6];
        if (Rg.kind == BC_REFLECTIVE_WALL) { // m - 2 (m.n) n is symmetric in m
            const double mn = Rg.nx * gb[1] + Rg.ny * gb[2];
            sb[0] = gb[0]; sb[1] = gb[1] - 2.0 * mn * Rg.nx; sb[2] = gb[2] - 2.0 * mn * Rg.ny;
            sb[3] = gb[3]; sb[4] = gb[4]; sb[5] = gb[5];
        } else if (Rg.kind == BC_ZEROTH_ORDER || Rg.kind == BC_PERIODIC) {
            for (int c = 0; c < 6; ++c) sb[c] = gb[c];
        } else {
            return; // Constant, TimeDependent: no state dependence
        }
        atomic_add6(Ubb + I.aoff, plane, Rg.src, sb);
    }
}

// Ub += W on fluid nodes
__global__ void k_adj_fluid(const Inst* __restrict__ insts, int k0, const double* __restrict__ Wb,
                            double* __restrict__ Ubb) {
    const Inst& I = insts[k0 + blockIdx.y];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)I.nx * I.ny) return;
    const long long n = node_of(I, (int)(t / I.ny), (int)(t % I.ny));
    if (!I.mask[n]) return;
    const double* W = Wb + I.aoff;
    double* Ub = Ubb + I.aoff;
    for (int c = 0; c < 6; ++c) Ub[c * I.plane + n] += W[c * I.plane + n];
}

// ---------------------------------------------------------------- launchers
void launch_adj_l(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, long long max_faces,
                  const GhostRec* heavy, int nh, const GhostRec* cheap, int nc, const double* hrec, const double* X,
                  const double* rbar, double* W, double* Ub, double* pbar) {
    if (n <= 0) return;
    const unsigned fb = (unsigned)((max_faces + 127) / 128), cb = (unsigned)((max_cells + 127) / 128);
    k_adj_faces<<<dim3(fb, n), 128, 0, s>>>(insts, k0, X, rbar, W, 0);
    k_adj_faces<<<dim3(fb, n), 128, 0, s>>>(insts, k0, X, rbar, W, 1);
    k_adj_cells<<<dim3(cb, n), 128, 0, s>>>(insts, k0, X, rbar, W, pbar);
    const int nbh = (nh + AG_WARPS - 1) / AG_WARPS, nbc = (nc + AG_WARPS * 32 - 1) / (AG_WARPS * 32);
    if (nbh + nbc > 0)
        k_adj_ghosts<<<nbh + nbc, AG_WARPS * 32, 0, s>>>(insts, heavy, nh, cheap, nc, hrec, X, W, Ub, pbar, nbh);
    k_adj_fluid<<<dim3(cb, n), 128, 0, s>>>(insts, k0, W, Ub);
}

int adj_l_launches(int nh, int nc) { return 4 + (nh + nc > 0 ? 1 : 0); }

// ---------------------------------------------------------------- RK3 step plumbing
// copy the 6 planes of stage buffer `which` (0 U, 1 A, 2 B) of instances
// [k0, k0 + n) to (dir 0) or from (dir 1) a plane set
__global__ void k_adj_copy(const Inst* __restrict__ insts, int k0, int which, double* __restrict__ set, int dir) {
    const Inst& I = insts[k0 + blockIdx.y];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6 * I.plane) return;
    double* buf = const_cast<double*>(stage_src(I, which));
    if (dir == 0) set[I.aoff + t] = buf[t];
    else buf[t] = set[I.aoff + t];
}

// AoS (6 per cell, i*ny+j, instance at 6*cell_off) <-> plane set, fluid cells
// (dir 0: AoS -> set, non-fluid nodes zeroed; dir 1: set -> AoS)
__global__ void k_adj_aos(const Inst* __restrict__ insts, int k0, double* __restrict__ aos, double* __restrict__ set,
                          int dir) {
    const Inst& I = insts[k0 + blockIdx.y];
    const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= (long long)I.nx * I.ny) return;
    const long long n = node_of(I, (int)(l / I.ny), (int)(l % I.ny));
    const bool f = I.mask[n] != 0;
    double* a = aos + 6 * (I.cell_off + l);
    double* p = set + I.aoff;
    for (int c = 0; c < 6; ++c) {
        if (dir == 0) p[c * I.plane + n] = f ? a[c] : 0.0;
        else a[c] = f ? p[c * I.plane + n] : 0.0;
    }
}

// Reverse of one stage update (main.rs:308-349), fluid nodes; Y is the
// cotangent of the stage output:
//   stage 2 (u3 = u0/3 + 2 u2/3 + 2dt/3 r2): U0 = Y/3, Uin = 2Y/3, rbar = 2dt/3 Y
//   stage 1 (u2 = 3u0/4 + u1/4 + dt/4 r1):   U0 += 3Y/4, Uin = Y/4, rbar = dt/4 Y
//   stage 0 (u1 = u0 + dt r0):               U0 += Y, rbar = dt Y
// and dtbar += (coef / dt) <Y, r> per instance. sc: the step's scalars.
__global__ void __launch_bounds__(256) k_adj_stage(const Inst* __restrict__ insts, int k0, int stage,
                                                   const double* __restrict__ Y, double* __restrict__ U0,
                                                   double* __restrict__ Uin, double* __restrict__ rbar,
                                                   const double* __restrict__ R, const DevScalars* __restrict__ sc,
                                                   double* __restrict__ dtbar) {
    __shared__ double red[8];
    const int k = k0 + blockIdx.y;
    const Inst& I = insts[k];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double dot = 0.0;
    if (t < (long long)I.nx * I.ny) {
        const long long n = node_of(I, (int)(t / I.ny), (int)(t % I.ny));
        if (I.mask[n]) {
            const double coef = sc[k].coef[stage];
            const double w0 = stage == 2 ? 1.0 / 3.0 : (stage == 1 ? 0.75 : 1.0);
            const double win = stage == 2 ? 2.0 / 3.0 : 0.25;
            const long long o = I.aoff;
            for (int c = 0; c < 6; ++c) {
                const long long m = o + c * I.plane + n;
                const double y = Y[m];
                if (stage == 2) U0[m] = w0 * y;
                else U0[m] += w0 * y;
                if (stage > 0) Uin[m] = win * y;
                rbar[m] = coef * y;
                dot += y * R[m];
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dot;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < 8; ++w) b += red[w];
        const double dcoef = stage == 2 ? 2.0 / 3.0 : (stage == 1 ? 0.25 : 1.0); // d coef / d dt
        if (b != 0.0) atomicAdd(&dtbar[k], dcoef * b);
    }
}

// dt = cfl * min_cells local_dt(u0) (main.rs:375-408, dt.rs:5-34): the
// derivative goes to the first cell, in i*ny+j order, whose local dt equals
// the minimum; one block per instance. Steps whose dt was clipped to t_final
// have none.
__global__ void __launch_bounds__(256) k_adj_dt(const Inst* __restrict__ insts, int k0, const double* __restrict__ X,
                                                const DevScalars* __restrict__ sc, const double* __restrict__ dtbar,
                                                double* __restrict__ U0, double* __restrict__ pbar) {
    __shared__ long long best;
    const int k = k0 + blockIdx.x;
    const Inst& I = insts[k];
    const DevScalars& S = sc[k];
    const double cfl = S.cfl_factor;
    if (!(S.dt == cfl * S.dt_cfl) || dtbar[k] == 0.0) return;
    if (threadIdx.x == 0) best = (long long)I.nx * I.ny;
    __syncthreads();
    const double* x = X + I.aoff;
    for (long long l = threadIdx.x; l < (long long)I.nx * I.ny; l += blockDim.x) {
        const long long n = node_of(I, (int)(l / I.ny), (int)(l % I.ny));
        if (!I.mask[n]) continue;
        double s[6];
        load6(x, I.plane, n, s);
        if (local_dt(s, I.dx, I.dy, I.P) == S.dt_cfl) atomicMin(&best, l);
    }
    __syncthreads();
    if (threadIdx.x != 0 || best >= (long long)I.nx * I.ny) return;
    const long long n = node_of(I, (int)(best / I.ny), (int)(best % I.ny));
    D8 s8[6];
    for (int c = 0; c < 6; ++c) s8[c] = D8::var(x[c * I.plane + n], c);
    const D8 d = local_dt_t<D8>(s8, I.dx, I.dy, I.P, D8::var(I.P.omega_ei, 6), D8::var(I.P.omega_er, 7));
    const double g = cfl * dtbar[k];
    for (int c = 0; c < 6; ++c) U0[I.aoff + c * I.plane + n] += g * d.d[c];
    pbar[8 * k + 6] += g * d.d[6];
    pbar[8 * k + 7] += g * d.d[7];
}

void launch_adj_copy(cudaStream_t s, const Inst* insts, int k0, int n, long long max_plane, int which, double* set,
                     int dir) {
    if (n <= 0) return;
    k_adj_copy<<<dim3((unsigned)((6 * max_plane + 255) / 256), n), 256, 0, s>>>(insts, k0, which, set, dir);
}
void launch_adj_aos(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, double* aos, double* set,
                    int dir) {
    if (n <= 0) return;
    k_adj_aos<<<dim3((unsigned)((max_cells + 255) / 256), n), 256, 0, s>>>(insts, k0, aos, set, dir);
}
void launch_adj_stage(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, int stage,
                      const double* Y, double* U0, double* Uin, double* rbar, const double* R, const DevScalars* sc,
                      double* dtbar) {
    if (n <= 0) return;
    k_adj_stage<<<dim3((unsigned)((max_cells + 255) / 256), n), 256, 0, s>>>(insts, k0, stage, Y, U0, Uin, rbar, R,
                                                                             sc, dtbar);
}
void launch_adj_dt(cudaStream_t s, const Inst* insts, int k0, int n, const double* X, const DevScalars* sc,
                   const double* dtbar, double* U0, double* pbar) {
    if (n <= 0) return;
    k_adj_dt<<<n, 256, 0, s>>>(insts, k0, X, sc, dtbar, U0, pbar);
}

} // namespace rh3t
