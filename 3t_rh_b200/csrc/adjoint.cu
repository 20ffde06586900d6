// Adjoint (vector-Jacobian products) of the semi-discrete operator l() and of
// the SSP-RK3 step (main.rs:135-373), hand-written per kernel of the forward
// path. No reference counterpart: the reference has no derivative code.
//
// vjp of l at a stage state X (ghost nodes of X set by the forward ghost
// update) for a cotangent rbar on the fluid cells, accumulated into Ubar:
//   k_adj_flux   x and y face tiles: the face flux cotangent from rbar, then
//                the reverse of weno.rs:685-802 (R g, WENO5 weights,
//                Lax-Friedrichs split, L projections, the Roe average of
//                points 2 and 3, the six physical fluxes) and of
//                diffusion.rs:27-50 -> node cotangents W (fluid and ghost
//                nodes, atomic adds);
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
// scalars (u, v, e_e, e_i, e_r). Since L = R^-1, the cotangent of L is
// turned into one of R (dL = -L dR L) and only R, which is polynomial in
// u, v and sqrt(cs2), is differentiated; the CFL time step of a cell is
// differentiated with dual numbers (dual.cuh). The rest is by hand.
// Kinks follow the values: d|x|/dx = +1 at 0, max/min pass the derivative to
// the first argument on ties, a FarField row switches on lambda < 0.
#include <algorithm>

#include "common.cuh"
#include "dual.cuh"
#include "kernels.cuh"
#include "physics.cuh"
#include "ghost_rows.cuh"

namespace rh3t {

using D8 = DualN<8>;
// the adjoint needs derivatives, not the forward's roundings: constant
// divisions become multiplications by reciprocals
constexpr double K3 = 1.0 / 3.0, K6 = 1.0 / 6.0;

// ---------------------------------------------------------------- pointwise vjps
// state.rs:245-276 primitives: cotangents of (u, v, e_e, e_i, e_r, p_e, p_i,
// p_r) -> state cotangent (added to sb)
__device__ __forceinline__ void prim_vjp(const double s[6], const DevParams& P, double bu, double bv, double bee,
                                         double bei, double ber, double bpe, double bpi, double bpr, double sb[6]) {
    const double rho = s[0], ir = 1.0 / rho, u = s[1] * ir, v = s[2] * ir;
    const double w2 = u * u + v * v;
    const double ge = P.gamma_e - 1.0, gi = P.gamma_i - 1.0, gr = P.gamma_r - 1.0;
    const double gp = ge * bpe + gi * bpi + gr * bpr;
    const double bw2 = -(bee + bei + ber) * K6 - gp * rho * K6;
    double brho = -(s[3] * bee + s[4] * bei + s[5] * ber) * ir * ir - gp * w2 * K6;
    const double bu2 = bu + 2.0 * u * bw2, bv2 = bv + 2.0 * v * bw2;
    brho -= (bu2 * u + bv2 * v) * ir;
    sb[0] += brho;
    sb[1] += bu2 * ir;
    sb[2] += bv2 * ir;
    sb[3] += bee * ir + ge * bpe;
    sb[4] += bei * ir + gi * bpi;
    sb[5] += ber * ir + gr * bpr;
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

// weno.rs:847-886 WENO5: cotangent gb of the result -> ub[5] (added); returns
// the value itself (formed with the same intermediates)
__device__ __forceinline__ double weno5_vjp(const double x[5], double eps, double gb, double ub[5]) {
    const double t0 = x[0] - 2.0 * x[1] + x[2], r0 = x[0] - 4.0 * x[1] + 3.0 * x[2];
    const double t1 = x[1] - 2.0 * x[2] + x[3], r1 = x[1] - x[3];
    const double t2 = x[2] - 2.0 * x[3] + x[4], r2 = 3.0 * x[2] - 4.0 * x[3] + x[4];
    const double c1312 = 13.0 / 12.0;
    const double e0 = 1.0 / (eps + (c1312 * t0 * t0 + 0.25 * r0 * r0));
    const double e1 = 1.0 / (eps + (c1312 * t1 * t1 + 0.25 * r1 * r1));
    const double e2 = 1.0 / (eps + (c1312 * t2 * t2 + 0.25 * r2 * r2));
    const double a0 = 0.1 * e0 * e0, a1 = 0.6 * e1 * e1, a2 = 0.3 * e2 * e2;
    const double iS = 1.0 / (a0 + a1 + a2);
    const double w0 = a0 * iS, w1 = a1 * iS, w2 = a2 * iS;
    const double p0 = x[0] * K3 - 7.0 / 6.0 * x[1] + 11.0 / 6.0 * x[2];
    const double p1 = -x[1] * K6 + 5.0 / 6.0 * x[2] + x[3] * K3;
    const double p2 = x[2] * K3 + 5.0 / 6.0 * x[3] - x[4] * K6;
    const double pb0 = w0 * gb, pb1 = w1 * gb, pb2 = w2 * gb;
    const double wb0 = p0 * gb, wb1 = p1 * gb, wb2 = p2 * gb;
    const double m = w0 * wb0 + w1 * wb1 + w2 * wb2;
    // alpha_k = d_k / (eps + b_k)^2, w_k = alpha_k / sum
    const double bb0 = -2.0 * (wb0 - m) * iS * a0 * e0, bb1 = -2.0 * (wb1 - m) * iS * a1 * e1,
                 bb2 = -2.0 * (wb2 - m) * iS * a2 * e2;
    ub[0] += pb0 * K3;
    ub[1] += -7.0 / 6.0 * pb0 - pb1 * K6;
    ub[2] += 11.0 / 6.0 * pb0 + 5.0 / 6.0 * pb1 + pb2 * K3;
    ub[3] += pb1 * K3 + 5.0 / 6.0 * pb2;
    ub[4] += -pb2 * K6;
    const double c0 = 13.0 / 6.0 * t0 * bb0, d0 = 0.5 * r0 * bb0;
    ub[0] += c0 + d0; ub[1] += -2.0 * c0 - 4.0 * d0; ub[2] += c0 + 3.0 * d0;
    const double c1 = 13.0 / 6.0 * t1 * bb1, d1 = 0.5 * r1 * bb1;
    ub[1] += c1 + d1; ub[2] += -2.0 * c1; ub[3] += c1 - d1;
    const double c2 = 13.0 / 6.0 * t2 * bb2, d2 = 0.5 * r2 * bb2;
    ub[2] += c2 + 3.0 * d2; ub[3] += -2.0 * c2 - 4.0 * d2; ub[4] += c2 + d2;
    return w0 * p0 + w1 * p1 + w2 * p2;
}

// column c of R and lambda_c (weno.rs:518-545) with reciprocals
template <int DIR>
__device__ __forceinline__ void r_col_adj(int c, const Roe& q, const DevParams& P, double R[6], double& lam) {
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    const double u = q.u, v = q.v, w2 = q.w2, cs = q.cs, vel = DIR == 0 ? u : v;
    const double w6 = w2 * K6;
    if (c == 0 || c == 5) {
        const double sg = c == 0 ? -1.0 : 1.0, vc = sg * vel * cs * K3;
        R[0] = 1.0;
        R[1] = DIR == 0 ? u + sg * cs : u;
        R[2] = DIR == 0 ? v : v + sg * cs;
        R[3] = GE * q.ee + w6 + vc; R[4] = GI * q.ei + w6 + vc; R[5] = GR * q.er + w6 + vc;
        lam = vel + sg * cs;
        return;
    }
    lam = vel;
    const int tr = DIR == 0 ? 4 : 1; // transverse column
    if (c == tr) {
        const double t3 = (DIR == 0 ? v : u) * K3;
        R[0] = 0.0;
        R[1] = DIR == 0 ? 0.0 : 1.0;
        R[2] = DIR == 0 ? 1.0 : 0.0;
        R[3] = t3; R[4] = t3; R[5] = t3;
        return;
    }
    const int k = DIR == 0 ? c - 1 : c - 2; // species 0 e, 1 i, 2 r
    const double gk = k == 0 ? ge : (k == 1 ? gi : gr);
    const double sp = gt * w2 * K6 / gk;
    R[0] = 1.0; R[1] = u; R[2] = v;
    if (k == 0) { R[3] = sp; R[4] = gr; R[5] = -gi; }
    else if (k == 1) { R[3] = -gr; R[4] = sp; R[5] = ge; }
    else { R[3] = gi; R[4] = -ge; R[5] = sp; }
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

// One side of roe_vjp: the cotangent of point 3 (side 0, sa) or point 2
// (side 1, sb_) only, added to g
__device__ __forceinline__ void roe_vjp_side(const double sa[6], const double sb_[6], const DevParams& P,
                                             const double bb[5], int side, double g[6]) {
    const Prim da = prim_from_state(sa, P), db = prim_from_state(sb_, P);
    const double ra = sqrt(sa[0]), rb = sqrt(sb_[0]), irs = 1.0 / (ra + rb);
    const double xa[5] = {da.u, da.v, da.e_e, da.e_i, da.e_r}, xb[5] = {db.u, db.v, db.e_e, db.e_i, db.e_r};
    const double rs_self = side == 0 ? ra : rb;
    double br = 0.0, pp[5];
    for (int k = 0; k < 5; ++k) {
        const double base = (xa[k] * ra + xb[k] * rb) * irs;
        pp[k] = bb[k] * rs_self * irs;
        br += bb[k] * ((side == 0 ? xa[k] : xb[k]) - base) * irs;
    }
    g[0] += br / (2.0 * rs_self);
    prim_vjp(side == 0 ? sa : sb_, P, pp[0], pp[1], pp[2], pp[3], pp[4], 0.0, 0.0, 0.0, g);
}

// Cotangents of R (Rb[c][i] = dJ/dR[i][c], weno.rs:518-545) and of the
// eigenvalues -> cotangents of the Roe base (u, v, e_e, e_i, e_r), added.
// R is written in u, v, w2 = u^2 + v^2, cs = sqrt(cs2) and the e_k.
template <int DIR>
__device__ __forceinline__ void r_base_vjp(const double base[5], const DevParams& P, const double Rb[6][6],
                                           const double lamb[6], double bb[5]) {
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    const double u = base[0], v = base[1];
    const double cs = sqrt(GE * ge * base[2] + GI * gi * base[3] + GR * gr * base[4]);
    const double vel = DIR == 0 ? u : v;
    double bvel = 0.0, bcs = 0.0, bw2 = 0.0, bu = 0.0, bv = 0.0, be[3] = {0.0, 0.0, 0.0};
    const double Gk[3] = {GE, GI, GR}, gk[3] = {ge, gi, gr};
    // acoustic columns 0 (-) and 5 (+): (1, [vel -+ cs], ..., G_k e_k + w2/6 -+ vel cs/3)
    for (int side = 0; side < 2; ++side) {
        const int c = side == 0 ? 0 : 5;
        const double sg = side == 0 ? -1.0 : 1.0;
        const double* r = Rb[c];
        if (DIR == 0) { bu += r[1]; bcs += sg * r[1]; bv += r[2]; }
        else { bu += r[1]; bv += r[2]; bcs += sg * r[2]; }
        for (int k = 0; k < 3; ++k) {
            be[k] += Gk[k] * r[3 + k];
            bw2 += r[3 + k] * K6;
            bvel += sg * cs * K3 * r[3 + k];
            bcs += sg * vel * K3 * r[3 + k];
        }
    }
    // transverse column (x: 4, y: 1): unit momentum, (t/3, t/3, t/3) with t = v (x) or u (y)
    {
        const int c = DIR == 0 ? 4 : 1;
        const double t3 = (Rb[c][3] + Rb[c][4] + Rb[c][5]) * K3;
        if (DIR == 0) bv += t3;
        else bu += t3;
    }
    // species columns (x: 1, 2, 3; y: 2, 3, 4): (1, u, v, ..., gt w2 / (6 g_k) at row 3 + k)
    for (int k = 0; k < 3; ++k) {
        const int c = DIR == 0 ? 1 + k : 2 + k;
        bu += Rb[c][1];
        bv += Rb[c][2];
        bw2 += gt * K6 / gk[k] * Rb[c][3 + k];
    }
    // eigenvalues: vel -+ cs, vel
    for (int c = 0; c < 6; ++c) bvel += lamb[c];
    bcs += lamb[5] - lamb[0];
    if (DIR == 0) bu += bvel;
    else bv += bvel;
    bu += 2.0 * u * bw2;
    bv += 2.0 * v * bw2;
    const double hc = 0.5 / cs;
    bb[0] += bu;
    bb[1] += bv;
    bb[2] += be[0] + GE * ge * hc * bcs;
    bb[3] += be[1] + GI * gi * hc * bcs;
    bb[4] += be[2] + GR * gr * hc * bcs;
}

// r_base_vjp for the two columns c0, c0 + 1 of R-bar (the other columns
// zero): the part of the Roe base cotangent they carry, added to bb
template <int DIR>
__device__ __forceinline__ void r_base_vjp2(const double base[5], const DevParams& P, int c0, const double Rb2[2][6],
                                            const double lamb2[2], double bb[5]) {
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    const double u = base[0], v = base[1];
    const double cs = sqrt(GE * ge * base[2] + GI * gi * base[3] + GR * gr * base[4]);
    const double vel = DIR == 0 ? u : v;
    double bvel = 0.0, bcs = 0.0, bw2 = 0.0, bu = 0.0, bv = 0.0, be[3] = {0.0, 0.0, 0.0};
    const double Gk[3] = {GE, GI, GR}, gk[3] = {ge, gi, gr};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int c = c0 + h;
        const double* r = Rb2[h];
        if (c == 0 || c == 5) { // acoustic: (1, [vel -+ cs], ..., G_k e_k + w2/6 -+ vel cs/3)
            const double sg = c == 0 ? -1.0 : 1.0;
            if (DIR == 0) { bu += r[1]; bcs += sg * r[1]; bv += r[2]; }
            else { bu += r[1]; bv += r[2]; bcs += sg * r[2]; }
            for (int k = 0; k < 3; ++k) {
                be[k] += Gk[k] * r[3 + k];
                bw2 += r[3 + k] * K6;
                bvel += sg * cs * K3 * r[3 + k];
                bcs += sg * vel * K3 * r[3 + k];
            }
            bcs += sg * lamb2[h];
        } else if (c == (DIR == 0 ? 4 : 1)) { // transverse: unit momentum, (t/3, t/3, t/3)
            const double t3 = (r[3] + r[4] + r[5]) * K3;
            if (DIR == 0) bv += t3;
            else bu += t3;
        } else { // species k: (1, u, v, ..., gt w2 / (6 g_k) at row 3 + k)
            // (selects, not an index: a runtime index would put Rb2 in local memory)
            const int k = DIR == 0 ? c - 1 : c - 2;
            const double rk = k == 0 ? r[3] : (k == 1 ? r[4] : r[5]);
            const double gkk = k == 0 ? gk[0] : (k == 1 ? gk[1] : gk[2]);
            bu += r[1];
            bv += r[2];
            bw2 += gt * K6 / gkk * rk;
        }
        bvel += lamb2[h];
    }
    if (DIR == 0) bu += bvel;
    else bv += bvel;
    bu += 2.0 * u * bw2;
    bv += 2.0 * v * bw2;
    const double hc = 0.5 / cs;
    bb[0] += bu;
    bb[1] += bv;
    bb[2] += be[0] + GE * ge * hc * bcs;
    bb[3] += be[1] + GI * gi * hc * bcs;
    bb[4] += be[2] + GR * gr * hc * bcs;
}

// L = R^-1, so dL = -L dR L and the cotangent Lb of L is one of R:
// Rb -= L^T Lb L^T. Rb[c][i] = dJ/dR[i][c], Lb[c][j] = dJ/dL[c][j],
// L[c][j] = L[6c + j].
__device__ __forceinline__ void fold_l_into_r(const double* L, const double Lb[6][6], double Rb[6][6]) {
    double Z[6][6]; // Z[j][c] = sum_k Lb[j][k] L[c][k]
    for (int j = 0; j < 6; ++j)
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0;
            for (int k = 0; k < 6; ++k) acc += Lb[j][k] * L[6 * c + k];
            Z[j][c] = acc;
        }
    for (int c = 0; c < 6; ++c)
        for (int i = 0; i < 6; ++i) {
            double acc = 0.0;
            for (int j = 0; j < 6; ++j) acc += L[6 * j + i] * Z[j][c];
            Rb[c][i] -= acc;
        }
}

__device__ __forceinline__ void atomic_add6(double* W, long long plane, long long n, const double v[6]) {
#pragma unroll
    for (int c = 0; c < 6; ++c)
        if (v[c] != 0.0) atomicAdd(&W[c * plane + n], v[c]);
}

// ---------------------------------------------------------------- face tiles
// The same 64-face tiles as the forward flux kernel (k_flux), block of 6
// warps:
//   1. staging: point states and physical fluxes of the tile, each face's Roe
//      state and flux cotangent Fb (from rbar);
//   2. warp c = characteristic field c, faces lane and lane + 32: the forward
//      reconstruction of field c, then its reverse: w-bar and f-bar of the six
//      points, L-bar of row c, lambda-bar; L row c and g_c kept for step 3;
//   3a. three threads per face: L-bar folded into R-bar (L = R^-1), the Roe
//      base cotangent and the Roe average's vjp -> W at points 2 and 3
//      (atomic), the diffusion flux's vjp, and per point k of the face
//      sum_c w-bar_ck L_c and sum_c f-bar_ck L_c;
//   3b. one thread per point: the sums of 3a over the faces that use it, the
//      physical flux's vjp -> W (atomic).
// per-face rows are padded to FLUX_FACES + 1 doubles: the three threads of a
// face in step 3a read different rows at the same face and land in different
// banks
constexpr int AFP = FLUX_FACES + 1;
struct AdjFluxShared {
    double2 U[3][FLUX_NPT];
    double2 F[3][FLUX_NPT];
    double Q[15][AFP];     // Roe state u v w2 ee ei er cs2 cs he hi hr b den, 1/cs2, 1/b
    double FB[6][AFP];     // face flux cotangent
    double G[6][AFP];      // g_c
    double LAMB[6][AFP];   // lambda-bar_c
    double LS[6][6][AFP];  // L row c
    double LB[6][6][AFP];  // L-bar row c
    double WB[6][6][AFP];  // w-bar [c][k]
    double FK[6][6][AFP];  // f-bar [c][k]
    int act[FLUX_FACES];
};
static_assert(14 * FLUX_NPT + FLUX_NPT / 8 + 1 <= 36 * AFP, "step-1 staging fits in LS");

template <int DIR>
__device__ __forceinline__ void adj_face_index(const Tile& t, int f, int& i, int& j, int& p0, int& ps) {
    const int r = f >> t.lg, cc = f & ((1 << t.lg) - 1);
    i = t.i + r;
    j = t.j0 + cc;
    if (DIR == 0) { p0 = f; ps = 1 << t.lg; }
    else { p0 = r * ((1 << t.lg) + 5) + cc; ps = 1; }
}

__device__ __forceinline__ Roe adj_load_q(const AdjFluxShared& S, int f) {
    Roe q;
    q.u = S.Q[0][f]; q.v = S.Q[1][f]; q.w2 = S.Q[2][f]; q.ee = S.Q[3][f]; q.ei = S.Q[4][f]; q.er = S.Q[5][f];
    q.cs2 = S.Q[6][f]; q.cs = S.Q[7][f]; q.he = S.Q[8][f]; q.hi = S.Q[9][f]; q.hr = S.Q[10][f]; q.b = S.Q[11][f];
    q.den = S.Q[12][f];
    return q;
}

__device__ __forceinline__ void adj_point(const AdjFluxShared& S, int p, double u[6], double F[6]) {
    const double2 a = S.U[0][p], b = S.U[1][p], c = S.U[2][p];
    const double2 x = S.F[0][p], y = S.F[1][p], z = S.F[2][p];
    u[0] = a.x; u[1] = a.y; u[2] = b.x; u[3] = b.y; u[4] = c.x; u[5] = c.y;
    F[0] = x.x; F[1] = x.y; F[2] = y.x; F[3] = y.y; F[4] = z.x; F[5] = z.y;
}

template <int DIR>
__device__ void adj_flux_tile(const Inst& I, const Tile& t, const double* __restrict__ X,
                              const double* __restrict__ rbar, double* __restrict__ W, AdjFluxShared& S) {
    const DevParams& P = I.P;
    const long long plane = I.plane;
    const int nx = I.nx, ny = I.ny;
    const int cols = 1 << t.lg, rows = FLUX_FACES >> t.lg;
    const int np = DIR == 0 ? (rows + 5) * cols : rows * (cols + 5);
    const double sc = DIR == 0 ? 1.0 / I.dx : 1.0 / I.dy;
    // ---- 1a. points of the tile: state, physical flux, primitives, mask and
    // rbar (fluid nodes of the grid, else 0); primitives, rbar and mask live in
    // the L rows' space until step 2
    double* const stage_tmp = &S.LS[0][0][0];
    double(*PR)[FLUX_NPT] = reinterpret_cast<double(*)[FLUX_NPT]>(stage_tmp);
    double(*RB)[FLUX_NPT] = reinterpret_cast<double(*)[FLUX_NPT]>(stage_tmp + 8 * FLUX_NPT);
    unsigned char* MK = reinterpret_cast<unsigned char*>(stage_tmp + 14 * FLUX_NPT);
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        int pi, pj;
        if (DIR == 0) { pi = t.i - 3 + (p >> t.lg); pj = t.j0 + (p & (cols - 1)); }
        else { const int r = p / (cols + 5); pi = t.i + r; pj = t.j0 - 3 + (p - r * (cols + 5)); }
        double s[6] = {1.0, 0.0, 0.0, 1.0, 1.0, 1.0};
        unsigned char mk = 0;
        long long n = 0;
        if (pi >= -RH3T_PAD && pi < nx + RH3T_PAD && pj >= -RH3T_PAD && pj < ny + RH3T_PAD) {
            n = node_of(I, pi, pj);
            load6(X, plane, n, s);
            mk = I.mask[n];
        }
        const Prim d = prim_from_state(s, P);
        double f[6];
        phys_flux<DIR>(s, d, f);
        for (int k = 0; k < 3; ++k) {
            S.U[k][p] = make_double2(s[2 * k], s[2 * k + 1]);
            S.F[k][p] = make_double2(f[2 * k], f[2 * k + 1]);
        }
        PR[0][p] = d.u; PR[1][p] = d.v; PR[2][p] = d.e_e; PR[3][p] = d.e_i; PR[4][p] = d.e_r;
        PR[5][p] = d.pe; PR[6][p] = d.pi; PR[7][p] = d.pr;
        const bool in = mk && pi >= 0 && pi < nx && pj >= 0 && pj < ny;
        for (int c = 0; c < 6; ++c) RB[c][p] = in ? rbar[c * plane + n] : 0.0;
        MK[p] = mk;
    }
    __syncthreads();
    // ---- 1b. faces: Roe state of points 3 and 2, flux cotangent Fb
    for (int f = threadIdx.x; f < FLUX_FACES; f += blockDim.x) {
        int i, j, p0, ps;
        adj_face_index<DIR>(t, f, i, j, p0, ps);
        const int p3 = p0 + 3 * ps, p2 = p0 + 2 * ps;
        const bool valid = (DIR == 0 ? (i <= nx && j < ny) : (i < nx && j <= ny)) && (MK[p3] | MK[p2]) != 0;
        S.act[f] = valid ? 1 : 0;
        if (!valid) continue;
        const Prim d3 = {PR[0][p3], PR[1][p3], PR[2][p3], PR[3][p3], PR[4][p3], PR[5][p3], PR[6][p3], PR[7][p3]};
        const Prim d2 = {PR[0][p2], PR[1][p2], PR[2][p2], PR[3][p2], PR[4][p2], PR[5][p2], PR[6][p2], PR[7][p2]};
        const Roe q = roe_average(S.U[0][p3].x, d3, S.U[0][p2].x, d2, P);
        const double qv[15] = {q.u,  q.v,  q.w2, q.ee, q.ei, q.er,  q.cs2,       q.cs,
                               q.he, q.hi, q.hr, q.b,  q.den, 1.0 / q.cs2, 1.0 / q.b};
        for (int k = 0; k < 15; ++k) S.Q[k][f] = qv[k];
        for (int c = 0; c < 6; ++c) S.FB[c][f] = (RB[c][p3] - RB[c][p2]) * sc;
    }
    __syncthreads();
    // ---- 2. warp c: field c of faces lane and lane + 32
    const int c = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int h = 0; h < FLUX_FACES / 32; ++h) {
        const int f = lane + 32 * h;
        if (!S.act[f]) continue;
        int i, j, p0, ps;
        adj_face_index<DIR>(t, f, i, j, p0, ps);
        const Roe q = adj_load_q(S, f);
        double Lc[6], Rc[6], lam;
        fastm::l_row<DIR>(c, q, S.Q[13][f], S.Q[14][f], P, Lc);
        r_col_adj<DIR>(c, q, P, Rc, lam);
        const double a = fabs(lam);
        double w[6], fp[6], fm[6];
        for (int k = 0; k < 6; ++k) {
            double u[6], F[6];
            adj_point(S, p0 + k * ps, u, F);
            double cf = 0.0, cs = 0.0;
            for (int m = 0; m < 6; ++m) { cf += Lc[m] * F[m]; cs += Lc[m] * u[m]; }
            w[k] = cs;
            fp[k] = 0.5 * (cf + a * cs);
            fm[k] = 0.5 * (cf - a * cs);
        }
        // g_c = weno5(f+) + weno5(f-) and its cotangent gb = (R^T Fb)_c: both
        // reconstructions are reversed with the intermediates of their value
        double gb = 0.0;
        for (int i2 = 0; i2 < 6; ++i2) gb += Rc[i2] * S.FB[i2][f];
        double fpb[6] = {0, 0, 0, 0, 0, 0}, fmb[6] = {0, 0, 0, 0, 0, 0};
        double gval = weno5_vjp(fp, P.eps, gb, fpb);
        {
            const double xm[5] = {fm[5], fm[4], fm[3], fm[2], fm[1]};
            double ubm[5] = {0, 0, 0, 0, 0};
            gval += weno5_vjp(xm, P.eps, gb, ubm);
            fmb[5] += ubm[0]; fmb[4] += ubm[1]; fmb[3] += ubm[2]; fmb[2] += ubm[3]; fmb[1] += ubm[4];
        }
        S.G[c][f] = gval;
        double ab = 0.0, Lb[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 6; ++k) {
            const double fbk = 0.5 * (fpb[k] + fmb[k]);
            const double wbk = 0.5 * a * (fpb[k] - fmb[k]);
            ab += 0.5 * w[k] * (fpb[k] - fmb[k]);
            double u[6], F[6];
            adj_point(S, p0 + k * ps, u, F);
            for (int m = 0; m < 6; ++m) Lb[m] += wbk * u[m] + fbk * F[m];
            S.WB[c][k][f] = wbk;
            S.FK[c][k][f] = fbk;
        }
        for (int m = 0; m < 6; ++m) { S.LS[c][m][f] = Lc[m]; S.LB[c][m][f] = Lb[m]; }
        S.LAMB[c][f] = lam < 0.0 ? -ab : ab;
    }
    __syncthreads();
    // ---- 3a. per face, three threads (two columns of R each): L-bar folded
    // into R-bar (L = R^-1), the Roe base cotangent; then the Roe average's
    // vjp and the diffusion flux's vjp on the first of the three
    {
        const int f = threadIdx.x / 3, part = threadIdx.x - 3 * (threadIdx.x / 3);
        const bool on = f < FLUX_FACES && S.act[f];
        double bb[5] = {0, 0, 0, 0, 0};
        if (on) {
            // own columns c0, c0 + 1 of R-bar: Fb g_c^T, then -= sum_j L[j][i] Z[j][c]
            // with Z[j][c] = sum_k Lb[j][k] L[c][k]
            const int c0 = 2 * part;
            double Rb2[2][6], lamb2[2], Z0[6] = {}, Z1[6] = {};
            lamb2[0] = S.LAMB[c0][f];
            lamb2[1] = S.LAMB[c0 + 1][f];
            const double g0 = S.G[c0][f], g1 = S.G[c0 + 1][f];
#pragma unroll
            for (int m = 0; m < 6; ++m) {
                const double fb = S.FB[m][f];
                Rb2[0][m] = fb * g0;
                Rb2[1][m] = fb * g1;
            }
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const double l0 = S.LS[c0][k][f], l1 = S.LS[c0 + 1][k][f];
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    const double lb = S.LB[j][k][f];
                    Z0[j] += lb * l0;
                    Z1[j] += lb * l1;
                }
            }
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                double a0 = 0.0, a1 = 0.0;
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    const double l = S.LS[j][i][f];
                    a0 += l * Z0[j];
                    a1 += l * Z1[j];
                }
                Rb2[0][i] -= a0;
                Rb2[1][i] -= a1;
            }
            const Roe q = adj_load_q(S, f);
            const double base[5] = {q.u, q.v, q.ee, q.ei, q.er};
            r_base_vjp2<DIR>(base, P, c0, Rb2, lamb2, bb);
        }
        // per face and point k of this part: V_k = sum_c wbar_ck L_c and
        // VF_k = sum_c fbar_ck L_c (the point sums of 3b read these)
        double V[2][6] = {}, VF[2][6] = {};
        if (on) {
            const int k0 = 2 * part;
#pragma unroll
            for (int c2 = 0; c2 < 6; ++c2) {
                const double w0 = S.WB[c2][k0][f], w1 = S.WB[c2][k0 + 1][f];
                const double q0 = S.FK[c2][k0][f], q1 = S.FK[c2][k0 + 1][f];
#pragma unroll
                for (int m = 0; m < 6; ++m) {
                    const double l = S.LS[c2][m][f];
                    V[0][m] += w0 * l;
                    V[1][m] += w1 * l;
                    VF[0][m] += q0 * l;
                    VF[1][m] += q1 * l;
                }
            }
        }
        __syncthreads(); // LB, WB, FK, G and LAMB are read: reuse them
        if (on) {
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                if (part == 0) S.FK[0][m][f] = bb[m];
                if (part == 1) S.G[m][f] = bb[m];
                if (part == 2) S.LAMB[m][f] = bb[m];
            }
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int m = 0; m < 6; ++m) {
                    S.LB[2 * part + h][m][f] = V[h][m];
                    S.WB[2 * part + h][m][f] = VF[h][m];
                }
        }
        __syncthreads();
        if (on && part < 2) { // the Roe average's vjp: point 3 on part 0, point 2 on part 1
#pragma unroll
            for (int m = 0; m < 5; ++m) bb[m] = S.FK[0][m][f] + (S.G[m][f] + S.LAMB[m][f]);
            int i, j, p0, ps;
            adj_face_index<DIR>(t, f, i, j, p0, ps);
            double u3[6], u2[6], F_[6];
            adj_point(S, p0 + 3 * ps, u3, F_);
            adj_point(S, p0 + 2 * ps, u2, F_);
            double g[6] = {0, 0, 0, 0, 0, 0};
            roe_vjp_side(u3, u2, P, bb, part, g);
            atomic_add6(W, plane, part == 0 ? node_of(I, i, j) : (DIR == 0 ? node_of(I, i - 1, j) : node_of(I, i, j - 1)),
                        g);
        }
        if (on && part == 2) {
            int i, j, p0, ps;
            adj_face_index<DIR>(t, f, i, j, p0, ps);
            double F_[6];
            if (I.diffusion) { // diffusion.rs:27-50: rhs += -(b - a) cx per face pair, cx = -1 / ds^2
                const double cx = DIR == 0 ? -1.0 / (I.dx * I.dx) : -1.0 / (I.dy * I.dy);
                const double Db[3] = {S.FB[3][f] / sc * cx, S.FB[4][f] / sc * cx, S.FB[5][f] / sc * cx};
                const double cf[6] = {-2.0, 25.0, -245.0, 245.0, -25.0, 2.0};
                const double kap[3] = {P.kappa_e, P.kappa_i, P.kappa_r};
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    double uk[6];
                    adj_point(S, p0 + k * ps, uk, F_);
                    double te, ti, tr;
                    temps_from_state(uk, P, te, ti, tr);
                    double sb[6] = {0, 0, 0, 0, 0, 0};
                    temps_vjp(uk, P, Db[0] * kap[0] * cf[k] / 180.0, Db[1] * kap[1] * cf[k] / 180.0,
                              Db[2] * kap[2] * cf[k] / 180.0 * 4.0 * tr * tr * tr, sb);
                    const long long nk = DIR == 0 ? node_of(I, i - 3 + k, j) : node_of(I, i, j - 3 + k);
                    atomic_add6(W, plane, nk, sb);
                }
            }
        }
    }
    // ---- 3b. per point: sum over the faces and fields that use it
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        // faces of this point: x tiles: same column, rows pr-5..pr; y tiles: same row, cols pc-5..pc
        int pr, pc, pi, pj;
        if (DIR == 0) { pr = p >> t.lg; pc = p & (cols - 1); pi = t.i - 3 + pr; pj = t.j0 + pc; }
        else { pr = p / (cols + 5); pc = p - pr * (cols + 5); pi = t.i + pr; pj = t.j0 - 3 + pc; }
        double ub[6] = {0, 0, 0, 0, 0, 0}, fb[6] = {0, 0, 0, 0, 0, 0};
        bool any = false;
        for (int k = 0; k < 6; ++k) {
            int f;
            if (DIR == 0) {
                const int r = pr - k;
                if (r < 0 || r >= rows) continue;
                f = r * cols + pc;
            } else {
                const int cc = pc - k;
                if (cc < 0 || cc >= cols) continue;
                f = pr * cols + cc;
            }
            if (!S.act[f]) continue;
            any = true;
#pragma unroll
            for (int m = 0; m < 6; ++m) {
                ub[m] += S.LB[k][m][f]; // V_k of face f
                fb[m] += S.WB[k][m][f]; // VF_k
            }
        }
        if (!any) continue;
        double u[6], F_[6];
        adj_point(S, p, u, F_);
        const Prim d = prim_from_state(u, P);
        flux_vjp<DIR>(u, d, P, fb, ub);
        atomic_add6(W, plane, node_of(I, pi, pj), ub);
    }
}

__global__ void __launch_bounds__(FLUX_THREADS, 2) k_adj_flux(const Inst* __restrict__ insts,
                                                           const Tile* __restrict__ tx, int ntx,
                                                           const Tile* __restrict__ ty, int nty,
                                                           const double* __restrict__ Xb,
                                                           const double* __restrict__ rbarb, double* __restrict__ Wb) {
    extern __shared__ __align__(16) unsigned char adj_flux_smem[];
    AdjFluxShared& S = *reinterpret_cast<AdjFluxShared*>(adj_flux_smem);
    const int b = blockIdx.x;
    if (b < ntx) {
        const Tile t = tx[b];
        const Inst& I = insts[t.inst];
        if (has_error(I)) return;
        adj_flux_tile<0>(I, t, Xb + I.aoff, rbarb + I.aoff, Wb + I.aoff, S);
    } else if (b < ntx + nty) {
        const Tile t = ty[b - ntx];
        const Inst& I = insts[t.inst];
        if (has_error(I)) return;
        adj_flux_tile<1>(I, t, Xb + I.aoff, rbarb + I.aoff, Wb + I.aoff, S);
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

// Fluid cells on the RHS tiles (a TI x TJ block of cells with its 4-node cross
// halo, shape per tile): the node primitives (p_e, p_i, p_r, u, v) of the
// tile and halo are formed once in shared memory; each cell adds the
// cotangents of its two 9-point stencils to a shared tile of primitive
// cotangents; each node then turns them into a state cotangent with one
// primitive vjp and one atomic add per component to W. The exchange source
// goes to W at the cell, its coefficient cotangents to pbar (block sums).
// pbar: per-instance parameter cotangents [u_inf (6), omega_ei, omega_er].
constexpr int ADJ_CELL_SMEM = 2 * 5 * RHS_NPT * (int)sizeof(double);

__global__ void __launch_bounds__(RHS_THREADS) k_adj_cells(const Inst* __restrict__ insts,
                                                           const Tile* __restrict__ tiles, int nt,
                                                           const double* __restrict__ Xb,
                                                           const double* __restrict__ rbarb, double* __restrict__ Wb,
                                                           double* __restrict__ pbar) {
    extern __shared__ __align__(16) double adj_cell_smem[];
    double* sP = adj_cell_smem;                // [5][RHS_NPT] p_e, p_i, p_r, u, v
    double* sB = adj_cell_smem + 5 * RHS_NPT;  // [5][RHS_NPT] their cotangents
    __shared__ double red[2][RHS_THREADS / 32];
    if ((int)blockIdx.x >= nt) return;
    const Tile t = tiles[blockIdx.x];
    const Inst& I = insts[t.inst];
    if (has_error(I)) return;
    const DevParams& P = I.P;
    const long long plane = I.plane;
    const double* X = Xb + I.aoff;
    const double* rb = rbarb + I.aoff;
    double* W = Wb + I.aoff;
    const int nx = I.nx, ny = I.ny;
    const int TJ = 1 << t.lg, TI = RHS_THREADS >> t.lg;
    const int HJ = TJ + 8, NPT = (TI + 8) * HJ;
    for (int p = threadIdx.x; p < NPT; p += blockDim.x) {
        const int hi = p / HJ, hj = p - hi * HJ;
        const bool corner = (hi < 4 || hi >= TI + 4) && (hj < 4 || hj >= TJ + 4);
        const int i = t.i - 4 + hi, j = t.j0 - 4 + hj;
        for (int q = 0; q < 5; ++q) sB[q * RHS_NPT + p] = 0.0;
        if (corner || i < -RH3T_PAD || i >= nx + RH3T_PAD || j < -RH3T_PAD || j >= ny + RH3T_PAD) continue;
        double s[6];
        load6(X, plane, node_of(I, i, j), s);
        const Prim d = prim_from_state(s, P);
        sP[p] = d.pe; sP[RHS_NPT + p] = d.pi; sP[2 * RHS_NPT + p] = d.pr;
        sP[3 * RHS_NPT + p] = d.u; sP[4 * RHS_NPT + p] = d.v;
    }
    __syncthreads();
    const int ti = threadIdx.x >> t.lg, tj = threadIdx.x & (TJ - 1);
    const int i = t.i + ti, j = t.j0 + tj;
    double oei_b = 0.0, oer_b = 0.0;
    if (i < nx && j < ny && I.mask[node_of(I, i, j)]) {
        const long long n = node_of(I, i, j);
        const double ob[3] = {rb[3 * plane + n], rb[4 * plane + n], rb[5 * plane + n]};
        const int hc = (ti + 4) * HJ + (tj + 4);
        for (int dir = 0; dir < 2; ++dir) {
            const int step = dir == 0 ? HJ : 1;
            double pe[9], pi[9], pr[9], vel[9];
            for (int q = 0; q < 9; ++q) {
                const int p = hc + (q - 4) * step;
                pe[q] = sP[p]; pi[q] = sP[RHS_NPT + p]; pr[q] = sP[2 * RHS_NPT + p];
                vel[q] = sP[(dir == 0 ? 3 : 4) * RHS_NPT + p];
            }
            double peb[9], pib[9], prb[9], velb[9];
            noncon9_vjp(pe, pi, pr, vel, dir == 0 ? I.dx : I.dy, ob, peb, pib, prb, velb);
            for (int q = 0; q < 9; ++q) {
                const int p = hc + (q - 4) * step;
                if (peb[q] != 0.0) atomicAdd(&sB[p], peb[q]);
                if (pib[q] != 0.0) atomicAdd(&sB[RHS_NPT + p], pib[q]);
                if (prb[q] != 0.0) atomicAdd(&sB[2 * RHS_NPT + p], prb[q]);
                if (velb[q] != 0.0) atomicAdd(&sB[(dir == 0 ? 3 : 4) * RHS_NPT + p], velb[q]);
            }
        }
        if (I.source) { // source.rs:7-21
            double s[6];
            load6(X, plane, n, s);
            double te, ti_, tr;
            temps_from_state(s, P, te, ti_, tr);
            const double oei = P.omega_ei, oer = P.omega_er;
            const double te3 = te * te * te, tr3 = tr * tr * tr;
            const double bte = -oei * ob[0] - oer * 4.0 * te3 * ob[0] + oei * ob[1] + oer * 4.0 * te3 * ob[2];
            const double bti = oei * ob[0] - oei * ob[1];
            const double btr = oer * 4.0 * tr3 * ob[0] - oer * 4.0 * tr3 * ob[2];
            double sb[6] = {0, 0, 0, 0, 0, 0};
            temps_vjp(s, P, bte, bti, btr, sb);
            atomic_add6(W, plane, n, sb);
            const double x4 = pow4d(te) - pow4d(tr);
            oei_b = -(te - ti_) * ob[0] + (te - ti_) * ob[1];
            oer_b = -x4 * ob[0] + x4 * ob[2];
        }
    }
    if (I.source) {
        for (int o = 16; o > 0; o >>= 1) {
            oei_b += __shfl_xor_sync(0xffffffffu, oei_b, o);
            oer_b += __shfl_xor_sync(0xffffffffu, oer_b, o);
        }
        if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = oei_b; red[1][threadIdx.x >> 5] = oer_b; }
    }
    __syncthreads();
    if (I.source && threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < RHS_THREADS / 32; ++w) { a += red[0][w]; b += red[1][w]; }
        if (a != 0.0) atomicAdd(&pbar[8 * t.inst + 6], a);
        if (b != 0.0) atomicAdd(&pbar[8 * t.inst + 7], b);
    }
    // primitive cotangents -> state cotangents, one node each
    for (int p = threadIdx.x; p < NPT; p += blockDim.x) {
        const double b0 = sB[p], b1 = sB[RHS_NPT + p], b2 = sB[2 * RHS_NPT + p], b3 = sB[3 * RHS_NPT + p],
                     b4 = sB[4 * RHS_NPT + p];
        if (b0 == 0.0 && b1 == 0.0 && b2 == 0.0 && b3 == 0.0 && b4 == 0.0) continue;
        const int hi = p / HJ, hj = p - hi * HJ;
        const long long m = node_of(I, t.i - 4 + hi, t.j0 - 4 + hj);
        double s[6];
        load6(X, plane, m, s);
        double sb[6] = {0, 0, 0, 0, 0, 0};
        prim_vjp(s, P, b3, b4, 0.0, 0.0, 0.0, b0, b1, b2, sb);
        atomic_add6(W, plane, m, sb);
    }
}

// ---------------------------------------------------------------- ghosts
// Heavy (FarField) ghosts in three launches:
//   k_adj_ghost_lr    one thread per ghost: L, R and lambda at the nearest
//                     node of X (bc1.rs:294-312), every thread running the
//                     same six rows, into the ghost's scratch slot;
//   k_adj_ghosts      one warp per ghost: the forward pass again (D, S d,
//                     beta, alpha, V, v) and its reverse down to the
//                     cotangents of the stencil states (-> Ub), of the
//                     FarField state and of R (L-bar folded in), which goes
//                     to the scratch slot; cheap ghosts, one thread each;
//   k_adj_ghost_tail  one thread per ghost: the Roe base of the nearest
//                     node's state from R-bar -> Ub at that node.
// A scratch slot holds AG_SLOT doubles: L (36), R by column (36), lambda (6),
// pad (2), R-bar (36).
constexpr int AG_WARPS = 3;
constexpr int AG_LR_THREADS = 128;
constexpr int AG_RB = 80;
__constant__ int kAStOff[6] = {0, 1, 5, 14, 30, 55};
__constant__ int kASOff[6] = {0, 1, 17, 98, 354, 979};
__constant__ int kAWOff[6] = {0, 1, 9, 36, 100, 225};


struct AdjGhostWarp {
    double L[36], R[36], lam[6];             // L[6c + j]; R column c at R[6c + i]
    double U6[6][56];                        // rotated stencil states
    double D[56][6];                         // d_c of stencil node a at row d_row(a)
    double ACC[6][56], STD[6][56];           // ACC: S d; STD: D-bar
    double alpha[6][5], beta[6][5], V[6][5][5];
    double v[5][6], x[5][6], ub[5][6], xb[5][6], vinf[6], vinfb[6];
    double Lb[6][6], Rb[6][6];
    double vb[5][6];
    double Z[6][6];
    double omm[6][5]; // omega_r * omega-bar_r per field
};

__device__ __forceinline__ int aorder(int a) { return a < 1 ? 0 : (a < 5 ? 1 : (a < 14 ? 2 : (a < 30 ? 3 : 4))); }

// the nearest node's state of ghost Rg, rotated to its (n, t) frame, and its Roe state
__device__ __forceinline__ Roe nearest_roe(const Inst& I, const GhostRec& Rg, const double* __restrict__ X,
                                           double q6[6]) {
    double s[6];
    load6(X, I.plane, Rg.src, s);
    q6[0] = s[0]; q6[1] = s[1] * Rg.nx + s[2] * Rg.ny; q6[2] = -s[1] * Rg.ny + s[2] * Rg.nx;
    q6[3] = s[3]; q6[4] = s[4]; q6[5] = s[5];
    const Prim d1 = prim_from_state(q6, I.P);
    return roe_average(q6[0], d1, q6[0], d1, I.P);
}

// L, R, lambda of FarField ghost g into its scratch slot, staged in shared
// memory ([value][thread]) and stored by whole warps
constexpr int AG_LR_SMEM = 80 * (AG_LR_THREADS + 1) * (int)sizeof(double);
__global__ void __launch_bounds__(AG_LR_THREADS) k_adj_ghost_lr(const Inst* __restrict__ insts,
                                                               const GhostRec* __restrict__ heavy, int nh,
                                                               const double* __restrict__ Xb,
                                                               double* __restrict__ slots) {
    extern __shared__ __align__(16) double lr_smem[];
    constexpr int ST = AG_LR_THREADS + 1;
    const int g0 = blockIdx.x * AG_LR_THREADS, g = g0 + threadIdx.x;
    if (g < nh) {
        const GhostRec Rg = heavy[g];
        const Inst& I = insts[Rg.inst];
        if (!has_error(I)) {
            double q6[6];
            const Roe q = nearest_roe(I, Rg, Xb + I.aoff, q6);
            double* o = lr_smem + threadIdx.x;
            for (int row = 0; row < 6; ++row) {
                double Lr[6], Rcol[6], lm;
                l_row<0>(row, q, I.P, Lr);
                r_col<0>(row, q, I.P, Rcol, lm);
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    o[(6 * row + k) * ST] = Lr[k];
                    o[(36 + 6 * row + k) * ST] = Rcol[k];
                }
                o[(72 + row) * ST] = lm;
            }
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int j = 0; j < 32; ++j) {
        const int t = 32 * w + j, gj = g0 + t;
        if (gj >= nh) break;
        double* o = slots + (size_t)gj * AG_SLOT;
        for (int e = lane; e < 78; e += 32) o[e] = lr_smem[e * ST + t];
    }
}

// A x = b for a 6x6 system by LU with partial pivoting (the forward's
// bc1.rs:467-469 solve6); A is overwritten; false if singular
__device__ bool lu_solve6(double A[6][6], double b[6]) {
    int piv[6];
    for (int j = 0; j < 6; ++j) {
        int p = j;
        double mx = fabs(A[j][j]);
        for (int i = j + 1; i < 6; ++i)
            if (fabs(A[i][j]) > mx) { mx = fabs(A[i][j]); p = i; }
        piv[j] = p;
        if (A[p][j] == 0.0) return false;
        if (p != j)
            for (int k = 0; k < 6; ++k) { const double t = A[j][k]; A[j][k] = A[p][k]; A[p][k] = t; }
        const double rcp = 1.0 / A[j][j];
        for (int i = j + 1; i < 6; ++i) A[i][j] *= rcp;
        for (int k = j + 1; k < 6; ++k)
            for (int i = j + 1; i < 6; ++i) A[i][k] -= A[i][j] * A[j][k];
    }
    for (int j = 0; j < 6; ++j)
        if (piv[j] != j) { const double t = b[j]; b[j] = b[piv[j]]; b[piv[j]] = t; }
    for (int k = 0; k < 6; ++k)
        for (int i = k + 1; i < 6; ++i) b[i] -= b[k] * A[i][k];
    for (int k = 5; k >= 0; --k) {
        b[k] /= A[k][k];
        for (int i = 0; i < k; ++i) b[i] -= b[k] * A[i][k];
    }
    return true;
}

// Wall (ILW, bc1.rs:691-756) or Outflow (LODI, bc1.rs:760-828) rows in
// reverse, on one lane: from ub[k] (cotangents of u_k) and the forward's v,
// L, R to vb[k] (cotangents of v_k), Rb (R columns) and Lb (L rows, from the
// ILW systems). Wall: u_0 = A_0^-1 r_0 with A_0 = L but row 0 = e_1 and
// r_0 = v_0 but r_0[0] = 0, u_1 = A_1^-1 r_1 with row 0 of A_1 the ILW
// momentum row of u_0, u_k = R v_k (k >= 2); so r-bar = A^-T u-bar and
// A-bar = -r-bar u^T. Outflow: u_k = R r_k with r_k = v_k except
// r_1[0] = l_1(u_0) / lambda_1(u_0) when lambda_1 = u_n - a < 0 (its
// gradient by dual numbers). Returns false if an ILW system is singular.
__device__ __noinline__ bool wall_outflow_vjp(const Inst& I, const GhostRec& Rg, AdjGhostWarp& G) {
    const DevParams& P = I.P;
    const double* L = G.L; // L[c][j] = L[6c + j]
    const double* Rc = G.R; // R[i][c] = Rc[6c + i]
    double Rb[6][6], Lb[6][6], vb[5][6];
    for (int c = 0; c < 6; ++c)
        for (int i = 0; i < 6; ++i) { Rb[c][i] = 0.0; Lb[c][i] = 0.0; }
    for (int k = 0; k < 5; ++k)
        for (int c = 0; c < 6; ++c) vb[k][c] = 0.0;
    // u_k = R v_k, k = 2..4 (both kinds)
    for (int k = 2; k <= 4; ++k)
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0;
            for (int i = 0; i < 6; ++i) {
                acc += Rc[6 * c + i] * G.ub[k][i];
                Rb[c][i] += G.ub[k][i] * G.v[k][c];
            }
            vb[k][c] = acc;
        }
    double u0b[6];
    for (int c = 0; c < 6; ++c) u0b[c] = G.ub[0][c];
    if (Rg.kind == BC_WALL) {
        const double gi = P.gamma_i - 1.0, ge = P.gamma_e - 1.0, gr = P.gamma_r - 1.0, gt = gi + ge + gr;
        double A0[6][6], u0[6], A1[6][6], u1[6], T[6][6];
        for (int i = 0; i < 6; ++i)
            for (int c = 0; c < 6; ++c) A0[i][c] = i == 0 ? (c == 1 ? 1.0 : 0.0) : L[6 * i + c];
        for (int c = 0; c < 6; ++c) u0[c] = c == 0 ? 0.0 : G.v[0][c];
        for (int i = 0; i < 6; ++i)
            for (int c = 0; c < 6; ++c) T[i][c] = A0[i][c];
        if (!lu_solve6(T, u0)) return false;
        const double a1 = u0[0], a3 = u0[2];
        const double row1[6] = {-gt * a3 * a3 / (6.0 * a1 * a1), 0.0, gt * a3 / (6.0 * a1), -ge, -gi, -gr};
        for (int i = 0; i < 6; ++i)
            for (int c = 0; c < 6; ++c) A1[i][c] = i == 0 ? row1[c] : L[6 * i + c];
        for (int c = 0; c < 6; ++c) u1[c] = c == 0 ? 0.0 : G.v[1][c];
        for (int i = 0; i < 6; ++i)
            for (int c = 0; c < 6; ++c) T[i][c] = A1[i][c];
        if (!lu_solve6(T, u1)) return false;
        // k = 1: r1-bar = A1^-T u1-bar, A1-bar = -r1-bar u1^T
        double r1b[6];
        for (int c = 0; c < 6; ++c) r1b[c] = G.ub[1][c];
        for (int i = 0; i < 6; ++i)
            for (int c = 0; c < 6; ++c) T[i][c] = A1[c][i];
        if (!lu_solve6(T, r1b)) return false;
        for (int c = 1; c < 6; ++c) vb[1][c] = r1b[c];
        for (int i = 1; i < 6; ++i)
            for (int c = 0; c < 6; ++c) Lb[i][c] -= r1b[i] * u1[c];
        // row 0 of A1 = the ILW row of u0 (u0[0], u0[2])
        const double b0 = -r1b[0] * u1[0], b2 = -r1b[0] * u1[2];
        u0b[0] += b0 * (gt * a3 * a3 / (3.0 * a1 * a1 * a1)) + b2 * (-gt * a3 / (6.0 * a1 * a1));
        u0b[2] += b0 * (-gt * a3 / (3.0 * a1 * a1)) + b2 * (gt / (6.0 * a1));
        // k = 0
        for (int i = 0; i < 6; ++i)
            for (int c = 0; c < 6; ++c) T[i][c] = A0[c][i];
        if (!lu_solve6(T, u0b)) return false;
        for (int c = 1; c < 6; ++c) vb[0][c] = u0b[c];
        for (int i = 1; i < 6; ++i)
            for (int c = 0; c < 6; ++c) Lb[i][c] -= u0b[i] * u0[c];
    } else {
        const DevBC& bc = I.bcs[Rg.bc];
        // forward: u0 = R v0, the LODI row test on it
        DualN<6> q[6];
        for (int i = 0; i < 6; ++i) {
            double acc = 0.0;
            for (int c = 0; c < 6; ++c) acc += Rc[6 * c + i] * G.v[0][c];
            q[i] = DualN<6>::var(acc, i);
        }
        const DualN<6> rho0 = q[0], un0 = q[1] / rho0, ut0 = q[2] / rho0;
        const DualN<6> w2 = un0 * un0 + ut0 * ut0;
        const DualN<6> ee1 = q[3] / rho0 - w2 * K6, ei1 = q[4] / rho0 - w2 * K6, er1 = q[5] / rho0 - w2 * K6;
        const double ge = P.gamma_e - 1.0, gi = P.gamma_i - 1.0, gr = P.gamma_r - 1.0;
        const DualN<6> p0 = rho0 * (ge * ee1 + gi * ei1 + gr * er1);
        const DualN<6> a = sqrt(P.gamma_e * ge * ee1 + P.gamma_i * gi * ei1 + P.gamma_r * gr * er1);
        const DualN<6> lambda1 = un0 - a;
        const bool lodi = lambda1.v < 0.0;
        double rhs1[6];
        for (int c = 0; c < 6; ++c) rhs1[c] = G.v[1][c];
        DualN<6> g;
        if (lodi) {
            const DualN<6> ml = fabs(un0 / a);
            const DualN<6> l1 = bc.sigma * (1.0 - ml * ml) * a / bc.l_domain * (p0 - bc.p_inf);
            g = l1 / lambda1;
            rhs1[0] = g.v;
        }
        // k = 1: u1 = R rhs1
        double r1b[6];
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0;
            for (int i = 0; i < 6; ++i) {
                acc += Rc[6 * c + i] * G.ub[1][i];
                Rb[c][i] += G.ub[1][i] * rhs1[c];
            }
            r1b[c] = acc;
        }
        for (int c = 0; c < 6; ++c) vb[1][c] = r1b[c];
        if (lodi) {
            vb[1][0] = 0.0;
            for (int i = 0; i < 6; ++i) u0b[i] += r1b[0] * g.d[i];
        }
        // k = 0: u0 = R v0
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0;
            for (int i = 0; i < 6; ++i) {
                acc += Rc[6 * c + i] * u0b[i];
                Rb[c][i] += u0b[i] * G.v[0][c];
            }
            vb[0][c] = acc;
        }
    }
    for (int c = 0; c < 6; ++c)
        for (int i = 0; i < 6; ++i) { G.Rb[c][i] = Rb[c][i]; G.Lb[c][i] = Lb[c][i]; }
    for (int k = 0; k < 5; ++k)
        for (int c = 0; c < 6; ++c) G.vb[k][c] = vb[k][c];
    return true;
}

// two rows of one order of the record (S_r transposed, stride m, or w_{r,k},
// stride 1; read from global memory, prefetched to L2) with the stencil
// data d, all six fields: an S row stores (S_r d_c)_a, a w row V^(k)_{c,r}
__device__ __forceinline__ void adj_dot_pair(AdjGhostWarp& G, const double* __restrict__ rec, unsigned codes) {
    if (codes == kPairNone) return;
    const unsigned c1 = codes & 0xffffu, c2 = codes >> 16;
    const int r = (int)((c1 >> 5) & 7u), m = (r + 1) * (r + 1);
    const int i1 = (int)(c1 & 31u), i2 = (int)(c2 & 31u);
    const bool w1 = (c1 >> 8) != 0, w2 = (c2 >> 8) != 0;
    const double* __restrict__ p1 = w1 ? rec + GH_W + kAWOff[r] + i1 * m : rec + GH_S + kASOff[r] + i1;
    const double* __restrict__ p2 = w2 ? rec + GH_W + kAWOff[r] + i2 * m : rec + GH_S + kASOff[r] + i2;
    const int s1 = w1 ? 1 : m, s2 = w2 ? 1 : m;
    const double(*__restrict__ D)[6] = G.D + kDOff[r];
    double a1[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, a2[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    // the record is read from L2: the loads of the next four terms are in
    // flight while four terms are summed (in order)
    constexpr int PF = 4;
    double x1[PF], x2[PF];
#pragma unroll
    for (int j = 0; j < PF; ++j) {
        x1[j] = j < m ? __ldg(p1 + j * s1) : 0.0;
        x2[j] = j < m ? __ldg(p2 + j * s2) : 0.0;
    }
    for (int b0 = 0; b0 < m; b0 += PF) {
        double y1[PF], y2[PF];
#pragma unroll
        for (int j = 0; j < PF; ++j) {
            const int bn = b0 + PF + j;
            y1[j] = bn < m ? __ldg(p1 + bn * s1) : 0.0;
            y2[j] = bn < m ? __ldg(p2 + bn * s2) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < PF; ++j) {
            if (b0 + j < m) {
                double d[6];
                load_d6(D[b0 + j], d);
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    a1[c] += x1[j] * d[c];
                    a2[c] += x2[j] * d[c];
                }
            }
        }
#pragma unroll
        for (int j = 0; j < PF; ++j) { x1[j] = y1[j]; x2[j] = y2[j]; }
    }
    const int off = kAStOff[r];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        if (w1) G.V[c][r][i1] = a1[c];
        else G.ACC[c][off + i1] = a1[c];
        if (w2) G.V[c][r][i2] = a2[c];
        else G.ACC[c][off + i2] = a2[c];
    }
}

// L2 prefetch of a ghost's record by the bulk-copy engine (16-byte aligned,
// size a multiple of 16; nothing waits on it)
__device__ __forceinline__ void prefetch_record_l2(const double* rec) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(rec), "r"((unsigned)(GH_REC * 8)) : "memory");
}

// one heavy ghost per warp; gb from W at the ghost node. WO: the Wall /
// Outflow instantiation (their rows on one lane through wall_outflow_vjp);
// the FarField one has no call and keeps its registers
template <bool WO>
__device__ void ghost_vjp_warp(const Inst& I, const GhostRec& Rg, const double* __restrict__ rec,
                               const double* __restrict__ X, const double* __restrict__ W, double* __restrict__ Ub,
                               double* __restrict__ pbar_k, double* __restrict__ slot, AdjGhostWarp& G, int lane) {
    const DevParams& P = I.P;
    const long long plane = I.plane;
    const double nx = Rg.nx, ny = Rg.ny;
    // the record's S_r and w are read in steps below: have them in L2 first
    if (lane == 0) prefetch_record_l2(rec);
    // L, R, lambda at the nearest node of X (k_adj_ghost_lr), the stencil
    // indices and then the stencil states: all loads in flight together
    double sl[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) sl[j] = lane + 32 * j < 78 ? slot[lane + 32 * j] : 0.0;
    // read much later, loaded now: the cotangent at the ghost node and the
    // FarField state, component `lane` on lanes 0-5
    const double w_gn = lane < 6 ? W[lane * plane + Rg.node] : 0.0;
    const double ui_l = lane < 6 ? I.bcs[Rg.bc].state[lane] : 0.0;
    const int32_t* st = reinterpret_cast<const int32_t*>(rec + GH_ST);
    const int i0 = __ldg(&st[lane]), i1 = lane + 32 < 55 ? __ldg(&st[lane + 32]) : 0;
    double sx0[6], sx1[6];
    load6(X, plane, i0, sx0);
    if (lane + 32 < 55) load6(X, plane, i1, sx1);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const int e = lane + 32 * j;
        if (e < 36) G.L[e] = sl[j];
        else if (e < 72) G.R[e - 36] = sl[j];
        else if (e < 78) G.lam[e - 72] = sl[j];
    }
    __syncwarp();
    const double* L = G.L;    // L[c][j] = L[6c + j]
    const double* Rc = G.R;   // R[i][c] = Rc[6c + i]
    const double* lam = G.lam;
    // ---- forward: D, ACC = S d, beta, alpha, V, v. S_r = P^T M_r P is
    // symmetric (bc1.rs:169-175), so d beta / d d = 2 S d: S^T d is not formed
    auto project = [&](int a, const double s[6]) {
        const double u6[6] = {s[0], s[1] * nx + s[2] * ny, -s[1] * ny + s[2] * nx, s[3], s[4], s[5]};
        for (int q = 0; q < 6; ++q) G.U6[q][a] = u6[q];
        double d[6];
        for (int c = 0; c < 6; ++c) {
            double acc = 0.0;
            for (int q = 0; q < 6; ++q) acc += L[6 * c + q] * u6[q];
            d[c] = acc;
        }
        store_d6(G.D[d_row(a)], d);
    };
    project(lane, sx0);
    if (lane + 32 < 55) project(lane + 32, sx1);
    __syncwarp();
    // the 70 rows (S d)_a and V^(k)_{c,r} = w_{r,k} . d_c, as pairs of rows of one order
    adj_dot_pair(G, rec, kSlotA[lane]);
    adj_dot_pair(G, rec, kSlotB[lane]);
    __syncwarp();
    if (lane < 30) {
        const int c = lane / 5, r = lane - 5 * (lane / 5);
        const int m = (r + 1) * (r + 1), off = kAStOff[r], doff = kDOff[r];
        double beta = 0.0;
#pragma unroll 5
        for (int a = 0; a < m; ++a) beta += G.D[doff + a][c] * G.ACC[c][off + a];
        G.beta[c][r] = beta;
        const double x = P.eps + beta;
        double xq;
        if (P.weno_q == 10.0) { const double x2 = x * x, x4 = x2 * x2, x8 = x4 * x4; xq = x8 * x2; }
        else xq = pow(x, P.weno_q);
        G.alpha[c][r] = rec[GH_D + r] / xq;
        for (int k = r + 1; k < 5; ++k) G.V[c][r][k] = 0.0;
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
    double ui[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) ui[q] = __shfl_sync(0xffffffffu, ui_l, q);
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
    double o[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) o[q] = __shfl_sync(0xffffffffu, w_gn, q);
    if (lane == 0) {
        // out1 = mn nx - mt ny, out2 = mn ny + mt nx
        const double gb[6] = {o[0], o[1] * nx + o[2] * ny, -o[1] * ny + o[2] * nx, o[3], o[4], o[5]};
        double coef = 1.0;
        for (int k = 0; k < 5; ++k) {
            if (k > 0) coef *= Rg.dist / (double)k;
            for (int c = 0; c < 6; ++c) G.ub[k][c] = coef * gb[c];
        }
    }
    __syncwarp();
    if (WO) {
        const bool ok = __shfl_sync(0xffffffffu, lane == 0 ? (wall_outflow_vjp(I, Rg, G) ? 1 : 0) : 0, 0) != 0;
        if (!ok) {
            if (lane == 0) report(I, 1, 3, (unsigned)Rg.gid);
            return;
        }
        __syncwarp();
    } else {
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
    } // FarField
    // v[k][c] = sum_r (alpha_r / sum) V_r^k -> V-bar, alpha-bar -> beta-bar,
    // lanes (c, r)
    const int oc = lane / 5, orr = lane - 5 * (lane / 5);
    double asum = 0.0, om = 0.0, omb = 0.0;
    if (lane < 30) {
        for (int r = 0; r < 5; ++r) asum += G.alpha[oc][r];
        om = G.alpha[oc][orr] / asum;
        for (int k = 0; k < 5; ++k) omb += G.V[oc][orr][k] * G.vb[k][oc];
        G.omm[oc][orr] = om * omb;
    }
    __syncwarp();
    if (lane < 30) {
        double m = 0.0;
        for (int r = 0; r < 5; ++r) m += G.omm[oc][r];
        const double ab = (omb - m) / asum;
        // alpha = d (eps + beta)^-q
        G.beta[oc][orr] = -P.weno_q * ab * G.alpha[oc][orr] / (P.eps + G.beta[oc][orr]); // now beta-bar
        for (int k = 0; k < 5; ++k) G.V[oc][orr][k] = om * G.vb[k][oc];                 // now V-bar
    }
    __syncwarp();
    // D-bar over the 55 nodes: beta = d^T S d, V = w . d (the w columns of
    // both of a lane's nodes are loaded together)
    {
        const int r0 = aorder(lane), m0 = (r0 + 1) * (r0 + 1), ar0 = lane - kAStOff[r0];
        const int ar1 = lane + 32 - kAStOff[4]; // the second node is of order 4
        double wv0[5], wv1[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            wv0[k] = k <= r0 ? __ldg(&rec[GH_W + kAWOff[r0] + k * m0 + ar0]) : 0.0;
            wv1[k] = lane + 32 < 55 ? __ldg(&rec[GH_W + kAWOff[4] + k * 25 + ar1]) : 0.0;
        }
        for (int c = 0; c < 6; ++c) {
            double acc = G.beta[c][r0] * (2.0 * G.ACC[c][lane]);
            for (int k = 0; k <= r0; ++k) acc += G.V[c][r0][k] * wv0[k];
            G.STD[c][lane] = acc; // D-bar
        }
        if (lane + 32 < 55) {
            for (int c = 0; c < 6; ++c) {
                double acc = G.beta[c][4] * (2.0 * G.ACC[c][lane + 32]);
#pragma unroll
                for (int k = 0; k < 5; ++k) acc += G.V[c][4][k] * wv1[k];
                G.STD[c][lane + 32] = acc;
            }
        }
    }
    __syncwarp();
    // D = L rot(u_a): Lb += DB rot(u_a)^T (18 lanes, entries (c, q) and (c, q + 1)),
    // rot(u_a)-bar = L^T DB
    if (lane < 18) {
        const int c = lane / 3, q = 2 * (lane - 3 * (lane / 3));
        double acc0 = 0.0, acc1 = 0.0;
        for (int a = 0; a < 55; ++a) {
            const double sd = G.STD[c][a];
            acc0 += sd * G.U6[q][a];
            acc1 += sd * G.U6[q + 1][a];
        }
        G.Lb[c][q] += acc0;
        G.Lb[c][q + 1] += acc1;
    }
    {
        // both of a lane's nodes per row of L (one read of L)
        const bool two = lane + 32 < 55;
        double ur0[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, ur1[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double d0 = G.STD[c][lane], d1 = two ? G.STD[c][lane + 32] : 0.0;
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                const double l = L[6 * c + q];
                ur0[q] += l * d0;
                ur1[q] += l * d1;
            }
        }
        const double sb0[6] = {ur0[0], ur0[1] * nx - ur0[2] * ny, ur0[1] * ny + ur0[2] * nx, ur0[3], ur0[4], ur0[5]};
        atomic_add6(Ub, plane, i0, sb0);
        if (two) {
            const double sb1[6] = {ur1[0], ur1[1] * nx - ur1[2] * ny, ur1[1] * ny + ur1[2] * nx, ur1[3], ur1[4],
                                   ur1[5]};
            atomic_add6(Ub, plane, i1, sb1);
        }
    }
    __syncwarp();
    // L, R of the nearest node: L-bar folded into R-bar (lanes over the 36
    // entries), then the Roe base of two equal rotated states
    for (int e = lane; e < 36; e += 32) {
        const int j = e / 6, c = e - 6 * (e / 6);
        double acc = 0.0;
        for (int k = 0; k < 6; ++k) acc += G.Lb[j][k] * L[6 * c + k];
        G.Z[j][c] = acc;
    }
    __syncwarp();
    for (int e = lane; e < 36; e += 32) {
        const int c = e / 6, i = e - 6 * (e / 6);
        double acc = 0.0;
        for (int j = 0; j < 6; ++j) acc += L[6 * j + i] * G.Z[j][c];
        G.Rb[c][i] -= acc;
    }
    __syncwarp();
    // R-bar to the scratch slot (k_adj_ghost_tail)
    for (int e = lane; e < 36; e += 32) slot[AG_RB + e] = G.Rb[e / 6][e - 6 * (e / 6)];
}

// the Roe base of the nearest node of FarField ghost g from its R-bar -> Ub
__global__ void __launch_bounds__(128) k_adj_ghost_tail(const Inst* __restrict__ insts,
                                                        const GhostRec* __restrict__ heavy, int nh,
                                                        const double* __restrict__ Xb,
                                                        const double* __restrict__ slots, double* __restrict__ Ubb) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nh) return;
    const GhostRec Rg = heavy[g];
    const Inst& I = insts[Rg.inst];
    if (has_error(I)) return;
    double q6[6];
    const Roe q = nearest_roe(I, Rg, Xb + I.aoff, q6);
    const double* o = slots + (size_t)g * AG_SLOT + AG_RB;
    double Rb[6][6];
    for (int e = 0; e < 36; ++e) Rb[e / 6][e - 6 * (e / 6)] = o[e];
    const double base[5] = {q.u, q.v, q.ee, q.ei, q.er};
    const double lamb[6] = {0, 0, 0, 0, 0, 0};
    double bb[5] = {0, 0, 0, 0, 0};
    r_base_vjp<0>(base, I.P, Rb, lamb, bb);
    double ga[6] = {0, 0, 0, 0, 0, 0}, gb2[6] = {0, 0, 0, 0, 0, 0};
    roe_vjp(q6, q6, I.P, bb, ga, gb2);
    double gr[6];
    for (int c = 0; c < 6; ++c) gr[c] = ga[c] + gb2[c];
    const double nx = Rg.nx, ny = Rg.ny;
    const double sb[6] = {gr[0], gr[1] * nx - gr[2] * ny, gr[1] * ny + gr[2] * nx, gr[3], gr[4], gr[5]};
    atomic_add6(Ubb + I.aoff, I.plane, Rg.src, sb);
}

template <bool WO>
__global__ void __launch_bounds__(AG_WARPS * 32, 5) k_adj_ghosts(const Inst* __restrict__ insts,
                                                             const GhostRec* __restrict__ heavy, int nh,
                                                             const GhostRec* __restrict__ cheap, int nc,
                                                             const double* __restrict__ hrec,
                                                             const double* __restrict__ Xb,
                                                             const double* __restrict__ Wb,
                                                             double* __restrict__ Ubb, double* __restrict__ pbar,
                                                             double* __restrict__ slots, int nbh) {
    __shared__ AdjGhostWarp G[AG_WARPS];
    const int lane = threadIdx.x & 31;
    if ((int)blockIdx.x < nbh) {
        const int g = blockIdx.x * AG_WARPS + (threadIdx.x >> 5);
        if (g >= nh) return;
        const GhostRec Rg = heavy[g];
        const Inst& I = insts[Rg.inst];
        if (has_error(I) || (Rg.kind != BC_FAR_FIELD) != WO) return;
        ghost_vjp_warp<WO>(I, Rg, hrec + (size_t)Rg.heavy * GH_REC, Xb + I.aoff, Wb + I.aoff, Ubb + I.aoff,
                       pbar + 8 * Rg.inst, slots + (size_t)g * AG_SLOT, G[threadIdx.x >> 5], lane);
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
void launch_adj_l(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, const Tile* tx, int ntx,
                  const Tile* ty, int nty, const Tile* tr, int ntr, const GhostRec* heavy, int nh,
                  const GhostRec* cheap, int nc, const double* hrec, const double* X, const double* rbar, double* W,
                  double* Ub, double* pbar, double* slots, int wall_outflow) {
    if (n <= 0) return;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_adj_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, ADJ_CELL_SMEM);
        cudaFuncSetAttribute(k_adj_flux, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(AdjFluxShared));
        cudaFuncSetAttribute(k_adj_ghost_lr, cudaFuncAttributeMaxDynamicSharedMemorySize, AG_LR_SMEM);
        attr = true;
    }
    if (nh > 0)
        k_adj_ghost_lr<<<(nh + AG_LR_THREADS - 1) / AG_LR_THREADS, AG_LR_THREADS, AG_LR_SMEM, s>>>(insts, heavy, nh,
                                                                                                  X, slots);
    const unsigned cb = (unsigned)((max_cells + 127) / 128);
    if (ntx + nty > 0)
        k_adj_flux<<<ntx + nty, FLUX_THREADS, sizeof(AdjFluxShared), s>>>(insts, tx, ntx, ty, nty, X, rbar, W);
    if (ntr > 0) k_adj_cells<<<ntr, RHS_THREADS, ADJ_CELL_SMEM, s>>>(insts, tr, ntr, X, rbar, W, pbar);
    const int nbh = (nh + AG_WARPS - 1) / AG_WARPS, nbc = (nc + AG_WARPS * 32 - 1) / (AG_WARPS * 32);
    if (nbh + nbc > 0)
        k_adj_ghosts<false><<<nbh + nbc, AG_WARPS * 32, 0, s>>>(insts, heavy, nh, cheap, nc, hrec, X, W, Ub, pbar,
                                                                 slots, nbh);
    if (wall_outflow && nbh > 0)
        k_adj_ghosts<true><<<nbh, AG_WARPS * 32, 0, s>>>(insts, heavy, nh, cheap, 0, hrec, X, W, Ub, pbar, slots, nbh);
    if (nh > 0) k_adj_ghost_tail<<<(nh + 127) / 128, 128, 0, s>>>(insts, heavy, nh, X, slots, Ub);
    k_adj_fluid<<<dim3(cb, n), 128, 0, s>>>(insts, k0, W, Ub);
}

int adj_l_launches(int nh, int nc, int wall_outflow) {
    return 3 + (nh + nc > 0 ? 1 : 0) + (nh > 0 ? 2 : 0) + (wall_outflow && nh > 0 ? 1 : 0);
}

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
// the minimum. Steps whose dt was clipped to t_final have none.
// k_adj_dt_find: that cell's index per instance (argmin initialised to ~0).
__global__ void __launch_bounds__(256) k_adj_dt_find(const Inst* __restrict__ insts, int k0,
                                                     const double* __restrict__ X, const DevScalars* __restrict__ sc,
                                                     const double* __restrict__ dtbar,
                                                     unsigned long long* __restrict__ argmin) {
    const int k = k0 + blockIdx.y;
    const Inst& I = insts[k];
    const DevScalars& S = sc[k];
    if (!(S.dt == S.cfl_factor * S.dt_cfl) || dtbar[k] == 0.0) return;
    const long long l = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= (long long)I.nx * I.ny) return;
    const long long n = node_of(I, (int)(l / I.ny), (int)(l % I.ny));
    if (!I.mask[n]) return;
    double s[6];
    load6(X + I.aoff, I.plane, n, s);
    if (local_dt(s, I.dx, I.dy, I.P) == S.dt_cfl) atomicMin(&argmin[k], (unsigned long long)l);
}

// k_adj_dt_apply: one thread per instance, dual numbers in the state and omegas
__global__ void k_adj_dt_apply(const Inst* __restrict__ insts, int k0, int n, const double* __restrict__ X,
                               const DevScalars* __restrict__ sc, const double* __restrict__ dtbar,
                               const unsigned long long* __restrict__ argmin, double* __restrict__ U0,
                               double* __restrict__ pbar) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int k = k0 + q;
    const Inst& I = insts[k];
    const DevScalars& S = sc[k];
    if (!(S.dt == S.cfl_factor * S.dt_cfl) || dtbar[k] == 0.0) return;
    const unsigned long long l = argmin[k];
    if (l >= (unsigned long long)I.nx * I.ny) return;
    const long long nd = node_of(I, (int)(l / I.ny), (int)(l % I.ny));
    const double* x = X + I.aoff;
    D8 s8[6];
    for (int c = 0; c < 6; ++c) s8[c] = D8::var(x[c * I.plane + nd], c);
    const D8 d = local_dt_t<D8>(s8, I.dx, I.dy, I.P, D8::var(I.P.omega_ei, 6), D8::var(I.P.omega_er, 7));
    const double g = S.cfl_factor * dtbar[k];
    for (int c = 0; c < 6; ++c) U0[I.aoff + c * I.plane + nd] += g * d.d[c];
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
void launch_adj_dt(cudaStream_t s, const Inst* insts, int k0, int n, long long max_cells, const double* X,
                   const DevScalars* sc, const double* dtbar, unsigned long long* argmin, double* U0, double* pbar) {
    if (n <= 0) return;
    cudaMemsetAsync(argmin + k0, 0xff, (size_t)n * sizeof(unsigned long long), s);
    k_adj_dt_find<<<dim3((unsigned)((max_cells + 255) / 256), n), 256, 0, s>>>(insts, k0, X, sc, dtbar, argmin);
    k_adj_dt_apply<<<(n + 63) / 64, 64, 0, s>>>(insts, k0, n, X, sc, dtbar, argmin, U0, pbar);
}

} // namespace rh3t
