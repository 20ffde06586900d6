// Device-side pointwise physics of the 3T_RH operator, FP64.
//
// Each function restates the reference expression with the same association
// order (colinhu123/3T_RH src/state.rs, weno.rs, noncon.rs, diffusion.rs,
// source.rs, dt.rs); the only arithmetic freedom taken is the compiler's
// mul+add -> FMA contraction (disabled in the RH3T_EXACT build).
#pragma once
#include "rh3t_dev.h"
#include "divrn.cuh"

namespace rh3t {

template <class T> __device__ __forceinline__ T sqd(T x) { return x * x; }
__device__ __forceinline__ double pow4d(double x) { return (x * x) * (x * x); }

// ---- correctly rounded powers for the two pow() calls of the reference
// (state.rs:261 powf(0.25), bc1.rs:241 powf(WENO_Q)). Double-double
// arithmetic (Dekker 1971: exact product by FMA, normalised sums) carries
// ~104 significant bits, so rounding the double-double result gives the
// correctly rounded power except within ~1e-31 of a rounding midpoint.
// Explicit __fma_rn / __dmul_rn / __dadd_rn keep the sequence identical in
// the FMA and the no-contraction builds.
struct DD {
    double hi, lo;
};
__device__ __forceinline__ DD dd_sq(double a) {
    double p = __dmul_rn(a, a);
    return {p, __fma_rn(a, a, -p)};
}
__device__ __forceinline__ DD dd_mul(DD a, DD b) {
    double p = __dmul_rn(a.hi, b.hi);
    double e = __fma_rn(a.hi, b.hi, -p);
    e = __fma_rn(a.hi, b.lo, e);
    e = __fma_rn(a.lo, b.hi, e);
    double s = __dadd_rn(p, e);
    return {s, __dsub_rn(e, __dsub_rn(s, p))};
}
// x^n for an integer n >= 1 by binary powering in double-double
__device__ __forceinline__ double cr_powi(double x, int n) {
    if (!isfinite(x) || x == 0.0) return pow(x, (double)n);
    DD r = {1.0, 0.0}, a = {x, 0.0};
    bool first = true;
    while (n > 0) {
        if (n & 1) { r = first ? a : dd_mul(r, a); first = false; }
        n >>= 1;
        if (n) a = (a.lo == 0.0) ? dd_sq(a.hi) : dd_mul(a, a);
    }
    if (!isfinite(r.hi)) return r.hi;
    return __dadd_rn(r.hi, r.lo);
}
// x^(1/4): sqrt(sqrt(x)) is within one ulp; of it and its two neighbours pick
// the one whose fourth power (double-double) is nearest to x.
__device__ __forceinline__ double cr_pow_quarter(double x) {
    double y = sqrt(sqrt(x));
    if (!(x > 0.0) || !isfinite(y) || !isfinite(x)) return y;
    const long long yb = __double_as_longlong(y); // y > 0 and finite here: neighbours by bit pattern
    double cand[3] = {__longlong_as_double(yb - 1), y, __longlong_as_double(yb + 1)};
    double best = y, bd = INFINITY;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        DD c2 = dd_sq(cand[k]);
        DD c4 = dd_mul(c2, c2);
        double d = fabs(__dadd_rn(__dsub_rn(c4.hi, x), c4.lo));
        if (d < bd || (d == bd && k == 1)) { bd = d; best = cand[k]; }
    }
    return best;
}
// powf(q) of the boundary WENO weights: integer q in double-double, else libdevice pow
__device__ __forceinline__ double pow_q(double x, double q) {
    if (q == 10.0) return cr_powi(x, 10);
    if (q >= 1.0 && q <= 64.0 && q == floor(q)) return cr_powi(x, (int)q);
    return pow(x, q);
}

// x / 3 and x / 6 written once for every scalar type: the IEEE quotient by
// divrn.cuh for double, the type's own division otherwise (dual numbers)
__device__ __forceinline__ double quot3(double x) { return div3_rn(x); }
__device__ __forceinline__ double quot6(double x) { return div6_rn(x); }
template <class T> __device__ __forceinline__ T quot3(const T& x) { return x / 3.0; }
template <class T> __device__ __forceinline__ T quot6(const T& x) { return x / 6.0; }

// Subset of state.rs:245-276 Derived::from_state needed by fluxes, L/R and noncon.
struct Prim {
    double u, v, e_e, e_i, e_r, pe, pi, pr;
};

// Every quotient is the IEEE one (divrn.cuh): the five by rho share one
// reciprocal, w2 / 6 and rho w2 / 6 are each formed once.
__device__ __forceinline__ Prim prim_from_state(const double s[6], const DevParams& P) {
    Prim d;
    const Recip r0 = recip(s[0]);
    d.u = div_rn(s[1], r0);
    d.v = div_rn(s[2], r0);
    double w2 = sqd(d.u) + sqd(d.v);
    const double w6 = div6_rn(w2), rw6 = div6_rn(s[0] * w2);
    d.e_e = div_rn(s[3], r0) - w6;
    d.e_i = div_rn(s[4], r0) - w6;
    d.e_r = div_rn(s[5], r0) - w6;
    d.pe = (P.gamma_e - 1.0) * (s[3] - rw6);
    d.pi = (P.gamma_i - 1.0) * (s[4] - rw6);
    d.pr = (P.gamma_r - 1.0) * (s[5] - rw6);
    return d;
}

// state.rs:245-276 te, ti, tr (diffusion and source only). r6e, r6i, ra:
// the instance's divisors 6 cve, 6 cvi and a_rad with their reciprocals
// (every quotient stays the IEEE one, divrn.cuh)
__device__ __forceinline__ void temps_from_state(const double s[6], const DevParams& P, const Recip& r6e,
                                                 const Recip& r6i, const Recip& ra, double& te, double& ti,
                                                 double& tr) {
    const Recip r0 = recip(s[0]);
    double u = div_rn(s[1], r0), v = div_rn(s[2], r0);
    double w2 = sqd(u) + sqd(v);
    te = s[3] / (s[0] * P.cve) - div_rn(w2, r6e);
    ti = s[4] / (s[0] * P.cvi) - div_rn(w2, r6i);
    double er_term = div_rn(s[5], r0) - div6_rn(w2);
    tr = cr_pow_quarter(div_rn(er_term * s[0], ra));
}

// the same values with plain IEEE divisions (callers without the instance's
// reciprocals at hand)
__device__ __forceinline__ void temps_from_state(const double s[6], const DevParams& P, double& te, double& ti,
                                                 double& tr) {
    const Recip r0 = recip(s[0]);
    double u = div_rn(s[1], r0), v = div_rn(s[2], r0);
    double w2 = sqd(u) + sqd(v);
    te = s[3] / (s[0] * P.cve) - w2 / (6.0 * P.cve);
    ti = s[4] / (s[0] * P.cvi) - w2 / (6.0 * P.cvi);
    double er_term = div_rn(s[5], r0) - div6_rn(w2);
    tr = cr_pow_quarter(er_term * s[0] / P.a_rad);
}

// state.rs:56-85 flux_from_derived
template <int DIR>
__device__ __forceinline__ void phys_flux(const double s[6], const Prim& d, double f[6]) {
    double u = d.u, v = d.v;
    double p = d.pe + d.pi + d.pr;
    double rho = s[0];
    if (DIR == 0) {
        f[0] = rho * u; f[1] = rho * u * u + p; f[2] = rho * u * v;
        f[3] = (s[3] + d.pe) * u; f[4] = (s[4] + d.pi) * u; f[5] = (s[5] + d.pr) * u;
    } else {
        f[0] = rho * v; f[1] = rho * u * v; f[2] = rho * v * v + p;
        f[3] = (s[3] + d.pe) * v; f[4] = (s[4] + d.pi) * v; f[5] = (s[5] + d.pr) * v;
    }
}

// Roe (sqrt(rho)-weighted) averages shared by weno.rs:28-78 build_l_plain and
// weno.rs:484-516 build_r_plain (state1 = points[3], state2 = points[2]).
template <class T> struct RoeT {
    T u, v, w2, ee, ei, er, cs2, cs, he, hi, hr, b, den;
};
using Roe = RoeT<double>;

__device__ __forceinline__ Roe roe_average(double rho_s1, const Prim& d3, double rho_s2, const Prim& d2,
                                           const DevParams& P) {
    Roe q;
    double rho1 = sqrt(rho_s1), rho2 = sqrt(rho_s2);
    double rho_sum = rho1 + rho2;
    const Recip rs = recip(rho_sum);
    q.u = div_rn(d3.u * rho1 + d2.u * rho2, rs);
    q.v = div_rn(d3.v * rho1 + d2.v * rho2, rs);
    q.w2 = sqd(q.u) + sqd(q.v);
    q.ee = div_rn(d3.e_e * rho1 + d2.e_e * rho2, rs);
    q.ei = div_rn(d3.e_i * rho1 + d2.e_i * rho2, rs);
    q.er = div_rn(d3.e_r * rho1 + d2.e_r * rho2, rs);
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    q.cs2 = GE * ge * q.ee + GI * gi * q.ei + GR * gr * q.er;
    q.cs = sqrt(q.cs2);
    q.he = 6.0 * gi * gr * (GI * q.ei - GR * q.er) + GE * gt * q.ee * q.w2;
    q.hi = 6.0 * ge * gr * (GR * q.er - GE * q.ee) + GI * gt * q.ei * q.w2;
    q.hr = 6.0 * ge * gi * (GE * q.ee - GI * q.ei) + GR * gt * q.er * q.w2;
    q.b = gt * (36.0 * ge * gi * gr + gt * sqd(q.w2)) * q.cs2;
    q.den = 12.0 * q.cs2;
    return q;
}

// Mode of left eigenvector row `row`: 0 acoustic-, 1 transverse, 2 electron,
// 3 ion, 4 radiation, 5 acoustic+. x faces order their rows
// [u-c, e, i, r, transverse, u+c], y faces [v-c, transverse, e, i, r, v+c].
// (Selects, not a table: a table indexed by a runtime row lives in local memory.)
template <int DIR> __device__ __forceinline__ int row_mode(int row) {
    if (DIR != 0) return row;
    return row == 0 ? 0 : (row == 5 ? 5 : (row == 4 ? 1 : row + 1));
}

// Row `row` of the left eigenvector matrix (weno.rs:79-458). DIR 0: rows
// [u-c, e, i, r, transverse, u+c]; DIR 1: [v-c, transverse, e, i, r, v+c].
// Written over the scalar type T (double; a dual-number type in the adjoint).
template <int DIR, class T>
__device__ __forceinline__ void l_row(int row, const RoeT<T>& q, const DevParams& P, T L[6]) {
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    const T u = q.u, v = q.v, w2 = q.w2, cs = q.cs, cs2 = q.cs2, b = q.b, den = q.den;
    const int mode = row_mode<DIR>(row);
    if (mode == 0 || mode == 5) {
        const double sgn = mode == 0 ? 1.0 : -1.0;
        if (DIR == 0) {
            L[0] = mode == 0 ? (gt * w2 + 6.0 * u * cs) / den : (gt * w2 - 6.0 * u * cs) / den;
            L[1] = mode == 0 ? (-2.0 * gt * u - 6.0 * cs) / den : (-2.0 * gt * u + 6.0 * cs) / den;
            L[2] = (-2.0 * gt * v) / den;
        } else {
            L[0] = mode == 0 ? (gt * w2 + 6.0 * v * cs) / den : (gt * w2 - 6.0 * v * cs) / den;
            L[1] = (-2.0 * gt * u) / den;
            L[2] = mode == 0 ? (-2.0 * gt * v - 6.0 * cs) / den : (-2.0 * gt * v + 6.0 * cs) / den;
        }
        (void)sgn;
        L[3] = 6.0 * ge / den;
        L[4] = 6.0 * gi / den;
        L[5] = 6.0 * gr / den;
    } else if (mode == 1) {
        if (DIR == 0) { L[0] = -v; L[1] = T(0.0); L[2] = T(1.0); }
        else { L[0] = -u; L[1] = T(1.0); L[2] = T(0.0); }
        L[3] = T(0.0); L[4] = T(0.0); L[5] = T(0.0);
    } else if (mode == 2) {
        const T he = q.he;
        L[0] = ge / gt - ge * w2 / (6.0 * cs2) - ge * gt * w2 / b * (he - cs2 * w2);
        L[1] = ge * u / (3.0 * cs2) + 2.0 * ge * gt * u / b * (he - cs2 * w2);
        L[2] = ge * v / (3.0 * cs2) + 2.0 * ge * gt * v / b * (he - cs2 * w2);
        L[3] = -sqd(ge) / (gt * cs2) - 6.0 * ge / b * (ge * he - gt * cs2 * w2);
        L[4] = -ge * gi / (gt * cs2) - 6.0 * ge * gi / b * (he - 6.0 * gr * cs2);
        L[5] = -ge * gr / (gt * cs2) - 6.0 * ge * gr / b * (he + 6.0 * gi * cs2);
    } else if (mode == 3) {
        const T hi = q.hi;
        L[0] = gi / gt - gi * w2 / (6.0 * cs2) - gi * gt * w2 / b * (hi - cs2 * w2);
        L[1] = gi * u / (3.0 * cs2) + 2.0 * gi * gt * u / b * (hi - cs2 * w2);
        L[2] = gi * v / (3.0 * cs2) + 2.0 * gi * gt * v / b * (hi - cs2 * w2);
        L[3] = -gi * ge / (gt * cs2) - 6.0 * gi * ge / b * (hi + 6.0 * gr * cs2);
        L[4] = -sqd(gi) / (gt * cs2) - 6.0 * gi / b * (gi * hi - gt * cs2 * w2);
        L[5] = -gi * gr / (gt * cs2) - 6.0 * gi * gr / b * (hi - 6.0 * ge * cs2);
    } else {
        const T hr = q.hr;
        L[0] = gr / gt - gr * w2 / (6.0 * cs2) - gr * gt * w2 / b * (hr - cs2 * w2);
        L[1] = gr * u / (3.0 * cs2) + 2.0 * gr * gt * u / b * (hr - cs2 * w2);
        L[2] = gr * v / (3.0 * cs2) + 2.0 * gr * gt * v / b * (hr - cs2 * w2);
        L[3] = -gr * ge / (gt * cs2) - 6.0 * gr * ge / b * (hr - 6.0 * gi * cs2);
        L[4] = -gr * gi / (gt * cs2) - 6.0 * gr * gi / b * (hr + 6.0 * ge * cs2);
        L[5] = -sqd(gr) / (gt * cs2) - 6.0 * gr / b * (gr * hr - gt * cs2 * w2);
    }
}

// Column `col` of the right eigenvector matrix and eigenvalue (weno.rs:518-545).
template <int DIR, class T>
__device__ __forceinline__ void r_col(int col, const RoeT<T>& q, const DevParams& P, T R[6], T& lam) {
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    const T u = q.u, v = q.v, w2 = q.w2, cs = q.cs;
    if (DIR == 0) {
        switch (col) {
        case 0:
            R[0] = 1.0; R[1] = u - cs; R[2] = v;
            R[3] = GE * q.ee + quot6(w2) - quot3(u * cs);
            R[4] = GI * q.ei + quot6(w2) - quot3(u * cs);
            R[5] = GR * q.er + quot6(w2) - quot3(u * cs);
            lam = u - cs; break;
        case 1: R[0] = 1.0; R[1] = u; R[2] = v; R[3] = gt * w2 / (6.0 * ge); R[4] = gr; R[5] = -gi; lam = u; break;
        case 2: R[0] = 1.0; R[1] = u; R[2] = v; R[3] = -gr; R[4] = gt * w2 / (6.0 * gi); R[5] = ge; lam = u; break;
        case 3: R[0] = 1.0; R[1] = u; R[2] = v; R[3] = gi; R[4] = -ge; R[5] = gt * w2 / (6.0 * gr); lam = u; break;
        case 4: R[0] = 0.0; R[1] = 0.0; R[2] = 1.0; R[3] = quot3(v); R[4] = quot3(v); R[5] = quot3(v); lam = u; break;
        default:
            R[0] = 1.0; R[1] = u + cs; R[2] = v;
            R[3] = GE * q.ee + quot6(w2) + quot3(u * cs);
            R[4] = GI * q.ei + quot6(w2) + quot3(u * cs);
            R[5] = GR * q.er + quot6(w2) + quot3(u * cs);
            lam = u + cs; break;
        }
    } else {
        switch (col) {
        case 0:
            R[0] = 1.0; R[1] = u; R[2] = v - cs;
            R[3] = GE * q.ee + quot6(w2) - quot3(v * cs);
            R[4] = GI * q.ei + quot6(w2) - quot3(v * cs);
            R[5] = GR * q.er + quot6(w2) - quot3(v * cs);
            lam = v - cs; break;
        case 1: R[0] = 0.0; R[1] = 1.0; R[2] = 0.0; R[3] = quot3(u); R[4] = quot3(u); R[5] = quot3(u); lam = v; break;
        case 2: R[0] = 1.0; R[1] = u; R[2] = v; R[3] = gt * w2 / (6.0 * ge); R[4] = gr; R[5] = -gi; lam = v; break;
        case 3: R[0] = 1.0; R[1] = u; R[2] = v; R[3] = -gr; R[4] = gt * w2 / (6.0 * gi); R[5] = ge; lam = v; break;
        case 4: R[0] = 1.0; R[1] = u; R[2] = v; R[3] = gi; R[4] = -ge; R[5] = gt * w2 / (6.0 * gr); lam = v; break;
        default:
            R[0] = 1.0; R[1] = u; R[2] = v + cs;
            R[3] = GE * q.ee + quot6(w2) + quot3(v * cs);
            R[4] = GI * q.ei + quot6(w2) + quot3(v * cs);
            R[5] = GR * q.er + quot6(w2) + quot3(v * cs);
            lam = v + cs; break;
        }
    }
}

// Row `row` of the right eigenvector matrix (weno.rs:518-545) and the
// eigenvalue of characteristic field `row`.
template <int DIR>
__device__ __forceinline__ void r_row(int row, const Roe& q, const DevParams& P, double R[6], double& lam) {
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    const double u = q.u, v = q.v, w2 = q.w2, cs = q.cs;
    const double vel = DIR == 0 ? u : v;
    lam = row == 0 ? vel - cs : (row == 5 ? vel + cs : vel);
    if (row >= 3) {
        // energy components k = 0, 1, 2 (e, i, r): one code path with the
        // component's operands. Entries 0 and 5: Gk ek + w2/6 -+ vel cs / 3;
        // the three others (x faces 1..3, y faces 2..4) hold gt w2 / (6 gk)
        // at position k and +-gl (l the third index, + for position
        // (k + 2) mod 3) elsewhere; the remaining entry is v / 3 (x faces,
        // position 4) or u / 3 (y faces, position 1)
        const int k = row - 3;
        const double Gk = k == 0 ? GE : (k == 1 ? GI : GR);
        const double ek = k == 0 ? q.ee : (k == 1 ? q.ei : q.er);
        const double gk = k == 0 ? ge : (k == 1 ? gi : gr);
        const double base = Gk * ek + div6_rn(w2);
        const double vc = div3_rn(vel * cs);
        R[0] = base - vc;
        R[5] = base + vc;
        const double dk = gt * w2 / (6.0 * gk);
        const int o = DIR == 0 ? 1 : 2;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const int l = 3 - k - m;
            const double gl = l == 0 ? ge : (l == 1 ? gi : gr);
            R[o + m] = m == k ? dk : (m == (k + 2) % 3 ? gl : -gl);
        }
        R[DIR == 0 ? 4 : 1] = div3_rn(DIR == 0 ? v : u);
    } else if (DIR == 0) {
        switch (row) {
        case 0: R[0] = 1.0; R[1] = 1.0; R[2] = 1.0; R[3] = 1.0; R[4] = 0.0; R[5] = 1.0; break;
        case 1: R[0] = u - cs; R[1] = u; R[2] = u; R[3] = u; R[4] = 0.0; R[5] = u + cs; break;
        default: R[0] = v; R[1] = v; R[2] = v; R[3] = v; R[4] = 1.0; R[5] = v; break;
        }
    } else {
        switch (row) {
        case 0: R[0] = 1.0; R[1] = 0.0; R[2] = 1.0; R[3] = 1.0; R[4] = 1.0; R[5] = 1.0; break;
        case 1: R[0] = u; R[1] = 1.0; R[2] = u; R[3] = u; R[4] = u; R[5] = u; break;
        default: R[0] = v - cs; R[1] = 0.0; R[2] = v; R[3] = v; R[4] = v; R[5] = v + cs; break;
        }
    }
}

// The divisors of one face's left eigenvector rows (weno.rs:79-458):
// 12 cs2, b, 6 cs2, 3 cs2, gt cs2 and gt, each with its reciprocal, formed
// once per face and shared by the rows (divrn.cuh: every quotient is still
// the IEEE one).
struct RoeDiv {
    Recip den, b, c6, c3, cg, gt;
};
__device__ __forceinline__ RoeDiv roe_div(const Roe& q, const DevParams& P) {
    const double gt = (P.gamma_i - 1.0) + (P.gamma_e - 1.0) + (P.gamma_r - 1.0);
    RoeDiv r;
    r.den = recip(q.den);
    r.b = recip(q.b);
    // den = RN(12 cs2) is exactly 2 RN(6 cs2) and 4 RN(3 cs2) (scaling by a
    // power of two commutes with rounding), so while den is in the fast range
    // (no overflow or underflow) RN(1 / (6 cs2)) = 2 RN(1 / den) and
    // RN(1 / (3 cs2)) = 4 RN(1 / den) exactly: two IEEE divisions fewer
    if (r.den.ok) {
        const double c6 = 6.0 * q.cs2, c3 = 3.0 * q.cs2;
        r.c6 = {c6, 2.0 * r.den.y, div_in_range(c6)};
        r.c3 = {c3, 4.0 * r.den.y, div_in_range(c3)};
    } else {
        r.c6 = recip(6.0 * q.cs2);
        r.c3 = recip(3.0 * q.cs2);
    }
    r.cg = recip(gt * q.cs2);
    r.gt = recip(gt);
    return r;
}

// l_row over double with the face's shared divisors: the same expressions
// as l_row<DIR, T> (weno.rs:79-458), the same roundings.
template <int DIR>
__device__ __forceinline__ void l_row(int row, const Roe& q, const RoeDiv& rd, const DevParams& P, double L[6]) {
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    const double u = q.u, v = q.v, w2 = q.w2, cs = q.cs, cs2 = q.cs2;
    const int mode = row_mode<DIR>(row);
    if (mode == 0 || mode == 5) {
        // the two acoustic rows differ only in the sign of one term of two
        // entries: x + s y with s = +-1 is x + y or x - y exactly
        const double s = mode == 0 ? 1.0 : -1.0;
        if (DIR == 0) {
            L[0] = div_rn(gt * w2 + s * (6.0 * u * cs), rd.den);
            L[1] = div_rn(-2.0 * gt * u + -s * (6.0 * cs), rd.den);
            L[2] = div_rn(-2.0 * gt * v, rd.den);
        } else {
            L[0] = div_rn(gt * w2 + s * (6.0 * v * cs), rd.den);
            L[1] = div_rn(-2.0 * gt * u, rd.den);
            L[2] = div_rn(-2.0 * gt * v + -s * (6.0 * cs), rd.den);
        }
        L[3] = div_rn(6.0 * ge, rd.den);
        L[4] = div_rn(6.0 * gi, rd.den);
        L[5] = div_rn(6.0 * gr, rd.den);
    } else if (mode == 1) {
        if (DIR == 0) { L[0] = -v; L[1] = 0.0; L[2] = 1.0; }
        else { L[0] = -u; L[1] = 1.0; L[2] = 0.0; }
        L[3] = 0.0; L[4] = 0.0; L[5] = 0.0;
    } else {
        // energy rows: k = 0, 1, 2 for e, i, r (modes 2, 3, 4), one code path
        // with the mode's operands. Entry 3 + j: on the diagonal (j == k)
        // -gk^2 / (gt cs2) - 6 gk / b (gk hk - gt cs2 w2); off it, with l the
        // third index, -gk gj / (gt cs2) - 6 gk gj / b (hk +- 6 gl cs2), the
        // sign + for j == (k + 2) mod 3: the reference's rows written per
        // mode, the same products in the same order
        const int k = mode - 2;
        const double gk = k == 0 ? ge : (k == 1 ? gi : gr);
        const double hk = k == 0 ? q.he : (k == 1 ? q.hi : q.hr);
        L[0] = div_rn(gk, rd.gt) - div_rn(gk * w2, rd.c6) - div_rn(gk * gt * w2, rd.b) * (hk - cs2 * w2);
        L[1] = div_rn(gk * u, rd.c3) + div_rn(2.0 * gk * gt * u, rd.b) * (hk - cs2 * w2);
        L[2] = div_rn(gk * v, rd.c3) + div_rn(2.0 * gk * gt * v, rd.b) * (hk - cs2 * w2);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const bool diag = j == k;
            const int l = 3 - k - j;
            const double gj = j == 0 ? ge : (j == 1 ? gi : gr);
            const double gl = l == 0 ? ge : (l == 1 ? gi : gr);
            const double t = 6.0 * gl * cs2;
            const double n2 = diag ? 6.0 * gk : 6.0 * gk * gj;
            const double f = diag ? gk * hk - gt * cs2 * w2 : hk + (j == (k + 2) % 3 ? t : -t);
            L[3 + j] = div_rn(-gk * gj, rd.cg) - div_rn(n2, rd.b) * f;
        }
    }
}

// ---------------------------------------------------------------- fast forms
// Same mathematics, fewer divisions (shared reciprocals, a single division per
// WENO5 reconstruction); used by the FMA build only. Rounding differs from the
// reference by a few ulps per operation, like FMA contraction does.
namespace fastm {

__device__ __forceinline__ Prim prim(const double s[6], const DevParams& P) {
    Prim d;
    const double ir = 1.0 / s[0];
    d.u = s[1] * ir;
    d.v = s[2] * ir;
    const double w2 = d.u * d.u + d.v * d.v;
    const double k = w2 * (1.0 / 6.0);
    d.e_e = s[3] * ir - k;
    d.e_i = s[4] * ir - k;
    d.e_r = s[5] * ir - k;
    const double rk = s[0] * k;
    d.pe = (P.gamma_e - 1.0) * (s[3] - rk);
    d.pi = (P.gamma_i - 1.0) * (s[4] - rk);
    d.pr = (P.gamma_r - 1.0) * (s[5] - rk);
    return d;
}

// Roe average from (sqrt(rho), u, v, e_e, e_i, e_r) of points[3] (a) and points[2] (b)
__device__ __forceinline__ Roe roe(const double a[6], const double b[6], const DevParams& P) {
    Roe q;
    const double inv = 1.0 / (a[0] + b[0]);
    q.u = (a[1] * a[0] + b[1] * b[0]) * inv;
    q.v = (a[2] * a[0] + b[2] * b[0]) * inv;
    q.w2 = q.u * q.u + q.v * q.v;
    q.ee = (a[3] * a[0] + b[3] * b[0]) * inv;
    q.ei = (a[4] * a[0] + b[4] * b[0]) * inv;
    q.er = (a[5] * a[0] + b[5] * b[0]) * inv;
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    q.cs2 = GE * ge * q.ee + GI * gi * q.ei + GR * gr * q.er;
    q.cs = sqrt(q.cs2);
    q.he = 6.0 * gi * gr * (GI * q.ei - GR * q.er) + GE * gt * q.ee * q.w2;
    q.hi = 6.0 * ge * gr * (GR * q.er - GE * q.ee) + GI * gt * q.ei * q.w2;
    q.hr = 6.0 * ge * gi * (GE * q.ee - GI * q.ei) + GR * gt * q.er * q.w2;
    q.b = gt * (36.0 * ge * gi * gr + gt * q.w2 * q.w2) * q.cs2;
    q.den = 12.0 * q.cs2;
    return q;
}

// ics2 = 1 / cs2 and ib = 1 / b of the face (formed once per face)
template <int DIR>
__device__ __forceinline__ void l_row(int row, const Roe& q, double ics2, double ib, const DevParams& P,
                                      double L[6]) {
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    const double u = q.u, v = q.v, w2 = q.w2, cs = q.cs, cs2 = q.cs2;
    const double iden = ics2 * (1.0 / 12.0);
    const int mode = row_mode<DIR>(row);
    if (mode == 0 || mode == 5) {
        const double sg = mode == 0 ? 6.0 : -6.0;
        const double vn = DIR == 0 ? u : v;
        L[0] = (gt * w2 + sg * vn * cs) * iden;
        if (DIR == 0) {
            L[1] = (-2.0 * gt * u - sg * cs) * iden;
            L[2] = (-2.0 * gt * v) * iden;
        } else {
            L[1] = (-2.0 * gt * u) * iden;
            L[2] = (-2.0 * gt * v - sg * cs) * iden;
        }
        L[3] = 6.0 * ge * iden;
        L[4] = 6.0 * gi * iden;
        L[5] = 6.0 * gr * iden;
    } else if (mode == 1) {
        if (DIR == 0) { L[0] = -v; L[1] = 0.0; L[2] = 1.0; }
        else { L[0] = -u; L[1] = 1.0; L[2] = 0.0; }
        L[3] = 0.0; L[4] = 0.0; L[5] = 0.0;
    } else {
        // electron / ion / radiation: gk = (ge, gi, gr)[k], hk = (he, hi, hr)[k]
        const double gk = mode == 2 ? ge : (mode == 3 ? gi : gr);
        const double hk = mode == 2 ? q.he : (mode == 3 ? q.hi : q.hr);
        const double t = (hk - cs2 * w2) * ib;
        L[0] = gk / gt - gk * w2 * (ics2 * (1.0 / 6.0)) - gk * gt * w2 * t;
        L[1] = gk * u * (ics2 * (1.0 / 3.0)) + 2.0 * gk * gt * u * t;
        L[2] = gk * v * (ics2 * (1.0 / 3.0)) + 2.0 * gk * gt * v * t;
        const double igc = ics2 / gt;
        const double c6 = 6.0 * gk * ib;
        if (mode == 2) {
            L[3] = -ge * ge * igc - c6 * (ge * hk - gt * cs2 * w2);
            L[4] = -ge * gi * igc - c6 * gi * (hk - 6.0 * gr * cs2);
            L[5] = -ge * gr * igc - c6 * gr * (hk + 6.0 * gi * cs2);
        } else if (mode == 3) {
            L[3] = -gi * ge * igc - c6 * ge * (hk + 6.0 * gr * cs2);
            L[4] = -gi * gi * igc - c6 * (gi * hk - gt * cs2 * w2);
            L[5] = -gi * gr * igc - c6 * gr * (hk - 6.0 * ge * cs2);
        } else {
            L[3] = -gr * ge * igc - c6 * ge * (hk - 6.0 * gi * cs2);
            L[4] = -gr * gi * igc - c6 * gi * (hk + 6.0 * ge * cs2);
            L[5] = -gr * gr * igc - c6 * (gr * hk - gt * cs2 * w2);
        }
    }
}

// WENO5 with one division: alpha_k = d_k / s_k^2 scaled by s0^2 s1^2 s2^2
__device__ __forceinline__ double weno5(double u0, double u1, double u2, double u3, double u4, double eps) {
    const double c1312 = 13.0 / 12.0;
    double t2 = u2 - 2.0 * u3 + u4, r2 = 3.0 * u2 - 4.0 * u3 + u4;
    double t1 = u1 - 2.0 * u2 + u3, r1 = u1 - u3;
    double t0 = u0 - 2.0 * u1 + u2, r0 = u0 - 4.0 * u1 + 3.0 * u2;
    double s0 = eps + (c1312 * t0 * t0 + 0.25 * r0 * r0);
    double s1 = eps + (c1312 * t1 * t1 + 0.25 * r1 * r1);
    double s2 = eps + (c1312 * t2 * t2 + 0.25 * r2 * r2);
    s0 *= s0; s1 *= s1; s2 *= s2;
    double a0 = 0.1 * (s1 * s2), a1 = 0.6 * (s0 * s2), a2 = 0.3 * (s0 * s1);
    double p0 = u0 * (1.0 / 3.0) - u1 * (7.0 / 6.0) + u2 * (11.0 / 6.0);
    double p1 = -u1 * (1.0 / 6.0) + u2 * (5.0 / 6.0) + u3 * (1.0 / 3.0);
    double p2 = u2 * (1.0 / 3.0) + u3 * (5.0 / 6.0) - u4 * (1.0 / 6.0);
    return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2);
}

} // namespace fastm

// weno.rs:847-886 weno5 (WENO-JS, p = 2)
__device__ __forceinline__ double weno5(double u0, double u1, double u2, double u3, double u4, double eps) {
    double beta2 = 13.0 / 12.0 * sqd(u2 - 2.0 * u3 + u4) + 0.25 * sqd(3.0 * u2 - 4.0 * u3 + u4);
    double beta1 = 13.0 / 12.0 * sqd(u1 - 2.0 * u2 + u3) + 0.25 * sqd(u1 - u3);
    double beta0 = 13.0 / 12.0 * sqd(u0 - 2.0 * u1 + u2) + 0.25 * sqd(u0 - 4.0 * u1 + 3.0 * u2);
    double a0 = 0.1 / sqd(eps + beta0);
    double a1 = 0.6 / sqd(eps + beta1);
    double a2 = 0.3 / sqd(eps + beta2);
    double sum_o = a0 + a1 + a2;
    const Recip rs = recip(sum_o); // the three weights share their divisor (IEEE quotients, divrn.cuh)
    double w0 = div_rn(a0, rs), w1 = div_rn(a1, rs), w2 = div_rn(a2, rs);
    double p0 = div3_rn(u0) - 7.0 / 6.0 * u1 + 11.0 / 6.0 * u2;
    double p1 = div6_rn(-u1) + 5.0 / 6.0 * u2 + div3_rn(u3);
    double p2 = div3_rn(u2) + 5.0 / 6.0 * u3 - div6_rn(u4);
    return w0 * p0 + w1 * p1 + w2 * p2;
}

// noncon.rs:49-57
__device__ __forceinline__ double q_pulse7(double b0, double b1, double b2, double b3, double b4, double b5,
                                           double b6) {
    return -0.00714285714285723 * b0 + 0.0595238095238118 * b1 - 0.240476190476197 * b2 +
           0.759523809523819 * b3 + 0.509523809523803 * b4 - 0.0904761904761891 * b5 +
           0.00952380952380977 * b6;
}

// noncon.rs:259-285 one component of n_jump_pre on an 8-point window a[0..7]
__device__ __forceinline__ double jump8(const double* a) {
    return q_pulse7(a[7], a[6], a[5], a[4], a[3], a[2], a[1]) - q_pulse7(a[0], a[1], a[2], a[3], a[4], a[5], a[6]);
}

// noncon.rs:26-44
__device__ __forceinline__ double d6(double qm3, double qm2, double qm1, double qp1, double qp2, double qp3,
                                     double dx) {
    return (qp3 - 9.0 * qp2 + 45.0 * qp1 - 45.0 * qm1 + 9.0 * qm2 - qm3) / (60.0 * dx);
}

// noncon.rs:288-332 nonconservative_direction_pre on a 9-point window
// (pe, pi, pr, transport velocity vel per point, index 4 = cell).
__device__ __forceinline__ void noncon9(const double pe[9], const double pi[9], const double pr[9],
                                        const double vel[9], double ds, double out[3]) {
    double v = vel[4];
    double dpe = d6(pe[1], pe[2], pe[3], pe[5], pe[6], pe[7], ds);
    double dpi = d6(pi[1], pi[2], pi[3], pi[5], pi[6], pi[7], ds);
    double dpr = d6(pr[1], pr[2], pr[3], pr[5], pr[6], pr[7], ds);
    double der_ee = 2.0 * dpe - dpi - dpr;
    double der_ei = 2.0 * dpi - dpe - dpr;
    double der_er = 2.0 * dpr - dpe - dpi;
    double nee[9], nei[9], ner[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        nee[k] = 2.0 * pe[k] - pi[k] - pr[k];
        nei[k] = 2.0 * pi[k] - pe[k] - pr[k];
        ner[k] = 2.0 * pr[k] - pe[k] - pi[k];
    }
    double jm_ee = jump8(nee), jm_ei = jump8(nei), jm_er = jump8(ner);
    double jp_ee = jump8(nee + 1), jp_ei = jump8(nei + 1), jp_er = jump8(ner + 1);
    double coef_left = fmax(fmax(v, vel[3]), 0.0) / 3.0;
    double coef_right = fmin(fmin(v, vel[5]), 0.0) / 3.0;
    out[0] = v / 3.0 * der_ee + (coef_left * jm_ee + coef_right * jp_ee) / ds;
    out[1] = v / 3.0 * der_ei + (coef_left * jm_ei + coef_right * jp_ei) / ds;
    out[2] = v / 3.0 * der_er + (coef_left * jm_er + coef_right * jp_er) / ds;
}

// noncon9 with the divisors 60 ds and ds given with their reciprocals (the
// same quotients, divrn.cuh), for callers that hold them for many cells
__device__ __forceinline__ void noncon9(const double pe[9], const double pi[9], const double pr[9],
                                        const double vel[9], const Recip& r60ds, const Recip& rds, double out[3]) {
    double v = vel[4];
    auto d6r = [&](const double* q) {
        return div_rn(q[7] - 9.0 * q[6] + 45.0 * q[5] - 45.0 * q[3] + 9.0 * q[2] - q[1], r60ds);
    };
    double dpe = d6r(pe), dpi = d6r(pi), dpr = d6r(pr);
    double der_ee = 2.0 * dpe - dpi - dpr;
    double der_ei = 2.0 * dpi - dpe - dpr;
    double der_er = 2.0 * dpr - dpe - dpi;
    double nee[9], nei[9], ner[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        nee[k] = 2.0 * pe[k] - pi[k] - pr[k];
        nei[k] = 2.0 * pi[k] - pe[k] - pr[k];
        ner[k] = 2.0 * pr[k] - pe[k] - pi[k];
    }
    double jm_ee = jump8(nee), jm_ei = jump8(nei), jm_er = jump8(ner);
    double jp_ee = jump8(nee + 1), jp_ei = jump8(nei + 1), jp_er = jump8(ner + 1);
    double coef_left = div3_rn(fmax(fmax(v, vel[3]), 0.0));
    double coef_right = div3_rn(fmin(fmin(v, vel[5]), 0.0));
    const double v3 = div3_rn(v);
    out[0] = v3 * der_ee + div_rn(coef_left * jm_ee + coef_right * jp_ee, rds);
    out[1] = v3 * der_ei + div_rn(coef_left * jm_ei + coef_right * jp_ei, rds);
    out[2] = v3 * der_er + div_rn(coef_left * jm_er + coef_right * jp_er, rds);
}

// dt.rs:5-34 get_local_dt (same association order; CVE^3 = CVE*(CVE*CVE)),
// over the scalar type T with the exchange coefficients as arguments (the
// adjoint differentiates it in the state and in them)
template <class T>
__device__ __forceinline__ T local_dt_t(const T s[6], double dx, double dy, const DevParams& P, T OEI, T OER) {
    T u = s[1] / s[0], v = s[2] / s[0];
    T ee = s[3] / s[0] - (sqd(u) + sqd(v)) / 6.0;
    T ei = s[4] / s[0] - (sqd(u) + sqd(v)) / 6.0;
    T er = s[5] / s[0] - (sqd(u) + sqd(v)) / 6.0;
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r, A = P.a_rad, CVE = P.cve, CVI = P.cvi;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    T cs = sqrt(GE * ge * ee + GI * gi * ei + GR * gr * er);
    const double c4 = (CVE * CVE) * (CVE * CVE), c3 = CVE * (CVE * CVE);
    T ee3 = ee * (ee * ee);
    T t1 = A * OEI * c4 + A * OEI * c3 * CVI + 4.0 * A * OER * CVI * ee3 + OER * c4 * CVI * s[0];
    T s1 = sqrt(sqd(t1) - 4.0 * A * OEI * OER * c4 * CVI * (4.0 * A * ee3 + c4 * s[0] + c3 * CVI * s[0]));
    T s2 = -(A * OEI * c4 + A * OEI * c3 * CVI + 4.0 * A * OER * CVI * ee3 + OER * c4 * CVI * s[0]);
    T sden = 2.0 * A * c4 * CVI * s[0];
    T alpha1 = fabs((-s1 + s2) / sden);
    T alpha2 = fabs((s1 + s2) / sden);
    T sj = fmax(alpha1, alpha2);
    T dj = fmax(fmax(P.kappa_e / (CVE * s[0]), P.kappa_i / (CVI * s[0])), T(P.kappa_r / A));
    T vj = (fabs(u) + cs) / dx + 2.0 * dj / (sqd(dx) + sqd(dy)) + sj + (fabs(v) + cs) / dy;
    return P.lambda / vj;
}

__device__ __forceinline__ double local_dt(const double s[6], double dx, double dy, const DevParams& P) {
    return local_dt_t<double>(s, dx, dy, P, P.omega_ei, P.omega_er);
}

namespace fastm {

// noncon.rs:288-332 with the divisions by 60 ds, 3 and ds as multiplications
__device__ __forceinline__ void noncon9(const double pe[9], const double pi[9], const double pr[9],
                                        const double vel[9], double inv_60ds, double inv_ds, double out[3]) {
    const double v = vel[4];
    auto d6f = [&](const double* q) {
        return (q[7] - 9.0 * q[6] + 45.0 * q[5] - 45.0 * q[3] + 9.0 * q[2] - q[1]) * inv_60ds;
    };
    const double dpe = d6f(pe), dpi = d6f(pi), dpr = d6f(pr);
    const double der[3] = {2.0 * dpe - dpi - dpr, 2.0 * dpi - dpe - dpr, 2.0 * dpr - dpe - dpi};
    double n[3][9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        n[0][k] = 2.0 * pe[k] - pi[k] - pr[k];
        n[1][k] = 2.0 * pi[k] - pe[k] - pr[k];
        n[2][k] = 2.0 * pr[k] - pe[k] - pi[k];
    }
    const double cl = fmax(fmax(v, vel[3]), 0.0) * (1.0 / 3.0) * inv_ds;
    const double cr = fmin(fmin(v, vel[5]), 0.0) * (1.0 / 3.0) * inv_ds;
    const double v3 = v * (1.0 / 3.0);
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = v3 * der[c] + (cl * jump8(n[c]) + cr * jump8(n[c] + 1));
}

} // namespace fastm

} // namespace rh3t
