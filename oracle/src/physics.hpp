// ORACLE — test infrastructure only. CPU restatement of the 3T_RH pointwise
// physics and interface operators, used as the parity reference for the CUDA
// path and as the timed CPU baseline. Product code never links this.
//
// Every function follows the reference Rust source operation for operation
// (same association order, no FMA contraction: build with -ffp-contract=off).
// Rust `x.powi(n)` is restated by `powi()` below (the binary-decomposition
// multiply sequence LLVM emits for powi), Rust `powf` by std::pow (libm).
#pragma once
#include <cmath>
#include <cstdint>

namespace oracle {

// constant.rs:1-25 — compile-time constants in the reference, runtime here so
// that configurations with diffusion/exchange switched on can be run. The
// defaults are the reference values.
struct Params {
    double gamma_e = 1.4, gamma_i = 1.4, gamma_r = 1.4;
    double cve = 1.0, cvi = 1.0, a_rad = 1.0;
    double kappa_e = 0.0, kappa_i = 0.0, kappa_r = 0.0;
    double omega_ei = 0.0, omega_er = 0.0;
    double lambda = 0.5;      // LAMBDA
    double weno_q = 10.0;     // WENO_Q
    double eps = 1e-12;       // DEFAULT_EPS
    double periodic_ly = 0.5; // bc1.rs:577 hardcodes ly = 0.5
    bool diffusion_active() const { return kappa_e != 0.0 || kappa_i != 0.0 || kappa_r != 0.0; }
    bool source_active() const { return omega_ei != 0.0 || omega_er != 0.0; }
};

// LLVM/compiler-rt powi: binary decomposition, r *= a on set bits, a *= a.
template <class T> inline T powi(T a, int b) {
    bool recip = b < 0;
    T r = T(1.0);
    for (;;) {
        if (b & 1) r = r * a;
        b /= 2;
        if (b == 0) break;
        a = a * a;
    }
    return recip ? T(1.0) / r : r;
}
template <class T> inline T sq(T x) { return x * x; }            // powi(x, 2)

// Rust `powf` (state.rs:261 x^0.25, bc1.rs:241 x^WENO_Q) is libm pow: glibc's
// is within 0.52 ulp and not always correctly rounded. Built with
// -DORACLE_CRPOW the restatement takes the correctly rounded power instead
// (double-double products, Dekker 1971), the power the CUDA path computes:
// that build separates what a last-bit change of libm does to a run from
// every other difference.
#ifdef ORACLE_CRPOW
struct DDPair {
    double hi, lo;
};
inline DDPair dd_product(DDPair a, DDPair b) {
    double p = a.hi * b.hi;
    double e = std::fma(a.hi, b.hi, -p);
    e = std::fma(a.hi, b.lo, e);
    e = std::fma(a.lo, b.hi, e);
    double s = p + e;
    return {s, e - (s - p)};
}
inline DDPair dd_square(double a) { // exact: a*a = hi + lo
    double p = a * a;
    return {p, std::fma(a, a, -p)};
}
inline double cr_int_power(double x, int n) { // n >= 1, binary powering in double-double
    if (!std::isfinite(x) || x == 0.0) return std::pow(x, (double)n);
    DDPair r = {1.0, 0.0}, a = {x, 0.0};
    bool first = true;
    while (n > 0) {
        if (n & 1) {
            r = first ? a : dd_product(r, a);
            first = false;
        }
        n >>= 1;
        if (n) a = (a.lo == 0.0) ? dd_square(a.hi) : dd_product(a, a);
    }
    if (!std::isfinite(r.hi)) return r.hi;
    return r.hi + r.lo;
}
inline double cr_quarter_power(double x) { // of sqrt(sqrt(x)) and its neighbours, the one whose 4th power is nearest x
    double y = std::sqrt(std::sqrt(x));
    if (!(x > 0.0) || !std::isfinite(x) || !std::isfinite(y)) return y;
    double cand[3] = {std::nextafter(y, 0.0), y, std::nextafter(y, INFINITY)};
    double best = y, bd = INFINITY;
    for (int k = 0; k < 3; ++k) {
        DDPair c2 = dd_square(cand[k]);
        DDPair c4 = dd_product(c2, c2);
        double d = std::fabs((c4.hi - x) + c4.lo);
        if (d < bd || (d == bd && k == 1)) {
            bd = d;
            best = cand[k];
        }
    }
    return best;
}
#endif
template <class T> inline T powf_ref(T x, double p) {
    using std::pow;
    return pow(x, p);
}
#ifdef ORACLE_CRPOW
template <> inline double powf_ref<double>(double x, double p) {
    if (p == 0.25) return cr_quarter_power(x);
    if (p >= 1.0 && p <= 64.0 && p == std::floor(p)) return cr_int_power(x, (int)p);
    return std::pow(x, p);
}
#endif
template <class T> inline T pow4(T x) { return (x * x) * (x * x); } // powi(x, 4)

enum Dir { DIR_X = 0, DIR_Y = 1 };

// state.rs:18-25
template <class T> struct StateT {
    T rho, mx, my, ee, ei, er;
    T& operator[](int k) { return (&rho)[k]; }
    const T& operator[](int k) const { return (&rho)[k]; }
};

// state.rs:213-226
template <class T> struct DerivedT {
    T u, v, e_e, e_i, e_r, pe, pi, pr, te, ti, tr;
};

// state.rs:245-276 Derived::from_state
template <class T> inline DerivedT<T> derived_from_state(const StateT<T>& s, const Params& P) {
    using std::pow;
    DerivedT<T> d;
    d.u = s.mx / s.rho;
    d.v = s.my / s.rho;
    T w2 = sq(d.u) + sq(d.v);
    d.e_e = s.ee / s.rho - w2 / 6.0;
    d.e_i = s.ei / s.rho - w2 / 6.0;
    d.e_r = s.er / s.rho - w2 / 6.0;
    d.pe = (P.gamma_e - 1.0) * (s.ee - s.rho * w2 / 6.0);
    d.pi = (P.gamma_i - 1.0) * (s.ei - s.rho * w2 / 6.0);
    d.pr = (P.gamma_r - 1.0) * (s.er - s.rho * w2 / 6.0);
    d.te = s.ee / (s.rho * P.cve) - w2 / (6.0 * P.cve);
    d.ti = s.ei / (s.rho * P.cvi) - w2 / (6.0 * P.cvi);
    T er_term = s.er / s.rho - w2 / 6.0;
    d.tr = powf_ref(er_term * s.rho / P.a_rad, 0.25);
    return d;
}

// state.rs:56-85 State::flux_from_derived
template <class T> inline StateT<T> flux_from_derived(const StateT<T>& s, const DerivedT<T>& d, Dir dir) {
    T u = d.u, v = d.v;
    T p = d.pe + d.pi + d.pr;
    T rho = s.rho;
    if (dir == DIR_X)
        return {rho * u, rho * u * u + p, rho * u * v, (s.ee + d.pe) * u, (s.ei + d.pi) * u, (s.er + d.pr) * u};
    return {rho * v, rho * u * v, rho * v * v + p, (s.ee + d.pe) * v, (s.ei + d.pi) * v, (s.er + d.pr) * v};
}

// weno.rs:28-459 Stencil6::build_l_plain (state1 = points[3], state2 = points[2])
template <class T>
inline void build_l_plain(const StateT<T>& state1, const StateT<T>& state2, const DerivedT<T>& d3,
                          const DerivedT<T>& d2, Dir dir, const Params& P, T L[6][6]) {
    using std::sqrt;
    T u1 = d3.u, u2 = d2.u, v1 = d3.v, v2 = d2.v;
    T ee1 = d3.e_e, ei1 = d3.e_i, er1 = d3.e_r;
    T ee2 = d2.e_e, ei2 = d2.e_i, er2 = d2.e_r;
    T rho1 = sqrt(state1.rho), rho2 = sqrt(state2.rho);
    T rho_sum = rho1 + rho2;
    T u = (u1 * rho1 + u2 * rho2) / rho_sum;
    T v = (v1 * rho1 + v2 * rho2) / rho_sum;
    T w2 = sq(u) + sq(v);
    T ee = (ee1 * rho1 + ee2 * rho2) / rho_sum;
    T ei = (ei1 * rho1 + ei2 * rho2) / rho_sum;
    T er = (er1 * rho1 + er2 * rho2) / rho_sum;
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    const double gt = gi + ge + gr;
    T cs2 = GE * ge * ee + GI * gi * ei + GR * gr * er;
    T cs = sqrt(cs2);
    T he = 6.0 * gi * gr * (GI * ei - GR * er) + GE * gt * ee * w2;
    T hi = 6.0 * ge * gr * (GR * er - GE * ee) + GI * gt * ei * w2;
    T hr = 6.0 * ge * gi * (GE * ee - GI * ei) + GR * gt * er * w2;
    T b = gt * (36.0 * ge * gi * gr + gt * sq(w2)) * cs2;
    T den = 12.0 * cs2;

    // electron / ion / radiation rows (identical in X and Y), weno.rs:119-235
    T E[6] = {ge / gt - ge * w2 / (6.0 * cs2) - ge * gt * w2 / b * (he - cs2 * w2),
              ge * u / (3.0 * cs2) + 2.0 * ge * gt * u / b * (he - cs2 * w2),
              ge * v / (3.0 * cs2) + 2.0 * ge * gt * v / b * (he - cs2 * w2),
              -sq(ge) / (gt * cs2) - 6.0 * ge / b * (ge * he - gt * cs2 * w2),
              -ge * gi / (gt * cs2) - 6.0 * ge * gi / b * (he - 6.0 * gr * cs2),
              -ge * gr / (gt * cs2) - 6.0 * ge * gr / b * (he + 6.0 * gi * cs2)};
    T I[6] = {gi / gt - gi * w2 / (6.0 * cs2) - gi * gt * w2 / b * (hi - cs2 * w2),
              gi * u / (3.0 * cs2) + 2.0 * gi * gt * u / b * (hi - cs2 * w2),
              gi * v / (3.0 * cs2) + 2.0 * gi * gt * v / b * (hi - cs2 * w2),
              -gi * ge / (gt * cs2) - 6.0 * gi * ge / b * (hi + 6.0 * gr * cs2),
              -sq(gi) / (gt * cs2) - 6.0 * gi / b * (gi * hi - gt * cs2 * w2),
              -gi * gr / (gt * cs2) - 6.0 * gi * gr / b * (hi - 6.0 * ge * cs2)};
    T R[6] = {gr / gt - gr * w2 / (6.0 * cs2) - gr * gt * w2 / b * (hr - cs2 * w2),
              gr * u / (3.0 * cs2) + 2.0 * gr * gt * u / b * (hr - cs2 * w2),
              gr * v / (3.0 * cs2) + 2.0 * gr * gt * v / b * (hr - cs2 * w2),
              -gr * ge / (gt * cs2) - 6.0 * gr * ge / b * (hr - 6.0 * gi * cs2),
              -gr * gi / (gt * cs2) - 6.0 * gr * gi / b * (hr + 6.0 * ge * cs2),
              -sq(gr) / (gt * cs2) - 6.0 * gr / b * (gr * hr - gt * cs2 * w2)};
    auto put = [&](int row, const T* src) { for (int c = 0; c < 6; ++c) L[row][c] = src[c]; };
    if (dir == DIR_X) {
        // weno.rs:89-107 and 249-267
        T a0[6] = {(gt * w2 + 6.0 * u * cs) / den, (-2.0 * gt * u - 6.0 * cs) / den, (-2.0 * gt * v) / den,
                   6.0 * ge / den, 6.0 * gi / den, 6.0 * gr / den};
        T a5[6] = {(gt * w2 - 6.0 * u * cs) / den, (-2.0 * gt * u + 6.0 * cs) / den, (-2.0 * gt * v) / den,
                   6.0 * ge / den, 6.0 * gi / den, 6.0 * gr / den};
        T tr[6] = {-v, T(0.0), T(1.0), T(0.0), T(0.0), T(0.0)};
        put(0, a0); put(1, E); put(2, I); put(3, R); put(4, tr); put(5, a5);
    } else {
        // weno.rs:280-311 and 437-455
        T a0[6] = {(gt * w2 + 6.0 * v * cs) / den, (-2.0 * gt * u) / den, (-2.0 * gt * v - 6.0 * cs) / den,
                   6.0 * ge / den, 6.0 * gi / den, 6.0 * gr / den};
        T a5[6] = {(gt * w2 - 6.0 * v * cs) / den, (-2.0 * gt * u) / den, (-2.0 * gt * v + 6.0 * cs) / den,
                   6.0 * ge / den, 6.0 * gi / den, 6.0 * gr / den};
        T tr[6] = {-u, T(1.0), T(0.0), T(0.0), T(0.0), T(0.0)};
        put(0, a0); put(1, tr); put(2, E); put(3, I); put(4, R); put(5, a5);
    }
}

// weno.rs:484-548 Stencil6::build_r_plain
template <class T>
inline void build_r_plain(const StateT<T>& state1, const StateT<T>& state2, const DerivedT<T>& d3,
                          const DerivedT<T>& d2, Dir dir, const Params& P, T lam[6], T Rm[6][6]) {
    using std::sqrt;
    T u1 = d3.u, u2 = d2.u, v1 = d3.v, v2 = d2.v;
    T ee1 = d3.e_e, ei1 = d3.e_i, er1 = d3.e_r;
    T ee2 = d2.e_e, ei2 = d2.e_i, er2 = d2.e_r;
    T rho1 = sqrt(state1.rho), rho2 = sqrt(state2.rho);
    T u = (u1 * rho1 + u2 * rho2) / (rho1 + rho2);
    T v = (v1 * rho1 + v2 * rho2) / (rho1 + rho2);
    T w2 = sq(u) + sq(v);
    T ee = (ee1 * rho1 + ee2 * rho2) / (rho1 + rho2);
    T ei = (ei1 * rho1 + ei2 * rho2) / (rho1 + rho2);
    T er = (er1 * rho1 + er2 * rho2) / (rho1 + rho2);
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    T cs = sqrt(GE * ge * ee + GI * gi * ei + GR * gr * er);
    const double gt = gi + ge + gr;
    if (dir == DIR_X) {
        T r[6][6] = {
            {T(1.0), T(1.0), T(1.0), T(1.0), T(0.0), T(1.0)},
            {u - cs, u, u, u, T(0.0), u + cs},
            {v, v, v, v, T(1.0), v},
            {GE * ee + w2 / 6.0 - u * cs / 3.0, gt * w2 / (6.0 * ge), T(-gr), T(gi), v / 3.0, GE * ee + w2 / 6.0 + u * cs / 3.0},
            {GI * ei + w2 / 6.0 - u * cs / 3.0, T(gr), gt * w2 / (6.0 * gi), T(-ge), v / 3.0, GI * ei + w2 / 6.0 + u * cs / 3.0},
            {GR * er + w2 / 6.0 - u * cs / 3.0, T(-gi), T(ge), gt * w2 / (6.0 * gr), v / 3.0, GR * er + w2 / 6.0 + u * cs / 3.0}};
        for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Rm[i][j] = r[i][j];
        T l[6] = {u - cs, u, u, u, u, u + cs};
        for (int i = 0; i < 6; ++i) lam[i] = l[i];
    } else {
        T r[6][6] = {
            {T(1.0), T(0.0), T(1.0), T(1.0), T(1.0), T(1.0)},
            {u, T(1.0), u, u, u, u},
            {v - cs, T(0.0), v, v, v, v + cs},
            {GE * ee + w2 / 6.0 - v * cs / 3.0, u / 3.0, gt * w2 / (6.0 * ge), T(-gr), T(gi), GE * ee + w2 / 6.0 + v * cs / 3.0},
            {GI * ei + w2 / 6.0 - v * cs / 3.0, u / 3.0, T(gr), gt * w2 / (6.0 * gi), T(-ge), GI * ei + w2 / 6.0 + v * cs / 3.0},
            {GR * er + w2 / 6.0 - v * cs / 3.0, u / 3.0, T(-gi), T(ge), gt * w2 / (6.0 * gr), GR * er + w2 / 6.0 + v * cs / 3.0}};
        for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) Rm[i][j] = r[i][j];
        T l[6] = {v - cs, v, v, v, v, v + cs};
        for (int i = 0; i < 6; ++i) lam[i] = l[i];
    }
}

// weno.rs:824-843 l_dot / r_dot
template <class T> inline void mat6_dot(const T M[6][6], const T x[6], T out[6]) {
    for (int i = 0; i < 6; ++i)
        out[i] = M[i][0] * x[0] + M[i][1] * x[1] + M[i][2] * x[2] + M[i][3] * x[3] + M[i][4] * x[4] + M[i][5] * x[5];
}

// weno.rs:847-886 weno5 (WENO-JS, p = 2)
template <class T> inline T weno5(T u0, T u1, T u2, T u3, T u4, double eps) {
    T beta2 = 13.0 / 12.0 * sq(u2 - 2.0 * u3 + u4) + 0.25 * sq(3.0 * u2 - 4.0 * u3 + u4);
    T beta1 = 13.0 / 12.0 * sq(u1 - 2.0 * u2 + u3) + 0.25 * sq(u1 - u3);
    T beta0 = 13.0 / 12.0 * sq(u0 - 2.0 * u1 + u2) + 0.25 * sq(u0 - 4.0 * u1 + 3.0 * u2);
    const double d0 = 0.1, d1 = 0.6, d2 = 0.3;
    T a0 = d0 / sq(eps + beta0);
    T a1 = d1 / sq(eps + beta1);
    T a2 = d2 / sq(eps + beta2);
    T sum_o = a0 + a1 + a2;
    T w0 = a0 / sum_o, w1 = a1 / sum_o, w2 = a2 / sum_o;
    T p0 = u0 / 3.0 - 7.0 / 6.0 * u1 + 11.0 / 6.0 * u2;
    T p1 = -u1 / 6.0 + 5.0 / 6.0 * u2 + u3 / 3.0;
    T p2 = u2 / 3.0 + 5.0 / 6.0 * u3 - u4 / 6.0;
    return w0 * p0 + w1 * p1 + w2 * p2;
}

// weno.rs:685-802 Stencil6::reconstruction_fast
template <class T>
inline StateT<T> reconstruction_fast(const StateT<T> pts[6], const DerivedT<T> d[6], Dir dir, bool recon_type,
                                     const Params& P) {
    T L[6][6], Rm[6][6], lam[6];
    build_l_plain(pts[3], pts[2], d[3], d[2], dir, P, L);
    build_r_plain(pts[3], pts[2], d[3], d[2], dir, P, lam, Rm);
    T cf[6][6], cs[6][6];
    for (int i = 0; i < 6; ++i) {
        StateT<T> fl = flux_from_derived(pts[i], d[i], dir);
        T fv[6] = {fl.rho, fl.mx, fl.my, fl.ee, fl.ei, fl.er};
        T sv[6] = {pts[i].rho, pts[i].mx, pts[i].my, pts[i].ee, pts[i].ei, pts[i].er};
        if (recon_type) {
            mat6_dot(L, fv, cf[i]);
            mat6_dot(L, sv, cs[i]);
        } else {
            for (int m = 0; m < 6; ++m) { cf[i][m] = fv[m]; cs[i][m] = sv[m]; }
        }
    }
    using std::fabs;
    T a[6];
    for (int m = 0; m < 6; ++m) a[m] = fabs(lam[m]);
    T fp[6][6], fm[6][6];
    for (int i = 0; i < 6; ++i)
        for (int m = 0; m < 6; ++m) {
            fp[i][m] = 0.5 * (cf[i][m] + a[m] * cs[i][m]);
            fm[i][m] = 0.5 * (cf[i][m] - a[m] * cs[i][m]);
        }
    T flux[6];
    for (int m = 0; m < 6; ++m) {
        T plus = weno5(fp[0][m], fp[1][m], fp[2][m], fp[3][m], fp[4][m], P.eps);
        T minus = weno5(fm[5][m], fm[4][m], fm[3][m], fm[2][m], fm[1][m], P.eps);
        flux[m] = plus + minus;
    }
    T c[6];
    mat6_dot(Rm, flux, c);
    return {c[0], c[1], c[2], c[3], c[4], c[5]};
}

// noncon.rs:26-44
template <class T> inline T sixth_order_derivative(T qm3, T qm2, T qm1, T qp1, T qp2, T qp3, double dx) {
    return (qp3 - 9.0 * qp2 + 45.0 * qp1 - 45.0 * qm1 + 9.0 * qm2 - qm3) / (60.0 * dx);
}

// noncon.rs:49-57
template <class T> inline T q_pulse(const T b[7]) {
    return -0.00714285714285723 * b[0] + 0.0595238095238118 * b[1] - 0.240476190476197 * b[2] +
           0.759523809523819 * b[3] + 0.509523809523803 * b[4] - 0.0904761904761891 * b[5] +
           0.00952380952380977 * b[6];
}

// noncon.rs:259-285 n_jump_pre (component jump q_pulse(rev(arr[1..8])) - q_pulse(arr[0..7]))
template <class T> inline T jump_component(const T arr[8]) {
    T b2[7] = {arr[0], arr[1], arr[2], arr[3], arr[4], arr[5], arr[6]};
    T b1[7] = {arr[7], arr[6], arr[5], arr[4], arr[3], arr[2], arr[1]};
    return q_pulse(b1) - q_pulse(b2);
}

// noncon.rs:288-332 nonconservative_direction_pre (+ dN_pre 235-257, n_jump_pre 259-285)
template <class T> inline StateT<T> nonconservative_pre(const DerivedT<T> d[9], double ds, Dir dir) {
    using std::fmax; using std::fmin;
    T v = dir == DIR_X ? d[4].u : d[4].v;
    // dN_pre on d[1..8]
    const DerivedT<T>* s7 = d + 1;
    T dpe = sixth_order_derivative(s7[0].pe, s7[1].pe, s7[2].pe, s7[4].pe, s7[5].pe, s7[6].pe, ds);
    T dpi = sixth_order_derivative(s7[0].pi, s7[1].pi, s7[2].pi, s7[4].pi, s7[5].pi, s7[6].pi, ds);
    T dpr = sixth_order_derivative(s7[0].pr, s7[1].pr, s7[2].pr, s7[4].pr, s7[5].pr, s7[6].pr, ds);
    T der_ee = 2.0 * dpe - dpi - dpr;
    T der_ei = 2.0 * dpi - dpe - dpr;
    T der_er = 2.0 * dpr - dpe - dpi;
    T nee[9], nei[9], ner[9];
    for (int k = 0; k < 9; ++k) {
        nee[k] = 2.0 * d[k].pe - d[k].pi - d[k].pr;
        nei[k] = 2.0 * d[k].pi - d[k].pe - d[k].pr;
        ner[k] = 2.0 * d[k].pr - d[k].pe - d[k].pi;
    }
    T jm_ee = jump_component(nee), jm_ei = jump_component(nei), jm_er = jump_component(ner);
    T jp_ee = jump_component(nee + 1), jp_ei = jump_component(nei + 1), jp_er = jump_component(ner + 1);
    T vm = dir == DIR_X ? d[3].u : d[3].v;
    T vp = dir == DIR_X ? d[5].u : d[5].v;
    T coef_left = fmax(fmax(v, vm), T(0.0)) / 3.0;
    T coef_right = fmin(fmin(v, vp), T(0.0)) / 3.0;
    StateT<T> o;
    o.rho = T(0.0); o.mx = T(0.0); o.my = T(0.0);
    o.ee = v / 3.0 * der_ee + (coef_left * jm_ee + coef_right * jp_ee) / ds;
    o.ei = v / 3.0 * der_ei + (coef_left * jm_ei + coef_right * jp_ei) / ds;
    o.er = v / 3.0 * der_er + (coef_left * jm_er + coef_right * jp_er) / ds;
    return o;
}

// diffusion.rs:27-50 build_diffusion_from_derived (only ee/ei/er are nonzero)
template <class T> inline StateT<T> diffusion_from_derived(const DerivedT<T> d[6], const Params& P) {
    const DerivedT<T>&sjp3 = d[5], &sjp2 = d[4], &sjp1 = d[3], &sj = d[2], &sjm1 = d[1], &sjm2 = d[0];
    T ee_term = P.kappa_e * (2.0 * sjp3.te - 25.0 * sjp2.te + 245.0 * sjp1.te - 245.0 * sj.te + 25.0 * sjm1.te -
                             2.0 * sjm2.te);
    T ei_term = P.kappa_i * (2.0 * sjp3.ti - 25.0 * sjp2.ti + 245.0 * sjp1.ti - 245.0 * sj.ti + 25.0 * sjm1.ti -
                             2.0 * sjm2.ti);
    T er_term = P.kappa_r * (2.0 * pow4(sjp3.tr) - 25.0 * pow4(sjp2.tr) + 245.0 * pow4(sjp1.tr) -
                             245.0 * pow4(sj.tr) + 25.0 * pow4(sjm1.tr) - 2.0 * pow4(sjm2.tr));
    return {T(0.0), T(0.0), T(0.0), ee_term / 180.0, ei_term / 180.0, er_term / 180.0};
}

// state.rs:118-135 State::te/ti/tr
template <class T> inline T state_te(const StateT<T>& s, const Params& P) {
    T u = s.mx / s.rho, v = s.my / s.rho;
    return s.ee / (s.rho * P.cve) - (sq(u) + sq(v)) / (6.0 * P.cve);
}
template <class T> inline T state_ti(const StateT<T>& s, const Params& P) {
    T u = s.mx / s.rho, v = s.my / s.rho;
    return s.ei / (s.rho * P.cvi) - (sq(u) + sq(v)) / (6.0 * P.cvi);
}
template <class T> inline T state_tr(const StateT<T>& s, const Params& P) {
    using std::pow;
    T u = s.mx / s.rho, v = s.my / s.rho;
    T er = s.er / s.rho - (sq(u) + sq(v)) / 6.0;
    return powf_ref(er * s.rho / P.a_rad, 0.25);
}

// source.rs:7-21
template <class T> inline StateT<T> source(const StateT<T>& s, const Params& P) {
    T te = state_te(s, P), tr = state_tr(s, P), ti = state_ti(s, P);
    return {T(0.0), T(0.0), T(0.0), -P.omega_ei * (te - ti) - P.omega_er * (pow4(te) - pow4(tr)),
            P.omega_ei * (te - ti), P.omega_er * (pow4(te) - pow4(tr))};
}

// dt.rs:5-34 get_local_dt
template <class T> inline T get_local_dt(const StateT<T>& s, double dx, double dy, const Params& P) {
    using std::sqrt; using std::fabs; using std::fmax;
    T u = s.mx / s.rho, v = s.my / s.rho;
    T ee = s.ee / s.rho - (sq(u) + sq(v)) / 6.0;
    T ei = s.ei / s.rho - (sq(u) + sq(v)) / 6.0;
    T er = s.er / s.rho - (sq(u) + sq(v)) / 6.0;
    const double GE = P.gamma_e, GI = P.gamma_i, GR = P.gamma_r, A = P.a_rad, CVE = P.cve, CVI = P.cvi;
    const double OEI = P.omega_ei, OER = P.omega_er;
    const double gi = GI - 1.0, ge = GE - 1.0, gr = GR - 1.0;
    T cs = sqrt(GE * ge * ee + GI * gi * ei + GR * gr * er);
    const double c4 = powi(CVE, 4), c3 = powi(CVE, 3);
    T ee3 = powi(ee, 3);
    T t1 = A * OEI * c4 + A * OEI * c3 * CVI + 4.0 * A * OER * CVI * ee3 + OER * c4 * CVI * s.rho;
    T s1 = sqrt(sq(t1) - 4.0 * A * OEI * OER * c4 * CVI * (4.0 * A * ee3 + c4 * s.rho + c3 * CVI * s.rho));
    T s2 = -(A * OEI * c4 + A * OEI * c3 * CVI + 4.0 * A * OER * CVI * ee3 + OER * c4 * CVI * s.rho);
    T sden = 2.0 * A * c4 * CVI * s.rho;
    T alpha1 = fabs((-s1 + s2) / sden);
    T alpha2 = fabs((s1 + s2) / sden);
    T sj = fmax(alpha1, alpha2);
    T dj = fmax(fmax(P.kappa_e / (CVE * s.rho), P.kappa_i / (CVI * s.rho)), T(P.kappa_r / A));
    T vj = (fabs(u) + cs) / dx + 2.0 * dj / (sq(dx) + sq(dy)) + sj + (fabs(v) + cs) / dy;
    return P.lambda / vj;
}

} // namespace oracle
