// ORACLE — test infrastructure only (see physics.hpp).
// Operation counting: the templated pointwise functions of physics.hpp
// instantiated on a scalar that counts its floating-point operations
// (add/sub/mul/div/sqrt/pow/fabs/fmin/fmax each 1). Gives the algorithmic
// FLOPs of the reference's per-face / per-cell work for the roofline.
#include <cmath>
#include <cstring>

#include "physics.hpp"

namespace oracle {

static long long g_ops = 0;

struct Cnt {
    double v;
    Cnt() : v(0) {}
    Cnt(double x) : v(x) {}
};
inline Cnt operator+(Cnt a, Cnt b) { ++g_ops; return Cnt(a.v + b.v); }
inline Cnt operator-(Cnt a, Cnt b) { ++g_ops; return Cnt(a.v - b.v); }
inline Cnt operator*(Cnt a, Cnt b) { ++g_ops; return Cnt(a.v * b.v); }
inline Cnt operator/(Cnt a, Cnt b) { ++g_ops; return Cnt(a.v / b.v); }
inline Cnt operator-(Cnt a) { return Cnt(-a.v); } // sign flip: not counted
inline Cnt operator+(Cnt a, double b) { return a + Cnt(b); }
inline Cnt operator+(double a, Cnt b) { return Cnt(a) + b; }
inline Cnt operator-(Cnt a, double b) { return a - Cnt(b); }
inline Cnt operator-(double a, Cnt b) { return Cnt(a) - b; }
inline Cnt operator*(Cnt a, double b) { return a * Cnt(b); }
inline Cnt operator*(double a, Cnt b) { return Cnt(a) * b; }
inline Cnt operator/(Cnt a, double b) { return a / Cnt(b); }
inline Cnt operator/(double a, Cnt b) { return Cnt(a) / b; }
inline bool operator<(Cnt a, double b) { return a.v < b; }
inline Cnt sqrt(Cnt a) { ++g_ops; return Cnt(std::sqrt(a.v)); }
inline Cnt pow(Cnt a, double b) { ++g_ops; return Cnt(std::pow(a.v, b)); }
inline Cnt fabs(Cnt a) { ++g_ops; return Cnt(std::fabs(a.v)); }
inline Cnt fmax(Cnt a, Cnt b) { ++g_ops; return Cnt(std::fmax(a.v, b.v)); }
inline Cnt fmin(Cnt a, Cnt b) { ++g_ops; return Cnt(std::fmin(a.v, b.v)); }

using CS = StateT<Cnt>;
using CD = DerivedT<Cnt>;

static CS mk(double a, double b, double c, double d, double e, double f) { return CS{a, b, c, d, e, f}; }

} // namespace oracle

using namespace oracle;

// out: [0] face flux X  [1] face flux Y  (reconstruction_fast incl. its six physical fluxes)
//      [2] Derived::from_state  [3] nonconservative term, one direction
//      [4] diffusion interface flux  [5] source term  [6] get_local_dt
//      [7] weno5  [8] build_l_plain  [9] build_r_plain  [10] flux_from_derived (X)
extern "C" void oracle_flop_counts(long long* out) {
    Params P;
    CS pts[6];
    CD d[6];
    for (int i = 0; i < 6; ++i) {
        pts[i] = mk(1.0 + 0.01 * i, 0.5, 0.3, 3.0, 2.0, 1.0);
    }
    for (int i = 0; i < 6; ++i) d[i] = derived_from_state(pts[i], P);
    g_ops = 0;
    reconstruction_fast(pts, d, DIR_X, true, P);
    out[0] = g_ops;
    g_ops = 0;
    reconstruction_fast(pts, d, DIR_Y, true, P);
    out[1] = g_ops;
    g_ops = 0;
    derived_from_state(pts[0], P);
    out[2] = g_ops;
    CD d9[9];
    for (int i = 0; i < 9; ++i) d9[i] = derived_from_state(mk(1.0 + 0.01 * i, 0.5, 0.3, 3.0, 2.0, 1.0), P);
    g_ops = 0;
    nonconservative_pre(d9, 0.1, DIR_X);
    out[3] = g_ops;
    g_ops = 0;
    P.kappa_e = P.kappa_i = P.kappa_r = 1e-3;
    diffusion_from_derived(d, P);
    out[4] = g_ops;
    g_ops = 0;
    P.omega_ei = P.omega_er = 1.0;
    source(pts[0], P);
    out[5] = g_ops;
    g_ops = 0;
    P = Params();
    get_local_dt(pts[0], 0.1, 0.1, P);
    out[6] = g_ops;
    g_ops = 0;
    weno5(Cnt(1.0), Cnt(2.0), Cnt(3.0), Cnt(4.0), Cnt(5.0), 1e-12);
    out[7] = g_ops;
    Cnt L[6][6], R[6][6], lam[6];
    g_ops = 0;
    build_l_plain(pts[3], pts[2], d[3], d[2], DIR_X, P, L);
    out[8] = g_ops;
    g_ops = 0;
    build_r_plain(pts[3], pts[2], d[3], d[2], DIR_X, P, lam, R);
    out[9] = g_ops;
    g_ops = 0;
    flux_from_derived(pts[0], d[0], DIR_X);
    out[10] = g_ops;
}
