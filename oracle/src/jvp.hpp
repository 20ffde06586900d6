// ORACLE — test infrastructure only (see physics.hpp). Forward-mode
// (dual-number) restatement of the reference l() (main.rs:135-305) with the
// ghost update (ghost.rs:199-268, bc1.rs:609-928): every function below is
// the double-precision function of solver.cpp written over a scalar type T.
// With T = Dual the value parts reproduce the double oracle bit for bit
// (same operations in the same order) and the tangent parts give the
// directional derivative J_l(u) du of l() for a state direction du, a
// FarField state direction and exchange-coefficient directions. It is the
// reference of the CUDA adjoint (vector-Jacobian products) in the tests.
#pragma once
#include "model.hpp"
#include <cmath>
#include <vector>

namespace oracle {

struct Dual {
    double v = 0.0, d = 0.0;
    Dual() = default;
    Dual(double x) : v(x), d(0.0) {}
    Dual(double x, double dx) : v(x), d(dx) {}
    Dual& operator+=(Dual b) { v += b.v; d += b.d; return *this; }
    Dual& operator-=(Dual b) { v -= b.v; d -= b.d; return *this; }
    Dual& operator*=(Dual b) { *this = Dual{v * b.v, d * b.v + v * b.d}; return *this; }
    Dual& operator/=(Dual b) { double q = v / b.v; *this = Dual{q, (d - q * b.d) / b.v}; return *this; }
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) {
    double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline bool operator==(Dual a, Dual b) { return a.v == b.v; }
inline Dual sqrt(Dual a) {
    double s = std::sqrt(a.v);
    return {s, a.d / (2.0 * s)};
}
inline Dual pow(Dual a, double p) {
    double r = std::pow(a.v, p);
    return {r, p * std::pow(a.v, p - 1.0) * a.d};
}
inline Dual fabs(Dual a) { return a.v < 0.0 ? -a : a; }
inline Dual fmax(Dual a, Dual b) { return a.v >= b.v ? a : b; }
inline Dual fmin(Dual a, Dual b) { return a.v <= b.v ? a : b; }

inline double val(double x) { return x; }
inline double val(Dual x) { return x.v; }
template <class T> T seed(double v, double d);
template <> inline double seed<double>(double v, double) { return v; }
template <> inline Dual seed<Dual>(double v, double d) { return Dual{v, d}; }

// tangent inputs of one l() evaluation
struct Tangent {
    const double* du = nullptr; // nx*ny*6 state direction (fluid cells)
    double duinf[6] = {0, 0, 0, 0, 0, 0}; // direction of every FarField BC state
    double domega_ei = 0.0, domega_er = 0.0;
};

} // namespace oracle
