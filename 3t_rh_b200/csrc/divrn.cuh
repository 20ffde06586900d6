// Correctly rounded FP64 division a / b by a reciprocal shared between
// several divisions with the same divisor, for the no-contraction build:
// every quotient equals the IEEE quotient bit for bit, at 5 (or, for the
// constants 3 and 6, 3) FP64 operations once the reciprocal is known.
//
// Method: Markstein's correction step (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res.
// Dev. 34(1), 1990; also Cornea, Harrison, Tang, "Scientific Computing on
// Itanium-based Systems", 2002). Let y = RN(1/b) and q a faithful
// approximation of z = a/b (one of the two doubles around z). Then
// r = a - b q is a double (computed exactly by one FMA) and
// RN(q + r y) = RN(z). Proof, b = B 2^(eb-52) with B in [2^52, 2^53), z in
// [2^E, 2^(E+1)): every midpoint mu between doubles near z is
// M 2^(E-53), M odd, so a - b mu = N 2^(eb+E-105) with N a nonzero integer
// (a quotient of two doubles is never a midpoint); r = R 2^(eb+E-104) with
// |R| < B; b y - 1 = K 2^-105 with |K| <= B/2 (y is within half an ulp of
// 1/b). Then b (q + r y - mu) = (a - b mu) + r (b y - 1)
//                             = 2^(eb+E-105) (N + R K 2^-104),
// and |R K 2^-104| < B^2 2^-105 < 1 <= |N|: q + r y lies on the same side of
// every midpoint as z (and is none), so both round to the same double.
//
// A faithful q: q0 = RN(a y) is within 1.5 ulp of z (|a y - z| < z 2^-53);
// q1 = RN(q0 + RN(a - b q0) y) is within (1/2 + 2^-51) ulp, hence faithful;
// q2 = RN(q1 + (a - b q1) y) = RN(z). For b = 3 or 6, RN(1/b) = (1 - 2^-54)/b
// exactly, so a y lies within half an ulp below z and RN(a y) is already
// faithful: one correction suffices.
//
// The argument needs no overflow, underflow or special value anywhere: the
// fast sequence is taken only when both exponents are within [-450, 450]
// (then z lies in [2^-901, 2^901], y in [2^-451, 2^450] and a nonzero r
// above 2^-557: all normal numbers); a zero numerator over such a divisor
// is the signed zero a y; anything else (subnormal, huge, infinite, NaN, a
// divisor out of range) takes the IEEE division. tests/test_gpu_math.py compares
// every routine here with the IEEE quotient bit for bit on random,
// near-midpoint and special operands (rh3t_div_check).
#pragma once

namespace rh3t {

__device__ __forceinline__ bool div_in_range(double x) {
    const unsigned e = (unsigned)__double2hiint(x) & 0x7ff00000u;
    return e - 0x23d00000u <= 0x38400000u; // biased exponent in [1023 - 450, 1023 + 450]
}

// the IEEE quotient, out of line: the rare operands outside the fast range
// take it, and one copy of its code serves every call site (the callers'
// code stays small enough for the instruction cache)
static __device__ __noinline__ double div_ieee(double a, double b) { return __ddiv_rn(a, b); }

// operands outside the fast range (b_ok: b is in it, y = RN(1/b)): a zero
// numerator over such a divisor, common where a flow is uniform, gives the
// signed zero a y (y is finite, nonzero and of b's sign, so the sign is a's
// XOR b's, as in IEEE division); anything else takes the IEEE quotient. The
// zero test is inline: zero numerators are too frequent for a call (batch
// of half-cylinder instances: with zeros through the IEEE division the flux
// kernels ran 9% and the RHS 26% slower, with the test out of line 2% and 6%)
__device__ __forceinline__ double div_edge(double a, double b, double y, bool b_ok) {
    return (b_ok && a == 0.0) ? __dmul_rn(a, y) : div_ieee(a, b);
}

struct Recip {
    double b, y;
    bool ok;
};

__device__ __forceinline__ Recip recip(double b) {
    Recip d;
    d.b = b;
    d.y = __ddiv_rn(1.0, b);
    d.ok = div_in_range(b);
    return d;
}

// a Recip from a divisor and its stored reciprocal RN(1/b)
__device__ __forceinline__ Recip recip_of(double b, double y) {
    Recip d;
    d.b = b;
    d.y = y;
    d.ok = div_in_range(b);
    return d;
}

// a / d.b, correctly rounded
__device__ __forceinline__ double div_rn(double a, const Recip& d) {
    if (!(d.ok && div_in_range(a))) return div_edge(a, d.b, d.y, d.ok);
    double q = __dmul_rn(a, d.y);
    double r = __fma_rn(-d.b, q, a);
    q = __fma_rn(r, d.y, q);
    r = __fma_rn(-d.b, q, a);
    return __fma_rn(r, d.y, q);
}

// a / 3.0 and a / 6.0, correctly rounded
__device__ __forceinline__ double div3_rn(double a) {
    const double y = 0x1.5555555555555p-2; // RN(1/3)
    if (!div_in_range(a)) return div_edge(a, 3.0, y, true);
    const double q = __dmul_rn(a, y);
    const double r = __fma_rn(-3.0, q, a);
    return __fma_rn(r, y, q);
}
__device__ __forceinline__ double div6_rn(double a) {
    const double y = 0x1.5555555555555p-3; // RN(1/6)
    if (!div_in_range(a)) return div_edge(a, 6.0, y, true);
    const double q = __dmul_rn(a, y);
    const double r = __fma_rn(-6.0, q, a);
    return __fma_rn(r, y, q);
}

} // namespace rh3t
