"""Device power routines (x^(1/4) for Tr, x^10 for the boundary WENO weights)
against correctly rounded values from mpmath. The reference calls libm pow
(state.rs:261, bc1.rs:241); the device replaces both with correctly rounded
double-double evaluations (3t_rh_b200/csrc/physics.cuh)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_correctly_rounded_powers(rh):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 200
    rng = np.random.default_rng(7)
    x = np.concatenate([np.exp(rng.uniform(-20, 20, 3000)), np.exp(rng.uniform(-27.6, 5, 1000))])
    L = rh.load()
    out = np.zeros(3 * len(x))
    assert L.rh3t_math_check(0, x.ctypes.data, len(x), 10.0, out.ctypes.data) == 0
    out = out.reshape(-1, 3)
    bad_q = bad_10 = 0
    for k, v in enumerate(x):
        m = mpmath.mpf(float(v))
        bad_q += out[k, 0] != float(m ** mpmath.mpf(0.25))
        bad_10 += out[k, 1] != float(m ** 10)
    assert bad_q == 0 and bad_10 == 0, (bad_q, bad_10)
    assert np.array_equal(out[:, 1], out[:, 2])


def test_shared_reciprocal_division_bitwise(rh):
    """Where one divisor serves several quotients, and for the constants 3
    and 6, the solver divides by a shared reciprocal (Markstein's correction
    step, csrc/divrn.cuh): every quotient must equal the IEEE one bit for
    bit. 4e9 device-generated pairs: random operands over the fast path's
    exponent range and beyond it, divisors with all-ones significands,
    quotients next to a rounding midpoint, special values, and the two
    constants; and the face's reciprocals of 6 c^2 and 3 c^2, which the
    flux kernel forms as 2 and 4 times RN(1 / (12 c^2))."""
    for exact in (True, False):
        L = rh.load(exact)
        counts = np.zeros(7, np.int64)
        first = np.zeros(3)
        seed = 1 if exact else 2
        assert L.rh3t_div_check(0, 2_000_000_000, seed, counts.ctypes.data, first.ctypes.data) == 0
        assert counts.sum() == 0, (counts.tolist(), first.tolist())
