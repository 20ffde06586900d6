"""The oracle's dual-number l() (oracle/src/jvp.hpp), the reference values of the
CUDA adjoint: its double instantiation reproduces the oracle's l() bit for
bit, its value parts do too, its tangent is linear in the direction, and it
matches central differences in the exchange coefficients (a direction that
moves no kink argument)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def case(O):
    c = O.Case.cylinder(h=0.1, omega_ei=0.5, omega_er=2.0)
    c.run(10, 0.05)
    return c


def test_templates_reproduce_oracle(case):
    r1, g1 = case.l()
    r2, g2 = case.l_t()
    assert np.array_equal(r1, r2) and np.array_equal(g1, g2)


def test_dual_values_are_the_oracle(case):
    r1, g1 = case.l()
    du = np.random.default_rng(0).standard_normal(r1.shape) * case.fluid()[:, None]
    r, _, g, _ = case.l_jvp(du, np.ones(6), [1.0, -1.0])
    assert np.array_equal(r, r1) and np.array_equal(g, g1)


def test_tangent_is_linear(case):
    rng = np.random.default_rng(1)
    fl = case.fluid()[:, None]
    a, b = rng.standard_normal((2, case.n, 6)) * fl
    _, ja, _, _ = case.l_jvp(a)
    _, jb, _, _ = case.l_jvp(b)
    _, jab, _, _ = case.l_jvp(2.0 * a - 3.0 * b)
    assert np.abs(jab - (2.0 * ja - 3.0 * jb)).max() <= 1e-9 * np.abs(jab).max()


def test_exchange_tangent_vs_central_difference(O):
    def rhs(oei, oer):
        c = O.Case.cylinder(h=0.1, omega_ei=oei, omega_er=oer)
        c.run(5, 0.05)
        return c

    base = rhs(0.5, 2.0)
    u = base.state()
    _, dr, _, _ = base.l_jvp(None, None, [1.0, 0.0])
    h = 1e-3  # l() is linear in omega_ei: a wide step loses nothing and keeps rounding small
    cp, cm = O.Case.cylinder(h=0.1, omega_ei=0.5 + h, omega_er=2.0), O.Case.cylinder(h=0.1, omega_ei=0.5 - h,
                                                                                      omega_er=2.0)
    for c in (cp, cm):
        c.set_state(u)
        c.time = base.time
    fd = (cp.l()[0] - cm.l()[0]) / (2 * h)
    fl = base.fluid()
    assert np.abs(fd[fl] - dr[fl]).max() <= 1e-8 * np.abs(dr[fl]).max()
