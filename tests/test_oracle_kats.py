"""The reference's own unit tests (colinhu123/3T_RH, #[cfg(test)] modules),
ported as known-answer tests of the oracle. They pin the CPU restatement to
the reference's behaviour; the reference itself cannot be built on this
image (no Rust toolchain), so these KATs and the op-for-op restatement are
the oracle's anchor.
"""
import math

import numpy as np
import pytest

X, Y = 0, 1
TOL = 1e-10  # weno.rs:895


def ref_state():
    return np.array([1.0, 0.5, 0.3, 3.0, 2.0, 1.0])  # weno.rs:915-924


# ------------------------------------------------------------------ weno.rs tests
def test_weno_constant(O):  # weno.rs:988-1001
    assert abs(O.weno5([5.0] * 5) - 5.0) < 1e-12


def test_weno5_accuracy(O):  # weno.rs:1003-1076
    errors = []
    for nx in (40, 80, 160, 320):
        dx = 2.0 * math.pi / nx
        err, cnt = 0.0, 0
        for j in range(3, nx - 3):
            x = j * dx
            sr = [math.sin(x - 2 * dx), math.sin(x - dx), math.sin(x), math.sin(x + dx), math.sin(x + 2 * dx)]
            xm = x - dx
            sl = [math.sin(xm - 2 * dx), math.sin(xm - dx), math.sin(xm), math.sin(xm + dx), math.sin(xm + 2 * dx)]
            num = (O.weno5(sr) - O.weno5(sl)) / dx
            err += abs(num - math.cos(x))
            cnt += 1
        errors.append(err / cnt)
    orders = [math.log2(errors[i - 1] / errors[i]) for i in range(1, len(errors))]
    for o in orders[1:]:
        assert o > 4.5, orders


@pytest.mark.parametrize("d", [X, Y])
def test_eigen_inverse(O, d):  # weno.rs:1108-1154
    s = ref_state()
    L, R, lam = O.build_lr(s, s, d)
    assert len(lam) == 6
    assert np.abs(L @ R - np.eye(6)).max() < TOL


@pytest.mark.parametrize("d", [X, Y])
def test_characteristic_round_trip(O, d):  # weno.rs:1160-1203
    s = ref_state()
    L, R, _ = O.build_lr(s, s, d)
    assert np.abs(R @ (L @ s) - s).max() < TOL


@pytest.mark.parametrize("d", [X, Y])
def test_constant_flux_preserving(O, d):  # weno.rs:1209-1242
    s = ref_state()
    r = O.reconstruction(np.tile(s, (6, 1)), d, True)
    assert np.abs(r - O.flux(s, d)).max() < TOL


@pytest.mark.parametrize("d", [X, Y])
def test_conservative_variant_applies_r(O, d):
    """weno.rs:1248-1281 expects reconstruction(false) == F for a constant
    stencil, but weno.rs:672-677 multiplies by R in both variants, so that
    reference test fails against its own code (by inspection). The
    restatement keeps the code's behaviour: R . F. Only recon = true is on the
    hot path (main.rs:179, 202)."""
    s = ref_state()
    r = O.reconstruction(np.tile(s, (6, 1)), d, False)
    _, R, _ = O.build_lr(s, s, d)
    assert np.abs(r - R @ O.flux(s, d)).max() < TOL * np.abs(R @ O.flux(s, d)).max()


def test_x_and_y_flux_are_direction_sensitive(O):  # weno.rs:1287-1317
    s = np.array([1.0, 0.7, 0.2, 3.0, 2.0, 1.0])
    fx, fy = O.flux(s, X), O.flux(s, Y)
    assert abs(fx[0] - fy[0]) > 1e-12
    assert abs(fx[0] - s[1]) < TOL and abs(fy[0] - s[2]) < TOL


def test_reconstruction_fast_matches_reconstruction(O):
    """main.rs:514-545: 100 stencils from the test's LCG (main.rs:493-498, seed
    12345; rho in [0.5, 1.5], momenta in [-0.5, 0.5], energies in [1, 2]),
    reconstruction_fast (weno.rs:685-802) against the ndarray reconstruction
    (weno.rs:599-679) for both recon types and directions, max abs difference
    < 1e-12."""
    seed = [12345]

    def rng():
        seed[0] = (seed[0] * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        return float(seed[0] >> 11) / float(1 << 53)

    worst = 0.0
    for _ in range(100):
        pts = np.array([[0.5 + rng(), rng() - 0.5, rng() - 0.5, 1.0 + rng(), 1.0 + rng(), 1.0 + rng()]
                        for _ in range(6)])
        for recon in (True, False):
            for d in (X, Y):
                a = O.reconstruction_slow(pts, d, recon)
                b = O.reconstruction(pts, d, recon)
                assert np.isfinite(b).all()
                worst = max(worst, np.abs(a - b).max())
    assert worst < 1e-12


# ------------------------------------------------------------------ noncon.rs tests
def _n_vector(O, s):
    d = O.derived(s)
    pe, pi, pr = d[5], d[6], d[7]
    return np.array([2 * pe - pi - pr, 2 * pi - pe - pr, 2 * pr - pe - pi])


def test_n_vector_zero_pressure(O):  # noncon.rs:373-392
    assert np.all(_n_vector(O, [1.0, 0, 0, 0, 0, 0]) == 0.0)


def test_n_vector_pressure_split_inverse(O):  # noncon.rs:394-418
    """The expected values (5/3, 5/3, -10/3) need gamma_e = gamma_i = 5/3 and
    gamma_r = 4/3 (py_utils/contour_gen.py:15-17), not constant.rs's 1.4, so
    the reference test fails against its own constants; with those gammas as
    runtime parameters the restatement reproduces them, and with 1.4 it gives
    N = 0 as the reference code does."""
    p = O.params_array(gamma_e=5.0 / 3.0, gamma_i=5.0 / 3.0, gamma_r=4.0 / 3.0)
    d = O.derived([1.0, 0, 0, 5.0, 5.0, 5.0], p)
    pe, pi, pr = d[5], d[6], d[7]
    n = [2 * pe - pi - pr, 2 * pi - pe - pr, 2 * pr - pe - pi]
    assert abs(n[0] - 5.0 / 3.0) < 1e-12 and abs(n[1] - 5.0 / 3.0) < 1e-12 and abs(n[2] + 10.0 / 3.0) < 1e-12
    assert np.abs(_n_vector(O, [1.0, 0, 0, 5.0, 5.0, 5.0])).max() < 1e-15


def test_sixth_order_derivative(O):  # noncon.rs:424-465
    assert abs(O.sixth_derivative([1.0] * 6, 0.1)) < 1e-14
    assert abs(O.sixth_derivative([-3.0, -2.0, -1.0, 1.0, 2.0, 3.0], 1.0) - 1.0) < 1e-12


@pytest.mark.parametrize("d", [X, Y])
def test_nonconservative_constant_state(O, d):  # noncon.rs:471-521, 563-629
    r = O.noncon(np.tile([1.0, 0.5, 0.8, 2.0, 2.0, 2.0], (9, 1)), 1.0, d)
    assert np.all(r[:3] == 0.0) and np.abs(r[3:]).max() < 1e-10
    r = O.noncon(np.tile([1.0, 0.0, 0.0, 3.0, 3.0, 3.0], (9, 1)), 1.0, d)
    assert np.abs(r).max() < 1e-14


def test_direction_velocity(O):  # noncon.rs:527-557
    d = O.derived([2.0, 6.0, 10.0, 1.0, 1.0, 1.0])
    assert abs(d[0] - 3.0) < 1e-14 and abs(d[1] - 5.0) < 1e-14


def test_nonconservative_zero_velocity(O):  # noncon.rs:635-701
    sx = np.array([[1.0, 0.0, 1.0, 0.9 + 0.1 * k, 1.9 + 0.1 * k, 2.9 + 0.1 * k] for k in range(9)])
    assert np.abs(O.noncon(sx, 1.0, X)).max() < 1e-10
    sy = np.array([[1.0, 1.0, 0.0, 0.9 + 0.1 * k, 1.9 + 0.1 * k, 2.9 + 0.1 * k] for k in range(9)])
    assert np.abs(O.noncon(sy, 1.0, Y)).max() < 1e-10


# ------------------------------------------------------------------ bc1.rs tests
def test_polynomial_least_squares_reproduces_degree4(O):  # bc1.rs:1713-1769
    def f(x, y):
        return (1 + 2 * x + 3 * y + 4 * x * x + 5 * x * y + 6 * y * y + 7 * x ** 3 + 8 * x ** 2 * y + 9 * x * y ** 2 +
                10 * y ** 3 + 11 * x ** 4 + 12 * x ** 3 * y + 13 * x ** 2 * y ** 2 + 14 * x * y ** 3 + 15 * y ** 4)

    h = 0.1
    data = np.array([(i * h, j * h, f(i * h, j * h)) for i in range(-2, 3) for j in range(-2, 3)])
    c = O.fit_poly(data, 4)
    assert len(c) == 15
    err = 0.0
    for x, y, ex in data:
        rec, col = 0.0, 0
        for t in range(5):
            for i in range(t + 1):
                rec += c[col] * x ** i * y ** (t - i)
                col += 1
        err = max(err, abs(rec - ex))
    assert err < 5e-10


def test_x_derivatives_at_origin(O):  # bc1.rs:1786-1816
    c = [1.0, 3.0, 2.0, 6.0, 5.0, 4.0, 10.0, 9.0, 8.0, 7.0, 15.0, 14.0, 13.0, 12.0, 11.0]
    for k, e in enumerate([1.0, 2.0, 8.0, 42.0, 264.0]):
        assert abs(O.x_derivative(c, 4, k) - e) < 1e-13


def test_constant_polynomial_fit(O):  # bc1.rs:2151-2177
    h = 0.0125
    data = np.array([(i * h, j * h, 1.0) for i in range(-2, 3) for j in range(-2, 3)])
    assert abs(O.fit_poly(data, 4)[0] - 1.0) < 1e-12


def _rect(O, n=80):
    # bc1.rs:1641-1702 with State::primi2con(1, 0, 0, 1, 1, 1) = (1, 0, 0, 2.5, 2.5, 2.5)
    return O.Case.rect(n, n, 1.0, 1.0, [1.0, 0.0, 0.0, 2.5, 2.5, 2.5], O.BC_WALL)


@pytest.mark.parametrize("ghost,vertical,step", [((-1, 40), True, 1), ((40, -1), False, 1)])
def test_paper_stencil_structure(O, ghost, vertical, step):  # bc1.rs:1827-1951
    c = _rect(O)
    p = c.project_outer(c.x0 + ghost[0] * c.dx, c.y0 + ghost[1] * c.dy)
    fl = c.fluid().reshape(c.nx, c.ny)
    for r in range(5):
        e = c.extractor(p, r)
        w = r + 1
        assert len(e) == w * w
        for l in range(w):
            s = e[l * w:(l + 1) * w]
            line, along = (0, 1) if vertical else (1, 0)
            assert np.all(s[:, line] == s[0, line])
            assert np.all(np.diff(s[:, along]) == 1)
            assert all(fl[i, j] for i, j in s)
        for l in range(1, w):
            line = 0 if vertical else 1
            assert e[l * w, line] == e[(l - 1) * w, line] + step


def test_oblique_boundary_paper_stencil(O):  # bc1.rs:2050-2149 (triangle (0,0),(1,0),(0,1))
    # the triangle fixture is restated through the rect case's extractor on a
    # projection onto x + y = 1 from (0.62, 0.42)
    c = O.Case.rect(100, 100, 1.0, 1.0, [1.0, 0, 0, 2.5, 2.5, 2.5], O.BC_WALL)
    n = np.array([1.0, 1.0]) / math.sqrt(2.0)
    p = np.array([0.62, 0.42])
    dist = (p[0] + p[1] - 1.0) / math.sqrt(2.0)
    p0 = p - dist * n
    e = c.extractor([p0[0], p0[1], n[0], n[1], dist], 4)
    assert len(e) == 25


def test_characteristic_weno_constant_state_zero_derivatives(O):  # bc1.rs:1964-1998
    """The reference test runs the per-call SVD path (bc1.rs:345-421); the
    solver runs the precomputed path (bc1.rs:193-255), whose V^(k) for a
    constant field is a sum of O(k!/h^k) weights that cancels to rounding.
    What reaches the ghost is V^(k) D^k / k! with |D| <= 4h (bc1.rs:733-739):
    that contribution is checked at the reference's 5e-10."""
    c = _rect(O)
    g = c.ghost_id(-1, 40)
    v = c.ghost_extrapolation(g)
    assert np.isfinite(v[0]).all()
    h = c.dx
    for k in range(1, 5):
        assert np.abs(v[k]).max() * (4 * h) ** k / math.factorial(k) < 5e-10


def test_final_wall_ghost_preserves_stationary_constant_state(O):  # bc1.rs:2006-2033
    c = _rect(O)
    exact = np.array([1.0, 0.0, 0.0, 2.5, 2.5, 2.5])
    worst = 0.0
    for idx in [(-1, 40), (-2, 40), (-3, 40), (80, 40), (81, 40), (82, 40), (40, -1), (40, -2), (40, -3), (40, 80),
                (40, 81), (40, 82)]:
        worst = max(worst, np.abs(c.ghost_value(c.ghost_id(*idx)) - exact).max())
    assert worst < 5e-10


# ------------------------------------------------------------------ geometry.rs arc tests
ARC = [0.0, -1.0, -1.0, 0.0, 0.0, 1.0]


def test_three_point_construction_left_semicircle(O):  # geometry.rs:689-703
    a = O.circle_from_three(ARC, 1)
    assert abs(a[0]) < 1e-12 and abs(a[1]) < 1e-12 and abs(a[2] - 1.0) < 1e-12
    assert O.arc_contains(a, 1, math.pi)
    assert not O.arc_contains(a, 1, 0.0) and not O.arc_contains(a, 1, 2.0 * math.pi)


def test_stagnation_projection(O):  # geometry.rs:705-721
    a = O.circle_from_three(ARC, 1)
    p = O.arc_project(a, 1, -1.2, 0.0)
    assert abs(p[0] + 1.0) < 1e-12 and abs(p[1]) < 1e-12
    assert abs(p[2] - 1.0) < 1e-12 and abs(p[3]) < 1e-12 and abs(p[4] + 0.2) < 1e-12


def test_upper_lower_mirror_symmetry(O):  # geometry.rs:723-740
    a = O.circle_from_three(ARC, 1)
    u, d = O.arc_project(a, 1, -1.1, 0.2), O.arc_project(a, 1, -1.1, -0.2)
    assert abs(u[0] - d[0]) < 1e-12 and abs(u[1] + d[1]) < 1e-12
    assert abs(u[2] - d[2]) < 1e-12 and abs(u[3] + d[3]) < 1e-12 and abs(u[4] - d[4]) < 1e-12


def test_finite_arc_endpoint_selection(O):  # geometry.rs:742-759
    a = O.circle_from_three(ARC, 1)
    p = O.arc_project(a, 1, 0.3, 0.7)
    assert abs(p[0]) < 1e-12 and abs(p[1] - 1.0) < 1e-12
    p = O.arc_project(a, 1, 0.3, -0.7)
    assert abs(p[0]) < 1e-12 and abs(p[1] + 1.0) < 1e-12


# ------------------------------------------------------------------ ghost.rs / main.rs tests
def test_default_offsets_radius_four_cross(O):  # ghost.rs:513-522
    c = _rect(O, 20)
    acc = c.access()
    assert acc.shape[1] == 17


def test_cylinder_arc_registration_is_shifted(O):
    """main.rs:615-637 expects the arc centre at y = 0; init.rs:268,318,336-344
    shifts every arc point by +0.0125, so that reference test fails against
    the reference's own init_cylinder. The restatement follows the code."""
    c = O.Case.cylinder()
    g = c.geometry()
    arc = g["arcs"][0]
    assert arc[0] == 2 and arc[1] == 361
    assert abs(arc[2]) < 1e-12 and abs(arc[3] - 0.0125) < 1e-12 and abs(arc[4] - 1.0) < 1e-12
    assert all(k == O.BC_REFLECTIVE_WALL for k in g["outer_kind"][2:362])


def test_cylinder_counts(O):
    c = O.Case.cylinder()
    assert c.nx == 121 and c.ny == 481
    assert c.fluid().sum() == 55132 and c.n_ghosts() == 4914 and c.n_heavy() == 4480
