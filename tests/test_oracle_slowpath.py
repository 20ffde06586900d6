"""The oracle's ghost update against the reference's own second witness: the
per-call least-squares path of set_ghost_point_value(.., None)
(bc1.rs:345-421 weno_extrapolation, bc1.rs:1039-1049 poly_regression,
bc1.rs:1557-1579 weno_data_preprocess), restated in oracle/src/slowpath.cpp
with an independent least-squares solve.

  - main.rs:548-613 ghost_bc_fast_matches_slow, ported: the initial
    half-cylinder (h = 1/40) at the test's eight grid points, projection and
    side formed as the test forms them, the precomputed path against the
    per-call one, max abs difference < 1e-10.
  - The reference's test only reaches inflow FarField ghosts, whose values do
    not depend on the extrapolation (every characteristic enters). Extended
    here to developed states and every Wall, Outflow and FarField ghost of
    three cases: the half-cylinder after 30 steps (outflow-side and
    transverse FarField sides), the double Mach reflection after 10 steps
    (Wall ghosts: ILW rows and both 6x6 solves) and the planar shock after 20
    steps (Outflow LODI row, subsonic-inflow FarField).
  - The precomputed path's r = 0 smoothness indicator is 2 h^2 v^2 (S_0 = 2 h^2
    used as a quadratic form, bc1.rs:167-168, 222-231) where the per-call
    path's is 2 h^2 (bc1.rs:1087-1089). With that term taken as the
    precomputed path takes it, the two paths agree to the rounding
    sensitivity of the boundary weights; with the per-call path's own term
    they differ by up to ~20% of the state on extrapolated ghosts, so the
    solver's (precomputed) behaviour is what the oracle and the CUDA path
    follow.

Tolerance of the extended check, relative to the ghost state's largest
component: 1e-7 on the half-cylinder and double Mach cases (measured
<= 1.1e-8); 1e-6 on the planar shock, where beta = d^T S d of near-uniform
data cancels to far below eps = 1e-12 and the q = 10 weights then move the
ghost values of the precomputed path by up to 6.4e-7 under a plain change of
rounding (the oracle built with FMA contraction, same state)."""
import numpy as np
import pytest

PLANAR = dict(kappa_e=1e-3, kappa_i=1e-3, kappa_r=1e-3, omega_ei=1.0, omega_er=1.0, periodic_ly=0.03125)


def test_ghost_bc_fast_matches_slow(O):
    c = O.Case.cylinder()
    for (i, j) in [(-1, 100), (-1, 240), (-2, 240), (-3, 240), (0, 0), (2, 240), (3, 240), (1, 100)]:
        proj, side = c.ghost_probe(i, j)
        a = c.ghost_value_at(i, j, proj, side, mode="slow")
        b = c.ghost_value_at(i, j, proj, side, mode="fast")
        assert np.abs(a - b).max() < 1e-10, (i, j)


def _scan(case):
    """per (boundary, side): ghosts, max rel. difference precomputed vs
    per-call (r = 0 term as precomputed), vs per-call (its own r = 0 term)"""
    gi = case.ghost_info()
    out = {}
    for gid in np.flatnonzero(gi["pre"] >= 0):
        i, j = (int(x) for x in gi["ij"][gid])
        proj, side, bnd = gi["proj"][gid], int(gi["side"][gid]), int(gi["boundary"][gid])
        ref = case.ghost_value(gid)
        assert np.array_equal(case.ghost_value_at(i, j, proj, side, bnd, "fast"), ref)
        sc = np.abs(ref).max()
        e0 = np.abs(case.ghost_value_at(i, j, proj, side, bnd, "slow_beta0") - ref).max() / sc
        e1 = np.abs(case.ghost_value_at(i, j, proj, side, bnd, "slow") - ref).max() / sc
        n, m0, m1 = out.get((bnd, side), (0, 0.0, 0.0))
        out[(bnd, side)] = (n + 1, max(m0, e0), max(m1, e1))
    return out


@pytest.mark.parametrize("case,steps,tol", [("cylinder", 30, 1e-7), ("double_mach", 10, 1e-7),
                                            ("planar", 20, 1e-6)])
def test_ghosts_fast_matches_slow_developed(O, case, steps, tol):
    c = {"cylinder": lambda: O.Case.cylinder(h=0.1), "double_mach": lambda: O.Case.double_mach(h=1.0 / 40.0),
         "planar": lambda: O.Case.planar_shock(nx=256, **PLANAR)}[case]()
    c.run(steps, 0.05)
    res = _scan(c)
    for k, (n, e0, e1) in sorted(res.items()):
        print(f"{case} boundary/side {k}: {n} ghosts, per-call (r=0 as precomputed) {e0:.2e}, per-call {e1:.2e}")
        assert e0 <= tol, k
    if case in ("cylinder", "double_mach"):
        # the r = 0 indicator of the two reference paths differs, and it shows
        assert max(e1 for _, _, e1 in res.values()) > 1e-3
