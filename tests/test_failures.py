"""Failures injected on the host, checked against the oracle.

The reference panics in these cases (bc1.rs:467-469 for a singular ILW
system, bc1.rs:594-604 for a periodic wrap that leaves the fluid); the
library returns the matching status and, in a batch, stops only the
instance that failed.

  - singular Wall system: a uniform state whose normal velocity equals the
    sound speed exactly (gamma = 3 for all three species, rho = 4,
    u = a = 1.5, specific energies 1/8: every quantity is a binary fraction,
    so no rounding takes part). The ILW system of bc1.rs:691-756 (the
    incoming-characteristic rows of L with the first row replaced by the
    no-penetration row) then has an exactly zero pivot on the wall the flow
    leaves through, and the reference's LAPACK solve fails there;
  - periodic wrap length that does not match the domain (ly = 0.5 on a
    strip 0.03125 high): the wrapped row of the bottom ghosts lies outside
    the grid.
"""
import numpy as np
import pytest

# rho = 4, rho*u = 6 (u = 1.5), E_k = rho*(1/8 + u^2/6) = 2; with gamma = 3,
# a^2 = sum gamma (gamma - 1) e_k = 6 * 3/8 = 2.25, so a = u = 1.5 exactly.
SONIC = np.array([4.0, 6.0, 0.0, 2.0, 2.0, 2.0])
SONIC_PARAMS = dict(gamma_e=3.0, gamma_i=3.0, gamma_r=3.0)
RECT_N = 16
DIRECTIONS = [(1, 0), (-1, 0), (0, 1), (0, -1)]


def _sonic_state(direction):
    s = SONIC.copy()
    s[1], s[2] = direction[0] * 6.0, direction[1] * 6.0
    return s


def _leaves(ij, idx, proj, direction):
    """True where ghost ij belongs to the wall the flow leaves through: the
    outward normal of its projection (a corner ghost takes the normal of the
    segment it projects onto) is the flow direction."""
    k = [tuple(x) for x in np.asarray(idx).tolist()].index(tuple(int(v) for v in ij))
    return proj[k][2] * direction[0] + proj[k][3] * direction[1] == 1.0


@pytest.mark.parametrize("direction", DIRECTIONS)
@pytest.mark.parametrize("variant", ["plain", "fma"])
def test_oracle_singular_wall(O, direction, variant):
    M = O if variant == "plain" else O.fma_variant()
    c = M.Case.rect(RECT_N, RECT_N, 1.0, 1.0, _sonic_state(direction), **SONIC_PARAMS)
    with pytest.raises(M.OracleError) as ei:
        c.l()
    assert ei.value.code == 3
    info = c.ghost_info()
    assert _leaves(ei.value.ij, info["ij"], info["proj"], direction)


def test_oracle_periodic_wrap_mismatch(O):
    c = O.Case.planar_shock(nx=64, ny=8, periodic_ly=0.5)
    with pytest.raises(O.OracleError) as ei:
        c.l()
    assert ei.value.code == 4


@pytest.mark.gpu
@pytest.mark.parametrize("exact", [False, True])
@pytest.mark.parametrize("direction", DIRECTIONS)
def test_singular_wall_reported(rh, O, direction, exact):
    f = rh.cases.rect_field(RECT_N, RECT_N, 1.0, 1.0, _sonic_state(direction), params=rh.Params(**SONIC_PARAMS))
    g = rh.GhostGrid.build(f)
    s = rh.Solver(f, g, exact=exact)
    with pytest.raises(rh.RH3TError) as ei:
        s.l()
    e = ei.value
    assert e.kind == "SINGULAR_ILW"
    assert _leaves((e.i, e.j), g.idx, g.proj, direction)
    # the oracle's solve fails on the same ghost
    c = O.Case.rect(RECT_N, RECT_N, 1.0, 1.0, _sonic_state(direction), **SONIC_PARAMS)
    with pytest.raises(O.OracleError) as oe:
        c.ghost_value(c.ghost_id(e.i, e.j))
    assert oe.value.code == 3
    s.close()


@pytest.mark.gpu
def test_singular_wall_instance_isolated(rh):
    good = [rh.cases.init_cylinder(h=1.0 / 10.0), rh.cases.init_double_mach(h=1.0 / 40.0)]
    bad = rh.cases.rect_field(RECT_N, RECT_N, 1.0, 1.0, _sonic_state((0, -1)), params=rh.Params(**SONIC_PARAMS))
    fields = [good[0], bad, good[1]]
    grids = [rh.GhostGrid.build(f) for f in fields]
    b = rh.Batch(fields, grids)
    with pytest.raises(rh.RH3TError) as ei:
        b.advance(3, 0.05)
    assert ei.value.kind == "SINGULAR_ILW" and ei.value.instance == 1
    st = b.status()
    assert st[1] == 3 and st[0] == 0 and st[2] == 0
    res = b.download()
    for q in (0, 2):
        s = rh.Solver(fields[q], grids[q])
        s.advance(3, 0.05)
        u, t = s.download()
        s.close()
        assert np.array_equal(res[q][0], u) and res[q][1] == t
    b.close()


@pytest.mark.gpu
def test_periodic_wrap_mismatch_reported(rh):
    f = rh.cases.planar_shock(nx=64, ny=8, params=rh.Params(periodic_ly=0.5))
    g = rh.GhostGrid.build(f)
    with pytest.raises(rh.RH3TError) as ei:
        rh.Solver(f, g)
    assert ei.value.kind == "PERIODIC_WRAP"
    assert "periodic wrapped point is not fluid" in str(ei.value)
    cyl = rh.cases.init_cylinder(h=1.0 / 10.0)
    with pytest.raises(rh.RH3TError) as ei:
        rh.Batch([cyl, f], [rh.GhostGrid.build(cyl), g])
    assert ei.value.kind == "PERIODIC_WRAP" and "instance 1" in str(ei.value)


@pytest.mark.gpu
def test_bounded_wait_gives_up(rh):
    """The ghost update's mbarrier wait is bounded (RH3T_ERR_DEVICE_TIMEOUT
    instead of a hang): on a barrier that nothing completes it gives up, on
    one whose phase completes it returns, and the device stays usable."""
    import ctypes as C
    import time
    L = rh.load()
    t = C.c_int32(-1)
    assert L.rh3t_wait_check(0, 1, C.byref(t)) == 0 and t.value == 0
    t0 = time.perf_counter()
    assert L.rh3t_wait_check(0, 0, C.byref(t)) == 0 and t.value == 1
    print(f"wait gave up after {time.perf_counter() - t0:.3f} s")
    assert time.perf_counter() - t0 < 30.0
    assert L.rh3t_wait_check(0, 1, C.byref(t)) == 0 and t.value == 0
