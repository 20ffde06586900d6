"""Committed fixtures (tests/golden/make_golden.py): the oracle must reproduce
them bit for bit; the GPU exact build must match them (bitwise for l(),
1e-10 normwise after the steps); the product case builders must produce the
same initial states."""
import os

import numpy as np
import pytest

from helpers import rel_linf

HERE = os.path.dirname(os.path.abspath(__file__))
PLANAR = dict(nx=256, ny=8, lx=1.0, ly=0.03125, x_shock=0.25, mach=2.0, sigma=0.25)
PLANAR_PARAMS = dict(kappa_e=1e-3, kappa_i=1e-3, kappa_r=1e-3, omega_ei=1.0, omega_er=1.0, periodic_ly=0.03125)


def fixture(name):
    return np.load(os.path.join(HERE, "golden", name))


def test_oracle_reproduces_cylinder_fixture(O):
    z = fixture("cyl31x121.npz")
    c = O.Case.cylinder(h=0.1)
    assert np.array_equal(c.fluid(), z["fluid"])
    assert np.array_equal(c.state(), z["u0"])
    rhs, gv = c.l()
    assert np.array_equal(rhs, z["rhs0"]) and np.array_equal(gv, z["ghosts0"])
    dts = c.run(10, 0.05)
    assert np.array_equal(dts, z["dts"]) and np.array_equal(c.state(), z["u10"])


def test_oracle_reproduces_planar_fixture(O):
    z = fixture("planar256x8.npz")
    p = O.Case.planar_shock(**PLANAR, **PLANAR_PARAMS)
    assert np.array_equal(p.state(), z["u0"])
    assert np.array_equal(p.run(20, 0.05), z["dts"])
    assert np.array_equal(p.state(), z["u20"])


def test_product_cases_build_the_fixture_inputs(rh):
    z = fixture("cyl31x121.npz")
    f = rh.cases.init_cylinder(h=0.1)
    assert np.array_equal(f.fluid, z["fluid"]) and np.array_equal(f.value, z["u0"])
    z = fixture("planar256x8.npz")
    f = rh.cases.planar_shock(params=rh.Params(**PLANAR_PARAMS), **PLANAR)
    assert np.array_equal(f.value, z["u0"])


@pytest.mark.gpu
def test_gpu_exact_build_matches_fixtures(rh):
    z = fixture("cyl31x121.npz")
    f = rh.cases.init_cylinder(h=0.1)
    g = rh.GhostGrid.build(f)
    s = rh.Solver(f, g, exact=True)
    rhs, gv = s.l(with_ghosts=True)
    assert np.array_equal(rhs, z["rhs0"]) and np.array_equal(gv, z["ghosts0"])
    s.advance(10, 0.05)
    u, t = s.download()
    assert rel_linf(u, z["u10"], f.fluid).max() <= 1e-10
    z = fixture("planar256x8.npz")
    f = rh.cases.planar_shock(params=rh.Params(**PLANAR_PARAMS), **PLANAR)
    s = rh.Solver(f, rh.GhostGrid.build(f), exact=True)
    s.advance(20, 0.05)
    u, _ = s.download()
    assert rel_linf(u, z["u20"], f.fluid).max() <= 1e-10
