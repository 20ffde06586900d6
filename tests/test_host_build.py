"""The product's host-side Field/GhostGrid build (C++, rh3t_geom_*) against
the oracle's restatement of field1.rs / ghost.rs / bc1.rs: ghost discovery,
projection and E_r stencils must be bit-identical (the reference's ghost
layout is part of its API); the least-squares tables must agree."""
import numpy as np
import pytest


def _compare(rh, O, f, oc):
    g = rh.GhostGrid.build(f, with_access=True)
    oi, op = oc.ghost_info(), oc.ghost_pre()
    assert np.array_equal(f.fluid, oc.fluid())
    assert g.len() == oc.n_ghosts() and g.n_heavy() == oc.n_heavy()
    assert np.array_equal(g.idx, oi["ij"])
    assert np.array_equal(g.boundary, oi["boundary"])
    assert np.array_equal(g.side, oi["side"])
    assert np.array_equal(g.proj.view(np.int64), oi["proj"].view(np.int64))  # bitwise
    assert np.array_equal(g.pre, oi["pre"])
    assert np.array_equal(g.nearest, op["nearest"])
    assert np.array_equal(g.stencil, op["stencil"])
    assert np.array_equal(g.access, oc.access())
    assert np.array_equal(g.d, op["d"])
    scale_s = np.abs(op["s"]).max(axis=1, keepdims=True) + 1e-300
    scale_w = np.abs(op["w"]).max(axis=1, keepdims=True) + 1e-300
    assert (np.abs(g.s - op["s"]) / scale_s).max() <= 1e-12
    assert (np.abs(g.w - op["w"]) / scale_w).max() <= 1e-12
    return g


def test_cylinder_reference_grid(rh, O):
    f = rh.cases.init_cylinder()
    oc = O.Case.cylinder()
    assert np.array_equal(f.value, oc.state())
    g = _compare(rh, O, f, oc)
    # counts of the reference case (121 x 481): fluid nodes, ghosts, heavy ghosts
    assert f.fluid.sum() == 55132 and g.len() == 4914 and g.n_heavy() == 4480


def test_cylinder_refined(rh, O):
    f = rh.cases.init_cylinder(h=1.0 / 160.0)
    oc = O.Case.cylinder(h=1.0 / 160.0)
    g = _compare(rh, O, f, oc)
    assert f.fluid.sum() == 881574 and g.len() == 19716


def test_planar_shock_corners_pick_farfield(rh, O):
    f = rh.cases.planar_shock()
    oc = O.Case.planar_shock()
    assert np.array_equal(f.value, oc.state())
    g = _compare(rh, O, f, oc)
    # the ghosts below / above column 0 project onto the corner and take the
    # higher-priority FarField side (ghost.rs:285-348)
    for j in (-1, -2, -3, -4, 8, 9, 10, 11):
        k = int(np.flatnonzero((g.idx[:, 0] == 0) & (g.idx[:, 1] == j))[0])
        assert g.side[k] == 3 and g.pre[k] >= 0
    assert g.len() == 8256 and g.n_heavy() == 72


def test_double_mach(rh, O):
    f = rh.cases.init_double_mach(h=1.0 / 80.0)
    oc = O.Case.double_mach(h=1.0 / 80.0)
    assert np.array_equal(f.value, oc.state())
    _compare(rh, O, f, oc)

