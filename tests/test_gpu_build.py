"""GPU ghost-grid build (rh3t_geom_build_ghosts_device): the least-squares
tables of the Wall / Outflow / FarField ghosts (bc1.rs:108-188 E_r
pseudo-inverses, S_r, w_r) computed on the device equal the host build's bit
for bit, for one geometry and for many uneven geometries in one pass; the
integer tables (ghost set, sides, projections, E_r stencils, access table)
are the host's by construction and are checked too.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TABLES = ("idx", "boundary", "side", "proj", "pre", "nearest", "stencil", "s", "w", "d")


def _same(a, b):
    for name in TABLES:
        x, y = getattr(a, name), getattr(b, name)
        assert x.shape == y.shape, name
        # bitwise: compare the bytes (NaN-free tables, -0.0 distinguished)
        assert x.tobytes() == y.tobytes(), f"{name} differs"


@pytest.mark.parametrize("case", ["cylinder40", "planar", "double_mach"])
def test_device_build_bitwise(rh, case):
    if case == "cylinder40":
        f = rh.cases.init_cylinder(h=1.0 / 40.0)
    elif case == "planar":
        f = rh.cases.planar_shock(params=rh.Params(periodic_ly=0.03125))
    else:
        f = rh.cases.init_double_mach(h=1.0 / 40.0)
    host = rh.GhostGrid.build(f, with_access=True)
    dev = rh.GhostGrid.build(f, device=0, with_access=True)
    assert host.n_heavy() > 0
    _same(host, dev)
    assert np.array_equal(host.access, dev.access)


def test_device_build_many_bitwise(rh):
    specs = rh.cases.batch_specs(9)
    fields = [rh.cases.batch_field(sp) for sp in specs]
    fields.append(rh.cases.init_double_mach(h=1.0 / 20.0))
    t0 = time.perf_counter()
    dev = rh.GhostGrid.build_many(fields, device=0)
    t_dev = time.perf_counter() - t0
    t0 = time.perf_counter()
    host = [rh.GhostGrid.build(f) for f in fields]
    t_host = time.perf_counter() - t0
    for a, b in zip(host, dev):
        _same(a, b)
    print(f"ghost-grid build of {len(fields)} fields ({sum(g.n_heavy() for g in host)} heavy ghosts): "
          f"host {t_host:.2f} s, device {t_dev:.2f} s")


def test_device_build_solver_runs(rh):
    """A solver built from device tables runs and equals one built from host tables."""
    f = rh.cases.init_cylinder(h=1.0 / 20.0)
    gh, gd = rh.GhostGrid.build(f), rh.GhostGrid.build(f, device=0)
    out = []
    for g in (gh, gd):
        s = rh.Solver(f, g)
        s.advance(5, 0.05)
        out.append(s.download()[0])
        s.close()
    assert np.array_equal(out[0], out[1])
