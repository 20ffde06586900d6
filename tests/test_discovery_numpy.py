"""A second, independent witness of the bit-exact part of the ghost-grid
build: a numpy restatement (written here, sharing no code with the library
or the C++ oracle) of the fluid mask (field1.rs:112-122 with the ray-crossing
test of geometry.rs:254-278) and of ghost discovery (ghost.rs:352-376: every
node that is not fluid and lies on the radius-4 cross of a fluid node, grid
bounds ignored, sorted by (i, j)). The library's mask and ghost list must
equal it exactly for the reference's half-cylinder, the planar shock and
double Mach."""
import numpy as np
import pytest


def _is_fluid(points, fluid_side, px, py):
    """geometry.rs:254-278 over arrays of points, same operations."""
    inside = np.zeros(px.shape, bool)
    n = len(points)
    if n < 3:
        return np.zeros(px.shape, bool)
    for k in range(n):
        ax, ay = points[k]
        bx, by = points[(k + 1) % n]
        cross = (ay > py) != (by > py)
        with np.errstate(divide="ignore", invalid="ignore"):
            xi = ax + (py - ay) * (bx - ax) / (by - ay)
        inside ^= cross & (px < xi)
    return inside if fluid_side == 0 else ~inside


def _in_domain(f, i, j):
    g = f.grid
    px = g.x0 + i.astype(np.float64) * g.dx
    py = g.y0 + j.astype(np.float64) * g.dy
    return (_is_fluid(f.outer_bound.points, f.outer_bound.fluid, px, py) &
            _is_fluid(f.inner_bound.points, f.inner_bound.fluid, px, py))


@pytest.mark.parametrize("case", ["cylinder", "planar", "double_mach"])
def test_numpy_mask_and_discovery(rh, case):
    if case == "cylinder":
        f = rh.cases.init_cylinder(h=1.0 / 40.0)
    elif case == "planar":
        f = rh.cases.planar_shock(params=rh.Params(periodic_ly=0.03125))
    else:
        f = rh.cases.init_double_mach(h=1.0 / 40.0)
    nx, ny = f.grid.nx, f.grid.ny
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    mask = _in_domain(f, ii.ravel(), jj.ravel())
    assert np.array_equal(mask, np.asarray(f.fluid, bool)), "fluid mask"
    # candidates: the radius-4 cross around every fluid node
    fi, fj = ii.ravel()[mask], jj.ravel()[mask]
    cand = set()
    for d in list(range(-4, 0)) + list(range(1, 5)):
        for a, b in ((fi + d, fj), (fi, fj + d)):
            inside = (a >= 0) & (a < nx) & (b >= 0) & (b < ny)
            fl = np.zeros(a.shape, bool)
            fl[inside] = mask[a[inside] * ny + b[inside]]
            out = ~inside
            if out.any():
                fl[out] = _in_domain(f, a[out], b[out])
            cand.update(zip(a[~fl].tolist(), b[~fl].tolist()))
    ghosts = np.array(sorted(cand), np.int64)
    g = rh.GhostGrid.build(f)
    assert g.len() == len(ghosts)
    assert np.array_equal(g.idx.astype(np.int64), ghosts)
