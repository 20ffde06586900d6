"""The GhostBC least-squares tables (bc1.rs:108-188 precompute_ghost_bc) against
an independent numpy computation.

The reference forms, per heavy ghost and order r = 0..4, the monomial matrix
A of the E_r stencil nodes in the ghost's local (normal, tangential) frame,
its pseudo-inverse P by nalgebra's SVD with an absolute singular-value cut of
1e-12, S_r = P^T M_r P (M_r the quadratic form of the smoothness indicator,
bc1.rs:62-81 / 1070-1196) and w_{r,k} = k! P[x^k row]. The builder computes P
with its own one-sided Jacobi SVD. Here numpy recomputes every table from the
stencil nodes and the projection alone:

  - P by np.linalg.pinv of A with its columns scaled by h^-degree (the
    scaled matrix is well conditioned, so its pseudo-inverse is accurate to
    a few ulps; for a full column rank A, pinv(A) = D pinv(A D));
  - M_r from the analytic integrals of the squared derivatives over the cell
    [-h/2, h/2]^2, written here independently of the builder;
  - the smallest singular value of the unscaled A, which nalgebra compares
    with the absolute cut: every retained one must stay well above 1e-12, or
    a change of geometry could silently change the truncation.

Checked on the half-cylinder at h = 1/40 (every heavy ghost) and h = 1/320
(961 x 3841 nodes; a sample of the heavy ghosts, which include the smallest
singular values of all the configurations)."""
import math

import numpy as np
import pytest

BC_STENCIL_OFF = (0, 1, 5, 14, 30, 55)
BC_S_OFF = (0, 1, 17, 98, 354, 979)
BC_W_OFF = (0, 1, 9, 36, 100, 225)
CUT = 1.0e-12


def monomials(r):
    """(i, j) exponents of x^i y^j in the reference's coefficient order
    (bc1.rs:1199-1214: total degree t = 0..r, then i = 0..t, j = t - i)."""
    return [(i, t - i) for t in range(r + 1) for i in range(t + 1)]


def cell_moment(p, h):
    """integral of s^p over [-h/2, h/2]"""
    return 0.0 if p % 2 else 2.0 * (h / 2.0) ** (p + 1) / (p + 1)


def quadratic_form(r, h):
    """M_r with beta(c) = c^T M_r c = sum over derivative orders 1 <= |a| <= r of
    |K|^(|a|-1) * integral over K of (D^a p)^2 (Jiang-Shu type indicator, the
    r = 0 case being a constant that does not use M)."""
    mons = monomials(r)
    n = len(mons)
    M = np.zeros((n, n))
    for ax in range(r + 1):
        for ay in range(r + 1 - ax):
            order = ax + ay
            if order == 0:
                continue
            scale = h ** (2 * (order - 1))
            der = []
            for (i, j) in mons:
                if i < ax or j < ay:
                    der.append(None)
                    continue
                f = math.perm(i, ax) * math.perm(j, ay)
                der.append((i - ax, j - ay, float(f)))
            for a in range(n):
                if der[a] is None:
                    continue
                for b in range(n):
                    if der[b] is None:
                        continue
                    ia, ja, fa = der[a]
                    ib, jb, fb = der[b]
                    M[a, b] += scale * fa * fb * cell_moment(ia + ib, h) * cell_moment(ja + jb, h)
    return M


def check_tables(field, grids, sample, rtol_s, rtol_w):
    g = field.grid
    h = math.sqrt(g.dx * g.dy)
    heavy = np.flatnonzero(grids.pre >= 0)
    if sample is not None:
        heavy = heavy[::sample]
    forms = [quadratic_form(r, h) for r in range(5)]
    worst_s, worst_w, min_sigma = 0.0, 0.0, math.inf
    for gid in heavy:
        slot = grids.pre[gid]
        p0x, p0y, nx, ny, _ = grids.proj[gid]
        st = grids.stencil[slot].astype(np.int64)
        ii, jj = st // g.ny, st % g.ny
        x = g.x0 + ii * g.dx
        y = g.y0 + jj * g.dy
        ddx, ddy = x - p0x, y - p0y
        nor = nx * ddx + ny * ddy      # geometry.rs:97-107 gloabl2local_coord
        tan = -ddx * ny + ddy * nx
        for r in range(5):
            m = (r + 1) ** 2
            sl = slice(BC_STENCIL_OFF[r], BC_STENCIL_OFF[r + 1])
            xn, yt = nor[sl], tan[sl]
            mons = monomials(r)
            A = np.stack([xn ** i * yt ** j for (i, j) in mons], axis=1)
            if r > 0:
                min_sigma = min(min_sigma, np.linalg.svd(A, compute_uv=False).min())
            D = np.array([h ** -(i + j) for (i, j) in mons])
            P = D[:, None] * np.linalg.pinv(A * D[None, :])
            s = grids.s[slot, BC_S_OFF[r]:BC_S_OFF[r + 1]].reshape(m, m)
            if r == 0:
                assert s[0, 0] == 2.0 * h * h  # bc1.rs:167-168: S_0 = 2 h^2, not P^T M P
            else:
                S = P.T @ forms[r] @ P
                worst_s = max(worst_s, np.abs(s - S).max() / np.abs(S).max())
            for k in range(r + 1):
                col = mons.index((k, 0))
                wk = math.factorial(k) * P[col]
                w = grids.w[slot, BC_W_OFF[r] + k * m:BC_W_OFF[r] + (k + 1) * m]
                worst_w = max(worst_w, np.abs(w - wk).max() / np.abs(wk).max())
    print(f"h={h:.6g}: {len(heavy)} ghosts, S rel {worst_s:.2e}, w rel {worst_w:.2e}, "
          f"smallest sigma {min_sigma:.3e} (cut {CUT:g})")
    assert worst_s <= rtol_s and worst_w <= rtol_w
    return min_sigma


def test_tables_h40(rh):
    f = rh.cases.init_cylinder(h=1.0 / 40.0)
    g = rh.GhostGrid.build(f)
    sig = check_tables(f, g, None, 1e-10, 1e-10)
    assert sig > 1e3 * CUT


def test_tables_h320_and_cut_margin(rh):
    f = rh.cases.init_cylinder(h=1.0 / 320.0)
    g = rh.GhostGrid.build(f)
    sig = check_tables(f, g, 23, 1e-10, 1e-10)
    # every singular value of every E_r fit is retained, with a margin of
    # more than two decades above the absolute cut
    assert sig > 100 * CUT
