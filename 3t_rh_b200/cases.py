"""Initial conditions / domains of the workloads (the builders the reference
keeps in init.rs, restated for inputs of the solver).

  init_cylinder     init.rs:116-510 with mesh width, Mach number and arc shift
                    as parameters (reference: h = 1/40, M = 3, shift 0.0125)
  init_double_mach  init.rs:26-113 (reference mesh width 1/320)
  planar_shock      translating Mach-2 shock, y-periodic (no reference builder)
  rect_field        bc1.rs:1641-1702 test fixture (one BC kind on all sides)
  batch_specs       seeded half-cylinder instances of uneven size and
                    parameters for the batched solver (the LCG of the
                    reference's parity tests, main.rs:493-498)
  SurfacePressure   the adjoint's objective: pressure integrated over the
                    cylinder arc (no reference counterpart)
"""
import math

import numpy as np

from .api import (FLUID_INSIDE, FLUID_OUTSIDE, ArcOverride, BCType, CircularArc, Field, GridInfo, Params,
                  Polygon)


def euler_to_three_energy(rho, ux, uy, p, gamma):
    """init.rs:7-24: equal split of the total energy."""
    kinetic = 0.5 * rho * (ux * ux + uy * uy)
    e_total = p / (gamma - 1.0) + kinetic
    return np.array([rho, rho * ux, rho * uy, e_total / 3.0, e_total / 3.0, e_total / 3.0])


def _dummy_inner():
    return Polygon([(-1002.0, -1002.0), (-1001.0, -1002.0), (-1001.0, -1001.0), (-1002.0, -1001.0)], FLUID_OUTSIDE)


def freestream(mach=3.0):
    gamma, rho_inf, p_inf = 1.4, 1.0, 1.0
    a_inf = math.sqrt(gamma * p_inf / rho_inf)
    return euler_to_three_energy(rho_inf, mach * a_inf, 0.0, p_inf, gamma)


def init_cylinder(h=1.0 / 40.0, mach=3.0, shift=0.0125, params=None):
    u_inf = freestream(mach)
    x0, y0, lx, ly = -3.0, -6.0, 3.0, 12.0
    nx = int(_round(lx / h)) + 1
    ny = int(_round(ly / h)) + 1
    grid = GridInfo(nx, ny, h, h, x0, y0)
    pts = [(-3.0, -6.0), (0.0, -6.0)]
    bcs = [BCType.FarField(u_inf)]
    pts.append((0.0, -1.0 + shift))
    bcs.append(BCType.FarField(u_inf))
    n_arc = 360
    arc_start = len(bcs)
    for k in range(1, n_arc + 1):
        s = float(k) / float(n_arc)
        theta = -0.5 * math.pi - math.pi * s
        pts.append((math.cos(theta), math.sin(theta) + shift))
        bcs.append(BCType.ReflectiveWall())
    arc_end = len(bcs) - 1
    arc = CircularArc.from_three_points((0.0, -1.0 + shift), (-1.0, 0.0 + shift), (0.0, 1.0 + shift), FLUID_OUTSIDE)
    pts.append((0.0, 6.0))
    bcs.append(BCType.FarField(u_inf))
    pts.append((-3.0, 6.0))
    bcs.append(BCType.FarField(u_inf))
    bcs.append(BCType.FarField(u_inf))
    f = Field(grid, [BCType.Wall()] * 4, bcs, np.zeros(6), Polygon(pts, FLUID_INSIDE), _dummy_inner(), 0.0,
              params=params)
    f.outer_arcs.append(ArcOverride(arc_start, arc_end, arc))
    f.value[f.fluid] = u_inf
    return f


def init_double_mach(h=1.0 / 320.0, params=None):
    sqrt3 = math.sqrt(3.0)
    a = (-0.5 - sqrt3 / 12.0, 0.0)
    b = (0.0, 0.0)
    c = (23.0 * sqrt3 / 12.0, 23.0 / 12.0)
    d = (c[0], 23.0 / 12.0 + sqrt3 / 2.0)
    e = (a[0], d[1])
    x0, y0, lx, ly = a[0], 0.0, c[0] - a[0], d[1]
    nx = int(math.ceil(lx / h)) + 1
    ny = int(math.ceil(ly / h)) + 1
    grid = GridInfo(nx, ny, h, h, x0, y0)
    pre = euler_to_three_energy(1.4, 0.0, 0.0, 1.0, 1.4)
    post = euler_to_three_energy(8.0, 8.25, 0.0, 116.5, 1.4)
    bcs = [BCType.Constant(post), BCType.Wall(), BCType.Constant(pre), BCType.ZerothOrder(), BCType.Constant(post)]
    f = Field(grid, [BCType.Wall()] * 4, bcs, np.zeros(6), Polygon([a, b, c, d, e], FLUID_INSIDE), _dummy_inner(),
              0.0, params=params)
    for i in range(nx):
        row = np.arange(ny) + i * ny
        fl = f.fluid[row]
        f.value[row[fl]] = post if grid.x(i) <= 0.0 else pre
    return f


def _solve_temperature(target, ce, ci, cr, rho, P):
    def fn(T):
        te, ti, tr = ce * T, ci * T, cr * T
        return P.cve * te + P.cvi * ti + P.a_rad * ((tr * tr) * (tr * tr)) / rho - target

    lo, hi = 0.0, 1.0
    while fn(hi) < 0.0:
        hi *= 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if fn(mid) < 0.0:
            lo = mid
        else:
            hi = mid
        if hi - lo <= 0.0:
            break
    return 0.5 * (lo + hi)


def _three_temp_state(rho, u, v, te, ti, tr, P):
    e_e, e_i, e_r = P.cve * te, P.cvi * ti, P.a_rad * ((tr * tr) * (tr * tr)) / rho
    k = rho * (u * u + v * v) / 6.0
    return np.array([rho, rho * u, rho * v, rho * e_e + k, rho * e_i + k, rho * e_r + k])


def planar_shock(nx=1024, ny=8, lx=4.0, ly=0.03125, x_shock=1.0, mach=2.0, sigma=0.25, params=None):
    """Mach-`mach` shock at x_shock moving into (rho, u, p) = (1, 0, 1),
    gamma = 1.4 Rankine-Hugoniot on the total energy; pre-shock
    Te = Ti = Tr, post-shock Te:Ti:Tr = 1 : 1.5 : 0.8. Bottom/top Periodic,
    right Outflow(p_inf = 1, sigma, l_domain = lx), left FarField(post)."""
    P = params if params is not None else Params(periodic_ly=ly)
    grid = GridInfo(nx, ny, lx / float(nx), ly / float(ny), 0.0, 0.0)
    g, rho1, u1, p1 = 1.4, 1.0, 0.0, 1.0
    c1 = math.sqrt(g * p1 / rho1)
    m2 = mach * mach
    rho2 = rho1 * (g + 1.0) * m2 / ((g - 1.0) * m2 + 2.0)
    p2 = p1 * (2.0 * g * m2 - (g - 1.0)) / (g + 1.0)
    ws = mach * c1
    u2 = ws * (1.0 - rho1 / rho2)
    t1 = _solve_temperature(p1 / ((g - 1.0) * rho1), 1.0, 1.0, 1.0, rho1, P)
    t2 = _solve_temperature(p2 / ((g - 1.0) * rho2), 1.0, 1.5, 0.8, rho2, P)
    pre = _three_temp_state(rho1, u1, 0.0, t1, t1, t1, P)
    post = _three_temp_state(rho2, u2, 0.0, t2, 1.5 * t2, 0.8 * t2, P)
    bcs = [BCType.Periodic(), BCType.Outflow(p1, sigma, lx), BCType.Periodic(), BCType.FarField(post)]
    f = Field(grid, [BCType.Wall()] * 4, bcs, np.zeros(6), Polygon([(0.0, 0.0), (lx, 0.0), (lx, ly), (0.0, ly)],
                                                                  FLUID_INSIDE), _dummy_inner(), 0.0, params=P)
    for i in range(nx):
        row = np.arange(ny) + i * ny
        fl = f.fluid[row]
        f.value[row[fl]] = post if grid.x(i) < x_shock else pre
    return f


def rect_field(nx, ny, lx, ly, value, kind=BCType.WALL, params=None):
    grid = GridInfo(nx, ny, lx / float(nx), ly / float(ny), 0.0, 0.0)
    b = BCType(kind, state=value)
    return Field(grid, [BCType.Wall()] * 4, [b] * 4, value,
                 Polygon([(0.0, 0.0), (lx, 0.0), (lx, ly), (0.0, ly)], FLUID_INSIDE), _dummy_inner(), 0.0,
                 params=params)


def _round(v):
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


# ------------------------------------------------------------------ batched workloads
BATCH_SEED = 20261203
BATCH_SIZES = (61, 91, 121)
OMEGA_BASE = 1.0  # the reference's exchange coefficients are 0 (constant.rs); the scaled base is 1


class Lcg:
    """main.rs:493-498: 64-bit LCG, uniform doubles in [0, 1) from the top 53 bits."""

    MASK = (1 << 64) - 1

    def __init__(self, seed):
        self.state = int(seed) & self.MASK

    def uniform(self):
        self.state = (self.state * 6364136223846793005 + 1442695040888963407) & self.MASK
        return float(self.state >> 11) / float(1 << 53)


def batch_specs(n=256, seed=BATCH_SEED, sizes=BATCH_SIZES, mach=(2.0, 4.0), omega_scale=(0.1, 10.0),
                omega_base=OMEGA_BASE):
    """n half-cylinder instances: nx uniform over `sizes` (ny = 4 (nx - 1) + 1,
    square cells h = 3 / (nx - 1)), inflow Mach uniform in `mach`, electron-ion
    and electron-radiation exchange coefficients log-uniform in `omega_scale`
    times `omega_base`. Draw order per instance: size, Mach, omega_ei, omega_er."""
    rng = Lcg(seed)
    lo, hi = math.log(omega_scale[0]), math.log(omega_scale[1])
    out = []
    for _ in range(n):
        nx = sizes[min(int(rng.uniform() * len(sizes)), len(sizes) - 1)]
        m = mach[0] + (mach[1] - mach[0]) * rng.uniform()
        oei = omega_base * math.exp(lo + (hi - lo) * rng.uniform())
        oer = omega_base * math.exp(lo + (hi - lo) * rng.uniform())
        out.append(dict(nx=nx, ny=4 * (nx - 1) + 1, h=3.0 / (nx - 1), mach=m, omega_ei=oei, omega_er=oer))
    return out


def batch_field(spec):
    """The half-cylinder Field of one batch_specs entry."""
    return init_cylinder(h=spec["h"], mach=spec["mach"],
                         params=Params(omega_ei=spec["omega_ei"], omega_er=spec["omega_er"]))


# ------------------------------------------------------------------ adjoint objective
class SurfacePressure:
    """J(u) = h * sum over the ghosts of the arc sides of p(u[n_g]), n_g the
    fluid node nearest to the ghost's boundary foot P0 (among the 3 x 3 nodes
    around its rounded grid index), p = p_e + p_i + p_r (state.rs:245-276) and
    h = sqrt(dx dy): the surface pressure integral on the cylinder, each
    ghost standing for one arc element of length h."""

    def __init__(self, field, ghosts, arc=0):
        g = field.grid
        a = field.outer_arcs[arc]
        sel = (ghosts.boundary == 0) & (ghosts.side >= a.side_start) & (ghosts.side <= a.side_end)
        nodes = []
        for p0x, p0y in ghosts.proj[sel, :2]:
            ic, jc = _round((p0x - g.x0) / g.dx), _round((p0y - g.y0) / g.dy)
            best, bn = math.inf, None
            for di in (0, -1, 1):
                for dj in (0, -1, 1):
                    i, j = int(ic) + di, int(jc) + dj
                    if 0 <= i < g.nx and 0 <= j < g.ny and field.fluid[i * g.ny + j]:
                        d2 = (g.x0 + i * g.dx - p0x) ** 2 + (g.y0 + j * g.dy - p0y) ** 2
                        if d2 < best:
                            best, bn = d2, i * g.ny + j
            if bn is None:
                raise ValueError("arc ghost without a fluid node near its foot")
            nodes.append(bn)
        self.nodes = np.array(nodes, np.int64)
        self.h = math.sqrt(g.dx * g.dy)
        P = field.params
        self.g3 = np.array([P.gamma_e - 1.0, P.gamma_i - 1.0, P.gamma_r - 1.0])

    def value(self, u):
        s = np.asarray(u)[self.nodes]
        rw2 = (s[:, 1] ** 2 + s[:, 2] ** 2) / s[:, 0]
        p = (self.g3[None, :] * (s[:, 3:6] - rw2[:, None] / 6.0)).sum(1)
        return self.h * p.sum()

    def grad(self, u):
        u = np.asarray(u)
        s = u[self.nodes]
        G = self.g3.sum()
        gp = np.zeros_like(s)
        gp[:, 0] = G * (s[:, 1] ** 2 + s[:, 2] ** 2) / (6.0 * s[:, 0] ** 2)
        gp[:, 1] = -G * s[:, 1] / (3.0 * s[:, 0])
        gp[:, 2] = -G * s[:, 2] / (3.0 * s[:, 0])
        gp[:, 3:6] = self.g3[None, :]
        out = np.zeros_like(u)
        np.add.at(out, self.nodes, self.h * gp)
        return out
