"""Adjoint of l() and of the SSP-RK3 time loop (rh3t_l_vjp,
rh3t_adjoint_forward / rh3t_adjoint_backward).

  - operator level, against the oracle's dual-number run of the reference
    l() (oracle/src/jvp.hpp) on the 31 x 121 half-cylinder: for random
    cotangents rbar and directions du (state), du_inf (FarField state) and
    domega (exchange coefficients), <rbar, J du> = <J^T rbar, du> to a
    relative 1e-9 (no-contraction build: both sides take the same branches at
    the kinks; the derivatives of the WENO weights, ~(eps + beta)^-3, amplify
    the adjoint's own roundings to ~1e-10 of the sum);
  - time loop, against FP64 central finite differences (h = 1e-6 relative)
    of J = surface pressure on the arc (cases.SurfacePressure) after N steps,
    with respect to the inflow Mach number and the two exchange coefficients
    (1e-5), and the initial state in directions near the cylinder (O(h)
    convergence near the shock);
  - Wall (ILW) and Outflow (LODI) ghosts: the operator vjp against the
    dual-number oracle on double Mach and the planar shock, and the time
    loop's gradient against central differences;
  - a batch's gradients equal those of its instances run alone.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OMEGA = dict(omega_ei=0.5, omega_er=2.0)


def _dev_state(rh, O, steps=10, h=0.1, **kw):
    """A developed 31 x 121 state from the oracle and the same Field."""
    ref = O.Case.cylinder(h=h, **kw)
    ref.run(steps, 0.05)
    f = rh.cases.init_cylinder(h=h, params=rh.Params(**kw))
    f.value[:] = ref.state()
    f.time = ref.time
    return f, ref


@pytest.mark.parametrize("which", ["state", "farfield", "omega"])
def test_l_vjp_matches_dual_oracle(rh, O, which):
    f, ref = _dev_state(rh, O, **OMEGA)
    g = rh.GhostGrid.build(f)
    b = rh.Batch([f], [g], exact=True)
    rng = np.random.default_rng(7)
    fl = f.fluid
    scale = np.abs(f.value[fl]).mean(0)
    rbar = rng.standard_normal(f.value.shape) * fl[:, None]
    du = rng.standard_normal(f.value.shape) * scale * fl[:, None] if which == "state" else None
    duinf = rng.standard_normal(6) if which == "farfield" else None
    dom = rng.standard_normal(2) if which == "omega" else None
    _, jdu, _, _ = ref.l_jvp(du, duinf, dom)
    lhs = float((rbar * jdu).sum())
    ub, pb = b.l_vjp(0, rbar)
    rhs = 0.0
    if du is not None:
        rhs += float((ub * du).sum())
    if duinf is not None:
        rhs += float(pb[:6] @ duinf)
    if dom is not None:
        rhs += float(pb[6:] @ dom)
    print(f"{which}: <rbar, J du> = {lhs:.15e}, <J^T rbar, du> = {rhs:.15e}")
    assert abs(lhs - rhs) <= 1e-9 * max(abs(lhs), 1e-300)


def test_l_vjp_fma_build_close(rh, O):
    """The FMA build takes other branches where a kink argument is zero up to
    rounding (|v| on the FarField corners, max/min of velocities): its vjp
    differs there locally, so the two builds are compared in norm. The
    adjoint the bench times is the no-contraction build's, the one held to
    the dual-number oracle (1e-9 above) and to central differences at
    121x481 after 200 steps (tests/test_gpu_configs.py)."""
    f, _ = _dev_state(rh, O, **OMEGA)
    g = rh.GhostGrid.build(f)
    rbar = np.random.default_rng(3).standard_normal(f.value.shape) * f.fluid[:, None]
    ue, pe = rh.Batch([f], [g], exact=True).l_vjp(0, rbar)
    uf, pf = rh.Batch([f], [g], exact=False).l_vjp(0, rbar)
    rel = np.linalg.norm(uf - ue) / np.linalg.norm(ue)
    print(f"FMA vs exact vjp: relative L2 difference {rel:.3e}, parameters {np.abs(pf - pe).max():.3e}")
    assert rel <= 1e-2
    assert np.abs(pf - pe).max() <= 1e-4 * np.abs(pe).max()


PLANAR = dict(kappa_e=1e-3, kappa_i=1e-3, kappa_r=1e-3, omega_ei=1.0, omega_er=1.0, periodic_ly=0.03125)


def _wall_outflow_case(rh, O, case, steps):
    """A developed oracle state and the same Field: double Mach (Wall ILW
    ghosts on the wedge, Constant, TimeDependent, ZerothOrder) or the planar
    shock (Outflow LODI at x = 4, FarField, Periodic, diffusion + exchange)."""
    if case == "double_mach":
        ref = O.Case.double_mach(h=1.0 / 40.0)
        f = rh.cases.init_double_mach(h=1.0 / 40.0)
    else:
        ref = O.Case.planar_shock(nx=256, **PLANAR)
        f = rh.cases.planar_shock(nx=256, params=rh.Params(**PLANAR))
    ref.run(steps, 0.05)
    f.value[:] = ref.state()
    f.time = ref.time
    return f, ref


@pytest.mark.parametrize("case", ["double_mach", "planar"])
def test_l_vjp_wall_outflow_matches_dual_oracle(rh, O, case):
    """Wall (two ILW solves) and Outflow (LODI row) ghosts in reverse:
    <rbar, J du> = <J^T rbar, du> against the oracle's dual-number l(), with
    du on the E_r stencils and nearest nodes of the Wall (double Mach: 536
    of 1864 ghosts) or Outflow (planar: 32) ghosts and rbar on the cells
    those ghosts reach, so that their rows carry the products. Measured:
    4.9e-10 (Wall; the ILW solves and the WENO weights near the reflected
    shock amplify the rounding of both sides) and 4e-16 (Outflow)."""
    f, ref = _wall_outflow_case(rh, O, case, 10)
    g = rh.GhostGrid.build(f)
    kind = rh.BCType.Wall().kind if case == "double_mach" else rh.BCType.Outflow(1.0, 1.0, 1.0).kind
    bcs = (f.bc_outer, f.bc_inner)
    sel = [k for k in range(g.len()) if g.pre[k] >= 0 and int(bcs[g.boundary[k]][g.side[k]].kind) == kind]
    assert sel
    ny = f.grid.ny
    nodes = np.unique(np.concatenate([g.stencil[g.pre[k]].astype(np.int64) for k in sel] +
                                     [[g.nearest[g.pre[k]][0] * ny + g.nearest[g.pre[k]][1]] for k in sel]))
    reach = np.zeros(f.grid.len(), bool)
    for k in sel:
        i, j = g.idx[k]
        for d in range(-4, 5):
            for a, c in ((i + d, j), (i, j + d)):
                if 0 <= a < f.grid.nx and 0 <= c < ny:
                    reach[a * ny + c] = True
    reach &= f.fluid
    b = rh.Batch([f], [g], exact=True)
    rng = np.random.default_rng(3)
    scale = np.abs(f.value[f.fluid]).mean(0)
    du = np.zeros(f.value.shape)
    du[nodes] = rng.standard_normal((len(nodes), 6)) * scale
    du *= f.fluid[:, None]
    rbar = rng.standard_normal(f.value.shape) * reach[:, None]
    _, jdu, _, _ = ref.l_jvp(du, None, None)
    lhs = float((rbar * jdu).sum())
    ub, _ = b.l_vjp(0, rbar)
    rhs = float((ub * du).sum())
    print(f"{case}: <rbar, J du> = {lhs:.15e}, <J^T rbar, du> = {rhs:.15e}")
    assert abs(lhs - rhs) <= 1e-8 * max(abs(lhs), 1e-300)


@pytest.mark.parametrize("case", ["double_mach", "planar"])
def test_wall_outflow_loop_gradient_vs_finite_differences(rh, O, case):
    """The checkpointed time loop over Wall / Outflow ghosts: the gradient of
    a linear functional J = <w, u_N> after N steps, in a random smooth
    direction of the initial state, against FP64 central differences."""
    f, _ = _wall_outflow_case(rh, O, case, 10)
    g = rh.GhostGrid.build(f)
    N = 6
    rng = np.random.default_rng(5)
    fl = f.fluid
    w = rng.standard_normal(f.value.shape) * fl[:, None]
    gr = f.grid
    x = gr.x0 + gr.dx * (np.arange(gr.len()) // gr.ny)
    y = gr.y0 + gr.dy * (np.arange(gr.len()) % gr.ny)
    bump = (1.0 + 0.5 * np.sin(3.0 * x) * np.cos(2.0 * y)) * fl
    delta = f.value * bump[:, None] * 1e-3
    u0 = f.value.copy()

    def J(eps):
        f.value[:] = u0 + eps * delta
        b = rh.Batch([f], [g], exact=True)
        b.advance(N, 0.05)
        u, _ = b.download(0)
        b.close()
        return float((w * u).sum())

    f.value[:] = u0
    b = rh.Batch([f], [g], exact=True)
    b.adjoint_forward(N, 0.05, ckpt_every=4)
    g0, _ = b.adjoint_backward([w])
    b.close()
    adj = float((g0[0] * delta).sum())
    fd = (J(1e-6) - J(-1e-6)) / 2e-6
    print(f"{case}: adjoint {adj:.12e} central difference {fd:.12e}")
    assert abs(adj - fd) <= 1e-5 * abs(fd)


def _objective(rh, mach, oei, oer, nsteps, u0=None, delta=None, eps=0.0, h=0.1):
    f = rh.cases.init_cylinder(h=h, mach=mach, params=rh.Params(omega_ei=oei, omega_er=oer))
    if u0 is not None:
        f.value[:] = u0
    if delta is not None:
        f.value[:] = f.value + eps * delta
    g = rh.GhostGrid.build(f)
    J = rh.cases.SurfacePressure(f, g)
    b = rh.Batch([f], [g], exact=True)
    b.advance(nsteps, 0.05)
    u, _ = b.download(0)
    return J.value(u), f, g, J


def _fd(fun, x, rel=1e-6):
    h = rel * abs(x)
    return (fun(x + h) - fun(x - h)) / (2.0 * h)


def test_gradient_vs_finite_differences(rh):
    mach, oei, oer, N = 3.0, 0.5, 2.0, 12
    J0, f, g, J = _objective(rh, mach, oei, oer, N)
    b = rh.Batch([f], [g], exact=True)
    b.adjoint_forward(N, 0.05, ckpt_every=5, max_records=1)  # two of the three segments recomputed
    assert b.adjoint_records() == 1
    uN, _ = b.download(0)
    assert abs(J.value(uN) - J0) <= 1e-14 * abs(J0)
    g0, gp = b.adjoint_backward([J.grad(uN)])
    # Mach: the FarField state and the initial state are both u_inf(M)
    hm = 1e-7
    dudm = (rh.cases.freestream(mach + hm) - rh.cases.freestream(mach - hm)) / (2 * hm)
    adj_m = float(gp[0, :6] @ dudm) + float((g0[0][f.fluid] @ dudm).sum())
    fd_m = _fd(lambda m: _objective(rh, m, oei, oer, N)[0], mach)
    adj_ei, adj_er = gp[0, 6], gp[0, 7]
    fd_ei = _fd(lambda o: _objective(rh, mach, o, oer, N)[0], oei)
    fd_er = _fd(lambda o: _objective(rh, mach, oei, o, N)[0], oer)
    print(f"dJ/dM adj {adj_m:.10e} fd {fd_m:.10e}; dJ/domega_ei adj {adj_ei:.10e} fd {fd_ei:.10e}; "
          f"dJ/domega_er adj {adj_er:.10e} fd {fd_er:.10e}")
    assert abs(adj_m - fd_m) <= 1e-5 * abs(fd_m)
    assert abs(adj_ei - fd_ei) <= 1e-5 * max(abs(fd_ei), 1e-3 * abs(fd_m))
    assert abs(adj_er - fd_er) <= 1e-5 * max(abs(fd_er), 1e-3 * abs(fd_m))


@pytest.mark.parametrize("comp", ["density_energy", "momentum"])
def test_initial_state_gradient_vs_finite_differences(rh, O, comp):
    """A smooth bump behind the bow shock, from a developed state. Near the
    shock the discrete operator is not smooth (WENO weights, kinks), so the
    central difference converges to the adjoint only at O(h): it must agree
    to 1e-4 at h = 1e-6 and to 2e-5 at h = 1e-7, and come closer as h
    shrinks."""
    mach, oei, oer, N = 3.0, 0.5, 2.0, 8
    f, _ = _dev_state(rh, O, steps=30, **OMEGA)
    gr = f.grid
    x = gr.x0 + gr.dx * (np.arange(gr.len()) // gr.ny)
    y = gr.y0 + gr.dy * (np.arange(gr.len()) % gr.ny)
    bump = np.exp(-((x + 0.5) ** 2 + (y - 1.4) ** 2) / 0.05) * f.fluid
    delta = np.zeros_like(f.value)
    if comp == "density_energy":
        delta[:, 0] = bump * f.value[:, 0]
        delta[:, 3:6] = bump[:, None] * f.value[:, 3:6]
    else:
        delta[:, 1] = 0.3 * bump
        delta[:, 2] = 0.3 * bump
    u0 = f.value.copy()
    _, _, g, J = _objective(rh, mach, oei, oer, N, u0=u0)
    b = rh.Batch([f], [g], exact=True)
    b.adjoint_forward(N, 0.05, ckpt_every=3)
    uN, _ = b.download(0)
    g0, _ = b.adjoint_backward([J.grad(uN)])
    adj = float((g0[0] * delta).sum())

    def fd(e):
        return (_objective(rh, mach, oei, oer, N, u0, delta, e)[0] -
                _objective(rh, mach, oei, oer, N, u0, delta, -e)[0]) / (2 * e)

    f5, f6, f7 = fd(1e-5), fd(1e-6), fd(1e-7)
    print(f"dJ/du0 . delta ({comp}): adj {adj:.10e} fd(1e-5) {f5:.10e} fd(1e-6) {f6:.10e} fd(1e-7) {f7:.10e}")
    assert abs(adj - f6) <= 1e-4 * abs(f6)
    assert abs(adj - f7) <= 2e-5 * abs(f7)
    assert abs(adj - f7) < abs(adj - f5)


def test_batch_adjoint_equals_single(rh):
    specs = rh.cases.batch_specs(n=3, sizes=(31, 41))
    fields = [rh.cases.batch_field(sp) for sp in specs]
    grids = [rh.GhostGrid.build(f) for f in fields]
    Js = [rh.cases.SurfacePressure(f, g) for f, g in zip(fields, grids)]
    b = rh.Batch(fields, grids, exact=True)
    b.adjoint_forward(6, 0.05, ckpt_every=4)
    res = b.download()
    g0, gp = b.adjoint_backward([J.grad(u) for J, (u, _) in zip(Js, res)])
    for k, (f, g, J) in enumerate(zip(fields, grids, Js)):
        s = rh.Batch([f], [g], exact=True)
        s.adjoint_forward(6, 0.05, ckpt_every=4)
        u, _ = s.download(0)
        assert np.array_equal(u, res[k][0])
        a0, ap = s.adjoint_backward([J.grad(u)])
        # atomic accumulation: the order of the additions differs between runs
        assert np.abs(a0[0] - g0[k]).max() <= 1e-10 * np.abs(a0[0]).max()
        assert np.abs(ap[0] - gp[k]).max() <= 1e-10 * np.abs(ap[0]).max()


def test_segment_records_do_not_change_the_gradient(rh):
    """The forward run keeps the records of its last segments (as many as
    fit, or a given cap) so the reverse sweep skips their recomputation:
    the gradients are those of the sweep that recomputes all but the last."""
    specs = rh.cases.batch_specs(n=2, sizes=(31,))
    fields = [rh.cases.batch_field(sp) for sp in specs]
    grids = [rh.GhostGrid.build(f) for f in fields]
    Js = [rh.cases.SurfacePressure(f, g) for f, g in zip(fields, grids)]
    out = {}
    for cap in (1, 2, 0):
        b = rh.Batch(fields, grids, exact=True)
        b.adjoint_forward(10, 0.05, ckpt_every=3, max_records=cap)
        res = b.download()
        out[cap] = (b.adjoint_records(),) + b.adjoint_backward([J.grad(u) for J, (u, _) in zip(Js, res)])
        b.close()
    assert out[1][0] == 1 and out[2][0] == 2 and out[0][0] == 4  # 4 segments, all fit
    for cap in (2, 0):
        for k in range(2):
            a0, b0 = out[1][1][k], out[cap][1][k]
            assert np.abs(a0 - b0).max() <= 1e-10 * np.abs(a0).max()
        assert np.abs(out[1][2] - out[cap][2]).max() <= 1e-10 * np.abs(out[1][2]).max()
