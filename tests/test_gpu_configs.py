"""The benchmark configurations at their stated sizes and step counts, in the
no-contraction build (the benched build), against the oracle.

  - the Mach-3 half-cylinder at scale: h = 1/160 (481 x 1921 nodes), one l()
    of a developed state and 20 SSP-RK3 steps; h = 1/320 (961 x 3841 nodes),
    one l() of a developed state;
  - the Mach-2 planar shock (1024 x 8, y-periodic, FarField and Outflow,
    diffusion and exchange on) for the full 500 steps;
  - the gradient of J (surface pressure on the arc) after 200 steps of the
    121 x 481 half-cylinder (checkpoints every 20) in the inflow Mach number
    and both exchange coefficients, against FP64 central differences with
    h = 1e-6 relative, for seeded instances advanced as a batch.

Parity tolerance: normwise relative L-infinity per field over fluid nodes
(tests/helpers.py rel_linf) <= 1e-10 against the oracle, and against the
oracle built with the correctly rounded power the CUDA path uses
(O.crpow_variant(); the only arithmetic in which it differs from the plain
oracle is the reference's two libm pow calls)."""
import numpy as np
import pytest

from helpers import rel_linf

pytestmark = pytest.mark.gpu

PLANAR = dict(kappa_e=1e-3, kappa_i=1e-3, kappa_r=1e-3, omega_ei=1.0, omega_er=1.0, periodic_ly=0.03125)


def _check(u, refs, fluid, tol, label):
    errs = {name: rel_linf(u, r, fluid).max() for name, r in refs.items()}
    print(f"{label}: " + ", ".join(f"vs {k} {v:.3e}" for k, v in errs.items()))
    for v in errs.values():
        assert v <= tol
    return errs


@pytest.mark.parametrize("h,steps_before,run_steps", [(1.0 / 160.0, 10, 20), (1.0 / 320.0, 4, 0)])
def test_half_cylinder_at_scale(rh, O, h, steps_before, run_steps):
    OC = O.crpow_variant()
    ref, refc = O.Case.cylinder(h=h), OC.Case.cylinder(h=h)
    refc.run(steps_before, 0.05)
    f = rh.cases.init_cylinder(h=h)
    f.value[:] = refc.state()
    f.time = refc.time
    ref.set_state(refc.state())
    ref.time = refc.time
    g = rh.GhostGrid.build(f)
    s = rh.Solver(f, g, exact=True)
    rhs, gv = s.l(with_ghosts=True)
    r1, g1 = ref.l()
    r2, g2 = refc.l()
    label = f"{f.grid.nx}x{f.grid.ny} l()"
    _check(rhs, {"oracle": r1, "oracle_crpow": r2}, f.fluid, 1e-10, label + " rhs")
    allg = np.ones(len(g1), bool)
    _check(gv, {"oracle": g1, "oracle_crpow": g2}, allg, 1e-10, label + " ghosts")
    if run_steps:
        s.advance(run_steps, 0.05)
        ref.run(run_steps, 0.05)
        refc.run(run_steps, 0.05)
        u, t = s.download()
        _check(u, {"oracle": ref.state(), "oracle_crpow": refc.state()}, f.fluid, 1e-10,
               f"{f.grid.nx}x{f.grid.ny} {run_steps} steps")
        assert abs(t - refc.time) <= 1e-12 * refc.time
    s.close()


def test_planar_shock_500_steps(rh, O):
    OC = O.crpow_variant()
    f = rh.cases.planar_shock(params=rh.Params(**PLANAR))
    ref, refc = O.Case.planar_shock(**PLANAR), OC.Case.planar_shock(**PLANAR)
    assert np.array_equal(f.value, ref.state())
    g = rh.GhostGrid.build(f)
    s = rh.Solver(f, g, exact=True)
    s.advance(500, 0.05)
    ref.run(500, 0.05)
    refc.run(500, 0.05)
    u, t = s.download()
    _check(u, {"oracle": ref.state(), "oracle_crpow": refc.state()}, f.fluid, 1e-10, "planar 1024x8 500 steps")
    assert abs(t - ref.time) <= 1e-12 * ref.time
    s.close()


def _fd(fun, x, rel=1e-6):
    h = rel * abs(x)
    return (fun(x + h) - fun(x - h)) / (2.0 * h)


def test_config5_gradient_121x481_200_steps(rh):
    """Two seeded 121 x 481 instances (Mach U[2,4], exchange coefficients
    log-U[0.1,10]) advanced as one batch for 200 steps with checkpoints every
    20; each instance's gradient against central differences of its own J."""
    N, CK = 200, 20
    specs = rh.cases.batch_specs(2, sizes=(121,))
    fields = [rh.cases.batch_field(sp) for sp in specs]
    grids = [rh.GhostGrid.build(f) for f in fields]
    Js = [rh.cases.SurfacePressure(f, g) for f, g in zip(fields, grids)]
    b = rh.Batch(fields, grids, exact=True)
    b.adjoint_forward(N, 0.05, ckpt_every=CK)
    res = b.download()
    g0, gp = b.adjoint_backward([J.grad(u) for J, (u, _) in zip(Js, res)])
    b.close()

    def objective(k, **change):
        sp = dict(specs[k])
        sp.update(change)
        f = rh.cases.batch_field(sp)
        s = rh.Batch([f], [grids[k]], exact=True)
        s.advance(N, 0.05)
        u, _ = s.download(0)
        s.close()
        return Js[k].value(u)

    for k, sp in enumerate(specs):
        hm = 1e-7
        dudm = (rh.cases.freestream(sp["mach"] + hm) - rh.cases.freestream(sp["mach"] - hm)) / (2 * hm)
        adj_m = float(gp[k, :6] @ dudm) + float((g0[k][fields[k].fluid] @ dudm).sum())
        fd_m = _fd(lambda m: objective(k, mach=m), sp["mach"])
        fd_ei = _fd(lambda o: objective(k, omega_ei=o), sp["omega_ei"])
        fd_er = _fd(lambda o: objective(k, omega_er=o), sp["omega_er"])
        adj_ei, adj_er = gp[k, 6], gp[k, 7]
        print(f"instance {k} M={sp['mach']:.4f}: dJ/dM adj {adj_m:.10e} fd {fd_m:.10e}; "
              f"dJ/domega_ei adj {adj_ei:.10e} fd {fd_ei:.10e}; dJ/domega_er adj {adj_er:.10e} fd {fd_er:.10e}")
        assert abs(adj_m - fd_m) <= 1e-5 * abs(fd_m)
        assert abs(adj_ei - fd_ei) <= 1e-5 * max(abs(fd_ei), 1e-3 * abs(fd_m))
        assert abs(adj_er - fd_er) <= 1e-5 * max(abs(fd_er), 1e-3 * abs(fd_m))
