"""Generate the oracle fixtures under tests/golden/ (run from the repo root:
`python tests/golden/make_golden.py`).

The reference ships no whole-run outputs and cannot be built on this image,
so these fixtures are produced by the oracle (the CPU restatement). They pin
the oracle against regressions and give the GPU tests committed vectors:

  cyl31x121.npz   half-cylinder at h = 1/10 (31 x 121 nodes): fluid mask,
                  initial state, l() of the initial state (rhs and ghost
                  values), the state after 10 SSP-RK3 steps and the 10 dts
  planar256x8.npz planar shock 256 x 8 on [0, 1] x [0, 0.03125] with
                  diffusion and exchange on: initial state, state after 20
                  steps and the 20 dts
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

PLANAR = dict(nx=256, ny=8, lx=1.0, ly=0.03125, x_shock=0.25, mach=2.0, sigma=0.25)
PLANAR_PARAMS = dict(kappa_e=1e-3, kappa_i=1e-3, kappa_r=1e-3, omega_ei=1.0, omega_er=1.0, periodic_ly=0.03125)


def make():
    from oracle import oracle as O
    c = O.Case.cylinder(h=0.1)
    u0 = c.state()
    rhs, gv = c.l()
    dts = c.run(10, 0.05)
    np.savez_compressed(os.path.join(HERE, "cyl31x121.npz"), fluid=c.fluid(), u0=u0, rhs0=rhs, ghosts0=gv,
                        u10=c.state(), dts=dts, t10=np.array([c.time]))
    p = O.Case.planar_shock(**PLANAR, **PLANAR_PARAMS)
    u0 = p.state()
    dts = p.run(20, 0.05)
    np.savez_compressed(os.path.join(HERE, "planar256x8.npz"), fluid=p.fluid(), u0=u0, u20=p.state(), dts=dts)


if __name__ == "__main__":
    make()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")
