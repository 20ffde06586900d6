"""Algorithmic FLOP model of one SSP-RK3 step (for the roofline).

Counts are the reference algorithm's value-dependent floating-point
operations (add, sub, mul, div, sqrt, pow, fabs, fmin, fmax = 1 each), taken
from an operation-counting instantiation of the oracle's templated pointwise
functions (tests/test_flops.py re-derives them):

  FACE_FLUX      weno.rs:685-802 reconstruction_fast incl. its six physical
                 fluxes (state.rs:56-85)                         per face
  DERIVED        state.rs:245-276                                per node and stage
  NONCON_DIR     noncon.rs:288-332, one direction               per cell and stage
  DIFFUSION      diffusion.rs:27-50                              per face (if on)
  SOURCE         source.rs:7-21                                  per cell (if on)
  LOCAL_DT       dt.rs:5-34                                      per cell and step
  BUILD_L/R      weno.rs:28-459 / 484-548

The heavy ghost (Wall / Outflow / FarField, bc1.rs:193-255 + 690-924) is
counted for one pass over its data (the reference repeats the pass for each
k = 0..4; the repeats compute nothing new and are not algorithmic work).
"""

FACE_FLUX = 2299
DERIVED = 40
NONCON_DIR = 309
DIFFUSION = 57
SOURCE = 50
LOCAL_DT = 72
BUILD_L = 240
BUILD_R = 85

# per-cell RHS assembly (main.rs:268-302): 2 directions x 6 components x
# (sub, mul) + 1 add, plus +ncx +ncy on three components
RHS_ASSEMBLY = 6 * (2 + 2 + 1) + 3 * 2
# stage updates (main.rs:308-349): RK1 6x(mul+add), RK2/RK3 6x(3 mul + 2 add);
# admissibility (main.rs:24-33): 2 div, 2 mul, 1 add, 1 div, 3 div, 3 sub
STAGE = (12 + 30 + 30) / 3.0 + 12


def heavy_ghost_flops(kind="far_field"):
    """One heavy ghost, one stage."""
    rotate_derived_lr = 6 + DERIVED + BUILD_L + BUILD_R
    data = 55 * (6 + 6 * 11)                    # rotate momentum, L.u6 for 6 characteristics
    beta = 6 * (2 * 979 + 2 * 55)               # d^T S_r d, r = 0..4
    vk = 6 * 2 * 225                            # w_{r,k} . d
    weights = 6 * (5 * 4 + 5 * 5 * 3)           # alpha_r, sum, normalised sums per k
    post = {"far_field": 72 + 5 * 72 + 6, "outflow": 5 * 72 + 30, "wall": 2 * 200 + 3 * 72}[kind]
    taylor = 4 * (2 + 12) + 6
    return rotate_derived_lr + data + beta + vk + weights + post + taylor


# Algorithmic HBM bytes of one heavy ghost per stage: its GhostBC tables
# (bc1.rs:50-57: S_0..S_4 979, w 225, d 5 doubles; the E_r stencil as 55
# 4-byte node indices), which no cache holds across stages at scale, plus the
# ghost value written (6 doubles). The stencil states are shared with the
# neighbouring ghosts and cells and are not counted.
HEAVY_GHOST_BYTES = (979 + 225 + 5) * 8 + 55 * 4 + 6 * 8


def ghost_launch_bytes(n_heavy):
    """Algorithmic bytes of one stage's ghost update (heavy ghosts' tables)."""
    return n_heavy * HEAVY_GHOST_BYTES


def step_flops(n_fluid, n_xfaces, n_yfaces, n_ghosts, n_heavy, diffusion=False, source=False):
    """Algorithmic FLOPs of one RK3 step (3 stages + the dt reduction)."""
    per_stage = (n_xfaces + n_yfaces) * (FACE_FLUX + (DIFFUSION if diffusion else 0))
    per_stage += n_fluid * (DERIVED + 2 * NONCON_DIR + RHS_ASSEMBLY + STAGE + (SOURCE if source else 0))
    per_stage += n_ghosts * DERIVED + n_heavy * heavy_ghost_flops()
    return 3 * per_stage + n_fluid * LOCAL_DT


def flux_launch_flops(n_xfaces, n_yfaces, diffusion=False):
    """FLOPs of one launch of the interface-flux kernel (all x and y faces)."""
    return (n_xfaces + n_yfaces) * (FACE_FLUX + (DIFFUSION if diffusion else 0))


def face_counts(fluid, nx, ny):
    """Active x faces (i-1/2, j) and y faces (i, j-1/2): one neighbour fluid (main.rs:168-204)."""
    import numpy as np
    f = np.asarray(fluid, bool).reshape(nx, ny)
    fx = np.zeros((nx + 1, ny), bool)
    fx[:nx] |= f
    fx[1:] |= f
    fy = np.zeros((nx, ny + 1), bool)
    fy[:, :ny] |= f
    fy[:, 1:] |= f
    return int(fx.sum()), int(fy.sum())
