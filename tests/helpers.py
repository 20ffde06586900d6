import numpy as np


def rel_linf(a, b, mask):
    """Normwise relative L-infinity deviation per field over fluid nodes:
    max|a - b| / scale, scale = max|b| for rho, ee, ei, er and the largest
    momentum magnitude max sqrt(mom_x^2 + mom_y^2) for both momentum
    components (a component that is identically ~0, like mom_y in a 1-D
    problem, is measured against the flow's momentum, not against itself)."""
    a, b = a[mask], b[mask]
    scale = np.abs(b).max(0)
    mom = np.sqrt(b[:, 1] ** 2 + b[:, 2] ** 2).max()
    scale[1] = scale[2] = mom
    scale[scale == 0] = 1.0
    return np.abs(a - b).max(0) / scale
