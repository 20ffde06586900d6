import numpy as np


def rel_linf(a, b, mask):
    """Normwise relative L-infinity per field: max|a-b| / max|b| over fluid nodes."""
    a, b = a[mask], b[mask]
    scale = np.abs(b).max(0)
    scale[scale == 0] = 1.0
    return np.abs(a - b).max(0) / scale
