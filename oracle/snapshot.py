"""Test infrastructure (reference values for tests, not the product): a numpy restatement of
the reference's RH3TBIN1 snapshot writer and reader (src/io.rs:1-123) and of
its energy-split tool (py_utils/energy_split.py:12-31), used to check the
library's device-packed snapshots, its restart path and its device
reduction."""
import math
import struct

import numpy as np

MAGIC = b"RH3TBIN1"                      # io.rs:5
HEADER = struct.Struct("<8sIIQQd")       # io.rs:9-20; energy_split.py:6
NAN = struct.unpack("<d", struct.pack("<Q", 0x7FF8000000000000))[0]  # Rust f64::NAN


def snapshot_bytes(value, fluid, nx, ny, dx, dy, x0, y0, time):
    """io.rs:25-99 save_data as bytes: value is nx*ny x 6 at i*ny + j (the
    Field::value layout), fluid the nx*ny mask; payload j-major / i-fastest,
    (x, y, rho, mom_x, mom_y, ee, ei, er), NaN state outside the fluid."""
    v = np.asarray(value, np.float64).reshape(nx, ny, 6)
    fl = np.asarray(fluid, bool).reshape(nx, ny)
    rec = np.empty((ny, nx, 8), np.float64)
    i = np.arange(nx, dtype=np.float64)
    j = np.arange(ny, dtype=np.float64)
    rec[:, :, 0] = (x0 + i * dx)[None, :]  # GridInfo::x, field1.rs:6-15
    rec[:, :, 1] = (y0 + j * dy)[:, None]
    st = np.transpose(v, (1, 0, 2)).copy()
    st[~fl.T] = NAN
    rec[:, :, 2:] = st
    return HEADER.pack(MAGIC, 1, 8, nx, ny, float(time)) + rec.astype("<f8").tobytes()


def read_snapshot(path):
    """io.rs:101-123 load_data's parse: (nx, ny, time, records (ny, nx, 8))."""
    with open(path, "rb") as f:
        raw = f.read()
    magic, version, nvar, nx, ny, t = HEADER.unpack(raw[:HEADER.size])
    if magic != MAGIC or version != 1 or nvar != 8:
        raise ValueError("not an RH3TBIN1 v1 file")
    a = np.frombuffer(raw, dtype="<f8", offset=HEADER.size, count=nx * ny * 8).reshape(ny, nx, 8)
    return nx, ny, t, a


def energy_split(records):
    """py_utils/energy_split.py:19-31 on one snapshot's records (ny, nx, 8):
    max, mean and rms of |Ee-Ei|, |Ee-Er|, |Ei-Er| over the finite nodes and
    (x, y) of the first maximum of |Ee-Er|."""
    x, y = records[:, :, 0], records[:, :, 1]
    ee, ei, er = records[:, :, 5], records[:, :, 6], records[:, :, 7]
    valid = np.isfinite(ee) & np.isfinite(ei) & np.isfinite(er)
    out = {}
    for name, d in (("Ee_Ei", np.abs(ee - ei)), ("Ee_Er", np.abs(ee - er)), ("Ei_Er", np.abs(ei - er))):
        m = np.where(valid, d, -np.inf)
        ij = np.unravel_index(int(np.argmax(m)), d.shape)
        out["max_" + name] = float(d[ij])
        out["mean_" + name] = float(np.mean(d[valid]))
        out["rms_" + name] = float(math.sqrt(np.mean(d[valid] ** 2)))
        if name == "Ee_Er":
            out["x_max_Ee_Er"], out["y_max_Ee_Er"] = float(x[ij]), float(y[ij])
    out["n_fluid"] = int(valid.sum())
    return out
