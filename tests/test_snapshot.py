"""RH3TBIN1 snapshots (io.rs:1-123) and the energy-split diagnostic
(py_utils/energy_split.py).

CPU: the oracle's restated writer produces the header the reference's own
tooling parses (struct "<8sIIQQd", energy_split.py:5-6) and round-trips
through its reader; the energy split of a hand-built snapshot.
GPU (marked): the library's device-packed snapshot is byte-identical to the
oracle's bytes for the same state, restart reproduces the state and time
bitwise, a corrupted or mismatched file is rejected with the reference's
messages, and the device energy split equals the tool's numbers.
"""
import os
import struct

import numpy as np
import pytest

from oracle import snapshot as S


def _state(nx, ny, seed=1):
    rng = np.random.default_rng(seed)
    v = rng.uniform(0.5, 2.0, (nx * ny, 6))
    fluid = rng.uniform(size=nx * ny) > 0.2
    return v, fluid


def test_oracle_snapshot_header_and_round_trip(tmp_path):
    nx, ny = 7, 5
    v, fluid = _state(nx, ny)
    raw = S.snapshot_bytes(v, fluid, nx, ny, 0.1, 0.2, -1.0, 3.0, 1.25)
    magic, version, nvar, gnx, gny, t = struct.unpack("<8sIIQQd", raw[:40])
    assert (magic, version, nvar, gnx, gny, t) == (b"RH3TBIN1", 1, 8, nx, ny, 1.25)
    assert len(raw) == 40 + nx * ny * 64
    p = tmp_path / "s.bin"
    p.write_bytes(raw)
    _, _, t2, a = S.read_snapshot(str(p))
    assert t2 == 1.25
    for i in range(nx):
        for j in range(ny):
            r = a[j, i]
            assert r[0] == -1.0 + i * 0.1 and r[1] == 3.0 + j * 0.2
            if fluid[i * ny + j]:
                assert np.array_equal(r[2:], v[i * ny + j])
            else:
                assert np.isnan(r[2:]).all()


def test_oracle_energy_split_by_hand():
    rec = np.full((2, 3, 8), np.nan)
    rec[:, :, 0] = [[0, 1, 2], [0, 1, 2]]
    rec[:, :, 1] = [[0, 0, 0], [1, 1, 1]]
    rec[0, 0, 5:] = [1.0, 2.0, 4.0]
    rec[1, 2, 5:] = [3.0, 3.0, 0.0]
    d = S.energy_split(rec)
    assert d["max_Ee_Ei"] == 1.0 and d["max_Ee_Er"] == 3.0 and d["max_Ei_Er"] == 3.0
    assert d["mean_Ee_Ei"] == 0.5 and d["mean_Ee_Er"] == 3.0
    assert (d["x_max_Ee_Er"], d["y_max_Ee_Er"]) == (0.0, 0.0)  # first of the tie in j-major order
    assert d["n_fluid"] == 2


@pytest.mark.gpu
def test_device_snapshot_bytes_restart_and_energy_split(rh, tmp_path):
    f = rh.cases.init_cylinder(h=1.0 / 20.0, params=rh.Params(omega_ei=0.5, omega_er=2.0))
    g = rh.GhostGrid.build(f)
    s = rh.Solver(f, g)
    s.advance(7, 0.05)
    u, t = s.download()
    gr = f.grid
    p = tmp_path / "solution_0007.bin"
    s.snapshot(str(p))
    s.snapshot_wait()
    assert not os.path.exists(str(p) + ".tmp")
    expect = S.snapshot_bytes(u, f.fluid, gr.nx, gr.ny, gr.dx, gr.dy, gr.x0, gr.y0, t)
    assert p.read_bytes() == expect
    # io.rs save_data layout under data_new/
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        s.save_data("solution_0000.bin")
        assert (tmp_path / "data_new" / "solution_0000.bin").read_bytes() == expect
    finally:
        os.chdir(cwd)
    # restart into a fresh solver: state and time bitwise
    s2 = rh.Solver(f, g)
    s2.load_data(str(p))
    u2, t2 = s2.download()
    assert t2 == t and np.array_equal(u2[f.fluid], u[f.fluid])
    # both continue identically
    s.advance(3, 0.05)
    s2.advance(3, 0.05)
    assert np.array_equal(s.download()[0], s2.download()[0])
    # energy split: device reduction vs the tool on the file
    _, _, _, rec = S.read_snapshot(str(p))
    ref = S.energy_split(rec)
    s3 = rh.Solver(f, g)
    s3.load_data(str(p))
    dev = s3.energy_split()
    for k, v in ref.items():
        if k.startswith(("mean", "rms")):
            assert abs(dev[k] - v) <= 1e-13 * abs(v), k
        else:
            assert dev[k] == v, k
    # rejected files: grid mismatch, bad magic, non-finite fluid state
    f2 = rh.cases.init_cylinder(h=1.0 / 10.0)
    s4 = rh.Solver(f2, rh.GhostGrid.build(f2))
    with pytest.raises(rh.RH3TError, match="restart grid mismatch"):
        s4.load_data(str(p))
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"RH3TBIN2" + expect[8:])
    with pytest.raises(rh.RH3TError, match="bad magic"):
        s2.load_data(str(bad))
    raw = bytearray(expect)
    l = int(np.nonzero(f.fluid)[0][0])
    i, j = l // gr.ny, l % gr.ny
    off = 40 + 8 * (8 * (j * gr.nx + i) + 2)
    raw[off:off + 8] = struct.pack("<d", float("inf"))
    bad.write_bytes(bytes(raw))
    with pytest.raises(rh.RH3TError, match="non-finite restart state"):
        s2.load_data(str(bad))
    for x in (s, s2, s3, s4):
        x.close()
