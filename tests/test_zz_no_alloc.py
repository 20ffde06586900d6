"""rh3t_calc_global_dt_noalloc, the time-step reduction for callers that
cannot allocate device memory (their device memory belongs to a host
framework or pool, or an allocation would synchronise the device where they
call): it must give the same dt_cfl as rh3t_calc_global_dt on the same
state, on two calls in a row (the second on a different state, so nothing
left in its shared scratch array can leak into a result). The caller owns
every buffer; here torch allocates the inputs and the output.

Kept in a file of its own that pytest collects last; it passes alone in a
fresh process and after the other tests."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_dt_matches_existing_entry_point_twice(rh):
    import torch
    f = rh.cases.init_cylinder()
    g = rh.GhostGrid.build(f)
    s = rh.Solver(f, g)
    L = s.L  # the same build as the solver the expected value comes from
    grid, prm = f.grid.to_c(), f.params.to_c()
    fluid_d = torch.tensor(f.fluid.astype(np.uint8), device="cuda")
    out_d = torch.zeros(1, dtype=torch.float64, device="cuda")
    seen = []
    for call in range(2):
        if call == 1:
            s.advance(5, 0.05)  # a different state for the second call
        u, _ = s.download()
        expected = s.calc_global_dt()
        u_d = torch.tensor(np.ascontiguousarray(u), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = L.rh3t_calc_global_dt_noalloc(C.byref(grid), C.byref(prm), u_d.data_ptr(), fluid_d.data_ptr(),
                                            out_d.data_ptr(), None)
        assert rc == 0
        torch.cuda.synchronize()
        got = float(out_d.item())
        # same device function as rh3t_calc_global_dt, same build: within the
        # dt tolerance of tests/test_gpu_parity.py
        assert abs(got - expected) <= 1e-15 * expected, (call, got, expected)
        seen.append(got)
    assert seen[0] != seen[1]


def test_noalloc_rejects_grids_beyond_its_scratch(rh):
    import torch
    L = rh.load()
    lib = __import__("importlib").import_module("3t_rh_b200._lib")
    big = lib.Grid(65536, 257, 0.01, 0.01, 0.0, 0.0)  # 65536 * 257 nodes > RH3T_DT_NOALLOC_MAX_CELLS
    prm = lib.Params()
    L.rh3t_default_params(C.byref(prm))
    dummy = torch.zeros(6, dtype=torch.float64, device="cuda")
    out_d = torch.zeros(1, dtype=torch.float64, device="cuda")
    # rejected on the host before anything is queued
    rc = L.rh3t_calc_global_dt_noalloc(C.byref(big), C.byref(prm), dummy.data_ptr(), dummy.data_ptr(),
                                        out_d.data_ptr(), None)
    assert rc == 7
