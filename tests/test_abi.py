"""The C ABI library: it loads, exports every function include/rh3t.h
declares, and the host-only entry points work without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "rh3t.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rh3t_[a-z0-9_]+)\s*\(", src)))


@pytest.mark.parametrize("exact", [False, True])
def test_library_exports_every_declared_symbol(rh, exact):
    L = C.CDLL(rh.lib_path(exact))
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_header(rh):
    from importlib import import_module
    lib = import_module("3t_rh_b200._lib")
    assert set(declared_functions()) <= set(lib.EXPORTS)


def test_default_params_are_the_reference_constants(rh):
    L = rh.load()
    from importlib import import_module
    lib = import_module("3t_rh_b200._lib")
    p = lib.Params()
    L.rh3t_default_params(C.byref(p))
    # constant.rs:1-25, bc1.rs:577
    assert (p.gamma_e, p.gamma_i, p.gamma_r) == (1.4, 1.4, 1.4)
    assert (p.cve, p.cvi, p.a_rad) == (1.0, 1.0, 1.0)
    assert (p.kappa_e, p.kappa_i, p.kappa_r, p.omega_ei, p.omega_er) == (0.0,) * 5
    assert (p.lambda_, p.weno_q, p.eps, p.periodic_ly) == (0.5, 10.0, 1e-12, 0.5)


def test_invalid_arguments_rejected_without_device(rh):
    L = rh.load()
    out = C.c_void_p()
    # null grid: rejected before any device call
    assert L.rh3t_create(None, None, None, 0, None, 0, None, None, 0, C.byref(out)) == 7
    assert L.rh3t_upload_state(None, None, 0.0) == 7


def test_geometry_errors_reported(rh):
    """A non-collinear check of the arc constructor (geometry.rs:514-517)."""
    f = rh.cases.init_cylinder(h=0.1)
    f.outer_arcs[0].arc.mid = (0.0, 0.0125)  # collinear with start and end
    with pytest.raises(rh.RH3TError):
        rh.GhostGrid.build(f)


def test_create_failure_message_without_device(rh):
    """A failed create returns no context; its status and message are kept
    per thread (rh3t_create_error): here, set-up on a machine without the
    requested device, and a malformed description."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("needs a machine without a CUDA device")
    L = rh.load()
    f = rh.cases.init_cylinder(h=1.0 / 10.0)
    g = rh.GhostGrid.build(f)
    with pytest.raises(rh.RH3TError) as ei:
        rh.Batch([f], [g])
    assert ei.value.kind == "NO_DEVICE" and "no such CUDA device" in str(ei.value)
    out = C.c_void_p()
    assert L.rh3t_batch_create(1, None, 0, C.byref(out)) == 7
    msg = C.create_string_buffer(192)
    assert L.rh3t_create_error(msg, 192) == 0  # a null description is rejected before the record is set
    inst = (C.c_byte * 256)()  # one instance description of null pointers
    assert L.rh3t_batch_create(1, C.addressof(inst), 0, C.byref(out)) == 7
    assert L.rh3t_create_error(msg, 192) == 7
    assert msg.value.decode() == "instance 0: missing or malformed description"
