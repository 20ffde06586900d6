"""ctypes binding of librh3t (include/rh3t.h). The library is the product: if
it is missing the import fails loudly; there is no CPU fallback."""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")

RH3T_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "NONPHYSICAL_STATE", 2: "NONFINITE_GHOST", 3: "SINGULAR_ILW", 4: "PERIODIC_WRAP",
    5: "STENCIL_FIT", 6: "GEOMETRY", 7: "INVALID_ARGUMENT", 8: "CUDA", 9: "NONPOSITIVE_DT", 10: "NO_DEVICE",
    11: "DEVICE_TIMEOUT",
}

# exported symbols of include/rh3t.h
EXPORTS = (
    "rh3t_geom_create", "rh3t_geom_fluid_mask", "rh3t_geom_build_ghosts", "rh3t_geom_build_ghosts_device",
    "rh3t_geom_ghost_table",
    "rh3t_geom_access_table", "rh3t_geom_last_error", "rh3t_geom_destroy", "rh3t_default_params", "rh3t_create",
    "rh3t_upload_state", "rh3t_download_state", "rh3t_l", "rh3t_calc_global_dt", "rh3t_rk3_ssp", "rh3t_advance",
    "rh3t_step_host", "rh3t_last_dt", "rh3t_profile_steps", "rh3t_fp64_peak", "rh3t_math_check", "rh3t_div_check",
    "rh3t_calc_global_dt_noalloc", "rh3t_synchronize", "rh3t_last_error", "rh3t_create_error", "rh3t_wait_check", "rh3t_step_host_batch", "rh3t_kernel_launches", "rh3t_stream",
    "rh3t_destroy", "rh3t_batch_create", "rh3t_instance_count", "rh3t_upload_batch", "rh3t_download_batch",
    "rh3t_upload_instance", "rh3t_download_instance", "rh3t_l_instance", "rh3t_calc_global_dt_batch",
    "rh3t_instance_times", "rh3t_instance_status", "rh3t_set_tile_shapes", "rh3t_get_tile_shapes",
    "rh3t_autotune", "rh3t_l_vjp", "rh3t_adjoint_forward", "rh3t_adjoint_backward", "rh3t_adjoint_records",
    "rh3t_adjoint_max_records", "rh3t_snapshot",
    "rh3t_snapshot_wait", "rh3t_restart", "rh3t_energy_split",
)


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("dx", C.c_double), ("dy", C.c_double),
                ("x0", C.c_double), ("y0", C.c_double)]


PARAM_FIELDS = ("gamma_e", "gamma_i", "gamma_r", "cve", "cvi", "a_rad", "kappa_e", "kappa_i", "kappa_r",
                "omega_ei", "omega_er", "lambda_", "weno_q", "eps", "periodic_ly")


class Params(C.Structure):
    _fields_ = [(n, C.c_double) for n in PARAM_FIELDS]


class BC(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("state", C.c_double * 6), ("p_inf", C.c_double),
                ("sigma", C.c_double), ("l_domain", C.c_double), ("td_x0", C.c_double), ("td_speed", C.c_double),
                ("td_left", C.c_double * 6), ("td_right", C.c_double * 6)]


class Arc(C.Structure):
    _fields_ = [("boundary", C.c_int32), ("side_start", C.c_int32), ("side_end", C.c_int32),
                ("fluid_side", C.c_int32), ("start", C.c_double * 2), ("mid", C.c_double * 2),
                ("end", C.c_double * 2)]


class GhostTable(C.Structure):
    _fields_ = [("n_ghosts", C.c_int32), ("idx", C.c_void_p), ("boundary", C.c_void_p), ("side", C.c_void_p),
                ("proj", C.c_void_p), ("pre", C.c_void_p), ("n_heavy", C.c_int32), ("nearest", C.c_void_p),
                ("stencil", C.c_void_p), ("s", C.c_void_p), ("w", C.c_void_p), ("d", C.c_void_p)]


class Error(C.Structure):
    _fields_ = [("code", C.c_int32), ("stage", C.c_int32), ("step", C.c_int64), ("i", C.c_int32),
                ("j", C.c_int32), ("ghost", C.c_int32), ("instance", C.c_int32), ("message", C.c_char * 160)]


class Instance(C.Structure):
    _fields_ = [("grid", C.c_void_p), ("params", C.c_void_p), ("fluid", C.c_void_p), ("n_outer_bc", C.c_int32),
                ("outer_bcs", C.c_void_p), ("n_inner_bc", C.c_int32), ("inner_bcs", C.c_void_p),
                ("ghosts", C.c_void_p)]


class TuneEntry(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("diffusion", C.c_int32), ("n_instances", C.c_int32),
                ("lg_fx", C.c_int32), ("lg_fy", C.c_int32), ("lg_rhs", C.c_int32), ("from_cache", C.c_int32),
                ("ms_fx", C.c_double * 3), ("ms_fy", C.c_double * 3), ("ms_rhs", C.c_double * 3)]


_libs = {}


def lib_path(exact=False):
    return os.path.join(BUILD_DIR, "librh3t_exact.so" if exact else "librh3t.so")


def load(exact=False):
    """Load librh3t (FMA build) or librh3t_exact (no contraction)."""
    if exact in _libs:
        return _libs[exact]
    path = lib_path(exact)
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python 3t_rh_b200/build.py` "
                          "(the rh3t solver has no CPU fallback)")
    L = C.CDLL(path)
    V, I, D, P = C.c_void_p, C.c_int, C.c_double, C.POINTER
    sig = {
        "rh3t_geom_create": (I, [P(Grid), P(Params), C.c_int32, V, C.c_int32, V, C.c_int32, V, C.c_int32, V,
                                 C.c_int32, V, P(V)]),
        "rh3t_geom_fluid_mask": (I, [V, V]),
        "rh3t_geom_build_ghosts": (I, [V, C.c_int32]),
        "rh3t_geom_build_ghosts_device": (I, [C.c_int32, V, C.c_int32, C.c_int32]),
        "rh3t_geom_ghost_table": (I, [V, P(GhostTable)]),
        "rh3t_geom_access_table": (I, [V, V]),
        "rh3t_geom_last_error": (C.c_char_p, [V]),
        "rh3t_geom_destroy": (None, [V]),
        "rh3t_default_params": (None, [P(Params)]),
        "rh3t_create": (I, [P(Grid), P(Params), V, C.c_int32, V, C.c_int32, V, P(GhostTable), C.c_int32, P(V)]),
        "rh3t_upload_state": (I, [V, V, D]),
        "rh3t_download_state": (I, [V, V, P(D)]),
        "rh3t_l": (I, [V, V, V]),
        "rh3t_calc_global_dt": (I, [V, P(D)]),
        "rh3t_rk3_ssp": (I, [V, D]),
        "rh3t_advance": (I, [V, C.c_int32, D, D, C.c_int32]),
        "rh3t_step_host": (I, [V, V, P(D), D, P(D)]),
        "rh3t_last_dt": (I, [V, P(D)]),
        "rh3t_profile_steps": (I, [V, C.c_int32, D, V, V]),
        "rh3t_fp64_peak": (I, [C.c_int32, P(D)]),
        "rh3t_math_check": (I, [C.c_int32, V, C.c_int32, D, V]),
        "rh3t_div_check": (I, [C.c_int32, C.c_int64, C.c_uint64, V, V]),
        "rh3t_calc_global_dt_noalloc": (I, [P(Grid), P(Params), V, V, V, V]),
        "rh3t_synchronize": (I, [V]),
        "rh3t_last_error": (I, [V, P(Error)]),
        "rh3t_create_error": (I, [C.c_char_p, C.c_int32]),
        "rh3t_wait_check": (I, [C.c_int32, C.c_int32, P(C.c_int32)]),
        "rh3t_step_host_batch": (I, [V, V, V, D, C.c_int32]),
        "rh3t_kernel_launches": (C.c_int64, [V]),
        "rh3t_stream": (V, [V]),
        "rh3t_destroy": (None, [V]),
        "rh3t_batch_create": (I, [C.c_int32, V, C.c_int32, P(V)]),
        "rh3t_instance_count": (C.c_int32, [V]),
        "rh3t_upload_batch": (I, [V, V, V]),
        "rh3t_download_batch": (I, [V, V, V]),
        "rh3t_upload_instance": (I, [V, C.c_int32, V, D]),
        "rh3t_download_instance": (I, [V, C.c_int32, V, P(D)]),
        "rh3t_l_instance": (I, [V, C.c_int32, V, V]),
        "rh3t_calc_global_dt_batch": (I, [V, V]),
        "rh3t_instance_times": (I, [V, V, V, V]),
        "rh3t_instance_status": (I, [V, V]),
        "rh3t_set_tile_shapes": (I, [V, C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
        "rh3t_get_tile_shapes": (I, [V, C.c_int32, V]),
        "rh3t_autotune": (I, [V, C.c_char_p, C.c_int32, V, C.c_int32, P(C.c_int32)]),
        "rh3t_l_vjp": (I, [V, C.c_int32, V, V, V]),
        "rh3t_adjoint_forward": (I, [V, C.c_int32, D, C.c_int32]),
        "rh3t_adjoint_backward": (I, [V, V, V, V]),
        "rh3t_adjoint_records": (C.c_int32, [V]),
        "rh3t_adjoint_max_records": (I, [V, C.c_int32]),
        "rh3t_snapshot": (I, [V, C.c_int32, C.c_char_p]),
        "rh3t_snapshot_wait": (I, [V]),
        "rh3t_restart": (I, [V, C.c_int32, C.c_char_p]),
        "rh3t_energy_split": (I, [V, C.c_int32, V]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _libs[exact] = L
    return L
