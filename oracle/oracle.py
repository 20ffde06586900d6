"""ORACLE — test infrastructure only.

ctypes front end of the CPU restatement of colinhu123/3T_RH's hot path
(``oracle/src``). Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may use it, and
only as the reference values of parity tests or the timed CPU baseline; the
product never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


_VARIANTS = {}


def _variant(libname):
    if libname not in _VARIANTS:
        import importlib.util
        spec = importlib.util.spec_from_file_location(f"oracle_variant_{libname}", os.path.abspath(__file__))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod._LIB_PATH = os.path.join(_HERE, "_build", libname)
        _VARIANTS[libname] = mod
    return _VARIANTS[libname]


def fma_variant():
    """A second instance of this module bound to liboracle_fma.so (the
    restatement compiled with FMA contraction): the rounding envelope of the
    reference algorithm."""
    return _variant("liboracle_fma.so")


def crpow_variant():
    """This module bound to liboracle_crpow.so: the restatement (no
    contraction) with the correctly rounded power in place of libm pow for
    the reference's two powf calls (state.rs:261, bc1.rs:241). Its distance
    from the plain oracle is how far a last-bit change of libm moves a run;
    on runs it moves, it is the parity reference of the no-contraction CUDA
    build, which computes the same correctly rounded power."""
    return _variant("liboracle_crpow.so")

# Order of the 15 runtime parameters (oracle/src/physics.hpp Params)
PARAM_NAMES = ("gamma_e", "gamma_i", "gamma_r", "cve", "cvi", "a_rad", "kappa_e", "kappa_i", "kappa_r",
               "omega_ei", "omega_er", "lambda_", "weno_q", "eps", "periodic_ly")
DEFAULT_PARAMS = (1.4, 1.4, 1.4, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.5, 10.0, 1e-12, 0.5)

BC_REFLECTIVE_WALL, BC_WALL, BC_PERIODIC, BC_CONSTANT, BC_TIME_DEPENDENT, BC_OUTFLOW, BC_ZEROTH_ORDER, \
    BC_FAR_FIELD = range(8)


def build():
    """Compile liboracle.so with the committed Makefile (g++, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P, D, I, LG = C.c_void_p, C.c_double, C.c_int, C.c_long
        dp = C.POINTER(C.c_double)
        for name, res, args in [
            ("oracle_create_cylinder", P, [D, D, D, dp, C.c_char_p, I]),
            ("oracle_create_double_mach", P, [D, dp, C.c_char_p, I]),
            ("oracle_create_planar_shock", P, [LG, LG, D, D, D, D, D, dp, C.c_char_p, I]),
            ("oracle_create_rect", P, [LG, LG, D, D, dp, I, dp, C.c_char_p, I]),
            ("oracle_destroy", None, [P]),
            ("oracle_dims", None, [P, C.POINTER(LG), C.POINTER(LG), dp]),
            ("oracle_params", None, [P, dp]),
            ("oracle_fluid", None, [P, C.c_void_p]),
            ("oracle_get_state", None, [P, C.c_void_p]),
            ("oracle_set_state", None, [P, C.c_void_p]),
            ("oracle_time", D, [P]),
            ("oracle_set_time", None, [P, D]),
            ("oracle_geometry_sizes", None, [P, C.c_void_p]),
            ("oracle_geometry", None, [P] + [C.c_void_p] * 7),
            ("oracle_n_ghosts", LG, [P]),
            ("oracle_n_heavy", LG, [P]),
            ("oracle_ghost_info", None, [P] + [C.c_void_p] * 6),
            ("oracle_ghost_pre", None, [P] + [C.c_void_p] * 5),
            ("oracle_access", None, [P, C.c_void_p]),
            ("oracle_last_error", I, [P, C.c_void_p, C.c_char_p, I]),
            ("oracle_l", I, [P, C.c_void_p, C.c_void_p]),
            ("oracle_l_jvp", I, [P] + [C.c_void_p] * 7),
            ("oracle_l_t", I, [P, C.c_void_p, C.c_void_p]),
            ("oracle_rk3", I, [P, D]),
            ("oracle_global_dt", D, [P]),
            ("oracle_run", I, [P, LG, D, C.c_void_p]),
            ("oracle_set_threads", None, [I]),
            ("oracle_max_threads", I, []),
            ("oracle_weno5", None, [dp, dp]),
            ("oracle_derived", None, [dp, dp, dp]),
            ("oracle_flux", None, [dp, I, dp, dp]),
            ("oracle_build_lr", None, [dp, dp, I, dp, dp, dp, dp]),
            ("oracle_reconstruction", None, [dp, I, I, dp, dp]),
            ("oracle_noncon", None, [dp, D, I, dp, dp]),
            ("oracle_diffusion", None, [dp, dp, dp]),
            ("oracle_source", None, [dp, dp, dp]),
            ("oracle_local_dt", D, [dp, D, D, dp]),
            ("oracle_sixth_derivative", D, [dp, D]),
            ("oracle_fit_poly", None, [dp, I, I, dp]),
            ("oracle_x_derivative", D, [dp, I, I]),
            ("oracle_smooth_indicator", D, [dp, I, D]),
            ("oracle_extractor", I, [P, dp, I, C.c_void_p]),
            ("oracle_project_outer", None, [P, D, D, dp]),
            ("oracle_ghost_value", I, [P, LG, dp]),
            ("oracle_arc", None, [P, I, dp]),
            ("oracle_circle_from_three", None, [dp, I, dp]),
            ("oracle_arc_project", None, [dp, I, D, D, dp]),
            ("oracle_arc_contains", I, [dp, I, D]),
            ("oracle_ghost_extrapolation", I, [P, LG, dp]),
            ("oracle_ghost_id", LG, [P, LG, LG]),
            ("oracle_flop_counts", None, [C.c_void_p]),
            ("oracle_reconstruction_slow", None, [dp, I, I, dp, dp]),
            ("oracle_ghost_probe", I, [P, LG, LG, dp]),
            ("oracle_ghost_value_at", I, [P, LG, LG, dp, I, I, I, dp]),
            ("oracle_wall_systems", I, [P, LG, dp, dp, dp, dp]),
            ("oracle_solve6", I, [dp, dp, dp]),
        ]:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def solve6(A, b):
    """bc1.rs:467-469 solve6 as the oracle restates it (LU with partial
    pivoting); None for a zero pivot."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(6)
    return None if lib().oracle_solve6(_dp(A), _dp(b), _dp(x)) else x


def _ptr(a):
    return None if a is None else a.ctypes.data


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def params_array(**kw):
    p = list(DEFAULT_PARAMS)
    for k, v in kw.items():
        p[PARAM_NAMES.index(k)] = float(v)
    return np.array(p, dtype=np.float64)


class OracleError(RuntimeError):
    def __init__(self, code, msg, ij):
        super().__init__(f"{msg} (code {code}) at {ij}")
        self.code, self.ij = code, ij


class Case:
    """One oracle instance: field + ghost grid + solver scratch."""

    def __init__(self, handle, params):
        if not handle:
            raise RuntimeError("oracle case construction failed")
        self.h = handle
        self.params = params
        nx, ny = C.c_long(), C.c_long()
        g = np.zeros(4)
        lib().oracle_dims(self.h, C.byref(nx), C.byref(ny), _dp(g))
        self.nx, self.ny = nx.value, ny.value
        self.dx, self.dy, self.x0, self.y0 = g

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    # ---- constructors
    @classmethod
    def cylinder(cls, h=1.0 / 40.0, mach=3.0, shift=0.0125, **params):
        p = params_array(**params)
        msg = C.create_string_buffer(256)
        return cls(lib().oracle_create_cylinder(h, mach, shift, _dp(p), msg, 256), p)

    @classmethod
    def double_mach(cls, h=1.0 / 320.0, **params):
        p = params_array(**params)
        msg = C.create_string_buffer(256)
        return cls(lib().oracle_create_double_mach(h, _dp(p), msg, 256), p)

    @classmethod
    def planar_shock(cls, nx=1024, ny=8, lx=4.0, ly=0.03125, x_shock=1.0, mach=2.0, sigma=0.25, **params):
        params.setdefault("periodic_ly", ly)
        p = params_array(**params)
        msg = C.create_string_buffer(256)
        return cls(lib().oracle_create_planar_shock(nx, ny, lx, ly, x_shock, mach, sigma, _dp(p), msg, 256), p)

    @classmethod
    def rect(cls, nx, ny, lx, ly, state, kind=BC_WALL, **params):
        p = params_array(**params)
        s = np.asarray(state, dtype=np.float64)
        msg = C.create_string_buffer(256)
        return cls(lib().oracle_create_rect(nx, ny, lx, ly, _dp(s), kind, _dp(p), msg, 256), p)

    # ---- state
    @property
    def n(self):
        return self.nx * self.ny

    def fluid(self):
        out = np.zeros(self.n, dtype=np.uint8)
        lib().oracle_fluid(self.h, out.ctypes.data)
        return out.astype(bool)

    def state(self):
        out = np.zeros((self.n, 6))
        lib().oracle_get_state(self.h, out.ctypes.data)
        return out

    def set_state(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64).reshape(self.n, 6)
        lib().oracle_set_state(self.h, s.ctypes.data)

    @property
    def time(self):
        return lib().oracle_time(self.h)

    @time.setter
    def time(self, t):
        lib().oracle_set_time(self.h, float(t))

    # ---- geometry / ghost grid
    def geometry(self):
        sizes = np.zeros(4, dtype=np.int64)
        lib().oracle_geometry_sizes(self.h, sizes.ctypes.data)
        no, ni = int(sizes[0]), int(sizes[1])
        oxy, ixy = np.zeros((no, 2)), np.zeros((ni, 2))
        ok, ik = np.zeros(no, np.int32), np.zeros(ni, np.int32)
        obc, ibc = np.zeros((no, 24)), np.zeros((ni, 24))
        fs = np.zeros(2, np.int32)
        lib().oracle_geometry(self.h, oxy.ctypes.data, ixy.ctypes.data, ok.ctypes.data, ik.ctypes.data,
                              obc.ctypes.data, ibc.ctypes.data, fs.ctypes.data)
        arcs = []
        for k in range(int(sizes[2])):
            a = np.zeros(8)
            lib().oracle_arc(self.h, k, _dp(a))
            arcs.append(a)
        return dict(outer_xy=oxy, inner_xy=ixy, outer_kind=ok, inner_kind=ik, outer_bc=obc, inner_bc=ibc,
                    fluid_sides=fs, arcs=arcs)

    def n_ghosts(self):
        return int(lib().oracle_n_ghosts(self.h))

    def n_heavy(self):
        return int(lib().oracle_n_heavy(self.h))

    def ghost_info(self):
        n = self.n_ghosts()
        ij = np.zeros((n, 2), np.int32)
        bnd, side, pre = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
        proj = np.zeros((n, 5))
        near = np.zeros((n, 2), np.int32)
        lib().oracle_ghost_info(self.h, ij.ctypes.data, bnd.ctypes.data, side.ctypes.data, proj.ctypes.data,
                                near.ctypes.data, pre.ctypes.data)
        return dict(ij=ij, boundary=bnd, side=side, proj=proj, nearest=near, pre=pre)

    def ghost_pre(self):
        m = self.n_heavy()
        near = np.zeros((m, 2), np.int32)
        st = np.zeros((m, 55), np.uint32)
        s, w, d = np.zeros((m, 979)), np.zeros((m, 225)), np.zeros((m, 5))
        lib().oracle_ghost_pre(self.h, near.ctypes.data, st.ctypes.data, s.ctypes.data, w.ctypes.data,
                               d.ctypes.data)
        return dict(nearest=near, stencil=st, s=s, w=w, d=d)

    def access(self):
        out = np.zeros(self.n * 17, np.uint32)
        lib().oracle_access(self.h, out.ctypes.data)
        return out.reshape(self.n, 17)

    # ---- operators
    def _check(self, rc):
        if rc:
            ij = np.zeros(2, np.int64)
            msg = C.create_string_buffer(256)
            code = lib().oracle_last_error(self.h, ij.ctypes.data, msg, 256)
            raise OracleError(code, msg.value.decode(), tuple(ij))

    def l(self):
        rhs = np.zeros((self.n, 6))
        gv = np.zeros((self.n_ghosts(), 6))
        self._check(lib().oracle_l(self.h, rhs.ctypes.data, gv.ctypes.data))
        return rhs, gv

    def l_jvp(self, du=None, duinf=None, domega=None):
        """Forward-mode directional derivative of l() (dual numbers): returns
        (rhs, d rhs, ghost values, d ghost values) for a state direction du
        (nx*ny x 6), a direction of every FarField state (6) and of
        (omega_ei, omega_er)."""
        rhs, drhs = np.zeros((self.n, 6)), np.zeros((self.n, 6))
        gv, dgv = np.zeros((self.n_ghosts(), 6)), np.zeros((self.n_ghosts(), 6))
        du = None if du is None else np.ascontiguousarray(du, np.float64)
        du6 = None if duinf is None else np.ascontiguousarray(duinf, np.float64)
        dom = None if domega is None else np.ascontiguousarray(domega, np.float64)
        self._check(lib().oracle_l_jvp(self.h, _ptr(du), _ptr(du6), _ptr(dom), rhs.ctypes.data, drhs.ctypes.data,
                                       gv.ctypes.data, dgv.ctypes.data))
        return rhs, drhs, gv, dgv

    def l_t(self):
        """l() through the scalar-type templates at T = double"""
        rhs = np.zeros((self.n, 6))
        gv = np.zeros((self.n_ghosts(), 6))
        self._check(lib().oracle_l_t(self.h, rhs.ctypes.data, gv.ctypes.data))
        return rhs, gv

    def rk3_ssp(self, dt):
        self._check(lib().oracle_rk3(self.h, float(dt)))

    def global_dt(self):
        return lib().oracle_global_dt(self.h)

    def run(self, nsteps, cfl_factor=0.05):
        dts = np.zeros(nsteps)
        self._check(lib().oracle_run(self.h, nsteps, cfl_factor, dts.ctypes.data))
        return dts

    def ghost_value(self, gid):
        out = np.zeros(6)
        rc = lib().oracle_ghost_value(self.h, gid, _dp(out))
        if rc:
            raise OracleError(rc, "ghost value", (gid, 0))
        return out

    def ghost_id(self, i, j):
        return int(lib().oracle_ghost_id(self.h, i, j))

    def ghost_extrapolation(self, gid):
        out = np.zeros((5, 6))
        if lib().oracle_ghost_extrapolation(self.h, gid, _dp(out)):
            raise ValueError("not a WENO-extrapolated ghost")
        return out

    def wall_systems(self, gid):
        """The two 6x6 ILW systems (A0, b0, A1, b1) of Wall ghost gid as the
        ghost update solves them (bc1.rs:691-740); None when the first is
        singular."""
        A0, A1, b0, b1 = np.zeros((6, 6)), np.zeros((6, 6)), np.zeros(6), np.zeros(6)
        rc = lib().oracle_wall_systems(self.h, gid, _dp(A0), _dp(b0), _dp(A1), _dp(b1))
        if rc < 0:
            raise ValueError("not a Wall ghost")
        return None if rc else (A0, b0, A1, b1)

    def extractor(self, proj5, r):
        out = np.zeros(((r + 1) ** 2, 2), np.int32)
        p = np.asarray(proj5, dtype=np.float64)
        n = lib().oracle_extractor(self.h, _dp(p), r, out.ctypes.data)
        if n < 0:
            raise OracleError(-n, "cannot fit paper substencil", (0, 0))
        return out

    def ghost_probe(self, i, j):
        """(projection[5], side) of grid point (i, j) on the outer polygon, as
        the reference's ghost_bc_fast_matches_slow forms them (main.rs:567-596)."""
        proj = np.zeros(5)
        side = lib().oracle_ghost_probe(self.h, i, j, _dp(proj))
        return proj, side

    def ghost_value_at(self, i, j, proj5, side, boundary=0, mode="fast"):
        """set_ghost_point_value at (i, j) for the given projection and side on
        the current state: mode "fast" (precomputed GhostBC, bc1.rs:108-255),
        "slow" (per-call least squares, bc1.rs:345-421) or "slow_beta0" (the
        per-call path with the precomputed path's r = 0 indicator)."""
        out = np.zeros(6)
        p = np.asarray(proj5, dtype=np.float64)
        rc = lib().oracle_ghost_value_at(self.h, i, j, _dp(p), boundary, side,
                                         {"fast": 0, "slow": 1, "slow_beta0": 2}[mode], _dp(out))
        if rc:
            raise OracleError(rc, "ghost value", (i, j))
        return out

    def project_outer(self, x, y):
        out = np.zeros(5)
        lib().oracle_project_outer(self.h, x, y, _dp(out))
        return out


def set_threads(n):
    lib().oracle_set_threads(int(n))


def max_threads():
    return int(lib().oracle_max_threads())


# ---- pointwise known-answer helpers
def flop_counts():
    out = np.zeros(11, np.int64)
    lib().oracle_flop_counts(out.ctypes.data)
    return dict(zip(("flux_x", "flux_y", "derived", "noncon_dir", "diffusion", "source", "local_dt", "weno5",
                     "build_l", "build_r", "phys_flux"), out.tolist()))


def weno5(u5):
    u = np.asarray(u5, dtype=np.float64)
    out = np.zeros(1)
    lib().oracle_weno5(_dp(u), _dp(out))
    return out[0]


def derived(s6, params=None):
    s = np.asarray(s6, dtype=np.float64)
    p = params if params is not None else params_array()
    out = np.zeros(11)
    lib().oracle_derived(_dp(s), _dp(p), _dp(out))
    return out


def flux(s6, direction, params=None):
    s = np.asarray(s6, dtype=np.float64)
    p = params if params is not None else params_array()
    out = np.zeros(6)
    lib().oracle_flux(_dp(s), direction, _dp(p), _dp(out))
    return out


def build_lr(s1, s2, direction, params=None):
    a, b = np.asarray(s1, dtype=np.float64), np.asarray(s2, dtype=np.float64)
    p = params if params is not None else params_array()
    L, R, lam = np.zeros((6, 6)), np.zeros((6, 6)), np.zeros(6)
    lib().oracle_build_lr(_dp(a), _dp(b), direction, _dp(p), _dp(L), _dp(R), _dp(lam))
    return L, R, lam


def reconstruction(pts, direction, recon=True, params=None):
    a = np.ascontiguousarray(pts, dtype=np.float64).reshape(36)
    p = params if params is not None else params_array()
    out = np.zeros(6)
    lib().oracle_reconstruction(_dp(a), direction, int(recon), _dp(p), _dp(out))
    return out


def reconstruction_slow(pts, direction, recon=True, params=None):
    """weno.rs:599-679 Stencil6::reconstruction (ndarray L/R, State::flux)"""
    a = np.ascontiguousarray(pts, dtype=np.float64).reshape(36)
    p = params if params is not None else params_array()
    out = np.zeros(6)
    lib().oracle_reconstruction_slow(_dp(a), direction, int(recon), _dp(p), _dp(out))
    return out


def noncon(pts9, ds, direction, params=None):
    a = np.ascontiguousarray(pts9, dtype=np.float64).reshape(54)
    p = params if params is not None else params_array()
    out = np.zeros(6)
    lib().oracle_noncon(_dp(a), ds, direction, _dp(p), _dp(out))
    return out


def diffusion(pts6, params=None):
    a = np.ascontiguousarray(pts6, dtype=np.float64).reshape(36)
    p = params if params is not None else params_array()
    out = np.zeros(6)
    lib().oracle_diffusion(_dp(a), _dp(p), _dp(out))
    return out


def source(s6, params=None):
    s = np.asarray(s6, dtype=np.float64)
    p = params if params is not None else params_array()
    out = np.zeros(6)
    lib().oracle_source(_dp(s), _dp(p), _dp(out))
    return out


def local_dt(s6, dx, dy, params=None):
    s = np.asarray(s6, dtype=np.float64)
    p = params if params is not None else params_array()
    return lib().oracle_local_dt(_dp(s), dx, dy, _dp(p))


def sixth_derivative(q6, dx):
    q = np.asarray(q6, dtype=np.float64)
    return lib().oracle_sixth_derivative(_dp(q), dx)


def fit_poly(xyz, degree):
    a = np.ascontiguousarray(xyz, dtype=np.float64)
    out = np.zeros((degree + 1) * (degree + 2) // 2)
    lib().oracle_fit_poly(_dp(a), a.shape[0], degree, _dp(out))
    return out


def x_derivative(coef, degree, k):
    c = np.asarray(coef, dtype=np.float64)
    return lib().oracle_x_derivative(_dp(c), degree, k)


def smooth_indicator(coef, r, h):
    c = np.asarray(coef, dtype=np.float64)
    return lib().oracle_smooth_indicator(_dp(c), r, h)


def circle_from_three(p6, fluid):
    a = np.asarray(p6, dtype=np.float64)
    out = np.zeros(5)
    lib().oracle_circle_from_three(_dp(a), fluid, _dp(out))
    return out


def arc_project(arc5, fluid, x, y):
    a = np.asarray(arc5, dtype=np.float64)
    out = np.zeros(5)
    lib().oracle_arc_project(_dp(a), fluid, x, y, _dp(out))
    return out


def arc_contains(arc5, fluid, theta):
    a = np.asarray(arc5, dtype=np.float64)
    return bool(lib().oracle_arc_contains(_dp(a), fluid, theta))
