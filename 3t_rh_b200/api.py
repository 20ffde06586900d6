"""Host-side mirror of the reference's Rust API for the 3T_RH hot path.

Names, argument meaning and error behaviour follow colinhu123/3T_RH:
  GridInfo, Field, Polygon, CircularArc/ArcOverride, BCType   (field1.rs, geometry.rs, bc1.rs)
  GhostGrid.build                                              (ghost.rs:50-118)
  l, rk3_ssp, calc_global_dt                                   (main.rs:135, 351, 375)
Every computation runs in librh3t (include/rh3t.h): the geometry / ghost-grid
build on the host in C++, the operator and the time stepping on the GPU.
Where the reference panics, these functions raise RH3TError carrying the
reference's message.
"""
import ctypes as C
import math
import os

import numpy as np

from . import _lib

FLUID_INSIDE, FLUID_OUTSIDE = 0, 1
OUTER, INNER = 0, 1


class RH3TError(RuntimeError):
    """A failure the reference reports with panic! (main.rs:30-33, ghost.rs:229-263, bc1.rs:467-469, ...)."""

    def __init__(self, code, message, stage=0, step=0, i=0, j=0, ghost=-1, instance=-1):
        self.code, self.stage, self.step, self.i, self.j, self.ghost = code, stage, step, i, j, ghost
        self.instance = instance
        self.kind = _lib.STATUS_NAMES.get(code, str(code))
        where = f", instance {instance}" if instance > 0 else ""
        super().__init__(f"{message} [{self.kind}; step {step}, stage {stage}, idx ({i}, {j}), ghost {ghost}{where}]")


def _raise_last(L, h, rc):
    e = _lib.Error()
    L.rh3t_last_error(h, C.byref(e))
    raise RH3TError(e.code or rc, e.message.decode(), e.stage, e.step, e.i, e.j, e.ghost, e.instance)


def _raise_create(L, rc, what):
    msg = C.create_string_buffer(192)
    code = L.rh3t_create_error(msg, 192)
    raise RH3TError(code or rc, f"{what}: {msg.value.decode()}" if msg.value else what)


def _arr(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _ptr(a):
    return a.ctypes.data if a is not None and a.size else None


# ------------------------------------------------------------------ bc1.rs:17-28
class BCType:
    REFLECTIVE_WALL, WALL, PERIODIC, CONSTANT, TIME_DEPENDENT, OUTFLOW, ZEROTH_ORDER, FAR_FIELD = range(8)

    def __init__(self, kind, state=None, p_inf=0.0, sigma=0.0, l_domain=1.0, td_x0=0.0, td_speed=0.0,
                 td_left=None, td_right=None):
        self.kind = kind
        self.state = np.zeros(6) if state is None else np.asarray(state, dtype=np.float64)
        self.p_inf, self.sigma, self.l_domain = float(p_inf), float(sigma), float(l_domain)
        self.td_x0, self.td_speed = float(td_x0), float(td_speed)
        self.td_left = np.zeros(6) if td_left is None else np.asarray(td_left, dtype=np.float64)
        self.td_right = np.zeros(6) if td_right is None else np.asarray(td_right, dtype=np.float64)

    @classmethod
    def ReflectiveWall(cls):
        return cls(cls.REFLECTIVE_WALL)

    @classmethod
    def Wall(cls):
        return cls(cls.WALL)

    @classmethod
    def Periodic(cls):
        return cls(cls.PERIODIC)

    @classmethod
    def Constant(cls, state):
        return cls(cls.CONSTANT, state=state)

    @classmethod
    def TimeDependent(cls, x0, speed, left, right):
        """The reference's closure type (bc1.rs:14) restricted to its one use
        (init.rs:61-65): U = left if P0.x <= x0 + speed*t else right."""
        return cls(cls.TIME_DEPENDENT, td_x0=x0, td_speed=speed, td_left=left, td_right=right)

    @classmethod
    def Outflow(cls, p_inf, sigma, l_domain):
        return cls(cls.OUTFLOW, p_inf=p_inf, sigma=sigma, l_domain=l_domain)

    @classmethod
    def ZerothOrder(cls):
        return cls(cls.ZEROTH_ORDER)

    @classmethod
    def FarField(cls, state):
        return cls(cls.FAR_FIELD, state=state)

    def to_c(self):
        b = _lib.BC()
        b.kind = self.kind
        for k in range(6):
            b.state[k] = self.state[k]
            b.td_left[k] = self.td_left[k]
            b.td_right[k] = self.td_right[k]
        b.p_inf, b.sigma, b.l_domain, b.td_x0, b.td_speed = self.p_inf, self.sigma, self.l_domain, self.td_x0, \
            self.td_speed
        return b


# ------------------------------------------------------------------ constant.rs
class Params:
    """constant.rs values as runtime parameters (defaults = the reference's)."""
    FIELDS = _lib.PARAM_FIELDS

    def __init__(self, **kw):
        self.gamma_e = self.gamma_i = self.gamma_r = 1.4
        self.cve = self.cvi = self.a_rad = 1.0
        self.kappa_e = self.kappa_i = self.kappa_r = 0.0
        self.omega_ei = self.omega_er = 0.0
        self.lambda_, self.weno_q, self.eps, self.periodic_ly = 0.5, 10.0, 1e-12, 0.5
        for k, v in kw.items():
            if k not in self.FIELDS:
                raise TypeError(f"unknown parameter {k}")
            setattr(self, k, float(v))

    def to_c(self):
        p = _lib.Params()
        for k in self.FIELDS:
            setattr(p, k, getattr(self, k))
        return p

    def as_array(self):
        return np.array([getattr(self, k) for k in self.FIELDS])


# ------------------------------------------------------------------ field1.rs:6-73
class GridInfo:
    def __init__(self, nx, ny, dx, dy, x0, y0):
        assert nx > 0 and ny > 0 and dx > 0.0 and dy > 0.0
        self.nx, self.ny, self.dx, self.dy, self.x0, self.y0 = int(nx), int(ny), float(dx), float(dy), float(x0), \
            float(y0)

    def x(self, i):
        return self.x0 + float(i) * self.dx

    def y(self, j):
        return self.y0 + float(j) * self.dy

    def len(self):
        return self.nx * self.ny

    def is_in_domain(self, idx):
        i, j = idx
        return 0 <= i < self.nx and 0 <= j < self.ny

    def coord2idx(self, p):
        return (int(_round_half_away((p[0] - self.x0) / self.dx)), int(_round_half_away((p[1] - self.y0) / self.dy)))

    def to_c(self):
        return _lib.Grid(self.nx, self.ny, self.dx, self.dy, self.x0, self.y0)


def _round_half_away(v):
    return math.floor(v + 0.5) if v >= 0 else -math.floor(-v + 0.5)


# ------------------------------------------------------------------ geometry.rs
class Polygon:
    def __init__(self, points, fluid=FLUID_INSIDE):
        self.points = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 2)
        self.fluid = fluid


class CircularArc:
    """geometry.rs:492-549: kept as its three construction points; the arc
    itself (centre, radius, angles) is formed in librh3t."""

    def __init__(self, start, mid, end, fluid):
        self.start, self.mid, self.end, self.fluid = tuple(start), tuple(mid), tuple(end), fluid

    @classmethod
    def from_three_points(cls, start, mid, end, fluid):
        return cls(start, mid, end, fluid)


class ArcOverride:
    def __init__(self, side_start, side_end, arc, boundary=OUTER):
        self.side_start, self.side_end, self.arc, self.boundary = int(side_start), int(side_end), arc, boundary

    def contains_side(self, side):
        return self.side_start <= side <= self.side_end

    def to_c(self):
        a = _lib.Arc()
        a.boundary, a.side_start, a.side_end, a.fluid_side = self.boundary, self.side_start, self.side_end, \
            self.arc.fluid
        for k in range(2):
            a.start[k], a.mid[k], a.end[k] = self.arc.start[k], self.arc.mid[k], self.arc.end[k]
        return a


# ------------------------------------------------------------------ field1.rs:75-136
class Field:
    """Field: grid, node values (nx*ny x 6, linear index i*ny+j), the two
    bounding polygons with one BCType per side, time, fluid mask, arcs."""

    def __init__(self, grid, bc_inner, bc_outer, value, outer_bound, inner_bound, time=0.0, params=None):
        assert outer_bound.fluid == FLUID_INSIDE, "Wrong outer boundary setting"
        assert inner_bound.fluid == FLUID_OUTSIDE, "Wrong inner boundary setting"
        assert len(bc_inner) == len(inner_bound.points)
        assert len(bc_outer) == len(outer_bound.points)
        self.grid = grid
        self.params = params if params is not None else Params()
        self.outer_bound, self.inner_bound = outer_bound, inner_bound
        self.bc_inner, self.bc_outer = list(bc_inner), list(bc_outer)
        self.time = float(time)
        self.outer_arcs, self.inner_arcs = [], []
        v = np.asarray(value, dtype=np.float64)
        self.value = np.tile(v.reshape(1, 6), (grid.len(), 1)) if v.size == 6 else _arr(v.reshape(-1, 6), np.float64)
        with _Geom(self, arcs=False) as g:
            self.fluid = g.fluid_mask()

    def is_in_domain(self, idx):
        i, j = idx
        return self.grid.is_in_domain(idx) and bool(self.fluid[i * self.grid.ny + j])

    def linear_index(self, idx):
        return idx[0] * self.grid.ny + idx[1]

    def set(self, idx, value):
        assert self.is_in_domain(idx), f"cannot write ghost cell {idx}"
        self.value[self.linear_index(idx)] = value

    def get_inside(self, idx):
        return self.value[self.linear_index(idx)]

    def empty_like(self):
        f = object.__new__(Field)
        f.__dict__.update(self.__dict__)
        f.value = np.zeros_like(self.value)
        return f


class _Geom:
    """Owner of an rh3t_geom handle (the C++ host build)."""

    def __init__(self, field, arcs=True):
        L = _lib.load()
        self.L = L
        ob, ib = field.outer_bound, field.inner_bound
        self._keep = []
        obc = (_lib.BC * len(field.bc_outer))(*[b.to_c() for b in field.bc_outer])
        ibc = (_lib.BC * max(1, len(field.bc_inner)))(*[b.to_c() for b in field.bc_inner])
        arc_list = (field.outer_arcs + field.inner_arcs) if arcs else []
        carcs = (_lib.Arc * max(1, len(arc_list)))(*[a.to_c() for a in arc_list])
        oxy, ixy = _arr(ob.points, np.float64), _arr(ib.points, np.float64)
        self._keep += [obc, ibc, carcs, oxy, ixy]
        h = C.c_void_p()
        grid, prm = field.grid.to_c(), field.params.to_c()
        rc = L.rh3t_geom_create(C.byref(grid), C.byref(prm), len(ob.points), oxy.ctypes.data, ob.fluid,
                                C.addressof(obc), len(ib.points), ixy.ctypes.data, ib.fluid, C.addressof(ibc),
                                len(arc_list), C.addressof(carcs), C.byref(h))
        if rc:
            raise RH3TError(rc, "geometry set-up failed")
        self.h = h
        self.n = field.grid.len()

    def fluid_mask(self):
        out = np.zeros(self.n, dtype=np.uint8)
        self.L.rh3t_geom_fluid_mask(self.h, out.ctypes.data)
        return out.astype(bool)

    def close(self):
        if self.h:
            self.L.rh3t_geom_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# ------------------------------------------------------------------ ghost.rs:30-118
class GhostGrid:
    """Static ghost layout: per ghost its grid index, final projection
    (P0, outward normal, signed distance), boundary and selected side, and for
    Wall / Outflow / FarField ghosts the GhostBC tables (bc1.rs:50-57)."""

    @classmethod
    def build(cls, field, n_threads=0, with_access=False, device=None):
        """GhostGrid::build (ghost.rs:50-118). device=None builds every table
        on the host; a device index computes the least-squares tables
        (bc1.rs:108-188) on that GPU (bit-identical results)."""
        if device is not None:
            return cls.build_many([field], device=device, n_threads=n_threads, with_access=with_access)[0]
        with _Geom(field) as geom:
            rc = geom.L.rh3t_geom_build_ghosts(geom.h, n_threads)
            if rc:
                raise RH3TError(rc, geom.L.rh3t_geom_last_error(geom.h).decode())
            return cls._from_geom(geom, field, with_access)

    @classmethod
    def build_many(cls, fields, device=0, n_threads=0, with_access=False):
        """GhostGrid::build of many fields at once, the least-squares tables of
        all their Wall / Outflow / FarField ghosts computed in one pass on
        GPU `device` (rh3t_geom_build_ghosts_device)."""
        geoms = [_Geom(f) for f in fields]
        try:
            L = geoms[0].L
            arr = (C.c_void_p * len(geoms))(*[g.h.value for g in geoms])
            rc = L.rh3t_geom_build_ghosts_device(len(geoms), arr, n_threads, device)
            if rc:
                msg = next((L.rh3t_geom_last_error(g.h).decode() for g in geoms if L.rh3t_geom_last_error(g.h)), "")
                raise RH3TError(rc, msg or "device ghost-grid build failed")
            return [cls._from_geom(g, f, with_access) for g, f in zip(geoms, fields)]
        finally:
            for g in geoms:
                g.close()

    @classmethod
    def _from_geom(cls, geom, field, with_access):
        g = cls()
        v = _lib.GhostTable()
        geom.L.rh3t_geom_ghost_table(geom.h, C.byref(v))
        n, m = v.n_ghosts, v.n_heavy

        def cp(ptr, count, dtype):
            if count == 0:
                return np.zeros(0, dtype=dtype)
            buf = (C.c_char * (count * np.dtype(dtype).itemsize)).from_address(ptr)
            return np.frombuffer(buf, dtype=dtype).copy()

        g.idx = cp(v.idx, 2 * n, np.int32).reshape(n, 2)
        g.boundary = cp(v.boundary, n, np.int32)
        g.side = cp(v.side, n, np.int32)
        g.proj = cp(v.proj, 5 * n, np.float64).reshape(n, 5)
        g.pre = cp(v.pre, n, np.int32)
        g.nearest = cp(v.nearest, 2 * m, np.int32).reshape(m, 2)
        g.stencil = cp(v.stencil, 55 * m, np.uint32).reshape(m, 55)
        g.s = cp(v.s, 979 * m, np.float64).reshape(m, 979)
        g.w = cp(v.w, 225 * m, np.float64).reshape(m, 225)
        g.d = cp(v.d, 5 * m, np.float64).reshape(m, 5)
        if with_access:
            g.access = np.zeros(field.grid.len() * 17, np.uint32)
            geom.L.rh3t_geom_access_table(geom.h, g.access.ctypes.data)
            g.access = g.access.reshape(-1, 17)
        return g

    @classmethod
    def from_arrays(cls, idx, boundary, side, proj, pre, nearest, stencil, s, w, d):
        """A GhostGrid handed over from another builder (the reference's Rust
        GhostGrid, or any table in the same layout)."""
        g = cls()
        g.idx = _arr(idx, np.int32).reshape(-1, 2)
        g.boundary, g.side, g.pre = _arr(boundary, np.int32), _arr(side, np.int32), _arr(pre, np.int32)
        g.proj = _arr(proj, np.float64).reshape(-1, 5)
        g.nearest = _arr(nearest, np.int32).reshape(-1, 2)
        g.stencil = _arr(stencil, np.uint32).reshape(-1, 55)
        g.s, g.w, g.d = (_arr(s, np.float64).reshape(-1, 979), _arr(w, np.float64).reshape(-1, 225),
                         _arr(d, np.float64).reshape(-1, 5))
        return g

    def len(self):
        return len(self.boundary)

    def n_heavy(self):
        return len(self.nearest)

    def to_c(self):
        t = _lib.GhostTable()
        t.n_ghosts, t.n_heavy = self.len(), self.n_heavy()
        t.idx, t.boundary, t.side, t.proj, t.pre = (_ptr(self.idx), _ptr(self.boundary), _ptr(self.side),
                                                    _ptr(self.proj), _ptr(self.pre))
        t.nearest, t.stencil, t.s, t.w, t.d = (_ptr(self.nearest), _ptr(self.stencil), _ptr(self.s), _ptr(self.w),
                                               _ptr(self.d))
        return t


# ------------------------------------------------------------------ device solver
class _SnapshotIO:
    """RH3TBIN1 snapshots, restart and the energy-split diagnostic of one
    instance (io.rs save_data / load_data, py_utils/energy_split.py)."""

    def snapshot(self, path, k=0):
        """Write instance k's state to `path` (RH3TBIN1); returns before the
        file is written (snapshot_wait joins)."""
        self._check(self.L.rh3t_snapshot(self.h, int(k), os.fsencode(path)))

    def snapshot_wait(self):
        self._check(self.L.rh3t_snapshot_wait(self.h))

    def save_data(self, filename, k=0, directory="data_new"):
        """io.rs:25-99 save_data: `directory`/`filename`, written through a
        .tmp file and a rename; waits for the file."""
        os.makedirs(directory, exist_ok=True)
        self.snapshot(os.path.join(directory, filename), k)
        self.snapshot_wait()

    def load_data(self, path, k=0):
        """io.rs:101-123 load_data: instance k's state and time from `path`."""
        self._check(self.L.rh3t_restart(self.h, int(k), os.fsencode(path)))

    def energy_split(self, k=0):
        """py_utils/energy_split.py for instance k: max, mean and rms of
        |Ee-Ei|, |Ee-Er|, |Ei-Er| over fluid nodes, and (x, y) of the max
        |Ee-Er| (first in j-major order)."""
        out = np.zeros(12)
        self._check(self.L.rh3t_energy_split(self.h, int(k), out.ctypes.data))
        names = ("max_Ee_Ei", "max_Ee_Er", "max_Ei_Er", "mean_Ee_Ei", "mean_Ee_Er", "mean_Ei_Er", "rms_Ee_Ei",
                 "rms_Ee_Er", "rms_Ei_Er", "x_max_Ee_Er", "y_max_Ee_Er")
        d = dict(zip(names, out[:11].tolist()))
        d["n_fluid"] = int(out[11])
        return d


class Solver(_SnapshotIO):
    """Device copy of a Field + GhostGrid + the l() scratch (main.rs:45-67):
    one rh3t_ctx on one CUDA stream.

    exact=True (default): librh3t_exact, the reference's expressions and
    roundings (no FMA contraction, IEEE quotients, correctly rounded pow);
    exact=False: librh3t, FMA contraction and shared reciprocals (faster; its
    roundings differ from the reference's by a few ulps per operation)."""

    def __init__(self, field, ghosts, device=0, exact=True):
        self.L = _lib.load(exact)
        self.exact = exact
        self.grid = field.grid
        self.n_ghosts = ghosts.len()
        obc = (_lib.BC * len(field.bc_outer))(*[b.to_c() for b in field.bc_outer])
        ibc = (_lib.BC * max(1, len(field.bc_inner)))(*[b.to_c() for b in field.bc_inner])
        fluid = _arr(field.fluid, np.uint8)
        table = ghosts.to_c()
        h = C.c_void_p()
        grid, prm = field.grid.to_c(), field.params.to_c()
        rc = self.L.rh3t_create(C.byref(grid), C.byref(prm), fluid.ctypes.data, len(field.bc_outer),
                                C.addressof(obc), len(field.bc_inner), C.addressof(ibc), C.byref(table), device,
                                C.byref(h))
        if rc:
            _raise_create(self.L, rc, "rh3t_create failed")
        self.h = h
        self.upload(field)

    def _check(self, rc):
        if rc:
            _raise_last(self.L, self.h, rc)

    def close(self):
        if getattr(self, "h", None):
            self.L.rh3t_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, field):
        v = _arr(field.value, np.float64)
        self._check(self.L.rh3t_upload_state(self.h, v.ctypes.data, field.time))

    def download(self, field=None):
        out = np.zeros((self.grid.len(), 6))
        t = C.c_double()
        self._check(self.L.rh3t_download_state(self.h, out.ctypes.data, C.byref(t)))
        if field is not None:
            fl = field.fluid
            field.value[fl] = out[fl]
            field.time = t.value
        return out, t.value

    def l(self, with_ghosts=False):
        rhs = np.zeros((self.grid.len(), 6))
        gv = np.zeros((self.n_ghosts, 6)) if with_ghosts else None
        self._check(self.L.rh3t_l(self.h, rhs.ctypes.data, _ptr(gv)))
        return (rhs, gv) if with_ghosts else rhs

    def calc_global_dt(self):
        d = C.c_double()
        self._check(self.L.rh3t_calc_global_dt(self.h, C.byref(d)))
        return d.value

    def rk3_ssp(self, dt):
        self._check(self.L.rh3t_rk3_ssp(self.h, float(dt)))

    def advance(self, nsteps, cfl_factor=0.05, t_final=math.inf, graph=True):
        self._check(self.L.rh3t_advance(self.h, int(nsteps), float(cfl_factor), float(t_final), int(bool(graph))))

    def step_host(self, value, time, cfl_factor=0.05):
        """One reference time-loop iteration on a host value array (in place)."""
        t = C.c_double(time)
        dt = C.c_double()
        self._check(self.L.rh3t_step_host(self.h, value.ctypes.data, C.byref(t), float(cfl_factor), C.byref(dt)))
        return t.value, dt.value

    def profile_steps(self, nsteps, cfl_factor=0.05):
        """Eager steps with CUDA events around every launch: device ms and
        launch counts per kernel class (ghosts, fluxes, rhs+stage, dt)."""
        ms = np.zeros(4)
        cnt = np.zeros(4, np.int64)
        self._check(self.L.rh3t_profile_steps(self.h, int(nsteps), float(cfl_factor), ms.ctypes.data, cnt.ctypes.data))
        return dict(zip(("ghosts", "flux", "rhs_stage", "dt"), zip(ms.tolist(), cnt.tolist())))

    def last_dt(self):
        d = C.c_double()
        self._check(self.L.rh3t_last_dt(self.h, C.byref(d)))
        return d.value

    def synchronize(self):
        self._check(self.L.rh3t_synchronize(self.h))

    @property
    def kernel_launches(self):
        return int(self.L.rh3t_kernel_launches(self.h))

    @property
    def stream(self):
        return self.L.rh3t_stream(self.h)


class Batch(_SnapshotIO):
    """Independent instances (Field + GhostGrid each, any sizes, parameters
    and BCs) resident together on one GPU (rh3t_batch_create). Every kernel
    launch covers all instances; each instance has its own dt reduction, time
    and error record, and advance() replays one CUDA graph per step of the
    whole batch. No reference counterpart: the reference runs one Field per
    process."""

    def __init__(self, fields, ghostgrids, device=0, exact=True):
        if len(fields) != len(ghostgrids) or not fields:
            raise ValueError("one GhostGrid per Field, at least one")
        self.L = _lib.load(exact)
        self.exact = exact
        self.n = len(fields)
        self.grids = [f.grid for f in fields]
        self.n_ghosts = [g.len() for g in ghostgrids]
        self.cells = np.array([f.grid.len() for f in fields], np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.cells)])
        keep = []  # the C views must outlive rh3t_batch_create
        desc = (_lib.Instance * self.n)()
        for k, (f, g) in enumerate(zip(fields, ghostgrids)):
            grid, prm = f.grid.to_c(), f.params.to_c()
            obc = (_lib.BC * max(1, len(f.bc_outer)))(*[b.to_c() for b in f.bc_outer])
            ibc = (_lib.BC * max(1, len(f.bc_inner)))(*[b.to_c() for b in f.bc_inner])
            fluid = _arr(f.fluid, np.uint8)
            table = g.to_c()
            keep += [grid, prm, obc, ibc, fluid, table]
            desc[k] = _lib.Instance(C.addressof(grid), C.addressof(prm), fluid.ctypes.data, len(f.bc_outer),
                                    C.addressof(obc), len(f.bc_inner), C.addressof(ibc), C.addressof(table))
        h = C.c_void_p()
        rc = self.L.rh3t_batch_create(self.n, C.addressof(desc), device, C.byref(h))
        if rc:
            _raise_create(self.L, rc, "rh3t_batch_create failed")
        self.h = h
        self.upload(fields)

    def _check(self, rc):
        if rc:
            _raise_last(self.L, self.h, rc)

    def close(self):
        if getattr(self, "h", None):
            self.L.rh3t_destroy(self.h)
            self.h = None

    __del__ = close

    def upload(self, fields):
        v = np.concatenate([_arr(f.value, np.float64).reshape(-1) for f in fields])
        t = np.array([f.time for f in fields], np.float64)
        self._check(self.L.rh3t_upload_batch(self.h, v.ctypes.data, t.ctypes.data))

    def upload_values(self, values, times):
        """values: all instances' value arrays concatenated (total_cells x 6)."""
        v = _arr(values, np.float64)
        t = _arr(times, np.float64)
        self._check(self.L.rh3t_upload_batch(self.h, v.ctypes.data, t.ctypes.data))

    def step_host(self, values, times, cfl_factor=0.05, groups=8):
        """One time-loop iteration of every instance on host arrays, in place
        (values: total_cells x 6, times: n; float64, C-contiguous; page-locked
        memory lets the copies of one instance group overlap the step of
        another)."""
        if values.dtype != np.float64 or not values.flags.c_contiguous or values.size != int(self.offsets[-1]) * 6:
            raise ValueError("values must be a C-contiguous float64 array of total_cells x 6")
        if times.dtype != np.float64 or not times.flags.c_contiguous or times.size != self.n:
            raise ValueError("times must be a C-contiguous float64 array of n instances")
        self._check(self.L.rh3t_step_host_batch(self.h, values.ctypes.data, times.ctypes.data, float(cfl_factor),
                                                int(groups)))
        return values, times

    def download_values(self, out=None, times=None):
        """(total_cells x 6 values of all instances, times[n]); out / times
        (float64, C-contiguous, e.g. pinned host memory) receive the copy
        when given."""
        if out is None:
            out = np.zeros((int(self.offsets[-1]), 6))
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size != int(self.offsets[-1]) * 6:
            raise ValueError("out must be a C-contiguous float64 array of total_cells x 6")
        t = np.zeros(self.n) if times is None else times
        self._check(self.L.rh3t_download_batch(self.h, out.ctypes.data, t.ctypes.data))
        return out, t

    def download(self, k=None):
        """[(value, time)] per instance, or one instance's (value, time)."""
        if k is not None:
            out = np.zeros((int(self.cells[k]), 6))
            t = C.c_double()
            self._check(self.L.rh3t_download_instance(self.h, int(k), out.ctypes.data, C.byref(t)))
            return out, t.value
        v, t = self.download_values()
        return [(v[self.offsets[k]:self.offsets[k + 1]], float(t[k])) for k in range(self.n)]

    def l(self, k, with_ghosts=False):
        rhs = np.zeros((int(self.cells[k]), 6))
        gv = np.zeros((self.n_ghosts[k], 6)) if with_ghosts else None
        self._check(self.L.rh3t_l_instance(self.h, int(k), rhs.ctypes.data, _ptr(gv)))
        return (rhs, gv) if with_ghosts else rhs

    def calc_global_dt(self):
        d = np.zeros(self.n)
        self._check(self.L.rh3t_calc_global_dt_batch(self.h, d.ctypes.data))
        return d

    def rk3_ssp(self, dt):
        self._check(self.L.rh3t_rk3_ssp(self.h, float(dt)))

    def advance(self, nsteps, cfl_factor=0.05, t_final=math.inf, graph=True):
        self._check(self.L.rh3t_advance(self.h, int(nsteps), float(cfl_factor), float(t_final), int(bool(graph))))

    def times(self):
        """(time, dt of the last step, steps taken) per instance"""
        t, dt, n = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n, np.int64)
        self._check(self.L.rh3t_instance_times(self.h, t.ctypes.data, dt.ctypes.data, n.ctypes.data))
        return t, dt, n

    def status(self):
        """per-instance status codes of the last synchronising call"""
        c = np.zeros(self.n, np.int32)
        self._check(self.L.rh3t_instance_status(self.h, c.ctypes.data))
        return c

    def set_tile_shapes(self, lg_fx, lg_fy, lg_rhs, k=-1):
        self._check(self.L.rh3t_set_tile_shapes(self.h, int(k), int(lg_fx), int(lg_fy), int(lg_rhs)))

    def tile_shapes(self, k):
        a = np.zeros(3, np.int32)
        self._check(self.L.rh3t_get_tile_shapes(self.h, int(k), a.ctypes.data))
        return tuple(int(x) for x in a)

    def autotune(self, cache_path=None, reps=5):
        """Time every admissible tile shape per (nx, ny, diffusion) class and
        apply the fastest; returns one dict per class."""
        out = (_lib.TuneEntry * 64)()
        n = C.c_int32()
        path = cache_path.encode() if cache_path else None
        self._check(self.L.rh3t_autotune(self.h, path, int(reps), C.addressof(out), 64, C.byref(n)))
        res = []
        for e in out[:n.value]:
            res.append(dict(nx=e.nx, ny=e.ny, diffusion=e.diffusion, n_instances=e.n_instances,
                            shape=(e.lg_fx, e.lg_fy, e.lg_rhs), from_cache=bool(e.from_cache),
                            ms_fx=list(e.ms_fx), ms_fy=list(e.ms_fy), ms_rhs=list(e.ms_rhs)))
        return res

    def profile_steps(self, nsteps, cfl_factor=0.05):
        ms = np.zeros(4)
        cnt = np.zeros(4, np.int64)
        self._check(self.L.rh3t_profile_steps(self.h, int(nsteps), float(cfl_factor), ms.ctypes.data, cnt.ctypes.data))
        return dict(zip(("ghosts", "flux", "rhs_stage", "dt"), zip(ms.tolist(), cnt.tolist())))

    # ---- adjoint (no reference counterpart)
    def l_vjp(self, k, rbar):
        """Cotangent of instance k's resident state for a cotangent rbar of
        its l() (nx*ny x 6); returns (ubar, pbar) with pbar = (FarField state
        (6), omega_ei, omega_er)."""
        rb = _arr(rbar, np.float64)
        ub = np.zeros((int(self.cells[k]), 6))
        pb = np.zeros(8)
        self._check(self.L.rh3t_l_vjp(self.h, int(k), rb.ctypes.data, ub.ctypes.data, pb.ctypes.data))
        return ub, pb

    def adjoint_forward(self, nsteps, cfl_factor=0.05, ckpt_every=20, max_records=None):
        """nsteps steps of every instance with checkpoints every ckpt_every;
        the last segments (as many as fit in a quarter of the free device
        memory, at most max_records when given) are kept recorded, so the
        reverse sweep does not recompute them."""
        if max_records is not None:
            self._check(self.L.rh3t_adjoint_max_records(self.h, int(max_records)))
        self._check(self.L.rh3t_adjoint_forward(self.h, int(nsteps), float(cfl_factor), int(ckpt_every)))

    def adjoint_records(self):
        """segment records the adjoint allocated"""
        return int(self.L.rh3t_adjoint_records(self.h))

    def adjoint_backward(self, dJ_du, out=None):
        """dJ_du: per-instance list of (nx*ny x 6) arrays or their
        concatenation. Returns ([dJ/du0 per instance], dJ/dparams (n x 8));
        out (total_cells x 6 float64, C-contiguous, e.g. pinned host memory)
        receives dJ/du0 when given."""
        if isinstance(dJ_du, (list, tuple)):
            dJ_du = np.concatenate([_arr(x, np.float64).reshape(-1, 6) for x in dJ_du])
        lam = _arr(dJ_du, np.float64)
        if out is None:
            g0 = np.zeros((int(self.offsets[-1]), 6))
        elif out.dtype != np.float64 or not out.flags.c_contiguous or out.size != int(self.offsets[-1]) * 6:
            raise ValueError("out must be a C-contiguous float64 array of total_cells x 6")
        else:
            g0 = out
        gp = np.zeros((self.n, 8))
        self._check(self.L.rh3t_adjoint_backward(self.h, lam.ctypes.data, g0.ctypes.data, gp.ctypes.data))
        return [g0[self.offsets[k]:self.offsets[k + 1]] for k in range(self.n)], gp

    def synchronize(self):
        self._check(self.L.rh3t_synchronize(self.h))

    @property
    def kernel_launches(self):
        return int(self.L.rh3t_kernel_launches(self.h))

    @property
    def stream(self):
        return self.L.rh3t_stream(self.h)


def fp64_peak_tflops(device=0):
    """Measured DFMA throughput of the device (TFLOP/s)."""
    L = _lib.load()
    t = C.c_double()
    rc = L.rh3t_fp64_peak(device, C.byref(t))
    if rc:
        raise RH3TError(rc, "fp64 peak probe failed")
    return t.value


# ------------------------------------------------------------------ main.rs functions
def l(u, ghosts, solver):
    """main.rs:135-305: semi-discrete operator of u; returns rhs (nx*ny x 6)."""
    solver.upload(u)
    return solver.l()


def calc_global_dt(u, solver):
    """main.rs:375-408"""
    solver.upload(u)
    return solver.calc_global_dt()


def rk3_ssp(u, ghosts, dt, solver):
    """main.rs:351-373: advances the host Field u in place by one SSP-RK3 step."""
    solver.upload(u)
    solver.rk3_ssp(dt)
    solver.download(u)
