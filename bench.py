"""Benchmark of the rh3t B200 solver: cell-updates/s of the SSP-RK3 step.

A step is one SSP-RK3 step (main.rs:459-466: dt = 0.05 * calc_global_dt, then
rk3_ssp) of every solver instance; a cell-update is one fluid node advanced by
one step. Default workload (batch256): 256 independent half-cylinder
instances of uneven size (nx in {61, 91, 121}, ny = 4 (nx - 1) + 1), inflow
Mach number and exchange coefficients (seeded, cases.batch_specs), advanced
together by the batched solver, each with its own dt; the line also carries
the plain solver run one instance at a time on the same instances. The plain
workloads are the reference's Mach-3 half-cylinder at h = 1/320 (cyl961,
961 x 3841 nodes), 1/160 and 1/40, and the planar shock. FP64 throughout.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--workload batch256|cyl961|cyl481|cyl121|planar] [--fma]

The benched build is librh3t_exact: the reference's expressions and
roundings (no FMA contraction, IEEE quotients, correctly rounded pow), the
build whose results are checked against the oracle at <= 1e-10 (the line's
`parity` object measures it on instances of the benched workload in the same
run). --fma benches librh3t (FMA contraction, shared reciprocals; faster,
its roundings differ from the reference's). The batched line also carries
the other build as a labelled second figure (`other_build`: its step time
and flux rate; `parity.other_build`: its deviation from the same oracle
runs); --no-other-build skips both.

--impl reference times the reference algorithm's CPU implementation (the
oracle restatement, OpenMP on all host cores; the Rust reference cannot be
built on this image) on the same workload and prints the same JSON line
(same metric, config, steps and warm-up; each step a bounded sample of the
workload, as its cpu_baseline.sample says).
Multi-GPU runs are independent replicas (one instance per GPU, no exchange):
value = all ranks' cell-updates / max-over-ranks device time.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "cyl961": dict(kind="cylinder", h=1.0 / 320.0, name="half-cylinder Mach-3, 961x3841 nodes (h=1/320)"),
    "cyl481": dict(kind="cylinder", h=1.0 / 160.0, name="half-cylinder Mach-3, 481x1921 nodes (h=1/160)"),
    "cyl121": dict(kind="cylinder", h=1.0 / 40.0, name="half-cylinder Mach-3, 121x481 nodes (h=1/40)"),
    "planar": dict(kind="planar", name="Mach-2 planar shock, 1024x8, y-periodic, diffusion+exchange on"),
    "batch256": dict(kind="batch", n=256, name="256 half-cylinder instances, nx in {61,91,121}, ny = 4(nx-1)+1, "
                     "Mach U[2,4], omega_ei/omega_er log-U[0.1,10] x 1.0, seed 20261203"),
    # the first 24 instances of batch256: the small case of the ncu captures
    "batch24": dict(kind="batch", n=24, name="the first 24 of the batch256 instances (profiling case)"),
}
PLANAR_PARAMS = dict(kappa_e=1e-3, kappa_i=1e-3, kappa_r=1e-3, omega_ei=1.0, omega_er=1.0, periodic_ly=0.03125)
CFL = 0.05
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one stage's
# fluxes on a plain workload, from an ncu capture of `bench.py --steps 3
# --warmup 3 --no-cpu --no-e2e` (FMA build, when x and y faces were one
# launch); None where no capture exists
FLUX_TRAFFIC_BYTES = {"fma": {"cyl961": 651.5e6}, "exact": {}}
# DRAM bytes per heavy ghost of one stage's ghost update (k_ghost_prep +
# k_ghosts) and per active face of one stage's k_flux<0> + k_flux<1>, from
# ncu captures on the batch24 workload (84,000 heavy ghosts, 860,240 x and
# 854,216 y faces), scaled by the heavy-ghost and face counts of the batched
# workloads. The no-contraction capture holds k_ghosts and both flux
# kernels; its ghost figure takes k_ghost_prep's bytes from the FMA-build
# capture (the same loads and stores in both builds).
GHOST_TRAFFIC_PER_HEAVY = {"fma": (902.88e6 + 7.24e6 + 15.32e6 + 9.25e6) / 84000,
                           "exact": (902.77e6 + 7.46e6 + 15.32e6 + 9.25e6) / 84000}
FLUX_TRAFFIC_PER_FACE = {"fma": (74.60e6 + 43.63e6) / 1714456,
                         "exact": (48.41e6 + 12.05e6 + 45.41e6 + 9.40e6) / 1714456}
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    """Measured copy bandwidth of this pool's B200s (GB/s) and its source."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s (of fallback)"


def make_field(rh, wl):
    spec = WORKLOADS[wl]
    if spec["kind"] == "cylinder":
        return rh.cases.init_cylinder(h=spec["h"])
    return rh.cases.planar_shock(params=rh.Params(**PLANAR_PARAMS))


def make_oracle(O, wl):
    spec = WORKLOADS[wl]
    if spec["kind"] == "cylinder":
        return O.Case.cylinder(h=spec["h"])
    return O.Case.planar_shock(**PLANAR_PARAMS)


def oracle_batch_case(O, sp):
    return O.Case.cylinder(h=sp["h"], mach=sp["mach"], omega_ei=sp["omega_ei"], omega_er=sp["omega_er"])


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def replica_value(ms_local, cells_local, steps, dist=None, device="cpu"):
    """Whole-job cell-updates/s of independent replicas: the sum of all ranks'
    cell-updates over the slowest rank's time (MAX all-reduce of the device
    times, SUM of the cells). Returns (value, max_ms)."""
    import torch
    if dist is None:
        return cells_local * steps / (ms_local * 1e-3), ms_local
    t = torch.tensor([ms_local], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor([float(cells_local)], dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    ms = float(t.item())
    return float(c.item()) * steps / (ms * 1e-3), ms


def batch_oracle_rate(O, specs, budget_s, max_steps=None):
    """Oracle cell-updates/s over the batch instances taken in order, one step
    each per round, until the time budget (or max_steps rounds) is spent."""
    cases, cells = [], []
    t_build = time.perf_counter()
    for sp in specs:
        cases.append(oracle_batch_case(O, sp))
        cells.append(int(cases[-1].fluid().sum()))
        if time.perf_counter() - t_build > budget_s:
            break
    build_s = time.perf_counter() - t_build
    done, steps, el = 0, 0, 0.0
    t0 = time.perf_counter()
    while True:
        for c, n in zip(cases, cells):
            c.run(1, CFL)
            done += n
        steps += 1
        el = time.perf_counter() - t0
        if el > budget_s or (max_steps is not None and steps >= max_steps):
            break
    return done / el, len(cases), steps, el, build_s


def cpu_baseline(O, wl, budget_s=20.0, specs=None):
    """The oracle (OpenMP, all host threads) on a bounded number of steps of the same workload,
    and a short one-thread sample beside it."""
    if specs is not None:
        threads = O.max_threads()
        v, n_inst, steps, el, build_s = batch_oracle_rate(O, specs, budget_s)
        O.set_threads(1)
        v1, n1, steps1, el1, _ = batch_oracle_rate(O, specs[:4], 3.0)
        O.set_threads(threads)
        return {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                "sample": f"{steps} SSP-RK3 step(s) of each of the first {n_inst} of the {len(specs)} instances, "
                          f"{el:.1f} s, after a {build_s:.1f} s ghost-grid build",
                "one_core": {"value": v1, "cores": 1,
                             "sample": f"{steps1} step(s) of the first {n1} instances, {el1:.1f} s"}}
    t0 = time.perf_counter()
    case = make_oracle(O, wl)
    build_s = time.perf_counter() - t0
    cells = int(case.fluid().sum())
    threads = O.max_threads()
    t0 = time.perf_counter()
    steps = 0
    while True:
        case.run(1, CFL)
        steps += 1
        el = time.perf_counter() - t0
        if el > budget_s or (el / steps) * (steps + 1) > budget_s * 1.5:
            break
    return {"value": cells * steps / el, "unit": "cell-updates/s", "cores": threads, "kind": "port",
            "sample": f"{steps} SSP-RK3 step(s) of the {wl} workload ({cells} fluid cells), "
                      f"{el:.1f} s, after a {build_s:.1f} s ghost-grid build"}


def rel_linf(a, b, mask):
    """Normwise relative L-infinity deviation per field over fluid nodes
    (max |a - b| / max |b|; both momentum components against the largest
    momentum magnitude)."""
    a, b = a[mask], b[mask]
    scale = np.abs(b).max(0)
    scale[1] = scale[2] = np.sqrt(b[:, 1] ** 2 + b[:, 2] ** 2).max()
    scale[scale == 0] = 1.0
    return np.abs(a - b).max(0) / scale


def batch_config(spec, specs, cells, ghosts, heavy, world, state_mb):
    """The `config` of a batch workload line: what defines the workload, the
    same for the repo arm and the reference arm."""
    classes = {}
    for sp in specs:
        classes[sp["nx"]] = classes.get(sp["nx"], 0) + 1
    return {"workload": spec["name"], "instances": len(specs), "instances_by_nx": classes,
            "scheme": "SSP-RK3, dt = 0.05 dt_cfl per step and instance", "fluid_cells": cells, "ghosts": ghosts,
            "heavy_ghosts": heavy, "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (state buffers 3 x %.0f MB)" % state_mb}


def run_reference(args):
    """The reference arm: the oracle (the reference algorithm restated in
    C++, OpenMP on all host threads) on the same workload, metric, config,
    step and warm-up counts. A step advances a bounded, rotating sample of
    the instances by one SSP-RK3 step each, sized so the whole run stays
    within about two minutes; the metric (cell-updates/s) is a rate."""
    from oracle import oracle as O
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    spec = WORKLOADS[args.workload]
    threads = O.max_threads()
    import importlib
    rh = importlib.import_module("3t_rh_b200")
    if spec["kind"] == "batch":
        specs = rh.cases.batch_specs(spec["n"])
        t0 = time.perf_counter()
        cases = [oracle_batch_case(O, sp) for sp in specs]
        build_s = time.perf_counter() - t0
        cells = [int(c.fluid().sum()) for c in cases]
        ghosts = sum(c.n_ghosts() for c in cases)
        heavy = sum(c.n_heavy() for c in cases)
        state_mb = 6 * 8 * sum((c.nx + 8) * (c.ny + 8) for c in cases) / 1e6
        total = sum(cells)
        # a short probe of one step per instance sizes the per-step sample
        t0 = time.perf_counter()
        probe = 0
        for c, n in zip(cases, cells):
            c.run(1, CFL)
            probe += n
            if time.perf_counter() - t0 > 2.0:
                break
        rate0 = probe / (time.perf_counter() - t0)
        budget = 120.0
        frac = min(1.0, budget * rate0 / (total * max(1, args.steps + args.warmup)))
        per_step = max(1, int(round(frac * total)))
        pos = [0]

        def step():
            done = 0
            while done < per_step:
                k = pos[0] % len(cases)
                cases[k].run(1, CFL)
                done += cells[k]
                pos[0] += 1
            return done

        for _ in range(args.warmup):
            step()
        t0 = time.perf_counter()
        done = 0
        for _ in range(args.steps):
            done += step()
        el = time.perf_counter() - t0
        v = done / el
        line = {"metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference",
                "config": batch_config(spec, specs, total, ghosts, heavy, args.gpus, state_mb),
                "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                                 "sample": f"each step advances the next instances of the {len(specs)} in turn by one "
                                           f"SSP-RK3 step until {per_step} fluid cells ({100 * per_step / total:.1f}% "
                                           f"of the workload's {total}) are advanced; {args.steps} timed steps, "
                                           f"{el:.1f} s; ghost-grid build {build_s:.1f} s not timed"},
                "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    case = make_oracle(O, args.workload)
    cells = int(case.fluid().sum())
    for _ in range(min(args.warmup, 1)):
        case.run(1, CFL)
    # each timed step is one full SSP-RK3 step; the number of steps is capped so
    # the run stays within a few minutes
    t0 = time.perf_counter()
    steps = 0
    while steps < args.steps:
        case.run(1, CFL)
        steps += 1
        if time.perf_counter() - t0 > 120.0:
            break
    el = time.perf_counter() - t0
    v = cells * steps / el
    line = {"metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": spec["name"], "fluid_cells": cells},
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                             "sample": f"{steps} of {args.steps} requested SSP-RK3 steps (capped at ~120 s)"},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


PARITY_SIZES = (61, 91, 121)


def parity_instances(rh, per_size=3):
    """The first `per_size` instances of each grid size of the batch256 workload."""
    specs_all = rh.cases.batch_specs(256)
    idx = []
    for nx in PARITY_SIZES:
        idx += [k for k, sp in enumerate(specs_all) if sp["nx"] == nx][:per_size]
    return idx, [specs_all[k] for k in idx]


def parity_record(rh, O, local, exact, steps=200, per_size=3, other_build=False):
    """The benched build against the oracle on instances of the batch256
    workload, advanced together for `steps` steps, each compared with the
    oracle (glibc pow, the reference's libm) and with the oracle built with
    the correctly rounded power the CUDA path computes. crpow_vs_oracle is
    how far that last-bit change of libm alone moves the reference
    algorithm. other_build: the other arithmetic build on the same instances
    against the same oracle runs (key `other_build`)."""
    idx, specs = parity_instances(rh, per_size)
    fields = [rh.cases.batch_field(sp) for sp in specs]
    grids = rh.GhostGrid.build_many(fields, device=local)
    runs = {}
    for ex in ((exact, not exact) if other_build else (exact,)):
        b = rh.Batch(fields, grids, device=local, exact=ex)
        b.advance(steps, CFL)
        runs[ex] = b.download()
        b.close()
    res = runs[exact]
    OC = O.crpow_variant()
    per, other = [], []
    t0 = time.perf_counter()
    for n, (k, sp, f, (u, _)) in enumerate(zip(idx, specs, fields, res)):
        ref, refc = oracle_batch_case(O, sp), oracle_batch_case(OC, sp)
        ref.run(steps, CFL)
        refc.run(steps, CFL)
        r, rc = ref.state(), refc.state()
        fl = f.fluid
        per.append({"instance": k, "nx": sp["nx"], "mach": round(sp["mach"], 4),
                    "vs_oracle": float(rel_linf(u, r, fl).max()),
                    "vs_oracle_crpow": float(rel_linf(u, rc, fl).max()),
                    "bitwise_vs_oracle_crpow": bool(np.array_equal(u[fl], rc[fl])),
                    "crpow_vs_oracle": float(rel_linf(rc, r, fl).max())})
        if other_build:
            uo = runs[not exact][n][0]
            other.append({"instance": k, "vs_oracle": float(rel_linf(uo, r, fl).max()),
                          "vs_oracle_crpow": float(rel_linf(uo, rc, fl).max())})
    rec = {"build": "no FMA contraction" if exact else "FMA contraction", "steps": steps,
            "instances_checked": len(per), "tolerance": 1e-10,
            "max_rel_linf_vs_oracle": max(p["vs_oracle"] for p in per),
            "max_rel_linf_vs_oracle_crpow": max(p["vs_oracle_crpow"] for p in per),
            "all_bitwise_vs_oracle_crpow": all(p["bitwise_vs_oracle_crpow"] for p in per),
            "max_crpow_vs_oracle": max(p["crpow_vs_oracle"] for p in per),
            "metric": "max over fields of max|gpu - oracle| / max|oracle| over fluid nodes",
            "oracle_s": round(time.perf_counter() - t0, 1), "per_instance": per}
    if other_build:
        rec["other_build"] = {"build": "FMA contraction" if exact else "no FMA contraction",
                              "max_rel_linf_vs_oracle": max(p["vs_oracle"] for p in other),
                              "max_rel_linf_vs_oracle_crpow": max(p["vs_oracle_crpow"] for p in other),
                              "per_instance": other}
    return rec


def scale_record(rh, torch, flops, local, exact, wl="cyl961", steps=20):
    """The plain solver on one large instance (the reference's half-cylinder
    at h = 1/320, 961 x 3841 nodes), the benched build: cell-updates/s over
    `steps` graph-replayed steps and the flux kernel's FP64 rate."""
    f = make_field(rh, wl)
    g = rh.GhostGrid.build_many([f], device=local)[0]
    s = rh.Solver(f, g, device=local, exact=exact)
    cells = int(f.fluid.sum())
    st = torch.cuda.ExternalStream(s.stream, device=torch.device(f"cuda:{local}"))
    s.advance(3, CFL)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    s.advance(steps, CFL)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    prof = s.profile_steps(5, CFL)
    nxf, nyf = flops.face_counts(f.fluid, f.grid.nx, f.grid.ny)
    fl_launch = flops.flux_launch_flops(nxf, nyf, False)
    flux_ms, flux_n = prof["flux"][0], 3 * 5  # per stage: the x-face and the y-face launch
    total = sum(v[0] for v in prof.values())
    s.close()
    return {"workload": WORKLOADS[wl]["name"], "fluid_cells": cells, "steps": steps, "ms_per_step": ms / steps,
            "value": cells * steps / (ms * 1e-3), "unit": "cell-updates/s",
            "flux_tflops": fl_launch / (flux_ms / flux_n * 1e-3) / 1e12,
            "kernel_share": {k: v[0] / total for k, v in prof.items()}}


def other_build_record(rh, torch, fields, grids, local, exact, cells, fl_launch, peak, steps=100):
    """The same batch in the other arithmetic build (FMA contraction when the
    benched build is the no-contraction one), a labelled second figure: the
    device-timed step over `steps` graph-replayed steps and the flux pair's
    FP64 rate. Its deviation from the oracle is in the parity record's
    `other_build`."""
    b = rh.Batch(fields, grids, device=local, exact=not exact)
    b.autotune(reps=3)
    st = torch.cuda.ExternalStream(b.stream, device=torch.device(f"cuda:{local}"))
    b.advance(5, CFL)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    b.advance(steps, CFL)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    prof = b.profile_steps(5, CFL)
    b.close()
    flux_stage_ms = prof["flux"][0] / (3 * 5)
    total = sum(v[0] for v in prof.values())
    fl_rate = fl_launch / (flux_stage_ms * 1e-3) / 1e12
    return {"build": "FMA contraction" if exact else "no FMA contraction", "steps": steps,
            "ms_per_step": ms / steps, "value": cells * steps / (ms * 1e-3), "unit": "cell-updates/s",
            "flux_tflops": fl_rate, "flux_frac_of_dfma": fl_rate / peak,
            "kernel_share": {k: v[0] / total for k, v in prof.items()},
            "note": "not the headline: on this workload its results are not within 1e-10 of the oracle "
                    "(parity.other_build)" if exact else "the build whose results are the reference's"}


def adjoint_bench(rh, torch, local, exact, nsteps=200, ckpt=20, n=32):
    """The adjoint workload: n seeded 121x481 half-cylinders (Mach U[2,4],
    exchange coefficients log-U[0.1,10]), J = surface pressure on the arc
    after nsteps, gradient with respect to the Mach number, the two exchange
    coefficients and the initial state, checkpoints every ckpt steps; device
    times of the forward solve and of the adjoint (checkpointed forward +
    reverse sweep)."""
    specs = rh.cases.batch_specs(n, sizes=(121,))
    fields = [rh.cases.batch_field(sp) for sp in specs]
    grids = rh.GhostGrid.build_many(fields, device=local)
    Js = [rh.cases.SurfacePressure(f, g) for f, g in zip(fields, grids)]
    dev = torch.device(f"cuda:{local}")

    def timed(fn, b):
        st = torch.cuda.ExternalStream(b.stream, device=dev)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(st)
        out = fn()
        e1.record(st)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1), 1e3 * (time.perf_counter() - t0)

    fwd = rh.Batch(fields, grids, device=local, exact=exact)
    fwd.advance(3, CFL)  # warm-up (graph capture)
    fwd.upload(fields)
    _, f_ms, f_wall = timed(lambda: fwd.advance(nsteps, CFL), fwd)
    fwd.close()
    b = rh.Batch(fields, grids, device=local, exact=exact)
    # warm-up with the timed run's checkpoint layout: its buffers (checkpoints,
    # the segment record) are allocated here, not inside the timed region
    b.adjoint_forward(nsteps, CFL, ckpt)
    b.adjoint_backward([np.zeros((int(c), 6)) for c in b.cells])
    b.upload(fields)

    # host buffers of the caller: pinned, as for any large device transfer
    total = int(b.offsets[-1])
    vals_h = torch.empty((total, 6), dtype=torch.float64, pin_memory=True).numpy()
    lam_h = torch.empty((total, 6), dtype=torch.float64, pin_memory=True).numpy()
    g0_h = torch.empty((total, 6), dtype=torch.float64, pin_memory=True).numpy()
    times_h = np.zeros(b.n)
    st = torch.cuda.ExternalStream(b.stream, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    def adjoint():
        ev[0].record(st)
        b.adjoint_forward(nsteps, CFL, ckpt)
        ev[1].record(st)
        b.download_values(out=vals_h, times=times_h)
        for k, J in enumerate(Js):
            o0, o1 = b.offsets[k], b.offsets[k + 1]
            lam_h[o0:o1] = J.grad(vals_h[o0:o1])
        ev[2].record(st)
        out = b.adjoint_backward(lam_h, out=g0_h)
        ev[3].record(st)
        return [(vals_h[b.offsets[k]:b.offsets[k + 1]], times_h[k]) for k in range(b.n)], out

    (res, (g0, gp)), a_ms, a_wall = timed(adjoint, b)
    n_rec = b.adjoint_records()
    lib_ms = ev[0].elapsed_time(ev[1]) + ev[2].elapsed_time(ev[3])
    dmach = []
    for k, sp in enumerate(specs):
        hm = 1e-7
        dudm = (rh.cases.freestream(sp["mach"] + hm) - rh.cases.freestream(sp["mach"] - hm)) / (2 * hm)
        dmach.append(float(gp[k, :6] @ dudm) + float((g0[k][fields[k].fluid] @ dudm).sum()))
    b.close()
    return {"workload": f"{n} half-cylinder instances 121x481, Mach U[2,4], omega log-U[0.1,10] x 1.0, "
                        f"seed 20261203; J = surface pressure on the arc after {nsteps} steps; gradient in Mach, "
                        f"omega_ei, omega_er and the initial state; checkpoints every {ckpt} steps",
            "forward_ms": f_ms, "adjoint_ms": a_ms, "adj_fwd_ratio": a_ms / f_ms,
            "adjoint_library_ms": lib_ms, "adj_fwd_ratio_library": lib_ms / f_ms,
            "segment_records": n_rec,
            "records_note": f"the forward run kept the records of its last {n_rec} of {-(-nsteps // ckpt)} segments "
                            "(as many as fit in a quarter of the free device memory): the reverse sweep "
                            "recomputes the others",
            "ratio_note": "adjoint_ms: checkpointed forward + download + host objective gradient + reverse sweep; "
                          "adjoint_library_ms: rh3t_adjoint_forward + rh3t_adjoint_backward only",
            "wall_ms": {"forward": f_wall, "adjoint": a_wall},
            "J_first": float(Js[0].value(res[0][0])), "dJ_dMach_first": dmach[0],
            "dJ_domega_first": [float(gp[0, 6]), float(gp[0, 7])]}


def run_batch(args, rh, flops, torch, dist, world, rank, local):
    """Batched workload: all instances in one Batch, one CUDA graph per step;
    then the plain solver on the same instances one at a time."""
    spec = WORKLOADS[args.workload]
    specs = rh.cases.batch_specs(spec["n"])
    t0 = time.perf_counter()
    fields = [rh.cases.batch_field(sp) for sp in specs]
    t1 = time.perf_counter()
    grids = rh.GhostGrid.build_many(fields, device=local)
    build_s = time.perf_counter() - t1
    fields_s = t1 - t0
    b = rh.Batch(fields, grids, device=local, exact=args.exact)
    cells = int(sum(int(f.fluid.sum()) for f in fields))
    tune = b.autotune(reps=5)
    step_fl, fl_launch, n_faces = 0.0, 0.0, 0
    for f, g in zip(fields, grids):
        nxf, nyf = flops.face_counts(f.fluid, f.grid.nx, f.grid.ny)
        n_faces += nxf + nyf
        step_fl += flops.step_flops(int(f.fluid.sum()), nxf, nyf, g.len(), g.n_heavy(), False, True)
        fl_launch += flops.flux_launch_flops(nxf, nyf, False)
    stream = torch.cuda.ExternalStream(b.stream, device=torch.device(f"cuda:{local}"))
    b.advance(args.warmup, CFL)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = b.kernel_launches
    ev0.record(stream)
    b.advance(args.steps, CFL)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = b.kernel_launches - l0
    value, ms = replica_value(ms, cells, args.steps, dist, f"cuda:{local}")
    sampler.stop()
    clocks = sampler.summary()
    k_prof = min(args.steps, 10)
    prof = b.profile_steps(k_prof, CFL)
    flux_ms, flux_n = prof["flux"][0], 3 * k_prof  # per stage: the x-face and the y-face launch
    achieved = fl_launch / (flux_ms / flux_n * 1e-3) / 1e12
    peak = rh.api.fp64_peak_tflops(local)
    total_prof_ms = sum(v[0] for v in prof.values())
    share = {k: v[0] / total_prof_ms for k, v in prof.items()}
    n_heavy = int(sum(g.n_heavy() for g in grids))
    ghost_stage_ms = prof["ghosts"][0] / (3 * k_prof)
    g_bytes = flops.ghost_launch_bytes(n_heavy)
    hbm, hbm_src = hbm_peak()
    g_achieved = g_bytes / (ghost_stage_ms * 1e-3) / 1e9
    bkey = "exact" if args.exact else "fma"
    rl_flux = {"bound": "fp64", "kernel": "k_flux<0> + k_flux<1> (x and y interface WENO5 fluxes of one stage, "
               "all instances)",
               "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
               "traffic": None if FLUX_TRAFFIC_PER_FACE[bkey] is None else FLUX_TRAFFIC_PER_FACE[bkey] * n_faces,
               "traffic_unit": "bytes per stage (both launches)",
               "peak_source": "measured DFMA loop on this GPU (rh3t_fp64_peak)",
               "flops_per_stage": fl_launch, "stage_ms": flux_ms / flux_n, "launches_per_stage": 2,
               "flop_count": "algorithmic: every add, sub, mul, div, sqrt of the reference's expressions = 1 "
                             "(a division costs 3-14 FP64 issue slots here)"}
    if args.exact:
        # every product and sum of the reference issues on its own: an FP64
        # stream without FMA peaks at half the DFMA FLOP rate
        rl_flux["no_fma_ceiling"] = peak / 2.0
        rl_flux["frac_of_no_fma_ceiling"] = achieved / (peak / 2.0)
    rl_ghost = {"bound": "hbm", "kernel": "k_ghost_prep + k_ghosts (one stage's ghost update, all instances)",
                "achieved": g_achieved, "peak": hbm, "unit": "GB/s", "frac": g_achieved / hbm,
                "traffic": None if GHOST_TRAFFIC_PER_HEAVY[bkey] is None else GHOST_TRAFFIC_PER_HEAVY[bkey] * n_heavy,
                "traffic_unit": "bytes per stage", "peak_source": hbm_src,
                "bytes_per_stage": g_bytes, "stage_ms": ghost_stage_ms,
                "bytes_model": f"{flops.HEAVY_GHOST_BYTES} B of GhostBC tables per heavy ghost x {n_heavy}"}
    dominant = "ghosts" if share["ghosts"] >= share["flux"] else "flux"
    roofline = dict(rl_ghost if dominant == "ghosts" else rl_flux)
    roofline.update({"kernel_share": share, "step_tflops": step_fl / (ms / args.steps * 1e-3) / 1e12,
                     "step_flops": step_fl, "other": {"flux": rl_flux} if dominant == "ghosts" else {"ghosts": rl_ghost}})

    # the plain GPU path on the same instances, one instance at a time
    k_plain = max(5, min(args.steps, 20))
    plain_ms, plain_cells = 0.0, 0
    for f, g in (zip(fields, grids) if not args.no_plain else ()):
        sv = rh.Solver(f, g, device=local, exact=args.exact)
        sv.advance(3, CFL)
        st = torch.cuda.ExternalStream(sv.stream, device=torch.device(f"cuda:{local}"))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        sv.advance(k_plain, CFL)
        e1.record(st)
        torch.cuda.synchronize()
        plain_ms += e0.elapsed_time(e1)
        plain_cells += int(f.fluid.sum())
        sv.close()
    plain_value = plain_cells * k_plain / (plain_ms * 1e-3) if plain_ms > 0 else None

    e2e = None
    if not args.no_e2e:
        vals, times = b.download_values()
        host = torch.empty(vals.shape, dtype=torch.float64, pin_memory=True).numpy()
        host[:] = vals
        times = np.ascontiguousarray(times)
        k_e2e = max(3, min(args.steps, 10))
        b.step_host(host, times, CFL, groups=args.e2e_groups)  # first call: its streams and buffer
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            b.step_host(host, times, CFL, groups=args.e2e_groups)
        el = time.perf_counter() - t0
        nb = host.size * 8
        e2e = {"value": world * cells * k_e2e / el, "unit": "cell-updates/s", "h2d_bytes_per_step": nb + 8 * b.n,
               "d2h_bytes_per_step": nb + 128 * b.n,
               "call": "rh3t_step_host_batch (every step: all Field::value arrays host -> device, one step, "
                       f"values and times device -> host; {args.e2e_groups} instance groups, the copies of one "
                       "overlapping the step of another; pinned host arrays; wall clock)",
               "steps": k_e2e}

    other = None
    if rank == 0 and world == 1 and not args.no_other_build:
        other = other_build_record(rh, torch, fields, grids, local, args.exact, cells, fl_launch, peak,
                                   steps=max(5, min(args.steps, 100)))

    adj = None
    if not args.no_adjoint:
        adj = adjoint_bench(rh, torch, local, args.exact, nsteps=args.adjoint_steps,
                            ckpt=min(20, args.adjoint_steps), n=args.adjoint_instances)

    cpu = parity = scale = None
    if rank == 0 and world == 1:
        from oracle import oracle as O  # timed CPU baseline and parity reference only
        if not args.no_cpu:
            cpu = cpu_baseline(O, args.workload, specs=specs)
        if not args.no_parity:
            parity = parity_record(rh, O, local, args.exact, steps=args.parity_steps,
                                   other_build=not args.no_other_build)
    if rank == 0 and world == 1 and not args.no_scale:
        scale = scale_record(rh, torch, flops, local, args.exact)

    if rank == 0:
        state_mb = 6 * 8 * sum((f.grid.nx + 8) * (f.grid.ny + 8) for f in fields) / 1e6
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": batch_config(spec, specs, cells, int(sum(g.len() for g in grids)),
                                   int(sum(g.n_heavy() for g in grids)), world, state_mb),
            "arithmetic": "no FMA contraction, IEEE quotients, correctly rounded pow (the reference's "
                          "roundings)" if args.exact else "FMA contraction, shared reciprocals",
            "setup": {"ghost_build_s": round(build_s, 3), "ghost_build": "rh3t_geom_build_ghosts_device",
                      "field_setup_s": round(fields_s, 3),
                      "tile_shapes": {f"{e['nx']}x{e['ny']}": e["shape"] for e in tune}},
            "parity": parity,
            "plain_at_scale": scale,
            "other_build": other,
            "instances_per_s": value / cells * b.n,
            "plain_one_at_a_time": None if plain_value is None else {
                "value": plain_value, "unit": "cell-updates/s", "steps_per_instance": k_plain,
                "batched_speedup": value / plain_value},
            "adjoint": adj,
            "roofline": roofline,
            "launch_gaps": {"graph_ms_per_step": ms / args.steps, "kernel_ms_per_step": total_prof_ms / k_prof,
                            "gap_fraction": 1.0 - (total_prof_ms / k_prof) / (ms / args.steps),
                            "note": "one step of the whole batch replays as one CUDA graph of "
                                    f"{launches // args.steps} kernels; kernel_ms_per_step sums CUDA-event "
                                    "durations of each kernel in eager profiled steps"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    b.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="batch256", choices=sorted(WORKLOADS))
    ap.add_argument("--fma", action="store_true", help="bench the FMA-contraction build (librh3t)")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle parity record")
    ap.add_argument("--parity-steps", type=int, default=200)
    ap.add_argument("--no-scale", action="store_true", help="skip the 961x3841 plain-solver record")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-groups", type=int, default=8, help="instance groups of the pipelined host step")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-other-build", action="store_true",
                    help="skip the labelled figure and parity of the other arithmetic build")
    ap.add_argument("--no-plain", action="store_true", help="skip the one-instance-at-a-time comparison")
    ap.add_argument("--adjoint-steps", type=int, default=200)
    ap.add_argument("--adjoint-instances", type=int, default=32)
    args = ap.parse_args()
    args.exact = not args.fma
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import importlib
    import torch

    rh = importlib.import_module("3t_rh_b200")
    from importlib import import_module
    flops = import_module("3t_rh_b200.flops")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))

    spec = WORKLOADS[args.workload]
    if spec["kind"] == "batch":
        run_batch(args, rh, flops, torch, dist, world, rank, local)
        if dist:
            dist.destroy_process_group()
        return
    f = make_field(rh, args.workload)
    t0 = time.perf_counter()
    g = rh.GhostGrid.build(f)
    build_s = time.perf_counter() - t0
    s = rh.Solver(f, g, device=local, exact=args.exact)
    cells = int(f.fluid.sum())
    nxf, nyf = flops.face_counts(f.fluid, f.grid.nx, f.grid.ny)
    diff = bool(any(getattr(f.params, k) != 0.0 for k in ("kappa_e", "kappa_i", "kappa_r")))
    src = bool(any(getattr(f.params, k) != 0.0 for k in ("omega_ei", "omega_er")))
    step_fl = flops.step_flops(cells, nxf, nyf, g.len(), g.n_heavy(), diff, src)
    stream = torch.cuda.ExternalStream(s.stream, device=torch.device(f"cuda:{local}"))

    s.advance(args.warmup, CFL)
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = s.kernel_launches
    ev0.record(stream)
    s.advance(args.steps, CFL)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = s.kernel_launches - l0
    value, ms = replica_value(ms, cells, args.steps, dist, f"cuda:{local}")
    sampler.stop()
    clocks = sampler.summary()

    # roofline of the dominant kernel: live per-launch durations (CUDA events)
    prof = s.profile_steps(min(args.steps, 20), CFL)
    flux_ms, flux_n = prof["flux"][0], 3 * min(args.steps, 20)  # per stage: the x-face and the y-face launch
    fl_launch = flops.flux_launch_flops(nxf, nyf, diff)
    achieved = fl_launch / (flux_ms / flux_n * 1e-3) / 1e12
    peak = rh.api.fp64_peak_tflops(local)
    total_prof_ms = sum(v[0] for v in prof.values())

    e2e = None
    if not args.no_e2e:
        n = f.grid.len()
        host = torch.empty((n, 6), dtype=torch.float64, pin_memory=True).numpy()
        u, tcur = s.download()
        host[:] = u
        k_e2e = max(3, min(args.steps, 20))
        s.step_host(host, tcur, CFL)  # warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            tcur, _dt = s.step_host(host, tcur, CFL)
        el = time.perf_counter() - t0
        e2e = {"value": world * cells * k_e2e / el, "unit": "cell-updates/s",
               "h2d_bytes_per_step": n * 6 * 8, "d2h_bytes_per_step": n * 6 * 8 + 16,
               "call": "rh3t_step_host (upload Field::value, dt reduction, rk3_ssp, download)", "steps": k_e2e}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O  # timed CPU baseline only
        cpu = cpu_baseline(O, args.workload)

    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": spec["name"], "scheme": "SSP-RK3, dt = 0.05 dt_cfl per step", "grid":
                       [f.grid.nx, f.grid.ny], "fluid_cells": cells, "ghosts": g.len(), "heavy_ghosts": g.n_heavy(),
                       "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2 (state buffers 3 x %.0f MB)" % (
                           6 * 8 * (f.grid.nx + 8) * (f.grid.ny + 8) / 1e6),
                       "ghost_build_s": round(build_s, 3)},
            "arithmetic": "no FMA contraction, IEEE quotients, correctly rounded pow (the reference's "
                          "roundings)" if args.exact else "FMA contraction, shared reciprocals",
            "roofline": {"bound": "fp64", "kernel": "k_flux<0> + k_flux<1> (x and y interface WENO5 fluxes of one "
                         "stage)", "achieved": achieved,
                         "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": FLUX_TRAFFIC_BYTES["exact" if args.exact else "fma"].get(args.workload),
                         "traffic_unit": "bytes per stage (both launches)",
                         "peak_source": "measured DFMA loop on this GPU (rh3t_fp64_peak)",
                         "flops_per_stage": fl_launch, "stage_ms": flux_ms / flux_n, "launches_per_stage": 2,
                         **({"no_fma_ceiling": peak / 2.0, "frac_of_no_fma_ceiling": achieved / (peak / 2.0)}
                            if args.exact else {}),
                         "kernel_share": {k: v[0] / total_prof_ms for k, v in prof.items()},
                         "step_tflops": step_fl / (ms / args.steps * 1e-3) / 1e12,
                         "step_flops": step_fl},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
