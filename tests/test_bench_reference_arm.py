"""bench.py --impl reference (the reference algorithm's CPU implementation,
timed on the host cores) keeps the bench line's contract: one JSON line with
the same metric, unit, step and warm-up counts and the same `config` keys as
the GPU arm, `impl` = "reference", a cpu_baseline describing the run and an
e2e object without host-device copies; under torchrun only rank 0 prints.
Run on the small batch workload (the first 24 batch instances)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CMD = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "batch24",
       "--steps", "1", "--warmup", "3"]


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run(CMD, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    return [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_line():
    lines = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference"
    assert d["metric"] == "cell-updates/s" and d["unit"] == "cell-updates/s"
    assert d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 3
    # the GPU arm builds its config with the same function (bench.batch_config)
    assert set(d["config"]) == {"workload", "instances", "instances_by_nx", "scheme", "fluid_cells", "ghosts",
                                "heavy_ghosts", "parallelism", "l2"}
    assert d["config"]["instances"] == 24
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    assert _run({"RANK": "1", "WORLD_SIZE": "2"}) == []
