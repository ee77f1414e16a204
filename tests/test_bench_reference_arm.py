"""CPU tests of bench.py's reference arm, the line the headline ratio is
computed against: `bench.py --impl reference` times the reference's
estimator (the oracle restatement, FP64, all host threads) on rank 0 and
prints one JSON line with the same metric, unit and config as this build's
arm, a cpu_baseline describing the run and an e2e object without copies;
every other rank exits 0 without work."""

from __future__ import annotations

import json
import os
import subprocess
import sys

from conftest import REPO


def _run(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "1", "--cpu-seconds", "1"], cwd=REPO, env=env, capture_output=True,
                          text=True, timeout=300)


def test_reference_arm_prints_one_contract_line():
    out = _run()
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["unit"] == "samples/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the same workload and threshold as this build's headline line
    assert d["config"]["workload"].startswith("learned proposal (config 4)")
    assert d["config"]["threshold"] == 0.005 and d["config"]["rays_per_sample"] == [100000, 1000000]


def test_reference_arm_other_ranks_exit_without_work():
    out = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
