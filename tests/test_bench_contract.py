"""The reference arm of ``bench.py`` runs on the host alone: its JSON line
keeps the benchmark contract (metric, unit, direction, e2e with no copies,
a CPU baseline describing the run), and ranks other than 0 print nothing."""
import json
import os
import subprocess
import sys

import pytest

from tests.conftest import ROOT


def run_bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, env=e, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return [json.loads(line) for line in out.stdout.splitlines() if line.startswith("{")]


@pytest.mark.parametrize("workload,extra", [
    ("fba", ["--envs", "64", "--cpu-sample", "12"]),
    ("cooperative", ["--envs", "16", "--coop-sample", "2"]),
])
def test_reference_arm_line(workload, extra):
    lines = run_bench("--impl", "reference", "--workload", workload, "--steps", "1", "--warmup", "0", *extra)
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference" and d["unit"] == "LPs/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0 and d["n_gpus"] == 1
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert d["data"].startswith("synthetic") and "workload" in d["config"]
    assert d["ms_per_step"] > 0 and d["vs_baseline"] is None


def test_reference_arm_other_ranks_print_nothing():
    assert run_bench("--impl", "reference", "--steps", "1", "--warmup", "0", "--envs", "16",
                     env={"RANK": "1"}) == []


def test_reference_arm_step_is_the_bounded_sample():
    """The reference arm's step is its bounded HiGHS sample: ms_per_step is
    that sample's wall time, and the full step's time is a projection."""
    d = run_bench("--impl", "reference", "--steps", "1", "--warmup", "0", "--envs", "32", "--cpu-sample", "6")[0]
    assert d["ms_per_step"] < d["projected_full_step_ms"]
    assert d["config"]["lps_per_step"] == 96 and "sample" in d["step"]


def test_gpus_flag_launches_that_many_ranks():
    """``--gpus 2`` outside torchrun re-launches the command as two ranks on
    this node; rank 0 alone prints the one line."""
    lines = run_bench("--gpus", "2", "--impl", "reference", "--steps", "1", "--warmup", "0", "--envs", "16",
                      "--cpu-sample", "6")
    assert len(lines) == 1 and lines[0]["n_gpus"] == 2 and lines[0]["impl"] == "reference"
