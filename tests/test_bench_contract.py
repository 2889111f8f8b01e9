"""The bench's one-line JSON contract, checked on small networks: every key the
line promises, with values of the right kind.  The reference arm (the
reference's kernels on the host cores) runs without a GPU; our arm needs one."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BASE_KEYS = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
             "scaling", "vs_baseline", "dtype", "data", "config"}


def bench_line(*args, timeout=900):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                       capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def check_base(d, steps, warmup):
    assert BASE_KEYS <= set(d), BASE_KEYS - set(d)
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["steps"] == steps and d["warmup"] == warmup and d["n_gpus"] == 1
    assert d["higher_is_better"] is True and d["scaling"] in ("weak", "strong")
    assert d["config"]["workload"].startswith("tensile_")
    assert d["config"]["l2"].startswith("working set within")  # small networks stay in L2


def test_reference_arm_line():
    d = bench_line("--impl", "reference", "--steps", "2", "--warmup", "3", "--fibres", "100")
    check_base(d, 2, 3)
    assert d["impl"] == "reference"
    cb = d["cpu_baseline"]
    assert {"value", "unit", "cores", "kind", "sample"} <= set(cb)
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


@pytest.mark.gpu
def test_our_arm_line():
    d = bench_line("--steps", "8", "--warmup", "3", "--fibres", "400", "--no-extras", "--cpu-seconds", "2")
    check_base(d, 8, 3)
    assert d.get("impl", "ours") == "ours"
    rl = d["roofline"]
    assert {"bound", "achieved", "peak", "unit", "frac", "traffic"} <= set(rl)
    assert rl["bound"] == "hbm" and rl["unit"] == "GB/s" and 0 < rl["frac"] < 2
    assert abs(rl["frac"] - rl["achieved"] / rl["peak"]) < 1e-9
    e2e = d["e2e"]
    assert {"value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"} <= set(e2e)
    assert 0 < e2e["value"] and e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    assert d["gpu_launches"] > 0
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(d["clocks"])
    assert d["cpu_baseline"]["value"] > 0
