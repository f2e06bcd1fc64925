"""bench.py's JSON contract on CPU: the reference arm's line (the CPU restatement timed on
the host cores) carries every key of the contract, and the helpers that read the
committed ncu summaries find the per-cell traffic of the kernels the bench runs."""
import json
import subprocess
import sys
from pathlib import Path

import bench

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([s for s in r.stdout.splitlines() if s.startswith("{")][-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    # the CPU times a fixed sample cube of the 512^3 workload, and the line names it
    assert line["config"]["workload"].startswith(f"porous periodic {bench.CPU_N}^3")
    assert line["config"]["sampled_for"].startswith("porous periodic 512^3")
    assert f"best of {bench.CPU_REPEATS} runs" in line["cpu_baseline"]["sample"]
    cpu = line["cpu_baseline"]
    assert cpu["value"] == line["value"] and cpu["cores"] >= 1 and cpu["kind"] == "port" and cpu["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_roofline_traffic_comes_from_the_committed_summaries():
    assert bench.step_kernel("fp32", 512) == "aa_pair_kernel"
    assert bench.step_kernel("fp16dev", 512) == "aa_octo_even_kernel / aa_pair_split_kernel"
    assert bench.step_kernel("fp64", 512) == "aa_step_kernel"
    for storage, algorithmic in (("fp32", 153), ("fp16dev", 77)):
        t = bench.profiled_traffic(storage, 512)
        assert t is not None
        per_cell = t / 512 ** 3
        assert 0.9 * algorithmic < per_cell < 1.1 * algorithmic, (storage, per_cell)
