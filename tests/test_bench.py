"""bench.py on the CPU: the reference arm's JSON line (the oracle port timed on
the host cores) carries the keys the benchmark contract asks for and the same
`config` object as the GPU arm, and the roofline fields the GPU arm reads from
the committed ncu summary of the headline kernel parse."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_profile_fields_parse():
    traffic = bench.profile_traffic("ensemble_4000x40")
    # DRAM bytes per launch: the replica state and the staged protein
    # conformations, about 1.7 MB
    assert traffic is not None and 1e6 < traffic < 1e7
    for key in ("sm__pipe_fma_cycles_active.avg.pct_of_peak_sustained_active",
                "sm__inst_executed_pipe_xu.avg.pct_of_peak_sustained_active"):
        v = bench.profile_metric("ensemble_4000x40", key)
        assert v is not None and 0.0 < v[0] <= 100.0


@pytest.mark.timeout(300)
def test_reference_arm_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], cwd=ROOT, capture_output=True, text=True,
                         timeout=280)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "replica-MC-steps/s" and line["unit"] == "replica-MC-steps/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    # the same workload description as the GPU arm's line
    w, cx, _ = bench.build_workload("ensemble_4000x40", 2024, oracle_tables=True)
    assert line["config"] == bench.workload_config(w, cx, 1)
