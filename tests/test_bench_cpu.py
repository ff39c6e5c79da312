"""bench.py on the CPU: the reference arm's JSON line keeps the contract, and the committed
profile files carry the per-cell traffic and instruction counts that the live bench reads."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3", "--size", "1024", "--window-steps", "1"], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "cell-updates/s"
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    # the reference arm times the window state the GPU arm's CPU baseline uses
    assert line["config"]["same_state_as"] == "the b200 arm's cpu_baseline"
    assert "from its FP64 state after 60 s from dry" in line["cpu_baseline"]["sample"]


@pytest.mark.parametrize("name", ["sweep_interior_kernel_f32_datum64", "sweep_interior_kernel_f64", "sweep_kernel_f32_datum64",
                                  "sweep_batch_kernel_f32_datum64", "stage_kernel_f64"])
def test_profile_files_carry_what_the_bench_reads(name):
    sys.path.insert(0, ROOT)
    import bench
    traffic = bench.profile_traffic(f"{name}_2048_traffic.json")
    inst = bench.profile_traffic(f"{name}_2048_traffic.json", "warp_inst_per_cell_per_launch")
    assert traffic and 40.0 < traffic < 200.0
    assert inst and 20.0 < inst < 200.0
    assert os.path.exists(os.path.join(ROOT, "profiles", f"{name}_config2.md"))
