"""The benchmark's reference arm (the FP64 C++ restatement on the host cores) prints one JSON
line that the GPU arm's line can be compared with: same metric name, unit, direction and
workload description, plus its own CPU-baseline and end-to-end entries.  Runs on CPU (one
oracle step of the 6 x 128^3 workload)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    sys.path.insert(0, ROOT)
    import bench
    from solar_b200 import configs

    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC
    assert line["unit"] == "grid-pt RK4 updates/s" and line["higher_is_better"] is True
    assert line["config"] == bench.run_config(configs.get("c2"), 1)
    assert line["value"] > 0 and line["steps"] == 1
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
