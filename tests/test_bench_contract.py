"""bench.py's reference arm (the CPU restatement on the host's cores) prints the contract's JSON
line on the same workload description as the GPU arm. Runs on the CPU."""

import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_reference_arm_json_line():
    import bench
    from hasteboots_b200 import tfhe
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--preset", "0", "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "bootstraps/s"
    assert line["higher_is_better"] is True and line["value"] > 0
    assert line["steps"] == 1 and line["warmup"] == 1 and line["n_gpus"] == 1
    assert line["dtype"] == "u32"
    # the GPU arm names the same workload
    params = tfhe.Parameters.preset(0)
    expect = bench.gates_workload(16384, params.name.replace("_PARAMETERS", ""), params.raw)
    assert line["config"]["workload"] == expect
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["value"] == line["value"] and cb["cores"] >= 1 and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": "bootstraps/s",
                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
