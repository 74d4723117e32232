"""bench.py's reference arm (the CPU oracle on a bounded sample) runs
without a GPU and prints the contract's JSON line: impl, metric and unit,
the sample's description, the e2e object and, beside the global LSA's
time, the partitioned branch's (cpu_baseline.parallel)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line(oracle_mod):
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--cpu-sample-scale", "0.002"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"].startswith("s to converge at matched final RMS")
    assert line["unit"] == "s" and line["higher_is_better"] is False and line["value"] > 0
    assert line["e2e"] == {"value": line["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] == 1 and cb["status"] == 0 and "sample" in cb
    par = cb["parallel"]
    if par is not None:
        assert par["status"] == 0 and par["partitions"] >= 2 and par["value"] > 0
        assert abs(par["exteval_sigma0"] - par["global_exteval_sigma0"]) < 0.05 * par["global_exteval_sigma0"]
