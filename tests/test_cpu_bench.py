"""bench.py's reference arm (the CPU oracle on a bounded sample) runs
without a GPU and prints the contract's JSON line: impl, metric and unit,
the workload's config, the sample's description and scale factor, the e2e
object, the partitioned branch (the reference's Threads=0 path, the value)
and the single-threaded global LSA beside it; and it loads no GPU code --
only the oracle's library."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line(oracle_mod):
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                        "--scale", "0.02", "--ref-sample-scale", "0.01", "--cpu-sample-scale", "0.004"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"].startswith("s to converge at matched final RMS")
    assert line["unit"] == "s" and line["higher_is_better"] is False and line["value"] > 0
    assert line["e2e"] == {"value": line["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["config"]["workload"].startswith("city") and line["config"]["n_obs"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and "sample" in cb and cb["value"] == line["value"]
    assert abs(cb["sample_seconds"] * cb["scale_factor"] - cb["value"]) <= 1e-9 * cb["value"]
    assert abs(cb["scale_factor"] - line["config"]["n_obs"] / int(cb["sample"].split("points, ")[1].split()[0])) < 1e-6
    par = cb["partitioned"]
    if par is not None:
        assert par["status"] == 0 and par["partitions"] >= 2 and par["value"] > 0 and cb["cores"] == par["cores"]
    g = cb["global_lsa"]
    assert g["status"] == 0 and g["cores"] == 1 and g["value"] > 0
    libs = line["loaded_repo_libraries"]
    assert libs == ["oracle/_build/liboracle.so"], libs
