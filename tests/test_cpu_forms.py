"""The per-form command (python -m rpba_b200.forms) rejects unknown forms
and configurations before it generates a scene or touches a device."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    return subprocess.run([sys.executable, "-m", "rpba_b200.forms", *args], cwd=ROOT, capture_output=True,
                          text=True, timeout=120)


def test_unknown_form_is_an_argument_error():
    r = _run("--forms", "plain,cholmod")
    assert r.returncode == 2
    assert "unknown form 'cholmod'" in r.stderr


def test_unknown_config_is_an_argument_error():
    r = _run("--config", "4")
    assert r.returncode == 2
    assert "invalid choice" in r.stderr


def test_partitioned_form_reports_its_partition_count_and_status():
    """The partitioned form's line: the reference's partition count for this
    host's cores and the call's status (on a host without a GPU, "no CUDA
    device" from the first merge pass)."""
    import json
    r = _run("--config", "1", "--scale", "0.2", "--forms", "partitioned", "--repeats", "1")
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["form"] == "partitioned" and line["n_images"] == 200
    assert line["partitions"] == min(os.cpu_count() or 1, 3)
    assert "status" in line
