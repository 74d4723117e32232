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
