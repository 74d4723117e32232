"""The `rpba` executable (rpba.cpp:45-176 over the C ABI) without a GPU:
the reference's `parameters` file is read (every key required, as
rpba.cpp:56-64 reads them), the BAL file parsed, and the reference's header
lines printed -- input file, flags, threads, cameras / points /
observations, unknowns and redundancy (rpba.cpp:194-205) -- before the
solve, which then reports the missing device and exits with status 2."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "rpba_b200", "rpba")

pytestmark = pytest.mark.skipif(not os.path.exists(EXE), reason="executable not built")


def _run(cwd, args=()):
    import torch
    env = dict(os.environ)
    if not torch.cuda.is_available():
        env["CUDA_VISIBLE_DEVICES"] = ""
    return subprocess.run([EXE, *args], cwd=cwd, env=env, capture_output=True, text=True, timeout=120)


@pytest.fixture
def workdir(tmp_path, oracle_mod):
    import rpba_b200 as rb
    from rpba_b200 import scenes
    blk = scenes.to_block(scenes.arc_scene(seed=2, n_cams=6, n_pts=80))
    (tmp_path / "data").mkdir()
    rb.OutputBlock(str(tmp_path / "data" / "scene.txt"), blk, k24out=True)
    return tmp_path, blk


def _params(path, **over):
    kv = {"InputDir": "data", "File": "scene.txt", "Robust": "1", "Exteval": "0", "Threads": "1", "k2": "1",
          "k4": "1", "f": "1", "k24out": "1"}
    kv.update(over)
    path.write_text("".join(f"{k}={v}\n" for k, v in kv.items() if v is not None))


def test_header_and_missing_device(workdir):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the solve would run")
    d, blk = workdir
    _params(d / "parameters", Threads="3", k4="0")
    r = _run(d)
    out = r.stdout
    nobs = blk.n_obs
    nadd = 2
    unk = 3 * blk.n_points + (blk.n_images - 2) * 6 + 5 + blk.n_images * nadd
    assert "Inputfile: data/scene.txt" in out
    assert "Robustflag: 1" in out and "Threads: 3" in out
    assert "K2: 1\nK4: 0\nFocal length: 1" in out
    assert f"Cameras: {blk.n_images}  Points: {blk.n_points} Observations {nobs}" in out
    assert f"Unknowns {unk}  Redundancy {2 * nobs - unk}" in out
    assert "no CUDA device" in r.stderr
    assert r.returncode == 2


@pytest.mark.parametrize("missing", ["InputDir", "Robust", "k24out", "Threads"])
def test_missing_key(workdir, missing):
    d, _ = workdir
    _params(d / "parameters", **{missing: None})
    r = _run(d)
    assert r.returncode == 1
    assert f"parameters: missing key {missing}" in r.stderr


def test_no_parameters_file_and_extra_argument(workdir):
    d, _ = workdir
    r = _run(d)
    assert r.returncode == 1 and 'cannot read file "parameters"' in r.stderr
    _params(d / "parameters")
    r = _run(d, ["x"])
    assert r.returncode == 1 and "Parameter file not used" in r.stdout


def test_partitioned_branch_header(tmp_path, oracle_mod):
    """Threads selects the reference's parallel branch where its rule does
    (min(Threads, iround(images / 70)) > 1, rpbacore.cpp:79-92): the
    '#threads' line and one 'Thread:' line per partition, then the device is
    needed; Threads=1 keeps the global branch."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the solve would run")
    import rpba_b200 as rb
    from rpba_b200 import scenes
    blk = scenes.to_block(scenes.arc_scene(seed=2, n_cams=150, n_pts=600))
    (tmp_path / "data").mkdir()
    rb.OutputBlock(str(tmp_path / "data" / "scene.txt"), blk, k24out=True)
    _params(tmp_path / "parameters", Threads="4")
    r = _run(tmp_path)
    assert "#threads: 2 2" in r.stdout
    lines = [l for l in r.stdout.splitlines() if l.startswith("Thread: ")]
    assert len(lines) == 2 and sum(int(l.split()[3]) for l in lines) == blk.n_images
    assert "no CUDA device" in r.stderr and r.returncode == 2
    # the global branch below the rule's threshold: no partition lines
    _params(tmp_path / "parameters", Threads="1")
    r = _run(tmp_path)
    assert "#threads" not in r.stdout and r.returncode == 2


def test_partition_count_follows_the_reference_rule(oracle_mod):
    """rpba_partition_count against the rule restated by the oracle
    (min(Threads, iround(images / 70)), partitioned above 1 with more than
    five images, never with Exteval), including the rounding at the halves."""
    import os
    import rpba_b200 as rb
    L = rb.load()
    for n in (5, 6, 50, 104, 105, 106, 139, 140, 175, 13700):
        for t in (1, 2, 3, 8, 64, 500):
            want = oracle_mod.parallel_threads(n, t)
            want = want if want > 1 and n > 5 else 1
            assert L.rpba_partition_count(n, t, 0) == want, (n, t)
            assert L.rpba_partition_count(n, t, 1) == 1
    hw = os.cpu_count() or 1
    assert L.rpba_partition_count(13700, 0, 0) == max(1, min(hw, 196)) if min(hw, 196) > 1 else 1
