"""BAL text I/O of large files runs in parallel (token-indexed parse,
per-thread output buffers).  Forced onto small files here through the
RPBA_IO_* environment knobs, it must give exactly what the serial path and
the oracle's reader give, whatever the line layout."""
import os

import numpy as np
import pytest

FIELDS = ("pmat", "K", "distpara", "XX", "img_obs_off", "xg", "wx", "wy", "wxy", "pt_obs_off", "pt_obs_image",
          "pt_obs_slot")


@pytest.fixture
def io_mode():
    saved = {k: os.environ.get(k) for k in ("RPBA_IO_PARALLEL_MIN_BYTES", "RPBA_IO_THREADS")}

    def set_mode(parallel: bool, threads: int = 5):
        os.environ["RPBA_IO_PARALLEL_MIN_BYTES"] = "0" if parallel else str(1 << 60)
        os.environ["RPBA_IO_THREADS"] = str(threads)

    yield set_mode
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v


def _one_value_per_line(src, dst):
    """Rewrite a BAL file in the layout of the public BAL files: observations
    one per line, then every camera and point value on its own line, with
    CRLF ends and stray tabs."""
    lines = open(src).read().split("\n")
    n_obs = int(lines[0].split()[2])
    out = [lines[0]] + [l.replace(" ", "\t", 1) for l in lines[1:1 + n_obs]]
    for l in lines[1 + n_obs:]:
        out += l.split()
    open(dst, "w", newline="").write("\r\n".join(out) + "\r\n")


def test_parallel_parse_matches_serial_and_oracle(tmp_path, oracle_mod, io_mode):
    import rpba_b200 as rb
    from rpba_b200 import scenes
    bal = scenes.arc_scene(seed=11, n_cams=23, n_pts=4000)
    p1, p2 = str(tmp_path / "a.txt"), str(tmp_path / "b.txt")
    scenes.write_bal(p1, bal)
    _one_value_per_line(p1, p2)
    for path in (p1, p2):
        for k24 in (True, False):
            ref = oracle_mod.input_block(path, k24)
            io_mode(False)
            ser = rb.InputBlock(path, 3, k24)
            for threads in (2, 7, 32):
                io_mode(True, threads)
                par = rb.InputBlock(path, 3, k24)
                for n in FIELDS:
                    assert np.array_equal(getattr(par, n), getattr(ser, n)), (path, k24, threads, n)
                    assert np.array_equal(getattr(par, n), getattr(ref, n)), (path, k24, threads, n)


def test_parallel_write_is_byte_identical(tmp_path, io_mode):
    import rpba_b200 as rb
    from rpba_b200 import scenes
    bal = scenes.arc_scene(seed=12, n_cams=17, n_pts=3000)
    p = str(tmp_path / "in.txt")
    scenes.write_bal(p, bal)
    blk = rb.InputBlock(p)
    io_mode(False)
    rb.OutputBlock(str(tmp_path / "s.txt"), blk.copy())
    io_mode(True, 6)
    rb.OutputBlock(str(tmp_path / "p.txt"), blk.copy())
    assert open(tmp_path / "s.txt", "rb").read() == open(tmp_path / "p.txt", "rb").read()


def test_parallel_parse_rejects_truncated_and_bad(tmp_path, io_mode):
    import rpba_b200 as rb
    from rpba_b200 import scenes
    bal = scenes.arc_scene(seed=13, n_cams=9, n_pts=500)
    p = str(tmp_path / "a.txt")
    scenes.write_bal(p, bal)
    text = open(p).read()
    cut = str(tmp_path / "cut.txt")
    open(cut, "w").write(text[: len(text) * 2 // 3])
    bad = str(tmp_path / "bad.txt")
    lines = text.split("\n")
    lines[5] = "0 999999 1.0 2.0"  # point index out of range
    open(bad, "w").write("\n".join(lines))
    for parallel in (False, True):
        io_mode(parallel, 4)
        for path in (cut, bad):
            with pytest.raises(Exception):
                rb.InputBlock(path)
