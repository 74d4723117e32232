"""The multi-GPU form is independent replicas: host-side timing and
reductions over ranks, tested here with world-size-2 gloo ranks on CPU, each
rank solving its own small scene with the CPU oracle.  A planted failure
(one rank raising before its first collective) must end the other rank's
next collective with an error within the group's short timeout."""
import multiprocessing as mp
import os
import socket
import time

import pytest


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, fail_rank, q):
    try:
        from rpba_b200.replicas import Group, time_steps
        import oracle
        import rpba_b200 as rb
        from rpba_b200 import scenes
        g = Group(rank, world, backend="gloo", timeout_s=15.0, init_method=f"tcp://127.0.0.1:{port}")
        blk = scenes.to_block(scenes.make_scene(0, scale=0.3, seed=500 + rank))
        reps = []

        def step():
            if rank == fail_rank:
                raise RuntimeError("planted failure")
            t0 = time.perf_counter()
            st, _, rep, _ = oracle.calc_plsa(blk, rb.make_options())
            reps.append(rep)
            return time.perf_counter() - t0

        res = time_steps(g, step, steps=2, warmup=1)
        stats = g.gather({"rank": rank, "rms": reps[-1]["rms"], "median": res["median"]})
        q.put(("ok", rank, res, stats))
        g.close()
    except Exception as e:  # reported to the parent
        q.put(("err", rank, repr(e)))


def _run(world, fail_rank, timeout):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, fail_rank, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = []
    deadline = time.time() + timeout
    while len(out) < world and time.time() < deadline:
        try:
            out.append(q.get(timeout=max(0.1, deadline - time.time())))
        except Exception:
            break
    for p in ps:
        p.join(timeout=5)
        if p.is_alive():
            p.kill()
    return out


def test_replicas_max_over_ranks_gloo():
    out = _run(2, -1, 240)
    assert len(out) == 2 and all(o[0] == "ok" for o in out), out
    by = {o[1]: o for o in out}
    meds = [by[r][2]["median"] for r in (0, 1)]
    for r in (0, 1):
        assert by[r][2]["max_over_ranks"] == pytest.approx(max(meds))
        stats = by[r][3]
        assert [s["rank"] for s in stats] == [0, 1]
        assert stats[0]["rms"] != stats[1]["rms"]  # each rank solved its own scene


def test_replicas_failure_surfaces_as_error_not_hang():
    t0 = time.time()
    out = _run(2, 1, 120)
    assert time.time() - t0 < 120
    by = {o[1]: o for o in out}
    assert by[1][0] == "err" and "planted failure" in by[1][2]
    assert 0 in by and by[0][0] == "err", out  # the survivor's collective failed
