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


def test_shard_balances_and_is_deterministic():
    from rpba_b200.replicas import shard
    from rpba_b200 import scenes
    costs = [kw["n_cams"] for kw in scenes.batch_scene_specs()]
    for world in (1, 2, 3, 8):
        own = shard(costs, world)
        assert own == shard(costs, world) and sorted(set(own)) == list(range(world))
        load = [sum(c for c, o in zip(costs, own) if o == r) for r in range(world)]
        assert max(load) - min(load) <= max(costs)


def _scene_worker(rank, world, port, q):
    try:
        from rpba_b200.replicas import Group, scene_parallel
        import oracle
        import rpba_b200 as rb
        from rpba_b200 import scenes
        g = Group(rank, world, backend="gloo", timeout_s=30.0, init_method=f"tcp://127.0.0.1:{port}")
        specs = scenes.batch_scene_specs(n_scenes=6, cmin=8, cmax=16, pts_per_cam=40)

        def solve(idx):
            t0 = time.perf_counter()
            out = []
            for i in idx:
                st, _, rep, _ = oracle.calc_plsa(scenes._arc_block(specs[i]), rb.make_options())
                out.append({"status": st, "rms": rep["rms"], "rank": rank})
            return out, time.perf_counter() - t0

        res = scene_parallel(g, [kw["n_cams"] for kw in specs], solve)
        q.put(("ok", rank, res))
        g.close()
    except Exception as e:
        q.put(("err", rank, repr(e)))


def test_scene_parallel_gloo():
    """Batched scenes split over two gloo ranks: every scene solved exactly
    once, by its owner, results gathered in scene order on both ranks, job
    time = max over the ranks' times."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_scene_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=240) for _ in range(2)]
    for p in ps:
        p.join(timeout=10)
    assert all(o[0] == "ok" for o in out), out
    by = {o[1]: o[2] for o in out}
    for r in (0, 1):
        res = by[r]
        assert len(res["scenes"]) == 6 and all(s is not None and s["status"] == 0 for s in res["scenes"])
        assert [s["rank"] for s in res["scenes"]] == res["owner"]
        assert res["job_seconds"] == pytest.approx(max(by[0]["rank_seconds"], by[1]["rank_seconds"]))
    assert by[0]["scenes"] == by[1]["scenes"]
    assert set(by[0]["owner"]) == {0, 1}
