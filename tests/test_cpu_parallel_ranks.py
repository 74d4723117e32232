"""The parallel RPBA over ranks (rpba_calc_plsa_parallel_ranks: one scene,
its partitions dealt to the ranks, the partition steps' results exchanged
by an all-gather after every round of steps) checked without a GPU.

The hosted form binds the oracle's partition step and merge, and the ranks
are gloo processes on this host exchanging through torch.distributed.  The
result on every rank must equal the oracle's one-process loop
(oracle_calc_plsa_parallel, rpbacore.cpp:100-510) bit for bit -- cameras,
points, tracks, sigma0, iterations and log -- whatever the number of ranks,
including ranks that own no partition.  A failed all-gather ends the call
with RPBA_ERR_COMM, and a partition step that fails on one rank is reported
by every rank."""
import ctypes as C
import multiprocessing as mp
import socket
import time
from datetime import timedelta

import numpy as np
import pytest

NAMES = ("pmat", "K", "distpara", "XX", "pt_obs_off", "pt_obs_image", "pt_obs_slot")
STEP_ARGS = (C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32,
             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t)


def _scene(case):
    from rpba_b200 import scenes
    if case == "arc":
        return scenes.to_block(scenes.arc_scene(seed=5, n_cams=50, n_pts=8000)), 4
    if case == "street":  # the street workload at full size: 1,000 cameras, 943k observations
        return scenes.to_block(scenes.make_scene(1, scale=1.0)), 8
    return scenes.to_block(scenes.city_scene(seed=8, n_clusters=3, cams_per_cluster=20, n_pts=8000)), 3


def _steps(oracle_mod):
    O = oracle_mod.lib()
    return C.cast(O.oracle_lsa_gcp_step_full, C.c_void_p), C.cast(O.oracle_merge, C.c_void_p)


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


OPTS = {"": {}, "plain": {"robust": False}, "noadd": {"addflags": (False, False, False)}}


def _rank_worker(rank, world, port, case, fail_rank, q, opts=""):
    try:
        import torch.distributed as dist
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                                timeout=timedelta(seconds=60))
        import oracle
        import rpba_b200 as rb
        from rpba_b200 import lib
        from rpba_b200.replicas import bytes_allgather
        blk, k = _scene(case)
        part = rb.partition_images(blk, k)
        step, merge = _steps(oracle)
        failing = None
        if rank == fail_rank:  # a partition step that reports a failed direct solve
            failing = C.CFUNCTYPE(C.c_int32, *STEP_ARGS)(lambda *a: 10)
            step = C.cast(failing, C.c_void_p)
        st, b, s, log = lib.calc_plsa_parallel_ranks(blk, part, k, rank, world, bytes_allgather(),
                                                     steps=(step, merge), **OPTS[opts])
        q.put(("ok", rank, st, {n: getattr(b, n) for n in NAMES}, s, log))
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        q.put(("err", rank, repr(e)))


def _run(world, case, fail_rank=-1, timeout=300, opts=""):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_rank_worker, args=(r, world, port, case, fail_rank, q, opts)) for r in range(world)]
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
        p.join(timeout=10)
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda r: r[1])


@pytest.fixture(scope="module")
def oracle_loops(oracle_mod):
    import rpba_b200 as rb
    res = {}
    for case in ("arc", "city", "street"):
        blk, k = _scene(case)
        part = rb.partition_images(blk, k)
        res[case] = oracle_mod.calc_plsa_parallel(blk, part, k, rb.make_options())
    blk, k = _scene("arc")
    part = rb.partition_images(blk, k)
    res["arc/plain"] = oracle_mod.calc_plsa_parallel(blk, part, k, rb.make_options(robust=False))
    blk, k = _scene("city")
    part = rb.partition_images(blk, k)
    res["city/noadd"] = oracle_mod.calc_plsa_parallel(blk, part, k, rb.make_options(k2=False, k4=False, f=False))
    return res


def _same(st, b, s, log, ref):
    st_o, b_o, s_o, log_o = ref
    assert st == st_o == 0
    assert s == s_o
    for n in NAMES:
        assert np.array_equal(b[n] if isinstance(b, dict) else getattr(b, n), getattr(b_o, n)), n
    assert log == log_o


def test_one_rank_through_the_exchange_equals_oracle_loop(oracle_mod, oracle_loops):
    """One rank with an all-gather that returns its own bytes: the exchange
    path runs (records written and read back) and the loop is unchanged."""
    import rpba_b200 as rb
    from rpba_b200 import lib
    blk, k = _scene("arc")
    part = rb.partition_images(blk, k)
    calls = []

    def gather(data):
        calls.append(len(data))
        return data

    st, b, s, log = lib.calc_plsa_parallel_ranks(blk, part, k, 0, 1, gather, steps=_steps(oracle_mod))
    _same(st, b, s, log, oracle_loops["arc"])
    assert len(calls) == 2 * (s["iterations"] - 1)  # sizes and records after every round of steps


@pytest.mark.parametrize("world,case,opts", [(2, "arc", ""), (3, "city", ""), (4, "city", ""), (2, "arc", "plain"),
                                             (2, "city", "noadd"), (4, "street", "")])
def test_ranks_equal_oracle_loop(oracle_loops, world, case, opts):
    """world 4 with 3 partitions: one rank owns none and only exchanges;
    also without robust reweighting and without additional parameters."""
    out = _run(world, case, opts=opts)
    assert len(out) == world, out
    for r in out:
        assert r[0] == "ok", r
        _same(r[2], r[3], r[4], r[5], oracle_loops[case + ("/" + opts if opts else "")])


def test_failed_allgather_is_reported(oracle_mod):
    import rpba_b200 as rb
    from rpba_b200 import lib
    blk, k = _scene("arc")
    part = rb.partition_images(blk, k)

    def gather(data):
        raise ConnectionError("planted: the transport failed")

    st = lib.calc_plsa_parallel_ranks(blk, part, k, 0, 1, gather, steps=_steps(oracle_mod))[0]
    assert st == 12  # RPBA_ERR_COMM


def test_step_failure_on_one_rank_is_returned_by_every_rank():
    out = _run(2, "arc", fail_rank=1)
    assert len(out) == 2, out
    assert [r[0] for r in out] == ["ok", "ok"], out
    assert [r[2] for r in out] == [10, 10]


def test_bad_rank_arguments(oracle_mod):
    import rpba_b200 as rb
    from rpba_b200 import lib
    blk, k = _scene("arc")
    part = rb.partition_images(blk, k)
    for rank, world in ((1, 1), (-1, 2), (0, 0)):
        st = lib.calc_plsa_parallel_ranks(blk, part, k, rank, world, lambda d: d * max(world, 1),
                                          steps=_steps(oracle_mod))[0]
        assert st == 1, (rank, world)


def _bench_worker(rank, world, port, q):
    try:
        import argparse
        import os
        import sys
        sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
        import bench
        from rpba_b200.replicas import Group
        g = Group(rank, world, backend="gloo", timeout_s=60.0, init_method=f"tcp://127.0.0.1:{port}")
        args = argparse.Namespace(ranks_scale=0.01, seed_offset=0)
        q.put(("ok", rank, bench.partitioned_over_ranks(args, g, 0)))
        g.close()
    except Exception as e:  # reported to the parent
        q.put(("err", rank, repr(e)))


def _has_cuda():
    import torch
    return torch.cuda.is_available()


@pytest.mark.skipif(_has_cuda(), reason="the failure it plants is the absence of a GPU")
def test_bench_leg_reports_a_failure_on_every_rank_without_hanging():
    """bench.py's one-scene-over-ranks leg takes the same collective steps on
    every rank whatever fails: here every rank fails to reach a GPU (none on
    this host) and both ranks return the leg's record with the errors."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = []
    deadline = time.time() + 240
    while len(out) < 2 and time.time() < deadline:
        try:
            out.append(q.get(timeout=max(0.1, deadline - time.time())))
        except Exception:
            break
    for p in ps:
        p.join(timeout=10)
        if p.is_alive():
            p.kill()
    assert len(out) == 2, out
    for r in out:
        assert r[0] == "ok", r
        assert r[2]["ranks"] == 2 and len(r[2]["errors"]) == 2, r[2]
