"""Work over ranks: one process per GPU.

The reference's global LSA does not shard (one linear system per LM step);
its own parallel form partitions the scene into independent LSAs
(rpbacore.cpp:100-510).  Across GPUs this library therefore splits work that
is independent by nature:

* one scene in the partitioned form: the partitions' steps dealt to the
  ranks, their results all-gathered after every round of steps
  (rpba_calc_plsa_parallel_ranks, whose transport is ``bytes_allgather``);
* replicas (one scene): every rank solves its own copy; the job's time is
  the slowest rank's (max over ranks);
* scene-parallel (many independent scenes, the batched workload): the scenes
  are dealt to ranks by size (``shard``), every rank solves its share, the
  per-scene results are gathered in scene order and the job's time is the
  slowest rank's (``scene_parallel``).

Only these host-side exchanges cross ranks, through torch.distributed
(NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import statistics
from datetime import timedelta
from typing import Callable


class Group:
    """torch.distributed plumbing of a replica job (world 1: no-op)."""

    def __init__(self, rank: int, world: int, backend: str = "nccl", timeout_s: float = 600.0,
                 device=None, init_method: str | None = None):
        import torch.distributed as dist
        self.rank, self.world, self.dist = rank, world, dist
        self.device = device
        if world > 1 and not dist.is_initialized():
            kw = {"timeout": timedelta(seconds=timeout_s)}
            if init_method:
                kw.update(init_method=init_method, rank=rank, world_size=world)
            if device is not None and backend == "nccl":
                kw["device_id"] = device
            dist.init_process_group(backend, **kw)

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """Max over ranks (every rank gets it)."""
        if self.world == 1:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64,
                         device=self.device if self.device is not None else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def gather(self, obj) -> list:
        """Every rank's object, in rank order (on every rank)."""
        if self.world == 1:
            return [obj]
        out = [None] * self.world
        self.dist.all_gather_object(out, obj)
        return out

    def close(self):
        if self.world > 1 and self.dist.is_initialized():
            self.dist.barrier()
            self.dist.destroy_process_group()


def bytes_allgather(device=None):
    """An all-gather of byte strings over the default torch.distributed
    group, as rpba_calc_plsa_parallel_ranks wants it: every rank passes the
    same number of bytes and gets every rank's, concatenated in rank order
    (one rank, no group: its own).  ``device``: where the buffers go for
    the collective (a CUDA device with NCCL; None with gloo)."""
    import torch
    import torch.distributed as dist

    def gather(data: bytes) -> bytes:
        if not dist.is_initialized() or dist.get_world_size() == 1:
            return data
        t = torch.frombuffer(bytearray(data), dtype=torch.uint8) if data else torch.empty(0, dtype=torch.uint8)
        if device is not None:
            t = t.to(device)
        outs = [torch.empty_like(t) for _ in range(dist.get_world_size())]
        dist.all_gather(outs, t)
        return b"".join(o.cpu().numpy().tobytes() for o in outs)

    return gather


def time_steps(g: Group, step: Callable[[], float], steps: int, warmup: int,
               before_step: Callable[[], None] | None = None) -> dict:
    """Warm-up, then `steps` timed calls of `step` (which returns its own
    device-measured seconds), a barrier before every step.  Returns this
    rank's step times, its median, and the max of the medians over ranks."""
    for _ in range(warmup):
        step()
    times = []
    for _ in range(steps):
        if before_step is not None:
            before_step()
        g.barrier()
        times.append(float(step()))
    g.barrier()
    med = statistics.median(times)
    return {"times": times, "median": med, "max_over_ranks": g.max(med)}


def shard(costs, world: int) -> list:
    """Owner rank of every item: largest first to the least-loaded rank
    (ties: lower index, lower rank), deterministic on every rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += costs[i]
    return owner


def scene_parallel(g: Group, costs, solve: Callable[[list], tuple]) -> dict:
    """Solve independent scenes split over the ranks.  ``solve(indices)``
    runs this rank's scenes and returns (per-scene result dicts in the order
    of ``indices``, its seconds).  Returns, on every rank, the results of all
    scenes in scene order, the owner of each, and the job's seconds (max over
    ranks of the ranks' seconds)."""
    owner = shard(costs, g.world)
    mine = [i for i, r in enumerate(owner) if r == g.rank]
    g.barrier()
    results, secs = solve(mine)
    job = g.max(secs)
    merged = [None] * len(costs)
    for part in g.gather(list(zip(mine, results))):
        for i, res in part:
            merged[i] = res
    return {"scenes": merged, "owner": owner, "job_seconds": job, "rank_seconds": secs}
