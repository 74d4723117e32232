#!/usr/bin/env python
"""Seconds to converge at matched final RMS reprojection error on one B200:
the learned-PCG solver against the plain one.

One step = one complete robust bundle adjustment (the reference's stop rule:
two LM passes, robust reweighting, RobustDelete) of a seeded synthetic scene
that is already resident in HBM, timed on the device (CUDA events around the
whole LM run).  The default workload is the city scene (13,700 cameras in 50
clustered blocks, 4.5M points, ~29M observations).

  ours   the learned two-level PCG solver in the mixed-precision form: FP32
         Jacobians / Schur blocks, the learned block-Jacobi correction plus
         the aggregate coarse space, inexact Newton with relative residual
         tolerance --tol, weights from rpba_b200/precond_weights.npy
  plain  the plain FP64 GPU solver: the reference's block-Jacobi PCG and its
         stop rule (the drop-in form), timed in the same run

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

value = ours' median seconds; "plain" carries the plain solver's time and the
matched-RMS check (ours' final RMS <= plain's x (1 + 1e-6)).  With N > 1
(torchrun, one rank per GPU) every rank solves its own copy of the scene
(independent replicas, no collective on the data path); the value is the
slowest rank's time.  ``--impl reference`` times the reference algorithm's
CPU implementation (the C++ restatement under oracle/, single-threaded like
the reference's global LSA) on a bounded sample of the workload, rank 0 only;
beside it ("parallel") the reference's partitioned branch, which it takes
with more than one thread, on the same sample with the host's cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s to converge at matched final RMS reproj error: learned-PCG vs plain, 1 B200"
UNIT = "s"
WORKLOADS = {
    4: "batch: 256 independent arc scenes of 20-400 cameras (scene-parallel over ranks)",
    0: "arc: 50 cameras, 8k points, ~32k observations",
    1: "street: 1000 cameras, 190k points, ~950k observations",
    2: "aerial: 3000 cameras, 310k points, ~1.65M observations",
    3: "city: 13700 cameras in 50 clusters, 4.5M points, ~29M observations",
}
RMS_MATCH = 1e-6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--tol", type=float, default=3e-5, help="relative PCG tolerance of the learned solver")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain solver")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-scale", type=float, default=0.01,
                    help="scale of the scene the CPU baseline solves (bounded sample)")
    ap.add_argument("--ref-sample-scale", type=float, default=0.04,
                    help="scale of the scene one step of --impl reference solves (bounded sample)")
    ap.add_argument("--seed-offset", type=int, default=0, help="generator seed offset (another scene)")
    ap.add_argument("--no-ablation", action="store_true", help="skip the preconditioner ablation solves")
    ap.add_argument("--batch-scenes", type=int, default=256, help="--config 4: scenes of the batched workload")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--ranks-scale", type=float, default=0.1,
                    help="scale of the city-family scene the partitioned branch solves over the ranks")
    ap.add_argument("--no-ranks", action="store_true", help="skip the partitioned branch over the ranks")
    return ap.parse_args()


def peaks():
    """HBM copy bandwidth (GB/s) from MEASURED_PEAKS.json (key hbm_gbs, a
    number or an object holding one), else the pool's earlier measurement."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            v = json.load(fh)["hbm_gbs"]
        if isinstance(v, dict):
            v = next(x for k, x in v.items() if isinstance(x, (int, float)) and k in ("value", "burst", "gbs"))
        return float(v), "measured"
    except (OSError, ValueError, KeyError, TypeError, StopIteration):
        return 6650.0, "fallback"


def traffic_ratio():
    """DRAM bytes / algorithmic bytes of the PCG kernel from the committed ncu
    summary (measured on a smaller case of the same scene family)."""
    path = os.path.join(ROOT, "profiles", "k_pcg_traffic.txt")
    if not os.path.exists(path):
        return None, None
    with open(path) as fh:
        for line in fh:
            if line.startswith("traffic_over_algorithmic:"):
                return float(line.split(":")[1]), "profiles/k_pcg_traffic.txt"
    return None, None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the run."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if gpu_id:
            cmd += ["-i", gpu_id]
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(cmd, stdout=self.fh, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 8:
                    continue
                try:
                    sm.append(float(parts[0]))
                    smax.append(float(parts[1]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[4:8]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def block_bytes(b) -> int:
    return int(sum(getattr(b, n).nbytes for n in ("pmat", "K", "distpara", "XX", "img_obs_off", "xg", "wx",
                                                     "wy", "wxy", "pt_obs_off", "pt_obs_image", "pt_obs_slot")))


def state_bytes(b) -> int:
    return int(sum(getattr(b, n).nbytes for n in ("pmat", "K", "distpara", "XX", "pt_obs_off", "pt_obs_image",
                                                     "pt_obs_slot")))


def make_block(config, scale, seed_offset=0):
    from rpba_b200 import scenes
    return scenes.to_block(scenes.make_scene(config, scale=scale, seed=20260 + config + seed_offset))


def pinned_copy(blk):
    """The block with every array in page-locked host memory (the e2e
    inputs are copied to the device from pinned memory)."""
    import torch
    from rpba_b200.block import Block, _ARRAYS
    keep, arrs = [], []
    for n in _ARRAYS:
        a = np.ascontiguousarray(getattr(blk, n))
        t = torch.empty(max(a.nbytes, 1), dtype=torch.uint8, pin_memory=True)
        keep.append(t)
        v = t.numpy()[:a.nbytes].view(a.dtype).reshape(a.shape)
        v[...] = a
        arrs.append(v)
    return Block(*arrs, _keep=keep)


def pinned_out(blk):
    """Page-locked arrays for the result (cameras, points, tracks); the
    observation arrays, which a solve does not change, are the block's."""
    import torch
    from rpba_b200.block import Block, _ARRAYS
    keep, arrs = [], []
    for n in _ARRAYS:
        a = np.ascontiguousarray(getattr(blk, n))
        if n in ("pmat", "K", "distpara", "XX", "pt_obs_off", "pt_obs_image", "pt_obs_slot"):
            t = torch.empty(max(a.nbytes, 1), dtype=torch.uint8, pin_memory=True)
            keep.append(t)
            a = t.numpy()[:a.nbytes].view(a.dtype).reshape(a.shape)
        arrs.append(a)
    return Block(*arrs, _keep=keep)


def learned_weights():
    from rpba_b200 import train_precond
    w = train_precond.load()
    if w is None:
        raise RuntimeError("rpba_b200/precond_weights.npy is missing: python -m rpba_b200.train_precond")
    return w


def cpu_sample(config, scale):
    """The oracle (C++ restatement of the reference's global LSA, one thread)
    on a bounded sample: one complete solve of a scene of the same family at
    `scale` of the workload's size."""
    import oracle
    import rpba_b200 as rb
    blk = make_block(config, scale)
    t0 = time.perf_counter()
    st, out, rep, _ = oracle.calc_plsa(blk, rb.make_options(solver=rb.SOLVER_PCG))
    return time.perf_counter() - t0, rep, st, blk, out


def cpu_sample_parallel(blk, out_global):
    """The reference's partitioned branch (Threads=0: min(host cores,
    iround(images / 70)) partitions, rpbacore.cpp:79-92, 100-510) as restated
    by the oracle, on the same sample, partition included in the time;
    None when that sample takes the global branch.  The partition (the
    stand-in for METIS) is the copy compiled into the oracle's library, so
    this leg loads no GPU code."""
    import oracle
    threads = oracle.parallel_threads(blk.n_images, os.cpu_count() or 1)
    if threads < 2 or blk.n_images <= 5:
        return None
    t0 = time.perf_counter()
    part = oracle.partition_images(blk, threads)
    st, out, stats, _ = oracle.calc_plsa_parallel(blk, part, threads)
    dt = time.perf_counter() - t0
    ev = lambda b: oracle.exteval(b)[1]["exteval_sigma0"]
    return {"value": dt, "unit": UNIT, "cores": threads, "partitions": threads, "status": st,
            "outer_iterations": stats["iterations"], "exteval_sigma0": ev(out),
            "global_exteval_sigma0": ev(out_global) if out_global is not None else None,
            "note": "Threads=0 branch of the reference: partition, per-partition GCP steps, CalcLSAXMulti merge"}


def rooflines(kstats, hbm, peak_kind):
    """Per-kernel device time share, achieved GB/s of its algorithmic bytes
    (counted per launch by the library) and fraction of the HBM peak, for
    every kernel at 3% of the solve or more; and the roofline object of the
    dominant one.  For the PCG also the fraction on the minimal bytes: each
    block of the reduced camera system read once with its entry, without the
    transposed products' round trip (80 B per off-diagonal block)."""
    rcs = kstats.pop("_rcs", None)
    total_ms = sum(v["ms"] for v in kstats.values()) or 1.0
    kernels = {}
    for k, v in sorted(kstats.items(), key=lambda kv: -kv[1]["ms"]):
        d = {"share": round(v["ms"] / total_ms, 4), "launches": v["launches"],
             "avg_ms": v["ms"] / max(v["launches"], 1)}
        if v.get("bytes", 0) > 0 and v["ms"] > 0 and d["share"] >= 0.03:
            ach = v["bytes"] / (v["ms"] * 1e-3) / 1e9
            d.update({"achieved_gbs": ach, "frac": ach / hbm, "algorithmic_bytes": v["bytes"] / v["launches"]})
        kernels[k] = d
    timed_k = {k: v for k, v in kstats.items() if v.get("bytes", 0) > 0}
    dom = max(timed_k, key=lambda k: timed_k[k]["ms"]) if timed_k else None
    if not dom:
        return None, kernels
    d = timed_k[dom]
    avg_s = d["ms"] * 1e-3 / d["launches"]
    alg = d["bytes"] / d["launches"]
    ach = alg / avg_s / 1e9
    ratio, src = traffic_ratio() if dom == "pcg" else (None, None)
    roofline = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": ach / hbm, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": alg * ratio if ratio else None,
                "traffic_note": (f"ncu DRAM bytes / algorithmic bytes = {ratio:.3f} from {src}, scaled to "
                                 "this launch's algorithmic bytes") if ratio else None,
                "algorithmic_bytes_per_launch": alg, "avg_launch_ms": d["ms"] / d["launches"]}
    if dom == "pcg" and rcs and rcs.get("fp32"):
        # the library's count per iteration (solver.cu): blocks with their
        # 16 B index, the transposed products' 64 B slots written and read,
        # the per-row vectors; minimal: each block once with an 8 B index
        nb, rows = rcs["offdiag_blocks"], rcs["rows"]
        per_row = rows * (648.0 + 22 * 72.0 + 2 * 720.0 + 2 * 72.0)
        full_it = 340.0 * (rows + nb) + 128.0 * nb + per_row
        min_it = 332.0 * (rows + nb) + per_row
        minimal = alg * min_it / full_it
        roofline["frac_minimal_bytes"] = minimal / avg_s / 1e9 / hbm
        roofline["minimal_bytes_note"] = ("each block read once with an 8 B index, no transposed-product round trip "
                                          "and no slot padding")
    return roofline, kernels


def config_dict(args, blk=None):
    d = {"workload": WORKLOADS[args.config], "scale": args.scale, "robust": True, "addflags": "k2 k4 f",
         "ours": f"learned two-level PCG, {args.precision}, relative tolerance {args.tol:g}",
         "plain": "FP64 block-Jacobi PCG, the reference's stop rule",
         "l2": "inputs larger than L2 (scene > 1 GB); 256 MB buffer written before every step",
         "parallelism": f"replicas x{args.gpus}"}
    if blk is not None:
        d.update({"n_images": blk.n_images, "n_points": blk.n_points, "n_obs": blk.n_obs})
    return d


def run_reference(args):
    """The reference's CPU path on the host cores: its default branch for
    this workload (Threads=0, the partitioned RPBA with min(cores,
    iround(images / 70)) partitions on OpenMP threads, restated by the
    oracle) on a bounded sample of the workload per step -- a scene of the
    same family at --ref-sample-scale of its size -- with the value scaled
    to the full workload by observation count.  The cost of the reference's
    solve grows faster than its observation count (more PCG iterations,
    larger partitions), so the scaled value is a lower bound of its
    full-workload time.  Beside it, once, the single-threaded global LSA
    (Threads=1, the algorithm the plain GPU form reproduces) on the
    --cpu-sample-scale sample, scaled the same way."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    import rpba_b200 as rb  # the options container only: no GPU library is loaded
    full = make_block(args.config, args.scale, args.seed_offset)  # the workload itself: its size and config
    cfg, n_full = config_dict(args, full), full.n_obs
    del full
    sblk = make_block(args.config, args.ref_sample_scale, args.seed_offset)
    threads = oracle.parallel_threads(sblk.n_images, os.cpu_count() or 1)
    times, par = [], None
    for i in range(args.warmup + args.steps):
        par = cpu_sample_parallel(sblk, None)
        if par is None:  # too small for the partitioned branch: the global LSA is the reference's path
            t0 = time.perf_counter()
            oracle.calc_plsa(sblk, rb.make_options(solver=rb.SOLVER_PCG))
            dt = time.perf_counter() - t0
        else:
            dt = par["value"]
        if i >= args.warmup:
            times.append(dt)
    t_sample = statistics.median(times)
    factor = n_full / sblk.n_obs
    v = t_sample * factor
    g_dt, g_rep, g_st, gblk, _ = cpu_sample(args.config, args.cpu_sample_scale)
    sample = (f"per step one complete solve of a scene of the same family at {args.ref_sample_scale:g} of the "
              f"workload ({sblk.n_images} cameras, {sblk.n_points} points, {sblk.n_obs} observations) by the "
              f"reference's Threads=0 branch on {threads if par else 1} host threads; value = median step time "
              f"x {factor:.1f} (full-workload observations / sample observations), a lower bound of the "
              f"full-workload time")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads if par else 1, "kind": "port",
                         "sample": sample, "sample_seconds": t_sample, "scale_factor": factor,
                         "step_times": times, "partitioned": par,
                         "global_lsa": {"value": g_dt * n_full / gblk.n_obs, "sample_seconds": g_dt, "cores": 1,
                                        "sample": (f"one complete solve at {args.cpu_sample_scale:g} of the "
                                                   f"workload ({gblk.n_images} cameras, {gblk.n_obs} "
                                                   "observations), one thread, scaled by observation count"),
                                        "linear_solves": g_rep["linear_solves"], "final_rms": g_rep["rms"],
                                        "status": g_st}},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "loaded_repo_libraries": repo_libraries(),
    }
    print(json.dumps(line), flush=True)
    return 0


def partitioned_over_ranks(args, g, local):
    """One scene over the ranks in the reference's own partitioned algorithm:
    the city family at --ranks-scale, every rank holding the whole scene,
    the partitions (the reference's count for the host's cores) dealt to the
    ranks and the partition steps' results all-gathered after every round
    (rpba_calc_plsa_parallel_ranks; one rank: rpba_calc_plsa_parallel).
    Wall time of the second of two runs, max over ranks; the same scene at
    every rank count (strong scaling).  Every rank takes the same
    collective steps whatever fails; a failure is reported, not raised."""
    import hashlib
    import math
    import torch
    import rpba_b200 as rb
    from rpba_b200.replicas import bytes_allgather
    sblk = make_block(3, args.ranks_scale, args.seed_offset)
    k = max(2, min(os.cpu_count() or 1, int(math.floor(sblk.n_images / 70 + 0.5))))
    err, dt, st, iters, h, part = None, float("nan"), None, None, None, None
    try:
        part = rb.partition_images(sblk, k)
    except Exception as e:
        err = f"{type(e).__name__}: {e}"
    gather = bytes_allgather(torch.device("cuda", local))
    for _ in range(2):
        g.barrier()
        if err is not None:
            continue
        try:
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if g.world == 1:
                st, b, stats, _ = rb.calc_plsa_parallel(sblk, part, k, device=local)
            else:
                st, b, stats, _ = rb.calc_plsa_parallel_ranks(sblk, part, k, g.rank, g.world, gather, device=local)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            iters = stats["iterations"]
            h = hashlib.sha1(b"".join(np.ascontiguousarray(getattr(b, n)).tobytes()
                                      for n in ("pmat", "K", "distpara", "XX", "pt_obs_off", "pt_obs_image",
                                                "pt_obs_slot"))).hexdigest()
        except Exception as e:
            err = f"{type(e).__name__}: {e}"
    infos = g.gather({"seconds": dt, "status": st, "hash": h, "error": err})
    return {"value": max(i["seconds"] for i in infos), "unit": UNIT, "scaling": "strong", "ranks": g.world,
            "partitions": k,
            "workload": (f"city family at {args.ranks_scale:g} scale ({sblk.n_images} cameras, {sblk.n_obs} "
                         "observations), the reference's partitioned branch, reference PCG in the steps"),
            "status": [i["status"] for i in infos], "outer_iterations": iters,
            "identical_on_all_ranks": len({i["hash"] for i in infos}) == 1,
            "errors": [i["error"] for i in infos if i["error"]]}


def repo_libraries():
    """Shared libraries of this repository mapped into the process (the
    reference arm must run the oracle's alone)."""
    try:
        with open("/proc/self/maps") as fh:
            paths = {ln.split()[-1] for ln in fh if ln.rstrip().endswith(".so")}
    except OSError:
        return None
    return sorted(os.path.relpath(p, ROOT) for p in paths if p.startswith(ROOT + os.sep))


def run_batch(args):
    """The batched workload (256 uneven arc scenes, 20-400 cameras) split
    scene-parallel over the ranks: every rank solves the scenes ``shard``
    deals it (by camera count) with rpba_solve_batch on its GPU, FP32
    assembly, and the per-scene results are gathered in scene order.  Value:
    scenes per second of the whole job (all scenes over the slowest rank's
    wall time, device synchronised on both sides); p50/p99 of the per-scene
    device times."""
    import torch
    import rpba_b200 as rb
    from rpba_b200 import scenes
    from rpba_b200.replicas import Group, scene_parallel
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    g = Group(rank, world, "nccl", 600.0, device=torch.device("cuda", local))
    specs = scenes.batch_scene_specs(n_scenes=args.batch_scenes)
    costs = [kw["n_cams"] for kw in specs]
    from rpba_b200.replicas import shard
    mine_all = [i for i, r in enumerate(shard(costs, world)) if r == rank]
    blocks = {i: scenes._arc_block(specs[i]) for i in mine_all}

    def solve(idx):
        bl = [blocks[i].copy() for i in idx]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st, reps, br = rb.solve_batch(bl, workers=0, precision=rb.PREC_MIXED, device=local)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        return [{"status": a, "solve_s": r["solve_seconds"], "rms": r["rms"]} for a, r in zip(st, reps)], dt

    for _ in range(args.warmup):
        scene_parallel(g, costs, solve)
    runs = [scene_parallel(g, costs, solve) for _ in range(args.steps)]
    job = statistics.median(r["job_seconds"] for r in runs)
    per = np.array([sc["solve_s"] for sc in runs[-1]["scenes"]])
    if rank == 0:
        line = {"metric": "scenes/s, batched uneven scenes", "value": len(specs) / job, "unit": "scenes/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": job * 1e3,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32/f64",
                "data": "synthetic",
                "config": {"workload": f"{len(specs)} arc scenes, 20-400 cameras, 150 points per camera",
                           "parallelism": f"scene-parallel x{world}"},
                "p50_scene_s": float(np.percentile(per, 50)), "p99_scene_s": float(np.percentile(per, 99)),
                "failed": int(sum(sc["status"] != 0 for sc in runs[-1]["scenes"]))}
        print(json.dumps(line), flush=True)
    g.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.config == 4:
        return run_batch(args)
    import torch
    import rpba_b200 as rb

    from rpba_b200.replicas import Group, time_steps

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    g = Group(rank, world, "nccl", 600.0, device=torch.device("cuda", local))
    barrier, max_over_ranks = g.barrier, g.max

    blk = make_block(args.config, args.scale, args.seed_offset)
    w = learned_weights()
    prec = rb.PREC_MIXED if args.precision == "mixed" else rb.PREC_FP64
    ours_kw = dict(solver=rb.SOLVER_LEARNED, precision=prec, pcg_tolerance=args.tol, device=local)
    plain_kw = dict(solver=rb.SOLVER_PCG, precision=rb.PREC_FP64, device=local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        uuid = None

    def timed(kw, weights, steps, warmup):
        S = rb.Solver(blk, **kw)
        if weights is not None:
            S.set_preconditioner(weights)
        reps = []

        def step():
            torch.cuda.synchronize()
            st, rep = S.solve()
            torch.cuda.synchronize()
            reps.append(rep)
            return rep["solve_seconds"]

        res = time_steps(g, step, steps, warmup, before_step=flush.zero_)
        S.close()
        return res, reps[warmup:]

    clk = Clocks(uuid)
    res, reps = timed(ours_kw, w, args.steps, args.warmup)
    clocks = clk.stop()
    times, value = res["times"], res["max_over_ranks"]
    plain = None
    if not args.no_plain:
        p_res, p_reps = timed(plain_kw, None, args.steps, args.warmup)
        p_times, pv = p_res["times"], p_res["max_over_ranks"]
        rms_o, rms_p = reps[-1]["rms"], p_reps[-1]["rms"]
        plain = {"value": pv, "unit": UNIT, "final_rms": rms_p, "pcg_iterations": p_reps[-1]["pcg_iterations"],
                 "linear_solves": p_reps[-1]["linear_solves"], "step_times": p_times,
                 "speedup": pv / value, "rms_rel_diff": (rms_o - rms_p) / rms_p,
                 "matched": bool(rms_o <= rms_p * (1 + RMS_MATCH))}

    # end to end through the C ABI with host buffers: rpba_create (scene
    # H2D), the weights, rpba_solve, rpba_get_state (D2H), rpba_destroy
    # (inputs and the caller's output arrays in page-locked memory, both
    # allocated before the timed steps)
    try:
        eblk, e2e_mem = pinned_copy(blk), "pinned"
        eout = pinned_out(blk)
    except Exception as e:  # page-locking refused: the caller's pageable arrays
        eblk, e2e_mem, eout = blk, f"pageable ({type(e).__name__})", None
    e2e_times = []
    for _ in range(max(1, args.e2e_steps)):
        flush.zero_()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S = rb.Solver(eblk, **ours_kw)
        S.set_preconditioner(w)
        S.solve()
        S.state(out=eout)
        S.close()
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
    e2e = max_over_ranks(statistics.median(e2e_times))

    # per-kernel device times of one more solve (CUDA events around
    # launches), after a warm-up solve on the same handle like the timed ones
    P = rb.Solver(blk, verbose=2, **ours_kw)
    P.set_preconditioner(w)
    P.solve()
    P.solve()
    kstats = P.kernel_stats()
    P.close()
    hbm, peak_kind = peaks()
    roofline, kernels = rooflines(kstats, hbm, peak_kind)
    kernel_share = {k: v["share"] for k, v in kernels.items()}

    # what each part of the preconditioner buys: the same learned solver
    # without the network (block-Jacobi part plus the coarse space), and
    # without the coarse space (network only), one solve each, same tolerance
    ablation = None
    if not args.no_ablation:
        ablation = {}
        for name, kw, wt in (("no_network", ours_kw, None),
                             ("no_coarse_space", dict(ours_kw, coarse_aggregates=-1), w)):
            S = rb.Solver(blk, **kw)
            S.set_preconditioner(wt)
            S.solve()  # warm-up, as the timed steps have
            flush.zero_()
            torch.cuda.synchronize()
            _, ra = S.solve()
            S.close()
            ablation[name] = {"value": ra["solve_seconds"], "unit": UNIT, "pcg_iterations": ra["pcg_iterations"],
                              "linear_solves": ra["linear_solves"], "pcg_fallbacks": ra["pcg_fallbacks"],
                              "final_rms": ra["rms"]}
        ablation["with_both"] = {"value": value, "pcg_iterations": reps[-1]["pcg_iterations"],
                                 "final_rms": reps[-1]["rms"]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        dt, rep_c, st_c, sblk, sout = cpu_sample(args.config, args.cpu_sample_scale)
        same = {}
        for name, kw, wt in (("ours", ours_kw, w), ("plain_fp64", plain_kw, None)):
            S = rb.Solver(sblk, **kw)
            S.set_preconditioner(wt)
            S.solve()
            _, rep_g = S.solve()
            S.close()
            same[name] = rep_g["solve_seconds"]
        # end to end through the C ABI from host buffers, as the e2e value
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S = rb.Solver(sblk, **ours_kw)
        S.set_preconditioner(w)
        S.solve()
        S.state()
        S.close()
        torch.cuda.synchronize()
        same["ours_e2e"] = time.perf_counter() - t0
        par = cpu_sample_parallel(sblk, sout)
        if par is not None:
            # the same branch on the GPU (rpba_calc_plsa_parallel: the partition
            # steps on host threads, their solves and the merge on the device),
            # same partition count, partition included; the first run warms up
            import oracle
            k = par["partitions"]
            try:
                for _ in range(2):
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    part_g = rb.partition_images(sblk, k)
                    st_p, b_p, s_p, _ = rb.calc_plsa_parallel(sblk, part_g, k)
                    torch.cuda.synchronize()
                    dt_p = time.perf_counter() - t0
                par.update({"gpu_same_sample_s": dt_p, "gpu_status": st_p,
                            "gpu_outer_iterations": s_p["iterations"],
                            "gpu_exteval_sigma0": oracle.exteval(b_p)[1]["exteval_sigma0"]})
            except Exception as e:  # a side measurement: reported, never fatal to the bench line
                par["gpu_error"] = f"{type(e).__name__}: {e}"
        cpu = {"value": dt, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": (f"one complete solve of the same scene family at {args.cpu_sample_scale:g} of the "
                          f"workload ({sblk.n_images} cameras, {sblk.n_obs} observations) on one host core"),
               "linear_solves": rep_c["linear_solves"], "final_rms": rep_c["rms"],
               "gpu_same_sample_s": same["ours"], "gpu_plain_fp64_same_sample_s": same["plain_fp64"],
               "gpu_e2e_same_sample_s": same["ours_e2e"], "parallel": par}

    ranks = None if args.no_ranks else partitioned_over_ranks(args, g, local)

    if rank == 0:
        r0 = reps[-1]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64" if prec else "f64", "data": "synthetic",
            "config": config_dict(args, blk),
            "plain": plain,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": block_bytes(blk),
                    "d2h_bytes_per_step": state_bytes(blk), "host_input_memory": e2e_mem,
                    "host_output_memory": e2e_mem},
            "gpu_launches": int(r0["kernel_launches"]),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "solve": {"linear_solves": r0["linear_solves"], "pcg_iterations": r0["pcg_iterations"],
                      "pcg_fallbacks": r0["pcg_fallbacks"], "final_rms": r0["rms"], "final_cost": r0["cost"],
                      "obs_deleted": r0["obs_deleted"], "step_times": times},
            "kernel_share": kernel_share,
            "kernels": kernels,
            "ablation": ablation,
            "one_scene_over_ranks": ranks,
        }
        print(json.dumps(line), flush=True)
    g.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
