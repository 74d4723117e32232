#!/usr/bin/env python
"""Time to converge of the robust bundle adjuster on B200.

One step = one complete robust bundle adjustment (the reference's own stop
rule: two passes, reweighting, RobustDelete) of a seeded synthetic scene
that is already resident in HBM.  The default workload is the street scene
(1,000 cameras, 189k points, 943k observations; the drop-in configuration)
solved by the plain FP64 form with the reference's block-Jacobi PCG.

  python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank solves its own scene
(independent replicas, no collective on the data path); the value is the
slowest rank's time.  ``--impl reference`` times the reference algorithm's
CPU implementation (the C++ restatement under oracle/, single-threaded like
the reference's global LSA) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s to converge at matched final RMS reproj error: learned-PCG vs plain, 1 B200"
UNIT = "s"
WORKLOADS = {
    0: "arc: 50 cameras, 8k points, ~32k observations",
    1: "street: 1000 cameras, 190k points, ~950k observations",
    2: "aerial: 3000 cameras, 310k points, ~1.65M observations",
    3: "city: 13700 cameras, 4.5M points, ~29M observations",
}
SOLVERS = {"pcg": 0, "direct": 1, "learned": 2}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--solver", default="pcg", choices=list(SOLVERS))
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=2)
    return ap.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


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


def make_block(config, scale, rank):
    from rpba_b200 import scenes
    seed = 20260 + config + 1000 * rank
    return scenes.to_block(scenes.make_scene(config, scale=scale, seed=seed))


def cpu_baseline(blk, opts_kw, max_seconds=60.0):
    """The oracle (C++ restatement of the reference's global LSA) on the host:
    one complete solve of the same scene, one thread."""
    import oracle
    import rpba_b200 as rb
    o = rb.make_options(**opts_kw)
    t0 = time.perf_counter()
    st, _, rep, _ = oracle.calc_plsa(blk, o)
    dt = time.perf_counter() - t0
    return dt, rep, st


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    blk = make_block(args.config, args.scale, 0)
    kw = dict(solver=SOLVERS["direct" if args.solver == "direct" else "pcg"])
    for _ in range(args.warmup):
        cpu_baseline(blk, kw)
    times = []
    for _ in range(args.steps):
        dt, rep, st = cpu_baseline(blk, kw)
        times.append(dt)
    v = statistics.mean(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.config], "scale": args.scale, "solver": args.solver,
                   "robust": True, "addflags": "k2 k4 f"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": "complete solves of the scene (reference stop rule)",
                         "linear_solves": rep["linear_solves"], "status": st},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist
    import rpba_b200 as rb

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    blk = make_block(args.config, args.scale, rank)
    solver_kw = dict(solver=SOLVERS[args.solver], precision=1 if args.precision == "mixed" else 0, device=local)
    S = rb.Solver(blk, **solver_kw)
    for _ in range(args.warmup):
        S.solve()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        uuid = None
    clk = Clocks(uuid)
    times, reps = [], []
    for _ in range(args.steps):
        flush.zero_()
        barrier()
        torch.cuda.synchronize()
        st, rep = S.solve()
        torch.cuda.synchronize()
        times.append(rep["solve_seconds"])
        reps.append(rep)
    barrier()
    clocks = clk.stop()
    t_mean = statistics.mean(times)
    t = torch.tensor([t_mean], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    value = float(t.item())

    # end to end through the C ABI with host buffers: create (H2D), solve,
    # get_state (D2H), destroy -- the reference-facing CalcPLSA call
    e2e_times = []
    for _ in range(max(1, args.e2e_steps)):
        b = blk.copy()
        flush.zero_()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st_e, _, rep_e = rb.CalcPLSA(b, solver=solver_kw["solver"], precision=solver_kw["precision"], device=local)
        torch.cuda.synchronize()
        e2e_times.append(time.perf_counter() - t0)
    te = torch.tensor([statistics.mean(e2e_times)], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)

    # per-kernel device times of one more solve (CUDA events around launches)
    P = rb.Solver(blk, verbose=2, **solver_kw)
    P.solve()
    kstats = P.kernel_stats()
    P.close()
    hbm, peak_kind = peaks()
    timed = {k: v for k, v in kstats.items() if v.get("bytes", 0) > 0}
    dom = max(timed, key=lambda k: timed[k]["ms"]) if timed else None
    roofline = None
    if dom:
        d = timed[dom]
        avg_s = d["ms"] * 1e-3 / d["launches"]
        ach = d["bytes"] / d["launches"] / avg_s / 1e9
        roofline = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                    "frac": ach / hbm, "peak_kind": peak_kind, "traffic": None,
                    "algorithmic_bytes_per_launch": d["bytes"] / d["launches"],
                    "avg_launch_ms": d["ms"] / d["launches"]}
    total_ms = sum(v["ms"] for v in kstats.values())
    kernel_share = {k: round(v["ms"] / total_ms, 4) for k, v in sorted(kstats.items(), key=lambda kv: -kv[1]["ms"])}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        dt, rep_c, st_c = cpu_baseline(blk, dict(solver=solver_kw["solver"]))
        cpu = {"value": dt, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": "one complete solve of the same scene on one host core",
               "linear_solves": rep_c["linear_solves"], "final_rms": rep_c["rms"]}

    if rank == 0:
        r0 = reps[-1]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.config], "scale": args.scale, "solver": args.solver,
                       "precision": args.precision, "robust": True, "addflags": "k2 k4 f",
                       "l2": "flushed before every step (256 MB write)", "parallelism": f"replicas x{world}",
                       "n_images": blk.n_images, "n_points": blk.n_points, "n_obs": blk.n_obs},
            "e2e": {"value": float(te.item()), "unit": UNIT, "h2d_bytes_per_step": block_bytes(blk),
                    "d2h_bytes_per_step": state_bytes(blk)},
            "gpu_launches": int(r0["kernel_launches"]),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "solve": {"linear_solves": r0["linear_solves"], "pcg_iterations": r0["pcg_iterations"],
                      "final_rms": r0["rms"], "final_cost": r0["cost"], "obs_deleted": r0["obs_deleted"],
                      "step_times": times},
            "kernel_share": kernel_share,
        }
        print(json.dumps(line), flush=True)
    S.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
