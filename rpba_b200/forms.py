"""One generated workload solved by each form of the library.

    python -m rpba_b200.forms [--config 2] [--scale 1.0] [--forms plain,direct,learned]
                              [--tol 3e-5] [--repeats 3]

Forms (the solver and precision options of rpba_create):
  plain          FP64, the reference's block-Jacobi PCG and its stop rule
  direct         FP64, the envelope Cholesky of the reduced camera system
  mixed_direct   FP32 assembly, the same direct solve
  learned        FP32 assembly, the learned two-level PCG at relative
                 tolerance --tol (weights from rpba_b200/precond_weights.npy)
  partitioned    the reference's partitioned branch (Threads=0): the
                 reference's partition count for this host's cores,
                 min(cores, iround(images / 70)), the partition included,
                 FP64 with the reference's PCG in the partition steps

Each solver form: one warm-up solve on its handle, then --repeats solves
from the same start state; prints one JSON line per form with the median
device time of the whole robust LM run (CUDA events inside the library),
the linear solve and PCG iteration counts, the final RMS reprojection error
and cost, and the status.  The partitioned form (host control around device
steps) reports the wall time of the last of 1 + --repeats runs, its outer
iterations and best sigma0.  A form the workload does not admit (the direct forms past
the envelope's size) reports its status instead of a time.
"""
from __future__ import annotations

import argparse
import json
import statistics
import time

FORMS = ("plain", "direct", "mixed_direct", "learned", "partitioned")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=2, choices=[0, 1, 2, 3])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--seed-offset", type=int, default=0)
    ap.add_argument("--forms", default=",".join(FORMS))
    ap.add_argument("--tol", type=float, default=3e-5, help="relative PCG tolerance of the learned form")
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    forms = [f for f in a.forms.split(",") if f]
    for f in forms:
        if f not in FORMS:
            ap.error(f"unknown form {f!r} (one of {', '.join(FORMS)})")
    from . import lib, scenes, train_precond
    from .block import PREC_FP64, PREC_MIXED, SOLVER_DIRECT, SOLVER_LEARNED, SOLVER_PCG
    kws = {
        "plain": dict(solver=SOLVER_PCG, precision=PREC_FP64),
        "direct": dict(solver=SOLVER_DIRECT, precision=PREC_FP64),
        "mixed_direct": dict(solver=SOLVER_DIRECT, precision=PREC_MIXED),
        "learned": dict(solver=SOLVER_LEARNED, precision=PREC_MIXED, pcg_tolerance=a.tol),
    }
    t0 = time.time()
    blk = scenes.to_block(scenes.make_scene(a.config, scale=a.scale, seed=20260 + a.config + a.seed_offset))
    gen = time.time() - t0
    weights = train_precond.load() if "learned" in forms else None
    if "learned" in forms and weights is None:
        raise SystemExit("rpba_b200/precond_weights.npy is missing: python -m rpba_b200.train_precond")
    for f in forms:
        if f == "partitioned":
            print(json.dumps(partitioned(lib, blk, a, gen)), flush=True)
            continue
        S = lib.Solver(blk, device=a.device, **kws[f])
        if f == "learned":
            S.set_preconditioner(weights)
        line = {"config": a.config, "scale": a.scale, "n_images": blk.n_images, "n_obs": blk.n_obs,
                "scene_generation_s": round(gen, 1), "form": f}
        if f == "learned":
            line["tolerance"] = a.tol
        st, rep = S.solve()
        times = []
        if st == 0:
            for _ in range(max(1, a.repeats)):
                st, rep = S.solve()
                times.append(rep["solve_seconds"])
        S.close()
        line.update({"status": st, "status_text": lib.load().rpba_status_string(st).decode()})
        if times:
            line.update({"seconds": statistics.median(times), "step_times": times,
                         "linear_solves": rep["linear_solves"], "pcg_iterations": rep["pcg_iterations"],
                         "pcg_fallbacks": rep["pcg_fallbacks"], "final_rms": rep["rms"], "final_cost": rep["cost"],
                         "obs_deleted": rep["obs_deleted"]})
        print(json.dumps(line), flush=True)


def partitioned(lib, blk, a, gen) -> dict:
    """The reference's Threads=0 branch on the GPU, wall time."""
    import math
    import os
    k = min(os.cpu_count() or 1, int(math.floor(blk.n_images / 70 + 0.5)))
    line = {"config": a.config, "scale": a.scale, "n_images": blk.n_images, "n_obs": blk.n_obs,
            "scene_generation_s": round(gen, 1), "form": "partitioned", "partitions": k}
    if k < 2:
        line.update({"status": None, "note": "one partition: the reference takes the global LSA"})
        return line
    times = []
    for _ in range(1 + max(1, a.repeats)):
        t0 = time.perf_counter()
        part = lib.partition_images(blk, k)
        st, _, stats, _ = lib.calc_plsa_parallel(blk, part, k, device=a.device)
        times.append(time.perf_counter() - t0)
    line.update({"status": st, "status_text": lib.load().rpba_status_string(st).decode(), "seconds": times[-1],
                 "step_times": times[1:], "outer_iterations": stats["iterations"], "sig0opt": stats["sig0opt"]})
    return line


if __name__ == "__main__":
    main()
