"""Batched workload: 256 independent arc scenes of uneven size (20-400
cameras, 150 points per camera, track length geometric mean 4), robust, FP32
assembly with FP64 accept/reject.

    python -m rpba_b200.batch_bench [--scenes 256] [--workers 0]

Note: with 150 points per camera and track length 4, the 256 scenes hold
about 34M observations, not 1.5M; the generator follows the per-scene
parameters.

Prints one JSON line: scenes/s and the per-scene time to converge (p50/p99,
device time of each scene's LM run) for one scene at a time ("one launch
sequence per scene") and for the batch (several scenes at once on their own
streams, worker count chosen by the library's autotuner unless given), and
whether the two give bitwise identical results.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=256)
    ap.add_argument("--workers", type=int, default=0)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    a = ap.parse_args()
    from . import lib, scenes
    prec = 1 if a.precision == "mixed" else 0
    t = time.time()
    blocks = scenes.batch_blocks(n_scenes=a.scenes)
    gen = time.time() - t
    n_obs = int(sum(b.n_obs for b in blocks))
    one = [b.copy() for b in blocks]
    st1, rep1, br1 = lib.solve_batch(one, workers=1, precision=prec)
    many = [b.copy() for b in blocks]
    st2, rep2, br2 = lib.solve_batch(many, workers=a.workers, precision=prec)
    same = all(np.array_equal(x.pmat, y.pmat) and np.array_equal(x.XX, y.XX) for x, y in zip(one, many))

    def pct(reps):
        t = np.array([r["solve_seconds"] for r in reps])
        return {"p50_s": float(np.percentile(t, 50)), "p99_s": float(np.percentile(t, 99))}

    line = {
        "workload": f"{a.scenes} arc scenes, 20-400 cameras, 150 points per camera, {n_obs} observations",
        "precision": a.precision, "scene_generation_s": round(gen, 1),
        "one_at_a_time": {"scenes_per_s": br1["scenes_per_second"], "wall_s": br1["seconds"], **pct(rep1),
                          "failed": br1["failed"]},
        "batched": {"scenes_per_s": br2["scenes_per_second"], "wall_s": br2["seconds"], **pct(rep2),
                    "workers": br2["workers"], "tune_s": br2["tune_seconds"], "failed": br2["failed"]},
        "speedup": br2["scenes_per_second"] / br1["scenes_per_second"],
        "identical_results": bool(same),
        "statuses_equal": st1 == st2,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
