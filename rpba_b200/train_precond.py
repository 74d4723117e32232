"""Train the learned block-Jacobi correction and write its weights.

    python -m rpba_b200.train_precond [--out rpba_b200/precond_weights.npy]

The training systems are the ones the plain FP64 direct solver's own LM
iterations assemble on seeded street-like and aerial-grid scenes (the styles
of the 1,000-camera street and 3,000-camera aerial workloads, at a few
hundred cameras each), recorded and trained entirely on the GPU by the
library's kernels (rpba_train_preconditioner).  The weights file is what
``Solver.set_preconditioner`` and the benchmark load.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "precond_weights.npy")


def training_scenes():
    from . import scenes
    blocks = [scenes.to_block(scenes.street_scene(seed=100 + i, n_cams=300, n_pts=57000)) for i in range(3)]
    blocks += [scenes.to_block(scenes.aerial_scene(seed=200 + i, nx=20, ny=15, n_pts=30000)) for i in range(2)]
    return blocks


def train(steps=1000, lr=1e-3, probes=4, seed=1):
    from . import lib
    t = time.time()
    blocks = training_scenes()
    t_gen = time.time() - t
    t = time.time()
    w, rep = lib.train_preconditioner(blocks, steps=steps, lr=lr, probes=probes, seed=seed)
    rep.update({"seconds": round(time.time() - t, 2), "scene_seconds": round(t_gen, 2), "lr": lr})
    return w, rep


def load(path: str = DEFAULT_OUT):
    """The committed weights (float32[1865]), or None when absent."""
    if not os.path.exists(path):
        return None
    w = np.load(path)
    return np.ascontiguousarray(w, np.float32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--probes", type=int, default=4)
    a = ap.parse_args()
    w, rep = train(a.steps, a.lr, a.probes)
    np.save(a.out, w.astype(np.float32))
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
