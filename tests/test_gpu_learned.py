"""Learned preconditioner: the GPU training kernels' loss and gradient
against an autograd reference on the CPU, and the trained network's effect
on PCG iterations."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_learned_gradient_matches_autograd():
    import rpba_b200 as rb
    from oracle import learned_ref as lr
    rng = np.random.default_rng(0)
    for trial in range(3):
        ts = lr.random_set(rng, systems=2 + trial, rows_per=10 + 3 * trial, probes=1 + trial)
        w = (rng.normal(size=rb.PRECOND_WEIGHTS) * 0.2).astype(np.float32)
        L_ref, g_ref = lr.loss(ts, w)
        L_gpu, g_gpu = rb.precond_loss_grad(ts, w)
        assert abs(L_gpu - L_ref) <= 1e-4 * max(1.0, abs(L_ref)), (L_gpu, L_ref)
        scale = np.abs(g_ref).max()
        assert np.abs(g_gpu - g_ref).max() <= 2e-3 * scale, (np.abs(g_gpu - g_ref).max(), scale)
