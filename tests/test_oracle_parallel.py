"""The oracle's restatement of the parallel RPBA's pieces (rpbacore.cpp:
100-510): the LSA's GCP mode (every camera free, shared points held by
3-D priors, one damped step per call).  No reference build exists here,
so the checks are behavioural: with every point a stiff GCP at the global
solution, GCP steps bring perturbed cameras back to that solution, and a
step taken at the solution barely moves them (no GPU needed)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def solved(oracle_mod):
    import rpba_b200 as rb
    from rpba_b200 import scenes
    blk = scenes.to_block(scenes.arc_scene(seed=31, n_cams=12, n_pts=1500, outlier_frac=0.0))
    st, out, rep, log = oracle_mod.calc_plsa(blk, rb.make_options(robust=False))
    assert st == 0
    return out


def _centres(blk):
    P = blk.pmat.astype(np.float64).reshape(-1, 3, 4)
    return np.stack([-p[:, :3].T @ p[:, 3] for p in P])


def _gcp_inputs(blk, w=1e4):
    n = blk.n_points
    gcpinfo = np.arange(n, dtype=np.int32)
    W3 = np.tile(np.array([w, w, w, 0, 0, 0], np.float32), (n, 1))
    return gcpinfo, W3, blk.XX.astype(np.float64).copy()


def test_gcp_steps_restore_cameras(oracle_mod, solved):
    import rpba_b200 as rb
    ref = _centres(solved)
    gi, W3, gd = _gcp_inputs(solved)
    # point 0 has GCP index 0: with a single observation the reference
    # would drop it, with two or more it is kept like the others
    blk = solved.copy()
    rng = np.random.default_rng(3)
    P = blk.pmat.reshape(-1, 3, 4)
    P[:, :, 3] += rng.normal(0, 0.05, (blk.n_images, 3)).astype(np.float32)
    err0 = np.abs(_centres(blk) - ref).max()
    for _ in range(4):
        st, log = oracle_mod.lsa_gcp_step(blk, gi, W3, gd, blk.n_images, rb.make_options(robust=False))
        assert st == 0, log
        assert "Sigma0AO:" in log
    err = np.abs(_centres(blk) - ref).max()
    print(f"camera centre error: {err0:.3e} -> {err:.3e}")
    assert err < 0.02 * err0


def test_gcp_step_at_solution_is_small(oracle_mod, solved):
    import rpba_b200 as rb
    ref = _centres(solved)
    gi, W3, gd = _gcp_inputs(solved)
    blk = solved.copy()
    st, log = oracle_mod.lsa_gcp_step(blk, gi, W3, gd, blk.n_images, rb.make_options(robust=False))
    assert st == 0, log
    scale = np.abs(ref).max()
    assert np.abs(_centres(blk) - ref).max() < 1e-4 * scale
