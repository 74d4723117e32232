"""The oracle's restatement of the per-point refinement (CalcLSAXMulti,
rpbacore.cpp:536-773) behaves as the algorithm should on a seeded scene:
refined points lower their weighted residuals, most points converge, and
the robust mode removes observations (no GPU needed)."""
import numpy as np


def _rms(oracle_mod, blk):
    import rpba_b200 as rb
    _, rep = oracle_mod.exteval(blk, rb.make_options(exteval=True))
    return rep["exteval_sigma0"]


def test_oracle_triangulation_refines_points(oracle_mod):
    from rpba_b200 import scenes
    blk = scenes.to_block(scenes.arc_scene(seed=21, n_cams=20, n_pts=1500, outlier_frac=0.0))
    r = oracle_mod.triangulate(blk, robustmode=0)
    assert r["conv"].mean() > 0.9
    after = blk.copy()
    after.XX = r["XX"].astype(np.float32)
    assert _rms(oracle_mod, after) < _rms(oracle_mod, blk)
    assert r["redundancy"] > 0 and r["sig0io"] > 0


def test_oracle_triangulation_robust_drops_outliers(oracle_mod):
    from rpba_b200 import scenes
    blk = scenes.to_block(scenes.arc_scene(seed=22, n_cams=20, n_pts=1500, outlier_frac=0.05))
    r1 = oracle_mod.triangulate(blk, robustmode=1)
    img = blk.pt_obs_image
    sig0w = np.zeros(blk.n_images, np.float32)
    for i in range(blk.n_images):
        v = np.sort(r1["sig0v"][img == i])
        sig0w[i] = np.float32(1.0) / (v[len(v) // 2] * np.float32(2.1981))
    r2 = oracle_mod.triangulate(blk, sig0w, robustmode=2)
    dropped = (r2["keep"] == 0).mean()
    assert 0.01 < dropped < 0.2
