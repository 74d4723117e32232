"""The GPU per-point refinement (rpba_triangulate, CalcLSAXMulti of
rpbacore.cpp:536-773) against the oracle's restatement on the same seeded
inputs: the kernel keeps the restatement's operation order and rounding, so
points, flags and statistics are compared bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    from rpba_b200 import scenes
    return scenes.to_block(scenes.city_scene(seed=41, n_clusters=3, cams_per_cluster=40, n_pts=30000))


def _thresholds(blk, sig0v):
    w = np.zeros(blk.n_images, np.float32)
    for i in range(blk.n_images):
        v = np.sort(sig0v[blk.pt_obs_image == i])
        w[i] = np.float32(1.0) / (v[len(v) // 2] * np.float32(2.1981)) if len(v) else np.float32(0)
    return w


@pytest.mark.parametrize("mode,weight_only", [(0, False), (1, False), (2, False), (2, True), (0, True)])
def test_triangulation_matches_oracle(oracle_mod, scene, mode, weight_only):
    import rpba_b200 as rb
    sig0w = None
    if mode == 2:
        sig0w = _thresholds(scene, oracle_mod.triangulate(scene, robustmode=1)["sig0v"])
    g = rb.triangulate(scene, sig0w, mode, weight_only)
    o = oracle_mod.triangulate(scene, sig0w, mode, weight_only)
    assert np.array_equal(g["conv"], o["conv"])
    assert np.array_equal(g["keep"], o["keep"])
    assert np.array_equal(g["XX"], o["XX"])
    assert np.array_equal(g["sig0v"], o["sig0v"])
    assert g["redundancy"] == o["redundancy"]
    assert g["sig0io"] == o["sig0io"]
    if mode == 2 and not weight_only:
        assert (g["keep"] == 0).any()
