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


@pytest.mark.parametrize("mode,weight_only,k", [(0, False, 3), (2, False, 4), (0, True, 3), (0, False, 1)])
def test_weight_blocks_match_oracle(oracle_mod, scene, mode, weight_only, k):
    """The per-partition weight blocks (rpba_triangulate_parts) against the
    oracle's, bit for bit, with the partition of rpba_partition_images; the
    other outputs equal rpba_triangulate's."""
    import rpba_b200 as rb
    part = rb.partition_images(scene, k)
    sig0w = None
    if mode == 2:
        sig0w = _thresholds(scene, oracle_mod.triangulate(scene, robustmode=1)["sig0v"])
    g = rb.triangulate_parts(scene, part, k, sig0w, mode, weight_only)
    o = oracle_mod.triangulate_parts(scene, part, k, sig0w, mode, weight_only)
    assert np.array_equal(g["w3d"], o["w3d"])
    assert (g["w3d"] != 0).any()
    plain = rb.triangulate(scene, sig0w, mode, weight_only)
    for name in ("XX", "keep", "sig0v", "conv"):
        assert np.array_equal(g[name], plain[name]), name
    assert g["redundancy"] == plain["redundancy"] and g["sig0io"] == plain["sig0io"]
