"""The oracle's error returns against the reference's (Adjust returns with
its last stored state after writing a 'BA-Error' line, and only when the
block has more than three images, rbacore.cpp:415-424, 470-476; a NaN or an
infinity in the step ends it before the cameras are decoded, 541-548).
No GPU needed."""
import numpy as np
import pytest

from rpba_b200 import scenes


def _drop_image_obs(blk, image):
    """Copy of blk where every observation of `image` is the only
    observation of a new point (its original points keep the others)."""
    import rpba_b200 as rb
    img = blk.pt_obs_image
    keep = img != image
    off = blk.pt_obs_off
    counts = np.add.reduceat(keep.astype(np.int64), off[:-1])
    extra = np.nonzero(~keep)[0]
    XX = np.concatenate([blk.XX, blk.XX[np.searchsorted(off, extra, side="right") - 1]])
    new_off = np.concatenate([[0], np.cumsum(counts)])
    return rb.Block(blk.pmat, blk.K, blk.distpara, XX.astype(np.float32), blk.img_obs_off, blk.xg, blk.wx, blk.wy,
                    blk.wxy, np.concatenate([new_off, new_off[-1] + np.arange(1, extra.size + 1)]).astype(np.int32),
                    np.concatenate([img[keep], img[extra]]).astype(np.int32),
                    np.concatenate([blk.pt_obs_slot[keep], blk.pt_obs_slot[extra]]).astype(np.int32))


@pytest.mark.parametrize("n_cams,line", [(8, True), (3, False)])
def test_no_observations_in_image(oracle_mod, n_cams, line):
    import rpba_b200 as rb
    blk = scenes.to_block(scenes.arc_scene(seed=3, n_cams=n_cams, n_pts=300))
    b = _drop_image_obs(blk, n_cams - 1)
    st, out, rep, log = oracle_mod.calc_plsa(b, rb.make_options())
    assert st == 3
    assert ("BA-Error: No observations in image %d (image index)" % (n_cams - 1) in log) == line
    # no stored state yet: the cameras and points are the input's, but for
    # camera 0, which the constructor rectified (PrepareIteration)
    assert np.array_equal(out.pmat[1:], b.pmat[1:]) and np.array_equal(out.XX, b.XX)
    assert np.abs(out.pmat[0] - b.pmat[0]).max() < 1e-6


@pytest.mark.parametrize("n_cams,line", [(6, True), (3, False)])
def test_low_redundancy(oracle_mod, n_cams, line):
    """Every point seen twice: 4 equations per point against 3 unknowns plus
    the cameras' -- too few points leave the redundancy negative."""
    import rpba_b200 as rb
    bal = scenes.arc_scene(seed=4, n_cams=n_cams, n_pts=400, outlier_frac=0.0)
    blk = scenes.to_block(bal)
    # keep 2 observations of the first few points only
    n_keep = 4 * n_cams
    off = blk.pt_obs_off
    sel = np.concatenate([np.arange(off[p], off[p] + 2) for p in range(n_keep)])
    b = blk.copy()
    b.XX = blk.XX[:n_keep].copy()
    b.pt_obs_off = (np.arange(n_keep + 1) * 2).astype(np.int32)
    b.pt_obs_image = blk.pt_obs_image[sel].copy()
    b.pt_obs_slot = blk.pt_obs_slot[sel].copy()
    assert all(len(set(b.pt_obs_image[b.pt_obs_off[i]:b.pt_obs_off[i + 1]])) == 2 for i in range(n_keep))
    covered = set(b.pt_obs_image.tolist())
    if len(covered) < n_cams:
        pytest.skip("the reduced scene leaves an image without observations")
    st, out, rep, log = oracle_mod.calc_plsa(b, rb.make_options())
    assert st == 4
    assert ("BA-Error: Low redundancy" in log) == line


def test_nan_camera_ends_with_nan_step(oracle_mod):
    """A NaN in one camera makes its residuals NaN (counted as zero, with the
    reweighting statistic 1e20) and the step NaN: the adjustment ends with
    the NaN-step status and the input state."""
    import rpba_b200 as rb
    blk = scenes.to_block(scenes.arc_scene(seed=6, n_cams=8, n_pts=400))
    b = blk.copy()
    b.pmat[3, 5] = np.nan
    st, out, rep, log = oracle_mod.calc_plsa(b, rb.make_options())
    assert st == 5
    assert np.array_equal(out.XX, b.XX)


def test_degenerate_block_is_an_argument_error(oracle_mod):
    import rpba_b200 as rb
    blk = scenes.to_block(scenes.arc_scene(seed=6, n_cams=8, n_pts=400))
    one = rb.Block(blk.pmat[:1], blk.K[:1], blk.distpara[:1], blk.XX[:0], blk.img_obs_off[:2], blk.xg[:blk.img_obs_off[1]],
                   blk.wx[:blk.img_obs_off[1]], blk.wy[:blk.img_obs_off[1]], blk.wxy[:blk.img_obs_off[1]],
                   np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32))
    st, _, _, _ = oracle_mod.calc_plsa(one, rb.make_options())
    assert st == 1
