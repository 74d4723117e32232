"""Batched form: many independent scenes of uneven size solved together on
one GPU give, scene by scene, exactly what solving each scene alone gives
(every kernel sums in a fixed order, so concurrency changes no bit)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch():
    from rpba_b200 import scenes
    return [scenes.to_block(b) for b in scenes.batch_scenes(seed=77, n_scenes=10, cmin=8, cmax=60)]


@pytest.mark.parametrize("workers,precision", [(4, 0), (0, 1)])
def test_batch_equals_individual_solves(batch, workers, precision):
    import rpba_b200 as rb
    alone = []
    for b in batch:
        c = b.copy()
        st, _, rep = rb.CalcPLSA(c, precision=precision)
        alone.append((st, c, rep))
    many = [b.copy() for b in batch]
    sts, reps, br = rb.solve_batch(many, workers=workers, precision=precision)
    print("batch", br)
    assert br["workers"] >= 1 and br["scenes_per_second"] > 0
    for (st, c, rep), st_b, m, rep_b in zip(alone, sts, many, reps):
        assert st_b == st
        assert rep_b["linear_solves"] == rep["linear_solves"]
        assert rep_b["cost"] == rep["cost"]
        for name in ("pmat", "K", "distpara", "XX", "pt_obs_off", "pt_obs_image", "pt_obs_slot"):
            assert np.array_equal(getattr(m, name), getattr(c, name)), name
