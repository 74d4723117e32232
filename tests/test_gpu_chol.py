"""The tiled FP64 Cholesky factorisation and inverse (chol.cu: one
cooperative launch, tile products on the FP64 tensor cores), which inverts
the learned solver's coarse operator, against numpy on random SPD matrices
of sizes around the 64-wide tiles and at the coarse operator's largest size
(148 aggregates x 10 = 1,480); a matrix that is not positive definite is
reported."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 9, 63, 64, 65, 130, 300, 1480])
def test_spd_inverse_matches_numpy(n):
    import rpba_b200 as rb
    rng = np.random.default_rng(n)
    M = rng.normal(size=(n, n))
    A = M @ M.T / n + np.diag(rng.uniform(0.05, 2.0, n))
    Ai = rb.spd_inverse(A)
    ref = np.linalg.inv(A)
    cond = np.linalg.cond(A)
    err = np.abs(Ai - ref).max() / np.abs(ref).max()
    print(f"n={n}: rel err {err:.2e} cond {cond:.1e}")
    assert err <= 1e-13 * cond * max(1.0, np.sqrt(n))
    assert np.allclose(Ai, Ai.T, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_spd_inverse_rejects_indefinite():
    import rpba_b200 as rb
    A = np.eye(70)
    A[40, 40] = -1.0
    with pytest.raises(rb.RpbaError) as e:
        rb.spd_inverse(A)
    assert e.value.status == 10
