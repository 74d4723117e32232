"""Known-answer tests pinning the oracle (the reference itself cannot be
built here): rotation conversions, the 3x3 and LU inverses, finite-difference
checks of every Jacobian column, a zero-noise scene, Exteval arithmetic and
the exact-sum model."""
import numpy as np
import pytest

from rpba_b200 import scenes


def test_cayley_small_angle_and_orthonormal(oracle_mod):
    R0 = oracle_mod.cayley(0.0, 0.0, 0.0)
    assert np.array_equal(R0, np.eye(3))
    rng = np.random.default_rng(0)
    for _ in range(20):
        a, b, c = rng.normal(0, 0.3, 3)
        R = oracle_mod.cayley(a, b, c)
        assert np.abs(R @ R.T - np.eye(3)).max() < 1e-14
        assert abs(np.linalg.det(R) - 1) < 1e-14
        # first order: I + [w]x with w = (a, b, c)
    R = oracle_mod.cayley(1e-6, -2e-6, 3e-6)
    W = np.array([[0, -3e-6, -2e-6], [3e-6, 0, -1e-6], [2e-6, 1e-6, 0]])
    assert np.abs(R - (np.eye(3) + W)).max() < 1e-11


def test_rectify_projects_to_rotation(oracle_mod):
    rng = np.random.default_rng(1)
    for _ in range(20):
        # away from pi, where the quaternion axis (from sin(theta)) is ill-conditioned
        aa = rng.normal(0, 1, 3)
        aa *= min(1.0, 2.5 / np.linalg.norm(aa))
        R = scenes.aa_to_R(aa[None])[0]
        Rn = R + rng.normal(0, 1e-6, (3, 3))
        Rr = oracle_mod.rectify3(Rn)
        assert np.abs(Rr @ Rr.T - np.eye(3)).max() < 1e-14
        assert np.abs(Rr - R).max() < 1e-5


def test_angleaxis_round_trip(oracle_mod):
    rng = np.random.default_rng(2)
    for _ in range(50):
        aa = rng.normal(0, 1, 3)
        aa *= min(1.0, 3.0 / np.linalg.norm(aa))
        R = oracle_mod.angleaxis_to_R(*aa)
        back = oracle_mod.R_to_angleaxis(R)
        assert np.abs(back - aa).max() < 2e-5, (aa, back)
    assert np.array_equal(oracle_mod.R_to_angleaxis(np.eye(3, dtype=np.float32)), np.zeros(3))


def test_inverses(oracle_mod):
    rng = np.random.default_rng(3)
    for _ in range(20):
        A = rng.normal(size=(3, 3)) + 3 * np.eye(3)
        Ai, det = oracle_mod.inv3(A)
        assert np.abs(Ai @ A - np.eye(3)).max() < 1e-13
        assert abs(det - np.linalg.det(A)) < 1e-12 * abs(det) * 10
        for n in (3, 5, 8, 9):
            B = rng.normal(size=(n, n))
            B = B @ B.T + n * np.eye(n)
            assert np.abs(oracle_mod.lu_inverse(B) @ B - np.eye(n)).max() < 1e-12


@pytest.mark.parametrize("addflags", [(1, 1, 1), (1, 0, 1), (0, 0, 0)])
def test_jacobians_match_finite_differences(oracle_mod, addflags):
    import rpba_b200 as rb
    blk = scenes.to_block(scenes.arc_scene(seed=5, n_cams=6, n_pts=60, outlier_frac=0.0))
    L = oracle_mod.OracleLSA(blk, rb.make_options(k2=addflags[0], k4=addflags[1], f=addflags[2]))
    xm = L.xm()
    nrioff = L.nrioff
    n = L.n_obs
    offs = blk.pt_obs_off
    worst = 0.0
    for o in range(0, n, 3):
        Bc, co, Bp = L.jacobian(o)
        p = int(np.searchsorted(offs, o, side="right") - 1)
        cols = [(co + j, Bc[:, j]) for j in range(Bc.shape[1])]
        cols += [(nrioff + 3 * p + j, Bp[:, j]) for j in range(3)]
        for j, an in cols:
            h = 1e-6 * max(1.0, abs(xm[j]))
            xp, xq = xm.copy(), xm.copy()
            xp[j] += h
            xq[j] -= h
            fd = (L.residuals(xp)[o] - L.residuals(xq)[o]) / (2 * h)
            err = np.abs(fd - an).max() / (np.abs(an).max() + 1e-3)
            worst = max(worst, err)
    L.close()
    assert worst < 1e-5, worst


def test_zero_noise_scene_converges_to_zero(oracle_mod):
    import rpba_b200 as rb
    bal = scenes.arc_scene(seed=9, n_cams=10, n_pts=600, outlier_frac=0.0, noise=0.0)
    st, b, rep, log = oracle_mod.calc_plsa(scenes.to_block(bal), rb.make_options(robust=False))
    assert st == 0
    assert rep["rms"] < 1e-3, rep["rms"]


def test_exteval_zero_for_consistent_block(oracle_mod):
    """A block whose observations are its own float projections has zero
    back-projection error up to float rounding of the observations."""
    import rpba_b200 as rb
    blk = scenes.to_block(scenes.arc_scene(seed=12, n_cams=5, n_pts=200, outlier_frac=0.0))
    n = blk.n_obs
    sl = blk.track_slots()
    P = blk.pmat.reshape(-1, 3, 4).astype(np.float64)
    pt = np.repeat(np.arange(blk.n_points), np.diff(blk.pt_obs_off))
    im = blk.pt_obs_image[:n]
    X = blk.XX[pt].astype(np.float64)
    p = np.einsum("nij,nj->ni", P[im, :, :3], X) + P[im, :, 3]
    p1, p2 = p[:, 0] / p[:, 2], p[:, 1] / p[:, 2]
    r2 = p1 * p1 + p2 * p2
    d = 1 + blk.distpara[im, 0].astype(np.float64) * r2 + blk.distpara[im, 1].astype(np.float64) * r2 * r2
    f = blk.K[im, 0].astype(np.float64)
    xg = blk.xg.copy()
    xg[sl, 0] = (p1 * d * f).astype(np.float32)
    xg[sl, 1] = (p2 * d * f).astype(np.float32)
    blk.xg = xg
    res, rep = oracle_mod.exteval(blk, rb.make_options())
    assert np.abs(res).max() < 1e-3
    assert rep["exteval_nrobs"] == 2 * n


def test_exact_sum_model_matches_sequential():
    """The binade-run method used by the GPU sums, modelled in numpy."""
    import math
    rng = np.random.default_rng(11)

    def model(v, H=2048):
        s, i, n = np.float32(0), 0, len(v)
        while i < n and (i < H or s < np.float32(2.0 ** -126)):
            s = np.float32(s + v[i])
            i += 1
        while i < n:
            E = math.frexp(float(s))[1] - 1
            u = 2.0 ** (E - 23)
            S = int(float(s) / u)
            f = v[i:].astype(np.float64) / u
            fl = np.floor(f)
            fr = f - fl
            r = fl + (fr > 0.5)
            R = np.concatenate([[0.0], np.cumsum(r)])
            ev = np.nonzero((S + R[:-1] + fl >= 2 ** 24) | (fr == 0.5))[0]
            if len(ev) == 0:
                return np.float32((S + R[-1]) * u)
            k = ev[0]
            s = np.float32(np.float32((S + R[k]) * u) + v[i + k])
            i += k + 1
        return s

    for kind in range(4):
        n = 150_000
        if kind == 0:
            v = (rng.normal(0, 0.5, n) ** 2).astype(np.float32)
        elif kind == 1:
            v = (rng.integers(0, 4, n) * 0.5).astype(np.float32)
        elif kind == 2:
            v = np.exp(rng.normal(0, 6, n)).astype(np.float32)
        else:
            v = np.full(n, 2.0, np.float32)
            v[rng.random(n) < 0.1] = np.float32(2e-4)
        assert model(v) == np.cumsum(v, dtype=np.float32)[-1]
