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


def _obs_normal(blk, p, X):
    """Per-observation normal matrices B^T W B of point p at X, restated in
    numpy from the projection and calibration of CalcLSAXMulti
    (rpbacore.cpp:594-626, 841-877), with the float roundings of its
    projection values."""
    out, ims = [], []
    for t in range(blk.pt_obs_off[p], blk.pt_obs_off[p + 1]):
        j = int(blk.pt_obs_image[t])
        sl = int(blk.img_obs_off[j] + blk.pt_obs_slot[t])
        P = blk.pmat[j].astype(np.float64)
        p1 = P[0] * X[0] + P[1] * X[1] + P[2] * X[2] + P[3]
        p2 = P[4] * X[0] + P[5] * X[1] + P[6] * X[2] + P[7]
        p3 = P[8] * X[0] + P[9] * X[1] + P[10] * X[2] + P[11]
        p3 = (1e3 if p3 > 0 else -1e3) if abs(p3) < 1e-3 else 1.0 / p3
        x, y, f3 = np.float32(p1 * p3), np.float32(p2 * p3), np.float32(p3)
        x, y, f3 = float(x), float(y), float(f3)
        xp = np.array([P[c] * f3 - P[8 + c] * (x * f3) for c in range(3)])
        yp = np.array([P[4 + c] * f3 - P[8 + c] * (y * f3) for c in range(3)])
        k2, k4 = float(blk.distpara[j][0]), float(blk.distpara[j][1])
        fx, fy, sk = float(blk.K[j][0]), float(blk.K[j][4]), float(blk.K[j][1])
        r2 = x * x + y * y
        r4 = r2 * r2
        axx = k4 * r4 + x * (2 * k2 * x + 4 * k4 * x * r2) + k2 * r2 + 1.0
        axy = x * (4 * k4 * r2 * y + 2 * k2 * y)
        ayx = y * (4 * k4 * x * r2 + 2 * k2 * x)
        ayy = y * (2 * k2 * y + 4 * k4 * r2 * y) + k4 * r4 + k2 * r2 + 1.0
        nx, ny = axx * xp + axy * yp, ayy * yp + ayx * xp
        bx, by = nx * fx + ny * sk, ny * fy
        wx, wy, wxy = float(blk.wx[sl]), float(blk.wy[sl]), float(blk.wxy[sl])
        w0, w1 = bx * wx + by * wxy, by * wy + bx * wxy
        out.append(np.outer(bx, w0) + np.outer(by, w1))
        ims.append(j)
    return out, ims


def test_oracle_weight_blocks(oracle_mod):
    """The per-partition weight blocks of CalcLSAXMulti (wxyflag): for every
    partition that sees a point, the normal matrix of the point's
    observations in the other partitions, at the accepted iterate; zero for
    the partitions that do not see it.  The weight-only pass evaluates at
    the input point, where the blocks are recomputed in numpy.  The
    partition changes none of the other outputs."""
    import rpba_b200 as rb
    from rpba_b200 import scenes
    blk = scenes.to_block(scenes.arc_scene(seed=23, n_cams=20, n_pts=600, outlier_frac=0.0))
    k = 3
    part = rb.partition_images(blk, k)
    r = oracle_mod.triangulate_parts(blk, part, k, weight_only=True)
    base = oracle_mod.triangulate(blk, weight_only=True)
    for name in ("XX", "keep", "sig0v", "conv"):
        assert np.array_equal(r[name], base[name]), name
    assert r["sig0io"] == base["sig0io"] and r["redundancy"] == base["redundancy"]
    idx = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    checked = 0
    for p in np.nonzero(r["conv"])[0]:
        X = blk.XX[p].astype(np.float32).astype(np.float64)
        mats, ims = _obs_normal(blk, p, X)
        seen = set(int(part[j]) for j in ims)
        for i in range(k):
            want = np.zeros((3, 3))
            if i in seen:
                for M, j in zip(mats, ims):
                    if part[j] != i:
                        want += M
            got = r["w3d"][p, i]
            exp = np.array([want[a, b] for a, b in idx], np.float32)
            scale = max(1e-30, float(np.abs(exp).max()))
            assert np.abs(got - exp).max() <= 1e-5 * scale, (p, i, got, exp)
            checked += 1
    assert checked > 1000
    # one partition: the blocks are the whole (undamped) normal matrix
    r1 = oracle_mod.triangulate_parts(blk, np.zeros(blk.n_images, np.int32), 1, weight_only=True)
    p = int(np.nonzero(r1["conv"])[0][0])
    mats, _ = _obs_normal(blk, p, blk.XX[p].astype(np.float64))
    want = sum(mats)
    exp = np.array([want[a, b] for a, b in idx], np.float32)
    assert np.abs(r1["w3d"][p, 0] - exp).max() <= 1e-5 * np.abs(exp).max()
