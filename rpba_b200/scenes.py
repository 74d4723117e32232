"""Seeded synthetic scenes in the BAL camera model.

Public BAL datasets are not available offline, so seeded synthetic scenes with
the shapes, sizes and value distributions of the benchmark configurations
stand in for them.  The camera model is BAL's: angle-axis rotation R,
translation t, focal length f and radial k1, k2; a point X projects to
P = R X + t, p = -P.xy / P.z, x = f (1 + k1 |p|^2 + k2 |p|^4) p.

``to_block`` converts BAL arrays to a ``Block`` with the quantisation of
InputBlock (rpba.cpp:180-284): rotation from the double angle-axis stored as
float, float translation / focal / distortion / points / observations,
observations negated (rpba.cpp:268-272), unit weights, and ``k24out``
handling of k1, k2 (rpba.cpp:255-262).

Scene families (sizes are those of the benchmark configurations):
  arc      50 cameras on a 10 m arc, 8k points in a 4 m box (config 0)
  street   1,000 forward cameras, 3 m spacing, 190k points (config 1)
  aerial   3,000 nadir cameras on a grid, 310k terrain points (config 2)
  city     13,700 cameras in 50 clusters, 4.5M points (config 3)
  batch    scenes of the arc family with 20..400 cameras (config 4)
"""
from __future__ import annotations

from dataclasses import dataclass

import os

import numpy as np

from .block import Block


@dataclass
class BAL:
    cam_aa: np.ndarray   # (n, 3) float64 angle-axis
    cam_t: np.ndarray    # (n, 3) float32
    cam_f: np.ndarray    # (n,) float32
    cam_k: np.ndarray    # (n, 2) float32 (k1, k2)
    pts: np.ndarray      # (p, 3) float32
    obs_cam: np.ndarray  # (o,) int32
    obs_pt: np.ndarray   # (o,) int32, non-decreasing (point-major file order)
    obs_xy: np.ndarray   # (o, 2) float32

    @property
    def n_cams(self):
        return int(self.cam_aa.shape[0])

    @property
    def n_pts(self):
        return int(self.pts.shape[0])

    @property
    def n_obs(self):
        return int(self.obs_cam.shape[0])


# ----------------------------------------------------------------- rotations


def host_share() -> int:
    """Host cores for this process's generator pool: the node's cores split
    between the processes torchrun starts on it (LOCAL_WORLD_SIZE), so that
    ranks generating their scenes at once do not oversubscribe the host."""
    local = max(1, int(os.environ.get("LOCAL_WORLD_SIZE", "1")))
    return max(1, (os.cpu_count() or 1) // local)

def aa_to_R(aa: np.ndarray) -> np.ndarray:
    """Angle-axis -> rotation (rpba.cpp:343-366 formula), float64."""
    a, b, c = aa[:, 0], aa[:, 1], aa[:, 2]
    a2, b2, c2 = a * a, b * b, c * c
    th = np.sqrt(a2 + b2 + c2)
    z = th == 0.0
    ths = np.where(z, 1.0, th)
    ct = np.where(z, 0.5, (1.0 - np.cos(ths)) / (ths * ths))
    st = np.where(z, 1.0, np.sin(ths) / ths)
    R = np.empty((aa.shape[0], 3, 3))
    R[:, 0, 0] = 1.0 - (b2 + c2) * ct
    R[:, 0, 1] = a * b * ct - c * st
    R[:, 0, 2] = a * c * ct + b * st
    R[:, 1, 0] = a * b * ct + c * st
    R[:, 1, 1] = 1.0 - (c2 + a2) * ct
    R[:, 1, 2] = b * c * ct - a * st
    R[:, 2, 0] = a * c * ct - b * st
    R[:, 2, 1] = b * c * ct + a * st
    R[:, 2, 2] = 1.0 - (a2 + b2) * ct
    return R


def R_to_aa(R: np.ndarray) -> np.ndarray:
    """Rotation -> angle-axis (log map) for rotations away from pi."""
    tr = np.clip((np.trace(R, axis1=1, axis2=2) - 1.0) * 0.5, -1.0, 1.0)
    th = np.arccos(tr)
    w = np.stack([R[:, 2, 1] - R[:, 1, 2], R[:, 0, 2] - R[:, 2, 0], R[:, 1, 0] - R[:, 0, 1]], 1)
    s = np.sin(th)
    fac = np.where(s > 1e-12, th / (2.0 * np.where(s > 1e-12, s, 1.0)), 0.5)
    return w * fac[:, None]


def look_at(C: np.ndarray, T: np.ndarray, up: np.ndarray) -> np.ndarray:
    """Rotations (world->camera) of cameras at C looking at T, BAL convention
    (the camera looks along its -z axis)."""
    fwd = T - C
    fwd /= np.linalg.norm(fwd, axis=1, keepdims=True)
    z = -fwd
    x = np.cross(np.broadcast_to(up, z.shape), z)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    y = np.cross(z, x)
    return np.stack([x, y, z], axis=1)


def small_rotation(rng, n, angle):
    ax = rng.normal(size=(n, 3))
    ax /= np.linalg.norm(ax, axis=1, keepdims=True)
    return aa_to_R(ax * angle)


# ------------------------------------------------------------- projection

def project(R, t, f, k, X, cam, pt):
    """BAL projection of points pt through cameras cam; returns (xy, P.z, |p|inf)."""
    P = np.einsum("nij,nj->ni", R[cam], X[pt]) + t[cam]
    pz = P[:, 2]
    safe = np.where(np.abs(pz) < 1e-9, -1e-9, pz)
    p = -P[:, :2] / safe[:, None]
    r2 = (p * p).sum(1)
    d = 1.0 + k[cam, 0] * r2 + k[cam, 1] * r2 * r2
    return f[cam, None] * d[:, None] * p, pz, np.abs(p).max(1)


def _select_tracks(rng, prop, vis, t_want):
    """First t_want distinct visible proposals of every row."""
    n, K = prop.shape
    order = np.argsort(prop, axis=1, kind="stable")
    sp = np.take_along_axis(prop, order, 1)
    dup_sorted = np.zeros_like(sp, dtype=bool)
    dup_sorted[:, 1:] = sp[:, 1:] == sp[:, :-1]
    # a duplicate only disqualifies later copies; keep the first visible copy
    vis_sorted = np.take_along_axis(vis, order, 1)
    # mark any copy after the first visible one as duplicate
    first_vis = np.zeros_like(vis_sorted)
    # group ids in sorted order
    grp = np.cumsum(~dup_sorted, axis=1)
    # first visible element of each group: visible and no earlier visible in group
    cum_vis = np.zeros_like(vis_sorted, dtype=np.int32)
    # per-group running count of visible entries
    for j in range(K):
        if j == 0:
            cum_vis[:, j] = vis_sorted[:, j]
        else:
            same = grp[:, j] == grp[:, j - 1]
            cum_vis[:, j] = np.where(same, cum_vis[:, j - 1], 0) + vis_sorted[:, j]
    first_vis = vis_sorted & (cum_vis == 1)
    keep = np.zeros_like(vis)
    np.put_along_axis(keep, order, first_vis, 1)
    rank = np.cumsum(keep, axis=1)
    take = keep & (rank <= t_want[:, None])
    return take


def _track_lengths(rng, n, mean, lo, hi):
    # lo + geometric(p) - 1 with mean `mean`
    p = 1.0 / (mean - lo + 1.0)
    t = lo + rng.geometric(p, size=n) - 1
    return np.minimum(t, hi)


def _chunk_tracks(job):
    """Tracks of the points [s, e): proposals, visibility, selection.  Each
    chunk draws from its own seed, so the result does not depend on how the
    chunks are spread over processes."""
    s, e, seed, props, vis_fn, t_want, n_c = job
    rng = np.random.default_rng(seed)
    prop = props(rng, s, e)
    n, K = prop.shape
    pt = np.repeat(np.arange(s, e), K)
    vis = vis_fn(prop.ravel(), pt).reshape(n, K)
    take = _select_tracks(rng, prop, vis, t_want[s:e])
    cnt = take.sum(1)
    take &= (cnt >= 2)[:, None]
    rows, cols = np.nonzero(take)
    c = prop[rows, cols]
    # cameras ascending within a track
    key = (rows + s).astype(np.int64) * (n_c + 1) + c
    o = np.argsort(key, kind="stable")
    return c[o].astype(np.int32), (rows[o] + s).astype(np.int32)


def _assemble(rng, R_true, C_true, f_true, k_true, X_true, props, vis_fn, t_want,
              noise=0.5, outlier_frac=0.03, outlier_px=50.0, rot_pert=0.01,
              t_pert=0.05, pt_pert=0.05, f_pert=0.02, chunk=200_000, workers=None):
    """Build a BAL problem from proposals; drops points seen < 2 times."""
    n_c = R_true.shape[0]
    t_true = -np.einsum("nij,nj->ni", R_true, C_true)
    n_p = X_true.shape[0]
    base = int(rng.integers(0, 2**62))
    jobs = [(s, min(s + chunk, n_p), base + s, props, vis_fn, t_want, n_c) for s in range(0, n_p, chunk)]
    if workers is None:
        workers = min(len(jobs), host_share(), 32) if n_p > 1_000_000 else 1
    if workers > 1:
        # spawn (not fork): callers may already hold a CUDA context
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
            res = list(ex.map(_chunk_tracks, jobs))
    else:
        res = [_chunk_tracks(j) for j in jobs]
    obs_cam = np.concatenate([r[0] for r in res])
    obs_pt = np.concatenate([r[1] for r in res])
    # re-index points seen >= 2 times
    used = np.unique(obs_pt)
    remap = -np.ones(X_true.shape[0], np.int64)
    remap[used] = np.arange(used.size)
    obs_pt = remap[obs_pt].astype(np.int32)
    X_true = X_true[used]
    xy = np.empty((obs_cam.size, 2))
    for s in range(0, obs_cam.size, 4 * chunk):
        e = min(s + 4 * chunk, obs_cam.size)
        xy[s:e], _, _ = project(R_true, t_true, f_true, k_true, X_true, obs_cam[s:e], obs_pt[s:e])
    xy += rng.normal(scale=noise, size=xy.shape)
    out = rng.random(obs_cam.size) < outlier_frac
    xy[out] += rng.uniform(-outlier_px, outlier_px, size=(int(out.sum()), 2))
    # initial state
    R0 = np.einsum("nij,njk->nik", small_rotation(rng, n_c, rot_pert), R_true)
    C0 = C_true + rng.normal(scale=t_pert / np.sqrt(3.0), size=C_true.shape)
    t0 = -np.einsum("nij,nj->ni", R0, C0)
    f0 = f_true * (1.0 + rng.normal(scale=f_pert, size=f_true.shape))
    X0 = X_true + rng.normal(scale=pt_pert / np.sqrt(3.0), size=X_true.shape)
    return BAL(R_to_aa(R0), t0.astype(np.float32), f0.astype(np.float32),
               k_true.astype(np.float32), X0.astype(np.float32), obs_cam, obs_pt,
               xy.astype(np.float32))


class _Vis:
    """Visibility: in front of the camera and inside the image."""

    def __init__(self, R, t, f, k, X, max_p, min_depth):
        self.a = (R, t, f, k, X)
        self.max_p, self.min_depth = max_p, min_depth

    def __call__(self, cam, pt):
        out = np.zeros(cam.size, bool)
        for s in range(0, cam.size, 2_000_000):
            e = min(s + 2_000_000, cam.size)
            _, pz, pinf = project(*self.a, cam[s:e], pt[s:e])
            out[s:e] = (pz < -self.min_depth) & (pinf < self.max_p)
        return out


class _ArcProps:
    def __init__(self, n_cams, K):
        self.n_cams, self.K = n_cams, K

    def __call__(self, rng, s, e):
        return np.argsort(rng.random((e - s, self.n_cams)), axis=1)[:, :self.K].astype(np.int64)


class _StreetProps:
    def __init__(self, xp, lo, hi, spacing, n_cams, K):
        self.xp, self.lo, self.hi, self.spacing, self.n_cams, self.K = xp, lo, hi, spacing, n_cams, K

    def __call__(self, rng, s, e):
        i_hi = np.floor((self.xp[s:e] - self.lo) / self.spacing).astype(np.int64)
        span = int(np.ceil((self.hi - self.lo) / self.spacing))
        off = rng.integers(0, span, size=(e - s, self.K))
        return np.clip(i_hi[:, None] - off, 0, self.n_cams - 1)


class _AerialProps:
    def __init__(self, xz, x0, y0, spacing, nx, ny, K):
        self.xz, self.x0, self.y0, self.spacing, self.nx, self.ny, self.K = xz, x0, y0, spacing, nx, ny, K

    def __call__(self, rng, s, e):
        ix = np.round((self.xz[s:e, 0] - self.x0) / self.spacing).astype(np.int64)
        iy = np.round((self.xz[s:e, 1] - self.y0) / self.spacing).astype(np.int64)
        dx = rng.integers(-2, 3, size=(e - s, self.K))
        dy = rng.integers(-2, 3, size=(e - s, self.K))
        cx = np.clip(ix[:, None] + dx, 0, self.nx - 1)
        cy = np.clip(iy[:, None] + dy, 0, self.ny - 1)
        return cy * self.nx + cx


class _CityProps:
    def __init__(self, pc, nbr_pad, is_inter, cpc, K):
        self.pc, self.nbr_pad, self.is_inter, self.cpc, self.K = pc, nbr_pad, is_inter, cpc, K

    def __call__(self, rng, s, e):
        n, K = e - s, self.K
        home = self.pc[s:e]
        own = home[:, None] * self.cpc + rng.integers(0, self.cpc, (n, K))
        other_c = self.nbr_pad[home, rng.integers(0, 8, n)]
        oth = other_c[:, None] * self.cpc + rng.integers(0, self.cpc, (n, K))
        use_oth = self.is_inter[s:e, None] & (rng.random((n, K)) < 0.3)
        return np.where(use_oth, oth, own)


def _intrinsics(rng, n, flo, fhi):
    f = rng.uniform(flo, fhi, n)
    k = np.stack([rng.normal(0, 1e-2, n), rng.normal(0, 1e-4, n)], 1)
    return f, k


# -------------------------------------------------------------- families

def arc_scene(seed=20260, n_cams=50, n_pts=8000, track_mean=4.0, track_max=12,
              outlier_frac=0.03, radius=10.0, box=4.0, noise=0.5, **kw) -> BAL:
    rng = np.random.default_rng(seed)
    th = np.linspace(-0.5 * np.pi, 0.5 * np.pi, n_cams) + rng.normal(0, 0.01, n_cams)
    C = np.stack([radius * np.sin(th), 1.5 + rng.normal(0, 0.1, n_cams), radius * np.cos(th)], 1)
    T = rng.normal(0, 0.2, (n_cams, 3))
    R = look_at(C, T, np.array([0.0, 1.0, 0.0]))
    f, k = _intrinsics(rng, n_cams, 400, 600)
    X = rng.uniform(-box / 2, box / 2, (n_pts, 3))
    t_want = _track_lengths(rng, n_pts, track_mean, 2, min(track_max, n_cams))
    K = min(n_cams, 3 * track_max)
    t = -np.einsum("nij,nj->ni", R, C)
    return _assemble(rng, R, C, f, k, X, _ArcProps(n_cams, K), _Vis(R, t, f, k, X, 1.5, 0.5), t_want,
                     outlier_frac=outlier_frac, noise=noise, **kw)


def street_scene(seed=20261, n_cams=1000, n_pts=190_000, spacing=3.0, track_mean=5.0,
                 track_max=30, outlier_frac=0.05, **kw) -> BAL:
    rng = np.random.default_rng(seed)
    L = n_cams * spacing
    xs = np.arange(n_cams) * spacing
    C = np.stack([xs, 2.0 + rng.normal(0, 0.05, n_cams), rng.normal(0, 0.3, n_cams)], 1)
    T = C + np.stack([np.full(n_cams, 20.0), rng.normal(0, 0.3, n_cams), rng.normal(0, 0.5, n_cams)], 1)
    R = look_at(C, T, np.array([0.0, 1.0, 0.0]))
    f, k = _intrinsics(rng, n_cams, 400, 600)
    lo, hi = 5.0, 110.0
    # points from the first camera's view to the last camera's
    X = np.stack([rng.uniform(lo, L - spacing + hi, n_pts), rng.uniform(0, 10, n_pts),
                  rng.uniform(-10, 10, n_pts)], 1)
    t_want = _track_lengths(rng, n_pts, track_mean, 2, track_max)
    K = 2 * track_max
    t = -np.einsum("nij,nj->ni", R, C)
    return _assemble(rng, R, C, f, k, X, _StreetProps(X[:, 0].copy(), lo, hi, spacing, n_cams, K),
                     _Vis(R, t, f, k, X, 1.2, 3.0), t_want, outlier_frac=outlier_frac, **kw)


def _height(x, y):
    return (8.0 * np.sin(x / 170.0) * np.cos(y / 230.0) + 5.0 * np.sin(x / 61.0 + 1.3) * np.sin(y / 83.0)
            + 2.0 * np.cos(x / 23.0 - y / 31.0) + 15.0)


def aerial_scene(seed=20262, nx=60, ny=50, n_pts=310_000, track_mean=5.3, track_max=30,
                 outlier_frac=0.03, **kw) -> BAL:
    rng = np.random.default_rng(seed)
    n_cams = nx * ny
    f, k = _intrinsics(rng, n_cams, 1000, 3000)
    h = 100.0 + 50.0 * (np.arange(n_cams) // nx % 3) / 2.0
    spacing = 0.4 * 2 * 0.45 * 125.0   # 60% overlap of a ~110 m footprint
    gx, gy = np.meshgrid(np.arange(nx) * spacing, np.arange(ny) * spacing)
    gx = gx.ravel() + rng.normal(0, 2, n_cams)
    gy = gy.ravel() + rng.normal(0, 2, n_cams)
    C = np.stack([gx, h + rng.normal(0, 1, n_cams), gy], 1)
    T = np.stack([gx + rng.normal(0, 3, n_cams), np.zeros(n_cams), gy + rng.normal(0, 3, n_cams)], 1)
    R = look_at(C, T, np.array([0.0, 0.0, 1.0]))
    px = rng.uniform(gx.min(), gx.max(), n_pts)
    pz = rng.uniform(gy.min(), gy.max(), n_pts)
    X = np.stack([px, _height(px, pz), pz], 1)
    t_want = _track_lengths(rng, n_pts, track_mean, 2, track_max)
    K = 2 * track_max
    t = -np.einsum("nij,nj->ni", R, C)
    return _assemble(rng, R, C, f, k, X, _AerialProps(X[:, [0, 2]].copy(), gx.min(), gy.min(), spacing, nx, ny, K),
                     _Vis(R, t, f, k, X, 0.45, 10.0), t_want, outlier_frac=outlier_frac, **kw)


def city_scene(seed=20263, n_clusters=50, cams_per_cluster=274, n_pts=4_500_000,
               track_mean=6.5, track_max=100, inter=0.2, outlier_frac=0.03, **kw) -> BAL:
    rng = np.random.default_rng(seed)
    gxn = 10
    n_cams = n_clusters * cams_per_cluster
    cid = np.repeat(np.arange(n_clusters), cams_per_cluster)
    centers = np.stack([(np.arange(n_clusters) % gxn) * 90.0, np.zeros(n_clusters),
                        (np.arange(n_clusters) // gxn) * 90.0], 1)
    th = rng.uniform(0, 2 * np.pi, n_cams)
    rad = rng.uniform(35.0, 55.0, n_cams)
    C = centers[cid] + np.stack([rad * np.cos(th), rng.uniform(2, 25, n_cams), rad * np.sin(th)], 1)
    T = centers[cid] + rng.normal(0, 8.0, (n_cams, 3)) * np.array([1.0, 0.3, 1.0])
    R = look_at(C, T, np.array([0.0, 1.0, 0.0]))
    f, k = _intrinsics(rng, n_cams, 400, 600)
    pc = rng.integers(0, n_clusters, n_pts)
    X = centers[pc] + rng.uniform(-1, 1, (n_pts, 3)) * np.array([30.0, 0.0, 30.0]) \
        + np.stack([np.zeros(n_pts), rng.uniform(0, 20, n_pts), np.zeros(n_pts)], 1)
    t_want = _track_lengths(rng, n_pts, track_mean, 2, track_max)
    K = int(1.5 * track_max)
    gx = np.arange(n_clusters) % gxn
    gy = np.arange(n_clusters) // gxn
    nbr = []
    for c in range(n_clusters):
        cand = [d for d in range(n_clusters) if d != c and abs(gx[d] - gx[c]) <= 1 and abs(gy[d] - gy[c]) <= 1]
        nbr.append(cand)
    nbr_pad = np.array([(n + n * 8)[:8] for n in nbr])
    is_inter = rng.random(n_pts) < inter
    t = -np.einsum("nij,nj->ni", R, C)
    return _assemble(rng, R, C, f, k, X, _CityProps(pc, nbr_pad, is_inter, cams_per_cluster, K),
                     _Vis(R, t, f, k, X, 1.0, 2.0), t_want, outlier_frac=outlier_frac, chunk=100_000, **kw)


def batch_scene_specs(seed=20264, n_scenes=256, cmin=20, cmax=400, pts_per_cam=150):
    """Keyword arguments of arc_scene for every scene of the batched workload."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_scenes):
        nc = int(rng.integers(cmin, cmax + 1))
        out.append(dict(seed=seed * 1000 + i, n_cams=nc, n_pts=pts_per_cam * nc, track_mean=4.0, track_max=12))
    return out


def _arc_block(kw):
    return to_block(arc_scene(**kw))


def batch_scenes(seed=20264, n_scenes=256, cmin=20, cmax=400, pts_per_cam=150):
    return [arc_scene(**kw) for kw in batch_scene_specs(seed, n_scenes, cmin, cmax, pts_per_cam)]


def batch_blocks(seed=20264, n_scenes=256, cmin=20, cmax=400, pts_per_cam=150, workers=None):
    """The batched workload as blocks, generated in parallel processes."""
    specs = batch_scene_specs(seed, n_scenes, cmin, cmax, pts_per_cam)
    workers = workers or min(len(specs), host_share(), 32)
    if workers <= 1:
        return [_arc_block(kw) for kw in specs]
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_arc_block, specs, chunksize=4))


CONFIGS = {
    0: ("arc", arc_scene),
    1: ("street", street_scene),
    2: ("aerial", aerial_scene),
    3: ("city", city_scene),
}


def make_scene(config: int, scale: float = 1.0, seed: int | None = None) -> BAL:
    """Scene of a benchmark configuration; ``scale`` < 1 shrinks cameras and
    points proportionally (for oracle-sized parity cases)."""
    name, fn = CONFIGS[config]
    s = 20260 + config if seed is None else seed
    if config == 0:
        return arc_scene(seed=s, n_cams=max(4, int(round(50 * scale))), n_pts=max(50, int(8000 * scale)))
    if config == 1:
        return street_scene(seed=s, n_cams=max(20, int(1000 * scale)), n_pts=max(500, int(190_000 * scale)))
    if config == 2:
        nx = max(6, int(round(60 * np.sqrt(scale))))
        ny = max(5, int(round(50 * np.sqrt(scale))))
        return aerial_scene(seed=s, nx=nx, ny=ny, n_pts=max(1000, int(310_000 * scale)))
    if config == 3:
        ncl = max(2, int(round(50 * scale)))
        return city_scene(seed=s, n_clusters=ncl, n_pts=max(2000, int(4_500_000 * scale)))
    raise ValueError(config)


# ---------------------------------------------------------------- block

def to_block(bal: BAL, k24out: bool = True) -> Block:
    """InputBlock's conversion (rpba.cpp:180-284) of in-memory BAL arrays."""
    n, npt, no = bal.n_cams, bal.n_pts, bal.n_obs
    R = aa_to_R(bal.cam_aa).astype(np.float32)
    pmat = np.zeros((n, 3, 4), np.float32)
    pmat[:, :, :3] = R
    pmat[:, :, 3] = bal.cam_t
    K = np.zeros((n, 3, 3), np.float32)
    K[:, 0, 0] = bal.cam_f
    K[:, 1, 1] = bal.cam_f
    K[:, 2, 2] = 1.0
    f = bal.cam_f.astype(np.float32)
    if k24out:
        dist = bal.cam_k.astype(np.float32)
    else:
        dist = np.stack([bal.cam_k[:, 0] * f * f, bal.cam_k[:, 1] * f * f * f * f], 1).astype(np.float32)
    # slots per image in file order
    cam = bal.obs_cam.astype(np.int64)
    cnt = np.bincount(cam, minlength=n)
    img_off = np.zeros(n + 1, np.int64)
    img_off[1:] = np.cumsum(cnt)
    order = np.argsort(cam, kind="stable")
    slot_global = np.empty(no, np.int64)
    slot_global[order] = np.arange(no)
    slot = slot_global - img_off[cam]
    xg = np.empty((no, 2), np.float32)
    xg[slot_global] = -bal.obs_xy
    pcnt = np.bincount(bal.obs_pt, minlength=npt)
    pt_off = np.zeros(npt + 1, np.int64)
    pt_off[1:] = np.cumsum(pcnt)
    porder = np.argsort(bal.obs_pt, kind="stable")
    return Block(pmat.reshape(n, 12), K.reshape(n, 9), dist, bal.pts.astype(np.float32).copy(),
                 img_off.astype(np.int32), xg, np.ones(no, np.float32), np.ones(no, np.float32),
                 np.zeros(no, np.float32), pt_off.astype(np.int32),
                 bal.obs_cam[porder].astype(np.int32), slot[porder].astype(np.int32))


def write_bal(path: str, bal: BAL) -> None:
    """BAL text (the format InputBlock reads)."""
    with open(path, "w") as fh:
        fh.write(f"{bal.n_cams} {bal.n_pts} {bal.n_obs}\n")
        for c, p, (x, y) in zip(bal.obs_cam.tolist(), bal.obs_pt.tolist(), bal.obs_xy.tolist()):
            fh.write(f"{c} {p} {x!r} {y!r}\n")
        for i in range(bal.n_cams):
            a, b, c = bal.cam_aa[i].tolist()
            t0, t1, t2 = (repr(float(np.float32(v))) for v in bal.cam_t[i])
            fh.write(f"{a!r} {b!r} {c!r} {t0} {t1} {t2} {float(bal.cam_f[i])!r} "
                     f"{float(bal.cam_k[i, 0])!r} {float(bal.cam_k[i, 1])!r}\n")
        for p in range(bal.n_pts):
            fh.write(" ".join(repr(float(v)) for v in bal.pts[p]) + "\n")
