"""Comparison helpers for GPU-vs-oracle parity tests.

Tolerances (stated by the drop-in contract):
  final cost         relative 1e-8
  parameters         relative 1e-6 (scaled by the array's magnitude)
  Exteval residuals  absolute 1e-10 px
"""
import numpy as np

COST_RTOL = 1e-8
PARAM_RTOL = 1e-6
EXTEVAL_ATOL = 1e-10


def scaled_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.size == 0:
        return 0.0
    scale = max(np.abs(b).max(), 1e-12)
    return float(np.abs(a - b).max() / scale)


def param_errors(gpu_blk, ora_blk):
    """Scaled relative errors of the adjusted parameters."""
    n = gpu_blk.n_images
    P_g = gpu_blk.pmat.reshape(n, 3, 4)
    P_o = ora_blk.pmat.reshape(n, 3, 4)
    return {
        "R": scaled_err(P_g[:, :, :3], P_o[:, :, :3]),
        "t": scaled_err(P_g[:, :, 3], P_o[:, :, 3]),
        "f": scaled_err(gpu_blk.K[:, 0], ora_blk.K[:, 0]),
        "k1": scaled_err(gpu_blk.distpara[:, 0], ora_blk.distpara[:, 0]),
        "k2": scaled_err(gpu_blk.distpara[:, 1], ora_blk.distpara[:, 1]),
        "XX": scaled_err(gpu_blk.XX, ora_blk.XX),
    }


def same_tracks(a, b):
    return (np.array_equal(a.pt_obs_off, b.pt_obs_off)
            and np.array_equal(a.pt_obs_image[: a.n_obs], b.pt_obs_image[: b.n_obs])
            and np.array_equal(a.pt_obs_slot[: a.n_obs], b.pt_obs_slot[: b.n_obs]))


SIGMA_RTOL = 1e-5  # printed float sigma0: a few float ulps of the cost sum


def log_float_dev(a: str, b: str) -> float:
    """Largest relative difference between the float words of two logs with
    the same layout (0 when the layouts differ)."""
    dev = 0.0
    for x, y in zip(a.strip().splitlines(), b.strip().splitlines()):
        for u, v in zip(x.split(), y.split()):
            if u != v and any(c in u + v for c in ".e"):
                try:
                    dev = max(dev, abs(float(u) - float(v)) / max(abs(float(v)), 1e-30))
                except ValueError:
                    pass
    return dev


def same_log(a: str, b: str, rtol: float = SIGMA_RTOL) -> bool:
    """Log lines agree: words equal, numbers with a '.' or 'e' within
    rtol (default SIGMA_RTOL), integers exactly."""
    la, lb = a.strip().splitlines(), b.strip().splitlines()
    if len(la) != len(lb):
        return False
    for x, y in zip(la, lb):
        wx, wy = x.split(), y.split()
        if len(wx) != len(wy):
            return False
        for u, v in zip(wx, wy):
            if u == v:
                continue
            try:
                fu, fv = float(u), float(v)
            except ValueError:
                return False
            if not any(c in u + v for c in ".e") or abs(fu - fv) > rtol * max(abs(fv), 1e-30):
                return False
    return True
