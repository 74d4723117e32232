"""Host-side block container: numpy arrays laid out exactly as ``rpba_block``
(``include/rpba_b200.h``), which mirrors the containers ``CalcPLSA`` takes
(rpba.h:693-703): float projection matrices, cameras, points, per-image
observation slots ``xg``/``wx``/``wy``/``wxy`` and per-point ``pointXXv``
track lists of ``IMAPNR`` (image, pointnr) entries (rpba.h:88-93).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

_f32p = C.POINTER(C.c_float)
_i32p = C.POINTER(C.c_int32)


class RpbaBlockC(C.Structure):
    _fields_ = [
        ("n_images", C.c_int32),
        ("n_points", C.c_int32),
        ("pmat", _f32p),
        ("K", _f32p),
        ("distpara", _f32p),
        ("XX", _f32p),
        ("img_obs_off", _i32p),
        ("xg", _f32p),
        ("wx", _f32p),
        ("wy", _f32p),
        ("wxy", _f32p),
        ("pt_obs_off", _i32p),
        ("pt_obs_image", _i32p),
        ("pt_obs_slot", _i32p),
    ]


class RpbaOptionsC(C.Structure):
    _fields_ = [
        ("robust", C.c_int32),
        ("exteval", C.c_int32),
        ("threads", C.c_int32),
        ("k2", C.c_int32),
        ("k4", C.c_int32),
        ("f", C.c_int32),
        ("solver", C.c_int32),
        ("precision", C.c_int32),
        ("max_lm_iterations", C.c_int32),
        ("pcg_max_iterations", C.c_int32),
        ("pcg_tolerance", C.c_double),
        ("device", C.c_int32),
        ("verbose", C.c_int32),
        ("coarse_aggregates", C.c_int32),
    ]


class RpbaReportC(C.Structure):
    _fields_ = [
        ("sigma0_in", C.c_float * 2),
        ("sigma0_out", C.c_float * 2),
        ("redundancy", C.c_int32 * 2),
        ("nrobs", C.c_int32 * 2),
        ("nrunknowns", C.c_int32 * 2),
        ("itt", C.c_int32 * 2),
        ("passes_done", C.c_int32),
        ("linear_solves", C.c_int32),
        ("pcg_iterations", C.c_int64),
        ("pcg_fallbacks", C.c_int32),
        ("coarse_rebuilds", C.c_int32),
        ("obs_deleted", C.c_int32),
        ("points_deleted", C.c_int32),
        ("points_used", C.c_int32),
        ("cost", C.c_double),
        ("rms", C.c_double),
        ("exteval_sigma0", C.c_float),
        ("exteval_nrobs", C.c_int64),
        ("exteval_redundancy", C.c_int64),
        ("solve_seconds", C.c_double),
        ("setup_seconds", C.c_double),
        ("status", C.c_int32),
        ("kernel_launches", C.c_int64),
    ]

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if isinstance(v, C.Array) else v
        return out


class RpbaTrainOptionsC(C.Structure):
    _fields_ = [("steps", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float), ("probes", C.c_int32),
                ("max_samples", C.c_int32), ("seed", C.c_uint64)]


class RpbaTrainReportC(C.Structure):
    _fields_ = [("samples", C.c_int32), ("steps", C.c_int32), ("loss_initial", C.c_float),
                ("loss_final", C.c_float), ("systems", C.c_int32), ("err_initial", C.c_float),
                ("err_final", C.c_float)]


class RpbaPrecondSetC(C.Structure):
    _fields_ = [("rows", C.c_int32), ("systems", C.c_int32), ("probes", C.c_int32), ("nent", C.c_int32),
                ("nblocks", C.c_int32), ("features", _f32p), ("sinv", _f32p), ("b", _f32p), ("xs", _f32p),
                ("np", _i32p), ("sys", _i32p), ("rowoff", _i32p), ("ent_col", _i32p), ("ent_blk", _i32p),
                ("blocks", _f32p), ("sys_row", _i32p), ("uc", _f32p)]


class RpbaPrecondBuffersC(C.Structure):
    _fields_ = [("rows_cap", C.c_int32), ("ents_cap", C.c_int32), ("blocks_cap", C.c_int32),
                ("systems_cap", C.c_int32), ("rows", C.c_int32), ("systems", C.c_int32), ("probes", C.c_int32),
                ("nent", C.c_int32), ("nblocks", C.c_int32), ("features", _f32p), ("sinv", _f32p), ("b", _f32p),
                ("xs", _f32p), ("blocks", _f32p), ("uc", _f32p), ("np", _i32p), ("sys", _i32p),
                ("rowoff", _i32p), ("ent_col", _i32p), ("ent_blk", _i32p), ("sys_row", _i32p)]


class RpbaTriOptionsC(C.Structure):
    _fields_ = [("robustmode", C.c_int32), ("weight_only", C.c_int32), ("device", C.c_int32)]


class RpbaBatchReportC(C.Structure):
    _fields_ = [("seconds", C.c_double), ("scenes_per_second", C.c_double), ("tune_seconds", C.c_double),
                ("workers", C.c_int32), ("failed", C.c_int32)]


PRECOND_WEIGHTS = 1865
SOLVER_PCG, SOLVER_DIRECT, SOLVER_LEARNED = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1


def make_options(robust=True, exteval=False, threads=1, k2=True, k4=True, f=True,
                 solver=SOLVER_PCG, precision=PREC_FP64, max_lm_iterations=-1,
                 pcg_max_iterations=0, pcg_tolerance=0.0, device=0, verbose=0,
                 coarse_aggregates=0) -> RpbaOptionsC:
    return RpbaOptionsC(int(robust), int(exteval), int(threads), int(k2), int(k4), int(f),
                        int(solver), int(precision), int(max_lm_iterations),
                        int(pcg_max_iterations), float(pcg_tolerance), int(device), int(verbose),
                        int(coarse_aggregates))


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


@dataclass
class Block:
    """In-memory block (the state ``InputBlock`` produces, rpba.cpp:180-284)."""

    pmat: np.ndarray          # (n_images, 12) float32, row-major [R | t]
    K: np.ndarray             # (n_images, 9) float32
    distpara: np.ndarray      # (n_images, 2) float32
    XX: np.ndarray            # (n_points, 3) float32
    img_obs_off: np.ndarray   # (n_images+1,) int32
    xg: np.ndarray            # (n_slots, 2) float32 (negated image coordinates)
    wx: np.ndarray            # (n_slots,) float32
    wy: np.ndarray
    wxy: np.ndarray
    pt_obs_off: np.ndarray    # (n_points+1,) int32
    pt_obs_image: np.ndarray  # (n_track_obs,) int32
    pt_obs_slot: np.ndarray   # (n_track_obs,) int32
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_images(self) -> int:
        return int(self.pmat.shape[0])

    @property
    def n_points(self) -> int:
        return int(self.XX.shape[0])

    @property
    def n_obs(self) -> int:
        return int(self.pt_obs_off[-1])

    def copy(self) -> "Block":
        return Block(*(np.array(getattr(self, n), copy=True) for n in _ARRAYS))

    def as_c(self) -> RpbaBlockC:
        for n in _ARRAYS:
            a = getattr(self, n)
            if not a.flags.c_contiguous:
                setattr(self, n, np.ascontiguousarray(a))
        return RpbaBlockC(
            self.n_images, self.n_points,
            _p(self.pmat, _f32p), _p(self.K, _f32p), _p(self.distpara, _f32p),
            _p(self.XX, _f32p), _p(self.img_obs_off, _i32p), _p(self.xg, _f32p),
            _p(self.wx, _f32p), _p(self.wy, _f32p), _p(self.wxy, _f32p),
            _p(self.pt_obs_off, _i32p), _p(self.pt_obs_image, _i32p), _p(self.pt_obs_slot, _i32p))

    def tracks(self):
        """Yield (point, images, slots) per point."""
        for p in range(self.n_points):
            s, e = self.pt_obs_off[p], self.pt_obs_off[p + 1]
            yield p, self.pt_obs_image[s:e], self.pt_obs_slot[s:e]

    def track_slots(self) -> np.ndarray:
        """Global slot index (into xg / w*) of every track observation."""
        n = self.n_obs
        return self.img_obs_off[self.pt_obs_image[:n]] + self.pt_obs_slot[:n]

    @staticmethod
    def from_c(c: RpbaBlockC) -> "Block":
        """Copy a library-allocated block into numpy arrays."""
        ni, npt = c.n_images, c.n_points
        ns = c.img_obs_off[ni]
        nt = c.pt_obs_off[npt]

        def arr(ptr, n, dt):
            if n == 0:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True)

        return Block(arr(c.pmat, 12 * ni, np.float32).reshape(ni, 12),
                     arr(c.K, 9 * ni, np.float32).reshape(ni, 9),
                     arr(c.distpara, 2 * ni, np.float32).reshape(ni, 2),
                     arr(c.XX, 3 * npt, np.float32).reshape(npt, 3),
                     arr(c.img_obs_off, ni + 1, np.int32),
                     arr(c.xg, 2 * ns, np.float32).reshape(ns, 2),
                     arr(c.wx, ns, np.float32), arr(c.wy, ns, np.float32), arr(c.wxy, ns, np.float32),
                     arr(c.pt_obs_off, npt + 1, np.int32),
                     arr(c.pt_obs_image, nt, np.int32), arr(c.pt_obs_slot, nt, np.int32))


_ARRAYS = ("pmat", "K", "distpara", "XX", "img_obs_off", "xg", "wx", "wy", "wxy",
           "pt_obs_off", "pt_obs_image", "pt_obs_slot")
