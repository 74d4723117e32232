"""ctypes wrapper of the C++ oracle (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from rpba_b200.block import Block, RpbaBlockC, RpbaOptionsC, RpbaReportC, make_options

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.oracle_calc_plsa.argtypes = [C.POINTER(RpbaBlockC), C.POINTER(RpbaOptionsC), C.c_char_p,
                                       C.c_size_t, C.POINTER(RpbaReportC)]
        L.oracle_calc_plsa.restype = C.c_int32
        L.oracle_calc_plsa_variant.argtypes = [C.POINTER(RpbaBlockC), C.POINTER(RpbaOptionsC),
                                               C.c_char_p, C.c_size_t, C.POINTER(RpbaReportC),
                                               C.c_int32]
        L.oracle_calc_plsa_variant.restype = C.c_int32
        L.oracle_exteval.argtypes = [C.POINTER(RpbaBlockC), C.POINTER(RpbaOptionsC), dp,
                                     C.POINTER(RpbaReportC)]
        L.oracle_exteval.restype = C.c_int32
        L.oracle_cayley.argtypes = [C.c_double] * 3 + [dp]
        L.oracle_rectify3.argtypes = [dp]
        L.oracle_angleaxis_to_R.argtypes = [C.c_double] * 3 + [C.POINTER(C.c_float)]
        L.oracle_R_to_angleaxis.argtypes = [C.POINTER(C.c_float), dp]
        L.oracle_inv3.argtypes = [dp, dp]
        L.oracle_inv3.restype = C.c_double
        L.oracle_lu_inverse.argtypes = [C.c_int, dp, dp]
        L.oracle_lsa_create.argtypes = [C.POINTER(RpbaBlockC), C.POINTER(RpbaOptionsC)]
        L.oracle_lsa_create.restype = C.c_void_p
        L.oracle_lsa_destroy.argtypes = [C.c_void_p]
        for n in ("oracle_lsa_xm_size", "oracle_lsa_n_track_obs", "oracle_lsa_nrioff",
                  "oracle_lsa_normcamera"):
            getattr(L, n).argtypes = [C.c_void_p]
            getattr(L, n).restype = C.c_int32
        L.oracle_lsa_get_xm.argtypes = [C.c_void_p, dp]
        L.oracle_lsa_residuals.argtypes = [C.c_void_p, dp, dp]
        L.oracle_lsa_jacobian.argtypes = [C.c_void_p, C.c_int, dp, C.POINTER(C.c_int),
                                          C.POINTER(C.c_int), dp]
        L.oracle_input_block.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.POINTER(RpbaBlockC)]
        L.oracle_input_block.restype = C.c_int32
        L.oracle_block_free.argtypes = [C.POINTER(RpbaBlockC)]
        L.oracle_output_block.argtypes = [C.c_char_p, C.POINTER(RpbaBlockC), C.c_int32]
        L.oracle_output_block.restype = C.c_int32
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def calc_plsa(block: Block, opts: RpbaOptionsC | None = None, log_cap: int = 1 << 16):
    """Run the oracle's CalcPLSA on a copy of ``block``.

    Returns (status, adjusted block, report dict, log text)."""
    b = block.copy()
    cb = b.as_c()
    o = opts if opts is not None else make_options()
    rep = RpbaReportC()
    buf = C.create_string_buffer(log_cap)
    st = lib().oracle_calc_plsa(C.byref(cb), C.byref(o), buf, log_cap, C.byref(rep))
    return st, b, rep.as_dict(), buf.value.decode()


def calc_plsa_variant(block: Block, opts: RpbaOptionsC | None = None, variant: int = 1,
                      log_cap: int = 1 << 16):
    """calc_plsa with the SpMV blocks of each column visited in another
    order (1 reversed, 2 rotated by half, >= 3 a shuffle seeded by the
    variant): the same arithmetic up to summation order (a self-sensitivity
    probe)."""
    b = block.copy()
    cb = b.as_c()
    o = opts if opts is not None else make_options()
    rep = RpbaReportC()
    buf = C.create_string_buffer(log_cap)
    st = lib().oracle_calc_plsa_variant(C.byref(cb), C.byref(o), buf, log_cap, C.byref(rep), variant)
    return st, b, rep.as_dict(), buf.value.decode()


def exteval(block: Block, opts: RpbaOptionsC | None = None):
    o = opts if opts is not None else make_options()
    cb = block.as_c()
    res = np.zeros(2 * max(block.n_obs, 1))
    rep = RpbaReportC()
    lib().oracle_exteval(C.byref(cb), C.byref(o), _dp(res), C.byref(rep))
    return res[: 2 * block.n_obs].reshape(-1, 2), rep.as_dict()


def triangulate(block: Block, sig0w=None, robustmode: int = 0, weight_only: bool = False) -> dict:
    """CalcLSAXMulti for every point (the oracle's restatement)."""
    from rpba_b200 import lib as rlib
    L = lib()
    L.oracle_triangulate.restype = C.c_int32
    L.oracle_triangulate.argtypes = [C.POINTER(RpbaBlockC), C.POINTER(C.c_float), C.c_int32, C.c_int32,
                                     C.POINTER(C.c_double), C.POINTER(C.c_uint8), C.POINTER(C.c_float),
                                     C.POINTER(C.c_uint8), C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    return rlib.triangulate(block, sig0w, robustmode, weight_only, fn=L.oracle_triangulate)


def triangulate_parts(block: Block, part, nparts: int, sig0w=None, robustmode: int = 0,
                      weight_only: bool = False) -> dict:
    """CalcLSAXMulti with the camera partition ``part`` (image -> 0 ..
    nparts - 1): also the per-partition weight blocks ``w3d`` (n_points x
    nparts x 6: XX, YY, ZZ, XY, XZ, YZ) of the reference's wxyflag."""
    cb = block.as_c()
    nt, np_ = block.n_obs, block.n_points
    part = np.ascontiguousarray(part, np.int32)
    out = {"XX": np.zeros(3 * np_), "keep": np.zeros(nt, np.uint8), "sig0v": np.zeros(nt, np.float32),
           "conv": np.zeros(np_, np.uint8), "w3d": np.zeros(np_ * nparts * 6, np.float32)}
    s0, red = C.c_double(), C.c_int64()
    w = None if sig0w is None else np.ascontiguousarray(sig0w, np.float32)
    L = lib()
    f = L.oracle_triangulate_parts
    f.restype = C.c_int32
    f.argtypes = [C.POINTER(RpbaBlockC), C.POINTER(C.c_float), C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                  C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_uint8), C.POINTER(C.c_float),
                  C.POINTER(C.c_uint8), C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_float)]
    st = f(C.byref(cb), None if w is None else w.ctypes.data_as(C.POINTER(C.c_float)), int(robustmode),
           int(weight_only), part.ctypes.data_as(C.POINTER(C.c_int32)), int(nparts),
           out["XX"].ctypes.data_as(C.POINTER(C.c_double)), out["keep"].ctypes.data_as(C.POINTER(C.c_uint8)),
           out["sig0v"].ctypes.data_as(C.POINTER(C.c_float)), out["conv"].ctypes.data_as(C.POINTER(C.c_uint8)),
           C.byref(s0), C.byref(red), out["w3d"].ctypes.data_as(C.POINTER(C.c_float)))
    if st != 0:
        raise RuntimeError(f"oracle_triangulate_parts: status {st}")
    out["XX"] = out["XX"].reshape(np_, 3)
    out["w3d"] = out["w3d"].reshape(np_, nparts, 6)
    out["sig0io"], out["redundancy"] = s0.value, red.value
    return out


def lsa_gcp_step(block: Block, gcpinfo, W3, gcpdata, ncam_total: int, opts: RpbaOptionsC | None = None,
                 log_cap: int = 1 << 16):
    """One GCP-mode step of the LSA on ``block`` (modified in place): the
    parallel RPBA's per-partition call.  gcpinfo: per point, GCP index or
    -1; W3: (n_gcp_kept, 6) float weights; gcpdata: (n_gcp, 3) doubles."""
    cb = block.as_c()
    o = opts if opts is not None else make_options()
    gi = np.ascontiguousarray(gcpinfo, np.int32)
    w3 = np.ascontiguousarray(W3, np.float32).reshape(-1)
    gd = np.ascontiguousarray(gcpdata, np.float64).reshape(-1)
    buf = C.create_string_buffer(log_cap)
    f = lib().oracle_lsa_gcp_step
    f.restype = C.c_int32
    f.argtypes = [C.POINTER(RpbaBlockC), C.POINTER(RpbaOptionsC), C.POINTER(C.c_int32), C.POINTER(C.c_float),
                  C.POINTER(C.c_double), C.c_int32, C.c_char_p, C.c_size_t]
    st = f(C.byref(cb), C.byref(o), gi.ctypes.data_as(C.POINTER(C.c_int32)),
           w3.ctypes.data_as(C.POINTER(C.c_float)), gd.ctypes.data_as(C.POINTER(C.c_double)), int(ncam_total),
           buf, log_cap)
    return st, buf.value.decode()


def lsa_gcp_step_full(block: Block, gcpinfo, W3, gcpdata, ncam_total: int, pmat_d=None,
                      opts: RpbaOptionsC | None = None, log_cap: int = 1 << 16):
    """oracle_lsa_gcp_step_full on a copy of ``block``: the GCP-mode step
    with the cameras in double precision in and out.  Returns (status,
    block, cameras (n_images, 12), point_used, log)."""
    b = block.copy()
    cb = b.as_c()
    o = opts if opts is not None else make_options()
    gi = np.ascontiguousarray(gcpinfo, np.int32)
    w3 = np.ascontiguousarray(W3, np.float32).reshape(-1)
    gd = np.ascontiguousarray(gcpdata, np.float64).reshape(-1)
    pin = None if pmat_d is None else np.ascontiguousarray(pmat_d, np.float64).reshape(-1)
    pout = np.zeros((b.n_images, 12))
    used = np.zeros(max(b.n_points, 1), np.uint8)
    buf = C.create_string_buffer(log_cap)
    f = lib().oracle_lsa_gcp_step_full
    f.restype = C.c_int32
    f.argtypes = [C.POINTER(RpbaBlockC), C.POINTER(RpbaOptionsC), C.POINTER(C.c_int32), C.POINTER(C.c_float),
                  C.c_int32, C.POINTER(C.c_double), C.c_int32, C.c_int32, C.POINTER(C.c_double),
                  C.POINTER(C.c_double), C.POINTER(C.c_uint8), C.c_void_p, C.c_char_p, C.c_size_t]
    st = f(C.byref(cb), C.byref(o), gi.ctypes.data_as(C.POINTER(C.c_int32)), w3.ctypes.data_as(C.POINTER(C.c_float)),
           int(w3.size // 6), _dp(gd), int(gd.size // 3), int(ncam_total), None if pin is None else _dp(pin),
           _dp(pout), used.ctypes.data_as(C.POINTER(C.c_uint8)), None, buf, log_cap)
    return st, b, pout, used[:b.n_points].astype(bool), buf.value.decode()


def parallel_threads(n_images: int, threads: int) -> int:
    """Partition count of CalcPLSA (rpbacore.cpp:79-85): min(Threads,
    iround(images / 70)), iround rounding halves away from zero; the
    partitioned branch runs when it is above 1 and images > 5."""
    q = n_images / 70.0
    return int(min(threads, int(q + 0.5)))


def partition_images(block: Block, nparts: int) -> np.ndarray:
    """The camera partition that stands in for METIS (PartitionpointXXv,
    rpbacore.cpp:945-1037): the library's own bisection, compiled into this
    library (oracle_partition_images) so that the CPU baseline loads no GPU
    code.  Part (0 .. nparts - 1) of every image."""
    part = np.zeros(block.n_images, np.int32)
    cb = block.as_c()
    f = lib().oracle_partition_images
    f.restype = C.c_int32
    f.argtypes = [C.POINTER(RpbaBlockC), C.c_int32, C.POINTER(C.c_int32)]
    st = f(C.byref(cb), int(nparts), part.ctypes.data_as(C.POINTER(C.c_int32)))
    if st != 0:
        raise RuntimeError(f"oracle_partition_images: status {st}")
    return part


def calc_plsa_parallel(block: Block, part, nthreads: int, opts: RpbaOptionsC | None = None,
                       log_cap: int = 1 << 20):
    """The parallel RPBA (the partitioned branch of CalcPLSA,
    rpbacore.cpp:100-510) on a copy of ``block`` with the camera partition
    ``part`` (per image, 0 .. nthreads - 1).

    Returns (status, adjusted block, {"sig0opt", "iterations"}, log text);
    the block's tracks are the best iteration's (pointXXvold)."""
    b = block.copy()
    cb = b.as_c()
    o = opts if opts is not None else make_options()
    pt = np.ascontiguousarray(part, np.int32)
    assert pt.shape == (b.n_images,)
    stats = np.zeros(2)
    buf = C.create_string_buffer(log_cap)
    f = lib().oracle_calc_plsa_parallel
    f.restype = C.c_int32
    f.argtypes = [C.POINTER(RpbaBlockC), C.POINTER(RpbaOptionsC), C.c_int32, C.POINTER(C.c_int32), C.c_char_p,
                  C.c_size_t, C.POINTER(C.c_double)]
    st = f(C.byref(cb), C.byref(o), int(nthreads), pt.ctypes.data_as(C.POINTER(C.c_int32)), buf, log_cap,
           _dp(stats))
    # the track arrays were rewritten in place with fewer or equal entries
    n = int(b.pt_obs_off[-1])
    b.pt_obs_image = b.pt_obs_image[:n].copy()
    b.pt_obs_slot = b.pt_obs_slot[:n].copy()
    return st, b, {"sig0opt": float(stats[0]), "iterations": int(stats[1])}, buf.value.decode()


def input_block(path: str, k24out: bool = True) -> Block:
    cb = RpbaBlockC()
    st = lib().oracle_input_block(path.encode(), 3, int(k24out), C.byref(cb))
    if st != 0:
        raise IOError(f"oracle_input_block failed: {st}")
    b = Block.from_c(cb)
    lib().oracle_block_free(C.byref(cb))
    return b


def output_block(path: str, block: Block, k24out: bool = True) -> int:
    cb = block.as_c()
    return lib().oracle_output_block(path.encode(), C.byref(cb), int(k24out))


def cayley(a, b, c):
    R = np.zeros(9)
    lib().oracle_cayley(a, b, c, _dp(R))
    return R.reshape(3, 3)


def rectify3(R):
    R = np.ascontiguousarray(R, dtype=np.float64).copy()
    lib().oracle_rectify3(_dp(R))
    return R


def angleaxis_to_R(a, b, c):
    R = np.zeros(9, np.float32)
    lib().oracle_angleaxis_to_R(a, b, c, R.ctypes.data_as(C.POINTER(C.c_float)))
    return R.reshape(3, 3)


def R_to_angleaxis(R):
    R = np.ascontiguousarray(R, dtype=np.float32)
    out = np.zeros(3)
    lib().oracle_R_to_angleaxis(R.ctypes.data_as(C.POINTER(C.c_float)), _dp(out))
    return out


def inv3(m):
    m = np.ascontiguousarray(m, dtype=np.float64)
    out = np.zeros(9)
    det = lib().oracle_inv3(_dp(m), _dp(out))
    return out.reshape(3, 3), det


def lu_inverse(A):
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    out = np.zeros(n * n)
    lib().oracle_lu_inverse(n, _dp(A), _dp(out))
    return out.reshape(n, n)


class OracleLSA:
    """An LSA after the pass-0 set-up (weights, EncodeCameras, DecodeCameras):
    exposes the state vector, residuals and analytic Jacobians for
    finite-difference known-answer tests."""

    def __init__(self, block: Block, opts: RpbaOptionsC | None = None):
        self._block = block
        self._cb = block.as_c()
        self._o = opts if opts is not None else make_options()
        self.h = lib().oracle_lsa_create(C.byref(self._cb), C.byref(self._o))
        if not self.h:
            raise ValueError("degenerate block")

    def close(self):
        if self.h:
            lib().oracle_lsa_destroy(self.h)
            self.h = None

    __del__ = close

    @property
    def n_xm(self):
        return lib().oracle_lsa_xm_size(self.h)

    @property
    def n_obs(self):
        return lib().oracle_lsa_n_track_obs(self.h)

    @property
    def nrioff(self):
        return lib().oracle_lsa_nrioff(self.h)

    @property
    def normcamera(self):
        return lib().oracle_lsa_normcamera(self.h)

    def xm(self):
        out = np.zeros(self.n_xm)
        lib().oracle_lsa_get_xm(self.h, _dp(out))
        return out

    def residuals(self, xm):
        xm = np.ascontiguousarray(xm, dtype=np.float64)
        out = np.zeros(2 * self.n_obs)
        lib().oracle_lsa_residuals(self.h, _dp(xm), _dp(out))
        return out.reshape(-1, 2)

    def jacobian(self, tobs):
        Bc = np.zeros(18)
        Bp = np.zeros(6)
        nc = C.c_int()
        co = C.c_int()
        lib().oracle_lsa_jacobian(self.h, tobs, _dp(Bc), C.byref(nc), C.byref(co), _dp(Bp))
        return Bc.reshape(2, 9)[:, : nc.value], co.value, Bp.reshape(2, 3)
