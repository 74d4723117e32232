"""ctypes binding of ``librpba_b200.so`` with the reference's entry points.

The names mirror RPBA's own functions (rpba.cpp / rpbacore.cpp):

* ``InputBlock(path, nraddpar, k24out)`` -- rpba.cpp:180-284
* ``OutputBlock(path, block, k24out)``   -- rpba.cpp:288-338
* ``CalcPLSA(block, ...)``               -- rpbacore.cpp:28-531; adjusts the
  block in place (cameras, points, track lists), returns (status, log, report)

plus ``Solver`` for the handle API (upload once, solve many times).

There is no CPU fallback: the library must be built (``__graft_entry__.build``
or ``make -C rpba_b200/csrc``) and a CUDA device must be present, otherwise
the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .block import (Block, RpbaBlockC, RpbaOptionsC, RpbaReportC, RpbaTrainOptionsC, RpbaTrainReportC,
                    RpbaPrecondSetC, RpbaPrecondBuffersC, RpbaBatchReportC, RpbaTriOptionsC,
                    make_options, PRECOND_WEIGHTS, SOLVER_PCG, SOLVER_DIRECT, SOLVER_LEARNED, PREC_FP64,
                    PREC_MIXED)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librpba_b200.so")

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "no observations in image",
          4: "low redundancy", 5: "NaN step", 6: "device timeout", 7: "I/O error",
          8: "unsupported input", 9: "no CUDA device", 10: "direct solve failed",
          11: "input too large for an allocation-free call", 12: "a collective between ranks failed"}

# Every entry point include/rpba_b200.h declares.
EXPORTS = ("rpba_status_string", "rpba_version", "rpba_input_block", "rpba_block_free",
           "rpba_output_block", "rpba_calc_plsa", "rpba_create", "rpba_solve",
           "rpba_get_state", "rpba_get_log", "rpba_exteval", "rpba_kernel_stats", "rpba_float_sequential_sum",
           "rpba_float_sequential_sum_noalloc", "rpba_train_preconditioner",
           "rpba_set_preconditioner", "rpba_precond_loss_grad", "rpba_record_systems", "rpba_solve_batch",
           "rpba_triangulate", "rpba_triangulate_parts", "rpba_partition_images", "rpba_lsa_gcp_step",
           "rpba_calc_plsa_parallel", "rpba_calc_plsa_parallel_hosted", "rpba_calc_plsa_parallel_ranks",
           "rpba_calc_plsa_parallel_ranks_hosted", "rpba_debug_barrier_timeout",
           "rpba_partition_count", "rpba_spd_inverse",
           "rpba_destroy")

_lib = None

# rpba_allgather_fn: (ctx, send, bytes, recv) -> 0 on success
AllgatherFn = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p)


def allgather_callback(gather, world: int) -> AllgatherFn:
    """An rpba_allgather_fn over a Python all-gather ``gather(data: bytes)
    -> bytes`` that returns every rank's bytes concatenated in rank order.
    A failure (an exception, or a result of the wrong length) returns 1 to
    the library, which ends the call with status 12 (keep the returned
    object alive for the call)."""

    def cb(ctx, send, n, recv):
        try:
            out = gather(C.string_at(send, n) if n else b"")
            if len(out) != world * n:
                return 1
            if out:
                C.memmove(recv, out, len(out))
            return 0
        except Exception:
            return 1

    return AllgatherFn(cb)


class RpbaError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        super().__init__(f"{what}: {STATUS.get(status, status)} ({status})")
        self.status = status


def load():
    """Load the library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    bp, op, rp = C.POINTER(RpbaBlockC), C.POINTER(RpbaOptionsC), C.POINTER(RpbaReportC)
    L.rpba_status_string.argtypes = [C.c_int32]
    L.rpba_status_string.restype = C.c_char_p
    L.rpba_version.restype = C.c_char_p
    L.rpba_input_block.argtypes = [C.c_char_p, C.c_int32, C.c_int32, bp]
    L.rpba_input_block.restype = C.c_int32
    L.rpba_block_free.argtypes = [bp]
    L.rpba_output_block.argtypes = [C.c_char_p, bp, C.c_int32]
    L.rpba_output_block.restype = C.c_int32
    L.rpba_calc_plsa.argtypes = [bp, op, C.c_char_p, C.c_size_t, rp]
    L.rpba_calc_plsa.restype = C.c_int32
    L.rpba_create.argtypes = [C.POINTER(C.c_void_p), bp, op]
    L.rpba_create.restype = C.c_int32
    L.rpba_solve.argtypes = [C.c_void_p, rp]
    L.rpba_solve.restype = C.c_int32
    L.rpba_get_state.argtypes = [C.c_void_p, bp]
    L.rpba_get_state.restype = C.c_int32
    L.rpba_get_log.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
    L.rpba_get_log.restype = C.c_int32
    L.rpba_exteval.argtypes = [C.c_void_p, C.POINTER(C.c_double), rp]
    L.rpba_exteval.restype = C.c_int32
    L.rpba_float_sequential_sum.argtypes = [C.POINTER(C.c_float), C.c_int64, C.c_int32,
                                            C.POINTER(C.c_float)]
    L.rpba_float_sequential_sum.restype = C.c_int32
    L.rpba_float_sequential_sum_noalloc.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    L.rpba_float_sequential_sum_noalloc.restype = C.c_int32
    fp = C.POINTER(C.c_float)
    L.rpba_train_preconditioner.argtypes = [bp, C.c_int32, op, C.POINTER(RpbaTrainOptionsC), fp,
                                            C.POINTER(RpbaTrainReportC)]
    L.rpba_train_preconditioner.restype = C.c_int32
    L.rpba_set_preconditioner.argtypes = [C.c_void_p, fp, C.c_int32]
    L.rpba_set_preconditioner.restype = C.c_int32
    L.rpba_precond_loss_grad.argtypes = [C.POINTER(RpbaPrecondSetC), fp, fp, fp]
    L.rpba_precond_loss_grad.restype = C.c_int32
    L.rpba_record_systems.argtypes = [bp, C.c_int32, op, C.POINTER(RpbaTrainOptionsC),
                                      C.POINTER(RpbaPrecondBuffersC)]
    L.rpba_record_systems.restype = C.c_int32
    L.rpba_solve_batch.argtypes = [bp, C.c_int32, op, C.c_int32, rp, C.POINTER(C.c_int32),
                                   C.POINTER(RpbaBatchReportC)]
    L.rpba_solve_batch.restype = C.c_int32
    L.rpba_triangulate_parts.argtypes = [bp, C.POINTER(C.c_float), C.POINTER(RpbaTriOptionsC),
                                         C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_double),
                                         C.POINTER(C.c_uint8), C.POINTER(C.c_float), C.POINTER(C.c_uint8),
                                         C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_float)]
    L.rpba_triangulate_parts.restype = C.c_int32
    L.rpba_partition_images.argtypes = [bp, C.c_int32, C.POINTER(C.c_int32)]
    L.rpba_partition_images.restype = C.c_int32
    L.rpba_lsa_gcp_step.argtypes = [bp, op, C.POINTER(C.c_int32), C.POINTER(C.c_float), C.c_int32,
                                    C.POINTER(C.c_double), C.c_int32, C.c_int32, C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.POINTER(C.c_uint8), rp, C.c_char_p, C.c_size_t]
    L.rpba_lsa_gcp_step.restype = C.c_int32
    L.rpba_calc_plsa_parallel.argtypes = [bp, op, C.c_int32, C.POINTER(C.c_int32), C.c_char_p, C.c_size_t,
                                          C.POINTER(C.c_double)]
    L.rpba_calc_plsa_parallel.restype = C.c_int32
    L.rpba_calc_plsa_parallel_hosted.argtypes = [bp, op, C.c_int32, C.POINTER(C.c_int32), C.c_char_p, C.c_size_t,
                                                 C.POINTER(C.c_double), C.c_void_p, C.c_void_p]
    L.rpba_calc_plsa_parallel_hosted.restype = C.c_int32
    L.rpba_calc_plsa_parallel_ranks.argtypes = [bp, op, C.c_int32, C.POINTER(C.c_int32), C.c_char_p, C.c_size_t,
                                                C.POINTER(C.c_double), C.c_int32, C.c_int32, AllgatherFn,
                                                C.c_void_p]
    L.rpba_calc_plsa_parallel_ranks.restype = C.c_int32
    L.rpba_calc_plsa_parallel_ranks_hosted.argtypes = [bp, op, C.c_int32, C.POINTER(C.c_int32), C.c_char_p,
                                                       C.c_size_t, C.POINTER(C.c_double), C.c_void_p, C.c_void_p,
                                                       C.c_int32, C.c_int32, AllgatherFn, C.c_void_p]
    L.rpba_calc_plsa_parallel_ranks_hosted.restype = C.c_int32
    L.rpba_triangulate.argtypes = [bp, C.POINTER(C.c_float), C.POINTER(RpbaTriOptionsC), C.POINTER(C.c_double),
                                   C.POINTER(C.c_uint8), C.POINTER(C.c_float), C.POINTER(C.c_uint8),
                                   C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    L.rpba_triangulate.restype = C.c_int32
    L.rpba_kernel_stats.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t]
    L.rpba_kernel_stats.restype = C.c_int32
    L.rpba_spd_inverse.argtypes = [C.POINTER(C.c_double), C.c_int32, C.POINTER(C.c_double), C.c_int32]
    L.rpba_spd_inverse.restype = C.c_int32
    L.rpba_partition_count.argtypes = [C.c_int32, C.c_int32, C.c_int32]
    L.rpba_partition_count.restype = C.c_int32
    L.rpba_debug_barrier_timeout.argtypes = [C.c_void_p, C.c_int32, C.c_int64]
    L.rpba_debug_barrier_timeout.restype = C.c_int32
    L.rpba_destroy.argtypes = [C.c_void_p]
    _lib = L
    return L


def InputBlock(path: str, nraddpar: int = 3, k24out: bool = True) -> Block:
    L = load()
    cb = RpbaBlockC()
    st = L.rpba_input_block(path.encode(), int(nraddpar), int(k24out), C.byref(cb))
    if st != 0:
        raise RpbaError(st, f"InputBlock({path})")
    b = Block.from_c(cb)
    L.rpba_block_free(C.byref(cb))
    return b


def OutputBlock(path: str, block: Block, k24out: bool = True) -> None:
    cb = block.as_c()
    st = load().rpba_output_block(path.encode(), C.byref(cb), int(k24out))
    if st != 0:
        raise RpbaError(st, f"OutputBlock({path})")


def CalcPLSA(block: Block, robust: bool = True, addflags=(True, True, True), threads: int = 1,
             exteval: bool = False, solver: int = SOLVER_PCG, precision: int = PREC_FP64,
             max_lm_iterations: int = -1, device: int = 0, log_cap: int = 1 << 20):
    """Adjust ``block`` in place on the GPU (or evaluate it, ``exteval``).

    Returns (status, log text, report dict).  Like the reference, the
    adjusted state is written back on the error returns that keep a stored
    state (no observations in an image, low redundancy, NaN step)."""
    o = make_options(robust=robust, exteval=exteval, threads=threads, k2=addflags[0],
                     k4=addflags[1], f=addflags[2], solver=solver, precision=precision,
                     max_lm_iterations=max_lm_iterations, device=device)
    cb = block.as_c()
    rep = RpbaReportC()
    buf = C.create_string_buffer(log_cap)
    st = load().rpba_calc_plsa(C.byref(cb), C.byref(o), buf, log_cap, C.byref(rep))
    if st in (2, 9):
        raise RpbaError(st, "CalcPLSA")
    return st, buf.value.decode(), rep.as_dict()


def lsa_gcp_step(block: Block, gcpinfo, W3, gcpdata, ncam_total: int, pmat_d=None, solver: int = SOLVER_PCG,
                 addflags=(True, True, True), device: int = 0, log_cap: int = 1 << 16):
    """One GCP-mode LSA step on a copy of ``block`` (rpba_lsa_gcp_step, the
    parallel RPBA's per-partition call).  gcpinfo: per point its GCP index
    or -1; W3: (rows, 6) weight blocks in the order of the kept GCP points;
    gcpdata: (n_gcp, 3).  Returns (status, block, cameras in double
    precision (n_images, 12), point_used, report, log)."""
    b = block.copy()
    cb = b.as_c()
    o = make_options(robust=False, k2=addflags[0], k4=addflags[1], f=addflags[2], solver=solver,
                     precision=PREC_FP64, device=device)
    gi = np.ascontiguousarray(gcpinfo, np.int32)
    w3 = np.ascontiguousarray(W3, np.float32).reshape(-1)
    gd = np.ascontiguousarray(gcpdata, np.float64).reshape(-1)
    pin = None if pmat_d is None else np.ascontiguousarray(pmat_d, np.float64).reshape(-1)
    pout = np.zeros((b.n_images, 12))
    used = np.zeros(max(b.n_points, 1), np.uint8)
    rep = RpbaReportC()
    buf = C.create_string_buffer(log_cap)
    dp = lambda a: None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))
    st = load().rpba_lsa_gcp_step(C.byref(cb), C.byref(o), gi.ctypes.data_as(C.POINTER(C.c_int32)),
                                  w3.ctypes.data_as(C.POINTER(C.c_float)), int(w3.size // 6), dp(gd),
                                  int(gd.size // 3), int(ncam_total), dp(pin), dp(pout),
                                  used.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(rep), buf, log_cap)
    return st, b, pout, used[:b.n_points].astype(bool), rep.as_dict(), buf.value.decode()


def calc_plsa_parallel(block: Block, part, nthreads: int, robust: bool = True, addflags=(True, True, True),
                       solver: int = SOLVER_PCG, device: int = 0, log_cap: int = 1 << 20):
    """The parallel RPBA (rpba_calc_plsa_parallel) on a copy of ``block``
    with the camera partition ``part``.  Returns (status, adjusted block,
    {"sig0opt", "iterations"}, log); the block's tracks are the best
    iteration's, trimmed to their length."""
    b = block.copy()
    cb = b.as_c()
    o = make_options(robust=robust, k2=addflags[0], k4=addflags[1], f=addflags[2], solver=solver,
                     precision=PREC_FP64, device=device)
    pt = np.ascontiguousarray(part, np.int32)
    stats = np.zeros(2)
    buf = C.create_string_buffer(log_cap)
    st = load().rpba_calc_plsa_parallel(C.byref(cb), C.byref(o), int(nthreads),
                                        pt.ctypes.data_as(C.POINTER(C.c_int32)), buf, log_cap,
                                        stats.ctypes.data_as(C.POINTER(C.c_double)))
    n = int(b.pt_obs_off[-1])
    b.pt_obs_image = b.pt_obs_image[:n].copy()
    b.pt_obs_slot = b.pt_obs_slot[:n].copy()
    return st, b, {"sig0opt": float(stats[0]), "iterations": int(stats[1])}, buf.value.decode()


def calc_plsa_parallel_ranks(block: Block, part, nthreads: int, rank: int, world: int, gather,
                             robust: bool = True, addflags=(True, True, True), solver: int = SOLVER_PCG,
                             device: int = 0, log_cap: int = 1 << 20, steps=None):
    """The parallel RPBA over ranks (rpba_calc_plsa_parallel_ranks) on a copy
    of ``block``: this rank runs its partitions' steps on ``device``;
    ``gather(data: bytes) -> bytes`` is the all-gather between the ranks
    (``replicas.bytes_allgather`` over torch.distributed).  ``steps``:
    (step, merge) C function pointers to run the hosted form instead (the
    host-side check binds the oracle's).  Returns what calc_plsa_parallel
    returns; every rank gets the same."""
    b = block.copy()
    cb = b.as_c()
    o = make_options(robust=robust, k2=addflags[0], k4=addflags[1], f=addflags[2], solver=solver,
                     precision=PREC_FP64, device=device)
    pt = np.ascontiguousarray(part, np.int32)
    stats = np.zeros(2)
    buf = C.create_string_buffer(log_cap)
    ag = allgather_callback(gather, world)
    args = (C.byref(cb), C.byref(o), int(nthreads), pt.ctypes.data_as(C.POINTER(C.c_int32)), buf, log_cap,
            stats.ctypes.data_as(C.POINTER(C.c_double)))
    if steps is None:
        st = load().rpba_calc_plsa_parallel_ranks(*args, int(rank), int(world), ag, None)
    else:
        st = load().rpba_calc_plsa_parallel_ranks_hosted(*args, steps[0], steps[1], int(rank), int(world), ag, None)
    n = int(b.pt_obs_off[-1])
    b.pt_obs_image = b.pt_obs_image[:n].copy()
    b.pt_obs_slot = b.pt_obs_slot[:n].copy()
    return st, b, {"sig0opt": float(stats[0]), "iterations": int(stats[1])}, buf.value.decode()


def float_sequential_sum(v, device: int = 0) -> np.float32:
    """Left-to-right float32 sum of ``v`` (values finite, >= 0) on the GPU,
    bitwise equal to the sequential loop."""
    a = np.ascontiguousarray(v, dtype=np.float32)
    out = C.c_float()
    st = load().rpba_float_sequential_sum(a.ctypes.data_as(C.POINTER(C.c_float)), a.size, device,
                                          C.byref(out))
    if st != 0:
        raise RpbaError(st, "rpba_float_sequential_sum")
    return np.float32(out.value)


def train_preconditioner(blocks, steps=300, batch=0, lr=3e-3, probes=2, seed=1, max_samples=0,
                         **opt_kw):
    """Train the learned block-Jacobi correction on the direct solver's own
    systems for ``blocks``; returns (weights float32[1865], report dict)."""
    arr = (RpbaBlockC * len(blocks))(*[b.as_c() for b in blocks])
    o = make_options(**opt_kw)
    t = RpbaTrainOptionsC(int(steps), int(batch), float(lr), int(probes), int(max_samples), int(seed))
    w = np.zeros(PRECOND_WEIGHTS, np.float32)
    rep = RpbaTrainReportC()
    st = load().rpba_train_preconditioner(arr, len(blocks), C.byref(o), C.byref(t),
                                          w.ctypes.data_as(C.POINTER(C.c_float)), C.byref(rep))
    if st != 0:
        raise RpbaError(st, "rpba_train_preconditioner")
    return w, {k: getattr(rep, k) for k, _ in rep._fields_}


def spd_inverse(A, device: int = 0) -> np.ndarray:
    """A^-1 of a dense SPD matrix by the library's tiled FP64 tensor-core
    Cholesky and inverse (rpba_spd_inverse)."""
    A = np.ascontiguousarray(A, np.float64)
    n = A.shape[0]
    out = np.zeros_like(A)
    st = load().rpba_spd_inverse(A.ctypes.data_as(C.POINTER(C.c_double)), n,
                                 out.ctypes.data_as(C.POINTER(C.c_double)), device)
    if st != 0:
        raise RpbaError(st, "rpba_spd_inverse")
    return out


def partition_images(block: Block, nparts: int) -> np.ndarray:
    """Part (0 .. nparts - 1) of every image: the camera partition of the
    reference's parallel RPBA (PartitionpointXXv, rpbacore.cpp:945-1037),
    contiguous parts of the covisibility graph.  Host code, no GPU."""
    part = np.zeros(block.n_images, np.int32)
    cb = block.as_c()
    st = load().rpba_partition_images(C.byref(cb), int(nparts), part.ctypes.data_as(C.POINTER(C.c_int32)))
    if st != 0:
        raise RpbaError(st, "rpba_partition_images")
    return part


def triangulate(block: Block, sig0w=None, robustmode: int = 0, weight_only: bool = False, device: int = 0,
                fn=None) -> dict:
    """Per-point refinement of every point against the block's fixed cameras
    (rpba_triangulate; ``fn`` substitutes another implementation with the
    same C signature, e.g. the oracle's)."""
    cb = block.as_c()
    nt, np_ = block.n_obs, block.n_points
    out = {"XX": np.zeros(3 * np_), "keep": np.zeros(nt, np.uint8), "sig0v": np.zeros(nt, np.float32),
           "conv": np.zeros(np_, np.uint8)}
    s0, red = C.c_double(), C.c_int64()
    w = None if sig0w is None else np.ascontiguousarray(sig0w, np.float32)
    wp = None if w is None else w.ctypes.data_as(C.POINTER(C.c_float))
    args = (C.byref(cb), wp)
    tail = (out["XX"].ctypes.data_as(C.POINTER(C.c_double)), out["keep"].ctypes.data_as(C.POINTER(C.c_uint8)),
            out["sig0v"].ctypes.data_as(C.POINTER(C.c_float)), out["conv"].ctypes.data_as(C.POINTER(C.c_uint8)),
            C.byref(s0), C.byref(red))
    if fn is None:
        o = RpbaTriOptionsC(int(robustmode), int(weight_only), int(device))
        st = load().rpba_triangulate(*args, C.byref(o), *tail)
    else:
        st = fn(*args, int(robustmode), int(weight_only), *tail)
    if st != 0:
        raise RpbaError(st, "rpba_triangulate")
    out["XX"] = out["XX"].reshape(np_, 3)
    out["sig0io"], out["redundancy"] = s0.value, red.value
    return out


def triangulate_parts(block: Block, part, nparts: int, sig0w=None, robustmode: int = 0,
                      weight_only: bool = False, device: int = 0) -> dict:
    """rpba_triangulate with the camera partition ``part`` (image -> 0 ..
    nparts - 1): also the per-partition weight blocks ``w3d`` (n_points x
    nparts x 6: XX, YY, ZZ, XY, XZ, YZ)."""
    cb = block.as_c()
    nt, np_ = block.n_obs, block.n_points
    part = np.ascontiguousarray(part, np.int32)
    out = {"XX": np.zeros(3 * np_), "keep": np.zeros(nt, np.uint8), "sig0v": np.zeros(nt, np.float32),
           "conv": np.zeros(np_, np.uint8), "w3d": np.zeros(np_ * nparts * 6, np.float32)}
    s0, red = C.c_double(), C.c_int64()
    w = None if sig0w is None else np.ascontiguousarray(sig0w, np.float32)
    o = RpbaTriOptionsC(int(robustmode), int(weight_only), int(device))
    st = load().rpba_triangulate_parts(
        C.byref(cb), None if w is None else w.ctypes.data_as(C.POINTER(C.c_float)), C.byref(o),
        part.ctypes.data_as(C.POINTER(C.c_int32)), int(nparts), out["XX"].ctypes.data_as(C.POINTER(C.c_double)),
        out["keep"].ctypes.data_as(C.POINTER(C.c_uint8)), out["sig0v"].ctypes.data_as(C.POINTER(C.c_float)),
        out["conv"].ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(s0), C.byref(red),
        out["w3d"].ctypes.data_as(C.POINTER(C.c_float)))
    if st != 0:
        raise RpbaError(st, "rpba_triangulate_parts")
    out["XX"] = out["XX"].reshape(np_, 3)
    out["w3d"] = out["w3d"].reshape(np_, nparts, 6)
    out["sig0io"], out["redundancy"] = s0.value, red.value
    return out


def solve_batch(blocks, workers: int = 0, **opt_kw):
    """Solve many independent scenes in place, several at once on one GPU
    (rpba_solve_batch; workers <= 0: chosen by the library).  Returns
    (status list, report dicts, batch report dict)."""
    n = len(blocks)
    cbs = [b.as_c() for b in blocks]
    arr = (RpbaBlockC * n)(*cbs)
    o = make_options(**opt_kw)
    reps = (RpbaReportC * n)()
    st = (C.c_int32 * n)()
    br = RpbaBatchReportC()
    r = load().rpba_solve_batch(arr, n, C.byref(o), int(workers), reps, st, C.byref(br))
    if r not in (0, 10):
        raise RpbaError(r, "rpba_solve_batch")
    # the results went straight into the blocks' arrays (as with CalcPLSA);
    # cbs keeps the C views alive until here
    del cbs
    return list(st), [rp.as_dict() for rp in reps], {k: getattr(br, k) for k, _ in br._fields_}


def record_systems(blocks, probes=2, seed=1, max_samples=0, caps=None, **opt_kw) -> dict:
    """The training set the GPU records for ``blocks`` (the direct solver's
    own systems, diagonally scaled), as a dict of numpy arrays laid out as
    ``precond_loss_grad`` takes them."""
    arr = (RpbaBlockC * len(blocks))(*[b.as_c() for b in blocks])
    o = make_options(**opt_kw)
    t = RpbaTrainOptionsC(0, 0, 0.0, int(probes), int(max_samples), int(seed))
    rows_cap, ents_cap, blocks_cap, sys_cap = caps or (0, 0, 0, 0)
    for attempt in range(2):
        P = 1 + max(0, int(probes))
        arrs = {"features": np.zeros((rows_cap, 19), np.float32), "sinv": np.zeros((rows_cap, 81), np.float32),
                "b": np.zeros((P, rows_cap, 9), np.float32), "xs": np.zeros((rows_cap, 9), np.float32),
                "blocks": np.zeros((blocks_cap, 81), np.float32), "uc": np.zeros((P, rows_cap, 9), np.float32),
                "np": np.zeros(rows_cap, np.int32), "sys": np.zeros(rows_cap, np.int32),
                "rowoff": np.zeros(rows_cap + 1, np.int32), "ent_col": np.zeros(ents_cap, np.int32),
                "ent_blk": np.zeros(ents_cap, np.int32), "sys_row": np.zeros(sys_cap + 1, np.int32)}
        fp = lambda k: arrs[k].ctypes.data_as(C.POINTER(C.c_float))
        ip = lambda k: arrs[k].ctypes.data_as(C.POINTER(C.c_int32))
        buf = RpbaPrecondBuffersC(rows_cap, ents_cap, blocks_cap, sys_cap, 0, 0, 0, 0, 0,
                                  fp("features"), fp("sinv"), fp("b"), fp("xs"), fp("blocks"), fp("uc"),
                                  ip("np"), ip("sys"), ip("rowoff"), ip("ent_col"), ip("ent_blk"), ip("sys_row"))
        st = load().rpba_record_systems(arr, len(blocks), C.byref(o), C.byref(t), C.byref(buf))
        if st == 11 and attempt == 0:  # too large: retry with the reported sizes
            rows_cap, ents_cap, blocks_cap, sys_cap = buf.rows, buf.nent, buf.nblocks, buf.systems
            continue
        if st != 0:
            raise RpbaError(st, "rpba_record_systems")
        break
    R, S = buf.rows, buf.systems
    out = {"rows": R, "systems": S, "probes": buf.probes,
           "features": arrs["features"][:R], "sinv": arrs["sinv"][:R], "b": arrs["b"][:, :R],
           "xs": arrs["xs"][:R], "blocks": arrs["blocks"][:buf.nblocks], "uc": arrs["uc"][:, :R],
           "np": arrs["np"][:R], "sys": arrs["sys"][:R], "rowoff": arrs["rowoff"][:R + 1],
           "ent_col": arrs["ent_col"][:buf.nent], "ent_blk": arrs["ent_blk"][:buf.nent],
           "sys_row": arrs["sys_row"][:S + 1]}
    return out


def precond_loss_grad(ts: dict, weights):
    """Training loss and gradient for a host training set (dict of numpy
    arrays laid out as rpba_precond_set), computed by the GPU kernels."""
    f32 = lambda k: np.ascontiguousarray(ts[k], np.float32)
    i32 = lambda k: np.ascontiguousarray(ts[k], np.int32)
    keep = {k: f32(k) for k in ("features", "sinv", "b", "xs", "blocks")}
    keep.update({k: i32(k) for k in ("np", "sys", "rowoff", "ent_col", "ent_blk", "sys_row")})
    if ts.get("uc") is not None:
        keep["uc"] = f32("uc")
    fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int32)
    st = RpbaPrecondSetC(int(ts["rows"]), int(ts["systems"]), int(ts["probes"]), int(keep["ent_col"].size),
                         int(keep["blocks"].shape[0]),
                         *(keep[k].ctypes.data_as(fp) for k in ("features", "sinv", "b", "xs")),
                         *(keep[k].ctypes.data_as(ip) for k in ("np", "sys", "rowoff", "ent_col", "ent_blk")),
                         keep["blocks"].ctypes.data_as(fp), keep["sys_row"].ctypes.data_as(ip),
                         keep["uc"].ctypes.data_as(fp) if "uc" in keep else None)
    w = np.ascontiguousarray(weights, np.float32)
    loss = C.c_float()
    g = np.zeros(PRECOND_WEIGHTS, np.float32)
    r = load().rpba_precond_loss_grad(C.byref(st), w.ctypes.data_as(fp), C.byref(loss), g.ctypes.data_as(fp))
    if r != 0:
        raise RpbaError(r, "rpba_precond_loss_grad")
    return loss.value, g


class Solver:
    """Handle API: the block is uploaded once; ``solve`` restarts from it."""

    def __init__(self, block: Block, **kw):
        self.block = block
        self.opts = make_options(**kw)
        self._cb = block.as_c()
        self.h = C.c_void_p()
        st = load().rpba_create(C.byref(self.h), C.byref(self._cb), C.byref(self.opts))
        if st != 0:
            self.h = None
            raise RpbaError(st, "rpba_create")

    def solve(self) -> tuple[int, dict]:
        rep = RpbaReportC()
        st = load().rpba_solve(self.h, C.byref(rep))
        if st in (2, 6, 9):
            raise RpbaError(st, "rpba_solve")
        return st, rep.as_dict()

    def log(self, cap: int = 1 << 20) -> str:
        buf = C.create_string_buffer(cap)
        load().rpba_get_log(self.h, buf, cap)
        return buf.value.decode()

    def state(self, out: Block | None = None) -> Block:
        """The adjusted block: new cameras, points and tracks (the
        observation arrays xg, wx, wy, wxy and img_obs_off, which a solve
        does not change, are shared with the input block).  The track
        arrays keep the input's length; entries past pt_obs_off[-1] are 0.
        ``out``: a block of the input's shape whose pmat, K, distpara, XX and
        track arrays receive the result (for example arrays in page-locked
        memory, reused from call to call); it is returned."""
        b = self.block
        if out is None:
            out = Block(np.empty_like(b.pmat), np.empty_like(b.K), np.empty_like(b.distpara), np.empty_like(b.XX),
                        b.img_obs_off, b.xg, b.wx, b.wy, b.wxy, np.empty_like(b.pt_obs_off),
                        np.zeros_like(b.pt_obs_image), np.zeros_like(b.pt_obs_slot))
        else:
            for name in ("pmat", "K", "distpara", "XX", "pt_obs_off", "pt_obs_image", "pt_obs_slot"):
                a, ref = getattr(out, name), getattr(b, name)
                if a.shape != ref.shape or a.dtype != ref.dtype or not a.flags.c_contiguous or not a.flags.writeable:
                    raise ValueError(f"state(out=...): {name} must be a writable C-contiguous {ref.dtype} "
                                     f"array of shape {ref.shape}")
        cb = out.as_c()
        st = load().rpba_get_state(self.h, C.byref(cb))
        if st != 0:
            raise RpbaError(st, "rpba_get_state")
        return out

    def exteval(self):
        n = self.block.n_obs
        res = np.zeros(2 * max(n, 1))
        rep = RpbaReportC()
        st = load().rpba_exteval(self.h, res.ctypes.data_as(C.POINTER(C.c_double)), C.byref(rep))
        if st != 0:
            raise RpbaError(st, "rpba_exteval")
        return res[: 2 * n].reshape(-1, 2), rep.as_dict()

    def set_preconditioner(self, weights):
        """Weights for RPBA_SOLVER_LEARNED solves (None: plain block-Jacobi)."""
        if weights is None:
            st = load().rpba_set_preconditioner(self.h, None, 0)
        else:
            self._w = np.ascontiguousarray(weights, np.float32)
            st = load().rpba_set_preconditioner(self.h, self._w.ctypes.data_as(C.POINTER(C.c_float)),
                                                self._w.size)
        if st != 0:
            raise RpbaError(st, "rpba_set_preconditioner")

    def kernel_stats(self) -> dict:
        """Per-kernel device time of the last solve (needs verbose=2)."""
        import json
        buf = C.create_string_buffer(1 << 16)
        load().rpba_kernel_stats(self.h, buf, 1 << 16)
        return json.loads(buf.value.decode())

    def debug_barrier_timeout(self, extra_ctas: int, timeout_ns: int):
        """Test hook: the PCG's grid barriers wait for `extra_ctas` CTAs that
        do not exist, for at most `timeout_ns`; (0, 0) restores them."""
        st = load().rpba_debug_barrier_timeout(self.h, int(extra_ctas), int(timeout_ns))
        if st != 0:
            raise RpbaError(st, "rpba_debug_barrier_timeout")

    def close(self):
        if self.h:
            load().rpba_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
