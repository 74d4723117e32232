"""The library's parallel RPBA loop (rpba_calc_plsa_parallel: host code in
parallel.cu around two device steps) checked without a GPU.
rpba_calc_plsa_parallel_hosted runs the same loop with its two steps bound
to the oracle's restatements of them (oracle_lsa_gcp_step_full: the
partition's GCP-mode LSA step; oracle_merge: CalcLSAXMulti over every point
with the weight blocks); the result must equal the oracle's own loop
(oracle_calc_plsa_parallel, rpbacore.cpp:100-510) bit for bit: cameras,
points, intrinsics, tracks, sigma0, iteration count and log.  The device
steps themselves are checked against the oracle on a GPU."""
import ctypes as C

import numpy as np
import pytest


def _hosted(oracle_mod, blk, part, k, **opts):
    import rpba_b200 as rb
    L, O = rb.load(), oracle_mod.lib()
    b = blk.copy()
    cb = b.as_c()
    o = rb.make_options(**opts)
    stats = np.zeros(2)
    cap = 1 << 20
    buf = C.create_string_buffer(cap)
    pt = np.ascontiguousarray(part, np.int32)
    st = L.rpba_calc_plsa_parallel_hosted(C.byref(cb), C.byref(o), int(k), pt.ctypes.data_as(C.POINTER(C.c_int32)),
                                          buf, cap, stats.ctypes.data_as(C.POINTER(C.c_double)),
                                          C.cast(O.oracle_lsa_gcp_step_full, C.c_void_p),
                                          C.cast(O.oracle_merge, C.c_void_p))
    n = int(b.pt_obs_off[-1])
    b.pt_obs_image = b.pt_obs_image[:n].copy()
    b.pt_obs_slot = b.pt_obs_slot[:n].copy()
    return st, b, {"sig0opt": float(stats[0]), "iterations": int(stats[1])}, buf.value.decode()


@pytest.fixture(scope="module")
def loop_scenes():
    from rpba_b200 import scenes
    return {
        "arc": scenes.to_block(scenes.arc_scene(seed=5, n_cams=50, n_pts=8000)),
        "city": scenes.to_block(scenes.city_scene(seed=8, n_clusters=3, cams_per_cluster=20, n_pts=8000)),
        "street": scenes.to_block(scenes.street_scene(seed=6, n_cams=80, n_pts=12000)),
    }


CASES = [("arc", 2, {}), ("arc", 4, {}), ("city", 3, {}), ("street", 2, {}),
         ("arc", 3, {"robust": False}), ("city", 2, {"k2": False, "k4": False, "f": False})]


@pytest.mark.parametrize("name,k,opts", CASES)
def test_library_loop_equals_oracle_loop(oracle_mod, loop_scenes, name, k, opts):
    import rpba_b200 as rb
    blk = loop_scenes[name]
    part = rb.partition_images(blk, k)
    st_o, b_o, s_o, log_o = oracle_mod.calc_plsa_parallel(blk, part, k, rb.make_options(**opts))
    st_h, b_h, s_h, log_h = _hosted(oracle_mod, blk, part, k, **opts)
    print(f"{name} k={k} {opts}: {s_h['iterations']} iterations, sigma0 {s_h['sig0opt']:.6f}, "
          f"{b_h.n_obs} of {blk.n_obs} observations")
    assert st_o == st_h == 0
    assert s_h == s_o
    for n in ("pmat", "K", "distpara", "XX", "pt_obs_off", "pt_obs_image", "pt_obs_slot"):
        assert np.array_equal(getattr(b_h, n), getattr(b_o, n)), n
    assert log_h == log_o


def test_library_loop_rejects_bad_arguments(oracle_mod, loop_scenes):
    import rpba_b200 as rb
    blk = loop_scenes["arc"]
    n = blk.n_images
    good = ((np.arange(n) * 2) // n).astype(np.int32)
    assert _hosted(oracle_mod, blk, good, 1)[0] == 1
    assert _hosted(oracle_mod, blk, np.where(good == 1, 2, 0), 2)[0] == 1
    assert _hosted(oracle_mod, blk, np.zeros(n, np.int32), 2)[0] == 1
    cb = blk.copy().as_c()
    o = rb.make_options(precision=rb.PREC_MIXED)
    st = rb.load().rpba_calc_plsa_parallel(C.byref(cb), C.byref(o), 2, good.ctypes.data_as(C.POINTER(C.c_int32)),
                                           None, 0, None)
    assert st == 8  # RPBA_ERR_UNSUPPORTED: the partition steps are FP64 only


def test_gcp_step_rejects_bad_arguments(loop_scenes):
    """rpba_lsa_gcp_step checks its arguments before touching a device."""
    import rpba_b200 as rb
    blk = loop_scenes["arc"]
    n = blk.n_points
    gi = np.full(n, -1, np.int32)
    W3 = np.zeros((0, 6), np.float32)
    gd = np.zeros((0, 3))
    st = rb.lsa_gcp_step(blk, gi, W3, gd, blk.n_images - 1)[0]
    assert st == 1  # ncam_total below the block's image count
    L = rb.load()
    b = blk.copy()
    cb = b.as_c()
    for o, want in ((rb.make_options(precision=rb.PREC_MIXED), 8), (rb.make_options(solver=rb.SOLVER_LEARNED), 8),
                    (rb.make_options(exteval=True), 8)):
        st = L.rpba_lsa_gcp_step(C.byref(cb), C.byref(o), gi.ctypes.data_as(C.POINTER(C.c_int32)), None, 0, None,
                                 0, blk.n_images, None, None, None, None, None, 0)
        assert st == want
    o = rb.make_options()
    st = L.rpba_lsa_gcp_step(C.byref(cb), C.byref(o), None, None, 0, None, 0, blk.n_images, None, None, None, None,
                             None, 0)
    assert st == 1  # no gcpinfo
