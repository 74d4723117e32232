"""Error returns of the GPU solver against the oracle's (whose rules are
checked against the reference's on the CPU, test_oracle_errors.py): low
redundancy and an image without observations end with the same status and
log line; a NaN camera ends with the NaN-step status; a PCG cap that the
learned solver cannot meet falls back to the block-Jacobi PCG and the
direct solve and still reaches the plain solver's RMS."""

import numpy as np
import pytest

from rpba_b200 import scenes

pytestmark = pytest.mark.gpu


def _pair(oracle_mod, blk, **kw):
    import rpba_b200 as rb
    st_o, out_o, rep_o, log_o = oracle_mod.calc_plsa(blk, rb.make_options(**kw))
    b = blk.copy()
    st_g, log_g, rep_g = rb.CalcPLSA(b, **kw)
    return (st_o, out_o, log_o), (st_g, b, log_g)


def test_low_redundancy_status_and_line(oracle_mod):
    bal = scenes.arc_scene(seed=4, n_cams=6, n_pts=400, outlier_frac=0.0)
    blk = scenes.to_block(bal)
    n_keep = 24
    off = blk.pt_obs_off
    sel = np.concatenate([np.arange(off[p], off[p] + 2) for p in range(n_keep)])
    b = blk.copy()
    b.XX = blk.XX[:n_keep].copy()
    b.pt_obs_off = (np.arange(n_keep + 1) * 2).astype(np.int32)
    b.pt_obs_image = blk.pt_obs_image[sel].copy()
    b.pt_obs_slot = blk.pt_obs_slot[sel].copy()
    (st_o, _, log_o), (st_g, _, log_g) = _pair(oracle_mod, b)
    assert st_o == st_g == 4
    assert ("BA-Error: Low redundancy" in log_g) == ("BA-Error: Low redundancy" in log_o)


def test_nan_camera_status(oracle_mod):
    blk = scenes.to_block(scenes.arc_scene(seed=6, n_cams=8, n_pts=400))
    b = blk.copy()
    b.pmat[3, 5] = np.nan
    (st_o, out_o, _), (st_g, out_g, _) = _pair(oracle_mod, b)
    assert st_o == st_g == 5
    assert np.array_equal(out_g.XX, out_o.XX)


def test_pcg_cap_falls_back(oracle_mod):
    import rpba_b200 as rb
    from rpba_b200 import train_precond
    blk = scenes.to_block(scenes.arc_scene(seed=5, n_cams=50, n_pts=8000))
    S = rb.Solver(blk, solver=rb.SOLVER_LEARNED, precision=rb.PREC_MIXED, pcg_tolerance=1e-9, pcg_max_iterations=3)
    S.set_preconditioner(train_precond.load())
    st, rep = S.solve()
    S.close()
    P = rb.Solver(blk, solver=rb.SOLVER_DIRECT)
    _, rep_d = P.solve()
    P.close()
    assert st == 0 and rep["pcg_fallbacks"] > 0
    assert abs(rep["rms"] - rep_d["rms"]) <= 1e-4 * rep_d["rms"]


def test_pcg_barrier_wait_runs_out_and_handle_recovers():
    """A bounded wait that runs out: the persistent PCG's grid barriers are
    made to wait for a CTA that does not exist (test hook), with a 20 ms
    limit.  The kernel sets the error word and returns, the solve ends with
    the device-timeout status instead of hanging, and the same handle then
    solves normally, equal to a fresh handle."""
    import time
    import rpba_b200 as rb
    blk = scenes.to_block(scenes.arc_scene(seed=5, n_cams=20, n_pts=2000))
    S = rb.Solver(blk)
    S.debug_barrier_timeout(1, 20_000_000)
    t0 = time.perf_counter()
    with pytest.raises(rb.RpbaError) as e:
        S.solve()
    dt = time.perf_counter() - t0
    assert e.value.status == 6, e.value
    assert dt < 30.0, dt
    S.debug_barrier_timeout(0, 0)
    st, rep = S.solve()
    S.close()
    F = rb.Solver(blk)
    st_f, rep_f = F.solve()
    F.close()
    assert st == st_f == 0
    assert rep["cost"] == rep_f["cost"] and rep["linear_solves"] == rep_f["linear_solves"]
    print(f"timed-out solve returned after {dt * 1e3:.0f} ms")
