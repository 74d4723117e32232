"""The parallel RPBA on the GPU against the oracle.

rpba_lsa_gcp_step (the GCP-mode LSA step: every camera free, shared points
held by 3-D priors, one damped step) against oracle_lsa_gcp_step_full, and
rpba_calc_plsa_parallel (the whole loop, rpbacore.cpp:100-510) against
oracle_calc_plsa_parallel.  The loop's host logic is checked bit for bit
without a GPU (test_cpu_parallel_loop.py); here the device steps.  Both
sides solve the partition systems with the dense direct solver, so the
bars are roundoff-level: cameras within 1e-9 (scaled), the same points
taken, the same log integers; the loop's iteration count equal and its
final Exteval sigma0 within 1e-6 relative."""
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solved(oracle_mod):
    import rpba_b200 as rb
    from rpba_b200 import scenes
    blk = scenes.to_block(scenes.arc_scene(seed=31, n_cams=12, n_pts=1500, outlier_frac=0.0))
    st, out, _, _ = oracle_mod.calc_plsa(blk, rb.make_options(robust=False))
    assert st == 0
    return out


def _ints(log):
    """The integer fields of the Sigma0 lines (redundancy, observations,
    unknowns, IT, ITT) and of the Sigma0AO line (prior observations)."""
    out = []
    for l in log.splitlines():
        m = re.match(r"Sigma0: \S+ \S+\s+(\d+) (\d+) (\d+)\s+IT: (\d+)\s+ITT: (\d+)", l)
        if m:
            out.append(m.groups())
        m = re.match(r"Sigma0AO: \S+\s+\S+ \S+\s+(\d+) ", l)
        if m:
            out.append(m.groups())
    return out


@pytest.mark.parametrize("every", [1, 3])
def test_gcp_step_matches_oracle(oracle_mod, solved, every):
    """Perturbed cameras, every `every`-th point a stiff GCP at the solution
    (GCP index 0 included: kept with two or more observations only)."""
    import rpba_b200 as rb
    blk = solved.copy()
    rng = np.random.default_rng(3)
    P = blk.pmat.reshape(-1, 3, 4)
    P[:, :, 3] += rng.normal(0, 0.05, (blk.n_images, 3)).astype(np.float32)
    n = blk.n_points
    gcpinfo = np.full(n, -1, np.int32)
    sel = np.arange(0, n, every)
    gcpinfo[sel] = np.arange(len(sel), dtype=np.int32)
    W3 = np.tile(np.array([1e4, 1e4, 1e4, 0, 0, 0], np.float32), (len(sel), 1))
    gd = solved.XX[sel].astype(np.float64)
    o = rb.make_options(robust=False, solver=rb.SOLVER_DIRECT)
    st_o, b_o, P_o, used_o, log_o = oracle_mod.lsa_gcp_step_full(blk, gcpinfo, W3, gd, blk.n_images, opts=o)
    st_g, b_g, P_g, used_g, rep, log_g = rb.lsa_gcp_step(blk, gcpinfo, W3, gd, blk.n_images,
                                                         solver=rb.SOLVER_DIRECT)
    assert st_o == st_g == 0, (log_o, log_g)
    assert np.array_equal(used_o, used_g)
    scale = np.abs(P_o).max()
    assert np.abs(P_g - P_o).max() <= 1e-9 * scale, np.abs(P_g - P_o).max()
    assert np.array_equal(b_g.K, b_o.K) or np.abs(b_g.K - b_o.K).max() <= 1e-6 * np.abs(b_o.K).max()
    assert _ints(log_g) == _ints(log_o), (log_g, log_o)


@pytest.mark.parametrize("k", [2, 3])
def test_parallel_loop_matches_oracle(oracle_mod, k):
    import rpba_b200 as rb
    from rpba_b200 import scenes
    blk = scenes.to_block(scenes.arc_scene(seed=5, n_cams=50, n_pts=8000))
    part = rb.partition_images(blk, k)
    o = rb.make_options(solver=rb.SOLVER_DIRECT)
    st_o, b_o, s_o, _ = oracle_mod.calc_plsa_parallel(blk, part, k, o)
    st_g, b_g, s_g, log_g = rb.calc_plsa_parallel(blk, part, k, solver=rb.SOLVER_DIRECT)
    assert st_o == st_g == 0, log_g[-2000:]
    assert s_g["iterations"] == s_o["iterations"]
    ev = lambda b: oracle_mod.exteval(b)[1]["exteval_sigma0"]
    e_o, e_g = ev(b_o), ev(b_g)
    print(f"k={k}: Exteval sigma0 GPU {e_g:.7f} oracle {e_o:.7f}, {s_g['iterations']} iterations")
    assert abs(e_g - e_o) <= 1e-6 * e_o


def test_calc_plsa_threads_selects_the_partitioned_branch(oracle_mod):
    """rpba_calc_plsa with threads = 4 on a 150-image scene takes the
    reference's partitioned branch (rpbacore.cpp:79-92: min(4, iround(150 /
    70)) = 2 partitions): the log opens with the reference's '#threads: 2 2'
    and 'Thread:' lines, and the block equals the partitioned loop's on the
    same partition; threads = 1 keeps the global branch."""
    import rpba_b200 as rb
    from rpba_b200 import scenes
    blk = scenes.to_block(scenes.arc_scene(seed=9, n_cams=150, n_pts=9000))
    b = blk.copy()
    st, log, rep = rb.CalcPLSA(b, threads=4, solver=rb.SOLVER_DIRECT)
    assert st == 0, log[-2000:]
    assert log.startswith("#threads: 2 2\n"), log[:200]
    assert sum(1 for l in log.splitlines() if l.startswith("Thread: ")) == 2
    part = oracle_mod.partition_images(blk, 2)
    st_o, b_o, s_o, _ = oracle_mod.calc_plsa_parallel(blk, part, 2, rb.make_options(solver=rb.SOLVER_DIRECT))
    assert st_o == 0
    ev = lambda x: oracle_mod.exteval(x)[1]["exteval_sigma0"]
    e_o, e_g = ev(b_o), ev(b)
    print(f"Threads=4 branch: Exteval sigma0 GPU {e_g:.7f} oracle {e_o:.7f}")
    assert abs(e_g - e_o) <= 1e-6 * e_o
    st1, log1, _ = rb.CalcPLSA(blk.copy(), threads=1, solver=rb.SOLVER_DIRECT)
    assert st1 == 0 and not log1.startswith("#threads")


def test_parallel_loop_is_reproducible():
    """The partition steps of an outer iteration run concurrently on host
    threads, each on its own handle and stream, with the reference's PCG as
    the partition solver (cooperative kernels one at a time); two runs give
    the same block, statistics and log bit for bit, whichever order the
    steps ran in."""
    import rpba_b200 as rb
    from rpba_b200 import scenes
    blk = scenes.to_block(scenes.arc_scene(seed=5, n_cams=50, n_pts=8000))
    part = rb.partition_images(blk, 4)
    st1, b1, s1, log1 = rb.calc_plsa_parallel(blk, part, 4)
    st2, b2, s2, log2 = rb.calc_plsa_parallel(blk, part, 4)
    assert st1 == st2 == 0, log1[-2000:]
    assert s1 == s2 and log1 == log2
    for name in ("pmat", "K", "distpara", "XX", "pt_obs_off", "pt_obs_image", "pt_obs_slot"):
        assert np.array_equal(getattr(b1, name), getattr(b2, name)), name


def test_ranks_form_on_one_rank_equals_the_loop():
    """rpba_calc_plsa_parallel_ranks on one rank, its all-gather returning
    the rank's own bytes: the exchange of the partition steps' results runs
    (written and read back after every round of steps) and the block,
    statistics and log equal rpba_calc_plsa_parallel's bit for bit.  (Over
    several ranks the loop is checked on CPU with gloo ranks,
    test_cpu_parallel_ranks.py.)"""
    import rpba_b200 as rb
    from rpba_b200 import lib, scenes
    blk = scenes.to_block(scenes.arc_scene(seed=5, n_cams=50, n_pts=8000))
    part = rb.partition_images(blk, 4)
    st1, b1, s1, log1 = rb.calc_plsa_parallel(blk, part, 4)
    calls = []

    def gather(data):
        calls.append(len(data))
        return data

    st2, b2, s2, log2 = lib.calc_plsa_parallel_ranks(blk, part, 4, 0, 1, gather)
    assert st1 == st2 == 0, log2[-2000:]
    assert s1 == s2 and log1 == log2
    assert len(calls) == 2 * (s2["iterations"] - 1)
    for name in ("pmat", "K", "distpara", "XX", "pt_obs_off", "pt_obs_image", "pt_obs_slot"):
        assert np.array_equal(getattr(b1, name), getattr(b2, name)), name
