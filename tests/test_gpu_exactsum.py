"""The GPU's exact float sequential sum against numpy's sequential float32
cumsum, bit for bit, on adversarial inputs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases():
    rng = np.random.default_rng(5)
    yield "empty", np.zeros(0, np.float32)
    yield "one", np.array([3.5], np.float32)
    yield "zeros", np.zeros(50_000, np.float32)
    yield "cost-like", (rng.normal(0, 0.5, 950_000) ** 2 * 2).astype(np.float32)
    v = (rng.normal(0, 0.5, 700_000) ** 2).astype(np.float32)
    v[rng.random(v.size) < 0.05] = rng.uniform(0, 5000, int((rng.random(v.size) < 0.05).sum()) or 1)[0]
    yield "outliers", v
    w = np.full(1_200_000, 2.0, np.float32)
    w[rng.random(w.size) < 0.07] = np.float32(2e-4)
    yield "weights", w
    yield "halves (ties)", (rng.integers(0, 4, 300_000) * 0.5).astype(np.float32)
    yield "heavy tail", np.exp(rng.normal(0, 6, 400_000)).astype(np.float32)
    t = np.zeros(200_000, np.float32)
    t[::1000] = 1e-40  # subnormal stretches
    t[100_000:] = (rng.random(100_000)).astype(np.float32)
    yield "subnormal start", t
    yield "huge first", np.concatenate([[np.float32(3e38)], rng.random(100_000).astype(np.float32)])
    # shrinking terms: the sum stays in one binade across many windows
    yield "shrinking terms", (1.0 / np.sqrt(1.0 + np.arange(2_000_000))).astype(np.float32)
    yield "growing terms", (np.arange(1_500_000) * 1e-3).astype(np.float32)


@pytest.mark.parametrize("name,v", list(_cases()), ids=[c[0] for c in _cases()])
def test_exact_sum_bitwise(name, v):
    import rpba_b200 as rb
    ref = np.cumsum(v, dtype=np.float32)[-1] if v.size else np.float32(0)
    got = rb.float_sequential_sum(v)
    assert got.tobytes() == np.float32(ref).tobytes(), (name, got, ref)


def test_exact_sum_bitwise_bench_size():
    """The bench's size: 29M cost-like terms (generated inside the test, not
    at collection)."""
    import rpba_b200 as rb
    rng = np.random.default_rng(6)
    v = (rng.normal(0, 0.5, 29_000_000) ** 2 * rng.uniform(0.1, 2.0, 29_000_000)).astype(np.float32)
    ref = np.cumsum(v, dtype=np.float32)[-1]
    got = rb.float_sequential_sum(v)
    assert got.tobytes() == np.float32(ref).tobytes(), (got, ref)
