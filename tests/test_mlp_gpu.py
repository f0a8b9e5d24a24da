"""The tcgen05 radiance-cache MLP against the FP64 CPU oracle (oracle/mlp_oracle.py).

Bars (BF16 operands, FP32 accumulation): forward outputs within 2e-2 relative; gradients of
every weight matrix with cosine similarity > 0.999 and relative L2 error < 2e-2; an Adam step
within 1e-3 relative of the oracle's; training on a smooth target lowers the loss tenfold; queries
run on the bias-corrected weight average when one is kept."""
from __future__ import annotations

import numpy as np
import pytest

import ptb200 as pt
import mlp_oracle as mo

pytestmark = pytest.mark.gpu
LO, HI = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)


def queries(n, seed):
    g = np.random.default_rng(seed)
    q = np.zeros(n, pt.CACHE_QUERY)
    q["position"] = g.uniform(-1, 1, (n, 3))
    d = g.normal(size=(n, 3)); d /= np.linalg.norm(d, axis=1, keepdims=True)
    q["direction"] = d
    nrm = g.normal(size=(n, 3)); nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    q["normal"] = nrm
    q["albedo"] = g.uniform(0.2, 0.8, (n, 3))
    q["roughness"] = g.uniform(0, 1, n)
    return q


def target_fn(q):
    p = q["position"].astype(np.float64)
    d = q["direction"].astype(np.float64)
    r = 0.5 + 0.4 * np.sin(2 * p[:, 0]) * np.cos(p[:, 1]) + 0.3 * d[:, 2] ** 2
    return np.stack([r, 0.8 * r + 0.1 * p[:, 2], 0.6 + 0.2 * d[:, 0]], axis=1).clip(0.05, None).astype(np.float32)


def to_dev(a):
    torch = pytest.importorskip("torch")
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).cuda()


@pytest.mark.parametrize("n", [1, 128, 1000, 4096])
def test_forward_matches_oracle(n):
    torch = pytest.importorskip("torch")
    cache = pt.RadianceCache(LO, HI, seed=3)
    q = queries(n, n)
    out = torch.zeros(n * 3, dtype=torch.float32, device="cuda")
    cache.query(to_dev(q), n, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(n, 3)
    want = mo.forward(cache.weights(), mo.encode(q, LO, HI))
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-6)
    assert rel.max() < 2e-2, rel.max()


@pytest.mark.parametrize("n", [128, 3000])
def test_gradients_match_oracle(n):
    cache = pt.RadianceCache(LO, HI, seed=5)
    q = queries(n, 100 + n)
    t = target_fn(q)
    loss, g = cache.gradients(to_dev(q), to_dev(t), n)
    want_loss, want = mo.loss_and_grad(cache.weights(), mo.encode(q, LO, HI), t)
    assert abs(loss - want_loss) <= 2e-2 * abs(want_loss)
    offsets = [0] + [4096 * (l + 1) for l in range(5)] + [pt.CACHE_WEIGHTS]
    for l in range(6):
        a, b = g[offsets[l]:offsets[l + 1]].astype(np.float64), want[offsets[l]:offsets[l + 1]].astype(np.float64)
        cos = float(a @ b / max(1e-30, np.linalg.norm(a) * np.linalg.norm(b)))
        rel = float(np.linalg.norm(a - b) / max(1e-30, np.linalg.norm(b)))
        assert cos > 0.999 and rel < 2e-2, (l, cos, rel)


def test_adam_step_matches_oracle():
    n = 1024
    cache = pt.RadianceCache(LO, HI, seed=7)
    q = queries(n, 77)
    t = target_fn(q)
    w0 = cache.weights().astype(np.float64)
    _, g = cache.gradients(to_dev(q), to_dev(t), n)
    cache.train(to_dev(q), to_dev(t), n)
    w1 = cache.weights().astype(np.float64)
    want, _, _ = mo.adam(w0, np.zeros_like(w0), np.zeros_like(w0), g.astype(np.float64), 1)
    assert np.abs(w1 - want).max() <= 1e-3 * max(1.0, np.abs(want).max())


def test_training_lowers_the_loss():
    n = 1 << 14
    cache = pt.RadianceCache(LO, HI, seed=11)
    q = queries(n, 5)
    t = target_fn(q)
    dq, dt = to_dev(q), to_dev(t)
    first = cache.train(dq, dt, n)
    for _ in range(300):
        last = cache.train(dq, dt, n)
    assert np.isfinite(last) and last < first / 10, (first, last)


def test_weight_average_is_what_queries_use():
    """With a decay d, queries run on sum_k (1-d) d^(t-k) w_k / (1 - d^t) over the weights after
    each of the t steps; pt_cache_average restarts the average."""
    torch = pytest.importorskip("torch")
    n, d = 2048, 0.9
    cache = pt.RadianceCache(LO, HI, seed=13)
    cache.average(d)
    q = queries(n, 31)
    t = target_fn(q)
    dq, dt = to_dev(q), to_dev(t)
    avg = np.zeros(pt.CACHE_WEIGHTS)
    for step in range(1, 6):
        cache.train(dq, dt, n)
        avg = d * avg + (1 - d) * cache.weights().astype(np.float64)
    expect_w = (avg / (1 - d ** 5)).astype(np.float32)
    out = torch.zeros(n * 3, dtype=torch.float32, device="cuda")
    cache.query(dq, n, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(n, 3)
    x = mo.encode(q, LO, HI)
    want = mo.forward(expect_w, x)
    assert (np.abs(got - want) / np.maximum(np.abs(want), 1e-6)).max() < 2e-2
    live = mo.forward(cache.weights(), x)
    assert np.abs(live - want).max() > 1e-3          # the average is not the live weights
    cache.average(0.0)                               # queries on the live weights again
    cache.query(dq, n, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(n, 3)
    assert (np.abs(got - live) / np.maximum(np.abs(live), 1e-6)).max() < 2e-2


def test_tensor_core_wait_timeout_is_reported_and_recoverable():
    """Failure detection of the tensor-core kernels without a GPU fault: with a limit of 0 try_wait
    attempts every bounded mbarrier wait runs out at once.  The forward pass and a training step
    then report PT_TIMEOUT, the weights stay as they were (no Adam step is applied), each kernel
    frees its TMEM after waiting for its own MMAs, and with the default limit back the same cache
    answers exactly as before."""
    torch = pytest.importorskip("torch")
    cache = pt.RadianceCache(LO, HI, seed=3)
    n = 4096
    q = queries(n, 11)
    t = target_fn(q)
    qd, td = to_dev(q), to_dev(t)
    out0 = torch.zeros(n * 3, dtype=torch.float32, device="cuda")
    cache.query(qd, n, out0)
    cache.sync()
    l0, g0 = cache.gradients(qd, td, n)
    w0 = cache.weights()
    cache.wait_limit(0)
    out1 = torch.full((n * 3,), -1.0, dtype=torch.float32, device="cuda")
    cache.query(qd, n, out1)
    with pytest.raises(pt.PtError) as e:
        cache.sync()
    assert e.value.status == 6                       # PT_TIMEOUT
    with pytest.raises(pt.PtError) as e:
        cache.train(qd, td, n, wait=True)
    assert e.value.status == 6
    assert np.array_equal(cache.weights(), w0)       # no step on a timed-out gradient pass
    cache.wait_limit(-1)
    cache.sync()                                     # nothing left pending
    out2 = torch.zeros(n * 3, dtype=torch.float32, device="cuda")
    cache.query(qd, n, out2)
    cache.sync()
    assert torch.equal(out0, out2)
    l2, g2 = cache.gradients(qd, td, n)
    assert np.array_equal(g0, g2) and l0 == l2
    cache.train(qd, td, n, wait=True)
    assert not np.array_equal(cache.weights(), w0)
