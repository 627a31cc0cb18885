"""The planner's learned cost model: CUDA gradients vs a CPU oracle, training,
recording from the engine's own timings, and the learned-vs-greedy A/B."""

import numpy as np
import pytest

from oracle import oracle as o

import dqsim
from dqsim import _core, workloads

pytestmark = pytest.mark.gpu
F, H = 16, 64


def unpack(P):
    W1 = P[0:H * F].reshape(H, F)
    b1 = P[H * F:H * F + H]
    o2 = H * F + H
    W2 = P[o2:o2 + H * H].reshape(H, H)
    b2 = P[o2 + H * H:o2 + H * H + H]
    o3 = o2 + H * H + H
    W3 = P[o3:o3 + H]
    b3 = P[o3 + H]
    return W1, b1, W2, b2, W3, b3


def numpy_gradients(P, X, y):
    """Backpropagation of the mean squared error in float64 (the CPU oracle)."""
    W1, b1, W2, b2, W3, b3 = (np.asarray(a, dtype=np.float64) for a in unpack(P))
    X = X.astype(np.float64)
    n = X.shape[0]
    a1 = np.maximum(X @ W1.T + b1, 0)
    a2 = np.maximum(a1 @ W2.T + b2, 0)
    yp = a2 @ W3 + b3
    d = 2 * (yp - y) / n
    gW3, gb3 = a2.T @ d, d.sum()
    dz2 = np.outer(d, W3) * (a2 > 0)
    gW2, gb2 = dz2.T @ a1, dz2.sum(0)
    dz1 = (dz2 @ W2) * (a1 > 0)
    gW1, gb1 = dz1.T @ X, dz1.sum(0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])


def test_gradients_match_cpu_oracle():
    m = _core.CostModel(seed=3)
    rng = np.random.default_rng(0)
    for n in (1, 37, 128):
        X = rng.normal(size=(n, F)).astype(np.float32)
        y = rng.normal(size=n).astype(np.float32)
        g = m.gradients(X, y)
        want = numpy_gradients(m.params[:-2], X, y)
        np.testing.assert_allclose(g, want, rtol=2e-3, atol=2e-5)


def test_training_fits_a_smooth_function():
    rng = np.random.default_rng(1)
    X = rng.uniform(0, 1, size=(4096, F)).astype(np.float32)
    y = (3 * X[:, 0] + np.sin(4 * X[:, 1]) + X[:, 2] * X[:, 3] + 5).astype(np.float32)
    m = _core.CostModel(seed=4)
    m.add_samples(X, y)
    mse = m.train(epochs=80, lr=3e-3)
    assert mse < 0.05, mse  # in units of the target's variance
    Xt = rng.uniform(0, 1, size=(512, F)).astype(np.float32)
    yt = 3 * Xt[:, 0] + np.sin(4 * Xt[:, 1]) + Xt[:, 2] * Xt[:, 3] + 5
    pred = m.predict(Xt)
    assert np.corrcoef(pred, yt)[0, 1] > 0.97


def test_engine_records_samples_and_learned_plan_is_judged_by_greedy():
    model = _core.CostModel(seed=5)
    for width in (1, 2, 3):
        sim = dqsim.StatevectorSimulator(seed=1, precision="complex64", fusion_width=width, max_memory_mb=1 << 13)
        for c in (workloads.brickwork(20, 8, seed=width, measure=False), workloads.qft(18, seed=width),
                  workloads.hea(19, 5, seed=width)):
            added = model.record(sim, c)
            assert added > 0
    X, y = model.samples()
    assert X.shape[0] == model.num_samples and np.all(np.isfinite(y)) and np.all(y > 0)
    model.train(epochs=40, lr=2e-3)
    sim = dqsim.StatevectorSimulator(seed=2, precision="complex64", max_memory_mb=1 << 13)
    _core.set_cost_model(sim, model)
    held_out = workloads.brickwork(21, 10, seed=77, measure=False)
    plan = _core.PreparedCircuit(sim, held_out)
    info = plan.planner()
    assert info["greedy_ms"] > 0 and info["learned_ms"] > 0
    assert info["used_learned"] != info["rejected"]
    log = _core.planner_log(sim)
    assert log and log[-1]["rejected"] == info["rejected"]
    # whichever plan was kept, the state is right
    plan.run()
    want = o.OracleSimulator(seed=2).simulate(held_out).statevector
    got = plan.statevector()
    assert abs(np.vdot(got, want)) ** 2 >= 1 - 1e-6
    _core.set_cost_model(sim, None)
