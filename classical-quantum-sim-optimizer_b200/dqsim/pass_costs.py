"""Training data and training of the learned fused-pass cost model.

The complex64 form runs its unitary runs as tensor-core passes of 12 tile
qubits, planned as a portfolio: one plan per cap on the pass's "spread" (how
far its tile qubits scatter the runs of amplitudes that the tiles in flight
read together).  Which plan is fastest depends on where each pass's tile
qubits sit in the state, how many blocks it holds and the state's size; the
hand-fitted rule prices it with constants fitted at 30 and 32 qubits.  A
CostModel of kind "fused_passes" learns it instead from device timings this
engine records itself: every distinct pass of the candidate plans of seeded
brickwork and QFT circuits of 24-30 qubits, plus seeded random passes at
24-32 qubits.  Attached to a simulator, the model picks the plan of least
predicted time; a prepared circuit times that plan against the hand rule's
and keeps the faster, logging a rejection when the learned plan is slower.

A recorded pass is a row: state qubits, tile-qubit mask, blocks, gates and
device milliseconds of one k_fused launch over one state.  The model's
features come from the library (dq_fused_pass_features); its target is the
log of device nanoseconds per tile.
"""

import numpy as np

from . import _core, workloads

# Seeded random passes per state size (the bulk of the training set).
RANDOM_PASSES = {24: 11000, 26: 11000, 28: 11000, 30: 9000, 31: 4000, 32: 3000}
# Circuits whose candidate plans' passes join the training set: depth-40 brickwork and QFT, 24-30 qubits.
TRAIN_CIRCUITS = ([("brickwork", n, 100 + 10 * n + s) for n in (24, 26, 28, 30) for s in range(2)]
                  + [("qft", n, 200 + n) for n in (24, 26, 28, 30)])
# Held-out circuits (seeds outside the training set): depth-40 brickwork at 26, 30 and 33 qubits, QFT at 32.
HELD_OUT = [("brickwork", 26, 9026), ("brickwork", 30, 9030), ("brickwork", 33, 9033), ("qft", 32, 9032)]
CHUNK = 1000


def circuit(kind, n, seed):
    """A seeded unitary workload circuit: depth-40 brickwork or the QFT."""
    if kind == "brickwork":
        return workloads.brickwork(n, 40, seed=seed, measure=False)
    if kind == "qft":
        return workloads.qft(n, seed=seed)
    raise ValueError(f"unknown circuit kind {kind!r}")


def rows_of(passes, n):
    """Recorded passes (the "passes" list of fused_portfolio / fused_random_passes) as row arrays."""
    mask = np.array([sum(1 << q for q in p["qubits"]) for p in passes], dtype=np.uint64)
    return {"n": np.full(len(passes), n, dtype=np.uint8), "mask": mask,
            "blocks": np.array([p["blocks"] for p in passes], dtype=np.uint8),
            "gates": np.array([p["gates"] for p in passes], dtype=np.uint16),
            "ms": np.array([p["ms"] for p in passes], dtype=np.float32)}


def concat(parts):
    return {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}


def tile_qubits(mask):
    m = int(mask)
    return [q for q in range(64) if (m >> q) & 1]


def features(rows):
    """The model's inputs, one row per recorded pass (computed by the library)."""
    X = np.empty((len(rows["ms"]), _core.MLP_FEATURES), dtype=np.float32)
    for i in range(X.shape[0]):
        X[i] = _core.fused_pass_features(int(rows["n"][i]), tile_qubits(rows["mask"][i]), int(rows["blocks"][i]),
                                         int(rows["gates"][i]))
    return X


def targets(rows):
    """Log of device nanoseconds per tile (a tile is 4096 amplitudes)."""
    tiles = np.exp2(rows["n"].astype(np.float64) - 12.0)
    return np.log(rows["ms"].astype(np.float64) * 1e6 / tiles).astype(np.float32)


def record(sim, random_passes=RANDOM_PASSES, circuits=TRAIN_CIRCUITS, seed=0):
    """Times the training passes on the simulator's device; returns their rows."""
    parts = []
    for n, count in random_passes.items():
        for c0 in range(0, count, CHUNK):
            out = _core.fused_random_passes(sim, n, min(CHUNK, count - c0), seed=seed * 1000003 + n * 1009 + c0,
                                            measure=True)
            parts.append(rows_of(out["passes"], n))
    for kind, n, s in circuits:
        pf = _core.fused_portfolio(sim, circuit(kind, n, s), wide=True, measure=True)
        parts.append(rows_of(pf["passes"], n))
    return concat(parts)


def train(rows, seed=0, epochs=60, lr=2e-3, device=0):
    """A fused-pass CostModel trained (on the device) on recorded rows; returns (model, final MSE)."""
    model = _core.CostModel(device=device, seed=seed, kind="fused_passes")
    model.add_samples(features(rows), targets(rows))
    mse = model.train(epochs=epochs, lr=lr)
    return model, mse


def portfolio_rows(pf):
    """A recorded portfolio's distinct passes as rows (their measured milliseconds included)."""
    return rows_of(pf["passes"], pf["n"])


def plan_ms(pf, pass_ms):
    """Total milliseconds of each candidate plan from per-pass milliseconds."""
    return [float(sum(pass_ms[i] for i in plan["passes"])) for plan in pf["plans"]]


def predicted_plan_ms(model, pf):
    """The model's predicted milliseconds of each candidate plan of a portfolio."""
    rows = portfolio_rows(pf)
    tiles = 2.0 ** (pf["n"] - 12)
    pass_ms = np.exp(model.predict(features(rows)).astype(np.float64)) * tiles * 1e-6
    return plan_ms(pf, pass_ms)
