"""The recorded fused-pass dataset matches the current planner (host only).

The learned planner's GPU test trains on tests/golden/fused_pass_costs_b200.npz
and judges its choices on tests/golden/fused_pass_portfolios_b200.json.  Here,
without a device, the held-out circuits are planned again and every candidate
plan and pass (tile qubits, blocks, gates, the hand rule's choice) must be the
one recorded, so the dataset describes the planner that ships; and every
recorded row must give finite features and targets.
"""

import json
from pathlib import Path

import numpy as np

import dqsim
from dqsim import _core, pass_costs

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_recorded_rows_give_finite_features_and_targets():
    rows = dict(np.load(GOLDEN / "fused_pass_costs_b200.npz"))
    assert len(rows["ms"]) >= 20000
    assert np.all(rows["ms"] > 0)
    sample = {k: v[::97] for k, v in rows.items()}
    X = pass_costs.features(sample)
    y = pass_costs.targets(sample)
    assert np.all(np.isfinite(X)) and np.all(np.isfinite(y))
    assert set(np.unique(rows["n"]).tolist()) >= {24, 26, 28, 30, 32}


def test_held_out_portfolios_are_the_current_planners():
    held = json.loads((GOLDEN / "fused_pass_portfolios_b200.json").read_text())["held_out"]
    assert [(h["kind"], h["n"], h["seed"]) for h in held] == [tuple(x) for x in pass_costs.HELD_OUT]
    sim = dqsim.StatevectorSimulator(precision="complex64")
    for h in held:
        now = _core.fused_portfolio(sim, pass_costs.circuit(h["kind"], h["n"], h["seed"]), wide=True, measure=False)
        rec = h["portfolio"]
        assert now["rule_choice"] == rec["rule_choice"]
        assert [p["passes"] for p in now["plans"]] == [p["passes"] for p in rec["plans"]]
        assert [p["cap"] for p in now["plans"]] == [p["cap"] for p in rec["plans"]]
        for a, b in zip(now["passes"], rec["passes"]):
            assert (a["qubits"], a["blocks"], a["gates"]) == (b["qubits"], b["blocks"], b["gates"])
            np.testing.assert_allclose(a["features"], b["features"], rtol=1e-5)
