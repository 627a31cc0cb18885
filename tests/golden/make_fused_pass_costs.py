"""Records the fused-pass timing fixture on a B200 (run on a GPU machine).

The learned planner's test trains a fused-pass cost model on these recorded
device timings and checks which candidate plan it picks for held-out circuits
against the plans' recorded times.  Recording needs the device; the test
itself then needs no new timings, so its outcome does not depend on which
B200 runs it.

Writes, next to this script (or to the directory given as the first argument):
  fused_pass_costs_b200.npz       training rows: state qubits, tile-qubit mask,
                                  blocks, gates and k_fused milliseconds of
                                  seeded random passes and of every distinct
                                  pass of the candidate plans of the training
                                  circuits (dqsim.pass_costs.RANDOM_PASSES,
                                  TRAIN_CIRCUITS);
  fused_pass_portfolios_b200.json the held-out circuits' candidate plans
                                  (dqsim.pass_costs.HELD_OUT): every distinct
                                  pass with its measured milliseconds, each
                                  plan's passes and the hand rule's choice.
"""

import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "classical-quantum-sim-optimizer_b200"))

import dqsim  # noqa: E402
from dqsim import _core, pass_costs  # noqa: E402


def main():
    out_dir = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent
    out_dir.mkdir(parents=True, exist_ok=True)
    sim = dqsim.StatevectorSimulator(precision="complex64", max_memory_mb=1 << 20)
    t0 = time.time()
    rows = pass_costs.record(sim)
    record_s = time.time() - t0
    np.savez_compressed(out_dir / "fused_pass_costs_b200.npz", **rows)
    held = []
    for kind, n, seed in pass_costs.HELD_OUT:
        pf = _core.fused_portfolio(sim, pass_costs.circuit(kind, n, seed), wide=True, measure=True)
        held.append({"kind": kind, "n": n, "seed": seed, "portfolio": pf})
    (out_dir / "fused_pass_portfolios_b200.json").write_text(json.dumps({"held_out": held}))
    print(json.dumps({"training_rows": int(len(rows["ms"])), "record_s": record_s,
                      "held_out": [{"kind": h["kind"], "n": h["n"], "rule_choice": h["portfolio"]["rule_choice"],
                                    "plan_ms": pass_costs.plan_ms(h["portfolio"],
                                                                  [p["ms"] for p in h["portfolio"]["passes"]])}
                                   for h in held]}))


if __name__ == "__main__":
    main()
