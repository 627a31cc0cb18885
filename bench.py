"""Benchmark: 30-qubit depth-40 random brickwork, plain complex128 vs complex64 form.

One step = one full circuit on one GPU: |0...0>, every compiled operation,
FP64 terminal probabilities, CDF and 10^5 seeded samples, with the circuit
plan and state buffers resident in HBM (dq_plan_*).  Each form is timed with
CUDA events on the engine's stream.  The 16 GiB / 8 GiB state is far larger
than the 126 MB L2, so no flush is needed between steps.

`value` is the circuit time of the complex64 form (seconds per circuit; for
N GPUs, replicas: N circuits / max-over-ranks time, reported as seconds per
circuit).  The plain complex128 time, both forms' algorithmic HBM GB/s, and the
complex64 state's fidelity / max amplitude error against the complex128 run
are reported beside it.

--impl reference times the CPU restatement of the reference's engine
(oracle/, OpenMP on every host core) on a bounded sample of the same circuit:
the first operations at 30 qubits, scaled by operation count.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "classical-quantum-sim-optimizer_b200"
for _p in (str(PKG), str(ROOT)):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "30q circuit time & HBM GB/s: fused FP32 vs plain FP64 at fidelity≥1−1e-6"
FALLBACK_HBM = 6650.0


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", FALLBACK_HBM)), "measured"
    return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, local, value):
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{local}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def time_form(dqsim, circuit, precision, local, steps, warmup, shots, seed, execution="auto"):
    sim = dqsim.StatevectorSimulator(seed=seed, max_memory_mb=1 << 20, precision=precision, device=local,
                                     execution=execution)
    plan = dqsim._core.PreparedCircuit(sim, circuit, shots=shots)
    for _ in range(warmup):
        plan.run()
    return sim, plan


def cpu_reference_sample(circuit, budget_s, threads=None):
    """Time the oracle's kernels on the first operations of the circuit at full size."""
    from oracle import oracle

    L = oracle.lib()
    if threads:
        L.orc_set_num_threads(threads)
    n, _, ops = oracle.circuit_ops(circuit.model_dump_json())
    unitary = [op for op in ops if op[0] not in ("measure", "reset", "cond")]
    import numpy as np

    t0 = time.perf_counter()
    state = np.zeros(1 << n, dtype=np.complex128)
    state[0] = 1.0
    alloc_s = time.perf_counter() - t0
    done = 0
    t1 = time.perf_counter()
    rng = oracle.ChaCha8Stream(0)
    while done < len(unitary) and time.perf_counter() - t1 < budget_s:
        oracle.apply_op(unitary[done], state, n, [], rng, True)
        done += 1
    per_op = (time.perf_counter() - t1) / max(done, 1)
    del state
    return {"per_op_s": per_op, "ops_timed": done, "ops_total": len(unitary), "alloc_s": alloc_s,
            "circuit_s": per_op * len(unitary), "threads": L.orc_num_threads(), "qubits": n}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import dqsim

    circuit = dqsim.workloads.brickwork(args.qubits, args.depth, seed=args.seed, measure=True)
    samples = []
    info = None
    for i in range(args.warmup + args.steps):
        info = cpu_reference_sample(circuit, args.cpu_budget / max(1, args.steps + args.warmup))
        if i >= args.warmup:
            samples.append(info["circuit_s"])
    value = statistics.mean(samples)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "higher_is_better": False,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)", "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": "s", "cores": info["threads"], "kind": "port",
                         "sample": f"first {info['ops_timed']} of {info['ops_total']} operations at "
                                   f"{info['qubits']} qubits per step, scaled by operation count"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def workload_config(args):
    return {"workload": f"brickwork-{args.qubits}q-d{args.depth}-seed{args.seed}-{args.shots}shots",
            "qubits": args.qubits, "depth": args.depth, "shots": args.shots, "seed": args.seed,
            "parallelism": "replicas", "l2": "state (16 GiB c128 / 8 GiB c64) exceeds L2; no flush"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--depth", type=int, default=40)
    ap.add_argument("--shots", type=int, default=100000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU baseline work")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--plain-steps", type=int, default=1)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    world, rank, local, pg = dist_setup(args)
    import dqsim

    peak, peak_kind = peaks()
    circuit = dqsim.workloads.brickwork(args.qubits, args.depth, seed=args.seed, measure=True)

    def bytes_of(stats):
        return sum(v["bytes"] for k, v in stats.items() if k != "sample")

    def summarize(stats, ms_):
        gbs = bytes_of(stats) / (ms_ * 1e-3) / 1e9
        return {"s": ms_ * 1e-3, "gbs": gbs, "frac_of_hbm": gbs / peak, "kernels": stats}

    # Plain complex128 form: the reference's arithmetic, one HBM pass per operation.
    sim128, plan128 = time_form(dqsim, circuit, "complex128", local, 1, 0, args.shots, args.seed,
                                execution="per_gate")
    t128 = [plan128.run() for _ in range(args.plain_steps)]
    plan128.run(record=True)
    st128 = plan128.stats()
    ms128 = statistics.mean(t128)
    per_gate = st128.get("gate1q")
    plain_kernel = None
    if per_gate:
        ach = per_gate["bytes"] / (per_gate["ms"] * 1e-3) / 1e9
        plain_kernel = {"kernel": "gate1q (c128, per-gate)", "achieved": ach, "frac": ach / peak,
                        "launches": per_gate["launches"]}

    # complex128 with shared-memory tile passes (same FP64 arithmetic, fused 4x4 within a pass).
    simt, plant = time_form(dqsim, circuit, "complex128", local, 1, 1, args.shots, args.seed)
    tt = [plant.run() for _ in range(args.plain_steps)]
    plant.run(record=True)
    stt = plant.stats()
    mst = statistics.mean(tt)
    tiled_fid, tiled_err = plant.compare(plan128)
    del plant, simt

    # Complex64 form (the chosen form).
    sim64, plan64 = time_form(dqsim, circuit, "complex64", local, 1, args.warmup, args.shots, args.seed)
    barrier(pg)
    with ClockSampler(local) as clocks:
        times = [plan64.run() for _ in range(args.steps)]
    barrier(pg)
    ms = max_over_ranks(pg, local, statistics.mean(times))
    plan64.run(record=True)
    st64 = plan64.stats()
    fidelity, max_err = plan64.compare(plan128)
    del plan128, sim128

    gb64 = bytes_of(st64) / (ms * 1e-3) / 1e9
    dom = max(st64.items(), key=lambda kv: kv[1]["ms"])
    dom_achieved = dom[1]["bytes"] / (dom[1]["ms"] * 1e-3) / 1e9

    # End to end through the public API: host JSON in, host counts out.
    e2e = None
    if True:
        api = dqsim.StatevectorSimulator(seed=args.seed, max_memory_mb=1 << 20, precision="complex64", device=local)
        api.simulate_shots(circuit, shots=args.shots)
        t0 = time.perf_counter()
        counts = api.simulate_shots(circuit, shots=args.shots)
        e2e_s = time.perf_counter() - t0
        assert sum(counts.values()) == args.shots
        e2e = {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": len(circuit.model_dump_json()),
               "d2h_bytes_per_step": 8 * args.shots}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        info = cpu_reference_sample(circuit, args.cpu_budget)
        cpu = {"value": info["circuit_s"], "unit": "s", "cores": info["threads"], "kind": "port",
               "sample": f"first {info['ops_timed']} of {info['ops_total']} operations at {info['qubits']} qubits "
                         f"(OpenMP C restatement of src/engine.rs), scaled by operation count"}

    value = (ms * 1e-3) / world
    launches = sum(v["launches"] for k, v in st64.items())
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 (f32, FP64 reductions)", "data": "synthetic",
        "config": workload_config(args),
        "forms": {
            "complex64": {**summarize(st64, ms), "fidelity": fidelity, "max_amp_err": max_err},
            "complex128_per_gate": {**summarize(st128, ms128), "dominant": plain_kernel},
            "complex128_tiled": {**summarize(stt, mst), "fidelity": tiled_fid, "max_amp_err": tiled_err},
            "speedup_c64_vs_plain": ms128 / ms,
        },
        "roofline": {"bound": "hbm", "kernel": dom[0], "achieved": dom_achieved, "peak": peak, "unit": "GB/s",
                     "frac": dom_achieved / peak, "peak_kind": peak_kind, "traffic": None},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches * args.steps,
        "clocks": clocks.summary(),
    }
    if rank == 0:
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
