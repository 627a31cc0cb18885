"""Benchmark: 30-qubit depth-40 random brickwork, plain complex128 vs the fused complex64 form.

One step = one full circuit on one GPU: |0...0>, every compiled operation,
FP64 terminal probabilities, CDF and 10^5 seeded samples, with the circuit
plan and state buffers resident in HBM (dq_plan_*).  Each form is timed with
CUDA events on the engine's stream.  The 16 GiB / 8 GiB state is far larger
than the 126 MB L2, so no flush is needed between steps.

`value` is the circuit time of the chosen complex64 form (fused 5-qubit blocks
on tcgen05 tensor cores; seconds per circuit; for N GPUs, replicas: N circuits
/ max-over-ranks time, reported as seconds per circuit).  The plain complex128
per-gate form (its per-pass HBM fraction), complex128 shared-memory tiles,
complex64 CUDA-core tiles, the algorithmic GB/s of each and every complex64
state's fidelity / max amplitude error against the plain run are reported
beside it.  The roofline is the fused kernel's tensor-pipe throughput (f16
FLOPs it issues: three 128x64x64 products per block and tile).

--impl reference times the CPU restatement of the reference's engine
(oracle/, OpenMP on every host core) on complete circuits: every step is one
whole simulate_shots call at 30 qubits (all operations, the FP64 marginal
table and CDF, 10^5 seeded draws), nothing extrapolated.  One such circuit
takes minutes, so the arm runs as many complete circuits as fit its wall-time
budget (at least one, at most --steps, no warm-up: the reference allocates
and first-touches a fresh state inside every call) and reports the count it
ran.  It loads the circuit generators from their file alone, never the
engine's library.

--workload selects the other measured configurations (their own JSON line):
qft (32-qubit QFT, complex64 fused vs complex128 plain), batch (512 uneven HEA
circuits in one persistent launch vs a per-circuit complex128 loop) and
learned (cost model trained on recorded timings; learned vs greedy plans on
held-out 26/30/33-qubit brickwork).
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

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "classical-quantum-sim-optimizer_b200"
for _p in (str(PKG), str(ROOT)):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "30q circuit time & HBM GB/s: fused FP32 vs plain FP64 at fidelity≥1−1e-6"
FALLBACK_HBM = 6650.0
FALLBACK_TFLOPS = 1590.0


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", FALLBACK_HBM)), "measured"
    return FALLBACK_HBM, "fallback"


def tensor_peak():
    """Dense f16/bf16 tensor peak (TFLOP/s): the measured burst cuBLAS bf16 figure."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "measured"
    return FALLBACK_TFLOPS, FALLBACK_TFLOPS, "fallback"


# f16 tensor FLOPs one fused block issues per 4096-amplitude tile: hi*hi, hi*lo
# and lo*hi products of the 128 x 64 operand with the 64 x 64 real gate image.
FUSED_FLOPS_PER_TILE_BLOCK = 3 * 2 * 128 * 64 * 64
# DRAM bytes (read + write) per tile of one k_fused launch, from the ncu capture
# of the first pass of the 28-qubit depth-40 brickwork (2 GiB complex64 state,
# 16x the L2): 2.147771 GB read + 2.088167 GB written over 2^16 tiles.  Traffic
# grows with the tiles, so a 30-qubit launch moves 2^18 times this.
FUSED_TRAFFIC_PER_TILE = (2.147771e9 + 2.088167e9) / 65536


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

        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:  # host-only ranks (the multi-rank logic tested on CPU)
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, local, value):
    if pg is None:
        return value
    import torch

    device = f"cuda:{local}" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, local, value):
    if pg is None:
        return value
    import torch

    device = f"cuda:{local}" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def time_form(dqsim, circuit, precision, local, steps, warmup, shots, seed, execution="auto", **kw):
    sim = dqsim.StatevectorSimulator(seed=seed, max_memory_mb=1 << 20, precision=precision, device=local,
                                     execution=execution, **kw)
    plan = dqsim._core.PreparedCircuit(sim, circuit, shots=shots)
    for _ in range(warmup):
        plan.run()
    return sim, plan


def load_workloads():
    """The seeded circuit generators, loaded from their file alone (importing the dqsim package would load
    the engine's library into the CPU-only arms)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("dqsim_workloads", PKG / "dqsim" / "workloads.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cpu_budget_mb(n):
    """max_memory_mb for terminal sampling on the CPU restatement: state (16 B per amplitude) plus the
    FP64 CDF, shots.rs:118-124."""
    return ((16 << n) + (8 << n)) // (1 << 20) + 64


def cpu_reference_sample(circuit, budget_s, shots, seed):
    """Bounded CPU baseline at full size: the first operations of the circuit timed one by one on a fresh
    state (the first includes first-touching it), the rest estimated from the timed ones' per-kind means,
    and the marginal table, CDF and seeded draws timed in full."""
    from oracle import oracle

    L = oracle.lib()
    n, _, ops = oracle.circuit_ops(circuit.model_dump_json())
    prefix_end = next((i for i, op in enumerate(ops) if not oracle.is_unitary(op)), len(ops))
    unitary = ops[:prefix_end]
    qubits = sorted({op[1] for op in ops[prefix_end:]}, reverse=True)

    def kind(op):
        return f"{op[0]}{len(op[3]) if op[0] == 'one' else len(op[2]) if op[0] == 'x' else ''}"

    t_start = time.perf_counter()
    state = oracle.zero_state(n)
    rng = oracle.ChaCha8Stream(seed)
    per_kind, first_s, done = {}, 0.0, 0
    while done < len(unitary) and (done < 2 or time.perf_counter() - t_start < budget_s):
        t0 = time.perf_counter()
        oracle.apply_op(unitary[done], state, n, [], rng, True)
        dt = time.perf_counter() - t0
        if done == 0:
            first_s = dt
        else:
            per_kind.setdefault(kind(unitary[done]), []).append(dt)
        done += 1
    timed_s = first_s + sum(sum(v) for v in per_kind.values())
    all_mean = sum(sum(v) for v in per_kind.values()) / max(1, sum(len(v) for v in per_kind.values()))
    rest_s = 0.0
    for op in unitary[done:]:
        v = per_kind.get(kind(op))
        rest_s += statistics.mean(v) if v else all_mean
    t0 = time.perf_counter()
    cdf = oracle.cdf_from_probs(oracle.marginal_probs(state, n, qubits))
    del state
    draws = oracle.first_draws(seed, shots)
    idx = np.minimum(np.searchsorted(cdf, draws, side="right"), len(cdf) - 1)
    np.unique(idx, return_counts=True)
    sample_s = time.perf_counter() - t0
    del cdf
    return {"circuit_s": timed_s + rest_s + sample_s, "ops_timed": done, "ops_total": len(unitary),
            "sampling_s": sample_s, "threads": L.orc_num_threads(), "qubits": n,
            "per_kind_ms": {k: 1e3 * statistics.mean(v) for k, v in per_kind.items()}}


def run_reference(args):
    """The reference arm: complete 30-qubit circuits through the CPU restatement's simulate_shots."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import oracle

    circuit = load_workloads().brickwork(args.qubits, args.depth, seed=args.seed, measure=True)
    threads = oracle.lib().orc_num_threads()
    sim = oracle.OracleSimulator(seed=args.seed, max_memory_mb=cpu_budget_mb(args.qubits))
    times = []
    t_start = time.perf_counter()
    while len(times) < max(1, args.steps):
        t0 = time.perf_counter()
        out = sim.simulate_shots_full(circuit, shots=args.shots)
        times.append(time.perf_counter() - t0)
        if out["strategy"] != "terminal_sampling" or sum(out["counts"].values()) != args.shots:
            raise RuntimeError("the CPU restatement did not sample the circuit terminally")
        if time.perf_counter() - t_start + 1.1 * max(times) > args.ref_budget:
            break
    value = statistics.mean(times)
    sample = (f"full circuit: every one of the circuit's operations at {args.qubits} qubits, the FP64 marginal "
              f"table and CDF and {args.shots} seeded draws per step (simulate_shots of the C restatement of "
              f"src/engine.rs + shots.rs), {len(times)} complete circuit(s) timed, no extrapolation")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "higher_is_better": False,
        "n_gpus": world, "steps": len(times), "warmup": 0, "ms_per_step": value * 1e3,
        "requested": {"steps": args.steps, "warmup": args.warmup,
                      "why": "one complete CPU circuit takes minutes; as many as fit the arm's budget are run"},
        "runs_s": times, "scaling": "weak", "vs_baseline": None, "dtype": "c128 (f64)", "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def workload_config(args):
    return {"workload": f"brickwork-{args.qubits}q-d{args.depth}-seed{args.seed}-{args.shots}shots",
            "qubits": args.qubits, "depth": args.depth, "shots": args.shots, "seed": args.seed,
            "parallelism": "replicas", "l2": "state (16 GiB c128 / 8 GiB c64) exceeds L2; no flush"}


def bytes_of(stats):
    return sum(v["bytes"] for k, v in stats.items() if k != "sample")


def summarize(stats, ms_, peak):
    gbs = bytes_of(stats) / (ms_ * 1e-3) / 1e9
    return {"s": ms_ * 1e-3, "gbs": gbs, "frac_of_hbm": gbs / peak, "kernels": stats}


def fused_roofline(plan, stats, n):
    """Tensor-pipe roofline of the fused kernel class from the plan's block count."""
    fused = stats.get("fused")
    if not fused or fused["ms"] <= 0:
        return None
    tiles = 1 << (n - 12)
    flops = tiles * plan.shape()["fused_blocks"] * FUSED_FLOPS_PER_TILE_BLOCK
    burst, sustained, kind = tensor_peak()
    achieved = flops / (fused["ms"] * 1e-3) / 1e12
    return {"bound": "tensor", "kernel": "k_fused (tcgen05 kind::f16)", "achieved": achieved, "peak": burst,
            "unit": "TFLOP/s", "frac": achieved / burst, "frac_of_sustained": achieved / sustained,
            "peak_kind": kind, "flops": flops, "launches": fused["launches"],
            "hbm_gbs": fused["bytes"] / (fused["ms"] * 1e-3) / 1e9,
            "traffic": FUSED_TRAFFIC_PER_TILE * tiles, "traffic_unit": "bytes per launch (scaled from 28 qubits)",
            "algorithmic_bytes_per_launch": 16.0 * tiles * 4096}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="brickwork", choices=["brickwork", "qft", "batch", "learned", "cases"])
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--depth", type=int, default=40)
    ap.add_argument("--shots", type=int, default=100000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of timed CPU operations (cpu_baseline)")
    ap.add_argument("--ref-budget", type=float, default=900.0,
                    help="wall seconds the reference arm may spend on complete circuits (at least one runs)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--forms", default="fused,c64_cuda_core,c128_tiled,c128_per_gate",
                    help="forms timed beside the fused one (profiling runs time the fused form alone)")
    ap.add_argument("--plain-steps", type=int, default=1)
    ap.add_argument("--learned-rows", default="",
                    help="--workload learned: train on these recorded pass rows (.npz) instead of recording anew")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "brickwork":
        return {"qft": run_qft, "batch": run_batch, "learned": run_learned, "cases": run_cases}[args.workload](args)

    world, rank, local, pg = dist_setup(args)
    import dqsim

    peak, peak_kind = peaks()
    circuit = dqsim.workloads.brickwork(args.qubits, args.depth, seed=args.seed, measure=True)

    forms = set(args.forms.split(","))
    unknown = forms - {"fused", "c64_cuda_core", "c128_tiled", "c128_per_gate"}
    if unknown or "fused" not in forms:
        raise SystemExit(f"--forms: the fused form is required; unknown forms {sorted(unknown)}")
    out_forms = {}
    plan128 = sim128 = None

    # Plain complex128 form: the reference's arithmetic, one HBM pass per operation.
    if "c128_per_gate" in forms:
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
        out_forms["complex128_per_gate"] = {**summarize(st128, ms128, peak), "dominant": plain_kernel}

    def compare_plain(plan):
        return plan.compare(plan128) if plan128 is not None else (None, None)

    # complex128 with shared-memory tile passes (same FP64 arithmetic, fused 4x4 within a pass).
    if "c128_tiled" in forms:
        simt, plant = time_form(dqsim, circuit, "complex128", local, 1, 1, args.shots, args.seed)
        tt = [plant.run() for _ in range(args.plain_steps)]
        plant.run(record=True)
        stt = plant.stats()
        mst = statistics.mean(tt)
        tiled_fid, tiled_err = compare_plain(plant)
        out_forms["complex128_tiled"] = {**summarize(stt, mst, peak), "fidelity": tiled_fid,
                                         "max_amp_err": tiled_err}
        tile = stt.get("tile")
        if tile and tile["ms"] > 0:
            # FP64 roofline of the tile kernel: its arithmetic over the device's FP64 FMA rate
            # (measured by the library's own kernel).
            fl = plant.flops()["cuda_core"]
            fp64 = dqsim._core.device_fp64_tflops(local)
            ach = fl / (tile["ms"] * 1e-3) / 1e12
            out_forms["complex128_tiled"]["fp64_roofline"] = {
                "kernel": "k_tile_phased_arg<double2> (register phases)", "bound": "fp64", "achieved": ach,
                "peak": fp64, "unit": "TFLOP/s",
                "frac": ach / fp64, "peak_kind": "measured (dq_device_fp64_tflops)", "flops": fl,
                "launches": tile["launches"]}
        del plant, simt

    # complex64 on CUDA cores (13-qubit tiles, width-2 fusion).
    if "c64_cuda_core" in forms:
        simc, planc = time_form(dqsim, circuit, "complex64", local, 1, 1, args.shots, args.seed,
                                tile_qubits=13, fusion_width=2)
        tc = [planc.run() for _ in range(args.plain_steps)]
        planc.run(record=True)
        stc = planc.stats()
        msc = statistics.mean(tc)
        cc_fid, cc_err = compare_plain(planc)
        out_forms["complex64_cuda_core"] = {**summarize(stc, msc, peak), "fidelity": cc_fid, "max_amp_err": cc_err}
        del planc, simc

    # The chosen form: complex64 with fused 5-qubit blocks on tensor cores.
    sim64, plan64 = time_form(dqsim, circuit, "complex64", local, 1, args.warmup, args.shots, args.seed)
    barrier(pg)
    with ClockSampler(local) as clocks:
        times = [plan64.run() for _ in range(args.steps)]
    barrier(pg)
    ms = max_over_ranks(pg, local, statistics.mean(times))
    plan64.run(record=True)
    st64 = plan64.stats()
    fidelity, max_err = compare_plain(plan64)
    shape64 = plan64.shape()
    roof = fused_roofline(plan64, st64, args.qubits)
    out_forms["complex64_fused"] = {**summarize(st64, ms, peak), "fidelity": fidelity, "max_amp_err": max_err,
                                    "passes": shape64["passes"], "fused_blocks": shape64["fused_blocks"]}
    if "complex128_per_gate" in out_forms:
        out_forms["speedup_fused_vs_plain"] = out_forms["complex128_per_gate"]["s"] * 1e3 / ms
    if "complex64_cuda_core" in out_forms:
        out_forms["speedup_fused_vs_c64_cuda_core"] = out_forms["complex64_cuda_core"]["s"] * 1e3 / ms
    del plan128, sim128

    # End to end through the public API: host JSON in, host counts out.  Five calls after the same warm-up
    # count as the device timing (the first calls also fill the engine's memory pool); every call is
    # reported with its host phase times.
    e2e = None
    if not args.no_e2e:
        api = dqsim.StatevectorSimulator(seed=args.seed, max_memory_mb=1 << 20, precision="complex64",
                                         device=local)
        warm_runs, warm_phases = [], []
        for _ in range(max(1, args.warmup)):
            t0 = time.perf_counter()
            api.simulate_shots(circuit, shots=args.shots)
            warm_runs.append(time.perf_counter() - t0)
            warm_phases.append({**{k: round(v * 1e3, 3) for k, v in dqsim._core.last_call_phases(api).items()},
                                "free_gb": round(dqsim._core.device_memory(local)["free"] / 1e9, 2)})
        e2e_runs, e2e_phases = [], []
        for _ in range(5):
            t0 = time.perf_counter()
            counts = api.simulate_shots(circuit, shots=args.shots)
            e2e_runs.append(time.perf_counter() - t0)
            e2e_phases.append({**{k: round(v * 1e3, 3) for k, v in dqsim._core.last_call_phases(api).items()},
                               "free_gb": round(dqsim._core.device_memory(local)["free"] / 1e9, 2)})
            assert sum(counts.values()) == args.shots
        e2e = {"value": statistics.median(e2e_runs), "unit": "s",
               "h2d_bytes_per_step": len(circuit.model_dump_json()), "d2h_bytes_per_step": 8 * args.shots,
               "runs_s": e2e_runs, "mean_s": statistics.mean(e2e_runs), "max_s": max(e2e_runs),
               "phases_ms": e2e_phases, "warmup_runs_s": warm_runs, "warmup_phases_ms": warm_phases}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        info = cpu_reference_sample(circuit, args.cpu_budget, args.shots, args.seed)
        cpu = {"value": info["circuit_s"], "unit": "s", "cores": info["threads"], "kind": "port",
               "sample": f"first {info['ops_timed']} of {info['ops_total']} operations at {info['qubits']} qubits "
                         f"timed on a fresh state, the rest estimated from their per-kind means "
                         f"({info['per_kind_ms']} ms), marginal table, CDF and {args.shots} draws timed in full "
                         f"({info['sampling_s']:.2f} s); OpenMP C restatement of src/engine.rs + shots.rs"}

    value = (ms * 1e-3) / world
    # Every kernel of a step: the recorded classes plus the basis-state initialisation.
    launches = sum(v["launches"] for k, v in st64.items()) + 1
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64 (f16x3 tensor products, f32 accumulate, FP64 reductions)",
        "data": "synthetic", "config": workload_config(args),
        "forms": out_forms,
        "roofline": roof,
        "hbm_peak": {"value": peak, "kind": peak_kind},
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


def run_qft(args):
    """32-qubit QFT: complex64 fused (32 GiB) vs complex128 per-gate (64 GiB), time and fidelity."""
    import dqsim

    n = args.qubits if args.qubits != 30 else 32
    circuit = dqsim.workloads.qft(n, seed=args.seed)
    _, plan128 = time_form(dqsim, circuit, "complex128", 0, 1, 0, 0, args.seed, execution="per_gate")
    t128 = [plan128.run() for _ in range(max(1, args.plain_steps))]
    sim64, plan64 = time_form(dqsim, circuit, "complex64", 0, 1, 1, 0, args.seed)
    t64 = [plan64.run() for _ in range(args.steps)]
    plan64.run(record=True)
    st64 = plan64.stats()
    fid, err = plan64.compare(plan128)
    print(json.dumps({"workload": f"qft-{n}q-seed{args.seed}", "complex64_fused_s": statistics.mean(t64) * 1e-3,
                      "complex128_per_gate_s": statistics.mean(t128) * 1e-3,
                      "speedup": statistics.mean(t128) / statistics.mean(t64), "fidelity": fid, "max_amp_err": err,
                      "shape": plan64.shape(), "roofline": fused_roofline(plan64, st64, n),
                      "state_gib": {"complex64": (8 << n) / 2 ** 30, "complex128": (16 << n) / 2 ** 30}}))
    return 0


def run_batch(args):
    """512 uneven HEA circuits (12..22 qubits, depth 4..16), 1024 shots and <Z0 Z1> each, in one CUDA graph
    (autotuned per qubit count: persistent tile kernel or tensor-core fused passes on side streams), vs a
    per-circuit complex128 per-gate loop on the device and the CPU restatement on a sample of the circuits.
    With N ranks every rank runs its longest-processing-time share of the circuits on its own GPU (no
    data-path collective); the batch time is the maximum over ranks and <Z0 Z1> merges in one all-reduce."""
    import dqsim
    from dqsim import sharding
    from oracle import oracle

    world, rank, local, pg = dist_setup(args)
    peak, peak_kind = peaks()
    all_circuits = dqsim.workloads.hea_batch(512, seed=args.seed)
    mine, circuits = sharding.shard(all_circuits, world, rank)
    sim = dqsim.StatevectorSimulator(seed=args.seed, precision="complex64", max_memory_mb=1 << 16, device=local)
    t0 = time.perf_counter()
    batch = dqsim._core.BatchedCircuits(sim, circuits, shots=1024, autotune=True)
    setup_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        batch.run()
    barrier(pg)
    ms = [batch.run() for _ in range(args.steps)]
    zz = batch.expect_zz()
    work = batch.work()
    batch_ms = max_over_ranks(pg, local, statistics.mean(ms))
    zz_all = sharding.merge_values(pg, mine, zz, len(all_circuits),
                                   device=f"cuda:{local}" if pg is not None and pg.get_backend() == "nccl" else "cpu")
    work = {k: (sum_over_ranks(pg, local, v) if k != "fused_circuits" else int(sum_over_ranks(pg, local, v)))
            for k, v in work.items()}
    burst, _, tkind = tensor_peak()
    roof = {"bound": "hbm", "achieved": work["bytes"] / (batch_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
            "peak_kind": peak_kind, "algorithmic_bytes": work["bytes"],
            "tensor_tflops": work["tensor_flops"] / (batch_ms * 1e-3) / 1e12, "tensor_peak": burst,
            "cuda_core_tflops": work["cuda_core_flops"] / (batch_ms * 1e-3) / 1e12}
    roof["frac"] = roof["achieved"] / (peak * world)  # whole-job rates against N GPUs' peaks
    roof["tensor_frac"] = roof["tensor_tflops"] / (burst * world)
    sim128 = dqsim.StatevectorSimulator(seed=args.seed, precision="complex128", max_memory_mb=1 << 16,
                                        execution="per_gate", device=local)
    loop_ms, zz_err = 0.0, 0.0
    t1 = time.perf_counter()
    for i, c in enumerate(circuits):
        plan = dqsim._core.PreparedCircuit(sim128, c, shots=1024)
        loop_ms += plan.run()
        if i < 16:  # <Z0 Z1> of the complex128 state for a spot check
            sv = plan.statevector()
            p = np.abs(sv) ** 2
            idx = np.arange(p.shape[0])
            sign = 1 - 2 * (((idx >> 0) & 1) ^ ((idx >> 1) & 1))
            zz_err = max(zz_err, abs(float(np.dot(p, sign)) - float(zz[i])))
        del plan
    loop_wall = time.perf_counter() - t1
    loop_ms = max_over_ranks(pg, local, loop_ms)
    zz_err = max_over_ranks(pg, local, zz_err)
    cpu = None
    if world == 1 and not args.no_cpu:
        # CPU restatement on a bounded sample: whole simulate_shots calls on circuits taken in a seeded order
        # until the budget is spent, scaled to the batch by amplitude-operations (2^n x gates per circuit).
        rng = np.random.default_rng(args.seed)
        order = rng.permutation(len(circuits))
        weight = [sharding.circuit_weight(c) for c in circuits]
        cpu_s, cpu_w, done = 0.0, 0, 0
        osim = oracle.OracleSimulator(seed=args.seed, max_memory_mb=1 << 16)
        t2 = time.perf_counter()
        for i in order:
            if time.perf_counter() - t2 > args.cpu_budget and done >= 4:
                break
            t3 = time.perf_counter()
            osim.simulate_shots(circuits[int(i)], shots=1024)
            cpu_s += time.perf_counter() - t3
            cpu_w += weight[int(i)]
            done += 1
        cpu = {"value": cpu_s * sum(weight) / cpu_w, "unit": "s", "cores": oracle.lib().orc_num_threads(),
               "kind": "port", "sample": f"{done} of {len(circuits)} circuits through simulate_shots "
                                         f"(1024 shots) in {cpu_s:.1f} s, scaled by 2^n x gates"}
    passes = int(sum_over_ranks(pg, local, batch.passes))
    if rank == 0:
        print(json.dumps({"workload": f"hea-batch-512-seed{args.seed}", "n_gpus": world,
                          "scaling": "strong", "batch_ms": batch_ms, "runs_ms": ms,
                          "circuits_per_s": len(all_circuits) / (batch_ms * 1e-3),
                          "batch_setup_s": setup_s, "passes": passes, "work_items": batch.items,
                          "fused_circuits": work["fused_circuits"], "roofline": roof,
                          "per_circuit_c128_device_ms": loop_ms, "per_circuit_c128_wall_s": loop_wall,
                          "speedup_device": loop_ms / batch_ms, "zz_max_err_first16": zz_err,
                          "zz_checksum": sum(zz_all), "cpu_baseline": cpu}))
    if pg is not None:
        pg.destroy_process_group()
    return 0


def run_cases(args):
    """The reference's own statevector benchmark cases (benchmarks/statevector_benchmark.py:60-90):
    median of 5 wall-clock repeats after one warm-up, through the public API, on the GPU engine
    (complex128, the reference's precision) and on the CPU restatement with every host thread."""
    import dqsim
    from oracle import oracle

    cases = dqsim.workloads.benchmark_cases()

    def timed(make_sim):
        sim = make_sim()
        out = {}
        for name, (circuit, shots) in cases.items():
            if name == "full_probabilities_14q":
                res = sim.simulate(circuit)
                call = res.probabilities
            elif shots is not None:
                call = lambda c=circuit, k=shots: sim.simulate_shots(c, shots=k)
            else:
                call = lambda c=circuit: sim.simulate(c)
            call()
            times = []
            for _ in range(5):
                t0 = time.perf_counter()
                r = call()
                times.append(time.perf_counter() - t0)
                if shots is not None:
                    assert sum(r.values()) == shots
                elif name == "full_probabilities_14q":
                    assert abs(sum(r.values()) - 1) < 1e-10
            out[name] = statistics.median(times)
        return out

    gpu = timed(lambda: dqsim.StatevectorSimulator(seed=71))
    cpu = timed(lambda: oracle.OracleSimulator(seed=71))
    print(json.dumps({"workload": "reference-statevector-benchmark-cases", "unit": "s (median of 5)",
                      "gpu_complex128": gpu, "cpu_restatement": cpu,
                      "cpu_threads": oracle.lib().orc_num_threads()}))
    return 0


def run_learned(args):
    """Learned fused-pass cost model: trained on the device on passes this engine times itself (seeded random
    passes at 24-32 qubits and every distinct pass of the candidate plans of brickwork and QFT circuits of
    24-30 qubits), then, on held-out circuits (depth-40 brickwork at 26, 30 and 33 qubits, QFT at 32), the plan
    it picks against the hand rule's: each prepared circuit A/B-times the two and keeps the faster."""
    import dqsim
    from dqsim import _core, pass_costs

    t0 = time.perf_counter()
    if args.learned_rows:
        # Rows this engine recorded earlier (tests/golden/make_fused_pass_costs.py writes them).
        rows = dict(np.load(args.learned_rows))
    else:
        rec = dqsim.StatevectorSimulator(seed=1, precision="complex64", max_memory_mb=1 << 20)
        rows = pass_costs.record(rec, seed=args.seed)
        del rec
    record_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    model, mse = pass_costs.train(rows, seed=args.seed)
    train_s = time.perf_counter() - t0
    results = []
    for kind, n, seed in pass_costs.HELD_OUT:
        circuit = pass_costs.circuit(kind, n, seed)
        sim = dqsim.StatevectorSimulator(seed=1, precision="complex64", max_memory_mb=1 << 20)
        _core.set_cost_model(sim, model)
        learned = _core.PreparedCircuit(sim, circuit)
        info = learned.planner()
        log = _core.planner_log(sim)[-1]
        greedy = _core.PreparedCircuit(dqsim.StatevectorSimulator(seed=1, precision="complex64",
                                                                  max_memory_mb=1 << 20), circuit)
        tl = min(learned.run() for _ in range(3))
        tg = min(greedy.run() for _ in range(3))
        fid, err = learned.compare(greedy)
        seg = log["fused_plans"][0] if log.get("fused_plans") else {}
        results.append({"circuit": f"{kind}-{n}q-seed{seed}", "greedy_ms": tg, "kept_ms": tl, "gain": tg / tl,
                        "ab_greedy_ms": info["greedy_ms"], "ab_learned_ms": info["learned_ms"],
                        "rejected": info["rejected"], "rule_choice": seg.get("rule_choice"),
                        "model_choice": seg.get("chosen"), "candidates": seg.get("candidates"),
                        "fidelity_vs_greedy": fid, "max_amp_err_vs_greedy": err})
        _core.set_cost_model(sim, None)
        del learned, greedy
    print(json.dumps({"workload": "learned-fused-planner-vs-hand-rule", "samples": int(len(rows["ms"])),
                      "rows_from": args.learned_rows or "recorded in this run",
                      "record_s": record_s, "train_s": train_s, "train_mse": mse, "results": results,
                      "rejection_rate": sum(r["rejected"] for r in results) / len(results)}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
