"""GPU backend entries for the reference's timing collector.

The reference collects backend timings for its selector with
scripts/collect_simulator_data.py: `options_for` (:40-50) builds a backend's
constructor options from the run settings, `measure` (:52-71) times the public
API (warm-ups, then repeats; loading, construction and checks untimed), and
`resource_preflight` (ml/circuit.py:201-217) rejects a dense state that cannot
fit before any work, assuming 16 bytes per amplitude of host memory.  These
functions keep those signatures and semantics and add the device backends, so
a collector can label circuits with them:

  statevector_gpu      complex128 on the device (the reference's precision),
  statevector_gpu_c64  complex64 with fused tensor-core blocks and FP64
                       reductions.

For the device backends `max_memory_mb` budgets device memory, and the
preflight also rejects a state that exceeds the device's total memory.
"""

import statistics
import struct
import time

from . import _core

GPU_BACKENDS = {"statevector_gpu": "complex128", "statevector_gpu_c64": "complex64"}
BACKENDS = ("statevector", "mps", "pblock", "stabilizer") + tuple(GPU_BACKENDS)
BYTES_PER_AMPLITUDE = {"statevector": 16, "statevector_gpu": 16, "statevector_gpu_c64": 8}


def options_for(backend, settings):
    """Constructor options of a backend from the collector's settings (collect_simulator_data.py:40-50)."""
    if backend not in BACKENDS:
        raise ValueError(f"unknown backend {backend!r}")
    options = dict(seed=settings["seed"], max_memory_mb=settings["max_memory_mb"],
                   max_parallel_shots=settings["parallel_shots"], sample_terminal=True)
    if backend == "mps":
        options.update(max_bond_dimension=None, truncation_threshold=0.0, max_discarded_weight=0.0)
    elif backend == "pblock":
        options.update(split_separable=False)
    elif backend == "stabilizer":
        options.update(clifford_tolerance=0.0)
    elif backend in GPU_BACKENDS:
        options.update(precision=GPU_BACKENDS[backend], device=int(settings.get("device", 0)))
    return options


def simulator_class(backend):
    """The simulator class a backend name selects (the device backends share StatevectorSimulator)."""
    if backend not in BACKENDS:
        raise ValueError(f"unknown backend {backend!r}")
    return {"statevector": _core.StatevectorSimulator, "mps": _core.MpsSimulator, "pblock": _core.PBlockSimulator,
            "stabilizer": _core.StabilizerSimulator}.get(backend, _core.StatevectorSimulator)


def measure(simulator, circuit, task, settings):
    """Times the public API only (collect_simulator_data.py:52-71): warm-ups, then timed repeats."""
    samples = []
    for iteration in range(settings["warmups"] + settings["repeats"]):
        start = time.perf_counter_ns()
        if task == "shots":
            result = simulator.simulate_shots(circuit, shots=settings["shots"])
        else:
            result = simulator.simulate(circuit)
        elapsed = (time.perf_counter_ns() - start) / 1e9
        if task == "shots" and sum(result.values()) != settings["shots"]:
            raise RuntimeError("Returned shot count does not match the requested count")
        if task == "evolve" and result.num_qubits != circuit.num_qubits:
            raise RuntimeError("Returned quantum width does not match the input")
        del result  # Do not retain quantum states or counts across repetitions.
        if iteration >= settings["warmups"]:
            samples.append(elapsed)
    return dict(samples_seconds=samples, median_seconds=statistics.median(samples),
                min_seconds=min(samples), max_seconds=max(samples),
                stdev_seconds=statistics.stdev(samples) if len(samples) > 1 else 0.0)


def resource_preflight(backend, num_qubits, settings, device_total_bytes=None):
    """Rejects only provably oversized dense states (ml/circuit.py:201-217), never compact backends.

    The dense backends need `BYTES_PER_AMPLITUDE` bytes per amplitude within max_memory_mb; a device backend
    also within the device's total memory (`device_total_bytes`, read from the device when None)."""
    if backend not in BYTES_PER_AMPLITUDE:
        return None
    budget = settings["max_memory_mb"] * 1024 ** 2
    amp_log2 = BYTES_PER_AMPLITUDE[backend].bit_length() - 1
    precision = "complex64" if amp_log2 == 3 else "complex128"
    # Workspaces cost extra; fitting this lower bound does not guarantee that execution will fit.
    if num_qubits + amp_log2 >= budget.bit_length():
        return dict(status="resource_exceeded", stage="preflight",
                    reason=f"A single {precision} statevector exceeds max_memory_mb",
                    minimum_state_bytes_power_of_two=num_qubits + amp_log2, memory_budget_bytes=budget)
    if num_qubits >= 8 * struct.calcsize("P"):
        return dict(status="resource_exceeded", stage="preflight",
                    reason="Qubit count exceeds native statevector index capacity")
    if backend in GPU_BACKENDS:
        total = device_total_bytes if device_total_bytes is not None else _core.device_memory(
            int(settings.get("device", 0)))["total"]
        if num_qubits + amp_log2 >= int(total).bit_length():
            return dict(status="resource_exceeded", stage="preflight",
                        reason=f"A single {precision} statevector exceeds the device's memory",
                        minimum_state_bytes_power_of_two=num_qubits + amp_log2, device_memory_bytes=int(total))
    return None
