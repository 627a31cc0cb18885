"""Device backend entries of the reference's timing collector (dqsim.collector).

The reference's collector (scripts/collect_simulator_data.py:40-71) and
resource preflight (ml/circuit.py:201-217) are mirrored with the device
backends added; the host logic is checked here without a device (a fake
simulator stands in, as the reference's collector tests fake their workers),
and one GPU test times a real circuit through `measure`.
"""

import pytest

from helpers import Circuit, inst

from dqsim import collector

SETTINGS = dict(seed=7, max_memory_mb=1024, parallel_shots=None, warmups=1, repeats=3, shots=64)


def test_options_for_keeps_the_reference_options_and_adds_precision():
    assert collector.options_for("statevector", SETTINGS) == dict(seed=7, max_memory_mb=1024, max_parallel_shots=None,
                                                                  sample_terminal=True)
    assert collector.options_for("mps", SETTINGS)["max_bond_dimension"] is None
    assert collector.options_for("pblock", SETTINGS)["split_separable"] is False
    gpu = collector.options_for("statevector_gpu", dict(SETTINGS, device=1))
    assert gpu["precision"] == "complex128" and gpu["device"] == 1 and gpu["sample_terminal"] is True
    assert collector.options_for("statevector_gpu_c64", SETTINGS)["precision"] == "complex64"
    with pytest.raises(ValueError):
        collector.options_for("qasm", SETTINGS)


def test_preflight_by_bytes_per_amplitude_and_device_memory():
    s = dict(SETTINGS, max_memory_mb=1024)  # 2^30 bytes
    # complex128: a state of 2^(n+4) bytes passes while n + 4 stays below the budget's bit length
    # (the reference's rule: 26 qubits fill the 1 GiB budget exactly, 27 do not fit)
    assert collector.resource_preflight("statevector", 26, s) is None
    assert collector.resource_preflight("statevector", 27, s)["status"] == "resource_exceeded"
    assert collector.resource_preflight("statevector_gpu", 27, s, device_total_bytes=1 << 40)["stage"] == "preflight"
    # complex64 needs half: one more qubit fits
    assert collector.resource_preflight("statevector_gpu_c64", 27, s, device_total_bytes=1 << 40) is None
    assert collector.resource_preflight("statevector_gpu_c64", 28, s, device_total_bytes=1 << 40) is not None
    big = dict(SETTINGS, max_memory_mb=1 << 30)
    b200 = 183_359 * 1024 ** 2  # one B200's memory
    r = collector.resource_preflight("statevector_gpu", 34, big, device_total_bytes=b200)  # 256 GiB
    assert r is not None and "device" in r["reason"]
    assert collector.resource_preflight("statevector_gpu", 33, big, device_total_bytes=b200) is None  # 128 GiB
    assert collector.resource_preflight("statevector_gpu_c64", 34, big, device_total_bytes=b200) is None
    assert collector.resource_preflight("mps", 200, s) is None  # compact backends are never rejected


class FakeSimulator:
    def __init__(self):
        self.calls = 0

    def simulate_shots(self, circuit, shots):
        self.calls += 1
        return {"0": shots}


def test_measure_times_warmups_then_repeats():
    sim = FakeSimulator()
    out = collector.measure(sim, object(), "shots", SETTINGS)
    assert sim.calls == 4 and len(out["samples_seconds"]) == 3
    assert out["min_seconds"] <= out["median_seconds"] <= out["max_seconds"]


@pytest.mark.gpu
def test_measure_a_circuit_on_each_device_backend():
    c = Circuit(14, [inst("h", qubit=q) for q in range(14)] + [inst("measure", qubit=q, cbit=q) for q in range(14)],
                cbits=14)
    for backend in ("statevector_gpu", "statevector_gpu_c64"):
        assert collector.resource_preflight(backend, 14, SETTINGS) is None
        sim = collector.simulator_class(backend)(**collector.options_for(backend, SETTINGS))
        out = collector.measure(sim, c, "shots", SETTINGS)
        assert len(out["samples_seconds"]) == 3 and out["median_seconds"] > 0
