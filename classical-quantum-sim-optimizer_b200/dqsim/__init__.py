"""Native quantum circuit simulators on NVIDIA B200 (dense statevector backend).

Circuit inputs expose ``model_dump_json()`` using the register/instruction
schema of the reference project (python/dqsim/__init__.py:1-41 re-exports the
same names).  The statevector simulator runs on sm_100a CUDA kernels behind
the C ABI in include/dqsim_sv.h; the other backends are named but not provided.
"""

from ._core import (
    MpsResult,
    MpsSimulator,
    PBlockResult,
    PBlockSimulator,
    SimulationProfile,
    SimulationResult,
    StabilizerResult,
    StabilizerSimulator,
    StatevectorSimulator,
    simulate_distributed,
    simulate_distributed_shots,
    simulate_monolithic,
    simulate_monolithic_shots,
)

from . import workloads  # noqa: E402  (seeded benchmark circuits)

__all__ = [
    "MpsSimulator",
    "MpsResult",
    "PBlockResult",
    "PBlockSimulator",
    "SimulationProfile",
    "SimulationResult",
    "StabilizerSimulator",
    "StabilizerResult",
    "StatevectorSimulator",
    "simulate_distributed",
    "simulate_distributed_shots",
    "simulate_monolithic",
    "simulate_monolithic_shots",
]


class QASMImportError(ValueError):
    """Raised by the OpenQASM helpers, which need Qiskit (not part of this engine)."""


class ImportedCircuit:  # pragma: no cover - placeholder for the reference's qasm transport
    def __init__(self, *args, **kwargs):
        raise NotImplementedError("OpenQASM import is not provided by the B200 statevector engine")


def from_qiskit(*args, **kwargs):
    raise NotImplementedError("OpenQASM import is not provided by the B200 statevector engine")


def load_qasm(*args, **kwargs):
    raise NotImplementedError("OpenQASM import is not provided by the B200 statevector engine")


__all__ += ["ImportedCircuit", "QASMImportError", "from_qiskit", "load_qasm"]
