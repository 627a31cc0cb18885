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


from .qasm import ImportedCircuit, QASMImportError, from_qiskit, load_qasm, parse_qasm  # noqa: E402

__all__ += ["ImportedCircuit", "QASMImportError", "from_qiskit", "load_qasm", "parse_qasm"]
