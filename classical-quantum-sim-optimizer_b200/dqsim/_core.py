"""``dqsim._core`` on the B200 engine.

Python surface of the reference's PyO3 module (src/lib.rs:16-31) for the dense
statevector backend: ``StatevectorSimulator``, ``SimulationResult``,
``SimulationProfile`` and the ``simulate_monolithic[_shots]`` wrappers, with
the same signatures, defaults, result types and exception classes
(src/monolithic/statevector/simulator.rs:14-372, src/simulator.rs:14-144,
src/codecs.rs:29-64).  Every call goes through the C ABI declared in
include/dqsim_sv.h (``libdqsim_sv.so``); ctypes releases the GIL for the
duration of each call, as the reference does with ``py.allow_threads``.

The other backends of the reference (MPS, stabilizer, P-block) are not part of
this engine; their names exist and raise ``NotImplementedError``.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_LIB_NAME = "libdqsim_sv.so"
_LIB_PATH = Path(__file__).resolve().parent / _LIB_NAME

if not _LIB_PATH.exists():
    raise ImportError(
        f"{_LIB_NAME} is not built; run `make -C classical-quantum-sim-optimizer_b200/csrc` "
        "(or __graft_entry__.build()) first"
    )

_lib = ctypes.CDLL(str(_LIB_PATH))

try:  # count dictionaries built in C (dqsim/_counts.c); the same dictionaries otherwise
    from . import _counts
except ImportError:
    _counts = None

_u64 = ctypes.c_uint64
_P = ctypes.c_void_p


class _Options(ctypes.Structure):
    _fields_ = [
        ("has_seed", ctypes.c_int),
        ("seed", _u64),
        ("profile", ctypes.c_int),
        ("max_memory_mb", _u64),
        ("has_max_parallel_shots", ctypes.c_int),
        ("max_parallel_shots", _u64),
        ("sample_terminal", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("device", ctypes.c_int),
        ("execution", ctypes.c_int),
        ("tile_qubits", ctypes.c_int),
        ("fusion_width", ctypes.c_int),
    ]


class _Profile(ctypes.Structure):
    _fields_ = [
        ("apply_one_qubit_calls", _u64),
        ("apply_one_qubit_time", ctypes.c_double),
        ("apply_n_qubit_calls", _u64),
        ("apply_n_qubit_time", ctypes.c_double),
        ("measure_qubit_calls", _u64),
        ("measure_qubit_time", ctypes.c_double),
        ("total_time", ctypes.c_double),
    ]


def _sig(name, args, res=ctypes.c_int):
    f = getattr(_lib, name)
    f.argtypes = args
    f.restype = res
    return f


_last_error = _sig("dq_last_error", [], ctypes.c_char_p)
_version = _sig("dq_version", [], ctypes.c_char_p)
_sim_create = _sig("dq_sim_create", [ctypes.POINTER(_Options), ctypes.POINTER(_P)])
_sim_destroy = _sig("dq_sim_destroy", [_P], None)
_simulate_shots = _sig("dq_simulate_shots", [_P, ctypes.c_char_p, ctypes.c_size_t, _u64, ctypes.c_int,
                                             ctypes.POINTER(_P)])
_simulate = _sig("dq_simulate", [_P, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(_P)])
_counts_size = _sig("dq_counts_size", [_P, ctypes.POINTER(_u64), ctypes.POINTER(_u64)])
_counts_copy = _sig("dq_counts_copy", [_P, _P, _P])
_counts_free = _sig("dq_counts_free", [_P], None)
_res_nq = _sig("dq_result_num_qubits", [_P, ctypes.POINTER(_u64)])
_res_ncb = _sig("dq_result_num_cbits", [_P, ctypes.POINTER(_u64)])
_res_sv = _sig("dq_result_statevector", [_P, _P, _u64])
_res_cbits = _sig("dq_result_classical_bits", [_P, _P, _u64])
_res_profile = _sig("dq_result_profile", [_P, ctypes.POINTER(_Profile), ctypes.POINTER(ctypes.c_int)])
_res_probs = _sig("dq_result_probabilities", [_P, _P, ctypes.c_size_t, ctypes.c_int, _P, _u64])
_res_counts = _sig("dq_result_counts", [_P, _u64, _P, ctypes.c_size_t, ctypes.c_int, _u64, ctypes.c_int,
                                        ctypes.POINTER(_P)])
_res_fidelity = _sig("dq_result_fidelity", [_P, _P, _u64, ctypes.POINTER(ctypes.c_double)])
_res_amps = _sig("dq_result_amplitudes", [_P, _P, _u64, _P])
_res_pauli = _sig("dq_result_pauli_expectation", [_P, _u64, _u64, ctypes.POINTER(ctypes.c_double),
                                                  ctypes.POINTER(ctypes.c_double)])
_res_free = _sig("dq_result_free", [_P], None)
_compile_dump = _sig("dq_compile_dump", [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_char_p)])
_string_free = _sig("dq_string_free", [ctypes.c_void_p], None)

_ERRORS = {
    1: ValueError,
    2: MemoryError,
    3: TypeError,
    4: RuntimeError,
    5: NotImplementedError,
    6: RuntimeError,
}

PRECISIONS = {"complex128": 0, "c128": 0, "fp64": 0, "complex64": 1, "c64": 1, "fp32": 1}


def _check(status):
    if status != 0:
        msg = _last_error().decode("utf-8", "replace")
        raise _ERRORS.get(status, RuntimeError)(msg)


def _as_u64(value, name):
    """PyO3 usize/u64 extraction: ints only, in range."""
    if isinstance(value, bool) or not isinstance(value, (int, np.integer)):
        raise TypeError(f"argument '{name}': '{type(value).__name__}' object cannot be interpreted as an integer")
    value = int(value)
    if value < 0 or value > (1 << 64) - 1:
        raise OverflowError(f"argument '{name}': out of range integral type conversion attempted")
    return value


def _as_bool(value, name):
    if not isinstance(value, (bool, np.bool_)):
        raise TypeError(f"argument '{name}': '{type(value).__name__}' object cannot be converted to 'PyBool'")
    return bool(value)


def _circuit_json(circuit):
    text = circuit.model_dump_json()
    if isinstance(text, bytes):
        return text
    if not isinstance(text, str):
        raise TypeError("model_dump_json() must return a string")
    return text.encode("utf-8")


def _take_counts(handle):
    try:
        n, w = _u64(), _u64()
        _check(_counts_size(handle, ctypes.byref(n), ctypes.byref(w)))
        n, w = n.value, w.value
        keys = ctypes.create_string_buffer(max(1, n * w))
        counts = np.zeros(max(1, n), dtype=np.uint64)
        _check(_counts_copy(handle, keys, counts.ctypes.data))
        if _counts is not None:
            return _counts.build(keys.raw[:n * w], w, counts[:n].tobytes())
        text = keys.raw[:n * w].decode("ascii")
        return dict(zip([text[i:i + w] for i in range(0, n * w, w)] if w else [""] * n, counts[:n].tolist()))
    finally:
        _counts_free(handle)


def _qubit_list(qubits):
    if qubits is None:
        return None
    return [_as_u64(q, "qubits") for q in qubits]


class SimulationProfile:
    """Per-category execution counters of one trajectory (simulator.rs:43-79)."""

    __slots__ = ("apply_one_qubit_calls", "apply_one_qubit_time", "apply_n_qubit_calls", "apply_n_qubit_time",
                 "measure_qubit_calls", "measure_qubit_time", "total_time")

    def __init__(self, p):
        for name in self.__slots__:
            setattr(self, name, getattr(p, name))

    def __repr__(self):
        total = max(self.total_time, 1e-9)
        return (
            f"SimulationProfile (total: {self.total_time * 1000.0:.2f} ms)\n"
            f"  apply_one_qubit : {self.apply_one_qubit_calls:4} calls  {self.apply_one_qubit_time * 1000.0:8.2f} ms"
            f"  ({100.0 * self.apply_one_qubit_time / total:.1f}%)\n"
            f"  apply_n_qubit   : {self.apply_n_qubit_calls:4} calls  {self.apply_n_qubit_time * 1000.0:8.2f} ms"
            f"  ({100.0 * self.apply_n_qubit_time / total:.1f}%)\n"
            f"  measure_qubit   : {self.measure_qubit_calls:4} calls  {self.measure_qubit_time * 1000.0:8.2f} ms"
            f"  ({100.0 * self.measure_qubit_time / total:.1f}%)"
        )


class SimulationResult:
    """A final state held in device memory (simulator.rs:85-191)."""

    def __init__(self, handle):
        self._h = handle
        n = _u64()
        _check(_res_nq(handle, ctypes.byref(n)))
        self._n = n.value
        ncb = _u64()
        _check(_res_ncb(handle, ctypes.byref(ncb)))
        self._ncb = ncb.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _res_free(h)
            self._h = None

    @property
    def num_qubits(self):
        return self._n

    @property
    def statevector(self):
        """An independent complex128 NumPy copy of shape (2^n,)."""
        out = np.empty(1 << self._n, dtype=np.complex128)
        _check(_res_sv(self._h, out.ctypes.data_as(_P), 2 * out.shape[0]))
        return out

    @property
    def classical_bits(self):
        buf = np.zeros(max(1, self._ncb), dtype=np.uint8)
        _check(_res_cbits(self._h, buf.ctypes.data_as(_P), self._ncb))
        return {i: int(buf[i]) for i in range(self._ncb)}

    @property
    def profile(self):
        p, has = _Profile(), ctypes.c_int()
        _check(_res_profile(self._h, ctypes.byref(p), ctypes.byref(has)))
        return SimulationProfile(p) if has.value else None

    def probabilities(self, qubits=None):
        """{basis index: probability} for p > 0; qubits[0] is the output MSB."""
        qs = _qubit_list(qubits)
        k = self._n if qs is None else len(qs)
        if qs is not None:
            for i, q in enumerate(qs):
                if q >= self._n or q in qs[:i]:
                    raise ValueError("Query qubits must be distinct and within the statevector's range")
        arr = np.asarray(qs if qs is not None else [0], dtype=np.uint64)
        out = np.empty(1 << k, dtype=np.float64)
        _check(_res_probs(self._h, arr.ctypes.data_as(_P), len(qs or []), 0 if qs is None else 1,
                          out.ctypes.data_as(_P), out.shape[0]))
        nz = np.flatnonzero(out > 0.0)
        return dict(zip(nz.tolist(), out[nz].tolist()))

    def counts(self, shots=1000, qubits=None, seed=None):
        """Sample the current state; one ChaCha8 stream for all shots (engine.rs:457-507)."""
        shots = _as_u64(shots, "shots")
        qs = _qubit_list(qubits)
        arr = np.asarray(qs if qs is not None else [0], dtype=np.uint64)
        has_seed = seed is not None
        seed_v = _as_u64(seed, "seed") if has_seed else 0
        h = _P()
        _check(_res_counts(self._h, shots, arr.ctypes.data_as(_P), len(qs or []), 0 if qs is None else 1, seed_v,
                           1 if has_seed else 0, ctypes.byref(h)))
        return _take_counts(h)

    def amplitude(self, bitstring):
        """One amplitude, read on the device; the bitstring has one binary digit
        per qubit, highest qubit first.  Extra query (the reference offers it on
        MPS and P-block results, src/monolithic/mps/result.rs:114-130)."""
        if not isinstance(bitstring, str) or len(bitstring) != self._n or any(ch not in "01" for ch in bitstring):
            raise ValueError("Expected one binary digit per qubit, MSB first")
        return complex(self.amplitudes([int(bitstring, 2)])[0]) if self._n else complex(self.amplitudes([0])[0])

    def amplitudes(self, indices):
        """Amplitudes at little-endian basis indices, as a complex128 array (device gather)."""
        arr = np.ascontiguousarray(np.asarray(indices, dtype=np.uint64).ravel())
        out = np.empty(arr.shape[0], dtype=np.complex128)
        _check(_res_amps(self._h, arr.ctypes.data_as(_P), arr.shape[0], out.ctypes.data_as(_P)))
        return out

    def expectation_value(self, pauli):
        """<psi|P|psi> for a Pauli string with one of I, X, Y, Z per qubit, highest
        qubit first, reduced in FP64 on the device.  Extra query (the reference
        offers it on MPS results, src/monolithic/mps/result.rs:209-236)."""
        if not isinstance(pauli, str) or len(pauli) != self._n:
            raise ValueError("Expected one Pauli per qubit")
        x = z = 0
        for pos, ch in enumerate(pauli):
            bit = 1 << (self._n - 1 - pos)
            if ch == "X":
                x |= bit
            elif ch == "Z":
                z |= bit
            elif ch == "Y":
                x |= bit
                z |= bit
            elif ch != "I":
                raise ValueError("Pauli string must contain only I, X, Y, Z")
        re, im = ctypes.c_double(), ctypes.c_double()
        _check(_res_pauli(self._h, x, z, ctypes.byref(re), ctypes.byref(im)))
        return re.value

    def fidelity(self, other):
        """|<self|other>|^2 for a complex128 array; 0.0 on a length mismatch."""
        arr = np.asarray(other)
        if arr.dtype != np.complex128 or arr.ndim != 1:
            raise TypeError("fidelity expects a one-dimensional complex128 array")
        arr = np.ascontiguousarray(arr)
        out = ctypes.c_double()
        _check(_res_fidelity(self._h, arr.ctypes.data_as(_P), arr.shape[0], ctypes.byref(out)))
        return out.value


class StatevectorSimulator:
    """Dense statevector simulator on one B200 (simulator.rs:213-372).

    ``max_memory_mb`` bounds device working memory with the reference's
    arithmetic (state + classical buffers + terminal CDF); ``max_parallel_shots``
    bounds the trajectories one device batch runs at once.  ``precision``
    selects the plain complex128 form (default) or the fused complex64 form.
    """

    def __init__(self, seed=None, profile=False, *, max_memory_mb=1024, max_parallel_shots=None,
                 sample_terminal=True, precision="complex128", device=0, execution="auto", tile_qubits=0,
                 fusion_width=0):
        o = _Options()
        o.has_seed = 0 if seed is None else 1
        o.seed = 0 if seed is None else _as_u64(seed, "seed")
        o.profile = 1 if _as_bool(profile, "profile") else 0
        o.max_memory_mb = _as_u64(max_memory_mb, "max_memory_mb")
        o.has_max_parallel_shots = 0 if max_parallel_shots is None else 1
        o.max_parallel_shots = 0 if max_parallel_shots is None else _as_u64(max_parallel_shots, "max_parallel_shots")
        o.sample_terminal = 1 if _as_bool(sample_terminal, "sample_terminal") else 0
        key = str(precision).lower()
        if key not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(set(PRECISIONS))}")
        o.precision = PRECISIONS[key]
        o.device = int(device)
        modes = {"auto": 0, "per_gate": 1, "tiled": 2}
        if execution not in modes:
            raise ValueError("execution must be 'auto', 'per_gate' or 'tiled'")
        o.execution = modes[execution]
        o.tile_qubits = int(tile_qubits)
        o.fusion_width = int(fusion_width)
        h = _P()
        _check(_sim_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.precision = "complex64" if o.precision else "complex128"

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _sim_destroy(h)
            self._h = None

    def simulate_shots(self, circuit, shots=1000, profile=False):
        """Classical-register counts (simulator.rs:256-317)."""
        text = _circuit_json(circuit)
        shots = _as_u64(shots, "shots")
        profile = _as_bool(profile, "profile")
        h = _P()
        _check(_simulate_shots(self._h, text, len(text), shots, 1 if profile else 0, ctypes.byref(h)))
        return _take_counts(h)

    def simulate(self, circuit):
        """One trajectory; measurements collapse the returned state (simulator.rs:319-371)."""
        text = _circuit_json(circuit)
        h = _P()
        _check(_simulate(self._h, text, len(text), ctypes.byref(h)))
        return SimulationResult(h)


# ---------------------------------------------------------------------------
# Wrappers, src/simulator.rs:14-144 and src/codecs.rs:29-64
# ---------------------------------------------------------------------------
def _parse_mode(mode):
    key = str(mode).strip().lower().replace("-", "_")
    if key in ("state_vector", "statevector", "sv"):
        return "sv"
    if key in ("mps", "matrix_product_state", "stabilizer", "stab"):
        raise NotImplementedError(f"The {key!r} backend is not provided by the B200 statevector engine")
    raise ValueError(f"Unsupported monolithic simulation mode {key!r}; expected 'state_vector' or 'mps'")


_SV_OPTIONS = ("max_memory_mb", "max_parallel_shots", "sample_terminal", "precision", "device", "execution",
               "tile_qubits", "fusion_width")


def _parse_options(options):
    out = {"max_memory_mb": 1024, "max_parallel_shots": None, "sample_terminal": True}
    for key, value in options.items():
        if key not in _SV_OPTIONS:
            raise TypeError(f"Unsupported statevector option {key!r}")
        out[key] = value
    return out


def simulate_monolithic(circuit, mode="state_vector", seed=None, profile=False, **options):
    _parse_mode(mode)
    opts = _parse_options(options)
    return StatevectorSimulator(seed, profile, **opts).simulate(circuit)


def simulate_monolithic_shots(circuit, mode="state_vector", shots=1000, seed=None, profile=False, **options):
    _parse_mode(mode)
    opts = _parse_options(options)
    return StatevectorSimulator(seed, False, **opts).simulate_shots(circuit, shots, profile)


def _not_provided(name):
    def __init__(self, *args, **kwargs):
        raise NotImplementedError(f"{name} is not provided by the B200 statevector engine")

    return type(name, (), {"__init__": __init__, "__doc__": f"{name}: not provided (statevector engine only)."})


MpsSimulator = _not_provided("MpsSimulator")
MpsResult = _not_provided("MpsResult")
StabilizerSimulator = _not_provided("StabilizerSimulator")
StabilizerResult = _not_provided("StabilizerResult")
PBlockSimulator = _not_provided("PBlockSimulator")
PBlockResult = _not_provided("PBlockResult")


def simulate_distributed(distributed, mode="p_block", seed=None, profile=False, **options):
    raise NotImplementedError("The P-block backend is not provided by the B200 statevector engine")


def simulate_distributed_shots(distributed, mode="p_block", shots=1000, seed=None, profile=False, **options):
    raise NotImplementedError("The P-block backend is not provided by the B200 statevector engine")


_plan_create = _sig("dq_plan_create", [_P, ctypes.c_char_p, ctypes.c_size_t, _u64, ctypes.POINTER(_P)])
_plan_run = _sig("dq_plan_run", [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_double)])
_plan_stats = _sig("dq_plan_stats", [_P, _P, _P, _P])
_plan_info = _sig("dq_plan_info", [_P, ctypes.POINTER(_u64), ctypes.POINTER(_u64), ctypes.POINTER(ctypes.c_double)])
_plan_sv = _sig("dq_plan_statevector", [_P, _P, _u64])
_plan_samples = _sig("dq_plan_samples", [_P, _P, _u64])
_plan_free = _sig("dq_plan_free", [_P], None)
_plan_compare = _sig("dq_plan_compare", [_P, _P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)])

KERNEL_CLASSES = ("gate1q", "controlled", "diagonal", "swap", "dense", "measure", "tile", "fused", "sample", "norm")


class PreparedCircuit:
    """A circuit compiled and resident on the device, run many times (dq_plan_*)."""

    def __init__(self, simulator, circuit, shots=0):
        text = _circuit_json(circuit)
        h = _P()
        _check(_plan_create(simulator._h, text, len(text), _as_u64(shots, "shots"), ctypes.byref(h)))
        self._h = h
        self._sim = simulator
        nq, nops, sb = _u64(), _u64(), ctypes.c_double()
        _check(_plan_info(h, ctypes.byref(nq), ctypes.byref(nops), ctypes.byref(sb)))
        self.num_qubits, self.num_ops, self.state_bytes = nq.value, nops.value, sb.value
        self.shots = shots

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _plan_free(h)
            self._h = None

    def run(self, record=False):
        """Device milliseconds of one run (CUDA events on the engine stream)."""
        ms = ctypes.c_double()
        _check(_plan_run(self._h, 1 if record else 0, ctypes.byref(ms)))
        return ms.value

    def stats(self):
        n = len(KERNEL_CLASSES)
        ms = np.zeros(n)
        launches = np.zeros(n, dtype=np.uint64)
        nbytes = np.zeros(n)
        _check(_plan_stats(self._h, ms.ctypes.data_as(_P), launches.ctypes.data_as(_P), nbytes.ctypes.data_as(_P)))
        return {k: {"ms": float(ms[i]), "launches": int(launches[i]), "bytes": float(nbytes[i])}
                for i, k in enumerate(KERNEL_CLASSES) if launches[i]}

    def statevector(self):
        out = np.empty(1 << self.num_qubits, dtype=np.complex128)
        _check(_plan_sv(self._h, out.ctypes.data_as(_P), 2 * out.shape[0]))
        return out

    def samples(self):
        out = np.empty(self.shots, dtype=np.uint64)
        _check(_plan_samples(self._h, out.ctypes.data_as(_P), self.shots))
        return out

    def planner(self):
        """Learned-vs-greedy outcome of this plan (all zero when no cost model was attached)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        u, r = ctypes.c_int(), ctypes.c_int()
        _check(_plan_planner(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(u), ctypes.byref(r)))
        return {"learned_ms": a.value, "greedy_ms": b.value, "used_learned": bool(u.value), "rejected": bool(r.value)}

    def flops(self):
        """Arithmetic of one run: CUDA-core real FLOPs and tensor-core f16 FLOPs (dq_plan_flops)."""
        c, tc = ctypes.c_double(), ctypes.c_double()
        _check(_plan_flops(self._h, ctypes.byref(c), ctypes.byref(tc)))
        return {"cuda_core": c.value, "tensor": tc.value}

    def shape(self):
        p, t, f = _u64(), _u64(), _u64()
        _check(_plan_shape(self._h, ctypes.byref(p), ctypes.byref(t), ctypes.byref(f)))
        return {"passes": p.value, "tile_ops": t.value, "fused_blocks": f.value}

    def compare(self, other):
        """(fidelity |<self|other>|^2 / (<self|self> <other|other>), max amplitude error) of the two final states."""
        f, e = ctypes.c_double(), ctypes.c_double()
        _check(_plan_compare(self._h, other._h, ctypes.byref(f), ctypes.byref(e)))
        return f.value, e.value


_batch_create = _sig("dq_batch_create", [_P, _P, _P, _u64, _u64, ctypes.c_int, ctypes.POINTER(_P)])
_batch_run = _sig("dq_batch_run", [_P, ctypes.c_int, ctypes.POINTER(ctypes.c_double)])
_batch_counts = _sig("dq_batch_counts", [_P, _u64, ctypes.POINTER(_P)])
_batch_zz = _sig("dq_batch_expect_zz", [_P, _P, _u64])
_batch_sv = _sig("dq_batch_statevector", [_P, _u64, _P, _u64])
_batch_info = _sig("dq_batch_info", [_P, ctypes.POINTER(_u64), ctypes.POINTER(_u64)])
_batch_work = _sig("dq_batch_work", [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_u64)])
_batch_free = _sig("dq_batch_free", [_P], None)


class BatchedCircuits:
    """Many terminal-measurement circuits of uneven sizes in one CUDA graph (dq_batch_*): a persistent
    tile kernel, and tensor-core fused passes on side streams where the autotuner picks them.

    Seeds: circuit i samples with seed + i * 0x9E3779B97F4A7C15 (mod 2^64), shot t
    of it with ChaCha8 seed_from_u64(that + t), as a single simulate_shots call would.
    """

    def __init__(self, simulator, circuits, shots=1024, autotune=False, tensor_cores=False):
        """autotune=True times candidate shapes per qubit count (tensor-core passes among them);
        tensor_cores=True runs every complex64 circuit of 12 or more qubits as tensor-core fused passes."""
        texts = [_circuit_json(c) for c in circuits]
        self._keep = [ctypes.create_string_buffer(t, len(t)) for t in texts]
        ptrs = (ctypes.c_void_p * len(texts))(*[ctypes.cast(b, ctypes.c_void_p) for b in self._keep])
        lens = (ctypes.c_size_t * len(texts))(*[len(t) for t in texts])
        h = _P()
        _check(_batch_create(simulator._h, ctypes.cast(ptrs, _P), ctypes.cast(lens, _P), len(texts),
                             _as_u64(shots, "shots"), 2 if tensor_cores else (1 if autotune else 0),
                             ctypes.byref(h)))
        self._h = h
        self._sim = simulator
        self.size = len(texts)
        self.num_qubits = [c.num_qubits if hasattr(c, "num_qubits") else None for c in circuits]
        p, i = _u64(), _u64()
        _check(_batch_info(h, ctypes.byref(p), ctypes.byref(i)))
        self.passes, self.items = p.value, i.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _batch_free(h)
            self._h = None

    def run(self, use_graph=True):
        ms = ctypes.c_double()
        _check(_batch_run(self._h, 1 if use_graph else 0, ctypes.byref(ms)))
        return ms.value

    def counts(self, i):
        h = _P()
        _check(_batch_counts(self._h, i, ctypes.byref(h)))
        return _take_counts(h)

    def expect_zz(self):
        out = np.empty(self.size)
        _check(_batch_zz(self._h, out.ctypes.data_as(_P), self.size))
        return out

    def statevector(self, i, n):
        out = np.empty(1 << n, dtype=np.complex128)
        _check(_batch_sv(self._h, i, out.ctypes.data_as(_P), 2 * out.shape[0]))
        return out

    def work(self):
        """One run's algorithmic HBM bytes, tensor and CUDA-core FLOPs, and tensor-core circuits."""
        b, tf, cf, fc = ctypes.c_double(), ctypes.c_double(), ctypes.c_double(), _u64()
        _check(_batch_work(self._h, ctypes.byref(b), ctypes.byref(tf), ctypes.byref(cf), ctypes.byref(fc)))
        return {"bytes": b.value, "tensor_flops": tf.value, "cuda_core_flops": cf.value, "fused_circuits": fc.value}


BATCH_SEED_STRIDE = 0x9E3779B97F4A7C15

MLP_FEATURES = 16
MLP_PARAMS = 5315
_cm_create = _sig("dq_cost_model_create_kind", [ctypes.c_int, _u64, ctypes.c_int, ctypes.POINTER(_P)])
_cm_kind = _sig("dq_cost_model_kind", [_P, ctypes.POINTER(ctypes.c_int)])
_fused_portfolio = _sig("dq_fused_portfolio", [_P, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, _P,
                                               ctypes.POINTER(ctypes.c_char_p)])
_fused_random = _sig("dq_fused_random_passes", [_P, ctypes.c_int, _u64, _u64, ctypes.c_int,
                                                ctypes.POINTER(ctypes.c_char_p)])
_cm_free = _sig("dq_cost_model_free", [_P], None)
_cm_add = _sig("dq_cost_model_add_samples", [_P, _P, _P, _u64])
_cm_record = _sig("dq_cost_model_record", [_P, _P, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(_u64)])
_cm_num = _sig("dq_cost_model_num_samples", [_P, ctypes.POINTER(_u64)])
_cm_samples = _sig("dq_cost_model_samples", [_P, _P, _P, _u64])
_cm_train = _sig("dq_cost_model_train", [_P, ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_double)])
_cm_predict = _sig("dq_cost_model_predict", [_P, _P, _u64, _P])
_cm_grads = _sig("dq_cost_model_gradients", [_P, _P, _P, _u64, _P])
_cm_get = _sig("dq_cost_model_get_params", [_P, _P, _u64])
_cm_set = _sig("dq_cost_model_set_params", [_P, _P, _u64])
_sim_set_cm = _sig("dq_sim_set_cost_model", [_P, _P])
_plan_planner = _sig("dq_plan_planner", [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)])
_plan_shape = _sig("dq_plan_shape", [_P, ctypes.POINTER(_u64), ctypes.POINTER(_u64), ctypes.POINTER(_u64)])
_plan_flops = _sig("dq_plan_flops", [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)])
_sim_log = _sig("dq_sim_planner_log", [_P, ctypes.POINTER(ctypes.c_char_p)])
_sim_phases = _sig("dq_sim_last_call_phases", [_P, _P, _u64])
_fp64_tflops = _sig("dq_device_fp64_tflops", [ctypes.c_int, ctypes.POINTER(ctypes.c_double)])
_measure_noalloc = _sig("dq_measure_noalloc", [_P, ctypes.c_int, _u64, _u64, _u64, ctypes.c_int, _P, _P, _P])


def _f32(a, cols=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if cols is not None and (a.ndim != 2 or a.shape[1] != cols):
        raise ValueError(f"expected an array of shape (n, {cols})")
    return a


COST_KINDS = {"tile_ops": 0, "fused_passes": 1}


class CostModel:
    """The planner's learned cost model (dq_cost_model_*): MLP 16-64-64-1, trained on device.

    kind "tile_ops" prices CUDA-core tile operations and tensor-core blocks (it picks each pass's fusion
    width); kind "fused_passes" prices whole tensor-core passes (it picks which candidate fused plan runs).
    """

    def __init__(self, device=0, seed=0, kind="tile_ops"):
        if kind not in COST_KINDS:
            raise ValueError(f"kind must be one of {sorted(COST_KINDS)}")
        h = _P()
        _check(_cm_create(int(device), _as_u64(seed, "seed"), COST_KINDS[kind], ctypes.byref(h)))
        self._h = h

    @property
    def kind(self):
        k = ctypes.c_int()
        _check(_cm_kind(self._h, ctypes.byref(k)))
        return {v: n for n, v in COST_KINDS.items()}[k.value]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _cm_free(h)
            self._h = None

    def add_samples(self, features, log_cycles):
        X = _f32(features, MLP_FEATURES)
        y = _f32(log_cycles).reshape(-1)
        if y.shape[0] != X.shape[0]:
            raise ValueError("features and targets differ in length")
        _check(_cm_add(self._h, X.ctypes.data_as(_P), y.ctypes.data_as(_P), y.shape[0]))

    def record(self, simulator, circuit):
        """Run a unitary circuit once with per-operation timing; returns samples added."""
        text = _circuit_json(circuit)
        n = _u64()
        _check(_cm_record(self._h, simulator._h, text, len(text), ctypes.byref(n)))
        return n.value

    @property
    def num_samples(self):
        n = _u64()
        _check(_cm_num(self._h, ctypes.byref(n)))
        return n.value

    def samples(self):
        n = self.num_samples
        X = np.empty((n, MLP_FEATURES), dtype=np.float32)
        y = np.empty(n, dtype=np.float32)
        _check(_cm_samples(self._h, X.ctypes.data_as(_P), y.ctypes.data_as(_P), n))
        return X, y

    def train(self, epochs=60, lr=2e-3):
        mse = ctypes.c_double()
        _check(_cm_train(self._h, int(epochs), float(lr), ctypes.byref(mse)))
        return mse.value

    def predict(self, features):
        X = _f32(features, MLP_FEATURES)
        out = np.empty(X.shape[0], dtype=np.float32)
        _check(_cm_predict(self._h, X.ctypes.data_as(_P), X.shape[0], out.ctypes.data_as(_P)))
        return out

    def gradients(self, features, targets):
        X = _f32(features, MLP_FEATURES)
        y = _f32(targets).reshape(-1)
        g = np.empty(MLP_PARAMS - 2, dtype=np.float32)
        _check(_cm_grads(self._h, X.ctypes.data_as(_P), y.ctypes.data_as(_P), X.shape[0], g.ctypes.data_as(_P)))
        return g

    @property
    def params(self):
        p = np.empty(MLP_PARAMS, dtype=np.float32)
        _check(_cm_get(self._h, p.ctypes.data_as(_P), MLP_PARAMS))
        return p

    @params.setter
    def params(self, value):
        p = _f32(value).reshape(-1)
        _check(_cm_set(self._h, p.ctypes.data_as(_P), p.shape[0]))


def _take_text(out):
    try:
        return out.value.decode()
    finally:
        _string_free(ctypes.cast(out, ctypes.c_void_p))


def fused_portfolio(simulator, circuit, wide=True, measure=False, model=None):
    """The candidate fused plans of a circuit's unitary prefix (dq_fused_portfolio) as a dict: per plan its
    spread cap, hand-rule cost and pass indices; per distinct pass its tile qubits, blocks, gates and
    features, with measure=True its device milliseconds and with a fused-pass model its prediction."""
    import json as _json

    text = _circuit_json(circuit)
    out = ctypes.c_char_p()
    _check(_fused_portfolio(simulator._h, text, len(text), 1 if wide else 0, 1 if measure else 0,
                            None if model is None else model._h, ctypes.byref(out)))
    return _json.loads(_take_text(out))


def fused_random_passes(simulator, num_qubits, count, seed=0, measure=True):
    """Seeded random fused passes with features and device milliseconds (dq_fused_random_passes)."""
    import json as _json

    out = ctypes.c_char_p()
    _check(_fused_random(simulator._h, int(num_qubits), _as_u64(count, "count"), _as_u64(seed, "seed"),
                         1 if measure else 0, ctypes.byref(out)))
    return _json.loads(_take_text(out))


_fused_features = _sig("dq_fused_pass_features", [ctypes.c_int, _P, ctypes.c_int, ctypes.c_int, _P])


def fused_pass_features(num_qubits, tile_qubits, blocks, gates):
    """The fused-pass cost model's features of one pass (dq_fused_pass_features)."""
    tq = np.ascontiguousarray(np.asarray(tile_qubits, dtype=np.int32).reshape(-1))
    if tq.shape[0] != 12:
        raise ValueError("a fused pass has 12 tile qubits")
    out = np.empty(MLP_FEATURES, dtype=np.float32)
    _check(_fused_features(int(num_qubits), tq.ctypes.data_as(_P), int(blocks), int(gates), out.ctypes.data_as(_P)))
    return out


def fused_pass_targets(passes, num_qubits):
    """Training targets of the fused-pass model: log of each pass's device nanoseconds per tile."""
    tiles = float(1 << (int(num_qubits) - 12))
    return np.log(np.array([p["ms"] for p in passes], dtype=np.float64) * 1e6 / tiles).astype(np.float32)


def set_cost_model(simulator, model):
    """Attach (or with None detach) a trained cost model to a simulator's planner."""
    _check(_sim_set_cm(simulator._h, None if model is None else model._h))
    simulator._cost_model = model


def planner_log(simulator):
    out = ctypes.c_char_p()
    _check(_sim_log(simulator._h, ctypes.byref(out)))
    try:
        import json as _json

        return [_json.loads(line) for line in out.value.decode().splitlines() if line.strip()]
    finally:
        _string_free(ctypes.cast(out, ctypes.c_void_p))


CALL_PHASES = ("parse", "compile", "state", "plan", "run", "sums", "sample", "keys", "release", "total", "table",
               "prefix_device")


def last_call_phases(simulator):
    """Host seconds per phase of the simulator's last simulate_shots call (dq_sim_last_call_phases)."""
    out = np.zeros(len(CALL_PHASES), dtype=np.float64)
    _check(_sim_phases(simulator._h, out.ctypes.data, len(CALL_PHASES)))
    return dict(zip(CALL_PHASES, out.tolist()))


_device_memory = _sig("dq_device_memory", [ctypes.c_int, ctypes.POINTER(_u64), ctypes.POINTER(_u64)])


def device_memory(device=0):
    """Free and total bytes of a CUDA device (dq_device_memory)."""
    f, t = _u64(), _u64()
    _check(_device_memory(int(device), ctypes.byref(f), ctypes.byref(t)))
    return {"free": f.value, "total": t.value}


_U8P = ctypes.POINTER(ctypes.c_uint8)
_blocks_create = _sig("dq_blocks_create", [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_P)])
_blocks_destroy = _sig("dq_blocks_destroy", [_P], None)
_blocks_sync = _sig("dq_blocks_sync", [_P])
_block_one = _sig("dq_block_apply_one_qubit", [_P, _P, _u64, _u64, _P, _P, _P, ctypes.c_size_t])
_block_x = _sig("dq_block_apply_x", [_P, _P, _u64, _u64, _P, _P, ctypes.c_size_t])
_block_swap = _sig("dq_block_apply_swap", [_P, _P, _u64, _u64, _u64, _P, _P, ctypes.c_size_t])
_block_diag = _sig("dq_block_apply_diagonal", [_P, _P, _u64, _P, ctypes.c_size_t, _P])
_block_dense = _sig("dq_block_apply_dense", [_P, _P, _u64, _P, ctypes.c_size_t, _P])
_block_measure = _sig("dq_block_measure", [_P, _P, _u64, _u64, ctypes.c_double, ctypes.POINTER(ctypes.c_int)])
_block_merge = _sig("dq_block_merge", [_P, _P, _u64, _P, _u64, _P])
_block_probs = _sig("dq_block_probabilities", [_P, _P, _u64, _P, ctypes.c_size_t, _P])
_block_sums = _sig("dq_block_running_sums", [_P, _P, _u64, _P])


def _ptr_arg(p):
    return ctypes.c_void_p(int(p))


class BlockContext:
    """Dense P-block blocks on the device (dq_blocks_* / dq_block_*).

    Blocks are device buffers the caller owns (e.g. CUDA tensors' data_ptr()), of 2^n complex128 or complex64
    amplitudes little-endian in the block's local qubits; calls run in order on the context's stream.
    """

    def __init__(self, device=0, precision="complex128"):
        prec = PRECISIONS[str(precision).lower()]
        h = _P()
        _check(_blocks_create(int(device), prec, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _blocks_destroy(h)
            self._h = None

    @staticmethod
    def _controls(controls):
        q = np.ascontiguousarray([c[0] for c in controls], dtype=np.uint64)
        v = np.ascontiguousarray([1 if c[1] else 0 for c in controls], dtype=np.uint8)
        return q, v

    def apply_one_qubit(self, state, n, target, matrix, controls=()):
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128).reshape(4))
        q, v = self._controls(controls)
        _check(_block_one(self._h, _ptr_arg(state), n, target, m.ctypes.data_as(_P), q.ctypes.data_as(_P),
                          v.ctypes.data_as(_P), len(controls)))

    def apply_x(self, state, n, target, controls=()):
        q, v = self._controls(controls)
        _check(_block_x(self._h, _ptr_arg(state), n, target, q.ctypes.data_as(_P), v.ctypes.data_as(_P),
                        len(controls)))

    def apply_swap(self, state, n, a, b, controls=()):
        q, v = self._controls(controls)
        _check(_block_swap(self._h, _ptr_arg(state), n, a, b, q.ctypes.data_as(_P), v.ctypes.data_as(_P),
                           len(controls)))

    def apply_diagonal(self, state, n, qubits, diagonal):
        q = np.ascontiguousarray(qubits, dtype=np.uint64)
        d = np.ascontiguousarray(np.asarray(diagonal, dtype=np.complex128).reshape(-1))
        _check(_block_diag(self._h, _ptr_arg(state), n, q.ctypes.data_as(_P), q.shape[0], d.ctypes.data_as(_P)))

    def apply_dense(self, state, n, qubits, matrix):
        q = np.ascontiguousarray(qubits, dtype=np.uint64)
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128).reshape(-1))
        _check(_block_dense(self._h, _ptr_arg(state), n, q.ctypes.data_as(_P), q.shape[0], m.ctypes.data_as(_P)))

    def measure(self, state, n, qubit, draw):
        out = ctypes.c_int()
        _check(_block_measure(self._h, _ptr_arg(state), n, qubit, float(draw), ctypes.byref(out)))
        return out.value

    def merge(self, left, left_qubits, right, right_qubits, out):
        _check(_block_merge(self._h, _ptr_arg(left), left_qubits, _ptr_arg(right), right_qubits, _ptr_arg(out)))

    def probabilities(self, state, n, qubits, out):
        q = np.ascontiguousarray(list(qubits or []), dtype=np.uint64)
        _check(_block_probs(self._h, _ptr_arg(state), n, q.ctypes.data_as(_P), q.shape[0], _ptr_arg(out)))

    def running_sums(self, state, n, out):
        _check(_block_sums(self._h, _ptr_arg(state), n, _ptr_arg(out)))

    def sync(self):
        _check(_blocks_sync(self._h))


def device_fp64_tflops(device=0):
    """FP64 FMA throughput of a device in TFLOP/s, measured by the library's own kernel."""
    out = ctypes.c_double()
    _check(_fp64_tflops(int(device), ctypes.byref(out)))
    return out.value


def measure_noalloc(states_ptr, precision, num_states, num_qubits, qubit, seeds, draw_index, reset=False):
    """dq_measure_noalloc: measure states already in device memory, allocating nothing on the device.

    states_ptr is a device address (e.g. a CUDA tensor's data_ptr()); returns the outcomes.
    """
    prec = PRECISIONS[str(precision).lower()] if not isinstance(precision, int) else precision
    s = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64).reshape(-1))
    d = np.ascontiguousarray(np.asarray(draw_index, dtype=np.uint64).reshape(-1))
    if s.shape[0] != num_states or d.shape[0] != num_states:
        raise ValueError("seeds and draw_index need one entry per state")
    out = np.zeros(num_states, dtype=np.int32)
    _check(_measure_noalloc(ctypes.c_void_p(int(states_ptr)), prec, num_states, num_qubits, qubit, 1 if reset else 0,
                            s.ctypes.data_as(_P), d.ctypes.data_as(_P), out.ctypes.data_as(_P)))
    return out.tolist()


def compile_dump(circuit_json):
    """Host-only: the fused operation list of a transport JSON string (for tests)."""
    import json as _json

    text = circuit_json.encode("utf-8") if isinstance(circuit_json, str) else circuit_json
    out = ctypes.c_char_p()
    _check(_compile_dump(text, len(text), ctypes.byref(out)))
    try:
        return _json.loads(out.value.decode("utf-8"))
    finally:
        _string_free(ctypes.cast(out, ctypes.c_void_p))


_tile_plan_dump = _sig("dq_tile_plan_dump", [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_char_p)])


def tile_plan_dump(circuit_json, tile_qubits=12, fusion_width=2):
    """Host-only: the shared-memory pass plan of a unitary circuit (for tests and inspection)."""
    import json as _json

    text = circuit_json.encode("utf-8") if isinstance(circuit_json, str) else circuit_json
    out = ctypes.c_char_p()
    _check(_tile_plan_dump(text, len(text), int(tile_qubits), int(fusion_width), ctypes.byref(out)))
    try:
        return _json.loads(out.value.decode("utf-8"))
    finally:
        _string_free(ctypes.cast(out, ctypes.c_void_p))


_fused_plan_dump = _sig("dq_fused_plan_dump", [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_char_p)])


def fused_plan_dump(circuit_json):
    """Host-only: the tensor-core fused plan of a unitary circuit (for tests and inspection)."""
    import json as _json

    text = circuit_json.encode("utf-8") if isinstance(circuit_json, str) else circuit_json
    out = ctypes.c_char_p()
    _check(_fused_plan_dump(text, len(text), ctypes.byref(out)))
    try:
        return _json.loads(out.value.decode("utf-8"))
    finally:
        _string_free(ctypes.cast(out, ctypes.c_void_p))


_debug_fused_fault = _sig("dq_debug_fused_fault", [ctypes.c_uint64, ctypes.c_double])


def debug_fused_fault(withhold_step=None, wait_ms=0.0):
    """Failure-path testing of the fused kernel: gate images of fused steps >=
    withhold_step are never fetched and its bounded waits give up after wait_ms
    (<= 0: about 2 s); the call then raises RuntimeError.  No arguments: normal."""
    step = (1 << 64) - 1 if withhold_step is None else int(withhold_step)
    _check(_debug_fused_fault(step, float(wait_ms)))


def library_path():
    return str(_LIB_PATH)


def version():
    return _version().decode()


__all__ = [
    "MpsSimulator", "MpsResult", "PBlockResult", "PBlockSimulator", "SimulationProfile", "SimulationResult",
    "StabilizerSimulator", "StabilizerResult", "StatevectorSimulator", "simulate_distributed",
    "simulate_distributed_shots", "simulate_monolithic", "simulate_monolithic_shots",
]

if os.environ.get("DQSIM_DEBUG_LIB"):
    print("dqsim loaded", _LIB_PATH)
