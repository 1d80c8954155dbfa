"""ctypes binding of the C ABI (include/snuqs_b200.h).

This is the binding a maintainer would add on the reference side to call the
engine without pybind11; the tests use it to drive the C ABI directly.  Every call checks its status and raises SqError with the
library's message.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsnuqs_b200.so")

SQ_OK, SQ_ERR_INVALID, SQ_ERR_CUDA, SQ_ERR_OOM, SQ_ERR_UNSUPPORTED, SQ_ERR_TIMEOUT = range(6)
SQ_C128, SQ_C64 = 0, 1
(SQ_OPT_FUSION, SQ_OPT_TILE_BITS, SQ_OPT_REORDER, SQ_OPT_TIMING, SQ_OPT_JIT, SQ_OPT_LOW_BITS,
 SQ_OPT_REMAP) = range(7)

GATE_NAMES = [
    "Identity", "Hadamard", "PauliX", "PauliY", "PauliZ", "CX", "CY", "CZ", "S", "Si", "T",
    "Ti", "V", "Vi", "PhaseShift", "CPhaseShift", "CPhaseShift00", "CPhaseShift01",
    "CPhaseShift10", "RotX", "RotY", "RotZ", "Swap", "ISwap", "PSwap", "XY", "XX", "YY", "ZZ",
    "CCNot", "CSwap", "U", "GPhase", "SwapA2A", "ECR", "CV", "PRx",
]
GATE_ID = {n: i for i, n in enumerate(GATE_NAMES)}

# Every entry point the header declares: name -> (restype, argtypes).
_P = ctypes.c_void_p
_U32, _U64, _I, _D = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
_PU32, _PU64, _PD = ctypes.POINTER(_U32), ctypes.POINTER(_U64), ctypes.POINTER(_D)
SIGNATURES = {
    "sq_version": (ctypes.c_char_p, []),
    "sq_last_error": (ctypes.c_char_p, []),
    "sq_device_count": (_I, [ctypes.POINTER(_I)]),
    "sq_get_device": (_I, [ctypes.POINTER(_I)]),
    "sq_set_device": (_I, [_I]),
    "sq_device_synchronize": (_I, []),
    "sq_mem_info": (_I, [ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    "sq_stream_create": (_I, [ctypes.POINTER(_P), _I]),
    "sq_stream_destroy": (_I, [_P]),
    "sq_stream_synchronize": (_I, [_P]),
    "sq_stream_wait_event": (_I, [_P, _P]),
    "sq_event_create": (_I, [ctypes.POINTER(_P)]),
    "sq_event_destroy": (_I, [_P]),
    "sq_event_record": (_I, [_P, _P]),
    "sq_event_synchronize": (_I, [_P]),
    "sq_event_elapsed": (_I, [_P, _P, ctypes.POINTER(ctypes.c_float)]),
    "sq_host_alloc": (_I, [ctypes.POINTER(_P), ctypes.c_size_t]),
    "sq_host_free": (_I, [_P]),
    "sq_gate_matrix": (_I, [_I, _PD, _U32, _PD, _PU32]),
    "sq_gate_qubits": (_I, [_I]),
    "sq_gate_matrix_derivative": (_I, [_I, _PD, _U32, _U32, _PD, _PU32]),
    "sq_state_create": (_I, [_U32, _I, ctypes.POINTER(_P)]),
    "sq_state_wrap": (_I, [_P, _U32, _I, ctypes.POINTER(_P)]),
    "sq_state_destroy": (_I, [_P]),
    "sq_state_data": (_P, [_P]),
    "sq_state_num_qubits": (_U32, [_P]),
    "sq_state_dtype": (_I, [_P]),
    "sq_set_option": (_I, [_P, _I, ctypes.c_int64]),
    "sq_init_zero": (_I, [_P, _P]),
    "sq_init_basis": (_I, [_P, _U64, _P]),
    "sq_apply_matrix": (_I, [_P, _PD, _PU32, _U32, _P]),
    "sq_apply_controlled_matrix": (_I, [_P, _PD, _PU32, _U32, _PU32,
                                        ctypes.POINTER(ctypes.c_uint8), _U32, _P]),
    "sq_apply_gate": (_I, [_P, _I, _PU32, _U32, _PD, _U32, _P]),
    "sq_flush": (_I, [_P, _P]),
    "sq_pending": (_I, [_P, _PU32]),
    "sq_launch_count": (_I, [_P, _PU64]),
    "sq_sweep_timing": (_I, [_P, _PD, _PU64]),
    "sq_jit_info": (_I, [ctypes.POINTER(_I), _PU64, _PU64]),
    "sq_jit_compile": (_I, [ctypes.c_char_p]),
    "sq_jit_source": (_I, [_U32, _I, _P, _U32, _U32, ctypes.c_char_p, _U64, _PU64, _PU32]),
    "sq_jit_adjoint_source": (_I, [_U32, _I, _P, _U32, _U32, ctypes.c_char_p, _U64, _PU64, _PU32]),
    "sq_jit_batch_adjoint_source": (_I, [_U32, _I, _P, _U32, ctypes.c_char_p, _U64, _PU64]),
    "sq_apply_gate_buffer": (_I, [_P, _P, _PU64, _U32, _U32, _U64, _P]),
    "sq_copy_to_host": (_I, [_P, _P, _P]),
    "sq_copy_from_host": (_I, [_P, _P, _P]),
    "sq_copy_state": (_I, [_P, _P, _P]),
    "sq_state_check": (_I, [_P, _P]),
    "sq_variance_pauli": (_I, [_P, ctypes.c_char_p, _PD, _U32, _PD, _P]),
    "sq_sample": (_I, [_P, _P, _U64, _P, _P]),
    "sq_sample_host": (_I, [_P, _PD, _U64, _PU64, _P]),
    "sq_amplitudes": (_I, [_P, _P, _U64, _P, _P]),
    "sq_marginal_probabilities": (_I, [_P, _PU32, _U32, _P, _P]),
    "sq_state_distance": (_I, [_P, _P, _PD, _PD, _P]),
    "sq_probabilities": (_I, [_P, _P, _P]),
    "sq_expect_pauli": (_I, [_P, ctypes.c_char_p, _PD, _U32, _PD, _P]),
    "sq_norm2": (_I, [_P, _PD, _P]),
    "sq_expect_pauli_noalloc": (_I, [_P, _U32, _I, ctypes.c_char_p, _PD, _U32, _P, _P]),
    "sq_adjoint_gradient": (_I, [_P, _P, _P, _U32, ctypes.c_char_p, _PD, _U32, _U32, _PD, _PD, _P]),
    "sq_batch_create": (_I, [_I, ctypes.POINTER(_P)]),
    "sq_batch_destroy": (_I, [_P]),
    "sq_batch_set_option": (_I, [_P, _I, ctypes.c_int64]),
    "sq_batch_add_hamiltonian": (_I, [_P, _U32, ctypes.c_char_p, _PD, _U32, _PU32]),
    "sq_batch_add_circuit": (_I, [_P, _U32, _P, _U32, _U32, _PU32]),
    "sq_batch_set_angles": (_I, [_P, _U32, _PD, _U32]),
    "sq_batch_num_circuits": (_I, [_P, _PU32]),
    "sq_batch_run": (_I, [_P, _PD, _P]),
    "sq_batch_run_gradients": (_I, [_P, _U32, _PD, _PD, _P]),
    "sq_batch_autotune": (_I, [_P, _U32, _P, _P]),
    "sq_batch_state": (_I, [_P, _U32, _P, _P]),
    "sq_batch_last_timing": (_I, [_P, _PD, _PU32]),
    "sq_batch_stats": (_I, [_P, _PU64, _PU64, _PU64]),
    "sq_batch_groups": (_I, [_P, _PU32, _PU32]),
    "sq_jit_multi_source": (_I, [_U32, _I, _P, _U32, _U32, _I, ctypes.c_char_p, _U64, _PU64, _PU32]),
}


class SqBatchConfig(ctypes.Structure):
    """sq_batch_config (include/snuqs_b200.h)."""
    _fields_ = [("tile_bits", ctypes.c_uint32), ("low_bits", ctypes.c_uint32),
                ("max_ops", ctypes.c_uint32), ("ctas_per_sm", ctypes.c_uint32),
                ("kernel_ms", ctypes.c_double)]


SQ_BOPT_KEEP_STATES, SQ_BOPT_TILE_BITS, SQ_BOPT_LOW_BITS, SQ_BOPT_MAX_OPS, SQ_BOPT_CTAS_PER_SM = range(5)


class SqCircuitOp(ctypes.Structure):
    """sq_circuit_op (include/snuqs_b200.h)."""
    _fields_ = [("gate", ctypes.c_int32), ("k", ctypes.c_uint32), ("qubits", ctypes.c_uint32 * 3),
                ("nangles", ctypes.c_uint32), ("angles", ctypes.c_double * 3),
                ("param", ctypes.c_int32 * 3), ("scale", ctypes.c_double * 3),
                ("matrix", ctypes.POINTER(ctypes.c_double))]


def jit_info():
    """(NVRTC available, JIT sweep launches, fallbacks to the generic kernel)."""
    av, a, b = ctypes.c_int(0), _U64(0), _U64(0)
    check(lib().sq_jit_info(ctypes.byref(av), ctypes.byref(a), ctypes.byref(b)))
    return bool(av.value), a.value, b.value


def jit_sources(n: int, ops, dtype: int = SQ_C128, limit: int | None = None, adjoint: bool = False,
                multi: bool = False, from_zero: bool = False):
    """CUDA sources of the JIT kernels of the fused sweeps of a circuit (with
    adjoint=True: of the reverse sweeps of its adjoint-gradient plan; with
    multi=True: the multi-state kernels of its batch energy plan, from_zero:
    their form that starts from |0...0>; "" for a sweep the generic kernel
    runs)."""
    if multi:
        raw = lib().sq_jit_multi_source
        fn = lambda *a: raw(*a[:5], int(from_zero), *a[5:])
    else:
        fn = lib().sq_jit_adjoint_source if adjoint else lib().sq_jit_source
    arr, keep = circuit_ops(ops)
    ln, ns = _U64(0), _U32(0)
    check(fn(n, dtype, ctypes.cast(arr, _P), len(ops), 0, None, 0, ctypes.byref(ln), ctypes.byref(ns)))
    out = []
    for i in range(ns.value if limit is None else min(limit, ns.value)):
        check(fn(n, dtype, ctypes.cast(arr, _P), len(ops), i, None, 0, ctypes.byref(ln), ctypes.byref(ns)))
        buf = ctypes.create_string_buffer(ln.value + 1)
        check(fn(n, dtype, ctypes.cast(arr, _P), len(ops), i, buf, ln.value + 1,
                 ctypes.byref(ln), ctypes.byref(ns)))
        out.append(buf.value.decode())
    del keep
    return out


def jit_batch_adjoint_source(n: int, ops, dtype: int = SQ_C128) -> str:
    """Source of the JIT batched-gradient kernel for batches of circuits
    sharing the structure of `ops` ("" when not covered)."""
    arr, keep = circuit_ops(ops)
    ln = _U64(0)
    check(lib().sq_jit_batch_adjoint_source(n, dtype, ctypes.cast(arr, _P), len(ops), None, 0, ctypes.byref(ln)))
    buf = ctypes.create_string_buffer(ln.value + 1)
    check(lib().sq_jit_batch_adjoint_source(n, dtype, ctypes.cast(arr, _P), len(ops), buf, ln.value + 1,
                                            ctypes.byref(ln)))
    del keep
    return buf.value.decode()


def jit_compile(source: str) -> None:
    """NVRTC-compiles a kernel source for sm_100a; raises SqError with the log."""
    check(lib().sq_jit_compile(source.encode()))


def circuit_ops(ops):
    """Array of SqCircuitOp from ops (name, qubits, angles[, params[, scales]]) or
    ("Unitary", qubits, (), matrix).  params[j] is the parameter index fed by
    angle j (-1 = constant).  Returns (array, keepalive)."""
    arr = (SqCircuitOp * max(1, len(ops)))()
    keep = []
    for i, op in enumerate(ops):
        o = arr[i]
        o.k = len(op[1])
        for j, q in enumerate(op[1]):
            o.qubits[j] = q
        for j in range(3):
            o.param[j] = -1
            o.scale[j] = 1.0
        if op[0] == "Unitary":
            m = np.ascontiguousarray(op[3], dtype=np.complex128)
            keep.append(m)
            o.gate = -1
            o.matrix = m.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            continue
        o.gate = GATE_ID[op[0]]
        o.nangles = len(op[2])
        for j, a in enumerate(op[2]):
            o.angles[j] = a
        if len(op) > 3:
            for j, p in enumerate(op[3]):
                o.param[j] = p
        if len(op) > 4:
            for j, sc in enumerate(op[4]):
                o.scale[j] = sc
    return arr, keep




class Batch:
    """Many small circuits and their Pauli-sum energies in one launch
    (sq_batch_*)."""

    def __init__(self, dtype: int = SQ_C128, keep_states: bool = False):
        h = _P()
        check(lib().sq_batch_create(dtype, ctypes.byref(h)))
        self.h, self.dtype = h, dtype
        self._hams = {}
        self._n = []
        if keep_states:
            check(lib().sq_batch_set_option(h, SQ_BOPT_KEEP_STATES, 1))

    def close(self):
        if self.h:
            check(lib().sq_batch_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_hamiltonian(self, n: int, terms) -> int:
        flat = "".join(p for _, p in terms).encode()
        w = np.ascontiguousarray([x for x, _ in terms] or [0.0], dtype=np.float64)
        hid = _U32(0)
        check(lib().sq_batch_add_hamiltonian(self.h, n, flat, _dp(w), len(terms), ctypes.byref(hid)))
        return hid.value

    def add_circuit(self, n: int, ops, ham: int) -> int:
        arr, keep = circuit_ops(ops)
        cid = _U32(0)
        check(lib().sq_batch_add_circuit(self.h, n, ctypes.cast(arr, _P), len(ops), ham,
                                         ctypes.byref(cid)))
        self._n.append(n)
        return cid.value

    def set_angles(self, circuit: int, angles) -> None:
        a = np.ascontiguousarray(angles, dtype=np.float64)
        check(lib().sq_batch_set_angles(self.h, circuit, _dp(a), a.size))

    def run(self, stream=None) -> np.ndarray:
        out = np.zeros(max(1, len(self._n)), dtype=np.float64)
        check(lib().sq_batch_run(self.h, _dp(out), stream))
        return out[: len(self._n)]

    def set_option(self, option: int, value: int) -> None:
        check(lib().sq_batch_set_option(self.h, option, value))

    def configure(self, config: dict) -> None:
        """Applies a launch configuration (the dict autotune() returns)."""
        for key, opt in (("tile_bits", SQ_BOPT_TILE_BITS), ("low_bits", SQ_BOPT_LOW_BITS),
                         ("max_ops", SQ_BOPT_MAX_OPS), ("ctas_per_sm", SQ_BOPT_CTAS_PER_SM)):
            self.set_option(opt, int(config.get(key, 0)))

    def signature(self) -> str:
        """Workload key of the autotuner cache: device, precision and the
        circuits' qubit-count histogram."""
        import hashlib

        dev = "unknown"
        try:
            import torch

            dev = torch.cuda.get_device_name()
        except Exception:
            pass
        hist = {}
        for n in self._n:
            hist[n] = hist.get(n, 0) + 1
        text = f"{dev}|{self.dtype}|{sorted(hist.items())}"
        return hashlib.sha1(text.encode()).hexdigest()[:16]

    def autotune(self, reps: int = 2, cache: str | None = None, stream=None) -> dict:
        """Picks tile size, low bits, fusion width and CTAs per SM by timing
        the energy kernel (sq_batch_autotune) and applies the fastest.  With
        `cache` (a JSON file), a result stored for the same signature() is
        applied without timing, and new results are stored there."""
        import json

        key = self.signature()
        store = {}
        if cache and os.path.exists(cache):
            try:
                with open(cache) as f:
                    store = json.load(f)
            except Exception:
                store = {}
        if key in store:
            self.configure(store[key])
            return dict(store[key], cached=True)
        c = SqBatchConfig()
        check(lib().sq_batch_autotune(self.h, reps, ctypes.byref(c), stream))
        out = {"tile_bits": c.tile_bits, "low_bits": c.low_bits, "max_ops": c.max_ops,
               "ctas_per_sm": c.ctas_per_sm, "kernel_ms": c.kernel_ms}
        if cache:
            store[key] = out
            os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
            with open(cache, "w") as f:
                json.dump(store, f, indent=1)
        return dict(out, cached=False)

    def run_gradients(self, n_params: int, stream=None):
        """(energies[ncircuits], grads[ncircuits, n_params]) in one launch."""
        nc = len(self._n)
        e = np.zeros(max(1, nc), dtype=np.float64)
        g = np.zeros((max(1, nc), max(1, n_params)), dtype=np.float64)
        check(lib().sq_batch_run_gradients(self.h, n_params, _dp(e), _dp(g), stream))
        return e[:nc], g[:nc, :n_params]

    def state(self, circuit: int) -> np.ndarray:
        a = np.empty(1 << self._n[circuit],
                     dtype=np.complex64 if self.dtype == SQ_C64 else np.complex128)
        check(lib().sq_batch_state(self.h, circuit, a.ctypes.data_as(_P), None))
        return a

    def stats(self):
        """(streamed circuits, their sweeps, their algorithmic HBM bytes) of
        the last run."""
        a, b, c = _U64(0), _U64(0), _U64(0)
        check(lib().sq_batch_stats(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def groups(self):
        """(structure groups, circuits in them) of the last run: circuits run
        by multi-state JIT sweeps."""
        g, c = _U32(0), _U32(0)
        check(lib().sq_batch_groups(self.h, ctypes.byref(g), ctypes.byref(c)))
        return g.value, c.value

    def last_timing(self):
        ms, ctas = _D(0), _U32(0)
        check(lib().sq_batch_last_timing(self.h, ctypes.byref(ms), ctypes.byref(ctas)))
        return ms.value, ctas.value


class SqError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"sq status {status}: {msg}")
        self.status = status


_lib = None


def lib() -> ctypes.CDLL:
    """Loads libsnuqs_b200.so.  Raises if it has not been built: there is no
    fallback implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with python -m snuqs_b200.build")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def check(status: int) -> None:
    if status != SQ_OK:
        raise SqError(status, lib().sq_last_error().decode())


def _u32(xs: Sequence[int]):
    return (_U32 * max(1, len(xs)))(*xs)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_PD)


def gate_matrix(name: str, angles: Sequence[float] = ()) -> np.ndarray:
    a = np.zeros(3, dtype=np.float64)
    a[: len(angles)] = angles
    out = np.zeros(64, dtype=np.complex128)
    k = _U32(0)
    check(lib().sq_gate_matrix(GATE_ID[name], _dp(a), len(angles), _dp(out), ctypes.byref(k)))
    d = 1 << k.value
    return out[: d * d].reshape(d, d).copy()


def gate_matrix_derivative(name: str, angles: Sequence[float], param: int) -> np.ndarray:
    a = np.zeros(3, dtype=np.float64)
    a[: len(angles)] = angles
    out = np.zeros(64, dtype=np.complex128)
    k = _U32(0)
    check(lib().sq_gate_matrix_derivative(GATE_ID[name], _dp(a), len(angles), param, _dp(out),
                                          ctypes.byref(k)))
    d = 1 << k.value
    return out[: d * d].reshape(d, d).copy()


class State:
    """Owning wrapper of an sq_state* (complex128 or complex64)."""

    def __init__(self, num_qubits: int, dtype: int = SQ_C128, stream=None):
        self.n = num_qubits
        self.dtype = dtype
        self.stream = stream
        h = _P()
        check(lib().sq_state_create(num_qubits, dtype, ctypes.byref(h)))
        self.h = h

    def close(self) -> None:
        if self.h:
            check(lib().sq_state_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def np_dtype(self):
        return np.complex64 if self.dtype == SQ_C64 else np.complex128

    def set_option(self, opt: int, value: int) -> None:
        check(lib().sq_set_option(self.h, opt, value))

    def init_basis(self, index: int = 0) -> None:
        check(lib().sq_init_basis(self.h, index, self.stream))

    def apply_matrix(self, m: np.ndarray, qubits: Sequence[int], controls: Sequence[int] = (),
                     control_values: Sequence[int] | None = None) -> None:
        mm = np.ascontiguousarray(m, dtype=np.complex128)
        if controls:
            cv = (ctypes.c_uint8 * len(controls))(*(control_values or [1] * len(controls)))
            check(lib().sq_apply_controlled_matrix(self.h, _dp(mm), _u32(qubits), len(qubits),
                                                   _u32(controls), cv, len(controls), self.stream))
        else:
            check(lib().sq_apply_matrix(self.h, _dp(mm), _u32(qubits), len(qubits), self.stream))

    def apply_gate(self, name: str, qubits: Sequence[int], angles: Sequence[float] = ()) -> None:
        a = np.ascontiguousarray(np.array(list(angles) + [0.0], dtype=np.float64))
        check(lib().sq_apply_gate(self.h, GATE_ID[name], _u32(qubits), len(qubits), _dp(a),
                                  len(angles), self.stream))

    def apply_ops(self, ops) -> None:
        for op in ops:
            if op[0] == "Unitary":
                self.apply_matrix(op[3], op[1])
            else:
                self.apply_gate(op[0], op[1], op[2])

    def flush(self) -> None:
        check(lib().sq_flush(self.h, self.stream))

    def launches(self) -> int:
        c = _U64(0)
        check(lib().sq_launch_count(self.h, ctypes.byref(c)))
        return c.value

    def sweep_timing(self):
        """(total ms, launches) of the fused sweeps recorded with SQ_OPT_TIMING."""
        ms, c = _D(0), _U64(0)
        check(lib().sq_sweep_timing(self.h, ctypes.byref(ms), ctypes.byref(c)))
        return ms.value, c.value

    def to_host(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(1 << self.n, dtype=self.np_dtype)
        check(lib().sq_copy_to_host(self.h, out.ctypes.data_as(_P), self.stream))
        check(lib().sq_state_check(self.h, self.stream))
        return out

    def from_host(self, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=self.np_dtype)
        check(lib().sq_copy_from_host(self.h, a.ctypes.data_as(_P), self.stream))
        check(lib().sq_stream_synchronize(self.stream))

    def expectation(self, terms) -> float:
        """terms: list of (weight, pauli string of length n)."""
        flat = "".join(p for _, p in terms).encode()
        w = np.ascontiguousarray([float(x) for x, _ in terms] or [0.0], dtype=np.float64)
        out = _D(0)
        check(lib().sq_expect_pauli(self.h, flat, _dp(w), len(terms), ctypes.byref(out),
                                    self.stream))
        return out.value

    def variance(self, terms) -> float:
        """<H^2> - <H>^2 of the Pauli sum `terms` (list of (weight, string))."""
        flat = "".join(p for _, p in terms).encode()
        w = np.ascontiguousarray([float(x) for x, _ in terms] or [0.0], dtype=np.float64)
        out = _D(0)
        check(lib().sq_variance_pauli(self.h, flat, _dp(w), len(terms), ctypes.byref(out),
                                      self.stream))
        return out.value

    def sample(self, uniforms) -> np.ndarray:
        """Basis-state indices of len(uniforms) shots (device inverse CDF)."""
        import torch

        u = torch.as_tensor(np.ascontiguousarray(uniforms, dtype=np.float64)).cuda()
        out = torch.empty(u.numel(), dtype=torch.int64, device="cuda")
        check(lib().sq_sample(self.h, ctypes.c_void_p(u.data_ptr()), u.numel(),
                              ctypes.c_void_p(out.data_ptr()), self.stream))
        check(lib().sq_state_check(self.h, self.stream))
        return out.cpu().numpy().astype(np.uint64)

    def amplitudes(self, indices) -> np.ndarray:
        import torch

        idx = torch.as_tensor(np.ascontiguousarray(indices, dtype=np.int64)).cuda()
        out = torch.empty((idx.numel(), 2), dtype=torch.float64, device="cuda")
        check(lib().sq_amplitudes(self.h, ctypes.c_void_p(idx.data_ptr()), idx.numel(),
                                  ctypes.c_void_p(out.data_ptr()), self.stream))
        o = out.cpu().numpy()
        return o[:, 0] + 1j * o[:, 1]

    def marginal_probabilities(self, qubits) -> np.ndarray:
        import torch

        out = torch.empty(1 << len(qubits), dtype=torch.float64, device="cuda")
        check(lib().sq_marginal_probabilities(self.h, _u32(qubits), len(qubits),
                                              ctypes.c_void_p(out.data_ptr()), self.stream))
        check(lib().sq_state_check(self.h, self.stream))
        return out.cpu().numpy()

    def distance(self, other: "State"):
        """(max-abs amplitude difference, 1 - fidelity) against `other`."""
        mx, fl = _D(0), _D(0)
        check(lib().sq_state_distance(self.h, other.h, ctypes.byref(mx), ctypes.byref(fl), self.stream))
        return mx.value, fl.value

    def norm2(self) -> float:
        out = _D(0)
        check(lib().sq_norm2(self.h, ctypes.byref(out), self.stream))
        return out.value

    def data_ptr(self) -> int:
        return lib().sq_state_data(self.h)
