"""ctypes wrapper for the test-only plan emulator (tests/native)."""
import ctypes
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from tests.native.build import build  # noqa: E402

_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        _lib.emu_run.restype = ctypes.c_int
    return _lib


def run(state, n, gates, tile_bits=12, reorder=True, low_bits=0):
    """gates: list of (matrix, qubits, controls, control_values). Returns
    (state, sweeps, unfused).  reorder: False/True, or "select" / "noselect"
    to force tile selection on / off."""
    psi = np.array(state, dtype=np.complex128)
    k, qoff, qs, nc, coff, cs, cv, moff, mats = [], [], [], [], [], [], [], [], []
    mo = 0
    for m, q, c, v in gates:
        k.append(len(q)); qoff.append(len(qs)); qs.extend(q)
        nc.append(len(c)); coff.append(len(cs)); cs.extend(c); cv.extend(v)
        moff.append(mo); mats.append(np.asarray(m, dtype=np.complex128).ravel()); mo += mats[-1].size
    arr = lambda x, t: np.ascontiguousarray(np.array(x if x else [0], dtype=t))
    K, QO, QS, NC, CO, CS, CV = (arr(x, np.int32) for x in (k, qoff, qs, nc, coff, cs, cv))
    MO = arr(moff, np.int64)
    M = np.ascontiguousarray(np.concatenate(mats) if mats else np.zeros(1, np.complex128))
    unf = ctypes.c_int(0)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    r = lib().emu_run(P(psi), n, len(gates), P(K), P(QO), P(QS), P(NC), P(CO), P(CS), P(CV),
                      P(MO), P(M), tile_bits, _reorder_code(reorder), low_bits,
                      ctypes.byref(unf))
    if r < 0:
        raise RuntimeError("emulator failed")
    return psi, r, unf.value


def run_rebuilt(state, n, gates_a, gates_b, tile_bits=12, reorder=True, low_bits=0):
    """Plans gates_a, re-emits the plan for gates_b (the same gates with other
    matrices) by rebuild_plan, emulates it; returns (state, sweeps, rebuilt)
    with rebuilt False when the plan was made anew instead."""
    psi = np.array(state, dtype=np.complex128)
    k, qoff, qs, nc, coff, cs, cv, moff, ma, mb = [], [], [], [], [], [], [], [], [], []
    mo = 0
    for (m, q, c, v), (m2, q2, c2, v2) in zip(gates_a, gates_b):
        assert tuple(q) == tuple(q2) and tuple(c) == tuple(c2) and tuple(v) == tuple(v2)
        k.append(len(q)); qoff.append(len(qs)); qs.extend(q)
        nc.append(len(c)); coff.append(len(cs)); cs.extend(c); cv.extend(v)
        moff.append(mo)
        ma.append(np.asarray(m, dtype=np.complex128).ravel())
        mb.append(np.asarray(m2, dtype=np.complex128).ravel())
        mo += ma[-1].size
    arr = lambda x, t: np.ascontiguousarray(np.array(x if x else [0], dtype=t))
    K, QO, QS, NC, CO, CS, CV = (arr(x, np.int32) for x in (k, qoff, qs, nc, coff, cs, cv))
    MO = arr(moff, np.int64)
    MA = np.ascontiguousarray(np.concatenate(ma))
    MB = np.ascontiguousarray(np.concatenate(mb))
    rebuilt = ctypes.c_int(0)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    r = lib().emu_rebuild(P(psi), n, len(gates_a), P(K), P(QO), P(QS), P(NC), P(CO), P(CS), P(CV),
                          P(MO), P(MA), P(MB), tile_bits, _reorder_code(reorder), low_bits,
                          ctypes.byref(rebuilt))
    if r < 0:
        raise RuntimeError("emulator failed")
    return psi, r, bool(rebuilt.value)


def _reorder_code(reorder):
    return {"select": 2, "noselect": 3, "remap": 4}.get(reorder, int(bool(reorder)))


def plan_stats(n, gates, tile_bits=12, reorder=True, low_bits=0):
    """{sweeps, phases, ops, kinds{...}, unfused, direct_load, direct_store}
    of the engine's plan (the last two count sweeps whose first / last phase
    leaves the low tile bits to the lanes)."""
    k, qoff, qs, nc, coff, cs, cv, moff, mats = [], [], [], [], [], [], [], [], []
    mo = 0
    for m, q, c, v in gates:
        k.append(len(q)); qoff.append(len(qs)); qs.extend(q)
        nc.append(len(c)); coff.append(len(cs)); cs.extend(c); cv.extend(v)
        moff.append(mo); mats.append(np.asarray(m, dtype=np.complex128).ravel()); mo += mats[-1].size
    arr = lambda x, t: np.ascontiguousarray(np.array(x if x else [0], dtype=t))
    K, QO, QS, NC, CO, CS, CV = (arr(x, np.int32) for x in (k, qoff, qs, nc, coff, cs, cv))
    MO = arr(moff, np.int64)
    M = np.ascontiguousarray(np.concatenate(mats))
    out = np.zeros(12, dtype=np.int64)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    if lib().emu_plan_stats(n, len(gates), P(K), P(QO), P(QS), P(NC), P(CO), P(CS), P(CV),
                            P(MO), P(M), tile_bits, _reorder_code(reorder), low_bits, P(out)) != 0:
        raise RuntimeError("planner failed")
    names = ["dense", "diag", "anti1", "xrot", "swap2", "phase"]
    return {"sweeps": int(out[0]), "phases": int(out[1]), "ops": int(out[2]),
            "kinds": {names[i]: int(out[3 + i]) for i in range(6)}, "unfused": int(out[9]),
            "direct_load": int(out[10]), "direct_store": int(out[11])}


def adjoint(n, ops, terms, nparams, tile_bits=10, select=-1):
    """(energy, grad, sweeps) from the host emulation of the adjoint plan."""
    from snuqs_b200 import capi
    arr, keep = capi.circuit_ops(ops)
    flat = "".join(p for _, p in terms).encode()
    w = np.ascontiguousarray([x for x, _ in terms], dtype=np.float64)
    e = ctypes.c_double(0)
    g = np.zeros(max(1, nparams), dtype=np.float64)
    lib().emu_adjoint.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_char_p,
                                  ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                  ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    r = lib().emu_adjoint(n, ctypes.cast(arr, ctypes.c_void_p), len(ops), flat,
                          w.ctypes.data_as(ctypes.c_void_p), len(terms), nparams, tile_bits,
                          select, ctypes.byref(e), g.ctypes.data_as(ctypes.c_void_p))
    if r < 0:
        raise RuntimeError("emulated adjoint failed")
    return e.value, g[:nparams], r
