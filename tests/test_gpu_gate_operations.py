"""Front-end gate operations on the GPU through the reference's calling
sequence (_C.functionals.apply): modifiers (ctrl / negctrl / pow / inv,
fractional powers) and the gates the reference drops (CV, ECR, PRx,
Unitary), against the oracle applying each operation's full matrix."""
import numpy as np
import pytest

import oracle
from snuqs_b200 import _C, circuits
from snuqs_b200 import gate_operations as go

pytestmark = pytest.mark.gpu


def test_modified_gates_through_functionals_apply(cuda_required):
    n = 9
    rng = np.random.default_rng(11)
    sv = _C.result_types.StateVector(_C.DeviceType.CUDA, n)
    _C.functionals.initialize_basis_z(sv)
    ref = oracle.basis_state(n)
    for h in range(n):  # a spread-out state first
        op = go.gate_operation("h", [h])
        _C.functionals.apply(sv, op, n, list(op.targets))
        oracle.apply_matrix(ref, n, np.array(op), [h])
    names = [("rx", 1, 1), ("U", 1, 3), ("xy", 2, 1), ("cv", 2, 0), ("ecr", 2, 0), ("prx", 1, 2),
             ("ccnot", 3, 0), ("iswap", 2, 0)]
    for i in range(60):
        name, k, na = names[i % len(names)]
        mods = [("ctrl", int(rng.integers(0, 2))), ("negctrl", int(rng.integers(0, 2)))]
        if i % 3 == 0:
            mods.append(("pow", float(rng.choice([0.5, 2, -1.5, 3]))))
        if i % 4 == 0:
            mods.append(("inv", None))
        ctrl, power = go.fold_modifiers(mods)
        qs = [int(q) for q in rng.choice(n, size=len(ctrl) + k, replace=False)]
        op = go.gate_operation(name, qs, list(rng.uniform(0, 6, size=na)), ctrl_modifiers=ctrl, power=power)
        _C.functionals.apply(sv, op, n, list(op.targets))
        oracle.apply_matrix(ref, n, np.array(op), qs)
    u = go.Unitary([2, 7], circuits.haar_unitary(4, rng), ctrl_modifiers=[], power=0.5)
    _C.functionals.apply(sv, u, n, list(u.targets))
    oracle.apply_matrix(ref, n, np.array(u), [2, 7])
    got = np.array(sv.cpu(), copy=False)
    assert np.abs(got - ref).max() <= 1e-12
