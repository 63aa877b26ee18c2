"""Circuit equivalence on the device (gq_unitary, gq_equivalent,
gq_equivalent_on_zero) against goqu's transpile/verify: its own test cases
(transpile/verify/verify_test.go:10-160), unitary columns against the
oracle's column-by-column construction (verify.go:45-90) within 1e-12, and
the same decisions as the oracle's restatement of stateVectorsClose /
unitariesClose on random pairs."""
import math

import numpy as np
import pytest

from goqu_b200 import circuit as ir, gate as G, verify, workloads
from oracle import verify as ov

from kat_util import random_circuit

pytestmark = pytest.mark.gpu


def circ(n, ops, name="c"):
    return ir.Circuit(name, n, 0, [ir.Operation(g, list(q)) for g, q in ops])


# verify_test.go:10-150, EquivalentOnZero
@pytest.mark.parametrize("n,a,b,tol,want", [
    (2, [(G.H, [0]), (G.CNOT, [0, 1])], [(G.H, [0]), (G.CNOT, [0, 1])], 1e-8, True),   # identical (:10-26)
    (1, [(G.H, [0])], [(G.X, [0])], 1e-8, False),                                        # different (:28-46)
    (1, [(G.RZ(1.0), [0])], [(G.RZ(1.0), [0])], 1e-8, True),                             # same RZ (:48-66)
    (2, [], [], 1e-8, True),                                                             # empty (:68-79)
    (2, [(G.H, [0]), (G.CNOT, [0, 1])],                                                   # decomposed Bell (:91-117)
     [(G.RZ(1.5707963267948966), [0]), (G.SX, [0]), (G.RZ(1.5707963267948966), [0]), (G.CNOT, [0, 1])], 1e-6, True),
    (1, [(G.I, [0])], [], 1e-8, True),                                                   # identity vs empty (:119-133)
    (1, [(G.X, [0]), (G.X, [0])], [], 1e-8, True),                                       # self inverse (:135-150)
])
def test_equivalent_on_zero_reference_cases(n, a, b, tol, want):
    ca, cb = circ(n, a, "a"), circ(n, b, "b")
    assert verify.EquivalentOnZero(ca, cb, tol) is want
    assert ov.equivalent_on_zero(ca, cb, tol) is want


@pytest.mark.parametrize("n,a,b,want", [
    (2, [(G.CNOT, [0, 1])], [(G.H, [1]), (G.CZ, [0, 1]), (G.H, [1])], True),
    (2, [(G.SWAP, [0, 1])], [(G.CNOT, [0, 1]), (G.CNOT, [1, 0]), (G.CNOT, [0, 1])], True),
    (1, [(G.RZ(0.7), [0])], [(G.Phase(0.7), [0])], True),      # a global phase apart
    (1, [(G.X, [0])], [(G.Y, [0])], False),                      # X = i Y Z: not a global phase
    (2, [(G.H, [0]), (G.CNOT, [0, 1])], [(G.H, [0])], False),
    (3, [(G.CCX, [0, 1, 2])], [(G.CCX, [1, 0, 2])], True),
    (3, [(G.CCX, [0, 1, 2])], [(G.CCX, [0, 2, 1])], False),
])
def test_equivalent_unitaries(n, a, b, want):
    ca, cb = circ(n, a, "a"), circ(n, b, "b")
    assert verify.Equivalent(ca, cb, 1e-9) is want
    assert ov.equivalent(ca, cb, 1e-9) is want


def test_unitary_columns_match_oracle():
    c = random_circuit(8, 60, 5, allow_3q=True, allow_ctrl=True, allow_reset=False)
    u = verify.Unitary(c)
    want = ov.unitary_columns(c)
    assert np.max(np.abs(u - want)) <= 1e-12


def test_random_pairs_same_decisions_as_oracle():
    rng = np.random.default_rng(7)
    for k in range(12):
        n = int(rng.integers(2, 7))
        a = random_circuit(n, 25, 100 + k, allow_3q=False, allow_ctrl=False, allow_reset=False)
        # b: a itself, a with one gate perturbed, or a global phase of a
        ops = list(a.Ops())
        kind = k % 3
        if kind == 1:
            i = int(rng.integers(len(ops)))
            q = ops[i].Qubits[0]
            ops.insert(i, ir.Operation(G.RZ(1e-3), [q]))
        elif kind == 2:
            ops.append(ir.Operation(G.GlobalPhase(0.4), [0]))
        b = ir.Circuit("b", n, 0, ops)
        for tol in (1e-9, 1e-2):
            assert verify.Equivalent(a, b, tol) == ov.equivalent(a, b, tol), (k, tol)
            assert verify.EquivalentOnZero(a, b, tol) == ov.equivalent_on_zero(a, b, tol), (k, tol)


def test_larger_than_goqu_through_the_c_abi():
    # 12 qubits: 4^12 entries per unitary, beyond goqu's 10-qubit limit
    import ctypes

    from goqu_b200 import _abi, encode
    c = workloads.random_layers(12, 3, seed=4)
    s = encode.statevector_ops(c)
    both = encode.OpStream(12)  # the circuit, then its inverse (daggers in reverse order)
    ident = encode.OpStream(12)
    for op in list(c.Ops()):
        m = np.asarray(op.Gate.Matrix(), dtype=np.complex128)
        both.add(_abi.GQ_OP_MATRIX, op.Qubits, m)
    for op in reversed(list(c.Ops())):
        m = np.asarray(op.Gate.Matrix(), dtype=np.complex128)
        d = int(math.isqrt(m.size))
        both.add(_abi.GQ_OP_MATRIX, op.Qubits, m.reshape(d, d).conj().T)
    eq = ctypes.c_int()
    _abi.check(_abi.lib().gq_equivalent(12, both.ptr(), len(both), ident.ptr(), 0, 1e-9, ctypes.byref(eq)))
    assert eq.value == 1
    _abi.check(_abi.lib().gq_equivalent(12, s.ptr(), len(s), ident.ptr(), 0, 1e-9, ctypes.byref(eq)))
    assert eq.value == 0
