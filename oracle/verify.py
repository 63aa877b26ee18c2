"""goqu's transpile/verify on the oracle (verify.go:14-155).

TEST INFRASTRUCTURE: the checker for the engine's gq_unitary / gq_equivalent
entry points, used by tests/ only. Columns are built the way goqu builds
them: X gates prepare |col>, then the circuit runs on a fresh state
(prependBasisPrep, verify.go:80-90); the comparisons restate
stateVectorsClose (:92-126) and unitariesClose (:128-155) loop for loop.
"""
from __future__ import annotations

import numpy as np

from goqu_b200 import circuit as ir, encode, gate as G

from . import binding as orc


def _prep(c, idx):
    n = c.NumQubits()
    ops = [ir.Operation(G.X, [q]) for q in range(n) if idx & (1 << q)]
    return ir.Circuit(c.Name(), n, c.NumClbits(), ops + list(c.Ops()))


def unitary_columns(c):
    """unitary[col] = the state of the circuit applied to |col>."""
    n = c.NumQubits()
    return np.array([orc.sv_evolve(encode.statevector_ops(_prep(c, col))) for col in range(1 << n)])


def state_vectors_close(a, b, tol):
    if len(a) != len(b):
        return False
    phase, found = 0j, False
    for i in range(len(a)):
        if abs(b[i]) > tol:
            if abs(a[i]) < tol:
                return False
            phase = a[i] / b[i]
            if abs(abs(phase) - 1) > tol:
                return False
            found = True
            break
        elif abs(a[i]) > tol:
            return False
    if not found:
        return True
    return bool(np.all(np.abs(a - phase * b) <= tol))


def unitaries_close(a, b, dim, tol):
    phase, found = 0j, False
    for i in range(dim):
        if abs(b[0][i]) > tol:
            if abs(a[0][i]) < tol:
                return False
            phase = a[0][i] / b[0][i]
            found = True
            break
    if not found:
        return True
    return bool(np.all(np.abs(a - phase * b) <= tol))


def equivalent_on_zero(a, b, tol):
    sa = orc.sv_evolve(encode.statevector_ops(a))
    sb = orc.sv_evolve(encode.statevector_ops(b))
    return state_vectors_close(sa, sb, tol)


def equivalent(a, b, tol):
    return unitaries_close(unitary_columns(a), unitary_columns(b), 1 << a.NumQubits(), tol)
