"""Circuit equivalence checks: goqu's transpile/verify (verify.go:16-155).

EquivalentOnZero compares the states the two circuits prepare from
|0...0>; Equivalent compares their unitaries. Both allow a global phase,
taken from the first entry of the second circuit's state (column 0 of its
unitary) whose modulus exceeds tol. goqu builds a unitary from 2^n
statevector runs that prepend X gates to prepare each basis column; the
engine evolves all columns at once as one 2n-qubit vector (gq_unitary), and
evaluates the comparisons on the device. The qubit limits and error messages
are goqu's (14 qubits on |0>, 10 for unitaries).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from . import encode as _encode

_D = ctypes.POINTER(ctypes.c_double)


def _pair(a, b, limit, what):
    n = a.NumQubits()
    if b.NumQubits() != n:
        raise ValueError(f"verify: qubit count mismatch: {n} vs {b.NumQubits()}")
    if n > limit:
        raise ValueError(f"verify: circuit too large for {what}: {n} qubits")
    return n, _encode.statevector_ops(a), _encode.statevector_ops(b)


def _call(fn, n, sa, sb, tol):
    eq = ctypes.c_int()
    if n == 0:  # nothing to compare: both are the empty state
        return True
    _abi.check(fn(n, sa.ptr(), len(sa), sb.ptr(), len(sb), float(tol), ctypes.byref(eq)))
    return bool(eq.value)


def EquivalentOnZero(a, b, tol):
    """verify.go:14-38: the states from |0...0> agree up to a global phase."""
    n, sa, sb = _pair(a, b, 14, "equivalence check")
    return _call(_abi.lib().gq_equivalent_on_zero, n, sa, sb, tol)


def Equivalent(a, b, tol):
    """verify.go:40-68: the unitaries agree up to a global phase."""
    n, sa, sb = _pair(a, b, 10, "full equivalence check")
    return _call(_abi.lib().gq_equivalent, n, sa, sb, tol)


def Unitary(c):
    """The circuit's unitary as goqu's column list: out[col][row] = U[row][col]."""
    n = c.NumQubits()
    s = _encode.statevector_ops(c)
    out = np.empty(1 << (2 * n), dtype=np.complex128)
    _abi.check(_abi.lib().gq_unitary(n, s.ptr(), len(s), out.view(np.float64).ctypes.data_as(_D), out.nbytes))
    return out.reshape(1 << n, 1 << n)
