"""Pauli strings and sums (goqu sim/pauli).

Symplectic encoding I=00, X=10, Z=01, Y=11 (pauli.go:19-24); x/z masks
(pauli.go:146-169). ``Parse`` maps character i to qubit i (pauli.go:57-80).
"""
from __future__ import annotations

from . import _abi

I, X, Z, Y = 0b00, 0b10, 0b01, 0b11
_NAMES = {I: "I", X: "X", Y: "Y", Z: "Z"}


class PauliString:
    def __init__(self, coeff, ops, num_qubits):
        if num_qubits < 1:
            raise ValueError("pauli: numQubits must be >= 1")
        self._coeff = complex(coeff)
        self._ops = list(ops)
        self._n = num_qubits

    def Coeff(self):
        return self._coeff

    def Op(self, q):
        if q < 0 or q >= self._n:
            return I
        return self._ops[q]

    def NumQubits(self):
        return self._n

    def Scale(self, c):
        return PauliString(self._coeff * c, self._ops, self._n)

    def IsIdentity(self):
        return all(p == I for p in self._ops)

    def XMask(self):
        return sum(1 << i for i, p in enumerate(self._ops) if p & 0b10)

    def ZMask(self):
        return sum(1 << i for i, p in enumerate(self._ops) if p & 0b01)

    def NumY(self):
        return sum(1 for p in self._ops if p == Y)

    def __str__(self):
        s = "".join(_NAMES[p] for p in self._ops)
        return s if self._coeff == 1 else f"{self._coeff}*{s}"


def NewPauliString(coeff, ops, num_qubits):
    """pauli.go:38-55: ops maps qubit -> Pauli."""
    if num_qubits < 1:
        raise ValueError("pauli: numQubits must be >= 1")
    paulis = [I] * num_qubits
    for q, p in (ops or {}).items():
        if q < 0 or q >= num_qubits:
            raise ValueError(f"pauli: qubit {q} out of range [0, {num_qubits})")
        paulis[q] = p
    return PauliString(coeff, paulis, num_qubits)


def Parse(s):
    if not s:
        raise ValueError("pauli: empty string")
    table = {"I": I, "X": X, "Y": Y, "Z": Z}
    ops = []
    for i, ch in enumerate(s):
        if ch not in table:
            raise ValueError(f"pauli: invalid character {ch!r} at position {i}")
        ops.append(table[ch])
    return PauliString(1, ops, len(s))


def ZOn(qubits, num_qubits):
    return NewPauliString(1, {q: Z for q in qubits}, num_qubits)


class PauliSum:
    def __init__(self, terms):
        if not terms:
            raise ValueError("pauli: empty term list")
        nq = terms[0].NumQubits()
        for i, t in enumerate(terms[1:]):
            if t.NumQubits() != nq:
                raise ValueError(f"pauli: term {i + 1} has {t.NumQubits()} qubits, expected {nq}")
        self._terms = list(terms)
        self._n = nq

    def Terms(self):
        return list(self._terms)

    def NumQubits(self):
        return self._n


def NewPauliSum(terms):
    return PauliSum(terms)


def to_terms(obj):
    """ctypes array of gq_pauli_term for a PauliString or PauliSum."""
    terms = obj.Terms() if isinstance(obj, PauliSum) else [obj]
    arr = (_abi.gq_pauli_term * len(terms))()
    for k, t in enumerate(terms):
        arr[k].coeff_re = t.Coeff().real
        arr[k].coeff_im = t.Coeff().imag
        arr[k].x_mask = t.XMask()
        arr[k].z_mask = t.ZMask()
    return arr
