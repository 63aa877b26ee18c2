"""Gate library: the same gates, names and matrices as goqu's circuit/gate.

Matrices are flat row-major ``numpy.complex128`` arrays of length 4^k; the
first listed qubit is the most significant bit of the local index
(circuit/gate/fixed.go:169-171, 316-317). Each gate carries ``kind``, the
dispatch tier goqu's simulator selects for it (pointer equality for the fixed
singletons, kernel2q.go:27-71; the optional interfaces ControlDiagonal2Q /
Diagonal2Q / ControlU2Q, gate.go:55-76; ControlledGate for >= 4 qubits,
sim/statevector/sim.go:146-152). The engine forwards it in ``gq_op.kind``.
"""
from __future__ import annotations

import cmath
import math

import numpy as np

from . import _abi

_S2 = 1.0 / math.sqrt(2.0)


class Gate:
    """A quantum gate (circuit/gate/gate.go:5-26)."""

    kind = _abi.GQ_OP_MATRIX

    def __init__(self, name, n, matrix, params=None, kind=None):
        self._name = name
        self._n = n
        self._matrix = None if matrix is None else np.asarray(matrix, dtype=np.complex128).reshape(-1)
        self._params = None if params is None else list(params)
        if kind is not None:
            self.kind = kind

    def Name(self):
        if callable(self._name):  # parameterised gates format their name on first use
            self._name = self._name()
        return self._name

    def Qubits(self):
        return self._n

    def Matrix(self):
        return self._matrix

    def Params(self):
        return self._params

    def Inverse(self):
        """Conjugate transpose (fixed.go:20-43, parameterized.go:23-42)."""
        dim = 1 << self._n
        m = self._matrix.reshape(dim, dim)
        inv = np.conj(m.T).reshape(-1)
        params = None if self._params is None else [-p for p in self._params]
        return Gate(self.Name() + "†", self._n, inv, params, kind=_inverse_kind(self.kind))

    def Decompose(self, qubits):
        return None

    def __repr__(self):
        return f"Gate({self._name})"


def _inverse_kind(kind):
    # Structural tiers survive inversion (controlDiag2Q.Inverse etc.,
    # parameterized.go:51-83); singletons other than the self-inverse ones do not.
    if kind in (_abi.GQ_OP_CTRL_DIAG_2Q, _abi.GQ_OP_DIAG_2Q, _abi.GQ_OP_CTRL_U_2Q):
        return kind
    return _abi.GQ_OP_MATRIX


class _Fixed(Gate):
    _SELF_INVERSE = {"I", "H", "X", "Y", "Z", "CNOT", "CZ", "SWAP", "CCX", "CSWAP", "ECR", "CCZ"}

    def Inverse(self):
        if self._name in self._SELF_INVERSE:
            return self
        pairs = {"S": "Sdg", "S†": "S", "T": "Tdg", "T†": "T"}
        if self._name in pairs:
            return globals()[pairs[self._name]]
        return Gate.Inverse(self)


def _fixed(name, n, entries, kind=_abi.GQ_OP_MATRIX):
    return _Fixed(name, n, entries, None, kind=kind)


# Single-qubit singletons (fixed.go:54-155).
I = _fixed("I", 1, [1, 0, 0, 1])
H = _fixed("H", 1, [_S2, _S2, _S2, -_S2])
X = _fixed("X", 1, [0, 1, 1, 0])
Y = _fixed("Y", 1, [0, -1j, 1j, 0])
Z = _fixed("Z", 1, [1, 0, 0, -1])
S = _fixed("S", 1, [1, 0, 0, 1j])
Sdg = _fixed("S†", 1, [1, 0, 0, -1j])
T = _fixed("T", 1, [1, 0, 0, complex(_S2, _S2)])
Tdg = _fixed("T†", 1, [1, 0, 0, complex(_S2, -_S2)])
SX = _fixed("SX", 1, [complex(0.5, 0.5), complex(0.5, -0.5), complex(0.5, -0.5), complex(0.5, 0.5)])

# Two-qubit singletons (fixed.go:163-311).
CNOT = _fixed("CNOT", 2, [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0], _abi.GQ_OP_CNOT)
CZ = _fixed("CZ", 2, [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, -1], _abi.GQ_OP_CZ)
SWAP = _fixed("SWAP", 2, [1, 0, 0, 0, 0, 0, 1, 0, 0, 1, 0, 0, 0, 0, 0, 1], _abi.GQ_OP_SWAP)
CY = _fixed("CY", 2, [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, -1j, 0, 0, 1j, 0], _abi.GQ_OP_CY)
ISWAP = _fixed("iSWAP", 2, [1, 0, 0, 0, 0, 0, 1j, 0, 0, 1j, 0, 0, 0, 0, 0, 1], _abi.GQ_OP_ISWAP)
ECR = _fixed("ECR", 2, [0, 0, _S2, 1j * _S2, 0, 0, 1j * _S2, _S2, _S2, -1j * _S2, 0, 0, -1j * _S2, _S2, 0, 0])
DCX = _fixed("DCX", 2, [1, 0, 0, 0, 0, 0, 0, 1, 0, 1, 0, 0, 0, 0, 1, 0])
CH = _fixed("CH", 2, [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, _S2, _S2, 0, 0, _S2, -_S2])
CSX = _fixed("CSX", 2, [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, complex(0.5, 0.5), complex(0.5, -0.5),
                        0, 0, complex(0.5, -0.5), complex(0.5, 0.5)])


def _perm_matrix(dim, pairs):
    m = np.eye(dim, dtype=np.complex128)
    for a, b in pairs:
        m[[a, b]] = m[[b, a]]
    return m.reshape(-1)


# Three-qubit singletons (fixed.go:313-365).
CCX = _fixed("CCX", 3, _perm_matrix(8, [(6, 7)]), _abi.GQ_OP_CCX)
CSWAP = _fixed("CSWAP", 3, _perm_matrix(8, [(5, 6)]), _abi.GQ_OP_CSWAP)
_ccz = np.eye(8, dtype=np.complex128)
_ccz[7, 7] = -1
CCZ = _fixed("CCZ", 3, _ccz.reshape(-1), _abi.GQ_OP_CCZ)

# Sycamore = FSim(pi/2, pi/6) (fixed.go:377-395).
Sycamore = _fixed("Sycamore", 2, [1, 0, 0, 0, 0, 0, -1j, 0, 0, -1j, 0, 0, 0, 0, 0,
                                  cmath.exp(complex(0, -math.pi / 6))], _abi.GQ_OP_SYCAMORE)


def _e(x):
    # cmplx.Exp(complex(0, x)) = complex(cos x, sin x)
    return cmath.exp(complex(0.0, x))


def _param(name, n, params, matrix, kind=_abi.GQ_OP_MATRIX):
    return Gate(name, n, matrix, params, kind=kind)


def _fmt(*vals):
    return ",".join(f"{v:.4f}" for v in vals)


# Parameterized gates (circuit/gate/parameterized.go:91-564).
def RX(theta):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    return _param(lambda: f"RX({_fmt(theta)})", 1, [theta], [complex(c, 0), complex(0, -s), complex(0, -s), complex(c, 0)])


def RY(theta):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    return _param(lambda: f"RY({_fmt(theta)})", 1, [theta], [complex(c, 0), complex(-s, 0), complex(s, 0), complex(c, 0)])


def RZ(theta):
    return _param(lambda: f"RZ({_fmt(theta)})", 1, [theta], [_e(-theta / 2), 0, 0, _e(theta / 2)])


def Phase(phi):
    return _param(lambda: f"P({_fmt(phi)})", 1, [phi], [1, 0, 0, _e(phi)])


def U3(theta, phi, lam):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    return _param(lambda: f"U3({_fmt(theta, phi, lam)})", 1, [theta, phi, lam],
                  [complex(c, 0), -_e(lam) * complex(s, 0), _e(phi) * complex(s, 0), _e(phi + lam) * complex(c, 0)])


def CP(phi):
    return _param(lambda: f"CP({_fmt(phi)})", 2, [phi], np.diag([1, 1, 1, _e(phi)]).reshape(-1), _abi.GQ_OP_CTRL_DIAG_2Q)


def CRZ(theta):
    return _param(lambda: f"CRZ({_fmt(theta)})", 2, [theta], np.diag([1, 1, _e(-theta / 2), _e(theta / 2)]).reshape(-1),
                  _abi.GQ_OP_CTRL_DIAG_2Q)


def _ctrl_u(u):
    m = np.eye(4, dtype=np.complex128)
    m[2:, 2:] = np.asarray(u, dtype=np.complex128).reshape(2, 2)
    return m.reshape(-1)


def CRX(theta):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    return _param(lambda: f"CRX({_fmt(theta)})", 2, [theta], _ctrl_u([complex(c, 0), complex(0, -s), complex(0, -s), complex(c, 0)]),
                  _abi.GQ_OP_CTRL_U_2Q)


def CRY(theta):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    return _param(lambda: f"CRY({_fmt(theta)})", 2, [theta], _ctrl_u([complex(c, 0), complex(-s, 0), complex(s, 0), complex(c, 0)]),
                  _abi.GQ_OP_CTRL_U_2Q)


def RXX(theta):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    cc, is_ = complex(c, 0), complex(0, -s)
    return _param(lambda: f"RXX({_fmt(theta)})", 2, [theta], [cc, 0, 0, is_, 0, cc, is_, 0, 0, is_, cc, 0, is_, 0, 0, cc])


def RYY(theta):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    cc, is_, nis = complex(c, 0), complex(0, s), complex(0, -s)
    return _param(lambda: f"RYY({_fmt(theta)})", 2, [theta], [cc, 0, 0, is_, 0, cc, nis, 0, 0, nis, cc, 0, is_, 0, 0, cc])


def RZZ(theta):
    em, ep = _e(-theta / 2), _e(theta / 2)
    return _param(lambda: f"RZZ({_fmt(theta)})", 2, [theta], [em, 0, 0, 0, 0, ep, 0, 0, 0, 0, ep, 0, 0, 0, 0, em],
                  _abi.GQ_OP_DIAG_2Q)


def ZZ(theta):
    em, ep = _e(-theta / 2), _e(theta / 2)
    return _param(lambda: f"ZZ({_fmt(theta)})", 2, [theta], np.diag([em, ep, ep, em]).reshape(-1), _abi.GQ_OP_DIAG_2Q)


def GPI(phi):
    return _param(lambda: f"GPI({_fmt(phi)})", 1, [phi], [0, _e(-phi), _e(phi), 0])


def GPI2(phi):
    inv = complex(_S2, 0)
    return _param(lambda: f"GPI2({_fmt(phi)})", 1, [phi], [inv, inv * complex(0, -1) * _e(-phi), inv * complex(0, -1) * _e(phi), inv])


def MS(phi0, phi1):
    inv = complex(_S2, 0)
    ep, em = _e(phi0 + phi1), _e(phi0 - phi1)
    mi = complex(0, -1)
    return _param(lambda: f"MS({_fmt(phi0, phi1)})", 2, [phi0, phi1],
                  [inv, 0, 0, inv * mi * ep.conjugate(), 0, inv, inv * mi * em, 0,
                   0, inv * mi * em.conjugate(), inv, 0, inv * mi * ep, 0, 0, inv])


def U1(lam):
    return _param(lambda: f"U1({_fmt(lam)})", 1, [lam], [1, 0, 0, _e(lam)])


def U2(phi, lam):
    s = complex(_S2, 0)
    return _param(lambda: f"U2({_fmt(phi, lam)})", 1, [phi, lam], [s, -_e(lam) * s, _e(phi) * s, _e(phi + lam) * s])


def Rot(phi, theta, omega):
    cth, sth = math.cos(theta / 2), math.sin(theta / 2)
    eipo, eimo = _e((phi + omega) / 2), _e((phi - omega) / 2)
    return _param(lambda: f"Rot({_fmt(phi, theta, omega)})", 1, [phi, theta, omega],
                  [eipo.conjugate() * complex(cth, 0), -eimo.conjugate() * complex(sth, 0),
                   eimo * complex(sth, 0), eipo * complex(cth, 0)])


def PhasedXZ(x, z, a):
    cx, sx = math.cos(math.pi * x / 2), math.sin(math.pi * x / 2)
    ez, ea = _e(math.pi * z), _e(math.pi * a)
    return _param(lambda: f"PhasedXZ({_fmt(x, z, a)})", 1, [x, z, a],
                  [complex(cx, 0), ea.conjugate() * complex(0, sx), ez * ea * complex(0, sx), ez * complex(cx, 0)])


def GlobalPhase(phi):
    ep = _e(phi)
    return _param(lambda: f"GlobalPhase({_fmt(phi)})", 1, [phi], [ep, 0, 0, ep])


def FSim(theta, phi):
    ct, st = math.cos(theta), math.sin(theta)
    return _param(lambda: f"FSim({_fmt(theta, phi)})", 2, [theta, phi],
                  [1, 0, 0, 0, 0, complex(ct, 0), complex(0, -st), 0, 0, complex(0, -st), complex(ct, 0), 0,
                   0, 0, 0, _e(-phi)])


def PSwap(phi):
    ep = _e(phi)
    return _param(lambda: f"PSwap({_fmt(phi)})", 2, [phi], [1, 0, 0, 0, 0, 0, ep, 0, 0, ep, 0, 0, 0, 0, 0, 1])


class ControlledGate(Gate):
    """Inner gate plus leading control qubits (circuit/gate/controlled.go:8-110)."""

    def __init__(self, inner, n_controls):
        self._inner = inner
        self._nc = n_controls
        super().__init__(f"C{n_controls}-{inner.Name()}", n_controls + inner.Qubits(), None, inner.Params())
        self.kind = _abi.GQ_OP_CONTROLLED if self._n >= 4 else _abi.GQ_OP_MATRIX

    def Inner(self):
        return self._inner

    def NumControls(self):
        return self._nc

    def Matrix(self):
        # Lazily built full matrix; panics beyond 10 qubits (controlled.go:84-110).
        if self._matrix is None:
            total = self.Qubits()
            if total > 10:
                raise ValueError(f"gate: Matrix() not supported for {total}-qubit controlled gate (max 10); "
                                 "use simulation kernel instead")
            dim = 1 << total
            inner_dim = 1 << self._inner.Qubits()
            m = np.eye(dim, dtype=np.complex128)
            m[dim - inner_dim:, dim - inner_dim:] = self._inner.Matrix().reshape(inner_dim, inner_dim)
            self._matrix = m.reshape(-1)
        return self._matrix

    def Inverse(self):
        return ControlledGate(self._inner.Inverse(), self._nc)


def Controlled(inner, n_controls):
    """controlled.go:27-51: well-known cases return the singletons."""
    if n_controls < 1:
        raise ValueError("gate: Controlled requires at least 1 control qubit")
    if n_controls == 1:
        if inner is X:
            return CNOT
        if inner is Z:
            return CZ
        if inner is Y:
            return CY
    if n_controls == 2 and inner is X:
        return CCX
    return ControlledGate(inner, n_controls)


def MCX(n_controls):
    return Controlled(X, n_controls)


def MCZ(n_controls):
    return Controlled(Z, n_controls)


def MCP(phi, n_controls):
    return Controlled(Phase(phi), n_controls)


class _Pseudo(Gate):
    def __init__(self, name, n, params=None):
        super().__init__(name, n, None, params)
        self.directive = name  # what the simulators switch on, without formatting names

    def Inverse(self):
        return self


# Pseudo-gates (circuit/gate/pseudo.go): no matrix; simulators treat them specially.
Reset = _Pseudo("reset", 1)


def Delay(duration, unit="ns"):
    g = _Pseudo("delay", 1, [duration])
    g.unit = unit
    return g


def Barrier(n):
    return _Pseudo("barrier", n)


def Unitary(name, matrix):
    """A user matrix gate (circuit/gate/unitary.go:36-88): must be unitary."""
    m = np.asarray(matrix, dtype=np.complex128).reshape(-1)
    dim = int(round(math.sqrt(m.size)))
    if dim * dim != m.size or dim & (dim - 1):
        raise ValueError("gate: matrix size is not a power-of-two square")
    n = dim.bit_length() - 1
    u = m.reshape(dim, dim)
    if not np.allclose(u @ u.conj().T, np.eye(dim), atol=1e-10):
        raise ValueError("gate: matrix is not unitary")
    return Gate(name, n, m)
