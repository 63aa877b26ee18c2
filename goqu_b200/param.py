"""Symbolic parameters and gates (goqu circuit/param).

``Parameter`` / ``Vector`` (param.go:10-60, names ``"θ[i]"``), expressions
(expr.go: Literal, Add, Sub, Mul, Div, Neg) and symbolic gates that bind
through their constructor (gate.go:13-200). Expressions also differentiate
themselves, which the adjoint gradient uses for the chain rule.
"""
from __future__ import annotations

import math

import numpy as np

from . import gate as _gate


class Expr:
    def Eval(self, bindings):
        raise NotImplementedError

    def Parameters(self):
        raise NotImplementedError

    def IsNumeric(self):
        return not self.Parameters()

    def Deriv(self, name, bindings):
        """d(self)/d(name) at `bindings`."""
        raise NotImplementedError


class _Literal(Expr):
    def __init__(self, v):
        self.v = float(v)

    def Eval(self, bindings):
        return self.v

    def Parameters(self):
        return []

    def Deriv(self, name, bindings):
        return 0.0

    def __str__(self):
        return repr(self.v)


def Literal(v):
    return _Literal(v)


class Parameter(Expr):
    """A named free parameter (param.go:10-28)."""

    def __init__(self, name):
        self._name = name

    def Name(self):
        return self._name

    def Expr(self):
        return self

    def Eval(self, bindings):
        if self._name not in bindings:
            raise KeyError(f"param: unbound parameter {self._name!r}")
        return float(bindings[self._name])

    def Parameters(self):
        return [self]

    def Deriv(self, name, bindings):
        return 1.0 if name == self._name else 0.0

    def __str__(self):
        return self._name


def New(name):
    return Parameter(name)


class Vector:
    """NewVector(name, size): parameters named "name[i]" (param.go:38-48)."""

    def __init__(self, name, size):
        self._name = name
        self._params = [Parameter(f"{name}[{i}]") for i in range(size)]

    def Name(self):
        return self._name

    def Size(self):
        return len(self._params)

    def At(self, i):
        if i < 0 or i >= len(self._params):
            raise IndexError(f"param.Vector.At: index {i} out of range [0, {len(self._params)})")
        return self._params[i]

    def Names(self):
        return [p.Name() for p in self._params]


def NewVector(name, size):
    return Vector(name, size)


def _merge(a, b):
    seen, out = set(), []
    for p in a + b:
        if p.Name() not in seen:
            seen.add(p.Name())
            out.append(p)
    return out


class _BinOp(Expr):
    def __init__(self, op, left, right):
        self.op, self.left, self.right = op, left, right

    def Eval(self, b):
        x, y = self.left.Eval(b), self.right.Eval(b)
        if self.op == "+":
            return x + y
        if self.op == "-":
            return x - y
        if self.op == "*":
            return x * y
        if y == 0:
            raise ZeroDivisionError("param: division by zero")
        return x / y

    def Parameters(self):
        return _merge(self.left.Parameters(), self.right.Parameters())

    def Deriv(self, name, b):
        dx, dy = self.left.Deriv(name, b), self.right.Deriv(name, b)
        if self.op == "+":
            return dx + dy
        if self.op == "-":
            return dx - dy
        x, y = self.left.Eval(b), self.right.Eval(b)
        if self.op == "*":
            return dx * y + x * dy
        return (dx * y - x * dy) / (y * y)

    def __str__(self):
        return f"({self.left} {self.op} {self.right})"


class _Neg(Expr):
    def __init__(self, inner):
        self.inner = inner

    def Eval(self, b):
        return -self.inner.Eval(b)

    def Parameters(self):
        return self.inner.Parameters()

    def Deriv(self, name, b):
        return -self.inner.Deriv(name, b)

    def __str__(self):
        return f"(-{self.inner})"


def _e(x):
    return x if isinstance(x, Expr) else Literal(x)


def Add(a, b):
    return _BinOp("+", _e(a), _e(b))


def Sub(a, b):
    return _BinOp("-", _e(a), _e(b))


def Mul(a, b):
    return _BinOp("*", _e(a), _e(b))


def Div(a, b):
    return _BinOp("/", _e(a), _e(b))


def Neg(a):
    return _Neg(_e(a))


# 5-point central stencil step for matrix derivatives: the gate matrices are
# trigonometric in their arguments, so the truncation error is ~h^4 ~ 1e-12.
_H = 1e-3


class SymbolicGate(_gate.Gate):
    """An unbound parameterized gate (circuit/param/gate.go:13-91)."""

    def __init__(self, base_name, n, exprs, constructor):
        super().__init__(base_name, n, None)
        self.base_name = base_name
        self.exprs = [_e(x) for x in exprs]
        self.constructor = constructor

    def Name(self):
        return f"{self.base_name}({{{','.join(str(e) for e in self.exprs)}}})"

    def Matrix(self):
        raise ValueError(f"param: cannot compute matrix for unbound symbolic gate {self.Name()}; call Bind() first")

    def Params(self):
        return None

    def Inverse(self):
        # param/gate.go:37-49: negate the expressions, keep the constructor
        return SymbolicGate(self.base_name + "†", self._n, [Neg(e) for e in self.exprs], self.constructor)

    def Bind(self, bindings):
        vals = [e.Eval(bindings) for e in self.exprs]
        return self.constructor(vals)

    def FreeParameters(self):
        names = self.__dict__.get("_free")
        if names is None:  # expressions are immutable: computed once per gate
            seen, names = set(), []
            for e in self.exprs:
                for p in e.Parameters():
                    if p.Name() not in seen:
                        seen.add(p.Name())
                        names.append(p.Name())
            self._free = names
        return list(names)

    def IsBound(self):
        return all(e.IsNumeric() for e in self.exprs)

    # exp(-i theta/2 G) with G^2 = I: dU/dtheta = U(theta + pi) / 2
    _SHIFT = {"RX", "RY", "RZ", "RXX", "RYY", "RZZ"}
    # diag(1, ..., 1, e^(i phi)): dU/dphi is i e^(i phi) on the last diagonal entry
    _PHASE = {"P", "CP", "U1"}

    def _dmatrix(self, k, vals):
        base = self.base_name.rstrip("†")
        if len(vals) == 1 and base in self._SHIFT:
            return self.constructor([vals[0] + math.pi]).Matrix() / 2
        if len(vals) == 1 and base in self._PHASE:
            u = np.asarray(self.constructor(vals).Matrix(), dtype=np.complex128)
            d = np.zeros_like(u)
            d[-1] = 1j * u[-1]
            return d
        if len(vals) == 1 and base == "GlobalPhase":
            return 1j * self.constructor(vals).Matrix()

        def m(v):
            vv = list(vals)
            vv[k] = v
            return self.constructor(vv).Matrix()

        x = vals[k]
        return (-m(x + 2 * _H) + 8 * m(x + _H) - 8 * m(x - _H) + m(x - 2 * _H)) / (12 * _H)

    def MatrixDerivative(self, name, bindings):
        """d(bound matrix)/d(parameter `name`) with the chain rule applied:
        closed forms for rotation and phase gates, a 5-point stencil otherwise."""
        vals = [e.Eval(bindings) for e in self.exprs]
        total = None
        for k, e in enumerate(self.exprs):
            de = e.Deriv(name, bindings)
            if de == 0.0:
                continue
            dm = self._dmatrix(k, vals)
            total = dm * de if total is None else total + dm * de
        if total is None:
            total = np.zeros_like(self.constructor(vals).Matrix())
        return total


def _sym(base, n, exprs, ctor):
    return SymbolicGate(base, n, exprs, ctor)


def SymRX(theta):
    return _sym("RX", 1, [theta], lambda v: _gate.RX(v[0]))


def SymRY(theta):
    return _sym("RY", 1, [theta], lambda v: _gate.RY(v[0]))


def SymRZ(theta):
    return _sym("RZ", 1, [theta], lambda v: _gate.RZ(v[0]))


def SymPhase(phi):
    return _sym("P", 1, [phi], lambda v: _gate.Phase(v[0]))


def SymU3(theta, phi, lam):
    return _sym("U3", 1, [theta, phi, lam], lambda v: _gate.U3(v[0], v[1], v[2]))


def SymCP(phi):
    return _sym("CP", 2, [phi], lambda v: _gate.CP(v[0]))


def SymRXX(theta):
    return _sym("RXX", 2, [theta], lambda v: _gate.RXX(v[0]))


def SymRYY(theta):
    return _sym("RYY", 2, [theta], lambda v: _gate.RYY(v[0]))


def SymRZZ(theta):
    return _sym("RZZ", 2, [theta], lambda v: _gate.RZZ(v[0]))


def SymU1(lam):
    return _sym("U1", 1, [lam], lambda v: _gate.U1(v[0]))


def SymU2(phi, lam):
    return _sym("U2", 1, [phi, lam], lambda v: _gate.U2(v[0], v[1]))


def SymRot(phi, theta, omega):
    return _sym("Rot", 1, [phi, theta, omega], lambda v: _gate.Rot(v[0], v[1], v[2]))


def SymFSim(theta, phi):
    return _sym("FSim", 2, [theta, phi], lambda v: _gate.FSim(v[0], v[1]))


def SymPSwap(phi):
    return _sym("PSwap", 2, [phi], lambda v: _gate.PSwap(v[0]))


def SymGlobalPhase(phi):
    return _sym("GlobalPhase", 1, [phi], lambda v: _gate.GlobalPhase(v[0]))
