"""Circuit IR and builder (goqu circuit/ir and circuit/builder).

``Operation`` (ir/circuit.go:79-85), an immutable ``Circuit`` with ``Bind``
(:206-250), ``FreeParameters`` in first-appearance order (:253-280) and
``IsDynamic`` (:298-322), and a ``Builder`` with the method names of
circuit/builder/builder.go that the simulator path uses.
"""
from __future__ import annotations

from dataclasses import dataclass, field

from . import gate as _gate
from . import param as _param


@dataclass
class Condition:
    clbit: int
    value: int


# Structured control flow (ir/circuit.go:94-129).
ControlFlowWhile, ControlFlowFor, ControlFlowSwitch, ControlFlowIfElse = 1, 2, 3, 4
MaxControlFlowIterations = 1000  # while-loop cap at simulation time


@dataclass
class ForRange:
    Start: int
    End: int  # exclusive
    Step: int


@dataclass
class SwitchArg:
    Clbits: list
    Cases: list  # case value of each body, in order


@dataclass
class ControlFlow:
    Type: int
    Condition: object = None  # While and IfElse
    Bodies: list = field(default_factory=list)  # While[0], IfElse[0]/[1], Switch[i] (+ default last)
    ForRange: object = None
    SwitchArg: object = None


@dataclass
class Operation:
    Gate: object = None
    Qubits: list = field(default_factory=list)
    Clbits: list = field(default_factory=list)
    Condition: object = None
    ControlFlow: object = None


class Circuit:
    def __init__(self, name, num_qubits, num_clbits, ops, metadata=None):
        self._name = name
        self._nq = num_qubits
        self._nc = num_clbits
        self._ops = list(ops)
        self._meta = dict(metadata or {})

    def Name(self):
        return self._name

    def NumQubits(self):
        return self._nq

    def NumClbits(self):
        return self._nc

    def Ops(self):
        return list(self._ops)

    def NumOps(self):
        return len(self._ops)

    def Op(self, i):
        return self._ops[i]

    def Metadata(self):
        return dict(self._meta)

    def IsDynamic(self):
        """ir/circuit.go:298-322."""
        last_gate = -1
        for i in range(len(self._ops) - 1, -1, -1):
            g = self._ops[i].Gate
            if g is not None and getattr(g, "directive", None) not in ("barrier", "reset"):
                last_gate = i
                break
        for i, op in enumerate(self._ops):
            if op.ControlFlow is not None or op.Condition is not None:
                return True
            if op.Gate is not None and getattr(op.Gate, "directive", None) == "reset":
                return True
            if op.Gate is None and op.Clbits and i < last_gate:
                return True
        return False


def Bind(c, bindings):
    """ir.Bind (ir/circuit.go:206-250)."""
    out = []
    for op in c.Ops():
        g = op.Gate
        if g is not None and hasattr(g, "Bind"):
            out.append(Operation(g.Bind(bindings), list(op.Qubits), list(op.Clbits), op.Condition))
        else:
            out.append(op)
    return Circuit(c.Name(), c.NumQubits(), c.NumClbits(), out, c.Metadata())


def FreeParameters(c):
    """Names in first-appearance order (ir/circuit.go:253-280)."""
    seen, names = set(), []
    for op in c.Ops():
        g = op.Gate
        if g is not None and hasattr(g, "FreeParameters"):
            for n in g.FreeParameters():
                if n not in seen:
                    seen.add(n)
                    names.append(n)
    return names


class Builder:
    """Fluent circuit construction (circuit/builder/builder.go)."""

    def __init__(self, name, num_qubits):
        self._name = name
        self._nq = num_qubits
        self._nc = 0
        self._ops = []
        self._err = None

    def WithClbits(self, n):
        self._nc = n
        return self

    def _check(self, qubits, arity):
        if self._err:
            return False
        if len(qubits) != arity:
            self._err = ValueError(f"gate expects {arity} qubits, got {len(qubits)}")
            return False
        for q in qubits:
            if q < 0 or q >= self._nq:
                self._err = ValueError(f"qubit {q} out of range [0, {self._nq})")
                return False
        if len(set(qubits)) != len(qubits):
            self._err = ValueError(f"duplicate qubits {qubits}")
            return False
        return True

    def Apply(self, g, *qubits):
        if self._check(list(qubits), g.Qubits()):
            self._ops.append(Operation(g, list(qubits)))
        return self

    # Fixed gates.
    def H(self, q): return self.Apply(_gate.H, q)
    def X(self, q): return self.Apply(_gate.X, q)
    def Y(self, q): return self.Apply(_gate.Y, q)
    def Z(self, q): return self.Apply(_gate.Z, q)
    def S(self, q): return self.Apply(_gate.S, q)
    def T(self, q): return self.Apply(_gate.T, q)
    def CNOT(self, c, t): return self.Apply(_gate.CNOT, c, t)
    def CZ(self, c, t): return self.Apply(_gate.CZ, c, t)
    def SWAP(self, a, b): return self.Apply(_gate.SWAP, a, b)
    def ISWAP(self, a, b): return self.Apply(_gate.ISWAP, a, b)
    def ECR(self, a, b): return self.Apply(_gate.ECR, a, b)
    def DCX(self, a, b): return self.Apply(_gate.DCX, a, b)
    def CH(self, c, t): return self.Apply(_gate.CH, c, t)
    def CSX(self, c, t): return self.Apply(_gate.CSX, c, t)
    def Sycamore(self, a, b): return self.Apply(_gate.Sycamore, a, b)
    def CCX(self, c0, c1, t): return self.Apply(_gate.CCX, c0, c1, t)
    def CCZ(self, c0, c1, t): return self.Apply(_gate.CCZ, c0, c1, t)

    def MCX(self, controls, target):
        return self.Apply(_gate.MCX(len(controls)), *controls, target)

    def MCZ(self, controls, target):
        return self.Apply(_gate.MCZ(len(controls)), *controls, target)

    def MCP(self, phi, controls, target):
        return self.Apply(_gate.MCP(phi, len(controls)), *controls, target)

    def Ctrl(self, g, controls, *targets):
        return self.Apply(_gate.Controlled(g, len(controls)), *controls, *targets)

    # Parameterized gates.
    def RX(self, t, q): return self.Apply(_gate.RX(t), q)
    def RY(self, t, q): return self.Apply(_gate.RY(t), q)
    def RZ(self, t, q): return self.Apply(_gate.RZ(t), q)
    def Phase(self, p, q): return self.Apply(_gate.Phase(p), q)
    def U3(self, t, p, l, q): return self.Apply(_gate.U3(t, p, l), q)
    def U1(self, l, q): return self.Apply(_gate.U1(l), q)
    def U2(self, p, l, q): return self.Apply(_gate.U2(p, l), q)
    def Rot(self, p, t, o, q): return self.Apply(_gate.Rot(p, t, o), q)
    def GlobalPhase(self, p, q): return self.Apply(_gate.GlobalPhase(p), q)
    def RXX(self, t, a, b): return self.Apply(_gate.RXX(t), a, b)
    def RYY(self, t, a, b): return self.Apply(_gate.RYY(t), a, b)
    def RZZ(self, t, a, b): return self.Apply(_gate.RZZ(t), a, b)
    def ZZ(self, t, a, b): return self.Apply(_gate.ZZ(t), a, b)
    def FSim(self, t, p, a, b): return self.Apply(_gate.FSim(t, p), a, b)
    def PSwap(self, p, a, b): return self.Apply(_gate.PSwap(p), a, b)

    def Unitary(self, name, matrix, *qubits):
        return self.Apply(_gate.Unitary(name, matrix), *qubits)

    # Symbolic gates (builder.go:288-360).
    def SymRX(self, e, q): return self.Apply(_param.SymRX(e), q)
    def SymRY(self, e, q): return self.Apply(_param.SymRY(e), q)
    def SymRZ(self, e, q): return self.Apply(_param.SymRZ(e), q)
    def SymPhase(self, e, q): return self.Apply(_param.SymPhase(e), q)
    def SymU3(self, t, p, l, q): return self.Apply(_param.SymU3(t, p, l), q)
    def SymCP(self, e, a, b): return self.Apply(_param.SymCP(e), a, b)
    def SymRXX(self, e, a, b): return self.Apply(_param.SymRXX(e), a, b)
    def SymRYY(self, e, a, b): return self.Apply(_param.SymRYY(e), a, b)
    def SymRZZ(self, e, a, b): return self.Apply(_param.SymRZZ(e), a, b)

    # Non-unitary instructions.
    def Measure(self, qubit, clbit):
        if self._check([qubit], 1):
            if clbit >= self._nc:
                self._nc = clbit + 1
            self._ops.append(Operation(None, [qubit], [clbit]))
        return self

    def MeasureAll(self):
        """builder.go:381-396: nil-gate ops, clbit i for qubit i."""
        if self._nc < self._nq:
            self._nc = self._nq
        for q in range(self._nq):
            self._ops.append(Operation(None, [q], [q]))
        return self

    def Reset(self, q):
        return self.Apply(_gate.Reset, q)

    # Classical control (builder.go:424-600).
    def _clbit(self, c):
        if self._err is None and c < 0:
            self._err = ValueError(f"clbit {c} out of range")
        if c >= self._nc:
            self._nc = c + 1
        return self._err is None

    def _sub(self, fn):
        sub = Builder(self._name, self._nq)
        sub._nc = self._nc
        fn(sub)
        if sub._err:
            self._err = sub._err
        self._nc = max(self._nc, sub._nc)
        return sub._ops

    def If(self, clbit, value, g, *qubits):
        """A gate applied only when clbit == value."""
        if self._clbit(clbit) and self._check(list(qubits), g.Qubits()):
            self._ops.append(Operation(g, list(qubits), Condition=Condition(clbit, value)))
        return self

    def IfBlock(self, clbit, value, fn):
        """Every op fn adds is conditioned on clbit == value."""
        if self._clbit(clbit):
            start = len(self._ops)
            fn(self)
            for op in self._ops[start:]:
                op.Condition = Condition(clbit, value)
        return self

    def IfElseBlock(self, clbit, value, if_body, else_body):
        if self._clbit(clbit):
            a, b = self._sub(if_body), self._sub(else_body)
            self._ops.append(Operation(ControlFlow=ControlFlow(ControlFlowIfElse, Condition(clbit, value), [a, b])))
        return self

    def While(self, clbit, value, body):
        if self._clbit(clbit):
            ops = self._sub(body)
            self._ops.append(Operation(ControlFlow=ControlFlow(ControlFlowWhile, Condition(clbit, value), [ops])))
        return self

    def For(self, clbit, start, end, step, body):
        if self._clbit(clbit):
            if step == 0:
                self._err = ValueError("for loop step must be non-zero")
                return self
            ops = self._sub(body)
            self._ops.append(Operation(ControlFlow=ControlFlow(ControlFlowFor, None, [ops],
                                                               ForRange=ForRange(start, end, step))))
        return self

    def Switch(self, clbits, cases, default_body=None):
        """cases: {value: body}; bodies in ascending case value, default last."""
        for c in clbits:
            self._clbit(c)
        if self._err:
            return self
        vals = sorted(cases)
        bodies = [self._sub(cases[v]) for v in vals]
        if default_body is not None:
            bodies.append(self._sub(default_body))
        self._ops.append(Operation(ControlFlow=ControlFlow(ControlFlowSwitch, None, bodies,
                                                           SwitchArg=SwitchArg(list(clbits), vals))))
        return self

    def Delay(self, q, duration, unit="ns"):
        return self.Apply(_gate.Delay(duration, unit), q)

    def Barrier(self, *qubits):
        qs = list(qubits) or list(range(self._nq))
        self._ops.append(Operation(_gate.Barrier(len(qs)), qs))
        return self

    def Build(self):
        if self._err:
            raise self._err
        return Circuit(self._name, self._nq, self._nc, self._ops)


def New(name, num_qubits):
    return Builder(name, num_qubits)
