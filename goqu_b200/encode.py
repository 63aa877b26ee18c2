"""Circuit -> gq_op stream (the records the C ABI consumes).

This is the host half of the boundary: it walks ``Circuit.Ops()`` once, the way
goqu's Apply loop does (sim/statevector/sim.go:92-157), and emits one POD
record per operation with the gate's own matrix, so the engine and the oracle
see identical inputs. Errors mirror the reference's messages.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from . import gate as _gate


class OpStream:
    """A ctypes gq_op array plus the numpy buffers its pointers reference."""

    def __init__(self, num_qubits):
        self.num_qubits = num_qubits
        self._ops = []
        self._keep = []
        self._arr = None
        self.n_params = 0

    def _buf(self, m):
        a = np.ascontiguousarray(np.asarray(m, dtype=np.complex128).reshape(-1)).view(np.float64)
        self._keep.append(a)
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    def add(self, kind, qubits, matrix=None, num_controls=0, num_kraus=0, params=()):
        if len(qubits) > _abi.GQ_MAX_OP_QUBITS:
            raise ValueError(f"op on {len(qubits)} qubits exceeds {_abi.GQ_MAX_OP_QUBITS}")
        op = _abi.gq_op()
        op.kind = kind
        op.num_qubits = len(qubits)
        op.num_controls = num_controls
        op.num_kraus = num_kraus
        for i, q in enumerate(qubits):
            op.qubits[i] = q
        if matrix is not None:
            op.matrix = self._buf(matrix)
        for k in range(_abi.GQ_MAX_OP_PARAMS):
            op.param_index[k] = -1
        for k, (pidx, dm) in enumerate(params):
            op.param_index[k] = pidx
            op.dmatrix[k] = self._buf(dm)
        self._ops.append(op)
        self._arr = None

    def __len__(self):
        return len(self._ops)

    def array(self):
        if self._arr is None:
            self._arr = (_abi.gq_op * max(1, len(self._ops)))(*self._ops)
        return self._arr

    def ptr(self):
        return ctypes.cast(self.array(), ctypes.POINTER(_abi.gq_op))


def _gate_record(stream, g, qubits, params=()):
    """Emit one unitary op for gate g on qubits (Apply's size switch)."""
    n = g.Qubits()
    if n >= 4:
        if isinstance(g, _gate.ControlledGate):
            stream.add(_abi.GQ_OP_CONTROLLED, qubits, g.Inner().Matrix(), num_controls=g.NumControls(), params=params)
            return
        raise ValueError(f"unsupported gate size: {n} qubits")
    m = g.Matrix()
    if m is None:
        raise ValueError(f"gate {g.Name()!r} has no matrix representation")
    stream.add(g.kind, qubits, m, params=params)


def statevector_ops(circuit, bindings=None, param_names=None):
    """The op stream of Sim.Apply for `circuit` (sim/statevector/sim.go:92-157).

    With `bindings` and `param_names`, symbolic gates are bound and carry the
    derivative of their matrix with respect to each parameter they use.
    """
    stream = OpStream(circuit.NumQubits())
    index = {name: i for i, name in enumerate(param_names or [])}
    stream.n_params = len(index)
    for op in circuit.Ops():
        g = op.Gate
        if g is None or g.Name() in ("barrier", "delay"):
            continue
        if g.Name() == "reset":
            stream.add(_abi.GQ_OP_RESET, [op.Qubits[0]])
            continue
        if hasattr(g, "Bind"):
            if bindings is None:
                raise ValueError(f"param: cannot compute matrix for unbound symbolic gate {g.Name()}; call Bind() first")
            params = []
            for name in g.FreeParameters():
                if name in index:
                    params.append((index[name], g.MatrixDerivative(name, bindings)))
            if len(params) > _abi.GQ_MAX_OP_PARAMS:
                raise ValueError("op depends on more than three parameters")
            _gate_record(stream, g.Bind(bindings), op.Qubits, params)
            continue
        _gate_record(stream, g, op.Qubits)
    return stream


def density_ops(circuit, noise_model=None):
    """Op stream of densitymatrix Sim.Apply (sim/densitymatrix/sim.go:87-191):
    gates followed by the channel NoiseModel.Lookup selects for them."""
    stream = OpStream(circuit.NumQubits())

    def channel(name, qubits):
        if noise_model is None:
            return
        ch = noise_model.Lookup(name, qubits)
        if ch is None:
            return
        kraus = ch.Kraus()
        stream.add(_abi.GQ_OP_CHANNEL, list(qubits[:ch.Qubits()]), np.concatenate(kraus), num_kraus=len(kraus))

    for op in circuit.Ops():
        g = op.Gate
        if g is None or g.Name() == "barrier":
            continue
        if getattr(g, "noise_only", None):  # a channel without its gate (dynamic resets)
            channel(g.noise_only, op.Qubits)
            continue
        if g.Name() == "delay":
            channel("delay", op.Qubits)
            continue
        if g.Name() == "reset":
            stream.add(_abi.GQ_OP_RESET, [op.Qubits[0]])
            channel("reset", op.Qubits)
            continue
        if g.Qubits() >= 3:
            # decomposeForDensity (sim.go:321-344) handles only controlled
            # single-qubit gates; the engine applies them exactly as one op.
            if not (isinstance(g, _gate.ControlledGate) and g.Inner().Qubits() == 1):
                raise ValueError(f"densitymatrix: unsupported gate size: {g.Qubits()} qubits")
            stream.add(_abi.GQ_OP_CONTROLLED, op.Qubits, g.Inner().Matrix(), num_controls=g.NumControls())
        else:
            m = g.Matrix()
            if m is None:
                continue
            stream.add(g.kind, op.Qubits, m)
        if not getattr(g, "noiseless", False):
            channel(g.Name(), op.Qubits)
    return stream
