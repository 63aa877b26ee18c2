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


def _op_dtype():
    f = _abi.gq_op
    return np.dtype({
        "names": ["kind", "num_qubits", "num_controls", "num_kraus", "qubits", "matrix", "param_index", "reserved",
                  "dmatrix"],
        "formats": [np.int32, np.int32, np.int32, np.int32, (np.int32, _abi.GQ_MAX_OP_QUBITS), np.uint64,
                    (np.int32, _abi.GQ_MAX_OP_PARAMS), np.int32, (np.uint64, _abi.GQ_MAX_OP_PARAMS)],
        "offsets": [f.kind.offset, f.num_qubits.offset, f.num_controls.offset, f.num_kraus.offset, f.qubits.offset,
                    f.matrix.offset, f.param_index.offset, f.reserved.offset, f.dmatrix.offset],
        "itemsize": ctypes.sizeof(f)})


_OP_DTYPE = _op_dtype()


class OpStream:
    """gq_op records (a numpy array with the struct's layout, built once the
    stream is complete) plus one buffer holding every matrix they point to."""

    _PAD = (0,) * _abi.GQ_MAX_OP_QUBITS

    def __init__(self, num_qubits):
        self.num_qubits = num_qubits
        self._hdr = []   # (kind, num_qubits, num_controls, num_kraus)
        self._qub = []   # qubits padded to GQ_MAX_OP_QUBITS
        self._pidx = []  # param indices padded with -1
        self._mats = []  # complex128 arrays, in order
        self._nmat = 0   # complex entries so far
        self._moff = []  # (record, field (-1 = matrix, k = dmatrix[k]), entry offset)
        self._rec = None
        self._data = None
        self.n_params = 0

    def _slot(self, m):
        a = np.asarray(m, dtype=np.complex128).reshape(-1)
        off = self._nmat
        self._mats.append(a)
        self._nmat += a.size
        return off

    def add(self, kind, qubits, matrix=None, num_controls=0, num_kraus=0, params=()):
        nq = len(qubits)
        if nq > _abi.GQ_MAX_OP_QUBITS:
            raise ValueError(f"op on {nq} qubits exceeds {_abi.GQ_MAX_OP_QUBITS}")
        i = len(self._hdr)
        self._hdr.append((kind, nq, num_controls, num_kraus))
        self._qub.append(tuple(qubits) + self._PAD[nq:])
        if matrix is not None:
            self._moff.append((i, -1, self._slot(matrix)))
        pi = [-1, -1, -1]
        for k, (pidx, dm) in enumerate(params):
            pi[k] = pidx
            self._moff.append((i, k, self._slot(dm)))
        self._pidx.append(pi)
        self._rec = None

    def __len__(self):
        return len(self._hdr)

    def _finish(self):
        if self._rec is not None:
            return
        n = len(self._hdr)
        rec = np.zeros(max(1, n), dtype=_OP_DTYPE)
        if n:
            h = np.array(self._hdr, dtype=np.int32)
            rec["kind"][:n], rec["num_qubits"][:n] = h[:, 0], h[:, 1]
            rec["num_controls"][:n], rec["num_kraus"][:n] = h[:, 2], h[:, 3]
            rec["qubits"][:n] = np.array(self._qub, dtype=np.int32)
            rec["param_index"][:n] = np.array(self._pidx, dtype=np.int32)
        data = np.concatenate(self._mats) if self._mats else np.zeros(1, dtype=np.complex128)
        self._data = np.ascontiguousarray(data)
        if self._moff:
            m = np.array(self._moff, dtype=np.int64)
            addr = (self._data.ctypes.data + 16 * m[:, 2]).astype(np.uint64)
            sel = m[:, 1] < 0
            rec["matrix"][m[sel, 0]] = addr[sel]
            for k in range(_abi.GQ_MAX_OP_PARAMS):
                sk = m[:, 1] == k
                rec["dmatrix"][m[sk, 0], k] = addr[sk]
        self._rec = rec

    def array(self):
        """The records as a ctypes gq_op array (a view of the same memory)."""
        self._finish()
        return (_abi.gq_op * max(1, len(self._hdr))).from_buffer(self._rec)

    def ptr(self):
        self._finish()
        return ctypes.cast(self._rec.ctypes.data, ctypes.POINTER(_abi.gq_op))


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
        if g is None:
            continue
        d = getattr(g, "directive", None)
        if d == "barrier" or d == "delay":
            continue
        if d == "reset":
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
        d = None if g is None else getattr(g, "directive", None)
        if g is None or d == "barrier":
            continue
        if getattr(g, "noise_only", None):  # a channel without its gate (dynamic resets)
            channel(g.noise_only, op.Qubits)
            continue
        if d == "delay":
            channel("delay", op.Qubits)
            continue
        if d == "reset":
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


# ---- parameterized templates (gq_sv_adjoint_template / gq_sv_minimize_adam) --

def _affine(expr, index):
    """(parameter index or -1, scale, shift) of an expression that is affine
    in at most one parameter, else None."""
    from . import param as _param
    if isinstance(expr, _param._Literal):
        return (-1, 0.0, expr.v)
    if isinstance(expr, _param.Parameter):
        i = index.get(expr.Name())
        return None if i is None else (i, 1.0, 0.0)
    if isinstance(expr, _param._Neg):
        a = _affine(expr.inner, index)
        return None if a is None else (a[0], -a[1], -a[2])
    if isinstance(expr, _param._BinOp):
        a, b = _affine(expr.left, index), _affine(expr.right, index)
        if a is None or b is None:
            return None
        if expr.op in "+-":
            sg = 1.0 if expr.op == "+" else -1.0
            if a[0] >= 0 and b[0] >= 0 and a[0] != b[0]:
                return None
            p = a[0] if a[0] >= 0 else b[0]
            return (p, a[1] + sg * b[1], a[2] + sg * b[2])
        if expr.op == "*":
            if a[0] < 0:
                return (b[0], a[2] * b[1], a[2] * b[2])
            if b[0] < 0:
                return (a[0], b[2] * a[1], b[2] * a[2])
            return None
        if expr.op == "/" and b[0] < 0 and b[2] != 0.0:
            return (a[0], a[1] / b[2], a[2] / b[2])
    return None


class Template:
    """A circuit's op stream with its symbolic gates as gq_param_gate entries
    the library rebinds from parameter values (angles affine in one
    parameter each). `ops` holds the stream; `pgates` the entries."""

    def __init__(self, ops, pgates, n_params):
        self.ops = ops
        self.pgates = pgates
        self.n_params = n_params

    def pgate_ptr(self):
        return ctypes.cast(self.pgates, ctypes.POINTER(_abi.gq_param_gate)) if len(self.pgates) else None


def param_template(circuit, param_names, x0=None):
    """The Template of `circuit` for parameters `param_names` (raises
    ValueError when a symbolic gate's family or expression cannot be bound
    by the library). Symbolic ops carry their matrix at x0 as a placeholder."""
    names = list(param_names)
    index = {nm: i for i, nm in enumerate(names)}
    x0 = np.zeros(len(names)) if x0 is None else np.asarray(x0, dtype=np.float64)
    bindings = {nm: float(x0[i]) for i, nm in enumerate(names)}
    stream = OpStream(circuit.NumQubits())
    stream.n_params = len(names)
    entries = []
    for op in circuit.Ops():
        g = op.Gate
        if g is None:
            continue
        d = getattr(g, "directive", None)
        if d == "barrier" or d == "delay":
            continue
        if d == "reset":
            raise ValueError("template: reset is not unitary")
        if hasattr(g, "Bind"):
            fam = _abi.GQ_PG.get(g.base_name)
            if fam is None:
                raise ValueError(f"template: symbolic gate {g.base_name} has no library binding")
            coeffs = [_affine(e, index) for e in g.exprs]
            if any(a is None for a in coeffs):
                raise ValueError(f"template: {g.Name()} is not affine in one parameter per angle")
            e = _abi.gq_param_gate()
            e.op_index = len(stream)
            e.gate = fam
            e.num_angles = len(coeffs)
            for k, (p, sc, sh) in enumerate(coeffs):
                e.param[k], e.scale[k], e.shift[k] = p, sc, sh
            entries.append(e)
            _gate_record(stream, g.Bind(bindings), op.Qubits)
            continue
        _gate_record(stream, g, op.Qubits)
    return Template(stream, (_abi.gq_param_gate * len(entries))(*entries) if entries else [], len(names))
