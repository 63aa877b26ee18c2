"""Dynamic circuits: mid-circuit measurement, feed-forward, reset, control flow.

goqu simulates every shot on its own (RunDynamic, sim/statevector/dynamic.go:
14-177): reset to |0..0>, walk the ops, collapse the state at each
measurement with that shot's PCG draw, and branch on classical bits.

Here the walk is the same, but shots that share a measurement history share
one device state: a group of shots runs its gates once, and a measurement
splits it by the shots' own uniforms (outcome 1 iff u >= P(0), dynamic.go:
197-200); a split copies the state on the device (gq_sv_copy_state) and each
side collapses (gq_sv_collapse). The outcome of every shot is the one its
own walk would give, so the counts match a per-shot loop over the same
uniforms; the work is one walk per distinct history, not per shot.

Uniforms: shot s's k-th draw (measurements and dynamic resets, in walk
order) is uniforms[s, k]. Without them they are drawn from ``rng``.
"""
from __future__ import annotations

import numpy as np

from . import _abi, encode as _encode, gate as _gate
from . import circuit as ir


class _Uniforms:
    def __init__(self, shots, rng, uniforms):
        self.shots = shots
        if uniforms is not None:
            u = np.asarray(uniforms, dtype=np.float64)
            if u.ndim != 2 or u.shape[0] != shots:
                raise ValueError(f"uniforms must have shape (shots, draws), got {u.shape}")
            self.u, self.rng = u, None
        else:
            self.rng = rng if rng is not None else np.random.default_rng()
            self.u = self.rng.random((shots, 8))

    def column(self, k):
        while k >= self.u.shape[1]:
            if self.rng is None:
                raise ValueError(f"a shot needs more than {self.u.shape[1]} uniforms")
            self.u = np.concatenate([self.u, self.rng.random((self.shots, self.u.shape[1]))], axis=1)
        return self.u[:, k]


class _Group:
    __slots__ = ("state", "shots", "clbits", "draws", "pending")

    def __init__(self, state, shots, clbits, draws, pending):
        self.state, self.shots, self.clbits, self.draws, self.pending = state, shots, clbits, draws, pending


class ResetNoise:
    """Marker op of the density-matrix walk: the noise model's "reset" channel
    on its qubits, applied after a dynamic reset's measure-and-flip
    (sim/densitymatrix/dynamic.go:85-97)."""

    noise_only = "reset"

    def Name(self):
        return "reset-noise"

    def Qubits(self):
        return 1


class NoiselessGate:
    """A gate the density-matrix walk applies without its noise channel: the
    X of a dynamic reset (applyGate1 directly, sim/densitymatrix/dynamic.go:87-89)."""

    noiseless = True

    def __init__(self, g):
        self._g = g
        self.kind = g.kind

    def Name(self):
        return self._g.Name()

    def Qubits(self):
        return self._g.Qubits()

    def Matrix(self):
        return self._g.Matrix()


class EngineBackend:
    """Device states of one qubit count and precision (gq_sv handles), reused
    through a free list; `max_states` bounds the live ones."""

    keeps_delays = False  # statevector: delays are no-ops (dynamic.go:72-75)

    def __init__(self, sim, max_states=None):
        from . import statevector
        self._sv = statevector
        self.n, self.prec = sim.NumQubits(), sim._prec
        self.free_list, self.live = [], 0
        if max_states is None:
            max_states = max(2, (16 << 30) // ((8 if self.prec == _abi.GQ_C64 else 16) << self.n))
        self.max_states = max_states

    def _new(self):
        if self.live >= self.max_states:
            raise MemoryError(f"dynamic circuit: more than {self.max_states} distinct measurement histories "
                              f"alive at once for {self.n} qubits; run fewer shots per call")
        self.live += 1
        return self.free_list.pop() if self.free_list else self._sv.New(self.n, self.prec)

    def fresh(self):
        s = self._new()
        s.Reset()
        return s

    def copy(self, s):
        d = self._new()
        _abi.check(_abi.lib().gq_sv_copy_state(d.handle, s.handle))
        return d

    def release(self, s):
        self.live -= 1
        self.free_list.append(s)

    def apply(self, s, ops):
        stream = _encode.statevector_ops(ir.Circuit("", self.n, 0, ops))
        if len(stream):
            s.apply_ops(stream)

    def prob0(self, s, q):
        import ctypes
        p = ctypes.c_double()
        _abi.check(_abi.lib().gq_sv_prob0(s.handle, q, ctypes.byref(p)))
        return p.value

    def collapse(self, s, q, outcome, p0):
        _abi.check(_abi.lib().gq_sv_collapse(s.handle, q, outcome, p0))

    def close(self):
        for s in self.free_list:
            s.Close()
        self.free_list = []


class DensityBackend(EngineBackend):
    """Device density matrices (gq_dm handles) with the simulator's noise
    model: gates are followed by their channels, delays and dynamic resets
    by theirs (sim/densitymatrix/dynamic.go:53-121)."""

    keeps_delays = True

    def __init__(self, sim, max_states=None):
        from . import densitymatrix
        self._dm = densitymatrix
        self.n, self.noise = sim.NumQubits(), sim._noise
        self.free_list, self.live = [], 0
        if max_states is None:
            max_states = max(2, (16 << 30) // (16 << (2 * self.n)))
        self.max_states = max_states

    def _new(self):
        if self.live >= self.max_states:
            raise MemoryError(f"dynamic circuit: more than {self.max_states} distinct measurement histories "
                              f"alive at once for a {self.n}-qubit density matrix; run fewer shots per call")
        self.live += 1
        return self.free_list.pop() if self.free_list else self._dm.New(self.n)

    def copy(self, s):
        d = self._new()
        _abi.check(_abi.lib().gq_dm_copy_state(d._h, s._h))
        return d

    def apply(self, s, ops):
        stream = _encode.density_ops(ir.Circuit("", self.n, 0, ops), self.noise)
        if len(stream):
            _abi.check(_abi.lib().gq_dm_apply(s._h, stream.ptr(), len(stream)))

    def prob0(self, s, q):
        import ctypes
        p = ctypes.c_double()
        _abi.check(_abi.lib().gq_dm_prob0(s._h, q, ctypes.byref(p)))
        return p.value

    def collapse(self, s, q, outcome, p0):
        _abi.check(_abi.lib().gq_dm_collapse(s._h, q, outcome, p0))


def _flush(be, g):
    if g.pending:
        be.apply(g.state, g.pending)
        g.pending = []


def _measure(be, g, qubit, U):
    """Splits g by its shots' next draw; returns [(group, outcome)]."""
    _flush(be, g)
    p0 = be.prob0(g.state, qubit)
    u = U.column(g.draws)[g.shots]
    one = u >= p0
    parts = []
    for outcome, sel in ((0, ~one), (1, one)):
        if sel.any():
            parts.append((outcome, g.shots[sel]))
    out = []
    for i, (outcome, shots) in enumerate(parts):
        st = g.state if i == len(parts) - 1 else be.copy(g.state)
        be.collapse(st, qubit, outcome, p0)
        out.append((_Group(st, shots, list(g.clbits), g.draws + 1, []), outcome))
    return out


def _exec(be, groups, ops, U):
    for op in ops:
        nxt = []
        for g in groups:
            nxt.extend(_exec_op(be, g, op, U))
        groups = nxt
    return groups


def _exec_op(be, g, op, U):
    cf = op.ControlFlow
    if cf is not None:
        return _exec_cf(be, g, cf, U)
    if op.Gate is None:  # measurement: nil gate with clbits (dynamic.go:64-70)
        if op.Clbits and op.Qubits:
            out = []
            for ng, outcome in _measure(be, g, op.Qubits[0], U):
                ng.clbits[op.Clbits[0]] = outcome
                out.append(ng)
            return out
        return [g]
    name = getattr(op.Gate, "directive", None)
    if name == "barrier":
        return [g]
    if name == "delay":
        if be.keeps_delays:
            g.pending.append(ir.Operation(op.Gate, list(op.Qubits)))
        return [g]
    if name == "reset":  # measure, then X on outcome 1 (dynamic.go:78-85)
        out = []
        for ng, outcome in _measure(be, g, op.Qubits[0], U):
            if outcome == 1:
                x = NoiselessGate(_gate.X) if be.keeps_delays else _gate.X
                ng.pending.append(ir.Operation(x, [op.Qubits[0]]))
            if be.keeps_delays:
                ng.pending.append(ir.Operation(ResetNoise(), [op.Qubits[0]]))
            out.append(ng)
        return out
    c = op.Condition
    if c is not None and g.clbits[c.clbit] != c.value:
        return [g]
    g.pending.append(ir.Operation(op.Gate, list(op.Qubits)))
    return [g]


def _exec_cf(be, g, cf, U):
    """executeControlFlow (dynamic.go:101-143), per group."""
    if cf.Type == ir.ControlFlowWhile:
        done, active = [], [g]
        for _ in range(ir.MaxControlFlowIterations):
            run = [x for x in active if x.clbits[cf.Condition.clbit] == cf.Condition.value]
            done.extend(x for x in active if x.clbits[cf.Condition.clbit] != cf.Condition.value)
            if not run:
                active = []
                break
            active = _exec(be, run, cf.Bodies[0], U)
        return done + active
    if cf.Type == ir.ControlFlowFor:
        r = cf.ForRange
        if r.Step <= 0 and r.Start < r.End:
            raise ValueError("for loop never reaches its end")
        groups, i = [g], r.Start
        while i < r.End:
            groups = _exec(be, groups, cf.Bodies[0], U)
            i += r.Step
        return groups
    if cf.Type == ir.ControlFlowIfElse:
        if g.clbits[cf.Condition.clbit] == cf.Condition.value:
            return _exec(be, [g], cf.Bodies[0], U)
        if len(cf.Bodies) > 1:
            return _exec(be, [g], cf.Bodies[1], U)
        return [g]
    if cf.Type == ir.ControlFlowSwitch:
        val = 0
        for i, idx in enumerate(cf.SwitchArg.Clbits):  # little-endian (dynamic.go:146-153)
            val |= g.clbits[idx] << i
        for i, case in enumerate(cf.SwitchArg.Cases):
            if val == case and i < len(cf.Bodies):
                return _exec(be, [g], cf.Bodies[i], U)
        if len(cf.Bodies) > len(cf.SwitchArg.Cases):
            return _exec(be, [g], cf.Bodies[-1], U)
        return [g]
    raise ValueError(f"unknown control flow type {cf.Type}")


def bitstring(clbits):
    """Classical bits as goqu prints them: clbit n-1 first (dynamic.go:38-46)."""
    return "".join("1" if v else "0" for v in reversed(clbits))


def run_groups(be, circuit, shots, rng=None, uniforms=None):
    """The walk over groups; returns the final groups (state, shots, clbits)."""
    if shots <= 0:
        raise ValueError(f"shots must be positive, got {shots}")
    U = _Uniforms(shots, rng, uniforms)
    g0 = _Group(be.fresh(), np.arange(shots), [0] * circuit.NumClbits(), 0, [])
    groups = _exec(be, [g0], circuit.Ops(), U)
    for g in groups:
        _flush(be, g)
    return groups


def run_dynamic_dm(sim, circuit, shots, rng=None, uniforms=None, max_states=None):
    """densitymatrix RunDynamic (sim/densitymatrix/dynamic.go:13-51); the
    simulator is left with the last shot's final density matrix."""
    if circuit.NumQubits() != sim.NumQubits():
        raise ValueError(f"circuit has {circuit.NumQubits()} qubits, simulator has {sim.NumQubits()}")
    be = DensityBackend(sim, max_states)
    try:
        groups = run_groups(be, circuit, shots, rng, uniforms)
        counts = {}
        for g in groups:
            key = bitstring(g.clbits)
            counts[key] = counts.get(key, 0) + int(g.shots.size)
            if (g.shots == shots - 1).any():
                _abi.check(_abi.lib().gq_dm_copy_state(sim._h, g.state._h))
            be.release(g.state)
        return counts
    finally:
        be.close()


def run_dynamic(sim, circuit, shots, rng=None, uniforms=None, max_states=None):
    """RunDynamic: counts of classical-bit strings over `shots` shots. The
    simulator's state is left as the last shot's final state, as in goqu."""
    if circuit.NumQubits() != sim.NumQubits():
        raise ValueError(f"circuit has {circuit.NumQubits()} qubits, simulator has {sim.NumQubits()}")
    be = EngineBackend(sim, max_states)
    try:
        groups = run_groups(be, circuit, shots, rng, uniforms)
        counts = {}
        for g in groups:
            key = bitstring(g.clbits)
            counts[key] = counts.get(key, 0) + int(g.shots.size)
            if (g.shots == shots - 1).any():
                _abi.check(_abi.lib().gq_sv_copy_state(sim.handle, g.state.handle))
            be.release(g.state)
        return counts
    finally:
        be.close()
