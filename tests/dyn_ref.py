"""Per-shot restatement of goqu's RunDynamic (sim/statevector/dynamic.go:
14-177) on the oracle, for the dynamic-circuit tests: every shot starts from
|0..0>, applies gates with the oracle, measures with or_sv_measure (the
restated measureQubit) using uniforms[shot, k] for its k-th draw, and
branches on its classical bits. TEST INFRASTRUCTURE.
"""
import numpy as np

from goqu_b200 import circuit as ir, encode, gate as G
from oracle import binding as orc


def _apply(st, n, op_list):
    stream = encode.statevector_ops(ir.Circuit("", n, 0, op_list))
    if len(stream):
        orc.sv_apply(st, stream)


def _exec(ops, st, n, clbits, draw):
    for op in ops:
        cf = op.ControlFlow
        if cf is not None:
            _exec_cf(cf, st, n, clbits, draw)
            continue
        if op.Gate is None:
            if op.Clbits and op.Qubits:
                clbits[op.Clbits[0]] = orc.sv_measure(st, op.Qubits[0], draw())
            continue
        name = op.Gate.Name()
        if name in ("barrier", "delay"):  # the pseudo-gates' names (gate.go)
            continue
        if name == "reset":
            if orc.sv_measure(st, op.Qubits[0], draw()) == 1:
                _apply(st, n, [ir.Operation(G.X, [op.Qubits[0]])])
            continue
        if op.Condition is not None and clbits[op.Condition.clbit] != op.Condition.value:
            continue
        _apply(st, n, [ir.Operation(op.Gate, list(op.Qubits))])


def _exec_cf(cf, st, n, clbits, draw):
    if cf.Type == ir.ControlFlowWhile:
        for _ in range(ir.MaxControlFlowIterations):
            if clbits[cf.Condition.clbit] != cf.Condition.value:
                break
            _exec(cf.Bodies[0], st, n, clbits, draw)
    elif cf.Type == ir.ControlFlowFor:
        i = cf.ForRange.Start
        while i < cf.ForRange.End:
            _exec(cf.Bodies[0], st, n, clbits, draw)
            i += cf.ForRange.Step
    elif cf.Type == ir.ControlFlowIfElse:
        if clbits[cf.Condition.clbit] == cf.Condition.value:
            _exec(cf.Bodies[0], st, n, clbits, draw)
        elif len(cf.Bodies) > 1:
            _exec(cf.Bodies[1], st, n, clbits, draw)
    elif cf.Type == ir.ControlFlowSwitch:
        val = 0
        for i, idx in enumerate(cf.SwitchArg.Clbits):
            val |= clbits[idx] << i
        for i, case in enumerate(cf.SwitchArg.Cases):
            if val == case and i < len(cf.Bodies):
                _exec(cf.Bodies[i], st, n, clbits, draw)
                return
        if len(cf.Bodies) > len(cf.SwitchArg.Cases):
            _exec(cf.Bodies[-1], st, n, clbits, draw)


def run_dynamic(circuit, shots, uniforms):
    """Counts and the last shot's final state."""
    n = circuit.NumQubits()
    counts, st = {}, None
    for s in range(shots):
        st = orc.zero_state(n)
        clbits = [0] * circuit.NumClbits()
        k = [0]

        def draw():
            v = uniforms[s, k[0]]
            k[0] += 1
            return float(v)

        _exec(circuit.Ops(), st, n, clbits, draw)
        key = "".join("1" if v else "0" for v in reversed(clbits))
        counts[key] = counts.get(key, 0) + 1
    return counts, st


# ---- circuits ---------------------------------------------------------------

def teleport():
    b = ir.Builder("teleport", 3)
    b.RY(1.1, 0).RZ(0.4, 0)
    b.H(1).CNOT(1, 2).CNOT(0, 1).H(0)
    b.Measure(0, 0).Measure(1, 1)
    b.If(1, 1, G.X, 2).If(0, 1, G.Z, 2)
    b.RY(0.7, 2).Measure(2, 2)
    return b.Build()


def reset_and_reuse():
    b = ir.Builder("reset", 3)
    b.H(0).CNOT(0, 1).Reset(0).RX(0.9, 0).CNOT(0, 2).Measure(0, 0).Reset(1).H(1).Measure(1, 1).Measure(2, 2)
    return b.Build()


def repeat_until_success():
    b = ir.Builder("rus", 2)
    b.H(0).Measure(0, 0)
    b.While(0, 1, lambda s: s.Reset(0).RY(1.3, 0).CNOT(0, 1).Measure(0, 0))
    b.Measure(1, 1)
    return b.Build()


def loops_and_switch():
    b = ir.Builder("cf", 3)
    b.H(0).H(1)
    b.For(2, 0, 3, 1, lambda s: s.RY(0.5, 2).Measure(2, 2))
    b.Measure(0, 0).Measure(1, 1)
    b.Switch([0, 1], {0: lambda s: s.X(2), 3: lambda s: s.RZ(0.3, 2).H(2)}, lambda s: s.RX(1.0, 2))
    b.IfElseBlock(2, 1, lambda s: s.H(0), lambda s: s.S(0).H(0))
    b.Measure(2, 2).Measure(0, 0)
    return b.Build()


def random_mid_circuit(n, layers, seed):
    rng = np.random.default_rng(seed)
    b = ir.Builder("mid", n)
    c = 0
    for layer in range(layers):
        for q in range(n):
            b.U3(*rng.uniform(0, 2 * np.pi, 3), q)
        for q in range(layer % 2, n - 1, 2):
            b.CNOT(q, q + 1)
        q = int(rng.integers(n))
        b.Measure(q, c % n)
        b.If(c % n, 1, G.X, (q + 1) % n)
        c += 1
    for q in range(n):
        b.Measure(q, q)
    return b.Build()


CIRCUITS = {"teleport": teleport, "reset": reset_and_reuse, "rus": repeat_until_success,
            "cf": loops_and_switch, "mid": lambda: random_mid_circuit(5, 6, 3)}


# ---- density matrix (sim/densitymatrix/dynamic.go:13-255) -------------------

def _dm_apply(rho, n, op_list, nm):
    stream = encode.density_ops(ir.Circuit("", n, 0, op_list), nm)
    if len(stream):
        orc.dm_apply(rho, stream)


def _dm_exec(ops, rho, n, nm, clbits, draw):
    from goqu_b200 import dynamic
    for op in ops:
        cf = op.ControlFlow
        if cf is not None:
            if cf.Type == ir.ControlFlowWhile:
                for _ in range(ir.MaxControlFlowIterations):
                    if clbits[cf.Condition.clbit] != cf.Condition.value:
                        break
                    _dm_exec(cf.Bodies[0], rho, n, nm, clbits, draw)
            elif cf.Type == ir.ControlFlowFor:
                i = cf.ForRange.Start
                while i < cf.ForRange.End:
                    _dm_exec(cf.Bodies[0], rho, n, nm, clbits, draw)
                    i += cf.ForRange.Step
            elif cf.Type == ir.ControlFlowIfElse:
                if clbits[cf.Condition.clbit] == cf.Condition.value:
                    _dm_exec(cf.Bodies[0], rho, n, nm, clbits, draw)
                elif len(cf.Bodies) > 1:
                    _dm_exec(cf.Bodies[1], rho, n, nm, clbits, draw)
            else:
                raise NotImplementedError("switch is covered by the statevector cases")
            continue
        if op.Gate is None:
            if op.Clbits and op.Qubits:
                clbits[op.Clbits[0]] = orc.dm_measure(rho, n, op.Qubits[0], draw())
            continue
        name = op.Gate.Name()
        if name == "barrier":
            continue
        if name == "delay":
            _dm_apply(rho, n, [op], nm)
            continue
        if name == "reset":
            if orc.dm_measure(rho, n, op.Qubits[0], draw()) == 1:
                _dm_apply(rho, n, [ir.Operation(G.X, [op.Qubits[0]])], None)  # no gate noise
            _dm_apply(rho, n, [ir.Operation(dynamic.ResetNoise(), [op.Qubits[0]])], nm)
            continue
        if op.Condition is not None and clbits[op.Condition.clbit] != op.Condition.value:
            continue
        _dm_apply(rho, n, [ir.Operation(op.Gate, list(op.Qubits))], nm)


def run_dynamic_dm(circuit, nm, shots, uniforms):
    n = circuit.NumQubits()
    counts, rho = {}, None
    for s in range(shots):
        rho = orc.dm_zero(n)
        clbits = [0] * circuit.NumClbits()
        k = [0]

        def draw():
            v = uniforms[s, k[0]]
            k[0] += 1
            return float(v)

        _dm_exec(circuit.Ops(), rho, n, nm, clbits, draw)
        key = "".join("1" if v else "0" for v in reversed(clbits))
        counts[key] = counts.get(key, 0) + 1
    return counts, rho


def noisy_model():
    from goqu_b200 import noise as N
    nm = N.New()
    nm.AddDefaultError(1, N.Depolarizing1Q(0.02))
    nm.AddDefaultError(2, N.Depolarizing2Q(0.03))
    nm.AddGateError("delay", N.AmplitudeDamping(0.1))
    nm.AddGateError("reset", N.BitFlip(0.05))
    return nm


def noisy_dynamic():
    b = ir.Builder("noisy", 3)
    b.H(0).CNOT(0, 1).Delay(2, 100).Measure(0, 0)
    b.If(0, 1, G.X, 2).Reset(1).RY(0.8, 1).CNOT(1, 2)
    b.IfElseBlock(0, 0, lambda s: s.H(2), lambda s: s.RX(0.4, 2))
    b.Measure(1, 1).Measure(2, 2)
    return b.Build()
