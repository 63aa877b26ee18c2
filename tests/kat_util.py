"""Helpers shared by the tests: build goqu_b200 circuits from the KAT specs in
tests/golden/kats.json and seeded random circuits for cross-validation."""
import json
import math
import os

import numpy as np

from goqu_b200 import circuit as ir
from goqu_b200 import gate as G
from goqu_b200 import noise as N
from goqu_b200 import pauli as P

HERE = os.path.dirname(os.path.abspath(__file__))


def load_kats():
    with open(os.path.join(HERE, "golden", "kats.json")) as f:
        return json.load(f)["kats"]


def make_gate(name, params):
    if name == "MCX":
        return G.MCX(int(params[0]))
    if name == "MCZ":
        return G.MCZ(int(params[0]))
    if name == "MCP":
        return G.MCP(params[0], int(params[1]))
    if name == "CTRL_SWAP":
        return G.Controlled(G.SWAP, int(params[0]))
    if name == "Reset":
        return G.Reset
    obj = getattr(G, name)
    if params:
        return obj(*params)
    return obj


def build_circuit(spec):
    b = ir.Builder(spec["name"], spec["n"])
    for entry in spec["ops"]:
        name, qubits = entry[0], entry[1]
        params = entry[2] if len(entry) > 2 else []
        b.Apply(make_gate(name, params), *qubits)
    return b.Build()


def build_noise(spec):
    if "noise" not in spec and "readout" not in spec:
        return None
    nm = N.New()
    for kind, key, ch_name, args in spec.get("noise", []):
        ch = getattr(N, ch_name)(*args)
        if kind == "default":
            nm.AddDefaultError(key, ch)
        else:
            nm.AddGateError(key, ch)
    for q, p01, p10 in spec.get("readout", []):
        nm.AddReadoutError(q, N.NewReadoutError(p01, p10))
    return nm


def pauli_sum_from_spec(n, entries):
    table = {"X": P.X, "Y": P.Y, "Z": P.Z, "I": P.I}
    terms = [P.NewPauliString(complex(re, im), {int(q): table[p] for q, p in ops.items()}, n)
             for re, im, ops in entries]
    return P.NewPauliSum(terms)


def cplx(v):
    return np.array([complex(a, b) for a, b in v], dtype=np.complex128)


ONE_Q = ["H", "X", "Y", "Z", "S", "T", "SX", "Sdg", "Tdg"]
ONE_Q_PARAM = [("RX", 1), ("RY", 1), ("RZ", 1), ("Phase", 1), ("U3", 3), ("U2", 2), ("Rot", 3),
               ("GPI", 1), ("GPI2", 1), ("PhasedXZ", 3), ("GlobalPhase", 1)]
TWO_Q = ["CNOT", "CZ", "SWAP", "CY", "ISWAP", "ECR", "DCX", "CH", "CSX", "Sycamore"]
TWO_Q_PARAM = [("CP", 1), ("CRZ", 1), ("CRX", 1), ("CRY", 1), ("RXX", 1), ("RYY", 1), ("RZZ", 1),
               ("MS", 2), ("FSim", 2), ("PSwap", 1)]
THREE_Q = ["CCX", "CSWAP", "CCZ"]


def random_circuit(n, n_gates, seed, allow_3q=True, allow_ctrl=True, allow_reset=False):
    """Seeded random circuit over every gate family the simulator dispatches."""
    rng = np.random.default_rng(seed)
    b = ir.Builder(f"rand{n}_{seed}", n)
    for _ in range(n_gates):
        r = rng.random()
        if n >= 3 and allow_3q and r < 0.08:
            q = rng.choice(n, 3, replace=False).tolist()
            if rng.random() < 0.5:
                b.Apply(getattr(G, THREE_Q[rng.integers(len(THREE_Q))]), *q)
            else:
                b.Apply(G.Controlled(G.U3(*rng.uniform(0, 2 * math.pi, 3)), 2), *q)
        elif n >= 4 and allow_ctrl and r < 0.14:
            k = int(rng.integers(4, min(n, 6) + 1))
            q = rng.choice(n, k, replace=False).tolist()
            inner_kind = rng.integers(3)
            if inner_kind == 0:
                g = G.MCX(k - 1)
            elif inner_kind == 1:
                g = G.Controlled(G.U3(*rng.uniform(0, 2 * math.pi, 3)), k - 1)
            else:
                g = G.Controlled(G.RXX(rng.uniform(0, 2 * math.pi)), k - 2)
            b.Apply(g, *q)
        elif n >= 2 and r < 0.5:
            q = rng.choice(n, 2, replace=False).tolist()
            if rng.random() < 0.5:
                b.Apply(getattr(G, TWO_Q[rng.integers(len(TWO_Q))]), *q)
            else:
                name, k = TWO_Q_PARAM[rng.integers(len(TWO_Q_PARAM))]
                b.Apply(getattr(G, name)(*rng.uniform(0, 2 * math.pi, k)), *q)
        elif allow_reset and r < 0.53:
            b.Reset(int(rng.integers(n)))
        else:
            q = int(rng.integers(n))
            if rng.random() < 0.3:
                b.Apply(getattr(G, ONE_Q[rng.integers(len(ONE_Q))]), q)
            else:
                name, k = ONE_Q_PARAM[rng.integers(len(ONE_Q_PARAM))]
                b.Apply(getattr(G, name)(*rng.uniform(0, 2 * math.pi, k)), q)
    return b.Build()


def dense_unitary_state(circuit):
    """Independent numpy check: apply every gate as a full 2^n x 2^n matrix
    built with einsum (no shared code with the oracle or the engine)."""
    n = circuit.NumQubits()
    psi = np.zeros(1 << n, dtype=np.complex128)
    psi[0] = 1
    for op in circuit.Ops():
        g = op.Gate
        if g is None or g.Name() in ("barrier", "delay"):
            continue
        k = len(op.Qubits)
        m = g.Matrix().reshape([2] * (2 * k))
        t = psi.reshape([2] * n)  # axis a <-> qubit n-1-a
        axes = [n - 1 - q for q in op.Qubits]
        t = np.tensordot(m, t, axes=(list(range(k, 2 * k)), axes))
        t = np.moveaxis(t, list(range(k)), axes)
        psi = t.reshape(-1)
    return psi


def chain_circuit(n, seed, low=5):
    """One-qubit chains on low qubits through X-type gates controlled from high
    qubits (CTA-index bits at small tiles): CNOT, CY (phased X), H-CNOT-H
    (a diagonal product: not fused), two controls on one target, and
    controlled phases from high qubits (run-time accumulators)."""
    rng = np.random.default_rng(seed)
    b = ir.Builder("chains", n)
    for layer in range(10):
        for q in range(low):
            b.U3(*rng.uniform(0, 2 * np.pi, 3), q)
        for q in range(low):
            c = int(rng.integers(low, n))
            kind = (layer + q) % 5
            if kind == 0:
                b.CNOT(c, q)
            elif kind == 1:
                b.Ctrl(G.Y, [c], q)
            elif kind == 2:
                b.H(q)
                b.CNOT(c, q)
                b.H(q)
            elif kind == 3:
                b.CNOT(c, q)
                b.U3(*rng.uniform(0, 2 * np.pi, 3), q)
                b.CNOT(int(rng.integers(low, n)), q)
            else:
                for c2 in rng.choice(np.arange(low, n), 3, replace=False):
                    b.MCP(rng.uniform(0, 2 * np.pi), [int(c2)], q)
        for q in range(low, n):
            if layer % 3 == 0:
                b.U3(*rng.uniform(0, 2 * np.pi, 3), q)
    return b.Build()
