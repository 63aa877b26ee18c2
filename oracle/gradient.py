"""goqu's parameter-shift and finite-difference gradients evaluated on the
oracle (algorithm/gradient/gradient.go:25-86).

TEST INFRASTRUCTURE: the checker for the engine's adjoint gradients, used by
tests/ and bench.py's parity extras only.

CostFunc (gradient.go:25-47) binds the circuit, evolves a fresh statevector
and returns Re sum_t c_t <psi|P_t|psi>. ParameterShift (gradient.go:49-66)
takes (E(x + pi/2 e_i) - E(x - pi/2 e_i)) / 2 per parameter. Here the two
shifted evolutions of parameter i start from the state just before the first
op that depends on it, computed once in a forward sweep: the ops ahead of that
point do not depend on parameter i, so the shifted circuits' prefixes are the
same operations on the same numbers and the result is bit-identical to
evolving each shifted circuit from |0...0>.
"""
from __future__ import annotations

import math

import numpy as np

from goqu_b200 import circuit as ir, encode, pauli as P

from . import binding as orc


def _bind(c, names, x):
    return ir.Bind(c, {nm: float(x[i]) for i, nm in enumerate(names)})


def _sub(c, ops):
    return ir.Circuit(c.Name(), c.NumQubits(), c.NumClbits(), list(ops))


def energy(c, names, x, h, threads=0):
    """CostFunc (gradient.go:25-47) on the oracle."""
    st = orc.sv_evolve(encode.statevector_ops(_bind(c, names, x)), threads=threads)
    return orc.expect_pauli_sum(st, P.to_terms(h), threads=threads).real


def first_use(c, names):
    """Index of the first op of `c` whose gate depends on each parameter."""
    where = {}
    for k, op in enumerate(c.Ops()):
        g = op.Gate
        if g is not None and hasattr(g, "FreeParameters"):
            for nm in g.FreeParameters():
                where.setdefault(nm, k)
    return [where.get(nm, len(c.Ops())) for nm in names]


def parameter_shift(c, names, x, h, idx=None, threads=0, shift=math.pi / 2, denom=2.0):
    """ParameterShift (gradient.go:49-66) for the parameters in `idx` (all by
    default), with shared forward prefixes. shift = h, denom = 2h gives the
    central finite difference of FiniteDifference (gradient.go:68-86)."""
    x = np.asarray(x, dtype=float)
    idx = list(range(len(names))) if idx is None else [int(i) for i in idx]
    terms = P.to_terms(h)
    pos = first_use(c, names)
    base_ops = _bind(c, names, x).Ops()
    state = orc.zero_state(c.NumQubits())
    at = 0
    out = {}
    for i in sorted(idx, key=lambda i: pos[i]):
        k = pos[i]
        if k > at:
            orc.sv_apply(state, encode.statevector_ops(_sub(c, base_ops[at:k])), threads)
            at = k
        e = []
        for sgn in (1.0, -1.0):
            xs = x.copy()
            xs[i] += sgn * shift
            tail = _bind(c, names, xs).Ops()[k:]
            st = orc.sv_apply(state.copy(), encode.statevector_ops(_sub(c, tail)), threads)
            e.append(orc.expect_pauli_sum(st, terms, threads=threads).real)
        out[i] = (e[0] - e[1]) / denom
    return np.array([out[i] for i in idx])


def stratified_hea_params(n, layers, per_layer_qubits=2, seed=1):
    """A parameter sample of the hardware-efficient ansatz (RY, RZ on every
    qubit per layer): RY and RZ of `per_layer_qubits` random qubits in every
    layer. Parameter 2 * (n * layer + q) is RY on qubit q, the next one RZ."""
    rng = np.random.default_rng(seed)
    out = []
    for layer in range(layers):
        for q in rng.choice(n, per_layer_qubits, replace=False):
            base = 2 * (n * layer + int(q))
            out += [base, base + 1]
    return sorted(out)
