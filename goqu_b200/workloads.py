"""Seeded synthetic workloads (the benchmark and parity-test circuits).

No public benchmark suite exists for this path; these generators build the
circuits with numpy's seeded PCG64 generator:

* random_layers / random_layers_qft: layers of U3(theta, phi, lambda) on every
  qubit (angles uniform in [0, 2 pi)) followed by a CNOT brickwork, pairs
  (2i, 2i+1) in even layers and (2i+1, 2i+2) in odd layers, optionally
  followed by the QFT of goqu's algorithm/qpe/qpe.go:170-182.
* hardware_efficient_ansatz: layers of symbolic RY, RZ on every qubit then a
  CZ ring, with a transverse-field Ising observable.
* qaoa_maxcut: goqu's QAOA circuit (algorithm/qaoa/qaoa.go:68-93) and
  MaxCutHamiltonian (maxcut.go:13-35) on seeded random 3-regular graphs.
* noisy_brickwork: the density-matrix circuit with delays on idle qubits and
  the depolarizing / amplitude-damping noise model.
"""
from __future__ import annotations

import math

import numpy as np

from . import circuit as ir
from . import gate as G
from . import noise as N
from . import param as prm
from . import pauli as P


def _brickwork_pairs(n, layer):
    start = 0 if layer % 2 == 0 else 1
    return [(q, q + 1) for q in range(start, n - 1, 2)]


def add_random_layers(b, n, layers, rng):
    for layer in range(layers):
        for q in range(n):
            th, ph, la = rng.uniform(0.0, 2.0 * math.pi, 3)
            b.U3(th, ph, la, q)
        for c, t in _brickwork_pairs(n, layer):
            b.CNOT(c, t)
    return b


def apply_qft(b, n):
    """applyQFT (algorithm/qpe/qpe.go:170-182)."""
    for i in range(n):
        b.H(i)
        for j in range(i + 1, n):
            b.Apply(G.CP(math.pi / float(1 << (j - i))), i, j)
    for i in range(n // 2):
        b.SWAP(i, n - 1 - i)
    return b


def random_layers(n, layers, seed):
    rng = np.random.default_rng(seed)
    return add_random_layers(ir.Builder(f"layers{n}x{layers}", n), n, layers, rng).Build()


def random_layers_qft(n, layers, seed):
    rng = np.random.default_rng(seed)
    b = add_random_layers(ir.Builder(f"layers{n}x{layers}+qft", n), n, layers, rng)
    return apply_qft(b, n).Build()


def count_gates(c):
    return sum(1 for op in c.Ops() if op.Gate is not None and op.Gate.Name() not in ("barrier", "delay"))


def hardware_efficient_ansatz(n, layers):
    """RY(theta), RZ(theta) on every qubit, then CZ(i, i+1 mod n); parameters
    theta[0..2*n*layers) in first-appearance order."""
    theta = prm.NewVector("θ", 2 * n * layers)
    b = ir.Builder(f"hea{n}x{layers}", n)
    k = 0
    for _ in range(layers):
        for q in range(n):
            b.SymRY(theta.At(k), q)
            b.SymRZ(theta.At(k + 1), q)
            k += 2
        for q in range(n):
            b.CZ(q, (q + 1) % n)
    return b.Build(), theta.Names()


def ising_hamiltonian(n, h=0.5):
    """sum_{i<n-1} Z_i Z_{i+1} + h sum_i X_i (open chain)."""
    terms = [P.NewPauliString(1.0, {i: P.Z, i + 1: P.Z}, n) for i in range(n - 1)]
    terms += [P.NewPauliString(h, {i: P.X}, n) for i in range(n)]
    return P.NewPauliSum(terms)


def random_3_regular(n, rng, max_tries=1000):
    """Pairing model with rejection (no self loops, no multi-edges)."""
    if n % 2:
        raise ValueError("a 3-regular graph needs an even vertex count")
    for _ in range(max_tries):
        stubs = np.repeat(np.arange(n), 3)
        rng.shuffle(stubs)
        pairs = stubs.reshape(-1, 2)
        edges = set()
        ok = True
        for a, b in pairs:
            a, b = int(a), int(b)
            if a == b or (min(a, b), max(a, b)) in edges:
                ok = False
                break
            edges.add((min(a, b), max(a, b)))
        if ok:
            return sorted(edges)
    raise RuntimeError("no 3-regular graph found")


def maxcut_hamiltonian(edges, n):
    """MaxCutHamiltonian (algorithm/qaoa/maxcut.go:13-35)."""
    if not edges:
        raise ValueError("qaoa: no edges provided")
    if n < 2:
        raise ValueError("qaoa: numQubits must be >= 2")
    terms = []
    for a, b in edges:
        terms.append(P.NewPauliString(-0.5, None, n))
        terms.append(P.NewPauliString(0.5, {a: P.Z, b: P.Z}, n))
    return P.NewPauliSum(terms)


def qaoa_circuit(h, p):
    """The symbolic QAOA circuit of qaoa.Run (algorithm/qaoa/qaoa.go:68-93):
    H on every qubit, then per layer RZ/RZZ(2*coeff*gamma_k) for each Z term
    (qaoa.go:164-196) and RX(2*beta_k) on every qubit."""
    nq = h.NumQubits()
    gammas = prm.NewVector("γ", p)
    betas = prm.NewVector("β", p)
    b = ir.Builder("QAOA", nq)
    for q in range(nq):
        b.H(q)
    for k in range(p):
        for term in h.Terms():
            coeff = term.Coeff().real
            if coeff == 0:
                continue
            zq, all_z = [], True
            for q in range(nq):
                o = term.Op(q)
                if o == P.Z:
                    zq.append(q)
                elif o != P.I:
                    all_z = False
                    break
            if not all_z or not zq:
                continue
            angle = prm.Mul(prm.Literal(2 * coeff), gammas.At(k))
            if len(zq) == 1:
                b.SymRZ(angle, zq[0])
            elif len(zq) == 2:
                b.SymRZZ(angle, zq[0], zq[1])
        for q in range(nq):
            b.SymRX(prm.Mul(prm.Literal(2), betas.At(k)), q)
    c = b.Build()
    return c, ir.FreeParameters(c)


def qaoa_batch(count, seed, n_values=(10, 12, 14, 16, 18, 20), p_range=(1, 4)):
    """Seeded batch of QAOA MaxCut instances: (circuit, names, hamiltonian, x)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice(n_values))
        p = int(rng.integers(p_range[0], p_range[1] + 1))
        edges = random_3_regular(n, rng)
        h = maxcut_hamiltonian(edges, n)
        c, names = qaoa_circuit(h, p)
        x = rng.uniform(0.0, math.pi, len(names))
        out.append((c, names, h, x))
    return out


def noisy_brickwork(n, layers, seed, p1=1e-3, p2=1e-3, gamma=1e-3):
    """U3 on every qubit, CNOT brickwork, a Delay on each idle qubit, and a
    noise model with Depolarizing1Q/2Q defaults and amplitude damping on delay."""
    rng = np.random.default_rng(seed)
    b = ir.Builder(f"noisy{n}x{layers}", n)
    for layer in range(layers):
        for q in range(n):
            th, ph, la = rng.uniform(0.0, 2.0 * math.pi, 3)
            b.U3(th, ph, la, q)
        pairs = _brickwork_pairs(n, layer)
        busy = set()
        for c, t in pairs:
            b.CNOT(c, t)
            busy.update((c, t))
        for q in range(n):
            if q not in busy:
                b.Delay(q, 50.0, "ns")
    nm = N.New()
    nm.AddDefaultError(1, N.Depolarizing1Q(p1))
    nm.AddDefaultError(2, N.Depolarizing2Q(p2))
    nm.AddGateError("delay", N.AmplitudeDamping(gamma))
    return b.Build(), nm
