"""Adjoint gradients on the GPU against goqu's parameter-shift and finite
differences evaluated by the oracle (gradient.go:49-86). Bar: <= 1e-10 at
small sizes and <= 1e-8 on the 20-qubit, 400-parameter ansatz (complex128);
complex64 adjoint gradients are reported against the oracle at 5e-4."""
import math

import numpy as np
import pytest

from goqu_b200 import _abi, circuit as ir, encode, gradient, param as prm, pauli as P, workloads
from oracle import binding as orc

pytestmark = pytest.mark.gpu


def oracle_energy(c, names, x, h, threads=0):
    bound = ir.Bind(c, {nm: float(x[i]) for i, nm in enumerate(names)})
    st = orc.sv_evolve(encode.statevector_ops(bound), threads=threads)
    return orc.expect_pauli_sum(st, P.to_terms(h), threads=threads).real


def oracle_shift(c, names, x, h, idx=None, threads=0):
    idx = range(len(names)) if idx is None else idx
    out = []
    for i in idx:
        xp, xm = x.copy(), x.copy()
        xp[i] += math.pi / 2
        xm[i] -= math.pi / 2
        out.append((oracle_energy(c, names, xp, h, threads) - oracle_energy(c, names, xm, h, threads)) / 2)
    return np.array(out)


@pytest.mark.parametrize("n,layers", [(2, 1), (5, 2), (8, 3), (12, 2)])
def test_adjoint_matches_parameter_shift(n, layers):
    c, names = workloads.hardware_efficient_ansatz(n, layers)
    h = workloads.ising_hamiltonian(n)
    x = np.random.default_rng(n).uniform(0, 2 * np.pi, len(names))
    ev = gradient.AdjointEvaluator(c, h, names)
    e, g = ev(x)
    assert abs(e - oracle_energy(c, names, x, h)) < 1e-12
    np.testing.assert_allclose(g, oracle_shift(c, names, x, h), atol=1e-10, rtol=0)


def test_adjoint_general_gates_and_expressions():
    th = prm.NewVector("t", 5)
    b = ir.Builder("g", 6)
    b.H(0).H(1).H(2).H(5)
    b.SymU3(th.At(0), prm.Mul(2.0, th.At(1)), th.At(2), 3)
    b.SymCP(th.At(3), 0, 4).SymRXX(prm.Add(th.At(4), 0.3), 1, 2).SymRZZ(th.At(0), 2, 3)
    b.SymRX(prm.Neg(th.At(1)), 4).CNOT(3, 0).SymRY(th.At(2), 1).CCX(0, 1, 5).SymRYY(th.At(3), 5, 2)
    c = b.Build()
    names = ir.FreeParameters(c)
    h = P.NewPauliSum([P.NewPauliString(0.7, {0: P.Z, 3: P.X}, 6), P.NewPauliString(-0.4, {1: P.Y, 2: P.Y}, 6),
                       P.NewPauliString(0.25, {4: P.X, 5: P.Z}, 6)])
    x = np.random.default_rng(3).uniform(0, 2 * np.pi, len(names))
    e, g = gradient.AdjointEvaluator(c, h, names)(x)
    fd = []
    for i in range(len(names)):
        xp, xm = x.copy(), x.copy()
        xp[i] += 1e-5
        xm[i] -= 1e-5
        fd.append((oracle_energy(c, names, xp, h) - oracle_energy(c, names, xm, h)) / 2e-5)
    assert abs(e - oracle_energy(c, names, x, h)) < 1e-12
    np.testing.assert_allclose(g, fd, atol=1e-7, rtol=0)


def test_adjoint_20q_400_params():
    # the 20-qubit hardware-efficient ansatz: 10 layers of RY,RZ + CZ ring
    c, names = workloads.hardware_efficient_ansatz(20, 10)
    assert len(names) == 400
    h = workloads.ising_hamiltonian(20)
    x = np.random.default_rng(20).uniform(0, 2 * np.pi, 400)
    e, g = gradient.AdjointEvaluator(c, h, names)(x)
    # the engine's own parameter shift on 24 parameters and the oracle's on 4
    f = gradient.CostFunc(c, h, names)
    sel = np.random.default_rng(1).choice(400, 24, replace=False)
    gps = []
    for i in sel:
        xp, xm = x.copy(), x.copy()
        xp[i] += math.pi / 2
        xm[i] -= math.pi / 2
        gps.append((f(xp) - f(xm)) / 2)
    assert np.max(np.abs(g[sel] - np.array(gps))) < 1e-8
    sel4 = sel[:4]
    assert np.max(np.abs(g[sel4] - oracle_shift(c, names, x, h, sel4, threads=8))) < 1e-8
    assert abs(e - oracle_energy(c, names, x, h, threads=8)) < 1e-10


def test_adjoint_phase_gates_on_populated_qubits():
    # P, U1 and CP whose phase lands on amplitudes that are populated: their
    # derivative is i e^(i phi) on the last diagonal entry only
    a, b = prm.New("a"), prm.New("b")
    c = (ir.Builder("ph", 3).H(0).H(1).H(2).SymPhase(a, 0).SymCP(a, 0, 1).Apply(prm.SymU1(prm.Mul(2.0, b)), 2)
         .CNOT(1, 2).SymCP(b, 2, 0).H(0).H(2).Build())
    h = P.NewPauliSum([P.NewPauliString(1.0, {0: P.X}, 3), P.NewPauliString(0.5, {0: P.Z, 1: P.Y}, 3),
                       P.NewPauliString(-0.3, {2: P.X, 1: P.X}, 3)])
    names = ir.FreeParameters(c)
    x = np.array([0.7, -1.1])
    e, g = gradient.AdjointEvaluator(c, h, names)(x)
    fd = []
    for i in range(len(names)):
        xp, xm = x.copy(), x.copy()
        xp[i] += 1e-5
        xm[i] -= 1e-5
        fd.append((oracle_energy(c, names, xp, h) - oracle_energy(c, names, xm, h)) / 2e-5)
    np.testing.assert_allclose(g, fd, atol=1e-8, rtol=0)


def test_adjoint_checkpoints_agree():
    c, names = workloads.hardware_efficient_ansatz(10, 4)
    h = workloads.ising_hamiltonian(10)
    x = np.random.default_rng(4).uniform(0, 2 * np.pi, len(names))
    ev = gradient.AdjointEvaluator(c, h, names)
    e1, g1 = ev(x)
    ev.sim.set_option(_abi.GQ_OPT_ADJOINT_SEGMENTS, 5)
    e2, g2 = ev(x)
    assert abs(e1 - e2) < 1e-13
    assert np.max(np.abs(g1 - g2)) < 1e-12


def test_adjoint_complex64_error():
    c, names = workloads.hardware_efficient_ansatz(10, 3)
    h = workloads.ising_hamiltonian(10)
    x = np.random.default_rng(5).uniform(0, 2 * np.pi, len(names))
    e, g = gradient.AdjointEvaluator(c, h, names, _abi.GQ_C64)(x)
    assert np.max(np.abs(g - oracle_shift(c, names, x, h))) < 5e-4


def test_adjoint_rejects_reset():
    c = ir.Builder("r", 2).SymRY(prm.New("a"), 0).Reset(1).Build()
    with pytest.raises(_abi.GQError, match="unitary"):
        gradient.AdjointEvaluator(c, workloads.ising_hamiltonian(2), ["a"])(np.array([0.3]))
