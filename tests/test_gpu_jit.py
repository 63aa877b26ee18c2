"""Parity of the specialised (run-time compiled) tile-pass kernels (GPU).

With GQ_OPT_JIT = 2 every pass waits for its compiled kernel, so the results
below come from the specialised kernels alone (checked through the stats);
the bars are those of the interpreted kernel: complex128 within 1e-12 of the
FP64 oracle, complex64 within 2e-5.
"""
import numpy as np
import pytest

from goqu_b200 import _abi, densitymatrix, encode, statevector, workloads
from oracle import binding as orc

from kat_util import chain_circuit, random_circuit

pytestmark = pytest.mark.gpu


def jit_sim(n, precision=_abi.GQ_C128, mode=2):
    sim = statevector.New(n, precision)
    sim.set_option(_abi.GQ_OPT_TIMING, 1)
    sim.set_option(_abi.GQ_OPT_JIT, mode)
    sim.set_option(_abi.GQ_OPT_JIT_MIN_QUBITS, 0)
    return sim


@pytest.mark.parametrize("n,seed", [(12, 1), (14, 2), (17, 3)])
def test_random_circuits_match_oracle(n, seed):
    c = random_circuit(n, 120, seed, allow_reset=True)
    want = orc.sv_evolve(encode.statevector_ops(c))
    sim = jit_sim(n)
    sim.Evolve(c)
    st = sim.stats()
    assert st["jit_passes"] == st["passes"] >= 1
    np.testing.assert_allclose(sim.StateVector(), want, atol=1e-12, rtol=0)


@pytest.mark.parametrize("n,seed", [(14, 21), (16, 22)])
def test_uniform_predicates_and_chains_match_oracle(n, seed):
    # X-type gates and phases controlled from CTA-index qubits: predicate
    # tables, fused one-qubit chains, run-time phase accumulators
    c = chain_circuit(n, seed, low=6)
    want = orc.sv_evolve(encode.statevector_ops(c))
    for prec, tol in ((_abi.GQ_C128, 1e-12), (_abi.GQ_C64, 2e-5)):
        sim = jit_sim(n, prec)
        sim.Evolve(c)
        st = sim.stats()
        assert st["jit_passes"] == st["passes"] >= 1
        assert np.max(np.abs(sim.StateVector() - want)) < tol


def test_complex64_matches_oracle():
    c = random_circuit(13, 100, 4, allow_reset=True)
    want = orc.sv_evolve(encode.statevector_ops(c))
    sim = jit_sim(13, _abi.GQ_C64)
    sim.Evolve(c)
    st = sim.stats()
    assert st["jit_passes"] == st["passes"]
    assert np.max(np.abs(sim.StateVector() - want)) < 2e-5


def test_layered_benchmark_20q_matches_interpreter_and_oracle():
    c = workloads.random_layers_qft(20, layers=6, seed=2028)
    want = orc.sv_evolve(encode.statevector_ops(c))
    sim = jit_sim(20)
    sim.Evolve(c)
    assert sim.stats()["jit_passes"] == sim.stats()["passes"]
    got = sim.StateVector()
    ref = statevector.New(20)
    ref.set_option(_abi.GQ_OPT_JIT, 0)
    ref.Evolve(c)
    assert ref.stats()["jit_passes"] == 0
    np.testing.assert_allclose(got, want, atol=1e-12, rtol=0)
    np.testing.assert_allclose(got, ref.StateVector(), atol=1e-13, rtol=0)


def test_async_mode_switches_to_compiled_kernels():
    # mode 1: the first evolve may run interpreted while compiling; a later
    # one of the same structure (other angles) runs compiled; both exact
    n = 12
    for k, seed in enumerate([11, 11, 11]):
        c = random_circuit(n, 60, seed)
        sim = jit_sim(n, mode=1)
        if k == 2:
            sim.set_option(_abi.GQ_OPT_JIT, 2)
        sim.Evolve(c)
        np.testing.assert_allclose(sim.StateVector(), orc.sv_evolve(encode.statevector_ops(c)), atol=1e-12, rtol=0)
        if k == 2:
            assert sim.stats()["jit_passes"] == sim.stats()["passes"]


def test_density_matrix_matches_oracle():
    c, nm = workloads.noisy_brickwork(6, layers=4, seed=3)
    want = orc.dm_evolve(encode.density_ops(c, nm))
    dm = densitymatrix.New(6).WithNoise(nm)
    dm.set_option(_abi.GQ_OPT_JIT, 2)
    dm.set_option(_abi.GQ_OPT_JIT_MIN_QUBITS, 0)
    dm.set_option(_abi.GQ_OPT_TIMING, 1)
    dm.Evolve(c)
    st = dm.stats()
    assert st["jit_passes"] == st["passes"] >= 1
    np.testing.assert_allclose(dm.DensityMatrix().reshape(-1), want, atol=1e-12, rtol=0)


@pytest.mark.parametrize("n,layers", [(9, 3), (12, 2), (20, 2)])
def test_specialised_reverse_passes_match_interpreted(n, layers):
    # the adjoint's reverse sweep on specialised dual kernels (GQ_OPT_JIT = 2,
    # every size) against the interpreted one (GQ_OPT_JIT = 0) and parameter shift
    from goqu_b200 import gradient
    c, names = workloads.hardware_efficient_ansatz(n, layers)
    h = workloads.ising_hamiltonian(n)
    x = np.random.default_rng(n).uniform(0, 2 * np.pi, len(names))
    ev_j = gradient.AdjointEvaluator(c, h, names)
    ev_j.sim.set_option(_abi.GQ_OPT_JIT, 2)
    ev_j.sim.set_option(_abi.GQ_OPT_JIT_MIN_QUBITS, 0)
    ev_i = gradient.AdjointEvaluator(c, h, names)
    ev_i.sim.set_option(_abi.GQ_OPT_JIT, 0)
    e_j, g_j = ev_j(x)
    st = ev_j.sim.stats()
    assert st["jit_passes"] == st["passes"]  # forward and reverse passes all specialised
    e_i, g_i = ev_i(x)
    assert ev_i.sim.stats()["jit_passes"] == 0
    assert abs(e_j - e_i) < 1e-12
    np.testing.assert_allclose(g_j, g_i, atol=1e-11, rtol=0)
    if n <= 12:
        ps = gradient.ParameterShift(gradient.CostFunc(c, h, names))(x)
        np.testing.assert_allclose(g_j, ps, atol=1e-9, rtol=0)


def test_specialised_reverse_passes_general_gates():
    # U3 / CP / RXX / RYY / RZZ / CCX and expressions: dense, diagonal, phase
    # and controlled gradient generators on the dual kernels, complex128 and complex64
    from goqu_b200 import circuit as ir, gradient, param as prm, pauli as P
    th = prm.NewVector("t", 6)
    b = ir.Builder("g", 10)
    for q in range(10):
        b.H(q)
    b.SymU3(th.At(0), prm.Mul(2.0, th.At(1)), th.At(2), 3).SymCP(th.At(3), 0, 9).SymRXX(th.At(4), 1, 2)
    b.SymRZZ(th.At(0), 2, 8).SymRX(prm.Neg(th.At(1)), 7).CNOT(3, 0).SymRY(th.At(5), 5).CCX(1, 2, 6)
    b.SymPhase(th.At(2), 4).SymRZ(th.At(4), 9).SymRYY(th.At(3), 4, 5)
    c = b.Build()
    names = ir.FreeParameters(c)
    h = P.NewPauliSum([P.NewPauliString(0.7, {0: P.Z, 3: P.X}, 10), P.NewPauliString(-0.4, {1: P.Y, 2: P.Y}, 10),
                       P.NewPauliString(0.25, {9: P.X, 6: P.Z}, 10)])
    x = np.random.default_rng(3).uniform(0, 2 * np.pi, len(names))
    for prec, tol in ((_abi.GQ_C128, 1e-11), (_abi.GQ_C64, 1e-4)):
        ev_j = gradient.AdjointEvaluator(c, h, names, prec)
        ev_j.sim.set_option(_abi.GQ_OPT_JIT, 2)
        ev_j.sim.set_option(_abi.GQ_OPT_JIT_MIN_QUBITS, 0)
        ev_i = gradient.AdjointEvaluator(c, h, names, prec)
        ev_i.sim.set_option(_abi.GQ_OPT_JIT, 0)
        e_j, g_j = ev_j(x)
        e_i, g_i = ev_i(x)
        assert ev_j.sim.stats()["jit_passes"] == ev_j.sim.stats()["passes"]
        assert abs(e_j - e_i) < tol
        np.testing.assert_allclose(g_j, g_i, atol=tol, rtol=0)


@pytest.mark.parametrize("n,seed,variant", [(16, 51, 0), (22, 52, 2)])
def test_zero_tile_skip_matches_full_launch(n, seed, variant):
    # Evolve from the reset state launches only the tiles inside the support
    # (GQ_OPT_ZERO_TILES, default on): the state must match the run that
    # launches every tile (the short passes' larger budgets may change the
    # schedule and its rounding, not the result), and the tile bytes shrink
    c = workloads.random_layers_qft(n, 3, seed) if n > 16 else random_circuit(n, 120, seed, allow_reset=True)
    states, tb = [], []
    for skip in (0, 1):
        sim = jit_sim(n)
        sim.set_option(_abi.GQ_OPT_KERNEL_VARIANT, variant)
        sim.set_option(_abi.GQ_OPT_ZERO_TILES, skip)
        sim.Evolve(c)
        st = sim.stats()
        assert st["jit_passes"] == st["passes"] >= 1
        if not skip:
            assert st["tile_bytes"] == st["passes"] * 2 * st["state_bytes"]
        states.append(sim.StateVector())
        tb.append(st["tile_bytes"])
        sim.Close()
    np.testing.assert_allclose(states[1], states[0], atol=1e-13, rtol=0)
    assert tb[1] < tb[0]
    if n <= 16:
        np.testing.assert_allclose(states[1], orc.sv_evolve(encode.statevector_ops(c)), atol=1e-12, rtol=0)


def test_zero_tile_skip_density_matrix_and_apply():
    c, nm = workloads.noisy_brickwork(10, layers=3, seed=53)
    rhos = []
    for skip in (0, 1):
        dm = densitymatrix.New(10).WithNoise(nm)
        dm.set_option(_abi.GQ_OPT_JIT, 2)
        dm.set_option(_abi.GQ_OPT_JIT_MIN_QUBITS, 0)
        dm.set_option(_abi.GQ_OPT_ZERO_TILES, skip)
        dm.Evolve(c)
        st = dm.stats()
        assert (st["tile_bytes"] < st["passes"] * 2 * st["state_bytes"]) == bool(skip)
        rhos.append(dm.DensityMatrix())
        dm.Close()
    np.testing.assert_allclose(rhos[1], rhos[0], atol=1e-13, rtol=0)
    # Apply composes on the current state: nothing may be skipped there
    g = random_circuit(16, 60, 54)
    sim = jit_sim(16)
    sim.Evolve(g)
    sim.Apply(g)
    st = sim.stats()
    assert st["tile_bytes"] == st["passes"] * 2 * st["state_bytes"]
    sim2 = jit_sim(16)
    sim2.set_option(_abi.GQ_OPT_ZERO_TILES, 0)
    sim2.Evolve(g)
    sim2.Apply(g)
    np.testing.assert_allclose(sim.StateVector(), sim2.StateVector(), atol=1e-13, rtol=0)


@pytest.mark.parametrize("variant", [0, 2])
def test_persistent_kernels_match_one_tile_per_cta(variant):
    # GQ_OPT_JIT_PERSISTENT: persistent CTAs refill their tile buffer with the
    # next tile during the last phase; the state must be bit-identical to one
    # CTA per tile, and match the oracle
    n = 20
    c = workloads.random_layers_qft(n, 4, 61)
    want = orc.sv_evolve(encode.statevector_ops(c))
    states = []
    for persistent in (0, 1):
        sim = jit_sim(n)
        sim.set_option(_abi.GQ_OPT_KERNEL_VARIANT, variant)
        sim.set_option(_abi.GQ_OPT_JIT_PERSISTENT, persistent)
        sim.Evolve(c)
        st = sim.stats()
        assert st["jit_passes"] == st["passes"] >= 1
        states.append(sim.StateVector())
        sim.Close()
    assert np.array_equal(states[0], states[1])
    np.testing.assert_allclose(states[1], want, atol=1e-12, rtol=0)


def test_persistent_kernels_complex64_and_random_gates():
    c = random_circuit(18, 150, 62, allow_reset=True)
    want = orc.sv_evolve(encode.statevector_ops(c))
    for prec, tol in ((_abi.GQ_C128, 1e-12), (_abi.GQ_C64, 5e-5)):
        sim = jit_sim(18, prec)
        sim.set_option(_abi.GQ_OPT_JIT_PERSISTENT, 1)
        sim.Evolve(c)
        st = sim.stats()
        assert st["jit_passes"] == st["passes"] >= 1
        assert np.max(np.abs(sim.StateVector() - want)) < tol
        sim.Close()
