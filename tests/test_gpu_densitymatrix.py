"""Parity of the density-matrix engine with the oracle (GPU): entries, traces,
<Z_i>, purity and fidelity within 1e-12; readout-mixed sampling bit-exact."""
import numpy as np
import pytest

from goqu_b200 import circuit as ir, densitymatrix, encode, noise as N, pauli as P, statevector, workloads
from oracle import binding as orc

from kat_util import build_circuit, build_noise, cplx, load_kats, random_circuit

pytestmark = pytest.mark.gpu

TOL = 1e-12
EPS = 1e-10

DM_KATS = [k for k in load_kats() if k.get("dm")]


@pytest.mark.parametrize("kat", DM_KATS, ids=lambda k: k["name"])
def test_known_answers(kat):
    n = kat["n"]
    c = build_circuit(kat)
    nm = build_noise(kat)
    dm = densitymatrix.New(n).WithNoise(nm) if nm else densitymatrix.New(n)
    dm.Evolve(c)
    rho = dm.DensityMatrix()
    dim = 1 << n
    for idx, v in kat.get("rho_at", []):
        assert abs(rho[idx] - complex(*v)) < EPS
    if "trace" in kat:
        assert abs(dm.Trace().real - kat["trace"]) < EPS
    if "purity_below" in kat:
        assert 0 < dm.Purity() < kat["purity_below"] - EPS
    if "diag_nonneg" in kat:
        assert all(rho[i * dim + i].real > -EPS for i in range(dim))
    if "fidelity_with_sv" in kat:
        sv = statevector.New(n)
        sv.Evolve(c)
        assert abs(dm.Fidelity(sv.StateVector()) - kat["fidelity_with_sv"]) < EPS
    if "readout_probs" in kat:
        got = dm.ApplyReadoutError(dm.DiagonalProbs())
        np.testing.assert_allclose(got, kat["readout_probs"], atol=EPS, rtol=0)


def _noise_model(rng):
    nm = N.New()
    nm.AddDefaultError(1, N.Depolarizing1Q(0.02))
    nm.AddDefaultError(2, N.Depolarizing2Q(0.03))
    nm.AddGateError("H", N.PhaseDamping(0.1))
    nm.AddGateError("delay", N.AmplitudeDamping(0.05))
    nm.AddGateQubitError("CNOT", [0, 1], N.BitFlip(0.2))
    nm.AddReadoutError(0, N.NewReadoutError(0.03, 0.07))
    return nm


@pytest.mark.parametrize("n,seed", [(1, 1), (2, 2), (3, 3), (5, 4), (6, 5), (7, 6)])
def test_noisy_random_circuits_match_oracle(n, seed):
    rng = np.random.default_rng(seed)
    c = random_circuit(n, 40, seed, allow_3q=False, allow_ctrl=False, allow_reset=True)
    nm = _noise_model(rng)
    ops = encode.density_ops(c, nm)
    want = orc.dm_evolve(ops)
    dm = densitymatrix.New(n).WithNoise(nm)
    dm.Evolve(c)
    got = dm.DensityMatrix()
    assert np.max(np.abs(got - want)) < TOL
    assert abs(dm.Purity() - orc.dm_purity(want, n)) < TOL
    h = workloads.ising_hamiltonian(n) if n >= 2 else P.NewPauliSum([P.Parse("X")])
    assert abs(dm.ExpectPauliSum(h) - orc.dm_expect_pauli_sum(want, n, P.to_terms(h)).real) < TOL
    psi = orc.sv_evolve(encode.statevector_ops(ir.Circuit("p", n, 0, [op for op in c.Ops()
                                                                         if op.Gate.Name() != "reset"])))
    assert abs(dm.Fidelity(psi) - orc.dm_fidelity(want, n, psi)) < TOL


def test_controlled_gates_decomposed_path():
    # MCZ / controlled-U on >= 3 qubits (sim/densitymatrix/sim_test.go:413-482)
    from goqu_b200 import gate as G
    b = ir.Builder("mc", 4).H(0).H(1).H(2).Apply(G.MCZ(2), 0, 1, 2).Apply(G.Controlled(G.RY(0.7), 2), 1, 2, 3)
    c = b.Apply(G.MCP(0.4, 3), 0, 1, 2, 3).Build()
    want = orc.dm_evolve(encode.density_ops(c))
    dm = densitymatrix.New(4)
    dm.Evolve(c)
    assert np.max(np.abs(dm.DensityMatrix() - want)) < TOL
    with pytest.raises(ValueError, match="unsupported gate size: 3 qubits"):
        dm.Evolve(ir.Builder("ccx", 4).CCX(0, 1, 2).Build())


def test_noisy_brickwork_8q_matches_oracle():
    c, nm = workloads.noisy_brickwork(8, layers=6, seed=3)
    want = orc.dm_evolve(encode.density_ops(c, nm), threads=8)
    dm = densitymatrix.New(8).WithNoise(nm)
    dm.Evolve(c)
    got = dm.DensityMatrix()
    assert np.max(np.abs(got - want)) < TOL
    for q in range(8):
        ps = P.ZOn([q], 8)
        assert abs(dm.ExpectPauliString(ps) - orc.dm_expect_pauli_sum(want, 8, P.to_terms(ps)).real) < TOL
    assert abs(dm.Trace() - 1.0) < 1e-12


def test_readout_sampling_bit_exact():
    rng = np.random.default_rng(2)
    n = 6
    c = random_circuit(n, 30, 77, allow_3q=False, allow_ctrl=False)
    nm = _noise_model(rng)
    nm.AddReadoutError(3, N.NewReadoutError(0.11, 0.05))
    dm = densitymatrix.New(n).WithNoise(nm)
    dm.Evolve(c)
    rho = dm.DensityMatrix()
    p01, p10 = dm._readout_arrays()
    probs = orc.dm_readout(orc.dm_diagonal_probs(rho, n), n, p01, p10)
    u = statevector.uniforms(2000, rng)
    assert np.array_equal(dm.Sample(u), orc.sample(probs, u))
    np.testing.assert_array_equal(dm.ApplyReadoutError(dm.DiagonalProbs()), probs)


@pytest.mark.parametrize("dense", [0, 1])
def test_long_stream_planned_in_two_halves(dense):
    # streams of >= 256 ops are analysed and scheduled in two halves (the
    # second on a worker thread): the result must not depend on it, in the
    # channel-form and the dense-superoperator modes, with the JIT on and off
    from goqu_b200 import _abi
    c, nm = workloads.noisy_brickwork(10, layers=12, seed=71)
    ops = encode.density_ops(c, nm)
    assert len(ops) >= 256
    want = orc.dm_evolve(ops, threads=8)
    for jit in (0, 2):
        dm = densitymatrix.New(10).WithNoise(nm)
        dm.set_option(_abi.GQ_OPT_DM_DENSE_CHANNELS, dense)
        dm.set_option(_abi.GQ_OPT_JIT, jit)
        dm.set_option(_abi.GQ_OPT_JIT_MIN_QUBITS, 0)
        dm.Evolve(c)
        assert np.max(np.abs(dm.DensityMatrix() - want)) < TOL
        dm.Close()
