"""Parity of the sm_100a statevector engine with the oracle (GPU).

Bars: complex128 amplitudes and expectations within 1e-12 absolute of the
FP64 oracle; complex64 amplitudes within 2e-5 (FP32 gate arithmetic, stated
per test); sampled indices bit-exact with goqu's sequential inverse CDF given
the same state and uniforms.
"""
import math

import numpy as np
import pytest

from goqu_b200 import _abi, circuit as ir, encode, gate as G, pauli as P, statevector, workloads
from oracle import binding as orc

from kat_util import build_circuit, cplx, load_kats, pauli_sum_from_spec, random_circuit

pytestmark = pytest.mark.gpu

TOL128 = 1e-12
TOL64 = 2e-5
EPS = 1e-10  # the reference tests' eps


def evolve(c, precision=_abi.GQ_C128, tile=None, budget=None):
    sim = statevector.New(c.NumQubits(), precision)
    if tile is not None:
        sim.set_option(_abi.GQ_OPT_TILE_QUBITS, tile)
    if budget is not None:
        sim.set_option(_abi.GQ_OPT_PASS_BUDGET, budget)
    sim.Evolve(c)
    return sim


SV_KATS = [k for k in load_kats() if not k.get("dm")]


@pytest.mark.parametrize("kat", SV_KATS, ids=lambda k: k["name"])
def test_known_answers(kat):
    c = build_circuit(kat)
    sim = evolve(c)
    sv = sim.StateVector()
    n = kat["n"]
    if "state" in kat:
        np.testing.assert_allclose(sv, cplx(kat["state"]), atol=EPS, rtol=0)
    if "abs_all" in kat:
        np.testing.assert_allclose(np.abs(sv), kat["abs_all"], atol=EPS, rtol=0)
    for idx, v in kat.get("abs_at", []):
        assert abs(abs(sv[idx]) - v) < EPS
    for idx, v in kat.get("amp_at", []):
        assert abs(sv[idx] - complex(*v)) < EPS
    if "prob_one" in kat:
        p = np.abs(sv) ** 2
        assert abs(p[kat["prob_one"]] - 1) < EPS
    for qubits, want in kat.get("expect_z", []):
        assert abs(sim.ExpectationValue(qubits) - want) < EPS
    for s, want in kat.get("pauli", []):
        assert abs(sim.ExpectPauliString(P.Parse(s)) - want) < EPS
    if "pauli_sum" in kat:
        h = pauli_sum_from_spec(n, kat["pauli_sum"])
        got = sim.expect_terms(P.to_terms(h))
        assert abs(got - complex(*kat["pauli_sum_value"])) < EPS


@pytest.mark.parametrize("n,seed,tile,budget", [
    (1, 1, None, None), (2, 2, None, None), (3, 3, None, None), (4, 4, None, None), (5, 5, None, None),
    (7, 6, None, None), (9, 7, None, None), (11, 8, None, None), (12, 9, None, None), (13, 10, None, None),
    (14, 11, 8, None), (15, 12, 10, 20), (16, 13, 11, 200), (12, 14, 6, 4)])
def test_random_circuits_match_oracle(n, seed, tile, budget):
    c = random_circuit(n, 120, seed, allow_3q=n >= 3, allow_ctrl=n >= 4, allow_reset=True)
    ops = encode.statevector_ops(c)
    want = orc.sv_evolve(ops)
    sim = evolve(c, tile=tile, budget=budget)
    got = sim.StateVector()
    assert np.max(np.abs(got - want)) < TOL128


@pytest.mark.parametrize("n,seed", [(6, 31), (12, 32), (17, 33)])
def test_complex64_error_vs_oracle(n, seed):
    c = random_circuit(n, 80, seed, allow_3q=n >= 3, allow_ctrl=n >= 4)
    want = orc.sv_evolve(encode.statevector_ops(c))
    got = evolve(c, _abi.GQ_C64).StateVector()
    assert np.max(np.abs(got - want)) < TOL64


def test_brickwork_20q_config_matches_oracle():
    c = workloads.random_layers(20, layers=20, seed=2024)
    assert workloads.count_gates(c) == 590
    ops = encode.statevector_ops(c)
    want = orc.sv_evolve(ops, threads=8)
    sim = evolve(c)
    got = sim.StateVector()
    assert np.max(np.abs(got - want)) < TOL128
    u = statevector.uniforms(1024, np.random.default_rng(1))
    assert np.array_equal(sim.Sample(u), orc.sample(orc.probabilities(got), u))


def test_layers_plus_qft_22q_matches_oracle():
    c = workloads.random_layers_qft(22, layers=4, seed=7)
    want = orc.sv_evolve(encode.statevector_ops(c), threads=8)
    got = evolve(c).StateVector()
    assert np.max(np.abs(got - want)) < TOL128


def test_expectations_match_oracle():
    c = random_circuit(13, 100, 41)
    sim = evolve(c)
    sv = sim.StateVector()
    h = workloads.ising_hamiltonian(13)
    got = sim.expect_terms(P.to_terms(h))
    want = orc.expect_pauli_sum(sv, P.to_terms(h))
    assert abs(got - want) < TOL128
    rng = np.random.default_rng(5)
    for _ in range(20):
        ops = {int(q): [P.X, P.Y, P.Z][rng.integers(3)] for q in rng.choice(13, 4, replace=False)}
        ps = P.NewPauliString(complex(*rng.normal(size=2)), ops, 13)
        assert abs(sim.expect_terms(P.to_terms(ps)) - orc.expect_pauli_sum(sv, P.to_terms(ps))) < TOL128
    for mask in (0b1, 0b101, 0b1111111111111):
        qs = [q for q in range(13) if mask >> q & 1]
        assert abs(sim.ExpectationValue(qs) - orc.expect_z(sv, mask, rounded=True)) < 2e-14


def test_sampling_bit_exact_random_uniforms():
    c = random_circuit(14, 80, 51)
    sim = evolve(c)
    probs = orc.probabilities(sim.StateVector())
    u = statevector.uniforms(4096, np.random.default_rng(3))
    assert np.array_equal(sim.Sample(u), orc.sample(probs, u))


def test_sampling_bit_exact_on_boundaries():
    # uniforms placed exactly on (and one ulp around) the sequential cumulative
    # sums force the flagged-shot exact path
    c = random_circuit(12, 60, 52)
    sim = evolve(c)
    probs = orc.probabilities(sim.StateVector())
    rng = np.random.default_rng(9)
    at = np.sort(rng.choice(probs.size - 1, 64, replace=False))
    _, cum = orc.cumsum_at(probs, at)
    u = np.concatenate([cum, np.nextafter(cum, 0), np.nextafter(cum, 2), [0.0, np.nextafter(1.0, 0)]])
    u = u[(u >= 0) & (u < 1)]
    assert np.array_equal(sim.Sample(u), orc.sample(probs, u))


@pytest.mark.parametrize("n,prec", [(20, _abi.GQ_C128), (24, _abi.GQ_C128), (22, _abi.GQ_C64)])
def test_sampling_bit_exact_large_states(n, prec):
    # large states: every interval p_i is far below any a-priori rounding
    # bound, so this exercises the exact binade-step sampler end to end
    c = workloads.random_layers(n, layers=3, seed=n)
    sim = evolve(c, prec)
    probs = orc.probabilities(sim.StateVector())
    u = statevector.uniforms(4096, np.random.default_rng(n))
    assert np.array_equal(sim.Sample(u), orc.sample_fast(probs, u))
    sel = np.random.default_rng(1).choice(probs.size - 1, 32, replace=False)
    _, cum = orc.cumsum_at(probs, sel)
    uu = np.concatenate([cum, np.nextafter(cum, 0), np.nextafter(cum, 2)])
    uu = uu[uu < 1.0]
    assert np.array_equal(sim.Sample(uu), orc.sample_fast(probs, uu))


def test_sampling_degenerate_states():
    # |0...0>: every uniform maps to index 0; uniform superposition: exact dyadic sums
    sim = statevector.New(12)
    u = statevector.uniforms(500, np.random.default_rng(4))
    assert np.all(sim.Sample(u) == 0)
    b = ir.Builder("h", 12)
    for q in range(12):
        b.H(q)
    sim.Evolve(b.Build())
    probs = orc.probabilities(sim.StateVector())
    edges = np.arange(1, 4096, 97) / 4096.0
    uu = np.concatenate([u, edges, np.nextafter(edges, 0)])
    assert np.array_equal(sim.Sample(uu), orc.sample(probs, uu))


@pytest.mark.parametrize("n", [18, 22])
def test_sampling_sparse_and_basis_states(n):
    # a basis state far into the vector (the running sum is exactly 1 from
    # there on, a long all-zero tail), and a sparse state whose few weights
    # span many binades (every crossing walks its chunk element by element)
    sim = statevector.New(n)
    u = statevector.uniforms(2000, np.random.default_rng(n))
    k = (1 << n) - 12345
    st = np.zeros(1 << n, dtype=np.complex128)
    st[k] = 1
    sim.SetStateVector(st)
    assert np.all(sim.Sample(u) == k)
    rng = np.random.default_rng(n + 1)
    idx = np.sort(rng.choice(1 << n, 40, replace=False))
    st = np.zeros(1 << n, dtype=np.complex128)
    st[idx] = rng.normal(size=40) * 2.0 ** rng.integers(-20, 0, size=40) + 1j * rng.normal(size=40) * 1e-3
    st /= np.linalg.norm(st)
    sim.SetStateVector(st)
    probs = orc.probabilities(sim.StateVector())
    _, cum = orc.cumsum_at(probs, idx[:-1])
    uu = np.concatenate([u, cum, np.nextafter(cum, 0), np.nextafter(cum, 2)])
    uu = uu[(uu >= 0) & (uu < 1)]
    assert np.array_equal(sim.Sample(uu), orc.sample_fast(probs, uu))


def test_run_counts_statistics():
    # sim/statevector/sim_test.go:135-167: Bell counts only "00"/"11", each ~5000
    c = ir.Builder("bell", 2).H(0).CNOT(0, 1).MeasureAll().Build()
    counts = statevector.New(2).Run(c, 10000, rng=np.random.default_rng(11))
    assert set(counts) <= {"00", "11"}
    assert 4000 < counts["00"] < 6000 and 4000 < counts["11"] < 6000


def test_apply_composes_without_reset():
    a = random_circuit(8, 30, 61)
    b = random_circuit(8, 30, 62)
    sim = evolve(a)
    sim.Apply(b)
    want = orc.sv_apply(orc.sv_evolve(encode.statevector_ops(a)), encode.statevector_ops(b))
    assert np.max(np.abs(sim.StateVector() - want)) < TOL128


def test_set_state_roundtrip_and_reset():
    rng = np.random.default_rng(8)
    psi = rng.normal(size=1 << 9) + 1j * rng.normal(size=1 << 9)
    psi /= np.linalg.norm(psi)
    sim = statevector.New(9)
    sim.SetStateVector(psi)
    assert np.array_equal(sim.StateVector(), psi)
    sim.Reset()
    e0 = np.zeros(1 << 9, dtype=complex)
    e0[0] = 1
    assert np.array_equal(sim.StateVector(), e0)


def test_errors_mirror_reference():
    sim = statevector.New(3)
    with pytest.raises(ValueError, match="circuit has 2 qubits, simulator has 3"):
        sim.Evolve(ir.Builder("x", 2).H(0).Build())
    with pytest.raises(ValueError, match="unsupported gate size: 4 qubits"):
        big = G.Unitary("U4", np.eye(16))
        statevector.New(5).Evolve(ir.Builder("x", 5).Apply(big, 0, 1, 2, 3).Build())
    with pytest.raises(ValueError, match="PauliString has 2 qubits"):
        sim.ExpectPauliString(P.Parse("ZZ"))
    with pytest.raises(_abi.GQError):
        sim.Sample(np.array([1.5]))


def test_large_state_properties_26q():
    # full-size property checks: norm preserved, circuit followed by its inverse
    # returns |0...0>, complex64 agrees with complex128
    n = 26
    c = workloads.random_layers_qft(n, layers=6, seed=99)
    inv_ops = []
    for op in reversed(c.Ops()):
        inv_ops.append(ir.Operation(op.Gate.Inverse(), op.Qubits))
    inv = ir.Circuit("inv", n, 0, inv_ops)
    sim = evolve(c)
    p = sim.Probabilities()
    assert abs(p.sum() - 1.0) < 1e-10
    sim64 = evolve(c, _abi.GQ_C64)
    d = np.max(np.abs(sim64.StateVector() - sim.StateVector()))
    assert d < 5e-5
    sim.Apply(inv)
    a0 = sim.StateVector()[0]
    assert abs(a0 - 1.0) < 1e-10


@pytest.mark.parametrize("n,seed", [(9, 71), (14, 72)])
def test_dense_fusion_option_matches_oracle(n, seed):
    c = random_circuit(n, 150, seed, allow_reset=True)
    want = orc.sv_evolve(encode.statevector_ops(c))
    sim = statevector.New(n)
    sim.set_option(_abi.GQ_OPT_FUSE_DENSE, 1)
    sim.Evolve(c)
    assert np.max(np.abs(sim.StateVector() - want)) < TOL128
