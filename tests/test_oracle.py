"""Pins the CPU oracle: goqu's own known-answer tests (tests/golden/kats.json)
and an independent dense-matrix numpy evaluation on random circuits."""
import math

import numpy as np
import pytest

from goqu_b200 import encode, pauli as P
from oracle import binding as orc

from kat_util import (build_circuit, build_noise, cplx, dense_unitary_state, load_kats,
                      pauli_sum_from_spec, random_circuit)

EPS = 1e-10  # the reference's eps (sim/statevector/sim_test.go:13)


def _sv(spec):
    c = build_circuit(spec)
    return orc.sv_evolve(encode.statevector_ops(c))


def _dm(spec):
    c = build_circuit(spec)
    nm = build_noise(spec)
    return orc.dm_evolve(encode.density_ops(c, nm)), nm


SV_KATS = [k for k in load_kats() if not k.get("dm")]
DM_KATS = [k for k in load_kats() if k.get("dm")]


@pytest.mark.parametrize("kat", SV_KATS, ids=lambda k: k["name"])
def test_oracle_statevector_kats(kat):
    n = kat["n"]
    sv = _sv(kat)
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
        assert np.all(np.delete(p, kat["prob_one"]) < EPS)
    if "norm" in kat:
        assert abs(np.sum(np.abs(sv) ** 2) - kat["norm"]) < EPS
    for qubits, want in kat.get("expect_z", []):
        mask = sum(1 << q for q in qubits)
        assert abs(orc.expect_z(sv, mask, rounded=True) - want) < EPS
    for s, want in kat.get("pauli", []):
        got = orc.expect_pauli_sum(sv, P.to_terms(P.Parse(s)))
        assert abs(got.real - want) < EPS and abs(got.imag) < EPS
    if "pauli_sum" in kat:
        h = pauli_sum_from_spec(n, kat["pauli_sum"])
        got = orc.expect_pauli_sum(sv, P.to_terms(h))
        assert abs(got - complex(*kat["pauli_sum_value"])) < EPS


@pytest.mark.parametrize("kat", DM_KATS, ids=lambda k: k["name"])
def test_oracle_density_kats(kat):
    n = kat["n"]
    rho, nm = _dm(kat)
    dim = 1 << n
    for idx, v in kat.get("rho_at", []):
        assert abs(rho[idx] - complex(*v)) < EPS
    if "trace" in kat:
        assert abs(sum(rho[i * dim + i].real for i in range(dim)) - kat["trace"]) < EPS
    if "purity_below" in kat:
        p = orc.dm_purity(rho, n)
        assert 0 < p < kat["purity_below"] - EPS
    if "diag_nonneg" in kat:
        assert all(rho[i * dim + i].real > -EPS for i in range(dim))
    if "fidelity_with_sv" in kat:
        psi = _sv(kat)
        assert abs(orc.dm_fidelity(rho, n, psi) - kat["fidelity_with_sv"]) < EPS
    if "readout_probs" in kat:
        probs = orc.dm_diagonal_probs(rho, n)
        p01 = np.full(n, -1.0)
        p10 = np.full(n, -1.0)
        for q in range(n):
            re = nm.ReadoutFor(q)
            if re is not None:
                p01[q], p10[q] = re.P01, re.P10
        got = orc.dm_readout(probs, n, p01, p10)
        np.testing.assert_allclose(got, kat["readout_probs"], atol=EPS, rtol=0)


@pytest.mark.parametrize("seed", range(12))
def test_oracle_matches_dense_numpy(seed):
    n = 3 + seed % 5
    c = random_circuit(n, 60, seed)
    got = orc.sv_evolve(encode.statevector_ops(c))
    want = dense_unitary_state(c)
    np.testing.assert_allclose(got, want, atol=1e-12, rtol=0)


def test_oracle_threaded_equals_serial():
    c = random_circuit(17, 25, 7)
    ops = encode.statevector_ops(c)
    a = orc.sv_evolve(ops, threads=0)
    b = orc.sv_evolve(ops, threads=4)
    assert np.array_equal(a, b)  # elementwise kernels: identical arithmetic


def test_oracle_sample_is_sequential_inverse_cdf():
    rng = np.random.default_rng(3)
    p = rng.random(64)
    p /= p.sum()
    u = rng.integers(0, 1 << 53, 200) / float(1 << 53)
    got = orc.sample(p, u)
    cum = np.cumsum(p)  # numpy cumsum of float64 is sequential
    want = [int(np.searchsorted(cum, r, side="right")) for r in u]
    want = [min(w, 63) for w in want]
    assert got.tolist() == want


def test_oracle_fast_sampler_equals_scan():
    rng = np.random.default_rng(4)
    p = rng.random(4096) ** 4
    p /= p.sum()
    u = np.concatenate([rng.integers(0, 1 << 53, 500) / float(1 << 53), [0.0, np.nextafter(1.0, 0)]])
    assert np.array_equal(orc.sample_fast(p, u), orc.sample(p, u))


def test_oracle_density_matches_statevector_noiseless():
    # sim/densitymatrix/sim_test.go:46-120: noiseless rho = |psi><psi|
    for seed in range(4):
        c = random_circuit(4, 30, 100 + seed, allow_3q=False, allow_ctrl=False)
        psi = orc.sv_evolve(encode.statevector_ops(c))
        rho = orc.dm_evolve(encode.density_ops(c))
        np.testing.assert_allclose(rho.reshape(16, 16), np.outer(psi, psi.conj()), atol=1e-12, rtol=0)


def test_kraus_completeness():
    # sim/noise/noise_test.go: sum_k E_k^dagger E_k = I for every channel
    from goqu_b200 import noise as N
    chans = [N.Depolarizing1Q(0.2), N.Depolarizing2Q(0.3), N.AmplitudeDamping(0.4), N.PhaseDamping(0.3),
             N.BitFlip(0.1), N.PhaseFlip(0.2), N.GeneralizedAmplitudeDamping(0.3, 0.6),
             N.ThermalRelaxation(50e-6, 70e-6, 1e-6)]
    for ch in chans:
        d = 1 << ch.Qubits()
        acc = sum(k.reshape(d, d).conj().T @ k.reshape(d, d) for k in ch.Kraus())
        np.testing.assert_allclose(acc, np.eye(d), atol=1e-12)


def test_expectation_value_rounding():
    # ExpectationValue rounds to 1e-14 (sim/statevector/sim.go:368-382)
    from goqu_b200 import circuit as ir
    c = ir.Builder("r", 2).RY(0.3, 0).RY(1.1, 1).Build()
    sv = orc.sv_evolve(encode.statevector_ops(c))
    v = orc.expect_z(sv, 0b11, rounded=True)
    assert v == math.floor(v * 1e14 + 0.5) / 1e14
