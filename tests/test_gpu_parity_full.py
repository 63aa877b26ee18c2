"""Parity at the benchmark configurations' own sizes against the FP64 oracle.

* 28-qubit statevector (the headline size): U3 + CNOT brickwork layers and a
  28-qubit QFT (algorithm/qpe/qpe.go:170-182), run by the specialised pass
  kernels (the 28-qubit pass structures: CTA-index predicates, fused chains,
  run-time controlled phases). Amplitudes within 1e-12 (complex128); 1024
  sampled indices bit-exact with the sequential inverse CDF
  (sim/statevector/sim.go:288-298); complex64 error stated and bounded.
* 12-qubit noisy density matrix (2^24 entries): the brickwork with
  depolarizing channels after every gate and amplitude damping on idle
  qubits (sim/densitymatrix/sim.go:80-255, sim/noise/channel.go): entries,
  <Z_i> and the trace within 1e-12.
* 20-qubit, 400-parameter adjoint gradient: 40 parameters (RY and RZ of two
  qubits per layer, every layer) against the oracle's parameter shift
  (algorithm/gradient/gradient.go:49-66) within 1e-8.
* 20-qubit QAOA circuits of the batch configuration: batched gradients
  against central differences of the oracle's energy.
The layer counts of the first two are below the benchmark's (4 of 40, 2 of
30) so that the oracle (goqu's loops on the host cores) finishes in about a
minute; the layers repeat the same structure, and the benchmark itself
checks the full 28-qubit circuit.
"""
import os

import numpy as np
import pytest

from goqu_b200 import _abi, batch, densitymatrix, encode, gradient, pauli as P, statevector, workloads
from oracle import binding as orc
from oracle import gradient as og

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 8


def max_abs_diff(a, b, chunk=1 << 24):
    m = 0.0
    for s in range(0, a.size, chunk):
        m = max(m, float(np.max(np.abs(a[s:s + chunk] - b[s:s + chunk]))))
    return m


def test_statevector_28q_layers_qft_matches_oracle():
    n = 28
    c = workloads.random_layers_qft(n, 4, 2028)
    stream = encode.statevector_ops(c)
    want = orc.sv_evolve(stream, threads=THREADS)
    sim = statevector.New(n)
    sim.set_option(_abi.GQ_OPT_JIT, 2)
    sim.evolve_ops(stream)
    assert sim.stats()["jit_passes"] == sim.stats()["passes"] > 0
    got = sim.StateVector()
    err = max_abs_diff(got, want)
    assert err <= 1e-12, err
    u = statevector.uniforms(1024, np.random.default_rng(2028))
    idx = sim.Sample(u)
    assert np.array_equal(idx, orc.sample_fast(orc.probabilities(got), u))
    sim.Close()
    del got
    # complex64 bulk on the same circuit: error against the same FP64 state
    s64 = statevector.New(n, _abi.GQ_C64)
    s64.set_option(_abi.GQ_OPT_JIT, 2)
    s64.evolve_ops(stream)
    g64 = s64.StateVector()
    s64.Close()
    err64 = max_abs_diff(g64, want)
    # amplitudes are ~2^-14 = 6e-5 here; FP32 rounding over ~600 gates stays
    # far below 1e-7 absolute
    assert err64 <= 1e-7, err64


def test_density_matrix_12q_noisy_matches_oracle():
    n = 12
    c, nm = workloads.noisy_brickwork(n, layers=2, seed=12)
    s = encode.density_ops(c, nm)
    assert any(op.kind == _abi.GQ_OP_CHANNEL for op in s.array()[:len(s)])
    want = orc.dm_evolve(s, threads=THREADS)
    dm = densitymatrix.New(n).WithNoise(nm)
    dm.set_option(_abi.GQ_OPT_JIT, 2)
    _abi.check(_abi.lib().gq_dm_evolve(dm._h, s.ptr(), len(s)))
    got = dm.DensityMatrix()
    assert max_abs_diff(got.reshape(-1), want.reshape(-1)) <= 1e-12
    for q in range(n):
        term = P.to_terms(P.ZOn([q], n))
        assert abs(dm.ExpectPauliString(P.ZOn([q], n)) - orc.dm_expect_pauli_sum(want, n, term).real) <= 1e-12
    tr = dm.Trace()
    assert abs(tr - np.trace(want.reshape(1 << n, 1 << n)).real) <= 1e-12
    dm.Close()


def test_adjoint_20q_400_params_vs_oracle_parameter_shift():
    c, names = workloads.hardware_efficient_ansatz(20, 10)
    h = workloads.ising_hamiltonian(20)
    x = np.random.default_rng(20).uniform(0, 2 * np.pi, 400)
    ev = gradient.AdjointEvaluator(c, h, names)
    ev.sim.set_option(_abi.GQ_OPT_JIT, 2)
    e, g = ev(x)
    sel = og.stratified_hea_params(20, 10)
    assert len(sel) == 40
    ref = og.parameter_shift(c, names, x, h, sel, threads=THREADS)
    assert np.max(np.abs(g[sel] - ref)) <= 1e-8
    assert abs(e - og.energy(c, names, x, h, threads=THREADS)) <= 1e-10


def test_qaoa_20q_batch_gradients_vs_oracle_central_differences():
    evals = [e for e in workloads.qaoa_batch(4096, seed=4) if e[0].NumQubits() == 20][:3]
    assert len(evals) == 3
    for prec, tol_e, tol_g in ((_abi.GQ_C128, 1e-10, 1e-6), (_abi.GQ_C64, 1e-4, 2e-3)):
        b = batch.Batch(prec)
        energies, grads = b.Run(evals)
        b.Close()
        for k, (c, names, h, x) in enumerate(evals):
            x = np.asarray(x, float)
            assert abs(energies[k] - og.energy(c, names, x, h, threads=THREADS)) < tol_e
            fd = og.parameter_shift(c, names, x, h, threads=THREADS, shift=1e-6, denom=2e-6)
            assert np.max(np.abs(grads[k] - fd)) < tol_g
