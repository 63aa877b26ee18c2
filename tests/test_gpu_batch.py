"""Batched evaluation (gq_batch_run) against single-circuit adjoint runs and
the oracle: QAOA MaxCut circuits of mixed sizes and depths (goqu
algorithm/qaoa), complex128 at 1e-10 and complex64 within 5e-4."""
import numpy as np
import pytest

from goqu_b200 import _abi, batch, circuit as ir, encode, gradient, pauli as P, workloads
from oracle import binding as orc

pytestmark = pytest.mark.gpu


def oracle_energy(c, names, x, h):
    bound = ir.Bind(c, {nm: float(x[i]) for i, nm in enumerate(names)})
    return orc.expect_pauli_sum(orc.sv_evolve(encode.statevector_ops(bound)), P.to_terms(h)).real


@pytest.mark.parametrize("prec,tol", [(_abi.GQ_C128, 1e-10), (_abi.GQ_C64, 5e-4)])
def test_batch_matches_single_runs(prec, tol):
    evals = workloads.qaoa_batch(40, seed=11, n_values=(4, 6, 8, 10, 12, 14, 16), p_range=(1, 4))
    b = batch.Batch(prec)
    energies, grads = b.Run([(c, names, h, x) for c, names, h, x in evals])
    for k, (c, names, h, x) in enumerate(evals[:12]):
        e_ref = oracle_energy(c, names, x, h)
        assert abs(energies[k] - e_ref) < tol
        e1, g1 = gradient.AdjointEvaluator(c, h, names)(x)
        assert np.max(np.abs(grads[k] - g1)) < tol
    # a second run with new angles replays the captured graph
    evals2 = [(c, names, h, (x + 0.1) % np.pi) for c, names, h, x in evals]
    e2, g2 = b.Run(evals2)
    for k in range(0, 40, 7):
        c, names, h, x = evals2[k]
        assert abs(e2[k] - oracle_energy(c, names, x, h)) < tol


def test_batch_energy_only_and_mixed_hamiltonians():
    evals = []
    rng = np.random.default_rng(3)
    for n in (2, 3, 5, 9, 13):
        c, names = workloads.hardware_efficient_ansatz(n, 2)
        evals.append((c, names, workloads.ising_hamiltonian(n), rng.uniform(0, 2 * np.pi, len(names))))
    b = batch.Batch(_abi.GQ_C128)
    b.set_option(_abi.GQ_OPT_USE_GRAPH, 0)
    energies, grads = b.Run(evals, gradients=False)
    assert grads is None
    for k, (c, names, h, x) in enumerate(evals):
        assert abs(energies[k] - oracle_energy(c, names, x, h)) < 1e-10


def test_qaoa_gradients_match_oracle_central_differences():
    # QAOA angles are shared by every RZZ / RX of their layer: check the batched
    # adjoint gradient against central differences of the FP64 oracle energy
    from oracle import binding as orc
    evals = workloads.qaoa_batch(6, seed=21, n_values=(10, 12))
    for prec, tol in ((_abi.GQ_C128, 1e-6), (_abi.GQ_C64, 2e-3)):  # central differences: ~1e-7 roundoff
        b = batch.Batch(prec)
        energies, grads = b.Run(evals)
        for k, (c, names, h, x) in enumerate(evals):
            def energy(xx):
                bound = ir.Bind(c, {nm: float(xx[i]) for i, nm in enumerate(names)})
                return orc.expect_pauli_sum(orc.sv_evolve(encode.statevector_ops(bound)), P.to_terms(h)).real
            assert abs(energies[k] - energy(x)) < (1e-12 if prec == _abi.GQ_C128 else 1e-4)
            for i in range(len(names)):
                xp, xm = np.array(x, float), np.array(x, float)
                xp[i] += 1e-6
                xm[i] -= 1e-6
                assert abs(grads[k][i] - (energy(xp) - energy(xm)) / 2e-6) < tol


def test_segmented_batch_matches_single_segment():
    # 1100 circuits run as two segments (host planning of one overlaps the
    # other's launches); every energy and gradient equals the same circuits
    # run in a batch of their own, and a second call replays both segments
    evals = workloads.qaoa_batch(1100, seed=31, n_values=(4, 6, 8, 10), p_range=(1, 3))
    b = batch.Batch(_abi.GQ_C128)
    energies, grads = b.Run(evals)
    energies2, grads2 = b.Run(evals)
    for k in list(range(0, 1100, 97)) + [549, 550, 551, 1099]:
        one = batch.Batch(_abi.GQ_C128)
        e1, g1 = one.Run([evals[k]])
        assert abs(energies[k] - e1[0]) < 1e-12 and abs(energies2[k] - e1[0]) < 1e-12
        assert np.max(np.abs(grads[k] - g1[0])) < 1e-12 and np.max(np.abs(grads2[k] - g1[0])) < 1e-12
