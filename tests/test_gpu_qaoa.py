"""The dedicated MaxCut QAOA path (gq_qaoa_maxcut_batch) against the general
batch path (gq_batch_run on the same circuits' gates) and the FP64 oracle:
goqu's qaoa.Run circuits (algorithm/qaoa/qaoa.go:68-93, 164-196) with
MaxCutHamiltonian (maxcut.go:13-35). Sizes cover the one-CTA path (n <= 12,
including n < 9 with a partial warp of work), one group pass (13..20) and two
(21); complex64 amplitudes, FP64 reductions."""
import os

import numpy as np
import pytest

from goqu_b200 import _abi, batch, qaoa, workloads
from oracle import gradient as og

pytestmark = pytest.mark.gpu
TH = os.cpu_count() or 8


def mixed_batch():
    evals = []
    for k, n in enumerate((4, 6, 8, 10, 12, 14, 16, 20, 22)):
        evals += workloads.qaoa_batch(3, seed=100 + k, n_values=(n,), p_range=(1, 4))
    return evals


def test_matches_general_batch_and_oracle():
    evals = mixed_batch()
    items = [qaoa.from_evaluation(e) for e in evals]
    e_fast, g_fast = qaoa.MaxCutBatch().Run(items)
    e_gen, g_gen = batch.Batch(_abi.GQ_C64).Run(evals)
    for k in range(len(evals)):
        assert abs(e_fast[k] - e_gen[k]) < 1e-4, (k, e_fast[k], e_gen[k])
        assert np.max(np.abs(g_fast[k] - g_gen[k])) < 5e-4, k
    for k in range(0, len(evals), 4):  # against the FP64 oracle
        c, names, h, x = evals[k]
        x = np.asarray(x, float)
        assert abs(e_fast[k] - og.energy(c, names, x, h, threads=TH)) < 1e-4
        fd = og.parameter_shift(c, names, x, h, threads=TH, shift=1e-6, denom=2e-6)
        assert np.max(np.abs(g_fast[k] - fd)) < 2e-3


def test_odd_sizes_and_two_group_passes():
    # odd n (3-regular graphs need even n: a ring plus chords instead) and n = 21, 23
    rng = np.random.default_rng(3)
    items, evals = [], []
    from goqu_b200 import circuit as ir
    for n in (5, 11, 13, 21):
        edges = [(i, (i + 1) % n) for i in range(n)] + [(i, (i + n // 2) % n) for i in range(0, n, 3)]
        edges = [(a, b) for a, b in edges if a != b]
        p = int(rng.integers(1, 4))
        gam, bet = rng.uniform(0, np.pi, p), rng.uniform(0, np.pi, p)
        h = workloads.maxcut_hamiltonian(edges, n)
        c, names = workloads.qaoa_circuit(h, p)
        x = np.empty(2 * p)
        x[0::2], x[1::2] = gam, bet
        items.append((n, edges, gam, bet))
        evals.append((c, names, h, x))
    e, g = qaoa.MaxCutBatch().Run(items)
    for k, (c, names, h, x) in enumerate(evals):
        assert abs(e[k] - og.energy(c, names, x, h, threads=TH)) < 2e-4
        fd = og.parameter_shift(c, names, x, h, threads=TH, shift=1e-6, denom=2e-6)
        assert np.max(np.abs(g[k] - fd)) < 3e-3


def test_deterministic_and_energy_only():
    items = [qaoa.from_evaluation(e) for e in workloads.qaoa_batch(40, seed=9, n_values=(10, 14, 18))]
    b = qaoa.MaxCutBatch()
    e1, g1 = b.Run(items)
    e2, g2 = b.Run(items)
    assert np.array_equal(e1, e2) and all(np.array_equal(a, c) for a, c in zip(g1, g2))
    e3, none = b.Run(items, gradients=False)
    assert none is None and np.array_equal(e3, e1)


def test_rejects_bad_items():
    with pytest.raises(_abi.GQError):
        qaoa.MaxCutBatch(_abi.GQ_C128).Run([(6, [(0, 1)], [0.1], [0.2])])
    with pytest.raises(_abi.GQError, match="edge out of range"):
        qaoa.MaxCutBatch().Run([(6, [(0, 6)], [0.1], [0.2])])
    with pytest.raises(_abi.GQError, match="num_qubits"):
        qaoa.MaxCutBatch().Run([(3, [(0, 1)], [0.1], [0.2])])
