"""Shot histograms built on the device (gq_sv_sample_counts,
gq_sv_run_counts, gq_dm_sample_counts): the (outcome, count) pairs must be
exactly the histogram of the per-shot indices that gq_sv_sample /
gq_dm_sample return for the same uniforms, in increasing outcome order, and
Run's map must equal goqu's map[bitstring]int built from those indices
(sim/statevector/sim.go:40-58, 306-316). Sizes cover partial sort tiles,
one to four radix passes (1 to 28 qubits), a single outcome and no shots."""
import ctypes

import numpy as np
import pytest

from goqu_b200 import _abi, densitymatrix, encode, noise as N, statevector, workloads
from goqu_b200 import circuit as ir

pytestmark = pytest.mark.gpu


def hist(idx):
    v, c = np.unique(np.asarray(idx, dtype=np.uint64), return_counts=True)
    return v, c.astype(np.uint64)


@pytest.mark.parametrize("n,shots,layers", [(1, 5, 1), (3, 1000, 2), (9, 1025, 3), (14, 4096, 4), (17, 100000, 3),
                                            (20, 300001, 6)])
def test_statevector_counts_equal_histogram_of_samples(n, shots, layers):
    sim = statevector.New(n)
    sim.Evolve(workloads.random_layers(n, layers, seed=n))
    u = statevector.uniforms(shots, np.random.default_rng(shots))
    idx = sim.Sample(u)
    outc, cnt = sim.SampleCounts(u)
    want_v, want_c = hist(idx)
    assert np.array_equal(outc, want_v) and np.array_equal(cnt, want_c)
    assert int(cnt.sum()) == shots
    sim.Close()


def test_single_outcome_and_no_shots():
    sim = statevector.New(6)
    sim.Evolve(ir.Builder("x", 6).X(2).X(5).Build())  # |100100>
    outc, cnt = sim.SampleCounts(statevector.uniforms(3000, np.random.default_rng(1)))
    assert outc.tolist() == [0b100100] and cnt.tolist() == [3000]
    outc, cnt = sim.SampleCounts(np.empty(0))
    assert outc.size == 0 and cnt.size == 0
    sim.Close()


def test_run_counts_c_abi_and_run_map():
    n = 12
    c = workloads.random_layers(n, 5, seed=3)
    stream = encode.statevector_ops(c)
    u = statevector.uniforms(20000, np.random.default_rng(9))
    sim = statevector.New(n)
    idx = np.empty(u.size, dtype=np.uint64)
    _abi.check(_abi.lib().gq_sv_run(sim.handle, stream.ptr(), len(stream), u.ctypes.data_as(ctypes.POINTER(
        ctypes.c_double)), u.size, idx.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
    outc = np.empty(u.size, dtype=np.uint64)
    cnt = np.empty(u.size, dtype=np.uint64)
    nd = ctypes.c_size_t()
    _abi.check(_abi.lib().gq_sv_run_counts(sim.handle, stream.ptr(), len(stream),
                                           u.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), u.size,
                                           outc.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                           cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), ctypes.byref(nd)))
    v, k = hist(idx)
    assert nd.value == v.size
    assert np.array_equal(outc[:nd.value], v) and np.array_equal(cnt[:nd.value], k)
    # Run's map equals the one built from per-shot indices with the same draws
    m = sim.Run(c, 5000, np.random.default_rng(4))
    sim.Evolve(c)
    ref = statevector.counts_from_indices(sim.Sample(statevector.uniforms(5000, np.random.default_rng(4))), n)
    assert m == ref
    sim.Close()


def test_counts_28q_four_radix_passes():
    # 28-bit outcomes: four 8-bit digit passes (bits 0-31) over 2^20 shots
    n = 28
    sim = statevector.New(n)
    b = ir.Builder("h", n)
    for q in range(n):
        b.H(q)
    sim.Evolve(b.Build())
    u = statevector.uniforms(1 << 20, np.random.default_rng(28))
    idx = sim.Sample(u)
    outc, cnt = sim.SampleCounts(u)
    v, k = hist(idx)
    assert np.array_equal(outc, v) and np.array_equal(cnt, k)
    sim.Close()


def test_density_matrix_counts_with_readout_error():
    n = 5
    c, nm = workloads.noisy_brickwork(n, layers=3, seed=5)
    for q in (0, 3):
        nm.AddReadoutError(q, N.NewReadoutError(0.02, 0.05))
    dm = densitymatrix.New(n).WithNoise(nm)
    dm.Evolve(c)
    u = statevector.uniforms(7777, np.random.default_rng(2))
    idx = dm.Sample(u)
    outc, cnt = dm.SampleCounts(u)
    v, k = hist(idx)
    assert np.array_equal(outc, v) and np.array_equal(cnt, k)
    dm.Close()
