"""Sweeps (gq_sweep_run, gq_sweep_run_density) against the oracle: goqu's
sweep.RunSim / RunDensitySim (sweep/run.go:27-171) bind the circuit per
point, Run it with `shots` samples and return the counts in sweep order.
Counts must equal the oracle's sequential inverse-CDF sampling
(sim/statevector/sim.go:288-298) of the oracle's own state with the same
uniforms; a failing point reports its status without stopping the others."""
import ctypes

import numpy as np
import pytest

from goqu_b200 import _abi, circuit as ir, encode, noise as N, param as prm, statevector, sweep
from oracle import binding as orc

pytestmark = pytest.mark.gpu


def ansatz(n, layers):
    th = prm.NewVector("t", 2 * n * layers)
    b = ir.Builder("sweep", n)
    k = 0
    for _ in range(layers):
        for q in range(n):
            b.SymRY(th.At(k), q).SymRZ(th.At(k + 1), q)
            k += 2
        for q in range(n - 1):
            b.CNOT(q, q + 1)
    return b.Build(), th.Names()


def bindings(names, count, seed):
    rng = np.random.default_rng(seed)
    return [{nm: float(v) for nm, v in zip(names, rng.uniform(0, 2 * np.pi, len(names)))} for _ in range(count)]


@pytest.mark.parametrize("precision", [_abi.GQ_C128, _abi.GQ_C64])
def test_run_sim_100_points_match_oracle_sampling(precision):
    n, shots = 7, 500
    c, names = ansatz(n, 2)
    pts = bindings(names, 100, 3)
    res = sweep.RunSim(c, shots, pts, rng=np.random.default_rng(11), precision=precision)
    assert [r.Index for r in res] == list(range(100))
    rng = np.random.default_rng(11)
    mismatched = 0
    for r, b in zip(res, pts):
        assert r.Err is None and r.Bindings == b
        u = statevector.uniforms(shots, rng)
        st = orc.sv_evolve(encode.statevector_ops(ir.Bind(c, b)))
        want = statevector.counts_from_indices(orc.sample_fast(orc.probabilities(st), u), n)
        if precision == _abi.GQ_C128:
            assert r.Counts == want
        else:  # complex64 states move CDF boundaries by ~1e-7: nearly every shot agrees
            mismatched += sum(abs(r.Counts.get(k, 0) - want.get(k, 0)) for k in set(want) | set(r.Counts))
        assert sum(r.Counts.values()) == shots
    assert mismatched <= 0.01 * 100 * shots


def test_run_density_sim_with_noise_and_readout_matches_oracle():
    n, shots = 4, 3000
    c, names = ansatz(n, 2)
    nm = N.New()
    nm.AddDefaultError(1, N.Depolarizing1Q(0.01))
    nm.AddDefaultError(2, N.Depolarizing2Q(0.02))
    nm.AddReadoutError(1, N.NewReadoutError(0.03, 0.06))
    pts = bindings(names, 20, 5)
    res = sweep.RunDensitySim(c, shots, pts, nm=nm, rng=np.random.default_rng(2))
    rng = np.random.default_rng(2)
    p01 = np.array([-1.0, 0.03, -1.0, -1.0])
    p10 = np.array([-1.0, 0.06, -1.0, -1.0])
    for r, b in zip(res, pts):
        assert r.Err is None
        u = statevector.uniforms(shots, rng)
        rho = orc.dm_evolve(encode.density_ops(ir.Bind(c, b), nm))
        probs = orc.dm_readout(orc.dm_diagonal_probs(rho, n), n, p01, p10)
        want = statevector.counts_from_indices(orc.sample_fast(probs, u), n)
        assert r.Counts == want


def test_failing_point_does_not_stop_the_others():
    n, shots = 3, 64
    good = encode.statevector_ops(ir.Builder("g", n).H(0).CNOT(0, 1).Build())
    bad = encode.OpStream(n)
    bad.add(_abi.GQ_OP_CNOT, [0, 7], np.eye(4))  # qubit 7 of a 3-qubit state
    u = [np.ascontiguousarray(statevector.uniforms(shots, np.random.default_rng(k))) for k in range(3)]
    pts = (_abi.gq_sweep_point * 3)()
    for i, s in enumerate((good, bad, good)):
        pts[i].ops, pts[i].n_ops = s.ptr(), len(s)
        pts[i].uniforms = u[i].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    stride = min(shots, 1 << n)
    outc = np.zeros(3 * stride, dtype=np.uint64)
    cnt = np.zeros(3 * stride, dtype=np.uint64)
    nd = (ctypes.c_size_t * 3)()
    st = (ctypes.c_int32 * 3)()
    rc = _abi.lib().gq_sweep_run(n, _abi.GQ_C128, pts, 3, shots, outc.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                 cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), nd, st)
    assert rc == _abi.GQ_OK
    assert list(st) == [_abi.GQ_OK, _abi.GQ_EINVAL, _abi.GQ_OK]
    assert b"point 1" in _abi.lib().gq_last_error()
    for i in (0, 2):
        assert set(outc[i * stride:i * stride + nd[i]].tolist()) <= {0, 3}
        assert int(cnt[i * stride:i * stride + nd[i]].sum()) == shots
