"""Autotuner on the device (GPU): it times the candidates for a 20-qubit
circuit, leaves the fastest set, and the tuned handle still matches the FP64
oracle within 1e-12."""
import numpy as np
import pytest

from goqu_b200 import _abi, autotune, batch, encode, statevector, workloads
from oracle import binding as orc

pytestmark = pytest.mark.gpu


def test_tune_statevector_keeps_results_exact():
    autotune.clear()
    c = workloads.random_layers(20, 6, 7)
    stream = encode.statevector_ops(c)
    sim = statevector.New(20)
    r = autotune.tune_statevector(sim, stream, repeats=2)
    assert not r["cached"] and len(r["timings_ms"]) == len(autotune.STATEVECTOR_CANDIDATES)
    assert all(t > 0 for t in r["timings_ms"])
    sim.Evolve(c)
    np.testing.assert_allclose(sim.StateVector(), orc.sv_evolve(stream), atol=1e-12, rtol=0)
    assert autotune.tune_statevector(statevector.New(20), stream)["cached"]


def test_tune_batch():
    autotune.clear()
    evals = workloads.qaoa_batch(32, seed=9, n_values=(10, 12))
    streams, terms = batch.Batch.encode(evals)
    b = batch.Batch(_abi.GQ_C64)
    npar = [len(e[1]) for e in evals]
    r = autotune.tune_batch(b, streams, terms, npar)
    assert len(r["timings_ms"]) == len(autotune.BATCH_CANDIDATES)
    e, g = b.run_encoded(streams, terms, npar)
    assert np.all(np.isfinite(e)) and len(g) == 32
