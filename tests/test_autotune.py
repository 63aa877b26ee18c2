"""Autotuner logic on the CPU with a stand-in handle whose timing depends on
the options set: the fastest candidate is chosen, left set, and remembered
per workload structure (angles do not matter)."""
import numpy as np

from goqu_b200 import _abi, autotune, encode, workloads


class FakeSim:
    def __init__(self, n, prec=_abi.GQ_C128):
        self.n, self._prec, self.opts, self.calls = n, prec, {}, 0

    def NumQubits(self):
        return self.n

    def set_option(self, k, v):
        self.opts[k] = v

    def evolve_ops(self, stream):
        self.calls += 1

    def stats(self):
        budget = self.opts.get(_abi.GQ_OPT_PASS_BUDGET, 0)
        variant = self.opts.get(_abi.GQ_OPT_KERNEL_VARIANT, 0)
        return {"last_ms": 10.0 + (0 if budget == 480 else 1.0) + 0.5 * variant}


def test_picks_fastest_and_caches_by_structure():
    autotune.clear()
    s1 = encode.statevector_ops(workloads.random_layers(6, 3, 1))
    sim = FakeSim(6)
    r = autotune.tune_statevector(sim, s1)
    assert r["best"] == {_abi.GQ_OPT_PASS_BUDGET: 480} and not r["cached"]
    assert sim.opts[_abi.GQ_OPT_PASS_BUDGET] == 480 and sim.opts[_abi.GQ_OPT_KERNEL_VARIANT] == 0
    assert len(r["timings_ms"]) == len(autotune.STATEVECTOR_CANDIDATES)
    # same structure, other angles: cached, no timing calls
    s2 = encode.statevector_ops(workloads.random_layers(6, 3, 2))
    assert autotune.signature(s1) == autotune.signature(s2)
    sim2 = FakeSim(6)
    r2 = autotune.tune_statevector(sim2, s2)
    assert r2["cached"] and sim2.calls == 0 and sim2.opts[_abi.GQ_OPT_PASS_BUDGET] == 480
    # another structure is timed again
    s3 = encode.statevector_ops(workloads.random_layers(6, 4, 1))
    assert autotune.signature(s3) != autotune.signature(s1)
    assert not autotune.tune_statevector(FakeSim(6), s3)["cached"]


def test_complex64_keeps_its_default_shape():
    autotune.clear()
    sim = FakeSim(6, _abi.GQ_C64)
    autotune.tune_statevector(sim, encode.statevector_ops(workloads.random_layers(6, 2, 3)),
                              candidates=[{}, {_abi.GQ_OPT_KERNEL_VARIANT: 2}])
    assert sim.opts[_abi.GQ_OPT_KERNEL_VARIANT] == 1
