"""Autotuner for the engine's launch choices.

The pass scheduler and the tile kernels have a few free choices whose best
values depend on the circuit and the device: the launch shape (kernel
variant, which fixes the tile size), the pass budget (FMA per amplitude a
pass may take before the next one starts) and, for the specialised kernels,
CTAs per SM. ``tune_statevector`` and ``tune_batch`` time each candidate on
the device (CUDA events on the handle's stream, GQ_OPT_TIMING) for the
caller's own workload, leave the fastest one set on the handle, and remember
it per workload structure (qubit count, precision, op kinds and qubits; not
the angles), so later calls with other parameters reuse the choice without
timing again.
"""
from __future__ import annotations

import hashlib

import numpy as np

from . import _abi

# Candidate option sets: {option key: value}. The first is the engine default.
STATEVECTOR_CANDIDATES = [
    {},
    {_abi.GQ_OPT_PASS_BUDGET: 160},
    {_abi.GQ_OPT_PASS_BUDGET: 480},
    {_abi.GQ_OPT_KERNEL_VARIANT: 2},
    {_abi.GQ_OPT_JIT_MIN_BLOCKS: 3},
    # the larger tiles (variant 2: 12 qubits for complex128, 13 for complex64)
    # with other budgets and occupancies
    {_abi.GQ_OPT_KERNEL_VARIANT: 2, _abi.GQ_OPT_PASS_BUDGET: 200},
    {_abi.GQ_OPT_KERNEL_VARIANT: 2, _abi.GQ_OPT_PASS_BUDGET: 240},
    {_abi.GQ_OPT_KERNEL_VARIANT: 2, _abi.GQ_OPT_PASS_BUDGET: 400},
    {_abi.GQ_OPT_KERNEL_VARIANT: 2, _abi.GQ_OPT_PASS_BUDGET: 480},
    {_abi.GQ_OPT_KERNEL_VARIANT: 2, _abi.GQ_OPT_JIT_MIN_BLOCKS: 3},
    # persistent CTAs that prefetch their next tile during the last phase
    {_abi.GQ_OPT_JIT_PERSISTENT: 1},
    {_abi.GQ_OPT_KERNEL_VARIANT: 2, _abi.GQ_OPT_JIT_PERSISTENT: 1},
]
BATCH_CANDIDATES = [
    {},
    {_abi.GQ_OPT_PASS_BUDGET: 96},
    {_abi.GQ_OPT_PASS_BUDGET: 640},
]

_cache = {}


def signature(stream):
    """Structure of an op stream: kinds, qubit lists and control counts."""
    h = hashlib.sha1()
    h.update(str(stream.num_qubits).encode())
    for op in stream.array()[:len(stream)]:
        h.update(bytes([op.kind & 0xff, op.num_qubits & 0xff, op.num_controls & 0xff, op.num_kraus & 0xff]))
        h.update(bytes(op.qubits[i] & 0xff for i in range(op.num_qubits)))
    return h.hexdigest()


def _time(run, stats, repeats):
    run()  # first call: scheduling, compilation of specialised kernels
    ms = []
    for _ in range(repeats):
        run()
        ms.append(stats()["last_ms"])
    return float(np.median(ms))


def _tune(key, apply, run, stats, candidates, repeats):
    if key in _cache:
        best = _cache[key]
        apply(best)
        return {"best": best, "cached": True}
    timings = []
    for cand in candidates:
        apply(cand)
        timings.append(_time(run, stats, repeats))
    best = candidates[int(np.argmin(timings))]
    apply(best)
    _cache[key] = best
    return {"best": best, "cached": False, "timings_ms": timings}


def tune_statevector(sim, stream, candidates=None, repeats=3):
    """Times Evolve of `stream` on `sim` for each candidate option set and
    leaves the fastest set on `sim`. Returns {"best", "cached", "timings_ms"}."""
    candidates = candidates or STATEVECTOR_CANDIDATES
    sim.set_option(_abi.GQ_OPT_TIMING, 1)
    sim.set_option(_abi.GQ_OPT_JIT, 2)  # time the kernel that will run, not the compile-time fallback
    defaults = {k: 0 for c in candidates for k in c}
    if _abi.GQ_OPT_KERNEL_VARIANT in defaults:  # the handle's default launch shape
        defaults[_abi.GQ_OPT_KERNEL_VARIANT] = 1 if sim._prec == _abi.GQ_C64 else 0

    def apply(cand):
        for k, v in defaults.items():
            sim.set_option(k, cand.get(k, v))

    key = ("sv", sim.NumQubits(), sim._prec, signature(stream))
    return _tune(key, apply, lambda: sim.evolve_ops(stream), sim.stats, candidates, repeats)


def tune_batch(b, streams, terms, n_params, candidates=None, repeats=2, gradients=True):
    """The same for a batch (gq_batch_run on the caller's circuits)."""
    candidates = candidates or BATCH_CANDIDATES
    b.set_option(_abi.GQ_OPT_TIMING, 1)
    defaults = {k: 0 for c in candidates for k in c}

    def apply(cand):
        for k, v in defaults.items():
            b.set_option(k, cand.get(k, v))

    h = hashlib.sha1()
    for s in streams:
        h.update(signature(s).encode())
    key = ("batch", b.precision, gradients, h.hexdigest())
    return _tune(key, apply, lambda: b.run_encoded(streams, terms, n_params, gradients), b.stats, candidates,
                 repeats)


def clear():
    _cache.clear()
