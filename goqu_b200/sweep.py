"""Parameter sweeps: goqu's sweep.RunSim and RunDensitySim (sweep/run.go:27-171).

Every sweep point binds the circuit's free parameters, runs it on a fresh
simulator with `shots` samples and reports its counts, in sweep order. Here
one gq_sweep_run call takes all points: the C++ side runs them on a pool of
workers, each owning a device state and stream, and builds every point's
counts on the device; a point that fails reports its own error (goqu's
PointResult.Err) without stopping the others.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from . import circuit as _ir
from . import encode as _encode
from .statevector import counts_from_pairs, uniforms as _uniforms

_D = ctypes.POINTER(ctypes.c_double)
_U64 = ctypes.POINTER(ctypes.c_uint64)


@dataclass
class PointResult:
    """One sweep point (sweep/run.go:17-22)."""
    Index: int
    Bindings: dict
    Counts: dict = field(default_factory=dict)
    Err: Exception | None = None


def _resolve(sw):
    return sw.Resolve() if hasattr(sw, "Resolve") else list(sw)


def _validate(c, points):
    free = _ir.FreeParameters(c)
    for b in points:
        missing = [p for p in free if p not in b]
        if missing:
            raise ValueError(f"sweep: circuit parameter {missing[0]!r} not covered by sweep")


def _run(c, shots, sw, rng, density, nm=None, precision=_abi.GQ_C128):
    points = _resolve(sw)
    _validate(c, points)
    n = c.NumQubits()
    rng = np.random.default_rng() if rng is None else rng
    streams, draws, errors = [], [], {}
    for i, b in enumerate(points):
        try:
            bound = _ir.Bind(c, b)
            streams.append(_encode.density_ops(bound, nm) if density else _encode.statevector_ops(bound))
        except Exception as exc:  # a point that cannot be bound reports its error
            errors[i] = exc
            streams.append(_encode.OpStream(n))
        draws.append(np.ascontiguousarray(_uniforms(shots, rng)))
    npts = len(points)
    arr = (_abi.gq_sweep_point * max(1, npts))()
    for i, (s, u) in enumerate(zip(streams, draws)):
        arr[i].ops = s.ptr()
        arr[i].n_ops = len(s)
        arr[i].uniforms = u.ctypes.data_as(_D)
    stride = max(1, min(shots, 1 << n))
    outc = np.zeros(max(1, npts * stride), dtype=np.uint64)
    cnt = np.zeros(max(1, npts * stride), dtype=np.uint64)
    nd = (ctypes.c_size_t * max(1, npts))()
    st = (ctypes.c_int32 * max(1, npts))()
    lib = _abi.lib()
    if density:
        p01 = np.full(n, -1.0)
        p10 = np.full(n, -1.0)
        if nm is not None:
            for q in range(n):
                re = nm.ReadoutFor(q)
                if re is not None:
                    p01[q], p10[q] = re.P01, re.P10
        _abi.check(lib.gq_sweep_run_density(n, p01.ctypes.data_as(_D), p10.ctypes.data_as(_D), arr, npts, shots,
                                            outc.ctypes.data_as(_U64), cnt.ctypes.data_as(_U64), nd, st))
    else:
        _abi.check(lib.gq_sweep_run(n, precision, arr, npts, shots, outc.ctypes.data_as(_U64),
                                    cnt.ctypes.data_as(_U64), nd, st))
    out = []
    for i, b in enumerate(points):
        if i in errors:
            out.append(PointResult(i, b, {}, errors[i]))
        elif st[i] != _abi.GQ_OK:
            out.append(PointResult(i, b, {}, _abi.GQError(st[i], f"sweep point {i} failed (status {st[i]})")))
        else:
            lo = i * stride
            out.append(PointResult(i, b, counts_from_pairs(outc[lo:lo + nd[i]], cnt[lo:lo + nd[i]], n)))
    return out


def RunSim(c, shots, sw, rng=None, precision=_abi.GQ_C128):
    """RunSim (sweep/run.go:27-97): statevector Run(bound, shots) per point."""
    return _run(c, shots, sw, rng, False, precision=precision)


def RunDensitySim(c, shots, sw, nm=None, rng=None):
    """RunDensitySim (sweep/run.go:100-171): density-matrix Run per point,
    with the noise model's channels and readout error."""
    return _run(c, shots, sw, rng, True, nm=nm)
