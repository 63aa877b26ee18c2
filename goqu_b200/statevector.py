"""statevector.Sim on the B200 engine: the API of goqu's sim/statevector
(New, Run, Evolve, Apply, Reset, StateVector, ExpectPauliString/Sum,
ExpectationValue, Close; sim/statevector/sim.go:27-382), executed by
libgqb200.so through its C ABI.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _abi
from . import encode as _encode
from . import pauli as _pauli

_D = ctypes.POINTER(ctypes.c_double)
_U64 = ctypes.POINTER(ctypes.c_uint64)


def uniforms(shots, rng=None):
    """Uniforms as goqu draws them: rand.Float64() = (53 random bits) / 2^53."""
    rng = np.random.default_rng() if rng is None else rng
    return rng.integers(0, 1 << 53, size=shots, dtype=np.int64).astype(np.float64) / float(1 << 53)


def format_bitstring(idx, n):
    """formatBitstring (sim/statevector/sim.go:306-316): qubit 0 rightmost."""
    return format(int(idx), "b").zfill(n)[-n:] if n else ""


def counts_from_indices(idx, n):
    vals, cnt = np.unique(np.asarray(idx, dtype=np.uint64), return_counts=True)
    return counts_from_pairs(vals, cnt, n)


def counts_from_pairs(outcomes, counts, n):
    """goqu's map[bitstring]int from (outcome, count) pairs."""
    return {format_bitstring(v, n): int(c) for v, c in zip(outcomes, counts)}


def sample_counts_call(fn, shots, *head):
    """Calls a *_sample_counts entry point: (distinct outcomes, counts)."""
    m = max(1, shots)
    outc = np.empty(m, dtype=np.uint64)
    cnt = np.empty(m, dtype=np.uint64)
    nd = ctypes.c_size_t()
    _abi.check(fn(*head, outc.ctypes.data_as(_U64), cnt.ctypes.data_as(_U64), ctypes.byref(nd)))
    return outc[:nd.value].copy(), cnt[:nd.value].copy()


class Sim:
    """A statevector simulator backed by one device handle."""

    def __init__(self, num_qubits, precision=_abi.GQ_C128):
        if num_qubits < 1 or num_qubits > 34:
            raise ValueError(f"statevector: numQubits {num_qubits} out of range [1, 34]")
        self._n = num_qubits
        self._prec = precision
        h = ctypes.c_void_p()
        _abi.check(_abi.lib().gq_sv_create(num_qubits, precision, ctypes.byref(h)))
        self._h = h

    # -- lifecycle ---------------------------------------------------------
    def Close(self):
        if self._h:
            _abi.lib().gq_sv_destroy(self._h)
            self._h = None
        return None

    def __del__(self):
        try:
            self.Close()
        except Exception:
            pass

    def NumQubits(self):
        return self._n

    @property
    def handle(self):
        return self._h

    # -- evolution ---------------------------------------------------------
    def _check_circuit(self, c):
        if c.NumQubits() != self._n:
            raise ValueError(f"circuit has {c.NumQubits()} qubits, simulator has {self._n}")

    def Reset(self):
        _abi.check(_abi.lib().gq_sv_reset(self._h))

    def Apply(self, c):
        self._check_circuit(c)
        self.apply_ops(_encode.statevector_ops(c))

    def Evolve(self, c):
        self._check_circuit(c)
        self.evolve_ops(_encode.statevector_ops(c))

    def apply_ops(self, stream):
        _abi.check(_abi.lib().gq_sv_apply(self._h, stream.ptr(), len(stream)))

    def evolve_ops(self, stream):
        _abi.check(_abi.lib().gq_sv_evolve(self._h, stream.ptr(), len(stream)))

    def Run(self, c, shots, rng=None):
        """Evolve then sample every qubit `shots` times (sim.go:40-58)."""
        if c.IsDynamic():
            from . import dynamic
            return dynamic.run_dynamic(self, c, shots, rng)
        self.Evolve(c)
        return counts_from_pairs(*self.SampleCounts(uniforms(shots, rng)), self._n)

    # -- readout -----------------------------------------------------------
    def StateVector(self):
        n = 1 << self._n
        if self._prec == _abi.GQ_C64:
            out = np.empty(n, dtype=np.complex64)
        else:
            out = np.empty(n, dtype=np.complex128)
        _abi.check(_abi.lib().gq_sv_get_state(self._h, out.ctypes.data_as(ctypes.c_void_p), out.nbytes))
        return out.astype(np.complex128, copy=False)

    def SetStateVector(self, amps):
        dt = np.complex64 if self._prec == _abi.GQ_C64 else np.complex128
        a = np.ascontiguousarray(np.asarray(amps, dtype=dt))
        _abi.check(_abi.lib().gq_sv_set_state(self._h, a.ctypes.data_as(ctypes.c_void_p), a.nbytes))

    def Probabilities(self):
        out = np.empty(1 << self._n, dtype=np.float64)
        _abi.check(_abi.lib().gq_sv_probabilities(self._h, out.ctypes.data_as(_D), out.size))
        return out

    def SampleCounts(self, u):
        """Distinct sampled outcomes and their counts, histogrammed on the device."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        return sample_counts_call(_abi.lib().gq_sv_sample_counts, u.size, self._h, u.ctypes.data_as(_D), u.size)

    def Sample(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty(u.size, dtype=np.uint64)
        _abi.check(_abi.lib().gq_sv_sample(self._h, u.ctypes.data_as(_D), u.size, out.ctypes.data_as(_U64)))
        return out

    def expect_terms(self, terms):
        re, im = ctypes.c_double(), ctypes.c_double()
        arr = terms
        _abi.check(_abi.lib().gq_sv_expect_pauli_sum(self._h, ctypes.cast(arr, ctypes.POINTER(_abi.gq_pauli_term)),
                                                     len(arr), ctypes.byref(re), ctypes.byref(im)))
        return complex(re.value, im.value)

    def ExpectPauliString(self, ps):
        if ps.NumQubits() != self._n:
            raise ValueError(f"statevector: PauliString has {ps.NumQubits()} qubits, simulator has {self._n}")
        return self.expect_terms(_pauli.to_terms(ps)).real

    def ExpectPauliSum(self, ps):
        if ps.NumQubits() != self._n:
            raise ValueError(f"statevector: PauliSum has {ps.NumQubits()} qubits, simulator has {self._n}")
        return self.expect_terms(_pauli.to_terms(ps)).real

    def ExpectationValue(self, qubits):
        """<Z...Z> on `qubits`, rounded to 1e-14 (sim.go:368-382)."""
        mask = 0
        for q in qubits:
            mask |= 1 << q
        v = ctypes.c_double()
        _abi.check(_abi.lib().gq_sv_expect_z_mask(self._h, mask, ctypes.byref(v)))
        return _round14(v.value)

    # -- engine ------------------------------------------------------------
    def set_option(self, key, value):
        _abi.check(_abi.lib().gq_sv_set_option(self._h, key, int(value)))

    def stats(self):
        s = _abi.gq_stats()
        _abi.check(_abi.lib().gq_sv_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _abi.gq_stats._fields_}


def _round14(ev):
    # math.Round(ev*1e14)/1e14: round half away from zero
    x = ev * 1e14
    a = abs(x)
    r = math.floor(a)
    if a - r >= 0.5:
        r += 1.0
    return math.copysign(r, x) / 1e14


def New(num_qubits, precision=_abi.GQ_C128):
    return Sim(num_qubits, precision)
