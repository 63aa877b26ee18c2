"""densitymatrix.Sim on the B200 engine: the API of goqu's sim/densitymatrix
(New, WithNoise, Run, Evolve, Apply, Reset, DensityMatrix, Purity, Fidelity,
ExpectPauliString/Sum, ExpectationValue, DiagonalProbs, ApplyReadoutError;
sim/densitymatrix/sim.go:32-313, measure.go:11-91).

rho is held on the device as a 2n-qubit vector; gates act as U on the row
qubits and conj(U) on the column qubits, Kraus channels as the superoperator
sum_k E_k (x) conj(E_k), folded into the gate that precedes them.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from . import encode as _encode
from . import pauli as _pauli
from .statevector import _round14, counts_from_pairs, sample_counts_call, uniforms

_D = ctypes.POINTER(ctypes.c_double)
_U64 = ctypes.POINTER(ctypes.c_uint64)


class Sim:
    def __init__(self, num_qubits):
        if num_qubits < 1 or num_qubits > 15:
            raise ValueError(f"densitymatrix: numQubits {num_qubits} out of range [1, 15]")
        self._n = num_qubits
        self._dim = 1 << num_qubits
        self._noise = None
        h = ctypes.c_void_p()
        _abi.check(_abi.lib().gq_dm_create(num_qubits, ctypes.byref(h)))
        self._h = h

    def WithNoise(self, nm):
        self._noise = nm
        return self

    def Close(self):
        if self._h:
            _abi.lib().gq_dm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.Close()
        except Exception:
            pass

    def NumQubits(self):
        return self._n

    def _check(self, c):
        if c.NumQubits() != self._n:
            raise ValueError(f"circuit has {c.NumQubits()} qubits, simulator has {self._n}")

    def Reset(self):
        _abi.check(_abi.lib().gq_dm_reset(self._h))

    def Apply(self, c):
        self._check(c)
        s = _encode.density_ops(c, self._noise)
        _abi.check(_abi.lib().gq_dm_apply(self._h, s.ptr(), len(s)))

    def Evolve(self, c):
        self._check(c)
        s = _encode.density_ops(c, self._noise)
        _abi.check(_abi.lib().gq_dm_evolve(self._h, s.ptr(), len(s)))

    def Run(self, c, shots, rng=None):
        """Evolve and sample the readout-mixed diagonal (sim.go:48-66); dynamic
        circuits run shot groups (RunDynamic, dynamic.go:13-51)."""
        if c.IsDynamic():
            from . import dynamic
            return dynamic.run_dynamic_dm(self, c, shots, rng)
        self.Evolve(c)
        return counts_from_pairs(*self.SampleCounts(uniforms(shots, rng)), self._n)

    def _readout_arrays(self):
        p01 = np.full(self._n, -1.0)
        p10 = np.full(self._n, -1.0)
        if self._noise is not None:
            for q in range(self._n):
                re = self._noise.ReadoutFor(q)
                if re is not None:
                    p01[q], p10[q] = re.P01, re.P10
        return p01, p10

    def SampleCounts(self, u):
        """Distinct outcomes of the readout-mixed sampling and their counts,
        histogrammed on the device."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        p01, p10 = self._readout_arrays()
        return sample_counts_call(_abi.lib().gq_dm_sample_counts, u.size, self._h, p01.ctypes.data_as(_D),
                                  p10.ctypes.data_as(_D), u.ctypes.data_as(_D), u.size)

    def Sample(self, u):
        """Inverse-CDF sampling of the readout-mixed diagonal (sim.go:45-60)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        p01, p10 = self._readout_arrays()
        out = np.empty(u.size, dtype=np.uint64)
        _abi.check(_abi.lib().gq_dm_sample(self._h, p01.ctypes.data_as(_D), p10.ctypes.data_as(_D),
                                           u.ctypes.data_as(_D), u.size, out.ctypes.data_as(_U64)))
        return out

    def DensityMatrix(self):
        out = np.empty(self._dim * self._dim, dtype=np.complex128)
        _abi.check(_abi.lib().gq_dm_get(self._h, out.view(np.float64).ctypes.data_as(_D), out.nbytes))
        return out

    def DiagonalProbs(self):
        out = np.empty(self._dim, dtype=np.float64)
        _abi.check(_abi.lib().gq_dm_diagonal_probs(self._h, out.ctypes.data_as(_D), out.size))
        return out

    def ApplyReadoutError(self, probs):
        """measure.go:29-71, on the host array the caller passes."""
        if self._noise is None:
            return probs
        result = np.array(probs, dtype=np.float64)
        for q in range(self._n):
            re = self._noise.ReadoutFor(q)
            if re is None:
                continue
            m = 1 << q
            idx = np.arange(self._dim)
            stay = np.where(idx & m, 1 - re.P10, 1 - re.P01)
            flip = np.where(idx & m, re.P10, re.P01)
            result = result * stay + result[idx ^ m] * flip[idx ^ m]
        return result

    def Purity(self):
        v = ctypes.c_double()
        _abi.check(_abi.lib().gq_dm_purity(self._h, ctypes.byref(v)))
        return v.value

    def Fidelity(self, psi):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        if psi.size != self._dim:
            raise ValueError(f"densitymatrix: pure state length {psi.size}, expected {self._dim}")
        v = ctypes.c_double()
        _abi.check(_abi.lib().gq_dm_fidelity(self._h, psi.view(np.float64).ctypes.data_as(_D), psi.size,
                                             ctypes.byref(v)))
        return v.value

    def Trace(self):
        re, im = ctypes.c_double(), ctypes.c_double()
        _abi.check(_abi.lib().gq_dm_trace(self._h, ctypes.byref(re), ctypes.byref(im)))
        return complex(re.value, im.value)

    def _expect(self, ps):
        arr = _pauli.to_terms(ps)
        re, im = ctypes.c_double(), ctypes.c_double()
        _abi.check(_abi.lib().gq_dm_expect_pauli_sum(self._h, ctypes.cast(arr, ctypes.POINTER(_abi.gq_pauli_term)),
                                                     len(arr), ctypes.byref(re), ctypes.byref(im)))
        return complex(re.value, im.value)

    def ExpectPauliString(self, ps):
        if ps.NumQubits() != self._n:
            raise ValueError(f"densitymatrix: PauliString has {ps.NumQubits()} qubits, simulator has {self._n}")
        return self._expect(ps).real

    def ExpectPauliSum(self, ps):
        if ps.NumQubits() != self._n:
            raise ValueError(f"densitymatrix: PauliSum has {ps.NumQubits()} qubits, simulator has {self._n}")
        return self._expect(ps).real

    def ExpectationValue(self, qubits):
        """sum_i (-1)^parity rho_ii rounded to 1e-14 (measure.go:76-91)."""
        ps = _pauli.ZOn(list(qubits), self._n) if qubits else _pauli.NewPauliString(1, None, self._n)
        return _round14(self._expect(ps).real)

    def set_option(self, key, value):
        _abi.check(_abi.lib().gq_dm_set_option(self._h, key, int(value)))

    def stats(self):
        s = _abi.gq_stats()
        _abi.check(_abi.lib().gq_dm_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _abi.gq_stats._fields_}


def New(num_qubits):
    return Sim(num_qubits)
