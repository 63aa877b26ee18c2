"""Noise channels and models (goqu sim/noise).

Kraus sets of channel.go:27-298, the lookup order of NoiseModel.Lookup
(noise.go:62-74: gate+qubits, then gate name, then qubit count) and readout
errors (readout.go).
"""
from __future__ import annotations

import math

import numpy as np


class Channel:
    def __init__(self, name, nq, kraus):
        self._name = name
        self._nq = nq
        self._kraus = [np.asarray(k, dtype=np.complex128).reshape(-1) for k in kraus]

    def Name(self):
        return self._name

    def Qubits(self):
        return self._nq

    def Kraus(self):
        return list(self._kraus)


def _check(name, v, what="p"):
    if v < 0 or v > 1:
        raise ValueError(f"noise.{name}: {what}={v:f} out of range [0,1]")


def Depolarizing1Q(p):
    _check("Depolarizing1Q", p)
    s0, sp = complex(math.sqrt(1 - p), 0), complex(math.sqrt(p / 3), 0)
    return Channel(f"depolarizing1q({p:.4f})", 1, [
        [s0, 0, 0, s0], [0, sp, sp, 0], [0, -sp * 1j, sp * 1j, 0], [sp, 0, 0, -sp]])


def _tensor2x2(a, b):
    # tensorProduct2x2 (channel.go:89-104)
    r = [0j] * 16
    for i in range(2):
        for j in range(2):
            for k in range(2):
                for l in range(2):
                    r[(i * 2 + k) * 4 + (j * 2 + l)] = a[i * 2 + j] * b[k * 2 + l]
    return r


def Depolarizing2Q(p):
    _check("Depolarizing2Q", p)
    pauli1 = [[1, 0, 0, 1], [0, 1, 1, 0], [0, -1j, 1j, 0], [1, 0, 0, -1]]
    s0, sp = math.sqrt(1 - p), math.sqrt(p / 15)
    kraus = []
    for i in range(4):
        for j in range(4):
            k = _tensor2x2(pauli1[i], pauli1[j])
            scale = complex(s0, 0) if (i == 0 and j == 0) else complex(sp, 0)
            kraus.append([x * scale for x in k])
    return Channel(f"depolarizing2q({p:.4f})", 2, kraus)


def AmplitudeDamping(gamma):
    _check("AmplitudeDamping", gamma, "gamma")
    sg, s1 = complex(math.sqrt(gamma), 0), complex(math.sqrt(1 - gamma), 0)
    return Channel(f"amplitude_damping({gamma:.4f})", 1, [[1, 0, 0, s1], [0, sg, 0, 0]])


def PhaseDamping(lam):
    _check("PhaseDamping", lam, "lambda")
    sl, s1 = complex(math.sqrt(lam), 0), complex(math.sqrt(1 - lam), 0)
    return Channel(f"phase_damping({lam:.4f})", 1, [[1, 0, 0, s1], [0, 0, 0, sl]])


def BitFlip(p):
    _check("BitFlip", p)
    s0, sp = complex(math.sqrt(1 - p), 0), complex(math.sqrt(p), 0)
    return Channel(f"bit_flip({p:.4f})", 1, [[s0, 0, 0, s0], [0, sp, sp, 0]])


def PhaseFlip(p):
    _check("PhaseFlip", p)
    s0, sp = complex(math.sqrt(1 - p), 0), complex(math.sqrt(p), 0)
    return Channel(f"phase_flip({p:.4f})", 1, [[s0, 0, 0, s0], [sp, 0, 0, -sp]])


def GeneralizedAmplitudeDamping(p, gamma):
    _check("GeneralizedAmplitudeDamping", p)
    _check("GeneralizedAmplitudeDamping", gamma, "gamma")
    sp, s1p = complex(math.sqrt(p), 0), complex(math.sqrt(1 - p), 0)
    sg, s1g = complex(math.sqrt(gamma), 0), complex(math.sqrt(1 - gamma), 0)
    return Channel(f"generalized_amplitude_damping({p:.4f},{gamma:.4f})", 1, [
        [sp, 0, 0, sp * s1g], [0, sp * sg, 0, 0], [s1p * s1g, 0, 0, s1p], [0, 0, s1p * sg, 0]])


def ThermalRelaxation(t1, t2, time):
    if t2 > 2 * t1:
        raise ValueError(f"noise.ThermalRelaxation: t2={t2:f} > 2*t1={2 * t1:f} is unphysical")
    if t1 <= 0 or t2 <= 0 or time < 0:
        raise ValueError("noise.ThermalRelaxation: t1, t2 must be positive, time must be non-negative")
    gamma = 1 - math.exp(-time / t1)
    e_lambda = math.exp(-time / t2)
    lam = 0.0
    if gamma < 1:
        ideal = math.sqrt(1 - gamma)
        if e_lambda < ideal:
            ratio = e_lambda / ideal
            lam = 1 - ratio * ratio
    sg, s1g = math.sqrt(gamma), math.sqrt(1 - gamma)
    sl, s1l = math.sqrt(lam), math.sqrt(1 - lam)
    kraus = [[1, 0, 0, complex(s1l * s1g, 0)], [0, complex(sg, 0), 0, 0]]
    if lam > 1e-15:
        kraus.append([0, 0, 0, complex(sl * s1g, 0)])
    return Channel(f"thermal_relaxation({t1:.4g},{t2:.4g},{time:.4g})", 1, kraus)


def Custom(name, nq, kraus, tol=1e-10):
    """A user Kraus set; must be trace preserving (custom.go:13-78)."""
    dim = 1 << nq
    acc = np.zeros((dim, dim), dtype=np.complex128)
    for k in kraus:
        e = np.asarray(k, dtype=np.complex128).reshape(dim, dim)
        acc += e.conj().T @ e
    if not np.allclose(acc, np.eye(dim), atol=tol):
        raise ValueError("noise.Custom: Kraus operators are not trace preserving")
    return Channel(name, nq, kraus)


class ReadoutError:
    def __init__(self, p01, p10):
        if not (0 <= p01 <= 1 and 0 <= p10 <= 1):
            raise ValueError("noise.NewReadoutError: probabilities must be in [0,1]")
        self.P01 = p01
        self.P10 = p10

    def Apply(self, p0, p1):
        return (1 - self.P01) * p0 + self.P10 * p1, self.P01 * p0 + (1 - self.P10) * p1


def NewReadoutError(p01, p10):
    return ReadoutError(p01, p10)


class NoiseModel:
    def __init__(self):
        self._by_gate_qubits = {}
        self._by_gate = {}
        self._by_qubits = {}
        self._readout = {}

    def AddGateError(self, name, ch):
        self._by_gate[name] = ch

    def AddGateQubitError(self, name, qubits, ch):
        self._by_gate_qubits[_key(name, qubits)] = ch

    def AddDefaultError(self, n_qubits, ch):
        self._by_qubits[n_qubits] = ch

    def AddReadoutError(self, qubit, re):
        self._readout[qubit] = re

    def Lookup(self, name, qubits):
        ch = self._by_gate_qubits.get(_key(name, qubits))
        if ch is not None:
            return ch
        ch = self._by_gate.get(name)
        if ch is not None:
            return ch
        return self._by_qubits.get(len(qubits))

    def ReadoutFor(self, qubit):
        return self._readout.get(qubit)


def _key(name, qubits):
    return name + ":" + ",".join(str(q) for q in qubits)


def New():
    return NoiseModel()
