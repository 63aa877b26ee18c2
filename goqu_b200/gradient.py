"""Gradients of E(theta) = <psi(theta)|H|psi(theta)> (goqu algorithm/gradient).

CostFunc, ParameterShift and FiniteDifference follow
algorithm/gradient/gradient.go:25-86 and run each evaluation on the engine.
Adjoint is new: one forward pass, lambda = H psi, and a reverse sweep that
un-applies every gate to psi and lambda and accumulates 2 Re <lambda| dU/dtheta
U^dagger |psi> per parameter, on the device (gq_sv_adjoint_gradient).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _abi
from . import circuit as ir
from . import encode as _encode
from . import pauli as _pauli
from . import statevector

_D = ctypes.POINTER(ctypes.c_double)


def CostFunc(circuit, hamiltonian, param_names, precision=_abi.GQ_C128):
    """gradient.go:25-43: bind, evolve a fresh simulator, ExpectPauliSum."""
    sim = statevector.New(circuit.NumQubits(), precision)

    def f(x):
        bindings = {name: float(x[i]) for i, name in enumerate(param_names)}
        bound = ir.Bind(circuit, bindings)
        sim.Evolve(bound)
        return sim.ExpectPauliSum(hamiltonian)

    f.sim = sim
    return f


def ParameterShift(f):
    """gradient.go:49-66: (f(x + pi/2 e_i) - f(x - pi/2 e_i)) / 2."""

    def grad(x):
        x = np.asarray(x, dtype=np.float64)
        g = np.empty_like(x)
        for i in range(x.size):
            xp = x.copy()
            xm = x.copy()
            xp[i] += 0.5 * math.pi
            xm[i] -= 0.5 * math.pi
            g[i] = (f(xp) - f(xm)) / 2
        return g

    return grad


def FiniteDifference(f, h):
    """gradient.go:70-86: central differences."""

    def grad(x):
        x = np.asarray(x, dtype=np.float64)
        g = np.empty_like(x)
        for i in range(x.size):
            xp = x.copy()
            xm = x.copy()
            xp[i] += h
            xm[i] -= h
            g[i] = (f(xp) - f(xm)) / (2 * h)
        return g

    return grad


class AdjointEvaluator:
    """Energy and gradient of a symbolic circuit on one device handle."""

    def __init__(self, circuit, hamiltonian, param_names, precision=_abi.GQ_C128):
        self.circuit = circuit
        self.names = list(param_names)
        self.terms = _pauli.to_terms(hamiltonian)
        self.sim = statevector.New(circuit.NumQubits(), precision)

    def __call__(self, x):
        x = np.asarray(x, dtype=np.float64)
        bindings = {name: float(x[i]) for i, name in enumerate(self.names)}
        stream = _encode.statevector_ops(self.circuit, bindings, self.names)
        grad = np.empty(len(self.names), dtype=np.float64)
        energy = ctypes.c_double()
        _abi.check(_abi.lib().gq_sv_adjoint_gradient(
            self.sim.handle, stream.ptr(), len(stream),
            ctypes.cast(self.terms, ctypes.POINTER(_abi.gq_pauli_term)), len(self.terms),
            len(self.names), grad.ctypes.data_as(_D), ctypes.byref(energy)))
        return energy.value, grad


def Adjoint(circuit, hamiltonian, param_names, precision=_abi.GQ_C128):
    """An optim.GradientFunc computing dE/dtheta with the adjoint method."""
    ev = AdjointEvaluator(circuit, hamiltonian, param_names, precision)

    def grad(x):
        return ev(x)[1]

    grad.evaluator = ev
    return grad
