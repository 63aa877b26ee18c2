"""Variational quantum eigensolver: goqu's algorithm/vqe (vqe.go:17-89).

Run minimises E(theta) = <psi(theta)|H|psi(theta)> over the ansatz's free
parameters. With an Adam optimiser and the adjoint gradient (the default
here), the whole loop is one library call (gq_sv_minimize_adam): the
library rebinds the circuit's symbolic gates from theta itself, and one
forward + reverse sweep per iteration gives the energy after the update and
the gradient for the next step, with the state kept on the device. Other
optimisers or gradients run the loop in Python over the same engine.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from . import circuit as _ir
from . import encode as _encode
from . import gradient as _gradient
from . import optim as _optim
from . import pauli as _pauli
from . import statevector as _statevector

_D = ctypes.POINTER(ctypes.c_double)


@dataclass
class Config:
    Hamiltonian: object
    Ansatz: object                 # a circuit, or an object with Circuit()
    Optimizer: object = None       # default optim.Adam()
    Gradient: object = "adjoint"   # "adjoint", an optim GradientFunc, or None
    InitialParams: object = None
    Options: object = None         # optim.Options
    Precision: int = _abi.GQ_C128


@dataclass
class Result:
    Energy: float = 0.0
    OptimalParams: np.ndarray = field(default_factory=lambda: np.empty(0))
    NumIters: int = 0
    NumEvals: int = 0
    Converged: bool = False
    History: list = field(default_factory=list)


def minimize_adam_on_device(circuit, hamiltonian, names, x0, adam=None, opts=None, precision=_abi.GQ_C128, sim=None):
    """Adam with adjoint gradients as one library call; returns (optim.Result,
    history of energies)."""
    adam = adam or _optim.Adam()
    opts = opts or _optim.Options()
    tmpl = _encode.param_template(circuit, names, x0)
    terms = _pauli.to_terms(hamiltonian)
    own = sim is None
    sim = sim or _statevector.New(circuit.NumQubits(), precision)
    lr, b1, b2, eps = adam.params()
    o = _abi.gq_adam_options(lr, b1, b2, eps, opts.max_iter(), 0, opts.fun_tol(), opts.grad_tol())
    x = np.array(x0, dtype=np.float64)
    hist = np.empty(opts.max_iter() + 1)
    res = _abi.gq_optim_result()
    try:
        _abi.check(_abi.lib().gq_sv_minimize_adam(
            sim.handle, tmpl.ops.ptr(), len(tmpl.ops), tmpl.pgate_ptr(), len(tmpl.pgates),
            ctypes.cast(terms, ctypes.POINTER(_abi.gq_pauli_term)), len(terms), len(names),
            x.ctypes.data_as(_D), ctypes.byref(o), ctypes.byref(res), hist.ctypes.data_as(_D), hist.size))
    finally:
        if own:
            sim.Close()
    r = _optim.Result(x, res.fun, res.iterations, res.func_evals, res.grad_evals, bool(res.converged),
                      "converged" if res.converged else "maximum iterations reached")
    return r, hist[:res.func_evals].tolist()


def Run(cfg):
    """vqe.go:50-89."""
    circ = cfg.Ansatz.Circuit() if hasattr(cfg.Ansatz, "Circuit") else cfg.Ansatz
    names = _ir.FreeParameters(circ)
    if not names:
        raise ValueError("vqe: ansatz has no free parameters")
    x0 = np.zeros(len(names)) if cfg.InitialParams is None else np.asarray(cfg.InitialParams, dtype=np.float64)
    opt = cfg.Optimizer or _optim.Adam()
    if isinstance(opt, _optim.Adam) and cfg.Gradient == "adjoint":
        res, hist = minimize_adam_on_device(circ, cfg.Hamiltonian, names, x0, opt, cfg.Options, cfg.Precision)
    else:
        cost = _gradient.CostFunc(circ, cfg.Hamiltonian, names)
        hist = []

        def f(x):
            v = cost(x)
            hist.append(v)
            return v

        grad = cfg.Gradient
        if grad == "adjoint":
            grad = _gradient.Adjoint(circ, cfg.Hamiltonian, names, cfg.Precision)
        res = opt.Minimize(f, x0, grad, cfg.Options)
    return Result(res.Fun, res.X, res.Iterations, res.FuncEvals, res.Converged, hist)
