"""Classical optimisers for variational loops: goqu's algorithm/optim.

Options and Result follow optim.go:21-69; Adam restates adam.go:9-140 (the
update, the defaults and the convergence tests in the same order). The
variational drivers (vqe.Run) hand an Adam run with an adjoint gradient to
the library as one call, gq_sv_minimize_adam, which keeps the loop on the
device side; this Python Adam serves every other objective and is the
reference the library loop is tested against.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Options:
    MaxIter: int = 0      # default 1000
    FunTol: float = 0.0   # default 1e-8
    XTol: float = 0.0     # default 1e-8
    GradTol: float = 0.0  # 0: disabled
    Callback: object = None

    def max_iter(self):
        return self.MaxIter if self.MaxIter > 0 else 1000

    def fun_tol(self):
        return self.FunTol if self.FunTol > 0 else 1e-8

    def grad_tol(self):
        return self.GradTol


@dataclass
class Result:
    X: np.ndarray = field(default_factory=lambda: np.empty(0))
    Fun: float = 0.0
    Iterations: int = 0
    FuncEvals: int = 0
    GradEvals: int = 0
    Converged: bool = False
    Message: str = ""


@dataclass
class Adam:
    """Adam (adam.go:9-49); zero fields take goqu's defaults."""
    LR: float = 0.0
    Beta1: float = 0.0
    Beta2: float = 0.0
    Epsilon: float = 0.0

    def Name(self):
        return "Adam"

    def params(self):
        return (self.LR if self.LR > 0 else 0.001, self.Beta1 if self.Beta1 > 0 else 0.9,
                self.Beta2 if self.Beta2 > 0 else 0.999, self.Epsilon if self.Epsilon > 0 else 1e-8)

    def Minimize(self, f, x0, grad, opts=None):
        """adam.go:51-140."""
        opts = opts or Options()
        x = np.array(x0, dtype=np.float64)
        n = x.size
        if n == 0:
            raise ValueError("adam: x0 must be non-empty")
        if grad is None:
            raise ValueError("adam: gradient function required")
        lr, b1, b2, eps = self.params()
        m = np.zeros(n)
        v = np.zeros(n)
        fx = f(x)
        f_evals, g_evals = 1, 0
        prev = fx
        converged = False
        it = 0
        while it < opts.max_iter():
            g = np.asarray(grad(x), dtype=np.float64)
            g_evals += 1
            if opts.grad_tol() > 0 and math.sqrt(float(np.sum(g * g))) < opts.grad_tol():
                converged = True
                break
            t = float(it + 1)
            for j in range(n):  # element by element, in goqu's operation order
                m[j] = b1 * m[j] + (1 - b1) * g[j]
                v[j] = b2 * v[j] + (1 - b2) * g[j] * g[j]
                mh = m[j] / (1 - math.pow(b1, t))
                vh = v[j] / (1 - math.pow(b2, t))
                x[j] -= lr * mh / (math.sqrt(vh) + eps)
            fx = f(x)
            f_evals += 1
            if abs(fx - prev) < opts.fun_tol():
                converged = True
                it += 1
                break
            prev = fx
            if opts.Callback is not None and opts.Callback(it, x.copy(), fx) is not None:
                return Result(x.copy(), fx, it + 1, f_evals, g_evals, False, "stopped by callback")
            it += 1
        return Result(x.copy(), fx, it, f_evals, g_evals, converged,
                      "converged" if converged else "maximum iterations reached")
