"""MaxCut QAOA: goqu's algorithm/qaoa circuits evaluated in batches.

qaoa.Run (qaoa.go:61-126) builds H^n followed by p layers of RZZ(gamma_k)
per edge of MaxCutHamiltonian (maxcut.go:13-35) and RX(2 beta_k) per qubit,
and minimises <H>. MaxCutBatch evaluates many such circuits at once through
gq_qaoa_maxcut_batch: energies and adjoint gradients in FreeParameters order
[gamma_0, beta_0, gamma_1, ...]. from_evaluation reads the graph and angles
back from a (circuit, names, hamiltonian, x) evaluation of
workloads.qaoa_batch, so both batch paths can be fed the same circuits.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from . import pauli as _pauli

_D = ctypes.POINTER(ctypes.c_double)


def edges_of(hamiltonian):
    """The (i, j) pairs of the Z_i Z_j terms of a MaxCut Hamiltonian, in term order."""
    n = hamiltonian.NumQubits()
    out = []
    for t in hamiltonian.Terms():
        zq = [q for q in range(n) if t.Op(q) == _pauli.Z]
        if len(zq) == 2 and t.Coeff().real != 0:
            out.append((zq[0], zq[1]))
    return out


def from_evaluation(ev):
    """(n, edges, gammas, betas) of a workloads.qaoa_batch evaluation."""
    c, names, h, x = ev
    x = np.asarray(x, dtype=np.float64)
    return c.NumQubits(), edges_of(h), x[0::2].copy(), x[1::2].copy()


class Encoded:
    """Items packed for gq_qaoa_maxcut_batch (the arrays the records point to
    are kept alive here); reuse it while the circuits stay the same."""

    def __init__(self, items):
        self.keep = []
        self.arr = (_abi.gq_qaoa_item * max(1, len(items)))()
        self.n = len(items)
        self.sizes = []
        for i, (n, edges, gammas, betas) in enumerate(items):
            e = np.ascontiguousarray(np.asarray(edges, dtype=np.int32).reshape(-1))
            g = np.ascontiguousarray(gammas, dtype=np.float64)
            b = np.ascontiguousarray(betas, dtype=np.float64)
            if g.size != b.size:
                raise ValueError("qaoa: gammas and betas differ in length")
            self.keep += [e, g, b]
            self.arr[i].num_qubits, self.arr[i].p = int(n), int(g.size)
            self.arr[i].edges = e.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            self.arr[i].n_edges = e.size // 2
            self.arr[i].gammas, self.arr[i].betas = g.ctypes.data_as(_D), b.ctypes.data_as(_D)
            self.sizes.append(2 * g.size)
        self.total = int(sum(self.sizes))


class MaxCutBatch:
    """Energies (and gradients) of MaxCut QAOA circuits on one device."""

    def __init__(self, precision=_abi.GQ_C64):
        self.precision = precision

    @staticmethod
    def encode(items):
        return Encoded(items)

    def run_encoded(self, enc, gradients=True):
        energies = np.empty(max(1, enc.n), dtype=np.float64)
        grads = np.empty(max(1, enc.total), dtype=np.float64)
        _abi.check(_abi.lib().gq_qaoa_maxcut_batch(self.precision, enc.arr, enc.n, 1 if gradients else 0,
                                                  energies.ctypes.data_as(_D), grads.ctypes.data_as(_D)))
        if not gradients:
            return energies[:enc.n], None
        out, off = [], 0
        for k in enc.sizes:
            out.append(grads[off:off + k].copy())
            off += k
        return energies[:enc.n], out

    def Run(self, items, gradients=True):
        """items: (n, edges, gammas, betas) each; returns (energies, list of gradient arrays or None)."""
        return self.run_encoded(Encoded(items), gradients)
