"""Batches of parameterised circuits evaluated together on the device.

goqu evaluates sweeps and variational costs one fresh simulator per point on
a goroutine pool (sweep/run.go:27-97, algorithm/qaoa/qaoa.go:100-126). Here a
whole batch -- circuits of different sizes and depths, each with its own
Pauli sum and parameter values -- is one gq_batch_run: energies
Re <psi|H|psi> and, optionally, adjoint gradients for every item.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from . import encode as _encode
from . import pauli as _pauli

_D = ctypes.POINTER(ctypes.c_double)


class Batch:
    def __init__(self, precision=_abi.GQ_C64):
        h = ctypes.c_void_p()
        _abi.check(_abi.lib().gq_batch_create(precision, ctypes.byref(h)))
        self._h = h
        self.precision = precision

    def Close(self):
        if self._h:
            _abi.lib().gq_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.Close()
        except Exception:
            pass

    def set_option(self, key, value):
        _abi.check(_abi.lib().gq_batch_set_option(self._h, key, int(value)))

    def stats(self):
        s = _abi.gq_stats()
        _abi.check(_abi.lib().gq_batch_stats(self._h, ctypes.byref(s)))
        return {f: getattr(s, f) for f, _ in _abi.gq_stats._fields_}

    @staticmethod
    def encode(evaluations):
        """(circuit, param_names, hamiltonian, x) -> (op streams, term arrays)."""
        streams, terms = [], []
        for c, names, h, x in evaluations:
            bindings = {nm: float(x[i]) for i, nm in enumerate(names)}
            streams.append(_encode.statevector_ops(c, bindings, names))
            terms.append(_pauli.to_terms(h))
        return streams, terms

    def run_encoded(self, streams, terms, n_params, gradients=True):
        n = len(streams)
        items = (_abi.gq_batch_item * n)()
        for i, (s, t) in enumerate(zip(streams, terms)):
            items[i].num_qubits = s.num_qubits
            items[i].ops = s.ptr()
            items[i].n_ops = len(s)
            items[i].terms = ctypes.cast(t, ctypes.POINTER(_abi.gq_pauli_term))
            items[i].n_terms = len(t)
            items[i].n_params = n_params[i]
        energies = np.empty(n, dtype=np.float64)
        grads = np.empty(max(1, int(sum(n_params))), dtype=np.float64)
        _abi.check(_abi.lib().gq_batch_run(self._h, items, n, 1 if gradients else 0, energies.ctypes.data_as(_D),
                                           grads.ctypes.data_as(_D)))
        out, off = [], 0
        for k in n_params:
            out.append(grads[off:off + k].copy())
            off += k
        return energies, (out if gradients else None)

    def Run(self, evaluations, gradients=True):
        streams, terms = self.encode(evaluations)
        return self.run_encoded(streams, terms, [len(e[1]) for e in evaluations], gradients)


def circuit_work(evaluation, gradients=True):
    """Device work of one batch item, in amplitude-ops: the state size 2^n
    times its gate count, the reverse sweep (two states, every gate again)
    counting twice more when gradients are taken. Depth matters as much as
    size: a QAOA circuit of depth 4 costs about four times one of depth 1."""
    c = evaluation[0]
    gates = sum(1 for op in c.Ops() if op.Gate is not None)
    return (1 << c.NumQubits()) * max(1, gates) * (3 if gradients else 1)


def split_by_work(evaluations, world, gradients=True):
    """Indices of each rank's share of a batch, balanced by device work
    (circuit_work): the largest items first, each to the rank with the least
    work so far."""
    work = [circuit_work(e, gradients) for e in evaluations]
    load = [0] * world
    shares = [[] for _ in range(world)]
    for i in sorted(range(len(evaluations)), key=lambda i: -work[i]):
        r = min(range(world), key=lambda k: (load[k], k))
        shares[r].append(i)
        load[r] += work[i]
    return [sorted(x) for x in shares]


def run_sharded(evaluations, rank, world, precision=_abi.GQ_C64, gradients=True, runner=None):
    """A batch split across ranks (one GPU each): every rank runs its share on
    its own device and the energies and gradients are all-gathered; returns
    the whole batch's results in input order on every rank. The gather of
    scalars is the only collective (torch.distributed, any backend)."""
    share = split_by_work(evaluations, world, gradients)[rank]
    mine = [evaluations[i] for i in share]
    if runner is None:
        b = Batch(precision)
        e, g = b.Run(mine, gradients) if mine else (np.empty(0), [])
        b.Close()
    else:
        e, g = runner(mine, gradients)
    local = (share, np.asarray(e, dtype=np.float64).tolist(),
             [np.asarray(x, dtype=np.float64).tolist() for x in g] if gradients else None)
    if world > 1:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, local)
    else:
        parts = [local]
    energies = np.empty(len(evaluations), dtype=np.float64)
    grads = [None] * len(evaluations) if gradients else None
    for idx, es, gs in parts:
        for j, i in enumerate(idx):
            energies[i] = es[j]
            if gradients:
                grads[i] = np.asarray(gs[j], dtype=np.float64)
    return energies, grads
