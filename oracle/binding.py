"""ctypes binding of oracle/liboracle.so, the FP64 CPU restatement of goqu.

TEST INFRASTRUCTURE: used by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg only. It consumes the same gq_op streams as the engine
(goqu_b200.encode), so both sides are fed identical matrices.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from goqu_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_U64 = ctypes.POINTER(ctypes.c_uint64)
_OPP = ctypes.POINTER(_abi.gq_op)
_TP = ctypes.POINTER(_abi.gq_pauli_term)


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        h = ctypes.CDLL(LIB)
        sig = {
            "or_sv_apply": (ctypes.c_int, [ctypes.c_int, _D, _OPP, ctypes.c_size_t, ctypes.c_int]),
            "or_sv_probabilities": (None, [ctypes.c_int, _D, _D]),
            "or_sample": (None, [_D, ctypes.c_uint64, _D, ctypes.c_size_t, _U64]),
            "or_cumsum_at": (None, [_D, ctypes.c_uint64, _U64, ctypes.c_size_t, _D]),
            "or_cumsum": (None, [_D, ctypes.c_uint64, _D]),
            "or_sv_expect_pauli_sum": (None, [ctypes.c_int, _D, _TP, ctypes.c_size_t, ctypes.c_int, _D, _D]),
            "or_sv_expect_z": (ctypes.c_double, [ctypes.c_int, _D, ctypes.c_uint64, ctypes.c_int]),
            "or_dm_apply": (ctypes.c_int, [ctypes.c_int, _D, _OPP, ctypes.c_size_t, ctypes.c_int]),
            "or_dm_expect_pauli_sum": (None, [ctypes.c_int, _D, _TP, ctypes.c_size_t, _D, _D]),
            "or_dm_purity": (ctypes.c_double, [ctypes.c_int, _D]),
            "or_dm_fidelity": (ctypes.c_double, [ctypes.c_int, _D, _D]),
            "or_dm_diagonal_probs": (None, [ctypes.c_int, _D, _D]),
            "or_dm_readout": (None, [ctypes.c_int, _D, _D, _D]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def _dp(a):
    return a.ctypes.data_as(_D)


def zero_state(nq):
    s = np.zeros(1 << nq, dtype=np.complex128)
    s[0] = 1
    return s


def sv_apply(state, stream, threads=0):
    """Apply an OpStream to `state` (complex128, modified in place)."""
    nq = stream.num_qubits
    assert state.dtype == np.complex128 and state.size == 1 << nq and state.flags.c_contiguous
    rc = lib().or_sv_apply(nq, _dp(state.view(np.float64)), stream.ptr(), len(stream), threads)
    if rc != 0:
        raise ValueError(f"unsupported gate size (oracle status {rc})")
    return state


def sv_evolve(stream, threads=0):
    return sv_apply(zero_state(stream.num_qubits), stream, threads)


def probabilities(state):
    nq = state.size.bit_length() - 1
    p = np.empty(state.size, dtype=np.float64)
    lib().or_sv_probabilities(nq, _dp(np.ascontiguousarray(state).view(np.float64)), _dp(p))
    return p


def sample(probs, uniforms):
    probs = np.ascontiguousarray(probs, dtype=np.float64)
    u = np.ascontiguousarray(uniforms, dtype=np.float64)
    out = np.empty(u.size, dtype=np.uint64)
    lib().or_sample(_dp(probs), probs.size, _dp(u), u.size, out.ctypes.data_as(_U64))
    return out


def sample_fast(probs, uniforms):
    """sampleIndex for many shots: the sequential running sum once, then a
    sorted search (first i with r < cum_i; the last index when none)."""
    probs = np.ascontiguousarray(probs, dtype=np.float64)
    cum = np.empty_like(probs)
    lib().or_cumsum(_dp(probs), probs.size, _dp(cum))
    idx = np.searchsorted(cum, np.asarray(uniforms, dtype=np.float64), side="right")
    return np.minimum(idx, probs.size - 1).astype(np.uint64)


def cumsum_at(probs, indices):
    probs = np.ascontiguousarray(probs, dtype=np.float64)
    idx = np.ascontiguousarray(np.sort(np.asarray(indices, dtype=np.uint64)))
    out = np.empty(idx.size, dtype=np.float64)
    lib().or_cumsum_at(_dp(probs), probs.size, idx.ctypes.data_as(_U64), idx.size, _dp(out))
    return idx, out


def expect_pauli_sum(state, terms, threads=0):
    nq = state.size.bit_length() - 1
    re, im = ctypes.c_double(), ctypes.c_double()
    lib().or_sv_expect_pauli_sum(nq, _dp(np.ascontiguousarray(state).view(np.float64)),
                                 ctypes.cast(terms, _TP), len(terms), threads, ctypes.byref(re), ctypes.byref(im))
    return complex(re.value, im.value)


def expect_z(state, mask, rounded=False):
    nq = state.size.bit_length() - 1
    return lib().or_sv_expect_z(nq, _dp(np.ascontiguousarray(state).view(np.float64)), mask, int(rounded))


def dm_zero(nq):
    r = np.zeros((1 << nq) * (1 << nq), dtype=np.complex128)
    r[0] = 1
    return r


def dm_apply(rho, stream, threads=0):
    nq = stream.num_qubits
    rc = lib().or_dm_apply(nq, _dp(rho.view(np.float64)), stream.ptr(), len(stream), threads)
    if rc != 0:
        raise ValueError(f"oracle dm status {rc}")
    return rho


def dm_evolve(stream, threads=0):
    return dm_apply(dm_zero(stream.num_qubits), stream, threads)


def dm_expect_pauli_sum(rho, nq, terms):
    re, im = ctypes.c_double(), ctypes.c_double()
    lib().or_dm_expect_pauli_sum(nq, _dp(rho.view(np.float64)), ctypes.cast(terms, _TP), len(terms),
                                 ctypes.byref(re), ctypes.byref(im))
    return complex(re.value, im.value)


def dm_purity(rho, nq):
    return lib().or_dm_purity(nq, _dp(rho.view(np.float64)))


def dm_fidelity(rho, nq, psi):
    psi = np.ascontiguousarray(psi, dtype=np.complex128)
    return lib().or_dm_fidelity(nq, _dp(rho.view(np.float64)), _dp(psi.view(np.float64)))


def dm_diagonal_probs(rho, nq):
    p = np.empty(1 << nq, dtype=np.float64)
    lib().or_dm_diagonal_probs(nq, _dp(rho.view(np.float64)), _dp(p))
    return p


def dm_readout(probs, nq, p01, p10):
    probs = np.array(probs, dtype=np.float64)
    a = np.ascontiguousarray(p01, dtype=np.float64)
    b = np.ascontiguousarray(p10, dtype=np.float64)
    lib().or_dm_readout(nq, _dp(probs), _dp(a), _dp(b))
    return probs


def sv_measure(state, qubit, u):
    """measureQubit with uniform u (in place); returns the outcome."""
    lib().or_sv_measure.restype = ctypes.c_int
    lib().or_sv_measure.argtypes = [ctypes.c_int, _D, ctypes.c_int, ctypes.c_double]
    nq = state.size.bit_length() - 1
    return lib().or_sv_measure(nq, _dp(state.view(np.float64)), qubit, u)


def dm_measure(rho, nq, qubit, u):
    """measureQubitDM with uniform u (in place); returns the outcome."""
    lib().or_dm_measure.restype = ctypes.c_int
    lib().or_dm_measure.argtypes = [ctypes.c_int, _D, ctypes.c_int, ctypes.c_double]
    return lib().or_dm_measure(nq, _dp(rho.view(np.float64)), qubit, u)
