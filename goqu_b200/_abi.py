"""ctypes view of the C ABI declared in include/gqb200.h.

Loading is strict: if ``libgqb200.so`` (built in-tree by ``build.py``) is
missing or fails to load, every engine entry point raises ``GQError``. There is
no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

GQ_OK = 0
GQ_EINVAL = 1
GQ_ENOMEM = 2
GQ_ECUDA = 3
GQ_EUNSUPPORTED = 4
GQ_ENODEVICE = 5
GQ_EDEVICE = 6

GQ_C128 = 0
GQ_C64 = 1

GQ_OP_MATRIX = 0
GQ_OP_CNOT = 1
GQ_OP_CZ = 2
GQ_OP_SWAP = 3
GQ_OP_CY = 4
GQ_OP_ISWAP = 5
GQ_OP_SYCAMORE = 6
GQ_OP_CCX = 7
GQ_OP_CSWAP = 8
GQ_OP_CCZ = 9
GQ_OP_CTRL_DIAG_2Q = 10
GQ_OP_DIAG_2Q = 11
GQ_OP_CTRL_U_2Q = 12
GQ_OP_CONTROLLED = 13
GQ_OP_RESET = 14
GQ_OP_CHANNEL = 15
GQ_OP_BARRIER = 16

GQ_MAX_OP_QUBITS = 16
GQ_MAX_OP_PARAMS = 3

GQ_OPT_TILE_QUBITS = 1
GQ_OPT_PASS_BUDGET = 2
GQ_OPT_LOW_QUBITS = 3
GQ_OPT_TIMING = 4
GQ_OPT_KERNEL_VARIANT = 5
GQ_OPT_ADJOINT_SEGMENTS = 6
GQ_OPT_USE_GRAPH = 7
GQ_OPT_FUSE_DENSE = 8
GQ_OPT_JIT = 9
GQ_OPT_JIT_MIN_QUBITS = 10
GQ_OPT_JIT_MIN_BLOCKS = 11
GQ_OPT_JIT_PERSISTENT = 12
GQ_OPT_DM_DENSE_CHANNELS = 13
GQ_OPT_ZERO_TILES = 14

GQ_NOALLOC_MAX_TERMS = 2048

_DBL_P = ctypes.POINTER(ctypes.c_double)


class gq_op(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("num_qubits", ctypes.c_int32),
        ("num_controls", ctypes.c_int32),
        ("num_kraus", ctypes.c_int32),
        ("qubits", ctypes.c_int32 * GQ_MAX_OP_QUBITS),
        ("matrix", _DBL_P),
        ("param_index", ctypes.c_int32 * GQ_MAX_OP_PARAMS),
        ("reserved", ctypes.c_int32),
        ("dmatrix", _DBL_P * GQ_MAX_OP_PARAMS),
    ]


class gq_pauli_term(ctypes.Structure):
    _fields_ = [
        ("coeff_re", ctypes.c_double),
        ("coeff_im", ctypes.c_double),
        ("x_mask", ctypes.c_uint64),
        ("z_mask", ctypes.c_uint64),
    ]


class gq_stats(ctypes.Structure):
    _fields_ = [
        ("gates_in", ctypes.c_int64),
        ("passes", ctypes.c_int64),
        ("kernel_launches", ctypes.c_int64),
        ("phases", ctypes.c_int64),
        ("state_bytes", ctypes.c_int64),
        ("last_ms", ctypes.c_double),
        ("pass_ms", ctypes.c_double),
        ("h2d_bytes", ctypes.c_int64),
        ("d2h_bytes", ctypes.c_int64),
        ("jit_passes", ctypes.c_int64),
        ("jit_compile_ms", ctypes.c_double),
        ("host_ms", ctypes.c_double),
        ("tile_bytes", ctypes.c_int64),
    ]


class gq_batch_item(ctypes.Structure):
    _fields_ = [
        ("num_qubits", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("ops", ctypes.POINTER(gq_op)),
        ("n_ops", ctypes.c_size_t),
        ("terms", ctypes.POINTER(gq_pauli_term)),
        ("n_terms", ctypes.c_size_t),
        ("n_params", ctypes.c_size_t),
    ]


class gq_sweep_point(ctypes.Structure):
    _fields_ = [
        ("ops", ctypes.POINTER(gq_op)),
        ("n_ops", ctypes.c_size_t),
        ("uniforms", ctypes.POINTER(ctypes.c_double)),
    ]


class gq_param_gate(ctypes.Structure):
    _fields_ = [
        ("op_index", ctypes.c_int32),
        ("gate", ctypes.c_int32),
        ("num_angles", ctypes.c_int32),
        ("param", ctypes.c_int32 * 3),
        ("scale", ctypes.c_double * 3),
        ("shift", ctypes.c_double * 3),
    ]


class gq_adam_options(ctypes.Structure):
    _fields_ = [
        ("lr", ctypes.c_double), ("beta1", ctypes.c_double), ("beta2", ctypes.c_double),
        ("epsilon", ctypes.c_double), ("max_iter", ctypes.c_int32), ("reserved", ctypes.c_int32),
        ("fun_tol", ctypes.c_double), ("grad_tol", ctypes.c_double),
    ]


class gq_optim_result(ctypes.Structure):
    _fields_ = [
        ("fun", ctypes.c_double), ("iterations", ctypes.c_int32), ("func_evals", ctypes.c_int32),
        ("grad_evals", ctypes.c_int32), ("converged", ctypes.c_int32),
    ]


GQ_PG = {"RX": 1, "RY": 2, "RZ": 3, "P": 4, "U1": 5, "U2": 6, "U3": 7, "Rot": 8, "CP": 9, "RXX": 10, "RYY": 11,
         "RZZ": 12, "FSim": 13, "PSwap": 14, "GlobalPhase": 15}


class gq_qaoa_item(ctypes.Structure):
    _fields_ = [
        ("num_qubits", ctypes.c_int32), ("p", ctypes.c_int32), ("edges", ctypes.POINTER(ctypes.c_int32)),
        ("n_edges", ctypes.c_size_t), ("gammas", ctypes.POINTER(ctypes.c_double)),
        ("betas", ctypes.POINTER(ctypes.c_double)),
    ]


class GQError(RuntimeError):
    """An engine call returned a non-zero status."""

    def __init__(self, code, msg):
        super().__init__(f"gqb200 error {code}: {msg}")
        self.code = code


LIB_NAME = "libgqb200.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

_lib = None
_lib_lock = threading.Lock()

# Exported symbols and their argument types (must match include/gqb200.h).
_VP = ctypes.c_void_p
_SZ = ctypes.c_size_t
_I = ctypes.c_int
_OPP = ctypes.POINTER(gq_op)
_TP = ctypes.POINTER(gq_pauli_term)
_U64P = ctypes.POINTER(ctypes.c_uint64)
SIGNATURES = {
    "gq_abi_version": (ctypes.c_int, []),
    "gq_last_error": (ctypes.c_char_p, []),
    "gq_device_count": (_I, [ctypes.POINTER(ctypes.c_int)]),
    "gq_sv_create": (_I, [_I, _I, ctypes.POINTER(_VP)]),
    "gq_sv_destroy": (_I, [_VP]),
    "gq_sv_num_qubits": (_I, [_VP, ctypes.POINTER(ctypes.c_int)]),
    "gq_sv_reset": (_I, [_VP]),
    "gq_sv_apply": (_I, [_VP, _OPP, _SZ]),
    "gq_sv_evolve": (_I, [_VP, _OPP, _SZ]),
    "gq_sv_get_state": (_I, [_VP, _VP, _SZ]),
    "gq_sv_set_state": (_I, [_VP, _VP, _SZ]),
    "gq_sv_probabilities": (_I, [_VP, _DBL_P, _SZ]),
    "gq_sv_sample": (_I, [_VP, _DBL_P, _SZ, _U64P]),
    "gq_sv_run": (_I, [_VP, _OPP, _SZ, _DBL_P, _SZ, _U64P]),
    "gq_sv_sample_counts": (_I, [_VP, _DBL_P, _SZ, _U64P, _U64P, ctypes.POINTER(_SZ)]),
    "gq_sv_run_counts": (_I, [_VP, _OPP, _SZ, _DBL_P, _SZ, _U64P, _U64P, ctypes.POINTER(_SZ)]),
    "gq_sv_expect_pauli_sum": (_I, [_VP, _TP, _SZ, _DBL_P, _DBL_P]),
    "gq_sv_expect_z_mask": (_I, [_VP, ctypes.c_uint64, _DBL_P]),
    "gq_sv_adjoint_gradient": (_I, [_VP, _OPP, _SZ, _TP, _SZ, _SZ, _DBL_P, _DBL_P]),
    "gq_sv_prob0": (_I, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "gq_sv_collapse": (_I, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
    "gq_sv_measure": (_I, [_VP, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]),
    "gq_sv_copy_state": (_I, [_VP, _VP]),
    "gq_sv_stats": (_I, [_VP, ctypes.POINTER(gq_stats)]),
    "gq_sv_set_option": (_I, [_VP, _I, ctypes.c_int64]),
    "gq_dm_create": (_I, [_I, ctypes.POINTER(_VP)]),
    "gq_dm_destroy": (_I, [_VP]),
    "gq_dm_reset": (_I, [_VP]),
    "gq_dm_apply": (_I, [_VP, _OPP, _SZ]),
    "gq_dm_evolve": (_I, [_VP, _OPP, _SZ]),
    "gq_dm_get": (_I, [_VP, _DBL_P, _SZ]),
    "gq_dm_set": (_I, [_VP, _DBL_P, _SZ]),
    "gq_dm_diagonal_probs": (_I, [_VP, _DBL_P, _SZ]),
    "gq_dm_expect_pauli_sum": (_I, [_VP, _TP, _SZ, _DBL_P, _DBL_P]),
    "gq_dm_trace": (_I, [_VP, _DBL_P, _DBL_P]),
    "gq_dm_purity": (_I, [_VP, _DBL_P]),
    "gq_dm_fidelity": (_I, [_VP, _DBL_P, _SZ, _DBL_P]),
    "gq_dm_sample": (_I, [_VP, _DBL_P, _DBL_P, _DBL_P, _SZ, _U64P]),
    "gq_dm_sample_counts": (_I, [_VP, _DBL_P, _DBL_P, _DBL_P, _SZ, _U64P, _U64P, ctypes.POINTER(_SZ)]),
    "gq_dm_prob0": (_I, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "gq_dm_collapse": (_I, [_VP, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
    "gq_dm_measure": (_I, [_VP, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]),
    "gq_dm_copy_state": (_I, [_VP, _VP]),
    "gq_dm_stats": (_I, [_VP, ctypes.POINTER(gq_stats)]),
    "gq_dm_set_option": (_I, [_VP, _I, ctypes.c_int64]),
    "gq_batch_create": (_I, [_I, ctypes.POINTER(_VP)]),
    "gq_batch_destroy": (_I, [_VP]),
    "gq_batch_run": (_I, [_VP, ctypes.POINTER(gq_batch_item), _SZ, _I, _DBL_P, _DBL_P]),
    "gq_batch_set_option": (_I, [_VP, _I, ctypes.c_int64]),
    "gq_batch_stats": (_I, [_VP, ctypes.POINTER(gq_stats)]),
    "gq_sv_adjoint_template": (_I, [_VP, _OPP, _SZ, ctypes.POINTER(gq_param_gate), _SZ, _DBL_P, _SZ, _TP, _SZ,
                                    _DBL_P, _DBL_P]),
    "gq_sv_minimize_adam": (_I, [_VP, _OPP, _SZ, ctypes.POINTER(gq_param_gate), _SZ, _TP, _SZ, _SZ, _DBL_P,
                                 ctypes.POINTER(gq_adam_options), ctypes.POINTER(gq_optim_result), _DBL_P, _SZ]),
    "gq_qaoa_maxcut_batch": (_I, [_I, ctypes.POINTER(gq_qaoa_item), _SZ, _I, _DBL_P, _DBL_P]),
    "gq_unitary": (_I, [_I, _OPP, _SZ, _DBL_P, _SZ]),
    "gq_equivalent": (_I, [_I, _OPP, _SZ, _OPP, _SZ, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]),
    "gq_equivalent_on_zero": (_I, [_I, _OPP, _SZ, _OPP, _SZ, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]),
    "gq_sweep_run": (_I, [_I, _I, ctypes.POINTER(gq_sweep_point), _SZ, _SZ, _U64P, _U64P, ctypes.POINTER(_SZ),
                          ctypes.POINTER(ctypes.c_int32)]),
    "gq_sweep_run_density": (_I, [_I, _DBL_P, _DBL_P, ctypes.POINTER(gq_sweep_point), _SZ, _SZ, _U64P, _U64P,
                                  ctypes.POINTER(_SZ), ctypes.POINTER(ctypes.c_int32)]),
    "gq_expect_pauli_sum_noalloc": (_I, [_VP, _I, _I, _TP, _SZ, _VP, _DBL_P, _DBL_P]),
}


def lib():
    """The loaded engine library; raises GQError when it cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise GQError(GQ_ENODEVICE, f"{LIB_NAME} is not built (run __graft_entry__.build())")
            try:
                handle = ctypes.CDLL(LIB_PATH)
            except OSError as exc:
                raise GQError(GQ_ENODEVICE, f"cannot load {LIB_PATH}: {exc}") from exc
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
    return _lib


def check(code):
    """Raise GQError carrying the engine's message for a non-zero status."""
    if code != GQ_OK:
        msg = lib().gq_last_error()
        raise GQError(code, msg.decode() if msg else "")
