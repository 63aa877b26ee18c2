"""CPU checks of the specialised tile-pass kernels (no device needed).

The engine's generator (goqu_b200/csrc/jit_gen.cpp) emits one kernel text per
pass; libgqb200_emu.so schedules a circuit the way the engine does and
compiles the distinct texts with NVRTC for sm_100a. Every text must compile,
and without register spills at the engine's launch bounds.
"""
import ctypes
import os

import pytest

from goqu_b200 import _abi, encode, workloads
from kat_util import random_circuit

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU = os.path.join(ROOT, "goqu_b200", "libgqb200_emu.so")


@pytest.fixture(scope="module")
def emu():
    if not os.path.exists(EMU):
        import build as _build
        _build.build_emulator()
    h = ctypes.CDLL(EMU)
    h.gqx_jit_check.restype = ctypes.c_int
    h.gqx_jit_check.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_abi.gq_op), ctypes.c_size_t, ctypes.c_int,
                                ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
    h.gqx_last_error.restype = ctypes.c_char_p
    return h


def check(emu, stream, n, precision=_abi.GQ_C128, dm=0, max_compile=2):
    out = (ctypes.c_int64 * 5)()
    rc = emu.gqx_jit_check(n, precision, stream.ptr(), len(stream), 0, 0, dm, max_compile, out)
    if rc == _abi.GQ_EUNSUPPORTED:
        pytest.skip("libnvrtc not available")
    assert rc == 0, emu.gqx_last_error().decode()[:3000]
    passes, planned, texts, compiled, spilled = list(out)
    assert planned == passes >= 1
    assert 1 <= texts <= passes and compiled >= 1
    assert spilled == 0
    return passes, texts


@pytest.mark.parametrize("precision", [_abi.GQ_C128, _abi.GQ_C64])
def test_random_circuit_kernels_compile(emu, precision):
    # every gate family: dense 1-3 qubit, controlled, SWAP, diagonal, reset
    c = random_circuit(12, 80, 7, allow_reset=True)
    check(emu, encode.statevector_ops(c), 12, precision)


def test_layered_benchmark_kernels_repeat(emu):
    # 40 U3+CNOT brickwork layers + QFT: passes of the same structure share a kernel text
    c = workloads.random_layers_qft(20, layers=40, seed=2028)
    passes, texts = check(emu, encode.statevector_ops(c), 20, max_compile=1)
    assert texts < passes


def test_density_matrix_kernels_compile(emu):
    c, nm = workloads.noisy_brickwork(6, layers=3, seed=1)
    check(emu, encode.density_ops(c, nm), 6, dm=1)
