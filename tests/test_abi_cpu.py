"""CPU-side checks of the C ABI: the library loads, exports every symbol the
header declares, and fails with a status (never a crash) without a GPU."""
import ctypes
import os
import re

import pytest

from goqu_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    with open(os.path.join(ROOT, "include", "gqb200.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(gq_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _abi.lib()
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_signatures_cover_header():
    assert set(header_symbols()) <= set(_abi.SIGNATURES), set(header_symbols()) - set(_abi.SIGNATURES)


def test_struct_layouts_match_header():
    # gq_op: 4 int32 + 16 int32 qubits + pointer + 3 int32 + pad int32 + 3 pointers
    assert ctypes.sizeof(_abi.gq_op) == 4 * 4 + 16 * 4 + 8 + 4 * 4 + 3 * 8
    assert ctypes.sizeof(_abi.gq_pauli_term) == 32
    assert ctypes.sizeof(_abi.gq_stats) == 104


def test_abi_version():
    assert _abi.lib().gq_abi_version() == 5


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES") is None and os.path.exists("/dev/nvidia0"),
                    reason="a GPU is present")
def test_create_without_gpu_fails_loudly():
    lib = _abi.lib()
    n = ctypes.c_int(-1)
    assert lib.gq_device_count(ctypes.byref(n)) == 0
    if n.value > 0:
        pytest.skip("an sm_100 device is visible")
    h = ctypes.c_void_p()
    rc = lib.gq_sv_create(5, 0, ctypes.byref(h))
    assert rc == _abi.GQ_ENODEVICE and not h.value
    assert lib.gq_last_error()
    with pytest.raises(_abi.GQError):
        from goqu_b200 import statevector
        statevector.New(3)


def test_invalid_arguments_rejected_before_device_use():
    lib = _abi.lib()
    h = ctypes.c_void_p()
    assert lib.gq_sv_create(0, 0, ctypes.byref(h)) == _abi.GQ_EINVAL
    assert lib.gq_sv_create(35, 0, ctypes.byref(h)) == _abi.GQ_EINVAL
    assert lib.gq_sv_create(3, 7, ctypes.byref(h)) == _abi.GQ_EINVAL
    assert lib.gq_dm_create(16, ctypes.byref(h)) == _abi.GQ_EINVAL
    assert b"out of range" in lib.gq_last_error()
