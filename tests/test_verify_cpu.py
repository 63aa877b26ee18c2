"""transpile/verify's argument errors, raised by the Python mirror before
the device is touched (verify_test.go:81-89, 152-160)."""
import pytest

from goqu_b200 import circuit as ir, verify


def test_qubit_mismatch_and_size_limits():
    with pytest.raises(ValueError, match="qubit count mismatch: 2 vs 3"):
        verify.EquivalentOnZero(ir.Circuit("a", 2, 0, []), ir.Circuit("b", 3, 0, []), 1e-8)
    with pytest.raises(ValueError, match="too large for equivalence check: 15 qubits"):
        verify.EquivalentOnZero(ir.Circuit("a", 15, 0, []), ir.Circuit("b", 15, 0, []), 1e-8)
    with pytest.raises(ValueError, match="too large for full equivalence check: 11 qubits"):
        verify.Equivalent(ir.Circuit("a", 11, 0, []), ir.Circuit("b", 11, 0, []), 1e-8)
