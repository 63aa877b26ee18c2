"""gq_expect_pauli_sum_noalloc: the expectation entry point for callers that
cannot let the library allocate device memory. The state is allocated by the
caller (here with torch); the result must equal the regular entry point's
(gq_sv_expect_pauli_sum) within the complex128 tolerance of the other tests,
on consecutive calls that reuse the library's static scratch array."""
import ctypes

import numpy as np
import pytest

from goqu_b200 import _abi, pauli as P, statevector, workloads

pytestmark = pytest.mark.gpu

TOL128 = 1e-12


def noalloc_expect(dev_ptr, nq, precision, terms):
    re, im = ctypes.c_double(), ctypes.c_double()
    _abi.check(_abi.lib().gq_expect_pauli_sum_noalloc(
        ctypes.c_void_p(dev_ptr), nq, precision, ctypes.cast(terms, ctypes.POINTER(_abi.gq_pauli_term)), len(terms),
        None, ctypes.byref(re), ctypes.byref(im)))
    return complex(re.value, im.value)


@pytest.mark.parametrize("precision,dtype", [(_abi.GQ_C128, "complex128"), (_abi.GQ_C64, "complex64")])
def test_noalloc_matches_regular_entry_point_twice(precision, dtype):
    import torch
    n = 14
    c = workloads.random_layers(n, layers=5, seed=77)
    sim = statevector.New(n, precision)
    sim.Evolve(c)
    host = sim.StateVector().astype(dtype)
    dev = torch.from_numpy(host).to("cuda")  # the caller's own device allocation
    torch.cuda.synchronize()
    rng = np.random.default_rng(5)
    hams = [workloads.ising_hamiltonian(n)]
    # second sum: random Pauli strings with complex coefficients (X, Y, Z mixed)
    terms = []
    for _ in range(40):
        ops = {int(q): [P.X, P.Y, P.Z][rng.integers(3)] for q in rng.choice(n, 3, replace=False)}
        terms.append(P.NewPauliString(complex(*rng.normal(size=2)), ops, n))
    hams.append(P.NewPauliSum(terms))
    for h in hams:  # two calls in a row on the same scratch
        t = P.to_terms(h)
        want = sim.expect_terms(t)
        got = noalloc_expect(dev.data_ptr(), n, precision, t)
        assert abs(got - want) < TOL128, (got, want)
    sim.Close()


def test_noalloc_rejects_oversized_sums():
    import torch
    dev = torch.zeros(1 << 4, dtype=torch.complex128, device="cuda")
    terms = (_abi.gq_pauli_term * (_abi.GQ_NOALLOC_MAX_TERMS + 1))()
    rc = _abi.lib().gq_expect_pauli_sum_noalloc(ctypes.c_void_p(dev.data_ptr()), 4, _abi.GQ_C128,
                                                ctypes.cast(terms, ctypes.POINTER(_abi.gq_pauli_term)), len(terms),
                                                None, None, None)
    assert rc == _abi.GQ_EINVAL
    assert b"GQ_NOALLOC_MAX_TERMS" in _abi.lib().gq_last_error()
