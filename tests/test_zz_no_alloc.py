"""gq_expect_pauli_sum_noalloc: the expectation entry point for callers that
cannot let the library allocate device memory. The state is allocated by the
caller (here with torch); the result must equal the regular entry point's
(gq_sv_expect_pauli_sum) within the complex128 tolerance of the other tests,
on consecutive calls that reuse the library's static scratch array."""
import ctypes

import numpy as np
import pytest

from goqu_b200 import _abi, encode, pauli as P, statevector, workloads
from oracle import binding as orc

pytestmark = pytest.mark.gpu

TOL128 = 1e-12


def noalloc_expect(dev_ptr, nq, precision, terms, stream=None):
    re, im = ctypes.c_double(), ctypes.c_double()
    tp = ctypes.cast(terms, ctypes.POINTER(_abi.gq_pauli_term)) if len(terms) else None
    _abi.check(_abi.lib().gq_expect_pauli_sum_noalloc(
        ctypes.c_void_p(dev_ptr), nq, precision, tp, len(terms),
        ctypes.c_void_p(stream) if stream else None, ctypes.byref(re), ctypes.byref(im)))
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
    tol = TOL128 if precision == _abi.GQ_C128 else 1e-5
    oracle_state = orc.sv_evolve(encode.statevector_ops(c))
    side = torch.cuda.Stream()  # a caller's own stream, passed as its cudaStream_t
    for h in hams:  # two calls in a row on the same scratch
        t = P.to_terms(h)
        want = sim.expect_terms(t)
        got = noalloc_expect(dev.data_ptr(), n, precision, t)
        assert abs(got - want) < TOL128, (got, want)
        got_side = noalloc_expect(dev.data_ptr(), n, precision, t, side.cuda_stream)
        assert abs(got_side - want) < TOL128, (got_side, want)
        # and against the FP64 oracle's expectation of the same circuit
        ref = orc.expect_pauli_sum(oracle_state, t)
        assert abs(got - ref) < tol, (got, ref)
    # the empty sum is zero, even though the scratch still holds the last call's tables
    assert noalloc_expect(dev.data_ptr(), n, precision, []) == 0
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


def test_noalloc_rejects_host_memory_and_capture():
    import torch
    host = np.zeros(16, dtype=np.complex128)
    host[0] = 1
    t = P.to_terms(P.NewPauliSum([P.ZOn([0], 4)]))
    re, im = ctypes.c_double(), ctypes.c_double()
    rc = _abi.lib().gq_expect_pauli_sum_noalloc(ctypes.c_void_p(host.ctypes.data), 4, _abi.GQ_C128,
                                                ctypes.cast(t, ctypes.POINTER(_abi.gq_pauli_term)), len(t), None,
                                                ctypes.byref(re), ctypes.byref(im))
    assert rc == _abi.GQ_EINVAL
    assert b"device memory" in _abi.lib().gq_last_error() or b"CUDA pointer" in _abi.lib().gq_last_error()
    # a capturing stream is refused before anything is enqueued on it
    dev = torch.zeros(16, dtype=torch.complex128, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        rc = _abi.lib().gq_expect_pauli_sum_noalloc(ctypes.c_void_p(dev.data_ptr()), 4, _abi.GQ_C128,
                                                    ctypes.cast(t, ctypes.POINTER(_abi.gq_pauli_term)), len(t),
                                                    ctypes.c_void_p(s.cuda_stream), ctypes.byref(re),
                                                    ctypes.byref(im))
        g.capture_end()
    assert rc == _abi.GQ_EINVAL
    assert b"capturing" in _abi.lib().gq_last_error()
