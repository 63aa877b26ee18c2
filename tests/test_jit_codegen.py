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
from kat_util import chain_circuit, random_circuit

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


# ---- the generated code run on the CPU --------------------------------------
# gqx_jit_emulate compiles the host form of every pass's generated code (the
# same segments as the kernel, threads of a CTA run in turn between barriers)
# and runs it with the packed parameter blocks: this checks the generator's
# pending-factor bookkeeping, the one-qubit shear decomposition and the
# parameter packing against the oracle without a GPU.

import numpy as np  # noqa: E402

from oracle import binding as orc  # noqa: E402

CSRC = os.path.join(ROOT, "goqu_b200", "csrc").encode()
_D = ctypes.POINTER(ctypes.c_double)


def jit_emulate(emu, stream, n, tmp_path, precision=_abi.GQ_C128, dm=0, tile=0):
    emu.gqx_jit_emulate.restype = ctypes.c_int
    emu.gqx_jit_emulate.argtypes = [ctypes.c_int, ctypes.c_int, _D, ctypes.POINTER(_abi.gq_op), ctypes.c_size_t,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p,
                                    ctypes.POINTER(ctypes.c_int64)]
    nv = 2 * n if dm else n
    st = np.zeros(1 << nv, dtype=np.complex128)
    st[0] = 1
    out = (ctypes.c_int64 * 2)()
    rc = emu.gqx_jit_emulate(n, precision, st.view(np.float64).ctypes.data_as(_D), stream.ptr(), len(stream), tile, 0,
                             dm, CSRC, str(tmp_path).encode(), out)
    assert rc == 0, emu.gqx_last_error().decode()
    passes, jitted = list(out)
    assert jitted == passes >= 1
    return st


@pytest.mark.parametrize("n,seed,tile", [(6, 1, 0), (9, 2, 7), (12, 3, 0), (13, 4, 10)])
def test_generated_code_matches_oracle(emu, tmp_path, n, seed, tile):
    # every gate family, with controls inside and outside the registers and resets
    c = random_circuit(n, 120, seed, allow_reset=True)
    ops = encode.statevector_ops(c)
    got = jit_emulate(emu, ops, n, tmp_path, tile=tile)
    np.testing.assert_allclose(got, orc.sv_evolve(ops), atol=1e-12, rtol=0)


def test_generated_code_layered_qft(emu, tmp_path):
    # U3 layers (shear form), CNOT permutations, QFT phases (pending factors)
    c = workloads.random_layers_qft(14, layers=10, seed=5)
    ops = encode.statevector_ops(c)
    want = orc.sv_evolve(ops)
    np.testing.assert_allclose(jit_emulate(emu, ops, 14, tmp_path), want, atol=1e-12, rtol=0)
    assert np.max(np.abs(jit_emulate(emu, ops, 14, tmp_path, precision=_abi.GQ_C64) - want)) < 2e-5


def test_generated_code_extreme_angles(emu, tmp_path):
    # rotations next to 0 and pi: tan(theta/2) near 0 and near 1e16
    from goqu_b200 import circuit as ir
    b = ir.Builder("x", 12)
    rng = np.random.default_rng(9)
    for layer in range(6):
        for q in range(12):
            th = [1e-14, np.pi - 1e-15, np.pi, 2 * np.pi - 1e-13, rng.uniform(0, 2 * np.pi)][(q + layer) % 5]
            b.U3(th, rng.uniform(0, 6.3), rng.uniform(0, 6.3), q)
        for q in range(layer % 2, 11, 2):
            b.CNOT(q, q + 1)
    ops = encode.statevector_ops(b.Build())
    np.testing.assert_allclose(jit_emulate(emu, ops, 12, tmp_path), orc.sv_evolve(ops), atol=1e-12, rtol=0)


def plan_stats(emu, stream, n, tile=0, precision=_abi.GQ_C128):
    emu.gqx_jit_plan_stats.restype = ctypes.c_int
    out = (ctypes.c_int64 * 6)()
    rc = emu.gqx_jit_plan_stats(n, precision, stream.ptr(), len(stream), tile, 0, out)
    assert rc == 0, emu.gqx_last_error().decode()
    return dict(zip(["passes", "planned", "chains", "candidates", "pred_phases", "acc_decls"], list(out)))


@pytest.mark.parametrize("n,seed,tile", [(12, 11, 7), (13, 12, 8), (14, 13, 0)])
def test_generated_code_uniform_predicates_and_chains(emu, tmp_path, n, seed, tile):
    # pending factors indexed by CTA-uniform predicates, fused one-qubit chains
    # and run-time phase accumulators, each checked to be in use
    ops = encode.statevector_ops(chain_circuit(n, seed))
    st = plan_stats(emu, ops, n, tile)
    assert st["planned"] == st["passes"]
    assert st["chains"] >= 1 and st["pred_phases"] >= 1 and st["acc_decls"] >= 1, st
    want = orc.sv_evolve(ops)
    np.testing.assert_allclose(jit_emulate(emu, ops, n, tmp_path, tile=tile), want, atol=1e-12, rtol=0)
    assert np.max(np.abs(jit_emulate(emu, ops, n, tmp_path, precision=_abi.GQ_C64, tile=tile) - want)) < 2e-5


def test_generated_code_unfusable_chains(emu, tmp_path):
    # H CNOT H with the control on a CTA-index bit: the chain's products are
    # I and Z (diagonal), which have no shear form, so the chain stays unfused
    from goqu_b200 import circuit as ir
    n = 12
    b = ir.Builder("hxh", n)
    rng = np.random.default_rng(4)
    for q in range(4, n):
        b.U3(*rng.uniform(0, 2 * np.pi, 3), q)
    for q in range(4):
        b.H(q)
        b.CNOT(8 + q, q)
        b.H(q)
    ops = encode.statevector_ops(b.Build())
    st = plan_stats(emu, ops, n, 7)
    assert st["planned"] == st["passes"] and st["candidates"] > st["chains"], st
    np.testing.assert_allclose(jit_emulate(emu, ops, n, tmp_path, tile=7), orc.sv_evolve(ops), atol=1e-12, rtol=0)


def test_layered_benchmark_uses_chains(emu):
    # the 28-qubit benchmark's brickwork: most CNOT targets fuse with their U3s
    c = workloads.random_layers_qft(28, layers=40, seed=2028)
    st = plan_stats(emu, encode.statevector_ops(c), 28)
    assert st["planned"] == st["passes"]
    assert st["chains"] >= 400, st


def test_generated_code_density_matrix(emu, tmp_path):
    c, nm = workloads.noisy_brickwork(5, layers=3, seed=1)
    ops = encode.density_ops(c, nm)
    np.testing.assert_allclose(jit_emulate(emu, ops, 5, tmp_path, dm=1), orc.dm_evolve(ops), atol=1e-12, rtol=0)


# ---- specialised reverse (adjoint) passes, host form -------------------------

def _adjoint(emu, circuit, names, x, h, tmp_path=None, tile=0):
    from goqu_b200 import pauli as P
    stream = encode.statevector_ops(circuit, {nm: float(x[i]) for i, nm in enumerate(names)}, names)
    terms = P.to_terms(h)
    grad = np.zeros(len(names))
    energy = ctypes.c_double()
    common = [circuit.NumQubits(), stream.ptr(), len(stream), ctypes.cast(terms, ctypes.POINTER(_abi.gq_pauli_term)),
              len(terms), len(names), tile, 0, grad.ctypes.data_as(_D), ctypes.byref(energy)]
    base = [ctypes.c_int, ctypes.POINTER(_abi.gq_op), ctypes.c_size_t, ctypes.POINTER(_abi.gq_pauli_term),
            ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, _D, _D]
    if tmp_path is None:
        emu.gqx_emulate_adjoint.restype = ctypes.c_int
        emu.gqx_emulate_adjoint.argtypes = base
        rc = emu.gqx_emulate_adjoint(*common)
        jitted = None
    else:
        emu.gqx_jit_emulate_adjoint.restype = ctypes.c_int
        emu.gqx_jit_emulate_adjoint.argtypes = base + [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64)]
        j = ctypes.c_int64()
        rc = emu.gqx_jit_emulate_adjoint(*common, CSRC, str(tmp_path).encode(), ctypes.byref(j))
        jitted = j.value
    assert rc == 0, emu.gqx_last_error().decode()
    return energy.value, grad, jitted


def _general_circuit():
    from goqu_b200 import circuit as ir, param as prm, pauli as P
    th = prm.NewVector("t", 6)
    b = ir.Builder("g", 9)
    for q in range(9):
        b.H(q)
    b.SymU3(th.At(0), prm.Mul(2.0, th.At(1)), th.At(2), 3).SymCP(th.At(3), 0, 8).SymRXX(th.At(4), 1, 2)
    b.SymRZZ(th.At(0), 2, 7).SymRX(prm.Neg(th.At(1)), 6).CNOT(3, 0).SymRY(th.At(5), 5).CCX(1, 2, 6)
    b.SymPhase(th.At(2), 4).SymRZ(th.At(4), 8).SymRYY(th.At(3), 4, 5)
    c = b.Build()
    h = P.NewPauliSum([P.NewPauliString(0.7, {0: P.Z, 3: P.X}, 9), P.NewPauliString(-0.4, {1: P.Y, 2: P.Y}, 9),
                       P.NewPauliString(0.25, {8: P.X, 6: P.Z}, 9)])
    from goqu_b200 import circuit as ir2
    return c, ir2.FreeParameters(c), h


@pytest.mark.parametrize("which,tile", [("hea6", 0), ("hea9", 6), ("general", 0), ("general", 5), ("qaoa", 0)])
def test_generated_dual_passes_match_interpreted_adjoint(emu, tmp_path, which, tile):
    if which.startswith("hea"):
        n = int(which[3:])
        c, names = workloads.hardware_efficient_ansatz(n, 3)
        h = workloads.ising_hamiltonian(n)
    elif which == "general":
        c, names, h = _general_circuit()
    else:
        c, names, h, x0 = workloads.qaoa_batch(1, seed=8, n_values=(10,))[0]
    x = np.random.default_rng(4).uniform(0, 2 * np.pi, len(names))
    e0, g0, _ = _adjoint(emu, c, names, x, h, tile=tile)
    e1, g1, jitted = _adjoint(emu, c, names, x, h, tmp_path, tile=tile)
    assert jitted >= 1
    assert abs(e0 - e1) < 1e-13
    np.testing.assert_allclose(g1, g0, atol=1e-12, rtol=0)


@pytest.mark.parametrize("precision", [_abi.GQ_C128, _abi.GQ_C64])
def test_dual_kernels_compile(emu, precision):
    # device text of the dual kernels (hardware-efficient ansatz; QAOA with
    # pair sums) compiles with NVRTC for sm_100a
    emu.gqx_jit_check_dual.restype = ctypes.c_int
    emu.gqx_jit_check_dual.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_abi.gq_op), ctypes.c_size_t,
                                       ctypes.c_size_t, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
    c, names = workloads.hardware_efficient_ansatz(12, 3)
    qc, qn, _, _ = workloads.qaoa_batch(1, seed=3, n_values=(12,))[0]
    for circ, nm in ((c, names), (qc, qn)):
        xv = np.random.default_rng(1).uniform(0, 6.2, len(nm))
        ops = encode.statevector_ops(circ, {k: float(xv[i]) for i, k in enumerate(nm)}, nm)
        out = (ctypes.c_int64 * 3)()
        rc = emu.gqx_jit_check_dual(circ.NumQubits(), precision, ops.ptr(), len(ops), len(nm), 2, out)
        if rc == _abi.GQ_EUNSUPPORTED:
            pytest.skip("libnvrtc not available")
        assert rc == 0, emu.gqx_last_error().decode()[:3000]
        passes, planned, compiled = list(out)
        assert planned == passes >= 1 and compiled >= 1


def test_on_disk_kernel_cache(emu, tmp_path, monkeypatch):
    # compiled kernels are stored under a hash of everything they depend on and
    # reused by later compilations (other processes included); a stored file
    # whose identity differs is never used
    f = emu.gqx_jit_compile_cached
    f.restype = ctypes.c_int64
    f.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
    monkeypatch.setenv("GQ_JIT_CACHE_DIR", str(tmp_path / "jit"))
    src = b"extern \"C\" __global__ void gqj_pass(double* x) { x[threadIdx.x] *= 2.0; }\n"
    hit = ctypes.c_int()
    n1 = f(src, ctypes.byref(hit))
    assert n1 > 0 and hit.value == 0
    files = list((tmp_path / "jit").iterdir())
    assert len(files) == 1 and files[0].suffix == ".cubin"
    n2 = f(src, ctypes.byref(hit))
    assert n2 == n1 and hit.value == 1
    # a different kernel text is a different entry
    assert f(src.replace(b"2.0", b"3.0"), ctypes.byref(hit)) > 0 and hit.value == 0
    # a file whose stored identity does not match is ignored and rewritten
    data = bytearray(files[0].read_bytes())
    data[20] ^= 0xFF
    files[0].write_bytes(bytes(data))
    assert f(src, ctypes.byref(hit)) == n1 and hit.value == 0
    assert f(src, ctypes.byref(hit)) == n1 and hit.value == 1
    monkeypatch.setenv("GQ_JIT_CACHE_DIR", "off")
    assert f(src, ctypes.byref(hit)) == n1 and hit.value == 0


@pytest.mark.parametrize("n,seed,tile", [(10, 41, 6), (12, 42, 7)])
def test_generated_code_skipping_zero_tiles(emu, tmp_path, n, seed, tile):
    # from the reset state, passes launch only the tiles inside the support
    # (fewer CTA-index bits, controls on zero qubits outside every table)
    emu.gqx_set_support0.argtypes = [ctypes.c_uint64]
    emu.gqx_last_ctas.restype = ctypes.c_int64
    c = random_circuit(n, 100, seed, allow_reset=True)
    ops = encode.statevector_ops(c)
    emu.gqx_set_support0(0)
    try:
        got = jit_emulate(emu, ops, n, tmp_path, tile=tile)
        ctas = emu.gqx_last_ctas()
    finally:
        emu.gqx_set_support0(2 ** 64 - 1)
    np.testing.assert_allclose(got, orc.sv_evolve(ops), atol=1e-12, rtol=0)
    full = jit_emulate(emu, ops, n, tmp_path, tile=tile)
    np.testing.assert_allclose(got, full, atol=1e-13, rtol=0)
    assert ctas < emu.gqx_last_ctas()


def test_generated_code_density_matrix_skipping_zero_tiles(emu, tmp_path):
    # the vectorised |0><0| has entry 0 only: the same support rule holds
    c, nm = workloads.noisy_brickwork(5, layers=3, seed=3)
    ops = encode.density_ops(c, nm)
    emu.gqx_set_support0.argtypes = [ctypes.c_uint64]
    emu.gqx_last_ctas.restype = ctypes.c_int64
    emu.gqx_set_support0(0)
    try:
        got = jit_emulate(emu, ops, 5, tmp_path, dm=1, tile=5)
        ctas = emu.gqx_last_ctas()
    finally:
        emu.gqx_set_support0(2 ** 64 - 1)
    np.testing.assert_allclose(got, orc.dm_evolve(ops), atol=1e-12, rtol=0)
    full = jit_emulate(emu, ops, 5, tmp_path, dm=1, tile=5)
    np.testing.assert_allclose(got, full, atol=1e-13, rtol=0)
    assert ctas < emu.gqx_last_ctas()


@pytest.mark.parametrize("precision", [_abi.GQ_C128, _abi.GQ_C64])
def test_persistent_kernels_compile(emu, precision):
    # persistent CTAs with one tile buffer refilled during the last phase
    # (GQ_OPT_JIT_PERSISTENT): the texts compile with NVRTC (at 2 CTAs of 256
    # threads per SM the loop holds up to 128 registers; the heaviest passes
    # spill a few words, which the autotuner's timing accounts for)
    emu.gqx_set_persistent.argtypes = [ctypes.c_int]
    c = workloads.random_layers_qft(24, 6, 7)
    s = encode.statevector_ops(c)
    out = (ctypes.c_int64 * 5)()
    emu.gqx_set_persistent(1)
    try:
        rc = emu.gqx_jit_check(24, precision, s.ptr(), len(s), 12, 0, 0, 4, out)
    finally:
        emu.gqx_set_persistent(0)
    if rc == _abi.GQ_EUNSUPPORTED:
        pytest.skip("libnvrtc not available")
    assert rc == 0, emu.gqx_last_error().decode()[:3000]
    passes, planned, texts, compiled, spilled = list(out)
    assert planned == passes >= 1 and compiled >= 1 and spilled <= compiled
