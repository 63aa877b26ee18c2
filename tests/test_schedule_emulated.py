"""CPU checks of the pass scheduler and the tile-pass index tables.

libgqb200_emu.so runs the engine's own scheduler and the same tile-pass code
the sm_100a kernel compiles (goqu_b200/csrc/tile_core.cuh), emulated on the
host. Results must match the oracle to 1e-12 (c128) on seeded random circuits
over every gate family, for several tile sizes and pass budgets.
"""
import ctypes
import os

import numpy as np
import pytest

from goqu_b200 import _abi, circuit as ir, encode, workloads
from oracle import binding as orc

from kat_util import build_circuit, cplx, load_kats, random_circuit

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU = os.path.join(ROOT, "goqu_b200", "libgqb200_emu.so")


@pytest.fixture(scope="module")
def emu():
    if not os.path.exists(EMU):
        import build as _build
        _build.build_emulator()
    h = ctypes.CDLL(EMU)
    h.gqx_emulate_sv.restype = ctypes.c_int
    h.gqx_emulate_sv.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(_abi.gq_op), ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    h.gqx_last_error.restype = ctypes.c_char_p
    return h


def run_emu(emu, stream, precision=_abi.GQ_C128, tile=0, budget=0):
    n = stream.num_qubits
    st = np.zeros(1 << n, dtype=np.complex128)
    st[0] = 1
    passes, phases = ctypes.c_int64(), ctypes.c_int64()
    rc = emu.gqx_emulate_sv(n, precision, st.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            stream.ptr(), len(stream), tile, budget, ctypes.byref(passes), ctypes.byref(phases))
    assert rc == 0, emu.gqx_last_error()
    return st, passes.value, phases.value


@pytest.mark.parametrize("kat", [k for k in load_kats() if not k.get("dm") and "state" in k],
                         ids=lambda k: k["name"])
def test_emulated_kats(emu, kat):
    st, _, _ = run_emu(emu, encode.statevector_ops(build_circuit(kat)))
    np.testing.assert_allclose(st, cplx(kat["state"]), atol=1e-10, rtol=0)


CASES = [(n, seed, tile, budget) for n, seed, tile, budget in [
    (4, 1, 0, 0), (5, 2, 0, 0), (6, 3, 0, 0), (7, 4, 0, 0), (8, 5, 7, 20), (9, 6, 8, 0), (10, 7, 8, 30),
    (11, 8, 9, 0), (12, 9, 10, 40), (13, 10, 12, 0), (14, 11, 11, 60), (13, 12, 13, 200), (10, 13, 6, 8),
    (9, 14, 5, 1)]]


@pytest.mark.parametrize("n,seed,tile,budget", CASES)
def test_emulated_random_circuits_match_oracle(emu, n, seed, tile, budget):
    c = random_circuit(n, 80, seed, allow_reset=True)
    ops = encode.statevector_ops(c)
    want = orc.sv_evolve(ops)
    got, passes, phases = run_emu(emu, ops, tile=tile, budget=budget)
    assert passes >= 1 and phases >= passes
    np.testing.assert_allclose(got, want, atol=1e-12, rtol=0)


@pytest.mark.parametrize("n,seed", [(3, 21), (2, 22), (1, 23), (9, 24), (12, 25)])
def test_emulated_small_and_c64(emu, n, seed):
    c = random_circuit(n, 40, seed, allow_3q=n >= 3, allow_ctrl=n >= 4)
    ops = encode.statevector_ops(c)
    want = orc.sv_evolve(ops)
    got, _, _ = run_emu(emu, ops)
    np.testing.assert_allclose(got, want, atol=1e-12, rtol=0)
    got64, _, _ = run_emu(emu, ops, precision=_abi.GQ_C64)
    assert np.max(np.abs(got64 - want)) < 5e-5


def test_emulated_qft_and_brickwork(emu):
    from goqu_b200 import workloads
    c = workloads.random_layers_qft(12, layers=6, seed=5)
    ops = encode.statevector_ops(c)
    want = orc.sv_evolve(ops)
    got, passes, _ = run_emu(emu, ops, tile=10)
    np.testing.assert_allclose(got, want, atol=1e-12, rtol=0)
    assert passes < len(ops)  # gates were fused into passes


def _emu_dm(emu, stream, tile=0, budget=0):
    n = stream.num_qubits
    rho = np.zeros(1 << (2 * n), dtype=np.complex128)
    rho[0] = 1
    emu.gqx_emulate_dm.restype = ctypes.c_int
    emu.gqx_emulate_dm.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_abi.gq_op),
                                   ctypes.c_size_t, ctypes.c_int, ctypes.c_int]
    rc = emu.gqx_emulate_dm(n, rho.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                            stream.ptr(), len(stream), tile, budget)
    assert rc == 0, emu.gqx_last_error()
    return rho


@pytest.mark.parametrize("n,seed,tile", [(1, 1, 0), (2, 2, 0), (3, 3, 0), (4, 4, 6), (5, 5, 8), (6, 6, 0)])
def test_emulated_density_matrix_matches_oracle(emu, n, seed, tile):
    from goqu_b200 import noise as N
    c = random_circuit(n, 30, seed, allow_3q=False, allow_ctrl=False, allow_reset=True)
    nm = N.New()
    nm.AddDefaultError(1, N.Depolarizing1Q(0.05))
    nm.AddDefaultError(2, N.Depolarizing2Q(0.05))
    nm.AddGateError("H", N.AmplitudeDamping(0.1))
    ops = encode.density_ops(c, nm)
    want = orc.dm_evolve(ops)
    got = _emu_dm(emu, ops, tile=tile)
    np.testing.assert_allclose(got, want, atol=1e-12, rtol=0)


@pytest.mark.parametrize("kind", ["depol", "amp", "phase", "gad", "thermal", "bitflip", "phaseflip"])
def test_emulated_density_matrix_channel_kinds(emu, kind):
    # population / coherence channels (depolarizing, amplitude, phase and
    # generalized amplitude damping, thermal relaxation, phase flip) take the
    # structured form after their gate; bit flip mixes coherences and keeps
    # the dense superoperator. Both against goqu's Kraus sums.
    from goqu_b200 import noise as N
    ch1 = {"depol": N.Depolarizing1Q(0.07), "amp": N.AmplitudeDamping(0.2), "phase": N.PhaseDamping(0.15),
           "gad": N.GeneralizedAmplitudeDamping(0.3, 0.2), "thermal": N.ThermalRelaxation(50.0, 40.0, 7.0),
           "bitflip": N.BitFlip(0.1), "phaseflip": N.PhaseFlip(0.1)}[kind]
    c = random_circuit(5, 40, 17, allow_3q=False, allow_ctrl=False, allow_reset=True)
    nm = N.New()
    nm.AddDefaultError(1, ch1)
    nm.AddDefaultError(2, N.Depolarizing2Q(0.05) if kind != "bitflip" else N.Custom(
        "bf2", 2, [np.kron(np.reshape(k1, (2, 2)), np.reshape(k2, (2, 2))) for k1 in N.BitFlip(0.1).Kraus()
                   for k2 in N.BitFlip(0.2).Kraus()]))
    ops = encode.density_ops(c, nm)
    np.testing.assert_allclose(_emu_dm(emu, ops), orc.dm_evolve(ops), atol=1e-12, rtol=0)


def test_emulated_noisy_brickwork(emu):
    from goqu_b200 import workloads
    c, nm = workloads.noisy_brickwork(5, layers=4, seed=1)
    ops = encode.density_ops(c, nm)
    np.testing.assert_allclose(_emu_dm(emu, ops), orc.dm_evolve(ops), atol=1e-12, rtol=0)


def _emu_adjoint(emu, circuit, names, x, h, tile=0, budget=0):
    from goqu_b200 import pauli as P
    bindings = {nm: float(x[i]) for i, nm in enumerate(names)}
    stream = encode.statevector_ops(circuit, bindings, names)
    terms = P.to_terms(h)
    grad = np.zeros(len(names))
    energy = ctypes.c_double()
    emu.gqx_emulate_adjoint.restype = ctypes.c_int
    emu.gqx_emulate_adjoint.argtypes = [ctypes.c_int, ctypes.POINTER(_abi.gq_op), ctypes.c_size_t,
                                        ctypes.POINTER(_abi.gq_pauli_term), ctypes.c_size_t, ctypes.c_size_t,
                                        ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_double)]
    rc = emu.gqx_emulate_adjoint(circuit.NumQubits(), stream.ptr(), len(stream),
                                 ctypes.cast(terms, ctypes.POINTER(_abi.gq_pauli_term)), len(terms), len(names),
                                 tile, budget, grad.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 ctypes.byref(energy))
    assert rc == 0, emu.gqx_last_error()
    return energy.value, grad


def _oracle_energy(circuit, names, x, h):
    from goqu_b200 import circuit as ir, pauli as P
    bound = ir.Bind(circuit, {nm: float(x[i]) for i, nm in enumerate(names)})
    st = orc.sv_evolve(encode.statevector_ops(bound))
    return orc.expect_pauli_sum(st, P.to_terms(h)).real


def _oracle_param_shift(circuit, names, x, h):
    import math
    g = np.zeros(len(names))
    for i in range(len(names)):
        xp, xm = x.copy(), x.copy()
        xp[i] += math.pi / 2
        xm[i] -= math.pi / 2
        g[i] = (_oracle_energy(circuit, names, xp, h) - _oracle_energy(circuit, names, xm, h)) / 2
    return g


@pytest.mark.parametrize("n,layers,tile", [(4, 2, 0), (6, 2, 0), (7, 3, 5), (9, 2, 6)])
def test_emulated_adjoint_matches_parameter_shift(emu, n, layers, tile):
    from goqu_b200 import workloads
    c, names = workloads.hardware_efficient_ansatz(n, layers)
    h = workloads.ising_hamiltonian(n)
    x = np.random.default_rng(n).uniform(0, 2 * np.pi, len(names))
    e, g = _emu_adjoint(emu, c, names, x, h, tile=tile)
    assert abs(e - _oracle_energy(c, names, x, h)) < 1e-12
    np.testing.assert_allclose(g, _oracle_param_shift(c, names, x, h), atol=1e-10, rtol=0)


def test_emulated_adjoint_general_gates(emu):
    # U3 / CP / RXX / RZZ / RX with expressions (chain rule) and shared parameters
    from goqu_b200 import circuit as ir, param as prm, pauli as P
    th = prm.NewVector("t", 5)
    b = ir.Builder("g", 5)
    b.H(0).H(1).H(2)
    b.SymU3(th.At(0), prm.Mul(2.0, th.At(1)), th.At(2), 3)
    b.SymCP(th.At(3), 0, 4).SymRXX(prm.Add(th.At(4), 0.3), 1, 2).SymRZZ(th.At(0), 2, 3)
    b.SymRX(prm.Neg(th.At(1)), 4).CNOT(3, 0).SymRY(th.At(2), 1)
    c = b.Build()
    names = ir.FreeParameters(c)
    h = P.NewPauliSum([P.NewPauliString(0.7, {0: P.Z, 3: P.X}, 5), P.NewPauliString(-0.4, {1: P.Y, 2: P.Y}, 5),
                       P.NewPauliString(0.25, {4: P.X}, 5)])
    x = np.random.default_rng(3).uniform(0, 2 * np.pi, len(names))
    e, g = _emu_adjoint(emu, c, names, x, h)
    fd = np.zeros(len(names))
    for i in range(len(names)):
        xp, xm = x.copy(), x.copy()
        xp[i] += 1e-5
        xm[i] -= 1e-5
        fd[i] = (_oracle_energy(c, names, xp, h) - _oracle_energy(c, names, xm, h)) / 2e-5
    assert abs(e - _oracle_energy(c, names, x, h)) < 1e-12
    np.testing.assert_allclose(g, fd, atol=1e-7, rtol=0)


@pytest.mark.parametrize("n,seed,tile", [(5, 31, 0), (8, 32, 7), (11, 33, 9), (13, 34, 11)])
def test_emulated_dense_fusion_matches_oracle(emu, n, seed, tile):
    # GQ_OPT_FUSE_DENSE: runs of register-local gates folded into dense blocks
    c = random_circuit(n, 120, seed, allow_reset=True)
    ops = encode.statevector_ops(c)
    want = orc.sv_evolve(ops)
    st = np.zeros(1 << n, dtype=np.complex128)
    st[0] = 1
    emu.gqx_emulate_sv_fused.restype = ctypes.c_int
    emu.gqx_emulate_sv_fused.argtypes = emu.gqx_emulate_sv.argtypes
    p, q = ctypes.c_int64(), ctypes.c_int64()
    rc = emu.gqx_emulate_sv_fused(n, 0, st.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  ops.ptr(), len(ops), tile, 400, ctypes.byref(p), ctypes.byref(q))
    assert rc == 0
    np.testing.assert_allclose(st, want, atol=1e-12, rtol=0)


def test_qaoa_layers_fuse_into_pair_sums(emu):
    # QAOA: the RZZ(gamma) of a layer fold into K_PAIRSUM ops (one table lookup
    # per amplitude); the result and the adjoint gradient stay exact
    from goqu_b200 import pauli as P
    emu.gqx_schedule_stats.restype = ctypes.c_int
    emu.gqx_schedule_stats.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_abi.gq_op), ctypes.c_size_t,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
    for c, names, h, x in workloads.qaoa_batch(4, seed=17, n_values=(8, 10, 12)):
        n = c.NumQubits()
        bound = ir.Bind(c, {nm: float(x[i]) for i, nm in enumerate(names)})
        ops = encode.statevector_ops(bound)
        out = (ctypes.c_int64 * 5)()
        assert emu.gqx_schedule_stats(n, 0, ops.ptr(), len(ops), 0, 0, 0, out) == 0
        assert out[4] >= 1  # fused
        got, _, _ = run_emu(emu, ops)
        np.testing.assert_allclose(got, orc.sv_evolve(ops), atol=1e-12, rtol=0)
        e, g = _emu_adjoint(emu, c, names, x, h)
        assert abs(e - _oracle_energy(c, names, x, h)) < 1e-12
        for i in range(len(names)):
            xp, xm = np.array(x, float), np.array(x, float)
            xp[i] += 1e-5
            xm[i] -= 1e-5
            fd = (_oracle_energy(c, names, xp, h) - _oracle_energy(c, names, xm, h)) / 2e-5
            assert abs(g[i] - fd) < 1e-6


def test_adjoint_checkpoints_fit_free_memory(emu):
    """The automatic checkpoint count of the adjoint (engine: after
    cudaMemGetInfo) never asks for more stored states than the free memory
    holds: a 33-qubit complex64 circuit of 2000 ops wants 8 segments, i.e. 7
    stored 64 GiB states, and gets what fits, down to none."""
    f = emu.gqx_adjoint_segments
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]
    gib = 1 << 30
    head = 256 << 20  # kept free for program and reduction buffers
    s33 = 64 * gib  # one 33-qubit complex64 state
    assert f(0, 1, 2000, s33, 1000 * gib) == 8
    assert f(0, 1, 2000, s33, 3 * s33 + head) == 4  # three stored states fit
    assert f(0, 1, 2000, s33, 3 * s33 + head - 1) == 3
    assert f(0, 1, 2000, s33, s33) == 1  # no room: no checkpoints, no failure
    assert f(0, 1, 2000, s33, 0) == 1
    # complex128 and short circuits take none; small states are unaffected
    assert f(0, 0, 2000, s33, 1000 * gib) == 1
    assert f(0, 1, 256, 1 << 20, 1000 * gib) == 1
    assert f(0, 1, 600, 1 << 20, 8 * gib) == 4
    # an explicit request is kept (capped at the op count only)
    assert f(5, 1, 2000, s33, 0) == 5
    assert f(5, 0, 3, s33, 0) == 3


# ---- passes from the reset state skip the tiles that are still zero ---------
# (SchedOptions::support0, GQ_OPT_ZERO_TILES): a pass launches only the CTAs
# whose outer qubits lie in the support reached so far.

def _with_support(emu, support0, fn):
    emu.gqx_set_support0.argtypes = [ctypes.c_uint64]
    emu.gqx_last_ctas.restype = ctypes.c_int64
    emu.gqx_set_support0(support0)
    try:
        return fn(), emu.gqx_last_ctas()
    finally:
        emu.gqx_set_support0(ctypes.c_uint64(~0 & (2 ** 64 - 1)))


@pytest.mark.parametrize("n,seed,tile,budget", [(8, 31, 5, 8), (10, 32, 6, 0), (12, 33, 7, 16), (13, 34, 6, 4),
                                                (11, 35, 9, 0)])
def test_zero_tile_skip_matches_oracle(emu, n, seed, tile, budget):
    # controls and diagonals on qubits outside the support, resets, 3-qubit gates
    c = random_circuit(n, 90, seed, allow_reset=True)
    ops = encode.statevector_ops(c)
    want = orc.sv_evolve(ops)
    full, ctas_full = _with_support(emu, 2 ** 64 - 1, lambda: run_emu(emu, ops, tile=tile, budget=budget)[0])
    got, ctas = _with_support(emu, 0, lambda: run_emu(emu, ops, tile=tile, budget=budget)[0])
    # the short passes take larger budgets, so the schedule (and the rounding) may differ
    np.testing.assert_allclose(got, full, atol=1e-13, rtol=0)
    np.testing.assert_allclose(got, want, atol=1e-12, rtol=0)
    assert ctas < ctas_full


def test_zero_tile_skip_late_support():
    # a circuit that touches qubit 0 only: every pass runs one tile
    from goqu_b200 import gate as G
    c = ir.Circuit("narrow", 12, 0, [ir.Operation(G.H, [0]), ir.Operation(G.RZ(0.3), [11]),
                                     ir.Operation(G.CNOT, [11, 0]), ir.Operation(G.RX(0.2), [0])])
    ops = encode.statevector_ops(c)
    h = ctypes.CDLL(EMU)
    h.gqx_emulate_sv.restype = ctypes.c_int
    h.gqx_emulate_sv.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(_abi.gq_op), ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    h.gqx_last_error.restype = ctypes.c_char_p
    got, ctas = _with_support(h, 0, lambda: run_emu(h, ops, tile=4)[0])
    np.testing.assert_allclose(got, orc.sv_evolve(ops), atol=1e-14, rtol=0)
    assert ctas == 1  # qubit 11 stays 0, so its control and diagonal act on zeros only


def test_zero_tile_skip_headline_openers(emu):
    # 28 qubits, 40 U3+CNOT brickwork layers + QFT28, 12-qubit tiles: the
    # first pass runs one CTA and the second 2^9 of 2^16; the rest are full.
    # The two short passes take larger budgets (64x), so they absorb more of
    # the opening layers and the full passes that follow carry less
    f = emu.gqx_schedule_passes
    f.restype = ctypes.c_int64
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_abi.gq_op), ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_int64), ctypes.c_int64]
    c = workloads.random_layers_qft(28, 40, 2028)
    ops = encode.statevector_ops(c)
    out_full = (ctypes.c_int64 * (5 * 400))()
    out = (ctypes.c_int64 * (5 * 400))()
    (np_full, _) = _with_support(emu, 2 ** 64 - 1, lambda: f(28, 0, ops.ptr(), len(ops), 12, 0, out_full, 400))
    (np_zero, _) = _with_support(emu, 0, lambda: f(28, 0, ops.ptr(), len(ops), 12, 0, out, 400))
    assert np_zero <= np_full
    bits = [out[5 * i + 4] for i in range(np_zero)]
    assert [out_full[5 * i + 4] for i in range(np_full)] == [16] * np_full
    assert bits[0] == 0 and bits[1] == 9 and all(b == 16 for b in bits[2:])
    cost = [out[5 * i + 2] for i in range(np_zero)]
    cost_full = [out_full[5 * i + 2] for i in range(np_full)]
    assert sum(cost) == sum(cost_full)  # the same gates, placed differently
    assert cost[0] > cost_full[0] and max(cost[2:]) <= max(cost_full)
