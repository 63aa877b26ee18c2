"""Parameter templates on the CPU: the library's matrices for goqu's
parameterized gates (circuit/gate/parameterized.go:91-564) equal the host
gate constructors, its derivatives equal finite differences and the
symbolic gates' own derivatives (circuit/param/gate.go), the affine
analysis of parameter expressions, the C layouts of the new structs, and
the Adam restatement (algorithm/optim/adam.go) on a quadratic."""
import ctypes
import math
import os
import subprocess

import numpy as np
import pytest

from goqu_b200 import _abi, encode, gate as G, optim, param as prm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EMU = os.path.join(ROOT, "goqu_b200", "libgqb200_emu.so")

FAMILIES = {  # family code: (angle count, host constructor)
    "RX": (1, G.RX), "RY": (1, G.RY), "RZ": (1, G.RZ), "P": (1, G.Phase), "U1": (1, G.U1), "U2": (2, G.U2),
    "U3": (3, G.U3), "Rot": (3, G.Rot), "CP": (1, G.CP), "RXX": (1, G.RXX), "RYY": (1, G.RYY), "RZZ": (1, G.RZZ),
    "FSim": (2, G.FSim), "PSwap": (1, G.PSwap), "GlobalPhase": (1, G.GlobalPhase),
}


@pytest.fixture(scope="module")
def emu():
    if not os.path.exists(EMU):
        from goqu_b200 import build
        build.build_emulator()
    h = ctypes.CDLL(EMU)
    h.gqx_param_gate.restype = ctypes.c_int
    h.gqx_param_gate.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_double)]
    return h


def lib_matrix(emu, fam, angles, k=-1):
    a = np.ascontiguousarray(angles, dtype=np.float64)
    out = np.zeros(32, dtype=np.complex128)
    n = emu.gqx_param_gate(_abi.GQ_PG[fam], a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size, k,
                           out.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert n > 0
    return out[:n]


@pytest.mark.parametrize("fam", sorted(FAMILIES))
def test_matrices_and_derivatives(emu, fam):
    na, ctor = FAMILIES[fam]
    rng = np.random.default_rng(len(fam))
    for _ in range(5):
        ang = rng.uniform(-7, 7, na)
        want = np.asarray(ctor(*ang).Matrix(), dtype=np.complex128).reshape(-1)
        assert np.max(np.abs(lib_matrix(emu, fam, ang) - want)) <= 1e-15
        for k in range(na):
            h = 1e-6
            ap, am = ang.copy(), ang.copy()
            ap[k] += h
            am[k] -= h
            fd = (np.asarray(ctor(*ap).Matrix()).reshape(-1) - np.asarray(ctor(*am).Matrix()).reshape(-1)) / (2 * h)
            assert np.max(np.abs(lib_matrix(emu, fam, ang, k) - fd)) <= 1e-8, (fam, k)


def test_derivatives_match_symbolic_gates(emu):
    # the symbolic gates' MatrixDerivative (closed forms, 5-point stencils)
    t = prm.NewVector("t", 3)
    x = {"t[0]": 0.7, "t[1]": -1.3, "t[2]": 2.1}
    for sym, fam, na in ((prm.SymU3, "U3", 3), (prm.SymRot, "Rot", 3), (prm.SymRXX, "RXX", 1), (prm.SymCP, "CP", 1)):
        g = sym(*[t.At(k) for k in range(na)])
        ang = [x[f"t[{k}]"] for k in range(na)]
        for k in range(na):
            want = np.asarray(g.MatrixDerivative(f"t[{k}]", x)).reshape(-1)
            assert np.max(np.abs(lib_matrix(emu, fam, ang, k) - want)) <= 1e-9


def test_affine_expressions():
    idx = {"a": 0, "b": 1}
    a, b = prm.New("a"), prm.New("b")
    assert encode._affine(prm.Mul(2.0, a), idx) == (0, 2.0, 0.0)
    assert encode._affine(prm.Add(prm.Mul(a, 3.0), 0.5), idx) == (0, 3.0, 0.5)
    assert encode._affine(prm.Neg(prm.Sub(a, 1.0)), idx) == (0, -1.0, 1.0)
    assert encode._affine(prm.Div(b, 4.0), idx) == (1, 0.25, 0.0)
    assert encode._affine(prm.Literal(1.5), idx) == (-1, 0.0, 1.5)
    assert encode._affine(prm.Add(a, b), idx) is None      # two parameters in one angle
    assert encode._affine(prm.Mul(a, a), idx) is None      # not affine
    assert encode._affine(prm.New("c"), idx) is None       # not a listed parameter


def test_struct_layouts_against_the_c_compiler(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "gqb200.h"\nint main(void) {\n'
                   '  printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(gq_op), sizeof(gq_param_gate),\n'
                   '         offsetof(gq_param_gate, scale), sizeof(gq_adam_options), offsetof(gq_adam_options, fun_tol),\n'
                   '         sizeof(gq_optim_result), sizeof(gq_sweep_point), sizeof(gq_stats));\n  return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_abi.gq_op), ctypes.sizeof(_abi.gq_param_gate), _abi.gq_param_gate.scale.offset,
            ctypes.sizeof(_abi.gq_adam_options), _abi.gq_adam_options.fun_tol.offset,
            ctypes.sizeof(_abi.gq_optim_result), ctypes.sizeof(_abi.gq_sweep_point), ctypes.sizeof(_abi.gq_stats)]
    assert got == want


def test_adam_on_a_quadratic():
    target = np.array([1.0, -2.0, 0.5])
    f = lambda x: float(np.sum((x - target) ** 2))  # noqa: E731
    g = lambda x: 2 * (x - target)  # noqa: E731
    r = optim.Adam(LR=0.05).Minimize(f, np.zeros(3), g, optim.Options(MaxIter=3000, FunTol=1e-14))
    assert r.Converged and np.max(np.abs(r.X - target)) < 1e-4
    assert r.FuncEvals == r.Iterations + 1 and r.GradEvals == r.Iterations
    with pytest.raises(ValueError, match="gradient function required"):
        optim.Adam().Minimize(f, np.zeros(3), None)


def test_reverse_plans_do_not_depend_on_the_angles(emu):
    # G = dU U^dagger of a rotation is -i/2 times a Pauli string at every
    # angle; the reverse passes' kernel keys must not change with theta, or
    # an optimisation loop would compile new kernels at every step
    from goqu_b200 import workloads
    f = emu.gqx_adjoint_plan_digest
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(_abi.gq_op), ctypes.c_size_t, ctypes.c_size_t,
                  ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int64)]
    c, names = workloads.hardware_efficient_ansatz(20, 10)
    digests = set()
    for seed in range(4):
        x = np.random.default_rng(seed).uniform(0, 2 * np.pi, len(names))
        s = encode.statevector_ops(c, {nm: float(x[i]) for i, nm in enumerate(names)}, names)
        d, n = ctypes.c_uint64(), ctypes.c_int64()
        assert f(20, _abi.GQ_C128, s.ptr(), len(s), len(names), ctypes.byref(d), ctypes.byref(n)) == 0
        digests.add(d.value)
    assert len(digests) == 1 and n.value > 10
