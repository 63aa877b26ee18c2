"""The optimisation loop (gq_sv_adjoint_template, gq_sv_minimize_adam,
vqe.Run): the library rebinds goqu's parameterized gates from theta and
keeps the loop on its side. Gradients must equal the host-encoded adjoint
gradient and central differences of the oracle energy; the Adam loop must
follow goqu's Adam (algorithm/optim/adam.go:51-140) step for step, as the
Python restatement does with host-encoded adjoint gradients."""
import ctypes

import numpy as np
import pytest

from goqu_b200 import _abi, circuit as ir, encode, gradient, optim, param as prm, pauli as P, statevector, vqe
from goqu_b200 import workloads
from oracle import gradient as og

pytestmark = pytest.mark.gpu
_D = ctypes.POINTER(ctypes.c_double)


def template_grad(sim, c, names, h, x):
    t = encode.param_template(c, names, x)
    terms = P.to_terms(h)
    g = np.empty(len(names))
    e = ctypes.c_double()
    _abi.check(_abi.lib().gq_sv_adjoint_template(
        sim.handle, t.ops.ptr(), len(t.ops), t.pgate_ptr(), len(t.pgates), np.asarray(x, float).ctypes.data_as(_D),
        len(names), ctypes.cast(terms, ctypes.POINTER(_abi.gq_pauli_term)), len(terms), g.ctypes.data_as(_D),
        ctypes.byref(e)))
    return e.value, g


def every_family(n=4):
    t = prm.NewVector("t", 8)
    b = ir.Builder("fam", n)
    for q in range(n):
        b.H(q)
    b.SymU3(t.At(0), prm.Mul(2.0, t.At(1)), prm.Add(t.At(2), 0.4), 0).SymRX(t.At(3), 1).SymRY(prm.Neg(t.At(4)), 2)
    b.SymRZ(t.At(5), 3).SymCP(t.At(6), 0, 1).SymRXX(t.At(7), 1, 2).SymRYY(t.At(0), 2, 3).SymRZZ(t.At(1), 3, 0)
    b.SymPhase(t.At(2), 1).CNOT(0, 2)
    b.Apply(prm.SymU2(t.At(3), t.At(4)), 2).Apply(prm.SymRot(t.At(5), t.At(6), t.At(7)), 3)
    b.Apply(prm.SymFSim(t.At(0), t.At(5)), 1, 3).Apply(prm.SymPSwap(t.At(2)), 0, 2)
    b.Apply(prm.SymU1(prm.Div(t.At(6), 2.0)), 1).Apply(prm.SymGlobalPhase(t.At(7)), 0)
    return b.Build(), t.Names()


def test_template_gradient_every_family():
    c, names = every_family()
    h = P.NewPauliSum([P.NewPauliString(0.7, {0: P.Z, 3: P.X}, 4), P.NewPauliString(-0.4, {1: P.Y, 2: P.Y}, 4),
                       P.NewPauliString(0.25, {2: P.X}, 4)])
    x = np.random.default_rng(3).uniform(-3, 3, len(names))
    sim = statevector.New(4)
    e, g = template_grad(sim, c, names, h, x)
    e2, g2 = gradient.AdjointEvaluator(c, h, names)(x)
    assert abs(e - e2) < 1e-12 and abs(e - og.energy(c, names, x, h)) < 1e-12
    assert np.max(np.abs(g - g2)) < 1e-9  # host derivatives use 5-point stencils for U2, U3, Rot, FSim, PSwap
    fd = og.parameter_shift(c, names, x, h, shift=1e-6, denom=2e-6)
    assert np.max(np.abs(g - fd)) < 1e-7
    sim.Close()


@pytest.mark.parametrize("which", ["hea", "qaoa"])
def test_template_matches_host_encoded_adjoint(which):
    if which == "hea":
        c, names = workloads.hardware_efficient_ansatz(12, 4)
        h = workloads.ising_hamiltonian(12)
        x = np.random.default_rng(1).uniform(0, 2 * np.pi, len(names))
    else:
        c, names, h, x = workloads.qaoa_batch(1, seed=5, n_values=(12,), p_range=(3, 3))[0]
    sim = statevector.New(c.NumQubits())
    e, g = template_grad(sim, c, names, h, x)
    e2, g2 = gradient.AdjointEvaluator(c, h, names)(x)
    assert abs(e - e2) < 1e-12 and np.max(np.abs(g - g2)) < 1e-12
    sim.Close()


def test_adam_loop_follows_goqus_adam():
    c, names = workloads.hardware_efficient_ansatz(6, 2)
    h = workloads.ising_hamiltonian(6)
    x0 = np.random.default_rng(2).uniform(0, 2 * np.pi, len(names))
    adam = optim.Adam(LR=0.05)
    opts = optim.Options(MaxIter=40)
    r_dev, hist = vqe.minimize_adam_on_device(c, h, names, x0, adam, opts)
    ev = gradient.AdjointEvaluator(c, h, names)
    hist_host = []

    def f(x):
        v = ev(x)[0]
        hist_host.append(v)
        return v

    r_host = adam.Minimize(f, x0, lambda x: ev(x)[1], opts)
    assert (r_dev.Iterations, r_dev.FuncEvals, r_dev.GradEvals, r_dev.Converged) == \
        (r_host.Iterations, r_host.FuncEvals, r_host.GradEvals, r_host.Converged)
    assert np.max(np.abs(r_dev.X - r_host.X)) < 1e-9
    assert np.max(np.abs(np.array(hist) - np.array(hist_host))) < 1e-9
    assert hist[-1] < hist[0]


def test_vqe_run_reaches_the_ground_energy():
    n = 4
    c, names = workloads.hardware_efficient_ansatz(n, 3)
    h = workloads.ising_hamiltonian(n)
    # exact ground energy from the dense Hamiltonian: (P psi)[i ^ x] = i^nY (-1)^popcount(i & z) psi[i]
    mat = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    terms = P.to_terms(h)
    idx = np.arange(1 << n)
    for t in terms:
        x, z = int(t.x_mask), int(t.z_mask)
        ny = bin(x & z).count("1")
        sign = np.array([(-1) ** bin(i & z).count("1") for i in idx]) * (1j ** ny)
        mat[idx ^ x, idx] += complex(t.coeff_re, t.coeff_im) * sign
    e0 = float(np.min(np.linalg.eigvalsh(mat)))
    res = vqe.Run(vqe.Config(Hamiltonian=h, Ansatz=c, Optimizer=optim.Adam(LR=0.05),
                             InitialParams=np.random.default_rng(4).uniform(0, 1, len(names)),
                             Options=optim.Options(MaxIter=1500, FunTol=1e-12)))
    assert res.Energy < e0 + 0.05 * abs(e0)
    assert len(res.History) == res.NumEvals
