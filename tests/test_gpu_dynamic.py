"""Dynamic circuits on the device (GPU): Sim.Run on a dynamic circuit walks
shot groups over device states (gq_sv_prob0 / gq_sv_collapse /
gq_sv_copy_state). Counts must equal the per-shot restatement of RunDynamic
(tests/dyn_ref.py) for the same uniforms, and the simulator is left in the
last shot's final state (within 1e-12, complex128).
"""
import ctypes

import numpy as np
import pytest

from goqu_b200 import _abi, dynamic, statevector

import dyn_ref

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(dyn_ref.CIRCUITS))
def test_counts_match_per_shot_loop(name):
    c = dyn_ref.CIRCUITS[name]()
    shots = 128
    u = np.random.default_rng(11).random((shots, 64))
    want, last = dyn_ref.run_dynamic(c, shots, u)
    sim = statevector.New(c.NumQubits())
    got = dynamic.run_dynamic(sim, c, shots, uniforms=u)
    assert got == want
    np.testing.assert_allclose(sim.StateVector(), last, atol=1e-12, rtol=0)


def test_run_dispatches_dynamic_circuits():
    c = dyn_ref.teleport()
    sim = statevector.New(3)
    counts = sim.Run(c, 200, rng=np.random.default_rng(3))
    assert sum(counts.values()) == 200 and all(len(k) == 3 for k in counts)


def test_measure_entry_point_and_copy():
    from goqu_b200 import circuit as ir
    sim = statevector.New(2)
    sim.Evolve(ir.Builder("bell", 2).H(0).CNOT(0, 1).Build())
    other = statevector.New(2)
    _abi.check(_abi.lib().gq_sv_copy_state(other.handle, sim.handle))
    out = ctypes.c_int()
    _abi.check(_abi.lib().gq_sv_measure(sim.handle, 0, 0.75, ctypes.byref(out)))
    assert out.value == 1
    np.testing.assert_allclose(sim.StateVector(), [0, 0, 0, 1], atol=1e-15)
    _abi.check(_abi.lib().gq_sv_measure(other.handle, 1, 0.25, ctypes.byref(out)))
    assert out.value == 0
    np.testing.assert_allclose(other.StateVector(), [1, 0, 0, 0], atol=1e-15)
    with pytest.raises(_abi.GQError):
        _abi.check(_abi.lib().gq_sv_measure(sim.handle, 2, 0.5, ctypes.byref(out)))


def test_wide_state_mid_circuit_measurement():
    # 20 qubits: the same walk on a state the tile passes (and specialised kernels) run
    c = dyn_ref.random_mid_circuit(20, 3, 5)
    shots = 16
    u = np.random.default_rng(2).random((shots, 40))
    want, last = dyn_ref.run_dynamic(c, shots, u)
    sim = statevector.New(20)
    assert dynamic.run_dynamic(sim, c, shots, uniforms=u) == want
    np.testing.assert_allclose(sim.StateVector(), last, atol=1e-12, rtol=0)


@pytest.mark.parametrize("which", ["noisy", "teleport", "reset"])
def test_density_matrix_counts_match_per_shot_loop(which):
    from goqu_b200 import densitymatrix
    nm = dyn_ref.noisy_model()
    c = {"noisy": dyn_ref.noisy_dynamic, "teleport": dyn_ref.teleport, "reset": dyn_ref.reset_and_reuse}[which]()
    shots = 64
    u = np.random.default_rng(13).random((shots, 16))
    want, last = dyn_ref.run_dynamic_dm(c, nm, shots, u)
    dm = densitymatrix.New(c.NumQubits()).WithNoise(nm)
    assert dynamic.run_dynamic_dm(dm, c, shots, uniforms=u) == want
    np.testing.assert_allclose(dm.DensityMatrix(), last, atol=1e-12, rtol=0)
    assert sum(dm.Run(c, 50, rng=np.random.default_rng(1)).values()) == 50
