"""Dynamic circuits: the shot-group walk of goqu_b200.dynamic against a
per-shot restatement of RunDynamic (tests/dyn_ref.py), on the CPU.

The walk runs here over oracle states (a numpy backend with measureQubit's
P(0) and collapse) so its grouping, splitting and classical control flow are
checked without a device: counts must equal the per-shot loop's exactly for
the same uniforms, and the final groups' states must equal those shots'.
"""
import numpy as np
import pytest

from goqu_b200 import circuit as ir, dynamic, encode
from oracle import binding as orc

import dyn_ref


class OracleBackend:
    keeps_delays = False

    def __init__(self, n):
        self.n = n

    def fresh(self):
        return orc.zero_state(self.n)

    def copy(self, s):
        return s.copy()

    def release(self, s):
        pass

    def apply(self, s, ops):
        stream = encode.statevector_ops(ir.Circuit("", self.n, 0, ops))
        if len(stream):
            orc.sv_apply(s, stream)

    def prob0(self, s, q):
        idx = np.arange(s.size)
        a = s[((idx >> q) & 1) == 0]
        return float(np.sum(a.real * a.real + a.imag * a.imag))

    def collapse(self, s, q, outcome, p0):
        norm = np.sqrt(p0) if outcome == 0 else np.sqrt(1 - p0)
        if norm < 1e-15:
            return
        keep = ((np.arange(s.size) >> q) & 1) == outcome
        s[keep] *= 1.0 / norm
        s[~keep] = 0


@pytest.mark.parametrize("name", sorted(dyn_ref.CIRCUITS))
def test_group_walk_matches_per_shot_loop(name):
    c = dyn_ref.CIRCUITS[name]()
    assert c.IsDynamic()
    shots = 64
    u = np.random.default_rng(7).random((shots, 64))
    want, last = dyn_ref.run_dynamic(c, shots, u)
    groups = dynamic.run_groups(OracleBackend(c.NumQubits()), c, shots, uniforms=u)
    got = {}
    for g in groups:
        key = dynamic.bitstring(g.clbits)
        got[key] = got.get(key, 0) + len(g.shots)
        if (g.shots == shots - 1).any():
            np.testing.assert_allclose(g.state, last, atol=1e-12, rtol=0)
    assert got == want
    assert sum(got.values()) == shots
    assert len(groups) <= shots


def test_measureqbit_restatement():
    # outcome rule and renormalisation on a Bell pair
    st = orc.zero_state(2)
    from goqu_b200 import gate as G
    orc.sv_apply(st, encode.statevector_ops(ir.Circuit("", 2, 0, [ir.Operation(G.H, [0]),
                                                                   ir.Operation(G.CNOT, [0, 1])])))
    s1 = st.copy()
    assert orc.sv_measure(s1, 0, 0.49) == 0
    np.testing.assert_allclose(s1, [1, 0, 0, 0], atol=1e-15)
    s2 = st.copy()
    assert orc.sv_measure(s2, 0, 0.51) == 1
    np.testing.assert_allclose(s2, [0, 0, 0, 1], atol=1e-15)


def test_uniforms_shape_checked():
    c = dyn_ref.teleport()
    with pytest.raises(ValueError):
        dynamic.run_groups(OracleBackend(3), c, 4, uniforms=np.zeros((3, 8)))
    with pytest.raises(ValueError):
        dynamic.run_groups(OracleBackend(3), c, 0)


class OracleDMBackend(OracleBackend):
    keeps_delays = True

    def __init__(self, n, nm):
        self.n, self.nm = n, nm

    def fresh(self):
        return orc.dm_zero(self.n)

    def apply(self, s, ops):
        stream = encode.density_ops(ir.Circuit("", self.n, 0, ops), self.nm)
        if len(stream):
            orc.dm_apply(s, stream)

    def prob0(self, s, q):
        d = np.real(s.reshape(1 << self.n, 1 << self.n).diagonal())
        return float(np.sum(d[((np.arange(d.size) >> q) & 1) == 0]))

    def collapse(self, s, q, outcome, p0):
        p = p0 if outcome == 0 else 1 - p0
        if p < 1e-15:
            return
        dim = 1 << self.n
        r = (np.arange(dim * dim) // dim >> q) & 1
        c = (np.arange(dim * dim) % dim >> q) & 1
        keep = (r == outcome) & (c == outcome)
        s[keep] *= 1.0 / p
        s[~keep] = 0


@pytest.mark.parametrize("which", ["noisy", "teleport", "reset"])
def test_density_matrix_group_walk_matches_per_shot_loop(which):
    nm = dyn_ref.noisy_model()
    c = {"noisy": dyn_ref.noisy_dynamic, "teleport": dyn_ref.teleport, "reset": dyn_ref.reset_and_reuse}[which]()
    shots = 48
    u = np.random.default_rng(5).random((shots, 16))
    want, last = dyn_ref.run_dynamic_dm(c, nm, shots, u)
    groups = dynamic.run_groups(OracleDMBackend(c.NumQubits(), nm), c, shots, uniforms=u)
    got = {}
    for g in groups:
        key = dynamic.bitstring(g.clbits)
        got[key] = got.get(key, 0) + len(g.shots)
        if (g.shots == shots - 1).any():
            np.testing.assert_allclose(g.state, last, atol=1e-12, rtol=0)
    assert got == want
