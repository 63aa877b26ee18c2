"""The exact sampler's O(1) rule (goqu_b200/csrc/kernels.cuh, k_chunk_steps /
k_chunk_walk), restated in numpy and checked against the sequential FP64 sum
that goqu's sampleIndex computes (sim/statevector/sim.go:288-298).

Inside one binade [2^e, 2^(e+1)) each addition s + p rounds to the grid
2^(e-52), so s advances by round-to-nearest(p / 2^(e-52)) steps, independent
of s unless p / 2^(e-52) has fraction exactly 1/2. A run of probabilities
without such a tie whose sum stays in the binade therefore ends at
s + (sum of steps) * 2^(e-52), exactly. The kernels take chunks (2048
elements) and sub-chunks (64) this way and sum the rest element by element.
"""
import numpy as np


def steps_rule(s, p):
    """(taken, s_end) for the run p starting at s, by the O(1) rule."""
    if not s > 2.0 ** -1000:
        return False, None
    e = np.frexp(s)[1] - 1
    lim = 2.0 ** (e + 1)
    if not s + p.sum() < lim * (1.0 - 2.0 ** -30):
        return False, None
    q = np.ldexp(p, 52 - e)
    f = np.floor(q)
    fr = q - f
    if np.any(fr == 0.5):
        return False, None
    k = int(f.astype(np.int64).sum() + np.count_nonzero(fr > 0.5))
    sn = s + np.ldexp(float(k), e - 52)
    return (sn < lim), sn


def sequential(s, p):
    for v in p:
        s = s + v  # one IEEE double addition per element, in order
    return s


def test_rule_matches_sequential_sum():
    rng = np.random.default_rng(11)
    taken = 0
    for trial in range(4000):
        e0 = int(rng.integers(-40, 0))
        s = float(np.ldexp(1.0 + rng.random(), e0))          # a start in binade e0
        scale = float(np.ldexp(1.0, e0 - int(rng.integers(3, 30))))
        p = rng.exponential(scale, 64)                        # Porter-Thomas-like probabilities
        if trial % 5 == 0:
            p[int(rng.integers(64))] = 0.0
        ok, sn = steps_rule(s, p)
        if ok:
            taken += 1
            assert sn == sequential(s, p)
    assert taken > 2000


def test_ties_and_binade_crossings_are_not_taken():
    e = -10
    s = 2.0 ** e
    ulp = 2.0 ** (e - 52)
    p = np.full(64, 3.0 * ulp)
    p[7] = 2.5 * ulp  # an exact half step: its rounding depends on the parity of s
    assert not steps_rule(s, p)[0]
    p = np.full(64, 2.0 ** e / 40)  # the run ends above 2^(e+1)
    assert not steps_rule(s, p)[0]
    assert not steps_rule(0.0, np.full(64, 1e-3))[0]
