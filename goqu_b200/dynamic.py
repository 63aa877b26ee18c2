"""Dynamic circuits (mid-circuit measurement, feed-forward).

goqu runs these per shot on the CPU (sim/statevector/dynamic.go:14-230). The
device engine does not execute them yet; Run raises instead of silently
falling back to a host simulator.
"""


def run_dynamic(sim, circuit, shots, rng=None):
    raise NotImplementedError("statevector: dynamic circuits are not supported by the device engine yet")
