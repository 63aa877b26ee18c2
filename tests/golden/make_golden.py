"""Writes tests/golden/kats.json: the known-answer tests of goqu's own test
suite for the simulator path, restated as data.

Each entry names the reference test it comes from (file:line in
github.com/splch/goqu), the circuit (gate name, qubits, parameters) and the
expected result exactly as that test asserts it (tolerance 1e-10, the
reference's `eps`). Run:  python tests/golden/make_golden.py
"""
import json
import math
import os

S2 = 1 / math.sqrt(2)
PI = math.pi


def c(re, im=0.0):
    return [re, im]


def state(*amps):
    return [a if isinstance(a, list) else c(a) for a in amps]


def basis(n, idx):
    v = [c(0.0)] * (1 << n)
    v = list(v)
    v[idx] = c(1.0)
    return v


KATS = [
    # --- statevector: sim/statevector/sim_test.go ---------------------------
    dict(name="bell", ref="sim/statevector/sim_test.go:15-34", n=2,
         ops=[["H", [0]], ["CNOT", [0, 1]]], state=state(S2, 0, 0, S2)),
    dict(name="ghz3", ref="sim/statevector/sim_test.go:36-55", n=3,
         ops=[["H", [0]], ["CNOT", [0, 1]], ["CNOT", [1, 2]]], state=state(S2, 0, 0, 0, 0, 0, 0, S2)),
    dict(name="x", ref="sim/statevector/sim_test.go:57-70", n=1, ops=[["X", [0]]], state=state(0, 1)),
    dict(name="h", ref="sim/statevector/sim_test.go:72-86", n=1, ops=[["H", [0]]], state=state(S2, S2)),
    dict(name="hh", ref="sim/statevector/sim_test.go:88-100", n=1, ops=[["H", [0]], ["H", [0]]], state=state(1, 0)),
    dict(name="qft3_zero", ref="sim/statevector/sim_test.go:102-133", n=3,
         ops=[["H", [0]], ["CP", [1, 0], [PI / 2]], ["CP", [2, 0], [PI / 4]], ["H", [1]],
              ["CP", [2, 1], [PI / 2]], ["H", [2]]], abs_all=1 / math.sqrt(8)),
    dict(name="toffoli", ref="sim/statevector/sim_test.go:169-200", n=3,
         ops=[["X", [1]], ["X", [2]], ["CCX", [2, 1, 0]]], state=basis(3, 7)),
    dict(name="swap", ref="sim/statevector/sim_test.go:202-221", n=2,
         ops=[["X", [0]], ["SWAP", [0, 1]]], state=state(0, 0, 1, 0)),
    dict(name="ev_zero", ref="sim/statevector/sim_test.go:223-237", n=1, ops=[], expect_z=[[[0], 1.0]]),
    dict(name="ev_one", ref="sim/statevector/sim_test.go:239-249", n=1, ops=[["X", [0]]], expect_z=[[[0], -1.0]]),
    dict(name="ev_plus", ref="sim/statevector/sim_test.go:251-262", n=1, ops=[["H", [0]]], expect_z=[[[0], 0.0]]),
    dict(name="cnot_nonadjacent", ref="sim/statevector/sim_test.go:279-300", n=4,
         ops=[["X", [0]], ["CNOT", [0, 2]]], state=basis(4, 5)),
    dict(name="cz", ref="sim/statevector/sim_test.go:302-325", n=2,
         ops=[["H", [0]], ["X", [1]], ["CZ", [0, 1]]], state=state(0, 0, S2, -S2)),
    dict(name="cy", ref="sim/statevector/sim_test.go:327-345", n=2,
         ops=[["X", [0]], ["CY", [0, 1]]], state=state(0, 0, 0, c(0, 1))),
    dict(name="cp_pi", ref="sim/statevector/sim_test.go:347-367", n=2,
         ops=[["H", [0]], ["X", [1]], ["CP", [0, 1], [PI]]], state=state(0, 0, S2, -S2)),
    dict(name="crz_pi", ref="sim/statevector/sim_test.go:369-390", n=2,
         ops=[["X", [0]], ["X", [1]], ["CRZ", [0, 1], [PI]]], state=state(0, 0, 0, c(0, 1))),
    dict(name="crx_pi", ref="sim/statevector/sim_test.go:392-411", n=2,
         ops=[["X", [0]], ["CRX", [0, 1], [PI]]], state=state(0, 0, 0, c(0, -1))),
    dict(name="cry_pi", ref="sim/statevector/sim_test.go:413-432", n=2,
         ops=[["X", [0]], ["CRY", [0, 1], [PI]]], state=state(0, 0, 0, 1)),
    dict(name="ms_00", ref="sim/statevector/sim_test.go:434-456", n=2,
         ops=[["MS", [0, 1], [0.0, 0.0]]], state=state(S2, 0, 0, c(0, -S2))),
    dict(name="ccx_nonadjacent", ref="sim/statevector/sim_test.go:462-485", n=5,
         ops=[["X", [0]], ["X", [2]], ["CCX", [0, 2, 4]]], state=basis(5, 21)),
    dict(name="cswap", ref="sim/statevector/sim_test.go:487-510", n=3,
         ops=[["X", [0]], ["X", [2]], ["CSWAP", [0, 1, 2]]], state=basis(3, 3)),
    dict(name="reset_x", ref="sim/statevector/sim_test.go:667-679", n=1,
         ops=[["X", [0]], ["Reset", [0]]], state=state(1, 0)),
    dict(name="reset_h", ref="sim/statevector/sim_test.go:681-693", n=1,
         ops=[["H", [0]], ["Reset", [0]]], state=state(1, 0)),
    dict(name="reset_bell_q0", ref="sim/statevector/sim_test.go:695-731", n=2,
         ops=[["H", [0]], ["CNOT", [0, 1]], ["Reset", [0]]], state=state(S2, 0, S2, 0), norm=1.0),
    dict(name="reset_zero", ref="sim/statevector/sim_test.go:733-745", n=1,
         ops=[["Reset", [0]]], state=state(1, 0)),
    dict(name="parallel_17q", ref="sim/statevector/sim_test.go:748-771", n=17,
         ops=[["H", [0]], ["CNOT", [0, 1]]], abs_at=[[0, S2], [3, S2]]),
    # --- sim/statevector/kernel_controlled_test.go --------------------------
    dict(name="mcx3_flip", ref="sim/statevector/kernel_controlled_test.go:13-40", n=4,
         ops=[["X", [0]], ["X", [1]], ["X", [2]], ["MCX", [0, 1, 2, 3], [3]]], prob_one=15),
    dict(name="mcx3_partial", ref="sim/statevector/kernel_controlled_test.go:42-67", n=4,
         ops=[["X", [0]], ["X", [1]], ["MCX", [0, 1, 2, 3], [3]]], prob_one=3),
    dict(name="mcz2_phase", ref="sim/statevector/kernel_controlled_test.go:89-99", n=3,
         ops=[["X", [0]], ["X", [1]], ["X", [2]], ["MCZ", [0, 1, 2], [2]]], amp_at=[[7, c(-1.0)]]),
    dict(name="mcp2_pi", ref="sim/statevector/kernel_controlled_test.go:101-110", n=3,
         ops=[["X", [0]], ["X", [1]], ["X", [2]], ["MCP", [0, 1, 2], [PI, 2]]], amp_at=[[7, c(-1.0)]]),
    dict(name="controlled_nonadjacent", ref="sim/statevector/kernel_controlled_test.go:112-135", n=4,
         ops=[["X", [0]], ["X", [3]], ["MCX", [0, 3, 1], [2]]], prob_one=11),
    dict(name="c1_swap", ref="sim/statevector/kernel_controlled_test.go:137-167", n=3,
         ops=[["X", [0]], ["X", [2]], ["CTRL_SWAP", [0, 1, 2], [1]]], state=basis(3, 3)),
    dict(name="mcx4", ref="sim/statevector/kernel_controlled_test.go:169-189", n=5,
         ops=[["X", [0]], ["X", [1]], ["X", [2]], ["X", [3]], ["MCX", [0, 1, 2, 3, 4], [4]]], prob_one=31),
    # --- sim/statevector/integration_test.go --------------------------------
    dict(name="qft4_qasm", ref="sim/statevector/integration_test.go:72-111", n=4,
         ops=[["X", [0]], ["X", [2]], ["H", [0]], ["CP", [1, 0], [PI / 2]], ["H", [1]], ["CP", [2, 0], [PI / 4]],
              ["CP", [2, 1], [PI / 2]], ["H", [2]], ["CP", [3, 0], [PI / 8]], ["CP", [3, 1], [PI / 4]],
              ["CP", [3, 2], [PI / 2]], ["H", [3]]], abs_all=0.25),
    # --- sim/pauli/expect_sv_test.go (prepared with gates) -------------------
    dict(name="pauli_single", ref="sim/pauli/expect_sv_test.go:35-66", n=1, ops=[["H", [0]]],
         pauli=[["X", 1.0], ["Z", 0.0], ["Y", 0.0], ["I", 1.0]]),
    dict(name="pauli_minus", ref="sim/pauli/expect_sv_test.go:46-55", n=1, ops=[["X", [0]], ["H", [0]]],
         pauli=[["X", -1.0]]),
    dict(name="pauli_plus_i", ref="sim/pauli/expect_sv_test.go:57-66", n=1, ops=[["H", [0]], ["S", [0]]],
         pauli=[["Y", 1.0]]),
    dict(name="pauli_bell", ref="sim/pauli/expect_sv_test.go:85-171", n=2, ops=[["H", [0]], ["CNOT", [0, 1]]],
         pauli=[["ZZ", 1.0], ["XX", 1.0], ["YY", -1.0], ["XY", 0.0], ["ZI", 0.0], ["II", 1.0]]),
    dict(name="pauli_sum_00", ref="sim/pauli/expect_sv_test.go:106-116", n=2, ops=[],
         pauli_sum=[[0.5, 0.0, {"0": "Z", "1": "Z"}], [0.3, 0.0, {"0": "X"}]], pauli_sum_value=[0.5, 0.0]),
    dict(name="pauli_complex_coeff", ref="sim/pauli/expect_sv_test.go:187-193", n=1, ops=[],
         pauli_sum=[[0.0, 1.0, {"0": "Z"}]], pauli_sum_value=[0.0, 1.0]),
    dict(name="pauli_zii", ref="sim/pauli/expect_sv_test.go:179-185", n=3, ops=[], pauli=[["ZII", 1.0]]),
    # --- sim/densitymatrix/sim_test.go --------------------------------------
    dict(name="dm_fidelity_h", ref="sim/densitymatrix/sim_test.go:120-140", n=1, dm=True,
         ops=[["H", [0]]], fidelity_with_sv=1.0),
    dict(name="dm_depol_mixed", ref="sim/densitymatrix/sim_test.go:163-186", n=1, dm=True,
         noise=[["default", 1, "Depolarizing1Q", [0.75]]], ops=[["X", [0]]],
         rho_at=[[0, c(0.5)], [3, c(0.5)]]),
    dict(name="dm_amp_damping", ref="sim/densitymatrix/sim_test.go:188-211", n=1, dm=True,
         noise=[["gate", "X", "AmplitudeDamping", [0.5]]], ops=[["X", [0]]],
         rho_at=[[0, c(0.5)], [3, c(0.5)]]),
    dict(name="dm_phase_damping", ref="sim/densitymatrix/sim_test.go:213-234", n=1, dm=True,
         noise=[["gate", "H", "PhaseDamping", [0.5]]], ops=[["H", [0]]],
         rho_at=[[1, c(0.5 * math.sqrt(0.5))]]),
    dict(name="dm_readout", ref="sim/densitymatrix/sim_test.go:236-253", n=1, dm=True,
         readout=[[0, 0.1, 0.2]], ops=[], readout_probs=[0.9, 0.1]),
    dict(name="dm_trace_bell_depol", ref="sim/densitymatrix/sim_test.go:255-277", n=2, dm=True,
         noise=[["default", 1, "Depolarizing1Q", [0.1]], ["default", 2, "Depolarizing2Q", [0.1]]],
         ops=[["H", [0]], ["CNOT", [0, 1]]], trace=1.0, purity_below=1.0),
    dict(name="dm_positivity", ref="sim/densitymatrix/sim_test.go:279-301", n=2, dm=True,
         noise=[["default", 1, "Depolarizing1Q", [0.3]]],
         ops=[["H", [0]], ["RZ", [1], [PI / 3]], ["CNOT", [0, 1]]], diag_nonneg=True, trace=1.0),
]


def main():
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kats.json")
    with open(out, "w") as f:
        json.dump({"source": "known-answer tests of github.com/splch/goqu (eps 1e-10)", "kats": KATS}, f, indent=1)
    print(f"wrote {len(KATS)} KATs to {out}")


if __name__ == "__main__":
    main()
