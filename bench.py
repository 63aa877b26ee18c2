"""Benchmark: 28-qubit complex128 random-circuit simulation on B200.

Workload (one step): goqu statevector Evolve of a seeded 28-qubit circuit of
40 layers (U3 with uniform [0, 2 pi) angles on every qubit, then a CNOT
brickwork) followed by a 28-qubit QFT (algorithm/qpe/qpe.go:170-182): 2080
gates on a 4 GiB complex128 state, 32x the B200 L2 cache, so every pass
streams HBM (no flush needed). The device is timed with CUDA events on the
engine's stream. e2e is the public C-ABI call gq_sv_run (Evolve + 1024
inverse-CDF shots) with the op stream coming from host memory and the sampled
indices copied back, timed on the host around the call.

Extras (N = 1 only; other configurations of the same path and parity checks,
reported in "extras"): the full 28-qubit circuit against the FP64 oracle
(complex128 amplitudes and samples, and the complex64 bulk with its error and
throughput); adjoint gradients of a 20-qubit 400-parameter ansatz against the
oracle's parameter shift; a noisy 12-qubit density matrix; a batch of 4096
QAOA MaxCut circuits (complex64, energies + gradients); the 20-qubit
configuration.

--impl reference times the CPU restatement of goqu's pure-Go path (the oracle,
threaded like goqu's auto-parallel kernels) on this host's cores: each step is
a stratified sample of the same circuit (one U3 layer, one CNOT layer of each
parity, the first QFT row and one SWAP, timed gate by gate), and the rate is
the full circuit's gate count over the class-weighted time. Multi-GPU runs
(torchrun) are independent replicas, one state per GPU.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

LAYERS = 40
SEED = 2028
SHOTS = 1024


def workload_name(n, precision):
    return (f"statevector {n}q {'complex64' if precision == 'c64' else 'complex128'}: {LAYERS} U3+CNOT "
            f"brickwork layers + QFT{n}, {SHOTS} shots")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dist_setup(backend=None):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE): NCCL
    when a GPU is present, gloo otherwise (the CPU tests of this plumbing)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for k, name in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def build_workload(n):
    from goqu_b200 import encode, workloads
    c = workloads.random_layers_qft(n, LAYERS, SEED)
    return c, encode.statevector_ops(c), workloads.count_gates(c)


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# Stratified CPU sample of the benchmark circuit: per gate class, the first
# occurrences covering one U3 layer, one CNOT layer of each parity, the first
# QFT row (H + its controlled phases) and one SWAP.
def sample_plan(c, n):
    names = [op.Gate.Name().split("(")[0] for op in c.Ops()
             if op.Gate is not None and op.Gate.Name() not in ("barrier", "delay")]
    want = {"U3": n, "CNOT": n - 1, "H": 1, "CP": n - 1, "SWAP": 1}
    picked, seen = [], {}
    for i, nm in enumerate(names):
        k = seen.get(nm, 0)
        if k < want.get(nm, 0):
            picked.append(i)
            seen[nm] = k + 1
    counts = {nm: names.count(nm) for nm in set(names)}
    return names, picked, counts


class CpuSample:
    """goqu's CPU path (the oracle, threaded like goqu's GOMAXPROCS workers)
    timed gate by gate on the stratified sample of the full-size circuit; the
    full-circuit rate weighs each class's mean gate time by its count."""

    def __init__(self, n, c, stream, threads=None):
        from oracle import binding as orc
        self.n, self.stream = n, stream
        self.threads = threads or os.cpu_count() or 1
        self.names, self.picked, self.counts = sample_plan(c, n)
        self.state = orc.zero_state(n)
        self.ops = stream.array()
        self._apply(self.picked[0])  # first touch of the state's pages, untimed

    def _apply(self, i):
        import ctypes

        from oracle import binding as orc
        one = (type(self.ops[0]) * 1)(self.ops[i])
        t0 = time.perf_counter()
        rc = orc.lib().or_sv_apply(self.n, self.state.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                   ctypes.cast(one, ctypes.POINTER(type(self.ops[0]))), 1, self.threads)
        dt = time.perf_counter() - t0
        assert rc == 0
        return dt

    def step(self):
        per = {}
        for i in self.picked:
            per.setdefault(self.names[i], []).append(self._apply(i))
        timed = sum(sum(v) for v in per.values())
        est = sum(self.counts[k] * float(np.mean(v)) for k, v in per.items())
        return sum(self.counts.values()) / est, timed, {k: len(v) for k, v in per.items()}

    def describe(self, value, timed_s, steps, per):
        total = sum(self.counts.values())
        mix = ", ".join(f"{per[k]} {k} of {self.counts[k]}" for k in sorted(per))
        return {"value": value, "unit": "gates/s", "cores": self.threads, "kind": "port", "cpu_model": cpu_model(),
                "sample": f"stratified sample of the {total}-gate circuit at {self.n} qubits (complex128), per step "
                          f"{len(self.picked)} gates ({mix}) timed one by one; rate = {total} gates / sum over "
                          f"classes of (class gate count x class mean time); {timed_s:.1f} s timed over {steps} "
                          f"step(s); oracle threaded like goqu's GOMAXPROCS workers",
                "gates_timed_per_step": len(self.picked), "seconds_timed": timed_s}


def cpu_baseline(n, c, stream, steps=3):
    cs = CpuSample(n, c, stream)
    vals, timed, per = [], 0.0, None
    for _ in range(steps):
        v, t, per = cs.step()
        vals.append(v)
        timed += t
    return cs.describe(float(np.mean(vals)), timed, steps, per)


def run_reference(args, world, rank):
    if rank != 0:
        return
    n = args.qubits
    c, stream, gates = build_workload(n)
    cs = CpuSample(n, c, stream)
    for _ in range(args.warmup):
        cs.step()
    vals, times, per = [], [], None
    for _ in range(args.steps):
        v, t, per = cs.step()
        vals.append(v)
        times.append(t)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": f"{n}q gates/s", "value": value, "unit": "gates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * float(np.mean(times)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(n, "c128"), "qubits": n, "gates": gates, "seed": SEED,
                       "l2": "state 4 GiB > 126 MB L2 (no flush needed)",
                       "step": "one stratified sample of the circuit's gate classes (ms_per_step is its measured "
                               "time); value is the full-circuit rate those class times give"},
            "cpu_baseline": cs.describe(value, float(np.sum(times)), args.steps, per),
            "e2e": {"value": value, "unit": "gates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def extra_adjoint():
    """20-qubit hardware-efficient ansatz (10 layers RY,RZ + CZ ring, 400
    parameters), transverse-field Ising observable: adjoint gradient vs the
    full 800-evaluation parameter shift on the same engine."""
    from goqu_b200 import _abi, gradient, workloads
    c, names = workloads.hardware_efficient_ansatz(20, 10)
    h = workloads.ising_hamiltonian(20)
    x = np.random.default_rng(20).uniform(0, 2 * np.pi, len(names))
    ev = gradient.AdjointEvaluator(c, h, names)
    ev.sim.set_option(_abi.GQ_OPT_TIMING, 1)
    ev.sim.set_option(_abi.GQ_OPT_JIT, 2)
    for _ in range(3):
        ev(x)
    dev, t0 = [], time.perf_counter()
    for _ in range(10):
        _, g_adj = ev(x)
        dev.append(ev.sim.stats()["last_ms"])
    wall = (time.perf_counter() - t0) / 10
    st = ev.sim.stats()
    adj_stats = {k: st[k] for k in ("passes", "jit_passes", "kernel_launches", "pass_ms")}
    f = gradient.CostFunc(c, h, names)
    f.sim.set_option(_abi.GQ_OPT_TIMING, 1)
    f.sim.set_option(_abi.GQ_OPT_JIT, 2)
    f(x)
    g_ps = np.empty(len(names))
    ps_dev, t1 = 0.0, time.perf_counter()
    for i in range(len(names)):
        xp, xm = x.copy(), x.copy()
        xp[i] += math.pi / 2
        xm[i] -= math.pi / 2
        ep = f(xp)
        ps_dev += f.sim.stats()["last_ms"]
        em = f(xm)
        ps_dev += f.sim.stats()["last_ms"]
        g_ps[i] = (ep - em) / 2
    ps_wall = time.perf_counter() - t1
    adj_ms = float(np.median(dev))
    from oracle import gradient as og
    sel = og.stratified_hea_params(20, 10)
    t_or = time.perf_counter()
    g_or = og.parameter_shift(c, names, x, h, sel, threads=os.cpu_count() or 1)
    t_or = time.perf_counter() - t_or
    return {"workload": "adjoint gradient, 20q HEA 10 layers, 400 params, Ising H (39 terms), complex128",
            "max_abs_diff_vs_oracle_param_shift": float(np.max(np.abs(g_adj[sel] - g_or))),
            "oracle_sample": f"{len(sel)} parameters: RY and RZ of 2 qubits in each of the 10 layers",
            "adjoint_grads_per_s": 1000.0 / adj_ms, "adjoint_ms_device": adj_ms, "adjoint_ms_wall": wall * 1e3,
            "adjoint_ms_device_calls": [round(v, 3) for v in dev], "adjoint_call_stats": adj_stats,
            "cpu_oracle": {"what": "FP64 oracle parameter shift (2 evaluations per parameter, prefixes shared) "
                                   "of the sampled parameters on the host cores",
                           "params": len(sel), "seconds": t_or, "cores": os.cpu_count(),
                           "grads_per_s_all_400_params": len(sel) / (len(names) * t_or)},
            "param_shift_grads_per_s": 1000.0 / ps_dev, "param_shift_ms_device": ps_dev,
            "param_shift_ms_wall": ps_wall * 1e3, "speedup_device": ps_dev / adj_ms,
            "speedup_wall": ps_wall / wall,
            "max_abs_diff_vs_engine_param_shift": float(np.max(np.abs(g_adj - g_ps)))}


def extra_vqe(iters=20):
    """Adam on the 20-qubit, 400-parameter ansatz with adjoint gradients:
    the loop inside the library (gq_sv_minimize_adam: rebinding, one forward
    + reverse sweep per iteration) against the same Adam driven from the host
    (gates bound and encoded on the host for every gradient and energy)."""
    from goqu_b200 import _abi, gradient, optim, vqe, workloads
    c, names = workloads.hardware_efficient_ansatz(20, 10)
    h = workloads.ising_hamiltonian(20)
    x0 = np.random.default_rng(20).uniform(0, 2 * np.pi, len(names))
    adam = optim.Adam(LR=0.01)
    opts = optim.Options(MaxIter=iters, FunTol=1e-300)
    from goqu_b200 import statevector
    sim = statevector.New(20)
    sim.set_option(_abi.GQ_OPT_JIT, 2)
    vqe.minimize_adam_on_device(c, h, names, x0, adam, optim.Options(MaxIter=2), sim=sim)  # kernels compiled
    t0 = time.perf_counter()
    r_dev, hist = vqe.minimize_adam_on_device(c, h, names, x0, adam, opts, sim=sim)
    dev_s = time.perf_counter() - t0
    sim.Close()
    ev = gradient.AdjointEvaluator(c, h, names)
    ev.sim.set_option(_abi.GQ_OPT_JIT, 2)
    ev(x0)
    t1 = time.perf_counter()
    r_host = adam.Minimize(lambda x: ev(x)[0], x0, lambda x: ev(x)[1], opts)
    host_s = time.perf_counter() - t1
    return {"workload": "Adam, 20q HEA 10 layers, 400 params, Ising H, adjoint gradients, complex128",
            "iterations": r_dev.Iterations, "ms_per_iteration_library_loop": 1e3 * dev_s / r_dev.Iterations,
            "ms_per_iteration_host_loop": 1e3 * host_s / r_host.Iterations,
            "device_evaluations_per_iteration": {"library_loop": 1, "host_loop": 2},
            "energy_first_last": [hist[0], hist[-1]],
            "max_abs_x_diff_library_vs_host": float(np.max(np.abs(r_dev.X - r_host.X)))}


def first_call(n=28):
    """Seconds of the first Evolve of the benchmark circuit in this process
    (specialised kernels compiled, or read from the on-disk cache, and loaded)."""
    from goqu_b200 import _abi, statevector
    c, stream, gates = build_workload(n)
    sim = statevector.New(n)
    sim.set_option(_abi.GQ_OPT_JIT, 2)
    t0 = time.perf_counter()
    sim.evolve_ops(stream)
    sim.Close()
    return time.perf_counter() - t0


def extra_cold_start():
    """The first call of a fresh process, once the kernels this run compiled
    are in the on-disk cache (GQ_JIT_CACHE_DIR), against this process's first
    call, which compiled them."""
    out = subprocess.run([sys.executable, os.path.abspath(__file__), "--first-call"], capture_output=True,
                         text=True, env=dict(os.environ), timeout=600)
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    if out.returncode != 0 or not line:
        return {"error": (out.stderr or out.stdout)[-400:]}
    return {"workload": workload_name(28, "c128"),
            "first_call_s_new_process_disk_cache": json.loads(line[-1])["first_call_s"],
            "cache": "on-disk cubins keyed by compiler, header and kernel text (GQ_JIT_CACHE_DIR)"}


def extra_density():
    """Noisy 12-qubit density matrix: 30 U3 + CNOT brickwork layers,
    depolarizing 1e-3 after every gate, amplitude damping 1e-3 on idle qubits."""
    from goqu_b200 import _abi, densitymatrix, encode, pauli, workloads
    from oracle import binding as orc
    c, nm = workloads.noisy_brickwork(12, layers=30, seed=12)
    dm = densitymatrix.New(12).WithNoise(nm)
    dm.set_option(_abi.GQ_OPT_TIMING, 1)
    dm.set_option(_abi.GQ_OPT_JIT, 2)
    s = encode.density_ops(c, nm)
    lib = _abi.lib()
    for _ in range(2):
        _abi.check(lib.gq_dm_evolve(dm._h, s.ptr(), len(s)))
    ms, pms = [], []
    for _ in range(5):
        _abi.check(lib.gq_dm_evolve(dm._h, s.ptr(), len(s)))
        ms.append(dm.stats()["last_ms"])
        pms.append(dm.stats()["pass_ms"])
    st = dm.stats()
    z = [dm.ExpectPauliString(pauli.ZOn([q], 12)) for q in range(12)]
    tr = dm.Trace()
    dm.Close()
    peak, peak_kind = peaks()
    # rho (2^24 complex128 entries) read and written once per pass, less the
    # tiles the first passes skip while they are still zero
    pass_bytes = st["tile_bytes"] / max(1, st["passes"])
    pass_ms = float(np.median(pms)) / max(1, st["passes"])
    achieved = pass_bytes / (pass_ms / 1000.0) / 1e9

    def check(n, layers):
        cc, nn = workloads.noisy_brickwork(n, layers=layers, seed=12)
        ss = encode.density_ops(cc, nn)
        t_or = time.perf_counter()
        want = orc.dm_evolve(ss, threads=os.cpu_count() or 1)
        t_or = time.perf_counter() - t_or
        d = densitymatrix.New(n).WithNoise(nn)
        d.set_option(_abi.GQ_OPT_JIT, 2)
        d.set_option(_abi.GQ_OPT_JIT_MIN_QUBITS, 0)
        _abi.check(lib.gq_dm_evolve(d._h, ss.ptr(), len(ss)))
        terms = [pauli.to_terms(pauli.ZOn([q], n)) for q in range(n)]
        z_err = max(abs(d.ExpectPauliString(pauli.ZOn([q], n)) - orc.dm_expect_pauli_sum(want, n, terms[q]).real)
                    for q in range(n))
        out = {"layers": layers, "max_abs_rho_error_vs_fp64_oracle": float(np.max(np.abs(d.DensityMatrix() - want))),
               "max_abs_z_error_vs_fp64_oracle": z_err,
               "trace_error_vs_fp64_oracle": abs(d.Trace() - np.trace(want.reshape(1 << n, 1 << n))),
               "cpu_oracle_s": t_or, "cpu_cores": os.cpu_count()}
        d.Close()
        return out

    return {"workload": "density matrix 12q, 30 noisy U3+CNOT layers (depolarizing + amplitude damping)",
            "ms_device": float(np.median(ms)), "gates": workloads.count_gates(c), "ops_with_channels": len(s),
            "passes": st["passes"], "trace_minus_one": abs(tr - 1.0), "z_expectations": z[:3],
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "algorithmic_bytes_per_launch": pass_bytes, "launch_ms": pass_ms},
            "error_check_12q": check(12, 2), "error_check_8q": check(8, 30)}


def extra_qaoa(qubits=0, count=0, calls=3, graph=True):
    """4096 QAOA MaxCut circuits on seeded random 3-regular graphs, n in
    {10..20} even, p in 1..4, complex64: energies + adjoint gradients in one
    batched call (later calls replay the captured CUDA graphs). qubits / count
    keep only the circuits of that size / the first `count` (profiling cases)."""
    from goqu_b200 import _abi, batch, workloads
    t0 = time.perf_counter()
    evals = workloads.qaoa_batch(4096, seed=4)
    if qubits:
        evals = [e for e in evals if e[0].NumQubits() == qubits]
    if count:
        evals = evals[:count]
    streams, terms = batch.Batch.encode(evals)
    host_s = time.perf_counter() - t0
    npar = [len(e[1]) for e in evals]
    b = batch.Batch(_abi.GQ_C64)
    b.set_option(_abi.GQ_OPT_TIMING, 1)
    b.set_option(_abi.GQ_OPT_USE_GRAPH, 1 if graph else 0)
    ms, dev, host = [], [], []
    for _ in range(calls):
        energies, grads = b.run_encoded(streams, terms, npar)
        ms.append(b.stats()["last_ms"])
        dev.append(b.stats()["pass_ms"])
        host.append(b.stats()["host_ms"])
    st = b.stats()
    # error against the FP64 oracle on a sample of the batch: energies, and
    # gradients against central differences of the oracle energy (each QAOA
    # angle drives every RZZ / RX of its layer, so the +-pi/2 shift rule of a
    # single gate does not apply)
    from oracle import gradient as og
    th = os.cpu_count() or 1
    e_err = g_err = 0.0
    for k in range(0, len(evals), max(1, len(evals) // 16)):
        c, names, h, x = evals[k]
        x = np.asarray(x, float)
        e_err = max(e_err, abs(energies[k] - og.energy(c, names, x, h, threads=th)))
        fd = og.parameter_shift(c, names, x, h, threads=th, shift=1e-6, denom=2e-6)
        g_err = max(g_err, float(np.max(np.abs(grads[k] - fd))))
    sub = "" if not (qubits or count) else f" (subset: {'n = %d, ' % qubits if qubits else ''}{len(evals)} circuits)"
    return {"workload": "4096 QAOA MaxCut circuits (n 10..20, p 1..4), complex64, energies + gradients" + sub,
            "circuits": len(evals), "circuits_per_s": len(evals) / (ms[-1] / 1000.0), "ms_call_first": ms[0],
            "ms_call_replay": ms[-1], "ms_device_replay": dev[-1], "ms_host_before_launch": host[-1],
            "timing": "call: host planning (overlapped with the device by segments) + upload + graphs + results "
                      "(CUDA events on the batch stream); device: span of the batched launches",
            "passes": st["passes"], "launches": st["kernel_launches"], "host_encode_s": host_s,
            "max_abs_energy_error_vs_fp64_oracle": e_err, "max_abs_grad_error_vs_fp64_central_difference": g_err,
            "error_sample": f"{len(range(0, len(evals), max(1, len(evals) // 16)))} circuits evenly spaced"}


def max_abs_diff(a, b, chunk=1 << 24):
    m = 0.0
    for k in range(0, a.size, chunk):
        m = max(m, float(np.max(np.abs(a[k:k + chunk] - b[k:k + chunk]))))
    return m


def extra_parity_28q(n=28, steps=3):
    """The benchmark circuit itself (40 layers + QFT28, 2080 gates) against the
    FP64 oracle: complex128 amplitudes and 1024 sampled indices, and the
    complex64 bulk's throughput, roofline and error against the same state."""
    import ctypes

    from goqu_b200 import _abi, statevector
    from oracle import binding as orc
    c, stream, gates = build_workload(n)
    u = statevector.uniforms(SHOTS, np.random.default_rng(SEED))
    peak, peak_kind = peaks()
    out = {"workload": workload_name(n, "c128") + " (complex128 and complex64)"}
    got = {}
    for prec, tag, amp in ((_abi.GQ_C128, "c128", 16), (_abi.GQ_C64, "c64", 8)):
        sim = statevector.New(n, prec)
        sim.set_option(_abi.GQ_OPT_TIMING, 1)
        sim.set_option(_abi.GQ_OPT_JIT, 2)
        for _ in range(2):
            sim.evolve_ops(stream)
        ms, pms, passes, tbytes = [], [], 0, 0
        for _ in range(steps):
            sim.evolve_ops(stream)
            st = sim.stats()
            ms.append(st["last_ms"])
            pms.append(st["pass_ms"])
            passes += st["passes"]
            tbytes += st["tile_bytes"]
        launch_ms = float(np.sum(pms)) / max(1, passes)
        achieved = tbytes / max(1, passes) / (launch_ms / 1000.0) / 1e9
        out[tag] = {"gates_per_s": gates / (float(np.median(ms)) / 1000.0), "ms_device": float(np.median(ms)),
                    "passes": passes // steps,
                    "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                 "frac": achieved / peak, "peak_kind": peak_kind, "launch_ms": launch_ms}}
        if prec == _abi.GQ_C128:
            got[tag] = sim.StateVector()
            idx = sim.Sample(u)
        else:  # kept as complex64 on the host (2 GiB) until the comparison
            got[tag] = np.empty(1 << n, dtype=np.complex64)
            _abi.check(_abi.lib().gq_sv_get_state(sim.handle, got[tag].ctypes.data_as(ctypes.c_void_p),
                                                  got[tag].nbytes))
        sim.Close()
    t0 = time.perf_counter()
    want = orc.sv_evolve(stream, threads=os.cpu_count() or 1)
    out["oracle_s"] = time.perf_counter() - t0
    out["c128"]["max_abs_amplitude_error_vs_fp64_oracle"] = max_abs_diff(got["c128"], want)
    out["c128"]["samples_bit_exact_vs_oracle"] = bool(
        np.array_equal(idx, orc.sample_fast(orc.probabilities(got["c128"]), u)))
    del got["c128"]
    out["c64"]["max_abs_amplitude_error_vs_fp64_oracle"] = max_abs_diff(got["c64"], want)
    return out


def extra_qaoa_dedicated(qubits=0, count=0, calls=3):
    """The same 4096 QAOA MaxCut circuits through the dedicated path
    (gq_qaoa_maxcut_batch): cut-count tables, whole circuits of <= 12 qubits
    in one CTA, batched tile passes above; energies and gradients against the
    general batch path and the FP64 oracle. qubits / count keep only the
    circuits of that size / the first `count` (profiling cases)."""
    from goqu_b200 import _abi, batch, qaoa
    evals = workloads_qaoa_4096()
    if qubits:
        evals = [e for e in evals if e[0].NumQubits() == qubits]
    if count:
        evals = evals[:count]
    t0 = time.perf_counter()
    items = [qaoa.from_evaluation(e) for e in evals]
    b = qaoa.MaxCutBatch()
    enc = b.encode(items)  # host packing of the records, once (as for the general batch)
    host_encode_s = time.perf_counter() - t0
    b.run_encoded(enc)  # buffers sized, kernels loaded
    ms = []
    for _ in range(calls):
        t0 = time.perf_counter()
        e_fast, g_fast = b.run_encoded(enc)
        ms.append(1e3 * (time.perf_counter() - t0))
    gen = batch.Batch(_abi.GQ_C64)
    e_gen, g_gen = gen.Run(evals)
    from oracle import gradient as og
    th = os.cpu_count() or 1
    t_or = time.perf_counter()
    e_err = g_err = 0.0
    for k in range(0, len(evals), max(1, len(evals) // 16)):
        c, names, h, x = evals[k]
        x = np.asarray(x, float)
        e_err = max(e_err, abs(e_fast[k] - og.energy(c, names, x, h, threads=th)))
        fd = og.parameter_shift(c, names, x, h, threads=th, shift=1e-6, denom=2e-6)
        g_err = max(g_err, float(np.max(np.abs(g_fast[k] - fd))))
    t_or = time.perf_counter() - t_or
    n_or = len(range(0, len(evals), max(1, len(evals) // 16)))
    # algorithmic bytes: per circuit above 12 qubits, every forward pass reads and
    # writes psi (8 B per amplitude), every reverse pass psi and lambda, plus the
    # cut table (1 B) wherever it is read; circuits of <= 12 qubits stay on chip
    alg = 0
    for n, edges, gam, bet in items:
        if n <= 12:
            continue
        p, groups = len(gam), (n - 12 + 7) // 8
        passes = p * (1 + groups)
        alg += (1 << n) * (passes * 16 + passes * 32 + 2 * p + 1)
    peak, peak_kind = peaks()
    best = min(ms)
    return {"workload": f"{len(items)} QAOA MaxCut circuits (n 10..20, p 1..4), complex64, energies + gradients, "
                        "dedicated path" + (f" (only n = {qubits})" if qubits else ""),
            "ms_call": best, "circuits_per_s": len(items) / (best / 1000.0),
            "timing": "wall time of the whole gq_qaoa_maxcut_batch call (host tables, upload, launches, results); "
                      "records packed once beforehand",
            "host_encode_s": host_encode_s,
            "max_abs_energy_diff_vs_general_batch": float(np.max(np.abs(np.asarray(e_fast) - np.asarray(e_gen)))),
            "max_abs_grad_diff_vs_general_batch": float(max(np.max(np.abs(a - c)) for a, c in zip(g_fast, g_gen))),
            "max_abs_energy_error_vs_fp64_oracle": e_err, "max_abs_grad_error_vs_fp64_central_difference": g_err,
            "cpu_oracle": {"what": "FP64 oracle energy + central-difference gradient (2 evaluations per parameter) "
                                   "of the sampled circuits on the host cores",
                           "circuits": n_or, "seconds": t_or, "cores": os.cpu_count(),
                           "circuits_per_s": n_or / t_or},
            "roofline": {"bound": "hbm", "algorithmic_bytes": alg,
                         "achieved": alg / (best / 1000.0) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / (best / 1000.0) / 1e9 / peak, "peak_kind": peak_kind,
                         "note": "whole-call wall time; circuits of <= 12 qubits add no HBM bytes"}}


def extra_sampling(n=28, calls=10):
    """Exact sampling of the benchmark circuit's 28-qubit state: 1024 shots
    per call (gq_sv_sample: chunk sums, scan, chunk step counts, the exact
    walk, per-shot search), wall time of the whole call (uniform upload,
    kernels, index download)."""
    from goqu_b200 import _abi, statevector
    c, stream, gates = build_workload(n)
    sim = statevector.New(n)
    sim.set_option(_abi.GQ_OPT_JIT, 2)
    sim.evolve_ops(stream)
    u = statevector.uniforms(SHOTS, np.random.default_rng(SEED))
    first = sim.Sample(u)
    ms = []
    for _ in range(calls):
        t0 = time.perf_counter()
        idx = sim.Sample(u)
        ms.append(1e3 * (time.perf_counter() - t0))
    same = bool(np.array_equal(idx, first))
    sim.Close()
    return {"workload": f"{SHOTS} shots of the {n}q benchmark state (complex128)", "ms_call_wall": float(np.median(ms)),
            "calls": calls, "repeatable": same,
            "note": "indices are checked bit-exact against the oracle in parity_28q and the GPU tests"}


def workloads_qaoa_4096():
    from goqu_b200 import workloads
    return workloads.qaoa_batch(4096, seed=4)


def extra_parity():
    """The 20-qubit configuration (20 U3 + CNOT brickwork layers, 590 gates,
    1024 shots): throughput and error against the FP64 oracle, complex128 and
    complex64; sampled indices against the oracle's sequential inverse CDF."""
    from goqu_b200 import _abi, encode, statevector, workloads
    from oracle import binding as orc
    c = workloads.random_layers(20, 20, 20)
    stream = encode.statevector_ops(c)
    gates = workloads.count_gates(c)
    want = orc.sv_evolve(stream)
    u = statevector.uniforms(SHOTS, np.random.default_rng(SEED))
    out = {"workload": f"statevector 20q: 20 U3+CNOT brickwork layers ({gates} gates), {SHOTS} shots"}
    for prec, tag in ((_abi.GQ_C128, "c128"), (_abi.GQ_C64, "c64")):
        sim = statevector.New(20, prec)
        sim.set_option(_abi.GQ_OPT_TIMING, 1)
        sim.set_option(_abi.GQ_OPT_JIT, 2)
        for _ in range(3):
            sim.evolve_ops(stream)
        ms = []
        for _ in range(5):
            sim.evolve_ops(stream)
            ms.append(sim.stats()["last_ms"])
        got = sim.StateVector()
        out[tag] = {"gates_per_s": gates / (float(np.median(ms)) / 1000.0), "ms_device": float(np.median(ms)),
                    "max_abs_amplitude_error_vs_fp64_oracle": float(np.max(np.abs(got - want)))}
        if prec == _abi.GQ_C128:
            probs = orc.probabilities(got)
            out[tag]["samples_bit_exact_vs_oracle"] = bool(np.array_equal(sim.Sample(u), orc.sample_fast(probs, u)))
        sim.Close()
    return out


def run_gpu(args, world, rank, local):
    import ctypes

    from goqu_b200 import _abi, statevector
    n = args.qubits
    c, stream, gates = build_workload(n)
    sim = statevector.New(n, _abi.GQ_C64 if args.precision == "c64" else _abi.GQ_C128)
    sim.set_option(_abi.GQ_OPT_TIMING, 1)
    sim.set_option(_abi.GQ_OPT_JIT, args.jit)
    if args.budget:
        sim.set_option(_abi.GQ_OPT_PASS_BUDGET, args.budget)
    if args.variant is not None:
        sim.set_option(_abi.GQ_OPT_KERNEL_VARIANT, args.variant)
    lib = _abi.lib()
    u = statevector.uniforms(SHOTS, np.random.default_rng(SEED))
    u_p = u.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    idx = np.empty(SHOTS, dtype=np.uint64)
    idx_p = idx.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))

    # ---- device-resident throughput: Evolve only, CUDA events on the engine stream
    # (the first warm-up call compiles the specialised pass kernels)
    t_first = time.perf_counter()
    for w in range(args.warmup):
        sim.evolve_ops(stream)
        if w == 0:
            t_first = time.perf_counter() - t_first
    # the autotuner picks the launch choices (pass budget, tile variant, CTAs
    # per SM) for this circuit, untimed; the timed steps run with its choice
    tuned = None
    if args.autotune and not args.budget and args.variant is None:
        from goqu_b200 import autotune
        t0 = time.perf_counter()
        tuned = autotune.tune_statevector(sim, stream)
        tuned = {"best": {str(k): v for k, v in tuned["best"].items()},
                 "candidates": [{str(k): v for k, v in c.items()} for c in autotune.STATEVECTOR_CANDIDATES],
                 "timings_ms": tuned.get("timings_ms"), "tuning_s": time.perf_counter() - t0,
                 "keys": "option numbers of include/gqb200.h (2 pass budget, 5 kernel variant, 11 jit min blocks, "
                         "12 persistent CTAs)"}
        sim.set_option(_abi.GQ_OPT_TIMING, 1)
        sim.set_option(_abi.GQ_OPT_JIT, args.jit)
        for _ in range(2):
            sim.evolve_ops(stream)
    barrier(world)
    step_ms, pass_ms, launches, passes, jit_passes, tile_bytes = [], [], 0, 0, 0, 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            sim.evolve_ops(stream)
            st = sim.stats()
            step_ms.append(st["last_ms"])
            pass_ms.append(st["pass_ms"])
            launches += st["kernel_launches"]
            passes += st["passes"]
            jit_passes += st["jit_passes"]
            tile_bytes += st["tile_bytes"]
    barrier(world)
    total_ms = max_over_ranks(float(np.sum(step_ms)), world)
    value = world * gates * args.steps / (total_ms / 1000.0)

    # ---- end to end through the public C ABI: gq_sv_run from host buffers
    for _ in range(2):
        _abi.check(lib.gq_sv_run(sim.handle, stream.ptr(), len(stream), u_p, SHOTS, idx_p))
    barrier(world)
    t0 = time.perf_counter()
    h2d = d2h = 0
    for _ in range(args.steps):
        _abi.check(lib.gq_sv_run(sim.handle, stream.ptr(), len(stream), u_p, SHOTS, idx_p))
        st = sim.stats()
        h2d += st["h2d_bytes"]
        d2h += st["d2h_bytes"]
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e = world * gates * args.steps / e2e_s

    # ---- roofline of the dominant kernel (the tile pass)
    peak, peak_kind = peaks()
    amp_bytes = 8 if args.precision == "c64" else 16
    full_bytes = 2 * amp_bytes * (1 << n)  # one read + one write of the whole state
    # bytes of the tiles the passes launched (the first passes from the reset
    # state skip the tiles that are still zero), averaged over the launches
    alg_bytes = tile_bytes / max(1, passes)
    per_launch_ms = float(np.sum(pass_ms)) / max(1, passes)
    achieved = alg_bytes / (per_launch_ms / 1000.0) / 1e9
    traffic = traffic_full = None
    tf = os.path.join(ROOT, "profiles", "tile_pass_traffic.json")
    if os.path.exists(tf):
        with open(tf) as f:
            tj = json.load(f)
        t = tj.get(args.precision, {})
        if t.get("bytes_per_launch"):
            traffic_full = t["bytes_per_launch"] * 2.0 ** (n - t["qubits"])  # a full-state launch; scales with 2^n
            traffic = traffic_full * alg_bytes / full_bytes

    clocks = clk.summary()
    line = {
        "metric": f"{n}q gates/s", "value": value, "unit": "gates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == "c64" else "f64",
        "data": "synthetic",
        "config": {"workload": workload_name(n, args.precision), "qubits": n, "gates": gates, "seed": SEED,
                   "precision": args.precision, "parallelism": f"replicas{world}" if world > 1 else "single",
                   "l2": f"state {amp_bytes << n >> 20} MiB vs 126 MB L2 (no flush between steps)",
                   "passes_per_step": passes / args.steps, "pass_ms_per_step": float(np.mean(pass_ms)),
                   # pass time in SM clock cycles: comparable across runs at other clocks
                   "pass_sm_mcycles_per_step": (float(np.mean(pass_ms)) * clocks["sm_mhz"] / 1000.0
                                                if clocks.get("sm_mhz") else None),
                   "zero_tile_skip": {"tile_bytes_per_step": tile_bytes / args.steps,
                                      "full_state_bytes_per_step": full_bytes * passes / args.steps}},
        "e2e": {"value": e2e, "unit": "gates/s", "h2d_bytes_per_step": h2d // args.steps,
                "d2h_bytes_per_step": d2h // args.steps},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "traffic_full_state_launch": traffic_full, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": alg_bytes, "full_state_bytes_per_launch": full_bytes,
                     "launch_ms": per_launch_ms},
        "gpu_launches": launches,
        "jit": {"mode": args.jit, "passes_specialised_per_step": jit_passes / args.steps,
                "first_call_s": t_first, "compile_ms_total": sim.stats()["jit_compile_ms"]},
        "clocks": clocks,
        "autotune": tuned,
    }
    sim.Close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n, c, stream, steps=args.cpu_steps)
    if rank == 0 and world == 1 and not args.no_extras:
        extras = {}
        for name, fn in (("parity_20q", extra_parity), ("adjoint", extra_adjoint), ("density_matrix", extra_density),
                         ("qaoa_batch", extra_qaoa), ("qaoa_dedicated", extra_qaoa_dedicated),
                         ("vqe_loop", extra_vqe), ("cold_start", extra_cold_start),
                         ("sampling", extra_sampling), ("parity_28q", extra_parity_28q)):
            try:
                extras[name] = fn()
            except Exception as exc:  # an extra must not hide the headline line
                extras[name] = {"error": repr(exc)}
        line["extras"] = extras
    if rank == 0:
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["c128", "c64"], default="c128")
    ap.add_argument("--qubits", type=int, default=28)
    ap.add_argument("--budget", type=int, default=0)
    ap.add_argument("--variant", type=int, default=None, help="fixed tile-pass launch shape (profiling; no autotuning)")
    ap.add_argument("--cpu-steps", type=int, default=3, help="stratified CPU samples for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--autotune", type=int, choices=[0, 1], default=1,
                    help="1: the autotuner picks the launch choices before the timed steps (default)")
    ap.add_argument("--jit", type=int, choices=[0, 1, 2], default=2,
                    help="specialised pass kernels: 0 off, 1 when compiled, 2 wait for them (default)")
    ap.add_argument("--only-extra", choices=["parity_20q", "adjoint", "density_matrix", "qaoa_batch", "parity_28q",
                                             "vqe_loop", "cold_start", "qaoa_dedicated", "sampling"],
                    help="run one extra workload alone and print its JSON (profiling)")
    ap.add_argument("--qaoa-qubits", type=int, default=0, help="qaoa_batch: keep the circuits of this size")
    ap.add_argument("--qaoa-count", type=int, default=0, help="qaoa_batch: keep the first N circuits")
    ap.add_argument("--qaoa-calls", type=int, default=3)
    ap.add_argument("--qaoa-graph", type=int, choices=[0, 1], default=1)
    ap.add_argument("--first-call", action="store_true", help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.first_call:
        print(json.dumps({"first_call_s": first_call(args.qubits)}))
        return
    # the run's first call compiles its kernels: a private, empty on-disk cache
    # (the cold_start extra then measures a new process reading it)
    if "GQ_JIT_CACHE_DIR" not in os.environ:
        import tempfile
        os.environ["GQ_JIT_CACHE_DIR"] = tempfile.mkdtemp(prefix="gqb200_jit_")
    if args.only_extra:
        fns = {"parity_20q": extra_parity, "adjoint": extra_adjoint, "density_matrix": extra_density,
               "parity_28q": extra_parity_28q, "vqe_loop": extra_vqe, "cold_start": extra_cold_start,
               "qaoa_dedicated": lambda: extra_qaoa_dedicated(args.qaoa_qubits, args.qaoa_count),
               "sampling": extra_sampling,
               "qaoa_batch": lambda: extra_qaoa(args.qaoa_qubits, args.qaoa_count, args.qaoa_calls,
                                                args.qaoa_graph == 1)}
        print(json.dumps({args.only_extra: fns[args.only_extra]()}))
        return
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_gpu(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
