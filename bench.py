"""Throughput of the matrix-free Lindblad path on one or more B200s.

Workload: the 12-qubit open transverse-field Ising chain (Hilbert D = 4096,
rho = 16.8M complex128 = 268 MB, 47 terms: 11 ZZ + 12 X Hamiltonian terms,
12 decay + 12 dephasing Lindblad terms; J ~ U[0.5,1.5], h ~ N(0, 0.2^2)
from a seeded generator).  One bench step is one integration segment of 25
fixed RK4 steps (dt = 0.01), i.e. 100 fused L.rho stage launches (one
time_step_sys call, whose host round trips are thus amortised over 100
applications).

metric: L.rho GB/s = applications x 32*D^2 algorithmic bytes (read rho,
write L rho, 16 B each per element) / time.  `value` has rho resident in
HBM; `e2e` goes through the C-ABI call quac_time_step_host with the state
in pinned host memory (H2D + segment + D2H every step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

For N > 1 every rank integrates its own replica (independent systems, no
collective on the data path); the time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "L·ρ GB/s; ensemble & steady-state solves/s vs plain FP64 GPU at ≤1e-8 error"
NQ = 12
DT = 0.01
RK_STEPS = 25
STAGES = 4 * RK_STEPS


def tfim_terms(S, n=NQ, seed=3):
    from quac_b200.systems import tfim
    return tfim(S, n, seed=seed)


def workload_config(n_gpus):
    return {"workload": f"tfim{NQ}_rk4_segment", "D": 2 ** NQ, "rho_bytes": 16 * 4 ** NQ,
            "rk": "rk4", "rk_steps_per_segment": RK_STEPS, "dt": DT,
            "lrho_per_step": STAGES, "terms": 47, "parallelism": f"replicas{n_gpus}",
            "l2": "inputs larger than L2 (268 MB state vs 126 MB L2)"}


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        def run():
            q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits"], capture_output=True,
                                         text=True, timeout=5).stdout.strip()
                    if out:
                        self.samples.append([x.strip() for x in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if len(s) > 3 + k and "Active" in s[3 + k] and "Not" not in s[3 + k]:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.samples)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """Per-launch DRAM bytes of the L.rho stage kernel from the committed ncu
    summary (profiles/lrho_tfim12.json), or None."""
    p = os.path.join(ROOT, "profiles", "lrho_tfim12.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get("dram_bytes_per_lrho")
    return None


def cpu_baseline(seconds=12.0, rows_frac=64):
    """The oracle's restatement of the reference algorithm (assembled CSR from
    the kron.c maps, one CSR SpMV per RK stage) on a row block of the same
    Liouvillian: 1/rows_frac of the rows, timed for about `seconds`."""
    from oracle import oracle as O
    S = O.OSys()
    tfim_terms(S)
    D = S.D
    nrows = D * D // rows_frac
    h = S.csr_handle(rows=(0, nrows))
    x = np.random.default_rng(0).normal(size=D * D) + 0j
    y = np.zeros(nrows, dtype=np.complex128)
    L = O.lib()
    import ctypes
    xp, yp = x.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p)
    L.orc_spmv(h, xp, yp)
    n = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        L.orc_spmv(h, xp, yp)
        n += 1
    dt = time.perf_counter() - t0
    O.free_csr(h)
    gbs = n * nrows * 32 / dt / 1e9
    return {"value": gbs, "unit": "GB/s", "cores": O.num_threads(), "kind": "port",
            "omp_threads": O.num_threads(), "mpi_ranks": 1,
            "sample": f"CSR SpMV over rows [0, D^2/{rows_frac}) of the D=4096 Liouvillian "
                      f"({nrows} rows), {n} applications in {dt:.1f} s, OpenMP"}


def cpu_baselines_other_configs(seconds_each=8.0):
    """The oracle's CPU restatement of the reference algorithm (assembled
    CSR, one SpMV per stage, OpenMP) on bounded samples of configs 1, 2
    and 4, in the units of their GPU sections."""
    from oracle import oracle as O
    from quac_b200 import systems as Sy
    out = {"omp_threads": O.num_threads(), "mpi_ranks": 1}
    # config 1: JC 2 x 10, fixed RK4 dt = 0.01 (no per-step observables on the CPU side)
    S = O.OSys()
    Sy.jc(S)
    h = S.csr_handle()
    y = np.zeros(400, dtype=complex)
    y[10 * 20 + 10] = 1.0
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds_each:
        y = O.rk4(h, y, 0.01, 1000)
        n += 1000
    O.free_csr(h)
    out["jc_rk4_steps_per_s"] = n / (time.perf_counter() - t0)
    # config 2: noisy 10-qubit circuit, gates (superoperator form) + 1.0 time unit of BS3 per layer
    S = O.OSys()
    Sy.noisy_qubits(S, 10)
    h = S.csr_handle()
    spec = Sy.noisy_circuit_layers(10, 40)
    y = np.zeros(1024 * 1024, dtype=complex)
    y[0] = 1.0
    n, t, t0 = 0, 0.0, time.perf_counter()
    while time.perf_counter() - t0 < seconds_each and n < len(spec):
        for g, qb, kw in spec[n]:
            y = O.gate_superop([2] * 10, y, g, list(qb), **kw)
        y, _, _ = O.bs3(h, y, t, t + 1.0, 0.1)
        t += 1.0
        n += 1
    O.free_csr(h)
    out["circuit_layers_per_s"] = n / (time.perf_counter() - t0)
    # config 4: driven JC instances one at a time, DP5 atol = rtol = 5e-7 to t = 100
    params = Sy.driven_jc_ensemble_params(4096)
    rng = np.random.default_rng(1)
    n, t0 = 0, time.perf_counter()
    for i in rng.permutation(4096):
        if time.perf_counter() - t0 >= seconds_each:
            break
        p = params[i]
        S = O.OSys()
        Sy.driven_jc(S, **p)
        h = S.csr_handle()
        O.dp5(h, Sy.excited_vacuum(p["nc"]), 0.0, 100.0, 0.05)
        O.free_csr(h)
        n += 1
    out["ensemble_solves_per_s"] = n / (time.perf_counter() - t0)
    out["samples"] = "JC: RK4 steps for ~8 s; circuit: layers for ~8 s; ensemble: random instances for ~8 s"
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    # each step: one RK4 segment's worth (STAGES applications) of CSR SpMV on the sample rows
    from oracle import oracle as O
    import ctypes
    S = O.OSys()
    tfim_terms(S)
    D = S.D
    frac = 64
    nrows = D * D // frac
    h = S.csr_handle(rows=(0, nrows))
    x = np.random.default_rng(0).normal(size=D * D) + 0j
    y = np.zeros(nrows, dtype=np.complex128)
    L = O.lib()
    xp, yp = x.ctypes.data_as(ctypes.c_void_p), y.ctypes.data_as(ctypes.c_void_p)
    for _ in range(args.warmup):
        L.orc_spmv(h, xp, yp)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for _ in range(STAGES):
            L.orc_spmv(h, xp, yp)
    dt = time.perf_counter() - t0
    O.free_csr(h)
    gbs = args.steps * STAGES * nrows * 32 / dt / 1e9
    sample = (f"each step = {STAGES} CSR SpMV over rows [0, D^2/{frac}) ({nrows} rows) of the "
              f"assembled D=4096 Liouvillian")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": gbs, "unit": "GB/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
        "data": "synthetic", "config": workload_config(args.gpus),
        "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": O.num_threads(), "kind": "port",
                         "omp_threads": O.num_threads(), "mpi_ranks": 1, "sample": sample},
        "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference PETSc build unavailable (PETSc/SLEPc absent); oracle port of the "
                "reference algorithm timed instead"}))


def ensemble_summary(q, n_inst=4096, tmax=100.0, dt0=0.05, plain_sample=8, tol=5e-7):
    """Driven Jaynes-Cummings ensemble (4096 instances, n_c ~ U{5..40}, each
    evolved to t = 100 with its own Dormand-Prince 5(4) step at atol = rtol
    = tol): solves/s of the persistent batched kernel in FP64 and with
    complex64 right-hand-side increments (steps whose error estimate lies
    within 0.1 of the accept threshold re-evaluated in complex128, and an
    instance whose estimated accumulated complex64 error passes 1e-7
    continued in complex128), against
    the plain path (time_step_sys, -ts_rk_type 5dp, one system at a time)
    timed on a sample, and the population error of the complex64 mode
    against the FP64 ensemble (which the parity tests hold to the oracle at
    1e-10)."""
    from quac_b200 import systems as Sy
    params = Sy.driven_jc_ensemble_params(n_inst)
    built = []
    for p in params:
        B = Sy.Builder(q)
        Sy.driven_jc(B, **p)
        built.append(B.qs)
    E = q.Ensemble(built)
    for qs in built:
        qs.destroy()
    rho0 = np.concatenate([Sy.excited_vacuum(p["nc"]) for p in params])
    out = {"workload": f"driven_jc_ensemble_{n_inst}", "t_end": tmax, "controller": f"DP5(4) atol=rtol={tol:g}"}
    states = {}
    for mode, name in ((0, "fp64"), (1, "fp32_rhs")):
        E.set_options(precision=mode, atol=tol, rtol=tol)
        E.set_states(rho0)
        E.run(0.0, 0.5, dt0)  # captures the graph
        E.set_states(rho0)
        t0 = time.perf_counter()
        E.run(0.0, tmax, dt0)
        dt = time.perf_counter() - t0
        states[mode] = E.get_states()
        st = E.stats()
        out[name] = {"solves_per_s": n_inst / dt, "seconds": dt, "mean_steps": float(st[:, 1].mean()),
                     "shape": list(E.shape())}
        if mode == 1:
            red = E.redone_steps()
            out[name]["redone_step_fraction"] = float(red.sum() / max(1.0, (st[:, 1] + st[:, 2]).sum()))
            f64 = E.f64_steps()
            out[name]["complex128_step_fraction"] = float(f64.sum() / max(1.0, st[:, 1].sum()))
            out[name]["instances_switched_to_complex128"] = int((f64 > 0).sum())
    pops = lambda x, i: E.state(x, i).diagonal().real
    err = np.array([np.abs(pops(states[0], i) - pops(states[1], i)).max() for i in range(n_inst)])
    out["fp32_rhs"]["pop_err_vs_fp64"] = {"median": float(np.median(err)), "p99": float(np.percentile(err, 99)),
                                          "max": float(err.max()), "frac_le_1e-8": float((err <= 1e-8).mean())}
    # plain path: one system at a time through time_step_sys
    q.set_ts_options(rk_type="5dp", adapt_type="basic", rtol=tol, atol=tol)
    rng = np.random.default_rng(0)
    tp, perr = 0.0, 0.0
    for i in rng.choice(n_inst, size=plain_sample, replace=False):
        p = params[i]
        B = Sy.Builder(q)
        Sy.driven_jc(B, **p)
        q.construct_matrix(B.qs)
        x = Sy.excited_vacuum(p["nc"])
        t0 = time.perf_counter()
        q.time_step_host(B.qs, x, 0.0, tmax, dt0, 10 ** 7)
        tp += time.perf_counter() - t0
        D = 2 * p["nc"]
        perr = max(perr, float(np.abs(x.reshape(D, D, order="F").diagonal().real - pops(states[0], i)).max()))
        B.qs.destroy()
    q.set_ts_options(rk_type="3bs", adapt_type="basic", rtol=5e-7, atol=5e-7)
    plain = plain_sample / tp
    out["plain_fp64_solves_per_s"] = plain
    out["plain_sample"] = plain_sample
    out["fp64"]["vs_plain"] = out["fp64"]["solves_per_s"] / plain
    out["fp32_rhs"]["vs_plain"] = out["fp32_rhs"]["solves_per_s"] / plain
    out["fp64"]["pop_err_vs_plain_max"] = perr
    E.destroy()
    return out


def ensemble_sharded_summary(q, rank, world, dev, n_inst=4096, tmax=100.0, dt0=0.05, tol=5e-7):
    """The config-4 ensemble on `world` GPUs: the instances are split over
    the ranks longest-first by their cost (D^2 of each instance, LPT), each
    rank integrates its share in one persistent ensemble launch (FP64
    mode), no collective on the data path; device time between CUDA events
    on the default stream, max over ranks."""
    import torch
    import torch.distributed as dist
    from quac_b200 import systems as Sy
    from quac_b200.replicas import lpt_partition, max_over_ranks
    params = Sy.driven_jc_ensemble_params(n_inst)
    costs = [(2 * p["nc"]) ** 2 for p in params]
    shares = lpt_partition(costs, world)
    mine = shares[rank]
    built = []
    for i in mine:
        B = Sy.Builder(q)
        Sy.driven_jc(B, **params[i])
        built.append(B.qs)
    E = q.Ensemble(built)
    for qs in built:
        qs.destroy()
    rho0 = np.concatenate([Sy.excited_vacuum(params[i]["nc"]) for i in mine])
    E.set_options(precision=0, atol=tol, rtol=tol)
    E.set_states(rho0)
    E.run(0.0, 0.5, dt0)  # captures the graph
    E.set_states(rho0)
    torch.cuda.synchronize()
    dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(torch.cuda.default_stream(dev))
    E.run(0.0, tmax, dt0)
    ev1.record(torch.cuda.default_stream(dev))
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    loads = [sum(costs[i] for i in s) for s in shares]
    [ms_max] = max_over_ranks([ms], device=dev)
    E.destroy()
    return {"workload": f"driven_jc_ensemble_{n_inst}", "t_end": tmax, "controller": f"DP5(4) atol=rtol={tol:g}",
            "partition": "longest-first by D^2 over ranks (lpt_partition)", "instances_per_rank":
            [len(s) for s in shares], "cost_imbalance": max(loads) / (sum(loads) / world),
            "solves_per_s": n_inst / (ms_max / 1e3), "ms_max_over_ranks": ms_max}


def precision_summary(q, qs, rho, x0, stream, steps, segment):
    """12-qubit TFIM with complex64 contraction: the headline segment timed
    again, and the full run of that workload (Dormand-Prince 5(4),
    rtol = atol = 1e-8, t = 0..50 from |0...0><0...0|) in both precisions
    with the errors of the complex64 run against the complex128 one."""
    import torch
    D = int(round(np.sqrt(x0.size)))
    out = {}
    q.set_lrho_precision(1)
    rho.from_numpy(x0)
    segment(0.0)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    t = 0.0
    for _ in range(steps):
        segment(t)
        t += RK_STEPS * DT
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    out["lrho_gbs"] = steps * STAGES * 32.0 * D * D / (ms / 1e3) / 1e9
    out["ms_per_step"] = ms / steps
    q.set_lrho_precision(0)
    states, secs = [], []
    q.set_ts_options(rk_type="5dp", adapt_type="basic", rtol=1e-8, atol=1e-8)
    for prec in (0, 1):
        q.set_lrho_precision(prec)
        z = np.zeros(D * D, dtype=np.complex128)
        z[0] = 1.0
        rho.from_numpy(z)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        q.time_step_sys(qs, rho, 0.0, 50.0, 0.01, 10 ** 7)
        torch.cuda.synchronize()
        secs.append(time.perf_counter() - t0)
        states.append(rho.to_numpy().reshape(D, D, order="F"))
    q.set_lrho_precision(0)
    q.set_ts_options(rk_type="4", adapt_type="none", rtol=5e-7, atol=5e-7)
    a, b = states
    out["run_t50_seconds"] = {"fp64": secs[0], "fp32_contraction": secs[1]}
    # Uhlmann fidelity (Tr sqrt(sqrt(a) b sqrt(a)))^2 of the two final
    # states, eigen-decompositions by torch on the GPU (measurement only)
    ta = torch.from_numpy((a + a.conj().T) / 2).cuda()
    tb = torch.from_numpy((b + b.conj().T) / 2).cuda()
    w, V = torch.linalg.eigh(ta)
    sa = (V * torch.sqrt(torch.clamp(w, min=0.0))) @ V.conj().T

    def uhlmann(t):
        ev = torch.linalg.eigvalsh(sa @ t @ sa)
        return float(torch.sum(torch.sqrt(torch.clamp(ev, min=0.0))) ** 2)

    fid = uhlmann(tb)
    # the same computation of the complex128 state against itself: the floor
    # set by the eigen-decompositions (sqrt of the state's rounding-level
    # eigenvalues), not by the complex64 contraction
    fid_self = uhlmann(ta)
    neg = float(-torch.clamp(w, max=0.0).sum())
    del ta, tb, w, V, sa
    out["errors_vs_fp64"] = {
        "trace": float(abs(np.trace(b) - np.trace(a))),
        "population_max": float(np.abs(a.diagonal().real - b.diagonal().real).max()),
        "state_rel_frobenius": float(np.linalg.norm(a - b) / np.linalg.norm(a)),
        "purity": float(abs(np.vdot(b, b).real - np.vdot(a, a).real)),
        # F(fp64, complex64) against F(fp64, fp64): the adaptive run's state
        # has slightly negative eigenvalues, which puts F(fp64, fp64) itself
        # below 1 by about twice their sum
        "fidelity": abs(fid - fid_self),
        "fidelity_floor_fp64_vs_itself": abs(1.0 - fid_self),
        "fp64_state_negative_eigenvalue_sum": neg,
    }
    return out


def jc_summary(q, t_end=200.0, dt=0.01):
    """Jaynes-Cummings (emitter 2 x cavity 10, QuaC's simple JC form): fixed
    RK4 dt = 0.01 to t = 200 (20,000 steps) with the emitter and cavity
    populations recorded after every step: through the device-side
    observable monitor (one-CTA kernel, values handed back in batches of
    1000 steps) and, for comparison, through a host TS monitor called after
    every step (simple_jc_test.c:76-90)."""
    from quac_b200.systems import Builder, jc
    out = {"workload": "jc_2x10_rk4_t200_monitored", "steps": int(round(t_end / dt))}
    for form in ("observable_monitor", "ts_monitor"):
        S = Builder(q)
        qb, cav = jc(S)
        q.construct_matrix(S.qs)
        rho = q.create_qvec_sys(S.qs)
        q.add_to_qvec(rho, 1.0, 10, 10)
        q.assemble_qvec(rho)
        pops = []
        if form == "observable_monitor":
            q.set_observable_monitor(S.qs, [(qb.n,), (cav.n,)], lambda st, tm, v: pops.extend(v.real.tolist()),
                                     batch=1000)
        else:
            q.set_ts_monitor_sys(S.qs, lambda step, t, v: pops.append(
                (q.get_expectation_value_qvec(rho, qb.n).real, q.get_expectation_value_qvec(rho, cav.n).real)))
        q.set_ts_options(rk_type="4", adapt_type="none")
        t0 = time.perf_counter()
        q.time_step_sys(S.qs, rho, 0.0, t_end, dt, 10 ** 7)
        sec = time.perf_counter() - t0
        q.set_ts_options(rk_type="3bs", adapt_type="basic")
        q.set_ts_monitor_sys(S.qs, None)
        q.set_observable_monitor(S.qs, None, None)
        nrec = len(pops) if form == "observable_monitor" else len(pops) - 1
        out[form] = {"seconds": sec, "steps_per_s": out["steps"] / sec, "records": nrec,
                     "final_populations": {"emitter": pops[-1][0], "cavity": pops[-1][1]}}
        rho.destroy()
        S.qs.destroy()
    out["steps_per_s"] = out["observable_monitor"]["steps_per_s"]
    out["vs_ts_monitor"] = out["observable_monitor"]["steps_per_s"] / out["ts_monitor"]["steps_per_s"]
    return out


def circuit_summary(q, nq=10, layers=40):
    """Noisy 10-qubit random circuit on rho (D = 1024): per layer the gates
    (superoperator convention, apply_circuit_to_qvec) and then 1.0 time unit
    of Lindblad evolution (default adaptive BS3); fidelity against the ideal
    state obtained by applying the same gates to a second, noiseless rho."""
    from quac_b200.systems import Builder, noisy_circuit_layers, noisy_qubits
    S = Builder(q)
    noisy_qubits(S, nq)
    q.construct_matrix(S.qs)
    rho = q.create_dm_sys(S.qs)
    ideal = q.create_dm_sys(S.qs)
    for v in (rho, ideal):
        q.add_to_qvec(v, 1.0, 0, 0)
        q.assemble_qvec(v)
    spec = noisy_circuit_layers(nq, layers)
    circs = []
    for layer in spec:
        c = q.create_circuit(len(layer))
        for g, qb, kw in layer:
            c.add_gate(0.0, g, *qb, **kw)
        circs.append(c)
    t0 = time.perf_counter()
    t = 0.0
    for c in circs:
        q.apply_circuit_to_qvec(S.qs, c, rho)
        q.time_step_sys(S.qs, rho, t, t + 1.0, 0.1, 10 ** 6)
        t += 1.0
    sec = time.perf_counter() - t0
    for c in circs:
        q.apply_circuit_to_qvec(S.qs, c, ideal)
    D = S.D
    a = rho.to_numpy()
    b = ideal.to_numpy()
    fid = float(np.vdot(b, a).real)  # Tr(rho_ideal rho) for a pure rho_ideal
    tr = complex(np.trace(a.reshape(D, D, order="F")))
    out = {"workload": f"noisy_random_circuit_{nq}q_{layers}layers", "seconds": sec, "layers_per_s": layers / sec,
           "fidelity_vs_ideal": fid, "trace_error": abs(tr - 1.0)}
    rho.destroy()
    ideal.destroy()
    S.qs.destroy()
    return out


def steady_summary(q):
    """Steady states of driven Tavis-Cummings at the configuration's size:
    6 emitters and 8 cavity levels (D = 512, Liouville dimension 262,144),
    a 4-D sweep of (Omega, Delta, kappa, gamma); 100 solver-generated
    training states and 20 held-out points (the configuration's 2,000 / 500
    would take about 10 minutes of generation alone).  Solves/s of plain
    complex128 GMRES(100) from e0 (one point: about 35 k iterations), of the
    same GMRES preconditioned by the exact inverse of the no-jump
    Liouvillian (the method, from e0) and of the learned start with the
    preconditioned complex64-inner / complex128-refined solver; every solve
    to ||b - A x|| <= 1e-12 (tighter than the configuration's 1e-10, so
    that the arms agree on populations to 1e-8)."""
    from quac_b200 import warmstart as WS
    out = WS.measure_sweep(q, WS.sweep_settings(ne=6, nc=8, train=100, held=20, precond=2, cold_sample=1,
                                                steps=4000, fp32=1, rtol=1e-12))
    return {k: out[k] for k in ("workload", "sweep", "train_states", "held_out", "rtol", "solver", "generation",
                                "training",
                                "cold", "method", "learned", "learned_vs_cold", "learned_vs_method",
                                "learned_vs_method_median_point",
                                "method_vs_cold", "decompositions", "pop_err_max", "residual_max")}


def run_ours(args, rank, world, local_rank):
    import torch
    import quac_b200 as q
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    q.lib()
    q.QuaC_initialize()
    from quac_b200.systems import Builder
    S = Builder(q)
    tfim_terms(S)
    qs = S.qs
    q.construct_matrix(qs)
    D = S.D
    n = D * D
    rho = q.create_dm_sys(qs)
    rng = np.random.default_rng(1234 + rank)
    X = (rng.standard_normal((D, D)) + 1j * rng.standard_normal((D, D))).astype(np.complex128)
    X = (X + X.conj().T) / 2.0
    x0 = np.ascontiguousarray(X.reshape(-1, order="F"))
    rho.from_numpy(x0)
    stream = torch.cuda.Stream(device=dev)
    q.set_stream(qs, stream.cuda_stream)
    q.set_ts_options(rk_type="4", adapt_type="none")

    def segment(t):
        q.time_step_sys(qs, rho, t, t + RK_STEPS * DT, DT, 10 ** 9)

    t = 0.0
    for _ in range(args.warmup):
        segment(t)
        t += RK_STEPS * DT
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    clocks = Clocks(local_rank)
    clocks.start()
    launches0 = q.kernel_launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    seg_ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    torch.cuda.synchronize()
    ev0.record(stream)
    for k in range(args.steps):
        seg_ev[k].record(stream)
        segment(t)
        t += RK_STEPS * DT
    seg_ev[args.steps].record(stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = q.kernel_launch_count() - launches0
    ms = ev0.elapsed_time(ev1)
    seg_ms = [seg_ev[k].elapsed_time(seg_ev[k + 1]) for k in range(args.steps)]
    clk = clocks.stop()
    # the same segment with Hermitian mode off (every element computed and
    # stored by both passes), for comparison with the headline
    q.set_hermitian_mode(0)
    segment(t)
    t += RK_STEPS * DT
    fe0 = torch.cuda.Event(enable_timing=True)
    fe1 = torch.cuda.Event(enable_timing=True)
    nfull = max(1, min(args.steps, 5))
    torch.cuda.synchronize()
    fe0.record(stream)
    for _ in range(nfull):
        segment(t)
        t += RK_STEPS * DT
    fe1.record(stream)
    torch.cuda.synchronize()
    full_ms = fe0.elapsed_time(fe1) / nfull
    q.set_hermitian_mode(1)
    # e2e through the C ABI with host (pinned) buffers
    host = torch.from_numpy(x0.copy()).pin_memory()
    hp = host.numpy()
    q.set_stream(qs, None)
    q.time_step_host(qs, hp, 0.0, RK_STEPS * DT, DT, 10 ** 9)
    torch.cuda.synchronize()
    e2e_steps = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ts = time.perf_counter()
        q.time_step_host(qs, hp, 0.0, RK_STEPS * DT, DT, 10 ** 9)
        e2e_steps.append((time.perf_counter() - ts) * 1e3)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3
    from quac_b200.replicas import max_over_ranks
    ms, e2e_ms = max_over_ranks([ms, e2e_ms], device=dev)
    alg_bytes = 32.0 * n
    total_apps = args.steps * STAGES * world
    value = total_apps * alg_bytes / (ms / 1e3) / 1e9
    e2e = total_apps * alg_bytes / (e2e_ms / 1e3) / 1e9
    per_launch_ms = ms / (args.steps * STAGES)
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    traffic = profiled_traffic()
    out = {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": workload_config(world),
        "e2e": {"value": e2e, "unit": "GB/s", "h2d_bytes_per_step": 16 * n,
                "d2h_bytes_per_step": 16 * n,
                "step_ms": {"min": min(e2e_steps), "median": statistics.median(e2e_steps), "max": max(e2e_steps)}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "frac_of_nominal_8tbs": achieved / 8000.0,
                     "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)",
                     "kernel": "Hermitian mode: k_qpass over tile pairs (a <= b) of the high-qubit pass, "
                               "then k_qpass over the blocks I <= J of the low-qubit pass with the fused RK "
                               "stage epilogue and conjugate-transposed writes",
                     "per": "one L.rho application (32*D^2 algorithmic bytes)"},
        "gpu_launches": int(launches),
        "clocks": clk,
        "segment_ms": {"min": min(seg_ms), "median": statistics.median(seg_ms), "max": max(seg_ms)},
        "full_mode": {"value": STAGES * 32.0 * n / (full_ms / 1e3) / 1e9, "unit": "GB/s", "ms_per_step": full_ms,
                      "note": "Hermitian mode off: both passes compute and store every element (segments after "
                              "the timed region, same workload)"},
    }
    if world > 1 and not args.no_ensemble:
        # every rank takes part (its share of the instances, one max over ranks)
        out["ensemble_sharded"] = ensemble_sharded_summary(q, rank, world, dev)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline()
    if rank == 0 and world == 1 and not args.no_ensemble:
        q.set_stream(qs, stream.cuda_stream)
        out["fp32_contraction"] = precision_summary(q, qs, rho, x0, stream, args.steps, segment)
        q.set_stream(qs, None)
        out["ensemble"] = ensemble_summary(q)
        out["ensemble_tight"] = ensemble_summary(q, tol=1e-10)
        out["jc"] = jc_summary(q)
        out["circuit"] = circuit_summary(q)
        out["steady_state"] = steady_summary(q)
        if not args.no_cpu_baseline:
            out["cpu_baseline_other_configs"] = cpu_baselines_other_configs()
    q.set_ts_options(rk_type="3bs", adapt_type="basic")
    rho.destroy()
    qs.destroy()
    return out


def run_profile(args):
    """Small cases of single kernels for profiler captures (no JSON line):

      --profile lrho     --qubits N --reps R [--fp32] [--path P]   L.x applications on device buffers
      --profile rk4      --qubits N --rk4-steps K [--fp32]         fixed RK4 from a Hermitian state
                                                                     (Hermitian mode of the pass kernel)
      --profile ensemble --instances N --t-end T [--fp32]          one persistent ensemble launch
      --profile gemm     --m M --n N --k K --reps R                 TF32 tensor-core GEMM
      --profile steady   --ne E --nc C --train T --held H --kd K --restart M --fp32-basis B --sweep2d
                         --precond P --cold-sample S --train-steps N --rtol R   one steady-state sweep
                                                                     learned warm-start sweep
    """
    import ctypes
    import torch
    import quac_b200 as q
    from quac_b200 import systems as Sy
    q.lib()
    q.QuaC_initialize()
    q.set_lrho_precision(1 if args.fp32 else 0)
    if args.profile in ("lrho", "rk4"):
        q.set_kernel_path(args.path)
        S = Sy.Builder(q)
        tfim_terms(S, n=args.qubits)
        q.construct_matrix(S.qs)
        D = S.D
        if args.profile == "rk4":
            q.set_stream(S.qs, torch.cuda.current_stream().cuda_stream)
            X = torch.randn(D, D, dtype=torch.complex128)
            X = (X + X.conj().T) / 2
            rho = q.create_dm_sys(S.qs)
            rho.from_numpy(X.T.contiguous().reshape(-1).numpy())  # column-stacked
            q.set_ts_options(rk_type="4", adapt_type="none")
            for rep in range(max(1, args.reps)):
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                ev0.record()
                q.time_step_sys(S.qs, rho, 0.0, DT * args.rk4_steps, DT, 10 ** 6)
                ev1.record()
                torch.cuda.synchronize()
                print(f"ok D={D} rk4 steps={args.rk4_steps} hermitian applications={q.hermitian_apply_count()} "
                      f"{ev0.elapsed_time(ev1) / (4 * args.rk4_steps) * 1e3:.1f} us per L.rho")
            return
        x = torch.randn(D * D, dtype=torch.complex128, device="cuda")
        y = torch.empty_like(x)
        for _ in range(args.reps):
            q.lrho_apply_device(S.qs, x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        print(f"ok D={D} reps={args.reps} launches={q.kernel_launch_count()}")
    elif args.profile == "ensemble":
        params = Sy.driven_jc_ensemble_params(args.instances)
        built = []
        for p in params:
            B = Sy.Builder(q)
            Sy.driven_jc(B, **p)
            built.append(B.qs)
        E = q.Ensemble(built)
        E.set_options(precision=1 if args.fp32 else 0)
        E.set_states(np.concatenate([Sy.excited_vacuum(p["nc"]) for p in params]))
        t0 = time.perf_counter()
        E.run(0.0, args.t_end, 0.05)
        print(f"ok {args.instances} instances to t={args.t_end} in {(time.perf_counter() - t0) * 1e3:.1f} ms")
        E.destroy()
    elif args.profile == "gemm":
        L = q.lib()
        L.quac_gemm_tf32.restype = ctypes.c_int
        L.quac_gemm_tf32.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int] * 4
        A = torch.randn(args.m, args.k, device="cuda")
        Bm = torch.randn(args.n, args.k, device="cuda")
        bias = torch.randn(args.n, device="cuda")
        C = torch.empty(args.m, args.n, device="cuda")
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for i in range(args.reps):
            if i == args.reps - 1:
                ev0.record()
            assert L.quac_gemm_tf32(A.data_ptr(), Bm.data_ptr(), C.data_ptr(), bias.data_ptr(),
                                    args.m, args.n, args.k, 0) == 0
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        print(f"ok {args.m}x{args.n}x{args.k}: {ms * 1e3:.1f} us per GEMM, "
              f"{2.0 * args.m * args.n * args.k / ms / 1e9:.1f} TFLOP/s")
    elif args.profile == "steady":
        from quac_b200 import warmstart
        a = warmstart.sweep_settings(ne=args.ne, nc=args.nc, train=args.train, held=args.held, kd=args.kd,
                                     restart=args.restart, fp32=args.fp32_basis, sweep2d=args.sweep2d,
                                     precond=args.precond, cold_sample=args.cold_sample, steps=args.train_steps,
                                     rtol=args.rtol)
        print(json.dumps(warmstart.measure_sweep(q, a)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true",
                    help="skip the sections beside the headline (complex64, ensemble, JC, circuit, steady state)")
    ap.add_argument("--profile", choices=["lrho", "rk4", "ensemble", "gemm", "steady"],
                    help="run one small case for a profiler capture instead of the benchmark")
    ap.add_argument("--qubits", type=int, default=NQ)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--path", type=int, default=0)
    ap.add_argument("--fp32", action="store_true")
    ap.add_argument("--rk4-steps", type=int, default=2)
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--t-end", type=float, default=2.0)
    ap.add_argument("--m", type=int, default=4096)
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--k", type=int, default=4096)
    ap.add_argument("--ne", type=int, default=3)
    ap.add_argument("--nc", type=int, default=4)
    ap.add_argument("--train", type=int, default=48)
    ap.add_argument("--held", type=int, default=12)
    ap.add_argument("--kd", type=int, default=8)
    ap.add_argument("--restart", type=int, default=300)
    ap.add_argument("--fp32-basis", type=int, default=1)
    ap.add_argument("--sweep2d", action="store_true")
    ap.add_argument("--precond", type=int, default=1)
    ap.add_argument("--cold-sample", type=int, default=None)
    ap.add_argument("--train-steps", type=int, default=8000)
    ap.add_argument("--rtol", type=float, default=1e-11)
    args = ap.parse_args()
    if args.profile:
        run_profile(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    out = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
