#!/usr/bin/env python
"""Benchmark: TJM trajectory-steps/s of the analog engine, mixed-precision
form against the plain FP64 form.

Workload (default): the L=30 Heisenberg chain H = sum(XX+YY+ZZ) + 0.3 sum Z
(init_general_hamiltonian(30,1,1,1,0,0,0.3)), dephasing (pauli_z, gamma=0.05)
on every site, dt=0.05, 1-site TDVP with 2-site growth up to bond dimension
64 (the local dynamic TDVP of the Python lineage; --tdvp 2site runs the Julia
reference's two_site_tdvp! instead), threshold 1e-9, second-order TJM with
sampling at every time index, <Z_i> on all 30 sites plus the half-chain
entropy, 1024 trajectories per GPU, Philox draws.  The start state is an MPS
with every bulk bond already at 64 (Gaussian entries, normalised by the
engine) so every timed step runs at chi=64; with --start neel the run
starts from the Neel state instead.

The default form is the mixed-precision one (H_eff products in complex FP32
on tcgen05, Lanczos/SVD/QR/norms in FP64); the plain ComplexF64 form is
timed beside it in the same process on the same problem and draws
(vs_baseline = mixed / plain, the metric's comparison), and every recorded
<Z_i> and S_half of the two runs gives the error against FP64.

A step is one recorded time index of every trajectory (two TDVP sweeps,
dissipation, jump, measurement).  W untimed steps, then K timed steps,
bracketed by a barrier and a device synchronisation; device time from CUDA
events on the launching stream; the trajectory states (2.5 GB) are larger
than L2.  Multi-GPU runs are independent replicas (one process per GPU,
launched by torchrun); the value is the sum of every rank's trajectory-steps
over the slowest rank's time.

--workload digital times the digital TJM instead: a Trotterised Ising
circuit on L=40 qubits (per Trotter layer RZZ(2 J dt) on odd then even
bonds, RX(2 g dt) on every qubit, a SAMPLE_OBSERVABLES barrier; J = g = 1,
dt = 0.05, 60 layers), Pauli X/Y/Z noise 0.01 per qubit after every 2-qubit
gate, TEBD with chi_max = 128 and threshold 1e-9, 512 trajectories, <Z_i> on
every qubit after every layer.  A step is one Trotter layer of every
trajectory.

--impl reference times the CPU restatement of the reference algorithm
(the reference itself is Julia, not runnable here) on all host cores with
its contractions on OpenBLAS zgemm, on bounded samples of the same workload.
"""
from __future__ import annotations

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

from yaqs_julia_b200 import _abi as A  # noqa: E402
from yaqs_julia_b200 import api  # noqa: E402

# the same for the digital workload: (L, trajectories, timed layers) -> bytes
DIG_TIMED_TRAFFIC = {(40, 512, 57): 4.458638080e9 + 15.767363584e9}

METRIC = "TJM trajectory-steps/s (L=30 Heisenberg, chi=64, 1024 trajectories) vs plain FP64 GPU"
# DRAM read + write bytes per trajectory-step of the trajectory kernel, from
# one small-case ncu capture per configuration: (precision, tdvp, L, chi) -> bytes
TRAFFIC_PER_TRAJ_STEP = {("mixed", "dynamic", 30, 64): 276.942e9 / 148 + 189.476e9 / 148,
                         ("fp64", "dynamic", 30, 64): 438.298e9 / 148 + 252.204e9 / 148}
TDVP_NAMES = {"dynamic": A.YAQS_TDVP_DYNAMIC, "2site": A.YAQS_TDVP_2SITE, "1site": A.YAQS_TDVP_1SITE}
TDVP = [A.YAQS_TDVP_DYNAMIC]  # set from --tdvp
TDVP_DESC = {"dynamic": "1-site TDVP with 2-site growth (local dynamic TDVP)", "2site": "2-site TDVP",
             "1site": "1-site TDVP"}
UNIT = "trajectory-steps/s"
SEED = 0xC0FFEE02


def workload(L, chi, n_times, num_traj, start):
    H = api.init_general_hamiltonian(L, 1, 1, 1, 0, 0, 0.3)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    obs.append(api.Observable("S_half", None, L // 2, kind="entropy"))
    cfg = api.TimeEvolutionConfig(obs, (n_times - 1) * 0.05, dt=0.05, num_traj=num_traj, max_bond_dim=chi,
                                  truncation_threshold=1e-9)
    assert len(cfg.times) == n_times, (len(cfg.times), n_times)
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [i], "strength": 0.05} for i in range(1, L + 1)], L)
    psi = api.random_mps(L, chi, seed=1) if start == "sat" else api.MPS(L, state="Neel")
    return psi, H, cfg, nm


DIG_METRIC = "digital TJM trajectory-layers/s (L=40 Ising Trotter circuit, chi=128, 512 trajectories)"
DIG_UNIT = "trajectory-layers/s"
DIG_SEED = 0xC0FFEE03
DIG_DEPTH = 60


def digital_workload(L, depth, num_traj, chi=128):
    J = g = 1.0
    dt = 0.05
    c = api.DigitalCircuit(L)
    for _ in range(depth):
        for i in list(range(1, L, 2)) + list(range(2, L, 2)):
            c.add_gate(api.Rzz(2 * J * dt), [i, i + 1])
        for i in range(1, L + 1):
            c.add_gate(api.Rx(2 * g * dt), [i])
        c.add_gate(api.Barrier(), [])
    nm = api.NoiseModel([{"name": n, "sites": [i], "strength": 0.01} for i in range(1, L + 1)
                         for n in ("pauli_x", "pauli_y", "pauli_z")], L)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=1.0, num_traj=num_traj, max_bond_dim=chi,
                                  truncation_threshold=1e-9)
    return api.MPS(L), c, cfg, nm


BATCH_SEED = 0xC0FFEE04
SERVE_SEED = 0xC0FFEE05


def batch_requests(n=64, steps=40, seed=BATCH_SEED):
    """64 independent analog simulations with seeded parameters: model in
    {Ising g~U[0.2,1.5], XY init_general_hamiltonian(L,1+a,1-a,0,0,0,0)
    a~U[0,1], Heisenberg (1,1,1,0,0,h) h~U[0,1]}, L in {8,...,64}, chi_max in
    {16,...,128}, 64..512 trajectories, lowering and pauli_z noise with
    gamma~U[0.01,0.2], dt = 0.05, `steps` steps, <Z_i> on every site.  Ising
    starts from |0...0>, XY and Heisenberg from the Neel state."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        model = int(rng.integers(3))
        L = int(rng.choice([8, 16, 24, 32, 48, 64]))
        chi = int(rng.choice([16, 32, 64, 128]))
        nt = int(rng.integers(64, 513))
        g1, g2 = rng.uniform(0.01, 0.2, 2)
        if model == 0:
            par = float(rng.uniform(0.2, 1.5))
            H, name, state = api.init_ising(L, 1.0, par), "ising", "zeros"
        elif model == 1:
            par = float(rng.uniform(0, 1))
            H, name, state = api.init_general_hamiltonian(L, 1 + par, 1 - par, 0, 0, 0, 0), "xy", "Neel"
        else:
            par = float(rng.uniform(0, 1))
            H, name, state = api.init_general_hamiltonian(L, 1, 1, 1, 0, 0, par), "heisenberg", "Neel"
        obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
        cfg = api.TimeEvolutionConfig(obs, steps * 0.05, dt=0.05, num_traj=nt, max_bond_dim=chi)
        nm = api.NoiseModel([{"name": "lowering", "sites": [i], "strength": g1} for i in range(1, L + 1)] +
                            [{"name": "pauli_z", "sites": [i], "strength": g2} for i in range(1, L + 1)], L)
        out.append({"name": name, "par": par, "L": L, "chi": chi, "nt": nt, "w": max(H.bond_dims),
                    "problem": (api.MPS(L, state=state), H, cfg, nm), "seed": 1000 + k})
    return out


def ring_request(rng):
    """A QAOA ring request: n in {12,20,32,48}, p in {1,2,4} layers of RZZ on
    every ring edge (odd bonds, even bonds, then the (n,1) edge through the
    SWAP chain) then RX, angles
    ~U[0,pi], Pauli X/Y/Z noise 0.005/3 each per gate, chi_max = 64,
    128..1024 trajectories, <Z_i Z_i+1> on the adjacent pairs."""
    n = int(rng.choice([12, 20, 32, 48]))
    p = int(rng.choice([1, 2, 4]))
    nt = int(rng.integers(128, 1025))
    c = api.DigitalCircuit(n)
    for _ in range(p):
        g, b = rng.uniform(0, np.pi, 2)
        for i in list(range(1, n, 2)) + list(range(2, n, 2)):  # odd then even bonds
            c.add_gate(api.Rzz(g), [i, i + 1])
        c.add_gate(api.Rzz(g), [n, 1])
        for i in range(1, n + 1):
            c.add_gate(api.Rx(b), [i])
    nm = api.NoiseModel([{"name": nme, "sites": [i], "strength": 0.005 / 3} for i in range(1, n + 1)
                         for nme in ("pauli_x", "pauli_y", "pauli_z")], n)
    obs = [api.Observable(f"ZZ{i}", np.kron(api.Z, api.Z), [i, i + 1]) for i in range(1, n)]
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=1.0, num_traj=nt, max_bond_dim=64)
    return {"n": n, "p": p, "nt": nt, "problem": (api.MPS(n), c, cfg, nm)}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        sm, smax, pw = [], [], []
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                pw.append(float(r[3]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(pw) if pw else None, "samples": len(sm), "reasons": sorted(reasons)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        return ws, rank, local, dist
    return 1, 0, 0, None


def barrier_sync(dist):
    if dist is not None:
        dist.barrier()
    import torch
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def reduce_max(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(dist, v):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def cpu_sample(L, chi, start):
    """The reference path on the host cores: the oracle (CPU restatement,
    test infrastructure) with its contractions on OpenBLAS zgemm (the
    reference's backend), one trajectory per core, 4 recorded time indices
    from the same saturated start.  Order-2 sampling runs 2 (n - 1) - 1 = 5
    TDVP sweeps for those 3 indices, and a timed GPU step runs 2, so the rate
    counts 5 / 2 trajectory-steps per trajectory.  Returns (trajectory-steps/s,
    cores, sample text, BLAS description)."""
    from oracle import oracle as O
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    psi, H, cfg, nm = workload(L, chi, 4, cores, start)
    d = api.Descriptors(psi, H, cfg, nm, seed=SEED, tdvp_mode=TDVP[0])
    blas = O.set_blas(True)
    try:
        t0 = time.perf_counter()
        O.analog_run(d, nthreads=cores)
        dt = time.perf_counter() - t0
    finally:
        O.set_blas(False)
    steps = cores * 2.5
    return (steps / dt, cores, f"{cores} trajectories x 4 time indices (5 TDVP sweeps = 2.5 trajectory-steps each) "
                               f"of the same workload from the same saturated start, {dt:.1f} s", blas)


def cpu_sample_digital(L, depth):
    """Oracle on all host cores: 2 full-circuit trajectories per core.
    Returns (trajectory-layers/s, cores, sample text)."""
    from oracle import oracle as O
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    psi, c, cfg, nm = digital_workload(L, depth, 2 * cores)
    d = api.CircuitDescriptors(psi, c, cfg, nm, seed=DIG_SEED)
    t0 = time.perf_counter()
    O.digital_run(d, nthreads=cores)
    dt = time.perf_counter() - t0
    return 2 * cores * depth / dt, cores, f"{2 * cores} trajectories x {depth} layers of the same circuit, {dt:.1f} s"


START_DESC = {"sat": "saturated start", "neel": "Neel start"}


def analog_config(args, L, chi, nt, ws):
    """The analog workload's config object (shared by both bench arms)."""
    return {"workload": f"analog TJM, L={L} Heisenberg XXX h=0.3, dephasing gamma=0.05, dt=0.05, "
                        f"{TDVP_DESC[args.tdvp]} chi_max={chi}, thr=1e-9, {nt} trajectories per GPU, "
                        f"start={'saturated chi MPS' if args.start == 'sat' else 'Neel'}",
            "L": L, "chi": chi, "num_traj": nt, "dt": 0.05, "parallelism": f"replicas x{ws}",
            "precision": args.precision, "tdvp": args.tdvp,
            "l2": "inputs larger than L2: %d trajectory states of up to %.1f MB each" % (
                nt, sum(min(2 ** min(b, L - b), chi) * 2 * min(2 ** min(b + 1, L - b - 1), chi)
                        for b in range(L)) * 16 / 1e6)}


def run_reference(args):
    ws, rank, local, dist = dist_setup()
    if rank != 0:
        return
    if args.workload == "digital":
        vals = []
        for k in range(args.warmup + args.steps):
            v, cores, sample = cpu_sample_digital(40, DIG_DEPTH)
            if k >= args.warmup:
                vals.append(v)
        value = float(np.mean(vals))
        line = {"impl": "reference", "metric": DIG_METRIC, "value": value, "unit": DIG_UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "c128", "data": "synthetic",
                "config": {"workload": "digital TJM, L=40 Ising Trotter circuit, 60 layers, chi=128"},
                "cpu_baseline": {"value": value, "unit": DIG_UNIT, "cores": cores, "kind": "port", "sample": sample},
                "e2e": {"value": value, "unit": DIG_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "reference Julia (Yaqs.jl) cannot run here; CPU restatement (oracle/tjm_oracle.cpp)"}
        print(json.dumps(line), flush=True)
        return
    vals = []
    nrep = max(1, min(args.steps, 3))  # bounded: each repetition is ~10 s of host work
    for k in range(min(args.warmup, 1) + nrep):
        v, cores, sample, blas = cpu_sample(args.L, args.chi, args.start)
        if k >= min(args.warmup, 1):
            vals.append(v)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": analog_config(args, args.L, args.chi, args.traj, args.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "blas": blas,
                             "sample": f"{nrep} timed samples after 1 untimed: " + sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Julia (Yaqs.jl) cannot run here; CPU restatement (oracle/tjm_oracle.cpp) in "
                    "ComplexF64 with its contractions on OpenBLAS zgemm"}
    print(json.dumps(line), flush=True)


def desc_bytes(desc, n_obs, n_out, num_traj, L):
    h2d = 0
    for t in desc._keep:
        if isinstance(t, np.ndarray):
            h2d += t.nbytes
        elif isinstance(t, list):
            h2d += sum(x.nbytes for x in t if isinstance(x, np.ndarray))
    h2d += C_sizeof(desc)
    d2h = num_traj * n_obs * n_out * 8 + n_obs * n_out * 8 + num_traj * n_out * 4 + num_traj * 4
    return h2d, d2h


def C_sizeof(desc):
    import ctypes as C
    return C.sizeof(desc.noise) + C.sizeof(desc.obs) + C.sizeof(desc.cfg) + C.sizeof(desc.rng)


def run_digital(args):
    """The digital TJM workload: W untimed Trotter layers, then the timed ones."""
    ws, rank, local, dist = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from yaqs_julia_b200 import _lib
    ctx = _lib.Context(local)
    L, nt, depth = 40, args.traj or 512, DIG_DEPTH
    K = args.steps if args.steps_given else depth - args.warmup
    if args.warmup + K > depth:
        raise SystemExit(f"--warmup + --steps must be <= {depth}")
    psi, c, cfg, nm = digital_workload(L, depth, nt)
    n_layers, n_samples = api.digital_plan(c)
    per = n_layers // depth
    assert per * depth == n_layers and n_samples == depth
    desc = api.CircuitDescriptors(psi, c, cfg, nm, seed=DIG_SEED, traj_offset=rank * nt)
    sess = api.Session(desc, ctx)
    sess.advance(1 + per * args.warmup)
    st0 = sess.stats()
    clocks = ClockSampler(local)
    barrier_sync(dist)
    clocks.start()
    dev_ms = sess.advance(per * K)
    barrier_sync(dist)
    ck = clocks.stop()
    st1 = sess.stats()
    phases = sess.profile() if args.profile else None
    res = sess.finish()
    t_max = reduce_max(dist, dev_ms / 1e3)
    value = reduce_sum(dist, nt * K) / t_max
    import ctypes as C
    pk = C.c_double(0.0)
    ctx.check(ctx._lib.yaqs_fp64_peak(ctx.handle, C.byref(pk)))
    achieved = (st1["flops"] - st0["flops"]) / (dev_ms / 1e3) / 1e12
    # end to end: the public call on host buffers (marshalling, uploads,
    # the run, result reads); the circuit object is the caller's input and
    # is built before the clock starts, as the analog leg builds its MPS/MPO
    e2e_psi = digital_workload(L, depth, nt)
    barrier_sync(dist)
    t0 = time.perf_counter()
    e2e_desc = api.CircuitDescriptors(*e2e_psi, seed=DIG_SEED, traj_offset=rank * nt)
    api.run_circuit_descriptors(e2e_desc, ctx)
    barrier_sync(dist)
    e2e_s = reduce_max(dist, time.perf_counter() - t0)
    e2e_value = reduce_sum(dist, nt * depth) / e2e_s
    h2d = (sum(t.nbytes for t in e2e_psi[0].tensors) + 4 * (L + 1) + C.sizeof(e2e_desc.gates) +
           C_sizeof(e2e_desc))
    d2h = nt * L * depth * 8 + L * depth * 8 + nt * depth * 4 + nt * 4
    cpu = None
    if rank == 0 and not args.no_cpu and ws == 1:
        v, cores, sample = cpu_sample_digital(L, depth)
        cpu = {"value": v, "unit": DIG_UNIT, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        line = {"metric": DIG_METRIC, "value": value, "unit": DIG_UNIT, "n_gpus": ws, "steps": K,
                "warmup": args.warmup, "ms_per_step": dev_ms / K, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "c128", "data": "synthetic",
                "config": {"workload": f"digital TJM, L={L} Ising Trotter circuit (RZZ odd/even, RX all; J=g=1, "
                                       f"dt=0.05), {depth} layers, Pauli XYZ noise 0.01 after every 2-qubit gate, "
                                       f"TEBD chi_max=128 thr=1e-9, {nt} trajectories per GPU",
                           "L": L, "chi": 128, "num_traj": nt, "layers": depth, "parallelism": f"replicas x{ws}",
                           "l2": "working set below L2 (bond dimensions stay small); every layer rereads the "
                                 "trajectory states, no flush"},
                "gpu_launches": 1,  # one digital_step_kernel launch covers the timed layers
                "roofline": {"bound": "tensor", "achieved": achieved, "peak": pk.value, "unit": "TFLOP/s",
                             "frac": achieved / pk.value if pk.value else None,
                             "traffic": DIG_TIMED_TRAFFIC.get((L, nt, K)),
                             "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the timed "
                                               "launch (profiles/digital_step_kernel_L40_ising_512traj.md); "
                                               "null for configurations not captured",
                             "kernel": "digital_step_kernel",
                             "peak_source": "measured FP64 DFMA probe (yaqs_fp64_peak) in this run",
                             "achieved_counts": "nominal TEBD work: theta merge GEMM + 4x4 gate + SVD as "
                                                "4 m n min(m,n) complex MACs (8 flops each)"},
                "e2e": {"value": e2e_value, "unit": DIG_UNIT, "h2d_bytes_per_step": h2d / depth,
                        "d2h_bytes_per_step": d2h / depth, "seconds": e2e_s},
                "cpu_baseline": cpu, "clocks": ck,
                "stats": {"jumps": res.stats["jumps"], "svds": res.stats["svds"],
                          "max_bond": int(res.max_bond.max())}}
        if phases:
            tot = phases["step"] or 1.0
            line["phases_pct_of_step"] = {k: round(100 * v / tot, 2) for k, v in phases.items()}
            line["phases_note"] = "tdvp_sweep = TEBD gate application, jump_step = gate noise step"
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_batch(args):
    """64 uneven analog simulations through one server (all admitted runs share
    each persistent launch); value = total trajectory-steps / wall time."""
    import torch
    torch.cuda.set_device(0)
    from yaqs_julia_b200 import _lib
    ctx = _lib.Context(0)
    steps = args.steps if args.steps_given else 40
    reqs = batch_requests(steps=steps)
    # bucket order: (chi, MPO width), so similar runs sit next to each other in every launch
    reqs.sort(key=lambda r: (r["chi"], r["w"], r["L"]))
    prec = args.precision
    clocks = ClockSampler(0)
    limit = args.time_limit
    with api.Server(max_L=64, max_bond_dim=128, max_mpo_width=5, mixed=True, chunk=args.chunk, ctx=ctx) as srv:
        clocks.start()
        t0 = time.perf_counter()
        ids = [srv.submit(*r["problem"], seed=r["seed"], precision=prec, tdvp=args.tdvp) for r in reqs]
        # wait for every run, printing a progress record each minute; with a
        # time limit, stop there and report what finished
        done, last = set(), t0
        while len(done) < len(ids):
            for k, i in enumerate(ids):
                if k not in done and srv.poll(i) >= 2:
                    done.add(k)
            now = time.perf_counter()
            if now - last >= 60 or len(done) == len(ids):
                last = now
                st = srv.stats()
                print(json.dumps({"progress": {"elapsed_s": round(now - t0, 1), "runs_done": len(done),
                                               "launches": st["launches"], "device_busy_s": round(st["busy_s"], 1),
                                               "trajectory_steps_of_finished_runs":
                                                   sum(reqs[k]["nt"] * steps for k in done)}}), flush=True)
            if limit and now - t0 > limit and len(done) < len(ids):
                break
            if len(done) < len(ids):
                time.sleep(2.0)
        wall = time.perf_counter() - t0
        ck = clocks.stop()
        st = srv.stats()
        if len(done) < len(ids):
            unfinished = [{"L": reqs[k]["L"], "chi": reqs[k]["chi"], "nt": reqs[k]["nt"], "model": reqs[k]["name"]}
                          for k in range(len(ids)) if k not in done]
            print(json.dumps({"metric": "TJM trajectory-steps/s, 64 uneven analog simulations served together",
                              "value": None, "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": 0,
                              "higher_is_better": True, "incomplete": True,
                              "time_limit_s": limit, "wall_s": wall, "runs_done": len(done),
                              "trajectory_steps_of_finished_runs": sum(reqs[k]["nt"] * steps for k in done),
                              "launches": st["launches"], "device_busy_s": st["busy_s"],
                              "unfinished_runs": unfinished, "clocks": ck,
                              "config": {"precision": prec, "tdvp": args.tdvp, "chunk": args.chunk}}), flush=True)
            return
        res = [srv.result(i) for i in ids]
    # error of every simulation against the FP64 form: its first 16
    # trajectories again in FP64 (same seed: the same Philox streams) over
    # the first err_steps steps, after the timed region
    per_sim = []
    err_steps = min(steps, args.err_steps)
    if prec == "mixed" and not args.no_plain:
        with api.Server(max_L=64, max_bond_dim=128, max_mpo_width=5, mixed=False, chunk=args.chunk,
                        ctx=ctx) as srv64:
            subs = []
            for r in reqs:
                psi, H, cfg, nm = r["problem"]
                c64 = api.TimeEvolutionConfig(cfg.observables, err_steps * cfg.dt, dt=cfg.dt,
                                              num_traj=min(16, r["nt"]), max_bond_dim=cfg.max_bond_dim,
                                              min_bond_dim=cfg.min_bond_dim,
                                              truncation_threshold=cfg.truncation_threshold,
                                              sample_timesteps=cfg.sample_timesteps, order=cfg.order)
                subs.append(srv64.submit(psi, H, c64, nm, seed=r["seed"], precision="fp64", tdvp=args.tdvp))
            ref = [srv64.result(i) for i in subs]
        for r, m, f in zip(reqs, res, ref):
            n, nc = f.trajectories.shape[0], f.trajectories.shape[2]
            per_sim.append(float(np.abs(m.trajectories[:n, :, :nc] - f.trajectories).max()))
    total = sum(r["nt"] * steps for r in reqs)
    line = {"metric": "TJM trajectory-steps/s, 64 uneven analog simulations served together", "value": total / wall,
            "unit": UNIT, "n_gpus": 1, "steps": steps, "warmup": 0, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64 contractions + c128 Lanczos/SVD/QR" if prec == "mixed" else "c128",
            "data": "synthetic",
            "config": {"workload": f"64 analog TJM simulations (seed 0x{BATCH_SEED:X}): Ising/XY/Heisenberg, "
                                   f"L in 8..64, chi_max in 16..128, 64..512 trajectories, lowering+dephasing, "
                                   f"dt=0.05, {steps} steps, {TDVP_DESC[args.tdvp]}; one server, chunk={args.chunk}",
                       "precision": prec, "tdvp": args.tdvp, "trajectory_steps": total},
            "wall_s": wall, "device_busy_s": st["busy_s"], "launches": st["launches"], "slots": st["slots"],
            "latency_p50_s": st["latency_p50_s"], "latency_p99_s": st["latency_p99_s"],
            "queue_p50_s": st["queue_p50_s"], "queue_p99_s": st["queue_p99_s"], "clocks": ck,
            "max_bond_reached": {f"chi{c}": int(max([r.max_bond.max() for q, r in zip(reqs, res) if q["chi"] == c],
                                                    default=0)) for c in (16, 32, 64, 128)},
            "jumps": int(sum(r.stats["jumps"] for r in res))}
    if prec == "mixed":
        line["autotune"] = autotune_summary(ctx)
    if per_sim:
        line["err_vs_fp64"] = {"z_max_abs_per_simulation": per_sim, "max": max(per_sim),
                               "median": float(np.median(per_sim)),
                               "simulations_above_1e-5": int(sum(e > 1e-5 for e in per_sim)),
                               "run": f"every <Z_i> at the first {err_steps + 1} recorded times of the first 16 "
                                      "trajectories of each simulation against the same trajectories (same seed) in "
                                      "the FP64 form"}
    print(json.dumps(line), flush=True)


def run_serve(args):
    """Poisson arrivals of QAOA ring requests at 0.8 x the measured capacity."""
    import torch
    torch.cuda.set_device(0)
    from yaqs_julia_b200 import _lib
    ctx = _lib.Context(0)
    rng = np.random.default_rng(SERVE_SEED)

    def work(r):  # trajectory-layers of a request
        return r["nt"] * api.digital_plan(r["problem"][1])[0]

    # mean work per request of the arrival distribution
    wrng = np.random.default_rng(SERVE_SEED + 1)
    mean_work = float(np.mean([work(ring_request(wrng)) for _ in range(400)]))
    with api.Server(max_L=48, max_bond_dim=64, max_mpo_width=1, mixed=False, chunk=args.chunk, ctx=ctx) as srv:
        # capacity: trajectory-layers/s of a calibration set submitted at once,
        # turned into requests/s with the distribution's mean work per request
        calib = [ring_request(rng) for _ in range(48)]
        t0 = time.perf_counter()
        ids = [srv.submit(*r["problem"], seed=SERVE_SEED + k) for k, r in enumerate(calib)]
        for i in ids:
            srv.result(i)
        cap_work = sum(work(r) for r in calib) / (time.perf_counter() - t0)
        cap = cap_work / mean_work
        lam = 0.8 * cap
        n_req = max(8, int(round(lam * args.duration)))
        reqs = [ring_request(rng) for _ in range(n_req)]
        gaps = rng.exponential(1.0 / lam, n_req)
        clocks = ClockSampler(0)
        base = srv.stats()
        clocks.start()
        t0 = time.perf_counter()
        ids = []
        t_next = t0
        for k, r in enumerate(reqs):
            t_next += gaps[k]
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            ids.append(srv.submit(*r["problem"], seed=SERVE_SEED + 100 + k))
        res = [srv.result(i) for i in ids]
        wall = time.perf_counter() - t0
        ck = clocks.stop()
        st = srv.stats()
    lat = np.array([r.times[2] for r in res])
    qd = np.array([r.times[0] for r in res])
    layers = sum(q["nt"] * q["p"] for q in reqs)
    line = {"metric": "served digital TJM requests: p50/p99 latency at 0.8 x capacity", "value": float(np.percentile(lat, 50)),
            "unit": "s (p50 latency)", "n_gpus": 1, "steps": n_req, "warmup": len(calib), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": f"QAOA ring requests (seed 0x{SERVE_SEED:X}): n in {{12,20,32,48}}, p in {{1,2,4}}, "
                                   "Pauli XYZ 0.005/3 per gate, chi_max=64, 128..1024 trajectories, Poisson arrivals "
                                   f"at 0.8 x measured capacity ({cap:.2f} req/s) for {args.duration:.0f} s",
                       "chunk": args.chunk},
            "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
            "queue_p50_s": float(np.percentile(qd, 50)), "queue_p99_s": float(np.percentile(qd, 99)),
            "capacity_req_s": cap, "capacity_traj_layers_s": cap_work, "mean_traj_layers_per_req": mean_work,
            "offered_req_s": lam, "completed": len(res), "wall_s": wall,
            "trajectory_layers_per_s": layers / wall, "device_busy_s": st["busy_s"] - base["busy_s"],
            "launches": st["launches"] - base["launches"], "clocks": ck}
    print(json.dumps(line), flush=True)


def autotune_summary(ctx):
    """The autotuner's measured product form per H_eff shape on this device
    (yaqs_autotune_results): tcgen05 or mma.sync, with both timings."""
    import ctypes as C
    n = C.c_int32(0)
    ctx.check(ctx._lib.yaqs_autotune_results(ctx.handle, None, 0, C.byref(n)))
    rows = np.zeros((max(n.value, 1), 8))
    ctx.check(ctx._lib.yaqs_autotune_results(ctx.handle, A.dptr(rows), n.value, C.byref(n)))
    shapes = [{"chi_l": int(r[0]), "D": int(r[1]), "chi_r": int(r[2]), "w": [int(r[3]), int(r[4])],
               "form": "mma.sync" if r[5] else "tcgen05", "us_tcgen05": round(float(r[6]), 1),
               "us_mma_sync": round(float(r[7]), 1)} for r in rows[:n.value]]
    return {"what": "mixed H_eff product form per shape, chosen by the engine's autotuner from timed launches "
                    "over every slot (tcgen05 128x64 tiles vs mma.sync 3xTF32 64x64 tiles)",
            "shapes": len(shapes), "mma_sync_chosen": sum(x["form"] == "mma.sync" for x in shapes),
            "table": shapes}


def measured_peaks():
    """Roofline denominators: the driver-measured peaks of this pool's B200s
    (MEASURED_PEAKS.json beside this file), else the stated fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]), "source": "measured"}
    except (OSError, ValueError, KeyError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def ensemble_gap_in_se(a, b):
    """max over (site, time) of |mean(a) - mean(b)| / SE(b), SE = std/sqrt(n),
    over the entries whose trajectories spread (SE > 1e-12); None if none do."""
    se = b.std(axis=0, ddof=1) / np.sqrt(b.shape[0]) if b.shape[0] > 1 else np.zeros(b.shape[1:])
    live = se > 1e-12
    if not live.any():
        return None
    return float((np.abs(a.mean(0) - b.mean(0))[live] / se[live]).max())


def timed_session(args, ctx, dist, local, problem, prec, rank, nt, n_steps):
    """One resident run: W untimed time indices, then n_steps timed ones in one
    launch (CUDA events on the launching stream, barrier + synchronize on both
    sides); returns device ms, the run's counters before/after, its results
    and the clock record."""
    psi, H, cfg, nm = problem
    desc = api.Descriptors(psi, H, cfg, nm, seed=SEED, traj_offset=rank * nt, precision=prec, tdvp_mode=TDVP[0])
    sess = api.Session(desc, ctx)
    for _ in range(args.warmup):
        sess.advance(1)
    st0 = sess.stats()
    clocks = ClockSampler(local)
    barrier_sync(dist)
    clocks.start()
    dev_ms = sess.advance(n_steps)
    barrier_sync(dist)
    ck = clocks.stop()
    st1 = sess.stats()
    phases = sess.profile() if args.profile else None
    res = sess.finish()
    return {"dev_ms": dev_ms, "st0": st0, "st1": st1, "res": res, "clocks": ck, "phases": phases}


def run_ours(args):
    ws, rank, local, dist = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from yaqs_julia_b200 import _lib
    ctx = _lib.Context(local)
    L, chi, nt = args.L, args.chi, args.traj
    K = args.steps
    mixed = args.precision == "mixed"
    problem = workload(L, chi, args.warmup + K + 1, nt, args.start)
    prec = A.YAQS_PREC_MIXED if mixed else A.YAQS_PREC_FP64
    main = timed_session(args, ctx, dist, local, problem, prec, rank, nt, K)
    t_max = reduce_max(dist, main["dev_ms"] / 1e3)
    value = reduce_sum(dist, nt * K) / t_max
    flops_timed = main["st1"]["flops"] - main["st0"]["flops"]
    matvecs_timed = main["st1"]["matvecs"] - main["st0"]["matvecs"]
    achieved = flops_timed / (main["dev_ms"] / 1e3) / 1e12
    import ctypes as C
    pk = C.c_double(0.0)
    ctx.check(ctx._lib.yaqs_fp64_peak(ctx.handle, C.byref(pk)))
    peaks = measured_peaks()
    # the plain ComplexF64 form on the same problem and draws, in the same
    # process: the metric's comparison and the reference of the error
    plain, err, ratio = None, None, None
    if mixed and not args.no_plain:
        Kp = min(K, args.plain_steps)
        pl = timed_session(args, ctx, dist, local, problem, A.YAQS_PREC_FP64, rank, nt, Kp)
        p_value = reduce_sum(dist, nt * Kp) / reduce_max(dist, pl["dev_ms"] / 1e3)
        ratio = value / p_value
        p_achieved = (pl["st1"]["flops"] - pl["st0"]["flops"]) / (pl["dev_ms"] / 1e3) / 1e12
        plain = {"what": "plain ComplexF64 GPU form (FP64 tensor-core products), same problem, same Philox draws, "
                         "same process", "value": p_value, "unit": UNIT, "steps": Kp,
                 "ms_per_step": pl["dev_ms"] / Kp, "clocks": pl["clocks"],
                 "roofline": {"bound": "tensor", "achieved": p_achieved, "peak": pk.value, "unit": "TFLOP/s",
                              "frac": p_achieved / pk.value if pk.value else None,
                              "peak_source": "measured FP64 DFMA probe (yaqs_fp64_peak) in this run"}}
        ncol = args.warmup + Kp + 1  # time indices both runs recorded
        a = main["res"].trajectories[:, :, :ncol]
        b = pl["res"].trajectories[:, :, :ncol]
        dz = np.abs(a[:, :L] - b[:, :L])
        ds = np.abs(a[:, L] - b[:, L])
        per_traj = dz.max(axis=(1, 2))
        err = {"z_max_abs": float(dz.max()), "z_mean_abs": float(dz.mean()), "s_half_max_abs": float(ds.max()),
               "s_half_mean_abs": float(ds.mean()),
               "z_traj_max_percentiles": {q: float(np.percentile(per_traj, q)) for q in (50, 90, 99)},
               "trajectories_above_1e-5": int((per_traj > 1e-5).sum()),
               "jumps": {"mixed": int(main["res"].stats["jumps"]), "plain": int(pl["res"].stats["jumps"])},
               "z_ensemble_mean_max_abs": float(np.abs(a[:, :L].mean(0) - b[:, :L].mean(0)).max()),
               # the ensemble means against the plain form's standard error of
               # the mean at every (site, time index) with a nonzero spread
               "z_ensemble_mean_max_in_se": ensemble_gap_in_se(a[:, :L], b[:, :L]),
               # largest per-trajectory <Z_i> difference at chosen time indices:
               # how the separation grows along the run
               "z_max_abs_by_time_index": {str(t): float(dz[:, :, t].max())
                                           for t in sorted({1, 2, 5, 10, 20, 50, ncol - 1}) if t < ncol},
               "trajectories_compared": nt, "time_indices_compared": ncol,
               "run": f"every <Z_i> and S_half at {ncol} recorded time indices ({START_DESC[args.start]}, {args.warmup} "
                      f"warm-up and {Kp} timed indices) of the two forms on the same Philox draws"}
    # end to end: the public C-ABI call on host buffers (marshalling, uploads,
    # allocation, a complete run of K time indices from t = 0 whose first
    # index costs one sweep, result download)
    e2e_problem = workload(L, chi, K + 1, nt, args.start)
    barrier_sync(dist)
    t0 = time.perf_counter()
    e2e_desc = api.Descriptors(*e2e_problem, seed=SEED, traj_offset=rank * nt, precision=prec, tdvp_mode=TDVP[0])
    api.run_descriptors(e2e_desc, ctx)
    barrier_sync(dist)
    e2e_s = reduce_max(dist, time.perf_counter() - t0)
    h2d, d2h = desc_bytes(e2e_desc, e2e_desc.n_obs, e2e_desc.n_out, nt, L)
    e2e_value = reduce_sum(dist, nt * K) / e2e_s
    cpu = None
    if rank == 0 and not args.no_cpu and ws == 1:
        v, cores, sample, blas = cpu_sample(L, chi, args.start)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "blas": blas, "sample": sample}
    if rank == 0:
        traffic_per = TRAFFIC_PER_TRAJ_STEP.get((args.precision, args.tdvp, L, chi))
        if mixed:
            tc_peak = peaks["bf16_tflops"] / 2
            roof = {"bound": "tensor", "achieved": achieved, "peak": tc_peak, "unit": "TFLOP/s",
                    "frac": achieved / tc_peak,
                    "peak_source": f"half the {peaks['source']} dense bf16 rate (MEASURED_PEAKS.json): the rate of "
                                   "the tcgen05 kind::tf32 MMAs the mixed products issue",
                    "achieved_counts": "H_eff product flops only, 8 per complex MAC (the tensor pipe executes 9 "
                                       "TF32 MMAs per 4 real MACs: 3-product complex form x 3xTF32 split)"}
        else:
            roof = {"bound": "tensor", "achieved": achieved, "peak": pk.value, "unit": "TFLOP/s",
                    "frac": achieved / pk.value if pk.value else None,
                    "peak_source": "measured FP64 DFMA probe (yaqs_fp64_peak) in this run; MEASURED_PEAKS.json "
                                   "has no FP64 entry",
                    "achieved_counts": "H_eff product flops only (8 flops per complex MAC)"}
        tt = traffic_per * nt * K if traffic_per else None
        roof.update({"kernel": "tjm_step_kernel_tc" if mixed else "tjm_step_kernel", "traffic": tt,
                     "traffic_source": "DRAM read+write bytes per trajectory-step from a one-launch ncu capture of "
                                       "148 trajectories of the same configuration (profiles/tjm_step_kernels_L30_"
                                       "chi64_148traj_traffic.md), scaled by the trajectory-steps of the timed launch "
                                       "(a lower bound: the full run keeps twice the slots in L2); null when not "
                                       "captured",
                     "traffic_gbs": tt / (main["dev_ms"] / 1e3) / 1e9 if tt else None,
                     "hbm_frac": tt / (main["dev_ms"] / 1e3) / 1e9 / peaks["hbm_gbs"] if tt else None})
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K,
                "warmup": args.warmup, "ms_per_step": main["dev_ms"] / K, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": ratio,
                "vs_baseline_note": "value / the plain ComplexF64 GPU form's value measured in the same run (the "
                                    "metric's own comparison; the reference publishes no throughput)"
                if ratio is not None else None,
                "dtype": "c64 contractions (tcgen05 3xTF32) + c128 Lanczos/SVD/QR/norms" if mixed else "c128",
                "data": "synthetic",
                "config": analog_config(args, L, chi, nt, ws),
                "gpu_launches": 1,  # one trajectory-kernel launch covers the K time indices
                "roofline": roof,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / K,
                        "d2h_bytes_per_step": d2h / K, "seconds": e2e_s, "steps": K,
                        "precision": args.precision},
                "cpu_baseline": cpu, "clocks": main["clocks"],
                "stats": {"matvecs_timed": matvecs_timed, "flops_timed": flops_timed,
                          "jumps": main["res"].stats["jumps"], "svd_sweeps": main["res"].stats["svd_sweeps"],
                          "svds": main["res"].stats["svds"], "max_bond": int(main["res"].max_bond.max())}}
        if mixed:
            line["autotune"] = autotune_summary(ctx)
        if plain is not None:
            line["plain_fp64"] = plain
        if err is not None:
            line["err_vs_fp64"] = err
        if main["phases"]:
            tot = main["phases"]["step"] or 1.0
            line["phases_pct_of_step"] = {k: round(100 * v / tot, 2) for k, v in main["phases"].items()}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--workload", default="analog", choices=["analog", "digital", "batch", "serve"])
    ap.add_argument("--tdvp", default="dynamic", choices=list(TDVP_NAMES),
                    help="analog sweep: dynamic (1-site TDVP with 2-site growth up to chi, the configuration's "
                         "mode), 2site (the Julia reference's two_site_tdvp!) or 1site")
    ap.add_argument("--chunk", type=int, default=2, help="batch/serve: positions each run advances per launch")
    ap.add_argument("--duration", type=float, default=60.0, help="serve: seconds of Poisson arrivals")
    ap.add_argument("--time-limit", type=float, default=0.0,
                    help="batch: stop waiting after this many seconds and report what finished (0: no limit)")
    ap.add_argument("--err-steps", type=int, default=10,
                    help="batch: steps over which every simulation is compared with its FP64 form")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"],
                    help="analog contraction precision: mixed (complex FP32 on the tensor cores, the metric's "
                         "subject; the plain FP64 form is timed beside it) or fp64 alone")
    ap.add_argument("--plain-steps", type=int, default=8,
                    help="mixed runs: timed time indices of the plain FP64 form measured beside it")
    ap.add_argument("--no-plain", action="store_true", help="mixed runs: skip the plain FP64 comparison")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--traj", type=int, default=None)
    ap.add_argument("--chi", type=int, default=64)
    ap.add_argument("--L", type=int, default=30)
    ap.add_argument("--start", default="sat", choices=["sat", "neel"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="enable the engine's per-phase device timers and report them (not for timing runs)")
    args = ap.parse_args()
    TDVP[0] = TDVP_NAMES[args.tdvp]
    args.steps_given = args.steps is not None
    if args.steps is None:
        args.steps = 2
    if args.traj is None and args.workload == "analog":
        args.traj = 1024
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.profile:
        os.environ["YAQS_PROFILE"] = "1"
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "digital":
        run_digital(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
