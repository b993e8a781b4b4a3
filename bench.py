#!/usr/bin/env python
"""Benchmark: TJM trajectory-steps/s of the analog engine.

Workload (default): the L=30 Heisenberg chain H = sum(XX+YY+ZZ) + 0.3 sum Z
(init_general_hamiltonian(30,1,1,1,0,0,0.3)), dephasing (pauli_z, gamma=0.05)
on every site, dt=0.05, 2-site TDVP, max bond dimension 64, threshold 1e-9,
second-order TJM with sampling at every time index, <Z_i> on all 30 sites
plus the half-chain entropy, 1024 trajectories per GPU, Philox draws.  The
start state is an MPS with every bulk bond already at 64 (Gaussian
entries, normalised by the engine) so every timed step runs at chi=64; with
--start neel the run starts from the Neel state instead.

A step is one recorded time index of every trajectory (two TDVP sweeps,
dissipation, jump, measurement).  W untimed steps, then K timed steps,
bracketed by a barrier and a device synchronisation; device time from CUDA
events on the launching stream; the trajectory states (3.6 GB) are larger
than L2.  Multi-GPU runs are independent replicas (one process per GPU,
launched by torchrun); the value is the sum of every rank's trajectory-steps
over the slowest rank's time.

--impl reference times the CPU restatement of the reference algorithm
(the reference itself is Julia, not runnable here) on all host cores, on
bounded samples of the same workload.
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

METRIC = "TJM trajectory-steps/s (L=30 Heisenberg, chi=64, 1024 trajectories)"
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
    """Oracle (CPU restatement, test infrastructure) on all host cores:
    3 recorded time indices (1.5 sweeps per trajectory-step) for one
    trajectory per core.  Returns (trajectory-steps/s, cores, sample text)."""
    from oracle import oracle as O
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    psi, H, cfg, nm = workload(L, chi, 3, cores, start)
    d = api.Descriptors(psi, H, cfg, nm, seed=SEED)
    t0 = time.perf_counter()
    O.analog_run(d, nthreads=cores)
    dt = time.perf_counter() - t0
    steps = cores * 2
    return steps / dt, cores, f"{cores} trajectories x 2 time indices (t=0..0.1) of the same workload, {dt:.1f} s"


def run_reference(args):
    ws, rank, local, dist = dist_setup()
    if rank != 0:
        return
    vals = []
    for k in range(args.warmup + args.steps):
        v, cores, sample = cpu_sample(args.L, args.chi, args.start)
        if k >= args.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": f"L={args.L} Heisenberg h=0.3, chi={args.chi}, dephasing 0.05, dt=0.05, "
                                   f"start={args.start}", "L": args.L, "chi": args.chi},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Julia (Yaqs.jl) cannot run here; CPU restatement (oracle/tjm_oracle.cpp)"}
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


def run_ours(args):
    ws, rank, local, dist = dist_setup()
    import torch
    torch.cuda.set_device(local)
    from yaqs_julia_b200 import _lib
    ctx = _lib.Context(local)
    L, chi, nt = args.L, args.chi, args.traj
    n_times = args.warmup + args.steps + 1
    psi, H, cfg, nm = workload(L, chi, n_times, nt, args.start)
    desc = api.Descriptors(psi, H, cfg, nm, seed=SEED, traj_offset=rank * nt)
    sess = api.Session(desc, ctx)
    for _ in range(args.warmup):
        sess.advance(1)
    st0 = sess.stats()
    clocks = ClockSampler(local)
    barrier_sync(dist)
    clocks.start()
    dev_ms = sess.advance(args.steps)
    barrier_sync(dist)
    ck = clocks.stop()
    st1 = sess.stats()
    phases = sess.profile() if args.profile else None
    res = sess.finish()
    t_max = reduce_max(dist, dev_ms / 1e3)
    steps_all = reduce_sum(dist, nt * args.steps)
    value = steps_all / t_max
    flops_timed = st1["flops"] - st0["flops"]
    matvecs_timed = st1["matvecs"] - st0["matvecs"]
    import ctypes as C
    pk = C.c_double(0.0)
    ctx.check(ctx._lib.yaqs_fp64_peak(ctx.handle, C.byref(pk)))
    achieved = flops_timed / (dev_ms / 1e3) / 1e12
    # end to end: the public C-ABI call on host buffers, K time indices
    e2e_cfg_psi, e2e_H, e2e_cfg, e2e_nm = workload(L, chi, args.steps + 1, nt, args.start)
    barrier_sync(dist)
    t0 = time.perf_counter()
    e2e_desc = api.Descriptors(e2e_cfg_psi, e2e_H, e2e_cfg, e2e_nm, seed=SEED, traj_offset=rank * nt)
    e2e_res = api.run_descriptors(e2e_desc, ctx)
    barrier_sync(dist)
    e2e_s = reduce_max(dist, time.perf_counter() - t0)
    h2d, d2h = desc_bytes(e2e_desc, e2e_desc.n_obs, e2e_desc.n_out, nt, L)
    e2e_value = reduce_sum(dist, nt * args.steps) / e2e_s
    cpu = None
    if rank == 0 and not args.no_cpu and ws == 1:
        v, cores, sample = cpu_sample(L, chi, args.start)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
                "config": {"workload": f"analog TJM, L={L} Heisenberg XXX h=0.3, dephasing gamma=0.05, dt=0.05, "
                                       f"2-site TDVP chi_max={chi}, thr=1e-9, {nt} trajectories per GPU, "
                                       f"start={'saturated chi MPS' if args.start == 'sat' else 'Neel'}",
                           "L": L, "chi": chi, "num_traj": nt, "dt": 0.05, "parallelism": f"replicas x{ws}",
                           "l2": "inputs larger than L2: %d trajectory states of up to %.1f MB each" % (
                               nt, sum(min(2 ** min(b, L - b), chi) * 2 * min(2 ** min(b + 1, L - b - 1), chi)
                                       for b in range(L)) * 16 / 1e6)},
                "gpu_launches": args.steps,
                "roofline": {"bound": "fp64", "achieved": achieved, "peak": pk.value, "unit": "TFLOP/s",
                             "frac": achieved / pk.value if pk.value else None, "traffic": None,
                             "kernel": "tjm_step_kernel",
                             "peak_source": "measured FP64 DFMA probe (yaqs_fp64_peak) in this run; "
                                            "MEASURED_PEAKS.json has no FP64 entry",
                             "achieved_counts": "H_eff product flops only (8 flops per complex MAC)"},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
                        "d2h_bytes_per_step": d2h / args.steps, "seconds": e2e_s},
                "cpu_baseline": cpu, "clocks": ck,
                "stats": {"matvecs_timed": matvecs_timed, "flops_timed": flops_timed,
                          "jumps": res.stats["jumps"], "svd_sweeps": res.stats["svd_sweeps"],
                          "svds": res.stats["svds"], "max_bond": int(res.max_bond.max())}}
        if phases:
            tot = phases["step"] or 1.0
            line["phases_pct_of_step"] = {k: round(100 * v / tot, 2) for k, v in phases.items()}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--traj", type=int, default=1024)
    ap.add_argument("--chi", type=int, default=64)
    ap.add_argument("--L", type=int, default=30)
    ap.add_argument("--start", default="sat", choices=["sat", "neel"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="enable the engine's per-phase device timers and report them (not for timing runs)")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.profile:
        os.environ["YAQS_PROFILE"] = "1"
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
