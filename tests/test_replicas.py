"""The multi-GPU form is replicas: each rank runs its own block of
trajectories (global index = rank * n + local index, which keys the Philox
streams) and only the timing is reduced.  Two gloo ranks on the CPU check
that the blocks reproduce one run of all trajectories, analog and digital,
and that the bench's max/sum reductions combine the ranks as the bench line
reports them."""
import os
import socket

import numpy as np


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _problem(nt, offset):
    from yaqs_julia_b200 import api
    L = 4
    H = api.init_ising(L, 1.0, 0.7)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 0.3, dt=0.1, num_traj=nt, max_bond_dim=8)
    nm = api.NoiseModel([{"name": "lowering", "sites": [i], "strength": 0.3} for i in range(1, L + 1)], L)
    return api.Descriptors(api.MPS(L, state="ones"), H, cfg, nm, seed=1234, traj_offset=offset)


def _rank(rank, world, port, nt, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    from oracle import oracle as O
    ws, r, _, dist = bench.dist_setup()
    assert (ws, r) == (world, rank)
    traj, _, st = O.analog_run(_problem(nt, rank * nt))
    np.save(os.path.join(out_dir, f"traj{rank}.npy"), traj)
    t_max = bench.reduce_max(dist, 1.0 + rank)      # per-rank device seconds
    units = bench.reduce_sum(dist, nt * 3)          # trajectory-steps of this rank
    np.save(os.path.join(out_dir, f"red{rank}.npy"), np.array([t_max, units, st["jumps"]]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_reproduce_one_run(oracle, tmp_path):
    import torch.multiprocessing as mp
    nt, world = 6, 2
    port = _free_port()
    mp.start_processes(_rank, args=(world, port, nt, str(tmp_path)), nprocs=world, start_method="spawn", join=True)
    parts = [np.load(tmp_path / f"traj{r}.npy") for r in range(world)]
    whole, _, st = oracle.analog_run(_problem(world * nt, 0))
    assert np.array_equal(np.concatenate(parts, axis=0), whole)
    for r in range(world):
        t_max, units, _ = np.load(tmp_path / f"red{r}.npy")
        assert t_max == 2.0 and units == world * nt * 3
    jumps = sum(int(np.load(tmp_path / f"red{r}.npy")[2]) for r in range(world))
    assert jumps == st["jumps"] > 0


def _circuit_problem(nt, offset):
    from yaqs_julia_b200 import api
    from yaqs_julia_b200 import circuits as CL
    L = 5
    c = CL.create_ising_circuit(L, 1.0, 0.7, 0.1, 3)
    nm = api.NoiseModel([{"name": n, "sites": [i], "strength": 0.05} for i in range(1, L + 1)
                         for n in ("pauli_x", "pauli_z")], L)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 3.0, dt=1.0, num_traj=nt, max_bond_dim=8)
    return api.CircuitDescriptors(api.MPS(L), c, cfg, nm, seed=77, traj_offset=offset)


def _digital_rank(rank, world, port, nt, out_dir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench
    from oracle import oracle as O
    _, _, _, dist = bench.dist_setup()
    traj, _, _ = O.digital_run(_circuit_problem(nt, rank * nt))
    np.save(os.path.join(out_dir, f"dig{rank}.npy"), traj)
    dist.barrier()
    dist.destroy_process_group()


def test_two_digital_replicas_reproduce_one_run(oracle, tmp_path):
    """The digital workload shards the same way: each rank's block of
    trajectories (Philox streams keyed by the global index) concatenates to
    one run of all of them."""
    import torch.multiprocessing as mp
    nt, world = 5, 2
    mp.start_processes(_digital_rank, args=(world, _free_port(), nt, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    parts = [np.load(tmp_path / f"dig{r}.npy") for r in range(world)]
    whole, _, st = oracle.digital_run(_circuit_problem(world * nt, 0))
    assert np.array_equal(np.concatenate(parts, axis=0), whole) and st["jumps"] > 0


def test_bench_ensemble_gap_in_standard_errors():
    """The mixed line's ensemble check: |mean(a) - mean(b)| / SE(b) over the
    (site, time) entries whose trajectories spread; None when none spread."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    rng = np.random.default_rng(5)
    b = rng.normal(size=(400, 3, 4))
    se = b.std(axis=0, ddof=1) / np.sqrt(400)
    a = b + 2.0 * se.max()
    assert abs(bench.ensemble_gap_in_se(a, b) - 2.0 * se.max() / se.min()) < 1e-9
    assert bench.ensemble_gap_in_se(b, b) == 0.0
    flat = np.ones((50, 2, 3))
    assert bench.ensemble_gap_in_se(flat + 1.0, flat) is None
