"""Serving (yaqs_server_*): many simulations of different kinds and sizes in
one persistent launch per step, admitted as memory frees up.  Each result
must equal the result of the same request run alone (bitwise: a
trajectory's arithmetic does not depend on its slot or batch)."""
import threading
import time

import numpy as np
import pytest

from yaqs_julia_b200 import _abi as A
from yaqs_julia_b200 import api

pytestmark = pytest.mark.gpu


def _ising(L, g, T, nt, chi, seed_state="zeros"):
    H = api.init_ising(L, 1.0, g)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, T, dt=0.05, num_traj=nt, max_bond_dim=chi)
    nm = api.NoiseModel([{"name": "lowering", "sites": [i], "strength": 0.05} for i in range(1, L + 1)] +
                        [{"name": "pauli_z", "sites": [i], "strength": 0.05} for i in range(1, L + 1)], L)
    return api.MPS(L, state=seed_state), H, cfg, nm


def _heis(L, h, T, nt, chi):
    H = api.init_general_hamiltonian(L, 1, 1, 1, 0, 0, h)
    obs = ([api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)] +
           [api.Observable("S", None, L // 2, kind="entropy")])
    cfg = api.TimeEvolutionConfig(obs, T, dt=0.05, num_traj=nt, max_bond_dim=chi)
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [i], "strength": 0.1} for i in range(1, L + 1)], L)
    return api.MPS(L, state="Neel"), H, cfg, nm


def _ring(n, p, nt, seed):
    rng = np.random.default_rng(seed)
    c = api.DigitalCircuit(n)
    c.add_gate(api.Barrier(), [])
    for _ in range(p):
        g, b = rng.uniform(0, np.pi, 2)
        for i in range(1, n):
            c.add_gate(api.Rzz(g), [i, i + 1])
        c.add_gate(api.Rzz(g), [n, 1])
        for i in range(1, n + 1):
            c.add_gate(api.Rx(b), [i])
        c.add_gate(api.Barrier(), [])
    nm = api.NoiseModel([{"name": nme, "sites": [i], "strength": 0.005 / 3} for i in range(1, n + 1)
                         for nme in ("pauli_x", "pauli_y", "pauli_z")], n)
    obs = [api.Observable(f"ZZ{i}", np.kron(api.Z, api.Z), [i, i + 1]) for i in range(1, n)]
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=1.0, num_traj=nt, max_bond_dim=32)
    return api.MPS(n), c, cfg, nm


def _alone(problem, seed, precision="fp64"):
    """The request run alone: FP64 requests as a direct run (the server's
    FP64 arithmetic is the direct run's), mixed ones alone in a server of the
    same shape (direct mixed runs take the tcgen05 products, served runs the
    mma.sync form)."""
    psi, op, cfg, nm = problem
    if isinstance(op, api.DigitalCircuit):
        return api.run_circuit_descriptors(api.CircuitDescriptors(psi, op, cfg, nm, seed=seed))
    if precision == "mixed":
        with api.Server(max_L=16, max_bond_dim=32, max_mpo_width=5, chunk=2) as srv:
            return srv.result(srv.submit(psi, op, cfg, nm, seed=seed, precision=precision), timeout=300)
    return api.run_descriptors(api.Descriptors(psi, op, cfg, nm, seed=seed, precision=A.YAQS_PREC_FP64))


def test_results_alone_equal_results_in_the_mix():
    problems = [(_ising(6, 0.5, 0.5, 40, 16), 11, "fp64"), (_heis(10, 0.3, 0.3, 24, 16), 12, "fp64"),
                (_ring(8, 2, 30, 5), 13, "fp64"), (_heis(8, 0.7, 0.25, 16, 8), 14, "mixed"),
                (_ising(12, 1.2, 0.3, 20, 32, "x+"), 15, "fp64")]
    alone = [_alone(p, s, pr) for p, s, pr in problems]
    with api.Server(max_L=16, max_bond_dim=32, max_mpo_width=5, chunk=2) as srv:
        ids = [srv.submit(*p, seed=s, precision=pr) for p, s, pr in problems]
        mixed = [srv.result(i, timeout=300) for i in ids]
        st = srv.stats()
    for a, m in zip(alone, mixed):
        assert np.array_equal(a.trajectories, m.trajectories)
        assert np.array_equal(a.max_bond, m.max_bond)
        assert a.stats["jumps"] == m.stats["jumps"]
    assert st["completed"] == len(problems) and st["failed"] == 0
    assert st["launches"] >= 1 and st["latency_p99_s"] >= st["latency_p50_s"] > 0


def test_admission_by_memory_budget_queues_requests():
    """With a budget that holds one request at a time, the rest wait in order and all finish."""
    probs = [(_ising(6, 0.4 + 0.1 * k, 0.3, 30, 16), 20 + k) for k in range(4)]
    alone = [_alone(p, s) for p, s in probs]
    with api.Server(max_L=8, max_bond_dim=16, max_mpo_width=3, chunk=1, hbm_budget=1) as srv:
        ids = [srv.submit(*p, seed=s) for p, s in probs]
        res = [srv.result(i, timeout=300) for i in ids]
        st = srv.stats()
    for a, r in zip(alone, res):
        assert np.array_equal(a.trajectories, r.trajectories)
    # FIFO admission: each later request waited for the earlier ones
    queued = [r.times[0] for r in res]
    assert queued == sorted(queued) and queued[-1] > 0
    assert st["completed"] == 4 and st["bytes_in_use"] == 0


def test_requests_join_while_others_run():
    long = _heis(12, 0.2, 3.0, 32, 16)
    short = _ising(6, 0.8, 0.2, 16, 8)
    with api.Server(max_L=12, max_bond_dim=16, max_mpo_width=5, chunk=1) as srv:
        a = srv.submit(*long, seed=1)
        t0 = time.time()
        while srv.poll(a) != A.YAQS_REQ_RUNNING and time.time() - t0 < 60:
            time.sleep(0.005)
        b = srv.submit(*short, seed=2)
        rb = srv.result(b, timeout=300)
        state_a = srv.poll(a)
        ra = srv.result(a, timeout=300)
    assert state_a == A.YAQS_REQ_RUNNING  # the short request finished inside the long one's run
    assert np.array_equal(rb.trajectories, _alone(short, 2).trajectories)
    assert np.array_equal(ra.trajectories, _alone(long, 1).trajectories)


def test_submit_from_many_threads():
    probs = [(_ising(6, 0.3 + 0.05 * k, 0.2, 12, 8), 40 + k) for k in range(8)]
    out = {}
    with api.Server(max_L=8, max_bond_dim=8, max_mpo_width=3, chunk=2) as srv:
        def worker(k):
            p, s = probs[k]
            rid = srv.submit(*p, seed=s)
            out[k] = srv.result(rid, timeout=300)
        th = [threading.Thread(target=worker, args=(k,)) for k in range(8)]
        for t in th:
            t.start()
        for t in th:
            t.join()
    for k, (p, s) in enumerate(probs):
        assert np.array_equal(out[k].trajectories, _alone(p, s).trajectories)


def test_failed_request_leaves_the_others_intact():
    ok = _ising(6, 0.5, 0.2, 8, 8)
    too_big = _ising(8, 0.5, 0.2, 8, 64)  # bond capacity 16 > the server's slot shape (8)
    with api.Server(max_L=8, max_bond_dim=8, max_mpo_width=3) as srv:
        a = srv.submit(*ok, seed=3)
        b = srv.submit(*too_big, seed=4)
        ra = srv.result(a, timeout=300)
        from yaqs_julia_b200._lib import EngineError
        with pytest.raises(EngineError, match="UNSUPPORTED"):
            srv.result(b, timeout=300)
        st = srv.stats()
    assert np.array_equal(ra.trajectories, _alone(ok, 3).trajectories)
    assert st["failed"] == 1 and st["completed"] == 1


def test_long_range_noise_is_refused_by_the_server():
    psi, H, cfg, _ = _ising(6, 0.5, 0.2, 8, 8)
    nm = api.NoiseModel([{"name": "crosstalk_zz", "sites": [1, 4], "strength": 0.1}], 6)
    from yaqs_julia_b200._lib import EngineError
    with api.Server(max_L=8, max_bond_dim=8, max_mpo_width=3) as srv:
        with pytest.raises(EngineError, match="UNSUPPORTED"):
            srv.submit(psi, H, cfg, nm, seed=1)
