"""Host MPS/MPO algebra, shots and measurement configs (src/MPS.jl,
src/MPO.jl:271-556, src/SimulationConfigs.jl:95-208) against dense
linear algebra; RepeatedDigitalCircuit (DigitalTJM.jl:452-536) against the
explicitly repeated circuit."""
import math

import numpy as np
import pytest

from yaqs_julia_b200 import api
from yaqs_julia_b200 import tensornet as T
from oracle import dense as D


def _rand_mps(L, chi, seed):
    m = api.random_mps(L, chi, seed=seed)
    return T.normalize(m)


def test_gauge_moves_keep_the_state_and_normalise():
    m = _rand_mps(6, 4, 1)
    v = m.to_vec()
    assert abs(np.linalg.norm(v) - 1) < 1e-12 and m.orth_center == 1
    for c in (4, 6, 2, 1):
        T.shift_orthogonality_center(m, c)
        assert np.allclose(m.to_vec(), v, atol=1e-12)
        assert abs(T.mps_norm(m) - 1) < 1e-12
    assert T.check_if_valid_mps(m) and T.write_max_bond_dim(m) == 4


def test_overlaps_and_expectations_match_dense():
    a, b = _rand_mps(5, 3, 2), _rand_mps(5, 4, 3)
    va, vb = a.to_vec(), b.to_vec()
    # the reference's convention: sum a * conj(b) = <b|a> (MPS.jl:528-585)
    assert abs(T.scalar_product(a, b) - np.vdot(vb, va)) < 1e-12
    assert abs(T.scalar_product(a, b) - np.conj(T.scalar_product(b, a))) < 1e-12
    for s in range(1, 6):
        assert abs(T.local_expect(a, api.X, s) - np.vdot(va, D.site_op(api.X, s, 5) @ va)) < 1e-12
    op = np.kron(api.Z, api.Y)
    for s in range(1, 5):
        ref = np.vdot(va, D.gate_op(op, [s, s + 1], 5) @ va)
        assert abs(T.local_expect_two_site(a, op, s, s + 1) - ref) < 1e-12
    ops = [api.Z, api.X, api.Y, api.Z, api.X]
    ev = T.evaluate_all_local_expectations(a, ops)
    assert np.allclose(ev, [np.vdot(va, D.site_op(o, i + 1, 5) @ va) for i, o in enumerate(ops)], atol=1e-12)


def test_truncate_keeps_at_least_two_and_caps_the_bond():
    m = _rand_mps(8, 8, 4)
    v = m.to_vec()
    err = T.truncate(m, threshold=1e-3, max_bond_dim=3)
    assert T.write_max_bond_dim(m) <= 3 and min(t.shape[2] for t in m.tensors[:-1]) >= 2
    assert abs(np.linalg.norm(m.to_vec()) - 1) < 1e-12 and err > 0
    assert abs(np.vdot(m.to_vec(), v)) > 0.5
    exact = _rand_mps(6, 2, 5)
    v2 = exact.to_vec()
    assert T.truncate(exact, threshold=1e-12) < 1e-20 and np.allclose(exact.to_vec(), v2, atol=1e-10)


def _literal_shot(mps, u):
    """single_shot_measure restated one site at a time with explicit tensors."""
    import copy
    psi = T.shift_orthogonality_center(copy.deepcopy(mps), 1)
    bits = 0
    for i in range(psi.length):
        A = psi.tensors[i]
        probs = [float(np.sum(np.abs(A[:, p, :]) ** 2)) for p in range(2)]
        acc, chosen = 0.0, 1
        for k in range(2):
            acc += probs[k]
            if u[i] <= acc:
                chosen = k
                break
        bits += chosen << i
        if i < psi.length - 1:
            Ap = A[:, chosen, :] / max(math.sqrt(probs[chosen]), 1e-300)
            N = psi.tensors[i + 1]
            psi.tensors[i + 1] = np.einsum("lr,rpq->lpq", Ap, N)
    return bits


def test_shots_follow_the_born_rule():
    m = _rand_mps(4, 3, 6)
    v = m.to_vec()
    u = np.random.default_rng(7).random((40, 4))
    counts = T.measure_shots(m, 40, uniforms=u)
    lit = [_literal_shot(m, u[s]) for s in range(40)]
    want = {}
    for b in lit:
        want[b] = want.get(b, 0) + 1
    assert counts == want
    n = 40000
    counts = T.measure_shots(m, n, rng=np.random.default_rng(8))
    p = np.abs(v) ** 2
    for b in range(16):
        assert abs(counts.get(b, 0) / n - p[b]) < 5 * math.sqrt(p[b] * (1 - p[b]) / n) + 1e-9
    bs = "".join(str((3 >> i) & 1) for i in range(4))
    assert abs(T.project_onto_bitstring(m, bs) - p[3]) < 1e-12
    assert T.single_shot_measure(api.MPS(3, state="basis", basis_string="101")) == 0b101


def test_mpo_algebra_matches_dense():
    L = 4
    H1 = api.init_ising(L, 1.0, 0.4)
    H2 = api.init_general_hamiltonian(L, 0.3, 0.2, 0.5, 0.1, 0.0, 0.2)
    M1, M2 = H1.to_matrix(), H2.to_matrix()
    assert np.allclose(T.mpo_add(H1, H2).to_matrix(), M1 + M2, atol=1e-12)
    assert np.allclose(T.mpo_scale(2.5j, H1).to_matrix(), 2.5j * M1, atol=1e-12)
    assert np.allclose(T.contract_mpo_mpo(H1, H2).to_matrix(), M1 @ M2, atol=1e-12)
    assert np.allclose(T.mpo_identity(L).to_matrix(), np.eye(2 ** L))
    assert np.allclose(T.mpo_zero(L).to_matrix(), 0)
    psi = _rand_mps(L, 3, 9)
    v = psi.to_vec()
    assert np.allclose(T.contract_mpo_mps(H1, psi).to_vec(), M1 @ v, atol=1e-12)
    assert abs(T.expect_mpo(H2, psi) - np.vdot(v, M2 @ v)) < 1e-12
    # a doubled Hamiltonian compresses back to its own width
    S = T.mpo_add(H1, H1)
    assert max(S.bond_dims) == 6
    err = T.mpo_truncate(S, threshold=1e-12)
    assert err < 1e-20 and max(S.bond_dims) <= 3 and np.allclose(S.to_matrix(), 2 * M1, atol=1e-10)
    O = T.orthogonalize(api.init_ising(L, 0.7, 1.1), 2)
    assert np.allclose(O.to_matrix(), api.init_ising(L, 0.7, 1.1).to_matrix(), atol=1e-12)


def test_measurement_configs():
    mc = T.MeasurementConfig(3)
    mc.measurements[0] = {1: 2, 3: 1}
    mc.measurements[2] = {1: 1}
    assert T.aggregate_measurements(mc) == {1: 3, 3: 1} and mc.results == {1: 3, 3: 1}
    obs = [api.Observable("Z1", api.Z, 1)]
    sc = T.StrongMeasurementConfig(obs, num_traj=2)
    obs[0].trajectories = np.array([[1.0, 0.5], [0.0, 0.5]], dtype=np.complex128)
    T.aggregate_strong(sc)
    assert np.allclose(obs[0].results, [0.5, 0.5])


def _step(L, seed, lead_barrier=True, tail_barrier=True):
    rng = np.random.default_rng(seed)
    c = api.DigitalCircuit(L)
    if lead_barrier:
        c.add_gate(api.Barrier(), [])
    for i in range(1, L + 1):
        c.add_gate(api.Rx(rng.uniform(0, 1)), [i])
    for i in list(range(1, L, 2)) + list(range(2, L, 2)):
        c.add_gate(api.Rzz(rng.uniform(0, 1)), [i, i + 1])
    if tail_barrier:
        c.add_gate(api.Barrier(), [])
    return c


@pytest.mark.parametrize("lead,tail", [(True, True), (False, True), (True, False)])
def test_repeated_circuit_sample_plan(oracle, lead, tail):
    L, R = 5, 3
    step = _step(L, 3, lead, tail)
    rep = api.RepeatedDigitalCircuit(step, R)
    layers_step, _ = api.process_circuit(step)
    start, after, n = api.sample_plan(rep)
    s_start, s_after, _ = api.sample_plan(step)
    assert start == s_start and len(api.process_circuit(rep)[0]) == R * len(layers_step)
    assert n == max(1, (1 if s_start else 0) + R * len(s_after))
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=1.0, num_traj=1, max_bond_dim=32, truncation_threshold=1e-14)
    tr, _, _ = oracle.digital_run(api.CircuitDescriptors(api.MPS(L, state="wall"), rep, cfg, None))
    U = np.eye(2 ** L, dtype=np.complex128)
    for g in step.gates:
        if not isinstance(g.op, api.Barrier):
            U = D.gate_op(g.op, g.sites, L) @ U
    psi = D.product_state([[1, 0]] * (L // 2) + [[0, 1]] * (L - L // 2))
    zs = lambda v: [np.real(np.vdot(v, D.site_op(api.Z, i, L) @ v)) for i in range(1, L + 1)]  # noqa: E731
    cols = [zs(psi)] if lead else []
    for _ in range(R):
        psi = U @ psi
        if tail:
            cols.append(zs(psi))
    if not cols:
        cols = [zs(psi)]
    assert tr.shape[2] == n == len(cols)
    assert np.abs(tr[0] - np.array(cols).T).max() < 1e-9 and np.abs(np.array(cols)).max() > 0.1


def test_simulation_config_known_answers():
    """test_SimulationConfigs.jl:28-114: times, defaults, buffer shapes of
    initialize!, expect on |++++>, and the trajectory mean."""
    c = api.TimeEvolutionConfig([api.Observable("X", api.X, 1)], 1.0, dt=0.2, sample_timesteps=True, num_traj=50)
    assert np.allclose(c.times, np.arange(0.0, 1.0 + 1e-12, 0.2), atol=1e-10) and c.num_traj == 50
    d = api.TimeEvolutionConfig([], 2.0)
    assert (d.dt, d.sample_timesteps, d.num_traj, d.max_bond_dim, d.truncation_threshold) == \
        (0.1, True, 1000, 4096, 1e-9)
    assert abs(d.times[-1] - 2.0) < 1e-10
    o = api.Observable("X", api.X, 1)
    T.initialize_observable(o, api.TimeEvolutionConfig([o], 1.0, dt=0.5, sample_timesteps=True, num_traj=10))
    assert o.results.shape == (3,) and o.trajectories.shape == (10, 3)
    T.initialize_observable(o, api.TimeEvolutionConfig([o], 1.0, dt=0.25, sample_timesteps=False, num_traj=5))
    assert o.results.shape == (1,) and o.trajectories.shape == (5, 1)
    s = T.StrongMeasurementConfig([o], num_traj=4, sample_layers=True)
    T.initialize_observable(o, s, num_layers=3)
    assert o.trajectories.shape == (4, 4)
    psi = api.MPS(4, state="x+")
    assert abs(T.expect(psi, api.Observable("X", api.X, 1)) - 1.0) < 1e-10
    assert abs(T.expect(psi, api.Observable("Z", api.Z, 1))) < 1e-10
    assert abs(T.expect(psi, api.Observable("XX", np.kron(api.X, api.X), [3, 2])) - 1.0) < 1e-10
    with pytest.raises(ValueError):
        T.expect(psi, api.Observable("XXX", np.eye(8), [1, 2, 3]))
    agg = api.TimeEvolutionConfig([o], 1.0, num_traj=2, sample_timesteps=False)
    T.initialize_observable(o, agg)
    o.trajectories[0, 0], o.trajectories[1, 0] = 1.0, 0.5
    T.aggregate_trajectories(agg)
    assert abs(o.results[0] - 0.75) < 1e-10


def test_mps_random_state_and_padding():
    """MPS(L; state="random") is normalised with bonds of at most 4
    (MPS.jl:92-103); pad= and pad_bond_dimension! grow every bond to the
    target and leave a normalised state that is the padded one up to the
    noise (MPS.jl:453-494)."""
    r = api.MPS(6, state="random", seed=3)
    assert T.check_if_valid_mps(r) and max(r.bond_dims) <= 4 and r.orth_center == 1
    assert abs(np.linalg.norm(r.to_vec()) - 1) < 1e-12
    p = api.MPS(5, state="x+", pad=4, seed=1)
    # padded to 4, then normalize!'s LQ sweep (L -> 2) trims the last bond to its rank
    assert p.bond_dims == [1, 4, 4, 4, 2, 1]
    assert abs(np.linalg.norm(p.to_vec()) - 1) < 1e-12
    plus = api.MPS(5, state="x+").to_vec()
    assert abs(abs(np.vdot(plus, p.to_vec())) - 1) < 1e-6
    with pytest.raises(ValueError):
        api.MPS(3).pad_bond_dimension(0)


def _randc(rng, *dims):
    return rng.normal(size=dims) + 1j * rng.normal(size=dims)


def test_decompositions_known_answers():
    """test_Decompositions.jl:18-117: right_qr / left_qr shapes,
    reconstruction and isometry; two_site_svd reconstruction, truncation by
    a large threshold and by max_bond_dim."""
    rng = np.random.default_rng(9)
    X = _randc(rng, 4, 2, 5)
    Q, R = T.right_qr(X)
    nb = Q.shape[2]
    assert Q.shape == (4, 2, nb) and R.shape == (nb, 5)
    assert np.allclose(np.einsum("lpk,kr->lpr", Q, R), X, atol=1e-12)
    Qm = np.reshape(Q, (8, nb), order="F")
    assert np.allclose(Qm.conj().T @ Qm, np.eye(nb), atol=1e-12)
    Y = _randc(rng, 5, 2, 4)
    Lm, Q2 = T.left_qr(Y)
    nb = Q2.shape[0]
    assert Lm.shape == (5, nb) and Q2.shape == (nb, 2, 4)
    assert np.allclose(np.einsum("lk,kpr->lpr", Lm, Q2), Y, atol=1e-12)
    Qm = np.reshape(Q2, (nb, 8), order="F")
    assert np.allclose(Qm @ Qm.conj().T, np.eye(nb), atol=1e-12)
    A, B = _randc(rng, 3, 2, 4), _randc(rng, 4, 2, 5)
    An, Bn = T.two_site_svd(A, B, 1e-15)
    assert np.allclose(np.einsum("lak,kbr->labr", A, B), np.einsum("lak,kbr->labr", An, Bn), atol=1e-11)
    At, _ = T.two_site_svd(A, B, 2.0)
    assert At.shape[2] < 6
    Al, Bl = T.two_site_svd(A, B, 1e-15, max_bond_dim=2)
    assert Al.shape[2] == 2 and Bl.shape[0] == 2


def test_two_site_svd_rank_rule_matches_the_oracle(oracle):
    """The kept count is the oracle's absolute rule (rule 0) on the same
    singular values, for thresholds across the spectrum."""
    rng = np.random.default_rng(2)
    A, B = _randc(rng, 4, 2, 6), _randc(rng, 6, 2, 4)
    S = np.linalg.svd(np.reshape(A, (8, 6), order="F") @ np.reshape(B, (6, 8), order="F"), compute_uv=False)
    for thr in (1e-15, 1e-3, 1.0, 10.0, 1e3, 1e6):
        for chi in (None, 3):
            An, _ = T.two_site_svd(A, B, thr, max_bond_dim=chi)
            assert An.shape[2] == oracle.truncation_rank(S, thr, chi or 1 << 30, 0), (thr, chi)


def test_mps_known_answers():
    """test_MPS.jl:97-214: scalar products of random / orthogonal states,
    local expectations, all-site expectations, shots on basis states, the
    recorded centre after a shift and normalize!, truncate! to bond 2."""
    rng = np.random.default_rng(4)
    r = api.MPS(3, state="random", seed=5)
    assert abs(T.scalar_product(r, r) - 1) < 1e-12
    assert abs(T.scalar_product(api.MPS(3, state="zeros"), api.MPS(3, state="ones"))) < 1e-12
    z = api.MPS(2, state="zeros")
    assert abs(T.local_expect(z, api.Z, 1) - 1) < 1e-12 and abs(T.local_expect(z, api.Z, 2) - 1) < 1e-12
    assert abs(T.local_expect(api.MPS(2, state="x+"), api.X, 1) - 1) < 1e-12
    r4 = api.MPS(4, state="random", seed=6)
    ind = [T.local_expect(r4, api.Z, i) for i in range(1, 5)]
    assert np.allclose(ind, T.evaluate_all_local_expectations(r4, [api.Z] * 4), atol=1e-12)
    assert T.measure_single_shot(api.MPS(3, state="zeros")) == 0
    ones = api.MPS(3, state="ones")
    assert T.measure_single_shot(ones) == 7
    assert T.measure_shots(ones, 100, rng=rng) == {7: 100}
    assert sum(T.measure_shots(api.MPS(4, state="x+"), 100, rng=rng).values()) == 100
    m = _rand_mps(4, 4, 8)
    T.shift_orthogonality_center(m, 2)
    assert T.check_canonical_form(m) == [2]
    T.normalize(m)
    assert m.orth_center == 1 and abs(T.scalar_product(m, m) - 1) < 1e-12
    big = api.MPS(6, tensors=[_randc(rng, 1, 2, 8)] + [_randc(rng, 8, 2, 8) for _ in range(4)] +
                  [_randc(rng, 8, 2, 1)])
    T.normalize(big)
    T.truncate(big, max_bond_dim=2)
    assert max(max(t.shape[0], t.shape[2]) for t in big.tensors) <= 2
    T.normalize(big)
    assert abs(T.scalar_product(big, big) - 1) < 1e-10


def test_mpo_known_answers():
    """test_MPO.jl:10-150: identity / zero MPOs, orthogonalize! keeps
    <psi|W|psi> and records the centre, truncate! caps the bonds and leaves
    the centre at L, H1 + H2 = init_ising(L, 1, 1) and compresses, c * W,
    X * X = I."""
    rng = np.random.default_rng(12)
    I4 = T.mpo_identity(4)
    assert I4.tensors[0][0, 0, 0, 0] == 1 and I4.tensors[0][0, 1, 1, 0] == 1 and I4.tensors[0][0, 0, 1, 0] == 0
    assert np.abs(T.mpo_zero(4).tensors[0]).sum() == 0 and I4.orth_center == 0
    W = api.MPO(4, [_randc(rng, 1, 2, 2, 4)] + [_randc(rng, 4, 2, 2, 4) for _ in range(2)] + [_randc(rng, 4, 2, 2, 1)])
    psi = api.MPS(4, state="random", seed=3)
    v0 = T.expect_mpo(W, psi)
    T.orthogonalize(W, 1)
    assert W.orth_center == 1 and abs(T.expect_mpo(W, psi) - v0) < 1e-10
    T.mpo_truncate(W, max_bond_dim=2)
    assert W.orth_center == 4 and max(max(t.shape[0], t.shape[3]) for t in W.tensors) <= 2
    assert np.isfinite(T.expect_mpo(W, psi))
    H1, H2 = api.init_ising(3, 1.0, 0.0), api.init_ising(3, 0.0, 1.0)
    Hs = H1 + H2
    p3 = api.MPS(3, state="random", seed=4)
    assert abs(T.expect_mpo(Hs, p3) - T.expect_mpo(api.init_ising(3, 1.0, 1.0), p3)) < 1e-10
    T.orthogonalize(Hs, 1)
    T.mpo_truncate(Hs, threshold=1e-10)
    assert Hs.tensors[1].shape[3] <= 5
    assert abs(T.expect_mpo(2.5 * H1, p3) - 2.5 * T.expect_mpo(H1, p3)) < 1e-12
    assert abs(T.expect_mpo(H1 * 2.5, p3) - 2.5 * T.expect_mpo(H1, p3)) < 1e-12
    X = api.MPO(2, [api.X.reshape(1, 2, 2, 1)] * 2)
    XX = T.contract_mpo_mpo(X, X)
    assert abs(T.expect_mpo(XX, api.MPS(2)) - 1) < 1e-10 and XX.tensors[0].shape[3] == 1


def test_available_cpus(monkeypatch):
    """test_Simulator.jl:23-32: the host's CPU count, or SLURM_CPUS_ON_NODE."""
    import os
    monkeypatch.delenv("SLURM_CPUS_ON_NODE", raising=False)
    assert api.available_cpus() == os.cpu_count()
    monkeypatch.setenv("SLURM_CPUS_ON_NODE", "8")
    assert api.available_cpus() == 8


def test_run_rejects_other_operators():
    """test_Simulator.jl:91-96: an operator that is neither an MPO nor a
    circuit is an error before anything runs (and parallel= is accepted)."""
    cfg = api.TimeEvolutionConfig([], 1.0)
    with pytest.raises(TypeError):
        api.run(api.MPS(2), "InvalidOperator", cfg, parallel=False)


def test_run_host_logic(oracle, monkeypatch):
    """Simulator.run's host side (Simulator.jl:22-141) on CPU: the device
    call is replaced by the oracle here, so only the host logic is under
    test: the config check comes first, a noiseless model runs one
    trajectory, the observables' buffers follow _run_analog / _run_digital,
    and the caller's initial state is left normalised with its centre at 1."""
    def fake_analog(desc, ctx=None):
        tr, chi, st = oracle.analog_run(desc)
        return api.RunResult(tr, tr.mean(0), chi, st)

    def fake_digital(desc, ctx=None):
        tr, chi, st = oracle.digital_run(desc)
        return api.RunResult(tr, tr.mean(0), chi, st)

    monkeypatch.setattr(api, "run_descriptors", fake_analog)
    monkeypatch.setattr(api, "run_circuit_descriptors", fake_digital)
    with pytest.raises(TypeError, match="Only TimeEvolutionConfig"):
        api.run(api.MPS(2), "InvalidOperator", T.StrongMeasurementConfig([]))
    L = 4
    psi = api.MPS(L, tensors=[2.0 * t for t in api.MPS(L, state="x+").tensors])  # norm 16
    psi.orth_center = 3
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 0.3, dt=0.1, num_traj=7, max_bond_dim=4)
    res = api.run(psi, api.init_ising(L, 1, 0.5), cfg, None)
    assert cfg.num_traj == 1 and res.trajectories.shape == (1, L, 4)
    assert obs[0].trajectories.shape == (1, 4) and obs[0].results.shape == (4,)
    assert psi.orth_center == 1 and abs(np.linalg.norm(psi.to_vec()) - 1) < 1e-12
    c = api.DigitalCircuit(L).add_gate(api.Barrier("SAMPLE_OBSERVABLES"), []).add_gate(api.Rx(0.4), [2])
    c.add_gate(api.Barrier("SAMPLE_OBSERVABLES"), [])
    cfg = api.TimeEvolutionConfig(obs, 5.0, dt=1.0, num_traj=3, max_bond_dim=4)
    api.run(api.MPS(L), c, cfg, None)
    assert obs[1].trajectories.shape == (1, 6) and abs(obs[1].results[1] - np.cos(0.4)) < 1e-12
    assert np.all(obs[1].results[2:] == 0)


def test_truncate_refuses_non_finite_tensors():
    """MPS.truncate! raises on NaN/Inf in a two-site tensor (MPS.jl:356-360)."""
    m = _rand_mps(4, 2, 3)
    m.tensors[2] = m.tensors[2].copy()
    m.tensors[2][0, 0, 0] = np.nan
    with pytest.raises(ValueError, match="non-finite"):
        T.truncate(m, max_bond_dim=2)


def _transfer_matrix_expectations(tensors, ops):
    """<O_i> = E_i (A_i^* O_i A_i) R_{i+1} with E_0 = R_L = 1 and the one-sided
    transfer matrices in between, for any gauge (the contraction the device
    uses for 1-site observables on tight chains)."""
    L = len(tensors)
    R = [None] * (L + 1)
    R[L] = np.ones((1, 1), complex)
    for b in range(L - 1, -1, -1):
        A = tensors[b]
        R[b] = np.einsum("xpr,rs,yps->xy", A, R[b + 1], A.conj())
    E = np.ones((1, 1), complex)
    out = []
    for i, A in enumerate(tensors):
        out.append(np.einsum("ab,aqr,pq,bps,rs->", E, A, ops[i], A.conj(), R[i + 1]).real)
        E = np.einsum("ab,apr,bps->rs", E, A, A.conj())
    return np.array(out)


def test_transfer_matrix_observables_equal_the_centre_sweep():
    """On a normalised state in mixed canonical form, the 1-site expectations
    contracted with transfer matrices (centre left in place) equal the
    reference's evaluation, which moves the orthogonality centre to every
    site (MPS.jl:608-676), and the thin QR / LQ steps of that sweep change
    no bond dimension of a tight chain."""
    L = 9
    m = api.random_mps(L, 8, seed=21)
    T.normalize(m)
    T.shift_orthogonality_center(m, 4)
    before = [t.copy() for t in m.tensors]
    dims = [t.shape[2] for t in m.tensors]
    ops = [api.Z if i % 3 == 0 else (api.X if i % 3 == 1 else np.array([[0, -1j], [1j, 0]])) for i in range(L)]
    got = _transfer_matrix_expectations(before, ops)
    ref = T.evaluate_all_local_expectations(m, ops).real
    assert np.abs(got - ref).max() < 1e-12
    assert [t.shape[2] for t in m.tensors] == dims
