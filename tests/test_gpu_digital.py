"""Digital TJM on the GPU (yaqs_digital_run) against the oracle: every
trajectory's observables within 1e-10 relative on the same draws, identical
bond dimensions and jump counts, plus the reference's known answers."""
import numpy as np
import pytest

from yaqs_julia_b200 import _abi as A
from yaqs_julia_b200 import api

pytestmark = pytest.mark.gpu


def _zs(L):
    return [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]


def _brickwork(L, depth, long_range=True, seed=0, ring=False):
    rng = np.random.default_rng(seed)
    c = api.DigitalCircuit(L)
    c.add_gate(api.Barrier(), [])
    for _ in range(depth):
        for i in list(range(1, L, 2)) + list(range(2, L, 2)):
            c.add_gate(api.Rzz(rng.uniform(0, 1)), [i, i + 1])
        if ring:
            c.add_gate(api.Rzz(rng.uniform(0, 1)), [L, 1])
        for i in range(1, L + 1):
            c.add_gate(api.Rx(rng.uniform(0, 1)), [i])
        if long_range:
            c.add_gate(api.Rxx(rng.uniform(0, 1)), [1, L])
            c.add_gate(api.CX, [L - 1, 2])
        c.add_gate(api.Barrier(), [])
    return c


def _compare(oracle, L, c, obs, nm=None, num_traj=1, chi=64, thr=1e-9, seed=1, uniforms=None, rtol=1e-10,
             psi=None):
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=1.0, num_traj=num_traj, max_bond_dim=chi, truncation_threshold=thr)
    mode = A.YAQS_RNG_INJECTED if uniforms is not None else A.YAQS_RNG_PHILOX
    d = api.CircuitDescriptors(psi if psi is not None else api.MPS(L), c, cfg, nm, rng_mode=mode, seed=seed, uniforms=uniforms)
    ref, chi_ref, st_ref = oracle.digital_run(d)
    got = api.run_circuit_descriptors(d)
    err = np.abs(got.trajectories - ref)
    assert err.max() <= rtol * max(1.0, np.abs(ref).max()), err.max()
    assert np.array_equal(got.max_bond, chi_ref)
    assert got.stats["jumps"] == st_ref["jumps"]
    return got, ref


def test_bell_state_known_answer():
    """test_DigitalTJM.jl:50-72."""
    c = api.DigitalCircuit(2).add_gate(api.H, [1]).add_gate(api.Rzz(np.pi / 2), [1, 2])
    cfg = api.TimeEvolutionConfig(_zs(2), 1.0, dt=1.0)
    api.run(api.MPS(2), c, cfg)
    assert abs(cfg.observables[0].results[0]) < 1e-10 and abs(cfg.observables[1].results[0] - 1) < 1e-10
    assert cfg.num_traj == 1


def test_noiseless_circuit_with_long_range_gates(oracle):
    L = 7
    _compare(oracle, L, _brickwork(L, 4), _zs(L), thr=0.0)


@pytest.mark.parametrize("chi,thr", [(4, 1e-9), (8, 1e-4), (64, 1e-9)])
def test_truncation_paths(oracle, chi, thr):
    L = 8
    _compare(oracle, L, _brickwork(L, 5, seed=3), _zs(L) + [api.Observable("S", None, 4, kind="entropy")],
             chi=chi, thr=thr)


def test_pauli_noise_injected_draws(oracle):
    L = 8
    nm = api.NoiseModel([{"name": n, "sites": [i], "strength": 0.05} for i in range(1, L + 1)
                         for n in ("pauli_x", "pauli_y", "pauli_z")], L)
    c = _brickwork(L, 4, seed=5)
    u = np.random.default_rng(3).random((12, api.max_draws_digital(c)))
    got, _ = _compare(oracle, L, c, _zs(L), nm=nm, num_traj=12, chi=16, uniforms=u)
    assert got.stats["jumps"] > 0


def test_relaxation_and_dephasing_philox(oracle):
    L = 6
    nm = api.NoiseModel([{"name": "lowering", "sites": [i], "strength": 0.1} for i in range(1, L + 1)] +
                        [{"name": "pauli_z", "sites": [i], "strength": 0.1} for i in range(1, L + 1)], L)
    c = _brickwork(L, 4, seed=6)
    psi = api.MPS(L, state="x+")
    got, _ = _compare(oracle, L, c, _zs(L), nm=nm, num_traj=10, chi=16, seed=0xBEEF, psi=psi)
    assert got.stats["jumps"] > 0


def test_two_site_processes_take_the_reference_sweeps(oracle):
    """Two-site dissipators that split run the full reference sweeps."""
    L = 5
    nm = api.NoiseModel([{"name": "crosstalk_xz", "sites": [2, 3], "strength": 0.3},
                         {"name": "lowering_two", "sites": [3, 4], "strength": 0.5},
                         {"name": "raising", "sites": [1], "strength": 0.2}], L)
    c = _brickwork(L, 3, seed=7, long_range=False)
    u = np.random.default_rng(9).random((6, api.max_draws_digital(c)))
    _compare(oracle, L, c, [api.Observable(f"X{i}", api.X, i) for i in range(1, L + 1)], nm=nm, num_traj=6,
             chi=8, uniforms=u, psi=api.MPS(L, state="x+"))


def test_ring_circuit_with_edge_gate(oracle):
    """The (L, 1) edge of a ring runs as a SWAP chain of 2(L-2) gates."""
    L = 10
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [i], "strength": 0.02} for i in range(1, L + 1)], L)
    _compare(oracle, L, _brickwork(L, 3, seed=8, ring=True, long_range=False), _zs(L), nm=nm, num_traj=6,
             chi=16, seed=4)


def test_untight_start_state(oracle):
    """A start state with oversized bonds takes the sweeps that shrink them."""
    L = 6
    psi = api.random_mps(L, 8, seed=1)
    ts = list(psi.tensors)
    rng = np.random.default_rng(2)
    ts[2] = rng.standard_normal((4, 2, 1)) + 0j  # bond 3 drops to 1: bond 2 (4) exceeds 2 x 1
    ts[3] = rng.standard_normal((1, 2, 4)) + 0j
    psi = api.MPS(L, tensors=ts)
    nm = api.NoiseModel([{"name": "pauli_x", "sites": [i], "strength": 0.1} for i in range(1, L + 1)], L)
    _compare(oracle, L, _brickwork(L, 2, seed=9), _zs(L), nm=nm, num_traj=4, chi=8, seed=5, psi=psi)


def test_no_sampling_barrier_measures_at_the_end(oracle):
    L = 4
    c = api.DigitalCircuit(L)
    for i in range(1, L):
        c.add_gate(api.CX, [i, i + 1])
    c.add_gate(api.Barrier("not a sample"), [])
    c.add_gate(api.H, [2])
    got, _ = _compare(oracle, L, c, _zs(L))
    assert got.trajectories.shape == (1, L, 1)


def test_injected_stream_exhaustion_reports_status():
    L = 4
    nm = api.NoiseModel([{"name": "pauli_x", "sites": [i], "strength": 0.5} for i in range(1, L + 1)], L)
    cfg = api.TimeEvolutionConfig(_zs(L), 1.0, dt=1.0, num_traj=2)
    c = _brickwork(L, 2)
    d = api.CircuitDescriptors(api.MPS(L), c, cfg, nm, rng_mode=A.YAQS_RNG_INJECTED,
                               uniforms=np.full((2, 1), 0.5))
    from yaqs_julia_b200._lib import EngineError
    with pytest.raises(EngineError, match="YAQS_E_RNG"):
        api.run_circuit_descriptors(d)


def test_library_plan_matches_host_plan():
    c = _brickwork(6, 3, ring=True)
    layers, _ = api.process_circuit(c)
    assert api.digital_plan(c) == (len(layers), api.sample_plan(c)[2])


def test_session_steps_match_one_call(oracle):
    """yaqs_digital_begin + advance per layer gives the one-call result."""
    L = 6
    nm = api.NoiseModel([{"name": "pauli_y", "sites": [i], "strength": 0.05} for i in range(1, L + 1)], L)
    c = _brickwork(L, 3, seed=11)
    cfg = api.TimeEvolutionConfig(_zs(L), 1.0, dt=1.0, num_traj=5, max_bond_dim=16)
    d = api.CircuitDescriptors(api.MPS(L), c, cfg, nm, seed=21)
    one = api.run_circuit_descriptors(d)
    sess = api.Session(d)
    n_layers, _ = api.digital_plan(c)
    assert sess.remaining == n_layers + 1
    while sess.remaining:
        sess.advance(2)
    res = sess.finish()
    assert np.array_equal(res.trajectories, one.trajectories)
    assert res.stats["flops"] > 0


def _tdvp_circuit(L, depth, seed, long_range=True):
    rng = np.random.default_rng(seed)
    c = api.DigitalCircuit(L)
    c.add_gate(api.Barrier(), [])
    for _ in range(depth):
        for i in range(1, L + 1):
            c.add_gate(api.Rx(rng.uniform(0, 1)), [i])
        for i in list(range(1, L, 2)) + list(range(2, L, 2)):
            g = [api.RzzGate, api.RxxGate, api.RyyGate][rng.integers(3)](rng.uniform(0, 1.5))
            c.add_gate(g, [i, i + 1])
        c.add_gate(api.CXGate(), [2, 3])
        if long_range:
            c.add_gate(api.RzzGate(rng.uniform(0, 1)), [1, L])
            c.add_gate(api.CPhaseGate(rng.uniform(0, 1)), [L - 1, 2])
        c.add_gate(api.Barrier(), [])
    return c


@pytest.mark.parametrize("chi", [4, 32])
def test_tdvp_window_gates_match_oracle(oracle, chi):
    """apply_window! with :TDVP, the reference's default TJMOptions (window
    MPO + forward circuit 2-site sweep), with Pauli noise after every gate."""
    L = 7
    c = _tdvp_circuit(L, 3, seed=12)
    nm = api.NoiseModel([{"name": n, "sites": [i], "strength": 0.03} for i in range(1, L + 1)
                         for n in ("pauli_x", "pauli_z")], L)
    cfg = api.TimeEvolutionConfig(_zs(L), 1.0, dt=1.0, num_traj=6, max_bond_dim=chi)
    u = np.random.default_rng(13).random((6, api.max_draws_digital(c)))
    d = api.CircuitDescriptors(api.MPS(L), c, cfg, nm, rng_mode=A.YAQS_RNG_INJECTED, uniforms=u,
                               local_method="tdvp", long_range_method="tdvp")
    ref, chi_ref, st_ref = oracle.digital_run(d)
    got = api.run_circuit_descriptors(d)
    assert np.abs(got.trajectories - ref).max() < 1e-10
    assert np.array_equal(got.max_bond, chi_ref)
    assert got.stats["jumps"] == st_ref["jumps"]


def test_tdvp_local_tebd_long_range_mix(oracle):
    L = 6
    c = _tdvp_circuit(L, 2, seed=14)
    cfg = api.TimeEvolutionConfig(_zs(L), 1.0, dt=1.0, num_traj=1, max_bond_dim=16)
    d = api.CircuitDescriptors(api.MPS(L), c, cfg, None, local_method="tdvp", long_range_method="tebd")
    ref, chi_ref, _ = oracle.digital_run(d)
    got = api.run_circuit_descriptors(d)
    assert np.abs(got.trajectories - ref).max() < 1e-10
    assert np.array_equal(got.max_bond, chi_ref)


@pytest.mark.parametrize("unravel", ["projector", "unitary_gauss"])
def test_unraveled_gate_noise(oracle, unravel):
    """Gate-local noise with unraveled processes (the paper's digital
    unraveling studies): device vs oracle on injected draws."""
    L = 6
    c = _brickwork(L, 2, seed=21)
    info = [{"name": n, "sites": [i], "strength": 0.05, "unraveling": unravel}
            for i in range(1, L + 1) for n in ("pauli_x", "pauli_z")]
    info += [{"name": "crosstalk_zz", "sites": [i, i + 1], "strength": 0.05, "unraveling": unravel}
             for i in range(1, L)]
    nm = api.NoiseModel(info, L)
    u = np.random.default_rng(5).random((8, api.max_draws_digital(c)))
    got, _ = _compare(oracle, L, c, _zs(L), nm=nm, num_traj=8, uniforms=u)
    assert got.stats["jumps"] > 0


@pytest.mark.parametrize("method", ["tebd", "tdvp"])
def test_long_range_gate_noise(oracle, method):
    """Long-range gates take the long-range processes on their own pair
    (DigitalTJM.jl:172-188): MPO jumps on the device vs the oracle."""
    L = 6
    c = _tdvp_circuit(L, 2, seed=41) if method == "tdvp" else _brickwork(L, 2, seed=41)
    info = [{"name": "crosstalk_zz", "sites": [1, L], "strength": 0.3, "unraveling": "projector"},
            {"name": "crosstalk_xy", "sites": [1, L], "strength": 0.2, "unraveling": "unitary_2pt"},
            {"name": "crosstalk_xx", "sites": [2, L - 1], "strength": 0.3, "unraveling": "unitary_gauss", "M": 3},
            {"name": "crosstalk_yy", "sites": [3, L - 1], "strength": 0.3},
            {"name": "pauli_x", "sites": [2], "strength": 0.05}]
    nm = api.NoiseModel(info, L)
    u = np.random.default_rng(43).random((8, api.max_draws_digital(c)))
    cfg = api.TimeEvolutionConfig(_zs(L), 1.0, dt=1.0, num_traj=8, max_bond_dim=16)
    d = api.CircuitDescriptors(api.MPS(L), c, cfg, nm, rng_mode=A.YAQS_RNG_INJECTED, uniforms=u,
                               local_method=method, long_range_method=method)
    ref, chi_ref, st_ref = oracle.digital_run(d)
    got = api.run_circuit_descriptors(d)
    assert np.abs(got.trajectories - ref).max() <= 1e-10
    assert np.array_equal(got.max_bond, chi_ref)
    assert got.stats["jumps"] == st_ref["jumps"] > 0


@pytest.mark.parametrize("method", ["tebd", "tdvp"])
def test_circuit_library_fermi_hubbard(oracle, method):
    """A circuit-library generator (1D Fermi-Hubbard: long-range on-site
    CPhase between j and j+L, descending hopping pairs) with gate noise."""
    from yaqs_julia_b200 import circuits as C
    c = C.create_1d_fermi_hubbard_circuit(3, 1.2, 0.8, 0.3, 1, 0.3, 2)
    c.gates.insert(0, api.DigitalGate(api.Barrier(), []))
    c.add_gate(api.Barrier(), [])
    L = c.num_qubits
    nm = api.NoiseModel([{"name": n, "sites": [i], "strength": 0.02} for i in range(1, L + 1)
                         for n in ("pauli_x", "pauli_z")], L)
    u = np.random.default_rng(47).random((6, api.max_draws_digital(c)))
    cfg = api.TimeEvolutionConfig(_zs(L), 1.0, dt=1.0, num_traj=6, max_bond_dim=16)
    psi = api.MPS(L, state="Neel")
    d = api.CircuitDescriptors(psi, c, cfg, nm, rng_mode=A.YAQS_RNG_INJECTED, uniforms=u,
                               local_method=method, long_range_method=method)
    ref, chi_ref, st_ref = oracle.digital_run(d)
    got = api.run_circuit_descriptors(d)
    assert np.abs(got.trajectories - ref).max() <= 1e-10
    assert np.array_equal(got.max_bond, chi_ref) and got.stats["jumps"] == st_ref["jumps"]


def test_run_repeated_library_circuit_defaults_to_tdvp_windows(oracle):
    """api.run on a RepeatedDigitalCircuit of library gates: the reference's
    default TJMOptions (TDVP windows) and its per-repetition sample plan."""
    from yaqs_julia_b200 import circuits as C
    L = 6
    step = C.create_ising_circuit(L, 1.0, 0.7, 0.1, 1, periodic=True)
    rep = api.RepeatedDigitalCircuit(step, 4)
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [i], "strength": 0.03} for i in range(1, L + 1)], L)
    obs = _zs(L)
    cfg = api.TimeEvolutionConfig(obs, 4.0, dt=1.0, num_traj=8, max_bond_dim=16)
    res = api.run(api.MPS(L, state="wall"), rep, cfg, nm, seed=61)
    d = api.CircuitDescriptors(api.MPS(L, state="wall"), rep, cfg, nm, seed=61, local_method="tdvp",
                               long_range_method="tdvp")
    ref, chi_ref, _ = oracle.digital_run(d)
    assert ref.shape[2] == 5
    assert np.abs(res.trajectories - ref).max() <= 1e-10 and np.array_equal(res.max_bond, chi_ref)


def test_session_state_snapshot():
    """yaqs_run_state: a trajectory's final state copied from the device
    reproduces the observables recorded at the last sample."""
    from yaqs_julia_b200 import tensornet as T
    L = 6
    c = _brickwork(L, 2, seed=71)
    nm = api.NoiseModel([{"name": "pauli_x", "sites": [i], "strength": 0.05} for i in range(1, L + 1)], L)
    cfg = api.TimeEvolutionConfig(_zs(L), 1.0, dt=1.0, num_traj=5, max_bond_dim=16)
    d = api.CircuitDescriptors(api.MPS(L), c, cfg, nm, seed=9)
    sess = api.Session(d)
    sess.advance(sess.remaining)
    states = [sess.state(k) for k in range(5)]
    res = sess.finish()
    for k, m in enumerate(states):
        assert T.check_if_valid_mps(m) and abs(np.linalg.norm(m.to_vec()) - 1) < 1e-10
        z = [T.local_expect(m, api.Z, i).real for i in range(1, L + 1)]
        assert np.abs(np.array(z) - res.trajectories[k, :, -1]).max() < 1e-10
        assert T.write_max_bond_dim(m) == res.max_bond[k, -1]


def test_checkpoint_restore_digital():
    L = 6
    c = _brickwork(L, 3, seed=73)
    nm = api.NoiseModel([{"name": "pauli_y", "sites": [i], "strength": 0.06} for i in range(1, L + 1)], L)
    cfg = api.TimeEvolutionConfig(_zs(L), 1.0, dt=1.0, num_traj=5, max_bond_dim=16)
    d = api.CircuitDescriptors(api.MPS(L), c, cfg, nm, seed=19)
    straight = api.run_circuit_descriptors(d)
    sess = api.Session(d)
    sess.advance(3)
    cp = sess.checkpoint()
    sess.advance(2)
    sess.restore(cp)
    sess.advance(sess.remaining)
    res = sess.finish()
    assert np.array_equal(res.trajectories, straight.trajectories)
    assert np.array_equal(res.max_bond, straight.max_bond)


def test_ising_circuit_bitflip_run(oracle):
    """test_Ising_Digital_TJM.jl:11-58 through run(): create_ising_circuit
    with custom-named bit-flip processes, a TimeEvolutionConfig of 51 time
    points (T = 50, dt = 1) holding the 11 samples, 200 trajectories; the
    results equal the oracle on the same draws and keep the reference's
    buffer length."""
    from yaqs_julia_b200 import circuits as CL
    L, steps, nt = 6, 10, 200
    c = CL.create_ising_circuit(L, 1.0, 1.0, 0.1, steps)
    nm = api.NoiseModel([{"name": f"bitflip_{i}", "sites": [i], "strength": 0.05, "matrix": api.X}
                         for i in range(1, L + 1)], L)
    obs = [api.Observable(f"Z_{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 50.0, dt=1.0, num_traj=nt, sample_timesteps=True)
    res = api.run(api.MPS(L, state="zeros"), c, cfg, nm, seed=4)
    z1 = obs[0].results
    assert len(z1) == 51 > steps and abs(z1[0] - 1.0) < 1e-12
    assert np.all(np.abs(z1) <= 1 + 1e-9) and np.all(z1[steps + 1:] == 0)
    d = api.CircuitDescriptors(api.MPS(L, state="zeros"), c, cfg, nm, seed=4,
                               **api._methods(c, None, None))
    ref, _, _ = oracle.digital_run(d)
    assert np.abs(res.trajectories - ref).max() <= 1e-10


@pytest.mark.parametrize("method", ["tebd", "tdvp"])
def test_program_sizes_agree(method, monkeypatch):
    """Direct digital runs use the 128-thread program kernel; the 256-thread
    kernel (YAQS_DIGITAL_THREADS=256) gives the same trajectories to rounding,
    the same bond dimensions and the same jumps, on a noisy circuit with
    long-range gates (TEBD SWAP chains or TDVP windows)."""
    L = 9
    nm = api.NoiseModel([{"name": n, "sites": [i], "strength": 0.03} for i in range(1, L + 1)
                         for n in ("pauli_x", "pauli_z", "lowering")], L)
    obs = _zs(L) + [api.Observable("S", None, 4, kind="entropy")]
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=1.0, num_traj=40, max_bond_dim=16, truncation_threshold=1e-9)
    c = _tdvp_circuit(L, 3, seed=11) if method == "tdvp" else _brickwork(L, 4, seed=11)

    def run():
        d = api.CircuitDescriptors(api.MPS(L), c, cfg, nm, seed=21, local_method=method, long_range_method=method)
        return api.run_circuit_descriptors(d)

    small = run()
    monkeypatch.setenv("YAQS_DIGITAL_THREADS", "256")
    big = run()
    assert np.abs(small.trajectories - big.trajectories).max() <= 1e-10
    assert np.array_equal(small.max_bond, big.max_bond)
    assert small.stats["jumps"] == big.stats["jumps"] > 0


def test_local_observables_by_transfer_matrices(oracle):
    """After a layer, 1-site observables on a tight chain are contracted with
    transfer matrices and the centre stays put, where the oracle moves the
    centre across the chain as the reference does; an entropy observable
    then moves the device's centre to its site only.  Both runs give the
    oracle's <Z_i> on the same draws, with the same jumps and bond
    dimensions, under Pauli and relaxation noise with long-range gates."""
    L = 10
    nm = api.NoiseModel([{"name": n, "sites": [i], "strength": 0.04} for i in range(1, L + 1)
                         for n in ("pauli_x", "pauli_z", "lowering")], L)
    c = _brickwork(L, 5, seed=17)
    z, _ = _compare(oracle, L, c, _zs(L), nm=nm, num_traj=24, chi=16)
    zs, _ = _compare(oracle, L, c, _zs(L) + [api.Observable("S", None, 5, kind="entropy")], nm=nm, num_traj=24,
                     chi=16)
    assert np.abs(z.trajectories - zs.trajectories[:, :L]).max() <= 1e-10
    assert np.array_equal(z.max_bond, zs.max_bond) and z.stats["jumps"] == zs.stats["jumps"] > 0
