"""Edge cases through the C-ABI against the oracle: the shortest chains,
zero-strength and absent noise, circuits without gates or without sample
barriers, every TDVP mode at L=2 and 3, bond capacities reached from the
start, and the argument checks."""
import numpy as np
import pytest

from yaqs_julia_b200 import _abi as A
from yaqs_julia_b200 import api

pytestmark = pytest.mark.gpu


def _analog(L, mode, nm, T=0.4, nt=3, chi=8, state="x+"):
    H = api.init_ising(L, 1.0, 0.8)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    if L >= 2:
        obs.append(api.Observable("ZZ", np.kron(api.Z, api.Z), [1, 2]))
    cfg = api.TimeEvolutionConfig(obs, T, dt=0.1, num_traj=nt, max_bond_dim=chi)
    return api.Descriptors(api.MPS(L, state=state), H, cfg, nm, seed=5, tdvp_mode=api.TDVP_MODES[mode])


@pytest.mark.parametrize("mode", ["2site", "1site", "dynamic"])
@pytest.mark.parametrize("L", [2, 3])
def test_shortest_chains(oracle, L, mode):
    nm = api.NoiseModel([{"name": "lowering", "sites": [i], "strength": 1.5} for i in range(1, L + 1)], L)
    d = _analog(L, mode, nm, T=0.6, nt=6)
    ref, chi_ref, st = oracle.analog_run(d)
    got = api.run_descriptors(d)
    assert np.abs(got.trajectories - ref).max() <= 1e-10
    assert np.array_equal(got.max_bond, chi_ref) and got.stats["jumps"] == st["jumps"] > 0


@pytest.mark.parametrize("nm", [None, "zero"])
def test_absent_and_zero_noise(oracle, nm):
    L = 5
    model = None if nm is None else api.NoiseModel(
        [{"name": "pauli_z", "sites": [i], "strength": 0.0} for i in range(1, L + 1)], L)
    d = _analog(L, "2site", model, nt=2)
    ref, _, st = oracle.analog_run(d)
    got = api.run_descriptors(d)
    assert np.abs(got.trajectories - ref).max() <= 1e-10 and got.stats["jumps"] == 0 == st["jumps"]
    # without noise the trajectories coincide
    assert np.array_equal(got.trajectories[0], got.trajectories[1])


def test_saturated_start_at_capacity(oracle):
    """Every bond of the start state already at max_bond_dim."""
    L, chi = 8, 8
    psi = api.random_mps(L, chi, seed=4)
    H = api.init_general_hamiltonian(L, 1, 1, 1, 0, 0, 0.2)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 0.3, dt=0.1, num_traj=3, max_bond_dim=chi)
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [i], "strength": 0.1} for i in range(1, L + 1)], L)
    for mode in ("2site", "dynamic"):
        d = api.Descriptors(psi, H, cfg, nm, seed=8, tdvp_mode=api.TDVP_MODES[mode])
        ref, chi_ref, _ = oracle.analog_run(d)
        got = api.run_descriptors(d)
        assert np.abs(got.trajectories - ref).max() <= 1e-10 and np.array_equal(got.max_bond, chi_ref)
        assert got.max_bond.max() == chi


def test_circuit_without_gates(oracle):
    L = 4
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=1.0, num_traj=2, max_bond_dim=8)
    for c in (api.DigitalCircuit(L), api.DigitalCircuit(L).add_gate(api.Barrier(), [])):
        d = api.CircuitDescriptors(api.MPS(L, state="Neel"), c, cfg, None)
        ref, _, _ = oracle.digital_run(d)
        got = api.run_circuit_descriptors(d)
        assert got.trajectories.shape == ref.shape and np.array_equal(got.trajectories, ref)
        assert np.allclose(got.trajectories[0, :, 0], [1, -1, 1, -1])


def test_one_qubit_gates_only_with_noise(oracle):
    """No 2-qubit gate: the gate-local noise never acts (DigitalTJM.jl:402-420)."""
    L = 3
    c = api.DigitalCircuit(L).add_gate(api.Barrier(), []).add_gate(api.Rx(0.7), [2]).add_gate(api.Barrier(), [])
    nm = api.NoiseModel([{"name": "pauli_x", "sites": [i], "strength": 1.0} for i in range(1, L + 1)], L)
    cfg = api.TimeEvolutionConfig([api.Observable("Z2", api.Z, 2)], 1.0, dt=1.0, num_traj=3, max_bond_dim=4)
    d = api.CircuitDescriptors(api.MPS(L), c, cfg, nm, seed=2)
    got = api.run_circuit_descriptors(d)
    ref, _, _ = oracle.digital_run(d)
    assert np.array_equal(got.trajectories, ref) and got.stats["jumps"] == 0
    assert np.allclose(got.trajectories[:, 0, -1], np.cos(0.7), atol=1e-12)


def test_argument_checks():
    from yaqs_julia_b200._lib import EngineError
    L = 4
    H = api.init_ising(L, 1.0, 0.5)
    cfg = api.TimeEvolutionConfig([api.Observable("Z1", api.Z, 1)], 0.2, dt=0.1, num_traj=2, max_bond_dim=4)
    d = api.Descriptors(api.MPS(L), H, cfg, None)
    d.cfg.krylov_dim = 0
    with pytest.raises(EngineError, match="krylov_dim"):
        api.run_descriptors(d)
    big = api.TimeEvolutionConfig([api.Observable("Z1", api.Z, 1)], 0.2, dt=0.1, num_traj=1, max_bond_dim=256)
    with pytest.raises(EngineError, match="128"):  # a 20-site chain could reach bond 256
        api.run_descriptors(api.Descriptors(api.MPS(20), api.init_ising(20, 1.0, 0.5), big, None))
    d = api.Descriptors(api.MPS(L), H, cfg, None, rng_mode=A.YAQS_RNG_INJECTED,
                        uniforms=np.zeros((2, 1)))
    d.rng.uniforms = None
    with pytest.raises(EngineError, match="injected"):
        api.run_descriptors(d)


@pytest.mark.parametrize("order", [2, 1])
@pytest.mark.parametrize("sample", [False, True])
def test_identity_hamiltonian_result_shapes(oracle, order, sample):
    """test_AnalogTJM.jl:44-100 through the C-ABI: identity MPO (bond width
    1), T = 0.2, dt = 0.1: one column without sampling, three with it."""
    from yaqs_julia_b200 import tensornet as T
    L = 5
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 0.2, dt=0.1, num_traj=1, max_bond_dim=8, sample_timesteps=sample,
                                  order=order)
    d = api.Descriptors(api.MPS(L, state="zeros"), T.mpo_identity(L), cfg, None)
    got = api.run_descriptors(d)
    ref, _, _ = oracle.analog_run(d)
    assert got.trajectories.shape == ref.shape == (1, L, 3 if sample else 1)
    assert np.abs(got.trajectories - ref).max() <= 1e-12 and np.allclose(got.trajectories, 1.0, atol=1e-12)


def test_simulator_run_without_sampling(oracle):
    """test_Simulator.jl:34-64: Simulator.run with lowering + pauli_z at 0.1,
    10 trajectories, max_bond_dim 4, threshold 1e-6, order 2, no sampling:
    one result per observable and one row per trajectory, equal to the
    oracle on the same Philox draws."""
    from yaqs_julia_b200 import tensornet as T
    L = 5
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=0.1, num_traj=10, max_bond_dim=4, truncation_threshold=1e-6,
                                  order=2, sample_timesteps=False)
    info = [{"name": n, "sites": [i], "strength": 0.1} for n in ("lowering", "pauli_z") for i in range(1, L + 1)]
    nm = api.NoiseModel(info, L)
    res = api.run(api.MPS(L, state="zeros"), T.mpo_identity(L), cfg, nm, seed=3)
    assert res.trajectories.shape == (10, L, 1)
    for o in cfg.observables:
        assert len(o.results) == 1 and o.trajectories.shape[0] == 10
    ref, _, _ = oracle.analog_run(api.Descriptors(api.MPS(L, state="zeros"), T.mpo_identity(L), cfg, nm, seed=3))
    assert np.abs(res.trajectories - ref).max() <= 1e-10
