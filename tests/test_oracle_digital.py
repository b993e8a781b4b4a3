"""Digital TJM oracle: reference known answers (test/test_DigitalTJM.jl,
test/test_DigitalTJM_Noise.jl), exact dense statevector / density-matrix
results, and the host-side circuit planning."""
import numpy as np
import pytest

from oracle import dense as D
from yaqs_julia_b200 import api


def _zs(L):
    return [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]


def test_process_circuit_layers():
    """test_DigitalTJM.jl:13-48: X1, X2 | Rzz(1,2), X3."""
    c = api.DigitalCircuit(4)
    c.add_gate(api.X, [1]).add_gate(api.X, [2]).add_gate(api.Rzz(np.pi / 2), [1, 2]).add_gate(api.X, [3])
    layers, _ = api.process_circuit(c)
    assert [len(l) for l in layers] == [2, 2]
    assert layers[1][0].sites == [1, 2] and layers[1][1].sites == [3]


def test_oracle_plan_matches_host_plan(oracle):
    c = api.DigitalCircuit(5)
    c.add_gate(api.Barrier(), [])
    c.add_gate(api.H, [1]).add_gate(api.CX, [1, 2]).add_gate(api.CX, [2, 3])
    c.add_gate(api.Barrier(), [])
    c.add_gate(api.Barrier("other"), [])
    c.add_gate(api.Rxx(0.3), [1, 5]).add_gate(api.X, [3])
    c.add_gate(api.Barrier(), [])
    layers, _ = api.process_circuit(c)
    start, after, n = api.sample_plan(c)
    nl, ns = oracle.digital_plan(api.CircuitDescriptors.pack_gates(c), len(c.gates))
    # H1 | CX12 | CX23 || Rxx15 X3 ||: four layers, samples at the start and after layers 3 and 4
    assert (nl, ns) == (len(layers), n) == (4, 3)
    assert start and after == [3, 4]


def test_local_noise_model_selection():
    """test_DigitalTJM_Noise.jl:17-51."""
    procs = [api.LocalNoiseProcess("p1", [1], 0.1, api.X), api.LocalNoiseProcess("p2", [2], 0.1, api.Z),
             api.LocalNoiseProcess("p12", [1, 2], 0.1, np.kron(api.X, api.X)),
             api.LocalNoiseProcess("p34", [3, 4], 0.1, np.kron(api.Z, api.Z))]
    nm = api.NoiseModel(procs)
    assert sorted(p.name for p in api.create_local_noise_model(nm, 1, 2).processes) == ["p1", "p12", "p2"]
    assert [p.name for p in api.create_local_noise_model(nm, 3, 4).processes] == ["p34"]
    assert [p.name for p in api.create_local_noise_model(nm, 2, 3).processes] == ["p2"]


def _run(oracle, L, c, obs, nm=None, num_traj=1, chi=64, thr=1e-9, seed=1, uniforms=None):
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=1.0, num_traj=num_traj, max_bond_dim=chi, truncation_threshold=thr)
    mode = api.A.YAQS_RNG_INJECTED if uniforms is not None else api.A.YAQS_RNG_PHILOX
    d = api.CircuitDescriptors(api.MPS(L), c, cfg, nm, rng_mode=mode, seed=seed, uniforms=uniforms)
    return oracle.digital_run(d)


def test_bell_state_known_answer(oracle):
    """test_DigitalTJM.jl:50-72: H(1), Rzz(pi/2)(1,2) gives <Z1> = 0, <Z2> = 1."""
    c = api.DigitalCircuit(2).add_gate(api.H, [1]).add_gate(api.Rzz(np.pi / 2), [1, 2])
    tr, _, _ = _run(oracle, 2, c, _zs(2))
    assert abs(tr[0, 0, 0]) < 1e-10 and abs(tr[0, 1, 0] - 1.0) < 1e-10


def test_entanglement_generation_known_answer(oracle):
    """test_DigitalTJM.jl:74-90: H(1), H(2), Rzz(pi/2) gives <Z1 Z2> = 0."""
    c = api.DigitalCircuit(2).add_gate(api.H, [1]).add_gate(api.H, [2]).add_gate(api.Rzz(np.pi / 2), [1, 2])
    tr, _, _ = _run(oracle, 2, c, [api.Observable("ZZ", np.kron(api.Z, api.Z), [1, 2])])
    assert abs(tr[0, 0, 0]) < 1e-10


def test_one_qubit_gates_take_no_noise(oracle):
    """test_DigitalTJM.jl:92-116: X(1) under Z noise leaves <Z1> = -1."""
    c = api.DigitalCircuit(2).add_gate(api.X, [1])
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [1], "strength": 0.2}], 2)
    tr, _, st = _run(oracle, 2, c, _zs(2), nm=nm, num_traj=4)
    assert np.allclose(tr[:, 0, 0], -1.0, atol=1e-10) and st["jumps"] == 0


def test_strong_noise_keeps_state_normalised(oracle):
    """test_DigitalTJM_Noise.jl:53-77: Rzz(0) with a gamma = 10 X process jumps and stays normalised."""
    c = api.DigitalCircuit(2).add_gate(api.Rzz(0.0), [1, 2])
    nm = api.NoiseModel([api.LocalNoiseProcess("flip", [1], 10.0, api.X)])
    tr, _, st = _run(oracle, 2, c, _zs(2) + [api.Observable("I", np.eye(2), 1)], nm=nm, num_traj=8)
    assert np.allclose(tr[:, 2, 0], 1.0, atol=1e-8)
    assert st["jumps"] == 8 and np.allclose(tr[:, 0, 0], -1.0, atol=1e-8)


def _brickwork(L, depth, long_range=True, seed=0):
    rng = np.random.default_rng(seed)
    c = api.DigitalCircuit(L)
    c.add_gate(api.Barrier(), [])
    for _ in range(depth):
        for i in list(range(1, L, 2)) + list(range(2, L, 2)):
            c.add_gate(api.Rzz(rng.uniform(0, 1)), [i, i + 1])
        for i in range(1, L + 1):
            c.add_gate(api.Rx(rng.uniform(0, 1)), [i])
        if long_range:
            c.add_gate(api.Rxx(rng.uniform(0, 1)), [1, L])
            c.add_gate(api.CX, [L - 1, 2])
        c.add_gate(api.Barrier(), [])
    return c


def test_noiseless_circuit_matches_statevector(oracle):
    L = 6
    c = _brickwork(L, 4)
    tr, chi, _ = _run(oracle, L, c, _zs(L), thr=0.0)
    layers, _ = api.process_circuit(c)
    ref = D.digital_pauli_density(L, layers, [], [D.site_op(api.Z, i, L) for i in range(1, L + 1)])
    # samples after layers that end with a barrier: every barrier-closed block
    _, after, _ = api.sample_plan(c)
    ref = ref[[0] + after]
    assert np.abs(tr[0].T - ref).max() < 1e-12
    assert chi.max() <= 2 ** (L // 2)


def test_pauli_noise_ensemble_matches_exact_channel(oracle):
    """Ensemble mean within 3 standard errors of the exact averaged channel."""
    L = 4
    c = _brickwork(L, 3, seed=4)
    procs = [(m, [i], 0.05) for i in range(1, L + 1) for m in (api.X, api.Y, api.Z)]
    nm = api.NoiseModel([{"name": n, "sites": [i], "strength": 0.05} for i in range(1, L + 1)
                         for n in ("pauli_x", "pauli_y", "pauli_z")], L)
    nt = 3000
    tr, _, st = _run(oracle, L, c, _zs(L), nm=nm, num_traj=nt, seed=99)
    layers, _ = api.process_circuit(c)
    _, after, _ = api.sample_plan(c)
    ref = D.digital_pauli_density(L, layers, procs, [D.site_op(api.Z, i, L) for i in range(1, L + 1)])[[0] + after]
    mean, se = tr.mean(0).T, tr.std(0).T / np.sqrt(nt)
    assert st["jumps"] > 100
    assert np.all(np.abs(mean - ref) <= 3 * se + 1e-12), np.abs(mean - ref) / (se + 1e-15)


@pytest.mark.parametrize("chi,thr", [(4, 1e-9), (64, 1e-3)])
def test_truncated_bond_dimensions_respect_caps(oracle, chi, thr):
    L = 8
    c = _brickwork(L, 5, seed=2)
    tr, mx, _ = _run(oracle, L, c, _zs(L), chi=chi, thr=thr)
    assert mx.max() <= chi
    assert np.all(np.abs(tr) <= 1 + 1e-9)


def _run_m(oracle, L, c, obs, method, nm=None, num_traj=1, chi=64, thr=0.0, seed=1, uniforms=None, psi=None):
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=1.0, num_traj=num_traj, max_bond_dim=chi, truncation_threshold=thr)
    mode = api.A.YAQS_RNG_INJECTED if uniforms is not None else api.A.YAQS_RNG_PHILOX
    d = api.CircuitDescriptors(psi or api.MPS(L), c, cfg, nm, rng_mode=mode, seed=seed, uniforms=uniforms,
                               local_method=method, long_range_method=method)
    return oracle.digital_run(d)


def test_generators_reproduce_gate_matrices():
    """exp(-i coeff g1 (x) g2) in the p1 + 2 p2 basis (g1 on the first site)
    is the gate for the symmetric gates; CX's generator puts the control on
    its first site while its matrix constant (GateLibrary.jl:144-150) has it
    on the second."""
    import scipy.linalg as sl
    for g in [api.RzzGate(0.7), api.RxxGate(-1.1), api.RyyGate(0.4), api.CZGate(), api.CPhaseGate(0.9)]:
        U = sl.expm(-1j * g.coeff * np.kron(g.generator[1], g.generator[0]))
        assert np.allclose(U, g.matrix, atol=1e-12), g.name
    cx = api.CXGate()
    U = sl.expm(-1j * cx.coeff * np.kron(cx.generator[1], cx.generator[0]))
    swap = api.SWAP
    assert np.allclose(U, swap @ cx.matrix @ swap, atol=1e-12)


def test_tdvp_window_adjacent_gates_are_exact(oracle):
    """A 2-site window is one Krylov exponential of coeff g1 (x) g2 between
    identity environments: the gate itself (DigitalTJM.jl:335-358)."""
    L = 5
    rng = np.random.default_rng(3)
    c = api.DigitalCircuit(L)
    c.add_gate(api.Barrier(), [])
    for _ in range(3):
        for i in range(1, L + 1):
            c.add_gate(api.Rx(rng.uniform(0, 1)), [i])
        for i in list(range(1, L, 2)) + list(range(2, L, 2)):
            g = [api.RzzGate, api.RxxGate, api.RyyGate][rng.integers(3)](rng.uniform(0, 1.5))
            c.add_gate(g, [i, i + 1])
        c.add_gate(api.CZGate(), [2, 3])
        c.add_gate(api.CPhaseGate(0.8), [4, 5])
        c.add_gate(api.Barrier(), [])
    tr_tdvp, chi_tdvp, _ = _run_m(oracle, L, c, _zs(L), "tdvp")
    tr_tebd, _, _ = _run_m(oracle, L, c, _zs(L), "tebd")
    assert np.abs(tr_tdvp - tr_tebd).max() < 1e-9


def test_tdvp_window_long_range_gate_matches_dense_with_full_bonds(oracle):
    """A long-range Rzz by the TDVP window against the exact gate: with bonds
    already at full rank the projected sweep reproduces it."""
    L = 4
    c = api.DigitalCircuit(L)
    for i in range(1, L + 1):
        c.add_gate(api.H, [i])
    for i in range(1, L):
        c.add_gate(api.CZGate(), [i, i + 1])
    c.add_gate(api.Barrier(), [])
    c.add_gate(api.RzzGate(0.6), [1, 4])
    c.add_gate(api.Barrier(), [])
    layers, _ = api.process_circuit(c)
    ref = D.digital_pauli_density(L, layers, [], [D.site_op(api.Z, i, L) for i in range(1, L + 1)] +
                                  [D.site_op(api.X, i, L) for i in range(1, L + 1)])
    obs = _zs(L) + [api.Observable(f"X{i}", api.X, i) for i in range(1, L + 1)]
    psi = api.MPS(L).pad_bond_dimension(4, 1e-9, seed=1)
    tr, _, _ = _run_m(oracle, L, c, obs, "tdvp", psi=psi, chi=4)
    _, after, _ = api.sample_plan(c)
    assert np.abs(tr[0].T - ref[after]).max() < 1e-8


def test_tdvp_method_needs_generators(oracle):
    c = api.DigitalCircuit(2).add_gate(api.SWAP, [1, 2])
    with pytest.raises(RuntimeError, match="generator"):
        _run_m(oracle, 2, c, _zs(2), "tdvp")


def test_ising_circuit_bitflip_ensemble(oracle):
    """test_Ising_Digital_TJM.jl:11-58: create_ising_circuit(6, 1, 1, 0.1,
    10) with custom-named bit-flip processes (an X matrix under names the
    Pauli name list does not hold) at 0.05, 200 trajectories: the sampled
    <Z_1> starts at 1, stays in [-1, 1] and decays; the ensemble agrees with
    the exact averaged channel within 3 standard errors."""
    from yaqs_julia_b200 import circuits as CL
    L, steps, nt = 6, 10, 200
    c = CL.create_ising_circuit(L, 1.0, 1.0, 0.1, steps)
    nm = api.NoiseModel([{"name": f"bitflip_{i}", "sites": [i], "strength": 0.05, "matrix": api.X}
                         for i in range(1, L + 1)], L)
    assert not any(api.is_pauli_name(p.name) for p in nm.processes)
    assert all(api.is_pauli_matrix(p.matrix) for p in nm.processes)
    tr, _, st = _run(oracle, L, c, _zs(L), nm=nm, num_traj=nt, seed=11)
    z1 = tr[:, 0, :].mean(0)
    assert tr.shape[2] == steps + 1 and abs(z1[0] - 1.0) < 1e-12
    assert np.all(np.abs(tr) <= 1 + 1e-9) and z1[-1] < z1[0] and st["jumps"] > 0
    layers, _ = api.process_circuit(c)
    _, after, _ = api.sample_plan(c)
    procs = [(p.matrix, p.sites, p.strength) for p in nm.processes]
    ref = D.digital_pauli_density(L, layers, procs, [D.site_op(api.Z, i, L) for i in range(1, L + 1)])[[0] + after]
    mean, se = tr.mean(0).T, tr.std(0, ddof=1).T / np.sqrt(nt)
    z = np.abs(mean - ref)[1:] / np.maximum(se[1:], 1.5 / nt)
    assert (z > 3).mean() < 0.05 and z.max() < 5, z.max()
