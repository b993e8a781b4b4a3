"""Noise unravelings (src/Noise.jl:134-420): the NoiseModel constructor
expands a process into several jump operators that share its Lindbladian.
Known answers from test/test_Noise.jl:24-73, the Lindbladian identity on
random density matrices, and oracle ensembles against the exact dynamics."""
import math
import warnings

import numpy as np
import pytest

from yaqs_julia_b200 import api
from oracle import dense as D


def test_projector_unraveling_known_answer():
    """test_Noise.jl:24-55: pauli_z at 0.2 -> I+Z and I-Z at 0.1 each."""
    m = api.NoiseModel([{"name": "pauli_z", "sites": [1], "strength": 0.2, "unraveling": "projector"}], 2)
    assert [p.name for p in m.processes] == ["projector_plus_pauli_z", "projector_minus_pauli_z"]
    assert all(p.strength == 0.1 for p in m.processes)
    assert np.array_equal(m.processes[0].matrix, np.eye(2) + api.Z)
    assert np.array_equal(m.processes[1].matrix, np.eye(2) - api.Z)


def test_unitary_2pt_unraveling_known_answer():
    """test_Noise.jl:57-73: pauli_x at 0.2 with theta0 = 0.1."""
    m = api.NoiseModel([{"name": "pauli_x", "sites": [1], "strength": 0.2, "unraveling": "unitary_2pt",
                         "theta0": 0.1}], 2)
    assert len(m.processes) == 2
    assert math.isclose(m.processes[0].strength, (0.2 / math.sin(0.1) ** 2) / 2, rel_tol=1e-15)
    u_plus = math.cos(0.1) * np.eye(2) + 1j * math.sin(0.1) * api.X
    assert np.allclose(m.processes[0].matrix, u_plus, atol=1e-14)
    assert np.allclose(m.processes[1].matrix, u_plus.conj(), atol=1e-14)
    assert [p.name for p in m.processes] == ["unitary2pt_plus_pauli_x", "unitary2pt_minus_pauli_x"]


def test_unitary_2pt_default_theta_and_stability_warning():
    m = api.NoiseModel([{"name": "pauli_y", "sites": [2], "strength": 0.3, "unraveling": "unitary_2pt"}], 2)
    # theta0 = pi/2: exp(+-i pi/2 Y) = +-iY at the full rate split in two
    assert np.allclose(m.processes[0].matrix, 1j * api.Y, atol=1e-15)
    assert math.isclose(m.processes[0].strength + m.processes[1].strength, 0.3, rel_tol=1e-15)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        api.NoiseModel([{"name": "pauli_z", "sites": [1], "strength": 0.1, "unraveling": "unitary_2pt",
                         "theta0": 0.2}], 2, dt=0.1)
    assert any("Stability Warning" in str(x.message) for x in w)


def test_unitary_gauss_grid():
    """Noise.jl:225-252 with the defaults sigma = 1, M = 11, k = 4."""
    gamma = 0.1
    m = api.NoiseModel([{"name": "pauli_z", "sites": [3], "strength": gamma, "unraveling": "unitary_gauss"}], 4)
    assert [p.name for p in m.processes] == [f"unitary_gauss_{k}_pauli_z" for k in range(11)]
    thetas, w = api.gauss_angles(1.0, 11, 4.0)
    assert np.allclose(thetas, np.linspace(-4, 4, 11), atol=1e-15)
    assert math.isclose(w.sum(), 1.0, rel_tol=1e-14) and np.array_equal(w, w[::-1])
    rates = np.array([p.strength for p in m.processes])
    # the rates reproduce the dephasing rate: sum_k r_k sin^2 theta_k = gamma
    assert math.isclose(float(np.sum(rates * np.sin(thetas) ** 2)), gamma, rel_tol=1e-13)
    for p, th in zip(m.processes, thetas):
        assert np.allclose(p.matrix, np.diag([np.exp(1j * th), np.exp(-1j * th)]), atol=1e-14)
    # per-process grid overrides
    m2 = api.NoiseModel([{"name": "pauli_z", "sites": [1], "strength": gamma, "unraveling": "unitary_gauss",
                          "M": 5, "theta_max": 1.0, "sigma": 0.5}], 2)
    assert len(m2.processes) == 5
    assert np.allclose(api.gauss_angles(0.5, 5, 1.0)[0], [-1, -0.5, 0, 0.5, 1])


def test_analog_auto_is_deprecated_standard():
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        m = api.NoiseModel([{"name": "lowering", "sites": [1], "strength": 0.1, "unraveling": "analog_auto"}], 2)
    assert any("deprecated" in str(x.message) for x in w)
    assert [p.name for p in m.processes] == ["lowering"] and np.array_equal(m.processes[0].matrix, api.LOWERING)


def test_long_range_processes_need_the_chain_length():
    with pytest.raises(ValueError, match="num_qubits"):
        api.NoiseModel([{"name": "crosstalk_xy", "sites": [1, 3], "strength": 0.05, "unraveling": "projector"}])


def _dissipator(ops, rho):
    out = np.zeros_like(rho)
    for g, L in ops:
        out += g * (L @ rho @ L.conj().T - 0.5 * (L.conj().T @ L @ rho + rho @ L.conj().T @ L))
    return out


@pytest.mark.parametrize("unravel", ["projector", "unitary_2pt", "unitary_gauss"])
@pytest.mark.parametrize("name,sites", [("pauli_x", [2]), ("pauli_y", [1]), ("crosstalk_zx", [2, 3])])
def test_unravelings_share_the_lindbladian(unravel, name, sites):
    L = 3
    gamma = 0.37
    std = api.NoiseModel([{"name": name, "sites": sites, "strength": gamma}], L)
    unr = api.NoiseModel([{"name": name, "sites": sites, "strength": gamma, "unraveling": unravel,
                           "theta0": 0.7}], L)
    rng = np.random.default_rng(5)
    a = rng.normal(size=(8, 8)) + 1j * rng.normal(size=(8, 8))
    rho = a @ a.conj().T
    rho /= np.trace(rho)

    def ops(m):
        return [(p.strength, D.gate_op(p.matrix, p.sites, L)) for p in m.processes]

    assert np.allclose(_dissipator(ops(std), rho), _dissipator(ops(unr), rho), atol=1e-13)


@pytest.mark.parametrize("unravel", ["projector", "unitary_2pt", "unitary_gauss"])
def test_analog_ensemble_matches_lindblad(oracle, unravel):
    """Ising L=4 from |+...+> under Z dephasing (and one crosstalk pair):
    each unraveling's ensemble stays within 3 standard errors of the exact
    Lindblad dynamics of the standard model."""
    L = 4
    H = api.init_ising(L, 1.0, 0.5)
    info = [{"name": "pauli_z", "sites": [i], "strength": 0.15} for i in range(1, L + 1)]
    info.append({"name": "crosstalk_xx", "sites": [2, 3], "strength": 0.1})
    for d in info:
        d["unraveling"] = unravel
        d["theta0"] = math.pi / 3
    nm = api.NoiseModel(info, L)
    Xs = [D.site_op(api.X, s, L) for s in range(1, L + 1)]
    jumps = [np.sqrt(0.15) * D.site_op(api.Z, s, L) for s in range(1, L + 1)]
    jumps.append(np.sqrt(0.1) * D.gate_op(np.kron(api.X, api.X), [2, 3], L))
    plus = np.array([1, 1]) / np.sqrt(2)
    ex = D.lindblad(H.to_matrix(), D.product_state([plus] * L), jumps, 0.05, 20, Xs, substeps=10)
    obs = [api.Observable(f"X{s}", api.X, s) for s in range(1, L + 1)]
    nt = 600
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=0.05, num_traj=nt, max_bond_dim=8)
    traj, _, st = oracle.analog_run(api.Descriptors(api.MPS(L, state="x+"), H, cfg, nm, seed=7))
    mean = traj.mean(0).T
    se = traj.std(0, ddof=1).T / np.sqrt(nt)
    z = np.abs(mean - ex)[1:] / np.maximum(se[1:], 1e-12)
    assert st["jumps"] > 50
    assert (z > 3).mean() < 0.03 and z.max() < 5, z.max()


@pytest.mark.parametrize("unravel", ["unitary_2pt", "unitary_gauss"])
def test_digital_unitary_unravelings_match_the_exact_channel(oracle, unravel):
    """Unitary jumps (U^dag U = I) keep the digital step's channel
    e^{-G} rho + (1 - e^{-G}) sum_k g_k/G U_k rho U_k^dag, computed densely."""
    from test_oracle_digital import _brickwork, _run, _zs
    L = 4
    c = _brickwork(L, 3, seed=8)
    info = [{"name": n, "sites": [i], "strength": 0.04, "unraveling": unravel, "theta0": math.pi / 3}
            for i in range(1, L + 1) for n in ("pauli_x", "pauli_z")]
    nm = api.NoiseModel(info, L)
    procs = [(p.matrix, p.sites, p.strength) for p in nm.processes]
    nt = 3000
    tr, _, st = _run(oracle, L, c, _zs(L), nm=nm, num_traj=nt, seed=123)
    layers, _ = api.process_circuit(c)
    _, after, _ = api.sample_plan(c)
    ref = D.digital_pauli_density(L, layers, procs, [D.site_op(api.Z, i, L) for i in range(1, L + 1)])[[0] + after]
    mean, se = tr.mean(0).T, tr.std(0, ddof=1).T / np.sqrt(nt)
    z = np.abs(mean - ref)[1:] / np.maximum(se[1:], 1e-12)
    assert st["jumps"] > 100
    assert (z > 3).mean() < 0.05 and z.max() < 5, z.max()
