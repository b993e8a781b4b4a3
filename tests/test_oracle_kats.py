"""Known answers of the reference's own unit tests, restated against the
oracle's building blocks: the TDVP eigenstate phase of both sweeps
(test/test_Algorithms.jl:37-95), calculate_stochastic_factor and
create_probability_distribution (test/test_StochasticProcess.jl:16-99) and
apply_dissipation (test/test_Dissipation.jl:24-85)."""
import cmath

import numpy as np
import pytest

from yaqs_julia_b200 import api
from yaqs_julia_b200 import tensornet as T


def _desc(psi, H, nm=None, T_=0.5, dt=0.1, mode="2site", chi=8):
    cfg = api.TimeEvolutionConfig([], T_, dt=dt, num_traj=1, max_bond_dim=chi)
    return api.Descriptors(psi, H, cfg, nm, tdvp_mode=api.TDVP_MODES[mode])


@pytest.mark.parametrize("mode", ["1site", "2site", "dynamic"])
def test_ising_eigenstate_phase(oracle, mode):
    """|0000> is an eigenstate of init_ising(4, 1, 0) with E = -3: five
    sweeps of dt = 0.1 give scalar_product(psi(t), psi0) = exp(1.5i).  The
    reference allows 1e-2 (Krylov/Trotter error); a bond-1 eigenstate is
    evolved exactly, so the oracle must meet it to round-off."""
    d = _desc(api.MPS(4, state="zeros"), api.init_ising(4, 1.0, 0.0), mode=mode)
    ov = oracle.tdvp_overlap(d, 5)
    assert abs(abs(ov) - 1.0) < 1e-12
    assert abs(ov - cmath.exp(1.5j)) < 1e-10


def test_eigenstate_phase_convention_of_the_host_overlap():
    """The host mirror uses the same convention: scalar_product(e^{ia} psi,
    psi) = e^{ia} (the second argument is conjugated)."""
    psi = api.MPS(4, state="zeros")
    rot = api.MPS(4, state="zeros")
    rot.tensors[0] = rot.tensors[0] * cmath.exp(1.5j)
    assert abs(T.scalar_product(rot, psi) - cmath.exp(1.5j)) < 1e-15


def test_stochastic_factor(oracle):
    """dp = 1 - <psi|psi>: 0 for MPS(2, "ones"), 0.75 once site 1 is scaled
    by 0.5 (test_StochasticProcess.jl:16-29)."""
    H = api.init_ising(2, 1.0, 0.5)
    psi = api.MPS(2, state="ones")
    assert abs(oracle.stochastic_factor(_desc(psi, H))) < 1e-12
    psi.tensors[0] = psi.tensors[0] * 0.5
    assert abs(oracle.stochastic_factor(_desc(psi, H)) - 0.75) < 1e-12


def test_probability_distribution_one_site_pauli(oracle):
    """pauli_z on site 1 at 0.5, dt = 0.1, |++>: one local_1 candidate of
    probability 1 (test_StochasticProcess.jl:31-48)."""
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [1], "strength": 0.5}], 2)
    probs, cands = oracle.probability_distribution(_desc(api.MPS(2, state="x+"), api.init_ising(2, 1, 0.5), nm),
                                                   0.1)
    assert len(probs) == 1 and abs(probs[0] - 1.0) < 1e-14
    assert cands == [("local_1", [1])]


def test_probability_distribution_two_site_custom(oracle):
    """A custom Z(x)Z process on (1, 2) at 0.2 with |11>: one local_2
    candidate of probability 1 (test_StochasticProcess.jl:50-73)."""
    proc = api.LocalNoiseProcess("custom_zz", [1, 2], 0.2, np.kron(api.Z, api.Z))
    nm = api.NoiseModel([proc], 2)
    probs, cands = oracle.probability_distribution(_desc(api.MPS(2, state="ones"), api.init_ising(2, 1, 0.5), nm),
                                                   0.1)
    assert len(probs) == 1 and abs(probs[0] - 1.0) < 1e-14
    assert cands == [("local_2", [1, 2])]


def test_probability_distribution_long_range_pauli(oracle):
    """crosstalk_zz on (1, 3) of L = 3 with its Pauli factors: one
    pauli_long_range candidate (test_StochasticProcess.jl:75-99)."""
    nm = api.NoiseModel([{"name": "crosstalk_zz", "sites": [1, 3], "strength": 0.1}], 3)
    probs, cands = oracle.probability_distribution(_desc(api.MPS(3, state="ones"), api.init_ising(3, 1, 0.5), nm),
                                                   0.1)
    assert len(probs) == 1 and abs(probs[0] - 1.0) < 1e-14
    assert cands == [("pauli_long_range", [1, 3])]


def test_probability_distribution_order_and_weights(oracle):
    """Several processes: 1-site candidates in site order, then the 2-site
    ones at their first site, then the long-range ones; weights
    dt gamma ||L psi||^2 normalised (StochasticProcess.jl:89-212), checked
    against the dense state."""
    from oracle import dense as D
    L, dt = 4, 0.05
    psi = api.random_mps(L, 3, seed=11)
    T.normalize(psi)
    info = [{"name": "lowering", "sites": [3], "strength": 0.3},
            {"name": "pauli_x", "sites": [1], "strength": 0.2},
            {"name": "crosstalk_xx", "sites": [1, 3], "strength": 0.15},
            {"name": "crosstalk_zx", "sites": [2, 3], "strength": 0.25},
            {"name": "raising", "sites": [2], "strength": 0.1}]
    nm = api.NoiseModel(info, L)
    probs, cands = oracle.probability_distribution(_desc(psi, api.init_ising(L, 1, 0.5), nm), dt)
    v = psi.to_vec()
    # candidate order of the reference
    assert cands == [("local_1", [1]), ("local_1", [2]), ("local_2", [2, 3]), ("local_1", [3]),
                     ("pauli_long_range", [1, 3])]
    # weights of the local candidates from the dense state
    w = []
    for p in (nm.processes[1], nm.processes[4], nm.processes[3], nm.processes[0]):
        op = D.site_op(p.matrix, p.sites[0], L) if len(p.sites) == 1 else D.gate_op(p.matrix, p.sites, L)
        w.append(dt * p.strength * np.linalg.norm(op @ v) ** 2)
    w.append(dt * 0.15 * np.linalg.norm(v) ** 2)  # Pauli long-range: the state norm
    assert np.allclose(probs, np.array(w) / sum(w), atol=1e-13)
    assert abs(probs.sum() - 1.0) < 1e-14


def _product_state(L, seed):
    """A random normalised product state, as test_Dissipation.jl:24-37 builds it."""
    rng = np.random.default_rng(seed)
    psi = api.MPS(L)
    for i in range(L):
        v = rng.normal(size=2) + 1j * rng.normal(size=2)
        psi.tensors[i] = (v / np.linalg.norm(v)).reshape(1, 2, 1)
    return psi


def _right_canonical(A):
    l = A.shape[0]
    M = np.reshape(A, (l, -1), order="F")
    return np.allclose(M @ M.conj().T, np.eye(l), atol=1e-12)


def _dense_dissipation(psi, nm, dt):
    """prod exp(-dt gamma L^dag L / 2) in the reference's order: sites from
    right to left, at each site its 1-site processes, then the 2-site ones
    that end there (Dissipation.jl:37-159)."""
    from scipy.linalg import expm
    from oracle import dense as D
    L = psi.length
    v = psi.to_vec()
    for i in range(L, 0, -1):
        for p in nm.processes:
            if len(p.sites) == 1 and p.sites[0] == i:
                m = np.asarray(p.matrix)
                v = D.site_op(expm(-0.5 * dt * p.strength * m.conj().T @ m), i, L) @ v
        for p in nm.processes:
            if len(p.sites) == 2 and p.sites[1] == i:
                m = np.asarray(p.matrix)
                v = D.gate_op(expm(-0.5 * dt * p.strength * m.conj().T @ m), p.sites, L) @ v
    return v


def _to_vec(tensors):
    st = api.MPS(len(tensors))
    st.tensors = tensors
    return st.to_vec()


@pytest.mark.parametrize("case", ["one_site", "two_site"])
def test_dissipation_leaves_the_centre_at_site_1(oracle, case):
    """test_Dissipation.jl:24-85: lowering + pauli_z on every site, or
    crosstalk_xx + crosstalk_yy on every bond, of a random product state:
    afterwards the recorded centre is site 1 (the reference's
    check_canonical_form returns the recorded centre, MPS.jl:510-512) and
    the state equals the dense product of the dissipators.  The product
    state's recorded centre is site 1, so the first shift moves right and
    the last site, dissipated off-centre, is not re-gauged, in the reference
    as here."""
    L, dt = 3, 0.1
    psi = _product_state(L, 1234 if case == "one_site" else 4321)
    if case == "one_site":
        info = [{"name": n, "sites": [i], "strength": 0.1} for i in range(1, L + 1) for n in ("lowering", "pauli_z")]
    else:
        info = [{"name": n, "sites": [i, i + 1], "strength": 0.1} for i in range(1, L)
                for n in ("crosstalk_xx", "crosstalk_yy")]
    nm = api.NoiseModel(info, L)
    cfg = api.TimeEvolutionConfig([], 0.1, dt=dt, num_traj=1, max_bond_dim=10, truncation_threshold=1e-10)
    out, oc = oracle.apply_dissipation(api.Descriptors(psi, api.init_ising(L, 1, 0.5), cfg, nm))
    assert oc == 1
    assert np.allclose(_to_vec(out), _dense_dissipation(psi, nm, dt), atol=1e-13)


def test_dissipation_non_pauli_two_site_process(oracle):
    """An entangled start (centre at site 1) and a non-Pauli 2-site process
    (merged, the 4x4 dissipator applied, split with the relative rule):
    equal to the dense dissipators, and sites 2..L right-canonical since no
    process acts on the last site."""
    L, dt = 5, 0.2
    psi = api.random_mps(L, 3, seed=21)
    T.normalize(psi)
    proc = api.LocalNoiseProcess("custom_lr", [2, 3], 0.4, np.kron(api.LOWERING, api.LOWERING.T))
    nm = api.NoiseModel([proc, {"name": "lowering", "sites": [4], "strength": 0.3},
                         {"name": "pauli_x", "sites": [2], "strength": 0.2}], L)
    cfg = api.TimeEvolutionConfig([], 0.2, dt=dt, num_traj=1, max_bond_dim=16, truncation_threshold=1e-14)
    out, oc = oracle.apply_dissipation(api.Descriptors(psi, api.init_ising(L, 1, 0.5), cfg, nm))
    assert oc == 1 and all(_right_canonical(A) for A in out[1:])
    assert np.allclose(_to_vec(out), _dense_dissipation(psi, nm, dt), atol=1e-12)


@pytest.mark.parametrize("order", [2, 1])
@pytest.mark.parametrize("sample", [False, True])
def test_analog_tjm_result_shapes(oracle, order, sample):
    """test_AnalogTJM.jl:44-100: identity Hamiltonian on |00000>, T = 0.2,
    dt = 0.1, no noise: one column without sampling, len(0:dt:T) = 3 with
    it, for analog_tjm_2 and analog_tjm_1; <Z_i> stays 1."""
    L = 5
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 0.2, dt=0.1, num_traj=1, max_bond_dim=8, sample_timesteps=sample,
                                  order=order)
    tr, chi, _ = oracle.analog_run(api.Descriptors(api.MPS(L, state="zeros"), T.mpo_identity(L), cfg, None))
    assert tr.shape == (1, L, 3 if sample else 1)
    # the 2-site split keeps at least two Schmidt values (Algorithms.jl:428-438)
    assert np.allclose(tr, 1.0, atol=1e-14) and chi.max() <= 2
