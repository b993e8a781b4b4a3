"""Long-range noise processes (MPONoiseProcess, src/Noise.jl:22-33,71-131,
155-290,355-400; jumps src/StochasticProcess.jl:46-82,169-202,304-313;
dissipation src/Dissipation.jl:161-204) in the host model and the oracle.

The oracle applies the operator as the reference does: as an MPO to a copy
of the state, then MPS.truncate! (which renormalises), so the candidate
weight of a non-null operator is dt*gamma whatever its norm; a standard
long-range Pauli process ("pauli_long_range") is chosen with weight
dt*gamma*||psi||^2 but never applied.  These tests pin both behaviours."""
import math

import numpy as np
import pytest

from yaqs_julia_b200 import _abi as A
from yaqs_julia_b200 import api
from oracle import dense as D


def test_long_range_projector_known_answer():
    """test_Noise.jl:75-93: crosstalk_xy on [1, 3] -> two MPO processes."""
    m = api.NoiseModel([{"name": "crosstalk_xy", "sites": [1, 3], "strength": 0.05, "unraveling": "projector"}], 4)
    assert len(m.processes) == 2
    p1, p2 = m.processes
    assert isinstance(p1, api.MPONoiseProcess) and p1.sites == [1, 3]
    assert p1.mpo.length == 4 and len(p1.mpo.tensors) == 4
    assert [t.shape for t in p1.mpo.tensors] == [(1, 2, 2, 2), (2, 2, 2, 2), (2, 2, 2, 1), (1, 2, 2, 1)]
    # sigma (the name's first letter) on site 1, tau on site 3 (Noise.jl:162-171)
    xy = D.site_op(api.X, 1, 4) @ D.site_op(api.Y, 3, 4)
    assert np.allclose(p1.mpo.to_matrix(), np.eye(16) + xy, atol=1e-14)
    assert np.allclose(p2.mpo.to_matrix(), np.eye(16) - xy, atol=1e-14)
    assert p1.strength == p2.strength == 0.025 and not p1.factors


@pytest.mark.parametrize("unravel", ["standard", "unitary_2pt", "unitary_gauss"])
def test_long_range_operators(unravel):
    L = 5
    m = api.NoiseModel([{"name": "crosstalk_zx", "sites": [4, 2], "strength": 0.2, "unraveling": unravel,
                         "theta0": 0.9}], L)
    zx = D.site_op(api.Z, 2, L) @ D.site_op(api.X, 4, L)
    eye = np.eye(2 ** L)
    for p in m.processes:
        assert p.sites == [2, 4]
        Op = p.mpo.to_matrix()
        if unravel == "standard":
            assert np.allclose(Op, zx, atol=1e-14) and len(p.factors) == 2
        else:
            # cos(theta) 1 + i sin(theta) P is the unitary exp(i theta P)
            assert np.allclose(Op.conj().T @ Op, eye, atol=1e-13)
    # each expansion keeps the dissipator gamma D[P]
    rng = np.random.default_rng(3)
    a = rng.normal(size=(32, 32)) + 1j * rng.normal(size=(32, 32))
    rho = a @ a.conj().T
    rho /= np.trace(rho)

    def diss(ops):
        out = np.zeros_like(rho)
        for g, Lk in ops:
            out += g * (Lk @ rho @ Lk.conj().T - 0.5 * (Lk.conj().T @ Lk @ rho + rho @ Lk.conj().T @ Lk))
        return out

    ref = diss([(0.2, zx)])
    assert np.allclose(diss([(p.strength, p.mpo.to_matrix()) for p in m.processes]), ref, atol=1e-13)


def test_dissipation_rates_and_candidate_kinds():
    m = api.NoiseModel([{"name": "crosstalk_xx", "sites": [1, 4], "strength": 0.3, "unraveling": "projector"},
                        {"name": "crosstalk_yy", "sites": [2, 5], "strength": 0.1},
                        {"name": "pauli_z", "sites": [3], "strength": 0.2},
                        {"name": "crosstalk_zz", "sites": [1, 3], "strength": 0.4, "unraveling": "unitary_2pt"}], 5)
    f = api.long_range_flags(m.processes)
    assert f[0] == (0.3, False) and f[1] == (0.0, False)  # the pair shares one decay
    assert f[2] == (0.1, True)  # standard crosstalk: pauli_long_range
    assert f[4] == (0.2, False) and f[5] == (0.2, False)  # unitary components: their own rates
    bad = api.NoiseModel([api.MPONoiseProcess("custom", [1, 3], 0.1, api.X, api.X, 0, 1, 4, factors=(api.X, api.X))])
    with pytest.raises(NotImplementedError, match="Non-Pauli long-range"):
        api.long_range_flags(bad.processes)


def _tilted(L, thetas):
    return api.MPS(L, tensors=[np.array([math.cos(t / 2), math.sin(t / 2)], dtype=np.complex128).reshape(1, 2, 1)
                               for t in thetas])


def _one_gate(oracle, psi, nm, u, L, obs):
    c = api.DigitalCircuit(L)
    c.add_gate(api.Rzz(0.0), [1, 3])
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=1.0, num_traj=1, max_bond_dim=16)
    d = api.CircuitDescriptors(psi, c, cfg, nm, rng_mode=A.YAQS_RNG_INJECTED, uniforms=np.array([u]))
    return oracle.digital_run(d)


def test_projector_candidates_are_equally_weighted(oracle):
    """The reference weighs an MPO candidate by the norm of its renormalised
    copy, so 1 + ZZ and 1 - ZZ are equally likely whatever <ZZ> is; a null
    branch keeps a negligible weight."""
    L = 4
    th = 0.7
    nm = api.NoiseModel([{"name": "crosstalk_zz", "sites": [1, 3], "strength": 0.5, "unraveling": "projector"}], L)
    obs = [api.Observable("Z1", api.Z, 1)]
    c2, s2 = math.cos(th / 2) ** 2, math.sin(th / 2) ** 2
    plus = (c2 ** 2 - s2 ** 2) / (c2 ** 2 + s2 ** 2)
    for u2, want in ((0.49, plus), (0.51, 0.0)):
        tr, _, st = _one_gate(oracle, _tilted(L, [th, 0, th, 0]), nm, [0.0, u2], L, obs)
        assert st["jumps"] == 1 and abs(tr[0, 0, -1] - want) < 1e-12, (u2, tr[0, 0, -1], want)
    # |0000>: 1 - ZZ annihilates the state, so the plus branch is taken for any u2
    tr, _, st = _one_gate(oracle, api.MPS(L), nm, [0.0, 0.99], L, obs)
    assert st["jumps"] == 1 and abs(tr[0, 0, -1] - 1.0) < 1e-12


def test_standard_long_range_pauli_is_never_applied(oracle):
    """The "pauli_long_range" candidate has no branch in the reference's
    jump application: the state is only renormalised."""
    L = 4
    nm = api.NoiseModel([{"name": "crosstalk_xx", "sites": [1, 3], "strength": 0.5}], L)
    obs = [api.Observable("Z1", api.Z, 1), api.Observable("Z3", api.Z, 3)]
    tr, _, st = _one_gate(oracle, api.MPS(L), nm, [0.0, 0.5], L, obs)
    assert st["jumps"] == 1 and np.allclose(tr[0, :, -1], [1.0, 1.0], atol=1e-12)


@pytest.mark.parametrize("unravel", ["unitary_2pt", "unitary_gauss"])
def test_long_range_unitary_unravelings_match_lindblad(oracle, unravel):
    """Only unitary MPO candidates: every weight is dt*gamma, as exact
    dynamics wants, so the ensemble follows the Lindblad equation of the
    standard operator (3 standard errors)."""
    L = 5
    H = api.init_ising(L, 1.0, 0.6)
    info = [{"name": "crosstalk_zz", "sites": [1, 4], "strength": 0.2, "unraveling": unravel, "theta0": math.pi / 3},
            {"name": "crosstalk_xy", "sites": [2, 5], "strength": 0.15, "unraveling": unravel,
             "theta0": math.pi / 3}]
    nm = api.NoiseModel(info, L)
    jumps = [np.sqrt(0.2) * D.site_op(api.Z, 1, L) @ D.site_op(api.Z, 4, L),
             np.sqrt(0.15) * D.site_op(api.X, 2, L) @ D.site_op(api.Y, 5, L)]
    Xs = [D.site_op(api.X, s, L) for s in range(1, L + 1)]
    plus = np.array([1, 1]) / np.sqrt(2)
    ex = D.lindblad(H.to_matrix(), D.product_state([plus] * L), jumps, 0.05, 20, Xs, substeps=10)
    obs = [api.Observable(f"X{s}", api.X, s) for s in range(1, L + 1)]
    nt = 500
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=0.05, num_traj=nt, max_bond_dim=16)
    traj, _, st = oracle.analog_run(api.Descriptors(api.MPS(L, state="x+"), H, cfg, nm, seed=31))
    mean = traj.mean(0).T
    # early samples see few jumps (an observable can have no spread at all),
    # so the standard error is floored at the size of one jump's effect
    se = np.maximum(traj.std(0, ddof=1).T / np.sqrt(nt), 1.5 / nt)
    z = np.abs(mean - ex)[1:] / se[1:]
    assert st["jumps"] > 50
    assert (z > 3).mean() < 0.05 and z.max() < 5, z.max()


def _digital_density(L, layers, procs, observables):
    """Exact average of the digital step with unitary jump operators given
    as full 2^L matrices (processes on the gate's pair or sites)."""
    psi = D.product_state([[1, 0]] * L)
    rho = np.outer(psi, psi.conj())
    out = [[np.trace(O @ rho).real for O in observables]]
    for layer in layers:
        for g in layer:
            if len(g.sites) == 1:
                U = D.gate_op(g.op, g.sites, L)
                rho = U @ rho @ U.conj().T
        for g in layer:
            if len(g.sites) != 2:
                continue
            U = D.gate_op(g.op, g.sites, L)
            rho = U @ rho @ U.conj().T
            sset = set(g.sites)
            loc = [(P, gm) for P, st, gm in procs
                   if (len(st) == 1 and st[0] in sset) or (len(st) == 2 and set(st) == sset)]
            G = sum(gm for _, gm in loc)
            if G > 0:
                jumped = sum((gm / G) * (P @ rho @ P.conj().T) for P, gm in loc)
                rho = np.exp(-G) * rho + (1 - np.exp(-G)) * jumped
        out.append([np.trace(O @ rho).real for O in observables])
    return np.array(out)


def test_digital_long_range_gate_noise_matches_exact_channel(oracle):
    """Long-range gates pick up the unitary_2pt crosstalk processes on their
    own pair (DigitalTJM.jl:172-188, 405-420); with unitary operators the
    unravelled step averages to the channel e^{-G} rho + (1 - e^{-G}) sum_k
    g_k/G U_k rho U_k^dag."""
    from test_oracle_digital import _brickwork, _run, _zs
    L = 5
    c = _brickwork(L, 3, seed=12)  # carries Rxx on (1, L) and CX on (L-1, 2)
    info = [{"name": "crosstalk_zz", "sites": [1, L], "strength": 0.06, "unraveling": "unitary_2pt",
             "theta0": math.pi / 3},
            {"name": "crosstalk_xx", "sites": [2, L - 1], "strength": 0.05, "unraveling": "unitary_2pt",
             "theta0": math.pi / 3},
            {"name": "pauli_x", "sites": [3], "strength": 0.04}]
    nm = api.NoiseModel(info, L)
    procs = [(p.mpo.to_matrix() if isinstance(p, api.MPONoiseProcess) else D.gate_op(p.matrix, p.sites, L),
              p.sites, p.strength) for p in nm.processes]
    nt = 3000
    tr, _, st = _run(oracle, L, c, _zs(L), nm=nm, num_traj=nt, seed=77)
    layers, _ = api.process_circuit(c)
    _, after, _ = api.sample_plan(c)
    ref = _digital_density(L, layers, procs, [D.site_op(api.Z, i, L) for i in range(1, L + 1)])[[0] + after]
    mean = tr.mean(0).T
    se = np.maximum(tr.std(0, ddof=1).T / np.sqrt(nt), 1.5 / nt)
    z = np.abs(mean - ref)[1:] / se[1:]
    assert st["jumps"] > 100
    assert (z > 3).mean() < 0.05 and z.max() < 5, z.max()
