"""Known-answer tests of the oracle's building blocks."""
import ctypes as C

import numpy as np
import pytest

from yaqs_julia_b200 import _abi as A
from yaqs_julia_b200 import api


def _rand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("m,n", [(1, 1), (2, 7), (7, 2), (16, 16), (33, 12), (12, 33), (128, 64)])
def test_svd_reconstructs_and_is_orthonormal(oracle, m, n):
    rng = np.random.default_rng(m * 100 + n)
    M = _rand(rng, m, n)
    U, S, SVt = oracle.svd(M)
    assert np.allclose(U @ SVt, M, atol=1e-12 * np.abs(M).max() * max(m, n))
    k = min(m, n)
    assert np.allclose(U.conj().T @ U, np.eye(k), atol=1e-13 * max(m, n))
    assert np.allclose(SVt @ SVt.conj().T, np.diag(S ** 2), atol=1e-12 * max(m, n) * np.abs(M).max() ** 2)
    assert np.all(np.diff(S) <= 0)
    assert np.allclose(S, np.linalg.svd(M, compute_uv=False), rtol=1e-12, atol=1e-13)


def test_svd_rank_deficient_null_vectors_are_orthonormal(oracle):
    rng = np.random.default_rng(5)
    M = _rand(rng, 8, 2) @ _rand(rng, 2, 8)  # rank 2
    U, S, SVt = oracle.svd(M)
    assert np.all(S[2:] == 0.0)
    assert np.allclose(U.conj().T @ U, np.eye(8), atol=1e-13)
    assert np.all(SVt[2:] == 0.0)
    assert np.allclose(U @ SVt, M, atol=1e-12)


@pytest.mark.parametrize("m,n", [(4, 2), (2, 4), (128, 64), (64, 128), (3, 3)])
def test_qr(oracle, m, n):
    rng = np.random.default_rng(m + 7 * n)
    M = _rand(rng, m, n)
    Q, R = oracle.qr(M)
    assert np.allclose(Q @ R, M, atol=1e-12 * max(m, n))
    assert np.allclose(Q.conj().T @ Q, np.eye(min(m, n)), atol=1e-13 * max(m, n))
    assert np.allclose(np.tril(R, -1), 0)
    assert np.allclose(np.diag(R).imag, 0)


def test_truncation_rank_rules(oracle):
    # test_truncation_comparison.jl:72-128 cases, against the implementation
    # rule MPS.jl:406-414 / Algorithms.jl:428-438.
    S = 10.0 ** -np.arange(1, 21)
    for thr in (1e-40, 1e-20, 1e-12, 1e-8, 1e-4, 1e-2):
        disc, keep = 0.0, len(S)
        for k in range(len(S), 0, -1):
            disc += S[k - 1] ** 2
            if disc >= thr:
                keep = max(k, 2)
                break
        assert oracle.truncation_rank(S, thr, 4096, 0) == keep
    assert oracle.truncation_rank(S, 1e-12, 3, 0) == 3
    # relative rule (Dissipation.jl:290-303): keep while tail > thr * |S|^2
    assert oracle.truncation_rank(np.array([1.0, 1e-6]), 1e-9, 64, 1) == 1
    assert oracle.truncation_rank(np.array([1.0, 1e-6]), 1e-11, 64, 1) == 1
    assert oracle.truncation_rank(np.array([1.0, 1e-6]), 1e-13, 64, 1) == 2
    assert oracle.truncation_rank(np.array([1.0, 1e-6]), 1e-13, 1, 1) == 1


def _ident_env(chi, w):
    E = np.zeros((chi, w, chi), dtype=np.complex128)
    for i in range(chi):
        E[i, 0, i] = 1
    return E


@pytest.mark.parametrize("op,v,dt", [(api.Z, [1, 0], 0.3), (api.X, [1, 0], 0.7), (api.Z, [0.6, 0.8j], -0.2)])
def test_krylov_expm_2x2(oracle, op, v, dt):
    # test_Algorithms.jl:17-35: exp(-i dt A) v for Pauli A, atol 1e-10.
    import scipy.linalg as sl
    W = np.asarray(op).reshape(1, 2, 2, 1)
    x = np.asarray(v, dtype=np.complex128).reshape(1, 2, 1)
    out, _ = oracle.expm_site(_ident_env(1, 1), _ident_env(1, 1), W, x, dt)
    assert np.allclose(out.reshape(2), sl.expm(-1j * dt * op) @ np.asarray(v), atol=1e-10)


def test_krylov_expm_matches_dense_on_random_heff(oracle):
    import scipy.linalg as sl
    rng = np.random.default_rng(3)
    chil, chir, wl, wr, D = 6, 5, 3, 3, 4
    Lh = _rand(rng, chil, wl, chil)
    Rh = _rand(rng, chir, wr, chir)
    W = _rand(rng, wl, D, D, wr)
    # make H_eff Hermitian: L[a,m,k] = conj(L[k,m,a]), R likewise, W[m,po,pi,mr] = conj(W[m,pi,po,mr])
    Lh = Lh + Lh.transpose(2, 1, 0).conj()
    Rh = Rh + Rh.transpose(2, 1, 0).conj()
    W = W + W.transpose(0, 2, 1, 3).conj()
    n = chil * D * chir
    Hm = np.zeros((n, n), dtype=np.complex128)
    for j in range(n):
        e = np.zeros(n, dtype=np.complex128)
        e[j] = 1
        Hm[:, j] = oracle.project_site(Lh, Rh, W, e.reshape(chil, D, chir, order="F")).reshape(-1, order="F")
    assert np.allclose(Hm, Hm.conj().T, atol=1e-10)
    x = _rand(rng, chil, D, chir)
    dt = 0.01
    for exit_tol in (0.0, 1e-12):
        out, mv = oracle.expm_site(Lh, Rh, W, x, dt, exit_tol=exit_tol)
        ref = sl.expm(-1j * dt * Hm) @ x.reshape(-1, order="F")
        assert np.abs(out.reshape(-1, order="F") - ref).max() < 1e-10 * np.abs(ref).max()
        assert mv <= 25


def test_mpo_energies(oracle):
    # test_MPO.jl:26-53: <000|H|000> = -2 and <+++|H|+++> = -1.5 for init_ising(3, 1, 0.5).
    Hm = api.init_ising(3, 1.0, 0.5).to_matrix()
    z = np.zeros(8)
    z[0] = 1
    plus = np.ones(8) / np.sqrt(8)
    assert np.isclose(z @ Hm @ z, -2.0)
    assert np.isclose(plus @ Hm @ plus, -1.5)
    Hh = api.init_general_hamiltonian(4, 1, 1, 1, 0, 0, 0.3).to_matrix()
    assert np.allclose(Hh, Hh.conj().T)


def test_philox_known_answers(oracle):
    # Random123 kat_vectors for philox4x32_10.
    f = oracle.lib().orc_philox4x32_10
    cases = [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
             ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
             ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
              [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]
    for ctr, key, want in cases:
        c, k, o = (C.c_uint32 * 4)(*ctr), (C.c_uint32 * 2)(*key), (C.c_uint32 * 4)()
        f(c, k, o)
        assert list(o) == want
    u = [oracle.philox_uniform(7, 3, i) for i in range(1000)]
    assert 0.0 <= min(u) and max(u) < 1.0 and abs(np.mean(u) - 0.5) < 0.05


def test_injected_draws_reproduce_and_exhaustion_errors(oracle):
    L = 4
    H = api.init_ising(L, 1.0, 0.5)
    obs = [api.Observable("Z1", api.Z, 1)]
    cfg = api.TimeEvolutionConfig(obs, 0.5, dt=0.1, num_traj=3, max_bond_dim=8)
    nm = api.NoiseModel([{"name": "lowering", "sites": [i], "strength": 0.3} for i in range(1, L + 1)], L)
    u = np.random.default_rng(0).random((3, api.max_draws(cfg)))
    a, _, _ = oracle.analog_run(api.Descriptors(api.MPS(L, state="x+"), H, cfg, nm, rng_mode=1, uniforms=u))
    b, _, _ = oracle.analog_run(api.Descriptors(api.MPS(L, state="x+"), H, cfg, nm, rng_mode=1, uniforms=u))
    assert np.array_equal(a, b)
    with pytest.raises(RuntimeError, match="YAQS_E_RNG"):
        oracle.analog_run(api.Descriptors(api.MPS(L, state="x+"), H, cfg, nm, rng_mode=1, uniforms=u[:, :2]))


def test_blas_backed_restatement_equals_the_loops(oracle):
    """The timed CPU baseline routes the contractions through OpenBLAS zgemm;
    its trajectories equal the plain-loop restatement's to rounding."""
    L = 8
    H = api.init_general_hamiltonian(L, 1, 1, 1, 0, 0, 0.3)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 0.2, dt=0.05, num_traj=2, max_bond_dim=8)
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [i], "strength": 0.05} for i in range(1, L + 1)], L)
    res = {}
    for tdvp in (A.YAQS_TDVP_2SITE, A.YAQS_TDVP_DYNAMIC):
        d = api.Descriptors(api.random_mps(L, 8, seed=2), H, cfg, nm, seed=3, tdvp_mode=tdvp)
        try:
            oracle.set_blas(False)
            ref, _, _ = oracle.analog_run(d, nthreads=2)
            desc = oracle.set_blas(True)
            got, _, _ = oracle.analog_run(d, nthreads=2)
        finally:
            oracle.set_blas(False)
        res[tdvp] = (np.abs(got - ref).max(), desc)
    for err, desc in res.values():
        assert "OpenBLAS" in desc, desc
        assert err < 1e-10, err


def test_dynamic_truncation_is_rounding_sensitive(oracle):
    """Why the dynamic sweep's parity bar is 1e-5 where a 2-site split
    truncates (tests/test_gpu_parity.py): the oracle against itself with
    another summation order (OpenBLAS zgemm instead of loops) on the same
    draws.  L = 10 Heisenberg from Neel: with chi_max = 32 (never binding) the
    two runs agree to rounding; with chi_max = 16 the middle split truncates
    32 values to 16 and the runs separate by orders of magnitude more."""
    L = 10
    H = api.init_general_hamiltonian(L, 1, 1, 1, 0, 0, 0.3)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [i], "strength": 0.05} for i in range(1, L + 1)], L)
    out = {}
    for chi in (32, 16):
        cfg = api.TimeEvolutionConfig(obs, 0.8, dt=0.05, num_traj=3, max_bond_dim=chi)
        u = np.random.default_rng(22).random((3, api.max_draws(cfg)))
        d = api.Descriptors(api.MPS(L, state="Neel"), H, cfg, nm, rng_mode=A.YAQS_RNG_INJECTED, uniforms=u,
                            tdvp_mode=A.YAQS_TDVP_DYNAMIC)
        try:
            oracle.set_blas(False)
            a, _, _ = oracle.analog_run(d, nthreads=3)
            oracle.set_blas(True)
            b, _, _ = oracle.analog_run(d, nthreads=3)
        finally:
            oracle.set_blas(False)
        out[chi] = np.abs(a - b).max()
    assert out[32] < 1e-12, out
    assert out[16] > 1e-9, out
