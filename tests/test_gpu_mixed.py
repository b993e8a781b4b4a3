"""Mixed-precision analog form (H_eff and environment contractions in complex
FP32 on the tensor cores, 3xTF32) against the FP64 oracle: on the same
injected draws every trajectory's <Z_i> stays within 1e-5 absolute, the
half-chain entropy within 1e-4, and the ensemble means within the same
bounds.  The FP64 engine run beside it is held to 1e-10."""
import numpy as np
import pytest

from yaqs_julia_b200 import _abi as A
from yaqs_julia_b200 import api

pytestmark = pytest.mark.gpu

Z_TOL = 1e-5


def _run(psi, H, cfg, nm, u, precision):
    d = api.Descriptors(psi, H, cfg, nm, rng_mode=A.YAQS_RNG_INJECTED, uniforms=u, precision=precision)
    return d, api.run_descriptors(d)


def test_mixed_ising_cfg1_like(oracle):
    L = 6
    H = api.init_ising(L, 1.0, 0.5)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 2.0, dt=0.1, num_traj=8, max_bond_dim=16, truncation_threshold=1e-10)
    nm = api.NoiseModel([{"name": "lowering", "sites": [i], "strength": 0.1} for i in range(1, L + 1)] +
                        [{"name": "pauli_z", "sites": [i], "strength": 0.1} for i in range(1, L + 1)], L)
    u = np.random.default_rng(5).random((8, api.max_draws(cfg)))
    d, mixed = _run(api.MPS(L), H, cfg, nm, u, A.YAQS_PREC_MIXED)
    ref, _, st = oracle.analog_run(d)
    err = np.abs(mixed.trajectories - ref)
    assert err.max() < Z_TOL, err.max()
    assert mixed.stats["jumps"] == st["jumps"]


def test_mixed_heisenberg_entropy(oracle):
    L = 12
    H = api.init_general_hamiltonian(L, 1, 1, 1, 0, 0, 0.3)
    obs = ([api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)] +
           [api.Observable("S_half", None, L // 2, kind="entropy")])
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=0.05, num_traj=6, max_bond_dim=32)
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [i], "strength": 0.05} for i in range(1, L + 1)], L)
    u = np.random.default_rng(6).random((6, api.max_draws(cfg)))
    d, mixed = _run(api.MPS(L, state="Neel"), H, cfg, nm, u, A.YAQS_PREC_MIXED)
    ref, _, _ = oracle.analog_run(d)
    ez = np.abs(mixed.trajectories[:, :L] - ref[:, :L]).max()
    es = np.abs(mixed.trajectories[:, L] - ref[:, L]).max()
    assert ez < Z_TOL and es < 1e-4, (ez, es)
    d64, fp64 = _run(api.MPS(L, state="Neel"), H, cfg, nm, u, A.YAQS_PREC_FP64)
    assert np.abs(fp64.trajectories - ref).max() < 1e-10
    # the mixed form is not the FP64 form under another name
    assert np.abs(mixed.trajectories - fp64.trajectories).max() > 1e-13


def test_mixed_saturated_chi32_start(oracle):
    """A start with every bulk bond saturated exercises full-size tiles."""
    L = 10
    H = api.init_general_hamiltonian(L, 1, 1, 1, 0, 0, 0.3)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 0.2, dt=0.05, num_traj=3, max_bond_dim=32)
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [i], "strength": 0.05} for i in range(1, L + 1)], L)
    u = np.random.default_rng(7).random((3, api.max_draws(cfg)))
    d, mixed = _run(api.random_mps(L, 32, seed=3), H, cfg, nm, u, A.YAQS_PREC_MIXED)
    ref, _, _ = oracle.analog_run(d)
    assert np.abs(mixed.trajectories - ref).max() < Z_TOL


def test_run_api_precision_flag():
    L = 6
    H = api.init_ising(L, 1.0, 0.5)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 0.5, dt=0.1)
    res = api.run(api.MPS(L), H, cfg, None, precision="mixed")
    cfg64 = api.TimeEvolutionConfig([api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)], 0.5, dt=0.1)
    res64 = api.run(api.MPS(L), H, cfg64, None)
    assert np.abs(res.trajectories - res64.trajectories).max() < Z_TOL


def test_digital_rejects_mixed():
    c = api.DigitalCircuit(2).add_gate(api.H, [1])
    cfg = api.TimeEvolutionConfig([api.Observable("Z1", api.Z, 1)], 1.0, dt=1.0, num_traj=1)
    d = api.CircuitDescriptors(api.MPS(2), c, cfg, None)
    d.cfg.precision = A.YAQS_PREC_MIXED
    from yaqs_julia_b200._lib import EngineError
    with pytest.raises(EngineError, match="UNSUPPORTED"):
        api.run_circuit_descriptors(d)


def test_autotuner_measures_the_shapes_of_a_mixed_run(oracle):
    """A direct mixed run first times both product forms on every H_eff
    shape it will meet (yaqs_autotune_results); the run, with the chosen
    forms, still matches the FP64 oracle within the mixed tolerance."""
    import ctypes as C
    from yaqs_julia_b200 import _lib
    L = 8
    H = api.init_general_hamiltonian(L, 1, 1, 1, 0, 0, 0.3)
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 0.2, dt=0.05, num_traj=4, max_bond_dim=16)
    nm = api.NoiseModel([{"name": "pauli_z", "sites": [i], "strength": 0.05} for i in range(1, L + 1)], L)
    u = np.random.default_rng(9).random((4, api.max_draws(cfg)))
    d, mixed = _run(api.MPS(L, state="Neel"), H, cfg, nm, u, A.YAQS_PREC_MIXED)
    ref, _, _ = oracle.analog_run(d)
    assert np.abs(mixed.trajectories - ref).max() < Z_TOL
    ctx = _lib.default_context()
    n = C.c_int32(0)
    ctx.check(ctx._lib.yaqs_autotune_results(ctx.handle, None, 0, C.byref(n)))
    rows = np.zeros((max(n.value, 1), 8))
    ctx.check(ctx._lib.yaqs_autotune_results(ctx.handle, A.dptr(rows), n.value, C.byref(n)))
    rows = rows[:n.value]
    shapes = {(int(r[0]), int(r[1]), int(r[2])) for r in rows}
    # bond caps 1 2 4 8 16 8 4 2 1: the centre bond, the sites beside it and a 2-site window over them
    assert {(16, 1, 16), (8, 2, 16), (16, 2, 8), (8, 4, 8)} <= shapes, sorted(shapes)
    assert set(rows[:, 5]) <= {0.0, 1.0} and (rows[:, 6] > 0).all() and (rows[:, 7] > 0).all()
