"""Gate library, circuit library and ingestion (src/GateLibrary.jl,
src/CircuitLibrary.jl, src/CircuitIngestion.jl): gate matrices and
generators, gate sequences of the generators, their physics against dense
evolution, and runs of generated circuits on the oracle."""
import math
import types

import numpy as np
import pytest
from scipy.linalg import expm

from yaqs_julia_b200 import api
from yaqs_julia_b200 import circuits as C
from oracle import dense as D

ALL_1Q = [C.IdGate(), C.XGate(), C.YGate(), C.ZGate(), C.HGate(), C.SGate(), C.TGate(), C.SdgGate(), C.TdgGate(),
          C.RxGate(0.3), C.RyGate(-0.7), C.RzGate(1.1), C.PhaseGate(0.4), C.UGate(0.3, 1.2, -0.4)]
ALL_2Q = [C.CXGate(), C.CYGate(), C.CZGate(), C.CHGate(), C.CPhaseGate(0.9), C.SWAPGate(), C.iSWAPGate(),
          C.RxxGate(0.5), C.RyyGate(-1.3), C.RzzGate(2.1)]


def test_gates_are_unitary_and_generators_reproduce_them():
    for g in ALL_1Q + ALL_2Q:
        assert C.is_unitary(g), g.name
        if g.generator is not None:
            U = expm(-1j * g.coeff * np.kron(g.generator[1], g.generator[0]))
            # CX's generator has its control on the first site, its matrix on the second
            want = api.SWAP @ g.matrix @ api.SWAP if g.name == "cx" else g.matrix
            assert np.allclose(U, want, atol=1e-12), g.name
    assert not C.is_unitary(api.LOWERING)


def test_gate_identities():
    assert np.allclose(C.SGate().matrix @ C.SGate().matrix, api.Z)
    assert np.allclose(C.TGate().matrix @ C.TGate().matrix, C.SGate().matrix)
    assert np.allclose(C.UGate(math.pi / 2, 0.0, math.pi).matrix, api.H, atol=1e-15)
    assert np.allclose(C.UGate(0.8, -math.pi / 2, math.pi / 2).matrix, api.Rx(0.8), atol=1e-15)
    # basis index p1 + 2 p2: controlled gates act on site 1 when site 2 is 1
    e = np.eye(4)
    assert np.allclose(C.CYGate().matrix @ e[2], 1j * e[3]) and np.allclose(C.CYGate().matrix @ e[1], e[1])
    assert np.allclose(C.SWAPGate().matrix @ e[1], e[2])
    assert np.allclose(C.iSWAPGate().matrix @ e[1], 1j * e[2])


def _unitary(circ):
    L = circ.num_qubits
    U = np.eye(2 ** L, dtype=np.complex128)
    for g in circ.gates:
        if isinstance(g.op, api.Barrier):
            continue
        U = D.gate_op(g.op, g.sites, L) @ U
    return U


def test_ising_circuit_is_a_first_order_trotterisation():
    L, J, g, T = 4, 1.0, 0.7, 0.4
    exact = expm(-1j * T * api.init_ising(L, J, g).to_matrix())
    errs = []
    for steps in (10, 20, 40):
        circ = C.create_ising_circuit(L, J, g, T / steps, steps)
        errs.append(np.abs(_unitary(circ) - exact).max())
    assert errs[2] < 6e-3 and 1.6 < errs[0] / errs[1] < 2.4 and 1.6 < errs[1] / errs[2] < 2.4
    c = C.create_ising_circuit(5, 1.0, 0.5, 0.1, 2, periodic=True)
    kinds = [type(g.op).__name__ if isinstance(g.op, api.Barrier) else len(g.sites) for g in c.gates]
    assert kinds == ["Barrier"] + ([1] * 5 + [2] * 5 + ["Barrier"]) * 2
    assert [g.sites for g in c.gates[6:11]] == [[1, 2], [3, 4], [2, 3], [4, 5], [1, 5]]


def test_heisenberg_circuit_signs():
    """Rotation angles -2 dt J implement exp(-i dt H') with
    H' = -(Jx XX + Jy YY + Jz ZZ) - h Z."""
    L, T, steps = 4, 0.3, 60
    Hp = api.init_general_hamiltonian(L, -0.8, -1.1, -0.6, 0, 0, -0.4).to_matrix()
    circ = C.create_heisenberg_circuit(L, 0.8, 1.1, 0.6, 0.4, T / steps, steps)
    assert np.abs(_unitary(circ) - expm(-1j * T * Hp)).max() < 5e-3


def test_2d_circuits_follow_the_snake_order():
    assert [C.site_index(r, c, 3) for r in (1, 2) for c in (1, 2, 3)] == [1, 2, 3, 6, 5, 4]
    c = C.create_2d_ising_circuit(2, 3, 1.0, 0.5, 0.1, 1)
    two = [g.sites for g in c.gates if len(g.sites) == 2]
    assert two == [[1, 2], [2, 3], [6, 5], [5, 4], [1, 6], [2, 5], [3, 4]]
    h = C.create_2d_heisenberg_circuit(3, 2, 1.0, 1.0, 1.0, 0.2, 0.1, 1)
    assert sum(1 for g in h.gates if len(g.sites) == 2) == 3 * 7 and all(
        not isinstance(g.op, api.Barrier) for g in h.gates)


def test_fermi_hubbard_1d_conserves_each_spin_number():
    L = 3
    circ = C.create_1d_fermi_hubbard_circuit(L, 1.3, 0.7, 0.4, 2, 0.1, 2)
    U = _unitary(circ)
    n_up = sum((np.eye(2 ** (2 * L)) - D.site_op(api.Z, j, 2 * L)) / 2 for j in range(1, L + 1))
    n_dn = sum((np.eye(2 ** (2 * L)) - D.site_op(api.Z, j, 2 * L)) / 2 for j in range(L + 1, 2 * L + 1))
    assert np.abs(U @ n_up - n_up @ U).max() < 1e-12 and np.abs(U @ n_dn - n_dn @ U).max() < 1e-12
    assert sum(1 for g in circ.gates if len(g.sites) == 2 and abs(g.sites[0] - g.sites[1]) == L) == 2 * 2 * 2 * L


def test_long_range_interaction_gate_sequence():
    c = api.DigitalCircuit(5)
    C.add_long_range_interaction(c, 1, 4, "X", 0.3)
    names = [(type(g.op).__name__ if isinstance(g.op, api.Barrier) else g.sites) for g in c.gates]
    ladder_down = [[3, 4], [2, 4], [1, 4]]
    assert names == ([[4]] + ladder_down + [[1], [4], [1], [4]] + ladder_down + [[4]] + ladder_down[::-1] +
                     [[1], [4]])
    assert np.allclose(c.gates[4].op, api.Ry(math.pi / 2)) and np.allclose(c.gates[-1].op, api.Ry(-math.pi / 2))
    c2 = api.DigitalCircuit(4)
    C.add_hopping_term(c2, 1, 3, 0.2)
    assert len(c2.gates) == 2 * (1 + 2 + 4 + 2 + 1 + 2 + 2)
    with pytest.raises(ValueError):
        C.add_long_range_interaction(c2, 3, 1, "X", 0.1)


def test_random_and_variational_layers():
    a = C.nearest_neighbour_random_circuit(6, 3, seed=5)
    b = C.nearest_neighbour_random_circuit(6, 3, seed=5)
    assert all(np.array_equal(x.op, y.op) for x, y in zip(a.gates, b.gates))
    two = [g.sites for g in a.gates if len(g.sites) == 2]
    assert two == [[2, 3], [4, 5], [1, 2], [3, 4], [5, 6], [2, 3], [4, 5]]
    q = C.qaoa_ising_layer(4, beta=0.3, gamma=0.2)
    assert np.allclose(q.gates[0].op, api.Rx(0.6)) and np.allclose(q.gates[4].op, api.Rzz(0.4))
    h = C.hea_layer(5, phis=[0.1] * 5, thetas=[0.2] * 5, lams=[0.3] * 5, start_parity=1)
    assert len(h.gates) == 15 + 2 and [g.sites for g in h.gates[15:]] == [[2, 3], [4, 5]]
    xy = C.xy_trotter_layer_longrange(4, 0.1)
    assert [g.sites for g in xy.gates[-2:]] == [[4, 1], [4, 1]] and np.allclose(xy.gates[0].op, api.Ryy(0.2))
    lt = C.longrange_test_circuit(5, 0.4)
    assert len(lt.gates) == 6 and lt.gates[-1].sites == [5, 1]
    for make in (C.create_clifford_cz_frame_circuit, C.create_echoed_xx_pi_over_2, C.create_sy_cz_parity_frame):
        assert all(C.is_unitary(g.op) for g in make(4, 2).gates)
    assert len(C.create_cz_brickwork_circuit(5, 2, periodic=True).gates) == 2 * 5
    assert len(C.create_rzz_pi_over_2_brickwork(4, 3).gates) == 9


class _Q:  # a stand-in for a Qiskit qubit
    def __init__(self, i):
        self._index = i


def _fake_qiskit(n, items):
    data = [types.SimpleNamespace(operation=types.SimpleNamespace(name=nm, params=pr, label=None),
                                  qubits=[_Q(q) for q in qs]) for nm, pr, qs in items]
    return types.SimpleNamespace(num_qubits=n, data=data)


def test_ingestion_front_layers():
    items = [("h", [], [0]), ("cx", [], [0, 1]), ("rz", [0.3], [2]), ("barrier", [], [0, 1, 2]),
             ("sx", [], [1]), ("rzz", [0.4], [1, 2]), ("measure", [], [2]), ("u", [0.1, 0.2, 0.3], [0])]
    circ = C.ingest_qiskit_circuit(_fake_qiskit(3, items))
    assert [g.sites for g in circ.gates] == [[1], [3], [1, 2], [2], [1], [2, 3]]
    assert np.allclose(circ.gates[3].op, api.Rx(math.pi / 2)) and all(
        not isinstance(g.op, api.Barrier) for g in circ.gates)
    same = C.ingest_qiskit_circuit((3, items))
    assert all(np.array_equal(x.op, y.op) and x.sites == y.sites for x, y in zip(circ.gates, same.gates))
    with pytest.raises(ValueError, match="Unsupported"):
        C.ingest_qiskit_circuit((2, [("cy", [], [0, 1])]))
    with pytest.raises(ValueError, match=">2"):
        C.ingest_qiskit_circuit((3, [("ccx", [], [0, 1, 2])]))
    op, sites = C.convert_instruction_to_gate("barrier", [], [0, 1])
    assert isinstance(op, api.Barrier) and op.label == "SAMPLE_OBSERVABLES" and sites == [1, 2]
    assert C.convert_instruction_to_gate("cy", [], [0, 1]) is None


@pytest.mark.parametrize("make", [
    lambda: C.create_heisenberg_circuit(6, 1.0, 0.8, 0.6, 0.3, 0.1, 3),
    lambda: C.create_1d_fermi_hubbard_circuit(3, 1.0, 0.6, 0.2, 1, 0.2, 2),
    lambda: C.nearest_neighbour_random_circuit(6, 4, seed=9),
])
def test_generated_circuits_run_on_the_oracle(oracle, make):
    circ = make()
    L = circ.num_qubits
    obs = [api.Observable(f"Z{i}", api.Z, i) for i in range(1, L + 1)]
    cfg = api.TimeEvolutionConfig(obs, 1.0, dt=1.0, num_traj=1, max_bond_dim=64, truncation_threshold=1e-14)
    d = api.CircuitDescriptors(api.MPS(L, state="x+"), circ, cfg, None)
    tr, _, _ = oracle.digital_run(d)
    psi = D.product_state([np.array([1, 1]) / np.sqrt(2)] * L)
    psi = _unitary(circ) @ psi
    ref = [np.real(np.vdot(psi, D.site_op(api.Z, i, L) @ psi)) for i in range(1, L + 1)]
    assert np.abs(tr[0, :, -1] - ref).max() < 1e-9


def test_ingestion_reference_circuit_layers():
    """test_CircuitIngestion.jl:25-88: h(0), cx(0,1), rx(0.5, 2), barrier,
    rzz(0.2, 1, 2) -> layer 1 holds H on 1 and Rx(0.5) on 3, layer 2 CX on
    (1, 2), layer 3 Rzz(0.2) on (2, 3)."""
    items = [("h", [], [0]), ("cx", [], [0, 1]), ("rx", [0.5], [2]), ("barrier", [], [0, 1, 2]),
             ("rzz", [0.2], [1, 2])]
    circ = C.ingest_qiskit_circuit(_fake_qiskit(3, items))
    assert isinstance(circ, api.DigitalCircuit) and circ.num_qubits == 3
    layers, _ = api.process_circuit(circ)
    assert len(layers) >= 2
    l1 = {tuple(g.sites): g.op for g in layers[0]}
    assert set(l1) == {(1,), (3,)}
    assert np.allclose(l1[(1,)], api.H) and np.allclose(l1[(3,)], api.Rx(0.5))
    assert [tuple(g.sites) for g in layers[1]] == [(1, 2)] and np.allclose(layers[1][0].op, api.CX)
    assert [tuple(g.sites) for g in layers[2]] == [(2, 3)] and np.allclose(layers[2][0].op, api.Rzz(0.2))
