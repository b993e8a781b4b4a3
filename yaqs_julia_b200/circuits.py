"""Gate library, circuit library and circuit ingestion: the front-ends that
build DigitalCircuit inputs for the digital engine.

* Gates (src/GateLibrary.jl:44-302): every gate the reference defines, as a
  GateOp carrying its matrix and, where the reference has one, its 2-qubit
  generator pair and coefficient (gate = exp(-i coeff g1 (x) g2)), which the
  TDVP-window method needs.  4x4 matrices use the engine's basis order
  p1 + 2*p2 (first site fastest), as the reference's column-major SMatrix
  literals do; CX, CY and CH therefore have their control on the second
  index (GateLibrary.jl:144-196).
* Circuits (src/CircuitLibrary.jl): Trotter circuits of the 1D/2D Ising and
  Heisenberg models and of 1D/2D Fermi-Hubbard, random nearest-neighbour
  circuits, QAOA and hardware-efficient layers, XY Trotter layers and the
  Clifford/benchmark brickworks, each with the reference's gate order.
* Ingestion (src/CircuitIngestion.jl): Qiskit-style circuits (objects with
  ``num_qubits`` and ``data`` of instructions, or plain
  ``(name, params, qubits)`` tuples) mapped gate by gate with the
  reference's name table and front-layer order.

Sites are 1-based, as in the reference.
"""
from __future__ import annotations

import cmath
import math

import numpy as np

from .api import (CX, CZ, H, I2, X, Y, Z, Barrier, CPhaseGate, CXGate, CZGate, DigitalCircuit, GateOp,  # noqa: F401
                  Rx, Rxx, RxxGate, Ry, Ryy, RyyGate, Rz, Rzz, RzzGate)

# ---------------------------------------------------------------------------
# Gate library (src/GateLibrary.jl)
# ---------------------------------------------------------------------------
_S = np.diag([1, 1j]).astype(np.complex128)
_T = np.diag([1, cmath.exp(1j * math.pi / 4)]).astype(np.complex128)


def IdGate():  # GateLibrary.jl:44-46
    return GateOp(I2, None, 1.0, "id")


def XGate():  # :48-50
    return GateOp(X, None, 1.0, "x")


def YGate():  # :52-54
    return GateOp(Y, None, 1.0, "y")


def ZGate():  # :56-58
    return GateOp(Z, None, 1.0, "z")


def HGate():  # :60-61
    return GateOp(H, None, 1.0, "h")


def SGate():  # :63-64
    return GateOp(_S, None, 1.0, "s")


def TGate():  # :66-67
    return GateOp(_T, None, 1.0, "t")


def SdgGate():  # :69-70
    return GateOp(_S.conj(), None, 1.0, "sdg")


def TdgGate():  # :72-73
    return GateOp(_T.conj(), None, 1.0, "tdg")


def RxGate(theta):  # :88-97, exp(-i theta/2 X)
    return GateOp(Rx(theta), None, theta / 2, "rx")


def RyGate(theta):  # :99-108
    return GateOp(Ry(theta), None, theta / 2, "ry")


def RzGate(theta):  # :110-119
    return GateOp(Rz(theta), None, theta / 2, "rz")


def PhaseGate(theta):  # :121-124, diag(1, e^{i theta})
    return GateOp(np.diag([1, cmath.exp(1j * theta)]).astype(np.complex128), None, 1.0, "p")


def UGate(theta, phi, lam):  # :126-140, the U3 convention
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    m = np.array([[c, -cmath.exp(1j * lam) * s],
                  [cmath.exp(1j * phi) * s, cmath.exp(1j * (phi + lam)) * c]], dtype=np.complex128)
    return GateOp(m, None, 1.0, "u")


def CYGate():  # :161-167, Y on the first index when the second is 1
    m = np.eye(4, dtype=np.complex128)
    m[2:, 2:] = Y
    return GateOp(m, None, 1.0, "cy")


def CHGate():  # :190-196
    m = np.eye(4, dtype=np.complex128)
    m[2:, 2:] = H
    return GateOp(m, None, 1.0, "ch")


def SWAPGate():  # :235-241
    m = np.eye(4, dtype=np.complex128)[[0, 2, 1, 3]]
    return GateOp(m, None, 1.0, "swap")


def iSWAPGate():  # :243-250
    m = np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]], dtype=np.complex128)
    return GateOp(m, None, 1.0, "iswap")


def is_unitary(op) -> bool:
    """GateLibrary.is_unitary (:38-41, 84): every gate, not the lowering operator."""
    m = np.asarray(op, dtype=np.complex128)
    return bool(np.allclose(m.conj().T @ m, np.eye(m.shape[0]), atol=1e-12))


# ---------------------------------------------------------------------------
# Circuit library (src/CircuitLibrary.jl)
# ---------------------------------------------------------------------------
def _sample(circ):
    circ.add_gate(Barrier("SAMPLE_OBSERVABLES"), [])


def _bricks(L):
    """Bonds (i, i+1) in brickwork order: odd i first, then even (1-based)."""
    return [(i, i + 1) for i in range(1, L, 2)] + [(i, i + 1) for i in range(2, L, 2)]


def site_index(row: int, col: int, num_cols: int) -> int:
    """Snake ordering of a 2D grid onto the chain (CircuitLibrary.jl:21-30):
    odd rows left to right, even rows right to left (1-based)."""
    if row % 2 == 1:
        return (row - 1) * num_cols + col
    return (row - 1) * num_cols + (num_cols - col + 1)


def lookup_qiskit_ordering(particle: int, spin: str) -> int:
    """Interleaved Fermi-Hubbard ordering (CircuitLibrary.jl:39-44):
    up_1, down_1, up_2, ... (1-based)."""
    return 2 * (particle - 1) + (1 if spin == "up" else 2)


def add_long_range_interaction(circ, i: int, j: int, outer_op: str, alpha: float):
    """add_long_range_interaction! (CircuitLibrary.jl:52-153): the gate
    sequence the reference emits for exp(-i alpha P_i Z...Z P_j), P = X or Y.
    The reference appends Rz(alpha) on j and a CX ladder (j-1..i onto j) and
    the basis change on i and j before its documented sandwich (basis change,
    ladder down, Rz(alpha), ladder up, inverse basis change); the sequence
    below is that emitted sequence, gate for gate."""
    if i >= j:
        raise ValueError("i must be less than j")
    if outer_op not in ("X", "Y"):
        raise ValueError("outer_op must be X or Y")
    basis = RyGate if outer_op == "X" else RxGate
    half = math.pi / 2
    circ.add_gate(RzGate(alpha), [j])
    for k in range(j - 1, i - 1, -1):
        circ.add_gate(CXGate(), [k, j])
    for _ in range(2):
        circ.add_gate(basis(half), [i])
        circ.add_gate(basis(half), [j])
    for k in range(j - 1, i - 1, -1):
        circ.add_gate(CXGate(), [k, j])
    circ.add_gate(RzGate(alpha), [j])
    for k in range(i, j):
        circ.add_gate(CXGate(), [k, j])
    circ.add_gate(basis(-half), [i])
    circ.add_gate(basis(-half), [j])
    return circ


def add_hopping_term(circ, i: int, j: int, alpha: float):
    """add_hopping_term! (CircuitLibrary.jl:156-159): the X and the Y
    long-range interactions in turn."""
    add_long_range_interaction(circ, i, j, "X", alpha)
    add_long_range_interaction(circ, i, j, "Y", alpha)
    return circ


def create_ising_circuit(L: int, J: float, g: float, dt: float, timesteps: int, periodic: bool = False):
    """First-order Trotter circuit of H = -J sum ZZ - g sum X
    (CircuitLibrary.jl:164-190): per step Rx(-2 dt g) on every site, then
    Rzz(-2 dt J) on the brickwork bonds (and (1, L) if periodic); a sample
    barrier at the start and after every step."""
    circ = DigitalCircuit(L)
    a, b = -2.0 * dt * g, -2.0 * dt * J
    _sample(circ)
    for _ in range(timesteps):
        for s in range(1, L + 1):
            circ.add_gate(RxGate(a), [s])
        for p in _bricks(L):
            circ.add_gate(RzzGate(b), list(p))
        if periodic and L > 1:
            circ.add_gate(RzzGate(b), [1, L])
        _sample(circ)
    return circ


def create_heisenberg_circuit(L: int, Jx: float, Jy: float, Jz: float, h: float, dt: float, timesteps: int,
                              periodic: bool = False):
    """Heisenberg Trotter circuit (CircuitLibrary.jl:192-244): per step Rz on
    every site, then the ZZ, XX and YY brickworks (each closing the ring if
    periodic), angles -2 dt times the couplings; sample barriers as in the
    Ising circuit."""
    circ = DigitalCircuit(L)
    txx, tyy, tzz, tz = (-2.0 * dt * v for v in (Jx, Jy, Jz, h))
    _sample(circ)
    for _ in range(timesteps):
        for s in range(1, L + 1):
            circ.add_gate(RzGate(tz), [s])
        for gate, th in ((RzzGate, tzz), (RxxGate, txx), (RyyGate, tyy)):
            for p in _bricks(L):
                circ.add_gate(gate(th), list(p))
            if periodic and L > 1:
                circ.add_gate(gate(th), [1, L])
        _sample(circ)
    return circ


def _grid_bonds(num_rows, num_cols):
    """Horizontal bonds row by row (odd columns, then even), then vertical
    bonds column by column (odd rows, then even), as chain sites."""
    hor, ver = [], []
    for r in range(1, num_rows + 1):
        for start in (1, 2):
            for c in range(start, num_cols, 2):
                hor.append((site_index(r, c, num_cols), site_index(r, c + 1, num_cols)))
    for c in range(1, num_cols + 1):
        for start in (1, 2):
            for r in range(start, num_rows, 2):
                ver.append((site_index(r, c, num_cols), site_index(r + 1, c, num_cols)))
    return hor, ver


def create_2d_ising_circuit(num_rows: int, num_cols: int, J: float, g: float, dt: float, timesteps: int):
    """2D Ising Trotter circuit on a snake-ordered grid (CircuitLibrary.jl:
    248-299): Rx on every site, then horizontal and vertical Rzz bricks.
    No sample barriers (the reference adds none)."""
    circ = DigitalCircuit(num_rows * num_cols)
    a, b = -2.0 * dt * g, -2.0 * dt * J
    hor, ver = _grid_bonds(num_rows, num_cols)
    for _ in range(timesteps):
        for r in range(1, num_rows + 1):
            for c in range(1, num_cols + 1):
                circ.add_gate(RxGate(a), [site_index(r, c, num_cols)])
        for p in hor + ver:
            circ.add_gate(RzzGate(b), list(p))
    return circ


def create_2d_heisenberg_circuit(num_rows: int, num_cols: int, Jx: float, Jy: float, Jz: float, h: float,
                                 dt: float, timesteps: int):
    """2D Heisenberg Trotter circuit (CircuitLibrary.jl:304-363): Rz on every
    site, then for ZZ, XX, YY in turn: horizontal odd, horizontal even,
    vertical odd, vertical even bonds."""
    n = num_rows * num_cols
    circ = DigitalCircuit(n)
    txx, tyy, tzz, tz = (-2.0 * dt * v for v in (Jx, Jy, Jz, h))
    hor_odd, hor_even, ver_odd, ver_even = [], [], [], []
    for r in range(1, num_rows + 1):
        for c in range(1, num_cols, 2):
            hor_odd.append((site_index(r, c, num_cols), site_index(r, c + 1, num_cols)))
    for r in range(1, num_rows + 1):
        for c in range(2, num_cols, 2):
            hor_even.append((site_index(r, c, num_cols), site_index(r, c + 1, num_cols)))
    for c in range(1, num_cols + 1):
        for r in range(1, num_rows, 2):
            ver_odd.append((site_index(r, c, num_cols), site_index(r + 1, c, num_cols)))
    for c in range(1, num_cols + 1):
        for r in range(2, num_rows, 2):
            ver_even.append((site_index(r, c, num_cols), site_index(r + 1, c, num_cols)))
    for _ in range(timesteps):
        for q in range(1, n + 1):
            circ.add_gate(RzGate(tz), [q])
        for gate, th in ((RzzGate, tzz), (RxxGate, txx), (RyyGate, tyy)):
            for p in hor_odd + hor_even + ver_odd + ver_even:
                circ.add_gate(gate(th), list(p))
    return circ


def create_1d_fermi_hubbard_circuit(L: int, u: float, t: float, mu: float, num_trotter_steps: int, dt: float,
                                    timesteps: int):
    """1D Fermi-Hubbard (CircuitLibrary.jl:367-425) on 2L qubits, spin up on
    1..L and spin down on L+1..2L.  Per Trotter slice: phases mu dt/(2n),
    on-site CPhase(-u dt/(2n)) between j and j+L, hopping Rxx then Ryy
    (-t dt/n) on the odd then even bonds of each spin (sites given as
    [j+1, j]), on-site again, phases again; n * timesteps slices."""
    circ = DigitalCircuit(2 * L)
    n = num_trotter_steps

    def chem():
        th = mu * dt / (2 * n)
        for j in range(1, L + 1):
            circ.add_gate(PhaseGate(th), [j])
            circ.add_gate(PhaseGate(th), [j + L])

    def onsite():
        th = -u * dt / (2 * n)
        for j in range(1, L + 1):
            circ.add_gate(CPhaseGate(th), [j, j + L])

    def hop():
        th = -dt * t / n
        for start in (1, 2):
            for j in range(start, L, 2):
                circ.add_gate(RxxGate(th), [j + 1, j])
                circ.add_gate(RyyGate(th), [j + 1, j])
                circ.add_gate(RxxGate(th), [j + 1 + L, j + L])
                circ.add_gate(RyyGate(th), [j + 1 + L, j + L])

    for _ in range(n * timesteps):
        chem()
        onsite()
        hop()
        onsite()
        chem()
    return circ


def create_2d_fermi_hubbard_circuit(Lx: int, Ly: int, u: float, t: float, mu: float, num_trotter_steps: int,
                                    dt: float, timesteps: int):
    """2D Fermi-Hubbard on an Lx x Ly lattice, interleaved spin ordering
    (CircuitLibrary.jl:429-517).  Per slice: phases -mu dt/(2n), on-site
    CPhase(-u dt/(2n)), hopping exp(-i alpha (XX + YY)) with alpha = t dt/n
    through add_hopping_term on horizontal odd, horizontal even, vertical odd,
    vertical even pairs (up then down), on-site, phases."""
    ns = Lx * Ly
    circ = DigitalCircuit(2 * ns)
    n = num_trotter_steps
    up = lambda p: lookup_qiskit_ordering(p, "up")  # noqa: E731
    dn = lambda p: lookup_qiskit_ordering(p, "down")  # noqa: E731

    def chem():
        th = -mu * dt / (2 * n)
        for j in range(1, ns + 1):
            circ.add_gate(PhaseGate(th), [up(j)])
            circ.add_gate(PhaseGate(th), [dn(j)])

    def onsite():
        th = -u * dt / (2 * n)
        for j in range(1, ns + 1):
            circ.add_gate(CPhaseGate(th), [up(j), dn(j)])

    def hop():
        alpha = t * dt / n
        pairs = []
        for start in (1, 2):
            for y in range(1, Ly + 1):
                for x in range(start, Lx, 2):
                    p1 = (y - 1) * Lx + x
                    pairs.append((p1, p1 + 1))
        for start in (1, 2):
            for y in range(start, Ly, 2):
                for x in range(1, Lx + 1):
                    p1 = (y - 1) * Lx + x
                    pairs.append((p1, p1 + Lx))
        for p1, p2 in pairs:
            add_hopping_term(circ, up(p1), up(p2), alpha)
            add_hopping_term(circ, dn(p1), dn(p2), alpha)

    for _ in range(timesteps):
        for _ in range(n):
            chem()
            onsite()
            hop()
            onsite()
            chem()
    return circ


def nearest_neighbour_random_circuit(n_qubits: int, layers: int, seed: int = 42, rng=None):
    """Random brickwork (CircuitLibrary.jl:522-597): per layer a U(theta in
    [0, pi), phi, lam in [0, 2 pi)) on every qubit, then CZ or CX (each with
    probability 1/2) on the bonds starting at site 2 in odd layers and at
    site 1 in even layers.  The draws come from numpy's generator seeded
    with ``seed`` (the reference draws from Julia's global generator)."""
    rng = np.random.default_rng(seed) if rng is None else rng
    circ = DigitalCircuit(n_qubits)
    for layer in range(1, layers + 1):
        for q in range(1, n_qubits + 1):
            th, ph, la = rng.random() * math.pi, rng.random() * 2 * math.pi, rng.random() * 2 * math.pi
            circ.add_gate(UGate(th, ph, la), [q])
        start = 2 if layer % 2 == 1 else 1
        for i in range(start, n_qubits, 2):
            circ.add_gate(CZGate() if rng.random() < 0.5 else CXGate(), [i, i + 1])
    return circ


def qaoa_ising_layer(n_qubits: int, beta: float | None = None, gamma: float | None = None, rng=None):
    """One QAOA layer for a 1D Ising cost (CircuitLibrary.jl:601-634):
    Rx(2 beta) on every qubit, then Rzz(2 gamma) brickwork; missing angles are
    drawn uniformly from [0, 2 pi)."""
    rng = np.random.default_rng() if rng is None else rng
    b = rng.random() * 2 * math.pi if beta is None else beta
    g = rng.random() * 2 * math.pi if gamma is None else gamma
    circ = DigitalCircuit(n_qubits)
    for q in range(1, n_qubits + 1):
        circ.add_gate(RxGate(2 * b), [q])
    for p in _bricks(n_qubits):
        circ.add_gate(RzzGate(2 * g), list(p))
    return circ


def hea_layer(n_qubits: int, phis=None, thetas=None, lams=None, start_parity: int | None = None, rng=None):
    """One hardware-efficient layer (CircuitLibrary.jl:641-693): Rz(phi),
    Ry(theta), Rz(lam) on every qubit, then CZ on the bonds starting at site
    1 + start_parity; missing parameters are drawn (phi, lam in [0, 2 pi),
    theta in [0, pi), parity 0 or 1)."""
    rng = np.random.default_rng() if rng is None else rng
    ps = [rng.random() * 2 * math.pi for _ in range(n_qubits)] if phis is None else list(phis)
    ts = [rng.random() * math.pi for _ in range(n_qubits)] if thetas is None else list(thetas)
    ls = [rng.random() * 2 * math.pi for _ in range(n_qubits)] if lams is None else list(lams)
    sp = int(rng.integers(0, 2)) if start_parity is None else int(start_parity)
    circ = DigitalCircuit(n_qubits)
    for q in range(1, n_qubits + 1):
        circ.add_gate(RzGate(ps[q - 1]), [q])
        circ.add_gate(RyGate(ts[q - 1]), [q])
        circ.add_gate(RzGate(ls[q - 1]), [q])
    for i in range(sp + 1, n_qubits, 2):
        circ.add_gate(CZGate(), [i, i + 1])
    return circ


def xy_trotter_layer(N: int, tau: float, order: str = "YX"):
    """XY Trotter layer (CircuitLibrary.jl:697-720): Ryy(2 tau) then
    Rxx(2 tau) brickworks for order "YX", the other way round otherwise."""
    circ = DigitalCircuit(N)
    seq = (RyyGate, RxxGate) if order == "YX" else (RxxGate, RyyGate)
    for gate in seq:
        for p in _bricks(N):
            circ.add_gate(gate(2 * tau), list(p))
    return circ


def xy_trotter_layer_longrange(N: int, tau: float, order: str = "YX"):
    """xy_trotter_layer plus the boundary pair (N, 1) in the same order
    (CircuitLibrary.jl:724-740)."""
    circ = xy_trotter_layer(N, tau, order)
    seq = (RyyGate, RxxGate) if order == "YX" else (RxxGate, RyyGate)
    for gate in seq:
        circ.add_gate(gate(2 * tau), [N, 1])
    return circ


def longrange_test_circuit(N: int, theta: float):
    """H on every qubit, then one Rzz(theta) on (N, 1) (CircuitLibrary.jl:756-770)."""
    circ = DigitalCircuit(N)
    for q in range(1, N + 1):
        circ.add_gate(HGate(), [q])
    circ.add_gate(RzzGate(theta), [N, 1])
    return circ


def create_clifford_cz_frame_circuit(L: int, timesteps: int):
    """Per step: H on every qubit, CZ brickwork (CircuitLibrary.jl:774-791)."""
    circ = DigitalCircuit(L)
    for _ in range(timesteps):
        for q in range(1, L + 1):
            circ.add_gate(HGate(), [q])
        for p in _bricks(L):
            circ.add_gate(CZGate(), list(p))
    return circ


def create_echoed_xx_pi_over_2(L: int, timesteps: int):
    """Per step: H, Rxx(pi/2) brickwork, H (CircuitLibrary.jl:795-810)."""
    circ = DigitalCircuit(L)
    for _ in range(timesteps):
        for q in range(1, L + 1):
            circ.add_gate(HGate(), [q])
        for p in _bricks(L):
            circ.add_gate(RxxGate(math.pi / 2), list(p))
        for q in range(1, L + 1):
            circ.add_gate(HGate(), [q])
    return circ


def create_sy_cz_parity_frame(L: int, timesteps: int):
    """Per step: H then Sdg on every qubit, CZ brickwork (CircuitLibrary.jl:814-827)."""
    circ = DigitalCircuit(L)
    for _ in range(timesteps):
        for q in range(1, L + 1):
            circ.add_gate(HGate(), [q])
            circ.add_gate(SdgGate(), [q])
        for p in _bricks(L):
            circ.add_gate(CZGate(), list(p))
    return circ


def create_cz_brickwork_circuit(L: int, timesteps: int, periodic: bool = False):
    """CZ brickwork, ring-closing CZ on (L, 1) if periodic (CircuitLibrary.jl:831-842)."""
    circ = DigitalCircuit(L)
    for _ in range(timesteps):
        for p in _bricks(L):
            circ.add_gate(CZGate(), list(p))
        if periodic and L > 1:
            circ.add_gate(CZGate(), [L, 1])
    return circ


def create_rzz_pi_over_2_brickwork(L: int, timesteps: int, periodic: bool = False):
    """Rzz(pi/2) brickwork, ring-closing on (L, 1) if periodic (CircuitLibrary.jl:846-857)."""
    circ = DigitalCircuit(L)
    for _ in range(timesteps):
        for p in _bricks(L):
            circ.add_gate(RzzGate(math.pi / 2), list(p))
        if periodic and L > 1:
            circ.add_gate(RzzGate(math.pi / 2), [L, 1])
    return circ


# ---------------------------------------------------------------------------
# Circuit ingestion (src/CircuitIngestion.jl)
# ---------------------------------------------------------------------------
def map_qiskit_name(name: str, params):
    """map_qiskit_name (CircuitIngestion.jl:262-310): the reference's
    gate-name table; "sx" becomes Rx(pi/2).  Other names raise ValueError."""
    p = [float(v) for v in params]
    table = {
        "x": XGate, "y": YGate, "z": ZGate, "h": HGate, "id": IdGate, "s": SGate, "t": TGate,
        "cx": CXGate, "cz": CZGate, "swap": SWAPGate,
    }
    if name in table:
        return table[name]()
    if name == "sx":
        return RxGate(math.pi / 2)
    if name in ("rx", "ry", "rz", "rxx", "ryy", "rzz"):
        return {"rx": RxGate, "ry": RyGate, "rz": RzGate, "rxx": RxxGate, "ryy": RyyGate, "rzz": RzzGate}[name](p[0])
    if name in ("p", "phase"):
        return PhaseGate(p[0])
    if name in ("u", "u3"):
        return UGate(p[0], p[1], p[2])
    raise ValueError(f"Unsupported Qiskit gate: {name}")


def _instructions(qc):
    """(name, params, 0-based qubits) of a Qiskit-style circuit: an object
    with ``num_qubits`` and ``data`` (CircuitInstruction-like items with
    ``operation.name``, ``operation.params`` and ``qubits``), or a
    (num_qubits, [(name, params, qubits), ...]) pair."""
    if isinstance(qc, tuple) and len(qc) == 2:
        n, items = qc
        return int(n), [(str(nm), list(pr), [int(q) for q in qs]) for nm, pr, qs in items]
    out = []
    for ins in qc.data:
        op = ins.operation
        qs = []
        for q in ins.qubits:
            qs.append(int(q._index) if getattr(q, "_index", None) is not None else int(qc.find_bit(q).index))
        out.append((str(op.name), [float(v) for v in op.params], qs))
    return int(qc.num_qubits), out


def ingest_qiskit_circuit(qc) -> DigitalCircuit:
    """ingest_qiskit_circuit (CircuitIngestion.jl:15-124): the circuit's
    dependency front layers in turn; in each, measurements and barriers are
    dropped (the reference removes them without adding a gate), then the
    1-qubit gates and then the 2-qubit gates are appended, in circuit order
    within the layer.  Gates on more than two qubits raise ValueError."""
    n, items = _instructions(qc)
    circ = DigitalCircuit(n)
    pending = list(range(len(items)))
    while pending:
        busy = set()
        front = []
        for idx in pending:
            qs = items[idx][2] or list(range(n))
            if not any(q in busy for q in qs):
                front.append(idx)
            busy.update(qs)
        singles, pairs = [], []
        for idx in front:
            name, params, qs = items[idx]
            if name in ("measure", "barrier"):
                continue
            if len(qs) == 1:
                singles.append(idx)
            elif len(qs) == 2:
                pairs.append(idx)
            else:
                raise ValueError("Gates with >2 qubits not supported")
        for idx in singles + pairs:
            name, params, qs = items[idx]
            circ.add_gate(map_qiskit_name(name, params), [q + 1 for q in qs])
        done = set(front)
        pending = [i for i in pending if i not in done]
    return circ


def convert_instruction_to_gate(name: str, params, qubits, label: str | None = None):
    """convert_instruction_to_gate (CircuitIngestion.jl:132-187) for one
    instruction: (op, 1-based sites).  A barrier becomes Barrier(label)
    ("SAMPLE_OBSERVABLES" when unlabelled); unsupported names give None."""
    sites = [int(q) + 1 for q in qubits]
    if name == "barrier":
        return Barrier(label or "SAMPLE_OBSERVABLES"), sites
    try:
        return map_qiskit_name(name, params), sites
    except ValueError:
        return None
