"""Host-side mirror of the Yaqs.jl API for the analog TJM path.

Names, argument meaning and defaults follow the reference so code written
against Yaqs.jl reads the same here:

* ``MPS(length; state=...)``            — src/MPS.jl:52-144
* ``init_ising``, ``init_general_hamiltonian`` — src/MPO.jl:92-260
* ``NoiseModel(processes, num_qubits)`` — src/Noise.jl:299-420 (standard
  unraveling of local processes)
* ``Observable``, ``TimeEvolutionConfig`` — src/SimulationConfigs.jl:23-92
* ``run(initial_state, H, sim_params, noise_model)`` — src/Simulator.jl:127-141

Sites are 1-based, as in Julia.  Tensors are numpy arrays in the
reference's index order, (left, phys, right) for MPS and
(left, phys_out, phys_in, right) for MPO, stored column-major
(Fortran order) so their buffers are exactly what a Julia caller passes
through the C-ABI.

``run`` executes on the GPU through ``libyaqs_b200.so``; there is no CPU
path.  If the library or a CUDA device is missing it raises.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import _abi as A

# ---------------------------------------------------------------------------
# Gate library (src/GateLibrary.jl).  Matrices as in the reference; 4x4
# operators use the basis index p1 + 2*p2 (first site fastest).
# ---------------------------------------------------------------------------
I2 = np.eye(2, dtype=np.complex128)
X = np.array([[0, 1], [1, 0]], dtype=np.complex128)
Y = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
Z = np.array([[1, 0], [0, -1]], dtype=np.complex128)
H = np.array([[1, 1], [1, -1]], dtype=np.complex128) / math.sqrt(2)
RAISING = np.array([[0, 0], [1, 0]], dtype=np.complex128)   # GateLibrary.jl:77-78
LOWERING = np.array([[0, 1], [0, 0]], dtype=np.complex128)  # GateLibrary.jl:80-81


def Rx(theta):
    c, s = math.cos(theta / 2), -1j * math.sin(theta / 2)
    return np.array([[c, s], [s, c]], dtype=np.complex128)


def Rz(theta):
    return np.diag([np.exp(-0.5j * theta), np.exp(0.5j * theta)]).astype(np.complex128)


def Rzz(theta):
    em, ep = np.exp(-0.5j * theta), np.exp(0.5j * theta)
    return np.diag([em, ep, ep, em]).astype(np.complex128)


SWAP = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=np.complex128)
# CX as GateLibrary.jl:144-150 writes it (control on the second site under the
# p1 + 2 p2 basis convention)
CX = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=np.complex128)
CZ = np.diag([1, 1, 1, -1]).astype(np.complex128)


def Ry(theta):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    return np.array([[c, -s], [s, c]], dtype=np.complex128)


def Rxx(theta):
    c, s = math.cos(theta / 2), -1j * math.sin(theta / 2)
    return np.array([[c, 0, 0, s], [0, c, s, 0], [0, s, c, 0], [s, 0, 0, c]], dtype=np.complex128)


def Ryy(theta):
    c, s = math.cos(theta / 2), -1j * math.sin(theta / 2)
    return np.array([[c, 0, 0, -s], [0, c, s, 0], [0, s, c, 0], [-s, 0, 0, c]], dtype=np.complex128)


def CPhase(theta):
    return np.diag([1, 1, 1, np.exp(1j * theta)]).astype(np.complex128)


class GateOp:
    """A gate as GateLibrary defines it: its matrix and, for the 2-qubit
    gates TDVP can apply, the generator pair and coefficient with
    gate = exp(-i coeff g1 (x) g2), g1 on the gate's first site
    (generator / hamiltonian_coeff, GateLibrary.jl:24-36).  Usable wherever a
    matrix is (np.asarray gives the matrix)."""

    def __init__(self, matrix, generator=None, coeff=1.0, name=""):
        self.matrix = np.asarray(matrix, dtype=np.complex128)
        self.generator = None if generator is None else tuple(np.asarray(g, dtype=np.complex128) for g in generator)
        self.coeff = float(coeff)
        self.name = name

    def __array__(self, dtype=None, copy=None):
        return self.matrix if dtype is None else self.matrix.astype(dtype)


_I_MINUS_Z = np.array([[0, 0], [0, 2]], dtype=np.complex128)
_I_MINUS_X = np.array([[1, -1], [-1, 1]], dtype=np.complex128)


def RxxGate(theta):  # GateLibrary.jl:258-272
    return GateOp(Rxx(theta), (X, X), theta / 2, "rxx")


def RyyGate(theta):  # GateLibrary.jl:274-288
    return GateOp(Ryy(theta), (Y, Y), theta / 2, "ryy")


def RzzGate(theta):  # GateLibrary.jl:290-302
    return GateOp(Rzz(theta), (Z, Z), theta / 2, "rzz")


def CXGate():  # GateLibrary.jl:142-157
    return GateOp(CX, (_I_MINUS_Z, _I_MINUS_X), math.pi / 4, "cx")


def CZGate():  # GateLibrary.jl:167-187
    return GateOp(CZ, (_I_MINUS_Z, _I_MINUS_Z), math.pi / 4, "cz")


def CPhaseGate(theta):  # GateLibrary.jl:197-233
    return GateOp(CPhase(theta), (_I_MINUS_Z, _I_MINUS_Z), -theta / 4, "cphase")


def kron2(a, b):
    """Julia's kron(a, b) reshaped to the (p1_out, p2_out, p1_in, p2_in)
    convention: kron(A, B) acts with B on the FIRST site (Noise.jl:47-57)."""
    return np.kron(a, b)


GATES = {"x": X, "y": Y, "z": Z, "h": H, "id": I2, "raising": RAISING, "lowering": LOWERING}


def _pauli(c):
    return {"x": X, "y": Y, "z": Z}[c]


def get_operator(name: str) -> np.ndarray:
    """Noise.get_operator (src/Noise.jl:41-61)."""
    if name == "pauli_x":
        return X.copy()
    if name == "pauli_y":
        return Y.copy()
    if name == "pauli_z":
        return Z.copy()
    if name == "raising":
        return RAISING.copy()
    if name == "lowering":
        return LOWERING.copy()
    if name == "raising_two":
        return np.kron(RAISING, RAISING)
    if name == "lowering_two":
        return np.kron(LOWERING, LOWERING)
    if name.startswith("crosstalk_") and len(name) == 12:
        return np.kron(_pauli(name[10]), _pauli(name[11]))
    raise ValueError(f"Unknown operator: {name}")


_PAULI_NAMES = {"pauli_x", "pauli_y", "pauli_z", "crosstalk_xx", "crosstalk_yy", "crosstalk_zz",
                "crosstalk_xy", "crosstalk_yx", "crosstalk_zy", "crosstalk_zx", "crosstalk_yz",
                "crosstalk_xz"}


def is_pauli_name(name: str) -> bool:
    """DissipationModule.is_pauli (src/Dissipation.jl:14-21)."""
    return name in _PAULI_NAMES


def is_pauli_matrix(op: np.ndarray) -> bool:
    """StochasticProcessModule.is_pauli (src/StochasticProcess.jl:336-341)."""
    d = op.shape[0]
    return bool(np.allclose(op.conj().T @ op, np.eye(d), rtol=0.0, atol=1e-10))


def is_pauli_proc(name: str, op: np.ndarray) -> bool:
    """StochasticProcessModule.is_pauli_proc (src/StochasticProcess.jl:343-357)."""
    if ("pauli" in name or "crosstalk" in name) and "projector" not in name:
        return True
    return is_pauli_matrix(op)


# ---------------------------------------------------------------------------
# MPS (src/MPS.jl)
# ---------------------------------------------------------------------------
class MPS:
    """Matrix product state; tensors are (left, phys, right) arrays."""

    def __init__(self, length: int, tensors=None, physical_dimensions=None, state: str = "zeros",
                 basis_string: str | None = None, pad: int | None = None, seed: int | None = None):
        """MPS(length; tensors, physical_dimensions, state, pad, basis_string)
        (MPS.jl:52-144).  state "random" draws complex Gaussian tensors with
        interior bonds 4 and normalises them (MPS.jl:92-103; ``seed`` seeds
        the draws, which the reference takes from the global RNG); ``pad``
        grows every bond to that dimension afterwards (pad_bond_dimension!)."""
        self.length = int(length)
        if physical_dimensions not in (None, 2) and not (
                isinstance(physical_dimensions, (list, tuple)) and set(physical_dimensions) == {2}):
            raise NotImplementedError("only qubits (d = 2) are served")
        self.phys_dims = [2] * self.length
        self.orth_center = 1
        if tensors is not None:
            assert len(tensors) == self.length
            self.tensors = [np.asfortranarray(np.asarray(t, dtype=np.complex128)) for t in tensors]
            return
        if state == "random":
            rng = np.random.default_rng(seed)
            ts = []
            for i in range(1, self.length + 1):
                l = 1 if i == 1 else 4
                r = 1 if i == self.length else 4
                z = (rng.standard_normal((l, 2, r)) + 1j * rng.standard_normal((l, 2, r))) / math.sqrt(2)
                ts.append(np.asfortranarray(z))
            self.tensors = ts
            from .tensornet import normalize
            normalize(self)
            if pad is not None:
                self.pad_bond_dimension(pad, seed=seed or 0)
            return
        ts = []
        for i in range(1, self.length + 1):  # MPS.jl:105-134
            v = np.zeros(2, dtype=np.complex128)
            if state == "basis":
                assert basis_string is not None and len(basis_string) == self.length
                v[int(basis_string[i - 1])] = 1.0
            elif state == "zeros":
                v[0] = 1.0
            elif state == "ones":
                v[1] = 1.0
            elif state == "x+":
                v[:] = [1 / math.sqrt(2), 1 / math.sqrt(2)]
            elif state == "x-":
                v[:] = [1 / math.sqrt(2), -1 / math.sqrt(2)]
            elif state == "y+":
                v[:] = [1 / math.sqrt(2), 1j / math.sqrt(2)]
            elif state == "y-":
                v[:] = [1 / math.sqrt(2), -1j / math.sqrt(2)]
            elif state == "Neel":
                v[0 if i % 2 != 0 else 1] = 1.0
            elif state == "wall":
                v[0 if i <= self.length // 2 else 1] = 1.0
            else:
                raise ValueError(f"Unknown state: {state}")
            ts.append(np.asfortranarray(v.reshape(1, 2, 1)))
        self.tensors = ts
        if pad is not None:
            self.pad_bond_dimension(pad, seed=seed or 0)

    @property
    def bond_dims(self):
        return [1] + [t.shape[2] for t in self.tensors]

    def pad_bond_dimension(self, target_dim: int, noise_scale: float = 1e-8, seed: int = 0):
        """pad_bond_dimension! (MPS.jl:453-494): normalize!, then grow every
        bond below target_dim to target_dim, filling the new slices with
        complex noise of amplitude noise_scale (seeded here; the reference
        draws from the global RNG), then normalize! again."""
        from .tensornet import normalize
        if target_dim <= 0:
            raise ValueError("target_dim must be positive")
        normalize(self)
        rng = np.random.default_rng(seed)
        for i in range(self.length - 1):
            A, B = self.tensors[i], self.tensors[i + 1]
            r = A.shape[2]
            if r >= target_dim:
                continue
            nA = np.zeros((A.shape[0], A.shape[1], target_dim), dtype=np.complex128)
            nA[:, :, :r] = A
            nA[:, :, r:] = noise_scale * (rng.standard_normal((A.shape[0], A.shape[1], target_dim - r)) +
                                          1j * rng.standard_normal((A.shape[0], A.shape[1], target_dim - r)))
            nB = np.zeros((target_dim, B.shape[1], B.shape[2]), dtype=np.complex128)
            nB[:r] = B
            nB[r:] = noise_scale * (rng.standard_normal((target_dim - r, B.shape[1], B.shape[2])) +
                                    1j * rng.standard_normal((target_dim - r, B.shape[1], B.shape[2])))
            self.tensors[i] = np.asfortranarray(nA)
            self.tensors[i + 1] = np.asfortranarray(nB)
        normalize(self)
        return self

    def to_vec(self) -> np.ndarray:
        """MPS.to_vec (src/MPS.jl:766-775): site 1 is the fastest index."""
        v = self.tensors[0]
        for t in self.tensors[1:]:
            l, p, _ = v.shape
            v = np.einsum("lpk,kqr->lpqr", v, t).reshape(l, p * t.shape[1], t.shape[2], order="F")
        return v.reshape(-1, order="F")


# ---------------------------------------------------------------------------
# MPO (src/MPO.jl)
# ---------------------------------------------------------------------------
class MPO:
    """Matrix product operator; tensors are (left, out, in, right) arrays."""

    def __init__(self, length: int, tensors):
        self.length = int(length)
        self.tensors = [np.asfortranarray(np.asarray(t, dtype=np.complex128)) for t in tensors]
        self.phys_dims = [2] * self.length
        self.orth_center = 0  # unknown until orthogonalize! (MPO.jl:44)

    @property
    def bond_dims(self):
        return [1] + [t.shape[3] for t in self.tensors]

    def __add__(self, other: "MPO") -> "MPO":
        """a + b (MPO.jl:486-521): the block-diagonal sum."""
        from .tensornet import mpo_add
        return mpo_add(self, other)

    def __mul__(self, c) -> "MPO":
        """mpo * c = c * mpo (MPO.jl:523-529): the first tensor scaled."""
        import numbers
        if not isinstance(c, numbers.Number):
            return NotImplemented
        from .tensornet import mpo_scale
        return mpo_scale(c, self)

    __rmul__ = __mul__

    def to_matrix(self) -> np.ndarray:
        """Dense operator in the to_vec basis (site 1 fastest); tests only."""
        W = self.tensors[0][0]  # (out, in, r)
        op = W
        for t in self.tensors[1:]:
            # op[(o1..), (i1..), k] * t[k, o, i, r]
            do, di, _ = op.shape
            op = np.einsum("abk,kcdr->acbdr", op, t).reshape(do * 2, di * 2, t.shape[3], order="F")
        return op[:, :, 0]


def _block_to_tensor(blocks):
    rows, cols = len(blocks), len(blocks[0])
    T = np.zeros((rows, 2, 2, cols), dtype=np.complex128, order="F")
    for r in range(rows):
        for c in range(cols):
            T[r, :, :, c] = blocks[r][c]
    return T


def _param(p, i):  # 1-based site i; vectors shorter than L give 0 (MPO.jl:102,186)
    if isinstance(p, (list, tuple, np.ndarray)):
        return float(p[i - 1]) if i <= len(p) else 0.0
    return float(p)


def init_ising(length: int, J, g) -> MPO:
    """H = -sum J Z_i Z_{i+1} - sum g X_i (src/MPO.jl:92-163), bond width 3."""
    Zr = np.zeros((2, 2), dtype=np.complex128)
    L = int(length)
    if L == 1:
        return MPO(1, [(-_param(g, 1) * X).reshape(1, 2, 2, 1)])
    ts = [_block_to_tensor([[I2, -_param(J, 1) * Z, -_param(g, 1) * X]])]
    for i in range(2, L):
        W = [[Zr] * 3 for _ in range(3)]
        W[0][0] = I2
        W[0][1] = -_param(J, i) * Z
        W[0][2] = -_param(g, i) * X
        W[1][2] = Z
        W[2][2] = I2
        ts.append(_block_to_tensor(W))
    ts.append(_block_to_tensor([[-_param(g, L) * X], [Z], [I2]]))
    return MPO(L, ts)


def init_general_hamiltonian(length: int, Jxx, Jyy, Jzz, hx, hy, hz) -> MPO:
    """H = sum(Jxx XX + Jyy YY + Jzz ZZ) + sum(hx X + hy Y + hz Z)
    (src/MPO.jl:175-260), bond width 5, signs as written (positive)."""
    Zr = np.zeros((2, 2), dtype=np.complex128)
    L = int(length)
    ts = []
    for i in range(1, L + 1):
        jxx = _param(Jxx, i) if i < L else 0.0
        jyy = _param(Jyy, i) if i < L else 0.0
        jzz = _param(Jzz, i) if i < L else 0.0
        loc = _param(hx, i) * X + _param(hy, i) * Y + _param(hz, i) * Z
        W = [[Zr] * 5 for _ in range(5)]
        W[0][0] = I2
        W[0][1] = jxx * X
        W[0][2] = jyy * Y
        W[0][3] = jzz * Z
        W[0][4] = loc
        W[1][4] = X
        W[2][4] = Y
        W[3][4] = Z
        W[4][4] = I2
        if i == 1:
            ts.append(loc.reshape(1, 2, 2, 1) if L == 1 else _block_to_tensor([W[0]]))
        elif i == L:
            ts.append(_block_to_tensor([[W[r][4]] for r in range(5)]))
        else:
            ts.append(_block_to_tensor(W))
    return MPO(L, ts)


# ---------------------------------------------------------------------------
# Noise (src/Noise.jl)
# ---------------------------------------------------------------------------
class LocalNoiseProcess:
    def __init__(self, name, sites, strength, matrix):
        self.name = name
        self.sites = list(sites)
        self.strength = float(strength)
        self.matrix = np.asarray(matrix, dtype=np.complex128)


class MPONoiseProcess:
    """MPONoiseProcess(name, sites, strength, mpo, factors) (src/Noise.jl:22-33):
    a process on two sites i < j that are not neighbours.  Its operator is
    O = a*1 + b*(sigma at i)(tau at j), the MPO of build_mpo_phys
    (Noise.jl:71-131), which ``mpo`` builds.  ``factors`` is (sigma, tau)
    for the standard unraveling and empty for the expansions, as in the
    reference."""

    def __init__(self, name, sites, strength, sigma, tau, a, b, num_qubits, factors=()):
        self.name = name
        self.sites = sorted(int(x) for x in sites)
        self.strength = float(strength)
        self.sigma = np.asarray(sigma, dtype=np.complex128)
        self.tau = np.asarray(tau, dtype=np.complex128)
        self.a = complex(a)
        self.b = complex(b)
        self.num_qubits = int(num_qubits)
        self.factors = [np.asarray(f, dtype=np.complex128) for f in factors]

    @property
    def mpo(self) -> "MPO":
        return build_mpo_phys(self.num_qubits, self.sites[0], self.sites[1], self.sigma, self.tau, self.a, self.b)


def build_mpo_phys(L: int, i: int, j: int, sigma, tau, a, b) -> "MPO":
    """MPO of O = a*1 + b*(sigma_i tau_j), 1 <= i < j <= L (Noise.jl:71-131):
    identity (1x1) outside [i, j], the row [1, sigma] at i, diag(1, 1)
    between, the column [a 1; b tau] at j.  Tensors (left, out, in, right)."""
    if not 1 <= i < j <= L:
        raise ValueError("Require 1 <= i < j <= L")
    tens = []
    for k in range(1, L + 1):
        if k < i or k > j:
            T = np.zeros((1, 2, 2, 1), dtype=np.complex128)
            T[0, :, :, 0] = I2
        elif k == i:
            T = np.zeros((1, 2, 2, 2), dtype=np.complex128)
            T[0, :, :, 0] = I2
            T[0, :, :, 1] = sigma
        elif k < j:
            T = np.zeros((2, 2, 2, 2), dtype=np.complex128)
            T[0, :, :, 0] = I2
            T[1, :, :, 1] = I2
        else:
            T = np.zeros((2, 2, 2, 1), dtype=np.complex128)
            T[0, :, :, 0] = a * I2
            T[1, :, :, 0] = b * np.asarray(tau)
        tens.append(T)
    return MPO(L, tens)


def _lr_factors(p: dict):
    """(sigma, tau) of a long-range process: the "factors" key, else the two
    Pauli letters that end the name, as in "crosstalk_xy" (Noise.jl:162-171)."""
    if "factors" in p:
        sig, tau = p["factors"]
        return np.asarray(sig, dtype=np.complex128), np.asarray(tau, dtype=np.complex128)
    suffix = p["name"].split("_")[-1]
    if len(suffix) != 2 or any(ch not in "xyz" for ch in suffix):
        raise ValueError(f"Unknown Pauli pair in {p['name']!r}")
    return _pauli(suffix[0]), _pauli(suffix[1])


def _expm(a: np.ndarray) -> np.ndarray:
    from scipy.linalg import expm
    return expm(np.asarray(a, dtype=np.complex128))


def _proc_operator(p: dict) -> np.ndarray:
    """Noise.get_operator_from_proc (src/Noise.jl:422-433): the "matrix" key
    wins, else the operator named by "name"."""
    if "matrix" in p:
        return np.asarray(p["matrix"], dtype=np.complex128)
    return get_operator(p["name"])


def _projector_expansion(p, sites, P, gamma):
    """add_projector_expansion! (src/Noise.jl:134-154): jump operators I +- P
    at rate gamma/2 each, named projector_plus_<name> / projector_minus_<name>."""
    eye = np.eye(P.shape[0], dtype=np.complex128)
    return [LocalNoiseProcess(f"projector_{comp}_{p['name']}", sites, gamma / 2.0, eye + sgn * P)
            for comp, sgn in (("plus", 1.0), ("minus", -1.0))]


def _unitary_2pt_expansion(p, sites, P, gamma, theta0):
    """add_unitary_2pt_expansion! (src/Noise.jl:184-197): U = exp(+-i theta0 P)
    at rate (gamma / sin^2 theta0) / 2 each, named unitary2pt_plus/minus_<name>."""
    s_val = math.sin(theta0) ** 2
    if not s_val > 0:
        raise ValueError("theta0 too small")
    lam = gamma / s_val
    return [LocalNoiseProcess(f"unitary2pt_{comp}_{p['name']}", sites, lam / 2.0, _expm(1j * sgn * theta0 * P))
            for comp, sgn in (("plus", 1.0), ("minus", -1.0))]


def gauss_angles(sigma: float, M: int, theta_max: float):
    """The angle grid and weights of add_unitary_gauss_expansion!
    (src/Noise.jl:225-240): (M+1)//2 equispaced angles on [0, theta_max]
    mirrored to negative angles, Gaussian weights exp(-theta^2 / 2 sigma^2)
    normalised to sum 1 and symmetrised."""
    n_pos = (M + 1) // 2
    if n_pos == 1 and theta_max != 0.0:
        raise ValueError("range(0, theta_max, length=1) needs theta_max == 0")
    pos = np.linspace(0.0, theta_max, n_pos)
    thetas = np.concatenate([-pos[1:][::-1], pos])
    w = np.exp(-0.5 * (thetas / sigma) ** 2)
    w = w / w.sum()
    w = 0.5 * (w + w[::-1])
    return thetas, w


def _unitary_gauss_expansion(p, sites, P, gamma, sigma, M, k):
    """add_unitary_gauss_expansion! (src/Noise.jl:225-252): one unitary
    U = exp(i theta_k P) per grid angle at rate lambda * w_k with
    lambda = gamma / sum_k w_k sin^2 theta_k, named unitary_gauss_<k>_<name>
    (k from 0).  Per-process "M" and "theta_max" override the grid."""
    M = int(p.get("M", M))
    theta_max = float(p.get("theta_max", k * sigma))
    thetas, w = gauss_angles(sigma, M, theta_max)
    s_weight = float(np.sum(w * np.sin(thetas) ** 2))
    if not s_weight > 1e-12:
        raise ValueError("E[sin^2 theta] too small")
    lam = gamma / s_weight
    return [LocalNoiseProcess(f"unitary_gauss_{idx}_{p['name']}", sites, lam * wk, _expm(1j * th * P))
            for idx, (wk, th) in enumerate(zip(w, thetas)) if wk > 0.0]


UNRAVELINGS = ("standard", "projector", "unitary_2pt", "unitary_gauss", "analog_auto")


def _long_range_processes(p, sites, gamma, unravel, L, theta0, dt, sigma, gauss_M, gauss_k):
    """The long-range branches of the NoiseModel constructor (Noise.jl:
    155-182 projector, 199-223 unitary_2pt, 254-290 unitary_gauss, 355-400
    standard)."""
    import warnings
    sig, tau = _lr_factors(p)
    name = p["name"]
    if unravel == "projector":
        return [MPONoiseProcess(f"projector_{comp}_{name}", sites, gamma / 2.0, sig, tau, 1.0, sgn, L)
                for comp, sgn in (("plus", 1.0), ("minus", -1.0))]
    if unravel == "unitary_2pt":
        th = float(p.get("theta0", theta0))
        s_val = math.sin(th) ** 2
        if not s_val > 1e-12:
            raise ValueError("theta0 too small")
        lam = gamma / s_val
        if dt is not None and lam * dt > 0.1:
            warnings.warn(f"Stability Warning: theta0={th} is too small for dt={dt} (lambda*dt = {lam * dt} > 0.1)")
        return [MPONoiseProcess(f"unitary2pt_{comp}_{name}", sites, lam / 2.0, sig, tau, math.cos(th),
                                1j * sgn * math.sin(th), L) for comp, sgn in (("plus", 1.0), ("minus", -1.0))]
    if unravel == "unitary_gauss":
        sg = float(p.get("sigma", sigma))
        M = int(p.get("M", gauss_M))
        theta_max = float(p.get("theta_max", float(p.get("gauss_k", gauss_k)) * sg))
        thetas, w = gauss_angles(sg, M, theta_max)
        lam = gamma / float(np.sum(w * np.sin(thetas) ** 2))
        return [MPONoiseProcess(f"unitary_gauss_{idx}_{name}", sites, lam * wk, sig, tau, math.cos(th),
                                1j * math.sin(th), L) for idx, (wk, th) in enumerate(zip(w, thetas)) if wk > 0.0]
    if unravel == "analog_auto":
        warnings.warn("Unraveling mode 'analog_auto' is deprecated. "
                      "Please choose 'unitary_2pt' or 'unitary_gauss' manually.")
    return [MPONoiseProcess(name, sites, gamma, sig, tau, 0.0, 1.0, L, factors=(sig, tau))]


_LR_SCALAR_PREFIXES = ("projector_", "unitary2pt_", "unitary_gauss_", "crosstalk_", "pauli_")


def long_range_flags(processes):
    """Per long-range process: (dissipation rate, pauli_long_range) as the
    reference decides them.  handle_longrange_scalar! (Dissipation.jl:161-204)
    decays the state by exp(-dt/2 * rate) at the process's right site: a
    projector pair shares one factor with the summed rate (the first of the
    pair carries it, the mate 0), unitary components and Pauli/crosstalk
    names use their own rate, any other name is an error.  A candidate is
    "pauli_long_range" when is_pauli_proc holds and factors are stored
    (StochasticProcess.jl:176-185, 343-357)."""
    out = {}
    done = set()
    for k, p in enumerate(processes):
        if not isinstance(p, MPONoiseProcess):
            continue
        nm = p.name
        if nm.startswith("projector_"):
            base = nm.replace("projector_plus_", "").replace("projector_minus_", "")
            key = (tuple(p.sites), base)
            if key in done:
                rate = 0.0
            else:
                mates = [q for q in processes if isinstance(q, MPONoiseProcess) and tuple(q.sites) == key[0]
                         and q.name.endswith(base) and q.name.startswith("projector_")]
                if len(mates) != 2:
                    raise ValueError(f"Incomplete projector pair for long-range channel {base} on {key[0]}")
                rate = mates[0].strength + mates[1].strength
                done.add(key)
        elif nm.startswith(_LR_SCALAR_PREFIXES):
            rate = p.strength
        else:
            raise NotImplementedError(f"Non-Pauli long-range processes not fully implemented for: {nm}")
        if ("pauli" in nm or "crosstalk" in nm) and "projector" not in nm:
            pauli = True
        else:
            pauli = bool(p.factors) and all(is_pauli_matrix(f) for f in p.factors)
        out[k] = (rate, pauli and bool(p.factors))
    return out


class NoiseModel:
    """NoiseModel(processes_info, num_qubits; theta0, dt, sigma, gauss_M,
    gauss_k) (src/Noise.jl:299-420).

    Each process dict has "name", "sites", "strength" and optionally
    "matrix" and "unraveling":
      - "standard": the jump operator itself (the matrix, or the named one);
      - "projector": I +- P at gamma/2 each;
      - "unitary_2pt": exp(+-i theta0 P) at gamma / (2 sin^2 theta0) each
        (per-process "theta0" overrides the keyword);
      - "unitary_gauss": exp(i theta_k P) on a Gaussian angle grid (per-process
        "sigma", "M", "gauss_k", "theta_max" override the keywords);
      - "analog_auto": deprecated, warns and falls back to "standard".
    All of these give the same Lindbladian for a Pauli P; they differ in the
    trajectories.  Expanded processes keep the given site order sorted (the
    reference keeps the unsorted order for expansions, so a descending
    adjacent pair would never be a jump candidate there).  With dt given, a
    unitary_2pt rate with lambda*dt > 0.1 warns as in the reference.

    Long-range processes (two sites more than one apart) become
    MPONoiseProcess entries (Noise.jl:155-182,199-223,254-290,355-400): the
    standard unraveling keeps O = sigma_i tau_j with its factors; projector
    gives 1 +- sigma_i tau_j, unitary_2pt cos(theta0) 1 +- i sin(theta0)
    sigma_i tau_j, unitary_gauss cos(theta_k) 1 + i sin(theta_k) sigma_i tau_j
    at the local expansions' rates."""

    def __init__(self, processes, num_qubits: int | None = None, *, theta0: float = math.pi / 2,
                 dt: float | None = None, sigma: float = 1.0, gauss_M: int = 11, gauss_k: float = 4.0):
        import warnings
        self.processes = []
        for p in processes:
            if isinstance(p, (LocalNoiseProcess, MPONoiseProcess)):
                self.processes.append(p)
                continue
            name = p["name"]
            sites = list(p["sites"])
            strength = float(p["strength"])
            unravel = p.get("unraveling", "standard")
            if unravel not in UNRAVELINGS:
                raise ValueError(f"unknown unraveling {unravel!r}")
            if len(sites) == 2:
                sites = sorted(sites)
            if not sites or len(sites) > 2:
                raise ValueError("Invalid sites")
            if len(sites) == 2 and sites[1] - sites[0] > 1:
                if num_qubits is None:
                    raise ValueError("long-range processes need num_qubits")
                if "mpo" in p:
                    raise NotImplementedError("processes given as an explicit MPO are not served")
                self.processes += _long_range_processes(p, sites, strength, unravel, int(num_qubits), theta0,
                                                        dt, sigma, gauss_M, gauss_k)
                continue
            if unravel == "projector":
                self.processes += _projector_expansion(p, sites, _proc_operator(p), strength)
                continue
            if unravel == "unitary_2pt":
                th = float(p.get("theta0", theta0))
                s_val = math.sin(th) ** 2
                if s_val > 1e-12 and dt is not None and strength / s_val * dt > 0.1:
                    warnings.warn(f"Stability Warning: theta0={th} is too small for dt={dt} "
                                  f"(lambda*dt = {strength / s_val * dt} > 0.1)")
                self.processes += _unitary_2pt_expansion(p, sites, _proc_operator(p), strength, th)
                continue
            if unravel == "unitary_gauss":
                self.processes += _unitary_gauss_expansion(
                    p, sites, _proc_operator(p), strength, float(p.get("sigma", sigma)),
                    int(p.get("M", gauss_M)), float(p.get("gauss_k", gauss_k)))
                continue
            if unravel == "analog_auto":
                warnings.warn("Unraveling mode 'analog_auto' is deprecated. "
                              "Please choose 'unitary_2pt' or 'unitary_gauss' manually.")
            self.processes.append(LocalNoiseProcess(name, sites, strength, _proc_operator(p)))


# ---------------------------------------------------------------------------
# Observables and configs (src/SimulationConfigs.jl)
# ---------------------------------------------------------------------------
class Observable:
    """Observable(name, op, sites).  op is a 2x2 / 4x4 matrix or a gate name
    ("x", "y", "z", ...).  kind="entropy" measures the von Neumann entropy
    across the bond right of sites[0] (an addition to the reference)."""

    def __init__(self, name, op=None, sites=None, kind=None):
        self.name = name
        if isinstance(sites, int):
            sites = [sites]
        self.sites = list(sites)
        self.kind = kind or ("local" if op is not None else "entropy")
        if isinstance(op, str):
            op = GATES[op.lower()]
        self.op = None if op is None else np.asarray(op, dtype=np.complex128)
        self.results = np.zeros(0)
        self.trajectories = np.zeros((0, 0))


def _range_len(total_time: float, dt: float) -> int:
    """length(0.0:dt:total_time) (SimulationConfigs.jl:89)."""
    n = total_time / dt
    r = round(n)
    if abs(n - r) <= 1e-10 * max(1.0, abs(n)):
        return int(r) + 1
    return int(math.floor(n)) + 1


class TimeEvolutionConfig:
    def __init__(self, observables, total_time: float, dt: float = 0.1, num_traj: int = 1000,
                 max_bond_dim: int = 4096, min_bond_dim: int = 2, truncation_threshold: float = 1e-9,
                 sample_timesteps: bool = True, order: int = 2):
        self.observables = list(observables)
        self.total_time = float(total_time)
        self.dt = float(dt)
        n = _range_len(self.total_time, self.dt)
        self.times = np.arange(n) * self.dt
        self.num_traj = int(num_traj)
        self.max_bond_dim = int(max_bond_dim)
        self.min_bond_dim = int(min_bond_dim)
        self.truncation_threshold = float(truncation_threshold)
        self.sample_timesteps = bool(sample_timesteps)
        self.order = int(order)


# ---------------------------------------------------------------------------
# Descriptor packing (what the Julia shim does before ccall)
# ---------------------------------------------------------------------------
def _c64(a) -> np.ndarray:
    """Column-major complex128 buffer viewed as interleaved doubles."""
    f = np.asfortranarray(np.asarray(a, dtype=np.complex128))
    return f.reshape(-1, order="F").view(np.float64)


class Descriptors:
    """Owns every buffer referenced by the C descriptors of one run."""

    def __init__(self, psi0: MPS, H: MPO, sim_params: TimeEvolutionConfig, noise_model: NoiseModel | None,
                 *, rng_mode: int = A.YAQS_RNG_PHILOX, seed: int = 0, uniforms: np.ndarray | None = None,
                 krylov_dim: int = 25, krylov_tol: float = 1e-10, krylov_exit_tol: float = 1e-12,
                 precision: int = A.YAQS_PREC_FP64, traj_offset: int = 0, num_traj: int | None = None,
                 tdvp_mode: int = A.YAQS_TDVP_2SITE):
        L = psi0.length
        if H.length != L:
            raise ValueError("MPO and MPS lengths differ")
        self._keep = []
        # MPS
        chi = np.array([1] + [t.shape[2] for t in psi0.tensors], dtype=np.int32)
        for i, t in enumerate(psi0.tensors):
            if t.shape[0] != chi[i] or t.shape[1] != 2:
                raise ValueError(f"bond dimension mismatch at site {i + 1}")
        bufs = [_c64(t) for t in psi0.tensors]
        ptrs = (A.DPTR * L)(*[A.dptr(b) for b in bufs])
        self._keep += [chi, bufs, ptrs]
        self.mps = A.MpsDesc(L, chi.ctypes.data_as(C.POINTER(C.c_int32)), ptrs)
        # MPO
        w = np.array([1] + [t.shape[3] for t in H.tensors], dtype=np.int32)
        wb = [_c64(t) for t in H.tensors]
        wp = (A.DPTR * L)(*[A.dptr(b) for b in wb])
        self._keep += [w, wb, wp]
        self.mpo = A.MpoDesc(L, w.ctypes.data_as(C.POINTER(C.c_int32)), wp)
        defect = mpo_antihermitian_part(H)
        if not defect <= HERMITIAN_TOL:
            raise ValueError(f"the Hamiltonian MPO is not Hermitian (relative anti-Hermitian part {defect:.3g}): "
                             "the engine runs Lanczos, where the reference's :auto Krylov mode switches to Arnoldi")
        # noise
        procs = noise_model.processes if noise_model is not None else []
        arr = (A.NoiseProc * max(1, len(procs)))()
        lr = long_range_flags(procs)
        for k, p in enumerate(procs):
            q = arr[k]
            if isinstance(p, MPONoiseProcess):
                # sigma, tau (column-major 2x2), a, b, dissipation rate
                q.nsites = 2
                q.site[0], q.site[1] = p.sites[0] - 1, p.sites[1] - 1
                q.strength = p.strength
                packed = np.concatenate([_c64(p.sigma), _c64(p.tau), [p.a.real, p.a.imag, p.b.real, p.b.imag,
                                                                      lr[k][0]]])
                for e in range(packed.size):
                    q.matrix[e] = packed[e]
                q.pauli_name = 1
                q.pauli_proc = int(lr[k][1])
                continue
            q.nsites = len(p.sites)
            q.site[0] = p.sites[0] - 1
            q.site[1] = (p.sites[1] - 1) if len(p.sites) == 2 else (p.sites[0] - 1)
            q.strength = p.strength
            m = _c64(p.matrix)
            for e in range(m.size):
                q.matrix[e] = m[e]
            q.pauli_name = int(is_pauli_name(p.name))
            q.pauli_proc = int(is_pauli_matrix(p.matrix) if len(p.sites) == 1 else is_pauli_proc(p.name, p.matrix))
        self._keep.append(arr)
        self.noise = A.NoiseDesc(int(noise_model is not None), len(procs), arr)
        self.all_zero = all(p.strength == 0 for p in procs)
        # observables
        obs = sim_params.observables
        oarr = (A.ObsDesc * max(1, len(obs)))()
        for k, o in enumerate(obs):
            d = oarr[k]
            if o.kind == "entropy":
                d.kind = A.YAQS_OBS_ENTROPY
                d.site[0] = d.site[1] = o.sites[0] - 1
            elif len(o.sites) == 1:
                d.kind = A.YAQS_OBS_LOCAL1
                d.site[0] = d.site[1] = o.sites[0] - 1
            elif len(o.sites) == 2:
                s1, s2 = sorted(o.sites)
                if s2 != s1 + 1:
                    raise ValueError("Only nearest neighbor supported efficiently")  # MPS.jl:627
                d.kind = A.YAQS_OBS_LOCAL2
                d.site[0], d.site[1] = s1 - 1, s2 - 1
            else:
                raise ValueError("Only 1 or 2 site observables supported")
            if o.op is not None:
                m = _c64(o.op)
                for e in range(m.size):
                    d.matrix[e] = m[e]
        self._keep.append(oarr)
        self.obs = oarr
        self.n_obs = len(obs)
        # config
        nt = sim_params.num_traj if num_traj is None else num_traj
        self.cfg = A.TevConfig(sim_params.dt, len(sim_params.times), nt, sim_params.max_bond_dim,
                               sim_params.truncation_threshold, sim_params.order,
                               int(sim_params.sample_timesteps), krylov_dim, krylov_tol, krylov_exit_tol,
                               precision, traj_offset, tdvp_mode)
        self.n_out = len(sim_params.times) if sim_params.sample_timesteps else 1
        # rng
        if rng_mode == A.YAQS_RNG_INJECTED:
            u = np.ascontiguousarray(uniforms, dtype=np.float64)
            if u.ndim != 2 or u.shape[0] < nt:
                raise ValueError("uniforms must be [num_traj, stride]")
            self._keep.append(u)
            self.rng = A.RngDesc(rng_mode, seed, A.dptr(u), u.shape[1])
        else:
            self.rng = A.RngDesc(rng_mode, seed, None, 0)
        self.num_traj = nt


def max_draws(sim_params: TimeEvolutionConfig) -> int:
    """Upper bound on uniforms one trajectory consumes (2 per stochastic step)."""
    n = len(sim_params.times)
    steps = (2 * n - 2) if sim_params.order == 2 else (n - 1)
    return 2 * max(steps, 1)


# ---------------------------------------------------------------------------
# Digital circuits (src/DigitalTJM.jl:35-168)
# ---------------------------------------------------------------------------
class Barrier:
    """GateLibrary.Barrier (src/GateLibrary.jl:305-311)."""

    def __init__(self, label: str = "SAMPLE_OBSERVABLES"):
        self.label = label


class DigitalGate:
    def __init__(self, op, sites, generator=None):
        self.generator, self.coeff = None, 1.0
        if isinstance(op, GateOp):
            self.generator, self.coeff = op.generator, op.coeff
        if generator is not None:  # add_gate!(...; generator=...) (DigitalTJM.jl:64-66): exp(-i g1 (x) g2)
            self.generator, self.coeff = tuple(np.asarray(g, dtype=np.complex128) for g in generator), 1.0
        self.op = op if isinstance(op, Barrier) else np.asarray(op, dtype=np.complex128)
        self.sites = list(sites)


class DigitalCircuit:
    """DigitalCircuit(num_qubits) with add_gate (add_gate!, DigitalTJM.jl:60-66).
    Gates are 2x2 / 4x4 matrices (4x4 in the p1 + 2 p2 basis of the smaller
    site first, as apply_local_gate_exact! reads them) or Barrier."""

    def __init__(self, num_qubits: int):
        self.num_qubits = int(num_qubits)
        self.gates: list[DigitalGate] = []

    def add_gate(self, op, sites, generator=None):
        if isinstance(sites, int):
            sites = [sites]
        self.gates.append(DigitalGate(op, sites, generator))
        return self


class RepeatedDigitalCircuit:
    """RepeatedDigitalCircuit(step, repeats) (DigitalTJM.jl:47-58, 452-536):
    ``step`` run ``repeats`` times.  The step's layers are formed once; a
    sample barrier before the step's first layer samples once at the start,
    every other sample barrier samples after its layer in every repetition.

    ``flatten`` gives the equivalent DigitalCircuit the engine runs: the step's
    gates per repetition, a layer break (a barrier that does not sample)
    between repetitions so layers never merge across them, and the leading
    sample barriers kept only in the first repetition."""

    def __init__(self, step: DigitalCircuit, repeats: int):
        if repeats < 0:
            raise ValueError("repeats must be >= 0")
        self.step = step
        self.repeats = int(repeats)

    @property
    def num_qubits(self) -> int:
        return self.step.num_qubits

    def flatten(self) -> DigitalCircuit:
        out = DigitalCircuit(self.step.num_qubits)
        lead = 0
        while lead < len(self.step.gates) and isinstance(self.step.gates[lead].op, Barrier):
            lead += 1
        for r in range(self.repeats):
            if r > 0:
                out.gates.append(DigitalGate(Barrier("LAYER_BREAK"), []))
            for k, g in enumerate(self.step.gates):
                if r > 0 and k < lead:
                    continue
                out.gates.append(g)
        if self.repeats == 0:
            out.gates = [g for g in self.step.gates[:lead]]
        return out


def as_circuit(circ) -> DigitalCircuit:
    """A DigitalCircuit for the engine (a RepeatedDigitalCircuit is flattened)."""
    return circ.flatten() if isinstance(circ, RepeatedDigitalCircuit) else circ


def add_gate(circ: DigitalCircuit, op, sites, generator=None):
    return circ.add_gate(op, sites, generator)


def process_circuit(circ: DigitalCircuit):
    """Greedy layering and barrier map (DigitalTJM.jl:86-145)."""
    circ = as_circuit(circ)
    layers, barrier_map, cur, busy = [], {}, [], set()
    for g in circ.gates:
        if isinstance(g.op, Barrier):
            if cur:
                layers.append(cur)
                cur, busy = [], set()
            barrier_map.setdefault(len(layers), []).append(g.op.label)
            continue
        if any(q in busy for q in g.sites):
            layers.append(cur)
            cur, busy = [], set()
        cur.append(g)
        busy.update(g.sites)
    if cur:
        layers.append(cur)
    return layers, barrier_map


def sample_plan(circ: DigitalCircuit):
    """(sample_at_start, sample_after, n_samples) of run_digital_tjm (DigitalTJM.jl:159-168, 375-379)."""
    layers, bm = process_circuit(circ)
    has = lambda i: any(lbl.upper() == "SAMPLE_OBSERVABLES" for lbl in bm.get(i, []))  # noqa: E731
    start = has(0)
    after = [l for l in range(1, len(layers) + 1) if has(l)]
    n = (1 if start else 0) + len(after)
    return start, after, max(n, 1)


class CircuitDescriptors:
    """Owns every buffer referenced by the C descriptors of a digital run."""

    def __init__(self, psi0: MPS, circ: DigitalCircuit, sim_params: TimeEvolutionConfig,
                 noise_model: NoiseModel | None, *, rng_mode: int = A.YAQS_RNG_PHILOX, seed: int = 0,
                 uniforms: np.ndarray | None = None, traj_offset: int = 0, num_traj: int | None = None,
                 local_method: str = "tebd", long_range_method: str = "tebd"):
        L = psi0.length
        circ = as_circuit(circ)
        if circ.num_qubits != L:
            raise ValueError("circuit and MPS sizes differ")
        # reuse the analog packer for the state, noise, observables and rng
        dummy = init_ising(L, 0.0, 0.0)
        base = Descriptors(psi0, dummy, sim_params, noise_model, rng_mode=rng_mode, seed=seed,
                           uniforms=uniforms, traj_offset=traj_offset, num_traj=num_traj)
        self._base = base
        self.mps, self.noise, self.obs, self.n_obs, self.rng = base.mps, base.noise, base.obs, base.n_obs, base.rng
        self.num_traj = base.num_traj
        self.gates = self.pack_gates(circ)
        self.n_gates = len(circ.gates)
        meth = {"tebd": A.YAQS_METHOD_TEBD, "tdvp": A.YAQS_METHOD_TDVP}
        self.cfg = A.CircuitConfig(self.num_traj, sim_params.max_bond_dim, sim_params.truncation_threshold,
                                   meth[local_method], meth[long_range_method], A.YAQS_PREC_FP64, traj_offset)
        self.n_out = sample_plan(circ)[2]

    @staticmethod
    def pack_gates(circ: DigitalCircuit):
        """yaqs_gate_desc array of the circuit (sites 0-based, matrices column-major)."""
        gd = (A.GateDesc * max(1, len(circ.gates)))()
        for k, g in enumerate(circ.gates):
            d = gd[k]
            if isinstance(g.op, Barrier):
                d.kind = A.YAQS_GATE_BARRIER
                d.sample = int(g.op.label.upper() == "SAMPLE_OBSERVABLES")
                continue
            if len(g.sites) == 1:
                d.kind = A.YAQS_GATE_1Q
                d.site[0] = d.site[1] = g.sites[0] - 1
            elif len(g.sites) == 2:
                d.kind = A.YAQS_GATE_2Q
                d.site[0], d.site[1] = g.sites[0] - 1, g.sites[1] - 1
            else:
                raise ValueError("gates act on 1 or 2 qubits")
            m = _c64(g.op)
            for e in range(m.size):
                d.matrix[e] = m[e]
            if g.generator is not None and len(g.sites) == 2:
                d.has_generator = 1
                d.coeff = g.coeff
                g1, g2 = _c64(g.generator[0]), _c64(g.generator[1])
                for e in range(8):
                    d.gen1[e] = g1[e]
                    d.gen2[e] = g2[e]
        return gd


def create_local_noise_model(noise_model: NoiseModel, site1: int, site2: int) -> NoiseModel:
    """Processes of a noise model that act after a gate on (site1, site2):
    1-site processes on either site and 2-site processes on exactly that pair
    (DigitalTJM.jl:172-188).  The engine applies the same selection on the
    device (proc_on in the CUDA sources)."""
    out = []
    for p in noise_model.processes:
        if len(p.sites) == 1 and p.sites[0] in (site1, site2):
            out.append(p)
        elif len(p.sites) == 2 and sorted(p.sites) == sorted((site1, site2)):
            out.append(p)
    return NoiseModel(out)


def max_draws_digital(circ: DigitalCircuit) -> int:
    """Upper bound on uniforms one digital trajectory consumes (2 per 2-qubit gate)."""
    circ = as_circuit(circ)
    return 2 * max(1, sum(1 for g in circ.gates if not isinstance(g.op, Barrier) and len(g.sites) == 2))


# ---------------------------------------------------------------------------
# Simulator.run (src/Simulator.jl:22-69, 127-141) on the GPU engine
# ---------------------------------------------------------------------------
class RunResult:
    def __init__(self, traj, mean, maxchi, stats):
        self.trajectories = traj      # [num_traj, n_obs, n_out]
        self.mean = mean              # [n_obs, n_out]
        self.max_bond = maxchi        # [num_traj, n_out]
        self.stats = stats

    @property
    def variance(self) -> np.ndarray:
        """Unbiased ensemble variance per observable and sample (an addition:
        the reference aggregates means only, SimulationConfigs.jl:168-181)."""
        n = self.trajectories.shape[0]
        return self.trajectories.var(axis=0, ddof=1) if n > 1 else np.zeros_like(self.mean)

    @property
    def standard_error(self) -> np.ndarray:
        """Standard error of the ensemble mean, sqrt(variance / num_traj)."""
        return np.sqrt(self.variance / self.trajectories.shape[0])


def run_descriptors(desc: Descriptors, ctx=None) -> RunResult:
    """Runs a packed problem through yaqs_analog_run."""
    from . import _lib
    ctx = ctx or _lib.default_context()
    nt, nobs, nout = desc.num_traj, desc.n_obs, desc.n_out
    traj = np.zeros((nt, max(nobs, 1), nout))
    mean = np.zeros((max(nobs, 1), nout))
    chi = np.zeros((nt, nout), dtype=np.int32)
    st = A.RunStats()
    ctx.check(ctx._lib.yaqs_analog_run(ctx.handle, C.byref(desc.mps), C.byref(desc.mpo), C.byref(desc.noise),
                                       desc.obs, nobs, C.byref(desc.cfg), C.byref(desc.rng), A.dptr(traj),
                                       A.dptr(mean), chi.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(st)))
    return RunResult(traj[:, :nobs, :], mean[:nobs, :], chi, st.as_dict())


def run_circuit_descriptors(desc: CircuitDescriptors, ctx=None) -> RunResult:
    """Runs a packed circuit problem through yaqs_digital_run."""
    from . import _lib
    ctx = ctx or _lib.default_context()
    nt, nobs, nout = desc.num_traj, desc.n_obs, desc.n_out
    traj = np.zeros((nt, max(nobs, 1), nout))
    mean = np.zeros((max(nobs, 1), nout))
    chi = np.zeros((nt, nout), dtype=np.int32)
    st = A.RunStats()
    ctx.check(ctx._lib.yaqs_digital_run(ctx.handle, C.byref(desc.mps), desc.gates, desc.n_gates,
                                        C.byref(desc.noise), desc.obs, nobs, C.byref(desc.cfg), C.byref(desc.rng),
                                        A.dptr(traj), A.dptr(mean), chi.ctypes.data_as(C.POINTER(C.c_int32)),
                                        C.byref(st)))
    return RunResult(traj[:, :nobs, :], mean[:nobs, :], chi, st.as_dict())


HERMITIAN_TOL = 1e-5  # largest relative anti-Hermitian part a run accepts


def mpo_antihermitian_part(H: MPO) -> float:
    """||H - H^dag||_F / ||H||_F by the transfer contractions the library uses
    (tr(H^dag H) and tr(H H) over two copies' bonds), in numpy: the host-side
    form of the check, so descriptors fail early without the library.
    Values below about 1e-7 are rounding."""
    e1 = np.ones((1, 1), dtype=np.complex128)
    e2 = np.ones((1, 1), dtype=np.complex128)
    for t in H.tensors:
        e1 = np.einsum("ab,aoir,bois->rs", e1, t.conj(), t)
        e2 = np.einsum("ab,aoir,bios->rs", e2, t, t)
    n1 = e1[0, 0].real
    if n1 == 0.0:
        return 0.0
    q = (2.0 * n1 - 2.0 * e2[0, 0].real) / n1
    return math.sqrt(q) if q > 0.0 else (0.0 if q == q else q)


def hermitian_defect(H: MPO) -> float:
    """||H - H^dag||_F / ||H||_F as yaqs_mpo_hermitian_defect computes it (host
    arithmetic in the library, no device): the check that stands in for the
    reference's _ishermitian_check (Algorithms.jl:120-137).  Runs refuse a
    Hamiltonian above 1e-5; values below about 1e-7 are rounding."""
    from . import _lib
    L = _lib.lib()
    w = np.array([1] + [t.shape[3] for t in H.tensors], dtype=np.int32)
    wb = [_c64(t) for t in H.tensors]
    wp = (A.DPTR * H.length)(*[A.dptr(b) for b in wb])
    desc = A.MpoDesc(H.length, w.ctypes.data_as(C.POINTER(C.c_int32)), wp)
    out = C.c_double(0.0)
    st = L.yaqs_mpo_hermitian_defect(C.byref(desc), C.byref(out))
    if st != 0:
        raise _lib.EngineError(st, L.yaqs_last_error(None).decode())
    return out.value


def digital_plan(circ: DigitalCircuit) -> tuple[int, int]:
    """(number of layers, number of measurement columns) as the library plans them."""
    from . import _lib
    L = _lib.lib()
    circ = as_circuit(circ)
    gd = CircuitDescriptors.pack_gates(circ)
    nl, ns = C.c_int32(0), C.c_int32(0)
    st = L.yaqs_digital_plan(gd, len(circ.gates), C.byref(nl), C.byref(ns))
    if st != 0:
        raise _lib.EngineError(st, L.yaqs_last_error(None).decode())
    return nl.value, ns.value


class Session:
    """A run held on the device (yaqs_analog_begin or yaqs_digital_begin,
    then advance / finish).

    ``advance(n)`` evolves the next n recorded time indices (analog) or
    circuit layers (digital; the first step prepares the states) of every
    trajectory and returns their device time in ms."""

    def __init__(self, desc, ctx=None):
        from . import _lib
        self.ctx = ctx or _lib.default_context()
        self.desc = desc
        h = C.c_void_p()
        if isinstance(desc, CircuitDescriptors):  # one advance step = one circuit layer (launch 0 prepares)
            self.ctx.check(self.ctx._lib.yaqs_digital_begin(self.ctx.handle, C.byref(desc.mps), desc.gates,
                                                            desc.n_gates, C.byref(desc.noise), desc.obs, desc.n_obs,
                                                            C.byref(desc.cfg), C.byref(desc.rng), C.byref(h)))
        else:
            self.ctx.check(self.ctx._lib.yaqs_analog_begin(self.ctx.handle, C.byref(desc.mps), C.byref(desc.mpo),
                                                           C.byref(desc.noise), desc.obs, desc.n_obs,
                                                           C.byref(desc.cfg), C.byref(desc.rng), C.byref(h)))
        self.handle = h

    @property
    def remaining(self) -> int:
        return self.ctx._lib.yaqs_analog_remaining(self.handle)

    def advance(self, n: int) -> float:
        ms = C.c_double(0.0)
        self.ctx.check(self.ctx._lib.yaqs_analog_advance(self.handle, n, C.byref(ms)))
        return ms.value

    PHASES = ("gemm", "mpo_apply", "lanczos_orth", "tridiag_exp", "svd_sweeps", "svd_vectors", "qr_factor",
              "qr_formq", "norm_contraction", "env_update", "dissipation", "jump_step", "observables", "tdvp_sweep",
              "step", "state_copy")

    def stats(self) -> dict:
        st = A.RunStats()
        self.ctx.check(self.ctx._lib.yaqs_analog_stats(self.handle, C.byref(st)))
        return st.as_dict()

    def state(self, traj: int) -> MPS:
        """The evolving state of trajectory ``traj`` (0-based within this
        run) after the last advance, copied from the device (yaqs_run_state)."""
        L = self.desc.mps.L
        chi = np.zeros(L + 1, dtype=np.int32)
        oc = C.c_int32(0)
        need = C.c_int64(0)
        ip = C.POINTER(C.c_int32)
        self.ctx.check(self.ctx._lib.yaqs_run_state(self.handle, traj, chi.ctypes.data_as(ip), C.byref(oc), None,
                                                    0, C.byref(need)))
        buf = np.zeros(need.value, dtype=np.float64)
        self.ctx.check(self.ctx._lib.yaqs_run_state(self.handle, traj, chi.ctypes.data_as(ip), C.byref(oc),
                                                    A.dptr(buf), need.value, C.byref(need)))
        z = buf.view(np.complex128)
        tens, pos = [], 0
        for i in range(L):
            n = int(chi[i]) * 2 * int(chi[i + 1])
            tens.append(z[pos:pos + n].reshape(int(chi[i]), 2, int(chi[i + 1]), order="F"))
            pos += n
        m = MPS(L, tensors=tens)
        m.orth_center = int(oc.value) + 1
        return m

    def checkpoint(self) -> dict:
        """Every trajectory's state and draw count at the current position
        (yaqs_run_position / yaqs_run_state / yaqs_run_rng)."""
        pos = C.c_int32(0)
        self.ctx.check(self.ctx._lib.yaqs_run_position(self.handle, C.byref(pos)))
        states, draws = [], []
        for k in range(self.desc.num_traj):
            states.append(self.state(k))
            d = C.c_int64(0)
            self.ctx.check(self.ctx._lib.yaqs_run_rng(self.handle, k, C.byref(d)))
            draws.append(d.value)
        return {"position": pos.value, "states": states, "draws": draws}

    def restore(self, cp: dict) -> None:
        """Put every trajectory back to a checkpoint of this run and make the
        next advance continue from its position (yaqs_run_restore /
        yaqs_run_seek)."""
        ip = C.POINTER(C.c_int32)
        for k, (m, d) in enumerate(zip(cp["states"], cp["draws"])):
            chi = np.array(m.bond_dims, dtype=np.int32)
            buf = np.concatenate([_c64(t) for t in m.tensors])
            self.ctx.check(self.ctx._lib.yaqs_run_restore(self.handle, k, chi.ctypes.data_as(ip), m.orth_center - 1,
                                                          A.dptr(buf), int(d)))
        self.ctx.check(self.ctx._lib.yaqs_run_seek(self.handle, cp["position"]))

    def profile(self) -> dict:
        out = np.zeros(16)
        self.ctx.check(self.ctx._lib.yaqs_analog_profile(self.handle, A.dptr(out)))
        return dict(zip(self.PHASES, out.tolist()))

    def finish(self) -> RunResult:
        d = self.desc
        nt, nobs, nout = d.num_traj, d.n_obs, d.n_out
        traj = np.zeros((nt, max(nobs, 1), nout))
        mean = np.zeros((max(nobs, 1), nout))
        chi = np.zeros((nt, nout), dtype=np.int32)
        st = A.RunStats()
        h, self.handle = self.handle, None
        self.ctx.check(self.ctx._lib.yaqs_analog_finish(h, A.dptr(traj), A.dptr(mean),
                                                        chi.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(st)))
        return RunResult(traj[:, :nobs, :], mean[:nobs, :], chi, st.as_dict())


class Server:
    """Request loop serving many simulations at once on one GPU
    (yaqs_server_*): requests of any size are admitted as device memory
    frees up, all admitted runs advance together in one persistent kernel
    launch per step, and each request's results equal those of running it
    alone.  ``submit`` copies the request and returns an id at once."""

    def __init__(self, max_L: int = 64, max_bond_dim: int = 128, max_mpo_width: int = 5, krylov_dim: int = 25,
                 mixed: bool = True, chunk: int = 1, hbm_budget: int = 0, ctx=None):
        from . import _lib
        self.ctx = ctx or _lib.default_context()
        self._lib = self.ctx._lib
        cfg = A.ServerConfig(max_L, max_bond_dim, max_mpo_width, krylov_dim, int(mixed), chunk, hbm_budget)
        h = C.c_void_p()
        self.ctx.check(self._lib.yaqs_server_create(self.ctx.handle, C.byref(cfg), C.byref(h)))
        self.handle = h
        self._meta = {}

    def _check_static(self, st):
        if st != A.YAQS_OK:
            from . import _lib
            raise _lib.EngineError(st, self._lib.yaqs_last_error(None).decode())

    def submit(self, initial_state: MPS, operator, sim_params: TimeEvolutionConfig,
               noise_model: NoiseModel | None = None, *, seed: int = 0, uniforms: np.ndarray | None = None,
               precision: str = "fp64", traj_offset: int = 0, tdvp: str = "2site") -> int:
        mode = A.YAQS_RNG_INJECTED if uniforms is not None else A.YAQS_RNG_PHILOX
        rid = C.c_int64(0)
        if isinstance(operator, (DigitalCircuit, RepeatedDigitalCircuit)):
            d = CircuitDescriptors(initial_state, operator, sim_params, noise_model, rng_mode=mode, seed=seed,
                                   uniforms=uniforms, traj_offset=traj_offset)  # server slots: TEBD gates
            st = self._lib.yaqs_server_submit_digital(self.handle, C.byref(d.mps), d.gates, d.n_gates,
                                                      C.byref(d.noise), d.obs, d.n_obs, C.byref(d.cfg),
                                                      C.byref(d.rng), C.byref(rid))
        else:
            prec = {"fp64": A.YAQS_PREC_FP64, "mixed": A.YAQS_PREC_MIXED}[precision]
            d = Descriptors(initial_state, operator, sim_params, noise_model, rng_mode=mode, seed=seed,
                            uniforms=uniforms, precision=prec, traj_offset=traj_offset, tdvp_mode=TDVP_MODES[tdvp])
            st = self._lib.yaqs_server_submit_analog(self.handle, C.byref(d.mps), C.byref(d.mpo), C.byref(d.noise),
                                                     d.obs, d.n_obs, C.byref(d.cfg), C.byref(d.rng), C.byref(rid))
        self._check_static(st)
        self._meta[rid.value] = (d.num_traj, d.n_obs, d.n_out)
        return rid.value

    def poll(self, rid: int) -> int:
        s = C.c_int32(0)
        self._check_static(self._lib.yaqs_server_poll(self.handle, rid, C.byref(s)))
        return s.value

    def wait(self, rid: int, timeout: float | None = None):
        self._check_static(self._lib.yaqs_server_wait(self.handle, rid, -1.0 if timeout is None else timeout))

    def result(self, rid: int, timeout: float | None = None) -> RunResult:
        """Waits for the request and returns its RunResult (``times`` = queued, running, total seconds)."""
        self.wait(rid, timeout)
        nt, nobs, nout = self._meta.pop(rid)
        traj = np.zeros((nt, max(nobs, 1), nout))
        mean = np.zeros((max(nobs, 1), nout))
        chi = np.zeros((nt, nout), dtype=np.int32)
        st = A.RunStats()
        times = np.zeros(3)
        code = self._lib.yaqs_server_take(self.handle, rid, A.dptr(traj), A.dptr(mean),
                                          chi.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(st), A.dptr(times))
        if code != A.YAQS_OK:
            from . import _lib
            raise _lib.EngineError(code, self._lib.yaqs_server_last_error(self.handle).decode())
        res = RunResult(traj[:, :nobs, :], mean[:nobs, :], chi, st.as_dict())
        res.times = times
        return res

    def stats(self) -> dict:
        s = A.ServerStats()
        self._check_static(self._lib.yaqs_server_stats_get(self.handle, C.byref(s)))
        return s.as_dict()

    def close(self):
        if getattr(self, "handle", None):
            self._lib.yaqs_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()


def random_mps(length: int, chi: int, seed: int = 0) -> MPS:
    """An MPS with every bond at min(2^b, 2^(L-b), chi) and Gaussian entries
    (a saturated-bond-dimension start state; normalised by the engine)."""
    rng = np.random.default_rng(seed)
    dims = [min(2 ** min(b, length - b), chi) for b in range(length + 1)]
    ts = [(rng.standard_normal((dims[i], 2, dims[i + 1])) + 1j * rng.standard_normal((dims[i], 2, dims[i + 1])))
          for i in range(length)]
    return MPS(length, tensors=ts)


TDVP_MODES = {"2site": A.YAQS_TDVP_2SITE, "1site": A.YAQS_TDVP_1SITE, "dynamic": A.YAQS_TDVP_DYNAMIC}


def _methods(circ, local_method, long_range_method):
    """Digital gate methods: the given ones, else the reference's default
    TJMOptions() (TDVP windows for every gate, DigitalTJM.jl:70-76) when every
    2-qubit gate carries a generator; gates given as bare matrices (which the
    reference's typed gates cannot express) run by TEBD."""
    circ = as_circuit(circ)
    all_gen = all(g.generator is not None for g in circ.gates
                  if not isinstance(g.op, Barrier) and len(g.sites) == 2)
    default = "tdvp" if all_gen else "tebd"
    return {"local_method": local_method or default, "long_range_method": long_range_method or default}


def available_cpus() -> int:
    """available_cpus (Simulator.jl:14-20): SLURM_CPUS_ON_NODE when set, else
    the host's logical CPU count."""
    if "SLURM_CPUS_ON_NODE" in os.environ:
        return int(os.environ["SLURM_CPUS_ON_NODE"])
    return os.cpu_count() or 1


def run(initial_state: MPS, operator, sim_params: TimeEvolutionConfig, noise_model: NoiseModel | None = None,
        *, parallel: bool = True, seed: int = 0, uniforms: np.ndarray | None = None, krylov_exit_tol: float = 1e-12,
        precision: str = "fp64", tdvp: str = "2site", local_method: str | None = None,
        long_range_method: str | None = None, ctx=None) -> RunResult:
    """Simulator.run (Simulator.jl:127-141) for an MPO (analog TJM) or a
    DigitalCircuit (digital TJM, TEBD gate application).  Fills every
    observable's ``trajectories`` and ``results`` like _run_analog /
    _run_digital; the result's ``max_bond`` holds the per-trajectory bond
    dimensions at each measurement.  As in the reference, a noiseless model
    runs one trajectory and mutates ``sim_params.num_traj`` (Simulator.jl:27-29).
    ``precision="mixed"`` runs the analog H_eff and environment contractions
    in complex FP32 on the tensor cores (Lanczos orthogonalisation, SVD/QR,
    norms and jump probabilities stay FP64).  ``tdvp`` selects the sweep:
    "2site" (two_site_tdvp!, the reference's analog path), "1site"
    (single_site_tdvp!) or "dynamic" (1-site TDVP with 2-site growth up to
    max_bond_dim, the Python lineage's local_dynamic_tdvp).  For circuits,
    ``local_method`` / ``long_range_method`` ("tebd" or "tdvp") are the
    TJMOptions; left unset they follow the reference's default (see
    _methods).  A RepeatedDigitalCircuit runs as its flattened circuit.
    ``parallel`` is accepted for the reference's signature; every trajectory
    of the run advances together on the device either way.  As in the
    reference, ``initial_state`` is left normalised (centre at site 1) and a
    configuration other than TimeEvolutionConfig is an error."""
    prec = {"fp64": A.YAQS_PREC_FP64, "mixed": A.YAQS_PREC_MIXED}[precision]
    if isinstance(operator, RepeatedDigitalCircuit):
        operator = operator.flatten()
    if not isinstance(sim_params, TimeEvolutionConfig):
        raise TypeError("Only TimeEvolutionConfig is supported.")
    if not isinstance(operator, (MPO, DigitalCircuit)):
        raise TypeError("Simulation requires MPO (Analog) or DigitalCircuit (Digital).")
    if noise_model is None or all(p.strength == 0 for p in noise_model.processes):
        sim_params.num_traj = 1
    mode = A.YAQS_RNG_INJECTED if uniforms is not None else A.YAQS_RNG_PHILOX
    if isinstance(operator, DigitalCircuit):  # _run_digital, Simulator.jl:71-125
        desc = CircuitDescriptors(initial_state, operator, sim_params, noise_model, rng_mode=mode, seed=seed,
                                  uniforms=uniforms, **_methods(operator, local_method, long_range_method))
        res = run_circuit_descriptors(desc, ctx)
    else:
        desc = Descriptors(initial_state, operator, sim_params, noise_model, rng_mode=mode, seed=seed,
                           uniforms=uniforms, krylov_exit_tol=krylov_exit_tol, precision=prec,
                           tdvp_mode=TDVP_MODES[tdvp])
        res = run_descriptors(desc, ctx)
    if isinstance(operator, DigitalCircuit):
        # obs buffers sized by sim_params.times; the first min(n_samples, columns) are filled (Simulator.jl:99-103)
        ncol = len(sim_params.times) if sim_params.sample_timesteps else 1
        n_copy = min(ncol, res.trajectories.shape[2])
        for k, o in enumerate(sim_params.observables):
            o.trajectories = np.zeros((sim_params.num_traj, ncol), dtype=np.complex128)
            o.trajectories[:, :n_copy] = res.trajectories[:, k, :n_copy]
            o.results = o.trajectories.real.sum(axis=0) / sim_params.num_traj
    else:
        for k, o in enumerate(sim_params.observables):
            o.trajectories = res.trajectories[:, k, :].astype(np.complex128)
            o.results = res.mean[k].copy()
    # the reference normalises the caller's initial state in place
    # (Simulator.jl:128, normalize! with the centre at site 1); the engine
    # normalised its own copy, so the caller's object is brought to the same
    # form here, after the run, leaving what the device received unchanged
    from .tensornet import normalize
    normalize(initial_state)
    return res
