"""Host-side MPS and MPO algebra and measurement: the callers' side of the
engine (building and compressing Hamiltonians, inspecting and sampling
states).  Plain numpy; nothing here runs on the device.

* Decompositions (src/Decompositions.jl): right_qr, left_qr, two_site_svd.
* MPS (src/MPS.jl): gauge moves, normalisation, truncation, overlaps,
  local expectations, projective shots and bitstring projections.
* MPO (src/MPO.jl:271-556): canonical form, compression, MPO x MPS,
  <psi|W|psi>, sums, scalar multiples and products.
* Measurement configs (src/SimulationConfigs.jl:42-56, 95-208):
  MeasurementConfig (shots) and StrongMeasurementConfig (trajectories) with
  their aggregation; expect, initialize! and aggregate_trajectories! for
  observables of either config.

Tensors follow the engine's layouts: MPS (left, phys, right), MPO (left,
out, in, right), column-major reshapes as in the reference; sites 1-based.
"""
from __future__ import annotations

import copy

import numpy as np

from .api import MPO, MPS, Observable

# ---------------------------------------------------------------------------
# small factorisations (thin QR / LQ as LinearAlgebra.qr / lq give them)
# ---------------------------------------------------------------------------


def _qr(M):
    Q, R = np.linalg.qr(M, mode="reduced")
    return Q, R


def _lq(M):
    Q, R = np.linalg.qr(M.conj().T, mode="reduced")
    return R.conj().T, Q.conj().T


def _f(a, shape):
    return np.reshape(a, shape, order="F")


def right_qr(tensor):
    """right_qr (Decompositions.jl:18-33): thin QR of the (left*phys, right)
    matricisation; returns Q as (left, phys, k) and R as (k, right)."""
    l, p, r = tensor.shape
    Q, R = _qr(_f(np.asarray(tensor, dtype=np.complex128), (l * p, r)))
    return _f(Q, (l, p, Q.shape[1])), R


def left_qr(tensor):
    """left_qr (Decompositions.jl:35-58): thin LQ of the (left, phys*right)
    matricisation; returns L as (left, k) and Q as (k, phys, right)."""
    l, p, r = tensor.shape
    Lm, Q = _lq(_f(np.asarray(tensor, dtype=np.complex128), (l, p * r)))
    return Lm, _f(Q, (Q.shape[0], p, r))


def two_site_svd(A, B, threshold: float, max_bond_dim: int | None = None):
    """two_site_svd (Decompositions.jl:85-164): merge A (l, pa, k) and
    B (k, pb, r), SVD the (l*pa, pb*r) matrix, keep by the absolute rule
    (discard from the smallest while the discarded weight stays below
    threshold, keep the crossing value, at least 2), at most max_bond_dim;
    returns U as (l, pa, keep) and S*Vt as (keep, pb, r).  The kept count is
    also capped at the number of singular values, where the reference would
    index past them."""
    la, pa, ra = A.shape
    lb, pb, rb = B.shape
    if ra != lb:
        raise ValueError("bond dimensions of A and B differ")
    theta = _f(A, (la * pa, ra)) @ _f(B, (lb, pb * rb))
    U, S, Vt = np.linalg.svd(theta, full_matrices=False)
    keep, disc = len(S), 0.0
    for k in range(len(S), 0, -1):
        disc += S[k - 1] ** 2
        if disc >= threshold:
            keep = max(k, 2)
            break
    if max_bond_dim is not None:
        keep = min(keep, max_bond_dim)
    keep = max(min(keep, len(S)), 1)
    return _f(U[:, :keep], (la, pa, keep)), _f(S[:keep, None] * Vt[:keep], (keep, pb, rb))


# ---------------------------------------------------------------------------
# MPS (src/MPS.jl)
# ---------------------------------------------------------------------------
def check_if_valid_mps(mps: MPS) -> bool:
    """check_if_valid_mps (MPS.jl:153-166): neighbouring bonds match."""
    return all(mps.tensors[i].shape[2] == mps.tensors[i + 1].shape[0] for i in range(mps.length - 1))


def check_canonical_form(mps: MPS) -> list[int]:
    """check_canonical_form (MPS.jl:510-512): the recorded centre, as a
    one-element list (the reference does not inspect the tensors)."""
    return [mps.orth_center]


def write_max_bond_dim(mps: MPS) -> int:
    """write_max_bond_dim (MPS.jl:168-174)."""
    return max(t.shape[2] for t in mps.tensors)


def shift_orthogonality_center(mps: MPS, new_center: int) -> MPS:
    """shift_orthogonality_center! (MPS.jl:182-266): QR steps to the right,
    LQ steps to the left, from the recorded centre (1-based)."""
    oc = mps.orth_center
    if not 1 <= oc <= mps.length:
        raise ValueError("the orthogonality centre is not known: normalize the state first")
    if new_center > oc:
        for i in range(oc - 1, new_center - 1):
            A = mps.tensors[i]
            l, d, r = A.shape
            Q, R = _qr(_f(A, (l * d, r)))
            rn = R.shape[0]
            mps.tensors[i] = _f(Q, (l, d, rn))
            N = mps.tensors[i + 1]
            mps.tensors[i + 1] = _f(R @ _f(N, (r, -1)), (rn, N.shape[1], N.shape[2]))
    elif new_center < oc:
        for i in range(oc - 1, new_center - 1, -1):
            A = mps.tensors[i]
            l, d, r = A.shape
            Lm, Q = _lq(_f(A, (l, d * r)))
            rn = Lm.shape[1]
            mps.tensors[i] = _f(Q, (rn, d, r))
            P = mps.tensors[i - 1]
            mps.tensors[i - 1] = _f(_f(P, (-1, l)) @ Lm, (P.shape[0], P.shape[1], rn))
    mps.orth_center = new_center
    return mps


def normalize(mps: MPS) -> MPS:
    """normalize! (MPS.jl:274-311): LQ sweep L -> 2, then site 1 scaled to
    unit norm when its norm exceeds 1e-13; the centre ends at site 1."""
    mps.orth_center = mps.length
    shift_orthogonality_center(mps, 1)
    nrm = np.linalg.norm(mps.tensors[0])
    if nrm > 1e-13:
        mps.tensors[0] = mps.tensors[0] / nrm
    mps.orth_center = 1
    return mps


def mps_norm(mps: MPS) -> float:
    """norm(mps) (MPS.jl:518-521): the norm of the centre tensor."""
    return float(np.linalg.norm(mps.tensors[mps.orth_center - 1]))


def scalar_product(psi: MPS, phi: MPS) -> complex:
    """scalar_product(psi, phi) as the reference computes it (MPS.jl:528-585):
    a left-to-right transfer contraction of psi with conj(phi), i.e.
    sum psi * conj(phi) = <phi|psi>.  The reference's docstring reads <a|b>,
    but its code conjugates the second argument; this follows the code, so
    scalar_product(psi(t), psi0) of an eigenstate is e^{-iEt} as in
    test_Algorithms.jl:37-95."""
    E = np.ones((1, 1), dtype=np.complex128)
    for A, B in zip(psi.tensors, phi.tensors):
        E = np.einsum("ab,apc,bpd->cd", E, A, B.conj())
    return complex(E[0, 0])


def truncate(mps: MPS, threshold: float = 1e-12, max_bond_dim: int | None = None) -> float:
    """MPS.truncate! (MPS.jl:320-440): centre to site 1, one SVD sweep with
    the absolute rule (discard from the smallest while the discarded weight
    stays below threshold, keep the crossing value, at least 2), at most
    max_bond_dim, then normalize!.  Returns the discarded weight."""
    shift_orthogonality_center(mps, 1)
    err = 0.0
    for i in range(mps.length - 1):
        A, B = mps.tensors[i], mps.tensors[i + 1]
        l, d1, k = A.shape
        _, d2, r = B.shape
        theta = _f(A, (l * d1, k)) @ _f(B, (k, d2 * r))
        scale = np.abs(theta).max() if theta.size else 0.0
        if not np.isfinite(scale):  # MPS.jl:356-360
            raise ValueError(f"truncate!: non-finite entries encountered in Theta (scale={scale})")
        U, S, Vh = np.linalg.svd(theta, full_matrices=False)
        keep, disc = len(S), 0.0
        for kk in range(len(S), 0, -1):
            disc += S[kk - 1] ** 2
            if disc >= threshold:
                keep = max(kk, 2)
                break
        if max_bond_dim is not None:
            keep = min(keep, max_bond_dim)
        keep = min(keep, len(S))
        err += float(np.sum(S[keep:] ** 2))
        mps.tensors[i] = _f(U[:, :keep], (l, d1, keep))
        mps.tensors[i + 1] = _f(S[:keep, None] * Vh[:keep], (keep, d2, r))
    mps.orth_center = mps.length
    normalize(mps)
    return err


def local_expect(mps: MPS, op, site: int) -> complex:
    """local_expect (MPS.jl:608-624): centre moved to the site, then
    <A| op |A> on its tensor."""
    shift_orthogonality_center(mps, site)
    A = mps.tensors[site - 1]
    return complex(np.einsum("lpr,pq,lqr->", A.conj(), np.asarray(op), A))


def local_expect_two_site(mps: MPS, op, s1: int, s2: int) -> complex:
    """local_expect_two_site (MPS.jl:626-651): adjacent sites only; op is
    4x4 in the p1 + 2 p2 basis."""
    if s2 != s1 + 1:
        raise ValueError("local_expect_two_site needs adjacent sites")
    shift_orthogonality_center(mps, s1)
    A, B = mps.tensors[s1 - 1], mps.tensors[s2 - 1]
    th = np.einsum("lpk,kqr->lpqr", A, B)
    O = np.reshape(np.asarray(op), (2, 2, 2, 2), order="F")  # (p1', p2', p1, p2)
    return complex(np.einsum("lpqr,pqst,lstr->", th.conj(), O, th))


def evaluate_all_local_expectations(mps: MPS, operators) -> np.ndarray:
    """evaluate_all_local_expectations (MPS.jl:658-676): one operator per site."""
    if len(operators) != mps.length:
        raise ValueError("one operator per site")
    shift_orthogonality_center(mps, 1)
    return np.array([local_expect(mps, operators[i], i + 1) for i in range(mps.length)])


def measure_shots(mps: MPS, shots: int, rng=None, uniforms=None) -> dict:
    """measure_shots / single_shot_measure (MPS.jl:683-749): projective
    measurement of every site in turn from the centre at site 1, outcome k
    of site i with probability ||A_i[:, k, :]||^2 given the earlier outcomes
    (the first k whose cumulative probability reaches the draw), the
    projected slice renormalised into site i+1.  Bitstrings are integers
    with site i as bit i-1.  All shots advance together; ``uniforms``
    (shots x L, the draws in the reference's order) replaces the generator."""
    psi = shift_orthogonality_center(copy.deepcopy(mps), 1)
    L = psi.length
    if uniforms is None:
        rng = np.random.default_rng() if rng is None else rng
        uniforms = rng.random((shots, L))
    uniforms = np.asarray(uniforms, dtype=np.float64)
    v = np.ones((shots, 1), dtype=np.complex128)  # per shot, the left boundary vector
    bits = np.zeros(shots, dtype=np.int64)
    for i in range(L):
        A = psi.tensors[i]
        d = A.shape[1]
        w = np.einsum("sl,lpr->spr", v, A)  # (shots, d, r)
        probs = np.sum(np.abs(w) ** 2, axis=2)
        acc = np.cumsum(probs, axis=1)
        hit = uniforms[:, i:i + 1] <= acc
        chosen = np.where(hit.any(axis=1), hit.argmax(axis=1), d - 1)
        bits += chosen.astype(np.int64) << i
        if i < L - 1:
            pr = probs[np.arange(shots), chosen]
            scale = np.where(np.sqrt(pr) > 1e-12, 1.0 / np.sqrt(np.maximum(pr, 1e-300)), 1.0)
            v = w[np.arange(shots), chosen, :] * scale[:, None]
    counts: dict = {}
    for b in bits.tolist():
        counts[b] = counts.get(b, 0) + 1
    return counts


def single_shot_measure(mps: MPS, rng=None, uniforms=None) -> int:
    """One shot as an integer bitstring (MPS.jl:683-737)."""
    (b,) = measure_shots(mps, 1, rng=rng, uniforms=None if uniforms is None else np.reshape(uniforms, (1, -1)))
    return int(b)


measure_single_shot = single_shot_measure


def project_onto_bitstring(mps: MPS, bitstring: str) -> float:
    """|<bitstring|psi>|^2 with bitstring[i] the outcome of site i+1 (MPS.jl:751-764)."""
    vec = np.ones(1, dtype=np.complex128)
    for i, ch in enumerate(bitstring):
        vec = vec @ mps.tensors[i][:, int(ch), :]
    return float(abs(vec[0]) ** 2)


# ---------------------------------------------------------------------------
# MPO algebra (src/MPO.jl:44-87, 271-556)
# ---------------------------------------------------------------------------
def mpo_identity(length: int) -> MPO:
    """MPO(length; identity=true) (MPO.jl:55-87)."""
    return MPO(length, [np.eye(2, dtype=np.complex128).reshape(1, 2, 2, 1) for _ in range(length)])


def mpo_zero(length: int) -> MPO:
    """MPO(length) with zero tensors (MPO.jl:80-86)."""
    return MPO(length, [np.zeros((1, 2, 2, 1), dtype=np.complex128) for _ in range(length)])


def orthogonalize(mpo: MPO, new_center: int) -> MPO:
    """orthogonalize! (MPO.jl:271-331): QR from site 1 up to the centre and
    LQ from site L down to it, with (out, in) as one physical index."""
    for i in range(new_center - 1):
        A = mpo.tensors[i]
        l, po, pi, r = A.shape
        Q, R = _qr(_f(A, (l * po * pi, r)))
        rn = R.shape[0]
        mpo.tensors[i] = np.asfortranarray(_f(Q, (l, po, pi, rn)))
        N = mpo.tensors[i + 1]
        mpo.tensors[i + 1] = np.asfortranarray(_f(R @ _f(N, (r, -1)), (rn,) + N.shape[1:]))
    for i in range(mpo.length - 1, new_center - 1, -1):
        A = mpo.tensors[i]
        l, po, pi, r = A.shape
        Lm, Q = _lq(_f(A, (l, po * pi * r)))
        rn = Lm.shape[1]
        mpo.tensors[i] = np.asfortranarray(_f(Q, (rn, po, pi, r)))
        P = mpo.tensors[i - 1]
        mpo.tensors[i - 1] = np.asfortranarray(_f(_f(P, (-1, l)) @ Lm, P.shape[:3] + (rn,)))
    mpo.orth_center = new_center
    return mpo


def mpo_truncate(mpo: MPO, threshold: float = 1e-12, max_bond_dim: int | None = None) -> float:
    """MPO truncate! (MPO.jl:338-400): centre to site 1, one SVD sweep with
    the relative rule (discard from the smallest while the discarded weight
    is at most threshold times the total, at least 1 kept), at most
    max_bond_dim.  Returns the discarded weight."""
    orthogonalize(mpo, 1)
    err = 0.0
    for i in range(mpo.length - 1):
        A, B = mpo.tensors[i], mpo.tensors[i + 1]
        l, po1, pi1, k = A.shape
        _, po2, pi2, r = B.shape
        theta = _f(A, (l * po1 * pi1, k)) @ _f(B, (k, po2 * pi2 * r))
        U, S, Vh = np.linalg.svd(theta, full_matrices=False)
        nsq = float(S @ S)
        keep, csum = len(S), 0.0
        for idx in range(len(S), 0, -1):
            csum += S[idx - 1] ** 2
            if csum > threshold * nsq:
                keep = idx
                break
            if idx == 1:
                keep = 1
        if max_bond_dim is not None:
            keep = min(keep, max_bond_dim)
        err += float(np.sum(S[keep:] ** 2))
        mpo.tensors[i] = np.asfortranarray(_f(U[:, :keep], (l, po1, pi1, keep)))
        mpo.tensors[i + 1] = np.asfortranarray(_f(S[:keep, None] * Vh[:keep], (keep, po2, pi2, r)))
    mpo.orth_center = mpo.length
    return err


def contract_mpo_mps(w: MPO, psi: MPS) -> MPS:
    """W|psi> as an MPS with the bonds multiplied, (W bond, MPS bond) merged
    with the W index fastest (MPO.jl:407-432)."""
    if w.length != psi.length:
        raise ValueError("length mismatch")
    out = []
    for W, A in zip(w.tensors, psi.tensors):
        C = np.einsum("wpkv,akb->wapvb", W, A)
        lw, la, p, rw, ra = C.shape
        out.append(np.asfortranarray(_f(C, (lw * la, p, rw * ra))))
    res = MPS(psi.length, tensors=out)
    res.orth_center = 0
    return res


def expect_mpo(w: MPO, psi: MPS) -> complex:
    """<psi|W|psi> by one left-to-right environment sweep (MPO.jl:442-479)."""
    E = np.ones((1, 1, 1), dtype=np.complex128)
    for W, A in zip(w.tensors, psi.tensors):
        T1 = np.einsum("bwc,cir->bwir", E, A)
        T2 = np.einsum("bwir,woiv->brov", T1, W)
        E = np.einsum("brov,bos->svr", T2, A.conj())
    return complex(E[0, 0, 0])


def mpo_add(a: MPO, b: MPO) -> MPO:
    """a + b by the direct sum of bonds (MPO.jl:486-521): row [A B] at the
    first site, column [A; B] at the last, block diagonal between.  A chain
    of one site adds the tensors."""
    if a.length != b.length:
        raise ValueError("length mismatch")
    L = a.length
    if L == 1:
        return MPO(1, [a.tensors[0] + b.tensors[0]])
    out = []
    for i, (A, B) in enumerate(zip(a.tensors, b.tensors)):
        la, po, pi, ra = A.shape
        lb, _, _, rb = B.shape
        if i == 0:
            C = np.zeros((1, po, pi, ra + rb), dtype=np.complex128)
            C[0, :, :, :ra] = A[0]
            C[0, :, :, ra:] = B[0]
        elif i == L - 1:
            C = np.zeros((la + lb, po, pi, 1), dtype=np.complex128)
            C[:la, :, :, 0] = A[..., 0]
            C[la:, :, :, 0] = B[..., 0]
        else:
            C = np.zeros((la + lb, po, pi, ra + rb), dtype=np.complex128)
            C[:la, :, :, :ra] = A
            C[la:, :, :, ra:] = B
        out.append(C)
    return MPO(L, out)


def mpo_scale(c: complex, mpo: MPO) -> MPO:
    """c * mpo: the first tensor scaled (MPO.jl:523-529)."""
    ts = [t.copy() for t in mpo.tensors]
    ts[0] = c * ts[0]
    out = MPO(mpo.length, ts)
    out.orth_center = mpo.orth_center
    return out


def contract_mpo_mpo(a: MPO, b: MPO) -> MPO:
    """a * b (a acting after b): a's input contracted with b's output, bonds
    merged with a's index fastest (MPO.jl:536-556)."""
    if a.length != b.length:
        raise ValueError("length mismatch")
    out = []
    for A, B in zip(a.tensors, b.tensors):
        C = np.einsum("aokr,bkis->aboirs", A, B)
        la, lb, po, pi, ra, rb = C.shape
        out.append(np.asfortranarray(_f(C, (la * lb, po, pi, ra * rb))))
    return MPO(a.length, out)


# ---------------------------------------------------------------------------
# Measurement configs (src/SimulationConfigs.jl:42-56, 95-208)
# ---------------------------------------------------------------------------
class MeasurementConfig:
    """MeasurementConfig (shots): per-shot outcome tallies and their sum."""

    def __init__(self, shots: int, max_bond_dim: int = 4096, min_bond_dim: int = 2,
                 truncation_threshold: float = 1e-9):
        self.shots = int(shots)
        self.max_bond_dim = int(max_bond_dim)
        self.min_bond_dim = int(min_bond_dim)
        self.truncation_threshold = float(truncation_threshold)
        self.measurements: list = [None] * self.shots
        self.results: dict = {}


def aggregate_measurements(config: MeasurementConfig) -> dict:
    """aggregate_measurements! (SimulationConfigs.jl:198-208): the per-shot
    tallies summed (unfilled entries skipped)."""
    total: dict = {}
    for res in config.measurements:
        if res is None:
            continue
        for k, v in res.items():
            total[k] = total.get(k, 0) + v
    config.results = total
    return total


class StrongMeasurementConfig:
    """StrongMeasurementConfig (trajectories): observables averaged over
    num_traj trajectories."""

    def __init__(self, observables, num_traj: int = 1000, max_bond_dim: int = 4096, min_bond_dim: int = 2,
                 truncation_threshold: float = 1e-9, sample_layers: bool = False):
        self.observables: list[Observable] = list(observables)
        self.num_traj = int(num_traj)
        self.max_bond_dim = int(max_bond_dim)
        self.min_bond_dim = int(min_bond_dim)
        self.truncation_threshold = float(truncation_threshold)
        self.sample_layers = bool(sample_layers)


def expect(mps: MPS, obs: Observable) -> float:
    """expect(psi, obs) (SimulationConfigs.jl:42-56): the real part of
    local_expect for a 1-site observable, of local_expect_two_site on the
    sorted pair for a 2-site one; more sites are an error, as there."""
    if obs.op is None:
        raise ValueError("expect needs an operator observable")
    if len(obs.sites) == 1:
        return float(local_expect(mps, obs.op, obs.sites[0]).real)
    if len(obs.sites) == 2:
        s1, s2 = sorted(obs.sites)
        return float(local_expect_two_site(mps, obs.op, s1, s2).real)
    raise ValueError("multi-site expectation is not implemented (as in the reference)")


def initialize_observable(obs: Observable, config, num_layers: int = 0) -> None:
    """initialize! (SimulationConfigs.jl:146-160): zeroed buffers for one
    observable.  A TimeEvolutionConfig gets len(times) columns when it
    samples every time step, else 1; a StrongMeasurementConfig gets
    num_layers + 1 columns when it samples layers, else 1."""
    if isinstance(config, StrongMeasurementConfig):
        n = num_layers + 1 if config.sample_layers else 1
    else:
        n = len(config.times) if config.sample_timesteps else 1
    obs.trajectories = np.zeros((config.num_traj, n), dtype=np.complex128)
    obs.results = np.zeros(n)


def aggregate_trajectories(config) -> None:
    """aggregate_trajectories! (SimulationConfigs.jl:168-190) for either
    config: results = sum of the real parts over trajectories / num_traj,
    for every observable that has trajectories."""
    for o in config.observables:
        tr = getattr(o, "trajectories", None)
        if tr is not None and np.size(tr):
            o.results = np.real(np.asarray(tr)).sum(axis=0) / config.num_traj


def aggregate_strong(config: StrongMeasurementConfig) -> None:
    """aggregate_trajectories! for StrongMeasurementConfig
    (SimulationConfigs.jl:182-190): results = sum of the real parts over
    trajectories / num_traj, for observables with trajectories."""
    for o in config.observables:
        tr = getattr(o, "trajectories", None)
        if tr is not None and np.size(tr):
            o.results = np.real(np.asarray(tr)).sum(axis=0) / config.num_traj
