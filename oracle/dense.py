"""Dense exact solvers for small chains — TEST INFRASTRUCTURE ONLY.

The reference checked its TJM ensembles against QuTiP's mesolve
(00_safety_checks_full_algorithms/analogTJM_check/benchmark_analog_tjm.jl:20-88)
and its TDVP against a dense exp(-iHt) (test/benchmark_tdvp.jl:94-160).
QuTiP is not installed here, so this module restates both with numpy:

* ``schrodinger``: psi(t+dt) = exp(-i dt H) psi(t)
* ``lindblad``: d rho/dt = -i[H, rho] + sum_k (L_k rho L_k^+ - 1/2 {L_k^+ L_k, rho})
  integrated by classical RK4 with ``substeps`` steps per dt.

Basis: site 1 is the fastest index (MPS.to_vec, src/MPS.jl:766-775).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sl


def site_op(op: np.ndarray, site: int, L: int) -> np.ndarray:
    """op acting on 1-based `site` of L qubits, site 1 fastest."""
    M = np.eye(1, dtype=np.complex128)
    for s in range(L, 0, -1):
        M = np.kron(M, op if s == site else np.eye(2))
    return M


def two_site_op(op4: np.ndarray, s1: int, L: int) -> np.ndarray:
    """4x4 op (basis p1 + 2 p2) on sites s1, s1+1."""
    # in the site-1-fastest basis, sites (s1, s1+1) form the factor kron(.., op_{s1+1,s1}, ..)
    left = np.eye(2 ** (L - s1 - 1))
    right = np.eye(2 ** (s1 - 1))
    return np.kron(np.kron(left, op4), right)


def product_state(vectors) -> np.ndarray:
    psi = np.ones(1, dtype=np.complex128)
    for v in reversed(vectors):
        psi = np.kron(psi, np.asarray(v, dtype=np.complex128))
    return psi


def schrodinger(Hm, psi0, dt, steps, observables):
    U = sl.expm(-1j * dt * Hm)
    psi = np.asarray(psi0, dtype=np.complex128)
    out = np.zeros((steps + 1, len(observables)))
    for t in range(steps + 1):
        out[t] = [(psi.conj() @ (O @ psi)).real for O in observables]
        psi = U @ psi
    return out


def lindblad(Hm, psi0, jump_ops, dt, steps, observables, substeps=20):
    """Returns <O>(t_j) for j = 0..steps.  jump_ops already include sqrt(gamma)."""
    rho = np.outer(psi0, np.conj(psi0))
    Ls = [np.asarray(Lk, dtype=np.complex128) for Lk in jump_ops]
    LdL = sum((Lk.conj().T @ Lk for Lk in Ls), np.zeros_like(Hm))
    Heff = Hm - 0.5j * LdL

    def f(r):
        out = -1j * (Heff @ r - r @ Heff.conj().T)
        for Lk in Ls:
            out += Lk @ r @ Lk.conj().T
        return out

    h = dt / substeps
    res = np.zeros((steps + 1, len(observables)))
    for t in range(steps + 1):
        res[t] = [np.trace(O @ rho).real for O in observables]
        if t == steps:
            break
        for _ in range(substeps):
            k1 = f(rho)
            k2 = f(rho + 0.5 * h * k1)
            k3 = f(rho + 0.5 * h * k2)
            k4 = f(rho + h * k3)
            rho = rho + (h / 6.0) * (k1 + 2 * k2 + 2 * k3 + k4)
    return res


def gate_op(op: np.ndarray, sites, L: int) -> np.ndarray:
    """Dense 2^L matrix of a 1-qubit gate, or of a 4x4 gate whose basis index
    is p1 + 2 p2 with p1 the smaller of the two (1-based) sites, as
    apply_local_gate_exact! reads it (DigitalTJM.jl:266-269)."""
    sites = sorted(sites)
    if len(sites) == 1:
        return site_op(op, sites[0], L)
    a, b = sites[0] - 1, sites[1] - 1
    n = 2 ** L
    idx = np.arange(n)
    ba, bb = (idx >> a) & 1, (idx >> b) & 1
    col = ba + 2 * bb
    M = np.zeros((n, n), dtype=np.complex128)
    for row in range(4):
        y = (idx & ~((1 << a) | (1 << b))) | ((row & 1) << a) | ((row >> 1) << b)
        M[y, idx] += op[row, col]
    return M


def digital_pauli_density(L, layers, pauli_procs, observables, psi0=None):
    """Exact ensemble of the digital TJM with Pauli noise.

    ``layers`` is the output of process_circuit (gates with .op and 1-based
    .sites); within a layer the 1-qubit gates act first, then every 2-qubit
    gate followed by the noise of its local model.  For Pauli processes the
    unravelled step (dissipation e^{-gamma/2}, jump with probability
    1 - e^{-Gamma}, process k chosen with weight gamma_k) averages to the
    channel rho -> e^{-Gamma} rho + (1 - e^{-Gamma}) sum_k gamma_k/Gamma P_k rho P_k.
    ``pauli_procs`` is a list of (matrix, 1-based sites, gamma).
    Returns <O> after every layer, shape (n_layers + 1, n_obs), row 0 the start."""
    psi = product_state([[1, 0]] * L) if psi0 is None else psi0
    rho = np.outer(psi, psi.conj())
    out = [[np.trace(O @ rho).real for O in observables]]
    for layer in layers:
        for g in layer:
            if len(g.sites) == 1:
                U = gate_op(g.op, g.sites, L)
                rho = U @ rho @ U.conj().T
        for g in layer:
            if len(g.sites) != 2:
                continue
            U = gate_op(g.op, g.sites, L)
            rho = U @ rho @ U.conj().T
            s = set(g.sites)
            loc = [(gate_op(m, st, L), gm) for (m, st, gm) in pauli_procs
                   if (len(st) == 1 and st[0] in s) or (len(st) == 2 and set(st) == s)]
            G = sum(gm for _, gm in loc)
            if G > 0:
                jumped = sum((gm / G) * (P @ rho @ P.conj().T) for P, gm in loc)
                rho = np.exp(-G) * rho + (1 - np.exp(-G)) * jumped
        out.append([np.trace(O @ rho).real for O in observables])
    return np.array(out)
