"""ctypes front of the C++ FP64 oracle (oracle/tjm_oracle.cpp).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py as the checker.  It takes the same C-ABI
descriptors as the product library (include/yaqs_tjm.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from yaqs_julia_b200 import _abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle_tjm.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ only)."""
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
            os.path.join(_HERE, "tjm_oracle.cpp")):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        P = C.POINTER
        L.orc_analog_run.argtypes = [P(A.MpsDesc), P(A.MpoDesc), P(A.NoiseDesc), P(A.ObsDesc), C.c_int32,
                                     P(A.TevConfig), P(A.RngDesc), C.c_int32, C.c_int32, C.c_int32,
                                     A.DPTR, P(C.c_int32), P(A.RunStats)]
        L.orc_digital_run.argtypes = [P(A.MpsDesc), P(A.GateDesc), C.c_int32, P(A.NoiseDesc), P(A.ObsDesc),
                                      C.c_int32, P(A.CircuitConfig), P(A.RngDesc), C.c_int32, C.c_int32,
                                      C.c_int32, A.DPTR, P(C.c_int32), P(A.RunStats)]
        L.orc_digital_plan.argtypes = [P(A.GateDesc), C.c_int32, P(C.c_int32), P(C.c_int32)]
        L.orc_tdvp_evolve.argtypes = [P(A.MpsDesc), P(A.MpoDesc), P(A.ObsDesc), C.c_int32, P(A.TevConfig),
                                      C.c_int32, A.DPTR]
        L.orc_tdvp_overlap.argtypes = [P(A.MpsDesc), P(A.MpoDesc), P(A.TevConfig), C.c_int32, A.DPTR]
        L.orc_stochastic_factor.argtypes = [P(A.MpsDesc), A.DPTR]
        L.orc_probability_distribution.argtypes = [P(A.MpsDesc), P(A.MpoDesc), P(A.NoiseDesc), P(A.TevConfig),
                                                   C.c_double, C.c_int32, A.DPTR, P(C.c_int32), P(C.c_int32),
                                                   P(C.c_int32)]
        L.orc_apply_dissipation.argtypes = [P(A.MpsDesc), P(A.MpoDesc), P(A.NoiseDesc), P(A.TevConfig),
                                            C.c_int32, C.c_int64, A.DPTR, P(C.c_int32), P(C.c_int32)]
        L.orc_svd.argtypes = [C.c_int32, C.c_int32, A.DPTR, A.DPTR, A.DPTR, A.DPTR]
        L.orc_qr.argtypes = [C.c_int32, C.c_int32, A.DPTR, A.DPTR, A.DPTR]
        L.orc_truncation_rank.argtypes = [C.c_int32, A.DPTR, C.c_double, C.c_int32, C.c_int32]
        L.orc_truncation_rank.restype = C.c_int32
        L.orc_expm_site.argtypes = [C.c_int32] * 5 + [A.DPTR] * 4 + [C.c_double, C.c_int32, C.c_double,
                                                                    C.c_double, A.DPTR, P(C.c_int32)]
        L.orc_project_site.argtypes = [C.c_int32] * 5 + [A.DPTR] * 5
        L.orc_philox_uniform.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.orc_philox_uniform.restype = C.c_double
        L.orc_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def _check(st):
    if st != A.YAQS_OK:
        raise RuntimeError(f"oracle: {A.STATUS_NAMES.get(st, st)}: {lib().orc_last_error().decode()}")


def analog_run(desc, t_begin=0, t_end=None, nthreads=None):
    """Run trajectories [t_begin, t_end) of a packed problem (api.Descriptors).
    Returns (traj [num_traj, n_obs, n_out], maxchi [num_traj, n_out], stats)."""
    L = lib()
    nt = desc.num_traj
    t_end = nt if t_end is None else t_end
    traj = np.zeros((nt, max(desc.n_obs, 1), desc.n_out))
    chi = np.zeros((nt, desc.n_out), dtype=np.int32)
    st = A.RunStats()
    nth = nthreads or os.cpu_count() or 1
    _check(L.orc_analog_run(C.byref(desc.mps), C.byref(desc.mpo), C.byref(desc.noise), desc.obs, desc.n_obs,
                            C.byref(desc.cfg), C.byref(desc.rng), t_begin, t_end, nth, A.dptr(traj),
                            chi.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(st)))
    return traj[:, :desc.n_obs, :], chi, st.as_dict()


_blas = {}


def openblas_zgemm():
    """The OpenBLAS that scipy ships (the reference's LinearAlgebra backend is
    OpenBLAS as well, Manifest.toml), set to one thread per caller: returns
    (address of its cblas_zgemm, description), or (None, reason)."""
    if "fn" in _blas:
        return _blas["fn"], _blas["desc"]
    import glob

    import scipy
    libdir = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas-*.so")))
    if not cands:
        _blas.update(fn=None, desc="scipy's OpenBLAS not found")
        return None, _blas["desc"]
    ob = C.CDLL(cands[0])
    ob.scipy_openblas_set_num_threads.argtypes = [C.c_int]
    ob.scipy_openblas_set_num_threads(1)  # trajectories run one per host thread
    fn = C.cast(ob.scipy_cblas_zgemm, C.c_void_p).value
    ver = ""
    if hasattr(ob, "scipy_openblas_get_config"):
        ob.scipy_openblas_get_config.restype = C.c_char_p
        ver = ob.scipy_openblas_get_config().decode().split()[1] if ob.scipy_openblas_get_config() else ""
    _blas.update(fn=fn, desc=f"OpenBLAS {ver} cblas_zgemm (scipy's build), 1 thread per trajectory", lib=ob)
    return fn, _blas["desc"]


def set_blas(enabled: bool):
    """Routes the oracle's contractions through OpenBLAS zgemm (enabled) or
    back to its plain loops.  Returns the description of what is in use."""
    L = lib()
    L.orc_set_zgemm.restype = C.c_void_p
    L.orc_set_zgemm.argtypes = [C.c_void_p]
    if not enabled:
        L.orc_set_zgemm(None)
        return "plain loops"
    fn, desc = openblas_zgemm()
    L.orc_set_zgemm(fn)
    return desc if fn else "plain loops (" + desc + ")"


def digital_run(desc, t_begin=0, t_end=None, nthreads=None):
    """Digital trajectories of a packed circuit problem (api.CircuitDescriptors)."""
    L = lib()
    nt = desc.num_traj
    t_end = nt if t_end is None else t_end
    traj = np.zeros((nt, max(desc.n_obs, 1), desc.n_out))
    chi = np.zeros((nt, desc.n_out), dtype=np.int32)
    st = A.RunStats()
    nth = nthreads or os.cpu_count() or 1
    _check(L.orc_digital_run(C.byref(desc.mps), desc.gates, desc.n_gates, C.byref(desc.noise), desc.obs,
                             desc.n_obs, C.byref(desc.cfg), C.byref(desc.rng), t_begin, t_end, nth, A.dptr(traj),
                             chi.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(st)))
    return traj[:, :desc.n_obs, :], chi, st.as_dict()


def digital_plan(gates, n_gates):
    """(n_layers, n_samples) of a yaqs_gate_desc array (process_circuit / _sample_plan)."""
    nl, ns = C.c_int32(0), C.c_int32(0)
    _check(lib().orc_digital_plan(gates, n_gates, C.byref(nl), C.byref(ns)))
    return nl.value, ns.value


def tdvp_evolve(desc, n_steps):
    out = np.zeros((n_steps + 1, max(desc.n_obs, 1)))
    _check(lib().orc_tdvp_evolve(C.byref(desc.mps), C.byref(desc.mpo), desc.obs, desc.n_obs, C.byref(desc.cfg),
                                 n_steps, A.dptr(out)))
    return out[:, :desc.n_obs]


def tdvp_overlap(desc, n_steps) -> complex:
    """scalar_product(psi(t), psi0) in the reference's convention after
    n_steps noise-free sweeps of the configured TDVP mode."""
    out = np.zeros(2)
    _check(lib().orc_tdvp_overlap(C.byref(desc.mps), C.byref(desc.mpo), C.byref(desc.cfg), n_steps,
                                  A.dptr(out)))
    return complex(out[0], out[1])


def stochastic_factor(desc) -> float:
    """calculate_stochastic_factor of the packed initial state, as given."""
    out = np.zeros(1)
    _check(lib().orc_stochastic_factor(C.byref(desc.mps), A.dptr(out)))
    return float(out[0])


CANDIDATE_TYPES = ("local_1", "local_2", "pauli_long_range", "mpo_general")


def probability_distribution(desc, dt):
    """create_probability_distribution on the packed initial state:
    (probabilities, [(type, sites 1-based)]) in the reference's order."""
    cap = max(1, desc.noise.n)  # one candidate per process at most
    probs = np.zeros(cap)
    kinds = np.zeros(cap, dtype=np.int32)
    sites = np.zeros(2 * cap, dtype=np.int32)
    n = C.c_int32(0)
    I32 = C.POINTER(C.c_int32)
    _check(lib().orc_probability_distribution(C.byref(desc.mps), C.byref(desc.mpo), C.byref(desc.noise),
                                              C.byref(desc.cfg), dt, cap, A.dptr(probs),
                                              kinds.ctypes.data_as(I32), sites.ctypes.data_as(I32), C.byref(n)))
    k = n.value
    cands = [(CANDIDATE_TYPES[kinds[i]],
              [int(sites[2 * i]) + 1] if kinds[i] == 0 else [int(sites[2 * i]) + 1, int(sites[2 * i + 1]) + 1])
             for i in range(k)]
    return probs[:k], cands


def apply_dissipation(desc, full_dt=True):
    """apply_dissipation on the packed initial state at cfg.dt (or dt/2).
    Returns (tensors as (left, phys, right) arrays, 1-based centre)."""
    L = desc.mps.L
    cap = 4 * L * max(int(desc.mps.chi[i]) for i in range(L + 1)) ** 2 * 2 + 64
    buf = np.zeros(2 * cap)
    chi = np.zeros(L + 1, dtype=np.int32)
    oc = C.c_int32(0)
    _check(lib().orc_apply_dissipation(C.byref(desc.mps), C.byref(desc.mpo), C.byref(desc.noise),
                                       C.byref(desc.cfg), int(full_dt), cap, A.dptr(buf),
                                       chi.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(oc)))
    z = buf.view(np.complex128)
    out, o = [], 0
    for i in range(L):
        n = chi[i] * 2 * chi[i + 1]
        out.append(np.reshape(z[o:o + n], (chi[i], 2, chi[i + 1]), order="F").copy())
        o += n
    return out, oc.value + 1


def svd(M):
    M = np.asfortranarray(M, dtype=np.complex128)
    m, n = M.shape
    k = min(m, n)
    U = np.zeros((m, k), dtype=np.complex128, order="F")
    Vt = np.zeros((k, n), dtype=np.complex128, order="F")
    S = np.zeros(k)
    _check(lib().orc_svd(m, n, A.dptr(M.reshape(-1, order="F").view(np.float64)),
                         A.dptr(U.reshape(-1, order="F").view(np.float64)), A.dptr(S),
                         A.dptr(Vt.reshape(-1, order="F").view(np.float64))))
    return U, S, Vt


def qr(M):
    M = np.asfortranarray(M, dtype=np.complex128)
    m, n = M.shape
    k = min(m, n)
    Q = np.zeros((m, k), dtype=np.complex128, order="F")
    R = np.zeros((k, n), dtype=np.complex128, order="F")
    _check(lib().orc_qr(m, n, A.dptr(M.reshape(-1, order="F").view(np.float64)),
                        A.dptr(Q.reshape(-1, order="F").view(np.float64)),
                        A.dptr(R.reshape(-1, order="F").view(np.float64))))
    return Q, R


def truncation_rank(S, thr, max_bond, rule):
    S = np.ascontiguousarray(S, dtype=np.float64)
    return lib().orc_truncation_rank(S.size, A.dptr(S), thr, max_bond, rule)


def _fbuf(a):
    return np.asfortranarray(a, dtype=np.complex128).reshape(-1, order="F").view(np.float64)


def project_site(Lenv, Renv, W, x):
    chil, wl, _ = Lenv.shape
    chir, wr, _ = Renv.shape
    D = W.shape[1]
    out = np.zeros((chil, D, chir), dtype=np.complex128, order="F")
    bl, br, bw, bx = _fbuf(Lenv), _fbuf(Renv), _fbuf(W), _fbuf(x)
    _check(lib().orc_project_site(chil, D, chir, wl, wr, A.dptr(bl), A.dptr(br), A.dptr(bw), A.dptr(bx),
                                  A.dptr(out.reshape(-1, order="F").view(np.float64))))
    return out


def expm_site(Lenv, Renv, W, x, dt, kdim=25, tol=1e-10, exit_tol=0.0):
    chil, wl, _ = Lenv.shape
    chir, wr, _ = Renv.shape
    D = W.shape[1]
    out = np.zeros((chil, D, chir), dtype=np.complex128, order="F")
    mv = C.c_int32(0)
    bl, br, bw, bx = _fbuf(Lenv), _fbuf(Renv), _fbuf(W), _fbuf(x)
    _check(lib().orc_expm_site(chil, D, chir, wl, wr, A.dptr(bl), A.dptr(br), A.dptr(bw), A.dptr(bx), dt, kdim,
                               tol, exit_tol, A.dptr(out.reshape(-1, order="F").view(np.float64)), C.byref(mv)))
    return out, mv.value


def philox_uniform(seed, stream, draw):
    return lib().orc_philox_uniform(seed, stream, draw)
