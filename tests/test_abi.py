"""The C-ABI library builds, loads and exports every declared symbol (CPU only, no device calls)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"^\s*(?:int|const char\*|double)\s+(yaqs_\w+)\s*\(", src, flags=re.M))
    return names


def test_header_declares_entry_points():
    names = _declared()
    assert {"yaqs_analog_run", "yaqs_ctx_create", "yaqs_batched_svd", "yaqs_batched_expm_site"} <= names


# The C-ABI surface as the bindings (yaqs_julia_b200/_lib.py) and the Julia
# shim know it; a new or removed declaration must be added here too.
ENTRY_POINTS = {
    "yaqs_version", "yaqs_last_error", "yaqs_ctx_create", "yaqs_ctx_destroy", "yaqs_mpo_hermitian_defect",
    "yaqs_analog_run", "yaqs_analog_begin", "yaqs_analog_advance", "yaqs_analog_remaining", "yaqs_analog_stats",
    "yaqs_analog_profile", "yaqs_analog_finish", "yaqs_run_state", "yaqs_run_position", "yaqs_run_rng",
    "yaqs_run_restore", "yaqs_run_seek", "yaqs_digital_plan", "yaqs_digital_begin", "yaqs_digital_run",
    "yaqs_server_create", "yaqs_server_submit_analog", "yaqs_server_submit_digital", "yaqs_server_poll",
    "yaqs_server_wait", "yaqs_server_take", "yaqs_server_last_error", "yaqs_server_stats_get",
    "yaqs_server_destroy", "yaqs_batched_svd", "yaqs_batched_qr", "yaqs_batched_project_site",
    "yaqs_batched_expm_site", "yaqs_batched_cgemm_tf32", "yaqs_batched_svd_noalloc", "yaqs_fp64_peak",
    "yaqs_autotune_results",
}


def test_headers_declare_exactly_the_bound_entry_points():
    """The headers declare the entry points the bindings know, no more, no fewer."""
    names = _declared()
    assert names == ENTRY_POINTS, (sorted(names - ENTRY_POINTS), sorted(ENTRY_POINTS - names))


def test_bindings_set_argtypes_for_every_entry_point():
    """Every entry point taking arguments has its ctypes signature in _lib.py."""
    src = open(os.path.join(ROOT, "yaqs_julia_b200", "_lib.py")).read()
    missing = sorted(n for n in ENTRY_POINTS if n != "yaqs_version" and f"L.{n}." not in src)
    assert not missing, missing


def test_library_exports_every_declared_symbol():
    from yaqs_julia_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("engine not built")
    lib = C.CDLL(_lib.LIB_PATH)
    for n in sorted(_declared()):
        assert hasattr(lib, n), n
    assert b"sm_100a" in _lib.lib().yaqs_version()


def test_abi_struct_layouts_match_header(tmp_path):
    """ctypes mirrors match the C compiler's sizeof/offsetof for every struct."""
    import shutil
    import subprocess
    from yaqs_julia_b200 import _abi as A
    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    structs = {"yaqs_mps_desc": A.MpsDesc, "yaqs_mpo_desc": A.MpoDesc, "yaqs_noise_proc": A.NoiseProc,
               "yaqs_noise_desc": A.NoiseDesc, "yaqs_obs_desc": A.ObsDesc, "yaqs_rng_desc": A.RngDesc,
               "yaqs_tev_config": A.TevConfig, "yaqs_run_stats": A.RunStats, "yaqs_gate_desc": A.GateDesc,
               "yaqs_circuit_config": A.CircuitConfig, "yaqs_server_config": A.ServerConfig,
               "yaqs_server_stats": A.ServerStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "yaqs_tjm.h"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split("\n")
               if line)
    for cname, py in structs.items():
        assert int(out[cname]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(out[f"{cname}.{f}"]) == getattr(py, f).offset, (cname, f)


def test_descriptor_validation_host_side():
    from yaqs_julia_b200 import api
    # a long-range process needs a Pauli pair in its name or factors (Noise.jl:399-404)
    with pytest.raises(ValueError, match="Pauli pair"):
        api.NoiseModel([{"name": "pauli_z", "sites": [1, 3], "strength": 0.1}], 4)
    with pytest.raises(ValueError):
        H = api.init_ising(4, 1, 1)
        cfg = api.TimeEvolutionConfig([api.Observable("zz", np.kron(api.Z, api.Z), [1, 3])], 1.0)
        api.Descriptors(api.MPS(4), H, cfg, None)


import numpy as np  # noqa: E402


def _dagger(W):
    from yaqs_julia_b200 import api
    return api.MPO(W.length, [np.conj(np.transpose(t, (0, 2, 1, 3))) for t in W.tensors])


def test_hamiltonian_hermiticity_check():
    """yaqs_mpo_hermitian_defect (host arithmetic, no device) stands in for
    the reference's _ishermitian_check (Algorithms.jl:120-137): zero for the
    library Hamiltonians, their sums and multiples and a Hermitian random
    MPO; the true relative defect for non-Hermitian ones, which runs refuse."""
    from yaqs_julia_b200 import api
    from yaqs_julia_b200 import tensornet as T
    rng = np.random.default_rng(3)
    herm = [api.init_ising(30, 1.0, 0.5), api.init_ising(6, [0.6, 1.2, 0.8, 1.4, 0.9], [0.7, 1.3, 0.5, 1.1, 0.8, 1.2]),
            api.init_general_hamiltonian(12, 0.3, -1.2, 0.7, 0.4, 0.9, -0.2), T.mpo_identity(5), T.mpo_zero(4),
            api.init_ising(8, 1, 0) + api.init_ising(8, 0, 1), 2.5 * api.init_general_hamiltonian(256, 1, 1, 1, 0, 0, 0.3)]
    W = api.MPO(5, [rng.normal(size=(1 if i == 0 else 3, 2, 2, 1 if i == 4 else 3)) +
                    1j * rng.normal(size=(1 if i == 0 else 3, 2, 2, 1 if i == 4 else 3)) for i in range(5)])
    herm.append(W + _dagger(W))
    for H in herm:
        assert api.hermitian_defect(H) < 1e-7
    # non-Hermitian: i H, a random MPO, a small anti-Hermitian admixture; dense check of the value
    for H in (1j * api.init_ising(6, 1, 0.5), W, (1 + 1e-3j) * (W + _dagger(W))):
        M = H.to_matrix()
        ref = np.linalg.norm(M - M.conj().T) / np.linalg.norm(M)
        assert abs(api.hermitian_defect(H) - ref) <= 1e-6 * max(ref, 1.0) + 1e-7
        assert ref > 1e-5


def test_descriptors_refuse_non_hermitian_hamiltonians():
    """The host check (numpy) equals the library's, and Descriptors refuses a
    Hamiltonian above the tolerance before anything reaches the device."""
    from yaqs_julia_b200 import api
    rng = np.random.default_rng(5)
    W = api.MPO(4, [rng.normal(size=(1 if i == 0 else 2, 2, 2, 1 if i == 3 else 2)) +
                    1j * rng.normal(size=(1 if i == 0 else 2, 2, 2, 1 if i == 3 else 2)) for i in range(4)])
    for H in (api.init_ising(10, 1, 0.5), W + _dagger(W), W, 1j * api.init_ising(4, 1, 0.2)):
        assert abs(api.mpo_antihermitian_part(H) - api.hermitian_defect(H)) < 1e-7
    cfg = api.TimeEvolutionConfig([api.Observable("Z1", api.Z, 1)], 0.2, dt=0.1, num_traj=1, max_bond_dim=4)
    with pytest.raises(ValueError, match="not Hermitian"):
        api.Descriptors(api.MPS(4), W, cfg, None)
    api.Descriptors(api.MPS(4), W + _dagger(W), cfg, None)
