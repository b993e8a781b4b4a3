"""Loads the engine's C-ABI library (libyaqs_b200.so, built in-tree).

There is no fallback: if the library is missing or no CUDA device is
visible, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libyaqs_b200.so")
_lib = None


class EngineError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{A.STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EngineError(A.YAQS_E_CUDA, f"{LIB_PATH} is not built (run __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        L.yaqs_version.restype = C.c_char_p
        L.yaqs_last_error.restype = C.c_char_p
        L.yaqs_last_error.argtypes = [C.c_void_p]
        L.yaqs_ctx_create.argtypes = [C.c_int32, P(C.c_void_p)]
        L.yaqs_ctx_destroy.argtypes = [C.c_void_p]
        L.yaqs_analog_run.argtypes = [C.c_void_p, P(A.MpsDesc), P(A.MpoDesc), P(A.NoiseDesc), P(A.ObsDesc),
                                      C.c_int32, P(A.TevConfig), P(A.RngDesc), A.DPTR, A.DPTR, P(C.c_int32),
                                      P(A.RunStats)]
        L.yaqs_analog_begin.argtypes = [C.c_void_p, P(A.MpsDesc), P(A.MpoDesc), P(A.NoiseDesc), P(A.ObsDesc),
                                        C.c_int32, P(A.TevConfig), P(A.RngDesc), P(C.c_void_p)]
        L.yaqs_analog_advance.argtypes = [C.c_void_p, C.c_int32, P(C.c_double)]
        L.yaqs_analog_remaining.argtypes = [C.c_void_p]
        L.yaqs_analog_profile.argtypes = [C.c_void_p, A.DPTR]
        L.yaqs_analog_stats.argtypes = [C.c_void_p, P(A.RunStats)]
        L.yaqs_run_state.argtypes = [C.c_void_p, C.c_int32, P(C.c_int32), P(C.c_int32), P(C.c_double), C.c_int64,
                                     P(C.c_int64)]
        L.yaqs_run_position.argtypes = [C.c_void_p, P(C.c_int32)]
        L.yaqs_run_rng.argtypes = [C.c_void_p, C.c_int32, P(C.c_int64)]
        L.yaqs_run_restore.argtypes = [C.c_void_p, C.c_int32, P(C.c_int32), C.c_int32, P(C.c_double), C.c_int64]
        L.yaqs_run_seek.argtypes = [C.c_void_p, C.c_int32]
        L.yaqs_analog_finish.argtypes = [C.c_void_p, A.DPTR, A.DPTR, P(C.c_int32), P(A.RunStats)]
        L.yaqs_digital_plan.argtypes = [P(A.GateDesc), C.c_int32, P(C.c_int32), P(C.c_int32)]
        L.yaqs_mpo_hermitian_defect.argtypes = [P(A.MpoDesc), P(C.c_double)]
        L.yaqs_digital_run.argtypes = [C.c_void_p, P(A.MpsDesc), P(A.GateDesc), C.c_int32, P(A.NoiseDesc),
                                       P(A.ObsDesc), C.c_int32, P(A.CircuitConfig), P(A.RngDesc), A.DPTR, A.DPTR,
                                       P(C.c_int32), P(A.RunStats)]
        L.yaqs_digital_begin.argtypes = [C.c_void_p, P(A.MpsDesc), P(A.GateDesc), C.c_int32, P(A.NoiseDesc),
                                         P(A.ObsDesc), C.c_int32, P(A.CircuitConfig), P(A.RngDesc), P(C.c_void_p)]
        L.yaqs_server_create.argtypes = [C.c_void_p, P(A.ServerConfig), P(C.c_void_p)]
        L.yaqs_server_submit_analog.argtypes = [C.c_void_p, P(A.MpsDesc), P(A.MpoDesc), P(A.NoiseDesc),
                                                P(A.ObsDesc), C.c_int32, P(A.TevConfig), P(A.RngDesc),
                                                P(C.c_int64)]
        L.yaqs_server_submit_digital.argtypes = [C.c_void_p, P(A.MpsDesc), P(A.GateDesc), C.c_int32,
                                                 P(A.NoiseDesc), P(A.ObsDesc), C.c_int32, P(A.CircuitConfig),
                                                 P(A.RngDesc), P(C.c_int64)]
        L.yaqs_server_poll.argtypes = [C.c_void_p, C.c_int64, P(C.c_int32)]
        L.yaqs_server_wait.argtypes = [C.c_void_p, C.c_int64, C.c_double]
        L.yaqs_server_take.argtypes = [C.c_void_p, C.c_int64, A.DPTR, A.DPTR, P(C.c_int32), P(A.RunStats),
                                       A.DPTR]
        L.yaqs_server_last_error.argtypes = [C.c_void_p]
        L.yaqs_server_last_error.restype = C.c_char_p
        L.yaqs_server_stats_get.argtypes = [C.c_void_p, P(A.ServerStats)]
        L.yaqs_server_destroy.argtypes = [C.c_void_p]
        L.yaqs_fp64_peak.argtypes = [C.c_void_p, P(C.c_double)]
        L.yaqs_autotune_results.argtypes = [C.c_void_p, A.DPTR, C.c_int32, P(C.c_int32)]
        L.yaqs_batched_svd_noalloc.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32] + [A.DPTR] * 4 + [
            C.c_void_p]
        L.yaqs_batched_svd.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32] + [A.DPTR] * 4
        L.yaqs_batched_qr.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32] + [A.DPTR] * 3
        L.yaqs_batched_project_site.argtypes = [C.c_void_p] + [C.c_int32] * 6 + [A.DPTR] * 5
        FPTR = P(C.c_float)
        L.yaqs_batched_cgemm_tf32.argtypes = ([C.c_void_p] + [C.c_int32] * 4 + [FPTR, C.c_int32, C.c_int32, FPTR,
                                              C.c_int32, C.c_int32, FPTR])
        L.yaqs_batched_expm_site.argtypes = ([C.c_void_p] + [C.c_int32] * 6 + [A.DPTR] * 4 +
                                             [C.c_double, C.c_int32, C.c_double, C.c_double, A.DPTR,
                                              P(C.c_int32)])
        _lib = L
    return _lib


class Context:
    """A device context (yaqs_ctx).  Use one per thread."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        h = C.c_void_p()
        st = self._lib.yaqs_ctx_create(device, C.byref(h))
        if st != A.YAQS_OK:
            raise EngineError(st, self._lib.yaqs_last_error(None).decode())
        self.handle = h

    def check(self, st):
        if st != A.YAQS_OK:
            raise EngineError(st, self._lib.yaqs_last_error(self.handle).decode())

    def close(self):
        if self.handle:
            self._lib.yaqs_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx
