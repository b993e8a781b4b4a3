"""ctypes mirror of include/yaqs_tjm.h (the C-ABI of the engine).

Every structure here matches the C declaration field for field; the
descriptors point at caller-owned, column-major, interleaved-complex
buffers exactly as a Julia caller would pass them.
"""
import ctypes as C

YAQS_OK = 0
YAQS_E_ARG = 1
YAQS_E_OOM = 2
YAQS_E_NONFINITE = 3
YAQS_E_NOCONV = 4
YAQS_E_TIMEOUT = 5
YAQS_E_CUDA = 6
YAQS_E_RNG = 7
YAQS_E_UNSUPPORTED = 8

YAQS_OBS_LOCAL1 = 1
YAQS_OBS_LOCAL2 = 2
YAQS_OBS_ENTROPY = 3

YAQS_RNG_PHILOX = 0
YAQS_RNG_INJECTED = 1

YAQS_PREC_FP64 = 0
YAQS_PREC_MIXED = 1
YAQS_TDVP_2SITE, YAQS_TDVP_1SITE, YAQS_TDVP_DYNAMIC = 0, 1, 2

STATUS_NAMES = {
    0: "YAQS_OK", 1: "YAQS_E_ARG", 2: "YAQS_E_OOM", 3: "YAQS_E_NONFINITE",
    4: "YAQS_E_NOCONV", 5: "YAQS_E_TIMEOUT", 6: "YAQS_E_CUDA", 7: "YAQS_E_RNG",
    8: "YAQS_E_UNSUPPORTED",
}

DPTR = C.POINTER(C.c_double)


class MpsDesc(C.Structure):
    _fields_ = [("L", C.c_int32), ("chi", C.POINTER(C.c_int32)),
                ("tensors", C.POINTER(DPTR))]


class MpoDesc(C.Structure):
    _fields_ = [("L", C.c_int32), ("w", C.POINTER(C.c_int32)),
                ("tensors", C.POINTER(DPTR))]


class NoiseProc(C.Structure):
    _fields_ = [("nsites", C.c_int32), ("site", C.c_int32 * 2),
                ("strength", C.c_double), ("matrix", C.c_double * 32),
                ("pauli_name", C.c_int32), ("pauli_proc", C.c_int32)]


class NoiseDesc(C.Structure):
    _fields_ = [("present", C.c_int32), ("n", C.c_int32),
                ("procs", C.POINTER(NoiseProc))]


class ObsDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("site", C.c_int32 * 2),
                ("matrix", C.c_double * 32)]


class RngDesc(C.Structure):
    _fields_ = [("mode", C.c_int32), ("seed", C.c_uint64),
                ("uniforms", DPTR), ("stride", C.c_int64)]


class TevConfig(C.Structure):
    _fields_ = [("dt", C.c_double), ("n_times", C.c_int32),
                ("num_traj", C.c_int32), ("max_bond_dim", C.c_int32),
                ("truncation_threshold", C.c_double), ("order", C.c_int32),
                ("sample_timesteps", C.c_int32), ("krylov_dim", C.c_int32),
                ("krylov_tol", C.c_double), ("krylov_exit_tol", C.c_double),
                ("precision", C.c_int32), ("traj_offset", C.c_int32), ("tdvp_mode", C.c_int32)]


YAQS_GATE_BARRIER = 0
YAQS_GATE_1Q = 1
YAQS_GATE_2Q = 2


class GateDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("site", C.c_int32 * 2), ("matrix", C.c_double * 32),
                ("sample", C.c_int32), ("has_generator", C.c_int32), ("coeff", C.c_double),
                ("gen1", C.c_double * 8), ("gen2", C.c_double * 8)]


class CircuitConfig(C.Structure):
    _fields_ = [("num_traj", C.c_int32), ("max_bond_dim", C.c_int32),
                ("truncation_threshold", C.c_double), ("local_method", C.c_int32),
                ("long_range_method", C.c_int32), ("precision", C.c_int32),
                ("traj_offset", C.c_int32)]


class RunStats(C.Structure):
    _fields_ = [("matvecs", C.c_int64), ("krylov_solves", C.c_int64),
                ("svds", C.c_int64), ("jumps", C.c_int64),
                ("nonfinite_fixes", C.c_int64), ("flops", C.c_double),
                ("device_ms", C.c_double), ("svd_sweeps", C.c_int64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def dptr(a):
    """double* of a C-contiguous float64/complex128 numpy buffer."""
    return a.ctypes.data_as(DPTR)


YAQS_REQ_QUEUED, YAQS_REQ_RUNNING, YAQS_REQ_DONE, YAQS_REQ_FAILED = 0, 1, 2, 3


class ServerConfig(C.Structure):
    _fields_ = [("max_L", C.c_int32), ("max_bond_dim", C.c_int32), ("max_mpo_width", C.c_int32),
                ("krylov_dim", C.c_int32), ("mixed", C.c_int32), ("chunk", C.c_int32), ("hbm_budget", C.c_int64)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64), ("launches", C.c_int64),
                ("queued_now", C.c_int64), ("running_now", C.c_int64), ("bytes_in_use", C.c_int64),
                ("hbm_budget", C.c_int64), ("slots", C.c_int32), ("latency_p50_s", C.c_double),
                ("latency_p99_s", C.c_double), ("queue_p50_s", C.c_double), ("queue_p99_s", C.c_double),
                ("busy_s", C.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}

YAQS_METHOD_TEBD, YAQS_METHOD_TDVP = 0, 1
