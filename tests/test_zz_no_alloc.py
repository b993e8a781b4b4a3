"""The allocation-free SVD entry point against the allocating one.

yaqs_batched_svd_noalloc serves callers that cannot call cudaMalloc (their
device memory belongs to their own pool allocator, or an allocation would
synchronise the device or could fail mid-run): it takes device buffers and
uses a fixed scratch array compiled into the library.  This file is named so
that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dptr(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))


def _host_svd(ctx, Mb, batch, m, n):
    from yaqs_julia_b200 import _abi as A
    k = min(m, n)
    U = np.zeros(batch * m * k * 2)
    S = np.zeros(batch * k)
    SVt = np.zeros(batch * k * n * 2)
    ctx.check(ctx._lib.yaqs_batched_svd(ctx.handle, batch, m, n, A.dptr(Mb), A.dptr(U), A.dptr(S), A.dptr(SVt)))
    return U, S, SVt


def test_noalloc_svd_matches_allocating_svd_on_two_calls():
    import torch
    from yaqs_julia_b200 import _lib
    ctx = _lib.default_context()
    rng = np.random.default_rng(2024)
    for batch, m, n in ((3, 48, 40), (2, 128, 128)):  # two calls in a row, different shapes
        k = min(m, n)
        Mb = (rng.standard_normal(batch * m * n) + 1j * rng.standard_normal(batch * m * n)).view(np.float64)
        U_ref, S_ref, SVt_ref = _host_svd(ctx, Mb, batch, m, n)
        dev = torch.device("cuda", 0)
        dM = torch.from_numpy(Mb.copy()).to(dev)
        dU = torch.zeros(batch * m * k * 2, dtype=torch.float64, device=dev)
        dS = torch.zeros(batch * k, dtype=torch.float64, device=dev)
        dSVt = torch.zeros(batch * k * n * 2, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        ctx.check(ctx._lib.yaqs_batched_svd_noalloc(ctx.handle, batch, m, n, _dptr(dM), _dptr(dU), _dptr(dS),
                                                    _dptr(dSVt), C.c_void_p(stream)))
        torch.cuda.synchronize(dev)
        scale = np.abs(Mb).max() * max(m, n)
        assert np.abs(dS.cpu().numpy() - S_ref).max() <= 1e-12 * scale
        assert np.abs(dU.cpu().numpy() - U_ref).max() <= 1e-12 * max(m, n)
        assert np.abs(dSVt.cpu().numpy() - SVt_ref).max() <= 1e-12 * scale


def test_noalloc_svd_rejects_sizes_beyond_its_scratch():
    from yaqs_julia_b200 import _lib
    from yaqs_julia_b200._lib import EngineError
    ctx = _lib.default_context()
    buf = (C.c_double * 2)()
    p = C.cast(buf, C.POINTER(C.c_double))
    with pytest.raises(EngineError, match="8 MiB"):
        ctx.check(ctx._lib.yaqs_batched_svd_noalloc(ctx.handle, 64, 128, 128, p, p, p, p, None))
