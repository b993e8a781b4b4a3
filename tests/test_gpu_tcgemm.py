"""The tensor-core complex FP32 product (tcgen05 MMAs in the 3-product
complex form with the 3xTF32 split, operands loaded by TMA) against a
complex128 numpy product.  It is the contraction kernel of the
mixed-precision form (the @tensor products of Algorithms.jl:199-226,
:330-361), so the bar is FP32 accuracy: |C - C_ref| <= 2e-6 * (|A| |B|)
elementwise, which a single-pass TF32 product (~5e-4) would fail."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from yaqs_julia_b200 import _lib
    return _lib.default_context()


def _run(ctx, A, B, a_kmajor, conj_a, b_kmajor, conj_b):
    batch, M, K = A.shape
    N = B.shape[2]
    ah = np.ascontiguousarray(A if a_kmajor else A.transpose(0, 2, 1)).astype(np.complex64)
    bh = np.ascontiguousarray(B.transpose(0, 2, 1) if b_kmajor else B).astype(np.complex64)
    c = np.zeros((batch, N, M), np.complex64)
    fp = C.POINTER(C.c_float)
    ctx.check(ctx._lib.yaqs_batched_cgemm_tf32(ctx.handle, batch, M, N, K, ah.ctypes.data_as(fp), a_kmajor, conj_a,
                                               bh.ctypes.data_as(fp), b_kmajor, conj_b, c.ctypes.data_as(fp)))
    return c.transpose(0, 2, 1)


def _check(A, B, Cg, conj_a, conj_b):
    Ar = A.astype(np.complex64).astype(np.complex128)
    Br = B.astype(np.complex64).astype(np.complex128)
    if conj_a:
        Ar = Ar.conj()
    if conj_b:
        Br = Br.conj()
    ref = Ar @ Br
    scale = np.abs(Ar) @ np.abs(Br)
    err = np.abs(Cg - ref) / np.maximum(scale, 1e-30)
    return float(err.max())


@pytest.mark.parametrize("M,N,K", [(128, 64, 8), (320, 128, 64), (64, 64, 320), (37, 19, 5), (256, 64, 320),
                                   (130, 66, 9), (8, 256, 64), (320, 256, 64)])
@pytest.mark.parametrize("a_kmajor,b_kmajor", [(0, 1), (0, 0), (1, 1), (1, 0)])
def test_tc_cgemm_matches_complex128(ctx, M, N, K, a_kmajor, b_kmajor):
    rng = np.random.default_rng(M * 1000 + N * 10 + K)
    batch = 3
    A = rng.standard_normal((batch, M, K)) + 1j * rng.standard_normal((batch, M, K))
    B = rng.standard_normal((batch, K, N)) + 1j * rng.standard_normal((batch, K, N))
    for conj_a, conj_b in [(0, 0), (1, 0), (0, 1)]:
        Cg = _run(ctx, A, B, a_kmajor, conj_a, b_kmajor, conj_b)
        assert _check(A, B, Cg, conj_a, conj_b) < 2e-6


def test_tc_cgemm_wide_dynamic_range(ctx):
    """Entries spanning 12 orders of magnitude (environment tensors of a
    long chain): the split keeps every product at FP32 accuracy."""
    rng = np.random.default_rng(11)
    M, N, K = 200, 96, 48
    mag = 10.0 ** rng.uniform(-6, 6, (1, M, K))
    A = mag * (rng.standard_normal((1, M, K)) + 1j * rng.standard_normal((1, M, K)))
    B = rng.standard_normal((1, K, N)) + 1j * rng.standard_normal((1, K, N))
    Cg = _run(ctx, A, B, 0, 0, 1, 0)
    assert _check(A, B, Cg, 0, 0) < 2e-6
