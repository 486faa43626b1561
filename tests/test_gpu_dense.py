"""FP64 GEMM of the Ritz step (SRC/cheblanNr.c:333-399 forms the Ritz vectors
V(:,1:K) Y; evsl_dgemm_device is the reference's device BLAS entry point)
through the C ABI: the 128 x 128 tiled kernel (cp.async double buffering,
8 x 8 accumulators per thread) against the 64 x 64 kernel -- both form each
entry as the FMA chain over k in order, so they agree bit for bit -- and
against numpy (1e-13 of the largest |C| entry): aligned and unaligned
operands (odd leading dimensions), ragged edges, beta 0 and 0.5.
"""
import ctypes as C

import numpy as np
import pytest

import evsl_b200

pytestmark = pytest.mark.gpu


def _gemm(lib, m, n, k, A, lda, B, ldb, Cm, ldc, alpha, beta, tiled):
    lib.lib.evslcu_set_dgemm_tiled(1 if tiled else 0)
    dA = evsl_b200.DeviceBuffer.from_host(lib.lib, A)
    dB = evsl_b200.DeviceBuffer.from_host(lib.lib, B)
    dC = evsl_b200.DeviceBuffer.from_host(lib.lib, Cm)
    ci = lambda v: C.byref(C.c_int(v))  # noqa: E731
    cd = lambda v: C.byref(C.c_double(v))  # noqa: E731
    lib.lib.evsl_dgemm_device(b"N", b"N", ci(m), ci(n), ci(k), cd(alpha), C.c_void_p(dA.ptr), ci(lda),
                              C.c_void_p(dB.ptr), ci(ldb), cd(beta), C.c_void_p(dC.ptr), ci(ldc))
    out = dC.to_host(shape=Cm.shape)
    lib.lib.evslcu_set_dgemm_tiled(1)
    return out


@pytest.mark.parametrize("m, n, k, pad", [(1000, 70, 333, 0), (1001, 64, 257, 0), (4096, 300, 1000, 0),
                                         (777, 129, 33, 3), (2048, 32, 16, 1), (513, 40, 1, 0)])
@pytest.mark.parametrize("beta", [0.0, 0.5])
def test_tiled_gemm_matches(gpu_lib, m, n, k, pad, beta):
    rng = np.random.default_rng(m + n + k)
    lda, ldb, ldc = m + pad, k + pad, m + pad
    A = rng.standard_normal((k, lda))  # column j of A is row j here (column-major storage)
    B = rng.standard_normal((n, ldb))
    C0 = rng.standard_normal((n, ldc))
    alpha = 1.0 if beta == 0.0 else -0.75
    got = _gemm(gpu_lib, m, n, k, A, lda, B, ldb, C0, ldc, alpha, beta, True)
    old = _gemm(gpu_lib, m, n, k, A, lda, B, ldb, C0, ldc, alpha, beta, False)
    assert np.array_equal(got, old)
    ref = alpha * (A[:, :m].T @ B[:, :k].T) + beta * C0[:, :m].T
    assert np.max(np.abs(got[:, :m].T - ref)) <= 1e-13 * np.max(np.abs(ref))
    # the padding rows of C are untouched
    assert np.array_equal(got[:, m:], C0[:, m:])
