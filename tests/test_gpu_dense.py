"""FP64 GEMM of the Ritz step (SRC/cheblanNr.c:333-399 forms the Ritz vectors
V(:,1:K) Y; evsl_dgemm_device is the reference's device BLAS entry point)
through the C ABI: the 128 x 128 tiled DFMA kernel (cp.async double
buffering, 8 x 8 accumulators per thread) against the 64 x 64 kernel -- both
form each entry as the FMA chain over k in order, so they agree bit for bit
-- and the default kernel on the FP64 tensor instruction against both and
numpy (1e-13 of the largest |C| entry): aligned and unaligned operands (odd
leading dimensions), ragged edges, beta 0 and 0.5.
"""
import ctypes as C

import numpy as np
import pytest

import evsl_b200

pytestmark = pytest.mark.gpu


def _gemm(lib, m, n, k, A, lda, B, ldb, Cm, ldc, alpha, beta, tiled):
    prev = lib.lib.evslcu_set_dgemm_tiled(int(tiled))
    dA = evsl_b200.DeviceBuffer.from_host(lib.lib, A)
    dB = evsl_b200.DeviceBuffer.from_host(lib.lib, B)
    dC = evsl_b200.DeviceBuffer.from_host(lib.lib, Cm)
    ci = lambda v: C.byref(C.c_int(v))  # noqa: E731
    cd = lambda v: C.byref(C.c_double(v))  # noqa: E731
    lib.lib.evsl_dgemm_device(b"N", b"N", ci(m), ci(n), ci(k), cd(alpha), C.c_void_p(dA.ptr), ci(lda),
                              C.c_void_p(dB.ptr), ci(ldb), cd(beta), C.c_void_p(dC.ptr), ci(ldc))
    out = dC.to_host(shape=Cm.shape)
    lib.lib.evslcu_set_dgemm_tiled(prev)
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


@pytest.mark.parametrize("n, m, b", [(20000, 100, 32), (5003, 45, 16), (40000, 33, 32)])
def test_block_cgs2_orthonormalises(gpu_lib, n, m, b):
    """Block Gram-Schmidt twice (the mixed-precision refinement's
    orthonormalisation; GEMM projections between blocks, CGS + DGKS as in
    SRC/misc_la.c:221-261 inside a block): the columns come out orthonormal to
    1e-13 and span the input columns (every input column is reproduced by its
    projection to 1e-12 of its norm), on well and badly conditioned inputs."""
    rng = np.random.default_rng(n + m)
    W0 = rng.standard_normal((m, n))  # row j = column j of the n x m block
    # a badly conditioned half: columns nearly dependent on the first ones
    W0[m // 2:] = W0[: m - m // 2] + 1e-6 * rng.standard_normal((m - m // 2, n))
    dW = evsl_b200.DeviceBuffer.from_host(gpu_lib.lib, W0)
    dH = evsl_b200.DeviceBuffer(gpu_lib.lib, 8 * m * m)
    dn = evsl_b200.DeviceBuffer(gpu_lib.lib, 8)
    gpu_lib.lib.evslcu_cgs_work_size.restype = C.c_size_t
    gpu_lib.lib.evslcu_cgs_work_size.argtypes = [C.c_int, C.c_int]
    work = evsl_b200.DeviceBuffer(gpu_lib.lib, 8 * int(gpu_lib.lib.evslcu_cgs_work_size(n, b)))
    fn = gpu_lib.lib.evslcu_block_cgs2
    fn.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    assert fn(n, m, dW.ptr, b, dH.ptr, dn.ptr, work.ptr) == 0
    Q = dW.to_host(shape=(m, n))
    G = Q @ Q.T
    assert np.max(np.abs(G - np.eye(m))) <= 1e-13
    P = (W0 @ Q.T) @ Q
    assert np.max(np.linalg.norm(W0 - P, axis=1) / np.linalg.norm(W0, axis=1)) <= 1e-12


@pytest.mark.parametrize("m, n, k, pad", [(1000, 70, 333, 0), (1001, 64, 257, 0), (4096, 300, 1000, 0),
                                         (777, 129, 33, 3), (2048, 32, 16, 1), (513, 40, 1, 0)])
@pytest.mark.parametrize("beta", [0.0, 0.5])
def test_mma_gemm_matches(gpu_lib, m, n, k, pad, beta):
    """The tall GEMM on the FP64 tensor instruction (mma.sync m8n8k4, same
    tiles and staging as the DFMA kernel, products summed in the
    instruction's order): within 1e-13 of numpy and of the DFMA kernel,
    aligned and unaligned operands, ragged edges, beta 0 and 0.5; the padding
    rows of C untouched."""
    rng = np.random.default_rng(m + 2 * n + k)
    lda, ldb, ldc = m + pad, k + pad, m + pad
    A = rng.standard_normal((k, lda))
    B = rng.standard_normal((n, ldb))
    C0 = rng.standard_normal((n, ldc))
    alpha = 1.0 if beta == 0.0 else -0.75
    got = _gemm(gpu_lib, m, n, k, A, lda, B, ldb, C0, ldc, alpha, beta, 2)
    dfma = _gemm(gpu_lib, m, n, k, A, lda, B, ldb, C0, ldc, alpha, beta, 1)
    ref = alpha * (A[:, :m].T @ B[:, :k].T) + beta * C0[:, :m].T
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got[:, :m].T - ref)) <= 1e-13 * scale
    assert np.max(np.abs(got - dfma)) <= 1e-13 * scale
    assert np.array_equal(got[:, m:], C0[:, m:])
