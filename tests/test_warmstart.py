"""Tensor-core dense layers and the learned steady-state warm start.

The TF32 GEMM (tcgen05) is checked against numpy on random matrices to
the TF32 input rounding bound (10-bit mantissa per operand).
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gemm(q, A, B, bias, act):
    import torch
    assert A.dtype == B.dtype == np.float32 and (bias is None or bias.dtype == np.float32)
    L = q.lib()
    L.quac_gemm_tf32.restype = ctypes.c_int
    L.quac_gemm_tf32.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int] * 4
    a = torch.from_numpy(A).cuda()
    b = torch.from_numpy(B).cuda()
    bi = torch.from_numpy(bias).cuda() if bias is not None else None
    c = torch.zeros((A.shape[0], B.shape[0]), dtype=torch.float32, device="cuda")
    rc = L.quac_gemm_tf32(a.data_ptr(), b.data_ptr(), c.data_ptr(), bi.data_ptr() if bi is not None else None,
                          A.shape[0], B.shape[0], A.shape[1], act)
    assert rc == 0, L.quac_last_error()
    return c.cpu().numpy()


@pytest.mark.parametrize("M,N,K,act", [(128, 128, 32, 0), (300, 200, 96, 1), (2000, 16384 // 16, 256, 0),
                                       (77, 513, 64, 1)])
def test_gemm_tf32_matches_numpy(quac, M, N, K, act):
    rng = np.random.default_rng(M + N + K)
    A = rng.normal(size=(M, K)).astype(np.float32)
    B = (rng.normal(size=(N, K)) / np.sqrt(K)).astype(np.float32)
    bias = rng.normal(size=N).astype(np.float32)
    C = _gemm(quac, A, B, bias, act)
    ref = A.astype(np.float64) @ B.T.astype(np.float64) + bias
    if act == 1:
        ref = np.tanh(ref)
    # TF32 keeps 10 mantissa bits of each operand: |error| <= 3 * 2^-10 * (|A| |B|^T) (tanh is 1-Lipschitz)
    bound = 3 * 2.0 ** -10 * (np.abs(A).astype(np.float64) @ np.abs(B).T.astype(np.float64)) + 1e-6
    assert np.all(np.abs(C - ref) <= bound)
    assert np.abs(C - ref).max() > 0  # really TF32 tensor-core arithmetic, not an FP32 fallback
