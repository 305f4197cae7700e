"""The tcgen05 GEMM (tensor-memory accumulator) against numpy on bf16-rounded operands and against the mma.sync
GEMM, including ragged M and N (partial tiles) and a K that is a multiple of 8 but not of the 64-wide K slice."""
import ctypes as C

import numpy as np
import pytest

import mlp_oracle
import pdhg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (256, 512, 512), (37, 203, 88), (300, 1000, 256), (8, 3, 8),
                                   (256, 33001, 512)])
def test_gemm_tc(engine_lib, M, N, K):
    import torch
    rng = np.random.default_rng(M * 7 + N + K)
    A = mlp_oracle.bf16(rng.standard_normal((M, K)))
    Bt = mlp_oracle.bf16(rng.standard_normal((N, K)))
    dev = torch.device("cuda")
    dA = torch.tensor(A, dtype=torch.bfloat16, device=dev)
    dB = torch.tensor(Bt, dtype=torch.bfloat16, device=dev)
    dC = torch.full((M, N), float("nan"), dtype=torch.float32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    code = pdhg.lib().taral_gemm_bf16_tc(M, N, K, C.c_void_p(dA.data_ptr()), C.c_void_p(dB.data_ptr()),
                                         C.c_void_p(dC.data_ptr()), C.c_void_p(err.data_ptr()), None)
    assert code == pdhg.OK
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    got = dC.cpu().numpy().astype(np.float64)
    ref = A @ Bt.T
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.sqrt(K) * np.max(np.abs(ref)) + 1e-6
    # the mma.sync GEMM on the same operands (B stored [N][K]: tb = 1)
    dC2 = torch.zeros((M, N), dtype=torch.float32, device=dev)
    code = pdhg.lib().taral_gemm_bf16(M, N, K, 0, 1, C.c_void_p(dA.data_ptr()), C.c_void_p(dB.data_ptr()),
                                      C.c_void_p(dC2.data_ptr()), 1, None, None)
    assert code == pdhg.OK
    torch.cuda.synchronize()
    assert np.max(np.abs(dC2.cpu().numpy() - got)) <= 1e-5 * np.sqrt(K) * np.max(np.abs(ref)) + 1e-6


def test_gemm_tc_rejects_bad_shapes(engine_lib):
    import torch
    d = torch.zeros(64, dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.zeros(64, dtype=torch.float32, device="cuda")
    p = C.c_void_p(d.data_ptr())
    assert pdhg.lib().taral_gemm_bf16_tc(4, 4, 12, p, p, C.c_void_p(out.data_ptr()),
                                         C.c_void_p(err.data_ptr()), None) == pdhg.ERR_INPUT  # K % 8
    assert pdhg.lib().taral_gemm_bf16_tc(4, 4, 8, C.c_void_p(d.data_ptr() + 2), p, C.c_void_p(out.data_ptr()),
                                         C.c_void_p(err.data_ptr()), None) == pdhg.ERR_INPUT  # misaligned A


def _umma(M, N, K, a_mn, b_mn, lda_pad=0, ldb_pad=0, ldc_pad=0, slices=1, seed=0):
    """taral_gemm_bf16_umma on operands stored in the given layouts (with padded row strides) against numpy."""
    import torch
    rng = np.random.default_rng(seed + 17 * M + 3 * N + K)
    A = mlp_oracle.bf16(rng.standard_normal((M, K)))
    B = mlp_oracle.bf16(rng.standard_normal((N, K)))
    dev = torch.device("cuda")

    def stored(X, mn, pad):  # X is (rows, K): K-major storage [rows][ld], MN-major storage [K][ld]
        S = X.T if mn else X
        ld = (S.shape[1] + 7) // 8 * 8 + pad  # 16-byte rows, as the entry point requires
        buf = np.zeros((S.shape[0], ld))
        buf[:, :S.shape[1]] = S
        return torch.tensor(buf, dtype=torch.bfloat16, device=dev), ld
    dA, lda = stored(A, a_mn, lda_pad)
    dB, ldb = stored(B, b_mn, ldb_pad)
    ldc = N + ldc_pad
    dC = torch.full((M, ldc), float("nan"), dtype=torch.float32, device=dev)
    ws = torch.zeros(max(slices, 1) * M * ldc, dtype=torch.float32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    code = pdhg.lib().taral_gemm_bf16_umma(M, N, K, C.c_void_p(dA.data_ptr()), lda, a_mn, C.c_void_p(dB.data_ptr()),
                                           ldb, b_mn, C.c_void_p(dC.data_ptr()), ldc, slices,
                                           C.c_void_p(ws.data_ptr()), C.c_void_p(err.data_ptr()), None)
    assert code == pdhg.OK
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    got = dC.cpu().numpy().astype(np.float64)
    ref = A @ B.T
    assert np.all(np.isfinite(got[:, :N]))
    if ldc_pad:
        assert np.all(np.isnan(got[:, N:]))  # the padding of C is left alone
    assert np.max(np.abs(got[:, :N] - ref)) <= 1e-5 * np.sqrt(K) * np.max(np.abs(ref)) + 1e-6, (M, N, K, a_mn, b_mn)


@pytest.mark.parametrize("a_mn,b_mn", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (256, 512, 256), (200, 300, 136), (64, 1000, 512)])
def test_gemm_umma_layouts(engine_lib, a_mn, b_mn, M, N, K):
    _umma(M, N, K, a_mn, b_mn)


def test_gemm_umma_padded_strides_and_split_k(engine_lib):
    _umma(256, 1001, 256, 1, 1, lda_pad=0, ldb_pad=8, ldc_pad=5)          # dW-shaped: both MN-major, padded dZ
    _umma(256, 512, 4096, 0, 1, lda_pad=8, ldb_pad=0, slices=9)           # dH-shaped: split K into slices
    _umma(256, 33001, 512, 0, 0)                                          # forward-shaped, ragged N
    _umma(100, 120, 1000, 1, 0, slices=64)                                # more slices than K blocks: clipped


def test_gemm_umma_rejects_bad_strides(engine_lib):
    import torch
    d = torch.zeros(4096, dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.zeros(4096, dtype=torch.float32, device="cuda")
    p, o, e = C.c_void_p(d.data_ptr()), C.c_void_p(out.data_ptr()), C.c_void_p(err.data_ptr())
    L = pdhg.lib()
    assert L.taral_gemm_bf16_umma(8, 8, 16, p, 12, 0, p, 16, 0, o, 8, 1, None, e, None) == pdhg.ERR_INPUT  # lda % 8
    assert L.taral_gemm_bf16_umma(8, 8, 16, p, 8, 0, p, 16, 0, o, 8, 1, None, e, None) == pdhg.ERR_INPUT   # lda < K
    assert L.taral_gemm_bf16_umma(8, 8, 16, p, 16, 0, p, 16, 0, o, 4, 1, None, e, None) == pdhg.ERR_INPUT  # ldc < N
    assert L.taral_gemm_bf16_umma(8, 8, 16, p, 16, 0, p, 16, 0, o, 8, 2, None, e, None) == pdhg.ERR_INPUT  # no ws
