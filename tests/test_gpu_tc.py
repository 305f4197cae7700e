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
