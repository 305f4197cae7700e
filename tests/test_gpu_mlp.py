"""The learned warm start's GPU kernels: the BF16 tensor-core GEMM and the MLP's forward / backward pass, checked
against the FP64 numpy restatement in oracle/mlp_oracle.py (which rounds to bfloat16 where the GPU stores
bfloat16, so the comparison measures the FP32 accumulation, not the input rounding)."""
import ctypes as C

import numpy as np
import pytest

import mlp_oracle
import pdhg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ta,tb", [(0, 0), (1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("M,N,K,slices", [(256, 384, 512, 1), (37, 203, 91, 1), (64, 512, 4096, 8), (128, 1000, 256, 3)])
def test_gemm_bf16(engine_lib, ta, tb, M, N, K, slices):
    import torch
    rng = np.random.default_rng(M + N + K)
    A = mlp_oracle.bf16(rng.standard_normal((K, M) if ta else (M, K)))
    B = mlp_oracle.bf16(rng.standard_normal((N, K) if tb else (K, N)))
    dev = torch.device("cuda")
    dA = torch.tensor(A, dtype=torch.bfloat16, device=dev)
    dB = torch.tensor(B, dtype=torch.bfloat16, device=dev)
    dC = torch.zeros((M, N), dtype=torch.float32, device=dev)
    ws = torch.zeros(slices * M * N, dtype=torch.float32, device=dev)
    code = pdhg.lib().taral_gemm_bf16(M, N, K, ta, tb, C.c_void_p(dA.data_ptr()), C.c_void_p(dB.data_ptr()),
                                      C.c_void_p(dC.data_ptr()), slices, C.c_void_p(ws.data_ptr()), None)
    assert code == pdhg.OK
    torch.cuda.synchronize()
    ref = (A.T if ta else A) @ (B.T if tb else B)
    got = dC.cpu().numpy().astype(np.float64)
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.sqrt(K) * np.max(np.abs(ref)) + 1e-6


def test_mlp_gradients_match_oracle(engine_lib):
    net = pdhg.Mlp(24, 64, 3, 136, max_batch=32)
    net.init(seed=3)
    p = net.get_params().astype(np.float64)
    rng = np.random.default_rng(1)
    x = rng.standard_normal((20, 24))
    t = rng.standard_normal((20, 136)) * 0.5
    y_gpu = net.forward(x)
    y_ref, _, _ = mlp_oracle.forward(p, net.shapes(), x)
    assert np.max(np.abs(y_gpu - y_ref)) <= 2e-3 * (1 + np.max(np.abs(y_ref)))
    loss, g = net.gradients(x, t)
    loss_ref, g_ref = mlp_oracle.loss_and_grads(p, net.shapes(), x, t)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    k = 0
    for (fi, fo), _ in net.shapes():  # per tensor: relative error of the gradient in the 2-norm
        for size in (fi * fo, fo):
            a, b = g[k:k + size], g_ref[k:k + size]
            assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-9, (k, size)
            k += size


def test_mlp_training_reduces_loss(engine_lib):
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, (512, 16))
    Wt = rng.standard_normal((16, 200)) * 0.5
    t = np.tanh(x @ Wt)  # a smooth target the network can fit
    net = pdhg.Mlp(16, 128, 3, 200, max_batch=64)
    net.init(seed=0)
    l0, _ = net.gradients(x[:64], t[:64])
    net.set_dataset(x, t)
    last = net.train(epochs=40, batch=64, lr=2e-3, seed=1)
    assert last < 0.1 * l0, (l0, last)
