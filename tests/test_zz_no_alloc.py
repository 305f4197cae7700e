"""taral_kkt_eval_noalloc: the KKT evaluation for callers that cannot allocate device memory.

Such callers (a host whose GPU memory is reserved up front by another allocator, or a loop that must not take
cudaMalloc's implicit synchronisation) hold the iterate vectors themselves and get the 10 KKT scalars computed
with a fixed, library-owned scratch array instead of per-context allocations. This test rebuilds, in torch
device buffers, the state a context reaches after one block of iterations (the point from pdhg_download, its
products from the existing SpMV entry point, the data vectors of the scaled problem), then checks two calls in
a row of the allocation-free entry point against the context's own pdhg_eval, to the 1e-9 relative tolerance of
the other FP64 step-level tests. Both storage types are covered: an FP64 context with double vectors and an FP32
context with float vectors (the same float inputs and the same FP64 reduction, so the scalars agree to the same
tolerance). This file is collected last so that a failure here comes after every other test has run."""
import ctypes as C

import numpy as np
import pytest

import lpgen
import oracle
import pdhg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [pdhg.FP64, pdhg.FP32], ids=["fp64", "fp32"])
def test_noalloc_eval_matches_context_eval(engine_lib, oracle_lib, precision):
    import torch
    lp = lpgen.general(300, 700, seed=3)
    sp = oracle.ScaledProblem(lp)
    eng = pdhg.Engine.from_scaled(sp, precision=precision)
    norm = sp.power_norm(200)
    eng.set_steps(0.95 / norm * 0.7, 0.95 / norm / 0.7)
    eng.start()
    eng.iterate(64)  # one block, no restart: x_last = clamp(0, l, u), z_last = 0
    expected = eng.eval(0, 1.0)
    x, z = eng.download(0, 1.0)

    dev = torch.device("cuda")
    # the context narrows every vector to its storage type with round-to-nearest, as numpy's astype does
    npt = np.float64 if precision == pdhg.FP64 else np.float32
    tt = torch.float64 if precision == pdhg.FP64 else torch.float32

    def t(a):
        return torch.tensor(np.ascontiguousarray(np.asarray(a, np.float64).astype(npt)), device=dev)

    A, AT = sp.A, sp.AT
    ax, atz = torch.zeros(sp.m, dtype=tt, device=dev), torch.zeros(sp.n, dtype=tt, device=dev)
    xs, zs = t(x), t(z)
    for (ptr, idx, val), vin, vout, cols in ((A, xs, ax, sp.n), (AT, zs, atz, sp.m)):
        plan = pdhg.SpmvPlan(ptr, cols, dtype=precision)
        d_ptr = torch.tensor(ptr.astype(np.int32), device=dev)
        d_idx = torch.tensor(idx.astype(np.int32), device=dev)
        d_val = t(val)
        plan.run(d_ptr.data_ptr(), d_idx.data_ptr(), d_val.data_ptr(), vin.data_ptr(), vout.data_ptr())
        torch.cuda.synchronize()
        plan.close()
    l_t, u_t = np.asarray(sp.l).astype(npt), np.asarray(sp.u).astype(npt)
    x0 = np.minimum(np.maximum(npt(0), l_t), u_t)
    vecs = dict(Ax=ax, z=zs, rl=t(sp.rl), ru=t(sp.ru), Dr=t(sp.Dr), zlast=t(np.zeros(sp.m)),
                x=xs, ATz=atz, c=t(sp.c), l=t(sp.l), u=t(sp.u), Dc=t(sp.Dc), xlast=t(x0))
    order = ["Ax", "z", "rl", "ru", "Dr", "zlast", "x", "ATz", "c", "l", "u", "Dc", "xlast"]
    for call in range(2):  # the scratch array keeps the previous call's contents; the second call must not care
        out = torch.full((10,), float("nan"), dtype=torch.float64, device=dev)
        code = pdhg.lib().taral_kkt_eval_noalloc(sp.m, sp.n, precision, 1.0,
                                                 *[C.c_void_p(vecs[k].data_ptr()) for k in order],
                                                 C.c_void_p(out.data_ptr()), None)
        assert code == pdhg.OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        scale = np.maximum(np.abs(expected), 1.0)
        assert np.all(np.abs(got - expected) <= 1e-9 * scale), (call, got, expected)


def test_noalloc_rejects_sizes_beyond_the_limit(engine_lib):
    code = pdhg.lib().taral_kkt_eval_noalloc(2_000_000_001, 10, pdhg.FP64, 1.0, *[C.c_void_p(1)] * 13,
                                             C.c_void_p(1), None)
    assert code == pdhg.ERR_INPUT
