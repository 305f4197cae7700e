"""Failure paths of the batched engine and the allocators, made on the host without faulting the GPU.

* A cancel request (taral_batch_cancel) from another host thread stops a running batch after its current block:
  the device's decision kernel reads the flag from pinned host memory, every running instance ends with status
  `cancelled`, the solve returns ERR_CANCELLED with the outcomes filled, and the next solve runs normally.
* The device iteration budget (max_iter, checked by the decision kernel) ends every instance at exactly that count,
  across launches of several blocks and a final partial block.
* Launching several blocks per graph changes no result.
* The allocation hook (taral_set_device_alloc_limit) makes context and batch creation fail with ERR_ALLOC, as an
  out-of-memory device would, and the library works normally once it is lifted."""
import threading
import time

import numpy as np
import pytest

import lpgen
from conftest import bounded_pdhg as pdhg

pytestmark = pytest.mark.gpu


def _family(count, periods, seed):
    base = lpgen.RefineryBase(periods, seed=seed)
    pert = lpgen.perturbations(count, seed=seed + 1)
    return [base.instance(periods, p) for p in pert]


def test_cancel_from_another_thread(engine_lib):
    lps = _family(32, 12, seed=21)  # several seconds of batched solve to 1e-6
    b = pdhg.Batch(lps, tol=1e-6, precision=pdhg.FP32, time_limit=300)
    timer = threading.Timer(0.3, b.cancel)
    t0 = time.perf_counter()
    timer.start()
    res, xs, ys = b.solve()
    wall = time.perf_counter() - t0
    timer.join()
    assert b.last_code == pdhg.ERR_CANCELLED
    assert all(r["status"] in ("cancelled", "near_optimal") for r in res)
    assert sum(r["status"] == "cancelled" for r in res) > 0
    its = [r["iterations"] for r in res]
    assert min(its) >= 64 and all(k % 64 == 0 for k in its)
    for lp, x in zip(lps, xs):  # the points of the stopped instances come back, finite, one entry per column
        assert x.shape == (lp.n,) and np.all(np.isfinite(x))
    # the request applied to that solve only: the same batch now solves to the tolerance, and takes longer
    t0 = time.perf_counter()
    res2, _, _ = b.solve()
    wall2 = time.perf_counter() - t0
    assert b.last_code == pdhg.OK and all(r["status"] == "near_optimal" for r in res2)
    assert wall < wall2, (wall, wall2)
    assert all(r2["iterations"] >= r["iterations"] for r, r2 in zip(res, res2))


def test_cancel_before_solve_stops_after_the_first_block(engine_lib):
    lps = _family(6, 4, seed=31)
    b = pdhg.Batch(lps, tol=1e-6, precision=pdhg.FP32, time_limit=300)
    b.cancel()
    res, _, _ = b.solve()
    assert b.last_code == pdhg.ERR_CANCELLED
    assert all(r["status"] == "cancelled" and r["iterations"] == 64 for r in res), res
    res2, _, _ = b.solve()
    assert b.last_code == pdhg.OK and all(r["status"] == "near_optimal" for r in res2)


def test_budget_across_multi_block_launches(engine_lib, monkeypatch):
    monkeypatch.setenv("TARAL_BATCH_BLOCKS", "4")
    lps = [lpgen.general(150, 350, seed=k) for k in range(3)]
    b = pdhg.Batch(lps, tol=1e-13, max_iter=4 * 64 * 2 + 64 + 17, time_limit=120)  # 2 launches, a block, 17 steps
    res, _, _ = b.solve()
    assert all(r["status"] == "iteration_limit" and r["iterations"] == 4 * 64 * 2 + 64 + 17 for r in res), res


@pytest.mark.parametrize("precision", [pdhg.FP64, pdhg.FP32], ids=["fp64", "fp32"])
def test_blocks_per_launch_change_nothing(engine_lib, monkeypatch, precision):
    base = lpgen.RefineryBase(4, seed=3)
    lps = [base.instance(3 + k % 2, p) for k, p in enumerate(lpgen.perturbations(6, seed=9))]
    outs = []
    for blocks in ("1", "4", "16"):
        monkeypatch.setenv("TARAL_BATCH_BLOCKS", blocks)
        monkeypatch.setenv("TARAL_TUNE", "0")
        b = pdhg.Batch(lps, tol=1e-6, precision=precision, time_limit=300)
        outs.append(b.solve())
        b.close()
    (r1, x1, _), (r4, x4, _), (r16, x16, _) = outs
    for a, b_, c in zip(r1, r4, r16):
        assert a["status"] == b_["status"] == c["status"] == "near_optimal"
        assert a["iterations"] == b_["iterations"] == c["iterations"] and a["objective"] == b_["objective"] == c["objective"]
    assert all(np.array_equal(p, q) and np.array_equal(p, r) for p, q, r in zip(x1, x4, x16))


def test_allocation_limit_hook(engine_lib):
    lp = lpgen.general(400, 900, seed=4)
    try:
        pdhg.set_device_alloc_limit(64 << 10)  # 64 KB: far below what a context of this model needs
        with pytest.raises(pdhg.TaralError) as e:
            pdhg.Engine.from_model(lp)
        assert e.value.code == pdhg.ERR_ALLOC
        with pytest.raises(pdhg.TaralError) as e:
            pdhg.Batch([lp, lp], tol=1e-6)
        assert e.value.code == pdhg.ERR_ALLOC
        with pytest.raises(pdhg.TaralError) as e:
            pdhg.solve(lp, tol=1e-6)
        assert e.value.code == pdhg.ERR_ALLOC
    finally:
        pdhg.set_device_alloc_limit(0)
    r, _, _ = pdhg.solve(lp, tol=1e-6)
    assert r["status"] == "near_optimal"
    res, _, _ = pdhg.Batch([lp, lp], tol=1e-6).solve()
    assert all(x["status"] == "near_optimal" and abs(x["iterations"] - r["iterations"]) <= 64 for x in res)


def test_batch_programmatic_launch_changes_nothing(engine_lib, monkeypatch):
    lps = _family(6, 3, seed=41)
    outs = []
    for flag in ("0", "1"):
        monkeypatch.setenv("TARAL_PDL", flag)
        b = pdhg.Batch(lps, tol=1e-6, precision=pdhg.FP32, time_limit=300)
        outs.append(b.solve())
        b.close()
    (r0, x0, _), (r1, x1, _) = outs
    assert [r["iterations"] for r in r0] == [r["iterations"] for r in r1]
    assert all(np.array_equal(p, q) for p, q in zip(x0, x1))
