"""Batched solves (taral_batch_*) against single-instance solves of the same models.

Each instance follows the reference driver's rules with its own restarts and stopping, evaluated on the device.
The batch sums its KKT scalars per row block and evaluates the restart rule in device FP64, so its arithmetic
matches the single-instance path to rounding: statuses agree, iteration counts agree to within one evaluation
block in FP64, objectives to 1e-7 relative."""
import numpy as np
import pytest

import lpgen
from conftest import bounded_pdhg as pdhg, rel

pytestmark = pytest.mark.gpu


def _single(lp, **kw):
    r, x, y = pdhg.solve(lp, **kw)
    return r


def test_batch_of_distinct_models_fp64(engine_lib):
    lps = [lpgen.general(120 + 20 * k, 300 + 30 * k, seed=k) for k in range(6)] + [lpgen.packing(1500, seed=4),
                                                                                  lpgen.transport(12, 17, seed=5)]
    b = pdhg.Batch(lps, tol=1e-6, time_limit=120)
    assert b.info()["distinct_matrices"] == len(lps)
    res, xs, ys = b.solve()
    for lp, r, x in zip(lps, res, xs):
        s = _single(lp, tol=1e-6)
        assert r["status"] == s["status"] == "near_optimal", (lp.name, r, s)
        assert abs(r["iterations"] - s["iterations"]) <= 64, (lp.name, r["iterations"], s["iterations"])
        assert rel(r["objective"], s["objective"]) < 1e-7, (lp.name, r["objective"], s["objective"])
        assert max(r["rel_primal"], r["rel_dual"], r["rel_gap"]) <= 1e-6
        assert len(x) == lp.n


def test_batch_matches_matrices_by_content(engine_lib):
    """Instances whose matrices are equal but held in separate arrays share one stored matrix; a matrix of the same
    sizes with one value changed is stored apart; each instance solves as it does alone."""
    import dataclasses
    base = lpgen.RefineryBase(2, seed=12)
    pert = lpgen.perturbations(3, seed=3)
    a = base.instance(2, pert[0])
    b = dataclasses.replace(base.instance(2, pert[1]), col_ptr=a.col_ptr.copy(), row_idx=a.row_idx.copy(),
                            val=a.val.copy())
    c0 = base.instance(2, pert[2])
    v = c0.val.copy()
    v[len(v) // 2] *= 1.5
    c = dataclasses.replace(c0, val=v)
    lps = [a, b, c]
    bt = pdhg.Batch(lps, tol=1e-6, precision=pdhg.FP64, time_limit=300)
    info = bt.info()
    assert info["distinct_matrices"] == 2 and info["nnz_stored"] == 2 * len(a.val)
    res, xs, _ = bt.solve()
    for lp, r, x in zip(lps, res, xs):
        s, xs1, _ = pdhg.solve(lp, tol=1e-6, precision=pdhg.FP64)
        assert r["status"] == s["status"] == "near_optimal"
        assert abs(r["iterations"] - s["iterations"]) <= 64 and rel(r["objective"], s["objective"]) < 1e-7


def test_batch_shares_matrices_fp32(engine_lib):
    base = lpgen.RefineryBase(3, seed=11)
    pert = lpgen.perturbations(5, seed=2)
    lps = [base.instance(2, pert[0]), base.instance(3, pert[1]), base.instance(2, pert[2]), base.instance(3, pert[3]),
           base.instance(2, pert[4])]
    b = pdhg.Batch(lps, tol=1e-6, precision=pdhg.FP32, time_limit=300)
    info = b.info()
    assert info["distinct_matrices"] == 2 and info["nnz_stored"] < info["nnz_total"]
    res, xs, ys = b.solve()
    for lp, r in zip(lps, res):
        assert r["status"] == "near_optimal", (lp.name, r)
        s = _single(lp, tol=1e-6)
        assert rel(r["objective"], s["objective"]) < 5e-6, (lp.name, r["objective"], s["objective"])


def test_batch_warm_start_and_limits(engine_lib):
    lps = [lpgen.general(150, 350, seed=k) for k in range(3)]
    b = pdhg.Batch(lps, tol=1e-6, time_limit=120)
    res, xs, ys = b.solve()
    res2, _, _ = b.solve(x0=xs, y0=ys)  # warm start from the answers: a few blocks at most
    for r, r2 in zip(res, res2):
        assert r2["status"] == "near_optimal" and r2["iterations"] < r["iterations"] / 4
    res3, _, _ = b.solve(x0=[xs[0], None, None], y0=[ys[0], None, None])  # only instance 0 warm
    assert res3[0]["iterations"] < res[0]["iterations"] / 4
    assert [r["iterations"] for r in res3[1:]] == [r["iterations"] for r in res[1:]]
    # initial primal weight: values that are not finite and positive keep the default
    res5, _, _ = b.solve(w0=[0.0, float("nan"), -1.0])
    assert [r["iterations"] for r in res5] == [r["iterations"] for r in res]
    res6, _, _ = b.solve(w0=[r["primal_weight"] * 8.0 for r in res])
    for r, r6 in zip(res, res6):
        assert r6["status"] == "near_optimal" and rel(r6["objective"], r["objective"]) < 1e-5
    assert [r["iterations"] for r in res6] != [r["iterations"] for r in res]
    b2 = pdhg.Batch(lps, tol=1e-12, max_iter=128, time_limit=120)
    res4, _, _ = b2.solve()
    assert all(r["status"] == "iteration_limit" and r["iterations"] == 128 for r in res4)


def test_batch_deterministic(engine_lib):
    lps = [lpgen.general(100, 260, seed=k) for k in range(4)]
    b = pdhg.Batch(lps, tol=1e-6, time_limit=120)
    r1, x1, _ = b.solve()
    r2, x2, _ = b.solve()
    assert [r["iterations"] for r in r1] == [r["iterations"] for r in r2]
    assert all(np.array_equal(a, c) for a, c in zip(x1, x2))


@pytest.mark.parametrize("width", ["1", "8"])
def test_batch_packs_match_single_solves(engine_lib, monkeypatch, width):
    # 11 scenarios of one matrix and 2 of another; with packs of up to 8 slots: a pack of 8, a pack of 4 with one
    # unused slot, a pack of 2. Each batched instance takes the iterates of the same LP solved alone.
    monkeypatch.setenv("TARAL_BATCH_PACK", width)
    monkeypatch.setenv("TARAL_TUNE", "0")  # both sides on the default row split, whatever their timings
    monkeypatch.setenv("TARAL_ROWORDER", "0")  # and the single solves in the model's row order, like the batch
    base = lpgen.RefineryBase(2, seed=5)
    pert = lpgen.perturbations(13, seed=8)
    lps = [base.instance(2, p) for p in pert[:11]] + [base.instance(1, p) for p in pert[11:]]
    b = pdhg.Batch(lps, tol=1e-6, precision=pdhg.FP32, time_limit=300)
    assert b.info()["distinct_matrices"] == 2
    res, xs, _ = b.solve()
    for lp, r, x in zip(lps, res, xs):
        s, xsol, _ = pdhg.solve(lp, tol=1e-6, precision=pdhg.FP32, time_limit=120)
        assert r["status"] == "near_optimal" and r["iterations"] == s["iterations"], (lp.name, r["iterations"], s["iterations"])
        assert rel(r["objective"], s["objective"]) < 1e-9
        assert np.max(np.abs(x - xsol)) <= 1e-9 * (1 + np.max(np.abs(xsol)))


@pytest.mark.parametrize("pack", ["1", "8"])
def test_batch_tail_compaction_changes_nothing(engine_lib, monkeypatch, pack):
    """Instances stop at different iterations; once a quarter of the running ones have stopped, the iteration lists
    are rebuilt without them. Compacted and full lists give identical counts and bit-identical points, and a second
    solve on the same batch (lists restored) repeats the first."""
    monkeypatch.setenv("TARAL_BATCH_PACK", pack)
    base = lpgen.RefineryBase(3, seed=3)
    pert = lpgen.perturbations(16, seed=7)
    lps = [base.instance(2 + k % 2, pert[k]) for k in range(16)]
    b = pdhg.Batch(lps, tol=1e-6, precision=pdhg.FP32, time_limit=300)
    r1, x1, y1 = b.solve()
    assert len({r["iterations"] for r in r1}) > 3  # the instances stop at different blocks
    r2, x2, y2 = b.solve()
    monkeypatch.setenv("TARAL_COMPACT", "0")
    r3, x3, y3 = b.solve()
    for a, c in ((r1, r2), (r1, r3)):
        assert [r["iterations"] for r in a] == [r["iterations"] for r in c]
        assert [r["objective"] for r in a] == [r["objective"] for r in c]
    for xa, xb, xc in zip(x1, x2, x3):
        assert np.array_equal(xa, xb) and np.array_equal(xa, xc)
    for ya, yc in zip(y1, y3):
        assert np.array_equal(ya, yc)
    assert all(r["status"] == "near_optimal" for r in r1)


@pytest.mark.parametrize("precision", [pdhg.FP64, pdhg.FP32])
def test_batch_row_thread_kernel_is_bit_identical(engine_lib, monkeypatch, precision):
    """The batched one-thread-per-row kernel (one warp per 32-row chunk of one scenario) on phases whose rows all hold
    at most 48 nonzeros gives the same counts and bit-identical points: in FP64 the refinery scenarios' A^T and both
    matrices of the packing LPs (their A, rows up to 112, stays on the row blocks); in FP32 the packing LPs."""
    lps = [lpgen.packing(1500, seed=k) for k in range(3)]
    if precision == pdhg.FP64:
        base = lpgen.RefineryBase(3, seed=3)
        pert = lpgen.perturbations(6, seed=9)
        lps = [base.instance(2 + k % 2, pert[k]) for k in range(6)] + lps
    outs = []
    for flag in ("0", "1"):
        monkeypatch.setenv("TARAL_ROWTHREAD", flag)
        b = pdhg.Batch(lps, tol=1e-6, precision=precision, time_limit=300)
        outs.append(b.solve())
    (r0, x0, y0), (r1, x1, y1) = outs
    assert [r["iterations"] for r in r0] == [r["iterations"] for r in r1]
    assert [r["objective"] for r in r0] == [r["objective"] for r in r1]
    assert all(np.array_equal(a, c) for a, c in zip(x0, x1)) and all(np.array_equal(a, c) for a, c in zip(y0, y1))
    assert all(r["status"] == "near_optimal" for r in r0)


def test_batch_row_thread_kernel_fp32_medium_rows(engine_lib, monkeypatch):
    """In FP32 the thread-per-row kernel also takes rows of up to 128 nonzeros (the refinery A): every row summed by
    one thread in entry order, a different order than the row blocks' warps, so the answers agree to the tolerance,
    not bitwise."""
    base = lpgen.RefineryBase(3, seed=3)
    pert = lpgen.perturbations(6, seed=9)
    lps = [base.instance(2 + k % 2, pert[k]) for k in range(6)]
    outs = []
    for flag in ("0", "1"):
        monkeypatch.setenv("TARAL_ROWTHREAD", flag)
        b = pdhg.Batch(lps, tol=1e-6, precision=pdhg.FP32, time_limit=300)
        outs.append(b.solve()[0])
    for a, c in zip(*outs):
        assert a["status"] == c["status"] == "near_optimal"
        assert rel(a["objective"], c["objective"]) < 5e-6, (a["objective"], c["objective"])


def test_batch_power_iteration_once_per_matrix(engine_lib):
    # instances sharing a matrix take the estimate of the first one (the power iteration runs once per distinct
    # matrix): the same norm, bit for bit, and the same run as each instance batched alone
    base = lpgen.RefineryBase(3, seed=11)
    lps = [base.instance(3, p) for p in lpgen.perturbations(4, seed=2)] + [base.instance(2, None)]
    res, _, _ = pdhg.Batch(lps, tol=1e-6, precision=pdhg.FP32, time_limit=300).solve()
    for lp, r in zip(lps, res):
        a = pdhg.Batch([lp], tol=1e-6, precision=pdhg.FP32, time_limit=300).solve()[0][0]
        assert r["norm_a"] == a["norm_a"] and r["iterations"] == a["iterations"], (r["norm_a"], a["norm_a"])
    assert len({r["norm_a"] for r in res[:4]}) == 1
