"""Standalone SpMV (taral_spmv_*, the counterpart of gpu/csr_matvec.cu:23-32) against the CPU oracle's CSR product.

Every row-split policy of the autotuner (forced through TARAL_ROWSPLIT) sums the same products in a fixed order of
its own, so in FP64 each row agrees with the oracle's sequential sum to rounding (bounded by n eps sum|a x|); in
FP32 the products are rounded to float and summed in FP64, then the sum is rounded to float. Matrices cover rows
longer than a block (the whole-CTA path), rows of 49..128 nonzeros (the 8-lane groups), empty rows, an empty matrix,
index / value arrays that are not 16-byte aligned (the scalar staging path) and a matrix whose rows all hold at most
48 nonzeros (one thread per row under policy 0, bit-identical to the staged kernel)."""
import numpy as np
import pytest

import lpgen
import oracle
import pdhg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _matrices():
    lp = lpgen.planted(3000, 8000, 8, seed=5, zipf=1.1, cap=3000, floor=1)  # one row > 2044 nonzeros
    yield "zipf_long_rows", lp.csr()
    rng = np.random.default_rng(3)
    lens = rng.choice([0, 3, 60, 100, 127, 128, 129, 300], size=700)
    ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    idx = np.concatenate([np.sort(rng.choice(5000, size=k, replace=False)) for k in lens]).astype(np.int32)
    val = rng.standard_normal(int(ptr[-1]))
    yield "mid_rows_and_empty", (ptr, idx, val)
    lens = rng.integers(0, 49, size=5000)  # every row <= 48 nonzeros: the one-thread-per-row kernel
    ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    idx = np.concatenate([np.sort(rng.choice(3000, size=k, replace=False)) for k in lens]).astype(np.int32)
    yield "short_rows", (ptr, idx, rng.standard_normal(int(ptr[-1])))


def _run(ptr, idx, val, x, dtype, offset=0):
    """y = A x through the C ABI; offset > 0 shifts idx / val by that many elements (breaks 16-byte alignment)."""
    dev = torch.device("cuda")
    tdt = torch.float64 if dtype == pdhg.FP64 else torch.float32
    d_ptr = torch.from_numpy(np.asarray(ptr, np.int32)).to(dev)
    d_idx = torch.zeros(len(idx) + offset + 1, dtype=torch.int32, device=dev)
    d_val = torch.zeros(len(val) + offset + 1, dtype=tdt, device=dev)
    d_idx[offset:offset + len(idx)] = torch.from_numpy(np.asarray(idx, np.int32)).to(dev)
    d_val[offset:offset + len(val)] = torch.from_numpy(np.asarray(val)).to(dev, tdt)
    d_x = torch.from_numpy(np.asarray(x)).to(dev, tdt)
    rows = len(ptr) - 1
    d_y = torch.full((max(rows, 1),), float("nan"), dtype=tdt, device=dev)
    plan = pdhg.SpmvPlan(ptr, len(x), dtype)
    try:
        es = d_idx.element_size()
        plan.run(d_ptr.data_ptr(), d_idx.data_ptr() + offset * es, d_val.data_ptr() + offset * d_val.element_size(),
                 d_x.data_ptr(), d_y.data_ptr())
        torch.cuda.synchronize()
    finally:
        plan.close()
    return d_y.double().cpu().numpy()[:rows]


@pytest.mark.parametrize("policy", ["0", "1", "2", "3", "4"])
@pytest.mark.parametrize("offset", [0, 1])
def test_spmv_policies_match_oracle(engine_lib, oracle_lib, monkeypatch, policy, offset):
    monkeypatch.setenv("TARAL_ROWSPLIT", policy)
    for name, (ptr, idx, val) in _matrices():
        n = int(idx.max()) + 1
        x = np.random.default_rng(7).standard_normal(n)
        ref = oracle.spmv(ptr, idx, val, x)
        absum = oracle.spmv(ptr, idx, np.abs(val), np.abs(x))
        y64 = _run(ptr, idx, val, x, pdhg.FP64, offset)
        lens = np.diff(ptr)
        assert np.all(np.abs(y64 - ref) <= (lens + 1) * 2.3e-16 * absum), (name, policy)
        # FP32: products of the float operands rounded to float (rows longer than a block: exact products), summed
        # in FP64, the sum rounded to float
        v32, x32 = val.astype(np.float32), x.astype(np.float32)
        exact = v32.astype(np.float64) * x32[idx].astype(np.float64)
        prod = np.where(np.repeat(lens, lens) > 2044, exact, (v32 * x32[idx]).astype(np.float64))
        ref32 = np.zeros(len(ptr) - 1)
        np.add.at(ref32, np.repeat(np.arange(len(ptr) - 1), lens), prod)
        psum = np.zeros(len(ptr) - 1)
        np.add.at(psum, np.repeat(np.arange(len(ptr) - 1), lens), np.abs(prod))
        y32 = _run(ptr, idx, v32, x32, pdhg.FP32, offset)
        tol = 6e-8 * np.abs(ref32) + (lens + 1) * 2.3e-16 * psum
        assert np.all(np.abs(y32 - ref32) <= tol), (name, policy, np.max(np.abs(y32 - ref32) - tol))


def test_spmv_empty_and_bad_input(engine_lib):
    assert len(_run(np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0), np.ones(4), pdhg.FP64)) == 0
    with pytest.raises(pdhg.TaralError):
        pdhg.SpmvPlan(np.array([0, 3, 2], np.int64), 4, pdhg.FP64)  # decreasing row pointer


@pytest.mark.parametrize("dtype", [pdhg.FP64, pdhg.FP32])
def test_spmv_row_thread_is_bit_identical(engine_lib, monkeypatch, dtype):
    ptr, idx, val = list(_matrices())[-1][1]
    x = np.random.default_rng(2).standard_normal(int(idx.max()) + 1)
    if dtype == pdhg.FP32:
        val, x = val.astype(np.float32), x.astype(np.float32)
    y_thread = _run(ptr, idx, val, x, dtype)
    monkeypatch.setenv("TARAL_ROWTHREAD", "0")
    y_staged = _run(ptr, idx, val, x, dtype)
    assert np.array_equal(y_thread, y_staged)
