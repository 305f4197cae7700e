"""The engine's host set-up (taral-lp_b200/csrc/scaling.cpp), on the CPU: the CSR transpose split over threads must
give, for every thread count, exactly the sequential counting-sort transpose of the reference (gpu/pdhg.cu:55-70:
rows ascending, entries of a row in input order), restated here with numpy; the model matrices must drop explicit
zeros before transposing (gpu/pdhg.cu:80-90) and read A^T straight from a model whose columns already are A^T, with
the same numbers as the copying form."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "native" / "host_setup.cpp"
I64, I32, F64 = C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("hs") / "libhost_setup.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(ROOT / "include"),
                    "-I", str(ROOT / "taral-lp_b200" / "csrc"), str(SRC),
                    str(ROOT / "taral-lp_b200" / "csrc" / "scaling.cpp"), "-o", str(out), "-lpthread"], check=True)
    L = C.CDLL(str(out))
    L.transpose_into.restype = C.c_int64
    L.transpose_into.argtypes = [I64, I32, F64, C.c_int, C.c_int, C.c_int, I64, I32, F64]
    L.model_matrices_into.restype = C.c_int64
    L.model_matrices_into.argtypes = [C.c_int, C.c_int, I64, I32, F64, C.c_int, C.c_int, I64, I32, F64, I64, I32, F64,
                                      C.POINTER(C.c_int)]
    return L


def p(a, t):
    return a.ctypes.data_as(t)


def seq_transpose(ptr, idx, val, rows, cols):
    """Sequential counting sort: output row j lists the input rows holding j in input order."""
    cnt = np.bincount(idx[ptr[0]:ptr[rows]], minlength=cols)
    optr = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
    src_row = np.repeat(np.arange(rows, dtype=np.int32), np.diff(ptr))
    order = np.argsort(idx[ptr[0]:ptr[rows]], kind="stable")
    return optr, src_row[order], val[ptr[0]:ptr[rows]][order]


def random_csc(m, n, per_col, seed, zeros=False, unsorted=False):
    rng = np.random.default_rng(seed)
    cnt = rng.integers(0, 2 * per_col + 1, n)
    ptr = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
    idx = np.empty(int(ptr[-1]), np.int32)
    for j in range(n):
        r = np.sort(rng.choice(m, size=int(cnt[j]), replace=False)).astype(np.int32)
        idx[ptr[j]:ptr[j + 1]] = rng.permutation(r) if unsorted else r
    val = rng.standard_normal(idx.size)
    if zeros:
        val[rng.random(idx.size) < 0.05] = 0.0
    return ptr, idx, val


@pytest.fixture(scope="module")
def big():
    return random_csc(20_000, 40_000, 14, seed=1)  # ~560k nonzeros: up to 8 ranges of 65,536


@pytest.mark.parametrize("threads", [1, 2, 3, 8, 16])
def test_threaded_transpose_is_the_sequential_one(lib, big, threads):
    ptr, idx, val = big
    m, n = 20_000, len(ptr) - 1
    nnz = int(ptr[-1])
    optr, oidx, oval = np.zeros(m + 1, np.int64), np.zeros(nnz, np.int32), np.zeros(nnz)
    assert lib.transpose_into(p(ptr, I64), p(idx, I32), p(val, F64), n, m, threads, p(optr, I64), p(oidx, I32),
                              p(oval, F64)) == nnz
    wp, wi, wv = seq_transpose(ptr, idx, val, n, m)
    assert np.array_equal(optr, wp) and np.array_equal(oidx, wi) and np.array_equal(oval, wv)


def test_transpose_of_an_offset_view_and_empty_rows(lib):
    ptr, idx, val = random_csc(300, 500, 3, seed=2)
    ptr2 = ptr[100:].copy()  # rows 100.. of the input: ptr2[0] > 0
    rows = len(ptr2) - 1
    nnz = int(ptr2[-1] - ptr2[0])
    optr, oidx, oval = np.zeros(301, np.int64), np.zeros(nnz, np.int32), np.zeros(nnz)
    lib.transpose_into(p(ptr2, I64), p(idx, I32), p(val, F64), rows, 300, 4, p(optr, I64), p(oidx, I32), p(oval, F64))
    wp, wi, wv = seq_transpose(ptr2, idx, val, rows, 300)
    assert np.array_equal(optr, wp) and np.array_equal(oidx, wi) and np.array_equal(oval, wv)


@pytest.mark.parametrize("kind", ["sorted", "zeros", "unsorted"])
@pytest.mark.parametrize("threads", [1, 5])
def test_model_matrices_reference_form(lib, kind, threads):
    m, n = 3000, 7000
    ptr, idx, val = random_csc(m, n, 9, seed=3, zeros=kind == "zeros", unsorted=kind == "unsorted")
    nnz = int(ptr[-1])
    outs = []
    for by_ref in (0, 1):
        a = (np.zeros(m + 1, np.int64), np.zeros(nnz, np.int32), np.zeros(nnz))
        t = (np.zeros(n + 1, np.int64), np.zeros(nnz, np.int32), np.zeros(nnz))
        flag = C.c_int(-1)
        k = lib.model_matrices_into(m, n, p(ptr, I64), p(idx, I32), p(val, F64), threads, by_ref, p(a[0], I64),
                                    p(a[1], I32), p(a[2], F64), p(t[0], I64), p(t[1], I32), p(t[2], F64),
                                    C.byref(flag))
        outs.append((k, a, t, flag.value))
    (k0, a0, t0, f0), (k1, a1, t1, f1) = outs
    assert f0 == 0 and f1 == (1 if kind == "sorted" else 0)
    assert k0 == k1
    assert np.array_equal(a0[0], a1[0]) and np.array_equal(t0[0], t1[0])  # row pointers
    for u, v in zip(a0[1:] + t0[1:], a1[1:] + t1[1:]):  # entries, up to the nonzero count
        assert np.array_equal(u[:k0], v[:k0])
    # A: the transpose of the model with its explicit zeros dropped, rows ascending inside every column of A^T
    keep = val != 0
    cols = np.repeat(np.arange(n, dtype=np.int32), np.diff(ptr))[keep]
    kept_ptr = np.concatenate([[0], np.cumsum(np.bincount(cols, minlength=n))]).astype(np.int64)
    wp, wi, wv = seq_transpose(kept_ptr, idx[keep], val[keep], n, m)
    assert k0 == wi.size
    assert np.array_equal(a0[0], wp) and np.array_equal(a0[1][:k0], wi) and np.array_equal(a0[2][:k0], wv)
    tp, ti, tv = seq_transpose(wp, wi, wv, m, n)
    assert np.array_equal(t1[0], tp) and np.array_equal(t1[1][:k0], ti) and np.array_equal(t1[2][:k0], tv)
