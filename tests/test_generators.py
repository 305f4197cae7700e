"""Workload generators: the reference-family generators reproduce the reference's gpu/gen_lp.py byte for byte,
and the planted families carry the optimum / feasible point they claim."""
import hashlib

import numpy as np
import pytest

import lpgen
from conftest import golden

SHA = golden("gen_lp_sha256.json")
MAKERS = {"packing_10000_s1": lambda: lpgen.packing(10000, seed=1), "packing_2000_s3": lambda: lpgen.packing(2000, seed=3),
          "transport_100x100_s1": lambda: lpgen.transport(100, 100, seed=1),
          "transport_30x40_s2": lambda: lpgen.transport(30, 40, seed=2)}


@pytest.mark.parametrize("key", sorted(SHA))
def test_reference_family_bytes(key):
    assert hashlib.sha256(MAKERS[key]().mps_text().encode()).hexdigest() == SHA[key]


def _dense(lp):
    A = np.zeros((lp.m, lp.n))
    cols = np.repeat(np.arange(lp.n), np.diff(lp.col_ptr))
    A[lp.row_idx, cols] = lp.val
    return A


def test_planted_optimum_satisfies_kkt():
    lp = lpgen.planted(200, 500, 5, seed=3)
    A = _dense(lp)
    x, y = lp.x_star, lp.y_star
    assert np.allclose(A @ x, lp.row_lo) and np.array_equal(lp.row_lo, lp.row_up)
    assert np.all(x >= 0) and np.all(x <= 10)
    d = lp.cost - A.T @ y
    # b and c are rounded to the 12 digits the MPS file carries, so the planted KKT holds to ~1e-11
    assert np.all(d[x == 0] >= 0.1 - 1e-9) and np.all(d[x == 10] <= -0.1 + 1e-9)
    assert np.allclose(d[(x > 0) & (x < 10)], 0, atol=1e-9)
    assert abs(lp.obj_star - lp.cost @ x) < 1e-9 * abs(lp.obj_star)
    assert np.all(np.diff(lp.col_ptr) == 5)


def test_zipf_row_lengths():
    L = lpgen.zipf_row_lengths(20000, 20000 * 25, s=1.2, cap=2000, floor=5)
    assert L.sum() == 20000 * 25 and L.max() <= 2000 and L.min() >= 5 and L.max() == 2000
    lp = lpgen.planted(2000, 5000, 10, seed=1, zipf=1.2, cap=500)
    rows = np.bincount(lp.row_idx, minlength=lp.m)
    assert rows.max() <= 500 and lp.nnz > 0.97 * 50000  # repeats of a heavy row within a column are dropped


def test_general_planted_points_feasible():
    lp = lpgen.general(150, 300, seed=5)
    # the generator's rows are feasible at its planted x0 by construction; check through the bounds only
    assert np.all(lp.col_lo <= lp.col_up) and np.all(lp.row_lo <= lp.row_up)
    kinds = {(np.isfinite(a), np.isfinite(b)) for a, b in zip(lp.col_lo, lp.col_up)}
    assert kinds == {(False, False), (True, False), (False, True), (True, True)}
    assert np.any(lp.col_lo == lp.col_up) and np.any(np.isfinite(lp.row_lo) & np.isfinite(lp.row_up) & (lp.row_lo < lp.row_up))


def test_r12_arithmetic_equals_text_rounding():
    """The arithmetic 12-digit rounding used by the generators gives the doubles of the '%.12g' text, bit for bit,
    on wide-range values, the generators' price and capacity products, ties, powers of ten and specials."""
    rng = np.random.default_rng(11)
    cases = [rng.standard_normal(200_000) * np.exp(rng.uniform(-25, 25, 200_000)),
             np.round(rng.uniform(-50, 50, 100_000), 4) * rng.uniform(0.8, 1.2, 100_000),
             np.round(rng.uniform(100, 1000, 100_000), 3) * rng.uniform(0.8, 1.2, 100_000),
             (rng.integers(1, 10**12, 50_000) * 2 + 1) / 2.0 / 10.0 ** rng.integers(0, 12, 50_000),
             np.array([10.0 ** k for k in range(-30, 30)] + [-(10.0 ** k) for k in range(-30, 30)]),
             np.array([0.0, -0.0, np.inf, -np.inf, np.nan, 5e-324, 1.7e308, 999999999999.5, 0.1, 1 / 3])]
    for v in cases:
        a, b = lpgen._r12(v), lpgen._r12_text(v)
        assert np.array_equal(a, b, equal_nan=True) and np.array_equal(np.signbit(a), np.signbit(b))
