"""The device's independent answer check (taral_check_models) against the reference checker and the oracle:
(a) on the reference PDHG's own answers of the pinned runs it reproduces gpu/vector_check.check_files
(tests/golden/reference_vector_check.json); (b) over a batch of scenarios it agrees with the oracle's restatement
(oracle/check_oracle.py) on this engine's answers, and repeated calls give identical results."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import check_oracle
import lpgen
from conftest import bounded_pdhg as pdhg

GOLD = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLD))
import make_golden  # noqa: E402

pytestmark = pytest.mark.gpu
FIELDS = [("objective", "chk_objective"), ("row_violation_rel", "chk_row_viol_rel"),
          ("bound_violation", "chk_bound_viol"), ("dual_bound", "chk_dual_bound"),
          ("dual_obj_loose", "chk_dual_obj_loose"), ("dual_infeas_rel", "chk_dual_infeas_rel"),
          ("dual_gap_rel", "chk_dual_gap_rel"), ("dual_sign", "chk_dual_sign")]


def close(a, b, tol=1e-9):
    if a is None or b is None:
        return a is None and b is None
    return abs(a - b) <= tol * max(1.0, abs(b))


def test_device_check_reproduces_reference_checker(engine_lib):
    gold = json.loads((GOLD / "reference_vector_check.json").read_text())
    vecs = np.load(GOLD / "reference_vectors.npz")
    names = [r[0] for r in make_golden.RUNS]
    lps = [r[1]() for r in make_golden.RUNS]
    res = pdhg.check_models(lps, [vecs[n + "/x"] for n in names], [vecs[n + "/y"] for n in names])
    for name, r in zip(names, res):
        for mine, ref in FIELDS:
            assert close(r[mine], gold[name][ref]), (name, mine, r[mine], gold[name][ref])


def test_device_check_over_a_batch(engine_lib):
    base = lpgen.RefineryBase(3, seed=7)
    lps = [base.instance(2 + (i % 2), p) for i, p in enumerate(lpgen.perturbations(6, seed=21))]
    b = pdhg.Batch(lps, tol=1e-6, precision=pdhg.FP32, time_limit=120)
    res, xs, ys = b.solve()
    assert all(r["status"] == "near_optimal" for r in res)
    c1 = pdhg.check_models(lps, xs, ys)
    c2 = pdhg.check_models(lps, xs, ys)
    assert c1 == c2
    for lp, x, y, r, c in zip(lps, xs, ys, res, c1):
        o = check_oracle.check(lp, x, y)
        for f in ("objective", "row_violation_rel", "bound_violation", "dual_obj_loose", "dual_infeas_rel",
                  "dual_gap_rel", "dual_sign", "dual_bound"):
            assert close(c[f], o[f], 1e-8), (f, c[f], o[f])
        assert abs(c["objective"] - r["objective"]) <= 1e-9 * max(1.0, abs(r["objective"]))
