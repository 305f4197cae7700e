"""Objective error against the FP64 CPU oracle on the refinery family: one 4-period scenario (6,000 rows x 16,000
columns) whose optimum the reference dual simplex computed (tests/golden/reference_refinery_T4.json, written by
make_golden.py --refinery). The plain engine (FP32 and FP64) and the batched engine (FP32, beside two other
scenarios) reach 1e-6 relative KKT error with objectives within 1e-6 relative of that optimum."""
import json
from pathlib import Path

import pytest

import lpgen
from conftest import bounded_pdhg as pdhg, rel

FIX = Path(__file__).resolve().parent / "golden" / "reference_refinery_T4.json"
pytestmark = pytest.mark.gpu


def scenario():
    return lpgen.RefineryBase(48, seed=7).instance(4, lpgen.perturbations(2, seed=3)[0])


def test_refinery_objective_against_reference_optimum(engine_lib):
    d = json.loads(FIX.read_text())
    lp = scenario()
    assert d["status"] == "optimal" and d["model_sha256"] == lp.digest()
    for precision in (pdhg.FP32, pdhg.FP64):
        r, _, _ = pdhg.solve(lp, tol=1e-6, precision=precision, time_limit=120)
        assert r["status"] == "near_optimal"
        assert rel(r["objective"], d["objective"]) < 1e-6, (precision, r["objective"], d["objective"])
    base = lpgen.RefineryBase(48, seed=7)
    others = [base.instance(4, p) for p in lpgen.perturbations(3, seed=11)[:2]]
    b = pdhg.Batch([lp] + others, tol=1e-6, precision=pdhg.FP32, time_limit=120)
    res, _, _ = b.solve(want_points=False)
    assert all(r["status"] == "near_optimal" for r in res)
    assert rel(res[0]["objective"], d["objective"]) < 1e-6, (res[0]["objective"], d["objective"])
