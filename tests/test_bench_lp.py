"""The benchmark LP (planted, Zipf rows, 200,000 x 500,000, ~5M nonzeros, seed 0) against the reference's own FP64
CPU solve of it (tests/golden/reference_bench_lp.json, written by make_golden.py --bench-lp): the fixture belongs
to this exact model, and the FP64 GPU path reproduces the reference's iteration and restart counts and objective at
full size."""
import json
from pathlib import Path

import pytest

import lpgen
from conftest import bounded_pdhg as pdhg, rel

FIX = Path(__file__).resolve().parent / "golden" / "reference_bench_lp.json"


def bench_lp():
    return lpgen.planted(200_000, 500_000, 10, seed=0, zipf=1.2, cap=2000, floor=5, name="PLANTED_ZIPF_0")


def test_fixture_is_the_bench_model():
    d = json.loads(FIX.read_text())
    lp = bench_lp()
    assert d["model_sha256"] == lp.digest() and d["rows"] == lp.m and d["cols"] == lp.n and d["nnz"] == lp.nnz
    assert d["status"] == "near_optimal"


@pytest.mark.gpu
def test_fp64_full_size_matches_reference(engine_lib):
    d = json.loads(FIX.read_text())
    lp = bench_lp()
    r, _, _ = pdhg.solve(lp, tol=1e-6, precision=pdhg.FP64, time_limit=300)
    assert r["status"] == "near_optimal"
    assert r["iterations"] == d["iterations"] and r["restarts"] == d["restarts"], (r["iterations"], d["iterations"])
    assert rel(r["objective"], d["objective"]) < 1e-9
