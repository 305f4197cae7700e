"""Whole-solve parity of the CUDA engine (taral_pdhg_solve / the pdhg CLI) with the reference.

FP64: iteration counts, restart counts and the answer's point type equal the reference's published ledgers and
the reference binary's runs; objectives and relative KKT errors agree to 1e-8 relative (summation order differs).
FP32 (FP32 matrix and iterates, FP64 averages and KKT): reaches the requested tolerance, with the objective
within 1e-6 relative of the FP64 optimum from the reference IPM or the planted optimum."""
import json
import subprocess

import numpy as np
import pytest

import lpgen
import oracle
import pdhg as _pdhg
from conftest import bounded_pdhg as pdhg
from conftest import golden, rel

pytestmark = pytest.mark.gpu

PINS = golden("ledger_pins.json")
RUNS = golden("reference_runs.json")
VECS = golden("reference_vectors.npz")
OPTIMA = golden("reference_optima.json")

LEDGER_MODELS = {"packing_10000": lambda: lpgen.packing(10000), "transport_100x100": lambda: lpgen.transport(100, 100)}
RUN_MODELS = {
    "packing_2000_s3": lambda: lpgen.packing(2000, seed=3),
    "transport_30x40_s2": lambda: lpgen.transport(30, 40, seed=2),
    "planted_300x700_s5": lambda: lpgen.planted(300, 700, 5, seed=5),
    "general_300x700_s3": lambda: lpgen.general(300, 700, seed=3),
    "general_300x700_s3_max": lambda: lpgen.general(300, 700, seed=3, maximize=True),
    "general_200x500_s7": lambda: lpgen.general(200, 500, seed=7),
}


def _flags_to_kw(flags):
    kw = {}
    it = iter(flags)
    for f in it:
        v = next(it)
        kw[{"--tol": "tol", "--row-rel": "row_rel", "--eval-freq": "eval_freq", "--max-iter": "max_iter"}[f]] = \
            float(v) if f in ("--tol", "--row-rel") else int(v)
    return kw


@pytest.mark.parametrize("key", sorted(PINS))
def test_ledger_pins_fp64(engine_lib, key):
    pin = PINS[key]
    lp = LEDGER_MODELS[pin["case"]]()
    r, x, y = pdhg.solve(lp, tol=float(pin["tol"]))
    assert r["status"] == pin["status"]
    assert r["iterations"] == int(pin["iterations"]) and r["restarts"] == int(pin["restarts"])
    assert rel(r["objective"], float(pin["objective"])) < 1e-10
    for k in ("rel_primal", "rel_dual", "rel_gap"):
        assert abs(r[k] - float(pin[k])) <= 1e-3 * abs(float(pin[k])) + 1e-12


@pytest.mark.parametrize("name", sorted(RUNS))
def test_reference_runs_fp64(engine_lib, name):
    ref = RUNS[name]
    base = next(k for k in sorted(RUN_MODELS, key=len, reverse=True) if name.startswith(k))
    lp = RUN_MODELS[base]()
    assert lp.digest() == ref["model_sha256"]
    r, x, y = pdhg.solve(lp, **_flags_to_kw(ref["flags"]))
    assert r["status"] == ref["status"] and r["iterations"] == ref["iterations"] and r["restarts"] == ref["restarts"]
    assert r["from_average"] == (ref["point"] == "average")
    assert rel(r["objective"], ref["objective"]) < 1e-8
    assert abs(r["primal_weight"] - ref["primal_weight"]) <= 1e-5 * ref["primal_weight"]
    assert np.allclose(x, VECS[name + "/x"], rtol=1e-6, atol=1e-7)
    assert np.allclose(y, VECS[name + "/y"], rtol=1e-6, atol=1e-7)


def test_oracle_and_engine_agree_on_general(engine_lib, oracle_lib):
    lp = lpgen.general(400, 900, seed=11)
    ro, xo, yo = oracle.solve(lp, tol=1e-6)
    rg, xg, yg = pdhg.solve(lp, tol=1e-6)
    assert (ro["status"], ro["iterations"], ro["restarts"]) == (rg["status"], rg["iterations"], rg["restarts"])
    assert rel(rg["objective"], ro["objective"]) < 1e-9


def test_fp32_planted_reaches_1e6(engine_lib):
    opt = OPTIMA["planted_2000x5000_s0"]
    lp = lpgen.planted(2000, 5000, 5, seed=0)
    assert lp.digest() == opt["model_sha256"]
    r, x, y = pdhg.solve(lp, tol=1e-6, precision=pdhg.FP32)
    assert r["status"] == "near_optimal"
    assert max(r["rel_primal"], r["rel_dual"], r["rel_gap"]) <= 1e-6
    assert rel(r["objective"], opt["objective"]) < 2e-6  # rel KKT 1e-6 bounds the objective error at ~1e-6
    # x is stored in float: a column at its bound sits at float(u / Dc), 6e-8 relative from u after unscaling
    assert r["max_bound_violation"] <= 1e-6 * 10


@pytest.mark.parametrize("make", [lambda: lpgen.packing(10000), lambda: lpgen.general(300, 700, seed=3),
                                  lambda: lpgen.transport(30, 40, seed=2)])
def test_fp32_converges_like_fp64(engine_lib, make):
    lp = make()
    r64, _, _ = pdhg.solve(lp, tol=1e-6)
    r32, _, _ = pdhg.solve(lp, tol=1e-6, precision=pdhg.FP32)
    assert r32["status"] == "near_optimal"
    assert r32["iterations"] <= 2 * r64["iterations"]
    assert rel(r32["objective"], r64["objective"]) < 5e-6


def test_warm_start_from_solution(engine_lib):
    lp = lpgen.general(300, 700, seed=3)
    r, x, y = pdhg.solve(lp, tol=1e-6)
    rw, xw, yw = pdhg.solve(lp, tol=1e-6, x0=x, y0=y)
    assert rw["status"] == "near_optimal" and rw["iterations"] < r["iterations"] / 4


def test_iteration_and_time_limits(engine_lib):
    lp = lpgen.packing(2000, seed=3)
    r, _, _ = pdhg.solve(lp, tol=1e-12, max_iter=100)
    assert r["status"] == "iteration_limit" and r["iterations"] == 100
    r, _, _ = pdhg.solve(lp, tol=1e-14, time_limit=0.2)
    assert r["status"] == "time_limit"


def test_empty_and_degenerate_models(engine_lib):
    # no rows: min c'x on a box
    lp = lpgen.LP(name="BOX", m=0, n=3, col_ptr=np.zeros(4, np.int64), row_idx=np.zeros(0, np.int32),
                  val=np.zeros(0), cost=np.array([1.0, -1.0, 0.0]), col_lo=np.zeros(3), col_up=np.ones(3),
                  row_lo=np.zeros(0), row_up=np.zeros(0))
    r, x, y = pdhg.solve(lp, tol=1e-8)
    assert r["status"] == "near_optimal" and abs(r["objective"] + 1.0) < 1e-8
    # an empty column and an empty row
    lp = lpgen.general(50, 80, seed=2)
    lp.col_ptr = np.concatenate([lp.col_ptr, [lp.col_ptr[-1]]])
    lp.n += 1
    for k, v in (("cost", 1.0), ("col_lo", 0.0), ("col_up", 5.0)):
        setattr(lp, k, np.append(getattr(lp, k), v))
    lp.m += 1
    lp.row_lo, lp.row_up = np.append(lp.row_lo, -1.0), np.append(lp.row_up, 1.0)
    ro, xo, _ = oracle.solve(lp, tol=1e-6)
    rg, xg, _ = pdhg.solve(lp, tol=1e-6)
    assert (rg["iterations"], rg["restarts"]) == (ro["iterations"], ro["restarts"])
    assert abs(xg[-1]) < 1e-9


def test_unsupported_model_rejected(engine_lib):
    lp = lpgen.general(20, 30, seed=1)
    lp.is_int = np.zeros(lp.n, np.uint8)
    lp.is_int[3] = 1
    with pytest.raises(pdhg.TaralError) as e:
        pdhg.solve(lp)
    assert e.value.code == pdhg.ERR_UNSUPPORTED


def test_cli_end_to_end(engine_lib, tmp_path):
    lp = lpgen.packing(2000, seed=3)
    f = tmp_path / "m.mps"
    lp.write_mps(f)
    j, s, d = tmp_path / "r.json", tmp_path / "r.sol", tmp_path / "r.dual"
    p = subprocess.run([str(pdhg.CLI_PATH), str(f), "--tol", "1e-6", "--json", str(j), "--sol", str(s), "--dual",
                        str(d)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    ref = RUNS["packing_2000_s3_tol1e-6"]
    assert p.stdout.startswith(f"status near_optimal objective ")
    rep = json.loads(j.read_text())
    assert rep["iterations"] == ref["iterations"] and rep["restarts"] == ref["restarts"]
    assert rep["rows"] == ref["rows"] and rep["cols"] == ref["cols"] and rep["nnz"] == ref["nnz"]
    xs = np.array([float(l.split()[1]) for l in s.read_text().splitlines()])
    ys = np.array([float(l.split()[1]) for l in d.read_text().splitlines()])
    assert np.allclose(xs, VECS["packing_2000_s3_tol1e-6/x"], rtol=1e-6, atol=1e-7)
    assert np.allclose(ys, VECS["packing_2000_s3_tol1e-6/y"], rtol=1e-6, atol=1e-7)
