"""Ledger compatibility: the reference harness gpu/bench_pdhg.py drives a PDHG binary through TARAL_PDHG and writes
one row per case in its FIELDS schema from the binary's JSON report and its .sol / .dual files. The harness itself
is not on the GPU machine, so its contract is a fixture (tests/golden/reference_ledger.json, made by
`make_golden.py --ledger` from the harness's source and from a run of the harness on the reference binary): its
FIELDS, the report keys it reads, the flags it passes, and the row it wrote for packing_10000 at 1e-6.

This test runs this repository's CLI exactly as the harness's run_pdhg() runs a binary for the `gpu` config,
rebuilds the row the way the harness's main() does (the independent answer check through the oracle's restatement
of gpu/vector_check.check_files), and requires every FIELDS entry, every report key, and the same status,
iteration and restart counts and objective as the reference's own row (FP64: the iterations are the reference's)."""
import json
import os
import subprocess

import numpy as np
import pytest

import check_oracle
import lpgen
from conftest import golden, rel
import pdhg

pytestmark = pytest.mark.gpu


def _read_named(path, names):
    vals = {}
    for line in path.read_text().splitlines():
        k, v = line.split()
        vals[k] = float(v)
    return np.array([vals[k] for k in names])


def test_cli_writes_the_reference_ledger_row(engine_lib, tmp_path):
    fx = golden("reference_ledger.json")
    lp = lpgen.packing(10000, seed=1)
    assert lp.digest() == fx["model_sha256"]
    f = tmp_path / "packing_10000.mps"
    lp.write_mps(f)
    out, sol, dual = tmp_path / "r.json", tmp_path / "r.json.sol", tmp_path / "r.json.dual"
    tol, limit = 1e-6, 60.0
    cmd = [str(pdhg.CLI_PATH), str(f), "--device", "gpu", "--tol", str(tol), "--time-limit", str(limit),
           "--json", str(out), "--sol", str(sol), "--dual", str(dual)]
    assert {c for c in cmd if c.startswith("--")} <= set(fx["pdhg_flags"])
    subprocess.run(cmd, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, timeout=limit + 120, check=True)
    r0 = json.loads(out.read_text())
    missing = [k for k in fx["json_keys"] if k not in r0]
    assert not missing, missing
    rn, cn = lp._names()
    x, y = _read_named(sol, cn), _read_named(dual, rn)
    chk = check_oracle.check(lp, x, y)
    ref_obj = fx["reference_objective_via_ref_json"]
    row = dict(case="packing_10000", rows=r0.get("rows"), cols=r0.get("cols"), nnz=r0.get("nnz"), device="gpu",
               threads=r0.get("threads"), precision=r0.get("precision"), tol=tol, status=r0.get("status"),
               objective=r0.get("objective"), highs_objective=ref_obj,
               objective_rel_error_vs_highs=abs(r0["objective"] - ref_obj) / max(1.0, abs(ref_obj)),
               rel_primal=r0.get("rel_primal"), rel_dual=r0.get("rel_dual"), rel_gap=r0.get("rel_gap"),
               max_row_violation=r0.get("max_row_violation"), iterations=r0.get("iterations"),
               restarts=r0.get("restarts"), setup_s=r0.get("setup_s"), solve_s=r0.get("solve_s"),
               total_s=r0.get("total_s"), total_s_min=r0.get("total_s"), total_s_max=r0.get("total_s"), repeats=1,
               device_mem_bytes=r0.get("device_mem_bytes"), highs_s=None, load_avg_1m=os.getloadavg()[0],
               chk_objective=chk["objective"], chk_row_viol_rel=chk["row_violation_rel"],
               chk_bound_viol=chk["bound_violation"], chk_dual_bound=chk["dual_bound"],
               chk_dual_obj_loose=chk["dual_obj_loose"], chk_dual_infeas_rel=chk["dual_infeas_rel"],
               chk_dual_gap_rel=chk["dual_gap_rel"], chk_dual_sign=chk["dual_sign"],
               chk_row_viol_rel_max_repeats=chk["row_violation_rel"], objective_identical_repeats=True)
    assert set(fx["fields"]) - {"chk_error"} <= set(row), set(fx["fields"]) - set(row)
    ref = fx["reference_row_cpu1"]
    for k in ("rows", "cols", "nnz", "precision", "status", "iterations", "restarts"):
        assert row[k] == ref[k], (k, row[k], ref[k])
    assert rel(row["objective"], ref["objective"]) < 1e-9
    assert row["objective_rel_error_vs_highs"] < 1e-9 and row["chk_dual_sign"] == ref["chk_dual_sign"]
    for k in ("chk_objective", "chk_dual_obj_loose"):
        assert rel(row[k], ref[k]) < 1e-9, (k, row[k], ref[k])
    for k in ("rel_primal", "rel_dual", "rel_gap", "chk_row_viol_rel", "chk_dual_gap_rel"):
        assert abs(row[k] - ref[k]) <= 1e-9 + 1e-6 * abs(ref[k]), (k, row[k], ref[k])
