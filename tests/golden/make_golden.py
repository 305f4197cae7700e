#!/usr/bin/env python3
"""Regenerate the golden fixtures of tests/golden/ from the reference implementation.

Needs the reference checkout (REF, default: the directory "reference" beside this repository's checkout) and the reference binaries built from it by
``make -C oracle ref`` (oracle/_ref/pdhg, oracle/_ref/taral). Writes:

* gen_lp_sha256.json     sha256 of the MPS text that the reference's gpu/gen_lp.py writes for a few seeds
* ledger_pins.json       the reference's published CPU-FP64 PDHG rows for packing_10000 and transport_100x100
                         (results/gpu_pdhg/synth_*_tol1e-{4,6}.csv), read from its ledgers
* reference_runs.json    reference `pdhg --device cpu --threads 1` (FP64) reports on generated models
* reference_vectors.npz  the .sol / .dual vectors of those runs
* reference_optima.json  the reference IPM optimum (`taral --method ipm`) of the planted 2000 x 5000 model
* reference_vector_check.json (with --vector-check) the reference's independent answer check
                         (gpu/vector_check.check_files) on the .sol / .dual of the runs in reference_runs.json
* reference_refinery_T4.json (with --refinery, ~2 minutes of CPU) the reference dual simplex optimum of one
                         4-period scenario of the refinery family (RefineryBase(48, seed=7), perturbations(2, seed=3)[0])
* reference_ledger.json  (with --ledger) the reference harness's ledger contract, read from gpu/bench_pdhg.py: its
                         FIELDS, the keys it reads from a PDHG JSON report, the flags it passes to the PDHG binary,
                         and the row it writes for packing_10000 at 1e-6 when it runs the reference binary
                         (--configs cpu1, the reference objective given through --ref-json)
* reference_bench_lp.json (with --bench-lp, minutes of CPU) the reference `pdhg --device cpu` FP64 report on the
                         benchmark LP (planted, Zipf rows, 200,000 x 500,000, seed 0) solved to 1e-6: the FP64
                         iteration count the benchmark's CPU baselines are projected to

Run from the repository root: python tests/golden/make_golden.py [--bench-lp | --refinery | --vector-check | --ledger]
"""
import csv
import hashlib
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
REF = Path(os.environ.get("REF", str(Path(__file__).resolve().parents[3] / "reference")))
OUT = Path(__file__).resolve().parent
PDHG = ROOT / "oracle" / "_ref" / "pdhg"
TARAL = ROOT / "oracle" / "_ref" / "taral"
sys.path.insert(0, str(ROOT / "taral-lp_b200"))
import lpgen  # noqa: E402

GEN_CASES = [("packing", ["10000"], 1), ("packing", ["2000"], 3), ("transport", ["100", "100"], 1),
             ("transport", ["30", "40"], 2)]

# (case name, model factory, pdhg flags)
RUNS = [
    ("packing_2000_s3_tol1e-4", lambda: lpgen.packing(2000, seed=3), ["--tol", "1e-4"]),
    ("packing_2000_s3_tol1e-6", lambda: lpgen.packing(2000, seed=3), ["--tol", "1e-6"]),
    ("transport_30x40_s2_tol1e-6", lambda: lpgen.transport(30, 40, seed=2), ["--tol", "1e-6"]),
    ("planted_300x700_s5_tol1e-6", lambda: lpgen.planted(300, 700, 5, seed=5), ["--tol", "1e-6"]),
    ("general_300x700_s3_tol1e-6", lambda: lpgen.general(300, 700, seed=3), ["--tol", "1e-6"]),
    ("general_300x700_s3_max_tol1e-6", lambda: lpgen.general(300, 700, seed=3, maximize=True), ["--tol", "1e-6"]),
    ("general_200x500_s7_rowrel100_tol1e-4", lambda: lpgen.general(200, 500, seed=7),
     ["--tol", "1e-4", "--row-rel", "100"]),
    ("general_200x500_s7_freq32_maxit3000", lambda: lpgen.general(200, 500, seed=7),
     ["--tol", "1e-9", "--eval-freq", "32", "--max-iter", "3000"]),
]


def sha(text):
    return hashlib.sha256(text.encode()).hexdigest()


def read_vec(path):
    return np.array([float(line.rsplit(None, 1)[1]) for line in open(path)])


def main():
    if not PDHG.exists() or not TARAL.exists():
        sys.exit("build the reference first: make -C oracle ref")
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        gen = {}
        for fam, args, seed in GEN_CASES:
            f = td / "g.mps"
            subprocess.run([sys.executable, str(REF / "gpu" / "gen_lp.py"), fam, *args, str(f), "--seed", str(seed)],
                           check=True)
            gen[f"{fam}_{'x'.join(args)}_s{seed}"] = sha(f.read_text())
        (OUT / "gen_lp_sha256.json").write_text(json.dumps(gen, indent=1) + "\n")

        pins = {}
        for tol in ("1e-4", "1e-6"):
            for fam in ("packing", "transport"):
                with open(REF / "results" / "gpu_pdhg" / f"synth_{fam}_tol{tol}.csv") as fh:
                    for row in csv.DictReader(fh):
                        if row["device"] == "cpu" and row["threads"] == "1" and row["case"] in (
                                "packing_10000", "transport_100x100"):
                            pins[f"{row['case']}_tol{tol}"] = {
                                k: row[k] for k in ("case", "tol", "status", "objective", "iterations", "restarts",
                                                    "rel_primal", "rel_dual", "rel_gap", "max_row_violation")}
        (OUT / "ledger_pins.json").write_text(json.dumps(pins, indent=1) + "\n")

        runs, vecs = {}, {}
        for name, make, flags in RUNS:
            lp = make()
            f = td / "m.mps"
            lp.write_mps(f)
            j, s, d = td / "r.json", td / "r.sol", td / "r.dual"
            subprocess.run([str(PDHG), str(f), "--device", "cpu", "--threads", "1", *flags, "--json", str(j),
                            "--sol", str(s), "--dual", str(d)], check=True, stdout=subprocess.DEVNULL)
            rep = json.loads(j.read_text())
            runs[name] = {"flags": flags, "model_sha256": lp.digest(),
                          **{k: rep[k] for k in ("status", "objective", "iterations", "restarts", "rel_primal",
                                                 "rel_dual", "rel_gap", "point", "max_row_violation",
                                                 "max_bound_violation", "norm_a", "primal_weight", "rows", "cols",
                                                 "nnz")}}
            vecs[name + "/x"] = read_vec(s)
            vecs[name + "/y"] = read_vec(d)
        (OUT / "reference_runs.json").write_text(json.dumps(runs, indent=1) + "\n")
        np.savez_compressed(OUT / "reference_vectors.npz", **vecs)

        lp = lpgen.planted(2000, 5000, 5, seed=0)
        f = td / "p.mps"
        lp.write_mps(f)
        j = td / "p.json"
        subprocess.run([str(TARAL), str(f), "--method", "ipm", "--time-limit", "600", "--json", str(j)], check=True,
                       stdout=subprocess.DEVNULL)
        rep = json.loads(j.read_text())
        opt = {"planted_2000x5000_s0": {"method": "ipm", "status": rep.get("status"), "objective": rep.get("objective"),
                                         "planted_objective": lp.obj_star, "model_sha256": lp.digest()}}
        (OUT / "reference_optima.json").write_text(json.dumps(opt, indent=1) + "\n")
    print("wrote", sorted(p.name for p in OUT.iterdir()))


def bench_lp():
    if not PDHG.exists():
        sys.exit("build the reference first: make -C oracle ref")
    sys.path.insert(0, str(ROOT))
    import bench  # the benchmark's workload definition
    lp = bench.make_lp(0)
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        f, j = Path(td) / "b.mps", Path(td) / "b.json"
        lp.write_mps(f)
        subprocess.run([str(PDHG), str(f), "--device", "cpu", "--threads", str(threads), "--tol", "1e-6", "--json",
                        str(j)], check=True, stdout=subprocess.DEVNULL)
        rep = json.loads(j.read_text())
    out = {"workload": bench.WORKLOAD_NAME, "seed": 0, "model_sha256": lp.digest(), "threads": threads,
           **{k: rep[k] for k in ("status", "objective", "iterations", "restarts", "rel_primal", "rel_dual", "rel_gap",
                                  "scale_s", "power_iter_s", "solve_s", "rows", "cols", "nnz")}}
    (OUT / "reference_bench_lp.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote reference_bench_lp.json:", out["status"], out["iterations"])


def vector_check():
    sys.path.insert(0, str(REF / "gpu"))
    import vector_check as vc  # the reference's checker (needs REF/benchmarks/orig_check.py)
    vecs = np.load(OUT / "reference_vectors.npz")
    out = {}
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        for name, make, _ in RUNS:
            lp = make()
            rn, cn = lp._names()
            f, sol, dual = td / "m.mps", td / "m.sol", td / "m.dual"
            lp.write_mps(f)
            sol.write_text("".join(f"{c} {v:.17g}\n" for c, v in zip(cn, vecs[name + "/x"])))
            dual.write_text("".join(f"{r} {v:.17g}\n" for r, v in zip(rn, vecs[name + "/y"])))
            out[name] = {"model_sha256": lp.digest(), **vc.check_files(str(f), str(sol), str(dual))}
    (OUT / "reference_vector_check.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote reference_vector_check.json:", len(out), "runs")


def refinery():
    if not TARAL.exists():
        sys.exit("build the reference first: make -C oracle ref")
    lp = lpgen.RefineryBase(48, seed=7).instance(4, lpgen.perturbations(2, seed=3)[0])
    with tempfile.TemporaryDirectory() as td:
        f, j = Path(td) / "r.mps", Path(td) / "r.json"
        lp.write_mps(f)
        subprocess.run([str(TARAL), str(f), "--method", "dual", "--time-limit", "600", "--json", str(j)], check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        rep = json.loads(j.read_text())
    out = {"scenario": "RefineryBase(48, seed=7).instance(4, perturbations(2, seed=3)[0])", "method": "dual",
           "model_sha256": lp.digest(), "rows": lp.m, "cols": lp.n, "nnz": lp.nnz,
           **{k: rep.get(k) for k in ("status", "objective", "dual_objective", "primal_res", "dual_res", "gap")}}
    (OUT / "reference_refinery_T4.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote reference_refinery_T4.json:", out["status"], out["objective"])


def ledger():
    import ast
    import re
    harness = REF / "gpu" / "bench_pdhg.py"
    src = harness.read_text()
    tree = ast.parse(src)
    fields = next(ast.literal_eval(n.value) for n in ast.walk(tree)
                  if isinstance(n, ast.Assign) and any(getattr(t, "id", None) == "FIELDS" for t in n.targets))
    json_keys = sorted(set(re.findall(r"r0\.get\('([a-z_0-9]+)'\)", src)) | set(re.findall(r"med\('([a-z_0-9]+)'\)", src)))
    run_pdhg = next(n for n in ast.walk(tree) if isinstance(n, ast.FunctionDef) and n.name == "run_pdhg")
    flags = sorted({c.value for c in ast.walk(run_pdhg) if isinstance(c, ast.Constant) and isinstance(c.value, str)
                    and c.value.startswith("--")})
    pins = json.loads((OUT / "ledger_pins.json").read_text())["packing_10000_tol1e-6"]
    lp = lpgen.packing(10000, seed=1)
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        f = td / "packing_10000.mps"
        lp.write_mps(f)
        refs = td / "refs.json"
        refs.write_text(json.dumps({"packing_10000": float(pins["objective"])}))
        env = dict(os.environ, TARAL_PDHG=str(PDHG))
        subprocess.run([sys.executable, str(harness), str(f), "--out", str(td / "led"), "--configs", "cpu1",
                        "--tol", "1e-6", "--repeats", "1", "--ref-json", str(refs)], check=True, env=env,
                       stdout=subprocess.DEVNULL)
        row = json.loads((td / "led.json").read_text())["rows"][0]
    out = {"harness": "gpu/bench_pdhg.py", "fields": fields, "json_keys": json_keys, "pdhg_flags": flags,
           "model_sha256": lp.digest(), "reference_objective_via_ref_json": float(pins["objective"]),
           "reference_row_cpu1": row}
    (OUT / "reference_ledger.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote reference_ledger.json:", len(fields), "fields,", row["status"], row["iterations"])


if __name__ == "__main__":
    if "--ledger" in sys.argv:
        ledger()
    elif "--bench-lp" in sys.argv:
        bench_lp()
    elif "--refinery" in sys.argv:
        refinery()
    elif "--vector-check" in sys.argv:
        vector_check()
    else:
        main()
