#!/usr/bin/env python3
"""Benchmark: time to 1e-6 relative KKT error per LP on one B200 (N GPUs: N independent replicas).

Workload: the planted-optimum LP with power-law rows (m = 200,000 rows, n = 500,000 columns, ~5M nonzeros,
row lengths Zipf s = 1.2 capped at 2,000), FP32 matrix and iterates with FP64 averages / KKT / restarts,
tolerance 1e-6, seeded synthetic data (seed = rank). One step = one full solve of the LP:

* value -- the device-resident solve (power iteration, the PDHG loop with its restarts and evaluations, the
  final download of x and z) on a context created before the timed region; CUDA-event time on the engine's
  stream, L2 flushed (256 MiB write) between steps; max over ranks; seconds per LP for the whole job.
* e2e   -- the same solve through the public C ABI taral_pdhg_solve() from host arrays: host transposes,
  host-to-device upload of A, A^T and the vectors, scaling on the device, the solve, the device-to-host download
  and the original-space check, every step.

Once per run on rank 0 at N = 1, after the timed region (each can be skipped by its flag):
* fp64      -- the same LP solved with FP64 iterates (the reference's precision): device time, iterations
               against the reference's own FP64 count on this LP (--no-fp64);
* learned   -- the learned warm start on 24-period scenarios (trained on 512 solutions the engine computes, on 128
               held-out scenarios; batched, with the cold-start fallback) against cold batched and plain solves
               (--no-learned);
* family    -- the batched scenario family (512 refinery LPs of 4-48 periods) in one batched context against the
               plain single-instance engine, every status, the independent FP64 check of all answers, and an FP64
               objective oracle (this engine in FP64 to 1e-9 with a weak-duality certificate) on a stratified
               sample plus the 48-period refinery LP (--no-family);
* cpu_baseline -- one complete run of the reference's CPU PDHG (FP64, all host threads) to 1e-6 on the LP,
               and the reference's CPU IPM and dual simplex on a small planted LP (--no-cpu-baseline).
Also reported: the roofline of the dominant kernel (mean CUDA-event duration of the row-phase and column-phase
kernels launched one at a time on the engine stream, algorithmic bytes per launch, against the measured HBM
copy bandwidth) beside the random-gather floor measured in the same run, SM clocks sampled during the timed
region, and the number of engine kernels launched in it.

  python bench.py [--gpus N] [--steps K] [--warmup W]        our engine
  python bench.py --impl reference ...                       the reference's own PDHG (oracle/_ref/pdhg, built from
                                                             its sources): complete FP64 solves of the LP on its GPU
                                                             backend, and one complete run of its CPU backend
  python bench.py [--impl reference] --workload ledger       the reference's published workloads, FP64 (either arm)
  python bench.py --profile-blocks B                         ncu capture mode: B blocks of 64 steps, no report
  python bench.py --workload family [--instances 512]        the family block alone
  python bench.py --workload family --profile-blocks B       ncu capture mode of the batched engine (16 scenarios)
  python bench.py --workload warmstart [--train 512]         the learned warm start on the 24-period family
  python bench.py --workload gemm                            the tcgen05 GEMM's TFLOP/s on the MLP's shapes
  python bench.py --workload seeds                           the small planted LP (seeds 0-9) and the bench LP
                                                             (seeds 0-2) on both engines, the reference's CPU IPM,
                                                             dual simplex and PDHG included
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "taral-lp_b200"
for p in (PKG, ROOT / "oracle"):
    sys.path.insert(0, str(p))

# one process per GPU: each rank sees only its own device (set before CUDA is initialised anywhere)
if "LOCAL_RANK" in os.environ and "CUDA_VISIBLE_DEVICES" not in os.environ:
    os.environ["CUDA_VISIBLE_DEVICES"] = os.environ["LOCAL_RANK"]

WORKLOAD = dict(m=200_000, n=500_000, per_col=10, zipf=1.2, cap=2000, floor=5, tol=1e-6)
WORKLOAD_NAME = "planted LP, Zipf rows: m=200000 n=500000 ~5M nnz (row lengths Zipf s=1.2, cap 2000), tol 1e-6"
METRIC = "time-to-1e-6 rel KKT per LP"


def dist_max(v, dist, device="cuda"):
    """The maximum over ranks of a per-rank time (whole-job time of the replicas); v itself with one rank."""
    if not dist:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return t.item()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def make_lp(seed):
    import lpgen
    w = WORKLOAD
    return lpgen.planted(w["m"], w["n"], w["per_col"], seed=seed, zipf=w["zipf"], cap=w["cap"], floor=w["floor"],
                         name=f"PLANTED_ZIPF_{seed}")


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.flush()
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]
        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) >= 9 and c[0] == vis:
                rows.append(c)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        load = [s for s in sm if s > 0.5 * mx] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


def flush_l2(torch, buf):
    buf.zero_()
    torch.cuda.synchronize()


# ------------------------------------------------------------------------------------------------ reference
def ref_binary():
    return ROOT / "oracle" / "_ref" / "pdhg"


def ref_cpu_solver(lp, method, cap_s):
    """One run of the reference's single-threaded CPU engine `method` ("ipm" or "dual": `oracle/_ref/taral --method`)
    on the LP, capped at cap_s seconds: wall seconds, status and the objective's error against the planted optimum."""
    taral = ROOT / "oracle" / "_ref" / "taral"
    with tempfile.TemporaryDirectory() as td:
        f, j = Path(td) / "p.mps", Path(td) / "p.json"
        lp.write_mps(f)
        t0 = time.perf_counter()
        try:
            subprocess.run([str(taral), str(f), "--method", method, "--time-limit", str(cap_s), "--json", str(j)],
                           check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=cap_s + 60)
            rep = json.loads(j.read_text())
            return {"s": time.perf_counter() - t0, "status": rep.get("status"),
                    "objective_rel_err": abs(rep["objective"] - lp.obj_star) / abs(lp.obj_star)}
        except (subprocess.SubprocessError, OSError, ValueError, KeyError) as e:
            return {"s": time.perf_counter() - t0, "status": f"failed: {type(e).__name__}"}


def cpu_solvers(cap_s=120.0, with_engine=True):
    """The reference's own CPU dual simplex and IPM (single-threaded engines of `oracle/_ref/taral`, each capped at
    cap_s seconds) and this engine on the small planted LP (2,000 x 5,000, 5 nonzeros per column, seed 1), timed
    in this run on this host, with the objective errors against the planted optimum. A reported baseline only."""
    import lpgen
    taral = ROOT / "oracle" / "_ref" / "taral"
    if not taral.exists():
        return None
    lp = lpgen.planted(2000, 5000, 5, seed=1)
    out = {"workload": "planted LP m=2000 n=5000, 5 nonzeros per column, seed 1, tol 1e-6", "cores": 1,
           "cap_s": cap_s, "planted_objective": lp.obj_star}
    for method in ("ipm", "dual"):
        out[method] = ref_cpu_solver(lp, method, cap_s)
    if not with_engine:
        return out
    import pdhg
    for name, prec in (("gpu_pdhg_fp32", pdhg.FP32), ("gpu_pdhg_fp64", pdhg.FP64)):
        pdhg.solve(lp, tol=1e-6, precision=prec)  # untimed first call
        ts, r = [], None
        for _ in range(3):
            t0 = time.perf_counter()
            r, _, _ = pdhg.solve(lp, tol=1e-6, precision=prec)
            ts.append(time.perf_counter() - t0)
        out[name] = {"s": sorted(ts)[1], "status": r["status"], "iterations": r["iterations"],
                     "objective_rel_err": abs(r["objective"] - lp.obj_star) / abs(lp.obj_star),
                     "what": "taral_pdhg_solve from host arrays, median of 3"}
    return out


_MPS_FILES = []  # (model, path): each model the reference binary reads is written once per process
_MPS_DIR = None


def mps_file(lp):
    """The model as an MPS file, written on first use into a temporary directory that lives as long as the process."""
    global _MPS_DIR
    for m, f in _MPS_FILES:
        if m is lp:
            return f
    if _MPS_DIR is None:
        _MPS_DIR = tempfile.TemporaryDirectory()
    f = Path(_MPS_DIR.name) / f"m{len(_MPS_FILES)}.mps"
    lp.write_mps(f)
    _MPS_FILES.append((lp, f))
    return f


def run_reference(lp, device, tol=1e-6, limit_s=900.0, threads=0, max_iter=None):
    """One run of the reference binary (oracle/_ref/pdhg, FP64, built from the reference's sources) on the model:
    its JSON report plus the wall time of the process, or {"status": "failed: ..."}."""
    f = mps_file(lp)
    cmd = [str(ref_binary()), str(f), "--device", device, "--tol", str(tol), "--time-limit", str(limit_s)]
    if device == "cpu":
        cmd += ["--threads", str(threads or os.cpu_count() or 1)]
    if max_iter:
        cmd += ["--max-iter", str(max_iter)]
    with tempfile.TemporaryDirectory() as td:
        j = Path(td) / "r.json"
        t0 = time.perf_counter()
        try:
            subprocess.run(cmd + ["--json", str(j)], check=True, stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL, timeout=limit_s + 300)
            rep = json.loads(j.read_text())
        except (subprocess.SubprocessError, OSError, ValueError) as e:
            return {"status": f"failed: {type(e).__name__}"}
        wall = time.perf_counter() - t0
    out = {k: rep.get(k) for k in ("status", "iterations", "restarts", "objective", "setup_s", "solve_s", "total_s",
                                   "power_iter_s", "precision", "device", "threads")}
    out["process_wall_s"] = wall
    return out


def reference_cpu_complete(lp, threads):
    """One complete run of the reference CPU PDHG (--device cpu, FP64, `threads` host threads) to 1e-6 on the LP,
    measured (no projection), as a cpu_baseline dict."""
    rep = run_reference(lp, "cpu", threads=threads, limit_s=1200.0)
    if not str(rep.get("status", "")).startswith("near"):
        return {"value": None, "unit": "s", "cores": threads, "kind": "reference", "complete_runs": 0,
                "sample": f"one run of the reference CPU PDHG (FP64, {threads} threads) to 1e-6: {rep.get('status')}"}
    return {"value": rep["solve_s"], "unit": "s", "cores": threads, "kind": "reference", "complete_runs": 1,
            "total_s": rep["total_s"], "iterations": rep["iterations"], "status": rep["status"],
            "objective": rep["objective"],
            "sample": f"one complete run of the reference CPU PDHG (oracle/_ref/pdhg --device cpu --threads {threads}, "
                      f"FP64) on this LP to 1e-6 rel KKT, measured: value = its solve time, total_s = with its MPS "
                      f"parse and scaling"}


REF_BENCH_LP = ROOT / "tests" / "golden" / "reference_bench_lp.json"


def fp64_iterations(lp):
    """The reference's own FP64 iteration count to 1e-6 on the benchmark LP (seed 0), from its full CPU run recorded
    by `tests/golden/make_golden.py --bench-lp` (the model's sha256 is checked against the fixture's)."""
    d = json.loads(REF_BENCH_LP.read_text())
    if d["model_sha256"] != lp.digest():
        raise RuntimeError("the benchmark LP differs from the one in " + REF_BENCH_LP.name)
    return d["iterations"], d["status"]


def lp_config(m, n, nnz):
    """The `config` object of both arms (the same workload, so the same keys and values)."""
    return {"workload": WORKLOAD_NAME, "m": m, "n": n, "nnz": nnz, "tol": WORKLOAD["tol"], "seed": "rank (0 at N=1)",
            "parallelism": "replicas (one LP per GPU)",
            "l2": "inputs larger than L2 (~190 MB of matrices and vectors); L2 flushed (256 MiB write) between steps "
                  "of this engine, every step of the reference re-reads its model and uploads it anew"}


def reference_arm(args, rank, world):
    """The reference's own implementation of the path, unmodified, through its public interface (the `pdhg` CLI on
    an MPS file): `value` is the median solve time of complete FP64 runs of its GPU backend to 1e-6 on this LP (W
    untimed runs, then K timed), and `e2e` carries the line's own value; the median of the same runs' totals (its
    MPS parse, host scaling, upload and solve, a span this engine's e2e does not match: it starts from host arrays)
    is reported beside it as `total_s_median`.
    Its FP32 mode does not reach 1e-6 on this LP (time_limit), so FP64 is the reference's configuration here.
    `cpu_baseline`: one complete run of its CPU backend on all host threads, measured."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    lp = make_lp(0)
    if not ref_binary().exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/pdhg was not built (make -C oracle ref)"}))
        return
    n_it, _ = fp64_iterations(lp) if REF_BENCH_LP.exists() else (None, None)
    runs = []
    for s in range(args.warmup + args.steps):
        rep = run_reference(lp, "gpu", limit_s=600.0)
        print(json.dumps({"reference_gpu_run": s, **rep}), file=sys.stderr, flush=True)
        if s >= args.warmup:
            runs.append(rep)
    ok = [r for r in runs if r.get("solve_s") is not None]
    if not ok:
        print(json.dumps({"impl": "reference", "unavailable": "the reference GPU backend failed: " +
                          str(runs[0].get("status") if runs else "no run")}))
        return
    v = statistics.median(r["solve_s"] for r in ok)
    e2e = statistics.median(r["total_s"] for r in ok)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp64", "data": "synthetic", "config": lp_config(lp.m, lp.n, lp.nnz),
            "run": {"what": "oracle/_ref/pdhg --device gpu --tol 1e-6 (FP64, its default) per step, the reference's "
                            "stock CLI on the LP written as MPS",
                    "statuses": [r.get("status") for r in runs], "iterations": [r.get("iterations") for r in runs],
                    "reference_fp64_iterations_on_cpu": n_it, "restarts": ok[-1].get("restarts"),
                    "objective": ok[-1].get("objective"),
                    "objective_rel_err_vs_planted": abs(ok[-1]["objective"] - lp.obj_star) / abs(lp.obj_star),
                    "solve_s": [r.get("solve_s") for r in runs], "total_s": [r.get("total_s") for r in runs],
                    "process_wall_s": [r.get("process_wall_s") for r in runs], "device": ok[-1].get("device")},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                    "what": "the line's own value (median solve_s); its copies happen inside its process",
                    "total_s_median": e2e,
                    "total_what": "median total_s of the timed runs: the reference's own clock from reading the MPS "
                                  "file to its answer (parse, host scaling, upload, solve, check)"}}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = reference_cpu_complete(lp, threads)
        line["cpu_baseline"]["solvers_small_lp"] = cpu_solvers(with_engine=False)
    print(json.dumps(line))


# ------------------------------------------------------------------------------------------------ our engine
def algorithmic_bytes(m, n, nnz, fp32=True):
    """Per-launch bytes the row-phase and column-phase kernels must move (each datum once):
    row phase (A, m rows):    8 nnz (val f32 + idx i32) + 4 (m+1) ptr + 4 n (x gathered once)
                              + 40 m (z r/w 8, Ax r/w 8, rl ru 8, zs f64 r/w 16)
    column phase (A^T, n rows): 8 nnz + 4 (n+1) + 4 m (z gathered once)
                              + 40 n (x r/w 8, c l u 12, xs f64 r/w 16, ATz w 4)"""
    vb = 4 if fp32 else 8
    row = (4 + vb) * nnz + 4 * (m + 1) + vb * n + (4 * vb + 8 + 16) * m
    col = (4 + vb) * nnz + 4 * (n + 1) + vb * m + (5 * vb + 16) * n
    return row, col


def traffic_from_profile():
    """DRAM bytes per launch of the row / column phase kernels from the committed ncu summary, or None."""
    p = ROOT / "profiles" / "roofline_traffic.txt"
    if not p.exists():
        return None
    out = {}
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) == 2 and not line.startswith("#"):
            out[parts[0]] = int(parts[1])
    return out


def gather_floor(nnz):
    """The random-gather floor of this GPU, measured now by the committed probe (bin/gather_floor: `nnz` int32 index +
    float value pairs and one uniformly random float gather each, L2 flushed before every launch): {vector length:
    microseconds per launch} for the vector lengths 500,000 (x, gathered by the row phase) and 200,000 (z, column
    phase), or None when the probe is missing or fails."""
    probe = ROOT / "taral-lp_b200" / "bin" / "gather_floor"
    if not probe.exists():
        return None
    try:
        out = subprocess.run([str(probe), str(int(nnz))], capture_output=True, text=True, timeout=300, check=True)
        rows = [json.loads(line) for line in out.stdout.splitlines() if line.startswith("{")]
        return {int(r["n"]): float(r["l2_gather_us"]) for r in rows}
    except (subprocess.SubprocessError, OSError, ValueError, KeyError):
        return None


def our_arm(args, rank, world, dist):
    import torch
    import pdhg
    torch.cuda.set_device(0)
    lp = make_lp(rank)
    eng = pdhg.Engine.from_model(lp, precision=pdhg.FP32)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    tol = WORKLOAD["tol"]

    if args.profile_blocks:  # ncu capture mode
        eng.set_steps(0.5, 0.5)
        eng.start()
        for _ in range(args.profile_blocks):
            eng.iterate(64)
        eng.eval_pair(1 / 64)
        return

    def barrier():
        if dist:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        eng.solve(eng.bnorm, eng.cnorm, tol=tol, want_point=False)
        flush_l2(torch, flush)
    clocks = Clocks()
    clocks.start()
    barrier()
    dev_s, launches, its, outs = 0.0, 0, [], []
    for _ in range(args.steps):
        r, _, _ = eng.solve(eng.bnorm, eng.cnorm, tol=tol)
        dev_s += r["device_s"]
        launches += r["kernel_launches"]
        its.append(r["iterations"])
        outs.append(r)
        flush_l2(torch, flush)
    barrier()
    clk = clocks.stop()
    value = dist_max(dev_s, dist) / (world * args.steps)  # LPs of all replicas / the slowest rank's time

    # e2e through the public API from host arrays (scaling, upload, solve, download, check every step), after one
    # untimed call (the first call in a process also loads the library's kernels)
    pdhg.solve(lp, tol=tol, precision=pdhg.FP32)
    barrier()
    t0 = time.perf_counter()
    e2e_out, e2e_steps = [], []
    for _ in range(args.steps):
        ts = time.perf_counter()
        r, x, y = pdhg.solve(lp, tol=tol, precision=pdhg.FP32)
        e2e_steps.append(time.perf_counter() - ts)
        e2e_out.append(r)
    torch.cuda.synchronize()
    e2e_value = dist_max(time.perf_counter() - t0, dist) / (world * args.steps)
    nnz = e2e_out[0]["nnz"]
    m, n = lp.m, lp.n
    # uploaded per solve: A and A^T unscaled (int32 ptr, int32 idx, f64 val: scaled and narrowed on the device),
    # c l u Dc (f32, n), rl ru Dr (f32, m), the power-iteration start vector (f64, n); downloaded: Dr, Dc (f64),
    # x and z (f64) and 20 KKT doubles per evaluated block
    h2d = 2 * 12 * nnz + 4 * (m + 1) + 4 * (n + 1) + 16 * n + 12 * m + 8 * n
    d2h = 16 * (m + n) + 8 * 20 * (e2e_out[0]["iterations"] // 64 + 2)

    # roofline of the dominant kernel: one-at-a-time launches bracketed by CUDA events on the engine stream
    row_ms, col_ms = eng.profile_phases(64)
    brow, bcol = algorithmic_bytes(m, n, nnz)
    row_gbs, col_gbs = brow / (row_ms * 1e-3) / 1e9, bcol / (col_ms * 1e-3) / 1e9
    peak, peak_kind = peaks()
    dom = "row" if row_ms >= col_ms else "col"
    tr = traffic_from_profile()
    traffic = tr.get(dom) if tr else None
    floor = gather_floor(nnz) if rank == 0 and (m, n) == (200_000, 500_000) else None

    if rank == 0:
        once = world == 1  # the once-per-run blocks: rank 0 at N = 1 only
        fp64 = fp64_block(lp) if once and not args.no_fp64 else None
        family = family_block(args) if once and not args.no_family else None
        learned = warmstart_block(512, 128, 4, args.epochs) if once and not args.no_learned else None
        cpu = None
        if once and not args.no_cpu_baseline and ref_binary().exists():
            cpu = reference_cpu_complete(lp, os.cpu_count() or 1)
            cpu["solvers_small_lp"] = cpu_solvers()
        r0 = outs[-1]
        line = {
            "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1e3 * world, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": lp_config(m, n, nnz),
            "run": {"precision": "fp32 matrix/iterates, fp64 averages/KKT/restarts", "iterations": its,
                    "restarts": r0["restarts"], "status": r0["status"],
                    "rel_kkt": max(r0["rel_primal"], r0["rel_dual"], r0["rel_gap"]),
                    "objective_rel_err_vs_planted": abs(e2e_out[-1]["objective"] - lp.obj_star) / abs(lp.obj_star)},
            "e2e": {"value": e2e_value, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "phases_s": {k: e2e_out[-1][k] for k in ("scale_s", "device_init_s", "transfer_s", "solve_s")},
                    "steps_s": e2e_steps, "warmup_calls": 1},
            "roofline": {"bound": "hbm", "kernel": f"{dom}-phase SpMV + fused step (" + ("k_rowblock" if dom == "row" else "k_rowthread or k_rowblock, the tuner's choice") + ")",
                         "achieved": row_gbs if dom == "row" else col_gbs, "peak": peak, "unit": "GB/s",
                         "frac": (row_gbs if dom == "row" else col_gbs) / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "row_ms": row_ms, "col_ms": col_ms,
                         "bytes_per_launch": {"row": brow, "col": bcol}, "other_gbs": col_gbs if dom == "row" else row_gbs,
                         "gather_floor": None if not floor else {
                             "row_us": floor.get(n), "col_us": floor.get(m),
                             "row_frac": floor[n] / (row_ms * 1e3) if n in floor else None,
                             "col_frac": floor[m] / (col_ms * 1e3) if m in floor else None,
                             "source": "bin/gather_floor in this run: the same count of random 4-byte gathers "
                                       "with their index/value stream, L2 flushed before each launch"}},
            "fp64": fp64,
            "family": family,
            "learned": learned,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line))


def fp64_block(lp):
    """The bench LP with FP64 iterates (the reference's precision): one solve through taral_pdhg_solve from host
    arrays (end to end, like `e2e`; it also loads the FP64 kernels), then one on a resident context, timed with CUDA
    events like `value`."""
    import pdhg
    tol = WORKLOAD["tol"]
    t0 = time.perf_counter()
    r_e2e, _, _ = pdhg.solve(lp, tol=tol, precision=pdhg.FP64)
    e2e_s = time.perf_counter() - t0
    eng = pdhg.Engine.from_model(lp, precision=pdhg.FP64)
    r, _, _ = eng.solve(eng.bnorm, eng.cnorm, tol=tol, want_point=False)
    eng.close()
    n_it, _ = fp64_iterations(lp) if REF_BENCH_LP.exists() else (None, None)
    return {"device_s": r["device_s"], "e2e_s": e2e_s, "iterations": r["iterations"], "restarts": r["restarts"],
            "status": r["status"], "reference_fp64_iterations": n_it,
            "iterations_equal_reference": None if n_it is None else (r["iterations"] == n_it == r_e2e["iterations"]),
            "objective": r_e2e["objective"],
            "objective_rel_err_vs_planted": abs(r_e2e["objective"] - lp.obj_star) / abs(lp.obj_star)}


# The reference's own published GPU workloads (gpu/gen_lp.py models, reproduced byte for byte by lpgen), FP64 to
# 1e-6, with the iteration counts of its ledgers (results/gpu_pdhg/synth_packing_tol1e-6.csv:12,
# synth_transport_tol1e-6.csv:12) and its published solve times on an RTX 5050 laptop GPU.
LEDGER = {"packing_1M": (lambda lpgen: lpgen.packing(1_000_000), 6848, 23.70),
          "transport_1000x1000": (lambda lpgen: lpgen.transport(1000, 1000), 73344, 35.41)}


def ledger_arm(args, reference):
    """`--workload ledger`: the reference's published PDHG workloads on this GPU, FP64 to 1e-6 (their ledger
    precision). Ours: `taral_pdhg_solve` from host arrays (median of `--steps` after one untimed call), FP64 and FP32.
    Reference (`--impl reference`): its own GPU backend, `oracle/_ref/pdhg --device gpu`, one run each."""
    import lpgen
    out = {}
    for name, (make, ledger_it, published_s) in LEDGER.items():
        lp = make(lpgen)
        row = {"ledger_iterations": ledger_it, "published_solve_s_rtx5050": published_s}
        if reference:
            row["reference_gpu_fp64"] = run_reference(lp, "gpu", limit_s=600.0)
        else:
            import pdhg
            for tag, prec in (("fp64", pdhg.FP64), ("fp32", pdhg.FP32)):
                pdhg.solve(lp, tol=1e-6, precision=prec)
                ts, r = [], None
                for _ in range(max(args.steps, 1)):
                    t0 = time.perf_counter()
                    r, _, _ = pdhg.solve(lp, tol=1e-6, precision=prec)
                    ts.append(time.perf_counter() - t0)
                row[tag] = {"e2e_s": statistics.median(ts), "solve_s": r["solve_s"], "iterations": r["iterations"],
                            "status": r["status"], "objective": r["objective"]}
        out[name] = row
        print(json.dumps({name: row}), file=sys.stderr, flush=True)
    print(json.dumps({"impl": "reference" if reference else "ours", "workload": "ledger", "tol": 1e-6,
                      "models": out}))


def family_lps(count, seed=2024):
    """The batched scenario family: `count` refinery LPs of 4 to 48 periods (seeded), prices and capacities scaled
    by independent U(0.8, 1.2) factors. Returns (lps, periods)."""
    import numpy as np
    import lpgen
    rng = np.random.default_rng(seed)
    periods = rng.integers(4, 49, size=count)
    base = lpgen.RefineryBase(48, seed=7)
    P = lpgen.perturbations(count, seed=seed + 1)
    return [base.instance(int(T), p) for T, p in zip(periods, P)], periods


def family_profile(args):
    """ncu capture mode of the batched engine: 16 scenarios of the family structure (8 of 20 periods, 8 of 24
    periods: two distinct matrices), `--profile-blocks` blocks of 64 iterations, no report."""
    import lpgen
    import pdhg
    base = lpgen.RefineryBase(24, seed=7)
    P = lpgen.perturbations(16, seed=5)
    lps = [base.instance(24 if i % 2 else 20, p) for i, p in enumerate(P)]
    b = pdhg.Batch(lps, tol=WORKLOAD["tol"], precision=pdhg.FP32, max_iter=64 * max(args.profile_blocks, 1))
    res, _, _ = b.solve(want_points=False)
    print("profiled", len(res), "scenarios,", res[0]["iterations"], "iterations")


def fp64_oracle(lp, tol=1e-9, time_limit=300.0):
    """The FP64 objective oracle of a refinery LP (only a feasible point is planted there): this engine with FP64
    iterates to `tol` relative KKT, and the weak-duality bound of its dual vector from the independent device check
    (the reference checker's rule): objective, certified relative gap between them, status and time."""
    import pdhg
    t0 = time.perf_counter()
    r, x, y = pdhg.solve(lp, tol=tol, precision=pdhg.FP64, time_limit=time_limit)
    dt = time.perf_counter() - t0
    c = pdhg.check_models([lp], [x], [y])[0]
    lb = c["dual_bound"] if c["dual_bound"] is not None else c["dual_obj_loose"]
    return {"objective": r["objective"], "status": r["status"], "iterations": r["iterations"], "seconds": dt,
            "dual_bound": lb, "strict_bound": c["dual_bound"] is not None,
            "certified_gap_rel": None if lb is None else abs(r["objective"] - lb) / max(1.0, abs(r["objective"]))}


def family_block(args):
    """The batched scenario family: all scenarios in one batched context (FP32 iterates, FP64 per-instance restart
    state) against the plain single-instance FP32 engine on a stratified sample (fastest of 3 runs each; the plain
    per-LP time of the whole family is the least-squares line in the period count through the sample, evaluated at
    every scenario's period count), the independent FP64 check of every answer, and the FP64 objective oracle on a
    stratified sample and on the 48-period refinery LP."""
    import numpy as np
    import lpgen
    import pdhg
    tol = WORKLOAD["tol"]
    t0 = time.perf_counter()
    lps, periods = family_lps(args.instances)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    b = pdhg.Batch(lps, tol=tol, precision=pdhg.FP32, time_limit=3000)
    res, bx, by = b.solve()
    batch_s = time.perf_counter() - t0
    info = b.info()
    b.close()
    t0 = time.perf_counter()
    chk = pdhg.check_models(lps, bx, by)
    check_s = time.perf_counter() - t0
    del bx, by
    order = np.argsort(periods, kind="stable")
    pick = order[np.linspace(0, len(order) - 1, min(args.sample, len(order))).round().astype(int)]
    plain_t, plain_T, obj_diff, plain_it = [], [], [], []
    for i in pick:
        dt = float("inf")
        for _ in range(3):
            t0 = time.perf_counter()
            r, _, _ = pdhg.solve(lps[i], tol=tol, precision=pdhg.FP32, time_limit=600)
            dt = min(dt, time.perf_counter() - t0)
        plain_t.append(dt)
        plain_T.append(int(periods[i]))
        plain_it.append(int(r["iterations"]))
        obj_diff.append(abs(r["objective"] - res[i]["objective"]) / max(1.0, abs(r["objective"])))
    slope, icpt = np.polyfit(np.array(plain_T, float), np.array(plain_t), 1)
    plain_per_lp = float(np.mean(np.maximum(slope * periods + icpt, 0.0)))
    # FP64 objective oracle: a stratified sample of the family, then the 48-period refinery LP itself
    oracle_rows = []
    for i in order[np.linspace(0, len(order) - 1, min(args.oracle_sample, len(order))).round().astype(int)]:
        o = fp64_oracle(lps[i])
        o.update({"scenario": int(i), "periods": int(periods[i]), "batched_objective": res[i]["objective"],
                  "batched_rel_diff": abs(res[i]["objective"] - o["objective"]) / max(1.0, abs(o["objective"]))})
        oracle_rows.append(o)
        print("fp64 oracle", json.dumps(o), file=sys.stderr, flush=True)
    refinery48 = None
    if args.oracle_sample > 0:  # the 48-period refinery LP: plain FP32 solve against its FP64 oracle
        lp48 = lpgen.RefineryBase(48, seed=7).instance(48)
        t0 = time.perf_counter()
        r48, _, _ = pdhg.solve(lp48, tol=tol, precision=pdhg.FP32, time_limit=600)
        s48 = time.perf_counter() - t0
        o48 = fp64_oracle(lp48)
        refinery48 = {"m": lp48.m, "n": lp48.n, "nnz": lp48.nnz, "fp32_status": r48["status"],
                      "fp32_iterations": r48["iterations"], "fp32_e2e_s": s48, "fp32_objective": r48["objective"],
                      "fp64_oracle": o48,
                      "fp32_rel_diff": abs(r48["objective"] - o48["objective"]) / max(1.0, abs(o48["objective"]))}
    k = len(lps)
    its = [r["iterations"] for r in res]
    statuses = {}
    for r in res:
        statuses[r["status"]] = statuses.get(r["status"], 0) + 1
    return {"metric": "time-to-1e-6 rel KKT per LP, batched scenario family vs the plain engine",
            "workload": f"refinery scenario family: {k} LPs of 4-48 periods (1,500 rows x 4,000 columns per period), "
                        f"prices and capacities x U(0.8,1.2), tol {tol}, FP32 iterates",
            "rows_total": int(sum(lp.m for lp in lps)), "cols_total": int(sum(lp.n for lp in lps)),
            "nnz_total": info["nnz_total"], "nnz_stored": info["nnz_stored"],
            "distinct_matrices": info["distinct_matrices"], "device_mem_bytes": info["device_mem_bytes"],
            "batched": {"wall_s": batch_s, "per_lp_s": batch_s / k, "device_s": res[0]["device_s"],
                        "statuses": statuses, "iterations_mean": float(np.mean(its)), "iterations_max": int(max(its))},
            "plain_single_instance": {"per_lp_s_fit": plain_per_lp, "sample": len(pick), "sample_periods": plain_T,
                                      "sample_s": plain_t, "sample_iterations": plain_it,
                                      "fit_s_per_period": float(slope), "fit_intercept_s": float(icpt)},
            "speedup_per_lp": plain_per_lp / (batch_s / k),
            "objective_max_rel_diff_batched_vs_plain": float(max(obj_diff)),
            "independent_check": {"seconds": check_s,
                                  "max_row_violation_rel": max(c["row_violation_rel"] for c in chk),
                                  "max_bound_violation": max(c["bound_violation"] for c in chk),
                                  "max_dual_gap_rel": max(abs(c["dual_gap_rel"]) for c in chk if c["dual_gap_rel"] is not None),
                                  "strict_dual_bounds": sum(c["dual_bound"] is not None for c in chk),
                                  "max_objective_diff_vs_solver": max(abs(c["objective"] - r["objective"]) /
                                                                      max(1.0, abs(r["objective"])) for c, r in zip(chk, res))},
            "fp64_oracle": {"what": "this engine in FP64 to 1e-9 rel KKT; certified_gap_rel = |objective - weak-duality "
                                    "bound of its y| / max(1, |objective|) from the independent check",
                            "sample": oracle_rows,
                            "max_batched_rel_diff": max(o["batched_rel_diff"] for o in oracle_rows) if oracle_rows else None,
                            "max_certified_gap_rel": max((o["certified_gap_rel"] or 0.0) for o in oracle_rows) if oracle_rows else None},
            "refinery_48_periods": refinery48,
            "generate_s": gen_s}


def family_arm(args):
    print(json.dumps(family_block(args)))


def warmstart_block(train, instances, sample, epochs):
    """The learned warm start on the 24-period family: train on solutions of `train` scenarios (seeds disjoint from
    the evaluation seeds), then solve `instances` held-out scenarios cold and warm (with the fallback rule), all in
    batched contexts, and `sample` of them with the plain single-instance engine from host arrays (wall time, like
    the family block). Per-LP times of the batched runs are their solve calls' wall time divided by the count."""
    import numpy as np
    import lpgen
    import pdhg
    import warmstart as W
    T = 24
    base = lpgen.RefineryBase(T, seed=7)
    Ptr, Pev = lpgen.perturbations(train, seed=100), lpgen.perturbations(instances, seed=999)
    t0 = time.perf_counter()
    tr = [base.instance(T, p) for p in Ptr]
    ev = [base.instance(T, p) for p in Pev]
    gen_s = time.perf_counter() - t0
    outs, xs, ys, data_s = W.solve_batch(tr, tol=1e-5)
    t0 = time.perf_counter()
    ws = W.train(Ptr, xs, ys, np.array([r["primal_weight"] for r in outs]), epochs=epochs)
    train_s = time.perf_counter() - t0
    del xs, ys
    res = W.evaluate(ev, Pev, ws, tol=WORKLOAD["tol"])
    plain, plain_it = [], []
    for i in range(min(sample, len(ev))):
        t0 = time.perf_counter()
        r, _, _ = pdhg.solve(ev[i], tol=WORKLOAD["tol"], precision=pdhg.FP32, time_limit=600)
        plain.append(time.perf_counter() - t0)
        plain_it.append(int(r["iterations"]))
    k = len(ev)
    warm_total = res["warm_s"] + res["probe_s"] + res["predict_s"]
    plain_lp = float(np.mean(plain)) if plain else None
    statuses = {}
    for st in res["warm_status"]:
        statuses[st] = statuses.get(st, 0) + 1
    return {"metric": "time-to-1e-6 rel KKT per LP, learned warm start + batched vs the plain engine",
            "workload": f"refinery family, {T} periods ({ev[0].m} rows x {ev[0].n} columns), {train} training / "
                        f"{k} held-out scenarios (disjoint seeds), tol {WORKLOAD['tol']}, FP32 iterates",
            "mlp": f"256 -> 512 x 3 (GELU) -> {ev[0].n + ev[0].m + 1}, bf16 weights, fp32 accumulate, tcgen05 GEMMs",
            "train": {"solutions_s": data_s, "train_s": train_s, "final_loss": ws.net.last_loss,
                      "generate_s": gen_s, "epochs": epochs},
            "cold_batched": {"per_lp_s": res["cold_s"] / k, "iterations_mean": float(np.mean(res["cold_iterations"]))},
            "learned_batched": {"per_lp_s": warm_total / k, "iterations_mean": float(np.mean(res["warm_iterations"])),
                                "used_warm": int(sum(res["used_warm"])), "probe_s": res["probe_s"],
                                "predict_s": res["predict_s"], "statuses": statuses},
            "plain_single_instance": {"per_lp_s": plain_lp, "sample": len(plain),
                                      "iterations_mean": float(np.mean(plain_it)) if plain_it else None},
            "speedup_learned_batched_vs_plain": None if plain_lp is None else plain_lp / (warm_total / k),
            "objective_max_rel_diff_warm_vs_cold": float(max(abs(a - b) / max(1.0, abs(a)) for a, b in
                                                             zip(res["cold_objective"], res["warm_objective"])))}


def warmstart_arm(args):
    print(json.dumps(warmstart_block(args.train, args.instances, args.sample, args.epochs)))


def gemm_arm(args):
    """`--workload gemm`: the tcgen05 GEMM (taral_gemm_bf16_umma) on the warm-start MLP's three GEMM shapes at the
    24-period output width (132,001) and batch 256, and on an 8192-cube, against the mma.sync GEMM
    (taral_gemm_bf16) on the same operands: CUDA-event time per call (mean of 20 after 3 warm-ups), TFLOP/s = 2 M N K /
    time, and the fraction of the measured dense BF16 peak."""
    import ctypes as C
    import torch
    import pdhg
    L = pdhg.lib()
    dev = torch.device("cuda")
    pk = ROOT / "MEASURED_PEAKS.json"
    peak, kind = (json.loads(pk.read_text()).get("bf16_tflops"), "measured") if pk.exists() else (1590.0, "fallback")
    if peak is None:
        peak, kind = 1590.0, "fallback"
    out_w, ld_w = 132001, 132008

    def bf(shape):
        return (torch.randn(shape, device=dev) * 0.1).to(torch.bfloat16)
    cases = [  # name, M, N, K, A (tensor, ld, mn), B (tensor, ld, mn), slices, mma.sync form (ta, tb) or None
        ("forward: Z = H W^T, last layer", 256, out_w, 512, (bf((256, 512)), 512, 0), (bf((out_w, 512)), 512, 0), 1,
         (0, 1)),
        ("dW = H^T dZ, last layer", 512, out_w, 256, (bf((256, 512)), 512, 1), (bf((256, ld_w)), ld_w, 1), 1, None),
        ("dH = dZ W^T, last layer (split K)", 256, 512, out_w, (bf((256, ld_w)), ld_w, 0), (bf((out_w, 512)), 512, 1),
         37, None),
        ("square 8192^3", 8192, 8192, 8192, (bf((8192, 8192)), 8192, 0), (bf((8192, 8192)), 8192, 0), 1, (0, 1)),
    ]
    rows = []
    for name, M, N, K, (a, lda, amn), (b, ldb, bmn), slices, mma in cases:
        c = torch.empty((M, N), dtype=torch.float32, device=dev)
        ws = torch.empty(max(slices, 1) * M * N if slices > 1 else 1, dtype=torch.float32, device=dev)
        err = torch.zeros(1, dtype=torch.int32, device=dev)

        def umma():
            code = L.taral_gemm_bf16_umma(M, N, K, C.c_void_p(a.data_ptr()), lda, amn, C.c_void_p(b.data_ptr()), ldb,
                                          bmn, C.c_void_p(c.data_ptr()), N, slices, C.c_void_p(ws.data_ptr()),
                                          C.c_void_p(err.data_ptr()), None)
            assert code == pdhg.OK, code

        def timed(fn, reps=20):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps * 1e-3
        t = timed(umma)
        assert int(err.item()) == 0
        row = {"gemm": name, "M": M, "N": N, "K": K, "tcgen05_us": t * 1e6, "tcgen05_tflops": 2.0 * M * N * K / t / 1e12}
        row["frac_of_peak"] = row["tcgen05_tflops"] / peak
        if mma is not None:
            wsz = torch.empty(1, dtype=torch.float32, device=dev)

            def sync_gemm():
                code = L.taral_gemm_bf16(M, N, K, mma[0], mma[1], C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                         C.c_void_p(c.data_ptr()), 1, C.c_void_p(wsz.data_ptr()), None)
                assert code == pdhg.OK, code
            t2 = timed(sync_gemm, reps=5)
            row["mma_sync_us"], row["mma_sync_tflops"] = t2 * 1e6, 2.0 * M * N * K / t2 / 1e12
        rows.append(row)
        print(json.dumps(row), file=sys.stderr, flush=True)
    print(json.dumps({"workload": "gemm", "peak_bf16_tflops": peak, "peak_kind": kind, "rows": rows}))


def seeds_arm(args):
    """`--workload seeds`: the two planted LPs over their seeds (small LP 0-9, bench LP 0-2), on both engines.
    * the small planted LP (2,000 x 5,000, 5 nonzeros per column, seeds 0-9): this engine in FP32 and FP64 from host
      arrays (median of 3 after a warm-up call), the reference's CPU PDHG (FP64, all host threads) and its
      single-threaded CPU IPM and dual simplex (one process per seed and method, run side by side on the host's
      cores, capped at --cap seconds), with every objective's error against the planted optimum;
    * the bench LP (seeds 0-2): this engine in FP32 and FP64 from host arrays and the reference's GPU backend (FP64).
    Prints one JSON line with the per-seed results and their medians."""
    import concurrent.futures as cf
    import lpgen
    import pdhg
    tol = WORKLOAD["tol"]

    def ours(lp, prec, reps):
        pdhg.solve(lp, tol=tol, precision=prec)
        ts, r = [], None
        for _ in range(reps):
            t0 = time.perf_counter()
            r, _, _ = pdhg.solve(lp, tol=tol, precision=prec)
            ts.append(time.perf_counter() - t0)
        return {"s": statistics.median(ts), "status": r["status"], "iterations": r["iterations"],
                "objective_rel_err": abs(r["objective"] - lp.obj_star) / abs(lp.obj_star)}

    def ref(lp, device):
        rep = run_reference(lp, device, tol=tol, limit_s=args.cap if device == "cpu" else 900.0)
        ok = str(rep.get("status", "")).startswith("near")
        return {"solve_s": rep.get("solve_s"), "total_s": rep.get("total_s"), "status": rep.get("status"),
                "iterations": rep.get("iterations"),
                "objective_rel_err": abs(rep["objective"] - lp.obj_star) / abs(lp.obj_star) if ok else None}

    small = [lpgen.planted(2000, 5000, 5, seed=k) for k in range(10)]
    rows = [{"seed": k, "fp32": ours(lp, pdhg.FP32, 3), "fp64": ours(lp, pdhg.FP64, 3),
             "ref_cpu_pdhg": ref(lp, "cpu")} for k, lp in enumerate(small)]
    cores = os.cpu_count() or 1
    with cf.ThreadPoolExecutor(max_workers=max(1, min(20, cores // 2))) as ex:
        jobs = {(k, m): ex.submit(ref_cpu_solver, lp, m, args.cap) for k, lp in enumerate(small) for m in ("ipm", "dual")}
        for (k, m), fut in jobs.items():
            rows[k]["ref_" + m] = fut.result()

    def med(key, field):
        v = [r[key][field] for r in rows if r[key].get(field) is not None]
        return statistics.median(v) if v else None

    small_out = {"workload": "planted LP m=2000 n=5000, 5 nonzeros per column, seeds 0-9, tol 1e-6",
                 "host_cores": cores, "cap_s": args.cap, "seeds": rows,
                 "median_s": {"fp32": med("fp32", "s"), "fp64": med("fp64", "s"),
                              "ref_cpu_pdhg_solve": med("ref_cpu_pdhg", "solve_s"),
                              "ref_cpu_pdhg_total": med("ref_cpu_pdhg", "total_s"),
                              "ref_ipm": med("ref_ipm", "s"), "ref_dual": med("ref_dual", "s")},
                 "how": "this engine: taral_pdhg_solve from host arrays, median of 3; reference PDHG: its own "
                        "solve_s / total_s; IPM and dual simplex: process wall time, up to "
                        f"{max(1, min(20, cores // 2))} single-threaded processes side by side"}
    big = []
    for k in range(3):
        lp = make_lp(k)
        big.append({"seed": k, "m": lp.m, "n": lp.n, "nnz": int(lp.col_ptr[-1]), "fp32": ours(lp, pdhg.FP32, 1),
                    "fp64": ours(lp, pdhg.FP64, 1), "ref_gpu_backend": ref(lp, "gpu")})
        del lp
    print(json.dumps({"workload": "seeds", "metric": METRIC, "unit": "s", "small_lp": small_out,
                      "bench_lp": {"workload": WORKLOAD_NAME, "seeds": big,
                                   "how": "this engine: taral_pdhg_solve from host arrays after a warm-up call; "
                                          "reference: its GPU backend (FP64), its solve_s and total_s"}}),
          flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--profile-blocks", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the complete CPU run of the reference")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 run of the bench LP")
    ap.add_argument("--no-family", action="store_true", help="skip the batched family block")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start block")
    ap.add_argument("--oracle-sample", type=int, default=4,
                    help="family scenarios given the FP64 objective oracle (0: no oracle, no 48-period LP)")
    ap.add_argument("--workload", choices=["lp", "family", "warmstart", "ledger", "gemm", "seeds"], default="lp",
                    help="lp: the single large LP (the bench line); family: the batched scenario family; "
                         "warmstart: the learned warm start on the 24-period family; ledger: the reference's "
                         "published PDHG workloads (both arms); seeds: every seed of the small planted LP and the "
                         "bench LP on both engines")
    ap.add_argument("--cap", type=float, default=120.0, help="seconds per reference CPU run in --workload seeds")
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--sample", type=int, default=12)
    ap.add_argument("--train", type=int, default=512)
    ap.add_argument("--epochs", type=int, default=400)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = world > 1
    if args.workload == "ledger":
        if rank == 0:
            ledger_arm(args, args.impl == "reference")
        return
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.workload == "gemm":
        if rank == 0:
            gemm_arm(args)
        return
    if args.workload == "seeds":
        if rank == 0:
            seeds_arm(args)
        return
    if args.workload in ("family", "warmstart"):
        if rank == 0:
            if args.workload == "family" and args.profile_blocks:
                family_profile(args)
            else:
                (family_arm if args.workload == "family" else warmstart_arm)(args)
        return
    if dist:
        import datetime
        import torch
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        our_arm(args, rank, world, dist)
    finally:
        if dist:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
