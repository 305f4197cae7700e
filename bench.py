#!/usr/bin/env python3
"""Benchmark: time to 1e-6 relative KKT error per LP on one B200 (N GPUs: N independent replicas).

Workload: the planted-optimum LP with power-law rows (m = 200,000 rows, n = 500,000 columns, ~5M nonzeros,
row lengths Zipf s = 1.2 capped at 2,000), FP32 matrix and iterates with FP64 averages / KKT / restarts,
tolerance 1e-6, seeded synthetic data (seed = rank). One step = one full solve of the LP:

* value -- the device-resident solve (power iteration, the PDHG loop with its restarts and evaluations, the
  final download of x and z) on a context created before the timed region; CUDA-event time on the engine's
  stream, L2 flushed (256 MiB write) between steps; max over ranks; seconds per LP for the whole job.
* e2e   -- the same solve through the public C ABI taral_pdhg_solve() from host arrays: host scaling,
  host-to-device upload of A, A^T and the vectors, the solve, the device-to-host download and the
  original-space check, every step.

Also reported: the roofline of the dominant kernel (mean CUDA-event duration of the row-phase and column-phase
kernels launched one at a time on the engine stream, algorithmic bytes per launch, against the measured HBM
copy bandwidth), the reference's own CPU PDHG timed on a bounded sample on this host, SM clocks sampled during
the timed region, and the number of engine kernels launched in it.

  python bench.py [--gpus N] [--steps K] [--warmup W]        our engine
  python bench.py --impl reference ...                       the reference CPU PDHG (oracle/_ref/pdhg)
  python bench.py --profile-blocks B                         ncu capture mode: B blocks of 64 steps, no report
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
REF_SAMPLE_ITERS = 256


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


def run_reference_sample(lp, iters, threads):
    """The reference CPU PDHG (--device cpu, FP64) on the model for `iters` iterations; per-iteration seconds."""
    with tempfile.TemporaryDirectory() as td:
        f, j = Path(td) / "m.mps", Path(td) / "r.json"
        lp.write_mps(f)
        subprocess.run([str(ref_binary()), str(f), "--device", "cpu", "--threads", str(threads), "--tol", "1e-6",
                        "--max-iter", str(iters), "--json", str(j)], check=True, stdout=subprocess.DEVNULL,
                       timeout=1800)
        rep = json.loads(j.read_text())
    per_it = (rep["solve_s"] - rep["power_iter_s"]) / max(rep["iterations"], 1)
    setup = rep["scale_s"] + rep["transfer_s"]
    return per_it, setup, rep


def fp64_iterations(lp):
    """Iterations the FP64 path needs to 1e-6 on this LP (equal to the reference's FP64 count: the FP64
    iteration counts agree with the reference on every pinned case)."""
    import pdhg
    r, _, _ = pdhg.solve(lp, tol=WORKLOAD["tol"], precision=pdhg.FP64)
    return r["iterations"], r["status"]


def reference_arm(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    lp = make_lp(0)
    if not ref_binary().exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/pdhg was not built (make -C oracle ref)"}))
        return
    n_it, st = fp64_iterations(lp)
    vals = []
    for s in range(args.warmup + args.steps):
        per_it, setup, rep = run_reference_sample(lp, REF_SAMPLE_ITERS, threads)
        if s >= args.warmup:
            vals.append(setup + rep["power_iter_s"] + per_it * n_it)
    v = statistics.median(vals)
    sample = (f"{REF_SAMPLE_ITERS} iterations of the reference CPU PDHG (--device cpu --threads {threads}, FP64) per "
              f"step; time-to-1e-6 = scale + power iteration + per-iteration time x {n_it} iterations (the FP64 "
              f"iteration count to 1e-6 on this LP)")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "seed": 0, "tol": WORKLOAD["tol"], "parallelism": "cpu threads",
                       "l2": "n/a (CPU)", "fp64_iterations_to_tol": n_it, "fp64_status": st},
            "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
    t = torch.tensor([dev_s], dtype=torch.float64, device="cuda")
    if dist:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    value = t.item() / (world * args.steps)

    # e2e through the public API from host arrays (scaling, upload, solve, download, check every step)
    barrier()
    t0 = time.perf_counter()
    e2e_out = []
    for _ in range(args.steps):
        r, x, y = pdhg.solve(lp, tol=tol, precision=pdhg.FP32)
        e2e_out.append(r)
    torch.cuda.synchronize()
    e2e_s = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
    if dist:
        torch.distributed.all_reduce(e2e_s, op=torch.distributed.ReduceOp.MAX)
    e2e_value = e2e_s.item() / (world * args.steps)
    nnz = e2e_out[0]["nnz"]
    m, n = lp.m, lp.n
    # uploaded per solve: A and A^T (int32 ptr, int32 idx, f32 val), c l u Dc (f32, n), rl ru Dr (f32, m), the
    # power-iteration start vector (f64, n); downloaded: x and z (f64) and 20 KKT doubles per evaluated block
    h2d = 2 * 8 * nnz + 4 * (m + 1) + 4 * (n + 1) + 16 * n + 12 * m + 8 * n
    d2h = 8 * (m + n) + 8 * 20 * (e2e_out[0]["iterations"] // 64 + 2)

    # roofline of the dominant kernel: one-at-a-time launches bracketed by CUDA events on the engine stream
    row_ms, col_ms = eng.profile_phases(64)
    brow, bcol = algorithmic_bytes(m, n, nnz)
    row_gbs, col_gbs = brow / (row_ms * 1e-3) / 1e9, bcol / (col_ms * 1e-3) / 1e9
    peak, peak_kind = peaks()
    dom = "row" if row_ms >= col_ms else "col"
    tr = traffic_from_profile()
    traffic = tr.get(dom) if tr else None

    if rank == 0:
        cpu = None
        if ref_binary().exists() and world == 1 and not args.no_cpu_baseline:
            n_it, _ = fp64_iterations(lp)
            threads = os.cpu_count() or 1
            per_it, setup, rep = run_reference_sample(lp, REF_SAMPLE_ITERS, threads)
            cpu = {"value": setup + rep["power_iter_s"] + per_it * n_it, "unit": "s", "cores": threads,
                   "kind": "reference",
                   "sample": f"{REF_SAMPLE_ITERS} iterations of the reference CPU PDHG (FP64, {threads} threads) "
                             f"on this LP, projected to the {n_it} FP64 iterations to 1e-6 plus its setup"}
        r0 = outs[-1]
        line = {
            "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * 1e3 * world, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "m": m, "n": n, "nnz": nnz, "tol": tol, "seed": "rank",
                       "precision": "fp32 matrix/iterates, fp64 averages/KKT/restarts",
                       "parallelism": f"replicas x{world}", "l2": "flushed between steps (256 MiB write)",
                       "iterations": its, "restarts": r0["restarts"], "status": r0["status"],
                       "rel_kkt": max(r0["rel_primal"], r0["rel_dual"], r0["rel_gap"]),
                       "objective_rel_err_vs_planted": abs(e2e_out[-1]["objective"] - lp.obj_star) / abs(lp.obj_star)},
            "e2e": {"value": e2e_value, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "kernel": f"{dom}-phase SpMV + fused step (k_rowblock)",
                         "achieved": row_gbs if dom == "row" else col_gbs, "peak": peak, "unit": "GB/s",
                         "frac": (row_gbs if dom == "row" else col_gbs) / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "row_ms": row_ms, "col_ms": col_ms,
                         "bytes_per_launch": {"row": brow, "col": bcol}, "other_gbs": col_gbs if dom == "row" else row_gbs},
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--profile-blocks", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = world > 1
    if args.impl == "reference":
        reference_arm(args, rank, world)
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
