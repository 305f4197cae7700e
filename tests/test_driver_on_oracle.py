"""The engine's host driver (run() in taral-lp_b200/csrc/host.hpp and the restart schedule in schedule.hpp, the
same schedule the batched engine's decision kernel runs) driven over the CPU oracle's FP64 step functions must take
the same decisions as the oracle's own restatement of the reference driver (gpu/pdhg.cu:761-849): equal status,
iteration and restart counts, final primal weight, residuals and scaled-space point, bit for bit."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

import lpgen
import oracle

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "native" / "driver_on_oracle.cpp"


@pytest.fixture(scope="module")
def driver_lib(tmp_path_factory, oracle_lib):
    out = tmp_path_factory.mktemp("drv") / "libdriver_on_oracle.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off",
                    "-I", str(ROOT / "include"), "-I", str(ROOT / "taral-lp_b200" / "csrc"),
                    "-I", str(ROOT / "oracle"), str(SRC), "-o", str(out), str(oracle.LIB),
                    f"-Wl,-rpath,{oracle.LIB.parent}"], check=True)
    L = C.CDLL(str(out))
    L.drive_on_oracle.argtypes = [C.POINTER(oracle.Scaled), C.POINTER(oracle.Options), C.POINTER(oracle.Outcome),
                                  C.POINTER(C.c_double), C.POINTER(C.c_double)]
    return L


CASES = [
    ("general_300x700", lambda: lpgen.general(300, 700, seed=3), dict(tol=1e-6)),
    ("planted_2000x5000", lambda: lpgen.planted(2000, 5000, 5, seed=1), dict(tol=1e-6)),
    ("planted_zipf", lambda: lpgen.planted(3000, 8000, 6, seed=2, zipf=1.2, cap=400, floor=3), dict(tol=1e-5)),
    ("packing_10000", lambda: lpgen.packing(10_000), dict(tol=1e-4)),
    ("transport_30x30_rowrel", lambda: lpgen.transport(30, 30), dict(tol=1e-6, row_rel=100.0)),
    ("general_eval32_cap", lambda: lpgen.general(200, 500, seed=9), dict(tol=1e-9, eval_freq=32, max_iter=3000)),
    ("general_maximize", lambda: lpgen.general(250, 600, seed=5, maximize=True), dict(tol=1e-6)),
]


@pytest.mark.parametrize("name,make,kw", CASES, ids=[c[0] for c in CASES])
def test_driver_matches_oracle_driver(driver_lib, name, make, kw):
    lp = make()
    want, _, _ = oracle.solve(lp, **kw)
    sp = oracle.ScaledProblem(lp)
    o = oracle.Options(kw.get("tol", 1e-4), 3600.0, kw.get("max_iter", 2_000_000_000), kw.get("eval_freq", 64),
                       kw.get("row_rel", 0.0), 0)
    r = oracle.Outcome()
    x, z = np.zeros(max(sp.n, 1)), np.zeros(max(sp.m, 1))
    assert driver_lib.drive_on_oracle(C.byref(sp._s), C.byref(o), C.byref(r),
                                      x.ctypes.data_as(C.POINTER(C.c_double)),
                                      z.ctypes.data_as(C.POINTER(C.c_double))) == 0
    got = {k: getattr(r, k) for k in ("status", "iterations", "restarts", "from_average", "rel_p", "rel_d",
                                      "rel_gap", "norm_a", "omega")}
    got["status"] = oracle.STATUS[got["status"]]
    for k, v in got.items():
        assert v == want[k], (name, k, v, want[k])
    # the oracle's point in original units is Dc x_s; the driver's scaled point must give the same numbers
    _, xo, yo = oracle.solve(lp, **kw)
    assert np.array_equal(x[:sp.n] * sp.Dc, xo)
    assert np.array_equal(sp.Dr * z[:sp.m], yo)
