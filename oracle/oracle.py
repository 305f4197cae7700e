"""ctypes binding of the C restatement (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and bench.py's CPU-baseline leg import this module, and only to check or time
against the CUDA engine. It restates the reference's gpu/pdhg.cu PDHG path in FP64 on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

STATUS = {0: "near_optimal", 1: "iteration_limit", 2: "time_limit", 3: "numerical_failure"}
KKT_NAMES = ["PR2S", "PR2O", "PR2R", "DROW", "DZ2", "DR2S", "DR2O", "POBJ", "DCOL", "DX2"]

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_int64)


class Model(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("col_ptr", _lp), ("row_idx", _ip), ("val", _dp),
                ("cost", _dp), ("col_lo", _dp), ("col_up", _dp), ("row_lo", _dp), ("row_up", _dp),
                ("obj_const", C.c_double), ("maximize", C.c_int)]


class Csr(C.Structure):
    _fields_ = [("rows", C.c_int), ("nnz", C.c_int64), ("ptr", _lp), ("idx", _ip), ("val", _dp)]


class Scaled(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("A", Csr), ("AT", Csr), ("c", _dp), ("l", _dp), ("u", _dp),
                ("rl", _dp), ("ru", _dp), ("Dr", _dp), ("Dc", _dp), ("bnorm", C.c_double), ("cnorm", C.c_double)]


class Options(C.Structure):
    _fields_ = [("tol", C.c_double), ("time_limit", C.c_double), ("max_iter", C.c_int64), ("eval_freq", C.c_int),
                ("row_rel", C.c_double), ("verbose", C.c_int)]


class Outcome(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int64), ("restarts", C.c_int), ("from_average", C.c_int),
                ("rel_p", C.c_double), ("rel_d", C.c_double), ("rel_gap", C.c_double), ("norm_a", C.c_double),
                ("omega", C.c_double), ("objective", C.c_double), ("max_row_viol", C.c_double),
                ("max_bound_viol", C.c_double), ("power_s", C.c_double), ("iterate_s", C.c_double)]


class State(C.Structure):
    _fields_ = [("P", C.POINTER(Scaled)), ("tau", C.c_double), ("sigma", C.c_double)] + [
        (k, _dp) for k in ("x", "z", "Ax", "ATz", "xs", "zs", "Axs", "ATzs", "xlast", "zlast")]


_lib = None


def build() -> Path:
    """Compile liboracle.so from pdhg_oracle.c (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.orc_solve.argtypes = [C.POINTER(Model), C.POINTER(Options), C.POINTER(Outcome), _dp, _dp]
        L.orc_build_scaled.argtypes = [C.POINTER(Model), C.c_double, C.POINTER(Scaled)]
        L.orc_free_scaled.argtypes = [C.POINTER(Scaled)]
        L.orc_power_norm.argtypes = [C.POINTER(Scaled), C.c_int]
        L.orc_power_norm.restype = C.c_double
        L.orc_spmv.argtypes = [C.POINTER(Csr), _dp, _dp]
        L.orc_state_init.argtypes = [C.POINTER(State), C.POINTER(Scaled)]
        L.orc_state_free.argtypes = [C.POINTER(State)]
        L.orc_set_steps.argtypes = [C.POINTER(State), C.c_double, C.c_double]
        L.orc_start.argtypes = [C.POINTER(State), _dp]
        L.orc_iterate.argtypes = [C.POINTER(State), C.c_int]
        L.orc_eval.argtypes = [C.POINTER(State), C.c_int, C.c_double, _dp]
        L.orc_restart.argtypes = [C.POINTER(State), C.c_int, C.c_double]
        L.orc_download.argtypes = [C.POINTER(State), C.c_int, C.c_double, _dp, _dp]
        _lib = L
    return _lib


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


class _ModelRef:
    """Keeps the numpy arrays alive while the C struct points at them."""

    def __init__(self, lp):
        self.arrs = dict(col_ptr=np.ascontiguousarray(lp.col_ptr, np.int64),
                         row_idx=np.ascontiguousarray(lp.row_idx, np.int32),
                         **{k: np.ascontiguousarray(getattr(lp, k), np.float64)
                            for k in ("val", "cost", "col_lo", "col_up", "row_lo", "row_up")})
        a = self.arrs
        self.s = Model(lp.m, lp.n, _p(a["col_ptr"], _lp), _p(a["row_idx"], _ip), _p(a["val"]), _p(a["cost"]),
                       _p(a["col_lo"]), _p(a["col_up"]), _p(a["row_lo"]), _p(a["row_up"]), float(lp.obj_const),
                       int(bool(lp.maximize)))


def solve(lp, tol=1e-4, time_limit=3600.0, max_iter=2_000_000_000, eval_freq=64, row_rel=0.0, verbose=False):
    """Whole FP64 solve; returns (outcome dict, x in original space, y = Dr z)."""
    L = lib()
    mr = _ModelRef(lp)
    o = Options(tol, time_limit, max_iter, eval_freq, row_rel, int(verbose))
    r = Outcome()
    x = np.zeros(max(lp.n, 1))
    y = np.zeros(max(lp.m, 1))
    if L.orc_solve(C.byref(mr.s), C.byref(o), C.byref(r), _p(x), _p(y)) != 0:
        raise MemoryError("oracle solve failed")
    out = {k: getattr(r, k) for k, _ in Outcome._fields_}
    out["status"] = STATUS[r.status]
    return out, x[:lp.n], y[:lp.m]


def _arr(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(max(n, 1),))[:n].copy()


class ScaledProblem:
    """The scaled problem of gpu/pdhg.cu:80-133 as numpy arrays (copied out of the C struct)."""

    def __init__(self, lp, sign=None):
        L = lib()
        mr = _ModelRef(lp)
        self._s = Scaled()
        if sign is None:
            sign = -1.0 if lp.maximize else 1.0
        if L.orc_build_scaled(C.byref(mr.s), float(sign), C.byref(self._s)) != 0:
            raise MemoryError("oracle scaling failed")
        s = self._s
        self.m, self.n = s.m, s.n
        self.A = (_arr(s.A.ptr, s.m + 1), _arr(s.A.idx, s.A.nnz), _arr(s.A.val, s.A.nnz))
        self.AT = (_arr(s.AT.ptr, s.n + 1), _arr(s.AT.idx, s.AT.nnz), _arr(s.AT.val, s.AT.nnz))
        for k in ("c", "l", "u", "Dc"):
            setattr(self, k, _arr(getattr(s, k), s.n))
        for k in ("rl", "ru", "Dr"):
            setattr(self, k, _arr(getattr(s, k), s.m))
        self.bnorm, self.cnorm = s.bnorm, s.cnorm

    def power_norm(self, iters=200):
        return lib().orc_power_norm(C.byref(self._s), iters)

    def __del__(self):
        try:
            lib().orc_free_scaled(C.byref(self._s))
        except Exception:
            pass


class Stepper:
    """Step-level twin of the reference backend concept (init/set_steps/start/iterate/eval/restart/download)."""

    def __init__(self, sp: ScaledProblem):
        self.sp = sp
        self.st = State()
        if lib().orc_state_init(C.byref(self.st), C.byref(sp._s)) != 0:
            raise MemoryError("oracle state init failed")

    def set_steps(self, tau, sigma):
        lib().orc_set_steps(C.byref(self.st), tau, sigma)

    def start(self, x0=None):
        lib().orc_start(C.byref(self.st), None if x0 is None else _p(np.ascontiguousarray(x0, np.float64)))

    def iterate(self, steps):
        lib().orc_iterate(C.byref(self.st), steps)

    def eval(self, avg, f):
        out = np.zeros(10)
        lib().orc_eval(C.byref(self.st), int(avg), float(f), _p(out))
        return out

    def restart(self, avg, f):
        lib().orc_restart(C.byref(self.st), int(avg), float(f))

    def download(self, avg, f):
        x = np.zeros(max(self.sp.n, 1))
        z = np.zeros(max(self.sp.m, 1))
        lib().orc_download(C.byref(self.st), int(avg), float(f), _p(x), _p(z))
        return x[:self.sp.n], z[:self.sp.m]

    def vec(self, name):
        n = self.sp.n if name in ("x", "ATz", "xs", "ATzs", "xlast") else self.sp.m
        return _arr(getattr(self.st, name), n)

    def __del__(self):
        try:
            lib().orc_state_free(C.byref(self.st))
        except Exception:
            pass


def spmv(ptr, idx, val, x):
    rows = len(ptr) - 1
    ptr = np.ascontiguousarray(ptr, np.int64)
    idx = np.ascontiguousarray(idx, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(max(rows, 1))
    a = Csr(rows, len(idx), _p(ptr, _lp), _p(idx, _ip), _p(val))
    lib().orc_spmv(C.byref(a), _p(x), _p(y))
    return y[:rows]
