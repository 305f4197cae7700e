"""Python binding of the engine's C ABI (include/taral_pdhg.h) over ctypes.

Mirrors the reference's interfaces for the PDHG path: the backend concept of gpu/pdhg.cu:313-514
(:class:`Engine`: power_norm, set_steps, start, iterate, eval, restart, download), the whole solve
(:func:`solve`, gpu/pdhg.cu:761-911 behind main), the input gate (:func:`input_error`,
gpu/pdhg_input.hpp:7-17), the MPS reader (:func:`read_mps`, src/mps.cpp:388) and the standalone CSR SpMV
(:class:`SpmvPlan`, gpu/csr_matvec.cu:23-32). Everything runs in lib/libtaral_pdhg.so; there is no Python or
CPU fallback, and loading fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path
from typing import Optional

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libtaral_pdhg.so"
CLI_PATH = PKG / "bin" / "pdhg"

OK, ERR_CUDA, ERR_ALLOC, ERR_INPUT, ERR_UNSUPPORTED, ERR_PARSE, ERR_STATE, ERR_NO_DEVICE = 0, -1, -2, -3, -4, -5, -6, -7
ERR_CANCELLED = -8
FP64, FP32 = 0, 1
STATUS = {0: "near_optimal", 1: "iteration_limit", 2: "time_limit", 3: "numerical_failure", 4: "cancelled"}
KKT_NAMES = ["PR2S", "PR2O", "PR2R", "DROW", "DZ2", "DR2S", "DR2O", "POBJ", "DCOL", "DX2"]
ERRORS = {ERR_CUDA: "CUDA error", ERR_ALLOC: "allocation failed", ERR_INPUT: "bad input",
          ERR_UNSUPPORTED: "unsupported model", ERR_PARSE: "parse error", ERR_STATE: "call out of order",
          ERR_NO_DEVICE: "no CUDA device", ERR_CANCELLED: "cancelled"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)
_ubp = C.POINTER(C.c_ubyte)


class TaralError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"{ERRORS.get(code, code)} ({code}){': ' + msg if msg else ''}")
        self.code = code


class CsrT(C.Structure):
    _fields_ = [("rows", C.c_int), ("cols", C.c_int), ("nnz", C.c_int64), ("ptr", _lp), ("idx", _ip), ("val", _dp)]


class ModelT(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("col_ptr", _lp), ("row_idx", _ip), ("val", _dp), ("cost", _dp),
                ("col_lo", _dp), ("col_up", _dp), ("row_lo", _dp), ("row_up", _dp), ("obj_const", C.c_double),
                ("maximize", C.c_int), ("is_int", _ubp), ("n_quadratic", C.c_int64)]


class OptionsT(C.Structure):
    _fields_ = [("tol", C.c_double), ("time_limit", C.c_double), ("max_iter", C.c_int64), ("eval_freq", C.c_int),
                ("row_rel", C.c_double), ("verbose", C.c_int), ("graph", C.c_int), ("precision", C.c_int)]


class OutcomeT(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int64), ("restarts", C.c_int), ("from_average", C.c_int),
                ("rel_primal", C.c_double), ("rel_dual", C.c_double), ("rel_gap", C.c_double),
                ("norm_a", C.c_double), ("primal_weight", C.c_double), ("objective", C.c_double),
                ("max_row_violation", C.c_double), ("max_bound_violation", C.c_double), ("scale_s", C.c_double),
                ("device_init_s", C.c_double), ("transfer_s", C.c_double), ("solve_s", C.c_double),
                ("power_iter_s", C.c_double), ("device_mem_bytes", C.c_size_t), ("kernel_launches", C.c_int64),
                ("nnz", C.c_int64), ("device_s", C.c_double)]


class CheckT(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("objective", "row_violation_rel", "bound_violation", "dual_bound",
                                          "dual_obj_loose", "dual_infeas_rel", "dual_gap_rel")] + \
               [("dual_sign", C.c_int), ("pad", C.c_int)]


# Every symbol the header declares, with its ctypes signature: (restype, argtypes).
SIGNATURES = {
    "pdhg_create": (C.c_int, [C.POINTER(CsrT), C.POINTER(CsrT)] + [_dp] * 7 +
                    [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint, C.POINTER(C.c_void_p)]),
    "pdhg_power_norm": (C.c_int, [C.c_void_p, C.c_int, _dp]),
    "pdhg_set_steps": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "pdhg_start": (C.c_int, [C.c_void_p, _dp, _dp]),
    "pdhg_iterate": (C.c_int, [C.c_void_p, C.c_int]),
    "pdhg_eval": (C.c_int, [C.c_void_p, C.c_int, C.c_double, _dp]),
    "pdhg_eval_pair": (C.c_int, [C.c_void_p, C.c_double, _dp, _dp]),
    "pdhg_restart": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "pdhg_download": (C.c_int, [C.c_void_p, C.c_int, C.c_double, _dp, _dp]),
    "pdhg_info": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "pdhg_create_model": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_uint, C.POINTER(C.c_void_p), _dp, _dp]),
    "pdhg_solve_ctx": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_void_p, _dp, _dp, C.c_void_p, _dp, _dp]),
    "pdhg_profile_phases": (C.c_int, [C.c_void_p, C.c_int, _dp, _dp]),
    "pdhg_kernel_launches": (C.c_int64, [C.c_void_p]),
    "pdhg_last_error": (C.c_char_p, [C.c_void_p]),
    "pdhg_destroy": (None, [C.c_void_p]),
    "taral_options_default": (None, [C.POINTER(OptionsT)]),
    "taral_pdhg_input_error": (C.c_char_p, [C.POINTER(ModelT)]),
    "taral_pdhg_solve": (C.c_int, [C.POINTER(ModelT), C.POINTER(OptionsT), C.POINTER(OutcomeT), _dp, _dp]),
    "taral_pdhg_solve_warm": (C.c_int, [C.POINTER(ModelT), C.POINTER(OptionsT), _dp, _dp, C.POINTER(OutcomeT),
                                        _dp, _dp]),
    "taral_mps_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "taral_mps_error": (C.c_char_p, []),
    "taral_mps_model": (C.c_int, [C.c_void_p, C.POINTER(ModelT)]),
    "taral_mps_col_name": (C.c_char_p, [C.c_void_p, C.c_int]),
    "taral_mps_row_name": (C.c_char_p, [C.c_void_p, C.c_int]),
    "taral_mps_name": (C.c_char_p, [C.c_void_p]),
    "taral_mps_free": (None, [C.c_void_p]),
    "taral_batch_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(OptionsT), C.POINTER(C.c_void_p)]),
    "taral_batch_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]),
    "taral_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_size_t), C.POINTER(C.c_int64),
                                   C.POINTER(C.c_int64)]),
    "taral_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "taral_batch_destroy": (None, [C.c_void_p]),
    "taral_batch_cancel": (C.c_int, [C.c_void_p]),
    "pdhg_scaled_problem": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp]),
    "taral_set_device_alloc_limit": (None, [C.c_size_t]),
    "taral_check_models": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "taral_kkt_eval_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double] + [C.c_void_p] * 13 +
                               [C.c_void_p, C.c_void_p]),
    "taral_mlp_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "taral_mlp_param_count": (C.c_int64, [C.c_void_p]),
    "taral_mlp_set_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "taral_mlp_get_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "taral_mlp_forward": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "taral_mlp_gradients": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), _dp,
                                      C.POINTER(C.c_float)]),
    "taral_mlp_set_dataset": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "taral_mlp_train": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_uint64, _dp]),
    "taral_mlp_last_error": (C.c_char_p, [C.c_void_p]),
    "taral_mlp_destroy": (None, [C.c_void_p]),
    "taral_gemm_bf16": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_int, C.c_void_p, C.c_void_p]),
    "taral_gemm_bf16_tc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]),
    "taral_gemm_bf16_umma": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                       C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                       C.c_void_p]),
    "taral_spmv_plan_create": (C.c_int, [C.c_int, C.c_int, _lp, C.c_int, C.POINTER(C.c_void_p)]),
    "taral_spmv_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p]),
    "taral_spmv_plan_blocks": (C.c_int, [C.c_void_p]),
    "taral_spmv_plan_destroy": (None, [C.c_void_p]),
}

_lib = None


def lib():
    """Load lib/libtaral_pdhg.so (raises if it is missing: build it with taral-lp_b200/build.py)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: the CUDA engine has not been built (run build.py)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def _check(code, ctx=None):
    if code != OK:
        msg = lib().pdhg_last_error(ctx).decode() if ctx else ""
        raise TaralError(code, msg)


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, np.float64)


class _Csr:
    def __init__(self, ptr, idx, val, cols):
        self.ptr = np.ascontiguousarray(ptr, np.int64)
        self.idx = np.ascontiguousarray(idx, np.int32)
        self.val = _f64(val)
        self.s = CsrT(len(self.ptr) - 1, cols, len(self.idx), _p(self.ptr, _lp), _p(self.idx, _ip), _p(self.val))


class _Model:
    """C view of a column-wise model (anything with the LP attributes of lpgen.LP); keeps the arrays alive."""

    def __init__(self, lp):
        self.a = dict(col_ptr=np.ascontiguousarray(lp.col_ptr, np.int64),
                      row_idx=np.ascontiguousarray(lp.row_idx, np.int32),
                      **{k: _f64(getattr(lp, k)) for k in ("val", "cost", "col_lo", "col_up", "row_lo", "row_up")})
        is_int = getattr(lp, "is_int", None)
        self.is_int = None if is_int is None else np.ascontiguousarray(is_int, np.uint8)
        a = self.a
        self.s = ModelT(int(lp.m), int(lp.n), _p(a["col_ptr"], _lp), _p(a["row_idx"], _ip), _p(a["val"]),
                        _p(a["cost"]), _p(a["col_lo"]), _p(a["col_up"]), _p(a["row_lo"]), _p(a["row_up"]),
                        float(getattr(lp, "obj_const", 0.0)), int(bool(getattr(lp, "maximize", False))),
                        None if self.is_int is None else _p(self.is_int, _ubp),
                        int(getattr(lp, "n_quadratic", 0)))


# ------------------------------------------------------------------------------------------------ backend concept
class Engine:
    """Device context over a scaled problem (A_s, A_s^T and the 7 scaled vectors)."""

    def __init__(self, A, AT, c, l, u, rl, ru, Dr, Dc, precision=FP64, eval_freq=64, graph=True):
        m, n = len(A[0]) - 1, len(AT[0]) - 1
        self.m, self.n = m, n
        a, at = _Csr(*A, cols=n), _Csr(*AT, cols=m)
        vecs = [_f64(v) for v in (c, l, u, rl, ru, Dr, Dc)]
        h = C.c_void_p()
        code = lib().pdhg_create(C.byref(a.s), C.byref(at.s), *[_p(v) for v in vecs], m, n, int(precision),
                                 int(eval_freq), 0 if graph else 1, C.byref(h))
        _check(code)
        self.h = h

    @classmethod
    def from_model(cls, lp, precision=FP64, eval_freq=64, graph=True):
        """Scale a column-wise model on the host (gpu/pdhg.cu:80-133) and upload it. Sets .bnorm / .cnorm."""
        mr = _Model(lp)
        h = C.c_void_p()
        bn, cn = C.c_double(), C.c_double()
        _check(lib().pdhg_create_model(C.byref(mr.s), int(precision), int(eval_freq), 0 if graph else 1, C.byref(h),
                                       C.byref(bn), C.byref(cn)))
        self = cls.__new__(cls)
        self.h, self.m, self.n, self.bnorm, self.cnorm = h, int(lp.m), int(lp.n), bn.value, cn.value
        return self

    @classmethod
    def from_scaled(cls, sp, **kw):
        """From an object with A, AT (ptr, idx, val) tuples and c, l, u, rl, ru, Dr, Dc arrays."""
        return cls(sp.A, sp.AT, sp.c, sp.l, sp.u, sp.rl, sp.ru, sp.Dr, sp.Dc, **kw)

    def power_norm(self, iters=200):
        v = C.c_double()
        _check(lib().pdhg_power_norm(self.h, iters, C.byref(v)), self.h)
        return v.value

    def set_steps(self, tau, sigma):
        _check(lib().pdhg_set_steps(self.h, tau, sigma), self.h)

    def start(self, x0=None, z0=None):
        x0 = None if x0 is None else _f64(x0)
        z0 = None if z0 is None else _f64(z0)
        _check(lib().pdhg_start(self.h, None if x0 is None else _p(x0), None if z0 is None else _p(z0)), self.h)

    def iterate(self, steps):
        _check(lib().pdhg_iterate(self.h, int(steps)), self.h)

    def eval(self, avg, f):
        out = np.zeros(10)
        _check(lib().pdhg_eval(self.h, int(avg), float(f), _p(out)), self.h)
        return out

    def eval_pair(self, f):
        cur, avg = np.zeros(10), np.zeros(10)
        _check(lib().pdhg_eval_pair(self.h, float(f), _p(cur), _p(avg)), self.h)
        return cur, avg

    def restart(self, avg, f):
        _check(lib().pdhg_restart(self.h, int(avg), float(f)), self.h)

    def download(self, avg, f):
        x, z = np.zeros(max(self.n, 1)), np.zeros(max(self.m, 1))
        _check(lib().pdhg_download(self.h, int(avg), float(f), _p(x), _p(z)), self.h)
        return x[:self.n], z[:self.m]

    def solve(self, bnorm, cnorm, tol=1e-4, time_limit=3600.0, max_iter=2_000_000_000, eval_freq=64, row_rel=0.0,
              x0=None, z0=None, want_point=True):
        """The reference driver (gpu/pdhg.cu:761-849) on this context. Returns (outcome dict, x, z) in the scaled
        space; outcome['device_s'] is the CUDA-event time of the solve."""
        o = OptionsT(tol, time_limit, max_iter, eval_freq, row_rel, 0, 1, 0)
        r = OutcomeT()
        x, z = (np.zeros(max(self.n, 1)), np.zeros(max(self.m, 1))) if want_point else (None, None)
        xa = None if x0 is None else _f64(x0)
        za = None if z0 is None else _f64(z0)
        _check(lib().pdhg_solve_ctx(self.h, float(bnorm), float(cnorm), C.byref(o), None if xa is None else _p(xa),
                                    None if za is None else _p(za), C.byref(r), None if x is None else _p(x),
                                    None if z is None else _p(z)), self.h)
        out = {k: getattr(r, k) for k, _ in OutcomeT._fields_}
        out["status"] = STATUS[r.status]
        return out, (None if x is None else x[:self.n]), (None if z is None else z[:self.m])

    def scaled_problem(self, nnz):
        """(Dr, Dc, A values, A^T values) of the scaled problem held on the device (pdhg_scaled_problem)."""
        dr, dc = np.zeros(max(self.m, 1)), np.zeros(max(self.n, 1))
        a, at = np.zeros(max(nnz, 1)), np.zeros(max(nnz, 1))
        _check(lib().pdhg_scaled_problem(self.h, _p(dr), _p(dc), _p(a), _p(at)), self.h)
        return dr[:self.m], dc[:self.n], a[:nnz], at[:nnz]

    def profile_phases(self, reps):
        """Mean CUDA-event milliseconds per launch of the row-phase and column-phase kernels over `reps` steps."""
        a, b = C.c_double(), C.c_double()
        _check(lib().pdhg_profile_phases(self.h, int(reps), C.byref(a), C.byref(b)), self.h)
        return a.value, b.value

    def info(self):
        buf = C.create_string_buffer(256)
        mem = C.c_size_t()
        _check(lib().pdhg_info(self.h, buf, 256, C.byref(mem)), self.h)
        return buf.value.decode(), mem.value

    @property
    def kernel_launches(self):
        return lib().pdhg_kernel_launches(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib().pdhg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------------------------------ whole solve
def default_options():
    o = OptionsT()
    lib().taral_options_default(C.byref(o))
    return o


def input_error(lp) -> Optional[str]:
    r = lib().taral_pdhg_input_error(C.byref(_Model(lp).s))
    return None if r is None else r.decode()


def solve(lp, tol=1e-4, time_limit=3600.0, max_iter=2_000_000_000, eval_freq=64, row_rel=0.0, precision=FP64,
          graph=True, verbose=False, x0=None, y0=None):
    """Solve one LP on the GPU. Returns (outcome dict, x (n, original space), y (m, y = Dr z)).

    x0 / y0: optional warm start in the original space (y in the minimisation form of the dual output)."""
    mr = _Model(lp)
    o = OptionsT(tol, time_limit, max_iter, eval_freq, row_rel, int(verbose), int(graph), int(precision))
    r = OutcomeT()
    x, y = np.zeros(max(lp.n, 1)), np.zeros(max(lp.m, 1))
    if x0 is None and y0 is None:
        code = lib().taral_pdhg_solve(C.byref(mr.s), C.byref(o), C.byref(r), _p(x), _p(y))
    else:
        xa = None if x0 is None else _f64(x0)
        ya = None if y0 is None else _f64(y0)
        code = lib().taral_pdhg_solve_warm(C.byref(mr.s), C.byref(o), None if xa is None else _p(xa),
                                           None if ya is None else _p(ya), C.byref(r), _p(x), _p(y))
    _check(code)
    out = {k: getattr(r, k) for k, _ in OutcomeT._fields_}
    out["status"] = STATUS[r.status]
    return out, x[:lp.n], y[:lp.m]


def set_device_alloc_limit(nbytes):
    """Fault-injection hook for tests (taral_set_device_alloc_limit): contexts and batches created from now on fail
    with ERR_ALLOC when their device allocations would exceed `nbytes`; 0 removes the limit."""
    lib().taral_set_device_alloc_limit(int(nbytes))


# ------------------------------------------------------------------------------------------------ check
def rhs_of(lp):
    """The rows' MPS right-hand sides b when the model knows its row types (up for L rows, lo otherwise, as the MPS
    writer puts them), else None (the library's default: b = lo where lo is finite, else up)."""
    types = getattr(lp, "row_types", None)
    if types is None:
        return None
    return np.where(np.asarray(types) == "L", np.asarray(lp.row_up, float), np.asarray(lp.row_lo, float))


def check_models(lps, xs, ys=None, rhs=None):
    """Independent FP64 check of answers on the original models, on the device (taral_check_models): a list of dicts
    with objective, row_violation_rel, bound_violation and the weak-duality fields (None where not checked)."""
    k = len(lps)
    models = [_Model(lp) for lp in lps]
    arr = (ModelT * k)(*[m.s for m in models])
    xa = [_f64(x) for x in xs]
    ya = None if ys is None else [None if y is None else _f64(y) for y in ys]
    ra = [rhs_of(lp) for lp in lps] if rhs is None else rhs
    ra = [None if r is None else _f64(r) for r in ra]

    def table(vs):
        if vs is None:
            return None, None
        t = (_dp * k)(*[None if v is None else _p(v) for v in vs])
        return t, C.cast(t, C.c_void_p)
    tx, ty, tr = table(xa), table(ya), table(ra)
    out = (CheckT * k)()
    _check(lib().taral_check_models(C.cast(arr, C.c_void_p), k, tr[1], tx[1], ty[1], C.cast(out, C.c_void_p)))
    res = []
    for o in out:
        d = {f: getattr(o, f) for f, _ in CheckT._fields_ if f != "pad"}
        for f in ("dual_bound", "dual_obj_loose", "dual_infeas_rel", "dual_gap_rel"):
            if np.isnan(d[f]):
                d[f] = None
        d["dual_sign"] = None if d["dual_sign"] == 0 else float(d["dual_sign"])
        res.append(d)
    return res


# ------------------------------------------------------------------------------------------------ batch
class Batch:
    """Many LPs solved together (taral_batch_*): per-instance restarts and stopping on the device, identical
    constraint matrices stored once. Keeps the models' arrays alive for the batch's lifetime."""

    def __init__(self, lps, tol=1e-4, time_limit=3600.0, max_iter=2_000_000_000, eval_freq=64, row_rel=0.0,
                 precision=FP64, graph=True):
        self.lps = list(lps)
        self._models = [_Model(lp) for lp in self.lps]
        arr = (ModelT * len(self._models))(*[m.s for m in self._models])
        self._arr = arr
        o = OptionsT(tol, time_limit, max_iter, eval_freq, row_rel, 0, int(graph), int(precision))
        h = C.c_void_p()
        _check(lib().taral_batch_create(C.cast(arr, C.c_void_p), len(self._models), C.byref(o), C.byref(h)))
        self.h = h

    def info(self):
        d, mem, ns, nt = C.c_int(), C.c_size_t(), C.c_int64(), C.c_int64()
        _check(lib().taral_batch_info(self.h, C.byref(d), C.byref(mem), C.byref(ns), C.byref(nt)))
        return {"distinct_matrices": d.value, "device_mem_bytes": mem.value, "nnz_stored": ns.value,
                "nnz_total": nt.value}

    def solve(self, x0=None, y0=None, want_points=True, w0=None):
        """Returns (list of outcome dicts, list of x, list of y). x0 / y0: optional lists of warm starts (entries
        may be None); w0: optional initial primal weights (entries <= 0 keep the default)."""
        k = len(self.lps)
        outs = (OutcomeT * k)()

        def table(arrs):  # array of double* (NULL where None), as a void*
            if arrs is None:
                return None, None
            t = (_dp * k)(*[None if a is None else _p(a) for a in arrs])
            return t, C.cast(t, C.c_void_p)
        xin = None if x0 is None else [None if v is None else _f64(v) for v in x0]
        yin = None if y0 is None else [None if v is None else _f64(v) for v in y0]
        xout = [np.zeros(max(lp.n, 1)) for lp in self.lps] if want_points else None
        yout = [np.zeros(max(lp.m, 1)) for lp in self.lps] if want_points else None
        tabs = [table(v) for v in (xin, yin, xout, yout)]
        wv = None if w0 is None else _f64(np.nan_to_num(np.asarray(w0, np.float64), nan=0.0))
        if wv is not None and wv.size != k:
            raise ValueError("w0 needs one entry per instance")
        code = lib().taral_batch_solve(self.h, tabs[0][1], tabs[1][1], None if wv is None else wv.ctypes.data,
                                       C.cast(outs, C.c_void_p), tabs[2][1], tabs[3][1])
        self.last_code = code  # ERR_CANCELLED: stopped by cancel(); the outcomes and points are filled all the same
        if code not in (OK, ERR_CANCELLED):
            raise TaralError(code, (lib().taral_batch_last_error(self.h) or b"").decode())
        res = []
        for i in range(k):
            d = {f: getattr(outs[i], f) for f, _ in OutcomeT._fields_}
            d["status"] = STATUS[outs[i].status]
            res.append(d)
        if not want_points:
            return res, None, None
        return res, [xout[i][:self.lps[i].n] for i in range(k)], [yout[i][:self.lps[i].m] for i in range(k)]

    def cancel(self):
        """Ask a running solve() (in another thread) to stop after its current block; see taral_batch_cancel."""
        _check(lib().taral_batch_cancel(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().taral_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------------------------------ MLP
_fp = C.POINTER(C.c_float)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


class Mlp:
    """The learned warm start's network (taral_mlp_*): in -> hidden x depth (GELU) -> out, BF16 tensor-core GEMMs,
    FP32 accumulate, Adam on FP32 master weights. Parameters are a flat float32 vector, per layer W (in x out) then
    b."""

    def __init__(self, in_dim, hidden, depth, out_dim, max_batch=256):
        self.dims = (in_dim, hidden, depth, out_dim)
        self.max_batch = max_batch
        h = C.c_void_p()
        _check(lib().taral_mlp_create(in_dim, hidden, depth, out_dim, max_batch, C.byref(h)))
        self.h = h

    def _err(self, code):
        if code != OK:
            raise TaralError(code, (lib().taral_mlp_last_error(self.h) or b"").decode())

    @property
    def param_count(self):
        return lib().taral_mlp_param_count(self.h)

    def shapes(self):
        i, hd, d, o = self.dims
        dims = [i] + [hd] * d + [o]
        return [((dims[l], dims[l + 1]), (dims[l + 1],)) for l in range(d + 1)]

    def init(self, seed=0, out_scale=1.0):
        """He-style initialisation: W ~ N(0, 2 / fan_in) (out_scale^2 / fan_in for the output layer), b = 0.
        out_scale = 0 starts the network at a zero output (with normalised targets: the training mean)."""
        rng = np.random.default_rng(seed)
        parts = []
        sh = self.shapes()
        for k, ((fi, fo), _) in enumerate(sh):
            s = np.sqrt((out_scale ** 2 if k == len(sh) - 1 else 2.0) / fi)
            parts += [rng.standard_normal(fi * fo) * s, np.zeros(fo)]
        self.set_params(np.concatenate(parts))

    def set_params(self, p):
        p = _f32(p)
        assert p.size == self.param_count
        self._err(lib().taral_mlp_set_params(self.h, p.ctypes.data_as(_fp)))

    def get_params(self):
        p = np.zeros(self.param_count, np.float32)
        self._err(lib().taral_mlp_get_params(self.h, p.ctypes.data_as(_fp)))
        return p

    def forward(self, x):
        x = _f32(np.atleast_2d(x))
        y = np.zeros((x.shape[0], self.dims[3]), np.float32)
        for b0 in range(0, x.shape[0], self.max_batch):
            xb = _f32(x[b0:b0 + self.max_batch])
            yb = np.zeros((xb.shape[0], self.dims[3]), np.float32)
            self._err(lib().taral_mlp_forward(self.h, xb.shape[0], xb.ctypes.data_as(_fp), yb.ctypes.data_as(_fp)))
            y[b0:b0 + xb.shape[0]] = yb
        return y

    def gradients(self, x, t):
        x, t = _f32(x), _f32(t)
        g = np.zeros(self.param_count, np.float32)
        loss = C.c_double()
        self._err(lib().taral_mlp_gradients(self.h, x.shape[0], x.ctypes.data_as(_fp), t.ctypes.data_as(_fp),
                                            C.byref(loss), g.ctypes.data_as(_fp)))
        return loss.value, g

    def set_dataset(self, x, t):
        x, t = _f32(x), _f32(t)
        self._err(lib().taral_mlp_set_dataset(self.h, x.shape[0], x.ctypes.data_as(_fp), t.ctypes.data_as(_fp)))

    def train(self, epochs, batch, lr, seed=0):
        loss = C.c_double()
        self._err(lib().taral_mlp_train(self.h, epochs, batch, lr, seed, C.byref(loss)))
        return loss.value

    def close(self):
        if getattr(self, "h", None):
            lib().taral_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------------------------------ MPS
class MpsModel:
    """A model read by the engine's MPS reader: numpy copies of the arrays plus row/column names."""

    def __init__(self, path):
        h = C.c_void_p()
        code = lib().taral_mps_read(str(path).encode(), C.byref(h))
        if code != OK:
            raise TaralError(code, (lib().taral_mps_error() or b"").decode())
        try:
            v = ModelT()
            _check(lib().taral_mps_model(h, C.byref(v)))
            self.m, self.n = v.m, v.n
            nnz = v.col_ptr[v.n] if v.n else 0

            def arr(p, k, dt):
                return np.ctypeslib.as_array(p, shape=(max(k, 1),))[:k].astype(dt, copy=True) if k else np.zeros(0, dt)
            self.col_ptr = np.ctypeslib.as_array(v.col_ptr, shape=(v.n + 1,)).astype(np.int64, copy=True)
            self.row_idx = arr(v.row_idx, nnz, np.int32)
            self.val = arr(v.val, nnz, np.float64)
            self.cost, self.col_lo, self.col_up = (arr(getattr(v, k), v.n, np.float64) for k in ("cost", "col_lo", "col_up"))
            self.row_lo, self.row_up = (arr(getattr(v, k), v.m, np.float64) for k in ("row_lo", "row_up"))
            self.obj_const, self.maximize = v.obj_const, bool(v.maximize)
            self.is_int = arr(v.is_int, v.n, np.uint8)
            self.n_quadratic = v.n_quadratic
            self.name = (lib().taral_mps_name(h) or b"").decode()
            self.col_names = [lib().taral_mps_col_name(h, j).decode() for j in range(v.n)]
            self.row_names = [lib().taral_mps_row_name(h, i).decode() for i in range(v.m)]
        finally:
            lib().taral_mps_free(h)

    @property
    def nnz(self):
        return int(self.col_ptr[-1])


def read_mps(path) -> MpsModel:
    return MpsModel(path)


# ------------------------------------------------------------------------------------------------ SpMV
class SpmvPlan:
    """Row-block plan of a CSR matrix for y = A x on device buffers (int32 ptr/idx, float32 or float64 val)."""

    def __init__(self, host_ptr, cols, dtype=FP32):
        ptr = np.ascontiguousarray(host_ptr, np.int64)
        h = C.c_void_p()
        _check(lib().taral_spmv_plan_create(len(ptr) - 1, int(cols), _p(ptr, _lp), int(dtype), C.byref(h)))
        self.h = h

    @property
    def blocks(self):
        return lib().taral_spmv_plan_blocks(self.h)

    def run(self, d_ptr, d_idx, d_val, d_x, d_y, stream=0):
        """Device pointers as ints (e.g. torch tensor .data_ptr()); stream: cudaStream_t as int (0 = default)."""
        _check(lib().taral_spmv_run(self.h, C.c_void_p(d_ptr), C.c_void_p(d_idx), C.c_void_p(d_val),
                                    C.c_void_p(d_x), C.c_void_p(d_y), C.c_void_p(stream or None)))

    def close(self):
        if getattr(self, "h", None):
            lib().taral_spmv_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def header_symbols(header: Path = PKG.parent / "include" / "taral_pdhg.h"):
    """Function names declared in the C header (for the export check)."""
    import re
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b((?:pdhg|taral)_[a-z0-9_]+)\s*\(", text)))
