"""Oracle (test infrastructure only): FP64 numpy restatement of the reference's independent check of an answer on the
ORIGINAL model -- the primal side of benchmarks/orig_check.py:63-88 and the weak-duality bound of
gpu/vector_check.py:46-74. Pinned against the reference module itself: tests/golden/reference_vector_check.json
(make_golden.py --vector-check runs gpu/vector_check.check_files on the reference PDHG's own .sol / .dual files).

    objective          c'x + const (the objective row's constant)
    row_violation_rel  max_i max(lo_i - a_i x, a_i x - up_i, 0) / (1 + |b_i|), b_i the row's right-hand side
    bound_violation    max_j max(l_j - x_j, x_j - u_j, 0)
    dual side (minimisation models only), for y and -y: LB = const + sum_i min_{r in [lo_i, up_i]} y_i r
        + sum_j min_{x in [l_j, u_j]} d_j x with d = c - A'y; a term whose minimising bound is infinite (|v| >= 1e20)
        is dropped and its size recorded (rows |y_i| / (1 + |y_i|), columns |d_j| / (1 + |c_j|)); the sign with the
        smaller largest dropped term is kept. dual_bound = LB if nothing was dropped (else None), dual_obj_loose = LB,
        dual_infeas_rel = the largest dropped term, dual_gap_rel = (objective - LB) / max(1, |objective|).
"""
import numpy as np

INF = 1e20


def rhs_of(lp):
    """The MPS right-hand side of every row: up for L rows, lo otherwise (the MPS writer's rule); without row types
    a row with a finite lower bound has b = lo, else b = up."""
    lo, up = np.asarray(lp.row_lo, float), np.asarray(lp.row_up, float)
    types = getattr(lp, "row_types", None)
    if types is not None:
        return np.where(np.asarray(types) == "L", up, lo)
    return np.where(np.isfinite(lo), lo, up)


def _min_over(coef, lo, up):
    """Vectorised _min_over: (value or nan where dropped, dropped size)."""
    v = np.where(coef > 0, lo, up)
    dropped = (coef != 0) & (np.abs(v) >= INF)
    val = np.where(coef == 0, 0.0, np.where(dropped, np.nan, coef * np.where(dropped, 0.0, v)))
    return val, np.where(dropped, np.abs(coef), 0.0)


def check(lp, x, y=None, rhs=None):
    m, n = lp.m, lp.n
    cols = np.repeat(np.arange(n), np.diff(lp.col_ptr))
    x = np.asarray(x, float)
    act = np.zeros(m)
    np.add.at(act, lp.row_idx, lp.val * x[cols])
    const = float(getattr(lp, "obj_const", 0.0))
    cost = np.asarray(lp.cost, float)
    objective = float(np.dot(cost, x)) + const
    lo, up = np.asarray(lp.row_lo, float), np.asarray(lp.row_up, float)
    b = rhs_of(lp) if rhs is None else np.asarray(rhs, float)
    rv = np.maximum(np.maximum(lo - act, act - up), 0.0) / (1.0 + np.abs(b))
    l, u = np.asarray(lp.col_lo, float), np.asarray(lp.col_up, float)
    bv = np.maximum(np.maximum(l - x, x - u), 0.0)
    out = dict(objective=objective, row_violation_rel=float(rv.max(initial=0.0)),
               bound_violation=float(bv.max(initial=0.0)), dual_bound=None, dual_obj_loose=None, dual_infeas_rel=None,
               dual_gap_rel=None, dual_sign=None)
    if y is None or getattr(lp, "maximize", False):
        return out
    # the reference reads +-1e20 bounds as infinite; the model here stores them as inf
    lo_c, up_c = np.where(np.isfinite(lo), lo, -INF * 10), np.where(np.isfinite(up), up, INF * 10)
    l_c, u_c = np.where(np.isfinite(l), l, -INF * 10), np.where(np.isfinite(u), u, INF * 10)
    best = None
    for sgn in (1.0, -1.0):
        ys = sgn * np.asarray(y, float)
        tr, ir = _min_over(ys, lo_c, up_c)
        aty = np.zeros(n)
        np.add.at(aty, cols, lp.val * ys[lp.row_idx])
        d = cost - aty
        tc, ic = _min_over(d, l_c, u_c)
        infeas = max(float((ir / (1.0 + np.abs(ys))).max(initial=0.0)), float((ic / (1.0 + np.abs(cost))).max(initial=0.0)))
        loose = const + float(np.nansum(tr)) + float(np.nansum(tc))
        strict = not (np.isnan(tr).any() or np.isnan(tc).any())
        if best is None or infeas < best[0]:
            best = (infeas, sgn, loose, strict)
    infeas, sgn, loose, strict = best
    out.update(dual_sign=sgn, dual_infeas_rel=infeas, dual_obj_loose=loose, dual_bound=loose if strict else None,
               dual_gap_rel=(objective - loose) / max(1.0, abs(objective)))
    return out
