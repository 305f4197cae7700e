"""Seeded synthetic LP families for the PDHG engine's tests and benchmarks (synthetic data, not real-world).

Every family returns an :class:`LP`, a column-wise model with the field semantics of the reference's
``Model`` (src/taral.hpp:22-35): ``min cost'x + obj_const  s.t.  row_lo <= A x <= row_up,
col_lo <= x <= col_up``, +-inf for absent bounds, entries of each column row-ascending.

* ``packing`` and ``transport`` draw the same random streams as the reference's gpu/gen_lp.py:46-101 and
  round every written number through ``%.12g`` as its MPS writer does, so the models equal what the
  reference's own MPS reader returns for its files; the published PDHG ledgers
  (results/gpu_pdhg/synth_*_tol1e-{4,6}.csv) therefore apply to them as known answers.
* ``planted`` is the planted-optimum family: A with N(0,1) values, equality rows A x = b, 0 <= x <= 10,
  and an optimal primal-dual pair (x*, y*) built in, so c'x* is the exact optimum at any size. Uniform
  rows (5 per column) or power-law (Zipf) row lengths to stress SpMV skew.
* ``refinery`` is the multi-period refinery-structured family (block-diagonal periods joined by inventory
  rows) with a planted feasible point, and perturbed scenario copies of it for batched solves.
"""
from __future__ import annotations

import dataclasses
import hashlib
from typing import Optional

import numpy as np

INF = float("inf")


@dataclasses.dataclass
class LP:
    """Column-wise LP. ``col_ptr`` (int64, n+1), ``row_idx`` (int32), ``val`` (float64) form CSC."""

    name: str
    m: int
    n: int
    col_ptr: np.ndarray
    row_idx: np.ndarray
    val: np.ndarray
    cost: np.ndarray
    col_lo: np.ndarray
    col_up: np.ndarray
    row_lo: np.ndarray
    row_up: np.ndarray
    obj_const: float = 0.0
    maximize: bool = False
    row_types: Optional[list] = None     # 'E' / 'L' / 'G' per row, for the MPS writer
    row_names: Optional[np.ndarray] = None
    col_names: Optional[np.ndarray] = None
    x_star: Optional[np.ndarray] = None  # planted optimum (planted family) or planted feasible point
    y_star: Optional[np.ndarray] = None
    obj_star: Optional[float] = None

    @property
    def nnz(self) -> int:
        return int(self.col_ptr[-1])

    def csr(self):
        """Row-wise copy (ptr int64, idx int32, val float64), columns ascending within each row."""
        cols = np.repeat(np.arange(self.n, dtype=np.int32), np.diff(self.col_ptr))
        order = np.lexsort((cols, self.row_idx))
        ptr = np.zeros(self.m + 1, np.int64)
        np.cumsum(np.bincount(self.row_idx, minlength=self.m), out=ptr[1:])
        return ptr, cols[order].astype(np.int32), self.val[order]

    def digest(self) -> str:
        """sha256 over the model arrays (exact doubles), for fixtures."""
        h = hashlib.sha256()
        for a in (self.col_ptr.astype(np.int64), self.row_idx.astype(np.int32), self.val, self.cost, self.col_lo,
                  self.col_up, self.row_lo, self.row_up):
            h.update(np.ascontiguousarray(a).tobytes())
        h.update(np.float64(self.obj_const).tobytes())
        return h.hexdigest()

    # ------------------------------------------------------------------ MPS
    def _names(self):
        rn = self.row_names if self.row_names is not None else np.char.add("R", np.arange(self.m).astype(str))
        cn = self.col_names if self.col_names is not None else np.char.add("X", np.arange(self.n).astype(str))
        return rn, cn

    def mps_text(self) -> str:
        """Free-format MPS in the layout of the reference's writer (gpu/gen_lp.py:24-43): one entry per line,
        OBJ first in each column, numbers as %.12g. Rows are written with their sense; ranged rows use RANGES."""
        rn, cn = self._names()
        types = self.row_types
        if types is None:
            types = []
            for lo, up in zip(self.row_lo, self.row_up):
                types.append("E" if lo == up else ("L" if lo == -INF else "G"))
        parts = [f"NAME {self.name}\n"]
        if self.maximize:
            parts.append("OBJSENSE\n MAX\n")
        parts.append("ROWS\n N OBJ\n")
        parts.append("".join(f" {t} {r}\n" for t, r in zip(types, rn)))
        parts.append("COLUMNS\n")
        cnt = np.diff(self.col_ptr)
        has_obj = self.cost != 0
        # per column: [OBJ line] + entries
        ncol_lines = cnt + has_obj
        tot = int(ncol_lines.sum())
        cn_all = np.repeat(cn, ncol_lines)
        start = np.zeros(self.n + 1, np.int64)
        np.cumsum(ncol_lines, out=start[1:])
        is_obj = np.zeros(tot, bool)
        is_obj[start[:-1][has_obj]] = True
        rn_all = np.empty(tot, dtype=object)
        v_all = np.empty(tot, np.float64)
        rn_all[is_obj] = "OBJ"
        v_all[is_obj] = self.cost[has_obj]
        rn_all[~is_obj] = rn[self.row_idx]
        v_all[~is_obj] = self.val
        lines = np.char.add(np.char.add(np.char.add(np.char.add("    ", cn_all.astype(str)), " "),
                                        np.char.add(rn_all.astype(str), " ")), np.char.mod("%.12g", v_all))
        if tot:
            parts.append("\n".join(lines.tolist()))
            parts.append("\n")
        parts.append("RHS\n")
        rhs, rng_rows = [], []
        for i, (t, lo, up) in enumerate(zip(types, self.row_lo, self.row_up)):
            b = up if t == "L" else lo
            rhs.append((rn[i], b))
            if t in "LG" and np.isfinite(lo) and np.isfinite(up):
                rng_rows.append((rn[i], up - lo))
            elif t == "E" and lo != up:
                rng_rows.append((rn[i], up - lo))
        if self.obj_const != 0:
            rhs.append(("OBJ", -self.obj_const))
        parts.append("".join(f"    RHS {r} {v:.12g}\n" for r, v in rhs))
        if rng_rows:
            parts.append("RANGES\n")
            parts.append("".join(f"    RNG {r} {v:.12g}\n" for r, v in rng_rows))
        blines = []
        for j in range(self.n):
            lo, up = self.col_lo[j], self.col_up[j]
            if lo == 0 and up == INF:
                continue
            if lo == up:
                blines.append(f" FX BND {cn[j]} {lo:.12g}")
                continue
            if lo == -INF and up == INF:
                blines.append(f" FR BND {cn[j]}")
                continue
            if lo == -INF:
                blines.append(f" MI BND {cn[j]}")
            elif lo != 0:
                blines.append(f" LO BND {cn[j]} {lo:.12g}")
            if up != INF:
                blines.append(f" UP BND {cn[j]} {up:.12g}")
        if blines:
            parts.append("BOUNDS\n")
            parts.append("\n".join(blines))
            parts.append("\n")
        parts.append("ENDATA\n")
        return "".join(parts)

    def write_mps(self, path) -> None:
        with open(path, "w") as f:
            f.write(self.mps_text())


def _r12_text(v):
    """Round doubles through the '%.12g' text the MPS writer emits (what a reader of that file sees)."""
    return np.char.mod("%.12g", np.asarray(v, np.float64)).astype(np.float64)


_POW10 = np.array([10.0 ** k for k in range(23)])  # exactly representable powers of ten


def _r12(v):
    """The same doubles as _r12_text, computed arithmetically: with e the decimal exponent of |v| and k = 11 - e,
    M = the integer nearest to v * 10^k (12 significant digits) and the result M / 10^k (or M * 10^-k), one
    correctly rounded IEEE operation on two exact operands, i.e. the double nearest to the decimal M * 10^-k, which
    is what reading the 12-digit text gives. Values where the float product v * 10^k lies within 4 ulps of a
    rounding tie, near a power of ten, or outside 10^-11 .. 10^22 go through the text instead."""
    v0 = np.asarray(v, np.float64)
    v = v0.ravel()
    out = v.copy()
    idx = np.nonzero(np.isfinite(v) & (v != 0))[0]
    if idx.size == 0:
        return out.reshape(v0.shape)
    a = np.abs(v[idx])
    lg = np.log10(a)
    e = np.floor(lg).astype(np.int64)
    k = 11 - e
    ok = (np.abs(lg - np.rint(lg)) > 1e-9) & (k >= 0) & (k <= 22)
    kk = np.clip(k, 0, 22)
    scaled = a * _POW10[kk]
    M = np.rint(scaled)
    tie = np.abs(scaled - np.floor(scaled) - 0.5) <= 4 * np.spacing(scaled)
    ok &= ~tie & (M >= 1e11) & (M <= 1e12)
    r = np.copysign(M / _POW10[kk], v[idx])
    out[idx[ok]] = r[ok]
    rest = idx[~ok]
    if rest.size:
        out[rest] = _r12_text(v[rest])
    return out.reshape(v0.shape)


def _csc_from_lists(n, rows_per_col, vals_per_col, keep=None):
    """CSC from (n, K) row and value arrays; entries with keep False are dropped; rows sorted per column."""
    if keep is None:
        keep = np.ones(rows_per_col.shape, bool)
    cnt = keep.sum(axis=1)
    col_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(cnt, out=col_ptr[1:])
    return col_ptr, rows_per_col[keep].astype(np.int32), vals_per_col[keep].astype(np.float64)


# ---------------------------------------------------------------------------------------------- reference families
def packing(N: int, K: int = 5, seed: int = 1) -> LP:
    """Packing LP of the reference's generator (gpu/gen_lp.py:71-101): min -p'x, A x <= b, 0 <= x <= 1,
    K random rows per column (repeats dropped), values U(0.1,1), b = A x0 * U(1,1.5) + 0.1."""
    rng = np.random.default_rng(seed)
    M = max(1, N // 2)
    rows = np.sort(rng.integers(0, M, (N, K)), axis=1)
    dup = np.zeros_like(rows, dtype=bool)
    dup[:, 1:] = rows[:, 1:] == rows[:, :-1]
    vals = rng.uniform(0.1, 1.0, (N, K))
    vals[dup] = 0
    x0 = rng.random(N)
    ax0 = np.zeros(M)
    np.add.at(ax0, rows.ravel(), (vals * x0[:, None]).ravel())
    b = ax0 * rng.uniform(1.0, 1.5, M) + 0.1
    p = rng.uniform(0.5, 1.5, N)
    col_ptr, ri, v = _csc_from_lists(N, rows, _r12(vals), keep=~dup)
    return LP(name=f"PACKING_{N}", m=M, n=N, col_ptr=col_ptr, row_idx=ri, val=v, cost=_r12(-p),
              col_lo=np.zeros(N), col_up=np.ones(N), row_lo=np.full(M, -INF), row_up=_r12(b),
              row_types=["L"] * M)


def transport(S: int, D: int, seed: int = 1) -> LP:
    """Transportation LP of the reference's generator (gpu/gen_lp.py:46-68): S supplies (L rows), D demands
    (G rows), one column per (i, j) with cost = distance of random points, total supply 1.25 x demand."""
    rng = np.random.default_rng(seed)
    ps, pd = rng.random((S, 2)), rng.random((D, 2))
    demand = rng.uniform(1, 10, D)
    supply = rng.uniform(1, 10, S)
    supply *= 1.25 * demand.sum() / supply.sum()
    ii = np.repeat(np.arange(S), D)
    jj = np.tile(np.arange(D), S)
    cost = np.sqrt(((ps[ii] - pd[jj]) ** 2).sum(axis=1))
    n = S * D
    rows = np.stack([ii, S + jj], axis=1)
    col_ptr, ri, v = _csc_from_lists(n, rows, np.ones((n, 2)))
    row_lo = np.concatenate([np.full(S, -INF), _r12(demand)])
    row_up = np.concatenate([_r12(supply), np.full(D, INF)])
    names = np.array([f"S{i}" for i in range(S)] + [f"D{j}" for j in range(D)])
    return LP(name=f"TRANSPORT_{S}x{D}", m=S + D, n=n, col_ptr=col_ptr, row_idx=ri, val=v, cost=_r12(cost),
              col_lo=np.zeros(n), col_up=np.full(n, INF), row_lo=row_lo, row_up=row_up,
              row_types=["L"] * S + ["G"] * D, row_names=names)


def reference_mps_text(lp: LP) -> str:
    """The exact bytes the reference's gpu/gen_lp.py writes for a packing or transport model."""
    if lp.name.startswith("PACKING"):
        return lp.mps_text()
    # transport: every column has its OBJ line; no BOUNDS section
    return lp.mps_text()


# ---------------------------------------------------------------------------------------------- planted optimum
def _distinct_rows(rng, m, n, k):
    """(n, k) row indices, k distinct uniform rows per column, sorted."""
    rows = np.sort(rng.integers(0, m, (n, k)), axis=1)
    for _ in range(64):
        dup = np.zeros(rows.shape, bool)
        dup[:, 1:] = rows[:, 1:] == rows[:, :-1]
        bad = np.nonzero(dup.any(axis=1))[0]
        if bad.size == 0:
            return rows
        rows[bad] = np.sort(rng.integers(0, m, (bad.size, k)), axis=1)
    raise RuntimeError("could not draw distinct rows")


def zipf_row_lengths(m: int, nnz: int, s: float = 1.2, cap: int = 2000, floor: int = 5) -> np.ndarray:
    """Deterministic power-law row lengths: the row of rank r gets clip(C r^-s, floor, cap), with C chosen so
    the lengths sum to nnz (the last few units are spread over the uncapped rows)."""
    r = np.arange(1, m + 1, dtype=np.float64)
    lo, hi = 0.0, float(cap) * m
    for _ in range(200):
        C = 0.5 * (lo + hi)
        tot = np.clip(C * r ** -s, floor, cap).sum()
        if tot < nnz:
            lo = C
        else:
            hi = C
    L = np.clip(np.floor(C * r ** -s), floor, cap).astype(np.int64)
    short = nnz - int(L.sum())
    free = np.nonzero(L < cap)[0]
    if short > 0:
        L[free[np.arange(short) % free.size]] += 1
    elif short < 0:
        big = np.nonzero(L > floor)[0]
        L[big[np.arange(-short) % big.size]] -= 1
    return L


def planted(m: int, n: int, per_col: int = 5, seed: int = 0, zipf: Optional[float] = None, cap: int = 2000,
            floor: int = 5, name: Optional[str] = None) -> LP:
    """Planted-optimum LP: min c'x s.t. A x = b, 0 <= x <= 10.

    A: per_col nonzeros per column with N(0,1) values, at distinct uniform-random rows, or (zipf=s) at rows
    whose lengths follow the power law of :func:`zipf_row_lengths` (rows shuffled). x*: 40% of the entries at
    0, 10% at 10, the rest U(0.5, 9.5); y* ~ N(0,1); b = A x*; reduced costs z* with |z*| ~ U(0.1, 1), >= 0 at
    lower-bound entries, <= 0 at upper-bound entries, 0 otherwise; c = A'y* + z*. (x*, y*) satisfies the KKT
    conditions, so c'x* is the optimum.
    """
    rng = np.random.default_rng(seed)
    if zipf is None:
        rows = _distinct_rows(rng, m, n, per_col)
        keep = np.ones(rows.shape, bool)
    else:
        L = zipf_row_lengths(m, n * per_col, s=zipf, cap=cap, floor=floor)
        L = L[rng.permutation(m)]
        slots = np.repeat(np.arange(m, dtype=np.int64), L)
        rng.shuffle(slots)
        rows = np.sort(slots.reshape(n, per_col), axis=1)
        keep = np.ones(rows.shape, bool)
        keep[:, 1:] = rows[:, 1:] != rows[:, :-1]
    vals = _r12(rng.standard_normal(rows.shape))
    col_ptr, ri, v = _csc_from_lists(n, rows, vals, keep=keep)
    u = rng.random(n)
    x = np.where(u < 0.4, 0.0, np.where(u < 0.5, 10.0, 0.0))
    mid = u >= 0.5
    x[mid] = rng.uniform(0.5, 9.5, int(mid.sum()))
    y = rng.standard_normal(m)
    mag = rng.uniform(0.1, 1.0, n)
    z = np.where(u < 0.4, mag, np.where(u < 0.5, -mag, 0.0))
    cols = np.repeat(np.arange(n), np.diff(col_ptr))
    b = np.zeros(m)
    np.add.at(b, ri, v * x[cols])
    aty = np.zeros(n)
    np.add.at(aty, cols, v * y[ri])
    b, c = _r12(b), _r12(aty + z)  # every number as the MPS file carries it; x*, y* stay optimal to ~1e-12
    obj = float(np.dot(c, x))
    return LP(name=name or f"PLANTED_{m}x{n}", m=m, n=n, col_ptr=col_ptr, row_idx=ri, val=v, cost=c,
              col_lo=np.zeros(n), col_up=np.full(n, 10.0), row_lo=b.copy(), row_up=b.copy(),
              row_types=["E"] * m, x_star=x, y_star=y, obj_star=obj)


# ---------------------------------------------------------------------------------------------- general LP
def general(m: int, n: int, per_col: int = 4, seed: int = 0, maximize: bool = False) -> LP:
    """Bounded LP with every row and bound kind: E, L, G and ranged rows; free, lower-only, upper-only, boxed
    and fixed columns. A planted primal point x0 is feasible (rows hold A x0 with slack on their open side) and
    planted multipliers y0 / reduced costs d make the dual feasible (sign of y by row kind, sign of d by which
    column bounds are finite), so the optimum is finite. Values N(0,1) rounded to 6 decimals."""
    rng = np.random.default_rng(seed)
    rows = _distinct_rows(rng, m, n, per_col)
    vals = np.round(rng.standard_normal(rows.shape), 6)
    vals[vals == 0] = 0.5
    col_ptr, ri, v = _csc_from_lists(n, rows, vals)
    ck = rng.choice(5, n, p=[0.1, 0.3, 0.1, 0.4, 0.1])  # 0 free, 1 lower, 2 upper, 3 boxed, 4 fixed
    x0 = np.round(rng.uniform(-2, 2, n), 3)
    lo = np.where(np.isin(ck, (1, 3)), x0 - np.round(rng.uniform(0, 2, n), 3), -INF)
    up = np.where(np.isin(ck, (2, 3)), x0 + np.round(rng.uniform(0, 2, n), 3), INF)
    lo = _r12(np.where(ck == 4, x0, lo))
    up = _r12(np.where(ck == 4, x0, up))
    cols = np.repeat(np.arange(n), np.diff(col_ptr))
    ax0 = np.zeros(m)
    np.add.at(ax0, ri, v * x0[cols])
    rk = rng.choice(4, m, p=[0.3, 0.3, 0.3, 0.1])  # 0 E, 1 L, 2 G, 3 ranged
    slack = np.round(rng.uniform(0, 1, m), 3)
    rlo = np.where(rk == 0, ax0, np.where(rk == 2, ax0 - slack, np.where(rk == 3, ax0 - slack, -INF)))
    rup = np.where(rk == 0, ax0, np.where(rk == 1, ax0 + slack, np.where(rk == 3, ax0 + 1 + slack, INF)))
    rlo, rup = _r12(rlo), _r12(rup)
    rup = np.where(rk == 3, rlo + _r12(1 + slack), rup)  # a ranged row is read back as lo + |R|
    y0 = np.round(rng.standard_normal(m), 3)
    y0 = np.where(rk == 1, -np.abs(y0), np.where(rk == 2, np.abs(y0), y0))  # min form: y <= 0 on L, >= 0 on G
    d = np.round(rng.uniform(0, 1, n), 3)
    d = np.where(ck == 0, 0.0, np.where(ck == 2, -d, np.where(ck == 3, rng.choice([-1, 1], n) * d, d)))
    aty = np.zeros(n)
    np.add.at(aty, cols, v * y0[ri])
    c = _r12(aty + d)
    types = ["E" if k == 0 else ("L" if k == 1 else "G") for k in rk]
    if maximize:
        c = -c
    return LP(name=f"GENERAL_{m}x{n}_{seed}", m=m, n=n, col_ptr=col_ptr, row_idx=ri, val=v, cost=c,
              col_lo=lo, col_up=up, row_lo=rlo, row_up=rup, obj_const=0.5, maximize=maximize, row_types=types)


# ---------------------------------------------------------------------------------------------- refinery family
# One period block: 1,500 rows x 4,000 columns.
#   columns  [0,1000) process (crude -> unit) activities   [1000,3000) intermediate flows to blend pools
#            [3000,3800) product sales                       [3800,4000) closing inventory of 200 storable items
#   rows     [0,500) yield balances (E)   [500,800) unit capacities (L)   [800,1300) blend quality (G)
#            [1300,1500) inventory balances (E)
# A process column yields into 26 intermediates with U(0,1) coefficients scaled to sum U(0.85,1) (<= 1) and uses
# 3 capacity rows (coefficient 1). A flow column consumes its intermediate (-1) and carries U(-1,1) quality
# coefficients into 12 quality rows; 10% also feed an inventory balance (+1). A sales column has U(-1,1) in 18
# quality rows and draws -1 from an inventory balance. An inventory column is -1 in its item's balance of period
# t and +1 in that of period t+1 (the linking rows). About 71k nonzeros per period (3.4M at 48 periods).
# Bounds 0 <= x <= U(100,1000) (capacities), costs U(-50,50) (prices). A point x0 in [0, 0.5 x capacity] is
# planted: yield and inventory rows are equalities at A x0, capacity rows allow 1.3 A x0 + 10, quality rows
# require at least A x0 - U(0,1)(1 + |A x0|). Perturbation: 128 price groups scale costs and 128 capacity groups
# scale column capacities and capacity-row limits, each by a factor in [0.8, 1.2]; x0 stays feasible.
REF_ROWS, REF_COLS, REF_GROUPS = 1500, 4000, 128


class RefineryBase:
    """The 48-period structure of one scenario family (matrix, planted point, base prices and capacities)."""

    def __init__(self, periods: int = 48, seed: int = 7):
        rng = np.random.default_rng(seed)
        R, Cn = REF_ROWS, REF_COLS
        self.periods, self.seed = periods, seed
        rows_l, cols_l, vals_l = [], [], []
        for t in range(periods):
            r0, c0 = t * R, t * Cn
            # process columns
            nP = 1000
            yr = np.sort(np.stack([rng.choice(500, 26, replace=False) for _ in range(nP)]), axis=1)
            yv = rng.uniform(0, 1, (nP, 26))
            yv *= (rng.uniform(0.85, 1.0, nP) / yv.sum(axis=1))[:, None]
            cr = np.sort(np.stack([rng.choice(300, 3, replace=False) for _ in range(nP)]), axis=1) + 500
            pc = np.repeat(np.arange(nP), 29)
            rows_l.append(r0 + np.concatenate([yr, cr], axis=1).ravel())
            cols_l.append(c0 + pc)
            vals_l.append(np.concatenate([yv, np.ones((nP, 3))], axis=1).ravel())
            # flow columns
            nF = 2000
            src = rng.integers(0, 500, nF)
            qr = np.stack([rng.choice(500, 12, replace=False) for _ in range(nF)]) + 800
            qv = rng.uniform(-1, 1, (nF, 12))
            inv = rng.random(nF) < 0.1
            invr = rng.integers(0, 200, nF) + 1300
            for_rows = [src, qr]
            fr = np.concatenate([src[:, None], qr], axis=1)
            fv = np.concatenate([-np.ones((nF, 1)), qv], axis=1)
            fc = np.repeat(np.arange(1000, 1000 + nF), 13)
            rows_l.append(r0 + fr.ravel()), cols_l.append(c0 + fc), vals_l.append(fv.ravel())
            rows_l.append(r0 + invr[inv]), cols_l.append(c0 + 1000 + np.nonzero(inv)[0]), vals_l.append(np.ones(inv.sum()))
            # sales columns
            nS = 800
            sr = np.stack([rng.choice(500, 18, replace=False) for _ in range(nS)]) + 800
            sv = rng.uniform(-1, 1, (nS, 18))
            sb = rng.integers(0, 200, nS) + 1300
            rows_l.append(r0 + np.concatenate([sr, sb[:, None]], axis=1).ravel())
            cols_l.append(c0 + np.repeat(np.arange(3000, 3000 + nS), 19))
            vals_l.append(np.concatenate([sv, -np.ones((nS, 1))], axis=1).ravel())
            # inventory columns: -1 in this period's balance, +1 in the next period's
            k = np.arange(200)
            rows_l.append(r0 + 1300 + k), cols_l.append(c0 + 3800 + k), vals_l.append(-np.ones(200))
            if t + 1 < periods:
                rows_l.append(r0 + R + 1300 + k), cols_l.append(c0 + 3800 + k), vals_l.append(np.ones(200))
        rows = np.concatenate(rows_l).astype(np.int64)
        cols = np.concatenate(cols_l).astype(np.int64)
        vals = _r12(np.concatenate(vals_l))
        order = np.lexsort((rows, cols))
        self.rows, self.cols, self.vals = rows[order].astype(np.int32), cols[order], vals[order]
        self.m, self.n = periods * R, periods * Cn
        self.cap = np.round(rng.uniform(100, 1000, self.n), 3)
        self.price = np.round(rng.uniform(-50, 50, self.n), 4)
        self.x0 = rng.uniform(0, 0.5, self.n) * self.cap
        self.qslack = rng.uniform(0, 1, self.m)
        self.price_group = np.tile(rng.integers(0, REF_GROUPS, Cn), periods)
        self.cap_group_col = np.tile(rng.integers(0, REF_GROUPS, Cn), periods)
        self.cap_group_row = np.tile(rng.integers(0, REF_GROUPS, R), periods)

    def instance(self, periods: int, perturb: Optional[np.ndarray] = None, name: Optional[str] = None) -> LP:
        """The LP of the first `periods` periods, with prices / capacities scaled by the 256-vector `perturb`
        (None: all ones). The links of the last period to a later one are dropped."""
        R, Cn = REF_ROWS, REF_COLS
        m, n = periods * R, periods * Cn
        st = self._structure(periods)
        p = np.ones(2 * REF_GROUPS) if perturb is None else np.asarray(perturb, np.float64)
        fprice = p[self.price_group[:n]]
        fcap_c = p[REF_GROUPS + self.cap_group_col[:n]]
        fcap_r = p[REF_GROUPS + self.cap_group_row[:m]]
        ax0, rtype = st["ax0"], st["rtype"]
        row_up = np.where(rtype == 0, ax0, np.where(rtype == 1, (1.3 * ax0 + 10) * fcap_r, INF))
        return LP(name=name or f"REFINERY_T{periods}", m=m, n=n, col_ptr=st["col_ptr"], row_idx=st["rows"],
                  val=st["vals"], cost=_r12(self.price[:n] * fprice), col_lo=np.zeros(n),
                  col_up=_r12(self.cap[:n] * fcap_c), row_lo=st["row_lo"], row_up=_r12(row_up),
                  row_types=st["row_types"], x_star=self.x0[:n])

    def _structure(self, periods: int) -> dict:
        """The parts of instance(periods) that the perturbation does not touch (computed once per period count;
        the arrays are shared by the instances and must not be modified)."""
        cache = self.__dict__.setdefault("_cache", {})
        if periods in cache:
            return cache[periods]
        R, Cn = REF_ROWS, REF_COLS
        m, n = periods * R, periods * Cn
        keep = (self.cols < n) & (self.rows < m)
        cols, rows, vals = self.cols[keep], self.rows[keep], self.vals[keep]
        col_ptr = np.zeros(n + 1, np.int64)
        np.cumsum(np.bincount(cols, minlength=n), out=col_ptr[1:])
        x0 = self.x0[:n]
        ax0 = np.bincount(rows, weights=vals * x0[cols], minlength=m)  # sequential adds in entry order
        rtype = np.empty(m, np.int8)
        loc = np.arange(m) % R
        rtype[loc < 500] = 0                      # E yield
        rtype[(loc >= 500) & (loc < 800)] = 1     # L capacity
        rtype[(loc >= 800) & (loc < 1300)] = 2    # G quality
        rtype[loc >= 1300] = 0                    # E inventory
        row_lo = np.where(rtype == 0, ax0, np.where(rtype == 2, ax0 - self.qslack[:m] * (1 + np.abs(ax0)), -INF))
        for a in (col_ptr, rows, vals):
            a.setflags(write=False)
        st = {"col_ptr": col_ptr, "rows": rows, "vals": vals, "ax0": ax0, "rtype": rtype, "row_lo": _r12(row_lo),
              "row_types": ["E" if k == 0 else ("L" if k == 1 else "G") for k in rtype]}
        cache[periods] = st
        return st


def refinery(periods: int = 48, seed: int = 7, perturb: Optional[np.ndarray] = None) -> LP:
    """Refinery-structured multi-period LP (48 periods: 72,000 rows x 192,000 columns, ~3.4M nonzeros)."""
    return RefineryBase(max(periods, 1), seed).instance(periods, perturb)


def perturbations(count: int, seed: int) -> np.ndarray:
    """`count` independent 256-vectors of price / capacity factors, U(0.8, 1.2)."""
    return np.random.default_rng(seed).uniform(0.8, 1.2, (count, 2 * REF_GROUPS))
