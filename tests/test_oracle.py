"""Pins of the CPU oracle (oracle/pdhg_oracle.c) before it is trusted as the checker.

1. The reference's published ledgers (results/gpu_pdhg/synth_*_tol1e-{4,6}.csv, CPU FP64 rows): iteration and
   restart counts, objective to the printed digits, relative KKT errors.
2. The reference binary built from its own sources (tests/golden/reference_runs.json, made by
   tests/golden/make_golden.py): counts, objectives, weights and the written .sol / .dual vectors.
3. The FP64 optimum of the reference's interior-point method on the planted 2000 x 5000 model."""
import numpy as np
import pytest

import lpgen
import oracle
from conftest import golden, rel

PINS = golden("ledger_pins.json")
RUNS = golden("reference_runs.json")
VECS = golden("reference_vectors.npz")
OPTIMA = golden("reference_optima.json")

LEDGER_MODELS = {"packing_10000": lambda: lpgen.packing(10000), "transport_100x100": lambda: lpgen.transport(100, 100)}
RUN_MODELS = {
    "packing_2000_s3": lambda: lpgen.packing(2000, seed=3),
    "transport_30x40_s2": lambda: lpgen.transport(30, 40, seed=2),
    "planted_300x700_s5": lambda: lpgen.planted(300, 700, 5, seed=5),
    "general_300x700_s3_max": lambda: lpgen.general(300, 700, seed=3, maximize=True),
    "general_300x700_s3": lambda: lpgen.general(300, 700, seed=3),
    "general_200x500_s7": lambda: lpgen.general(200, 500, seed=7),
}


def flags_to_kw(flags):
    kw, it = {}, iter(flags)
    for f in it:
        v = next(it)
        key = {"--tol": "tol", "--row-rel": "row_rel", "--eval-freq": "eval_freq", "--max-iter": "max_iter"}[f]
        kw[key] = float(v) if key in ("tol", "row_rel") else int(v)
    return kw


def model_for(name):
    base = next(k for k in sorted(RUN_MODELS, key=len, reverse=True) if name.startswith(k))
    return RUN_MODELS[base]()


@pytest.mark.parametrize("key", sorted(PINS))
def test_oracle_reproduces_published_ledger(oracle_lib, key):
    pin = PINS[key]
    r, _, _ = oracle.solve(LEDGER_MODELS[pin["case"]](), tol=float(pin["tol"]))
    assert r["status"] == pin["status"]
    assert r["iterations"] == int(pin["iterations"]) and r["restarts"] == int(pin["restarts"])
    assert f"{r['objective']:.12g}" == pin["objective"]
    for k, kk in (("rel_p", "rel_primal"), ("rel_d", "rel_dual"), ("rel_gap", "rel_gap")):
        assert f"{r[k]:.6e}" == f"{float(pin[kk]):.6e}"
    assert f"{r['max_row_viol']:.6e}" == f"{float(pin['max_row_violation']):.6e}"


@pytest.mark.parametrize("name", sorted(RUNS))
def test_oracle_reproduces_reference_binary(oracle_lib, name):
    ref = RUNS[name]
    lp = model_for(name)
    assert lp.digest() == ref["model_sha256"]
    r, x, y = oracle.solve(lp, **flags_to_kw(ref["flags"]))
    assert (r["status"], r["iterations"], r["restarts"]) == (ref["status"], ref["iterations"], ref["restarts"])
    assert bool(r["from_average"]) == (ref["point"] == "average")
    assert rel(r["objective"], ref["objective"]) < 1e-12
    assert f"{r['omega']:.6e}" == f"{ref['primal_weight']:.6e}" and f"{r['norm_a']:.6e}" == f"{ref['norm_a']:.6e}"
    assert np.allclose(x, VECS[name + "/x"], rtol=1e-12, atol=1e-13)
    assert np.allclose(y, VECS[name + "/y"], rtol=1e-12, atol=1e-13)


def test_oracle_reaches_reference_ipm_optimum(oracle_lib):
    opt = OPTIMA["planted_2000x5000_s0"]
    lp = lpgen.planted(2000, 5000, 5, seed=0)
    assert lp.digest() == opt["model_sha256"]
    assert rel(opt["objective"], opt["planted_objective"]) < 1e-9  # the planted optimum is the true optimum
    r, _, _ = oracle.solve(lp, tol=1e-7)
    assert r["status"] == "near_optimal" and rel(r["objective"], opt["objective"]) < 1e-6


def test_oracle_spmv_and_transpose(oracle_lib):
    lp = lpgen.general(60, 90, seed=1)
    ptr, idx, val = lp.csr()
    x = np.random.default_rng(0).standard_normal(lp.n)
    dense = np.zeros((lp.m, lp.n))
    for i in range(lp.m):
        dense[i, idx[ptr[i]:ptr[i + 1]]] = val[ptr[i]:ptr[i + 1]]
    assert np.allclose(oracle.spmv(ptr, idx, val, x), dense @ x, rtol=1e-13, atol=1e-13)
    sp = oracle.ScaledProblem(lp)
    a_s = np.zeros((lp.m, lp.n))
    for i in range(lp.m):
        a_s[i, sp.A[1][sp.A[0][i]:sp.A[0][i + 1]]] = sp.A[2][sp.A[0][i]:sp.A[0][i + 1]]
    at_s = np.zeros((lp.n, lp.m))
    for j in range(lp.n):
        at_s[j, sp.AT[1][sp.AT[0][j]:sp.AT[0][j + 1]]] = sp.AT[2][sp.AT[0][j]:sp.AT[0][j + 1]]
    assert np.array_equal(a_s.T, at_s)
    assert np.allclose(a_s, sp.Dr[:, None] * dense * sp.Dc[None, :], rtol=1e-13, atol=0)


def test_oracle_nan_cost_semantics(oracle_lib):
    """A NaN cost leaves the primal measure finite while the dual and gap measures are NaN. The reference's
    worst() is std::max(p, std::max(d, g)), which returns p when the other argument is NaN, so the run stops
    as near_optimal with a NaN objective instead of numerical_failure. The restatement keeps that behaviour."""
    lp = lpgen.general(30, 50, seed=4)
    lp.cost = lp.cost.copy()
    lp.cost[0] = np.nan
    r, _, _ = oracle.solve(lp, tol=1e-6, max_iter=20000)
    assert r["status"] == "near_optimal" and np.isnan(r["objective"]) and np.isnan(r["rel_d"])


def test_mlp_oracle_gradients_by_finite_differences():
    """The numpy MLP restatement's analytic gradient agrees with central differences (no bf16 rounding)."""
    import mlp_oracle
    rng = np.random.default_rng(0)
    shapes = [((5, 7), (7,)), ((7, 7), (7,)), ((7, 4), (4,))]
    n = sum(a * b + b for (a, b), _ in shapes)
    p = rng.standard_normal(n) * 0.4
    x, t = rng.standard_normal((6, 5)), rng.standard_normal((6, 4))
    saved = mlp_oracle.bf16
    mlp_oracle.bf16 = lambda a: np.asarray(a, np.float64)
    try:
        _, g = mlp_oracle.loss_and_grads(p, shapes, x, t)
        for i in rng.choice(n, 12, replace=False):
            e = np.zeros(n)
            e[i] = 1e-6
            fd = (mlp_oracle.loss_and_grads(p + e, shapes, x, t)[0] - mlp_oracle.loss_and_grads(p - e, shapes, x, t)[0]) / 2e-6
            assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i]))
    finally:
        mlp_oracle.bf16 = saved
