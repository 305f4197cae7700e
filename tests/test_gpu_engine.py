"""Step-level parity of the CUDA engine with the CPU oracle (backend concept of gpu/pdhg.cu:313-514).

Both sides start from the same scaled problem (the oracle's scaling) and execute the same calls; FP64 results
must agree to rounding (different summation orders), FP32 results to single precision."""
import numpy as np
import pytest

import lpgen
import oracle
import pdhg
from conftest import rel

pytestmark = pytest.mark.gpu

CASES = {
    "packing_2000": lambda: lpgen.packing(2000, seed=3),
    "transport_30x40": lambda: lpgen.transport(30, 40, seed=2),
    "general_300x700": lambda: lpgen.general(300, 700, seed=3),
    "planted_zipf": lambda: lpgen.planted(3000, 6000, 8, seed=1, zipf=1.2, cap=3000),
}


def _pair(lp, precision=pdhg.FP64):
    sp = oracle.ScaledProblem(lp)
    eng = pdhg.Engine.from_scaled(sp, precision=precision)
    ref = oracle.Stepper(sp)
    return sp, eng, ref


def _close(a, b, rtol, atol=1e-300):
    a, b = np.asarray(a), np.asarray(b)
    scale = np.maximum(np.abs(b), 1.0)
    return np.all(np.abs(a - b) <= rtol * scale + atol)


@pytest.mark.parametrize("case", sorted(CASES))
def test_power_norm_fp64(engine_lib, oracle_lib, case):
    sp, eng, _ = _pair(CASES[case]())
    assert abs(eng.power_norm(200) - sp.power_norm(200)) <= 1e-12 * sp.power_norm(200)


@pytest.mark.parametrize("case", sorted(CASES))
def test_steps_match_oracle_fp64(engine_lib, oracle_lib, case):
    """start -> eval -> 3 blocks of 64 steps with a restart to the average and one to the current point."""
    sp, eng, ref = _pair(CASES[case]())
    norm = sp.power_norm(200)
    tau = sigma = 0.95 / norm
    for b in (eng, ref):
        b.set_steps(tau * 0.7, sigma / 0.7)
        b.start()
    assert _close(eng.eval(0, 1.0), ref.eval(0, 1.0), 1e-11)
    for blk, action in enumerate(("avg", "cur", None)):
        for b in (eng, ref):
            b.iterate(64)
        f = 1.0 / 64
        cur, avg = eng.eval_pair(f)
        assert _close(cur, ref.eval(0, 1.0), 1e-9), (blk, cur, ref.eval(0, 1.0))
        assert _close(avg, ref.eval(1, f), 1e-9), (blk, avg, ref.eval(1, f))
        xg, zg = eng.download(1, f)
        xo, zo = ref.download(1, f)
        assert _close(xg, xo, 1e-9) and _close(zg, zo, 1e-9)
        if action:
            for b in (eng, ref):
                b.restart(action == "avg", f)
    xg, zg = eng.download(0, 1.0)
    xo, zo = ref.download(0, 1.0)
    assert _close(xg, xo, 1e-9) and _close(zg, zo, 1e-9)


@pytest.mark.parametrize("case", ["packing_2000", "general_300x700"])
def test_steps_fp32_track_fp64(engine_lib, oracle_lib, case):
    """FP32 iterates follow the FP64 trajectory to single-precision accuracy over one block."""
    sp, eng, ref = _pair(CASES[case](), pdhg.FP32)
    norm = sp.power_norm(200)
    for b in (eng, ref):
        b.set_steps(0.95 / norm, 0.95 / norm)
        b.start()
        b.iterate(64)
    xg, zg = eng.download(1, 1 / 64)
    xo, zo = ref.download(1, 1 / 64)
    assert _close(xg, xo, 1e-4) and _close(zg, zo, 1e-4)


def test_deterministic(engine_lib, oracle_lib):
    """Fixed-order reductions: two contexts give bit-identical KKT scalars and iterates."""
    lp = CASES["planted_zipf"]()
    outs = []
    for _ in range(2):
        sp, eng, _ = _pair(lp)
        eng.set_steps(0.5, 0.5)
        eng.start()
        eng.iterate(64)
        outs.append((eng.eval_pair(1 / 64), eng.download(0, 1.0)))
    (c1, a1), (x1, z1) = outs[0]
    (c2, a2), (x2, z2) = outs[1]
    assert np.array_equal(c1, c2) and np.array_equal(a1, a2) and np.array_equal(x1, x2) and np.array_equal(z1, z2)


def test_graph_and_direct_launch_agree(engine_lib, oracle_lib):
    lp = CASES["general_300x700"]()
    sp = oracle.ScaledProblem(lp)
    res = []
    for graph in (True, False):
        eng = pdhg.Engine.from_scaled(sp, graph=graph)
        eng.set_steps(0.4, 0.6)
        eng.start()
        eng.iterate(64)
        eng.iterate(64)
        res.append(eng.download(0, 1.0))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


def test_warm_start_point(engine_lib, oracle_lib):
    lp = CASES["general_300x700"]()
    sp = oracle.ScaledProblem(lp)
    eng = pdhg.Engine.from_scaled(sp)
    rng = np.random.default_rng(0)
    x0, z0 = rng.standard_normal(sp.n), rng.standard_normal(sp.m)
    eng.set_steps(0.5, 0.5)
    eng.start(x0, z0)
    x, z = eng.download(0, 1.0)
    assert np.array_equal(x, x0) and np.array_equal(z, z0)


def test_state_errors(engine_lib, oracle_lib):
    sp = oracle.ScaledProblem(CASES["packing_2000"]())
    eng = pdhg.Engine.from_scaled(sp)
    with pytest.raises(pdhg.TaralError) as e:
        eng.iterate(8)
    assert e.value.code == pdhg.ERR_STATE
    bad_idx = sp.A[1].copy()
    bad_idx[-1] = sp.n  # a column index out of range is rejected before anything reaches the device
    with pytest.raises(pdhg.TaralError) as e:
        pdhg.Engine((sp.A[0], bad_idx, sp.A[2]), sp.AT, sp.c, sp.l, sp.u, sp.rl, sp.ru, sp.Dr, sp.Dc)
    assert e.value.code == pdhg.ERR_INPUT


def test_kernel_launch_count(engine_lib, oracle_lib):
    sp = oracle.ScaledProblem(CASES["packing_2000"]())
    eng = pdhg.Engine.from_scaled(sp)
    eng.set_steps(0.5, 0.5)
    eng.start()
    before = eng.kernel_launches
    eng.iterate(64)
    eng.iterate(64)
    assert eng.kernel_launches - before == 2 * (1 + 2 * 64)


@pytest.mark.parametrize("policy", ["0", "1", "2", "3", "4"])
def test_row_split_policies_agree(engine_lib, monkeypatch, policy):
    # the five row-split policies of the autotuner (hybrid, thread per row in uniform blocks, balanced segmented
    # sums, 8-lane groups for rows of 49..128 nonzeros, uniform blocks plus groups) on a Zipf LP whose long rows span
    # many threads of a block: each reaches the tolerance at the same objective (they differ only in the FP64
    # summation order of the products)
    monkeypatch.setenv("TARAL_ROWSPLIT", policy)
    lp = lpgen.planted(20_000, 50_000, 10, seed=4, zipf=1.2, cap=2000, floor=5)
    r, x, _ = pdhg.solve(lp, tol=1e-6, precision=pdhg.FP32, time_limit=120)
    assert r["status"] == "near_optimal", r
    assert rel(r["objective"], lp.obj_star) < 1e-5, (r["objective"], lp.obj_star)


@pytest.mark.parametrize("precision", [pdhg.FP64, pdhg.FP32])
def test_row_thread_kernel_is_bit_identical(engine_lib, monkeypatch, precision):
    # matrices whose rows all hold at most 48 nonzeros may run on the one-thread-per-row kernel: the same products
    # summed in the same order as the row blocks' thread path, so the whole solve is bit-identical either way
    lp = lpgen.packing(2000, seed=3)  # rows of A ~10, of A^T 5 nonzeros
    outs = []
    for flag in ("0", "1"):
        monkeypatch.setenv("TARAL_ROWTHREAD", flag)
        r, x, y = pdhg.solve(lp, tol=1e-6, precision=precision)
        outs.append((r, x, y))
    (r0, x0, y0), (r1, x1, y1) = outs
    assert r0["status"] == r1["status"] == "near_optimal"
    assert (r0["iterations"], r0["restarts"], r0["objective"]) == (r1["iterations"], r1["restarts"], r1["objective"])
    assert np.array_equal(x0, x1) and np.array_equal(y0, y1)


@pytest.mark.parametrize("precision", [pdhg.FP64, pdhg.FP32], ids=["fp64", "fp32"])
def test_row_order(engine_lib, monkeypatch, precision):
    # Contexts run with their rows sorted by length inside the engine (TARAL_ROWORDER=1, the default; the same
    # kernels as in the model's order): the same answer, and the dual vector comes back in the model's row order.
    # FP64: every row's products are summed in the same order, only the FP64 KKT sums over rows change order; the
    # iteration and restart counts stay those of the model's order and the answer agrees to rounding.
    lp = lpgen.planted(20_000, 50_000, 10, seed=4, zipf=1.2, cap=2000, floor=5)
    monkeypatch.setenv("TARAL_ROWORDER", "0")
    r0, x0, y0 = pdhg.solve(lp, tol=1e-6, precision=precision, time_limit=120)
    monkeypatch.setenv("TARAL_ROWORDER", "1")
    r1, x1, y1 = pdhg.solve(lp, tol=1e-6, precision=precision, time_limit=120)
    assert r0["status"] == r1["status"] == "near_optimal"
    assert rel(r1["objective"], lp.obj_star) < 1e-5 and rel(r1["objective"], r0["objective"]) < 1e-6
    if precision == pdhg.FP64:
        assert (r1["iterations"], r1["restarts"]) == (r0["iterations"], r0["restarts"])
        assert rel(r1["objective"], r0["objective"]) < 1e-12
        assert np.max(np.abs(x1 - x0)) <= 1e-9 * max(1.0, np.max(np.abs(x0)))
        assert np.max(np.abs(y1 - y0)) <= 1e-9 * max(1.0, np.max(np.abs(y0)))
    else:
        assert abs(r1["iterations"] - r0["iterations"]) <= 0.1 * r0["iterations"], (r0["iterations"], r1["iterations"])
        assert np.max(np.abs(y1 - y0)) <= 1e-3 * max(1.0, np.max(np.abs(y0)))  # rows in the model's order
    # a start point goes in and comes back in the model's order (translated both ways)
    eng = pdhg.Engine.from_model(lp, precision=precision)
    rng = np.random.default_rng(5)
    xs, zs = rng.standard_normal(lp.n), rng.standard_normal(lp.m)
    eng.set_steps(0.5, 0.5)
    eng.start(xs, zs)
    xb, zb = eng.download(0, 1.0)
    cast = np.float32 if precision == pdhg.FP32 else np.float64
    assert np.array_equal(xb, xs.astype(cast).astype(np.float64))
    assert np.array_equal(zb, zs.astype(cast).astype(np.float64))


@pytest.mark.parametrize("precision", [pdhg.FP64, pdhg.FP32], ids=["fp64", "fp32"])
def test_device_scaling_equals_host_scaling(engine_lib, oracle_lib, precision):
    """The set-up scales the model on the device (Ruiz x10, then Pock-Chambolle, in FP64 with the reference's
    operation order): Dr, Dc and the scaled values of A and A^T equal the oracle's host restatement of
    gpu/pdhg.cu:80-133 element by element (FP32 contexts: the same values narrowed to float). The models cover
    explicit zeros in the columns, a maximisation, power-law rows (FP32: rows held in length order internally),
    free and fixed columns."""
    zeros = lpgen.general(250, 600, seed=8)
    zeros.val = zeros.val.copy()
    zeros.val[::17] = 0.0  # explicit zeros: dropped before scaling, as the reference's column-wise copy drops them
    models = [zeros, lpgen.general(300, 700, seed=3, maximize=True), lpgen.packing(3000, seed=2),
              lpgen.planted(3000, 8000, 6, seed=2, zipf=1.2, cap=400, floor=3), lpgen.transport(20, 30, seed=4)]
    narrow = (lambda v: v) if precision == pdhg.FP64 else (lambda v: np.asarray(v).astype(np.float32).astype(np.float64))
    for lp in models:
        sp = oracle.ScaledProblem(lp)
        eng = pdhg.Engine.from_model(lp, precision=precision)
        dr, dc, a, at = eng.scaled_problem(len(sp.A[2]))
        assert np.array_equal(dr, narrow(sp.Dr)) and np.array_equal(dc, narrow(sp.Dc)), lp.name
        assert np.array_equal(a, narrow(sp.A[2])) and np.array_equal(at, narrow(sp.AT[2])), lp.name
        assert eng.bnorm == sp.bnorm and eng.cnorm == sp.cnorm, lp.name
        eng.close()


@pytest.mark.parametrize("precision", [pdhg.FP64, pdhg.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("case", ["packing_2000", "general_300x700", "transport_30x40"])
def test_programmatic_launch_changes_nothing(engine_lib, oracle_lib, monkeypatch, precision, case):
    """TARAL_PDL=1 launches the phase kernels with programmatic dependent launch. On these small grids a whole phase
    fits the GPU at once, the case where an early release would let a kernel read vectors its predecessor's
    predecessor is still writing: the iterates must equal the plain launches' bit for bit, through restarts."""
    outs = []
    for flag in ("0", "1"):
        monkeypatch.setenv("TARAL_PDL", flag)
        sp, eng, _ = _pair(CASES[case](), precision)
        eng.set_steps(0.5 / sp.power_norm(200), 0.5 / sp.power_norm(200))
        eng.start()
        for action in ("avg", "cur", None):
            eng.iterate(64)
            if action:
                eng.restart(action == "avg", 1 / 64)
        outs.append((eng.eval_pair(1 / 64), eng.download(0, 1.0)))
        eng.close()
    (c0, a0), (x0, z0) = outs[0]
    (c1, a1), (x1, z1) = outs[1]
    assert np.array_equal(c0, c1) and np.array_equal(a0, a1) and np.array_equal(x0, x1) and np.array_equal(z0, z1)


@pytest.mark.parametrize("precision", [pdhg.FP64, pdhg.FP32], ids=["fp64", "fp32"])
def test_power_norm_replay_and_repeated_solves(engine_lib, oracle_lib, precision):
    """The power iteration replays one captured chunk of steps: a second call on the same context and a context
    without graphs give the same estimate (FP64: the oracle's to 1e-12); two solves on one context give the same
    outcome and point."""
    lp = CASES["planted_zipf"]()
    sp = oracle.ScaledProblem(lp)
    eng = pdhg.Engine.from_scaled(sp, precision=precision)
    direct = pdhg.Engine.from_scaled(sp, precision=precision, graph=False)
    a, b, c = eng.power_norm(200), eng.power_norm(200), direct.power_norm(200)
    assert a == b == c, (a, b, c)
    if precision == pdhg.FP64:
        assert abs(a - sp.power_norm(200)) <= 1e-12 * a
    e2 = pdhg.Engine.from_model(lp, precision=precision)
    (r0, x0, z0), (r1, x1, z1) = [e2.solve(e2.bnorm, e2.cnorm, tol=1e-6) for _ in range(2)]
    assert r0["status"] == r1["status"] == "near_optimal"
    assert (r0["iterations"], r0["restarts"], r0["objective"]) == (r1["iterations"], r1["restarts"], r1["objective"])
    assert np.array_equal(x0, x1) and np.array_equal(z0, z1)
