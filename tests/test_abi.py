"""The C-ABI library loads, exports every function include/taral_pdhg.h declares, and rejects bad input
before touching a device (no GPU needed)."""
import ctypes as C

import numpy as np
import pytest

import lpgen
import pdhg
from conftest import has_gpu


def test_exports_every_declared_symbol(engine_lib):
    declared = pdhg.header_symbols()
    assert len(declared) >= 25
    missing = [s for s in declared if not hasattr(engine_lib, s)]
    assert not missing, missing
    assert set(declared) == set(pdhg.SIGNATURES), set(declared) ^ set(pdhg.SIGNATURES)


def test_default_options(engine_lib):
    o = pdhg.default_options()
    assert (o.tol, o.time_limit, o.max_iter, o.eval_freq, o.row_rel, o.graph, o.precision) == \
        (1e-4, 3600.0, 2_000_000_000, 64, 0.0, 1, pdhg.FP64)


def test_create_rejects_bad_csr(engine_lib):
    lp = lpgen.general(20, 30, seed=1)
    ptr, idx, val = lp.csr()
    a = pdhg._Csr(ptr, idx, val, lp.n)
    bad = pdhg._Csr(ptr, np.where(idx == idx.max(), lp.n + 5, idx), val, lp.n)
    v = [np.ones(lp.n)] * 3 + [np.ones(lp.m)] * 2 + [np.ones(lp.m), np.ones(lp.n)]
    h = C.c_void_p()
    code = engine_lib.pdhg_create(C.byref(bad.s), C.byref(a.s), *[pdhg._p(x) for x in v], lp.m, lp.n, 0, 64, 0,
                                  C.byref(h))
    assert code == pdhg.ERR_INPUT and not h.value
    code = engine_lib.pdhg_create(C.byref(a.s), C.byref(a.s), *[pdhg._p(x) for x in v], lp.m, lp.n, 7, 64, 0,
                                  C.byref(h))
    assert code == pdhg.ERR_INPUT


def test_null_context_calls(engine_lib):
    assert engine_lib.pdhg_iterate(None, 1) == pdhg.ERR_INPUT
    assert engine_lib.pdhg_last_error(None) == b"NULL context"
    engine_lib.pdhg_destroy(None)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_device_is_reported(engine_lib):
    with pytest.raises(pdhg.TaralError) as e:
        pdhg.solve(lpgen.general(20, 30, seed=1))
    assert e.value.code == pdhg.ERR_NO_DEVICE


def test_solve_rejects_unsupported_before_device(engine_lib):
    lp = lpgen.general(20, 30, seed=1)
    lp.n_quadratic = 2
    with pytest.raises(pdhg.TaralError) as e:
        pdhg.solve(lp)
    assert e.value.code == pdhg.ERR_UNSUPPORTED
