"""Parity with the reference's own GPU backend on the same B200: `oracle/_ref/pdhg --device gpu` (gpu/pdhg.cu built
for sm_100a from its sources, FP64, its default) against this engine's FP64 path, model by model.

The reference's GPU FP64 run reproduces its CPU FP64 run (the ledgers), so the iteration and restart counts must
agree exactly and the objectives to 1e-9 relative; both report near_optimal at 1e-6."""
import json
import subprocess
import tempfile
from pathlib import Path

import pytest

import lpgen
from conftest import ROOT, bounded_pdhg as pdhg, rel

pytestmark = pytest.mark.gpu

REF = ROOT / "oracle" / "_ref" / "pdhg"

MODELS = {
    "packing_10000": lambda: lpgen.packing(10000),
    "transport_100x100": lambda: lpgen.transport(100, 100),
    "planted_2000x5000_s1": lambda: lpgen.planted(2000, 5000, 5, seed=1),
    "planted_zipf_20000x50000": lambda: lpgen.planted(20_000, 50_000, 10, seed=4, zipf=1.2, cap=2000, floor=5),
}


def _reference_gpu(lp, extra=()):
    with tempfile.TemporaryDirectory() as td:
        f, j = Path(td) / "m.mps", Path(td) / "r.json"
        lp.write_mps(f)
        subprocess.run([str(REF), str(f), "--device", "gpu", "--tol", "1e-6", "--time-limit", "120", "--json", str(j),
                        *extra], check=True, stdout=subprocess.DEVNULL, timeout=600)
        return json.loads(j.read_text())


@pytest.mark.skipif(not REF.exists(), reason="oracle/_ref/pdhg not built (make -C oracle ref)")
@pytest.mark.parametrize("name", sorted(MODELS))
def test_fp64_matches_reference_gpu_backend(engine_lib, name):
    lp = MODELS[name]()
    ref = _reference_gpu(lp)
    r, _, _ = pdhg.solve(lp, tol=1e-6, precision=pdhg.FP64)
    assert ref["status"] == r["status"] == "near_optimal", (name, ref["status"], r["status"])
    assert (r["iterations"], r["restarts"]) == (ref["iterations"], ref["restarts"]), (name, r, ref)
    assert rel(r["objective"], ref["objective"]) < 1e-9, (name, r["objective"], ref["objective"])
