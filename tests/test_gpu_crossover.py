"""Crossover handoff: the .sol / .dual files of this engine's CLI start the reference simplex (`taral --warm-sol F
--warm-dual F`, src/main.cpp:661-683, built from the reference's sources into oracle/_ref/) and the simplex ends at
the same optimum as its cold solve. The file formats (one `name value` line per column / row) are the reference
PDHG's, so the reference harness can hand either engine's output to its crossover unchanged."""
import json
import subprocess
from pathlib import Path

import pytest

import lpgen
from conftest import rel

ROOT = Path(__file__).resolve().parents[1]
CLI = ROOT / "taral-lp_b200" / "bin" / "pdhg"
TARAL = ROOT / "oracle" / "_ref" / "taral"

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [lambda: lpgen.transport(30, 40, seed=2), lambda: lpgen.packing(2000, seed=3)],
                         ids=["transport_30x40", "packing_2000"])
def test_pdhg_solution_warm_starts_reference_crossover(engine_lib, tmp_path, make):
    if not TARAL.exists():
        pytest.skip("reference binary not built (make -C oracle ref)")
    lp = make()
    mps, sol, dual = tmp_path / "m.mps", tmp_path / "m.sol", tmp_path / "m.dual"
    lp.write_mps(mps)
    subprocess.run([str(CLI), str(mps), "--tol", "1e-6", "--sol", str(sol), "--dual", str(dual), "--json",
                    str(tmp_path / "p.json")], check=True, stdout=subprocess.DEVNULL, timeout=300)
    assert json.loads((tmp_path / "p.json").read_text())["status"] == "near_optimal"
    runs = {}
    for name, extra in (("cold", []), ("warm", ["--warm-sol", str(sol), "--warm-dual", str(dual)])):
        j = tmp_path / f"{name}.json"
        subprocess.run([str(TARAL), str(mps), "--method", "dual", "--time-limit", "120", "--json", str(j), *extra],
                       check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=300)
        runs[name] = json.loads(j.read_text())
    assert runs["cold"]["status"] == "optimal" and runs["warm"]["status"] == "optimal"
    assert rel(runs["warm"]["objective"], runs["cold"]["objective"]) < 1e-9
