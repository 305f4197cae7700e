"""The oracle's restatement of the reference's independent answer check (oracle/check_oracle.py) against the
reference checker itself: gpu/vector_check.check_files on the reference PDHG's .sol / .dual of the pinned runs
(tests/golden/reference_vector_check.json)."""
import json
import sys
from pathlib import Path

import numpy as np
import pytest

import check_oracle

GOLD = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLD))
import make_golden  # noqa: E402  (the runs' model factories)

FIELDS = [("objective", "chk_objective"), ("row_violation_rel", "chk_row_viol_rel"),
          ("bound_violation", "chk_bound_viol"), ("dual_bound", "chk_dual_bound"),
          ("dual_obj_loose", "chk_dual_obj_loose"), ("dual_infeas_rel", "chk_dual_infeas_rel"),
          ("dual_gap_rel", "chk_dual_gap_rel"), ("dual_sign", "chk_dual_sign")]


def close(a, b):
    if a is None or b is None:
        return a is None and b is None
    return abs(a - b) <= 1e-9 * max(1.0, abs(b))


@pytest.mark.parametrize("name,make", [(r[0], r[1]) for r in make_golden.RUNS], ids=[r[0] for r in make_golden.RUNS])
def test_check_restatement_matches_reference(name, make):
    gold = json.loads((GOLD / "reference_vector_check.json").read_text())[name]
    vecs = np.load(GOLD / "reference_vectors.npz")
    lp = make()
    assert lp.digest() == gold["model_sha256"]
    out = check_oracle.check(lp, vecs[name + "/x"], vecs[name + "/y"])
    for mine, ref in FIELDS:
        assert close(out[mine], gold[ref]), (mine, out[mine], gold[ref])
