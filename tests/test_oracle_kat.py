"""Pins the CPU oracle's insertion DDA to hand-derived known answers (tests/golden)."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = json.loads((Path(__file__).parent / "golden" / "dda_kat.json").read_text())


def _point(c):
    return [float("nan") if (c["nan"] and v is None) else float(v) for v in c["point"]]


@pytest.mark.parametrize("case", GOLDEN["cases"], ids=[c["name"] for c in GOLDEN["cases"]])
@pytest.mark.parametrize("rounding", [0, 1])
def test_dda_known_answers(case, rounding):
    R = np.eye(3, dtype=np.float32).reshape(-1)
    ev = O.trace(R, np.array(case["eye"], np.float64), 1.0, np.float32(case["max_range"]),
                 rounding, _point(case))
    got = [] if ev is None else ev.tolist()
    assert got == case["events"]


def test_kat_covers_edge_cases():
    names = {c["name"] for c in GOLDEN["cases"]}
    for must in ("zero point", "NaN point", "beyond max range", "corner tie xyz",
                 "end point in the eye voxel", "axis -x across zero"):
        assert must in names
