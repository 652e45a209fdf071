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


def test_oracle_voxel_filter_properties():
    """Voxel filter restatement (filterCloud.cu:84-133, 279-318): one output per end-point
    voxel, counts summing to the traced points, each mean inside its voxel, voxel order."""
    rng = np.random.default_rng(3)
    pts = rng.uniform(-2.0, 2.0, (20000, 3)).astype(np.float32)  # all within the 4 m range
    pts[::50] = pts[1::50]  # duplicates land in the same voxel
    pts[3::101] = (4.5, 0.0, 0.0)  # beyond the range: dropped
    pts[4::103] = np.nan  # dropped
    R = np.eye(3, dtype=np.float32).reshape(-1)
    res = 0.1
    eye, mt = O.frame_setup((0.123, -0.456, 0.789), res, 4.0, 1)
    fp, cnt = O.voxel_filter(R, eye, res, mt, 1, pts)
    fc, cnt_c = O.voxel_filter(R, eye, res, mt, 1, pts, centre=True)
    assert np.array_equal(cnt, cnt_c)
    assert int(cnt.sum()) == int(np.count_nonzero(np.all(np.abs(pts) <= 2.0, axis=1)))
    v_mean = np.floor(eye + fp.astype(np.float64) / res)
    v_cent = np.floor(eye + fc.astype(np.float64) / res)
    assert np.array_equal(v_mean, v_cent)          # each mean lies in its voxel
    assert len(np.unique(v_cent, axis=0)) == len(v_cent)
    keys = [tuple(v) for v in v_cent.astype(np.int64)]
    assert keys == sorted(keys)                    # x, then y, then z
    # the mean of one point is that point
    one, c1 = O.voxel_filter(R, eye, res, mt, 1, pts[:1])
    assert c1.tolist() == [1] and np.allclose(one[0], pts[0], atol=1e-5)
