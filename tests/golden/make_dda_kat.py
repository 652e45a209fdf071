"""Generates tests/golden/dda_kat.json: known-answer cases for the insertion DDA.

Each case is evaluated here with exact rational arithmetic (fractions.Fraction) on the
published Amanatides & Woo traversal, independently of the C++ oracle and of the GPU code:

* index space = world / res (res = 1 here, so eye = sensor position);
* the ray direction is the double-precision unit vector of the point (its exact binary value
  is taken as a rational);
* start voxel floor(eye); next crossing per axis = (boundary - eye) / dir; step the axis with
  the smallest next crossing, ties to the higher axis; zero components never step;
* every voxel left by a step whose crossing time is <= |p| / res is a miss; the voxel holding
  the end point is a hit when the crossing that leaves it is below max_range / res;
* points with |p| / res >= max_range / res, NaN or zero length produce nothing.

Rays are chosen so that double rounding cannot flip a comparison, except the deliberate
exact ties (equal direction components), which tie in both arithmetics.

Run: python tests/golden/make_dda_kat.py
"""
from __future__ import annotations

import json
import math
from fractions import Fraction
from pathlib import Path

OUT = Path(__file__).with_name("dda_kat.json")


def exact_dda(eye, p, max_range):
    if any(math.isnan(c) for c in p):
        return []
    length = math.sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2])
    if not (length < max_range) or length <= 1e-7:
        return []
    d = [Fraction(c / length) for c in p]  # exact value of the double-rounded unit vector
    e = [Fraction(c) for c in eye]
    t1 = Fraction(length)
    vox = [math.floor(c) for c in eye]
    nxt, dlt, stp = [], [], []
    for a in range(3):
        if d[a] == 0:
            nxt.append(None)
            dlt.append(None)
            stp.append(0)
        elif d[a] > 0:
            nxt.append((vox[a] + 1 - e[a]) / d[a])
            dlt.append(1 / d[a])
            stp.append(1)
        else:
            nxt.append((vox[a] - e[a]) / d[a])
            dlt.append(-1 / d[a])
            stp.append(-1)

    def less(x, y):
        if x is None:
            return False
        if y is None:
            return True
        return x < y

    events = []
    cur = list(vox)
    while True:
        n0, n1, n2 = nxt
        a = (0 if less(n0, n2) else 2) if less(n0, n1) else (1 if less(n1, n2) else 2)
        t = nxt[a]
        nxt[a] = t + dlt[a]
        vox[a] += stp[a]
        if not (t <= t1):
            break
        events.append(cur + [0])
        cur = list(vox)
    if t < Fraction(max_range):
        events.append(cur + [1])
    return events


CASES = [
    ("axis +x", (0.5, 0.5, 0.5), (3.2, 0.0, 0.0), 10.0),
    ("axis -x across zero", (0.5, 0.5, 0.5), (-3.2, 0.0, 0.0), 10.0),
    ("axis +z into the next leaf", (0.25, 0.75, 6.5), (0.0, 0.0, 3.0), 10.0),
    ("axis -y negative leaf", (-0.5, -7.5, 0.5), (0.0, -2.25, 0.0), 10.0),
    ("end point in the eye voxel", (0.5, 0.5, 0.5), (0.2, 0.1, -0.3), 10.0),
    ("beyond max range", (0.5, 0.5, 0.5), (12.0, 0.0, 0.0), 10.0),
    ("exactly max range", (0.5, 0.5, 0.5), (10.0, 0.0, 0.0), 10.0),
    ("end voxel leaves past max range", (0.5, 0.5, 0.5), (9.8, 0.0, 0.0), 10.0),
    ("zero point", (0.5, 0.5, 0.5), (0.0, 0.0, 0.0), 10.0),
    ("NaN point", (0.5, 0.5, 0.5), (float("nan"), 1.0, 0.0), 10.0),
    ("diagonal xy", (0.25, 0.5, 0.5), (2.0, 1.4, 0.0), 10.0),
    ("corner tie xyz", (0.5, 0.5, 0.5), (2.0, 2.0, 2.0), 10.0),
    ("corner tie xy", (0.5, 0.5, 0.5), (-1.6, -1.6, 0.0), 10.0),
    ("general 3d", (3.1, -2.7, 1.3), (4.3, 2.9, -1.7), 10.0),
    ("general 3d negative", (-10.3, 20.6, -0.4), (-3.7, -5.1, 2.3), 10.0),
    ("eye on a voxel face", (2.0, 3.0, 4.0), (1.7, -0.9, 0.4), 10.0),
    ("long ray", (100.25, -50.5, 8.75), (7.3, -4.1, 2.2), 10.0),
]


def main():
    cases = []
    for name, eye, p, mr in CASES:
        cases.append({"name": name, "eye": list(eye), "point": [None if math.isnan(c) else c for c in p],
                      "nan": any(math.isnan(c) for c in p), "max_range": mr,
                      "events": exact_dda(eye, p, mr)})
    OUT.write_text(json.dumps({"res": 1.0, "rounding": "nearest", "cases": cases}, indent=1))
    print(f"wrote {OUT} ({len(cases)} cases)")


if __name__ == "__main__":
    main()
