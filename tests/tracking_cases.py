"""Inputs for the Tracking tests: the reference's known-answer cases (Tests_CPU/test_tr_Tracks.cpp), its golden CSVs
(tests/golden/tracking.npz with the localizations they were linked from) and seeded synthetic tracks.
"""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_cases():
    """[(name, points [n, 4] (Id, Plane, X, Y), {Id: Track})] from the reference's tracking CSVs (maxDistance 5):
    the localizations with positive integrated intensity (test_tr_Tracks.cpp:256-261)."""
    locs = np.load(os.path.join(GOLDEN, "localizations.npz"))
    tracks = np.load(os.path.join(GOLDEN, "tracking.npz"))
    cases = []
    for key in sorted(tracks.files):
        suffix = key[len("stack-tracking-"):-len("-5")]
        rows = locs["stack-localizations-" + suffix]
        rows = rows[rows[:, 7] > 0]
        pts = np.ascontiguousarray(rows[:, [0, 1, 4, 5]])
        expected = {int(r[2]): int(r[0]) for r in tracks[key]}
        cases.append((key, pts, expected))
    return cases


# (points, maxDistance, expected output) from Tests_CPU/test_tr_Tracks.cpp
KNOWN = {
    # TrackingWithGaps (:210-247)
    "gaps": ([[1, 3, 0.0, 0.0], [2, 3, 10.0, 10.0], [3, 3, 5.0, 5.0], [4, 4, 0.2, 0.0], [5, 4, 0.6, 0.0],
              [6, 4, 5.2, 5.0], [7, 6, 0.3, 0.0], [8, 6, 20.0, 20.0], [9, 7, 0.4, 0.0], [10, 7, 20.2, 20.0]], 1.0,
             [1, 1, 2, 2, 3, 3, 4, 1, 5, 4, 6, 3, 7, 5, 8, 6, 9, 5, 10, 6]),
    # ResolvesConflicts, exact ties and fallback neighbour (:181-196)
    "ties": ([[1, 1, 0, 0], [2, 1, 0.0, 0], [3, 2, 1, 0], [4, 2, -1.0, 0]], 1.0, [1, 1, 2, 2, 3, 1, 4, 2]),
    "fallback": ([[1, 1, 0, 0], [2, 1, 2.2, 0], [3, 2, 1, 0], [4, 2, 3.7, 0]], 2.0, [1, 1, 2, 2, 3, 1, 4, 2]),
}


def known_cases():
    out = []
    for name, (pts, r, expected) in KNOWN.items():
        pts = np.array(pts, dtype=np.float64)
        out.append((name, pts, r, np.array(expected, dtype=np.uint64)))
        out.append((name + "_reversed", pts[::-1].copy(), r, np.array(expected, dtype=np.uint64)))
    # ResolvesCloseDistances (:199-207): two distances closer than an epsilon are not ties
    d = np.sqrt(np.finfo(np.float64).eps / 2)
    out.append(("close", np.array([[1, 1, d, 0], [2, 1, 0, 0], [3, 2, 0, 0]], dtype=np.float64), 1.0, None))
    return out


def synthetic(seed, planes=50, per_plane=200, size=512.0, step=0.8, blink=0.1, gap_every=0, shuffle=True):
    """Seeded emitters drifting by ~step px per plane, each visible with probability 1 - blink, plus planes left
    empty every gap_every planes; Ids numbered in (Plane, order of appearance), rows shuffled when asked."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, size, (per_plane, 2))
    rows = []
    nid = 1
    for p in range(1, planes + 1):
        pos = pos + rng.normal(0, step, pos.shape)
        if gap_every and p % gap_every == 0:
            continue
        vis = rng.random(per_plane) >= blink
        for x, y in pos[vis]:
            rows.append([nid, p, x, y])
            nid += 1
    pts = np.array(rows, dtype=np.float64)
    if shuffle:
        pts = pts[rng.permutation(len(pts))]
    return pts
