"""Comparison helpers shared by the tests.

``match_rows`` restates the reference's golden-CSV rule (Tests_CPU/test_Palm.cpp:55-76): each actual row is paired
with the nearest unused expected row of the same Plane and Channel (squared distance in X, Y, Z), and every column
must satisfy |a - e| <= atol + rtol * |e| (numpy.isclose-style, rtol 1e-5).
"""
import numpy as np

COLS = 18
C_ID, C_PLANE, C_INDEX, C_CHANNEL, C_X, C_Y, C_Z = 0, 1, 2, 3, 4, 5, 6
C_INTENSITY, C_SX, C_SY, C_THETA, C_QXY, C_QZ, C_AMP, C_OFF, C_SEGI, C_SURF, C_CIRC = range(7, 18)


def theta_to_degrees(rows, fit):
    """The golden CSVs store theta in degrees folded into [-90, 90) for fit 4 (test_Palm.cpp:41-48)."""
    rows = rows.copy()
    if fit == 4 and len(rows):
        ok = (rows[:, C_SX] > 0) & (rows[:, C_SY] > 0)
        a = np.fmod(rows[ok, C_THETA] + np.pi / 2, np.pi)
        a[a < 0] += np.pi
        rows[ok, C_THETA] = (a - np.pi / 2) * 180 / np.pi
    return rows


def match_rows(actual, expected, atol=1e-3, rtol=1e-5, columns=None, keys=(C_X, C_Y, C_Z)):
    """Returns (n_bad_rows, worst_excess, pairs). ``pairs`` maps each actual row to its matched expected row;
    ``keys`` are the columns of the nearest-row distance (X, Y, Z as in the reference test; X, Y where Z is in nm)."""
    actual = np.asarray(actual, dtype=np.float64).reshape(-1, COLS)
    expected = np.asarray(expected, dtype=np.float64).reshape(-1, COLS)
    if actual.shape[0] != expected.shape[0]:
        return max(actual.shape[0], expected.shape[0]), np.inf, None
    cols = np.arange(COLS) if columns is None else np.asarray(columns)
    used = np.zeros(expected.shape[0], dtype=bool)
    pairs = np.full(actual.shape[0], -1)
    bad = 0
    worst = 0.0
    keyed = {}
    for j in range(expected.shape[0]):
        keyed.setdefault((expected[j, C_PLANE], expected[j, C_CHANNEL]), []).append(j)
    for i, row in enumerate(actual):
        cand = [j for j in keyed.get((row[C_PLANE], row[C_CHANNEL]), []) if not used[j]]
        if not cand:
            bad += 1
            worst = np.inf
            continue
        e = expected[cand]
        d = np.zeros(len(cand))
        for k in keys:
            d += (e[:, k] - row[k]) ** 2
        j = cand[int(np.argmin(d))]
        used[j] = True
        pairs[i] = j
        tol = atol + rtol * np.abs(expected[j, cols])
        excess = np.abs(row[cols] - expected[j, cols]) - tol
        excess = np.where(np.isnan(excess), np.where(np.isnan(row[cols]) & np.isnan(expected[j, cols]), -1.0, np.inf), excess)
        if np.any(excess > 0):
            bad += 1
            worst = max(worst, float(np.max(excess)))
    return bad, worst, pairs


def error_table(actual, expected, pairs, columns):
    """Per-column |actual - expected| percentiles over matched rows: {name: (median, p99, max)}."""
    out = {}
    ok = pairs >= 0
    for name, c in columns.items():
        d = np.abs(actual[ok, c] - expected[pairs[ok], c])
        if d.size == 0:
            out[name] = (0.0, 0.0, 0.0)
        else:
            out[name] = (float(np.median(d)), float(np.percentile(d, 99)), float(np.max(d)))
    return out
