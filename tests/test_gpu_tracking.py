"""Tracking on the GPU (the Tracking export and PTB_TrackingDevice) against the oracle, bit for bit: the reference's
golden CSVs and known answers, seeded drifting emitters with blinking and empty planes, equal distances everywhere,
segments longer than the shared-memory sort (one plane of 5000 points, a transition with more than 2048 pairs),
radius edge values, and a large stack."""
import numpy as np
import pytest

import tracking_cases as tc
from test_tracking import _edge_cases

pytestmark = pytest.mark.gpu


def test_tracking_golden_and_known(lib, orc):
    for name, pts, expected in tc.golden_cases():
        for p in (pts, pts[::-1].copy()):
            got = lib.tracking(p, 5.0)
            assert np.array_equal(got, orc.tracking(p, 5.0)), name
            assert {int(a): int(b) for a, b in got} == expected, name
    for name, pts, r, expected in tc.known_cases():
        got = lib.tracking(pts, r)
        assert np.array_equal(got, orc.tracking(pts, r)), name
        if expected is not None:
            assert np.array_equal(got.reshape(-1), expected), name
    assert lib.tracking(np.zeros((0, 4)), 5.0).shape == (0, 2)


def test_tracking_edge_cases(lib, orc):
    for name, pts, r in _edge_cases():
        assert np.array_equal(lib.tracking(pts, r), orc.tracking(pts, r)), name
    rng = np.random.default_rng(21)
    # one plane with 5000 points (global-memory sort of the plane), then a dense transition with > 2048 pairs
    big_plane = np.c_[np.arange(1, 5001), np.ones(5000), rng.uniform(0, 100, (5000, 2))]
    assert np.array_equal(lib.tracking(big_plane, 2.0), orc.tracking(big_plane, 2.0))
    dense = np.r_[np.c_[np.arange(1, 101), np.ones(100), rng.uniform(0, 5, (100, 2))],
                  np.c_[np.arange(101, 201), np.full(100, 2.0), rng.uniform(0, 5, (100, 2))]]
    assert np.array_equal(lib.tracking(dense, 4.0), orc.tracking(dense, 4.0))
    # Ids far apart and planes starting high
    sparse = tc.synthetic(9, planes=20, per_plane=100)
    sparse[:, 0] = sparse[:, 0] * 1e9
    sparse[:, 1] += 123456
    assert np.array_equal(lib.tracking(sparse, 2.0), orc.tracking(sparse, 2.0))


def _boundary_points(x0, y0, r, seed):
    """A source point and targets on and just around the circle of radius r (the window search's edge cases)."""
    rng = np.random.default_rng(seed)
    rows = [[1, 1, x0, y0]]
    targets = [(x0 + r, y0), (x0 - r, y0), (np.nextafter(x0 + r, np.inf), y0), (np.nextafter(x0 - r, -np.inf), y0),
               (x0, y0 + r), (x0, np.nextafter(y0 - r, -np.inf))]
    for t in rng.uniform(0, 2 * np.pi, 40):
        targets.append((x0 + r * np.cos(t), y0 + r * np.sin(t)))
    for k, (x, y) in enumerate(targets):
        rows.append([k + 2, 2, x, y])
    # more sources in plane 1 on the same circle, so that many pairs sit at distance ~r
    for k, t in enumerate(rng.uniform(0, 2 * np.pi, 20)):
        rows.append([100 + k, 1, x0 + r * np.cos(t), y0 + r * np.sin(t)])
    return np.array(rows, dtype=np.float64)


@pytest.mark.parametrize("r", [2.0, 0.1, 5.0, 1e-140, 1e140, 3.0e-5])
@pytest.mark.parametrize("x0", [0.0, 1000.3, 1.0e6 + 0.123])
def test_tracking_window_boundary(lib, orc, r, x0):
    pts = _boundary_points(x0, 17.25, r, seed=int(x0) % 97 + 3)
    for radius in (r, np.nextafter(r, 0.0), np.nextafter(r, np.inf)):
        assert np.array_equal(lib.tracking(pts, radius), orc.tracking(pts, radius)), radius


def test_tracking_large(lib, orc):
    pts = tc.synthetic(33, planes=400, per_plane=1500, size=2048.0, step=1.0, blink=0.2, gap_every=37)
    assert pts.shape[0] > 400000
    assert np.array_equal(lib.tracking(pts, 3.0), orc.tracking(pts, 3.0))


def test_tracking_device_entry(lib, orc):
    import torch
    pts = tc.synthetic(5, planes=30, per_plane=300)
    d_in = torch.from_numpy(pts).cuda()
    d_out = torch.full((pts.shape[0], 2), 7, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    n = lib.load().PTB_TrackingDevice(d_in.data_ptr(), d_out.data_ptr(), pts.shape[0], 2.0, stream)
    torch.cuda.synchronize()
    assert n == 2 * pts.shape[0]
    assert np.array_equal(d_out.cpu().numpy().view(np.uint64), orc.tracking(pts, 2.0))
