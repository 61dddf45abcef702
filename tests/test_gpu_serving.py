"""Serving (PTB_ServerStart / PTB_SubmitStack / PTB_StackResult): every stack's result is the same when it runs in a
mix of concurrent stacks of other shapes, lengths and fit modes as when it runs alone, and equals Localization's.
The maximum-likelihood fits of concurrent requests are fused into shared launches; stacks wait for device memory
when the budget admits only one at a time.

The fit mapping is pinned (PTB_MLE_LANES=1) so that the autotuner of each slot cannot pick a different, equally
valid mapping; with it the kernels are deterministic per ROI and the rows must match bit for bit.
"""
import numpy as np
import pytest

from conftest import GAUSS_PARAMS

pytestmark = pytest.mark.gpu

MLE6 = np.array([7.0, 1.3, 100.0, 2.0, 20, 0.0])
ASTIG = [150.0, 400.0, 0.05, 0.0, 1.3 * 160, -150.0, 400.0, -0.05, 0.0, 1.3 * 160]
MLE7 = np.array([11.0, 160.0] + ASTIG + [100.0, 2.0, 20, -600.0, 600.0, 0.0])


def _mix(orc):
    import synth
    cases = []
    for k, (workload, frames, size, fit, params) in enumerate([
            ("c1", 5, None, 6, MLE6), ("c1", 3, (128, 128), 2, GAUSS_PARAMS), ("c3", 2, None, 7, MLE7),
            ("c1", 1, None, 0, GAUSS_PARAMS), ("c2", 2, None, 6, MLE6), ("c1", 4, (256, 512), 4, GAUSS_PARAMS),
            ("c1", 6, (128, 256), 6, MLE6), ("c3", 1, (256, 256), 7, MLE7)]):
        s, _ = synth.stack(workload, frames=frames, seed=500 + k, size=size)
        thr = synth.mad_threshold(orc.planes(s[0])[1])
        cases.append((s, thr, fit, params))
    return cases


@pytest.mark.parametrize("fuse", ["1", "0"])
def test_served_mix_equals_alone(lib, orc, monkeypatch, fuse):
    monkeypatch.setenv("PTB_MLE_LANES", "1")
    monkeypatch.setenv("PTB_FUSE_FITS", fuse)
    # a long window: the fit stage waits for every busy slot's chunk, so concurrent requests are fused for sure
    monkeypatch.setenv("PTB_FUSE_WINDOW_US", "200000")
    cases = _mix(orc)
    alone = [lib.localization(s, thr, 0.0, fit, p) for s, thr, fit, p in cases]
    server = lib.Server(slots=4, budget_bytes=8 << 30)
    try:
        # all at once: the stacks overlap on the device
        tickets = [server.submit(s, thr, 0.0, fit, p) for s, thr, fit, p in cases]
        mixed = [server.result(t) for t in tickets]
        fused = server.fuse_stats()
        # one at a time through the server
        served_alone = []
        for s, thr, fit, p in cases:
            served_alone.append(server.result(server.submit(s, thr, 0.0, fit, p)))
    finally:
        server.stop()
    print("fused fit launches", fused)
    if fuse == "1":
        # chunks of different requests (modes 6 and 7 separately) shared launches
        assert fused["launches"] >= 1 and fused["chunks"] > fused["launches"], fused
    else:
        assert fused == {"launches": 0, "chunks": 0}
    for i, (ref, (m, q, lat), (a, _, _)) in enumerate(zip(alone, mixed, served_alone)):
        assert ref.shape[0] > 0 or cases[i][2] == 0
        assert m.shape == ref.shape and np.array_equal(m, ref), i
        assert a.shape == ref.shape and np.array_equal(a, ref), i
        assert 0.0 <= q <= lat


def test_server_reports_errors_and_restarts(lib):
    server = lib.Server(slots=2, budget_bytes=1 << 30)
    try:
        with pytest.raises(RuntimeError):
            server.result(987654321)  # unknown ticket
        s = np.zeros((1, 64, 64), np.uint16)
        rows, _, _ = server.result(server.submit(s, 100.0, 0.0, 2, GAUSS_PARAMS))
        assert rows.shape == (0, 18)
    finally:
        server.stop()
    server = lib.Server(slots=1)
    server.stop()


def test_budget_admission_makes_stacks_wait(lib, orc, monkeypatch):
    """A budget below one stack's estimate admits one stack at a time: every later stack waits in the queue until the
    one before it has completed (all are submitted together)."""
    import synth
    monkeypatch.setenv("PTB_MLE_LANES", "1")
    cases = []
    for k in range(3):
        st, _ = synth.stack("c1", frames=40, seed=700 + k)
        cases.append((st, synth.mad_threshold(orc.planes(st[0])[1])))
    server = lib.Server(slots=3, budget_bytes=1)
    try:
        tickets = [server.submit(st, thr, 0.0, 6, MLE6) for st, thr in cases]
        res = [server.result(t) for t in tickets]
    finally:
        server.stop()
    for i in range(1, len(res)):
        (_, q_prev, lat_prev), (_, q, _) = res[i - 1], res[i]
        assert q >= 0.9 * lat_prev, (i, q, lat_prev)
    for (st, thr), (rows, _, _) in zip(cases, res):
        assert np.array_equal(rows, lib.localization(st, thr, 0.0, 6, MLE6))
