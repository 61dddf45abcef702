"""Serving (PTB_ServerStart / PTB_SubmitStack / PTB_StackResult): every stack's result is the same when it runs in a
mix of concurrent stacks of other shapes, lengths and fit modes as when it runs alone, and equals Localization's.

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


def test_served_mix_equals_alone(lib, orc, monkeypatch):
    monkeypatch.setenv("PTB_MLE_LANES", "1")
    cases = _mix(orc)
    alone = [lib.localization(s, thr, 0.0, fit, p) for s, thr, fit, p in cases]
    server = lib.Server(slots=4, budget_bytes=8 << 30)
    try:
        # all at once: the stacks overlap on the device
        tickets = [server.submit(s, thr, 0.0, fit, p) for s, thr, fit, p in cases]
        mixed = [server.result(t) for t in tickets]
        # one at a time through the server
        served_alone = []
        for s, thr, fit, p in cases:
            served_alone.append(server.result(server.submit(s, thr, 0.0, fit, p)))
    finally:
        server.stop()
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
