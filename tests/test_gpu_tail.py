"""The MLE fits' tail hand-off leaves every row unchanged.

Once a warp of the thread-per-ROI LM or polish has an empty work queue and few busy lanes, it saves those ROIs'
state in their output rows and a resume launch finishes them (csrc/fit_mle.cu). Each ROI must then follow the same
FP32 operations as without the hand-off, so the rows must be bitwise equal with it on (the default) and off
(PTB_MLE_TAIL=0). The setting is read once per process, so each run is a child process; both force the
thread-per-ROI mapping (PTB_MLE_LANES=1), the one that hands off.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[2])
import ptb, synth
mode, out = int(sys.argv[3]), sys.argv[4]
params = {6: np.array([7.0, 1.3, 100.0, 2.0, 20.0, 0.0]),
          7: np.array([11.0, 160.0, 150.0, 400.0, 0.05, 0.0, 1.3 * 160, -150.0, 400.0, -0.05, 0.0, 1.3 * 160,
                       100.0, 2.0, 20, -600.0, 600.0, 0.0])}[mode]
s, _ = synth.stack("c2" if mode == 6 else "c3", frames=24, seed=77, size=(512, 512))
thr = float(sys.argv[5])
ptb.set_profiling(1)
ptb.mle_evaluations()
rows = ptb.localization(s, thr, 0.0, mode, params)
ev = ptb.mle_evaluations()
np.save(out, rows)
print(ev["lm_handoff"], ev["polish_handoff"])
"""


def _run(tmp_path, mode, thr, tail):
    out = str(tmp_path / ("rows_%d_%d.npy" % (mode, tail)))
    env = dict(os.environ, PTB_MLE_LANES="1", PTB_MLE_TAIL=str(tail))
    r = subprocess.run([sys.executable, "-c", CHILD, os.path.join(ROOT, "palmtracer-cpp_b200"), HERE, str(mode), out,
                        repr(thr)], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lm, polish = map(int, r.stdout.split()[-2:])
    return np.load(out), lm, polish


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [6, 7])
def test_tail_handoff_rows_bitwise(tmp_path, orc, mode):
    import synth
    s, _ = synth.stack("c2" if mode == 6 else "c3", frames=1, seed=77, size=(512, 512))
    thr = synth.mad_threshold(orc.planes(s[0])[1])
    with_tail, lm, polish = _run(tmp_path, mode, thr, 1)
    without, lm0, polish0 = _run(tmp_path, mode, thr, 0)
    print("mode", mode, "rows", len(with_tail), "handed off: LM", lm, "polish", polish)
    assert lm0 == 0 and polish0 == 0
    assert lm > 0 and polish > 0  # the hand-off ran in both kernels
    assert with_tail.shape == without.shape and len(with_tail) > 1000
    assert np.array_equal(with_tail.view(np.uint64), without.view(np.uint64))
