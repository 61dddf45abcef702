"""Launch-chain graphs: a chunk whose launch chain recurs is captured into a CUDA graph on its second occurrence and
replayed after that; the rows are bit-identical to direct launches (PTB_GRAPHS=0).

Covers the per-frame form (one-frame host calls repeated, as a front end that calls Localization frame by frame
makes them), a multi-chunk stack on two chunk slots through the device entry point, and every fit family.
The fit mapping is pinned (PTB_MLE_LANES=1) so that no autotuning chunk is launched directly.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GAUSS_PARAMS

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, os, sys
import numpy as np
sys.path[:0] = [os.path.join(sys.argv[1], "palmtracer-cpp_b200"), os.path.join(sys.argv[1], "tests")]
import torch, ptb
data = np.load(sys.argv[2])
out, stats = {}, {}
ptb.graph_stats()
for key in ("g", "m", "a"):
    s, thr, fit, params = data["stack"], float(data["thr"]), int(data["fit_" + key]), data["params_" + key]
    # per-frame form: the same frame four times, then the next frames
    rows = [ptb.localization(s[i % 2:i % 2 + 1], thr, 0.0, fit, params) for i in range(6)]
    for i, r in enumerate(rows):
        out["frame_%s_%d" % (key, i)] = r
    stats["frame_" + key] = ptb.graph_stats()
# multi-chunk stack through the device entry point, three times
s, thr = data["stack"], float(data["thr"])
z, h, w = s.shape
cap = ((h * w) // 5 + 1) * z * 18
d_in = torch.from_numpy(np.ascontiguousarray(s).view(np.int16)).cuda()
for rep in range(3):
    d_out = torch.full((cap,), -7.0, dtype=torch.float64, device="cuda")
    n = ptb.localization_device(d_in.data_ptr(), d_out.data_ptr(), cap, s.shape, thr, 0.0, 6, data["params_m"],
                                torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    out["stack_%d" % rep] = d_out[:n].cpu().numpy().reshape(-1, 18)
stats["stack"] = ptb.graph_stats()
np.savez(sys.argv[3], **out)
with open(sys.argv[3] + ".json", "w") as f:
    json.dump(stats, f)
"""


def _run(tmp_path, inp, tag, graphs):
    outp = tmp_path / ("out_%s.npz" % tag)
    env = dict(os.environ, PTB_GRAPHS=graphs, PTB_MLE_LANES="1", PTB_WORKSPACE_MB="12")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(inp), str(outp)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    with open(str(outp) + ".json") as f:
        return np.load(outp), json.load(f)


def test_graph_replays_match_direct_launches(orc, tmp_path):
    import synth
    from test_gpu_serving import MLE6, MLE7
    s, _ = synth.stack("c1", frames=6, seed=91)
    thr = synth.mad_threshold(orc.planes(s[0])[1])
    inp = tmp_path / "in.npz"
    np.savez(inp, stack=s, thr=thr, fit_g=2, params_g=GAUSS_PARAMS, fit_m=6, params_m=MLE6, fit_a=7, params_a=MLE7)
    on, st_on = _run(tmp_path, inp, "on", "1")
    off, st_off = _run(tmp_path, inp, "off", "0")
    for key in on.files:
        assert on[key].shape == off[key].shape and np.array_equal(on[key], off[key]), key
    for key in ("g", "m", "a"):
        # frames 0 and 1 alternate in one staging buffer, so all six calls have one launch chain: direct on the first
        # call, captured on the second, replayed on the other four
        assert st_on["frame_" + key] == {"captured": 1, "replayed": 4, "direct": 1}, (key, st_on)
        assert st_off["frame_" + key] == {"captured": 0, "replayed": 0, "direct": 6}, (key, st_off)
        assert on["frame_%s_0" % key].shape[0] > 5
        for i in range(2, 6):
            assert np.array_equal(on["frame_%s_%d" % (key, i)], on["frame_%s_%d" % (key, i % 2)])
    # the stack spans several chunks on two slots; its third run replays every chunk
    n_chunks = st_on["stack"]["direct"]
    assert n_chunks >= 3 and st_on["stack"] == {"captured": n_chunks, "replayed": n_chunks, "direct": n_chunks}, st_on
    for rep in (1, 2):
        assert np.array_equal(on["stack_%d" % rep], on["stack_0"])
