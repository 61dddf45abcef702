"""Chunked processing: a stack split into many chunks (small device-memory budget) gives the same rows as one chunk.

With host buffers the library copies chunk k + 1 in and the rows of chunk k - 1 out while chunk k computes, using three
device staging slots for the frames and two chunk slots (stream, workspace) for the compute, and numbers rows across
chunks with a device-side count. A budget of a few MB forces one to three frames per chunk, so every slot is reused
several times; the rows (Id numbering included) must be bit-identical to a run that holds the whole stack in one
chunk, through both the host-buffer and the device-buffer entry points. PTB_CHUNK_SLOTS=1 runs the chunks on one
chunk slot, one after the other.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GAUSS_PARAMS

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MLE6 = np.array([7.0, 1.3, 100.0, 2.0, 20, 0.0])

CHILD = r"""
import os, sys
import numpy as np
sys.path[:0] = [os.path.join(sys.argv[1], "palmtracer-cpp_b200"), os.path.join(sys.argv[1], "tests")]
import torch, ptb, synth
data = np.load(sys.argv[2])
out = {}
for key in ("g", "m"):
    s, thr, fit, params = data["stack"], float(data["thr"]), int(data["fit_" + key]), data["params_" + key]
    out["host_" + key] = ptb.localization(s, thr, 0.0, fit, params)
    z, h, w = s.shape
    cap = ((h * w) // 5 + 1) * z * 18
    d_in = torch.from_numpy(np.ascontiguousarray(s).view(np.int16)).cuda()
    d_out = torch.full((cap,), -7.0, dtype=torch.float64, device="cuda")
    n = ptb.localization_device(d_in.data_ptr(), d_out.data_ptr(), cap, s.shape, thr, 0.0, fit, params,
                                torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    out["dev_" + key] = d_out[:n].cpu().numpy().reshape(-1, 18)
np.savez(sys.argv[3], **out)
"""


def _one_chunk(lib, s, thr, fit, params):
    return lib.localization(s, thr, 0.0, fit, params)


# 8 MB: 1 frame per chunk; 30 MB: 3 per chunk, the first split and the end shrinking (1, 2, 3, 2, 1)
@pytest.mark.parametrize("budget_mb,slots", [("8", "2"), ("30", "2"), ("8", "1"), ("30", "1")])
def test_many_chunks_match_one_chunk(lib, orc, tmp_path, monkeypatch, budget_mb, slots):
    import synth
    monkeypatch.setenv("PTB_MLE_LANES", "1")
    s, _ = synth.stack("c1", frames=9, seed=77)
    thr = synth.mad_threshold(orc.planes(s[0])[1])
    ref_g = _one_chunk(lib, s, thr, 2, GAUSS_PARAMS)
    ref_m = _one_chunk(lib, s, thr, 6, MLE6)
    assert ref_g.shape[0] > 100 and ref_m.shape[0] > 100
    inp = tmp_path / "in.npz"
    outp = tmp_path / "out.npz"
    np.savez(inp, stack=s, thr=thr, fit_g=2, params_g=GAUSS_PARAMS, fit_m=6, params_m=MLE6)
    env = dict(os.environ, PTB_WORKSPACE_MB=budget_mb, PTB_MLE_LANES="1", PTB_CHUNK_SLOTS=slots)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(inp), str(outp)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got = np.load(outp)
    for key, ref in (("g", ref_g), ("m", ref_m)):
        for via in ("host", "dev"):
            a = got[via + "_" + key]
            assert a.shape == ref.shape, (via, key, a.shape, ref.shape)
            assert np.array_equal(a, ref), (via, key, float(np.max(np.abs(a - ref))))
            assert np.array_equal(a[:, 0], np.arange(1, a.shape[0] + 1))  # Ids run on across chunks
