"""Regenerates the golden fixtures in this folder from the reference's own test inputs.

Reads (text and TIFF only, nothing executed) from the reference tree:
  Tests_CPU/Input/stack.tif, Tests_CPU/Input/stack_quadrant.tif           -> stacks.npz
  Tests_CPU/Input/ref/stack-localizations-*.csv,
  Tests_CPU/Input/ref/stack_quadrant-localizations-*.csv                  -> localizations.npz
  Tests_CPU/Input/ref/stack-tracking-*-5.csv                              -> tracking.npz
  Tests_CPU/Input/Beads.tiff (a 29 x 29 x 61 crop around the bead at x 25, y 19 that the reference's spline
  calibration test lists first, Tests_CPU/test_sp_Spline.cpp:47-51; focus near plane 88) -> beads.npz
The AutoThreshold known answers come from Tests_CPU/test_Palm.cpp:307-310 and are stored beside them.

Usage: python tests/golden/make_golden.py REFERENCE_ROOT   (or set PTB_REFERENCE_ROOT)
"""
import glob
import os
import sys

import numpy as np
from PIL import Image

HERE = os.path.dirname(os.path.abspath(__file__))

# Tests_CPU/test_Palm.cpp:307-310 (per-plane AutoThreshold of stack.tif, roi 7, tolerance 1e-5)
AUTO_THRESHOLD = [63.651749, 66.142910, 63.192296, 64.368855, 63.954150,
                  63.400043, 66.521994, 63.373237, 62.613244, 63.866017]


def load_tiff_stack(path):
    img = Image.open(path)
    frames = []
    for i in range(img.n_frames):
        img.seek(i)
        frames.append(np.array(img, dtype=np.uint16))
    return np.stack(frames)


def load_csv(path):
    with open(path) as f:
        header = f.readline().strip().split(",")
    data = np.loadtxt(path, delimiter=",", skiprows=1, ndmin=2)
    return header, data


def main(ref_root):
    inp = os.path.join(ref_root, "Tests_CPU", "Input")
    stacks = {
        "stack": load_tiff_stack(os.path.join(inp, "stack.tif")),
        "stack_quadrant": load_tiff_stack(os.path.join(inp, "stack_quadrant.tif")),
    }
    np.savez_compressed(os.path.join(HERE, "stacks.npz"), **stacks,
                        auto_threshold=np.array(AUTO_THRESHOLD))
    locs = {}
    header = None
    for path in sorted(glob.glob(os.path.join(inp, "ref", "*localizations*.csv"))):
        header, data = load_csv(path)
        key = os.path.basename(path)[:-4]
        locs[key] = data
    locs["__header__"] = np.array(header)
    np.savez_compressed(os.path.join(HERE, "localizations.npz"), **locs)
    # Tracking known answers (Tests_CPU/test_tr_Tracks.cpp:250-268): Track, Plane, Id, ... of the localizations with
    # positive integrated intensity, linked with maxDistance 5
    tracks = {}
    for path in sorted(glob.glob(os.path.join(inp, "ref", "stack-tracking-*.csv"))):
        _, data = load_csv(path)
        tracks[os.path.basename(path)[:-4]] = data
    np.savez_compressed(os.path.join(HERE, "tracking.npz"), **tracks)
    beads = load_tiff_stack(os.path.join(inp, "Beads.tiff"))
    crop = beads[58:119, 19 - 14:19 + 15, 25 - 14:25 + 15]
    np.savez_compressed(os.path.join(HERE, "beads.npz"), bead=crop, origin=np.array([25 - 14, 19 - 14, 58]))
    print({k: v.shape for k, v in stacks.items()}, len(locs) - 1, "csv tables", "bead crop", crop.shape)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PTB_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set PTB_REFERENCE_ROOT)")
    main(root)
