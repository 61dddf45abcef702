"""TIFF stack reader (PTB_TiffInfo / PTB_TiffRead; host-only, no GPU needed).

Pinned three ways: the reference's own test stacks decode to the golden arrays (when the reference tree is present;
the golden arrays were decoded from them with PIL by tests/golden/make_golden.py), files written by PIL decode to
PIL's own reading of them, and every layout of tests/tiffgen.py (classic and BigTIFF, both byte orders, one or many
rows per strip, scattered strips) decodes to the frames it was written from. The reference's loader
(Tests_CPU/TiffManagement.hpp:8-55) rejects pages that are not 16-bit or differ in size; so does this one, and it
also rejects what it cannot decode (compressed or tiled pages) and malformed files instead of reading past them.
"""
import os

import numpy as np
import pytest

import tiffgen

def _reference_input():
    from oracle.oracle import reference_root
    root = reference_root()
    return os.path.join(root, "Tests_CPU", "Input") if root else None


REF_INPUT = _reference_input()


@pytest.fixture(scope="module")
def ptbmod():
    import ptb
    return ptb


def _frames(seed, n=4, h=37, w=53):
    rng = np.random.default_rng(seed)
    return [rng.integers(0, 65536, (h, w), dtype=np.uint16) for _ in range(n)]


@pytest.mark.parametrize("name", ["stack", "stack_quadrant"])
def test_reference_stacks_decode_to_golden(ptbmod, name):
    if REF_INPUT is None or not os.path.exists(os.path.join(REF_INPUT, name + ".tif")):
        pytest.skip("reference test inputs not present (set PTB_REFERENCE_ROOT)")
    path = os.path.join(REF_INPUT, name + ".tif")
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "stacks.npz"))[name]
    assert ptbmod.tiff_info(path) == (golden.shape[2], golden.shape[1], golden.shape[0])
    assert np.array_equal(ptbmod.tiff_read(path), golden)
    assert np.array_equal(ptbmod.tiff_read(path, 3, 4), golden[3:7])


@pytest.mark.parametrize("big_endian", [False, True])
@pytest.mark.parametrize("bigtiff", [False, True])
@pytest.mark.parametrize("rows_per_strip,scatter", [(None, False), (1, False), (7, True), (16, False)])
def test_layouts_round_trip(ptbmod, tmp_path, big_endian, bigtiff, rows_per_strip, scatter):
    frames = _frames(3)
    path = str(tmp_path / "s.tif")
    tiffgen.write(path, frames, big_endian=big_endian, bigtiff=bigtiff, rows_per_strip=rows_per_strip, scatter=scatter)
    assert ptbmod.tiff_info(path) == (53, 37, 4)
    assert np.array_equal(ptbmod.tiff_read(path), np.stack(frames))
    assert np.array_equal(ptbmod.tiff_read(path, 1, 2), np.stack(frames[1:3]))
    assert ptbmod.tiff_read(path, 4, 0).shape == (0, 37, 53)


def test_missing_strip_byte_counts(ptbmod, tmp_path):
    frames = _frames(4, n=2)
    path = str(tmp_path / "s.tif")
    tiffgen.write(path, frames, rows_per_strip=5, omit_counts=True)
    assert np.array_equal(ptbmod.tiff_read(path), np.stack(frames))


def test_pil_written_stack(ptbmod, tmp_path):
    from PIL import Image
    frames = _frames(5, n=3, h=64, w=40)
    path = str(tmp_path / "pil.tif")
    imgs = [Image.fromarray(f) for f in frames]
    imgs[0].save(path, save_all=True, append_images=imgs[1:])
    im = Image.open(path)
    pil = []
    for i in range(im.n_frames):
        im.seek(i)
        pil.append(np.array(im, dtype=np.uint16))
    got = ptbmod.tiff_read(path)
    assert np.array_equal(got, np.stack(pil)) and np.array_equal(got, np.stack(frames))


def test_large_stack_multithreaded_read(ptbmod, tmp_path):
    # > 8 MiB so that the read is split over threads; big-endian so every piece is byte-swapped
    rng = np.random.default_rng(6)
    frames = [rng.integers(0, 65536, (512, 512), dtype=np.uint16) for _ in range(40)]
    path = str(tmp_path / "big.tif")
    tiffgen.write(path, frames, big_endian=True)
    assert np.array_equal(ptbmod.tiff_read(path), np.stack(frames))


@pytest.mark.parametrize("case,message", [
    ("bits8", "16 bits"),
    ("mismatch", "same dimensions"),
    ("lzw", "compressed"),
    ("loop", "loops"),
    ("truncated", "outside the file"),
    ("not_tiff", "not a TIFF"),
    ("missing", "cannot open"),
])
def test_rejected_files(ptbmod, tmp_path, case, message):
    path = str(tmp_path / "bad.tif")
    frames = _frames(7, n=3)
    if case == "bits8":
        tiffgen.write(path, [f.astype(np.uint8) for f in frames], bits=8)
    elif case == "mismatch":
        tiffgen.write(path, frames[:2] + [np.zeros((10, 10), np.uint16)])
    elif case == "lzw":
        tiffgen.write(path, frames, compression=5)
    elif case == "loop":
        tiffgen.write(path, frames, loop=True)
    elif case == "truncated":
        size = tiffgen.write(path, frames, rows_per_strip=4)
        os.truncate(path, size - 40)  # the last page's directory (written after the pixels) now runs past the end
    elif case == "not_tiff":
        with open(path, "wb") as fh:
            fh.write(b"PK\x03\x04" + b"\0" * 64)
    elif case == "missing":
        path = str(tmp_path / "does_not_exist.tif")
    with pytest.raises(RuntimeError, match=message):
        ptbmod.tiff_read(path)


def test_page_range_outside_stack(ptbmod, tmp_path):
    path = str(tmp_path / "s.tif")
    tiffgen.write(path, _frames(8, n=3))
    out = np.empty((2, 37, 53), np.uint16)
    assert ptbmod.load().PTB_TiffRead(os.fsencode(path), out.ctypes.data_as(ptbmod._u16p), 2, 2) == 0
    assert "outside the stack" in ptbmod.last_error()
