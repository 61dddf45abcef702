"""Writes multi-page TIFF files for the TIFF reader's tests: classic or BigTIFF, either byte order, any rows per
strip, strips stored in file order or scattered, 8-bit pages, a compression tag, a looping IFD chain.

Test infrastructure only. Layout follows the TIFF 6.0 specification (header, IFD entries sorted by tag, values
inline when they fit) and the BigTIFF extension (version 43, 8-byte offsets, 20-byte entries).
"""
import struct

import numpy as np

SHORT, LONG, LONG8 = 3, 4, 16


def write(path, frames, big_endian=False, bigtiff=False, rows_per_strip=None, scatter=False, bits=16, loop=False,
          compression=1, omit_counts=False):
    """frames: list of 2-D uint16 (or uint8 with bits=8) arrays; returns the file size."""
    bo = ">" if big_endian else "<"
    off_fmt, off_size = ("Q", 8) if bigtiff else ("I", 4)
    dtype = np.dtype(bo + ("u2" if bits == 16 else "u1"))
    blob = bytearray()
    header_size = 16 if bigtiff else 8
    blob += b"MM" if big_endian else b"II"
    if bigtiff:
        blob += struct.pack(bo + "HHHQ", 43, 8, 0, 0)
    else:
        blob += struct.pack(bo + "HI", 42, 0)
    assert len(blob) == header_size
    # pixel data first (strips), then the IFDs
    strip_tables = []
    for f in frames:
        h, w = f.shape
        rps = rows_per_strip or h
        pieces = [np.ascontiguousarray(f[r:r + rps]).astype(dtype).tobytes() for r in range(0, h, rps)]
        order = list(range(len(pieces)))
        if scatter:
            order = order[::-1]
        offsets = [0] * len(pieces)
        for i in order:
            if len(blob) % 2:
                blob += b"\0"
            offsets[i] = len(blob)
            blob += pieces[i]
            if scatter:
                blob += b"\xab" * 6  # gap between strips
        strip_tables.append((offsets, [len(p) for p in pieces], rps))
    ifd_offsets = []
    for k, f in enumerate(frames):
        h, w = f.shape
        offsets, counts, rps = strip_tables[k]
        entries = [(256, LONG, [w]), (257, LONG, [h]), (258, SHORT, [bits]), (259, SHORT, [compression]),
                   (262, SHORT, [1]), (273, LONG8 if bigtiff else LONG, offsets), (277, SHORT, [1]), (278, LONG, [rps])]
        if not omit_counts:
            entries.append((279, LONG8 if bigtiff else LONG, counts))
        entries.sort()
        if len(blob) % 2:
            blob += b"\0"
        # out-of-line values first
        fixed = []
        for tag, typ, vals in entries:
            fmt = bo + {SHORT: "H", LONG: "I", LONG8: "Q"}[typ] * len(vals)
            raw = struct.pack(fmt, *vals)
            if len(raw) <= off_size:
                fixed.append((tag, typ, len(vals), raw.ljust(off_size, b"\0")))
            else:
                if len(blob) % 2:
                    blob += b"\0"
                pos = len(blob)
                blob += raw
                fixed.append((tag, typ, len(vals), struct.pack(bo + off_fmt, pos)))
        if len(blob) % 2:
            blob += b"\0"
        ifd_offsets.append(len(blob))
        blob += struct.pack(bo + ("Q" if bigtiff else "H"), len(fixed))
        for tag, typ, n, raw in fixed:
            blob += struct.pack(bo + "HH" + ("Q" if bigtiff else "I"), tag, typ, n) + raw
        blob += struct.pack(bo + off_fmt, 0)  # next IFD, patched below
    # chain the IFDs (the last one points back to the first when loop is set)
    for k, pos in enumerate(ifd_offsets):
        n = struct.unpack_from(bo + ("Q" if bigtiff else "H"), blob, pos)[0]
        nxt = pos + (8 if bigtiff else 2) + n * (20 if bigtiff else 12)
        target = ifd_offsets[k + 1] if k + 1 < len(ifd_offsets) else (ifd_offsets[0] if loop else 0)
        struct.pack_into(bo + off_fmt, blob, nxt, target)
    struct.pack_into(bo + off_fmt, blob, 8 if bigtiff else 4, ifd_offsets[0])
    with open(path, "wb") as fh:
        fh.write(bytes(blob))
    return len(blob)
