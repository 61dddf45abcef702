"""The C-ABI library loads without a GPU and exports every symbol include/palmtracer_b200.h declares."""
import ctypes
import os
import re
import subprocess

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "palmtracer_b200.h")


def declared():
    text = open(HEADER).read()
    return re.findall(r"PTB_API\s+[\w\s\*]+?\b(\w+)\s*\(", text)


def test_header_declares_reference_exports():
    names = declared()
    for n in ("Localization", "Fitting", "Wavelett", "AutoThreshold", "Astigmatism3DEstimation"):
        assert n in names


def test_library_exports_every_declared_symbol():
    import ptb
    lib = ptb.load()
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", ptb.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(declared()) <= exported
    assert set(ptb.EXPORTS) == set(declared())

