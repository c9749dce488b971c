"""The C ABI library loads and exports every function include/*.h declares (no device needed)."""
import ctypes
import glob
import os
import re

from photonoxide_b200.fdtd import LIB_PATH

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for path in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(path).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b((?:fdtd|pxs)_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_function():
    lib = ctypes.CDLL(LIB_PATH)
    names = declared()
    assert len(names) > 30
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
