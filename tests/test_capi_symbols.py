"""The C-ABI library loads and exports every symbol include/*.h declares (no GPU calls)."""
import glob
import os
import re

import pytest

from ugks2d_high_order_b200 import build as ub
from ugks2d_high_order_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(hdr).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(ugks_[a-z0-9_]+)\s*\(", text):
            syms.add(m.group(1))
    return sorted(syms)


def test_library_builds_and_exports_every_declared_symbol():
    lib_path = ub.build()
    import ctypes
    L = ctypes.CDLL(lib_path)
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), f"{s} declared in include/ but not exported"
    assert set(capi.EXPORTS) <= set(syms)
