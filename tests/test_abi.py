"""The C-ABI library loads and exports every function include/hb_gpu.h declares (no GPU needed)."""

import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "hb_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert "hb_gate_device" in names and "hb_external_product_device" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(hb):
    from hasteboots_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == declared()
