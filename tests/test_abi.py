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


def test_every_entry_point_refuses_null_arguments(hb):
    """Each function, called with null handles and pointers and zero scalars, returns HB_ERR_INVALID
    (or, where it returns no status, does nothing) without touching a device."""
    from hasteboots_b200 import _lib
    L = _lib.lib()
    for name in declared():
        fn = getattr(L, name)
        args = []
        for t in fn.argtypes:
            if t in (ctypes.c_double, ctypes.c_float):
                args.append(0.0)
            elif t in (ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t,
                       ctypes.c_longlong):
                args.append(0)
            else:
                args.append(None)
        rc = fn(*args)
        if fn.restype is None:
            assert rc is None, name
        elif fn.restype in (ctypes.c_size_t, ctypes.c_uint64):
            assert rc == 0, name
        else:
            assert _lib.ERRORS.get(rc) == "HB_ERR_INVALID", (name, rc)


def test_c_client_compiles_and_links():
    """A C caller builds against include/hb_gpu.h and links libhb_gpu.so (tests/c_client; run by
    tests/test_gpu_c_client.py on a GPU)."""
    import subprocess
    import tempfile
    from hasteboots_b200 import build
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(tempfile.mkdtemp(), "nand_client")
    libdir = os.path.dirname(build.OUT)
    subprocess.run(["gcc", "-O2", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "c_client", "nand_client.c"), "-o", exe,
                    "-L", libdir, "-lhb_gpu", "-Wl,-rpath," + libdir], check=True)
    assert os.path.exists(exe)
