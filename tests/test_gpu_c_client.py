"""The C ABI from C: tests/c_client/nand_client.c, built with gcc against include/hb_gpu.h and
linked to libhb_gpu.so, generates the BABYBEAR and GOLDILOCKS keys on the device from seed 0,
bootstraps the golden NAND inputs through hb_gate and decrypts them, as the reference's
nand_* examples do (tfhe/examples/nand_babybear.rs); every output word must equal the golden
oracle output and the bits the NAND truth table."""

import os
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_seed0.npz")


@pytest.fixture(scope="module")
def client(hb):
    from hasteboots_b200 import build
    d = tempfile.mkdtemp()
    exe = os.path.join(d, "nand_client")
    libdir = os.path.dirname(build.OUT)
    subprocess.run(["gcc", "-O2", "-std=c11", "-Wall", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_client", "nand_client.c"), "-o", exe,
                    "-L", libdir, "-lhb_gpu", "-Wl,-rpath," + libdir], check=True)
    return exe


@pytest.mark.parametrize("pid", [0, 1])
def test_c_client_nand_matches_golden(client, oracle, pid):
    g = np.load(GOLDEN)
    name = oracle.PRESET_NAMES[pid]
    c0, c1 = g[f"{name}/c0"], g[f"{name}/c1"]
    d = tempfile.mkdtemp()
    paths = [os.path.join(d, f) for f in ("c0", "c1", "out")]
    c0.astype(c0.dtype.newbyteorder("<")).tofile(paths[0])
    c1.astype(c1.dtype.newbyteorder("<")).tofile(paths[1])
    r = subprocess.run([client, str(pid), str(len(c0)), *paths], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(paths[2], dtype=c0.dtype).reshape(c0.shape)
    assert (out == g[f"{name}/nand"]).all()
    assert r.stdout.strip() == "1110"
