"""ctypes binding of the CPU oracle (oracle/libhb_oracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg and reference arm
(--impl reference) use this module; tests and smoke() use it as the checker. It restates the reference's TFHE gate-bootstrapping path on the CPU; see hb_oracle.h for
the reference files it follows and its parity status.
"""

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhb_oracle.so")

FIELD_BABYBEAR = 0
FIELD_GOLDILOCKS = 1
FIELD_DEFAULT_U32 = 2

PRESET_BABYBEAR = 0
PRESET_GOLDILOCKS = 1
PRESET_ZAMA = 2
PRESET_DEFAULT_TERNARY = 3
PRESET_CUSTOM_TERNARY = 4
PRESET_NAMES = {
    PRESET_BABYBEAR: "BABYBEAR_BINARY_128_BITS",
    PRESET_GOLDILOCKS: "GOLDILOCKS_BINARY_128_BITS",
    PRESET_ZAMA: "ZAMA_BINARY_128_BITS",
    PRESET_DEFAULT_TERNARY: "DEFAULT_TERNARY_128_BITS",
    PRESET_CUSTOM_TERNARY: "CUSTOM_TERNARY_128_BITS",
}

# Key sets the tests use: the presets, plus CUSTOM_TERNARY_128_BITS with a ternary LWE key (no
# reference preset configures one; TernaryBlindRotationKey,
# fhe_core/src/blind_rotation/rlwe/ternary.rs, serves it).
SET_TERNARY_LWE = 100
SET_NAMES = dict(PRESET_NAMES)
SET_NAMES[SET_TERNARY_LWE] = "CUSTOM_TERNARY_128_BITS_TERNARY_LWE_KEY"
# Sets with n' = next_pow2(n) < N on the other two fields (key switching in N/n' chunks).
SET_GOLDILOCKS_N500 = 101
SET_BABYBEAR_N300 = 102

GATES = {"nand": 0, "and": 1, "or": 2, "nor": 3, "xor": 4, "xnor": 5, "majority": 6,
         "not": 7, "mux": 8}

MODULUS = {FIELD_BABYBEAR: 0x78000001, FIELD_GOLDILOCKS: 0xFFFFFFFF00000001,
           FIELD_DEFAULT_U32: 132120577}


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("field_id", ctypes.c_int32),
        ("ring_dim", ctypes.c_uint32),
        ("lwe_dim", ctypes.c_uint32),
        ("br_bits", ctypes.c_uint32),
        ("br_len", ctypes.c_uint32),
        ("ks_bits", ctypes.c_uint32),
        ("ks_len", ctypes.c_uint32),
        ("ring_ternary", ctypes.c_uint32),
        ("lwe_ternary", ctypes.c_uint32),
        ("lwe_noise_std", ctypes.c_double),
        ("ring_noise_std", ctypes.c_double),
        ("ks_noise_std", ctypes.c_double),
    ]


def build():
    """Compile the oracle library with its Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None
_lib_path = LIB_PATH


def use_native_build():
    """Before the first lib() call: build the oracle for this host's CPU (-march=native, `make
    native`) and load that build. Returns a description of the build used; falls back to the
    portable library when the native build fails."""
    global _lib_path
    if _lib is not None:
        return "portable (loaded before the native build was requested)"
    try:
        subprocess.run(["make", "-s", "-C", HERE, "native"], check=True, capture_output=True, timeout=600)
        _lib_path = os.path.join(HERE, "libhb_oracle_native.so")
        return "-O3 -march=native, built on this host"
    except (OSError, subprocess.SubprocessError):
        return "-O3 portable (the native build failed)"


def lib():
    global _lib
    if _lib is None:
        if _lib_path == LIB_PATH and not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(_lib_path)
        vp, sz, u64, i32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int
        P = ctypes.POINTER(OrcParams)
        L.orc_params_preset.argtypes = [i32, P]
        L.orc_prg.restype = u64
        L.orc_prg.argtypes = [u64, u64, u64]
        L.orc_keygen.argtypes = [P, u64, vp, vp, vp, vp, i32]
        L.orc_encrypt.argtypes = [P, vp, u64, u64, vp, sz, vp]
        L.orc_decrypt.argtypes = [P, vp, vp, sz, vp, vp]
        L.orc_gate.argtypes = [P, vp, vp, i32, vp, vp, vp, vp, sz, i32]
        L.orc_eval_create.argtypes = [P, vp, vp, i32, ctypes.POINTER(vp)]
        L.orc_eval_free.argtypes = [vp]
        L.orc_eval_free.restype = None
        L.orc_eval_gate.argtypes = [vp, i32, vp, vp, vp, vp, sz, i32]
        L.orc_bootstrap_lut.argtypes = [P, vp, vp, vp, vp, vp, sz, i32]
        L.orc_modswitch.argtypes = [P, vp, vp]
        L.orc_blind_rotate.argtypes = [P, vp, vp, vp, ctypes.c_uint32, vp]
        L.orc_blind_rotate_trace.argtypes = [P, vp, vp, vp, vp, vp]
        L.orc_ntt_roundtrip.argtypes = [i32, ctypes.c_uint32, vp, vp]
        L.orc_negacyclic_mul.argtypes = [i32, ctypes.c_uint32, vp, vp, vp, i32]
        L.orc_external_product.argtypes = [i32, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.c_uint32, vp, vp, vp, sz, i32]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _check(rc, what):
    if rc != 0:
        raise ValueError(f"oracle {what} failed with status {rc}")


def dtype_of(field_id):
    return np.uint64 if field_id == FIELD_GOLDILOCKS else np.uint32


def preset(pid):
    p = OrcParams()
    _check(lib().orc_params_preset(pid, ctypes.byref(p)), "params_preset")
    return p


def params(set_id):
    """Parameters of a key set (SET_NAMES)."""
    if set_id == SET_TERNARY_LWE:
        p = preset(PRESET_CUSTOM_TERNARY)
        p.lwe_ternary = 1
        return p
    if set_id in (SET_GOLDILOCKS_N500, SET_BABYBEAR_N300):
        p = preset(PRESET_GOLDILOCKS if set_id == SET_GOLDILOCKS_N500 else PRESET_BABYBEAR)
        p.lwe_dim = 500 if set_id == SET_GOLDILOCKS_N500 else 300
        return p
    return preset(set_id)


def sizes(p):
    N, n, L, Lks = p.ring_dim, p.lwe_dim, p.br_len, p.ks_len
    pairs = 2 if p.lwe_ternary else 1
    return {"lwe_sk": n, "ring_sk": N, "bsk": n * pairs * 2 * L * 2 * N, "ksk": Lks * 2 * N,
            "lwe": n + 1}


class Keys:
    def __init__(self, p, lwe_sk, ring_sk, bsk, ksk):
        self.p, self.lwe_sk, self.ring_sk, self.bsk, self.ksk = p, lwe_sk, ring_sk, bsk, ksk
        self._eval = None

    def evaluator(self, threads=None):
        """Evaluator::new: the keys transformed once (orc_eval_create), reused by every gate."""
        if self._eval is None:
            h = ctypes.c_void_p()
            _check(lib().orc_eval_create(ctypes.byref(self.p), _ptr(self.bsk), _ptr(self.ksk),
                                         threads or os.cpu_count(), ctypes.byref(h)), "eval_create")
            self._eval = h
        return self._eval

    def __del__(self):
        if getattr(self, "_eval", None) is not None and _lib is not None:
            _lib.orc_eval_free(self._eval)
            self._eval = None


def keygen(p, seed, threads=None):
    dt = dtype_of(p.field_id)
    s = sizes(p)
    lwe_sk = np.zeros(s["lwe_sk"], dt)
    ring_sk = np.zeros(s["ring_sk"], dt)
    bsk = np.zeros(s["bsk"], dt)
    ksk = np.zeros(s["ksk"], dt)
    _check(lib().orc_keygen(ctypes.byref(p), seed, _ptr(lwe_sk), _ptr(ring_sk), _ptr(bsk),
                            _ptr(ksk), threads or os.cpu_count()), "keygen")
    return Keys(p, lwe_sk, ring_sk, bsk, ksk)


def encrypt(p, lwe_sk, seed, index0, bits):
    bits = np.ascontiguousarray(bits, dtype=np.uint8)
    out = np.zeros((len(bits), p.lwe_dim + 1), dtype_of(p.field_id))
    _check(lib().orc_encrypt(ctypes.byref(p), _ptr(lwe_sk), seed, index0, _ptr(bits), len(bits),
                             _ptr(out)), "encrypt")
    return out


def decrypt(p, lwe_sk, cts):
    cts = np.ascontiguousarray(cts, dtype=dtype_of(p.field_id)).reshape(-1, p.lwe_dim + 1)
    bits = np.zeros(len(cts), np.uint8)
    noise = np.zeros(len(cts), np.uint64)
    _check(lib().orc_decrypt(ctypes.byref(p), _ptr(lwe_sk), _ptr(cts), len(cts), _ptr(bits),
                             _ptr(noise)), "decrypt")
    return bits, noise


def gate(keys, name, c0, c1=None, c2=None, threads=None):
    p = keys.p
    dt = dtype_of(p.field_id)
    c0 = np.ascontiguousarray(c0, dtype=dt).reshape(-1, p.lwe_dim + 1)
    c1 = None if c1 is None else np.ascontiguousarray(c1, dtype=dt).reshape(-1, p.lwe_dim + 1)
    c2 = None if c2 is None else np.ascontiguousarray(c2, dtype=dt).reshape(-1, p.lwe_dim + 1)
    out = np.zeros_like(c0)
    _check(lib().orc_eval_gate(keys.evaluator(threads), GATES[name], _ptr(c0), _ptr(c1), _ptr(c2),
                               _ptr(out), len(c0), threads or os.cpu_count()), "gate")
    return out


def bootstrap_lut(keys, c, lut, threads=None):
    p = keys.p
    dt = dtype_of(p.field_id)
    c = np.ascontiguousarray(c, dtype=dt).reshape(-1, p.lwe_dim + 1)
    lut = np.ascontiguousarray(lut, dtype=dt)
    out = np.zeros_like(c)
    _check(lib().orc_bootstrap_lut(ctypes.byref(p), _ptr(keys.bsk), _ptr(keys.ksk), _ptr(c),
                                   _ptr(lut), _ptr(out), len(c), threads or os.cpu_count()),
           "bootstrap_lut")
    return out


def modswitch(p, c):
    c = np.ascontiguousarray(c, dtype=dtype_of(p.field_id))
    out = np.zeros(p.lwe_dim + 1, np.uint32)
    _check(lib().orc_modswitch(ctypes.byref(p), _ptr(c), _ptr(out)), "modswitch")
    return out


def blind_rotate(keys, c, lut, steps):
    p = keys.p
    dt = dtype_of(p.field_id)
    c = np.ascontiguousarray(c, dtype=dt)
    lut = np.ascontiguousarray(lut, dtype=dt)
    out = np.zeros(2 * p.ring_dim, dt)
    _check(lib().orc_blind_rotate(ctypes.byref(p), _ptr(keys.bsk), _ptr(c), _ptr(lut), steps,
                                  _ptr(out)), "blind_rotate")
    return out


def blind_rotate_trace(keys, c, lut, digits=False):
    """The accumulator after every blind-rotation step: [n, 2N] (a then b, canonical); with
    digits=True also every step's gadget digits of E.a then E.b, [n, 2, l, N] uint8."""
    p = keys.p
    dt = dtype_of(p.field_id)
    c = np.ascontiguousarray(c, dtype=dt)
    lut = np.ascontiguousarray(lut, dtype=dt)
    out = np.zeros((p.lwe_dim, 2 * p.ring_dim), dt)
    dig = np.zeros((p.lwe_dim, 2, p.br_len, p.ring_dim), np.uint8) if digits else None
    _check(lib().orc_blind_rotate_trace(ctypes.byref(p), _ptr(keys.bsk), _ptr(c), _ptr(lut),
                                        _ptr(out), _ptr(dig)), "blind_rotate_trace")
    return (out, dig) if digits else out


def ntt_roundtrip(field_id, log_n, x):
    x = np.ascontiguousarray(x, dtype=dtype_of(field_id))
    out = np.zeros_like(x)
    _check(lib().orc_ntt_roundtrip(field_id, log_n, _ptr(x), _ptr(out)), "ntt_roundtrip")
    return out


def negacyclic_mul(field_id, log_n, x, y, schoolbook=False):
    dt = dtype_of(field_id)
    x = np.ascontiguousarray(x, dtype=dt)
    y = np.ascontiguousarray(y, dtype=dt)
    out = np.zeros_like(x)
    _check(lib().orc_negacyclic_mul(field_id, log_n, _ptr(x), _ptr(y), _ptr(out),
                                    1 if schoolbook else 0), "negacyclic_mul")
    return out


def external_product(field_id, log_n, bits, length, rlwe, rgsw, threads=None):
    dt = dtype_of(field_id)
    rlwe = np.ascontiguousarray(rlwe, dtype=dt)
    rgsw = np.ascontiguousarray(rgsw, dtype=dt)
    n = 1 << log_n
    count = rlwe.size // (2 * n)
    out = np.zeros_like(rlwe)
    _check(lib().orc_external_product(field_id, log_n, bits, length, _ptr(rlwe), _ptr(rgsw),
                                      _ptr(out), count, threads or os.cpu_count()),
           "external_product")
    return out


def lut_poly(field_id, name, N):
    """LUT polynomial of a gate (tfhe/src/bfhe/evaluate.rs:267-465), lut_step 1."""
    q = MODULUS[field_id]
    q8, nq8 = q >> 3, q - (q >> 3)
    table = {
        "nand": (3 * N // 4, q8, nq8), "and": (3 * N // 4, nq8, q8),
        "majority": (3 * N // 4, nq8, q8), "or": (N // 4, nq8, q8), "mux": (N // 4, nq8, q8),
        "nor": (N // 4, q8, nq8), "xor": (N // 2, nq8, q8), "xnor": (N // 2, q8, nq8),
    }
    mid, lo, hi = table[name]
    out = np.full(N, hi, dtype_of(field_id))
    out[:mid] = lo
    return out
