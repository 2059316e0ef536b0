"""ctypes binding of libhb_gpu.so (include/hb_gpu.h).

The library is the product: there is no CPU fallback for device entry points. Importing this module
without the built library raises immediately.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# HB_GPU_LIB selects another build of the same library (for example one with different build flags).
LIB_PATH = os.environ.get("HB_GPU_LIB") or os.path.join(HERE, "libhb_gpu.so")

HB_OK = 0
ERRORS = {-1: "HB_ERR_INVALID", -2: "HB_ERR_CUDA", -3: "HB_ERR_NOMEM", -4: "HB_ERR_TIMEOUT",
          -5: "HB_ERR_UNSUPPORTED", -6: "HB_ERR_BUSY"}

FIELD_BABYBEAR = 0
FIELD_GOLDILOCKS = 1
FIELD_DEFAULT_U32 = 2
MODULUS = {FIELD_BABYBEAR: 0x78000001, FIELD_GOLDILOCKS: 0xFFFFFFFF00000001,
           FIELD_DEFAULT_U32: 132120577}

EXPORTS = [
    "hb_params_preset", "hb_params_validate", "hb_params_sizes", "hb_keygen", "hb_encrypt",
    "hb_decrypt", "hb_ctx_create", "hb_ctx_destroy", "hb_last_error", "hb_ctx_stream",
    "hb_ctx_synchronize", "hb_ctx_hbm_in_use", "hb_keys_upload", "hb_keys_free", "hb_keys_params",
    "hb_gate", "hb_gate_device", "hb_gate_device_plain", "hb_bootstrap_lut", "hb_bootstrap_trace",
    "hb_bootstrap_trace_device",
    "hb_ntt_forward_device", "hb_ntt_inverse_device", "hb_ntt_roundtrip_device", "hb_rgsw_upload",
    "hb_rgsw_free", "hb_external_product_device", "hb_autotune", "hb_keys_set_config",
    "hb_keys_config", "hb_keys_set_rate", "hb_batch_create", "hb_batch_launch", "hb_batch_free",
    "hb_batch_info", "hb_serve_start", "hb_serve_submit", "hb_serve_poll", "hb_serve_next_done",
    "hb_serve_fetch", "hb_serve_stats", "hb_serve_stop", "hb_gate_mux_device_noalloc",
    "hb_probe_modmul", "hb_ctx_launches", "hb_ctx_set_wait_limit", "hb_ctx_test_withhold_keys",
    "hb_keys_generate", "hb_encrypt_device", "hb_keys_device_words", "hb_keys_download",
]


class HbParams(ctypes.Structure):
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


class HbJob(ctypes.Structure):
    _fields_ = [
        ("keys", ctypes.c_void_p),
        ("gate", ctypes.c_int32),
        ("count", ctypes.c_uint32),
        ("c0", ctypes.c_void_p),
        ("c1", ctypes.c_void_p),
        ("c2", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
    ]


class HbServeConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_size_t), ("max_wave_gates", ctypes.c_uint32),
                ("max_inflight_waves", ctypes.c_uint32), ("max_queue_s", ctypes.c_double)]


class HbServeStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("submitted", "admitted", "completed", "failed",
                                                "queued", "waves", "gates_completed")] + \
               [(n, ctypes.c_double) for n in ("p50_latency_s", "p99_latency_s", "mean_latency_s",
                                                "max_latency_s", "gates_per_s")] + \
               [("hbm_in_use", ctypes.c_size_t), ("hbm_peak", ctypes.c_size_t), ("rejected", ctypes.c_uint64)]


class HbError(RuntimeError):
    def __init__(self, code, what, detail=""):
        self.code = code
        super().__init__(f"{what} failed: {ERRORS.get(code, code)}" + (f": {detail}" if detail else ""))


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m hasteboots_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp, sz, u32, u64, i32 = (ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64,
                             ctypes.c_int)
    P = ctypes.POINTER(HbParams)
    pp = ctypes.POINTER(ctypes.c_void_p)
    sig = {
        "hb_params_preset": (i32, [i32, P]),
        "hb_params_validate": (i32, [P]),
        "hb_params_sizes": (i32, [P, ctypes.POINTER(sz)] + [ctypes.POINTER(sz)] * 4),
        "hb_keygen": (i32, [P, u64, vp, vp, vp, vp, i32]),
        "hb_encrypt": (i32, [P, vp, u64, u64, vp, sz, vp]),
        "hb_decrypt": (i32, [P, vp, vp, sz, vp, vp]),
        "hb_ctx_create": (i32, [i32, sz, pp]),
        "hb_ctx_destroy": (None, [vp]),
        "hb_last_error": (i32, [vp, ctypes.c_char_p, sz]),
        "hb_ctx_stream": (i32, [vp, pp]),
        "hb_ctx_synchronize": (i32, [vp]),
        "hb_ctx_hbm_in_use": (sz, [vp]),
        "hb_keys_upload": (i32, [vp, P, vp, vp, pp]),
        "hb_keys_free": (None, [vp, vp]),
        "hb_keys_params": (i32, [vp, P]),
        "hb_gate": (i32, [vp, vp, i32, vp, vp, vp, vp, sz]),
        "hb_gate_device": (i32, [vp, vp, i32, vp, vp, vp, vp, sz]),
        "hb_gate_device_plain": (i32, [vp, vp, i32, vp, vp, vp, sz]),
        "hb_bootstrap_lut": (i32, [vp, vp, vp, vp, vp, sz]),
        "hb_bootstrap_trace_device": (i32, [vp, vp, vp, vp, vp, sz, vp, vp]),
        "hb_bootstrap_trace": (i32, [vp, vp, vp, vp, vp, vp]),
        "hb_ntt_forward_device": (i32, [vp, i32, u32, vp, sz]),
        "hb_ntt_inverse_device": (i32, [vp, i32, u32, vp, sz]),
        "hb_ntt_roundtrip_device": (i32, [vp, i32, u32, vp, vp, sz]),
        "hb_rgsw_upload": (i32, [vp, i32, u32, u32, u32, vp, pp]),
        "hb_rgsw_free": (None, [vp, vp]),
        "hb_external_product_device": (i32, [vp, i32, u32, u32, u32, vp, vp, vp, sz]),
        "hb_autotune": (i32, [vp, vp, u32, ctypes.POINTER(i32), ctypes.POINTER(i32),
                              ctypes.POINTER(ctypes.c_double)]),
        "hb_keys_set_config": (i32, [vp, vp, i32, i32]),
        "hb_keys_config": (i32, [vp, ctypes.POINTER(i32), ctypes.POINTER(i32)]),
        "hb_batch_create": (i32, [vp, ctypes.POINTER(HbJob), sz, pp]),
        "hb_batch_launch": (i32, [vp, vp]),
        "hb_batch_free": (None, [vp, vp]),
        "hb_batch_info": (i32, [vp, ctypes.POINTER(u64), ctypes.POINTER(i32), ctypes.POINTER(i32), i32]),
        "hb_keys_set_rate": (i32, [vp, ctypes.c_double]),
        "hb_serve_start": (i32, [vp, ctypes.POINTER(HbServeConfig), pp]),
        "hb_serve_submit": (i32, [vp, vp, i32, vp, vp, vp, u32, ctypes.POINTER(u64)]),
        "hb_serve_poll": (i32, [vp, u64, ctypes.POINTER(i32)]),
        "hb_serve_next_done": (i32, [vp, ctypes.POINTER(u64), ctypes.c_double]),
        "hb_serve_fetch": (i32, [vp, u64, vp, ctypes.POINTER(ctypes.c_double)]),
        "hb_serve_stats": (i32, [vp, ctypes.POINTER(HbServeStats)]),
        "hb_serve_stop": (i32, [vp]),
        "hb_gate_mux_device_noalloc": (i32, [vp, vp, vp, vp, vp, vp, sz]),
        "hb_probe_modmul": (i32, [vp, i32, ctypes.POINTER(ctypes.c_double)]),
        "hb_ctx_launches": (u64, [vp]),
        "hb_ctx_set_wait_limit": (i32, [vp, ctypes.c_longlong]),
        "hb_ctx_test_withhold_keys": (i32, [vp, i32]),
        "hb_keys_generate": (i32, [vp, P, u64, vp, vp, pp]),
        "hb_encrypt_device": (i32, [vp, P, vp, u64, u64, vp, sz, vp]),
        "hb_keys_device_words": (i32, [vp, ctypes.POINTER(sz), ctypes.POINTER(sz)]),
        "hb_keys_download": (i32, [vp, vp, vp, sz, vp, sz]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error(ctx):
    if not ctx:
        return ""
    buf = ctypes.create_string_buffer(512)
    lib().hb_last_error(ctx, buf, 512)
    return buf.value.decode(errors="replace")


def check(rc, what, ctx=None):
    if rc != HB_OK:
        raise HbError(rc, what, last_error(ctx))
