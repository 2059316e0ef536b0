"""Host-side mirror of the reference tfhe crate API over the C ABI of libhb_gpu.so.

Names follow the reference (tfhe/src/lib.rs:1-13): parameter statics, KeyGen, SecretKeyPack,
Encryptor, Decryptor, Evaluator with nand/and/or/nor/xor/xnor/majority/not/mux/bootstrap
(tfhe/src/bfhe/evaluate.rs:65-262). Ciphertexts are numpy arrays (host) or torch CUDA tensors
(device), shape [count, n + 1], dtype uint64 (Goldilocks) / uint32 (BabyBear, DefaultFieldU32),
canonical values.
Host arrays go through hb_gate (copies in and out included); device tensors through hb_gate_device
on the context stream.
"""

import ctypes
import os

import numpy as np

from . import _lib
from ._lib import HbParams, check, lib

GATE_IDS = {"nand": 0, "and": 1, "or": 2, "nor": 3, "xor": 4, "xnor": 5, "majority": 6,
            "not": 7, "mux": 8}


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(ctypes.c_void_p)
    return ctypes.c_void_p(a.data_ptr())  # torch tensor


class Parameters:
    """fhe_core::Parameters for RLWE bootstrapping with the RLWE key switch."""

    def __init__(self, raw: HbParams, name=""):
        check(lib().hb_params_validate(ctypes.byref(raw)), "Parameters::new")
        self.raw = raw
        self.name = name

    @classmethod
    def preset(cls, pid):
        raw = HbParams()
        check(lib().hb_params_preset(pid, ctypes.byref(raw)), "hb_params_preset")
        names = {0: "BABYBEAR_BINARY_128_BITS_PARAMETERS",
                 1: "GOLDILOCKS_BINARY_128_BITS_PARAMETERS", 2: "ZAMA_BINARY_128_BITS_PARAMETERS",
                 3: "DEFAULT_TERNARY_128_BITS_PARAMETERS", 4: "CUSTOM_TERNARY_128_BITS_PARAMETERS"}
        return cls(raw, names[pid])

    def with_ternary_lwe_key(self):
        """The same set with a ternary LWE secret key (LWESecretKeyType::Ternary,
        fhe_core/src/secret_key.rs:12-18); DefaultFieldU32 sets only."""
        raw = HbParams.from_buffer_copy(self.raw)
        raw.lwe_ternary = 1
        return Parameters(raw, self.name + "+TERNARY_LWE_KEY")

    @property
    def field_id(self):
        return self.raw.field_id

    @property
    def dtype(self):
        return np.uint64 if self.raw.field_id == _lib.FIELD_GOLDILOCKS else np.uint32

    @property
    def modulus(self):
        return _lib.MODULUS[self.raw.field_id]

    def lwe_dimension(self):
        return self.raw.lwe_dim

    def ring_dimension(self):
        return self.raw.ring_dim

    def sizes(self):
        out = [ctypes.c_size_t() for _ in range(5)]
        check(lib().hb_params_sizes(ctypes.byref(self.raw), *[ctypes.byref(o) for o in out]),
              "hb_params_sizes")
        keys = ("lwe_sk", "ring_sk", "bsk", "ksk", "lwe")
        return {k: o.value for k, o in zip(keys, out)}


def BABYBEAR_BINARY_128_BITS_PARAMETERS():
    return Parameters.preset(0)


def DEFAULT_TERNARY_128_BITS_PARAMETERS():
    return Parameters.preset(3)


def CUSTOM_TERNARY_128_BITS_PARAMETERS():
    return Parameters.preset(4)


def GOLDILOCKS_BINARY_128_BITS_PARAMETERS():
    return Parameters.preset(1)


def ZAMA_BINARY_128_BITS_PARAMETERS():
    return Parameters.preset(2)


class SecretKeyPack:
    """fhe_core::SecretKeyPack (fhe_core/src/secret_key.rs:42-89), seeded."""

    def __init__(self, params: Parameters, seed=0):
        self.params = params
        self.seed = seed
        s = params.sizes()
        self.lwe_secret_key = np.zeros(s["lwe_sk"], params.dtype)
        self.ring_secret_key = np.zeros(s["ring_sk"], params.dtype)
        check(lib().hb_keygen(ctypes.byref(params.raw), seed, _ptr(self.lwe_secret_key),
                              _ptr(self.ring_secret_key), None, None, 0), "KeyGen")
        self._next_index = 0

    def evaluation_key_material(self, threads=0):
        """BSK and KSK (coefficient domain) of this key pack (Evaluator::new's key generation)."""
        s = self.params.sizes()
        lwe = np.zeros(s["lwe_sk"], self.params.dtype)
        ring = np.zeros(s["ring_sk"], self.params.dtype)
        bsk = np.zeros(s["bsk"], self.params.dtype)
        ksk = np.zeros(s["ksk"], self.params.dtype)
        check(lib().hb_keygen(ctypes.byref(self.params.raw), self.seed, _ptr(lwe), _ptr(ring),
                              _ptr(bsk), _ptr(ksk), threads), "KeyGen")
        return bsk, ksk

    def encrypt(self, bits, index0=None):
        bits = np.ascontiguousarray(np.atleast_1d(bits), dtype=np.uint8)
        if index0 is None:
            index0 = self._next_index
        self._next_index = index0 + len(bits)
        out = np.zeros((len(bits), self.params.lwe_dimension() + 1), self.params.dtype)
        check(lib().hb_encrypt(ctypes.byref(self.params.raw), _ptr(self.lwe_secret_key), self.seed,
                               index0, _ptr(bits), len(bits), _ptr(out)), "encrypt")
        return out

    def decrypt_with_noise(self, cts):
        cts = np.ascontiguousarray(cts, dtype=self.params.dtype).reshape(
            -1, self.params.lwe_dimension() + 1)
        bits = np.zeros(len(cts), np.uint8)
        noise = np.zeros(len(cts), np.uint64)
        check(lib().hb_decrypt(ctypes.byref(self.params.raw), _ptr(self.lwe_secret_key), _ptr(cts),
                               len(cts), _ptr(bits), _ptr(noise)), "decrypt")
        return bits, noise

    def decrypt(self, cts):
        return self.decrypt_with_noise(cts)[0]


class KeyGen:
    @staticmethod
    def generate_secret_key(params: Parameters, seed=0):
        return SecretKeyPack(params, seed)


class Encryptor:
    def __init__(self, sk: SecretKeyPack):
        self.sk = sk

    def encrypt(self, bits, index0=None):
        return self.sk.encrypt(bits, index0)


class Decryptor:
    def __init__(self, sk: SecretKeyPack):
        self.sk = sk

    def decrypt(self, cts):
        return self.sk.decrypt(cts)

    def decrypt_with_noise(self, cts):
        return self.sk.decrypt_with_noise(cts)


class Context:
    """One CUDA device + stream + HBM budget (hb_ctx)."""

    def __init__(self, device=0, hbm_budget=0):
        h = ctypes.c_void_p()
        check(lib().hb_ctx_create(device, hbm_budget, ctypes.byref(h)), "hb_ctx_create")
        self.handle = h
        self.device = device

    def stream_ptr(self):
        s = ctypes.c_void_p()
        check(lib().hb_ctx_stream(self.handle, ctypes.byref(s)), "hb_ctx_stream", self.handle)
        return s.value or 0

    def synchronize(self):
        check(lib().hb_ctx_synchronize(self.handle), "hb_ctx_synchronize", self.handle)

    def hbm_in_use(self):
        return lib().hb_ctx_hbm_in_use(self.handle)

    def close(self):
        if self.handle:
            lib().hb_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceKeys:
    """Device-resident BSK/KSK (hb_keys)."""

    def __init__(self, ctx: Context, params: Parameters, bsk=None, ksk=None, handle=None):
        if handle is None:
            h = ctypes.c_void_p()
            bsk = np.ascontiguousarray(bsk, params.dtype)
            ksk = np.ascontiguousarray(ksk, params.dtype)
            check(lib().hb_keys_upload(ctx.handle, ctypes.byref(params.raw), _ptr(bsk), _ptr(ksk),
                                       ctypes.byref(h)), "hb_keys_upload", ctx.handle)
            handle = h
        self.ctx = ctx
        self.params = params
        self.handle = handle

    @classmethod
    def generate(cls, ctx: Context, params: Parameters, seed=0):
        """Evaluator::new's key material generated on the device (hb_keys_generate): the same
        words as the host generator followed by an upload. Returns (keys, lwe_sk, ring_sk)."""
        s = params.sizes()
        lwe = np.zeros(s["lwe_sk"], params.dtype)
        ring = np.zeros(s["ring_sk"], params.dtype)
        h = ctypes.c_void_p()
        check(lib().hb_keys_generate(ctx.handle, ctypes.byref(params.raw), seed, _ptr(lwe), _ptr(ring),
                                     ctypes.byref(h)), "hb_keys_generate", ctx.handle)
        return cls(ctx, params, handle=h), lwe, ring

    def download(self):
        """The device words of the keys (transformed, scaled, kernel slot layout): (bsk, ksk)."""
        nb, nk = ctypes.c_size_t(), ctypes.c_size_t()
        check(lib().hb_keys_device_words(self.handle, ctypes.byref(nb), ctypes.byref(nk)),
              "hb_keys_device_words")
        bsk = np.zeros(nb.value, self.params.dtype)
        ksk = np.zeros(nk.value, self.params.dtype)
        check(lib().hb_keys_download(self.ctx.handle, self.handle, _ptr(bsk), nb.value, _ptr(ksk),
                                     nk.value), "hb_keys_download", self.ctx.handle)
        return bsk, ksk

    def free(self):
        if self.handle and self.ctx.handle:
            lib().hb_keys_free(self.ctx.handle, self.handle)
        self.handle = None


class Evaluator:
    """tfhe::Evaluator (tfhe/src/bfhe/evaluate.rs:65-262) on one B200."""

    def __init__(self, sk: SecretKeyPack, ctx: Context = None, keys=None, device_keygen=True):
        """Keys generated on the device by default (hb_keys_generate); device_keygen=False runs the
        host generator and uploads its coefficient-domain keys. Both give the same device words."""
        self.params = sk.params
        self.ctx = ctx or Context()
        if keys is None and device_keygen:
            keys, lwe, ring = DeviceKeys.generate(self.ctx, self.params, sk.seed)
            if not ((lwe == sk.lwe_secret_key).all() and (ring == sk.ring_secret_key).all()):
                keys.free()
                raise ValueError("secret keys differ from the key pack's")
        elif keys is None:
            bsk, ksk = sk.evaluation_key_material()
            keys = DeviceKeys(self.ctx, self.params, bsk, ksk)
        self.keys = keys

    def parameters(self):
        return self.params

    def _gate(self, name, c0, c1=None, c2=None):
        gid = GATE_IDS[name]
        w = self.params.lwe_dimension() + 1
        if isinstance(c0, np.ndarray):
            dt = self.params.dtype
            c0 = np.ascontiguousarray(c0, dt).reshape(-1, w)
            c1 = None if c1 is None else np.ascontiguousarray(c1, dt).reshape(-1, w)
            c2 = None if c2 is None else np.ascontiguousarray(c2, dt).reshape(-1, w)
            out = np.zeros_like(c0)
            check(lib().hb_gate(self.ctx.handle, self.keys.handle, gid, _ptr(c0), _ptr(c1), _ptr(c2),
                                _ptr(out), len(c0)), name, self.ctx.handle)
            return out
        import torch  # device tensors
        out = torch.empty_like(c0)
        torch.cuda.current_stream().synchronize()
        check(lib().hb_gate_device(self.ctx.handle, self.keys.handle, gid, _ptr(c0), _ptr(c1),
                                   _ptr(c2), _ptr(out), c0.shape[0]), name, self.ctx.handle)
        self.ctx.synchronize()
        return out

    def nand(self, c0, c1):
        return self._gate("nand", c0, c1)

    def and_(self, c0, c1):
        return self._gate("and", c0, c1)

    def or_(self, c0, c1):
        return self._gate("or", c0, c1)

    def nor(self, c0, c1):
        return self._gate("nor", c0, c1)

    def xor(self, c0, c1):
        return self._gate("xor", c0, c1)

    def xnor(self, c0, c1):
        return self._gate("xnor", c0, c1)

    def majority(self, c0, c1, c2):
        return self._gate("majority", c0, c1, c2)

    def not_(self, c0):
        return self._gate("not", c0)

    def mux(self, c0, c1, c2):
        return self._gate("mux", c0, c1, c2)

    def bootstrap(self, c, lut):
        dt = self.params.dtype
        c = np.ascontiguousarray(c, dt).reshape(-1, self.params.lwe_dimension() + 1)
        lut = np.ascontiguousarray(lut, dt)
        out = np.zeros_like(c)
        check(lib().hb_bootstrap_lut(self.ctx.handle, self.keys.handle, _ptr(c), _ptr(lut),
                                     _ptr(out), len(c)), "bootstrap", self.ctx.handle)
        return out

    def bootstrap_with_trace(self, c, lut):
        """bootstrap of one ciphertext plus the accumulator after every blind-rotation step (the
        AccTrace of vfhe's bootstrap, vfhe/src/bfhe/evaluate.rs:47-141): returns (out [n + 1],
        trace [n, 2N] with a in [:, :N] and b in [:, N:])."""
        dt = self.params.dtype
        n, N = self.params.lwe_dimension(), self.params.ring_dimension()
        c = np.ascontiguousarray(c, dt).reshape(n + 1)
        lut = np.ascontiguousarray(lut, dt)
        out = np.zeros(n + 1, dt)
        trace = np.zeros((n, 2 * N), dt)
        check(lib().hb_bootstrap_trace(self.ctx.handle, self.keys.handle, _ptr(c), _ptr(lut),
                                       _ptr(out), _ptr(trace)), "bootstrap_with_trace", self.ctx.handle)
        return out, trace


    def bootstrap_with_trace_batch(self, c, lut, digits=True):
        """bootstrap of a batch of ciphertexts (one persistent launch) with, per ciphertext, the
        accumulator after every blind-rotation step and, with digits=True, every step's gadget
        digits of (X^a_i - 1) ACC (hb_bootstrap_trace_device). Host arrays in; returns
        (out [count, n + 1], acc [count, n, 2N], digits [count, n, 2, l, N] uint8 or None)."""
        import torch
        dt = self.params.dtype
        raw = self.params.raw
        n, N, L = raw.lwe_dim, raw.ring_dim, raw.br_len
        c = np.ascontiguousarray(c, dt).reshape(-1, n + 1)
        count = len(c)
        tdt = torch.int64 if dt == np.uint64 else torch.int32
        ivt = np.int64 if dt == np.uint64 else np.int32
        dc = torch.from_numpy(c.view(ivt).copy()).cuda()
        dl = torch.from_numpy(np.ascontiguousarray(lut, dt).view(ivt).copy()).cuda()
        dout = torch.zeros_like(dc)
        dacc = torch.zeros((count, n, 2 * N), dtype=tdt, device="cuda")
        ddig = torch.zeros((count, n, 2, L, N), dtype=torch.uint8, device="cuda") if digits else None
        torch.cuda.synchronize()
        check(lib().hb_bootstrap_trace_device(self.ctx.handle, self.keys.handle, _ptr(dc), _ptr(dl),
                                              _ptr(dout), count, _ptr(dacc), _ptr(ddig)),
              "bootstrap_with_trace_batch", self.ctx.handle)
        self.ctx.synchronize()
        return (dout.cpu().numpy().view(dt), dacc.cpu().numpy().view(dt),
                ddig.cpu().numpy() if digits else None)


# ------------------------------------------------------------------------------------------------
# Autotuning and mixed-set batches
# ------------------------------------------------------------------------------------------------

AUTOTUNE_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_autotune_cache.json")


def _device_name(device):
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return "cuda:%d" % device


def _tune_key(ev):
    r = ev.params.raw
    return "|".join(str(x) for x in (_device_name(ev.ctx.device), r.field_id, r.ring_dim, r.lwe_dim,
                                     r.br_bits, r.br_len, r.ks_bits, r.ks_len))


def autotune(ev, sample_gates=0, use_cache=True):
    """Pick the fastest compiled kernel variant -- threads per gate (NTT tile) and gates per CTA --
    for this evaluator's key set (hb_autotune), remembering the choice per device and parameter set
    in AUTOTUNE_CACHE. Returns ((threads_per_gate, gates_per_cta), gates_per_s, from_cache)."""
    import json
    key = _tune_key(ev)
    cache = {}
    if use_cache and os.path.exists(AUTOTUNE_CACHE):
        try:
            cache = json.load(open(AUTOTUNE_CACHE))
        except ValueError:
            cache = {}
    if use_cache and key in cache and "threads_per_gate" in cache[key]:
        c = cache[key]
        if lib().hb_keys_set_config(ev.ctx.handle, ev.keys.handle, c["threads_per_gate"],
                                    c["gates_per_cta"]) == 0:
            lib().hb_keys_set_rate(ev.keys.handle, c["gates_per_s"])
            return (c["threads_per_gate"], c["gates_per_cta"]), c["gates_per_s"], True
    t = ctypes.c_int()
    g = ctypes.c_int()
    rate = ctypes.c_double()
    check(lib().hb_autotune(ev.ctx.handle, ev.keys.handle, sample_gates, ctypes.byref(t),
                            ctypes.byref(g), ctypes.byref(rate)), "hb_autotune", ev.ctx.handle)
    if use_cache:
        cache[key] = {"threads_per_gate": t.value, "gates_per_cta": g.value, "gates_per_s": rate.value}
        # best effort: processes of one job (one per GPU) may write the same cache at once
        tmp = f"{AUTOTUNE_CACHE}.{os.getpid()}.tmp"
        try:
            with open(tmp, "w") as f:
                json.dump(cache, f, indent=1)
            os.replace(tmp, AUTOTUNE_CACHE)
        except OSError:
            pass
    return (t.value, g.value), rate.value, False


class Batch:
    """A planned batch of gate jobs that may mix parameter sets (hb_batch): one CUDA graph holding
    one persistent launch per key set. jobs: iterable of (evaluator, gate_name, c0, c1, c2, out)
    with torch CUDA tensors (c2 may be None)."""

    def __init__(self, ctx: Context, jobs):
        from ._lib import HbJob
        jobs = list(jobs)
        arr = (HbJob * max(1, len(jobs)))()
        self._keep = jobs
        for i, (ev, gate, c0, c1, c2, out) in enumerate(jobs):
            arr[i].keys = ev.keys.handle
            arr[i].gate = GATE_IDS[gate]
            arr[i].count = c0.shape[0]
            arr[i].c0 = c0.data_ptr()
            arr[i].c1 = c1.data_ptr() if c1 is not None else None
            arr[i].c2 = c2.data_ptr() if c2 is not None else None
            arr[i].out = out.data_ptr()
        h = ctypes.c_void_p()
        check(lib().hb_batch_create(ctx.handle, arr, len(jobs), ctypes.byref(h)), "hb_batch_create",
              ctx.handle)
        self.ctx = ctx
        self.handle = h

    def info(self):
        gates = ctypes.c_uint64()
        launches = ctypes.c_int()
        grid = (ctypes.c_int * 8)()
        check(lib().hb_batch_info(self.handle, ctypes.byref(gates), ctypes.byref(launches), grid, 8),
              "hb_batch_info")
        return {"gates": gates.value, "launches": launches.value,
                "sm_split": list(grid)[:launches.value]}

    def launch(self):
        check(lib().hb_batch_launch(self.ctx.handle, self.handle), "hb_batch_launch", self.ctx.handle)

    def free(self):
        if self.handle:
            lib().hb_batch_free(self.ctx.handle, self.handle)
            self.handle = None


class Server:
    """Request loop with continuous batching (hb_serve_*). Submissions take host ciphertext arrays
    (pinned memory recommended), which this wrapper keeps alive until fetched."""

    def __init__(self, ctx: Context, hbm_budget=0, max_wave_gates=0, max_inflight_waves=0, max_queue_s=0.0):
        from ._lib import HbServeConfig
        cfg = HbServeConfig(hbm_budget, max_wave_gates, max_inflight_waves, max_queue_s)
        h = ctypes.c_void_p()
        check(lib().hb_serve_start(ctx.handle, ctypes.byref(cfg), ctypes.byref(h)), "hb_serve_start",
              ctx.handle)
        self.ctx = ctx
        self.handle = h
        self._live = {}

    def submit(self, ev: "Evaluator", gate, c0, c1, c2=None):
        """Returns the request id, or None when the server refuses the request: its predicted
        completion lies beyond max_queue_s (load shedding), or the server is stopping."""
        rid = ctypes.c_uint64()
        arrays = [a for a in (c0, c1, c2) if a is not None]
        rc = lib().hb_serve_submit(self.handle, ev.keys.handle, GATE_IDS[gate], _ptr(c0), _ptr(c1),
                                   _ptr(c2), len(c0), ctypes.byref(rid))
        if rc == -6 and rid.value == 0:  # HB_ERR_BUSY: refused by the queue-delay bound
            return None
        check(rc, "hb_serve_submit")
        self._live[rid.value] = (arrays, ev.params, len(c0))
        return rid.value

    def state(self, rid):
        st = ctypes.c_int()
        check(lib().hb_serve_poll(self.handle, rid, ctypes.byref(st)), "hb_serve_poll")
        return st.value

    def next_done(self, timeout=10.0):
        rid = ctypes.c_uint64()
        rc = lib().hb_serve_next_done(self.handle, ctypes.byref(rid), timeout)
        return rid.value if rc == 0 else None

    def fetch(self, rid, out=None):
        arrays, params, count = self._live.pop(rid)
        if out is None:
            out = np.zeros((count, params.lwe_dimension() + 1), params.dtype)
        lat = ctypes.c_double()
        check(lib().hb_serve_fetch(self.handle, rid, _ptr(out), ctypes.byref(lat)), "hb_serve_fetch")
        return out, lat.value

    def stats(self):
        from ._lib import HbServeStats
        st = HbServeStats()
        lib().hb_serve_stats(self.handle, ctypes.byref(st))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def stop(self):
        if self.handle:
            rc = lib().hb_serve_stop(self.handle)
            self.handle = None
            return rc
        return 0
