/*
 * hb_gpu.h -- C ABI of the B200 (sm_100a) TFHE gate-bootstrapping library (libhb_gpu.so).
 *
 * Drop-in boundary for HasteBoots' bootstrapping path: the tfhe crate's Evaluator / KeyGen /
 * Encryptor / Decryptor (tfhe/src/lib.rs:1-13, tfhe/src/bfhe/evaluate.rs), the lattice crate's
 * RLWE x RGSW external product (lattice/src/rlwe.rs:573-596) and the algebra crate's NTT-table trait
 * (algebra/src/transformation/mod.rs:20-96). A Rust binding (hb-gpu-sys) declares these functions
 * verbatim in an `extern "C"` block.
 *
 * Conventions
 *  - Every function returns an int status: HB_OK (0) or a negative HB_ERR_* code. After an error,
 *    hb_last_error() on the same context returns a one-line description. The Rust shim maps
 *    non-zero statuses to panics where the reference panics (tfhe/src/bfhe/evaluate.rs:56) and to
 *    Err where it returns Result (Parameters::new, fhe_core/src/parameter.rs:111).
 *  - Field words are canonical little-endian values: uint64_t for Goldilocks
 *    (Q = 2^64 - 2^32 + 1), uint32_t for BabyBear (Q = 2^31 - 2^27 + 1) and DefaultFieldU32
 *    (Q = 132120577 = 2^27 - 2^21 + 1, fhe_core/src/parameter.rs:286-290).
 *  - An LWE ciphertext is n+1 words: a[0..n) then b. Batches are contiguous arrays of them.
 *  - Key material in host buffers is coefficient domain: BSK layout
 *    [i < n][pair][part: 0 = c_neg_s_m, 1 = c_m][j < br_len][0 = a, 1 = b][N] with one pair for a
 *    binary LWE key and two -- RGSW(s_i == 1), RGSW(s_i == -1) -- for a ternary one; KSK layout
 *    [c < N/n'][j < ks_len][0 = a, 1 = b][n'] with n' = next_pow2(n) (NTTRGSW
 *    lattice/src/rgsw.rs:212-218, TernaryBlindRotationKey
 *    fhe_core/src/blind_rotation/rlwe/ternary.rs:13-16, NTTGadgetRLWE
 *    lattice/src/gadget/rlwe.rs:235-240, KeySwitchingRLWEKey fhe_core/src/key_switch/rlwe.rs:23-28,
 *    one gadget RLWE per n'-word chunk of the ring key, :79-108).
 *  - Functions named *_device take device pointers and enqueue on the context's stream without
 *    synchronising; all other functions take host pointers and return when results are in place.
 *  - A context is used by one host thread at a time.
 */
#ifndef HB_GPU_H
#define HB_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HB_OK 0
#define HB_ERR_INVALID (-1)     /* bad argument or parameter set */
#define HB_ERR_CUDA (-2)        /* CUDA runtime error */
#define HB_ERR_NOMEM (-3)       /* allocation would exceed the context's HBM budget */
#define HB_ERR_TIMEOUT (-4)     /* a kernel's bounded wait ran out; results are invalid */
#define HB_ERR_UNSUPPORTED (-5) /* parameter combination without a compiled kernel */
#define HB_ERR_BUSY (-6)        /* serving queue full */

#define HB_FIELD_BABYBEAR 0
#define HB_FIELD_GOLDILOCKS 1
#define HB_FIELD_DEFAULT_U32 2 /* DefaultFieldU32, Q = 132120577 */

/* Parameter-set ids (tfhe/src/bfhe/parameters.rs:7-117). The two *_TERNARY_* sets configure
 * binary LWE and ring keys over DefaultFieldU32; n = 1024 and n = 512 (two key-switching chunks). */
#define HB_PRESET_BABYBEAR_BINARY_128_BITS 0
#define HB_PRESET_GOLDILOCKS_BINARY_128_BITS 1
#define HB_PRESET_ZAMA_BINARY_128_BITS 2
#define HB_PRESET_DEFAULT_TERNARY_128_BITS 3
#define HB_PRESET_CUSTOM_TERNARY_128_BITS 4

/* Gate ids (Evaluator::{nand, and, or, nor, xor, xnor, majority, not, mux},
 * tfhe/src/bfhe/evaluate.rs:98-262). */
#define HB_GATE_NAND 0
#define HB_GATE_AND 1
#define HB_GATE_OR 2
#define HB_GATE_NOR 3
#define HB_GATE_XOR 4
#define HB_GATE_XNOR 5
#define HB_GATE_MAJORITY 6
#define HB_GATE_NOT 7
#define HB_GATE_MUX 8

typedef struct hb_ctx hb_ctx;
typedef struct hb_keys hb_keys;

/* fhe_core::ConstParameters (fhe_core/src/parameter.rs:81-107) with the RLWE key switch. */
typedef struct hb_params {
  int32_t field_id;      /* HB_FIELD_* */
  uint32_t ring_dim;     /* N (1024 is compiled) */
  uint32_t lwe_dim;      /* n <= N; the key switch works in dimension n' = next_pow2(n) */
  uint32_t br_bits;      /* blind_rotation_basis_bits */
  uint32_t br_len;       /* ceil(bits(Q) / br_bits) (Basis::new, algebra/src/decompose_basis.rs:29-40) */
  uint32_t ks_bits;      /* key_switching_basis_bits */
  uint32_t ks_len;       /* ceil(bits(Q) / ks_bits) */
  uint32_t ring_ternary; /* ring secret key: 1 ternary, 0 binary */
  uint32_t lwe_ternary;  /* LWE secret key: 1 ternary (HB_FIELD_DEFAULT_U32 only; LWESecretKeyType,
                            fhe_core/src/secret_key.rs:12-18), 0 binary */
  double lwe_noise_std;
  double ring_noise_std;
  double ks_noise_std;
} hb_params;

/* ---- parameters -------------------------------------------------------------------------- */

/* Replaces the LazyLock parameter statics (tfhe/src/bfhe/parameters.rs:45-117). */
int hb_params_preset(int preset, hb_params *out);
/* Replaces Parameters::new's checks (fhe_core/src/parameter.rs:111-172). */
int hb_params_validate(const hb_params *p);
/* Word counts of the host buffers for p: lwe_sk, ring_sk, bsk, ksk, and one LWE ciphertext. */
int hb_params_sizes(const hb_params *p, size_t *lwe_sk, size_t *ring_sk, size_t *bsk, size_t *ksk,
                    size_t *lwe);

/* ---- client side (host CPU) --------------------------------------------------------------- */

/* KeyGen::generate_secret_key + Evaluator::new key material (tfhe/src/key_gen.rs:12,
 * fhe_core/src/secret_key.rs:67-89, fhe_core/src/blind_rotation/rlwe/binary.rs:207-239,
 * fhe_core/src/key_switch/rlwe.rs:37-112) from a 64-bit seed: the reference seeds from OS entropy,
 * this library derives every sample from a counter PRG of (seed, stream, counter). */
int hb_keygen(const hb_params *p, uint64_t seed, void *lwe_sk, void *ring_sk, void *bsk, void *ksk,
              int threads);
/* Encryptor::encrypt / SecretKeyPack::encrypt (fhe_core/src/secret_key.rs:129-149); ciphertext i
 * uses sample index index0 + i. */
int hb_encrypt(const hb_params *p, const void *lwe_sk, uint64_t seed, uint64_t index0,
               const uint8_t *bits, size_t count, void *lwe_out);
/* hb_encrypt on the device: d_lwe_sk (n words), d_bits (count bytes) and d_out (count ciphertexts)
 * are device buffers; enqueued on the context stream. Same ciphertexts as hb_encrypt. */
int hb_encrypt_device(hb_ctx *ctx, const hb_params *p, const void *d_lwe_sk, uint64_t seed,
                      uint64_t index0, const uint8_t *d_bits, size_t count, void *d_out);
/* Decryptor::decrypt / SecretKeyPack::decrypt_with_noise (fhe_core/src/secret_key.rs:151-188);
 * noise_out may be NULL. */
int hb_decrypt(const hb_params *p, const void *lwe_sk, const void *lwe, size_t count,
               uint8_t *bits_out, uint64_t *noise_out);

/* ---- device context ----------------------------------------------------------------------- */

/* One CUDA device, one stream, an HBM budget (bytes, 0 = unlimited) for key and batch memory. */
int hb_ctx_create(int device, size_t hbm_budget, hb_ctx **out);
void hb_ctx_destroy(hb_ctx *ctx);
int hb_last_error(const hb_ctx *ctx, char *buf, size_t len);
/* The context's cudaStream_t, for callers that enqueue their own copies around *_device calls. */
int hb_ctx_stream(hb_ctx *ctx, void **stream);
int hb_ctx_synchronize(hb_ctx *ctx);
/* Bytes of device memory the context currently holds against its budget. */
size_t hb_ctx_hbm_in_use(const hb_ctx *ctx);

/* ---- evaluation keys (Evaluator::new, tfhe/src/bfhe/evaluate.rs:26-39) ---------------------- */

/* Upload coefficient-domain BSK/KSK; transforms and lays them out on the device. */
int hb_keys_upload(hb_ctx *ctx, const hb_params *p, const void *bsk, const void *ksk, hb_keys **out);
/* KeyGen::generate_secret_key + Evaluator::new (tfhe/src/key_gen.rs:12,
 * tfhe/src/bfhe/evaluate.rs:26-39, fhe_core/src/blind_rotation/rlwe/binary.rs:207-239,
 * ternary.rs:123-183, fhe_core/src/key_switch/rlwe.rs:37-112) with the key material generated on
 * the device: the secret keys (n and N words) are written to lwe_sk / ring_sk, and the evaluation
 * keys come out identical, word for word, to hb_keygen followed by hb_keys_upload. */
int hb_keys_generate(hb_ctx *ctx, const hb_params *p, uint64_t seed, void *lwe_sk, void *ring_sk,
                     hb_keys **out);
void hb_keys_free(hb_ctx *ctx, hb_keys *keys);
int hb_keys_params(const hb_keys *keys, hb_params *out);
/* No counterpart in the reference: the words of the device-resident keys (transformed, scaled,
 * in the bootstrap kernel's slot layout), for inspection and for tests of key generation. */
int hb_keys_device_words(const hb_keys *keys, size_t *bsk_words, size_t *ksk_words);
int hb_keys_download(hb_ctx *ctx, const hb_keys *keys, void *bsk, size_t bsk_words, void *ksk,
                     size_t ksk_words);

/* ---- gate bootstrapping --------------------------------------------------------------------- */

/* Evaluator::{nand,and,or,nor,xor,xnor,majority,not,mux} over `count` independent gates
 * (tfhe/src/bfhe/evaluate.rs:98-262). c2 is read by MAJORITY and MUX only. Host buffers. */
int hb_gate(hb_ctx *ctx, hb_keys *keys, int gate, const void *c0, const void *c1, const void *c2,
            void *out, size_t count);
/* Same on device buffers, enqueued on the context stream (one launch per bootstrap layer: MUX takes
 * two). A layer of at most one gate per SM runs the latency form -- with a binary LWE key a cluster
 * of CTAs per gate (4 for the Goldilocks sets, 2 for the 32-bit fields) while the layer holds at
 * most one cluster CTA per SM, else one CTA per gate -- and larger layers the persistent batched
 * kernel. */
int hb_gate_device(hb_ctx *ctx, hb_keys *keys, int gate, const void *c0, const void *c1,
                   const void *c2, void *out, size_t count);
/* The plain form: one kernel launch per gate. */
int hb_gate_device_plain(hb_ctx *ctx, hb_keys *keys, int gate, const void *c0, const void *c1,
                         void *out, size_t count);
/* EvaluationKey::bootstrap(c, lut) (tfhe/src/bfhe/evaluate.rs:42-60) for count ciphertexts sharing
 * one LUT polynomial of N words. Host buffers. */
int hb_bootstrap_lut(hb_ctx *ctx, hb_keys *keys, const void *c, const void *lut, void *out,
                     size_t count);
/* EvaluationKey::bootstrap(c, lut) of one ciphertext that also returns the blind-rotation
 * accumulator after every step, the AccTrace that vfhe's bootstrap records for its proof
 * (vfhe/src/bfhe/evaluate.rs:47-141): acc_trace receives n x 2N canonical words, step i's
 * accumulator a at [i][0, N) and b at [i][N, 2N), before b[0] += Q/8 and the key switch. Steps
 * with a zero rotation leave the accumulator as it was. Host buffers; binary LWE keys
 * (HB_ERR_UNSUPPORTED for a ternary one). */
int hb_bootstrap_trace(hb_ctx *ctx, hb_keys *keys, const void *c, const void *lut, void *out,
                       void *acc_trace);
/* The traced bootstrap of vfhe (vfhe/src/bfhe/evaluate.rs:47-141) for a batch of count ciphertexts
 * sharing one LUT polynomial, in one persistent launch (two gates per CTA). Per gate g:
 *  - acc_trace[g][i] = the accumulator after blind-rotation step i, n x 2N canonical words (a then
 *    b): AccTrace's rows (trace/src/acc_trace.rs, blind_rotate_w_trace,
 *    fhe_core/src/blind_rotation/rlwe/binary.rs:106-205);
 *  - digit_trace[g][i][part][j] (may be NULL) = the N unsigned gadget digits j of E.a (part 0) and
 *    E.b (part 1), E = (X^a_i - 1) ACC, one byte each, [count][n][2][l][N]: the bit polynomials
 *    of SumHadamardTrace (append_bit_poly in mul_polynomial_inplace_fast_w_traces,
 *    lattice/src/gadget/rlwe.rs:426-457); a step with a_i = 0 has E = 0 and zero digits.
 * The digits' NTTs and the NTT-domain key rows the reference records as well are not produced:
 * their slot order is concrete-ntt's. Device pointers; c and out are [count][n + 1] words, lut N
 * words; enqueued on the context stream (hb_ctx_synchronize reports device-side waits that ran
 * out). Binary LWE keys; digit traces need a gadget base of at most 2^8 (every preset's).
 * HB_ERR_UNSUPPORTED otherwise. */
int hb_bootstrap_trace_device(hb_ctx *ctx, hb_keys *keys, const void *c, const void *lut, void *out,
                              size_t count, void *acc_trace, void *digit_trace);

/* ---- NTT table trait and external product (device slices) ---------------------------------- */

/* AbstractNTT::transform_slice over count polynomials of 2^log_n words, in place. Output slot
 * order is bit-reversed evaluation order at odd powers of a primitive 2N-th root (the reference's
 * concrete-ntt order is unspecified; only round trips and products are part of the contract). */
int hb_ntt_forward_device(hb_ctx *ctx, int field_id, uint32_t log_n, void *data, size_t count);
/* AbstractNTT::inverse_transform_slice (inverse + normalise), in place. */
int hb_ntt_inverse_device(hb_ctx *ctx, int field_id, uint32_t log_n, void *data, size_t count);
/* Forward then inverse (round trip) from `in` to `out`. */
int hb_ntt_roundtrip_device(hb_ctx *ctx, int field_id, uint32_t log_n, const void *in, void *out,
                            size_t count);
/* NTTRGSW from a coefficient-domain RGSW (host buffer, layout of one BSK entry); the returned
 * device handle feeds hb_external_product_device and is released with hb_rgsw_free. */
int hb_rgsw_upload(hb_ctx *ctx, int field_id, uint32_t log_n, uint32_t bits, uint32_t len,
                   const void *rgsw, void **d_rgsw);
void hb_rgsw_free(hb_ctx *ctx, void *d_rgsw);
/* RLWE::mul_assign_ntt_rgsw (lattice/src/rlwe.rs:573-596): out_i = rlwe_i x RGSW for count
 * coefficient-domain RLWEs (2 * 2^log_n words each). */
int hb_external_product_device(hb_ctx *ctx, int field_id, uint32_t log_n, uint32_t bits,
                               uint32_t len, const void *d_rgsw, const void *rlwe_in,
                               void *rlwe_out, size_t count);

/* ---- autotuning and mixed-set batches ----------------------------------------------------- */

/* Times every compiled variant of the persistent kernel for this key set -- threads per gate T
 * (the NTT tile: 64 threads x 16 words or 128 threads x 8 words, which fixes the device key
 * layout) and gates per CTA G -- on sample_gates NAND gates (0: 24 per SM), keeps the fastest for
 * later launches (re-laying the keys out if T changes) and reports it with its throughput.
 * No counterpart in the reference (its path is single-threaded CPU). */
int hb_autotune(hb_ctx *ctx, hb_keys *keys, uint32_t sample_gates, int *threads_per_gate,
                int *gates_per_cta, double *gates_per_s);
/* Restores a cached autotuner choice; HB_ERR_UNSUPPORTED if that variant is not compiled. */
int hb_keys_set_config(hb_ctx *ctx, hb_keys *keys, int threads_per_gate, int gates_per_cta);
int hb_keys_config(const hb_keys *keys, int *threads_per_gate, int *gates_per_cta);
/* Restores a cached autotuner rate (gates per second of this key set alone), which the serving
 * loop uses to predict queue delay; hb_autotune sets it. No counterpart in the reference. */
int hb_keys_set_rate(hb_keys *keys, double gates_per_s);

/* One bootstrapped-gate job of a batch: `count` gates (NAND..MAJORITY) of one key set on device
 * buffers. Batching across gates of the reference's Evaluator (tfhe/src/bfhe/evaluate.rs:113-237). */
typedef struct hb_job {
  hb_keys *keys;
  int32_t gate;
  uint32_t count;
  const void *c0, *c1, *c2;
  void *out;
} hb_job;
typedef struct hb_batch hb_batch;

/* Plans a batch of jobs that may mix parameter sets and gate kinds: one launch per key set on its own
 * stream, each with a full grid (the block scheduler hands SMs to the next set's CTAs as the previous
 * set's retire), all captured into one CUDA graph. */
int hb_batch_create(hb_ctx *ctx, const hb_job *jobs, size_t njobs, hb_batch **out);
/* Enqueues the whole batch as one graph launch on the context stream. */
int hb_batch_launch(hb_ctx *ctx, hb_batch *batch);
void hb_batch_free(hb_ctx *ctx, hb_batch *batch);
/* Gates in the batch, kernels per launch, and the grid of each (up to grid_cap entries). */
int hb_batch_info(const hb_batch *batch, uint64_t *gates, int *launches, int *grid, int grid_cap);

/* ---- serving: request loop with continuous batching ----------------------------------------
 * No counterpart in the reference (its Evaluator is a synchronous single-gate CPU call). */

typedef struct hb_server hb_server;
typedef struct hb_serve_config {
  size_t hbm_budget;           /* bytes of request memory (inputs + output) on the device; 0 = 120 GiB */
  uint32_t max_wave_gates;     /* gates packed into one wave at most; 0 = no limit */
  uint32_t max_inflight_waves; /* waves on the GPU at once (1..4); 0 = 2 */
  double max_queue_s;          /* load shedding: hb_serve_submit refuses (HB_ERR_BUSY) a request whose
                                  predicted completion, from the work ahead of it and the key sets'
                                  calibrated rates, lies more than this many seconds away; 0 = admit all */
} hb_serve_config;
typedef struct hb_serve_stats {
  uint64_t submitted, admitted, completed, failed, queued, waves, gates_completed;
  double p50_latency_s, p99_latency_s, mean_latency_s, max_latency_s;
  double gates_per_s; /* completed gates / (last completion - first submission) */
  size_t hbm_in_use, hbm_peak;
  uint64_t rejected; /* submissions refused by the max_queue_s bound */
} hb_serve_statistics;

/* Starts the request loop of a context (one worker thread). Keys used by requests must outlive it. */
int hb_serve_start(hb_ctx *ctx, const hb_serve_config *cfg, hb_server **out);
/* Queues `count` single-bootstrap gates (NAND..MAJORITY) on host input buffers, which must stay
 * valid until the request is admitted (its state leaves 0). Thread-safe. */
int hb_serve_submit(hb_server *s, hb_keys *keys, int gate, const void *c0, const void *c1,
                    const void *c2, uint32_t count, uint64_t *id);
/* State of a request: 0 queued, 1 admitted, 2 running, 3 done, -1 failed. */
int hb_serve_poll(hb_server *s, uint64_t id, int *state);
/* Id of the next request to finish (done or failed), waiting up to timeout_s; HB_ERR_BUSY on timeout. */
int hb_serve_next_done(hb_server *s, uint64_t *id, double timeout_s);
/* Copies a finished request's output ciphertexts to `out` (host, may be NULL), reports its latency
 * (submission to completion on the device) and returns its memory to the budget. */
int hb_serve_fetch(hb_server *s, uint64_t id, void *out, double *latency_s);
int hb_serve_stats(hb_server *s, hb_serve_statistics *out);
/* Stops admitting, lets the waves on the GPU finish, cancels the rest and frees everything. */
int hb_serve_stop(hb_server *s);

/* Evaluator::mux for callers that cannot allocate device memory during a call: a serving process
 * that reserves its whole HBM budget at start-up and may not take a cudaMalloc on its request path
 * (cudaMalloc can synchronise the device and fragments the heap), or a host that hands out all
 * device memory from its own pool. No counterpart in the reference.
 * The intermediate ciphertexts, job table and status word live in a 16 MiB array compiled into the
 * library, which every GPU that loads the library holds until the process exits. count is at most
 * (16 MiB - 1 KiB) / (2 (n + 1) word bytes): 1438 gates for the Goldilocks sets, 2876 for BabyBear,
 * 2045 for DEFAULT_TERNARY, 4087 for CUSTOM_TERNARY; larger counts return HB_ERR_INVALID. The
 * first call on a context looks up the array's device address, so make that call before any stream
 * capture. A wait that runs out in the first of the two bootstrap layers returns HB_ERR_TIMEOUT
 * without running the second. Every call uses the same array: calls whose work overlaps on the GPU (other streams,
 * contexts or host threads) race and must be serialised. Device pointers in; returns when `out`
 * holds the result (synchronises the context stream). The keys must have been created (uploaded or
 * generated) on this context. */
int hb_gate_mux_device_noalloc(hb_ctx *ctx, hb_keys *keys, const void *c0, const void *c1,
                               const void *c2, void *out, size_t count);

/* ---- diagnostics ------------------------------------------------------------------------ */

/* Field-multiplication throughput of this device (independent register chains, all SMs): the
 * integer-pipe ceiling against which bootstrapping's modular multiplies are measured. No
 * counterpart in the reference, which publishes CPU timings only. */
int hb_probe_modmul(hb_ctx *ctx, int field_id, double *modmul_per_s);
/* Kernel launches the context has issued for bootstrapping (batched, latency and plain forms). */
uint64_t hb_ctx_launches(const hb_ctx *ctx);
/* Limit, in SM clock cycles, of every bounded wait inside this context's kernels (waits for key
 * chunks in flight); 0 restores the default (about 2 s). A wait that runs out makes the call return
 * HB_ERR_TIMEOUT and leaves the context usable; tests use a tiny limit to exercise that path.
 * No counterpart in the reference. */
int hb_ctx_set_wait_limit(hb_ctx *ctx, long long clock_cycles);
/* Test hook for the path above: while on, bootstrapping launches of this context issue no key
 * copies, so their first wait for a key chunk runs out (a flag that nothing sets) and the call
 * returns HB_ERR_TIMEOUT. No counterpart in the reference. */
int hb_ctx_test_withhold_keys(hb_ctx *ctx, int on);

#ifdef __cplusplus
}
#endif

#endif /* HB_GPU_H */
