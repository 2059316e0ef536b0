// hb_kernels.cuh -- sm_100a kernels of the TFHE gate-bootstrapping path.
//
//  * prepare_polys_kernel   coefficient-domain key polynomials -> device NTT slot layout, scaled by
//                           N^-1 (and R for BabyBear) so the inverse transform needs no normalising
//  * relayout_kernel        moves a resident key between the slot layouts of two NTT tiles
//  * ntt_batch_kernel       batched forward, inverse or round-trip negacyclic NTT on device slices
//                           (AbstractNTT::{transform_slice, inverse_transform_slice})
//  * ext_product_kernel     RLWE x RGSW external product for many RLWEs sharing one RGSW
//  * bootstrap_kernel       persistent batched gate bootstrapping: modulus switch, blind rotation
//                           with accumulators in shared memory, key switching and sample extraction,
//                           G gates per CTA sharing every bootstrapping-key chunk, which the TMA unit
//                           streams into a ring of shared-memory stages
//  * bootstrap_dp_kernel    the same bootstrap for launches of at most one gate per SM: one gate
//                           per CTA (or per cluster of CTAs) with its gadget digits spread over the
//                           thread groups
//  * modmul_probe_kernel    field-multiply throughput (the roofline denominator)
#pragma once

#include "hb_field.cuh"
#include "hb_ntt.cuh"
#include "hb_sync.cuh"

namespace hb {

enum : int { STATUS_OK = 0, STATUS_TIMEOUT = 1 };

// Clock budget of the wait, on an abort, for bulk copies still in flight into shared memory. It is
// independent of the launch's wait limit: a CTA must not exit while a copy can still land.
constexpr long long kDrainBudget = 4000000000LL;

// ------------------------------------------------------------------------------------------
// Shared pieces
// ------------------------------------------------------------------------------------------

// lwe_modulus_switch (fhe_core/src/modulus_switch.rs:12-38): round(f64(v) * 2N / f64(Q)) mod 2N
// with IEEE round-to-nearest conversion, multiply and divide, and round-half-away-from-zero.
template <class F>
__device__ __forceinline__ uint32_t modswitch(typename F::W v, uint32_t two_n) {
  const double x = __ull2double_rn((unsigned long long)F::value(v));
  const double q = __ull2double_rn((unsigned long long)F::P);
  const double r = round(__ddiv_rn(__dmul_rn(x, (double)two_n), q));
  const uint32_t t = (uint32_t)(unsigned long long)r;
  return t < two_n ? t : t - two_n;
}

template <class F>
__device__ __forceinline__ typename F::W canon_neg(typename F::W x) {
  x = F::canon(x);
  return x == 0 ? 0 : F::P - x;
}

// s * x for s in {-2,...,2}, canonical result.
template <class F>
__device__ __forceinline__ typename F::W small_mul(typename F::W x, int s) {
  using W = typename F::W;
  x = F::canon(x);
  W y = s == 2 || s == -2 ? F::canon(F::add(x, x)) : (s == 0 ? 0 : x);
  return s < 0 ? canon_neg<F>(y) : y;
}

// One gate job: `count` gates whose input LWE ciphertexts are combined as
// c = s0*c0 + s1*c1 + s2*c2 (+ add_b on the body), then bootstrapped with a LUT that is either a
// caller polynomial (`lut`) or the piecewise constant {lo on [0, mid), hi on [mid, N)} of the gate
// LUT builders (tfhe/src/bfhe/evaluate.rs:267-465).
struct GateJob {
  const void *in0, *in1, *in2;
  void *out;
  const void *lut;
  unsigned long long lut_lo, lut_hi, add_b;
  uint32_t lut_mid;
  int32_t s0, s1, s2;
  uint32_t count;
  uint32_t first_batch;
};

// Ring of S shared-memory stages fed by the TMA unit with consecutive 2N-word chunks of key
// material (cp.async.bulk, no multicast), consumed by G independent thread groups without a
// CTA-wide barrier: each group releases a stage after its own barrier by counting itself in
// `cnt`; the group whose count completes a multiple of G refills the stage. Groups can therefore
// drift up to S - 1 chunks apart (one may run its multiply-heavy accumulate while another runs the
// add-heavy transform). `issued` counts the copies per stage so that an aborting CTA can wait for
// the ones in flight.
template <class W, int N, int S, int G>
struct GroupPipe {
  W *stages;
  uint64_t *bars;
  uint32_t *cnt, *issued;
  volatile int *abort_flag;
  int *status;
  long long budget;
  unsigned long long next;
  unsigned long long total;
  static constexpr uint32_t WORDS = 2 * N;
  static constexpr uint32_t BYTES = WORDS * sizeof(W);

  template <class Src>
  __device__ __forceinline__ void prime(const Src &src) {
    if (threadIdx.x == 0)
      for (unsigned long long c = 0; c < (unsigned long long)S && c < total; ++c) {
        issued[c] = 1;
        mbar_arrive_expect_tx(&bars[c], BYTES);
        bulk_g2s(stages + c * WORDS, src(c), BYTES, &bars[c]);
      }
  }
  __device__ __forceinline__ const W *acquire() {
    const int st = (int)(next % S);
    const uint32_t par = (uint32_t)((next / S) & 1);
    if (!mbar_wait_bounded(&bars[st], par, budget)) {
      *abort_flag = 1;
      atomicOr(status, STATUS_TIMEOUT);
    }
    return stages + st * WORDS;
  }
  // The chunk after the current one, held together with it (two releases follow). Cannot deadlock
  // with S >= 2: that chunk's copy waits only on the releases of chunk next + 1 - S, which every
  // group passed before it took chunk next.
  __device__ __forceinline__ const W *acquire_next() {
    static_assert(S >= 2, "two chunks held at once need two stages");
    const unsigned long long c = next + 1;
    const int st = (int)(c % S);
    const uint32_t par = (uint32_t)((c / S) & 1);
    if (!mbar_wait_bounded(&bars[st], par, budget)) {
      *abort_flag = 1;
      atomicOr(status, STATUS_TIMEOUT);
    }
    return stages + st * WORDS;
  }
  // Group-wide release of the current chunk (t: the thread's index in its group); false when the
  // launch must stop.
  template <class Src, class Sync>
  __device__ __forceinline__ bool release(const Src &src, int t, const Sync &sync) {
    sync();  // every thread of this group is done reading the stage
    if (*abort_flag) return false;
    if (t == 0) {
      const int st = (int)(next % S);
      __threadfence_block();
      // Counts only grow (no reset to order against other groups). They stay far below 2^32: a
      // stage takes G releases per S chunks, about 40 per gate of a launch, and no launch can
      // hold 10^8 gates' ciphertexts in HBM.
      if ((atomicAdd(&cnt[st], 1u) + 1) % G == 0) {
        __threadfence_block();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (next + S < total) {
          issued[st] += 1;
          mbar_arrive_expect_tx(&bars[st], BYTES);
          bulk_g2s(stages + st * WORDS, src(next + S), BYTES, &bars[st]);
        }
      }
    }
    ++next;
    return true;
  }
  // After an abort, with every thread of the CTA past its loops: wait (bounded) for the last copy
  // issued into each stage.
  __device__ __forceinline__ void drain() {
    if (threadIdx.x != 0) return;
    for (int st = 0; st < S; ++st)
      if (issued[st]) mbar_wait_bounded(&bars[st], (issued[st] - 1) & 1, kDrainBudget);
  }
};

// ------------------------------------------------------------------------------------------
// Key preparation
// ------------------------------------------------------------------------------------------

// in: npolys coefficient-domain polynomials (natural order, canonical); out: same count in the
// device slot layout out[poly][v*T + t] = scale * NTT(in)[slot t*V + v].
template <class F, int LOGN, int T>
__global__ void __launch_bounds__(2 * T) prepare_polys_kernel(const typename F::W *__restrict__ in,
                                                             typename F::W *__restrict__ out,
                                                             unsigned long long npolys,
                                                             const typename F::W *__restrict__ tw_g,
                                                             typename F::W scale) {
  using W = typename F::W;
  using NT = GroupNtt<F, LOGN, T>;
  constexpr int N = 1 << LOGN, V = NT::V;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int TWN = N * F::TW_WORDS;  // words of a twiddle table
  W *s_tw = reinterpret_cast<W *>(smem_raw);
  W *s_x = s_tw + TWN;
  const int g = threadIdx.x / T, t = threadIdx.x % T;
  for (int i = threadIdx.x; i < TWN; i += blockDim.x) s_tw[i] = tw_g[i];
  __syncthreads();
  GroupSync<T> sync{1 + g};
  W *xbuf = s_x + g * 2 * N;
  int ping = 0;
  for (unsigned long long poly = (unsigned long long)blockIdx.x * 2 + g; poly < npolys;
       poly += (unsigned long long)gridDim.x * 2) {
    W x[V];
    const W *src = in + poly * N;
#pragma unroll
    for (int v = 0; v < V; ++v) x[v] = F::canon(src[NT::natural_pos(t, v)]);
    NT::forward(x, xbuf, ping, s_tw, t, sync);
    W *dst = out + poly * N;
#pragma unroll
    for (int v = 0; v < V; ++v) dst[v * T + t] = F::mul(x[v], scale);
  }
}

// Moves key polynomials from the slot layout of a T_from-thread group to that of a T_to-thread
// group: slot s = t*V + v is stored at v*T + t (V = N/T).
template <class W>
__global__ void __launch_bounds__(256) relayout_kernel(const W *__restrict__ in, W *__restrict__ out,
                                                       unsigned long long words, int N, int t_from,
                                                       int t_to) {
  const int v_from = N / t_from, v_to = N / t_to;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < words;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long base = i - i % N;
    const int p = (int)(i % N);
    const int slot = (p % t_from) * v_from + p / t_from;
    out[base + (slot % v_to) * t_to + slot / v_to] = in[i];
  }
}

// ------------------------------------------------------------------------------------------
// Batched NTT kernels (one polynomial per thread group)
// ------------------------------------------------------------------------------------------

// mode 0: forward then inverse with N^-1 (round trip), 1: forward only (slot order out),
// 2: inverse only (slot order in, N^-1 applied).
template <class F, int LOGN, int T, int GPB>
__global__ void __launch_bounds__(GPB * T) ntt_batch_kernel(const typename F::W *in,  // may alias out
                                                           typename F::W *out,
                                                           unsigned long long npolys,
                                                           const typename F::W *__restrict__ tw_g,
                                                           const typename F::W *__restrict__ itw_g,
                                                           typename F::W n_inv, int mode) {
  using W = typename F::W;
  using NT = GroupNtt<F, LOGN, T>;
  constexpr int N = 1 << LOGN, V = NT::V;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int TWN = N * F::TW_WORDS;
  W *s_tw = reinterpret_cast<W *>(smem_raw);
  W *s_itw = s_tw + TWN;
  W *s_x = s_itw + TWN;
  const int g = threadIdx.x / T, t = threadIdx.x % T;
  for (int i = threadIdx.x; i < TWN; i += blockDim.x) {
    s_tw[i] = tw_g[i];
    s_itw[i] = itw_g[i];
  }
  __syncthreads();
  GroupSync<T> sync{1 + g};
  W *xbuf = s_x + g * 2 * N;
  int ping = 0;
  for (unsigned long long poly = (unsigned long long)blockIdx.x * GPB + g; poly < npolys;
       poly += (unsigned long long)gridDim.x * GPB) {
    W x[V];
    const W *src = in + poly * N;
    W *dst = out + poly * N;
    if (mode == 2) {
#pragma unroll
      for (int v = 0; v < V; ++v) x[v] = src[NT::slot_pos(t, v)];
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v) x[v] = src[NT::natural_pos(t, v)];
    }
    if (mode != 2) NT::forward(x, xbuf, ping, s_tw, t, sync);
    if (mode == 1) {
#pragma unroll
      for (int v = 0; v < V; ++v) dst[NT::slot_pos(t, v)] = F::canon(x[v]);
      continue;
    }
    NT::inverse(x, xbuf, ping, s_itw, t, sync);
#pragma unroll
    for (int v = 0; v < V; ++v) dst[NT::natural_pos(t, v)] = F::mul(x[v], n_inv);
  }
}

// ------------------------------------------------------------------------------------------
// External product: out_i = RLWE_i x RGSW (lattice/src/rlwe.rs:573-596) for many RLWEs
// ------------------------------------------------------------------------------------------

// Digit j of the unsigned LSB-first decomposition (Polynomial::decompose_lsb_bits_inplace,
// algebra/src/polynomial/univariate/native_polynomial.rs:340-348) of the words e[v * T + t]:
// (e >> sh) & mask with sh = j * bits uniform, as one funnel shift of the word's halves (or one
// shift of the high half) and a mask.
template <class W, int V, int T>
__device__ __forceinline__ void digits(W (&x)[V], const W *e, int t, uint32_t sh, uint32_t mask) {
  if constexpr (sizeof(W) == 8) {
    if (sh < 32) {
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const uint64_t w = e[v * T + t];
        x[v] = __funnelshift_r((uint32_t)w, (uint32_t)(w >> 32), sh) & mask;
      }
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v) x[v] = ((uint32_t)(e[v * T + t] >> 32) >> (sh - 32)) & mask;
    }
  } else {
#pragma unroll
    for (int v = 0; v < V; ++v) x[v] = (e[v * T + t] >> sh) & mask;
  }
}

// The same on words held in registers.
template <class W, int V>
__device__ __forceinline__ void digits_reg(W (&x)[V], const W (&e)[V], uint32_t sh, uint32_t mask) {
  if constexpr (sizeof(W) == 8) {
    if (sh < 32) {
#pragma unroll
      for (int v = 0; v < V; ++v) x[v] = __funnelshift_r((uint32_t)e[v], (uint32_t)(e[v] >> 32), sh) & mask;
    } else {
#pragma unroll
      for (int v = 0; v < V; ++v) x[v] = ((uint32_t)(e[v] >> 32) >> (sh - 32)) & mask;
    }
  } else {
#pragma unroll
    for (int v = 0; v < V; ++v) x[v] = (e[v] >> sh) & mask;
  }
}

// A lazy accumulator that already took `nprod` products must be folded (acc_fold) before the
// next one: every FOLD products (never for accumulators that need no folds).
template <int FOLD>
__device__ __forceinline__ bool fold_due_n(uint32_t nprod) {
  if constexpr (FOLD >= (1 << 20)) {
    return false;
  } else {
    return nprod != 0 && nprod % FOLD == 0;
  }
}
template <class F>
__device__ __forceinline__ bool fold_due(uint32_t nprod) {
  return fold_due_n<F::FOLD>(nprod);
}

// Accumulator of the latency form, whose groups each sum only a few products per phase: the
// field's lazy accumulator for Goldilocks, and for the 32-bit fields a word reduced at every
// product (their 64-bit sums cost 32 registers at 16 words per thread, more than their
// instructions save on a few products).
template <class F, bool REDUCED = sizeof(typename F::W) == 4>
struct FewAcc {
  using A = typename F::Acc;
  static constexpr int FOLD = F::FOLD;
  __device__ __forceinline__ static void clear(A &a) { F::acc_clear(a); }
  __device__ __forceinline__ static void mac(A &a, typename F::W x, typename F::W k) { F::acc_mac(a, x, k); }
  __device__ __forceinline__ static void fold(A &a) { F::acc_fold(a); }
  __device__ __forceinline__ static typename F::W value(const A &a, typename F::W off) { return F::acc_value(a, off); }
};
template <class F>
struct FewAcc<F, true> {
  struct A {
    typename F::W w;
  };
  static constexpr int FOLD = 1 << 30;
  __device__ __forceinline__ static void clear(A &a) { a.w = 0; }
  __device__ __forceinline__ static void mac(A &a, typename F::W x, typename F::W k) { a.w = F::mac(a.w, x, k); }
  __device__ __forceinline__ static void fold(A &) {}
  __device__ __forceinline__ static typename F::W value(const A &a, typename F::W) { return a.w; }
};

template <class F, int LOGN, int T, int G, int S>
__global__ void __launch_bounds__(G * T, 1)
    ext_product_kernel(const typename F::W *__restrict__ rlwe_in, typename F::W *__restrict__ rlwe_out,
                       unsigned long long count, const typename F::W *__restrict__ rgsw,
                       uint32_t len, uint32_t bits, const typename F::W *__restrict__ tw_g,
                       const typename F::W *__restrict__ itw_g, int *status, long long budget) {
  using W = typename F::W;
  using NT = GroupNtt<F, LOGN, T>;
  constexpr int N = 1 << LOGN, V = NT::V;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int TWN = N * F::TW_WORDS;
  W *s_tw = reinterpret_cast<W *>(smem_raw);
  W *s_itw = s_tw + TWN;
  W *s_k = s_itw + TWN;
  W *s_x = s_k + S * 2 * N;
  uint64_t *s_bar = reinterpret_cast<uint64_t *>(s_x + G * 2 * N);
  uint32_t *s_cnt = reinterpret_cast<uint32_t *>(s_bar + S);
  uint32_t *s_issued = s_cnt + S;
  volatile int *s_abort = reinterpret_cast<volatile int *>(s_issued + S);
  const int tid = threadIdx.x, g = tid / T, t = tid % T;
  for (int i = tid; i < TWN; i += blockDim.x) {
    s_tw[i] = tw_g[i];
    s_itw[i] = itw_g[i];
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&s_bar[s], 1);
      s_cnt[s] = 0;
      s_issued[s] = 0;
    }
    mbar_fence_init();
    *s_abort = 0;
  }
  __syncthreads();
  GroupSync<T> sync{1 + g};
  W *xbuf = s_x + g * 2 * N;
  int ping = 0;

  const unsigned long long batches = (count + G - 1) / G;
  const unsigned long long my_batches =
      blockIdx.x < batches ? (batches - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const uint32_t cpb = 2 * len;
  GroupPipe<W, N, S, G> pipe{s_k, s_bar, s_cnt, s_issued, s_abort, status, budget, 0, my_batches * cpb};
  auto src = [&](unsigned long long c) { return rgsw + (size_t)(c % cpb) * 2 * N; };
  pipe.prime(src);
  const uint32_t mask = bits >= 32 ? 0xFFFFFFFFu : ((1u << bits) - 1);
  const W off = F::acc_offset(2 * len);  // every slot sums 2 len products

  for (unsigned long long b = blockIdx.x; b < batches; b += gridDim.x) {
    const unsigned long long item = b * G + g;
    const bool active = item < count;
    typename F::Acc acc_a[V], acc_b[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      F::acc_clear(acc_a[v]);
      F::acc_clear(acc_b[v]);
    }
    uint32_t nprod = 0;  // products in the accumulators since the last fold
    for (int part = 0; part < 2; ++part) {
      W e[V];
      if (active) {
        const W *src_poly = rlwe_in + (item * 2 + part) * N;
#pragma unroll
        for (int v = 0; v < V; ++v) e[v] = F::value(src_poly[NT::natural_pos(t, v)]);
      }
      for (uint32_t j = 0; j < len; ++j) {
        W x[V];
        if (active) {
          digits_reg<W, V>(x, e, j * bits, mask);
          NT::forward_small(x, xbuf, ping, s_tw, t, sync);
        }
        const W *k = pipe.acquire();
        if (active) {
          if (fold_due<F>(nprod)) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
              F::acc_fold(acc_a[v]);
              F::acc_fold(acc_b[v]);
            }
          }
#pragma unroll
          for (int v = 0; v < V; ++v) {
            F::acc_mac(acc_a[v], x[v], k[v * T + t]);
            F::acc_mac(acc_b[v], x[v], k[N + v * T + t]);
          }
        }
        ++nprod;
        if (!pipe.release(src, t, sync)) goto aborted;
      }
    }
    if (active) {
      W fa[V], fb[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        fa[v] = F::acc_value(acc_a[v], off);
        fb[v] = F::acc_value(acc_b[v], off);
      }
      NT::inverse(fa, xbuf, ping, s_itw, t, sync);
      NT::inverse(fb, xbuf, ping, s_itw, t, sync);
      W *dst = rlwe_out + item * 2 * N;
#pragma unroll
      for (int v = 0; v < V; ++v) {
        dst[NT::natural_pos(t, v)] = F::canon(fa[v]);
        dst[N + NT::natural_pos(t, v)] = F::canon(fb[v]);
      }
    }
  }
aborted:
  __syncthreads();
  if (*s_abort) pipe.drain();
}

// ------------------------------------------------------------------------------------------
// Persistent batched bootstrapping (EvaluationKey::bootstrap, tfhe/src/bfhe/evaluate.rs:42-60)
// ------------------------------------------------------------------------------------------

template <class W>
struct BootParams {
  const W *bsk;  // [n][pairs][2][len][2][N] slot layout, scaled (one 2N-word chunk per row)
  const W *ksk;  // [ks_chunks][ks_len][2][N] slot layout, scaled (chunk keys spread to N words)
  const W *tw, *itw;
  const W *itw_w;  // bootstrap_dp_kernel: inverse twiddles of its half-CTA groups
  const GateJob *jobs;
  int njobs;
  uint32_t total_batches;
  uint32_t n, len, bits, ks_len, ks_bits;
  uint32_t ks_n, ks_chunks;  // key-switch dimension n' = next_pow2(n) and its N / n' chunks
  int *status;
  long long budget;
  int withhold;  // test hook: issue no key-chunk copy, so the first wait runs out (bounded)
  W *trace;      // the accumulator after every blind-rotation step, [gate][n][a | b][N] canonical
                 // words (bootstrap_dp_kernel: one gate; bootstrap_kernel: its TRACE variant, one
                 // job); null records nothing
  uint8_t *digits;  // bootstrap_kernel's TRACE variant: every step's gadget digits of E.a then E.b,
                    // [gate][n][2][len][N] bytes (bases up to 2^8); null records nothing
};

// Shared memory needed by bootstrap_kernel: twiddles (2N words), S key-chunk stages (2N words
// each), per gate the accumulator (2N), the exchange buffers (2N) and the decomposition source
// (N), the modulus-switched input (n + 1 halves) and the stage barriers.
// Exchange buffers of the bootstrap kernel's transforms: two per gate (one barrier per exchange) or
// one (a second barrier per exchange). One buffer with the freed 32 KB spent on four key stages
// measured 0.75 % slower for GOLDILOCKS at G = 4, so two is the default.
#ifndef HB_BOOT_PINGPONG
#define HB_BOOT_PINGPONG 1
#endif
constexpr bool kBootPingPong = HB_BOOT_PINGPONG != 0;
// Digit pairs: a bootstrap kernel variant that transforms two digits at once (GroupNtt::
// forward_small2) gives each thread two independent transforms to interleave. Measured on B200
// (16384 gates per launch), it pays for BabyBear where the launch leaves 128 registers per thread
// (T G = 512 threads: T = 64, G = 8: 439.4 -> 427.7 ms; T = 128, G = 4: 501.7 -> 487.0 ms) and
// costs elsewhere (BabyBear T = 64, G = 6: 447.9 -> 460.1 ms; DefaultFieldU32, whose 64-bit sums
// already hold 32 more registers: up to 23 % slower), so only those variants use it.
template <class F, int T, int G>
__host__ __device__ constexpr bool boot_dual() {
  if constexpr (sizeof(typename F::W) == 4) {
    return !F::WIDE && T * G >= 512;
  } else {
    return false;
  }
}
constexpr int kBootXbuf = kBootPingPong ? 2 : 1;  // exchange buffers of N words per gate

template <class W, int N, int G, int S>
__host__ __device__ constexpr size_t boot_smem_bytes(uint32_t n) {
  return sizeof(W) * (size_t)(2 * tw_words<W>() * N + S * 2 * N + G * (3 + kBootXbuf) * N) +
         sizeof(uint16_t) * (size_t)G * ((n + 8) & ~7u) + sizeof(uint64_t) * S + 2 * sizeof(uint32_t) * S + 16;
}

// Key-chunk stages of a bootstrap_kernel variant: 3 when they fit the 227 KB of shared memory a
// CTA can have (for LWE dimensions up to 1016), else 2.
template <class W, int N, int G>
__host__ __device__ constexpr int boot_stages() {
  return boot_smem_bytes<W, N, G, 3>(1016) <= 232448 ? 3 : 2;
}

// TERN: ternary LWE key (TernaryBlindRotationKey, fhe_core/src/blind_rotation/rlwe/ternary.rs:26-119)
// with two RGSWs per key coefficient, for fields whose words stay canonical. E = (X^a_i - 1) ACC is
// the product the reference's comment names (ternary.rs:91); its code forms it from an
// untransformed NTT-domain monomial (:93-100), which this kernel does not reproduce.
// KSC: key switch in ks_chunks chunks of n' = next_pow2(n) < N words; without it the key switch is
// the single chunk n' = N of the reference presets, with no chunk bookkeeping in the kernel.
// TRACE (binary LWE key, one job): every gate also writes the accumulator after each blind-rotation
// step to p.trace and, when p.digits is set, each step's gadget digits to p.digits (the witness of
// vfhe's traced bootstrap, vfhe/src/bfhe/evaluate.rs:47-141).
template <class F, int LOGN, int T, int G, int S, bool TERN = false, bool KSC = false, bool TRACE = false>
__global__ void __launch_bounds__(G * T, 1) bootstrap_kernel(const BootParams<typename F::W> p) {
  using W = typename F::W;
  using NT = GroupNtt<F, LOGN, T, kBootPingPong>;
  constexpr int N = 1 << LOGN, V = NT::V, TWN = N * F::TW_WORDS;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  W *s_tw = reinterpret_cast<W *>(smem_raw);
  W *s_itw = s_tw + TWN;
  W *s_k = s_itw + TWN;
  W *s_grp = s_k + S * 2 * N;
  W *s_e = s_grp + G * (2 + kBootXbuf) * N;
  const uint32_t msz = (p.n + 8) & ~7u;
  uint16_t *s_ms = reinterpret_cast<uint16_t *>(s_e + G * N);
  uint64_t *s_bar = reinterpret_cast<uint64_t *>(s_ms + G * msz);
  uint32_t *s_cnt = reinterpret_cast<uint32_t *>(s_bar + S);
  uint32_t *s_issued = s_cnt + S;
  volatile int *s_abort = reinterpret_cast<volatile int *>(s_issued + S);

  const int tid = threadIdx.x, g = tid / T, t = tid % T;
  for (int i = tid; i < TWN; i += blockDim.x) {
    s_tw[i] = p.tw[i];
    s_itw[i] = p.itw[i];
  }
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&s_bar[s], 1);
      s_cnt[s] = 0;
      s_issued[s] = 0;
    }
    mbar_fence_init();
    *s_abort = 0;
  }
  __syncthreads();

  GroupSync<T> sync{1 + g};
  W *acc_a = s_grp + g * (2 + kBootXbuf) * N;
  W *acc_b = acc_a + N;
  W *xbuf = acc_b + N;
  W *ebuf = s_e + g * N;  // decomposition source, thread t owns words v * T + t
  uint16_t *ms = s_ms + g * msz;
  int ping = 0;

  const uint32_t n = p.n;
  constexpr uint32_t PAIRS = TERN ? 2 : 1;
  const uint32_t br_chunks = n * PAIRS * 2 * p.len;
  const uint32_t ks_chunks = KSC ? p.ks_chunks : 1;
  const uint32_t cpb = br_chunks + ks_chunks * p.ks_len;
  const uint32_t my_batches =
      blockIdx.x < p.total_batches ? (p.total_batches - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  GroupPipe<W, N, S, G> pipe{s_k, s_bar, s_cnt, s_issued, s_abort, p.status, p.budget, 0,
                             p.withhold ? 0ull : (unsigned long long)my_batches * cpb};
  // Chunks in consumption order: per step (i, part, j) and, for a ternary key, both RGSWs' rows
  // of that digit in turn (stored [i][pair][part][j]); then the key switch's [c][j] rows.
  auto src = [&](unsigned long long c) -> const W * {
    const uint32_t q = (uint32_t)(c % cpb);
    if (q >= br_chunks) return p.ksk + (size_t)(q - br_chunks) * 2 * N;
    if constexpr (TERN) {
      const uint32_t L = p.len, i = q / (4 * L), r = q % (4 * L);
      const uint32_t part = r / (2 * L), j = (r >> 1) % L, pair = r & 1;
      return p.bsk + ((size_t)((i * 2 + pair) * 2 + part) * L + j) * 2 * N;
    } else {
      return p.bsk + (size_t)q * 2 * N;
    }
  };
  pipe.prime(src);

  const uint32_t two_n = 2 * N;
  // Offsets that remove the per-product bookkeeping of the lazy accumulators (F::acc_value): a
  // blind-rotation step sums 2 len products per slot, the key switch ks_len.
  const W off_br = F::acc_offset(2 * p.len);
  const W off_ks = F::acc_offset(ks_chunks * p.ks_len);

  for (uint32_t batch = blockIdx.x; batch < p.total_batches; batch += gridDim.x) {
    int jx = 0;
    while (jx + 1 < p.njobs && p.jobs[jx + 1].first_batch <= batch) ++jx;
    const GateJob &job = p.jobs[jx];
    const uint32_t gate = (batch - job.first_batch) * G + g;
    const bool active = gate < job.count;
    const size_t lwe_words = (size_t)n + 1;

    // ---- input combine + modulus switch (Evaluator::nand etc., evaluate.rs:113-119) ----
    if (active) {
      const W *c0 = reinterpret_cast<const W *>(job.in0) + gate * lwe_words;
      const W *c1 = job.in1 ? reinterpret_cast<const W *>(job.in1) + gate * lwe_words : nullptr;
      const W *c2 = job.in2 ? reinterpret_cast<const W *>(job.in2) + gate * lwe_words : nullptr;
      for (uint32_t k = t; k <= n; k += T) {
        W c = small_mul<F>(c0[k], job.s0);
        if (c1) c = F::canon(F::add(c, small_mul<F>(c1[k], job.s1)));
        if (c2) c = F::canon(F::add(c, small_mul<F>(c2[k], job.s2)));
        if (k == n) c = F::canon(F::add(c, (W)job.add_b));
        ms[k] = (uint16_t)modswitch<F>(c, two_n);
      }
    }
    sync();
    // ---- ACC = (0, LUT * X^{-b}) (fhe_core/src/blind_rotation/rlwe/binary.rs:40-64) ----
    if (active) {
      const uint32_t bt = ms[n];
      const int e = bt ? (int)(two_n - bt) : 0;
      const W *lut = reinterpret_cast<const W *>(job.lut);
      for (int k = t; k < N; k += T) {
        int s = k - e;
        bool neg = false;
        if (s < 0) {
          s += N;
          neg = true;
          if (s < 0) {
            s += N;
            neg = false;
          }
        }
        W f = lut ? F::canon(lut[s]) : (W)((uint32_t)s < job.lut_mid ? job.lut_lo : job.lut_hi);
        acc_a[k] = 0;
        acc_b[k] = neg ? F::neg_ref(f) : f;
      }
    }
    sync();

    // ---- blind rotation (binary.rs:66-103), then key switching (key_switch/rlwe.rs:115-137) ----
    // One loop of 2n + ks_chunks phases shares a single forward-NTT and a single inverse-NTT call
    // site: phase 2i + part decomposes E.a (part 0) or E.b (part 1) of step i, phase 2n + c
    // decomposes the key switch's chunk c of -acc.a.
    typename F::Acc acc_x[V], acc_y[V];
    typename F::Acc acc_x1[TERN ? V : 1], acc_y1[TERN ? V : 1];  // ternary: RGSW(s_i == -1) products
#pragma unroll
    for (int v = 0; v < V; ++v) {
      F::acc_clear(acc_x[v]);
      F::acc_clear(acc_y[v]);
      if constexpr (TERN) {
        F::acc_clear(acc_x1[v]);
        F::acc_clear(acc_y1[v]);
      }
    }
    uint32_t nprod = 0;  // products in the accumulators since their last fold or clear
    const uint32_t phases = 2 * n + ks_chunks;
    for (uint32_t ph = 0; ph < phases; ++ph) {
      const bool ks = KSC ? ph >= 2 * n : ph == 2 * n;
      const uint32_t part = ph & 1;
      if (active) {
        if (!ks) {
          // E = ACC * (X^r - 1) (lattice/src/rlwe.rs:437-487) in the reference's representation,
          // then canonical for the unsigned decomposition.
          const int r = (int)ms[ph >> 1];
          const W *y = part == 0 ? acc_a : acc_b;
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const int k = NT::natural_pos(t, v);
            int s = k - r;
            W rot;
            if (s >= 0) {
              rot = y[s];
            } else if (s >= -N) {
              rot = F::neg_ref(y[s + N]);
            } else {
              rot = y[s + 2 * N];
            }
            ebuf[v * T + t] = F::value(F::sub(rot, y[k]));
          }
        } else if (!KSC) {
          // sub_assign_gadget_rlwe_mul_polynomial_inplace_fast: p = -acc.a (lattice/src/rlwe.rs:1147-1166)
#pragma unroll
          for (int v = 0; v < V; ++v) ebuf[v * T + t] = F::value(F::neg_ref(acc_a[NT::natural_pos(t, v)]));
        } else {
          // n' < N (fhe_core/src/key_switch/rlwe.rs:123-131): a[0] = -a[0], a[1..] reversed, then on
          // chunk c the same again, so chunk word u is -a[N - c n'] (u = 0; a[0] negated twice for
          // c = 0) or a[N - (c + 1) n' + u]; the chunk is then negated (p = -chunk) and placed at
          // every ks_stride-th slot, the ring embedding X -> X^ks_stride of the n'-word product.
          const uint32_t c = ph - 2 * n, kn = p.ks_n, ks_stride = N / kn;
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const int k = NT::natural_pos(t, v);
            W d = 0;
            if ((uint32_t)k % ks_stride == 0) {
              const uint32_t u = (uint32_t)k / ks_stride;
              W w;
              if (u != 0)
                w = acc_a[N - (c + 1) * kn + u];
              else
                w = c == 0 ? F::neg_ref(F::neg_ref(acc_a[0])) : F::neg_ref(acc_a[N - c * kn]);
              d = F::value(F::neg_ref(w));
            }
            ebuf[v * T + t] = d;
          }
        }
      }
      const uint32_t L = ks ? p.ks_len : p.len;
      const uint32_t bits = ks ? p.ks_bits : p.bits;
      const uint64_t mask = (1ULL << bits) - 1;
      // multiply-accumulate of one transformed digit against its key chunk(s): false when the
      // launch must stop
      auto mac_digit = [&](W(&x)[V]) -> bool {
        const W *k = pipe.acquire();
        if (active) {
          if (fold_due<F>(nprod)) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
              F::acc_fold(acc_x[v]);
              F::acc_fold(acc_y[v]);
              if constexpr (TERN) {
                F::acc_fold(acc_x1[v]);
                F::acc_fold(acc_y1[v]);
              }
            }
          }
#pragma unroll
          for (int v = 0; v < V; ++v) {
            F::acc_mac(acc_x[v], x[v], k[v * T + t]);
            F::acc_mac(acc_y[v], x[v], k[N + v * T + t]);
          }
        }
        ++nprod;
        if (!pipe.release(src, t, sync)) return false;
        if constexpr (TERN) {
          if (!ks) {  // the same digit against RGSW(s_i == -1)
            const W *k1 = pipe.acquire();
            if (active) {
#pragma unroll
              for (int v = 0; v < V; ++v) {
                F::acc_mac(acc_x1[v], x[v], k1[v * T + t]);
                F::acc_mac(acc_y1[v], x[v], k1[N + v * T + t]);
              }
            }
            if (!pipe.release(src, t, sync)) return false;
          }
        }
        return true;
      };
      // DUAL, binary key: two transformed digits against their consecutive key chunks, held at once;
      // the two products of a slot share one reduction (F::acc_mac2; BABYBEAR 16384 gates, same GPU:
      // T = 64, G = 8 352.6 -> 341.8 ms, T = 128, G = 4 416.1 -> 395.4 ms)
      auto mac_pair = [&](W(&x)[V], W(&y)[V]) -> bool {
        const W *k0 = pipe.acquire();
        const W *k1 = pipe.acquire_next();
        if (active) {
#pragma unroll
          for (int v = 0; v < V; ++v) {
            F::acc_mac2(acc_x[v], x[v], k0[v * T + t], y[v], k1[v * T + t]);
            F::acc_mac2(acc_y[v], x[v], k0[N + v * T + t], y[v], k1[N + v * T + t]);
          }
        }
        nprod += 2;
        if (!pipe.release(src, t, sync)) return false;
        return pipe.release(src, t, sync);
      };
      // TRACE: digit j of E.part at step ph / 2; coefficient v T + t is in x[v]
      auto trace_digit = [&](const W(&x)[V], uint32_t j) {
        if constexpr (TRACE) {
          if (!ks && p.digits) {
            uint8_t *dd = p.digits + ((((size_t)gate * n + (ph >> 1)) * 2 + part) * p.len + j) * N;
#pragma unroll
            for (int v = 0; v < V; ++v) dd[v * T + t] = (uint8_t)x[v];
          }
        }
      };
      constexpr bool DUAL = boot_dual<F, T, G>();
      uint32_t j = 0;
      if constexpr (DUAL) {
        for (; j + 1 < L; j += 2) {
          W x[V], y[V];
          if (active) {
            digits<W, V, T>(x, ebuf, t, j * bits, (uint32_t)mask);
            digits<W, V, T>(y, ebuf, t, (j + 1) * bits, (uint32_t)mask);
            trace_digit(x, j);
            trace_digit(y, j + 1);
            NT::forward_small2(x, y, xbuf, ping, s_tw, t, sync);
          }
          if constexpr (!TERN && !F::WIDE) {
            if (!mac_pair(x, y)) goto aborted;
          } else {
            if (!mac_digit(x) || !mac_digit(y)) goto aborted;
          }
        }
      }
      for (; j < L; ++j) {
        W x[V];
        if (active) {
          digits<W, V, T>(x, ebuf, t, j * bits, (uint32_t)mask);
          trace_digit(x, j);
          NT::forward_small(x, xbuf, ping, s_tw, t, sync);
        }
        if (!mac_digit(x)) goto aborted;
      }
      if (KSC ? (ks ? ph + 1 < phases : part == 0) : (part == 0 && !ks)) continue;
      if constexpr (TERN) {
        if (!ks) {
          // Ternary step (ternary.rs:78-114): the evaluation key RGSW_0 + RGSW_1 * (-X^-a) is
          // linear in the RGSWs, so ACC += INTT(acc_0) + (-X^(2N - a)) * INTT(acc_1) per
          // polynomial. h even: INTT of the pair-1 sum into ebuf; h odd: ACC += INTT(pair-0 sum)
          // minus ebuf rotated by d = 2N - a (negacyclic). The chain acc_x1, acc_x, acc_y1, acc_y
          // shifts one place per h.
          const int d = (int)(2 * N) - (int)ms[ph >> 1];
#pragma unroll 1
          for (int h = 0; h < 4; ++h) {
            if (active) {
              W f[V];
#pragma unroll
              for (int v = 0; v < V; ++v) f[v] = F::acc_value(acc_x1[v], off_br);
              NT::inverse(f, xbuf, ping, s_itw, t, sync);
              if ((h & 1) == 0) {
#pragma unroll
                for (int v = 0; v < V; ++v) ebuf[NT::natural_pos(t, v)] = F::canon(f[v]);
              } else {
                W *y = h == 1 ? acc_a : acc_b;
#pragma unroll
                for (int v = 0; v < V; ++v) {
                  const int k = NT::natural_pos(t, v);
                  const int s = k - d;
                  W rot;
                  if (s >= 0) {
                    rot = ebuf[s];
                  } else if (s >= -N) {
                    rot = F::neg_ref(ebuf[s + N]);
                  } else {
                    rot = ebuf[s + 2 * N];
                  }
                  y[k] = F::add(y[k], F::sub(F::canon(f[v]), rot));
                }
              }
#pragma unroll
              for (int v = 0; v < V; ++v) {
                acc_x1[v] = acc_x[v];
                acc_x[v] = acc_y1[v];
                acc_y1[v] = acc_y[v];
                F::acc_clear(acc_y[v]);
              }
            }
            sync();  // ebuf written (h even) or read (h odd) by the whole group
          }
          nprod = 0;
          continue;
        }
      }
      // Inverse transforms of both accumulators through one call site: h = 0 handles acc_x (the
      // a polynomial), then acc_y moves into acc_x for h = 1 (the b polynomial).
      const W off = ks ? off_ks : off_br;
      W b0 = 0;
      W *out = reinterpret_cast<W *>(job.out) + gate * lwe_words;
      if (ks && active) b0 = F::canon(F::add(acc_b[0], (W)(F::P >> 3)));  // evaluate.rs:52
#pragma unroll 1
      for (int h = 0; h < 2; ++h) {
        if (active) {
          W f[V];
#pragma unroll
          for (int v = 0; v < V; ++v) f[v] = F::acc_value(acc_x[v], off);
          NT::inverse(f, xbuf, ping, s_itw, t, sync);
          if (!ks) {
            W *y = h == 0 ? acc_a : acc_b;
#pragma unroll
            for (int v = 0; v < V; ++v) {
              const int k = NT::natural_pos(t, v);
              y[k] = F::add(y[k], F::canon(f[v]));  // RLWE::add_assign_element_wise
              if constexpr (TRACE)
                p.trace[(((size_t)gate * n + (ph >> 1)) * 2 + h) * N + k] = F::canon(y[k]);
            }
          } else {
            // extract_partial_lwe_locally (lattice/src/rlwe.rs:393-402): a' = [A0, -A_{N-1}, ...],
            // b' = b0 + B0; with KSC the n'-word result sits at every (N/n')-th slot and
            // a' = [A0, -A_{n'-1}, ..., -A_{n'-n+1}]
            const int kn = KSC ? (int)p.ks_n : N, ks_stride = N / kn;
#pragma unroll
            for (int v = 0; v < V; ++v) {
              const int k = NT::natural_pos(t, v);
              const W val = F::canon(f[v]);
              if (h == 0) {
                if (!KSC || k % ks_stride == 0) {
                  const int u = KSC ? k / ks_stride : k;
                  if (u == 0)
                    out[0] = val;
                  else if (u >= kn - (int)n + 1)
                    out[kn - u] = F::neg_ref(val);
                }
              } else if (k == 0) {
                out[n] = F::canon(F::add(val, b0));
              }
            }
          }
#pragma unroll
          for (int v = 0; v < V; ++v) {
            acc_x[v] = acc_y[v];
            F::acc_clear(acc_y[v]);
          }
        }
      }
      nprod = 0;
      sync();
    }
  }

  // Every thread ends here, including the groups that stopped on an abort, so that copies still
  // in flight into shared memory are waited for before the CTA exits.
aborted:
  __syncthreads();
  if (*s_abort) pipe.drain();
}

// ------------------------------------------------------------------------------------------
// Latency form: one gate per CTA, its gadget digits spread over D thread groups
// ------------------------------------------------------------------------------------------

// Threads per group of bootstrap_dp_kernel with C CTAs per gate, over keys laid out for KT threads:
// the key layout's width, except in the 32-bit fields' cluster form, whose groups transform a digit
// with 128 threads (a 64-thread key layout is then read in the 128-thread slot order), so that
// BabyBear's 2l = 8 digits give each of the 2 x 4 groups of a 2-CTA cluster one digit.
template <class W, int KT, int C = 1>
__host__ __device__ constexpr int dp_group_threads() {
  return sizeof(W) == 4 && C > 1 ? 128 : KT;
}

// Groups per CTA of bootstrap_dp_kernel: as many groups as 512 threads hold (the 64-bit transforms
// keep about 128 registers a thread, so 4 groups of 128 or of 64).
template <class W, int KT, int C = 1>
__host__ __device__ constexpr int dp_groups() {
  return sizeof(W) == 8 ? 4 : 512 / dp_group_threads<W, KT, C>();
}

// Words per thread of the half-CTA groups (D/2 groups) that sum and inverse-transform the a and b
// polynomials in bootstrap_dp_kernel.
template <class W, int N, int KT, int C = 1>
__host__ __device__ constexpr int dp_wide_words() {
  return N / (dp_groups<W, KT, C>() / 2 * dp_group_threads<W, KT, C>());
}

// Shared memory of bootstrap_dp_kernel: twiddle tables (forward, inverse of the half-CTA layout;
// N entries each), the accumulator (2N), the decomposition sources E.a and E.b (2N), per group two exchange
// buffers (2N) that also carry the group's partial sums, with KST the key words of its digit (2N), in a
// cluster two buffers of the CTA's partial sums that the other CTAs read (2 x 2N), and the
// modulus-switched input.
template <class W, int N, int D, int C, bool KST>
__host__ __device__ constexpr size_t dp_smem_bytes(uint32_t n) {
  return sizeof(W) * (size_t)(2 * tw_words<W>() + 4 + (KST ? 4 : 2) * D + (C > 1 ? 4 : 0)) * N +
         sizeof(uint16_t) * (size_t)((n + 8) & ~7u);
}

// Cluster barrier halves (all threads of every CTA of the cluster, warp-uniform): arrive releases
// this thread's shared-memory writes and reads, wait acquires every other thread's.
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// Generic address of the same shared-memory word in CTA `rank` of the cluster.
template <class W>
__device__ __forceinline__ const W *cluster_peer(const W *p, uint32_t rank) {
  uint64_t in = (uint64_t)p, out;
  asm volatile("mapa.u64 %0, %1, %2;" : "=l"(out) : "l"(in), "r"(rank));
  return reinterpret_cast<const W *>(out);
}

// The same bootstrap as bootstrap_kernel (binary LWE key, one key-switching chunk) with the
// latency of one gate cut instead of the cost of many: per blind-rotation step the 2l digit
// polynomials of E = ACC (X^r - 1) go to D groups (digit d to group d mod D), each transforms its
// digits and multiply-accumulates them with their key rows, the groups' partial sums meet in shared
// memory, and the two halves of the CTA, each one group of D/2 * T threads, inverse-transform the
// a and b sums and add them to the accumulator. The key switch spreads its l_ks digits the same
// way. Used for launches of at most one gate per SM.
//
// KST: every thread copies its key words of a digit into shared memory (cp.async) before the
// digit's transform and waits for them after it; otherwise the key words are read from global
// memory after the transform (with an L2 prefetch before it for the 64-bit keys, which exceed L2).
//
// C > 1: a cluster of C CTAs (C SMs) per gate. The digits go to the C * D groups of the cluster;
// each CTA sums its groups' partials, the CTAs read each other's sums through distributed shared
// memory, and every CTA inverse-transforms the total itself, so every CTA keeps the same
// accumulator without a broadcast. One cluster barrier per phase, after the CTA sums are written:
// the sums alternate between two buffers, and a CTA passes phase k's barrier only after every CTA
// arrived there, that is after every CTA finished reading phase k-1's sums, so the buffer written
// in phase k+1 is free. A last barrier keeps every CTA until the others have read its sums.
//
// KSC: the key switch in ks_chunks chunks of n' < N words (as bootstrap_kernel's KSC): digit d of
// the key-switch phase is digit d mod l_ks of chunk d / l_ks, whose source words are formed from
// the accumulator where the digit is taken, and the extraction reads every (N/n')-th coefficient.
//
// KT < T: the key rows are laid out for KT-thread groups (word v KT + t' holds slot t' (N/KT) + v);
// a group of T threads reads the same slots in its own order.
//
// TERN (ternary LWE key, one CTA per gate): in a blind-rotation step the first half of the groups
// multiplies all 2l digits by RGSW(s_i == 1), the second half by RGSW(s_i == -1), so no group
// holds two sets of sums. Each CTA half then reads both pairs' sums of its polynomial,
// inverse-transforms the pair-1 sum into a stage and the pair-0 sum in registers, and adds
// INTT(pair-0 sum) - X^(2N - a_i) INTT(pair-1 sum) to the accumulator: the evaluation key
// RGSW_0 + RGSW_1 (-X^-a_i) of bootstrap_kernel's TERN step (ternary.rs:78-114).
template <class F, int LOGN, int T, int D, int C = 1, bool KSC = false, bool TERN = false, int KT = T,
          bool KST = false>
__global__ void __launch_bounds__(D * T, 1) bootstrap_dp_kernel(const BootParams<typename F::W> p) {
  using W = typename F::W;
  using NT = GroupNtt<F, LOGN, T>;
  constexpr int N = 1 << LOGN, V = NT::V, NT_ALL = D * T;
  static_assert(D >= 2 && D % 2 == 0, "two half-CTA groups transform the a and b sums");
  static_assert(!TERN || (C == 1 && D >= 4), "ternary keys: one CTA per gate, a pair per CTA half");
  static_assert(KT <= T && T % KT == 0, "a group reads a key layout of at most its own width");
  constexpr int TW = D / 2 * T;  // threads of a half-CTA group
  using NW = GroupNtt<F, LOGN, TW>;
  constexpr int VW = NW::V;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int TWN = N * F::TW_WORDS;
  W *s_tw = reinterpret_cast<W *>(smem_raw);
  W *s_itw_w = s_tw + TWN;
  W *acc_a = s_itw_w + TWN;
  W *acc_b = acc_a + N;
  W *s_e = acc_b + N;  // E.a then E.b (the key switch: -acc.a), natural order
  W *s_x = s_e + 2 * N;
  W *s_k = s_x + D * 2 * N;  // KST, per group: its digit's key words at (v T + t) and N + (v T + t)
  W *s_cp = s_k + (KST ? D * 2 * N : 0);  // C > 1: this CTA's partial sums (a then b) x 2, read by the cluster
  uint16_t *ms = reinterpret_cast<uint16_t *>(s_cp + (C > 1 ? 4 * N : 0));

  const int tid = threadIdx.x, g = tid / T, t = tid % T;
  // key word of the group's (t, v): slot t V + v sits at (slot % (N/KT)) KT + slot / (N/KT)
  constexpr int KM = T / KT;
  const int kbase = (t % KM) * V * KT + t / KM;
  const uint32_t rank = C > 1 ? cluster_rank() : 0;
  const int gg = (int)rank * D + g;  // the group's index in the cluster (digits gg, gg + C D, ...)
  uint32_t cp_turn = 0;              // C > 1: which sum buffer this phase writes
  for (int i = tid; i < TWN; i += NT_ALL) {
    s_tw[i] = p.tw[i];
    s_itw_w[i] = p.itw_w[i];
  }
  __syncthreads();
  GroupSync<T> sync{1 + g};
  W *xbuf = s_x + g * 2 * N;
  W *kbuf = s_k + g * 2 * N;
  int ping = 0;
  // half 0 (groups 0 .. D/2-1) sums and transforms the a polynomial, half 1 the b polynomial
  const int half = g / (D / 2), tw = tid % TW;
  GroupSync<TW> wsync{D + 1 + half};
  W *wbuf = half == 0 ? s_e : s_x;  // free once every partial sum has been read
  int ping_w = 0;

  const uint32_t n = p.n, L = p.len, two_n = 2 * N;
  // products each group accumulates per phase (digits gg, gg + C D, ...), for the lazy offsets
  const uint32_t nd_br = 2 * L, nd_ks = (KSC ? p.ks_chunks : 1) * p.ks_len;
  // TERN: a blind-rotation step's digits go to the D/2 groups of the CTA half of the group's pair
  const uint32_t br_lanes = TERN ? D / 2 : C * D;
  const uint32_t br_first = TERN ? (uint32_t)(g % (D / 2)) : (uint32_t)gg;
  const uint32_t br_pair = TERN ? (uint32_t)(g / (D / 2)) : 0;
  const uint32_t my_br = br_first < nd_br ? (nd_br - 1 - br_first) / br_lanes + 1 : 0;
  const uint32_t my_ks = (uint32_t)gg < nd_ks ? (nd_ks - 1 - gg) / (C * D) + 1 : 0;
  const W off_br = F::acc_offset(my_br);
  const W off_ks = F::acc_offset(my_ks);

  for (uint32_t gi = blockIdx.x / C; gi < p.total_batches; gi += gridDim.x / C) {
    int jx = 0;
    while (jx + 1 < p.njobs && p.jobs[jx + 1].first_batch <= gi) ++jx;
    const GateJob &job = p.jobs[jx];
    const uint32_t gate = gi - job.first_batch;  // one gate per batch
    const size_t lwe_words = (size_t)n + 1;

    // ---- input combine + modulus switch (as bootstrap_kernel) ----
    {
      const W *c0 = reinterpret_cast<const W *>(job.in0) + gate * lwe_words;
      const W *c1 = job.in1 ? reinterpret_cast<const W *>(job.in1) + gate * lwe_words : nullptr;
      const W *c2 = job.in2 ? reinterpret_cast<const W *>(job.in2) + gate * lwe_words : nullptr;
      for (uint32_t k = tid; k <= n; k += NT_ALL) {
        W c = small_mul<F>(c0[k], job.s0);
        if (c1) c = F::canon(F::add(c, small_mul<F>(c1[k], job.s1)));
        if (c2) c = F::canon(F::add(c, small_mul<F>(c2[k], job.s2)));
        if (k == n) c = F::canon(F::add(c, (W)job.add_b));
        ms[k] = (uint16_t)modswitch<F>(c, two_n);
      }
    }
    __syncthreads();
    // ---- ACC = (0, LUT * X^{-b}) (fhe_core/src/blind_rotation/rlwe/binary.rs:40-64) ----
    {
      const uint32_t bt = ms[n];
      const int e = bt ? (int)(two_n - bt) : 0;
      const W *lut = reinterpret_cast<const W *>(job.lut);
      for (int k = tid; k < N; k += NT_ALL) {
        int s = k - e;
        bool neg = false;
        if (s < 0) {
          s += N;
          neg = true;
          if (s < 0) {
            s += N;
            neg = false;
          }
        }
        W f = lut ? F::canon(lut[s]) : (W)((uint32_t)s < job.lut_mid ? job.lut_lo : job.lut_hi);
        acc_a[k] = 0;
        acc_b[k] = neg ? F::neg_ref(f) : f;
      }
    }
    __syncthreads();

    // ---- phases 0 .. n-1: blind-rotation steps; phase n: key switch ----
    for (uint32_t ph = 0; ph <= n; ++ph) {
      const bool ks = ph == n;
      if (!ks) {
        // E = ACC * (X^r - 1) in the reference's representation (lattice/src/rlwe.rs:437-487)
        const int r = (int)ms[ph];
        for (int q = tid; q < 2 * N; q += NT_ALL) {
          const int k = q & (N - 1);
          const W *y = q < N ? acc_a : acc_b;
          const int s = k - r;
          W rot;
          if (s >= 0) {
            rot = y[s];
          } else if (s >= -N) {
            rot = F::neg_ref(y[s + N]);
          } else {
            rot = y[s + 2 * N];
          }
          s_e[q] = F::value(F::sub(rot, y[k]));
        }
      } else if (!KSC) {
        // p = -acc.a (lattice/src/rlwe.rs:1147-1166)
        for (int k = tid; k < N; k += NT_ALL) s_e[k] = F::value(F::neg_ref(acc_a[k]));
      }
      __syncthreads();
      const uint32_t nd = ks ? nd_ks : nd_br;
      const uint32_t bits = ks ? p.ks_bits : p.bits;
      const uint32_t mask = (1u << bits) - 1;
      using FA = FewAcc<F>;
      typename FA::A ax[V], ay[V];
#pragma unroll
      for (int v = 0; v < V; ++v) {
        FA::clear(ax[v]);
        FA::clear(ay[v]);
      }
      uint32_t nprod = 0;  // products in ax / ay since their last fold
      for (uint32_t d = ks ? (uint32_t)gg : br_first; d < nd; d += ks ? C * D : br_lanes) {
        const uint32_t part = ks ? 0 : d / L, j = ks ? d % p.ks_len : d % L;
        const W *krow = ks     ? p.ksk + (size_t)d * 2 * N
                        : TERN ? p.bsk + ((((size_t)ph * 2 + br_pair) * 2 + part) * L + j) * 2 * N
                               : p.bsk + ((size_t)(ph * 2 + part) * L + j) * 2 * N;
        if constexpr (KST) {
          // the thread's key words of this digit, copied to its own slots of the group's key stage
          // while the digit is decomposed and transformed; the thread reads back only the words it
          // copied, after its own wait
#pragma unroll
          for (int v = 0; v < V; ++v) {
            cp_async_word(kbuf + v * T + t, krow + kbase + v * KT);
            cp_async_word(kbuf + N + v * T + t, krow + N + kbase + v * KT);
          }
          cp_async_commit();
        } else if constexpr (sizeof(W) == 8) {
          // Goldilocks keys (191-310 MB) exceed L2: start the key row's way from HBM into L2 while
          // the digit transform runs (the loads below come after the transform's barriers)
#pragma unroll
          for (int v = 0; v < V; ++v) {
            asm volatile("prefetch.global.L2 [%0];" ::"l"(krow + kbase + v * KT));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(krow + N + kbase + v * KT));
          }
        }
        W x[V];
        if (KSC && ks) {
          // chunk c of the permuted -acc.a (fhe_core/src/key_switch/rlwe.rs:123-131), word u at
          // slot u * stride: -a[N - c n'] for u = 0 (a[0] negated twice for c = 0), else
          // a[N - (c + 1) n' + u], then negated
          const uint32_t c = d / p.ks_len, kn = p.ks_n, stride = N / kn;
          W e[V];
#pragma unroll
          for (int v = 0; v < V; ++v) {
            const uint32_t k = (uint32_t)NT::natural_pos(t, v);
            W w = 0;
            if (k % stride == 0) {
              const uint32_t u = k / stride;
              const W a = u != 0 ? acc_a[N - (c + 1) * kn + u]
                                 : (c == 0 ? F::neg_ref(F::neg_ref(acc_a[0])) : F::neg_ref(acc_a[N - c * kn]));
              w = F::value(F::neg_ref(a));
            }
            e[v] = w;
          }
          digits_reg<W, V>(x, e, j * bits, mask);
        } else {
          digits<W, V, T>(x, s_e + part * N, t, j * bits, mask);
        }
        NT::forward_small(x, xbuf, ping, s_tw, t, sync);
        if (fold_due_n<FA::FOLD>(nprod)) {
#pragma unroll
          for (int v = 0; v < V; ++v) {
            FA::fold(ax[v]);
            FA::fold(ay[v]);
          }
        }
        if constexpr (KST) {
          cp_async_wait_all();
#pragma unroll
          for (int v = 0; v < V; ++v) {
            FA::mac(ax[v], x[v], kbuf[v * T + t]);
            FA::mac(ay[v], x[v], kbuf[N + v * T + t]);
          }
        } else {
#pragma unroll
          for (int v = 0; v < V; ++v) {
            FA::mac(ax[v], x[v], krow[kbase + v * KT]);
            FA::mac(ay[v], x[v], krow[N + kbase + v * KT]);
          }
        }
        ++nprod;
      }
      sync();  // the group's last exchange has been read: its buffers take the partial sums
      {
        const W off = ks ? off_ks : off_br;
#pragma unroll
        for (int v = 0; v < V; ++v) {
          xbuf[v * T + t] = FA::value(ax[v], off);
          xbuf[N + v * T + t] = FA::value(ay[v], off);
        }
      }
      __syncthreads();
      if constexpr (TERN) {
        if (!ks) {
          // the half's polynomial: both pairs' sums (groups [0, D/2) and [D/2, D)) in its layout
          W f0[VW], f1[VW];
#pragma unroll
          for (int vw = 0; vw < VW; ++vw) {
            const int slot = tw * VW + vw;
            const int at = half * N + (slot % V) * T + slot / V;
            W s0 = s_x[at], s1 = s_x[(D / 2) * 2 * N + at];
#pragma unroll 1
            for (int h = 1; h < D / 2; ++h) {
              s0 = F::add(s0, s_x[h * 2 * N + at]);
              s1 = F::add(s1, s_x[(D / 2 + h) * 2 * N + at]);
            }
            f0[vw] = s0;
            f1[vw] = s1;
          }
          __syncthreads();  // every partial read: the group buffers are free
          // INTT(pair-1 sum) to a stage in group 1's buffer (the halves' exchange buffers are E's
          // and group 0's), then INTT(pair-0 sum) in registers
          W *st = s_x + 2 * N + half * N;
          NW::inverse(f1, wbuf, ping_w, s_itw_w, tw, wsync);
#pragma unroll
          for (int vw = 0; vw < VW; ++vw) st[NW::natural_pos(tw, vw)] = F::canon(f1[vw]);
          NW::inverse(f0, wbuf, ping_w, s_itw_w, tw, wsync);
          wsync();  // the stage is complete
          W *y = half == 0 ? acc_a : acc_b;
          const int dr = (int)two_n - (int)ms[ph];
#pragma unroll
          for (int vw = 0; vw < VW; ++vw) {
            const int k = NW::natural_pos(tw, vw);
            const int sidx = k - dr;
            W rot;
            if (sidx >= 0) {
              rot = st[sidx];
            } else if (sidx >= -N) {
              rot = F::neg_ref(st[sidx + N]);
            } else {
              rot = st[sidx + 2 * N];
            }
            y[k] = F::add(y[k], F::sub(F::canon(f0[vw]), rot));
          }
          __syncthreads();
          continue;
        }
      }
      {
        // the half's sum over all groups' partials, read in its own layout: slot tw*VW + vw sits at
        // (slot % V) * T + slot / V in a group's buffer
        W f[VW];
        if constexpr (C == 1) {
#pragma unroll
          for (int vw = 0; vw < VW; ++vw) {
            const int slot = tw * VW + vw;
            const int at = half * N + (slot % V) * T + slot / V;
            W sum = s_x[at];
#pragma unroll 1
            for (int h = 1; h < D; ++h) sum = F::add(sum, s_x[h * 2 * N + at]);
            f[vw] = sum;
          }
          __syncthreads();  // every partial read: the exchange buffers are free
        } else {
          W *cp = s_cp + (cp_turn & 1) * 2 * N;
          ++cp_turn;
          for (int q = tid; q < 2 * N; q += NT_ALL) {
            W sum = s_x[q];
#pragma unroll 1
            for (int h = 1; h < D; ++h) sum = F::add(sum, s_x[h * 2 * N + q]);
            cp[q] = sum;
          }
          cluster_arrive();
          cluster_wait();  // every CTA's sums are written (and this CTA's group buffers are read)
#pragma unroll
          for (int vw = 0; vw < VW; ++vw) {
            const int slot = tw * VW + vw;
            const int at = half * N + (slot % V) * T + slot / V;
            // the same order of terms in every CTA, so every CTA forms the same words
            W sum = cluster_peer(cp, 0)[at];
#pragma unroll 1
            for (uint32_t r = 1; r < (uint32_t)C; ++r) sum = F::add(sum, cluster_peer(cp, r)[at]);
            f[vw] = sum;
          }
        }
        NW::inverse(f, wbuf, ping_w, s_itw_w, tw, wsync);
        if (!ks) {
          W *y = half == 0 ? acc_a : acc_b;
          // the accumulator trace of vfhe's bootstrap (vfhe/src/bfhe/evaluate.rs:47-141), written
          // by one CTA of the cluster (every CTA forms the same words)
          W *tr = p.trace != nullptr && rank == 0 ? p.trace + ((size_t)ph * 2 + half) * N : nullptr;
#pragma unroll
          for (int vw = 0; vw < VW; ++vw) {
            const int k = NW::natural_pos(tw, vw);
            y[k] = F::add(y[k], F::canon(f[vw]));  // RLWE::add_assign_element_wise
            if (tr) tr[k] = F::canon(y[k]);
          }
        } else if (rank == 0) {
          // extract_partial_lwe_locally (lattice/src/rlwe.rs:393-402); b' = acc.b[0] + Q/8 + B0; with
          // KSC the n'-word result sits at every (N/n')-th slot
          W *out = reinterpret_cast<W *>(job.out) + gate * lwe_words;
          const int kn = KSC ? (int)p.ks_n : N, ks_stride = N / kn;
#pragma unroll
          for (int vw = 0; vw < VW; ++vw) {
            const int k = NW::natural_pos(tw, vw);
            const W val = F::canon(f[vw]);
            if (half == 0) {
              if (!KSC || k % ks_stride == 0) {
                const int u = KSC ? k / ks_stride : k;
                if (u == 0)
                  out[0] = val;
                else if (u >= kn - (int)n + 1)
                  out[kn - u] = F::neg_ref(val);
              }
            } else if (k == 0) {
              const W b0 = F::canon(F::add(acc_b[0], (W)(F::P >> 3)));  // evaluate.rs:52
              out[n] = F::canon(F::add(val, b0));
            }
          }
        }
      }
      __syncthreads();
    }
  }
  if constexpr (C > 1) {  // no CTA leaves while another may still read its shared memory
    cluster_arrive();
    cluster_wait();
  }
}

// ------------------------------------------------------------------------------------------
// Integer-pipe modmul throughput probe (roofline denominator): every thread runs 8 independent
// chains of F::mul on register operands; the result is stored so nothing is dead code.
// ------------------------------------------------------------------------------------------
template <class F>
__global__ void __launch_bounds__(256) modmul_probe_kernel(typename F::W *out, uint32_t iters,
                                                            typename F::W seed) {
  using W = typename F::W;
  W x[8];
  const W w = (W)(seed | 3u);
#pragma unroll
  for (int i = 0; i < 8; ++i) x[i] = F::canon((W)(seed + threadIdx.x * 8u + i + blockIdx.x * 977u));
  for (uint32_t it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = F::mul(x[i], w);
  }
  W acc = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) acc ^= x[i];
  out[blockIdx.x * (size_t)blockDim.x + threadIdx.x] = acc;
}

}  // namespace hb
