// hb_ntt.cuh -- negacyclic NTT/INTT of one polynomial by a group of T threads, V = N/T words per
// thread held in registers, exchanges through a swizzled shared-memory buffer between passes.
//
// Forward: Cooley-Tukey with merged psi powers (natural order in, bit-reversed slot order out).
// Inverse: Gentleman-Sande (bit-reversed slot order in, natural order out), without the final
// N^-1 scaling (callers fold N^-1 into the key material they multiply by, or scale explicitly).
// This replaces concrete-ntt's Plan::fwd / Plan::inv + normalize behind
// AbstractNTT::{transform_slice, inverse_transform_slice} (algebra/src/transformation/concrete.rs:116-148).
//
// Register layout of a pass with "low" position `lo`: thread t, register v holds element
//   idx(t, v, lo) = ((t >> lo) << (lo + LOGV)) | (v << lo) | (t & ((1 << lo) - 1)).
// Forward passes cover butterfly bits from the top down (LOGV bits per pass); the last forward
// pass and the first inverse pass share layout lo = 0 (thread t holds slots t*V .. t*V+V-1), so the
// pointwise multiply-accumulate between them needs no exchange.
#pragma once

#include "hb_field.cuh"

namespace hb {

__host__ __device__ constexpr int ilog2c(int x) { return x <= 1 ? 0 : 1 + ilog2c(x >> 1); }

// Words per entry of a twiddle table for word type W: the 32-bit fields keep a Shoup quotient
// beside each twiddle (Mont32::Tw), Goldilocks the twiddle alone.
template <class W>
__host__ __device__ constexpr int tw_words() {
  return sizeof(W) == 4 ? 2 : 1;
}

// Synchronisation of one thread group: a warp (T == 32) or a named barrier (T > 32).
template <int T>
struct GroupSync {
  int bar_id;
  __device__ __forceinline__ void operator()() const {
    if constexpr (T == 32) {
      __syncwarp();
    } else {
      asm volatile("bar.sync %0, %1;" ::"r"(bar_id), "r"(T) : "memory");
    }
  }
};

// PP: two exchange buffers used in turn (one barrier per exchange); otherwise one buffer and a
// second barrier after each exchange's reads.
template <class F, int LOGN, int T, bool PP = true>
struct GroupNtt {
  using W = typename F::W;
  using TwT = typename F::Tw;  // table entry: F::TW_WORDS words (the 32-bit fields add a Shoup quotient)
  static constexpr int TW_WORDS = F::TW_WORDS;
  static_assert(TW_WORDS == tw_words<W>() && sizeof(TwT) == TW_WORDS * sizeof(W), "twiddle entry layout");
  static constexpr int N = 1 << LOGN;
  static constexpr int V = N / T;
  static constexpr int LOGV = ilog2c(V);
  static constexpr int LOGT = LOGN - LOGV;
  static constexpr int SWZ = sizeof(W) == 8 ? 15 : 31;
  static_assert((1 << LOGV) == V && V >= 2, "V must be a power of two >= 2");
  static_assert(T % 32 == 0, "groups are whole warps");

  // Physical slot of element q in an exchange buffer: an XOR swizzle that makes every pass layout
  // conflict-free (half-warp distinct banks for 8-byte words, warp-distinct for 4-byte words).
  __device__ __forceinline__ static int phys(int q) { return q ^ ((q >> LOGV) & SWZ); }

  template <int LO>
  __device__ __forceinline__ static int idx(int t, int v) {
    return ((t >> LO) << (LO + LOGV)) | (v << LO) | (t & ((1 << LO) - 1));
  }

  // Natural-order position held by (t, v) at the forward input / inverse output layout.
  __device__ __forceinline__ static int natural_pos(int t, int v) { return v * T + t; }
  // Slot held by (t, v) at the forward output / inverse input layout.
  __device__ __forceinline__ static int slot_pos(int t, int v) { return t * V + v; }

  // phys is XOR-linear and idx(t, v) = idx(t, 0) ^ (v << LO) (disjoint bits), so
  // phys(idx(t, v)) = phys(idx(t, 0)) ^ phys(v << LO): a per-thread base and a compile-time constant.
  __host__ __device__ static constexpr int cphys(int q) { return q ^ ((q >> LOGV) & SWZ); }

  template <int LO_FROM, int LO_TO>
  __device__ __forceinline__ static void exchange(W (&x)[V], W *buf, int t, const GroupSync<T> &sync) {
    const int pf = phys(idx<LO_FROM>(t, 0));
    const int pt = phys(idx<LO_TO>(t, 0));
#pragma unroll
    for (int v = 0; v < V; ++v) buf[pf ^ cphys(v << LO_FROM)] = x[v];
    sync();
#pragma unroll
    for (int v = 0; v < V; ++v) x[v] = buf[pt ^ cphys(v << LO_TO)];
  }

  // Twiddle tables (N entries of F::Tw, N * F::TW_WORDS words) are stored stage by stage; within
  // the 2^S entries of a stage, entry high * K + k (the k-th distinct twiddle of the threads whose
  // bits above the pass are `high`) sits at high + k * (2^S / K), so the loads of a warp are
  // broadcasts or consecutive entries (build_tables in hb_api.cu writes this layout).

  __host__ __device__ static constexpr int brvc(int x, int bits) {
    int r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1) << (bits - 1 - i);
    return r;
  }
  // Exponent E with psi^brv(2^S + k) = 2^E when the tables' psi satisfies psi^(N/32) = 8
  // (brv(2^S + k) is a multiple of N/32 for S <= 4).
  template <int S, int k>
  __host__ __device__ static constexpr int pow2_exponent() {
    return (int)((96LL * brvc((1 << S) + k, LOGN)) >> LOGN);
  }
  // Stage S of the first forward pass (layout LO = LOGT, where t >> LO = 0 for every thread): the
  // k-th twiddle is psi^brv(2^S + k), a compile-time power of two for S <= 4.
  template <int RB, int S, int k>
  __device__ __forceinline__ static void pow2_stage(W (&x)[V]) {
    constexpr int K = V >> (RB + 1);
    if constexpr (k < K) {
      static_assert(S >= 0 && S <= 4 && ((96LL * brvc((1 << S) + k, LOGN)) & (N - 1)) == 0,
                    "twiddle is not a power of two");
      constexpr int E = pow2_exponent<S, k>();
#pragma unroll
      for (int l = 0; l < (1 << RB); ++l) {
        const int v = (k << (RB + 1)) | l;
        F::template ct_pow2<E>(x[v], x[v | (1 << RB)]);
      }
      pow2_stage<RB, S, k + 1>(x);
    }
  }

  // Radix-8 passes (fields with power-of-two eighth roots of unity, V = 8). The three stages of a
  // pass act on groups of 8 elements at stride L/8 inside a block of length L whose modulus is
  // X^L - theta^8, theta = psi^brv(2^(S0+2) + 4m) for block m of the pass's first stage S0. They
  // equal one pre-multiplication of element k by theta^k (7 products) followed by an 8-point DFT
  // whose twiddles are the eighth roots of unity 2^24, 2^48, 2^72 (shifts), with the result of
  // frequency brv3(p) at position p. The inverse pass is the transposed form: an 8-point inverse
  // DFT on the bit-reversed group, then a post-multiplication by theta^-k. The tables hold theta^k
  // (theta^-k) at 2^S0 + (k - 1) 2^S0 + m (build_tables in hb_api.cu writes them).
  static constexpr bool R8 = F::RADIX8 && LOGV == 3;
  __host__ __device__ static constexpr int brv3(int p) { return ((p & 1) << 2) | (p & 2) | ((p >> 2) & 1); }
  // (u, v) -> (u + v, u - v) for a canonical v.
  __device__ __forceinline__ static void bf(W &u, W &v) {
    const W a = u;
    u = F::add_c(a, v);
    v = F::sub_c(a, v);
  }
  __device__ __forceinline__ static void bf_canon(W &u, W &v) {
    v = F::canon(v);
    bf(u, v);
  }
  // (u, v) -> (u - 2^E v, u + 2^E v): the twiddle -2^E = 2^(E + 96).
  template <int E>
  __device__ __forceinline__ static void bf_negpow2(W &u, W &v) {
    const W s = F::template mul_pow2<E>(v);
    const W a = u;
    u = F::sub_c(a, s);
    v = F::add_c(a, s);
  }

  template <int LO, int S0>
  __device__ __forceinline__ static void fwd_r8(W (&x)[V], const W *__restrict__ tw, int t) {
    const W *th = tw + (1 << S0) + (t >> LO);
    W b[8];
    b[0] = x[0];
#pragma unroll
    for (int p = 1; p < 8; ++p) b[p] = F::mul(x[brv3(p)], th[(brv3(p) - 1) << S0]);
    // 8-point DFT, decimation in time: bit-reversed input, natural output.
#pragma unroll
    for (int i = 0; i < 4; ++i) bf(b[2 * i], b[2 * i + 1]);  // b[odd] are products (canonical)
#pragma unroll
    for (int blk = 0; blk < 8; blk += 4) {
      bf_canon(b[blk], b[blk + 2]);
      F::template ct_pow2<48>(b[blk + 1], b[blk + 3]);
    }
    bf_canon(b[0], b[4]);
    F::template ct_pow2<24>(b[1], b[5]);
    F::template ct_pow2<48>(b[2], b[6]);
    F::template ct_pow2<72>(b[3], b[7]);
#pragma unroll
    for (int p = 0; p < 8; ++p) x[p] = b[brv3(p)];
  }

  template <int LO, int S0>
  __device__ __forceinline__ static void inv_r8(W (&x)[V], const W *__restrict__ itw, int t) {
    const W *th = itw + (1 << S0) + (t >> LO);
    // 8-point inverse DFT (twiddles 2^-24 = -2^72, 2^-48 = -2^48, 2^-72 = -2^24), decimation in
    // time: the bit-reversed group in, natural order out.
#pragma unroll
    for (int i = 0; i < 4; ++i) bf_canon(x[2 * i], x[2 * i + 1]);
#pragma unroll
    for (int blk = 0; blk < 8; blk += 4) {
      bf_canon(x[blk], x[blk + 2]);
      bf_negpow2<48>(x[blk + 1], x[blk + 3]);
    }
    bf_canon(x[0], x[4]);
    bf_negpow2<72>(x[1], x[5]);
    bf_negpow2<48>(x[2], x[6]);
    bf_negpow2<24>(x[3], x[7]);
#pragma unroll
    for (int k = 1; k < 8; ++k) x[k] = F::mul(x[k], th[(k - 1) << S0]);
  }

  // One forward (CT) stage on butterfly bit BB in a pass of layout LO. SMALL: inputs are words
  // below 2^15 (gadget digits) and this is the first stage, whose twiddle is 2^48.
  template <int LO, int BB, bool SMALL>
  __device__ __forceinline__ static void fwd_stage(W (&x)[V], const W *__restrict__ tw, int t) {
    constexpr int RB = BB - LO;
    constexpr int S = LOGN - 1 - BB;
    constexpr int K = V >> (RB + 1);  // distinct twiddles per thread in this stage
    constexpr int HIGHS = (1 << S) / K;
    if constexpr (SMALL && S == 0 && F::SMALL_FIRST_GEN != 0) {
#pragma unroll
      for (int v = 0; v < V; ++v)
        if (!((v >> RB) & 1)) F::ct_small_first(x[v], x[v | (1 << RB)]);
    } else if constexpr (F::SMALL_FIRST_GEN != 0 && LO == LOGT && S <= 4) {
      pow2_stage<RB, S, 0>(x);
    } else {
      const int base = (1 << S) + (t >> LO);
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const TwT w = reinterpret_cast<const TwT *>(tw)[base + k * HIGHS];
#pragma unroll
        for (int l = 0; l < (1 << RB); ++l) {
          const int v = (k << (RB + 1)) | l;
          F::ct(x[v], x[v | (1 << RB)], w);
        }
      }
    }
  }

  template <int LO, int BB>
  __device__ __forceinline__ static void inv_stage(W (&x)[V], const W *__restrict__ itw, int t) {
    constexpr int RB = BB - LO;
    constexpr int H = N >> (BB + 1);
    constexpr int K = V >> (RB + 1);
    constexpr int HIGHS = H / K;
    const int base = H + (t >> LO);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const TwT w = reinterpret_cast<const TwT *>(itw)[base + k * HIGHS];
#pragma unroll
      for (int l = 0; l < (1 << RB); ++l) {
        const int v = (k << (RB + 1)) | l;
        F::gs(x[v], x[v | (1 << RB)], w);
      }
    }
  }

  // Forward pass whose top butterfly bit is TOP-1; recurses to the next pass.
  template <int TOP, int BB, bool SMALL>
  __device__ __forceinline__ static void fwd_stages(W (&x)[V], const W *tw, int t) {
    constexpr int LO = TOP - LOGV > 0 ? TOP - LOGV : 0;
    constexpr int LAST = TOP - LOGV > 0 ? TOP - LOGV : 0;
    fwd_stage<LO, BB, SMALL>(x, tw, t);
    if constexpr (BB - 1 >= LAST) fwd_stages<TOP, BB - 1, SMALL>(x, tw, t);
  }
  template <int TOP, bool SMALL>
  __device__ __forceinline__ static void fwd_pass(W (&x)[V], W *buf, int &ping, const W *tw, int t,
                                                  const GroupSync<T> &sync) {
    constexpr int LO = TOP - LOGV > 0 ? TOP - LOGV : 0;
    if constexpr (R8 && TOP < LOGN && TOP - LO == 3)
      fwd_r8<LO, LOGN - TOP>(x, tw, t);
    else
      fwd_stages<TOP, TOP - 1, SMALL>(x, tw, t);
    if constexpr (LO > 0) {
      constexpr int NEXT = LO - LOGV > 0 ? LO - LOGV : 0;
      if constexpr (PP) {
        exchange<LO, NEXT>(x, buf + ping * N, t, sync);
        ping ^= 1;
      } else {
        exchange<LO, NEXT>(x, buf, t, sync);
        sync();
      }
      fwd_pass<LO, false>(x, buf, ping, tw, t, sync);
    }
  }

  // Inverse pass processing bits [B0, min(B0+LOGV, LOGN)) in layout LO = min(B0, LOGN-LOGV).
  template <int B0, int BB>
  __device__ __forceinline__ static void inv_stages(W (&x)[V], const W *itw, int t) {
    constexpr int LO = B0 < LOGN - LOGV ? B0 : LOGN - LOGV;
    constexpr int END = B0 + LOGV < LOGN ? B0 + LOGV : LOGN;
    inv_stage<LO, BB>(x, itw, t);
    if constexpr (BB + 1 < END) inv_stages<B0, BB + 1>(x, itw, t);
  }
  template <int B0>
  __device__ __forceinline__ static void inv_pass(W (&x)[V], W *buf, int &ping, const W *itw, int t,
                                                  const GroupSync<T> &sync) {
    constexpr int LO = B0 < LOGN - LOGV ? B0 : LOGN - LOGV;
    constexpr int END = B0 + LOGV < LOGN ? B0 + LOGV : LOGN;
    if constexpr (R8 && END - B0 == 3)
      inv_r8<LO, LOGN - 3 - B0>(x, itw, t);
    else
      inv_stages<B0, B0>(x, itw, t);
    if constexpr (END < LOGN) {
      constexpr int NLO = END < LOGN - LOGV ? END : LOGN - LOGV;
      if constexpr (PP) {
        exchange<LO, NLO>(x, buf + ping * N, t, sync);
        ping ^= 1;
      } else {
        exchange<LO, NLO>(x, buf, t, sync);
        sync();
      }
      inv_pass<END>(x, buf, ping, itw, t, sync);
    }
  }

  // Two independent forward transforms advanced pass by pass, so that the compiler can interleave
  // their instructions between the exchanges (each exchange of each transform as in fwd_pass).
  template <int TOP, bool SMALL>
  __device__ __forceinline__ static void fwd_pass2(W (&x)[V], W (&y)[V], W *buf, int &ping, const W *tw, int t,
                                                   const GroupSync<T> &sync) {
    constexpr int LO = TOP - LOGV > 0 ? TOP - LOGV : 0;
    if constexpr (R8 && TOP < LOGN && TOP - LO == 3) {
      fwd_r8<LO, LOGN - TOP>(x, tw, t);
      fwd_r8<LO, LOGN - TOP>(y, tw, t);
    } else {
      fwd_stages<TOP, TOP - 1, SMALL>(x, tw, t);
      fwd_stages<TOP, TOP - 1, SMALL>(y, tw, t);
    }
    if constexpr (LO > 0) {
      constexpr int NEXT = LO - LOGV > 0 ? LO - LOGV : 0;
      static_assert(PP, "paired transforms use the two exchange buffers in turn");
      exchange<LO, NEXT>(x, buf + ping * N, t, sync);
      ping ^= 1;
      exchange<LO, NEXT>(y, buf + ping * N, t, sync);
      ping ^= 1;
      fwd_pass2<LO, false>(x, y, buf, ping, tw, t, sync);
    }
  }
  // forward_small of two digit polynomials at once.
  __device__ __forceinline__ static void forward_small2(W (&x)[V], W (&y)[V], W *buf, int &ping, const W *tw,
                                                        int t, const GroupSync<T> &sync) {
    fwd_pass2<LOGN, true>(x, y, buf, ping, tw, t, sync);
  }

  // x: natural-order values at natural_pos(t, v) -> slots at slot_pos(t, v).
  // buf: the group's exchange buffers (2 N words with PP, else N).
  __device__ __forceinline__ static void forward(W (&x)[V], W *buf, int &ping, const W *tw, int t,
                                                 const GroupSync<T> &sync) {
    fwd_pass<LOGN, false>(x, buf, ping, tw, t, sync);
  }
  // Forward transform of a polynomial whose coefficients are below 2^15 (gadget digits).
  __device__ __forceinline__ static void forward_small(W (&x)[V], W *buf, int &ping, const W *tw,
                                                       int t, const GroupSync<T> &sync) {
    fwd_pass<LOGN, true>(x, buf, ping, tw, t, sync);
  }
  // x: slots at slot_pos(t, v) -> N * (natural-order values) at natural_pos(t, v).
  __device__ __forceinline__ static void inverse(W (&x)[V], W *buf, int &ping, const W *itw, int t,
                                                 const GroupSync<T> &sync) {
    inv_pass<0>(x, buf, ping, itw, t, sync);
  }
};

}  // namespace hb
