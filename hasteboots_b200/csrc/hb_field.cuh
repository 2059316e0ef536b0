// hb_field.cuh -- Goldilocks, BabyBear and DefaultFieldU32 arithmetic for sm_100a on the integer pipe.
//
// Goldilocks Q = 2^64 - 2^32 + 1 (algebra/src/modulus/goldilocks/mod.rs:9-11): 64x64->128 products
// folded with 2^64 = 2^32 - 1 and 2^96 = -1 (mod Q); values may sit anywhere in [0, 2^64) and are
// canonicalised only where a canonical value is observed (decomposition, outputs).
// The accumulator additions and negations use the reference's exact u64 operations
// (algebra/src/modulus/goldilocks/ops.rs:26-73) because a non-canonical accumulator word is
// negated by `P - x` there, and bit-exact outputs must follow that.
//
// BabyBear Q = 2^31 - 2^27 + 1 (algebra/src/modulus/baby_bear/mod.rs:11) and DefaultFieldU32
// Q = 2^27 - 2^21 + 1 (fhe_core/src/parameter.rs:286-290): data words are canonical residues;
// constants that multiply data (twiddles, keys) are stored premultiplied by R = 2^32 so a
// Montgomery product returns a canonical residue of the plain product.
#pragma once

#include <cstdint>
#include <type_traits>

#ifdef __CUDACC__
#include "hb_gl_ptx.cuh"
#endif

#ifndef HB_HD
#ifdef __CUDACC__
#define HB_HD __host__ __device__ __forceinline__
#else
#define HB_HD inline
#endif
#endif

namespace hb {

struct Goldilocks {
  using W = uint64_t;
  static constexpr W P = 0xFFFFFFFF00000001ULL;
  static constexpr W EPS = 0xFFFFFFFFULL;  // 2^64 mod P
  static constexpr int BITS = 64;
  static constexpr int FIELD_ID = 1;

  HB_HD static W canon(W x) {
#ifdef __CUDA_ARCH__
    return glx::canon(x);
#else
    return x >= P ? x - P : x;
#endif
  }

  // Fold a 128-bit value (lo + hi*2^64) to [0, 2^64).
  HB_HD static W fold(W lo, W hi) {
    const uint32_t hh = (uint32_t)(hi >> 32);
    const uint32_t hl = (uint32_t)hi;
    W t0 = lo - hh;
    if (lo < hh) t0 -= EPS;
    const W t1 = ((W)hl << 32) - hl;  // hl * (2^32 - 1)
    W r = t0 + t1;
    if (r < t1) r += EPS;
    return r;
  }
  HB_HD static W mul_lazy(W a, W b) {
#ifdef __CUDA_ARCH__
    return fold(a * b, __umul64hi(a, b));
#else
    unsigned __int128 x = (unsigned __int128)a * b;
    return fold((W)x, (W)(x >> 64));
#endif
  }
  // Product with a canonical result.
  HB_HD static W mul(W a, W b) {
#ifdef __CUDA_ARCH__
    return glx::mul_canon(a, b);
#else
    return canon(mul_lazy(a, b));
#endif
  }
  // Sum/difference where `b` is canonical (< P): one carry fix-up suffices.
  HB_HD static W add_c(W a, W b) {
#ifdef __CUDA_ARCH__
    return glx::add_c(a, b);
#else
    W s = a + b;
    if (s < b) s += EPS;
    return s;
#endif
  }
  HB_HD static W sub_c(W a, W b) {
#ifdef __CUDA_ARCH__
    return glx::sub_c(a, b);
#else
    W d = a - b;
    if (a < b) d -= EPS;
    return d;
#endif
  }
  // Sum/difference of arbitrary words: the reference's add_reduce / sub_reduce
  // (algebra/src/modulus/goldilocks/ops.rs:26-57).
  HB_HD static W add(W a, W b) {
    W s = a + b;
    W c = s < a ? EPS : 0;
    W s2 = s + c;
    if (s2 < c) s2 += EPS;
    return s2;
  }
  HB_HD static W sub(W a, W b) {
    W d = a - b;
    W c = a < b ? EPS : 0;
    W d2 = d - c;
    if (d < c) d2 -= EPS;
    return d2;
  }
  // neg_reduce (ops.rs:69-73): `P - x`, which wraps for non-canonical x.
  HB_HD static W neg_ref(W a) { return a == 0 ? 0 : P - a; }
  HB_HD static W value(W a) { return canon(a); }
  // Plain (non-Montgomery) constant: identity for Goldilocks.
  HB_HD static W to_mont(W a) { return a; }
  // NTT twiddle table entry: the twiddle itself (one word).
  using Tw = W;
  static constexpr int TW_WORDS = 1;
  HB_HD static Tw make_tw(W w) { return w; }
#ifdef __CUDA_ARCH__
  // Device hot path: PTX carry-chain arithmetic (hb_gl_ptx.cuh).
  // CT butterfly: (x, y) -> (x + w y, x - w y).
  __device__ __forceinline__ static void ct(W &x, W &y, W w) {
    const W t = glx::mul_canon(y, w);
    const W u = x;
    x = glx::add_c(u, t);
    y = glx::sub_c(u, t);
  }
  // GS butterfly: (x, y) -> (x + y, (x - y) w).
  __device__ __forceinline__ static void gs(W &x, W &y, W w) {
    const W v = glx::canon(y), u = x;
    x = glx::add_c(u, v);
    y = glx::mul_lazy(glx::sub_c(u, v), w);
  }
  template <int E>
  __device__ __forceinline__ static W mul_pow2(W y) { return glx::mul_pow2<E>(y); }
  // CT butterfly with the twiddle 2^E (compile-time 0 < E < 96): the product comes from shifts.
  template <int E>
  __device__ __forceinline__ static void ct_pow2(W &x, W &y) {
    const W t = glx::mul_pow2<E>(y);
    const W u = x;
    x = glx::add_c(u, t);
    y = glx::sub_c(u, t);
  }
  // acc += x * k.
  __device__ __forceinline__ static W mac(W acc, W x, W k) { return glx::add_c(acc, glx::mul_canon(x, k)); }
  // Accumulator of a sum of m products, reduced once at the end (glx::mac_lazy).
  struct Acc {
    W lo;
    uint32_t cnt;
  };
  __device__ __forceinline__ static void acc_clear(Acc &a) {
    a.lo = 0;
    a.cnt = 0;
  }
  __device__ __forceinline__ static void acc_mac(Acc &a, W x, W k) { glx::mac_lazy(a.lo, a.cnt, x, k); }
  __device__ __forceinline__ static void acc_mac2(Acc &a, W x, W kx, W y, W ky) {
    glx::mac_lazy(a.lo, a.cnt, x, kx);
    glx::mac_lazy(a.lo, a.cnt, y, ky);
  }
  static constexpr bool WIDE = false;  // products accumulate lazily in 96 bits, not as 64-bit sums
  // The carry count never overflows for the sums here (at most 2^32 products): no folds.
  static constexpr int FOLD = 1 << 30;
  __device__ __forceinline__ static void acc_fold(Acc &) {}
  // off = acc_offset(m) for an accumulator that took m products.
  __device__ __forceinline__ static W acc_value(const Acc &a, W off) { return glx::mac_lazy_value(a.lo, a.cnt, off); }
  // First forward stage on words below 2^15 with twiddle 2^48 (the fourth root of unity that the
  // device tables use): x + 2^48 y and x - 2^48 y need no reduction.
  __device__ __forceinline__ static void ct_small_first(W &x, W &y) {
    const W t = y << 48;
    const W u = x;
    x = u + t;
    y = (u + P) - t;
  }
#else
  static void ct(W &x, W &y, W w) {
    const W t = mul(y, w);
    const W u = x;
    x = add_c(u, t);
    y = sub_c(u, t);
  }
  static void gs(W &x, W &y, W w) {
    const W u = x, v = y;
    x = add(u, v);
    y = mul(sub(u, v), w);
  }
  static W mac(W acc, W x, W k) { return add_c(acc, mul(x, k)); }
#endif
  HB_HD static W acc_offset(uint32_t products) { return products ? P - (W)products * EPS : 0; }
  // The device tables pick psi with psi^(2N/64) = 8, so psi^(N/2) = 2^48 and every twiddle
  // psi^e with e a multiple of N/32 is the power of two 2^(96 e / N) (GroupNtt::fwd_stage uses
  // ct_pow2 for those stages).
  static constexpr uint64_t SMALL_FIRST_GEN = 8;
  // The eighth roots of unity 2^24k make radix-8 passes cheaper than three radix-2 stages.
  static constexpr bool RADIX8 = true;
};

// 32-bit prime fields P < 2^31 with canonical data words and Montgomery-form constants.
// Twiddle table entry of the 32-bit fields: the twiddle w (canonical, not in Montgomery form) and
// its Shoup quotient q = floor(w 2^32 / P), read with one 8-byte load.
struct alignas(8) TwPair {
  uint32_t w, q;
};

template <uint32_t PP, uint32_t PINV, int BB, int ID>
struct Mont32 {
  using W = uint32_t;
  static constexpr W P = PP;
  static constexpr W PINV_NEG = PINV;  // -P^-1 mod 2^32
  static constexpr int BITS = BB;      // bits(Q): the decomposition covers this many bits
  static constexpr int FIELD_ID = ID;

  // x - P when x >= P, else x, as an unsigned minimum (x - P wraps above x when x < P): one add
  // and one min instead of a compare, a subtract and a select.
  HB_HD static W umin(W x, W y) { return y < x ? y : x; }
  HB_HD static W canon(W x) { return umin(x, x - P); }
  // (t + m P) / 2^32 with m = -t P^-1 mod 2^32: t 2^-32 mod P, below 2P for t < P 2^32 (no final
  // subtraction).
  HB_HD static uint64_t redc_lazy(uint64_t t) {
    const uint32_t m = (uint32_t)t * PINV_NEG;
    return (t + (uint64_t)m * P) >> 32;
  }
  // Montgomery product a*b*2^-32 mod P for a*b < P*2^32; canonical result.
  HB_HD static W mont(W a, W b) {
    const uint64_t t = (uint64_t)a * b;
    const uint32_t m = (uint32_t)t * PINV_NEG;
    const uint64_t u = (t + (uint64_t)m * P) >> 32;
    return canon((uint32_t)u);
  }
  HB_HD static W mul(W a, W b_mont) { return mont(a, b_mont); }
  HB_HD static W add(W a, W b) { return canon(a + b); }
  // Canonical a - b: a - b, or a - b + P when it wrapped (then a - b + P < P <= the wrapped word).
  HB_HD static W sub(W a, W b) {
    const W d = a - b;
    return umin(d, d + P);
  }
  HB_HD static W add_c(W a, W b) { return add(a, b); }
  HB_HD static W sub_c(W a, W b) { return sub(a, b); }
  HB_HD static W neg_ref(W a) { return a == 0 ? 0 : P - a; }
  HB_HD static W value(W a) { return a; }
  HB_HD static W to_mont(W a) { return (W)(((uint64_t)a << 32) % P); }
  HB_HD static void ct(W &x, W &y, W w) {
    const W t = mont(y, w);
    const W u = x;
    x = add(u, t);
    y = sub(u, t);
  }
  HB_HD static void gs(W &x, W &y, W w) {
    const W u = x, v = y;
    x = add(u, v);
    y = mont(sub(u, v), w);
  }
  // Shoup product a w mod P for any 32-bit a, canonical: with h = floor(a q / 2^32),
  // a w - h P lies in [0, 2P) (below 2^32 since P < 2^31), so it is computed mod 2^32 -- a high
  // and two low multiplies where the Montgomery product takes two wide ones and a low one (a
  // throughput probe of the two chains on B200: 4504 vs 3113 G products/s).
  HB_HD static W shoup(W a, W w, W q) {
#ifdef __CUDA_ARCH__
    const W h = __umulhi(a, q);
#else
    const W h = (W)(((uint64_t)a * q) >> 32);
#endif
    const W r = a * w - h * P;
    return canon(r);
  }
  using Tw = TwPair;
  static constexpr int TW_WORDS = 2;
  HB_HD static Tw make_tw(W w) { return TwPair{w, (W)(((uint64_t)w << 32) / P)}; }
  // Butterflies with table twiddles.
  HB_HD static void ct(W &x, W &y, Tw w) {
    const W t = shoup(y, w.w, w.q);
    const W u = x;
    x = add(u, t);
    y = sub(u, t);
  }
  HB_HD static void gs(W &x, W &y, Tw w) {
    const W u = x, v = y;
    x = add(u, v);
    y = shoup(sub(u, v), w.w, w.q);
  }
  HB_HD static W mac(W acc, W x, W k) { return add(acc, mont(x, k)); }
  // Sums of products x k (x, k < P) in the multiply-accumulate of the external product.
  //  * WIDE (P < 2^28, DefaultFieldU32): t is a 64-bit sum of unreduced products, one 32x32 -> 64
  //    multiply-add each (10.8 % off a DEFAULT_TERNARY launch). fold() keeps t's residue and brings
  //    it below 2^32 (C + 1), C = 2^32 mod P, with one multiply-add, t_hi C + t_lo; FOLD products
  //    fit between two folds (t < 2^64). The value is the Montgomery reduction of the folded t,
  //    which is below P 2^32, so it lands in [0, 2P).
  //  * otherwise (BabyBear, whose products reach 2^62): every product is reduced at once. A 64-bit
  //    sum costs 32 more registers at 16 words per thread, and a 32-bit word with lazily reduced
  //    products and carries folded back as C (6 instructions per product instead of 8) measured
  //    1.2 % slower: the kernel is latency-bound and the fold lengthens the dependent chain.
  static constexpr uint32_t C32 = (uint32_t)((1ull << 32) % PP);
  static constexpr bool WIDE = PP < (1u << 28);
  static constexpr int FOLD =
      WIDE ? (int)((~0ull - (1ull << 32) * (C32 + 1ull)) / ((unsigned long long)PP * PP)) : (1 << 30);
  struct Acc {
    typename std::conditional<WIDE, uint64_t, uint32_t>::type t;
  };
  HB_HD static void acc_clear(Acc &a) { a.t = 0; }
  HB_HD static void acc_mac(Acc &a, W x, W k) {
    if constexpr (WIDE) {
      a.t += (uint64_t)x * k;
    } else {
      a.t = mac(a.t, x, k);
    }
  }
  // a += x kx + y ky. Per-product reduction (BabyBear): the two products share one Montgomery
  // reduction, since x kx + y ky < 2 P^2 < P 2^32 (2P < 2^32) keeps it below 2P.
  HB_HD static void acc_mac2(Acc &a, W x, W kx, W y, W ky) {
    if constexpr (WIDE) {
      a.t += (uint64_t)x * kx;
      a.t += (uint64_t)y * ky;
    } else {
      const uint64_t t = (uint64_t)x * kx + (uint64_t)y * ky;
      a.t = add(a.t, canon((W)redc_lazy(t)));
    }
  }
  HB_HD static void acc_fold(Acc &a) {
    if constexpr (WIDE) a.t = (uint64_t)(uint32_t)(a.t >> 32) * C32 + (uint32_t)a.t;
  }
  HB_HD static W acc_value(const Acc &a, W) {
    if constexpr (WIDE) {
      return canon((W)redc_lazy((uint64_t)(uint32_t)(a.t >> 32) * C32 + (uint32_t)a.t));
    } else {
      return a.t;
    }
  }
  HB_HD static W acc_offset(uint32_t) { return 0; }
  static constexpr uint64_t SMALL_FIRST_GEN = 0;  // no special first stage
  static constexpr bool RADIX8 = false;
};

// BabyBear Q = 2^31 - 2^27 + 1 (algebra/src/modulus/baby_bear/mod.rs:11-15).
using BabyBear = Mont32<0x78000001U, 0x77FFFFFFU, 31, 0>;
// DefaultFieldU32 Q = 132120577 = 2^27 - 2^21 + 1 (fhe_core/src/parameter.rs:286-290), bits(Q) = 27.
using DefaultFieldU32 = Mont32<0x07E00001U, 0x07DFFFFFU, 27, 2>;

// Host-side exact helpers used to build tables.
template <class F>
inline typename F::W host_mulmod(typename F::W a, typename F::W b) {
  return (typename F::W)(((unsigned __int128)a * b) % F::P);
}
template <class F>
inline typename F::W host_powmod(typename F::W b, uint64_t e) {
  typename F::W r = 1;
  while (e) {
    if (e & 1) r = host_mulmod<F>(r, b);
    b = host_mulmod<F>(b, b);
    e >>= 1;
  }
  return r;
}

}  // namespace hb
