// hb_sample.cuh -- the samplers of the project's seeded key convention, shared by the host key
// generator (hb_client.cpp) and the device key generator (keygen_rows_kernel), so that both draw
// the same keys word for word.
//
// Every random value is rand(seed, stream, ctr) = mix(mix(seed + g) ^ mix(stream ^ c) + ctr * g)
// (mix = the splitmix64 finaliser); streams pack (tag, i, part, j, which) into 64 bits.
// Distributions follow the reference: uniform field elements; the discrete Gaussian of
// FieldDiscreteGaussianSampler (algebra/src/random.rs:156-171: N(0, sigma), reject |x| >= 6 sigma,
// round half away from zero, negative r -> Q - |r|) with normal deviates from the Marsaglia polar
// method and a logarithm built from IEEE double operations only; and, for error polynomials with
// sigma exactly 3.2, the centered binomial sampler (algebra/src/random.rs:91-92,
// algebra/src/utils/sample.rs:54-75). The double arithmetic is spelled out as single correctly
// rounded operations (no contraction into fused multiply-adds), so host and device agree.
#pragma once

#include <cstdint>

#ifndef HB_HD
#ifdef __CUDACC__
#define HB_HD __host__ __device__ __forceinline__
#else
#define HB_HD inline
#endif
#endif

namespace hb {
namespace smp {

constexpr uint64_t kTagLweSk = 1, kTagRingSk = 2, kTagBsk = 3, kTagKsk = 4, kTagEnc = 5;

HB_HD uint64_t mix(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

HB_HD uint64_t rnd(uint64_t seed, uint64_t stream, uint64_t ctr) {
  const uint64_t key = mix(seed + 0x9E3779B97F4A7C15ULL) ^ mix(stream ^ 0xD1B54A32D192ED03ULL);
  return mix(key + ctr * 0x9E3779B97F4A7C15ULL);
}

HB_HD uint64_t stream_of(uint64_t tag, uint64_t i, uint64_t part, uint64_t j, uint64_t which) {
  return (tag << 56) | ((i & 0xFFFFFFFFULL) << 24) | ((part & 0xFF) << 16) | ((j & 0xFF) << 8) |
         (which & 0xFF);
}

// Correctly rounded double operations, one rounding each.
HB_HD double dadd(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
HB_HD double dsub(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
HB_HD double dmul(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
HB_HD double ddiv(double a, double b) {
#ifdef __CUDA_ARCH__
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
HB_HD double dsqrt(double a) {
#ifdef __CUDA_ARCH__
  return __dsqrt_rn(a);
#else
  return __builtin_sqrt(a);
#endif
}
HB_HD double dround(double a) {  // half away from zero
#ifdef __CUDA_ARCH__
  return round(a);
#else
  return __builtin_round(a);
#endif
}
HB_HD double dabs(double a) { return a < 0.0 ? -a : a; }

HB_HD double bits_to_double(uint64_t b) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)b);
#else
  double d;
  __builtin_memcpy(&d, &b, sizeof d);
  return d;
#endif
}
HB_HD uint64_t double_to_bits(double d) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t b;
  __builtin_memcpy(&b, &d, sizeof b);
  return b;
#endif
}

// s = m 2^e with m in [0.5, 1), for a positive normal double s (exact: a field split).
HB_HD double split_exponent(double s, int *e) {
  const uint64_t b = double_to_bits(s);
  *e = (int)((b >> 52) & 0x7FF) - 1022;
  return bits_to_double((b & 0x800FFFFFFFFFFFFFULL) | (1022ULL << 52));
}

// ln(s), s in (0, 1): s = m 2^e with m in [1/sqrt2, sqrt2), ln s = e ln2 + 2 atanh((m-1)/(m+1)),
// atanh by its odd power series (24 terms; |y| <= 0.1716). s is a sum of squares of multiples of
// 2^-52, so it is normal.
HB_HD double log_unit(double s) {
  int e;
  double m = split_exponent(s, &e);
  if (m < 0.70710678118654752440) {
    m = dmul(m, 2.0);
    e = e - 1;
  }
  const double y = ddiv(dsub(m, 1.0), dadd(m, 1.0));
  const double y2 = dmul(y, y);
  double acc = 0.0;
  double pw = y;
  for (int k = 0; k < 24; ++k) {
    acc = dadd(acc, ddiv(pw, (double)(2 * k + 1)));
    pw = dmul(pw, y2);
  }
  return dadd(dmul(2.0, acc), dmul((double)e, 0.693147180559945309417232121458));
}

HB_HD double to_unit(uint64_t r) { return dmul((double)(r >> 11), 1.0 / 9007199254740992.0); }

template <class F>
HB_HD typename F::W sample_gauss(uint64_t seed, uint64_t stream, uint64_t coeff, double sigma) {
  const double bound = dmul(sigma, 6.0);
  for (uint64_t attempt = 0;; ++attempt) {
    const uint64_t ctr = (coeff << 20) | (attempt << 1);
    const double u = dsub(dmul(2.0, to_unit(rnd(seed, stream, ctr))), 1.0);
    const double v = dsub(dmul(2.0, to_unit(rnd(seed, stream, ctr | 1))), 1.0);
    const double s = dadd(dmul(u, u), dmul(v, v));
    if (!(s > 0.0 && s < 1.0)) continue;
    const double z = dmul(u, dsqrt(ddiv(dmul(-2.0, log_unit(s)), s)));
    const double val = dmul(sigma, z);
    if (dabs(val) >= bound) continue;
    const double r = dround(val);
    if (r < 0.0) return (typename F::W)((uint64_t)F::P - (uint64_t)(-r));
    return (typename F::W)(uint64_t)r;
  }
}

template <class F>
HB_HD typename F::W sample_uniform(uint64_t seed, uint64_t stream, uint64_t k) {
  return (typename F::W)(rnd(seed, stream, k) % (uint64_t)F::P);
}

HB_HD uint32_t popcount64(uint64_t x) {
#ifdef __CUDA_ARCH__
  return (uint32_t)__popcll(x);
#else
  return (uint32_t)__builtin_popcountll(x);
#endif
}

// sample_cbd_field_vec (algebra/src/utils/sample.rs:54-75) on the low six bytes of one PRG word:
// popcounts a (bytes 0, 1 and 5 bits of byte 2) and b (bytes 3, 4 and 5 bits of byte 5). For a < b
// the reference's `modulus - (a - b)` wraps its u32 subtraction (release builds), which leaves
// Field::new of the wrapped word in the field's width: b - a for 32-bit fields,
// P - (2^32 - (b - a)) for Goldilocks.
template <class F>
HB_HD typename F::W sample_cbd(uint64_t seed, uint64_t stream, uint64_t k) {
  using W = typename F::W;
  const uint64_t r = rnd(seed, stream, k);
  const uint32_t a = popcount64(r & 0xFF) + popcount64((r >> 8) & 0xFF) + popcount64((r >> 16) & 0x1F);
  const uint32_t b = popcount64((r >> 24) & 0xFF) + popcount64((r >> 32) & 0xFF) + popcount64((r >> 40) & 0x1F);
  const uint32_t d = a - b;
  if (a >= b) return (W)d;
  const W v = (W)((W)F::P - (W)d);
  return (W)((uint64_t)v % (uint64_t)F::P);
}

// One coefficient of an error polynomial (Polynomial::random_with_gaussian,
// algebra/src/polynomial/univariate/native_polynomial.rs:232-246).
template <class F>
HB_HD typename F::W error_coeff(uint64_t seed, uint64_t stream, uint64_t k, double sigma) {
  return sigma == 3.2 ? sample_cbd<F>(seed, stream, k) : sample_gauss<F>(seed, stream, k, sigma);
}

// Canonical (a + b) mod P of canonical words.
template <class F>
HB_HD typename F::W add_mod(typename F::W a, typename F::W b) {
  using W = typename F::W;
  if constexpr (sizeof(W) == 8) {
    W r = a + b;
    if (r < a || r >= F::P) r = (W)(r - F::P);
    return r;
  } else {
    const uint64_t s = (uint64_t)a + b;
    return (W)(s >= F::P ? s - F::P : s);
  }
}

// tfhe encoding of a message m in Z_4 (fhe_core/src/plaintext.rs:64-75): round(m * (Q / 4)).
template <class F>
HB_HD uint64_t encode_msg(uint64_t m) {
  const double q = (double)(uint64_t)F::P;
  return (uint64_t)dround(dmul((double)m, ddiv(q, 4.0)));
}

}  // namespace smp
}  // namespace hb
