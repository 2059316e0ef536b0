// hb_client.cpp -- host-side parameters, key generation, encryption and decryption
// (the tfhe crate's KeyGen / Encryptor / Decryptor and Evaluator::new key material).
//
// Seeded key convention: every random value is drawn from the counter PRG of hb_sample.cuh, so key
// generation parallelises over polynomials and is identical on every host and on the device
// (hb_keys_generate). Distributions follow the reference: binary or ternary {0,0,1,-1}[r&3] LWE and
// ring keys (algebra/src/utils/sample.rs:6-51), uniform field elements, the discrete Gaussian and,
// for error polynomials with sigma exactly 3.2, the centered binomial sampler (hb_sample.cuh).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/hb_gpu.h"
#include "hb_field.cuh"
#include "hb_sample.cuh"

namespace {

using u64 = uint64_t;
using u128 = unsigned __int128;

// ---- field helpers (host, canonical) ----
template <class F>
struct HostField {
  using W = typename F::W;
  static W add(W a, W b) {
    u64 s = (u64)a + b;
    if (sizeof(W) == 8) {
      // a, b < P < 2^64: detect wrap
      W r = (W)s;
      if (r < a || r >= F::P) r = (W)(r - F::P);
      return r;
    }
    return (W)(s >= F::P ? s - F::P : s);
  }
  static W sub(W a, W b) { return a >= b ? (W)(a - b) : (W)(a + (F::P - b)); }
  static W mul(W a, W b) { return (W)(((u128)a * b) % F::P); }
  static W neg(W a) { return a == 0 ? 0 : (W)(F::P - a); }
};

// ---- samplers (hb_sample.cuh, shared with the device key generator) ----
using hb::smp::error_coeff;
using hb::smp::kTagBsk;
using hb::smp::kTagEnc;
using hb::smp::kTagKsk;
using hb::smp::kTagLweSk;
using hb::smp::kTagRingSk;
using hb::smp::rnd;
using hb::smp::sample_gauss;
using hb::smp::sample_uniform;
using hb::smp::stream_of;

// Calls fn(F{}) with the field type of a field id (Goldilocks, BabyBear or DefaultFieldU32).
template <class Fn>
void with_field(int field_id, Fn fn) {
  if (field_id == HB_FIELD_GOLDILOCKS)
    fn(hb::Goldilocks{});
  else if (field_id == HB_FIELD_BABYBEAR)
    fn(hb::BabyBear{});
  else
    fn(hb::DefaultFieldU32{});
}

// ---- host negacyclic multiplication for key generation (radix-2, twisted cyclic NTT) ----
template <class F>
struct HostRing {
  using W = typename F::W;
  using H = HostField<F>;
  uint32_t n, logn;
  std::vector<W> twist, untwist, roots, iroots;
  std::vector<uint32_t> rev;
  W ninv;

  explicit HostRing(uint32_t logn_) : n(1u << logn_), logn(logn_) {
    const u64 order = (u64)F::P - 1;
    W psi = 0;
    for (W g = 2; g < 64 && !psi; ++g) {
      W c = hb::host_powmod<F>(g, order / (2ull * n));
      if (hb::host_powmod<F>(c, n) == (W)(F::P - 1)) psi = c;
    }
    const W psi_inv = hb::host_powmod<F>(psi, (u64)F::P - 2);
    twist.resize(n);
    untwist.resize(n);
    W a = 1, b = 1;
    ninv = hb::host_powmod<F>((W)n, (u64)F::P - 2);
    for (uint32_t i = 0; i < n; ++i) {
      twist[i] = a;
      untwist[i] = H::mul(b, ninv);
      a = H::mul(a, psi);
      b = H::mul(b, psi_inv);
    }
    const W w = H::mul(psi, psi), wi = H::mul(psi_inv, psi_inv);
    roots.assign(n, 0);
    iroots.assign(n, 0);
    for (uint32_t half = 1; half < n; half <<= 1) {
      const W step = hb::host_powmod<F>(w, n / (2 * half));
      const W istep = hb::host_powmod<F>(wi, n / (2 * half));
      W x = 1, y = 1;
      for (uint32_t j = 0; j < half; ++j) {
        roots[half + j] = x;
        iroots[half + j] = y;
        x = H::mul(x, step);
        y = H::mul(y, istep);
      }
    }
    rev.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
      uint32_t r = 0;
      for (uint32_t b2 = 0; b2 < logn; ++b2) r |= ((i >> b2) & 1) << (logn - 1 - b2);
      rev[i] = r;
    }
  }
  void dft(W *a, const std::vector<W> &rt) const {
    for (uint32_t i = 0; i < n; ++i)
      if (i < rev[i]) std::swap(a[i], a[rev[i]]);
    for (uint32_t half = 1; half < n; half <<= 1)
      for (uint32_t i = 0; i < n; i += 2 * half)
        for (uint32_t j = 0; j < half; ++j) {
          const W u = a[i + j], v = H::mul(a[i + j + half], rt[half + j]);
          a[i + j] = H::add(u, v);
          a[i + j + half] = H::sub(u, v);
        }
  }
  void to_eval(W *a) const {
    for (uint32_t i = 0; i < n; ++i) a[i] = H::mul(a[i], twist[i]);
    dft(a, roots);
  }
  void to_coeff(W *a) const {
    dft(a, iroots);
    for (uint32_t i = 0; i < n; ++i) a[i] = H::mul(a[i], untwist[i]);
  }
  // out = x * y where y_eval is y in evaluation form
  void mul(const W *x, const W *y_eval, W *out) const {
    std::vector<W> t(x, x + n);
    to_eval(t.data());
    for (uint32_t i = 0; i < n; ++i) t[i] = H::mul(t[i], y_eval[i]);
    to_coeff(t.data());
    std::memcpy(out, t.data(), sizeof(W) * n);
  }
};

u64 modulus_of(int field_id) {
  return field_id == HB_FIELD_GOLDILOCKS ? hb::Goldilocks::P
         : field_id == HB_FIELD_BABYBEAR ? (u64)hb::BabyBear::P
                                         : (u64)hb::DefaultFieldU32::P;
}

bool check_params(const hb_params *p) {
  if (!p) return false;
  if (p->field_id != HB_FIELD_BABYBEAR && p->field_id != HB_FIELD_GOLDILOCKS &&
      p->field_id != HB_FIELD_DEFAULT_U32)
    return false;
  const uint32_t N = p->ring_dim;
  if (N < 4 || N > 4096 || (N & (N - 1))) return false;
  // The RLWE key switch pads the LWE key to next_pow2(n) <= N words
  // (fhe_core/src/key_switch/rlwe.rs:40-43).
  if (p->lwe_dim == 0 || p->lwe_dim > N) return false;
  // A ternary LWE key takes TernaryBlindRotationKey, whose NTT-domain monomial the reference marks
  // incompatible with BabyBear and Goldilocks (fhe_core/src/blind_rotation/rlwe/ternary.rs:80).
  if (p->lwe_ternary > 1 || (p->lwe_ternary && p->field_id != HB_FIELD_DEFAULT_U32)) return false;
  if (p->ring_ternary > 1) return false;
  // Parameters::new: 2N | Q - 1 (fhe_core/src/parameter.rs:131-138)
  const u64 q = modulus_of(p->field_id);
  if ((q - 1) % (2ull * N) != 0) return false;
  const uint32_t qbits = p->field_id == HB_FIELD_GOLDILOCKS ? 64 : p->field_id == HB_FIELD_BABYBEAR ? 31 : 27;
  if (p->br_bits == 0 || p->br_bits > 16 || p->ks_bits == 0 || p->ks_bits > 16) return false;
  if (p->br_len != (qbits + p->br_bits - 1) / p->br_bits) return false;
  if (p->ks_len != (qbits + p->ks_bits - 1) / p->ks_bits) return false;
  if (!(p->lwe_noise_std >= 0) || !(p->ring_noise_std >= 0) || !(p->ks_noise_std >= 0)) return false;
  return true;
}

template <class F>
void keygen_impl(const hb_params *p, u64 seed, typename F::W *lwe_sk, typename F::W *ring_sk,
                 typename F::W *bsk, typename F::W *ksk, int threads) {
  using W = typename F::W;
  using H = HostField<F>;
  const uint32_t N = p->ring_dim, n = p->lwe_dim, L = p->br_len;
  const W tern[4] = {0, 0, 1, (W)(F::P - 1)};
  for (uint32_t i = 0; i < n; ++i) {
    const u64 r = rnd(seed, stream_of(kTagLweSk, 0, 0, 0, 0), i);
    lwe_sk[i] = p->lwe_ternary ? tern[r & 3] : (W)(r & 1);
  }
  for (uint32_t k = 0; k < N; ++k) {
    const u64 r = rnd(seed, stream_of(kTagRingSk, 0, 0, 0, 0), k);
    ring_sk[k] = p->ring_ternary ? tern[r & 3] : (W)(r & 1);
  }
  if (!bsk) return;
  uint32_t logn = 0;
  while ((1u << logn) < N) ++logn;
  HostRing<F> ring(logn);
  std::vector<W> z_eval(ring_sk, ring_sk + N);
  ring.to_eval(z_eval.data());

  // One RLWE zero sample in the ring of rg: a uniform, b = a*key + e.
  auto zero_sample = [&](const HostRing<F> &rg, const W *key_eval, u64 sa, u64 se, double sigma, W *a,
                         W *b) {
    for (uint32_t k = 0; k < rg.n; ++k) a[k] = sample_uniform<F>(seed, sa, k);
    rg.mul(a, key_eval, b);
    for (uint32_t k = 0; k < rg.n; ++k) b[k] = H::add(b[k], error_coeff<F>(seed, se, k, sigma));
  };

  // BSK: per LWE key coefficient an NTTRGSW zero sample (s_i = 0) or one sample (s_i = 1)
  // (lattice/src/rgsw.rs:343-395): c_neg_s_m rows (a + B^j, b) / c_m rows (a, b + B^j). A ternary
  // key holds the pair (RGSW(s_i == 1), RGSW(s_i == -1)) per coefficient
  // (fhe_core/src/blind_rotation/rlwe/ternary.rs:123-183); pair 1 draws from streams part + 2.
  const uint32_t pairs = p->lwe_ternary ? 2 : 1;
  const size_t rows_total = (size_t)n * pairs * 2 * L;
  std::atomic<size_t> next{0};
  auto worker = [&] {
    for (size_t q; (q = next.fetch_add(1)) < rows_total;) {
      const uint32_t i = (uint32_t)(q / (pairs * 2 * L));
      const uint32_t pair = (uint32_t)((q / (2 * L)) % pairs);
      const uint32_t part = (uint32_t)((q / L) % 2);
      const uint32_t j = (uint32_t)(q % L);
      W *a = bsk + q * 2 * N;
      W *b = a + N;
      zero_sample(ring, z_eval.data(), stream_of(kTagBsk, i, part + 2 * pair, j, 0),
                  stream_of(kTagBsk, i, part + 2 * pair, j, 1), p->ring_noise_std, a, b);
      const bool one = pairs == 1 ? lwe_sk[i] != 0 : lwe_sk[i] == (pair == 0 ? (W)1 : (W)(F::P - 1));
      if (one) {
        const W bj = (W)((u64)1 << (j * p->br_bits));
        if (part == 0)
          a[0] = H::add(a[0], bj);
        else
          b[0] = H::add(b[0], bj);
      }
    }
  };
  const int nt = std::max(1, threads);
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) pool.emplace_back(worker);
  for (auto &th : pool) th.join();

  // KSK (fhe_core/src/key_switch/rlwe.rs:37-112): the LWE key padded to n' = next_pow2(n) words;
  // per n'-word chunk z_c of the ring key (z itself when n' == N) rows j = zero samples of
  // dimension n' plus z_c * B_ks^j on b. Layout [c][j][ab][n'].
  uint32_t M = 1, logm = 0;
  while (M < n) {
    M <<= 1;
    ++logm;
  }
  HostRing<F> kring(logm);
  std::vector<W> s_eval(M, 0);
  for (uint32_t i = 0; i < n; ++i) s_eval[i] = lwe_sk[i];
  kring.to_eval(s_eval.data());
  const W bks = (W)(1u << p->ks_bits);
  for (uint32_t c = 0; c < N / M; ++c) {
    std::vector<W> zpow(ring_sk + (size_t)c * M, ring_sk + (size_t)(c + 1) * M);
    for (uint32_t j = 0; j < p->ks_len; ++j) {
      W *a = ksk + ((size_t)c * p->ks_len + j) * 2 * M;
      W *b = a + M;
      zero_sample(kring, s_eval.data(), stream_of(kTagKsk, c, 0, j, 0), stream_of(kTagKsk, c, 0, j, 1),
                  p->ks_noise_std, a, b);
      for (uint32_t k = 0; k < M; ++k) b[k] = H::add(b[k], zpow[k]);
      for (uint32_t k = 0; k < M; ++k) zpow[k] = H::mul(zpow[k], bks);
    }
  }
}

template <class F>
u64 encode_msg(u64 m) {
  return hb::smp::encode_msg<F>(m);  // fhe_core/src/plaintext.rs:64-75, t = 4
}
template <class F>
u64 decode_msg(u64 c) {
  const double q = (double)(u64)F::P;
  const u64 r = (u64)std::round((double)c * 4.0 / q);  // plaintext.rs:87-97
  return r < 4 ? r : r - 4;
}

template <class F>
void encrypt_impl(const hb_params *p, const typename F::W *sk, u64 seed, u64 index0,
                  const uint8_t *bits, size_t count, typename F::W *out) {
  using W = typename F::W;
  using H = HostField<F>;
  const uint32_t n = p->lwe_dim;
  for (size_t c = 0; c < count; ++c) {
    W *ct = out + c * (n + 1);
    const u64 idx = index0 + c;
    W dot = 0;
    for (uint32_t i = 0; i < n; ++i) {
      ct[i] = sample_uniform<F>(seed, stream_of(kTagEnc, idx, 0, 0, 0), i);
      dot = H::add(dot, H::mul(ct[i], sk[i]));
    }
    const W e = sample_gauss<F>(seed, stream_of(kTagEnc, idx, 0, 0, 1), 0, p->lwe_noise_std);
    ct[n] = H::add(H::add(dot, e), (W)encode_msg<F>(bits[c] & 1));
  }
}

template <class F>
void decrypt_impl(const hb_params *p, const typename F::W *sk, const typename F::W *in, size_t count,
                  uint8_t *bits, uint64_t *noise) {
  using W = typename F::W;
  using H = HostField<F>;
  const uint32_t n = p->lwe_dim;
  for (size_t c = 0; c < count; ++c) {
    const W *ct = in + c * (n + 1);
    W dot = 0;
    for (uint32_t i = 0; i < n; ++i) dot = H::add(dot, H::mul((W)(ct[i] % F::P), sk[i]));
    const W pt = H::sub((W)(ct[n] % F::P), dot);
    const u64 m = decode_msg<F>(pt);
    if (bits) bits[c] = (uint8_t)m;
    if (noise) {
      const W fresh = (W)encode_msg<F>(m);
      noise[c] = std::min<u64>(H::sub(pt, fresh), H::sub(fresh, pt));
    }
  }
}

}  // namespace

extern "C" {

int hb_params_preset(int preset, hb_params *out) {
  if (!out) return HB_ERR_INVALID;
  std::memset(out, 0, sizeof(*out));
  out->ring_dim = 1024;
  out->lwe_dim = 728;
  out->ring_ternary = 1;
  out->ks_bits = 5;
  if (preset == HB_PRESET_DEFAULT_TERNARY_128_BITS || preset == HB_PRESET_CUSTOM_TERNARY_128_BITS) {
    // tfhe/src/bfhe/parameters.rs:7-42: both sets configure binary LWE and ring keys.
    const bool dflt = preset == HB_PRESET_DEFAULT_TERNARY_128_BITS;
    out->field_id = HB_FIELD_DEFAULT_U32;
    out->lwe_dim = dflt ? 1024 : 512;
    out->ring_ternary = 0;
    out->br_bits = dflt ? 3 : 7;
    out->br_len = dflt ? 9 : 4;
    out->ks_bits = dflt ? 1 : 7;
    out->ks_len = dflt ? 27 : 4;
    out->lwe_noise_std = 3.20;
    out->ring_noise_std = 3.20 * 2.0;
    out->ks_noise_std = 3.2 * 2.0;
    return HB_OK;
  }
  if (preset == HB_PRESET_BABYBEAR_BINARY_128_BITS) {
    out->field_id = HB_FIELD_BABYBEAR;
    out->br_bits = 8;
    out->br_len = 4;
    out->ks_len = 7;
    out->lwe_noise_std = 11000.0;
    out->ring_noise_std = 41.9;
    out->ks_noise_std = 11000.0;
    return HB_OK;
  }
  if (preset == HB_PRESET_GOLDILOCKS_BINARY_128_BITS || preset == HB_PRESET_ZAMA_BINARY_128_BITS) {
    const bool zama = preset == HB_PRESET_ZAMA_BINARY_128_BITS;
    out->field_id = HB_FIELD_GOLDILOCKS;
    out->br_bits = zama ? 5 : 8;
    out->br_len = zama ? 13 : 8;
    out->ks_len = 13;
    out->lwe_noise_std = 2.9 * (double)(1ULL << 45);
    out->ring_noise_std = 2.3 * (double)(1ULL << 37);
    out->ks_noise_std = 2.9 * (double)(1ULL << 45);
    return HB_OK;
  }
  return HB_ERR_INVALID;
}

int hb_params_validate(const hb_params *p) { return check_params(p) ? HB_OK : HB_ERR_INVALID; }

int hb_params_sizes(const hb_params *p, size_t *lwe_sk, size_t *ring_sk, size_t *bsk, size_t *ksk,
                    size_t *lwe) {
  if (!check_params(p)) return HB_ERR_INVALID;
  const size_t N = p->ring_dim, n = p->lwe_dim;
  if (lwe_sk) *lwe_sk = n;
  if (ring_sk) *ring_sk = N;
  if (bsk) *bsk = n * (p->lwe_ternary ? 2 : 1) * 2 * p->br_len * 2 * N;
  if (ksk) *ksk = (size_t)p->ks_len * 2 * N;
  if (lwe) *lwe = n + 1;
  return HB_OK;
}

int hb_keygen(const hb_params *p, uint64_t seed, void *lwe_sk, void *ring_sk, void *bsk, void *ksk,
              int threads) {
  // bsk and ksk may both be NULL: only the secret keys are produced (KeyGen::generate_secret_key).
  if (!check_params(p) || !lwe_sk || !ring_sk || (!bsk != !ksk)) return HB_ERR_INVALID;
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  with_field(p->field_id, [&](auto f) {
    using F = decltype(f);
    using W = typename F::W;
    keygen_impl<F>(p, seed, (W *)lwe_sk, (W *)ring_sk, (W *)bsk, (W *)ksk, threads);
  });
  return HB_OK;
}

int hb_encrypt(const hb_params *p, const void *lwe_sk, uint64_t seed, uint64_t index0,
               const uint8_t *bits, size_t count, void *lwe_out) {
  if (!check_params(p) || !lwe_sk || (count && (!bits || !lwe_out))) return HB_ERR_INVALID;
  with_field(p->field_id, [&](auto f) {
    using F = decltype(f);
    using W = typename F::W;
    encrypt_impl<F>(p, (const W *)lwe_sk, seed, index0, bits, count, (W *)lwe_out);
  });
  return HB_OK;
}

int hb_decrypt(const hb_params *p, const void *lwe_sk, const void *lwe, size_t count,
               uint8_t *bits_out, uint64_t *noise_out) {
  if (!check_params(p) || !lwe_sk || (count && !lwe)) return HB_ERR_INVALID;
  with_field(p->field_id, [&](auto f) {
    using F = decltype(f);
    using W = typename F::W;
    decrypt_impl<F>(p, (const W *)lwe_sk, (const W *)lwe, count, bits_out, noise_out);
  });
  return HB_OK;
}

}  // extern "C"
