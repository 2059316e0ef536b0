// hb_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see hb_oracle.h for scope and parity status).
//
// CPU restatement of the reference's TFHE NAND/gate bootstrapping path. Every function cites
// the reference file:line it follows. Transforms are exact over Z/QZ with canonical inputs and
// outputs (Goldilocks words may leave [0, Q) between butterflies, never between calls); where the
// reference's own code fixes a (possibly non-canonical) Goldilocks representation that can leak
// into results -- accumulator additions and negations -- this file reproduces the reference's
// exact u64 operations (algebra/src/modulus/goldilocks/ops.rs).
//
// Assumption (the reference's NTT lives in the un-vendored concrete-ntt crate): its forward and
// inverse transforms are exact over Z/QZ and the inverse returns canonical values in [0, Q).

#include "hb_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace {

typedef unsigned __int128 u128;

// ------------------------------------------------------------------------------------------
// Fields
// ------------------------------------------------------------------------------------------

// Goldilocks Q = 2^64 - 2^32 + 1 (algebra/src/modulus/goldilocks/mod.rs:9-11).
struct Gold {
  using T = uint64_t;
  static constexpr T P = 0xFFFFFFFF00000001ULL;
  static constexpr T EPS = 0xFFFFFFFFULL;  // 2^64 mod P
  static constexpr int BITS = 64;          // bits(Q) (algebra/src/goldilocks/mod.rs:69-75)

  static T canon(T x) { return x - (P & mask(x >= P)); }

  // All-ones when c holds: the folds and corrections below are written without data-dependent
  // branches (about half of them fire on random data).
  static T mask(bool c) { return (T)0 - (T)c; }

  // 128-bit -> 64-bit folding using 2^64 = 2^32 - 1 and 2^96 = -1 (mod P) (the reduce128 of
  // algebra/src/modulus/goldilocks/mod.rs:139-150). Result in [0, 2^64), not canonical.
  static T fold128(u128 x) {
    const T lo = (T)x, hi = (T)(x >> 64);
    const T hh = hi >> 32, hl = hi & EPS;
    const T t0 = lo - hh - (EPS & mask(lo < hh));  // a borrow wraps by 2^64 = P + EPS
    const T t1 = hl * EPS;
    const T s = t0 + t1;
    return s + (EPS & mask(s < t1));  // after a carry s < t1 <= 2^64 - 2^33 + 1: no second carry
  }

  // Canonical arithmetic.
  static T add(T a, T b) {
    const u128 s = (u128)canon(a) + canon(b);
    return (T)(s >= P ? s - P : s);
  }
  static T sub(T a, T b) {
    a = canon(a);
    b = canon(b);
    const T d = a - b;
    return a >= b ? d : d + P;
  }
  static T mul(T a, T b) { return canon(fold128((u128)a * b)); }
  // Operations on canonical inputs (the transforms keep every word canonical).
  static T add_cc(T a, T b) {
    const T s = a + b;
    return s - (P & mask((s < a) | (s >= P)));
  }
  static T sub_cc(T a, T b) { return a - b + (P & mask(a < b)); }
  // Lazy operations for the transforms: any word in [0, 2^64) stands for its residue. A carry out
  // of a + b is worth 2^64 = EPS (mod P); after one carry the sum is at most 2^64 - 2, so adding
  // EPS carries at most once more, and then the word is below 2^33. A borrow is worth -EPS the
  // same way; a second borrow leaves at least 2^64 - 2 EPS, so the third subtraction cannot wrap.
  static T add_lz(T a, T b) {
    const T s = a + b, e = EPS & mask(s < a), s2 = s + e;
    return s2 + (EPS & mask(s2 < e));
  }
  static T sub_lz(T a, T b) {
    const T d = a - b, e = EPS & mask(a < b);
    return d - e - (EPS & mask(d < e));
  }
  static T mul_lz(T a, T b) { return fold128((u128)a * b); }
  // Sum of products reduced once: fold128 values (< 2^64) added in 128 bits.
  typedef u128 Acc;
  static void acc_mac(Acc &acc, T a, T b) { acc += fold128((u128)a * b); }
  static T acc_value(Acc acc) { return canon(fold128(acc)); }
  static T neg(T a) {
    a = canon(a);
    return a == 0 ? 0 : P - a;
  }

  // The reference's exact representation-level operations.
  // add_reduce: algebra/src/modulus/goldilocks/ops.rs:26-35
  static T add_ref(T a, T b) {
    T s = a + b;
    bool over = s < a;
    T s2 = s + (over ? EPS : 0);
    bool over2 = s2 < s;
    if (over2) s2 += EPS;
    return s2;
  }
  // sub_reduce: algebra/src/modulus/goldilocks/ops.rs:48-57
  static T sub_ref(T a, T b) {
    T d = a - b;
    bool under = a < b;
    T c = under ? EPS : 0;
    T d2 = d - c;
    bool under2 = d < c;
    if (under2) d2 -= EPS;
    return d2;
  }
  // neg_reduce: algebra/src/modulus/goldilocks/ops.rs:69-73 (`P - self`, wrapping when self > P)
  static T neg_ref(T a) { return a == 0 ? 0 : P - a; }
  // Field::value (algebra/src/goldilocks/mod.rs:53-56)
  static T value(T a) { return canon(a); }
  static T from_u64(uint64_t v) { return v; }  // Goldilocks::new stores the word unchanged
};

// 32-bit prime fields with canonical words:
//  - BabyBear Q = 2^31 - 2^27 + 1 (algebra/src/modulus/baby_bear/mod.rs:11). The reference stores
//    Montgomery form; every operation on the path returns canonical residues, so the oracle works
//    on canonical values directly. bits(Q) = 31 (algebra/src/baby_bear/mod.rs:73-79).
//  - DefaultFieldU32 Q = 132120577 = 2^27 - 2^21 + 1 (fhe_core/src/parameter.rs:286-290): a
//    derived Barrett field storing the plain residue (algebra_derive/src/field.rs:91-120) with the
//    usual add/sub/neg reductions (algebra_derive/src/ops.rs:25-113); bits(Q) = 27, the bit length
//    of the modulus (algebra/src/modulus/barrett/internal_macros.rs:74-76). Its lazy FheField
//    products (algebra_derive/src/fhe_field.rs:31-42) only feed inverse transforms, whose outputs
//    are canonical, so exact products give the same coefficients.
template <uint32_t PP, int BB>
struct Prime32 {
  using T = uint32_t;
  static constexpr T P = PP;
  static constexpr int BITS = BB;

  static T canon(T x) { return x % P; }
  static T add(T a, T b) {
    uint32_t s = a + b;  // a, b < 2^31
    return s >= P ? s - P : s;
  }
  static T sub(T a, T b) { return a >= b ? a - b : a + P - b; }
  static T mul(T a, T b) { return (T)(((uint64_t)a * b) % P); }
  static T add_cc(T a, T b) { return add(a, b); }
  static T sub_cc(T a, T b) { return sub(a, b); }
  typedef uint64_t Acc;  // sum of canonical products (each < 2^62), reduced per product
  static void acc_mac(Acc &acc, T a, T b) { acc += mul(a, b); }
  static T acc_value(Acc acc) { return (T)(acc % P); }
  static T neg(T a) { return a == 0 ? 0 : P - a; }
  static T add_ref(T a, T b) { return add(a, b); }  // ops.rs:9-17
  static T sub_ref(T a, T b) { return sub(a, b); }  // ops.rs:28-35
  static T neg_ref(T a) { return neg(a); }          // ops.rs:47-51
  static T value(T a) { return a; }
  static T from_u64(uint64_t v) { return (T)(v % P); }
};
using Baby = Prime32<0x78000001U, 31>;
using Dflt = Prime32<0x07E00001U, 27>;

// bits(Q) of a field id (the decomposition length is ceil(bits(Q) / basis bits)).
inline int field_bits(int field_id) {
  return field_id == ORC_FIELD_GOLDILOCKS ? 64 : field_id == ORC_FIELD_BABYBEAR ? 31 : 27;
}

template <class F>
typename F::T fpow(typename F::T b, uint64_t e) {
  typename F::T r = 1;
  while (e) {
    if (e & 1) r = F::mul(r, b);
    b = F::mul(b, b);
    e >>= 1;
  }
  return r;
}

template <class F>
typename F::T finv(typename F::T a) {
  return fpow<F>(a, (uint64_t)F::P - 2);
}

// ------------------------------------------------------------------------------------------
// Negacyclic NTT: Cooley-Tukey with the psi twist merged into the twiddles (natural order in,
// bit-reversed slot order out) and the matching Gentleman-Sande inverse (bit-reversed in, natural
// out, times N^-1). Slot order is internal: every NTT-domain operation on the path is pointwise,
// and the constant polynomial c still transforms to [c; N], which the reference's key switch
// initialiser relies on (fhe_core/src/key_switch/rlwe.rs:118-121).
// ------------------------------------------------------------------------------------------

inline uint32_t bit_reverse(uint32_t x, uint32_t bits) {
  uint32_t r = 0;
  for (uint32_t i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

template <class F>
struct Ntt {
  using T = typename F::T;
  uint32_t logn = 0, n = 0;
  std::vector<T> zeta, izeta;  // zeta[k] = psi^brv(k), izeta[k] = psi^-brv(k), k in [1, n)
  T n_inv = 0;
  bool ok = false;
  // 32-bit fields: Shoup's precomputed quotients w' = floor(w 2^32 / P) of every constant factor
  // (V. Shoup's NTL MulModPrecon; D. Harvey, "Faster arithmetic for number-theoretic transforms",
  // J. Symb. Comput. 60, 2014): for a < 2^32 and w < P < 2^31, a w - floor(a w' / 2^32) P lies in
  // [0, 2P), so one conditional subtraction gives the canonical a w mod P.
  std::vector<uint32_t> zeta_q, izeta_q;
  uint32_t n_inv_q = 0;

  static uint32_t quotient(T w) { return (uint32_t)(((uint64_t)w << 32) / F::P); }
  static T mul_q(T a, T w, uint32_t wq) {
    if constexpr (sizeof(T) == 4) {
      const uint32_t q = (uint32_t)(((uint64_t)a * wq) >> 32);
      const uint32_t r = (uint32_t)a * (uint32_t)w - q * (uint32_t)F::P;
      return (T)(r >= F::P ? r - F::P : r);
    } else {
      (void)wq;
      return F::mul(a, w);
    }
  }
  // Butterfly operations: Goldilocks words stay lazy inside a transform (canonical at its end),
  // the 32-bit fields' words stay canonical.
  static T bf_add(T a, T b) {
    if constexpr (sizeof(T) == 8) return F::add_lz(a, b); else return F::add_cc(a, b);
  }
  static T bf_sub(T a, T b) {
    if constexpr (sizeof(T) == 8) return F::sub_lz(a, b); else return F::sub_cc(a, b);
  }
  static T bf_mul(T a, T w, uint32_t wq) {
    if constexpr (sizeof(T) == 8) return F::mul_lz(a, w); else return mul_q(a, w, wq);
  }

  explicit Ntt(uint32_t log_n) : logn(log_n), n(1u << log_n) {
    uint64_t order = (uint64_t)F::P - 1;
    if (order % (2ull * n) != 0) return;
    T psi = 0;
    for (T g = 2; g < 100; ++g) {
      T c = fpow<F>(g, order / (2ull * n));
      if (fpow<F>(c, n) == F::P - 1) {
        psi = c;
        break;
      }
    }
    if (!psi) return;
    const T psi_inv = finv<F>(psi);
    std::vector<T> pw(n), ipw(n);
    T a = 1, b = 1;
    for (uint32_t i = 0; i < n; ++i) {
      pw[i] = a;
      ipw[i] = b;
      a = F::mul(a, psi);
      b = F::mul(b, psi_inv);
    }
    zeta.assign(n, 0);
    izeta.assign(n, 0);
    for (uint32_t k = 1; k < n; ++k) {
      zeta[k] = pw[bit_reverse(k, logn)];
      izeta[k] = ipw[bit_reverse(k, logn)];
    }
    n_inv = finv<F>((T)n);
    if constexpr (sizeof(T) == 4) {
      zeta_q.assign(n, 0);
      izeta_q.assign(n, 0);
      for (uint32_t k = 1; k < n; ++k) {
        zeta_q[k] = quotient(zeta[k]);
        izeta_q[k] = quotient(izeta[k]);
      }
      n_inv_q = quotient(n_inv);
    }
    ok = true;
  }

  // AbstractNTT::transform_slice (algebra/src/transformation/mod.rs:85)
  void forward(T *a) const {
    for (uint32_t i = 0; i < n; ++i) a[i] = F::canon(a[i]);
    uint32_t k = 1;
    for (uint32_t len = n >> 1; len >= 1; len >>= 1)
      for (uint32_t start = 0; start < n; start += 2 * len) {
        const T w = zeta[k];
        const uint32_t wq = sizeof(T) == 4 ? zeta_q[k] : 0;
        ++k;
        T *__restrict lo = a + start;  // the two halves of a block never overlap
        T *__restrict hi = lo + len;
        for (uint32_t j = 0; j < len; ++j) {
          const T t = bf_mul(hi[j], w, wq);
          const T u = lo[j];
          lo[j] = bf_add(u, t);
          hi[j] = bf_sub(u, t);
        }
      }
    if constexpr (sizeof(T) == 8)
      for (uint32_t i = 0; i < n; ++i) a[i] = F::canon(a[i]);
  }
  // AbstractNTT::inverse_transform_slice (algebra/src/transformation/mod.rs:95): inverse + normalize
  void inverse(T *a) const {
    for (uint32_t i = 0; i < n; ++i) a[i] = F::canon(a[i]);
    for (uint32_t len = 1; len < n; len <<= 1) {
      const uint32_t blocks = n / (2 * len);
      for (uint32_t blk = 0; blk < blocks; ++blk) {
        const T w = izeta[blocks + blk];
        const uint32_t wq = sizeof(T) == 4 ? izeta_q[blocks + blk] : 0;
        T *__restrict lo = a + 2 * len * blk;
        T *__restrict hi = lo + len;
        for (uint32_t j = 0; j < len; ++j) {
          const T u = lo[j], v = hi[j];
          lo[j] = bf_add(u, v);
          hi[j] = bf_mul(bf_sub(u, v), w, wq);
        }
      }
    }
    for (uint32_t i = 0; i < n; ++i) a[i] = mul_q(a[i], n_inv, n_inv_q);
  }
};

template <class F>
const Ntt<F> &ntt_table(uint32_t logn) {
  // NTTField::get_ntt_table caches one table per log_n (algebra/src/goldilocks/goldilocks_ntt.rs:136-160)
  static std::unique_ptr<Ntt<F>> tables[16];
  static std::once_flag flags[16];
  std::call_once(flags[logn], [&] { tables[logn].reset(new Ntt<F>(logn)); });
  return *tables[logn];
}

template <class F>
void schoolbook_negacyclic(const typename F::T *x, const typename F::T *y, typename F::T *out,
                           uint32_t n) {
  using T = typename F::T;
  std::vector<T> acc(n, 0);
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t j = 0; j < n; ++j) {
      T p = F::mul(x[i], y[j]);
      uint32_t k = i + j;
      if (k < n)
        acc[k] = F::add(acc[k], p);
      else
        acc[k - n] = F::sub(acc[k - n], p);
    }
  std::copy(acc.begin(), acc.end(), out);
}

// ------------------------------------------------------------------------------------------
// Seeded PRG and samplers (the project's key convention; the distributions follow
// algebra/src/utils/sample.rs:6-51 and algebra/src/random.rs:82-96,156-171).
// ------------------------------------------------------------------------------------------

inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

inline uint64_t prg(uint64_t seed, uint64_t stream, uint64_t ctr) {
  uint64_t k = mix64(seed + 0x9E3779B97F4A7C15ULL) ^ mix64(stream ^ 0xD1B54A32D192ED03ULL);
  return mix64(k + ctr * 0x9E3779B97F4A7C15ULL);
}

enum : uint64_t { TAG_LWE_SK = 1, TAG_RING_SK = 2, TAG_BSK = 3, TAG_KSK = 4, TAG_ENC = 5 };

inline uint64_t stream_id(uint64_t tag, uint64_t i, uint64_t part, uint64_t j, uint64_t which) {
  return (tag << 56) | ((i & 0xFFFFFFFFULL) << 24) | ((part & 0xFF) << 16) | ((j & 0xFF) << 8) |
         (which & 0xFF);
}

// Natural logarithm for s in (0, 1] from IEEE-exact operations only (frexp, +, -, *, /), so the
// sampled noise is identical on every x86-64 host: ln s = e ln2 + 2 atanh((m-1)/(m+1)).
double ln_exact(double s) {
  int e = 0;
  double m = std::frexp(s, &e);
  if (m < 0.70710678118654752440) {
    m *= 2.0;
    e -= 1;
  }
  double y = (m - 1.0) / (m + 1.0);
  double y2 = y * y;
  double sum = 0.0, term = y;
  for (int k = 0; k < 24; ++k) {
    sum += term / (double)(2 * k + 1);
    term *= y2;
  }
  return 2.0 * sum + (double)e * 0.693147180559945309417232121458;
}

inline double unit_double(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

// FieldDiscreteGaussianSampler::sample (algebra/src/random.rs:156-171): N(0, sigma), reject
// |x| >= 6 sigma, round half away from zero, negative r -> Q - |r|. The normal deviate comes from
// the Marsaglia polar method on the project's PRG.
template <class F>
typename F::T gaussian(uint64_t seed, uint64_t stream, uint64_t coeff, double sigma) {
  const double max_dev = sigma * 6.0;
  for (uint64_t attempt = 0;; ++attempt) {
    uint64_t base = (coeff << 20) | (attempt << 1);
    double u = 2.0 * unit_double(prg(seed, stream, base)) - 1.0;
    double v = 2.0 * unit_double(prg(seed, stream, base | 1)) - 1.0;
    double s = u * u + v * v;
    if (!(s > 0.0 && s < 1.0)) continue;
    double x = u * std::sqrt(-2.0 * ln_exact(s) / s);
    double value = sigma * x;
    if (std::fabs(value) < max_dev) {
      double r = std::round(value);
      if (r < 0.0) return (typename F::T)((uint64_t)F::P - (uint64_t)(-r));
      return (typename F::T)(uint64_t)r;
    }
  }
}

template <class F>
typename F::T uniform(uint64_t seed, uint64_t stream, uint64_t k) {
  return (typename F::T)(prg(seed, stream, k) % (uint64_t)F::P);
}

// random_with_gaussian draws error polynomials from sample_cbd_field_vec instead of the Gaussian
// when the sampler has mean 0 and sigma exactly 3.2 (algebra/src/random.rs:91-92,
// algebra/src/polynomial/univariate/native_polynomial.rs:232-246).
inline bool cbd_enabled(double sigma) { return sigma == 3.2; }

// sample_cbd_field_vec (algebra/src/utils/sample.rs:54-75): six random bytes (here the low six
// bytes of one PRG word), the third and sixth masked to 5 bits; a and b are the popcounts of the
// first and last three. For a < b the reference evaluates `modulus - (a - b)` with a u32
// subtraction that wraps in release builds, so the value is Field::new of that wrapped word in
// the field's word width: b - a for the 32-bit fields, P - (2^32 - (b - a)) for Goldilocks.
template <class F>
typename F::T cbd(uint64_t seed, uint64_t stream, uint64_t coeff) {
  using T = typename F::T;
  const uint64_t r = prg(seed, stream, coeff);
  auto pc = [](uint64_t x) { return (uint32_t)__builtin_popcountll(x); };
  const uint32_t a = pc(r & 0xFF) + pc((r >> 8) & 0xFF) + pc((r >> 16) & 0x1F);
  const uint32_t b = pc((r >> 24) & 0xFF) + pc((r >> 32) & 0xFF) + pc((r >> 40) & 0x1F);
  const uint32_t d = a - b;  // wraps when a < b
  if (a >= b) return (T)d;
  return F::from_u64((uint64_t)(T)((T)F::P - (T)d));
}

// One error coefficient of an RLWE zero sample.
template <class F>
typename F::T error_coeff(uint64_t seed, uint64_t stream, uint64_t coeff, double sigma) {
  return cbd_enabled(sigma) ? cbd<F>(seed, stream, coeff) : gaussian<F>(seed, stream, coeff, sigma);
}

// ------------------------------------------------------------------------------------------
// Parameters
// ------------------------------------------------------------------------------------------

struct Dims {
  uint32_t N, logN, n, bits, len, ks_bits, ks_len;
  uint32_t ks_n, ks_logn, chunks;  // key switch: n' = next_pow2(n), N / n' key chunks
  uint32_t pairs;                  // RGSWs per LWE key coefficient: 1 binary, 2 ternary
};

bool dims_of(const orc_params *p, Dims &d) {
  if (!p) return false;
  if (p->field_id != ORC_FIELD_GOLDILOCKS && p->field_id != ORC_FIELD_BABYBEAR &&
      p->field_id != ORC_FIELD_DEFAULT_U32)
    return false;
  d.N = p->ring_dim;
  d.n = p->lwe_dim;
  if (d.N < 2 || (d.N & (d.N - 1)) || d.N > 4096) return false;
  d.logN = 0;
  while ((1u << d.logN) < d.N) ++d.logN;
  if (d.n == 0 || d.n > d.N) return false;
  // KeySwitchingRLWEKey::generate: extended_lwe_dimension = next_pow2(n) <= N, and the ring key
  // splits into N / n' chunks when it is smaller (fhe_core/src/key_switch/rlwe.rs:40-43,79-108)
  d.ks_n = 1;
  d.ks_logn = 0;
  while (d.ks_n < d.n) {
    d.ks_n <<= 1;
    ++d.ks_logn;
  }
  d.chunks = d.N / d.ks_n;
  // Ternary LWE keys take TernaryBlindRotationKey (fhe_core/src/blind_rotation/rlwe/ternary.rs),
  // whose NTT-domain monomial is marked incompatible with BabyBear and Goldilocks there (:80).
  if (p->lwe_ternary > 1 || (p->lwe_ternary && p->field_id != ORC_FIELD_DEFAULT_U32)) return false;
  d.pairs = p->lwe_ternary ? 2 : 1;
  d.bits = p->br_bits;
  d.len = p->br_len;
  d.ks_bits = p->ks_bits;
  d.ks_len = p->ks_len;
  int fb = field_bits(p->field_id);
  auto want = [&](uint32_t b) { return (uint32_t)((fb + (int)b - 1) / (int)b); };
  if (d.bits == 0 || d.bits > 16 || d.len != want(d.bits)) return false;
  if (d.ks_bits == 0 || d.ks_bits > 16 || d.ks_len != want(d.ks_bits)) return false;
  return true;
}

// ------------------------------------------------------------------------------------------
// Key generation (fhe_core/src/secret_key.rs:67-89, fhe_core/src/blind_rotation/rlwe/binary.rs:207-239,
// lattice/src/rgsw.rs:343-395, lattice/src/gadget/rlwe.rs:478-552, lattice/src/rlwe.rs:1215-1252,
// fhe_core/src/key_switch/rlwe.rs:37-112), restated in the coefficient domain.
// ------------------------------------------------------------------------------------------

template <class F>
void negacyclic_mul(const Ntt<F> &ntt, const typename F::T *x, const typename F::T *y_ntt,
                    typename F::T *out) {
  std::vector<typename F::T> t(x, x + ntt.n);
  ntt.forward(t.data());
  for (uint32_t k = 0; k < ntt.n; ++k) t[k] = F::mul(t[k], y_ntt[k]);
  ntt.inverse(t.data());
  std::copy(t.begin(), t.end(), out);
}

template <class F>
void rlwe_zero_sample(const Ntt<F> &ntt, const typename F::T *key_ntt, uint64_t seed,
                      uint64_t stream_a, uint64_t stream_e, double sigma, typename F::T *a,
                      typename F::T *b) {
  // NTTRLWE::generate_random_zero_sample (lattice/src/rlwe.rs:1215-1230): b = a*s + e
  uint32_t N = ntt.n;
  for (uint32_t k = 0; k < N; ++k) a[k] = uniform<F>(seed, stream_a, k);
  negacyclic_mul<F>(ntt, a, key_ntt, b);
  for (uint32_t k = 0; k < N; ++k) b[k] = F::add(b[k], error_coeff<F>(seed, stream_e, k, sigma));
}

template <class F>
void keygen(const orc_params *p, const Dims &d, uint64_t seed, typename F::T *lwe_sk,
            typename F::T *ring_sk, typename F::T *bsk, typename F::T *ksk, int threads) {
  using T = typename F::T;
  const uint32_t N = d.N, n = d.n;
  const Ntt<F> &ntt = ntt_table<F>(d.logN);
  // sample_binary_field_vec / sample_ternary_field_vec (algebra/src/utils/sample.rs:6-51;
  // fhe_core/src/secret_key.rs:60-63): a bit, or {0, 0, 1, -1}[r & 3]
  const T tern[4] = {0, 0, 1, (T)(F::P - 1)};
  for (uint32_t i = 0; i < n; ++i) {
    const uint64_t r = prg(seed, stream_id(TAG_LWE_SK, 0, 0, 0, 0), i);
    lwe_sk[i] = d.pairs == 2 ? tern[r & 3] : (T)(r & 1);
  }
  // random_with_ternary / random_with_binary (fhe_core/src/secret_key.rs:74-79)
  for (uint32_t k = 0; k < N; ++k) {
    uint64_t r = prg(seed, stream_id(TAG_RING_SK, 0, 0, 0, 0), k);
    ring_sk[k] = p->ring_ternary ? tern[r & 3] : (T)(r & 1);
  }
  std::vector<T> z_ntt(ring_sk, ring_sk + N);
  ntt.forward(z_ntt.data());

  // Blind-rotation key: per LWE key coefficient one NTTRGSW of s_i (binary,
  // fhe_core/src/blind_rotation/rlwe/binary.rs:207-239), or the pair (RGSW(s_i == 1),
  // RGSW(s_i == -1)) (ternary, fhe_core/src/blind_rotation/rlwe/ternary.rs:123-183). Layout
  // [i][pair][part][j][ab][N]; pair 1 draws from streams part + 2.
  const uint32_t L = d.len;
  const size_t row = 2 * (size_t)N;            // one RLWE (a, b)
  const size_t entry = 2 * (size_t)L * row;    // one RGSW = (c_neg_s_m, c_m)
  auto work = [&](uint32_t i0, uint32_t i1) {
    for (uint32_t i = i0; i < i1; ++i) {
      for (uint32_t pair = 0; pair < d.pairs; ++pair) {
        const bool one = d.pairs == 1 ? lwe_sk[i] != 0 : lwe_sk[i] == (pair == 0 ? (T)1 : (T)(F::P - 1));
        T basis_pow = 1;
        for (uint32_t j = 0; j < L; ++j) {
          for (uint32_t part = 0; part < 2; ++part) {
            T *a = bsk + ((size_t)i * d.pairs + pair) * entry + ((size_t)part * L + j) * row;
            T *b = a + N;
            rlwe_zero_sample<F>(ntt, z_ntt.data(), seed, stream_id(TAG_BSK, i, part + 2 * pair, j, 0),
                                stream_id(TAG_BSK, i, part + 2 * pair, j, 1), p->ring_noise_std, a, b);
            if (one && part == 0) {
              // generate_random_neg_secret_sample: every NTT slot of a += B^j, i.e. a[0] += B^j
              // (lattice/src/gadget/rlwe.rs:526-551)
              a[0] = F::add(a[0], basis_pow);
            } else if (one && part == 1) {
              // generate_random_value_sample: e[0] += B^j before the transform (lattice/src/rlwe.rs:1233-1252)
              b[0] = F::add(b[0], basis_pow);
            }
          }
          // basis_power = lazy_new(basis_power.value() * basis) (lattice/src/gadget/rlwe.rs:518,546)
          basis_pow = (T)((uint64_t)basis_pow << d.bits);
        }
      }
    }
  };
  int nt = std::max(1, threads);
  std::vector<std::thread> pool;
  uint32_t chunk = (n + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    uint32_t i0 = t * chunk, i1 = std::min(n, i0 + chunk);
    if (i0 >= i1) break;
    pool.emplace_back(work, i0, i1);
  }
  for (auto &th : pool) th.join();

  // KeySwitchingRLWEKey::generate (fhe_core/src/key_switch/rlwe.rs:37-112): the LWE key padded to
  // n' = next_pow2(n) words; one gadget RLWE of dimension n' per n'-word chunk z_c of the ring key
  // (a single one, z itself, when n' == N). Row j of chunk c encrypts z_c * B_ks^j; layout
  // [c][j][ab][n'].
  const uint32_t M = d.ks_n;
  const Ntt<F> &kntt = ntt_table<F>(d.ks_logn);
  std::vector<T> s_ext(M, 0);
  for (uint32_t i = 0; i < n; ++i) s_ext[i] = lwe_sk[i];
  kntt.forward(s_ext.data());
  const T basis_ks = F::from_u64(1ull << d.ks_bits);
  for (uint32_t c = 0; c < d.chunks; ++c) {
    std::vector<T> zk(ring_sk + (size_t)c * M, ring_sk + (size_t)(c + 1) * M);
    for (uint32_t j = 0; j < d.ks_len; ++j) {
      T *a = ksk + ((size_t)c * d.ks_len + j) * 2 * M;
      T *b = a + M;
      rlwe_zero_sample<F>(kntt, s_ext.data(), seed, stream_id(TAG_KSK, c, 0, j, 0),
                          stream_id(TAG_KSK, c, 0, j, 1), p->ks_noise_std, a, b);
      for (uint32_t k = 0; k < M; ++k) b[k] = F::add(b[k], zk[k]);
      if (j + 1 < d.ks_len)
        for (uint32_t k = 0; k < M; ++k) zk[k] = F::mul(zk[k], basis_ks);
    }
  }
}

// ------------------------------------------------------------------------------------------
// Encode / decode / encrypt / decrypt (fhe_core/src/plaintext.rs:64-97, fhe_core/src/secret_key.rs:129-188)
// ------------------------------------------------------------------------------------------

template <class F>
uint64_t encode(uint64_t m) {
  double qf = (double)(uint64_t)F::P;
  return (uint64_t)std::round((double)m * (qf / 4.0));
}

template <class F>
uint64_t decode(uint64_t c) {
  double qf = (double)(uint64_t)F::P;
  uint64_t r = (uint64_t)std::round((double)c * 4.0 / qf);
  return r < 4 ? r : r - 4;
}

template <class F>
void encrypt(const Dims &d, const orc_params *p, const typename F::T *sk, uint64_t seed,
             uint64_t index, int bit, typename F::T *out) {
  using T = typename F::T;
  // LWE::generate_random_zero_sample_field (lattice/src/lwe.rs:389-404)
  T acc = 0;
  for (uint32_t i = 0; i < d.n; ++i) {
    out[i] = uniform<F>(seed, stream_id(TAG_ENC, index, 0, 0, 0), i);
    acc = F::add(acc, F::mul(out[i], sk[i]));
  }
  T e = gaussian<F>(seed, stream_id(TAG_ENC, index, 0, 0, 1), 0, p->lwe_noise_std);
  T b = F::add(acc, e);
  out[d.n] = F::add(b, F::from_u64(encode<F>((uint64_t)bit)));
}

template <class F>
void decrypt(const Dims &d, const typename F::T *sk, const typename F::T *c, uint8_t *bit,
             uint64_t *noise) {
  using T = typename F::T;
  T acc = 0;
  for (uint32_t i = 0; i < d.n; ++i) acc = F::add(acc, F::mul(F::canon(c[i]), sk[i]));
  T pt = F::sub(F::canon(c[d.n]), acc);
  uint64_t m = decode<F>(F::value(pt));
  if (bit) *bit = (uint8_t)m;
  if (noise) {
    T fresh = F::from_u64(encode<F>(m));
    T x = F::sub(pt, fresh), y = F::sub(fresh, pt);
    *noise = std::min<uint64_t>(x, y);
  }
}

// ------------------------------------------------------------------------------------------
// Bootstrapping
// ------------------------------------------------------------------------------------------

template <class F>
struct EvalKey {
  using T = typename F::T;
  Dims d;
  std::vector<T> bsk_ntt;  // [i][pair][part][j][ab][N] in this oracle's NTT domain
  std::vector<T> ksk_ntt;  // [c][j][ab][n'] (n'-point transforms)
};

template <class F>
EvalKey<F> *make_eval(const Dims &d, const typename F::T *bsk, const typename F::T *ksk,
                      int threads) {
  auto *ek = new EvalKey<F>();
  ek->d = d;
  const Ntt<F> &ntt = ntt_table<F>(d.logN);
  size_t polys = (size_t)d.n * d.pairs * 2 * d.len * 2;
  ek->bsk_ntt.assign(bsk, bsk + polys * d.N);
  int nt = std::max(1, threads);
  std::vector<std::thread> pool;
  size_t chunk = (polys + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    size_t p0 = t * chunk, p1 = std::min(polys, p0 + chunk);
    if (p0 >= p1) break;
    pool.emplace_back([&, p0, p1] {
      for (size_t q = p0; q < p1; ++q) ntt.forward(ek->bsk_ntt.data() + q * d.N);
    });
  }
  for (auto &th : pool) th.join();
  const Ntt<F> &kntt = ntt_table<F>(d.ks_logn);
  const size_t kpolys = (size_t)d.chunks * d.ks_len * 2;
  ek->ksk_ntt.assign(ksk, ksk + kpolys * d.ks_n);
  for (size_t q = 0; q < kpolys; ++q) kntt.forward(ek->ksk_ntt.data() + q * d.ks_n);
  return ek;
}

// lwe_modulus_switch (fhe_core/src/modulus_switch.rs:12-38)
template <class F>
void modswitch(const Dims &d, const typename F::T *c, uint32_t *out) {
  const double before = (double)(uint64_t)F::P;
  const double after = (double)(2 * d.N);
  for (uint32_t i = 0; i <= d.n; ++i) {
    double v = (double)(uint64_t)F::value(c[i]);
    double r = std::round(v * after / before);
    uint64_t t = (uint64_t)r;
    out[i] = (uint32_t)(t < 2ull * d.N ? t : t - 2ull * d.N);
  }
}

// Polynomial::decompose_lsb_bits_inplace (algebra/src/polynomial/univariate/native_polynomial.rs:340-348)
// with Goldilocks/BabyBear::decompose_lsb_bits_at (algebra/src/goldilocks/mod.rs:123-127,
// algebra/src/baby_bear/mod.rs:127-131): digit = value & mask, poly = value >> bits.
template <class F>
void decompose_step(typename F::T *poly, typename F::T *digit, uint32_t N, uint32_t bits) {
  const uint64_t mask = (1ull << bits) - 1;
  for (uint32_t k = 0; k < N; ++k) {
    uint64_t v = (uint64_t)F::value(poly[k]);
    digit[k] = (typename F::T)(v & mask);
    poly[k] = (typename F::T)(v >> bits);
  }
}

// RLWE::mul_monic_monomial_sub_one_inplace (lattice/src/rlwe.rs:437-487): dst = src*(X^r - 1)
template <class F>
void monomial_sub_one(const typename F::T *y, typename F::T *x, uint32_t N, uint32_t r) {
  if (r <= N) {
    uint32_t nsr = N - r;
    for (uint32_t k = 0; k < r; ++k) x[k] = F::neg_ref(y[nsr + k]);
    for (uint32_t k = r; k < N; ++k) x[k] = y[k - r];
  } else {
    uint32_t rr = r - N;
    uint32_t nsr = N - rr;
    for (uint32_t k = 0; k < rr; ++k) x[k] = y[nsr + k];
    for (uint32_t k = rr; k < N; ++k) x[k] = F::neg_ref(y[k - rr]);
  }
  for (uint32_t k = 0; k < N; ++k) x[k] = F::sub_ref(x[k], y[k]);
}

// RLWE::mul_assign_ntt_rgsw (lattice/src/rlwe.rs:573-596): c_neg_s_m x E.a + c_m x E.b, then INTT.
// rgsw_ntt layout [part][j][ab][N]. With `digits` (bits <= 8), the coefficient-domain gadget digits
// go to digits[(part L + j) N + k]: the bit polynomials that the traced product records
// (mul_polynomial_inplace_fast_w_traces, lattice/src/gadget/rlwe.rs:426-457, append_bit_poly).
template <class F>
void external_product(const Ntt<F> &ntt, uint32_t bits, uint32_t L, const typename F::T *rgsw_ntt,
                      typename F::T *ea, typename F::T *eb, uint8_t *digits = nullptr) {
  using T = typename F::T;
  using Acc = typename F::Acc;
  const uint32_t N = ntt.n;
  // Per-thread scratch, addressed through plain pointers inside the loops (a thread_local
  // object's address is looked up per access in a shared library).
  thread_local std::vector<T> tl_w;
  thread_local std::vector<Acc> tl_acc;
  tl_w.resize((size_t)4 * N);
  tl_acc.assign((size_t)2 * N, 0);
  T *ma = tl_w.data(), *mb = ma + N, *poly = mb + N, *digit = poly + N;
  Acc *sa = tl_acc.data(), *sb = sa + N;
  for (uint32_t part = 0; part < 2; ++part) {
    const T *src = part == 0 ? ea : eb;
    std::copy(src, src + N, poly);
    for (uint32_t j = 0; j < L; ++j) {
      decompose_step<F>(poly, digit, N, bits);
      if (digits)
        for (uint32_t k = 0; k < N; ++k) digits[((size_t)part * L + j) * N + k] = (uint8_t)digit[k];
      ntt.forward(digit);
      const T *ka = rgsw_ntt + ((size_t)part * L + j) * 2 * N;
      const T *kb = ka + N;
      // ntt_add_mul_assign_fast (algebra/src/polynomial/univariate/ntt_polynomial.rs:620-629);
      // the sums are exact, so reducing once per slot gives the same canonical result
      for (uint32_t k = 0; k < N; ++k) {
        F::acc_mac(sa[k], digit[k], ka[k]);
        F::acc_mac(sb[k], digit[k], kb[k]);
      }
    }
  }
  for (uint32_t k = 0; k < N; ++k) {
    ma[k] = F::acc_value(sa[k]);
    mb[k] = F::acc_value(sb[k]);
  }
  ntt.inverse(ma);
  ntt.inverse(mb);
  std::copy(ma, ma + N, ea);
  std::copy(mb, mb + N, eb);
}

// One row of an accumulator trace: [a | b] canonical (the rows of AccTrace, trace/src/acc_trace.rs).
template <class F>
void trace_row(const typename F::T *acc_a, const typename F::T *acc_b, uint32_t N, typename F::T *row) {
  for (uint32_t k = 0; k < N; ++k) {
    row[k] = F::canon(acc_a[k]);
    row[N + k] = F::canon(acc_b[k]);
  }
}

// BinaryBlindRotationKey::blind_rotate (fhe_core/src/blind_rotation/rlwe/binary.rs:28-104).
// acc_a/acc_b hold the reference's representation of the accumulator. With `trace`, the accumulator
// after every step i goes to trace[i] (blind_rotate_w_trace, binary.rs:106-205, which does not skip
// a_i = 0; such a step leaves the accumulator unchanged). With `digits`, step i's gadget digits of
// E.a and E.b go to digits[i][2 L][N] (zero for a step with a_i = 0, whose E is zero).
template <class F>
void blind_rotate(const EvalKey<F> &ek, const uint32_t *ms, const typename F::T *lut_in,
                  uint32_t steps, typename F::T *acc_a, typename F::T *acc_b,
                  typename F::T *trace = nullptr, uint8_t *digits = nullptr) {
  using T = typename F::T;
  const Dims &d = ek.d;
  const uint32_t N = d.N;
  const Ntt<F> &ntt = ntt_table<F>(d.logN);
  std::vector<T> lut(lut_in, lut_in + N);
  uint32_t b = ms[d.n];
  if (b != 0) {
    // lut * X^{-b} by rotate_right + negate (binary.rs:40-62)
    uint32_t neg_b = 2 * N - b;
    std::vector<T> t(N);
    if (neg_b <= N) {
      for (uint32_t k = 0; k < N; ++k) t[(k + neg_b) % N] = lut[k];
      for (uint32_t k = 0; k < neg_b; ++k) t[k] = F::neg_ref(t[k]);
    } else {
      uint32_t r = neg_b - N;
      for (uint32_t k = 0; k < N; ++k) t[(k + r) % N] = lut[k];
      for (uint32_t k = r; k < N; ++k) t[k] = F::neg_ref(t[k]);
    }
    lut.swap(t);
  }
  std::fill(acc_a, acc_a + N, (T)0);
  std::copy(lut.begin(), lut.end(), acc_b);
  std::vector<T> ea(N), eb(N);
  const size_t entry = (size_t)2 * d.len * 2 * N;
  for (uint32_t i = 0; i < d.n && i < steps; ++i) {
    const uint32_t ai = ms[i];
    if (ai != 0) {  // binary.rs:70
      monomial_sub_one<F>(acc_a, ea.data(), N, ai);
      monomial_sub_one<F>(acc_b, eb.data(), N, ai);
      external_product<F>(ntt, d.bits, d.len, ek.bsk_ntt.data() + i * entry, ea.data(), eb.data(),
                          digits ? digits + (size_t)i * 2 * d.len * N : nullptr);
      // RLWE::add_assign_element_wise (lattice/src/rlwe.rs:287-290)
      for (uint32_t k = 0; k < N; ++k) {
        acc_a[k] = F::add_ref(acc_a[k], ea[k]);
        acc_b[k] = F::add_ref(acc_b[k], eb[k]);
      }
    }
    if (trace) trace_row<F>(acc_a, acc_b, N, trace + (size_t)i * 2 * N);
  }
}

// NTT of the monomial c * X^deg, deg in [0, 2N) (X^N = -1), as
// MonomialNTT::transform_monomial / transform_coeff_neg_one_monomial
// (algebra/src/transformation/concrete.rs:63-84) produce it.
template <class F>
void monomial_ntt(const Ntt<F> &ntt, typename F::T c, uint32_t deg, typename F::T *out) {
  const uint32_t N = ntt.n;
  std::fill(out, out + N, (typename F::T)0);
  if (deg < N)
    out[deg] = c;
  else
    out[deg - N] = F::neg(c);
  ntt.forward(out);
}

// TernaryBlindRotationKey::blind_rotate (fhe_core/src/blind_rotation/rlwe/ternary.rs:26-119): the
// LUT rotated by an NTT product with X^-b; per step with a_i != 0 the evaluation key
// RGSW(s_i == 1) + RGSW(s_i == -1) * NTT(-X^-a_i) (lattice/src/rgsw.rs:321-338) multiplies
// E = (X^a_i - 1) * ACC and ACC += the product. The fields this path accepts keep canonical words,
// so the reference's representation-level operations are the canonical ones. E is the product
// the reference's comment names (ternary.rs:91), formed here through the transform of the monomial
// X^a_i; the reference's code places +-1 at index a_i of the NTT-domain vector without transforming
// it (:93-100), which depends on concrete-ntt's slot order and is not that product.
template <class F>
void blind_rotate_ternary(const EvalKey<F> &ek, const uint32_t *ms, const typename F::T *lut_in,
                          uint32_t steps, typename F::T *acc_a, typename F::T *acc_b,
                          typename F::T *trace = nullptr) {
  using T = typename F::T;
  const Dims &d = ek.d;
  const uint32_t N = d.N;
  const Ntt<F> &ntt = ntt_table<F>(d.logN);
  std::vector<T> lut(lut_in, lut_in + N), mono(N), t(N);
  const uint32_t b = ms[d.n];
  if (b != 0) {  // ternary.rs:43-56
    monomial_ntt<F>(ntt, (T)1, 2 * N - b, mono.data());
    ntt.forward(lut.data());
    for (uint32_t k = 0; k < N; ++k) lut[k] = F::mul(lut[k], mono[k]);
    ntt.inverse(lut.data());
  }
  std::fill(acc_a, acc_a + N, (T)0);
  std::copy(lut.begin(), lut.end(), acc_b);
  const size_t rgsw = (size_t)2 * d.len * 2 * N;
  std::vector<T> evk(rgsw), ea(N), eb(N);
  for (uint32_t i = 0; i < d.n && i < steps; ++i) {
    const uint32_t ai = ms[i];
    if (ai == 0) {  // ternary.rs:73
      if (trace) trace_row<F>(acc_a, acc_b, N, trace + (size_t)i * 2 * N);
      continue;
    }
    // evaluation_key = RGSW_0 + RGSW_1 * NTT(-X^(2N - a_i)) (ternary.rs:78-89)
    monomial_ntt<F>(ntt, (T)(F::P - 1), 2 * N - ai, mono.data());
    const T *k0 = ek.bsk_ntt.data() + (size_t)i * 2 * rgsw;
    const T *k1 = k0 + rgsw;
    for (size_t q = 0; q < rgsw; ++q) evk[q] = F::add(k0[q], F::mul(k1[q], mono[q % N]));
    // external_product = (X^a_i - 1) * ACC through the NTT (ternary.rs:91-103)
    monomial_ntt<F>(ntt, (T)1, ai, mono.data());
    for (int part = 0; part < 2; ++part) {
      const T *y = part == 0 ? acc_a : acc_b;
      T *e = part == 0 ? ea.data() : eb.data();
      std::copy(y, y + N, t.data());
      ntt.forward(t.data());
      for (uint32_t k = 0; k < N; ++k) t[k] = F::mul(t[k], mono[k]);
      ntt.inverse(t.data());
      for (uint32_t k = 0; k < N; ++k) e[k] = F::sub(t[k], y[k]);
    }
    external_product<F>(ntt, d.bits, d.len, evk.data(), ea.data(), eb.data());
    for (uint32_t k = 0; k < N; ++k) {  // ternary.rs:114
      acc_a[k] = F::add(acc_a[k], ea[k]);
      acc_b[k] = F::add(acc_b[k], eb[k]);
    }
    if (trace) trace_row<F>(acc_a, acc_b, N, trace + (size_t)i * 2 * N);
  }
}

// KeySwitchingRLWEKey::key_switch_for_rlwe (fhe_core/src/key_switch/rlwe.rs:115-137) with
// key_switch_inner (SubAMulS, :250-286) and extract_partial_lwe_locally (lattice/src/rlwe.rs:393-402).
// With n' = next_pow2(n) < N the accumulator's a is first negated at 0 and reversed on [1, N),
// then the same on every n'-word chunk (:123-131), and each chunk is switched with its own key.
template <class F>
void key_switch(const EvalKey<F> &ek, const typename F::T *acc_a, const typename F::T *acc_b,
                typename F::T *out) {
  using T = typename F::T;
  const Dims &d = ek.d;
  const uint32_t N = d.N, M = d.ks_n;
  const Ntt<F> &ntt = ntt_table<F>(d.ks_logn);
  std::vector<T> a(acc_a, acc_a + N);
  if (M != N) {
    a[0] = F::neg_ref(a[0]);
    std::reverse(a.begin() + 1, a.end());
    for (uint32_t c = 0; c < d.chunks; ++c) {
      T *ch = a.data() + (size_t)c * M;
      ch[0] = F::neg_ref(ch[0]);
      std::reverse(ch + 1, ch + M);
    }
  }
  std::vector<T> ia(M, 0), ib(M, F::canon(acc_b[0]));  // NTTRLWE(0, [b0; n'])
  std::vector<T> poly(M), digit(M);
  for (uint32_t c = 0; c < d.chunks; ++c) {
    // sub_assign_gadget_rlwe_mul_polynomial_inplace_fast (lattice/src/rlwe.rs:1147-1166): negate, then add
    for (uint32_t k = 0; k < M; ++k) poly[k] = F::neg_ref(a[(size_t)c * M + k]);
    for (uint32_t j = 0; j < d.ks_len; ++j) {
      decompose_step<F>(poly.data(), digit.data(), M, d.ks_bits);
      ntt.forward(digit.data());
      const T *ka = ek.ksk_ntt.data() + ((size_t)c * d.ks_len + j) * 2 * M;
      const T *kb = ka + M;
      for (uint32_t k = 0; k < M; ++k) {
        ia[k] = F::add(ia[k], F::mul(digit[k], ka[k]));
        ib[k] = F::add(ib[k], F::mul(digit[k], kb[k]));
      }
    }
  }
  ntt.inverse(ia.data());
  ntt.inverse(ib.data());
  out[0] = ia[0];
  for (uint32_t k = 1; k < d.n; ++k) out[k] = F::neg_ref(ia[M - k]);
  out[d.n] = ib[0];
}

// EvaluationKey::bootstrap (tfhe/src/bfhe/evaluate.rs:42-60)
template <class F>
void bootstrap(const EvalKey<F> &ek, const typename F::T *c, const typename F::T *lut,
               typename F::T *out) {
  using T = typename F::T;
  const Dims &d = ek.d;
  std::vector<uint32_t> ms(d.n + 1);
  modswitch<F>(d, c, ms.data());
  std::vector<T> acc_a(d.N), acc_b(d.N);
  if (d.pairs == 2)
    blind_rotate_ternary<F>(ek, ms.data(), lut, d.n, acc_a.data(), acc_b.data());
  else
    blind_rotate<F>(ek, ms.data(), lut, d.n, acc_a.data(), acc_b.data());
  acc_b[0] = F::add_ref(acc_b[0], (T)((uint64_t)F::P >> 3));  // evaluate.rs:52
  key_switch<F>(ek, acc_a.data(), acc_b.data(), out);
}

// LUT builders (tfhe/src/bfhe/evaluate.rs:267-465) with lut_step 1.
template <class F>
void make_lut(int gate, uint32_t N, typename F::T *lut) {
  using T = typename F::T;
  const T q8 = (T)((uint64_t)F::P >> 3);
  const T nq8 = (T)((uint64_t)F::P - q8);
  T lo, hi;
  uint32_t mid;
  switch (gate) {
    case ORC_GATE_NAND: mid = N / 2 + N / 4; lo = q8; hi = nq8; break;
    case ORC_GATE_AND:
    case ORC_GATE_MAJORITY: mid = N / 2 + N / 4; lo = nq8; hi = q8; break;
    case ORC_GATE_OR:
    case ORC_GATE_MUX: mid = N / 4; lo = nq8; hi = q8; break;
    case ORC_GATE_NOR: mid = N / 4; lo = q8; hi = nq8; break;
    case ORC_GATE_XOR: mid = N / 2; lo = nq8; hi = q8; break;
    case ORC_GATE_XNOR: mid = N / 2; lo = q8; hi = nq8; break;
    default: mid = N; lo = 0; hi = 0;
  }
  for (uint32_t k = 0; k < N; ++k) lut[k] = k < mid ? lo : hi;
}

// Evaluator gate front-ends (tfhe/src/bfhe/evaluate.rs:98-262).
template <class F>
void gate_one(const EvalKey<F> &ek, int gate, const typename F::T *c0, const typename F::T *c1,
              const typename F::T *c2, typename F::T *out) {
  using T = typename F::T;
  const Dims &d = ek.d;
  const uint32_t m = d.n + 1;
  std::vector<T> c(m), lut(d.N);
  auto not_ = [&](const T *x, T *y) {  // evaluate.rs:98-105
    for (uint32_t i = 0; i < m; ++i) y[i] = F::neg(x[i]);
    y[d.n] = F::add(y[d.n], (T)((uint64_t)F::P >> 2));
  };
  switch (gate) {
    case ORC_GATE_NOT:
      not_(c0, out);
      return;
    case ORC_GATE_NAND:
    case ORC_GATE_AND:
    case ORC_GATE_OR:
    case ORC_GATE_NOR:
      for (uint32_t i = 0; i < m; ++i) c[i] = F::add(c0[i], c1[i]);
      break;
    case ORC_GATE_XOR:
    case ORC_GATE_XNOR:
      for (uint32_t i = 0; i < m; ++i) {
        T s = F::sub(c0[i], c1[i]);
        c[i] = F::add(s, s);
      }
      break;
    case ORC_GATE_MAJORITY:
      for (uint32_t i = 0; i < m; ++i) c[i] = F::add(F::add(c0[i], c1[i]), c2[i]);
      break;
    case ORC_GATE_MUX: {  // evaluate.rs:245-262
      std::vector<T> nc0(m), t0(m), t1(m);
      not_(c0, nc0.data());
      gate_one<F>(ek, ORC_GATE_AND, c0, c1, nullptr, t0.data());
      gate_one<F>(ek, ORC_GATE_AND, nc0.data(), c2, nullptr, t1.data());
      for (uint32_t i = 0; i < m; ++i) c[i] = F::add(t0[i], t1[i]);
      break;
    }
    default:
      return;
  }
  make_lut<F>(gate, d.N, lut.data());
  bootstrap<F>(ek, c.data(), lut.data(), out);
}

template <class Fn>
void parallel_for(size_t count, int threads, Fn fn) {
  int nt = (int)std::min<size_t>(std::max(1, threads), std::max<size_t>(count, 1));
  if (nt <= 1) {
    for (size_t i = 0; i < count; ++i) fn(i);
    return;
  }
  std::vector<std::thread> pool;
  std::atomic<size_t> next{0};
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&] {
      for (size_t i; (i = next.fetch_add(1)) < count;) fn(i);
    });
  for (auto &th : pool) th.join();
}

}  // namespace

// ------------------------------------------------------------------------------------------
// C API
// ------------------------------------------------------------------------------------------

extern "C" {

int orc_params_preset(int preset, orc_params *out) {
  if (!out) return -1;
  std::memset(out, 0, sizeof(*out));
  out->ring_dim = 1024;
  out->lwe_dim = 728;
  out->ring_ternary = 1;
  out->ks_bits = 5;
  switch (preset) {
    case 0:  // BABYBEAR_BINARY_128_BITS_PARAMETERS (tfhe/src/bfhe/parameters.rs:45-61)
      out->field_id = ORC_FIELD_BABYBEAR;
      out->br_bits = 8;
      out->br_len = 4;
      out->ks_len = 7;
      out->lwe_noise_std = 11000.0;
      out->ring_noise_std = 41.9;
      out->ks_noise_std = 11000.0;
      return 0;
    case 1:  // GOLDILOCKS_BINARY_128_BITS_PARAMETERS (tfhe/src/bfhe/parameters.rs:64-80)
    case 2:  // ZAMA_BINARY_128_BITS_PARAMETERS (tfhe/src/bfhe/parameters.rs:83-98)
      out->field_id = ORC_FIELD_GOLDILOCKS;
      out->br_bits = preset == 1 ? 8 : 5;
      out->br_len = preset == 1 ? 8 : 13;
      out->ks_len = 13;
      out->lwe_noise_std = 2.9 * (double)(1ULL << 45);
      out->ring_noise_std = 2.3 * (double)(1ULL << 37);
      out->ks_noise_std = 2.9 * (double)(1ULL << 45);
      return 0;
    case 3:  // DEFAULT_TERNARY_128_BITS_PARAMETERS (tfhe/src/bfhe/parameters.rs:7-23)
    case 4:  // CUSTOM_TERNARY_128_BITS_PARAMETERS (tfhe/src/bfhe/parameters.rs:26-42)
      // Both sets name their ring "ternary" but configure binary LWE and ring keys.
      out->field_id = ORC_FIELD_DEFAULT_U32;
      out->lwe_dim = preset == 3 ? 1024 : 512;
      out->ring_ternary = 0;
      out->br_bits = preset == 3 ? 3 : 7;
      out->br_len = preset == 3 ? 9 : 4;
      out->ks_bits = preset == 3 ? 1 : 7;
      out->ks_len = preset == 3 ? 27 : 4;
      out->lwe_noise_std = 3.20;
      out->ring_noise_std = 3.20 * 2.0;
      out->ks_noise_std = 3.2 * 2.0;
      return 0;
    default:
      return -1;
  }
}

uint64_t orc_prg(uint64_t seed, uint64_t stream, uint64_t ctr) { return prg(seed, stream, ctr); }

#define ORC_DISPATCH(p, BODY)                                  \
  do {                                                         \
    if ((p)->field_id == ORC_FIELD_GOLDILOCKS) {               \
      using F = Gold;                                          \
      BODY;                                                    \
    } else if ((p)->field_id == ORC_FIELD_BABYBEAR) {          \
      using F = Baby;                                          \
      BODY;                                                    \
    } else if ((p)->field_id == ORC_FIELD_DEFAULT_U32) {       \
      using F = Dflt;                                          \
      BODY;                                                    \
    } else {                                                   \
      return -1;                                               \
    }                                                          \
  } while (0)

int orc_keygen(const orc_params *p, uint64_t seed, void *lwe_sk, void *ring_sk, void *bsk,
               void *ksk, int threads) {
  Dims d;
  if (!dims_of(p, d) || !lwe_sk || !ring_sk || !bsk || !ksk) return -1;
  ORC_DISPATCH(p, {
    using T = F::T;
    keygen<F>(p, d, seed, (T *)lwe_sk, (T *)ring_sk, (T *)bsk, (T *)ksk, threads);
  });
  return 0;
}

int orc_encrypt(const orc_params *p, const void *lwe_sk, uint64_t seed, uint64_t index0,
                const uint8_t *bits, size_t count, void *lwe_out) {
  Dims d;
  if (!dims_of(p, d)) return -1;
  ORC_DISPATCH(p, {
    using T = F::T;
    for (size_t i = 0; i < count; ++i)
      encrypt<F>(d, p, (const T *)lwe_sk, seed, index0 + i, bits[i] & 1,
                 (T *)lwe_out + i * (d.n + 1));
  });
  return 0;
}

int orc_decrypt(const orc_params *p, const void *lwe_sk, const void *lwe, size_t count,
                uint8_t *bits_out, uint64_t *noise_out) {
  Dims d;
  if (!dims_of(p, d)) return -1;
  ORC_DISPATCH(p, {
    using T = F::T;
    for (size_t i = 0; i < count; ++i)
      decrypt<F>(d, (const T *)lwe_sk, (const T *)lwe + i * (d.n + 1),
                 bits_out ? bits_out + i : nullptr, noise_out ? noise_out + i : nullptr);
  });
  return 0;
}

struct orc_eval {
  orc_params p;
  Dims d;
  void *ek;  // EvalKey<F> of the parameter set's field
};

int orc_eval_create(const orc_params *p, const void *bsk, const void *ksk, int threads, orc_eval **out) {
  Dims d;
  if (!out || !dims_of(p, d)) return -1;
  *out = nullptr;
  ORC_DISPATCH(p, {
    using T = F::T;
    orc_eval *e = new orc_eval();
    e->p = *p;
    e->d = d;
    e->ek = make_eval<F>(d, (const T *)bsk, (const T *)ksk, threads);
    *out = e;
  });
  return 0;
}

void orc_eval_free(orc_eval *e) {
  if (!e) return;
  if (e->p.field_id == ORC_FIELD_GOLDILOCKS)
    delete (EvalKey<Gold> *)e->ek;
  else if (e->p.field_id == ORC_FIELD_BABYBEAR)
    delete (EvalKey<Baby> *)e->ek;
  else
    delete (EvalKey<Dflt> *)e->ek;
  delete e;
}

int orc_eval_gate(const orc_eval *e, int gate, const void *c0, const void *c1, const void *c2,
                  void *out, size_t count, int threads) {
  if (!e || gate < 0 || gate > ORC_GATE_MUX) return -1;
  if ((gate == ORC_GATE_MAJORITY || gate == ORC_GATE_MUX) && !c2) return -1;
  const Dims &d = e->d;
  ORC_DISPATCH(&e->p, {
    using T = F::T;
    const EvalKey<F> &ek = *(const EvalKey<F> *)e->ek;
    const size_t m = d.n + 1;
    parallel_for(count, threads, [&](size_t i) {
      gate_one<F>(ek, gate, (const T *)c0 + i * m, c1 ? (const T *)c1 + i * m : nullptr,
                  c2 ? (const T *)c2 + i * m : nullptr, (T *)out + i * m);
    });
  });
  return 0;
}

int orc_gate(const orc_params *p, const void *bsk, const void *ksk, int gate, const void *c0,
             const void *c1, const void *c2, void *out, size_t count, int threads) {
  Dims d;
  if (!dims_of(p, d) || gate < 0 || gate > ORC_GATE_MUX) return -1;
  if ((gate == ORC_GATE_MAJORITY || gate == ORC_GATE_MUX) && !c2) return -1;
  ORC_DISPATCH(p, {
    using T = F::T;
    std::unique_ptr<EvalKey<F>> ek(make_eval<F>(d, (const T *)bsk, (const T *)ksk, threads));
    const size_t m = d.n + 1;
    parallel_for(count, threads, [&](size_t i) {
      gate_one<F>(*ek, gate, (const T *)c0 + i * m, c1 ? (const T *)c1 + i * m : nullptr,
                  c2 ? (const T *)c2 + i * m : nullptr, (T *)out + i * m);
    });
  });
  return 0;
}

int orc_bootstrap_lut(const orc_params *p, const void *bsk, const void *ksk, const void *c,
                      const void *lut, void *out, size_t count, int threads) {
  Dims d;
  if (!dims_of(p, d)) return -1;
  ORC_DISPATCH(p, {
    using T = F::T;
    std::unique_ptr<EvalKey<F>> ek(make_eval<F>(d, (const T *)bsk, (const T *)ksk, threads));
    const size_t m = d.n + 1;
    parallel_for(count, threads, [&](size_t i) {
      bootstrap<F>(*ek, (const T *)c + i * m, (const T *)lut, (T *)out + i * m);
    });
  });
  return 0;
}

int orc_modswitch(const orc_params *p, const void *c, uint32_t *out) {
  Dims d;
  if (!dims_of(p, d)) return -1;
  ORC_DISPATCH(p, { modswitch<F>(d, (const F::T *)c, out); });
  return 0;
}

// The accumulator after `steps` steps (acc_out: 2N words), and with `trace` every step's row.
static int blind_rotate_probe(const orc_params *p, const void *bsk, const void *c, const void *lut,
                       uint32_t steps, void *acc_out, void *trace, uint8_t *digits = nullptr) {
  Dims d;
  if (!dims_of(p, d)) return -1;
  ORC_DISPATCH(p, {
    using T = F::T;
    // only the first `steps` BSK entries are needed: transform just those
    Dims dd = d;
    std::unique_ptr<EvalKey<F>> ek(new EvalKey<F>());
    ek->d = dd;
    const Ntt<F> &ntt = ntt_table<F>(d.logN);
    uint32_t used = std::min(steps, d.n);
    size_t entry = (size_t)d.pairs * 2 * d.len * 2 * d.N;
    ek->bsk_ntt.assign((const T *)bsk, (const T *)bsk + used * entry);
    for (size_t q = 0; q < used * (size_t)d.pairs * 2 * d.len * 2; ++q)
      ntt.forward(ek->bsk_ntt.data() + q * d.N);
    std::vector<uint32_t> ms(d.n + 1);
    modswitch<F>(d, (const T *)c, ms.data());
    T *acc = (T *)acc_out;
    if (d.pairs == 2)
      blind_rotate_ternary<F>(*ek, ms.data(), (const T *)lut, used, acc, acc + d.N, (T *)trace);
    else
      blind_rotate<F>(*ek, ms.data(), (const T *)lut, used, acc, acc + d.N, (T *)trace, digits);
    for (uint32_t k = 0; k < 2 * d.N; ++k) acc[k] = F::canon(acc[k]);
  });
  return 0;
}

int orc_blind_rotate(const orc_params *p, const void *bsk, const void *c, const void *lut,
                     uint32_t steps, void *acc_out) {
  return blind_rotate_probe(p, bsk, c, lut, steps, acc_out, nullptr);
}

int orc_blind_rotate_trace(const orc_params *p, const void *bsk, const void *c, const void *lut,
                           void *trace_out, void *digits_out) {
  if (!p || !trace_out) return -1;
  if (digits_out && (p->br_bits > 8 || p->lwe_ternary)) return -1;
  if (digits_out)
    std::memset(digits_out, 0, (size_t)p->lwe_dim * 2 * p->br_len * p->ring_dim);
  std::vector<uint64_t> acc(2 * (size_t)p->ring_dim);  // room for either word size
  return blind_rotate_probe(p, bsk, c, lut, p->lwe_dim, acc.data(), trace_out, (uint8_t *)digits_out);
}

int orc_ntt_roundtrip(int field_id, uint32_t log_n, const void *in, void *out) {
  if (log_n < 1 || log_n > 15) return -1;
  orc_params p;
  p.field_id = field_id;
  ORC_DISPATCH(&p, {
    using T = F::T;
    const Ntt<F> &ntt = ntt_table<F>(log_n);
    if (!ntt.ok) return -1;
    std::vector<T> t((const T *)in, (const T *)in + ntt.n);
    ntt.forward(t.data());
    ntt.inverse(t.data());
    std::copy(t.begin(), t.end(), (T *)out);
  });
  return 0;
}

int orc_negacyclic_mul(int field_id, uint32_t log_n, const void *x, const void *y, void *out,
                       int schoolbook) {
  if (log_n < 1 || log_n > 15) return -1;
  orc_params p;
  p.field_id = field_id;
  ORC_DISPATCH(&p, {
    using T = F::T;
    const uint32_t n = 1u << log_n;
    if (schoolbook) {
      schoolbook_negacyclic<F>((const T *)x, (const T *)y, (T *)out, n);
    } else {
      const Ntt<F> &ntt = ntt_table<F>(log_n);
      if (!ntt.ok) return -1;
      std::vector<T> yy((const T *)y, (const T *)y + n);
      ntt.forward(yy.data());
      negacyclic_mul<F>(ntt, (const T *)x, yy.data(), (T *)out);
    }
  });
  return 0;
}

int orc_external_product(int field_id, uint32_t log_n, uint32_t bits, uint32_t len,
                         const void *rlwe, const void *rgsw, void *out, size_t count,
                         int threads) {
  if (log_n < 1 || log_n > 15 || bits == 0 || bits > 16 || len == 0) return -1;
  orc_params p;
  p.field_id = field_id;
  ORC_DISPATCH(&p, {
    using T = F::T;
    const Ntt<F> &ntt = ntt_table<F>(log_n);
    if (!ntt.ok) return -1;
    const uint32_t n = 1u << log_n;
    std::vector<T> k((const T *)rgsw, (const T *)rgsw + (size_t)2 * len * 2 * n);
    for (size_t q = 0; q < (size_t)2 * len * 2; ++q) ntt.forward(k.data() + q * n);
    parallel_for(count, threads, [&](size_t i) {
      std::vector<T> a((const T *)rlwe + i * 2 * n, (const T *)rlwe + i * 2 * n + n);
      std::vector<T> b((const T *)rlwe + i * 2 * n + n, (const T *)rlwe + (i + 1) * 2 * n);
      external_product<F>(ntt, bits, len, k.data(), a.data(), b.data());
      std::copy(a.begin(), a.end(), (T *)out + i * 2 * n);
      std::copy(b.begin(), b.end(), (T *)out + i * 2 * n + n);
    });
  });
  return 0;
}

}  // extern "C"
