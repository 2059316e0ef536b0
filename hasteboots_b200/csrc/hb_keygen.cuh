// hb_keygen.cuh -- key generation and LWE encryption on the device, word for word what the host
// generator (hb_client.cpp) produces under the project's seeded key convention (hb_sample.cuh).
//
//  * keygen_rows_kernel   RGSW / key-switching rows: RLWE zero samples b = a * key + e plus their
//                         message, stored transformed, scaled and in the bootstrap kernel's slot
//                         layout -- the words prepare_polys_kernel makes of the host's rows
//  * lwe_encrypt_kernel   LWE encryptions of bits, one warp per ciphertext
#pragma once

#include "hb_field.cuh"
#include "hb_ntt.cuh"
#include "hb_sample.cuh"
#include "hb_sync.cuh"

namespace hb {

template <class W>
struct KeygenParams {
  W *out;             // rows x 2N words: a then b of every row, transformed, scaled, slot layout
  const W *key;       // NTT(key) * N^-1 in the slot layout (prepare_polys_kernel of the key)
  const W *lwe_sk;    // n words: BSK rows encrypt one where the key coefficient selects them
  const W *ring_sk;   // N words: KSK rows encrypt the ring key's chunk z_c times B_ks^j
  const W *tw, *itw;
  W scale;            // the key scale of the tables (N^-1, and R for the 32-bit fields)
  unsigned long long seed;
  double sigma;
  uint32_t rows;
  uint32_t ksk;       // 0: BSK rows [i][pair][part][j]; 1: KSK rows [c][j]
  uint32_t n, len, bits, pairs;
  uint32_t ks_n, ks_len;
  W ks_pow[64];       // B_ks^j mod P in the multiplier form of F::mul
};

// One RLWE row per group of T threads (two groups per block). BSK row (i, pair, part, j)
// (NTTRGSW::generate_random_{zero,one}_sample, lattice/src/rgsw.rs:343-395): a uniform, b = a*z + e
// under the ring key z, plus B^j on a[0] (part 0) or b[0] (part 1) when the RGSW encrypts one.
// KSK row (c, j) (fhe_core/src/key_switch/rlwe.rs:57-108): a uniform in dimension n', b = a*s + e
// under the LWE key padded to n' words, plus z_c * B_ks^j; with n' < N every n'-word polynomial
// sits at every (N/n')-th of N slots (the ring embedding the bootstrap kernel's key switch uses).
template <class F, int LOGN, int T>
__global__ void __launch_bounds__(2 * T) keygen_rows_kernel(const KeygenParams<typename F::W> p) {
  using W = typename F::W;
  using NT = GroupNtt<F, LOGN, T>;
  constexpr int N = 1 << LOGN, V = NT::V, TWN = N * F::TW_WORDS;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  W *s_tw = reinterpret_cast<W *>(smem_raw);
  W *s_itw = s_tw + TWN;
  W *s_x = s_itw + TWN;
  const int g = threadIdx.x / T, t = threadIdx.x % T;
  for (int i = threadIdx.x; i < TWN; i += blockDim.x) {
    s_tw[i] = p.tw[i];
    s_itw[i] = p.itw[i];
  }
  __syncthreads();
  GroupSync<T> sync{1 + g};
  W *xbuf = s_x + g * 2 * N;
  int ping = 0;
  const uint32_t stride = p.ksk ? N / p.ks_n : 1;
  for (uint32_t row = blockIdx.x * 2 + g; row < p.rows; row += gridDim.x * 2) {
    uint64_t sa, se;
    bool one = false;
    uint32_t part = 0, c = 0, j = 0;
    if (!p.ksk) {
      const uint32_t L = p.len, i = row / (p.pairs * 2 * L), pair = (row / (2 * L)) % p.pairs;
      part = (row / L) % 2;
      j = row % L;
      sa = smp::stream_of(smp::kTagBsk, i, part + 2 * pair, j, 0);
      se = smp::stream_of(smp::kTagBsk, i, part + 2 * pair, j, 1);
      const W s = p.lwe_sk[i];
      one = p.pairs == 1 ? s != 0 : s == (pair == 0 ? (W)1 : (W)(F::P - 1));
    } else {
      c = row / p.ks_len;
      j = row % p.ks_len;
      sa = smp::stream_of(smp::kTagKsk, c, 0, j, 0);
      se = smp::stream_of(smp::kTagKsk, c, 0, j, 1);
    }
    const W bj = p.ksk ? (W)0 : (W)(1ULL << (j * p.bits));  // B^j < 2^(bits(Q) - 1) <= P
    const bool amod = !p.ksk && one && part == 0;
    W *out_a = p.out + (size_t)row * 2 * N;
    W *out_b = out_a + N;

    // a (coefficient k of an n'-word row at slot k * stride), its transform and a * key
    W x[V], y[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const uint32_t k = (uint32_t)NT::natural_pos(t, v);
      x[v] = k % stride ? (W)0 : smp::sample_uniform<F>(p.seed, sa, k / stride);
    }
    NT::forward(x, xbuf, ping, s_tw, t, sync);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      y[v] = F::mul(x[v], p.key[v * T + t]);
      if (!amod) out_a[v * T + t] = F::mul(x[v], p.scale);
    }
    NT::inverse(y, xbuf, ping, s_itw, t, sync);
    // b = a * key + e + message, canonical, then transformed like a host row at upload
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const uint32_t k = (uint32_t)NT::natural_pos(t, v);
      W b = F::canon(y[v]);
      if (k % stride == 0) {
        const uint32_t u = k / stride;
        b = smp::add_mod<F>(b, smp::error_coeff<F>(p.seed, se, u, p.sigma));
        if (!p.ksk) {
          if (one && part == 1 && k == 0) b = smp::add_mod<F>(b, bj);
        } else {
          const W z = p.ring_sk[c * p.ks_n + u];
          b = smp::add_mod<F>(b, F::canon(F::mul(z, p.ks_pow[j])));
        }
      }
      y[v] = b;
    }
    NT::forward(y, xbuf, ping, s_tw, t, sync);
#pragma unroll
    for (int v = 0; v < V; ++v) out_b[v * T + t] = F::mul(y[v], p.scale);
    if (amod) {  // a[0] += B^j after b was formed (lattice/src/gadget/rlwe.rs:526-551)
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const uint32_t k = (uint32_t)NT::natural_pos(t, v);
        const W a = smp::sample_uniform<F>(p.seed, sa, k);
        x[v] = k == 0 ? smp::add_mod<F>(a, bj) : a;
      }
      NT::forward(x, xbuf, ping, s_tw, t, sync);
#pragma unroll
      for (int v = 0; v < V; ++v) out_a[v * T + t] = F::mul(x[v], p.scale);
    }
  }
}

// Exact canonical a * b mod P of canonical words.
template <class F>
__device__ __forceinline__ typename F::W mul_mod(typename F::W a, typename F::W b) {
  if constexpr (sizeof(typename F::W) == 8)
    return F::canon(F::mul(a, b));
  else
    return (typename F::W)(((uint64_t)a * b) % F::P);
}

// SecretKeyPack::encrypt (fhe_core/src/secret_key.rs:129-149) of bits[c] with sample index
// index0 + c: a uniform, b = <a, s> + e + round(m Q / 4). One warp per ciphertext.
template <class F>
__global__ void __launch_bounds__(256) lwe_encrypt_kernel(const typename F::W *__restrict__ sk,
                                                           const uint8_t *__restrict__ bits,
                                                           typename F::W *__restrict__ out,
                                                           unsigned long long count, uint32_t n,
                                                           unsigned long long seed,
                                                           unsigned long long index0, double sigma) {
  using W = typename F::W;
  const int lane = threadIdx.x & 31;
  const unsigned long long warps = (unsigned long long)gridDim.x * (blockDim.x / 32);
  for (unsigned long long ct = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; ct < count; ct += warps) {
    const unsigned long long idx = index0 + ct;
    const uint64_t sa = smp::stream_of(smp::kTagEnc, idx, 0, 0, 0);
    W *o = out + ct * (n + 1);
    W dot = 0;
    for (uint32_t i = lane; i < n; i += 32) {
      const W a = smp::sample_uniform<F>(seed, sa, i);
      o[i] = a;
      dot = smp::add_mod<F>(dot, mul_mod<F>(a, sk[i]));
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) dot = smp::add_mod<F>(dot, __shfl_xor_sync(0xFFFFFFFFu, dot, off));
    if (lane == 0) {
      const W e = smp::sample_gauss<F>(seed, smp::stream_of(smp::kTagEnc, idx, 0, 0, 1), 0, sigma);
      const W m = (W)smp::encode_msg<F>(bits[ct] & 1);
      o[n] = smp::add_mod<F>(smp::add_mod<F>(dot, e), m);
    }
  }
}

}  // namespace hb
