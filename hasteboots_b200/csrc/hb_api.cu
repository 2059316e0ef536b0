// hb_api.cu -- device context, NTT tables, key upload and kernel launches behind include/hb_gpu.h.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hb_gpu.h"
#include "hb_keygen.cuh"
#include "hb_kernels.cuh"
#include "hb_launch.cuh"
#include "hb_runtime.h"

using hb::BabyBear;
using hb::DefaultFieldU32;
using hb::GateJob;
using hb::Goldilocks;

// ------------------------------------------------------------------------------------------
// Context helpers
// ------------------------------------------------------------------------------------------

namespace hbrt {

int fail(hb_ctx *ctx, int code, const char *fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

int cuda_fail(hb_ctx *ctx, cudaError_t e, const char *what) {
  return fail(ctx, HB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int dev_alloc(hb_ctx *ctx, size_t bytes, void **out) {
  *out = nullptr;
  if (bytes == 0) return HB_OK;
  if (ctx->budget && ctx->in_use + bytes > ctx->budget)
    return fail(ctx, HB_ERR_NOMEM, "allocation of %zu bytes exceeds the HBM budget (%zu of %zu in use)",
                bytes, ctx->in_use, ctx->budget);
  cudaError_t e = cudaMalloc(out, bytes);
  if (e != cudaSuccess) {
    *out = nullptr;
    return cuda_fail(ctx, e, "cudaMalloc");
  }
  ctx->in_use += bytes;
  ctx->sizes.push_back({*out, bytes});
  return HB_OK;
}

void dev_free(hb_ctx *ctx, void *p) {
  if (!p) return;
  for (size_t i = 0; i < ctx->sizes.size(); ++i)
    if (ctx->sizes[i].first == p) {
      ctx->in_use -= ctx->sizes[i].second;
      ctx->sizes.erase(ctx->sizes.begin() + i);
      break;
    }
  cudaFree(p);
}

// Grow-only scratch buffer owned by the context.
int scratch(hb_ctx *ctx, Scratch &s, size_t bytes) {
  if (s.cap >= bytes) return HB_OK;
  dev_free(ctx, s.ptr);
  s.ptr = nullptr;
  s.cap = 0;
  int rc = dev_alloc(ctx, bytes, &s.ptr);
  if (rc == HB_OK) s.cap = bytes;
  return rc;
}

uint32_t brv(uint32_t x, uint32_t bits) {
  uint32_t r = 0;
  for (uint32_t b = 0; b < bits; ++b) r |= ((x >> b) & 1u) << (bits - 1 - b);
  return r;
}

// Device twiddle tables for a group NTT with 2^logv words per thread. Entry layout within each
// stage follows GroupNtt::fwd_stage / inv_stage (hb_ntt.cuh): the twiddle of block i = high*K + k
// is stored at stage_base + k * (stage_size / K) + high.
template <class F>
int build_tables(hb_ctx *ctx, uint32_t logn, uint32_t logv, DevTables &t) {
  using W = typename F::W;
  const uint32_t N = 1u << logn;
  const uint32_t V = 1u << logv;
  const uint64_t order = (uint64_t)F::P - 1;
  if (order % (2ull * N)) return fail(ctx, HB_ERR_UNSUPPORTED, "2N does not divide Q-1");
  W psi = 0;
  for (W g = 2; g < 64 && !psi; ++g) {
    W c = hb::host_powmod<F>(g, order / (2ull * N));
    if (hb::host_powmod<F>(c, N) == (W)(F::P - 1)) psi = c;
  }
  if (F::SMALL_FIRST_GEN) {
    // Pick the primitive 2N-th root whose (2N/64)-th power is 8, so psi^(N/2) = 8^16 = 2^48 and the
    // first forward stage on gadget digits is a shift (Goldilocks::ct_small_first).
    const W omega = hb::host_powmod<F>(psi, 2ull * N / 64);
    W chosen = 0;
    for (uint32_t j = 1; j < 64 && !chosen; j += 2)
      if (hb::host_powmod<F>(omega, j) == (W)F::SMALL_FIRST_GEN) chosen = hb::host_powmod<F>(psi, j);
    if (!chosen || hb::host_powmod<F>(chosen, N / 2) != (W)(1ULL << 48))
      return fail(ctx, HB_ERR_UNSUPPORTED, "no root of unity with the required power of two");
    psi = chosen;
  }
  const W psi_inv = hb::host_powmod<F>(psi, order - 1);
  using Tw = typename F::Tw;  // the twiddle (and for the 32-bit fields its Shoup quotient)
  std::vector<W> pw(N), ipw(N);
  std::vector<Tw> tw(N, F::make_tw(0)), itw(N, F::make_tw(0));
  W a = 1, b = 1;
  for (uint32_t i = 0; i < N; ++i) {
    pw[i] = a;
    ipw[i] = b;
    a = hb::host_mulmod<F>(a, psi);
    b = hb::host_mulmod<F>(b, psi_inv);
  }
  if (F::SMALL_FIRST_GEN) {
    // The first forward pass multiplies by its twiddles with shifts (GroupNtt::pow2_stage): stages
    // s <= 4 must hold psi^e = 2^(96 e / N).
    for (uint32_t s = 0; s <= 4 && s < logn; ++s)
      for (uint32_t i = 0; i < (1u << s); ++i) {
        const uint32_t e = brv((1u << s) + i, logn);
        if ((96ull * e) % N || pw[e] != hb::host_powmod<F>((W)2, (96ull * e) / N))
          return fail(ctx, HB_ERR_UNSUPPORTED, "twiddle psi^%u is not the expected power of two", e);
      }
  }
  for (uint32_t bb = 0; bb < logn; ++bb) {
    // forward stage s = logn-1-bb: blocks i in [0, 2^s), twiddle psi^brv(2^s + i)
    {
      const uint32_t s = logn - 1 - bb;
      const uint32_t p = (logn - 1 - bb) / logv;
      const int lo_i = (int)logn - (int)((p + 1) * logv);
      const uint32_t lo = lo_i > 0 ? (uint32_t)lo_i : 0;
      const uint32_t rb = bb - lo;
      const uint32_t K = V >> (rb + 1), highs = (1u << s) / K;
      for (uint32_t i = 0; i < (1u << s); ++i)
        tw[(1u << s) + (i % K) * highs + i / K] = F::make_tw(pw[brv((1u << s) + i, logn)]);
    }
    // inverse stage on bit bb: blocks i in [0, H), twiddle psi^-brv(H + i)
    {
      const uint32_t H = N >> (bb + 1);
      const uint32_t b0 = (bb / logv) * logv;
      const uint32_t lo = std::min(b0, logn - logv);
      const uint32_t rb = bb - lo;
      const uint32_t K = V >> (rb + 1), highs = H / K;
      for (uint32_t i = 0; i < H; ++i)
        itw[H + (i % K) * highs + i / K] = F::make_tw(ipw[brv(H + i, logn)]);
    }
  }
  if (F::RADIX8 && logv == 3) {
    // Radix-8 passes (GroupNtt::fwd_r8 / inv_r8): every forward pass but the first, and every
    // inverse pass, that spans three stages holds theta_m^k (theta_m^-k) at 2^S0 + (k-1) 2^S0 + m,
    // theta_m = psi^brv(2^(S0+2) + 4m) for the 2^S0 blocks of its first stage S0.
    auto fill = [&](std::vector<Tw> &tab, uint32_t s0, bool inverse) {
      const uint32_t blocks = 1u << s0;
      for (uint32_t m = 0; m < blocks; ++m) {
        const uint32_t e = brv((1u << (s0 + 2)) + 4 * m, logn);
        const W th = inverse ? ipw[e] : pw[e];
        W pk = th;
        for (uint32_t k = 1; k < 8; ++k) {
          tab[blocks + (k - 1) * blocks + m] = F::make_tw(pk);
          pk = hb::host_mulmod<F>(pk, th);
        }
      }
    };
    for (int top = (int)logn - 3; top >= 3; top -= 3) fill(tw, logn - (uint32_t)top, false);
    for (uint32_t b0 = 0; b0 + 3 <= logn; b0 += 3) fill(itw, logn - 3 - b0, true);
  }
  const W ninv = hb::host_powmod<F>((W)N, order - 1);
  t.n_inv = F::to_mont(ninv);
  // keys: mul(x, scale) must give x * N^-1 in the Montgomery domain of the key words
  t.key_scale = F::to_mont(F::to_mont(ninv));
  if (sizeof(W) == 8) t.key_scale = ninv;
  void *dtw = nullptr, *ditw = nullptr;
  int rc = dev_alloc(ctx, sizeof(Tw) * N, &dtw);
  if (rc) return rc;
  rc = dev_alloc(ctx, sizeof(Tw) * N, &ditw);
  if (rc) {
    dev_free(ctx, dtw);
    return rc;
  }
  cudaMemcpy(dtw, tw.data(), sizeof(Tw) * N, cudaMemcpyHostToDevice);
  cudaMemcpy(ditw, itw.data(), sizeof(Tw) * N, cudaMemcpyHostToDevice);
  t.tw = dtw;
  t.itw = ditw;
  return HB_OK;
}

int tables(hb_ctx *ctx, int field_id, uint32_t logn, DevTables **out, uint32_t logv) {
  if (logn < 6 || logn > 12 || logv < 1 || logv > 5 || field_id < 0 || field_id > 2)
    return fail(ctx, HB_ERR_UNSUPPORTED, "no NTT tables for field %d log_n %u", field_id, logn);
  DevTables &t = ctx->tables[field_id][logn][logv];
  if (!t.tw) {
    int rc = field_id == HB_FIELD_GOLDILOCKS ? build_tables<Goldilocks>(ctx, logn, logv, t)
             : field_id == HB_FIELD_BABYBEAR ? build_tables<BabyBear>(ctx, logn, logv, t)
                                             : build_tables<DefaultFieldU32>(ctx, logn, logv, t);
    if (rc) return rc;
  }
  *out = &t;
  return HB_OK;
}

int check_status(hb_ctx *ctx) {
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "kernel execution");
  if (h) {
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return fail(ctx, HB_ERR_TIMEOUT, "a device-side wait exceeded its limit (status %d)", h);
  }
  return HB_OK;
}

// ~2 s of SM clocks per bounded wait unless the context sets another limit (hb_ctx_set_wait_limit)
long long wait_budget(const hb_ctx *ctx) { return ctx && ctx->wait_limit > 0 ? ctx->wait_limit : 4000000000LL; }

uint64_t modulus_of(int field_id) {
  return field_id == HB_FIELD_GOLDILOCKS ? Goldilocks::P
         : field_id == HB_FIELD_BABYBEAR ? (uint64_t)BabyBear::P
                                         : (uint64_t)DefaultFieldU32::P;
}

// The key switch's dimension n' = next_pow2(n) (fhe_core/src/key_switch/rlwe.rs:40-43).
uint32_t ks_dim(const hb_params &p) {
  uint32_t m = 1;
  while (m < p.lwe_dim) m <<= 1;
  return m;
}

// Twiddle tables of bootstrap_dp_kernel for keys laid out for T threads, for one CTA per gate and
// for the cluster form: those of its groups' digit transforms (hb::dp_group_threads) and of its
// half-CTA groups (words per thread: hb::dp_wide_words).
int dp_tables(hb_ctx *ctx, const hb_params &p, int T) {
  if (p.ring_dim != 1024) return HB_OK;
  const int ws = p.field_id == HB_FIELD_GOLDILOCKS ? 8 : 4;
  for (int cl = 0; cl < 2; ++cl) {
    // hb::dp_group_threads, hb::dp_groups: the groups' own transforms and the half-CTA groups'
    const int tg = ws == 4 && cl ? 128 : T, D = ws == 8 ? 4 : 512 / tg;
    for (int words : {1024 / tg, 1024 / (D / 2 * tg)}) {
      uint32_t logv = 0;
      while ((1 << logv) < words) ++logv;
      DevTables *tb;
      const int rc = tables(ctx, p.field_id, 10, &tb, logv);
      if (rc) return rc;
    }
  }
  return HB_OK;
}

// Device words of the key-switching key: every n'-word chunk key polynomial spread to N words.
size_t ksk_device_words(const hb_params &p) {
  return (size_t)(p.ring_dim / ks_dim(p)) * p.ks_len * 2 * p.ring_dim;
}

}  // namespace hbrt

using namespace hbrt;

// ------------------------------------------------------------------------------------------
// Kernel configurations
// ------------------------------------------------------------------------------------------

namespace {

constexpr int kStages = 3;

template <class F, int LOGN, int T>
int launch_prepare(hb_ctx *ctx, const void *d_in, void *d_out, size_t npolys) {
  DevTables *tb;
  int rc = tables(ctx, F::FIELD_ID, LOGN, &tb, hb::GroupNtt<F, LOGN, T>::LOGV);
  if (rc) return rc;
  using W = typename F::W;
  constexpr int N = 1 << LOGN;
  auto kern = hb::prepare_polys_kernel<F, LOGN, T>;
  const size_t smem = sizeof(W) * (hb::tw_words<W>() * N + 2 * 2 * N);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const unsigned grid = (unsigned)std::min<size_t>((npolys + 1) / 2, (size_t)ctx->sms * 4);
  kern<<<std::max(1u, grid), 2 * T, smem, ctx->stream>>>((const W *)d_in, (W *)d_out, npolys,
                                                          (const W *)tb->tw, (W)tb->key_scale);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? HB_OK : cuda_fail(ctx, e, "prepare_polys launch");
}

// Key polynomials are laid out for a group of T threads (slot t*V + v stored at v*T + t).
template <class F>
int prepare_any(hb_ctx *ctx, uint32_t logn, int T, const void *d_in, void *d_out, size_t npolys) {
  if (logn == 10 && T == 64) return launch_prepare<F, 10, 64>(ctx, d_in, d_out, npolys);
  if (logn == 10 && T == 128) return launch_prepare<F, 10, 128>(ctx, d_in, d_out, npolys);
  if (logn == 11 && T == 128) return launch_prepare<F, 11, 128>(ctx, d_in, d_out, npolys);
  if (logn == 11 && T == 256) return launch_prepare<F, 11, 256>(ctx, d_in, d_out, npolys);
  return fail(ctx, HB_ERR_UNSUPPORTED, "ring dimension 2^%u with %d threads has no compiled kernel", logn, T);
}

int prepare_field(hb_ctx *ctx, int field, uint32_t logn, int T, const void *d_in, void *d_out, size_t npolys) {
  if (field == HB_FIELD_GOLDILOCKS) return prepare_any<Goldilocks>(ctx, logn, T, d_in, d_out, npolys);
  if (field == HB_FIELD_BABYBEAR) return prepare_any<BabyBear>(ctx, logn, T, d_in, d_out, npolys);
  return prepare_any<DefaultFieldU32>(ctx, logn, T, d_in, d_out, npolys);
}

// The group size of the NTT and external-product kernels: 8 words per thread, so their passes of
// three stages take the radix-8 form (GroupNtt::fwd_r8 / inv_r8) for Goldilocks.
int std_threads(uint32_t logn) { return logn == 10 ? 128 : 256; }

template <class F, int LOGN, int T, int GPB>
int launch_ntt(hb_ctx *ctx, const void *in, void *out, size_t count, int mode) {
  DevTables *tb;
  int rc = tables(ctx, F::FIELD_ID, LOGN, &tb, hb::GroupNtt<F, LOGN, T>::LOGV);
  if (rc) return rc;
  using W = typename F::W;
  constexpr int N = 1 << LOGN;
  auto kern = hb::ntt_batch_kernel<F, LOGN, T, GPB>;
  const size_t smem = sizeof(W) * (2 * hb::tw_words<W>() * N + GPB * 2 * N);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, GPB * T, smem);
  const size_t want = (count + GPB - 1) / GPB;
  const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>(want, (size_t)ctx->sms * std::max(1, per_sm)));
  kern<<<grid, GPB * T, smem, ctx->stream>>>((const W *)in, (W *)out, count, (const W *)tb->tw,
                                              (const W *)tb->itw, (W)tb->n_inv, mode);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? HB_OK : cuda_fail(ctx, e, "ntt launch");
}

int ntt_dispatch(hb_ctx *ctx, int field, uint32_t logn, const void *in, void *out, size_t count, int mode) {
  if (field == HB_FIELD_GOLDILOCKS) {
    if (logn == 10) return launch_ntt<Goldilocks, 10, 128, 2>(ctx, in, out, count, mode);
    if (logn == 11) return launch_ntt<Goldilocks, 11, 256, 1>(ctx, in, out, count, mode);
  } else if (field == HB_FIELD_BABYBEAR) {
    if (logn == 10) return launch_ntt<BabyBear, 10, 128, 2>(ctx, in, out, count, mode);
    if (logn == 11) return launch_ntt<BabyBear, 11, 256, 1>(ctx, in, out, count, mode);
  } else if (field == HB_FIELD_DEFAULT_U32) {
    if (logn == 10) return launch_ntt<DefaultFieldU32, 10, 128, 2>(ctx, in, out, count, mode);
    if (logn == 11) return launch_ntt<DefaultFieldU32, 11, 256, 1>(ctx, in, out, count, mode);
  }
  return fail(ctx, HB_ERR_UNSUPPORTED, "no NTT kernel for field %d, log_n %u", field, logn);
}

template <class F, int LOGN, int T, int G>
int launch_ext(hb_ctx *ctx, const void *rgsw, uint32_t bits, uint32_t len, const void *in, void *out,
               size_t count) {
  DevTables *tb;
  int rc = tables(ctx, F::FIELD_ID, LOGN, &tb, hb::GroupNtt<F, LOGN, T>::LOGV);
  if (rc) return rc;
  using W = typename F::W;
  constexpr int N = 1 << LOGN;
  auto kern = hb::ext_product_kernel<F, LOGN, T, G, kStages>;
  const size_t smem = sizeof(W) * (2 * hb::tw_words<W>() * N + kStages * 2 * N + G * 2 * N) + sizeof(uint64_t) * kStages +
                      2 * sizeof(uint32_t) * kStages + 16;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const size_t batches = (count + G - 1) / G;
  const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>(batches, (size_t)ctx->sms));
  kern<<<grid, G * T, smem, ctx->stream>>>((const W *)in, (W *)out, count, (const W *)rgsw, len, bits,
                                            (const W *)tb->tw, (const W *)tb->itw, ctx->d_status,
                                            wait_budget(ctx));
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? HB_OK : cuda_fail(ctx, e, "external product launch");
}

// ---- bootstrapping ----

struct LutSpec {
  uint32_t mid;
  uint64_t lo, hi;
};

LutSpec lut_of(uint64_t P, int gate, uint32_t N) {
  const uint64_t q8 = P >> 3, nq8 = P - q8;
  switch (gate) {  // tfhe/src/bfhe/evaluate.rs:267-465
    case HB_GATE_NAND: return {3 * N / 4, q8, nq8};
    case HB_GATE_AND:
    case HB_GATE_MAJORITY: return {3 * N / 4, nq8, q8};
    case HB_GATE_OR:
    case HB_GATE_MUX: return {N / 4, nq8, q8};
    case HB_GATE_NOR: return {N / 4, q8, nq8};
    case HB_GATE_XOR: return {N / 2, nq8, q8};
    case HB_GATE_XNOR: return {N / 2, q8, nq8};
  }
  return {N, 0, 0};
}

// P: the field modulus (modulus_of)
GateJob make_job(uint64_t P, int gate, uint32_t N, const void *c0, const void *c1, const void *c2,
                 void *out, uint32_t count) {
  GateJob j{};
  j.in0 = c0;
  j.in1 = c1;
  j.in2 = nullptr;
  j.out = out;
  j.lut = nullptr;
  LutSpec l = lut_of(P, gate, N);
  j.lut_mid = l.mid;
  j.lut_lo = l.lo;
  j.lut_hi = l.hi;
  j.add_b = 0;
  j.s0 = 1;
  j.s1 = 1;
  j.s2 = 0;
  if (gate == HB_GATE_XOR || gate == HB_GATE_XNOR) {  // evaluate.rs:182-208: 2 (c0 - c1)
    j.s0 = 2;
    j.s1 = -2;
  } else if (gate == HB_GATE_MAJORITY) {  // evaluate.rs:220-237: c0 + c1 + c2
    j.in2 = c2;
    j.s2 = 1;
  }
  j.count = count;
  return j;
}


// Launches of at most one gate per SM (G = 1 outside the plain form) run the latency form: one gate
// per CTA, its digits spread over the CTA's thread groups. With a binary LWE key a gate takes a
// cluster of CTAs instead while the launch holds at most one cluster CTA per SM: kDpCluster64 CTAs
// of 4 groups for the Goldilocks sets (2l = 16 digits), kDpCluster32 CTAs of 4 groups of 128
// threads for the 32-bit fields (BabyBear's 2l = 8 digits one per group), so that each SM
// transforms a share of a step's digits and every CTA inverse-transforms the summed a and b
// polynomials itself.
constexpr int kDpCluster64 = 4;
constexpr int kDpCluster32 = 2;

template <class F, int LOGN, int T, int C, bool KSC, bool TERN, bool KST>
int launch_dp_k(hb_ctx *ctx, const hb::BootParams<typename F::W> &prm, cudaStream_t stream, int *max_clusters) {
  using W = typename F::W;
  constexpr int N = 1 << LOGN, D = hb::dp_groups<W, T, C>(), TG = hb::dp_group_threads<W, T, C>();
  auto kern = hb::bootstrap_dp_kernel<F, LOGN, TG, D, C, KSC, TERN, T, KST>;
  const size_t smem = hb::dp_smem_bytes<W, N, D, C, KST>(prm.n);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "bootstrap smem attribute");
  if constexpr (C == 1) {
    const unsigned grid = std::max(1u, std::min<unsigned>(prm.total_batches, (unsigned)ctx->sms));
    kern<<<grid, D * TG, smem, stream>>>(prm);
  } else {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(D * TG);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (max_clusters) {  // how many clusters of this shape the GPU holds at once
      cfg.gridDim = dim3(C);
      int m = 0;
      e = cudaOccupancyMaxActiveClusters(&m, kern, &cfg);
      *max_clusters = e == cudaSuccess ? m : 0;
      return HB_OK;
    }
    cfg.gridDim = dim3(prm.total_batches * C);
    e = cudaLaunchKernelEx(&cfg, kern, prm);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "bootstrap cluster launch");
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "bootstrap launch");
  ctx->launches += 1;
  return HB_OK;
}

// The latency form with C CTAs per gate. Key words staged through shared memory (KST) only for the
// 32-bit fields' clusters whose groups take more than one digit per step (DEFAULT_TERNARY: 18
// digits over 8 groups, one gate 10.75 -> 10.09 ms); a single digit per group (BABYBEAR,
// CUSTOM_TERNARY) and the Goldilocks sets measured 4-7 % slower with it.
template <class F, int LOGN, int T, int C, bool KSC, bool TERN = false>
int launch_dp_c(hb_ctx *ctx, const hb::BootParams<typename F::W> &prm, cudaStream_t stream, int *max_clusters) {
  using W = typename F::W;
  if constexpr (sizeof(W) == 4 && C > 1 && !TERN) {
    if (2 * prm.len > (uint32_t)(C * hb::dp_groups<W, T, C>()))
      return launch_dp_k<F, LOGN, T, C, KSC, TERN, true>(ctx, prm, stream, max_clusters);
  }
  return launch_dp_k<F, LOGN, T, C, KSC, TERN, false>(ctx, prm, stream, max_clusters);
}

// Twiddles of the latency form with C CTAs per gate over keys laid out for T threads: those of the
// groups' digit transforms and the half-CTA groups' inverse twiddles. Built with the keys
// (hb_keys_upload / hb_keys_generate / relayout), never inside a capture; false if missing.
template <class F, int LOGN, int T, int C>
bool dp_twiddles(hb_ctx *ctx, hb::BootParams<typename F::W> &prm) {
  using W = typename F::W;
  constexpr int N = 1 << LOGN;
  constexpr int LOGV = hb::ilog2c(N / hb::dp_group_threads<W, T, C>());
  constexpr int LOGVW = hb::ilog2c(hb::dp_wide_words<W, N, T, C>());
  prm.tw = (const W *)ctx->tables[F::FIELD_ID][LOGN][LOGV].tw;
  prm.itw = (const W *)ctx->tables[F::FIELD_ID][LOGN][LOGV].itw;
  prm.itw_w = (const W *)ctx->tables[F::FIELD_ID][LOGN][LOGVW].itw;
  return prm.tw && prm.itw && prm.itw_w;
}

template <class F, int LOGN, int T, bool KSC, bool TERN = false>
int launch_dp(hb_ctx *ctx, hb::BootParams<typename F::W> prm, cudaStream_t stream) {
  using W = typename F::W;
  constexpr int CL = sizeof(W) == 8 ? kDpCluster64 : kDpCluster32;
  if constexpr (!TERN) {
    std::atomic<int> &cached = ctx->dp_clusters[(sizeof(W) == 8 ? 0 : 2) + (T == 128 ? 1 : 0)];
    int m = cached.load();
    hb::BootParams<W> cp = prm;
    if (!dp_twiddles<F, LOGN, T, CL>(ctx, cp)) return fail(ctx, HB_ERR_INVALID, "keys were not prepared on this context");
    if (m < 0) {  // the same shared memory and threads with or without KSC
      const int rc = launch_dp_c<F, LOGN, T, CL, KSC>(ctx, cp, stream, &m);
      if (rc) return rc;
      m = std::min(m, ctx->sms / CL);  // one cluster CTA per SM
      cached.store(m);
    }
    if (cp.total_batches <= (uint32_t)m) return launch_dp_c<F, LOGN, T, CL, KSC>(ctx, cp, stream, nullptr);
  }
  if (!dp_twiddles<F, LOGN, T, 1>(ctx, prm)) return fail(ctx, HB_ERR_INVALID, "keys were not prepared on this context");
  return launch_dp_c<F, LOGN, T, 1, KSC, TERN>(ctx, prm, stream, nullptr);
}

template <class F, int LOGN, int T, int G, bool TERN, bool KSC>
int launch_boot(hb_ctx *ctx, hb_keys *keys, std::vector<GateJob> &jobs, bool plain, void *trace) {
  using W = typename F::W;
  constexpr int N = 1 << LOGN;
  DevTables *tb;
  int rc = tables(ctx, F::FIELD_ID, LOGN, &tb, hb::GroupNtt<F, LOGN, T>::LOGV);
  if (rc) return rc;
  // Batched: jobs are laid end to end in batch space. Plain: every launch holds one job whose
  // batches start at 0.
  uint32_t batches = 0;
  for (auto &j : jobs) {
    j.first_batch = plain ? 0 : batches;
    batches += (j.count + G - 1) / G;
  }
  if (batches == 0) return HB_OK;
  rc = scratch(ctx, ctx->jobs, sizeof(GateJob) * jobs.size());
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(ctx->jobs.ptr, jobs.data(), sizeof(GateJob) * jobs.size(),
                                  cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "job table upload");
  hb::BootParams<W> prm{};
  boot_params(prm, ctx, keys, tb);
  prm.trace = (W *)trace;
  constexpr int S = hb::boot_stages<W, N, G>();
  auto kern = hb::bootstrap_kernel<F, LOGN, T, G, S, TERN, KSC>;
  const size_t smem = hb::boot_smem_bytes<W, N, G, S>(prm.n);
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "bootstrap smem attribute");
  const GateJob *djobs = (const GateJob *)ctx->jobs.ptr;
  const unsigned grid = plain ? 1u : std::min<unsigned>(batches, (unsigned)ctx->sms);
  const unsigned block = G * T;
  if (!plain) {
    prm.jobs = djobs;
    prm.njobs = (int)jobs.size();
    prm.total_batches = batches;
    if constexpr (G == 1) return launch_dp<F, LOGN, T, KSC, TERN>(ctx, prm, ctx->stream);
    kern<<<grid, block, smem, ctx->stream>>>(prm);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "bootstrap launch");
    ctx->launches += 1;
    return HB_OK;
  }
  // plain form: one launch per job (each job is one gate)
  for (size_t i = 0; i < jobs.size(); ++i) {
    prm.jobs = djobs + i;
    prm.njobs = 1;
    prm.total_batches = 1;
    hb::BootParams<W> one = prm;
    kern<<<1, block, smem, ctx->stream>>>(one);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "bootstrap launch");
    ctx->launches += 1;
  }
  return HB_OK;
}

// Compiled variants of the persistent bootstrapping kernel: (field, threads per gate T, gates per
// CTA G, ternary LWE key, key switch in chunks of n' < N words). The key layout fixes T at upload;
// the autotuner picks G among the variants of that T. G = 1 is the plain one-gate-per-launch form.
#define HB_BOOT_VARIANTS(X)                                                                          \
  X(Goldilocks, 64, 1, false, false) X(Goldilocks, 64, 3, false, false)                             \
  X(Goldilocks, 64, 4, false, false) X(Goldilocks, 128, 1, false, false)                            \
  X(Goldilocks, 128, 3, false, false) X(Goldilocks, 128, 4, false, false)                           \
  X(Goldilocks, 128, 1, false, true) X(Goldilocks, 128, 4, false, true)                             \
  X(BabyBear, 64, 1, false, false) X(BabyBear, 64, 4, false, false) X(BabyBear, 64, 6, false, false) \
  X(BabyBear, 64, 8, false, false) X(BabyBear, 128, 1, false, false)                                \
  X(BabyBear, 128, 4, false, false) X(BabyBear, 128, 6, false, false)                               \
  X(BabyBear, 64, 1, false, true) X(BabyBear, 64, 6, false, true)                                   \
  X(DefaultFieldU32, 64, 1, false, false) X(DefaultFieldU32, 64, 4, false, false)                   \
  X(DefaultFieldU32, 64, 6, false, false) X(DefaultFieldU32, 64, 8, false, false)                   \
  X(DefaultFieldU32, 128, 1, false, false) X(DefaultFieldU32, 128, 4, false, false)                 \
  X(DefaultFieldU32, 128, 6, false, false) X(DefaultFieldU32, 64, 1, false, true)                   \
  X(DefaultFieldU32, 64, 4, false, true) X(DefaultFieldU32, 64, 8, false, true)                     \
  X(DefaultFieldU32, 128, 1, false, true) X(DefaultFieldU32, 128, 4, false, true)                   \
  X(DefaultFieldU32, 64, 1, true, false) X(DefaultFieldU32, 64, 4, true, false)                     \
  X(DefaultFieldU32, 128, 1, true, false) X(DefaultFieldU32, 128, 4, true, false)                   \
  X(DefaultFieldU32, 64, 1, true, true) X(DefaultFieldU32, 64, 4, true, true)                       \
  X(DefaultFieldU32, 128, 1, true, true) X(DefaultFieldU32, 128, 4, true, true)

template <class F>
constexpr int field_of() { return F::FIELD_ID; }

// trace: the accumulator trace of a one-gate launch (the latency form records it), or null.
int run_jobs(hb_ctx *ctx, hb_keys *keys, std::vector<GateJob> &jobs, bool plain, void *trace = nullptr) {
  if (keys->p.ring_dim != 1024)
    return fail(ctx, HB_ERR_UNSUPPORTED, "bootstrapping is compiled for N = 1024");
  uint64_t gates = 0;
  for (auto &j : jobs) gates += j.count;
  const int G = plain ? 1 : launch_gates_per_cta(ctx, keys, gates), T = keys->threads_per_gate,
            fld = keys->p.field_id;
  const bool tern = keys->p.lwe_ternary != 0, ksc = ks_dim(keys->p) < keys->p.ring_dim;
  if (trace && (plain || G != 1 || tern || gates != 1))
    return fail(ctx, HB_ERR_UNSUPPORTED, "accumulator traces are recorded for one gate under a binary LWE key");
#define HB_CASE(FLD, TT, GG, TN, KC)                                             \
  if (fld == field_of<FLD>() && T == TT && G == GG && tern == TN && ksc == KC) \
    return launch_boot<FLD, 10, TT, GG, TN, KC>(ctx, keys, jobs, plain, trace);
  HB_BOOT_VARIANTS(HB_CASE)
#undef HB_CASE
  return fail(ctx, HB_ERR_UNSUPPORTED, "no compiled kernel with %d threads per gate and %d gates per CTA", T, G);
}

// Gates-per-CTA variants compiled for a parameter set and group size (the autotuner's candidates).
std::vector<int> variants(const hb_params &p, int T) {
  std::vector<int> v;
  const bool tern = p.lwe_ternary != 0, ksc = ks_dim(p) < p.ring_dim;
#define HB_CASE(FLD, TT, GG, TN, KC) \
  if (p.field_id == field_of<FLD>() && T == TT && GG > 1 && tern == TN && ksc == KC) v.push_back(GG);
  HB_BOOT_VARIANTS(HB_CASE)
#undef HB_CASE
  return v;
}

uint32_t batches_of(const std::vector<GateJob> &jobs, int G) {
  uint32_t b = 0;
  for (auto &j : jobs) b += (j.count + G - 1) / G;
  return b;
}

// One batched persistent launch over a device job table that is already in place.
template <class F, int LOGN, int T, int G, bool TERN, bool KSC>
int launch_table(hb_ctx *ctx, hb_keys *keys, const GateJob *djobs, int njobs, uint32_t batches,
                 unsigned grid, cudaStream_t stream) {
  using W = typename F::W;
  constexpr int N = 1 << LOGN;
  DevTables *tb;
  int rc = tables(ctx, F::FIELD_ID, LOGN, &tb, hb::GroupNtt<F, LOGN, T>::LOGV);
  if (rc) return rc;
  hb::BootParams<W> prm{};
  boot_params(prm, ctx, keys, tb);
  prm.jobs = djobs;
  prm.njobs = njobs;
  prm.total_batches = batches;
  if constexpr (G == 1) return launch_dp<F, LOGN, T, KSC, TERN>(ctx, prm, stream);
  constexpr int S = hb::boot_stages<W, N, G>();
  auto kern = hb::bootstrap_kernel<F, LOGN, T, G, S, TERN, KSC>;
  const size_t smem = hb::boot_smem_bytes<W, N, G, S>(prm.n);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "bootstrap smem attribute");
  grid = std::max(1u, std::min(grid, batches));
  kern<<<grid, G * T, smem, stream>>>(prm);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "bootstrap launch");
  ctx->launches += 1;
  return HB_OK;
}

int launch_table_any(hb_ctx *ctx, hb_keys *keys, int G, const GateJob *djobs, int njobs,
                     uint32_t batches, unsigned grid, cudaStream_t stream) {
  const int T = keys->threads_per_gate, fld = keys->p.field_id;
  const bool tern = keys->p.lwe_ternary != 0, ksc = ks_dim(keys->p) < keys->p.ring_dim;
#define HB_CASE(FLD, TT, GG, TN, KC)                                             \
  if (fld == field_of<FLD>() && T == TT && G == GG && tern == TN && ksc == KC) \
    return launch_table<FLD, 10, TT, GG, TN, KC>(ctx, keys, djobs, njobs, batches, grid, stream);
  HB_BOOT_VARIANTS(HB_CASE)
#undef HB_CASE
  return fail(ctx, HB_ERR_UNSUPPORTED, "no compiled kernel with %d threads per gate and %d gates per CTA", T, G);
}

bool single_bootstrap_gate(int gate) { return gate >= HB_GATE_NAND && gate <= HB_GATE_MAJORITY; }

template <class F>
__global__ void lwe_not_kernel(const typename F::W *in, typename F::W *out, size_t words,
                               uint32_t width) {
  // Evaluator::not (tfhe/src/bfhe/evaluate.rs:98-105): -c, then b += Q >> 2
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < words; i += (size_t)gridDim.x * blockDim.x) {
    typename F::W v = hb::canon_neg<F>(in[i]);
    if (i % width == width - 1) v = F::canon(F::add(v, (typename F::W)(F::P >> 2)));
    out[i] = v;
  }
}

size_t word_size(const hb_params &p) { return p.field_id == HB_FIELD_GOLDILOCKS ? 8 : 4; }

int default_threads_per_gate(int field_id) {
  const char *env = getenv("HB_THREADS_PER_GATE");
  if (env && (atoi(env) == 64 || atoi(env) == 128)) return atoi(env);
  return field_id == HB_FIELD_GOLDILOCKS ? 128 : 64;  // measured best tiles on B200
}

int default_gates_per_cta(int field_id) {
  const char *env = getenv("HB_GATES_PER_CTA");
  if (env && atoi(env) > 0) return atoi(env);
  // measured best on B200 before autotuning: Goldilocks (T = 128) 4, BabyBear (T = 64, paired
  // digit transforms) 8, DefaultFieldU32 (T = 64) 6
  return field_id == HB_FIELD_GOLDILOCKS ? 4 : field_id == HB_FIELD_BABYBEAR ? 8 : 6;
}

}  // namespace

// ------------------------------------------------------------------------------------------
// C API
// ------------------------------------------------------------------------------------------

extern "C" {

int hb_ctx_create(int device, size_t hbm_budget, hb_ctx **out) {
  if (!out) return HB_ERR_INVALID;
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return HB_ERR_CUDA;
  hb_ctx *ctx = new hb_ctx();
  ctx->device = device;
  ctx->budget = hbm_budget;
  cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
  e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete ctx;
    return HB_ERR_CUDA;
  }
  void *st = nullptr;
  if (dev_alloc(ctx, sizeof(int) * 4, &st) != HB_OK) {
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return HB_ERR_CUDA;
  }
  ctx->d_status = (int *)st;
  cudaMemset(ctx->d_status, 0, sizeof(int) * 4);
  *out = ctx;
  return HB_OK;
}

void hb_ctx_destroy(hb_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto &kv : ctx->sizes) cudaFree(kv.first);
  ctx->sizes.clear();
  cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int hb_last_error(const hb_ctx *ctx, char *buf, size_t len) {
  if (!ctx || !buf || !len) return HB_ERR_INVALID;
  snprintf(buf, len, "%s", ctx->err.c_str());
  return HB_OK;
}

int hb_ctx_stream(hb_ctx *ctx, void **stream) {
  if (!ctx || !stream) return HB_ERR_INVALID;
  *stream = (void *)ctx->stream;
  return HB_OK;
}

int hb_ctx_synchronize(hb_ctx *ctx) {
  if (!ctx) return HB_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return check_status(ctx);
}

size_t hb_ctx_hbm_in_use(const hb_ctx *ctx) { return ctx ? ctx->in_use : 0; }

int hb_keys_upload(hb_ctx *ctx, const hb_params *p, const void *bsk, const void *ksk, hb_keys **out) {
  if (!ctx || !out || !bsk || !ksk) return HB_ERR_INVALID;
  *out = nullptr;
  if (hb_params_validate(p) != HB_OK) return fail(ctx, HB_ERR_INVALID, "invalid parameter set");
  cudaSetDevice(ctx->device);
  size_t nb = 0, nk = 0;
  hb_params_sizes(p, nullptr, nullptr, &nb, &nk, nullptr);
  const size_t ws = word_size(*p);
  uint32_t logn = 0;
  while ((1u << logn) < p->ring_dim) ++logn;
  hb_keys *k = new hb_keys();
  k->p = *p;
  // The key switch's n'-word chunk keys (n' = next_pow2(n) < N) are spread to N words, every
  // (N/n')-th slot, so their products come out of the N-point transforms of the bootstrap kernel
  // (the ring embedding X -> X^(N/n')).
  const size_t nkd = ksk_device_words(*p);
  std::vector<unsigned char> spread;
  const void *ksk_src = ksk;
  if (nkd != nk) {
    const size_t M = ks_dim(*p), stride = p->ring_dim / M, polys = nk / M;
    spread.assign(nkd * ws, 0);
    for (size_t q = 0; q < polys; ++q)
      for (size_t u = 0; u < M; ++u)
        std::memcpy(spread.data() + (q * p->ring_dim + u * stride) * ws,
                    (const unsigned char *)ksk + (q * M + u) * ws, ws);
    ksk_src = spread.data();
  }
  int rc = dev_alloc(ctx, nb * ws, &k->bsk);
  if (!rc) rc = dev_alloc(ctx, nkd * ws, &k->ksk);
  void *staging = nullptr;
  if (!rc) rc = dev_alloc(ctx, std::max(nb, nkd) * ws, &staging);
  if (rc) {
    dev_free(ctx, k->bsk);
    dev_free(ctx, k->ksk);
    delete k;
    return rc;
  }
  k->threads_per_gate = default_threads_per_gate(p->field_id);
  cudaError_t e = cudaMemcpyAsync(staging, bsk, nb * ws, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    rc = prepare_field(ctx, p->field_id, logn, k->threads_per_gate, staging, k->bsk, nb / p->ring_dim);
  if (e == cudaSuccess && !rc) e = cudaStreamSynchronize(ctx->stream);
  if (e == cudaSuccess && !rc) e = cudaMemcpyAsync(staging, ksk_src, nkd * ws, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess && !rc)
    rc = prepare_field(ctx, p->field_id, logn, k->threads_per_gate, staging, k->ksk, nkd / p->ring_dim);
  if (e == cudaSuccess && !rc) e = cudaStreamSynchronize(ctx->stream);
  dev_free(ctx, staging);
  if (e != cudaSuccess || rc) {
    dev_free(ctx, k->bsk);
    dev_free(ctx, k->ksk);
    delete k;
    return e != cudaSuccess ? cuda_fail(ctx, e, "key upload") : rc;
  }
  k->bytes = (nb + nkd) * ws;
  k->gates_per_cta = default_gates_per_cta(p->field_id);
  const std::vector<int> cand = variants(*p, k->threads_per_gate);
  if (cand.size() && std::find(cand.begin(), cand.end(), k->gates_per_cta) == cand.end())
    k->gates_per_cta = cand.back();
  rc = dp_tables(ctx, *p, k->threads_per_gate);
  if (rc) {
    hb_keys_free(ctx, k);
    return rc;
  }
  *out = k;
  return HB_OK;
}

void hb_keys_free(hb_ctx *ctx, hb_keys *keys) {
  if (!ctx || !keys) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  dev_free(ctx, keys->bsk);
  dev_free(ctx, keys->ksk);
  delete keys;
}

int hb_keys_params(const hb_keys *keys, hb_params *out) {
  if (!keys || !out) return HB_ERR_INVALID;
  *out = keys->p;
  return HB_OK;
}

int hb_keys_device_words(const hb_keys *keys, size_t *bsk_words, size_t *ksk_words) {
  if (!keys) return HB_ERR_INVALID;
  size_t nb = 0;
  hb_params_sizes(&keys->p, nullptr, nullptr, &nb, nullptr, nullptr);
  if (bsk_words) *bsk_words = nb;
  if (ksk_words) *ksk_words = ksk_device_words(keys->p);
  return HB_OK;
}

int hb_keys_download(hb_ctx *ctx, const hb_keys *keys, void *bsk, size_t bsk_words, void *ksk,
                     size_t ksk_words) {
  if (!ctx || !keys || !bsk || !ksk) return HB_ERR_INVALID;
  size_t nb = 0, nk = 0;
  hb_keys_device_words(keys, &nb, &nk);
  if (bsk_words != nb || ksk_words != nk)
    return fail(ctx, HB_ERR_INVALID, "key buffers of %zu / %zu words, the keys hold %zu / %zu", bsk_words,
                ksk_words, nb, nk);
  cudaSetDevice(ctx->device);
  const size_t ws = word_size(keys->p);
  cudaError_t e = cudaMemcpyAsync(bsk, keys->bsk, nb * ws, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ksk, keys->ksk, nk * ws, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? HB_OK : cuda_fail(ctx, e, "key download");
}

int hb_gate_device(hb_ctx *ctx, hb_keys *keys, int gate, const void *c0, const void *c1,
                   const void *c2, void *out, size_t count) {
  if (!ctx || !keys) return HB_ERR_INVALID;
  if (gate < HB_GATE_NAND || gate > HB_GATE_MUX) return fail(ctx, HB_ERR_INVALID, "unknown gate %d", gate);
  if (count == 0) return HB_OK;
  if (count > 0xFFFFFFFFull) return fail(ctx, HB_ERR_INVALID, "too many gates in one call");
  if (!c0 || !out || (gate != HB_GATE_NOT && !c1) ||
      ((gate == HB_GATE_MAJORITY || gate == HB_GATE_MUX) && !c2))
    return fail(ctx, HB_ERR_INVALID, "missing ciphertext buffer");
  cudaSetDevice(ctx->device);
  const hb_params &p = keys->p;
  const uint32_t N = p.ring_dim;
  const size_t width = p.lwe_dim + 1;
  const uint64_t P = modulus_of(p.field_id);
  if (gate == HB_GATE_NOT) {
    const size_t words = count * width;
    const unsigned grid = (unsigned)std::min<size_t>((words + 255) / 256, 4096);
    if (p.field_id == HB_FIELD_GOLDILOCKS)
      lwe_not_kernel<Goldilocks><<<grid, 256, 0, ctx->stream>>>((const uint64_t *)c0, (uint64_t *)out, words, (uint32_t)width);
    else if (p.field_id == HB_FIELD_BABYBEAR)
      lwe_not_kernel<BabyBear><<<grid, 256, 0, ctx->stream>>>((const uint32_t *)c0, (uint32_t *)out, words, (uint32_t)width);
    else
      lwe_not_kernel<DefaultFieldU32><<<grid, 256, 0, ctx->stream>>>((const uint32_t *)c0, (uint32_t *)out, words, (uint32_t)width);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? HB_OK : cuda_fail(ctx, e, "not launch");
  }
  std::vector<GateJob> jobs;
  if (gate != HB_GATE_MUX) {
    jobs.push_back(make_job(P, gate, N, c0, c1, c2, out, (uint32_t)count));
    return run_jobs(ctx, keys, jobs, false);
  }
  // MUX (evaluate.rs:245-262): t0 = and(c0, c1), t1 = and(not c0, c2), out = bootstrap(t0 + t1, or)
  const size_t bytes = count * width * word_size(p);
  int rc = scratch(ctx, ctx->mux_tmp, 2 * bytes);
  if (rc) return rc;
  char *t0 = (char *)ctx->mux_tmp.ptr, *t1 = t0 + bytes;
  GateJob a = make_job(P, HB_GATE_AND, N, c0, c1, nullptr, t0, (uint32_t)count);
  GateJob b = a;
  b.in1 = c2;
  b.out = t1;
  b.s0 = -1;  // not(c0) = -c0 + Q/4 on the body
  b.add_b = P >> 2;
  jobs = {a, b};
  rc = run_jobs(ctx, keys, jobs, false);
  if (rc) return rc;
  jobs = {make_job(P, HB_GATE_MUX, N, t0, t1, nullptr, out, (uint32_t)count)};
  return run_jobs(ctx, keys, jobs, false);
}

int hb_gate_device_plain(hb_ctx *ctx, hb_keys *keys, int gate, const void *c0, const void *c1,
                         void *out, size_t count) {
  if (!ctx || !keys || !c0 || !c1 || !out) return HB_ERR_INVALID;
  if (gate < HB_GATE_NAND || gate > HB_GATE_XNOR) return fail(ctx, HB_ERR_INVALID, "plain form covers two-input gates");
  cudaSetDevice(ctx->device);
  const hb_params &p = keys->p;
  const size_t width = p.lwe_dim + 1, ws = word_size(p);
  std::vector<GateJob> jobs;
  jobs.reserve(count);
  for (size_t i = 0; i < count; ++i) {
    const char *a = (const char *)c0 + i * width * ws;
    const char *b = (const char *)c1 + i * width * ws;
    char *o = (char *)out + i * width * ws;
    jobs.push_back(make_job(modulus_of(p.field_id), gate, p.ring_dim, a, b, nullptr, o, 1));
  }
  return run_jobs(ctx, keys, jobs, true);
}

int hb_gate(hb_ctx *ctx, hb_keys *keys, int gate, const void *c0, const void *c1, const void *c2,
            void *out, size_t count) {
  if (!ctx || !keys) return HB_ERR_INVALID;
  if (count == 0) return HB_OK;
  cudaSetDevice(ctx->device);
  const size_t bytes = count * (keys->p.lwe_dim + 1) * word_size(keys->p);
  const int nin = gate == HB_GATE_NOT ? 1 : (gate == HB_GATE_MAJORITY || gate == HB_GATE_MUX ? 3 : 2);
  int rc = scratch(ctx, ctx->io, bytes * (nin + 1));
  if (rc) return rc;
  char *base = (char *)ctx->io.ptr;
  const void *srcs[3] = {c0, c1, c2};
  void *dins[3] = {nullptr, nullptr, nullptr};
  for (int i = 0; i < nin; ++i) {
    if (!srcs[i]) return fail(ctx, HB_ERR_INVALID, "missing ciphertext buffer");
    dins[i] = base + i * bytes;
    cudaMemcpyAsync(dins[i], srcs[i], bytes, cudaMemcpyHostToDevice, ctx->stream);
  }
  void *dout = base + nin * bytes;
  rc = hb_gate_device(ctx, keys, gate, dins[0], dins[1], dins[2], dout, count);
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "result copy");
  return check_status(ctx);
}

int hb_bootstrap_lut(hb_ctx *ctx, hb_keys *keys, const void *c, const void *lut, void *out, size_t count) {
  if (!ctx || !keys || !c || !lut || !out) return HB_ERR_INVALID;
  if (count == 0) return HB_OK;
  cudaSetDevice(ctx->device);
  const hb_params &p = keys->p;
  const size_t ws = word_size(p), bytes = count * (p.lwe_dim + 1) * ws, lbytes = p.ring_dim * ws;
  int rc = scratch(ctx, ctx->io, 2 * bytes + lbytes);
  if (rc) return rc;
  char *din = (char *)ctx->io.ptr, *dout = din + bytes, *dlut = dout + bytes;
  cudaMemcpyAsync(din, c, bytes, cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(dlut, lut, lbytes, cudaMemcpyHostToDevice, ctx->stream);
  GateJob j{};
  j.in0 = din;
  j.out = dout;
  j.lut = dlut;
  j.s0 = 1;
  j.count = (uint32_t)count;
  std::vector<GateJob> jobs{j};
  rc = run_jobs(ctx, keys, jobs, false);
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "result copy");
  return check_status(ctx);
}

int hb_bootstrap_trace(hb_ctx *ctx, hb_keys *keys, const void *c, const void *lut, void *out,
                       void *acc_trace) {
  if (!ctx || !keys || !c || !lut || !out || !acc_trace) return HB_ERR_INVALID;
  if (keys->p.lwe_ternary)
    return fail(ctx, HB_ERR_UNSUPPORTED, "accumulator traces are recorded under binary LWE keys");
  cudaSetDevice(ctx->device);
  const hb_params &p = keys->p;
  const size_t ws = word_size(p), bytes = (p.lwe_dim + 1) * ws, lbytes = p.ring_dim * ws;
  const size_t tbytes = (size_t)p.lwe_dim * 2 * p.ring_dim * ws;
  int rc = scratch(ctx, ctx->io, 2 * bytes + lbytes + tbytes);
  if (rc) return rc;
  // every part starts at a multiple of the word size
  char *din = (char *)ctx->io.ptr, *dout = din + bytes, *dlut = dout + bytes, *dtrace = dlut + lbytes;
  cudaMemcpyAsync(din, c, bytes, cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(dlut, lut, lbytes, cudaMemcpyHostToDevice, ctx->stream);
  GateJob j{};
  j.in0 = din;
  j.out = dout;
  j.lut = dlut;
  j.s0 = 1;
  j.count = 1;
  std::vector<GateJob> jobs{j};
  rc = run_jobs(ctx, keys, jobs, false, dtrace);
  if (rc) return rc;
  cudaError_t e = cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(acc_trace, dtrace, tbytes, cudaMemcpyDeviceToHost, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "result copy");
  return check_status(ctx);
}

int hb_ntt_forward_device(hb_ctx *ctx, int field_id, uint32_t log_n, void *data, size_t count) {
  if (!ctx || !data) return HB_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return ntt_dispatch(ctx, field_id, log_n, data, data, count, 1);
}

int hb_ntt_inverse_device(hb_ctx *ctx, int field_id, uint32_t log_n, void *data, size_t count) {
  if (!ctx || !data) return HB_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return ntt_dispatch(ctx, field_id, log_n, data, data, count, 2);
}

int hb_ntt_roundtrip_device(hb_ctx *ctx, int field_id, uint32_t log_n, const void *in, void *out,
                            size_t count) {
  if (!ctx || !in || !out) return HB_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return ntt_dispatch(ctx, field_id, log_n, in, out, count, 0);
}

int hb_rgsw_upload(hb_ctx *ctx, int field_id, uint32_t log_n, uint32_t bits, uint32_t len,
                   const void *rgsw, void **d_rgsw) {
  if (!ctx || !rgsw || !d_rgsw || bits == 0 || bits > 16 || len == 0 || (uint64_t)(len - 1) * bits >= 64)
    return HB_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (field_id < 0 || field_id > 2) return fail(ctx, HB_ERR_INVALID, "unknown field %d", field_id);
  const size_t N = (size_t)1 << log_n, ws = field_id == HB_FIELD_GOLDILOCKS ? 8 : 4;
  const size_t words = 2 * (size_t)len * 2 * N;
  void *dst = nullptr, *staging = nullptr;
  int rc = dev_alloc(ctx, words * ws, &dst);
  if (!rc) rc = dev_alloc(ctx, words * ws, &staging);
  if (rc) {
    dev_free(ctx, dst);
    return rc;
  }
  cudaMemcpyAsync(staging, rgsw, words * ws, cudaMemcpyHostToDevice, ctx->stream);
  rc = prepare_field(ctx, field_id, log_n, std_threads(log_n), staging, dst, words / N);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  dev_free(ctx, staging);
  if (rc || e != cudaSuccess) {
    dev_free(ctx, dst);
    return rc ? rc : cuda_fail(ctx, e, "rgsw upload");
  }
  *d_rgsw = dst;
  return HB_OK;
}

void hb_rgsw_free(hb_ctx *ctx, void *d_rgsw) {
  if (!ctx || !d_rgsw) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  dev_free(ctx, d_rgsw);
}

int hb_external_product_device(hb_ctx *ctx, int field_id, uint32_t log_n, uint32_t bits, uint32_t len,
                               const void *d_rgsw, const void *rlwe_in, void *rlwe_out, size_t count) {
  if (!ctx || !d_rgsw || !rlwe_in || !rlwe_out || bits == 0 || bits > 16 || len == 0 ||
      (uint64_t)(len - 1) * bits >= 64)
    return HB_ERR_INVALID;
  if (count == 0) return HB_OK;
  cudaSetDevice(ctx->device);
  if (field_id == HB_FIELD_GOLDILOCKS) {
    if (log_n == 10) return launch_ext<Goldilocks, 10, 128, 4>(ctx, d_rgsw, bits, len, rlwe_in, rlwe_out, count);
    if (log_n == 11) return launch_ext<Goldilocks, 11, 256, 2>(ctx, d_rgsw, bits, len, rlwe_in, rlwe_out, count);
  } else if (field_id == HB_FIELD_BABYBEAR) {
    if (log_n == 10) return launch_ext<BabyBear, 10, 128, 4>(ctx, d_rgsw, bits, len, rlwe_in, rlwe_out, count);
    if (log_n == 11) return launch_ext<BabyBear, 11, 256, 2>(ctx, d_rgsw, bits, len, rlwe_in, rlwe_out, count);
  } else if (field_id == HB_FIELD_DEFAULT_U32) {
    if (log_n == 10) return launch_ext<DefaultFieldU32, 10, 128, 4>(ctx, d_rgsw, bits, len, rlwe_in, rlwe_out, count);
    if (log_n == 11) return launch_ext<DefaultFieldU32, 11, 256, 2>(ctx, d_rgsw, bits, len, rlwe_in, rlwe_out, count);
  }
  return fail(ctx, HB_ERR_UNSUPPORTED, "no external-product kernel for field %d, log_n %u", field_id, log_n);
}

int hb_probe_modmul(hb_ctx *ctx, int field_id, double *modmul_per_s) {
  if (!ctx || !modmul_per_s || field_id < 0 || field_id > 2) return HB_ERR_INVALID;
  cudaSetDevice(ctx->device);
  const unsigned blocks = (unsigned)ctx->sms * 8, threads = 256;
  const uint32_t iters = field_id == HB_FIELD_GOLDILOCKS ? 4096 : 16384;
  void *buf = nullptr;
  int rc = dev_alloc(ctx, (size_t)blocks * threads * 8, &buf);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0, ctx->stream);
    if (field_id == HB_FIELD_GOLDILOCKS)
      hb::modmul_probe_kernel<Goldilocks><<<blocks, threads, 0, ctx->stream>>>((uint64_t *)buf, iters, 12345 + rep);
    else if (field_id == HB_FIELD_BABYBEAR)
      hb::modmul_probe_kernel<BabyBear><<<blocks, threads, 0, ctx->stream>>>((uint32_t *)buf, iters, 12345 + rep);
    else
      hb::modmul_probe_kernel<DefaultFieldU32><<<blocks, threads, 0, ctx->stream>>>((uint32_t *)buf, iters, 12345 + rep);
    cudaEventRecord(e1, ctx->stream);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0) best = std::min(best, ms);
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dev_free(ctx, buf);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "modmul probe");
  *modmul_per_s = (double)blocks * threads * 8.0 * iters / (best * 1e-3);
  return HB_OK;
}

uint64_t hb_ctx_launches(const hb_ctx *ctx) { return ctx ? ctx->launches.load() : 0; }

int hb_ctx_set_wait_limit(hb_ctx *ctx, long long clock_cycles) {
  if (!ctx || clock_cycles < 0) return HB_ERR_INVALID;
  ctx->wait_limit = clock_cycles;
  return HB_OK;
}

int hb_ctx_test_withhold_keys(hb_ctx *ctx, int on) {
  if (!ctx) return HB_ERR_INVALID;
  ctx->withhold_keys = on ? 1 : 0;
  return HB_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Key generation and encryption on the device
// ------------------------------------------------------------------------------------------

namespace {

template <class F, int LOGN, int T>
int launch_keygen(hb_ctx *ctx, hb::KeygenParams<typename F::W> &prm) {
  using W = typename F::W;
  constexpr int N = 1 << LOGN;
  DevTables *tb;
  int rc = tables(ctx, F::FIELD_ID, LOGN, &tb, hb::GroupNtt<F, LOGN, T>::LOGV);
  if (rc) return rc;
  prm.tw = (const W *)tb->tw;
  prm.itw = (const W *)tb->itw;
  prm.scale = (W)tb->key_scale;
  auto kern = hb::keygen_rows_kernel<F, LOGN, T>;
  const size_t smem = sizeof(W) * (2 * hb::tw_words<W>() * N + 2 * 2 * N);
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>((prm.rows + 1) / 2, (size_t)ctx->sms * 4));
  kern<<<grid, 2 * T, smem, ctx->stream>>>(prm);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? HB_OK : cuda_fail(ctx, e, "keygen launch");
}

// BSK and KSK rows of p on the device into keys->bsk / keys->ksk (slot layout of keys'
// threads_per_gate), from the secret keys lwe_sk / ring_sk (host words).
template <class F>
int generate_keys(hb_ctx *ctx, const hb_params &p, uint64_t seed, const void *lwe_sk,
                  const void *ring_sk, hb_keys *k) {
  using W = typename F::W;
  const uint32_t N = p.ring_dim, n = p.lwe_dim, M = ks_dim(p), stride = N / M;
  if (N != 1024) return fail(ctx, HB_ERR_UNSUPPORTED, "device key generation is compiled for N = 1024");
  // device copies: LWE key, ring key, and both multiplier keys (ring key z for the BSK rows, the
  // LWE key padded to n' words and spread to N for the KSK rows) before their transforms
  std::vector<W> host(2 * (size_t)N, 0);
  std::memcpy(host.data(), ring_sk, sizeof(W) * N);
  for (uint32_t u = 0; u < n; ++u) host[N + (size_t)u * stride] = ((const W *)lwe_sk)[u];
  void *d_tmp = nullptr;
  int rc = dev_alloc(ctx, sizeof(W) * (6 * (size_t)N + n), &d_tmp);
  if (rc) return rc;
  W *d_raw = (W *)d_tmp, *d_keys = d_raw + 2 * N, *d_ring = d_keys + 2 * N, *d_lwe = d_ring + N;
  cudaError_t e = cudaMemcpyAsync(d_raw, host.data(), sizeof(W) * 2 * N, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_ring, ring_sk, sizeof(W) * N, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_lwe, lwe_sk, sizeof(W) * n, cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) rc = cuda_fail(ctx, e, "key generation upload");
  const int T = k->threads_per_gate;
  if (!rc) rc = prepare_field(ctx, p.field_id, 10, T, d_raw, d_keys, 2);
  hb::KeygenParams<W> prm{};
  prm.lwe_sk = d_lwe;
  prm.ring_sk = d_ring;
  prm.seed = seed;
  prm.n = n;
  prm.len = p.br_len;
  prm.bits = p.br_bits;
  prm.pairs = p.lwe_ternary ? 2 : 1;
  prm.ks_n = M;
  prm.ks_len = p.ks_len;
  W pw = 1;
  const W bks = (W)(1ULL << p.ks_bits);
  for (uint32_t j = 0; j < p.ks_len && j < 64; ++j) {
    prm.ks_pow[j] = F::to_mont(pw);
    pw = hb::host_mulmod<F>(pw, bks);
  }
  auto launch = [&](void) -> int {
    if (T == 64) return launch_keygen<F, 10, 64>(ctx, prm);
    if (T == 128) return launch_keygen<F, 10, 128>(ctx, prm);
    return fail(ctx, HB_ERR_UNSUPPORTED, "no key generation kernel for %d threads per gate", T);
  };
  if (!rc) {  // RGSW rows under the ring key
    prm.out = (W *)k->bsk;
    prm.key = d_keys;
    prm.sigma = p.ring_noise_std;
    prm.rows = n * prm.pairs * 2 * p.br_len;
    prm.ksk = 0;
    rc = launch();
  }
  if (!rc) {  // key-switching rows under the padded LWE key
    prm.out = (W *)k->ksk;
    prm.key = d_keys + N;
    prm.sigma = p.ks_noise_std;
    prm.rows = (N / M) * p.ks_len;
    prm.ksk = 1;
    rc = launch();
  }
  e = cudaStreamSynchronize(ctx->stream);
  dev_free(ctx, d_tmp);
  if (!rc && e != cudaSuccess) rc = cuda_fail(ctx, e, "key generation");
  return rc;
}

}  // namespace

extern "C" int hb_keys_generate(hb_ctx *ctx, const hb_params *p, uint64_t seed, void *lwe_sk,
                                void *ring_sk, hb_keys **out) {
  if (!ctx || !out || !lwe_sk || !ring_sk) return HB_ERR_INVALID;
  *out = nullptr;
  if (hb_params_validate(p) != HB_OK) return fail(ctx, HB_ERR_INVALID, "invalid parameter set");
  if (p->ks_len > 64) return fail(ctx, HB_ERR_UNSUPPORTED, "more than 64 key-switching digits");
  // the secret keys are drawn on the host (n + N words): KeyGen::generate_secret_key
  int rc = hb_keygen(p, seed, lwe_sk, ring_sk, nullptr, nullptr, 1);
  if (rc) return fail(ctx, rc, "secret key generation");
  cudaSetDevice(ctx->device);
  size_t nb = 0;
  hb_params_sizes(p, nullptr, nullptr, &nb, nullptr, nullptr);
  const size_t nkd = ksk_device_words(*p), ws = word_size(*p);
  hb_keys *k = new hb_keys();
  k->p = *p;
  k->threads_per_gate = default_threads_per_gate(p->field_id);
  rc = dev_alloc(ctx, nb * ws, &k->bsk);
  if (!rc) rc = dev_alloc(ctx, nkd * ws, &k->ksk);
  if (!rc) {
    if (p->field_id == HB_FIELD_GOLDILOCKS)
      rc = generate_keys<Goldilocks>(ctx, *p, seed, lwe_sk, ring_sk, k);
    else if (p->field_id == HB_FIELD_BABYBEAR)
      rc = generate_keys<BabyBear>(ctx, *p, seed, lwe_sk, ring_sk, k);
    else
      rc = generate_keys<DefaultFieldU32>(ctx, *p, seed, lwe_sk, ring_sk, k);
  }
  if (rc) {
    dev_free(ctx, k->bsk);
    dev_free(ctx, k->ksk);
    delete k;
    return rc;
  }
  k->bytes = (nb + nkd) * ws;
  k->gates_per_cta = default_gates_per_cta(p->field_id);
  const std::vector<int> cand = variants(*p, k->threads_per_gate);
  if (cand.size() && std::find(cand.begin(), cand.end(), k->gates_per_cta) == cand.end())
    k->gates_per_cta = cand.back();
  rc = dp_tables(ctx, *p, k->threads_per_gate);
  if (rc) {
    hb_keys_free(ctx, k);
    return rc;
  }
  *out = k;
  return HB_OK;
}

extern "C" int hb_encrypt_device(hb_ctx *ctx, const hb_params *p, const void *d_lwe_sk, uint64_t seed,
                                 uint64_t index0, const uint8_t *d_bits, size_t count, void *d_out) {
  if (!ctx || !d_lwe_sk || (count && (!d_bits || !d_out))) return HB_ERR_INVALID;
  if (hb_params_validate(p) != HB_OK) return fail(ctx, HB_ERR_INVALID, "invalid parameter set");
  if (count == 0) return HB_OK;
  cudaSetDevice(ctx->device);
  const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>((count + 7) / 8, (size_t)ctx->sms * 16));
  if (p->field_id == HB_FIELD_GOLDILOCKS)
    hb::lwe_encrypt_kernel<Goldilocks><<<grid, 256, 0, ctx->stream>>>(
        (const uint64_t *)d_lwe_sk, d_bits, (uint64_t *)d_out, count, p->lwe_dim, seed, index0, p->lwe_noise_std);
  else if (p->field_id == HB_FIELD_BABYBEAR)
    hb::lwe_encrypt_kernel<BabyBear><<<grid, 256, 0, ctx->stream>>>(
        (const uint32_t *)d_lwe_sk, d_bits, (uint32_t *)d_out, count, p->lwe_dim, seed, index0, p->lwe_noise_std);
  else
    hb::lwe_encrypt_kernel<DefaultFieldU32><<<grid, 256, 0, ctx->stream>>>(
        (const uint32_t *)d_lwe_sk, d_bits, (uint32_t *)d_out, count, p->lwe_dim, seed, index0, p->lwe_noise_std);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? HB_OK : cuda_fail(ctx, e, "encrypt launch");
}

// ------------------------------------------------------------------------------------------
// Allocation-free MUX (hb_gate_mux_device_noalloc)
//
// For callers that may not allocate device memory during a call. Everything the two-layer MUX
// needs beyond its inputs and outputs -- the status word, the job table and the two intermediate
// ciphertext batches -- lives in one array compiled into this library.
// ------------------------------------------------------------------------------------------

namespace {

constexpr size_t kNoAllocBytes = 16u << 20;  // 16 MiB, held by every GPU that loads the library
constexpr size_t kNoAllocStatus = 0;         // int status word
constexpr size_t kNoAllocJobs = 256;         // three GateJob records
constexpr size_t kNoAllocData = 1024;        // t0 | t1, count * (n + 1) words each

static_assert(kNoAllocStatus + sizeof(int) <= kNoAllocJobs, "status word overlaps the job table");
static_assert(kNoAllocJobs + 3 * sizeof(GateJob) <= kNoAllocData, "job table overlaps the ciphertexts");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;

// Host code only sees a host-side stand-in named g_noalloc_scratch; the kernels need the device
// address, looked up with the context's device current by the first call on each context (kept
// on the context, so a context created after a device reset never uses a stale address).
int noalloc_address(hb_ctx *ctx, unsigned char **out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!ctx->noalloc_addr) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress(no-allocation scratch)");
    ctx->noalloc_addr = p;
  }
  *out = (unsigned char *)ctx->noalloc_addr;
  return HB_OK;
}

// Gates per CTA of the allocation-free MUX: the keys' variant, or, when that is the one-gate
// latency variant (which the batched launches here do not use), the smallest compiled G > 1 for
// the keys' group size.
int noalloc_gates_per_cta(const hb_keys *keys) {
  if (keys->gates_per_cta > 1) return keys->gates_per_cta;
  std::vector<int> v = variants(keys->p, keys->threads_per_gate);
  return v.empty() ? 0 : *std::min_element(v.begin(), v.end());
}

template <class F, int LOGN, int T, int G, bool TERN, bool KSC>
int launch_noalloc(hb_ctx *ctx, hb_keys *keys, const DevTables *tb, const GateJob *djobs, int njobs,
                   uint32_t batches, int *dstatus) {
  using W = typename F::W;
  constexpr int N = 1 << LOGN;
  hb::BootParams<W> prm{};
  boot_params(prm, ctx, keys, tb);
  prm.jobs = djobs;
  prm.njobs = njobs;
  prm.total_batches = batches;
  prm.status = dstatus;  // withhold keeps the context's test setting (boot_params)
  constexpr int S = hb::boot_stages<W, N, G>();
  auto kern = hb::bootstrap_kernel<F, LOGN, T, G, S, TERN, KSC>;
  const size_t smem = hb::boot_smem_bytes<W, N, G, S>(prm.n);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "bootstrap smem attribute");
  const unsigned grid = std::min<unsigned>(batches, (unsigned)ctx->sms);
  kern<<<grid, G * T, smem, ctx->stream>>>(prm);
  e = cudaGetLastError();
  return e == cudaSuccess ? HB_OK : cuda_fail(ctx, e, "bootstrap launch");
}

int noalloc_layer(hb_ctx *ctx, hb_keys *keys, const DevTables *tb, const GateJob *djobs, int njobs,
                  uint32_t batches, int *dstatus, int G) {
  const int T = keys->threads_per_gate, fld = keys->p.field_id;
  const bool tern = keys->p.lwe_ternary != 0, ksc = ks_dim(keys->p) < keys->p.ring_dim;
#define HB_CASE(FLD, TT, GG, TN, KC)                                                       \
  if (fld == field_of<FLD>() && T == TT && G == GG && GG > 1 && tern == TN && ksc == KC) \
    return launch_noalloc<FLD, 10, TT, GG, TN, KC>(ctx, keys, tb, djobs, njobs, batches, dstatus);
  HB_BOOT_VARIANTS(HB_CASE)
#undef HB_CASE
  return fail(ctx, HB_ERR_UNSUPPORTED, "no compiled kernel with %d gates per CTA", G);
}

}  // namespace

extern "C" int hb_gate_mux_device_noalloc(hb_ctx *ctx, hb_keys *keys, const void *c0, const void *c1,
                                          const void *c2, void *out, size_t count) {
  if (!ctx || !keys) return HB_ERR_INVALID;
  if (!c0 || !c1 || !c2 || !out) return fail(ctx, HB_ERR_INVALID, "missing ciphertext buffer");
  if (count == 0) return HB_OK;
  const hb_params &p = keys->p;
  if (p.ring_dim != 1024) return fail(ctx, HB_ERR_UNSUPPORTED, "bootstrapping is compiled for N = 1024");
  const uint64_t P = modulus_of(p.field_id);
  const size_t width = (size_t)p.lwe_dim + 1, ws = word_size(p);
  const size_t max_gates = (kNoAllocBytes - kNoAllocData) / (2 * width * ws);
  if (count > max_gates)
    return fail(ctx, HB_ERR_INVALID,
                "%zu gates exceed the no-allocation scratch of %zu bytes (at most %zu gates for this "
                "parameter set)", count, kNoAllocBytes, max_gates);
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  // The NTT tables were built when the keys were uploaded; this path must not build (allocate) them.
  const int lv = keys->threads_per_gate == 128 ? 3 : 4;
  const DevTables *tb = &ctx->tables[p.field_id][10][lv];
  if (!tb->tw) return fail(ctx, HB_ERR_INVALID, "keys were not uploaded on this context");
  unsigned char *base = nullptr;
  int rc = noalloc_address(ctx, &base);
  if (rc) return rc;
  int *dstatus = (int *)(base + kNoAllocStatus);
  GateJob *djobs = (GateJob *)(base + kNoAllocJobs);
  unsigned char *t0 = base + kNoAllocData, *t1 = t0 + count * width * ws;

  // MUX (tfhe/src/bfhe/evaluate.rs:245-262): t0 = and(c0, c1), t1 = and(not c0, c2) in one launch,
  // then out = bootstrap(t0 + t1, or) in a second.
  const int G = noalloc_gates_per_cta(keys);
  if (G <= 1) return fail(ctx, HB_ERR_UNSUPPORTED, "no batched kernel compiled for these keys");
  GateJob jobs[3];
  jobs[0] = make_job(P, HB_GATE_AND, p.ring_dim, c0, c1, nullptr, t0, (uint32_t)count);
  jobs[1] = jobs[0];
  jobs[1].in1 = c2;
  jobs[1].out = t1;
  jobs[1].s0 = -1;  // not(c0) = -c0 + Q/4 on the body
  jobs[1].add_b = P >> 2;
  jobs[2] = make_job(P, HB_GATE_MUX, p.ring_dim, t0, t1, nullptr, out, (uint32_t)count);
  const uint32_t per_job = (uint32_t)((count + G - 1) / G);
  jobs[0].first_batch = 0;
  jobs[1].first_batch = per_job;
  jobs[2].first_batch = 0;

  // The array keeps the previous call's contents: the status word must start at zero.
  e = cudaMemsetAsync(dstatus, 0, sizeof(int), ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(djobs, jobs, sizeof(jobs), cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "no-allocation scratch setup");
  // The second layer reads t0 and t1, so it runs only when the first one finished all its waits.
  int h = 0;
  for (int layer = 0; layer < 2; ++layer) {
    rc = layer == 0 ? noalloc_layer(ctx, keys, tb, djobs, 2, 2 * per_job, dstatus, G)
                    : noalloc_layer(ctx, keys, tb, djobs + 2, 1, per_job, dstatus, G);
    if (rc) return rc;
    e = cudaMemcpyAsync(&h, dstatus, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "no-allocation MUX");
    if (h) return fail(ctx, HB_ERR_TIMEOUT, "a device-side wait exceeded its limit (status %d)", h);
  }
  return HB_OK;
}

// ------------------------------------------------------------------------------------------
// Autotuner and mixed-set batches
// ------------------------------------------------------------------------------------------

namespace {

// Re-lays the device keys out for groups of T threads (stream-ordered on the context stream).
int relayout_keys(hb_ctx *ctx, hb_keys *keys, int T) {
  if (keys->threads_per_gate == T) return HB_OK;
  const size_t ws = word_size(keys->p);
  size_t nb = 0;
  hb_params_sizes(&keys->p, nullptr, nullptr, &nb, nullptr, nullptr);
  const size_t nk = ksk_device_words(keys->p);
  uint32_t logn = 0;
  while ((1u << logn) < keys->p.ring_dim) ++logn;
  DevTables *tb;
  const uint32_t logv = logn - (T == 128 ? 7 : 6);
  int rc = tables(ctx, keys->p.field_id, logn, &tb, logv);  // the new group size's twiddles
  void *nbsk = nullptr, *nksk = nullptr;
  if (!rc) rc = dev_alloc(ctx, nb * ws, &nbsk);
  if (!rc) rc = dev_alloc(ctx, nk * ws, &nksk);
  if (rc) {
    dev_free(ctx, nbsk);
    return rc;
  }
  const unsigned grid = (unsigned)ctx->sms * 8;
  const int N = (int)keys->p.ring_dim, Tf = keys->threads_per_gate;
  if (ws == 8) {
    hb::relayout_kernel<uint64_t><<<grid, 256, 0, ctx->stream>>>((const uint64_t *)keys->bsk, (uint64_t *)nbsk, nb, N, Tf, T);
    hb::relayout_kernel<uint64_t><<<grid, 256, 0, ctx->stream>>>((const uint64_t *)keys->ksk, (uint64_t *)nksk, nk, N, Tf, T);
  } else {
    hb::relayout_kernel<uint32_t><<<grid, 256, 0, ctx->stream>>>((const uint32_t *)keys->bsk, (uint32_t *)nbsk, nb, N, Tf, T);
    hb::relayout_kernel<uint32_t><<<grid, 256, 0, ctx->stream>>>((const uint32_t *)keys->ksk, (uint32_t *)nksk, nk, N, Tf, T);
  }
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    dev_free(ctx, nbsk);
    dev_free(ctx, nksk);
    return cuda_fail(ctx, e, "key relayout");
  }
  dev_free(ctx, keys->bsk);
  dev_free(ctx, keys->ksk);
  keys->bsk = nbsk;
  keys->ksk = nksk;
  keys->threads_per_gate = T;
  return dp_tables(ctx, keys->p, T);
}

bool compiled(const hb_params &p, int T, int G) {
  for (int g : variants(p, T))
    if (g == G) return true;
  return false;
}

}  // namespace

extern "C" int hb_keys_set_config(hb_ctx *ctx, hb_keys *keys, int threads_per_gate, int gates_per_cta) {
  if (!ctx || !keys) return HB_ERR_INVALID;
  if (!compiled(keys->p, threads_per_gate, gates_per_cta))
    return fail(ctx, HB_ERR_UNSUPPORTED, "no compiled kernel with %d threads per gate and %d gates per CTA",
                threads_per_gate, gates_per_cta);
  cudaSetDevice(ctx->device);
  int rc = relayout_keys(ctx, keys, threads_per_gate);
  if (rc) return rc;
  keys->gates_per_cta = gates_per_cta;
  return HB_OK;
}

extern "C" int hb_keys_set_rate(hb_keys *keys, double gates_per_s) {
  if (!keys || !(gates_per_s >= 0)) return HB_ERR_INVALID;
  keys->gates_per_s = gates_per_s;
  return HB_OK;
}

extern "C" int hb_keys_config(const hb_keys *keys, int *threads_per_gate, int *gates_per_cta) {
  if (!keys) return HB_ERR_INVALID;
  if (threads_per_gate) *threads_per_gate = keys->threads_per_gate;
  if (gates_per_cta) *gates_per_cta = keys->gates_per_cta;
  return HB_OK;
}

extern "C" int hb_autotune(hb_ctx *ctx, hb_keys *keys, uint32_t sample_gates, int *chosen_threads,
                           int *chosen, double *gates_per_s) {
  if (!ctx || !keys) return HB_ERR_INVALID;
  if (keys->p.ring_dim != 1024) return fail(ctx, HB_ERR_UNSUPPORTED, "bootstrapping is compiled for N = 1024");
  cudaSetDevice(ctx->device);
  if (sample_gates == 0) sample_gates = (uint32_t)ctx->sms * 24;  // whole waves for every candidate G
  const size_t width = (size_t)keys->p.lwe_dim + 1, ws = word_size(keys->p);
  const size_t bytes = (size_t)sample_gates * width * ws;
  void *buf = nullptr, *tab = nullptr;
  int rc = dev_alloc(ctx, 2 * bytes, &buf);
  if (!rc) rc = dev_alloc(ctx, sizeof(GateJob), &tab);
  if (rc) {
    dev_free(ctx, buf);
    return rc;
  }
  cudaMemsetAsync(buf, 0, 2 * bytes, ctx->stream);  // any ciphertexts time the same: zeros
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int best_g = keys->gates_per_cta, best_t = keys->threads_per_gate;
  double best_rate = 0;
  for (int T : {64, 128})
  for (int G : variants(keys->p, T)) {
    if (!rc) rc = relayout_keys(ctx, keys, T);
    if (rc) break;
    std::vector<GateJob> jobs{make_job(modulus_of(keys->p.field_id), HB_GATE_NAND, 1024, buf, buf,
                                       nullptr, (char *)buf + bytes, sample_gates)};
    jobs[0].first_batch = 0;
    const uint32_t batches = batches_of(jobs, G);
    cudaMemcpyAsync(tab, jobs.data(), sizeof(GateJob), cudaMemcpyHostToDevice, ctx->stream);
    float best_ms = 1e30f;
    for (int rep = 0; rep < 3 && !rc; ++rep) {  // rep 0 warms up
      cudaEventRecord(e0, ctx->stream);
      rc = launch_table_any(ctx, keys, G, (const GateJob *)tab, 1, batches, ctx->sms, ctx->stream);
      cudaEventRecord(e1, ctx->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) rc = cuda_fail(ctx, cudaGetLastError(), "autotune");
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0) best_ms = std::min(best_ms, ms);
    }
    if (rc) break;
    const double rate = sample_gates / (best_ms * 1e-3);
    if (rate > best_rate) {
      best_rate = rate;
      best_g = G;
      best_t = T;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dev_free(ctx, buf);
  dev_free(ctx, tab);
  if (!rc) rc = check_status(ctx);
  if (!rc) rc = relayout_keys(ctx, keys, best_t);
  if (rc) return rc;
  keys->gates_per_cta = best_g;
  keys->gates_per_s = best_rate;
  if (chosen_threads) *chosen_threads = best_t;
  if (chosen) *chosen = best_g;
  if (gates_per_s) *gates_per_s = best_rate;
  return HB_OK;
}

struct hb_batch {
  struct Group {
    hb_keys *keys = nullptr;
    void *djobs = nullptr;
    int njobs = 0;
    uint32_t batches = 0;
    unsigned grid = 0;
    int gates_per_cta = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
  };
  std::vector<Group> groups;
  cudaEvent_t fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint64_t gates = 0;
};

extern "C" void hb_batch_free(hb_ctx *ctx, hb_batch *b) {
  if (!ctx || !b) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto &g : b->groups) {
    dev_free(ctx, g.djobs);
    if (g.stream) cudaStreamDestroy(g.stream);
    if (g.done) cudaEventDestroy(g.done);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  delete b;
}

extern "C" int hb_batch_create(hb_ctx *ctx, const hb_job *jobs, size_t njobs, hb_batch **out) {
  if (!ctx || !out || (njobs && !jobs)) return HB_ERR_INVALID;
  *out = nullptr;
  cudaSetDevice(ctx->device);
  // group the jobs by key set: one persistent launch per parameter set
  std::vector<hb_keys *> keysets;
  std::vector<std::vector<GateJob>> tables_h;
  uint64_t gates = 0;
  for (size_t i = 0; i < njobs; ++i) {
    const hb_job &j = jobs[i];
    if (!j.keys || !j.c0 || !j.out || !single_bootstrap_gate(j.gate) || (j.count && !j.c1) ||
        (j.gate == HB_GATE_MAJORITY && !j.c2))
      return fail(ctx, HB_ERR_INVALID, "job %zu: bad keys, buffers or gate (batches take single-bootstrap gates)", i);
    if (j.keys->p.ring_dim != 1024) return fail(ctx, HB_ERR_UNSUPPORTED, "bootstrapping is compiled for N = 1024");
    if (j.count == 0) continue;
    size_t k = 0;
    while (k < keysets.size() && keysets[k] != j.keys) ++k;
    if (k == keysets.size()) {
      keysets.push_back(j.keys);
      tables_h.emplace_back();
    }
    tables_h[k].push_back(make_job(modulus_of(j.keys->p.field_id), j.gate, 1024, j.c0, j.c1, j.c2, j.out,
                                   j.count));
    gates += j.count;
  }
  hb_batch *b = new hb_batch();
  b->gates = gates;
  // Every set's kernel gets a full grid on its own stream: the block scheduler backfills SMs
  // from the next set's CTAs as the previous set's CTAs retire, which measured within 2 % of
  // the sum of the per-set full-GPU times (a static SM split by estimated work lost 28 %).
  int rc = HB_OK;
  for (size_t k = 0; k < keysets.size() && !rc; ++k) {
    hb_batch::Group grp;
    grp.keys = keysets[k];
    auto &tab = tables_h[k];
    uint64_t set_gates = 0;
    for (auto &t : tab) set_gates += t.count;
    const int G = launch_gates_per_cta(ctx, grp.keys, set_gates);
    grp.gates_per_cta = G;
    uint32_t bsum = 0;
    for (auto &t : tab) {
      t.first_batch = bsum;
      bsum += (t.count + G - 1) / G;
    }
    grp.batches = bsum;
    grp.njobs = (int)tab.size();
    grp.grid = std::max(1u, std::min((unsigned)ctx->sms, bsum));
    rc = dev_alloc(ctx, sizeof(GateJob) * tab.size(), &grp.djobs);
    if (!rc) {
      cudaMemcpy(grp.djobs, tab.data(), sizeof(GateJob) * tab.size(), cudaMemcpyHostToDevice);
      if (cudaStreamCreateWithFlags(&grp.stream, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&grp.done, cudaEventDisableTiming) != cudaSuccess)
        rc = fail(ctx, HB_ERR_CUDA, "stream creation");
    }
    b->groups.push_back(grp);
  }
  if (!rc && cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
    rc = fail(ctx, HB_ERR_CUDA, "event creation");
  // capture: fork from the context stream, one persistent kernel per set on its own stream, join
  if (!rc) {
    cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) e = cudaEventRecord(b->fork, ctx->stream);
    for (auto &grp : b->groups) {
      if (e != cudaSuccess || rc) break;
      e = cudaStreamWaitEvent(grp.stream, b->fork, 0);
      if (e == cudaSuccess)
        rc = launch_table_any(ctx, grp.keys, grp.gates_per_cta, (const GateJob *)grp.djobs, grp.njobs,
                              grp.batches, grp.grid, grp.stream);
      if (e == cudaSuccess && !rc) e = cudaEventRecord(grp.done, grp.stream);
      if (e == cudaSuccess && !rc) e = cudaStreamWaitEvent(ctx->stream, grp.done, 0);
    }
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &g);
    if (e == cudaSuccess) e = e2;
    b->graph = g;
    if (e == cudaSuccess && !rc) e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess && !rc) rc = cuda_fail(ctx, e, "batch graph capture");
  }
  if (rc) {
    hb_batch_free(ctx, b);
    return rc;
  }
  ctx->launches -= b->groups.size();  // capture is not execution: count launches when replayed
  *out = b;
  return HB_OK;
}

extern "C" int hb_batch_launch(hb_ctx *ctx, hb_batch *b) {
  if (!ctx || !b || !b->exec) return HB_ERR_INVALID;
  cudaSetDevice(ctx->device);
  cudaError_t e = cudaGraphLaunch(b->exec, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph launch");
  ctx->launches += b->groups.size();
  return HB_OK;
}

extern "C" int hb_batch_info(const hb_batch *b, uint64_t *gates, int *launches, int *grid_out, int grid_cap) {
  if (!b) return HB_ERR_INVALID;
  if (gates) *gates = b->gates;
  if (launches) *launches = (int)b->groups.size();
  for (int k = 0; grid_out && k < grid_cap && k < (int)b->groups.size(); ++k) grid_out[k] = (int)b->groups[k].grid;
  return HB_OK;
}

// ------------------------------------------------------------------------------------------
// Helpers shared with the serving loop (hb_serve.cu)
// ------------------------------------------------------------------------------------------

namespace hbrt {

int launch_set(hb_ctx *ctx, hb_keys *keys, int G, const GateJob *djobs, int njobs, uint32_t batches,
               cudaStream_t stream) {
  return launch_table_any(ctx, keys, G, djobs, njobs, batches, (unsigned)ctx->sms, stream);
}

// Gates per CTA for one launch of `gates` gates: the keys' autotuned (throughput) choice, unless that
// leaves SMs idle; then the smallest compiled variant that still gives every CTA an SM of its own,
// so that fewer gates share an SM and a small launch finishes sooner.
int launch_gates_per_cta(const hb_ctx *ctx, const hb_keys *keys, uint64_t gates) {
  const int tuned = keys->gates_per_cta;
  const uint64_t sms = (uint64_t)std::max(1, ctx->sms);
  if (gates >= sms * (uint64_t)tuned) return tuned;
  std::vector<int> cand = variants(keys->p, keys->threads_per_gate);
  cand.push_back(1);
  std::sort(cand.begin(), cand.end());
  for (int g : cand)
    if (g <= tuned && (gates + g - 1) / g <= sms) return g;
  return tuned;
}

int gate_job(const hb_params &p, int gate, const void *c0, const void *c1, const void *c2, void *out,
             uint32_t count, GateJob *job) {
  if (!single_bootstrap_gate(gate) || p.ring_dim != 1024) return HB_ERR_INVALID;
  *job = make_job(modulus_of(p.field_id), gate, 1024, c0, c1, c2, out, count);
  return HB_OK;
}

}  // namespace hbrt

