// hb_trace.cu -- traced bootstrapping of a batch (hb_bootstrap_trace_device).
//
// vfhe's bootstrap (vfhe/src/bfhe/evaluate.rs:47-141) records, while it bootstraps, the witness of
// its proof: the accumulator after every blind-rotation round (AccTrace, trace/src/acc_trace.rs,
// filled by blind_rotate_w_trace, fhe_core/src/blind_rotation/rlwe/binary.rs:106-205) and, per
// round, the gadget digits of (X^a_i - 1) ACC that the external product decomposes (the bit
// polynomials of SumHadamardTrace, appended by mul_polynomial_inplace_fast_w_traces,
// lattice/src/gadget/rlwe.rs:426-457). Here a whole batch of gates runs in one persistent launch of
// the batched kernel's TRACE variant, two gates per CTA, each gate writing its own slab of both.
// The digits' NTTs and the NTT-domain key rows that the reference also records are left out: their
// slot order is concrete-ntt's, which nothing here can reproduce.

#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/hb_gpu.h"
#include "hb_kernels.cuh"
#include "hb_launch.cuh"
#include "hb_runtime.h"

using hb::BabyBear;
using hb::DefaultFieldU32;
using hb::GateJob;
using hb::Goldilocks;
using namespace hbrt;

namespace {

constexpr int kTraceGates = 2;  // gates per CTA of the traced launch

template <class F, int T, bool KSC>
int launch_trace(hb_ctx *ctx, hb_keys *keys, const GateJob *djob, uint32_t count, void *acc_trace,
                 void *digit_trace) {
  using W = typename F::W;
  constexpr int LOGN = 10, N = 1 << LOGN, G = kTraceGates;
  DevTables *tb;
  int rc = tables(ctx, F::FIELD_ID, LOGN, &tb, hb::GroupNtt<F, LOGN, T>::LOGV);
  if (rc) return rc;
  hb::BootParams<W> prm{};
  boot_params(prm, ctx, keys, tb);
  prm.jobs = djob;
  prm.njobs = 1;
  prm.total_batches = (count + G - 1) / G;
  prm.trace = (W *)acc_trace;
  prm.digits = (uint8_t *)digit_trace;
  constexpr int S = hb::boot_stages<W, N, G>();
  auto kern = hb::bootstrap_kernel<F, LOGN, T, G, S, false, KSC, true>;
  const size_t smem = hb::boot_smem_bytes<W, N, G, S>(prm.n);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "traced bootstrap smem attribute");
  const unsigned grid = std::min<unsigned>(prm.total_batches, (unsigned)ctx->sms);
  kern<<<grid, G * T, smem, ctx->stream>>>(prm);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "traced bootstrap launch");
  ctx->launches += 1;
  return HB_OK;
}

// Compiled traced variants: (field, threads per gate, key switch in chunks of n' < N words); the
// group size follows the keys' slot layout.
#define HB_TRACE_VARIANTS(X)                                                                    \
  X(Goldilocks, 128, false) X(Goldilocks, 128, true) X(Goldilocks, 64, false)                 \
  X(BabyBear, 64, false) X(BabyBear, 64, true) X(BabyBear, 128, false)                        \
  X(DefaultFieldU32, 64, false) X(DefaultFieldU32, 64, true) X(DefaultFieldU32, 128, false)   \
  X(DefaultFieldU32, 128, true)

}  // namespace

extern "C" int hb_bootstrap_trace_device(hb_ctx *ctx, hb_keys *keys, const void *c, const void *lut,
                                         void *out, size_t count, void *acc_trace, void *digit_trace) {
  if (!ctx || !keys || !c || !lut || !out || !acc_trace) return HB_ERR_INVALID;
  if (count == 0) return HB_OK;
  const hb_params &p = keys->p;
  if (count > 0xFFFFFFFFull) return fail(ctx, HB_ERR_INVALID, "too many gates in one call");
  if (p.lwe_ternary) return fail(ctx, HB_ERR_UNSUPPORTED, "traces are recorded under binary LWE keys");
  if (p.ring_dim != 1024) return fail(ctx, HB_ERR_UNSUPPORTED, "bootstrapping is compiled for N = 1024");
  if (digit_trace && p.br_bits > 8)
    return fail(ctx, HB_ERR_UNSUPPORTED, "digit traces hold bytes: the gadget base must be at most 2^8");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
  GateJob job{};
  job.in0 = c;
  job.out = out;
  job.lut = lut;
  job.s0 = 1;
  job.count = (uint32_t)count;
  job.first_batch = 0;
  int rc = scratch(ctx, ctx->jobs, sizeof(GateJob));
  if (rc) return rc;
  e = cudaMemcpyAsync(ctx->jobs.ptr, &job, sizeof(GateJob), cudaMemcpyHostToDevice, ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "job table upload");
  const GateJob *djob = (const GateJob *)ctx->jobs.ptr;
  const int T = keys->threads_per_gate, fld = p.field_id;
  const bool ksc = ks_dim(p) < p.ring_dim;
#define HB_CASE(FLD, TT, KC)                                                 \
  if (fld == FLD::FIELD_ID && T == TT && ksc == KC)                         \
    return launch_trace<FLD, TT, KC>(ctx, keys, djob, (uint32_t)count, acc_trace, digit_trace);
  HB_TRACE_VARIANTS(HB_CASE)
#undef HB_CASE
  return fail(ctx, HB_ERR_UNSUPPORTED, "no traced kernel for %d threads per gate", T);
}
