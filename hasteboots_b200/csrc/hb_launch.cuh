// hb_launch.cuh -- launch-parameter setup shared by the translation units that launch the
// bootstrapping kernels (hb_api.cu, hb_trace.cu).
#pragma once

#include "hb_kernels.cuh"
#include "hb_runtime.h"

namespace hbrt {

// The launch-independent fields of a bootstrap launch's parameters.
template <class W>
void boot_params(hb::BootParams<W> &prm, hb_ctx *ctx, const hb_keys *keys, const DevTables *tb) {
  prm.bsk = (const W *)keys->bsk;
  prm.ksk = (const W *)keys->ksk;
  prm.tw = (const W *)tb->tw;
  prm.itw = (const W *)tb->itw;
  prm.n = keys->p.lwe_dim;
  prm.len = keys->p.br_len;
  prm.bits = keys->p.br_bits;
  prm.ks_len = keys->p.ks_len;
  prm.ks_bits = keys->p.ks_bits;
  prm.ks_n = ks_dim(keys->p);
  prm.ks_chunks = keys->p.ring_dim / prm.ks_n;
  prm.status = ctx->d_status;
  prm.budget = wait_budget(ctx);
  prm.withhold = ctx->withhold_keys;
}

}  // namespace hbrt
