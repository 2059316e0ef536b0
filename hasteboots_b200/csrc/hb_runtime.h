// hb_runtime.h -- host-side context and key handles shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <string>
#include <utility>
#include <vector>

#include "../../include/hb_gpu.h"

namespace hb {
struct GateJob;
}

namespace hbrt {

struct DevTables {
  void *tw = nullptr;   // N entries of F::Tw: psi^brv(k) (the 32-bit fields: with its Shoup quotient)
  void *itw = nullptr;  // psi^-brv(k), the same way
  unsigned long long n_inv = 0;      // multiplier giving x * N^-1
  unsigned long long key_scale = 0;  // multiplier applied to key words at upload
};

struct Scratch {
  void *ptr = nullptr;
  size_t cap = 0;
};

}  // namespace hbrt

struct hb_ctx {
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  int *d_status = nullptr;
  size_t budget = 0;
  size_t in_use = 0;
  std::vector<std::pair<void *, size_t>> sizes;
  std::string err;
  hbrt::DevTables tables[3][13][6];  // [field][log2 N][log2 words per thread]
  hbrt::Scratch jobs, io, mux_tmp;
  std::atomic<unsigned long long> launches{0};  // bootstrap kernel launches issued by this context
  long long wait_limit = 0;                     // SM clock cycles per bounded wait; 0 = default
  int withhold_keys = 0;                        // test hook: bootstrap launches issue no key copies
  // latency-form clusters the GPU holds with one cluster CTA per SM ([Goldilocks, 32-bit fields] x
  // [T = 64, 128]); -1 unknown. Atomic: the serving loop's worker thread launches on the context too.
  std::atomic<int> dp_clusters[4] = {-1, -1, -1, -1};
  // device address of the allocation-free MUX's in-library array, looked up by the first such call
  // on this context (a context made after a device reset looks it up again)
  void *noalloc_addr = nullptr;
};

struct hb_keys {
  hb_params p{};
  void *bsk = nullptr;
  void *ksk = nullptr;
  size_t bytes = 0;
  int threads_per_gate = 64;  // T: key slot layout and kernel group size
  int gates_per_cta = 4;      // persistent-kernel variant (autotuned)
  double gates_per_s = 0;   // measured by hb_autotune (0: not calibrated)
};

namespace hbrt {
int fail(hb_ctx *ctx, int code, const char *fmt, ...);
int cuda_fail(hb_ctx *ctx, cudaError_t e, const char *what);
int dev_alloc(hb_ctx *ctx, size_t bytes, void **out);
void dev_free(hb_ctx *ctx, void *p);
int scratch(hb_ctx *ctx, Scratch &s, size_t bytes);
int tables(hb_ctx *ctx, int field_id, uint32_t logn, DevTables **out, uint32_t logv = 4);
int check_status(hb_ctx *ctx);
long long wait_budget(const hb_ctx *ctx);
// The key switch's dimension n' = next_pow2(n) (fhe_core/src/key_switch/rlwe.rs:40-43).
uint32_t ks_dim(const hb_params &p);
// One persistent bootstrapping launch over a device job table (full grid, the keys' variant).
int launch_set(hb_ctx *ctx, hb_keys *keys, int gates_per_cta, const hb::GateJob *djobs, int njobs,
               uint32_t batches, cudaStream_t stream);
int launch_gates_per_cta(const hb_ctx *ctx, const hb_keys *keys, uint64_t gates);
// The job record of `count` single-bootstrap gates (NAND..MAJORITY) of parameter set p.
int gate_job(const hb_params &p, int gate, const void *c0, const void *c1, const void *c2, void *out,
             uint32_t count, hb::GateJob *job);
}  // namespace hbrt
