// hb_serve.cu -- request loop with continuous batching over the persistent bootstrapping kernel.
//
// Clients submit bootstrap requests (1..2^32-1 gates of one key set, host input buffers) from any
// thread. One worker thread per server:
//  1. admits queued requests in FIFO order while the HBM budget allows (stream-ordered
//     cudaMallocAsync for inputs + output, inputs copied to the device on the upload stream);
//  2. packs every admitted, not-yet-running request into a wave: one job table and one persistent
//     launch per key set, each on its own stream, joined by a wave event;
//  3. keeps up to `max_inflight_waves` waves on the GPU, so a new wave's CTAs take SMs as the previous
//     wave's CTAs retire (requests that arrive while others run are admitted and overlap on device);
//  4. marks requests done when their wave's event completes. Outputs stay on the device until the
//     client fetches them (hb_serve_fetch), which also returns the request's memory to the budget.
// Optional load shedding (max_queue_s): the server keeps the predicted seconds of work ahead of a
// new request (sum of count / calibrated gates-per-second of every request not yet completed; the
// persistent kernels of different key sets share the GPU, so their times add) and refuses a
// submission that would complete later than max_queue_s from now. Without a bound the queue is
// FIFO and its latency grows without limit under overload.
// No counterpart in the reference (its Evaluator is a synchronous single-gate CPU call).

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/hb_gpu.h"
#include "hb_kernels.cuh"
#include "hb_runtime.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

enum ReqState { QUEUED = 0, ADMITTED = 1, RUNNING = 2, DONE = 3, FAILED = -1 };

struct Request {
  uint64_t id = 0;
  hb_keys *keys = nullptr;
  int gate = 0;
  uint32_t count = 0;
  const void *h_in[3] = {nullptr, nullptr, nullptr};
  int nin = 0;
  size_t lwe_bytes = 0;  // one batch of count ciphertexts
  size_t bytes = 0;      // nin inputs + 1 output
  unsigned char *d_buf = nullptr;
  int state = QUEUED;
  double t_submit = 0, t_done = 0;
  double work_s = 0;  // predicted GPU seconds (count / calibrated rate), 0 when uncalibrated
};

struct Wave {
  std::vector<Request *> reqs;
  std::vector<void *> tables;
  cudaEvent_t done = nullptr;
  int slot = 0;
  bool failed = false;  // a launch of this wave failed: its requests complete as failed
};

// Key sets per wave (one persistent launch, on its own stream, per key set): wave selection leaves
// the requests of a further set for the next wave.
constexpr int kMaxSets = 4;

}  // namespace

struct hb_server {
  hb_ctx *ctx = nullptr;
  hb_serve_config cfg{};
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_done, cv_work;
  bool stopping = false;
  std::deque<Request *> queued;
  std::vector<Request *> ready;
  std::unordered_map<uint64_t, Request *> reqs;
  std::deque<uint64_t> done_ids;
  uint64_t next_id = 1;
  size_t in_use = 0, peak = 0;
  // statistics
  uint64_t submitted = 0, admitted = 0, completed = 0, failed = 0, waves = 0, gates_done = 0, rejected = 0;
  double backlog_s = 0;  // predicted seconds of work submitted and not yet completed
  std::vector<double> latencies;
  double t_first_submit = 0, t_last_done = 0;
  // worker-owned CUDA objects
  cudaStream_t up = nullptr, fetch = nullptr;
  std::vector<cudaStream_t> set_streams;  // max_inflight * kMaxSets
  std::vector<cudaStream_t> wave_streams; // max_inflight: joins a wave's set streams
  cudaEvent_t uploaded = nullptr;
  std::deque<Wave> inflight;
  int error = HB_OK;
  std::string error_text;
};

namespace {

void fail_request(hb_server *s, Request *r) {
  r->state = FAILED;
  ++s->failed;
  s->backlog_s = std::max(0.0, s->backlog_s - r->work_s);
  s->done_ids.push_back(r->id);
}

// Admission: FIFO while the budget allows. Returns the requests whose uploads were enqueued.
std::vector<Request *> admit(hb_server *s) {
  std::vector<Request *> newly;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    while (!s->queued.empty()) {
      Request *r = s->queued.front();
      if (s->in_use + r->bytes > s->cfg.hbm_budget && s->in_use > 0) break;  // wait for memory
      s->queued.pop_front();
      s->in_use += r->bytes;
      s->peak = std::max(s->peak, s->in_use);
      newly.push_back(r);
    }
  }
  for (Request *r : newly) {
    cudaError_t e = cudaMallocAsync((void **)&r->d_buf, r->bytes, s->up);
    for (int i = 0; i < r->nin && e == cudaSuccess; ++i)
      e = cudaMemcpyAsync(r->d_buf + i * r->lwe_bytes, r->h_in[i], r->lwe_bytes, cudaMemcpyHostToDevice, s->up);
    std::lock_guard<std::mutex> lock(s->mu);
    if (e != cudaSuccess) {
      s->in_use -= r->bytes;
      if (r->d_buf) cudaFreeAsync(r->d_buf, s->up);
      r->d_buf = nullptr;
      fail_request(s, r);
      s->cv_done.notify_all();
    } else {
      r->state = ADMITTED;
      ++s->admitted;
    }
  }
  if (!newly.empty()) cudaEventRecord(s->uploaded, s->up);
  return newly;
}

int launch_wave(hb_server *s, std::vector<Request *> reqs, int slot) {
  hb_ctx *ctx = s->ctx;
  Wave w;
  w.slot = slot;
  w.reqs = reqs;
  cudaStream_t ws = s->wave_streams[slot];
  cudaStreamWaitEvent(ws, s->uploaded, 0);
  std::vector<hb_keys *> sets;
  std::vector<std::vector<hb::GateJob>> tabs;
  for (Request *r : reqs) {
    size_t k = 0;
    while (k < sets.size() && sets[k] != r->keys) ++k;
    if (k == sets.size()) {
      sets.push_back(r->keys);
      tabs.emplace_back();
    }
    hb::GateJob j;
    unsigned char *b = r->d_buf;
    hbrt::gate_job(r->keys->p, r->gate, b, r->nin > 1 ? b + r->lwe_bytes : nullptr,
                   r->nin > 2 ? b + 2 * r->lwe_bytes : nullptr, b + r->nin * r->lwe_bytes, r->count, &j);
    tabs[k].push_back(j);
  }
  if ((int)sets.size() > kMaxSets) {  // wave selection never takes more sets; fail rather than strand
    std::lock_guard<std::mutex> lock(s->mu);
    for (Request *r : reqs) fail_request(s, r);
    s->cv_done.notify_all();
    return HB_ERR_UNSUPPORTED;
  }
  cudaEvent_t fork;
  cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
  cudaEventRecord(fork, ws);
  std::vector<cudaEvent_t> joins;
  int rc = HB_OK;
  for (size_t k = 0; k < sets.size() && !rc; ++k) {
    uint64_t set_gates = 0;
    for (auto &j : tabs[k]) set_gates += j.count;
    const int G = hbrt::launch_gates_per_cta(ctx, sets[k], set_gates);
    uint32_t batches = 0;
    for (auto &j : tabs[k]) {
      j.first_batch = batches;
      batches += (j.count + G - 1) / G;
    }
    cudaStream_t st = s->set_streams[slot * kMaxSets + k];
    void *dtab = nullptr;
    cudaStreamWaitEvent(st, fork, 0);
    cudaError_t e = cudaMallocAsync(&dtab, sizeof(hb::GateJob) * tabs[k].size(), st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(dtab, tabs[k].data(), sizeof(hb::GateJob) * tabs[k].size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
      rc = HB_ERR_CUDA;
      break;
    }
    w.tables.push_back(dtab);
    rc = hbrt::launch_set(ctx, sets[k], G, (const hb::GateJob *)dtab, (int)tabs[k].size(), batches, st);
    cudaEvent_t j;
    cudaEventCreateWithFlags(&j, cudaEventDisableTiming);
    cudaEventRecord(j, st);
    cudaStreamWaitEvent(ws, j, 0);
    joins.push_back(j);
  }
  cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming);
  cudaEventRecord(w.done, ws);
  cudaEventDestroy(fork);
  for (auto j : joins) cudaEventDestroy(j);  // destruction is deferred until the event completes
  w.failed = rc != HB_OK;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    for (Request *r : reqs) r->state = RUNNING;
    ++s->waves;
  }
  s->inflight.push_back(std::move(w));
  return rc;
}

void complete_waves(hb_server *s) {
  while (!s->inflight.empty()) {
    Wave &w = s->inflight.front();
    cudaError_t q = cudaEventQuery(w.done);
    if (q == cudaErrorNotReady) break;
    const double t = now_s();
    for (void *tab : w.tables) cudaFreeAsync(tab, s->wave_streams[w.slot]);
    {
      std::lock_guard<std::mutex> lock(s->mu);
      for (Request *r : w.reqs) {
        if (q != cudaSuccess || w.failed) {
          fail_request(s, r);
          continue;
        }
        r->state = DONE;
        r->t_done = t;
        ++s->completed;
        s->backlog_s = std::max(0.0, s->backlog_s - r->work_s);
        s->gates_done += r->count;
        s->latencies.push_back(t - r->t_submit);
        s->t_last_done = t;
        s->done_ids.push_back(r->id);
      }
    }
    cudaEventDestroy(w.done);
    s->inflight.pop_front();
    s->cv_done.notify_all();
  }
}

void worker_main(hb_server *s) {
  cudaSetDevice(s->ctx->device);
  while (true) {
    {
      std::unique_lock<std::mutex> lock(s->mu);
      if (s->stopping && s->inflight.empty()) break;
      if (s->queued.empty() && s->ready.empty() && s->inflight.empty())
        s->cv_work.wait_for(lock, std::chrono::milliseconds(5));
    }
    bool stopping;
    {
      std::lock_guard<std::mutex> lock(s->mu);
      stopping = s->stopping;
    }
    bool progress = false;
    if (!stopping) {
      std::vector<Request *> newly = admit(s);
      s->ready.insert(s->ready.end(), newly.begin(), newly.end());
      progress |= !newly.empty();
    }
    const size_t before = s->inflight.size();
    complete_waves(s);
    progress |= s->inflight.size() != before;
    if (!stopping && !s->ready.empty() && (int)s->inflight.size() < (int)s->cfg.max_inflight_waves) {
      // slot: the wave stream not used by a wave in flight
      int slot = 0;
      for (; slot < (int)s->cfg.max_inflight_waves; ++slot) {
        bool used = false;
        for (auto &w : s->inflight) used |= w.slot == slot;
        if (!used) break;
      }
      std::vector<Request *> take;
      std::vector<hb_keys *> keysets;
      uint64_t gates = 0;
      size_t i = 0;
      for (; i < s->ready.size(); ++i) {
        Request *r = s->ready[i];
        if (!take.empty() && s->cfg.max_wave_gates && gates + r->count > s->cfg.max_wave_gates) break;
        if (std::find(keysets.begin(), keysets.end(), r->keys) == keysets.end()) {
          if ((int)keysets.size() == kMaxSets) break;  // the next set starts the next wave
          keysets.push_back(r->keys);
        }
        take.push_back(r);
        gates += r->count;
      }
      s->ready.erase(s->ready.begin(), s->ready.begin() + i);
      int rc = launch_wave(s, take, slot);
      if (rc) {
        std::lock_guard<std::mutex> lock(s->mu);
        s->error = rc;
        s->error_text = "wave launch failed";
      }
    } else if (!progress) {
      // waves running, or requests waiting for budget that only fetches return: poll gently
      std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
  }
  // Stopping: requests never launched are cancelled and their memory released.
  std::lock_guard<std::mutex> lock(s->mu);
  for (Request *r : s->ready) {
    if (r->d_buf) cudaFreeAsync(r->d_buf, s->up);
    r->d_buf = nullptr;
    s->in_use -= r->bytes;
    fail_request(s, r);
  }
  s->ready.clear();
  for (Request *r : s->queued) fail_request(s, r);
  s->queued.clear();
  cudaStreamSynchronize(s->up);
  s->cv_done.notify_all();
}

size_t word_bytes(const hb_params &p) { return p.field_id == HB_FIELD_GOLDILOCKS ? 8 : 4; }

}  // namespace

extern "C" {

int hb_serve_start(hb_ctx *ctx, const hb_serve_config *cfg, hb_server **out) {
  if (!ctx || !out) return HB_ERR_INVALID;
  *out = nullptr;
  cudaSetDevice(ctx->device);
  hb_server *s = new hb_server();
  s->ctx = ctx;
  s->cfg.hbm_budget = cfg && cfg->hbm_budget ? cfg->hbm_budget : (size_t)120 << 30;
  s->cfg.max_wave_gates = cfg ? cfg->max_wave_gates : 0;
  s->cfg.max_inflight_waves = cfg && cfg->max_inflight_waves ? std::min(cfg->max_inflight_waves, 4u) : 2;
  s->cfg.max_queue_s = cfg && cfg->max_queue_s > 0 ? cfg->max_queue_s : 0;
  cudaStreamCreateWithFlags(&s->up, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&s->fetch, cudaStreamNonBlocking);
  s->set_streams.resize(s->cfg.max_inflight_waves * kMaxSets);
  s->wave_streams.resize(s->cfg.max_inflight_waves);
  for (auto &st : s->set_streams) cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  for (auto &st : s->wave_streams) cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  cudaEventCreateWithFlags(&s->uploaded, cudaEventDisableTiming);
  cudaEventRecord(s->uploaded, s->up);
  // keep freed request memory in the device pool for reuse instead of returning it to the driver
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, ctx->device) == cudaSuccess) {
    uint64_t keep = s->cfg.hbm_budget;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    delete s;
    return hbrt::cuda_fail(ctx, e, "server start");
  }
  s->worker = std::thread(worker_main, s);
  *out = s;
  return HB_OK;
}

int hb_serve_submit(hb_server *s, hb_keys *keys, int gate, const void *c0, const void *c1,
                    const void *c2, uint32_t count, uint64_t *id) {
  if (!s || !keys || !c0 || count == 0 || gate < HB_GATE_NAND || gate > HB_GATE_MAJORITY) return HB_ERR_INVALID;
  if (!c1 || (gate == HB_GATE_MAJORITY && !c2)) return HB_ERR_INVALID;
  if (keys->p.ring_dim != 1024) return HB_ERR_UNSUPPORTED;
  Request *r = new Request();
  r->keys = keys;
  r->gate = gate;
  r->count = count;
  r->nin = gate == HB_GATE_MAJORITY ? 3 : 2;
  r->h_in[0] = c0;
  r->h_in[1] = c1;
  r->h_in[2] = c2;
  r->lwe_bytes = (size_t)count * (keys->p.lwe_dim + 1) * word_bytes(keys->p);
  r->bytes = (r->nin + 1) * r->lwe_bytes;
  r->t_submit = now_s();
  if (keys->gates_per_s > 0) r->work_s = count / keys->gates_per_s;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stopping) {
      delete r;
      return HB_ERR_BUSY;
    }
    if (r->bytes > s->cfg.hbm_budget) {
      delete r;
      return HB_ERR_NOMEM;
    }
    if (s->cfg.max_queue_s > 0 && r->work_s > 0 && s->backlog_s + r->work_s > s->cfg.max_queue_s) {
      ++s->rejected;
      delete r;
      if (id) *id = 0;
      return HB_ERR_BUSY;
    }
    s->backlog_s += r->work_s;
    r->id = s->next_id++;
    s->reqs[r->id] = r;
    s->queued.push_back(r);
    ++s->submitted;
    if (s->t_first_submit == 0) s->t_first_submit = r->t_submit;
    if (id) *id = r->id;
  }
  s->cv_work.notify_one();
  return HB_OK;
}

int hb_serve_poll(hb_server *s, uint64_t id, int *state) {
  if (!s || !state) return HB_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return HB_ERR_INVALID;
  *state = it->second->state;
  return HB_OK;
}

int hb_serve_next_done(hb_server *s, uint64_t *id, double timeout_s) {
  if (!s || !id) return HB_ERR_INVALID;
  std::unique_lock<std::mutex> lock(s->mu);
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
  while (s->done_ids.empty()) {
    if (s->cv_done.wait_until(lock, deadline) == std::cv_status::timeout && s->done_ids.empty())
      return HB_ERR_BUSY;  // nothing completed within the timeout
  }
  *id = s->done_ids.front();
  s->done_ids.pop_front();
  return HB_OK;
}

int hb_serve_fetch(hb_server *s, uint64_t id, void *out, double *latency_s) {
  if (!s) return HB_ERR_INVALID;
  Request *r;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return HB_ERR_INVALID;
    r = it->second;
    if (r->state != DONE && r->state != FAILED) return HB_ERR_BUSY;
    s->reqs.erase(it);
  }
  int rc = HB_OK;
  cudaSetDevice(s->ctx->device);
  if (r->state == DONE) {
    if (out) {
      cudaError_t e = cudaMemcpyAsync(out, r->d_buf + r->nin * r->lwe_bytes, r->lwe_bytes,
                                      cudaMemcpyDeviceToHost, s->fetch);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s->fetch);
      if (e != cudaSuccess) rc = HB_ERR_CUDA;
    }
    if (latency_s) *latency_s = r->t_done - r->t_submit;
  } else {
    rc = HB_ERR_CUDA;
  }
  if (r->d_buf) {
    cudaFreeAsync(r->d_buf, s->fetch);
    std::lock_guard<std::mutex> lock(s->mu);
    s->in_use -= r->bytes;
  }
  delete r;
  s->cv_work.notify_one();
  return rc;
}

int hb_serve_stats(hb_server *s, hb_serve_statistics *out) {
  if (!s || !out) return HB_ERR_INVALID;
  std::lock_guard<std::mutex> lock(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->submitted = s->submitted;
  out->admitted = s->admitted;
  out->completed = s->completed;
  out->failed = s->failed;
  out->queued = s->queued.size();
  out->waves = s->waves;
  out->gates_completed = s->gates_done;
  out->hbm_in_use = s->in_use;
  out->hbm_peak = s->peak;
  out->rejected = s->rejected;
  if (!s->latencies.empty()) {
    std::vector<double> l = s->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) { return l[std::min(l.size() - 1, (size_t)(q * (l.size() - 1) + 0.5))]; };
    out->p50_latency_s = pct(0.50);
    out->p99_latency_s = pct(0.99);
    out->max_latency_s = l.back();
    double sum = 0;
    for (double v : l) sum += v;
    out->mean_latency_s = sum / l.size();
  }
  if (s->t_last_done > s->t_first_submit && s->t_first_submit > 0)
    out->gates_per_s = s->gates_done / (s->t_last_done - s->t_first_submit);
  return s->error;
}

int hb_serve_stop(hb_server *s) {
  if (!s) return HB_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->ctx->device);
  cudaDeviceSynchronize();
  for (auto &kv : s->reqs) {
    if (kv.second->d_buf) cudaFreeAsync(kv.second->d_buf, s->fetch);
    delete kv.second;
  }
  s->reqs.clear();
  cudaStreamSynchronize(s->fetch);
  for (auto st : s->set_streams) cudaStreamDestroy(st);
  for (auto st : s->wave_streams) cudaStreamDestroy(st);
  cudaStreamDestroy(s->up);
  cudaStreamDestroy(s->fetch);
  cudaEventDestroy(s->uploaded);
  const int rc = s->error;
  delete s;
  return rc;
}

}  // extern "C"
