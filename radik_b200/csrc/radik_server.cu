// radik_server.cu -- continuous-batching top-k request loop (C ABI in
// include/radik_b200.h, radik_server_*).
//
// Requests (one row each: device values, n, k, dtype, flags, device output
// buffers) are queued by any host thread.  A worker thread admits queued
// requests into batches while a batch slot is free and the in-flight bytes
// stay under the memory budget, launches each batch as ONE radik_topk_rows
// call (rows addressed in place: the batch's base is its lowest value
// pointer, each row an element offset from it), scatters the results to the
// requests' own buffers with one small kernel, and retires the batch when its
// event completes.  Requests that arrive while batches run join the next
// batch; several slots on their own streams keep batches in flight at once.
//
// SMs are the third resource a batch is admitted by, beside its slot and the
// memory budget: the engine runs one CTA per SM, so a batch asks for one CTA
// per 2^16 keys (at least 32 on an idle device) and at most three quarters
// of the device when several slots exist, and starts only when that many SMs
// are free of other batches.  The
// engines of concurrent batches therefore sit on disjoint SMs and run side by
// side: a batch of small requests does not wait for a large one to finish.
//
// Per-request mode (radik_server_config::mode = 1) is the plain baseline: one
// radik_topk launch per request, in arrival order on one stream.
//
// RadiK has no serving layer; its callers launch one topKRadixSelectL per
// request batch they form themselves (radik/RadixSelect/topk_radixselect.h).

#include "radik_common.cuh"
#include "radik_b200.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstddef>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace radik {
namespace {

double now_us() {
  using namespace std::chrono;
  return duration<double, std::micro>(steady_clock::now().time_since_epoch()).count();
}

struct Req {
  uint64_t id;
  int dtype;
  uint32_t flags;
  const void* val;
  int n, k;
  void* vout;
  void* iout;
  double t_arrival;  // microseconds, steady clock
};

struct ScatterDesc {
  int64_t src;  // first output slot in the batch's output region
  void* vdst;
  void* idst;
  int32_t k;
  int32_t pad;
};

// One block per request: copies its k values and indices from the batch's
// output region to the request's own buffers.
__global__ void scatter_kernel(const ScatterDesc* d, const uint8_t* vsrc, const uint8_t* isrc, int es, int is) {
  const ScatterDesc s = d[blockIdx.x];
  const int64_t vb = (int64_t)s.k * es, ib = (int64_t)s.k * is;
  const uint8_t* v = vsrc + s.src * es;
  const uint8_t* ix = isrc + s.src * is;
  for (int64_t j = threadIdx.x; j < vb; j += blockDim.x) static_cast<uint8_t*>(s.vdst)[j] = v[j];
  for (int64_t j = threadIdx.x; j < ib; j += blockDim.x) static_cast<uint8_t*>(s.idst)[j] = ix[j];
}

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  void* ws = nullptr;
  size_t ws_bytes = 0;
  uint8_t* vout = nullptr;
  uint8_t* iout = nullptr;
  radik_row_desc* desc_h = nullptr;  // pinned
  radik_row_desc* desc_d = nullptr;
  ScatterDesc* sc_h = nullptr;  // pinned
  ScatterDesc* sc_d = nullptr;
  int32_t* status_h = nullptr;  // pinned copy of the call's device status word
  std::vector<Req> reqs;
  size_t bytes = 0;
  int ctas = 0;  // engine CTAs (SMs) the batch holds
  bool busy = false;
};

// Keys per engine CTA a batch asks for.  At 2^16 fp32 keys (256 KB) a CTA
// streams its share in a few microseconds, about the engine's fixed cost.
// A batch that finds no other batch in flight takes at least kIdleBatchCtas:
// a row of 128K keys on two CTAs streams for longer than the engine's fixed
// cost.  Under load it takes only its share, so that small batches never
// hold the SMs a large one is waiting for (a floor of 16 CTAs for every batch
// raised p99 at 50k requests/s from 0.50 to 1.49 ms).
constexpr int64_t kKeysPerCta = (int64_t)1 << 16;
constexpr int kIdleBatchCtas = 32;

}  // namespace

struct Server {
  radik_server_config cfg{};
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Req> pending;
  std::vector<radik_completion> completed;
  std::atomic<uint64_t> next_id{1};
  std::atomic<int64_t> outstanding{0};
  size_t inflight_bytes = 0;
  int ctas_total = 0;     // engine CTAs the device runs at once (one per SM)
  int ctas_cap = 0;       // most CTAs one batch may take
  int ctas_inflight = 0;  // CTAs held by batches in flight
  radik_server_stats stats{};
  bool stop = false;
  std::thread worker;
  std::string error;
  int first_error = RADIK_OK;

  static size_t req_bytes(const Req& r) {
    const size_t es = r.dtype == kF32 ? 4 : 2;
    const size_t is = (r.flags & kFlagIdx64) ? 8 : 4;
    return (size_t)r.n * es + (size_t)r.k * (es + is);
  }

  void complete(const Req& r, int status, double t_done) {
    radik_completion c{};
    c.id = r.id;
    c.status = status;
    c.latency_us = t_done - r.t_arrival;
    completed.push_back(c);
  }

  // Retires finished batches.  Caller holds mu.
  void retire() {
    for (Slot& s : slots) {
      if (!s.busy) continue;
      const cudaError_t q = cudaEventQuery(s.done);
      if (q == cudaErrorNotReady) continue;
      const double t = now_us();
      int st = RADIK_OK;
      if (q != cudaSuccess) {
        st = RADIK_ECUDA;
        error = std::string("radik_server: ") + cudaGetErrorString(q);
      } else if (*s.status_h & kStatusTimeout) {
        st = RADIK_ETIMEOUT;
      } else if (*s.status_h & kStatusCapacity) {
        st = RADIK_EWORKSPACE;
      } else if (*s.status_h) {
        st = RADIK_EINTERNAL;
      }
      if (st != RADIK_OK && first_error == RADIK_OK) first_error = st;
      for (const Req& r : s.reqs) complete(r, st, t);
      release(s);
    }
  }

  // Returns slot s's requests, bytes and SMs.  Caller holds mu.
  void release(Slot& s) {
    outstanding -= (int64_t)s.reqs.size();
    inflight_bytes -= s.bytes;
    ctas_inflight -= s.ctas;
    s.reqs.clear();
    s.bytes = 0;
    s.ctas = 0;
    s.busy = false;
    cv.notify_all();
  }

  // Engine CTAs a batch of `keys` keys asks for.
  int want_ctas(int64_t keys) const {
    int64_t w = (keys + kKeysPerCta - 1) / kKeysPerCta;
    if (ctas_inflight == 0) w = std::max<int64_t>(w, kIdleBatchCtas);
    return (int)std::max<int64_t>(1, std::min<int64_t>(w, ctas_cap));
  }

  // Takes one batch for slot s from the pending queue: the oldest request's
  // (dtype, flags) group, in arrival order, within the slot's row, key and
  // output limits, the memory budget and the free SMs; reserves the slot and
  // the batch's SMs.  Caller holds mu.
  bool form(Slot& s) {
    if (pending.empty()) return false;
    const int dtype = pending.front().dtype;
    const uint32_t flags = pending.front().flags;
    const int free_ctas = ctas_total - ctas_inflight;
    int64_t keys = 0, outs = 0;
    size_t bytes = 0;
    s.reqs.clear();
    for (auto it = pending.begin(); it != pending.end();) {
      if ((int)s.reqs.size() >= cfg.max_batch_rows) break;
      if (it->dtype != dtype || it->flags != flags) {
        ++it;
        continue;
      }
      const size_t b = req_bytes(*it);
      if (s.reqs.empty()) {
        if (inflight_bytes > 0 && inflight_bytes + b > cfg.budget_bytes) return false;  // wait for memory
        if (want_ctas(it->n) > free_ctas) return false;                                 // wait for SMs
      } else if (keys + it->n > cfg.max_batch_keys || outs + it->k > (int64_t)cfg.max_batch_rows * cfg.max_k ||
                 inflight_bytes + bytes + b > cfg.budget_bytes || want_ctas(keys + it->n) > free_ctas) {
        break;
      }
      s.reqs.push_back(*it);
      keys += it->n;
      outs += it->k;
      bytes += b;
      it = pending.erase(it);
    }
    if (s.reqs.empty()) return false;
    s.bytes = bytes;
    s.ctas = want_ctas(keys);
    s.busy = true;
    inflight_bytes += bytes;
    ctas_inflight += s.ctas;
    return true;
  }

  // Launches slot s's batch (no lock held): descriptors, one radik_topk_rows,
  // the scatter to the requests' buffers, the status read-back, the event.
  // Per-request mode launches its single request with radik_topk instead.
  int issue(Slot& s) {
    const Req& r0 = s.reqs.front();
    const int dtype = r0.dtype;
    const uint32_t flags = r0.flags;
    const int es = dtype == kF32 ? 4 : 2;
    const int is = (flags & kFlagIdx64) ? 8 : 4;
    int rc = RADIK_OK;
    cudaError_t e = cudaSuccess;
    if (cfg.mode == 1) {
      const int n = r0.n;
      rc = radik_topk(dtype, flags, r0.val, nullptr, r0.vout, r0.iout, s.ws, s.ws_bytes, &n, 1, r0.k, s.stream);
    } else {
      // rows addressed from the batch's lowest value pointer
      uintptr_t base = UINTPTR_MAX;
      int n_max = 0, k_max = 0;
      int64_t keys = 0, oo = 0;
      for (const Req& r : s.reqs) {
        base = std::min(base, reinterpret_cast<uintptr_t>(r.val));
        n_max = std::max(n_max, r.n);
        k_max = std::max(k_max, r.k);
        keys += r.n;
      }
      for (size_t i = 0; i < s.reqs.size(); ++i) {
        const Req& r = s.reqs[i];
        s.desc_h[i].in_off = (int64_t)((reinterpret_cast<uintptr_t>(r.val) - base) / (uintptr_t)es);
        s.desc_h[i].out_off = oo;
        s.desc_h[i].n = r.n;
        s.desc_h[i].k = r.k;
        s.sc_h[i].src = oo;
        s.sc_h[i].vdst = r.vout;
        s.sc_h[i].idst = r.iout;
        s.sc_h[i].k = r.k;
        oo += r.k;
      }
      const int B = (int)s.reqs.size();
      e = cudaMemcpyAsync(s.desc_d, s.desc_h, sizeof(radik_row_desc) * B, cudaMemcpyHostToDevice, s.stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(s.sc_d, s.sc_h, sizeof(ScatterDesc) * B, cudaMemcpyHostToDevice, s.stream);
      if (e != cudaSuccess) return RADIK_ECUDA;
      rc = radik_topk_rows_ctas(dtype, flags, reinterpret_cast<const void*>(base), nullptr, s.vout, s.iout, s.ws,
                                s.ws_bytes, s.desc_d, B, keys, n_max, k_max, s.ctas, s.stream);
      if (rc == RADIK_OK) {
        scatter_kernel<<<B, 128, 0, s.stream>>>(s.sc_d, s.vout, s.iout, es, is);
        e = cudaGetLastError();
      }
    }
    if (rc != RADIK_OK) return rc;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s.status_h, static_cast<uint8_t*>(s.ws) + offsetof(Header, status), sizeof(int32_t),
                          cudaMemcpyDeviceToHost, s.stream);
    if (e == cudaSuccess) e = cudaEventRecord(s.done, s.stream);
    return e == cudaSuccess ? RADIK_OK : RADIK_ECUDA;
  }

  void run() {
    cudaSetDevice(cfg.device);
    std::unique_lock<std::mutex> lock(mu);
    while (true) {
      retire();
      Slot* ready = nullptr;
      for (Slot& s : slots) {
        if (s.busy) continue;
        if (cfg.mode == 1 && &s != &slots[0]) continue;
        if (cfg.mode == 1 ? !pending.empty() : true) {
          if (cfg.mode == 1) {
            s.reqs.assign(1, pending.front());
            pending.pop_front();
            s.bytes = req_bytes(s.reqs[0]);
            s.ctas = ctas_total;
            s.busy = true;
            inflight_bytes += s.bytes;
            ctas_inflight += s.ctas;
            ready = &s;
          } else if (form(s)) {
            ready = &s;
          }
        }
        if (ready) break;
      }
      if (ready) {
        int others = 0;
        for (const Slot& o : slots) others += (o.busy && &o != ready) ? 1 : 0;
        ++stats.batches;
        stats.requests += (int64_t)ready->reqs.size();
        if (others > 0) ++stats.batches_beside_others;
        stats.max_batches_in_flight = std::max(stats.max_batches_in_flight, others + 1);
        stats.max_ctas_in_flight = std::max(stats.max_ctas_in_flight, ctas_inflight);
        lock.unlock();
        const int rc = issue(*ready);
        lock.lock();
        if (rc != RADIK_OK) {
          if (first_error == RADIK_OK) first_error = rc;
          error = std::string("radik_server: launch failed: ") + radik_last_error();
          const double t = now_us();
          for (const Req& r : ready->reqs) complete(r, rc, t);
          release(*ready);
        }
        continue;
      }
      bool busy = false;
      for (const Slot& s : slots) busy = busy || s.busy;
      if (stop && pending.empty() && !busy) break;
      if (busy) {
        // poll the in-flight batches; release the lock so submitters proceed
        lock.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(2));
        lock.lock();
      } else {
        cv.wait_for(lock, std::chrono::microseconds(200), [&] { return stop || !pending.empty(); });
      }
    }
  }
};

}  // namespace radik

using namespace radik;

extern "C" {

struct radik_server {
  Server s;
};

int radik_server_create(const radik_server_config* cfg_in, radik_server** out) {
  if (!cfg_in || !out) return RADIK_EINVAL;
  *out = nullptr;
  radik_server_config cfg = *cfg_in;
  if (cfg.mode != 0 && cfg.mode != 1) return RADIK_EINVAL;
  if (cfg.slots <= 0) cfg.slots = 3;
  if (cfg.max_batch_rows <= 0) cfg.max_batch_rows = 512;
  if (cfg.max_batch_keys <= 0) cfg.max_batch_keys = (int64_t)1 << 27;
  if (cfg.max_n <= 0) cfg.max_n = 1 << 24;
  if (cfg.max_k <= 0) cfg.max_k = 2048;
  if (cfg.budget_bytes == 0) cfg.budget_bytes = (size_t)40 << 30;
  if (cfg.mode == 1) cfg.slots = 1;
  if (cfg.max_n > cfg.max_batch_keys) cfg.max_batch_keys = cfg.max_n;
  cudaError_t e = cudaSetDevice(cfg.device);
  if (e != cudaSuccess) return RADIK_ECUDA;
  int ctas = 0;
  if (radik_engine_ctas(&ctas) != RADIK_OK || ctas <= 0) return RADIK_ECUDA;
  auto* h = new radik_server();
  Server& S = h->s;
  S.cfg = cfg;
  S.ctas_total = ctas;
  S.ctas_cap = cfg.slots > 1 ? std::max(1, ctas * 3 / 4) : ctas;
  S.slots.resize(cfg.slots);
  const uint32_t all = kFlagSorted | kFlagLargest | kFlagIdx64;
  for (Slot& sl : S.slots) {
    size_t ws = 0;
    int rc = cfg.mode == 0 ? radik_get_workspace_size_rows(kF32, all, cfg.max_batch_rows, cfg.max_batch_keys,
                                                           cfg.max_n, cfg.max_k, &ws)
                           : radik_get_workspace_size(kF32, all, cfg.max_k, cfg.max_n, 1, &ws);
    if (rc != RADIK_OK) {
      radik_server_destroy(h);
      return rc;
    }
    sl.ws_bytes = ws;
    const size_t outs = (size_t)cfg.max_batch_rows * cfg.max_k;
    bool ok = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) == cudaSuccess &&
              cudaMalloc(&sl.ws, ws) == cudaSuccess && cudaMalloc((void**)&sl.vout, outs * 4) == cudaSuccess &&
              cudaMalloc((void**)&sl.iout, outs * 8) == cudaSuccess &&
              cudaMalloc((void**)&sl.desc_d, sizeof(radik_row_desc) * cfg.max_batch_rows) == cudaSuccess &&
              cudaMalloc((void**)&sl.sc_d, sizeof(ScatterDesc) * cfg.max_batch_rows) == cudaSuccess &&
              cudaMallocHost((void**)&sl.desc_h, sizeof(radik_row_desc) * cfg.max_batch_rows) == cudaSuccess &&
              cudaMallocHost((void**)&sl.sc_h, sizeof(ScatterDesc) * cfg.max_batch_rows) == cudaSuccess &&
              cudaMallocHost((void**)&sl.status_h, sizeof(int32_t)) == cudaSuccess;
    if (!ok) {
      radik_server_destroy(h);
      return RADIK_ECUDA;
    }
  }
  S.worker = std::thread([&S] { S.run(); });
  *out = h;
  return RADIK_OK;
}

int radik_server_submit(radik_server* h, int dtype, uint32_t flags, const void* values, int n, int k, void* val_out,
                        void* idx_out, uint64_t* id) {
  if (!h || !values || !val_out || !idx_out) return RADIK_EINVAL;
  Server& S = h->s;
  if (dtype != kF32 && dtype != kF16 && dtype != kBF16) return RADIK_EINVAL;
  if (flags & (kFlagWithIdxIn | kFlagWithScale)) return RADIK_ENOTSUP;
  if (n <= 0 || k <= 0 || n > S.cfg.max_n || k > S.cfg.max_k) return RADIK_EINVAL;
  Req r{};
  r.id = S.next_id++;
  r.dtype = dtype;
  r.flags = flags;
  r.val = values;
  r.n = n;
  r.k = k;
  r.vout = val_out;
  r.iout = idx_out;
  r.t_arrival = now_us();
  {
    std::lock_guard<std::mutex> lock(S.mu);
    S.pending.push_back(r);
    ++S.outstanding;
  }
  S.cv.notify_all();
  if (id) *id = r.id;
  return RADIK_OK;
}

int radik_server_poll(radik_server* h, radik_completion* out, int max, int* count) {
  if (!h || !count) return RADIK_EINVAL;
  Server& S = h->s;
  std::lock_guard<std::mutex> lock(S.mu);
  const int c = std::min<int>(max, (int)S.completed.size());
  if (out && c > 0) std::copy(S.completed.begin(), S.completed.begin() + c, out);
  S.completed.erase(S.completed.begin(), S.completed.begin() + c);
  *count = c;
  return RADIK_OK;
}

int radik_server_get_stats(radik_server* h, radik_server_stats* out) {
  if (!h || !out) return RADIK_EINVAL;
  Server& S = h->s;
  std::lock_guard<std::mutex> lock(S.mu);
  *out = S.stats;
  out->ctas_total = S.ctas_total;
  out->ctas_cap = S.ctas_cap;
  return RADIK_OK;
}

int radik_server_drain(radik_server* h) {
  if (!h) return RADIK_EINVAL;
  Server& S = h->s;
  std::unique_lock<std::mutex> lock(S.mu);
  S.cv.wait(lock, [&] { return S.outstanding.load() == 0; });
  return S.first_error;
}

int radik_server_run_trace(radik_server* h, const radik_trace_item* items, int count, double* latency_us) {
  if (!h || (!items && count > 0)) return RADIK_EINVAL;
  Server& S = h->s;
  std::vector<uint64_t> ids(count);
  const double t0 = now_us();
  for (int i = 0; i < count; ++i) {
    const radik_trace_item& it = items[i];
    const double due = t0 + it.arrival_us;
    // sleep through long gaps, then spin the last stretch for an exact arrival
    const double early = due - now_us() - 150.0;
    if (early > 0) std::this_thread::sleep_for(std::chrono::microseconds((int64_t)early));
    while (now_us() < due) {
    }
    const int rc = radik_server_submit(h, it.dtype, it.flags, it.values, it.n, it.k, it.val_out, it.idx_out, &ids[i]);
    if (rc != RADIK_OK) return rc;
  }
  const int rc = radik_server_drain(h);
  if (latency_us && count > 0) {
    // Take this trace's completions (ids are consecutive from ids[0], as no
    // other thread submits meanwhile); completions of requests submitted
    // before the trace stay queued for radik_server_poll.
    std::lock_guard<std::mutex> lock(S.mu);
    size_t w = 0;
    for (size_t r = 0; r < S.completed.size(); ++r) {
      const radik_completion& c = S.completed[r];
      const uint64_t j = c.id - ids[0];
      if (c.id >= ids[0] && j < (uint64_t)count) latency_us[j] = c.latency_us;
      else S.completed[w++] = c;
    }
    S.completed.resize(w);
  }
  return rc;
}

int radik_server_destroy(radik_server* h) {
  if (!h) return RADIK_EINVAL;
  Server& S = h->s;
  if (S.worker.joinable()) {
    {
      std::lock_guard<std::mutex> lock(S.mu);
      S.stop = true;
    }
    S.cv.notify_all();
    S.worker.join();
  }
  for (Slot& sl : S.slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    cudaFree(sl.ws);
    cudaFree(sl.vout);
    cudaFree(sl.iout);
    cudaFree(sl.desc_d);
    cudaFree(sl.sc_d);
    cudaFreeHost(sl.desc_h);
    cudaFreeHost(sl.sc_h);
    cudaFreeHost(sl.status_h);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
  }
  delete h;
  return RADIK_OK;
}

}  // extern "C"
