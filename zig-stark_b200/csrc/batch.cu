// Batched and served proving.
//
// A proof is a chain of device phases separated by host transcript steps (every
// commitment root is absorbed before the next challenge). One proof therefore
// leaves the GPU idle between its small kernels and during its host round trips.
// Proving many traces at once fills those gaps: each worker thread owns a CUDA
// stream and its own transcript, takes the next job from a shared queue, and the
// device interleaves the kernels of all workers' proofs. Admission is bounded by
// an estimate of each proof's HBM footprint so the stream of requests never
// overcommits device memory; a job waits until enough of the budget is free.
//
// Every proof is computed by the same stark_prove as a single call, so each result
// is byte-identical to proving that trace alone.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/zs_m31.h"
#include "airs.cuh"
#include "host.cuh"
#include "stark.cuh"
#include "staging.cuh"

namespace zs {

namespace {

// Device bytes a proof of this shape holds at its peak: codewords, coefficients and
// values (16 B per element) of every committed column -- preprocessed, main and one
// LogUp accumulator per relation, counted from the AIR itself -- one Merkle tree per
// committed column plus the quotient and FRI layers (64 B per leaf), NTT tables and
// temporaries.
uint64_t estimate_footprint(const zs_m31_job& j) {
  if (!j.params || j.params_len < 2) return 64u << 20;  // malformed: the job fails on its own status
  const unsigned tl = j.params[0], lb = j.params[1];
  if (tl + lb > 40) return 64u << 20;
  const uint64_t n = (uint64_t)1 << tl, N = (uint64_t)1 << (tl + lb);
  uint64_t c = 0;
  try {
    const AirInfo air = make_air(j.air_id, j.public_inputs, j.public_inputs_len);
    c = (uint64_t)air.m + air.n_rel + air.n_pre;
  } catch (...) {
    // unknown AIR or malformed public inputs: the job fails on its own status; size it
    // from the column headers of its buffers
    uint64_t cols = 0, pcols = 0;
    if (j.trace_len >= 8) std::memcpy(&cols, j.trace, 8);
    if (j.preprocessed_len >= 8) std::memcpy(&pcols, j.preprocessed, 8);
    c = std::min<uint64_t>(cols + pcols + 1, 1u << 10);
  }
  return c * (N * 16 + 2 * n * 16) + (c + 2) * N * 64 + N * 16 * 3 + (64u << 20);
}

struct HbmBudget {
  std::mutex mu;
  std::condition_variable cv;
  uint64_t limit, used = 0;
  explicit HbmBudget(uint64_t l) : limit(l) {}
  void acquire(uint64_t b) {
    std::unique_lock<std::mutex> lk(mu);
    // a job larger than the whole budget runs alone rather than never
    cv.wait(lk, [&] { return used == 0 || used + b <= limit; });
    used += b;
  }
  void release(uint64_t b) {
    {
      std::lock_guard<std::mutex> lk(mu);
      used -= b;
    }
    cv.notify_all();
  }
};

// The footprint estimates leave some slack for the pool's fragmentation.
uint64_t default_budget() {
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return (uint64_t)8 << 30;
  return (uint64_t)(free_b * 0.7);
}

// A job's arguments. Batch jobs point into the caller's buffers, which outlive the
// call; a server copies each request's buffers into one allocation of its own.
struct Job {
  zs_m31_job v{};
  std::unique_ptr<uint8_t[]> owned;
  uint64_t footprint = 0;
};

Job view_job(const zs_m31_job& j) {
  Job o;
  o.v = j;
  return o;
}

Job copy_job(const zs_m31_job& j) {
  Job o;
  o.v = j;
  const size_t total = j.params_len + j.public_inputs_len + j.preprocessed_len + j.trace_len + j.channel_sep_len;
  o.owned.reset(new uint8_t[total ? total : 1]);  // not value-initialized: filled by the copies below
  uint8_t* p = o.owned.get();
  auto cp = [&](const uint8_t* src, size_t n) -> const uint8_t* {
    if (n == 0) return nullptr;
    host_copy(p, src, n);
    const uint8_t* r = p;
    p += n;
    return r;
  };
  o.v.params = cp(j.params, j.params_len);
  o.v.public_inputs = cp(j.public_inputs, j.public_inputs_len);
  o.v.preprocessed = cp(j.preprocessed, j.preprocessed_len);
  o.v.trace = cp(j.trace, j.trace_len);
  o.v.channel_sep = cp(j.channel_sep, j.channel_sep_len);
  return o;
}

int32_t run_job(const Job& j, cudaStream_t st, std::vector<uint8_t>& out) {
  const zs_m31_job& v = j.v;
  try {
    out = stark_prove(v.air_id, v.params, v.params_len, v.public_inputs, v.public_inputs_len, v.preprocessed,
                      v.preprocessed_len, v.trace, v.trace_len, v.channel_sep, v.channel_sep_len, st);
    return ZS_OK;
  } catch (const Error& e) {
    cudaStreamSynchronize(st);
    return e.code;
  } catch (const std::bad_alloc&) {
    cudaStreamSynchronize(st);
    return ZS_ENOMEM;
  } catch (...) {
    cudaStreamSynchronize(st);
    return ZS_EGENERIC;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Server: continuous batching over a request queue
// ---------------------------------------------------------------------------

struct Server {
  struct Entry {
    Job job;
    int32_t status = 1;  // 1 = pending
    std::vector<uint8_t> proof;
    std::chrono::steady_clock::time_point t_submit, t_start, t_done;
  };
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Entry>> entries;
  uint64_t next_ticket = 1;
  bool stopping = false;
  HbmBudget budget;
  int device = 0;
  std::vector<std::thread> workers;

  Server(uint32_t n_workers, uint64_t hbm_budget) : budget(hbm_budget ? hbm_budget : default_budget()) {
    ZS_CUDA(cudaGetDevice(&device));
    if (n_workers == 0) n_workers = 1;
    for (uint32_t w = 0; w < n_workers; ++w) workers.emplace_back([this] { loop(); });
  }
  ~Server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stopping = true;
    }
    cv_work.notify_all();
    for (auto& t : workers) t.join();
  }

  // Each worker proves on its own stream.
  // Each worker proves on its own streams: proofs with a footprint of at least
  // kLargeProof bytes on a high-priority stream, so a long proof is not stretched by
  // the many short ones sharing the device with it (their blocks fill its gaps).
  static constexpr uint64_t kLargeProof = (uint64_t)1 << 30;
  void loop() {
    cudaSetDevice(device);
    int lo_prio = 0, hi_prio = 0;
    cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
    cudaStream_t st_lo = nullptr, st_hi = nullptr;
    cudaStreamCreateWithPriority(&st_lo, cudaStreamNonBlocking, lo_prio);
    cudaStreamCreateWithPriority(&st_hi, cudaStreamNonBlocking, hi_prio);
    for (;;) {
      uint64_t ticket;
      Entry* e;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stopping || !queue.empty(); });
        if (queue.empty()) break;
        ticket = queue.front();
        queue.pop_front();
        e = entries.at(ticket).get();
      }
      budget.acquire(e->job.footprint);
      e->t_start = std::chrono::steady_clock::now();
      std::vector<uint8_t> out;
      const int32_t rc = run_job(e->job, e->job.footprint >= kLargeProof ? st_hi : st_lo, out);
      budget.release(e->job.footprint);
      {
        std::lock_guard<std::mutex> lk(mu);
        e->proof = std::move(out);
        e->t_done = std::chrono::steady_clock::now();
        e->status = rc;
        e->job = Job();  // inputs are no longer needed
      }
      cv_done.notify_all();
    }
    cudaStreamDestroy(st_lo);
    cudaStreamDestroy(st_hi);
  }

  // Queues a job; `copy` makes the server's own copy of the caller's buffers.
  uint64_t submit(const zs_m31_job& j, bool copy) {
    const auto t_submit = std::chrono::steady_clock::now();  // a request's latency includes taking its copy
    Job job = copy ? copy_job(j) : view_job(j);
    job.footprint = estimate_footprint(j);
    auto e = std::make_unique<Entry>();
    e->job = std::move(job);
    e->t_submit = t_submit;
    uint64_t t;
    {
      std::lock_guard<std::mutex> lk(mu);
      t = next_ticket++;
      entries[t] = std::move(e);
      queue.push_back(t);
    }
    cv_work.notify_one();
    return t;
  }
};

}  // namespace zs

using namespace zs;

struct zs_m31_server {
  std::unique_ptr<Server> s;
};

namespace {
template <typename F>
int32_t guarded_b(F&& f) {
  try {
    f();
    return ZS_OK;
  } catch (const Error& e) {
    return e.code;
  } catch (const std::bad_alloc&) {
    return ZS_ENOMEM;
  } catch (...) {
    return ZS_EGENERIC;
  }
}
void check_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw Error(ZS_EDEVICE, "no CUDA device");
}
}  // namespace

extern "C" {

int32_t zs_m31_prove_batch(zs_host_allocator host, size_t n_jobs, const zs_m31_job* jobs, uint32_t concurrency,
                           uint64_t hbm_budget_bytes, zs_m31_result* results) {
  return guarded_b([&] {
    if ((n_jobs && (!jobs || !results)) || !host.alloc) throw Error(ZS_EMALFORMED, "null argument");
    check_device();
    for (size_t i = 0; i < n_jobs; ++i) results[i] = zs_m31_result{nullptr, 0, 1};
    if (n_jobs == 0) return;
    Server srv(concurrency, hbm_budget_bytes);
    // largest proofs first, so the long ones overlap with the many short ones
    std::vector<uint64_t> fp(n_jobs);
    for (size_t i = 0; i < n_jobs; ++i)
      fp[i] = estimate_footprint(jobs[i]);
    std::vector<size_t> order(n_jobs);
    for (size_t i = 0; i < n_jobs; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return fp[a] > fp[b]; });
    std::vector<uint64_t> tickets(n_jobs);
    for (size_t i : order) tickets[i] = srv.submit(jobs[i], false);  // the caller's buffers outlive the call
    for (size_t i = 0; i < n_jobs; ++i) {
      std::unique_lock<std::mutex> lk(srv.mu);
      Server::Entry* e = srv.entries.at(tickets[i]).get();
      srv.cv_done.wait(lk, [&] { return e->status != 1; });
      results[i].status = e->status;
      if (e->status == ZS_OK) {
        uint8_t* buf = (uint8_t*)host.alloc(host.ctx, e->proof.size() ? e->proof.size() : 1);
        if (!buf) {
          results[i].status = ZS_ENOMEM;
          continue;
        }
        std::memcpy(buf, e->proof.data(), e->proof.size());
        results[i].proof = buf;
        results[i].len = e->proof.size();
      }
      e->proof.clear();
      e->proof.shrink_to_fit();
    }
  });
}

int32_t zs_m31_server_create(uint32_t workers, uint64_t hbm_budget_bytes, zs_m31_server** out) {
  return guarded_b([&] {
    if (!out) throw Error(ZS_EMALFORMED, "null out");
    check_device();
    auto s = std::make_unique<zs_m31_server>();
    s->s = std::make_unique<Server>(workers, hbm_budget_bytes);
    *out = s.release();
  });
}

void zs_m31_server_destroy(zs_m31_server* server) { delete server; }

int32_t zs_m31_server_submit(zs_m31_server* server, const zs_m31_job* job, uint64_t* ticket) {
  return guarded_b([&] {
    if (!server || !job || !ticket) throw Error(ZS_EMALFORMED, "null argument");
    *ticket = server->s->submit(*job, true);
  });
}

int32_t zs_m31_server_poll(zs_m31_server* server, uint64_t ticket, int32_t wait, zs_host_allocator host,
                           zs_m31_result* result, double* latency_ms) {
  return guarded_b([&] {
    if (!server || !result) throw Error(ZS_EMALFORMED, "null argument");
    Server& s = *server->s;
    std::unique_lock<std::mutex> lk(s.mu);
    auto it = s.entries.find(ticket);
    if (it == s.entries.end()) throw Error(ZS_EMALFORMED, "unknown ticket");
    Server::Entry* e = it->second.get();
    if (wait) s.cv_done.wait(lk, [&] { return e->status != 1; });
    *result = zs_m31_result{nullptr, 0, e->status};
    if (e->status == 1) return;
    if (latency_ms)
      *latency_ms = std::chrono::duration<double, std::milli>(e->t_done - e->t_submit).count();
    if (e->status == ZS_OK) {
      if (!host.alloc) throw Error(ZS_EMALFORMED, "null allocator");
      uint8_t* buf = (uint8_t*)host.alloc(host.ctx, e->proof.size() ? e->proof.size() : 1);
      if (!buf) throw Error(ZS_ENOMEM, "host allocator returned null");
      std::memcpy(buf, e->proof.data(), e->proof.size());
      result->proof = buf;
      result->len = e->proof.size();
    }
    s.entries.erase(it);
  });
}

}  // extern "C"
