// Pinned, double-buffered, multi-threaded host staging for uploads.
#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "staging.cuh"

namespace zs {

namespace {

constexpr size_t kChunk = (size_t)16 << 20;  // bytes per staging buffer
constexpr size_t kSmall = (size_t)1 << 20;   // below this the driver's pageable path is as fast

thread_local bool t_upload_high = false;

// A fork-join pool of host threads: run(n, f) calls f(0..n-1) spread over the pool
// and the caller, and returns when every call has finished. A caller that finds the
// pool busy runs its calls itself, unless its uploads have priority: then it waits
// for the pool.
class HostPool {
 public:
  static HostPool& get() {
    static HostPool pool;
    return pool;
  }
  size_t width() const { return threads_.size() + 1; }
  void run(size_t n, const std::function<void(size_t)>& f) {
    std::unique_lock<std::mutex> call(call_mu_, std::defer_lock);
    if (t_upload_high)
      call.lock();
    else
      (void)call.try_lock();
    if (!call.owns_lock()) {  // the pool serves another caller: copy on this thread
      for (size_t i = 0; i < n; ++i) f(i);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      task_ = &f;
      n_ = n;
      next_ = 0;
      busy_ = threads_.size();
      ++gen_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return busy_ == 0; });
    task_ = nullptr;
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }

 private:
  HostPool() {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned extra = std::min(7u, std::max(1u, hw / 2) - 1);  // up to half the cores
    for (unsigned i = 0; i < extra; ++i) threads_.emplace_back([this] { loop(); });
  }
  void work() {
    for (;;) {
      size_t i;
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (!task_ || next_ >= n_) return;
        i = next_++;
      }
      (*task_)(i);
    }
  }
  void loop() {
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
      }
      work();
      {
        std::lock_guard<std::mutex> lk(mu_);
        --busy_;
      }
      done_cv_.notify_all();
    }
  }
  std::vector<std::thread> threads_;
  std::mutex call_mu_, mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(size_t)>* task_ = nullptr;
  size_t n_ = 0, next_ = 0, busy_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

// Two pinned upload buffers, each guarded by the event of the DMA that last read it.
struct Stager {
  void* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  uint64_t next = 0;  // alternates across calls too
  bool ok = false;
  Stager() {
    ok = cudaHostAlloc(&buf[0], kChunk, cudaHostAllocDefault) == cudaSuccess &&
         cudaHostAlloc(&buf[1], kChunk, cudaHostAllocDefault) == cudaSuccess &&
         cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) == cudaSuccess &&
         cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) == cudaSuccess;
  }
};

// Bump-allocated pinned blocks; a region stays valid until the next reset.
struct Arena {
  std::vector<std::pair<uint8_t*, size_t>> blocks;  // (base, capacity)
  size_t cur = 0, used = 0;
  void reset() {
    cur = 0;
    used = 0;
  }
  uint8_t* take(size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    while (cur < blocks.size() && used + bytes > blocks[cur].second) ++cur, used = 0;
    if (cur == blocks.size()) {
      size_t cap = blocks.empty() ? ((size_t)1 << 20) : blocks.back().second * 2;
      while (cap < bytes) cap *= 2;
      void* p = nullptr;
      ZS_CUDA(cudaHostAlloc(&p, cap, cudaHostAllocDefault));
      blocks.emplace_back(static_cast<uint8_t*>(p), cap);
      used = 0;
    }
    uint8_t* r = blocks[cur].first + used;
    used += bytes;
    return r;
  }
};

struct Slot {
  Stager stager;
  Arena arena;
};

// Slots are created on demand and kept for the life of the process.
class SlotBank {
 public:
  static SlotBank& get() {
    static SlotBank* bank = new SlotBank();
    return *bank;
  }
  Slot* take() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (!idle_.empty()) {
        Slot* s = idle_.back();
        idle_.pop_back();
        return s;
      }
    }
    return new Slot();
  }
  void give(Slot* s) {
    std::lock_guard<std::mutex> lk(mu_);
    idle_.push_back(s);
  }

 private:
  std::mutex mu_;
  std::vector<Slot*> idle_;
};

thread_local Slot* t_slot = nullptr;

}  // namespace

UploadPriority::UploadPriority(bool high) : prev_(t_upload_high) { t_upload_high = high; }
UploadPriority::~UploadPriority() { t_upload_high = prev_; }

PinnedScope::PinnedScope(cudaStream_t st) : st_(st), slot_(SlotBank::get().take()), prev_(t_slot) {
  Slot* s = static_cast<Slot*>(slot_);
  s->arena.reset();
  t_slot = s;
}

PinnedScope::~PinnedScope() {
  cudaStreamSynchronize(st_);
  t_slot = static_cast<Slot*>(prev_);
  SlotBank::get().give(static_cast<Slot*>(slot_));
}

void h2d_small(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return;
  if (!t_slot) {
    ZS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return;
  }
  uint8_t* r = t_slot->arena.take(bytes);
  std::memcpy(r, src, bytes);
  ZS_CUDA(cudaMemcpyAsync(dst, r, bytes, cudaMemcpyHostToDevice, st));
}

void d2h_small(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return;
  if (!t_slot) {
    ZS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    ZS_CUDA(cudaStreamSynchronize(st));
    return;
  }
  uint8_t* r = t_slot->arena.take(bytes);
  ZS_CUDA(cudaMemcpyAsync(r, src, bytes, cudaMemcpyDeviceToHost, st));
  ZS_CUDA(cudaStreamSynchronize(st));
  std::memcpy(dst, r, bytes);
}

void d2h_many(const D2H* c, size_t count, cudaStream_t st) {
  if (count == 0) return;
  if (!t_slot) {
    for (size_t k = 0; k < count; ++k)
      if (c[k].bytes) ZS_CUDA(cudaMemcpyAsync(c[k].dst, c[k].src, c[k].bytes, cudaMemcpyDeviceToHost, st));
    ZS_CUDA(cudaStreamSynchronize(st));
    return;
  }
  std::vector<uint8_t*> r(count);
  for (size_t k = 0; k < count; ++k) {
    if (!c[k].bytes) continue;
    r[k] = t_slot->arena.take(c[k].bytes);
    ZS_CUDA(cudaMemcpyAsync(r[k], c[k].src, c[k].bytes, cudaMemcpyDeviceToHost, st));
  }
  ZS_CUDA(cudaStreamSynchronize(st));
  for (size_t k = 0; k < count; ++k)
    if (c[k].bytes) std::memcpy(c[k].dst, r[k], c[k].bytes);
}

void host_copy(void* dst, const void* src, size_t bytes) {
  constexpr size_t kPart = (size_t)8 << 20;  // bytes per pool task
  if (bytes < 2 * kPart) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t parts = (bytes + kPart - 1) / kPart;
  HostPool::get().run(parts, [&](size_t i) {
    const size_t off = i * kPart;
    std::memcpy(static_cast<uint8_t*>(dst) + off, static_cast<const uint8_t*>(src) + off,
                std::min(kPart, bytes - off));
  });
}

void upload_bytes(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return;
  Stager* sg = (bytes < kSmall || !t_slot) ? nullptr : &t_slot->stager;
  if (!sg || !sg->ok) {
    ZS_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return;
  }
  HostPool& pool = HostPool::get();
  const size_t parts = pool.width();
  const uint8_t* s = static_cast<const uint8_t*>(src);
  uint8_t* d = static_cast<uint8_t*>(dst);
  for (size_t off = 0; off < bytes; off += kChunk) {
    const size_t len = std::min(kChunk, bytes - off);
    const int b = (int)(sg->next++ & 1);
    ZS_CUDA(cudaEventSynchronize(sg->ev[b]));  // the DMA that last read this buffer is done
    uint8_t* pin = static_cast<uint8_t*>(sg->buf[b]);
    const size_t piece = ((len + parts - 1) / parts + 63) & ~(size_t)63;
    pool.run(parts, [&](size_t i) {
      const size_t a = std::min(len, i * piece), e = std::min(len, a + piece);
      if (e > a) std::memcpy(pin + a, s + off + a, e - a);
    });
    ZS_CUDA(cudaMemcpyAsync(d + off, pin, len, cudaMemcpyHostToDevice, st));
    ZS_CUDA(cudaEventRecord(sg->ev[b], st));
  }
}

void upload_low_words(uint32_t* dst, const uint8_t* const* cols, uint32_t C, size_t n, uint8_t* high,
                      cudaStream_t st) {
  Stager* sg = t_slot ? &t_slot->stager : nullptr;
  if (!sg || !sg->ok) throw Error(ZS_EGENERIC, "upload_low_words needs pinned staging");
  HostPool& pool = HostPool::get();
  const size_t parts = pool.width();
  const size_t per_chunk = kChunk / 4;  // elements per staging buffer
  // Element g of the upload is element g mod n of column g / n, and the columns are
  // adjacent in `dst`, so a staging buffer is filled across column boundaries: one
  // pool run and one copy per buffer, however short the columns.
  const size_t total = (size_t)C * n;
  std::vector<uint8_t> part_high(parts * C, 0);
  for (size_t g0 = 0; g0 < total; g0 += per_chunk) {
    const size_t len = std::min(per_chunk, total - g0);
    const int b = (int)(sg->next++ & 1);
    ZS_CUDA(cudaEventSynchronize(sg->ev[b]));
    uint32_t* pin = static_cast<uint32_t*>(sg->buf[b]);
    const size_t piece = (len + parts - 1) / parts;
    pool.run(parts, [&](size_t i) {
      size_t a = std::min(len, i * piece);
      const size_t e = std::min(len, a + piece);
      while (a < e) {
        const size_t g = g0 + a, j = g / n, off = g % n;
        const size_t run = std::min(e - a, n - off);
        const uint8_t* src = cols[j] + 16 * off;
        uint32_t acc = 0;
        for (size_t k = 0; k < run; ++k) {
          uint32_t w[4];
          std::memcpy(w, src + 16 * k, 16);
          pin[a + k] = w[0];
          acc |= w[1] | w[2] | w[3];
        }
        if (acc) part_high[i * C + j] = 1;
        a += run;
      }
    });
    ZS_CUDA(cudaMemcpyAsync(dst + g0, pin, len * 4, cudaMemcpyHostToDevice, st));
    ZS_CUDA(cudaEventRecord(sg->ev[b], st));
  }
  for (uint32_t j = 0; j < C; ++j) {
    high[j] = 0;
    for (size_t i = 0; i < parts; ++i) high[j] |= part_high[i * C + j];
  }
}

}  // namespace zs
