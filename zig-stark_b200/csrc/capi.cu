// extern "C" entry points declared in include/zs_m31.h.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <thread>

#include "../../include/zs_m31.h"
#include "circle.cuh"
#include "commit.cuh"
#include "stark.cuh"
#include "verify.cuh"

using namespace zs;

namespace {

template <typename F>
int32_t guarded(F&& f) {
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

void ensure_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw Error(ZS_EDEVICE, "no CUDA device");
}

struct DeviceBuffer {
  void* p = nullptr;
  explicit DeviceBuffer(size_t bytes) { ZS_CUDA(cudaMalloc(&p, bytes ? bytes : 4)); }
  ~DeviceBuffer() { cudaFree(p); }
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

int32_t circle_transform(const uint32_t* in, uint32_t n_columns, uint32_t ox, uint32_t oy, uint32_t sx, uint32_t sy,
                         uint32_t log_half, uint32_t* out, bool inverse) {
  return guarded([&] {
    if (!in || !out || n_columns == 0) throw Error(ZS_EMALFORMED, "null buffer or no columns");
    if (log_half > 27) throw Error(ZS_EMALFORMED, "log_half above 27");
    if (ox >= P || oy >= P || sx >= P || sy >= P) throw Error(ZS_EMALFORMED, "non-canonical coset point");
    ensure_device();
    const unsigned lg = log_half + 1;
    const size_t n = (size_t)1 << lg;
    cudaStream_t st = nullptr;
    CircleDomain dom(lg, cpoint{ox, oy}, cpoint{sx, sy}, st);
    DeviceBuffer a(n * n_columns * 4), b(n * n_columns * 4), s(n * n_columns * 4);
    ZS_CUDA(cudaMemcpy(a.p, in, n * n_columns * 4, cudaMemcpyHostToDevice));
    if (inverse)
      circle_ifft(a.as<uint32_t>(), b.as<uint32_t>(), n_columns, dom, s.as<uint32_t>(), st);
    else
      circle_fft(a.as<uint32_t>(), b.as<uint32_t>(), n_columns, dom, s.as<uint32_t>(), st);
    ZS_CUDA(cudaMemcpy(out, b.p, n * n_columns * 4, cudaMemcpyDeviceToHost));
  });
}

}  // namespace

struct zs_commit_plan {
  std::unique_ptr<CommitPlan> plan;
};

extern "C" {

int32_t zs_m31_circle_fft(const uint32_t* coeffs, uint32_t n_columns, uint32_t offset_x, uint32_t offset_y,
                          uint32_t step_x, uint32_t step_y, uint32_t log_half, uint32_t* evals) {
  return circle_transform(coeffs, n_columns, offset_x, offset_y, step_x, step_y, log_half, evals, false);
}

int32_t zs_m31_circle_ifft(const uint32_t* evals, uint32_t n_columns, uint32_t offset_x, uint32_t offset_y,
                           uint32_t step_x, uint32_t step_y, uint32_t log_half, uint32_t* coeffs) {
  return circle_transform(evals, n_columns, offset_x, offset_y, step_x, step_y, log_half, coeffs, true);
}

int32_t zs_m31_commit_plan_create(uint32_t n_columns, uint32_t log_rows, uint32_t log_blowup, uint32_t n_folds,
                                  zs_commit_plan** out) {
  return guarded([&] {
    if (!out) throw Error(ZS_EMALFORMED, "null out");
    ensure_device();
    auto p = std::make_unique<zs_commit_plan>();
    p->plan = std::make_unique<CommitPlan>(n_columns, log_rows, log_blowup, n_folds);
    *out = p.release();
  });
}

void zs_m31_commit_plan_destroy(zs_commit_plan* plan) { delete plan; }

int32_t zs_m31_commit_plan_set_challenges(zs_commit_plan* plan, const uint32_t* gammas, const uint32_t* alphas) {
  return guarded([&] {
    if (!plan || !gammas || (!alphas && plan->plan->F > 0)) throw Error(ZS_EMALFORMED, "null argument");
    plan->plan->set_challenges(gammas, alphas);
  });
}

uint32_t* zs_m31_commit_plan_trace_buffer(zs_commit_plan* plan) { return plan ? plan->plan->trace : nullptr; }

int32_t zs_m31_commit_plan_upload(zs_commit_plan* plan, const uint32_t* host_trace, void* stream) {
  return guarded([&] {
    if (!plan || !host_trace) throw Error(ZS_EMALFORMED, "null argument");
    CommitPlan& p = *plan->plan;
    ZS_CUDA(cudaMemcpyAsync(p.trace, host_trace, ((size_t)p.C << p.L) * 4, cudaMemcpyHostToDevice,
                            (cudaStream_t)stream));
  });
}

int32_t zs_m31_commit_plan_run_device(zs_commit_plan* plan, const uint32_t* d_trace, void* stream) {
  return guarded([&] {
    if (!plan) throw Error(ZS_EMALFORMED, "null plan");
    plan->plan->run(d_trace, (cudaStream_t)stream);
  });
}

int32_t zs_m31_commit_plan_run_host(zs_commit_plan* plan, const uint32_t* host_trace, void* stream) {
  return guarded([&] {
    if (!plan || !host_trace) throw Error(ZS_EMALFORMED, "null argument");
    plan->plan->run_host(host_trace, (cudaStream_t)stream);
  });
}

int32_t zs_m31_commit_plan_run_phase(zs_commit_plan* plan, int32_t phase, const uint32_t* d_trace, void* stream) {
  return guarded([&] {
    if (!plan) throw Error(ZS_EMALFORMED, "null plan");
    plan->plan->run_phase(phase, d_trace, (cudaStream_t)stream);
  });
}

int32_t zs_m31_commit_plan_results(zs_commit_plan* plan, void* stream, uint8_t* lde_root, uint8_t* layer_roots,
                                   uint32_t* final_layer) {
  return guarded([&] {
    if (!plan) throw Error(ZS_EMALFORMED, "null plan");
    CommitPlan& p = *plan->plan;
    cudaStream_t st = (cudaStream_t)stream;
    if (lde_root) ZS_CUDA(cudaMemcpyAsync(lde_root, p.row_tree.root(), 32, cudaMemcpyDeviceToHost, st));
    if (layer_roots)
      for (unsigned i = 0; i < p.F; ++i)
        ZS_CUDA(cudaMemcpyAsync(layer_roots + 32 * i, p.layer_trees[i].root(), 32, cudaMemcpyDeviceToHost, st));
    if (final_layer)
      ZS_CUDA(cudaMemcpyAsync(final_layer, p.layers[p.F], ((size_t)1 << (p.L + p.B - p.F)) * sizeof(qm31),
                              cudaMemcpyDeviceToHost, st));
    ZS_CUDA(cudaStreamSynchronize(st));
  });
}

int32_t zs_m31_commit_plan_copy_lde(zs_commit_plan* plan, uint32_t* host_out) {
  return guarded([&] {
    if (!plan || !host_out) throw Error(ZS_EMALFORMED, "null argument");
    CommitPlan& p = *plan->plan;
    ZS_CUDA(cudaDeviceSynchronize());
    ZS_CUDA(cudaMemcpy(host_out, p.lde, ((size_t)p.C << (p.L + p.B)) * 4, cudaMemcpyDeviceToHost));
  });
}

int32_t zs_m31_commit_plan_copy_layer(zs_commit_plan* plan, uint32_t layer, uint32_t* host_out) {
  return guarded([&] {
    if (!plan || !host_out) throw Error(ZS_EMALFORMED, "null argument");
    CommitPlan& p = *plan->plan;
    if (layer > p.F) throw Error(ZS_EMALFORMED, "layer index above n_folds");
    ZS_CUDA(cudaDeviceSynchronize());
    ZS_CUDA(cudaMemcpy(host_out, p.layers[layer], ((size_t)1 << (p.L + p.B - layer)) * sizeof(qm31),
                       cudaMemcpyDeviceToHost));
  });
}

uint32_t zs_m31_commit_plan_launches(const zs_commit_plan* plan) { return plan ? plan->plan->launches() : 0; }

int32_t zs_m31_circle_commit(const uint32_t* trace, uint32_t n_columns, uint32_t log_rows, uint32_t log_blowup,
                             const uint32_t* gammas, const uint32_t* alphas, uint32_t n_folds, uint8_t* lde_root,
                             uint8_t* layer_roots, uint32_t* final_layer) {
  zs_commit_plan* plan = nullptr;
  int32_t rc = zs_m31_commit_plan_create(n_columns, log_rows, log_blowup, n_folds, &plan);
  if (rc != 0) return rc;
  rc = zs_m31_commit_plan_set_challenges(plan, gammas, alphas);
  if (rc == 0) rc = zs_m31_commit_plan_upload(plan, trace, nullptr);
  if (rc == 0) rc = zs_m31_commit_plan_run_device(plan, nullptr, nullptr);
  if (rc == 0) rc = zs_m31_commit_plan_results(plan, nullptr, lde_root, layer_roots, final_layer);
  zs_m31_commit_plan_destroy(plan);
  return rc;
}

namespace {

// The calling thread's current device for the lifetime of the scope is `device`.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int device) {
    ZS_CUDA(cudaGetDevice(&prev));
    if (prev != device) ZS_CUDA(cudaSetDevice(device));
  }
  ~DeviceScope() {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;
};

// The argument checks of zs_m31_prove, made before any device is touched.
void check_prove_args(zs_host_allocator host, const uint8_t* params, size_t params_len, const uint8_t* public_inputs,
                      size_t public_inputs_len, const uint8_t* preprocessed, size_t preprocessed_len,
                      const uint8_t* trace, size_t trace_len, const uint8_t* channel_sep, size_t channel_sep_len,
                      uint8_t** out_proof, size_t* out_len) {
  if (!out_proof || !out_len || !host.alloc) throw Error(ZS_EMALFORMED, "null output or allocator");
  if ((!params && params_len) || (!public_inputs && public_inputs_len) || (!preprocessed && preprocessed_len) ||
      (!trace && trace_len) || (!channel_sep && channel_sep_len))
    throw Error(ZS_EMALFORMED, "null input buffer with a non-zero length");
}

// zs_m31_prove on stream `st` of the current device: proves and hands the bytes to the
// caller's allocator.
void prove_on(cudaStream_t st, zs_host_allocator host, uint32_t air_id, const uint8_t* params, size_t params_len,
              const uint8_t* public_inputs, size_t public_inputs_len, const uint8_t* preprocessed,
              size_t preprocessed_len, const uint8_t* trace, size_t trace_len, const uint8_t* channel_sep,
              size_t channel_sep_len, uint8_t** out_proof, size_t* out_len) {
  std::vector<uint8_t> bytes;
  try {
    bytes = stark_prove(air_id, params, params_len, public_inputs, public_inputs_len, preprocessed, preprocessed_len,
                        trace, trace_len, channel_sep, channel_sep_len, st);
  } catch (...) {
    cudaStreamSynchronize(st);
    throw;
  }
  uint8_t* buf = (uint8_t*)host.alloc(host.ctx, bytes.size() ? bytes.size() : 1);
  if (!buf) throw Error(ZS_ENOMEM, "host allocator returned null");
  std::memcpy(buf, bytes.data(), bytes.size());
  *out_proof = buf;
  *out_len = bytes.size();
}

}  // namespace

struct zs_m31_ctx {
  int device = 0;
  cudaStream_t st = nullptr;
  std::mutex mu;  // one call at a time on this context
};

int32_t zs_m31_prove(zs_host_allocator host, uint32_t air_id, const uint8_t* params, size_t params_len,
                     const uint8_t* public_inputs, size_t public_inputs_len, const uint8_t* preprocessed,
                     size_t preprocessed_len, const uint8_t* trace, size_t trace_len, const uint8_t* channel_sep,
                     size_t channel_sep_len, uint8_t** out_proof, size_t* out_len) {
  return guarded([&] {
    check_prove_args(host, params, params_len, public_inputs, public_inputs_len, preprocessed, preprocessed_len, trace,
                     trace_len, channel_sep, channel_sep_len, out_proof, out_len);
    ensure_device();
    cudaStream_t st = nullptr;
    thread_stream(0, &st);  // the calling thread's stream on the current device
    prove_on(st, host, air_id, params, params_len, public_inputs, public_inputs_len, preprocessed, preprocessed_len,
             trace, trace_len, channel_sep, channel_sep_len, out_proof, out_len);
  });
}

int32_t zs_m31_ctx_create(int32_t device, zs_m31_ctx** out) {
  return guarded([&] {
    if (!out) throw Error(ZS_EMALFORMED, "null output");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw Error(ZS_EDEVICE, "no CUDA device");
    if (device < 0 || device >= n) throw Error(ZS_EDEVICE, "device ordinal out of range");
    DeviceScope scope(device);
    auto c = std::make_unique<zs_m31_ctx>();
    c->device = device;
    ZS_CUDA(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    *out = c.release();
  });
}

void zs_m31_ctx_destroy(zs_m31_ctx* ctx) {
  if (!ctx) return;
  {
    std::lock_guard<std::mutex> lock(ctx->mu);
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(ctx->device) == cudaSuccess) {
      cudaStreamSynchronize(ctx->st);
      cudaStreamDestroy(ctx->st);
    }
    if (prev >= 0) cudaSetDevice(prev);
  }
  delete ctx;
}

int32_t zs_m31_ctx_device(const zs_m31_ctx* ctx) { return ctx ? ctx->device : ZS_EMALFORMED; }

int32_t zs_m31_prove_ctx(zs_m31_ctx* ctx, zs_host_allocator host, uint32_t air_id, const uint8_t* params,
                         size_t params_len, const uint8_t* public_inputs, size_t public_inputs_len,
                         const uint8_t* preprocessed, size_t preprocessed_len, const uint8_t* trace,
                         size_t trace_len, const uint8_t* channel_sep, size_t channel_sep_len, uint8_t** out_proof,
                         size_t* out_len) {
  return guarded([&] {
    if (!ctx) throw Error(ZS_EMALFORMED, "null context");
    check_prove_args(host, params, params_len, public_inputs, public_inputs_len, preprocessed, preprocessed_len, trace,
                     trace_len, channel_sep, channel_sep_len, out_proof, out_len);
    std::lock_guard<std::mutex> lock(ctx->mu);
    DeviceScope scope(ctx->device);
    prove_on(ctx->st, host, air_id, params, params_len, public_inputs, public_inputs_len, preprocessed,
             preprocessed_len, trace, trace_len, channel_sep, channel_sep_len, out_proof, out_len);
  });
}

int32_t zs_m31_verify(zs_host_allocator host, uint32_t air_id, const uint8_t* params, size_t params_len,
                      const uint8_t* public_inputs, size_t public_inputs_len, const uint8_t* proof, size_t proof_len,
                      const uint8_t* channel_sep, size_t channel_sep_len, int* out_ok) {
  (void)host;
  return guarded([&] {
    if (!out_ok) throw Error(ZS_EMALFORMED, "null out_ok");
    if ((!params && params_len) || (!public_inputs && public_inputs_len) || (!proof && proof_len) ||
        (!channel_sep && channel_sep_len))
      throw Error(ZS_EMALFORMED, "null input buffer with a non-zero length");
    *out_ok = 0;
    *out_ok = stark_verify(air_id, params, params_len, public_inputs, public_inputs_len, proof, proof_len,
                           channel_sep, channel_sep_len)
                  ? 1
                  : 0;
  });
}

int32_t zs_m31_verify_batch(size_t n_jobs, const zs_m31_verify_job* jobs, uint32_t threads, int* out_ok,
                            int32_t* statuses) {
  return guarded([&] {
    if (n_jobs && (!jobs || !out_ok || !statuses)) throw Error(ZS_EMALFORMED, "null argument");
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    if (threads > n_jobs) threads = (uint32_t)std::max<size_t>(n_jobs, 1);
    std::atomic<size_t> next{0};
    auto work = [&] {
      for (size_t i; (i = next.fetch_add(1)) < n_jobs;) {
        const zs_m31_verify_job& j = jobs[i];
        int ok = 0;
        statuses[i] = zs_m31_verify(zs_host_allocator{}, j.air_id, j.params, j.params_len, j.public_inputs,
                                    j.public_inputs_len, j.proof, j.proof_len, j.channel_sep, j.channel_sep_len, &ok);
        out_ok[i] = ok;
      }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
  });
}

int32_t zs_m31_commit_columns(zs_host_allocator host, uint8_t trace_log, uint8_t log_blowup, const uint8_t* columns,
                              size_t columns_len, uint8_t** out_roots, size_t* out_len) {
  return guarded([&] {
    if (!out_roots || !out_len || !host.alloc) throw Error(ZS_EMALFORMED, "null output or allocator");
    if (!columns && columns_len) throw Error(ZS_EMALFORMED, "null input buffer with a non-zero length");
    ensure_device();
    cudaStream_t st = nullptr;
    ZS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    std::vector<uint8_t> bytes;
    try {
      bytes = commit_columns(columns, columns_len, trace_log, log_blowup, st);
    } catch (...) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
      throw;
    }
    cudaStreamDestroy(st);
    uint8_t* buf = (uint8_t*)host.alloc(host.ctx, bytes.size());
    if (!buf) throw Error(ZS_ENOMEM, "host allocator returned null");
    std::memcpy(buf, bytes.data(), bytes.size());
    *out_roots = buf;
    *out_len = bytes.size();
  });
}

void zs_free(zs_host_allocator host, uint8_t* ptr, size_t len) {
  if (ptr && host.free) host.free(host.ctx, ptr, len);
}

const char* zs_version(void) { return "zs-b200 0.1.0 (sm_100a, M31 DEEP-FRI commitment path)"; }

}  // extern "C"
