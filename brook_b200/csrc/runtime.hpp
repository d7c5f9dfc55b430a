// Host runtime of brook_b200: one context per device with one non-blocking stream, stream-ordered
// allocations from the device's memory pool, typed device buffers and the error types the C ABI
// maps to status codes.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace bk {

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const std::string &where)
      : std::runtime_error(where + ": " + cudaGetErrorString(c)), code(c) {}
};

#define BK_CUDA(call)                                                                        \
  do {                                                                                       \
    cudaError_t bk_status_ = (call);                                                         \
    if (bk_status_ != cudaSuccess) throw ::bk::CudaError(bk_status_, #call);                 \
  } while (0)

// Restores the caller's current device when a public call returns.
class DeviceGuard {
  int previous_ = -1;

 public:
  explicit DeviceGuard(int device) {
    BK_CUDA(cudaGetDevice(&previous_));
    if (previous_ != device) BK_CUDA(cudaSetDevice(device));
  }
  ~DeviceGuard() {
    if (previous_ >= 0) cudaSetDevice(previous_);
  }
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;
};

// Launch choices of the object engine for one workload class (0 / -1: the built-in rule).
struct Tuning {
  int trace_cluster_ctas = 0;             // CTAs per cluster for the large objects: 4 or 8
  long long trace_cluster_voxels = 0;     // objects above this trace on clusters
  long long prepare_cluster_voxels = 0;   // objects from this size prepare on clusters
  int lone_first_percent = -1;            // share of clusters that start on the small objects
};

class Context {
 public:
  explicit Context(int device);
  ~Context();
  Context(const Context &) = delete;
  Context &operator=(const Context &) = delete;

  int device() const { return device_; }
  cudaStream_t stream() const { return stream_; }
  // A second stream, for host-to-device copies that overlap the main stream's kernels (created on
  // first use). The main stream waits on its events before it reads what they copied.
  cudaStream_t copy_stream();
  int sm_count() const { return sm_count_; }
  void synchronize() const { BK_CUDA(cudaStreamSynchronize(stream_)); }
  // Stream-ordered device memory with a per-context cache: a released block goes to a free list
  // of its size class (8 classes per power of two) and the next allocation of that class reuses
  // it, in the stream's order, without a driver call. Cached bytes beyond a cap are returned to
  // the device's pool; when an allocation fails, every cached block is returned and it is tried
  // once more.
  void *allocate(size_t bytes);
  void release(void *p);
  void trim();  // returns every cached block to the device's pool
  // Bytes this context holds: handed out and not released (`live`), kept in its free lists
  // (`cached`), and the most handed out at once since the last reset_peak().
  size_t live_bytes() const { return live_; }
  size_t cached_bytes() const { return cached_; }
  size_t peak_bytes() const { return peak_; }
  void reset_peak() { peak_ = live_; }
  std::mutex &mutex() { return mutex_; }
  // Per-call statistics: stage times (ms, CUDA events on this context's stream) and work counters.
  std::map<std::string, double> stats;
  // Kernels of this library launched by the current call.
  long long launches = 0;
  // Tuned engine launch choices by workload class (see workload_class in the pipeline), filled by
  // the autotuner or from a saved table; `forced` overrides them while the autotuner measures.
  std::map<unsigned long long, Tuning> tuning;
  const Tuning *forced = nullptr;
  // The share (percent, 1-100) of the device's resident clusters the engine's persistent launches
  // take; below 100 another context's kernels find free CTA slots while this one traces.
  int engine_percent = 100;
  unsigned long long last_class = 0;  // the workload class of the last call
  // Launches a captured graph of the engine's launches: the context keeps one executable graph and
  // updates it in place when the new graph has the same topology (else instantiates it anew).
  void launch_graph(cudaGraph_t graph);

 private:
  int device_ = 0, sm_count_ = 0;
  cudaStream_t stream_ = nullptr, copy_ = nullptr;
  std::mutex mutex_;
  std::map<size_t, std::vector<void *>> free_;  // size class -> cached blocks
  std::map<void *, size_t> class_of_;           // live and cached blocks -> size class
  size_t cached_ = 0, live_ = 0, peak_ = 0;
  cudaGraphExec_t engine_exec_ = nullptr;
};

// Device storage that outlives the context that made it (plain cudaMalloc / cudaFree on its
// device): results handed to callers.
struct DeviceStorage {
  void *ptr = nullptr;
  size_t bytes = 0;
  int device = 0;
  DeviceStorage(size_t n, int dev) : bytes(n), device(dev) {
    if (n) {
      cudaError_t s = cudaMalloc(&ptr, n);
      if (s != cudaSuccess) { cudaGetLastError(); throw CudaError(s, "cudaMalloc"); }
    }
  }
  ~DeviceStorage() {
    if (ptr) {
      int previous = -1;
      cudaGetDevice(&previous);
      cudaSetDevice(device);
      cudaFree(ptr);
      if (previous >= 0) cudaSetDevice(previous);
    }
  }
  DeviceStorage(const DeviceStorage &) = delete;
  DeviceStorage &operator=(const DeviceStorage &) = delete;
};

// A typed stream-ordered device allocation owned by one context.
template <class T>
class Buffer {
  Context *ctx_ = nullptr;
  T *ptr_ = nullptr;
  size_t count_ = 0;

 public:
  Buffer() = default;
  Buffer(Context &ctx, size_t count) : ctx_(&ctx), count_(count) {
    if (count) ptr_ = static_cast<T *>(ctx.allocate(count * sizeof(T)));
  }
  ~Buffer() { reset(); }
  Buffer(Buffer &&o) noexcept : ctx_(o.ctx_), ptr_(o.ptr_), count_(o.count_) { o.ptr_ = nullptr; o.count_ = 0; }
  Buffer &operator=(Buffer &&o) noexcept {
    if (this != &o) { reset(); ctx_ = o.ctx_; ptr_ = o.ptr_; count_ = o.count_; o.ptr_ = nullptr; o.count_ = 0; }
    return *this;
  }
  Buffer(const Buffer &) = delete;
  Buffer &operator=(const Buffer &) = delete;
  void reset() {
    if (ptr_ && ctx_) ctx_->release(ptr_);
    ptr_ = nullptr;
    count_ = 0;
  }
  T *data() const { return ptr_; }
  size_t size() const { return count_; }
  size_t bytes() const { return count_ * sizeof(T); }
  void zero() const {
    if (count_) BK_CUDA(cudaMemsetAsync(ptr_, 0, bytes(), ctx_->stream()));
  }
  void fill_bytes(int value) const {
    if (count_) BK_CUDA(cudaMemsetAsync(ptr_, value, bytes(), ctx_->stream()));
  }
  void upload(const T *host, size_t n, size_t offset = 0) const {
    if (n) BK_CUDA(cudaMemcpyAsync(ptr_ + offset, host, n * sizeof(T), cudaMemcpyHostToDevice, ctx_->stream()));
  }
  void upload(const std::vector<T> &host) const { upload(host.data(), host.size()); }
  // Synchronous download of the first n elements.
  std::vector<T> download(size_t n, size_t offset = 0) const {
    std::vector<T> out(n);
    if (n) {
      BK_CUDA(cudaMemcpyAsync(out.data(), ptr_ + offset, n * sizeof(T), cudaMemcpyDeviceToHost, ctx_->stream()));
      ctx_->synchronize();
    }
    return out;
  }
  std::vector<T> download() const { return download(count_); }
};

// Stage boundaries recorded as CUDA events on the context's stream; finish() adds each stage's
// elapsed time to ctx.stats["ms_<stage>"]. Each mark also adds the host time since the previous
// mark to ctx.stats["host_ms_<stage>"] (near the device time: the device waited for the host).
class StageClock {
  Context &ctx_;
  std::vector<std::pair<std::string, cudaEvent_t>> marks_;
  std::chrono::steady_clock::time_point host_ = std::chrono::steady_clock::now();
  bool capturing_ = false;

 public:
  explicit StageClock(Context &ctx) : ctx_(ctx) { mark("start"); }
  // While the stream is captured into a graph, marks become event record nodes of the graph (they
  // record when the graph runs).
  void capturing(bool on) { capturing_ = on; }
  ~StageClock() {
    for (auto &m : marks_) cudaEventDestroy(m.second);
  }
  void mark(const std::string &stage) {
    const auto now = std::chrono::steady_clock::now();
    if (!marks_.empty()) ctx_.stats["host_ms_" + stage] += std::chrono::duration<double, std::milli>(now - host_).count();
    host_ = now;
    cudaEvent_t e;
    BK_CUDA(cudaEventCreate(&e));
    marks_.push_back({stage, e});
    BK_CUDA(cudaEventRecordWithFlags(e, ctx_.stream(), capturing_ ? cudaEventRecordExternal : cudaEventRecordDefault));
  }
  void finish() {
    if (marks_.size() < 2) return;
    BK_CUDA(cudaEventSynchronize(marks_.back().second));
    for (size_t i = 1; i < marks_.size(); ++i) {
      float ms = 0;
      BK_CUDA(cudaEventElapsedTime(&ms, marks_[i - 1].second, marks_[i].second));
      ctx_.stats["ms_" + marks_[i].first] += ms;
    }
    float total = 0;
    BK_CUDA(cudaEventElapsedTime(&total, marks_.front().second, marks_.back().second));
    ctx_.stats["ms_total"] += total;
  }
};

template <class T>
Buffer<T> to_device(Context &ctx, const std::vector<T> &host) {
  Buffer<T> b(ctx, host.size());
  b.upload(host);
  return b;
}

inline unsigned blocks_for(long long n, int threads = 256) { return static_cast<unsigned>((n + threads - 1) / threads); }

}  // namespace bk
