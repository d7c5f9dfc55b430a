#include "runtime.hpp"

#include <cstdint>

namespace bk {

Context::Context(int device) : device_(device) {
  int count = 0;
  BK_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) throw std::invalid_argument("device index out of range");
  DeviceGuard guard(device);
  cudaDeviceProp prop{};
  BK_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) throw std::invalid_argument("brook_b200 requires a compute capability 10.x (Blackwell) GPU");
  sm_count_ = prop.multiProcessorCount;
  BK_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  // Keep freed blocks in this process's pool between calls: repeated calls of one shape then
  // allocate nothing from the driver.
  cudaMemPool_t pool;
  BK_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t threshold = UINT64_MAX;
  BK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
}

cudaStream_t Context::copy_stream() {
  if (!copy_) {
    DeviceGuard guard(device_);
    BK_CUDA(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
  }
  return copy_;
}

void Context::launch_graph(cudaGraph_t graph) {
  if (engine_exec_) {
    cudaGraphExecUpdateResultInfo info{};
    if (cudaGraphExecUpdate(engine_exec_, graph, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(engine_exec_);
      engine_exec_ = nullptr;
    } else stats["graph_updates"] += 1;
  }
  if (!engine_exec_) {
    const cudaError_t made = cudaGraphInstantiate(&engine_exec_, graph, 0);
    if (made != cudaSuccess) {
      engine_exec_ = nullptr;
      cudaGraphDestroy(graph);
      throw CudaError(made, "cudaGraphInstantiate");
    }
    stats["graph_instantiations"] += 1;
  }
  const cudaError_t launched = cudaGraphLaunch(engine_exec_, stream_);
  cudaGraphDestroy(graph);
  BK_CUDA(launched);
  stats["graph_launches"] += 1;
}

Context::~Context() {
  if (stream_) {
    int previous = -1;
    cudaGetDevice(&previous);
    cudaSetDevice(device_);
    if (engine_exec_) cudaGraphExecDestroy(engine_exec_);
    if (copy_) {
      cudaStreamSynchronize(copy_);
      cudaStreamDestroy(copy_);
    }
    for (auto &entry : free_)
      for (void *p : entry.second) cudaFreeAsync(p, stream_);
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(stream_);
    if (previous >= 0) cudaSetDevice(previous);
  }
}

namespace {

constexpr size_t kCacheCap = size_t(24) << 30;  // cached bytes kept per context at most

size_t size_class(size_t bytes) {
  if (bytes <= 256) return 256;
  int top = 63 - __builtin_clzll((unsigned long long)(bytes - 1));
  const size_t step = size_t(1) << (top >= 3 ? top - 3 : 0);  // 8 classes per power of two
  return (bytes + step - 1) / step * step;
}

}  // namespace

void *Context::allocate(size_t bytes) {
  const size_t cls = size_class(bytes);
  auto it = free_.find(cls);
  if (it != free_.end() && !it->second.empty()) {
    void *p = it->second.back();
    it->second.pop_back();
    cached_ -= cls;
    live_ += cls;
    if (live_ > peak_) peak_ = live_;
    return p;
  }
  void *p = nullptr;
  cudaError_t status = cudaMallocAsync(&p, cls, stream_);
  if (status != cudaSuccess) {
    cudaGetLastError();
    trim();
    status = cudaMallocAsync(&p, cls, stream_);
    if (status != cudaSuccess) {
      cudaGetLastError();
      throw CudaError(status, "cudaMallocAsync(" + std::to_string(bytes) + " bytes)");
    }
  }
  class_of_[p] = cls;
  live_ += cls;
  if (live_ > peak_) peak_ = live_;
  return p;
}

void Context::release(void *p) {
  if (!p) return;
  auto it = class_of_.find(p);
  if (it == class_of_.end()) {  // not ours: hand it back as it is
    cudaFreeAsync(p, stream_);
    return;
  }
  const size_t cls = it->second;
  live_ -= cls;
  if (cached_ + cls > kCacheCap) {
    class_of_.erase(it);
    cudaFreeAsync(p, stream_);
    return;
  }
  free_[cls].push_back(p);
  cached_ += cls;
}

void Context::trim() {
  for (auto &entry : free_)
    for (void *p : entry.second) {
      class_of_.erase(p);
      cudaFreeAsync(p, stream_);
    }
  free_.clear();
  cached_ = 0;
  cudaStreamSynchronize(stream_);
}

}  // namespace bk
