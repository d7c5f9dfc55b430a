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

Context::~Context() {
  if (stream_) {
    int previous = -1;
    cudaGetDevice(&previous);
    cudaSetDevice(device_);
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(stream_);
    if (previous >= 0) cudaSetDevice(previous);
  }
}

void *Context::allocate(size_t bytes) {
  void *p = nullptr;
  cudaError_t status = cudaMallocAsync(&p, bytes, stream_);
  if (status != cudaSuccess) {
    cudaGetLastError();
    throw CudaError(status, "cudaMallocAsync(" + std::to_string(bytes) + " bytes)");
  }
  return p;
}

void Context::release(void *p) {
  if (p) cudaFreeAsync(p, stream_);
}

}  // namespace bk
