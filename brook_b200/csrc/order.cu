// Object voxel lists and target orders, with CUB's device sorts:
//  * the voxels of every object, grouped by object and ascending in flat index (a compaction of
//    the foreground in flat order and a stable radix sort by object);
//  * per object the target order: descending DAF (infinite -> 0), ties -> higher flat index first
//    (lockstep_order.cu:21-45 of giorgioangel/brook), as one segmented sort of 64-bit keys
//    (~daf bits, ~flat).
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include "order.hpp"

namespace bk {
namespace {

struct InObject {
  const uint32_t *ids;
  const int *rank;
  __device__ bool operator()(int i) const {
    const uint32_t id = ids[i];
    return id != 0 && rank[id] >= 0;
  }
};

__global__ void object_keys(const int *vox, const uint32_t *ids, const int *rank, uint32_t *keys, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keys[i] = uint32_t(rank[ids[vox[i]]]);
}

__global__ void order_keys(const int *vox, const float *daf, unsigned long long *keys, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int v = vox[i];
  float d = daf[v];
  if (isinf(d) || d == 0.0f) d = 0.0f;
  keys[i] = (static_cast<unsigned long long>(0xFFFFFFFFu - __float_as_uint(d)) << 32) | (0xFFFFFFFFu - unsigned(v));
}

__global__ void unpack_order(const unsigned long long *keys, int *order, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) order[i] = int(0xFFFFFFFFu - unsigned(keys[i]));
}

}  // namespace

Buffer<int> object_voxels(Context &ctx, const uint32_t *ids, long long n, const int *rank, int nobj, long long total) {
  cudaStream_t s = ctx.stream();
  Buffer<int> picked(ctx, n > total ? n : (total > 0 ? total : 1)), count(ctx, 1);  // room for every voxel
  thrust::counting_iterator<int> index(0);
  size_t temp = 0;
  BK_CUDA(cub::DeviceSelect::If(nullptr, temp, index, picked.data(), count.data(), (int)n, InObject{ids, rank}, s));
  Buffer<unsigned char> scratch(ctx, temp);
  BK_CUDA(cub::DeviceSelect::If(scratch.data(), temp, index, picked.data(), count.data(), (int)n, InObject{ids, rank}, s));
  const int got = count.download(1)[0];
  if (got != total) throw std::runtime_error("object voxel count mismatch");
  Buffer<uint32_t> keys(ctx, total), keys_out(ctx, total);
  Buffer<int> vox(ctx, total);
  if (total == 0) return vox;
  object_keys<<<blocks_for(total), 256, 0, s>>>(picked.data(), ids, rank, keys.data(), (int)total); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  int bits = 1;
  while ((1LL << bits) < nobj) ++bits;
  temp = 0;
  BK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, keys.data(), keys_out.data(), picked.data(), vox.data(),
                                          (int)total, 0, bits, s));
  scratch = Buffer<unsigned char>(ctx, temp);
  BK_CUDA(cub::DeviceRadixSort::SortPairs(scratch.data(), temp, keys.data(), keys_out.data(), picked.data(), vox.data(),
                                          (int)total, 0, bits, s));
  return vox;
}

Buffer<int> target_orders(Context &ctx, const int *vox, const float *daf, long long total, const int *begin,
                          const int *end, int nobj) {
  cudaStream_t s = ctx.stream();
  Buffer<int> order(ctx, total > 0 ? total : 1);
  if (total == 0) return order;
  Buffer<unsigned long long> keys(ctx, total), sorted(ctx, total);
  order_keys<<<blocks_for(total), 256, 0, s>>>(vox, daf, keys.data(), (int)total); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  size_t temp = 0;
  BK_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, temp, keys.data(), sorted.data(), (int)total, nobj, begin, end, s));
  Buffer<unsigned char> scratch(ctx, temp);
  BK_CUDA(cub::DeviceSegmentedSort::SortKeys(scratch.data(), temp, keys.data(), sorted.data(), (int)total, nobj, begin,
                                             end, s));
  unpack_order<<<blocks_for(total), 256, 0, s>>>(sorted.data(), order.data(), (int)total); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  return order;
}

}  // namespace bk
