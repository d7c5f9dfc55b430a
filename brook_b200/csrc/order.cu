// Object voxel lists and target orders, with CUB's device sorts:
//  * the voxels of every object of every volume of a call, grouped by object and ascending in
//    flat index (one compaction of the arena in flat order and one stable radix sort by object);
//  * per object the target order: descending DAF (infinite -> 0), ties -> higher flat index first
//    (lockstep_order.cu:21-45 of giorgioangel/brook). Inside an object the voxel list ascends in
//    flat index, so "higher flat first" is "later list position first": the composite key
//    (object rank, 0x7FFFFFFF - DAF bits, last position - position) orders every object at once in
//    one device-wide radix sort over all SMs (a non-negative float's sign bit is 0, so 31 DAF bits
//    suffice). The key is a 64-bit word when the object, DAF and position bits fit, else a
//    (32-bit, 64-bit) pair sorted through a decomposer over only the bits in use.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include "order.hpp"

namespace bk {
namespace {

// The object of arena voxel i, or -1: the listed volume whose range holds i, then its id's object.
constexpr int kBlockShift = 12;  // voxels per entry of the volume lookup: 4096

struct ArenaObject {
  const uint32_t *ids;
  const long long *begin, *end;  // per listed volume, ascending
  const int *id_base;            // per listed volume: where its id -> object table starts
  const int *object_of;
  const int *block_volume;       // per 4096-voxel block: the last volume that begins at or before it
  int nvol;
  __device__ int operator()(long long i) const {
    // from the block's volume, forward over the few volumes that begin within the block
    int lo = __ldg(block_volume + (i >> kBlockShift));
    while (lo + 1 < nvol && __ldg(begin + lo + 1) <= i) ++lo;
    if (i < __ldg(begin + lo) || i >= __ldg(end + lo)) return -1;
    const uint32_t id = ids[i];
    return id == 0 ? -1 : __ldg(object_of + __ldg(id_base + lo) + int(id));
  }
};

struct InArenaObject {
  ArenaObject at;
  __device__ bool operator()(int i) const { return at(i) >= 0; }
};

__global__ void arena_object_keys(const int *vox, ArenaObject at, uint32_t *keys, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keys[i] = uint32_t(at(vox[i]));
}

__global__ void mark_alive(const int *vox, uint8_t *alive, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) alive[vox[i]] = 1;
}

// The composite key's fields for list position i of object o: o << (lbits + 31) | (0x7FFFFFFF -
// daf bits) << lbits | (2^lbits - 1 - position in o).
struct WideKey {
  unsigned long long lo;
  uint32_t hi;
};

struct WideKeyParts {
  __host__ __device__ cuda::std::tuple<uint32_t &, unsigned long long &> operator()(WideKey &k) const {
    return {k.hi, k.lo};
  }
};

__device__ __forceinline__ int object_of_position(const int *begin, int nobj, int i) {
  int lo = 0, hi = nobj - 1;  // the last object whose range begins at or before i
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(begin + mid) <= i) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ unsigned long long order_low(const int *vox, const float *daf, const int *begin, int o,
                                                        int i, int lbits) {
  float d = daf[vox[i]];
  if (isinf(d) || d == 0.0f) d = 0.0f;
  const unsigned long long lmask = (1ULL << lbits) - 1;
  return (static_cast<unsigned long long>(0x7FFFFFFFu - __float_as_uint(d)) << lbits) |
         (lmask - unsigned(i - __ldg(begin + o)));
}

__global__ void order_keys64(const int *vox, const float *daf, const int *begin, int nobj, int lbits,
                             unsigned long long *keys, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = object_of_position(begin, nobj, i);
  keys[i] = (static_cast<unsigned long long>(o) << (lbits + 31)) | order_low(vox, daf, begin, o, i, lbits);
}

__global__ void order_keys96(const int *vox, const float *daf, const int *begin, int nobj, int lbits, WideKey *keys,
                             int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int o = object_of_position(begin, nobj, i);
  const int shift = lbits + 31;  // 31 .. 62
  WideKey k;
  k.lo = (static_cast<unsigned long long>(o) << shift) | order_low(vox, daf, begin, o, i, lbits);
  k.hi = uint32_t(static_cast<unsigned long long>(o) >> (64 - shift));
  keys[i] = k;
}

// Sorted key -> voxel: the object from the top field, the position from the low field.
__device__ __forceinline__ int order_voxel(const int *vox, const int *begin, int o, unsigned long long lo, int lbits) {
  const unsigned long long lmask = (1ULL << lbits) - 1;
  return vox[__ldg(begin + o) + int(lmask - (lo & lmask))];
}

__global__ void unpack_order64(const unsigned long long *keys, const int *vox, const int *begin, int lbits, int *order,
                               int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned long long k = keys[i];
  order[i] = order_voxel(vox, begin, int(k >> (lbits + 31)), k, lbits);
}

__global__ void unpack_order96(const WideKey *keys, const int *vox, const int *begin, int lbits, int *order, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const WideKey k = keys[i];
  const int shift = lbits + 31;
  const int o = int((k.lo >> shift) | (static_cast<unsigned long long>(k.hi) << (64 - shift)));
  order[i] = order_voxel(vox, begin, o, k.lo, lbits);
}

}  // namespace

Buffer<int> arena_object_voxels(Context &ctx, const uint32_t *ids, long long n, const std::vector<ArenaVolume> &volumes,
                                const std::vector<int> &object_of, int nobj, long long total, uint8_t *alive) {
  cudaStream_t s = ctx.stream();
  Buffer<int> vox(ctx, total > 0 ? total : 1);
  if (total == 0 || volumes.empty()) {
    if (total != 0) throw std::runtime_error("object voxel count mismatch");
    return vox;
  }
  std::vector<long long> begin, end;
  std::vector<int> base;
  for (const auto &v : volumes) {
    begin.push_back(v.begin);
    end.push_back(v.end);
    base.push_back(v.id_base);
  }
  std::vector<int> block_volume(size_t((n >> kBlockShift) + 1), 0);
  for (size_t b = 0, v = 0; b < block_volume.size(); ++b) {
    const long long at = (long long)b << kBlockShift;
    while (v + 1 < begin.size() && begin[v + 1] <= at) ++v;
    block_volume[b] = int(v);
  }
  Buffer<long long> d_begin = to_device(ctx, begin), d_end = to_device(ctx, end);
  Buffer<int> d_base = to_device(ctx, base), d_object_of = to_device(ctx, object_of);
  Buffer<int> d_block_volume = to_device(ctx, block_volume);
  const ArenaObject at{ids, d_begin.data(), d_end.data(), d_base.data(), d_object_of.data(), d_block_volume.data(),
                       int(volumes.size())};
  Buffer<int> picked(ctx, total), count(ctx, 1);
  thrust::counting_iterator<int> index(0);
  size_t temp = 0;
  BK_CUDA(cub::DeviceSelect::If(nullptr, temp, index, picked.data(), count.data(), (int)n, InArenaObject{at}, s));
  Buffer<unsigned char> scratch(ctx, temp);
  BK_CUDA(cub::DeviceSelect::If(scratch.data(), temp, index, picked.data(), count.data(), (int)n, InArenaObject{at}, s));
  Buffer<uint32_t> keys(ctx, total), keys_out(ctx, total);
  arena_object_keys<<<blocks_for(total), 256, 0, s>>>(picked.data(), at, keys.data(), (int)total); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  int bits = 1;
  while ((1LL << bits) < nobj) ++bits;
  temp = 0;
  BK_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, keys.data(), keys_out.data(), picked.data(), vox.data(),
                                          (int)total, 0, bits, s));
  scratch = Buffer<unsigned char>(ctx, temp);
  BK_CUDA(cub::DeviceRadixSort::SortPairs(scratch.data(), temp, keys.data(), keys_out.data(), picked.data(), vox.data(),
                                          (int)total, 0, bits, s));
  mark_alive<<<blocks_for(total), 256, 0, s>>>(vox.data(), alive, (int)total); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  if (count.download(1)[0] != total) throw std::runtime_error("object voxel count mismatch");
  return vox;
}

OrderPlan plan_target_orders(Context &ctx, long long total, int nobj, long long largest, bool wide) {
  OrderPlan p;
  p.total = total;
  p.nobj = nobj;
  p.order = Buffer<int>(ctx, total > 0 ? total : 1);
  if (total == 0) return p;
  auto bits_for = [](long long values) {  // bits that hold 0 .. values-1
    int b = 0;
    while ((1LL << b) < values) ++b;
    return b;
  };
  p.lbits = bits_for(largest);
  p.end_bit = p.lbits + 31 + bits_for(nobj);
  p.wide = wide || p.end_bit > 64;
  const size_t key_bytes = p.wide ? sizeof(WideKey) : sizeof(unsigned long long);
  p.keys = Buffer<unsigned char>(ctx, total * key_bytes);
  p.sorted = Buffer<unsigned char>(ctx, total * key_bytes);
  // the scratch size is a host computation (no stream work)
  if (!p.wide)
    BK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, p.temp, reinterpret_cast<unsigned long long *>(p.keys.data()),
                                           reinterpret_cast<unsigned long long *>(p.sorted.data()), (int)total, 0,
                                           p.end_bit, ctx.stream()));
  else
    BK_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, p.temp, reinterpret_cast<WideKey *>(p.keys.data()),
                                           reinterpret_cast<WideKey *>(p.sorted.data()), (int)total, WideKeyParts{}, 0,
                                           p.end_bit, ctx.stream()));
  p.scratch = Buffer<unsigned char>(ctx, p.temp > 0 ? p.temp : 1);
  return p;
}

void run_target_orders(Context &ctx, OrderPlan &p, const int *vox, const float *daf, const int *begin) {
  if (p.total == 0) return;
  cudaStream_t s = ctx.stream();
  const long long total = p.total;
  size_t temp = p.temp;
  if (!p.wide) {
    auto *keys = reinterpret_cast<unsigned long long *>(p.keys.data());
    auto *sorted = reinterpret_cast<unsigned long long *>(p.sorted.data());
    order_keys64<<<blocks_for(total), 256, 0, s>>>(vox, daf, begin, p.nobj, p.lbits, keys, (int)total);
    ++ctx.launches;
    BK_CUDA(cudaGetLastError());
    BK_CUDA(cub::DeviceRadixSort::SortKeys(p.scratch.data(), temp, keys, sorted, (int)total, 0, p.end_bit, s));
    unpack_order64<<<blocks_for(total), 256, 0, s>>>(sorted, vox, begin, p.lbits, p.order.data(), (int)total);
  } else {
    auto *keys = reinterpret_cast<WideKey *>(p.keys.data());
    auto *sorted = reinterpret_cast<WideKey *>(p.sorted.data());
    order_keys96<<<blocks_for(total), 256, 0, s>>>(vox, daf, begin, p.nobj, p.lbits, keys, (int)total);
    ++ctx.launches;
    BK_CUDA(cudaGetLastError());
    BK_CUDA(cub::DeviceRadixSort::SortKeys(p.scratch.data(), temp, keys, sorted, (int)total, WideKeyParts{}, 0,
                                           p.end_bit, s));
    unpack_order96<<<blocks_for(total), 256, 0, s>>>(sorted, vox, begin, p.lbits, p.order.data(), (int)total);
  }
  ++ctx.launches;
  BK_CUDA(cudaGetLastError());
}

Buffer<int> target_orders(Context &ctx, const int *vox, const float *daf, long long total, const int *begin, int nobj,
                          long long largest, bool wide) {
  OrderPlan p = plan_target_orders(ctx, total, nobj, largest, wide);
  run_target_orders(ctx, p, vox, daf, begin);
  return std::move(p.order);
}

}  // namespace bk
