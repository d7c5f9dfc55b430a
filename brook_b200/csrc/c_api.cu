// The C ABI (include/brook_b200.h): argument checks, input staging into Fortran-ordered device
// buffers, exception -> brook_status mapping with thread-local error text, result handles.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>

#include "../../include/brook_b200.h"
#include "../../include/brook_b200_dlpack.h"
#include "engine.hpp"
#include "common.cuh"
#include "merge.hpp"
#include "post.hpp"
#include "streamed.hpp"
#include "pipeline.hpp"

#ifndef BROOK_B200_VERSION
#define BROOK_B200_VERSION "0.1.0"
#endif

struct brook_context {
  bk::Context value;
  explicit brook_context(int device) : value(device) {}
};

using bk::DeviceStorage;

struct brook_array {
  std::shared_ptr<DeviceStorage> storage;
  brook_volume view{};
  size_t bytes = 0;
  // the array as a tensor for DLPack: extents and strides in elements (a volume: (x, y, z) with
  // x fastest; a skeleton buffer: its row-major (rows, width) or (rows,) form)
  std::vector<int64_t> shape, strides;
};

struct brook_components {
  std::shared_ptr<DeviceStorage> storage;
  brook_volume view{};
  size_t bytes = 0;
  std::vector<int64_t> mapping, roots;
};

struct brook_host_components {
  std::vector<unsigned char> ids;  // narrowed to the smallest of u8 / u16 / u32 that holds the count
  brook_volume view{};
  std::vector<int64_t> mapping, roots;
};

struct brook_skeletons {
  bk::Packed packed;
  // a device result's host copy, made by the first brook_skeletons_get_view
  mutable std::once_flag host_copy;
};

namespace {

thread_local std::string g_error;

template <class F>
brook_status protect(F &&fn) noexcept {
  try {
    g_error.clear();
    fn();
    return BROOK_SUCCESS;
  } catch (const std::invalid_argument &e) {
    g_error = e.what();
    return BROOK_INVALID_ARGUMENT;
  } catch (const std::bad_alloc &e) {
    g_error = e.what();
    return BROOK_OUT_OF_MEMORY;
  } catch (const bk::CudaError &e) {
    g_error = e.what();
    return e.code == cudaErrorMemoryAllocation ? BROOK_OUT_OF_MEMORY : BROOK_CUDA_ERROR;
  } catch (const std::exception &e) {
    g_error = e.what();
    return BROOK_INTERNAL_ERROR;
  } catch (...) {
    g_error = "unknown exception";
    return BROOK_INTERNAL_ERROR;
  }
}

void require(bool ok, const char *what = "null brook argument") {
  if (!ok) throw std::invalid_argument(what);
}

// The slab copies of one staged volume: the events the main stream waits on before it reads a
// slab. On release the host waits for the last one (the caller's buffer is borrowed for the call
// only) and so does the main stream, so that the staged buffer goes back to the context's cache
// (in the main stream's order) only after the copies into it.
struct SlabCopies {
  cudaStream_t main = nullptr;
  bk::Slabs slabs;
  ~SlabCopies() {
    if (!slabs.empty()) {
      cudaEventSynchronize(slabs.back().second);
      cudaStreamWaitEvent(main, slabs.back().second, 0);
    }
    for (auto &s : slabs) cudaEventDestroy(s.second);
  }
};

// A volume gathered into Fortran order on the device (or borrowed when it already is).
struct Staged {
  bk::Buffer<unsigned char> owned;
  bk::DeviceVolume volume;
  std::shared_ptr<SlabCopies> copies;  // released first: the main stream waits for the copies
};

// Host input in page-locked memory is copied in slabs of about this many bytes on the copy
// stream; the components' tile unions start on each slab as it arrives.
constexpr long long kSlabBytes = 64LL << 20;

__global__ void gather_strided(const unsigned char *src, unsigned char *dst, int sx, int sy, int sz, long long s0,
                               long long s1, long long s2, int b) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)sx * sy * sz;
  if (i >= n) return;
  const long long z = i / ((long long)sx * sy), r = i - z * sx * sy, y = r / sx, x = r - y * sx;
  const unsigned char *p = src + x * s0 + y * s1 + z * s2;
  unsigned char *q = dst + i * b;
  for (int k = 0; k < b; ++k) q[k] = p[k];
}

// slabs: host input may arrive by slabs (the caller reads it only through connected_components,
// which waits per slab).
Staged stage(bk::Context &ctx, const brook_volume &v, bool slabs = false) {
  require(v.struct_size >= sizeof(brook_volume) && v.abi_version == BROOK_ABI_VERSION, "incompatible brook_volume");
  require(v.dtype >= BROOK_U8 && v.dtype <= BROOK_I64, "integer labels required");
  for (int a = 0; a < 3; ++a) require(v.shape[a] >= 0 && v.shape[a] < (1LL << 31), "invalid volume shape");
  Staged st;
  st.volume.dtype = int(v.dtype);
  st.volume.d = bk::VolumeDims{int(v.shape[0]), int(v.shape[1]), int(v.shape[2])};
  const long long n = st.volume.d.n();
  require(n < (1LL << 31) - 1, "volumes of 2^31 voxels or more are not supported");
  if (n == 0) return st;
  require(v.data != nullptr);
  const long long b = (long long)bk::label_bytes(v.dtype);
  const long long sx = v.shape[0], sy = v.shape[1], sz = v.shape[2];
  auto matches = [&](long long e0, long long e1, long long e2) {
    return (sx == 1 || v.strides[0] == e0) && (sy == 1 || v.strides[1] == e1) && (sz == 1 || v.strides[2] == e2);
  };
  const bool fortran = matches(b, b * sx, b * sx * sy);
  const bool c_order = matches(b * sy * sz, b * sz, b);
  cudaStream_t s = ctx.stream();
  if (v.memory == BROOK_DEVICE) {
    cudaPointerAttributes attr{};
    BK_CUDA(cudaPointerGetAttributes(&attr, v.data));
    require(attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged, "device volume is not device memory");
    require(attr.type == cudaMemoryTypeManaged || attr.device == ctx.device(), "device volume is on another device");
    if (fortran) { st.volume.data = v.data; return st; }
    st.owned = bk::Buffer<unsigned char>(ctx, n * b);
    gather_strided<<<bk::blocks_for(n), 256, 0, s>>>(static_cast<const unsigned char *>(v.data), st.owned.data(), int(sx),
                                                    int(sy), int(sz), v.strides[0], v.strides[1], v.strides[2], int(b)); ++ctx.launches;
    BK_CUDA(cudaGetLastError());
    st.volume.data = st.owned.data();
    return st;
  }
  require(v.memory == BROOK_HOST, "invalid memory kind");
  st.owned = bk::Buffer<unsigned char>(ctx, n * b);
  bool pinned = false;
  if (fortran && slabs && n * b >= 2 * kSlabBytes && sz >= 16) {
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, v.data) == cudaSuccess) pinned = attr.type == cudaMemoryTypeHost;
    else cudaGetLastError();
  }
  if (pinned) {
    // planes per slab: a multiple of the union tiles' depth (8)
    const long long plane = b * sx * sy;
    const int per = int(std::max(8LL, (kSlabBytes / plane) / 8 * 8));
    cudaStream_t copy = ctx.copy_stream();
    st.copies = std::make_shared<SlabCopies>();
    st.copies->main = s;
    cudaEvent_t ready;  // the staged buffer may be a block the main stream used before
    BK_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    BK_CUDA(cudaEventRecord(ready, s));
    const cudaError_t waited = cudaStreamWaitEvent(copy, ready, 0);
    cudaEventDestroy(ready);
    BK_CUDA(waited);
    for (int z0 = 0; z0 < int(sz); z0 += per) {
      const int z1 = int(std::min<long long>(sz, z0 + per));
      BK_CUDA(cudaMemcpyAsync(st.owned.data() + z0 * plane, static_cast<const unsigned char *>(v.data) + z0 * plane,
                              (z1 - z0) * plane, cudaMemcpyHostToDevice, copy));
      cudaEvent_t e;
      BK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      const cudaError_t recorded = cudaEventRecord(e, copy);
      if (recorded != cudaSuccess) cudaEventDestroy(e);
      BK_CUDA(recorded);
      st.copies->slabs.push_back({z1, e});
    }
    st.volume.slabs = &st.copies->slabs;
  } else if (fortran) {
    BK_CUDA(cudaMemcpyAsync(st.owned.data(), v.data, n * b, cudaMemcpyHostToDevice, s));
  } else if (c_order) {
    bk::Buffer<unsigned char> raw(ctx, n * b);
    BK_CUDA(cudaMemcpyAsync(raw.data(), v.data, n * b, cudaMemcpyHostToDevice, s));
    gather_strided<<<bk::blocks_for(n), 256, 0, s>>>(raw.data(), st.owned.data(), int(sx), int(sy), int(sz), b * sy * sz,
                                                    b * sz, b, int(b)); ++ctx.launches;
    BK_CUDA(cudaGetLastError());
    ctx.synchronize();
  } else {
    std::vector<unsigned char> host(n * b);
    const unsigned char *base = static_cast<const unsigned char *>(v.data);
    for (long long z = 0; z < sz; ++z)
      for (long long y = 0; y < sy; ++y)
        for (long long x = 0; x < sx; ++x)
          std::memcpy(&host[((z * sy + y) * sx + x) * b], base + x * v.strides[0] + y * v.strides[1] + z * v.strides[2], b);
    BK_CUDA(cudaMemcpyAsync(st.owned.data(), host.data(), n * b, cudaMemcpyHostToDevice, s));
    ctx.synchronize();
  }
  st.volume.data = st.owned.data();
  return st;
}

bk::Options options_of(const brook_skeletonize_options *p) {
  require(p->struct_size >= sizeof(brook_skeletonize_options) && p->abi_version == BROOK_ABI_VERSION,
          "incompatible skeletonization options");
  const uint32_t known = BROOK_FIX_BRANCHING | BROOK_FIX_BORDERS | BROOK_FILTER_OBJECTS | BROOK_DEVICE_OUTPUT |
                         BROOK_FILL_HOLES | BROOK_FIX_AVOCADOS;
  require(!(p->flags & ~known), "unknown skeletonization flags");
  if (p->voxel_graph) throw std::invalid_argument("voxel_graph is not supported by this build");
  bk::Options o;
  auto &t = o.teasar;
  t.scale = p->teasar.scale;
  t.constant = p->teasar.constant;
  t.pdrf_scale = p->teasar.pdrf_scale;
  t.pdrf_exponent = p->teasar.pdrf_exponent;
  t.soma_detection = p->teasar.soma_detection_threshold;
  t.soma_acceptance = p->teasar.soma_acceptance_threshold;
  t.soma_scale = p->teasar.soma_invalidation_scale;
  t.soma_constant = p->teasar.soma_invalidation_const;
  if (p->teasar.has_max_paths) t.max_paths = p->teasar.max_paths;
  for (int a = 0; a < 3; ++a) o.anisotropy[a] = p->anisotropy[a];
  o.dust = p->dust_threshold;
  o.fix_branching = (p->flags & BROOK_FIX_BRANCHING) != 0;
  o.fix_borders = (p->flags & BROOK_FIX_BORDERS) != 0;
  o.device_output = (p->flags & BROOK_DEVICE_OUTPUT) != 0;
  o.fill_holes = (p->flags & BROOK_FILL_HOLES) != 0;
  o.fix_avocados = (p->flags & BROOK_FIX_AVOCADOS) != 0;
  if (p->flags & BROOK_FILTER_OBJECTS) {
    require(p->object_ids || !p->object_ids_count);
    o.object_ids = std::vector<int64_t>(p->object_ids, p->object_ids + p->object_ids_count);
  }
  auto points = [](const int64_t *data, size_t count) {
    require(data || !count);
    std::vector<bk::Point> out;
    for (size_t i = 0; i < count; ++i) out.push_back({data[3 * i], data[3 * i + 1], data[3 * i + 2]});
    return out;
  };
  if (p->targets_before_count || p->targets_after_count) {
    o.targets_before.push_back(points(p->targets_before, p->targets_before_count));
    o.targets_after.push_back(points(p->targets_after, p->targets_after_count));
  }
  return o;
}

__global__ void pdrf_values_kernel(const float *dbf, const float *daf, float *out, long long n, float M, float inv,
                                   float scale, int squarings, float exponent) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = bk::pdrf_value(dbf[i], daf[i], M, inv, scale, squarings, exponent);
}

__global__ void narrow_ids(const uint32_t *ids, void *out, long long n, int bytes) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t v = ids[i];
  if (bytes == 1) static_cast<uint8_t *>(out)[i] = uint8_t(v);
  else if (bytes == 2) static_cast<uint16_t *>(out)[i] = uint16_t(v);
  else static_cast<uint32_t *>(out)[i] = v;
}

size_t element_bytes(brook_dtype t) {
  if (t == BROOK_F32) return 4;
  if (t == BROOK_F64) return 8;
  return bk::label_bytes(t);
}

brook_volume device_view(const void *data, brook_dtype dtype, bk::VolumeDims d) {
  brook_volume v{};
  v.struct_size = sizeof(v);
  v.abi_version = BROOK_ABI_VERSION;
  v.data = data;
  v.dtype = dtype;
  v.memory = BROOK_DEVICE;
  v.shape[0] = d.sx; v.shape[1] = d.sy; v.shape[2] = d.sz;
  const size_t b = element_bytes(dtype);
  v.strides[0] = int64_t(b); v.strides[1] = int64_t(b) * d.sx; v.strides[2] = int64_t(b) * d.sx * d.sy;
  return v;
}

// Device view of a row-major (rows x width) array of 4-byte elements: shape (width, rows, 1), x
// (the element within a row) fastest.
brook_volume skeleton_view(const DeviceStorage &s, brook_dtype dtype, int width, size_t rows) {
  brook_volume v{};
  v.struct_size = sizeof(v);
  v.abi_version = BROOK_ABI_VERSION;
  v.data = s.ptr;
  v.dtype = dtype;
  v.memory = BROOK_DEVICE;
  v.shape[0] = width; v.shape[1] = int64_t(rows); v.shape[2] = 1;
  v.strides[0] = 4; v.strides[1] = 4LL * width; v.strides[2] = 4LL * width * int64_t(rows);
  return v;
}

void volume_tensor(brook_array &a) {
  a.shape = {a.view.shape[0], a.view.shape[1], a.view.shape[2]};
  a.strides = {1, a.view.shape[0], a.view.shape[0] * a.view.shape[1]};
}

// A row-major (rows x width) skeleton buffer as a tensor: (rows, width), or (rows,) for width 1.
void rows_tensor(brook_array &a, int width, size_t rows) {
  if (width == 1) { a.shape = {int64_t(rows)}; a.strides = {1}; }
  else { a.shape = {int64_t(rows), width}; a.strides = {width, 1}; }
}

// A Fortran-ordered device copy of any volume (host or device memory, any strides, any of the
// ten element types), in the context's stream order; the host waits for the copy.
brook_array *upload_array(bk::Context &ctx, const brook_volume &v) {
  require(v.struct_size >= sizeof(brook_volume) && v.abi_version == BROOK_ABI_VERSION, "incompatible brook_volume");
  require(v.dtype >= BROOK_U8 && v.dtype <= BROOK_F64, "invalid element type");
  for (int a = 0; a < 3; ++a) require(v.shape[a] >= 0 && v.shape[a] < (1LL << 31), "invalid volume shape");
  const long long sx = v.shape[0], sy = v.shape[1], sz = v.shape[2], n = sx * sy * sz;
  const long long b = (long long)element_bytes(v.dtype);
  auto handle = std::make_unique<brook_array>();
  handle->storage = std::make_shared<DeviceStorage>(size_t(n * b), ctx.device());
  handle->bytes = size_t(n * b);
  handle->view = device_view(handle->storage->ptr, v.dtype, bk::VolumeDims{int(sx), int(sy), int(sz)});
  volume_tensor(*handle);
  if (!n) return handle.release();
  require(v.data != nullptr, "null volume data");
  require(v.memory == BROOK_HOST || v.memory == BROOK_DEVICE, "invalid memory kind");
  auto matches = [&](long long e0, long long e1, long long e2) {
    return (sx == 1 || v.strides[0] == e0) && (sy == 1 || v.strides[1] == e1) && (sz == 1 || v.strides[2] == e2);
  };
  const bool fortran = matches(b, b * sx, b * sx * sy);
  unsigned char *dst = static_cast<unsigned char *>(handle->storage->ptr);
  cudaStream_t s = ctx.stream();
  if (v.memory == BROOK_DEVICE) {
    cudaPointerAttributes attr{};
    BK_CUDA(cudaPointerGetAttributes(&attr, v.data));
    require(attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged, "device volume is not device memory");
    require(attr.type == cudaMemoryTypeManaged || attr.device == ctx.device(), "device volume is on another device");
    if (fortran) BK_CUDA(cudaMemcpyAsync(dst, v.data, n * b, cudaMemcpyDeviceToDevice, s));
    else {
      gather_strided<<<bk::blocks_for(n), 256, 0, s>>>(static_cast<const unsigned char *>(v.data), dst, int(sx), int(sy),
                                                      int(sz), v.strides[0], v.strides[1], v.strides[2], int(b)); ++ctx.launches;
      BK_CUDA(cudaGetLastError());
    }
  } else if (fortran) {
    BK_CUDA(cudaMemcpyAsync(dst, v.data, n * b, cudaMemcpyHostToDevice, s));
  } else {
    std::vector<unsigned char> host(n * b);
    const unsigned char *base = static_cast<const unsigned char *>(v.data);
    for (long long z = 0; z < sz; ++z)
      for (long long y = 0; y < sy; ++y)
        for (long long x = 0; x < sx; ++x)
          std::memcpy(&host[((z * sy + y) * sx + x) * b], base + x * v.strides[0] + y * v.strides[1] + z * v.strides[2], b);
    BK_CUDA(cudaMemcpyAsync(dst, host.data(), n * b, cudaMemcpyHostToDevice, s));
    ctx.synchronize();
  }
  ctx.synchronize();
  return handle.release();
}

// One DLPack export of an array: owns a reference to the array's storage and the extents, so
// that it outlives the array handle and the context; the consumer's call of the deleter frees it.
template <class Tensor>
struct Export {
  Tensor tensor{};
  std::shared_ptr<DeviceStorage> storage;
  std::vector<int64_t> shape, strides;
};

template <class Tensor>
void release_export(Tensor *t) noexcept {
  delete static_cast<Export<Tensor> *>(t->manager_ctx);
}

template <class Tensor>
Tensor *export_array(const brook_array &a) {
  auto e = std::make_unique<Export<Tensor>>();
  e->storage = a.storage;
  e->shape = a.shape;
  e->strides = a.strides;
  e->tensor.manager_ctx = e.get();
  e->tensor.deleter = release_export<Tensor>;
  DLTensor &t = e->tensor.dl_tensor;
  t.data = a.bytes ? a.storage->ptr : nullptr;
  t.device = DLDevice{kDLCUDA, int32_t(a.storage->device)};
  t.ndim = int32_t(e->shape.size());
  t.shape = e->shape.empty() ? nullptr : e->shape.data();
  t.strides = e->strides.empty() ? nullptr : e->strides.data();
  t.byte_offset = 0;
  const brook_dtype d = a.view.dtype;
  const uint8_t code = d <= BROOK_U64 ? kDLUInt : d <= BROOK_I64 ? kDLInt : kDLFloat;
  t.dtype = DLDataType{code, uint8_t(8 * element_bytes(d)), 1};
  return &e.release()->tensor;
}

brook_status skeletonize_many(brook_context *ctx, const brook_volume *volumes, size_t count,
                              const brook_skeletonize_options *p, const brook_sample_targets *targets,
                              brook_skeletons **out) {
  return protect([&] {
    require(ctx && (volumes || !count) && p && out);
    for (size_t i = 0; i < count; ++i) out[i] = nullptr;
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    bk::Options options = options_of(p);
    if (count > 1 && !options.targets_before.empty())
      throw std::invalid_argument("the options' extra targets are for one volume: give a batch its targets per sample "
                                  "(brook_skeletonize_batch_targets)");
    if (targets) {
      require(options.targets_before.empty(), "extra targets are given both in the options and per sample");
      options.targets_before.resize(count);
      options.targets_after.resize(count);
      for (size_t i = 0; i < count; ++i) {
        const brook_sample_targets &t = targets[i];
        require((t.before || !t.before_count) && (t.after || !t.after_count));
        for (size_t k = 0; k < t.before_count; ++k)
          options.targets_before[i].push_back({t.before[3 * k], t.before[3 * k + 1], t.before[3 * k + 2]});
        for (size_t k = 0; k < t.after_count; ++k)
          options.targets_after[i].push_back({t.after[3 * k], t.after[3 * k + 1], t.after[3 * k + 2]});
      }
    }
    std::vector<Staged> staged;
    std::vector<bk::DeviceVolume> vols;
    for (size_t i = 0; i < count; ++i) {
      staged.push_back(stage(ctx->value, volumes[i], true));
      vols.push_back(staged.back().volume);
    }
    auto results = bk::skeletonize(ctx->value, vols, options);
    ctx->value.synchronize();
    std::vector<std::unique_ptr<brook_skeletons>> handles;
    for (auto &r : results) {
      if (options.device_output && !r.on_device()) {  // nothing traced: empty device arrays
        r.device_vertices = std::make_shared<DeviceStorage>(0, ctx->value.device());
        r.device_edges = std::make_shared<DeviceStorage>(0, ctx->value.device());
        r.device_radii = std::make_shared<DeviceStorage>(0, ctx->value.device());
      }
      handles.emplace_back(new brook_skeletons());
      handles.back()->packed = std::move(r);
    }
    for (size_t i = 0; i < count; ++i) out[i] = handles[i].release();
  });
}

}  // namespace

namespace {

// A post-processing call on the context: its statistics and launch count are the call's own.
template <class F>
void post_call(brook_context *ctx, const brook_skeletons *input, F &&body) {
  require(ctx && input);
  std::lock_guard<std::mutex> lock(ctx->value.mutex());
  bk::DeviceGuard guard(ctx->value.device());
  const bk::Packed &p = input->packed;
  if (p.on_device()) require(p.device_vertices->device == ctx->value.device(), "the skeletons are on another device");
  ctx->value.stats.clear();
  ctx->value.launches = 0;
  body(p);
  ctx->value.stats["launches"] = double(ctx->value.launches);
}

}  // namespace

extern "C" {

uint32_t brook_abi_version(void) { return BROOK_ABI_VERSION; }
const char *brook_version(void) { return BROOK_B200_VERSION; }
const char *brook_last_error(void) { return g_error.c_str(); }

brook_status brook_context_create(int device, brook_context **out) {
  return protect([&] {
    require(out);
    *out = nullptr;
    *out = new brook_context(device);
  });
}
void brook_context_destroy(brook_context *ctx) { delete ctx; }
brook_status brook_context_synchronize(brook_context *ctx) {
  return protect([&] {
    require(ctx);
    ctx->value.synchronize();
  });
}

brook_status brook_context_set_engine_share(brook_context *ctx, int percent) {
  return protect([&] {
    require(ctx && percent >= 1 && percent <= 100, "the engine share is a percentage from 1 to 100");
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    ctx->value.engine_percent = percent;
  });
}

brook_status brook_context_trim(brook_context *ctx) {
  return protect([&] {
    require(ctx);
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    ctx->value.trim();
    cudaMemPool_t pool;
    BK_CUDA(cudaDeviceGetDefaultMemPool(&pool, ctx->value.device()));
    BK_CUDA(cudaMemPoolTrimTo(pool, 0));
  });
}

void brook_array_destroy(brook_array *a) { delete a; }
brook_status brook_array_view(const brook_array *a, brook_volume *out) {
  return protect([&] {
    require(a && out);
    *out = a->view;
  });
}
brook_status brook_array_copy_to_host(const brook_array *a, void *out, size_t bytes) {
  return protect([&] {
    require(a && (out || !bytes));
    require(bytes >= a->bytes, "output buffer too small");
    bk::DeviceGuard guard(a->storage->device);
    if (a->bytes) BK_CUDA(cudaMemcpy(out, a->storage->ptr, a->bytes, cudaMemcpyDeviceToHost));
  });
}

brook_status brook_array_upload(brook_context *ctx, const brook_volume *input, brook_array **out) {
  return protect([&] {
    require(ctx && input && out);
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    *out = upload_array(ctx->value, *input);
  });
}

brook_status brook_array_to_dlpack(const brook_array *a, DLManagedTensor **out) {
  return protect([&] {
    require(a && out);
    *out = nullptr;
    *out = export_array<DLManagedTensor>(*a);
  });
}

brook_status brook_array_to_dlpack_versioned(const brook_array *a, uint32_t max_minor, DLManagedTensorVersioned **out) {
  return protect([&] {
    require(a && out);
    *out = nullptr;
    DLManagedTensorVersioned *t = export_array<DLManagedTensorVersioned>(*a);
    t->version = DLPackVersion{DLPACK_MAJOR_VERSION, std::min<uint32_t>(max_minor, DLPACK_MINOR_VERSION)};
    t->flags = 0;  // shared, writable storage: no copy was made
    *out = t;
  });
}

brook_status brook_context_wait_stream(brook_context *ctx, int64_t producer) {
  return protect([&] {
    require(ctx);
    require(producer >= 0, "invalid producer stream handle");
    bk::DeviceGuard guard(ctx->value.device());
    cudaStream_t stream = producer <= 1 ? cudaStreamLegacy
                          : producer == 2 ? cudaStreamPerThread
                                          : reinterpret_cast<cudaStream_t>(static_cast<uintptr_t>(producer));
    cudaEvent_t event = nullptr;
    BK_CUDA(cudaEventCreateWithFlags(&event, cudaEventDisableTiming));
    cudaError_t status = cudaEventRecord(event, stream);
    if (status == cudaSuccess) status = cudaStreamWaitEvent(ctx->value.stream(), event, 0);
    cudaEventDestroy(event);
    BK_CUDA(status);
  });
}

brook_status brook_connected_components(brook_context *ctx, const brook_volume *labels, brook_components **out) {
  return protect([&] {
    require(ctx && labels && out);
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    Staged st = stage(ctx->value, *labels);
    const long long n = st.volume.d.n();
    bk::Buffer<uint32_t> ids(ctx->value, n > 0 ? n : 1);
    auto cc = n ? bk::connected_components(ctx->value, st.volume.data, st.volume.dtype, st.volume.d, ids.data())
                : bk::ComponentsResult{0, {0}, {}};
    const brook_dtype dtype = cc.count <= 0xFF ? BROOK_U8 : cc.count <= 0xFFFF ? BROOK_U16 : BROOK_U32;
    const size_t b = bk::label_bytes(dtype);
    auto handle = std::make_unique<brook_components>();
    handle->storage = std::make_shared<DeviceStorage>(size_t(n) * b, ctx->value.device());
    handle->bytes = size_t(n) * b;
    if (n) {
      narrow_ids<<<bk::blocks_for(n), 256, 0, ctx->value.stream()>>>(ids.data(), handle->storage->ptr, n, int(b)); ++ctx->value.launches;
      BK_CUDA(cudaGetLastError());
    }
    ctx->value.synchronize();
    handle->view = device_view(handle->storage->ptr, dtype, st.volume.d);
    handle->mapping = cc.mapping;
    if (handle->mapping.empty()) handle->mapping.push_back(0);
    handle->roots = cc.roots;
    *out = handle.release();
  });
}
void brook_components_destroy(brook_components *c) { delete c; }
brook_status brook_components_view(const brook_components *c, brook_volume *labels, const int64_t **mapping,
                                   const int64_t **roots, size_t *count) {
  return protect([&] {
    require(c);
    if (labels) *labels = c->view;
    if (mapping) *mapping = c->mapping.data();
    if (roots) *roots = c->roots.data();
    if (count) *count = c->roots.size();
  });
}
brook_status brook_components_labels(const brook_components *c, brook_array **out) {
  return protect([&] {
    require(c && out);
    *out = nullptr;
    auto handle = std::make_unique<brook_array>();
    handle->storage = c->storage;
    handle->view = c->view;
    handle->bytes = c->bytes;
    volume_tensor(*handle);
    *out = handle.release();
  });
}

brook_status brook_components_copy_to_host(const brook_components *c, void *out, size_t bytes) {
  return protect([&] {
    require(c && (out || !bytes));
    require(bytes >= c->bytes, "output buffer too small");
    bk::DeviceGuard guard(c->storage->device);
    if (c->bytes) BK_CUDA(cudaMemcpy(out, c->storage->ptr, c->bytes, cudaMemcpyDeviceToHost));
  });
}

brook_status brook_edt(brook_context *ctx, const brook_volume *labels, const float anisotropy[3], int black_border,
                       brook_array **out) {
  return protect([&] {
    require(ctx && labels && anisotropy && out);
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    Staged st = stage(ctx->value, *labels);
    const long long n = st.volume.d.n();
    auto handle = std::make_unique<brook_array>();
    handle->storage = std::make_shared<DeviceStorage>(size_t(n) * 4, ctx->value.device());
    handle->bytes = size_t(n) * 4;
    if (n) {
      bk::Buffer<uint32_t> ids(ctx->value, n);
      bk::connected_components(ctx->value, st.volume.data, st.volume.dtype, st.volume.d, ids.data());
      bk::edt(ctx->value, ids.data(), st.volume.d, anisotropy, black_border != 0, 3,
              static_cast<float *>(handle->storage->ptr));
    }
    ctx->value.synchronize();
    handle->view = device_view(handle->storage->ptr, BROOK_F32, st.volume.d);
    volume_tensor(*handle);
    *out = handle.release();
  });
}

void brook_skeletonize_options_init(brook_skeletonize_options *p) {
  if (!p) return;
  *p = brook_skeletonize_options{};
  p->struct_size = sizeof(*p);
  p->abi_version = BROOK_ABI_VERSION;
  p->teasar.scale = 1.5;
  p->teasar.constant = 300;
  p->teasar.pdrf_scale = 100000;
  p->teasar.pdrf_exponent = 4;
  p->teasar.soma_detection_threshold = 750;
  p->teasar.soma_acceptance_threshold = 3500;
  p->teasar.soma_invalidation_scale = 2;
  p->teasar.soma_invalidation_const = 300;
  p->anisotropy[0] = p->anisotropy[1] = p->anisotropy[2] = 1;
  p->dust_threshold = 1000;
  p->flags = BROOK_FIX_BRANCHING | BROOK_FIX_BORDERS;
}

brook_status brook_skeletonize(brook_context *ctx, const brook_volume *labels, const brook_skeletonize_options *p,
                               brook_skeletons **out) {
  if (!labels) return protect([] { require(false); });
  return skeletonize_many(ctx, labels, 1, p, nullptr, out);
}

brook_status brook_skeletonize_batch(brook_context *ctx, const brook_volume *volumes, size_t count,
                                     const brook_skeletonize_options *p, brook_skeletons **out) {
  return skeletonize_many(ctx, volumes, count, p, nullptr, out);
}

brook_status brook_skeletonize_batch_targets(brook_context *ctx, const brook_volume *volumes, size_t count,
                                             const brook_skeletonize_options *p, const brook_sample_targets *targets,
                                             brook_skeletons **out) {
  return skeletonize_many(ctx, volumes, count, p, targets, out);
}

brook_status brook_skeletons_get_view(const brook_skeletons *r, brook_skeletons_view *out) {
  return protect([&] {
    require(r && out);
    if (r->packed.on_device()) {  // a device result: one host copy, made on first use
      std::call_once(r->host_copy, [&] {
        auto &p = const_cast<bk::Packed &>(r->packed);
        bk::DeviceGuard guard(p.device_vertices->device);
        p.vertices.resize(p.device_vertices->bytes / sizeof(float));
        p.radii.resize(p.device_radii->bytes / sizeof(float));
        p.edges.resize(p.device_edges->bytes / sizeof(uint32_t));
        if (!p.vertices.empty()) BK_CUDA(cudaMemcpy(p.vertices.data(), p.device_vertices->ptr, p.device_vertices->bytes, cudaMemcpyDeviceToHost));
        if (!p.radii.empty()) BK_CUDA(cudaMemcpy(p.radii.data(), p.device_radii->ptr, p.device_radii->bytes, cudaMemcpyDeviceToHost));
        if (!p.edges.empty()) BK_CUDA(cudaMemcpy(p.edges.data(), p.device_edges->ptr, p.device_edges->bytes, cudaMemcpyDeviceToHost));
      });
    }
    const auto &p = r->packed;
    out->skeleton_count = p.labels.size();
    out->vertex_count = p.radii.size();
    out->edge_count = p.edges.size() / 2;
    out->labels = p.labels.data();
    out->vertex_offsets = p.vertex_offsets.data();
    out->edge_offsets = p.edge_offsets.data();
    out->vertices = p.vertices.data();
    out->edges = p.edges.data();
    out->radii = p.radii.data();
    for (int a = 0; a < 3; ++a) out->anisotropy[a] = p.anisotropy[a];
  });
}
void brook_skeletons_destroy(brook_skeletons *r) { delete r; }

brook_status brook_skeletons_get_device_view(const brook_skeletons *r, brook_skeletons_device_view *out) {
  return protect([&] {
    require(r && out);
    *out = {};
    const auto &p = r->packed;
    if (!p.on_device()) throw std::invalid_argument("skeleton result was not requested with BROOK_DEVICE_OUTPUT");
    out->skeleton_count = p.labels.size();
    out->vertex_count = size_t(p.vertex_offsets.back());
    out->edge_count = size_t(p.edge_offsets.back());
    out->labels = p.labels.data();
    out->vertex_offsets = p.vertex_offsets.data();
    out->edge_offsets = p.edge_offsets.data();
    out->vertices = skeleton_view(*p.device_vertices, BROOK_F32, 3, out->vertex_count);
    out->edges = skeleton_view(*p.device_edges, BROOK_U32, 2, out->edge_count);
    out->radii = skeleton_view(*p.device_radii, BROOK_F32, 1, out->vertex_count);
    for (int a = 0; a < 3; ++a) out->anisotropy[a] = p.anisotropy[a];
  });
}

brook_status brook_skeletons_get_array(const brook_skeletons *r, brook_skeleton_buffer buffer, brook_array **out) {
  return protect([&] {
    require(r && out);
    *out = nullptr;
    const auto &p = r->packed;
    if (!p.on_device()) throw std::invalid_argument("skeleton result was not requested with BROOK_DEVICE_OUTPUT");
    const size_t V = size_t(p.vertex_offsets.back()), E = size_t(p.edge_offsets.back());
    auto handle = std::make_unique<brook_array>();
    switch (buffer) {
      case BROOK_VERTICES:
        handle->storage = p.device_vertices; handle->view = skeleton_view(*p.device_vertices, BROOK_F32, 3, V);
        rows_tensor(*handle, 3, V);
        break;
      case BROOK_EDGES:
        handle->storage = p.device_edges; handle->view = skeleton_view(*p.device_edges, BROOK_U32, 2, E);
        rows_tensor(*handle, 2, E);
        break;
      case BROOK_RADII:
        handle->storage = p.device_radii; handle->view = skeleton_view(*p.device_radii, BROOK_F32, 1, V);
        rows_tensor(*handle, 1, V);
        break;
      default: throw std::invalid_argument("invalid skeleton buffer");
    }
    handle->bytes = handle->storage->bytes;
    *out = handle.release();
  });
}

brook_status brook_edt_device_noalloc(const brook_volume *labels, const float anisotropy[3], int black_border,
                                      float *out, void *stream) {
  return protect([&] {
    require(labels && anisotropy && out);
    const brook_volume &v = *labels;
    require(v.struct_size >= sizeof(brook_volume) && v.abi_version == BROOK_ABI_VERSION, "incompatible brook_volume");
    require(v.memory == BROOK_DEVICE, "brook_edt_device_noalloc reads device memory (memory = BROOK_DEVICE)");
    require(v.dtype == BROOK_U32, "brook_edt_device_noalloc takes uint32 labels");
    for (int a = 0; a < 3; ++a) require(v.shape[a] >= 0 && v.shape[a] < (1LL << 31), "invalid volume shape");
    const bk::VolumeDims d{int(v.shape[0]), int(v.shape[1]), int(v.shape[2])};
    require(d.n() < (1LL << 31) - 1, "volumes of 2^31 voxels or more are not supported");
    if (d.n() == 0) return;
    require(v.data != nullptr);
    const long long sx = v.shape[0], sy = v.shape[1], sz = v.shape[2];
    require((sx == 1 || v.strides[0] == 4) && (sy == 1 || v.strides[1] == 4 * sx) && (sz == 1 || v.strides[2] == 4 * sx * sy),
            "brook_edt_device_noalloc takes Fortran-contiguous labels");
    int device = 0;
    BK_CUDA(cudaGetDevice(&device));
    for (const void *p : {v.data, static_cast<const void *>(out)}) {
      cudaPointerAttributes attr{};
      BK_CUDA(cudaPointerGetAttributes(&attr, p));
      require(attr.type == cudaMemoryTypeManaged || (attr.type == cudaMemoryTypeDevice && attr.device == device),
              "labels and output must be device memory of the current device");
    }
    bk::edt_fixed_scratch(static_cast<const uint32_t *>(v.data), d, anisotropy, black_border != 0, out,
                          static_cast<cudaStream_t>(stream));
  });
}

namespace {
bk::Tuning tuning_of(const brook_tuning &t) {
  bk::Tuning out;
  out.trace_cluster_ctas = t.trace_cluster_ctas;
  out.trace_cluster_voxels = t.trace_cluster_voxels;
  out.prepare_cluster_voxels = t.prepare_cluster_voxels;
  out.lone_first_percent = t.lone_first_percent;
  return out;
}
brook_tuning tuning_to_c(const bk::Tuning &t) {
  brook_tuning out{};
  out.trace_cluster_ctas = t.trace_cluster_ctas;
  out.trace_cluster_voxels = t.trace_cluster_voxels;
  out.prepare_cluster_voxels = t.prepare_cluster_voxels;
  out.lone_first_percent = t.lone_first_percent;
  return out;
}
}  // namespace

brook_status brook_autotune(brook_context *ctx, const brook_volume *volumes, size_t count,
                            const brook_skeletonize_options *p, uint64_t *workload_class, brook_tuning *best,
                            double *best_ms) {
  return protect([&] {
    require(ctx && (volumes || !count) && p);
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    bk::Context &c = ctx->value;
    const bk::Options options = options_of(p);
    std::vector<Staged> staged;
    std::vector<bk::DeviceVolume> vols;
    for (size_t i = 0; i < count; ++i) {
      staged.push_back(stage(c, volumes[i]));
      vols.push_back(staged.back().volume);
    }
    // one candidate: the engine's device time (prepare, target orders, trace), best of two calls
    auto measure = [&](const bk::Tuning &t) {
      double ms = INFINITY;
      for (int rep = 0; rep < 2; ++rep) {
        c.forced = &t;
        try {
          bk::skeletonize(c, vols, options);
        } catch (...) {
          c.forced = nullptr;
          throw;
        }
        c.forced = nullptr;
        c.synchronize();
        ms = std::min(ms, c.stats["ms_prepare"] + c.stats["ms_order"] + c.stats["ms_trace"]);
      }
      return ms;
    };
    bk::Tuning chosen;
    double chosen_ms = measure(chosen);  // the built-in rule
    const unsigned long long cls = c.last_class;
    const double foreground = c.stats["foreground"];
    auto consider = [&](bk::Tuning t) {
      const double ms = measure(t);
      if (ms < chosen_ms) { chosen_ms = ms; chosen = t; }
    };
    // coordinate search: cluster width, the trace's cluster threshold, the lone-first share, the
    // preparation's cluster threshold
    for (int ctas : {bk::kClusterCtas, bk::kWideClusterCtas}) {
      bk::Tuning t = chosen;
      t.trace_cluster_ctas = ctas;
      consider(t);
    }
    const long long rule = bk::trace_cluster_voxels((long long)foreground);
    for (double f : {0.5, 2.0, 4.0}) {
      bk::Tuning t = chosen;
      t.trace_cluster_voxels = std::max(1LL, (long long)(double(rule) * f));
      consider(t);
    }
    for (int percent : {0, 25}) {
      bk::Tuning t = chosen;
      t.lone_first_percent = percent;
      consider(t);
    }
    for (long long v : {4096LL, 32768LL}) {
      bk::Tuning t = chosen;
      t.prepare_cluster_voxels = v;
      consider(t);
    }
    c.tuning[cls] = chosen;
    c.stats["autotune_ms"] = chosen_ms;
    if (workload_class) *workload_class = cls;
    if (best) *best = tuning_to_c(chosen);
    if (best_ms) *best_ms = chosen_ms;
  });
}

brook_status brook_skeletons_create(const brook_skeletons_view *v, brook_skeletons **out) {
  return protect([&] {
    require(v && out);
    *out = nullptr;
    const size_t k = v->skeleton_count, nv = v->vertex_count, ne = v->edge_count;
    require((v->labels || !k) && v->vertex_offsets && v->edge_offsets, "incomplete skeletons view");
    require((v->vertices && v->radii) || !nv, "incomplete skeletons view");
    require(v->edges || !ne, "incomplete skeletons view");
    require(v->vertex_offsets[0] == 0 && v->edge_offsets[0] == 0 && size_t(v->vertex_offsets[k]) == nv &&
                size_t(v->edge_offsets[k]) == ne,
            "inconsistent skeleton offsets");
    auto handle = std::make_unique<brook_skeletons>();
    bk::Packed &p = handle->packed;
    p.labels.assign(v->labels, v->labels + k);
    p.vertex_offsets.assign(v->vertex_offsets, v->vertex_offsets + k + 1);
    p.edge_offsets.assign(v->edge_offsets, v->edge_offsets + k + 1);
    for (size_t i = 0; i < k; ++i)
      require(p.vertex_offsets[i] <= p.vertex_offsets[i + 1] && p.edge_offsets[i] <= p.edge_offsets[i + 1],
              "inconsistent skeleton offsets");
    p.vertices.assign(v->vertices, v->vertices + 3 * nv);
    p.radii.assign(v->radii, v->radii + nv);
    p.edges.assign(v->edges, v->edges + 2 * ne);
    for (int a = 0; a < 3; ++a) p.anisotropy[a] = v->anisotropy[a];
    *out = handle.release();
  });
}

// A host volume of integer labels for the streamed entry points.
bk::HostVolume host_labels(const brook_volume *v) {
  require(v, "null volume");
  require(v->struct_size >= sizeof(brook_volume) && v->abi_version == BROOK_ABI_VERSION, "incompatible brook_volume");
  require(v->memory == BROOK_HOST, "streamed calls take host volumes");
  require(v->dtype >= BROOK_U8 && v->dtype <= BROOK_I64, "integer labels required");
  for (int a = 0; a < 3; ++a) require(v->shape[a] >= 0 && v->shape[a] < (1LL << 31), "invalid volume shape");
  bk::HostVolume hv;
  hv.data = v->data;
  hv.dtype = int(v->dtype);
  hv.d = bk::VolumeDims{int(v->shape[0]), int(v->shape[1]), int(v->shape[2])};
  for (int a = 0; a < 3; ++a) hv.strides[a] = v->strides[a];
  require(hv.data || hv.d.n() == 0);
  return hv;
}

brook_status brook_connected_components_streamed(brook_context *ctx, const brook_volume *labels, size_t budget_bytes,
                                                 brook_host_components **out) {
  return protect([&] {
    require(ctx && labels && out);
    *out = nullptr;
    const bk::HostVolume hv = host_labels(labels);
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    ctx->value.stats.clear();
    ctx->value.launches = 0;
    auto cc = bk::connected_components_streamed(ctx->value, hv, bk::stream_budget(budget_bytes), nullptr);
    auto handle = std::make_unique<brook_host_components>();
    const brook_dtype dtype = cc.count <= 0xFF ? BROOK_U8 : cc.count <= 0xFFFF ? BROOK_U16 : BROOK_U32;
    const size_t b = bk::label_bytes(dtype), n = cc.ids.size();
    handle->ids.resize(n * b);
    if (b == 4) std::memcpy(handle->ids.data(), cc.ids.data(), n * 4);
    else if (b == 2) for (size_t i = 0; i < n; ++i) reinterpret_cast<uint16_t *>(handle->ids.data())[i] = uint16_t(cc.ids[i]);
    else for (size_t i = 0; i < n; ++i) handle->ids[i] = uint8_t(cc.ids[i]);
    brook_volume &v = handle->view;
    v.struct_size = sizeof(v);
    v.abi_version = BROOK_ABI_VERSION;
    v.data = handle->ids.data();
    v.dtype = dtype;
    v.memory = BROOK_HOST;
    v.shape[0] = hv.d.sx; v.shape[1] = hv.d.sy; v.shape[2] = hv.d.sz;
    v.strides[0] = int64_t(b); v.strides[1] = int64_t(b) * hv.d.sx; v.strides[2] = int64_t(b) * hv.d.sx * hv.d.sy;
    handle->mapping = std::move(cc.mapping);
    handle->roots = std::move(cc.roots);
    ctx->value.stats["streamed_slabs"] = cc.slabs;
    ctx->value.stats["launches"] = double(ctx->value.launches);
    *out = handle.release();
  });
}

void brook_host_components_destroy(brook_host_components *c) { delete c; }

brook_status brook_host_components_view(const brook_host_components *c, brook_volume *labels, const int64_t **mapping,
                                        const int64_t **roots, size_t *count) {
  return protect([&] {
    require(c);
    if (labels) *labels = c->view;
    if (mapping) *mapping = c->mapping.data();
    if (roots) *roots = c->roots.data();
    if (count) *count = c->roots.size();
  });
}

brook_status brook_edt_streamed(brook_context *ctx, const brook_volume *labels, const float anisotropy[3],
                                int black_border, size_t budget_bytes, float *output, size_t output_bytes) {
  return protect([&] {
    require(ctx && labels && anisotropy);
    const bk::HostVolume hv = host_labels(labels);
    const size_t n = size_t(hv.d.n());
    require(output_bytes / sizeof(float) >= n && (output || !n), "the output does not hold the volume's float32 field");
    const size_t in_bytes = n * bk::label_bytes(hv.dtype);
    const auto *a = static_cast<const unsigned char *>(hv.data), *o = reinterpret_cast<const unsigned char *>(output);
    require(!n || o + n * sizeof(float) <= a || a + in_bytes <= o, "input and output overlap");
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    ctx->value.stats.clear();
    ctx->value.launches = 0;
    bk::edt_streamed(ctx->value, hv, anisotropy, black_border != 0, budget_bytes, output);
    ctx->value.stats["launches"] = double(ctx->value.launches);
  });
}

brook_status brook_skeletonize_streamed(brook_context *ctx, const brook_volume *labels,
                                        const brook_skeletonize_options *p, size_t budget_bytes,
                                        brook_skeletons **out) {
  return protect([&] {
    require(ctx && labels && p && out);
    *out = nullptr;
    const bk::HostVolume hv = host_labels(labels);
    const bk::Options options = options_of(p);
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    auto handle = std::make_unique<brook_skeletons>();
    handle->packed = bk::skeletonize_streamed(ctx->value, hv, options, budget_bytes);
    *out = handle.release();
  });
}

brook_status brook_skeletons_create_device(brook_context *ctx, const brook_skeletons_device_view *v,
                                           brook_skeletons **out) {
  return protect([&] {
    require(ctx && v && out);
    *out = nullptr;
    const size_t k = v->skeleton_count, nv = v->vertex_count, ne = v->edge_count;
    require((v->labels || !k) && v->vertex_offsets && v->edge_offsets, "incomplete skeletons view");
    require(v->vertex_offsets[0] == 0 && v->edge_offsets[0] == 0 && size_t(v->vertex_offsets[k]) == nv &&
                size_t(v->edge_offsets[k]) == ne,
            "inconsistent skeleton offsets");
    for (size_t i = 0; i < k; ++i)
      require(v->vertex_offsets[i] <= v->vertex_offsets[i + 1] && v->edge_offsets[i] <= v->edge_offsets[i + 1],
              "inconsistent skeleton offsets");
    // row-major device arrays: (3, V), (2, E), (1, V) elements of 4 bytes
    auto check_rows = [&](const brook_volume &a, brook_dtype dtype, int width, size_t rows) {
      require(a.struct_size >= sizeof(brook_volume) && a.abi_version == BROOK_ABI_VERSION, "incompatible brook_volume");
      if (!rows) return;
      require(a.data && a.memory == BROOK_DEVICE && a.dtype == dtype, "skeleton arrays must be device arrays");
      require(a.shape[0] == width && size_t(a.shape[1]) == rows && a.strides[0] == 4 && a.strides[1] == 4LL * width,
              "skeleton arrays must be row major and contiguous");
    };
    check_rows(v->vertices, BROOK_F32, 3, nv);
    check_rows(v->edges, BROOK_U32, 2, ne);
    check_rows(v->radii, BROOK_F32, 1, nv);
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    auto handle = std::make_unique<brook_skeletons>();
    bk::Packed &p = handle->packed;
    p.labels.assign(v->labels, v->labels + k);
    p.vertex_offsets.assign(v->vertex_offsets, v->vertex_offsets + k + 1);
    p.edge_offsets.assign(v->edge_offsets, v->edge_offsets + k + 1);
    for (int a = 0; a < 3; ++a) p.anisotropy[a] = v->anisotropy[a];
    const int dev = ctx->value.device();
    p.device_vertices = std::make_shared<DeviceStorage>(nv * 3 * sizeof(float), dev);
    p.device_edges = std::make_shared<DeviceStorage>(ne * 2 * sizeof(uint32_t), dev);
    p.device_radii = std::make_shared<DeviceStorage>(nv * sizeof(float), dev);
    cudaStream_t st = ctx->value.stream();
    if (nv) {
      BK_CUDA(cudaMemcpyAsync(p.device_vertices->ptr, v->vertices.data, nv * 3 * sizeof(float), cudaMemcpyDeviceToDevice, st));
      BK_CUDA(cudaMemcpyAsync(p.device_radii->ptr, v->radii.data, nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
    if (ne) BK_CUDA(cudaMemcpyAsync(p.device_edges->ptr, v->edges.data, ne * 2 * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    ctx->value.synchronize();
    *out = handle.release();
  });
}

brook_status brook_merge_skeletons(brook_context *ctx, const brook_skeletons *const *fragments, const float *origins,
                                   size_t count, brook_skeletons **out) {
  return protect([&] {
    require(ctx && out && (fragments || !count));
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    std::vector<const bk::Packed *> parts;
    std::vector<std::array<float, 3>> shifts;
    for (size_t i = 0; i < count; ++i) {
      require(fragments[i] != nullptr);
      const bk::Packed &p = fragments[i]->packed;
      if (p.on_device()) require(p.device_vertices->device == ctx->value.device(), "a fragment is on another device");
      parts.push_back(&p);
      shifts.push_back(origins ? std::array<float, 3>{origins[3 * i], origins[3 * i + 1], origins[3 * i + 2]}
                               : std::array<float, 3>{0, 0, 0});
    }
    auto handle = std::make_unique<brook_skeletons>();
    handle->packed = bk::merge_fragments(ctx->value, parts, shifts);
    *out = handle.release();
  });
}

brook_status brook_postprocess_canonical(brook_context *ctx, const brook_skeletons *input, double dust_threshold,
                                         double tick_threshold, brook_skeletons **out) {
  return protect([&] {
    require(out);
    *out = nullptr;
    post_call(ctx, input, [&](const bk::Packed &p) {
      auto handle = std::make_unique<brook_skeletons>();
      handle->packed = bk::post_process(ctx->value, p, bk::kPostprocess, dust_threshold, tick_threshold);
      *out = handle.release();
    });
  });
}

brook_status brook_postprocess_step(brook_context *ctx, const brook_skeletons *input, int step, double threshold,
                                    brook_skeletons **out) {
  return protect([&] {
    require(out);
    *out = nullptr;
    require(step >= BROOK_POST_REMOVE_DUST && step <= BROOK_POST_PRUNE_UNUSED, "unknown post-processing step");
    post_call(ctx, input, [&](const bk::Packed &p) {
      auto handle = std::make_unique<brook_skeletons>();
      handle->packed = bk::post_process(ctx->value, p, step, threshold, 0.0);
      *out = handle.release();
    });
  });
}

brook_status brook_skeleton_components(brook_context *ctx, const brook_skeletons *input, brook_array **out) {
  return protect([&] {
    require(out);
    *out = nullptr;
    post_call(ctx, input, [&](const bk::Packed &p) {
      size_t n = 0;
      auto handle = std::make_unique<brook_array>();
      handle->storage = bk::skeleton_components(ctx->value, p, &n);
      brook_volume v{};
      v.struct_size = sizeof(v);
      v.abi_version = BROOK_ABI_VERSION;
      v.data = handle->storage->ptr;
      v.dtype = BROOK_I64;
      v.memory = BROOK_DEVICE;
      v.shape[0] = 1; v.shape[1] = int64_t(n); v.shape[2] = 1;
      v.strides[0] = 8; v.strides[1] = 8; v.strides[2] = 8LL * int64_t(n);
      handle->view = v;
      handle->bytes = n * sizeof(int64_t);
      rows_tensor(*handle, 1, n);
      *out = handle.release();
    });
  });
}

brook_status brook_pdrf_values(brook_context *ctx, const float *dbf, const float *daf, size_t n, double maximum,
                               double max_daf, double scale, double exponent, float *out) {
  return protect([&] {
    require(ctx && ((dbf && daf && out) || !n));
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    bk::DeviceGuard guard(ctx->value.device());
    if (!n) return;
    // the engine's per-object constants (the reference's pdrf, trace_primitives.cu:119-129)
    const float M = float(1.0 / std::pow(maximum, 1.01));
    const float inv = max_daf != 0 ? float(1.0 / max_daf) : 0.0f;
    int squarings = -1;
    if (exponent > 0 && exponent < 65536 && std::floor(exponent) == exponent && !(int(exponent) & (int(exponent) - 1))) {
      squarings = 0;
      for (int e = int(exponent); e > 1; e >>= 1) ++squarings;
    }
    bk::Buffer<float> d_dbf(ctx->value, n), d_daf(ctx->value, n), d_out(ctx->value, n);
    d_dbf.upload(dbf, n);
    d_daf.upload(daf, n);
    pdrf_values_kernel<<<bk::blocks_for((long long)n), 256, 0, ctx->value.stream()>>>(
        d_dbf.data(), d_daf.data(), d_out.data(), (long long)n, M, inv, float(scale), squarings, float(exponent));
    ++ctx->value.launches;
    BK_CUDA(cudaGetLastError());
    BK_CUDA(cudaMemcpyAsync(out, d_out.data(), n * sizeof(float), cudaMemcpyDeviceToHost, ctx->value.stream()));
    ctx->value.synchronize();
  });
}

brook_status brook_context_set_tuning(brook_context *ctx, uint64_t workload_class, const brook_tuning *t) {
  return protect([&] {
    require(ctx);
    std::lock_guard<std::mutex> lock(ctx->value.mutex());
    if (t) ctx->value.tuning[workload_class] = tuning_of(*t);
    else ctx->value.tuning.erase(workload_class);
  });
}

brook_status brook_context_stats(brook_context *ctx, char *json, size_t capacity, size_t *length) {
  return protect([&] {
    require(ctx);
    std::string out = "{";
    bool first = true;
    // the context's own memory at the time of the query beside the last call's figures
    auto stats = ctx->value.stats;
    stats["context_cached_bytes"] = double(ctx->value.cached_bytes());
    stats["context_live_bytes"] = double(ctx->value.live_bytes());
    for (const auto &kv : stats) {
      char value[64];
      std::snprintf(value, sizeof(value), "%.17g", kv.second);
      out += (first ? "\"" : ", \"") + kv.first + "\": " + value;
      first = false;
    }
    out += "}";
    if (length) *length = out.size() + 1;
    if (json && capacity) {
      const size_t n = std::min(capacity - 1, out.size());
      std::memcpy(json, out.data(), n);
      json[n] = 0;
    }
  });
}

}  // extern "C"
