// Out-of-core skeletonization: the reference's streamed mode (brook_skeletonize_streamed and
// brook_connected_components_streamed, cpp/include/brook/brook.h:173-206; streaming_ccl.cu and
// streaming_trace.cu:99-162 of giorgioangel/brook) for host volumes whose in-core state does not fit
// on the device.
//
// Components: z-slabs sized to the budget go through the in-core CCL one after another (labels
// copied straight from the caller's memory or gathered on the host, ids copied back to host memory); the seam between two slabs
// gives the pairs (id in the last plane of one, id in the first plane of the next) of 26-adjacent
// voxels with the same label, one kernel and one radix sort per seam; a union-find over the slabs'
// ids on the host, by smallest (slab, id), numbers the components by ascending first flat index,
// which is the in-core numbering; the host id volume is renumbered in place by threads.
// Skeletons: each traced component (more voxels than dust, a box of two or more voxels) runs in its
// bounding box as a crop of its own voxels. A crop's EDT has a wall on every face where the box is
// inside the volume (the voxels beyond belong to other components or the background) and the
// volume's black-border rule where the box meets the volume's edge, so its distances are the whole
// volume's; its border targets come from the six faces of the whole volume (planar stage over a
// face stack built on the host), its extra targets by the component they fall on; vertices come out
// in the volume's frame. Crops run batched (the in-core pipeline, one call per batch) within the
// budget, and the crops' skeletons are merged per label on the device (same points, same
// consolidation: the in-core skeletons), labels in the in-core order.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>

#include "merge.hpp"
#include "streamed.hpp"

namespace bk {
namespace {

using u64 = unsigned long long;

template <class F>
void parallel_for(long long n, F &&fn) {
  const long long threads = std::max(1LL, std::min<long long>(n, std::thread::hardware_concurrency()));
  if (threads <= 1) {
    for (long long i = 0; i < n; ++i) fn(i);
    return;
  }
  std::vector<std::thread> pool;
  for (long long t = 0; t < threads; ++t)
    pool.emplace_back([&, t] {
      for (long long i = t; i < n; i += threads) fn(i);
    });
  for (auto &th : pool) th.join();
}

// A large copy split over the host's threads.
void parallel_copy(void *dst, const void *src, size_t bytes) {
  const size_t piece = size_t(16) << 20;
  const long long pieces = (long long)((bytes + piece - 1) / piece);
  parallel_for(pieces, [&](long long k) {
    const size_t at = size_t(k) * piece;
    std::memcpy(static_cast<char *>(dst) + at, static_cast<const char *>(src) + at, std::min(piece, bytes - at));
  });
}

// z planes [z0, z1) of the host volume into an F-ordered buffer.
void gather_slab(const HostVolume &hv, int z0, int z1, unsigned char *dst) {
  const size_t b = label_bytes(hv.dtype), sx = size_t(hv.d.sx), sy = size_t(hv.d.sy);
  const auto *src = static_cast<const unsigned char *>(hv.data);
  const auto &st = hv.strides;
  if (st[0] == (long long)b && st[1] == (long long)(b * sx) && st[2] == (long long)(b * sx * sy)) {
    parallel_copy(dst, src + size_t(z0) * sx * sy * b, size_t(z1 - z0) * sx * sy * b);
    return;
  }
  parallel_for(z1 - z0, [&](long long k) {
    const long long z = z0 + k;
    for (size_t y = 0; y < sy; ++y) {
      unsigned char *out = dst + ((size_t(k) * sy + y) * sx) * b;
      const unsigned char *row = src + z * st[2] + (long long)y * st[1];
      if (st[0] == (long long)b) {
        std::memcpy(out, row, sx * b);
      } else {
        for (size_t x = 0; x < sx; ++x) std::memcpy(out + x * b, row + (long long)x * st[0], b);
      }
    }
  });
}

// The 26-adjacent same-label pairs across a seam: voxel (x, y) of the next slab's first plane and
// (x + dx, y + dy) of the previous slab's last plane, as (previous id << 32 | next id); all ones
// where there is none.
template <class T>
__global__ void seam_pairs(const T *prev_labels, const uint32_t *prev_ids, const T *next_labels,
                           const uint32_t *next_ids, int sx, int sy, u64 *pairs) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)sx * sy) return;
  u64 *out = pairs + 9 * i;
  for (int k = 0; k < 9; ++k) out[k] = ~0ull;
  const T l = next_labels[i];
  if (l == T(0)) return;
  const int x = int(i % sx), y = int(i / sx);
  const u64 id = next_ids[i];
  int k = 0;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx) {
      const int px = x + dx, py = y + dy;
      if (px < 0 || py < 0 || px >= sx || py >= sy) continue;
      const long long j = px + (long long)sx * py;
      if (prev_labels[j] == l) out[k++] = (u64(prev_ids[j]) << 32) | id;
    }
}

void launch_seam(Context &ctx, int dtype, const void *prev_labels, const uint32_t *prev_ids, const void *next_labels,
                 const uint32_t *next_ids, int sx, int sy, u64 *pairs) {
  const long long plane = (long long)sx * sy;
  const unsigned grid = blocks_for(plane);
  cudaStream_t s = ctx.stream();
#define BK_SEAM(T)                                                                                              \
  seam_pairs<T><<<grid, 256, 0, s>>>(static_cast<const T *>(prev_labels), prev_ids,                             \
                                      static_cast<const T *>(next_labels), next_ids, sx, sy, pairs)
  switch (dtype) {
    case U8: BK_SEAM(uint8_t); break;
    case U16: BK_SEAM(uint16_t); break;
    case U32: BK_SEAM(uint32_t); break;
    case U64: BK_SEAM(uint64_t); break;
    case I8: BK_SEAM(int8_t); break;
    case I16: BK_SEAM(int16_t); break;
    case I32: BK_SEAM(int32_t); break;
    case I64: BK_SEAM(int64_t); break;
    default: throw std::invalid_argument("integer labels required");
  }
#undef BK_SEAM
  ++ctx.launches;
  BK_CUDA(cudaGetLastError());
}

struct UnionFind {
  std::vector<int64_t> parent;
  explicit UnionFind(size_t n) : parent(n) { std::iota(parent.begin(), parent.end(), 0); }
  int64_t find(int64_t x) {
    while (parent[x] != x) x = parent[x] = parent[parent[x]];
    return x;
  }
  void unite(int64_t a, int64_t b) {
    a = find(a);
    b = find(b);
    if (a != b) parent[std::max(a, b)] = std::min(a, b);
  }
};

double ms_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

}  // namespace

size_t stream_budget(size_t requested) {
  if (requested) return requested;  // a slab is at least one plane and a batch one crop, whatever it says
  if (const char *env = std::getenv("BROOK_STREAM_BUDGET_MB")) {
    char *end = nullptr;
    const unsigned long long mb = std::strtoull(env, &end, 10);
    if (!*env || *end || mb == 0 || mb > (~size_t(0) >> 20))
      throw std::invalid_argument("BROOK_STREAM_BUDGET_MB must be a positive integer number of MiB");
    return size_t(mb) << 20;
  }
  size_t free = 0, total = 0;
  BK_CUDA(cudaMemGetInfo(&free, &total));
  return std::max(free / 4, size_t(64) << 20);
}

StreamedComponents connected_components_streamed(Context &ctx, const HostVolume &hv, size_t budget,
                                                 const std::vector<int64_t> *object_ids) {
  StreamedComponents out;
  out.d = hv.d;
  out.mapping.assign(1, 0);
  out.boxes.assign(1, Box{});
  const long long n = hv.d.n();
  if (n <= 0) return out;
  if (!hv.data) throw std::invalid_argument("null host volume");
  const size_t b = label_bytes(hv.dtype);
  const long long plane = (long long)hv.d.sx * hv.d.sy;
  if (plane >= (1LL << 31) / 9) throw std::invalid_argument("an xy plane of the streamed volume is too large");
  // a slab: labels, ids, the CCL's scratch and the seam keys per voxel, within the budget
  const long long depth = std::max(1LL, std::min<long long>(hv.d.sz, (long long)(budget / (size_t(plane) * (b + 40)))));
  if (plane * depth >= (1LL << 31) - 1) throw std::invalid_argument("a slab of the streamed volume is too large");
  cudaStream_t s = ctx.stream();
  // Fortran-ordered input is copied to the device straight from the caller's memory; any other
  // layout is gathered into one of two host buffers (the next slab's while the device works on this
  // one). Copies from and to pageable memory: page-locking buffers of a slab's size costs more time
  // than the driver's own staging.
  const auto &st = hv.strides;
  const bool fortran = st[0] == (long long)b && st[1] == (long long)b * hv.d.sx && st[2] == (long long)b * plane;
  std::vector<unsigned char> stage_a(fortran ? 0 : size_t(plane * depth) * b), stage_b(fortran ? 0 : size_t(plane * depth) * b);
  unsigned char *stages[2] = {stage_a.data(), stage_b.data()};
  Buffer<unsigned char> labels(ctx, size_t(plane * depth) * b), prev_labels(ctx, size_t(plane) * b);
  Buffer<uint32_t> ids(ctx, size_t(plane * depth)), prev_ids(ctx, size_t(plane));
  Buffer<u64> keys(ctx, 9 * size_t(plane)), sorted(ctx, 9 * size_t(plane));
  Buffer<int> unique_count(ctx, 1);
  Buffer<unsigned char> scratch;
  out.ids.resize(size_t(n));
  {  // fault the pages in on every thread (a copy into fresh pageable memory faults them one by one)
    const size_t piece = size_t(4) << 20;
    const long long pieces = (long long)((size_t(n) + piece - 1) / piece);
    parallel_for(pieces, [&](long long k) {
      const size_t at = size_t(k) * piece;
      std::memset(out.ids.data() + at, 0, std::min(piece, size_t(n) - at) * sizeof(uint32_t));
    });
  }
  struct Slab {
    int z0, depth;
    int64_t base, count;
    ComponentsResult cc;
    std::vector<Box> boxes;
  };
  std::vector<Slab> slabs;
  std::vector<std::pair<int64_t, int64_t>> seams;  // node pairs to unite
  int64_t nodes = 0;
  const int nslabs = int((hv.d.sz + depth - 1) / depth);
  auto slab_z = [&](int k) { return int(std::min<long long>((long long)k * depth, hv.d.sz)); };
  if (!fortran) gather_slab(hv, 0, slab_z(1), stages[0]);
  for (int k = 0; k < nslabs; ++k) {
    Slab sl;
    sl.z0 = slab_z(k);
    sl.depth = slab_z(k + 1) - sl.z0;
    const VolumeDims sd{hv.d.sx, hv.d.sy, sl.depth};
    const long long m = sd.n();
    const unsigned char *from = fortran ? static_cast<const unsigned char *>(hv.data) + size_t(sl.z0) * size_t(plane) * b
                                        : stages[k % 2];
    BK_CUDA(cudaMemcpyAsync(labels.data(), from, size_t(m) * b, cudaMemcpyHostToDevice, s));
    // the next slab's gather runs on a host thread meanwhile (its buffer's last copy has ended:
    // the stream was synchronised at the end of the previous slab)
    std::thread next;
    if (!fortran && k + 1 < nslabs)
      next = std::thread([&, k] { gather_slab(hv, slab_z(k + 1), slab_z(k + 2), stages[(k + 1) % 2]); });
    try {
      const void *lab = labels.data();
      Buffer<unsigned char> selected;
      if (object_ids) {
        selected = select_labels(ctx, DeviceVolume{labels.data(), hv.dtype, sd}, *object_ids);
        lab = selected.data();
      }
      sl.cc = connected_components(ctx, lab, hv.dtype, sd, ids.data());
      sl.count = sl.cc.count;
      sl.base = nodes;
      nodes += sl.count;
      sl.boxes = sl.count ? analyze(ctx, ids.data(), sd, sl.count) : std::vector<Box>(1);
      if (!slabs.empty()) {
        launch_seam(ctx, hv.dtype, prev_labels.data(), prev_ids.data(), lab, ids.data(), hv.d.sx, hv.d.sy, keys.data());
        const int nk = int(9 * plane);
        auto with_scratch = [&](auto op) {
          size_t bytes = 0;
          BK_CUDA(op(nullptr, bytes));
          bytes = std::max<size_t>(bytes, 16);
          if (bytes > scratch.size()) scratch = Buffer<unsigned char>(ctx, bytes);
          BK_CUDA(op(scratch.data(), bytes));
        };
        with_scratch([&](void *t, size_t &bb) { return cub::DeviceRadixSort::SortKeys(t, bb, keys.data(), sorted.data(), nk, 0, 64, s); });
        with_scratch([&](void *t, size_t &bb) {
          return cub::DeviceSelect::Unique(t, bb, sorted.data(), keys.data(), unique_count.data(), nk, s);
        });
        const int u = unique_count.download(1)[0];
        const auto pairs = keys.download(size_t(u));
        const Slab &prev = slabs.back();
        for (u64 key : pairs) {
          if (key == ~0ull) continue;
          seams.push_back({prev.base + int64_t(key >> 32) - 1, sl.base + int64_t(uint32_t(key)) - 1});
        }
      }
      // the last plane for the next seam
      BK_CUDA(cudaMemcpyAsync(prev_labels.data(), static_cast<const unsigned char *>(lab) + size_t(m - plane) * b,
                              size_t(plane) * b, cudaMemcpyDeviceToDevice, s));
      BK_CUDA(cudaMemcpyAsync(prev_ids.data(), ids.data() + (m - plane), size_t(plane) * sizeof(uint32_t),
                              cudaMemcpyDeviceToDevice, s));
      BK_CUDA(cudaMemcpyAsync(out.ids.data() + size_t(sl.z0) * size_t(plane), ids.data(), size_t(m) * sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, s));
      ctx.synchronize();
    } catch (...) {
      if (next.joinable()) next.join();
      throw;
    }
    if (next.joinable()) next.join();
    slabs.push_back(std::move(sl));
  }
  out.slabs = int(slabs.size());
  // components across the seams: the smallest (slab, id) of each set names it
  UnionFind uf(static_cast<size_t>(nodes));
  for (const auto &p : seams) uf.unite(p.first, p.second);
  std::vector<uint32_t> gid(static_cast<size_t>(nodes), 0);
  std::vector<int> slab_of(static_cast<size_t>(nodes));
  for (size_t k = 0; k < slabs.size(); ++k)
    for (int64_t j = 0; j < slabs[k].count; ++j) slab_of[size_t(slabs[k].base + j)] = int(k);
  int64_t count = 0;
  for (int64_t v = 0; v < nodes; ++v) {
    const int64_t r = uf.find(v);
    if (r == v) {
      if (count >= int64_t(UINT32_MAX) - 1) throw std::invalid_argument("too many components");
      gid[size_t(v)] = uint32_t(++count);
      const Slab &sl = slabs[size_t(slab_of[size_t(v)])];
      const int64_t local = v - sl.base + 1;
      out.mapping.push_back(sl.cc.mapping[size_t(local)]);
      out.roots.push_back(int64_t(sl.z0) * plane + sl.cc.roots[size_t(local - 1)]);
      Box box{};
      for (int a = 0; a < 3; ++a) { box.lo[a] = INT32_MAX; box.hi[a] = -1; }
      box.count = 0;
      out.boxes.push_back(box);
    } else {
      gid[size_t(v)] = gid[size_t(r)];
    }
  }
  out.count = count;
  for (int64_t v = 0; v < nodes; ++v) {
    const Slab &sl = slabs[size_t(slab_of[size_t(v)])];
    const Box &in = sl.boxes[size_t(v - sl.base + 1)];
    Box &o = out.boxes[gid[size_t(v)]];
    o.count += in.count;
    for (int a = 0; a < 3; ++a) {
      const int shift = a == 2 ? sl.z0 : 0;
      o.lo[a] = std::min(o.lo[a], in.lo[a] + shift);
      o.hi[a] = std::max(o.hi[a], in.hi[a] + shift);
    }
  }
  // the host ids renumbered, plane by plane on the host's threads
  std::vector<int> slab_of_z(static_cast<size_t>(hv.d.sz));
  for (size_t k = 0; k < slabs.size(); ++k)
    for (int z = slabs[k].z0; z < slabs[k].z0 + slabs[k].depth; ++z) slab_of_z[size_t(z)] = int(k);
  parallel_for(hv.d.sz, [&](long long z) {
    const int64_t base = slabs[size_t(slab_of_z[size_t(z)])].base;
    uint32_t *p = out.ids.data() + size_t(z) * size_t(plane);
    for (long long i = 0; i < plane; ++i)
      if (p[i]) p[i] = gid[size_t(base + p[i] - 1)];
  });
  return out;
}

void edt_streamed(Context &ctx, const HostVolume &hv, const float aniso[3], bool black_border, size_t budget,
                  float *out) {
  for (int a = 0; a < 3; ++a)
    if (!(aniso[a] > 0) || !std::isfinite(aniso[a])) throw std::invalid_argument("anisotropy must be finite and positive");
  const long long n = hv.d.n();
  if (n <= 0) return;
  budget = stream_budget(budget);
  StreamedComponents cc = connected_components_streamed(ctx, hv, budget, nullptr);
  cudaStream_t s = ctx.stream();
  const int sx = hv.d.sx, sy = hv.d.sy, sz = hv.d.sz;
  const long long plane = (long long)sx * sy;
  // device bytes per voxel of a piece: ids, field, and the envelope stacks of its lines
  const size_t per_voxel = 4 + 4 + 16;
  // x and y passes, slab by slab: squared distances into `out`
  {
    const long long depth = std::max(1LL, std::min<long long>(sz, (long long)(budget / (size_t(plane) * per_voxel))));
    if (plane * depth >= (1LL << 31) - 1) throw std::invalid_argument("a slab of the streamed volume is too large");
    Buffer<uint32_t> ids(ctx, size_t(plane * depth));
    Buffer<float> field(ctx, size_t(plane * depth));
    for (int z0 = 0; z0 < sz; z0 += int(depth)) {
      const int dz = int(std::min<long long>(depth, sz - z0));
      const long long m = plane * dz;
      BK_CUDA(cudaMemcpyAsync(ids.data(), cc.ids.data() + size_t(z0) * size_t(plane), size_t(m) * 4,
                              cudaMemcpyHostToDevice, s));
      edt_xy_squared(ctx, ids.data(), VolumeDims{sx, sy, dz}, aniso, black_border, field.data());
      BK_CUDA(cudaMemcpyAsync(out + size_t(z0) * size_t(plane), field.data(), size_t(m) * 4, cudaMemcpyDeviceToHost, s));
      ctx.synchronize();
    }
  }
  // z pass, by tiles of whole columns: rows [y0, y0 + ty) of every plane
  {
    const long long column = (long long)sx * sz;
    const long long ty = std::max(1LL, std::min<long long>(sy, (long long)(budget / (size_t(column) * per_voxel))));
    if (column * ty >= (1LL << 31) - 1) throw std::invalid_argument("a column tile of the streamed volume is too large");
    const long long tile = column * ty;
    Buffer<uint32_t> ids(ctx, size_t(tile));
    Buffer<float> field(ctx, size_t(tile));
    std::vector<uint32_t> id_stage(static_cast<size_t>(tile));
    std::vector<float> field_stage(static_cast<size_t>(tile));
    uint32_t *is = id_stage.data();
    float *fs = field_stage.data();
    for (int y0 = 0; y0 < sy; y0 += int(ty)) {
      const int dy = int(std::min<long long>(ty, sy - y0));
      const size_t rows = size_t(sx) * size_t(dy);
      parallel_for(sz, [&](long long z) {
        const size_t from = size_t(z) * size_t(plane) + size_t(y0) * size_t(sx), to = size_t(z) * rows;
        std::memcpy(is + to, cc.ids.data() + from, rows * 4);
        std::memcpy(fs + to, out + from, rows * 4);
      });
      const size_t m = rows * size_t(sz);
      BK_CUDA(cudaMemcpyAsync(ids.data(), is, m * 4, cudaMemcpyHostToDevice, s));
      BK_CUDA(cudaMemcpyAsync(field.data(), fs, m * 4, cudaMemcpyHostToDevice, s));
      edt_z_finish(ctx, ids.data(), VolumeDims{sx, dy, sz}, aniso[2], black_border, field.data());
      BK_CUDA(cudaMemcpyAsync(fs, field.data(), m * 4, cudaMemcpyDeviceToHost, s));
      ctx.synchronize();
      parallel_for(sz, [&](long long z) {
        std::memcpy(out + size_t(z) * size_t(plane) + size_t(y0) * size_t(sx), fs + size_t(z) * rows, rows * 4);
      });
    }
  }
}

Packed skeletonize_streamed(Context &ctx, const HostVolume &hv, const Options &opt, size_t budget) {
  if (opt.fill_holes || opt.fix_avocados)
    throw std::invalid_argument("streamed skeletonization does not support fill_holes or fix_avocados");
  for (float a : opt.anisotropy)
    if (!std::isfinite(a) || a <= 0) throw std::invalid_argument("anisotropy must be finite and positive");
  {
    const double e = opt.teasar.pdrf_exponent;
    if (std::isfinite(e) && e == std::floor(e) && std::fmod(e, 2.0) == 1.0)
      throw std::invalid_argument("odd pdrf_exponent makes the background penalty negative");
  }
  if (opt.targets_before.size() > 1 || opt.targets_after.size() > 1)
    throw std::invalid_argument("extra targets are given for more volumes than the call holds");
  std::map<std::string, double> stats;
  long long launches = 0;
  auto t0 = std::chrono::steady_clock::now();
  Packed result;
  result.anisotropy = opt.anisotropy;
  const long long n = hv.d.n();
  auto finish = [&](Packed p) {
    stats["host_ms_streamed_total"] = ms_since(t0);
    launches += ctx.launches;
    stats["launches"] = double(launches);
    ctx.stats = stats;
    ctx.launches = launches;
    return p;
  };
  if (n <= 0 || double(n) <= opt.dust) {
    if (opt.device_output) {
      result.device_vertices = std::make_shared<DeviceStorage>(0, ctx.device());
      result.device_edges = std::make_shared<DeviceStorage>(0, ctx.device());
      result.device_radii = std::make_shared<DeviceStorage>(0, ctx.device());
    }
    return finish(result);
  }
  budget = stream_budget(budget);
  StreamedComponents cc = connected_components_streamed(ctx, hv, budget, opt.object_ids ? &*opt.object_ids : nullptr);
  stats["host_ms_streamed_components"] = ms_since(t0);
  stats["streamed_slabs"] = cc.slabs;
  stats["objects"] = 0;
  const int sx = hv.d.sx, sy = hv.d.sy, sz = hv.d.sz;
  const bool black_border = cc.count == 1 && cc.boxes[1].count == n;
  // border targets of the whole volume's faces (global frame)
  std::vector<std::vector<Point>> borders(size_t(cc.count) + 1);
  if (opt.fix_borders && cc.count) {
    auto tb = std::chrono::steady_clock::now();
    const std::vector<BorderVolume> bv{{0, hv.d, cc.count}};
    int W = 1, H = 1;
    const std::vector<Face> faces = face_list(bv, W, H);
    std::vector<uint32_t> stack(size_t(W) * H * faces.size(), 0);
    for (size_t f = 0; f < faces.size(); ++f) {
      const Face &fc = faces[f];
      for (int pa = 0; pa < fc.fx(); ++pa)
        for (int pb = 0; pb < fc.fy(); ++pb) {
          long long p[3];
          p[fc.a] = pa;
          p[fc.b] = pb;
          p[fc.c] = fc.fixed;
          stack[size_t(pb) + size_t(W) * (size_t(pa) + size_t(H) * f)] = cc.ids[size_t(p[0] + sx * (p[1] + sy * p[2]))];
        }
    }
    Buffer<uint32_t> dstack = to_device(ctx, stack);
    const float aniso[3] = {opt.anisotropy[0], opt.anisotropy[1], opt.anisotropy[2]};
    borders = border_targets(ctx, nullptr, bv, aniso, dstack.data())[0];
    stats["host_ms_streamed_borders"] = ms_since(tb);
  }
  // extra targets by the component they fall on (a negative coordinate counts from the end)
  std::vector<std::vector<Point>> before(size_t(cc.count) + 1), after(size_t(cc.count) + 1);
  for (int list = 0; list < 2; ++list) {
    const auto &lists = list ? opt.targets_after : opt.targets_before;
    if (lists.empty()) continue;
    const long long shape[3] = {sx, sy, sz};
    for (auto p : lists[0]) {
      for (int a = 0; a < 3; ++a) {
        if (p[a] < 0) p[a] += shape[a];
        if (p[a] < 0 || p[a] >= shape[a]) throw std::invalid_argument("extra target is outside the input volume");
      }
      const uint32_t id = cc.ids[size_t(p[0] + sx * (p[1] + sy * p[2]))];
      if (id) (list ? after : before)[id].push_back(p);
    }
  }
  // The traced components, grouped into crops: components whose boxes' centres fall in one cell of
  // a grid of kCell voxels share a crop (the union of their boxes) while it stays within its share
  // of the budget. Every other voxel of a crop is 0 and each member takes a crop id by its first
  // voxel in the crop's flat order, which is the crop's own component numbering; its distances,
  // objects and paths are the same as alone (other components were walls or other objects anyway).
  std::vector<int64_t> traced;
  auto box_voxels = [](const Box &b) {
    return (long long)(b.hi[0] - b.lo[0] + 1) * (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1);
  };
  for (int64_t id = 1; id <= cc.count; ++id) {
    const Box &bx = cc.boxes[size_t(id)];
    if (!bx.count || double(bx.count) <= opt.dust || box_voxels(bx) <= 1) continue;
    traced.push_back(id);
  }
  stats["objects"] = double(traced.size());
  const size_t per_voxel = 4 + 160;  // a crop voxel's label and in-core state
  const long long cap = std::max<long long>(1, std::min<long long>((long long)(budget / per_voxel), (1LL << 31) - 2));
  constexpr int kCell = 128;
  const long long crop_cap = std::min<long long>(cap, 64LL << 20);
  struct Crop {
    Box box;
    std::vector<int64_t> members;  // then ordered by crop id
  };
  std::vector<Crop> crops;
  {
    const long long ncx = (sx + kCell - 1) / kCell, ncy = (sy + kCell - 1) / kCell;
    std::vector<std::pair<long long, int64_t>> keyed;
    for (int64_t id : traced) {
      const Box &b = cc.boxes[size_t(id)];
      const long long c = ((b.lo[0] + b.hi[0]) / 2) / kCell + ncx * (((b.lo[1] + b.hi[1]) / 2) / kCell +
                                                                      ncy * (((b.lo[2] + b.hi[2]) / 2) / kCell));
      keyed.push_back({c, id});
    }
    std::sort(keyed.begin(), keyed.end());
    long long cell = -1;
    for (const auto &[c, id] : keyed) {
      const Box &b = cc.boxes[size_t(id)];
      if (!crops.empty() && c == cell) {
        Box u = crops.back().box;
        for (int a = 0; a < 3; ++a) { u.lo[a] = std::min(u.lo[a], b.lo[a]); u.hi[a] = std::max(u.hi[a], b.hi[a]); }
        if (box_voxels(u) <= crop_cap) {
          crops.back().box = u;
          crops.back().members.push_back(id);
          continue;
        }
      }
      crops.push_back({b, {id}});
      cell = c;
    }
  }
  std::vector<int> crop_of(size_t(cc.count) + 1, -1);
  std::vector<uint32_t> local_of(size_t(cc.count) + 1, 0);
  for (size_t c = 0; c < crops.size(); ++c)
    for (int64_t id : crops[c].members) crop_of[size_t(id)] = int(c);
  std::vector<Packed> pieces;
  std::vector<std::pair<int64_t, int64_t>> made;  // (component, label) of every skeleton made
  std::vector<uint32_t> crop_stage;  // the batch's crops on the host (reused)
  size_t batches = 0;
  for (size_t i = 0; i < crops.size();) {
    size_t j = i;
    long long voxels = 0;
    while (j < crops.size()) {
      const long long v = box_voxels(crops[j].box);
      if (j > i && (voxels + v > cap || voxels + v >= (1LL << 31) - 1)) break;
      voxels += v;
      ++j;
    }
    crop_stage.resize(size_t(voxels));
    uint32_t *crop_host = crop_stage.data();
    std::vector<long long> at(j - i + 1, 0);
    for (size_t k = i; k < j; ++k) at[k - i + 1] = at[k - i] + box_voxels(crops[k].box);
    parallel_for((long long)(j - i), [&](long long q) {
      Crop &cr = crops[i + size_t(q)];
      const Box &bx = cr.box;
      const int cx = bx.hi[0] - bx.lo[0] + 1, cy = bx.hi[1] - bx.lo[1] + 1;
      uint32_t *dst = crop_host + at[size_t(q)];
      const int me = int(i + size_t(q));
      uint32_t next = 0;
      std::vector<int64_t> ordered;
      for (int z = bx.lo[2]; z <= bx.hi[2]; ++z)
        for (int y = bx.lo[1]; y <= bx.hi[1]; ++y) {
          const uint32_t *row = cc.ids.data() + size_t(bx.lo[0]) + size_t(sx) * (size_t(y) + size_t(sy) * size_t(z));
          uint32_t *o = dst + size_t(cx) * (size_t(y - bx.lo[1]) + size_t(cy) * size_t(z - bx.lo[2]));
          for (int x = 0; x < cx; ++x) {
            const uint32_t g = row[x];
            uint32_t v = 0;
            if (g && crop_of[g] == me) {
              if (!local_of[g]) { local_of[g] = ++next; ordered.push_back(g); }
              v = local_of[g];
            }
            o[x] = v;
          }
        }
      cr.members = std::move(ordered);
    });
    Buffer<uint32_t> dev_crops(ctx, size_t(voxels));
    dev_crops.upload(crop_host, size_t(voxels));
    std::vector<DeviceVolume> volumes;
    std::vector<std::vector<std::vector<Point>>> given(j - i);
    Options o = opt;
    o.object_ids.reset();
    o.device_output = false;
    o.targets_before.assign(j - i, {});
    o.targets_after.assign(j - i, {});
    for (size_t k = i; k < j; ++k) {
      const Crop &cr = crops[k];
      const Box &bx = cr.box;
      DeviceVolume v;
      v.data = dev_crops.data() + at[k - i];
      v.dtype = U32;
      v.d = VolumeDims{bx.hi[0] - bx.lo[0] + 1, bx.hi[1] - bx.lo[1] + 1, bx.hi[2] - bx.lo[2] + 1};
      const int shape[3] = {sx, sy, sz};
      int faces = 0;
      for (int a = 0; a < 3; ++a) {
        if (bx.lo[a] > 0 || black_border) faces |= 1 << (2 * a);
        if (bx.hi[a] < shape[a] - 1 || black_border) faces |= 2 << (2 * a);
      }
      v.faces = faces;
      v.origin = {bx.lo[0], bx.lo[1], bx.lo[2]};
      auto frame = [&](const std::vector<Point> &pts, std::vector<Point> &into) {
        for (auto p : pts) {
          for (int a = 0; a < 3; ++a) p[a] -= bx.lo[a];
          into.push_back(p);
        }
      };
      auto &g = given[k - i];
      g.assign(cr.members.size() + 1, {});
      for (size_t m = 0; m < cr.members.size(); ++m) {
        const int64_t id = cr.members[m];
        frame(borders[size_t(id)], g[m + 1]);
        frame(before[size_t(id)], o.targets_before[k - i]);
        frame(after[size_t(id)], o.targets_after[k - i]);
      }
      v.borders = &g;
      volumes.push_back(v);
    }
    launches += ctx.launches;
    auto parts = skeletonize(ctx, volumes, o);
    for (const auto &kv : ctx.stats)
      if (kv.first != "objects") stats[kv.first] += kv.second;
    launches += ctx.launches;
    ctx.launches = 0;
    for (size_t k = i; k < j; ++k) {
      Packed &p = parts[k - i];
      if (p.labels.empty()) continue;
      for (auto &label : p.labels) {  // crop id -> component -> its label
        const int64_t id = crops[k].members[size_t(label) - 1];
        label = cc.mapping[size_t(id)];
        made.push_back({id, label});
      }
      pieces.push_back(std::move(p));
    }
    ++batches;
    i = j;
  }
  stats["streamed_batches"] = double(batches);
  stats["streamed_crops"] = double(crops.size());
  // the pieces merged per label (device), then the labels in the in-core order: by the first
  // component of each label that made a skeleton
  std::vector<const Packed *> refs;
  for (const auto &p : pieces) refs.push_back(&p);
  std::vector<std::array<float, 3>> zero(refs.size(), {0.0f, 0.0f, 0.0f});
  Packed merged = merge_fragments(ctx, refs, zero);
  std::sort(made.begin(), made.end());
  std::vector<int64_t> order;
  {
    std::map<int64_t, bool> seen;
    for (const auto &m : made)
      if (!seen[m.second]) { seen[m.second] = true; order.push_back(m.second); }
  }
  const size_t K = merged.labels.size();
  const size_t V = size_t(merged.vertex_offsets.back()), E = size_t(merged.edge_offsets.back());
  std::vector<float> mv(3 * V), mr(V);
  std::vector<uint32_t> me(2 * E);
  if (V) {
    BK_CUDA(cudaMemcpy(mv.data(), merged.device_vertices->ptr, mv.size() * sizeof(float), cudaMemcpyDeviceToHost));
    BK_CUDA(cudaMemcpy(mr.data(), merged.device_radii->ptr, mr.size() * sizeof(float), cudaMemcpyDeviceToHost));
  }
  if (E) BK_CUDA(cudaMemcpy(me.data(), merged.device_edges->ptr, me.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  std::map<int64_t, size_t> index;
  for (size_t k = 0; k < K; ++k) index[merged.labels[k]] = k;
  for (int64_t label : order) {
    const size_t k = index.at(label);
    result.labels.push_back(label);
    const int64_t v0 = merged.vertex_offsets[k], v1 = merged.vertex_offsets[k + 1];
    const int64_t e0 = merged.edge_offsets[k], e1 = merged.edge_offsets[k + 1];
    result.vertices.insert(result.vertices.end(), mv.begin() + 3 * v0, mv.begin() + 3 * v1);
    result.radii.insert(result.radii.end(), mr.begin() + v0, mr.begin() + v1);
    result.edges.insert(result.edges.end(), me.begin() + 2 * e0, me.begin() + 2 * e1);
    result.vertex_offsets.push_back(result.vertex_offsets.back() + (v1 - v0));
    result.edge_offsets.push_back(result.edge_offsets.back() + (e1 - e0));
  }
  if (opt.device_output) {
    const int dev = ctx.device();
    result.device_vertices = std::make_shared<DeviceStorage>(result.vertices.size() * sizeof(float), dev);
    result.device_radii = std::make_shared<DeviceStorage>(result.radii.size() * sizeof(float), dev);
    result.device_edges = std::make_shared<DeviceStorage>(result.edges.size() * sizeof(uint32_t), dev);
    if (!result.vertices.empty()) {
      BK_CUDA(cudaMemcpy(result.device_vertices->ptr, result.vertices.data(), result.vertices.size() * sizeof(float),
                         cudaMemcpyHostToDevice));
      BK_CUDA(cudaMemcpy(result.device_radii->ptr, result.radii.data(), result.radii.size() * sizeof(float),
                         cudaMemcpyHostToDevice));
    }
    if (!result.edges.empty())
      BK_CUDA(cudaMemcpy(result.device_edges->ptr, result.edges.data(), result.edges.size() * sizeof(uint32_t),
                         cudaMemcpyHostToDevice));
    result.vertices.clear();
    result.radii.clear();
    result.edges.clear();
  }
  return finish(result);
}

}  // namespace bk
