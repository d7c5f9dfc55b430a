// Orchestration of the skeletonizer over one flat index space that holds every volume of a call
// (an arena per volume). Each stage covers every volume at once (launches per volume where a
// volume's shape sets the grid, one download for all):
//   connected components (a volume arriving by slabs has its unions queued slab by slab), boxes,
//   EDT, neighbour masks, DBF maxima, border targets, object voxel lists;
//   every object of every volume in the engine: prepare (roots, DAF, PDRF), target orders, trace;
//   assembly into packed skeletons per volume.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <numeric>
#include <stdexcept>

#include "assembly.hpp"
#include "common.cuh"
#include "engine.hpp"
#include "order.hpp"
#include "pipeline.hpp"

namespace bk {
namespace {

template <class L>
__global__ void filter_labels(const L *in, L *out, long long n, const long long *ids, int count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long v = (long long)in[i];
  int lo = 0, hi = count;
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if (ids[mid] < v) lo = mid + 1; else hi = mid;
  }
  out[i] = (lo < count && ids[lo] == v) ? in[i] : L(0);
}

// Compacts the used prefix of every object's store region.
__global__ void gather_store(const int *store, const long long *store_begin, const long long *dst_begin,
                             const int *nstore, int nobj, int *out) {
  const int o = blockIdx.x;
  if (o >= nobj) return;
  const int n = nstore[o];
  const int *src = store + store_begin[o];
  const long long dst = dst_begin[o];
  for (int i = threadIdx.x; i < n; i += blockDim.x) out[dst + i] = src[i];
}

__global__ void gather_records(const int *rs, const int *rl, const long long *rec_begin, const long long *dst_begin,
                               const int *npaths, int nobj, int *out_start, int *out_len) {
  const int o = blockIdx.x;
  if (o >= nobj) return;
  const int n = npaths[o];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    out_start[dst_begin[o] + i] = rs[rec_begin[o] + i];
    out_len[dst_begin[o] + i] = rl[rec_begin[o] + i];
  }
}

// A box of a volume (ids or DBF) into a contiguous crop: out[c] for crop voxel c of the box at
// (lx, ly, lz) with extents (cx, cy, cz). With `keep`, crop voxels where keep is 0 get 0.
template <class T>
__global__ void gather_box(const T *src, int sx, int sy, int lx, int ly, int lz, int cx, int cy, long long n,
                           const uint32_t *keep, T *out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long z = i / ((long long)cx * cy), r = i - z * cx * cy, y = r / cx, x = r - y * cx;
  const T value = src[(x + lx) + (long long)sx * ((y + ly) + (long long)sy * (z + lz))];
  out[i] = keep && !keep[i] ? T(0) : value;
}

// The soma root (trace.cu:55-73, batched.cu:58-105): among the crop voxels at the DBF maximum,
// sorted by (x, y, z), the first nearest (float64 squared distance, voxel units) to their float32
// centroid. Returns the crop flat index.
long long soma_root(const std::vector<float> &dbf, const std::vector<uint32_t> &mask, float maximum, int cx, int cy) {
  std::vector<std::array<long long, 3>> points;
  std::array<long long, 3> sum{0, 0, 0};
  for (long long v = 0; v < (long long)dbf.size(); ++v)
    if (mask[v] && dbf[v] == maximum) {
      const long long z = v / ((long long)cx * cy), r = v - z * cx * cy, y = r / cx, x = r - y * cx;
      points.push_back({x, y, z});
      sum[0] += x; sum[1] += y; sum[2] += z;
    }
  if (points.empty()) throw std::runtime_error("no soma maximum");
  std::sort(points.begin(), points.end());
  float centre[3];
  for (int k = 0; k < 3; ++k) centre[k] = float(double(sum[k]) / double(points.size()));
  double best = INFINITY;
  std::array<long long, 3> root = points.front();
  for (const auto &p : points) {
    double cost = 0;
    for (int k = 0; k < 3; ++k) { const double d = double(p[k]) - double(centre[k]); cost += d * d; }
    if (cost < best) { best = cost; root = p; }
  }
  return root[0] + cx * (root[1] + (long long)cy * root[2]);
}

template <class L>
Buffer<unsigned char> filtered(Context &ctx, const DeviceVolume &v, const std::vector<int64_t> &ids) {
  std::vector<long long> sorted(ids.begin(), ids.end());
  std::sort(sorted.begin(), sorted.end());
  sorted.erase(std::unique(sorted.begin(), sorted.end()), sorted.end());
  Buffer<long long> d = to_device(ctx, sorted);
  Buffer<unsigned char> out(ctx, v.d.n() * sizeof(L));
  filter_labels<L><<<blocks_for(v.d.n()), 256, 0, ctx.stream()>>>(static_cast<const L *>(v.data),
                                                                  reinterpret_cast<L *>(out.data()), v.d.n(),
                                                                  d.data(), (int)sorted.size()); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  return out;
}

Buffer<unsigned char> filter_volume(Context &ctx, const DeviceVolume &v, const std::vector<int64_t> &ids) {
  switch (v.dtype) {
    case U8: return filtered<uint8_t>(ctx, v, ids);
    case U16: return filtered<uint16_t>(ctx, v, ids);
    case U32: return filtered<uint32_t>(ctx, v, ids);
    case U64: return filtered<uint64_t>(ctx, v, ids);
    case I8: return filtered<int8_t>(ctx, v, ids);
    case I16: return filtered<int16_t>(ctx, v, ids);
    case I32: return filtered<int32_t>(ctx, v, ids);
    case I64: return filtered<int64_t>(ctx, v, ids);
    default: throw std::invalid_argument("integer labels required");
  }
}

// The workload class the tuned launch choices are kept by: the bit lengths of the foreground
// voxels, of the largest object's voxels and of the object count.
unsigned long long workload_class(long long foreground, long long largest, int objects) {
  auto bits = [](long long v) { int b = 0; while (v > 0) { ++b; v >>= 1; } return (unsigned long long)b; };
  return (bits(foreground) << 16) | (bits(largest) << 8) | bits(objects);
}

struct VolumeState {
  VolumeDims d;
  long long offset = 0;
  ComponentsResult cc;
  std::vector<Box> boxes;
  std::vector<std::vector<Point>> borders;
  std::vector<float> dbf_max;
  std::vector<int> object_of;  // id -> global object index, -1 when inactive
  bool empty = true;
  bool black_border = false;   // one component filling the volume as given
  int faces = -1;              // the EDT's walls of a crop (DeviceVolume::faces)
  std::array<int, 3> origin{0, 0, 0};
  const std::vector<std::vector<Point>> *given_borders = nullptr;
};

}  // namespace

Buffer<unsigned char> select_labels(Context &ctx, const DeviceVolume &v, const std::vector<int64_t> &ids) {
  return filter_volume(ctx, v, ids);
}

std::vector<Packed> skeletonize(Context &ctx, const std::vector<DeviceVolume> &volumes, const Options &opt) {
  cudaStream_t s = ctx.stream();
  ctx.stats.clear();
  ctx.launches = 0;
  ctx.reset_peak();
  StageClock clock(ctx);
  const auto &t = opt.teasar;
  for (float a : opt.anisotropy)
    if (!std::isfinite(a) || a <= 0) throw std::invalid_argument("anisotropy must be finite and positive");
  {
    const double e = t.pdrf_exponent;
    if (std::isfinite(e) && e == std::floor(e) && std::fmod(e, 2.0) == 1.0)
      throw std::invalid_argument("odd pdrf_exponent makes the background penalty negative");
  }
  if (opt.targets_before.size() > volumes.size() || opt.targets_after.size() > volumes.size())
    throw std::invalid_argument("extra targets are given for more volumes than the call holds");
  // a power-of-two exponent is repeated squaring, any other one powf (the reference's lockstep
  // and per-component arithmetic, batched_regular.inc:93-108 and trace_primitives.cu:119-129)
  const double exponent = t.pdrf_exponent;
  int squarings = -1;
  if (exponent > 0 && exponent < 65536 && exponent == std::floor(exponent) && !(int(exponent) & (int(exponent) - 1))) {
    squarings = 0;
    for (int e = int(exponent); e > 1; e >>= 1) ++squarings;
  }

  std::vector<Packed> results(volumes.size());
  for (auto &r : results) std::copy(opt.anisotropy.begin(), opt.anisotropy.end(), r.anisotropy.begin());
  // ---- one flat index space for all volumes
  std::vector<VolumeState> vs(volumes.size());
  long long N = 0;
  for (size_t v = 0; v < volumes.size(); ++v) {
    vs[v].d = volumes[v].d;
    vs[v].offset = N;
    vs[v].faces = volumes[v].faces;
    vs[v].origin = volumes[v].origin;
    vs[v].given_borders = volumes[v].borders;
    const long long n = volumes[v].d.n();
    if (n > 0 && double(n) > opt.dust) { N += n; vs[v].empty = false; }
  }
  if (N >= (1LL << 31) - 1) throw std::invalid_argument("the volumes of one call must hold fewer than 2^31 voxels");
  if (N == 0) return results;
  Buffer<uint32_t> ids(ctx, N), mask(ctx, N);
  Buffer<float> dbf(ctx, N);
  const float aniso[3] = {opt.anisotropy[0], opt.anisotropy[1], opt.anisotropy[2]};
  // ---- connected components of every volume at once, then boxes per volume
  std::vector<Buffer<unsigned char>> masked(volumes.size());
  {
    std::vector<CcVolume> cv;
    std::vector<size_t> which;
    for (size_t v = 0; v < volumes.size(); ++v) {
      if (vs[v].empty) continue;
      const void *labels = volumes[v].data;
      const Slabs *slabs = volumes[v].slabs;
      if (opt.object_ids) {
        if (slabs && !slabs->empty()) BK_CUDA(cudaStreamWaitEvent(s, slabs->back().second, 0));
        masked[v] = filter_volume(ctx, volumes[v], *opt.object_ids);
        labels = masked[v].data();
        slabs = nullptr;
      }
      cv.push_back({labels, volumes[v].dtype, vs[v].d, vs[v].offset, slabs});
      which.push_back(v);
    }
    auto cc = connected_components(ctx, cv, ids.data());
    for (size_t j = 0; j < which.size(); ++j) vs[which[j]].cc = std::move(cc[j]);
    clock.mark("ccl");
  }
  {
    std::vector<IdVolume> iv;
    std::vector<size_t> which;
    for (size_t v = 0; v < vs.size(); ++v) {
      auto &st = vs[v];
      if (st.empty) continue;
      st.object_of.assign(st.cc.count + 1, -1);
      if (!st.cc.count) { st.empty = true; continue; }
      iv.push_back({st.offset, st.d, st.cc.count});
      which.push_back(v);
    }
    auto boxes = analyze(ctx, ids.data(), iv);
    for (size_t j = 0; j < which.size(); ++j) vs[which[j]].boxes = std::move(boxes[j]);
    // black border from the volume as given, before any void is filled (skeletonize.cu:82-85)
    for (auto &st : vs) st.black_border = !st.empty && st.cc.count == 1 && st.boxes[1].count == st.d.n();
    clock.mark("analyze");
    // ---- voids of every component filled (skeletonize.cu:86-90): the ids change, then the boxes
    // and counts are taken again
    if (opt.fill_holes && !iv.empty()) {
      std::vector<HoleVolume> hv;
      for (size_t j : which) hv.push_back({vs[j].offset, vs[j].d, &vs[j].boxes});
      const long long filled = fill_holes(ctx, ids.data(), hv);
      ctx.stats["hole_filled_voxels"] = double(filled);
      if (filled) {
        auto again = analyze(ctx, ids.data(), iv);
        for (size_t j = 0; j < which.size(); ++j) vs[which[j]].boxes = std::move(again[j]);
      }
      clock.mark("holes");
    }
  }
  // ---- EDT of every volume at once (the y and z passes of all volumes' lines in one launch each)
  {
    std::vector<EdtVolume> ev;
    for (const auto &st : vs)
      if (!st.empty) ev.push_back({st.offset, st.d, st.black_border, st.faces});
    edt_volumes(ctx, ids.data(), ev, aniso, dbf.data());
    clock.mark("edt");
  }
  // ---- the avocado stage per volume (skeletonize.cu:92-96): pits merged into the objects around
  // them, ids renumbered, the field refreshed where a pass merged; then boxes and counts again
  if (opt.fix_avocados) {
    int passes = 0;
    std::vector<IdVolume> iv;
    std::vector<size_t> which;
    for (size_t v = 0; v < vs.size(); ++v) {
      auto &st = vs[v];
      if (st.empty) continue;
      passes = std::max(passes, fix_avocados(ctx, ids.data() + st.offset, dbf.data() + st.offset, st.d, st.cc,
                                             t.soma_detection, aniso, st.black_border));
      st.object_of.assign(st.cc.count + 1, -1);
      if (!st.cc.count) { st.empty = true; continue; }
      iv.push_back({st.offset, st.d, st.cc.count});
      which.push_back(v);
    }
    ctx.stats["avocado_passes"] = passes;
    auto again = analyze(ctx, ids.data(), iv);
    for (size_t j = 0; j < which.size(); ++j) vs[which[j]].boxes = std::move(again[j]);
    clock.mark("avocados");
  }
  {
    std::vector<IdVolume> iv;
    std::vector<size_t> which;
    for (size_t v = 0; v < vs.size(); ++v) {
      auto &st = vs[v];
      if (st.empty) continue;
      neighbour_mask(ctx, ids.data() + st.offset, st.d, mask.data() + st.offset);
      st.borders.assign(st.cc.count + 1, {});
      iv.push_back({st.offset, st.d, st.cc.count});
      which.push_back(v);
    }
    clock.mark("mask");
    auto maxima = segment_max(ctx, dbf.data(), ids.data(), iv);
    for (size_t j = 0; j < which.size(); ++j) vs[which[j]].dbf_max = std::move(maxima[j]);
    clock.mark("dbf_max");
  }
  // ---- border targets of every volume in one pass
  if (opt.fix_borders) {
    std::vector<BorderVolume> bv;
    std::vector<size_t> which;
    for (size_t v = 0; v < vs.size(); ++v) {
      if (vs[v].empty) continue;
      if (vs[v].given_borders) {
        if (vs[v].given_borders->size() < size_t(vs[v].cc.count) + 1)
          throw std::invalid_argument("given border targets do not cover the volume's components");
        vs[v].borders = *vs[v].given_borders;
        continue;
      }
      bv.push_back({vs[v].offset, vs[v].d, vs[v].cc.count});
      which.push_back(v);
    }
    auto picks = border_targets(ctx, ids.data(), bv, aniso);
    for (size_t j = 0; j < which.size(); ++j) vs[which[j]].borders = std::move(picks[j]);
    clock.mark("borders");
  }
  // ---- objects: more voxels than dust and a bounding box of two or more voxels (batched.cu:187-191).
  // An object whose DBF maximum passes soma_detection_threshold is a soma candidate: it is prepared
  // and traced in a private arena, the crop of its box appended to the flat index space
  // (prepare_component and soma.cu:141-237): its voids filled, the DBF recomputed on the crop when
  // anything was filled (black border when the fill covers the crop), else the input's; a soma
  // when the crop's maximum passes soma_acceptance_threshold.
  struct Object {
    int volume;     // the input volume the object belongs to
    uint32_t id;
    int64_t count;  // voxels it is traced with (a candidate's: its filled crop)
    int arena;      // the engine arena it is traced in (its volume, or its private crop)
    int soma;       // index into `somas`, or -1
  };
  struct SomaArena {
    int volume;
    uint32_t id;
    std::array<int, 3> lo, dims;
    long long offset = 0, valid = 0, filled = 0;
    std::vector<uint32_t> mask;  // the filled crop, 1 / 0
    float maximum = 0;
    bool soma = false;
    long long root = -1;         // crop flat index of the soma root
  };
  std::vector<Object> objects;
  std::vector<SomaArena> somas;
  for (size_t v = 0; v < vs.size(); ++v) {
    auto &st = vs[v];
    if (st.empty) continue;
    for (int64_t id = 1; id <= st.cc.count; ++id) {
      const Box &b = st.boxes[id];
      const long long bbox = (long long)(b.hi[0] - b.lo[0] + 1) * (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1);
      if (!b.count || double(b.count) <= opt.dust || bbox <= 1) continue;
      st.object_of[id] = int(objects.size());
      int soma = -1;
      if (double(st.dbf_max[id]) > t.soma_detection) {
        soma = int(somas.size());
        SomaArena sa;
        sa.volume = int(v);
        sa.id = uint32_t(id);
        for (int a = 0; a < 3; ++a) { sa.lo[a] = b.lo[a]; sa.dims[a] = b.hi[a] - b.lo[a] + 1; }
        somas.push_back(std::move(sa));
      }
      objects.push_back({int(v), uint32_t(id), b.count, int(v), soma});
    }
  }
  const int nobj = int(objects.size());
  if (nobj == 0) return results;
  long long NT = N;  // voxels of the flat index space, private arenas included
  if (!somas.empty()) {
    // the candidates' crops: ids gathered on the device; every crop's voids (fill_voids' rule) from
    // one batched flood over all the boxes
    std::vector<VoidBox> boxes_of;
    for (const auto &sa : somas) boxes_of.push_back({vs[sa.volume].offset, vs[sa.volume].d, vs[sa.volume].boxes[sa.id], sa.id});
    const Voids voids = component_voids(ctx, ids.data(), boxes_of);
    for (size_t j = 0; j < somas.size(); ++j) {
      auto &sa = somas[j];
      const auto &st = vs[sa.volume];
      const long long n = (long long)sa.dims[0] * sa.dims[1] * sa.dims[2];
      Buffer<uint32_t> crop(ctx, n);
      gather_box<uint32_t><<<blocks_for(n), 256, 0, s>>>(ids.data() + st.offset, st.d.sx, st.d.sy, sa.lo[0], sa.lo[1],
                                                         sa.lo[2], sa.dims[0], sa.dims[1], n, nullptr, crop.data());
      ++ctx.launches;
      BK_CUDA(cudaGetLastError());
      sa.mask = crop.download();
      for (auto &m : sa.mask) m = m == sa.id ? 1u : 0u;
      sa.filled = voids.count[j];
      sa.valid = st.boxes[sa.id].count + sa.filled;
      sa.offset = NT;
      NT += n;
    }
    for (size_t k = 0; k < voids.voxel.size(); ++k) {
      auto &sa = somas[size_t(voids.box[k])];
      const auto &st = vs[sa.volume];
      const long long local = voids.voxel[k] - st.offset;
      const long long x = local % st.d.sx, y = (local / st.d.sx) % st.d.sy, z = local / ((long long)st.d.sx * st.d.sy);
      sa.mask[(x - sa.lo[0]) + sa.dims[0] * ((y - sa.lo[1]) + (long long)sa.dims[1] * (z - sa.lo[2]))] = 1u;
    }
    if (NT >= (1LL << 31) - 1) throw std::invalid_argument("the volumes of one call must hold fewer than 2^31 voxels");
    // ids, masks and DBF over the whole space: the volumes', then every private crop's
    Buffer<uint32_t> ids2(ctx, NT), mask2(ctx, NT);
    Buffer<float> dbf2(ctx, NT);
    BK_CUDA(cudaMemcpyAsync(ids2.data(), ids.data(), N * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    BK_CUDA(cudaMemcpyAsync(mask2.data(), mask.data(), N * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    BK_CUDA(cudaMemcpyAsync(dbf2.data(), dbf.data(), N * sizeof(float), cudaMemcpyDeviceToDevice, s));
    for (auto &sa : somas) {
      const auto &st = vs[sa.volume];
      const long long n = (long long)sa.mask.size();
      const VolumeDims cd{sa.dims[0], sa.dims[1], sa.dims[2]};
      ids2.upload(sa.mask.data(), n, sa.offset);
      if (sa.filled)
        edt(ctx, ids2.data() + sa.offset, cd, aniso, sa.valid == n, 3, dbf2.data() + sa.offset);
      else {
        gather_box<float><<<blocks_for(n), 256, 0, s>>>(dbf.data() + st.offset, st.d.sx, st.d.sy, sa.lo[0], sa.lo[1],
                                                        sa.lo[2], sa.dims[0], sa.dims[1], n, ids2.data() + sa.offset,
                                                        dbf2.data() + sa.offset);
        ++ctx.launches;
        BK_CUDA(cudaGetLastError());
      }
      neighbour_mask(ctx, ids2.data() + sa.offset, cd, mask2.data() + sa.offset);
      const auto crop_dbf = dbf2.download(n, sa.offset);
      for (long long c = 0; c < n; ++c)
        if (sa.mask[c]) sa.maximum = std::max(sa.maximum, crop_dbf[c]);
      sa.soma = double(sa.maximum) > t.soma_acceptance;
      if (sa.soma) sa.root = soma_root(crop_dbf, sa.mask, sa.maximum, sa.dims[0], sa.dims[1]);
    }
    ids = std::move(ids2);
    mask = std::move(mask2);
    dbf = std::move(dbf2);
    for (auto &ob : objects)
      if (ob.soma >= 0) {
        ob.count = somas[ob.soma].valid;
        ob.arena = int(vs.size()) + ob.soma;
      }
    clock.mark("somata");
  }
  // After the avocado stage a foreground voxel can hold distance zero (background it painted
  // without a refresh): +inf to the tracer from here on, in the volumes' part of the space
  // (lockstep.cu:61-82; a soma's crop keeps its own field).
  if (opt.fix_avocados) ctx.stats["zero_distances"] = double(zero_distances_to_infinity(ctx, ids.data(), dbf.data(), N));
  // a point of a volume (x, y, z) as the flat index of the arena its object is traced in
  auto arena_flat = [&](const Object &ob, const Point &p) -> int {
    if (ob.soma < 0) {
      const auto &st = vs[ob.volume];
      return int(st.offset + p[0] + (long long)st.d.sx * (p[1] + (long long)st.d.sy * p[2]));
    }
    const auto &sa = somas[ob.soma];
    return int(sa.offset + (p[0] - sa.lo[0]) + (long long)sa.dims[0] * ((p[1] - sa.lo[1]) + (long long)sa.dims[1] * (p[2] - sa.lo[2])));
  };
  // extra targets by the component they fall on (skeletonize.cu:16-25, 61-65 of the reference): a
  // negative coordinate counts from the end of its axis; a point outside the volume is an error;
  // points on the background or on objects that are not traced are dropped. Each volume's points
  // are in its own frame.
  std::vector<std::vector<int>> before_of(nobj), after_of(nobj);
  {
    struct Pick { size_t volume; bool after; long long flat; Point p; };
    std::vector<Pick> picks;
    for (size_t v = 0; v < volumes.size(); ++v)
      for (int list = 0; list < 2; ++list) {
        const auto &lists = list ? opt.targets_after : opt.targets_before;
        if (v >= lists.size()) continue;
        const auto &st = vs[v];
        const long long shape[3] = {volumes[v].d.sx, volumes[v].d.sy, volumes[v].d.sz};
        for (auto p : lists[v]) {
          for (int a = 0; a < 3; ++a) {
            if (p[a] < 0) p[a] += shape[a];
            if (p[a] < 0 || p[a] >= shape[a]) throw std::invalid_argument("extra target is outside the input volume");
          }
          if (st.empty) continue;  // a volume at or below the dust threshold traces nothing
          picks.push_back({v, list == 1, st.offset + p[0] + shape[0] * (p[1] + shape[1] * p[2]), p});
        }
      }
    if (!picks.empty()) {
      std::vector<uint32_t> at(picks.size());
      for (size_t i = 0; i < picks.size(); ++i)
        BK_CUDA(cudaMemcpyAsync(&at[i], ids.data() + picks[i].flat, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      ctx.synchronize();
      for (size_t i = 0; i < picks.size(); ++i) {
        const int o = at[i] ? vs[picks[i].volume].object_of[at[i]] : -1;
        if (o < 0) continue;
        (picks[i].after ? after_of : before_of)[o].push_back(arena_flat(objects[o], picks[i].p));
      }
    }
  }
  std::vector<int> after_begin(nobj), after_count(nobj), after;
  // per object: voxel range, arena, border root, manual targets, path budget, store regions
  std::vector<int> obj_begin(nobj), obj_count(nobj), obj_arena(nobj), border_root(nobj, -1);
  std::vector<float> M(nobj), free_radius(nobj, 0.0f);
  std::vector<double> soma_radius(nobj, -1.0);
  std::vector<int> manual_begin(nobj), manual_count(nobj), manual;
  std::vector<long long> max_paths(nobj), store_begin(nobj), store_cap(nobj), rec_begin(nobj), rec_cap(nobj);
  long long F = 0, store_total = 0, rec_total = 0;
  for (int o = 0; o < nobj; ++o) {
    const auto &ob = objects[o];
    const auto &st = vs[ob.volume];
    const SomaArena *sa = ob.soma >= 0 ? &somas[ob.soma] : nullptr;
    const bool soma = sa && sa->soma;
    obj_begin[o] = int(F);
    obj_count[o] = int(ob.count);
    F += ob.count;
    obj_arena[o] = ob.arena;
    // the maximum of the DBF the object is traced with (a candidate's: its crop's)
    M[o] = float(1.0 / std::pow(double(sa ? sa->maximum : st.dbf_max[ob.id]), 1.01));
    const auto &b = st.borders[ob.id];
    auto flat = [&](const Point &p) { return arena_flat(ob, p); };
    if (soma) {
      // the soma root, the DAF seeded through free space within the maximum of it, the paths
      // trimmed to maximum * soma_invalidation_scale + soma_invalidation_const (trace.cu:114-124)
      border_root[o] = int(sa->offset + sa->root);
      free_radius[o] = sa->maximum;
      soma_radius[o] = double(sa->maximum) * t.soma_scale + t.soma_constant;
    } else if (!b.empty()) border_root[o] = flat(b.back());
    // manual targets in pop order: the border points except the last (the root), then the extra
    // targets before, all last first (lockstep.cu:127-134); none: the object's own target (-1,
    // resolved on the device). A soma's border root, if any, comes first in the list (traced last
    // of them), and a soma has no default target (lockstep.cu:131-135, trace.cu:163).
    // Extra targets after: last first, once no voxel is alive.
    std::vector<int> listed;
    if (soma && !b.empty()) listed.push_back(flat(b.back()));
    for (size_t i = 0; i + 1 < b.size(); ++i) listed.push_back(flat(b[i]));
    listed.insert(listed.end(), before_of[o].begin(), before_of[o].end());
    manual_begin[o] = int(manual.size());
    if (listed.empty()) {
      if (!soma) manual.push_back(-1);
    } else manual.insert(manual.end(), listed.rbegin(), listed.rend());
    manual_count[o] = int(manual.size()) - manual_begin[o];
    after_begin[o] = int(after.size());
    after.insert(after.end(), after_of[o].rbegin(), after_of[o].rend());
    after_count[o] = int(after.size()) - after_begin[o];
    const int64_t budget = t.max_paths.value_or(ob.count);
    max_paths[o] = manual_count[o] + after_count[o] >= budget ? 0 : budget;
    store_begin[o] = store_total;
    // a soma's trimmed paths may end with the root: one more vertex per path
    store_cap[o] = (2 + (soma ? 1 : 0) + (long long)after_count[o]) * ob.count + manual_count[o] + 2;
    store_total += store_cap[o];
    rec_begin[o] = rec_total;
    rec_cap[o] = ob.count + manual_count[o] + after_count[o] + 1;
    rec_total += rec_cap[o];
  }
  if (F >= (1LL << 31)) throw std::invalid_argument("too many foreground voxels");
  // global per-voxel state
  Buffer<float> pdrf(ctx, NT), dist(ctx, NT), daf(ctx, NT);
  Buffer<uint32_t> flags(ctx, NT);
  Buffer<uint8_t> alive(ctx, NT);
  Buffer<unsigned long long> key(ctx, NT);
  fill_float(ctx, pdrf.data(), NT, INFINITY);
  fill_float(ctx, dist.data(), NT, INFINITY);
  fill_float(ctx, daf.data(), NT, INFINITY);
  flags.zero();
  alive.zero();
  key.fill_bytes(0xFF);
  // object voxel lists of all volumes at once (grouped by global object index), marking them alive
  std::vector<ArenaVolume> listed;
  std::vector<int> object_table;
  for (size_t v = 0; v < vs.size(); ++v) {
    auto &st = vs[v];
    if (st.empty) continue;
    bool any = false;
    for (int64_t id = 1; id <= st.cc.count && !any; ++id) any = st.object_of[id] >= 0;
    if (!any) continue;
    listed.push_back({st.offset, st.offset + st.d.n(), int(object_table.size())});
    object_table.push_back(-1);  // id 0
    for (int64_t id = 1; id <= st.cc.count; ++id) {  // a soma candidate is traced in its crop
      const int o = st.object_of[id];
      object_table.push_back(o >= 0 && objects[o].soma >= 0 ? -1 : o);
    }
  }
  for (size_t j = 0; j < somas.size(); ++j) {  // a crop holds its object as id 1
    const long long n = (long long)somas[j].mask.size();
    listed.push_back({somas[j].offset, somas[j].offset + n, int(object_table.size())});
    object_table.push_back(-1);
    object_table.push_back(vs[somas[j].volume].object_of[somas[j].id]);
  }
  Buffer<int> vox = arena_object_voxels(ctx, ids.data(), NT, listed, object_table, nobj, F, alive.data());
  clock.mark("object_voxels");
  const size_t arenas = vs.size() + somas.size();
  std::vector<int> arena_offset(arenas), arena_dims(3 * arenas);
  for (size_t v = 0; v < vs.size(); ++v) {
    arena_offset[v] = int(vs[v].offset);
    arena_dims[3 * v] = vs[v].d.sx; arena_dims[3 * v + 1] = vs[v].d.sy; arena_dims[3 * v + 2] = vs[v].d.sz;
  }
  for (size_t j = 0; j < somas.size(); ++j) {
    const size_t r = vs.size() + j;
    arena_offset[r] = int(somas[j].offset);
    for (int k = 0; k < 3; ++k) arena_dims[3 * r + k] = somas[j].dims[k];
  }
  // largest objects first; the leading objects above a size threshold go to clusters
  std::vector<int> schedule(nobj);
  std::iota(schedule.begin(), schedule.end(), 0);
  std::stable_sort(schedule.begin(), schedule.end(), [&](int a, int b) { return obj_count[a] > obj_count[b]; });
  // the engine's launch choices: a test's environment knob, else the autotuner's (or the saved)
  // choice for this workload class, else the built-in rule
  const long long largest = nobj ? obj_count[schedule[0]] : 0;
  ctx.last_class = workload_class(F, largest, nobj);
  Tuning tune;
  if (ctx.forced) tune = *ctx.forced;
  else if (auto it = ctx.tuning.find(ctx.last_class); it != ctx.tuning.end()) tune = it->second;
  auto leading = [&](const char *knob, long long voxels) {  // knob: tuning override from the environment
    if (const char *e = std::getenv(knob)) voxels = std::atoll(e);
    int n = 0;
    while (n < nobj && obj_count[schedule[n]] >= voxels) ++n;
    return n;
  };
  const int nbig_prepare = leading("BROOK_B200_PREPARE_CLUSTER_VOXELS",
                                   tune.prepare_cluster_voxels > 0 ? tune.prepare_cluster_voxels : kPrepareClusterVoxels);
  const int nbig_trace = leading("BROOK_B200_TRACE_CLUSTER_VOXELS",
                                 tune.trace_cluster_voxels > 0 ? tune.trace_cluster_voxels : trace_cluster_voxels(F));
  auto d_arena_offset = to_device(ctx, arena_offset), d_arena_dims = to_device(ctx, arena_dims);
  auto d_obj_arena = to_device(ctx, obj_arena), d_obj_begin = to_device(ctx, obj_begin), d_obj_count = to_device(ctx, obj_count);
  auto d_schedule = to_device(ctx, schedule), d_border_root = to_device(ctx, border_root);
  auto d_M = to_device(ctx, M), d_free_radius = to_device(ctx, free_radius);
  auto d_soma_radius = to_device(ctx, soma_radius);
  auto d_manual_begin = to_device(ctx, manual_begin), d_manual_count = to_device(ctx, manual_count);
  auto d_manual = to_device(ctx, manual.empty() ? std::vector<int>{0} : manual);
  auto d_after_begin = to_device(ctx, after_begin), d_after_count = to_device(ctx, after_count);
  auto d_after = to_device(ctx, after.empty() ? std::vector<int>{0} : after);
  auto d_max_paths = to_device(ctx, max_paths), d_store_begin = to_device(ctx, store_begin), d_store_cap = to_device(ctx, store_cap);
  auto d_rec_begin = to_device(ctx, rec_begin), d_rec_cap = to_device(ctx, rec_cap);
  Buffer<int> queue(ctx, 2), status(ctx, nobj), root(ctx, nobj), target(ctx, nobj), npaths(ctx, nobj), nstore(ctx, nobj);
  Buffer<float> max_daf(ctx, nobj);
  Buffer<int> lists(ctx, 5 * F), store(ctx, store_total), rec_start(ctx, rec_total), rec_len(ctx, rec_total);
  Buffer<unsigned long long> wide(ctx, F), side(ctx, 2 * F), work(ctx, 4), profile(ctx, 8LL * nobj);
  queue.zero();
  status.zero();
  work.zero();

  EngineArgs a{};
  a.arena_offset = d_arena_offset.data(); a.arena_dims = d_arena_dims.data(); a.obj_arena = d_obj_arena.data();
  a.mask = mask.data(); a.dbf = dbf.data(); a.pdrf = pdrf.data(); a.dist = dist.data(); a.daf = daf.data();
  a.flags = flags.data(); a.alive = alive.data(); a.key = key.data();
  a.nobj = nobj; a.obj_begin = d_obj_begin.data(); a.obj_count = d_obj_count.data(); a.vox = vox.data();
  a.schedule = d_schedule.data(); a.queue = queue.data(); a.status = status.data();
  a.lists = lists.data(); a.wide = wide.data(); a.side = side.data(); a.F = F;
  a.border_root = d_border_root.data(); a.M = d_M.data(); a.pdrf_scale = float(t.pdrf_scale); a.squarings = squarings;
  a.exponent = float(exponent);
  a.fix_branching = opt.fix_branching ? 1 : 0;
  a.free_radius = d_free_radius.data();
  a.soma_radius = d_soma_radius.data();
  a.soma_scale = float(t.soma_scale);
  a.soma_constant = float(t.soma_constant);
  {
    const double x = aniso[0], y = aniso[1], z = aniso[2];
    const double pairs[3] = {std::sqrt(x * x + y * y), std::sqrt(y * y + z * z), std::sqrt(x * x + z * z)};
    for (int k = 0; k < 6; ++k) a.w[k] = aniso[k / 2];
    for (int k = 6; k < 18; ++k) a.w[k] = float(pairs[(k - 6) / 4]);
    for (int k = 18; k < 26; ++k) a.w[k] = float(std::sqrt(x * x + y * y + z * z));
  }
  a.root = root.data(); a.target = target.data(); a.max_daf = max_daf.data();
  a.manual_begin = d_manual_begin.data(); a.manual_count = d_manual_count.data(); a.manual = d_manual.data();
  a.after_begin = d_after_begin.data(); a.after_count = d_after_count.data(); a.after = d_after.data();
  a.max_paths = d_max_paths.data(); a.store = store.data(); a.store_begin = d_store_begin.data(); a.store_cap = d_store_cap.data();
  a.rec_start = rec_start.data(); a.rec_len = rec_len.data(); a.rec_begin = d_rec_begin.data(); a.rec_cap = d_rec_cap.data();
  a.npaths = npaths.data(); a.nstore = nstore.data(); a.work = work.data(); a.profile = profile.data();
  a.wx = aniso[0]; a.wy = aniso[1]; a.wz = aniso[2];
  a.scale = float(t.scale); a.constant = float(t.constant);
  a.delta = std::min({aniso[0], aniso[1], aniso[2]});
  a.round_limit = 0;
  if (const char *e = std::getenv("BROOK_B200_TEST_ROUND_LIMIT")) a.round_limit = std::atoll(e);  // test knob
  a.rail_band = kRailBand;
  a.grid_percent = ctx.engine_percent;
  if (const char *e = std::getenv("BROOK_B200_RAIL_BAND")) a.rail_band = float(std::atof(e));  // tuning knob

  clock.mark("state");
  const int ctas = tune.trace_cluster_ctas == kWideClusterCtas || tune.trace_cluster_ctas == kClusterCtas
                       ? tune.trace_cluster_ctas
                       : cluster_ctas(largest, F);
  int prepare_ctas = ctas;
  if (const char *e = std::getenv("BROOK_B200_PREPARE_CLUSTER_CTAS")) {  // tuning knob: 4 or 8
    const int v = std::atoi(e);
    if (v == kClusterCtas || v == kWideClusterCtas) prepare_ctas = v;
  }
  int lone_percent = tune.lone_first_percent >= 0 ? tune.lone_first_percent : kLoneFirstPercent;
  if (const char *e = std::getenv("BROOK_B200_LONE_FIRST_PERCENT")) lone_percent = std::atoi(e);  // tuning knob
  lone_percent = std::max(0, std::min(100, lone_percent));
  const char *fields = std::getenv("BROOK_B200_DUMP_FIELDS");
  const bool wide_order = std::getenv("BROOK_B200_WIDE_ORDER_KEY") != nullptr;  // test knob: the 96-bit key path
  OrderPlan orders = plan_target_orders(ctx, F, nobj, largest, wide_order);
  a.order = orders.order.data();
  // the engine's launches, prepare -> target orders -> trace, as one CUDA graph (every buffer is
  // made above; the graph holds kernels, a memset and the stage marks): one submission per call,
  // and the context's executable graph is updated in place while the topology holds
  const char *graph_knob = std::getenv("BROOK_B200_GRAPH");
  const bool as_graph = !fields && !(graph_knob && std::string(graph_knob) == "0");
  auto engine = [&] {
    launch_prepare(a, nbig_prepare, prepare_ctas, s);
    ++ctx.launches;
    clock.mark("prepare");
    if (fields) {
      // diagnostics: the prepared DAF and PDRF (root rails included) as raw float32 files
      const auto hd = daf.download(), hp = pdrf.download(), hb = dbf.download();
      for (auto item : {std::make_pair("daf", &hd), std::make_pair("pdrf", &hp), std::make_pair("dbf", &hb)}) {
        FILE *f = std::fopen((std::string(fields) + "." + item.first).c_str(), "wb");
        if (f) { std::fwrite(item.second->data(), sizeof(float), size_t(N), f); std::fclose(f); }  // the volumes' part
      }
    }
    run_target_orders(ctx, orders, vox.data(), daf.data(), d_obj_begin.data());
    BK_CUDA(cudaMemsetAsync(queue.data(), 0, 2 * sizeof(int), s));
    clock.mark("order");
    launch_trace(a, nbig_trace, ctas, lone_percent, s);
    ++ctx.launches;
    clock.mark("trace");
  };
  if (as_graph) {
    const auto graph_start = std::chrono::steady_clock::now();
    prepare_engine_launches(prepare_ctas, ctas, s);  // device queries, before the capture
    BK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    clock.capturing(true);
    try {
      engine();
    } catch (...) {
      clock.capturing(false);
      cudaGraph_t broken = nullptr;
      cudaStreamEndCapture(s, &broken);
      if (broken) cudaGraphDestroy(broken);
      cudaGetLastError();
      throw;
    }
    clock.capturing(false);
    cudaGraph_t graph = nullptr;
    BK_CUDA(cudaStreamEndCapture(s, &graph));
    const auto captured = std::chrono::steady_clock::now();
    ctx.launch_graph(graph);
    const auto launched = std::chrono::steady_clock::now();
    ctx.stats["host_ms_graph_capture"] = std::chrono::duration<double, std::milli>(captured - graph_start).count();
    ctx.stats["host_ms_graph_launch"] = std::chrono::duration<double, std::milli>(launched - captured).count();
  } else {
    engine();
  }

  // ---- results
  const auto st_host = status.download();
  for (int o = 0; o < nobj; ++o)
    if (st_host[o] != kOk) {
      static const char *what[] = {"ok", "a loop bound was reached", "no rail reachable from a target", "path store full",
                                   "path records full"};
      throw std::runtime_error(std::string("tracing failed: ") + what[std::min(st_host[o], 4)]);
    }
  const auto np = npaths.download(), ns = nstore.download();
  const char *dump = std::getenv("BROOK_B200_DUMP");
  std::vector<long long> vdst(nobj), rdst(nobj);
  long long vt = 0, rt = 0;
  for (int o = 0; o < nobj; ++o) { vdst[o] = vt; vt += ns[o]; rdst[o] = rt; rt += np[o]; }
  Buffer<int> cstore(ctx, std::max(vt, 1LL)), cstart(ctx, std::max(rt, 1LL)), clen(ctx, std::max(rt, 1LL));
  auto d_vdst = to_device(ctx, vdst), d_rdst = to_device(ctx, rdst);
  gather_store<<<nobj, 256, 0, s>>>(store.data(), d_store_begin.data(), d_vdst.data(), nstore.data(), nobj, cstore.data());
  ++ctx.launches;
  gather_records<<<nobj, 256, 0, s>>>(rec_start.data(), rec_len.data(), d_rec_begin.data(), d_rdst.data(), npaths.data(),
                                      nobj, cstart.data(), clen.data()); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  const auto hstart = cstart.download(rt), hlen = clen.download(rt);
  if (dump && *dump) {
    const auto hstore = cstore.download(vt);
    // diagnostics: the intermediate results a parity investigation compares with the oracle
    FILE *f = std::fopen(dump, "w");
    if (f) {
      const auto hroot = root.download(), htarget = target.download();
      const auto hmax = max_daf.download();
      for (size_t v = 0; v < vs.size(); ++v) {
        const auto &st = vs[v];
        if (st.empty) continue;
        for (int64_t id = 1; id <= st.cc.count; ++id) {
          std::fprintf(f, "borders %zu %lld", v, (long long)id);
          for (const auto &p : st.borders[id]) std::fprintf(f, " %lld,%lld,%lld", (long long)p[0], (long long)p[1], (long long)p[2]);
          std::fprintf(f, "\n");
        }
      }
      const auto hprof = profile.download();
      for (int o = 0; o < nobj; ++o) {
        const unsigned long long *pr = hprof.data() + 8LL * o;
        std::fprintf(f, "object %d volume %d id %u voxels %d root %d target %d max_daf %.9g paths %d "
                     "t0 %llu t1 %llu target_ns %llu rail_ns %llu back_ns %llu inval_ns %llu rail_rounds %llu inval_rounds %llu\n",
                     o, objects[o].volume, objects[o].id, obj_count[o], hroot[o], htarget[o], hmax[o], np[o], pr[0], pr[1],
                     pr[2], pr[3], pr[4], pr[5], pr[6], pr[7]);
        for (int p = 0; p < np[o]; ++p) {
          std::fprintf(f, "path %d %d:", o, p);
          for (int q = 0; q < hlen[rdst[o] + p]; ++q) std::fprintf(f, " %d", hstore[vdst[o] + hstart[rdst[o] + p] + q]);
          std::fprintf(f, "\n");
        }
      }
      std::fclose(f);
    }
  }
  // skeletons: per volume, one per original label (first seen in id order) whose objects made a
  // path of two or more vertices; the label's objects contribute in id order
  AssemblyPaths ap;
  std::vector<std::vector<int64_t>> group_labels(vs.size());
  std::vector<int> group_begin(vs.size() + 1, 0);
  for (size_t v = 0; v < vs.size(); ++v) {
    auto &st = vs[v];
    group_begin[v] = ap.groups;
    if (st.empty) continue;
    std::vector<int64_t> &label_order = group_labels[v];
    std::vector<std::vector<int>> label_objects;
    for (int64_t id = 1; id <= st.cc.count; ++id) {
      const int o = st.object_of[id];
      if (o < 0) continue;
      bool has_edge = false;
      for (int p = 0; p < np[o]; ++p) has_edge |= hlen[rdst[o] + p] >= 2;
      if (!has_edge) continue;
      const int64_t label = st.cc.mapping[id];
      auto it = std::find(label_order.begin(), label_order.end(), label);
      if (it == label_order.end()) { label_order.push_back(label); label_objects.push_back({o}); }
      else label_objects[it - label_order.begin()].push_back(o);
    }
    for (size_t j = 0; j < label_order.size(); ++j, ++ap.groups)
      for (int o : label_objects[j])
        for (int p = 0; p < np[o]; ++p) {
          const int len = hlen[rdst[o] + p];
          if (len < 2) continue;
          ap.src.push_back(int(vdst[o] + hstart[rdst[o] + p]));
          ap.len.push_back(len);
          ap.group.push_back(ap.groups);
          ap.volume.push_back(obj_arena[o]);
        }
  }
  group_begin[vs.size()] = ap.groups;
  std::vector<long long> arena_off(arenas);
  std::vector<std::array<int, 3>> arena_dim(arenas), arena_origin(arenas, {0, 0, 0});
  for (size_t r = 0; r < arenas; ++r) {
    arena_off[r] = arena_offset[r];
    arena_dim[r] = {arena_dims[3 * r], arena_dims[3 * r + 1], arena_dims[3 * r + 2]};
  }
  for (size_t v = 0; v < vs.size(); ++v) arena_origin[v] = vs[v].origin;
  for (size_t j = 0; j < somas.size(); ++j)
    for (int k = 0; k < 3; ++k) arena_origin[vs.size() + j][k] = somas[j].lo[k] + vs[somas[j].volume].origin[k];
  AssemblyResult asmb = assemble(ctx, cstore.data(), dbf.data(), ap, arena_off, arena_dim, arena_origin, aniso);
  const long long V = asmb.vertex_offsets.back(), E = asmb.edge_offsets.back();
  std::vector<float> hvert, hrad;
  std::vector<uint32_t> hedge;
  if (!opt.device_output) {
    hvert.resize(3 * V);
    hrad.resize(V);
    hedge.resize(2 * E);
    if (V) {
      BK_CUDA(cudaMemcpyAsync(hvert.data(), asmb.vertices.data(), hvert.size() * sizeof(float), cudaMemcpyDeviceToHost, s));
      BK_CUDA(cudaMemcpyAsync(hrad.data(), asmb.radii.data(), hrad.size() * sizeof(float), cudaMemcpyDeviceToHost, s));
    }
    if (E) BK_CUDA(cudaMemcpyAsync(hedge.data(), asmb.edges.data(), hedge.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  }
  for (size_t v = 0; v < vs.size(); ++v) {
    Packed &out = results[v];
    // a volume's skeletons are one contiguous range (groups are volume-major; a group without
    // edges has no vertices either)
    const int64_t vbase = asmb.vertex_offsets[group_begin[v]], ebase = asmb.edge_offsets[group_begin[v]];
    const int64_t vend = asmb.vertex_offsets[group_begin[v + 1]], eend = asmb.edge_offsets[group_begin[v + 1]];
    for (int g = group_begin[v]; g < group_begin[v + 1]; ++g) {
      if (asmb.edge_offsets[g + 1] == asmb.edge_offsets[g]) continue;
      out.labels.push_back(group_labels[v][g - group_begin[v]]);
      out.vertex_offsets.push_back(asmb.vertex_offsets[g + 1] - vbase);
      out.edge_offsets.push_back(asmb.edge_offsets[g + 1] - ebase);
    }
    if (opt.device_output) {
      out.device_vertices = std::make_shared<DeviceStorage>(size_t(vend - vbase) * 3 * sizeof(float), ctx.device());
      out.device_radii = std::make_shared<DeviceStorage>(size_t(vend - vbase) * sizeof(float), ctx.device());
      out.device_edges = std::make_shared<DeviceStorage>(size_t(eend - ebase) * 2 * sizeof(uint32_t), ctx.device());
      if (vend > vbase) {
        BK_CUDA(cudaMemcpyAsync(out.device_vertices->ptr, asmb.vertices.data() + 3 * vbase, out.device_vertices->bytes,
                                cudaMemcpyDeviceToDevice, s));
        BK_CUDA(cudaMemcpyAsync(out.device_radii->ptr, asmb.radii.data() + vbase, out.device_radii->bytes,
                                cudaMemcpyDeviceToDevice, s));
      }
      if (eend > ebase)
        BK_CUDA(cudaMemcpyAsync(out.device_edges->ptr, asmb.edges.data() + 2 * ebase, out.device_edges->bytes,
                                cudaMemcpyDeviceToDevice, s));
    }
  }
  ctx.synchronize();
  if (!opt.device_output)
    for (size_t v = 0; v < vs.size(); ++v) {
      Packed &out = results[v];
      const int64_t vbase = asmb.vertex_offsets[group_begin[v]], ebase = asmb.edge_offsets[group_begin[v]];
      const int64_t vend = asmb.vertex_offsets[group_begin[v + 1]], eend = asmb.edge_offsets[group_begin[v + 1]];
      out.vertices.assign(hvert.begin() + 3 * vbase, hvert.begin() + 3 * vend);
      out.radii.assign(hrad.begin() + vbase, hrad.begin() + vend);
      out.edges.assign(hedge.begin() + 2 * ebase, hedge.begin() + 2 * eend);
    }
  clock.mark("assembly");
  clock.finish();
  {
    // the device memory pool after the call (bytes): reserved from the driver, and in use at the high-water mark
    cudaMemPool_t pool;
    BK_CUDA(cudaDeviceGetDefaultMemPool(&pool, ctx.device()));
    uint64_t reserved = 0, high = 0;
    BK_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    BK_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &high));
    ctx.stats["pool_reserved_bytes"] = double(reserved);
    ctx.stats["pool_used_high_bytes"] = double(high);
    ctx.stats["context_peak_bytes"] = double(ctx.peak_bytes());  // most this call held at once
  }
  const auto w = work.download();
  ctx.stats["paths"] = double(w[3]);
  ctx.stats["railroad_settled"] = double(w[0]);
  ctx.stats["railroad_touched"] = double(w[1]);
  ctx.stats["invalidated"] = double(w[2]);
  ctx.stats["objects"] = nobj;
  ctx.stats["soma_candidates"] = double(somas.size());
  {
    long long n = 0;
    for (const auto &sa : somas) n += sa.soma ? 1 : 0;
    ctx.stats["somata"] = double(n);
  }
  ctx.stats["voxels"] = double(N);
  ctx.stats["foreground"] = double(F);
  ctx.stats["launches"] = double(ctx.launches);
  long long kmax = 0;
  for (const auto &st : vs) kmax = std::max<long long>(kmax, st.cc.count);
  ctx.stats["label_bytes"] = kmax <= 0xFF ? 1 : kmax <= 0xFFFF ? 2 : kmax <= 0xFFFFFFFFLL ? 4 : 8;
  double input_bytes = 0;
  for (size_t v = 0; v < vs.size(); ++v)
    if (volumes[v].d.n() > 0 && double(volumes[v].d.n()) > opt.dust)  // the volumes the call read
      input_bytes += double(volumes[v].d.n()) * double(label_bytes(volumes[v].dtype));
  ctx.stats["input_bytes"] = input_bytes;
  ctx.stats["path_vertices"] = double(vt);
  ctx.stats["vertices"] = double(V);
  ctx.stats["edges"] = double(E);
  return results;
}

}  // namespace bk
