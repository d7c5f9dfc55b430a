// Hole filling of components (the reference's fill_all_holes, holes.cu:38-67, called after the
// components and their boxes in skeletonize.cu:86-90 and batch.cu:217-220).
//
// The reference fills components one at a time in ascending id: the voxels of the current ids equal
// to the id, within the id's original box, form a mask; the mask's voids (background not
// 6-connected to a face of the box) are filled and painted with the id; a painted voxel that held
// another component disables that component, which is then skipped. An id that is not disabled
// still holds exactly its own voxels when its turn comes (only its own fill paints it, and a fill
// that painted one of its voxels would have disabled it), so every component's filled set F(L)
// depends on the original ids alone. Here all F(L) are computed at once, independent of order:
//
//   per eligible component, two bit planes over its box (32 voxels of a row per word): `free`
//   (voxels that are not the component) and `reach` (free voxels 6-connected to the box's faces),
//   seeded with the free face voxels and closed by rounds of three sweeps: rows (a warp per row,
//   runs filled inside a word by shift-doubling and across words by a warp scan), columns along y
//   and columns along z (a thread per column of words, both directions). A round that changes no
//   word ends the flood. The holes are free & ~reach.
//
// The holes are then listed as (voxel, component, id the voxel holds) and the order-dependent part
// is resolved on the host: ascending, a component is filled unless an earlier filled component's
// holes held one of its voxels; a voxel ends with the last (largest) filled component that holds it
// in its holes; the count is the filled components' hole voxels.
#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <vector>

#include "kernels.hpp"

namespace bk {
namespace {

// One component's box: its id, the volume it lies in and the box's word layout.
struct HoleJob {
  long long base;        // first word of its planes
  long long vol_offset;  // flat index of the volume's first voxel
  int vsx, vsy;          // volume extents (x, y)
  int lx, ly, lz;        // box low corner
  int bx, by, bz;        // box extents
  int words;             // words per row: ceil(bx / 32)
  uint32_t id;
};

__device__ int job_of(const HoleJob *jobs, int njobs, long long word) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {  // the last job whose base is <= word
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].base <= word) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// free / reach words of every job: one warp per word, lane i the voxel x = 32 w + i
__global__ void hole_planes(const uint32_t *__restrict__ ids, const HoleJob *__restrict__ jobs, int njobs,
                            long long total_words, uint32_t *__restrict__ freew, uint32_t *__restrict__ reach) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long w = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < total_words; w += warps) {
    const HoleJob J = jobs[job_of(jobs, njobs, w)];
    long long r = w - J.base;
    const int xw = int(r % J.words);
    r /= J.words;
    const int y = int(r % J.by), z = int(r / J.by);
    const int x = xw * 32 + lane;
    bool f = false, seed = false;
    if (x < J.bx) {
      const long long v = J.vol_offset + (long long)(J.lx + x) + (long long)J.vsx * ((J.ly + y) + (long long)J.vsy * (J.lz + z));
      f = ids[v] != J.id;
      seed = f && (x == 0 || x == J.bx - 1 || y == 0 || y == J.by - 1 || z == 0 || z == J.bz - 1);
    }
    const uint32_t fw = __ballot_sync(0xffffffffu, f), rw = __ballot_sync(0xffffffffu, seed);
    if (lane == 0) {
      freew[w] = fw;
      reach[w] = rw;
    }
  }
}

// Bits of f reachable from the bits of r (r within f) through contiguous bits of f, both ways.
__device__ __forceinline__ uint32_t fill_word(uint32_t r, uint32_t f) {
  uint32_t gu = r & f, pu = f, gd = r & f, pd = f;
#pragma unroll
  for (int s = 1; s < 32; s <<= 1) {
    gu |= pu & (gu << s);
    pu &= pu << s;
    gd |= pd & (gd >> s);
    pd &= pd >> s;
  }
  return gu | gd;
}

__device__ __forceinline__ uint32_t run_from_low(uint32_t f) { return f & ~(f + 1u); }
__device__ __forceinline__ uint32_t run_from_high(uint32_t f) { return __brev(run_from_low(__brev(f))); }

// The x sweep: one warp per row; 32 words at a time, carries across the chunks left to right and
// then right to left.
__global__ void hole_rows(const HoleJob *__restrict__ jobs, int njobs, const long long *__restrict__ row_begin,
                          long long total_rows, const uint32_t *__restrict__ freew, uint32_t *__restrict__ reach,
                          int *changed) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  bool any = false;
  for (long long row = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < total_rows; row += warps) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (row_begin[mid] <= row) lo = mid;
      else hi = mid - 1;
    }
    const HoleJob J = jobs[lo];
    const long long first = J.base + (row - row_begin[lo]) * J.words;
    for (int pass = 0; pass < 2; ++pass) {
      // pass 0: chunks left to right, carrying rightward; pass 1: right to left, carrying leftward
      const int chunks = (J.words + 31) / 32;
      uint32_t carry = 0;
      for (int c = 0; c < chunks; ++c) {
        const int chunk = pass == 0 ? c : chunks - 1 - c;
        const int j = chunk * 32 + lane;
        const bool in = j < J.words;
        const uint32_t f = in ? freew[first + j] : 0u;
        const uint32_t r0 = in ? reach[first + j] : 0u;
        uint32_t r = fill_word(r0, f);
        const bool full = f == 0xffffffffu;
        // rightward: a word passes a carry on when its top bit is reached, or when it is full and
        // one came in (an inclusive scan of (generate, propagate) over the lanes)
        uint32_t gen = (r >> 31) & 1u, prop = full ? 1u : 0u;
        if (pass == 0) {
          if (lane == 0) gen |= prop & carry;
#pragma unroll
          for (int s = 1; s < 32; s <<= 1) {
            const uint32_t g2 = __shfl_up_sync(0xffffffffu, gen, s), p2 = __shfl_up_sync(0xffffffffu, prop, s);
            if (lane >= s) { gen |= prop & g2; prop &= p2; }
          }
          uint32_t in_left = __shfl_up_sync(0xffffffffu, gen, 1);
          if (lane == 0) in_left = carry;
          if (in_left) r |= run_from_low(f);
          carry = __shfl_sync(0xffffffffu, gen, 31);
        } else {
          gen = r & 1u;
          prop = full ? 1u : 0u;
          if (lane == 31) gen |= prop & carry;
#pragma unroll
          for (int s = 1; s < 32; s <<= 1) {
            const uint32_t g2 = __shfl_down_sync(0xffffffffu, gen, s), p2 = __shfl_down_sync(0xffffffffu, prop, s);
            if (lane + s < 32) { gen |= prop & g2; prop &= p2; }
          }
          uint32_t in_right = __shfl_down_sync(0xffffffffu, gen, 1);
          if (lane == 31) in_right = carry;
          if (in_right) r |= run_from_high(f);
          carry = __shfl_sync(0xffffffffu, gen, 0);
        }
        if (in && r != r0) {
          reach[first + j] = r;
          any = true;
        }
      }
    }
  }
  if (__any_sync(0xffffffffu, any) && lane == 0) atomicOr(changed, 1);
}

// The y (axis 1) or z (axis 2) sweep: one thread per column of words, up then down.
__global__ void hole_columns(const HoleJob *__restrict__ jobs, int njobs, const long long *__restrict__ col_begin,
                             long long total_cols, int axis, const uint32_t *__restrict__ freew,
                             uint32_t *__restrict__ reach, int *changed) {
  bool any = false;
  for (long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x; col < total_cols;
       col += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (col_begin[mid] <= col) lo = mid;
      else hi = mid - 1;
    }
    const HoleJob J = jobs[lo];
    const long long c = col - col_begin[lo];
    long long start, stride;
    int length;
    if (axis == 1) {  // columns (w, z), along y
      const long long w = c % J.words, z = c / J.words;
      start = J.base + w + (long long)J.words * J.by * z;
      stride = J.words;
      length = J.by;
    } else {  // columns (w, y), along z
      start = J.base + c;  // c = w + words * y
      stride = (long long)J.words * J.by;
      length = J.bz;
    }
    uint32_t prev = 0;
    for (int k = 0; k < length; ++k) {
      const long long i = start + k * stride;
      const uint32_t r0 = reach[i], r = r0 | (prev & freew[i]);
      if (r != r0) { reach[i] = r; any = true; }
      prev = r;
    }
    prev = 0;
    for (int k = length - 1; k >= 0; --k) {
      const long long i = start + k * stride;
      const uint32_t r0 = reach[i], r = r0 | (prev & freew[i]);
      if (r != r0) { reach[i] = r; any = true; }
      prev = r;
    }
  }
  if (any) atomicOr(changed, 1);
}

// Per job the number of hole voxels (free & ~reach), and with `out` set the holes themselves as
// (flat index, job, id the voxel holds), each job's from out_begin[job] on.
__global__ void hole_list(const uint32_t *__restrict__ ids, const HoleJob *__restrict__ jobs, int njobs,
                          long long total_words, const uint32_t *__restrict__ freew, const uint32_t *__restrict__ reach,
                          unsigned long long *counts, const long long *out_begin, int *out_voxel, int *out_job,
                          uint32_t *out_held) {
  for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < total_words;
       w += (long long)gridDim.x * blockDim.x) {
    uint32_t h = freew[w] & ~reach[w];
    if (!h) continue;
    const int j = job_of(jobs, njobs, w);
    const HoleJob J = jobs[j];
    const unsigned long long at = atomicAdd(counts + j, (unsigned long long)__popc(h));
    if (!out_voxel) continue;
    long long r = w - J.base;
    const int xw = int(r % J.words);
    r /= J.words;
    const int y = int(r % J.by), z = int(r / J.by);
    long long k = out_begin[j] + (long long)at;
    while (h) {
      const int bit = __ffs(h) - 1;
      h &= h - 1;
      const long long v = J.vol_offset + (long long)(J.lx + xw * 32 + bit) +
                          (long long)J.vsx * ((J.ly + y) + (long long)J.vsy * (J.lz + z));
      out_voxel[k] = int(v);
      out_job[k] = j;
      out_held[k] = ids[v];
      ++k;
    }
  }
}

__global__ void paint_voxels(uint32_t *ids, const int *voxel, const uint32_t *value, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) ids[voxel[i]] = value[i];
}

constexpr int kMaxRounds = 1 << 20;  // a round that changes nothing ends the flood long before

}  // namespace

Voids component_voids(Context &ctx, const uint32_t *ids, const std::vector<VoidBox> &boxes) {
  cudaStream_t s = ctx.stream();
  Voids out;
  out.count.assign(boxes.size(), 0);
  // the voids of every box, in batches of at most `budget` plane words (256 MiB a plane; a larger
  // box runs alone)
  constexpr long long budget = 1LL << 26;
  size_t next = 0;
  while (next < boxes.size()) {
    std::vector<HoleJob> jobs;
    std::vector<size_t> job_box;
    std::vector<long long> row_begin, ycol_begin, zcol_begin;
    long long words = 0, rows = 0, ycols = 0, zcols = 0;
    while (next < boxes.size()) {
      const VoidBox &e = boxes[next];
      const Box &b = e.box;
      HoleJob J{};
      J.vol_offset = e.vol_offset;
      J.vsx = e.d.sx;
      J.vsy = e.d.sy;
      J.lx = b.lo[0]; J.ly = b.lo[1]; J.lz = b.lo[2];
      J.bx = b.hi[0] - b.lo[0] + 1; J.by = b.hi[1] - b.lo[1] + 1; J.bz = b.hi[2] - b.lo[2] + 1;
      J.words = (J.bx + 31) / 32;
      J.id = e.id;
      const long long w = (long long)J.words * J.by * J.bz;
      if (!jobs.empty() && words + w > budget) break;
      J.base = words;
      jobs.push_back(J);
      job_box.push_back(next++);
      row_begin.push_back(rows);
      ycol_begin.push_back(ycols);
      zcol_begin.push_back(zcols);
      words += w;
      rows += (long long)J.by * J.bz;
      ycols += (long long)J.words * J.bz;
      zcols += (long long)J.words * J.by;
    }
    const int njobs = int(jobs.size());
    auto d_jobs = to_device(ctx, jobs);
    auto d_rows = to_device(ctx, row_begin), d_ycols = to_device(ctx, ycol_begin), d_zcols = to_device(ctx, zcol_begin);
    Buffer<uint32_t> freew(ctx, words), reach(ctx, words);
    Buffer<int> changed(ctx, 1);
    const int grid = ctx.sm_count() * 8;
    hole_planes<<<grid, 256, 0, s>>>(ids, d_jobs.data(), njobs, words, freew.data(), reach.data());
    ++ctx.launches;
    BK_CUDA(cudaGetLastError());
    int rounds = 0;
    for (;; ++rounds) {
      if (rounds >= kMaxRounds) throw std::runtime_error("hole filling did not converge (loop bound)");
      changed.zero();
      hole_rows<<<std::max<long long>(1, std::min<long long>(grid, (rows + 7) / 8)), 256, 0, s>>>(
          d_jobs.data(), njobs, d_rows.data(), rows, freew.data(), reach.data(), changed.data());
      hole_columns<<<std::max<long long>(1, std::min<long long>(grid, blocks_for(ycols))), 256, 0, s>>>(
          d_jobs.data(), njobs, d_ycols.data(), ycols, 1, freew.data(), reach.data(), changed.data());
      hole_columns<<<std::max<long long>(1, std::min<long long>(grid, blocks_for(zcols))), 256, 0, s>>>(
          d_jobs.data(), njobs, d_zcols.data(), zcols, 2, freew.data(), reach.data(), changed.data());
      ctx.launches += 3;
      BK_CUDA(cudaGetLastError());
      if (!changed.download(1)[0]) break;
    }
    ctx.stats["hole_rounds"] += rounds + 1;
    Buffer<unsigned long long> counts(ctx, njobs);
    counts.zero();
    hole_list<<<grid, 256, 0, s>>>(ids, d_jobs.data(), njobs, words, freew.data(), reach.data(), counts.data(), nullptr,
                                   nullptr, nullptr, nullptr);
    ++ctx.launches;
    BK_CUDA(cudaGetLastError());
    const auto hc = counts.download();
    std::vector<long long> out_begin(njobs + 1, 0);
    for (int j = 0; j < njobs; ++j) out_begin[j + 1] = out_begin[j] + (long long)hc[j];
    const long long H = out_begin[njobs];
    if (H == 0) continue;
    if (H >= (1LL << 31)) throw std::invalid_argument("too many hole voxels in one call");
    counts.zero();
    auto d_begin = to_device(ctx, out_begin);
    Buffer<int> ov(ctx, H), oj(ctx, H);
    Buffer<uint32_t> oh(ctx, H);
    hole_list<<<grid, 256, 0, s>>>(ids, d_jobs.data(), njobs, words, freew.data(), reach.data(), counts.data(),
                                   d_begin.data(), ov.data(), oj.data(), oh.data());
    ++ctx.launches;
    BK_CUDA(cudaGetLastError());
    const auto hv = ov.download(), hj = oj.download();
    const auto hh = oh.download();
    for (long long k = 0; k < H; ++k) {
      const size_t box = job_box[hj[k]];
      out.voxel.push_back(hv[k]);
      out.box.push_back(int(box));
      out.held.push_back(hh[k]);
      out.count[box] += 1;
    }
  }
  return out;
}

long long fill_holes(Context &ctx, uint32_t *ids, const std::vector<HoleVolume> &volumes) {
  cudaStream_t s = ctx.stream();
  // eligible components: a box of three or more voxels along every axis that the component does
  // not fill (no other box can enclose a void)
  std::vector<VoidBox> eligible;
  std::vector<size_t> volume_of;
  for (size_t v = 0; v < volumes.size(); ++v) {
    const auto &boxes = *volumes[v].boxes;
    for (size_t id = 1; id < boxes.size(); ++id) {
      const Box &b = boxes[id];
      if (!b.count) continue;
      const int bx = b.hi[0] - b.lo[0] + 1, by = b.hi[1] - b.lo[1] + 1, bz = b.hi[2] - b.lo[2] + 1;
      const long long n = (long long)bx * by * bz;
      if (bx <= 2 || by <= 2 || bz <= 2 || n == b.count) continue;
      eligible.push_back({volumes[v].offset, volumes[v].d, b, uint32_t(id)});
      volume_of.push_back(v);
    }
  }
  const Voids voids = component_voids(ctx, ids, eligible);
  std::vector<int> hole_voxel, hole_job_volume;
  std::vector<uint32_t> hole_id, hole_held;
  std::vector<std::vector<long long>> filled_of(volumes.size());
  for (size_t v = 0; v < volumes.size(); ++v) filled_of[v].assign(volumes[v].boxes->size(), 0);
  for (size_t k = 0; k < voids.voxel.size(); ++k) {
    const size_t j = size_t(voids.box[k]);
    hole_voxel.push_back(voids.voxel[k]);
    hole_job_volume.push_back(int(volume_of[j]));
    hole_id.push_back(eligible[j].id);
    hole_held.push_back(voids.held[k]);
    filled_of[volume_of[j]][eligible[j].id] += 1;
  }
  if (hole_voxel.empty()) return 0;
  // the order-dependent part, per volume: ascending ids, a component is filled unless disabled by
  // an earlier filled one; the last filled component holding a voxel paints it
  std::vector<std::vector<uint8_t>> disabled(volumes.size());
  for (size_t v = 0; v < volumes.size(); ++v) disabled[v].assign(volumes[v].boxes->size(), 0);
  std::vector<size_t> order(hole_voxel.size());
  for (size_t k = 0; k < order.size(); ++k) order[k] = k;
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
    if (hole_job_volume[a] != hole_job_volume[b]) return hole_job_volume[a] < hole_job_volume[b];
    if (hole_id[a] != hole_id[b]) return hole_id[a] < hole_id[b];
    return hole_voxel[a] < hole_voxel[b];
  });
  long long total = 0;
  std::vector<uint8_t> painted(order.size(), 0);
  for (size_t i = 0; i < order.size();) {
    size_t e = i;
    const int vol = hole_job_volume[order[i]];
    const uint32_t id = hole_id[order[i]];
    while (e < order.size() && hole_job_volume[order[e]] == vol && hole_id[order[e]] == id) ++e;
    if (!disabled[vol][id]) {
      total += filled_of[vol][id];
      for (size_t k = i; k < e; ++k) {
        const uint32_t held = hole_held[order[k]];
        if (held && held != id) disabled[vol][held] = 1;
        painted[k] = 1;
      }
    }
    i = e;
  }
  // per voxel the largest painting id (the list is ascending in id within a volume, and a voxel
  // belongs to one volume)
  std::vector<std::pair<int, uint32_t>> paint;
  for (size_t k = 0; k < order.size(); ++k)
    if (painted[k]) paint.push_back({hole_voxel[order[k]], hole_id[order[k]]});
  std::stable_sort(paint.begin(), paint.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
  std::vector<int> pv;
  std::vector<uint32_t> pid;
  for (size_t k = 0; k < paint.size(); ++k)
    if (k + 1 == paint.size() || paint[k + 1].first != paint[k].first) {
      pv.push_back(paint[k].first);
      pid.push_back(paint[k].second);
    }
  if (!pv.empty()) {
    auto d_v = to_device(ctx, pv);
    auto d_id = to_device(ctx, pid);
    paint_voxels<<<blocks_for((long long)pv.size()), 256, 0, s>>>(ids, d_v.data(), d_id.data(), (long long)pv.size());
    ++ctx.launches;
    BK_CUDA(cudaGetLastError());
  }
  return total;
}

}  // namespace bk
