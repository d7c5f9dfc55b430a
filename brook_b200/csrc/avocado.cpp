// The avocado stage (the reference's fix_avocados, avocado.cpp:223-239, which restates Kimimaro
// 5.8.1's engage_avocado_protection): a pit inside another object (the nucleus inside a soma) is
// merged into that object. Like the reference, the stage works on host copies of one volume's
// component ids and distance field, one candidate at a time in the order of a CPython set; the
// distance field it refreshes after a merging pass comes from the device EDT.
#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <map>
#include <vector>

#include "kernels.hpp"

namespace bk {
namespace {

// A set of non-negative ints that iterates like a CPython 3.12 set of them (hash(k) == k): a table
// of 2^k slots, 8 at first; probe the home slot k & mask and, while 9 more slots fit before the
// table's end, those 9 after it, then jump to (5 i + 1 + perturb) & mask with perturb shifted right
// by 5 bits each jump. A removed key leaves a dummy; a new key takes the last dummy its probe
// passed before an empty slot. An insertion into an empty slot that brings the filled slots to 3/5
// of the table regrows it for 4x the live keys (2x past 50000), keeping the old table's order.
class IntSetPy {
  static constexpr long long kEmpty = -1, kDummy = -2;
  std::vector<long long> slot_ = std::vector<long long>(8, kEmpty);
  long long live_ = 0, filled_ = 0;

  long long mask() const { return (long long)slot_.size() - 1; }
  // where `k` is, else where it goes; `fresh`: a table without dummies or duplicates
  long long probe(long long k, bool fresh) const {
    unsigned long long perturb = (unsigned long long)k, i = (unsigned long long)(k & mask());
    long long dummy = -1;
    for (;;) {
      const unsigned long long run = i + 9 <= (unsigned long long)mask() ? 9 : 0;
      for (unsigned long long j = i; j <= i + run; ++j) {
        const long long e = slot_[j];
        if (e == kEmpty) return dummy >= 0 ? dummy : (long long)j;
        if (fresh) continue;
        if (e == k) return (long long)j;
        if (e == kDummy) dummy = (long long)j;
      }
      perturb >>= 5;
      i = (i * 5 + 1 + perturb) & (unsigned long long)mask();
    }
  }
  void regrow(long long least) {
    long long size = 8;
    while (size <= least) size *= 2;
    if (size == 8 && slot_.size() == 8 && filled_ == live_) return;
    std::vector<long long> old(size, kEmpty);
    old.swap(slot_);
    filled_ = live_;
    for (long long e : old)
      if (e >= 0) slot_[probe(e, true)] = e;
  }
  long long growth() const { return live_ > 50000 ? 2 * live_ : 4 * live_; }

 public:
  long long size() const { return live_; }
  bool has(long long k) const { return slot_[probe(k, false)] == k; }
  void insert(long long k) {
    const long long at = probe(k, false);
    if (slot_[at] == k) return;
    const bool was_empty = slot_[at] == kEmpty;
    slot_[at] = k;
    ++live_;
    if (was_empty && ++filled_ * 5 >= mask() * 3) regrow(growth());
  }
  void erase(long long k) {
    const long long at = probe(k, false);
    if (slot_[at] == k) { slot_[at] = kDummy; --live_; }
  }
  void minus(const IntSetPy &o) {  // a -= o
    for (long long e : o.slot_)
      if (e >= 0) erase(e);
    if (filled_ - live_ > mask() / 4) regrow(growth());
  }
  void plus(const IntSetPy &o) {  // a |= o
    if (&o == this || !o.live_) return;
    if ((filled_ + o.live_) * 5 >= mask() * 3) regrow((live_ + o.live_) * 2);
    if (!filled_ && slot_.size() == o.slot_.size() && o.filled_ == o.live_) {
      *this = o;
      return;
    }
    if (!filled_) {
      filled_ = live_ = o.live_;
      for (long long e : o.slot_)
        if (e >= 0) slot_[probe(e, true)] = e;
      return;
    }
    for (long long e : o.slot_)
      if (e >= 0) insert(e);
  }
  std::vector<long long> in_order() const {
    std::vector<long long> out;
    for (long long e : slot_)
      if (e >= 0) out.push_back(e);
    return out;
  }
};

using Pos = std::array<long long, 3>;

// A box of the volume walked in x-fastest order: fn(crop index, volume index).
struct Crop {
  Pos lo, ext;
  long long n() const { return ext[0] * ext[1] * ext[2]; }
  template <class Fn>
  void each(const VolumeDims &d, Fn fn) const {
    long long c = 0;
    for (long long z = 0; z < ext[2]; ++z)
      for (long long y = 0; y < ext[1]; ++y) {
        long long g = lo[0] + d.sx * ((lo[1] + y) + (long long)d.sy * (lo[2] + z));
        for (long long x = 0; x < ext[0]; ++x) fn(c++, g++);
      }
  }
};

// fill_voids 2.1.2's hole filling of a binary image (1 object, 0 background), returned as 1 inside
// the object or its holes and 0 where the background reaches a face. In 3D the flood starts, on each
// face scanned row after row, from the first background voxel of every background run (a run may
// continue from one row into the next) and spreads over face neighbours; in 2D from every border
// background pixel over edge neighbours.
void fill_holes_of(std::vector<uint8_t> &m, const Pos &e, int dims) {
  std::vector<long long> queue;
  auto index = [&](const Pos &p) { return p[0] + e[0] * (p[1] + e[1] * p[2]); };
  if (dims == 3) {
    static const int faces[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
    for (const auto &f : faces)
      for (long long fixed : {0LL, e[f[2]] - 1}) {
        bool in_run = false;
        for (long long v = 0; v < e[f[1]]; ++v)
          for (long long u = 0; u < e[f[0]]; ++u) {
            Pos p;
            p[f[0]] = u;
            p[f[1]] = v;
            p[f[2]] = fixed;
            const long long i = index(p);
            if (!m[i] && !in_run) queue.push_back(i);
            in_run = !m[i];
          }
      }
    for (long long i : queue) m[i] = 2;
  } else {
    for (long long y = 0; y < e[1]; ++y)
      for (long long x = 0; x < e[0]; ++x) {
        const long long i = x + e[0] * y;
        if (!m[i] && (x == 0 || y == 0 || x == e[0] - 1 || y == e[1] - 1)) { m[i] = 2; queue.push_back(i); }
      }
  }
  for (size_t q = 0; q < queue.size(); ++q) {
    const long long i = queue[q];
    const Pos p{i % e[0], (i / e[0]) % e[1], i / (e[0] * e[1])};
    for (int a = 0; a < dims; ++a)
      for (long long step : {-1LL, 1LL}) {
        Pos r = p;
        r[a] += step;
        if (r[a] < 0 || r[a] >= e[a]) continue;
        const long long j = index(r);
        if (!m[j]) { m[j] = 2; queue.push_back(j); }
      }
  }
  for (auto &v : m) v = v == 2 ? 0 : 1;
}

class AvocadoStage {
 public:
  AvocadoStage(std::vector<uint32_t> &ids, std::vector<float> &dbf, VolumeDims d, size_t table)
      : ids_(ids), dbf_(dbf), d_(d), table_(table) {}

  enum Outcome { kNoCandidate, kNoMerge, kMerged };
  // One pass over the candidates (ids with a voxel deeper than threshold / 2.5 that no earlier
  // pass left unchanged).
  Outcome pass(double threshold) {
    const float cutoff = float(threshold / 2.5);
    const long long n = d_.n();
    std::vector<uint8_t> deep(table_, 0);
    for (long long i = 0; i < n; ++i) deep[dbf_[i] > cutoff ? ids_[i] : 0] = 1;
    IntSetPy candidates;
    for (size_t id = 0; id < table_; ++id)
      if (deep[id]) candidates.insert((long long)id);
    candidates.minus(unchanged_);
    candidates.erase(0);
    if (!candidates.size()) return kNoCandidate;
    boxes();
    IntSetPy still, merged;
    for (long long label : candidates.in_order()) {
      const Crop c{{lo_[label][0], lo_[label][1], lo_[label][2]},
                   {hi_[label][0] - lo_[label][0] + 1, hi_[label][1] - lo_[label][1] + 1,
                    hi_[label][2] - lo_[label][2] + 1}};
      std::vector<uint8_t> m(c.n());
      c.each(d_, [&](long long k, long long g) { m[k] = ids_[g] == uint32_t(label); });
      close_faces(m, c.ext);
      const Pos centre = deepest(m, c);
      const auto po = pit_and_owner(centre);
      const long long pit = po.first, owner = po.second;
      if (pit == owner && !merged.has(pit)) still.insert(pit);
      else {
        still.erase(pit);
        still.erase(owner);
        merged.insert(pit);
        merged.insert(owner);
        c.each(d_, [&](long long k, long long g) { m[k] |= ids_[g] == uint32_t(owner); });
      }
      fill_holes_of(m, c.ext, 3);
      c.each(d_, [&](long long k, long long g) { if (m[k]) ids_[g] = uint32_t(owner); });
    }
    unchanged_.plus(still);
    return merged.size() ? kMerged : kNoMerge;
  }

 private:
  std::vector<uint32_t> &ids_;
  std::vector<float> &dbf_;
  VolumeDims d_;
  size_t table_;
  IntSetPy unchanged_;
  std::vector<Pos> lo_, hi_;

  void boxes() {
    lo_.assign(table_, {LLONG_MAX, LLONG_MAX, LLONG_MAX});
    hi_.assign(table_, {-1, -1, -1});
    long long g = 0;
    for (long long z = 0; z < d_.sz; ++z)
      for (long long y = 0; y < d_.sy; ++y)
        for (long long x = 0; x < d_.sx; ++x, ++g) {
          const uint32_t id = ids_[g];
          if (!id) continue;
          const Pos p{x, y, z};
          for (int a = 0; a < 3; ++a) { lo_[id][a] = std::min(lo_[id][a], p[a]); hi_[id][a] = std::max(hi_[id][a], p[a]); }
        }
  }

  // The crop's six faces each filled as an image, in the order (x, y | z), (x, z | y), (y, z | x),
  // low side then high side.
  static void close_faces(std::vector<uint8_t> &m, const Pos &e) {
    static const int faces[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
    for (const auto &f : faces)
      for (long long fixed : {0LL, e[f[2]] - 1}) {
        const Pos pe{e[f[0]], e[f[1]], 1};
        std::vector<uint8_t> image(pe[0] * pe[1]);
        auto at = [&](long long u, long long v) {
          Pos p;
          p[f[0]] = u;
          p[f[1]] = v;
          p[f[2]] = fixed;
          return p[0] + e[0] * (p[1] + e[1] * p[2]);
        };
        for (long long v = 0; v < pe[1]; ++v)
          for (long long u = 0; u < pe[0]; ++u) image[u + pe[0] * v] = m[at(u, v)];
        fill_holes_of(image, pe, 2);
        for (long long v = 0; v < pe[1]; ++v)
          for (long long u = 0; u < pe[0]; ++u) m[at(u, v)] = image[u + pe[0] * v];
      }
  }

  // np.argmax of mask * DBF over the crop in x-fastest order (the first maximum; a NaN wins), as a
  // volume position.
  Pos deepest(const std::vector<uint8_t> &m, const Crop &c) const {
    long long best = 0;
    float top = 0.0f;
    bool first = true;
    c.each(d_, [&](long long k, long long g) {
      const float v = float(m[k]) * dbf_[g];
      if (first) { top = v; first = false; return; }
      if (!(v <= top) && !std::isnan(top)) { top = v; best = k; }
    });
    return {c.lo[0] + best % c.ext[0], c.lo[1] + (best / c.ext[0]) % c.ext[1], c.lo[2] + best / (c.ext[0] * c.ext[1])};
  }

  // Six rays from the centre: up each axis to the volume's last voxel, down each to coordinate 1;
  // a ray ends at background or at the first voxel of another id, which counts as a hit. With three
  // or more hits, the most hit id (the least of them on a tie) owns the pit, unless more rays than
  // allowed (none of three hits, one of four or more) went elsewhere.
  std::pair<long long, long long> pit_and_owner(const Pos &c) const {
    auto at = [&](const Pos &p) { return ids_[p[0] + d_.sx * (p[1] + (long long)d_.sy * p[2])]; };
    const long long pit = at(c);
    const long long ext[3] = {d_.sx, d_.sy, d_.sz};
    std::map<long long, int> hits;
    int rays = 0;
    for (int a = 0; a < 3; ++a)
      for (int dir : {1, -1})
        for (Pos p = c; dir > 0 ? p[a] < ext[a] : p[a] > 0; p[a] += dir) {
          const long long v = at(p);
          if (!v) break;
          if (v != pit) { ++hits[v]; ++rays; break; }
        }
    if (rays < 3) return {pit, pit};
    long long owner = pit;
    int most = 0;
    for (const auto &h : hits)
      if (h.second > most) { owner = h.first; most = h.second; }
    const int allowed = rays > 3 ? 1 : 0;
    return rays - most > allowed ? std::make_pair(pit, pit) : std::make_pair(pit, owner);
  }
};

}  // namespace

int fix_avocados(Context &ctx, uint32_t *ids, float *dbf, VolumeDims d, ComponentsResult &cc, double threshold,
                 const float aniso[3], bool black_border) {
  const long long n = d.n();
  if (!n || !cc.count) return 0;
  cudaStream_t s = ctx.stream();
  std::vector<uint32_t> labels(n);
  std::vector<float> field(n);
  BK_CUDA(cudaMemcpyAsync(labels.data(), ids, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  BK_CUDA(cudaMemcpyAsync(field.data(), dbf, n * sizeof(float), cudaMemcpyDeviceToHost, s));
  ctx.synchronize();
  const std::vector<uint32_t> before = labels;
  const size_t table = size_t(cc.count) + 1;
  AvocadoStage stage(labels, field, d, table);
  Buffer<uint32_t> current;
  Buffer<float> refreshed;
  // up to 20 passes: a pass without candidates ends the stage uncounted, one that merged nothing
  // ends it counted, one that merged refreshes the field (avocado.cpp:92-115)
  int passes = 0;
  for (; passes < 20; ++passes) {
    const auto outcome = stage.pass(threshold);
    if (outcome == AvocadoStage::kNoCandidate) break;
    if (outcome == AvocadoStage::kNoMerge) { ++passes; break; }
    if (!current.data()) { current = Buffer<uint32_t>(ctx, n); refreshed = Buffer<float>(ctx, n); }
    current.upload(labels);
    edt(ctx, current.data(), d, aniso, black_border, 3, refreshed.data());
    BK_CUDA(cudaMemcpyAsync(field.data(), refreshed.data(), n * sizeof(float), cudaMemcpyDeviceToHost, s));
    ctx.synchronize();
  }
  // ids renumbered by first voxel; a new id maps to the original label of the old id at its last
  // run start in index order (fastremap's renumber and get_mapping, avocado.cpp:117-131)
  std::vector<uint32_t> renumber(table, 0);
  std::vector<int64_t> mapping{0}, roots;
  uint32_t previous = UINT32_MAX;
  for (long long i = 0; i < n; ++i) {
    uint32_t &k = renumber[labels[i]];
    if (labels[i] && !k) {
      roots.push_back(i);
      mapping.push_back(0);
      k = uint32_t(roots.size());
    }
    labels[i] = k;
    if (k != previous) {
      if (k) mapping[k] = before[i] ? cc.mapping[before[i]] : 0;
      previous = k;
    }
  }
  cc.count = int64_t(roots.size());
  cc.mapping = std::move(mapping);
  cc.roots = std::move(roots);
  BK_CUDA(cudaMemcpyAsync(ids, labels.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  if (refreshed.data()) BK_CUDA(cudaMemcpyAsync(dbf, refreshed.data(), n * sizeof(float), cudaMemcpyDeviceToDevice, s));
  ctx.synchronize();
  return passes;
}

}  // namespace bk
