// Border targets (fix_borders): for each of the six faces, a 2D CC and a 2D EDT (black border) of
// the face's component ids run on the GPU; the host then picks, per face component, the farthest
// pixel with Kimimaro's tie-break (nearest the component's centroid, then the face centre, the
// corners and the edges) and collects the picks per 3D component in the insertion order of a
// CPython set of integer 3-tuples, which decides the reference's root and target order
// (borders.cu:53-116 and point_set.hpp of giorgioangel/brook).
#include <algorithm>
#include <limits>

#include "kernels.hpp"

namespace bk {
namespace {

// CPython 3.12's set of integer 3-tuples: xxHash-based tuple hash over int hashes (value modulo
// 2^61 - 1, sign kept, -1 -> -2); open addressing with 9 linear probes and perturbed jumps;
// growth to the next power of two above 4x the entries (2x beyond 50000) when fill * 5 >= mask * 3.
class TupleSet {
  struct Slot {
    Point p{};
    uint64_t h = 0;
    bool live = false;
  };
  std::vector<Slot> table_ = std::vector<Slot>(8);
  size_t used_ = 0;

  static uint64_t hash_int(int64_t v) {
    const uint64_t modulus = (uint64_t{1} << 61) - 1;
    const uint64_t magnitude = v < 0 ? uint64_t(-(v + 1)) + 1 : uint64_t(v);
    int64_t h = int64_t(magnitude % modulus);
    if (v < 0) h = -h;
    if (h == -1) h = -2;
    return uint64_t(h);
  }
  static uint64_t hash(const Point &p) {
    const uint64_t prime1 = 11400714785074694791ull, prime2 = 14029467366897019727ull, prime5 = 2870177450012600261ull;
    uint64_t acc = prime5;
    for (int64_t v : p) {
      acc += hash_int(v) * prime2;
      acc = (acc << 31) | (acc >> 33);
      acc *= prime1;
    }
    acc += uint64_t{3} ^ (prime5 ^ 3527539ull);
    return acc == ~uint64_t{0} ? 1546275796ull : acc;
  }
  bool place(const Point &p, uint64_t h, bool compare) {
    const size_t mask = table_.size() - 1;
    size_t i = h & mask;
    uint64_t perturb = h;
    for (;;) {
      const size_t probes = i + 9 <= mask ? 9 : 0;
      for (size_t j = 0; j <= probes; ++j) {
        Slot &slot = table_[i + j];
        if (!slot.live) { slot.p = p; slot.h = h; slot.live = true; return true; }
        if (compare && slot.h == h && slot.p == p) return false;
      }
      perturb >>= 5;
      i = (i * 5 + 1 + perturb) & mask;
    }
  }

 public:
  void add(const Point &p) {
    if (!place(p, hash(p), true)) return;
    ++used_;
    if (used_ * 5 < (table_.size() - 1) * 3) return;
    const size_t target = used_ * (used_ > 50000 ? 2 : 4);
    size_t size = 8;
    while (size <= target) size *= 2;
    std::vector<Slot> old = std::move(table_);
    table_.assign(size, Slot{});
    for (const Slot &slot : old)
      if (slot.live) place(slot.p, slot.h, false);
  }
  std::vector<Point> values() const {
    std::vector<Point> out;
    out.reserve(used_);
    for (const Slot &slot : table_)
      if (slot.live) out.push_back(slot.p);
    return out;
  }
};

float sqdist(float x, float y, float a, float b, float wx, float wy) {
  const float dx = wx * (x - a), dy = wy * (y - b);
  return dx * dx + dy * dy;
}

std::array<float, 4> tie_keys(int64_t ix, int64_t iy, float cx, float cy, int64_t nx, int64_t ny, float wx, float wy) {
  const float x = float(ix), y = float(iy), fx = float(nx), fy = float(ny);
  const float centre_x = float(double(wx * fx) / 2.0), centre_y = float(double(wy * fy) / 2.0);
  const float far_x = float(double(fx) - 0.5), far_y = float(double(fy) - 0.5);
  const float corner = std::min({sqdist(x, y, -0.5f, -0.5f, wx, wy), sqdist(x, y, far_x, -0.5f, wx, wy),
                                 sqdist(x, y, far_x, far_y, wx, wy), sqdist(x, y, -0.5f, far_x, wx, wy)});
  const float edge = float(std::min({double(wx) * (double(x) - 0.5), double(wx) * (double(fx) - 0.5 - double(x)),
                                     double(wy) * (double(y) - 0.5), double(wy) * (double(fy) - 0.5 - double(y))}));
  return {sqdist(x, y, cx, cy, wx, wy), sqdist(x, y, centre_x, centre_y, wx, wy), corner, edge};
}

}  // namespace

std::vector<std::vector<Point>> border_targets(Context &ctx, const uint32_t *ids, VolumeDims d, int64_t count,
                                               const float aniso[3]) {
  std::vector<TupleSet> sets(count + 1);
  const int shape[3] = {d.sx, d.sy, d.sz};
  const int axes[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
  for (int face = 0; face < 6; ++face) {
    const int a = axes[face / 2][0], b = axes[face / 2][1], c = axes[face / 2][2];
    const int fixed = face % 2 ? shape[c] - 1 : 0;
    const int64_t fx = shape[a], fy = shape[b];
    const VolumeDims pd{int(fy), int(fx), 1};
    Buffer<uint32_t> plane(ctx, fx * fy);
    extract_face(ctx, ids, d, a, b, c, fixed, plane.data());
    Buffer<uint32_t> plane_ids(ctx, fx * fy);
    ComponentsResult pc = connected_components(ctx, plane.data(), U32, pd, plane_ids.data());
    if (pc.count == 0) continue;
    const float plane_aniso[3] = {aniso[b], aniso[a], 1.0f};
    Buffer<float> dist(ctx, fx * fy);
    edt(ctx, plane_ids.data(), pd, plane_aniso, true, 2, dist.data());
    const std::vector<uint32_t> lab = plane_ids.download();
    const std::vector<float> dd = dist.download();
    const size_t k = size_t(pc.count) + 1;
    std::vector<float> maxdist(k, 0.0f), sumx(k, 0.0f), sumy(k, 0.0f);
    std::vector<uint32_t> sizes(k, 0);
    std::vector<int64_t> first(k, std::numeric_limits<int64_t>::max()), pick(k, -1);
    // Kimimaro's sequential float32 centroid sums, x outer
    for (int64_t x = 0; x < fx; ++x)
      for (int64_t y = 0; y < fy; ++y) {
        const size_t i = size_t(y + fy * x);
        const uint32_t l = lab[i];
        if (!l) continue;
        sumx[l] += float(x);
        sumy[l] += float(y);
        ++sizes[l];
        if (dd[i] > 0) { maxdist[l] = std::max(maxdist[l], dd[i]); first[l] = std::min(first[l], x + fx * y); }
      }
    const float wx = aniso[a], wy = aniso[b];
    std::vector<float> cx(k, 0.0f), cy(k, 0.0f);
    for (size_t l = 1; l < k; ++l)
      if (sizes[l]) {
        float px = (wx * sumx[l]) / float(sizes[l]), py = (wy * sumy[l]) / float(sizes[l]);
        if (px - (wx * float(fx)) / 2.0f < 0) px = px + wx;
        if (py - (wy * float(fy)) / 2.0f < 0) py = py + wy;
        cx[l] = float(int(px / wx));
        cy[l] = float(int(py / wy));
      }
    std::vector<std::array<float, 4>> best(k);
    for (int64_t y = 0; y < fy; ++y)
      for (int64_t x = 0; x < fx; ++x) {
        const size_t i = size_t(y + fy * x);
        const uint32_t l = lab[i];
        if (!l || dd[i] == 0 || dd[i] != maxdist[l]) continue;
        const auto key = tie_keys(x, y, cx[l], cy[l], fx, fy, wx, wy);
        if (pick[l] < 0 || key < best[l]) { best[l] = key; pick[l] = x + fx * y; }
      }
    std::vector<size_t> order;
    for (size_t l = 1; l < k; ++l)
      if (pick[l] >= 0) order.push_back(l);
    std::sort(order.begin(), order.end(), [&](size_t u, size_t v) { return first[u] < first[v]; });
    for (size_t l : order) {
      Point p{};
      p[a] = pick[l] % fx;
      p[b] = pick[l] / fx;
      p[c] = fixed;
      sets.at(size_t(pc.mapping[l])).add(p);
    }
  }
  std::vector<std::vector<Point>> out;
  out.reserve(sets.size());
  for (const auto &s : sets) out.push_back(s.values());
  return out;
}

}  // namespace bk
