// Border targets (fix_borders): every face of every volume goes into one stack of slices; a planar
// CCL and planar EDTs (black border) run over the stack on the GPU, and per face component the
// device gathers the pixel count, the coordinate sums, the largest distance, the first pixel with
// a positive distance and the pixels at the largest distance. The host then picks, per face
// component, the farthest pixel with Kimimaro's tie-break (nearest the component's centroid, then
// the face centre, the corners and the edges) and collects the picks per 3D component in the
// insertion order of a CPython set of integer 3-tuples, which decides the reference's root and
// target order (borders.cu:53-116 and point_set.hpp of giorgioangel/brook).
#include <algorithm>
#include <chrono>
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

std::vector<Face> face_list(const std::vector<BorderVolume> &volumes, int &W, int &H) {
  // faces grouped by axis pair t: (a, b) = (x, y), (x, z), (y, z); within a group volume-major,
  // the low face (c = 0) before the high one
  const int axes[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
  std::vector<Face> faces;
  W = 1;
  H = 1;
  for (int t = 0; t < 3; ++t)
    for (const auto &v : volumes)
      for (int side = 0; side < 2; ++side) {
        const int a = axes[t][0], b = axes[t][1], c = axes[t][2];
        const int shape[3] = {v.d.sx, v.d.sy, v.d.sz};
        Face f{v.offset, v.d, a, b, c, side ? shape[c] - 1 : 0};
        W = std::max(W, f.fy());
        H = std::max(H, f.fx());
        faces.push_back(f);
      }
  return faces;
}

std::vector<std::vector<std::vector<Point>>> border_targets(Context &ctx, const uint32_t *ids,
                                                            const std::vector<BorderVolume> &volumes,
                                                            const float aniso[3], const uint32_t *given_stack) {
  const int axes[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
  int W = 1, H = 1;
  const std::vector<Face> faces = face_list(volumes, W, H);
  std::vector<std::vector<std::vector<Point>>> out(volumes.size());
  for (size_t v = 0; v < volumes.size(); ++v) out[v].resize(size_t(volumes[v].count) + 1);
  if (volumes.empty()) return out;
  if (faces.size() > 65535) throw std::invalid_argument("too many volumes for one border pass");
  const long long slice = (long long)W * H, S = (long long)faces.size();
  if (slice * S >= (1LL << 31) - 1) throw std::invalid_argument("border faces exceed 2^31 pixels");
  // host time of the steps (the device waits on the host in this stage)
  auto t0 = std::chrono::steady_clock::now();
  auto lap = [&](const char *step) {
    const auto now = std::chrono::steady_clock::now();
    ctx.stats[std::string("host_ms_borders_") + step] += std::chrono::duration<double, std::milli>(now - t0).count();
    t0 = now;
  };
  Buffer<uint32_t> stack(ctx, slice * S), stack_ids(ctx, slice * S);
  if (given_stack)
    BK_CUDA(cudaMemcpyAsync(stack.data(), given_stack, size_t(slice * S) * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                            ctx.stream()));
  else
    extract_faces(ctx, ids, faces, W, H, stack.data());
  const VolumeDims sd{W, H, int(S)};
  ComponentsResult pc = connected_components(ctx, stack.data(), U32, sd, stack_ids.data(), true);
  lap("components");
  if (pc.count == 0) return out;
  // 2D EDT (black border) of each group with its own spacing: the slice's x axis is b, y is a
  Buffer<float> dist(ctx, slice * S);
  const long long per_group = 2LL * (long long)volumes.size();
  {
    float wx[3], wy[3];
    for (int t = 0; t < 3; ++t) { wx[t] = aniso[axes[t][1]]; wy[t] = aniso[axes[t][0]]; }
    edt_planes(ctx, stack_ids.data(), W, H, 3, int(per_group), wx, wy, dist.data());
  }
  // per component: counts, coordinate sums, largest distance, first pixel, and the pixels at the
  // largest distance, from the device; the host does the per-component selection
  const FaceStats st = face_stats(ctx, stack_ids.data(), dist.data(), faces, W, H, pc.count);
  lap("stats");
  const size_t K = size_t(pc.count) + 1;
  // a component's face: the stack slice of its first pixel
  std::vector<int> face_of(K, -1);
  for (size_t l = 1; l < K; ++l) face_of[l] = int(pc.roots[l - 1] / slice);
  // Kimimaro's centroid sums are sequential float32 sums over the face in (pa outer, pb inner)
  // order: exact integers while the total stays within 2^24; larger ones are redone that way
  const double exact = 16777216.0;
  std::vector<float> sum_a(K, 0.0f), sum_b(K, 0.0f);
  std::vector<char> redo_face(faces.size(), 0);
  for (size_t l = 1; l < K; ++l) {
    sum_a[l] = float(st.sum_a[l]);
    sum_b[l] = float(st.sum_b[l]);
    if (double(st.sum_a[l]) > exact || double(st.sum_b[l]) > exact) redo_face[face_of[l]] = 1;
  }
  for (size_t fi = 0; fi < faces.size(); ++fi) {
    if (!redo_face[fi]) continue;
    const Face &f = faces[fi];
    const std::vector<uint32_t> lab = stack_ids.download(size_t(slice), size_t(slice) * fi);
    std::vector<float> sa(K, 0.0f), sb(K, 0.0f);
    for (int pa = 0; pa < f.fx(); ++pa)
      for (int pb = 0; pb < f.fy(); ++pb) {
        const uint32_t l = lab[size_t(pb) + size_t(W) * pa];
        if (!l) continue;
        sa[l] += float(pa);
        sb[l] += float(pb);
      }
    for (size_t l = 1; l < K; ++l)
      if (face_of[l] == int(fi)) { sum_a[l] = sa[l]; sum_b[l] = sb[l]; }
  }
  // per component the pick: among its pixels at the largest distance, the least tie keys, the
  // first in (pb outer, pa inner) order among equals
  std::vector<int64_t> pick(K, -1);
  std::vector<std::array<float, 4>> best(K);
  std::vector<float> cx(K, 0.0f), cy(K, 0.0f);
  for (size_t l = 1; l < K; ++l) {
    if (!st.count[l]) continue;
    const Face &f = faces[face_of[l]];
    const float wx = aniso[f.a], wy = aniso[f.b];
    float px = (wx * sum_a[l]) / float(st.count[l]), py = (wy * sum_b[l]) / float(st.count[l]);
    if (px - (wx * float(f.fx())) / 2.0f < 0) px = px + wx;
    if (py - (wy * float(f.fy())) / 2.0f < 0) py = py + wy;
    cx[l] = float(int(px / wx));
    cy[l] = float(int(py / wy));
  }
  const size_t ncand = st.candidates.size() / 3;
  std::vector<size_t> cands(ncand);
  for (size_t j = 0; j < ncand; ++j) cands[j] = j;
  auto flat = [&](size_t j) {
    const int l = st.candidates[3 * j];
    return int64_t(st.candidates[3 * j + 1]) + int64_t(faces[face_of[l]].fx()) * st.candidates[3 * j + 2];
  };
  std::sort(cands.begin(), cands.end(), [&](size_t u, size_t w) {
    const int lu = st.candidates[3 * u], lw = st.candidates[3 * w];
    return lu != lw ? lu < lw : flat(u) < flat(w);
  });
  for (size_t j : cands) {
    const int l = st.candidates[3 * j];
    const Face &f = faces[face_of[l]];
    const auto key = tie_keys(st.candidates[3 * j + 1], st.candidates[3 * j + 2], cx[l], cy[l], f.fx(), f.fy(),
                              aniso[f.a], aniso[f.b]);
    if (pick[l] < 0 || key < best[l]) { best[l] = key; pick[l] = flat(j); }
  }
  // per volume and component id, the picks in the reference's face order (each volume's faces
  // come in that order in the stack), within a face by first pixel with a positive distance
  std::vector<std::vector<size_t>> by_face(faces.size());
  for (size_t l = 1; l < K; ++l)
    if (pick[l] >= 0) by_face[face_of[l]].push_back(l);
  std::vector<std::vector<TupleSet>> sets(volumes.size());
  for (size_t v = 0; v < volumes.size(); ++v) sets[v].resize(size_t(volumes[v].count) + 1);
  for (size_t fi = 0; fi < faces.size(); ++fi) {
    auto &order = by_face[fi];
    if (order.empty()) continue;
    const Face &f = faces[fi];
    const size_t v = size_t(fi % per_group) / 2;
    std::sort(order.begin(), order.end(), [&](size_t u, size_t w) { return st.first[u] < st.first[w]; });
    for (size_t l : order) {
      Point p{};
      p[f.a] = pick[l] % f.fx();
      p[f.b] = pick[l] / f.fx();
      p[f.c] = f.fixed;
      sets[v].at(size_t(pc.mapping[l])).add(p);
    }
  }
  for (size_t v = 0; v < volumes.size(); ++v)
    for (size_t id = 0; id < sets[v].size(); ++id) out[v][id] = sets[v][id].values();
  lap("select");
  return out;
}

}  // namespace bk
