// CPU oracle for the TEASAR hot path of giorgioangel/brook (v0.1.0).
//
// TEST INFRASTRUCTURE ONLY. This file is a plain C++ restatement of the reference algorithm, used
// by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the checker. The product
// (brook_b200) never links, loads or calls it.
//
// Everything works on one label volume in Fortran order (x fastest), flat index
// i = x + sx * (y + sy * z). Each function cites the reference file:line whose behaviour it
// restates; the tie and rounding rules are the reference's, because its output is the parity target:
//   * connected components: ids 1..K by ascending first flat index (ccl.cu:25-63, ccl_kernels.cuh:108-133)
//   * EDT: float32 spacing accumulation along x, float64 lower envelope along y and z, float32
//     storage, sqrt at the end (edt_kernels.cuh:15-144, edt.cu:12-15)
//   * border targets (fix_borders): per face a 2D CC + 2D EDT, farthest pixel with the
//     centroid/centre/corner/edge tie-break, ordered by first pixel, collected in a CPython set
//     (borders.cu:53-116, point_set.hpp)
//   * argmax ties -> lowest flat (batched_regular.inc:9-22)
//   * DAF: 26-connected geometric distance with float32 weights (batched.cu:211-215)
//   * PDRF: (1 - dbf * M)^(2^s) * scale + daf * inv, no FMA (batched_regular.inc:93-108)
//   * target order: descending DAF (inf -> 0), ties -> higher flat first (lockstep_order.cu:21-45)
//   * railroad: vertex-weighted SSSP with the one-ulp step, nearest rail by (dist, flat), warp
//     backtrace rule (lowest neighbour index on ties) and the dijkstra3d join
//     (common.cuh:113-127, lockstep_coop.inc:71-305, lockstep_regular.inc:61-155)
//   * invalidation: claim-order flood in bands of the bottleneck distance, round-synchronous
//     inside a band, pulls at band boundaries (invalidation_kernels.cuh:11-297)
//   * assembly: unique vertices sorted by (x,y,z), edges (min,max) sorted unique, unused vertices
//     dropped, radius = DBF (skeleton.cpp:13-40, assembly.cu:88-160)
// Soma handling (dbf_max > soma_detection_threshold) is not restated: the oracle reports an
// error for such objects.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <memory>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <mutex>
#include <numeric>
#include <queue>
#include <stdexcept>
#include <string>
#include <thread>
#include <map>
#include <vector>

namespace {

using i64 = int64_t;
constexpr float kInf = std::numeric_limits<float>::infinity();

// ---------------------------------------------------------------------------------------------
// Neighbourhood tables. The reference fixes one 26-neighbour order for every kernel
// (common.cuh:33-47): the six faces (-x,+x,-y,+y,-z,+z), then the xy, yz and xz edges, each pair
// of signs in lexicographic order, then the eight corners lexicographic with z fastest. The
// dijkstra3d order (common.cuh:63-76) differs only in the corners. Both are built here from
// those rules.
struct Tables {
  int dx[26], dy[26], dz[26], opp[26], d3rank[26], d3inv[26];
  int bit[26];  // the voxel-graph bit (cc3d's order) that permits step k (common.cuh:48-55)
  Tables() {
    int k = 0;
    auto put = [&](int x, int y, int z) { dx[k] = x; dy[k] = y; dz[k] = z; ++k; };
    put(-1, 0, 0); put(1, 0, 0); put(0, -1, 0); put(0, 1, 0); put(0, 0, -1); put(0, 0, 1);
    for (int a : {-1, 1}) for (int b : {-1, 1}) put(a, b, 0);
    for (int a : {-1, 1}) for (int b : {-1, 1}) put(0, a, b);
    for (int a : {-1, 1}) for (int b : {-1, 1}) put(a, 0, b);
    for (int a : {-1, 1}) for (int b : {-1, 1}) for (int c : {-1, 1}) put(a, b, c);
    for (int i = 0; i < 26; ++i)
      for (int j = 0; j < 26; ++j)
        if (dx[j] == -dx[i] && dy[j] == -dy[i] && dz[j] == -dz[i]) opp[i] = j;
    // dijkstra3d corner order: (-,-,-)(+,-,-)(-,+,-)(-,-,+)(+,+,-)(+,-,+)(-,+,+)(+,+,+)
    const int corners[8][3] = {{-1,-1,-1},{1,-1,-1},{-1,1,-1},{-1,-1,1},{1,1,-1},{1,-1,1},{-1,1,1},{1,1,1}};
    for (int i = 0; i < 18; ++i) { d3rank[i] = i; d3inv[i] = i; }
    for (int r = 0; r < 8; ++r)
      for (int j = 18; j < 26; ++j)
        if (dx[j] == corners[r][0] && dy[j] == corners[r][1] && dz[j] == corners[r][2]) { d3inv[18 + r] = j; d3rank[j] = 18 + r; }
    // cc3d's bit order: faces +x -x +y -y +z -z, the xy edges, the xz and yz edges with +z, then
    // with -z, the corners with +z, then with -z, x fastest and + before - within each group
    const int cc3d[26][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1},
                             {1,1,0},{-1,1,0},{1,-1,0},{-1,-1,0},{1,0,1},{-1,0,1},{0,1,1},{0,-1,1},
                             {1,0,-1},{-1,0,-1},{0,1,-1},{0,-1,-1},
                             {1,1,1},{-1,1,1},{1,-1,1},{-1,-1,1},{1,1,-1},{-1,1,-1},{1,-1,-1},{-1,-1,-1}};
    for (int i = 0; i < 26; ++i)
      for (int b = 0; b < 26; ++b)
        if (dx[i] == cc3d[b][0] && dy[i] == cc3d[b][1] && dz[i] == cc3d[b][2]) bit[i] = b;
  }
};
const Tables T;

struct Shape {
  i64 sx, sy, sz;
  i64 n() const { return sx * sy * sz; }
  i64 idx(i64 x, i64 y, i64 z) const { return x + sx * (y + sy * z); }
  void xyz(i64 i, i64 &x, i64 &y, i64 &z) const { z = i / (sx * sy); i -= z * sx * sy; y = i / sx; x = i - y * sx; }
  bool inside(i64 x, i64 y, i64 z) const { return x >= 0 && y >= 0 && z >= 0 && x < sx && y < sy && z < sz; }
};

inline uint32_t fbits(float f) { uint32_t b; std::memcpy(&b, &f, 4); return b; }
inline float bitsf(uint32_t b) { float f; std::memcpy(&f, &b, 4); return f; }

// fn(begin, end) over [0, n) in chunks of `grain`, on `threads` threads (the caller's among
// them). Every use below splits work whose items write disjoint data, so the result does not
// depend on the thread count.
template <class F>
void parallel_for(i64 n, int threads, i64 grain, F &&fn) {
  if (n <= 0) return;
  const int workers = int(std::max<i64>(1, std::min<i64>(threads, (n + grain - 1) / grain)));
  if (workers == 1) { fn(i64(0), n); return; }
  std::atomic<i64> next{0};
  auto work = [&] {
    for (;;) {
      const i64 b = next.fetch_add(grain);
      if (b >= n) return;
      fn(b, std::min(n, b + grain));
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < workers; ++t) pool.emplace_back(work);
  work();
  for (auto &t : pool) t.join();
}

// ---------------------------------------------------------------------------------------------
// Connected components (ccl.cu:25-63): 26-connected components of equal nonzero labels. The
// union-find root of a component is its lowest flat index; ids 1..K follow ascending roots.
struct Components {
  std::vector<uint32_t> ids;    // per voxel, 0 = background
  std::vector<int64_t> mapping; // id -> original label (index 0 unused)
  std::vector<int64_t> roots;   // id-1 -> first flat index
};

// Linking the larger root under the smaller one keeps every tree's root at its least flat index,
// whatever order the unions come in: z-slabs are joined in parallel (every union inside a slab
// touches only that slab's entries), then the pairs across slab boundaries one by one.
template <class L>
Components connected_components(const L *labels, const Shape &s, int threads = 1) {
  const i64 n = s.n();
  std::vector<i64> parent(n);
  std::iota(parent.begin(), parent.end(), i64(0));
  auto find = [&](i64 v) {
    i64 r = v;
    while (parent[r] != r) r = parent[r];
    while (parent[v] != r) { i64 next = parent[v]; parent[v] = r; v = next; }
    return r;
  };
  auto unite_from = [&](i64 v, i64 zlo, i64 zhi) {  // v's forward neighbours with z in [zlo, zhi)
    if (labels[v] == 0) return;
    i64 x, y, z; s.xyz(v, x, y, z);
    for (int k = 0; k < 26; ++k) {
      i64 nx = x + T.dx[k], ny = y + T.dy[k], nz = z + T.dz[k];
      if (!s.inside(nx, ny, nz) || nz < zlo || nz >= zhi) continue;
      i64 u = s.idx(nx, ny, nz);
      if (u <= v || labels[u] != labels[v]) continue;
      i64 a = find(v), b = find(u);
      if (a != b) { if (a < b) parent[b] = a; else parent[a] = b; }
    }
  };
  const i64 plane = s.sx * s.sy, depth = std::max<i64>(1, (s.sz + threads - 1) / std::max(threads, 1));
  const i64 slabs = (s.sz + depth - 1) / depth;
  parallel_for(slabs, threads, 1, [&](i64 b, i64 e) {
    for (i64 k = b; k < e; ++k) {
      const i64 z0 = k * depth, z1 = std::min(s.sz, z0 + depth);
      for (i64 v = z0 * plane; v < z1 * plane; ++v) unite_from(v, z0, z1);
    }
  });
  for (i64 k = 1; k < slabs; ++k)  // plane z0 - 1 with plane z0
    for (i64 v = (k * depth - 1) * plane; v < k * depth * plane; ++v) unite_from(v, k * depth, k * depth + 1);
  Components c;
  c.ids.assign(n, 0);
  c.mapping.push_back(0);
  std::vector<uint32_t> id_of(n, 0);
  for (i64 v = 0; v < n; ++v) {
    if (labels[v] == 0) continue;
    i64 r = find(v);
    if (r == v) {  // roots appear in ascending flat order
      c.roots.push_back(v);
      c.mapping.push_back(static_cast<int64_t>(labels[v]));
      id_of[v] = static_cast<uint32_t>(c.roots.size());
    }
    c.ids[v] = id_of[r];
  }
  return c;
}

Components components_any(const void *labels, int dtype, const Shape &s, int threads) {
  switch (dtype) {
    case 0: return connected_components(static_cast<const uint8_t *>(labels), s, threads);
    case 1: return connected_components(static_cast<const uint16_t *>(labels), s, threads);
    case 2: return connected_components(static_cast<const uint32_t *>(labels), s, threads);
    case 3: return connected_components(static_cast<const uint64_t *>(labels), s, threads);
    case 4: return connected_components(static_cast<const int8_t *>(labels), s, threads);
    case 5: return connected_components(static_cast<const int16_t *>(labels), s, threads);
    case 6: return connected_components(static_cast<const int32_t *>(labels), s, threads);
    case 7: return connected_components(static_cast<const int64_t *>(labels), s, threads);
    default: throw std::invalid_argument("integer labels required");
  }
}

// ---------------------------------------------------------------------------------------------
// Multi-label anisotropic EDT (edt_kernels.cuh:15-144, edt.cu:12-15). Distance of each voxel to
// the nearest voxel of a different label; with black_border the volume edge counts as such a
// voxel. `dims` = 2 skips the z pass (the 2D face transforms of the border targets).
void edt_pass_x(const uint32_t *lab, float *D, const Shape &s, float w, bool bb, int threads) {
  std::vector<float> acc(s.sx + 2, 0.0f);
  for (size_t k = 1; k < acc.size(); ++k) acc[k] = acc[k - 1] + w;  // one float32 rounding per step
  parallel_for(s.sy * s.sz, threads, 256, [&](i64 lb, i64 le) {
  for (i64 line = lb; line < le; ++line) {
    const i64 base = s.sx * line;
    i64 i = 0;
    while (i < s.sx) {
      const uint32_t L = lab[base + i];
      i64 c = i, d = i;
      while (d + 1 < s.sx && lab[base + d + 1] == L) ++d;
      const bool leftw = c > 0 || bb, rightw = d < s.sx - 1 || bb;
      for (i64 p = c; p <= d; ++p) {
        float best = kInf;
        if (leftw) { float dd = acc[p - (c - 1)]; float v = dd * dd; if (v < best) best = v; }
        if (rightw) { float dd = acc[(d + 1) - p]; float v = dd * dd; if (v < best) best = v; }
        D[base + p] = best;
      }
      i = d + 1;
    }
  }
  });
}

// One line of the y / z pass: lower envelope of the parabolas of a run's finite heights and its
// walls (height 0), evaluated in double. The reference compiles this pass with FMA contraction;
// the two sums of a product and a height are written as explicit fused operations here (exact
// for integer spacings, where every product is an integer below 2^53).
void edt_line_fh(const uint32_t *lab, float *D, i64 base, i64 stride, i64 n, float w, bool bb,
                 std::vector<i64> &V, std::vector<float> &H, std::vector<double> &Z) {
  const double w2 = static_cast<double>(w * w);
  i64 i = 0;
  while (i < n) {
    const uint32_t L = lab[base + i * stride];
    i64 c = i, d = i;
    while (d + 1 < n && lab[base + (d + 1) * stride] == L) ++d;
    const bool leftw = c > 0 || bb, rightw = d < n - 1 || bb;
    int k = -1;
    auto place = [&](i64 pp, double ph) {
      bool placed = false;
      while (k >= 0 && !placed) {
        const double num = std::fma(w2 * static_cast<double>(pp), static_cast<double>(pp), ph) -
                           std::fma(w2 * static_cast<double>(V[k]), static_cast<double>(V[k]), static_cast<double>(H[k]));
        const double s = num / (2.0 * w2 * (static_cast<double>(pp) - static_cast<double>(V[k])));
        if (s <= Z[k]) --k;
        else { ++k; V[k] = pp; H[k] = static_cast<float>(ph); Z[k] = s; placed = true; }
      }
      if (!placed) { k = 0; V[0] = pp; H[0] = static_cast<float>(ph); Z[0] = -1e300; }
    };
    if (leftw) { k = 0; V[0] = c - 1; H[0] = 0.0f; Z[0] = -1e300; }
    for (i64 p = c; p <= d; ++p) {
      const float hf = D[base + p * stride];
      if (!(hf < kInf)) continue;
      place(p, static_cast<double>(hf));
    }
    if (rightw) place(d + 1, 0.0);
    if (k < 0) {
      for (i64 q = c; q <= d; ++q) D[base + q * stride] = kInf;
    } else {
      int kk = 0;
      for (i64 q = c; q <= d; ++q) {
        while (kk < k && Z[kk + 1] < static_cast<double>(q)) ++kk;
        const double dq = static_cast<double>(q) - static_cast<double>(V[kk]);
        D[base + q * stride] = static_cast<float>(std::fma(w2 * dq, dq, static_cast<double>(H[kk])));
      }
    }
    i = d + 1;
  }
}

std::vector<float> edt(const uint32_t *lab, const Shape &s, const float aniso[3], bool bb, int dims = 3,
                       int threads = 1) {
  std::vector<float> D(s.n());
  edt_pass_x(lab, D.data(), s, aniso[0], bb, threads);
  const i64 longest = std::max(s.sy, s.sz) + 3;
  // every line of a pass is independent: planes (y pass) and rows (z pass) go to the threads
  auto lines = [&](i64 outer, auto &&line) {
    parallel_for(outer, threads, 1, [&](i64 b, i64 e) {
      std::vector<i64> V(longest); std::vector<float> H(longest); std::vector<double> Z(longest);
      for (i64 o = b; o < e; ++o)
        for (i64 x = 0; x < s.sx; ++x) line(o, x, V, H, Z);
    });
  };
  if (dims >= 2)
    lines(s.sz, [&](i64 z, i64 x, auto &V, auto &H, auto &Z) {
      edt_line_fh(lab, D.data(), x + s.sx * s.sy * z, s.sx, s.sy, aniso[1], bb, V, H, Z);
    });
  if (dims >= 3)
    lines(s.sy, [&](i64 y, i64 x, auto &V, auto &H, auto &Z) {
      edt_line_fh(lab, D.data(), x + s.sx * y, s.sx * s.sy, s.sz, aniso[2], bb, V, H, Z);
    });
  parallel_for(s.n(), threads, 1 << 16, [&](i64 b, i64 e) {
    for (i64 i = b; i < e; ++i) D[i] = lab[i] == 0 ? 0.0f : std::sqrt(D[i]);
  });
  return D;
}

// ---------------------------------------------------------------------------------------------
// Border targets: CPython 3.12's insertion-ordered hash set of integer 3-tuples (the collection
// Kimimaro gathers border points in; point_set.hpp restates it for the reference). Tuple hash:
// CPython's xxHash-based tuplehash; int hash: value mod (2^61 - 1) with the sign kept, -1 -> -2;
// set probing: 9 linear probes then perturbed jumps; resize when fill * 5 >= mask * 3.
class TupleSet {
  struct Slot { std::array<i64, 3> p{}; uint64_t h = 0; bool live = false; };
  std::vector<Slot> table_ = std::vector<Slot>(8);
  size_t used_ = 0;
  static uint64_t hash_int(i64 v) {
    const uint64_t modulus = (uint64_t{1} << 61) - 1;
    uint64_t mag = v < 0 ? uint64_t(-(v + 1)) + 1 : uint64_t(v);
    i64 h = static_cast<i64>(mag % modulus);
    if (v < 0) h = -h;
    if (h == -1) h = -2;
    return static_cast<uint64_t>(h);
  }
  static uint64_t hash(const std::array<i64, 3> &p) {
    const uint64_t prime1 = 11400714785074694791ull, prime2 = 14029467366897019727ull, prime5 = 2870177450012600261ull;
    uint64_t acc = prime5;
    for (i64 v : p) { acc += hash_int(v) * prime2; acc = (acc << 31) | (acc >> 33); acc *= prime1; }
    acc += uint64_t{3} ^ (prime5 ^ 3527539ull);
    return acc == ~uint64_t{0} ? 1546275796ull : acc;
  }
  bool place(const std::array<i64, 3> &p, uint64_t h, bool compare) {
    const size_t mask = table_.size() - 1;
    size_t i = h & mask; uint64_t perturb = h;
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
  void add(const std::array<i64, 3> &p) {
    if (!place(p, hash(p), true)) return;
    ++used_;
    if (used_ * 5 < (table_.size() - 1) * 3) return;
    const size_t target = used_ * (used_ > 50000 ? 2 : 4);
    size_t size = 8;
    while (size <= target) size *= 2;
    std::vector<Slot> old = std::move(table_);
    table_.assign(size, Slot{});
    for (const Slot &slot : old) if (slot.live) place(slot.p, slot.h, false);
  }
  std::vector<std::array<i64, 3>> values() const {
    std::vector<std::array<i64, 3>> out;
    for (const Slot &slot : table_) if (slot.live) out.push_back(slot.p);
    return out;
  }
};

// Kimimaro's tie-break keys among a face component's farthest pixels (borders.cu:38-52).
float sqdist2(float x, float y, float a, float b, float wx, float wy) {
  const float dx = wx * (x - a), dy = wy * (y - b);
  return dx * dx + dy * dy;
}
std::array<float, 4> border_keys(i64 ix, i64 iy, float cx, float cy, i64 nx, i64 ny, float wx, float wy) {
  const float x = float(ix), y = float(iy), fx = float(nx), fy = float(ny);
  const float centre_x = float(double(wx * fx) / 2.0), centre_y = float(double(wy * fy) / 2.0);
  const float far_x = float(double(fx) - 0.5), far_y = float(double(fy) - 0.5);
  const float corner = std::min({sqdist2(x, y, -0.5f, -0.5f, wx, wy), sqdist2(x, y, far_x, -0.5f, wx, wy),
                                 sqdist2(x, y, far_x, far_y, wx, wy), sqdist2(x, y, -0.5f, far_x, wx, wy)});
  const float edge = float(std::min({double(wx) * (double(x) - 0.5), double(wx) * (double(fx) - 0.5 - double(x)),
                                     double(wy) * (double(y) - 0.5), double(wy) * (double(fy) - 0.5 - double(y))}));
  return {sqdist2(x, y, cx, cy, wx, wy), sqdist2(x, y, centre_x, centre_y, wx, wy), corner, edge};
}

// Per face: a 2D CC of the face's component ids, a 2D EDT with black border, and per face
// component the farthest pixel (borders.cu:53-116). Returns, per component id, its border points.
std::vector<std::vector<std::array<i64, 3>>> border_targets(const std::vector<uint32_t> &cc, const Shape &s, size_t count,
                                                            const float aniso[3]) {
  std::vector<TupleSet> sets(count + 1);
  const i64 shape[3] = {s.sx, s.sy, s.sz};
  const int axes[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
  for (int face = 0; face < 6; ++face) {
    const int a = axes[face / 2][0], b = axes[face / 2][1], c = axes[face / 2][2];
    const i64 fixed = face % 2 ? shape[c] - 1 : 0, fx = shape[a], fy = shape[b];
    // the face as a (fy, fx) plane: plane x = the b coordinate, plane y = the a coordinate
    const Shape ps{fy, fx, 1};
    std::vector<uint32_t> plane(fx * fy);
    for (i64 pa = 0; pa < fx; ++pa)
      for (i64 pb = 0; pb < fy; ++pb) {
        i64 p[3]; p[a] = pa; p[b] = pb; p[c] = fixed;
        plane[pb + fy * pa] = cc[s.idx(p[0], p[1], p[2])];
      }
    Components pc = connected_components(plane.data(), ps);
    const float plane_aniso[3] = {aniso[b], aniso[a], 1.0f};
    std::vector<float> d = edt(pc.ids.data(), ps, plane_aniso, true, 2);
    const size_t k = pc.mapping.size();
    std::vector<float> maxdist(k, 0.0f), sumx(k, 0.0f), sumy(k, 0.0f);
    std::vector<uint32_t> sizes(k, 0);
    std::vector<i64> first(k, std::numeric_limits<i64>::max()), pick(k, -1);
    for (i64 x = 0; x < fx; ++x)
      for (i64 y = 0; y < fy; ++y) {
        const size_t i = y + fy * x; const uint32_t label = pc.ids[i];
        if (!label) continue;
        sumx[label] += float(x); sumy[label] += float(y); ++sizes[label];
        if (d[i] > 0) { maxdist[label] = std::max(maxdist[label], d[i]); first[label] = std::min(first[label], x + fx * y); }
      }
    const float wx = aniso[a], wy = aniso[b];
    std::vector<float> cx(k, 0.0f), cy(k, 0.0f);
    for (size_t label = 1; label < k; ++label)
      if (sizes[label]) {
        float px = (wx * sumx[label]) / float(sizes[label]), py = (wy * sumy[label]) / float(sizes[label]);
        if (px - (wx * float(fx)) / 2.0f < 0) px = px + wx;
        if (py - (wy * float(fy)) / 2.0f < 0) py = py + wy;
        cx[label] = float(int(px / wx)); cy[label] = float(int(py / wy));
      }
    std::vector<std::array<float, 4>> best(k);
    for (i64 y = 0; y < fy; ++y)
      for (i64 x = 0; x < fx; ++x) {
        const size_t i = y + fy * x; const uint32_t label = pc.ids[i];
        if (!label || d[i] == 0 || d[i] != maxdist[label]) continue;
        const auto key = border_keys(x, y, cx[label], cy[label], fx, fy, wx, wy);
        if (pick[label] < 0 || key < best[label]) { best[label] = key; pick[label] = x + fx * y; }
      }
    std::vector<size_t> order;
    for (size_t label = 1; label < k; ++label) if (pick[label] >= 0) order.push_back(label);
    std::sort(order.begin(), order.end(), [&](size_t u, size_t v) { return first[u] < first[v]; });
    for (size_t label : order) {
      std::array<i64, 3> p{};
      p[a] = pick[label] % fx; p[b] = pick[label] / fx; p[c] = fixed;
      sets.at(pc.mapping[label]).add(p);
    }
  }
  std::vector<std::vector<std::array<i64, 3>>> out;
  for (const auto &set : sets) out.push_back(set.values());
  return out;
}

// ---------------------------------------------------------------------------------------------
// 26-connected geometric distance within one component (the DAF flood, batched.cu:211-232;
// weights: faces = spacing, edges = |pair|, corners = |spacing|, each rounded to float32 from
// double). Dijkstra over float32 sums: fl(d + w) is monotone in d, so the fixed point the
// reference's Bellman-Ford reaches is the one this search settles.
struct Weights { float w[26]; };
Weights geometric_weights(const float aniso[3]) {
  const double x = aniso[0], y = aniso[1], z = aniso[2];
  Weights W;
  const float faces[3] = {float(x), float(y), float(z)};
  for (int k = 0; k < 6; ++k) W.w[k] = faces[k / 2];
  const double pairs[3] = {std::sqrt(x * x + y * y), std::sqrt(y * y + z * z), std::sqrt(x * x + z * z)};
  for (int k = 6; k < 18; ++k) W.w[k] = float(pairs[(k - 6) / 4]);
  for (int k = 18; k < 26; ++k) W.w[k] = float(std::sqrt(x * x + y * y + z * z));
  return W;
}

void geometric_flood(const std::vector<uint32_t> &ids, const Shape &s, uint32_t label, i64 source, const Weights &W,
                     std::vector<float> &dist, const std::vector<i64> &voxels, const std::vector<float> *seeds = nullptr) {
  using Item = std::pair<float, i64>;
  std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
  for (i64 v : voxels) {
    dist[v] = seeds ? (*seeds)[v] : kInf;
    if (dist[v] < kInf) heap.push({dist[v], v});
  }
  if (dist[source] != 0.0f) { dist[source] = 0.0f; heap.push({0.0f, source}); }
  while (!heap.empty()) {
    auto [d, u] = heap.top(); heap.pop();
    if (d > dist[u]) continue;
    i64 x, y, z; s.xyz(u, x, y, z);
    for (int k = 0; k < 26; ++k) {
      const i64 nx = x + T.dx[k], ny = y + T.dy[k], nz = z + T.dz[k];
      if (!s.inside(nx, ny, nz)) continue;
      const i64 v = s.idx(nx, ny, nz);
      if (ids[v] != label) continue;
      const float cand = d + W.w[k];
      if (cand < dist[v]) { dist[v] = cand; heap.push({cand, v}); }
    }
  }
}

// argmax over a component's voxels: largest finite value, ties -> lowest flat (batched_regular.inc:9-22)
i64 argmax(const std::vector<float> &f, const std::vector<i64> &voxels, float &value) {
  i64 best = -1; value = 0;
  for (i64 v : voxels) {  // voxels ascend, so strict > keeps the lowest flat among ties
    const float x = f[v];
    if (!(x < kInf)) continue;
    if (best < 0 || fbits(x) > fbits(value)) { best = v; value = x; }
  }
  return best;
}

// ---------------------------------------------------------------------------------------------
// One vertex-weighted step (common.cuh:113-127): fl(d + f), advanced by one ulp where f > 0 is
// absorbed, so that distances strictly increase along every step.
inline float vw_step(float d, float f) {
  float c = d + f;
  if (c == d && f > 0.0f && d < kInf) c = bitsf(fbits(d) + 1);
  return c;
}

struct Params {
  double scale, constant, pdrf_scale, pdrf_exponent;
  double soma_detection, soma_acceptance, soma_scale, soma_constant;
  int64_t max_paths; int has_max_paths;
  float anisotropy[3];
  double dust;
  int fix_branching, fix_borders;
  int fill_holes = 0, fix_avocados = 0;
  // extra targets (x, y, z triples): `before` traced first, `after` once no voxel is left
  std::vector<std::array<i64, 3>> before, after;
  // a PDRF field (float32 per voxel, Fortran order) that replaces the computed one: tests use it
  // to trace from another implementation's field where the power itself is not bit-reproducible
  const float *pdrf_field = nullptr;
};

// Per-object tracing state over the shared volume. Every array is indexed by global flat index;
// an object only ever touches its own voxels, so objects can be traced concurrently.
struct Volume {
  Shape s;
  const std::vector<uint32_t> *ids;
  std::vector<float> dbf, pdrf, dist;
  std::vector<uint8_t> alive, inq;
  std::vector<uint64_t> key;
  const uint32_t *graph = nullptr;  // a voxel graph (cc3d bits per voxel), or none
};

// Voxel-graph gates (common.cuh:85-100): the step from u along k is permitted by graph[u]'s bit
// for k (push); the step into v from its neighbour u = v + N[k] is the step u -> v, permitted by
// graph[u]'s bit for the opposite offset (pull). Without a graph every step is permitted.
bool push_ok(const Volume &V, i64 u, int k) { return !V.graph || ((V.graph[u] >> T.bit[k]) & 1u); }
bool pull_ok(const Volume &V, i64 u, int k) { return push_ok(V, u, T.opp[k]); }

constexpr uint64_t kUnclaimed = ~uint64_t{0};

// Railroad (lockstep_coop.inc:71-305 semantics; trace_primitives.cu:282-311): SSSP from `target`
// over the object's voxels, entering v costs pdrf[v] (vw_step); rails (pdrf == 0) absorb. The
// nearest rail is the least (distance bits, flat); the path walks back from it by the argmin
// neighbour distance (non-rail neighbours, lowest table index on ties), after re-picking the join
// as the last road voxel's first rail in dijkstra3d order (lockstep_regular.inc:61-155).
// Returns the path target-first, or an empty path when no rail is reachable.
std::vector<i64> railroad(Volume &V, uint32_t label, i64 target, std::vector<i64> &touched,
                          bool keep_distances = false) {
  const Shape &s = V.s; const auto &ids = *V.ids;
  if (V.pdrf[target] == 0.0f) return {target};
  using Item = std::pair<float, i64>;
  std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
  touched.clear();
  V.dist[target] = 0.0f; touched.push_back(target); heap.push({0.0f, target});
  uint64_t best = ~uint64_t{0};
  while (!heap.empty()) {
    auto [d, u] = heap.top();
    if (best != ~uint64_t{0} && d > bitsf(uint32_t(best >> 32))) break;
    heap.pop();
    if (d > V.dist[u]) continue;
    if (V.pdrf[u] == 0.0f) continue;  // rails absorb
    i64 x, y, z; s.xyz(u, x, y, z);
    for (int k = 0; k < 26; ++k) {
      const i64 nx = x + T.dx[k], ny = y + T.dy[k], nz = z + T.dz[k];
      if (!s.inside(nx, ny, nz)) continue;
      const i64 v = s.idx(nx, ny, nz);
      if (ids[v] != label || !push_ok(V, u, k)) continue;
      const float cand = vw_step(d, V.pdrf[v]);
      if (cand < V.dist[v]) {
        if (V.dist[v] == kInf) touched.push_back(v);
        V.dist[v] = cand;
        if (V.pdrf[v] == 0.0f) {
          const uint64_t key = (uint64_t(fbits(cand)) << 32) | uint64_t(uint32_t(v));
          best = std::min(best, key);
        }
        heap.push({cand, v});
      }
    }
  }
  std::vector<i64> walk;
  if (best != ~uint64_t{0}) {
    i64 cur = i64(uint32_t(best));
    i64 x, y, z; s.xyz(cur, x, y, z);
    for (int step = 0;; ++step) {
      int kb = -1;
      if (cur != target) {
        uint32_t mb = 0x7f800000u;
        for (int k = 0; k < 26; ++k) {
          const i64 nx = x + T.dx[k], ny = y + T.dy[k], nz = z + T.dz[k];
          if (!s.inside(nx, ny, nz)) continue;
          const i64 u = s.idx(nx, ny, nz);
          if (ids[u] != label || V.pdrf[u] == 0.0f || !pull_ok(V, u, k)) continue;
          const uint32_t db = fbits(V.dist[u]);
          if (db < mb) { mb = db; kb = k; }
        }
      }
      if (step == 0 && kb >= 0) {  // the join: u's first rail in dijkstra3d order
        const i64 ux = x + T.dx[kb], uy = y + T.dy[kb], uz = z + T.dz[kb];
        const i64 road = s.idx(ux, uy, uz);
        for (int r = 0; r < 26; ++r) {
          const int k = T.d3inv[r];
          const i64 nx = ux + T.dx[k], ny = uy + T.dy[k], nz = uz + T.dz[k];
          if (!s.inside(nx, ny, nz)) continue;
          const i64 v = s.idx(nx, ny, nz);
          if (ids[v] != label || V.pdrf[v] != 0.0f || !push_ok(V, road, k)) continue;
          x = nx; y = ny; z = nz; cur = v; kb = T.opp[k];
          break;
        }
      }
      walk.push_back(cur);
      if (kb < 0) break;
      x += T.dx[kb]; y += T.dy[kb]; z += T.dz[kb];
      cur = s.idx(x, y, z);
    }
    std::reverse(walk.begin(), walk.end());
  }
  if (!keep_distances)
    for (i64 v : touched) V.dist[v] = kInf;
  return walk;
}

// fix_branching=False (trace.cu:151-160, trace_primitives.cu:187-211; lockstep batched.cu:246-250,
// batched_regular.inc:113-152): one vertex-weighted SSSP from the root over the object's PDRF (no
// rails), kept for the object's whole trace; every path walks from its target to the root through
// the argmin-distance neighbour (lowest neighbour index among ties). Paths are written
// target-first, like the railroad's (the assembly does not depend on the order).
void parental_field(Volume &V, uint32_t label, i64 root, const std::vector<i64> &voxels) {
  const Shape &s = V.s; const auto &ids = *V.ids;
  for (i64 v : voxels) V.dist[v] = kInf;
  using Item = std::pair<float, i64>;
  std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
  V.dist[root] = 0.0f; heap.push({0.0f, root});
  while (!heap.empty()) {
    auto [d, u] = heap.top(); heap.pop();
    if (d > V.dist[u]) continue;
    i64 x, y, z; s.xyz(u, x, y, z);
    for (int k = 0; k < 26; ++k) {
      const i64 nx = x + T.dx[k], ny = y + T.dy[k], nz = z + T.dz[k];
      if (!s.inside(nx, ny, nz)) continue;
      const i64 v = s.idx(nx, ny, nz);
      if (ids[v] != label) continue;
      const float cand = vw_step(d, V.pdrf[v]);
      if (cand < V.dist[v]) { V.dist[v] = cand; heap.push({cand, v}); }
    }
  }
}

std::vector<i64> parent_walk(const Volume &V, uint32_t label, i64 target, i64 root, i64 limit) {
  const Shape &s = V.s; const auto &ids = *V.ids;
  std::vector<i64> walk;
  i64 cur = target;
  while (i64(walk.size()) < limit) {
    walk.push_back(cur);
    if (cur == root || !(V.dist[cur] < kInf)) break;
    i64 x, y, z; s.xyz(cur, x, y, z);
    float best = kInf; i64 next = -1;
    for (int k = 0; k < 26; ++k) {
      const i64 nx = x + T.dx[k], ny = y + T.dy[k], nz = z + T.dz[k];
      if (!s.inside(nx, ny, nz)) continue;
      const i64 u = s.idx(nx, ny, nz);
      if (ids[u] != label) continue;
      if (V.dist[u] < best) { best = V.dist[u]; next = u; }
    }
    if (next < 0) break;
    cur = next;
  }
  return walk;
}

// Claim-order invalidation (invalidation_kernels.cuh:105-297; lockstep_coop.inc:530-845). Path
// vertices still alive become sources (bottleneck M = 0). A claimed voxel u holding (M, s) offers
// an alive neighbour v of the object the source s when |aniso * (v - s)| < scale * DBF[s] + const,
// with M' = max(M, |v - s|). Offers inside the current band [k delta, (k+1) delta) claim at once,
// keeping the least (M bits, source); rounds inside a band are synchronous (every frontier voxel
// offers from its key at the round boundary). Voxels offered beyond the band wait; at the band
// boundary each takes the best offer of its claimed neighbours, the smallest of those names the
// next band, and those inside it are claimed. Returns the number of voxels invalidated.
i64 invalidate(Volume &V, uint32_t label, const std::vector<i64> &path, const Params &P, double reach_scale,
               double reach_constant, std::vector<i64> &touched, std::vector<i64> &frontier, std::vector<i64> &next,
               std::vector<i64> &far, std::vector<i64> &keep, std::vector<uint64_t> &snap) {
  const Shape &s = V.s; const auto &ids = *V.ids;
  const float wx = P.anisotropy[0], wy = P.anisotropy[1], wz = P.anisotropy[2];
  const float scale = float(reach_scale), constant = float(reach_constant);
  const float delta = std::min({wx, wy, wz});
  touched.clear(); frontier.clear(); far.clear();
  for (i64 p : path) {
    if (!V.alive[p]) continue;
    if (V.key[p] == kUnclaimed) {
      V.key[p] = uint64_t(uint32_t(p));
      V.inq[p] = 1; frontier.push_back(p); touched.push_back(p);
    }
  }
  auto distance = [&](i64 vx, i64 vy, i64 vz, i64 src) {
    i64 qx, qy, qz; s.xyz(src, qx, qy, qz);
    const float dvx = wx * float(vx - qx), dvy = wy * float(vy - qy), dvz = wz * float(vz - qz);
    return std::sqrt(dvx * dvx + dvy * dvy + dvz * dvz);
  };
  auto reach = [&](i64 src) { return scale * V.dbf[src] + constant; };
  auto band_of = [&](uint32_t mbits, int kmin) {
    const float m = bitsf(mbits);
    int k = int(m / delta);
    while (float(k + 1) * delta <= m) ++k;
    while (k > 0 && float(k) * delta > m) --k;
    return k < kmin ? kmin : k;
  };
  int band = 0;
  for (;;) {
    uint32_t hi = fbits(float(band + 1) * delta);
    while (!frontier.empty()) {
      snap.resize(frontier.size());
      for (size_t i = 0; i < frontier.size(); ++i) { snap[i] = V.key[frontier[i]]; V.inq[frontier[i]] = 0; }
      next.clear();
      for (size_t i = 0; i < frontier.size(); ++i) {
        const i64 u = frontier[i];
        const i64 src = i64(uint32_t(snap[i]));
        const uint32_t mu = uint32_t(snap[i] >> 32);
        const float maxd = reach(src);
        i64 x, y, z; s.xyz(u, x, y, z);
        for (int k = 0; k < 26; ++k) {
          const i64 nx = x + T.dx[k], ny = y + T.dy[k], nz = z + T.dz[k];
          if (!s.inside(nx, ny, nz)) continue;
          const i64 v = s.idx(nx, ny, nz);
          if (!V.alive[v] || ids[v] != label) continue;
          const float d = distance(nx, ny, nz, src);
          if (d >= maxd) continue;
          uint32_t mb = fbits(d);
          if (mb < mu) mb = mu;
          if (mb < hi) {
            const uint64_t cand = (uint64_t(mb) << 32) | uint64_t(uint32_t(src));
            if (cand < V.key[v]) {
              if (V.key[v] == kUnclaimed) touched.push_back(v);
              V.key[v] = cand;
              if (V.inq[v] != 1) { V.inq[v] = 1; next.push_back(v); }
            }
          } else if (V.key[v] == kUnclaimed && V.inq[v] == 0) {
            V.inq[v] = 2; far.push_back(v);
          }
        }
      }
      frontier.swap(next);
    }
    if (far.empty()) break;
    // band boundary: every waiting voxel pulls the best offer of its claimed neighbours
    std::vector<uint64_t> pulled(far.size(), kUnclaimed);
    std::vector<uint8_t> state(far.size(), 0);  // 0 no offer, 1 offer, 2 claimed meanwhile
    uint32_t lowest = 0x7f800000u;
    for (size_t i = 0; i < far.size(); ++i) {
      const i64 c = far[i];
      if (V.key[c] != kUnclaimed) { state[i] = 2; continue; }
      i64 x, y, z; s.xyz(c, x, y, z);
      uint64_t bestk = kUnclaimed;
      for (int k = 0; k < 26; ++k) {
        const i64 nx = x + T.dx[k], ny = y + T.dy[k], nz = z + T.dz[k];
        if (!s.inside(nx, ny, nz)) continue;
        const i64 u = s.idx(nx, ny, nz);
        if (ids[u] != label || V.key[u] == kUnclaimed) continue;
        const i64 src = i64(uint32_t(V.key[u]));
        const float d = distance(x, y, z, src);
        if (d >= reach(src)) continue;
        uint32_t mb = fbits(d); const uint32_t mu = uint32_t(V.key[u] >> 32);
        if (mb < mu) mb = mu;
        bestk = std::min(bestk, (uint64_t(mb) << 32) | uint64_t(uint32_t(src)));
      }
      if (bestk != kUnclaimed) { state[i] = 1; pulled[i] = bestk; lowest = std::min(lowest, uint32_t(bestk >> 32)); }
    }
    if (lowest != 0x7f800000u) band = band_of(lowest, band + 1);
    hi = fbits(float(band + 1) * delta);
    keep.clear();
    for (size_t i = 0; i < far.size(); ++i) {
      const i64 c = far[i];
      if (state[i] == 2) continue;
      if (state[i] == 0) { V.inq[c] = 0; continue; }
      if (uint32_t(pulled[i] >> 32) < hi) {
        V.key[c] = pulled[i]; touched.push_back(c); frontier.push_back(c); V.inq[c] = 1;
      } else keep.push_back(c);
    }
    far.swap(keep);
  }
  for (i64 v : touched) { V.alive[v] = 0; V.key[v] = kUnclaimed; V.inq[v] = 0; }
  for (i64 v : far) V.inq[v] = 0;
  return i64(touched.size());
}

struct ObjectPlan {
  uint32_t id;
  i64 root, target;
  std::vector<i64> voxels;     // ascending flat
  std::vector<i64> order;      // target order
  std::vector<i64> manual;     // manual targets in pop order
  std::vector<i64> after;      // targets after the automatic ones, in pop order
  i64 max_paths;
  Volume *vol = nullptr;       // the volume the object is traced in (the input, or its own crop)
  uint32_t label = 0;          // the object's id in that volume
  std::array<i64, 3> origin{}; // where that volume's (0, 0, 0) lies in the input
  bool soma = false;
  double soma_radius = 0;      // paths are trimmed to this distance from the root
};

// The trace loop of one object (trace.cu:196-246 order, lockstep.cu:91-183 targets): manual
// targets first, then the first alive voxel of the target order, then, once no voxel is alive,
// the targets after (trace.cu:209-212); railroad; invalidation; the path becomes rails.
// Soma trimming (trace.cu:222-236): a path keeps its first vertex and every vertex farther than
// the soma radius from the root (float64 distance from the float32 root); with fix_branching a
// rail end within the radius gives way to the root. Without fix_branching the reference's paths
// are root-first, so the kept first vertex is the root.
std::vector<i64> trim_to_soma(const Shape &s, const std::vector<i64> &path, i64 root, double radius, const Params &P) {
  if (path.empty()) return path;
  i64 rx, ry, rz; s.xyz(root, rx, ry, rz);
  const double r[3] = {double(float(rx)), double(float(ry)), double(float(rz))};
  auto far = [&](i64 v) {
    i64 x, y, z; s.xyz(v, x, y, z);
    const double p[3] = {double(x), double(y), double(z)};
    double squared = 0;
    for (int k = 0; k < 3; ++k) { const double d = double(P.anisotropy[k]) * (p[k] - r[k]); squared += d * d; }
    return std::sqrt(squared) > radius;
  };
  std::vector<i64> ordered = path;
  if (!P.fix_branching) std::reverse(ordered.begin(), ordered.end());  // root first
  std::vector<i64> out = {ordered.front()};
  bool last_far = true;
  for (i64 v : ordered) {
    last_far = far(v);
    if (last_far) out.push_back(v);
  }
  if (P.fix_branching && !last_far) out.push_back(root);
  return out;
}

std::vector<std::vector<i64>> trace_object(Volume &V, const ObjectPlan &plan, const Params &P) {
  std::vector<std::vector<i64>> paths;
  std::vector<i64> touched, frontier, next, far, keep, rtouched;
  std::vector<uint64_t> snap;
  const uint32_t label = plan.label;
  if (plan.soma)  // the soma's ball first, with the soma's reach (trace.cu:199)
    invalidate(V, label, {plan.root}, P, P.soma_scale, P.soma_constant, touched, frontier, next, far, keep, snap);
  if (plan.max_paths <= 0) return paths;
  if (P.fix_branching) V.pdrf[plan.root] = 0.0f;  // the root is the first rail
  else parental_field(V, label, plan.root, plan.voxels);
  size_t cursor = 0, after = 0;
  while (i64(paths.size()) < plan.max_paths) {
    i64 t = -1;
    bool from_order = false;
    const size_t iter = paths.size();
    if (iter < plan.manual.size()) t = plan.manual[iter];
    else {
      while (cursor < plan.order.size() && !V.alive[plan.order[cursor]]) ++cursor;
      if (cursor < plan.order.size()) { t = plan.order[cursor]; from_order = true; }
      else if (after < plan.after.size()) t = plan.after[after++];
      else break;
    }
    std::vector<i64> path = P.fix_branching ? railroad(V, label, t, rtouched)
                                            : parent_walk(V, label, t, plan.root, i64(plan.voxels.size()) + 1);
    if (path.empty()) {
      // No rail is reachable from t (an infinite penalty walls it off: a cavity the avocado stage
      // painted without refreshing the field). A target of the DAF order ends the object, since
      // it would be picked again and again (trace.cu:218-224); a manual target leaves an empty path.
      if (from_order) break;
      paths.push_back({});
      continue;
    }
    if (plan.soma) path = trim_to_soma(V.s, path, plan.root, plan.soma_radius, P);
    invalidate(V, label, path, P, P.scale, P.constant, touched, frontier, next, far, keep, snap);
    if (P.fix_branching)
      for (i64 v : path) V.pdrf[v] = 0.0f;
    paths.push_back(std::move(path));
  }
  if (!P.fix_branching)
    for (i64 v : plan.voxels) V.dist[v] = kInf;
  return paths;
}

// consolidate (skeleton.cpp:13-40) on voxel coordinates, then physical vertices and radii. A path
// is a list of input-volume voxel coordinates with the DBF of the volume it was traced in.
struct Skeleton {
  int64_t label = 0;
  std::vector<std::array<i64, 3>> vox;
  std::vector<float> radius;
  std::vector<std::array<uint32_t, 2>> edges;
};

struct CoordPath {
  std::vector<std::array<i64, 3>> pts;
  std::vector<float> radius;
};

Skeleton assemble(const std::vector<CoordPath> &paths) {
  Skeleton out;
  std::vector<std::array<i64, 3>> vertices;
  std::vector<float> radius;
  std::vector<std::array<uint32_t, 2>> edges;
  for (const auto &path : paths) {
    if (path.pts.size() < 2) continue;
    const uint32_t base = uint32_t(vertices.size());
    for (size_t j = 0; j < path.pts.size(); ++j) {
      vertices.push_back(path.pts[j]);
      radius.push_back(path.radius[j]);
      if (j) edges.push_back({uint32_t(base + j - 1), uint32_t(base + j)});
    }
  }
  if (vertices.empty() || edges.empty()) return out;
  std::vector<uint32_t> order(vertices.size()), inverse(vertices.size());
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return vertices[a] < vertices[b]; });
  std::vector<std::array<i64, 3>> uniq;
  std::vector<float> uniq_radius;
  for (uint32_t old : order) {
    if (uniq.empty() || uniq.back() != vertices[old]) { uniq.push_back(vertices[old]); uniq_radius.push_back(radius[old]); }
    inverse[old] = uint32_t(uniq.size() - 1);
  }
  std::vector<std::array<uint32_t, 2>> e2;
  for (auto e : edges) {
    std::array<uint32_t, 2> f = {inverse[e[0]], inverse[e[1]]};
    if (f[0] > f[1]) std::swap(f[0], f[1]);
    if (f[0] != f[1]) e2.push_back(f);
  }
  std::sort(e2.begin(), e2.end());
  e2.erase(std::unique(e2.begin(), e2.end()), e2.end());
  std::vector<uint8_t> used(uniq.size(), 0);
  for (auto e : e2) used[e[0]] = used[e[1]] = 1;
  std::vector<uint32_t> remap(uniq.size(), 0);
  for (size_t i = 0; i < uniq.size(); ++i)
    if (used[i]) { remap[i] = uint32_t(out.vox.size()); out.vox.push_back(uniq[i]); out.radius.push_back(uniq_radius[i]); }
  for (auto &e : e2) e = {remap[e[0]], remap[e[1]]};
  out.edges = std::move(e2);
  return out;
}

// ---------------------------------------------------------------------------------------------
// Somata (trace.cu:98-131, soma.cu:141-237). fill_voids (trace_primitives.cu:238-253,
// fillvoids_kernels.cuh): background voxels of the crop that are not 6-connected to the crop's
// faces become foreground. Returns the number filled.
i64 fill_voids(std::vector<uint32_t> &mask, const Shape &s) {
  std::vector<uint8_t> seen(mask.size(), 0);
  std::vector<i64> stack;
  for (i64 v = 0; v < s.n(); ++v) {
    if (mask[v]) continue;
    i64 x, y, z; s.xyz(v, x, y, z);
    if (x == 0 || y == 0 || z == 0 || x == s.sx - 1 || y == s.sy - 1 || z == s.sz - 1) { seen[v] = 1; stack.push_back(v); }
  }
  while (!stack.empty()) {
    const i64 u = stack.back(); stack.pop_back();
    i64 x, y, z; s.xyz(u, x, y, z);
    for (int k = 0; k < 6; ++k) {
      const i64 nx = x + T.dx[k], ny = y + T.dy[k], nz = z + T.dz[k];
      if (!s.inside(nx, ny, nz)) continue;
      const i64 v = s.idx(nx, ny, nz);
      if (mask[v] || seen[v]) continue;
      seen[v] = 1; stack.push_back(v);
    }
  }
  i64 filled = 0;
  for (i64 v = 0; v < s.n(); ++v)
    if (!mask[v] && !seen[v]) { mask[v] = 1; ++filled; }
  return filled;
}

// fill_holes (holes.cu:38-67; its call in skeletonize.cu:86-90 and batch.cu:217-220): components
// in ascending id, each in its original box; the voxels of the current ids equal to the id form a
// mask whose voids are filled (fill_voids); every voxel of the filled mask is painted with the id,
// and a painted voxel's earlier nonzero id (another component) disables that component, which is
// then filled no more. `box` holds the original boxes (lo x y z, hi x y z, count). Returns the
// voxels filled by the components that were filled.
i64 fill_all_holes(std::vector<uint32_t> &ids, const Shape &s, const std::vector<std::array<i64, 7>> &box) {
  std::vector<uint8_t> disabled(box.size(), 0);
  i64 total = 0;
  for (size_t id = 1; id < box.size(); ++id) {
    const auto &b = box[id];
    if (!b[6] || disabled[id]) continue;
    const Shape cs{b[3] - b[0] + 1, b[4] - b[1] + 1, b[5] - b[2] + 1};
    std::vector<uint32_t> mask(cs.n());
    for (i64 c = 0; c < cs.n(); ++c) {
      i64 x, y, z; cs.xyz(c, x, y, z);
      mask[c] = ids[s.idx(x + b[0], y + b[1], z + b[2])] == uint32_t(id) ? 1u : 0u;
    }
    const i64 filled = fill_voids(mask, cs);
    if (!filled) continue;
    total += filled;
    for (i64 c = 0; c < cs.n(); ++c) {
      if (!mask[c]) continue;
      i64 x, y, z; cs.xyz(c, x, y, z);
      uint32_t &v = ids[s.idx(x + b[0], y + b[1], z + b[2])];
      if (v && v != uint32_t(id)) disabled[v] = 1;
      v = uint32_t(id);
    }
  }
  return total;
}

// ---------------------------------------------------------------------------------------------
// The avocado stage (avocado.cpp:223-239, restating Kimimaro 5.8.1's engage_avocado_protection).
// Its candidates are iterated in the order of a CPython 3.12 set of ints, restated here from
// CPython's setobject.c rules: table of 2^k slots (8 at first), hash(k) == k, probe i, then up to 9
// slots after it, then i = (5 i + 1 + perturb) & mask with perturb >>= 5; a deleted slot is a
// dummy, and a new key takes the last dummy its probe passed before reaching an empty slot; the
// table grows to hold 4x the live keys (2x past 50000) when fill reaches 3/5 of it.
struct PySet {
  std::vector<i64> key;          // -1 empty, -2 dummy, else the key
  i64 used = 0, fill = 0;
  PySet() : key(8, -1) {}
  i64 mask() const { return i64(key.size()) - 1; }
  // the slot holding k, or where k would go (the last dummy passed before an empty slot, else
  // that empty slot)
  i64 find(i64 k, bool clean) const {
    uint64_t perturb = uint64_t(k);
    i64 i = k & mask(), dummy = -1;
    for (;;) {
      const i64 probes = i + 9 <= mask() ? 9 : 0;
      for (i64 j = 0; j <= probes; ++j) {
        const i64 e = key[i + j];
        if (e == -1) return dummy >= 0 ? dummy : i + j;
        if (!clean && e == k) return i + j;
        if (!clean && e == -2) dummy = i + j;  // the last dummy passed takes the key
      }
      perturb >>= 5;
      i = i64((uint64_t(i) * 5 + 1 + perturb) & uint64_t(mask()));
    }
  }
  void resize(i64 minused) {
    i64 size = 8;
    while (size <= minused) size <<= 1;
    if (size == 8 && i64(key.size()) == 8 && fill == used) return;
    std::vector<i64> old;
    old.swap(key);
    key.assign(size, -1);
    fill = used;
    for (i64 e : old) if (e >= 0) key[find(e, true)] = e;
  }
  bool contains(i64 k) const { return key[find(k, false)] == k; }
  void add(i64 k) {
    const i64 at = find(k, false);
    if (key[at] == k) return;
    const bool fresh = key[at] == -1;
    key[at] = k;
    ++used;
    if (fresh && ++fill * 5 >= mask() * 3) resize(used > 50000 ? used * 2 : used * 4);
  }
  void discard(i64 k) {
    const i64 at = find(k, false);
    if (key[at] == k) { key[at] = -2; --used; }
  }
  void difference_update(const PySet &o) {
    for (i64 e : o.key) if (e >= 0) discard(e);
    if (fill - used > mask() / 4) resize(used > 50000 ? used * 2 : used * 4);
  }
  void update(const PySet &o) {
    if (&o == this || !o.used) return;
    if ((fill + o.used) * 5 >= mask() * 3) resize((used + o.used) * 2);
    if (!fill && key.size() == o.key.size() && o.fill == o.used) { key = o.key; fill = o.fill; used = o.used; return; }
    if (!fill) {
      fill = used = o.used;
      for (i64 e : o.key) if (e >= 0) key[find(e, true)] = e;
      return;
    }
    for (i64 e : o.key) if (e >= 0) add(e);
  }
  std::vector<i64> items() const {
    std::vector<i64> out;
    for (i64 e : key) if (e >= 0) out.push_back(e);
    return out;
  }
};

// fill_voids 2.1.2 on a binary crop (avocado.cpp:23-52): background reached from the crop's faces
// becomes 0, everything else 1. In 3D the seeds are, on each face scanned row after row, the first
// background voxel of every background run (the run state carries over from one row to the next);
// in 2D every background pixel on the border. The flood is 6- (4-) connected.
void avocado_fill(std::vector<uint8_t> &m, const i64 s[3], int dims) {
  std::vector<i64> queue;
  auto at = [&](const i64 p[3]) { return p[0] + s[0] * (p[1] + s[1] * p[2]); };
  if (dims == 3) {
    const int axes[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
    for (const auto &ax : axes)
      for (int side = 0; side < 2; ++side) {
        bool background = false;
        for (i64 v = 0; v < s[ax[1]]; ++v)
          for (i64 u = 0; u < s[ax[0]]; ++u) {
            i64 p[3];
            p[ax[0]] = u; p[ax[1]] = v; p[ax[2]] = side ? s[ax[2]] - 1 : 0;
            const i64 i = at(p);
            if (!m[i] && !background) queue.push_back(i);
            background = !m[i];
          }
      }
    for (i64 i : queue) m[i] = 2;
  } else {
    for (i64 y = 0; y < s[1]; ++y)
      for (i64 x = 0; x < s[0]; ++x) {
        const i64 i = x + s[0] * y;
        if (!m[i] && (x == 0 || x == s[0] - 1 || y == 0 || y == s[1] - 1)) { m[i] = 2; queue.push_back(i); }
      }
  }
  for (size_t head = 0; head < queue.size(); ++head) {
    const i64 i = queue[head];
    const i64 p[3] = {i % s[0], (i / s[0]) % s[1], i / (s[0] * s[1])};
    for (int a = 0; a < dims; ++a)
      for (int d = -1; d <= 1; d += 2) {
        i64 q[3] = {p[0], p[1], p[2]};
        q[a] += d;
        if (q[a] < 0 || q[a] >= s[a]) continue;
        const i64 j = at(q);
        if (!m[j]) { m[j] = 2; queue.push_back(j); }
      }
  }
  for (auto &v : m) v = v == 2 ? 0 : 1;
}

// Each of the crop's six faces filled as a 2D image, in the order (x, y | z low, high),
// (x, z | y low, high), (y, z | x low, high) (avocado.cpp:53-66).
void avocado_walls(std::vector<uint8_t> &m, const i64 s[3]) {
  const int axes[3][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}};
  for (const auto &ax : axes)
    for (int side = 0; side < 2; ++side) {
      const i64 ps[3] = {s[ax[0]], s[ax[1]], 1};
      std::vector<uint8_t> plane(ps[0] * ps[1]);
      auto voxel = [&](i64 u, i64 v) {
        i64 p[3];
        p[ax[0]] = u; p[ax[1]] = v; p[ax[2]] = side ? s[ax[2]] - 1 : 0;
        return p[0] + s[0] * (p[1] + s[1] * p[2]);
      };
      for (i64 v = 0; v < ps[1]; ++v)
        for (i64 u = 0; u < ps[0]; ++u) plane[u + ps[0] * v] = m[voxel(u, v)];
      avocado_fill(plane, ps, 2);
      for (i64 v = 0; v < ps[1]; ++v)
        for (i64 u = 0; u < ps[0]; ++u) m[voxel(u, v)] = plane[u + ps[0] * v];
    }
}

// The rays from `c` (avocado.cpp:67-80): along each axis up (to the last voxel) and down (to
// coordinate 1), each stops at background or at the first other id (a hit). Fewer than three hits:
// (pit, pit); else the most hit id (the least such id on ties) owns the pit unless more rays than
// (one, with four or more hits; none with three) missed it.
std::pair<i64, i64> avocado_fruit(const std::vector<uint32_t> &ids, const Shape &s, const i64 c[3]) {
  const i64 pit = ids[s.idx(c[0], c[1], c[2])];
  std::map<i64, int> hits;
  int rays = 0;
  const i64 ext[3] = {s.sx, s.sy, s.sz};
  for (int a = 0; a < 3; ++a)
    for (int d : {1, -1}) {
      i64 p[3] = {c[0], c[1], c[2]};
      for (; d > 0 ? p[a] < ext[a] : p[a] > 0; p[a] += d) {
        const i64 v = ids[s.idx(p[0], p[1], p[2])];
        if (!v) break;
        if (v != pit) { ++hits[v]; ++rays; break; }
      }
    }
  if (rays < 3) return {pit, pit};
  i64 owner = pit;
  int most = 0;
  for (const auto &h : hits)
    if (h.second > most) { owner = h.first; most = h.second; }
  if (rays - most > (rays > 3 ? 1 : 0)) return {pit, pit};
  return {pit, owner};
}

// The stage on one volume: cc (ids, mapping, first voxels) and its DBF, both changed in place.
// Up to 20 passes: the ids holding a voxel beyond threshold / 2.5 that no earlier pass left
// unchanged are the candidates; each candidate's crop (its box at the pass's start) gets its faces'
// holes filled, its DBF-weighted argmax is the centre of the rays; a pit merges into its owner
// (the crop's owner voxels join the mask), and the mask's voids are painted with the owner. A pass
// that merged something refreshes the DBF. Finally the ids are renumbered by first voxel, each new
// id mapped to the original label of the old id at its last run start (fastremap's get_mapping).
// Returns the passes run.
int fix_avocados(Components &cc, std::vector<float> &dbf, const Shape &s, double threshold, const float aniso[3],
                 bool bb, int threads) {
  auto &ids = cc.ids;
  const i64 n = s.n();
  const size_t table = cc.mapping.size();
  const std::vector<uint32_t> original = ids;
  PySet unchanged;
  int passes = 0;
  for (; passes < 20; ++passes) {
    const float cutoff = float(threshold / 2.5);
    std::vector<uint8_t> present(table, 0);
    for (i64 i = 0; i < n; ++i) present[dbf[i] > cutoff ? ids[i] : 0] = 1;
    PySet candidates;
    for (size_t id = 0; id < table; ++id) if (present[id]) candidates.add(i64(id));
    candidates.difference_update(unchanged);
    candidates.discard(0);
    if (!candidates.used) break;
    std::vector<std::array<i64, 6>> box(table, {INT64_MAX, INT64_MAX, INT64_MAX, -1, -1, -1});
    for (i64 i = 0; i < n; ++i)
      if (ids[i]) {
        i64 p[3]; s.xyz(i, p[0], p[1], p[2]);
        auto &b = box[ids[i]];
        for (int a = 0; a < 3; ++a) { b[a] = std::min(b[a], p[a]); b[3 + a] = std::max(b[3 + a], p[a]); }
      }
    PySet cycle, changed;
    for (i64 label : candidates.items()) {
      const auto &b = box[label];
      const i64 cs[3] = {b[3] - b[0] + 1, b[4] - b[1] + 1, b[5] - b[2] + 1};
      const i64 cn = cs[0] * cs[1] * cs[2];
      auto global = [&](i64 c) { return s.idx(b[0] + c % cs[0], b[1] + (c / cs[0]) % cs[1], b[2] + c / (cs[0] * cs[1])); };
      std::vector<uint8_t> m(cn);
      for (i64 c = 0; c < cn; ++c) m[c] = ids[global(c)] == uint32_t(label);
      avocado_walls(m, cs);
      // np.argmax of mask * dbf over the crop in x-fastest order: the first maximum, a NaN wins
      i64 best = 0;
      float maximum = float(m[0]) * dbf[global(0)];
      for (i64 c = 0; c < cn; ++c) {
        const float v = float(m[c]) * dbf[global(c)];
        if (!(v <= maximum) && !std::isnan(maximum)) { maximum = v; best = c; }
      }
      const i64 centre[3] = {b[0] + best % cs[0], b[1] + (best / cs[0]) % cs[1], b[2] + best / (cs[0] * cs[1])};
      const auto [pit, owner] = avocado_fruit(ids, s, centre);
      if (pit == owner && !changed.contains(pit)) cycle.add(pit);
      else {
        cycle.discard(pit); cycle.discard(owner);
        changed.add(pit); changed.add(owner);
        for (i64 c = 0; c < cn; ++c) m[c] |= ids[global(c)] == uint32_t(owner);
      }
      avocado_fill(m, cs, 3);
      for (i64 c = 0; c < cn; ++c) if (m[c]) ids[global(c)] = uint32_t(owner);
    }
    unchanged.update(cycle);
    if (!changed.used) { ++passes; break; }
    dbf = edt(ids.data(), s, aniso, bb, 3, threads);
  }
  // renumbering by first voxel (avocado.cpp:117-131)
  std::vector<i64> compact(table, 0);
  std::vector<int64_t> mapping{0}, roots;
  i64 previous = -1;
  for (i64 i = 0; i < n; ++i) {
    i64 &k = compact[ids[i]];
    if (ids[i] && !k) { k = i64(roots.size()) + 1; roots.push_back(i); mapping.push_back(0); }
    ids[i] = uint32_t(k);
    if (k != previous) {
      if (k) mapping[k] = original[i] ? cc.mapping[original[i]] : 0;
      previous = k;
    }
  }
  cc.mapping = std::move(mapping);
  cc.roots = std::move(roots);
  return passes;
}

// The soma root (trace.cu:55-73, batched.cu:58-105): among the voxels at the DBF maximum, sorted
// by (x, y, z), the first nearest (float64 squared distance, voxel units) to their float32 centroid.
i64 soma_root(const std::vector<float> &dbf, const std::vector<i64> &voxels, float maximum, const Shape &s) {
  std::vector<std::array<i64, 3>> points;
  for (i64 v : voxels)
    if (dbf[v] == maximum) { i64 x, y, z; s.xyz(v, x, y, z); points.push_back({x, y, z}); }
  if (points.empty()) throw std::runtime_error("no soma maximum");
  std::array<i64, 3> sum{0, 0, 0};
  for (const auto &p : points) for (int k = 0; k < 3; ++k) sum[k] += p[k];
  std::sort(points.begin(), points.end());
  float centre[3];
  for (int k = 0; k < 3; ++k) centre[k] = float(double(sum[k]) / double(points.size()));
  double best = INFINITY;
  std::array<i64, 3> root = points.front();
  for (const auto &p : points) {
    double cost = 0;
    for (int k = 0; k < 3; ++k) { const double d = double(p[k]) - double(centre[k]); cost += d * d; }
    if (cost < best) { best = cost; root = p; }
  }
  return s.idx(root[0], root[1], root[2]);
}

// The free-space seed of a soma's DAF (sssp_kernels.cuh:14-35): every object voxel within the
// radius (float32 physical distance) of the root starts at its 26-connected distance through
// empty space.
void freespace_seed(std::vector<float> &dist, const std::vector<i64> &voxels, const Shape &s, i64 root,
                    const float a[3], float radius) {
  i64 rx, ry, rz; s.xyz(root, rx, ry, rz);
  const float wx = a[0], wy = a[1], wz = a[2];
  for (i64 v : voxels) {
    i64 x, y, z; s.xyz(v, x, y, z);
    const float rdx = wx * float(x - rx), rdy = wy * float(y - ry), rdz = wz * float(z - rz);
    if (rdx * rdx + rdy * rdy + rdz * rdz > radius * radius) continue;
    const float dx = std::fabs(float(x - rx)), dy = std::fabs(float(y - ry)), dz = std::fabs(float(z - rz));
    const float dxyz = std::min(std::min(dx, dy), dz);
    const float dxy = std::min(dx, dy), dyz = std::min(dy, dz), dxz = std::min(dx, dz);
    const float val = dxyz * std::sqrt(wx * wx + wy * wy + wz * wz) + wx * (dx - dxyz) + wy * (dy - dxyz) +
                      wz * (dz - dxyz) + (dxy - dxyz) * (std::sqrt(wx * wx + wy * wy) - wx - wy) +
                      (dxz - dxyz) * (std::sqrt(wx * wx + wz * wz) - wx - wz) +
                      (dyz - dxyz) * (std::sqrt(wy * wy + wz * wz) - wy - wz);
    dist[v] = val;
  }
}

// ---------------------------------------------------------------------------------------------
// The whole path (skeletonize.cu:70-183 with the lockstep inputs of batched.cu:177-255), in three
// steps: prepare (components, boxes, EDT, border targets, roots, DAF, PDRF, target orders), trace
// (objects in largest-first order, any sub-range of that order at a time), finish (assembly).
struct Staged;

struct Result {
  std::vector<int64_t> labels, vertex_offsets{0}, edge_offsets{0};
  std::vector<float> vertices, radii;
  std::vector<uint32_t> edges;
  std::string error;
  int64_t filled = 0;  // voxels fill_holes filled
  int64_t avocado_passes = 0;
  // stage outputs
  Components cc;
  std::vector<float> dbf, daf, pdrf;
  std::vector<int64_t> roots, targets, boxes;  // boxes: per id lo xyz, hi xyz, count
  std::vector<std::vector<std::array<i64, 3>>> borders;
  std::vector<int64_t> orders;                 // concatenated target orders of active ids
  std::vector<int64_t> order_offsets;          // per id (count+2)
  std::vector<int64_t> paths_flat, path_offsets{0}, path_labels;
  // wall-clock ms of the steps: components, boxes, edt, borders, daf, pdrf, orders, trace, assembly
  std::vector<double> stage_ms = std::vector<double>(9, 0.0);
  std::shared_ptr<Staged> staged;  // between prepare and finish
};

// A soma candidate's own crop: its (filled) mask as ids 0/1, and the volume state over it.
struct PrivateVolume {
  std::vector<uint32_t> ids;
  Volume V;
  std::array<i64, 3> origin{};
};

struct Staged {
  Shape s;
  Params P;
  Volume V;
  std::vector<std::unique_ptr<PrivateVolume>> privates;
  int keep_stages = 0;
  std::vector<std::array<i64, 7>> box;
  std::vector<ObjectPlan> plans;
  std::vector<size_t> schedule;  // plans, largest first
  std::vector<std::vector<std::vector<i64>>> traced;
};

struct Lap {
  std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
  double next() {
    const auto now = std::chrono::steady_clock::now();
    const double ms = std::chrono::duration<double, std::milli>(now - t).count();
    t = now;
    return ms;
  }
};

void prepare(Result &R, const void *labels, int dtype, const Shape &s, const Params &P, int threads, int keep_stages) {
  auto st = std::make_shared<Staged>();
  st->s = s; st->P = P; st->keep_stages = keep_stages;
  R.staged = st;
  const i64 n = s.n();
  if (n == 0 || double(n) <= P.dust) return;
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(P.anisotropy[a]) || P.anisotropy[a] <= 0) throw std::invalid_argument("anisotropy must be finite and positive");
  {
    const double e = P.pdrf_exponent;
    if (std::isfinite(e) && e == std::floor(e) && std::fmod(e, 2.0) == 1.0)
      throw std::invalid_argument("odd pdrf_exponent makes the background penalty negative");
  }
  Lap lap;
  R.cc = components_any(labels, dtype, s, threads);
  R.stage_ms[0] = lap.next();
  const auto &ids = R.cc.ids;
  size_t count = R.cc.roots.size();
  if (!count) return;
  // bounding boxes and counts (preamble.cu:10-29), and each id's voxels; with `refresh_first` the
  // first voxels too (preamble.cu:77-90: an id left without voxels keeps its old one)
  auto &box = st->box;
  std::vector<std::vector<i64>> voxels;
  auto analyze_ids = [&](bool refresh_first) {
    box.assign(count + 1, {INT32_MAX, INT32_MAX, INT32_MAX, -1, -1, -1, 0});
    voxels.assign(count + 1, {});
    for (i64 v = 0; v < n; ++v) {
      const uint32_t id = ids[v];
      if (!id) continue;
      i64 x, y, z; s.xyz(v, x, y, z);
      auto &b = box[id];
      b[0] = std::min(b[0], x); b[1] = std::min(b[1], y); b[2] = std::min(b[2], z);
      b[3] = std::max(b[3], x); b[4] = std::max(b[4], y); b[5] = std::max(b[5], z); ++b[6];
      if (refresh_first && voxels[id].empty()) R.cc.roots[id - 1] = v;
      voxels[id].push_back(v);
    }
  };
  analyze_ids(false);
  R.stage_ms[1] = lap.next();
  // black border from the volume as given, before any hole is filled (skeletonize.cu:82-85)
  const bool black_border = count == 1 && box[1][6] == n;
  if (P.fill_holes) {
    R.filled = fill_all_holes(R.cc.ids, s, box);
    if (R.filled) analyze_ids(true);
  }
  Volume &V = st->V;
  V.s = s; V.ids = &R.cc.ids;
  V.dbf = edt(ids.data(), s, P.anisotropy, black_border, 3, threads);
  if (P.fix_avocados) {
    // the avocado stage (skeletonize.cu:92-96): ids renumbered, the field refreshed when it merged
    R.avocado_passes = fix_avocados(R.cc, V.dbf, s, P.soma_detection, P.anisotropy, black_border, threads);
    count = R.cc.roots.size();
    if (!count) return;
    analyze_ids(false);
  }
  R.stage_ms[2] = lap.next();
  std::vector<std::vector<std::array<i64, 3>>> borders(count + 1);
  if (P.fix_borders) borders = border_targets(ids, s, count, P.anisotropy);
  R.stage_ms[3] = lap.next();
  // active objects (batched.cu:187-191): more voxels than dust and a bounding box of 2+ voxels
  std::vector<uint8_t> active(count + 1, 0), candidate(count + 1, 0);
  std::vector<float> dbf_max(count + 1, 0.0f);
  for (size_t id = 1; id <= count; ++id) {
    const auto &b = box[id];
    const i64 bbox = (b[3] - b[0] + 1) * (b[4] - b[1] + 1) * (b[5] - b[2] + 1);
    float m; argmax(V.dbf, voxels[id], m); dbf_max[id] = m;
    if (double(b[6]) <= P.dust || bbox <= 1) continue;
    active[id] = 1;
    // a soma candidate is prepared and traced in a crop of its own (its voids filled)
    if (double(dbf_max[id]) > P.soma_detection) candidate[id] = 1;
  }
  // roots and DAF per object: every object's floods touch only its own voxels
  const Weights W = geometric_weights(P.anisotropy);
  std::vector<float> daf(n, kInf);
  std::vector<int64_t> roots(count + 1, -1), targets(count + 1, -1);
  std::vector<float> max_daf(count + 1, 0.0f);
  parallel_for(i64(count), threads, 1, [&](i64 b, i64 e) {
    for (i64 j = b; j < e; ++j) {
      const size_t id = size_t(j) + 1;
      if (!active[id] || candidate[id]) continue;
      i64 root;
      if (!borders[id].empty()) { const auto &p = borders[id].back(); root = s.idx(p[0], p[1], p[2]); }
      else {
        geometric_flood(ids, s, uint32_t(id), R.cc.roots[id - 1], W, daf, voxels[id]);
        float m; root = argmax(daf, voxels[id], m);
      }
      geometric_flood(ids, s, uint32_t(id), root, W, daf, voxels[id]);
      float m; const i64 target = argmax(daf, voxels[id], m);
      roots[id] = root; targets[id] = target; max_daf[id] = m;
    }
  });
  R.stage_ms[4] = lap.next();
  // PDRF (batched.cu:234-245, batched_regular.inc:93-108, trace_primitives.cu:119-129, 213-229):
  // (1 - dbf * M)^e * scale + daf * inv. A power-of-two e is repeated squaring in float32, as in
  // the reference; any other e is the reference's powf, restated here as the float64 power
  // rounded to float32 (within a few ulp of CUDA's powf, not bit for bit).
  const double exponent = P.pdrf_exponent;
  int squarings = -1;
  if (exponent > 0 && exponent < 65536 && exponent == std::floor(exponent) && !(int(exponent) & (int(exponent) - 1))) {
    squarings = 0;
    for (int e = int(exponent); e > 1; e >>= 1) ++squarings;
  }
  V.pdrf.assign(n, kInf);
  {
    std::vector<float> M(count + 1, 0.0f), inv(count + 1, 0.0f);
    std::vector<uint8_t> use(count + 1, 0);
    for (size_t id = 1; id <= count; ++id)
      if (active[id] && !candidate[id]) {
        M[id] = float(1.0 / std::pow(double(dbf_max[id]), 1.01));
        if (max_daf[id] != 0) { inv[id] = float(1.0 / double(max_daf[id])); use[id] = 2; } else use[id] = 1;
      }
    const float scale = float(P.pdrf_scale);
    parallel_for(n, threads, 1 << 16, [&](i64 b, i64 e) {
      for (i64 i = b; i < e; ++i) {
        const uint32_t L = ids[i];
        if (L == 0 || use[L] == 0) continue;
        float d = V.dbf[i];
        if (d == 0.0f) d = kInf;
        float p = 1.0f - d * M[L];
        if (squarings >= 0) for (int k = 0; k < squarings; ++k) p = p * p;
        else p = float(std::pow(double(p), exponent));
        p = p * scale;
        if (use[L] == 2) { float dd = daf[i]; if (std::isinf(dd)) dd = 0.0f; p = p + dd * inv[L]; }
        V.pdrf[i] = p;
      }
    });
  }
  if (P.pdrf_field) {  // a test's field replaces the computed one over the traced objects' voxels
    for (i64 i = 0; i < n; ++i)
      if (ids[i] && active[ids[i]] && !candidate[ids[i]]) V.pdrf[i] = P.pdrf_field[i];
  }
  R.stage_ms[5] = lap.next();
  if (keep_stages) { R.dbf = V.dbf; R.daf = daf; R.pdrf = V.pdrf; }
  // extra targets by the component they fall on (skeletonize.cu:16-25, 61-65): a negative
  // coordinate counts from the end of its axis; a point outside the volume is an error
  std::vector<std::vector<i64>> before_of(count + 1), after_of(count + 1);
  for (int list = 0; list < 2; ++list)
    for (auto p : list ? P.after : P.before) {
      const i64 shape[3] = {s.sx, s.sy, s.sz};
      for (int a = 0; a < 3; ++a) {
        if (p[a] < 0) p[a] += shape[a];
        if (p[a] < 0 || p[a] >= shape[a]) throw std::invalid_argument("extra target is outside the input volume");
      }
      const i64 flat = s.idx(p[0], p[1], p[2]);
      (list ? after_of : before_of)[ids[flat]].push_back(flat);
    }
  // target orders and manual targets (lockstep.cu:120-142, lockstep_order.cu:21-45)
  auto &plans = st->plans;
  for (size_t id = 1; id <= count; ++id) {
    if (!active[id] || candidate[id]) continue;
    ObjectPlan plan;
    plan.id = uint32_t(id); plan.root = roots[id]; plan.target = targets[id];
    plan.vol = &V; plan.label = uint32_t(id);
    plan.voxels = std::move(voxels[id]);
    std::vector<i64> manual;
    for (const auto &p : borders[id]) manual.push_back(s.idx(p[0], p[1], p[2]));
    if (!manual.empty()) manual.pop_back();
    manual.insert(manual.end(), before_of[id].begin(), before_of[id].end());
    if (manual.empty()) plan.manual.push_back(targets[id]);
    else plan.manual.assign(manual.rbegin(), manual.rend());
    plan.after.assign(after_of[id].rbegin(), after_of[id].rend());
    const i64 budget = P.has_max_paths ? P.max_paths : box[id][6];
    plan.max_paths = i64(plan.manual.size() + plan.after.size()) >= budget ? 0 : budget;
    plans.push_back(std::move(plan));
  }
  // soma candidates (prepare_component, trace.cu:98-131): the crop of the object's box with its
  // voids filled; the DBF recomputed on that crop when anything was filled (black border when it
  // fills the crop), else the input's; a soma when the maximum passes soma_acceptance_threshold:
  // the root at the maximum nearest the maxima's centroid, the DAF seeded through free space
  // within the maximum of the root, the border root traced last among the manual targets and no
  // default target
  std::vector<size_t> soma_ids;
  for (size_t id = 1; id <= count; ++id) if (candidate[id]) soma_ids.push_back(id);
  std::vector<ObjectPlan> soma_plans(soma_ids.size());
  st->privates.resize(soma_ids.size());
  parallel_for(i64(soma_ids.size()), threads, 1, [&](i64 b, i64 e) {
    for (i64 j = b; j < e; ++j) {
      const size_t id = soma_ids[j];
      const auto &bx = box[id];
      auto pv = std::make_unique<PrivateVolume>();
      const Shape cs{bx[3] - bx[0] + 1, bx[4] - bx[1] + 1, bx[5] - bx[2] + 1};
      pv->origin = {bx[0], bx[1], bx[2]};
      pv->ids.assign(cs.n(), 0);
      std::vector<float> crop_dbf(cs.n(), 0.0f);
      for (i64 v : voxels[id]) {
        i64 x, y, z; s.xyz(v, x, y, z);
        const i64 c = cs.idx(x - bx[0], y - bx[1], z - bx[2]);
        pv->ids[c] = 1;
        crop_dbf[c] = V.dbf[v];
      }
      const i64 filled = fill_voids(pv->ids, cs);
      const i64 valid = bx[6] + filled;
      Volume &PV = pv->V;
      PV.s = cs; PV.ids = &pv->ids;
      PV.dbf = filled ? edt(pv->ids.data(), cs, P.anisotropy, valid == cs.n(), 3, 1) : std::move(crop_dbf);
      std::vector<i64> cvox;
      for (i64 c = 0; c < cs.n(); ++c) if (pv->ids[c]) cvox.push_back(c);
      float maximum; argmax(PV.dbf, cvox, maximum);
      ObjectPlan plan;
      plan.id = uint32_t(id); plan.vol = &PV; plan.label = 1; plan.origin = pv->origin;
      plan.soma = double(maximum) > P.soma_acceptance;
      auto crop_flat = [&](std::array<i64, 3> p) { return cs.idx(p[0] - bx[0], p[1] - bx[1], p[2] - bx[2]); };
      auto to_crop = [&](i64 v) { i64 x, y, z; s.xyz(v, x, y, z); return cs.idx(x - bx[0], y - bx[1], z - bx[2]); };
      std::vector<float> cdaf(cs.n(), kInf);
      i64 root;
      if (plan.soma) {
        root = soma_root(PV.dbf, cvox, maximum, cs);
        plan.soma_radius = double(maximum) * P.soma_scale + P.soma_constant;
        std::vector<float> seeds(cs.n(), kInf);
        freespace_seed(seeds, cvox, cs, root, P.anisotropy, maximum);
        geometric_flood(pv->ids, cs, 1, root, W, cdaf, cvox, &seeds);
      } else {
        if (!borders[id].empty()) root = crop_flat(borders[id].back());
        else {
          geometric_flood(pv->ids, cs, 1, cvox.front(), W, cdaf, cvox);
          float m; root = argmax(cdaf, cvox, m);
        }
        geometric_flood(pv->ids, cs, 1, root, W, cdaf, cvox);
      }
      float far_daf; const i64 target = argmax(cdaf, cvox, far_daf);
      // PDRF of the crop (the maximum and the farthest DAF of the crop's fields)
      PV.pdrf.assign(cs.n(), kInf);
      const float M = float(1.0 / std::pow(double(maximum), 1.01));
      const float inv = far_daf != 0 ? float(1.0 / double(far_daf)) : 0.0f;
      for (i64 c : cvox) {
        float d = PV.dbf[c];
        if (d == 0.0f) d = kInf;
        float q = 1.0f - d * M;
        if (squarings >= 0) for (int k = 0; k < squarings; ++k) q = q * q;
        else q = float(std::pow(double(q), exponent));
        q = q * float(P.pdrf_scale);
        if (far_daf != 0) { float dd = cdaf[c]; if (std::isinf(dd)) dd = 0.0f; q = q + dd * inv; }
        PV.pdrf[c] = q;
      }
      std::vector<i64> manual;
      for (const auto &p : borders[id]) manual.push_back(crop_flat(p));
      if (!manual.empty()) manual.pop_back();
      if (plan.soma && !borders[id].empty()) manual.insert(manual.begin(), crop_flat(borders[id].back()));
      for (i64 v : before_of[id]) manual.push_back(to_crop(v));
      if (manual.empty() && !plan.soma) plan.manual.push_back(target);
      else plan.manual.assign(manual.rbegin(), manual.rend());
      for (auto it = after_of[id].rbegin(); it != after_of[id].rend(); ++it) plan.after.push_back(to_crop(*it));
      const i64 budget = P.has_max_paths ? P.max_paths : valid;
      plan.max_paths = i64(plan.manual.size() + plan.after.size()) >= budget ? 0 : budget;
      plan.root = root; plan.target = target;
      plan.voxels = cvox;
      plan.order = cvox;
      std::sort(plan.order.begin(), plan.order.end(), [&](i64 a, i64 c) {
        float x = cdaf[a], y = cdaf[c];
        if (std::isinf(x)) x = 0;
        if (std::isinf(y)) y = 0;
        return x == y ? a > c : x > y;
      });
      PV.dist.assign(cs.n(), kInf);
      PV.alive.assign(pv->ids.begin(), pv->ids.end());
      PV.inq.assign(cs.n(), 0);
      PV.key.assign(cs.n(), kUnclaimed);
      auto to_input = [&](i64 c) { i64 x, y, z; cs.xyz(c, x, y, z); return s.idx(x + bx[0], y + bx[1], z + bx[2]); };
      roots[id] = to_input(root); targets[id] = to_input(target);
      soma_plans[j] = std::move(plan);
      st->privates[j] = std::move(pv);
    }
  });
  parallel_for(i64(plans.size()), threads, 1, [&](i64 b, i64 e) {
    for (i64 j = b; j < e; ++j) {
      ObjectPlan &plan = plans[j];
      plan.order = plan.voxels;
      std::sort(plan.order.begin(), plan.order.end(), [&](i64 a, i64 c) {
        float x = daf[a], y = daf[c];
        if (std::isinf(x)) x = 0;
        if (std::isinf(y)) y = 0;
        return x == y ? a > c : x > y;
      });
    }
  });
  for (auto &plan : soma_plans) plans.push_back(std::move(plan));
  R.stage_ms[6] = lap.next();
  // A foreground voxel at distance zero (background the avocado stage painted without refreshing
  // the field) is +inf to the tracer: its penalty (above), invalidation reach and radius
  // (lockstep.cu:61-82).
  for (i64 i = 0; i < n; ++i)
    if (ids[i] && V.dbf[i] == 0.0f) V.dbf[i] = kInf;
  V.dist.assign(n, kInf);
  V.alive.assign(n, 0);
  for (i64 i = 0; i < n; ++i) V.alive[i] = ids[i] ? active[ids[i]] && !candidate[ids[i]] : 0;
  V.inq.assign(n, 0);
  V.key.assign(n, kUnclaimed);
  st->traced.assign(plans.size(), {});
  // largest objects first, so that a pool of threads finishes together
  st->schedule.resize(plans.size());
  std::iota(st->schedule.begin(), st->schedule.end(), size_t(0));
  std::stable_sort(st->schedule.begin(), st->schedule.end(),
                   [&](size_t a, size_t b) { return plans[a].voxels.size() > plans[b].voxels.size(); });
  R.roots = roots; R.targets = targets; R.borders = std::move(borders);
}

// Traces the objects schedule[begin, end) on `threads` threads (objects never touch each other's
// voxels, so they run concurrently).
void trace(Result &R, size_t begin, size_t end, int threads) {
  Staged &st = *R.staged;
  end = std::min(end, st.schedule.size());
  if (begin >= end) return;
  Lap lap;
  std::atomic<size_t> next{begin};
  std::mutex failure;
  std::string message;
  auto worker = [&] {
    for (;;) {
      const size_t j = next.fetch_add(1);
      if (j >= end) return;
      const size_t i = st.schedule[j];
      try { st.traced[i] = trace_object(*st.plans[i].vol, st.plans[i], st.P); }
      catch (const std::exception &e) { std::lock_guard<std::mutex> lock(failure); message = e.what(); }
    }
  };
  const int workers = std::max(1, std::min<int>(threads, int(end - begin)));
  std::vector<std::thread> pool;
  for (int t = 1; t < workers; ++t) pool.emplace_back(worker);
  worker();
  for (auto &t : pool) t.join();
  R.stage_ms[7] += lap.next();
  if (!message.empty()) throw std::runtime_error(message);
}

// Assembly: one skeleton per original label, components merged in id order (skeletonize.cu:130-181).
void finish(Result &R) {
  Staged &st = *R.staged;
  Lap lap;
  const auto &plans = st.plans;
  const auto &traced = st.traced;
  // every path in input coordinates with the radii of the volume it was traced in; components of
  // one label merge in id order (plans are in id order, the soma candidates' last, so sort)
  std::vector<size_t> by_id(plans.size());
  std::iota(by_id.begin(), by_id.end(), size_t(0));
  std::stable_sort(by_id.begin(), by_id.end(), [&](size_t a, size_t b) { return plans[a].id < plans[b].id; });
  auto coords = [&](size_t j) {
    const ObjectPlan &plan = plans[j];
    const Volume &PV = *plan.vol;
    std::vector<CoordPath> out;
    for (const auto &path : traced[j]) {
      CoordPath cp;
      for (i64 v : path) {
        i64 x, y, z; PV.s.xyz(v, x, y, z);
        cp.pts.push_back({x + plan.origin[0], y + plan.origin[1], z + plan.origin[2]});
        cp.radius.push_back(PV.dbf[v]);
      }
      out.push_back(std::move(cp));
    }
    return out;
  };
  std::vector<int64_t> label_order;
  std::vector<std::vector<CoordPath>> merged;
  for (size_t j : by_id) {
    const int64_t label = R.cc.mapping[plans[j].id];
    auto cps = coords(j);
    Skeleton sk = assemble(cps);
    if (sk.edges.empty()) continue;
    auto it = std::find(label_order.begin(), label_order.end(), label);
    if (it == label_order.end()) { label_order.push_back(label); merged.push_back(std::move(cps)); }
    else { auto &m = merged[it - label_order.begin()]; m.insert(m.end(), cps.begin(), cps.end()); }
  }
  for (size_t j = 0; j < label_order.size(); ++j) {
    Skeleton sk = assemble(merged[j]);
    R.labels.push_back(label_order[j]);
    for (size_t q = 0; q < sk.vox.size(); ++q) {
      for (int a = 0; a < 3; ++a) R.vertices.push_back(float(sk.vox[q][a]) * st.P.anisotropy[a]);
      R.radii.push_back(sk.radius[q]);
    }
    for (const auto &e : sk.edges) { R.edges.push_back(e[0]); R.edges.push_back(e[1]); }
    R.vertex_offsets.push_back(int64_t(R.radii.size()));
    R.edge_offsets.push_back(int64_t(R.edges.size() / 2));
  }
  if (st.keep_stages) {
    const size_t count = R.cc.roots.size();
    R.boxes.clear();
    for (size_t id = 0; id < st.box.size(); ++id) for (int a = 0; a < 7; ++a) R.boxes.push_back(st.box[id][a]);
    R.order_offsets.assign(count + 2, 0);
    for (size_t id = 1; id <= count; ++id) {
      R.order_offsets[id + 1] = R.order_offsets[id];
      auto it = std::find_if(plans.begin(), plans.end(), [&](const ObjectPlan &p) { return p.id == id; });
      if (it == plans.end() || it->vol != &st.V) continue;  // a soma candidate's order is in its crop
      R.orders.insert(R.orders.end(), it->order.begin(), it->order.end());
      R.order_offsets[id + 1] += i64(it->order.size());
    }
    for (size_t j : by_id)
      for (const auto &cp : coords(j)) {
        for (const auto &q : cp.pts) R.paths_flat.push_back(st.s.idx(q[0], q[1], q[2]));
        R.path_offsets.push_back(i64(R.paths_flat.size()));
        R.path_labels.push_back(plans[j].id);
      }
  } else {
    R.roots.clear(); R.targets.clear(); R.borders.clear();
  }
  R.stage_ms[8] = lap.next();
  R.staged.reset();
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// C interface for the Python test harness (ctypes).
extern "C" {

// The penalty of n voxels from their DBF and DAF values, restating the reference's normalisation
// and PDRF arithmetic (cpp/tests/pdrf_fusion_smoke.cu:10-40, trace_primitives.cu:119-129): a DBF of
// 0 becomes +inf and an infinite DAF 0; m = float(1 / maximum^1.01), inverse = float(1 / max_daf)
// when max_daf is not 0; p = 1 - dbf * m, squared log2(exponent) times for a power of two below
// 65536, else pow; times scale; plus daf * inverse when inverse is not 0. The power other than by
// squaring is float(pow(double, double)), which CUDA's powf need not match in the last place.
void oracle_pdrf_values(const float *dbf, const float *daf, int64_t n, double maximum, double max_daf, double scale,
                        double exponent, float *out) {
  const float m = float(1.0 / std::pow(maximum, 1.01));
  const float inverse = max_daf != 0 ? float(1.0 / max_daf) : 0.0f;
  int squarings = -1;
  if (exponent > 0 && exponent < 65536 && std::floor(exponent) == exponent && !(int(exponent) & (int(exponent) - 1))) {
    squarings = 0;
    for (int e = int(exponent); e > 1; e >>= 1) ++squarings;
  }
  for (int64_t i = 0; i < n; ++i) {
    float d = dbf[i], a = daf[i];
    if (d == 0) d = std::numeric_limits<float>::infinity();
    if (std::isinf(a)) a = 0;
    float p = 1.0f - d * m;
    if (squarings >= 0) for (int k = 0; k < squarings; ++k) p = p * p;
    else p = float(std::pow(double(p), exponent));
    p = p * float(scale);
    if (inverse != 0) p = p + a * inverse;
    out[i] = p;
  }
}


struct oracle_params {
  double scale, constant, pdrf_scale, pdrf_exponent;
  double soma_detection, soma_acceptance, soma_scale, soma_constant;
  int64_t max_paths; int32_t has_max_paths;
  float anisotropy[3];
  double dust;
  int32_t fix_branching, fix_borders;
  const int64_t *targets_before; int64_t n_before;  // x, y, z triples
  const int64_t *targets_after; int64_t n_after;
  const float *pdrf_field;  // optional (null: computed)
  int32_t fill_holes;
  int32_t fix_avocados;
};

namespace {
Params params_of(const oracle_params *p) {
    Params P{};
    P.scale = p->scale; P.constant = p->constant; P.pdrf_scale = p->pdrf_scale; P.pdrf_exponent = p->pdrf_exponent;
    P.soma_detection = p->soma_detection; P.soma_acceptance = p->soma_acceptance;
    P.soma_scale = p->soma_scale; P.soma_constant = p->soma_constant;
    P.max_paths = p->max_paths; P.has_max_paths = p->has_max_paths;
    for (int a = 0; a < 3; ++a) P.anisotropy[a] = p->anisotropy[a];
    P.dust = p->dust; P.fix_branching = p->fix_branching; P.fix_borders = p->fix_borders;
    for (int64_t i = 0; i < p->n_before; ++i)
      P.before.push_back({p->targets_before[3 * i], p->targets_before[3 * i + 1], p->targets_before[3 * i + 2]});
    for (int64_t i = 0; i < p->n_after; ++i)
      P.after.push_back({p->targets_after[3 * i], p->targets_after[3 * i + 1], p->targets_after[3 * i + 2]});
    P.pdrf_field = p->pdrf_field;
    P.fill_holes = p->fill_holes;
    P.fix_avocados = p->fix_avocados;
    return P;
}
}  // namespace

// The whole path in one call.
void *oracle_run(const void *labels, int dtype, int64_t sx, int64_t sy, int64_t sz, const oracle_params *p,
                 int threads, int keep_stages) {
  auto *r = new Result();
  try {
    prepare(*r, labels, dtype, Shape{sx, sy, sz}, params_of(p), threads, keep_stages);
    trace(*r, 0, r->staged->schedule.size(), threads);
    finish(*r);
  } catch (const std::exception &e) {
    r->error = e.what();
    r->staged.reset();
  }
  return r;
}

// The same path in steps: oracle_prepare, then oracle_trace over sub-ranges of the largest-first
// object order (oracle_objects of them), then oracle_finish. Errors go to oracle_error.
void *oracle_prepare(const void *labels, int dtype, int64_t sx, int64_t sy, int64_t sz, const oracle_params *p,
                     int threads) {
  auto *r = new Result();
  try {
    prepare(*r, labels, dtype, Shape{sx, sy, sz}, params_of(p), threads, 0);
  } catch (const std::exception &e) {
    r->error = e.what();
    r->staged.reset();
  }
  return r;
}
int64_t oracle_objects(void *h) {
  auto *r = static_cast<Result *>(h);
  return r->staged ? int64_t(r->staged->schedule.size()) : 0;
}
int oracle_trace(void *h, int64_t begin, int64_t end, int threads) {
  auto *r = static_cast<Result *>(h);
  if (!r->staged) return 1;
  try {
    trace(*r, size_t(std::max<int64_t>(begin, 0)), size_t(std::max<int64_t>(end, 0)), threads);
    return 0;
  } catch (const std::exception &e) {
    r->error = e.what();
    return 1;
  }
}
int oracle_finish(void *h) {
  auto *r = static_cast<Result *>(h);
  if (!r->staged) return 1;
  try {
    finish(*r);
    return 0;
  } catch (const std::exception &e) {
    r->error = e.what();
    return 1;
  }
}
void oracle_free(void *h) { delete static_cast<Result *>(h); }
const char *oracle_error(void *h) { return static_cast<Result *>(h)->error.c_str(); }

// Array accessors: name -> (pointer, element count). Element types are fixed per name.
const void *oracle_array(void *h, const char *name, int64_t *count) {
  auto *r = static_cast<Result *>(h);
  const std::string k(name);
  auto give = [&](const auto &v) -> const void * { *count = int64_t(v.size()); return v.data(); };
  if (k == "labels") return give(r->labels);
  if (k == "vertex_offsets") return give(r->vertex_offsets);
  if (k == "edge_offsets") return give(r->edge_offsets);
  if (k == "vertices") return give(r->vertices);
  if (k == "radii") return give(r->radii);
  if (k == "edges") return give(r->edges);
  if (k == "cc") return give(r->cc.ids);
  if (k == "mapping") return give(r->cc.mapping);
  if (k == "cc_roots") return give(r->cc.roots);
  if (k == "dbf") return give(r->dbf);
  if (k == "daf") return give(r->daf);
  if (k == "pdrf") return give(r->pdrf);
  if (k == "roots") return give(r->roots);
  if (k == "targets") return give(r->targets);
  if (k == "boxes") return give(r->boxes);
  if (k == "orders") return give(r->orders);
  if (k == "order_offsets") return give(r->order_offsets);
  if (k == "paths") return give(r->paths_flat);
  if (k == "path_offsets") return give(r->path_offsets);
  if (k == "path_labels") return give(r->path_labels);
  if (k == "stage_ms") return give(r->stage_ms);
  if (k == "filled") { *count = 1; return &r->filled; }
  if (k == "avocado_passes") { *count = 1; return &r->avocado_passes; }
  *count = -1;
  return nullptr;
}
// Border points of component `id`, flattened (x, y, z) triples in set order.
int64_t oracle_borders(void *h, int64_t id, int64_t *out, int64_t capacity) {
  auto *r = static_cast<Result *>(h);
  if (id < 0 || size_t(id) >= r->borders.size()) return -1;
  const auto &b = r->borders[id];
  for (size_t i = 0; i < b.size() && int64_t(3 * i + 2) < capacity; ++i)
    for (int a = 0; a < 3; ++a) out[3 * i + a] = b[i][a];
  return int64_t(b.size());
}

// Standalone stages, for known-answer tests.
int oracle_edt(const uint32_t *labels, int64_t sx, int64_t sy, int64_t sz, const float aniso[3], int black_border,
               int dims, float *out) {
  try {
    auto d = edt(labels, Shape{sx, sy, sz}, aniso, black_border != 0, dims);
    std::copy(d.begin(), d.end(), out);
    return 0;
  } catch (...) { return 1; }
}
// Railroad on a raw penalty field of one component (all voxels of `labels` equal to 1 belong to it).
int64_t oracle_railroad_graph(const float *field, const uint32_t *labels, const uint32_t *graph, int64_t sx,
                              int64_t sy, int64_t sz, int64_t target, int64_t *out, int64_t capacity);
int64_t oracle_railroad(const float *field, const uint32_t *labels, int64_t sx, int64_t sy, int64_t sz,
                        int64_t target, int64_t *out, int64_t capacity) {
  return oracle_railroad_graph(field, labels, nullptr, sx, sy, sz, target, out, capacity);
}
// The same with a voxel graph (cc3d bits per voxel, or null): relaxations and the join step only
// where the graph permits, the walk back only over permitted steps (lockstep_regular.inc:108, 123;
// lockstep_coop.inc:153-245).
int64_t oracle_railroad_graph(const float *field, const uint32_t *labels, const uint32_t *graph, int64_t sx,
                              int64_t sy, int64_t sz, int64_t target, int64_t *out, int64_t capacity) {
  Volume V; V.s = Shape{sx, sy, sz};
  V.graph = graph;
  std::vector<uint32_t> ids(labels, labels + V.s.n());
  V.ids = &ids;
  V.pdrf.assign(field, field + V.s.n());
  V.dist.assign(V.s.n(), kInf);
  std::vector<i64> touched;
  auto path = railroad(V, 1, target, touched);
  for (size_t i = 0; i < path.size() && int64_t(i) < capacity; ++i) out[i] = path[i];
  return int64_t(path.size());
}
// The railroad's float32 distance field of the same search (+inf where it never reached): the
// SSSP distances the path walks back on, for comparison with a float64 search.
int oracle_railroad_distances(const float *field, const uint32_t *labels, int64_t sx, int64_t sy, int64_t sz,
                              int64_t target, float *dist_out) {
  try {
    Volume V; V.s = Shape{sx, sy, sz};
    std::vector<uint32_t> ids(labels, labels + V.s.n());
    V.ids = &ids;
    V.pdrf.assign(field, field + V.s.n());
    V.dist.assign(V.s.n(), kInf);
    std::vector<i64> touched;
    railroad(V, 1, target, touched, true);
    std::copy(V.dist.begin(), V.dist.end(), dist_out);
    return 0;
  } catch (...) { return 1; }
}
// The CPython set restatement on a script of operations (code, key) pairs: 0 add to A, 1 discard
// from A, 2 add to B, 3 A -= B (B emptied), 4 A |= B (B emptied), 5 A emptied. Writes A's
// iteration order; returns its size.
int64_t oracle_pyset(const int64_t *ops, int64_t n, int64_t *out, int64_t capacity) {
  PySet A, B;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t code = ops[2 * i], key = ops[2 * i + 1];
    if (code == 0) A.add(key);
    else if (code == 1) A.discard(key);
    else if (code == 2) B.add(key);
    else if (code == 3) { A.difference_update(B); B = PySet(); }
    else if (code == 4) { A.update(B); B = PySet(); }
    else A = PySet();
  }
  const auto items = A.items();
  for (size_t i = 0; i < items.size() && int64_t(i) < capacity; ++i) out[i] = items[i];
  return int64_t(items.size());
}
// Target order rule on a flat (mask, daf) pair: descending daf (inf -> 0), ties -> higher index.
int64_t oracle_target_order(const uint8_t *mask, const float *daf, int64_t n, int64_t *out) {
  std::vector<int64_t> order;
  for (int64_t i = 0; i < n; ++i) if (mask[i]) order.push_back(i);
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
    float x = daf[a], y = daf[b];
    if (std::isinf(x) || x == 0) x = 0;
    if (std::isinf(y) || y == 0) y = 0;
    return x == y ? a > b : x > y;
  });
  std::copy(order.begin(), order.end(), out);
  return int64_t(order.size());
}
}
