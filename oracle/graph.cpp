// CPU restatement of the reference's voxel-graph preamble: the components of a voxel connectivity
// graph (brook_graph_components, cpp/src/c_api.cpp:201-207; cpp/src/graph_components.cu:14-154)
// and the graph-aware EDT (brook_graph_edt, cpp/src/c_api.cpp:209-216; cpp/src/graph_edt.cu:9-150).
//
// TEST INFRASTRUCTURE ONLY: the checker for a device implementation of these two calls; the
// product never links it.
//
// The graph is cc3d's: bit b of graph[v] permits the step from voxel v along offset b of kSteps
// (tests/python/test_package.py:1246-1252 of the reference lists the same table). A uint8 graph is
// the compact 2D form: bits 6 and up of the 3D table sit two places lower
// (graph_components.cu:19), and the EDT reads it widened to 32 bits unchanged
// (graph_components.cu:148-164).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <vector>

extern "C" int oracle_edt(const uint32_t *labels, int64_t sx, int64_t sy, int64_t sz, const float aniso[3],
                          int black_border, int dims, float *out);

namespace {

struct Step {
  int dx, dy, dz;
};
// cc3d's bit order (bit b: the step kSteps[b])
constexpr Step kSteps[26] = {{1, 0, 0},   {-1, 0, 0},  {0, 1, 0},   {0, -1, 0},   {0, 0, 1},   {0, 0, -1},
                             {1, 1, 0},   {-1, 1, 0},  {1, -1, 0},  {-1, -1, 0},  {1, 0, 1},   {-1, 0, 1},
                             {0, 1, 1},   {0, -1, 1},  {1, 0, -1},  {-1, 0, -1},  {0, 1, -1},  {0, -1, -1},
                             {1, 1, 1},   {-1, 1, 1},  {1, -1, 1},  {-1, -1, 1},  {1, 1, -1},  {-1, 1, -1},
                             {1, -1, -1}, {-1, -1, -1}};

uint32_t edges_of(const void *graph, bool compact, int64_t v) {
  return compact ? static_cast<const uint8_t *>(graph)[v] : static_cast<const uint32_t *>(graph)[v];
}

int64_t find(std::vector<int64_t> &parent, int64_t a) {
  while (parent[a] != a) {
    parent[a] = parent[parent[a]];
    a = parent[a];
  }
  return a;
}

}  // namespace

extern "C" {

// labels: uint64 per voxel (Fortran order, x fastest); graph: uint32 (graph_u8 = 0) or uint8
// (graph_u8 = 1) per voxel. Writes ids[n] (0 for background voxels) and, for compact ids
// 0..count, mapping[count + 1] (the label at the start of the id's last run of voxels in flat
// order; mapping[0] = 0), roots[count] (the id's lowest voxel) and keys[count + 1] (the id's
// rank among all graph components, background ones included, by lowest voxel; keys[0] = 0).
// The output arrays hold n + 1 entries. Returns count, or -1 on bad arguments.
int64_t oracle_graph_components(const uint64_t *labels, const void *graph, int graph_u8, int64_t sx, int64_t sy,
                                int64_t sz, uint32_t *ids, int64_t *mapping, int64_t *roots, int64_t *keys) {
  if (sx < 0 || sy < 0 || sz < 0) return -1;
  const int64_t n = sx * sy * sz;
  const bool compact = graph_u8 != 0;
  // unions along every permitted step to a lower voxel (graph_components.cu:14-26): the edge is
  // read at its higher end only; roots end up at each component's lowest voxel
  std::vector<int64_t> parent(n);
  std::iota(parent.begin(), parent.end(), 0);
  for (int64_t v = 0; v < n; ++v) {
    const int64_t x = v % sx, y = (v / sx) % sy, z = v / (sx * sy);
    const uint32_t e = edges_of(graph, compact, v);
    for (int b = 0; b < 26; ++b) {
      const int bit = compact && b >= 6 ? b - 2 : b;
      if (bit >= (compact ? 8 : 32) || !((e >> bit) & 1u)) continue;
      const int64_t nx = x + kSteps[b].dx, ny = y + kSteps[b].dy, nz = z + kSteps[b].dz;
      if (nx < 0 || ny < 0 || nz < 0 || nx >= sx || ny >= sy || nz >= sz) continue;
      const int64_t u = nx + sx * (ny + sy * nz);
      if (u >= v) continue;
      const int64_t a = find(parent, v), c = find(parent, u);
      if (a != c) parent[std::max(a, c)] = std::min(a, c);
    }
  }
  // sparse ids: the rank of each component's root among all roots (graph_components.cu:27-42)
  std::vector<int64_t> rank(n, 0);
  int64_t roots_seen = 0;
  for (int64_t v = 0; v < n; ++v)
    if (find(parent, v) == v) rank[v] = ++roots_seen;
  std::vector<int64_t> sparse(n, 0);
  for (int64_t v = 0; v < n; ++v) sparse[v] = labels[v] > 0 ? rank[find(parent, v)] : 0;
  // compact ids: the present sparse ids renumbered 1.. in their order (graph_components.cu:43-55)
  std::vector<int64_t> compact_of(n + 1, 0);
  for (int64_t v = 0; v < n; ++v)
    if (sparse[v]) compact_of[sparse[v]] = 1;
  int64_t count = 0;
  std::vector<int64_t> key_of;
  key_of.push_back(0);
  for (int64_t s = 1; s <= n; ++s)
    if (compact_of[s]) {
      compact_of[s] = ++count;
      key_of.push_back(s);
    }
  for (int64_t v = 0; v < n; ++v) ids[v] = uint32_t(sparse[v] ? compact_of[sparse[v]] : 0);
  // per id: the start of its last run and its lowest voxel (graph_components.cu:56-66, 69-71)
  std::vector<int64_t> last_run(count + 1, -1), lowest(count + 1, INT64_MAX);
  for (int64_t v = 0; v < n; ++v) {
    const int64_t id = ids[v];
    if (!id) continue;
    if (v == 0 || int64_t(ids[v - 1]) != id) last_run[id] = std::max(last_run[id], v);
    lowest[id] = std::min(lowest[id], v);
  }
  for (int64_t c = 0; c <= count; ++c) {
    mapping[c] = c && last_run[c] >= 0 ? int64_t(labels[last_run[c]]) : 0;
    keys[c] = key_of[c];
    if (c) roots[c - 1] = lowest[c];
  }
  return count;
}

// The graph EDT (graph_edt.cu:9-29, 66-150): a binary grid of twice the extent per axis, where
// doubled position (x, y, z) belongs to voxel (x/2, y/2, z/2) and is 0 when that voxel is
// background, at the +x, +y or +z face interface (odd along exactly that one axis) when the
// voxel's graph lacks that step (bits 0, 2, 4), and, with a black border, on the last doubled
// slice of every axis; every other position is 1. Its EDT with half the spacing, sampled at the
// voxels' own (even) positions, is the result (0 for background voxels).
int oracle_graph_edt(const uint64_t *labels, const void *graph, int graph_u8, int64_t sx, int64_t sy, int64_t sz,
                     const float aniso[3], int black_border, float *out) {
  if (sx < 0 || sy < 0 || sz < 0) return 1;
  for (int a = 0; a < 3; ++a)
    if (!(aniso[a] > 0) || !std::isfinite(aniso[a])) return 1;
  const int64_t n = sx * sy * sz;
  if (!n) return 0;
  const bool compact = graph_u8 != 0;
  const int64_t X = 2 * sx, Y = 2 * sy, Z = 2 * sz;
  std::vector<uint32_t> mask(size_t(X * Y * Z));
  for (int64_t z = 0; z < Z; ++z)
    for (int64_t y = 0; y < Y; ++y)
      for (int64_t x = 0; x < X; ++x) {
        uint32_t m = 1;
        if (black_border && (x == X - 1 || y == Y - 1 || z == Z - 1)) {
          m = 0;
        } else {
          const int64_t source = (x >> 1) + sx * ((y >> 1) + sy * (z >> 1));
          if (!(labels[source] > 0)) {
            m = 0;
          } else {
            const uint32_t e = edges_of(graph, compact, source);  // widened unchanged
            const int sub = int((x & 1) | ((y & 1) << 1) | ((z & 1) << 2));
            if (sub == 1) m = (e & 1u) != 0;
            else if (sub == 2) m = (e & 4u) != 0;
            else if (sub == 4) m = (e & 16u) != 0;
          }
        }
        mask[size_t(x + X * (y + Y * z))] = m;
      }
  const float half[3] = {aniso[0] * 0.5f, aniso[1] * 0.5f, aniso[2] * 0.5f};
  std::vector<float> doubled(mask.size());
  if (oracle_edt(mask.data(), X, Y, Z, half, black_border, 3, doubled.data())) return 1;
  for (int64_t z = 0; z < sz; ++z)
    for (int64_t y = 0; y < sy; ++y)
      for (int64_t x = 0; x < sx; ++x) {
        const int64_t i = x + sx * (y + sy * z);
        out[i] = labels[i] > 0 ? doubled[size_t(2 * x + X * (2 * y + Y * 2 * z))] : 0.0f;
      }
  return 0;
}

}  // extern "C"
