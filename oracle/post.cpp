// CPU oracle for the canonical post-processing of packed skeletons of giorgioangel/brook
// (brook_postprocess_canonical, cpp/include/brook/brook.h:238-239; cpp/src/post.cu:646-650 and
// the per-component kernels of cpp/src/post_kernels.cuh, which follow Kimimaro 5.8.1's
// remove_dust, remove_loops, join_close_components and remove_ticks with the reference's tie rules).
//
// TEST INFRASTRUCTURE ONLY: the checker of brook_b200's device post-processing; the product never
// links, loads or calls it. Plain data structures, whole-graph recomputation where the device code
// is incremental; every float operation rounds on its own (-ffp-contract=off), as in the
// reference's --fmad=false build.
//
// A packed set holds K labels; skeleton k owns vertices [voff[k], voff[k+1]) (x, y, z float32) and
// edges [eoff[k], eoff[k+1]) whose endpoints are local to the skeleton. A vertex's global id is
// voff[k] + local. Components are the connected components of the edges, named by their smallest
// global vertex id (the reference's min-index union-find, ccl_kernels.cuh:16-50 and post.cu:36-58).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace {

struct Packed {
  std::vector<int64_t> labels, voff{0}, eoff{0};
  std::vector<float> v, r;  // v: 3 per vertex
  std::vector<uint32_t> e;  // 2 per edge, local
};

struct Graph {
  int n = 0, m = 0, k = 0;
  std::vector<int> vlabel, elabel, root, degree;
  std::vector<std::array<int, 2>> edges;  // global endpoints, orientation as given
};

// post.cu:36-58: global endpoints, degrees (a self loop counts twice), components by smallest id.
Graph graph_of(const Packed &p) {
  Graph g;
  g.k = int(p.labels.size());
  g.n = int(p.voff.back());
  g.m = int(p.eoff.back());
  g.vlabel.resize(g.n);
  g.elabel.resize(g.m);
  g.degree.assign(g.n, 0);
  g.edges.resize(g.m);
  for (int l = 0; l < g.k; ++l) {
    for (int64_t i = p.voff[l]; i < p.voff[l + 1]; ++i) g.vlabel[i] = l;
    const int64_t nv = p.voff[l + 1] - p.voff[l];
    for (int64_t i = p.eoff[l]; i < p.eoff[l + 1]; ++i) {
      const uint32_t a = p.e[2 * i], b = p.e[2 * i + 1];
      if (a >= nv || b >= nv) throw std::invalid_argument("packed edge is out of bounds");
      g.elabel[i] = l;
      g.edges[i] = {int(p.voff[l] + a), int(p.voff[l] + b)};
    }
  }
  std::vector<int> parent(g.n);
  for (int i = 0; i < g.n; ++i) parent[i] = i;
  auto find = [&](int x) {
    while (parent[x] != x) x = parent[x] = parent[parent[x]];
    return x;
  };
  for (auto &e : g.edges) {
    ++g.degree[e[0]];
    ++g.degree[e[1]];
    int a = find(e[0]), b = find(e[1]);
    if (a != b) parent[std::max(a, b)] = std::min(a, b);
  }
  g.root.resize(g.n);
  for (int i = 0; i < g.n; ++i) g.root[i] = find(i);
  return g;
}

// post.cu:72-105 (select): the vertices with keep set, in order; the edges whose two ends are kept,
// in order and orientation, renumbered. Every label stays (possibly empty).
Packed select(const Packed &p, const Graph &g, const std::vector<uint8_t> &keep) {
  Packed out;
  out.labels = p.labels;
  std::vector<int> renum(g.n, -1);
  int next = 0;
  for (int l = 0; l < g.k; ++l) {
    const int base = next;
    for (int64_t i = p.voff[l]; i < p.voff[l + 1]; ++i)
      if (keep[i]) {
        renum[i] = next++ - base;
        for (int a = 0; a < 3; ++a) out.v.push_back(p.v[3 * i + a]);
        out.r.push_back(p.r[i]);
      }
    out.voff.push_back(next);
    for (int64_t i = p.eoff[l]; i < p.eoff[l + 1]; ++i) {
      const auto &e = g.edges[i];
      if (keep[e[0]] && keep[e[1]]) {
        out.e.push_back(uint32_t(renum[e[0]]));
        out.e.push_back(uint32_t(renum[e[1]]));
      }
    }
    out.eoff.push_back(int64_t(out.e.size() / 2));
  }
  return out;
}

// post.cu:293-306 (edge_result): the edges become the sorted distinct (lower, higher) global keys
// (the all-ones key marks an edge to drop); vertices unchanged.
Packed edge_result(const Packed &p, const Graph &g, std::vector<uint64_t> keys) {
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  if (!keys.empty() && keys.back() == ~0ull) keys.pop_back();
  Packed out = p;
  out.e.clear();
  out.eoff.assign(1, 0);
  std::vector<int64_t> count(g.k, 0);
  for (uint64_t key : keys) {
    const int a = int(key >> 32), b = int(uint32_t(key));
    const int l = g.vlabel[a];
    ++count[l];
    out.e.push_back(uint32_t(a - p.voff[l]));
    out.e.push_back(uint32_t(b - p.voff[l]));
  }
  for (int l = 0; l < g.k; ++l) out.eoff.push_back(out.eoff.back() + count[l]);
  return out;
}

uint64_t pair_key(int a, int b) { return (uint64_t(uint32_t(std::min(a, b))) << 32) | uint32_t(std::max(a, b)); }

// post.cu:415-426 (prune_unused): vertices on no edge are dropped when there are any.
Packed prune(const Packed &p) {
  if (p.voff.back() == 0) return p;
  Graph g = graph_of(p);
  bool any = false;
  std::vector<uint8_t> keep(g.n);
  for (int i = 0; i < g.n; ++i) any |= !(keep[i] = g.degree[i] != 0);
  return any ? select(p, g, keep) : p;
}

// NumPy's float32 pairwise summation (blocks of eight lanes below 128 values, halves above; the
// reference cites NumPy 2.4.6, post.cu:129-141).
float pairwise_sum(const float *x, size_t n) {
  if (n < 8) {
    float s = -0.0f;
    for (size_t i = 0; i < n; ++i) s += x[i];
    return s;
  }
  if (n <= 128) {
    float lane[8];
    for (int j = 0; j < 8; ++j) lane[j] = x[j];
    size_t i = 8;
    for (; i < n - n % 8; i += 8)
      for (int j = 0; j < 8; ++j) lane[j] += x[i + j];
    float s = ((lane[0] + lane[1]) + (lane[2] + lane[3])) + ((lane[4] + lane[5]) + (lane[6] + lane[7]));
    for (; i < n; ++i) s += x[i];
    return s;
  }
  size_t half = n / 2;
  half -= half % 8;
  return pairwise_sum(x, half) + pairwise_sum(x + half, n - half);
}

// post.cu:427-468 (remove_dust): a component is kept when its cable length exceeds the threshold.
// The length is the double sum of the edges' lengths (float32 differences, double squares and
// root); within count * 2^-23 * threshold of the threshold the decision is NumPy's float32
// pairwise sum of float32 lengths in edge order instead.
Packed remove_dust(const Packed &p, double threshold) {
  if (threshold == 0 || p.voff.back() == 0) return p;
  Graph g = graph_of(p);
  std::vector<double> total(g.n, 0.0);
  std::vector<int> count(g.n, 0);
  std::vector<std::vector<float>> lengths(g.n);
  for (int i = 0; i < g.m; ++i) {
    const int a = g.edges[i][0], b = g.edges[i][1];
    const double x = double(p.v[3 * b] - p.v[3 * a]), y = double(p.v[3 * b + 1] - p.v[3 * a + 1]),
                 z = double(p.v[3 * b + 2] - p.v[3 * a + 2]);
    const int c = g.root[a];
    total[c] += std::sqrt((x * x + y * y) + z * z);
    ++count[c];
    float fx = p.v[3 * b] - p.v[3 * a], fy = p.v[3 * b + 1] - p.v[3 * a + 1], fz = p.v[3 * b + 2] - p.v[3 * a + 2];
    fx = fx * fx;
    fy = fy * fy;
    fz = fz * fz;
    lengths[c].push_back(std::sqrt((fx + fy) + fz));
  }
  std::vector<uint8_t> keep_root(g.n), keep(g.n);
  for (int c = 0; c < g.n; ++c) {
    const bool near = count[c] > 0 && std::fabs(total[c] - threshold) <= count[c] * (1.0 / 8388608.0) * threshold;
    keep_root[c] = near ? double(pairwise_sum(lengths[c].data(), lengths[c].size())) > threshold
                        : total[c] > threshold;
  }
  for (int i = 0; i < g.n; ++i) keep[i] = keep_root[g.root[i]];
  return select(p, g, keep);
}

// ---- remove_loops (post.cu:469-489; the per-component rules of post_kernels.cuh:23-192) ----
//
// One component with a cycle, vertices numbered 0..nv-1 in ascending global order, its edges as
// rows in edge order. Each round: a depth-first search from the first live row's first vertex
// (neighbours pushed in their adjacency order, popped last first, the parent node skipped) stops
// at the first node it reaches twice; the path from that node's first place is the cycle. Branch
// nodes are the cycle's nodes with three or more row ends. 0 branches: the cycle's edges go.
// 1: they go and an edge joins the branch node to the cycle node farthest from it (float32
// squared distance, ties to the lower node). 2: the edges off the side with fewer path positions
// go. 3+: the node of the whole component nearest the branch nodes' float32 centroid (first
// minimum) either replaces the cycle, joined to every branch node, or, when the farthest branch
// node is beyond its radius, only the cycle's first edge goes. Removing an edge removes all its
// duplicate rows. A self loop (a cycle of one node) or no cycle ends the rounds.
struct LoopComponent {
  struct Adj {
    int to, row, mult;
  };
  const float *P, *R;
  int nv;
  std::vector<std::array<int, 2>> rows;
  std::vector<uint8_t> live;
  std::vector<std::vector<Adj>> adj;  // distinct neighbours in insertion order
  std::vector<int> cnt;
  int nlive = 0, first = 0;

  Adj *find(int a, int b) {
    for (auto &x : adj[a])
      if (x.to == b) return &x;
    return nullptr;
  }
  void add_row(int x, int y) {
    const int r = int(rows.size());
    rows.push_back({x, y});
    live.push_back(1);
    ++nlive;
    ++cnt[x];
    ++cnt[y];
    if (Adj *f = find(x, y)) {
      ++f->mult;
      ++find(y, x)->mult;  // the same entry again for a self loop, as the reference counts it
    } else {
      adj[x].push_back({y, r, 1});
      adj[y].push_back({x, r, 1});
    }
  }
  void unlink(int a, int b) {
    auto &l = adj[a];
    for (size_t i = 0; i < l.size(); ++i)
      if (l[i].to == b) {
        l.erase(l.begin() + i);
        return;
      }
  }
  float sq(int a, int b) const {
    const float dx = P[3 * a] - P[3 * b], dy = P[3 * a + 1] - P[3 * b + 1], dz = P[3 * a + 2] - P[3 * b + 2];
    return (dx * dx + dy * dy) + dz * dz;
  }

  void run() {
    cnt.assign(nv, 0);
    adj.assign(nv, {});
    std::vector<std::array<int, 2>> initial;
    initial.swap(rows);
    for (auto &r : initial) add_row(r[0], r[1]);
    int app0 = int(rows.size()), app1 = app0;
    std::vector<uint8_t> visited(nv), drop(nv);
    for (;;) {
      if (nlive == 0) break;
      while (!live[first]) ++first;
      // the depth-first search
      struct Item {
        int node, parent, depth;
      };
      std::vector<Item> stack{{rows[first][0], -1, 0}};
      std::vector<int> path;
      std::fill(visited.begin(), visited.end(), 0);
      int node = -1;
      bool found = false;
      while (!stack.empty()) {
        const Item it = stack.back();
        stack.pop_back();
        node = it.node;
        if (int(path.size()) > it.depth) path.resize(it.depth);
        path.push_back(node);
        if (visited[node]) {
          found = true;
          break;
        }
        visited[node] = 1;
        for (const Adj &x : adj[node])
          if (x.to != it.parent) stack.push_back({x.to, node, it.depth + 1});
      }
      const int plen = int(path.size());
      if (!found || plen <= 1) break;
      int i0 = 0;
      while (i0 < plen - 1 && path[i0] != node) ++i0;
      if (plen - i0 < 3) break;
      const std::vector<int> cy(path.begin() + i0, path.end());  // cy.front() == cy.back()
      const int cl = int(cy.size());
      std::vector<int> branch;
      for (int j = 0; j + 1 < cl; ++j)
        if (cnt[cy[j]] >= 3) branch.push_back(cy[j]);
      std::sort(branch.begin(), branch.end());
      const int nb = int(branch.size());
      std::fill(drop.begin(), drop.end(), 0);  // drop[cy[j]]: cycle edge j (cy[j], cy[j+1]) goes
      std::vector<std::array<int, 2>> added;
      if (nb == 0) {
        for (int j = 0; j + 1 < cl; ++j) drop[cy[j]] = 1;
      } else if (nb == 1) {
        const int b = branch[0];
        int end = -1;
        float best = -1.0f;
        for (int j = 0; j + 1 < cl; ++j) {
          const int v = cy[j];
          const float d = sq(v, b);
          if (end < 0 || d > best || (d == best && v < end)) {
            best = d;
            end = v;
          }
        }
        for (int j = 0; j + 1 < cl; ++j) drop[cy[j]] = 1;
        added.push_back({b, end});
      } else if (nb == 2) {
        // the path is cy[1..cl-1]; p0 < p1 its two branch positions
        const int L = cl - 1;
        int p0 = -1, p1 = -1;
        for (int j = 0; j < L; ++j)
          if (cnt[cy[j + 1]] >= 3) (p0 < 0 ? p0 : p1) = j;
        const bool inner = double(p1 - p0) < double(L) / 2.0;
        for (int j = 0; j + 1 < cl; ++j) {
          const bool on_inner = j - 1 >= 0 && j - 1 >= p0 && j <= p1;
          if (inner != on_inner) drop[cy[j]] = 1;
        }
      } else {
        float cx = 0.0f, cyy = 0.0f, cz = 0.0f;
        for (int v : branch) {
          cx += P[3 * v];
          cyy += P[3 * v + 1];
          cz += P[3 * v + 2];
        }
        cx /= float(nb);
        cyy /= float(nb);
        cz /= float(nb);
        int inter = -1;
        float best = 0.0f;
        for (int v = 0; v < nv; ++v) {
          const float dx = P[3 * v] - cx, dy = P[3 * v + 1] - cyy, dz = P[3 * v + 2] - cz;
          const float d = (dx * dx + dy * dy) + dz * dz;
          if (inter < 0 || d < best) {
            best = d;
            inter = v;
          }
        }
        float far = 0.0f;
        for (int i = 0; i < nb; ++i) {
          const float d = sq(branch[i], inter);
          if (i == 0 || d > far) far = d;
        }
        if (std::sqrt(far) > R[inter]) {
          drop[cy[0]] = 1;
        } else {
          for (int j = 0; j + 1 < cl; ++j) drop[cy[j]] = 1;
          for (int v : branch)
            if (v != inter) added.push_back({v, inter});
        }
      }
      // the rows added last round become (lower, higher); the dropped edges go with their duplicates
      for (int r = app0; r < app1; ++r)
        if (live[r] && rows[r][0] > rows[r][1]) std::swap(rows[r][0], rows[r][1]);
      for (int j = 0; j + 1 < cl; ++j) {
        const int a = cy[j], b = cy[j + 1];
        if (!drop[a]) continue;
        Adj *e = find(a, b);
        if (!e) continue;
        const int m = e->mult;
        if (m == 1) {
          live[e->row] = 0;
        } else {
          const int lo = std::min(a, b), hi = std::max(a, b);
          for (int r = first; r < int(rows.size()); ++r)
            if (live[r] && rows[r][0] == lo && rows[r][1] == hi) live[r] = 0;
        }
        nlive -= m;
        cnt[a] -= m;
        cnt[b] -= m;
        unlink(a, b);
        unlink(b, a);
      }
      app0 = int(rows.size());
      for (auto &x : added) add_row(x[0], x[1]);
      app1 = int(rows.size());
    }
  }
};

Packed remove_loops(const Packed &p) {
  if (p.voff.back() == 0 || p.eoff.back() == 0) return p;
  Graph g = graph_of(p);
  std::vector<int> nv(g.n, 0), ne(g.n, 0);
  for (int i = 0; i < g.n; ++i) ++nv[g.root[i]];
  for (auto &e : g.edges) ++ne[g.root[e[0]]];
  std::vector<int> work;
  for (int c = 0; c < g.n; ++c)
    if (ne[c] > 0 && ne[c] - nv[c] + 1 > 0) work.push_back(c);
  if (work.empty()) return p;
  std::vector<int> slot(g.n, -1);
  for (size_t s = 0; s < work.size(); ++s) slot[work[s]] = int(s);
  std::vector<std::vector<int>> verts(work.size()), erows(work.size());
  std::vector<int> local(g.n, -1);
  for (int i = 0; i < g.n; ++i)
    if (slot[g.root[i]] >= 0) {
      auto &vs = verts[slot[g.root[i]]];
      local[i] = int(vs.size());
      vs.push_back(i);
    }
  std::vector<uint64_t> keys;
  for (int i = 0; i < g.m; ++i) {
    const auto &e = g.edges[i];
    const int s = slot[g.root[e[0]]];
    if (s >= 0) erows[s].push_back(i);
    else keys.push_back(e[0] != e[1] ? pair_key(e[0], e[1]) : ~0ull);
  }
  std::vector<uint8_t> emptied(work.size(), 0);
  for (size_t s = 0; s < work.size(); ++s) {
    const auto &vs = verts[s];
    std::vector<float> P, R;
    for (int v : vs) {
      for (int a = 0; a < 3; ++a) P.push_back(p.v[3 * v + a]);
      R.push_back(p.r[v]);
    }
    LoopComponent lc;
    lc.P = P.data();
    lc.R = R.data();
    lc.nv = int(vs.size());
    for (int i : erows[s]) lc.rows.push_back({local[g.edges[i][0]], local[g.edges[i][1]]});
    lc.run();
    int kept = 0;
    for (size_t r = 0; r < lc.rows.size(); ++r)
      if (lc.live[r]) {
        ++kept;
        const int a = vs[lc.rows[r][0]], b = vs[lc.rows[r][1]];
        if (a != b) keys.push_back(pair_key(a, b));
      }
    emptied[s] = kept == 0;
  }
  Packed out = edge_result(p, g, keys);
  if (std::find(emptied.begin(), emptied.end(), 1) != emptied.end()) {
    Graph h = graph_of(out);
    std::vector<uint8_t> keep(g.n);
    for (int i = 0; i < g.n; ++i) keep[i] = slot[g.root[i]] < 0 || !emptied[slot[g.root[i]]];
    return select(out, h, keep);
  }
  return out;
}

// ---- join_close_components (post.cu:589-645; join_scan and join_fuse, post_kernels.cuh:204-311) ----
//
// Within each label with more than one component: reach = 2 x the label's largest positive radius
// (0 without one). Candidate pairs join two vertices of different components closer than reach +
// 1e-6 (double distance of float32 coordinates); per pair of components the nearest candidate,
// ties to the lower (lower vertex, higher vertex). Then, greedily, the nearest pair in float32 (ties
// to the lower pair of list positions, where the newest fused cluster heads the list) is joined if
// no farther than reach; pairs longer than the float32 sum of their two vertices' radii never join.
// After a fusion the fused cluster keeps, towards every other cluster, the nearer of its two pairs.
Packed join_components(const Packed &input) {
  Packed p = prune(input);
  if (p.voff.back() == 0 || p.eoff.back() == 0) return p;
  Graph g = graph_of(p);
  struct Label {
    int l;
    double reach, bound;
    std::vector<int> roots, verts;
  };
  std::vector<Label> multi;
  {
    std::vector<int> ncomp(g.k, 0);
    std::vector<float> rmax(g.k, 0.0f);
    for (int i = 0; i < g.n; ++i) {
      if (g.root[i] == i) ++ncomp[g.vlabel[i]];
      if (p.r[i] > 0 && p.r[i] > rmax[g.vlabel[i]]) rmax[g.vlabel[i]] = p.r[i];
    }
    for (int l = 0; l < g.k; ++l)
      if (ncomp[l] > 1) {
        const double reach = std::max(2.0 * double(rmax[l]), 0.0);
        Label L{l, reach, reach + 0.000001, {}, {}};
        for (int64_t i = p.voff[l]; i < p.voff[l + 1]; ++i) {
          L.verts.push_back(int(i));
          if (g.root[i] == i) L.roots.push_back(int(i));
        }
        multi.push_back(std::move(L));
      }
  }
  if (multi.empty()) return p;
  std::vector<std::array<int, 2>> made;
  for (const Label &L : multi) {
    // the nearest candidate per pair of components (a < b by component id)
    struct Cand {
      double d;
      int lo, hi, va, vb;
    };
    std::map<std::pair<int, int>, Cand> best;
    const float b32 = float(L.bound);
    const float limit = b32 * b32 * 1.0001f + 1e-30f;
    for (int i : L.verts)
      for (int j : L.verts) {
        if (g.root[j] <= g.root[i]) continue;
        const float fx = p.v[3 * j] - p.v[3 * i], fy = p.v[3 * j + 1] - p.v[3 * i + 1], fz = p.v[3 * j + 2] - p.v[3 * i + 2];
        if ((fx * fx + fy * fy) + fz * fz > limit) continue;
        const double ex = double(p.v[3 * j]) - double(p.v[3 * i]), ey = double(p.v[3 * j + 1]) - double(p.v[3 * i + 1]),
                     ez = double(p.v[3 * j + 2]) - double(p.v[3 * i + 2]);
        const double d = std::sqrt((ex * ex + ey * ey) + ez * ez);
        if (!(d < L.bound)) continue;
        Cand c{d, std::min(i, j), std::max(i, j), i, j};
        auto key = std::make_pair(g.root[i], g.root[j]);
        auto it = best.find(key);
        if (it == best.end()) best.emplace(key, c);
        else {
          const Cand &o = it->second;
          if (c.d < o.d || (c.d == o.d && (c.lo < o.lo || (c.lo == o.lo && c.hi < o.hi)))) it->second = c;
        }
      }
    // greedy fusion over the list (pairs in (a, b) order)
    std::map<int, int> index;  // component id -> local index (ascending ids)
    for (size_t c = 0; c < L.roots.size(); ++c) index[L.roots[c]] = int(c);
    struct Pair {
      int cx, cy;
      double d;
      int va, vb;
      bool alive;
    };
    std::vector<Pair> pairs;
    for (auto &kv : best)
      pairs.push_back({index[kv.first.first], index[kv.first.second], kv.second.d, kv.second.va, kv.second.vb, true});
    std::vector<int> pos(L.roots.size());
    for (size_t c = 0; c < pos.size(); ++c) pos[c] = int(c);
    int fusions = 0;
    for (;;) {
      int best_p = -1, bi = 0, bj = 0;
      float bd = 0.0f;
      for (size_t q = 0; q < pairs.size(); ++q) {
        const Pair &x = pairs[q];
        if (!x.alive) continue;
        if (x.d > double(float(p.r[x.va] + p.r[x.vb]))) continue;
        const float d32 = float(x.d);
        int ia = pos[x.cx], ib = pos[x.cy];
        if (ia > ib) std::swap(ia, ib);
        if (best_p < 0 || d32 < bd || (d32 == bd && (ia < bi || (ia == bi && ib < bj)))) {
          best_p = int(q);
          bd = d32;
          bi = ia;
          bj = ib;
        }
      }
      if (best_p < 0 || double(bd) > L.reach) break;
      const int X = pairs[best_p].cx, Y = pairs[best_p].cy;
      made.push_back({pairs[best_p].va, pairs[best_p].vb});
      pairs[best_p].alive = false;
      ++fusions;
      std::map<int, int> toward;  // other cluster -> its surviving pair
      for (size_t q = 0; q < pairs.size(); ++q) {
        Pair &x = pairs[q];
        if (!x.alive) continue;
        if (x.cx == Y) x.cx = X;
        if (x.cy == Y) x.cy = X;
        if (x.cx == x.cy) {
          x.alive = false;
          continue;
        }
        if (x.cx != X && x.cy != X) continue;
        const int other = x.cx == X ? x.cy : x.cx;
        auto it = toward.find(other);
        if (it == toward.end()) {
          toward[other] = int(q);
          continue;
        }
        Pair &y = pairs[it->second];
        const int xl = std::min(x.va, x.vb), xh = std::max(x.va, x.vb), yl = std::min(y.va, y.vb), yh = std::max(y.va, y.vb);
        const bool x_wins = x.d < y.d || (x.d == y.d && (xl < yl || (xl == yl && xh < yh)));
        if (x_wins) {
          y.alive = false;
          it->second = int(q);
        } else {
          x.alive = false;
        }
      }
      pos[X] = -fusions;
    }
  }
  if (made.empty()) return p;
  std::vector<uint64_t> keys;
  for (auto &e : g.edges) keys.push_back(pair_key(e[0], e[1]));
  for (auto &e : made) keys.push_back(pair_key(e[0], e[1]));
  return edge_result(p, g, keys);
}

// ---- remove_ticks (post.cu:490-519; remove_ticks_k, post_kernels.cuh:314-405) ----
//
// Components that are trees with a branch node. Critical nodes (one or three-plus neighbours)
// split the tree into chains; a chain's length is the float32 sum, from the end nearer the first
// leaf (lowest local id), of its edges' float32 lengths. Chains touching a leaf are eligible.
// Repeatedly the eligible chain with the least (length, lower end, higher end) goes, unless both
// its ends have one chain left or it is at least the threshold; a branch node left with two
// chains fuses them into one eligible chain of the double sum of their lengths.
Packed remove_ticks(const Packed &p, double threshold) {
  if (threshold == 0 || p.voff.back() == 0 || p.eoff.back() == 0) return p;
  Graph g = graph_of(p);
  std::vector<int> nv(g.n, 0), ne(g.n, 0), branch(g.n, 0);
  for (int i = 0; i < g.n; ++i) {
    ++nv[g.root[i]];
    if (g.degree[i] >= 3) branch[g.root[i]] = 1;
  }
  for (auto &e : g.edges) ++ne[g.root[e[0]]];
  std::vector<uint8_t> live(g.m, 1);
  std::vector<std::vector<int>> verts(g.n), erows(g.n);
  for (int i = 0; i < g.n; ++i) verts[g.root[i]].push_back(i);
  for (int i = 0; i < g.m; ++i) erows[g.root[g.edges[i][0]]].push_back(i);
  for (int c = 0; c < g.n; ++c) {
    if (!(branch[c] && ne[c] == nv[c] - 1)) continue;
    const auto &vs = verts[c];
    const int n = int(vs.size());
    std::map<int, int> local;
    for (int i = 0; i < n; ++i) local[vs[i]] = i;
    std::vector<std::vector<std::pair<int, int>>> nbr(n);  // (neighbour, row)
    for (int r : erows[c]) {
      const int a = local[g.edges[r][0]], b = local[g.edges[r][1]];
      nbr[a].push_back({b, r});
      nbr[b].push_back({a, r});
    }
    auto deg = [&](int v) { return int(nbr[v].size()); };
    int start = -1;
    for (int v = 0; v < n && start < 0; ++v)
      if (deg(v) == 1) start = v;
    if (start < 0) continue;
    struct Chain {
      int u, v;
      double len;
      bool alive, eligible;
      std::vector<int> rows;
    };
    std::vector<Chain> chains;
    // walk the tree from the start leaf; a chain starts at every critical node
    struct Item {
      int node, parent, root, chain;
      float dist;
    };
    std::vector<Item> stack{{start, -1, start, -1, 0.0f}};
    while (!stack.empty()) {
      Item it = stack.back();
      stack.pop_back();
      const int d = deg(it.node);
      if ((d == 1 || d >= 3) && it.node != it.root) {
        Chain &ch = chains[it.chain];
        ch.u = it.root;
        ch.v = it.node;
        ch.len = double(it.dist);
        ch.alive = true;
        ch.eligible = deg(it.root) == 1 || d == 1;
        it.dist = 0.0f;
        it.root = it.node;
      }
      for (auto [child, row] : nbr[it.node]) {
        if (child == it.parent) continue;
        const float *a = &p.v[3 * vs[it.node]], *b = &p.v[3 * vs[child]];
        float dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
        dx *= dx;
        dy *= dy;
        dz *= dz;
        int ch = it.chain;
        if (it.node == it.root) {
          ch = int(chains.size());
          chains.push_back({-1, -1, 0.0, false, false, {}});
        }
        chains[ch].rows.push_back(row);
        stack.push_back({child, it.node, it.root, ch, it.dist + std::sqrt((dx + dy) + dz)});
      }
    }
    std::vector<int> bc(n);
    for (int v = 0; v < n; ++v) bc[v] = deg(v) >= 3 ? deg(v) : 0;
    int nalive = 0;
    for (auto &ch : chains) nalive += ch.alive;
    while (nalive > 1) {
      int best = -1;
      for (size_t s = 0; s < chains.size(); ++s) {
        const Chain &x = chains[s];
        if (!x.alive || !x.eligible) continue;
        if (best < 0) {
          best = int(s);
          continue;
        }
        const Chain &y = chains[best];
        const int xl = std::min(x.u, x.v), xh = std::max(x.u, x.v), yl = std::min(y.u, y.v), yh = std::max(y.u, y.v);
        if (x.len < y.len || (x.len == y.len && (xl < yl || (xl == yl && xh < yh)))) best = int(s);
      }
      if (best < 0) break;
      Chain &b = chains[best];
      const int e1 = b.u, e2 = b.v;
      if (bc[e1] == 1 && bc[e2] == 1) break;
      if (b.len >= threshold) break;
      for (int r : b.rows) live[r] = 0;
      b.alive = false;
      --nalive;
      --bc[e1];
      --bc[e2];
      for (int v : {e1, e2}) {
        if (bc[v] != 2) continue;
        int x = -1, y = -1;
        for (size_t s = 0; s < chains.size(); ++s)
          if (chains[s].alive && (chains[s].u == v || chains[s].v == v)) (x < 0 ? x : y) = int(s);
        if (x < 0 || y < 0) {
          bc[v] = 0;
          continue;
        }
        Chain &A = chains[x], &B = chains[y];
        const int ea = A.u == v ? A.v : A.u, eb = B.u == v ? B.v : B.u;
        A.len = (0.0 + A.len) + B.len;
        A.u = ea;
        A.v = eb;
        A.alive = A.eligible = true;
        A.rows.insert(A.rows.end(), B.rows.begin(), B.rows.end());
        B.alive = false;
        --nalive;
        bc[v] = 0;
      }
    }
  }
  // select_edge_rows (post.cu:381-396): the surviving edges in order; vertices unchanged
  Packed out = p;
  out.e.clear();
  out.eoff.assign(1, 0);
  for (int l = 0; l < g.k; ++l) {
    for (int64_t i = p.eoff[l]; i < p.eoff[l + 1]; ++i)
      if (live[i]) {
        out.e.push_back(p.e[2 * i]);
        out.e.push_back(p.e[2 * i + 1]);
      }
    out.eoff.push_back(int64_t(out.e.size() / 2));
  }
  return out;
}

struct PostResult {
  Packed p;
  std::vector<int64_t> components;
  std::string error;
};

}  // namespace

extern "C" {

// op: 0 postprocess(a = dust, b = ticks) (post.cu:646-650), 1 remove_dust(a), 2 remove_loops,
// 3 join_components, 4 remove_ticks(a), 5 prune_unused, 6 components (the component id of every
// vertex, post.cu:407-411).
void *oracle_post(const int64_t *labels, int64_t k, const int64_t *voff, const int64_t *eoff, const float *vertices,
                  const uint32_t *edges, const float *radii, int op, double a, double b) {
  auto *res = new PostResult();
  try {
    Packed p;
    p.labels.assign(labels, labels + k);
    p.voff.assign(voff, voff + k + 1);
    p.eoff.assign(eoff, eoff + k + 1);
    const int64_t n = p.voff.back(), m = p.eoff.back();
    p.v.assign(vertices, vertices + 3 * n);
    p.r.assign(radii, radii + n);
    p.e.assign(edges, edges + 2 * m);
    switch (op) {
      case 0: {
        Packed q = remove_dust(p, a);
        q = remove_loops(q);
        q = join_components(q);
        q = remove_ticks(q, b);
        res->p = prune(q);
        break;
      }
      case 1: res->p = remove_dust(p, a); break;
      case 2: res->p = remove_loops(p); break;
      case 3: res->p = join_components(p); break;
      case 4: res->p = remove_ticks(p, a); break;
      case 5: res->p = prune(p); break;
      case 6: {
        Graph g = graph_of(p);
        res->components.assign(g.root.begin(), g.root.end());
        res->p = p;
        break;
      }
      default: throw std::invalid_argument("unknown post-processing step");
    }
  } catch (const std::exception &e) {
    res->error = e.what();
  }
  return res;
}

const char *oracle_post_error(void *h) {
  auto *r = static_cast<PostResult *>(h);
  return r->error.empty() ? nullptr : r->error.c_str();
}

// sizes[0..3] = labels, vertices, edges, components
void oracle_post_sizes(void *h, int64_t *sizes) {
  auto *r = static_cast<PostResult *>(h);
  sizes[0] = int64_t(r->p.labels.size());
  sizes[1] = r->p.voff.back();
  sizes[2] = r->p.eoff.back();
  sizes[3] = int64_t(r->components.size());
}

void oracle_post_copy(void *h, int64_t *labels, int64_t *voff, int64_t *eoff, float *vertices, uint32_t *edges,
                      float *radii, int64_t *components) {
  auto *r = static_cast<PostResult *>(h);
  const Packed &p = r->p;
  std::copy(p.labels.begin(), p.labels.end(), labels);
  std::copy(p.voff.begin(), p.voff.end(), voff);
  std::copy(p.eoff.begin(), p.eoff.end(), eoff);
  std::copy(p.v.begin(), p.v.end(), vertices);
  std::copy(p.e.begin(), p.e.end(), edges);
  std::copy(p.r.begin(), p.r.end(), radii);
  std::copy(r->components.begin(), r->components.end(), components);
}

void oracle_post_free(void *h) { delete static_cast<PostResult *>(h); }

}  // extern "C"
