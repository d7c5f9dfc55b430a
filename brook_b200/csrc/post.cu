// Canonical post-processing of packed skeletons on the device: the reference's
// brook_postprocess_canonical (cpp/include/brook/brook.h:238-239; cpp/src/post.cu:646-650 of
// giorgioangel/brook, whose per-component rules follow Kimimaro 5.8.1's remove_dust, remove_loops,
// join_close_components and remove_ticks with the reference's tie rules,
// cpp/src/post_kernels.cuh).
//
// Layout: a packed set stays in three flat device arrays (vertices x, y, z float32; edges as local
// uint32 pairs; radii) with its per-label offsets on the host. Every step first builds the global
// graph in one pass over the edges (global endpoints, degrees, a lock-free union-find whose roots
// are the smallest vertex id of each component), then:
//   * remove_dust: per-component cable length by double atomics; components within
//     count * 2^-23 * threshold of the threshold are decided by NumPy's float32 pairwise sum of
//     their edges in edge order, one thread per such component over the edges sorted by component;
//   * remove_loops / remove_ticks: the components that need work (a cycle / a branched tree) are
//     gathered into contiguous arenas (radix sort by component) and one thread walks each
//     component sequentially, with per-component workspaces sized on the host. The loop walker
//     keeps the graph's 2-core by peeling leaves incrementally, so a round's depth-first search
//     visits the cyclic part only; the tick walker keeps the shortest eligible chain in a binary
//     heap with versioned entries;
//   * join_components: vertices of labels with several components sorted into grid cells of
//     the label's reach (four stable radix passes), one thread per vertex scans the 27 cells
//     around it, the candidates sorted by (components, distance, vertices) in three 64-bit radix
//     passes keep the nearest per pair of components, and one thread per label runs the greedy
//     fusion;
//   * edge results: (lower, higher) global keys radix-sorted and made unique.
// Each step reads back only per-label or per-component counts to size its outputs.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "post.hpp"

namespace bk {
namespace {

using u64 = unsigned long long;

// ---------------------------------------------------------------- a packed set on the device ----

struct Set {
  std::vector<int64_t> labels, voff{0}, eoff{0};
  std::array<float, 3> anisotropy{1, 1, 1};
  std::shared_ptr<Buffer<float>> vbuf, rbuf;  // owners when this file made the arrays
  std::shared_ptr<Buffer<uint32_t>> ebuf;
  const float *v = nullptr, *r = nullptr;
  const uint32_t *e = nullptr;
  int n() const { return int(voff.back()); }
  int m() const { return int(eoff.back()); }
  int k() const { return int(labels.size()); }
};

// A CUB call with scratch sized by its own query.
struct Cub {
  Context &ctx;
  Buffer<unsigned char> tmp;
  template <class Op>
  void operator()(Op op) {
    size_t bytes = 0;
    BK_CUDA(op(nullptr, bytes));
    bytes = std::max<size_t>(bytes, 16);
    if (bytes > tmp.size()) tmp = Buffer<unsigned char>(ctx, bytes);
    BK_CUDA(op(tmp.data(), bytes));
  }
};

Set set_of(Context &ctx, const Packed &p) {
  Set s;
  s.labels = p.labels;
  s.voff = p.vertex_offsets;
  s.eoff = p.edge_offsets;
  s.anisotropy = p.anisotropy;
  const size_t k = s.labels.size();
  if (s.voff.size() != k + 1 || s.eoff.size() != k + 1 || s.voff[0] != 0 || s.eoff[0] != 0 ||
      !std::is_sorted(s.voff.begin(), s.voff.end()) || !std::is_sorted(s.eoff.begin(), s.eoff.end()))
    throw std::invalid_argument("invalid packed graph");
  if (s.voff.back() >= INT32_MAX || s.eoff.back() >= INT32_MAX / 2 || k >= size_t(INT32_MAX))
    throw std::invalid_argument("packed graph exceeds int32 work capacity");
  if (p.on_device()) {
    s.v = static_cast<const float *>(p.device_vertices->ptr);
    s.r = static_cast<const float *>(p.device_radii->ptr);
    s.e = static_cast<const uint32_t *>(p.device_edges->ptr);
  } else {
    if (p.vertices.size() != size_t(3 * s.voff.back()) || p.radii.size() != size_t(s.voff.back()) ||
        p.edges.size() != size_t(2 * s.eoff.back()))
      throw std::invalid_argument("invalid packed graph");
    s.vbuf = std::make_shared<Buffer<float>>(to_device(ctx, p.vertices));
    s.rbuf = std::make_shared<Buffer<float>>(to_device(ctx, p.radii));
    s.ebuf = std::make_shared<Buffer<uint32_t>>(to_device(ctx, p.edges));
    s.v = s.vbuf->data();
    s.r = s.rbuf->data();
    s.e = s.ebuf->data();
  }
  return s;
}

// ------------------------------------------------------------------------------- the graph ----

struct Graph {
  int n = 0, m = 0, k = 0;
  Buffer<long long> voff, eoff;
  Buffer<int> vlabel, root, degree;
  Buffer<int2> edges;  // global endpoints, orientation as given
};

// The label owning flat index i: the largest l with off[l] <= i.
__device__ __forceinline__ int owner(const long long *off, int k, long long i) {
  int lo = 0, hi = k;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= i) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void graph_vertices(const long long *voff, int k, int n, int *vlabel, int *parent, int *degree) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  vlabel[i] = owner(voff, k, i);
  parent[i] = i;
  degree[i] = 0;
}

// Root of x with path halving; every pointer goes to a smaller id, so a racing halving write stores
// an ancestor either way.
__device__ __forceinline__ int find_root(int *parent, int x) {
  for (;;) {
    const int p = parent[x];
    if (p == x) return x;
    const int g = parent[p];
    if (g != p) parent[x] = g;
    x = g;
  }
}

// Links the larger root under the smaller until the two agree.
__device__ __forceinline__ void unite(int *parent, int a, int b) {
  for (;;) {
    a = find_root(parent, a);
    b = find_root(parent, b);
    if (a == b) return;
    if (a < b) { const int t = a; a = b; b = t; }
    if (atomicCAS(parent + a, a, b) == a) return;
  }
}

__global__ void graph_edges(const uint32_t *e, const long long *voff, const long long *eoff, int k, int m,
                            int2 *edges, int *degree, int *parent, int *error) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int l = owner(eoff, k, i);
  const unsigned a = e[2LL * i], b = e[2LL * i + 1];
  const long long nv = voff[l + 1] - voff[l];
  if (a >= nv || b >= nv) {
    atomicExch(error, 1);
    edges[i] = make_int2(0, 0);
    return;
  }
  const int ga = int(voff[l] + a), gb = int(voff[l] + b);
  edges[i] = make_int2(ga, gb);
  atomicAdd(degree + ga, 1);
  atomicAdd(degree + gb, 1);
  unite(parent, ga, gb);
}

// Read-only walk to the root, one write of the vertex's own entry.
__global__ void flatten(int *parent, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int x = parent[i];
  for (int p; (p = parent[x]) != x;) x = p;
  parent[i] = x;
}

Graph graph_of(Context &ctx, const Set &s) {
  cudaStream_t st = ctx.stream();
  Graph g;
  g.n = s.n();
  g.m = s.m();
  g.k = s.k();
  std::vector<long long> vo(s.voff.begin(), s.voff.end()), eo(s.eoff.begin(), s.eoff.end());
  g.voff = to_device(ctx, vo);
  g.eoff = to_device(ctx, eo);
  g.vlabel = Buffer<int>(ctx, g.n);
  g.root = Buffer<int>(ctx, g.n);
  g.degree = Buffer<int>(ctx, g.n);
  g.edges = Buffer<int2>(ctx, g.m);
  if (g.n) {
    graph_vertices<<<blocks_for(g.n), 256, 0, st>>>(g.voff.data(), g.k, g.n, g.vlabel.data(), g.root.data(),
                                                     g.degree.data());
    ++ctx.launches;
  }
  if (g.m) {
    Buffer<int> error(ctx, 1);
    error.zero();
    graph_edges<<<blocks_for(g.m), 256, 0, st>>>(s.e, g.voff.data(), g.eoff.data(), g.k, g.m, g.edges.data(),
                                                  g.degree.data(), g.root.data(), error.data());
    ++ctx.launches;
    if (g.n) {
      flatten<<<blocks_for(g.n), 256, 0, st>>>(g.root.data(), g.n);
      ++ctx.launches;
    }
    BK_CUDA(cudaGetLastError());
    if (error.download(1)[0]) throw std::invalid_argument("packed edge is out of bounds");
  }
  BK_CUDA(cudaGetLastError());
  return g;
}

// ------------------------------------------------------------------ selections and results ----

// new_off[l] = number of kept items before off[l] (rank is an inclusive scan of the kept flags)
__global__ void offsets_from_rank(const long long *off, int k, const int *rank, long long *out) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l > k) return;
  out[l] = off[l] == 0 ? 0 : rank[off[l] - 1];
}

struct KeepVertex {
  const unsigned char *keep;
  __device__ int operator()(int i) const { return keep[i] != 0; }
};
struct KeepEdge {
  const unsigned char *keep;
  const int2 *edges;
  __device__ int operator()(int i) const {
    const int2 e = edges[i];
    return keep[e.x] && keep[e.y];
  }
};
struct KeepFlag {
  const unsigned char *keep;
  __device__ int operator()(int i) const { return keep[i] != 0; }
};

__global__ void write_kept_vertices(const float *v, const float *r, const unsigned char *keep, const int *rank, int n,
                                    float *ov, float *orad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !keep[i]) return;
  const int j = rank[i] - 1;
  for (int a = 0; a < 3; ++a) ov[3LL * j + a] = v[3LL * i + a];
  orad[j] = r[i];
}

__global__ void write_kept_edges(KeepEdge keep, const int *erank, const int *vrank, const int *vlabel, int m,
                                 const long long *new_voff, uint32_t *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m || !keep(i)) return;
  const int2 e = keep.edges[i];
  const int j = erank[i] - 1;
  const long long base = new_voff[vlabel[e.x]];
  out[2LL * j] = uint32_t(vrank[e.x] - 1 - base);
  out[2LL * j + 1] = uint32_t(vrank[e.y] - 1 - base);
}

Set empty_like(const Set &s) {
  Set o;
  o.labels = s.labels;
  o.anisotropy = s.anisotropy;
  return o;
}

// The vertices with keep set, in order; the edges with both ends kept, in order and orientation,
// renumbered; every label stays (post.cu:72-105).
Set select(Context &ctx, const Set &s, const Graph &g, const Buffer<unsigned char> &keep) {
  if (!g.n) return s;
  cudaStream_t st = ctx.stream();
  Cub cub_call{ctx};
  Buffer<int> vrank(ctx, g.n), erank(ctx, std::max(g.m, 1));
  auto seq = thrust::counting_iterator<int>(0);
  auto vflags = thrust::make_transform_iterator(seq, KeepVertex{keep.data()});
  cub_call([&](void *t, size_t &b) { return cub::DeviceScan::InclusiveSum(t, b, vflags, vrank.data(), g.n, st); });
  KeepEdge ke{keep.data(), g.edges.data()};
  if (g.m) {
    auto eflags = thrust::make_transform_iterator(seq, ke);
    cub_call([&](void *t, size_t &b) { return cub::DeviceScan::InclusiveSum(t, b, eflags, erank.data(), g.m, st); });
  }
  Buffer<long long> nvoff(ctx, g.k + 1), neoff(ctx, g.k + 1);
  offsets_from_rank<<<blocks_for(g.k + 1), 256, 0, st>>>(g.voff.data(), g.k, vrank.data(), nvoff.data());
  ++ctx.launches;
  if (g.m) {
    offsets_from_rank<<<blocks_for(g.k + 1), 256, 0, st>>>(g.eoff.data(), g.k, erank.data(), neoff.data());
    ++ctx.launches;
  } else {
    neoff.zero();
  }
  BK_CUDA(cudaGetLastError());
  const auto hv = nvoff.download(g.k + 1), he = neoff.download(g.k + 1);
  Set o = empty_like(s);
  o.voff.assign(hv.begin(), hv.end());
  o.eoff.assign(he.begin(), he.end());
  const int nv = o.n(), ne = o.m();
  o.vbuf = std::make_shared<Buffer<float>>(ctx, 3 * size_t(nv));
  o.rbuf = std::make_shared<Buffer<float>>(ctx, size_t(nv));
  o.ebuf = std::make_shared<Buffer<uint32_t>>(ctx, 2 * size_t(ne));
  o.v = o.vbuf->data();
  o.r = o.rbuf->data();
  o.e = o.ebuf->data();
  write_kept_vertices<<<blocks_for(g.n), 256, 0, st>>>(s.v, s.r, keep.data(), vrank.data(), g.n, o.vbuf->data(),
                                                        o.rbuf->data());
  ++ctx.launches;
  if (g.m) {
    write_kept_edges<<<blocks_for(g.m), 256, 0, st>>>(ke, erank.data(), vrank.data(), g.vlabel.data(), g.m,
                                                       nvoff.data(), o.ebuf->data());
    ++ctx.launches;
  }
  BK_CUDA(cudaGetLastError());
  return o;
}

__global__ void count_key_labels(const u64 *keys, int n, const int *vlabel, int *counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(counts + vlabel[int(keys[i] >> 32)], 1);
}

__global__ void write_key_edges(const u64 *keys, int n, const int *vlabel, const long long *voff, uint32_t *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int a = int(keys[i] >> 32), b = int(unsigned(keys[i]));
  const long long base = voff[vlabel[a]];
  out[2LL * i] = uint32_t(a - base);
  out[2LL * i + 1] = uint32_t(b - base);
}

// The edges become the sorted distinct (lower, higher) global keys of keys[0, count) (the all-ones
// key drops an edge); the vertices stay (post.cu:293-306). keys must hold count + 1 entries.
Set edge_result(Context &ctx, const Set &s, const Graph &g, Buffer<u64> &keys, int count) {
  cudaStream_t st = ctx.stream();
  Cub cub_call{ctx};
  BK_CUDA(cudaMemsetAsync(keys.data() + count, 0xFF, sizeof(u64), st));  // the sentinel sorts last
  Buffer<u64> sorted(ctx, size_t(count) + 1);
  Buffer<int> selected(ctx, 1);
  cub_call([&](void *t, size_t &b) {
    return cub::DeviceRadixSort::SortKeys(t, b, keys.data(), sorted.data(), count + 1, 0, 64, st);
  });
  cub_call([&](void *t, size_t &b) {
    return cub::DeviceSelect::Unique(t, b, sorted.data(), keys.data(), selected.data(), count + 1, st);
  });
  const int ne = selected.download(1)[0] - 1;
  Buffer<int> counts(ctx, std::max(g.k, 1));
  counts.zero();
  Set o = s;
  o.ebuf = std::make_shared<Buffer<uint32_t>>(ctx, 2 * size_t(ne));
  o.e = o.ebuf->data();
  if (ne) {
    count_key_labels<<<blocks_for(ne), 256, 0, st>>>(keys.data(), ne, g.vlabel.data(), counts.data());
    write_key_edges<<<blocks_for(ne), 256, 0, st>>>(keys.data(), ne, g.vlabel.data(), g.voff.data(), o.ebuf->data());
    ctx.launches += 2;
  }
  BK_CUDA(cudaGetLastError());
  const auto hc = counts.download(g.k);
  o.eoff.assign(1, 0);
  for (int l = 0; l < g.k; ++l) o.eoff.push_back(o.eoff.back() + hc[l]);
  return o;
}

__global__ void degree_keep(const int *degree, int n, unsigned char *keep) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keep[i] = degree[i] != 0;
}

struct IsZero {
  const int *x;
  __device__ int operator()(int i) const { return x[i] == 0; }
};

// Vertices on no edge are dropped when there are any (post.cu:415-426).
Set prune(Context &ctx, const Set &s) {
  if (!s.n()) return s;
  Graph g = graph_of(ctx, s);
  Cub cub_call{ctx};
  Buffer<int> zeros(ctx, 1);
  auto flags = thrust::make_transform_iterator(thrust::counting_iterator<int>(0), IsZero{g.degree.data()});
  cub_call([&](void *t, size_t &b) { return cub::DeviceReduce::Sum(t, b, flags, zeros.data(), g.n, ctx.stream()); });
  if (!zeros.download(1)[0]) return s;
  Buffer<unsigned char> keep(ctx, g.n);
  degree_keep<<<blocks_for(g.n), 256, 0, ctx.stream()>>>(g.degree.data(), g.n, keep.data());
  ++ctx.launches;
  return select(ctx, s, g, keep);
}

// ------------------------------------------------------------------------------ remove_dust ----

__global__ void cable_lengths(const float *v, const int2 *edges, const int *root, int m, double *total, int *count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int2 e = edges[i];
  const double x = double(v[3LL * e.y] - v[3LL * e.x]), y = double(v[3LL * e.y + 1] - v[3LL * e.x + 1]),
               z = double(v[3LL * e.y + 2] - v[3LL * e.x + 2]);
  const int c = root[e.x];
  atomicAdd(total + c, sqrt((x * x + y * y) + z * z));
  atomicAdd(count + c, 1);
}

// Components whose double length is too near the threshold to decide.
struct NearThreshold {
  const double *total;
  const int *count;
  double threshold;
  __device__ int operator()(int i) const {
    return count[i] > 0 && fabs(total[i] - threshold) <= count[i] * (1.0 / 8388608.0) * threshold;
  }
};

__global__ void keep_by_length(const double *total, int n, double threshold, unsigned char *keep_root) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keep_root[i] = total[i] > threshold;
}

__global__ void edge_component_keys(const int2 *edges, const int *root, int m, int *keys, int *index) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  keys[i] = root[edges[i].x];
  index[i] = i;
}

__global__ void segment_bounds(const int *keys, int m, int *begin, int *end) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  if (i == 0 || keys[i - 1] != keys[i]) begin[keys[i]] = i;
  if (i + 1 == m || keys[i + 1] != keys[i]) end[keys[i]] = i + 1;
}

// The float32 length of edge `i` (float differences, squares and sum, float root).
__device__ __forceinline__ float edge_length32(const float *v, int2 e) {
  float x = v[3LL * e.y] - v[3LL * e.x], y = v[3LL * e.y + 1] - v[3LL * e.x + 1], z = v[3LL * e.y + 2] - v[3LL * e.x + 2];
  x = x * x;
  y = y * y;
  z = z * z;
  return sqrtf((x + y) + z);
}

struct EdgeLengths {
  const float *v;
  const int2 *edges;
  const int *order;  // edges sorted by component (stable)
  __device__ float operator()(long long i) const { return edge_length32(v, edges[order[i]]); }
};

// NumPy's pairwise float32 summation over x[0, n): below 8 values a plain sum, up to 128 eight lanes
// and their tree, above that the two halves (cut at a multiple of 8) summed alike; iterative.
__device__ float numpy_pairwise(const EdgeLengths &x, long long first, long long n) {
  struct Frame {
    long long off, n;
    float left;
    int stage;
  };
  Frame st[48];
  int sp = 0;
  st[0] = {first, n, 0.0f, 0};
  float ret = 0.0f;
  while (sp >= 0) {
    Frame &f = st[sp];
    if (f.n <= 128) {
      if (f.n < 8) {
        float s = -0.0f;
        for (long long i = 0; i < f.n; ++i) s += x(f.off + i);
        ret = s;
      } else {
        float lane[8];
        for (int j = 0; j < 8; ++j) lane[j] = x(f.off + j);
        long long i = 8;
        for (; i < f.n - f.n % 8; i += 8)
          for (int j = 0; j < 8; ++j) lane[j] += x(f.off + i + j);
        float s = ((lane[0] + lane[1]) + (lane[2] + lane[3])) + ((lane[4] + lane[5]) + (lane[6] + lane[7]));
        for (; i < f.n; ++i) s += x(f.off + i);
        ret = s;
      }
      --sp;
      continue;
    }
    long long half = f.n / 2;
    half -= half % 8;
    if (f.stage == 0) {
      f.stage = 1;
      st[sp + 1] = {f.off, half, 0.0f, 0};
      ++sp;
    } else if (f.stage == 1) {
      f.left = ret;
      f.stage = 2;
      st[sp + 1] = {f.off + half, f.n - half, 0.0f, 0};
      ++sp;
    } else {
      ret = f.left + ret;
      --sp;
    }
  }
  return ret;
}

__global__ void decide_near(const int *near, int count, const int *begin, const int *end, EdgeLengths lengths,
                            double threshold, unsigned char *keep_root) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int c = near[i];
  keep_root[c] = double(numpy_pairwise(lengths, begin[c], end[c] - begin[c])) > threshold;
}

__global__ void broadcast_keep(const unsigned char *keep_root, const int *root, int n, unsigned char *keep) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keep[i] = keep_root[root[i]];
}

// post.cu:427-468.
Set remove_dust(Context &ctx, const Set &s, double threshold) {
  if (threshold == 0 || !s.n()) return s;
  cudaStream_t st = ctx.stream();
  Cub cub_call{ctx};
  Graph g = graph_of(ctx, s);
  Buffer<double> total(ctx, g.n);
  Buffer<int> count(ctx, g.n);
  total.zero();
  count.zero();
  if (g.m) {
    cable_lengths<<<blocks_for(g.m), 256, 0, st>>>(s.v, g.edges.data(), g.root.data(), g.m, total.data(), count.data());
    ++ctx.launches;
  }
  Buffer<unsigned char> keep_root(ctx, g.n), keep(ctx, g.n);
  keep_by_length<<<blocks_for(g.n), 256, 0, st>>>(total.data(), g.n, threshold, keep_root.data());
  ++ctx.launches;
  NearThreshold near_pred{total.data(), count.data(), threshold};
  auto seq = thrust::counting_iterator<int>(0);
  auto near_flags = thrust::make_transform_iterator(seq, near_pred);
  Buffer<int> nsel(ctx, 1);
  cub_call([&](void *t, size_t &b) { return cub::DeviceReduce::Sum(t, b, near_flags, nsel.data(), g.n, st); });
  const int nnear = nsel.download(1)[0];
  if (nnear) {
    Buffer<int> near(ctx, nnear);
    cub_call([&](void *t, size_t &b) {
      return cub::DeviceSelect::Flagged(t, b, seq, near_flags, near.data(), nsel.data(), g.n, st);
    });
    Buffer<int> keys(ctx, g.m), keys_sorted(ctx, g.m), index(ctx, g.m), order(ctx, g.m), begin(ctx, g.n),
        end(ctx, g.n);
    edge_component_keys<<<blocks_for(g.m), 256, 0, st>>>(g.edges.data(), g.root.data(), g.m, keys.data(), index.data());
    ++ctx.launches;
    cub_call([&](void *t, size_t &b) {
      return cub::DeviceRadixSort::SortPairs(t, b, keys.data(), keys_sorted.data(), index.data(), order.data(), g.m, 0,
                                             32, st);
    });
    segment_bounds<<<blocks_for(g.m), 256, 0, st>>>(keys_sorted.data(), g.m, begin.data(), end.data());
    decide_near<<<blocks_for(nnear, 64), 64, 0, st>>>(near.data(), nnear, begin.data(), end.data(),
                                                       EdgeLengths{s.v, g.edges.data(), order.data()}, threshold,
                                                       keep_root.data());
    ctx.launches += 2;
  }
  broadcast_keep<<<blocks_for(g.n), 256, 0, st>>>(keep_root.data(), g.root.data(), g.n, keep.data());
  ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  return select(ctx, s, g, keep);
}

// ------------------------------------------------------------------------ component arenas ----

// The components that need work, each with its vertices (ascending ids, local ids 0..nv-1) and its
// edge rows (ascending edge index, local endpoints) in contiguous ranges.
struct Arena {
  int count = 0, n = 0, m = 0;
  std::vector<long long> hvs, hes;  // per-component offsets on the host (count + 1)
  Buffer<long long> vs, es;
  Buffer<int> slot;                 // per vertex id: the component's index when it is a root, else -1
  Buffer<int> vertices, edges;      // global vertex ids / global edge indices, by component
  Buffer<int2> rows;                // local endpoints of edges[]
  Buffer<float> xyz, radii;         // component-local copies
};

__global__ void component_sizes(const int *root, const int *degree, int n, const int2 *edges, int m, int *nv, int *ne,
                                int *branch) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    atomicAdd(nv + root[i], 1);
    if (degree[i] >= 3) branch[root[i]] = 1;
  }
  if (i < m) atomicAdd(ne + root[edges[i].x], 1);
}

// trees: a branched tree (remove_ticks); else: a component with at least as many edges as
// vertices (remove_loops), as post.cu:152-155 counts them (duplicate rows and self loops included).
struct WorkComponent {
  const int *nv, *ne, *branch;
  bool trees;
  __device__ int operator()(int i) const {
    return trees ? (branch[i] && ne[i] == nv[i] - 1) : (ne[i] > 0 && ne[i] - nv[i] + 1 > 0);
  }
};

__global__ void set_slots(const int *roots, int count, int *slot, const int *nv, const int *ne, int *sizes) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int r = roots[i];
  slot[r] = i;
  sizes[2 * i] = nv[r];
  sizes[2 * i + 1] = ne[r];
}

struct InWork {
  const int *root, *slot;
  __device__ int operator()(int i) const { return slot[root[i]] >= 0; }
};
struct EdgeInWork {
  const int2 *edges;
  const int *root, *slot;
  __device__ int operator()(int i) const { return slot[root[edges[i].x]] >= 0; }
};

__global__ void slot_keys(const int *ids, int n, const int *root, const int *slot, const int2 *edges, bool edge,
                          unsigned *keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int v = edge ? edges[ids[i]].x : ids[i];
  keys[i] = unsigned(slot[root[v]]);
}

__global__ void arena_vertices(const int *ids, int n, const int *root, const int *slot, const long long *vs,
                               const float *v, const float *r, int *local, float *xyz, float *radii) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int g = ids[i];
  local[g] = int(i - vs[slot[root[g]]]);
  for (int a = 0; a < 3; ++a) xyz[3LL * i + a] = v[3LL * g + a];
  radii[i] = r[g];
}

__global__ void arena_rows(const int *ids, int n, const int2 *edges, const int *local, int2 *rows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int2 e = edges[ids[i]];
  rows[i] = make_int2(local[e.x], local[e.y]);
}

Arena arena_of(Context &ctx, const Set &s, const Graph &g, bool trees) {
  cudaStream_t st = ctx.stream();
  Cub cub_call{ctx};
  Arena a;
  Buffer<int> nv(ctx, g.n), ne(ctx, g.n), branch(ctx, g.n);
  nv.zero();
  ne.zero();
  branch.zero();
  component_sizes<<<blocks_for(std::max(g.n, g.m)), 256, 0, st>>>(g.root.data(), g.degree.data(), g.n, g.edges.data(),
                                                                   g.m, nv.data(), ne.data(), branch.data());
  ++ctx.launches;
  WorkComponent pred{nv.data(), ne.data(), branch.data(), trees};
  auto seq = thrust::counting_iterator<int>(0);
  auto flags = thrust::make_transform_iterator(seq, pred);
  Buffer<int> count(ctx, 1);
  cub_call([&](void *t, size_t &b) { return cub::DeviceReduce::Sum(t, b, flags, count.data(), g.n, st); });
  a.count = count.download(1)[0];
  if (!a.count) return a;
  Buffer<int> roots(ctx, a.count), sizes(ctx, 2 * size_t(a.count));
  a.slot = Buffer<int>(ctx, g.n);
  a.slot.fill_bytes(0xFF);
  cub_call([&](void *t, size_t &b) {
    return cub::DeviceSelect::Flagged(t, b, seq, flags, roots.data(), count.data(), g.n, st);
  });
  set_slots<<<blocks_for(a.count), 256, 0, st>>>(roots.data(), a.count, a.slot.data(), nv.data(), ne.data(),
                                                  sizes.data());
  ++ctx.launches;
  const auto hs = sizes.download(2 * size_t(a.count));
  a.hvs.assign(1, 0);
  a.hes.assign(1, 0);
  for (int c = 0; c < a.count; ++c) {
    a.hvs.push_back(a.hvs.back() + hs[2 * c]);
    a.hes.push_back(a.hes.back() + hs[2 * c + 1]);
  }
  a.n = int(a.hvs.back());
  a.m = int(a.hes.back());
  a.vs = to_device(ctx, a.hvs);
  a.es = to_device(ctx, a.hes);
  // the members, then a stable radix sort by component
  auto members = [&](Buffer<int> &ids, int total, int universe, auto pred2, bool edge) {
    Buffer<int> picked(ctx, std::max(total, 1)), keyed(ctx, std::max(total, 1));
    cub_call([&](void *t, size_t &b) {
      return cub::DeviceSelect::If(t, b, seq, picked.data(), count.data(), universe, pred2, st);
    });
    Buffer<unsigned> keys(ctx, std::max(total, 1)), sorted(ctx, std::max(total, 1));
    slot_keys<<<blocks_for(total), 256, 0, st>>>(picked.data(), total, g.root.data(), a.slot.data(), g.edges.data(),
                                                  edge, keys.data());
    ++ctx.launches;
    cub_call([&](void *t, size_t &b) {
      return cub::DeviceRadixSort::SortPairs(t, b, keys.data(), sorted.data(), picked.data(), keyed.data(), total, 0,
                                             32, st);
    });
    ids = std::move(keyed);
  };
  members(a.vertices, a.n, g.n, InWork{g.root.data(), a.slot.data()}, false);
  if (a.m) members(a.edges, a.m, g.m, EdgeInWork{g.edges.data(), g.root.data(), a.slot.data()}, true);
  else a.edges = Buffer<int>(ctx, 1);
  Buffer<int> local(ctx, g.n);
  a.xyz = Buffer<float>(ctx, 3 * size_t(a.n));
  a.radii = Buffer<float>(ctx, a.n);
  a.rows = Buffer<int2>(ctx, std::max(a.m, 1));
  arena_vertices<<<blocks_for(a.n), 256, 0, st>>>(a.vertices.data(), a.n, g.root.data(), a.slot.data(), a.vs.data(),
                                                   s.v, s.r, local.data(), a.xyz.data(), a.radii.data());
  ++ctx.launches;
  if (a.m) {
    arena_rows<<<blocks_for(a.m), 256, 0, st>>>(a.edges.data(), a.m, g.edges.data(), local.data(), a.rows.data());
    ++ctx.launches;
  }
  BK_CUDA(cudaGetLastError());
  return a;
}

// ----------------------------------------------------------------------------- remove_loops ----
//
// One thread per component with a cycle; the rules are post_kernels.cuh:23-192's (Kimimaro's
// _remove_loops): rounds of "find a cycle by depth-first search from the first live row's first
// node, resolve it by its number of branch nodes", until no cycle or a one-node cycle is found.
// Bookkeeping of this walker:
//   rows      cap = 2 * E0 + 2 slots; dead rows have x = -1; compacted (order kept) when full
//   adjacency per node a doubly linked list of distinct neighbours in insertion order, entries
//             from a pool with a free list; an entry holds its first row and the row multiplicity
//   2-core    a node whose count of non-peeled neighbour entries drops to one or zero is peeled
//             and remembers the neighbour it hangs from; the search does not enter a peeled
//             node from the node it hangs from (such a subtree has no cycle and one way in, so the
//             search's other steps and its result are unchanged). A new row first un-peels both
//             ends and the chains they hang from.

struct LoopWalker {
  enum : int { kPeeled = 1, kVisited = 2, kDrop = 4, kQueued = 8 };
  int nv, cap;
  const float *P, *R;
  int2 *rows;
  int nrows = 0, nlive = 0, first = 0;
  int *to, *row, *mult, *nxt, *prv;
  int used = 0, freehead = -1;
  int *head, *tail, *cnt, *cdeg, *hang, *flags, *queue, *list, *path;
  int *stack;
  int qn = 0;
  bool full = false;  // a bound was reached (only duplicate rows given in both orientations can do it)

  __device__ int find(int a, int b) const {
    for (int e = head[a]; e >= 0; e = nxt[e])
      if (to[e] == b) return e;
    return -1;
  }
  __device__ void link(int a, int b, int r) {
    int e;
    if (freehead >= 0) { e = freehead; freehead = nxt[e]; } else { e = used++; }
    to[e] = b;
    row[e] = r;
    mult[e] = 1;
    nxt[e] = -1;
    prv[e] = tail[a];
    if (tail[a] >= 0) nxt[tail[a]] = e; else head[a] = e;
    tail[a] = e;
  }
  __device__ void unlink(int a, int e) {
    if (prv[e] >= 0) nxt[prv[e]] = nxt[e]; else head[a] = nxt[e];
    if (nxt[e] >= 0) prv[nxt[e]] = prv[e]; else tail[a] = prv[e];
    nxt[e] = freehead;
    freehead = e;
  }
  __device__ void enqueue(int v) {
    if (!(flags[v] & kQueued)) { flags[v] |= kQueued; queue[qn++] = v; }
  }
  __device__ void unpeel(int v) {
    while (v >= 0 && (flags[v] & kPeeled)) {
      flags[v] &= ~kPeeled;
      int c = 0;
      for (int e = head[v]; e >= 0; e = nxt[e]) {
        const int w = to[e];
        if (!(flags[w] & kPeeled)) {
          ++c;
          if (w != v) ++cdeg[w];
        }
      }
      cdeg[v] = c;
      enqueue(v);
      v = hang[v];
    }
  }
  __device__ void peel() {
    while (qn > 0) {
      const int c = queue[--qn];
      flags[c] &= ~kQueued;
      if ((flags[c] & kPeeled) || cdeg[c] > 1) continue;
      int u = -1;
      for (int e = head[c]; e >= 0; e = nxt[e])
        if (!(flags[to[e]] & kPeeled)) { u = to[e]; break; }
      flags[c] |= kPeeled;
      hang[c] = u;
      if (u >= 0 && --cdeg[u] <= 1) enqueue(u);
    }
  }
  __device__ void add_row(int x, int y) {
    if (nrows >= cap || (freehead < 0 && used + 2 > 2 * cap)) { full = true; return; }
    unpeel(x);
    unpeel(y);
    const int r = nrows++;
    rows[r] = make_int2(x, y);
    ++nlive;
    ++cnt[x];
    ++cnt[y];
    const int f = find(x, y);
    if (f >= 0) {
      ++mult[f];
      ++mult[find(y, x)];
    } else {
      link(x, y, r);
      link(y, x, r);
      ++cdeg[x];
      ++cdeg[y];
    }
    enqueue(x);
    enqueue(y);
  }
  // all rows of the edge (a, b) go (post_kernels.cuh:157-172, duplicates matched as (lower, higher))
  __device__ void drop_edge(int a, int b) {
    const int e = find(a, b);
    if (e < 0) return;
    const int m = mult[e];
    if (m == 1) {
      rows[row[e]].x = -1;
    } else {
      const int lo = min(a, b), hi = max(a, b);
      for (int r = first; r < nrows; ++r)
        if (rows[r].x == lo && rows[r].y == hi) rows[r].x = -1;
    }
    nlive -= m;
    cnt[a] -= m;
    cnt[b] -= m;
    const int f = find(b, a);
    unlink(a, e);
    unlink(b, f);
    --cdeg[a];
    --cdeg[b];
    enqueue(a);
    enqueue(b);
  }
  __device__ void compact() {
    int w = 0;
    for (int r = 0; r < nrows; ++r) {
      int moved = -1;
      if (rows[r].x >= 0) { rows[w] = rows[r]; moved = w++; }
      stack[r] = moved;
    }
    for (int v = 0; v < nv; ++v)
      for (int e = head[v]; e >= 0; e = nxt[e]) row[e] = stack[row[e]];
    nrows = w;
    first = 0;
  }
  // the depth-first search; returns the node reached twice (or -1) and the path length
  __device__ int search(int start, int &plen) {
    int sp = 1, seen = 0, node = -1;
    bool found = false;
    plen = 0;
    stack[0] = start;
    stack[1] = -1;
    stack[2] = 0;
    while (sp > 0) {
      --sp;
      node = stack[3 * sp];
      const int parent = stack[3 * sp + 1], depth = stack[3 * sp + 2];
      if (plen > depth) plen = depth;
      path[plen++] = node;
      if (flags[node] & kVisited) { found = true; break; }
      flags[node] |= kVisited;
      list[seen++] = node;
      for (int e = head[node]; e >= 0; e = nxt[e]) {
        const int c = to[e];
        if (c == parent || ((flags[c] & kPeeled) && hang[c] == node)) continue;
        stack[3 * sp] = c;
        stack[3 * sp + 1] = node;
        stack[3 * sp + 2] = depth + 1;
        ++sp;
      }
    }
    for (int j = 0; j < seen; ++j) flags[list[j]] &= ~kVisited;
    return found ? node : -1;
  }
  __device__ float sq(int a, int b) const {
    const float dx = P[3 * a] - P[3 * b], dy = P[3 * a + 1] - P[3 * b + 1], dz = P[3 * a + 2] - P[3 * b + 2];
    return (dx * dx + dy * dy) + dz * dz;
  }

  __device__ void run(int E0) {
    for (int v = 0; v < nv; ++v) {
      head[v] = tail[v] = -1;
      cnt[v] = cdeg[v] = 0;
      hang[v] = -1;
      flags[v] = 0;
    }
    // the component's rows arrive in rows[0, E0)
    nrows = 0;
    for (int i = 0; i < E0; ++i) {
      const int2 r = rows[i];
      const int x = r.x, y = r.y;
      // re-adding in place: add_row writes rows[nrows] == rows[i]
      add_row(x, y);
    }
    int app0 = nrows, app1 = nrows;
    peel();
    for (;;) {
      if (nlive == 0) break;
      while (rows[first].x < 0) ++first;
      int plen = 0;
      const int node = search(rows[first].x, plen);
      if (node < 0 || plen <= 1) break;
      int i0 = 0;
      while (i0 < plen - 1 && path[i0] != node) ++i0;
      if (plen - i0 < 3) break;
      const int *cy = path + i0;
      const int cl = plen - i0;
      int nb = 0;
      for (int j = 0; j + 1 < cl; ++j)
        if (cnt[cy[j]] >= 3) list[nb++] = cy[j];
      for (int i = 1; i < nb; ++i) {  // branch nodes ascending
        const int x = list[i];
        int j = i - 1;
        while (j >= 0 && list[j] > x) { list[j + 1] = list[j]; --j; }
        list[j + 1] = x;
      }
      int add_a = -1, add_b = -1, inter = -1;
      bool many = false;
      if (nb == 0) {
        for (int j = 0; j + 1 < cl; ++j) flags[cy[j]] |= kDrop;
      } else if (nb == 1) {
        const int b = list[0];
        int end = -1;
        float best = -1.0f;
        for (int j = 0; j + 1 < cl; ++j) {
          const int v = cy[j];
          const float d = sq(v, b);
          if (end < 0 || d > best || (d == best && v < end)) { best = d; end = v; }
        }
        for (int j = 0; j + 1 < cl; ++j) flags[cy[j]] |= kDrop;
        add_a = b;
        add_b = end;
      } else if (nb == 2) {
        const int L = cl - 1;
        int p0 = -1, p1 = -1;
        for (int j = 0; j < L; ++j)
          if (cnt[cy[j + 1]] >= 3) { if (p0 < 0) p0 = j; else p1 = j; }
        const bool inner = double(p1 - p0) < double(L) / 2.0;
        for (int j = 0; j + 1 < cl; ++j) {
          const bool on_inner = j - 1 >= 0 && j - 1 >= p0 && j <= p1;
          if (inner != on_inner) flags[cy[j]] |= kDrop;
        }
      } else {
        float cx = 0.0f, cyy = 0.0f, cz = 0.0f;
        for (int i = 0; i < nb; ++i) {
          cx += P[3 * list[i]];
          cyy += P[3 * list[i] + 1];
          cz += P[3 * list[i] + 2];
        }
        cx /= float(nb);
        cyy /= float(nb);
        cz /= float(nb);
        float best = 0.0f;
        for (int v = 0; v < nv; ++v) {
          const float dx = P[3 * v] - cx, dy = P[3 * v + 1] - cyy, dz = P[3 * v + 2] - cz;
          const float d = (dx * dx + dy * dy) + dz * dz;
          if (inter < 0 || d < best) { best = d; inter = v; }
        }
        float far = 0.0f;
        for (int i = 0; i < nb; ++i) {
          const float d = sq(list[i], inter);
          if (i == 0 || d > far) far = d;
        }
        if (sqrtf(far) > R[inter]) {
          flags[cy[0]] |= kDrop;
        } else {
          for (int j = 0; j + 1 < cl; ++j) flags[cy[j]] |= kDrop;
          many = true;
        }
      }
      for (int r = app0; r < app1; ++r)
        if (rows[r].x > rows[r].y) rows[r] = make_int2(rows[r].y, rows[r].x);
      for (int j = 0; j + 1 < cl; ++j)
        if (flags[cy[j]] & kDrop) drop_edge(cy[j], cy[j + 1]);
      const int adds = many ? nb : (add_b >= 0 ? 1 : 0);
      if (nrows + adds > cap) compact();
      if (nrows + adds > cap) break;
      app0 = nrows;
      if (add_b >= 0) add_row(add_a, add_b);
      if (many)
        for (int i = 0; i < nb; ++i)
          if (list[i] != inter) add_row(list[i], inter);
      app1 = nrows;
      for (int j = 0; j + 1 < cl; ++j) flags[cy[j]] &= ~kDrop;
      peel();
      if (full) break;
    }
  }
};

// Per-component workspace sizes (ints): rows 2 * cap, entries 5 * 2 * cap, nodes 9 * nv + 1,
// stack 3 * (2 * cap + 1); cap = 2 * E0 + 2. Live rows never outnumber the component's E0 rows (a
// round removes at least as many rows as it adds), live entries are two per distinct edge, and a
// search pushes at most one item per entry of the nodes it visits once each.
__host__ __device__ inline long long loop_ints(long long nv, long long e0) {
  const long long cap = 2 * e0 + 2;
  const long long ints = 2 * cap + 10 * cap + 9 * nv + 1 + 3 * (2 * cap + 1);
  return (ints + 1) & ~1LL;  // even, so that the next component's rows (int2) stay 8-byte aligned
}

__global__ void loops_kernel(int count, const long long *vs, const long long *es, const long long *base,
                             const float *xyz, const float *radii, int2 *rows_io, int *kept, int *work) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= count) return;
  const long long v0 = vs[c], e0 = es[c];
  const int nv = int(vs[c + 1] - v0), E0 = int(es[c + 1] - e0);
  const int cap = 2 * E0 + 2, E = 2 * cap;
  int *w = work + base[c];
  LoopWalker lw;
  lw.nv = nv;
  lw.cap = cap;
  lw.P = xyz + 3 * v0;
  lw.R = radii + v0;
  lw.rows = reinterpret_cast<int2 *>(w);
  w += 2 * cap;
  lw.to = w; w += E;
  lw.row = w; w += E;
  lw.mult = w; w += E;
  lw.nxt = w; w += E;
  lw.prv = w; w += E;
  lw.head = w; w += nv;
  lw.tail = w; w += nv;
  lw.cnt = w; w += nv;
  lw.cdeg = w; w += nv;
  lw.hang = w; w += nv;
  lw.flags = w; w += nv;
  lw.queue = w; w += nv;
  lw.list = w; w += nv;
  lw.path = w; w += nv + 1;
  lw.stack = w;
  for (int i = 0; i < E0; ++i) lw.rows[i] = rows_io[e0 + i];
  lw.run(E0);
  int out = 0;
  for (int r = 0; r < lw.nrows; ++r)
    if (lw.rows[r].x >= 0) rows_io[e0 + out++] = lw.rows[r];
  kept[c] = out;
}

__global__ void plain_keys(const int2 *edges, const int *root, const int *slot, int m, u64 *keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int2 e = edges[i];
  u64 key = ~0ull;
  if (slot[root[e.x]] < 0 && e.x != e.y)
    key = (u64(unsigned(min(e.x, e.y))) << 32) | unsigned(max(e.x, e.y));
  keys[i] = key;
}

__global__ void loop_keys(const int *edge_ids, const int2 *rows, int total, const int *comp, const long long *es,
                          const long long *vs, const int *kept, const int *vertices, u64 *keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const int c = comp[i];
  u64 key = ~0ull;
  if (i - es[c] < kept[c]) {
    const int2 r = rows[i];
    const unsigned a = unsigned(vertices[vs[c] + r.x]), b = unsigned(vertices[vs[c] + r.y]);
    if (a != b) key = (u64(min(a, b)) << 32) | max(a, b);
  }
  keys[edge_ids[i]] = key;
}

__global__ void row_components(const long long *es, int count, int *comp) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= count) return;
  for (long long i = es[c]; i < es[c + 1]; ++i) comp[i] = c;
}

__global__ void keep_unemptied(const int *root, const int *slot, const int *kept, int n, unsigned char *keep) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = slot[root[i]];
  keep[i] = c < 0 || kept[c] > 0;
}

// post.cu:469-489.
Set remove_loops(Context &ctx, const Set &s) {
  if (!s.n() || !s.m()) return s;
  cudaStream_t st = ctx.stream();
  Graph g = graph_of(ctx, s);
  Arena a = arena_of(ctx, s, g, false);
  if (!a.count) return s;
  std::vector<long long> base(a.count + 1, 0);
  for (int c = 0; c < a.count; ++c)
    base[c + 1] = base[c] + loop_ints(a.hvs[c + 1] - a.hvs[c], a.hes[c + 1] - a.hes[c]);
  Buffer<long long> d_base = to_device(ctx, base);
  Buffer<int> work(ctx, size_t(base.back())), kept(ctx, a.count), comp(ctx, std::max(a.m, 1));
  loops_kernel<<<blocks_for(a.count, 64), 64, 0, st>>>(a.count, a.vs.data(), a.es.data(), d_base.data(), a.xyz.data(),
                                                       a.radii.data(), a.rows.data(), kept.data(), work.data());
  row_components<<<blocks_for(a.count, 64), 64, 0, st>>>(a.es.data(), a.count, comp.data());
  Buffer<u64> keys(ctx, size_t(g.m) + 1);
  plain_keys<<<blocks_for(g.m), 256, 0, st>>>(g.edges.data(), g.root.data(), a.slot.data(), g.m, keys.data());
  loop_keys<<<blocks_for(a.m), 256, 0, st>>>(a.edges.data(), a.rows.data(), a.m, comp.data(), a.es.data(), a.vs.data(),
                                             kept.data(), a.vertices.data(), keys.data());
  ctx.launches += 4;
  BK_CUDA(cudaGetLastError());
  Set out = edge_result(ctx, s, g, keys, g.m);
  const auto hk = kept.download(a.count);
  if (std::find(hk.begin(), hk.end(), 0) == hk.end()) return out;
  Buffer<unsigned char> keep(ctx, g.n);
  keep_unemptied<<<blocks_for(g.n), 256, 0, st>>>(g.root.data(), a.slot.data(), kept.data(), g.n, keep.data());
  ++ctx.launches;
  Graph h = graph_of(ctx, out);
  return select(ctx, out, h, keep);
}

// ----------------------------------------------------------------------------- remove_ticks ----
//
// One warp per branched tree; the rules are post_kernels.cuh:314-405's (Kimimaro's remove_ticks):
// chains between critical nodes (one or three-plus neighbours), each measured as the float32 sum of
// its edges' float32 lengths from the end nearer the first leaf (lowest local id), and the shortest
// eligible chain removed while it is shorter than the threshold and not between two nodes with one
// chain left; a branch node left with two chains fuses them. The result does not depend on the
// order the tree is walked in, so the warp builds the adjacency with atomics, walks every chain
// from both of its ends at once (a lane per walk), roots the small tree of critical nodes at the
// first leaf on one lane to pick each chain's measured end, and runs the heap loop over the chains
// on one lane; the rows' fate is written back by all lanes.

// Per-component workspace layout (ints, then doubles); shared by the host (sizes) and the kernel.
struct TickLayout {
  long long nv, e0, slots;
  __host__ __device__ TickLayout(long long nv_, long long e0_) : nv(nv_), e0(e0_), slots(2 * e0_) {}
  // ints: off (nv + 1), cursor (nv), src, nbr, nrow, wend, wother (slots each), chain_of_row (e0),
  // chain_at (slots), queue (nv), seen (nv), su, sv, sflag, ver, lhead, ltail, lnext, dead (e0 each),
  // ihead (nv), ito, inext (3 e0 + 1 each), hlo, hhi, hid, hver (2 e0 + 1 each); wlen as floats (slots)
  __host__ __device__ long long ints() const {
    return (nv + 1) + nv + 5 * slots + e0 + slots + 2 * nv + 8 * e0 + nv + 2 * (3 * e0 + 1) + 4 * (2 * e0 + 1) + slots;
  }
  __host__ __device__ long long doubles() const { return e0 + (2 * e0 + 1); }  // len, hlen
};

struct TickState {
  enum : int { kAlive = 1, kEligible = 2 };
  int nv, e0;
  const float *P;
  const int2 *rows;
  int *off, *cursor, *src, *nbr, *nrow, *wend, *wother, *chain_of_row, *chain_at, *queue, *seen;
  float *wlen;
  int *su, *sv, *sflag, *ver, *lhead, *ltail, *lnext, *dead;
  int *ihead, *ito, *inext;
  int *hlo, *hhi, *hid, *hver;
  double *len, *hlen;
  int in_used = 0, hn = 0;

  __device__ TickState(long long nv_, long long e0_, int *w, double *d) {
    nv = int(nv_);
    e0 = int(e0_);
    const long long slots = 2 * e0_;
    off = w; w += nv + 1;
    cursor = w; w += nv;
    src = w; w += slots;
    nbr = w; w += slots;
    nrow = w; w += slots;
    wend = w; w += slots;
    wother = w; w += slots;
    chain_of_row = w; w += e0;
    chain_at = w; w += slots;
    queue = w; w += nv;
    seen = w; w += nv;
    su = w; w += e0;
    sv = w; w += e0;
    sflag = w; w += e0;
    ver = w; w += e0;
    lhead = w; w += e0;
    ltail = w; w += e0;
    lnext = w; w += e0;
    dead = w; w += e0;
    ihead = w; w += nv;
    ito = w; w += 3 * e0 + 1;
    inext = w; w += 3 * e0 + 1;
    hlo = w; w += 2 * e0 + 1;
    hhi = w; w += 2 * e0 + 1;
    hid = w; w += 2 * e0 + 1;
    hver = w; w += 2 * e0 + 1;
    wlen = reinterpret_cast<float *>(w);
    len = d;
    hlen = d + e0;
  }
  __device__ int deg(int v) const { return off[v + 1] - off[v]; }
  __device__ float edge(int u, int v) const {
    float dx = P[3 * u] - P[3 * v], dy = P[3 * u + 1] - P[3 * v + 1], dz = P[3 * u + 2] - P[3 * v + 2];
    dx *= dx;
    dy *= dy;
    dz *= dz;
    return sqrtf((dx + dy) + dz);
  }
  __device__ void incident(int v, int s) {
    ito[in_used] = s;
    inext[in_used] = ihead[v];
    ihead[v] = in_used++;
  }
  __device__ bool less(int i, int j) const {
    return hlen[i] < hlen[j] || (hlen[i] == hlen[j] && (hlo[i] < hlo[j] || (hlo[i] == hlo[j] && hhi[i] < hhi[j])));
  }
  __device__ void swap_entries(int i, int j) {
    const double d = hlen[i]; hlen[i] = hlen[j]; hlen[j] = d;
    int t;
    t = hlo[i]; hlo[i] = hlo[j]; hlo[j] = t;
    t = hhi[i]; hhi[i] = hhi[j]; hhi[j] = t;
    t = hid[i]; hid[i] = hid[j]; hid[j] = t;
    t = hver[i]; hver[i] = hver[j]; hver[j] = t;
  }
  __device__ void push(int s) {
    int i = hn++;
    hlen[i] = len[s];
    hlo[i] = min(su[s], sv[s]);
    hhi[i] = max(su[s], sv[s]);
    hid[i] = s;
    hver[i] = ver[s];
    while (i > 0) {
      const int p = (i - 1) >> 1;
      if (!less(i, p)) break;
      swap_entries(i, p);
      i = p;
    }
  }
  __device__ void pop() {
    --hn;
    if (hn == 0) return;
    swap_entries(0, hn);
    int i = 0;
    for (;;) {
      const int l = 2 * i + 1, r = l + 1;
      int m = i;
      if (l < hn && less(l, m)) m = l;
      if (r < hn && less(r, m)) m = r;
      if (m == i) break;
      swap_entries(i, m);
      i = m;
    }
  }
};

__host__ __device__ inline long long tick_ints(long long nv, long long e0) { return TickLayout(nv, e0).ints(); }
__host__ __device__ inline long long tick_doubles(long long e0) { return TickLayout(0, e0).doubles(); }

constexpr int kTickWarps = 4;  // components per block (a warp each)

__global__ void ticks_kernel(int count, const long long *vs, const long long *es, const long long *ibase,
                             const long long *dbase, double threshold, const float *xyz, const int2 *rows, int *iwork,
                             double *dwork, int *keep_rows) {
  const int c = blockIdx.x * kTickWarps + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= count) return;
  const long long v0 = vs[c], r0 = es[c];
  TickState t(vs[c + 1] - v0, es[c + 1] - r0, iwork + ibase[c], dwork + dbase[c]);
  t.P = xyz + 3 * v0;
  t.rows = rows + r0;
  const int nv = t.nv, e0 = t.e0, slots = 2 * e0;
  int *keep = keep_rows + r0;
  // adjacency: degrees, offsets (warp scan), slots filled with atomics (any order)
  for (int v = lane; v <= nv; v += 32) t.off[v] = 0;
  __syncwarp();
  for (int r = lane; r < e0; r += 32) {
    atomicAdd(t.off + t.rows[r].x + 1, 1);
    atomicAdd(t.off + t.rows[r].y + 1, 1);
  }
  __syncwarp();
  int carry = 0;
  for (int base = 1; base <= nv; base += 32) {
    const int v = base + lane;
    int x = v <= nv ? t.off[v] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if (lane >= o) x += y;
    }
    if (v <= nv) t.off[v] = x + carry;
    carry += __shfl_sync(0xFFFFFFFFu, x, 31);
  }
  __syncwarp();
  for (int v = lane; v < nv; v += 32) t.cursor[v] = t.off[v];
  __syncwarp();
  for (int r = lane; r < e0; r += 32) {
    const int a = t.rows[r].x, b = t.rows[r].y;
    int q = atomicAdd(t.cursor + a, 1);
    t.src[q] = a; t.nbr[q] = b; t.nrow[q] = r;
    q = atomicAdd(t.cursor + b, 1);
    t.src[q] = b; t.nbr[q] = a; t.nrow[q] = r;
  }
  __syncwarp();
  // every chain walked from each of its ends (a lane per walk): its far end, the slot it arrives
  // by there, and its float32 length from this end; its rows keyed by the lower of its two slots
  for (int q = lane; q < slots; q += 32) {
    const int c0 = t.src[q];
    if (t.deg(c0) == 2) continue;
    int prev = c0, cur = t.nbr[q], row = t.nrow[q];
    float dist = 0.0f + t.edge(prev, cur);
    while (t.deg(cur) == 2) {
      const int s0 = t.off[cur];
      const int k = t.nbr[s0] == prev && t.nrow[s0] == row ? s0 + 1 : s0;
      const int next = t.nbr[k];
      row = t.nrow[k];
      dist = dist + t.edge(cur, next);
      prev = cur;
      cur = next;
    }
    int back = -1;  // the far end's slot of the chain's last edge
    for (int k = t.off[cur]; k < t.off[cur + 1]; ++k)
      if (t.nrow[k] == row) { back = k; break; }
    t.wend[q] = cur;
    t.wother[q] = back;
    t.wlen[q] = dist;
    const int key = min(q, back);
    // the rows of the chain, walked again from this end
    int p2 = c0, c2 = t.nbr[q], r2 = t.nrow[q];
    t.chain_of_row[r2] = key;
    while (t.deg(c2) == 2) {
      const int s0 = t.off[c2];
      const int k = t.nbr[s0] == p2 && t.nrow[s0] == r2 ? s0 + 1 : s0;
      r2 = t.nrow[k];
      t.chain_of_row[r2] = key;
      p2 = c2;
      c2 = t.nbr[k];
    }
  }
  __syncwarp();
  if (lane == 0) {
    int start = -1;
    for (int v = 0; v < nv && start < 0; ++v)
      if (t.deg(v) == 1) start = v;
    if (start >= 0) {
      // the tree of critical nodes rooted at the start leaf: each chain from its end nearer it
      for (int v = 0; v < nv; ++v) { t.seen[v] = 0; t.ihead[v] = -1; }
      int qh = 0, qt = 0, ns = 0;
      t.queue[qt++] = start;
      t.seen[start] = 1;
      while (qh < qt) {
        const int u = t.queue[qh++];
        for (int q = t.off[u]; q < t.off[u + 1]; ++q) {
          const int d = t.wend[q];
          if (t.seen[d]) continue;
          t.seen[d] = 1;
          t.queue[qt++] = d;
          const int s = ns++;
          t.chain_at[min(q, t.wother[q])] = s;
          t.su[s] = u;
          t.sv[s] = d;
          t.len[s] = double(t.wlen[q]);
          t.ver[s] = 0;
          t.sflag[s] = TickState::kAlive | ((t.deg(u) == 1 || t.deg(d) == 1) ? TickState::kEligible : 0);
          t.lhead[s] = t.ltail[s] = s;
          t.lnext[s] = -1;
          t.dead[s] = 0;
          t.incident(u, s);
          t.incident(d, s);
          if (t.sflag[s] & TickState::kEligible) t.push(s);
        }
      }
      int* bc = t.cursor;  // the chain count left at each node (its degree for branch nodes, else 0)
      for (int v = 0; v < nv; ++v) bc[v] = t.deg(v) >= 3 ? t.deg(v) : 0;
      int nalive = ns;
      while (nalive > 1) {
        while (t.hn > 0 && (!(t.sflag[t.hid[0]] & TickState::kAlive) || t.ver[t.hid[0]] != t.hver[0])) t.pop();
        if (t.hn == 0) break;
        const int best = t.hid[0];
        const int e1 = t.su[best], e2 = t.sv[best];
        if (bc[e1] == 1 && bc[e2] == 1) break;
        if (t.len[best] >= threshold) break;
        t.pop();
        for (int o = t.lhead[best]; o >= 0; o = t.lnext[o]) t.dead[o] = 1;
        t.sflag[best] = 0;
        --nalive;
        --bc[e1];
        --bc[e2];
        for (int side = 0; side < 2; ++side) {
          const int v = side ? e2 : e1;
          if (bc[v] != 2) continue;
          int a = -1, b = -1;
          for (int k = t.ihead[v]; k >= 0; k = t.inext[k]) {
            const int o = t.ito[k];
            if (!(t.sflag[o] & TickState::kAlive) || (t.su[o] != v && t.sv[o] != v) || o == a) continue;
            if (a < 0) a = o; else { b = o; break; }
          }
          if (a < 0 || b < 0) { bc[v] = 0; continue; }
          const int ea = t.su[a] == v ? t.sv[a] : t.su[a], eb = t.su[b] == v ? t.sv[b] : t.su[b];
          t.len[a] = (0.0 + t.len[a]) + t.len[b];
          t.su[a] = ea;
          t.sv[a] = eb;
          t.sflag[a] = TickState::kAlive | TickState::kEligible;
          t.lnext[t.ltail[a]] = t.lhead[b];
          t.ltail[a] = t.ltail[b];
          t.sflag[b] = 0;
          --nalive;
          t.incident(eb, a);
          ++t.ver[a];
          t.push(a);
          bc[v] = 0;
        }
      }
    }
    t.seen[0] = start;  // tells the lanes whether the tree was walked
  }
  __syncwarp();
  const bool walked = t.seen[0] >= 0;
  for (int r = lane; r < e0; r += 32) keep[r] = walked ? !t.dead[t.chain_at[t.chain_of_row[r]]] : 1;
}

__global__ void live_edges(const int *edge_ids, const int *keep_rows, int total, unsigned char *live) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) live[edge_ids[i]] = keep_rows[i] != 0;
}

__global__ void write_live_edges(const uint32_t *e, const unsigned char *live, const int *rank, int m, uint32_t *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m || !live[i]) return;
  const int j = rank[i] - 1;
  out[2LL * j] = e[2LL * i];
  out[2LL * j + 1] = e[2LL * i + 1];
}

// post.cu:490-519 and select_edge_rows (381-396): the surviving edges in order; vertices unchanged.
Set remove_ticks(Context &ctx, const Set &s, double threshold) {
  if (threshold == 0 || !s.n() || !s.m()) return s;
  cudaStream_t st = ctx.stream();
  Cub cub_call{ctx};
  Graph g = graph_of(ctx, s);
  Arena a = arena_of(ctx, s, g, true);
  if (!a.count) return s;
  std::vector<long long> ib(a.count + 1, 0), db(a.count + 1, 0);
  for (int c = 0; c < a.count; ++c) {
    const long long nv = a.hvs[c + 1] - a.hvs[c], e0 = a.hes[c + 1] - a.hes[c];
    ib[c + 1] = ib[c] + tick_ints(nv, e0);
    db[c + 1] = db[c] + tick_doubles(e0);
  }
  Buffer<long long> d_ib = to_device(ctx, ib), d_db = to_device(ctx, db);
  Buffer<int> iwork(ctx, size_t(ib.back())), keep_rows(ctx, std::max(a.m, 1));
  Buffer<double> dwork(ctx, size_t(db.back()));
  ticks_kernel<<<(a.count + kTickWarps - 1) / kTickWarps, 32 * kTickWarps, 0, st>>>(
      a.count, a.vs.data(), a.es.data(), d_ib.data(), d_db.data(), threshold, a.xyz.data(), a.rows.data(),
      iwork.data(), dwork.data(), keep_rows.data());
  Buffer<unsigned char> live(ctx, g.m);
  live.fill_bytes(1);
  live_edges<<<blocks_for(a.m), 256, 0, st>>>(a.edges.data(), keep_rows.data(), a.m, live.data());
  ctx.launches += 2;
  Buffer<int> rank(ctx, g.m);
  auto flags = thrust::make_transform_iterator(thrust::counting_iterator<int>(0), KeepFlag{live.data()});
  cub_call([&](void *t, size_t &b) { return cub::DeviceScan::InclusiveSum(t, b, flags, rank.data(), g.m, st); });
  Buffer<long long> neoff(ctx, g.k + 1);
  offsets_from_rank<<<blocks_for(g.k + 1), 256, 0, st>>>(g.eoff.data(), g.k, rank.data(), neoff.data());
  ++ctx.launches;
  const auto he = neoff.download(g.k + 1);
  Set o = s;
  o.eoff.assign(he.begin(), he.end());
  o.ebuf = std::make_shared<Buffer<uint32_t>>(ctx, 2 * size_t(o.m()));
  o.e = o.ebuf->data();
  write_live_edges<<<blocks_for(g.m), 256, 0, st>>>(s.e, live.data(), rank.data(), g.m, o.ebuf->data());
  ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  return o;
}

// -------------------------------------------------------------------------- join_components ----

__global__ void label_statistics(const int *root, const int *vlabel, const float *radii, int n, int *ncomp,
                                 unsigned *rmax) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int l = vlabel[i];
  if (root[i] == i) atomicAdd(ncomp + l, 1);
  const float r = radii[i];
  if (r > 0) atomicMax(rmax + l, __float_as_uint(r));
}

struct InMultiLabel {
  const int *vlabel, *rank;
  __device__ int operator()(int i) const { return rank[vlabel[i]] >= 0; }
};
struct MultiRoot {
  const int *vlabel, *rank, *root;
  __device__ int operator()(int i) const { return root[i] == i && rank[vlabel[i]] >= 0; }
};

// key of sorted position i for one pass: a cell coordinate (floor of the coordinate over the bound)
// or, for axis 3, the label's rank
__global__ void cell_pass_keys(const int *ids, const int *order, int n, const float *v, const int *vlabel,
                               const int *rank, const double *bound, int axis, long long *keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int g = ids[order[i]], l = rank[vlabel[g]];
  keys[i] = axis == 3 ? l : (long long)floor(double(v[3LL * g + axis]) / bound[l]);
}

__global__ void iota(int *x, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = i;
}

struct Cells {
  int *kl;
  long long *kx, *ky, *kz;
  float *xyz;
  int *gid, *comp;
};

__global__ void ordered_cells(const int *ids, const int *order, int n, const float *v, const int *root,
                              const int *vlabel, const int *rank, const double *bound, Cells c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int g = ids[order[i]], l = rank[vlabel[g]];
  c.kl[i] = l;
  c.gid[i] = g;
  c.comp[i] = root[g];
  for (int a = 0; a < 3; ++a) c.xyz[3LL * i + a] = v[3LL * g + a];
  c.kx[i] = (long long)floor(double(v[3LL * g]) / bound[l]);
  c.ky[i] = (long long)floor(double(v[3LL * g + 1]) / bound[l]);
  c.kz[i] = (long long)floor(double(v[3LL * g + 2]) / bound[l]);
}

__device__ __forceinline__ int cell_cmp(const Cells &c, int i, int l, long long x, long long y, long long z) {
  if (c.kl[i] != l) return c.kl[i] < l ? -1 : 1;
  if (c.kx[i] != x) return c.kx[i] < x ? -1 : 1;
  if (c.ky[i] != y) return c.ky[i] < y ? -1 : 1;
  if (c.kz[i] != z) return c.kz[i] < z ? -1 : 1;
  return 0;
}

struct Candidates {
  int *a, *b, *v, *u;  // components (a < b) and the two vertices (global ids)
  double *d;
};

// Candidates of vertex i: per higher component within the bound, its nearest vertex (ties to the
// lower id); up to 8 components are kept in registers, further ones go out as they come (the pair
// selection afterwards keeps the nearest per pair either way). mode 0 counts, mode 1 writes.
__global__ void join_scan(int n, int mode, Cells c, const double *bound, long long *counts, const long long *offsets,
                          Candidates out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int l = c.kl[i];
  const double bnd = bound[l];
  float b32 = float(bnd);
  b32 = b32 * b32 * 1.0001f + 1e-30f;
  constexpr int kSlots = 8;
  int s_comp[kSlots], s_j[kSlots];
  double s_d[kSlots];
  int ns = 0;
  long long emitted = 0;
  const long long base = mode ? offsets[i] : 0;
  const float px = c.xyz[3LL * i], py = c.xyz[3LL * i + 1], pz = c.xyz[3LL * i + 2];
  const int ci = c.comp[i];
  auto emit = [&](int comp_j, double d, int j) {
    if (mode) {
      const long long o = base + emitted;
      out.a[o] = ci;
      out.b[o] = comp_j;
      out.d[o] = d;
      out.v[o] = c.gid[i];
      out.u[o] = c.gid[j];
    }
    ++emitted;
  };
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const long long x = c.kx[i] + dx, y = c.ky[i] + dy, z = c.kz[i] + dz;
        int lo = 0, hi = n;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (cell_cmp(c, mid, l, x, y, z) < 0) lo = mid + 1; else hi = mid;
        }
        for (int j = lo; j < n && cell_cmp(c, j, l, x, y, z) == 0; ++j) {
          const int cj = c.comp[j];
          if (cj <= ci) continue;
          const float fx = c.xyz[3LL * j] - px, fy = c.xyz[3LL * j + 1] - py, fz = c.xyz[3LL * j + 2] - pz;
          if ((fx * fx + fy * fy) + fz * fz > b32) continue;
          const double ex = double(c.xyz[3LL * j]) - double(px), ey = double(c.xyz[3LL * j + 1]) - double(py),
                       ez = double(c.xyz[3LL * j + 2]) - double(pz);
          const double d = sqrt((ex * ex + ey * ey) + ez * ez);
          if (!(d < bnd)) continue;
          int s = -1;
          for (int t = 0; t < ns; ++t)
            if (s_comp[t] == cj) { s = t; break; }
          if (s >= 0) {
            if (d < s_d[s] || (d == s_d[s] && c.gid[j] < c.gid[s_j[s]])) { s_d[s] = d; s_j[s] = j; }
          } else if (ns < kSlots) {
            s_comp[ns] = cj;
            s_d[ns] = d;
            s_j[ns] = j;
            ++ns;
          } else {
            emit(cj, d, j);
          }
        }
      }
  for (int t = 0; t < ns; ++t) emit(s_comp[t], s_d[t], s_j[t]);
  if (!mode) counts[i] = emitted;
}

// sort keys of the candidates, least significant first: (lower, higher vertex), distance, (a, b)
__global__ void candidate_keys(const int *order, int n, Candidates c, int pass, u64 *keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = order[i];
  if (pass == 0) {
    const unsigned lo = unsigned(min(c.v[p], c.u[p])), hi = unsigned(max(c.v[p], c.u[p]));
    keys[i] = (u64(lo) << 32) | hi;
  } else if (pass == 1) {
    keys[i] = u64(__double_as_longlong(c.d[p]));
  } else {
    keys[i] = (u64(unsigned(c.a[p])) << 32) | unsigned(c.b[p]);
  }
}

struct FirstOfPair {
  const int *order;
  Candidates c;
  __device__ int operator()(int i) const {
    if (i == 0) return 1;
    const int x = order[i - 1], y = order[i];
    return c.a[x] != c.a[y] || c.b[x] != c.b[y];
  }
};

__global__ void root_positions(const int *roots, int nr, const int *vlabel, const int *rank, const long long *cs,
                               int *local) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nr) local[roots[i]] = int(i - cs[rank[vlabel[roots[i]]]]);
}

struct PairList {
  int *cx, *cy, *va, *vb;
  double *d;
};

__global__ void compact_pairs(const int *picked, int np, Candidates c, const int *local, const int *vlabel,
                              const int *rank, PairList out, int *counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int p = picked[i];
  out.cx[i] = local[c.a[p]];
  out.cy[i] = local[c.b[p]];
  out.d[i] = c.d[p];
  out.va[i] = c.v[p];
  out.vb[i] = c.u[p];
  atomicAdd(counts + rank[vlabel[c.a[p]]], 1);
}

// The greedy fusion of one label (post_kernels.cuh:251-311, Kimimaro's join_close_components).
__global__ void join_fuse(int nm, const long long *ps, const long long *cs, const double *reach, PairList pl,
                          const float *radii, int *alive, int *pos, int *slot, int *out_a, int *out_b, int *made_out) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= nm) return;
  const long long p0 = ps[l], p1 = ps[l + 1], c0 = cs[l];
  const int nc = int(cs[l + 1] - c0);
  int *POS = pos + c0, *SLOT = slot + c0;
  for (int k = 0; k < nc; ++k) { POS[k] = k; SLOT[k] = -1; }
  int fusions = 0, made = 0;
  for (;;) {
    long long best = -1;
    float bd = 0.0f;
    int bi = 0, bj = 0;
    for (long long p = p0; p < p1; ++p) {
      if (!alive[p]) continue;
      const double d = pl.d[p];
      if (d > double(radii[pl.va[p]] + radii[pl.vb[p]])) continue;
      const float d32 = float(d);
      int ia = POS[pl.cx[p]], ib = POS[pl.cy[p]];
      if (ia > ib) { const int t = ia; ia = ib; ib = t; }
      if (best < 0 || d32 < bd || (d32 == bd && (ia < bi || (ia == bi && ib < bj)))) {
        best = p;
        bd = d32;
        bi = ia;
        bj = ib;
      }
    }
    if (best < 0 || double(bd) > reach[l]) break;
    const int X = pl.cx[best], Y = pl.cy[best];
    out_a[c0 + made] = pl.va[best];
    out_b[c0 + made] = pl.vb[best];
    ++made;
    alive[best] = 0;
    ++fusions;
    for (long long p = p0; p < p1; ++p) {
      if (!alive[p]) continue;
      if (pl.cx[p] == Y) pl.cx[p] = X;
      if (pl.cy[p] == Y) pl.cy[p] = X;
      if (pl.cx[p] == pl.cy[p]) { alive[p] = 0; continue; }
      if (pl.cx[p] != X && pl.cy[p] != X) continue;
      const int k = pl.cx[p] == X ? pl.cy[p] : pl.cx[p];
      const int q0 = SLOT[k];
      if (q0 < 0) { SLOT[k] = int(p - p0); continue; }
      const long long q = p0 + q0;
      const int lp = min(pl.va[p], pl.vb[p]), hp = max(pl.va[p], pl.vb[p]);
      const int lq = min(pl.va[q], pl.vb[q]), hq = max(pl.va[q], pl.vb[q]);
      const bool p_wins = pl.d[p] < pl.d[q] || (pl.d[p] == pl.d[q] && (lp < lq || (lp == lq && hp < hq)));
      if (p_wins) { alive[q] = 0; SLOT[k] = int(p - p0); } else { alive[p] = 0; }
    }
    for (long long p = p0; p < p1; ++p)
      if (alive[p]) { SLOT[pl.cx[p]] = -1; SLOT[pl.cy[p]] = -1; }
    POS[X] = -fusions;
  }
  made_out[l] = made;
}

__global__ void join_keys(const int2 *edges, int m, const int *out_a, const int *out_b, int nr, const long long *cs,
                          int nm, const int *made, u64 *keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) {
    const int2 e = edges[i];
    keys[i] = (u64(unsigned(min(e.x, e.y))) << 32) | unsigned(max(e.x, e.y));
  }
  if (i < nr) {
    const int l = owner(cs, nm, i);
    u64 key = ~0ull;
    if (i - cs[l] < made[l]) key = (u64(unsigned(min(out_a[i], out_b[i]))) << 32) | unsigned(max(out_a[i], out_b[i]));
    keys[m + i] = key;
  }
}

__global__ void fill_ints(int *x, int n, int value) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = value;
}

// post.cu:589-645.
Set join_components(Context &ctx, const Set &input) {
  Set p = prune(ctx, input);
  if (!p.n() || !p.m()) return p;
  cudaStream_t st = ctx.stream();
  Cub cub_call{ctx};
  Graph g = graph_of(ctx, p);
  Buffer<int> ncomp(ctx, g.k);
  Buffer<unsigned> rbits(ctx, g.k);
  ncomp.zero();
  rbits.zero();
  label_statistics<<<blocks_for(g.n), 256, 0, st>>>(g.root.data(), g.vlabel.data(), p.r, g.n, ncomp.data(),
                                                     rbits.data());
  ++ctx.launches;
  const auto hn = ncomp.download(g.k);
  const auto hr = rbits.download(g.k);
  std::vector<int> rank(g.k, -1);
  std::vector<double> reach, bound;
  std::vector<long long> cs{0};
  int ns = 0;
  for (int l = 0; l < g.k; ++l)
    if (hn[l] > 1) {
      rank[l] = int(reach.size());
      float r;
      std::memcpy(&r, &hr[l], sizeof(float));
      const double R = std::max(2.0 * double(r), 0.0);
      reach.push_back(R);
      bound.push_back(R + 0.000001);
      cs.push_back(cs.back() + hn[l]);
      ns += int(p.voff[l + 1] - p.voff[l]);
    }
  const int nm = int(reach.size()), nr = int(cs.back());
  if (!nm) return p;
  Buffer<int> d_rank = to_device(ctx, rank);
  Buffer<double> d_bound = to_device(ctx, bound), d_reach = to_device(ctx, reach);
  Buffer<long long> d_cs = to_device(ctx, cs);
  auto seq = thrust::counting_iterator<int>(0);
  Buffer<int> ids(ctx, ns), roots(ctx, nr), nsel(ctx, 1);
  cub_call([&](void *t, size_t &b) {
    return cub::DeviceSelect::If(t, b, seq, ids.data(), nsel.data(), g.n, InMultiLabel{g.vlabel.data(), d_rank.data()},
                                 st);
  });
  cub_call([&](void *t, size_t &b) {
    return cub::DeviceSelect::If(t, b, seq, roots.data(), nsel.data(), g.n,
                                 MultiRoot{g.vlabel.data(), d_rank.data(), g.root.data()}, st);
  });
  // grid cells: stable passes by z, y, x cell and then the label's rank
  Buffer<int> order(ctx, ns), order2(ctx, ns);
  Buffer<long long> key(ctx, ns), key2(ctx, ns);
  iota<<<blocks_for(ns), 256, 0, st>>>(order.data(), ns);
  ++ctx.launches;
  for (int axis : {2, 1, 0, 3}) {
    cell_pass_keys<<<blocks_for(ns), 256, 0, st>>>(ids.data(), order.data(), ns, p.v, g.vlabel.data(), d_rank.data(),
                                                   d_bound.data(), axis, key.data());
    ++ctx.launches;
    cub_call([&](void *t, size_t &b) {
      return cub::DeviceRadixSort::SortPairs(t, b, key.data(), key2.data(), order.data(), order2.data(), ns, 0, 64, st);
    });
    std::swap(order, order2);
  }
  Buffer<int> kl(ctx, ns), gid(ctx, ns), comp(ctx, ns);
  Buffer<long long> kx(ctx, ns), ky(ctx, ns), kz(ctx, ns);
  Buffer<float> xyz(ctx, 3 * size_t(ns));
  Cells cells{kl.data(), kx.data(), ky.data(), kz.data(), xyz.data(), gid.data(), comp.data()};
  ordered_cells<<<blocks_for(ns), 256, 0, st>>>(ids.data(), order.data(), ns, p.v, g.root.data(), g.vlabel.data(),
                                                d_rank.data(), d_bound.data(), cells);
  ++ctx.launches;
  // the candidates: count, scan, write
  Buffer<long long> ccount(ctx, ns), coff(ctx, size_t(ns) + 1);
  BK_CUDA(cudaMemsetAsync(coff.data(), 0, sizeof(long long), st));
  join_scan<<<blocks_for(ns, 128), 128, 0, st>>>(ns, 0, cells, d_bound.data(), ccount.data(), nullptr, Candidates{});
  ++ctx.launches;
  cub_call([&](void *t, size_t &b) {
    return cub::DeviceScan::InclusiveSum(t, b, ccount.data(), coff.data() + 1, ns, st);
  });
  const long long total = coff.download(1, ns)[0];
  if (!total) return p;
  if (total >= INT32_MAX) throw std::invalid_argument("join candidates exceed int32 capacity");
  const int nt = int(total);
  Buffer<int> ca(ctx, nt), cb(ctx, nt), cv(ctx, nt), cu(ctx, nt);
  Buffer<double> cd(ctx, nt);
  Candidates cand{ca.data(), cb.data(), cv.data(), cu.data(), cd.data()};
  join_scan<<<blocks_for(ns, 128), 128, 0, st>>>(ns, 1, cells, d_bound.data(), nullptr, coff.data(), cand);
  ++ctx.launches;
  // nearest candidate per pair of components
  Buffer<int> porder(ctx, nt), porder2(ctx, nt);
  Buffer<u64> pk(ctx, nt), pk2(ctx, nt);
  iota<<<blocks_for(nt), 256, 0, st>>>(porder.data(), nt);
  ++ctx.launches;
  for (int pass = 0; pass < 3; ++pass) {
    candidate_keys<<<blocks_for(nt), 256, 0, st>>>(porder.data(), nt, cand, pass, pk.data());
    ++ctx.launches;
    cub_call([&](void *t, size_t &b) {
      return cub::DeviceRadixSort::SortPairs(t, b, pk.data(), pk2.data(), porder.data(), porder2.data(), nt, 0, 64, st);
    });
    std::swap(porder, porder2);
  }
  auto first_flags = thrust::make_transform_iterator(seq, FirstOfPair{porder.data(), cand});
  cub_call([&](void *t, size_t &b) { return cub::DeviceReduce::Sum(t, b, first_flags, nsel.data(), nt, st); });
  const int np = nsel.download(1)[0];
  Buffer<int> picked(ctx, np);
  cub_call([&](void *t, size_t &b) {
    return cub::DeviceSelect::Flagged(t, b, porder.data(), first_flags, picked.data(), nsel.data(), nt, st);
  });
  Buffer<int> local(ctx, g.n), pcx(ctx, np), pcy(ctx, np), pva(ctx, np), pvb(ctx, np), pcount(ctx, nm);
  Buffer<double> pd(ctx, np);
  pcount.zero();
  root_positions<<<blocks_for(nr), 256, 0, st>>>(roots.data(), nr, g.vlabel.data(), d_rank.data(), d_cs.data(),
                                                 local.data());
  PairList pl{pcx.data(), pcy.data(), pva.data(), pvb.data(), pd.data()};
  compact_pairs<<<blocks_for(np), 256, 0, st>>>(picked.data(), np, cand, local.data(), g.vlabel.data(), d_rank.data(),
                                                pl, pcount.data());
  ctx.launches += 2;
  const auto hpc = pcount.download(nm);
  std::vector<long long> ps{0};
  for (int c : hpc) ps.push_back(ps.back() + c);
  Buffer<long long> d_ps = to_device(ctx, ps);
  Buffer<int> alive(ctx, np), pos(ctx, nr), slot(ctx, nr), made(ctx, nm), out_a(ctx, nr), out_b(ctx, nr);
  fill_ints<<<blocks_for(np), 256, 0, st>>>(alive.data(), np, 1);
  join_fuse<<<blocks_for(nm, 64), 64, 0, st>>>(nm, d_ps.data(), d_cs.data(), d_reach.data(), pl, p.r, alive.data(),
                                               pos.data(), slot.data(), out_a.data(), out_b.data(), made.data());
  ctx.launches += 2;
  BK_CUDA(cudaGetLastError());
  const auto hm = made.download(nm);
  if (*std::max_element(hm.begin(), hm.end()) == 0) return p;  // no join: the edge order stays
  Buffer<u64> keys(ctx, size_t(g.m) + nr + 1);
  join_keys<<<blocks_for(std::max(g.m, nr)), 256, 0, st>>>(g.edges.data(), g.m, out_a.data(), out_b.data(), nr,
                                                           d_cs.data(), nm, made.data(), keys.data());
  ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  return edge_result(ctx, p, g, keys, g.m + nr);
}

// ----------------------------------------------------------------------------------- output ----

Packed packed_of(Context &ctx, const Set &s) {
  Packed out;
  out.labels = s.labels;
  out.vertex_offsets = s.voff;
  out.edge_offsets = s.eoff;
  out.anisotropy = s.anisotropy;
  const size_t nv = size_t(s.n()), ne = size_t(s.m());
  out.device_vertices = std::make_shared<DeviceStorage>(nv * 3 * sizeof(float), ctx.device());
  out.device_radii = std::make_shared<DeviceStorage>(nv * sizeof(float), ctx.device());
  out.device_edges = std::make_shared<DeviceStorage>(ne * 2 * sizeof(uint32_t), ctx.device());
  cudaStream_t st = ctx.stream();
  if (nv) {
    BK_CUDA(cudaMemcpyAsync(out.device_vertices->ptr, s.v, nv * 3 * sizeof(float), cudaMemcpyDeviceToDevice, st));
    BK_CUDA(cudaMemcpyAsync(out.device_radii->ptr, s.r, nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
  }
  if (ne) BK_CUDA(cudaMemcpyAsync(out.device_edges->ptr, s.e, ne * 2 * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
  ctx.synchronize();
  return out;
}

__global__ void widen(const int *x, int n, long long *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = x[i];
}

}  // namespace

Packed post_process(Context &ctx, const Packed &input, int step, double a, double b) {
  StageClock clock(ctx);
  Set s = set_of(ctx, input);
  switch (step) {
    case kPostprocess:
      s = remove_dust(ctx, s, a);
      clock.mark("post_dust");
      s = remove_loops(ctx, s);
      clock.mark("post_loops");
      s = join_components(ctx, s);
      clock.mark("post_join");
      s = remove_ticks(ctx, s, b);
      clock.mark("post_ticks");
      s = prune(ctx, s);
      clock.mark("post_prune");
      break;
    case kRemoveDust: s = remove_dust(ctx, s, a); clock.mark("post_dust"); break;
    case kRemoveLoops: s = remove_loops(ctx, s); clock.mark("post_loops"); break;
    case kJoinComponents: s = join_components(ctx, s); clock.mark("post_join"); break;
    case kRemoveTicks: s = remove_ticks(ctx, s, a); clock.mark("post_ticks"); break;
    case kPruneUnused: s = prune(ctx, s); clock.mark("post_prune"); break;
    default: throw std::invalid_argument("unknown post-processing step");
  }
  Packed out = packed_of(ctx, s);
  clock.finish();
  return out;
}

std::shared_ptr<DeviceStorage> skeleton_components(Context &ctx, const Packed &input, size_t *count) {
  Set s = set_of(ctx, input);
  Graph g = graph_of(ctx, s);
  auto out = std::make_shared<DeviceStorage>(size_t(g.n) * sizeof(long long), ctx.device());
  if (g.n) {
    widen<<<blocks_for(g.n), 256, 0, ctx.stream()>>>(g.root.data(), g.n, static_cast<long long *>(out->ptr));
    ++ctx.launches;
  }
  BK_CUDA(cudaGetLastError());
  ctx.synchronize();
  *count = size_t(g.n);
  return out;
}

}  // namespace bk
