// Multi-label anisotropic EDT on sm_100a, three separable passes with the reference's arithmetic
// (edt_kernels.cuh:15-144 of giorgioangel/brook):
//   x: distance to the walls of each run of equal ids, from a float32 table of accumulated
//      spacings (one rounding per step); one warp per x-line, coalesced, with run starts and ends
//      found by warp max/min scans and the starts staged in shared memory;
//   y, z: float64 lower envelope of parabolas per run, stored as float32; one thread per line,
//      lines x-consecutive across a warp (coalesced), envelope stacks interleaved across lines;
//   the last pass takes the square root (background: 0).
// The reference compiles the envelope with FMA contraction; its two product-plus-height sums are
// written as explicit fused operations here, everything else rounds per operation (--fmad=false).
#include <algorithm>
#include <climits>
#include <cmath>
#include <mutex>

#include "common.cuh"
#include "kernels.hpp"

namespace bk {
namespace {

constexpr int kWarpsX = 4;
// The x pass's dynamic shared memory (kWarpsX line starts per CTA) is at most this.
constexpr size_t kEdtXMaxSmem = 200 * 1024;

// bb (here and in the envelope passes): walls beyond the line's ends, bit 0 before the first voxel,
// bit 1 after the last (a black border sets both).
__global__ void edt_x(const uint32_t *__restrict__ ids, float *__restrict__ D, Dims d, const float *__restrict__ acc,
                      int bb, int finish) {
  extern __shared__ int s_start[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long line = (long long)blockIdx.x * kWarpsX + warp;
  if (line >= (long long)d.sy * d.sz) return;
  const int sx = d.sx;
  int *start = s_start + warp * sx;
  const long long base = line * sx;
  int carry_start = 0;
  uint32_t carry_label = 0;
  for (int c0 = 0; c0 < sx; c0 += 32) {
    const int p = c0 + lane;
    const bool in = p < sx;
    const uint32_t lab = in ? ids[base + p] : 0xFFFFFFFFu;
    uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, lab, 1);
    if (lane == 0) prev = carry_label;
    int st = (in && (p == 0 || lab != prev)) ? p : -1;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int o = __shfl_up_sync(0xFFFFFFFFu, st, off);
      if (lane >= off) st = max(st, o);
    }
    st = max(st, carry_start);
    if (in) start[p] = st;
    carry_start = __shfl_sync(0xFFFFFFFFu, st, 31);
    carry_label = __shfl_sync(0xFFFFFFFFu, lab, 31);
  }
  __syncwarp();
  int carry_end = sx - 1;
  uint32_t carry_next = 0;
  for (int c0 = ((sx - 1) / 32) * 32; c0 >= 0; c0 -= 32) {
    const int p = c0 + lane;
    const bool in = p < sx;
    const uint32_t lab = in ? ids[base + p] : 0xFFFFFFFFu;
    uint32_t next = __shfl_down_sync(0xFFFFFFFFu, lab, 1);
    if (lane == 31) next = carry_next;
    int en = (in && (p == sx - 1 || lab != next)) ? p : INT_MAX;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int o = __shfl_down_sync(0xFFFFFFFFu, en, off);
      if (lane + off < 32) en = min(en, o);
    }
    en = min(en, carry_end);
    if (in) {
      const int c = start[p];
      float best = __uint_as_float(BK_INF_BITS);
      if (c > 0 || (bb & 1)) { const float dd = acc[p - c + 1]; const float v = __fmul_rn(dd, dd); if (v < best) best = v; }
      if (en < sx - 1 || (bb & 2)) { const float dd = acc[en + 1 - p]; const float v = __fmul_rn(dd, dd); if (v < best) best = v; }
      if (finish) best = lab == 0 ? 0.0f : sqrtf(best);
      D[base + p] = best;
    }
    carry_end = __shfl_sync(0xFFFFFFFFu, en, 0);
    carry_next = __shfl_sync(0xFFFFFFFFu, lab, 0);
  }
}

// Lets every edt_x launch of this device use up to kEdtXMaxSmem of dynamic shared memory. The
// limit is a process-wide attribute of the kernel: set per call to the call's own need, it races
// with other threads' launches of other extents (a launch above the limit another thread just
// set fails), so it is raised once per device to the bound every launch is checked against.
void allow_edt_x_smem() {
  static std::mutex lock;
  static bool raised[256] = {};
  int device = 0;
  BK_CUDA(cudaGetDevice(&device));
  if (device < 0 || device >= 256) throw std::invalid_argument("device index out of range");
  std::lock_guard<std::mutex> guard(lock);
  if (raised[device]) return;
  BK_CUDA(cudaFuncSetAttribute(edt_x, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEdtXMaxSmem));
  raised[device] = true;
}

// One line of the y or z pass: n voxels from `base` with `stride`. Stacks V/H/Z are interleaved:
// entry k of this thread's stack is at [k * pitch]. One streaming sweep: ids and heights are read
// four voxels ahead of use (independent loads, so their latency overlaps the envelope work), a run
// ends where the id changes, and the top of the stack is kept in registers, so that only a pop
// reads the stack back from memory. The envelope is the reference's per run: parabolas are
// placed in order with the same float64 operations, and the fill walks the stack forward.
__device__ void envelope_line(const uint32_t *__restrict__ ids, float *__restrict__ D, long long base, long long stride,
                              int n, float w, int bb, int *V, float *H, double *Z, long long pitch, int finish) {
  const double w2 = (double)__fmul_rn(w, w);
  const float kInf = __uint_as_float(BK_INF_BITS);
  int c = 0;        // first voxel of the current run
  uint32_t L = 0;   // its id
  int k = -1;       // stack top (-1: empty)
  int vt = 0;       // the top entry, also in memory
  float ht = 0.0f;
  double zt = 0.0;
  auto push = [&](int at, int v, float h, double z) {
    V[(long long)at * pitch] = v; H[(long long)at * pitch] = h; Z[(long long)at * pitch] = z;
    vt = v; ht = h; zt = z;
  };
  // the parabola of height ph at p joins the lower envelope
  auto place = [&](int p, double ph) {
    while (k >= 0) {
      const double num = __dsub_rn(__fma_rn(__dmul_rn(w2, (double)p), (double)p, ph),
                                   __fma_rn(__dmul_rn(w2, (double)vt), (double)vt, (double)ht));
      const double sv = __ddiv_rn(num, __dmul_rn(__dmul_rn(2.0, w2), __dsub_rn((double)p, (double)vt)));
      if (sv <= zt) {
        if (--k >= 0) {
          vt = V[(long long)k * pitch]; ht = H[(long long)k * pitch]; zt = Z[(long long)k * pitch];
        }
      } else {
        ++k;
        push(k, p, (float)ph, sv);
        return;
      }
    }
    k = 0;
    push(0, p, (float)ph, -1e300);
  };
  // the run [c, e] ends; rightw: a wall follows it
  auto finish_run = [&](int e, bool rightw) {
    if (L == 0) {
      if (finish)
        for (int q = c; q <= e; ++q) D[base + (long long)q * stride] = 0.0f;
      return;
    }
    if (rightw) place(e + 1, 0.0);
    if (k < 0) {
      for (int q = c; q <= e; ++q) D[base + (long long)q * stride] = kInf;
      return;
    }
    // entry kk serves the voxels q up to Z[kk + 1] (the last entry: the rest); the next entry is
    // read while this one's voxels are written
    int q = c;
    int vk = V[0];
    float hk = H[0];
    double zn = k > 0 ? Z[pitch] : 0.0;
    for (int kk = 0; q <= e; ++kk) {
      int vn = 0;
      float hn = 0.0f;
      double znn = 0.0;
      if (kk < k) {
        vn = V[(long long)(kk + 1) * pitch];
        hn = H[(long long)(kk + 1) * pitch];
        if (kk + 1 < k) znn = Z[(long long)(kk + 2) * pitch];
      }
      for (; q <= e && (kk == k || !(zn < (double)q)); ++q) {
        const double dq = __dsub_rn((double)q, (double)vk);
        float v = __double2float_rn(__fma_rn(__dmul_rn(w2, dq), dq, (double)hk));
        if (finish) v = sqrtf(v);
        D[base + (long long)q * stride] = v;
      }
      vk = vn; hk = hn; zn = znn;
    }
  };
  auto step = [&](int p, uint32_t lab, float hf) {
    if (p == 0 || lab != L) {
      if (p > 0) finish_run(p - 1, true);
      c = p;
      L = lab;
      k = -1;
      if (L != 0 && (c > 0 || (bb & 1))) { k = 0; push(0, c - 1, 0.0f, -1e300); }
    }
    if (L != 0 && hf < kInf) place(p, (double)hf);
  };
  auto id_at = [&](int p) { return p < n ? ids[base + (long long)p * stride] : 0u; };
  auto d_at = [&](int p) { return p < n ? D[base + (long long)p * stride] : 0.0f; };
  uint32_t a0 = id_at(0), a1 = id_at(1), a2 = id_at(2), a3 = id_at(3);
  float f0 = d_at(0), f1 = d_at(1), f2 = d_at(2), f3 = d_at(3);
  for (int p = 0; p < n; p += 4) {
    const uint32_t b0 = id_at(p + 4), b1 = id_at(p + 5), b2 = id_at(p + 6), b3 = id_at(p + 7);
    const float g0 = d_at(p + 4), g1 = d_at(p + 5), g2 = d_at(p + 6), g3 = d_at(p + 7);
    step(p, a0, f0);
    if (p + 1 < n) step(p + 1, a1, f1);
    if (p + 2 < n) step(p + 2, a2, f2);
    if (p + 3 < n) step(p + 3, a3, f3);
    a0 = b0; a1 = b1; a2 = b2; a3 = b3;
    f0 = g0; f1 = g1; f2 = g2; f3 = g3;
  }
  finish_run(n - 1, (bb & 2) != 0);
}

// Line `line` of the y (axis 1) or z (axis 2) pass of a (sx, sy, sz) volume at `offset`.
__device__ __forceinline__ bool line_of(long long line, long long offset, Dims d, int axis, long long &base,
                                        long long &stride, int &n) {
  const long long x = line % d.sx, rest = line / d.sx;
  if (axis == 1) {
    if (rest >= d.sz) return false;
    base = offset + x + (long long)d.sx * d.sy * rest; stride = d.sx; n = d.sy;
  } else {
    if (rest >= d.sy) return false;
    base = offset + x + (long long)d.sx * rest; stride = (long long)d.sx * d.sy; n = d.sz;
  }
  return true;
}

__global__ void edt_envelope(const uint32_t *__restrict__ ids, float *__restrict__ D, Dims d, int axis, float w, int bb,
                             long long line0, long long nbatch, int *__restrict__ Vs, float *__restrict__ Hs,
                             double *__restrict__ Zs, int finish) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= nbatch) return;
  long long base, stride;
  int n;
  if (!line_of(line0 + tid, 0, d, axis, base, stride, n)) return;
  envelope_line(ids, D, base, stride, n, w, bb, Vs + tid, Hs + tid, Zs + tid, nbatch, finish);
}

// The y pass of a stack of 2D images in groups of `per_group` slices, each group with its own
// spacing w[group] (the border targets' face stack: one group per axis pair).
struct GroupSpacing {
  float w[3];
};
__global__ void edt_envelope_groups(const uint32_t *__restrict__ ids, float *__restrict__ D, Dims d, GroupSpacing gs,
                                    int per_group, int bb, long long line0, long long nbatch, int *__restrict__ Vs,
                                    float *__restrict__ Hs, double *__restrict__ Zs) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= nbatch) return;
  long long base, stride;
  int n;
  const long long line = line0 + tid;
  if (!line_of(line, 0, d, 1, base, stride, n)) return;
  const int group = int((line / d.sx) / per_group);
  envelope_line(ids, D, base, stride, n, gs.w[group], bb, Vs + tid, Hs + tid, Zs + tid, nbatch, 1);
}

// The y or z pass of several volumes of one flat index space in one launch: volume v's lines are
// [line_begin[v], line_begin[v + 1]) of the launch's line space.
struct EnvelopeVolume {
  long long offset, line_begin;
  int sx, sy, sz, bb;
};

__global__ void edt_envelope_volumes(const uint32_t *__restrict__ ids, float *__restrict__ D,
                                     const EnvelopeVolume *__restrict__ vols, int nvol, int axis, float w,
                                     long long line0, long long nbatch, int *__restrict__ Vs, float *__restrict__ Hs,
                                     double *__restrict__ Zs, int finish) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (tid >= nbatch) return;
  const long long line = line0 + tid;
  int lo = 0, hi = nvol - 1;  // the last volume whose first line is <= line
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (vols[mid].line_begin <= line) lo = mid; else hi = mid - 1;
  }
  const EnvelopeVolume v = vols[lo];
  long long base, stride;
  int n;
  if (!line_of(line - v.line_begin, v.offset, Dims{v.sx, v.sy, v.sz}, axis, base, stride, n)) return;
  envelope_line(ids, D, base, stride, n, w, v.bb, Vs + tid, Hs + tid, Zs + tid, nbatch, finish);
}

}  // namespace

void edt(Context &ctx, const uint32_t *ids, VolumeDims vd, const float aniso[3], bool black_border, int dims,
         float *D) {
  const Dims d{vd.sx, vd.sy, vd.sz};
  const long long n = vd.n();
  if (!n) return;
  for (int a = 0; a < 3; ++a)
    if (!(aniso[a] > 0) || !std::isfinite(aniso[a])) throw std::invalid_argument("anisotropy must be finite and positive");
  if (dims < 2 && (vd.sy != 1 || vd.sz != 1)) throw std::invalid_argument("1D EDT of a volume");
  cudaStream_t s = ctx.stream();
  // x pass
  std::vector<float> acc(vd.sx + 2, 0.0f);
  for (size_t k = 1; k < acc.size(); ++k) acc[k] = acc[k - 1] + aniso[0];
  Buffer<float> dacc = to_device(ctx, acc);
  const size_t smem = size_t(kWarpsX) * vd.sx * sizeof(int);
  if (smem > kEdtXMaxSmem) throw std::invalid_argument("x extent too large for the EDT x pass");
  allow_edt_x_smem();
  const long long xlines = (long long)vd.sy * vd.sz;
  const bool only_x = dims == 1 || (vd.sy == 1 && vd.sz == 1 && dims == 1);
  edt_x<<<(unsigned)((xlines + kWarpsX - 1) / kWarpsX), kWarpsX * 32, smem, s>>>(ids, D, d, dacc.data(),
                                                                                black_border ? 3 : 0, only_x ? 1 : 0); ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  for (int axis = 1; axis < dims; ++axis) {
    const int len = axis == 1 ? vd.sy : vd.sz;
    const long long lines = axis == 1 ? (long long)vd.sx * vd.sz : (long long)vd.sx * vd.sy;
    const long long budget = 4LL << 30;  // bytes of envelope stacks per batch
    long long batch = std::max(1LL, std::min(lines, budget / (16LL * (len + 3))));
    Buffer<int> V(ctx, batch * (len + 3));
    Buffer<float> H(ctx, batch * (len + 3));
    Buffer<double> Z(ctx, batch * (len + 3));
    const int last = axis == dims - 1;
    for (long long l0 = 0; l0 < lines; l0 += batch) {
      const long long nb = std::min(batch, lines - l0);
      edt_envelope<<<blocks_for(nb, 128), 128, 0, s>>>(ids, D, d, axis, aniso[axis], black_border ? 3 : 0, l0, nb,
                                                      V.data(), H.data(), Z.data(), last); ++ctx.launches;
      BK_CUDA(cudaGetLastError());
    }
  }
}

void edt_xy_squared(Context &ctx, const uint32_t *ids, VolumeDims vd, const float aniso[3], bool black_border, float *D) {
  const Dims d{vd.sx, vd.sy, vd.sz};
  if (!vd.n()) return;
  cudaStream_t s = ctx.stream();
  std::vector<float> acc(vd.sx + 2, 0.0f);
  for (size_t k = 1; k < acc.size(); ++k) acc[k] = acc[k - 1] + aniso[0];
  Buffer<float> dacc = to_device(ctx, acc);
  const size_t smem = size_t(kWarpsX) * vd.sx * sizeof(int);
  if (smem > kEdtXMaxSmem) throw std::invalid_argument("x extent too large for the EDT x pass");
  allow_edt_x_smem();
  const long long xlines = (long long)vd.sy * vd.sz;
  edt_x<<<(unsigned)((xlines + kWarpsX - 1) / kWarpsX), kWarpsX * 32, smem, s>>>(ids, D, d, dacc.data(),
                                                                                black_border ? 3 : 0, 0);
  ++ctx.launches;
  BK_CUDA(cudaGetLastError());
  const long long lines = (long long)vd.sx * vd.sz;
  const long long batch = std::max(1LL, std::min(lines, (4LL << 30) / (16LL * (vd.sy + 3))));
  Buffer<int> V(ctx, batch * (vd.sy + 3));
  Buffer<float> H(ctx, batch * (vd.sy + 3));
  Buffer<double> Z(ctx, batch * (vd.sy + 3));
  for (long long l0 = 0; l0 < lines; l0 += batch) {
    const long long nb = std::min(batch, lines - l0);
    edt_envelope<<<blocks_for(nb, 128), 128, 0, s>>>(ids, D, d, 1, aniso[1], black_border ? 3 : 0, l0, nb, V.data(),
                                                    H.data(), Z.data(), 0);
    ++ctx.launches;
    BK_CUDA(cudaGetLastError());
  }
}

void edt_z_finish(Context &ctx, const uint32_t *ids, VolumeDims vd, float wz, bool black_border, float *D) {
  const Dims d{vd.sx, vd.sy, vd.sz};
  if (!vd.n()) return;
  cudaStream_t s = ctx.stream();
  const long long lines = (long long)vd.sx * vd.sy;
  const long long batch = std::max(1LL, std::min(lines, (4LL << 30) / (16LL * (vd.sz + 3))));
  Buffer<int> V(ctx, batch * (vd.sz + 3));
  Buffer<float> H(ctx, batch * (vd.sz + 3));
  Buffer<double> Z(ctx, batch * (vd.sz + 3));
  for (long long l0 = 0; l0 < lines; l0 += batch) {
    const long long nb = std::min(batch, lines - l0);
    edt_envelope<<<blocks_for(nb, 128), 128, 0, s>>>(ids, D, d, 2, wz, black_border ? 3 : 0, l0, nb, V.data(),
                                                    H.data(), Z.data(), 1);
    ++ctx.launches;
    BK_CUDA(cudaGetLastError());
  }
}

void edt_planes(Context &ctx, const uint32_t *ids, int W, int H, int groups, int per_group, const float wx[3],
                const float wy[3], float *D) {
  if (groups < 1 || groups > 3 || per_group < 1) throw std::invalid_argument("planar EDT groups out of range");
  const long long slice = (long long)W * H, S = (long long)groups * per_group;
  if (!slice) return;
  cudaStream_t s = ctx.stream();
  const size_t smem = size_t(kWarpsX) * W * sizeof(int);
  if (smem > kEdtXMaxSmem) throw std::invalid_argument("x extent too large for the EDT x pass");
  allow_edt_x_smem();
  // x passes, one per group (its spacing table)
  for (int g = 0; g < groups; ++g) {
    std::vector<float> acc(W + 2, 0.0f);
    for (size_t k = 1; k < acc.size(); ++k) acc[k] = acc[k - 1] + wx[g];
    Buffer<float> dacc = to_device(ctx, acc);
    const long long lines = (long long)H * per_group;
    edt_x<<<(unsigned)((lines + kWarpsX - 1) / kWarpsX), kWarpsX * 32, smem, s>>>(
        ids + slice * per_group * g, D + slice * per_group * g, Dims{W, H, per_group}, dacc.data(), 3, 0);
    ++ctx.launches;
  }
  BK_CUDA(cudaGetLastError());
  // the y pass of every group in one launch
  const long long lines = (long long)W * S;
  const long long budget = 4LL << 30;
  const long long batch = std::max(1LL, std::min(lines, budget / (16LL * (H + 3))));
  Buffer<int> V(ctx, batch * (H + 3));
  Buffer<float> Hb(ctx, batch * (H + 3));
  Buffer<double> Z(ctx, batch * (H + 3));
  GroupSpacing gs{{wy[0], groups > 1 ? wy[1] : 0.0f, groups > 2 ? wy[2] : 0.0f}};
  for (long long l0 = 0; l0 < lines; l0 += batch) {
    const long long nb = std::min(batch, lines - l0);
    edt_envelope_groups<<<blocks_for(nb, 128), 128, 0, s>>>(ids, D, Dims{W, H, int(S)}, gs, per_group, 3, l0, nb,
                                                            V.data(), Hb.data(), Z.data());
    ++ctx.launches;
    BK_CUDA(cudaGetLastError());
  }
}

// The walls of a volume's lines along `axis`: bit 0 the low end, bit 1 the high end.
static int walls(const EdtVolume &v, int axis) {
  if (v.faces < 0) return v.black_border ? 3 : 0;
  return (v.faces >> (2 * axis)) & 3;
}

void edt_volumes(Context &ctx, const uint32_t *ids, const std::vector<EdtVolume> &vols, const float aniso[3], float *D) {
  if (vols.empty()) return;
  for (int a = 0; a < 3; ++a)
    if (!(aniso[a] > 0) || !std::isfinite(aniso[a])) throw std::invalid_argument("anisotropy must be finite and positive");
  cudaStream_t s = ctx.stream();
  int maxx = 1;
  for (const auto &v : vols) maxx = std::max(maxx, v.d.sx);
  // x pass, volume by volume (a warp per line fills the GPU on its own), one spacing table
  std::vector<float> acc(maxx + 2, 0.0f);
  for (size_t k = 1; k < acc.size(); ++k) acc[k] = acc[k - 1] + aniso[0];
  Buffer<float> dacc = to_device(ctx, acc);
  const size_t smem = size_t(kWarpsX) * maxx * sizeof(int);
  if (smem > kEdtXMaxSmem) throw std::invalid_argument("x extent too large for the EDT x pass");
  allow_edt_x_smem();
  for (const auto &v : vols) {
    if (!v.d.n()) continue;
    const long long xlines = (long long)v.d.sy * v.d.sz;
    edt_x<<<(unsigned)((xlines + kWarpsX - 1) / kWarpsX), kWarpsX * 32, smem, s>>>(
        ids + v.offset, D + v.offset, Dims{v.d.sx, v.d.sy, v.d.sz}, dacc.data(), walls(v, 0), 0);
    ++ctx.launches;
  }
  BK_CUDA(cudaGetLastError());
  // y and z passes: every volume's lines in one launch (a thread per line)
  for (int axis = 1; axis <= 2; ++axis) {
    std::vector<EnvelopeVolume> table;
    long long lines = 0;
    int len = 1;
    for (const auto &v : vols) {
      if (!v.d.n()) continue;
      table.push_back({v.offset, lines, v.d.sx, v.d.sy, v.d.sz, walls(v, axis)});
      lines += axis == 1 ? (long long)v.d.sx * v.d.sz : (long long)v.d.sx * v.d.sy;
      len = std::max(len, axis == 1 ? v.d.sy : v.d.sz);
    }
    if (!lines) continue;
    Buffer<EnvelopeVolume> dtable = to_device(ctx, table);
    const long long budget = 4LL << 30;  // bytes of envelope stacks per launch
    const long long batch = std::max(1LL, std::min(lines, budget / (16LL * (len + 3))));
    Buffer<int> V(ctx, batch * (len + 3));
    Buffer<float> H(ctx, batch * (len + 3));
    Buffer<double> Z(ctx, batch * (len + 3));
    for (long long l0 = 0; l0 < lines; l0 += batch) {
      const long long nb = std::min(batch, lines - l0);
      edt_envelope_volumes<<<blocks_for(nb, 128), 128, 0, s>>>(ids, D, dtable.data(), int(table.size()), axis,
                                                              aniso[axis], l0, nb, V.data(), H.data(), Z.data(),
                                                              axis == 2 ? 1 : 0);
      ++ctx.launches;
      BK_CUDA(cudaGetLastError());
    }
  }
}

// ---------------------------------------------------------------------------------------------
// The EDT with a fixed device scratch, for callers that cannot allocate device memory: code that
// runs inside another framework's memory budget (a caching allocator or a pre-reserved pool that
// owns the device's free memory), code on a path where an allocation would synchronise the device
// or fail under memory pressure at the worst moment, and embedded callers that keep a fixed
// device-memory footprint. The envelope stacks and the spacing table live in one file-scope
// device array of kFixedScratchBytes (32 MiB) that every GPU loading this library holds until the
// process exits; nothing is allocated per call.
namespace {

constexpr size_t kFixedScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_edt_scratch[kFixedScratchBytes];

// acc[k] = the spacing added k times in float32, one rounding per step (the host loop of edt()).
__global__ void spacing_table(float *acc, int n, float w) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  float a = 0.0f;
  acc[0] = a;
  for (int k = 1; k < n; ++k) {
    a = __fadd_rn(a, w);
    acc[k] = a;
  }
}

std::mutex g_scratch_mutex;
void *g_scratch_address[256];

// The device address of g_edt_scratch on the current device. Host code cannot use the array's
// name as a device address (it is a host-side stand-in), so the address is looked up once per
// device, with that device current, and cached.
void *fixed_scratch() {
  int device = 0;
  BK_CUDA(cudaGetDevice(&device));
  if (device < 0 || device >= 256) throw std::invalid_argument("device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_address[device]) {
    void *p = nullptr;
    const cudaError_t status = cudaGetSymbolAddress(&p, g_edt_scratch);
    if (status != cudaSuccess) {
      cudaGetLastError();
      throw CudaError(status, "cudaGetSymbolAddress(EDT scratch)");
    }
    g_scratch_address[device] = p;
  }
  return g_scratch_address[device];
}

}  // namespace

size_t edt_fixed_scratch_bytes() { return kFixedScratchBytes; }

// The EDT of uint32 labels (Fortran order) into D on `stream`, using only the fixed scratch. The
// result equals edt() on the labels' component ids (runs of equal labels along a line are runs of
// one component). Nothing in the scratch must start at zero: the spacing table is rewritten by
// every call and every stack entry is written before it is read. Calls that overlap on the GPU
// (two streams, two threads) share the scratch and race.
void edt_fixed_scratch(const uint32_t *labels, VolumeDims vd, const float aniso[3], bool black_border, float *D,
                       cudaStream_t s) {
  const Dims d{vd.sx, vd.sy, vd.sz};
  const long long n = vd.n();
  if (n <= 0) return;
  for (int a = 0; a < 3; ++a)
    if (!(aniso[a] > 0) || !std::isfinite(aniso[a])) throw std::invalid_argument("anisotropy must be finite and positive");
  const size_t smem = size_t(kWarpsX) * vd.sx * sizeof(int);
  const size_t table = (size_t(vd.sx + 2) * sizeof(float) + 255) / 256 * 256;
  const size_t line = 16 * size_t(std::max(vd.sy, vd.sz) + 3);
  if (smem > kEdtXMaxSmem || table + line > kFixedScratchBytes)
    throw std::invalid_argument("volume too large for the EDT's fixed 32 MiB scratch (x extent at most 12800 and "
                                "16 * (max(y, z) extent + 3) + 4 * (x extent + 2) bytes within it)");
  unsigned char *base = static_cast<unsigned char *>(fixed_scratch());
  float *acc = reinterpret_cast<float *>(base);
  spacing_table<<<1, 1, 0, s>>>(acc, vd.sx + 2, aniso[0]);
  BK_CUDA(cudaGetLastError());
  allow_edt_x_smem();
  const long long xlines = (long long)vd.sy * vd.sz;
  edt_x<<<(unsigned)((xlines + kWarpsX - 1) / kWarpsX), kWarpsX * 32, smem, s>>>(labels, D, d, acc,
                                                                                black_border ? 3 : 0, 0);
  BK_CUDA(cudaGetLastError());
  for (int axis = 1; axis < 3; ++axis) {
    const int len = axis == 1 ? vd.sy : vd.sz;
    const long long lines = axis == 1 ? (long long)vd.sx * vd.sz : (long long)vd.sx * vd.sy;
    const long long room = (long long)((kFixedScratchBytes - table) / (16 * size_t(len + 3)));
    const long long batch = std::max(1LL, std::min(lines, room));
    // stacks of one batch: Z (8 bytes per entry, 256-aligned after the table), then V, then H
    double *Z = reinterpret_cast<double *>(base + table);
    int *V = reinterpret_cast<int *>(Z + batch * (len + 3));
    float *H = reinterpret_cast<float *>(V + batch * (len + 3));
    for (long long l0 = 0; l0 < lines; l0 += batch) {
      const long long nb = std::min(batch, lines - l0);
      edt_envelope<<<blocks_for(nb, 128), 128, 0, s>>>(labels, D, d, axis, aniso[axis], black_border ? 3 : 0, l0, nb,
                                                      V, H, Z, axis == 2);
      BK_CUDA(cudaGetLastError());
    }
  }
}

}  // namespace bk
