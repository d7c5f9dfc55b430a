// The object engine: persistent kernels in which one CTA owns one object at a time (objects are
// pulled from a queue, largest first) and runs that object's whole sequential chain inside the
// CTA, so that every round of a flood costs a block barrier instead of a grid barrier:
//   prepare: root search flood + argmax, DAF flood + argmax, the object's PDRF, its root rail;
//   trace:   target, railroad flood, warp backtrace with the dijkstra3d join, claim-order
//            invalidation, rails, repeated until the object has no alive voxel left.
// Objects never read or write another object's voxels (every step is gated by the same-id
// neighbour mask), so concurrent CTAs need no synchronisation with one another.
#pragma once
#include <cstdint>

namespace bk {

constexpr int kEngineThreads = 512;  // threads per CTA

// Per-voxel flag bits (uint32 per voxel, 0 at rest).
constexpr unsigned kNearQueued = 1u;   // railroad / flood: in the next near list
constexpr unsigned kFarQueued = 2u;    // railroad: on the far list
constexpr unsigned kFront = 4u;        // invalidation: in the next frontier
constexpr unsigned kWaiting = 8u;      // invalidation: on the waiting list
constexpr unsigned kOnPath = 16u;      // without fix_branching: on a stored path of the object

enum EngineStatus : int {
  kOk = 0,
  kBudget = 1,        // a loop bound was reached (never expected; guards against hangs)
  kNoRail = 2,        // no rail reachable from a target
  kStoreFull = 3,     // path store region exhausted (cannot happen on a valid field)
  kRecordsFull = 4,
};

struct EngineArgs {
  // Arenas: volumes laid end to end in one flat index space (one arena per volume of a batch).
  // Arena r starts at arena_offset[r] and has shape arena_dims[3r .. 3r+2]; a voxel's neighbours
  // never leave its arena (the neighbour mask says so).
  const int *arena_offset, *arena_dims;
  const int *obj_arena;  // per object
  const uint32_t *mask;  // same-id neighbour mask per voxel
  const float *dbf;
  float *pdrf;           // penalty; rails are 0
  float *dist;           // railroad distances, +inf at rest
  float *daf;            // DAF, +inf before prepare
  uint32_t *flags;       // 0 at rest
  uint8_t *alive;
  unsigned long long *key;  // invalidation keys, all ones at rest

  int nobj;
  const int *obj_begin;  // offset of the object's voxels in vox and in the list pool
  const int *obj_count;
  const int *vox;        // voxels of every object, ascending flat index
  const int *schedule;   // processing order (object indices): large objects first, then the rest
  int nbig;              // schedule[0, nbig) run on clusters (set by launch_prepare / launch_trace)
  int lone_first;        // trace: clusters [0, lone_first) take the small objects first
  int *queue;            // two work counters (large, small), both 0 at launch
  int *status;           // per object
  int *lists;            // 5 lists of F ints: list w of object o at lists + w * F + obj_begin[o]
  unsigned long long *wide;  // F entries: object o at wide + obj_begin[o] (per-entry staging)
  unsigned long long *side;  // 2F entries: two more staging arrays (packed coordinates)
  long long F;

  // prepare
  const int *border_root;  // per object: flat index, or -1 (search)
  const float *M;          // per object: float(1 / dbf_max^1.01)
  float pdrf_scale;
  int squarings;           // the exponent is 2^squarings; -1: any other exponent (powf)
  float exponent;
  // fix_branching: each path runs to the nearest rail (the root, then every earlier path). Without
  // it, one SSSP from the root over the PDRF is kept for the object's whole trace and each path
  // walks from its target to the root (trace.cu:151-160, batched_regular.inc:113-152).
  int fix_branching;
  // somata (trace.cu:98-131): per object the free-space radius of its DAF seed (the DBF maximum;
  // 0: none) and the soma radius its paths are trimmed to (< 0: not a soma); the soma's own ball is
  // invalidated first with soma_scale / soma_constant as the reach
  const float *free_radius;
  const double *soma_radius;
  float soma_scale, soma_constant;
  float w[26];             // geometric step weights
  int *root, *target;
  float *max_daf;

  // trace
  const int *order;            // target order of every object at obj_begin
  const int *manual_begin, *manual_count, *manual;  // manual targets in pop order
  const int *after_begin, *after_count, *after;     // targets once no voxel is alive, in pop order
  const long long *max_paths;
  int *store;                  // path vertices, target first
  const long long *store_begin, *store_cap;
  int *rec_start, *rec_len;    // per path: offset in the object's store region, length
  const long long *rec_begin, *rec_cap;
  int *npaths, *nstore;
  // work counters (added over all objects): [0] voxels a railroad settled (distance <= its rail's),
  // [1] voxels a railroad touched, [2] voxels invalidated, [3] paths
  unsigned long long *work;
  // per object (8 entries, nanoseconds of %globaltimer): start, end, time in target search,
  // railroad, backtrace, invalidation; railroad rounds; invalidation rounds
  unsigned long long *profile;
  float wx, wy, wz, scale, constant, delta;
  // A lower cap on the round bounds of every flood (0: none). The bounds guard against a loop
  // that does not end; the cap lets a test make one run out and check that the call fails with
  // kBudget and leaves the device usable.
  long long round_limit;
  // The railroad's band past the nearest deferred voxel: its distance plus rail_band times its
  // penalty (at least 5e-4 of the distance). Any band gives the same distances; wider bands take
  // fewer band ends and more re-relaxations.
  float rail_band;
  // The share (percent) of the device's resident clusters the persistent launches take: below 100
  // they leave CTA slots free for another stream's kernels (a second batch's preamble).
  int grid_percent;
};

// Objects with at least kPrepareClusterVoxels voxels (preparation) or more voxels than
// trace_cluster_voxels (tracing) run on a cluster of CTAs that share the object's frontiers
// through distributed shared memory; smaller objects on one CTA each. Tracing keeps clusters for
// the objects whose lone-CTA chain would outlast the kernel's even share of the work: a cluster
// spends more CTA-time per object than a lone CTA, which pays only where the object's own chain
// would otherwise set the kernel's length. Clusters have kClusterCtas CTAs, or kWideClusterCtas
// when the largest object holds at least 1/kWideClusterShare of the foreground (its chain is
// then the kernel's length whatever else runs beside it).
constexpr int kClusterCtas = 4;
constexpr int kWideClusterCtas = 8;
constexpr long long kWideClusterShare = 16;
int cluster_ctas(long long largest, long long foreground);
constexpr int kPrepareClusterVoxels = 8192;
constexpr long long kTraceClusterFloor = 16384;
// Half the foreground voxels per resident engine CTA (largest-first scheduling then leaves the
// clusters' objects as the only ones longer than a CTA's share), at least kTraceClusterFloor.
long long trace_cluster_voxels(long long foreground);

// One pass of the engine: clusters take schedule[0, nbig) (large objects, largest first), then
// every CTA takes schedule[nbig, nobj) alone. queue[0] and queue[1] must be zero.
void launch_prepare(const EngineArgs &a, int nbig, int cluster_ctas, cudaStream_t stream);
// lone_percent: the share of clusters (percent) whose CTAs take small objects first.
void launch_trace(const EngineArgs &a, int nbig, int cluster_ctas, int lone_percent, cudaStream_t stream);
constexpr int kLoneFirstPercent = 10;
// The railroad band's width in penalties of the nearest deferred voxel (EngineArgs::rail_band).
// Measured on the 512^3 dense workload (trace ms): 0.1 69.8, 0.25 59.0, 0.5 56.1, 1 58.4, 2 60.6,
// 4 66.8, 8 80.6, 16 117.7; narrower bands take more band ends, wider ones more re-relaxations.
constexpr float kRailBand = 0.5f;
// The device queries the launches above make (resident clusters per kernel), done ahead so that
// a stream capture of the launches holds launches only.
void prepare_engine_launches(int prepare_cluster_ctas, int trace_cluster_ctas, cudaStream_t stream);

}  // namespace bk
