/* brook_b200 C ABI: the skeletonization entry points of giorgioangel/brook's C SDK
 * (cpp/include/brook/brook.h), implemented for NVIDIA B200 (sm_100a).
 *
 * Structures, enumerations and function names are the reference's, so that a consumer of the
 * reference's C API for this path links against libbrook_b200.so instead. Every declaration below
 * names the reference declaration it replaces. Calls block; errors return a brook_status and
 * brook_last_error() holds the text (thread-local, valid until the next call on that thread).
 * Volumes are indexed (x, y, z) with byte strides; the library works on Fortran-ordered copies.
 */
#ifndef BROOK_B200_H
#define BROOK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* brook.h:15 */
#define BROOK_ABI_VERSION 1u

typedef struct brook_context brook_context;     /* brook.h:17 */
typedef struct brook_array brook_array;         /* brook.h:18 */
typedef struct brook_components brook_components; /* brook.h:19 */
typedef struct brook_skeletons brook_skeletons; /* brook.h:21 */
typedef struct brook_host_components brook_host_components; /* brook.h:20 */
/* brook.h:22-24: include brook_b200_dlpack.h (or the standard dlpack/dlpack.h) to read the
 * exported tensors' fields. */
typedef struct DLManagedTensor DLManagedTensor;
typedef struct DLManagedTensorVersioned DLManagedTensorVersioned;

/* brook.h:26-29 */
typedef enum brook_status {
  BROOK_SUCCESS = 0, BROOK_INVALID_ARGUMENT = 1, BROOK_OUT_OF_MEMORY = 2,
  BROOK_CUDA_ERROR = 3, BROOK_INTERNAL_ERROR = 4
} brook_status;

/* brook.h:31-35 */
typedef enum brook_dtype {
  BROOK_U8 = 0, BROOK_U16 = 1, BROOK_U32 = 2, BROOK_U64 = 3,
  BROOK_I8 = 4, BROOK_I16 = 5, BROOK_I32 = 6, BROOK_I64 = 7,
  BROOK_F32 = 8, BROOK_F64 = 9
} brook_dtype;

/* brook.h:37 */
typedef enum brook_memory { BROOK_HOST = 0, BROOK_DEVICE = 1 } brook_memory;

/* brook.h:42-50: data points to logical (0,0,0); byte strides (host strides may be negative).
 * Zero-initialize and set struct_size/abi_version. Input is borrowed for the call; device input
 * must be on the context's device and ready before the call. */
typedef struct brook_volume {
  size_t struct_size;
  uint32_t abi_version;
  const void *data;
  int64_t shape[3];
  int64_t strides[3];
  brook_dtype dtype;
  brook_memory memory;
} brook_volume;

/* brook.h:52-58 */
typedef struct brook_teasar_parameters {
  double scale, constant, pdrf_scale, pdrf_exponent;
  double soma_detection_threshold, soma_acceptance_threshold;
  double soma_invalidation_scale, soma_invalidation_const;
  int64_t max_paths;
  uint32_t has_max_paths;
} brook_teasar_parameters;

/* brook.h:60-67 */
enum brook_skeletonize_flags {
  BROOK_FIX_BRANCHING = 1u, BROOK_FIX_BORDERS = 2u, BROOK_FILTER_OBJECTS = 4u,
  BROOK_DEVICE_OUTPUT = 8u, BROOK_FILL_HOLES = 16u, BROOK_FIX_AVOCADOS = 32u
};

/* brook.h:68-84 */
typedef struct brook_skeletonize_options {
  size_t struct_size;
  uint32_t abi_version;
  brook_teasar_parameters teasar;
  float anisotropy[3];
  double dust_threshold;
  uint32_t flags;
  const int64_t *object_ids;
  size_t object_ids_count;
  const int64_t *targets_before;
  size_t targets_before_count;
  const int64_t *targets_after;
  size_t targets_after_count;
  const brook_volume *voxel_graph;
} brook_skeletonize_options;

/* brook.h:86-95: host packed result. Offsets have skeleton_count+1 entries; edge indices are
 * local to each skeleton; vertices row major, physical coordinates. */
typedef struct brook_skeletons_view {
  size_t skeleton_count, vertex_count, edge_count;
  const int64_t *labels, *vertex_offsets, *edge_offsets;
  const float *vertices;
  const uint32_t *edges;
  const float *radii;
  float anisotropy[3];
} brook_skeletons_view;

/* brook.h:96-101: a result made with BROOK_DEVICE_OUTPUT. Labels and offsets on the host; the
 * vertices (shape {3, vertex_count, 1}), edges ({2, edge_count, 1}) and radii ({vertex_count, 1,
 * 1}) are device arrays of the context's device, row major, owned by the result handle. */
typedef struct brook_skeletons_device_view {
  size_t skeleton_count, vertex_count, edge_count;
  const int64_t *labels, *vertex_offsets, *edge_offsets;
  brook_volume vertices, edges, radii;
  float anisotropy[3];
} brook_skeletons_device_view;

/* brook.h:102 */
typedef enum brook_skeleton_buffer { BROOK_VERTICES = 0, BROOK_EDGES = 1, BROOK_RADII = 2 } brook_skeleton_buffer;

uint32_t brook_abi_version(void);       /* brook.h:147 */
const char *brook_version(void);        /* brook.h:148 */
const char *brook_last_error(void);     /* brook.h:150 */

/* brook.h:154: device >= 0 and a Blackwell (compute capability 10.x) GPU. */
brook_status brook_context_create(int device, brook_context **out);
void brook_context_destroy(brook_context *context);              /* brook.h:155 */
brook_status brook_context_synchronize(brook_context *context);  /* brook.h:156 */
/* No counterpart in the reference. Waits for the context's stream, hands every device block the
 * context keeps for reuse back to the device's default memory pool and trims that pool, so the
 * memory returns to the driver. The next call allocates again. */
brook_status brook_context_trim(brook_context *context);
/* No counterpart in the reference. The share (percent, 1 to 100, default 100) of the device's
 * resident thread-block clusters that this context's persistent engine launches take. Below 100,
 * kernels of other contexts (another request's preamble) run beside them instead of waiting for
 * them to end; a call alone on the GPU runs faster at 100. */
brook_status brook_context_set_engine_share(brook_context *context, int percent);

/* brook.h:159-162: device arrays owned by the handle. brook_array_upload copies a volume (host
 * or device memory of the context's device, any strides, any of the ten element types) into a
 * Fortran-ordered device array of the same shape and type; the copy is complete on return. */
brook_status brook_array_upload(brook_context *context, const brook_volume *input, brook_array **out);
void brook_array_destroy(brook_array *array);
brook_status brook_array_view(const brook_array *array, brook_volume *out);
brook_status brook_array_copy_to_host(const brook_array *array, void *out, size_t bytes);
/* brook.h:163-167: zero-copy DLPack exports of an array's device storage (kDLCUDA, the array's
 * device). A volume exports as shape (x, y, z) with strides (1, x, x*y) elements; a skeleton
 * buffer as its row-major (rows, 3), (rows, 2) or (rows,) form. Each export holds its own
 * reference to the storage, so it stays valid after the array handle and the context are
 * destroyed; the consumer calls the returned tensor's deleter exactly once. The versioned form
 * reports DLPack 1.min(max_minor, 1) and no flags. */
brook_status brook_array_to_dlpack(const brook_array *array, DLManagedTensor **out);
brook_status brook_array_to_dlpack_versioned(const brook_array *array, uint32_t max_minor,
                                             DLManagedTensorVersioned **out);

/* brook.h:169-177: 26-connected components; ids 1..K by ascending first voxel (Fortran order),
 * stored in the narrowest unsigned type that holds K. */
brook_status brook_connected_components(brook_context *context, const brook_volume *labels,
                                        brook_components **out);
void brook_components_destroy(brook_components *components);
brook_status brook_components_view(const brook_components *components, brook_volume *labels,
                                   const int64_t **mapping, const int64_t **roots, size_t *count);
brook_status brook_components_copy_to_host(const brook_components *components, void *out, size_t bytes);
/* brook.h:182: the component ids as an array handle sharing the components' storage (it stays
 * valid after brook_components_destroy). */
brook_status brook_components_labels(const brook_components *components, brook_array **out);

/* brook.h:180-181: anisotropic distance to the nearest voxel of another label (float32). */
brook_status brook_edt(brook_context *context, const brook_volume *labels, const float anisotropy[3],
                       int black_border, brook_array **out);

/* brook.h:201-203: defaults of the Python skeletonize() (DEFAULT_TEASAR_PARAMS, dust 1000,
 * fix_branching and fix_borders). */
void brook_skeletonize_options_init(brook_skeletonize_options *options);
brook_status brook_skeletonize(brook_context *context, const brook_volume *labels,
                               const brook_skeletonize_options *options, brook_skeletons **out);

/* The C form of the reference's Python skeletonize_batch (src/brook/batch.py:193; its C++ form
 * brook::skeletonize_batch, batch.cu:430): `count` volumes traced in one pass of the object
 * engine; out receives `count` result handles (one per volume, in input order). */
brook_status brook_skeletonize_batch(brook_context *context, const brook_volume *volumes, size_t count,
                                     const brook_skeletonize_options *options, brook_skeletons **out);

/* Per-sample extra targets of a batch (the reference's Python skeletonize_batch takes them as one
 * sequence per sample, src/brook/batch.py:173-190, 206-220): x, y, z triples in the sample's own
 * frame, as brook_skeletonize_options' targets_before / targets_after are for one volume. */
typedef struct brook_sample_targets {
  const int64_t *before;
  size_t before_count;
  const int64_t *after;
  size_t after_count;
} brook_sample_targets;
/* brook_skeletonize_batch with targets[i] for volumes[i] (`count` entries); the options must then
 * carry no targets of their own. */
brook_status brook_skeletonize_batch_targets(brook_context *context, const brook_volume *volumes, size_t count,
                                             const brook_skeletonize_options *options,
                                             const brook_sample_targets *targets, brook_skeletons **out);

/* Makes the context's stream wait for the work queued so far on a producer's stream, without
 * blocking the host: call it before passing device memory that a kernel on another stream is
 * still writing. producer: 0 or 1 the legacy default stream, 2 the per-thread default stream,
 * anything else a cudaStream_t of the context's device (the CUDA array interface's convention).
 * The reference's Python binding does the same for every device input (fence_producer,
 * cpp/python/bindings.cpp:104-120); its C header leaves it to the caller. */
brook_status brook_context_wait_stream(brook_context *context, int64_t producer);

/* brook.h:238-252. A device result (BROOK_DEVICE_OUTPUT) is copied to the host on the first call. */
brook_status brook_skeletons_get_view(const brook_skeletons *result, brook_skeletons_view *out);
void brook_skeletons_destroy(brook_skeletons *result);
/* brook.h:232: device arrays of a result made with BROOK_DEVICE_OUTPUT (INVALID_ARGUMENT otherwise). */
brook_status brook_skeletons_get_device_view(const brook_skeletons *result, brook_skeletons_device_view *out);
/* brook.h:233: one of those arrays as an array handle sharing the result's storage. */
brook_status brook_skeletons_get_array(const brook_skeletons *result, brook_skeleton_buffer buffer, brook_array **out);

/* No counterpart in the reference. The EDT of brook_edt for callers that cannot allocate device
 * memory: code running inside another framework's memory budget (a caching allocator or a
 * pre-reserved pool that owns the free device memory), code where an allocation would synchronise
 * the device or fail under memory pressure, and callers that must keep a fixed device footprint.
 * It allocates nothing and needs no context: labels are Fortran-contiguous uint32 device memory
 * (memory = BROOK_DEVICE) of the current device, out is the caller's float32 device array of
 * shape[0]*shape[1]*shape[2] entries, and the work is queued on `stream` (a cudaStream_t; NULL
 * is the legacy default stream) without synchronising: out is ready when the stream gets there.
 * The result equals brook_edt's on the same labels. Scratch is one fixed 32 MiB device array of
 * the library (every GPU that loads the library holds it until the process exits); volumes whose
 * x extent exceeds 12800 or whose 16 * (max(y, z) extent + 3) + 4 * (x extent + 2) bytes exceed
 * it are rejected with BROOK_INVALID_ARGUMENT. The first call on a device looks up the array's
 * device address; make that first call before any stream capture. Calls share the array, so calls
 * that overlap on the GPU (different streams or threads) race. */
brook_status brook_edt_device_noalloc(const brook_volume *labels, const float anisotropy[3], int black_border,
                                      float *out, void *stream);

/* No counterpart in the reference's C header (its Python binding builds the same from packed
 * arrays, PackedSkeletons.to_core): a host result handle holding a copy of a packed view, e.g. to
 * merge skeletons a program kept as arrays. */
brook_status brook_skeletons_create(const brook_skeletons_view *view, brook_skeletons **out);
/* brook.h:171-177: the components of a host volume of any size through slabs of the device
 * (budget_bytes of device memory; 0: BROOK_STREAM_BUDGET_MB, a positive number of MiB, else a
 * quarter of the free device memory and at least 64 MiB; a slab holds at least one xy plane). The handle owns the host id volume
 * (ids 1..count by ascending first flat index, Fortran order, u8 / u16 / u32 by the count), the
 * mapping id -> label (count + 1 entries) and the first flat index of every component. */
brook_status brook_connected_components_streamed(brook_context *context, const brook_volume *labels,
                                                 size_t budget_bytes, brook_host_components **out);
void brook_host_components_destroy(brook_host_components *components);
brook_status brook_host_components_view(const brook_host_components *components, brook_volume *labels,
                                        const int64_t **mapping, const int64_t **roots, size_t *count);
/* brook.h:185-191: the multi-label EDT brook_edt gives, for a host volume of any size, into the
 * caller's host float32 array (output_bytes must cover the volume; Fortran order; input and
 * output must not overlap): components by slabs, the x and y passes by z-slabs, the z pass by
 * tiles of whole columns, within budget_bytes of device memory (as above). */
brook_status brook_edt_streamed(brook_context *context, const brook_volume *labels, const float anisotropy[3],
                                int black_border, size_t budget_bytes, float *output, size_t output_bytes);
/* brook.h:202-206: the skeletons brook_skeletonize gives, for a host volume whose in-core state does
 * not fit on the device (any size, each axis below 2^31): components by slabs, then every traced
 * component in its bounding box within budget_bytes of device memory (as above). fill_holes and
 * fix_avocados are refused (BROOK_INVALID_ARGUMENT). */
brook_status brook_skeletonize_streamed(brook_context *context, const brook_volume *labels,
                                        const brook_skeletonize_options *options, size_t budget_bytes,
                                        brook_skeletons **out);
/* No counterpart in the reference's C header (its Python binding wraps device PackedSkeletons the
 * same way, PackedSkeletons.to_core): a device result holding a copy, made on the context's stream,
 * of packed skeletons whose vertices ({3, V}), edges ({2, E}) and radii ({1, V}) are row-major
 * contiguous device arrays of the context's device; labels and offsets on the host. Work that
 * produced the arrays on another stream must be ordered before the call (brook_context_wait_stream). */
brook_status brook_skeletons_create_device(brook_context *context, const brook_skeletons_device_view *view,
                                           brook_skeletons **out);
/* brook.h:244-247: one skeleton per label over `count` fragments (the pieces of overlapping chunks),
 * fragment i's vertices shifted by origins[3i .. 3i+2] (physical units; NULL: no shift). Vertices
 * of one label at the same physical point merge (the first fragment's radius), edges are mapped,
 * deduplicated and sorted, vertices on no edge are dropped, labels come out ascending. The result
 * is a device result (as with BROOK_DEVICE_OUTPUT). */
brook_status brook_merge_skeletons(brook_context *context, const brook_skeletons *const *fragments,
                                   const float *origins, size_t count, brook_skeletons **out);

/* brook.h:238-239: canonical post-processing of skeletons (host or device result) on the device:
 * remove_dust(dust_threshold), remove_loops, join_close_components, remove_ticks(tick_threshold)
 * and the removal of vertices on no edge, with the reference's tie rules (post.cu:646-650). A
 * threshold of 0 skips its step. Every label of the input stays, possibly empty. The result is a
 * device result (as with BROOK_DEVICE_OUTPUT). */
brook_status brook_postprocess_canonical(brook_context *context, const brook_skeletons *input,
                                         double dust_threshold, double tick_threshold, brook_skeletons **out);
/* No counterpart in the reference's C header (its Python binding exposes the same steps as context
 * methods, src/brook/_device_post.py:23-44): one step of the canonical post-processing on its own;
 * `threshold` is the dust or tick threshold of those two steps and is ignored by the others. */
typedef enum brook_post_step {
  BROOK_POST_REMOVE_DUST = 1, BROOK_POST_REMOVE_LOOPS = 2, BROOK_POST_JOIN_COMPONENTS = 3,
  BROOK_POST_REMOVE_TICKS = 4, BROOK_POST_PRUNE_UNUSED = 5
} brook_post_step;
brook_status brook_postprocess_step(brook_context *context, const brook_skeletons *input, int step,
                                    double threshold, brook_skeletons **out);
/* No counterpart in the reference's C header (src/brook/_device_post.py:13-16): the connected
 * component of every packed vertex, named by the smallest global vertex index in it, as an int64
 * device array (one row per vertex). */
brook_status brook_skeleton_components(brook_context *context, const brook_skeletons *input, brook_array **out);

/* No counterpart in the reference's C header (the reference checks the same arithmetic through its
 * internal brook::pdrf, cpp/tests/pdrf_fusion_smoke.cu:57-88): the penalty the engine computes for
 * n voxels of host DBF / DAF values, with an object's DBF maximum `maximum`, its largest DAF
 * `max_daf` (0: no DAF term), pdrf_scale and pdrf_exponent — the engine's own device arithmetic, for
 * checks of it. */
brook_status brook_pdrf_values(brook_context *context, const float *dbf, const float *daf, size_t n, double maximum,
                               double max_daf, double scale, double exponent, float *out);

/* No counterpart in the reference's C header (the reference sizes its cooperative grids by a timed
 * probe, cooperative.cu:18-47). The object engine's launch choices for one workload class: the
 * CTAs per thread-block cluster of the large objects (4 or 8), the voxel counts from which objects
 * prepare / trace on clusters, and the percent of clusters that start on the small objects.
 * 0 (-1 for the percent) keeps the built-in rule. A workload class is a key of the foreground
 * voxel count, the largest object's voxel count and the object count (their bit lengths). */
typedef struct brook_tuning {
  int32_t trace_cluster_ctas;
  int64_t trace_cluster_voxels;
  int64_t prepare_cluster_voxels;
  int32_t lone_first_percent;
} brook_tuning;
/* Measures the engine (prepare and trace, CUDA events) on these volumes with candidate launch
 * choices (a coordinate search from the built-in rule, each candidate timed twice), installs the
 * fastest in the context for the volumes' workload class and returns the class, the choice and
 * its time. Calls of that class through this context then use it. */
brook_status brook_autotune(brook_context *context, const brook_volume *volumes, size_t count,
                            const brook_skeletonize_options *options, uint64_t *workload_class,
                            brook_tuning *best, double *best_ms);
/* Installs (or, with tuning NULL, removes) the launch choice of a workload class, e.g. one a
 * program saved from an earlier brook_autotune. */
brook_status brook_context_set_tuning(brook_context *context, uint64_t workload_class, const brook_tuning *tuning);

/* The statistics of the context's last call as a JSON object (the reference keeps the same map as
 * Context.stats, runtime.hpp:59 and bindings.cpp:343-347): "ms_<stage>" stage times measured with
 * CUDA events on the context's stream, and counters (paths, railroad_settled, railroad_touched,
 * invalidated, objects, voxels, foreground, launches, label_bytes). *length receives the size
 * needed including the terminating zero; json (capacity bytes) receives as much as fits. */
brook_status brook_context_stats(brook_context *context, char *json, size_t capacity, size_t *length);

#ifdef __cplusplus
}
#endif
#endif
