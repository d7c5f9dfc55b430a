/* The DLPack exchange structures (DLPack ABI 1.x, https://dmlc.github.io/dlpack/latest/) that
 * brook_array_to_dlpack and brook_array_to_dlpack_versioned hand out.
 *
 * The layouts are the DLPack standard's, field for field, so a consumer that already includes
 * the standard dlpack/dlpack.h can use it instead: both headers share the include guard
 * DLPACK_DLPACK_H_, and whichever comes first defines the types. The reference ships the same
 * standard header (cpp/include/brook/dlpack.h) for the same two calls (brook.h:165-167).
 */
#ifndef DLPACK_DLPACK_H_
#define DLPACK_DLPACK_H_

#include <stdint.h>

#define DLPACK_MAJOR_VERSION 1
#define DLPACK_MINOR_VERSION 1

/* Flags of DLManagedTensorVersioned.flags */
#define DLPACK_FLAG_BITMASK_READ_ONLY (1UL << 0UL)
#define DLPACK_FLAG_BITMASK_IS_COPIED (1UL << 1UL)
#define DLPACK_FLAG_BITMASK_IS_SUBBYTE_TYPE_PADDED (1UL << 2UL)

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  uint32_t major;
  uint32_t minor;
} DLPackVersion;

/* The device kinds this library exports: host memory and CUDA device memory. The numbering is
 * the standard's, which lists further kinds this library never produces. */
typedef enum {
  kDLCPU = 1,
  kDLCUDA = 2,
  kDLCUDAHost = 3,
  kDLCUDAManaged = 13
} DLDeviceType;

typedef struct {
  DLDeviceType device_type;
  int32_t device_id;
} DLDevice;

typedef enum {
  kDLInt = 0U,
  kDLUInt = 1U,
  kDLFloat = 2U,
  kDLOpaqueHandle = 3U,
  kDLBfloat = 4U,
  kDLComplex = 5U,
  kDLBool = 6U
} DLDataTypeCode;

typedef struct {
  uint8_t code;   /* a DLDataTypeCode */
  uint8_t bits;   /* bits per lane */
  uint16_t lanes; /* 1 for scalars */
} DLDataType;

typedef struct {
  void *data;
  DLDevice device;
  int32_t ndim;
  DLDataType dtype;
  int64_t *shape;
  int64_t *strides; /* in elements; NULL means compact row major */
  uint64_t byte_offset;
} DLTensor;

/* The consumer calls deleter(self) exactly once when it no longer needs the tensor. */
typedef struct DLManagedTensor {
  DLTensor dl_tensor;
  void *manager_ctx;
  void (*deleter)(struct DLManagedTensor *self);
} DLManagedTensor;

typedef struct DLManagedTensorVersioned {
  DLPackVersion version;
  void *manager_ctx;
  void (*deleter)(struct DLManagedTensorVersioned *self);
  uint64_t flags;
  DLTensor dl_tensor;
} DLManagedTensorVersioned;

#ifdef __cplusplus
}
#endif
#endif /* DLPACK_DLPACK_H_ */
