"""brook_b200: TEASAR skeletonization of 3D label volumes on NVIDIA B200 (sm_100a).

A drop-in for the reference's `brook.skeletonize` / `brook.skeletonize_batch` and its C SDK
entry points (include/brook_b200.h). The compute path is the CUDA library
brook_b200/_lib/libbrook_b200.so (built by brook_b200/build.py); there is no CPU fallback.
"""
from __future__ import annotations

__version__ = "0.1.0"

from ._intake import DEFAULT_TEASAR_PARAMS, DimensionError, skeletonize  # noqa: E402
from ._packed import PackedSkeletons, Skeleton  # noqa: E402
from .batch import BatchedSkeletons, skeletonize_batch  # noqa: E402
from .chunked import merge_fragments, skeletonize_chunked  # noqa: E402
from . import device_post  # noqa: E402

__all__ = ["skeletonize", "skeletonize_batch", "skeletonize_chunked", "merge_fragments", "BatchedSkeletons",
           "PackedSkeletons", "Skeleton", "DEFAULT_TEASAR_PARAMS", "DimensionError", "device_post", "__version__"]
