"""B200-native intra rate-distortion search of an AV1 still-image encoder (the hot path of maddog107/av1gpu).

The search runs in hand-written sm_100a CUDA kernels in libisearch.so (built in-tree by av1gpu_b200.build); this
package is the host-side mirror of the reference's GpEncoder interface over that library's C ABI
(include/is_api.h).  There is no CPU fallback: without the library every entry point raises.
"""
from .isearch import Encoder, Record, load_library, LIB_PATH  # noqa: F401
from . import synth  # noqa: F401

__all__ = ["Encoder", "Record", "load_library", "LIB_PATH", "synth"]
