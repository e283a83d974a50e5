"""B200-native intra rate-distortion search of an AV1 still-image encoder (the hot path of maddog107/av1gpu).

The search runs in hand-written sm_100a CUDA kernels in libisearch.so (built in-tree by av1gpu_b200.build); this
package is the host-side mirror of the reference's GpEncoder interface over that library's C ABI
(include/is_api.h).  There is no CPU fallback: without the library every entry point raises.
"""
import os as _os

# Serving sessions keep a persistent closed-loop kernel running while other streams work; with the driver's default of 8
# hardware work queues, a stream that shares a queue with such a kernel waits behind it.  More queues (read when the
# process creates its CUDA context, so this takes effect when the package is imported first) keep streams apart.
_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from .isearch import Encoder, Record, load_library, LIB_PATH  # noqa: F401,E402
from . import synth  # noqa: F401,E402

__all__ = ["Encoder", "Record", "load_library", "LIB_PATH", "synth"]
