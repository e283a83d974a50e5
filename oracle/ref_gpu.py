"""ctypes wrapper of oracle/_ref/libref_gpu.so: the reference's own GPU search (maddog107/av1gpu GpEncoder::encode,
encoder/src/pipeline.h:191-211) built from its sources by oracle/refgpu.mk, with the plain knob set (oracle/ref_gpu.cpp).
Measurement infrastructure only: the speed bar of the B200 build and the reference's own decisions for BD-rate
comparisons.  8-bit 4:2:0 pictures."""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libref_gpu.so")
_lib = None


def available():
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB)
        vp = C.c_void_p
        L.ref_gpu_error.restype = C.c_char_p
        L.ref_gpu_search.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp, C.c_int, vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                     C.POINTER(C.c_uint64)]
        L.ref_gpu_copy.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.ref_gpu_check.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_int), vp]
        _lib = L
    return _lib


class RefResult:
    pass


def search(planes, qindex, reps=1, record=True):
    """Search (Y, U, V) uint8 4:2:0 host planes with the reference's GPU encoder reps times; the last run's GpTimes
    (ms: setup, analysis, dp, recon, pack, total) and, with record, its DecisionRecord and reconstruction."""
    from oracle import BLOCK_DT, TXB_DT
    y, u, v = [np.ascontiguousarray(p, np.uint8) for p in planes]
    h, w = y.shape
    t = np.zeros(6, np.float32)
    nb, nt, nc = C.c_uint32(), C.c_uint32(), C.c_uint64()
    L = lib()
    if L.ref_gpu_search(w, h, qindex, y.ctypes.data, u.ctypes.data, v.ctypes.data, reps, t.ctypes.data, C.byref(nb), C.byref(nt), C.byref(nc)):
        raise RuntimeError("reference GPU search failed: " + L.ref_gpu_error().decode(errors="replace"))
    r = RefResult()
    r.times = dict(zip(("setup", "analysis", "dp", "recon", "pack", "total"), map(float, t)))
    r.search_ms = float(t[0] + t[1] + t[2] + t[3] + t[4])
    if record:
        r.blocks = np.zeros(nb.value, BLOCK_DT)
        r.block_txb = np.zeros(nb.value + 1, np.uint32)
        r.txb = np.zeros(nt.value, TXB_DT)
        r.coeffs = np.zeros(nc.value, np.int16)
        r.recon = [np.zeros((h, w), np.uint8), np.zeros(((h + 1) // 2, (w + 1) // 2), np.uint8), np.zeros(((h + 1) // 2, (w + 1) // 2), np.uint8)]
        if L.ref_gpu_copy(r.blocks.ctypes.data, r.block_txb.ctypes.data, r.txb.ctypes.data, r.coeffs.ctypes.data, r.recon[0].ctypes.data,
                          r.recon[1].ctypes.data, r.recon[2].ctypes.data):
            raise RuntimeError("reference GPU copy failed: " + L.ref_gpu_error().decode(errors="replace"))
        # av1g_encode of the record with the reference's own frame parameters: OBU size and the exactness check
        nbytes, eq = C.c_uint64(), C.c_int()
        fp = np.zeros(256, np.uint8)
        if L.ref_gpu_check(C.byref(nbytes), C.byref(eq), fp.ctypes.data):
            raise RuntimeError("av1g_encode rejected the reference's record: " + L.ref_gpu_error().decode(errors="replace"))
        r.obu_bytes, r.recon_exact = nbytes.value, bool(eq.value)
    return r
