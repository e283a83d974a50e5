"""Host mirror of the reference's GpEncoder (encoder/src/pipeline.h:191-211) over libisearch.so's C ABI.

    enc = Encoder(device=0)                 # GpEncoder::init
    rec = enc.encode(planes, qindex)        # GpEncoder::encode with host planes (upload inside the call)
    rec = enc.encode_device(tensors, q)     # device planes (torch CUDA uint8 tensors), GpFrameIn-style
    rec.blocks, rec.block_txb, rec.txb, rec.coeffs, rec.recon   # av1core DecisionRecord + reconstruction

Errors raise RuntimeError with the library's message (the reference returns -1 + a message, pipeline.cpp:31-39).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libisearch.so")

# av1core DecisionRecord layouts (av1core/include/av1g/decisions.h:225-252), 16 bytes each
BLOCK_DT = np.dtype([("mi_row", "<u2"), ("mi_col", "<u2"), ("bsize", "u1"), ("skip", "u1"), ("tx_depth", "u1"),
                     ("y_mode", "u1"), ("angle_delta_y", "i1"), ("uv_mode", "u1"), ("angle_delta_uv", "i1"),
                     ("cfl_alpha_u", "i1"), ("cfl_alpha_v", "i1"), ("filter_intra", "u1"), ("cdef_idx", "i1"),
                     ("sb_qindex", "u1")])
TXB_DT = np.dtype([("coeff_off", "<u4"), ("x4", "<u2"), ("y4", "<u2"), ("plane", "u1"), ("tx_size", "u1"),
                   ("tx_type", "u1"), ("flags", "u1"), ("eob", "<u2"), ("reserved", "<u2")])

# av1g_frame_params (av1core/include/av1g/decisions.h:254-296): 88 bytes; the offsets of the fields the bindings write
FRAME_PARAMS_BYTES = 88
FP_BASE_Q_IDX, FP_TILE_LOG2, FP_QM, FP_CHROMA_FORMAT, FP_BIT_DEPTH = 13, 16, 28, 72, 73
AV1G_DECISIONS_VERSION = 5

IS_ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of device memory", -4: "wavefront wait timeout",
             -5: "no result", -6: "too large for the static scratch", -7: "serving session busy"}
IS_ERR_INVALID, IS_ERR_CUDA, IS_ERR_OOM, IS_ERR_TIMEOUT, IS_ERR_STATE, IS_ERR_TOO_LARGE, IS_ERR_BUSY = -1, -2, -3, -4, -5, -6, -7


class IsError(RuntimeError):
    """A failed entry point: .code is the library's status (IS_ERR_*), the message the handle's last error."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class IsParams(C.Structure):
    _fields_ = [("bit_depth", C.c_int32), ("chroma_444", C.c_int32), ("device", C.c_int32), ("reserved", C.c_int32 * 5)]


class IsFrame(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("qindex", C.c_int32), ("bit_depth", C.c_int32),
                ("planes", C.c_void_p * 3), ("pitch", C.c_int32 * 3), ("chroma_444", C.c_int32)]


class IsTimes(C.Structure):
    _fields_ = [("upload", C.c_float), ("analysis", C.c_float), ("dp", C.c_float), ("recon", C.c_float),
                ("pack", C.c_float), ("total", C.c_float), ("sbs", C.c_uint32), ("blocks", C.c_uint32)]


# every entry point declared in include/is_api.h
EXPORTS = ["is_create", "is_destroy", "is_last_error", "is_encode_device", "is_encode_host", "is_record_counts",
           "is_record_copy", "is_record_device", "is_times_get", "is_test_fwd_quant", "is_test_inverse",
           "is_test_predict", "is_debug_analysis", "is_debug_leaves", "is_debug_tables", "is_probe_int32", "is_set_trace", "is_get_trace",
           "is_fwd_quant_static", "is_encode_batch", "is_batch_counts", "is_batch_copy", "is_set_batch_options",
           "is_autotune_batch", "is_workspace_bytes", "is_workspace_bytes_format", "is_sl_create", "is_sl_destroy", "is_sl_set_params",
           "is_sl_get_params", "is_sl_forward", "is_sl_grads", "is_sl_train_step", "is_nn_gemm", "is_sl_dataset", "is_sl_infer",
           "is_set_shortlist_model",
           "is_set_wait_limits", "is_set_workspace_limit", "is_set_poison", "is_set_search_options", "is_set_closed_loop_warps", "is_serve_open", "is_serve_start", "is_serve_submit", "is_serve_poll",
           "is_serve_counts", "is_serve_copy", "is_serve_stop", "is_serve_close", "is_entropy_scratch_bytes", "is_entropy_batch",
           "is_obu_assemble", "is_encode_obu", "is_postfilter", "is_postfilter_from_q",
           "is_avif_mux"]

_lib = None


def load_library():
    """The CUDA library; raises if it was not built (there is no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libisearch.so missing: run `python -m av1gpu_b200.build` (the search has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.is_create.argtypes = [C.POINTER(IsParams), C.POINTER(vp)]
    L.is_destroy.argtypes = [vp]
    L.is_destroy.restype = None
    L.is_last_error.argtypes = [vp]
    L.is_last_error.restype = C.c_char_p
    L.is_encode_device.argtypes = [vp, C.POINTER(IsFrame), vp]
    L.is_encode_host.argtypes = [vp, C.POINTER(IsFrame), vp]
    L.is_record_counts.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
    L.is_record_copy.argtypes = [vp, vp, vp, vp, vp, vp, vp * 3, vp]
    L.is_record_device.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]
    L.is_times_get.argtypes = [vp, C.POINTER(IsTimes)]
    L.is_test_fwd_quant.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp]
    L.is_test_inverse.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, vp, vp]
    L.is_test_predict.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, vp, vp]
    L.is_debug_analysis.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp]
    L.is_debug_leaves.argtypes = [vp, C.c_uint32, vp, vp, vp]
    L.is_debug_tables.argtypes = [vp, C.c_int, vp, C.c_size_t, vp, vp, vp, C.c_int, C.POINTER(C.c_int64),
                                  C.POINTER(C.c_int64)]
    L.is_probe_int32.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_float)]
    L.is_set_trace.argtypes = [C.c_void_p, C.c_int]
    L.is_get_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint32)]
    L.is_fwd_quant_static.argtypes = [C.c_int, C.c_int, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp]
    L.is_encode_batch.argtypes = [vp, C.POINTER(IsFrame), C.c_int, C.c_int, vp]
    L.is_batch_counts.argtypes = [vp, C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
    L.is_batch_copy.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp * 3, vp]
    L.is_set_batch_options.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    L.is_workspace_bytes.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint64)]
    L.is_workspace_bytes_format.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64)]
    L.is_sl_create.argtypes = [C.c_int, C.c_int, C.POINTER(vp)]
    L.is_sl_destroy.argtypes = [vp]
    L.is_sl_destroy.restype = None
    L.is_sl_set_params.argtypes = [vp, vp]
    L.is_sl_get_params.argtypes = [vp, vp]
    L.is_sl_forward.argtypes = [vp, vp, C.c_int, vp, vp]
    L.is_sl_grads.argtypes = [vp, vp, vp, C.c_int, vp, C.POINTER(C.c_float), C.POINTER(C.c_int)]
    L.is_sl_train_step.argtypes = [vp, vp, vp, C.c_int, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_int)]
    L.is_nn_gemm.argtypes = [C.c_int, C.c_int, C.c_int, vp, C.c_int, vp, C.c_int, vp, C.c_int, vp, C.c_int, vp]
    L.is_sl_dataset.argtypes = [vp, C.c_int, vp, vp, C.c_int, C.POINTER(C.c_int)]
    L.is_sl_infer.argtypes = [vp, vp, C.c_int, vp, C.c_int, C.POINTER(C.c_int)]
    L.is_set_shortlist_model.argtypes = [vp, vp, C.c_float, C.c_int, C.c_float, C.c_int, C.c_float, C.c_int]
    L.is_autotune_batch.argtypes = [vp, C.POINTER(IsFrame), C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float)]
    L.is_set_closed_loop_warps.argtypes = [vp, C.c_int]
    L.is_set_wait_limits.argtypes = [vp, C.c_int, C.c_longlong]
    L.is_set_workspace_limit.argtypes = [vp, C.c_uint64]
    L.is_set_poison.argtypes = [vp, C.c_int]
    L.is_set_search_options.argtypes = [vp, C.c_int, C.c_int]
    L.is_serve_open.argtypes = [vp, C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_uint64, C.c_int]
    L.is_serve_start.argtypes = [vp]
    L.is_serve_submit.argtypes = [vp, C.POINTER(IsFrame), C.c_int, C.POINTER(C.c_int)]
    L.is_serve_poll.argtypes = [vp, vp, C.c_int, C.POINTER(C.c_int)]
    L.is_serve_counts.argtypes = [vp, C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
    L.is_serve_copy.argtypes = [vp, C.c_int, vp, vp, vp, vp, vp, vp * 3, vp]
    L.is_serve_stop.argtypes = [vp]
    L.is_serve_close.argtypes = [vp]
    L.is_entropy_scratch_bytes.argtypes = [vp, C.c_int, C.c_uint64, C.POINTER(C.c_uint64)]
    L.is_entropy_batch.argtypes = [C.c_int, vp, C.c_int, C.c_uint64, vp, C.c_uint64, vp, vp, vp]
    L.is_obu_assemble.argtypes = [vp, vp, vp, C.c_uint32, vp, C.c_uint64, C.POINTER(C.c_uint64)]
    L.is_encode_obu.argtypes = [vp, C.c_int, C.c_int, vp, C.c_uint64, vp, C.POINTER(C.c_float)]
    L.is_postfilter.argtypes = [vp, C.c_int, vp, vp, C.POINTER(C.c_float)]
    L.is_postfilter_from_q.argtypes = [C.c_int, C.c_int, vp]
    L.is_avif_mux.argtypes = [vp, vp, C.c_uint64, vp, C.c_uint64, C.POINTER(C.c_uint64)]
    _lib = L
    return L


def workspace_bytes(width, height, bit_depth=8, chroma_444=False):
    """Device workspace of one image in a batch (bytes); no GPU needed."""
    b = C.c_uint64()
    if load_library().is_workspace_bytes_format(width, height, bit_depth, int(bool(chroma_444)), C.byref(b)) != 0:
        raise ValueError("invalid image %dx%d (bit depth %d, 4:4:4 %s)" % (width, height, bit_depth, chroma_444))
    return b.value


def frame_params(width, height, qindex, bit_depth=8, chroma_444=False):
    """The av1g_frame_params bytes the search writes for an image (is_batch_copy's fp)."""
    fp = np.zeros(FRAME_PARAMS_BYTES, np.uint8)
    fp[:12].view(np.uint32)[:] = (AV1G_DECISIONS_VERSION, width, height)
    fp[FP_BASE_Q_IDX] = qindex
    fp[FP_TILE_LOG2:FP_TILE_LOG2 + 2] = 0xFF        # tile_cols_log2 = tile_rows_log2 = -1: the minimum legal tiling
    fp[FP_QM:FP_QM + 3] = 15                        # qm_y, qm_u, qm_v
    fp[FP_CHROMA_FORMAT] = 1 if chroma_444 else 0
    fp[FP_BIT_DEPTH] = bit_depth
    return fp


def avif_mux(fp, obu):
    """The AVIF file (bytes) around an OBU stream written for fp (av1g_frame_params bytes)."""
    L = load_library()
    fp = np.ascontiguousarray(fp, np.uint8)
    src = np.frombuffer(bytes(obu), np.uint8)
    size = C.c_uint64()
    rc = L.is_avif_mux(fp.ctypes.data, src.ctypes.data, len(src), None, 0, C.byref(size))
    if rc not in (0, IS_ERR_TOO_LARGE):
        raise IsError(rc, "is_avif_mux failed (%d)" % rc)
    out = np.zeros(size.value, np.uint8)
    rc = L.is_avif_mux(fp.ctypes.data, src.ctypes.data, len(src), out.ctypes.data, size.value, C.byref(size))
    if rc != 0:
        raise IsError(rc, "is_avif_mux failed (%d)" % rc)
    return out.tobytes()


def postfilter_from_q(fp, qindex, bit_depth=8):
    """fp (av1g_frame_params bytes) with the reference's default deblocking levels, sharpness and CDEF damping."""
    fp = np.ascontiguousarray(fp, np.uint8).copy()
    rc = load_library().is_postfilter_from_q(qindex, bit_depth, fp.ctypes.data)
    if rc != 0:
        raise IsError(rc, "is_postfilter_from_q failed (%d)" % rc)
    return fp


def obu_assemble(fp, payload, tile_offsets):
    """The OBU stream (sequence header + frame OBU) of a frame from its tile payloads (host bytes) and offsets."""
    L = load_library()
    pay = np.frombuffer(bytes(payload), np.uint8) if not isinstance(payload, np.ndarray) else np.ascontiguousarray(payload, np.uint8)
    off = np.ascontiguousarray(tile_offsets, np.uint64)
    size = C.c_uint64()
    fp = np.ascontiguousarray(fp, np.uint8)
    rc = L.is_obu_assemble(fp.ctypes.data, pay.ctypes.data, off.ctypes.data, len(off) - 1, None, 0, C.byref(size))
    if rc not in (0, IS_ERR_TOO_LARGE):
        raise IsError(rc, "is_obu_assemble failed (%d)" % rc)
    out = np.zeros(size.value, np.uint8)
    rc = L.is_obu_assemble(fp.ctypes.data, pay.ctypes.data, off.ctypes.data, len(off) - 1, out.ctypes.data, size.value, C.byref(size))
    if rc != 0:
        raise IsError(rc, "is_obu_assemble failed (%d)" % rc)
    return out.tobytes()


def plane_format(planes):
    """(bit depth, 4:4:4) of (Y, U, V) planes: 16-bit samples are 10-bit, chroma of the luma size is 4:4:4."""
    y, u = planes[0], planes[1]
    dt = str(y.dtype)
    bd = 10 if ("uint16" in dt or "int16" in dt) else 8
    return bd, tuple(u.shape) == tuple(y.shape)


def _recon_arrays(width, height, bit_depth, chroma_444):
    dt = np.uint16 if bit_depth == 10 else np.uint8
    cw, ch = (width, height) if chroma_444 else ((width + 1) // 2, (height + 1) // 2)
    return [np.zeros((height, width), dt), np.zeros((ch, cw), dt), np.zeros((ch, cw), dt)]


def probe_int32(device=0):
    """Measured INT32 instruction throughput (Gop/s) and the probe kernel's time (ms)."""
    g, ms = C.c_double(), C.c_float()
    rc = load_library().is_probe_int32(device, C.byref(g), C.byref(ms))
    if rc != 0:
        raise RuntimeError("is_probe_int32 failed (%d)" % rc)
    return g.value, ms.value


def host_tables(qctx, qindex=120):
    """Fixed-point tables the library uploads (no GPU needed): cost table, avgY, avgPart, avgSkip0, lambda, sqrt."""
    L = load_library()
    n = L.is_debug_tables(None, qctx, None, 0, None, None, None, qindex, None, None)
    cost = np.zeros(n, np.uint16)
    y, p, s = np.zeros(13, np.int32), np.zeros(50, np.int32), np.zeros(1, np.int32)
    lam, sq = C.c_int64(), C.c_int64()
    L.is_debug_tables(None, qctx, cost.ctypes.data, n, y.ctypes.data, p.ctypes.data, s.ctypes.data, qindex,
                      C.byref(lam), C.byref(sq))
    return cost, y, p.reshape(5, 10), int(s[0]), lam.value, sq.value


class Record:
    """One encoded image: the DecisionRecord arrays (decode order) and the cropped reconstruction."""

    def __init__(self, width, height, qindex, blocks, block_txb, txb, coeffs, recon, times, bit_depth=8, chroma_444=False):
        self.width, self.height, self.qindex = width, height, qindex
        self.bit_depth, self.chroma_444 = bit_depth, chroma_444
        self.blocks, self.block_txb, self.txb, self.coeffs = blocks, block_txb, txb, coeffs
        self.recon = recon
        self.times = times

    def digest(self):
        """BLAKE2b of every record array and reconstruction plane: equal digests = bit-equal results."""
        import hashlib
        h = hashlib.blake2b(digest_size=20)
        for a in (self.blocks, self.block_txb, self.txb, self.coeffs, *self.recon):
            h.update(np.ascontiguousarray(a).view(np.uint8).tobytes())
        return h.hexdigest()


class Encoder:
    """GpEncoder-shaped handle (one host thread at a time)."""

    def __init__(self, device=0):
        self.L = load_library()
        p = IsParams()
        p.bit_depth, p.chroma_444, p.device = 8, 0, device
        h = C.c_void_p()
        rc = self.L.is_create(C.byref(p), C.byref(h))
        if rc != 0:
            raise IsError(rc, "is_create failed (%d: %s)" % (rc, IS_ERRORS.get(rc, "?")))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.is_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            msg = self.L.is_last_error(self.h).decode(errors="replace")
            raise IsError(rc, "%s failed (%d: %s): %s" % (what, rc, IS_ERRORS.get(rc, "?"), msg))

    @staticmethod
    def _frame(planes, qindex, host):
        """is_frame of (Y, U, V) planes: numpy arrays (host) or torch CUDA tensors; uint8 8-bit, 16-bit samples 10-bit."""
        y = planes[0]
        bd, c444 = plane_format(planes)
        f = IsFrame()
        f.width, f.height, f.qindex = y.shape[1], y.shape[0], qindex
        f.bit_depth, f.chroma_444 = bd, int(c444)
        for p in range(3):
            f.planes[p] = planes[p].ctypes.data if host else planes[p].data_ptr()
            f.pitch[p] = planes[p].strides[0] // planes[p].itemsize if host else planes[p].stride(0)
        return f

    def encode_host_async(self, planes, qindex, stream=None):
        """Queue an encode of host planes (Y, U, V numpy uint8 / uint16, row-contiguous); returns after the record sizes
        are known."""
        f = self._frame(planes, qindex, True)
        self._check(self.L.is_encode_host(self.h, C.byref(f), stream), "is_encode_host")
        return f

    def encode_device_async(self, planes, qindex, stream=None):
        """Queue an encode of device planes (torch CUDA uint8 / 16-bit tensors, row-contiguous)."""
        f = self._frame(planes, qindex, False)
        self._check(self.L.is_encode_device(self.h, C.byref(f), stream), "is_encode_device")
        return f

    def counts(self):
        nb, nt, nc = C.c_uint32(), C.c_uint32(), C.c_uint64()
        self._check(self.L.is_record_counts(self.h, C.byref(nb), C.byref(nt), C.byref(nc)), "is_record_counts")
        return nb.value, nt.value, nc.value

    def times(self):
        t = IsTimes()
        self._check(self.L.is_times_get(self.h, C.byref(t)), "is_times_get")
        return {k: getattr(t, k) for k, _ in IsTimes._fields_}

    def fetch(self, width, height, qindex, out=None, bit_depth=8, chroma_444=False):
        """Copy the last record and reconstruction to host memory (numpy arrays, or the preallocated `out` dict)."""
        nb, nt, nc = self.counts()
        if out is None:
            out = {"blocks": np.zeros(nb, BLOCK_DT), "block_txb": np.zeros(nb + 1, np.uint32),
                   "txb": np.zeros(nt, TXB_DT), "coeffs": np.zeros(nc, np.int16),
                   "recon": _recon_arrays(width, height, bit_depth, chroma_444)}
        rp = (C.c_void_p * 3)(*[r.ctypes.data for r in out["recon"]])
        pitches = (C.c_int32 * 3)(*[r.strides[0] // r.itemsize for r in out["recon"]])
        self._check(self.L.is_record_copy(self.h, None, out["blocks"].ctypes.data, out["block_txb"].ctypes.data,
                                          out["txb"].ctypes.data, out["coeffs"].ctypes.data, rp, pitches),
                    "is_record_copy")
        return Record(width, height, qindex, out["blocks"][:nb], out["block_txb"][:nb + 1], out["txb"][:nt],
                      out["coeffs"][:nc], out["recon"], self.times(), bit_depth, chroma_444)

    def encode(self, planes, qindex):
        """Encode host planes end to end: upload, search, download of the record and the reconstruction."""
        planes = [np.ascontiguousarray(p) for p in planes]
        bd, c444 = plane_format(planes)
        self.encode_host_async(planes, qindex)
        return self.fetch(planes[0].shape[1], planes[0].shape[0], qindex, bit_depth=bd, chroma_444=c444)

    def encode_device(self, planes, qindex):
        bd, c444 = plane_format(planes)
        self.encode_device_async(planes, qindex)
        return self.fetch(planes[0].shape[1], planes[0].shape[0], qindex, bit_depth=bd, chroma_444=c444)

    # ---- batched form ----
    def _frames(self, images, qindices, host):
        """is_frame array for a list of (Y, U, V) planes: numpy arrays (host) or torch CUDA tensors (device)."""
        fr = (IsFrame * len(images))()
        for i, (planes, q) in enumerate(zip(images, qindices)):
            fr[i] = self._frame(planes, q, host)
        return fr

    def encode_batch_async(self, images, qindices, host=True, stream=None):
        """Queue one batch (host numpy planes, or torch CUDA planes with host=False); returns after the record sizes
        of every image are known."""
        fr = self._frames(images, qindices, host)
        self._check(self.L.is_encode_batch(self.h, fr, len(images), 1 if host else 0, stream), "is_encode_batch")
        return fr

    def batch_counts(self, i):
        nb, nt, nc = C.c_uint32(), C.c_uint32(), C.c_uint64()
        self._check(self.L.is_batch_counts(self.h, i, C.byref(nb), C.byref(nt), C.byref(nc)), "is_batch_counts")
        return nb.value, nt.value, nc.value

    def batch_fetch(self, i, width, height, qindex, bit_depth=8, chroma_444=False):
        nb, nt, nc = self.batch_counts(i)
        out = {"blocks": np.zeros(nb, BLOCK_DT), "block_txb": np.zeros(nb + 1, np.uint32), "txb": np.zeros(nt, TXB_DT),
               "coeffs": np.zeros(nc, np.int16), "recon": _recon_arrays(width, height, bit_depth, chroma_444)}
        rp = (C.c_void_p * 3)(*[r.ctypes.data for r in out["recon"]])
        pitches = (C.c_int32 * 3)(*[r.strides[0] // r.itemsize for r in out["recon"]])
        self._check(self.L.is_batch_copy(self.h, i, None, out["blocks"].ctypes.data, out["block_txb"].ctypes.data,
                                         out["txb"].ctypes.data, out["coeffs"].ctypes.data, rp, pitches), "is_batch_copy")
        return Record(width, height, qindex, out["blocks"], out["block_txb"], out["txb"], out["coeffs"], out["recon"],
                      self.times(), bit_depth, chroma_444)

    def encode_batch(self, images, qindices):
        """Encode a list of host images ((Y, U, V) planes, uint8 8-bit or uint16 10-bit, 4:2:0 or 4:4:4) with their
        qindices in one batch; a list of Records."""
        images = [[np.ascontiguousarray(p) for p in planes] for planes in images]
        self.encode_batch_async(images, qindices, host=True)
        out = []
        for i, (im, q) in enumerate(zip(images, qindices)):
            bd, c444 = plane_format(im)
            out.append(self.batch_fetch(i, im[0].shape[1], im[0].shape[0], q, bd, c444))
        return out

    def obu(self, first=0, n=1, timed=False):
        """Images first .. first + n - 1 of the last encode entropy-coded on the device in one batch: a list of OBU
        streams (bytes, av1g_encode()'s obu), and with timed=True also the device time of the coding (ms)."""
        offs = np.zeros(n + 1, np.uint64)
        ms = C.c_float()
        px = 0
        for i in range(first, first + n):
            nb, _, nc = self.batch_counts(i)
            px += nc + 16 * nb
        buf = np.empty(8 * px + 65536, np.uint8)   # above any stream of these records: one coding in the common case
        rc = self.L.is_encode_obu(self.h, first, n, buf.ctypes.data, buf.size, offs.ctypes.data, C.byref(ms))
        if rc == IS_ERR_TOO_LARGE:
            buf = np.empty(int(offs[n]), np.uint8)
            rc = self.L.is_encode_obu(self.h, first, n, buf.ctypes.data, buf.size, offs.ctypes.data, C.byref(ms))
        self._check(rc, "is_encode_obu")
        out = [buf[int(offs[k]):int(offs[k + 1])].tobytes() for k in range(n)]
        return (out, ms.value) if timed else out

    def frame_params(self, i=0):
        """The av1g_frame_params bytes of image i of the last encode (with the post-filters once applied)."""
        fp = np.zeros(FRAME_PARAMS_BYTES, np.uint8)
        self._check(self.L.is_batch_copy(self.h, i, fp.ctypes.data, None, None, None, None, (C.c_void_p * 3)(), None), "is_batch_copy")
        return fp

    def avif(self, first=0, n=1):
        """Images first .. first + n - 1 of the last encode as AVIF files (bytes): device entropy coding in one batch,
        then the container on the host."""
        return [avif_mux(self.frame_params(first + k), s) for k, s in enumerate(self.obu(first, n))]

    def postfilter(self, fp, sb_cdef=None, i=0):
        """Deblocking + CDEF in place on image i's reconstruction (fp: av1g_frame_params bytes with the filter fields,
        sb_cdef: int8 cdef_idx per 64x64 or None); the device time (ms)."""
        fp = np.ascontiguousarray(fp, np.uint8)
        sb = None if sb_cdef is None else np.ascontiguousarray(sb_cdef, np.int8)
        ms = C.c_float()
        self._check(self.L.is_postfilter(self.h, i, fp.ctypes.data, None if sb is None else sb.ctypes.data, C.byref(ms)), "is_postfilter")
        return ms.value

    def set_wait_limits(self, leaf_wait_iters=0, ready_wait_ns=0):
        """Closed-loop wait budgets (0: the defaults); a wait that runs out makes the encode raise IsError(-4)."""
        self._check(self.L.is_set_wait_limits(self.h, int(leaf_wait_iters), int(ready_wait_ns)), "is_set_wait_limits")

    def set_workspace_limit(self, nbytes=0):
        """Device-memory budget of the workspace (0: none); an encode over it raises IsError(-3) before allocating."""
        self._check(self.L.is_set_workspace_limit(self.h, int(nbytes)), "is_set_workspace_limit")

    def set_poison(self, on=True):
        """Poison mode: workspace bytes and kernel shared memory start as garbage (results must not change)."""
        self._check(self.L.is_set_poison(self.h, 1 if on else 0), "is_set_poison")

    def set_search_options(self, rd_k=4, tx_keep=0):
        """Non-learned pruning: RD candidates per analysed block (1 .. 4) and the tx types (0 = all, 1 .. 3 best by the
        analysis' cost) the closed loop's tx-type pass keeps per block.  The defaults are the plain form."""
        self._check(self.L.is_set_search_options(self.h, rd_k, tx_keep), "is_set_search_options")

    # ---- serving session: continuous admission into a running closed loop ----
    def serve_open(self, bit_depth=8, chroma_444=False, arena_bytes=4 << 30, max_images=64, max_leaves=1 << 22, recon_ctas=0,
                   start=True):
        """Allocate a serving session (and start its loop; with several sessions in a process, open all with
        start=False, then serve_start each: allocations wait for running loops)."""
        self._check(self.L.is_serve_open(self.h, bit_depth, int(bool(chroma_444)), int(arena_bytes), max_images, int(max_leaves),
                                         recon_ctas), "is_serve_open")
        if start:
            self.serve_start()

    def serve_start(self):
        self._check(self.L.is_serve_start(self.h), "is_serve_start")

    def serve_submit(self, planes, qindex, host=True):
        """Queue one image into the running closed loop; its ticket, or None when the session has no room now."""
        f = self._frame(planes, qindex, host)
        t = C.c_int()
        rc = self.L.is_serve_submit(self.h, C.byref(f), 1 if host else 0, C.byref(t))
        if rc == IS_ERR_BUSY:
            return None
        self._check(rc, "is_serve_submit")
        return t.value

    def serve_poll(self, cap=256):
        """Tickets of the images whose records are ready (packed; read them with serve_fetch)."""
        out = np.zeros(cap, np.int32)
        n = C.c_int()
        self._check(self.L.is_serve_poll(self.h, out.ctypes.data, cap, C.byref(n)), "is_serve_poll")
        return [int(v) for v in out[:n.value]]

    def serve_fetch(self, ticket, width, height, qindex, bit_depth=8, chroma_444=False):
        nb, nt, nc = C.c_uint32(), C.c_uint32(), C.c_uint64()
        self._check(self.L.is_serve_counts(self.h, ticket, C.byref(nb), C.byref(nt), C.byref(nc)), "is_serve_counts")
        nb, nt, nc = nb.value, nt.value, nc.value
        out = {"blocks": np.zeros(nb, BLOCK_DT), "block_txb": np.zeros(nb + 1, np.uint32), "txb": np.zeros(nt, TXB_DT),
               "coeffs": np.zeros(nc, np.int16), "recon": _recon_arrays(width, height, bit_depth, chroma_444)}
        rp = (C.c_void_p * 3)(*[r.ctypes.data for r in out["recon"]])
        pitches = (C.c_int32 * 3)(*[r.strides[0] // r.itemsize for r in out["recon"]])
        self._check(self.L.is_serve_copy(self.h, ticket, None, out["blocks"].ctypes.data, out["block_txb"].ctypes.data,
                                         out["txb"].ctypes.data, out["coeffs"].ctypes.data, rp, pitches), "is_serve_copy")
        return Record(width, height, qindex, out["blocks"], out["block_txb"], out["txb"], out["coeffs"], out["recon"], {},
                      bit_depth, chroma_444)

    def serve_stop(self):
        self._check(self.L.is_serve_stop(self.h), "is_serve_stop")

    def serve_close(self):
        self._check(self.L.is_serve_close(self.h), "is_serve_close")

    def set_batch_options(self, use_graph=False, front_streams=0, recon_ctas=0):
        self._check(self.L.is_set_batch_options(self.h, 1 if use_graph else 0, front_streams, recon_ctas),
                    "is_set_batch_options")

    def set_shortlist(self, params=None, tau=0.9, max_cand=8, conf=0.0, rd_k=2, tx_tau=0.9, max_tx=2):
        """Use a trained shortlist network (IS_SL_PARAMS fp32 parameters) in this handle's searches; None: the plain
        form.  Candidates per scored block: the most probable (mode, delta) pairs covering tau (at most max_cand), the
        best rd_k of them by SATD into the RD, the tx types covering tx_tau (at most max_tx); blocks whose top
        probability is below conf search in full."""
        if params is None:
            self._check(self.L.is_set_shortlist_model(self.h, None, C.c_float(1.0), 1, C.c_float(0.0), 4, C.c_float(1.0), 0),
                        "is_set_shortlist_model")
            return
        p = np.ascontiguousarray(params, np.float32).ravel()
        self._keep_params = p
        self._check(self.L.is_set_shortlist_model(self.h, p.ctypes.data, C.c_float(tau), max_cand, C.c_float(conf), rd_k,
                                                  C.c_float(tx_tau), max_tx), "is_set_shortlist_model")

    def autotune_batch(self, images, qindices, host=True, with_warps=False):
        """Time the batch with 1 / 2 / 4 front-end streams x 4 / 6 / all closed-loop warps per CTA and keep the fastest
        for the handle; returns (streams, ms), or (streams, warps, ms) with with_warps (warps 0: all)."""
        fr = self._frames(images, qindices, host)
        k, w, ms = C.c_int(), C.c_int(), C.c_float()
        self._check(self.L.is_autotune_batch(self.h, fr, len(images), 1 if host else 0, C.byref(k), C.byref(w), C.byref(ms)),
                    "is_autotune_batch")
        return (k.value, w.value, ms.value) if with_warps else (k.value, ms.value)

    def set_closed_loop_warps(self, warps=0):
        """Warps per CTA of the closed loop (0: all the shared memory holds)."""
        self._check(self.L.is_set_closed_loop_warps(self.h, warps), "is_set_closed_loop_warps")

    # ---- kernel-level entry points (parity tests) ----
    def test_fwd_quant(self, res, tx_size, tx_type, plane, qindex, ctx):
        res = np.ascontiguousarray(res, np.int32)
        n = res.shape[0]
        h, w = res.shape[1], res.shape[2]
        nc = min(w, 32) * min(h, 32)
        coef, lv = np.zeros((n, nc), np.int32), np.zeros((n, nc), np.int16)
        D, R, eob = np.zeros(n, np.int64), np.zeros(n, np.int64), np.zeros(n, np.int32)
        cx = np.array(ctx, np.int32)
        self._check(self.L.is_test_fwd_quant(self.h, n, res.ctypes.data, tx_size, tx_type, plane, qindex, cx.ctypes.data,
                                             coef.ctypes.data, lv.ctypes.data, D.ctypes.data, R.ctypes.data,
                                             eob.ctypes.data), "is_test_fwd_quant")
        return coef, lv, D, R, eob

    def test_inverse(self, levels, tx_size, tx_type, qindex, w, h):
        levels = np.ascontiguousarray(levels, np.int16)
        n = levels.shape[0]
        res, fl = np.zeros((n, h * w), np.int32), np.zeros(n, np.uint32)
        self._check(self.L.is_test_inverse(self.h, n, levels.ctypes.data, tx_size, tx_type, qindex, res.ctypes.data,
                                           fl.ctypes.data), "is_test_inverse")
        return res.reshape(n, h, w), fl

    def test_predict(self, plane, params):
        plane = np.ascontiguousarray(plane, np.uint8)
        params = np.ascontiguousarray(params, np.int32)
        n = params.shape[0]
        out = np.zeros((n, 4096), np.uint8)
        self._check(self.L.is_test_predict(self.h, n, plane.ctypes.data, plane.shape[1], plane.shape[0],
                                           params.ctypes.data, out.ctypes.data), "is_test_predict")
        return out

    def debug_analysis(self, bsize, tx_mask=False):
        """Analysis records of one shape of the last encode: J, cand [n x 4], ncand, tx (and the closed loop's tx masks)."""
        n = self.L.is_debug_analysis(self.h, bsize, None, None, None, None, None)
        if n < 0:
            raise RuntimeError("is_debug_analysis failed")
        J, cand = np.zeros(n, np.int64), np.zeros((n, 4), np.uint8)
        nc, tx, tm = np.zeros(n, np.uint8), np.zeros(n, np.uint8), np.zeros(n, np.uint16)
        self.L.is_debug_analysis(self.h, bsize, J.ctypes.data, cand.ctypes.data, nc.ctypes.data, tx.ctypes.data, tm.ctypes.data)
        return (J, cand, nc, tx, tm) if tx_mask else (J, cand, nc, tx)

    def set_trace(self, on=True):
        self._check(self.L.is_set_trace(self.h, 1 if on else 0), "is_set_trace")

    TRACE_STAMPS = 10

    def trace(self):
        """Per queued leaf of the last encode (queue order; in a batch, image 0's format group), 10 values: globaltimer ns
        at slot claimed, slot read, luma prologue done, luma pass 1 done, pass 2 done, luma published, chroma waits done,
        chroma RD done, leaf done; then the queue entry (image << 32 | sb << 8 | leaf)."""
        k = self.TRACE_STAMPS
        n = C.c_uint32()
        self._check(self.L.is_get_trace(self.h, None, 0, C.byref(n)), "is_get_trace")
        out = np.zeros(n.value * k, np.uint64)
        self._check(self.L.is_get_trace(self.h, out.ctypes.data, out.size, C.byref(n)), "is_get_trace")
        return out.reshape(-1, k)

    def debug_leaves(self, sb):
        b, x, y = (np.zeros(256, np.uint8) for _ in range(3))
        n = self.L.is_debug_leaves(self.h, sb, b.ctypes.data, x.ctypes.data, y.ctypes.data)
        if n < 0:
            raise RuntimeError("is_debug_leaves failed")
        return b[:n].copy(), x[:n].copy(), y[:n].copy()
