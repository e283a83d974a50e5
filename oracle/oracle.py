"""ctypes wrapper of the CPU oracle (oracle/_ref/liboracle.so).  TEST INFRASTRUCTURE ONLY: imported by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker, never by the product."""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "liboracle.so")

# av1core DecisionRecord POD layouts (av1core/include/av1g/decisions.h:225-252)
BLOCK_DT = np.dtype([("mi_row", "<u2"), ("mi_col", "<u2"), ("bsize", "u1"), ("skip", "u1"), ("tx_depth", "u1"),
                     ("y_mode", "u1"), ("angle_delta_y", "i1"), ("uv_mode", "u1"), ("angle_delta_uv", "i1"),
                     ("cfl_alpha_u", "i1"), ("cfl_alpha_v", "i1"), ("filter_intra", "u1"), ("cdef_idx", "i1"),
                     ("sb_qindex", "u1")])
TXB_DT = np.dtype([("coeff_off", "<u4"), ("x4", "<u2"), ("y4", "<u2"), ("plane", "u1"), ("tx_size", "u1"),
                   ("tx_type", "u1"), ("flags", "u1"), ("eob", "<u2"), ("reserved", "<u2")])
assert BLOCK_DT.itemsize == 16 and TXB_DT.itemsize == 16


class OrcImage(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("bit_depth", C.c_int), ("chroma_444", C.c_int),
                ("qindex", C.c_int), ("planes", C.c_void_p * 3), ("stride", C.c_int * 3)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("oracle library missing: build it with `make -C oracle` (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        L.orc_encode.argtypes = [C.POINTER(OrcImage), C.c_int, C.POINTER(C.c_void_p)]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_counts.argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]
        L.orc_copy_record.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_copy_recon.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.orc_analysis.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_analysis.restype = C.c_uint32
        L.orc_leaves.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_av1g_recon_arrays.argtypes = [C.c_int] * 5 + [C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                                            C.c_uint64, C.c_void_p, C.c_void_p * 3, C.c_char_p,
                                                            C.c_size_t, C.POINTER(C.c_uint64)]
        L.orc_av1g_obu_arrays.argtypes = [C.c_int] * 5 + [C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                                          C.c_uint64, C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64),
                                                          C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p, C.c_uint32,
                                                          C.POINTER(C.c_uint64), C.c_char_p, C.c_size_t]
        L.orc_av1g_obu_fp.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p,
                                      C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.c_void_p, C.c_void_p,
                                      C.c_uint32, C.POINTER(C.c_uint64), C.c_char_p, C.c_size_t]
        L.orc_set_uv_open_loop.argtypes = [C.c_int]
        L.orc_set_edge_filter.argtypes = [C.c_int]
        L.orc_mux_avif.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]
        L.orc_ref_lf_from_q.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_av1g_encode_fp.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                         C.c_uint64, C.c_void_p, C.c_void_p * 3, C.c_char_p, C.c_size_t]
        L.orc_av1g_postfilter.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p * 3, C.c_int * 3]
        L.orc_fwd2d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.orc_inv2d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.orc_inv2d.restype = C.c_uint32
        L.orc_quant_rate.argtypes = [C.c_void_p] + [C.c_int] * 10 + [C.c_int64, C.c_void_p, C.POINTER(C.c_int64),
                                                                     C.POINTER(C.c_int64), C.POINTER(C.c_int)]
        L.orc_cost_table.argtypes = [C.c_int, C.c_void_p, C.c_size_t]
        L.orc_cost_table.restype = C.c_size_t
        L.orc_avg_bits.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_lambda.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_predict.argtypes = [C.c_void_p] + [C.c_int] * 13 + [C.c_void_p]
        L.orc_op_counts.argtypes = [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.orc_qstep.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_ref_engine.argtypes = [C.POINTER(OrcImage), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib = L
    return _lib


def _image(planes, qindex, bit_depth=8, chroma_444=False):
    y = planes[0]
    img = OrcImage()
    img.width, img.height = y.shape[1], y.shape[0]
    img.bit_depth, img.chroma_444, img.qindex = bit_depth, int(chroma_444), qindex
    for p in range(3):
        a = planes[p]
        assert a.flags["C_CONTIGUOUS"]
        img.planes[p] = a.ctypes.data
        img.stride[p] = a.shape[1]
    return img


class Result:
    """Decisions, record and reconstruction of one oracle run."""

    def __init__(self, handle, width, height, bit_depth, chroma_444, qindex):
        self.h = handle
        self.width, self.height, self.bit_depth, self.chroma_444, self.qindex = width, height, bit_depth, chroma_444, qindex
        L = lib()
        nb, nt, nc = C.c_uint32(), C.c_uint32(), C.c_uint64()
        L.orc_counts(handle, C.byref(nb), C.byref(nt), C.byref(nc))
        self.blocks = np.zeros(nb.value, BLOCK_DT)
        self.block_txb = np.zeros(nb.value + 1, np.uint32)
        self.txb = np.zeros(nt.value, TXB_DT)
        self.coeffs = np.zeros(nc.value, np.int16)
        L.orc_copy_record(handle, None, self.blocks.ctypes.data, self.block_txb.ctypes.data, self.txb.ctypes.data,
                          self.coeffs.ctypes.data)
        dt = np.uint16 if bit_depth == 10 else np.uint8
        cw, ch = (width, height) if chroma_444 else ((width + 1) // 2, (height + 1) // 2)
        self.recon = []
        for p, (w, h) in enumerate(((width, height), (cw, ch), (cw, ch))):
            a = np.zeros((h, w), dt)
            L.orc_copy_recon(handle, p, a.ctypes.data)
            self.recon.append(a)

    def analysis(self, bsize):
        L = lib()
        n = L.orc_analysis(self.h, bsize, None, None, None, None)
        J = np.zeros(n, np.int64)
        cand = np.zeros((n, 4), np.uint8)
        ncand = np.zeros(n, np.uint8)
        tx = np.zeros(n, np.uint8)
        L.orc_analysis(self.h, bsize, J.ctypes.data, cand.ctypes.data, ncand.ctypes.data, tx.ctypes.data)
        return J, cand, ncand, tx

    def leaves(self, sb):
        L = lib()
        b, x, y = (np.zeros(256, np.uint8) for _ in range(3))
        n = L.orc_leaves(self.h, sb, b.ctypes.data, x.ctypes.data, y.ctypes.data)
        return b[:n].copy(), x[:n].copy(), y[:n].copy()

    def op_counts(self):
        """Algorithmic INT32 operations of this search: (open-loop analysis, closed loop)."""
        a, c = C.c_uint64(), C.c_uint64()
        lib().orc_op_counts(self.h, C.byref(a), C.byref(c))
        return a.value, c.value

    def __del__(self):
        try:
            lib().orc_free(self.h)
        except Exception:
            pass


def encode(planes, qindex, bit_depth=8, chroma_444=False, threads=None):
    img = _image(planes, qindex, bit_depth, chroma_444)
    h = C.c_void_p()
    rc = lib().orc_encode(C.byref(img), threads or os.cpu_count() or 1, C.byref(h))
    if rc != 0:
        raise RuntimeError("orc_encode failed: %d" % rc)
    return Result(h.value, img.width, img.height, bit_depth, bool(chroma_444), qindex)


def av1g_recon(width, height, qindex, blocks, block_txb, txb, coeffs, bit_depth=8, chroma_444=False):
    """av1core's reconstruction (av1g_layout check + av1g_encode) of a record: (planes, OBU bytes)."""
    dt = np.uint16 if bit_depth == 10 else np.uint8
    cw, ch = (width, height) if chroma_444 else ((width + 1) // 2, (height + 1) // 2)
    outs = [np.zeros((height, width), dt), np.zeros((ch, cw), dt), np.zeros((ch, cw), dt)]
    ptrs = (C.c_void_p * 3)(*[o.ctypes.data for o in outs])
    err = C.create_string_buffer(256)
    nbytes = C.c_uint64()
    blocks = np.ascontiguousarray(blocks)
    block_txb = np.ascontiguousarray(block_txb, np.uint32)
    txb = np.ascontiguousarray(txb).copy()
    coeffs = np.ascontiguousarray(coeffs, np.int16).copy()
    rc = lib().orc_av1g_recon_arrays(width, height, qindex, bit_depth, int(chroma_444), len(blocks), blocks.ctypes.data,
                                     block_txb.ctypes.data, len(txb), txb.ctypes.data, len(coeffs), coeffs.ctypes.data,
                                     ptrs, err, 256, C.byref(nbytes))
    if rc != 0:
        raise RuntimeError("av1g_encode rejected the record (%d): %s" % (rc, err.value.decode(errors="replace")))
    return outs, nbytes.value


def av1g_obu(width, height, qindex, blocks, block_txb, txb, coeffs, bit_depth=8, chroma_444=False, symbols=False):
    """av1g_encode()'s OBU stream of a record (bytes) and the tile payloads' (offset, size) in it, from av1g_parse();
    with symbols=True also the number of symbols av1g_encode() coded."""
    blocks = np.ascontiguousarray(blocks)
    block_txb = np.ascontiguousarray(block_txb, np.uint32)
    txb = np.ascontiguousarray(txb).copy()
    coeffs = np.ascontiguousarray(coeffs, np.int16).copy()
    err = C.create_string_buffer(256)
    size, nt, nsym = C.c_uint64(), C.c_uint32(), C.c_uint64()
    toff, tby = np.zeros(4096, np.uint64), np.zeros(4096, np.uint32)
    args = (width, height, qindex, bit_depth, int(chroma_444), len(blocks), blocks.ctypes.data, block_txb.ctypes.data, len(txb),
            txb.ctypes.data, len(coeffs), coeffs.ctypes.data)
    rc = lib().orc_av1g_obu_arrays(*args, None, 0, C.byref(size), C.byref(nt), toff.ctypes.data, tby.ctypes.data, 4096, C.byref(nsym),
                                   err, 256)
    if rc != 0:
        raise RuntimeError("av1g_encode rejected the record (%d): %s" % (rc, err.value.decode(errors="replace")))
    obu = np.zeros(size.value, np.uint8)
    rc = lib().orc_av1g_obu_arrays(*args, obu.ctypes.data, size.value, C.byref(size), C.byref(nt), toff.ctypes.data, tby.ctypes.data,
                                   4096, None, err, 256)
    if rc != 0:
        raise RuntimeError("av1g_encode rejected the record (%d): %s" % (rc, err.value.decode(errors="replace")))
    tiles = [(int(toff[i]), int(tby[i])) for i in range(nt.value)]
    return (obu.tobytes(), tiles, nsym.value) if symbols else (obu.tobytes(), tiles)


AV1G_ENC_PREFILTER_RECON = 0x20


def av1g_obu_fp(fp, blocks, block_txb, txb, coeffs):
    """av1g_encode()'s OBU stream of a record with frame parameters fp (av1g_frame_params bytes) and its tile payloads'
    (offset, size)."""
    fp = np.ascontiguousarray(fp, np.uint8)
    blocks = np.ascontiguousarray(blocks)
    block_txb = np.ascontiguousarray(block_txb, np.uint32)
    txb = np.ascontiguousarray(txb).copy()
    coeffs = np.ascontiguousarray(coeffs, np.int16).copy()
    err = C.create_string_buffer(256)
    size, nt = C.c_uint64(), C.c_uint32()
    toff, tby = np.zeros(4096, np.uint64), np.zeros(4096, np.uint32)
    args = (fp.ctypes.data, len(blocks), blocks.ctypes.data, block_txb.ctypes.data, len(txb), txb.ctypes.data, len(coeffs), coeffs.ctypes.data)
    for obu in (None, True):
        buf = np.zeros(size.value, np.uint8) if obu else None
        rc = lib().orc_av1g_obu_fp(*args, None if buf is None else buf.ctypes.data, size.value if obu else 0, C.byref(size), C.byref(nt),
                                   toff.ctypes.data, tby.ctypes.data, 4096, None, err, 256)
        if rc != 0:
            raise RuntimeError("av1g_encode rejected the record (%d): %s" % (rc, err.value.decode(errors="replace")))
    return buf.tobytes(), [(int(toff[i]), int(tby[i])) for i in range(nt.value)]


def av1g_encode_fp(fp, blocks, block_txb, txb, coeffs, prefilter=False):
    """av1g_encode() of a record with frame parameters fp (av1g_frame_params bytes): the reconstruction planes, cropped
    and post-filtered, or (prefilter) the unfiltered coded area (MiCols * 4 x MiRows * 4, chroma subsampled)."""
    fp = np.ascontiguousarray(fp, np.uint8)
    w, h = (int(v) for v in fp[4:12].view(np.uint32))
    c444, bd = int(fp[72]) == 1, 10 if int(fp[73]) == 10 else 8
    if prefilter:
        w, h = 8 * ((w + 7) // 8), 8 * ((h + 7) // 8)
    cw, ch = (w, h) if c444 else ((w + 1) // 2, (h + 1) // 2)
    dt = np.uint16 if bd == 10 else np.uint8
    outs = [np.zeros((h, w), dt), np.zeros((ch, cw), dt), np.zeros((ch, cw), dt)]
    err = C.create_string_buffer(256)
    blocks = np.ascontiguousarray(blocks)
    txb = np.ascontiguousarray(txb).copy()
    coeffs = np.ascontiguousarray(coeffs, np.int16).copy()
    block_txb = np.ascontiguousarray(block_txb, np.uint32)
    rc = lib().orc_av1g_encode_fp(fp.ctypes.data, AV1G_ENC_PREFILTER_RECON if prefilter else 0, len(blocks), blocks.ctypes.data,
                                  block_txb.ctypes.data, len(txb), txb.ctypes.data, len(coeffs), coeffs.ctypes.data,
                                  (C.c_void_p * 3)(*[o.ctypes.data for o in outs]), err, 256)
    if rc != 0:
        raise RuntimeError("av1g_encode rejected the record (%d): %s" % (rc, err.value.decode(errors="replace")))
    return outs


def mux_avif(obu, width, height):
    """av1core's AVIF file (av1g_mux_avif) around an OBU stream (bytes)."""
    src = np.frombuffer(obu, np.uint8)
    size = C.c_uint64()
    rc = lib().orc_mux_avif(src.ctypes.data, len(src), width, height, None, 0, C.byref(size))
    if rc != 0:
        raise RuntimeError("av1g_mux_avif failed (%d)" % rc)
    out = np.zeros(size.value, np.uint8)
    lib().orc_mux_avif(src.ctypes.data, len(src), width, height, out.ctypes.data, size.value, C.byref(size))
    return out.tobytes()


def set_edge_filter(on):
    """Experiment switch of the oracle: the search with the intra edge filter (records for enable_intra_edge_filter 1)."""
    lib().orc_set_edge_filter(1 if on else 0)


def set_uv_open_loop(on):
    """Experiment switch of the oracle: chroma screening on source edges (the reference's open-loop chroma shortlist)."""
    lib().orc_set_uv_open_loop(1 if on else 0)


def ref_lf_from_q(base, bit_depth=8):
    """The reference's default deblocking level (effective, with the intra delta), sharpness and CDEF damping."""
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    lib().orc_ref_lf_from_q(base, bit_depth, C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


def av1g_postfilter(fp, blocks, planes):
    """av1core's deblocking + CDEF in place on planes (numpy, at least the coded area) for the record's blocks."""
    fp = np.ascontiguousarray(fp, np.uint8)
    blocks = np.ascontiguousarray(blocks)
    rc = lib().orc_av1g_postfilter(fp.ctypes.data, len(blocks), blocks.ctypes.data, (C.c_void_p * 3)(*[p.ctypes.data for p in planes]),
                                   (C.c_int * 3)(*[p.strides[0] // p.itemsize for p in planes]))
    if rc != 0:
        raise RuntimeError("av1g_postfilter failed (%d)" % rc)


def fwd2d(res, tx_size, tx_type, bit_depth=8):
    res = np.ascontiguousarray(res, np.int32)
    h, w = res.shape
    out = np.zeros((min(h, 32), min(w, 32)), np.int32)
    lib().orc_fwd2d(res.ctypes.data, tx_size, tx_type, bit_depth, out.ctypes.data)
    return out


def inv2d(levels, tx_size, tx_type, dcq, acq, w, h, bit_depth=8):
    levels = np.ascontiguousarray(levels, np.int16)
    out = np.zeros((h, w), np.int32)
    err = lib().orc_inv2d(levels.ctypes.data, tx_size, tx_type, bit_depth, dcq, acq, out.ctypes.data)
    return out, err


def quant_rate(coef, tx_size, tx_type, plane, dcq, acq, skip_ctx, dc_ctx, intra_dir, qctx, res_energy=0, bit_depth=8):
    coef = np.ascontiguousarray(coef, np.int32)
    lv = np.zeros(coef.size, np.int16)
    D, R, eob = C.c_int64(), C.c_int64(), C.c_int()
    lib().orc_quant_rate(coef.ctypes.data, tx_size, tx_type, plane, bit_depth, dcq, acq, skip_ctx, dc_ctx, intra_dir, qctx,
                         res_energy, lv.ctypes.data, C.byref(D), C.byref(R), C.byref(eob))
    return lv.reshape(coef.shape), D.value, R.value, eob.value


def cost_table(qctx):
    n = lib().orc_cost_table(qctx, None, 0)
    out = np.zeros(n, np.uint16)
    lib().orc_cost_table(qctx, out.ctypes.data, n)
    return out


def avg_bits():
    y, p, s = np.zeros(13, np.int32), np.zeros(50, np.int32), np.zeros(1, np.int32)
    lib().orc_avg_bits(y.ctypes.data, p.ctypes.data, s.ctypes.data)
    return y, p.reshape(5, 10), int(s[0])


def lam(qindex, bit_depth=8):
    a, b = C.c_int64(), C.c_int64()
    lib().orc_lambda(qindex, bit_depth, C.byref(a), C.byref(b))
    return a.value, b.value


def ref_engine_seconds(planes, qindex):
    """The reference's own CPU decision engine (ref_engine_encode): (decide s, encode s)."""
    img = _image(planes, qindex)
    d, e = C.c_double(), C.c_double()
    rc = lib().orc_ref_engine(C.byref(img), C.byref(d), C.byref(e))
    if rc != 0:
        raise RuntimeError("ref_engine_encode failed: %d" % rc)
    return d.value, e.value


def qstep(qindex, bit_depth=8):
    """(dc_q, ac_q) of a qindex (av1core's spec tables)."""
    d, a = C.c_int(), C.c_int()
    lib().orc_qstep(qindex, bit_depth, C.byref(d), C.byref(a))
    return d.value, a.value
