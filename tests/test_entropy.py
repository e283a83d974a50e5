"""Entropy coding of the records: the device coder (is_encode_obu / is_entropy_batch) against av1core's CPU writer
(av1g_encode, built from the reference sources), byte for byte.  CPU tests check the host side: the OBU framing (sequence
header, frame header, tile sizes) of is_obu_assemble around av1g_encode's own tile payloads, and its refusals; GPU tests
check the device payloads over the formats, qindex range, multi-tile frames and batches."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from av1gpu_b200 import synth
from av1gpu_b200.isearch import IS_ERR_INVALID, IS_ERR_TOO_LARGE, frame_params, load_library, obu_assemble


def _payloads(obu, tiles):
    pay = b"".join(obu[o:o + n] for o, n in tiles)
    off = np.cumsum([0] + [n for _, n in tiles]).astype(np.uint64)
    return pay, off


@pytest.mark.parametrize("w,h,q,bd,c444,seed", [(96, 64, 120, 8, False, 1), (131, 77, 40, 8, False, 2), (64, 48, 200, 10, True, 3),
                                                (40, 24, 90, 10, False, 4), (4160, 40, 60, 8, False, 5)])
def test_obu_framing_matches_av1core(w, h, q, bd, c444, seed):
    """The OBU stream assembled around av1g_encode()'s own tile payloads is av1g_encode()'s stream: the headers, the
    tile-size fields (the 4160-wide frame has two tile columns) and the OBU sizes."""
    im = synth.make_image(w, h, seed, edges=True, bit_depth=bd, chroma_444=c444)
    r = O.encode(im, q, bit_depth=bd, chroma_444=c444, threads=4)
    obu, tiles = O.av1g_obu(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs, bit_depth=bd, chroma_444=c444)
    assert (len(tiles) > 1) == (w > 4096)
    pay, off = _payloads(obu, tiles)
    got = obu_assemble(frame_params(w, h, q, bd, c444), pay, off)
    assert got == obu


# av1g_frame_params offsets of the header-only fields (av1core/include/av1g/decisions.h:254-296)
FP_DQ, FP_EDGE, FP_QM_ON, FP_QM, FP_LF, FP_SHARP, FP_CD, FP_CP, FP_TC, FP_MC = 18, 24, 27, 28, 31, 35, 74, 75, 76, 77


@pytest.mark.parametrize("case", range(8))
def test_obu_framing_header_fields(case):
    """Frame parameters that change only the headers (plane delta_q values with and without separate U / V, quantizer
    matrices, loop-filter levels and sharpness, the intra edge filter flag, colour descriptions incl. the implied-range
    and unspecified forms, 10-bit 4:4:4): the framing still equals av1g_encode()'s stream."""
    rng = np.random.default_rng(100 + case)
    bd, c444 = (10, True) if case in (3, 6) else (8, False)
    w, h, q = 72, 40, 100
    im = synth.make_image(w, h, 900 + case, edges=True, bit_depth=bd, chroma_444=c444)
    r = O.encode(im, q, bit_depth=bd, chroma_444=c444, threads=2)
    fp = frame_params(w, h, q, bd, c444)
    dq = rng.integers(-20, 21, 5).astype(np.int8)
    if case % 2:
        dq[3:] = dq[1:3]                    # V equal to U: no separate_uv_delta_q
    fp[FP_DQ:FP_DQ + 5] = dq.view(np.uint8)
    if case in (2, 5, 6):
        fp[FP_QM_ON] = 1
        fp[FP_QM:FP_QM + 3] = rng.integers(0, 16, 3)
    lv = rng.integers(0, 64, 4)
    if case == 4:
        lv[:] = 0
    fp[FP_LF:FP_LF + 4] = lv
    fp[FP_SHARP] = rng.integers(0, 8)
    fp[FP_EDGE] = case % 2
    cicp = [(1, 13, 6), (1, 13, 0), (2, 2, 2), (9, 16, 9)][case % 4]
    if case >= 4:
        fp[FP_CD] = 1
        fp[FP_CP:FP_CP + 3] = cicp
        if cicp[2] == 0 and not c444:
            fp[FP_CP:FP_CP + 3] = (1, 13, 6)   # identity matrix needs 4:4:4
    want, tiles = O.av1g_obu_fp(fp, r.blocks, r.block_txb, r.txb, r.coeffs)
    pay, off = _payloads(want, tiles)
    assert obu_assemble(fp, pay, off) == want


@pytest.mark.parametrize("bd,c444,bits,seed", [(8, False, 2, 1), (10, True, 3, 2), (8, False, 0, 3)])
def test_obu_framing_with_post_filters(bd, c444, bits, seed):
    """A record with deblocking levels and CDEF (presets, damping, cdef_bits, a cdef_idx per 64x64): the framing around
    av1g_encode()'s payloads (which carry the cdef_idx literals) equals its stream, cdef_params of the frame header
    included."""
    rng = np.random.default_rng(seed)
    w, h, q = 200, 136, 90
    im = synth.make_image(w, h, 40 + seed, edges=True, bit_depth=bd, chroma_444=c444)
    r = O.encode(im, q, bit_depth=bd, chroma_444=c444, threads=4)
    fp = frame_params(w, h, q, bd, c444)
    fp[FP_LF:FP_LF + 4] = rng.integers(1, 64, 4)
    fp[36], fp[37], fp[38] = 1, rng.integers(0, 4), bits          # enable_cdef, cdef_damping_minus_3, cdef_bits
    fp[39:47], fp[55:63] = rng.integers(0, 16, 8), rng.integers(0, 16, 8)
    fp[47:55], fp[63:71] = rng.choice([0, 1, 2, 4], 8), rng.choice([0, 1, 2, 4], 8)
    sbc, sbr = (2 * ((w + 7) // 8) + 15) // 16, (2 * ((h + 7) // 8) + 15) // 16
    sb = rng.integers(0, 1 << bits, sbr * sbc)
    blocks = r.blocks.copy()
    blocks["cdef_idx"] = sb[(blocks["mi_row"].astype(np.int64) >> 4) * sbc + (blocks["mi_col"].astype(np.int64) >> 4)]
    want, tiles = O.av1g_obu_fp(fp, blocks, r.block_txb, r.txb, r.coeffs)
    pay, off = _payloads(want, tiles)
    assert obu_assemble(fp, pay, off) == want


@pytest.mark.parametrize("w,h,bd,c444,cicp,seed", [(96, 64, 8, False, None, 1), (64, 48, 10, True, None, 2), (72, 40, 8, False, (2, 2, 2), 3),
                                                (64, 64, 8, True, (1, 13, 0), 4), (80, 56, 10, False, (9, 16, 9), 5), (4160, 40, 8, False, None, 6)])
def test_avif_matches_av1core(w, h, bd, c444, cicp, seed):
    """The AVIF file around av1g_encode()'s OBU stream equals av1core's av1g_mux_avif (formats, colour descriptions incl.
    unspecified and identity, a two-tile frame's level)."""
    from av1gpu_b200.isearch import avif_mux
    im = synth.make_image(w, h, 60 + seed, edges=True, bit_depth=bd, chroma_444=c444)
    q = 110
    r = O.encode(im, q, bit_depth=bd, chroma_444=c444, threads=4)
    fp = frame_params(w, h, q, bd, c444)
    if cicp:
        fp[FP_CD] = 1
        fp[FP_CP:FP_CP + 3] = cicp
    obu, _ = O.av1g_obu_fp(fp, r.blocks, r.block_txb, r.txb, r.coeffs)
    assert avif_mux(fp, obu) == O.mux_avif(obu, w, h)


def test_obu_assemble_refusals():
    """Frames outside the coder's toolset, a tile count that does not match the tiling, and a short buffer."""
    L = load_library()
    pay = np.zeros(8, np.uint8)
    off = np.array([0, 8], np.uint64)
    size = C.c_uint64()
    fp = frame_params(64, 64, 100)
    assert L.is_obu_assemble(fp.ctypes.data, pay.ctypes.data, off.ctypes.data, 1, None, 0, C.byref(size)) == IS_ERR_TOO_LARGE
    assert size.value > 8
    two = np.array([0, 4, 8], np.uint64)
    assert L.is_obu_assemble(fp.ctypes.data, pay.ctypes.data, two.ctypes.data, 2, None, 0, C.byref(size)) == IS_ERR_INVALID
    for k, v in ((13, 0), (72, 2), (73, 12), (12, 1)):   # lossless, bad chroma format, bad bit depth, monochrome
        bad = fp.copy()
        bad[k] = v
        assert L.is_obu_assemble(bad.ctypes.data, pay.ctypes.data, off.ctypes.data, 1, None, 0, C.byref(size)) == IS_ERR_INVALID


def test_entropy_scratch_refusals():
    """The device entry points refuse bad frames before any GPU work (no GPU needed)."""
    L = load_library()
    b = C.c_uint64()
    assert L.is_entropy_scratch_bytes(None, 1, 0, C.byref(b)) == IS_ERR_INVALID
    assert L.is_entropy_scratch_bytes(None, 0, 0, C.byref(b)) == IS_ERR_INVALID


# ---------------------------------------------------------------------------------------------------------------
# GPU: the device coder's payloads against av1g_encode
# ---------------------------------------------------------------------------------------------------------------
GPU_CASES = [(320, 240, 120, 8, False, 11), (333, 197, 40, 8, False, 12), (256, 160, 220, 8, False, 13),
             (200, 128, 60, 10, False, 14), (192, 128, 100, 8, True, 15), (160, 96, 160, 10, True, 16),
             (4160, 64, 90, 8, False, 17), (16, 16, 120, 8, False, 18)]


def _check(enc, im, w, h, q, bd, c444):
    r = enc.encode(im, q)
    want, tiles = O.av1g_obu(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs, bit_depth=bd, chroma_444=c444)
    got = enc.obu()[0]
    if got != want:   # name the first differing tile for the report
        n = min(len(got), len(want))
        first = next((i for i in range(n) if got[i] != want[i]), n)
        tile = next((k for k, (o, s) in enumerate(tiles) if o <= first < o + s), None)
        raise AssertionError("OBU differs at byte %d of %d / %d (tile %s of %d)" % (first, len(got), len(want), tile, len(tiles)))


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,q,bd,c444,seed", GPU_CASES)
def test_device_entropy_matches_av1core(enc, w, h, q, bd, c444, seed):
    im = synth.make_image(w, h, seed, edges=True, bit_depth=bd, chroma_444=c444)
    _check(enc, im, w, h, q, bd, c444)


@pytest.mark.gpu
def test_device_entropy_reference_picture(enc):
    """The reference's CfL test picture at three qindex values."""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "gate_cfl_edge_211x149.npz"))
    im = (g["y"], g["u"], g["v"])
    for q in (60, 120, 200):
        _check(enc, im, 211, 149, q, 8, False)


@pytest.mark.gpu
def test_device_entropy_batch(enc):
    """Nine images of mixed sizes, formats and qindex searched as one batch and entropy-coded in one device call: every
    stream equals av1g_encode() of that image's record."""
    spec = [(96, 64, 80, 8, False), (130, 70, 150, 8, False), (64, 64, 60, 10, True), (200, 40, 200, 8, False),
            (48, 200, 30, 10, False), (128, 96, 120, 8, True), (24, 24, 250, 8, False), (300, 180, 100, 8, False),
            (72, 56, 45, 10, True)]
    ims = [synth.make_image(w, h, 500 + i, edges=True, bit_depth=bd, chroma_444=c) for i, (w, h, _, bd, c) in enumerate(spec)]
    recs = enc.encode_batch(ims, [s[2] for s in spec])
    streams, ms = enc.obu(0, len(spec), timed=True)
    assert ms > 0
    for (w, h, q, bd, c), r, got in zip(spec, recs, streams):
        want, _ = O.av1g_obu(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs, bit_depth=bd, chroma_444=c)
        assert got == want
    # a sub-range of the batch
    assert enc.obu(3, 2) == streams[3:5]
    # the AVIF files of the batch: av1core's container around the same streams
    for (w, h, q, bd, c), got, f in zip(spec, streams, enc.avif(0, len(spec))):
        assert f == O.mux_avif(got, w, h)


@pytest.mark.gpu
def test_device_entropy_speed(enc):
    """The 12 MP bench picture at qindex 120: the device coder's kernel time (CUDA events) against av1core's CPU writer
    (av1g_encode, bitstream only, one host thread) on the same record; the streams are equal."""
    import json
    import time
    w, h, q = 4000, 3000, 120
    r = enc.encode(synth.make_image(w, h, 12, edges=True), q)
    ms = min(enc.obu(timed=True)[1] for _ in range(3))
    t0 = time.perf_counter()
    want, tiles, nsym = O.av1g_obu(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs, symbols=True)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    assert enc.obu()[0] == want
    print(json.dumps({"image": "%dx%d q%d" % (w, h, q), "tiles": len(tiles), "symbols": nsym, "bytes": len(want),
                      "device_ms": round(ms, 1), "cpu_av1g_encode_ms": round(cpu_ms, 1),
                      "ns_per_symbol_per_tile": round(ms * 1e6 / (nsym / len(tiles)), 1)}))
    assert ms < cpu_ms


class _DevBytes:
    """A device byte range as a __cuda_array_interface__ object (torch.as_tensor reads it without a copy)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "|u1", "data": (int(ptr), False), "version": 3}


@pytest.mark.gpu
def test_device_entropy_rejects_bad_records(enc):
    """is_entropy_batch on a record whose blocks are out of decode order, or whose luma tx type is outside its tx set,
    reports IS_ENT_ERR_RECORD in the device status head (no payload); the intact record codes to av1g_encode()'s
    payload through the same entry point."""
    import torch
    w, h, q = 128, 64, 100
    im = synth.make_image(w, h, 7, edges=True)
    r = enc.encode(im, q)
    L = load_library()

    class EntFrame(C.Structure):
        _fields_ = [("fp", C.c_uint8 * 88), ("blocks", C.c_void_p), ("block_txb", C.c_void_p), ("txb", C.c_void_p),
                    ("coeffs", C.c_void_p), ("n_blocks", C.c_uint32), ("n_txb", C.c_uint32)]

    class EntOut(C.Structure):
        _fields_ = [("result", C.c_void_p), ("result_bytes", C.c_uint64), ("payload", C.c_void_p),
                    ("payload_capacity", C.c_uint64), ("n_tiles", C.c_uint32)]

    def run(blocks, txb):
        d = [torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda() for a in (blocks, r.block_txb, txb, r.coeffs)]
        f = EntFrame()
        f.fp[:] = frame_params(w, h, q).tolist()
        f.blocks, f.block_txb, f.txb, f.coeffs = (t.data_ptr() for t in d)
        f.n_blocks, f.n_txb = len(blocks), len(txb)
        nb = C.c_uint64()
        assert L.is_entropy_scratch_bytes(C.byref(f), 1, 0, C.byref(nb)) == 0
        scratch = torch.empty(nb.value + 256, dtype=torch.uint8, device="cuda")
        base = (scratch.data_ptr() + 255) & ~255
        out = EntOut()
        t0 = (C.c_uint32 * 2)()
        torch.cuda.synchronize()
        assert L.is_entropy_batch(0, C.byref(f), 1, 0, base, nb.value, None, C.byref(out), t0) == 0
        torch.cuda.synchronize()
        head = torch.as_tensor(_DevBytes(out.result, out.result_bytes), device="cuda").cpu().numpy()
        err = int(head[:4].view(np.int32)[0])
        nbytes = int(head[24:32].view(np.uint64)[0])
        pay = torch.as_tensor(_DevBytes(out.payload, nbytes), device="cuda").cpu().numpy().tobytes() if not err else b""
        assert out.n_tiles == 1 and list(t0) == [0, 1]
        return err, pay

    err, pay = run(r.blocks, r.txb)
    want, tiles = O.av1g_obu(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs)
    assert err == 0 and pay == want[tiles[0][0]:tiles[0][0] + tiles[0][1]]
    swapped = r.blocks.copy()
    swapped[[1, 2]] = swapped[[2, 1]]
    assert run(swapped, r.txb)[0] == 4
    bad = r.txb.copy()
    k = next(i for i in range(len(bad)) if bad[i]["plane"] == 0 and not r.blocks[np.searchsorted(r.block_txb, i, "right") - 1]["skip"]
             and np.any(r.coeffs[bad[i]["coeff_off"]:bad[i]["coeff_off"] + 16]))
    bad[k]["tx_type"] = 4   # FLIPADST_DCT: in no intra tx set
    assert run(r.blocks, bad)[0] == 4
