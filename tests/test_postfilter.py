"""The post-filters (deblocking, spec 7.14, then CDEF, spec 7.15): the library's filter arithmetic
(av1gpu_b200/csrc/is_postfilter.cuh) against av1core's av1g_postfilter, the reference's CPU post-filter, on the CPU
through a host build of the same functions (tests/pf_host.cpp); on the GPU, is_postfilter on a searched image's
reconstruction against av1g_encode() of the record with the same filter parameters."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from av1gpu_b200 import synth
from av1gpu_b200.isearch import frame_params

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# av1g_frame_params field offsets (av1core/include/av1g/decisions.h:254-296)
FP_LF, FP_SHARP, FP_CDEF, FP_DAMP, FP_BITS, FP_YPRI, FP_YSEC, FP_UVPRI, FP_UVSEC = 31, 35, 36, 37, 38, 39, 47, 55, 63


def filter_params(w, h, q, bd, c444, rng, cdef=True):
    """The frame parameters of a picture with seeded deblocking levels / sharpness and CDEF presets."""
    fp = frame_params(w, h, q, bd, c444)
    lv = rng.integers(0, 64, 4)
    if rng.random() < 0.2:
        lv[1] = 0                                  # luma horizontal edges off
    if not lv[0] and not lv[1]:
        lv[0] = 1                                  # chroma levels need a luma level
    fp[FP_LF:FP_LF + 4] = lv
    fp[FP_SHARP] = rng.integers(0, 8)
    if cdef:
        fp[FP_CDEF] = 1
        fp[FP_DAMP] = rng.integers(0, 4)
        fp[FP_BITS] = rng.integers(0, 4)
        fp[FP_YPRI:FP_YPRI + 8] = rng.integers(0, 16, 8)
        fp[FP_UVPRI:FP_UVPRI + 8] = rng.integers(0, 16, 8)
        fp[FP_YSEC:FP_YSEC + 8] = rng.choice([0, 1, 2, 4], 8)
        fp[FP_UVSEC:FP_UVSEC + 8] = rng.choice([0, 1, 2, 4], 8)
    return fp


def sb_cdef_map(w, h, fp, rng):
    sbc, sbr = (2 * ((w + 7) // 8) + 15) // 16, (2 * ((h + 7) // 8) + 15) // 16
    return rng.integers(0, 1 << int(fp[FP_BITS]), sbr * sbc).astype(np.int8), sbc


def with_cdef_idx(blocks, sb, sbc):
    b = blocks.copy()
    b["cdef_idx"] = sb[(b["mi_row"].astype(np.int64) >> 4) * sbc + (b["mi_col"].astype(np.int64) >> 4)]
    return b


_harness = None


def harness():
    """tests/pf_host.cpp built by oracle/Makefile (with the oracle, by the package build); rebuilt here when the av1core
    headers are at hand and the sources are newer."""
    global _harness
    if _harness is None:
        from av1gpu_b200 import build
        out = os.path.join(ROOT, "oracle", "_ref", "libpfhost.so")
        src = os.path.join(HERE, "pf_host.cpp")
        hdr = os.path.join(ROOT, "av1gpu_b200", "csrc", "is_postfilter.cuh")
        stale = not os.path.exists(out) or os.path.getmtime(out) < max(os.path.getmtime(src), os.path.getmtime(hdr))
        if stale and build.REF and os.path.isdir(build.REF):
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "REF=" + build.REF, "_ref/libpfhost.so"], check=True)
        elif not os.path.exists(out):
            pytest.skip("the post-filter host harness is not built (oracle/Makefile with the reference checkout)")
        L = C.CDLL(out)
        L.pfh_apply.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p * 3, C.c_int * 3]
        _harness = L
    return _harness


@pytest.mark.parametrize("w,h,q,bd,c444,seed", [(96, 80, 120, 8, False, 1), (131, 77, 60, 8, False, 2), (72, 64, 200, 10, False, 3),
                                                (64, 56, 90, 8, True, 4), (80, 48, 160, 10, True, 5), (200, 136, 40, 8, False, 6)])
def test_postfilter_arithmetic_matches_av1core(w, h, q, bd, c444, seed):
    """Deblocking and CDEF of the library's functions (host build) equal av1g_postfilter on the unfiltered coded area of
    an oracle record, over seeded levels, sharpness, damping and CDEF presets (three parameter draws per record, one
    without CDEF)."""
    L = harness()
    rng = np.random.default_rng(seed)
    im = synth.make_image(w, h, seed, edges=True, bit_depth=bd, chroma_444=c444)
    r = O.encode(im, q, bit_depth=bd, chroma_444=c444, threads=4)
    for k in range(3):
        fp = filter_params(w, h, q, bd, c444, rng, cdef=k != 2)
        sb, sbc = sb_cdef_map(w, h, fp, rng)
        blocks = with_cdef_idx(r.blocks, sb, sbc)
        pre = O.av1g_encode_fp(fp, blocks, r.block_txb, r.txb, r.coeffs, prefilter=True)
        want = [p.copy() for p in pre]
        O.av1g_postfilter(fp, blocks, want)
        got = [p.copy() for p in pre]
        L.pfh_apply(fp.ctypes.data, blocks.ctypes.data, len(blocks), (C.c_void_p * 3)(*[p.ctypes.data for p in got]),
                    (C.c_int * 3)(*[p.strides[0] // p.itemsize for p in got]))
        for p in range(3):
            assert np.array_equal(got[p], want[p]), (k, p, int(np.sum(got[p] != want[p])))
        assert any(not np.array_equal(want[p], pre[p]) for p in range(3))   # the filters did change the picture


def test_postfilter_arithmetic_bench_picture():
    """The 12 MP bench picture (4000x3000, qindex 120, the oracle's record): deblocking with the reference's default
    levels (level from Q) and CDEF with seeded presets, the host build of the library's functions against av1g_postfilter
    over the whole coded area."""
    from av1gpu_b200.isearch import postfilter_from_q
    L = harness()
    rng = np.random.default_rng(77)
    w, h, q = 4000, 3000, 120
    im = synth.make_image(w, h, 12, edges=True)
    r = O.encode(im, q)
    fp = filter_params(w, h, q, 8, False, rng)
    fp = postfilter_from_q(fp, q, 8)
    sb, sbc = sb_cdef_map(w, h, fp, rng)
    blocks = with_cdef_idx(r.blocks, sb, sbc)
    pre = O.av1g_encode_fp(fp, blocks, r.block_txb, r.txb, r.coeffs, prefilter=True)
    want = [p.copy() for p in pre]
    O.av1g_postfilter(fp, blocks, want)
    got = [p.copy() for p in pre]
    L.pfh_apply(fp.ctypes.data, blocks.ctypes.data, len(blocks), (C.c_void_p * 3)(*[p.ctypes.data for p in got]),
                (C.c_int * 3)(*[p.strides[0] // p.itemsize for p in got]))
    for p in range(3):
        assert np.array_equal(got[p], want[p]), (p, int(np.sum(got[p] != want[p])))


def test_postfilter_from_q_matches_reference():
    """is_postfilter_from_q (the reference's default deblocking: level from Q with the intra delta, sharpness, CDEF
    damping) equals the reference's own av1f_tuneiq_frame_init for every qindex at 8 and 10 bits."""
    from av1gpu_b200.isearch import postfilter_from_q
    for bd in (8, 10):
        for q in range(1, 256):
            fp = postfilter_from_q(frame_params(64, 64, q, bd), q, bd)
            lvl, sharp, damp = O.ref_lf_from_q(q, bd)
            assert list(fp[FP_LF:FP_LF + 4]) == [lvl] * 4 and fp[FP_SHARP] == sharp and fp[FP_DAMP] + 3 == damp, (bd, q)


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,q,bd,c444,seed", [(320, 240, 120, 8, False, 11), (211, 149, 60, 8, False, 12), (192, 128, 100, 10, False, 13),
                                                (160, 96, 80, 8, True, 14), (128, 96, 150, 10, True, 15)])
def test_device_postfilter_matches_av1core(enc, w, h, q, bd, c444, seed):
    """is_postfilter on the searched image's reconstruction equals av1g_encode()'s filtered reconstruction of the record
    with the same parameters (the record's cdef_idx written by the call)."""
    rng = np.random.default_rng(seed)
    im = synth.make_image(w, h, seed, edges=True, bit_depth=bd, chroma_444=c444)
    r = enc.encode(im, q)
    fp = filter_params(w, h, q, bd, c444, rng)
    sb, sbc = sb_cdef_map(w, h, fp, rng)
    ms = enc.postfilter(fp, sb)
    assert ms > 0
    got = enc.fetch(w, h, q, bit_depth=bd, chroma_444=c444)
    assert np.array_equal(got.blocks["cdef_idx"], with_cdef_idx(r.blocks, sb, sbc)["cdef_idx"])
    want = O.av1g_encode_fp(fp, got.blocks, got.block_txb, got.txb, got.coeffs)
    for p in range(3):
        assert np.array_equal(got.recon[p], want[p]), (p, int(np.sum(got.recon[p] != want[p])))
    assert any(not np.array_equal(got.recon[p], r.recon[p]) for p in range(3))


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,q,bd,c444,seed", [(256, 160, 110, 8, False, 21), (144, 112, 70, 10, True, 22)])
def test_device_postfilter_then_bitstream(enc, w, h, q, bd, c444, seed):
    """Search, post-filters, then the device entropy coder: the OBU stream signals the filters (frame header levels and
    cdef_params, each SB's cdef_idx literal) and equals av1g_encode()'s stream of the record with the same parameters."""
    rng = np.random.default_rng(seed)
    im = synth.make_image(w, h, seed, edges=True, bit_depth=bd, chroma_444=c444)
    enc.encode(im, q)
    fp = filter_params(w, h, q, bd, c444, rng)
    sb, sbc = sb_cdef_map(w, h, fp, rng)
    enc.postfilter(fp, sb)
    got = enc.fetch(w, h, q, bit_depth=bd, chroma_444=c444)
    want, _ = O.av1g_obu_fp(fp, got.blocks, got.block_txb, got.txb, got.coeffs)
    assert enc.obu()[0] == want

