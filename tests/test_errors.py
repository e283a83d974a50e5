"""The library's error paths: argument checks (IS_ERR_INVALID), the workspace budget (IS_ERR_OOM), closed-loop waits
that run out (IS_ERR_TIMEOUT, with no hang), reads of state that does not exist (IS_ERR_STATE), and poison mode (every
workspace byte and every kernel's shared memory start as garbage: the results must not change).

The checks that return before any GPU work run on the CPU; the rest need the GPU.  A failed encode leaves the handle
usable: the next encode with sane settings gives the same result as a fresh handle."""
import ctypes as C

import numpy as np
import pytest

from av1gpu_b200 import Encoder, isearch, synth
from av1gpu_b200.isearch import IS_ERR_INVALID, IS_ERR_OOM, IS_ERR_STATE, IS_ERR_TIMEOUT, IsError, IsFrame, IsParams


def _records_equal(a, b):
    return (np.array_equal(a.blocks.view(np.uint8), b.blocks.view(np.uint8)) and np.array_equal(a.block_txb, b.block_txb)
            and np.array_equal(a.txb.view(np.uint8), b.txb.view(np.uint8)) and np.array_equal(a.coeffs, b.coeffs)
            and all(np.array_equal(a.recon[p], b.recon[p]) for p in range(3)))


# ---------------------------------------------------------------- CPU: refused before any GPU work
@pytest.mark.parametrize("bd,c444", [(9, 0), (12, 0), (8, 2), (10, -1)])
def test_create_rejects_bad_format(bd, c444):
    L = isearch.load_library()
    p = IsParams()
    p.bit_depth, p.chroma_444, p.device = bd, c444, 0
    h = C.c_void_p()
    assert L.is_create(C.byref(p), C.byref(h)) == IS_ERR_INVALID
    assert L.is_create(None, C.byref(h)) == IS_ERR_INVALID


@pytest.mark.parametrize("w,h,bd,c444", [(0, 64, 8, 0), (64, 0, 8, 0), (16385, 64, 8, 0), (64, 16385, 8, 0), (64, 64, 9, 0),
                                         (64, 64, 8, 3), (-5, 64, 10, 1)])
def test_workspace_bytes_rejects_bad_frames(w, h, bd, c444):
    L = isearch.load_library()
    b = C.c_uint64()
    assert L.is_workspace_bytes_format(w, h, bd, c444, C.byref(b)) == IS_ERR_INVALID


def test_null_handle_everywhere():
    L = isearch.load_library()
    f = IsFrame()
    assert L.is_encode_device(None, C.byref(f), None) == IS_ERR_INVALID
    assert L.is_encode_host(None, C.byref(f), None) == IS_ERR_INVALID
    assert L.is_encode_batch(None, C.byref(f), 1, 1, None) == IS_ERR_INVALID
    assert L.is_set_wait_limits(None, 0, 0) == IS_ERR_INVALID
    assert L.is_set_workspace_limit(None, 0) == IS_ERR_INVALID
    assert L.is_set_poison(None, 1) == IS_ERR_INVALID
    assert L.is_set_batch_options(None, 0, 1, 0) == IS_ERR_INVALID
    n = C.c_uint32()
    assert L.is_record_counts(None, C.byref(n), None, None) == IS_ERR_STATE
    assert L.is_batch_counts(None, 0, C.byref(n), None, None) == IS_ERR_STATE


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_encode_rejects_bad_frames():
    enc = Encoder(0)
    try:
        L = enc.L
        y = np.zeros((64, 96), np.uint8)
        u = np.zeros((32, 48), np.uint8)
        keep = []

        def frame(**kw):
            f = IsFrame()
            f.width, f.height, f.qindex, f.bit_depth, f.chroma_444 = 96, 64, 120, 8, 0
            for p, a in enumerate((y, u, u)):
                keep.append(a)
                f.planes[p] = a.ctypes.data
                f.pitch[p] = a.shape[1]
            for k, v in kw.items():
                if k == "planes":
                    for p, a in enumerate(v):
                        f.planes[p] = a
                elif k == "pitch":
                    for p, a in enumerate(v):
                        f.pitch[p] = a
                else:
                    setattr(f, k, v)
            return f
        bad = [dict(width=0), dict(height=0), dict(width=16385), dict(qindex=0), dict(qindex=256), dict(bit_depth=9),
               dict(bit_depth=8, chroma_444=2), dict(planes=(y.ctypes.data, None, u.ctypes.data)),
               dict(pitch=(95, 48, 48)), dict(pitch=(96, 47, 48))]
        for kw in bad:
            f = frame(**kw)
            assert L.is_encode_host(enc.h, C.byref(f), None) == IS_ERR_INVALID, kw
        assert L.is_encode_batch(enc.h, None, 1, 1, None) == IS_ERR_INVALID
        f = frame()
        assert L.is_encode_batch(enc.h, C.byref(f), 0, 1, None) == IS_ERR_INVALID
        assert L.is_set_wait_limits(enc.h, -1, 0) == IS_ERR_INVALID
        assert L.is_set_wait_limits(enc.h, 0, -1) == IS_ERR_INVALID
        # no result yet on this handle
        n = C.c_uint32()
        assert L.is_record_counts(enc.h, C.byref(n), None, None) == IS_ERR_STATE
        # and the handle still works
        planes = synth.make_image(96, 64, 3)
        r = enc.encode(planes, 120)
        assert len(r.blocks) > 0
    finally:
        enc.close()


@pytest.mark.gpu
def test_workspace_limit_gives_oom_then_recovers(enc):
    planes = synth.make_image(320, 240, 4)
    want = enc.encode(planes, 100)
    need = isearch.workspace_bytes(320, 240)
    enc.set_workspace_limit(need // 2)
    with pytest.raises(IsError) as ei:
        enc.encode(planes, 100)
    assert ei.value.code == IS_ERR_OOM
    enc.set_workspace_limit(0)
    assert _records_equal(enc.encode(planes, 100), want)


@pytest.mark.gpu
@pytest.mark.parametrize("iters,ns", [(1, 0), (0, 1), (1, 1)])
def test_wait_budget_runs_out_without_hang(iters, ns):
    """Waits of one spin / one nanosecond run out at once on a picture with dependencies: the kernel returns, the encode
    reports IS_ERR_TIMEOUT, and the handle's next encode with the default budgets is exact."""
    enc = Encoder(0)
    try:
        planes = synth.make_image(640, 480, 12, edges=True)
        want = enc.encode(planes, 120)
        enc.set_wait_limits(iters, ns)
        with pytest.raises(IsError) as ei:
            enc.encode(planes, 120)
        assert ei.value.code == IS_ERR_TIMEOUT
        enc.set_wait_limits(0, 0)
        assert _records_equal(enc.encode(planes, 120), want)
    finally:
        enc.close()


@pytest.mark.gpu
@pytest.mark.parametrize("w,h,q,fmt", [(333, 200, 120, (8, False)), (211, 149, 60, (8, False)), (200, 136, 160, (10, True)),
                                       (130, 66, 40, (10, False)), (96, 72, 200, (8, True))])
def test_poison_does_not_change_results(enc, w, h, q, fmt):
    planes = synth.make_image(w, h, 31, edges=True, bit_depth=fmt[0], chroma_444=fmt[1])
    want = enc.encode(planes, q)
    enc.set_poison(True)
    try:
        got = enc.encode(planes, q)
    finally:
        enc.set_poison(False)
    assert _records_equal(got, want)


@pytest.mark.gpu
def test_poison_batch_does_not_change_results(enc):
    imgs = [synth.make_image(w, h, s) for w, h, s in ((160, 96, 1), (64, 200, 2), (300, 120, 3))]
    qs = [60, 140, 220]
    want = enc.encode_batch(imgs, qs)
    enc.set_poison(True)
    try:
        got = enc.encode_batch(imgs, qs)
    finally:
        enc.set_poison(False)
    for a, b in zip(got, want):
        assert _records_equal(a, b)
