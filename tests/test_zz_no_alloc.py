"""is_fwd_quant_static (forward transform + quantisation + rate with a fixed static scratch, no device allocation)
against the allocating entry point is_test_fwd_quant, both called through the C ABI with the same inputs.

Two calls in a row with different sizes reuse the one scratch, also on a caller's stream; a request larger than the
scratch and bad arguments are refused before any GPU work (those cases need no GPU).  The file name sorts last so the
test also runs after everything else in the session."""
import ctypes as C

import numpy as np
import pytest

from av1gpu_b200 import isearch

IS_ERR_INVALID, IS_ERR_TOO_LARGE = -1, -6
TX_16X16, TX_64X64, TX_8X32 = 2, 4, 15


def _static(L, res, tx_size, tx_type, plane, qindex, ctx, device=0, stream=None):
    n, h, w = res.shape
    nc = min(w, 32) * min(h, 32)
    res = np.ascontiguousarray(res, np.int32)
    coef, lv = np.zeros((n, nc), np.int32), np.zeros((n, nc), np.int16)
    D, R, eob = np.zeros(n, np.int64), np.zeros(n, np.int64), np.zeros(n, np.int32)
    cx = np.array(ctx, np.int32)
    rc = L.is_fwd_quant_static(device, n, res.ctypes.data, tx_size, tx_type, plane, qindex, cx.ctypes.data, coef.ctypes.data,
                               lv.ctypes.data, D.ctypes.data, R.ctypes.data, eob.ctypes.data, stream)
    return rc, (coef, lv, D, R, eob)


@pytest.mark.gpu
def test_static_scratch_matches_allocating_entry_point(enc):
    L = isearch.load_library()
    rng = np.random.default_rng(2024)
    cases = ((TX_64X64, 0, 0, 120, (3, 0, 0), 64, 64, 150),    # DCT_DCT luma, 150 blocks of 64x64
             (TX_16X16, 9, 0, 60, (1, 2, 0), 16, 16, 700),     # IDTX
             (TX_8X32, 0, 1, 200, (7, 1, 0), 8, 32, 300))      # chroma plane, rectangular
    for tx_size, tx_type, plane, q, ctx, w, h, n in cases:
        res = rng.integers(-255, 256, (n, h, w)).astype(np.int32)
        res[: n // 4] //= 16                                   # low-energy blocks: short and empty eobs too
        want = enc.test_fwd_quant(res, tx_size, tx_type, plane, q, ctx)
        rc, got = _static(L, res, tx_size, tx_type, plane, q, ctx)
        assert rc == 0
        for a, b in zip(want, got):
            assert np.array_equal(a, b)


@pytest.mark.gpu
def test_static_scratch_on_a_caller_stream(enc):
    """The same results through a caller's non-default stream; the calling thread's device stays current."""
    import torch
    L = isearch.load_library()
    rng = np.random.default_rng(7)
    res = rng.integers(-200, 201, (64, 8, 8)).astype(np.int32)
    want = enc.test_fwd_quant(res, 1, 3, 0, 90, (4, 0, 5))     # TX_8X8, ADST_ADST
    s = torch.cuda.Stream(device=0)
    for _ in range(2):
        rc, got = _static(L, res, 1, 3, 0, 90, (4, 0, 5), stream=s.cuda_stream)
        assert rc == 0
        for a, b in zip(want, got):
            assert np.array_equal(a, b)
    assert torch.cuda.current_device() == 0


def test_static_scratch_refuses_oversized_request():
    """Refused before any GPU work (no GPU needed)."""
    L = isearch.load_library()
    res = np.zeros((187, 64, 64), np.int32)                    # 186 blocks of 64x64 is the most that fits
    rc, _ = _static(L, res, TX_64X64, 0, 0, 120, (0, 0, 0))
    assert rc == IS_ERR_TOO_LARGE


@pytest.mark.parametrize("tx_size,tx_type,ctx,device", [
    (TX_16X16, 0, (13, 0, 0), 0),      # skip context beyond the txb_skip table
    (TX_16X16, 0, (0, 3, 0), 0),       # dc-sign context beyond its table
    (TX_16X16, 0, (0, 0, -1), 0),      # negative intra direction
    (TX_16X16, 0, (0, 0, 13), 0),      # intra direction beyond the tx-set tables
    (TX_64X64, 9, (0, 0, 0), 0),       # IDTX: not in the (DCT-only) set of 64x64
    (TX_16X16, 4, (0, 0, 0), 0),       # FLIPADST_DCT: not an intra type
    (TX_16X16, 0, (0, 0, 0), -1),      # no such device
])
def test_static_scratch_refuses_bad_arguments(tx_size, tx_type, ctx, device):
    """Bad contexts, tx types outside the intra set of the size and bad devices return IS_ERR_INVALID before any GPU
    work (no GPU needed)."""
    L = isearch.load_library()
    w = h = 64 if tx_size == TX_64X64 else 16
    rc, _ = _static(L, np.zeros((2, h, w), np.int32), tx_size, tx_type, 0, 120, ctx, device=device)
    assert rc == IS_ERR_INVALID
