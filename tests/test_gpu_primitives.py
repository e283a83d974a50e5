"""Kernel-level parity: the search's own device functions (through libisearch.so's C ABI) against the CPU oracle and
av1core's dsp.h on seeded random blocks - every tx size and intra tx type, the quantiser / rate / distortion, the
exact inverse (including out-of-range levels), every prediction mode and angle delta.  Bit-exact."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

# (tx size enum, W, H) for the 19 AV1 sizes
TX = [(0, 4, 4), (1, 8, 8), (2, 16, 16), (3, 32, 32), (4, 64, 64), (5, 4, 8), (6, 8, 4), (7, 8, 16), (8, 16, 8),
      (9, 16, 32), (10, 32, 16), (11, 32, 64), (12, 64, 32), (13, 4, 16), (14, 16, 4), (15, 8, 32), (16, 32, 8),
      (17, 16, 64), (18, 64, 16)]
SET1 = [0, 1, 2, 3, 9, 10, 11]     # DCT_DCT, ADST_DCT, DCT_ADST, ADST_ADST, IDTX, V_DCT, H_DCT
SET2 = [0, 1, 2, 3, 9]


def types_of(w, h):
    up = max(w, h)
    if up >= 32:
        return [0]
    return SET2 if min(w, h) == 16 else SET1


def residuals(rng, n, w, h):
    r = rng.integers(-255, 256, (n, h, w)).astype(np.int32)
    r[0] = 255                                        # extremes: the forward transform's range bound
    r[1] = -255
    r[2] = np.where((np.add.outer(np.arange(h), np.arange(w)) & 1) == 0, 255, -255)
    r[3] = np.where(np.arange(w)[None, :] < w // 2, 255, -255)
    r[4] = (rng.normal(0, 6, (h, w))).round().clip(-255, 255)   # small residuals (typical)
    return r


@pytest.mark.parametrize("tx", TX, ids=["%dx%d" % (t[1], t[2]) for t in TX])
def test_forward_quant_rate_parity(enc, tx):
    t, w, h = tx
    rng = np.random.default_rng(1000 + t)
    for tt in types_of(w, h):
        for q, plane in ((40, 0), (120, 0), (220, 1)):
            res = residuals(rng, 12, w, h)
            ctx = (int(rng.integers(0, 5)) if plane == 0 else 7 + int(rng.integers(0, 6)), int(rng.integers(0, 3)),
                   int(rng.integers(0, 13)))
            coef, lv, D, R, eob = enc.test_fwd_quant(res, t, tt, plane, q, ctx)
            qctx = 0 if q <= 20 else 1 if q <= 60 else 2 if q <= 120 else 3
            dcq, acq = _q(q)
            for i in range(res.shape[0]):
                oc = O.fwd2d(res[i], t, tt)
                assert np.array_equal(coef[i], oc.ravel()), "forward transform differs (type %d, block %d)" % (tt, i)
                e = int((res[i].astype(np.int64) ** 2).sum()) if (w == 64 or h == 64) else 0
                olv, oD, oR, oeob = O.quant_rate(oc, t, tt, plane, dcq, acq, ctx[0], ctx[1], ctx[2], qctx, e)
                assert np.array_equal(lv[i], olv.ravel()), "levels differ (type %d, block %d)" % (tt, i)
                assert (D[i], R[i], eob[i]) == (oD, oR, oeob), "D/R/eob differ (type %d, block %d)" % (tt, i)


def _q(q):
    return O.qstep(q)


@pytest.mark.parametrize("tx", TX, ids=["%dx%d" % (t[1], t[2]) for t in TX])
def test_inverse_parity(enc, tx):
    t, w, h = tx
    rng = np.random.default_rng(2000 + t)
    tw, th = min(w, 32), min(h, 32)
    for tt in types_of(w, h):
        for q in (40, 200):
            lv = np.zeros((10, th * tw), np.int16)
            for i in range(10):
                k = int(rng.integers(1, 12))
                pos = rng.integers(0, th * tw, k)
                lv[i, pos] = rng.integers(-40, 41, k)
            lv[8, :] = rng.integers(-2000, 2001, th * tw)   # out of the conformance range: flags set, values still defined
            lv[9, 0] = 16383
            res, fl = enc.test_inverse(lv, t, tt, q, w, h)
            dcq, acq = _q(q)
            for i in range(10):
                ores, oerr = O.inv2d(lv[i], t, tt, dcq, acq, w, h)
                assert (fl[i] != 0) == (oerr != 0), "range flags differ (type %d, block %d)" % (tt, i)
                if oerr == 0:
                    assert np.array_equal(res[i], ores), "inverse differs (type %d, block %d)" % (tt, i)


def test_prediction_parity(enc):
    rng = np.random.default_rng(7)
    plane = rng.integers(0, 256, (200, 200)).astype(np.uint8)
    plane[:, 100:] = np.clip(np.arange(100)[None, :] * 2 + plane[:, 100:] // 8, 0, 255)   # smooth part
    params = []
    for lw in range(2, 7):
        for lh in range(2, 7):
            if abs(lw - lh) > 2:
                continue
            for mode in range(13):
                for d in ((-3, -1, 0, 2, 3) if 1 <= mode <= 8 else (0,)):
                    bw, bh = 1 << lw, 1 << lh
                    x = int(rng.integers(1, 200 - 2 * bw)) if 200 - 2 * bw > 1 else 1
                    y = int(rng.integers(1, 200 - 2 * bh)) if 200 - 2 * bh > 1 else 1
                    hl, ha, har, hbl = (int(v) for v in rng.integers(0, 2, 4))
                    params.append([x, y, lw, lh, hl, ha, har, hbl, mode, d])
    params = np.array(params, np.int32)
    out = enc.test_predict(plane, params)
    for i, p in enumerate(params):
        bw, bh = 1 << p[2], 1 << p[3]
        ref = np.zeros(bw * bh, np.uint8)
        O.lib().orc_predict(plane.ctypes.data, 200, int(p[0]), int(p[1]), int(p[2]), int(p[3]), int(p[4]), int(p[5]),
                            int(p[6]), int(p[7]), 199, 199, int(p[8]), int(p[9]), ref.ctypes.data)
        assert np.array_equal(out[i, :bw * bh], ref), "prediction differs for %s" % list(p)
