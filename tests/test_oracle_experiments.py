"""Measurements on the CPU oracle that decide what is not built, against the plain form on 16 held-out images
(384 x 256, qindex 40 .. 200; rate from av1g_encode): the reference's open-loop chroma shortlist
(encoder/src/k_leafprep.cu:1-30, the chroma screening on source edges so that it leaves the closed loop: BD-rate of
PSNR-Y and of PSNR-YUV 6:1:1, the closed loop's algorithmic INT32 operations), and the intra edge filter (spec
7.11.2.11-12, one of the tools the reference's CLI enables: BD-rate; the oracle's edge-filter records reconstruct as
av1g_encode does with enable_intra_edge_filter 1)."""
import json

import numpy as np

import oracle as O
from av1gpu_b200 import synth
from av1gpu_b200.isearch import frame_params
from av1gpu_b200.shortlist import bd_rate

QS = (40, 80, 120, 160, 200)


def _psnr(a, b):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return 10 * np.log10(255.0 ** 2 / max(mse, 1e-12))


def _curve(im, w, h):
    rate, py, pyuv, ops = [], [], [], [0, 0]
    for q in QS:
        r = O.encode(im, q)
        _, nbytes = O.av1g_recon(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs)
        a, c = r.op_counts()
        ops[0] += a
        ops[1] += c
        rate.append(nbytes)
        y, u, v = (_psnr(im[p], r.recon[p]) for p in range(3))
        py.append(y)
        pyuv.append((6 * y + u + v) / 8)
    return rate, py, pyuv, ops


def test_open_loop_chroma_screening_cost():
    w, h, n = 384, 256, 16
    bd_y, bd_yuv, closed, opened = [], [], [0, 0], [0, 0]
    try:
        for i in range(n):
            im = synth.make_image(w, h, 995000 + i, edges=True)
            O.set_uv_open_loop(False)
            a = _curve(im, w, h)
            O.set_uv_open_loop(True)
            b = _curve(im, w, h)
            bd_y.append(bd_rate(a[0], a[1], b[0], b[1]))
            bd_yuv.append(bd_rate(a[0], a[2], b[0], b[2]))
            closed[0] += a[3][1]; closed[1] += b[3][1]
            opened[0] += a[3][0]; opened[1] += b[3][0]
    finally:
        O.set_uv_open_loop(False)
    line = {"images": n, "size": "%dx%d" % (w, h), "bd_rate_psnr_y_mean_pct": round(float(np.mean(bd_y)), 3),
            "bd_rate_psnr_yuv611_mean_pct": round(float(np.mean(bd_yuv)), 3), "closed_loop_ops_ratio": round(closed[1] / closed[0], 4),
            "open_loop_ops_ratio": round(opened[1] / opened[0], 4)}
    print(json.dumps(line))
    assert line["closed_loop_ops_ratio"] < 0.9 and line["open_loop_ops_ratio"] > 1.0
    assert line["bd_rate_psnr_yuv611_mean_pct"] > 0


def test_intra_edge_filter_gain():
    w, h, n = 384, 256, 16
    fp_on = lambda q: _fp_edge(w, h, q)  # noqa: E731
    bd_y, bd_yuv = [], []
    try:
        for i in range(n):
            im = synth.make_image(w, h, 996000 + i, edges=True)
            O.set_edge_filter(False)
            a = _curve(im, w, h)
            O.set_edge_filter(True)
            rate, py, pyuv = [], [], []
            for q in QS:
                r = O.encode(im, q)
                if i == 0 and q in (40, 200):   # the records decode to the oracle's reconstruction
                    rec = O.av1g_encode_fp(fp_on(q), r.blocks, r.block_txb, r.txb, r.coeffs)
                    assert all(np.array_equal(rec[p], r.recon[p]) for p in range(3))
                obu, _ = O.av1g_obu_fp(fp_on(q), r.blocks, r.block_txb, r.txb, r.coeffs)
                rate.append(len(obu))
                y, u, v = (_psnr(im[p], r.recon[p]) for p in range(3))
                py.append(y)
                pyuv.append((6 * y + u + v) / 8)
            bd_y.append(bd_rate(a[0], a[1], rate, py))
            bd_yuv.append(bd_rate(a[0], a[2], rate, pyuv))
    finally:
        O.set_edge_filter(False)
    line = {"images": n, "size": "%dx%d" % (w, h), "bd_rate_psnr_y_mean_pct": round(float(np.mean(bd_y)), 3),
            "bd_rate_psnr_yuv611_mean_pct": round(float(np.mean(bd_yuv)), 3)}
    print(json.dumps(line))   # the sign depends on the content (the filter smooths the edges these pictures are made of)


def _fp_edge(w, h, q):
    fp = frame_params(w, h, q)
    fp[24] = 1   # enable_intra_edge_filter
    return fp

