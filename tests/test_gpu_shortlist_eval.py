"""The trained shortlist (av1gpu_b200/shortlist_weights.npz, written by `python -m av1gpu_b200.shortlist`) against
the plain form on held-out images: BD-rate (PSNR-Y; rate = av1g_encode bytes of each record) and the analysis time of
a 12 MP search.  Every shortlist record is decoded exactly (av1g_encode's reconstruction equals the GPU's)."""
import json
import os

import numpy as np
import pytest

import oracle as O
from av1gpu_b200 import shortlist as SL
from av1gpu_b200 import synth

pytestmark = pytest.mark.gpu
WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "av1gpu_b200", "shortlist_weights.npz")
QS = (40, 80, 120, 160, 200)


def _psnr(a, b):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return 10 * np.log10(255.0 ** 2 / max(mse, 1e-12))


def _curve(enc, im, w, h):
    rates, qual = [], []
    for q in QS:
        r = enc.encode(im, q)
        rec, nbytes = O.av1g_recon(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs)
        assert all(np.array_equal(rec[p], r.recon[p]) for p in range(3))
        rates.append(nbytes)
        qual.append(_psnr(im[0], r.recon[0]))
    return rates, qual


@pytest.mark.parametrize("tau,max_modes,conf,rd_k,bound", [(0.95, 8, 0.0, 4, 1.0), (0.95, 8, 0.0, 2, 2.0), (0.9, 6, 0.0, 2, 2.5),
                                                         (0.8, 4, 0.0, 1, 5.0)])
def test_shortlist_bd_rate_and_speed(enc, tau, max_modes, conf, rd_k, bound):
    weights = SL.load_weights(WEIGHTS)
    w, h = 512, 384
    bds = []
    for i in range(4):   # held out: seeds the training script does not use
        im = synth.make_image(w, h, 777000 + i, edges=True)
        enc.set_shortlist(None)
        ra, qa = _curve(enc, im, w, h)
        enc.set_shortlist(weights, tau=tau, max_modes=max_modes, conf=conf, rd_k=rd_k)
        try:
            rb, qb = _curve(enc, im, w, h)
        finally:
            enc.set_shortlist(None)
        bds.append(SL.bd_rate(ra, qa, rb, qb))
    big = synth.make_image(2000, 1500, 5, edges=True)
    t = {}
    for name, wt in (("plain", None), ("shortlist", weights)):
        enc.set_shortlist(wt, tau=tau, max_modes=max_modes, conf=conf, rd_k=rd_k)
        try:
            for _ in range(2):
                enc.encode(big, 120)
            t[name] = enc.times()
        finally:
            enc.set_shortlist(None)
    line = {"tau": tau, "max_modes": max_modes, "rd_k": rd_k, "bd_rate_psnr_y_pct": [round(b, 3) for b in bds],
            "bd_rate_mean_pct": round(float(np.mean(bds)), 3),
            "analysis_ms_plain": round(t["plain"]["analysis"], 2), "analysis_ms_shortlist": round(t["shortlist"]["analysis"], 2),
            "total_ms_plain": round(t["plain"]["total"], 2), "total_ms_shortlist": round(t["shortlist"]["total"], 2)}
    print(json.dumps(line))
    assert float(np.mean(bds)) < bound


def test_shortlist_bd_rate_10bit_444(enc):
    """The network (trained on 8-bit images) on held-out 10-bit 4:4:4 images, whose features it reads at a quarter of
    the sample value: BD-rate of PSNR-Y against the plain form, every record decoded exactly."""
    weights = SL.load_weights(WEIGHTS)
    w, h = 384, 256
    bds = []
    for i in range(2):
        im = synth.make_image(w, h, 778000 + i, edges=True, bit_depth=10, chroma_444=True)
        curves = []
        for wt in (None, weights):
            enc.set_shortlist(wt, tau=0.9, max_modes=6, rd_k=2)
            try:
                rates, qual = [], []
                for q in QS:
                    r = enc.encode(im, q)
                    rec, nbytes = O.av1g_recon(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs, bit_depth=10, chroma_444=True)
                    assert all(np.array_equal(rec[p], r.recon[p]) for p in range(3))
                    mse = np.mean((im[0].astype(np.float64) - r.recon[0].astype(np.float64)) ** 2)
                    rates.append(nbytes)
                    qual.append(10 * np.log10(1023.0 ** 2 / max(mse, 1e-12)))
                curves.append((rates, qual))
            finally:
                enc.set_shortlist(None)
        bds.append(SL.bd_rate(curves[0][0], curves[0][1], curves[1][0], curves[1][1]))
    print(json.dumps({"format": "10-bit 4:4:4", "tau": 0.9, "max_modes": 6, "rd_k": 2, "bd_rate_psnr_y_pct": [round(b, 3) for b in bds]}))
    assert float(np.mean(bds)) < 2.5


def _ssim_db(a, b, peak):
    """SSIM of two planes (Gaussian window, sigma 1.5, K1 0.01, K2 0.03) as -10 log10(1 - SSIM)."""
    from scipy.ndimage import gaussian_filter
    a, b = a.astype(np.float64), b.astype(np.float64)
    c1, c2 = (0.01 * peak) ** 2, (0.03 * peak) ** 2
    f = lambda x: gaussian_filter(x, 1.5, truncate=3.5)
    ma, mb = f(a), f(b)
    va, vb, cov = f(a * a) - ma * ma, f(b * b) - mb * mb, f(a * b) - ma * mb
    s = np.mean(((2 * ma * mb + c1) * (2 * cov + c2)) / ((ma * ma + mb * mb + c1) * (va + vb + c2)))
    return -10 * np.log10(max(1.0 - s, 1e-12))


def test_shortlist_heldout_200(enc):
    """The trained network on 200 held-out seeded images (384 x 256, seeds the training script does not use): BD-rate
    of PSNR-Y and of SSIM-Y against the plain form over qindex 40 .. 200, with and without the confidence fallback,
    and the fallback rate, coverage and mask size on the held-out images' own blocks."""
    import torch
    weights = SL.load_weights(WEIGHTS)
    settings = {"tau0.9_max6_rdk2": (0.9, 6, 0.0, 2), "tau0.9_max6_conf0.25_rdk2": (0.9, 6, 0.25, 2)}
    w, h, n = 384, 256, 200
    bd = {k: ([], []) for k in settings}
    feats, labels = [], []
    for i in range(n):
        im = synth.make_image(w, h, 990000 + i, edges=True)
        curves = {}
        for name, st in [("plain", None)] + list(settings.items()):
            if st is None:
                enc.set_shortlist(None)
            else:
                enc.set_shortlist(weights, tau=st[0], max_modes=st[1], conf=st[2], rd_k=st[3])
            try:
                rates, ps, ss = [], [], []
                for q in QS:
                    r = enc.encode(im, q)
                    rec, nbytes = O.av1g_recon(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs)
                    assert all(np.array_equal(rec[p], r.recon[p]) for p in range(3))
                    rates.append(nbytes)
                    ps.append(_psnr(im[0], r.recon[0]))
                    ss.append(_ssim_db(im[0], r.recon[0], 255.0))
                curves[name] = (rates, ps, ss)
            finally:
                enc.set_shortlist(None)
        for name in settings:
            bd[name][0].append(SL.bd_rate(curves["plain"][0], curves["plain"][1], curves[name][0], curves[name][1]))
            bd[name][1].append(SL.bd_rate(curves["plain"][0], curves["plain"][2], curves[name][0], curves[name][2]))
        if i < 40:   # the blocks of the first 40 images for the mask statistics
            X, y = SL.dataset(enc, [im], [120], per_image=4096, seed=i)
            feats.append(X)
            labels.append(y)
    lrn = SL.Learner(max_batch=4096)
    try:
        lrn.set_weights(weights)
        Xh, yh = torch.cat(feats), torch.cat(labels)
        line = {"images": n, "size": "%dx%d" % (w, h), "qindex": list(QS)}
        for name, (tau, mm, cf, rdk) in settings.items():
            p, s = np.array(bd[name][0]), np.array(bd[name][1])
            line[name] = {"bd_rate_psnr_y_mean_pct": round(float(p.mean()), 3), "bd_rate_psnr_y_median_pct": round(float(np.median(p)), 3),
                          "bd_rate_ssim_y_mean_pct": round(float(s.mean()), 3), "bd_rate_ssim_y_median_pct": round(float(np.median(s)), 3),
                          **{k: round(v, 4) for k, v in SL.evaluate(lrn, Xh, yh, tau=tau, max_modes=mm, conf=cf).items()}}
        print(json.dumps(line))
    finally:
        lrn.close()
    for name in settings:
        assert float(np.mean(bd[name][0])) < 0.5 and float(np.mean(bd[name][1])) < 0.5
