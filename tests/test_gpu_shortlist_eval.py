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
