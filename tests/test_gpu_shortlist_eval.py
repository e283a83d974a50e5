"""The trained shortlist (av1gpu_b200/shortlist_weights.npz, written by `python -m av1gpu_b200.shortlist`) against
the plain form and against the non-learned pruning on held-out images: BD-rate (PSNR-Y and SSIM-Y; rate = av1g_encode
bytes of each record), the speed of the analysis and of a batch, and the fallback rate.  Every record is decoded
exactly (av1g_encode's reconstruction equals the GPU's)."""
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
# the learned form of the batched + shortlist workload, and the non-learned pruning it is compared with
LEARNED = SL.LEARNED                # the selection rule
LEARNED_NL = SL.LEARNED_OTHER       # the blocks the network does not score (4x4, 4x8, 8x4)
NONLEARNED = dict(rd_k=2)           # the same RD count for every block, no network


def _psnr(a, b, peak=255.0):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return 10 * np.log10(peak ** 2 / max(mse, 1e-12))


def _ssim_db(a, b, peak):
    """SSIM of two planes (Gaussian window, sigma 1.5, K1 0.01, K2 0.03) as -10 log10(1 - SSIM)."""
    from scipy.ndimage import gaussian_filter
    a, b = a.astype(np.float64), b.astype(np.float64)
    c1, c2 = (0.01 * peak) ** 2, (0.03 * peak) ** 2
    f = lambda x: gaussian_filter(x, 1.5, truncate=3.5)  # noqa: E731
    ma, mb = f(a), f(b)
    va, vb, cov = f(a * a) - ma * ma, f(b * b) - mb * mb, f(a * b) - ma * mb
    s = np.mean(((2 * ma * mb + c1) * (2 * cov + c2)) / ((ma * ma + mb * mb + c1) * (va + vb + c2)))
    return -10 * np.log10(max(1.0 - s, 1e-12))


def _form(enc, params, learned=None, nonlearned=None):
    enc.set_shortlist(None)
    enc.set_search_options()
    if learned:
        enc.set_shortlist(params, **learned)
    if nonlearned:
        enc.set_search_options(**nonlearned)


def _curve(enc, im, w, h, ssim=False, bit_depth=8, chroma_444=False):
    peak = 1023.0 if bit_depth == 10 else 255.0
    rates, ps, ss = [], [], []
    for q in QS:
        r = enc.encode(im, q)
        rec, nbytes = O.av1g_recon(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs, bit_depth=bit_depth, chroma_444=chroma_444)
        assert all(np.array_equal(rec[p], r.recon[p]) for p in range(3))
        rates.append(nbytes)
        ps.append(_psnr(im[0], r.recon[0], peak))
        if ssim:
            ss.append(_ssim_db(im[0], r.recon[0], peak))
    return rates, ps, ss


def _analysis_ms(enc, big):
    for _ in range(2):
        enc.encode(big, 120)
    return enc.times()


def test_learned_against_non_learned(enc):
    """On 6 held-out 512 x 384 images: the learned form and the non-learned pruning, each against the plain form
    (BD-rate of PSNR-Y), and the time of a 3 MP search.  The network must keep the BD-rate within 0.5 % and make the
    analysis faster than the non-learned pruning at the same RD count."""
    params = SL.load_params(WEIGHTS)
    w, h = 512, 384
    ims = [synth.make_image(w, h, 777000 + i, edges=True) for i in range(6)]   # seeds the training never used
    big = synth.make_image(2000, 1500, 5, edges=True)
    forms = {"plain": (None, None), "learned": (LEARNED, LEARNED_NL), "non-learned": (None, NONLEARNED)}
    curves, times = {}, {}
    try:
        for name, (lf, nf) in forms.items():
            _form(enc, params, lf, nf)
            curves[name] = [_curve(enc, im, w, h) for im in ims]
            times[name] = _analysis_ms(enc, big)
    finally:
        _form(enc, params)
    bd = {k: [SL.bd_rate(a[0], a[1], b[0], b[1]) for a, b in zip(curves["plain"], curves[k])] for k in ("learned", "non-learned")}
    line = {k: {"bd_rate_psnr_y_pct": [round(v, 3) for v in bd[k]], "bd_mean_pct": round(float(np.mean(bd[k])), 3),
                "analysis_ms": round(times[k]["analysis"], 2), "total_ms": round(times[k]["total"], 2)} for k in bd}
    line["plain"] = {"analysis_ms": round(times["plain"]["analysis"], 2), "total_ms": round(times["plain"]["total"], 2)}
    print(json.dumps(line))
    assert float(np.mean(bd["learned"])) < 0.5
    assert times["learned"]["analysis"] < times["plain"]["analysis"] * 0.8
    assert times["learned"]["analysis"] < times["non-learned"]["analysis"]


def test_learned_batch_speed(enc):
    """A batch of 32 mixed images (the batched workload's generator): the learned form against the plain batch and the
    one-at-a-time plain search, with every image of the learned batch equal to that image searched alone in the same
    form."""
    import time
    import torch
    from av1gpu_b200.batchbench import workload
    from av1gpu_b200.isearch import plane_format
    params = SL.load_params(WEIGHTS)
    work = workload(32, 5, 6.0)
    dev = [[torch.from_numpy(p.astype(np.int16) if p.dtype == np.uint16 else p).cuda() for p in planes] for planes, _ in work]
    qs = [q for _, q in work]
    mp = sum(p[0].shape[0] * p[0].shape[1] for p, _ in work) / 1e6

    def timed(f):
        f()
        torch.cuda.synchronize()
        t = time.perf_counter()
        f()
        torch.cuda.synchronize()
        return time.perf_counter() - t

    def one_by_one():
        for planes, q in zip(dev, qs):
            enc.encode_device_async(planes, q)

    def batch():
        enc.encode_batch_async(dev, qs, host=False)

    try:
        _form(enc, params)
        t_plain = timed(one_by_one)
        enc.set_batch_options(use_graph=True, front_streams=2)
        t_batch = timed(batch)
        _form(enc, params, LEARNED, LEARNED_NL)
        t_learned = timed(batch)
        fmt = [plane_format(p) for p, _ in work]
        got = [enc.batch_fetch(i, p[0].shape[1], p[0].shape[0], q, *f).digest() for i, ((p, q), f) in enumerate(zip(work, fmt))]
        enc.set_batch_options(use_graph=False, front_streams=1)
        for i in range(0, len(work), 5):
            (p, q), f = work[i], fmt[i]
            enc.encode_device_async(dev[i], q)
            assert enc.fetch(p[0].shape[1], p[0].shape[0], q, bit_depth=f[0], chroma_444=f[1]).digest() == got[i]
    finally:
        enc.set_batch_options(use_graph=False, front_streams=1)
        _form(enc, params)
    line = {"images": len(work), "mp": round(mp, 1), "plain_mps": round(mp / t_plain, 2), "batched_mps": round(mp / t_batch, 2),
            "batched_learned_mps": round(mp / t_learned, 2), "x_plain": round(t_plain / t_learned, 2)}
    print(json.dumps(line))
    assert t_learned < t_batch * 0.9


def test_shortlist_bd_rate_10bit_444(enc):
    """The network (trained on 8-bit images) on held-out 10-bit 4:4:4 images, whose features it reads at a quarter of
    the sample value: BD-rate of PSNR-Y against the plain form, every record decoded exactly."""
    params = SL.load_params(WEIGHTS)
    w, h = 384, 256
    bds = []
    try:
        for i in range(2):
            im = synth.make_image(w, h, 778000 + i, edges=True, bit_depth=10, chroma_444=True)
            _form(enc, params)
            a = _curve(enc, im, w, h, bit_depth=10, chroma_444=True)
            _form(enc, params, LEARNED, LEARNED_NL)
            b = _curve(enc, im, w, h, bit_depth=10, chroma_444=True)
            bds.append(SL.bd_rate(a[0], a[1], b[0], b[1]))
    finally:
        _form(enc, params)
    print(json.dumps({"format": "10-bit 4:4:4", **LEARNED, "bd_rate_psnr_y_pct": [round(b, 3) for b in bds]}))
    assert float(np.mean(bds)) < 1.0


def test_shortlist_heldout_200(enc):
    """The trained network on 200 held-out seeded images (384 x 256, seeds the training script does not use): BD-rate of
    PSNR-Y and of SSIM-Y against the plain form over qindex 40 .. 200 for the learned form with and without the
    confidence fallback and for the non-learned pruning, and the network's statistics on the held-out images' own blocks
    (top-1, coverage of the search's choice, list sizes, fallback rate)."""
    import torch
    params = SL.load_params(WEIGHTS)
    settings = {"learned": (LEARNED, LEARNED_NL), "learned_conf0.2": (dict(LEARNED, conf=0.2), LEARNED_NL),
                "non-learned": (None, NONLEARNED)}
    w, h, n = 384, 256, 200
    bd = {k: ([], []) for k in settings}
    feats, labels = [], []
    try:
        for i in range(n):
            im = synth.make_image(w, h, 990000 + i, edges=True)
            _form(enc, params)
            base = _curve(enc, im, w, h, ssim=True)
            if i < 40:   # the blocks of the first 40 images (plain search) for the network's statistics
                enc.encode(im, 120)
                X, y = SL.image_rows(enc)
                feats.append(X)
                labels.append(y)
            for name, (lf, nf) in settings.items():
                _form(enc, params, lf, nf)
                c = _curve(enc, im, w, h, ssim=True)
                bd[name][0].append(SL.bd_rate(base[0], base[1], c[0], c[1]))
                bd[name][1].append(SL.bd_rate(base[0], base[2], c[0], c[2]))
    finally:
        _form(enc, params)
    lrn = SL.Learner(max_batch=4096)
    try:
        lrn.set_params(params)
        Xh, yh = torch.cat(feats), torch.cat(labels)
        line = {"images": n, "size": "%dx%d" % (w, h), "qindex": list(QS)}
        for name, (lf, _) in settings.items():
            p, s = np.array(bd[name][0]), np.array(bd[name][1])
            line[name] = {"bd_rate_psnr_y_mean_pct": round(float(p.mean()), 3), "bd_rate_psnr_y_median_pct": round(float(np.median(p)), 3),
                          "bd_rate_ssim_y_mean_pct": round(float(s.mean()), 3), "bd_rate_ssim_y_median_pct": round(float(np.median(s)), 3)}
            if lf:
                line[name].update({k: round(v, 4) for k, v in SL.evaluate(lrn, Xh, yh, lf["tau"], lf["max_cand"], lf["conf"],
                                                                          lf["tx_tau"], lf["max_tx"]).items()})
        print(json.dumps(line))
    finally:
        lrn.close()
    for name in ("learned", "learned_conf0.2"):
        assert float(np.mean(bd[name][0])) < 0.5 and float(np.mean(bd[name][1])) < 0.5
