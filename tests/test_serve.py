"""Serving loop: admission by HBM budget (CPU), and on the GPU every served result equals the same image searched
alone, whatever batch it was admitted into."""
from collections import deque

import numpy as np
import pytest

from av1gpu_b200 import serve, synth


def _req(i, nbytes):
    r = serve.Request(i, [np.zeros((8, 8), np.uint8)] * 3, 120, 0.0)
    r.nbytes = nbytes
    return r


def test_take_batch_budget_and_order():
    pending = deque(_req(i, b) for i, b in enumerate([40, 30, 50, 10, 10]))
    b1 = serve.take_batch(pending, 100, 8)
    assert [r.rid for r in b1] == [0, 1]              # 40 + 30 fit, + 50 would not
    b2 = serve.take_batch(pending, 100, 2)
    assert [r.rid for r in b2] == [2, 3]              # max_batch 2
    big = deque([_req(9, 500), _req(10, 1)])
    assert [r.rid for r in serve.take_batch(big, 100, 8)] == [9]   # larger than the budget: runs alone
    assert [r.rid for r in serve.take_batch(big, 100, 8)] == [10]
    assert serve.take_batch(deque(), 100, 8) == []


def test_latency_stats():
    rs = [_req(i, 1) for i in range(100)]
    for i, r in enumerate(rs):
        r.t_arrive, r.t_done = 0.0, (i + 1) / 1000.0
    s = serve.latency_stats(rs)
    assert s["n"] == 100 and abs(s["p50_ms"] - 50.5) < 1e-6 and s["max_ms"] == 100.0


def test_workspace_bytes_grows_with_the_image():
    from av1gpu_b200.isearch import workspace_bytes
    a, b = workspace_bytes(640, 480), workspace_bytes(4000, 3000)
    assert 0 < a < b and b > 4000 * 3000 * 10
    assert workspace_bytes(4000, 3000, 8, True) > b and workspace_bytes(4000, 3000, 10, True) > workspace_bytes(4000, 3000, 8, True)


def _mixed_requests():
    sizes = [(160, 120), (96, 64), (211, 149), (64, 200), (300, 90), (128, 128), (77, 45), (256, 96)]
    qs = [60, 120, 200, 90, 150, 40, 220, 120]
    # formats mixed as requests arrive: images 2 and 5 10-bit 4:4:4, image 6 8-bit 4:4:4
    fmts = {2: (10, True), 5: (10, True), 6: (8, True)}
    images = [synth.make_image(w, h, 50 + i, edges=True, bit_depth=fmts.get(i, (8, False))[0], chroma_444=fmts.get(i, (8, False))[1])
              for i, (w, h) in enumerate(sizes)]
    return images, qs


@pytest.mark.gpu
@pytest.mark.parametrize("learned", [False, True])
def test_served_results_equal_alone(enc, learned):
    """Each served result (plain, or batched + learned shortlist) equals the same image searched alone with the same
    search settings, whatever batch it was admitted into."""
    images, qs = _mixed_requests()
    sl = None
    if learned:
        from av1gpu_b200.shortlist import load_params
        import os
        w = load_params(os.path.join(os.path.dirname(serve.__file__), "shortlist_weights.npz"))
        sl = {"params": w, "tau": 0.9, "max_cand": 8, "rd_k": 2, "tx_tau": 0.9, "max_tx": 2}
        enc.set_shortlist(**sl)
    try:
        alone = [enc.encode(im, q) for im, q in zip(images, qs)]
    finally:
        enc.set_shortlist(None)
    srv = serve.Server(device=0, hbm_budget=1 << 30, pipelines=2, max_batch=4, recon_ctas=96, shortlist=sl)
    try:
        t = serve.poisson_arrivals(400.0, len(images), seed=3)
        reqs = srv.run([(float(ti), im, q) for ti, im, q in zip(t, images, qs)])
    finally:
        srv.close()
    for r in reqs:
        a = alone[r.rid]
        assert np.array_equal(r.record.blocks.view(np.uint8), a.blocks.view(np.uint8)), "request %d" % r.rid
        assert np.array_equal(r.record.coeffs, a.coeffs) and np.array_equal(r.record.txb.view(np.uint8), a.txb.view(np.uint8))
        for p in range(3):
            assert np.array_equal(r.record.recon[p], a.recon[p])
    st = serve.latency_stats(reqs)
    assert st["n"] == len(images) and st["p99_ms"] >= st["p50_ms"] > 0
