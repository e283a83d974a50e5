"""Continuous admission into a running closed loop (is_serve_*): images submitted while others are already in the
persistent closed loop join it, each completes on its own, and each result equals the same image searched alone."""
import time

import numpy as np
import pytest

from av1gpu_b200 import Encoder, serve, synth

pytestmark = pytest.mark.gpu


def _pinned(planes):
    """Planes in pinned host memory (made before a session opens: nothing is allocated or freed while its loop runs)."""
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in planes]


def _run_until_done(e, tickets, timeout_s=60.0):
    order, t0 = [], time.perf_counter()
    while len(order) < len(tickets):
        for tk in e.serve_poll():
            order.append(tk)
        assert time.perf_counter() - t0 < timeout_s, "serving session did not finish"
        time.sleep(0.0005)
    return order


def test_image_submitted_mid_loop_finishes_first_and_equals_alone(enc):
    big = synth.make_image(1920, 1088, 71, edges=True)
    small = synth.make_image(160, 120, 72, edges=True)
    want_big, want_small, want3 = enc.encode(big, 120).digest(), enc.encode(small, 60).digest(), enc.encode(small, 200).digest()
    big, small = _pinned(big), _pinned(small)
    e = Encoder(0)
    try:
        e.serve_open(8, False, arena_bytes=1 << 30, max_images=8, max_leaves=1 << 20)
        tb = e.serve_submit(big, 120)
        time.sleep(0.03)                       # the big image's front end is done: its closed loop is running
        ts = e.serve_submit(small, 60)
        order = _run_until_done(e, [tb, ts])
        assert order[0] == ts, "the image submitted mid-loop did not finish first"
        rb = e.serve_fetch(tb, 1920, 1088, 120)
        rs = e.serve_fetch(ts, 160, 120, 60)
        assert rb.digest() == want_big and rs.digest() == want_small
        # the slots are free again: a third image in the same session
        t3 = e.serve_submit(small, 200)
        _run_until_done(e, [t3])
        assert e.serve_fetch(t3, 160, 120, 200).digest() == want3
    finally:
        e.serve_close()
        e.close()


@pytest.mark.parametrize("bd,c444", [(8, False), (10, True)])
def test_stream_session_many_images_equal_alone(enc, bd, c444):
    sizes = [(211, 149), (96, 64), (320, 240), (64, 200), (130, 66), (256, 96)]
    qs = [60, 120, 200, 90, 150, 40]
    images = [synth.make_image(w, h, 80 + i, edges=True, bit_depth=bd, chroma_444=c444) for i, (w, h) in enumerate(sizes)]
    want = [enc.encode(im, q).digest() for im, q in zip(images, qs)]
    images = [_pinned(im) for im in images]
    e = Encoder(0)
    try:
        e.serve_open(bd, c444, arena_bytes=256 << 20, max_images=4, max_leaves=1 << 20)   # fewer slots than images
        tickets, done = {}, {}
        pending = list(range(len(images)))
        t0 = time.perf_counter()
        while len(done) < len(images):
            while pending:
                i = pending[0]
                tk = e.serve_submit(images[i], qs[i])
                if tk is None:
                    break
                tickets[tk] = i
                pending.pop(0)
            for tk in e.serve_poll():
                i = tickets.pop(tk)
                h, w = images[i][0].shape
                done[i] = e.serve_fetch(tk, w, h, qs[i], bd, c444).digest()
            assert time.perf_counter() - t0 < 60
            time.sleep(0.0005)
        assert [done[i] for i in range(len(images))] == want
    finally:
        e.serve_close()
        e.close()


def test_stream_server_requests_equal_alone(enc):
    """The StreamServer over a mixed-format arrival stream: every result equals its image searched alone."""
    images, qs = [], []
    fmts = [(8, False), (8, False), (10, True), (8, False), (10, True), (8, False)]
    for i, (bd, c444) in enumerate(fmts):
        images.append(synth.make_image(96 + 32 * i, 64 + 16 * i, 90 + i, edges=True, bit_depth=bd, chroma_444=c444))
        qs.append(40 + 30 * i)
    want = [enc.encode(im, q).digest() for im, q in zip(images, qs)]
    srv = serve.StreamServer(hbm_budget=1 << 30, max_images=8, recon_ctas={(8, False): 64, (10, True): 32})
    try:
        reqs = srv.run([(0.005 * i, im, q) for i, (im, q) in enumerate(zip(images, qs))])
    finally:
        srv.close()
    assert [r.record.digest() for r in reqs] == want
    assert all(r.t_done >= r.t_arrive for r in reqs)
