"""The batched form: images of uneven sizes and mixed qindex searched in one batch (one persistent closed-loop launch
over a shared ready queue) give, image by image, exactly the single-image result and the oracle's record; the same
holds with the front ends on several streams and with the batch captured and replayed as a CUDA graph."""
import numpy as np
import pytest

import oracle as O
from av1gpu_b200 import synth

pytestmark = pytest.mark.gpu

BATCH = [(160, 120, 60, 31), (211, 149, 120, 32), (64, 72, 200, 33), (333, 77, 40, 34), (96, 200, 150, 35)]


def _images():
    return [synth.make_image(w, h, seed, edges=True) for w, h, _, seed in BATCH], [q for _, _, q, _ in BATCH]


def _same(a, b):
    return (np.array_equal(a.blocks.view(np.uint8), b.blocks.view(np.uint8)) and np.array_equal(a.block_txb, b.block_txb)
            and np.array_equal(a.txb.view(np.uint8), b.txb.view(np.uint8)) and np.array_equal(a.coeffs, b.coeffs)
            and all(np.array_equal(x, y) for x, y in zip(a.recon, b.recon)))


def test_batch_equals_single_and_oracle(enc):
    images, qs = _images()
    singles = [enc.encode(im, q) for im, q in zip(images, qs)]
    enc.set_batch_options(use_graph=False, front_streams=1)
    batch = enc.encode_batch(images, qs)
    for i, (s, b) in enumerate(zip(singles, batch)):
        assert _same(s, b), "image %d of the batch differs from its single-image search" % i
    for i in (0, 3):
        o = O.encode(images[i], qs[i])
        assert np.array_equal(batch[i].blocks.view(np.uint8), o.blocks.view(np.uint8))
        assert np.array_equal(batch[i].coeffs, o.coeffs)
        for p in range(3):
            assert np.array_equal(batch[i].recon[p], o.recon[p])


def test_batch_streams_and_graph_replay(enc):
    images, qs = _images()
    enc.set_batch_options(use_graph=False, front_streams=1)
    ref = enc.encode_batch(images, qs)
    enc.set_batch_options(use_graph=False, front_streams=4)
    multi = enc.encode_batch(images, qs)
    enc.set_batch_options(use_graph=True, front_streams=2)
    g1 = enc.encode_batch(images, qs)          # captured
    g2 = enc.encode_batch(images, qs)          # replayed (same signature)
    enc.set_batch_options(use_graph=False, front_streams=1)
    for i in range(len(images)):
        assert _same(ref[i], multi[i]) and _same(ref[i], g1[i]) and _same(ref[i], g2[i]), "image %d" % i


def test_autotune_batch(enc):
    """The autotuner's choice (front-end streams x closed-loop warps per CTA) changes the speed, not the results."""
    images, qs = _images()
    planes = [[np.ascontiguousarray(p) for p in im] for im in images]
    ref = [enc.encode(im, q) for im, q in zip(images, qs)]
    k, w, ms = enc.autotune_batch(planes, qs, with_warps=True)
    assert k in (1, 2, 4) and w in (0, 4, 6) and ms > 0
    try:
        for warps in (1, 3):
            enc.set_closed_loop_warps(warps)
            got = enc.encode_batch(planes, qs)
            for i in range(len(images)):
                assert _same(ref[i], got[i]), (warps, i)
    finally:
        enc.set_closed_loop_warps(0)
        enc.set_batch_options(use_graph=False, front_streams=1)


def test_batched_workload_slice_equals_one_at_a_time(enc):
    """A 16-image slice of the batched-form workload: the benchmark's 12 MP image plus crops of smaller 8-bit 4:2:0 and
    10-bit 4:4:4 pictures (the workload generator with reduced base pictures), mixed qindex.  The batch, captured and
    replayed as a CUDA graph with 4 front-end streams, gives every image bit for bit its one-at-a-time result."""
    from av1gpu_b200 import batchbench
    from av1gpu_b200.isearch import plane_format
    work = batchbench.workload(15, seed=5, max_mp=2.0, frac10=0.3, base8=(2000, 1500), base10=(1600, 1000))
    images = [synth.make_image(4000, 3000, 12, edges=True)] + [p for p, _ in work]
    qs = [120] + [q for _, q in work]
    assert sum(plane_format(im)[0] == 10 for im in images) >= 2 and images[0][0].size >= 12e6
    singles = [enc.encode(im, q).digest() for im, q in zip(images, qs)]
    enc.set_batch_options(use_graph=True, front_streams=4)
    try:
        enc.encode_batch(images, qs)                 # captured
        batch = enc.encode_batch(images, qs)         # replayed
    finally:
        enc.set_batch_options(use_graph=False, front_streams=1)
    for i, (s, b) in enumerate(zip(singles, batch)):
        assert s == b.digest(), "image %d (%dx%d, q%d) of the batch differs from its one-at-a-time search" % (
            i, images[i][0].shape[1], images[i][0].shape[0], qs[i])
