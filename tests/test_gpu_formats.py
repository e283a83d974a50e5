"""10-bit and 4:4:4: the GPU search against the CPU oracle for each format (analysis records of every shape, DP leaves,
the record, the reconstruction) and the GPU reconstruction against av1core's av1g_encode() of the GPU's own record,
bit-exact; 4:4:4 blocks with a 64-sample side (several chroma tx blocks per plane) included.  A batch that mixes
formats gives, image by image, the single-image result."""
import numpy as np
import pytest

import oracle as O
from av1gpu_b200 import synth

pytestmark = pytest.mark.gpu

SHAPES = [s for s in range(22) if not (13 <= s <= 15)]
FORMATS = [(10, False), (8, True), (10, True)]


def _image(w, h, seed, bd, c444, smooth):
    if smooth:
        return synth.make_smooth_image(w, h, seed, bd, c444)
    return synth.make_image(w, h, seed, edges=True, bit_depth=bd, chroma_444=c444)


def _same_record(a, b):
    return (len(a.blocks) == len(b.blocks) and np.array_equal(a.blocks.view(np.uint8), b.blocks.view(np.uint8))
            and np.array_equal(a.block_txb, b.block_txb) and np.array_equal(a.txb.view(np.uint8), b.txb.view(np.uint8))
            and np.array_equal(a.coeffs, b.coeffs) and all(np.array_equal(x, y) for x, y in zip(a.recon, b.recon)))


def check(enc, w, h, q, seed, bd, c444, smooth=False):
    planes = _image(w, h, seed, bd, c444, smooth)
    g = enc.encode(planes, q)
    o = O.encode(planes, q, bit_depth=bd, chroma_444=c444)
    for s in SHAPES:
        gJ, gc, gn, gt = enc.debug_analysis(s)
        oJ, oc, on, ot = o.analysis(s)
        bad = np.nonzero((gJ != oJ) | (gn != on) | (gt != ot) | np.any(gc != oc, axis=1))[0]
        assert len(bad) == 0, "analysis of shape %d differs at block %d" % (s, bad[0])
    nsb = ((2 * ((w + 7) >> 3) + 15) >> 4) * ((2 * ((h + 7) >> 3) + 15) >> 4)
    for sb in range(nsb):
        for a, b in zip(enc.debug_leaves(sb), o.leaves(sb)):
            assert np.array_equal(a, b), "leaves of SB %d differ" % sb
    assert len(g.blocks) == len(o.blocks) and len(g.txb) == len(o.txb) and len(g.coeffs) == len(o.coeffs)
    gb, ob = g.blocks.view(np.uint8).reshape(-1, 16), o.blocks.view(np.uint8).reshape(-1, 16)
    bad = np.nonzero(np.any(gb != ob, axis=1))[0]
    assert len(bad) == 0, "block %d differs: gpu %s oracle %s" % (bad[0], g.blocks[bad[0]], o.blocks[bad[0]])
    assert np.array_equal(g.block_txb, o.block_txb)
    gt, ot = g.txb.view(np.uint8).reshape(-1, 16), o.txb.view(np.uint8).reshape(-1, 16)
    bad = np.nonzero(np.any(gt != ot, axis=1))[0]
    assert len(bad) == 0, "txb %d differs: gpu %s oracle %s" % (bad[0], g.txb[bad[0]], o.txb[bad[0]])
    assert np.array_equal(g.coeffs, o.coeffs)
    for p in range(3):
        assert np.array_equal(g.recon[p], o.recon[p]), "reconstruction plane %d differs from the oracle" % p
    rec, _ = O.av1g_recon(w, h, q, g.blocks, g.block_txb, g.txb, g.coeffs, bit_depth=bd, chroma_444=c444)
    for p in range(3):
        assert np.array_equal(rec[p], g.recon[p]), "av1g_encode reconstruction of the GPU record differs (plane %d)" % p
    return g


@pytest.mark.parametrize("bd,c444", FORMATS)
@pytest.mark.parametrize("w,h,q,seed", [(211, 149, 120, 41), (96, 72, 40, 42)])
def test_formats_match_oracle(enc, bd, c444, w, h, q, seed):
    check(enc, w, h, q, seed, bd, c444)


@pytest.mark.parametrize("bd,c444", FORMATS)
@pytest.mark.parametrize("w,h,q", [(192, 160, 200), (150, 100, 180), (97, 130, 220)])
def test_formats_large_blocks(enc, bd, c444, w, h, q):
    """Smooth images: 64-sample-side blocks (4:4:4: 2 or 4 chroma tx blocks per plane, some cut by the frame edge)."""
    g = check(enc, w, h, q, 43, bd, c444, smooth=True)
    assert np.isin(g.blocks["bsize"], [10, 11, 12, 20, 21]).any()


def test_mixed_format_batch(enc):
    """One batch of 8-bit 4:2:0, 10-bit 4:4:4, 8-bit 4:4:4 and 10-bit 4:2:0 images (one closed-loop group per format)
    equals the single-image searches, with and without graph capture."""
    spec = [(160, 120, 60, 8, False, False), (150, 100, 180, 10, True, True), (211, 149, 120, 8, True, False),
            (96, 200, 150, 10, False, False), (128, 96, 200, 8, False, True)]
    images = [_image(w, h, 50 + i, bd, c444, sm) for i, (w, h, _, bd, c444, sm) in enumerate(spec)]
    qs = [s[2] for s in spec]
    singles = [enc.encode(im, q) for im, q in zip(images, qs)]
    for graph in (False, True):
        enc.set_batch_options(use_graph=graph, front_streams=2)
        batch = enc.encode_batch(images, qs)
        for i, (s, b) in enumerate(zip(singles, batch)):
            assert _same_record(s, b), "image %d of the mixed batch differs (graph %s)" % (i, graph)
    enc.set_batch_options(use_graph=False, front_streams=1)
