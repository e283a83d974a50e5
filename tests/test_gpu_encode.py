"""Whole-path parity of the plain form: the GPU search (C ABI) against the CPU oracle on the same seeded synthetic
images - analysis records of every shape, DP leaves, every DecisionRecord field, every level - and the GPU
reconstruction against av1core's av1g_encode() of the GPU's own record.  Bit-exact."""
import os

import numpy as np
import pytest

import oracle as O
from av1gpu_b200 import synth

pytestmark = pytest.mark.gpu

SHAPES = [s for s in range(22) if not (13 <= s <= 15)]


def first_diff(a, b):
    idx = np.nonzero(a != b)[0]
    return int(idx[0]) if len(idx) else -1


def check_image(enc, w, h, q, seed, edges=False, threads=None):
    return check_planes(enc, synth.make_image(w, h, seed, edges=edges), q, threads)


def check_planes(enc, planes, q, threads=None):
    h, w = planes[0].shape
    g = enc.encode(planes, q)
    o = O.encode(planes, q, threads=threads)
    # analysis (every shape, every position) and leaves: localise a difference before comparing the record
    for s in SHAPES:
        gJ, gc, gn, gt = enc.debug_analysis(s)
        oJ, oc, on, ot = o.analysis(s)
        assert len(gJ) == len(oJ)
        bad = np.nonzero((gJ != oJ) | (gn != on) | (gt != ot) | np.any(gc != oc, axis=1))[0]
        assert len(bad) == 0, "analysis of shape %d differs at block %d: gpu J=%d c=%s tx=%d, oracle J=%d c=%s tx=%d" % (
            s, bad[0], gJ[bad[0]], list(gc[bad[0]]), gt[bad[0]], oJ[bad[0]], list(oc[bad[0]]), ot[bad[0]])
    nsb = ((2 * ((w + 7) >> 3) + 15) >> 4) * ((2 * ((h + 7) >> 3) + 15) >> 4)
    for sb in range(nsb):
        gl, ol = enc.debug_leaves(sb), o.leaves(sb)
        for a, b in zip(gl, ol):
            assert np.array_equal(a, b), "leaves of SB %d differ" % sb
    assert len(g.blocks) == len(o.blocks) and len(g.txb) == len(o.txb) and len(g.coeffs) == len(o.coeffs)
    gb, ob = g.blocks.view(np.uint8).reshape(-1, 16), o.blocks.view(np.uint8).reshape(-1, 16)
    bad = np.nonzero(np.any(gb != ob, axis=1))[0]
    assert len(bad) == 0, "block %d differs: gpu %s oracle %s" % (bad[0], g.blocks[bad[0]], o.blocks[bad[0]])
    assert np.array_equal(g.block_txb, o.block_txb)
    gt, ot = g.txb.view(np.uint8).reshape(-1, 16), o.txb.view(np.uint8).reshape(-1, 16)
    bad = np.nonzero(np.any(gt != ot, axis=1))[0]
    assert len(bad) == 0, "txb %d differs: gpu %s oracle %s" % (bad[0], g.txb[bad[0]], o.txb[bad[0]])
    d = first_diff(g.coeffs, o.coeffs)
    assert d < 0, "coefficient %d differs" % d
    for p in range(3):
        assert np.array_equal(g.recon[p], o.recon[p]), "reconstruction plane %d differs from the oracle" % p
    rec, nbytes = O.av1g_recon(w, h, q, g.blocks, g.block_txb, g.txb, g.coeffs)
    for p in range(3):
        assert np.array_equal(rec[p], g.recon[p]), "av1g_encode reconstruction of the GPU record differs (plane %d)" % p
    return g, nbytes


def test_encode_config1_512(enc):
    """The reference's CPU-runnable case: 512x512 8-bit 4:2:0, qindex 120."""
    check_image(enc, 512, 512, 120, seed=1)


@pytest.mark.parametrize("w,h,q,seed", [(211, 149, 60, 2), (333, 77, 200, 3), (8, 8, 255, 4), (64, 72, 40, 5),
                                        (130, 66, 1, 6), (96, 200, 160, 7)])
def test_encode_odd_sizes(enc, w, h, q, seed):
    """Frame edges that cut superblocks and blocks, minimum sizes, the qindex extremes."""
    check_image(enc, w, h, q, seed)


def test_encode_two_tile_columns(enc):
    """A picture wider than 4096 samples has two tile columns: availability and contexts are tile-local."""
    check_image(enc, 4160, 72, 120, seed=8, edges=True)


@pytest.mark.parametrize("q", [60, 120, 200])
def test_encode_edges_qindex(enc, q):
    """The step-edge recipe of the 12 MP workload at its three qindex values (reduced size)."""
    check_image(enc, 640, 384, q, seed=9, edges=True)


@pytest.mark.parametrize("q", [60, 120, 200])
def test_encode_bench_image_full_size(enc, q):
    """The benchmark's own image at full size (4000x3000 12 MP, seed 12, step edges) at the three qindex values of the
    12 MP workload: every analysis record, leaf and record field against the oracle (on all host cores), and the
    reconstruction through av1g_encode."""
    check_image(enc, 4000, 3000, q, seed=12, edges=True, threads=os.cpu_count())


@pytest.mark.parametrize("q", [60, 120, 200])
def test_encode_reference_gate_picture(enc, q):
    """The reference's own test picture for CfL at the frame edge (tests/gate_images/cfl_edge_211x149.png, converted
    by tests/golden/make_gate_fixture.py), against the oracle and av1g_encode."""
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "gate_cfl_edge_211x149.npz"))
    g, _ = check_planes(enc, (z["y"], z["u"], z["v"]), q)
    assert np.array_equal(g.coeffs, z["coeffs_%d" % q]) and np.array_equal(g.blocks.view(np.uint8), z["blocks_%d" % q])


def test_repeat_deterministic(enc):
    """Two encodes of the same input give identical records (the wavefront's run order does not matter)."""
    planes = synth.make_image(300, 200, 11)
    a = enc.encode(planes, 100)
    b = enc.encode(planes, 100)
    assert np.array_equal(a.coeffs, b.coeffs) and np.array_equal(a.blocks, b.blocks)
    for p in range(3):
        assert np.array_equal(a.recon[p], b.recon[p])
