"""The reference's own GPU search (maddog107/av1gpu GpEncoder::encode with the plain knob set, built from its sources by
oracle/refgpu.mk) beside this build's search on the same seeded pictures:
  - its records reconstruct exactly through av1g_encode (the reference's own --check criterion), so the comparison is
    between two valid encoders;
  - this build's decisions against the reference's as a BD-rate (rate = av1g_encode bytes, quality PSNR-Y, qindex
    40 / 80 / 120 / 160 / 200, PCHIP Bjontegaard).  The reference's forward transform and costs are floating point, this
    build's are integer (its decisions are pinned to the oracle, not to the reference's), so the two differ on near
    ties; the test bounds the difference and prints it (-s)."""
import numpy as np
import pytest

import oracle as O
import ref_gpu
from av1gpu_b200 import synth
from av1gpu_b200.shortlist import bd_rate

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_gpu.available(), reason="oracle/_ref/libref_gpu.so not built")]

QS = (40, 80, 120, 160, 200)


def _psnr(a, b):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return 10 * np.log10(255.0 ** 2 / max(mse, 1e-12))


def test_reference_gpu_search_reconstructs_exactly():
    planes = synth.make_image(640, 384, 9, edges=True)
    h, w = planes[0].shape
    for q in (60, 200):
        r = ref_gpu.search(planes, q)
        assert r.obu_bytes > 0 and r.recon_exact, "av1g_encode does not reproduce the reference GPU search's reconstruction"


def test_bd_rate_against_reference_gpu_search(enc):
    res = []
    for seed in (101, 102, 103, 104):
        planes = synth.make_image(512, 384, seed, edges=True)
        h, w = planes[0].shape
        curves = {"b200": ([], []), "ref": ([], [])}
        for q in QS:
            g = enc.encode(planes, q)
            recon, nbytes = O.av1g_recon(w, h, q, g.blocks, g.block_txb, g.txb, g.coeffs)
            assert np.array_equal(recon[0], g.recon[0])
            curves["b200"][0].append(nbytes)
            curves["b200"][1].append(_psnr(planes[0], g.recon[0]))
            r = ref_gpu.search(planes, q)
            assert r.recon_exact
            curves["ref"][0].append(r.obu_bytes)
            curves["ref"][1].append(_psnr(planes[0], r.recon[0]))
        bd = bd_rate(curves["ref"][0], curves["ref"][1], curves["b200"][0], curves["b200"][1])
        res.append(bd)
        print("seed %d: BD-rate PSNR-Y of this build against the reference GPU search %+.2f %%" % (seed, bd))
    print("mean %+.2f %%" % float(np.mean(res)))
    assert abs(float(np.mean(res))) < 5.0
