"""Writes tests/golden/gate_cfl_edge_211x149.npz: the reference's own test picture for CfL at the frame edge with a
split luma transform (tests/gate_images/cfl_edge_211x149.png of maddog107/av1gpu, used by its decoder gate,
CMakeLists.txt:244-255), converted to the 8-bit 4:2:0 planes the reference encodes from it, plus the oracle's record of
it at qindex 60 / 120 / 200 (a regression pin of the oracle; the GPU test compares the kernels with the oracle).

The conversion restates the reference's PNG ingest (encoder/src/imageio.cpp:336-372): full-range BT.601 RGB -> YCbCr,
each value rounded to nearest and clamped, chroma the rounded mean of each 2 x 2 luma-grid area (edge samples
replicated for odd sizes).  Run from the repository root with the reference checkout's location:

    python tests/golden/make_gate_fixture.py <reference checkout>
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

QS = (60, 120, 200)


def rgb_to_420(rgb):
    """8-bit RGB (h, w, 3) -> (Y, Cb, Cr) uint8 planes, chroma ((w + 1) // 2, (h + 1) // 2)."""
    r, g, b = (rgb[..., k].astype(np.float64) for k in range(3))
    cl = lambda v: np.clip(np.rint(v), 0, 255).astype(np.int64)   # noqa: E731  (lrint: round half to even)
    y = cl(0.299 * r + 0.587 * g + 0.114 * b)
    cb = cl(-0.168735892 * r - 0.331264108 * g + 0.5 * b + 128)
    cr = cl(0.5 * r - 0.418687589 * g - 0.081312411 * b + 128)
    h, w = y.shape
    ch, cw = (h + 1) // 2, (w + 1) // 2
    ys = np.minimum(np.arange(2 * ch), h - 1)
    xs = np.minimum(np.arange(2 * cw), w - 1)

    def sub(c):
        e = c[np.ix_(ys, xs)]
        s = e[0::2, 0::2] + e[0::2, 1::2] + e[1::2, 0::2] + e[1::2, 1::2]
        return ((s + 2) >> 2).astype(np.uint8)
    return y.astype(np.uint8), sub(cb), sub(cr)


def main():
    from PIL import Image
    import oracle as O
    ref = sys.argv[1]
    png = os.path.join(ref, "tests", "gate_images", "cfl_edge_211x149.png")
    rgb = np.asarray(Image.open(png).convert("RGB"))
    planes = rgb_to_420(rgb)
    h, w = planes[0].shape
    out = dict(w=w, h=h, y=planes[0], u=planes[1], v=planes[2], qs=np.array(QS))
    for q in QS:
        r = O.encode(planes, q, threads=1)
        rec, nbytes = O.av1g_recon(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs)
        for p in range(3):
            assert np.array_equal(rec[p], r.recon[p])
        out.update({"blocks_%d" % q: r.blocks.view(np.uint8), "block_txb_%d" % q: r.block_txb, "txb_%d" % q: r.txb.view(np.uint8),
                    "coeffs_%d" % q: r.coeffs, "recon_y_%d" % q: r.recon[0], "recon_u_%d" % q: r.recon[1],
                    "recon_v_%d" % q: r.recon[2], "obu_bytes_%d" % q: nbytes})
        cfl = int(np.sum(r.blocks["uv_mode"] == 13))
        print("q%d: %d blocks (%d CfL), %d OBU bytes" % (q, len(r.blocks), cfl, nbytes))
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "gate_cfl_edge_211x149.npz"), **out)


if __name__ == "__main__":
    main()
