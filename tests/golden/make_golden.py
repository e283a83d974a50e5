"""Writes tests/golden/oracle_*.npz: the oracle's full DecisionRecord, reconstruction and av1core OBU size for small
seeded synthetic images (regression pins of the CPU oracle; the GPU tests compare the kernels against the same
records).  Run from the repository root: python tests/golden/make_golden.py"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402
from av1gpu_b200 import synth  # noqa: E402

CASES = [("oracle_96x64_q120", 96, 64, 120, 21, False), ("oracle_67x45_q200", 67, 45, 200, 22, True),
         ("oracle_128x128_q40", 128, 128, 40, 23, True)]


def main():
    for name, w, h, q, seed, edges in CASES:
        planes = synth.make_image(w, h, seed, edges=edges)
        r = O.encode(planes, q, threads=1)
        rec, nbytes = O.av1g_recon(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs)
        for p in range(3):
            assert np.array_equal(rec[p], r.recon[p])
        np.savez_compressed(os.path.join(ROOT, "tests", "golden", name + ".npz"), w=w, h=h, q=q, seed=seed, edges=edges,
                            y=planes[0], u=planes[1], v=planes[2], blocks=r.blocks.view(np.uint8), block_txb=r.block_txb,
                            txb=r.txb.view(np.uint8), coeffs=r.coeffs, recon_y=r.recon[0], recon_u=r.recon[1],
                            recon_v=r.recon[2], obu_bytes=nbytes)
        print(name, len(r.blocks), "blocks", nbytes, "OBU bytes")


if __name__ == "__main__":
    main()
