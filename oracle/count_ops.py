"""Algorithmic INT32 operation count of the 12 MP workload, from the oracle's counters (test / measurement
infrastructure).  Prints ops per pixel of the open-loop analysis and of the closed loop; the bench's roofline uses the
values this script printed, frozen in av1gpu_b200/roofline.py.

    python oracle/count_ops.py [qindex ...]
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from av1gpu_b200 import synth  # noqa: E402

W, H, SEED = 4000, 3000, 12
planes = synth.make_image(W, H, SEED, edges=True)
for q in [int(a) for a in sys.argv[1:]] or [120]:
    r = O.encode(planes, q)
    a, c = r.op_counts()
    print("qindex %d: analysis %.1f ops/px, closed loop %.1f ops/px (blocks %d)" % (q, a / (W * H), c / (W * H), len(r.blocks)))
