"""CPU-only tests (no GPU): the oracle against its golden records and against av1core's own reconstruction, the
independent restatements of the forward transform (generated CUDA networks vs the oracle), the fixed-point tables the
library uploads vs the oracle's, and the C ABI's exported symbols."""
import glob
import os
import re
import subprocess
import sys

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "oracle_*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_golden(path):
    """The oracle reproduces its committed golden records, and av1core reconstructs them sample for sample."""
    g = np.load(path)
    w, h, q = int(g["w"]), int(g["h"]), int(g["q"])
    planes = (g["y"], g["u"], g["v"])
    r = O.encode(planes, q, threads=2)
    assert np.array_equal(r.blocks.view(np.uint8).ravel(), g["blocks"].ravel())
    assert np.array_equal(r.block_txb, g["block_txb"])
    assert np.array_equal(r.txb.view(np.uint8).ravel(), g["txb"].ravel())
    assert np.array_equal(r.coeffs, g["coeffs"])
    for p, k in enumerate(("recon_y", "recon_u", "recon_v")):
        assert np.array_equal(r.recon[p], g[k])
    rec, nbytes = O.av1g_recon(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs)
    assert nbytes == int(g["obu_bytes"])
    for p in range(3):
        assert np.array_equal(rec[p], r.recon[p])


@pytest.mark.parametrize("w,h,q,seed", [(256, 192, 120, 31), (200, 136, 60, 32), (72, 300, 220, 33), (4, 4, 10, 34)])
def test_oracle_recon_is_av1core(w, h, q, seed):
    """Every oracle record is a valid DecisionRecord whose av1core reconstruction is the oracle's own."""
    from av1gpu_b200 import synth
    planes = synth.make_image(w, h, seed, edges=True)
    r = O.encode(planes, q)
    rec, _ = O.av1g_recon(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs)
    for p in range(3):
        assert np.array_equal(rec[p], r.recon[p])


@pytest.mark.parametrize("bd,c444,w,h,q,smooth", [(10, False, 200, 136, 120, False), (8, True, 200, 136, 120, False),
                                                  (10, True, 150, 100, 180, True), (8, True, 192, 160, 200, True)])
def test_oracle_formats_recon_is_av1core(bd, c444, w, h, q, smooth):
    """10-bit and 4:4:4 oracle records are valid DecisionRecords whose av1core reconstruction is the oracle's own,
    including 4:4:4 blocks with a 64-sample side (2 or 4 chroma tx blocks per plane)."""
    from av1gpu_b200 import synth
    planes = (synth.make_smooth_image(w, h, 7, bd, c444) if smooth else synth.make_image(w, h, 7, edges=True, bit_depth=bd,
                                                                                          chroma_444=c444))
    r = O.encode(planes, q, bit_depth=bd, chroma_444=c444)
    if smooth:
        assert np.isin(r.blocks["bsize"], [10, 11, 12, 20, 21]).any()   # a 64-sample side
    rec, _ = O.av1g_recon(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs, bit_depth=bd, chroma_444=c444)
    for p in range(3):
        assert np.array_equal(rec[p], r.recon[p])


def test_oracle_reference_gate_picture():
    """The oracle reproduces its committed records of the reference's CfL frame-edge picture (8-bit 4:2:0 planes from
    tests/gate_images/cfl_edge_211x149.png) at qindex 60 / 120 / 200, and av1core reconstructs them exactly."""
    z = np.load(os.path.join(ROOT, "tests", "golden", "gate_cfl_edge_211x149.npz"))
    planes = (z["y"], z["u"], z["v"])
    h, w = planes[0].shape
    assert (w, h) == (211, 149)
    for q in z["qs"]:
        q = int(q)
        r = O.encode(planes, q, threads=2)
        assert np.array_equal(r.blocks.view(np.uint8), z["blocks_%d" % q]) and np.array_equal(r.block_txb, z["block_txb_%d" % q])
        assert np.array_equal(r.txb.view(np.uint8), z["txb_%d" % q]) and np.array_equal(r.coeffs, z["coeffs_%d" % q])
        for p, k in enumerate("yuv"):
            assert np.array_equal(r.recon[p], z["recon_%s_%d" % (k, q)])
        rec, nbytes = O.av1g_recon(w, h, q, r.blocks, r.block_txb, r.txb, r.coeffs)
        assert nbytes == int(z["obu_bytes_%d" % q])
        for p in range(3):
            assert np.array_equal(rec[p], r.recon[p])
    assert np.any(z["blocks_60"].reshape(-1, 16)[:, 9] == 13)   # uv_mode byte: CfL blocks at the frame edge


def test_oracle_thread_independent():
    """The wavefront over host threads gives the same record as one thread."""
    from av1gpu_b200 import synth
    planes = synth.make_image(300, 200, 35)
    a, b = O.encode(planes, 90, threads=1), O.encode(planes, 90, threads=8)
    assert np.array_equal(a.coeffs, b.coeffs) and np.array_equal(a.blocks, b.blocks)


def _simulate_fwd2d(res, W, H, kind_c, kind_r):
    """2-D forward transform from gen_txfm.py's step lists (what the CUDA header is generated from), in Python."""
    sys.path.insert(0, os.path.join(ROOT, "av1gpu_b200", "csrc"))
    import gen_txfm as g

    def run(ops, T):
        T = list(T)
        for op in reversed(ops):
            if op[0] == 'P':
                src, sgn = op[1], op[2]
                c = list(T)
                for i in range(len(src)):
                    T[src[i]] = sgn[i] * c[i]
            elif op[0] == 'B':
                _, a, b, ang, fl = op
                ang = ang if fl else -ang
                cc, s = g.cos128(ang), g.sin128(ang)
                x = (T[a] * cc - T[b] * s + 2048) >> 12
                y = (T[a] * s + T[b] * cc + 2048) >> 12
                T[a], T[b] = (y, x) if fl else (x, y)
            else:
                _, a, b, fl = op
                if fl:
                    a, b = b, a
                x, y = T[a], T[b]
                T[a], T[b] = x + y, x - y
        return T

    def fwd1(kind, n, T):
        if n >= 32 or kind == 0:
            return run(g.idct_ops(n.bit_length() - 1), T)
        if kind == 1:
            if n == 4:
                S = g.adst4_matrix()
                return [(sum(S[i][j] * T[i] for i in range(4)) + 2048) >> 12 for j in range(4)]
            return run(g.iadst8_ops() if n == 8 else g.iadst16_ops(), T)
        return [((t * 5793 + 2048) >> 12) if n == 4 else (t * 2 if n == 8 else ((t * 11586 + 2048) >> 12)) for t in T]

    lw, lh = W.bit_length() - 1, H.bit_length() - 1
    rowshift = {(4, 4): 0, (4, 8): 0, (8, 4): 0, (16, 16): 2, (32, 32): 2, (64, 64): 2, (8, 32): 2, (32, 8): 2, (16, 64): 2,
                (64, 16): 2}.get((W, H), 1)
    E = rowshift + 4 + 3 - (lw + lh - 2)
    s0 = max(0, 17 - 8 - lh)
    s1 = lw
    s2 = s0 - s1 - E
    th, tw = min(H, 32), min(W, 32)
    tmp = [[0] * W for _ in range(th)]
    for j in range(W):
        col = fwd1(kind_c, H, [int(res[i][j]) << s0 for i in range(H)])
        for i in range(th):
            tmp[i][j] = (col[i] + (1 << (s1 - 1))) >> s1
    out = np.zeros((th, tw), np.int64)
    rect = abs(lw - lh) == 1
    for i in range(th):
        row = fwd1(kind_r, W, tmp[i])
        for j in range(tw):
            v = row[j]
            if rect:
                v = (v * 5793 + 2048) >> 12
            v = (v + (1 << (s2 - 1))) >> s2 if s2 > 0 else v * (1 << -s2)
            out[i, j] = v
    return out


@pytest.mark.parametrize("tx", [(0, 4, 4, 3), (1, 8, 8, 1), (2, 16, 16, 2), (5, 4, 8, 11), (8, 16, 8, 9), (13, 4, 16, 10),
                                (3, 32, 32, 0), (18, 64, 16, 0)])
def test_generated_transform_matches_oracle(tx):
    """The generated straight-line networks of the kernels and the oracle's recorded-and-transposed step lists are two
    independent restatements of the spec's inverse step lists: their forward transforms agree exactly."""
    t, W, H, ttype = tx
    kind = {0: (0, 0), 1: (1, 0), 2: (0, 1), 3: (1, 1), 9: (2, 2), 10: (0, 2), 11: (2, 0)}[ttype]
    rng = np.random.default_rng(t)
    for _ in range(3):
        res = rng.integers(-255, 256, (H, W))
        assert np.array_equal(_simulate_fwd2d(res, W, H, kind[0], kind[1]), O.fwd2d(res, t, ttype))


def test_generated_header_current():
    """txfm_gen.cuh is what gen_txfm.py generates."""
    gen = os.path.join(ROOT, "av1gpu_b200", "csrc", "gen_txfm.py")
    code = subprocess.run([sys.executable, gen], check=True, capture_output=True, text=True).stdout
    with open(os.path.join(ROOT, "av1gpu_b200", "csrc", "txfm_gen.cuh")) as f:
        assert f.read() == code


def test_library_exports_and_tables():
    """libisearch.so loads without a GPU, exports every entry point of include/is_api.h, and its fixed-point tables
    (costs of every CDF symbol, averaged bits, lambda) equal the oracle's."""
    from av1gpu_b200 import isearch
    L = isearch.load_library()
    with open(os.path.join(ROOT, "include", "is_api.h")) as f:
        names = set(re.findall(r"^\s*(?:int|void|const char \*)\s*(is_\w+)\(", f.read(), re.M))
    assert names and names <= set(isearch.EXPORTS)
    for n in names:
        assert hasattr(L, n), n
    for qctx, q in ((0, 10), (1, 60), (2, 120), (3, 230)):
        cost, y, p, s, lam, sq = isearch.host_tables(qctx, q)
        assert np.array_equal(cost, O.cost_table(qctx))
        oy, op, os_ = O.avg_bits()
        assert np.array_equal(y, oy) and np.array_equal(p, op) and s == os_
        assert (lam, sq) == O.lam(q)


def test_ref_engine_runs():
    """The reference's own CPU decision engine (timed beside the search by bench.py) runs from the oracle build."""
    from av1gpu_b200 import synth
    d, e = O.ref_engine_seconds(synth.make_image(128, 96, 36), 120)
    assert d >= 0 and e >= 0
