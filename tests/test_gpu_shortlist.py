"""The learned shortlist's kernels: the BF16 tensor-core GEMM against a PyTorch fp32 reference of the same op, the
training forward pass and gradients against the CPU restatement (oracle/shortlist_ref.py), the features against a numpy
restatement, the fused inference kernel against the GEMM path, the dataset against the analysis records, a short
training run, and the search with a shortlist (fallback = plain form; exact reconstruction; the lists obeyed)."""
import ctypes as C

import numpy as np
import pytest

import shortlist_ref as R
from av1gpu_b200 import shortlist as SL
from av1gpu_b200 import synth

pytestmark = pytest.mark.gpu

SCORED = [3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 16, 17, 18, 19, 20, 21]   # compact order of the scored shapes
DIMS = {3: (8, 8), 4: (8, 16), 5: (16, 8), 6: (16, 16), 7: (16, 32), 8: (32, 16), 9: (32, 32), 10: (32, 64), 11: (64, 32),
        12: (64, 64), 16: (4, 16), 17: (16, 4), 18: (8, 32), 19: (32, 8), 20: (16, 64), 21: (64, 16)}


def _rows(rng, n):
    X = (rng.standard_normal((n, R.N_FEAT)) * 0.5).astype(np.float32)
    y = np.zeros((n, 3), np.int32)
    y[:, 0] = rng.integers(0, R.N_MD, n)
    sets = [0b111000001111, 0b1000001111, 0]
    for r in range(n):
        v = sets[r % 3]
        y[r, 2] = v
        ks = [k for k in range(16) if (v >> k) & 1]
        y[r, 1] = rng.choice(ks) if ks else -1
    return X, y


def test_gemm_matches_torch_fp32():
    import torch
    from av1gpu_b200.isearch import load_library
    L = load_library()
    g = torch.Generator(device="cpu").manual_seed(1)
    for (M, N, K) in ((1000, 160, 288), (16, 128, 4096), (4096, 16, 144), (77, 50, 24), (65536, 8, 16)):
        A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
        B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
        bias = torch.randn(N, generator=g).cuda()
        Cm = torch.empty(M, N, device="cuda")
        rc = L.is_nn_gemm(M, N, K, C.c_void_p(A.data_ptr()), K, C.c_void_p(B.data_ptr()), K, C.c_void_p(Cm.data_ptr()), N,
                          C.c_void_p(bias.data_ptr()), 1, None)
        assert rc == 0
        ref = torch.relu(A.float() @ B.float().T + bias)
        tol = 1e-3 * (K ** 0.5) * 4   # fp32 accumulation in another order than the reference (relative to |entries| ~ sqrt(K))
        assert float((Cm - ref).abs().max()) < tol, (M, N, K, float((Cm - ref).abs().max()))


def test_forward_and_gradients_match_the_cpu_restatement():
    import torch
    rng = np.random.default_rng(3)
    n = 96
    X, y = _rows(rng, n)
    p = SL.init_params(5)
    p[-80:] = rng.standard_normal(80).astype(np.float32) * 0.2
    lrn = SL.Learner(max_batch=256)
    try:
        lrn.set_params(p)
        Xt = torch.from_numpy(X).to(torch.bfloat16).cuda()
        S = lrn.forward(Xt).cpu().numpy()
        g, loss, corr = lrn.grads(Xt, torch.from_numpy(y).cuda())
    finally:
        lrn.close()
    Xb = R.bf16(X)
    f = R.forward(Xb, p.astype(np.float64))
    assert np.abs(S - f["s"]).max() < 2e-2 * (np.abs(f["s"]).max() + 1)
    gr, lref, cref = R.grads(Xb, y, p.astype(np.float64))
    assert abs(loss - lref) < 2e-3 * max(1.0, lref)
    assert abs(corr - cref) <= 2
    o = 0
    for name, shp in R.SHAPES:
        k = int(np.prod(shp))
        a, b = g[o:o + k], gr[o:o + k]
        err = np.abs(a - b).max() / (np.abs(b).max() + 1e-12)
        assert err < 5e-2, (name, err)   # bf16 operands of the backward GEMMs: ~1e-2 relative
        o += k


def _padded_luma(planes):
    Y = planes[0].astype(np.float64)
    h, w = Y.shape
    H, W = (h + 63) // 64 * 64 + 64, (w + 63) // 64 * 64 + 64
    return np.pad(Y, ((0, H - h), (0, W - w)), mode="edge")


def _cells(Yp, bs, x, y):
    w, h = DIMS[bs]
    mx, my = (w + 7) // 8, (h + 7) // 8
    RW, RH, x0, y0 = w + mx, h + my, x - mx, y - my
    out = np.zeros((32, 32))
    for i in range(32):
        r0, r1 = y0 + (i * RH) // 32, y0 + ((i + 1) * RH) // 32
        r1 = max(r1, r0 + 1)
        for j in range(32):
            c0, c1 = x0 + (j * RW) // 32, x0 + ((j + 1) * RW) // 32
            c1 = max(c1, c0 + 1)
            out[i, j] = Yp[np.ix_(np.maximum(np.arange(r0, r1), 0), np.maximum(np.arange(c0, c1), 0))].mean()
    return out


def _hist(c):
    gx = c[:, np.minimum(np.arange(32) + 1, 31)] - c[:, np.maximum(np.arange(32) - 1, 0)]
    gy = c[np.minimum(np.arange(32) + 1, 31), :] - c[np.maximum(np.arange(32) - 1, 0), :]
    m = np.abs(gx) + np.abs(gy)
    flip = (gy < 0) | ((gy == 0) & (gx < 0))
    ax, ay = np.where(flip, -gx, gx), np.where(flip, -gy, gy)
    t1, t2 = 0.41421356, 2.41421356
    b = np.where(ax >= 0, np.where(ay <= t1 * ax, 0, np.where(ay <= ax, 1, np.where(ay <= t2 * ax, 2, 3))),
                 np.where(ay >= -t2 * ax, 4, np.where(ay >= -ax, 5, np.where(ay >= -t1 * ax, 6, 7))))
    hist = np.array([m[b == q].sum() for q in range(8)])
    return hist / (hist.sum() + 1)


def test_features_match_a_numpy_restatement(enc):
    w, h, q = 200, 136, 120
    im = synth.make_image(w, h, 47, edges=True)
    enc.encode(im, q)
    X, y = SL.image_rows(enc, keep_outside=True)
    X = X.float().cpu().numpy()
    Yp = _padded_luma(im)
    fw, fh = 2 * ((w + 7) >> 3) * 4, 2 * ((h + 7) >> 3) * 4
    rng = np.random.default_rng(0)
    row = 0
    checked = 0
    for s in SCORED:
        bw, bh = DIMS[s]
        nbx, nby = (fw + bw - 1) // bw, (fh + bh - 1) // bh
        picks = set(rng.integers(0, nbx * nby, 6).tolist())
        for r in range(nbx * nby):
            x, yy = (r % nbx) * bw, (r // nbx) * bh
            if r in picks and x < fw and yy < fh:
                c = _cells(Yp, s, x, yy)
                ref = (c - c.mean()) / 64.0
                got = X[row + r, :1024].reshape(32, 32)
                assert np.all(np.abs(got - ref) <= 2 ** -7 * np.maximum(np.abs(ref), 2 ** -6) + 1e-6), (s, x, yy)
                ext = X[row + r, 1024:]
                assert np.allclose(ext[:8], _hist(c), atol=4e-3), (s, x, yy)
                onehot = np.zeros(16)
                onehot[SCORED.index(s)] = 1
                assert np.array_equal(ext[8:24], onehot) and abs(ext[24] - q / 255) < 4e-3 and ext[25] == 1
                checked += 1
        row += nbx * nby
    assert row == X.shape[0] and checked > 40


def test_dataset_labels_are_the_search_choices(enc):
    im = synth.make_image(192, 128, 41, edges=True)
    enc.encode(im, 120)
    X, y = SL.image_rows(enc, keep_outside=True)
    y = y.cpu().numpy()
    fw, fh = 192, 128
    row = 0
    for s in SCORED:
        J, cand, nc, tx = enc.debug_analysis(s)
        bw, bh = DIMS[s]
        nbx = (fw + bw - 1) // bw
        for r in range(len(J)):
            x, yy = (r % nbx) * bw, (r // nbx) * bh
            if x < fw and yy < fh:
                assert SL.CLASS_CAND[y[row + r, 0]] == cand[r, 0]
                dct_only = s not in (3, 4, 5, 6, 16, 17)   # tx sizes with a 32- or 64-sample side
                assert y[row + r, 1] == (-1 if dct_only else tx[r])
            else:
                assert y[row + r, 0] == -1
        row += len(J)
    assert row == len(y)


def test_fused_inference_matches_the_gemm_path(enc):
    import torch
    im = synth.make_image(256, 192, 48, edges=True)
    enc.encode(im, 90)
    X, y = SL.image_rows(enc, keep_outside=True)
    p = SL.init_params(9)
    p[-80:] = np.random.default_rng(1).standard_normal(80).astype(np.float32) * 0.3
    lrn = SL.Learner(max_batch=4096)
    try:
        lrn.set_params(p)
        Sg = lrn.forward(X)
        Sf = torch.full_like(Sg, float("nan"))
        n = C.c_int()
        assert enc.L.is_sl_infer(enc.h, lrn.h, 0, C.c_void_p(Sf.data_ptr()), Sf.shape[0], C.byref(n)) == 0 and n.value == X.shape[0]
    finally:
        lrn.close()
    inside = y[:, 0] >= 0
    a, b = Sf[inside], Sg[inside]
    assert torch.isfinite(a).all()
    scale = float(b.abs().max()) + 1
    assert float((a - b).abs().max()) < 2e-2 * scale
    assert float((a[:, :61].argmax(1) == b[:, :61].argmax(1)).float().mean()) > 0.99


def test_training_lowers_the_loss(enc):
    ims = [synth.make_image(256, 192, 60 + i, edges=True) for i in range(3)]
    X, y = SL.dataset(enc, ims, [60, 120, 200])
    lrn = SL.Learner(max_batch=2048)
    try:
        lrn.set_params(SL.init_params(0))
        hist = SL.train(lrn, X, y, epochs=6, batch=512, lr=3e-3)
        ev = SL.evaluate(lrn, X, y, tau=0.9, max_cand=8)
    finally:
        lrn.close()
    assert hist[-1][0] < hist[0][0] * 0.9
    assert ev["coverage"] >= ev["top1"] and ev["mean_cand"] <= 8


def test_search_with_every_block_falling_back_equals_plain(enc):
    im = synth.make_image(211, 149, 43, edges=True)
    plain = enc.encode(im, 120)
    enc.set_shortlist(SL.init_params(1), conf=1.0)   # no top probability reaches 1: every block searches in full
    try:
        same = enc.encode(im, 120)
    finally:
        enc.set_shortlist(None)
    assert np.array_equal(plain.blocks.view(np.uint8), same.blocks.view(np.uint8))
    assert np.array_equal(plain.coeffs, same.coeffs)


def test_search_with_shortlist_is_exact_and_obeys_the_lists(enc):
    import torch
    import oracle as O
    w, h, q = 256, 160, 120
    im = synth.make_image(w, h, 44, edges=True)
    p = SL.init_params(2)
    enc.set_shortlist(p, tau=0.6, max_cand=3, rd_k=2, tx_tau=0.5, max_tx=1)   # untrained net: arbitrary small lists
    try:
        a = enc.encode(im, q)
        b = enc.encode(im, q)
        recs = {s: enc.debug_analysis(s, tx_mask=True) for s in SCORED}
        X, y = SL.image_rows(enc, keep_outside=True)
    finally:
        enc.set_shortlist(None)
    assert np.array_equal(a.blocks.view(np.uint8), b.blocks.view(np.uint8)) and np.array_equal(a.coeffs, b.coeffs)
    rec, nbytes = O.av1g_recon(w, h, q, a.blocks, a.block_txb, a.txb, a.coeffs)
    for pl in range(3):
        assert np.array_equal(rec[pl], a.recon[pl])
    assert nbytes > 0
    # the analysis took its candidates and tx types from the lists the selection rule gives for the network's scores
    lrn = SL.Learner(max_batch=4096)
    try:
        lrn.set_params(p)
        S = lrn.forward(X)
    finally:
        lrn.close()
    # (the kernel's scores differ from the GEMM path's in the last bits: a list at a slightly larger / smaller tau is a
    # superset / subset of the kernel's)
    mask, _, tmask = SL.select(S, y[:, 2], tau=0.65, max_cand=3, conf=0.0, tx_tau=0.55, max_tx=1)
    _, _, tsub = SL.select(S, y[:, 2], tau=0.55, max_cand=3, conf=0.0, tx_tau=0.45, max_tx=1)
    mask, tmask, tsub, y = mask.cpu().numpy(), tmask.cpu().numpy(), tsub.cpu().numpy(), y.cpu().numpy()
    row, checked = 0, 0
    for s in SCORED:
        J, cand, nc, tx, tm = recs[s]
        for r in range(len(J)):
            k = row + r
            if y[k, 0] < 0:
                continue
            allowed = set(SL.CLASS_CAND[np.nonzero(mask[k])[0]].tolist())
            assert cand[r, 0] in allowed and nc[r] <= 2
            sup = sum(1 << t for t in np.nonzero(tmask[k])[0].tolist())
            sub = sum(1 << t for t in np.nonzero(tsub[k])[0].tolist())
            assert tx[r] == 0 or (sup >> int(tx[r])) & 1
            assert (int(tm[r]) & ~sup) == 0 and (sub & ~int(tm[r])) == 0
            checked += 1
        row += len(J)
    assert checked > 100
