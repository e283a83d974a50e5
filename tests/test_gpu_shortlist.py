"""The learned shortlist's kernels: the BF16 tensor-core GEMM against a PyTorch fp32 reference of the same op, the
training gradients against the CPU restatement (oracle/shortlist_ref.py), the dataset against the analysis records,
and a short training run that lowers the loss."""
import numpy as np
import pytest

import shortlist_ref as R
from av1gpu_b200 import shortlist as SL
from av1gpu_b200 import synth

pytestmark = pytest.mark.gpu


def test_gemm_matches_torch_fp32():
    import torch
    from av1gpu_b200.isearch import load_library
    L = load_library()
    g = torch.Generator(device="cpu").manual_seed(1)
    for (M, N, K) in ((1000, 128, 288), (16, 128, 4096), (4096, 16, 128), (77, 50, 24)):
        A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
        B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
        bias = torch.randn(N, generator=g).cuda()
        Cm = torch.empty(M, N, device="cuda")
        import ctypes as C
        rc = L.is_nn_gemm(M, N, K, C.c_void_p(A.data_ptr()), K, C.c_void_p(B.data_ptr()), K, C.c_void_p(Cm.data_ptr()), N,
                          C.c_void_p(bias.data_ptr()), 1, None)
        assert rc == 0
        ref = torch.relu(A.float() @ B.float().T + bias)
        tol = 1e-3 * (K ** 0.5) * 4   # fp32 accumulation in another order than the reference (relative to |entries| ~ sqrt(K))
        assert float((Cm - ref).abs().max()) < tol, (M, N, K, float((Cm - ref).abs().max()))


def test_gradients_match_the_cpu_restatement():
    import torch
    rng = np.random.default_rng(3)
    n = 256
    X = rng.standard_normal((n, SL.N_IN)).astype(np.float32) * 0.5
    y = rng.integers(0, SL.N_MODES, n).astype(np.int32)
    w = SL.init_weights(5)
    lr = SL.Learner(max_batch=1024)
    try:
        lr.set_weights(w)
        Xt = torch.from_numpy(X).to(torch.bfloat16).cuda()
        g, loss, corr = lr.grads(Xt, torch.from_numpy(y).cuda())
    finally:
        lr.close()
    Xb = R.bf16(X)
    wb = [R.bf16(w[0]), w[1].astype(np.float64), R.bf16(w[2]), w[3].astype(np.float64)]
    gr, lref, cref = R.grads(Xb, y, *wb)
    assert abs(loss - lref) < 2e-3 * max(1.0, lref)
    assert abs(corr - cref) <= 2
    for a, b, name in zip(g, gr, ("w1", "b1", "w2", "b2")):
        err = np.abs(a - b).max() / (np.abs(b).max() + 1e-12)
        assert err < 3e-2, (name, err)   # bf16 operands of the backward GEMMs: ~1e-2 relative


def test_dataset_labels_are_the_search_choices(enc):
    import torch
    im = synth.make_image(192, 128, 41, edges=True)
    X, y = SL.dataset(enc, [im], [120])
    assert X.shape[1] == SL.N_IN and X.shape[0] == y.shape[0] > 0
    # the labels are the analysis records' best modes, shape by shape
    modes = []
    for s in range(22):
        if 13 <= s <= 15:
            continue
        J, cand, nc, tx = enc.debug_analysis(s)
        modes.append(cand[:, 0] >> 3)
    assert np.array_equal(np.concatenate(modes).astype(np.int32), y.cpu().numpy())
    assert torch.isfinite(X.float()).all()


def test_training_lowers_the_loss(enc):
    ims = [synth.make_image(256, 192, 60 + i, edges=True) for i in range(3)]
    X, y = SL.dataset(enc, ims, [60, 120, 200])
    lr = SL.Learner(max_batch=2048)
    try:
        lr.set_weights(SL.init_weights(0))
        hist = SL.train(lr, X, y, epochs=6, batch=1024, lr=3e-3)
        ev = SL.evaluate(lr, X, y, tau=0.9, max_modes=6)
    finally:
        lr.close()
    assert hist[-1][0] < hist[0][0] * 0.9
    assert ev["coverage"] > ev["top1"] and ev["mean_modes"] <= 6


def test_search_with_full_masks_equals_plain(enc):
    im = synth.make_image(211, 149, 43, edges=True)
    plain = enc.encode(im, 120)
    enc.set_shortlist(SL.init_weights(1), tau=0.9, max_modes=0)   # every mask full: the plain form
    try:
        same = enc.encode(im, 120)
    finally:
        enc.set_shortlist(None)
    assert np.array_equal(plain.blocks.view(np.uint8), same.blocks.view(np.uint8))
    assert np.array_equal(plain.coeffs, same.coeffs)


def test_search_with_shortlist_is_exact_and_deterministic(enc):
    import oracle as O
    w, h, q = 256, 160, 120
    im = synth.make_image(w, h, 44, edges=True)
    enc.set_shortlist(SL.init_weights(2), tau=0.6, max_modes=3)   # untrained net: arbitrary small mode sets
    try:
        a = enc.encode(im, q)
        b = enc.encode(im, q)
    finally:
        enc.set_shortlist(None)
    assert np.array_equal(a.blocks.view(np.uint8), b.blocks.view(np.uint8)) and np.array_equal(a.coeffs, b.coeffs)
    rec, nbytes = O.av1g_recon(w, h, q, a.blocks, a.block_txb, a.txb, a.coeffs)
    for p in range(3):
        assert np.array_equal(rec[p], a.recon[p])
    assert nbytes > 0
