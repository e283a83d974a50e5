// is_testapi.cuh - kernel-level entry points for the parity tests and debug readers (include/is_api.h, bottom part).
// Each test kernel runs the same device functions as the search, one warp per block.
#pragma once

namespace {

struct TestScr { int32_t buf[64 * 65]; int16_t q[1024]; };

// one warp per block: the search's own grp_eval (one task, 32 lanes) with a residual array as the source; the
// coefficients are read back from the scratch (quantisation writes only the levels)
__global__ void k_test_fwd_quant(int n, const int32_t *res, int txSz, int txType, int plane, int dcQ, int acQ, int qctx, int skipCtx,
                                 int dcCtx, int intraDir, int32_t *coef, int16_t *lv, long long *D, long long *R, int32_t *eob) {
    extern __shared__ __align__(16) unsigned char tsm[];
    TestScr &S = reinterpret_cast<TestScr *>(tsm)[threadIdx.x >> 5];
    const int b = blockIdx.x * 2 + (threadIdx.x >> 5);
    if (b >= n) return;
    const int W = txw(txSz), H = txh(txSz), tw = min(W, 32), th = min(H, 32), nc = tw * th, lw = 31 - __clz(W);
    const EvalIn e{txType, plane, skipCtx, dcCtx, intraDir, dcQ, acQ, rate_tabs_global(qctx)};
    ResFn<uint8_t> rf{nullptr, 0, nullptr, lw, res + (size_t)b * W * H};
    const EvalOut o = grp_eval<8, uint8_t>(txSz, rf, e, S.buf, S.q, lane_id(), 32);
    for (int idx = lane_id(); idx < nc; idx += 32) {
        coef[(size_t)b * nc + idx] = S.buf[(idx / tw) * (W + 1) + idx % tw];
        lv[(size_t)b * nc + idx] = S.q[idx];
    }
    (void)th;
    if (lane_id() == 0) { D[b] = o.D; R[b] = o.R; eob[b] = o.eob; }
}

__global__ void k_test_inverse(int n, const int16_t *lv, int txSz, int txType, int dcQ, int acQ, int32_t *res, uint32_t *flags) {
    extern __shared__ __align__(16) unsigned char tsm[];
    TestScr &S = reinterpret_cast<TestScr *>(tsm)[threadIdx.x >> 5];
    const int b = blockIdx.x * 2 + (threadIdx.x >> 5);
    if (b >= n) return;
    const int W = txw(txSz), H = txh(txSz), nc = min(W, 32) * min(H, 32);
    const uint32_t f = grp_inverse<8>(txSz, lv + (size_t)b * nc, txType, dcQ, acQ, S.buf, lane_id(), 32);
    for (int p = lane_id(); p < W * H; p += 32) res[(size_t)b * W * H + p] = S.buf[(p / W) * (W + 1) + p % W];
    if (lane_id() == 0) flags[b] = f;
}

__global__ void k_test_predict(int n, const uint8_t *plane, int pw, int ph, const int32_t *params, uint8_t *out) {
    __shared__ uint8_t E[4][2][EDGE_LEN];
    const int b = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (b >= n) return;
    const int32_t *p = params + (size_t)b * 10;
    const int x = p[0], y = p[1], lw = p[2], lh = p[3], hL = p[4], hA = p[5], hAR = p[6], hBL = p[7], mode = p[8], delta = p[9];
    const int w = 1 << lw, h = 1 << lh;
    uint8_t *A = E[threadIdx.x >> 5][0] + EDGE_OFF, *L = E[threadIdx.x >> 5][1] + EDGE_OFF;
    build_edges<8>(plane, pw, x, y, w, h, hL, hA, hAR, hBL, pw - 1, ph - 1, A, L, lane_id(), 32);
    __syncwarp();
    const int dcv = warp_dc<8>(A, L, hL, hA, lw, lh);
    const int pa = pangle(mode, delta);
    for (int q = lane_id(); q < w * h; q += 32) out[(size_t)b * 4096 + q] = (uint8_t)pred_px(mode, pa, q >> lw, q & (w - 1), lw, lh, A, L, dcv);
}

template <typename T>
int dev_upload(is_handle *h, T **d, const T *src, size_t n) {
    if (cudaMalloc((void **)d, n * sizeof(T) + 16) != cudaSuccess) return h->setErr(IS_ERR_OOM, "test alloc");
    if (src && cudaMemcpy(*d, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return h->setErr(IS_ERR_CUDA, "test upload");
    return 0;
}

}  // namespace

extern "C" {

int is_test_fwd_quant(is_handle *h, int n, const int32_t *res, int txSz, int txType, int plane, int qindex, const int32_t ctx[3], int32_t *coef,
                      int16_t *levels, int64_t *D, int64_t *R, int32_t *eob) {
    if (!h || n < 1 || txSz < 0 || txSz > 18 || qindex < 1 || qindex > 255) return IS_ERR_INVALID;
    IS_CK(cudaSetDevice(h->device));
    const int W = AV1G_T(Tx_Width)[txSz], H = AV1G_T(Tx_Height)[txSz], nc = std::min(W, 32) * std::min(H, 32);
    int32_t *dres = nullptr, *dcoef = nullptr, *deob = nullptr;
    int16_t *dlv = nullptr;
    long long *dD = nullptr, *dR = nullptr;
    int rc = dev_upload(h, &dres, res, (size_t)n * W * H);
    if (!rc) rc = dev_upload<int32_t>(h, &dcoef, nullptr, (size_t)n * nc);
    if (!rc) rc = dev_upload<int16_t>(h, &dlv, nullptr, (size_t)n * nc);
    if (!rc) rc = dev_upload<long long>(h, &dD, nullptr, n);
    if (!rc) rc = dev_upload<long long>(h, &dR, nullptr, n);
    if (!rc) rc = dev_upload<int32_t>(h, &deob, nullptr, n);
    if (!rc) {
        cudaFuncSetAttribute(k_test_fwd_quant, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * (int)sizeof(TestScr));
        k_test_fwd_quant<<<(n + 1) / 2, 64, 2 * sizeof(TestScr)>>>(n, dres, txSz, txType, plane, AV1G_T(Dc_Qlookup)[0][qindex], AV1G_T(Ac_Qlookup)[0][qindex],
                                               av1g_coeff_cdf_q_ctx(qindex), ctx[0], ctx[1], ctx[2], dcoef, dlv, dD, dR, deob);
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) rc = h->setErr(IS_ERR_CUDA, "k_test_fwd_quant: %s", cudaGetErrorString(e));
    }
    if (!rc) {
        cudaMemcpy(coef, dcoef, (size_t)n * nc * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(levels, dlv, (size_t)n * nc * 2, cudaMemcpyDeviceToHost);
        cudaMemcpy(D, dD, (size_t)n * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(R, dR, (size_t)n * 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(eob, deob, (size_t)n * 4, cudaMemcpyDeviceToHost);
    }
    cudaFree(dres); cudaFree(dcoef); cudaFree(dlv); cudaFree(dD); cudaFree(dR); cudaFree(deob);
    return rc;
}

int is_test_inverse(is_handle *h, int n, const int16_t *levels, int txSz, int txType, int qindex, int32_t *res, uint32_t *flags) {
    if (!h || n < 1 || txSz < 0 || txSz > 18 || qindex < 1 || qindex > 255) return IS_ERR_INVALID;
    IS_CK(cudaSetDevice(h->device));
    const int W = AV1G_T(Tx_Width)[txSz], H = AV1G_T(Tx_Height)[txSz], nc = std::min(W, 32) * std::min(H, 32);
    int16_t *dlv = nullptr;
    int32_t *dres = nullptr;
    uint32_t *dfl = nullptr;
    int rc = dev_upload(h, &dlv, levels, (size_t)n * nc);
    if (!rc) rc = dev_upload<int32_t>(h, &dres, nullptr, (size_t)n * W * H);
    if (!rc) rc = dev_upload<uint32_t>(h, &dfl, nullptr, n);
    if (!rc) {
        cudaFuncSetAttribute(k_test_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * (int)sizeof(TestScr));
        k_test_inverse<<<(n + 1) / 2, 64, 2 * sizeof(TestScr)>>>(n, dlv, txSz, txType, AV1G_T(Dc_Qlookup)[0][qindex], AV1G_T(Ac_Qlookup)[0][qindex], dres, dfl);
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) rc = h->setErr(IS_ERR_CUDA, "k_test_inverse: %s", cudaGetErrorString(e));
    }
    if (!rc) {
        cudaMemcpy(res, dres, (size_t)n * W * H * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(flags, dfl, (size_t)n * 4, cudaMemcpyDeviceToHost);
    }
    cudaFree(dlv); cudaFree(dres); cudaFree(dfl);
    return rc;
}

int is_test_predict(is_handle *h, int n, const uint8_t *plane, int w, int hgt, const int32_t *params, uint8_t *out) {
    if (!h || n < 1 || w < 1 || hgt < 1) return IS_ERR_INVALID;
    IS_CK(cudaSetDevice(h->device));
    for (int b = 0; b < n; b++) {   // every edge sample the prediction may read lies inside the plane
        const int32_t *p = params + (size_t)b * 10;
        const int x = p[0], y = p[1], bw = 1 << p[2], bh = 1 << p[3];
        if (p[2] < 2 || p[2] > 6 || p[3] < 2 || p[3] > 6 || x < 1 || y < 1 || x + 2 * bw > w || y + 2 * bh > hgt || p[8] < 0 || p[8] > 12 ||
            p[9] < -3 || p[9] > 3)
            return h->setErr(IS_ERR_INVALID, "prediction test block %d out of range", b);
    }
    uint8_t *dp = nullptr, *dout = nullptr;
    int32_t *dpar = nullptr;
    int rc = dev_upload(h, &dp, plane, (size_t)w * hgt);
    if (!rc) rc = dev_upload(h, &dpar, params, (size_t)n * 10);
    if (!rc) rc = dev_upload<uint8_t>(h, &dout, nullptr, (size_t)n * 4096);
    if (!rc) {
        k_test_predict<<<(n + 3) / 4, 128>>>(n, dp, w, hgt, dpar, dout);
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) rc = h->setErr(IS_ERR_CUDA, "k_test_predict: %s", cudaGetErrorString(e));
    }
    if (!rc) cudaMemcpy(out, dout, (size_t)n * 4096, cudaMemcpyDeviceToHost);
    cudaFree(dp); cudaFree(dpar); cudaFree(dout);
    return rc;
}

int is_debug_analysis(is_handle *h, int bs, int64_t *J, uint8_t *cand, uint8_t *ncand, uint8_t *tx, uint16_t *tx_mask) {
    if (!h || !h->have || bs < 0 || bs >= 22) return IS_ERR_STATE;
    const FrameDesc &F = h->F;
    const size_t n = (size_t)F.shNbx[bs] * F.shNby[bs];
    if (!n) return 0;
    std::vector<BlockRes> v(n);
    IS_CK(cudaMemcpy(v.data(), F.blk + F.shOff[bs], n * sizeof(BlockRes), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; i++) {
        if (J) J[i] = v[i].J;
        if (cand) memcpy(cand + 4 * i, v[i].cand, 4);
        if (ncand) ncand[i] = v[i].ncand;
        if (tx) tx[i] = v[i].tx;
        if (tx_mask) tx_mask[i] = v[i].txMask;
    }
    return (int)n;
}

int is_debug_leaves(is_handle *h, uint32_t sb, uint8_t *bsize, uint8_t *x4, uint8_t *y4) {
    if (!h || !h->have || sb >= (uint32_t)h->nSb) return IS_ERR_STATE;
    uint16_t nl = 0;
    IS_CK(cudaMemcpy(&nl, h->F.nLeaves + sb, 2, cudaMemcpyDeviceToHost));
    std::vector<Leaf> v(nl);
    if (nl) IS_CK(cudaMemcpy(v.data(), h->F.leaves + (size_t)sb * SB_MAX_LEAVES, nl * sizeof(Leaf), cudaMemcpyDeviceToHost));
    for (int i = 0; i < nl; i++) {
        if (bsize) bsize[i] = v[i].bsize;
        if (x4) x4[i] = v[i].x4;
        if (y4) y4[i] = v[i].y4;
    }
    return nl;
}

int is_debug_tables(is_handle *h, int qctx, uint16_t *cost, size_t cap, int32_t *avgY, int32_t *avgPart, int32_t *avgSkip0, int qindex,
                    int64_t *lam, int64_t *sq) {
    (void)h;   // host tables: no device needed
    const HostTables &T = host_tables();
    if (cost) memcpy(cost, T.cost[qctx & 3].data(), std::min(cap, (size_t)NCDF) * 2);
    if (avgY) for (int i = 0; i < 13; i++) avgY[i] = T.avgY[i];
    if (avgPart) for (int i = 0; i < 50; i++) avgPart[i] = T.avgPart[i / 10][i % 10];
    if (avgSkip0) *avgSkip0 = T.avgSkip0;
    long long a = 0, b = 0;
    lambda_fx(qindex, 8, &a, &b);
    if (lam) *lam = a;
    if (sq) *sq = b;
    return NCDF;
}

}  // extern "C"

// ---- INT32 issue-rate probe (the roofline denominator of this integer path) ----
// Every thread runs 8 independent chains of x = x * K + (y ^ C) (IMAD + LOP3: 2 INT32 instructions per link), the
// shape of the search's arithmetic (multiply-adds, xors / selects); ops = 2 x 8 x iterations x threads.
namespace {
__global__ void __launch_bounds__(256) k_int32_probe(int iters, uint32_t *sink) {
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = threadIdx.x * (k + 1) + blockIdx.x;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int r = 0; r < 16; r++)
#pragma unroll
            for (int k = 0; k < 8; k++) v[k] = v[k] * 0x01000193u + (v[(k + 1) & 7] ^ 0x5bd1e995u);
    }
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s ^= v[k];
    if (s == 0x12345678u) sink[blockIdx.x] = s;   // keeps the chains alive
}
}  // namespace

extern "C" int is_probe_int32(int device, double *gops, float *ms) {
    if (cudaSetDevice(device) != cudaSuccess) return IS_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return IS_ERR_CUDA;
    uint32_t *sink = nullptr;
    if (cudaMalloc(&sink, 1 << 16) != cudaSuccess) return IS_ERR_OOM;
    const int blocks = prop.multiProcessorCount * 8, iters = 512;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_int32_probe<<<blocks, 256>>>(iters, sink);   // warm-up (clocks, module load)
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(a);
        k_int32_probe<<<blocks, 256>>>(iters, sink);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float t = 0;
        cudaEventElapsedTime(&t, a, b);
        best = t < best ? t : best;
    }
    const cudaError_t e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess) return IS_ERR_CUDA;
    const double ops = 2.0 * 8 * 16 * (double)iters * blocks * 256;
    *gops = ops / (best * 1e-3) / 1e9;
    *ms = best;
    return IS_OK;
}

// ---- closed-loop trace (debug): per queued leaf TRACE_STAMPS values (the phases' globaltimer ns and the queue entry) ----
extern "C" int is_set_trace(is_handle *h, int on) {
    if (!h) return IS_ERR_INVALID;
    h->trace = on != 0;
    return IS_OK;
}
extern "C" int is_get_trace(is_handle *h, unsigned long long *out, size_t cap, uint32_t *n) {
    if (!h || !h->have || !h->F.leafTrace) return IS_ERR_STATE;
    // the leaves of the ready queue image 0 took part in: its own, or those of its format group in a batch
    int tot = 0;
    IS_CK(cudaMemcpy(&tot, h->F.rq + 1, 4, cudaMemcpyDeviceToHost));
    *n = (uint32_t)tot;
    const size_t m = std::min(cap, (size_t)tot * TRACE_STAMPS);
    IS_CK(cudaMemcpy(out, h->F.leafTrace, m * 8, cudaMemcpyDeviceToHost));
    return IS_OK;
}
