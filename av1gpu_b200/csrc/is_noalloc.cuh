// is_noalloc.cuh - is_fwd_quant_static: the forward transform + quantisation + rate kernel (k_test_fwd_quant) run
// with its device buffers in one fixed, module-level scratch instead of per-call device allocations.
//
// For callers that may not allocate device memory: a process whose device memory is owned by a pool or budgeted
// elsewhere (an allocation there can fail or evict), or code that must not reach the allocator's implicit
// synchronisation.  The scratch is a static __device__ array of NOALLOC_SCRATCH_BYTES per device, reserved when the
// module loads; its address is looked up once per device with cudaGetSymbolAddress.  Nothing of it has to start at
// zero: each call copies its residuals in before the launch, and the kernel writes every output word that the call
// reads back.  The first call on a device uploads the search's tables and looks the address up; it must not be made
// while the stream is being captured (it returns IS_ERR_INVALID then), and a failed set-up is retried by the next call.  Calls on one device share the scratch, so they must not overlap: two calls in flight at once on the
// same device (other threads, other streams) race on it and can return each other's results.
#pragma once

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)4 << 20;   // 4 MiB per device (IS_STATIC_SCRATCH_BYTES)
static_assert(NOALLOC_SCRATCH_BYTES == IS_STATIC_SCRATCH_BYTES, "scratch size and its public constant differ");
static __device__ __align__(256) unsigned char g_noallocScratch[NOALLOC_SCRATCH_BYTES];

// per device: the scratch address once its set-up succeeded (a failed set-up is retried by the next call)
std::mutex g_noallocMu;
unsigned char *g_noallocPtr[64];

// the scratch sections of n blocks of tx size W x H (nc kept coefficients): residuals, coefficients, levels, D, R, eob
struct NoallocLayout {
    size_t res, coef, lv, D, R, eob, end;
};
NoallocLayout noalloc_layout(int n, int W, int H, int nc) {
    NoallocLayout l;
    l.res = 0;
    l.coef = l.res + align256((size_t)n * W * H * 4);
    l.lv = l.coef + align256((size_t)n * nc * 4);
    l.D = l.lv + align256((size_t)n * nc * 2);
    l.R = l.D + align256((size_t)n * 8);
    l.eob = l.R + align256((size_t)n * 8);
    l.end = l.eob + align256((size_t)n * 4);
    return l;
}

}  // namespace

extern "C" int is_fwd_quant_static(int device, int n, const int32_t *res, int txSz, int txType, int plane, int qindex, const int32_t ctx[3],
                                   int32_t *coef, int16_t *levels, int64_t *D, int64_t *R, int32_t *eob, void *stream) {
    if (device < 0 || device >= 64 || n < 1 || txSz < 0 || txSz > 18 || txType < 0 || txType > 15 || plane < 0 || plane > 2 ||
        qindex < 1 || qindex > 255 || !res || !ctx || !coef || !levels || !D || !R || !eob)
        return IS_ERR_INVALID;
    // the contexts index the cost tables (txb_skip [13], dc_sign [3], the tx-set CDFs' intra direction [13])
    if (ctx[0] < 0 || ctx[0] >= 13 || ctx[1] < 0 || ctx[1] >= 3 || ctx[2] < 0 || ctx[2] >= 13) return IS_ERR_INVALID;
    // only the types the intra set of the size allows (get_tx_set, reduced_tx_set 0: DCT_DCT alone from 32 a side up)
    {
        const int up = AV1G_T(Tx_Size_Sqr_Up)[txSz];
        const int set = up >= AV1G_TX_32X32 ? AV1G_TX_SET_DCTONLY : AV1G_T(Tx_Size_Sqr)[txSz] == AV1G_TX_16X16 ? AV1G_TX_SET_INTRA_2
                                                                                                            : AV1G_TX_SET_INTRA_1;
        if (!AV1G_T(Tx_Type_In_Set_Intra)[set][txType]) return IS_ERR_INVALID;
    }
    const int W = AV1G_T(Tx_Width)[txSz], H = AV1G_T(Tx_Height)[txSz], nc = std::min(W, 32) * std::min(H, 32);
    if (n > (int)(NOALLOC_SCRATCH_BYTES / 16)) return IS_ERR_TOO_LARGE;   // keeps the layout arithmetic far from overflow
    const NoallocLayout l = noalloc_layout(n, W, H, nc);
    if (l.end > NOALLOC_SCRATCH_BYTES) return IS_ERR_TOO_LARGE;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return IS_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = IS_OK;
    unsigned char *s = nullptr;
    {   // first successful call on the device: the tables of the search and the scratch address (device current).  The
        // table upload cannot run while the stream is being captured: refuse before touching anything then.
        std::lock_guard<std::mutex> lk(g_noallocMu);
        s = g_noallocPtr[device];
        if (!s) {
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
                rc = IS_ERR_INVALID;
            } else {
                void *p = nullptr;
                if (upload_tables(device) || cudaGetSymbolAddress(&p, g_noallocScratch) != cudaSuccess || !p || ((uintptr_t)p & 255)) rc = IS_ERR_CUDA;
                else s = g_noallocPtr[device] = (unsigned char *)p;
            }
        }
    }
    if (rc == IS_OK) {
        int32_t *dres = (int32_t *)(s + l.res), *dcoef = (int32_t *)(s + l.coef), *deob = (int32_t *)(s + l.eob);
        int16_t *dlv = (int16_t *)(s + l.lv);
        long long *dD = (long long *)(s + l.D), *dR = (long long *)(s + l.R);
        cudaError_t e = cudaMemcpyAsync(dres, res, (size_t)n * W * H * 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            k_test_fwd_quant<<<(n + 1) / 2, 64, 2 * sizeof(TestScr), st>>>(n, dres, txSz, txType, plane, AV1G_T(Dc_Qlookup)[0][qindex],
                                                                     AV1G_T(Ac_Qlookup)[0][qindex], av1g_coeff_cdf_q_ctx(qindex), ctx[0],
                                                                     ctx[1], ctx[2], dcoef, dlv, dD, dR, deob);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(coef, dcoef, (size_t)n * nc * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(levels, dlv, (size_t)n * nc * 2, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(D, dD, (size_t)n * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(R, dR, (size_t)n * 8, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(eob, deob, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
        const cudaError_t es = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = es;
        if (e != cudaSuccess) rc = IS_ERR_CUDA;
    }
    cudaSetDevice(prev);
    return rc;
}
