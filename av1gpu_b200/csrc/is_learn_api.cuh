// is_learn_api.cuh - C ABI of the learned shortlist: the learner (weights, Adam state, training buffers; one training
// step = forward, softmax cross-entropy, backward, Adam, all on the device with the kernels of is_learn.cuh), the
// dataset extraction from a finished search, and the network GEMM for the numerics tests.
#pragma once

struct is_learner {
    int device = 0, cap = 0;
    std::string err;
    // fp32 masters, Adam moments, gradients; bf16 copies of the weights
    float *w1 = nullptr, *b1 = nullptr, *w2 = nullptr, *b2 = nullptr;
    float *m = nullptr, *v = nullptr, *g = nullptr;     // [NP] each, parameter order w1 | b1 | w2 | b2
    __nv_bfloat16 *w1b = nullptr, *w2b = nullptr, *w2tb = nullptr;
    // activations and gradients of a batch
    __nv_bfloat16 *Hb = nullptr, *dSb = nullptr, *dHb = nullptr, *Xt = nullptr, *Ht = nullptr, *dSt = nullptr, *dHt = nullptr;
    float *S = nullptr, *loss = nullptr;
    int *correct = nullptr;
    int step = 0;
    int setErr(const char *m_) { err = m_; return IS_ERR_CUDA; }
};

namespace {
constexpr int SL_NW1 = SL_HID * SL_IN, SL_NW2 = SL_OUT * SL_HID, SL_NP = SL_NW1 + SL_HID + SL_NW2 + SL_OUT;

int sl_gemm(int M, int N, int K, const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, float *C, int ldc, const float *bias,
            int relu, __nv_bfloat16 *Cb, int ldcb, cudaStream_t st) {
    if (M <= 0 || N <= 0 || K <= 0 || (K & 7) || (lda & 7) || (ldb & 7)) return IS_ERR_INVALID;
    const dim3 grid((N + GT_N - 1) / GT_N, (M + GT_M - 1) / GT_M);
    k_gemm_abt<<<grid, 128, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, relu, Cb, ldcb);
    return cudaGetLastError() == cudaSuccess ? IS_OK : IS_ERR_CUDA;
}
template <typename T> int sl_transpose(int rows, int cols, const T *in, int ldi, __nv_bfloat16 *out, int ldo, cudaStream_t st) {
    k_transpose_bf16<T><<<dim3((cols + 31) / 32, (rows + 31) / 32), dim3(32, 8), 0, st>>>(rows, cols, in, ldi, out, ldo);
    return cudaGetLastError() == cudaSuccess ? IS_OK : IS_ERR_CUDA;
}
__global__ void k_f2bf(int n, const float *__restrict__ a, __nv_bfloat16 *__restrict__ b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = __float2bfloat16(a[i]);
}
// forward of a batch: H = relu(X W1^T + b1) (bf16), S = H W2^T + b2 (fp32)
int sl_forward(is_learner *L, const __nv_bfloat16 *X, int n, float *S, cudaStream_t st) {
    int rc = sl_gemm(n, SL_HID, SL_IN, X, SL_IN, L->w1b, SL_IN, nullptr, 0, L->b1, 1, L->Hb, SL_HID, st);
    if (!rc) rc = sl_gemm(n, SL_OUT, SL_HID, L->Hb, SL_HID, L->w2b, SL_HID, S, SL_OUT, L->b2, 0, nullptr, 0, st);
    return rc;
}
// gradients of the mean cross-entropy of a batch into L->g (parameter order); loss / correct into L->loss / correct
int sl_backward(is_learner *L, const __nv_bfloat16 *X, const int32_t *y, int n, cudaStream_t st) {
    int rc = sl_forward(L, X, n, L->S, st);
    if (rc) return rc;
    cudaMemsetAsync(L->loss, 0, 4, st);
    cudaMemsetAsync(L->correct, 0, 4, st);
    k_sl_softmax_ce<<<(n + 127) / 128, 128, 0, st>>>(n, L->S, y, L->dSb, L->loss, L->correct);
    float *gw1 = L->g, *gb1 = gw1 + SL_NW1, *gw2 = gb1 + SL_HID, *gb2 = gw2 + SL_NW2;
    // dW2 = dS^T H, db2 = colsum dS
    rc = sl_transpose(n, SL_OUT, L->dSb, SL_OUT, L->dSt, L->cap, st);
    if (!rc) rc = sl_transpose(n, SL_HID, L->Hb, SL_HID, L->Ht, L->cap, st);
    if (!rc) rc = sl_gemm(SL_OUT, SL_HID, n, L->dSt, L->cap, L->Ht, L->cap, gw2, SL_HID, nullptr, 0, nullptr, 0, st);
    k_colsum<<<SL_OUT, 256, 0, st>>>(n, SL_OUT, L->dSb, gb2);
    // dH = dS W2 (masked by H > 0), dW1 = dH^T X, db1 = colsum dH
    if (!rc) rc = sl_transpose(SL_OUT, SL_HID, L->w2b, SL_HID, L->w2tb, SL_OUT, st);
    if (!rc) rc = sl_gemm(n, SL_HID, SL_OUT, L->dSb, SL_OUT, L->w2tb, SL_OUT, nullptr, 0, nullptr, 0, L->dHb, SL_HID, st);
    if (rc) return rc;
    k_relu_grad<<<(unsigned)(((size_t)n * SL_HID + 255) / 256), 256, 0, st>>>((size_t)n * SL_HID, L->Hb, L->dHb);
    rc = sl_transpose(n, SL_HID, L->dHb, SL_HID, L->dHt, L->cap, st);
    if (!rc) rc = sl_transpose(n, SL_IN, X, SL_IN, L->Xt, L->cap, st);
    if (!rc) rc = sl_gemm(SL_HID, SL_IN, n, L->dHt, L->cap, L->Xt, L->cap, gw1, SL_IN, nullptr, 0, nullptr, 0, st);
    k_colsum<<<SL_HID, 256, 0, st>>>(n, SL_HID, L->dHb, gb1);
    return rc ? rc : (cudaGetLastError() == cudaSuccess ? IS_OK : IS_ERR_CUDA);
}
int sl_refresh_bf16(is_learner *L, cudaStream_t st) {
    k_f2bf<<<(SL_NW1 + 255) / 256, 256, 0, st>>>(SL_NW1, L->w1, L->w1b);
    k_f2bf<<<(SL_NW2 + 255) / 256, 256, 0, st>>>(SL_NW2, L->w2, L->w2b);
    return cudaGetLastError() == cudaSuccess ? IS_OK : IS_ERR_CUDA;
}
// dataset labels: the best mode of each listed block (cand[0] of its analysis record)
__global__ void k_sl_labels(const FrameDesc F, const SlBlock *__restrict__ blocks, int n, int32_t *__restrict__ y) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const SlBlock bl = blocks[b];
    const int W = 4 * ST(Num_4x4_Blocks_Wide)[bl.bs], H = 4 * ST(Num_4x4_Blocks_High)[bl.bs];
    const int x = (bl.sb % F.sbCols) * 64 + bl.x4 * 4, y0 = (bl.sb / F.sbCols) * 64 + bl.y4 * 4;
    y[b] = F.blk[F.shOff[bl.bs] + (uint32_t)(y0 / H) * F.shNbx[bl.bs] + x / W].cand[0] >> 3;
}
}  // namespace

// every analysed block of an image, shape by shape in the analysis record order (SB-major inside a shape)
static std::vector<SlBlock> sl_block_list(const FrameDesc &F) {
    std::vector<SlBlock> v;
    const int FW = F.MiCols * 4, FH = F.MiRows * 4;
    for (int s = 0; s < AV1G_BLOCK_INVALID; s++) {
        if (s >= 13 && s <= 15) continue;
        const int w4 = AV1G_T(Num_4x4_Blocks_Wide)[s], h4 = AV1G_T(Num_4x4_Blocks_High)[s];
        for (int by = 0; by < F.shNby[s]; by++)
            for (int bx = 0; bx < F.shNbx[s]; bx++) {
                const int x = bx * w4 * 4, y = by * h4 * 4;
                if (x >= FW || y >= FH) continue;
                SlBlock b;
                b.bs = (uint8_t)s; b.x4 = (uint8_t)((x & 63) >> 2); b.y4 = (uint8_t)((y & 63) >> 2); b.pad = 0;
                b.sb = (uint32_t)((y >> 6) * F.sbCols + (x >> 6));
                v.push_back(b);
            }
    }
    return v;
}

extern "C" {

int is_sl_create(int device, int max_batch, is_learner **out) {
    if (!out || max_batch < 32 || (max_batch & 31)) return IS_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return IS_ERR_CUDA;
    if (upload_tables(device)) return IS_ERR_CUDA;
    is_learner *L = new is_learner();
    L->device = device;
    L->cap = max_batch;
    bool ok = true;
    auto A = [&](void **p, size_t b) { if (ok && cudaMalloc(p, b) != cudaSuccess) ok = false; };
    A((void **)&L->w1, SL_NP * 4);
    L->b1 = L->w1 + SL_NW1; L->w2 = L->b1 + SL_HID; L->b2 = L->w2 + SL_NW2;
    A((void **)&L->m, SL_NP * 4); A((void **)&L->v, SL_NP * 4); A((void **)&L->g, SL_NP * 4);
    A((void **)&L->w1b, SL_NW1 * 2); A((void **)&L->w2b, SL_NW2 * 2); A((void **)&L->w2tb, SL_NW2 * 2);
    const size_t n = (size_t)max_batch;
    A((void **)&L->Hb, n * SL_HID * 2); A((void **)&L->dSb, n * SL_OUT * 2); A((void **)&L->dHb, n * SL_HID * 2);
    A((void **)&L->Xt, n * SL_IN * 2); A((void **)&L->Ht, n * SL_HID * 2); A((void **)&L->dSt, n * SL_OUT * 2);
    A((void **)&L->dHt, n * SL_HID * 2); A((void **)&L->S, n * SL_OUT * 4); A((void **)&L->loss, 4); A((void **)&L->correct, 4);
    if (!ok) { is_sl_destroy(L); return IS_ERR_OOM; }
    *out = L;
    return IS_OK;
}

void is_sl_destroy(is_learner *L) {
    if (!L) return;
    cudaSetDevice(L->device);
    void *ps[] = {L->w1, L->m, L->v, L->g, L->w1b, L->w2b, L->w2tb, L->Hb, L->dSb, L->dHb, L->Xt, L->Ht, L->dSt, L->dHt, L->S, L->loss, L->correct};
    for (void *p : ps)
        if (p) cudaFree(p);
    delete L;
}

int is_sl_set_weights(is_learner *L, const float *w1, const float *b1, const float *w2, const float *b2) {
    if (!L || !w1 || !b1 || !w2 || !b2) return IS_ERR_INVALID;
    cudaSetDevice(L->device);
    if (cudaMemcpy(L->w1, w1, SL_NW1 * 4, cudaMemcpyHostToDevice) || cudaMemcpy(L->b1, b1, SL_HID * 4, cudaMemcpyHostToDevice) ||
        cudaMemcpy(L->w2, w2, SL_NW2 * 4, cudaMemcpyHostToDevice) || cudaMemcpy(L->b2, b2, SL_OUT * 4, cudaMemcpyHostToDevice))
        return IS_ERR_CUDA;
    cudaMemset(L->m, 0, SL_NP * 4);
    cudaMemset(L->v, 0, SL_NP * 4);
    L->step = 0;
    if (sl_refresh_bf16(L, 0)) return IS_ERR_CUDA;
    return cudaDeviceSynchronize() == cudaSuccess ? IS_OK : IS_ERR_CUDA;
}

int is_sl_get_weights(is_learner *L, float *w1, float *b1, float *w2, float *b2) {
    if (!L) return IS_ERR_INVALID;
    cudaSetDevice(L->device);
    if ((w1 && cudaMemcpy(w1, L->w1, SL_NW1 * 4, cudaMemcpyDeviceToHost)) || (b1 && cudaMemcpy(b1, L->b1, SL_HID * 4, cudaMemcpyDeviceToHost)) ||
        (w2 && cudaMemcpy(w2, L->w2, SL_NW2 * 4, cudaMemcpyDeviceToHost)) || (b2 && cudaMemcpy(b2, L->b2, SL_OUT * 4, cudaMemcpyDeviceToHost)))
        return IS_ERR_CUDA;
    return IS_OK;
}

int is_sl_forward(is_learner *L, const void *X, int n, float *S, void *stream) {
    if (!L || !X || !S || n < 1 || n > L->cap) return IS_ERR_INVALID;
    cudaSetDevice(L->device);
    return sl_forward(L, (const __nv_bfloat16 *)X, n, S, (cudaStream_t)stream);
}

// gradients (host, parameter order w1 | b1 | w2 | b2), mean loss and correct count of one batch, weights unchanged
int is_sl_grads(is_learner *L, const void *X, const int32_t *y, int n, float *grads, float *loss, int *correct) {
    if (!L || !X || !y || n < 32 || n > L->cap || (n & 31)) return IS_ERR_INVALID;
    cudaSetDevice(L->device);
    int rc = sl_backward(L, (const __nv_bfloat16 *)X, y, n, 0);
    if (rc) return rc;
    if (cudaDeviceSynchronize() != cudaSuccess) return IS_ERR_CUDA;
    if (grads && cudaMemcpy(grads, L->g, SL_NP * 4, cudaMemcpyDeviceToHost)) return IS_ERR_CUDA;
    float ls = 0;
    int c = 0;
    cudaMemcpy(&ls, L->loss, 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(&c, L->correct, 4, cudaMemcpyDeviceToHost);
    if (loss) *loss = ls / n;
    if (correct) *correct = c;
    return IS_OK;
}

// one Adam step on a batch (n a multiple of 32); returns the batch's mean loss and correct count
int is_sl_train_step(is_learner *L, const void *X, const int32_t *y, int n, float lr, float *loss, int *correct) {
    if (!L || !X || !y || n < 32 || n > L->cap || (n & 31)) return IS_ERR_INVALID;
    cudaSetDevice(L->device);
    int rc = sl_backward(L, (const __nv_bfloat16 *)X, y, n, 0);
    if (rc) return rc;
    L->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)L->step), c2 = 1.f - powf(b2, (float)L->step);
    k_adam<<<(SL_NP + 255) / 256, 256>>>(SL_NP, L->w1, L->g, L->m, L->v, lr, b1, b2, 1e-8f, c1, c2, nullptr);
    if (sl_refresh_bf16(L, 0)) return IS_ERR_CUDA;
    float ls = 0;
    int c = 0;
    if (cudaMemcpy(&ls, L->loss, 4, cudaMemcpyDeviceToHost) || cudaMemcpy(&c, L->correct, 4, cudaMemcpyDeviceToHost)) return IS_ERR_CUDA;
    if (loss) *loss = ls / n;
    if (correct) *correct = c;
    return IS_OK;
}

// C = A B^T on device bf16 operands (the network's GEMM, for the numerics tests)
int is_nn_gemm(int M, int N, int K, const void *A, int lda, const void *B, int ldb, float *C, int ldc, const float *bias, int relu,
               void *stream) {
    if (!A || !B || !C) return IS_ERR_INVALID;
    const int rc = sl_gemm(M, N, K, (const __nv_bfloat16 *)A, lda, (const __nv_bfloat16 *)B, ldb, C, ldc, bias, relu, nullptr, 0,
                           (cudaStream_t)stream);
    if (rc) return rc;
    return cudaStreamSynchronize((cudaStream_t)stream) == cudaSuccess ? IS_OK : IS_ERR_CUDA;
}

// Training data of image i of the last batch: the features (bf16, n x 288) and labels (best analysed mode) of its
// analysed blocks, written to device buffers of capacity cap; n = the number of blocks (returned even when > cap).
int is_sl_dataset(is_handle *h, int i, void *X, int32_t *y, int cap, int *n) {
    if (!h || !h->have || i < 0 || i >= h->bN || !n) return IS_ERR_STATE;
    IS_CK(cudaSetDevice(h->device));
    const FrameDesc &F = h->bF[i];
    const std::vector<SlBlock> bl = sl_block_list(F);
    *n = (int)bl.size();
    if (!X || !y || (int)bl.size() > cap) return IS_OK;
    SlBlock *d = nullptr;
    IS_CK(cudaMalloc(&d, bl.size() * sizeof(SlBlock)));
    cudaError_t e = cudaMemcpy(d, bl.data(), bl.size() * sizeof(SlBlock), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_sl_features<<<(unsigned)((bl.size() + 7) / 8), 256>>>(F, d, (int)bl.size(), (__nv_bfloat16 *)X);
        k_sl_labels<<<(unsigned)((bl.size() + 255) / 256), 256>>>(F, d, (int)bl.size(), y);
        e = cudaDeviceSynchronize();
    }
    cudaFree(d);
    IS_CK(e);
    return IS_OK;
}

}  // extern "C"
