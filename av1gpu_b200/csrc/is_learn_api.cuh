// is_learn_api.cuh - C ABI of the learned shortlist: the learner (master weights, Adam state, training buffers; one
// training step = forward, the two heads' softmax cross-entropy, backward, Adam, all on the device with the kernels of
// is_learn.cuh), the dataset extraction from a finished search, the fused inference of a search's image, and the
// network GEMM for the numerics tests.
#pragma once

struct is_learner {
    int device = 0, cap = 0;
    std::string err;
    float *P = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;   // [SL_NPARAM] each: masters, Adam moments, gradient
    SlNet net{};                                                  // bf16 weights (and the biases in P)
    __nv_bfloat16 *c2t = nullptr, *c3t = nullptr, *f1t = nullptr, *f2t = nullptr;   // transposed bf16 weights
    // activations and gradients of a batch of cap rows
    __nv_bfloat16 *Xc1 = nullptr, *A1 = nullptr, *Xc2 = nullptr, *A2 = nullptr, *Xc3 = nullptr, *A3 = nullptr, *Z = nullptr, *H = nullptr;
    float *S = nullptr;
    __nv_bfloat16 *dS = nullptr, *dH = nullptr, *dA3 = nullptr, *dA2 = nullptr, *dA1 = nullptr;
    float *dZ = nullptr, *dXc3 = nullptr, *dXc2 = nullptr;
    __nv_bfloat16 *TA = nullptr, *TB = nullptr;   // transposes of the weight gradients' operands
    float *parts = nullptr, *gtmp = nullptr;      // split-K partial sums; conv1's padded weight gradient
    float *loss = nullptr;
    int *correct = nullptr;
    int step = 0;
};

namespace {
constexpr int SL_PARTS_MAX = 64;
constexpr size_t SL_PART_FLOATS = (size_t)SL_PARTS_MAX * SL_HID * SL_Z;

bool sl_launch_ok() { return cudaGetLastError() == cudaSuccess; }

int sl_gemm(int M, int N, int K, const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, float *C, int ldc, const float *bias,
            int relu, __nv_bfloat16 *Cb, int ldcb, cudaStream_t st) {
    if (M <= 0 || N <= 0 || K <= 0 || (K & 7) || (lda & 7) || (ldb & 7)) return IS_ERR_INVALID;
    const dim3 grid((N + GT_N - 1) / GT_N, (M + GT_M - 1) / GT_M, 1);
    k_gemm_abt<<<grid, 128, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, relu, Cb, ldcb, K);
    return sl_launch_ok() ? IS_OK : IS_ERR_CUDA;
}
template <typename T> int sl_transpose(int rows, int cols, const T *in, int ldi, __nv_bfloat16 *out, int ldo, cudaStream_t st) {
    k_transpose_bf16<T><<<dim3((rows + 31) / 32, (cols + 31) / 32), dim3(32, 8), 0, st>>>(rows, cols, in, ldi, out, ldo);
    return sl_launch_ok() ? IS_OK : IS_ERR_CUDA;
}
unsigned sl_grid(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

// weight gradient out[M][N] (fp32, row stride N) = dY^T X over P rows: dY [P][M], X [P][N] (bf16, row-major); both
// transposed, then a split-K GEMM and a deterministic sum of the parts
int sl_wgrad(is_learner *L, int M, int N, int P, const __nv_bfloat16 *dY, const __nv_bfloat16 *X, float *out, cudaStream_t st) {
    int rc = sl_transpose(P, M, dY, M, L->TA, P, st);
    if (!rc) rc = sl_transpose(P, N, X, N, L->TB, P, st);
    if (rc) return rc;
    const int parts = std::max(1, std::min(SL_PARTS_MAX, P / 8192));
    const int chunk = ((P + parts - 1) / parts + GT_K - 1) / GT_K * GT_K;
    const int z = (P + chunk - 1) / chunk;
    if (z == 1) {
        k_gemm_abt<<<dim3((N + GT_N - 1) / GT_N, (M + GT_M - 1) / GT_M, 1), 128, 0, st>>>(M, N, P, L->TA, P, L->TB, P, out, N, nullptr, 0,
                                                                                          nullptr, 0, P);
        return sl_launch_ok() ? IS_OK : IS_ERR_CUDA;
    }
    k_gemm_abt<<<dim3((N + GT_N - 1) / GT_N, (M + GT_M - 1) / GT_M, z), 128, 0, st>>>(M, N, P, L->TA, P, L->TB, P, L->parts, N, nullptr, 0,
                                                                                      nullptr, 0, chunk);
    k_sum_parts<<<(M * N + 255) / 256, 256, 0, st>>>(M * N, z, L->parts, out);
    return sl_launch_ok() ? IS_OK : IS_ERR_CUDA;
}

// bf16 copies of the masters (and the transposed ones of the backward pass)
int sl_refresh(is_learner *L, cudaStream_t st) {
    k_sl_weights<<<(SL_HID * SL_Z + 255) / 256, 256, 0, st>>>(L->P, L->net);
    int rc = sl_launch_ok() ? IS_OK : IS_ERR_CUDA;
    if (!rc) rc = sl_transpose(SL_C2, SL_K2, L->net.c2, SL_K2, L->c2t, SL_C2, st);
    if (!rc) rc = sl_transpose(SL_C3, SL_K3, L->net.c3, SL_K3, L->c3t, SL_C3, st);
    if (!rc) rc = sl_transpose(SL_HID, SL_Z, L->net.f1, SL_Z, L->f1t, SL_HID, st);
    if (!rc) rc = sl_transpose(SL_OUT, SL_HID, L->net.f2, SL_HID, L->f2t, SL_OUT, st);
    return rc;
}

// forward of n feature rows X [n][SL_FEAT]: scores S [n][SL_OUT] (fp32); activations kept for the backward pass
int sl_forward(is_learner *L, const __nv_bfloat16 *X, int n, float *S, cudaStream_t st) {
    const SlNet &N = L->net;
    k_im2col<<<sl_grid((size_t)n * 256 * SL_K1P), 256, 0, st>>>(n, 32, 32, 1, X, SL_FEAT, SL_K1P, L->Xc1);
    int rc = sl_launch_ok() ? IS_OK : IS_ERR_CUDA;
    if (!rc) rc = sl_gemm(n * 256, SL_C1, SL_K1P, L->Xc1, SL_K1P, N.c1, SL_K1P, nullptr, 0, N.b1, 1, L->A1, SL_C1, st);
    if (rc) return rc;
    k_im2col<<<sl_grid((size_t)n * 64 * SL_K2), 256, 0, st>>>(n, 16, 16, SL_C1, L->A1, 256 * SL_C1, SL_K2, L->Xc2);
    rc = sl_launch_ok() ? IS_OK : IS_ERR_CUDA;
    if (!rc) rc = sl_gemm(n * 64, SL_C2, SL_K2, L->Xc2, SL_K2, N.c2, SL_K2, nullptr, 0, N.b2, 1, L->A2, SL_C2, st);
    if (rc) return rc;
    k_im2col<<<sl_grid((size_t)n * 16 * SL_K3), 256, 0, st>>>(n, 8, 8, SL_C2, L->A2, 64 * SL_C2, SL_K3, L->Xc3);
    rc = sl_launch_ok() ? IS_OK : IS_ERR_CUDA;
    if (!rc) rc = sl_gemm(n * 16, SL_C3, SL_K3, L->Xc3, SL_K3, N.c3, SL_K3, nullptr, 0, N.b3, 1, L->A3, SL_C3, st);
    if (rc) return rc;
    k_sl_zrows<<<sl_grid((size_t)n * SL_Z), 256, 0, st>>>(n, L->A3, X, L->Z);
    rc = sl_launch_ok() ? IS_OK : IS_ERR_CUDA;
    if (!rc) rc = sl_gemm(n, SL_HID, SL_Z, L->Z, SL_Z, N.f1, SL_Z, nullptr, 0, N.bf1, 1, L->H, SL_HID, st);
    if (!rc) rc = sl_gemm(n, SL_OUT, SL_HID, L->H, SL_HID, N.f2, SL_HID, S, SL_OUT, N.bf2, 0, nullptr, 0, st);
    return rc;
}

// gradients of the mean loss of a batch into L->g (parameter order); loss sum / correct count into L->loss / correct
int sl_backward(is_learner *L, const __nv_bfloat16 *X, const int32_t *y, int n, cudaStream_t st) {
    int rc = sl_forward(L, X, n, L->S, st);
    if (rc) return rc;
    cudaMemsetAsync(L->loss, 0, 4, st);
    cudaMemsetAsync(L->correct, 0, 4, st);
    k_sl_softmax_ce<<<(n + 127) / 128, 128, 0, st>>>(n, L->S, y, L->dS, L->loss, L->correct);
    float *g = L->g;
    // fc2: dW = dS^T H, db = colsum dS; dH = dS W (where H > 0)
    rc = sl_wgrad(L, SL_OUT, SL_HID, n, L->dS, L->H, g + SLP_F2W, st);
    k_colsum<<<SL_OUT, 256, 0, st>>>(n, SL_OUT, L->dS, g + SLP_F2B);
    if (!rc) rc = sl_gemm(n, SL_HID, SL_OUT, L->dS, SL_OUT, L->f2t, SL_OUT, nullptr, 0, nullptr, 0, L->dH, SL_HID, st);
    if (rc) return rc;
    k_relu_grad<<<(unsigned)(((size_t)n * SL_HID + 255) / 256), 256, 0, st>>>((size_t)n * SL_HID, L->H, L->dH);
    // fc1: dW = dH^T Z, db = colsum dH; dZ = dH W; conv3's output gradient = dZ[:, :256] where A3 > 0
    rc = sl_wgrad(L, SL_HID, SL_Z, n, L->dH, L->Z, g + SLP_F1W, st);
    k_colsum<<<SL_HID, 256, 0, st>>>(n, SL_HID, L->dH, g + SLP_F1B);
    if (!rc) rc = sl_gemm(n, SL_Z, SL_HID, L->dH, SL_HID, L->f1t, SL_HID, L->dZ, SL_Z, nullptr, 0, nullptr, 0, st);
    if (rc) return rc;
    k_sl_dz<<<sl_grid((size_t)n * 256), 256, 0, st>>>(n, L->dZ, L->A3, L->dA3);
    // conv3: dW = dA3^T Xc3; dXc3 = dA3 W3 -> conv2's output gradient (col2im, where A2 > 0)
    rc = sl_wgrad(L, SL_C3, SL_K3, n * 16, L->dA3, L->Xc3, g + SLP_C3W, st);
    k_colsum<<<SL_C3, 256, 0, st>>>(n * 16, SL_C3, L->dA3, g + SLP_C3B);
    if (!rc) rc = sl_gemm(n * 16, SL_K3, SL_C3, L->dA3, SL_C3, L->c3t, SL_C3, L->dXc3, SL_K3, nullptr, 0, nullptr, 0, st);
    if (rc) return rc;
    k_col2im_relu<<<sl_grid((size_t)n * 64 * SL_C2), 256, 0, st>>>(n, 8, 8, SL_C2, L->dXc3, SL_K3, L->A2, L->dA2);
    // conv2: dW = dA2^T Xc2; dXc2 = dA2 W2 -> conv1's output gradient
    rc = sl_wgrad(L, SL_C2, SL_K2, n * 64, L->dA2, L->Xc2, g + SLP_C2W, st);
    k_colsum<<<SL_C2, 256, 0, st>>>(n * 64, SL_C2, L->dA2, g + SLP_C2B);
    if (!rc) rc = sl_gemm(n * 64, SL_K2, SL_C2, L->dA2, SL_C2, L->c2t, SL_C2, L->dXc2, SL_K2, nullptr, 0, nullptr, 0, st);
    if (rc) return rc;
    k_col2im_relu<<<sl_grid((size_t)n * 256 * SL_C1), 256, 0, st>>>(n, 16, 16, SL_C1, L->dXc2, SL_K2, L->A1, L->dA1);
    // conv1: dW = dA1^T Xc1 (taps 0..8 of the padded 16)
    rc = sl_wgrad(L, SL_C1, SL_K1P, n * 256, L->dA1, L->Xc1, L->gtmp, st);
    k_colsum<<<SL_C1, 256, 0, st>>>(n * 256, SL_C1, L->dA1, g + SLP_C1B);
    if (rc) return rc;
    if (cudaMemcpy2DAsync(g + SLP_C1W, SL_K1 * 4, L->gtmp, SL_K1P * 4, SL_K1 * 4, SL_C1, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return IS_ERR_CUDA;
    return sl_launch_ok() ? IS_OK : IS_ERR_CUDA;
}

}  // namespace

extern "C" {

int is_sl_create(int device, int max_batch, is_learner **out) {
    if (!out || max_batch < 32 || (max_batch & 31) || max_batch > (1 << 16)) return IS_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return IS_ERR_CUDA;
    if (upload_tables(device)) return IS_ERR_CUDA;
    is_learner *L = new is_learner();
    L->device = device;
    L->cap = max_batch;
    bool ok = true;
    auto A = [&](void **p, size_t b) { if (ok && cudaMalloc(p, b) != cudaSuccess) { ok = false; *p = nullptr; } };
    A((void **)&L->P, SL_NPARAM * 4); A((void **)&L->m, SL_NPARAM * 4); A((void **)&L->v, SL_NPARAM * 4); A((void **)&L->g, SL_NPARAM * 4);
    A((void **)&L->net.c1, SL_C1 * SL_K1P * 2); A((void **)&L->net.c2, SL_C2 * SL_K2 * 2); A((void **)&L->net.c3, SL_C3 * SL_K3 * 2);
    A((void **)&L->net.f1, SL_HID * SL_Z * 2); A((void **)&L->net.f2, SL_OUT * SL_HID * 2);
    A((void **)&L->c2t, SL_C2 * SL_K2 * 2); A((void **)&L->c3t, SL_C3 * SL_K3 * 2); A((void **)&L->f1t, SL_HID * SL_Z * 2);
    A((void **)&L->f2t, SL_OUT * SL_HID * 2);
    const size_t n = (size_t)max_batch;
    A((void **)&L->Xc1, n * 256 * SL_K1P * 2); A((void **)&L->A1, n * 256 * SL_C1 * 2); A((void **)&L->Xc2, n * 64 * SL_K2 * 2);
    A((void **)&L->A2, n * 64 * SL_C2 * 2); A((void **)&L->Xc3, n * 16 * SL_K3 * 2); A((void **)&L->A3, n * 16 * SL_C3 * 2);
    A((void **)&L->Z, n * SL_Z * 2); A((void **)&L->H, n * SL_HID * 2); A((void **)&L->S, n * SL_OUT * 4);
    A((void **)&L->dS, n * SL_OUT * 2); A((void **)&L->dH, n * SL_HID * 2); A((void **)&L->dZ, n * SL_Z * 4);
    A((void **)&L->dA3, n * 256 * 2); A((void **)&L->dXc3, n * 16 * SL_K3 * 4); A((void **)&L->dA2, n * 64 * SL_C2 * 2);
    A((void **)&L->dXc2, n * 64 * SL_K2 * 4); A((void **)&L->dA1, n * 256 * SL_C1 * 2);
    A((void **)&L->TA, n * 256 * SL_C1 * 2);   // the largest dY^T: 8 x 256 n (conv1) = 16 x 64 n (conv2) > 160 n
    A((void **)&L->TB, n * 64 * SL_K2 * 2);    // the largest X^T: 72 x 64 n (conv2) > 16 x 256 n (conv1)
    A((void **)&L->parts, SL_PART_FLOATS * 4); A((void **)&L->gtmp, SL_C1 * SL_K1P * 4);
    A((void **)&L->loss, 4); A((void **)&L->correct, 4);
    L->net.b1 = L->P + SLP_C1B; L->net.b2 = L->P + SLP_C2B; L->net.b3 = L->P + SLP_C3B; L->net.bf1 = L->P + SLP_F1B; L->net.bf2 = L->P + SLP_F2B;
    if (!ok) { is_sl_destroy(L); return IS_ERR_OOM; }
    *out = L;
    return IS_OK;
}

void is_sl_destroy(is_learner *L) {
    if (!L) return;
    cudaSetDevice(L->device);
    void *ps[] = {L->P, L->m, L->v, L->g, L->net.c1, L->net.c2, L->net.c3, L->net.f1, L->net.f2, L->c2t, L->c3t, L->f1t, L->f2t,
                  L->Xc1, L->A1, L->Xc2, L->A2, L->Xc3, L->A3, L->Z, L->H, L->S, L->dS, L->dH, L->dZ, L->dA3, L->dXc3, L->dA2,
                  L->dXc2, L->dA1, L->TA, L->TB, L->parts, L->gtmp, L->loss, L->correct};
    for (void *p : ps)
        if (p) cudaFree(p);
    delete L;
}

int is_sl_set_params(is_learner *L, const float *params) {
    if (!L || !params) return IS_ERR_INVALID;
    cudaSetDevice(L->device);
    if (cudaMemcpy(L->P, params, SL_NPARAM * 4, cudaMemcpyHostToDevice) != cudaSuccess) return IS_ERR_CUDA;
    cudaMemset(L->m, 0, SL_NPARAM * 4);
    cudaMemset(L->v, 0, SL_NPARAM * 4);
    L->step = 0;
    if (sl_refresh(L, 0)) return IS_ERR_CUDA;
    return cudaDeviceSynchronize() == cudaSuccess ? IS_OK : IS_ERR_CUDA;
}

int is_sl_get_params(is_learner *L, float *params) {
    if (!L || !params) return IS_ERR_INVALID;
    cudaSetDevice(L->device);
    return cudaMemcpy(params, L->P, SL_NPARAM * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? IS_OK : IS_ERR_CUDA;
}

int is_sl_forward(is_learner *L, const void *X, int n, float *S, void *stream) {
    if (!L || !X || !S || n < 1 || n > L->cap) return IS_ERR_INVALID;
    cudaSetDevice(L->device);
    return sl_forward(L, (const __nv_bfloat16 *)X, n, S, (cudaStream_t)stream);
}

// gradients (host, parameter order), mean loss and correct count of one batch, weights unchanged
int is_sl_grads(is_learner *L, const void *X, const int32_t *y, int n, float *grads, float *loss, int *correct) {
    if (!L || !X || !y || n < 32 || n > L->cap || (n & 31)) return IS_ERR_INVALID;
    cudaSetDevice(L->device);
    int rc = sl_backward(L, (const __nv_bfloat16 *)X, y, n, 0);
    if (rc) return rc;
    if (cudaDeviceSynchronize() != cudaSuccess) return IS_ERR_CUDA;
    if (grads && cudaMemcpy(grads, L->g, SL_NPARAM * 4, cudaMemcpyDeviceToHost)) return IS_ERR_CUDA;
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
    k_adam<<<(SL_NPARAM + 255) / 256, 256>>>(SL_NPARAM, L->P, L->g, L->m, L->v, lr, b1, b2, 1e-8f, c1, c2);
    if (sl_refresh(L, 0)) return IS_ERR_CUDA;
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

// Training rows of image i of the last batch: features (bf16, n x IS_SL_FEAT) and labels (n x 3 int32) of its scored
// records in compact order (records outside the frame: class -1), into device buffers of capacity cap; n = the number
// of records (also when it exceeds cap: then nothing is written).
int is_sl_dataset(is_handle *h, int i, void *X, int32_t *y, int cap, int *n) {
    if (!h || !h->have || i < 0 || i >= h->bN || !n) return IS_ERR_STATE;
    IS_CK(cudaSetDevice(h->device));
    FrameDesc F = h->bF[i];
    uint32_t ns = sl_scored_layout(F, F.slIdx);
    *n = (int)ns;
    if (!X || !y || (int)ns > cap) return IS_OK;
    for (uint32_t i0 = 0; i0 < ns; i0 += 1u << 20) {
        const int cn = (int)std::min<uint32_t>(1u << 20, ns - i0);
        k_sl_dataset<<<(cn + 7) / 8, 256>>>(F, i0, cn, (__nv_bfloat16 *)X + (size_t)i0 * SL_FEAT, y + (size_t)i0 * 3);
    }
    IS_CK(cudaGetLastError());
    IS_CK(cudaDeviceSynchronize());
    return IS_OK;
}

// The search's inference kernels on image i of the last batch with the learner's weights: scores (device fp32, n x
// SL_OUT) of its scored records in compact order (rows of records outside the frame: whatever the GEMMs make of zero
// rows).
int is_sl_infer(is_handle *h, is_learner *L, int i, float *S, int cap, int *n) {
    if (!h || !L || !h->have || i < 0 || i >= h->bN || !n) return IS_ERR_STATE;
    IS_CK(cudaSetDevice(h->device));
    FrameDesc F = h->bF[i];
    const uint32_t ns = sl_scored_layout(F, F.slIdx);
    *n = (int)ns;
    if (!S || (int)ns > cap) return IS_OK;
    __nv_bfloat16 *Z = nullptr, *Hb = nullptr;
    float *Sc = nullptr;
    cudaError_t e = cudaMalloc(&Z, (size_t)SL_CHUNK * SL_Z * 2);
    if (e == cudaSuccess) e = cudaMalloc(&Hb, (size_t)SL_CHUNK * SL_HID * 2);
    if (e == cudaSuccess) e = cudaMalloc(&Sc, (size_t)SL_CHUNK * SL_OUT * 4);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_sl_conv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SlcSmem));
    if (e == cudaSuccess) e = sl_infer_image(F, L->net, SlSel{1.f, 0.f, 1.f, 8, 7}, h->nSm, Z, Hb, Sc, nullptr, S, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(Z);
    cudaFree(Hb);
    cudaFree(Sc);
    IS_CK(e);
    return IS_OK;
}

}  // extern "C"
