// is_learn.cuh - the learned mode shortlist: BF16 tensor-core kernels for its network's training and inference.
//
// Network (per analysed block): 288 features (a 16x16 luma patch resampled from the block, an 8-bin gradient
// orientation histogram, the block shape one-hot) -> 128 ReLU -> 16 scores (13 intra modes + 3 unused).  Every
// layer is a GEMM C = A B^T with A [M x K] and B [N x K] both K-contiguous BF16, FP32 accumulation on the tensor cores
// (mma.sync m16n8k16 bf16), K a multiple of 16.  Training keeps FP32 master weights (Adam) and BF16 copies.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace is {

constexpr int SL_IN = 288, SL_HID = 128, SL_OUT = 16, SL_MODES = 13;
constexpr uint32_t SL_CHUNK = 65536;   // analysis records scored per inference pass of the search

// ---- C[M x N] (fp32, row stride ldc) = A[M x K] . B[N x K]^T (+ bias[N]) (ReLU if relu); optional bf16 copy ----
// CTA tile 64 x 64, 4 warps each 32 x 32 (2 x 4 mma tiles of 16 x 8), K step 32 staged in shared memory.
constexpr int GT_M = 64, GT_N = 64, GT_K = 32;
__device__ __forceinline__ uint32_t pack_bf16x2(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

__global__ void __launch_bounds__(128) k_gemm_abt(int M, int N, int K, const __nv_bfloat16 *__restrict__ A, int lda,
                                                  const __nv_bfloat16 *__restrict__ B, int ldb, float *__restrict__ C, int ldc,
                                                  const float *__restrict__ bias, int relu, __nv_bfloat16 *__restrict__ Cb, int ldcb) {
    __shared__ __align__(16) __nv_bfloat16 sA[GT_M][GT_K + 8];
    __shared__ __align__(16) __nv_bfloat16 sB[GT_N][GT_K + 8];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * GT_M, n0 = blockIdx.x * GT_N;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) acc[i][j][r] = 0.f;
    const int g = lane >> 2, tq = lane & 3;
    for (int k0 = 0; k0 < K; k0 += GT_K) {
        // stage A and B tiles (zero outside the matrices), 8 bf16 per thread-load
        for (int e = tid; e < GT_M * GT_K / 8; e += 128) {
            const int r = e / (GT_K / 8), c = (e % (GT_K / 8)) * 8;
            const int gm = m0 + r, gk = k0 + c;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gm < M && gk + 8 <= K) v = *reinterpret_cast<const uint4 *>(A + (size_t)gm * lda + gk);
            *reinterpret_cast<uint4 *>(&sA[r][c]) = v;
        }
        for (int e = tid; e < GT_N * GT_K / 8; e += 128) {
            const int r = e / (GT_K / 8), c = (e % (GT_K / 8)) * 8;
            const int gn = n0 + r, gk = k0 + c;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gn < N && gk + 8 <= K) v = *reinterpret_cast<const uint4 *>(B + (size_t)gn * ldb + gk);
            *reinterpret_cast<uint4 *>(&sB[r][c]) = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GT_K; kk += 16) {
            uint32_t a[2][4], b[4][2];
#pragma unroll
            for (int i = 0; i < 2; i++) {   // A fragment (16 x 16, row): rows g / g+8, columns 2tq.. / 2tq+8..
                const int r = wm + i * 16 + g;
                a[i][0] = pack_bf16x2(&sA[r][kk + 2 * tq]);
                a[i][1] = pack_bf16x2(&sA[r + 8][kk + 2 * tq]);
                a[i][2] = pack_bf16x2(&sA[r][kk + 2 * tq + 8]);
                a[i][3] = pack_bf16x2(&sA[r + 8][kk + 2 * tq + 8]);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {   // B fragment (16 x 8, col): column g of the tile, rows 2tq.. / 2tq+8..
                const int c = wn + j * 8 + g;
                b[j][0] = pack_bf16x2(&sB[c][kk + 2 * tq]);
                b[j][1] = pack_bf16x2(&sB[c][kk + 2 * tq + 8]);
            }
#pragma unroll
            for (int i = 0; i < 2; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
                    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                                 "{%0,%1,%2,%3};"
                                 : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
                                 : "r"(a[i][0]), "r"(a[i][1]), "r"(a[i][2]), "r"(a[i][3]), "r"(b[j][0]), "r"(b[j][1]));
        }
        __syncthreads();
    }
    // epilogue: accumulator (i, j, r): row wm + 16i + g (+8 for r >= 2), column wn + 8j + 2tq + (r & 1)
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) {
                const int row = m0 + wm + i * 16 + g + (r >= 2 ? 8 : 0), col = n0 + wn + j * 8 + 2 * tq + (r & 1);
                if (row >= M || col >= N) continue;
                float v = acc[i][j][r] + (bias ? bias[col] : 0.f);
                if (relu) v = fmaxf(v, 0.f);
                if (C) C[(size_t)row * ldc + col] = v;
                if (Cb) Cb[(size_t)row * ldcb + col] = __float2bfloat16(v);
            }
}

// transpose + convert: out[c][r] = bf16(in[r][c]) (in rows x cols fp32 or bf16)
template <typename T>
__global__ void k_transpose_bf16(int rows, int cols, const T *__restrict__ in, int ldi, __nv_bfloat16 *__restrict__ out, int ldo) {
    __shared__ float t[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        t[k][threadIdx.x] = (r < rows && c < cols) ? (float)in[(size_t)r * ldi + c] : 0.f;
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (c < cols && r < rows) out[(size_t)c * ldo + r] = __float2bfloat16(t[threadIdx.x][k]);
    }
}

}  // namespace is

namespace is {

// ---- per-block features: 16 x 16 luma patch (box average of the block resampled to 16 x 16, minus the block mean,
// / 64), 8-bin gradient orientation histogram (orientation mod 180 degrees, |gx| + |gy| weighted, sum-normalised),
// the shape one-hot (22), qindex / 255, 1 ----
struct SlBlock { uint8_t bs, x4, y4, pad; uint32_t sb; };   // block of shape bs at SB sb, 4x4-unit offset (x4, y4)

// the features of a block of shape bs at (x, y) into out[288], by one warp; 10-bit samples count a quarter (the
// features stay on the 8-bit scale the network is trained on)
__device__ __forceinline__ void sl_features_of(const FrameDesc &F, int bs, int x, int y, __nv_bfloat16 *out) {
    const int lane = threadIdx.x & 31;
    const int W = 4 * ST(Num_4x4_Blocks_Wide)[bs], H = 4 * ST(Num_4x4_Blocks_High)[bs];
    const bool hi = F.bd > 8;
    const uint8_t *src8 = F.src[0];
    const uint16_t *src16 = reinterpret_cast<const uint16_t *>(F.src[0]);
    auto src = [&](size_t i) -> int { return hi ? (int)src16[i] : (int)src8[i]; };
    const float scale = hi ? 0.25f : 1.f;
    const int sp = F.spitch[0];
    // the patch: lane handles 8 of the 256 cells
    float cell[8], sum = 0.f;
    const int sw = max(W / 16, 1), sh = max(H / 16, 1);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int c = lane * 8 + k, ci = c >> 4, cj = c & 15;
        const int px = x + (cj * W) / 16, py = y + (ci * H) / 16;
        int s = 0;
        for (int i = 0; i < sh; i++)
            for (int j = 0; j < sw; j++) s += src((size_t)(py + i) * sp + px + j);
        cell[k] = (float)s / (float)(sw * sh) * scale;
        sum += cell[k];
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    const float mean = sum / 256.f;
#pragma unroll
    for (int k = 0; k < 8; k++) out[lane * 8 + k] = __float2bfloat16((cell[k] - mean) / 64.f);
    // orientation histogram over the same 16 x 16 grid (central differences on the source)
    float hist[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int c = lane * 8 + k, ci = c >> 4, cj = c & 15;
        const int px = x + (cj * W) / 16, py = y + (ci * H) / 16;
        // central differences clamped to the block (samples of the padded source plane only)
        const int xl = max(px - 1, x), xr = min(px + 1, x + W - 1), yu = max(py - 1, y), yd = min(py + 1, y + H - 1);
        const float gx = ((float)src((size_t)py * sp + xr) - (float)src((size_t)py * sp + xl)) * scale;
        const float gy = ((float)src((size_t)yd * sp + px) - (float)src((size_t)yu * sp + px)) * scale;
        const float m = fabsf(gx) + fabsf(gy);
        // orientation in [0, 180): fold to gy >= 0, then 8 bins of 22.5 degrees by comparisons with tan(22.5/67.5)
        float ax = gx, ay = gy;
        if (ay < 0.f || (ay == 0.f && ax < 0.f)) { ax = -ax; ay = -ay; }
        int bin;
        if (ax >= 0.f) bin = ay <= 0.41421356f * ax ? 0 : ay <= ax ? 1 : ay <= 2.41421356f * ax ? 2 : 3;
        else bin = ay >= -2.41421356f * ax ? 4 : ay >= -ax ? 5 : ay >= -0.41421356f * ax ? 6 : 7;
#pragma unroll
        for (int q = 0; q < 8; q++) hist[q] += q == bin ? m : 0.f;
    }
    float tot = 0.f;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        for (int o = 16; o > 0; o >>= 1) hist[q] += __shfl_xor_sync(0xffffffffu, hist[q], o);
        tot += hist[q];
    }
    if (lane < 8) {
        float hv = 0.f;
#pragma unroll
        for (int q = 0; q < 8; q++) hv = q == lane ? hist[q] : hv;
        out[256 + lane] = __float2bfloat16(hv / (tot + 1.f));
    }
    if (lane < 22) out[264 + lane] = __float2bfloat16(lane == bs ? 1.f : 0.f);
    if (lane == 22) out[286] = __float2bfloat16((float)F.qidx / 255.f);
    if (lane == 23) out[287] = __float2bfloat16(1.f);
}

// features of a list of blocks (training data), one warp per block
__global__ void k_sl_features(const FrameDesc F, const SlBlock *__restrict__ blocks, int n, __nv_bfloat16 *__restrict__ X) {
    const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (b >= n) return;
    const SlBlock bl = blocks[b];
    sl_features_of(F, bl.bs, (bl.sb % F.sbCols) * 64 + bl.x4 * 4, (bl.sb / F.sbCols) * 64 + bl.y4 * 4, X + (size_t)b * SL_IN);
}

// the analysis record (shape, position) of record index i; false when i is out of range or the block lies outside the
// frame
__device__ __forceinline__ bool sl_record_block(const FrameDesc &F, uint32_t i, int &bs, int &x, int &y) {
    bs = -1;
#pragma unroll 1
    for (int s = 0; s < 22; s++) {
        if (s >= 13 && s <= 15) continue;
        const uint32_t n = (uint32_t)F.shNbx[s] * (uint32_t)F.shNby[s];
        if (i >= F.shOff[s] && i < F.shOff[s] + n) { bs = s; break; }
    }
    if (bs < 0) return false;
    const uint32_t k = i - F.shOff[bs];
    x = (int)(k % (uint32_t)F.shNbx[bs]) * 4 * ST(Num_4x4_Blocks_Wide)[bs];
    y = (int)(k / (uint32_t)F.shNbx[bs]) * 4 * ST(Num_4x4_Blocks_High)[bs];
    return x < F.MiCols * 4 && y < F.MiRows * 4;
}

// features of the analysis records [i0, i0 + n) (zero rows for blocks outside the frame), one warp per record
__global__ void k_sl_features_rec(const FrameDesc F, uint32_t i0, int n, __nv_bfloat16 *__restrict__ X) {
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= n) return;
    int bs, x, y;
    __nv_bfloat16 *out = X + (size_t)r * SL_IN;
    if (sl_record_block(F, i0 + r, bs, x, y)) {
        sl_features_of(F, bs, x, y, out);
    } else {
        for (int k = lane; k < SL_IN; k += 32) out[k] = __float2bfloat16(0.f);
    }
}

// ---- softmax cross-entropy over the first SL_MODES of SL_OUT scores: loss sum (atomic) and dS = (p - onehot) / n
// (bf16, padded columns 0) ----
__global__ void k_sl_softmax_ce(int n, const float *__restrict__ S, const int *__restrict__ y, __nv_bfloat16 *__restrict__ dS,
                                float *__restrict__ loss, int *__restrict__ correct) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const float *s = S + (size_t)r * SL_OUT;
    float mx = s[0];
    int am = 0;
    for (int k = 1; k < SL_MODES; k++) if (s[k] > mx) { mx = s[k]; am = k; }
    float z = 0.f;
    for (int k = 0; k < SL_MODES; k++) z += __expf(s[k] - mx);
    const int t = y[r];
    atomicAdd(loss, -(s[t] - mx - __logf(z)));
    if (am == t) atomicAdd(correct, 1);
    for (int k = 0; k < SL_OUT; k++) {
        const float p = k < SL_MODES ? __expf(s[k] - mx) / z : 0.f;
        dS[(size_t)r * SL_OUT + k] = __float2bfloat16((p - (k == t ? 1.f : 0.f)) / (float)n);
    }
}

// dH (bf16, in place) *= (H > 0)
__global__ void k_relu_grad(size_t n, const __nv_bfloat16 *__restrict__ H, __nv_bfloat16 *__restrict__ dH) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !((float)H[i] > 0.f)) dH[i] = __float2bfloat16(0.f);
}

// column sums of a bf16 matrix (rows x cols) -> out[cols] (fp32)
__global__ void k_colsum(int rows, int cols, const __nv_bfloat16 *__restrict__ G, float *__restrict__ out) {
    const int c = blockIdx.x;
    float s = 0.f;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) s += (float)G[(size_t)r * cols + c];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float w[32];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += w[k];
        out[c] = t;
    }
}

// Adam step on fp32 master weights p with gradient g; refreshes the bf16 copy pb (may be null)
__global__ void k_adam(int n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v, float lr,
                       float b1, float b2, float eps, float c1, float c2, __nv_bfloat16 *__restrict__ pb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    m[i] = b1 * m[i] + (1.f - b1) * gi;
    v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
    p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
    if (pb) pb[i] = __float2bfloat16(p[i]);
}

// ---- shortlist mask of each block from its scores: the smallest set of modes (by probability) whose probabilities
// add up to tau, at most maxModes; all 13 modes when the most likely one is below conf (the fallback) ----
__global__ void k_sl_mask(int n, const float *__restrict__ S, float tau, int maxModes, float conf, uint16_t *__restrict__ mask) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    if (maxModes <= 0) { mask[r] = 0x1FFF; return; }
    const float *s = S + (size_t)r * SL_OUT;
    float p[SL_MODES], mx = s[0], z = 0.f;
    for (int k = 1; k < SL_MODES; k++) mx = fmaxf(mx, s[k]);
    for (int k = 0; k < SL_MODES; k++) { p[k] = __expf(s[k] - mx); z += p[k]; }
    uint32_t m = 0;
    float acc = 0.f, top = 0.f;
    for (int t = 0; t < maxModes && acc < tau; t++) {
        int b = -1;
        for (int k = 0; k < SL_MODES; k++)
            if (!((m >> k) & 1) && (b < 0 || p[k] > p[b])) b = k;
        if (t == 0) top = p[b] / z;
        m |= 1u << b;
        acc += p[b] / z;
    }
    mask[r] = (uint16_t)(top < conf ? 0x1FFF : m);
}

}  // namespace is
