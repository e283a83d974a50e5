// is_learn.cuh - the learned shortlist: BF16 tensor-core kernels for its network's training and inference.
//
// Network (per analysed block of the 16 shapes of 8x8 .. 64x64 with at least 64 samples: all but 4x4, 4x8, 8x4):
//   input   a 32 x 32 luma patch resampled from the block and a margin of an eighth of its size (at least one sample)
//           above and left (box averages, mean removed, / 64), and 32 extras: an 8-bin gradient-orientation histogram of
//           the patch, the shape one-hot (16), qindex / 255, 1
//   conv1   3x3 stride 2, 1 -> 8 channels, ReLU (16 x 16)
//   conv2   3x3 stride 2, 8 -> 16, ReLU (8 x 8)
//   conv3   3x3 stride 2, 16 -> 16, ReLU (4 x 4)
//   fc1     256 conv features + the 32 extras -> 160, ReLU
//   fc2     160 -> 80 scores: [0, 61) the (mode, angle delta) candidates (5 non-directional modes, 8 directional modes x
//           7 deltas), [64, 80) the 16 tx types; together they score the 61 x 16 (mode, delta, tx type) triples of a
//           block as the product of the two softmaxes
// 62,688 parameters.  Every layer is a GEMM C = A B^T with A [M x K] and B [N x K] both K-contiguous BF16 and FP32
// accumulation on the tensor cores (mma.sync m16n8k16), K a multiple of 16 (a convolution as an implicit GEMM over its
// 3x3 taps: k = tap * Cin + channel).  Training keeps FP32 master weights (Adam) and BF16 copies; the search runs the
// inference kernels k_sl_conv (source plane to each block's fc1 input), the fc GEMMs and k_sl_select.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace is {

constexpr int SL_PATCH = 32, SL_NPIX = SL_PATCH * SL_PATCH, SL_NEXTRA = 32, SL_FEAT = SL_NPIX + SL_NEXTRA;
constexpr int SL_C1 = 8, SL_C2 = 16, SL_C3 = 16;       // output channels of the three convolutions
constexpr int SL_K1 = 9, SL_K1P = 16, SL_K2 = 72, SL_K3 = 144;   // their GEMM K (conv1 padded to 16)
constexpr int SL_Z = 16 * SL_C3 + SL_NEXTRA;           // fc1 input: 288
constexpr int SL_HID = 160, SL_OUT = 80, SL_MD = 61, SL_TX0 = 64;
constexpr int SL_NSHAPE = 16;
// parameter offsets in the flat fp32 array (conv weights [Cout][9 Cin], fc weights [out][in], then the bias)
constexpr int SLP_C1W = 0, SLP_C1B = SLP_C1W + SL_C1 * SL_K1, SLP_C2W = SLP_C1B + SL_C1, SLP_C2B = SLP_C2W + SL_C2 * SL_K2,
              SLP_C3W = SLP_C2B + SL_C2, SLP_C3B = SLP_C3W + SL_C3 * SL_K3, SLP_F1W = SLP_C3B + SL_C3,
              SLP_F1B = SLP_F1W + SL_HID * SL_Z, SLP_F2W = SLP_F1B + SL_HID, SLP_F2B = SLP_F2W + SL_OUT * SL_HID,
              SL_NPARAM = SLP_F2B + SL_OUT;
static_assert(SL_NPARAM == 62688, "parameter count");

// the shapes the network scores, and each one's class (-1: not scored): 8x8 8x16 16x8 16x16 16x32 32x16 32x32 32x64
// 64x32 64x64 4x16 16x4 8x32 32x8 16x64 64x16
__host__ __device__ __forceinline__ int sl_shape_class(int bs) {
    return (bs >= 3 && bs <= 12) ? bs - 3 : (bs >= 16 && bs <= 21) ? bs - 6 : -1;
}
// (mode, delta) candidate code (mode << 3 | delta + 3) of class k of the first head, and back
__host__ __device__ __forceinline__ int sl_class_cand(int k) {
    if (k < 5) return (k == 0 ? 0 : 8 + k) << 3 | 3;   // DC, SMOOTH, SMOOTH_V, SMOOTH_H, PAETH
    const int m = 1 + (k - 5) / 7, d = (k - 5) % 7;      // V .. D67, delta -3 .. 3
    return m << 3 | d;
}
__host__ __device__ __forceinline__ int sl_cand_class(int c) {
    const int m = c >> 3, d = c & 7;
    if (m == 0) return 0;
    if (m >= 9) return m - 8;
    return 5 + (m - 1) * 7 + d;
}

// the selection rule: candidates by probability until tau is covered (at most maxCand), tx types likewise
struct SlSel {
    float tau, conf, txTau;
    int maxCand, maxTx;
};

// ---- C[M x N] (fp32, row stride ldc) = A[M x K] . B[N x K]^T (+ bias[N]) (ReLU if relu); optional bf16 copy ----
// CTA tile 64 x 64, 4 warps each 32 x 32 (2 x 4 mma tiles of 16 x 8), K step 32 staged in shared memory.  Split K:
// CTA z takes k in [z kChunk, (z + 1) kChunk) and writes its partial sums to C + z M ldc (no bias, no ReLU, no copy).
constexpr int GT_M = 64, GT_N = 64, GT_K = 32;
__device__ __forceinline__ uint32_t pack_bf16x2(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__global__ void __launch_bounds__(128) k_gemm_abt(int M, int N, int K, const __nv_bfloat16 *__restrict__ A, int lda,
                                                  const __nv_bfloat16 *__restrict__ B, int ldb, float *__restrict__ C, int ldc,
                                                  const float *__restrict__ bias, int relu, __nv_bfloat16 *__restrict__ Cb, int ldcb,
                                                  int kChunk) {
    __shared__ __align__(16) __nv_bfloat16 sA[GT_M][GT_K + 8];
    __shared__ __align__(16) __nv_bfloat16 sB[GT_N][GT_K + 8];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * GT_M, n0 = blockIdx.x * GT_N;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int kBeg = blockIdx.z * kChunk, kEnd = min(K, kBeg + kChunk);
    const bool split = gridDim.z > 1;
    if (split) C += (size_t)blockIdx.z * M * ldc;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int r = 0; r < 4; r++) acc[i][j][r] = 0.f;
    const int g = lane >> 2, tq = lane & 3;
    for (int k0 = kBeg; k0 < kEnd; k0 += GT_K) {
        // stage A and B tiles (zero outside the matrices and the K range), 8 bf16 per thread-load
        for (int e = tid; e < GT_M * GT_K / 8; e += 128) {
            const int r = e / (GT_K / 8), c = (e % (GT_K / 8)) * 8;
            const int gm = m0 + r, gk = k0 + c;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gm < M && gk + 8 <= kEnd) v = *reinterpret_cast<const uint4 *>(A + (size_t)gm * lda + gk);
            *reinterpret_cast<uint4 *>(&sA[r][c]) = v;
        }
        for (int e = tid; e < GT_N * GT_K / 8; e += 128) {
            const int r = e / (GT_K / 8), c = (e % (GT_K / 8)) * 8;
            const int gn = n0 + r, gk = k0 + c;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gn < N && gk + 8 <= kEnd) v = *reinterpret_cast<const uint4 *>(B + (size_t)gn * ldb + gk);
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
                for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], a[i], b[j][0], b[j][1]);
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
                if (split) { C[(size_t)row * ldc + col] = acc[i][j][r]; continue; }
                float v = acc[i][j][r] + (bias ? bias[col] : 0.f);
                if (relu) v = fmaxf(v, 0.f);
                if (C) C[(size_t)row * ldc + col] = v;
                if (Cb) Cb[(size_t)row * ldcb + col] = __float2bfloat16(v);
            }
}

// out[i] = sum over z of part[z][i] (the split-K partial sums, in z order: deterministic)
__global__ void k_sum_parts(int n, int parts, const float *__restrict__ part, float *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.f;
    for (int z = 0; z < parts; z++) s += part[(size_t)z * n + i];
    out[i] = s;
}

// transpose + convert: out[c][r] = bf16(in[r][c]) (in rows x cols fp32 or bf16)
// (grid: x over the row tiles, which may be millions, y over the column tiles)
template <typename T>
__global__ void k_transpose_bf16(int rows, int cols, const T *__restrict__ in, int ldi, __nv_bfloat16 *__restrict__ out, int ldo) {
    __shared__ float t[32][33];
    const int c0 = blockIdx.y * 32, r0 = blockIdx.x * 32;
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

// ---- the patch and extras of a block, by one warp ----
// Cell (i, j) of the 32 x 32 patch is the box average of source rows [y0 + i RH / 32, y0 + (i + 1) RH / 32) and
// columns likewise (one sample when the range is empty: upsampling), over the region of RW x RH = (W + mx) x (H + my)
// samples at (x0, y0) = (x - mx, y - my), the margins mx = ceil(W / 8), my = ceil(H / 8); coordinates clamped to the
// frame's first row / column (the padded plane covers the right and bottom).  10-bit samples count a quarter (the
// 8-bit scale the network is trained on).  Lane j computes column j; v[i] = cell (i, j).  The shape is a template
// parameter: every source row of the region is read once (a lane reads its column span, at most ceil(RW / 32)
// samples) and added to the cells whose row span holds it, the spans fixed at compile time.
template <int W, int H>
__device__ __forceinline__ void sl_cells_t(const FrameDesc &F, int x, int y, float (&v)[32]) {
    constexpr int mx = (W + 7) / 8, my = (H + 7) / 8, RW = W + mx, RH = H + my, CMAX = (RW + 31) / 32;
    const int lane = threadIdx.x & 31;
    const int x0 = x - mx, y0 = y - my;
    const bool hi = F.bd > 8;
    const uint8_t *s8 = F.src[0];
    const uint16_t *s16 = reinterpret_cast<const uint16_t *>(F.src[0]);
    const int sp = F.spitch[0];
    const int cx0 = x0 + (lane * RW) / 32, nc = max(x0 + ((lane + 1) * RW) / 32 - cx0, 1);
    int acc[32];
#pragma unroll
    for (int i = 0; i < 32; i++) acc[i] = 0;
#pragma unroll
    for (int r = 0; r < RH; r++) {
        const size_t row = (size_t)max(y0 + r, 0) * sp;
        int rs = 0;
#pragma unroll
        for (int b = 0; b < CMAX; b++)
            if (b < nc) rs += hi ? (int)s16[row + max(cx0 + b, 0)] : (int)s8[row + max(cx0 + b, 0)];
#pragma unroll
        for (int i = 0; i < 32; i++) {
            const int r0 = (i * RH) / 32, r1 = max(((i + 1) * RH) / 32, r0 + 1);
            if (r >= r0 && r < r1) acc[i] += rs;
        }
    }
    const float inv = hi ? 0.25f : 1.f;
#pragma unroll
    for (int i = 0; i < 32; i++) {
        const int r0 = (i * RH) / 32, nr = max(((i + 1) * RH) / 32, r0 + 1) - r0;
        v[i] = (float)acc[i] / (float)(nr * nc) * inv;
    }
}
__device__ __forceinline__ void sl_cells(const FrameDesc &F, int bs, int x, int y, float (&v)[32]) {
    switch (bs) {
    case AV1G_BLOCK_8X8: sl_cells_t<8, 8>(F, x, y, v); break;
    case AV1G_BLOCK_8X16: sl_cells_t<8, 16>(F, x, y, v); break;
    case AV1G_BLOCK_16X8: sl_cells_t<16, 8>(F, x, y, v); break;
    case AV1G_BLOCK_16X16: sl_cells_t<16, 16>(F, x, y, v); break;
    case AV1G_BLOCK_16X32: sl_cells_t<16, 32>(F, x, y, v); break;
    case AV1G_BLOCK_32X16: sl_cells_t<32, 16>(F, x, y, v); break;
    case AV1G_BLOCK_32X32: sl_cells_t<32, 32>(F, x, y, v); break;
    case AV1G_BLOCK_32X64: sl_cells_t<32, 64>(F, x, y, v); break;
    case AV1G_BLOCK_64X32: sl_cells_t<64, 32>(F, x, y, v); break;
    case AV1G_BLOCK_64X64: sl_cells_t<64, 64>(F, x, y, v); break;
    case AV1G_BLOCK_4X16: sl_cells_t<4, 16>(F, x, y, v); break;
    case AV1G_BLOCK_16X4: sl_cells_t<16, 4>(F, x, y, v); break;
    case AV1G_BLOCK_8X32: sl_cells_t<8, 32>(F, x, y, v); break;
    case AV1G_BLOCK_32X8: sl_cells_t<32, 8>(F, x, y, v); break;
    case AV1G_BLOCK_16X64: sl_cells_t<16, 64>(F, x, y, v); break;
    default: sl_cells_t<64, 16>(F, x, y, v); break;   // AV1G_BLOCK_64X16
    }
}
// From the cells: the normalised patch value of cell (i, lane) -> patch(i, lane) and the 32 extras -> extra(k)
// (lanes write their own entries).  Histogram: central differences on the cell grid (clamped at its border),
// orientation mod 180 degrees in 8 bins of 22.5 degrees, |gx| + |gy| weighted, divided by (sum + 1).
template <typename PatchFn, typename ExtraFn>
__device__ __forceinline__ void sl_features(const FrameDesc &F, int bs, const float (&v)[32], float *hs, PatchFn patch, ExtraFn extra) {
    const int lane = threadIdx.x & 31;
    float sum = 0.f;
#pragma unroll
    for (int i = 0; i < 32; i++) sum += v[i];
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    const float mean = sum / 1024.f;
#pragma unroll
    for (int i = 0; i < 32; i++) patch(i, lane, __float2bfloat16((v[i] - mean) / 64.f));
    float *hr = hs + lane * 9;   // the lane's 8 bins in shared memory (row stride 9: distinct banks)
#pragma unroll
    for (int q = 0; q < 8; q++) hr[q] = 0.f;
#pragma unroll
    for (int i = 0; i < 32; i++) {
        const float l = __shfl_sync(0xffffffffu, v[i], max(lane - 1, 0)), r = __shfl_sync(0xffffffffu, v[i], min(lane + 1, 31));
        const float gx = r - l, gy = v[i < 31 ? i + 1 : 31] - v[i > 0 ? i - 1 : 0];
        const float m = fabsf(gx) + fabsf(gy);
        float ax = gx, ay = gy;
        if (ay < 0.f || (ay == 0.f && ax < 0.f)) { ax = -ax; ay = -ay; }
        int bin;
        if (ax >= 0.f) bin = ay <= 0.41421356f * ax ? 0 : ay <= ax ? 1 : ay <= 2.41421356f * ax ? 2 : 3;
        else bin = ay >= -2.41421356f * ax ? 4 : ay >= -ax ? 5 : ay >= -0.41421356f * ax ? 6 : 7;
        hr[bin] += m;
    }
    float hist[8];
#pragma unroll
    for (int q = 0; q < 8; q++) hist[q] = hr[q];
    float tot = 0.f;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        for (int o = 16; o > 0; o >>= 1) hist[q] += __shfl_xor_sync(0xffffffffu, hist[q], o);
        tot += hist[q];
    }
    float hv = 0.f;
#pragma unroll
    for (int q = 0; q < 8; q++) hv = q == lane ? hist[q] : hv;
    const int cls = sl_shape_class(bs);
    float e = 0.f;
    if (lane < 8) e = hv / (tot + 1.f);
    else if (lane < 8 + SL_NSHAPE) e = lane - 8 == cls ? 1.f : 0.f;
    else if (lane == 8 + SL_NSHAPE) e = (float)F.qidx / 255.f;
    else if (lane == 9 + SL_NSHAPE) e = 1.f;
    extra(lane, __float2bfloat16(e));
}

// the compact layout of an image's scored records: first compact index of each scored shape (-1 for the others), and
// their count
static inline uint32_t sl_scored_layout(const FrameDesc &F, int *slIdx) {
    uint32_t n = 0;
    for (int s = 0; s < 22; s++) {
        slIdx[s] = -1;
        if (sl_shape_class(s) < 0) continue;
        slIdx[s] = (int)n;
        n += (uint32_t)F.shNbx[s] * (uint32_t)F.shNby[s];
    }
    return n;
}

// compact index of the scored records (shape by shape in scoring order, records in the analysis order): shape and
// record of compact index i; false when i is out of range
__device__ __forceinline__ bool sl_scored_record(const FrameDesc &F, uint32_t i, int &bs, uint32_t &rec) {
#pragma unroll 1
    for (int s = 0; s < 22; s++) {
        if (F.slIdx[s] < 0) continue;
        const uint32_t n = (uint32_t)F.shNbx[s] * (uint32_t)F.shNby[s];
        if (i >= (uint32_t)F.slIdx[s] && i < (uint32_t)F.slIdx[s] + n) { bs = s; rec = i - (uint32_t)F.slIdx[s]; return true; }
    }
    return false;
}
__device__ __forceinline__ void sl_record_xy(const FrameDesc &F, int bs, uint32_t rec, int &x, int &y) {
    x = (int)(rec % (uint32_t)F.shNbx[bs]) * 4 * ST(Num_4x4_Blocks_Wide)[bs];
    y = (int)(rec / (uint32_t)F.shNbx[bs]) * 4 * ST(Num_4x4_Blocks_High)[bs];
}

// training rows of the scored records [i0, i0 + n) of an image: features X [n][SL_FEAT] and labels y [n][3] = (class of
// the analysis' best (mode, delta), its tx type or -1 when the set is DCT_DCT alone, the set's types as a bit mask);
// records outside the frame get zero features and class -1.  One warp per record.
__global__ void k_sl_dataset(const FrameDesc F, uint32_t i0, int n, __nv_bfloat16 *__restrict__ X, int32_t *__restrict__ y) {
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= n) return;
    int bs;
    uint32_t rec;
    __nv_bfloat16 *out = X + (size_t)r * SL_FEAT;
    int x = 0, yy = 0;
    const bool ok = sl_scored_record(F, i0 + r, bs, rec) && (sl_record_xy(F, bs, rec, x, yy), x < F.MiCols * 4 && yy < F.MiRows * 4);
    if (!ok) {
        for (int k = lane; k < SL_FEAT; k += 32) out[k] = __float2bfloat16(0.f);
        if (lane == 0) { y[3 * r] = -1; y[3 * r + 1] = -1; y[3 * r + 2] = 0; }
        return;
    }
    __shared__ float hs[8][32 * 9];   // (256 threads: 8 warps)
    float v[32];
    sl_cells(F, bs, x, yy, v);
    sl_features(F, bs, v, hs[(threadIdx.x >> 5) & 7], [&](int i, int j, __nv_bfloat16 b) { out[i * SL_PATCH + j] = b; },
                [&](int k, __nv_bfloat16 b) { out[SL_NPIX + k] = b; });
    if (lane == 0) {
        const BlockRes br = F.blk[F.shOff[bs] + rec];
        const int txSz = ST(Max_Tx_Size_Rect)[bs], set = tx_set_intra(txSz);
        uint32_t valid = 0;
        for (int t = 0; t < 16; t++) valid |= tx_in_set(set, t) ? 1u << t : 0u;
        y[3 * r] = sl_cand_class(br.cand[0]);
        y[3 * r + 1] = set == AV1G_TX_SET_DCTONLY ? -1 : (int)br.tx;
        y[3 * r + 2] = set == AV1G_TX_SET_DCTONLY ? 0 : (int)valid;
    }
}

// ---- convolution as an implicit GEMM: im2col / col2im of a 3x3 stride-2 pad-1 convolution ----
// in: per sample IH x IW x C (channel fastest) at in + s * sstride; out rows (s, oy, ox), columns k = tap * C + c for
// k < 9 C, zero up to Kp
__global__ void k_im2col(int n, int IH, int IW, int C, const __nv_bfloat16 *__restrict__ in, int sstride, int Kp,
                         __nv_bfloat16 *__restrict__ out) {
    const int OH = IH / 2, OW = IW / 2;
    const size_t total = (size_t)n * OH * OW * Kp;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(e % Kp);
        const size_t row = e / Kp;
        const int p = (int)(row % (OH * OW)), s = (int)(row / (OH * OW));
        __nv_bfloat16 v = __float2bfloat16(0.f);
        if (k < 9 * C) {
            const int tap = k / C, c = k % C, iy = 2 * (p / OW) + tap / 3 - 1, ix = 2 * (p % OW) + tap % 3 - 1;
            if (iy >= 0 && ix >= 0 && iy < IH && ix < IW) v = in[(size_t)s * sstride + ((size_t)iy * IW + ix) * C + c];
        }
        out[e] = v;
    }
}
// gradient of the input activations: dA[s][iy][ix][c] = (sum over the taps that read it of dcol) where act > 0, bf16
__global__ void k_col2im_relu(int n, int IH, int IW, int C, const float *__restrict__ dcol, int Kp, const __nv_bfloat16 *__restrict__ act,
                              __nv_bfloat16 *__restrict__ dA) {
    const int OH = IH / 2, OW = IW / 2;
    const size_t total = (size_t)n * IH * IW * C;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e % C);
        const size_t q = e / C;
        const int pix = (int)(q % (IH * IW)), s = (int)(q / (IH * IW)), iy = pix / IW, ix = pix % IW;
        float sum = 0.f;
#pragma unroll
        for (int ky = 0; ky < 3; ky++) {
            const int ty = iy + 1 - ky;
            if (ty < 0 || (ty & 1) || ty / 2 >= OH) continue;
#pragma unroll
            for (int kx = 0; kx < 3; kx++) {
                const int tx = ix + 1 - kx;
                if (tx < 0 || (tx & 1) || tx / 2 >= OW) continue;
                sum += dcol[((size_t)s * OH * OW + (ty / 2) * OW + tx / 2) * Kp + (ky * 3 + kx) * C + c];
            }
        }
        dA[e] = __float2bfloat16((float)act[e] > 0.f ? sum : 0.f);
    }
}
// fc1 input rows: Z[s] = conv3 output (16 positions x 16 channels) then the sample's 32 extras
__global__ void k_sl_zrows(int n, const __nv_bfloat16 *__restrict__ A3, const __nv_bfloat16 *__restrict__ X, __nv_bfloat16 *__restrict__ Z) {
    const size_t total = (size_t)n * SL_Z;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(e % SL_Z);
        const size_t s = e / SL_Z;
        Z[e] = k < 256 ? A3[s * 256 + k] : X[s * SL_FEAT + SL_NPIX + (k - 256)];
    }
}
// conv3 output gradient from fc1's input gradient: dA3 = dZ[:, :256] where A3 > 0, bf16
__global__ void k_sl_dz(int n, const float *__restrict__ dZ, const __nv_bfloat16 *__restrict__ A3, __nv_bfloat16 *__restrict__ dA3) {
    const size_t total = (size_t)n * 256;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t s = e / 256;
        const int k = (int)(e % 256);
        dA3[e] = __float2bfloat16((float)A3[e] > 0.f ? dZ[s * SL_Z + k] : 0.f);
    }
}

// ---- loss: softmax cross-entropy of the (mode, delta) head plus that of the tx head over the block's set (rows whose
// tx label is -1 have no tx term); dS = gradient of the mean loss (bf16; unused columns 0), loss sum and the count of
// rows whose most probable (mode, delta) is the label ----
__global__ void k_sl_softmax_ce(int n, const float *__restrict__ S, const int *__restrict__ y, __nv_bfloat16 *__restrict__ dS,
                                float *__restrict__ loss, int *__restrict__ correct) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const float *s = S + (size_t)r * SL_OUT;
    const int t = y[3 * r], tt = y[3 * r + 1];
    const uint32_t valid = (uint32_t)y[3 * r + 2];
    float mx = s[0];
    int am = 0;
    for (int k = 1; k < SL_MD; k++) if (s[k] > mx) { mx = s[k]; am = k; }
    float z = 0.f;
    for (int k = 0; k < SL_MD; k++) z += __expf(s[k] - mx);
    float l = -(s[t] - mx - __logf(z));
    float tmx = -1e30f, tz = 0.f;
    if (tt >= 0) {
        for (int k = 0; k < 16; k++) if ((valid >> k) & 1) tmx = fmaxf(tmx, s[SL_TX0 + k]);
        for (int k = 0; k < 16; k++) if ((valid >> k) & 1) tz += __expf(s[SL_TX0 + k] - tmx);
        l += -(s[SL_TX0 + tt] - tmx - __logf(tz));
    }
    atomicAdd(loss, l);
    if (am == t) atomicAdd(correct, 1);
    const float inv = 1.f / (float)n;
    for (int k = 0; k < SL_OUT; k++) {
        float g = 0.f;
        if (k < SL_MD) g = (__expf(s[k] - mx) / z - (k == t ? 1.f : 0.f)) * inv;
        else if (k >= SL_TX0 && tt >= 0 && ((valid >> (k - SL_TX0)) & 1))
            g = (__expf(s[k] - tmx) / tz - (k - SL_TX0 == tt ? 1.f : 0.f)) * inv;
        dS[(size_t)r * SL_OUT + k] = __float2bfloat16(g);
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

// Adam step on fp32 master weights p with gradient g
__global__ void k_adam(int n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    m[i] = b1 * m[i] + (1.f - b1) * gi;
    v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
    p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

// ---- BF16 copies of the weights for the GEMMs (row-major [out][K], conv1's K padded to 16) and the fused kernel ----
struct SlNet {
    __nv_bfloat16 *c1, *c2, *c3, *f1, *f2;   // [8][16], [16][72], [16][144], [160][288], [80][160]
    const float *b1, *b2, *b3, *bf1, *bf2;   // biases (fp32, in the master array)
};
__global__ void k_sl_weights(const float *__restrict__ P, SlNet net) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < SL_C1 * SL_K1P) {
        const int o = i / SL_K1P, k = i % SL_K1P;
        net.c1[i] = __float2bfloat16(k < SL_K1 ? P[SLP_C1W + o * SL_K1 + k] : 0.f);
    }
    if (i < SL_C2 * SL_K2) net.c2[i] = __float2bfloat16(P[SLP_C2W + i]);
    if (i < SL_C3 * SL_K3) net.c3[i] = __float2bfloat16(P[SLP_C3W + i]);
    if (i < SL_HID * SL_Z) net.f1[i] = __float2bfloat16(P[SLP_F1W + i]);
    if (i < SL_OUT * SL_HID) net.f2[i] = __float2bfloat16(P[SLP_F2W + i]);
}

// ---- inference in the search: the convolutions per block (k_sl_conv), fc1 / fc2 as GEMMs over a chunk of blocks
// (k_gemm_abt), then each block's shortlist (k_sl_select) ----
// k_sl_conv: SLC_WARPS warps per CTA, two CTAs per SM; the CTA stages the BF16 conv weights in shared memory (rows
// padded so that the fragment loads of a warp hit 32 distinct banks); each warp takes scored records one at a time:
// the patch and extras, then conv1..3 as implicit GEMMs on mma.sync over its shared-memory activations, and writes the
// record's fc1 input row Z (conv3's 256 outputs, position-major, then the 32 extras; zeros for a record outside the
// frame).
constexpr int SLC_WARPS = 8;
constexpr int SLI_W1S = 24, SLI_W2S = 88, SLI_W3S = 152, SLI_PS = 40;
constexpr uint32_t SL_CHUNK = 65536;   // scored records per inference chunk (the Z / H / S buffers of a front stream)
struct SlcWarp {
    __nv_bfloat16 patch[SL_PATCH * SLI_PS];   // 32 x 32 (+ pad)
    __nv_bfloat16 act1[256 * SL_C1];          // 16 x 16 x 8
    __nv_bfloat16 act2[64 * SL_C2];           // 8 x 8 x 16
    float hist[32 * 9];                       // the lanes' orientation-histogram bins
};
struct SlcSmem {
    __nv_bfloat16 w1[SL_C1 * SLI_W1S], w2[SL_C2 * SLI_W2S], w3[SL_C3 * SLI_W3S];
    float b1[SL_C1], b2[SL_C2], b3[SL_C3];
    SlcWarp w[SLC_WARPS];
};
static_assert(2 * sizeof(SlcSmem) <= 227 * 1024, "k_sl_conv: two CTAs per SM");

__global__ void __launch_bounds__(SLC_WARPS * 32, 2) k_sl_conv(const __grid_constant__ FrameDesc F, SlNet net, uint32_t i0, int n,
                                                                __nv_bfloat16 *__restrict__ Z) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SlcSmem &S = *reinterpret_cast<SlcSmem *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, tq = lane & 3;
    if (F.poison) {
        smem_poison(smem_raw, sizeof(SlcSmem), tid, SLC_WARPS * 32);
        __syncthreads();
    }
    for (int i = tid; i < SL_C1 * SLI_W1S; i += blockDim.x) {
        const int r = i / SLI_W1S, c = i % SLI_W1S;
        S.w1[i] = c < SL_K1P ? net.c1[r * SL_K1P + c] : __float2bfloat16(0.f);
    }
    for (int i = tid; i < SL_C2 * SLI_W2S; i += blockDim.x) {   // K 72 -> 80 zero-padded (and the row pad)
        const int r = i / SLI_W2S, c = i % SLI_W2S;
        S.w2[i] = c < SL_K2 ? net.c2[r * SL_K2 + c] : __float2bfloat16(0.f);
    }
    for (int i = tid; i < SL_C3 * SLI_W3S; i += blockDim.x) {
        const int r = i / SLI_W3S, c = i % SLI_W3S;
        S.w3[i] = c < SL_K3 ? net.c3[r * SL_K3 + c] : __float2bfloat16(0.f);
    }
    if (tid < SL_C1) S.b1[tid] = net.b1[tid];
    if (tid < SL_C2) S.b2[tid] = net.b2[tid];
    if (tid < SL_C3) S.b3[tid] = net.b3[tid];
    __syncthreads();
    SlcWarp &Wp = S.w[warp];
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    // conv1's A fragment: lane (g, tq) holds taps k = 2tq, 2tq + 1, 2tq + 8, 2tq + 9 of output columns ox = g and g + 8
    // of output row mt; the patch offsets of those taps relative to input row 2 mt, and whether they exist (k < 9, the
    // column inside the patch; the row is outside only for mt = 0 and ky = 0)
    int kOff[4][2];
    bool kOk[4][2], kTop[4];
#pragma unroll
    for (int a = 0; a < 4; a++) {
        const int k = 2 * tq + (a & 1) + (a >> 1) * 8, ky = k / 3, kx = k % 3;
        kTop[a] = ky == 0;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int ix = 2 * (g + 8 * h) + kx - 1;
            kOk[a][h] = k < SL_K1 && ix >= 0 && ix < SL_PATCH;
            kOff[a][h] = (ky - 1) * SLI_PS + ix;
        }
    }
    const uint32_t bw0 = pack_bf16x2(&S.w1[g * SLI_W1S + 2 * tq]), bw1 = pack_bf16x2(&S.w1[g * SLI_W1S + 2 * tq + 8]);
    for (int r = blockIdx.x * SLC_WARPS + warp; r < n; r += gridDim.x * SLC_WARPS) {
        __nv_bfloat16 *zr = Z + (size_t)r * SL_Z;
        int bs = -1, x = 0, y = 0;
        uint32_t rec;
        bool ok = sl_scored_record(F, i0 + r, bs, rec);
        if (ok) {
            sl_record_xy(F, bs, rec, x, y);
            ok = x < F.MiCols * 4 && y < F.MiRows * 4;
        }
        if (!ok) {
            for (int k = lane; k < SL_Z / 2; k += 32) reinterpret_cast<uint32_t *>(zr)[k] = 0u;
            continue;
        }
        {
            float v[32];
            sl_cells(F, bs, x, y, v);
            sl_features(F, bs, v, Wp.hist, [&](int i, int j, __nv_bfloat16 val) { Wp.patch[i * SLI_PS + j] = val; },
                        [&](int k, __nv_bfloat16 val) { zr[256 + k] = val; });
        }
        __syncwarp();
        // conv1: M = 256 output positions (tile mt = output row mt), N = 8, K = 16 (taps 0..8, the rest zero)
        {
            const float bi0 = S.b1[2 * tq], bi1 = S.b1[2 * tq + 1];
#pragma unroll 4
            for (int mt = 0; mt < 16; mt++) {
                const __nv_bfloat16 *base = Wp.patch + 2 * mt * SLI_PS;
                __nv_bfloat16 e[4][2];
#pragma unroll
                for (int a = 0; a < 4; a++)
#pragma unroll
                    for (int h = 0; h < 2; h++) e[a][h] = (kOk[a][h] && !(mt == 0 && kTop[a])) ? base[kOff[a][h]] : zero;
                uint32_t A[4];
                {
                    __nv_bfloat162 t;
                    t.x = e[0][0]; t.y = e[1][0]; A[0] = *reinterpret_cast<uint32_t *>(&t);
                    t.x = e[0][1]; t.y = e[1][1]; A[1] = *reinterpret_cast<uint32_t *>(&t);
                    t.x = e[2][0]; t.y = e[3][0]; A[2] = *reinterpret_cast<uint32_t *>(&t);
                    t.x = e[2][1]; t.y = e[3][1]; A[3] = *reinterpret_cast<uint32_t *>(&t);
                }
                float d[4] = {0.f, 0.f, 0.f, 0.f};
                mma_bf16(d, A, bw0, bw1);
                const int p0 = mt * 16 + g, p1 = p0 + 8;
                __nv_bfloat162 o0, o1;
                o0.x = __float2bfloat16(fmaxf(d[0] + bi0, 0.f));
                o0.y = __float2bfloat16(fmaxf(d[1] + bi1, 0.f));
                o1.x = __float2bfloat16(fmaxf(d[2] + bi0, 0.f));
                o1.y = __float2bfloat16(fmaxf(d[3] + bi1, 0.f));
                *reinterpret_cast<__nv_bfloat162 *>(&Wp.act1[p0 * SL_C1 + 2 * tq]) = o0;
                *reinterpret_cast<__nv_bfloat162 *>(&Wp.act1[p1 * SL_C1 + 2 * tq]) = o1;
            }
        }
        __syncwarp();
        // conv2: M = 64 (tile mt = output rows 2 mt, 2 mt + 1), N = 16 (2 tiles), K = 80 (72 + zero), k = tap * 8 + c: the
        // fragment's k and k + 8 are taps 2 ks and 2 ks + 1 at channel 2 tq
        {
#pragma unroll 1
            for (int mt = 0; mt < 4; mt++) {
                float d[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
                for (int ks = 0; ks < 5; ks++) {
                    uint32_t A[4];
#pragma unroll
                    for (int a = 0; a < 4; a++) {   // (row g / g + 8) x (tap 2 ks / 2 ks + 1)
                        const int tap = 2 * ks + (a >> 1), oy = 2 * mt + (a & 1), ox = g;
                        const int iy = 2 * oy + tap / 3 - 1, ix = 2 * ox + tap % 3 - 1;
                        A[a] = (tap < 9 && iy >= 0 && ix >= 0 && ix < 16) ? pack_bf16x2(&Wp.act1[(iy * 16 + ix) * SL_C1 + 2 * tq]) : 0u;
                    }
#pragma unroll
                    for (int nt = 0; nt < 2; nt++) {
                        const __nv_bfloat16 *wr = &S.w2[(nt * 8 + g) * SLI_W2S + ks * 16 + 2 * tq];
                        mma_bf16(d[nt], A, pack_bf16x2(wr), pack_bf16x2(wr + 8));
                    }
                }
                const int p0 = mt * 16 + g, p1 = p0 + 8;
#pragma unroll
                for (int nt = 0; nt < 2; nt++) {
                    const int c = nt * 8 + 2 * tq;
                    __nv_bfloat162 o0, o1;
                    o0.x = __float2bfloat16(fmaxf(d[nt][0] + S.b2[c], 0.f));
                    o0.y = __float2bfloat16(fmaxf(d[nt][1] + S.b2[c + 1], 0.f));
                    o1.x = __float2bfloat16(fmaxf(d[nt][2] + S.b2[c], 0.f));
                    o1.y = __float2bfloat16(fmaxf(d[nt][3] + S.b2[c + 1], 0.f));
                    *reinterpret_cast<__nv_bfloat162 *>(&Wp.act2[p0 * SL_C2 + c]) = o0;
                    *reinterpret_cast<__nv_bfloat162 *>(&Wp.act2[p1 * SL_C2 + c]) = o1;
                }
            }
        }
        __syncwarp();
        // conv3: M = 16 (one tile: output rows g >> 2 and 2 + (g >> 2)), N = 16, K = 144 (one tap per k step)
        {
            const int p0 = g, p1 = g + 8;
            auto pair = [&](int p, int tap, int c) -> uint32_t {
                const int iy = 2 * (p >> 2) + tap / 3 - 1, ix = 2 * (p & 3) + tap % 3 - 1;
                if (iy < 0 || ix < 0 || iy >= 8 || ix >= 8) return 0u;
                return pack_bf16x2(&Wp.act2[(iy * 8 + ix) * SL_C2 + c]);
            };
            float d[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
            for (int tap = 0; tap < 9; tap++) {
                uint32_t A[4] = {pair(p0, tap, 2 * tq), pair(p1, tap, 2 * tq), pair(p0, tap, 2 * tq + 8), pair(p1, tap, 2 * tq + 8)};
#pragma unroll
                for (int nt = 0; nt < 2; nt++) {
                    const __nv_bfloat16 *wr = &S.w3[(nt * 8 + g) * SLI_W3S + tap * 16 + 2 * tq];
                    mma_bf16(d[nt], A, pack_bf16x2(wr), pack_bf16x2(wr + 8));
                }
            }
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                const int c = nt * 8 + 2 * tq;
                __nv_bfloat162 o0, o1;
                o0.x = __float2bfloat16(fmaxf(d[nt][0] + S.b3[c], 0.f));
                o0.y = __float2bfloat16(fmaxf(d[nt][1] + S.b3[c + 1], 0.f));
                o1.x = __float2bfloat16(fmaxf(d[nt][2] + S.b3[c], 0.f));
                o1.y = __float2bfloat16(fmaxf(d[nt][3] + S.b3[c + 1], 0.f));
                *reinterpret_cast<__nv_bfloat162 *>(&zr[p0 * SL_C3 + c]) = o0;
                *reinterpret_cast<__nv_bfloat162 *>(&zr[p1 * SL_C3 + c]) = o1;
            }
        }
        __syncwarp();
    }
}

// the shortlist of one block from its scores (one thread)
__device__ __forceinline__ SlCand sl_select(const float *s, int bs, const SlSel &P) {
    SlCand out;
#pragma unroll
    for (int k = 0; k < 8; k++) out.c[k] = 0;
#pragma unroll
    for (int k = 0; k < 5; k++) out.pad[k] = 0;
    float mx = s[0];
    for (int k = 1; k < SL_MD; k++) mx = fmaxf(mx, s[k]);
    float z = 0.f;
    for (int k = 0; k < SL_MD; k++) z += __expf(s[k] - mx);
    uint64_t taken0 = 0;   // classes 0..60
    float acc = 0.f;
    int n = 0;
    for (; n < P.maxCand && acc < P.tau; n++) {
        int b = -1;
        float bv = -1e30f;
        for (int k = 0; k < SL_MD; k++)
            if (!((taken0 >> k) & 1) && s[k] > bv) { bv = s[k]; b = k; }   // the lower class of equal scores
        const float p = __expf(bv - mx) / z;
        if (n == 0 && p < P.conf) break;
        taken0 |= 1ull << b;
        out.c[n] = (uint8_t)sl_class_cand(b);
        acc += p;
    }
    out.n = (uint8_t)n;
    // tx types of the block's set by probability
    const int set = tx_set_intra(ST(Max_Tx_Size_Rect)[bs]);
    uint32_t mask = 0;
    if (n > 0 && set != AV1G_TX_SET_DCTONLY && P.maxTx > 0) {
        float tmx = -1e30f, tz = 0.f;
        for (int t = 0; t < 16; t++) if (tx_in_set(set, t)) tmx = fmaxf(tmx, s[SL_TX0 + t]);
        for (int t = 0; t < 16; t++) if (tx_in_set(set, t)) tz += __expf(s[SL_TX0 + t] - tmx);
        float ta = 0.f;
        for (int k = 0; k < P.maxTx && ta < P.txTau; k++) {
            int b = -1;
            float bv = -1e30f;
            for (int t = 0; t < 16; t++)
                if (tx_in_set(set, t) && !((mask >> t) & 1) && s[SL_TX0 + t] > bv) { bv = s[SL_TX0 + t]; b = t; }
            if (b < 0) break;
            mask |= 1u << b;
            ta += __expf(bv - tmx) / tz;
        }
    }
    out.txMask = (uint16_t)mask;
    return out;
}

// shortlists of the scored records [i0, i0 + n) from their scores S [n][SL_OUT] (records outside the frame: none)
__global__ void k_sl_select(const __grid_constant__ FrameDesc F, const float *__restrict__ S, uint32_t i0, int n, SlSel P,
                            SlCand *__restrict__ outC) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int bs, x, y;
    uint32_t rec;
    if (!sl_scored_record(F, i0 + r, bs, rec)) return;
    sl_record_xy(F, bs, rec, x, y);
    if (x >= F.MiCols * 4 || y >= F.MiRows * 4) return;
    outC[i0 + r] = sl_select(S + (size_t)r * SL_OUT, bs, P);
}

// The learned shortlists of an image's scored records on stream s, in chunks of SL_CHUNK records through the chunk
// buffers Z [SL_CHUNK][SL_Z], H [SL_CHUNK][SL_HID] (bf16), S [SL_CHUNK][SL_OUT] (fp32): k_sl_conv, fc1 and fc2 on the
// tensor cores, k_sl_select.  scores (optional): every chunk's S copied to scores + i0 SL_OUT.
static inline cudaError_t sl_infer_image(const FrameDesc &F, const SlNet &net, const SlSel &sel, int nSm, __nv_bfloat16 *Z,
                                         __nv_bfloat16 *H, float *S, SlCand *outC, float *scores, cudaStream_t s) {
    int idx[22];
    const uint32_t ns = sl_scored_layout(F, idx);
    for (uint32_t i0 = 0; i0 < ns; i0 += SL_CHUNK) {
        const int cn = (int)std::min<uint32_t>(SL_CHUNK, ns - i0);
        const unsigned grid = (unsigned)std::max(1, std::min(2 * nSm, (cn + SLC_WARPS - 1) / SLC_WARPS));
        k_sl_conv<<<grid, SLC_WARPS * 32, sizeof(SlcSmem), s>>>(F, net, i0, cn, Z);
        k_gemm_abt<<<dim3((SL_HID + GT_N - 1) / GT_N, (cn + GT_M - 1) / GT_M, 1), 128, 0, s>>>(cn, SL_HID, SL_Z, Z, SL_Z, net.f1, SL_Z,
                                                                                              nullptr, 0, net.bf1, 1, H, SL_HID, SL_Z);
        k_gemm_abt<<<dim3((SL_OUT + GT_N - 1) / GT_N, (cn + GT_M - 1) / GT_M, 1), 128, 0, s>>>(cn, SL_OUT, SL_HID, H, SL_HID, net.f2, SL_HID,
                                                                                              S, SL_OUT, net.bf2, 0, nullptr, 0, SL_HID);
        if (outC) k_sl_select<<<(cn + 127) / 128, 128, 0, s>>>(F, S, i0, cn, sel, outC);
        if (scores) {
            const cudaError_t e = cudaMemcpyAsync(scores + (size_t)i0 * SL_OUT, S, (size_t)cn * SL_OUT * 4, cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaGetLastError();
}

}  // namespace is
