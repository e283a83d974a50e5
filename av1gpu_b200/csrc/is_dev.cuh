// is_dev.cuh - device building blocks of the B200 intra search (sm_100a).
//
// Everything here is integer arithmetic on the INT32 pipes; warp primitives (shuffles, ballots) do the reductions.
//   - spec geometry rules (block / tx sizes, tx sets, scans, chroma ownership) over the AV1 spec tables of av1core's
//     spec_tables.h (data only; av1core's dsp.h / blockinfo.h functions are not used by the product)
//   - intra prediction of one sample (spec 7.11.2, intra edge filter off) and edge preparation from a plane
//   - the forward 2-D transform: transposed spec butterfly networks (txfm_gen.cuh), one lane per column, then one lane
//     per row, registers only
//   - dead-zone quantiser, transform-domain distortion and the exact coefficient rate with every in-block context
//   - the exact inverse transform with the spec's conformance checks (for the reconstruction)
// Fixed-point conventions (shared with the CPU oracle, which restates them independently): coefficients carry FB = 3
// fractional bits; D is pixel SSE * 2^16; R is in 1/256 bit; lambda in 1/256; J = D + lambda * R (int64).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <type_traits>
#include "av1g/decisions.h"
#include "av1g/enums_gen.h"
#include "av1g/spec_tables.h"
#include "av1g/cdfctx.h"
#include "txfm_gen.cuh"

namespace is {

typedef long long i64;
constexpr i64 INF = 1LL << 60;
constexpr int FB = 3;
constexpr int NCDF = (int)(sizeof(av1g_cdfs) / 2);
// plain-form knobs (reference GpConfig defaults, encoder/src/pipeline.cpp:41-76)
constexpr int K_TOP = 4, K_RECHECK = 2, UV_K = 2;
constexpr int UV_OVERHEAD = 384;   // uvOverheadBits 1.5 in 1/256 bit
constexpr int EDGE_OFF = 16, EDGE_LEN = 16 + 2 * 64 + 16;

// ---- fixed-point tables (host-built, uploaded once per process) ----
static __device__ uint16_t g_cost[4][NCDF];   // -log2(p) * 256 of every CDF symbol of av1g_cdfs, per coefficient q-context
static __constant__ int c_avgY[13];           // y_mode bits averaged over its 25 contexts
static __constant__ int c_avgPart[5][10];     // partition bits averaged over contexts, per block-size level
static __constant__ int c_avgSkip0;           // skip = 0 averaged over contexts

// ---- the spec tables of the device code, in constant memory (av1core spec_tables.h values, copied from its host
// tables when the library uploads its tables): uniform-index reads hit the constant cache instead of global memory ----
#define IS_SPEC_TABLES(X) \
    X(uint8_t, Adjusted_Tx_Size, [19]) \
    X(uint8_t, Coeff_Base_Pos_Ctx_Offset, [3]) \
    X(uint16_t, Dr_Intra_Derivative, [90]) \
    X(uint8_t, Intra_Mode_Context, [13]) \
    X(uint8_t, Mag_Ref_Offset_With_Tx_Class, [3][3][2]) \
    X(uint8_t, Max_Tx_Size_Rect, [22]) \
    X(uint8_t, Mode_To_Angle, [13]) \
    X(uint8_t, Mode_To_Txfm, [14]) \
    X(uint8_t, Num_4x4_Blocks_High, [22]) \
    X(uint8_t, Num_4x4_Blocks_Wide, [22]) \
    X(uint8_t, Partition_Subsize, [10][22]) \
    X(uint8_t, Sig_Ref_Diff_Offset, [3][5][2]) \
    X(uint8_t, Sm_Weights_Tx_16x16, [16]) \
    X(uint8_t, Sm_Weights_Tx_32x32, [32]) \
    X(uint8_t, Sm_Weights_Tx_4x4, [4]) \
    X(uint8_t, Sm_Weights_Tx_64x64, [64]) \
    X(uint8_t, Sm_Weights_Tx_8x8, [8]) \
    X(uint8_t, Subsampled_Size, [22][2][2]) \
    X(uint8_t, Transform_Row_Shift, [19]) \
    X(uint8_t, Tx_Height, [19]) \
    X(uint8_t, Tx_Height_Log2, [19]) \
    X(uint8_t, Tx_Size_Sqr, [19]) \
    X(uint8_t, Tx_Size_Sqr_Up, [19]) \
    X(uint8_t, Tx_Type_In_Set_Intra, [3][16]) \
    X(uint8_t, Tx_Type_Intra_Inv_Set1, [7]) \
    X(uint8_t, Tx_Type_Intra_Inv_Set2, [5]) \
    X(uint8_t, Tx_Width, [19]) \
    X(uint8_t, Tx_Width_Log2, [19])
#define IS_DECL_SPEC_TABLE(T, name, dims) static __constant__ T c_##name dims;
IS_SPEC_TABLES(IS_DECL_SPEC_TABLE)
#define ST(name) c_##name

// ---- the tables of the rate loop: the cost table of the image's q-context, every scan of the intra tx sizes /
// classes (packed), the 2-D base-context offsets.  A kernel whose few warps each run a long dependent chain (the
// closed loop) stages them once per CTA in shared memory (RateStage); the others read them from global memory. ----
constexpr int SCAN_PACK = 4912;
static __device__ uint16_t g_scanPack[SCAN_PACK];     // the scans, packed (host-built from the spec tables)
static __device__ uint8_t g_baseCtx[19 * 25];         // Coeff_Base_Ctx_Offset
static __constant__ uint16_t c_scanOff[19][3];        // offset of the scan of (tx size, class 2D / VERT / HORIZ) in the pack
struct RateTabs {
    const uint16_t *cost, *scan;
    const uint8_t *baseCtx;                    // [19][5][5]
};
struct __align__(16) RateStage {
    uint16_t cost[NCDF];
    uint16_t scan[SCAN_PACK];
    uint8_t baseCtx[19 * 25];
    uint8_t pad[5];
};
// staged with 16-byte vector stores (cost, scan) and followed by 16-byte-aligned buffers in the kernels' shared memory
static_assert(sizeof(RateStage) % 16 == 0 && (NCDF * 2) % 16 == 0 && (SCAN_PACK * 2) % 16 == 0, "RateStage layout");
__device__ __forceinline__ RateTabs rate_tabs_global(int qctx) { return RateTabs{g_cost[qctx], g_scanPack, g_baseCtx}; }
// all threads of the CTA; followed by __syncthreads() at the caller
__device__ __forceinline__ RateTabs rate_tabs_stage(RateStage &T, int qctx, int tid, int nt) {
    const uint4 *c = reinterpret_cast<const uint4 *>(g_cost[qctx]);
    for (int i = tid; i < NCDF / 8; i += nt) reinterpret_cast<uint4 *>(T.cost)[i] = c[i];
    for (int i = tid; i < SCAN_PACK / 8; i += nt) reinterpret_cast<uint4 *>(T.scan)[i] = reinterpret_cast<const uint4 *>(g_scanPack)[i];
    for (int i = tid; i < 19 * 25; i += nt) T.baseCtx[i] = g_baseCtx[i];
    return RateTabs{T.cost, T.scan, T.baseCtx};
}

// ---- index of an entry of av1g_cdfs (uint16 units) ----
#define IS_CB(f) ((int)(offsetof(av1g_cdfs, f) / 2))
#define IS_CD(f, d) ((int)std::extent<decltype(av1g_cdfs::f), d>::value)
__device__ __forceinline__ int ci_y_mode(int a, int l) { return IS_CB(y_mode) + (a * IS_CD(y_mode, 1) + l) * IS_CD(y_mode, 2); }
__device__ __forceinline__ int ci_uv_cfl(int y) { return IS_CB(uv_mode_cfl_allowed) + y * IS_CD(uv_mode_cfl_allowed, 1); }
__device__ __forceinline__ int ci_uv_nocfl(int y) { return IS_CB(uv_mode_cfl_not_allowed) + y * IS_CD(uv_mode_cfl_not_allowed, 1); }
__device__ __forceinline__ int ci_angle(int m) { return IS_CB(angle_delta) + m * IS_CD(angle_delta, 1); }
__device__ __forceinline__ int ci_set1(int s, int d) { return IS_CB(intra_tx_set1) + (s * IS_CD(intra_tx_set1, 1) + d) * IS_CD(intra_tx_set1, 2); }
__device__ __forceinline__ int ci_set2(int s, int d) { return IS_CB(intra_tx_set2) + (s * IS_CD(intra_tx_set2, 1) + d) * IS_CD(intra_tx_set2, 2); }
__device__ __forceinline__ int ci_cfl_sign() { return IS_CB(cfl_sign); }
__device__ __forceinline__ int ci_cfl_alpha(int c) { return IS_CB(cfl_alpha) + c * IS_CD(cfl_alpha, 1); }
__device__ __forceinline__ int ci_txb_skip(int a, int b) { return IS_CB(txb_skip) + (a * IS_CD(txb_skip, 1) + b) * IS_CD(txb_skip, 2); }
__device__ __forceinline__ int ci_eob_pt(int ms, int p, int c) {
    switch (ms) {
    case 0: return IS_CB(eob_pt_16) + (p * 2 + c) * IS_CD(eob_pt_16, 2);
    case 1: return IS_CB(eob_pt_32) + (p * 2 + c) * IS_CD(eob_pt_32, 2);
    case 2: return IS_CB(eob_pt_64) + (p * 2 + c) * IS_CD(eob_pt_64, 2);
    case 3: return IS_CB(eob_pt_128) + (p * 2 + c) * IS_CD(eob_pt_128, 2);
    case 4: return IS_CB(eob_pt_256) + (p * 2 + c) * IS_CD(eob_pt_256, 2);
    case 5: return IS_CB(eob_pt_512) + p * IS_CD(eob_pt_512, 1);
    default: return IS_CB(eob_pt_1024) + p * IS_CD(eob_pt_1024, 1);
    }
}
__device__ __forceinline__ int ci_eob_extra(int s, int p, int k) {
    return IS_CB(eob_extra) + ((s * IS_CD(eob_extra, 1) + p) * IS_CD(eob_extra, 2) + k) * IS_CD(eob_extra, 3);
}
__device__ __forceinline__ int ci_dc_sign(int p, int c) { return IS_CB(dc_sign) + (p * IS_CD(dc_sign, 1) + c) * IS_CD(dc_sign, 2); }
__device__ __forceinline__ int ci_base_eob(int s, int p, int c) {
    return IS_CB(coeff_base_eob) + ((s * IS_CD(coeff_base_eob, 1) + p) * IS_CD(coeff_base_eob, 2) + c) * IS_CD(coeff_base_eob, 3);
}
__device__ __forceinline__ int ci_base(int s, int p, int c) {
    return IS_CB(coeff_base) + ((s * IS_CD(coeff_base, 1) + p) * IS_CD(coeff_base, 2) + c) * IS_CD(coeff_base, 3);
}
__device__ __forceinline__ int ci_br(int s, int p, int c) {
    return IS_CB(coeff_br) + ((s * IS_CD(coeff_br, 1) + p) * IS_CD(coeff_br, 2) + c) * IS_CD(coeff_br, 3);
}

// ---- shared-memory poison (is_set_poison): every word of a kernel's shared memory starts as a fixed garbage pattern,
// so a read before the kernel's own write changes the results instead of finding a benign leftover.  The caller
// synchronises the CTA after it. ----
__device__ __forceinline__ void smem_poison(unsigned char *base, size_t bytes, int tid, int nt) {
    for (size_t i = tid; i < bytes / 4; i += nt) reinterpret_cast<uint32_t *>(base)[i] = 0xA5C3E1F7u;
}

// ---- warp helpers ----
__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ int warp_sum(int v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ i64 warp_sum64(i64 v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ int warp_max(int v) {
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// index of the smallest (v, i) over the warp; the first of equal values (a serial scan's pick); -1 if all are >= INF
__device__ __forceinline__ int warp_argmin(i64 v, int i) {
    for (int o = 16; o > 0; o >>= 1) {
        const i64 ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, i, o);
        if (ov < v || (ov == v && oi < i)) { v = ov; i = oi; }
    }
    return v < INF ? i : -1;
}

// The best (at most 3) tx types of an analysed block by open-loop RD cost, the first evaluated of equal costs ahead:
// the tx types FrameDesc::txKeep lets the closed loop's second pass try (BlockRes::txMask).
struct TxRank {
    i64 j[3];
    int t[3];
    __device__ __forceinline__ TxRank() : j{INF, INF, INF}, t{0, 0, 0} {}
    __device__ __forceinline__ void add(i64 v, int ty) {   // after every kept entry of cost <= v
        const int pos = (j[0] <= v) + (j[1] <= v) + (j[2] <= v);
#pragma unroll
        for (int s = 2; s >= 0; s--) {
            if (s > pos) { j[s] = j[s > 0 ? s - 1 : 0]; t[s] = t[s > 0 ? s - 1 : 0]; }
            else if (s == pos) { j[s] = v; t[s] = ty; }
        }
    }
    __device__ __forceinline__ uint16_t mask(int keep) const {   // 0 (every type) when keep is 0
        uint32_t m = 0;
#pragma unroll
        for (int s = 0; s < 3; s++)
            if (s < keep && j[s] < INF) m |= 1u << t[s];
        return (uint16_t)m;
    }
};

// ---- geometry (spec tables) ----
__device__ __forceinline__ int bw4(int bs) { return ST(Num_4x4_Blocks_Wide)[bs]; }
__device__ __forceinline__ int bh4(int bs) { return ST(Num_4x4_Blocks_High)[bs]; }
__device__ __forceinline__ int txw(int t) { return ST(Tx_Width)[t]; }
__device__ __forceinline__ int txh(int t) { return ST(Tx_Height)[t]; }
__device__ __forceinline__ bool is_dir(int m) { return m >= AV1G_V_PRED && m <= AV1G_D67_PRED; }
__device__ __forceinline__ int cand_mode(int c) { return c >> 3; }
__device__ __forceinline__ int cand_delta(int c) { return (c & 7) - 3; }
__device__ __forceinline__ int cand_pack(int m, int d) { return (m << 3) | (d + 3); }
__device__ __forceinline__ int pangle(int m, int d) { return is_dir(m) ? ST(Mode_To_Angle)[m] + d * AV1G_ANGLE_STEP : 0; }

// get_tx_set() for intra (spec 5.11.48), reduced_tx_set = 0
__device__ __forceinline__ int tx_set_intra(int txSz) {
    const int up = ST(Tx_Size_Sqr_Up)[txSz];
    if (up >= AV1G_TX_32X32) return AV1G_TX_SET_DCTONLY;
    if (ST(Tx_Size_Sqr)[txSz] == AV1G_TX_16X16) return AV1G_TX_SET_INTRA_2;
    return AV1G_TX_SET_INTRA_1;
}
__device__ __forceinline__ bool tx_in_set(int set, int t) { return ST(Tx_Type_In_Set_Intra)[set][t] != 0; }
// 1-D kinds of a 2-D type: 0 DCT, 1 ADST, 2 identity (no FLIPADST occurs in the intra sets)
__device__ __forceinline__ int col_kind(int t) {
    return (t == AV1G_DCT_DCT || t == AV1G_DCT_ADST || t == AV1G_V_DCT) ? 0 : (t == AV1G_IDTX || t == AV1G_H_DCT) ? 2 : 1;
}
__device__ __forceinline__ int row_kind(int t) {
    return (t == AV1G_DCT_DCT || t == AV1G_ADST_DCT || t == AV1G_H_DCT) ? 0 : (t == AV1G_IDTX || t == AV1G_V_DCT) ? 2 : 1;
}
__device__ __forceinline__ int tx_class(int t) {
    return t == AV1G_V_DCT ? AV1G_TX_CLASS_VERT : t == AV1G_H_DCT ? AV1G_TX_CLASS_HORIZ : AV1G_TX_CLASS_2D;
}
// chroma type (spec compute_tx_type for plane > 0): Mode_To_Txfm if in the set, else DCT_DCT
__device__ __forceinline__ int chroma_tx_type(int uvTx, int uvMode) {
    if (ST(Tx_Size_Sqr_Up)[uvTx] > AV1G_TX_32X32) return AV1G_DCT_DCT;
    const int t = ST(Mode_To_Txfm)[uvMode];
    return tx_in_set(tx_set_intra(uvTx), t) ? t : AV1G_DCT_DCT;
}
// get_scan() (spec 5.11.41), intra types only (no flips): the scan of the size's class in the packed tables
__device__ __forceinline__ const uint16_t *get_scan(const RateTabs &T, int txSz, int txType) {
    const int cls = txType == AV1G_IDTX ? 0 : tx_class(txType);
    return T.scan + c_scanOff[txSz][cls];
}
__device__ __forceinline__ int dq_denom(int txSz) {
    if (txSz == AV1G_TX_32X32 || txSz == AV1G_TX_16X32 || txSz == AV1G_TX_32X16 || txSz == AV1G_TX_16X64 || txSz == AV1G_TX_64X16) return 2;
    if (txSz == AV1G_TX_64X64 || txSz == AV1G_TX_32X64 || txSz == AV1G_TX_64X32) return 4;
    return 1;
}
// spec 7.12.3 step 1 without quantizer matrices: (|l q| & 0xFFFFFF) / den, signed, clamped to 2^(7 + BitDepth)
template <int BD> __device__ __forceinline__ int dequant(int l, int q, int den) {
    const int dq = l * q;
    int a = (dq < 0 ? -dq : dq) & 0xFFFFFF;
    a /= den;
    if (dq < 0) a = -a;
    return min(max(a, -(1 << (7 + BD))), (1 << (7 + BD)) - 1);
}
// HasChroma (spec decode_block); 4:2:0 when ss = 1
__device__ __forceinline__ bool has_chroma(int bs, int mi_row, int mi_col, int ss) {
    if (ss && bh4(bs) == 1 && (mi_row & 1) == 0) return false;
    if (ss && bw4(bs) == 1 && (mi_col & 1) == 0) return false;
    return true;
}
__device__ __forceinline__ int uv_bsize(int bs, int ss) { return ST(Subsampled_Size)[bs][ss][ss]; }
__device__ __forceinline__ int uv_tx_size(int bs, int ss) {
    const int t = ST(Max_Tx_Size_Rect)[uv_bsize(bs, ss)];
    const int w = txw(t), h = txh(t);
    if (w == 64 || h == 64) return w == 16 ? AV1G_TX_16X32 : h == 16 ? AV1G_TX_32X16 : AV1G_TX_32X32;
    return t;
}

// ---------------------------------------------------------------------------------------------------------------
// intra prediction of one sample (spec 7.11.2.2 / .4 / .5 / .6, edge filter and upsampling off).  A / L point at
// AboveRow[0] / LeftCol[0] (index -1 valid).
// ---------------------------------------------------------------------------------------------------------------
template <typename P>
__device__ __forceinline__ int pred_px(int mode, int pAng, int i, int j, int lw, int lh, const P *A, const P *L, int dcv) {
    const int w = 1 << lw, h = 1 << lh;
    if (mode == AV1G_DC_PRED) return dcv;
    if (is_dir(mode)) {
        if (pAng == 90) return A[j];
        if (pAng == 180) return L[i];
        if (pAng < 90) {
            const int dx = ST(Dr_Intra_Derivative)[pAng];
            const int idx = (i + 1) * dx, base = (idx >> 6) + j, sh = (idx >> 1) & 0x1F;
            const int maxBaseX = w + h - 1;
            return base < maxBaseX ? (A[base] * (32 - sh) + A[base + 1] * sh + 16) >> 5 : A[maxBaseX];
        }
        if (pAng < 180) {
            const int dx = ST(Dr_Intra_Derivative)[180 - pAng];
            int idx = (j << 6) - (i + 1) * dx;
            int base = idx >> 6;
            if (base >= -1) {
                const int sh = (idx >> 1) & 0x1F;
                return (A[base] * (32 - sh) + A[base + 1] * sh + 16) >> 5;
            }
            const int dy = ST(Dr_Intra_Derivative)[pAng - 90];
            idx = (i << 6) - (j + 1) * dy;
            base = idx >> 6;
            const int sh = (idx >> 1) & 0x1F;
            return (L[base] * (32 - sh) + L[base + 1] * sh + 16) >> 5;
        }
        const int dy = ST(Dr_Intra_Derivative)[270 - pAng];
        const int idx = (j + 1) * dy, base = (idx >> 6) + i, sh = (idx >> 1) & 0x1F;
        return (L[base] * (32 - sh) + L[base + 1] * sh + 16) >> 5;
    }
    if (mode == AV1G_PAETH_PRED) {
        const int a = A[j], l = L[i], tl = A[-1], base = a + l - tl;
        const int pL = abs(base - l), pT = abs(base - a), pTL = abs(base - tl);
        return (pL <= pT && pL <= pTL) ? l : pT <= pTL ? a : tl;
    }
    const uint8_t *wx = lw == 2 ? ST(Sm_Weights_Tx_4x4) : lw == 3 ? ST(Sm_Weights_Tx_8x8) : lw == 4 ? ST(Sm_Weights_Tx_16x16)
                      : lw == 5 ? ST(Sm_Weights_Tx_32x32) : ST(Sm_Weights_Tx_64x64);
    const uint8_t *wy = lh == 2 ? ST(Sm_Weights_Tx_4x4) : lh == 3 ? ST(Sm_Weights_Tx_8x8) : lh == 4 ? ST(Sm_Weights_Tx_16x16)
                      : lh == 5 ? ST(Sm_Weights_Tx_32x32) : ST(Sm_Weights_Tx_64x64);
    if (mode == AV1G_SMOOTH_PRED)
        return (wy[i] * A[j] + (256 - wy[i]) * L[h - 1] + wx[j] * L[i] + (256 - wx[j]) * A[w - 1] + 256) >> 9;
    if (mode == AV1G_SMOOTH_V_PRED) return (wy[i] * A[j] + (256 - wy[i]) * L[h - 1] + 128) >> 8;
    return (wx[j] * L[i] + (256 - wx[j]) * A[w - 1] + 128) >> 8;   // SMOOTH_H
}

// One 4x4 sub-block (rows sy.., cols sx..) of a block's prediction into p[16], the values of pred_px with the mode
// dispatch hoisted out of the samples (one branch per sub-block instead of per sample).  Not inlined: one copy
// (~30 KB of code) serves every caller of a kernel instead of one per call site, which keeps the kernels' hot code
// within reach of the instruction caches.
template <typename P>
__device__ __forceinline__ void pred4_inl(int mode, int pAng, int sy, int sx, int lw, int lh, const P *A, const P *L, int dcv, int *p) {
    const int w = 1 << lw, h = 1 << lh;
    if (mode == AV1G_DC_PRED) {
#pragma unroll
        for (int k = 0; k < 16; k++) p[k] = dcv;
        return;
    }
    if (is_dir(mode)) {
        if (pAng == 90) {
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) p[i * 4 + j] = A[sx + j];
        } else if (pAng == 180) {
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) p[i * 4 + j] = L[sy + i];
        } else if (pAng < 90) {
            const int dx = ST(Dr_Intra_Derivative)[pAng], maxBaseX = w + h - 1;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int idx = (sy + i + 1) * dx, base = (idx >> 6) + sx, sh = (idx >> 1) & 0x1F;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int k = base + j;
                    p[i * 4 + j] = k < maxBaseX ? (A[k] * (32 - sh) + A[k + 1] * sh + 16) >> 5 : A[maxBaseX];
                }
            }
        } else if (pAng > 180) {
            const int dy = ST(Dr_Intra_Derivative)[270 - pAng];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int idx = (sx + j + 1) * dy, base = (idx >> 6) + sy, sh = (idx >> 1) & 0x1F;
#pragma unroll
                for (int i = 0; i < 4; i++) p[i * 4 + j] = (L[base + i] * (32 - sh) + L[base + i + 1] * sh + 16) >> 5;
            }
        } else {
            const int dx = ST(Dr_Intra_Derivative)[180 - pAng], dy = ST(Dr_Intra_Derivative)[pAng - 90];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    int idx = ((sx + j) << 6) - (sy + i + 1) * dx;
                    const P *E = A;
                    if ((idx >> 6) < -1) { idx = ((sy + i) << 6) - (sx + j + 1) * dy; E = L; }
                    const int b = idx >> 6, sh = (idx >> 1) & 0x1F;
                    p[i * 4 + j] = (E[b] * (32 - sh) + E[b + 1] * sh + 16) >> 5;
                }
        }
        return;
    }
    if (mode == AV1G_PAETH_PRED) {
        const int tl = A[-1];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int a = A[sx + j], l = L[sy + i], base = a + l - tl;
                const int pL = abs(base - l), pT = abs(base - a), pTL = abs(base - tl);
                p[i * 4 + j] = (pL <= pT && pL <= pTL) ? l : pT <= pTL ? a : tl;
            }
        return;
    }
    // SMOOTH / SMOOTH_V / SMOOTH_H: sum of the vertical and horizontal terms of the modes that use them
    const uint8_t *wx = (lw == 2 ? ST(Sm_Weights_Tx_4x4) : lw == 3 ? ST(Sm_Weights_Tx_8x8) : lw == 4 ? ST(Sm_Weights_Tx_16x16)
                       : lw == 5 ? ST(Sm_Weights_Tx_32x32) : ST(Sm_Weights_Tx_64x64)) + sx;
    const uint8_t *wy = (lh == 2 ? ST(Sm_Weights_Tx_4x4) : lh == 3 ? ST(Sm_Weights_Tx_8x8) : lh == 4 ? ST(Sm_Weights_Tx_16x16)
                       : lh == 5 ? ST(Sm_Weights_Tx_32x32) : ST(Sm_Weights_Tx_64x64)) + sy;
    const int bl = L[h - 1], tr = A[w - 1];
    const int sh = mode == AV1G_SMOOTH_PRED ? 9 : 8, useV = mode != AV1G_SMOOTH_H_PRED, useH = mode != AV1G_SMOOTH_V_PRED;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int v = useV ? wy[i] * A[sx + j] + (256 - wy[i]) * bl : 0;
            const int hz = useH ? wx[j] * L[sy + i] + (256 - wx[j]) * tr : 0;
            p[i * 4 + j] = (v + hz + (1 << (sh - 1))) >> sh;
        }
}

// 4x4 Hadamard: sum of |coefficients| (the reference's SATD proxy, 4 x the orthonormal SATD)
__device__ __forceinline__ int hadamard4_sum(int *d) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
        int *r = d + 4 * i;
        const int s0 = r[0] + r[1], s1 = r[0] - r[1], s2 = r[2] + r[3], s3 = r[2] - r[3];
        r[0] = s0 + s2; r[1] = s1 + s3; r[2] = s0 - s2; r[3] = s1 - s3;
    }
    int sum = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int s0 = d[j] + d[4 + j], s1 = d[j] - d[4 + j], s2 = d[8 + j] + d[12 + j], s3 = d[8 + j] - d[12 + j];
        sum += abs(s0 + s2) + abs(s1 + s3) + abs(s0 - s2) + abs(s1 - s3);
    }
    return sum;
}

// One 4x4 sub-block of a candidate's prediction (row sy, column sx of a W x H block), kept in registers: with out, it
// is stored there (row stride W) and 0 returned; otherwise its SATD against src (row stride sp, the block's sample
// (0, 0)) is returned.  The one out-of-line copy of the predictor serves both the screening and whole predictions.
template <typename P, typename O>
__device__ __noinline__ int pred4_x(int mode, int pAng, int sy, int sx, int lw, int lh, const P *A, const P *L, int dcv, const P *src, int sp,
                                    O *out) {
    int d[16];
    pred4_inl(mode, pAng, sy, sx, lw, lh, A, L, dcv, d);
    if (out) {
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) out[((sy + i) << lw) + sx + j] = (O)d[i * 4 + j];
        return 0;
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) d[i * 4 + j] = (int)src[(sy + i) * sp + sx + j] - d[i * 4 + j];
    return hadamard4_sum(d);
}
template <typename P>
__device__ __forceinline__ int pred4_satd(int mode, int pAng, int sy, int sx, int lw, int lh, const P *A, const P *L, int dcv, const P *src, int sp) {
    return pred4_x<P, P>(mode, pAng, sy, sx, lw, lh, A, L, dcv, src, sp, (P *)nullptr);
}

// the whole prediction of a W x H block into out (row stride W) by the G lanes of a group: 4x4 sub-blocks over the
// lanes, or, when the block has fewer sub-blocks than the group has lanes, samples over the lanes (pred_px: the same
// values, the work spread over every lane instead of one lane per sub-block)
template <typename P, typename O>
__device__ __noinline__ void grp_predict(int mode, int pAng, int lw, int lh, const P *A, const P *L, int dcv, O *out, int g, int G) {
    const int nsx = 1 << (lw - 2), nsub = 1 << (lw + lh - 4);
    if (nsub < G) {
        for (int q = g; q < (1 << (lw + lh)); q += G) out[q] = (O)pred_px(mode, pAng, q >> lw, q & ((1 << lw) - 1), lw, lh, A, L, dcv);
        return;
    }
    for (int sb = g; sb < nsub; sb += G) {
        const int sx = (sb & (nsx - 1)) * 4, sy = (sb >> (lw - 2)) * 4;
        pred4_x<P, O>(mode, pAng, sy, sx, lw, lh, A, L, dcv, nullptr, 0, out);
    }
}
// CfL prediction (spec 7.11.5 with the DC prediction dcv) of a W x H chroma block into out (row stride W)
template <typename O>
__device__ __forceinline__ void grp_predict_cfl(int lw, int lh, int dcv, const int16_t *cfl, int alpha, int avg, int maxv, O *out, int g, int G) {
    for (int p = g; p < (1 << (lw + lh)); p += G) {
        const int v = alpha * (cfl[p] - avg);
        const int s = v >= 0 ? (v + 32) >> 6 : -((-v + 32) >> 6);
        out[p] = (O)min(max(dcv + s, 0), maxv);
    }
}

// AboveRow / LeftCol preparation (spec 7.11.2, "intra edge" arrays): lanes t = 0..nt-1 of a group fill
// A[-1 .. w+h-1] / L[-1 .. w+h-1] from a plane (pointer at sample (0, 0), pitch in samples).
template <int BD, typename P>
__device__ __forceinline__ void build_edges(const P *plane, int pitch, int x, int y, int w, int h, int haveL, int haveA, int haveAR,
                                            int haveBL, int maxX, int maxY, P *A, P *L, int t, int nt) {
    const int n = w + h;
    const int alim = min(x + (haveAR ? 2 * w : w) - 1, maxX), llim = min(y + (haveBL ? 2 * h : h) - 1, maxY);
    for (int i = t; i < n; i += nt) {
        P a, l;
        if (haveA) a = plane[(size_t)(y - 1) * pitch + min(x + i, alim)];
        else a = haveL ? plane[(size_t)y * pitch + x - 1] : (P)((1 << (BD - 1)) - 1);
        if (haveL) l = plane[(size_t)min(y + i, llim) * pitch + x - 1];
        else l = haveA ? plane[(size_t)(y - 1) * pitch + x] : (P)((1 << (BD - 1)) + 1);
        A[i] = a;
        L[i] = l;
    }
    if (t == 0) {
        P c;
        if (haveA && haveL) c = plane[(size_t)(y - 1) * pitch + x - 1];
        else if (haveA) c = plane[(size_t)(y - 1) * pitch + x];
        else if (haveL) c = plane[(size_t)y * pitch + x - 1];
        else c = (P)(1 << (BD - 1));
        A[-1] = c;
        L[-1] = c;
    }
}
// DC value (spec 7.11.2.5), sums over the warp
template <int BD, typename P>
__device__ __forceinline__ int warp_dc(const P *A, const P *L, int haveL, int haveA, int lw, int lh) {
    const int w = 1 << lw, h = 1 << lh, lane = lane_id();
    int sa = 0, sl = 0;
    for (int k = lane; k < w; k += 32) sa += A[k];
    for (int k = lane; k < h; k += 32) sl += L[k];
    sa = warp_sum(sa);
    sl = warp_sum(sl);
    if (haveL && haveA) return (sa + sl + ((w + h) >> 1)) / (w + h);
    if (haveL) return min((sl + (h >> 1)) >> lh, (1 << BD) - 1);
    if (haveA) return min((sa + (w >> 1)) >> lw, (1 << BD) - 1);
    return 1 << (BD - 1);
}


// ---------------------------------------------------------------------------------------------------------------
// 1-D transforms on a strided int32 vector in shared memory.  Each (kind, length) network exists ONCE in the binary
// (the dispatchers are not inlined): the kernels' instruction footprint stays small enough for the instruction
// caches, whatever mix of block sizes the warps of an SM are working on.
//   forward: T = v << pre; the transposed spec network (txfm_gen.cuh); out i < nout: (rect: Round2(T * 5793, 12)),
//            then Round2(., post) for post > 0 or << -post
//   inverse: T = v (preRect: Round2(T * 2896, 12)); the spec network with its checks at r bits; out: Round2(., post),
//            clamped to clampBits when nonzero
// ---------------------------------------------------------------------------------------------------------------
template <int N> __device__ __forceinline__ void fwd1d(int kind, int32_t *T) {
    if (N >= 32 || kind == 0) {
        if constexpr (N == 4) fwd_dct4(T);
        else if constexpr (N == 8) fwd_dct8(T);
        else if constexpr (N == 16) fwd_dct16(T);
        else if constexpr (N == 32) fwd_dct32(T);
        else fwd_dct64(T);
    } else if (kind == 1) {
        if constexpr (N == 4) fwd_adst4(T);
        else if constexpr (N == 8) fwd_adst8(T);
        else if constexpr (N == 16) fwd_adst16(T);
    } else {
#pragma unroll
        for (int i = 0; i < N; i++) {
            if constexpr (N == 4) T[i] = (T[i] * 5793 + 2048) >> 12;
            else if constexpr (N == 8) T[i] = T[i] * 2;
            else T[i] = (T[i] * 11586 + 2048) >> 12;
        }
    }
}
template <int N>
__device__ __forceinline__ void fwd_mem_n(int kind, int32_t *p, int stride, int pre, int nout, int rect, int post) {
    int32_t T[N];
#pragma unroll
    for (int i = 0; i < N; i++) T[i] = p[i * stride] * (1 << pre);
    fwd1d<N>(kind, T);
#pragma unroll
    for (int i = 0; i < N; i++) {
        if (i < nout) {
            int32_t v = T[i];
            if (rect) v = (v * 5793 + 2048) >> 12;
            v = post > 0 ? (v + (1 << (post - 1))) >> post : v * (1 << -post);
            p[i * stride] = v;
        }
    }
}
static __device__ __noinline__ void fwd1d_mem(int kind, int n, int32_t *p, int stride, int pre, int nout, int rect, int post) {
    switch (n) {
    case 4: fwd_mem_n<4>(kind, p, stride, pre, nout, rect, post); break;
    case 8: fwd_mem_n<8>(kind, p, stride, pre, nout, rect, post); break;
    case 16: fwd_mem_n<16>(kind, p, stride, pre, nout, rect, post); break;
    case 32: fwd_mem_n<32>(0, p, stride, pre, nout, rect, post); break;
    default: fwd_mem_n<64>(0, p, stride, pre, nout, rect, post); break;
    }
}

// runtime geometry of a tx size: the forward transform's shifts (the range rule: s0 = 17 - BD - log2 H keeps every
// column intermediate inside int32 rotations, s1 = log2 W the row inputs, s2 brings the result to the dequantisation
// domain with FB fractional bits, DQ = M_H^T R M_W 2^(rowShift + 4) / (H W / 4) / rect) and the distortion scale
// (pixel SSE = sum (DQ - dequant)^2 2^-(2 FB + k))
struct TxRt {
    int W, H, lw, lh, tw, th, ltw, n, TS, rowShift, rect, s0, s1, s2, dsh;
};
__device__ __forceinline__ TxRt tx_rt(int txSz, int bd) {
    TxRt d;
    d.W = txw(txSz); d.H = txh(txSz);
    d.lw = ST(Tx_Width_Log2)[txSz]; d.lh = ST(Tx_Height_Log2)[txSz];
    d.tw = min(d.W, 32); d.th = min(d.H, 32); d.ltw = min(d.lw, 5); d.n = d.tw * d.th;
    d.TS = d.W + 1;
    d.rowShift = ST(Transform_Row_Shift)[txSz];
    d.rect = (d.lw - d.lh == 1 || d.lh - d.lw == 1) ? 1 : 0;
    const int E = d.rowShift + 4 + FB - (d.lw + d.lh - 2);
    d.s0 = max(0, 17 - bd - d.lh);
    d.s1 = d.lw;
    d.s2 = d.s0 - d.s1 - E;
    d.dsh = 16 - 2 * FB - (2 * (d.rowShift + 4) - (d.lw + d.lh - 2) + d.rect);
    return d;
}

// Residual source of an evaluation: src - a prediction already in shared memory (row stride 1 << lw), or a given
// residual array (kernel tests).
template <typename P>
struct ResFn {
    const P *src;        // sample (0, 0) of the block
    int sp;
    const P *pred;       // the prediction, W x H
    int lw;
    const int32_t *arr;  // residual array (H x W row-major) instead of src - prediction
    __device__ __forceinline__ int operator()(int i, int j) const {
        return arr ? arr[(i << lw) + j] : (int)src[i * sp + j] - (int)pred[(i << lw) + j];
    }
};

// ---- lane groups: G lanes (a power of two) evaluate one task; reductions stay inside the aligned group ----
__device__ __forceinline__ int grp_sum(int v, int G) {
    for (int o = G >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ i64 grp_sum64(i64 v, int G) {
    for (int o = G >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ int grp_max(int v, int G) {
    for (int o = G >> 1; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// lanes per evaluation task for a tx size in the analysis / closed loop: every task runs its column and row passes on
// at least as many lanes as it has columns / rows, the warp holds 32 / G tasks
__device__ __forceinline__ int grp_size(int txSz) {
    const int W = txw(txSz), H = txh(txSz);
    return (W >= 32 || H >= 32) ? 32 : max(max(W, H), 8);
}
// lanes per task for a closed-loop pass of n tasks: as few rounds of 32 / G tasks as the tx size allows - at least
// max(W, H) / 2 lanes (two columns / rows a lane), at least 4 (32 / G <= 8 groups), and 32 / G tasks' levels within
// one 1024-entry buffer - and no more lanes than grp_size.  The results do not depend on G: every task computes the
// same integers, costs are compared in task order.
__device__ __forceinline__ int round_group(int txSz, int n) {
    const int W = txw(txSz), H = txh(txSz), nq = min(W, 32) * min(H, 32);
    const int gmin = max(4, max(max(W, H) >> 1, nq >> 5)), gmax = grp_size(txSz);
    int p = 1;
    while (p < n && p < 32) p <<= 1;   // tasks rounded up to a power of two
    return min(gmax, max(gmin, 32 / p));
}
// scratch of one task: int32 buffer H x (W + 1), levels tw x th
__device__ __forceinline__ int task_buf_ints(int txSz) { return txh(txSz) * (txw(txSz) + 1); }

// ---------------------------------------------------------------------------------------------------------------
// quantisation + distortion + exact rate (warp)
// ---------------------------------------------------------------------------------------------------------------
struct EvalIn {
    int txType, plane, skipCtx, dcCtx, intraDir, dcQ, acQ;
    RateTabs T;          // cost table of the image's q-context, scans, base-context offsets
};
struct EvalOut { i64 D, R; int eob; };

__device__ __forceinline__ int tx_index_in_set(int set, int t) {
    if (set == AV1G_TX_SET_INTRA_1) { for (int i = 0; i < 7; i++) if (ST(Tx_Type_Intra_Inv_Set1)[i] == t) return i; }
    else { for (int i = 0; i < 5; i++) if (ST(Tx_Type_Intra_Inv_Set2)[i] == t) return i; }
    return 0;
}

// txb_skip, tx type, eob position bits
__device__ __forceinline__ i64 base_bits_inl(int txSz, const EvalIn &e, int eob) {
    const int txSzCtx = (ST(Tx_Size_Sqr)[txSz] + ST(Tx_Size_Sqr_Up)[txSz] + 1) >> 1;
    const uint16_t *C = e.T.cost;
    if (eob == 0) return C[ci_txb_skip(txSzCtx, e.skipCtx) + 1];
    i64 b = C[ci_txb_skip(txSzCtx, e.skipCtx)];
    const int ptype = e.plane > 0;
    if (e.plane == 0) {
        const int set = tx_set_intra(txSz);
        if (set > 0) {
            const int sqr = ST(Tx_Size_Sqr)[txSz], idx = tx_index_in_set(set, e.txType);
            b += set == AV1G_TX_SET_INTRA_1 ? C[ci_set1(sqr, e.intraDir) + idx] : C[ci_set2(sqr, e.intraDir) + idx];
        }
    }
    const int ms = min((int)ST(Tx_Width_Log2)[txSz], 5) + min((int)ST(Tx_Height_Log2)[txSz], 5) - 4;
    const int eobPt = eob <= 2 ? eob : 2 + (31 - __clz(eob - 1));
    b += C[ci_eob_pt(ms, ptype, tx_class(e.txType) == AV1G_TX_CLASS_2D ? 0 : 1) + eobPt - 1];
    if (eobPt >= 3) {
        const int rem = eob - ((1 << (eobPt - 2)) + 1);
        b += C[ci_eob_extra(txSzCtx, ptype, eobPt - 3) + ((rem >> (eobPt - 3)) & 1)];
        b += (eobPt - 3) * 256;
    }
    return b;
}
// out of line with scalar arguments: no structure of the caller has to be written to memory for the call
static __device__ __noinline__ i64 base_bits(int txSz, int txType, int plane, int skipCtx, int intraDir, const uint16_t *cost, int eob) {
    EvalIn e;
    e.txType = txType; e.plane = plane; e.skipCtx = skipCtx; e.intraDir = intraDir;
    e.T.cost = cost;
    return base_bits_inl(txSz, e, eob);
}

// bits of the coefficient at scan position c < eob (levels q natural order, row stride = adjusted width)
__device__ __forceinline__ int coeff_bits(int c, int eob, const int16_t *q, const uint16_t *scan, int txSz, int txClass, int ptype,
                                          int dcCtx, const RateTabs &T) {
    const uint16_t *C = T.cost;
    const int txSzCtx = (ST(Tx_Size_Sqr)[txSz] + ST(Tx_Size_Sqr_Up)[txSz] + 1) >> 1;
    const int adj = ST(Adjusted_Tx_Size)[txSz];
    const int bwl = ST(Tx_Width_Log2)[adj];
    const int width = 1 << bwl, height = ST(Tx_Height)[adj];
    const int pos = scan[c];
    const int qv = q[pos], v = abs(qv), level = min(v, 15);
    const int row = pos >> bwl, col = pos - (row << bwl);
    int b;
    if (c == eob - 1) {
        const int area = height << bwl;
        const int bctx = c == 0 ? 0 : c <= area / 8 ? 1 : c <= area / 4 ? 2 : 3;
        b = C[ci_base_eob(txSzCtx, ptype, bctx) + min(level, 3) - 1];
    } else {
        int mag = 0;
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const int rr = row + ST(Sig_Ref_Diff_Offset)[txClass][k][0], cc = col + ST(Sig_Ref_Diff_Offset)[txClass][k][1];
            if (rr < height && cc < width) mag += min(abs((int)q[(rr << bwl) + cc]), 3);
        }
        int bctx = min((mag + 1) >> 1, 4);
        if (txClass == AV1G_TX_CLASS_2D) bctx = (row == 0 && col == 0) ? 0 : bctx + T.baseCtx[txSz * 25 + min(row, 4) * 5 + min(col, 4)];
        else bctx += ST(Coeff_Base_Pos_Ctx_Offset)[min(txClass == AV1G_TX_CLASS_VERT ? row : col, 2)];
        b = C[ci_base(txSzCtx, ptype, bctx) + min(level, 3)];
    }
    if (level > 2) {
        int mag = 0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int rr = row + ST(Mag_Ref_Offset_With_Tx_Class)[txClass][k][0], cc = col + ST(Mag_Ref_Offset_With_Tx_Class)[txClass][k][1];
            if (rr < height && cc < width) mag += min(abs((int)q[rr * width + cc]), 15);
        }
        mag = min((mag + 1) >> 1, 6);
        const int brctx = pos == 0 ? mag
                        : txClass == AV1G_TX_CLASS_2D ? ((row < 2 && col < 2) ? mag + 7 : mag + 14)
                        : txClass == AV1G_TX_CLASS_HORIZ ? (col == 0 ? mag + 7 : mag + 14) : (row == 0 ? mag + 7 : mag + 14);
        const int cid = ci_br(min(txSzCtx, (int)AV1G_TX_32X32), ptype, brctx);
        int rem = level - 3;
        for (int i = 0; i < 4; i++) {
            const int k = min(rem, 3);
            b += C[cid + k];
            rem -= k;
            if (k < 3) break;
        }
    }
    if (v) {
        b += c == 0 ? C[ci_dc_sign(ptype, dcCtx) + (qv < 0)] : 256;
        if (v > 14) b += (2 * (31 - __clz(v - 14)) + 1) * 256;
    }
    return b;
}

// One evaluation (group of G lanes, all 32 lanes of the warp call it together with the same txSz): residual into
// buf, forward transform in place (columns, then rows), dead-zone quantisation into q (zbin 21/32, rounding 3/8 of
// the step, the reference's 0.656 / 0.375; levels capped at 16383), transform-domain distortion, exact rate.  The
// coefficients stay in buf (th x tw, row stride W + 1).
template <int BD, typename Px>
__device__ __noinline__ EvalOut grp_eval_x(int txSz, const Px *rsrc, int rsp, const Px *rpred, int rlw, const int32_t *rarr, int txType,
                                           int plane, int skipCtx, int dcCtx, int intraDir, int dcQ, int acQ, const uint16_t *cost,
                                           const uint16_t *scanT, const uint8_t *baseCtx, int32_t *buf, int16_t *q, int g, int G) {
    // the arguments come as scalars and the structures are rebuilt here, in registers: a structure passed by address
    // would live in the caller's local memory and be re-read after every store through buf / q
    const ResFn<Px> rf{rsrc, rsp, rpred, rlw, rarr};
    EvalIn e;
    e.txType = txType; e.plane = plane; e.skipCtx = skipCtx; e.dcCtx = dcCtx; e.intraDir = intraDir; e.dcQ = dcQ; e.acQ = acQ;
    e.T.cost = cost; e.T.scan = scanT; e.T.baseCtx = baseCtx;
    const TxRt d = tx_rt(txSz, BD);
    const int ck = col_kind(e.txType), rk = row_kind(e.txType);
    const bool big = d.W == 64 || d.H == 64;
    i64 en = 0;
    for (int j = g; j < d.W; j += G) {
        for (int i = 0; i < d.H; i++) {
            const int r = rf(i, j);
            en += r * r;
            buf[i * d.TS + j] = r;
        }
        fwd1d_mem(ck, d.H, buf + j, d.TS, d.s0, d.th, 0, d.s1);
    }
    __syncwarp();
    for (int i = g; i < d.th; i += G) fwd1d_mem(rk, d.W, buf + i * d.TS, 1, 0, d.tw, d.rect, d.s2);
    __syncwarp();
    const int den = dq_denom(txSz);
    i64 dist = 0, kept = 0;
    for (int idx = g; idx < d.n; idx += G) {
        const int v = buf[(idx >> d.ltw) * d.TS + (idx & (d.tw - 1))];
        const int step = idx == 0 ? e.dcQ : e.acQ;
        const int a = abs(v) * den, S = step << FB;
        int l = 0;
        if (a * 32 >= 21 * S) l = min((8 * a + 3 * S) / (8 * S), 16383);
        const int qv = v < 0 ? -l : l;
        q[idx] = (int16_t)qv;
        const int dq = l ? dequant<BD>(qv, step, den) * (1 << FB) : 0;
        const i64 df = (i64)(v - dq);
        dist += df * df;
        kept += (i64)v * v;
    }
    dist = grp_sum64(dist, G);
    __syncwarp();
    const uint16_t *scan = get_scan(e.T, txSz, e.txType);
    int last = 0;
    for (int c = g; c < d.n; c += G)
        if (q[scan[c]]) last = c + 1;
    const int eob = grp_max(last, G);
    int b = 0;
    const int cls = tx_class(e.txType);
    for (int c = g; c < eob; c += G) b += coeff_bits(c, eob, q, scan, txSz, cls, e.plane > 0, e.dcCtx, e.T);
    EvalOut o;
    o.R = grp_sum(b, G) + base_bits(txSz, e.txType, e.plane, e.skipCtx, e.intraDir, e.T.cost, eob);
    o.D = dist << d.dsh;
    if (big) {
        en = grp_sum64(en, G);
        kept = grp_sum64(kept, G);
        const i64 extra = (en << 16) - (kept << d.dsh);
        o.D += extra > 0 ? extra : 0;
    }
    o.eob = eob;
    return o;
}
template <int BD, typename Px>
__device__ __forceinline__ EvalOut grp_eval(int txSz, const ResFn<Px> &rf, const EvalIn &e, int32_t *buf, int16_t *q, int g, int G) {
    return grp_eval_x<BD, Px>(txSz, rf.src, rf.sp, rf.pred, rf.lw, rf.arr, e.txType, e.plane, e.skipCtx, e.dcCtx, e.intraDir, e.dcQ, e.acQ,
                              e.T.cost, e.T.scan, e.T.baseCtx, buf, q, g, G);
}

// ---------------------------------------------------------------------------------------------------------------
// exact inverse transform (spec 7.13.3, Lossless = 0) + conformance flags.  Rows on lanes, then columns on lanes
// (warp), residual rows stored in res (H x W int32 scratch).
// ---------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t inv_adst4(int32_t *T, int r) {   // spec 7.13.2.6 with its range checks
    const i64 s0 = 1321LL * T[0], s1 = 2482LL * T[0], s2 = 3344LL * T[1], s3 = 3803LL * T[2], s4 = 1321LL * T[2];
    const i64 s5 = 2482LL * T[3], s6 = 3803LL * T[3];
    const i64 a7 = (i64)T[0] - T[2], b7 = a7 + T[3];
    uint32_t e = 0;
    auto chk = [&](i64 v, int bits) { if (v < -(1LL << (bits - 1)) || v > (1LL << (bits - 1)) - 1) e |= 2; };
    chk(a7, r + 1); chk(b7, r);
    chk(s0, r + 12); chk(s1, r + 12); chk(s2, r + 12); chk(s3, r + 12); chk(s4, r + 12); chk(s5, r + 12); chk(s6, r + 12);
    i64 t0 = s0 + s3, t1 = s1 - s4, t3 = s2, t2 = 3344LL * b7;
    chk(t0, r + 12); chk(t1, r + 12); chk(t2, r + 12);
    t0 += s5; t1 -= s6;
    chk(t0, r + 12); chk(t1, r + 12);
    const i64 x0 = t0 + t3, x1 = t1 + t3, x2 = t2;
    i64 x3 = t0 + t1;
    chk(x3, r + 12);
    x3 -= t3;
    chk(x0, r + 12); chk(x1, r + 12); chk(x2, r + 12); chk(x3, r + 12);
    T[0] = (int32_t)((x0 + 2048) >> 12); T[1] = (int32_t)((x1 + 2048) >> 12);
    T[2] = (int32_t)((x2 + 2048) >> 12); T[3] = (int32_t)((x3 + 2048) >> 12);
    return e;
}
template <int N> __device__ __forceinline__ uint32_t inv1d(int kind, int32_t *T, int r) {
    if (N >= 32 || kind == 0) {
        if constexpr (N == 4) return inv_dct4(T, r);
        else if constexpr (N == 8) return inv_dct8(T, r);
        else if constexpr (N == 16) return inv_dct16(T, r);
        else if constexpr (N == 32) return inv_dct32(T, r);
        else return inv_dct64(T, r);
    } else if (kind == 1) {
        if constexpr (N == 4) return inv_adst4(T, r);
        else if constexpr (N == 8) return inv_adst8(T, r);
        else if constexpr (N == 16) return inv_adst16(T, r);
    } else {
#pragma unroll
        for (int i = 0; i < N; i++) {
            if constexpr (N == 4) T[i] = (int32_t)(((i64)T[i] * 5793 + 2048) >> 12);
            else if constexpr (N == 8) T[i] = T[i] * 2;
            else T[i] = (int32_t)(((i64)T[i] * 11586 + 2048) >> 12);
        }
    }
    return 0;
}
template <int N>
__device__ __forceinline__ uint32_t inv_mem_n(int kind, int32_t *p, int stride, int r, int preRect, int post, int clampBits) {
    int32_t T[N];
#pragma unroll
    for (int i = 0; i < N; i++) {
        T[i] = p[i * stride];
        if (preRect) T[i] = (int32_t)(((i64)T[i] * 2896 + 2048) >> 12);
    }
    const uint32_t e = inv1d<N>(kind, T, r);
#pragma unroll
    for (int i = 0; i < N; i++) {
        int32_t v = post ? (int32_t)(((i64)T[i] + (1 << (post - 1))) >> post) : T[i];
        if (clampBits) v = min(max(v, -(1 << (clampBits - 1))), (1 << (clampBits - 1)) - 1);
        p[i * stride] = v;
    }
    return e;
}
static __device__ __noinline__ uint32_t inv1d_mem(int kind, int n, int32_t *p, int stride, int r, int preRect, int post, int clampBits) {
    switch (n) {
    case 4: return inv_mem_n<4>(kind, p, stride, r, preRect, post, clampBits);
    case 8: return inv_mem_n<8>(kind, p, stride, r, preRect, post, clampBits);
    case 16: return inv_mem_n<16>(kind, p, stride, r, preRect, post, clampBits);
    case 32: return inv_mem_n<32>(0, p, stride, r, preRect, post, clampBits);
    default: return inv_mem_n<64>(0, p, stride, r, preRect, post, clampBits);
    }
}

// levels q (tw x th) -> residual in buf (H x W, row stride W + 1) of the spec's 2-D inverse (7.13.3, Lossless = 0:
// dequantisation, row transforms at BitDepth + 8 bits with the 2:1 rectangular scaling, Round2 by the row shift,
// clamp to colClampRange, column transforms, Round2(., 4)); returns the OR of the conformance flags (group)
template <int BD>
__device__ __noinline__ uint32_t grp_inverse(int txSz, const int16_t *q, int txType, int dcQ, int acQ, int32_t *buf, int g, int G) {
    const TxRt d = tx_rt(txSz, BD);
    constexpr int rowR = BD + 8, colR = (BD + 6) > 16 ? BD + 6 : 16;
    const int den = dq_denom(txSz);
    const int ck = col_kind(txType), rk = row_kind(txType);
    for (int p = g; p < d.W * d.H; p += G) {
        const int i = p >> d.lw, j = p & (d.W - 1);
        int v = 0;
        if (i < d.th && j < d.tw) {
            const int l = q[i * d.tw + j];
            v = l ? dequant<BD>(l, (i == 0 && j == 0) ? dcQ : acQ, den) : 0;
        }
        buf[i * d.TS + j] = v;
    }
    __syncwarp();
    uint32_t err = 0;
    for (int i = g; i < d.H; i += G) err |= inv1d_mem(rk, d.W, buf + i * d.TS, 1, rowR, d.rect, d.rowShift, colR);
    __syncwarp();
    for (int j = g; j < d.W; j += G) err |= inv1d_mem(ck, d.H, buf + j, d.TS, colR, 0, 4, 0);
    __syncwarp();
    return (uint32_t)grp_max((int)err, G);
}

// ---------------------------------------------------------------------------------------------------------------
// runtime dispatch over the 19 tx sizes (host-side self-checks)
// ---------------------------------------------------------------------------------------------------------------
#define IS_TX_SWITCH(txSz, M)            \
    switch (txSz) {                      \
    case AV1G_TX_4X4: M(4, 4); break;    \
    case AV1G_TX_8X8: M(8, 8); break;    \
    case AV1G_TX_16X16: M(16, 16); break; \
    case AV1G_TX_32X32: M(32, 32); break; \
    case AV1G_TX_64X64: M(64, 64); break; \
    case AV1G_TX_4X8: M(4, 8); break;    \
    case AV1G_TX_8X4: M(8, 4); break;    \
    case AV1G_TX_8X16: M(8, 16); break;  \
    case AV1G_TX_16X8: M(16, 8); break;  \
    case AV1G_TX_16X32: M(16, 32); break; \
    case AV1G_TX_32X16: M(32, 16); break; \
    case AV1G_TX_32X64: M(32, 64); break; \
    case AV1G_TX_64X32: M(64, 32); break; \
    case AV1G_TX_4X16: M(4, 16); break;  \
    case AV1G_TX_16X4: M(16, 4); break;  \
    case AV1G_TX_8X32: M(8, 32); break;  \
    case AV1G_TX_32X8: M(32, 8); break;  \
    case AV1G_TX_16X64: M(16, 64); break; \
    default: M(64, 16); break;           \
    }

}  // namespace is
