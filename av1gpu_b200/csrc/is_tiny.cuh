// is_tiny.cuh - open-loop analysis of the small blocks, one thread per block: 4x4, 4x8 and 8x4 with everything in
// registers (k_analysis_tiny); 8x8, 4x16 and 16x4 with the transform in registers and edges / levels in per-thread
// shared-memory slots (k_analysis_mid).
//
// The same search as an_block (the reference's k_analysis, encoder/src/k_analysis.cuh:496-689) for the three smallest
// shapes - 512 of the 836 analysed blocks of an SB.  A warp-per-block search leaves most lanes idle or divergent on
// blocks this small (13 candidates of one 4x4 sub-block each); here each thread owns one block, the geometry and the
// prediction angles are compile-time constants, so every array is a register array with static indices and the
// threads of a warp run the same instruction stream:
//   edges from the staged SB tile, DC value, SATD of the 13 modes at delta 0 (no angle deltas below 8x8), the top 4
//   kept with their predictions (insertion in cost order, earlier candidate first on ties), exact-rate RD of the top 4
//   with DCT_DCT, then the other tx types of the set for the winner.
// One CTA of 256 threads per SB: the 256 4x4 blocks, then the 128 4x8 (warps 0-3) and 128 8x4 blocks (warps 4-7).
#pragma once
#include "is_dev.cuh"
#include "is_frame.cuh"
#include "is_analysis.cuh"

namespace is {

// Spec constants used as compile-time indices: Sig_Ref_Diff_Offset, Mag_Ref_Offset_With_Tx_Class (spec 8.3.2 / the
// av1core tables; the library checks them against av1core's at upload) and Dr_Intra_Derivative at 23, 45, 67 degrees.
// (row, column) offset d of neighbour k for tx class c (0 2D, 1 HORIZ, 2 VERT)
__host__ __device__ constexpr int sig_ref(int c, int k, int d) {
    return k == 0 ? (d == 0 ? 0 : 1) : k == 1 ? (d == 0 ? 1 : 0)
         : c == 0 ? (k == 2 ? 1 : k == 3 ? (d == 0 ? 0 : 2) : (d == 0 ? 2 : 0))
         : c == 1 ? (d == 0 ? 0 : k) : (d == 0 ? k : 0);
}
__host__ __device__ constexpr int mag_ref(int c, int k, int d) {
    return k == 0 ? (d == 0 ? 0 : 1) : k == 1 ? (d == 0 ? 1 : 0)
         : c == 0 ? 1 : c == 1 ? (d == 0 ? 0 : 2) : (d == 0 ? 2 : 0);
}
constexpr int kDr23 = 151, kDr45 = 64, kDr67 = 27;

constexpr int TINY_THREADS = 256;
template <typename Px> struct TinySmem {      // Px: the sample type (uint8_t 8-bit, uint16_t 10-bit)
    static constexpr int TW = 144, TH = 65;   // the SB tile of the analysis (columns sbx-16 .., rows sby-1 ..)
    Px tile[TH * TW];
    uint8_t iscan[3][3][32];                  // scan position of each coefficient: (4x4, 4x8, 8x4) x (2D, HORIZ, VERT)
    RateStage T;
};

// ---- prediction of mode M at delta 0 of a W x H block; A[k + 1] = AboveRow[k], L[k + 1] = LeftCol[k], k >= -1 ----
template <int W, int H, int M>
__device__ __forceinline__ void tpred(const int *A, const int *L, int dcv, int *p) {
    constexpr int NE = W + H;
    if constexpr (M == AV1G_DC_PRED) {
#pragma unroll
        for (int k = 0; k < W * H; k++) p[k] = dcv;
    } else if constexpr (M == AV1G_V_PRED) {
#pragma unroll
        for (int i = 0; i < H; i++)
#pragma unroll
            for (int j = 0; j < W; j++) p[i * W + j] = A[1 + j];
    } else if constexpr (M == AV1G_H_PRED) {
#pragma unroll
        for (int i = 0; i < H; i++)
#pragma unroll
            for (int j = 0; j < W; j++) p[i * W + j] = L[1 + i];
    } else if constexpr (M == AV1G_D45_PRED || M == AV1G_D67_PRED) {   // 0 < angle < 90: the above row only
        constexpr int dx = M == AV1G_D45_PRED ? kDr45 : kDr67, maxBaseX = NE - 1;
#pragma unroll
        for (int i = 0; i < H; i++)
#pragma unroll
            for (int j = 0; j < W; j++) {
                const int idx = (i + 1) * dx, base = (idx >> 6) + j, sh = (idx >> 1) & 0x1F;
                p[i * W + j] = base < maxBaseX ? (A[1 + base] * (32 - sh) + A[2 + base] * sh + 16) >> 5 : A[1 + maxBaseX];
            }
    } else if constexpr (M == AV1G_D113_PRED || M == AV1G_D135_PRED || M == AV1G_D157_PRED) {   // 90 < angle < 180
        constexpr int dx = M == AV1G_D113_PRED ? kDr67 : M == AV1G_D135_PRED ? kDr45 : kDr23;
        constexpr int dy = M == AV1G_D113_PRED ? kDr23 : M == AV1G_D135_PRED ? kDr45 : kDr67;
#pragma unroll
        for (int i = 0; i < H; i++)
#pragma unroll
            for (int j = 0; j < W; j++) {
                const int ia = (j << 6) - (i + 1) * dx, ba = ia >> 6;
                if (ba >= -1) {
                    const int sh = (ia >> 1) & 0x1F;
                    p[i * W + j] = (A[1 + ba] * (32 - sh) + A[2 + ba] * sh + 16) >> 5;
                } else {
                    const int il = (i << 6) - (j + 1) * dy, bl = il >> 6, sh = (il >> 1) & 0x1F;
                    p[i * W + j] = (L[1 + bl] * (32 - sh) + L[2 + bl] * sh + 16) >> 5;
                }
            }
    } else if constexpr (M == AV1G_D203_PRED) {   // 180 < angle < 270: the left column only
        constexpr int dy = kDr67;
#pragma unroll
        for (int i = 0; i < H; i++)
#pragma unroll
            for (int j = 0; j < W; j++) {
                const int idx = (j + 1) * dy, base = (idx >> 6) + i, sh = (idx >> 1) & 0x1F;
                p[i * W + j] = (L[1 + base] * (32 - sh) + L[2 + base] * sh + 16) >> 5;
            }
    } else if constexpr (M == AV1G_PAETH_PRED) {
        const int tl = A[0];
#pragma unroll
        for (int i = 0; i < H; i++)
#pragma unroll
            for (int j = 0; j < W; j++) {
                const int a = A[1 + j], l = L[1 + i], base = a + l - tl;
                const int pL = abs(base - l), pT = abs(base - a), pTL = abs(base - tl);
                p[i * W + j] = (pL <= pT && pL <= pTL) ? l : pT <= pTL ? a : tl;
            }
    } else {   // SMOOTH, SMOOTH_V, SMOOTH_H
        const uint8_t *wx = W == 4 ? ST(Sm_Weights_Tx_4x4) : ST(Sm_Weights_Tx_8x8);
        const uint8_t *wy = H == 4 ? ST(Sm_Weights_Tx_4x4) : ST(Sm_Weights_Tx_8x8);
        const int bl = L[H], tr = A[W];
        constexpr int sh = M == AV1G_SMOOTH_PRED ? 9 : 8;
#pragma unroll
        for (int i = 0; i < H; i++)
#pragma unroll
            for (int j = 0; j < W; j++) {
                const int v = M != AV1G_SMOOTH_H_PRED ? wy[i] * A[1 + j] + (256 - wy[i]) * bl : 0;
                const int hz = M != AV1G_SMOOTH_V_PRED ? wx[j] * L[1 + i] + (256 - wx[j]) * tr : 0;
                p[i * W + j] = (v + hz + (1 << (sh - 1))) >> sh;
            }
    }
}

// ---- rate of the levels q (natural order) of a 4- or 8-point tx block of class CLS: coeff_bits over the scan
// positions c < eob, walked in natural order through the inverse scan ----
template <int LW, int LH, int CLS>
__device__ __forceinline__ int tcoeff_rate(const int *q, const uint8_t *iscan, int eob, int txSz, int ptype, int dcCtx, const RateTabs &T) {
    constexpr int W = 1 << LW, H = 1 << LH, N = W * H;
    const uint16_t *C = T.cost;
    const int txSzCtx = (ST(Tx_Size_Sqr)[txSz] + ST(Tx_Size_Sqr_Up)[txSz] + 1) >> 1;
    int b = 0;
#pragma unroll
    for (int pos = 0; pos < N; pos++) {
        const int c = iscan[pos];
        if (c >= eob) continue;
        const int row = pos >> LW, col = pos & (W - 1);
        const int qv = q[pos], v = abs(qv), level = min(v, 15);
        int bb;
        if (c == eob - 1) {
            const int bctx = c == 0 ? 0 : c <= N / 8 ? 1 : c <= N / 4 ? 2 : 3;
            bb = C[ci_base_eob(txSzCtx, ptype, bctx) + min(level, 3) - 1];
        } else {
            int mag = 0;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                const int rr = row + sig_ref(CLS, k, 0), cc = col + sig_ref(CLS, k, 1);
                if (rr < H && cc < W) mag += min(abs(q[rr * W + cc]), 3);
            }
            int bctx = min((mag + 1) >> 1, 4);
            if (CLS == AV1G_TX_CLASS_2D) bctx = pos == 0 ? 0 : bctx + T.baseCtx[txSz * 25 + min(row, 4) * 5 + min(col, 4)];
            else bctx += ST(Coeff_Base_Pos_Ctx_Offset)[min(CLS == AV1G_TX_CLASS_VERT ? row : col, 2)];
            bb = C[ci_base(txSzCtx, ptype, bctx) + min(level, 3)];
        }
        if (level > 2) {
            int mag = 0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const int rr = row + mag_ref(CLS, k, 0), cc = col + mag_ref(CLS, k, 1);
                if (rr < H && cc < W) mag += min(abs(q[rr * W + cc]), 15);
            }
            mag = min((mag + 1) >> 1, 6);
            const int brctx = pos == 0 ? mag
                            : CLS == AV1G_TX_CLASS_2D ? ((row < 2 && col < 2) ? mag + 7 : mag + 14)
                            : CLS == AV1G_TX_CLASS_HORIZ ? (col == 0 ? mag + 7 : mag + 14) : (row == 0 ? mag + 7 : mag + 14);
            const int cid = ci_br(min(txSzCtx, (int)AV1G_TX_32X32), ptype, brctx);
            int rem = level - 3;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int k = min(rem, 3);
                bb += C[cid + k];
                rem -= k;
                if (k < 3) break;
            }
        }
        if (v) {
            bb += c == 0 ? C[ci_dc_sign(ptype, dcCtx) + (qv < 0)] : 256;
            if (v > 14) bb += (2 * (31 - __clz(v - 14)) + 1) * 256;
        }
        b += bb;
    }
    return b;
}

// ---- one evaluation by one thread (grp_eval's arithmetic for a 4- or 8-point tx size): forward transform of the
// residual, dead-zone quantisation into q, transform-domain distortion, exact rate ----
template <int BD, int LW, int LH>
__device__ __forceinline__ EvalOut thr_eval(int txSz, const int *res, const EvalIn &e, const uint8_t *iscan, int istride, int *q) {
    constexpr int W = 1 << LW, H = 1 << LH, N = W * H;
    const int rowShift = ST(Transform_Row_Shift)[txSz];
    constexpr int rect = (LW - LH == 1 || LH - LW == 1) ? 1 : 0;
    const int E = rowShift + 4 + FB - (LW + LH - 2);
    const int s0 = max(0, 17 - BD - LH), s2 = s0 - LW - E;
    const int dsh = 16 - 2 * FB - (2 * (rowShift + 4) - (LW + LH - 2) + rect);
    const int ck = col_kind(e.txType), rk = row_kind(e.txType);
    int buf[N];
#pragma unroll
    for (int j = 0; j < W; j++) {
        int t[H];
#pragma unroll
        for (int i = 0; i < H; i++) t[i] = res[i * W + j] * (1 << s0);
        fwd1d<H>(ck, t);
#pragma unroll
        for (int i = 0; i < H; i++) buf[i * W + j] = (t[i] + (1 << (LW - 1))) >> LW;
    }
#pragma unroll
    for (int i = 0; i < H; i++) {
        int t[W];
#pragma unroll
        for (int j = 0; j < W; j++) t[j] = buf[i * W + j];
        fwd1d<W>(rk, t);
#pragma unroll
        for (int j = 0; j < W; j++) {
            int v = t[j];
            if (rect) v = (v * 5793 + 2048) >> 12;
            buf[i * W + j] = s2 > 0 ? (v + (1 << (s2 - 1))) >> s2 : v * (1 << -s2);
        }
    }
    const int cls = e.txType == AV1G_IDTX ? AV1G_TX_CLASS_2D : tx_class(e.txType);
    const uint8_t *isc = iscan + cls * istride;
    i64 dist = 0;
    int eob = 0;
#pragma unroll
    for (int idx = 0; idx < N; idx++) {
        const int v = buf[idx];
        const int step = idx == 0 ? e.dcQ : e.acQ;
        const int a = abs(v), S = step << FB;   // dequantisation denominator 1 for these sizes
        int l = 0;
        if (a * 32 >= 21 * S) l = min((8 * a + 3 * S) / (8 * S), 16383);
        const int qv = v < 0 ? -l : l;
        q[idx] = qv;
        const int dq = l ? dequant<BD>(qv, step, 1) * (1 << FB) : 0;
        const i64 df = (i64)(v - dq);
        dist += df * df;
        if (qv) eob = max(eob, isc[idx] + 1);
    }
    int b = 0;
    if (eob) {
        const int ptype = e.plane > 0;
        if (cls == AV1G_TX_CLASS_2D) b = tcoeff_rate<LW, LH, AV1G_TX_CLASS_2D>(q, isc, eob, txSz, ptype, e.dcCtx, e.T);
        else if (cls == AV1G_TX_CLASS_HORIZ) b = tcoeff_rate<LW, LH, AV1G_TX_CLASS_HORIZ>(q, isc, eob, txSz, ptype, e.dcCtx, e.T);
        else b = tcoeff_rate<LW, LH, AV1G_TX_CLASS_VERT>(q, isc, eob, txSz, ptype, e.dcCtx, e.T);
    }
    EvalOut o;
    o.R = b + base_bits_inl(txSz, e, eob);
    o.D = dist << dsh;
    o.eob = eob;
    return o;
}

// ---- the search of one W x H block (bs) at (x, y), one thread ----
template <int BD, int LW, int LH, typename Px>
__device__ __forceinline__ void tiny_block(const FrameDesc &F, const TinySmem<Px> &S, const RateTabs &T, int bs, int txSz, int sizeIdx, int x,
                                           int y, int sbx, int sby, int tx0, int ty0, int tx1, int ty1) {
    constexpr int W = 1 << LW, H = 1 << LH, N = W * H, NE = W + H;
    constexpr int TW = TinySmem<Px>::TW;
    // the kept predictions are packed PPW samples to a 32-bit word: 4 bytes (8-bit), 2 halves (10-bit)
    constexpr int PPW = sizeof(Px) == 1 ? 4 : 2, PB = 32 / PPW, NWD = N / PPW;
    constexpr uint32_t PMASK = (1u << PB) - 1u;
    const Px *tile = S.tile;
    const int haveL = x > tx0, haveA = y > ty0;
    const int haveAR = ol_decoded(x + W, y - 1, x, y, tx0, ty0, tx1, ty1), haveBL = ol_decoded(x - 1, y + H, x, y, tx0, ty0, tx1, ty1);
    const int lx = x - sbx + 16, ly = y - sby + 1;
    const int mX = F.MiCols * 4 - 1 - sbx + 16, mY = F.MiRows * 4 - 1 - sby + 1;
    // edges (build_edges on the tile)
    int A[NE + 1], L[NE + 1];
    {
        const int alim = min(lx + (haveAR ? 2 * W : W) - 1, mX), llim = min(ly + (haveBL ? 2 * H : H) - 1, mY);
        const int dA = haveL ? tile[ly * TW + lx - 1] : (1 << (BD - 1)) - 1;
        const int dL = haveA ? tile[(ly - 1) * TW + lx] : (1 << (BD - 1)) + 1;
#pragma unroll
        for (int k = 0; k < NE; k++) {
            A[k + 1] = haveA ? tile[(ly - 1) * TW + min(lx + k, alim)] : dA;
            L[k + 1] = haveL ? tile[min(ly + k, llim) * TW + lx - 1] : dL;
        }
        const int c = (haveA && haveL) ? tile[(ly - 1) * TW + lx - 1] : haveA ? tile[(ly - 1) * TW + lx] : haveL ? tile[ly * TW + lx - 1]
                                                                                                             : (1 << (BD - 1));
        A[0] = c;
        L[0] = c;
    }
    int dcv;
    {
        int sa = 0, sl = 0;
#pragma unroll
        for (int k = 0; k < W; k++) sa += A[1 + k];
#pragma unroll
        for (int k = 0; k < H; k++) sl += L[1 + k];
        if (haveL && haveA) dcv = (sa + sl + (NE >> 1)) / NE;
        else if (haveL) dcv = min((sl + (H >> 1)) >> LH, (1 << BD) - 1);
        else if (haveA) dcv = min((sa + (W >> 1)) >> LW, (1 << BD) - 1);
        else dcv = 1 << (BD - 1);
    }
    int src[N];
#pragma unroll
    for (int i = 0; i < H; i++)
#pragma unroll
        for (int j = 0; j < W; j++) src[i * W + j] = tile[(ly + i) * TW + lx + j];
    // ---- SATD screening of the 13 modes; the 4 best kept in cost order with their predictions (packed) ----
    i64 topJ[4];
    int topM[4];
    uint32_t topP[4][NWD];
#pragma unroll
    for (int k = 0; k < 4; k++) { topJ[k] = INF; topM[k] = 0; }
    auto screen = [&](auto modeTag) {
        constexpr int M = decltype(modeTag)::value;
        int p[N];
        tpred<W, H, M>(A, L, dcv, p);
        int satd = 0;
#pragma unroll
        for (int sy = 0; sy < H; sy += 4)
#pragma unroll
            for (int sx = 0; sx < W; sx += 4) {
                int d[16];
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) d[i * 4 + j] = src[(sy + i) * W + sx + j] - p[(sy + i) * W + sx + j];
                satd += hadamard4_sum(d);
            }
        const i64 js = ((i64)satd << 14) + F.sqlam * c_avgY[M];
        uint32_t pk[NWD];
#pragma unroll
        for (int k = 0; k < NWD; k++) {
            uint32_t v = 0;
#pragma unroll
            for (int u = 0; u < PPW; u++) v |= (uint32_t)p[PPW * k + u] << (PB * u);
            pk[k] = v;
        }
        // insertion: after every kept entry of cost <= js (the earlier candidate wins a tie)
        const int pos = (topJ[0] <= js) + (topJ[1] <= js) + (topJ[2] <= js) + (topJ[3] <= js);
#pragma unroll
        for (int s = 3; s >= 0; s--) {
            if (s > pos) {
                topJ[s] = topJ[s - 1 < 0 ? 0 : s - 1];
                topM[s] = topM[s - 1 < 0 ? 0 : s - 1];
#pragma unroll
                for (int k = 0; k < NWD; k++) topP[s][k] = topP[s - 1 < 0 ? 0 : s - 1][k];
            } else if (s == pos) {
                topJ[s] = js;
                topM[s] = M;
#pragma unroll
                for (int k = 0; k < NWD; k++) topP[s][k] = pk[k];
            }
        }
    };
    screen(std::integral_constant<int, 0>{});
    screen(std::integral_constant<int, 1>{});
    screen(std::integral_constant<int, 2>{});
    screen(std::integral_constant<int, 3>{});
    screen(std::integral_constant<int, 4>{});
    screen(std::integral_constant<int, 5>{});
    screen(std::integral_constant<int, 6>{});
    screen(std::integral_constant<int, 7>{});
    screen(std::integral_constant<int, 8>{});
    screen(std::integral_constant<int, 9>{});
    screen(std::integral_constant<int, 10>{});
    screen(std::integral_constant<int, 11>{});
    screen(std::integral_constant<int, 12>{});
    // ---- RD: the top 4 with DCT_DCT, then the other types of the set for the winner (first of equal costs wins) ----
    const bool hasC = has_chroma(bs, y >> 2, x >> 2, F.ssx);
    const int overhead = (hasC ? UV_OVERHEAD : 0) + c_avgSkip0;
    const uint8_t *iscan = &S.iscan[sizeIdx][0][0];
    auto rd = [&](const uint32_t *pw, int m, int t) -> i64 {
        int res[N], q[N];
#pragma unroll
        for (int i = 0; i < N; i++) res[i] = src[i] - (int)((pw[i / PPW] >> (PB * (i % PPW))) & PMASK);
        const EvalIn e{t, 0, 0, 0, m, F.dcQ, F.acQ, T};
        const EvalOut o = thr_eval<BD, LW, LH>(txSz, res, e, iscan, 32, q);
        return o.D + F.lam * (o.R + c_avgY[m] + overhead);
    };
    i64 bestJ = INF;
    int bestK = 0, bestTx = AV1G_DCT_DCT;
    const int kMax = F.rdK;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (topJ[k] == INF || k >= kMax) continue;   // fewer candidates screened or taken (shortlist)
        const i64 j = rd(topP[k], topM[k], AV1G_DCT_DCT);
        if (j < bestJ) { bestJ = j; bestK = k; }
    }
    // the winner's prediction and mode (static register indices for the type loop)
    uint32_t wp[NWD];
    int wm = topM[0];
#pragma unroll
    for (int k = 0; k < NWD; k++) wp[k] = topP[0][k];
#pragma unroll
    for (int s = 1; s < 4; s++)
        if (bestK == s) {
            wm = topM[s];
#pragma unroll
            for (int k = 0; k < NWD; k++) wp[k] = topP[s][k];
        }
    // 4- and 8-point sizes are in TX_SET_INTRA_1: IDTX, DCT_DCT, V_DCT, H_DCT, ADST_ADST, ADST_DCT, DCT_ADST
    TxRank rank;
    rank.add(bestJ, AV1G_DCT_DCT);
#pragma unroll 1
    for (int t = 1; t < 16; t++) {
        if (!tx_in_set(AV1G_TX_SET_INTRA_1, t)) continue;
        const i64 j = rd(wp, wm, t);
        if (j < bestJ) { bestJ = j; bestTx = t; }
        rank.add(j, t);
    }
    BlockRes r;
    r.J = bestJ;
    r.tx = (uint8_t)bestTx;
    r.cand[0] = (uint8_t)cand_pack(wm, 0);
    r.cand[1] = r.cand[2] = r.cand[3] = 0;
    int n = 1;
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (k != bestK && topJ[k] < INF && k < kMax) r.cand[n++ & 3] = (uint8_t)cand_pack(topM[k], 0);
    r.ncand = (uint8_t)n;
    r.txMask = rank.mask(F.txKeep);
    F.blk[F.shOff[bs] + (uint32_t)(y >> LH) * F.shNbx[bs] + (x >> LW)] = r;
}

// 8-bit: two CTAs per SM (128 registers a thread, some spilled) ran 2 % faster than one CTA with 255 registers; the
// 10-bit instance keeps one CTA per SM (with 128 registers it spills more than 6 KB a thread)
template <int BD>
__global__ void __launch_bounds__(TINY_THREADS, BD == 8 ? 2 : 1) k_analysis_tiny(const __grid_constant__ FrameDesc F) {
    typedef typename std::conditional<BD == 8, uint8_t, uint16_t>::type Px;
    typedef TinySmem<Px> Sm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Sm &S = *reinterpret_cast<Sm *>(smem_raw);
    const int sb = blockIdx.x, sbr = sb / F.sbCols, sbc = sb % F.sbCols;
    const int sbx = sbc * 64, sby = sbr * 64;
    const int tid = threadIdx.x;
    if (F.poison) {
        smem_poison(smem_raw, sizeof(Sm), tid, TINY_THREADS);
        __syncthreads();
    }
    {   // the SB tile (as an_sb), the rate tables, the inverse scans of the three sizes
        constexpr int V = Sm::TW * (int)sizeof(Px) / 16;
        const Px *s0 = (const Px *)F.src[0] + (size_t)(sby - 1) * F.spitch[0] + (sbx - 16);
        for (int k = tid; k < Sm::TH * V; k += TINY_THREADS) {
            const int r = k / V, c = k % V;
            reinterpret_cast<uint4 *>(S.tile + r * Sm::TW)[c] = __ldg(reinterpret_cast<const uint4 *>(s0 + (size_t)r * F.spitch[0]) + c);
        }
    }
    const RateTabs T = rate_tabs_stage(S.T, F.qctx, tid, TINY_THREADS);
    __syncthreads();
    for (int k = tid; k < 3 * 3 * 32; k += TINY_THREADS) {
        const int si = k / 96, cls = (k / 32) % 3, c = k % 32;
        const int txSz = si == 0 ? AV1G_TX_4X4 : si == 1 ? AV1G_TX_4X8 : AV1G_TX_8X4;
        if (c < (si == 0 ? 16 : 32)) S.iscan[si][cls][T.scan[c_scanOff[txSz][cls] + c]] = (uint8_t)c;
    }
    __syncthreads();
    int tc = 0, tr = 0;
    while (tc + 1 < F.tileCols && sbx >= F.tileColStart[tc + 1] * 4) tc++;
    while (tr + 1 < F.tileRows && sby >= F.tileRowStart[tr + 1] * 4) tr++;
    const int tx0 = F.tileColStart[tc] * 4, tx1 = F.tileColStart[tc + 1] * 4, ty0 = F.tileRowStart[tr] * 4, ty1 = F.tileRowStart[tr + 1] * 4;
    const int FW = F.MiCols * 4, FH = F.MiRows * 4;
    {   // 4x4: thread = (column, row) of the 16 x 16 grid
        const int x = sbx + (tid & 15) * 4, y = sby + (tid >> 4) * 4;
        if (x < FW && y < FH) tiny_block<BD, 2, 2>(F, S, T, AV1G_BLOCK_4X4, AV1G_TX_4X4, 0, x, y, sbx, sby, tx0, ty0, tx1, ty1);
    }
    if (tid < 128) {   // 4x8: 16 columns x 8 rows
        const int x = sbx + (tid & 15) * 4, y = sby + (tid >> 4) * 8;
        if (x < FW && y < FH) tiny_block<BD, 2, 3>(F, S, T, AV1G_BLOCK_4X8, AV1G_TX_4X8, 1, x, y, sbx, sby, tx0, ty0, tx1, ty1);
    } else {           // 8x4: 8 columns x 16 rows
        const int t = tid - 128, x = sbx + (t & 7) * 8, y = sby + (t >> 3) * 4;
        if (x < FW && y < FH) tiny_block<BD, 3, 2>(F, S, T, AV1G_BLOCK_8X4, AV1G_TX_8X4, 2, x, y, sbx, sby, tx0, ty0, tx1, ty1);
    }
}


// ================================================================================================================
// 8x8, 4x16 and 16x4: one thread per block.  Angle deltas (+-1..3 around the two best directional modes) make the
// prediction angles run-time values, so the edges live in a per-thread shared-memory slot and the prediction is
// pred4's sub-block code; every candidate and every RD task goes through ONE loop body (one copy of the prediction, the
// transform and the rate in the binary).  Levels go to a per-thread slot for the rate's context reads.
// ================================================================================================================
// One CTA runs ONE shape on the 64 blocks of each of MID_SBS superblocks, so that all its warps (and the co-resident
// CTAs, which the grid order gives the same shape) share one instruction stream.
constexpr int MID_SBS = 3, MID_THREADS = 64 * MID_SBS;
template <typename Px> struct MidSmem {   // Px: the sample type
    static constexpr int TW = 144, TH = 65;
    Px tile[MID_SBS][TH * TW];
    uint8_t iscan[3][64];                // the shape's tx size x (2D, HORIZ, VERT)
    Px edge[MID_THREADS][2][24];         // per thread: AboveRow[-1 .. 22], LeftCol[-1 .. 22]
    int16_t q[MID_THREADS][64];          // per thread: levels of the evaluation in progress
    RateStage T;
};

// forward transform of an N = W x H residual block in registers (grp_eval's column and row passes with their shifts)
template <int BD, int LW, int LH>
__device__ __forceinline__ void thr_fwd(int txSz, int txType, const int *res, int *buf) {
    constexpr int W = 1 << LW, H = 1 << LH;
    const int rowShift = ST(Transform_Row_Shift)[txSz];
    constexpr int rect = (LW - LH == 1 || LH - LW == 1) ? 1 : 0;
    const int E = rowShift + 4 + FB - (LW + LH - 2);
    const int s0 = max(0, 17 - BD - LH), s2 = s0 - LW - E;
    const int ck = col_kind(txType), rk = row_kind(txType);
#pragma unroll
    for (int j = 0; j < W; j++) {
        int t[H];
#pragma unroll
        for (int i = 0; i < H; i++) t[i] = res[i * W + j] * (1 << s0);
        fwd1d<H>(ck, t);
#pragma unroll
        for (int i = 0; i < H; i++) buf[i * W + j] = (t[i] + (1 << (LW - 1))) >> LW;
    }
#pragma unroll
    for (int i = 0; i < H; i++) {
        int t[W];
#pragma unroll
        for (int j = 0; j < W; j++) t[j] = buf[i * W + j];
        fwd1d<W>(rk, t);
#pragma unroll
        for (int j = 0; j < W; j++) {
            int v = t[j];
            if (rect) v = (v * 5793 + 2048) >> 12;
            buf[i * W + j] = s2 > 0 ? (v + (1 << (s2 - 1))) >> s2 : v * (1 << -s2);
        }
    }
}

// one evaluation of a <= 16-point-side block by one thread: transform in registers, levels to qs (shared memory),
// rate by coeff_bits over the scan
template <int BD, int LW, int LH>
__device__ __forceinline__ EvalOut mid_eval(int txSz, const int *res, const EvalIn &e, const uint8_t *iscan, int istride, int16_t *qs) {
    constexpr int W = 1 << LW, H = 1 << LH, N = W * H;
    int buf[N];
    thr_fwd<BD, LW, LH>(txSz, e.txType, res, buf);
    const int rowShift = ST(Transform_Row_Shift)[txSz];
    constexpr int rect = (LW - LH == 1 || LH - LW == 1) ? 1 : 0;
    const int dsh = 16 - 2 * FB - (2 * (rowShift + 4) - (LW + LH - 2) + rect);
    const int cls = e.txType == AV1G_IDTX ? AV1G_TX_CLASS_2D : tx_class(e.txType);
    const uint8_t *isc = iscan + cls * istride;
    i64 dist = 0;
    int eob = 0;
#pragma unroll
    for (int idx = 0; idx < N; idx++) {
        const int v = buf[idx];
        const int step = idx == 0 ? e.dcQ : e.acQ;
        const int a = abs(v), S = step << FB;   // dequantisation denominator 1 for these sizes
        int l = 0;
        if (a * 32 >= 21 * S) l = min((8 * a + 3 * S) / (8 * S), 16383);
        const int qv = v < 0 ? -l : l;
        qs[idx] = (int16_t)qv;
        const int dq = l ? dequant<BD>(qv, step, 1) * (1 << FB) : 0;
        const i64 df = (i64)(v - dq);
        dist += df * df;
        if (qv) eob = max(eob, isc[idx] + 1);
    }
    const uint16_t *scan = get_scan(e.T, txSz, e.txType);
    int b = 0;
    for (int c = 0; c < eob; c++) b += coeff_bits(c, eob, qs, scan, txSz, cls, e.plane > 0, e.dcCtx, e.T);
    EvalOut o;
    o.R = b + base_bits_inl(txSz, e, eob);
    o.D = dist << dsh;
    o.eob = eob;
    return o;
}

template <int BD, int LW, int LH, typename Px>
__device__ __forceinline__ void mid_block(const FrameDesc &F, MidSmem<Px> &S, const RateTabs &T, int bs, int txSz, const Px *tile, int x,
                                          int y, int sbx, int sby, int tx0, int ty0, int tx1, int ty1) {
    constexpr int W = 1 << LW, H = 1 << LH, N = W * H, NE = W + H;
    constexpr int TW = MidSmem<Px>::TW;
    const int tid = threadIdx.x;
    const int haveL = x > tx0, haveA = y > ty0;
    const int haveAR = ol_decoded(x + W, y - 1, x, y, tx0, ty0, tx1, ty1), haveBL = ol_decoded(x - 1, y + H, x, y, tx0, ty0, tx1, ty1);
    const int lx = x - sbx + 16, ly = y - sby + 1;
    const int mX = F.MiCols * 4 - 1 - sbx + 16, mY = F.MiRows * 4 - 1 - sby + 1;
    Px *A = S.edge[tid][0] + 1, *L = S.edge[tid][1] + 1;
    build_edges<BD>(tile, TW, lx, ly, W, H, haveL, haveA, haveAR, haveBL, mX, mY, A, L, 0, 1);
    int dcv;
    {
        int sa = 0, sl = 0;
#pragma unroll
        for (int k = 0; k < W; k++) sa += A[k];
#pragma unroll
        for (int k = 0; k < H; k++) sl += L[k];
        if (haveL && haveA) dcv = (sa + sl + (NE >> 1)) / NE;
        else if (haveL) dcv = min((sl + (H >> 1)) >> LH, (1 << BD) - 1);
        else if (haveA) dcv = min((sa + (W >> 1)) >> LW, (1 << BD) - 1);
        else dcv = 1 << (BD - 1);
    }
    const Px *src = tile + ly * TW + lx;
    const uint16_t *C = T.cost;
    auto mbits = [&](int c) -> int {
        const int m = cand_mode(c);
        int b = c_avgY[m];
        if (is_dir(m)) b += C[ci_angle(m - AV1G_V_PRED) + cand_delta(c) + 3];
        return b;
    };
    const bool hasC = has_chroma(bs, y >> 2, x >> 2, F.ssx);
    const int overhead = (hasC ? UV_OVERHEAD : 0) + c_avgSkip0;
    const uint8_t *iscan = &S.iscan[0][0];
    int16_t *qs = S.q[tid];
    i64 topJ[4] = {INF, INF, INF, INF};
    int topC[4] = {0, 0, 0, 0};
    i64 dJ0 = INF, dJ1 = INF;
    int b0 = AV1G_V_PRED, b1 = AV1G_V_PRED;
    i64 bestJ = INF;
    int bestK = 0, bestTx = AV1G_DCT_DCT, winC = 0;
    // a block with a learned shortlist screens its (mode, delta) list (most probable first) instead of the 13 modes and
    // the deltas, and tries only its list's tx types
    const SlCand *slc = (F.slCand && F.slIdx[bs] >= 0) ? F.slCand + F.slIdx[bs] + (uint32_t)(y >> LH) * F.shNbx[bs] + (x >> LW) : nullptr;
    const uint2 slw = slc ? *reinterpret_cast<const uint2 *>(slc->c) : make_uint2(0u, 0u);
    const int nsl = slc ? slc->n : 0;
    const uint32_t slTx = slc ? slc->txMask : 0u;
    const int kMax = nsl > 0 ? F.slRdK : F.rdK;
    TxRank rank;   // the winner's types by cost (txKeep)
    // jobs: 0-12 the 13 modes (a shortlisted block: its list's entries 0-7), 13-24 the deltas of the two best
    // directional modes (SATD); 25-28 the top 4 with DCT_DCT, 29-34 the other types of TX_SET_INTRA_1 for the winner (a
    // shortlisted block: the types of its list, in type order) (RD); a job no thread of the warp needs is skipped
#pragma unroll 1
    for (int job = 0; job < 35; job++) {
        int c, t = AV1G_DCT_DCT;
        bool need;
        if (job < 13) {
            c = nsl > 0 ? (int)(((job < 4 ? slw.x >> (8 * job) : slw.y >> (8 * (job - 4)))) & 0xFFu) : cand_pack(job, 0);
            need = nsl > 0 ? job < nsl && job < 8 : true;
        } else if (job < 25) {
            const int k = job - 13, kk = k % 6;
            c = cand_pack(k < 6 ? b0 : b1, kk < 3 ? -(kk + 1) : kk - 2);
        } else if (job < 29) {
            const int k = job - 25;
            c = topC[0];
#pragma unroll
            for (int s = 1; s < 4; s++) if (k == s) c = topC[s];
        } else {
            c = winC;
            const int k = job - 29;   // ADST_DCT, DCT_ADST, ADST_ADST, IDTX, V_DCT, H_DCT
            t = k < 3 ? k + 1 : k + 6;
            if (slTx) {   // the k-th type of the list beyond DCT_DCT
                const uint32_t m = slTx & ~1u;
                t = k < __popc(m) ? (int)__fns(m, 0, k + 1) : -1;
            }
        }
        if (job >= 13)
            need = job < 25 ? ((job - 13 < 6) ? dJ0 < INF : dJ1 < INF) : job < 29 ? (topJ[job - 25] < INF && job - 25 < kMax) : t >= 0;
        if (!__any_sync(__activemask(), need)) continue;
        if (t < 0) t = AV1G_DCT_DCT;   // (a thread past its list's types: its result is not used)
        const int m = cand_mode(c), pa = pangle(m, cand_delta(c));
        // the prediction, one 4x4 sub-block at a time (one copy of the predictor): SATD of the residual while screening,
        // the prediction into the thread's slot for an RD task
        int satd = 0;
#pragma unroll 1
        for (int k = 0; k < N / 16; k++) {
            const int sy = (k >> (LW - 2)) * 4, sx = (k & ((W >> 2) - 1)) * 4;
            int p[16];
            pred4_inl(m, pa, sy, sx, LW, LH, A, L, dcv, p);
            if (job < 25) {
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) p[i * 4 + j] = (int)src[(sy + i) * TW + sx + j] - p[i * 4 + j];
                satd += hadamard4_sum(p);
            } else {
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) qs[(sy + i) * W + sx + j] = (int16_t)p[i * 4 + j];
            }
        }
        if (job < 25) {
            const i64 js = ((i64)satd << 14) + F.sqlam * mbits(c);
            const int pos = need ? (topJ[0] <= js) + (topJ[1] <= js) + (topJ[2] <= js) + (topJ[3] <= js) : 4;
#pragma unroll
            for (int s = 3; s >= 0; s--) {
                if (s > pos) { topJ[s] = topJ[s > 0 ? s - 1 : 0]; topC[s] = topC[s > 0 ? s - 1 : 0]; }
                else if (s == pos) { topJ[s] = js; topC[s] = c; }
            }
            if (need && nsl == 0 && job >= AV1G_V_PRED && job <= AV1G_D67_PRED) {   // the two best directional modes (first of equals)
                if (js < dJ0) { dJ1 = dJ0; b1 = b0; dJ0 = js; b0 = job; }
                else if (js < dJ1) { dJ1 = js; b1 = job; }
            }
        } else {
            int res[N];
#pragma unroll
            for (int i = 0; i < H; i++)
#pragma unroll
                for (int j = 0; j < W; j++) res[i * W + j] = (int)src[i * TW + j] - qs[i * W + j];
            const EvalIn e{t, 0, 0, 0, m, F.dcQ, F.acQ, T};
            const EvalOut o = mid_eval<BD, LW, LH>(txSz, res, e, iscan, 64, qs);
            const i64 J = o.D + F.lam * (o.R + mbits(c) + overhead);
            if (need && job == 29) rank.add(bestJ, AV1G_DCT_DCT);   // the winner's DCT_DCT cost, before its other types
            if (need && job >= 29) rank.add(J, t);
            if (need && J < bestJ) {
                bestJ = J;
                if (job < 29) { bestK = job - 25; winC = c; }
                else bestTx = t;
            }
        }
    }
    if (rank.j[0] >= INF) rank.add(bestJ, bestTx);   // no type job ran for this block: its own type only
    BlockRes r;
    r.J = bestJ;
    r.tx = (uint8_t)bestTx;
    r.cand[0] = (uint8_t)winC;
    r.cand[1] = r.cand[2] = r.cand[3] = 0;
    int n = 1;
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (k != bestK && topJ[k] < INF && k < kMax) r.cand[n++ & 3] = (uint8_t)topC[k];
    r.ncand = (uint8_t)n;
    r.txMask = F.txKeep ? rank.mask(F.txKeep) : (uint16_t)slTx;
    F.blk[F.shOff[bs] + (uint32_t)(y >> LH) * F.shNbx[bs] + (x >> LW)] = r;
}

// grid: 3 x ceil(nSb / MID_SBS) CTAs, shape-major (8x8, then 4x16, then 16x4)
template <int BD>
__global__ void __launch_bounds__(MID_THREADS, 2) k_analysis_mid(const __grid_constant__ FrameDesc F) {
    typedef typename std::conditional<BD == 8, uint8_t, uint16_t>::type Px;
    typedef MidSmem<Px> Sm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Sm &S = *reinterpret_cast<Sm *>(smem_raw);
    const int nSb = F.sbCols * F.sbRows, groups = (nSb + MID_SBS - 1) / MID_SBS;
    const int shape = blockIdx.x / groups, sb0 = (blockIdx.x % groups) * MID_SBS;
    const int tid = threadIdx.x;
    const int txSz = shape == 0 ? AV1G_TX_8X8 : shape == 1 ? AV1G_TX_4X16 : AV1G_TX_16X4;
    if (F.poison) {
        smem_poison(smem_raw, sizeof(Sm), tid, MID_THREADS);
        __syncthreads();
    }
    constexpr int V = Sm::TW * (int)sizeof(Px) / 16;
    for (int k = tid; k < MID_SBS * Sm::TH * V; k += MID_THREADS) {
        const int u = k / (Sm::TH * V), r = (k / V) % Sm::TH, c = k % V, sb = sb0 + u;
        if (sb >= nSb) continue;
        const int sbx = (sb % F.sbCols) * 64, sby = (sb / F.sbCols) * 64;
        const Px *s0 = (const Px *)F.src[0] + (size_t)(sby - 1) * F.spitch[0] + (sbx - 16);
        reinterpret_cast<uint4 *>(S.tile[u] + r * Sm::TW)[c] = __ldg(reinterpret_cast<const uint4 *>(s0 + (size_t)r * F.spitch[0]) + c);
    }
    const RateTabs T = rate_tabs_stage(S.T, F.qctx, tid, MID_THREADS);
    __syncthreads();
    for (int k = tid; k < 3 * 64; k += MID_THREADS) {
        const int cls = k / 64, c = k % 64;
        S.iscan[cls][T.scan[c_scanOff[txSz][cls] + c]] = (uint8_t)c;
    }
    __syncthreads();
    const int u = tid >> 6, b = tid & 63, sb = sb0 + u;
    if (sb >= nSb) return;
    const int sbx = (sb % F.sbCols) * 64, sby = (sb / F.sbCols) * 64;
    int tc = 0, tr = 0;
    while (tc + 1 < F.tileCols && sbx >= F.tileColStart[tc + 1] * 4) tc++;
    while (tr + 1 < F.tileRows && sby >= F.tileRowStart[tr + 1] * 4) tr++;
    const int tx0 = F.tileColStart[tc] * 4, tx1 = F.tileColStart[tc + 1] * 4, ty0 = F.tileRowStart[tr] * 4, ty1 = F.tileRowStart[tr + 1] * 4;
    const int FW = F.MiCols * 4, FH = F.MiRows * 4;
    if (shape == 0) {          // 8x8: 8 columns x 8 rows
        const int x = sbx + (b & 7) * 8, y = sby + (b >> 3) * 8;
        if (x < FW && y < FH) mid_block<BD, 3, 3>(F, S, T, AV1G_BLOCK_8X8, AV1G_TX_8X8, S.tile[u], x, y, sbx, sby, tx0, ty0, tx1, ty1);
    } else if (shape == 1) {   // 4x16: 16 columns x 4 rows
        const int x = sbx + (b & 15) * 4, y = sby + (b >> 4) * 16;
        if (x < FW && y < FH) mid_block<BD, 2, 4>(F, S, T, AV1G_BLOCK_4X16, AV1G_TX_4X16, S.tile[u], x, y, sbx, sby, tx0, ty0, tx1, ty1);
    } else {                   // 16x4: 4 columns x 16 rows
        const int x = sbx + (b & 3) * 16, y = sby + (b >> 2) * 4;
        if (x < FW && y < FH) mid_block<BD, 4, 2>(F, S, T, AV1G_BLOCK_16X4, AV1G_TX_16X4, S.tile[u], x, y, sbx, sby, tx0, ty0, tx1, ty1);
    }
}

}  // namespace is
