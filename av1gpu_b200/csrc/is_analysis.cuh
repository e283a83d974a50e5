// is_analysis.cuh - open-loop analysis kernel: every block shape at every aligned position of a superblock.
//
// One CTA per 64x64 SB (8 warps).  The CTA stages the SB's source tile with its edges - rows sby-1 .. sby+63,
// columns sbx-16 .. sbx+127 - in shared memory with 128-bit loads (every edge an open-loop block can read: the
// above-right reach of a block at the SB's top row is 2W <= 128 columns; below-left never leaves the SB's rows).
// Warps then take blocks from the SB's task list (largest shapes first) and run, per block, the search of the
// reference's k_analysis (encoder/src/k_analysis.cuh:496-689):
//   edges from the source (haveAR / haveBL by the Z-order guess), DC value,
//   SATD screening of the 13 modes, then +-1..3 around the two best directional modes (bsize >= 8x8),
//   top-4 by SATD * 2^14 + sqrt(lambda) * mode bits, exact-rate RD of the top-4 with DCT_DCT, tx-type search of the
//   winner, -> BlockRes {J, candidates best first, tx}.
#pragma once
#include "is_dev.cuh"
#include "is_frame.cuh"

namespace is {

// Two kernels share the block search: k_analysis for the 132 blocks of the shapes up to 32 samples a side from 8x16 /
// 16x8 / 8x32 / 32x8 up (8 warps, 2 CTAs per SM: 128 registers a thread; 3 CTAs with 80 registers spilled more and ran
// 2.5 % slower), k_analysis_big for the 13 blocks with a 64-sample side (4 warps with
// the larger scratch).  The 704 blocks of 4x4, 4x8, 8x4, 8x8, 4x16 and 16x4 have the per-thread searches of
// is_tiny.cuh.
constexpr int AN_WARPS = 8, ANB_WARPS = 4;
constexpr int AN_TASKS = 132, ANB_TASKS = 13;
constexpr int AN_BUF_INTS = 1088;             // evaluation scratch per warp: 32 / G tasks of H x (W + 1) int32 (<= 32x32)
constexpr int ANB_BUF_INTS = 64 * 65;
static __constant__ uint8_t c_anTask[AN_TASKS][3];   // (bsize, x4, y4) largest area first, then shape, then raster
static __constant__ uint8_t c_anTaskBig[ANB_TASKS][3];
// Each CTA runs the blocks of ONE shape of one SB (grid: shapes x SBs, shape-major), so that the warps of an SM work
// through the same code; the task ranges of the shapes in the lists above.  The 64-sided list runs in three groups
// instead of its five shapes: 64x64 with 32x64 and 64x32 (5 blocks for the 4 warps; alone, 64x64 left three warps of
// its CTA idle and 32x64 / 64x32 two), then 16x64, then 64x16 (4 blocks each).
constexpr int AN_SHAPES = 8, ANB_SHAPES = 5, ANB_GROUPS = 3;
static __constant__ int c_anShapeStart[AN_SHAPES + 1], c_anShapeStartBig[ANB_GROUPS + 1];

template <typename Px, int BUFI> struct AnWarp {
    int32_t buf[BUFI];
    int16_t q[1024];
    Px pred[BUFI > 2048 ? 4096 : 1024];   // predictions of the tasks' candidates, W x H per group
    int predC[8];                         // candidate whose prediction a group's slice holds (-1: none)
    i64 taskJ[8];
    i64 txJ[16];                          // the winner's open-loop cost per tx type (INF: not evaluated)
    Px ea[EDGE_LEN], el[EDGE_LEN];
    int satd[32];
    int cand[32];
};
template <typename Px, int NW, int BUFI> struct AnSmem {
    static constexpr int TW = 144, TH = 65;   // tile: columns sbx-16 .. sbx+127, rows sby-1 .. sby+63
    Px tile[TH * TW];
    AnWarp<Px, BUFI> w[NW];
    int next;
};

// open-loop "decoded before (x, y)" guess (the reference's ol_decoded, dev_common.cuh:153-163): previous SB row and
// left SB as the spec's BlockDecoded init, Z-order inside the SB; luma pixel units, tile box in pixels
__device__ __forceinline__ int zorder16(int x, int y) {
    int z = 0;
#pragma unroll
    for (int b = 0; b < 4; b++) z |= (((x >> b) & 1) << (2 * b)) | (((y >> b) & 1) << (2 * b + 1));
    return z;
}
__device__ __forceinline__ bool ol_decoded(int px, int py, int x, int y, int tx0, int ty0, int tx1, int ty1) {
    if (px < tx0 || py < ty0 || px >= tx1 || py >= ty1) return false;
    const int sbx = x & ~63, sby = y & ~63;
    if (py < sby) return true;
    if (px < sbx) return py < sby + 64;
    if (px >= sbx + 64 || py >= sby + 64) return false;
    return zorder16(((px - sbx) >> 2) & 15, ((py - sby) >> 2) & 15) < zorder16(((x - sbx) >> 2) & 15, ((y - sby) >> 2) & 15);
}

template <int BD, typename Px, int BUFI>
__device__ __noinline__ void an_block(const FrameDesc &F, const Px *tile, AnWarp<Px, BUFI> &S, int bs, int x, int y, int sbx, int sby,
                                      int tx0, int ty0, int tx1, int ty1) {
    constexpr int TW = 144;
    const int lane = lane_id();
    const int txSz = ST(Max_Tx_Size_Rect)[bs];
    const int W = txw(txSz), H = txh(txSz), lw = 31 - __clz(W), lh = 31 - __clz(H);
    const int maxX = F.MiCols * 4 - 1, maxY = F.MiRows * 4 - 1;
    const int haveL = x > tx0, haveA = y > ty0;
    const int haveAR = ol_decoded(x + W, y - 1, x, y, tx0, ty0, tx1, ty1), haveBL = ol_decoded(x - 1, y + H, x, y, tx0, ty0, tx1, ty1);
    // tile-local coordinates (tile column 0 = sbx - 16, row 0 = sby - 1)
    const int lx = x - sbx + 16, ly = y - sby + 1;
    Px *A = S.ea + EDGE_OFF, *L = S.el + EDGE_OFF;
    build_edges<BD>(tile, TW, lx, ly, W, H, haveL, haveA, haveAR, haveBL, maxX - sbx + 16, maxY - sby + 1, A, L, lane, 32);
    __syncwarp();
    const int dcv = warp_dc<BD>(A, L, haveL, haveA, lw, lh);
    const Px *src = tile + ly * TW + lx;
    const RateTabs T = rate_tabs_global(F.qctx);
    const uint16_t *C = T.cost;
    auto mbits = [&](int c) -> int {
        const int m = cand_mode(c);
        int b = c_avgY[m];
        if (bs >= AV1G_BLOCK_8X8 && is_dir(m)) b += C[ci_angle(m - AV1G_V_PRED) + cand_delta(c) + 3];
        return b;
    };
    // ---- SATD screening of candidates [c0, c1): (candidate, 4x4 sub-block) items over the lanes ----
    const int nsx = W >> 2, lnsx = lw - 2, nsub = (W >> 2) * (H >> 2), lnsub = lw + lh - 4;
    auto screen = [&](int c0, int c1) {
        const int items = (c1 - c0) * nsub;
        for (int it0 = 0; it0 < items; it0 += 32) {
            const int it = it0 + lane;
            const int ci = c0 + (it >> lnsub);
            int t = 0;
            if (it < items) {
                const int sb = it & (nsub - 1), sx = (sb & (nsx - 1)) * 4, sy = (sb >> lnsx) * 4;
                const int c = S.cand[ci], m = cand_mode(c);
                t = pred4_satd(m, pangle(m, cand_delta(c)), sy, sx, lw, lh, A, L, dcv, src, TW);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                if (o < nsub) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (it < items && (lane & (nsub - 1)) == 0) S.satd[ci] += t;
            __syncwarp();
        }
    };
    // the candidates screened: a block with a learned shortlist screens its list (most probable first, so ties go to
    // the more probable one); the others the 13 modes, then +-1..3 around the two best directional modes
    const uint32_t recIdx = (uint32_t)(y / H) * F.shNbx[bs] + x / W;
    const SlCand *slc = (F.slCand && F.slIdx[bs] >= 0) ? F.slCand + F.slIdx[bs] + recIdx : nullptr;
    const int nsl = slc ? slc->n : 0;
    const uint32_t slTx = slc ? slc->txMask : 0u;
    const int nm = nsl > 0 ? nsl : 13;
    S.satd[lane] = 0;
    if (lane < nm) S.cand[lane] = nsl > 0 ? (int)slc->c[lane] : cand_pack(lane, 0);
    __syncwarp();
    screen(0, nm);
    i64 js = lane < nm ? ((i64)S.satd[lane] << 14) + F.sqlam * mbits(S.cand[lane]) : INF;
    int nc = nm;
    if (nsl == 0 && bs >= AV1G_BLOCK_8X8) {
        const i64 jd = (lane < nm && is_dir(cand_mode(S.cand[lane]))) ? js : INF;
        const int l0 = warp_argmin(jd, lane);
        const int l1 = warp_argmin(lane == l0 ? INF : jd, lane);
        const int b0 = l0 >= 0 ? cand_mode(S.cand[l0]) : -1, b1 = l1 >= 0 ? cand_mode(S.cand[l1]) : -1;
        const int nd = (b0 >= 0 ? 6 : 0) + (b1 >= 0 ? 6 : 0);   // 12 with the plain form's two directional modes
        __syncwarp();
        if (lane < nd) {
            const int m = lane < 6 ? b0 : b1, k = lane % 6;
            S.cand[nm + lane] = cand_pack(m, k < 3 ? -(k + 1) : (k - 2));
        }
        __syncwarp();
        screen(nm, nm + nd);
        if (lane >= nm && lane < nm + nd) js = ((i64)S.satd[lane] << 14) + F.sqlam * mbits(S.cand[lane]);
        nc = nm + nd;
    }
    (void)nc;
    int top[K_TOP];
    int nK = 0;
    const int kMax = nsl > 0 ? F.slRdK : F.rdK;   // a shortlisted block: its best slRdK candidates only
#pragma unroll
    for (int k = 0; k < K_TOP; k++) {
        top[k] = warp_argmin(js, lane);
        if (top[k] >= 0 && k < kMax) nK = k + 1;
        if (lane == top[k]) js = INF;
    }
    // ---- RD: the top-K with DCT_DCT, then the other types of the set for the winner; 32 / G tasks at a time, the
    //      costs compared afterwards in evaluation order (strict <: the first of equal costs wins, as a serial loop) ----
    const int set = tx_set_intra(txSz);
    const bool hasC = has_chroma(bs, y >> 2, x >> 2, F.ssx);
    const int overhead = (hasC ? UV_OVERHEAD : 0) + c_avgSkip0;
    const int G = grp_size(txSz), ng = 32 / G, grp = lane / G, g = lane & (G - 1);
    const int bufInts = task_buf_ints(txSz), nq = min(W, 32) * min(H, 32);
    int32_t *tb = S.buf + grp * bufInts;
    int16_t *tq = S.q + grp * nq;
    Px *tp = S.pred + grp * (W * H);
    if (lane < 8) S.predC[lane] = -1;
    __syncwarp();
    // the group's task: its candidate's prediction into the group's slice (kept while the candidate repeats)
    auto evalc = [&](int c, int t) -> EvalOut {
        const int m = cand_mode(c);
        if (S.predC[grp] != c) grp_predict(m, pangle(m, cand_delta(c)), lw, lh, A, L, dcv, tp, g, G);
        __syncwarp();
        if (g == 0) S.predC[grp] = c;
        const EvalIn e{t, 0, 0, 0, m, F.dcQ, F.acQ, T};
        return grp_eval<BD, Px>(txSz, ResFn<Px>{src, TW, tp, lw, nullptr}, e, tb, tq, g, G);
    };
    i64 bestJ = INF;
    int bestK = 0, bestTx = AV1G_DCT_DCT;
    // stage 1: candidates top[0 .. nK) with DCT_DCT
    for (int r0 = 0; r0 < nK; r0 += ng) {
        const int k = min(r0 + grp, nK - 1);   // groups past the end repeat the last task (their results are unused)
        const int c = S.cand[top[k]];
        const EvalOut o = evalc(c, AV1G_DCT_DCT);
        if (g == 0 && r0 + grp < nK) S.taskJ[grp] = o.D + F.lam * (o.R + mbits(c) + overhead);
        __syncwarp();
        for (int t = 0; t < ng && r0 + t < nK; t++)
            if (S.taskJ[t] < bestJ) { bestJ = S.taskJ[t]; bestK = r0 + t; }
        __syncwarp();
    }
    // stage 2: the other tx types of the set for the winner
    if (lane < 16) S.txJ[lane] = lane == AV1G_DCT_DCT ? bestJ : INF;   // the winner's costs per type (txKeep)
    __syncwarp();
    if (set != AV1G_TX_SET_DCTONLY) {
        int types[8], nt = 0;
        for (int t = 1; t < 16; t++)   // a shortlisted block: the types of its list
            if (tx_in_set(set, t) && (!slTx || ((slTx >> t) & 1))) types[nt++] = t;
        const int c = S.cand[top[bestK]];
        for (int r0 = 0; r0 < nt; r0 += ng) {
            const int tt = types[min(r0 + grp, nt - 1)];
            const EvalOut o = evalc(c, tt);
            if (g == 0 && r0 + grp < nt) {
                const i64 J = o.D + F.lam * (o.R + mbits(c) + overhead);
                S.taskJ[grp] = J;
                S.txJ[tt] = J;
            }
            __syncwarp();
            for (int t = 0; t < ng && r0 + t < nt; t++)
                if (S.taskJ[t] < bestJ) { bestJ = S.taskJ[t]; bestTx = types[r0 + t]; }
            __syncwarp();
        }
    }
    // the txKeep best types by cost (the lower type of equal costs: the one evaluated first)
    uint32_t txMask = 0;
    if (F.txKeep && set != AV1G_TX_SET_DCTONLY) {
        i64 v = lane < 16 ? S.txJ[lane] : INF;
        for (int k = 0; k < F.txKeep; k++) {
            const int b = warp_argmin(v, lane);
            if (b < 0) break;
            txMask |= 1u << b;
            if (lane == b) v = INF;
        }
    }
    if (lane == 0) {
        BlockRes r;
        r.J = bestJ;
        r.tx = (uint8_t)bestTx;
        int n = 0;
        r.cand[n++] = (uint8_t)S.cand[top[bestK]];
        for (int k = 0; k < nK; k++) if (k != bestK) r.cand[n++] = (uint8_t)S.cand[top[k]];
        for (int k = n; k < 4; k++) r.cand[k] = 0;
        r.ncand = (uint8_t)n;
        r.txMask = (uint16_t)(txMask ? txMask : slTx);
        F.blk[F.shOff[bs] + (uint32_t)(y / H) * F.shNbx[bs] + x / W] = r;
    }
    __syncwarp();
}

// the task list of a kernel: 0 the shapes up to 32 a side, 1 those with a 64-sample side
template <int LIST> __device__ __forceinline__ const uint8_t *an_task(int t) { return LIST == 0 ? c_anTask[t] : c_anTaskBig[t]; }
template <int LIST> __device__ __forceinline__ int an_shape_start(int s) { return LIST == 0 ? c_anShapeStart[s] : c_anShapeStartBig[s]; }

// one CTA per SB: stage the tile, then the warps take the blocks of the task list
template <int BD, int NW, int BUFI, int LIST>
__device__ __forceinline__ void an_sb(const FrameDesc &F, unsigned char *smem_raw) {
    typedef typename std::conditional<BD == 8, uint8_t, uint16_t>::type Px;
    typedef AnSmem<Px, NW, BUFI> Sm;
    Sm &S = *reinterpret_cast<Sm *>(smem_raw);
    const int nSb = F.sbCols * F.sbRows, shape = blockIdx.x / nSb, sb = blockIdx.x % nSb;
    const int sbr = sb / F.sbCols, sbc = sb % F.sbCols;
    const int sbx = sbc * 64, sby = sbr * 64;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int t0 = an_shape_start<LIST>(shape), t1 = an_shape_start<LIST>(shape + 1);
    if (F.poison) {
        smem_poison(smem_raw, sizeof(Sm), tid, NW * 32);
        __syncthreads();
    }
    {   // the SB tile with 128-bit loads (rows and the tile's first column are 16-byte aligned by the layout)
        constexpr int V = Sm::TW * (int)sizeof(Px) / 16;
        const Px *s0 = (const Px *)F.src[0] + (size_t)(sby - 1) * F.spitch[0] + (sbx - 16);
        for (int k = tid; k < Sm::TH * V; k += NW * 32) {
            const int r = k / V, c = k % V;
            reinterpret_cast<uint4 *>(S.tile + r * Sm::TW)[c] = __ldg(reinterpret_cast<const uint4 *>(s0 + (size_t)r * F.spitch[0]) + c);
        }
        if (tid == 0) S.next = t0 + NW;
    }
    __syncthreads();
    int tc = 0, tr = 0;
    while (tc + 1 < F.tileCols && sbx >= F.tileColStart[tc + 1] * 4) tc++;
    while (tr + 1 < F.tileRows && sby >= F.tileRowStart[tr + 1] * 4) tr++;
    const int tx0 = F.tileColStart[tc] * 4, tx1 = F.tileColStart[tc + 1] * 4, ty0 = F.tileRowStart[tr] * 4, ty1 = F.tileRowStart[tr + 1] * 4;
    const int FW = F.MiCols * 4, FH = F.MiRows * 4;
    int t = t0 + warp;
    while (t < t1) {
        const uint8_t *tk = an_task<LIST>(t);
        const int bs = tk[0], x = sbx + tk[1] * 4, y = sby + tk[2] * 4;
        if (x < FW && y < FH) an_block<BD, Px, BUFI>(F, S.tile, S.w[warp], bs, x, y, sbx, sby, tx0, ty0, tx1, ty1);
        int n = 0;
        if (lane == 0) n = atomicAdd(&S.next, 1);
        t = __shfl_sync(0xffffffffu, n, 0);
    }
}

template <int BD>
__global__ void __launch_bounds__(AN_WARPS * 32, 2) k_analysis(const __grid_constant__ FrameDesc F) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    an_sb<BD, AN_WARPS, AN_BUF_INTS, 0>(F, smem_raw);
}
template <int BD>
__global__ void __launch_bounds__(ANB_WARPS * 32, 2) k_analysis_big(const __grid_constant__ FrameDesc F) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    an_sb<BD, ANB_WARPS, ANB_BUF_INTS, 1>(F, smem_raw);
}


}  // namespace is
