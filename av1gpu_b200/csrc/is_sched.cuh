// is_sched.cuh - the closed loop's schedule and the pack: per SB the map of leaf indices and record offsets, the
// global leaf queue, the dataflow graph (per-leaf luma dependency counters and dependents lists, the initial ready
// leaves), and the compaction of the per-SB output slots into the DecisionRecord in decode order (the reference's
// k_pack and host offsets, encoder/src/k_misc.cu:46-105, pipeline.cpp:878-903).
#pragma once
#include "is_recon.cuh"

namespace is {

// Dependencies of leaf li of SB sb: the distinct leaves (unit_leaf rule) covering a unit of its above strip (row y4 - 1
// from the above-left corner to the above-right reach x4 + 2 bw) or of its left strip (column x4 - 1 down to the
// below-left reach y4 + 2 bh) - every sample its luma prediction and its luma contexts read - and, for a 4:2:0 chroma
// carrier, the leaves of the strips its chroma waits on (rc_leaf's chroma rc_wait; with 4:4:4 they are among the
// first).  A leaf is queued when all of them have published their luma, so a chroma wait is always on leaves whose
// warps are running (their chroma follows their luma in the same warp): however long the queue, waits cannot
// accumulate on leaves that no warp has taken yet.  At most 2 bw + 1 + 2 bh + 5 (REV_PER_SB).
static __device__ int luma_deps(const FrameDesc &F, int sb, int li, uint32_t *out) {
    const Leaf lf = F.leaves[(size_t)sb * SB_MAX_LEAVES + li];
    const int bw = bw4(lf.bsize), bh = bh4(lf.bsize);
    const int sbr = sb / F.sbCols, sbc = sb % F.sbCols;
    int tC0, tC1, tR0, tR1;
    tile_box(F, sbr * 16 + lf.y4, sbc * 16 + lf.x4, tC0, tC1, tR0, tR1);
    int n = 0;
    auto add = [&](int yy, int xx) {
        const int id = unit_leaf(F, sb, li, sbr, sbc, yy, xx, tC0, tC1, tR0);
        if (id < 0 || (n > 0 && out[n - 1] == (uint32_t)id)) return;
        bool seen = false;
        for (int k = 0; k < n; k++) seen |= out[k] == (uint32_t)id;
        if (!seen) out[n++] = (uint32_t)id;
    };
    for (int c = lf.x4 - 1; c < lf.x4 + 2 * bw; c++) add(lf.y4 - 1, c);
    for (int r = lf.y4; r < lf.y4 + 2 * bh; r++) add(r, lf.x4 - 1);
    if (F.ssx && has_chroma(lf.bsize, sbr * 16 + lf.y4, sbc * 16 + lf.x4, 1)) {
        const int cx0 = lf.x4 & ~1, cy0 = lf.y4 & ~1, cw = max(bw, 2), ch = max(bh, 2);
        for (int c = cx0 - 1; c < cx0 + 2 * cw; c += 2) add(cy0 - 1, c);
        for (int r = cy0 + 1; r < cy0 + 2 * ch; r += 2) add(r, cx0 - 1);
    }
    return n;
}

// ---- before the closed loop: per SB the map of leaf indices, per leaf its first tx block and coefficient (SB-local),
// per SB the output counts; then the global leaf queue (SBs in wavefront order, leaves in decode order) ----
__global__ void k_leaf_prep(const __grid_constant__ FrameDesc F, int nSb) {
    const int sb = blockIdx.x, tid = threadIdx.x;
    if (sb >= nSb) return;
    __shared__ uint8_t om[256];
    const int nl = F.nLeaves[sb];
    om[tid] = 255;
    F.leafDone[(size_t)sb * SB_MAX_LEAVES + tid] = 0;
    F.revCnt[(size_t)sb * SB_MAX_LEAVES + tid] = 0;
    F.revFill[(size_t)sb * SB_MAX_LEAVES + tid] = 0;
    __syncthreads();
    if (tid < nl) {
        const Leaf l = F.leaves[(size_t)sb * SB_MAX_LEAVES + tid];
        const int w4 = bw4(l.bsize), h4 = bh4(l.bsize);
        for (int r = l.y4; r < min(16, l.y4 + h4); r++)
            for (int c = l.x4; c < min(16, l.x4 + w4); c++) om[r * 16 + c] = (uint8_t)tid;
    }
    __syncthreads();
    F.ordmap[(size_t)sb * 256 + tid] = om[tid];
    if (tid == 0) {
        const int sbr = sb / F.sbCols, sbc = sb % F.sbCols;
        int nt = 0, ncf = 0;
        for (int i = 0; i < nl; i++) {
            F.leafTxb[(size_t)sb * SB_MAX_LEAVES + i] = (uint16_t)nt;
            F.leafCoef[(size_t)sb * SB_MAX_LEAVES + i] = (uint16_t)ncf;
            const Leaf l = F.leaves[(size_t)sb * SB_MAX_LEAVES + i];
            const int yt = ST(Max_Tx_Size_Rect)[l.bsize];
            nt += 1;
            ncf += min(txw(yt), 32) * min(txh(yt), 32);
            const int mi_row = sbr * 16 + l.y4, mi_col = sbc * 16 + l.x4;
            if (has_chroma(l.bsize, mi_row, mi_col, F.ssx)) {
                // 2 x the coded chroma tx blocks of a plane (more than one: 4:4:4 blocks with a 64-sample side)
                const int ut = uv_tx_size(l.bsize, F.ssx), ss = F.ssx;
                const int W = txw(ut), H = txh(ut);
                const int nTxX = ss ? 1 : max(1, 4 * bw4(l.bsize) / W), nTxY = ss ? 1 : max(1, 4 * bh4(l.bsize) / H);
                const int cx4 = mi_col >> ss, cy4 = mi_row >> ss, cCols4 = F.MiCols >> ss, cRows4 = F.MiRows >> ss;
                int nc = 0;
                for (int t = 0; t < nTxX * nTxY; t++)
                    nc += t == 0 || (cx4 + (t % nTxX) * (W >> 2) < cCols4 && cy4 + (t / nTxX) * (H >> 2) < cRows4);
                nt += 2 * nc;
                ncf += 2 * nc * min(W, 32) * min(H, 32);
            }
        }
        SbCount c;
        c.nBlocks = (uint32_t)nl; c.nTxb = (uint32_t)nt; c.nCoeffs = (uint32_t)ncf; c.pad = 0;
        F.sbCount[sb] = c;
    }
}
// exclusive prefix of the leaf counts over the wavefront order (one CTA of 1024 threads), then every SB's leaves into
// the queue
__global__ void k_leaf_queue_scan(const __grid_constant__ FrameDesc F, int nSb) {
    __shared__ uint32_t sN[1024];
    const int tid = threadIdx.x;
    const int per = (nSb + 1023) / 1024, i0 = min(nSb, tid * per), i1 = min(nSb, i0 + per);
    uint32_t n = 0;
    for (int i = i0; i < i1; i++) n += F.nLeaves[F.sbOrder[i]];
    sN[tid] = n;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const uint32_t v = tid >= o ? sN[tid - o] : 0;
        __syncthreads();
        sN[tid] += v;
        __syncthreads();
    }
    uint32_t at = sN[tid] - n;
    for (int i = i0; i < i1; i++) {
        const uint32_t sb = F.sbOrder[i];
        F.leafStart[sb] = at;
        at += F.nLeaves[sb];
    }
    if (tid == 1023) *F.leafTotal = sN[1023];
}
// The dataflow graph of the closed loop, one thread per leaf, in four passes: 0 counts each leaf's luma dependencies
// and its dependents, 1 gives each leaf its range of revList, 2 writes the dependents, 3 queues the leaves without
// dependencies.  The queueing comes last so that a closed loop already running (a serving session) never takes a leaf
// whose dependents list is not written yet.
template <int PASS>
__global__ void k_leaf_deps(const __grid_constant__ FrameDesc F, int nSb) {
    const int sb = blockIdx.x, tid = threadIdx.x;
    if (sb >= nSb || tid >= F.nLeaves[sb]) return;
    const uint32_t me = (uint32_t)sb * SB_MAX_LEAVES + tid;
    const uint32_t cap = (uint32_t)nSb * REV_PER_SB;   // never reached (see REV_PER_SB); checked all the same
    if (PASS == 1) {
        const uint32_t off = (uint32_t)atomicAdd(F.queue + 2, F.revCnt[me]);
        F.revOff[me] = off;
        if (off + (uint32_t)F.revCnt[me] > cap) atomicCAS(F.err, 0, KERR_CAPACITY);
        return;
    }
    if (PASS == 3) {
        if (F.depCnt[me] == 0) push_ready(F, me);
        return;
    }
    uint32_t d[72];
    const int n = luma_deps(F, sb, tid, d);
    if (PASS == 0) F.depCnt[me] = n;
    for (int k = 0; k < n; k++) {
        if (PASS == 0) {
            atomicAdd(F.revCnt + d[k], 1);
        } else {
            const uint32_t at = F.revOff[d[k]] + (uint32_t)atomicAdd(F.revFill + d[k], 1);
            if (at < cap) F.revList[at] = me;
        }
    }
}

// ---- pack: per-SB slots -> DecisionRecord arrays in decode order ----
__global__ void k_pack_scan(const __grid_constant__ FrameDesc F, int nSb) {
    // exclusive prefix sums of the per-SB counts over the decode order (one CTA of 1024 threads)
    __shared__ uint32_t sB[1024], sT[1024];
    __shared__ unsigned long long sC[1024];
    const int tid = threadIdx.x;
    const int per = (nSb + 1023) / 1024, i0 = min(nSb, tid * per), i1 = min(nSb, i0 + per);
    uint32_t b = 0, t = 0;
    unsigned long long c = 0;
    for (int i = i0; i < i1; i++) {
        const SbCount k = F.sbCount[F.sbDecodeOrder[i]];
        b += k.nBlocks; t += k.nTxb; c += k.nCoeffs;
    }
    sB[tid] = b; sT[tid] = t; sC[tid] = c;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        uint32_t vb = 0, vt = 0;
        unsigned long long vc = 0;
        if (tid >= o) { vb = sB[tid - o]; vt = sT[tid - o]; vc = sC[tid - o]; }
        __syncthreads();
        sB[tid] += vb; sT[tid] += vt; sC[tid] += vc;
        __syncthreads();
    }
    b = sB[tid] - b; t = sT[tid] - t; c = sC[tid] - c;
    for (int i = i0; i < i1; i++) {
        F.offBlk[i] = b; F.offTxb[i] = t; F.offCoef[i] = c;
        const SbCount k = F.sbCount[F.sbDecodeOrder[i]];
        b += k.nBlocks; t += k.nTxb; c += k.nCoeffs;
    }
    if (tid == 1023) { F.offBlk[nSb] = sB[1023]; F.offTxb[nSb] = sT[1023]; F.offCoef[nSb] = sC[1023]; }
}

__global__ void k_pack(const __grid_constant__ FrameDesc F, int nSb) {
    const int i = blockIdx.x;
    if (i >= nSb) return;
    const int sb = (int)F.sbDecodeOrder[i];
    const SbCount k = F.sbCount[sb];
    const uint32_t ob = F.offBlk[i], ot = F.offTxb[i];
    const uint64_t oc = F.offCoef[i];
    for (uint32_t j = threadIdx.x; j < k.nBlocks; j += blockDim.x) {
        F.recBlocks[ob + j] = F.oBlocks[(size_t)sb * SB_MAX_LEAVES + j];
        F.recBlockTxb[ob + j] = ot + F.oBlockTxb[(size_t)sb * SB_MAX_LEAVES + j];
    }
    for (uint32_t j = threadIdx.x; j < k.nTxb; j += blockDim.x) {
        av1g_txb t = F.oTxb[(size_t)sb * SB_MAX_TXB + j];
        t.coeff_off = (uint32_t)(oc + t.coeff_off);
        F.recTxb[ot + j] = t;
    }
    // coefficients: 16-byte vectors (every tx block holds a multiple of 16 levels, SB slots are 16-byte aligned)
    const uint4 *s = reinterpret_cast<const uint4 *>(F.oCoeffs + (size_t)sb * SB_MAX_COEF);
    int16_t *d = F.recCoeffs + oc;
    if ((oc & 7) == 0) {
        uint4 *dv = reinterpret_cast<uint4 *>(d);
        for (uint32_t j = threadIdx.x; j < k.nCoeffs / 8; j += blockDim.x) dv[j] = s[j];
    } else {
        const int16_t *ss = F.oCoeffs + (size_t)sb * SB_MAX_COEF;
        for (uint32_t j = threadIdx.x; j < k.nCoeffs; j += blockDim.x) d[j] = ss[j];
    }
    if (i == nSb - 1 && threadIdx.x == 0) F.recBlockTxb[F.offBlk[nSb]] = F.offTxb[nSb];
}

}  // namespace is
