// is_recon.cuh - closed-loop decision + reconstruction: warps as independent workers over a global leaf queue.
//
// The leaves (the DP's blocks) of every SB form one global queue in topological order - SBs by wavefront step
// (tile-local col + 2 row), the leaves of an SB in decode order - so every leaf a leaf depends on comes earlier.  A
// persistent grid of warps (co-resident: cooperative launch) takes leaves from the queue; a warp waits - bounded spins
// on acquire loads of per-leaf done flags - only for the earlier leaves whose area meets its leaf's neighbourhood
// (edges with their above-right / below-left reach, coefficient and mode contexts, 4:2:0 chroma pairs), in its own SB
// or in the SBs above, above-right and left.  Leaves of neighbouring superblocks therefore overlap, and every leaf still
// sees exactly the state of a sequential decode-order pass.  Data written by other warps (reconstruction, maps) is read
// with L1-bypassing loads after the acquire.  Per leaf (one warp; the reference's rc_luma / rc_chroma,
// encoder/src/k_recon.cuh:822-1686):
//   luma    real edges from the reconstruction, exact contexts; pass 1 = the analysis' top-2 with DCT_DCT (+ its winner
//           with its tx type), pass 2 = the other tx types of the pass-1 winner; tasks in lane groups; final levels ->
//           exact inverse (with the conformance repair) -> reconstruction, record
//   chroma  CfL luma from the reconstruction, least-squares alpha + +-1 refinement; SATD screening of 13 UV modes
//           (+ +-1..3 around the best directional one); top-2 + CfL through the exact RD of U and V; final U, V
// The BlockDecoded state of the spec is derived from the SB's map of leaf indices (a unit is decoded for leaf li iff its
// leaf index is below li) and the SB border rules of clear_block_decoded_flags outside it.
#pragma once
#include "is_dev.cuh"
#include "is_frame.cuh"

namespace is {

// warps per CTA: independent workers, as many as the shared memory of one CTA per SM holds (at most 8; rc_warps below)
constexpr int RC_MAX_WARPS = 8;
// per-warp scratch: a task round of tx sizes up to 32 x 32 (32 / G tasks of H x (W + 1) int32: at most 16 x 80 in the
// small sizes' single round (G >= 2, 4x16), 4 x 272 / 2 x 544 / 1 x 1056 in the others (round_group's G)) and
// predictions up to 32 x 32 (16 x 64 in the single round); the luma of a leaf with a 64-sample side (rare: large flat
// blocks) uses the CTA's one large buffer (RcBig) instead, under a lock
constexpr int RC_BUF_INTS = 1280;
// bounded waits (defaults; FrameDesc::waitIters / readyWaitNs carry the values of a run): a wait that runs out records
// an error and moves on, and once any error is recorded no further wait starts (the host discards the result)
constexpr int LEAF_WAIT_ITERS = 1 << 20;
// closed-loop trace (is_set_trace): per queued leaf, globaltimer ns at: 0 slot claimed, 1 slot read, 2 luma prologue
// done (loads, edges, contexts), 3 luma pass 1 done, 4 pass 2 done, 5 luma published, 6 chroma waits done, 7 chroma
// screening and RD done, 8 leaf done; 9 the queue entry (image << 32 | sb << 8 | leaf)
constexpr int TRACE_STAMPS = 10;
constexpr long long READY_WAIT_NS = 4000000000ll;

template <typename Px, int SS> struct RcWarp {   // SS: chroma subsampling (1 4:2:0, 0 4:4:4)
    int32_t buf[RC_BUF_INTS];  // evaluation scratch (32 / G tasks) and the inverse transform's residual (tx <= 32 x 32)
    int16_t q[1024];           // levels of the tasks of a round
    int16_t qb[2][1024];       // best levels (chroma: U, V)
    Px pred[1024];             // predictions of the tasks (W x H per group); the final prediction (tx <= 32 x 32)
    i64 taskJ[16];
    int predC[8];
    Px ea[3][EDGE_LEN], el[3][EDGE_LEN];
    __align__(16) Px srcS[3][1024];   // the source of the leaf's tx blocks (Y, U, V) when <= 32 x 32, staged once per
                                      // leaf with 16-byte vector stores
    int16_t cfl[SS ? 256 : 1024];   // CfL luma values of a chroma block up to 16 x 16 (4:2:0) / 32 x 32 (4:4:4)
    int satd[32];
    int cand[32];
    int job;
};
template <typename Px> struct RcBig {   // the CTA's scratch for luma tx sizes with a 64-sample side
    int32_t buf[64 * 65];
    Px pred[64 * 64];
    int lock;                           // 0 free, 1 taken
    int pad[3];
};
template <typename Px, int SS> struct RcSlot {   // one warp's part: its copy of its image's descriptor, its scratch
    FrameDesc F;
    RcWarp<Px, SS> w;
};
// The warps' parts come last: a launch with fewer working warps allocates only theirs (rc_smem_bytes), which leaves the
// SM a larger L1 for the warps' stacks.
template <typename Px, int SS, int NW> struct RcSmem {
    RateStage T;                         // scans, base-context offsets (and the cost table of q-context 0)
    RcBig<Px> big;
    uint16_t cost[3][NCDF];              // the cost tables of q-contexts 1 .. 3 (the images of a batch mix qindex)
    RcSlot<Px, SS> ws[NW];
};
template <typename Px, int SS> constexpr size_t rc_smem_bytes(int warps) {
    typedef RcSmem<Px, SS, 1> S1;
    typedef RcSlot<Px, SS> Slot;
    return offsetof(S1, ws) + (size_t)warps * sizeof(Slot);
}
// the most warps (<= RC_MAX_WARPS) whose shared memory fits one CTA (8 for 8-bit 4:2:0, fewer for the larger formats)
template <typename Px, int SS> constexpr int rc_warps() {
    return sizeof(RcSmem<Px, SS, 8>) <= 227 * 1024 ? 8 : sizeof(RcSmem<Px, SS, 7>) <= 227 * 1024 ? 7
         : sizeof(RcSmem<Px, SS, 6>) <= 227 * 1024 ? 6 : sizeof(RcSmem<Px, SS, 5>) <= 227 * 1024 ? 5 : 4;
}
template <typename Px, int SS> constexpr bool rc_smem_ok() {
    typedef RcWarp<Px, SS> Wt;
    typedef RcSmem<Px, SS, rc_warps<Px, SS>()> St;
    typedef RcSlot<Px, SS> Sl;
    return sizeof(St) <= 227 * 1024 && offsetof(Wt, srcS) % 16 == 0 && sizeof(Wt) % 16 == 0 && offsetof(St, ws) % 16 == 0 &&
           offsetof(St, cost) % 16 == 0 && sizeof(Sl) % 16 == 0 && offsetof(Sl, w) % 16 == 0 &&
           rc_smem_bytes<Px, SS>(rc_warps<Px, SS>()) == sizeof(St);
}
static_assert(rc_smem_ok<uint8_t, 1>() && rc_smem_ok<uint8_t, 0>() && rc_smem_ok<uint16_t, 1>() && rc_smem_ok<uint16_t, 0>() &&
                  sizeof(FrameDesc) % 16 == 0,
              "the closed loop's shared memory: at most 227 KB, staged sources and descriptors 16-byte aligned");
static_assert(rc_warps<uint8_t, 1>() == 8 && rc_warps<uint8_t, 0>() >= 7 && rc_warps<uint16_t, 1>() >= 6 && rc_warps<uint16_t, 0>() >= 5,
              "closed-loop warps per CTA");

// Waits poll with relaxed loads and acquire once, with a fence after the awaited value was seen (the acquire pattern of
// the PTX memory model: a strong read that observes a release, then fence.acq_rel): one acquire per wait instead of one
// per poll.
__device__ __forceinline__ int ld_relaxed(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void fence_acquire() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
// the release side: the writes before it (the thread's own, and those ordered before it by a warp barrier) are visible
// to a thread that acquires a later relaxed store or atomic of this thread (an acquire-release fence, not the
// sequentially consistent one of __threadfence, which costs a global ordering step)
__device__ __forceinline__ void fence_release() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void st_release(int *p, int v) { asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory"); }
template <typename P> __device__ __forceinline__ P ldcg(const P *p);
template <> __device__ __forceinline__ uint8_t ldcg<uint8_t>(const uint8_t *p) { return __ldcg(p); }
template <> __device__ __forceinline__ uint16_t ldcg<uint16_t>(const uint16_t *p) { return __ldcg(p); }

// AboveRow / LeftCol from the reconstruction (other warps' data: L1-bypassing loads), as build_edges
template <int BD, typename P>
__device__ __forceinline__ void rec_edges(const P *plane, int pitch, int x, int y, int w, int h, int haveL, int haveA, int haveAR,
                                          int haveBL, int maxX, int maxY, P *A, P *L) {
    const int t = lane_id(), n = w + h;
    const int alim = min(x + (haveAR ? 2 * w : w) - 1, maxX), llim = min(y + (haveBL ? 2 * h : h) - 1, maxY);
    for (int i = t; i < n; i += 32) {
        P a, l;
        if (haveA) a = ldcg(plane + (size_t)(y - 1) * pitch + min(x + i, alim));
        else a = haveL ? ldcg(plane + (size_t)y * pitch + x - 1) : (P)((1 << (BD - 1)) - 1);
        if (haveL) l = ldcg(plane + (size_t)min(y + i, llim) * pitch + x - 1);
        else l = haveA ? ldcg(plane + (size_t)(y - 1) * pitch + x) : (P)((1 << (BD - 1)) + 1);
        A[i] = a;
        L[i] = l;
    }
    if (t == 0) {
        P c;
        if (haveA && haveL) c = ldcg(plane + (size_t)(y - 1) * pitch + x - 1);
        else if (haveA) c = ldcg(plane + (size_t)(y - 1) * pitch + x);
        else if (haveL) c = ldcg(plane + (size_t)y * pitch + x - 1);
        else c = (P)(1 << (BD - 1));
        A[-1] = c;
        L[-1] = c;
    }
}

// exact inverse + reconstruction of a tx block (warp), the levels halved until conformant (AV1G_ENC_FIX_RANGE's
// repair, the reference's cta_inverse_add, k_recon.cuh:140-197); writes prediction + residual into the plane
template <int BD, typename Px>
__device__ void rc_reconstruct(int txSz, int txType, int16_t *q, int dcQ, int acQ, const Px *pred, Px *dst, int pitch, int32_t *buf) {
    const int lane = lane_id();
    const int W = txw(txSz), H = txh(txSz), n = min(W, 32) * min(H, 32), TS = W + 1;
    bool any = false;
    for (;;) {
        int nz = 0;
        for (int i = lane; i < n; i += 32) nz |= q[i] != 0;
        if (!__any_sync(0xffffffffu, nz)) { any = false; break; }
        const uint32_t err = grp_inverse<BD>(txSz, q, txType, dcQ, acQ, buf, lane, 32);
        if (!err) { any = true; break; }
        for (int i = lane; i < n; i += 32) q[i] = (int16_t)(q[i] / 2);
        __syncwarp();
    }
    const int lw = 31 - __clz(W);
    for (int p = lane; p < W * H; p += 32) {
        const int i = p >> lw, j = p & (W - 1);
        int v = (int)pred[p] + (any ? buf[i * TS + j] : 0);
        v = min(max(v, 0), (1 << BD) - 1);
        dst[(size_t)i * pitch + j] = (Px)v;
    }
    __syncwarp();
}

// the edges of a W x H (<= 32 x 32) tx block at (px, py) of plane pl from the reconstruction, whole warp: the rule of
// the reference's rec_edges (availability, above-right / below-left reach, frame clamp), as the leaf's first tx blocks
template <int BD, typename Px>
__device__ void rc_edges_rec(const FrameDesc &F, int pl, int px, int py, int W, int H, int haveL, int haveA, int haveAR, int haveBL, Px *A, Px *L) {
    const int lane = lane_id();
    const int ss = pl ? F.ssx : 0;
    const Px *rp = (const Px *)F.rec[pl];
    const int pitch = F.rpitch[pl], n = W + H;
    const int aLim = min(px + 2 * W - 1, ((F.MiCols * 4) >> ss) - 1), lLim = min(py + 2 * H - 1, ((F.MiRows * 4) >> ss) - 1);
    Px ra[2], rl[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const int i = lane + 32 * k;
        ra[k] = i < n ? ldcg(rp + (size_t)(py - 1) * pitch + min(px + i, aLim)) : (Px)0;
        rl[k] = i < n ? ldcg(rp + (size_t)min(py + i, lLim) * pitch + px - 1) : (Px)0;
    }
    const Px rcorner = ldcg(rp + (size_t)(py - 1) * pitch + px - 1);
    const Px aW = (Px)__shfl_sync(0xffffffffu, (int)ra[0], W - 1), lH = (Px)__shfl_sync(0xffffffffu, (int)rl[0], H - 1);
    const Px a0 = (Px)__shfl_sync(0xffffffffu, (int)ra[0], 0), l0 = (Px)__shfl_sync(0xffffffffu, (int)rl[0], 0);
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const int i = lane + 32 * k;
        if (i < n) {
            A[i] = haveA ? ((!haveAR && i >= W) ? aW : ra[k]) : (haveL ? l0 : (Px)((1 << (BD - 1)) - 1));
            L[i] = haveL ? ((!haveBL && i >= H) ? lH : rl[k]) : (haveA ? a0 : (Px)((1 << (BD - 1)) + 1));
        }
    }
    if (lane == 0) {
        const Px c = (haveA && haveL) ? rcorner : haveA ? a0 : haveL ? l0 : (Px)(1 << (BD - 1));
        A[-1] = c;
        L[-1] = c;
    }
    __syncwarp();
}

// record a finished tx block: eob, culLevel / dc category into the context maps, the txb entry and its levels
static __device__ int rc_record(const FrameDesc &F, const RateTabs &T, int sb, int plane, int txSz, int txType, int x4, int y4, const int16_t *q,
                         int txbIdx, int coefOff) {
    const int lane = lane_id();
    const int W = txw(txSz), H = txh(txSz), n = min(W, 32) * min(H, 32);
    const uint16_t *scan = get_scan(T, txSz, txType);
    int last = 0;
    for (int c = lane; c < n; c += 32) if (q[scan[c]]) last = c + 1;
    const int eob = warp_max(last);
    int cul = 0;
    for (int c = lane; c < eob; c += 32) cul += abs((int)q[scan[c]]);
    cul = min(warp_sum(cul), 63);
    const int dcCat = q[0] < 0 ? 1 : q[0] > 0 ? 2 : 0;
    const int ss = plane ? F.ssx : 0;
    const int stride = F.MiCols >> ss, rows = F.MiRows >> ss;
    const int w4 = W >> 2, h4 = H >> 2;
    for (int k = lane; k < w4 * h4; k += 32) {
        const int yy = y4 + k / w4, xx = x4 + k % w4;
        if (yy < rows && xx < stride) {
            F.cLvl[plane][(size_t)yy * stride + xx] = (uint8_t)(eob ? cul : 0);
            F.cDc[plane][(size_t)yy * stride + xx] = (uint8_t)(eob ? dcCat : 0);
        }
    }
    int16_t *oc = F.oCoeffs + (size_t)sb * SB_MAX_COEF + coefOff;
    for (int i = lane; i < n; i += 32) oc[i] = q[i];
    if (lane == 0) {
        av1g_txb t;
        t.coeff_off = (uint32_t)coefOff;
        t.x4 = (uint16_t)x4; t.y4 = (uint16_t)y4;
        t.plane = (uint8_t)plane; t.tx_size = (uint8_t)txSz;
        t.tx_type = (uint8_t)(plane == 0 && eob == 0 ? AV1G_DCT_DCT : txType);
        t.flags = 0; t.eob = (uint16_t)eob; t.reserved = 0;
        F.oTxb[(size_t)sb * SB_MAX_TXB + txbIdx] = t;
    }
    __syncwarp();
    return eob;
}

// txb skip / dc-sign contexts from the 4x4 maps (spec get_tx_size_context and the reference's txb_ctx,
// k_recon.cuh:204-238): lane k reads above entry k and left entry k (w4, h4 <= 16).  Split into the loads (issued with
// the other loads of a leaf) and the reduction.
struct CtxLd { int la, da, ll, dl; };
__device__ __forceinline__ CtxLd rc_txb_ctx_load(const FrameDesc &F, int plane, int txSz, int x4, int y4, int tileX4, int tileY4) {
    const int lane = lane_id();
    const int ss = plane ? F.ssx : 0;
    const int stride = F.MiCols >> ss, maxX4 = F.MiCols >> ss, maxY4 = F.MiRows >> ss;
    const bool hasAbove = y4 > (tileY4 >> ss), hasLeft = x4 > (tileX4 >> ss);
    const int w4 = txw(txSz) >> 2, h4 = txh(txSz) >> 2;
    const bool a = hasAbove && lane < w4 && x4 + lane < maxX4, l = hasLeft && lane < h4 && y4 + lane < maxY4;
    const uint8_t *Lv = F.cLvl[plane], *Dc = F.cDc[plane];
    CtxLd c;
    c.la = a ? __ldcg(Lv + (size_t)(y4 - 1) * stride + x4 + lane) : 0;
    c.da = a ? __ldcg(Dc + (size_t)(y4 - 1) * stride + x4 + lane) : 0;
    c.ll = l ? __ldcg(Lv + (size_t)(y4 + lane) * stride + x4 - 1) : 0;
    c.dl = l ? __ldcg(Dc + (size_t)(y4 + lane) * stride + x4 - 1) : 0;
    return c;
}
__device__ __forceinline__ void rc_txb_ctx_finish(const FrameDesc &F, const CtxLd &c, int plane, int txSz, int bsize, int *skipCtx, int *dcCtx) {
    const int ss = plane ? F.ssx : 0;
    const int w = txw(txSz), h = txh(txSz);
    const int la = c.la, da = c.da, ll = c.ll, dl = c.dl;
    const bool nzA = __any_sync(0xffffffffu, plane ? (la | da) != 0 : la != 0);
    const bool nzL = __any_sync(0xffffffffu, plane ? (ll | dl) != 0 : ll != 0);
    const int dcSign = warp_sum((da == 2) - (da == 1) + (dl == 2) - (dl == 1));
    *dcCtx = dcSign < 0 ? 1 : dcSign > 0 ? 2 : 0;
    if (plane == 0) {
        const bool gtA = __any_sync(0xffffffffu, la > 3), gtL = __any_sync(0xffffffffu, ll > 3);
        if (4 * bw4(bsize) == w && 4 * bh4(bsize) == h) *skipCtx = 0;
        else if (!nzA && !nzL) *skipCtx = 1;
        else if (!nzA || !nzL) *skipCtx = 2 + (gtA || gtL);
        else if (!gtA && !gtL) *skipCtx = 4;
        else if (!gtA || !gtL) *skipCtx = 5;
        else *skipCtx = 6;
    } else {
        const int ub = uv_bsize(bsize, ss);
        *skipCtx = (int)nzA + (int)nzL + 7 + ((16 * bw4(ub) * bh4(ub) > w * h) ? 3 : 0);
    }
}
__device__ __forceinline__ void rc_txb_ctx(const FrameDesc &F, int plane, int txSz, int x4, int y4, int bsize, int tileX4, int tileY4,
                                           int *skipCtx, int *dcCtx) {
    const CtxLd c = rc_txb_ctx_load(F, plane, txSz, x4, y4, tileX4, tileY4);
    rc_txb_ctx_finish(F, c, plane, txSz, bsize, skipCtx, dcCtx);
}

// a block of H rows of W bytes (<= 64; a W x H <= 32 x 32 block of samples) at src (row pitch in bytes) into dst (row
// stride W bytes), vector loads of up to 16 bytes (rows and the block's first byte are aligned to its width).  Coherent
// L2 loads, not the read-only path: a serving session's loop runs while new images are written into reused memory.
__device__ __forceinline__ void stage_block(const uint8_t *src, int pitch, int W, int H, uint8_t *dst) {
    const int lane = lane_id();
    if (W >= 16) {
        const int v = W >> 4;
        for (int k = lane; k < v * H; k += 32)
            reinterpret_cast<uint4 *>(dst)[k] = __ldcg(reinterpret_cast<const uint4 *>(src + (size_t)(k / v) * pitch) + (k % v));
    } else if (W == 8) {
        for (int k = lane; k < H; k += 32) reinterpret_cast<uint2 *>(dst)[k] = __ldcg(reinterpret_cast<const uint2 *>(src + (size_t)k * pitch));
    } else {
        for (int k = lane; k < H; k += 32) reinterpret_cast<uint32_t *>(dst)[k] = __ldcg(reinterpret_cast<const uint32_t *>(src + (size_t)k * pitch));
    }
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// The leaf decoded before leaf li of SB sb that covers the luma 4x4 unit (yy, xx) (SB-local; negative / >= 16 reach
// the SBs above, above-right and left) as sb << 8 | leaf, or -1: outside the tile or the frame, in the SBs below or to
// the right (decoded later), uncovered, or a later leaf of this SB.
__device__ __forceinline__ int unit_leaf(const FrameDesc &F, int sb, int li, int sbr, int sbc, int yy, int xx, int tC0, int tC1, int tR0) {
    const int Y = sbr * 16 + yy, X = sbc * 16 + xx;            // luma 4x4 unit, frame coordinates
    if (Y < tR0 || X < tC0 || X >= tC1 || Y >= F.MiRows || X >= F.MiCols) return -1;
    if (yy >= 16 || (yy >= 0 && xx >= 16)) return -1;
    int osb = sb, oy = yy, ox = xx;
    if (yy < 0 || xx < 0 || xx >= 16) { osb = (Y >> 4) * F.sbCols + (X >> 4); oy = Y & 15; ox = X & 15; }
    const int o = F.ordmap[(size_t)osb * 256 + oy * 16 + ox];
    if (o == 255 || (osb == sb && o >= li)) return -1;
    return osb * SB_MAX_LEAVES + o;
}

// Wait until the leaves decoded before leaf li of SB sb that cover the luma 4x4 units of two strips have published
// flag >= level: the row rTop, columns c0, c0 + st, ... < c1, and the column cLeft, rows r0, r0 + st, ... < r1 (the
// unit_leaf rule).  Returns false when a wait ran out of its budget or another warp reported an error (F.err set); the
// leaf is then abandoned.
static __device__ __noinline__ bool rc_wait(const FrameDesc &F, int sb, int li, int sbr, int sbc, int rTop, int c0, int c1, int cLeft, int r0,
                                     int r1, int st, int level, int tC0, int tC1, int tR0) {
    const int lane = lane_id();
    const int nTop = c1 > c0 ? (c1 - c0 + st - 1) / st : 0, nLeft = r1 > r0 ? (r1 - r0 + st - 1) / st : 0;
    bool ok = true;
    for (int u = lane; u < nTop + nLeft; u += 32) {
        const int yy = u < nTop ? rTop : r0 + (u - nTop) * st, xx = u < nTop ? c0 + u * st : cLeft;
        const int id = unit_leaf(F, sb, li, sbr, sbc, yy, xx, tC0, tC1, tR0);
        if (id < 0) continue;
        const int *flag = F.leafDone + id;
        int it = 0;
        while (ld_relaxed(flag) < level) {
            if (++it > F.waitIters || *(volatile int *)F.err) { ok = false; break; }
            __nanosleep(64);
        }
    }
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && lane == 0) atomicCAS(F.err, 0, KERR_WAIT_LEAF);
    if (ok) fence_acquire();   // every lane: its awaited flags were seen, the neighbours' data may be read now
    __syncwarp();
    return ok;
}

// Take the CTA's large buffer (RcBig; its holder gives it back right after its evaluation and waits on nothing while it
// holds it): a spin of at most F.waitIters polls.  False when it ran out or another warp reported an error (F.err set);
// the leaf is then abandoned.
__device__ __forceinline__ bool rc_big_lock(const FrameDesc &F, int &lock) {
    int ok = 1;
    if (lane_id() == 0) {
        int it = 0;
        while (atomicCAS(&lock, 0, 1) != 0) {
            if (++it > F.waitIters || *(volatile int *)F.err) { ok = 0; break; }
            __nanosleep(64);
        }
        if (!ok) atomicCAS(F.err, 0, KERR_WAIT_LEAF);
        __threadfence_block();   // the buffer's previous holder is done with it
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    return ok != 0;
}

// tile box (mi units) of the 4x4 unit (mi_row, mi_col)
__device__ __forceinline__ void tile_box(const FrameDesc &F, int mi_row, int mi_col, int &tC0, int &tC1, int &tR0, int &tR1) {
    int tc = 0, tr = 0;
    while (tc + 1 < F.tileCols && mi_col >= F.tileColStart[tc + 1]) tc++;
    while (tr + 1 < F.tileRows && mi_row >= F.tileRowStart[tr + 1]) tr++;
    tC0 = F.tileColStart[tc]; tC1 = F.tileColStart[tc + 1]; tR0 = F.tileRowStart[tr]; tR1 = F.tileRowStart[tr + 1];
}

// A queue slot given up by an idle worker of a serving session (the worker claimed it and left before a leaf came).
constexpr unsigned long long SLOT_ABANDONED = ~0ull;
// append leaf id (sb << 8 | leaf) of the image to the ready queue, after a fence that releases everything this thread
// wrote before (a running loop may take the leaf at once); a slot that an idle serving worker abandoned is skipped
__device__ __forceinline__ void push_ready(const FrameDesc &F, uint32_t id) {
    const unsigned long long v = 1ull + (((unsigned long long)F.img << 32) | id);
    fence_release();
    for (;;) {
        const int pos = atomicAdd(F.rq + 1, 1);
        if ((uint32_t)pos >= F.readyCap) {   // the queue's positions are used up: the image cannot complete
            atomicCAS(F.err, 0, KERR_CAPACITY);
            return;
        }
        if (atomicCAS(F.readyQ + pos, 0ull, v) == 0ull) break;
    }
}

// The further chroma tx blocks of plane pl of a 4:4:4 block with a 64-sample side (2 or 4 per plane in raster order;
// the first is coded by the caller, the block's mode bestC chosen on it): each takes its edges from the reconstruction
// (the block's earlier tx blocks included), its own coefficient contexts and a closed-loop quantisation of the chosen
// mode (the reference's rc_chroma, k_recon.cuh:1636-1678); tx blocks that start outside the coded area are not coded.
// tIdx counts the leaf's coded chroma tx blocks (txb slot txb0 + tIdx, coefficients at coef0 + tIdx x the tx area).
// Returns the OR of the eobs.
template <int BD, typename Px>
__device__ __noinline__ int rc_chroma_more(const FrameDesc &F, RcWarp<Px, 0> &Wp, const RateTabs &T, int sb, int li, int pl, int txSz, int uvType,
                                           int bestC, int bsize, int cx, int cy, int csr, int csc, int nTxX, int nTxY, int availLC, int availUC,
                                           int tC0, int tR0, int sbW4, int sbH4, int txb0, int coef0, int *tIdx) {
    const int lane = lane_id();
    const int W = txw(txSz), H = txh(txSz), lw = 31 - __clz(W), lh = 31 - __clz(H), nq = min(W, 32) * min(H, 32);
    const int bw = bw4(bsize), bh = bh4(bsize);
    const int cx4 = cx >> 2, cy4 = cy >> 2, cCols4 = F.MiCols, cRows4 = F.MiRows;   // 4:4:4: plane units = luma units
    const uint8_t *ordmap = F.ordmap + (size_t)sb * 256;
    int eobs = 0;
    for (int t = 1; t < nTxX * nTxY; t++) {
        const int tx = t % nTxX, ty = t / nTxX, ox = tx * W, oy = ty * H;
        if (cx4 + (ox >> 2) >= cCols4 || cy4 + (oy >> 2) >= cRows4) continue;
        const int r4 = csr + (oy >> 2), c4 = csc + (ox >> 2);   // SB-relative 4x4 units
        // BlockDecoded: the leaves before this one (the SB's leaf map and its above / left rule), and this leaf's tx
        // blocks before t
        auto dec = [&](int yy, int xx) -> bool {
            if (yy >= csr && xx >= csc && yy < csr + bh && xx < csc + bw) return ((yy - csr) * 4 / H) * nTxX + ((xx - csc) * 4 / W) < t;
            if (yy < 0) return xx < sbW4;
            if (xx < 0) return yy < sbH4 && yy != 16;
            if (yy >= 16 || xx >= 16) return false;
            return ordmap[yy * 16 + xx] < li;
        };
        const int haveL = availLC || tx > 0, haveA = availUC || ty > 0;
        const int haveAR = dec(r4 - 1, c4 + (W >> 2)), haveBL = dec(r4 + (H >> 2), c4 - 1);
        Px *A = Wp.ea[pl] + EDGE_OFF, *L = Wp.el[pl] + EDGE_OFF;
        rc_edges_rec<BD, Px>(F, pl, cx + ox, cy + oy, W, H, haveL, haveA, haveAR, haveBL, A, L);
        const int dcv = warp_dc<BD>(A, L, haveL, haveA, lw, lh);
        const int m = cand_mode(bestC);
        grp_predict(m, pangle(m, cand_delta(bestC)), lw, lh, A, L, dcv, Wp.pred, lane, 32);
        __syncwarp();
        __threadfence_block();   // the context maps of this leaf's earlier tx blocks (written by this warp)
        int sc, dcc;
        rc_txb_ctx(F, pl, txSz, cx4 + (ox >> 2), cy4 + (oy >> 2), bsize, tC0, tR0, &sc, &dcc);
        const EvalIn e{uvType, pl, sc, dcc, 0, F.dcQ, F.acQ, T};
        const Px *so = (const Px *)F.src[pl] + (size_t)(cy + oy) * F.spitch[pl] + cx + ox;
        int16_t *lv = Wp.qb[pl - 1];
        grp_eval<BD, Px>(txSz, ResFn<Px>{so, F.spitch[pl], Wp.pred, lw, nullptr}, e, Wp.buf, lv, lane, 32);
        Px *dst = (Px *)F.rec[pl] + (size_t)(cy + oy) * F.rpitch[pl] + cx + ox;
        rc_reconstruct<BD, Px>(txSz, uvType, lv, F.dcQ, F.acQ, Wp.pred, dst, F.rpitch[pl], Wp.buf);
        eobs |= rc_record(F, T, sb, pl, txSz, uvType, cx4 + (ox >> 2), cy4 + (oy >> 2), lv, txb0 + *tIdx, coef0 + *tIdx * nq);
        (*tIdx)++;
    }
    return eobs;
}

template <int BD, typename Px, int SS>
__device__ void rc_leaf(const FrameDesc &F, RcWarp<Px, SS> &Wp, RcBig<Px> &Big, const RateTabs &T, int sb, int li, unsigned long long *trace) {
    const int lane = lane_id();
    const Leaf lf = F.leaves[(size_t)sb * SB_MAX_LEAVES + li];
    const int bsize = lf.bsize;
    const int sbr = sb / F.sbCols, sbc = sb % F.sbCols;
    const int sbx = sbc * 64, sby = sbr * 64;
    const int x = sbx + lf.x4 * 4, y = sby + lf.y4 * 4, mi_row = y >> 2, mi_col = x >> 2;
    const int bw = bw4(bsize), bh = bh4(bsize);
    const int ss = SS;   // (the image's F.ssx: one instance per subsampling)
    const uint8_t *ordmap = F.ordmap + (size_t)sb * 256;
    int tC0, tC1, tR0, tR1;
    tile_box(F, mi_row, mi_col, tC0, tC1, tR0, tR1);
    // (the leaf came from the ready queue: the luma of every leaf of luma_deps() is published)
    const int availU = mi_row - 1 >= tR0, availL = mi_col - 1 >= tC0;
    const bool hasC = has_chroma(bsize, mi_row, mi_col, ss);
    const int availUC = (ss && bh == 1) ? (mi_row - 2 >= tR0) : availU;
    const int availLC = (ss && bw == 1) ? (mi_col - 2 >= tC0) : availL;
    const uint16_t *C = T.cost;
    const uint32_t me = (uint32_t)sb * SB_MAX_LEAVES + li;
    const int txbBase = F.leafTxb[me], coefBase = F.leafCoef[me];
    // the leaf's dependents (prefetched here, used when its luma is published)
    const int relN = F.revCnt[me];
    const uint32_t relOff = F.revOff[me];
    // BlockDecoded of a 4x4 unit (SB-relative, plane units; ps = 0 luma, ss chroma) for this leaf
    auto decoded = [&](int ps, int yy, int xx) -> bool {
        const int sz = 16 >> ps;
        const int sbW4 = (tC1 - sbc * 16) >> ps, sbH4 = (tR1 - sbr * 16) >> ps;
        if (yy < 0) return xx < sbW4;
        if (xx < 0) return yy < sbH4 && yy != sz;
        if (yy >= sz || xx >= sz) return false;
        const int o = ps ? ordmap[((yy << ps) + 1) * 16 + (xx << ps) + 1] : ordmap[yy * 16 + xx];
        return o < li;
    };
    // ================= luma =================
    int yMode, yDelta, eobY;
    {
        const int txSz = ST(Max_Tx_Size_Rect)[bsize];
        const int W = txw(txSz), H = txh(txSz), lw = 31 - __clz(W), lh = 31 - __clz(H);
        // ---- the luma's global loads, issued together (one round of memory latency): the raw edge samples up to the
        //      longest reach, the analysis record, the neighbours' y modes, the coefficient-context maps, the
        //      decoded-ness of the above-right / below-left units, the source block ----
        const Px *recY = (const Px *)F.rec[0];
        const int rp = F.rpitch[0], n = W + H;
        const int aLim = min(x + 2 * W - 1, F.MiCols * 4 - 1), lLim = min(y + 2 * H - 1, F.MiRows * 4 - 1);
        Px ra[4], rl[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int i = lane + 32 * k;
            ra[k] = i < n ? ldcg(recY + (size_t)(y - 1) * rp + min(x + i, aLim)) : (Px)0;
            rl[k] = i < n ? ldcg(recY + (size_t)min(y + i, lLim) * rp + x - 1) : (Px)0;
        }
        const Px rcorner = ldcg(recY + (size_t)(y - 1) * rp + x - 1);
        const BlockRes br = F.blk[F.shOff[bsize] + (uint32_t)(y / H) * F.shNbx[bsize] + x / W];
        const int ymA = availU ? __ldcg(F.mYMode + (size_t)(mi_row - 1) * F.MiCols + mi_col) : AV1G_DC_PRED;
        const int ymL = availL ? __ldcg(F.mYMode + (size_t)mi_row * F.MiCols + mi_col - 1) : AV1G_DC_PRED;
        const CtxLd cl = rc_txb_ctx_load(F, 0, txSz, x >> 2, y >> 2, tC0, tR0);
        const int haveAR = decoded(0, lf.y4 - 1, lf.x4 + (W >> 2)), haveBL = decoded(0, lf.y4 + (H >> 2), lf.x4 - 1);
        const bool staged = W <= 32 && H <= 32;
        if (staged)
            stage_block((const uint8_t *)((const Px *)F.src[0] + (size_t)y * F.spitch[0] + x), F.spitch[0] * (int)sizeof(Px), W * (int)sizeof(Px), H,
                        (uint8_t *)Wp.srcS[0]);
        // ---- the edges: rec_edges' rule (availability, above-right / below-left reach, frame clamp) on the raw samples ----
        Px *A = Wp.ea[0] + EDGE_OFF, *L = Wp.el[0] + EDGE_OFF;
        {
            const Px aW = (Px)__shfl_sync(0xffffffffu, (int)(W > 32 ? ra[1] : ra[0]), (W - 1) & 31);
            const Px lH = (Px)__shfl_sync(0xffffffffu, (int)(H > 32 ? rl[1] : rl[0]), (H - 1) & 31);
            const Px a0 = (Px)__shfl_sync(0xffffffffu, (int)ra[0], 0), l0 = (Px)__shfl_sync(0xffffffffu, (int)rl[0], 0);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int i = lane + 32 * k;
                if (i < n) {
                    A[i] = availU ? ((!haveAR && i >= W) ? aW : ra[k]) : (availL ? l0 : (Px)((1 << (BD - 1)) - 1));
                    L[i] = availL ? ((!haveBL && i >= H) ? lH : rl[k]) : (availU ? a0 : (Px)((1 << (BD - 1)) + 1));
                }
            }
            if (lane == 0) {
                const Px c = (availU && availL) ? rcorner : availU ? a0 : availL ? l0 : (Px)(1 << (BD - 1));
                A[-1] = c;
                L[-1] = c;
            }
        }
        __syncwarp();
        const int dcv = warp_dc<BD>(A, L, availL, availU, lw, lh);
        int skipCtx, dcCtx;
        rc_txb_ctx_finish(F, cl, 0, txSz, bsize, &skipCtx, &dcCtx);
        const int am = ST(Intra_Mode_Context)[ymA], lm = ST(Intra_Mode_Context)[ymL];
        auto mbits = [&](int c) -> int {
            const int m = cand_mode(c);
            int b = C[ci_y_mode(am, lm) + m];
            if (bsize >= AV1G_BLOCK_8X8 && is_dir(m)) b += C[ci_angle(m - AV1G_V_PRED) + cand_delta(c) + 3];
            return b;
        };
        const Px *src = staged ? (const Px *)Wp.srcS[0] : (const Px *)F.src[0] + (size_t)y * F.spitch[0] + x;
        const int srcPitch = staged ? W : F.spitch[0];
        const int set = tx_set_intra(txSz);
        const int nq = min(W, 32) * min(H, 32);
        // scratch of the evaluation rounds, the prediction and the inverse: the warp's own, or for a tx size with a
        // 64-sample side the CTA's large buffer, taken under its lock for the evaluation only (its holder waits on
        // nothing until it gives it back)
        const bool bigTx = W == 64 || H == 64;
        if (bigTx && !rc_big_lock(F, Big.lock)) return;   // (the wait ran out: the error is recorded)
        int32_t *lbuf = bigTx ? Big.buf : Wp.buf;
        Px *lpred = bigTx ? Big.pred : Wp.pred;
        int16_t *best = Wp.qb[0];
        i64 bestJ = INF;
        int bestC = br.cand[0], bestT = br.tx;
        bool have = false;
        int curG = 0;
        // tasks (candidate, tx type) in rounds of 32 / G (G per pass: round_group); costs compared in task order (first
        // of equal costs wins); the round's winner, if it beats the best so far, leaves its levels in `best`
        auto run = [&](const int *tcand, const int *ttype, int n) {
            const int G = round_group(txSz, n), ng = 32 / G, grp = lane / G, g = lane & (G - 1);
            int32_t *tb = lbuf + grp * task_buf_ints(txSz);
            int16_t *tq = Wp.q + grp * nq;
            Px *tp = lpred + grp * (W * H);
            if (G != curG) {   // the groups' cached predictions belong to another grouping
                if (lane < 8) Wp.predC[lane] = -1;
                __syncwarp();
                curG = G;
            }
            for (int r0 = 0; r0 < n; r0 += ng) {
                const int k = min(r0 + grp, n - 1);
                const int c = tcand[k], t = ttype[k], m = cand_mode(c);
                if (Wp.predC[grp] != c) grp_predict(m, pangle(m, cand_delta(c)), lw, lh, A, L, dcv, tp, g, G);
                __syncwarp();
                if (g == 0) Wp.predC[grp] = c;
                const EvalIn e{t, 0, skipCtx, dcCtx, m, F.dcQ, F.acQ, T};
                const EvalOut o = grp_eval<BD, Px>(txSz, ResFn<Px>{src, srcPitch, tp, lw, nullptr}, e, tb, tq, g, G);
                if (g == 0 && r0 + grp < n) Wp.taskJ[grp] = o.D + F.lam * (o.R + mbits(c));
                __syncwarp();
                int win = -1;
                for (int u = 0; u < ng && r0 + u < n; u++)
                    if (Wp.taskJ[u] < bestJ) { bestJ = Wp.taskJ[u]; bestC = tcand[r0 + u]; bestT = ttype[r0 + u]; win = u; have = true; }
                if (win >= 0)
                    for (int i = lane; i < nq; i += 32) best[i] = Wp.q[win * nq + i];
                __syncwarp();
            }
        };
        const int nc = max(1, min((int)br.ncand, K_RECHECK));
        // the types pass 2 may try for cand[0]: its open-loop shortlist (with DCT_DCT and the analysis' type), or all
        const uint32_t txAllow = br.txMask ? (uint32_t)br.txMask | (1u << AV1G_DCT_DCT) | (1u << br.tx) : 0xFFFFu;
        int tcand[8], ttype[8], n1 = 0;
        for (int k = 0; k < nc; k++) { tcand[n1] = br.cand[k]; ttype[n1] = AV1G_DCT_DCT; n1++; }
        if (br.tx != AV1G_DCT_DCT) { tcand[n1] = br.cand[0]; ttype[n1] = br.tx; n1++; }
        const bool skip1 = n1 == 1;
        if (trace && lane == 0) trace[2] = gtimer();
        if (W * H <= 64 && set != AV1G_TX_SET_DCTONLY) {
            // Small tx sizes (4x4 .. 8x8, 4x16, 16x4; nine leaves in ten): pass 1 and the pass-2 tx types of BOTH possible
            // pass-1 winners in one round of at most 16 tasks (2 lanes each), then the winner taken in the order of the two
            // passes - pass 1 in task order, then pass 2 of the pass-1 winner in type order, the first of equal costs -
            // which is exactly the result of running pass 2 after pass 1.  A round's latency hardly depends on its task
            // count, so this saves the second round.
            const int c0 = br.cand[0], c1 = nc >= 2 ? br.cand[1] : br.cand[0];
            const int tt = lane & 15;   // pass-2 types: lanes 0-15 for the first candidate, 16-31 for the second
            const bool ok = lane < 16 ? tx_in_set(set, tt) && ((txAllow >> tt) & 1) && !(!skip1 && (tt == AV1G_DCT_DCT || tt == br.tx))
                                      : nc >= 2 && tx_in_set(set, tt) && tt != AV1G_DCT_DCT;
            const unsigned bal = __ballot_sync(0xffffffffu, ok), m0 = bal & 0xFFFFu, m1 = bal >> 16;
            const int p1 = skip1 ? 0 : n1, n2a = __popc(m0), n2b = __popc(m1), nt = p1 + n2a + n2b;
            const int G = nt > 8 ? 2 : nt > 4 ? 4 : 8, grp = lane / G, g = lane & (G - 1);
            {   // every lane takes part (the evaluation's warp-wide reductions); groups past the last task repeat it
                const int k = min(grp, nt - 1);
                int c, ty;
                if (k < p1) { c = k < nc ? (int)br.cand[k] : c0; ty = k < nc ? AV1G_DCT_DCT : br.tx; }
                else if (k < p1 + n2a) { c = c0; ty = __fns(m0, 0, k - p1 + 1); }
                else { c = c1; ty = __fns(m1, 0, k - p1 - n2a + 1); }
                const int m = cand_mode(c);
                Px *tp = lpred + grp * (W * H);
                grp_predict(m, pangle(m, cand_delta(c)), lw, lh, A, L, dcv, tp, g, G);
                __syncwarp();
                const EvalIn e{ty, 0, skipCtx, dcCtx, m, F.dcQ, F.acQ, T};
                const EvalOut o = grp_eval<BD, Px>(txSz, ResFn<Px>{src, srcPitch, tp, lw, nullptr}, e, lbuf + grp * task_buf_ints(txSz),
                                                   Wp.q + grp * nq, g, G);
                if (g == 0 && grp < nt) Wp.taskJ[grp] = o.D + F.lam * (o.R + mbits(c));
            }
            __syncwarp();
            int win = -1;
            if (!skip1) {
                for (int k = 0; k < p1; k++)
                    if (Wp.taskJ[k] < bestJ) { bestJ = Wp.taskJ[k]; bestC = k < nc ? (int)br.cand[k] : c0; bestT = k < nc ? AV1G_DCT_DCT : br.tx; win = k; }
            } else {
                bestC = c0; bestT = AV1G_DCT_DCT;
            }
            const bool first = bestC == c0;
            const int base = first ? p1 : p1 + n2a, cnt = first ? n2a : n2b;
            const unsigned mk = first ? m0 : m1;
            for (int j = 0; j < cnt; j++)
                if (Wp.taskJ[base + j] < bestJ) { bestJ = Wp.taskJ[base + j]; bestT = __fns(mk, 0, j + 1); win = base + j; }
            if (win >= 0) {
                have = true;
                for (int i = lane; i < nq; i += 32) best[i] = Wp.q[win * nq + i];
            }
            __syncwarp();
            if (trace && lane == 0) trace[3] = trace[4] = gtimer();
        } else {
        if (!skip1) run(tcand, ttype, n1);
        else { bestC = br.cand[0]; bestT = AV1G_DCT_DCT; }
        if (trace && lane == 0) trace[3] = gtimer();
        if (set != AV1G_TX_SET_DCTONLY) {
            const int c1 = bestC;
            const bool isC0 = c1 == br.cand[0];
            int n2 = 0;
            for (int t = 0; t < 16; t++) {
                if (!tx_in_set(set, t)) continue;
                if (!skip1 && (t == AV1G_DCT_DCT || (isC0 && t == br.tx))) continue;
                if (isC0 && !((txAllow >> t) & 1)) continue;
                tcand[n2] = c1; ttype[n2] = t; n2++;
            }
            run(tcand, ttype, n2);
        }
        if (trace && lane == 0) trace[4] = gtimer();
        }
        // the winner's prediction (whole warp) for its levels (single-candidate case) and the reconstruction
        const int bm = cand_mode(bestC);
        grp_predict(bm, pangle(bm, cand_delta(bestC)), lw, lh, A, L, dcv, lpred, lane, 32);
        __syncwarp();
        if (!have) {
            const EvalIn e{bestT, 0, skipCtx, dcCtx, bm, F.dcQ, F.acQ, T};
            grp_eval<BD, Px>(txSz, ResFn<Px>{src, srcPitch, lpred, lw, nullptr}, e, lbuf, best, lane, 32);
        }
        Px *dst = (Px *)F.rec[0] + (size_t)y * F.rpitch[0] + x;
        rc_reconstruct<BD, Px>(txSz, bestT, best, F.dcQ, F.acQ, lpred, dst, F.rpitch[0], lbuf);
        if (bigTx) {   // the large buffer back (the reconstruction is written; the levels are in the warp's own qb)
            __syncwarp();
            if (lane == 0) {
                __threadfence_block();
                atomicExch(&Big.lock, 0);
            }
        }
        eobY = rc_record(F, T, sb, 0, txSz, bestT, x >> 2, y >> 2, best, txbBase, coefBase);
        yMode = bm;
        yDelta = cand_delta(bestC);
        for (int k = lane; k < bw * bh; k += 32) {
            const int r = mi_row + k / bw, c = mi_col + k % bw;
            if (r < F.MiRows && c < F.MiCols) F.mYMode[(size_t)r * F.MiCols + c] = (uint8_t)yMode;
        }
    }
    // publish the luma (reconstruction, y modes, luma coefficient contexts) for the luma of the later leaves
    __syncwarp();
    if (lane == 0) {   // (the release store is cumulative: it also releases the other lanes' writes, ordered by the barrier)
        st_release(F.leafDone + (size_t)sb * SB_MAX_LEAVES + li, 1);
        if (trace) trace[5] = gtimer();
    }
    {   // the dependents whose last luma dependency this was enter the ready queue (the taker of a leaf acquires each of
        // its dependencies' flags itself before it reads their data; push_ready releases what this thread wrote)
        __syncwarp();
        for (int k = lane; k < relN; k += 32) {
            const uint32_t d = F.revList[relOff + k];
            if (atomicSub(F.depCnt + d, 1) == 1) push_ready(F, d);
        }
    }
    // ================= chroma =================
    int uv = 0, duv = 0, aU = 0, aV = 0, eobU = 0, eobV = 0;
    if (hasC) {
        // chroma neighbourhood: the leaves carrying the chroma units above (from the above-left corner to the above-right
        // reach of 2 x chroma width) and left (to the below-left reach of 2 x chroma height) are done (flag 2); with
        // subsampling a chroma unit's carrier covers the bottom-right luma unit of its 2 x 2 area
        if (ss) {
            const int cx0 = lf.x4 & ~1, cy0 = lf.y4 & ~1, cw = max(bw, 2), ch = max(bh, 2);
            if (!rc_wait(F, sb, li, sbr, sbc, cy0 - 1, cx0 - 1, cx0 + 2 * cw, cx0 - 1, cy0 + 1, cy0 + 2 * ch, 2, 2, tC0, tC1, tR0)) return;
        } else {
            if (!rc_wait(F, sb, li, sbr, sbc, lf.y4 - 1, lf.x4 - 1, lf.x4 + 2 * bw, lf.x4 - 1, lf.y4, lf.y4 + 2 * bh, 1, 2, tC0, tC1, tR0)) return;
        }
        if (trace && lane == 0) trace[6] = gtimer();
        const int txSz = uv_tx_size(bsize, ss);
        const int W = txw(txSz), H = txh(txSz), lw = 31 - __clz(W), lh = 31 - __clz(H);
        const int cx = (mi_col >> ss) * 4, cy = (mi_row >> ss) * 4, cx4 = cx >> 2, cy4 = cy >> 2;
        const int csr = (mi_row & 15) >> ss, csc = (mi_col & 15) >> ss;
        // ---- the chroma's global loads, issued together: raw U / V edge samples up to the longest reach, the
        //      coefficient-context maps, the decoded-ness of the above-right / below-left units, the U / V sources ----
        const int n = W + H;   // <= 64
        const int aLim = min(cx + 2 * W - 1, ((F.MiCols * 4) >> ss) - 1), lLim = min(cy + 2 * H - 1, ((F.MiRows * 4) >> ss) - 1);
        Px ra[2][2], rl[2][2], rcorner[2];
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const Px *rp = (const Px *)F.rec[1 + q];
            const int pitch = F.rpitch[1 + q];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int i = lane + 32 * k;
                ra[q][k] = i < n ? ldcg(rp + (size_t)(cy - 1) * pitch + min(cx + i, aLim)) : (Px)0;
                rl[q][k] = i < n ? ldcg(rp + (size_t)min(cy + i, lLim) * pitch + cx - 1) : (Px)0;
            }
            rcorner[q] = ldcg(rp + (size_t)(cy - 1) * pitch + cx - 1);
        }
        const CtxLd cl1 = rc_txb_ctx_load(F, 1, txSz, cx4, cy4, tC0, tR0), cl2 = rc_txb_ctx_load(F, 2, txSz, cx4, cy4, tC0, tR0);
        const int haveAR = decoded(ss, csr - 1, csc + (W >> 2)), haveBL = decoded(ss, csr + (H >> 2), csc - 1);
        for (int q = 1; q <= 2; q++)
            stage_block((const uint8_t *)((const Px *)F.src[q] + (size_t)cy * F.spitch[q] + cx), F.spitch[q] * (int)sizeof(Px), W * (int)sizeof(Px), H,
                        (uint8_t *)Wp.srcS[q]);
        // ---- the edges of U and V (rec_edges' rule on the raw samples) ----
        Px *A[3], *L[3];
        int dcv[3];
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int pl = 1 + q;
            A[pl] = Wp.ea[pl] + EDGE_OFF; L[pl] = Wp.el[pl] + EDGE_OFF;
            const Px aW = (Px)__shfl_sync(0xffffffffu, (int)(W > 32 ? ra[q][1] : ra[q][0]), (W - 1) & 31);
            const Px lH = (Px)__shfl_sync(0xffffffffu, (int)(H > 32 ? rl[q][1] : rl[q][0]), (H - 1) & 31);
            const Px a0 = (Px)__shfl_sync(0xffffffffu, (int)ra[q][0], 0), l0 = (Px)__shfl_sync(0xffffffffu, (int)rl[q][0], 0);
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int i = lane + 32 * k;
                if (i < n) {
                    A[pl][i] = availUC ? ((!haveAR && i >= W) ? aW : ra[q][k]) : (availLC ? l0 : (Px)((1 << (BD - 1)) - 1));
                    L[pl][i] = availLC ? ((!haveBL && i >= H) ? lH : rl[q][k]) : (availUC ? a0 : (Px)((1 << (BD - 1)) + 1));
                }
            }
            if (lane == 0) {
                const Px c = (availUC && availLC) ? rcorner[q] : availUC ? a0 : availLC ? l0 : (Px)(1 << (BD - 1));
                A[pl][-1] = c;
                L[pl][-1] = c;
            }
        }
        __syncwarp();
        for (int pl = 1; pl <= 2; pl++) dcv[pl] = warp_dc<BD>(A[pl], L[pl], availLC, availUC, lw, lh);
        // the staged sources (row stride W)
        const Px *sP[3] = {nullptr, (const Px *)Wp.srcS[1], (const Px *)Wp.srcS[2]};
        const bool cflAllowed = bw <= 8 && bh <= 8;
        auto uvbits = [&](int m) -> int { return cflAllowed ? C[ci_uv_cfl(yMode) + m] : C[ci_uv_nocfl(yMode) + m]; };
        auto uvcbits = [&](int c) -> int {
            const int m = cand_mode(c);
            int b = uvbits(m);
            if (bsize >= AV1G_BLOCK_8X8 && is_dir(m)) b += C[ci_angle(m - AV1G_V_PRED) + cand_delta(c) + 3];
            return b;
        };
        // ---- CfL (spec 7.11.5 luma values; least-squares alpha, then the best of alpha - 1 .. + 1 by SSE) ----
        int alpha[3] = {0, 0, 0}, cflAvg = 0;
        if (cflAllowed) {
            const int maxLumaW = x + 4 * bw, maxLumaH = y + 4 * bh;   // tx_depth 0: one luma tx block, starting inside
            const Px *luma = (const Px *)F.rec[0];
            const int lp = F.rpitch[0];
            int sum = 0;
            for (int p = lane; p < W * H; p += 32) {
                const int i = p >> lw, j = p & (W - 1);
                int v;
                if (ss) {
                    const int ly = min((cy + i) << 1, maxLumaH - 2), lx = min((cx + j) << 1, maxLumaW - 2);
                    v = ((int)ldcg(luma + (size_t)ly * lp + lx) + ldcg(luma + (size_t)ly * lp + lx + 1) + ldcg(luma + (size_t)(ly + 1) * lp + lx) +
                         ldcg(luma + (size_t)(ly + 1) * lp + lx + 1)) << 1;
                } else {
                    v = (int)ldcg(luma + (size_t)min(cy + i, maxLumaH - 1) * lp + min(cx + j, maxLumaW - 1)) << 3;
                }
                Wp.cfl[p] = (int16_t)v;
                sum += v;
            }
            sum = warp_sum(sum);
            cflAvg = (sum + (1 << (lw + lh - 1))) >> (lw + lh);
            __syncwarp();
            i64 num1 = 0, num2 = 0, den = 0;
            for (int p = lane; p < W * H; p += 32) {
                const int i = p >> lw, j = p & (W - 1);
                const i64 l = Wp.cfl[p] - cflAvg;
                num1 += l * ((int)sP[1][i * W + j] - dcv[1]);
                num2 += l * ((int)sP[2][i * W + j] - dcv[2]);
                den += l * l;
            }
            num1 = warp_sum64(num1); num2 = warp_sum64(num2); den = warp_sum64(den);
            for (int pl = 1; pl <= 2; pl++) {
                const i64 num = pl == 1 ? num1 : num2;
                int a = 0;
                if (den > 0) {
                    const i64 n = 64 * num;
                    a = (int)(n >= 0 ? (2 * n + den) / (2 * den) : -((-2 * n + den) / (2 * den)));
                }
                a = max(-16, min(16, a));
                i64 sse[3] = {0, 0, 0};
                for (int p = lane; p < W * H; p += 32) {
                    const int i = p >> lw, j = p & (W - 1);
                    const int l = Wp.cfl[p] - cflAvg, s = sP[pl][i * W + j];
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        const int ak = max(-16, min(16, a + k - 1));
                        const int v = ak * l, sc = v >= 0 ? (v + 32) >> 6 : -((-v + 32) >> 6);
                        const int pr = min(max(dcv[pl] + sc, 0), (1 << BD) - 1);
                        sse[k] += (i64)(s - pr) * (s - pr);
                    }
                }
                for (int k = 0; k < 3; k++) sse[k] = warp_sum64(sse[k]);
                int bk = 1;
                for (int k = 0; k < 3; k++) if (sse[k] < sse[bk]) bk = k;
                alpha[pl] = max(-16, min(16, a + bk - 1));
            }
        }
        // ---- SATD screening of the UV modes over U and V ----
        const int nsx = W >> 2, nsub2 = 2 * (W >> 2) * (H >> 2);   // items per candidate: U then V 4x4 sub-blocks
        auto screen = [&](int c0, int c1) {
            const int items = (c1 - c0) * nsub2;
            for (int it0 = 0; it0 < items; it0 += 32) {
                const int it = it0 + lane;
                const int ci = c0 + it / nsub2;
                int t = 0;
                if (it < items) {
                    const int r = it % nsub2, pl = 1 + (r >= (nsub2 >> 1)), sbk = r % (nsub2 >> 1);
                    const int sx = (sbk % nsx) * 4, sy = (sbk / nsx) * 4;
                    const int c = Wp.cand[ci], m = cand_mode(c);
                    t = pred4_satd(m, pangle(m, cand_delta(c)), sy, sx, lw, lh, A[pl], L[pl], dcv[pl], sP[pl], W);
                }
                for (int o = 16; o > 0; o >>= 1)
                    if (o < nsub2) t += __shfl_xor_sync(0xffffffffu, t, o);
                if (it < items && (lane & (nsub2 - 1)) == 0) Wp.satd[ci] += t;
                __syncwarp();
            }
        };
        Wp.satd[lane] = 0;
        Wp.cand[lane] = lane < 13 ? cand_pack(lane, 0) : 0;
        __syncwarp();
        screen(0, 13);
        i64 js = lane < 13 ? ((i64)Wp.satd[lane] << 14) + F.sqlam * uvcbits(Wp.cand[lane]) : INF;
        if (bsize >= AV1G_BLOCK_8X8) {
            const int bm = warp_argmin((lane >= AV1G_V_PRED && lane <= AV1G_D67_PRED) ? js : INF, lane);
            if (lane < 6) Wp.cand[13 + lane] = cand_pack(bm, lane < 3 ? -(lane + 1) : (lane - 2));
            __syncwarp();
            screen(13, 19);
            if (lane >= 13 && lane < 19) js = ((i64)Wp.satd[lane] << 14) + F.sqlam * uvcbits(Wp.cand[lane]);
        }
        int chosen[UV_K + 1], nch = 0;
        for (int k = 0; k < UV_K; k++) {
            const int b = warp_argmin(js, lane);
            if (b < 0) break;
            chosen[nch++] = Wp.cand[b];
            if (lane == b) js = INF;
        }
        if (cflAllowed && (alpha[1] || alpha[2])) chosen[nch++] = 255;
        int skipCtx[3], dcCtx[3];
        rc_txb_ctx_finish(F, cl1, 1, txSz, bsize, &skipCtx[1], &dcCtx[1]);
        rc_txb_ctx_finish(F, cl2, 2, txSz, bsize, &skipCtx[2], &dcCtx[2]);
        // prediction of (plane, candidate) by a group of G lanes into out
        auto predict = [&](int pl, int c, Px *out, int g, int G) {
            if (c == 255) grp_predict_cfl(lw, lh, dcv[pl], Wp.cfl, alpha[pl], cflAvg, (1 << BD) - 1, out, g, G);
            else grp_predict(cand_mode(c), pangle(cand_mode(c), cand_delta(c)), lw, lh, A[pl], L[pl], dcv[pl], out, g, G);
        };
        // (candidate, plane) tasks in rounds of 32 / G; each candidate's cost = U + V + lambda * its mode bits; the
        // winner's two planes are evaluated once more for their levels
        const int nq = min(W, 32) * min(H, 32);
        i64 pj[2 * (UV_K + 1)];
        const int ntask = 2 * nch;
        const int G = round_group(txSz, ntask), ng = 32 / G, grp = lane / G, g = lane & (G - 1);
        int32_t *tb = Wp.buf + grp * task_buf_ints(txSz);
        int16_t *tq = Wp.q + grp * nq;
        Px *tp = Wp.pred + grp * (W * H);
        for (int r0 = 0; r0 < ntask; r0 += ng) {
            const int k = min(r0 + grp, ntask - 1), c = chosen[k >> 1], pl = 1 + (k & 1);
            predict(pl, c, tp, g, G);
            __syncwarp();
            const int txType = chroma_tx_type(txSz, c == 255 ? AV1G_UV_CFL_PRED : cand_mode(c));
            const EvalIn e{txType, pl, skipCtx[pl], dcCtx[pl], 0, F.dcQ, F.acQ, T};
            const EvalOut o = grp_eval<BD, Px>(txSz, ResFn<Px>{sP[pl], W, tp, lw, nullptr}, e, tb, tq, g, G);
            if (g == 0 && r0 + grp < ntask) Wp.taskJ[grp] = o.D + F.lam * o.R;
            __syncwarp();
            for (int u = 0; u < ng && r0 + u < ntask; u++) pj[r0 + u] = Wp.taskJ[u];
            __syncwarp();
        }
        i64 bJ = INF;
        int bestC = cand_pack(AV1G_DC_PRED, 0);
        for (int k = 0; k < nch; k++) {
            const int c = chosen[k];
            i64 J = pj[2 * k] + pj[2 * k + 1];
            int b;
            if (c == 255) {
                const int a1 = alpha[1], a2 = alpha[2];
                const int sU = a1 == 0 ? 0 : a1 < 0 ? 1 : 2, sV = a2 == 0 ? 0 : a2 < 0 ? 1 : 2;
                b = uvbits(AV1G_UV_CFL_PRED) + C[ci_cfl_sign() + sU * 3 + sV - 1];
                if (sU) b += C[ci_cfl_alpha((sU - 1) * 3 + sV) + abs(a1) - 1];
                if (sV) b += C[ci_cfl_alpha((sV - 1) * 3 + sU) + abs(a2) - 1];
            } else {
                b = uvcbits(c);
            }
            J += F.lam * b;
            if (J < bJ) { bJ = J; bestC = c; }
        }
        if (trace && lane == 0) trace[7] = gtimer();
        const bool cfl = bestC == 255;
        uv = cfl ? AV1G_UV_CFL_PRED : cand_mode(bestC);
        const int uvType = chroma_tx_type(txSz, uv);
        // chroma tx blocks per plane (the reference's rc_chroma, k_recon.cuh:1588-1680): one in 4:2:0 and in 4:4:4 up
        // to 32 x 32; 2 or 4 in raster order for a 4:4:4 block with a 64-sample side (rc_chroma_more codes those after
        // the first).  Record order: U's tx blocks, then V's.
        const int nTxX = ss ? 1 : max(1, 4 * bw / W), nTxY = ss ? 1 : max(1, 4 * bh / H);
        const int yt = ST(Max_Tx_Size_Rect)[bsize];
        const int lumaN = min(txw(yt), 32) * min(txh(yt), 32);
        int tIdx = 0;   // coded chroma tx blocks so far
        for (int pl = 1; pl <= 2; pl++) {
            Px *dst = (Px *)F.rec[pl] + (size_t)cy * F.rpitch[pl] + cx;
            int16_t *lv = Wp.qb[pl - 1];
            predict(pl, bestC, Wp.pred, lane, 32);
            __syncwarp();
            const EvalIn e{uvType, pl, skipCtx[pl], dcCtx[pl], 0, F.dcQ, F.acQ, T};
            grp_eval<BD, Px>(txSz, ResFn<Px>{sP[pl], W, Wp.pred, lw, nullptr}, e, Wp.buf, lv, lane, 32);
            rc_reconstruct<BD, Px>(txSz, uvType, lv, F.dcQ, F.acQ, Wp.pred, dst, F.rpitch[pl], Wp.buf);
            int e2 = rc_record(F, T, sb, pl, txSz, uvType, cx4, cy4, lv, txbBase + 1 + tIdx, coefBase + lumaN + tIdx * nq);
            tIdx++;
            if constexpr (SS == 0) {
                if (nTxX * nTxY > 1) {   // (4:4:4, a 64-sample side: rare, out of line)
                    const int sbW4 = tC1 - sbc * 16, sbH4 = tR1 - sbr * 16;
                    e2 |= rc_chroma_more<BD, Px>(F, Wp, T, sb, li, pl, txSz, uvType, bestC, bsize, cx, cy, csr, csc, nTxX, nTxY, availLC,
                                                 availUC, tC0, tR0, sbW4, sbH4, txbBase + 1, coefBase + lumaN, &tIdx);
                }
            }
            if (pl == 1) eobU = e2; else eobV = e2;
        }
        duv = cfl ? 0 : cand_delta(bestC);
        aU = cfl ? alpha[1] : 0;
        aV = cfl ? alpha[2] : 0;
    }
    if (lane == 0) {
        av1g_block b;
        b.mi_row = (uint16_t)mi_row; b.mi_col = (uint16_t)mi_col;
        b.bsize = (uint8_t)bsize;
        b.skip = (uint8_t)((eobY == 0 && eobU == 0 && eobV == 0) ? 1 : 0);
        b.tx_depth = 0;
        b.y_mode = (uint8_t)yMode;
        b.angle_delta_y = (int8_t)(bsize >= AV1G_BLOCK_8X8 && is_dir(yMode) ? yDelta : 0);
        b.uv_mode = (uint8_t)(hasC ? uv : 0);
        b.angle_delta_uv = (int8_t)(hasC && bsize >= AV1G_BLOCK_8X8 && is_dir(uv) ? duv : 0);
        b.cfl_alpha_u = (int8_t)aU; b.cfl_alpha_v = (int8_t)aV;
        b.filter_intra = 0; b.cdef_idx = 0; b.sb_qindex = 0;
        F.oBlocks[(size_t)sb * SB_MAX_LEAVES + li] = b;
        F.oBlockTxb[(size_t)sb * SB_MAX_LEAVES + li] = (uint16_t)txbBase;
    }
    __syncwarp();
    if (lane == 0) {
        st_release(F.leafDone + (size_t)sb * SB_MAX_LEAVES + li, 2);
        if (trace) trace[8] = gtimer();
        // serving session: the image's last leaf tells the host (its record can be packed while others run on)
        if (F.leafDoneCnt && atomicAdd(F.leafDoneCnt, 1) + 1 == (int)*F.leafTotal) {
            __threadfence_system();
            *F.doneFlag = F.img;
        }
    }
}

// Persistent grid of independent warps over a ready queue (one instance per bit depth BD and chroma subsampling SS):
// a warp takes the next slot, waits until a leaf has been written there (bounded in time), brings the descriptor of the
// leaf's image into its shared copy when the image changes, and runs the leaf.  Two modes:
//   batch    the nImg images of Fs (one format group of a batch): the loop ends once every leaf of them is taken;
//   serving  (ctl.serving) images keep arriving: each submitted image's front end writes its descriptor into the table
//            Fs and pushes its first ready leaves into the same queue while the loop runs.  A warp that finds no leaf in
//            its slot for readyWaitNs gives the slot up and leaves: the loop ends when it is idle, and the host launches it
//            again once an image's front end has queued leaves (the queue counters carry on).
struct RcCtl {
    int *rq;                       // [0] next slot to take, [1] next slot to write
    const unsigned long long *readyQ;      // (serving: idle workers write SLOT_ABANDONED into their slots)
    int *err;
    int serving;                   // a serving session's loop (else a batch's)
    uint32_t cap;                  // positions of readyQ
    unsigned long long readyWaitNs;
    unsigned long long *trace;     // optional leaf trace (batch mode)
    int poison;
    int warps;                     // warps per CTA that work (the rest leave after the CTA's staging); at most NW
};
template <int BD> using RcPxOf = typename std::conditional<BD == 8, uint8_t, uint16_t>::type;
template <int BD, int SS> constexpr int rc_warps_of() { return rc_warps<RcPxOf<BD>, SS>(); }
template <int BD, int SS>
__global__ void __launch_bounds__(rc_warps_of<BD, SS>() * 32, 1) k_recon(const FrameDesc *Fs, int nImg, const RcCtl ctl) {
    typedef RcPxOf<BD> Px;
    constexpr int NW = rc_warps_of<BD, SS>();
    typedef RcSmem<Px, SS, NW> Sm;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Sm &S = *reinterpret_cast<Sm *>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = lane_id();
    RcWarp<Px, SS> &Wp = S.ws[warp].w;
    FrameDesc &F = S.ws[warp].F;
    if (ctl.poison) {   // (the shared memory of the launch: the working warps' parts only)
        smem_poison(smem_raw, rc_smem_bytes<Px, SS>(ctl.warps), threadIdx.x, blockDim.x);
        __syncthreads();
    }
    {   // all four cost tables (q-context 0 in the RateStage), the scans and base-context offsets
        rate_tabs_stage(S.T, 0, threadIdx.x, blockDim.x);
        for (int q = 1; q < 4; q++) {
            const uint4 *c = reinterpret_cast<const uint4 *>(g_cost[q]);
            for (int i = threadIdx.x; i < NCDF / 8; i += blockDim.x) reinterpret_cast<uint4 *>(S.cost[q - 1])[i] = c[i];
        }
    }
    if (threadIdx.x == 0) S.big.lock = 0;
    __syncthreads();
    if (warp >= ctl.warps) return;   // (uniform per warp; no CTA barrier follows)
    int *rq = ctl.rq;
    const unsigned long long *readyQ = ctl.readyQ;
    int *err = ctl.err;
    const unsigned long long readyWait = ctl.readyWaitNs;
    unsigned long long *traceBase = ctl.trace;
    const bool serving = ctl.serving != 0;
    int total = 0x7FFFFFFF;
    if (!serving) {
        total = 0;
        for (int i = 0; i < nImg; i++) total += (int)*Fs[i].leafTotal;
    }
    int cur = -1;
    for (;;) {
        unsigned long long e = 0;
        int h = 0, bad = 0;
        if (lane == 0 && serving) {
            // serving: a ticket of its own (no two workers poll one word); a worker that finds no leaf in its slot for
            // readyWait - or sees the stop word - gives the slot up (a producer that comes later skips it) and leaves, so
            // the loop ends when idle (the host launches it again while images are in it; the counters carry on)
            h = atomicAdd(rq, 1);
            const unsigned long long t0 = gtimer();
            if ((uint32_t)h >= ctl.cap) {   // no position left: nothing more can come
                bad = 1;
            } else {
                for (;;) {
                    e = ld_relaxed64(readyQ + h);
                    if (e) break;
                    if (*(volatile int *)err || gtimer() - t0 > readyWait) {
                        e = atomicCAS(const_cast<unsigned long long *>(readyQ) + h, 0ull, SLOT_ABANDONED);
                        if (!e) bad = 1;   // given up; otherwise a leaf came just now: take it
                        break;
                    }
                    __nanosleep(128);
                }
            }
        } else if (lane == 0) {
            h = atomicAdd(rq, 1);
            if (h >= total) {
                bad = 1;
            } else {
                const unsigned long long t0 = gtimer();
                for (;;) {
                    e = ld_relaxed64(readyQ + h);
                    if (e || gtimer() - t0 > readyWait || *(volatile int *)err) break;
                    __nanosleep(128);
                }
                if (!e) {
                    atomicCAS(err, 0, KERR_WAIT_LEAF);
                    bad = 1;
                }
                if (traceBase) {
                    unsigned long long *tr = traceBase + (size_t)h * TRACE_STAMPS;
                    tr[0] = t0; tr[1] = gtimer(); tr[9] = e - 1;
                }
            }
        }
        if (__shfl_sync(0xffffffffu, bad, 0)) break;
        e = __shfl_sync(0xffffffffu, e, 0);
        h = __shfl_sync(0xffffffffu, h, 0);
        fence_acquire();   // the slot's entry was released by the warp that queued the leaf: its data and that of the
                           // leaves it waited on are visible from here on
        const unsigned long long v = e - 1;
        const int img = (int)(v >> 32);
        const uint32_t id = (uint32_t)v;
        if (img != cur) {   // the descriptor of the leaf's image into the warp's shared copy (tags differ per slot use);
                            // coherent loads: a serving session rewrites table slots while its loop runs
            const uint4 *src = reinterpret_cast<const uint4 *>(Fs + (img & 0xFFFF));
            for (int k = lane; k < (int)(sizeof(FrameDesc) / 16); k += 32) reinterpret_cast<uint4 *>(&F)[k] = __ldcg(src + k);
            __syncwarp();
            cur = img;
        }
        const RateTabs T{F.qctx == 0 ? S.T.cost : S.cost[F.qctx - 1], S.T.scan, S.T.baseCtx};
        unsigned long long *trace = traceBase ? traceBase + (size_t)h * TRACE_STAMPS : nullptr;
        rc_leaf<BD, Px, SS>(F, Wp, S.big, T, (int)(id >> 8), (int)(id & 255), trace);
    }
}

}  // namespace is
