// is_k_ent.cu - entropy coding of DecisionRecords on the device: a batch of records (each frame's arrays wherever they
// lie in device memory) in, the AV1 tile payloads out, byte for byte what av1core's CPU writer produces
// (av1core/src/encoder.cpp:415-1315 encode_partition / encode_block / code_txb / code_coeffs / encode_tile), plus the
// sequence and frame headers and the OBU framing on the host (encoder.cpp:1317-1441 write_headers, :1571-1600).
//
// Every context of the intra syntax is a function of the record alone (neighbouring blocks' sizes, modes and skip
// flags, neighbouring tx blocks' cumulative levels and DC signs), never of the adapted CDF values, so the symbols are
// made in parallel and only the range coder with its CDF adaptation runs in order, per tile:
//   k_ent_blocks  one thread per block: the 4x4 mode-info maps (size, luma mode, skip), each SB's first block, the
//                 owner block of each tx block
//   k_ent_txb     one thread per tx block: end of block, cumulative level and DC category (into per-plane 4x4 maps),
//                 the number of its coefficient symbols
//   k_ent_sb      one thread per SB: the partition walk over its blocks (partition symbols with their contexts) and
//                 each block's mode-info symbols, into a fixed slot of the block
//   scans         exclusive sums of the blocks' and tx blocks' symbol counts: where each block's and tx block's
//                 symbols start in the batch's stream, which is in bitstream order
//   k_ent_emit_*  the symbols into the stream (one thread per block / tx block)
//   k_ent_code    two warps per tile: the CDF state in shared memory; one warp adapts the CDFs and works out the
//                 symbols' interval bounds 32 at a time, one lane range-codes the bounds of the batch before, then
//                 resolves the carries
//   k_ent_pack    the tiles' payloads back to back, offsets in the result head
// A symbol is one 32-bit word: kind (adaptive / equiprobable bit / split-or-horizontal / split-or-vertical), alphabet
// size, value and the CDF's offset inside av1g_cdfs.
#include "is_units.cuh"
#include "is_api.h"
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>
#include "av1g/levels_gen.h"

namespace is {

static __constant__ uint8_t c_miWLog2[22], c_miHLog2[22];
static __device__ uint16_t g_cdfInit[4][NCDF];   // av1g_cdfs of each coefficient q-context at the start of a tile

constexpr uint32_t NONE32 = 0xFFFFFFFFu;
constexpr int HEAD_WORDS = 16;   // partition symbols (at most 4: 64, 32, 16, 8) + mode info (at most 10) of a block
enum { SYM_ADAPT = 0, SYM_BIT = 1, SYM_SPLIT_H = 2, SYM_SPLIT_V = 3 };

__device__ __forceinline__ uint32_t sym_word(int kind, int cdf, int s, int N) {
    return (uint32_t)kind | ((uint32_t)(N - 1) << 2) | ((uint32_t)s << 6) | ((uint32_t)cdf << 16);
}

struct EntFrameD {
    const av1g_block *blocks;
    const uint32_t *blockTxb;
    const av1g_txb *txb;
    const int16_t *coeffs;
    int MiCols, MiRows, ss, qctx;
    int cdefBits;                 // enable_cdef: the bits of a SB's cdef_idx; -1 without CDEF
    int sbCols, sbRows, tileWSb, tileHSb, tileCols, tileRows;
    uint32_t blockBase, nBlocks, txbBase, nTxb, sbBase, tileBase;
    uint64_t miBase, ctxBase[3];
    int ctxW[3], ctxH[3];
};

struct EntArgs {
    const EntFrameD *fr;
    int nF;
    const uint32_t *fBlock, *fTxb, *fSb, *fTile;   // [nF + 1] first global block / tx block / SB / tile of each frame
    uint32_t nB, nT, nSb, nTiles;
    uint8_t *miSize, *yMode, *skip, *cul, *dcc, *txbType;
    uint16_t *txbEob;
    uint32_t *sbFirst, *txbBlock, *txbCnt, *headCnt, *headW;
    uint32_t *syms;
    uint64_t cap;
    uint64_t *symBegin;                            // [nTiles + 1]
    uint16_t *pre;                                 // precarry entries, per tile at 2 * symBegin + 16 * tile
    uint8_t *tbytes;                               // the tiles' resolved bytes, same places
    uint32_t *tileBytes;
    is_ent_status *status;
    uint64_t *tileOff;                             // [nTiles + 1], right after the status
    uint8_t *out;
};

__device__ __forceinline__ int ent_find(const uint32_t *base, int n, uint32_t i) {   // last f with base[f] <= i
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (base[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ void ent_fail(const EntArgs &A, int bit) { atomicOr(&A.status->error, bit); }

// symbols of a level v of a non-skip tx block beyond the base symbol: coeff_br words, the sign, the Golomb bits
__device__ __forceinline__ uint32_t level_extra_syms(int v) {
    const int a = abs(v);
    if (!a) return 0;
    uint32_t n = 1;
    if (a > 2) n += min((min(a, 15) - 3) / 3 + 1, 4);
    if (a > 14) n += 2 * (31 - __clz(a - 14)) + 1;
    return n;
}
__device__ __forceinline__ int eob_pt_of(int eob) { return eob <= 2 ? eob : 2 + (31 - __clz(eob - 1)); }

// ---- per block: mode-info maps, SB starts, owners of the tx blocks ----
__global__ void k_ent_blocks(EntArgs A) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= A.nB) return;
    const EntFrameD &F = A.fr[ent_find(A.fBlock, A.nF, g)];
    const uint32_t b = g - F.blockBase;
    const av1g_block B = F.blocks[b];
    const int r = B.mi_row, c = B.mi_col, bs = B.bsize;
    if (bs >= 22 || (bs >= 13 && bs <= 15) || r >= F.MiRows || c >= F.MiCols) { ent_fail(A, IS_ENT_ERR_RECORD); return; }
    const int r1 = min(r + bh4(bs), F.MiRows), c1 = min(c + bw4(bs), F.MiCols);
    for (int y = r; y < r1; y++)
        for (int x = c; x < c1; x++) {
            const uint64_t m = F.miBase + (uint64_t)y * F.MiCols + x;
            A.miSize[m] = (uint8_t)bs;
            A.yMode[m] = B.y_mode;
            A.skip[m] = B.skip;
        }
    if (!(r & 15) && !(c & 15)) A.sbFirst[F.sbBase + (r >> 4) * F.sbCols + (c >> 4)] = g;
    const uint32_t t0 = F.blockTxb[b], t1 = F.blockTxb[b + 1];
    if (t0 > t1 || t1 > F.nTxb) { ent_fail(A, IS_ENT_ERR_RECORD); return; }
    for (uint32_t t = t0; t < t1; t++) A.txbBlock[F.txbBase + t] = g;
}

// ---- per tx block: eob, type, cumulative level and DC category, symbol count ----
__global__ void k_ent_txb(EntArgs A) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= A.nT) return;
    const uint32_t gb = A.txbBlock[g];
    A.txbCnt[g] = 0;
    if (gb == NONE32) { ent_fail(A, IS_ENT_ERR_RECORD); return; }
    const EntFrameD &F = A.fr[ent_find(A.fTxb, A.nF, g)];
    const av1g_txb X = F.txb[g - F.txbBase];
    const av1g_block B = F.blocks[gb - F.blockBase];
    const int plane = X.plane, txSz = X.tx_size;
    if (plane > 2 || txSz >= 19 || (plane == 0 && X.tx_type >= 16) || B.uv_mode > AV1G_UV_CFL_PRED) { ent_fail(A, IS_ENT_ERR_RECORD); return; }
    int eob = 0, type = AV1G_DCT_DCT, cul = 0, dc = 0;
    uint32_t cnt = 0;
    if (!B.skip) {
        type = plane == 0 ? X.tx_type : chroma_tx_type(txSz, B.uv_mode);
        const int n = min(txw(txSz), 32) * min(txh(txSz), 32);
        const int16_t *q = F.coeffs + X.coeff_off;
        const bool legal = plane > 0 || tx_in_set(tx_set_intra(txSz), type);
        const uint16_t *scan = get_scan(rate_tabs_global(0), txSz, legal ? type : AV1G_DCT_DCT);
        for (int c = n - 1; c >= 0; c--)
            if (q[scan[c]]) { eob = c + 1; break; }
        if (eob && !legal) { ent_fail(A, IS_ENT_ERR_RECORD); return; }
        if (!eob) type = AV1G_DCT_DCT;
        cnt = 1;
        if (eob) {
            const int pt = eob_pt_of(eob);
            cnt += 1 + (plane == 0 && tx_set_intra(txSz) > 0) + (pt >= 3 ? pt - 2 : 0) + eob;
            int sum = 0;
            for (int c = 0; c < eob; c++) {
                const int v = q[scan[c]];
                sum += abs(v);
                cnt += level_extra_syms(v);
            }
            cul = min(sum, 63);
            dc = q[0] < 0 ? 1 : q[0] > 0 ? 2 : 0;
        }
    }
    A.txbEob[g] = (uint16_t)eob;
    A.txbType[g] = (uint8_t)type;
    A.txbCnt[g] = cnt;
    const int W = F.ctxW[plane], H = F.ctxH[plane];
    const int x1 = min(X.x4 + (txw(txSz) >> 2), W), y1 = min(X.y4 + (txh(txSz) >> 2), H);
    for (int y = X.y4; y < y1; y++)
        for (int x = X.x4; x < x1; x++) {
            const uint64_t m = F.ctxBase[plane] + (uint64_t)y * W + x;
            A.cul[m] = (uint8_t)cul;
            A.dcc[m] = (uint8_t)dc;
        }
}

// ---- per SB: partition walk and mode info ----
struct Walk {
    const EntArgs *A;
    const EntFrameD *F;
    int rowStart, colStart;     // the tile's first row / column (mi)
    uint32_t cur, end;          // next block (global), end of the frame's blocks
    int k;                      // words in the current block's slot
    int cdef;                   // the SB's cdef_idx once coded (-1: not yet)
    bool bad;
};

__device__ __forceinline__ int mi_at(const uint8_t *map, const EntFrameD &F, int r, int c) {
    return map[F.miBase + (uint64_t)r * F.MiCols + c];
}
__device__ __forceinline__ void put_word(Walk &W, uint32_t w) {
    if (W.k < HEAD_WORDS) W.A->headW[(uint64_t)W.cur * HEAD_WORDS + W.k] = w;
    W.k++;
}
__device__ __forceinline__ bool blk_at(const Walk &W, uint32_t i, int r, int c, int bs) {
    if (i >= W.end) return false;
    const av1g_block &B = W.F->blocks[i - W.F->blockBase];
    return B.mi_row == r && B.mi_col == c && B.bsize == bs;
}

// mode info of the block at (r, c) of size bs (spec 5.11.5 intra_frame_mode_info, as av1core codes it:
// encoder.cpp:491-600 with the toolset of these records)
__device__ void walk_block(Walk &W, int r, int c, int bs) {
    const EntFrameD &F = *W.F;
    const EntArgs &A = *W.A;
    if (!blk_at(W, W.cur, r, c, bs)) { W.bad = true; return; }
    const av1g_block B = F.blocks[W.cur - F.blockBase];
    const bool aU = r - 1 >= W.rowStart, aL = c - 1 >= W.colStart;
    const bool dirOk = bs >= AV1G_BLOCK_8X8;
    const bool hasC = has_chroma(bs, r, c, F.ss);
    const bool cflOk = bw4(bs) <= 8 && bh4(bs) <= 8;
    // fields these records may carry
    if (B.skip > 1 || B.tx_depth || B.filter_intra || B.y_mode > AV1G_PAETH_PRED ||
        (B.angle_delta_y && !(dirOk && is_dir(B.y_mode))) || B.angle_delta_y < -3 || B.angle_delta_y > 3 ||
        (hasC && (B.uv_mode > AV1G_UV_CFL_PRED || (B.uv_mode == AV1G_UV_CFL_PRED && !cflOk) ||
                  (B.angle_delta_uv && !(dirOk && is_dir(B.uv_mode))) || B.angle_delta_uv < -3 || B.angle_delta_uv > 3 ||
                  (B.uv_mode == AV1G_UV_CFL_PRED && ((!B.cfl_alpha_u && !B.cfl_alpha_v) || B.cfl_alpha_u < -16 ||
                                                     B.cfl_alpha_u > 16 || B.cfl_alpha_v < -16 || B.cfl_alpha_v > 16))))) {
        W.bad = true;
        return;
    }
    const int sctx = (aU ? mi_at(A.skip, F, r - 1, c) : 0) + (aL ? mi_at(A.skip, F, r, c - 1) : 0);
    put_word(W, sym_word(SYM_ADAPT, IS_CB(skip) + sctx * IS_CD(skip, 1), B.skip, 2));
    if (F.cdefBits >= 0 && !B.skip) {   // read_cdef: the SB's cdef_idx with its first coded block, a literal
        if (B.cdef_idx < 0 || B.cdef_idx >= (1 << F.cdefBits) || (W.cdef >= 0 && B.cdef_idx != W.cdef)) { W.bad = true; return; }
        if (W.cdef < 0) {
            for (int i = F.cdefBits - 1; i >= 0; i--) put_word(W, sym_word(SYM_BIT, 0, (B.cdef_idx >> i) & 1, 2));
            W.cdef = B.cdef_idx;
        }
    }
    const int am = ST(Intra_Mode_Context)[aU ? mi_at(A.yMode, F, r - 1, c) : AV1G_DC_PRED];
    const int lm = ST(Intra_Mode_Context)[aL ? mi_at(A.yMode, F, r, c - 1) : AV1G_DC_PRED];
    put_word(W, sym_word(SYM_ADAPT, ci_y_mode(am, lm), B.y_mode, 13));
    if (dirOk && is_dir(B.y_mode)) put_word(W, sym_word(SYM_ADAPT, ci_angle(B.y_mode - AV1G_V_PRED), B.angle_delta_y + 3, 7));
    if (hasC) {
        put_word(W, cflOk ? sym_word(SYM_ADAPT, ci_uv_cfl(B.y_mode), B.uv_mode, 14)
                          : sym_word(SYM_ADAPT, ci_uv_nocfl(B.y_mode), B.uv_mode, 13));
        if (B.uv_mode == AV1G_UV_CFL_PRED) {
            // joint sign: 0 zero, 1 negative, 2 positive per plane; the pair (0, 0) does not occur
            const int sU = B.cfl_alpha_u == 0 ? 0 : B.cfl_alpha_u < 0 ? 1 : 2;
            const int sV = B.cfl_alpha_v == 0 ? 0 : B.cfl_alpha_v < 0 ? 1 : 2;
            put_word(W, sym_word(SYM_ADAPT, ci_cfl_sign(), sU * 3 + sV - 1, 8));
            if (sU) put_word(W, sym_word(SYM_ADAPT, ci_cfl_alpha((sU - 1) * 3 + sV), abs(B.cfl_alpha_u) - 1, 16));
            if (sV) put_word(W, sym_word(SYM_ADAPT, ci_cfl_alpha((sV - 1) * 3 + sU), abs(B.cfl_alpha_v) - 1, 16));
        }
        if (dirOk && is_dir(B.uv_mode)) put_word(W, sym_word(SYM_ADAPT, ci_angle(B.uv_mode - AV1G_V_PRED), B.angle_delta_uv + 3, 7));
    }
    if (W.k > HEAD_WORDS) { W.bad = true; return; }
    A.headCnt[W.cur] = (uint32_t)W.k;
    W.cur++;
    W.k = 0;
}

// the partition node at (r, c) of size bs (spec 5.11.4 decode_partition); the partition type is the one the block
// sequence implies (the record stores no tree: av1core/include/av1g/decisions.h "Block order", encoder.cpp:375-413)
__device__ void walk_node(Walk &W, int r, int c, int bs) {
    const EntFrameD &F = *W.F;
    if (W.bad || r >= F.MiRows || c >= F.MiCols) return;
    const int half = bw4(bs) >> 1, quarter = half >> 1;
    const bool hasRows = r + half < F.MiRows, hasCols = c + half < F.MiCols;
    int p = AV1G_PARTITION_NONE;
    if (bs >= AV1G_BLOCK_8X8) {
        if (W.cur >= W.end) { W.bad = true; return; }
        const av1g_block &B = F.blocks[W.cur - F.blockBase];
        if (B.mi_row != r || B.mi_col != c) { W.bad = true; return; }
        const int hz = ST(Partition_Subsize)[AV1G_PARTITION_HORZ][bs], vt = ST(Partition_Subsize)[AV1G_PARTITION_VERT][bs];
        const int sp = ST(Partition_Subsize)[AV1G_PARTITION_SPLIT][bs];
        const int h4 = ST(Partition_Subsize)[AV1G_PARTITION_HORZ_4][bs], v4 = ST(Partition_Subsize)[AV1G_PARTITION_VERT_4][bs];
        const bool big = bs > AV1G_BLOCK_8X8, both = hasRows && hasCols;
        const int s = B.bsize;
        if (s == bs) p = AV1G_PARTITION_NONE;
        else if (s == hz) p = blk_at(W, W.cur + 1, r + half, c, sp) ? AV1G_PARTITION_HORZ_B : AV1G_PARTITION_HORZ;
        else if (s == vt) p = blk_at(W, W.cur + 1, r, c + half, sp) ? AV1G_PARTITION_VERT_B : AV1G_PARTITION_VERT;
        else if (s == sp && big && both && blk_at(W, W.cur + 1, r + half, c, sp)) p = AV1G_PARTITION_VERT_A;
        else if (s == sp && big && both && blk_at(W, W.cur + 1, r, c + half, sp) && blk_at(W, W.cur + 2, r + half, c, hz))
            p = AV1G_PARTITION_HORZ_A;
        else if (big && s == h4) p = AV1G_PARTITION_HORZ_4;
        else if (big && s == v4) p = AV1G_PARTITION_VERT_4;
        else p = AV1G_PARTITION_SPLIT;
        const bool ok = (bs == AV1G_BLOCK_8X8 && p > AV1G_PARTITION_SPLIT) ? false
                      : both ? true
                      : hasCols ? (p == AV1G_PARTITION_HORZ || p == AV1G_PARTITION_SPLIT)
                      : hasRows ? (p == AV1G_PARTITION_VERT || p == AV1G_PARTITION_SPLIT)
                      : p == AV1G_PARTITION_SPLIT;
        if (!ok) { W.bad = true; return; }
        // context: neighbours narrower (above) / shorter (left) than this node
        const int bsl = c_miWLog2[bs];
        const int above = (r - 1 >= W.rowStart) && c_miWLog2[mi_at(W.A->miSize, F, r - 1, c)] < bsl;
        const int left = (c - 1 >= W.colStart) && c_miHLog2[mi_at(W.A->miSize, F, r, c - 1)] < bsl;
        const int ctx = left * 2 + above;
        const int cdf = bsl == 1 ? IS_CB(partition_w8) + ctx * IS_CD(partition_w8, 1)
                      : bsl == 2 ? IS_CB(partition_w16) + ctx * IS_CD(partition_w16, 1)
                      : bsl == 3 ? IS_CB(partition_w32) + ctx * IS_CD(partition_w32, 1)
                                 : IS_CB(partition_w64) + ctx * IS_CD(partition_w64, 1);
        if (both) put_word(W, sym_word(SYM_ADAPT, cdf, p, bsl == 1 ? 4 : 10));
        else if (hasCols) put_word(W, sym_word(SYM_SPLIT_H, cdf, p == AV1G_PARTITION_SPLIT, 2));
        else if (hasRows) put_word(W, sym_word(SYM_SPLIT_V, cdf, p == AV1G_PARTITION_SPLIT, 2));
    }
    const int sub = ST(Partition_Subsize)[p][bs], sp = ST(Partition_Subsize)[AV1G_PARTITION_SPLIT][bs];
    switch (p) {
    case AV1G_PARTITION_NONE: walk_block(W, r, c, sub); break;
    case AV1G_PARTITION_HORZ:
        walk_block(W, r, c, sub);
        if (hasRows && !W.bad) walk_block(W, r + half, c, sub);
        break;
    case AV1G_PARTITION_VERT:
        walk_block(W, r, c, sub);
        if (hasCols && !W.bad) walk_block(W, r, c + half, sub);
        break;
    case AV1G_PARTITION_SPLIT:
        walk_node(W, r, c, sub);
        walk_node(W, r, c + half, sub);
        walk_node(W, r + half, c, sub);
        walk_node(W, r + half, c + half, sub);
        break;
    case AV1G_PARTITION_HORZ_A:
        walk_block(W, r, c, sp);
        if (!W.bad) walk_block(W, r, c + half, sp);
        if (!W.bad) walk_block(W, r + half, c, sub);
        break;
    case AV1G_PARTITION_HORZ_B:
        walk_block(W, r, c, sub);
        if (!W.bad) walk_block(W, r + half, c, sp);
        if (!W.bad) walk_block(W, r + half, c + half, sp);
        break;
    case AV1G_PARTITION_VERT_A:
        walk_block(W, r, c, sp);
        if (!W.bad) walk_block(W, r + half, c, sp);
        if (!W.bad) walk_block(W, r, c + half, sub);
        break;
    case AV1G_PARTITION_VERT_B:
        walk_block(W, r, c, sub);
        if (!W.bad) walk_block(W, r, c + half, sp);
        if (!W.bad) walk_block(W, r + half, c + half, sp);
        break;
    case AV1G_PARTITION_HORZ_4:
        for (int i = 0; i < 4 && !W.bad; i++)
            if (i < 3 || r + quarter * 3 < F.MiRows) walk_block(W, r + quarter * i, c, sub);
        break;
    default:   // VERT_4
        for (int i = 0; i < 4 && !W.bad; i++)
            if (i < 3 || c + quarter * 3 < F.MiCols) walk_block(W, r, c + quarter * i, sub);
        break;
    }
}

__global__ void k_ent_sb(EntArgs A) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= A.nSb) return;
    const EntFrameD &F = A.fr[ent_find(A.fSb, A.nF, g)];
    const int s = (int)(g - F.sbBase), sr = s / F.sbCols, sc = s - sr * F.sbCols;
    Walk W;
    W.A = &A;
    W.F = &F;
    W.rowStart = (sr / F.tileHSb) * F.tileHSb * 16;
    W.colStart = (sc / F.tileWSb) * F.tileWSb * 16;
    W.cur = A.sbFirst[g];
    W.end = F.blockBase + F.nBlocks;
    W.k = 0;
    W.cdef = -1;
    W.bad = W.cur == NONE32;
    if (!W.bad) walk_node(W, sr * 16, sc * 16, AV1G_BLOCK_64X64);
    // the walk must end where the next SB of the decode order starts
    if (!W.bad) {
        const int tc = sc / F.tileWSb, tr = sr / F.tileHSb;
        const int c1 = min(F.sbCols, (tc + 1) * F.tileWSb), r1 = min(F.sbRows, (tr + 1) * F.tileHSb);
        int nr = sr, nc = sc + 1;
        if (nc >= c1) { nc = tc * F.tileWSb; nr++; }
        uint32_t want;
        if (nr < r1) want = A.sbFirst[F.sbBase + nr * F.sbCols + nc];
        else {   // the first SB of the next tile in raster order, or the frame's end
            int ntc = tc + 1, ntr = tr;
            if (ntc >= F.tileCols) { ntc = 0; ntr++; }
            want = ntr < F.tileRows ? A.sbFirst[F.sbBase + ntr * F.tileHSb * F.sbCols + ntc * F.tileWSb] : W.end;
        }
        if (W.cur != want) W.bad = true;
    }
    if (W.bad) ent_fail(A, IS_ENT_ERR_RECORD);
}

// ---- exclusive sums (in place; a[n] gets the total) ----
constexpr int SCAN_T = 1024;
__device__ __forceinline__ uint32_t cta_exclusive(uint32_t v, uint32_t *sh, uint32_t *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = sh[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    const uint32_t before = (w ? sh[w - 1] : 0) + x - v;
    *total = sh[31];
    return before;
}
__global__ void __launch_bounds__(SCAN_T) k_scan_local(uint32_t *a, uint32_t n, uint32_t *part) {
    __shared__ uint32_t sh[32];
    const uint32_t i = blockIdx.x * SCAN_T + threadIdx.x;
    const uint32_t v = i < n ? a[i] : 0;
    uint32_t tot;
    const uint32_t e = cta_exclusive(v, sh, &tot);
    if (i < n) a[i] = e;
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}
__global__ void __launch_bounds__(SCAN_T) k_scan_parts(uint32_t *part, uint32_t np) {
    __shared__ uint32_t sh[32];
    uint32_t carry = 0;
    for (uint32_t b = 0; b < np; b += SCAN_T) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t v = i < np ? part[i] : 0;
        uint32_t tot;
        const uint32_t e = cta_exclusive(v, sh, &tot);
        if (i < np) part[i] = e + carry;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) part[np] = carry;
}
__global__ void k_scan_add(uint32_t *a, uint32_t n, const uint32_t *part, uint32_t np) {
    const uint32_t i = blockIdx.x * SCAN_T + threadIdx.x;
    if (i < n) a[i] += part[blockIdx.x];
    if (i == 0) a[n] = part[np];
}

// ---- where each tile's symbols begin; capacity check ----
__device__ __forceinline__ uint64_t head_pos(const EntArgs &A, uint32_t gb) {
    const EntFrameD &F = A.fr[ent_find(A.fBlock, A.nF, gb)];
    return (uint64_t)A.headCnt[gb] + A.txbCnt[F.txbBase + F.blockTxb[gb - F.blockBase]];
}
__global__ void k_ent_tiles(EntArgs A) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g == 0) {
        const uint64_t total = (uint64_t)A.headCnt[A.nB] + A.txbCnt[A.nT];
        A.symBegin[A.nTiles] = total;
        A.status->symbols = total;
        A.status->capacity = A.cap;
        if (total > A.cap) ent_fail(A, IS_ENT_ERR_SYMBOLS);
    }
    if (g >= A.nTiles) return;
    if (A.status->error & IS_ENT_ERR_RECORD) { A.symBegin[g] = 0; return; }   // a bad record's offsets are not trusted
    const EntFrameD &F = A.fr[ent_find(A.fTile, A.nF, g)];
    const int t = (int)(g - F.tileBase), tr = t / F.tileCols, tc = t - tr * F.tileCols;
    const uint32_t gb = A.sbFirst[F.sbBase + tr * F.tileHSb * F.sbCols + tc * F.tileWSb];
    A.symBegin[g] = gb == NONE32 ? 0 : head_pos(A, gb);
}

// ---- symbols into the stream ----
__global__ void k_ent_emit_head(EntArgs A) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= A.nB || A.status->error) return;
    const uint64_t o = head_pos(A, g);
    const uint32_t n = A.headCnt[g + 1] - A.headCnt[g];
    for (uint32_t k = 0; k < n; k++) A.syms[o + k] = A.headW[(uint64_t)g * HEAD_WORDS + k];
}

struct SymOut {
    uint32_t *p;
    uint32_t n, cap;
    __device__ __forceinline__ void put(uint32_t w) { if (n < cap) p[n] = w; n++; }
};

// the coefficient syntax of one tx block (spec 5.11.39 coeffs, as av1core codes it: encoder.cpp:1073-1288)
__global__ void k_ent_emit_txb(EntArgs A) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= A.nT || A.status->error) return;
    const uint32_t cnt = A.txbCnt[g + 1] - A.txbCnt[g];
    if (!cnt) return;
    const uint32_t gb = A.txbBlock[g];
    const EntFrameD &F = A.fr[ent_find(A.fTxb, A.nF, g)];
    const av1g_txb X = F.txb[g - F.txbBase];
    const av1g_block B = F.blocks[gb - F.blockBase];
    const int plane = X.plane, txSz = X.tx_size, ptype = plane > 0, ssp = plane ? F.ss : 0;
    const int eob = A.txbEob[g], type = A.txbType[g];
    const int x4 = X.x4, y4 = X.y4, w4 = txw(txSz) >> 2, h4 = txh(txSz) >> 2;
    const int W = F.ctxW[plane], H = F.ctxH[plane];
    const uint8_t *cul = A.cul + F.ctxBase[plane], *dcc = A.dcc + F.ctxBase[plane];
    // the tile's first row / column in this plane's 4x4 units: neighbours before them were reset
    const int tr0 = (((int)(B.mi_row >> 4) / F.tileHSb) * F.tileHSb * 16) >> ssp;
    const int tc0 = (((int)(B.mi_col >> 4) / F.tileWSb) * F.tileWSb * 16) >> ssp;
    const bool hasA = y4 - 1 >= tr0, hasL = x4 - 1 >= tc0;
    SymOut S{A.syms + (uint64_t)(A.headCnt[gb + 1]) + A.txbCnt[g], 0, cnt};
    const int txSzCtx = (ST(Tx_Size_Sqr)[txSz] + ST(Tx_Size_Sqr_Up)[txSz] + 1) >> 1;
    // all_zero
    int ctx;
    {
        const int bsz = plane ? uv_bsize(B.bsize, F.ss) : B.bsize;
        const int bw = 4 * bw4(bsz), bh = 4 * bh4(bsz), w = txw(txSz), h = txh(txSz);
        if (plane == 0) {
            int top = 0, left = 0;
            if (hasA) for (int k = 0; k < w4 && x4 + k < W; k++) top = max(top, (int)cul[(uint64_t)(y4 - 1) * W + x4 + k]);
            if (hasL) for (int k = 0; k < h4 && y4 + k < H; k++) left = max(left, (int)cul[(uint64_t)(y4 + k) * W + x4 - 1]);
            const int mx = max(top, left), mn = min(top, left);
            ctx = (bw == w && bh == h) ? 0 : (top == 0 && left == 0) ? 1 : (top == 0 || left == 0) ? 2 + (mx > 3)
                : mx <= 3 ? 4 : mn <= 3 ? 5 : 6;
        } else {
            int above = 0, left = 0;
            if (hasA) for (int k = 0; k < w4 && x4 + k < W; k++) above |= cul[(uint64_t)(y4 - 1) * W + x4 + k] | dcc[(uint64_t)(y4 - 1) * W + x4 + k];
            if (hasL) for (int k = 0; k < h4 && y4 + k < H; k++) left |= cul[(uint64_t)(y4 + k) * W + x4 - 1] | dcc[(uint64_t)(y4 + k) * W + x4 - 1];
            ctx = (above != 0) + (left != 0) + 7 + (bw * bh > w * h ? 3 : 0);
        }
    }
    S.put(sym_word(SYM_ADAPT, ci_txb_skip(txSzCtx, ctx), eob == 0, 2));
    if (eob) {
        if (plane == 0) {
            const int set = tx_set_intra(txSz);
            if (set > 0) {
                const int sqr = ST(Tx_Size_Sqr)[txSz], idx = tx_index_in_set(set, type);
                S.put(set == AV1G_TX_SET_INTRA_1 ? sym_word(SYM_ADAPT, ci_set1(sqr, B.y_mode), idx, 7)
                                                 : sym_word(SYM_ADAPT, ci_set2(sqr, B.y_mode), idx, 5));
            }
        }
        const int cls = tx_class(type);
        const int ms = min((int)ST(Tx_Width_Log2)[txSz], 5) + min((int)ST(Tx_Height_Log2)[txSz], 5) - 4;
        const int pt = eob_pt_of(eob);
        S.put(sym_word(SYM_ADAPT, ci_eob_pt(ms, ptype, cls == AV1G_TX_CLASS_2D ? 0 : 1), pt - 1, ms + 5));
        if (pt >= 3) {
            const int rem = eob - ((1 << (pt - 2)) + 1);
            S.put(sym_word(SYM_ADAPT, ci_eob_extra(txSzCtx, ptype, pt - 3), (rem >> (pt - 3)) & 1, 2));
            for (int sh = pt - 4; sh >= 0; sh--) S.put(sym_word(SYM_BIT, 0, (rem >> sh) & 1, 2));
        }
        const int16_t *q = F.coeffs + X.coeff_off;
        const uint16_t *scan = get_scan(rate_tabs_global(0), txSz, type);
        const int adj = ST(Adjusted_Tx_Size)[txSz];
        const int bwl = ST(Tx_Width_Log2)[adj], width = 1 << bwl, height = ST(Tx_Height)[adj];
        const int area = height << bwl;
        // base levels and ranges in reverse scan order; a level's context neighbours come later in the scan, so they
        // are already coded: their levels are the coefficients' (capped)
        for (int c = eob - 1; c >= 0; c--) {
            const int pos = scan[c];
            const int level = min(abs((int)q[pos]), 15);
            const int row = pos >> bwl, col = pos - (row << bwl);
            if (c == eob - 1) {
                const int bctx = c == 0 ? 0 : c <= area / 8 ? 1 : c <= area / 4 ? 2 : 3;
                S.put(sym_word(SYM_ADAPT, ci_base_eob(txSzCtx, ptype, bctx), min(level, 3) - 1, 3));
            } else {
                int mag = 0;
                for (int k = 0; k < 5; k++) {
                    const int rr = row + ST(Sig_Ref_Diff_Offset)[cls][k][0], cc = col + ST(Sig_Ref_Diff_Offset)[cls][k][1];
                    if (rr < height && cc < width) mag += min(abs((int)q[(rr << bwl) + cc]), 3);
                }
                int bctx = min((mag + 1) >> 1, 4);
                if (cls == AV1G_TX_CLASS_2D) bctx = (row == 0 && col == 0) ? 0 : bctx + g_baseCtx[txSz * 25 + min(row, 4) * 5 + min(col, 4)];
                else bctx += ST(Coeff_Base_Pos_Ctx_Offset)[min(cls == AV1G_TX_CLASS_VERT ? row : col, 2)];
                S.put(sym_word(SYM_ADAPT, ci_base(txSzCtx, ptype, bctx), min(level, 3), 4));
            }
            if (level > 2) {
                int mag = 0;
                for (int k = 0; k < 3; k++) {
                    const int rr = row + ST(Mag_Ref_Offset_With_Tx_Class)[cls][k][0], cc = col + ST(Mag_Ref_Offset_With_Tx_Class)[cls][k][1];
                    if (rr < height && cc < width) mag += min(abs((int)q[rr * width + cc]), 15);
                }
                mag = min((mag + 1) >> 1, 6);
                const int brctx = pos == 0 ? mag
                                : cls == AV1G_TX_CLASS_2D ? ((row < 2 && col < 2) ? mag + 7 : mag + 14)
                                : cls == AV1G_TX_CLASS_HORIZ ? (col == 0 ? mag + 7 : mag + 14) : (row == 0 ? mag + 7 : mag + 14);
                const int cid = ci_br(min(txSzCtx, (int)AV1G_TX_32X32), ptype, brctx);
                int rem = level - 3;
                for (int i = 0; i < 4; i++) {
                    const int k = min(rem, 3);
                    S.put(sym_word(SYM_ADAPT, cid, k, 4));
                    rem -= k;
                    if (k < 3) break;
                }
            }
        }
        // signs and Golomb remainders in scan order
        for (int c = 0; c < eob; c++) {
            const int v = q[scan[c]];
            if (!v) continue;
            if (c == 0) {
                int d = 0;
                if (hasA) for (int k = 0; k < w4 && x4 + k < W; k++) { const int z = dcc[(uint64_t)(y4 - 1) * W + x4 + k]; d += z == 2 ? 1 : z == 1 ? -1 : 0; }
                if (hasL) for (int k = 0; k < h4 && y4 + k < H; k++) { const int z = dcc[(uint64_t)(y4 + k) * W + x4 - 1]; d += z == 2 ? 1 : z == 1 ? -1 : 0; }
                S.put(sym_word(SYM_ADAPT, ci_dc_sign(ptype, d < 0 ? 1 : d > 0 ? 2 : 0), v < 0, 2));
            } else {
                S.put(sym_word(SYM_BIT, 0, v < 0, 2));
            }
            const int a = abs(v);
            if (a > 14) {   // Exp-Golomb of a - 14: len zero bits, a one, then the len low bits of x
                const uint32_t x = (uint32_t)(a - 14);
                const int len = 31 - __clz(x);
                for (int i = 0; i < len; i++) S.put(sym_word(SYM_BIT, 0, 0, 2));
                S.put(sym_word(SYM_BIT, 0, 1, 2));
                for (int i = len - 1; i >= 0; i--) S.put(sym_word(SYM_BIT, 0, (x >> i) & 1, 2));
            }
        }
    }
    if (S.n != cnt) ent_fail(A, IS_ENT_ERR_RECORD);
}

// ---- the range coder: AV1's multi-symbol arithmetic coder (spec 8.2.6 read_symbol, from the encoder's side; the
// interval split (15-bit probabilities, 4 per symbol reserved), renormalisation and flush follow libaom's
// od_ec_encode_q15 / od_ec_enc_done, which the decoder's arithmetic fixes to the bit).  Output goes to a precarry buffer of 16-bit entries (a byte plus a possible carry);
// the carries are resolved backwards when the tile is done. ----
struct RangeEnc {
    uint32_t low, rng;
    int cnt;           // bits of low waiting below the next output byte, minus 16 (starts at -9)
    uint32_t n, cap;
    uint16_t *pre;
    bool over;
    __device__ void init(uint16_t *p, uint32_t c) { low = 0; rng = 0x8000; cnt = -9; n = 0; cap = c; pre = p; over = false; }
    __device__ __forceinline__ void out(uint32_t v) {
        if (n < cap) pre[n] = (uint16_t)v; else over = true;
        n++;
    }
    // one symbol from its packed step (pack_step): the interval split of the symbol, then renormalisation of the range
    // to 16 bits, where every 8 bits of low that pass the window go out.  The arithmetic chain through the range is
    // kept short: the probability terms come precomputed.
    __device__ __forceinline__ void step(uint32_t e) {
        const uint32_t r = rng, r8 = r >> 8;
        const uint32_t ev = (e >> 20) & 63u;
        const uint32_t v = ((r8 * ((e >> 10) & 0x3FFu)) >> 1) + ev;
        const uint32_t u = (e >> 26) ? r : ((r8 * (e & 0x3FFu)) >> 1) + ev + 4u;
        uint32_t l = low + (r - u);
        const uint32_t rn = u - v;
        const int d = __clz(rn) - 16;
        int s = cnt + d;
        if (s >= 0) {
            int c = cnt + 16;
            const int bytes = s >= 8 ? 2 : 1;
            for (int i = 0; i < bytes; i++) {
                out(l >> c);
                l &= (1u << c) - 1;
                c -= 8;
            }
            s = c + d - 16;
        }
        low = l << d;
        rng = rn << d;
        cnt = s;
    }
    // flush: the shortest tail that keeps the final interval decodable, then the carries; returns the byte count
    __device__ uint32_t finish(uint8_t *bytes) {
        uint32_t e = ((low + 0x3FFFu) & ~0x3FFFu) | 0x4000u;
        int c = cnt, s = c + 10;
        if (s > 0) {
            uint32_t m = (1u << (c + 16)) - 1;
            do {
                out(e >> (c + 16));
                e &= m;
                s -= 8;
                c -= 8;
                m >>= 8;
            } while (s > 0);
        }
        if (over) return 0;
        uint32_t carry = 0;
        for (uint32_t i = n; i-- > 0;) {
            carry += pre[i];
            bytes[i] = (uint8_t)carry;
            carry >>= 8;
        }
        return n;
    }
};
// the coder's inputs of symbol s of an alphabet of nm1 + 1 symbols with bounds fl / fh (32768 x the probability of the
// symbols after s - 1 / after s): fl >> 6, fh >> 6, 4 (nm1 - s), and whether fl is the whole range
__device__ __forceinline__ uint32_t pack_step(uint32_t fl, uint32_t fh, int s, int nm1) {
    return (fl >> 6) | ((fh >> 6) << 10) | ((uint32_t)(4 * (nm1 - s)) << 20) | ((fl >= 32768u ? 1u : 0u) << 26);
}

// CDF adaptation (spec 8.2.6 symbol decoding process, disable_cdf_update 0): spec-format CDF (cumulative, last
// entry 32768) followed by its counter
__device__ __forceinline__ void adapt(uint16_t *cdf, int s, int N) {
    const int count = cdf[N];
    const int rate = 3 + (count > 15) + (count > 31) + (N > 3 ? 2 : 1);
    for (int i = 0; i < N - 1; i++) {
        const int v = cdf[i];
        cdf[i] = (uint16_t)(i < s ? v - (v >> rate) : v + ((32768 - v) >> rate));
    }
    cdf[N] = (uint16_t)(count + (count < 32));
}

// the probability mass of the partitions that split the bottom half (split_or_horz) or the right half
// (split_or_vert) of a node at the frame edge (spec 9.3.1, split_or_horz / split_or_vert cdf)
__device__ __forceinline__ uint32_t split_mass(const uint16_t *pc, bool vert) {
    auto P = [&](int x) { return (uint32_t)pc[x] - (x ? (uint32_t)pc[x - 1] : 0u); };
    return vert ? P(AV1G_PARTITION_HORZ) + P(AV1G_PARTITION_SPLIT) + P(AV1G_PARTITION_HORZ_A) + P(AV1G_PARTITION_HORZ_B) +
                      P(AV1G_PARTITION_VERT_A) + P(AV1G_PARTITION_HORZ_4)
                : P(AV1G_PARTITION_VERT) + P(AV1G_PARTITION_SPLIT) + P(AV1G_PARTITION_HORZ_A) + P(AV1G_PARTITION_VERT_A) +
                      P(AV1G_PARTITION_VERT_B) + P(AV1G_PARTITION_VERT_4);
}

// Two warps per tile.  Warp 0 turns the symbols into coder inputs 32 at a time: a symbol's interval bounds (fl, fh)
// depend on its CDF as the earlier symbols left it, so the symbols of a window that share a CDF form a group (lanes
// with equal CDF offsets) whose lowest lane walks them in order, adapting the CDF - in registers for alphabets of up
// to 4 symbols (the coefficient CDFs, which carry long runs), in shared memory otherwise; groups and the equiprobable
// bits proceed side by side; each symbol leaves its coder step (pack_step).  Lane 0 of warp 1 runs only the range
// coder's arithmetic over the previous batch of steps, so the two overlap batch by batch.
constexpr int CODE_BATCH = 1024;   // symbols per batch (a multiple of 32)

// the coder step of symbol s of a CDF of up to 4 symbols held as c0..c2 (the last entry is 32768), then its adaptation
__device__ __forceinline__ uint32_t bounds_small(uint32_t c[3], uint32_t &count, int s, int N) {
    const uint32_t cs = s == 0 ? c[0] : s == 1 ? (N > 2 ? c[1] : 32768u) : s == 2 ? (N > 3 ? c[2] : 32768u) : 32768u;
    const uint32_t cp = s == 1 ? c[0] : s == 2 ? c[1] : c[2];
    const uint32_t fl = s ? 32768u - cp : 32768u, fh = 32768u - cs;
    const int rate = 3 + (count > 15) + (count > 31) + (N > 3 ? 2 : 1);
#pragma unroll
    for (int i = 0; i < 3; i++)
        if (i < N - 1) c[i] = i < s ? c[i] - (c[i] >> rate) : c[i] + ((32768u - c[i]) >> rate);
    count += count < 32;
    return pack_step(fl, fh, s, N - 1);
}

__global__ void __launch_bounds__(64) k_ent_code(EntArgs A) {
    __shared__ __align__(16) uint16_t cdf[NCDF];
    __shared__ uint32_t bnd[2][CODE_BATCH];   // the coder steps (pack_step)
    __shared__ uint32_t words[CODE_BATCH];    // warp 0's batch of symbol words
    const uint32_t g = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (A.status->error) return;
    const EntFrameD &F = A.fr[ent_find(A.fTile, A.nF, g)];
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(g_cdfInit[F.qctx]);
        for (int i = threadIdx.x; i < NCDF / 8; i += 64) reinterpret_cast<uint4 *>(cdf)[i] = src[i];
    }
    const uint64_t s0 = A.symBegin[g], s1 = A.symBegin[g + 1];
    const uint64_t base = 2 * s0 + 16 * (uint64_t)g;
    const uint32_t nb = (uint32_t)((s1 - s0 + CODE_BATCH - 1) / CODE_BATCH);
    RangeEnc E;
    E.init(A.pre + base, (uint32_t)(2 * (s1 - s0) + 16));
    __syncthreads();
    for (uint32_t b = 0; b <= nb; b++) {
        if (warp == 0 && b < nb) {
            const uint64_t at = s0 + (uint64_t)b * CODE_BATCH;
            const int n = (int)min((uint64_t)CODE_BATCH, s1 - at);
            uint32_t *pb = bnd[b & 1];
#pragma unroll 8
            for (int j = lane; j < n; j += 32) words[j] = A.syms[at + j];   // the batch's loads in flight together
            __syncwarp();
            for (int j = 0; j < n; j += 32) {
                const bool live = j + lane < n;
                const uint32_t w = live ? words[j + lane] : (uint32_t)SYM_BIT;
                const int kind = w & 3, nm1 = (w >> 2) & 15, s = (w >> 6) & 15;
                const uint32_t key = kind == SYM_BIT ? 0x80000000u | lane : (w >> 16);
                const uint32_t same = __match_any_sync(0xffffffffu, key);
                if (live) {
                    if (kind == SYM_BIT) {
                        pb[j + lane] = pack_step(s ? 16384u : 32768u, s ? 0u : 16384u, s, 1);
                    } else if (lane == __ffs(same) - 1) {   // the group's leader walks its members in order
                        uint16_t *c = cdf + (w >> 16);
                        const uint32_t m = same;   // only live lanes carry CDF keys
                        bool small = kind == SYM_ADAPT && nm1 < 4;
                        for (uint32_t t = m; t && small; t &= t - 1) small = (words[j + __ffs(t) - 1] & 3) == SYM_ADAPT;
                        if (small) {
                            const int N = nm1 + 1;
                            uint32_t cv[3] = {c[0], N > 2 ? c[1] : 0u, N > 3 ? c[2] : 0u};
                            uint32_t count = c[N];
                            int k = j + __ffs(m) - 1;
                            uint32_t wk = words[k];
                            for (uint32_t t = m; t;) {   // the next member's word is loaded while this one is coded
                                const uint32_t tn = t & (t - 1);
                                const int kn = tn ? j + __ffs(tn) - 1 : k;
                                const uint32_t wn = words[kn];
                                pb[k] = bounds_small(cv, count, (wk >> 6) & 15, N);
                                t = tn;
                                k = kn;
                                wk = wn;
                            }
                            c[0] = (uint16_t)cv[0];
                            if (N > 2) c[1] = (uint16_t)cv[1];
                            if (N > 3) c[2] = (uint16_t)cv[2];
                            c[N] = (uint16_t)count;
                        } else {
                            for (uint32_t t = m; t; t &= t - 1) {
                                const int k = j + __ffs(t) - 1;
                                const uint32_t wk = words[k];
                                const int kk = wk & 3, nk = (wk >> 2) & 15, sk = (wk >> 6) & 15;
                                uint32_t fl, fh;
                                if (kk == SYM_ADAPT) {
                                    fl = sk ? 32768u - c[sk - 1] : 32768u;
                                    fh = 32768u - c[sk];
                                    adapt(c, sk, nk + 1);
                                } else {
                                    const uint32_t ms = split_mass(c, kk == SYM_SPLIT_V);
                                    fl = sk ? ms : 32768u;
                                    fh = sk ? 0u : ms;
                                }
                                pb[k] = pack_step(fl, fh, sk, nk);
                            }
                        }
                    }
                }
                __syncwarp();
            }
        }
        if (warp == 1 && lane == 0 && b > 0) {
            const uint64_t at = s0 + (uint64_t)(b - 1) * CODE_BATCH;
            const int n = (int)min((uint64_t)CODE_BATCH, s1 - at);
            const uint32_t *pb = bnd[(b - 1) & 1];
#pragma unroll 4
            for (int j = 0; j < n; j++) E.step(pb[j]);
        }
        __syncthreads();
    }
    if (warp == 1 && lane == 0) {
        const uint32_t bytes = E.finish(A.tbytes + base);
        if (E.over) ent_fail(A, IS_ENT_ERR_OUTPUT);
        A.tileBytes[g] = bytes;
    }
}

// ---- payloads back to back ----
__global__ void __launch_bounds__(SCAN_T) k_ent_offsets(EntArgs A) {
    __shared__ uint32_t sh[32];
    uint64_t carry = 0;
    for (uint32_t b = 0; b < A.nTiles; b += SCAN_T) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t v = i < A.nTiles ? A.tileBytes[i] : 0;
        uint32_t tot;
        const uint32_t e = cta_exclusive(v, sh, &tot);
        if (i < A.nTiles) A.tileOff[i] = carry + e;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        A.tileOff[A.nTiles] = carry;
        A.status->bytes = carry;
    }
}
__global__ void k_ent_pack(EntArgs A) {
    const uint32_t g = blockIdx.x;
    if (A.status->error) return;
    const uint64_t src = 2 * A.symBegin[g] + 16 * (uint64_t)g, dst = A.tileOff[g];
    const uint32_t n = A.tileBytes[g];
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) A.out[dst + i] = A.tbytes[src + i];
}

// ---------------------------------------------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------------------------------------------
cudaError_t ent_upload(const TableBlob &B) {
    cudaError_t e = upload_common(B);
    uint8_t w[22], h[22];
    for (int i = 0; i < 22; i++) { w[i] = AV1G_T(Mi_Width_Log2)[i]; h[i] = AV1G_T(Mi_Height_Log2)[i]; }
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_miWLog2, w, sizeof w);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_miHLog2, h, sizeof h);
    std::vector<uint16_t> init((size_t)4 * NCDF);
    const int qrep[4] = {20, 60, 120, 255};
    for (int q = 0; q < 4; q++) {
        av1g_cdfs c;
        av1g_cdfs_init(&c, qrep[q]);
        memcpy(init.data() + (size_t)q * NCDF, &c, sizeof c);
    }
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_cdfInit, init.data(), init.size() * 2);
    return e;
}

// spec 5.9.15 tile_info with uniform spacing: the requested log2 counts (-1: the minimum legal tiling)
bool tile_info(int W, int H, int colsLog2, int rowsLog2, TileGeom &t) {
    const int MiCols = 2 * ((W + 7) >> 3), MiRows = 2 * ((H + 7) >> 3);
    const int sbCols = (MiCols + 15) >> 4, sbRows = (MiRows + 15) >> 4;
    auto tlog2 = [](int blk, int target) { int k = 0; while ((blk << k) < target) k++; return k; };
    const int maxWSb = 4096 >> 6, maxAreaSb = (4096 * 2304) >> 12;
    t.minLog2Cols = tlog2(maxWSb, sbCols);
    t.maxLog2Cols = tlog2(1, std::min(sbCols, 64));
    t.maxLog2Rows = tlog2(1, std::min(sbRows, 64));
    const int minLog2Tiles = std::max(t.minLog2Cols, tlog2(maxAreaSb, sbRows * sbCols));
    if (colsLog2 < 0) colsLog2 = t.minLog2Cols;
    if (colsLog2 < t.minLog2Cols || colsLog2 > t.maxLog2Cols) return false;
    t.colsLog2 = colsLog2;
    t.wSb = (sbCols + (1 << colsLog2) - 1) >> colsLog2;
    t.cols = (sbCols + t.wSb - 1) / t.wSb;
    t.minLog2Rows = std::max(minLog2Tiles - colsLog2, 0);
    const bool autoRows = rowsLog2 < 0;
    if (autoRows) rowsLog2 = t.minLog2Rows;
    for (;; rowsLog2++) {
        if (rowsLog2 < t.minLog2Rows || rowsLog2 > t.maxLog2Rows) return false;
        const int hSb = (sbRows + (1 << rowsLog2) - 1) >> rowsLog2;
        if (t.wSb * hSb <= maxAreaSb) {
            t.rowsLog2 = rowsLog2;
            t.hSb = hSb;
            t.rows = (sbRows + hSb - 1) / hSb;
            return true;
        }
        if (!autoRows) return false;
    }
}

namespace {

// the frame parameters this coder handles: the toolset of the search's records (no delta-q, palette, filter intra,
// tx-size or reduced-set syntax; lossy; 4:2:0 or 4:4:4; 8- or 10-bit) with CDEF (its per-SB cdef_idx); header-only
// fields are free
bool frame_ok(const av1g_frame_params &fp, std::string *err) {
    const char *why = nullptr;
    if (fp.width < 1 || fp.height < 1 || fp.width > 65536 || fp.height > 65536) why = "size";
    else if (fp.monochrome) why = "monochrome";
    else if (fp.base_q_idx == 0) why = "lossless (base_q_idx 0)";
    else if (fp.bit_depth != 0 && fp.bit_depth != 8 && fp.bit_depth != 10) why = "bit_depth";
    else if (fp.chroma_format > 1) why = "chroma_format";
    else if (fp.tx_mode_select || fp.reduced_tx_set || fp.delta_q_present || fp.enable_filter_intra || fp.allow_screen_content_tools)
        why = "a coding tool outside the search's toolset (tx_mode_select, reduced_tx_set, delta_q, filter intra, palette)";
    else if (fp.enable_cdef > 1 || fp.cdef_bits > 3 || fp.cdef_damping_minus_3 > 3) why = "CDEF parameters";
    if (why && err) *err = std::string("frame parameters: ") + why;
    return !why;
}

struct Plan {
    std::vector<EntFrameD> fr;
    std::vector<uint32_t> fBlock, fTxb, fSb, fTile;
    uint32_t nB = 0, nT = 0, nSb = 0, nTiles = 0;
    uint64_t nMi = 0, nCtx = 0, cap = 0;
    size_t bytes = 0;
    // offsets in the scratch
    size_t oFr, oBases, oMi, oCtx, oType, oEob, oSbFirst, oTxbBlock, oTxbCnt, oHeadCnt, oHeadW, oPartB, oPartT, oSyms,
        oBegin, oPre, oTb, oTileBytes, oResult, oOut;
};

size_t al(size_t v) { return (v + 255) & ~(size_t)255; }

int plan(const is_ent_frame *frames, int n, uint64_t cap, Plan &P, std::string *err) {
    if (n < 1 || !frames) { if (err) *err = "no frames"; return IS_ERR_INVALID; }
    P.fr.resize(n);
    uint64_t defCap = 0;
    for (int i = 0; i < n; i++) {
        const is_ent_frame &f = frames[i];
        if (!frame_ok(f.fp, err)) return IS_ERR_INVALID;
        if (!f.blocks || !f.block_txb || (!f.txb && f.n_txb) || (!f.coeffs && f.n_txb) || !f.n_blocks) {
            if (err) *err = "frame " + std::to_string(i) + ": record arrays missing";
            return IS_ERR_INVALID;
        }
        TileGeom t;
        if (!tile_info((int)f.fp.width, (int)f.fp.height, f.fp.tile_cols_log2, f.fp.tile_rows_log2, t)) {
            if (err) *err = "frame " + std::to_string(i) + ": tiling not allowed";
            return IS_ERR_INVALID;
        }
        EntFrameD &D = P.fr[i];
        memset(&D, 0, sizeof D);
        D.blocks = f.blocks; D.blockTxb = f.block_txb; D.txb = f.txb; D.coeffs = f.coeffs;
        D.MiCols = 2 * (((int)f.fp.width + 7) >> 3);
        D.MiRows = 2 * (((int)f.fp.height + 7) >> 3);
        D.ss = f.fp.chroma_format == AV1G_CHROMA_444 ? 0 : 1;
        D.cdefBits = f.fp.enable_cdef ? f.fp.cdef_bits : -1;
        const int q = f.fp.base_q_idx;
        D.qctx = q <= 20 ? 0 : q <= 60 ? 1 : q <= 120 ? 2 : 3;
        D.sbCols = (D.MiCols + 15) >> 4; D.sbRows = (D.MiRows + 15) >> 4;
        D.tileWSb = t.wSb; D.tileHSb = t.hSb; D.tileCols = t.cols; D.tileRows = t.rows;
        D.blockBase = P.nB; D.nBlocks = f.n_blocks; D.txbBase = P.nT; D.nTxb = f.n_txb;
        D.sbBase = P.nSb; D.tileBase = P.nTiles;
        D.miBase = P.nMi;
        for (int p = 0; p < 3; p++) {
            const int s = p ? D.ss : 0;
            D.ctxW[p] = D.MiCols >> s;
            D.ctxH[p] = D.MiRows >> s;
            D.ctxBase[p] = P.nCtx;
            P.nCtx += (uint64_t)D.ctxW[p] * D.ctxH[p];
        }
        P.fBlock.push_back(P.nB); P.fTxb.push_back(P.nT); P.fSb.push_back(P.nSb); P.fTile.push_back(P.nTiles);
        if ((uint64_t)P.nB + f.n_blocks >= 0xFFFFFFF0ull || (uint64_t)P.nT + f.n_txb >= 0xFFFFFFF0ull) {
            if (err) *err = "batch too large";
            return IS_ERR_INVALID;
        }
        P.nB += f.n_blocks; P.nT += f.n_txb;
        P.nSb += (uint32_t)(D.sbCols * D.sbRows);
        P.nTiles += (uint32_t)(t.cols * t.rows);
        P.nMi += (uint64_t)D.MiCols * D.MiRows;
        const uint64_t px = (uint64_t)D.MiCols * D.MiRows * 16;
        defCap += px * (D.ss ? 2 : 4) + 16ull * f.n_blocks + 8ull * f.n_txb;
    }
    P.fBlock.push_back(P.nB); P.fTxb.push_back(P.nT); P.fSb.push_back(P.nSb); P.fTile.push_back(P.nTiles);
    P.cap = cap ? cap : defCap;
    if (P.cap > 0xF0000000ull) P.cap = 0xF0000000ull;   // stream offsets are 32-bit sums
    const uint32_t npB = (P.nB + SCAN_T - 1) / SCAN_T, npT = (P.nT + SCAN_T - 1) / SCAN_T;
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t at = o; o = al(o + bytes); return at; };
    P.oFr = take(sizeof(EntFrameD) * n);
    P.oBases = take(4ull * 4 * (n + 1));
    P.oMi = take(3 * P.nMi);
    P.oCtx = take(2 * P.nCtx);
    P.oType = take(P.nT + 1);
    P.oEob = take(2ull * (P.nT + 1));
    P.oSbFirst = take(4ull * P.nSb);
    P.oTxbBlock = take(4ull * (P.nT + 1));
    P.oTxbCnt = take(4ull * (P.nT + 1));
    P.oHeadCnt = take(4ull * (P.nB + 1));
    P.oHeadW = take(4ull * HEAD_WORDS * P.nB);
    P.oPartB = take(4ull * (npB + 1));
    P.oPartT = take(4ull * (npT + 1));
    P.oSyms = take(4ull * P.cap);
    P.oBegin = take(8ull * (P.nTiles + 1));
    const uint64_t preN = 2 * P.cap + 16ull * P.nTiles;
    P.oPre = take(2 * preN);
    P.oTb = take(preN);
    P.oTileBytes = take(4ull * P.nTiles);
    P.oResult = take(sizeof(is_ent_status) + 8ull * (P.nTiles + 1));
    P.oOut = take(preN);
    P.bytes = o;
    return IS_OK;
}

}  // namespace

int ent_scratch(const is_ent_frame *frames, int n, uint64_t cap, size_t *bytes, std::string *err) {
    Plan P;
    const int rc = plan(frames, n, cap, P, err);
    if (rc == IS_OK) *bytes = P.bytes;
    return rc;
}

int ent_launch(const is_ent_frame *frames, int n, uint64_t cap, void *scratch, size_t scratchBytes, cudaStream_t s, is_ent_out *out,
               uint32_t *frameTile0, std::string *err) {
    Plan P;
    int rc = plan(frames, n, cap, P, err);
    if (rc != IS_OK) return rc;
    if (!scratch || scratchBytes < P.bytes || ((uintptr_t)scratch & 255)) {
        if (err) *err = "scratch missing, too small or not 256-byte aligned";
        return IS_ERR_INVALID;
    }
    uint8_t *S = (uint8_t *)scratch;
    EntArgs A;
    memset(&A, 0, sizeof A);
    A.fr = (const EntFrameD *)(S + P.oFr);
    A.nF = n;
    uint32_t *bases = (uint32_t *)(S + P.oBases);
    A.fBlock = bases; A.fTxb = bases + (n + 1); A.fSb = bases + 2 * (n + 1); A.fTile = bases + 3 * (n + 1);
    A.nB = P.nB; A.nT = P.nT; A.nSb = P.nSb; A.nTiles = P.nTiles;
    A.miSize = S + P.oMi; A.yMode = A.miSize + P.nMi; A.skip = A.yMode + P.nMi;
    A.cul = S + P.oCtx; A.dcc = A.cul + P.nCtx;
    A.txbType = S + P.oType;
    A.txbEob = (uint16_t *)(S + P.oEob);
    A.sbFirst = (uint32_t *)(S + P.oSbFirst);
    A.txbBlock = (uint32_t *)(S + P.oTxbBlock);
    A.txbCnt = (uint32_t *)(S + P.oTxbCnt);
    A.headCnt = (uint32_t *)(S + P.oHeadCnt);
    A.headW = (uint32_t *)(S + P.oHeadW);
    A.syms = (uint32_t *)(S + P.oSyms);
    A.cap = P.cap;
    A.symBegin = (uint64_t *)(S + P.oBegin);
    A.pre = (uint16_t *)(S + P.oPre);
    A.tbytes = S + P.oTb;
    A.tileBytes = (uint32_t *)(S + P.oTileBytes);
    A.status = (is_ent_status *)(S + P.oResult);
    A.tileOff = (uint64_t *)(S + P.oResult + sizeof(is_ent_status));
    A.out = S + P.oOut;
    std::vector<uint32_t> hb;
    hb.insert(hb.end(), P.fBlock.begin(), P.fBlock.end());
    hb.insert(hb.end(), P.fTxb.begin(), P.fTxb.end());
    hb.insert(hb.end(), P.fSb.begin(), P.fSb.end());
    hb.insert(hb.end(), P.fTile.begin(), P.fTile.end());
    cudaError_t e = cudaMemcpyAsync(S + P.oFr, P.fr.data(), sizeof(EntFrameD) * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(bases, hb.data(), hb.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(A.status, 0, sizeof(is_ent_status), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(A.sbFirst, 0xFF, 4ull * P.nSb, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(A.txbBlock, 0xFF, 4ull * (P.nT + 1), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(A.headCnt, 0, 4ull * (P.nB + 1), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(A.txbCnt, 0, 4ull * (P.nT + 1), s);
    auto grid = [](uint64_t n, int t) { return (unsigned)std::max<uint64_t>(1, (n + t - 1) / t); };
    if (e == cudaSuccess) {
        k_ent_blocks<<<grid(P.nB, 256), 256, 0, s>>>(A);
        if (P.nT) k_ent_txb<<<grid(P.nT, 128), 128, 0, s>>>(A);
        k_ent_sb<<<grid(P.nSb, 64), 64, 0, s>>>(A);
        const uint32_t npB = (P.nB + SCAN_T - 1) / SCAN_T, npT = (P.nT + SCAN_T - 1) / SCAN_T;
        uint32_t *partB = (uint32_t *)(S + P.oPartB), *partT = (uint32_t *)(S + P.oPartT);
        k_scan_local<<<npB, SCAN_T, 0, s>>>(A.headCnt, P.nB, partB);
        k_scan_parts<<<1, SCAN_T, 0, s>>>(partB, npB);
        k_scan_add<<<npB, SCAN_T, 0, s>>>(A.headCnt, P.nB, partB, npB);
        if (P.nT) {
            k_scan_local<<<npT, SCAN_T, 0, s>>>(A.txbCnt, P.nT, partT);
            k_scan_parts<<<1, SCAN_T, 0, s>>>(partT, npT);
            k_scan_add<<<npT, SCAN_T, 0, s>>>(A.txbCnt, P.nT, partT, npT);
        }
        k_ent_tiles<<<grid(P.nTiles, 128), 128, 0, s>>>(A);
        k_ent_emit_head<<<grid(P.nB, 256), 256, 0, s>>>(A);
        if (P.nT) k_ent_emit_txb<<<grid(P.nT, 128), 128, 0, s>>>(A);
        k_ent_code<<<P.nTiles, 64, 0, s>>>(A);
        k_ent_offsets<<<1, SCAN_T, 0, s>>>(A);
        k_ent_pack<<<P.nTiles, 256, 0, s>>>(A);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        if (err) *err = std::string("entropy launch: ") + cudaGetErrorString(e);
        return IS_ERR_CUDA;
    }
    out->result = S + P.oResult;
    out->result_bytes = sizeof(is_ent_status) + 8ull * (P.nTiles + 1);
    out->payload = A.out;
    out->payload_capacity = 2 * P.cap + 16ull * P.nTiles;
    out->n_tiles = P.nTiles;
    if (frameTile0)
        for (int i = 0; i <= n; i++) frameTile0[i] = P.fTile[i];
    return IS_OK;
}

// ---- OBU framing (host): sequence header, frame header, tile group; spec 5.5 (reduced still-picture sequence
// header), 5.9 (uncompressed header of a key frame with reduced_still_picture_header), 5.11.1 (tile group) ----
namespace {
struct Bits {
    std::vector<uint8_t> b;
    int bit = 0;   // bits used in the last byte
    void put(uint32_t v, int n) {
        for (int i = n - 1; i >= 0; i--) {
            if (!bit) b.push_back(0);
            if ((v >> i) & 1) b.back() |= (uint8_t)(0x80 >> bit);
            bit = (bit + 1) & 7;
        }
    }
    void su(int v, int n) { put((uint32_t)v & ((1u << n) - 1), n); }
    void align() { bit = 0; }
    void trailing() { put(1, 1); align(); }
};
void leb128(std::vector<uint8_t> &o, uint64_t v) {
    do {
        uint8_t x = v & 0x7F;
        v >>= 7;
        if (v) x |= 0x80;
        o.push_back(x);
    } while (v);
}
int seq_level(uint32_t W, uint32_t H, int tiles, int cols) {
    if (W < 16 || H < 16) return 31;
    for (int i = 0; i < AV1G_NUM_LEVELS; i++) {
        const uint32_t *L = av1g_levels[i];
        if ((uint64_t)W * H <= L[1] && W <= L[2] && H <= L[3] && (uint32_t)tiles <= L[4] && (uint32_t)cols <= L[5]) return (int)L[0];
    }
    return 31;
}
}  // namespace

int obu_assemble(const av1g_frame_params &fp, const uint8_t *payload, const uint64_t *off, uint32_t nTiles, std::vector<uint8_t> &o,
                 std::string *err) {
    if (!frame_ok(fp, err)) return IS_ERR_INVALID;
    TileGeom t;
    if (!tile_info((int)fp.width, (int)fp.height, fp.tile_cols_log2, fp.tile_rows_log2, t) || (uint32_t)(t.cols * t.rows) != nTiles) {
        if (err) *err = "tile count does not match the frame's tiling";
        return IS_ERR_INVALID;
    }
    for (uint32_t i = 0; i < nTiles; i++)
        if (off[i + 1] <= off[i]) { if (err) *err = "empty tile payload"; return IS_ERR_INVALID; }
    uint64_t maxSz = 0;
    for (uint32_t i = 0; i + 1 < nTiles; i++) maxSz = std::max<uint64_t>(maxSz, off[i + 1] - off[i] - 1);
    const int tsb = maxSz < (1u << 8) ? 1 : maxSz < (1u << 16) ? 2 : maxSz < (1u << 24) ? 3 : 4;
    const int W = (int)fp.width, H = (int)fp.height, bd10 = fp.bit_depth == 10;
    const int ss = fp.chroma_format == AV1G_CHROMA_444 ? 0 : 1;
    const int diffUv = fp.delta_q_v_dc != fp.delta_q_u_dc || fp.delta_q_v_ac != fp.delta_q_u_ac;
    const int sepUv = diffUv || (fp.using_qmatrix && fp.qm_v != fp.qm_u);
    Bits sq, fh;
    // sequence header
    sq.put(ss ? 0 : 1, 3);                            // seq_profile: Main (4:2:0), High (4:4:4)
    sq.put(1, 1);                                     // still_picture
    sq.put(1, 1);                                     // reduced_still_picture_header
    sq.put(seq_level(fp.width, fp.height, t.cols * t.rows, t.cols), 5);
    int wb = 1, hb = 1;
    while ((uint32_t)(W - 1) >> wb) wb++;
    while ((uint32_t)(H - 1) >> hb) hb++;
    sq.put(wb - 1, 4); sq.put(hb - 1, 4);
    sq.put(W - 1, wb); sq.put(H - 1, hb);
    sq.put(0, 1);                                     // use_128x128_superblock
    sq.put(fp.enable_filter_intra, 1);
    sq.put(fp.enable_intra_edge_filter, 1);
    sq.put(0, 1);                                     // enable_superres
    sq.put(fp.enable_cdef, 1);
    sq.put(0, 1);                                     // enable_restoration
    sq.put(bd10, 1);                                  // high_bitdepth
    if (ss) sq.put(0, 1);                             // mono_chrome (not coded in the High profile)
    const int cp = fp.color_description ? fp.color_primaries : 1, tc = fp.color_description ? fp.transfer_characteristics : 13,
              mc = fp.color_description ? fp.matrix_coefficients : 6;
    const int cdp = !(cp == 2 && tc == 2 && mc == 2);
    sq.put(cdp, 1);
    if (cdp) { sq.put(cp, 8); sq.put(tc, 8); sq.put(mc, 8); }
    if (!(cp == 1 && tc == 13 && mc == 0)) sq.put(1, 1);   // color_range full (sRGB: implied)
    if (ss) sq.put(0, 2);                             // chroma_sample_position unknown (4:2:0)
    sq.put(sepUv, 1);
    sq.put(0, 1);                                     // film_grain_params_present
    sq.trailing();
    // frame header
    fh.put(0, 1);                                     // disable_cdf_update
    fh.put(0, 1);                                     // allow_screen_content_tools
    fh.put(0, 1);                                     // render_and_frame_size_different
    fh.put(1, 1);                                     // uniform_tile_spacing_flag
    for (int k = t.minLog2Cols; k < t.maxLog2Cols; k++) {
        fh.put(k < t.colsLog2, 1);
        if (k >= t.colsLog2) break;
    }
    for (int k = t.minLog2Rows; k < t.maxLog2Rows; k++) {
        fh.put(k < t.rowsLog2, 1);
        if (k >= t.rowsLog2) break;
    }
    if (t.colsLog2 > 0 || t.rowsLog2 > 0) {
        fh.put(0, t.colsLog2 + t.rowsLog2);           // context_update_tile_id
        fh.put(tsb - 1, 2);                           // tile_size_bytes_minus_1
    }
    fh.put(fp.base_q_idx, 8);
    auto dq = [&](int v) { if (v) { fh.put(1, 1); fh.su(v, 7); } else fh.put(0, 1); };
    dq(fp.delta_q_y_dc);
    if (sepUv) fh.put(diffUv, 1);
    dq(fp.delta_q_u_dc);
    dq(fp.delta_q_u_ac);
    if (diffUv) { dq(fp.delta_q_v_dc); dq(fp.delta_q_v_ac); }
    fh.put(fp.using_qmatrix, 1);
    if (fp.using_qmatrix) {
        fh.put(fp.qm_y, 4); fh.put(fp.qm_u, 4);
        if (sepUv) fh.put(fp.qm_v, 4);
    }
    fh.put(0, 1);                                     // segmentation_enabled
    fh.put(0, 1);                                     // delta_q_present
    fh.put(fp.loop_filter_level[0], 6);
    fh.put(fp.loop_filter_level[1], 6);
    if (fp.loop_filter_level[0] || fp.loop_filter_level[1]) { fh.put(fp.loop_filter_level[2], 6); fh.put(fp.loop_filter_level[3], 6); }
    fh.put(fp.loop_filter_sharpness, 3);
    fh.put(0, 1);                                     // loop_filter_delta_enabled
    if (fp.enable_cdef) {                             // cdef_params (secondary strength 4 is coded as 3)
        fh.put(fp.cdef_damping_minus_3, 2);
        fh.put(fp.cdef_bits, 2);
        for (int i = 0; i < (1 << fp.cdef_bits); i++) {
            fh.put(fp.cdef_y_pri[i], 4); fh.put(fp.cdef_y_sec[i] == 4 ? 3 : fp.cdef_y_sec[i], 2);
            fh.put(fp.cdef_uv_pri[i], 4); fh.put(fp.cdef_uv_sec[i] == 4 ? 3 : fp.cdef_uv_sec[i], 2);
        }
    }
    fh.put(0, 1);                                     // tx_mode_select
    fh.put(0, 1);                                     // reduced_tx_set
    fh.align();
    std::vector<uint8_t> frame = fh.b;
    if (nTiles > 1) frame.push_back(0);               // tile_start_and_end_present_flag 0 + byte_alignment
    for (uint32_t i = 0; i < nTiles; i++) {
        const uint64_t sz = off[i + 1] - off[i];
        if (i + 1 < nTiles)
            for (int k = 0; k < tsb; k++) frame.push_back((uint8_t)((sz - 1) >> (8 * k)));
        frame.insert(frame.end(), payload + off[i], payload + off[i + 1]);
    }
    o.clear();
    o.push_back(0x0A);                                // OBU_SEQUENCE_HEADER with obu_size
    leb128(o, sq.b.size());
    o.insert(o.end(), sq.b.begin(), sq.b.end());
    o.push_back(0x32);                                // OBU_FRAME with obu_size
    leb128(o, frame.size());
    o.insert(o.end(), frame.begin(), frame.end());
    return IS_OK;
}

// ---- AVIF container (host): the still-image HEIF layout libavif writes (ftyp / meta: hdlr, pitm, iinf, iloc, iprp
// with ispe, av1C, pixi, colr nclx / mdat), the av1C, pixi and colr values from the frame parameters the sequence header
// was written from; av1core's av1g_mux_avif (av1core/src/avif.cpp) writes the same bytes ----
namespace {
struct Box {
    std::vector<uint8_t> b;
    void u8(uint32_t v) { b.push_back((uint8_t)v); }
    void u16(uint32_t v) { u8(v >> 8); u8(v); }
    void u32(uint32_t v) { u16(v >> 16); u16(v & 0xFFFF); }
    void tag(const char *t) { for (int i = 0; i < 4; i++) u8((uint8_t)t[i]); }
    void add(const std::vector<uint8_t> &x) { b.insert(b.end(), x.begin(), x.end()); }
};
// a box of type t around payload p; full boxes carry version and flags first
std::vector<uint8_t> boxed(const char *t, const std::vector<uint8_t> &p, int version = -1, uint32_t flags = 0) {
    Box o;
    o.u32((uint32_t)(8 + (version >= 0 ? 4 : 0) + p.size()));
    o.tag(t);
    if (version >= 0) o.u32(((uint32_t)version << 24) | (flags & 0xFFFFFF));
    o.add(p);
    return o.b;
}
}  // namespace

int avif_write(const av1g_frame_params &fp, const uint8_t *obu, size_t n, std::vector<uint8_t> &out, std::string *err) {
    if (!frame_ok(fp, err)) return IS_ERR_INVALID;
    TileGeom t;
    if (!tile_info((int)fp.width, (int)fp.height, fp.tile_cols_log2, fp.tile_rows_log2, t)) {
        if (err) *err = "tiling not allowed";
        return IS_ERR_INVALID;
    }
    const bool c444 = fp.chroma_format == AV1G_CHROMA_444, hbd = fp.bit_depth == 10;
    const int cp = fp.color_description ? fp.color_primaries : 1, tc = fp.color_description ? fp.transfer_characteristics : 13,
              mc = fp.color_description ? fp.matrix_coefficients : 6;
    // properties of the item: ispe (size), av1C (the sequence header's configuration), pixi (3 channels), colr (CICP,
    // full range: the sequence header always codes or implies color_range 1)
    Box ispe, av1c, pixi, colr;
    ispe.u32(fp.width); ispe.u32(fp.height);
    av1c.u8(0x81);                                                        // marker, version 1
    av1c.u8(((c444 ? 1u : 0u) << 5) | (uint32_t)seq_level(fp.width, fp.height, t.cols * t.rows, t.cols));
    av1c.u8(((hbd ? 1u : 0u) << 6) | ((c444 ? 0u : 1u) << 3) | ((c444 ? 0u : 1u) << 2));   // tier 0, mono 0, CSP unknown
    av1c.u8(0);                                                           // no initial presentation delay
    pixi.u8(3);
    for (int k = 0; k < 3; k++) pixi.u8(hbd ? 10 : 8);
    colr.tag("nclx"); colr.u16(cp); colr.u16(tc); colr.u16(mc); colr.u8(0x80);
    Box ipco;
    ipco.add(boxed("ispe", ispe.b, 0));
    ipco.add(boxed("av1C", av1c.b));
    ipco.add(boxed("pixi", pixi.b, 0));
    ipco.add(boxed("colr", colr.b));
    Box ipma;                                                             // item 1: ispe, av1C essential; pixi, colr
    ipma.u32(1); ipma.u16(1); ipma.u8(4); ipma.u8(0x81); ipma.u8(0x82); ipma.u8(0x03); ipma.u8(0x04);
    Box iprp;
    iprp.add(boxed("ipco", ipco.b));
    iprp.add(boxed("ipma", ipma.b, 0));
    Box hdlr, pitm, infe, iinf;
    hdlr.u32(0); hdlr.tag("pict"); for (int k = 0; k < 12; k++) hdlr.u8(0); hdlr.u8(0);   // no name
    pitm.u16(1);
    infe.u16(1); infe.u16(0); infe.tag("av01"); infe.u8(0);
    iinf.u16(1); iinf.add(boxed("infe", infe.b, 2));
    auto meta = [&](uint32_t dataAt) {
        Box iloc, m;
        iloc.u8(0x44); iloc.u8(0x00);                                     // 4-byte offsets and lengths, no base offset
        iloc.u16(1); iloc.u16(1); iloc.u16(0); iloc.u16(1); iloc.u32(dataAt); iloc.u32((uint32_t)n);
        m.add(boxed("hdlr", hdlr.b, 0));
        m.add(boxed("pitm", pitm.b, 0));
        m.add(boxed("iinf", iinf.b, 0));
        m.add(boxed("iloc", iloc.b, 0));
        m.add(boxed("iprp", iprp.b));
        return boxed("meta", m.b, 0);
    };
    Box ftyp;
    ftyp.tag("avif"); ftyp.u32(0); ftyp.tag("avif"); ftyp.tag("mif1");
    const std::vector<uint8_t> ft = boxed("ftyp", ftyp.b);
    const size_t metaBytes = meta(0).size();                              // the offset field does not change the size
    const uint32_t at = (uint32_t)(ft.size() + metaBytes + 8);
    Box file;
    file.add(ft);
    file.add(meta(at));
    file.u32((uint32_t)(8 + n)); file.tag("mdat");
    file.b.insert(file.b.end(), obu, obu + n);
    out.swap(file.b);
    return IS_OK;
}

}  // namespace is
