// is_postfilter.cuh - the decoder's post-filters of an intra frame, as host + device functions: the deblocking loop
// filter (spec 7.14) and CDEF (spec 7.15), for 8- and 10-bit samples, 4:2:0 and 4:4:4, no segmentation / delta-lf /
// lossless.  The device kernels (is_k_pf.cu) run one thread per filtered line (deblocking) and per output sample
// (CDEF); the same functions compiled for the host let the tests pin the arithmetic on the CPU against av1core's
// av1g_postfilter (av1core/src/encoder.cpp:1998-2041), the reference's CPU post-filter.
//
// Maps (built from the record's blocks by pf_mark_block, one thread per block): Skips per luma 4x4, the loop-filter tx
// size of every 4x4 of each plane, the cdef_idx of every 64x64 (-1 where no block of it is coded: CDEF leaves it).
// Order: deblocking pass 0 (vertical edges) of every plane, then pass 1 (horizontal edges) - within a pass every edge
// is independent (a filter never reaches the samples another edge of the pass changes) - then CDEF from the deblocked
// frame into a separate frame (every sample independent).
#pragma once
#include <stddef.h>
#include <stdint.h>
#include "av1g/decisions.h"
#include "av1g/enums_gen.h"
#include "av1g/spec_tables.h"

#if defined(__CUDACC__)
#define IS_PF_HD __host__ __device__ __forceinline__
#else
#define IS_PF_HD static inline
#endif

namespace is {

// the filter parameters of a frame and its maps
struct PfFrame {
    int W, H, MiRows, MiCols, ssx, ssy, bd;
    int lvl[4];                   // effective deblocking levels: Y vertical edges, Y horizontal edges, U, V (0: off)
    int sharp;                    // loop_filter_sharpness
    int cdefOn, damping;          // enable_cdef, CdefDamping (cdef_damping_minus_3 + 3)
    int yPri[8], ySec[8], uvPri[8], uvSec[8];
    int sbCols;
    uint8_t *skip;                // Skips, MiRows x MiCols
    uint8_t *txs[3];              // loop-filter tx sizes per 4x4 of each plane: luma MiRows x MiCols, chroma >> ss
    int8_t *cdefIdx;              // per 64x64 (raster over sbCols), -1: no CDEF
};

IS_PF_HD int pf_abs(int v) { return v < 0 ? -v : v; }
IS_PF_HD int pf_clip(int lo, int hi, int v) { return v < lo ? lo : v > hi ? hi : v; }
IS_PF_HD int pf_log2(unsigned v) {   // FloorLog2 of v > 0
    int k = 0;
    while (v >> (k + 1)) k++;
    return k;
}

// frame parameters from the record's av1g_frame_params (effective levels: no chroma deblocking without a luma level)
IS_PF_HD void pf_init(const av1g_frame_params &fp, PfFrame &f) {
    f.W = (int)fp.width;
    f.H = (int)fp.height;
    f.MiCols = 2 * ((f.W + 7) >> 3);
    f.MiRows = 2 * ((f.H + 7) >> 3);
    f.ssx = f.ssy = fp.chroma_format == AV1G_CHROMA_444 ? 0 : 1;
    f.bd = fp.bit_depth == 10 ? 10 : 8;
    const bool luma = fp.loop_filter_level[0] || fp.loop_filter_level[1];
    for (int i = 0; i < 4; i++) f.lvl[i] = (i < 2 || luma) ? fp.loop_filter_level[i] : 0;
    f.sharp = fp.loop_filter_sharpness;
    f.cdefOn = fp.enable_cdef;
    f.damping = fp.cdef_damping_minus_3 + 3;
    for (int i = 0; i < 8; i++) {
        f.yPri[i] = fp.cdef_y_pri[i]; f.ySec[i] = fp.cdef_y_sec[i];
        f.uvPri[i] = fp.cdef_uv_pri[i]; f.uvSec[i] = fp.cdef_uv_sec[i];
    }
    f.sbCols = (f.MiCols + 15) >> 4;
}

// one block's entries of the maps (tx_depth 0: the luma tx size is the block's largest; chroma as the record layout)
IS_PF_HD void pf_mark_block(const PfFrame &f, const av1g_block &b) {
    const int r0 = b.mi_row, c0 = b.mi_col, bs = b.bsize;
    const int w4 = AV1G_T(Num_4x4_Blocks_Wide)[bs], h4 = AV1G_T(Num_4x4_Blocks_High)[bs];
    const int txY = AV1G_T(Max_Tx_Size_Rect)[bs];
    for (int y = r0; y < r0 + h4 && y < f.MiRows; y++)
        for (int x = c0; x < c0 + w4 && x < f.MiCols; x++) {
            f.skip[(size_t)y * f.MiCols + x] = b.skip;
            f.txs[0][(size_t)y * f.MiCols + x] = (uint8_t)txY;
        }
    const bool hasC = !(f.ssy && h4 == 1 && !(r0 & 1)) && !(f.ssx && w4 == 1 && !(c0 & 1));
    if (hasC) {
        const int cbs = AV1G_T(Subsampled_Size)[bs][f.ssx][f.ssy];
        int t = AV1G_T(Max_Tx_Size_Rect)[cbs];
        const int tw = AV1G_T(Tx_Width)[t], th = AV1G_T(Tx_Height)[t];
        if (tw == 64 || th == 64) t = tw == 16 ? AV1G_TX_16X32 : th == 16 ? AV1G_TX_32X16 : AV1G_TX_32X32;   // chroma <= 32
        const int cw = f.MiCols >> f.ssx, ch = f.MiRows >> f.ssy, y0 = r0 >> f.ssy, x0 = c0 >> f.ssx;
        const int bw = AV1G_T(Num_4x4_Blocks_Wide)[cbs], bh = AV1G_T(Num_4x4_Blocks_High)[cbs];
        for (int y = y0; y < y0 + bh && y < ch; y++)
            for (int x = x0; x < x0 + bw && x < cw; x++) {
                f.txs[1][(size_t)y * cw + x] = (uint8_t)t;
                f.txs[2][(size_t)y * cw + x] = (uint8_t)t;
            }
    }
    if (f.cdefOn && !b.skip) f.cdefIdx[(size_t)(r0 >> 4) * f.sbCols + (c0 >> 4)] = b.cdef_idx;
}

// ---------------------------------------------------------------------------------------------------------------
// deblocking
// ---------------------------------------------------------------------------------------------------------------
// the edge of the 4x4 at plane position (x4, y4) in a pass: false when there is none to filter; else the filter size
// (4, 6 / 8, 16 taps class) and the level's limits (spec 7.14.2 edge_loop_filter, 7.14.4 filter size, 7.14.5 adaptive
// filter strength without deltas)
struct PfEdge { int size, limit, blimit, thresh; };
IS_PF_HD bool pf_edge(const PfFrame &f, int plane, int pass, int x4, int y4, PfEdge &e) {
    const int sx = plane ? f.ssx : 0, sy = plane ? f.ssy : 0;
    const int lx = (x4 << sx) * 4, ly = (y4 << sy) * 4;   // the luma position of the 4x4's mode-info unit
    if (lx >= f.W || ly >= f.H) return false;
    if (pass == 0 ? x4 == 0 : y4 == 0) return false;
    const int lvl = f.lvl[plane == 0 ? pass : plane + 1];
    if (!lvl) return false;
    const int pw = f.MiCols >> sx;
    const uint8_t *t = f.txs[plane];
    const int cur = t[(size_t)y4 * pw + x4], prev = pass == 0 ? t[(size_t)y4 * pw + x4 - 1] : t[(size_t)(y4 - 1) * pw + x4];
    const int dc = pass == 0 ? AV1G_T(Tx_Width)[cur] : AV1G_T(Tx_Height)[cur];
    const int dp = pass == 0 ? AV1G_T(Tx_Width)[prev] : AV1G_T(Tx_Height)[prev];
    if (((pass == 0 ? x4 : y4) * 4) % dc) return false;   // not a tx edge (an intra block filters every tx edge)
    const int base = dc < dp ? dc : dp, cap = plane ? 8 : 16;
    e.size = base < cap ? base : cap;
    const int shift = f.sharp > 4 ? 2 : f.sharp > 0 ? 1 : 0;
    int limit = lvl >> shift;
    limit = f.sharp > 0 ? pf_clip(1, 9 - f.sharp, limit) : (limit > 1 ? limit : 1);
    e.limit = limit;
    e.blimit = 2 * (lvl + 2) + limit;
    e.thresh = lvl >> 4;
    return true;
}

// the wide filter (spec 7.14.6.4) of n samples each side; the taps within `wide` of the edge count twice
template <int N, int TWICE, int LOG2, typename P>
IS_PF_HD void pf_wide(P *q0, ptrdiff_t step) {
    int v[2 * N + 2];
#pragma unroll
    for (int k = 0; k < 2 * N + 2; k++) v[k] = q0[(k - N - 1) * step];   // v[N + 1 + i] = sample i (q side from 0)
    int out[2 * N];
#pragma unroll
    for (int i = -N; i < N; i++) {
        int t = 0;
#pragma unroll
        for (int j = -N; j <= N; j++) {
            const int k = i + j < -(N + 1) ? -(N + 1) : i + j > N ? N : i + j;
            t += v[k + N + 1] * ((j < 0 ? -j : j) <= TWICE ? 2 : 1);
        }
        out[i + N] = (t + (1 << (LOG2 - 1))) >> LOG2;
    }
#pragma unroll
    for (int i = -N; i < N; i++) q0[i * step] = (P)out[i + N];
}

// sample filtering (spec 7.14.6) of one line across an edge: q0 points at the first sample after the edge, step to the
// next one across it
template <typename P>
IS_PF_HD void pf_line(P *q0, ptrdiff_t step, int plane, const PfEdge &e, int bd) {
    const int sh = bd - 8;
    const int limit = e.limit << sh, blimit = e.blimit << sh, thresh = e.thresh << sh, flat = 1 << sh;
    const int taps = e.size == 4 ? 4 : plane ? 6 : e.size == 8 ? 8 : 16;
    const int p0 = q0[-step], p1 = q0[-2 * step], qa = q0[0], q1 = q0[step];
    bool bad = pf_abs(p1 - p0) > limit || pf_abs(q1 - qa) > limit || pf_abs(p0 - qa) * 2 + pf_abs(p1 - q1) / 2 > blimit;
    int p2 = 0, q2 = 0, p3 = 0, q3 = 0;
    if (taps >= 6) {
        p2 = q0[-3 * step]; q2 = q0[2 * step];
        bad = bad || pf_abs(p2 - p1) > limit || pf_abs(q2 - q1) > limit;
    }
    if (taps >= 8) {
        p3 = q0[-4 * step]; q3 = q0[3 * step];
        bad = bad || pf_abs(p3 - p2) > limit || pf_abs(q3 - q2) > limit;
    }
    if (bad) return;
    const bool hev = pf_abs(p1 - p0) > thresh || pf_abs(q1 - qa) > thresh;
    bool isFlat = false, isFlat2 = false;
    if (e.size >= 8) {
        isFlat = pf_abs(p1 - p0) <= flat && pf_abs(q1 - qa) <= flat && pf_abs(p2 - p0) <= flat && pf_abs(q2 - qa) <= flat;
        if (taps >= 8) isFlat = isFlat && pf_abs(p3 - p0) <= flat && pf_abs(q3 - qa) <= flat;
    }
    if (e.size >= 16 && isFlat) {
        isFlat2 = true;
        for (int k = 4; k <= 6; k++)
            isFlat2 = isFlat2 && pf_abs((int)q0[-(k + 1) * step] - p0) <= flat && pf_abs((int)q0[k * step] - qa) <= flat;
    }
    if (e.size == 4 || !isFlat) {   // narrow filter (7.14.6.3), in signed sample units
        const int half = 0x80 << sh, lo = -(1 << (bd - 1)), hi = (1 << (bd - 1)) - 1;
        const int ps1 = p1 - half, ps0 = p0 - half, qs0 = qa - half, qs1 = q1 - half;
        int fv = hev ? pf_clip(lo, hi, ps1 - qs1) : 0;
        fv = pf_clip(lo, hi, fv + 3 * (qs0 - ps0));
        const int f1 = pf_clip(lo, hi, fv + 4) >> 3, f2 = pf_clip(lo, hi, fv + 3) >> 3;
        q0[0] = (P)(pf_clip(lo, hi, qs0 - f1) + half);
        q0[-step] = (P)(pf_clip(lo, hi, ps0 + f2) + half);
        if (!hev) {
            const int a = (f1 + 1) >> 1;
            q0[step] = (P)(pf_clip(lo, hi, qs1 - a) + half);
            q0[-2 * step] = (P)(pf_clip(lo, hi, ps1 + a) + half);
        }
        return;
    }
    if (e.size >= 16 && isFlat2) pf_wide<6, 1, 4>(q0, step);
    else if (plane == 0) pf_wide<3, 0, 3>(q0, step);
    else pf_wide<2, 1, 3>(q0, step);
}

// ---------------------------------------------------------------------------------------------------------------
// CDEF
// ---------------------------------------------------------------------------------------------------------------
// the spec's Cdef_Directions: (row, col) of the first and second tap of each of the 8 directions
#if defined(__CUDACC__)
static __device__ const int8_t c_pfCdefDir[8][2][2] = {{{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}}, {{0, 1}, {0, 2}}, {{0, 1}, {1, 2}},
                                                       {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},  {{1, 0}, {2, 0}}, {{1, 0}, {2, -1}}};
#endif
static const int8_t h_pfCdefDir[8][2][2] = {{{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}}, {{0, 1}, {0, 2}}, {{0, 1}, {1, 2}},
                                            {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},  {{1, 0}, {2, 0}}, {{1, 0}, {2, -1}}};
#if defined(__CUDA_ARCH__)
#define IS_PF_DIR c_pfCdefDir
#else
#define IS_PF_DIR h_pfCdefDir
#endif

// direction search (spec 7.15.2) of the 8x8 luma block at src: the direction of the line pattern the block follows
// best and the variance term of the luma strength adjustment
template <typename P>
IS_PF_HD void pf_cdef_dir(const P *src, ptrdiff_t stride, int bd, int &dir, int &var) {
    int part[8][15];
    for (int d = 0; d < 8; d++)
        for (int k = 0; k < 15; k++) part[d][k] = 0;
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) {
            const int x = ((int)src[i * stride + j] >> (bd - 8)) - 128;
            part[0][i + j] += x;
            part[1][i + (j >> 1)] += x;
            part[2][i] += x;
            part[3][3 + i - (j >> 1)] += x;
            part[4][7 + i - j] += x;
            part[5][3 - (i >> 1) + j] += x;
            part[6][j] += x;
            part[7][(i >> 1) + j] += x;
        }
    // 840 / n for a line of n samples (the spec's Div_Table), so every direction's cost is on one scale
    const int div[9] = {0, 840, 420, 280, 210, 168, 140, 120, 105};
    int cost[8];
    for (int d = 0; d < 8; d += 2) {   // straight and diagonal directions
        int c = 0;
        if (d == 2 || d == 6) {
            for (int k = 0; k < 8; k++) c += part[d][k] * part[d][k];
            c *= div[8];
        } else {
            for (int k = 0; k < 7; k++) c += (part[d][k] * part[d][k] + part[d][14 - k] * part[d][14 - k]) * div[k + 1];
            c += part[d][7] * part[d][7] * div[8];
        }
        cost[d] = c;
    }
    for (int d = 1; d < 8; d += 2) {   // the four directions between
        int c = 0;
        for (int k = 3; k < 8; k++) c += part[d][k] * part[d][k];
        c *= div[8];
        for (int k = 0; k < 3; k++) c += (part[d][k] * part[d][k] + part[d][10 - k] * part[d][10 - k]) * div[2 * k + 2];
        cost[d] = c;
    }
    int best = 0, bc = 0;
    for (int d = 0; d < 8; d++)
        if (cost[d] > bc) { bc = cost[d]; best = d; }
    dir = best;
    var = (bc - cost[(best + 4) & 7]) >> 10;
}

// the CDEF of one 8x8 block (spec 7.15.1): -1 when it is left as it is, else its cdef_idx
IS_PF_HD int pf_cdef_idx(const PfFrame &f, int r, int c) {   // r, c: luma 4x4 position (even)
    if (!f.cdefOn) return -1;
    const int idx = f.cdefIdx[(size_t)(r >> 4) * f.sbCols + (c >> 4)];
    if (idx < 0) return -1;
    const size_t w = (size_t)f.MiCols;
    const uint8_t *s = f.skip;
    return (s[r * w + c] && s[r * w + c + 1] && s[(r + 1) * w + c] && s[(r + 1) * w + c + 1]) ? -1 : idx;
}

// strengths and direction of a plane in a filtered block (spec 7.15.1): pri, sec (<< (BitDepth - 8), luma primary
// adjusted by the block's variance), the direction (0 without a primary strength)
struct PfCdef { int pri, sec, dir, damping; };
IS_PF_HD PfCdef pf_cdef_plane(const PfFrame &f, int plane, int idx, int dir, int var) {
    PfCdef o;
    const int sh = f.bd - 8;
    if (plane == 0) {
        const int pri = f.yPri[idx] << sh;
        int adj = 0;
        if (var >> 6) { adj = pf_log2((unsigned)(var >> 6)); adj = adj < 12 ? adj : 12; }
        o.pri = var ? (pri * (4 + adj) + 8) >> 4 : 0;
        o.sec = f.ySec[idx] << sh;
        o.dir = pri ? dir : 0;
        o.damping = f.damping + sh;
    } else {
        o.pri = f.uvPri[idx] << sh;
        o.sec = f.uvSec[idx] << sh;
        o.dir = o.pri ? dir : 0;
        o.damping = f.damping + sh - 1;
    }
    return o;
}

IS_PF_HD int pf_constrain(int diff, int strength, int damping) {
    if (!strength) return 0;
    int adj = damping - pf_log2((unsigned)strength);
    adj = adj > 0 ? adj : 0;
    const int a = pf_abs(diff);
    const int v = pf_clip(0, a, strength - (a >> adj));
    return diff < 0 ? -v : v;
}

// the CDEF filter (spec 7.15.3) of the sample at plane position (x, y) of the deblocked plane src; taps outside the
// frame's coded area are not available
template <typename P>
IS_PF_HD int pf_cdef_sample(const PfFrame &f, const P *src, ptrdiff_t stride, int plane, int x, int y, const PfCdef &c) {
    const int sx = plane ? f.ssx : 0, sy = plane ? f.ssy : 0;
    const int x0 = src[(size_t)y * stride + x];
    const int odd = (c.pri >> (f.bd - 8)) & 1;
    int sum = 0, mx = x0, mn = x0;
    for (int k = 0; k < 2; k++)
        for (int sg = -1; sg <= 1; sg += 2)
            for (int t = 0; t < 3; t++) {   // the primary tap, then the secondary ones at direction -2 / +2
                const int d = t == 0 ? c.dir : (c.dir + (t == 1 ? 6 : 2)) & 7;
                const int yy = y + sg * IS_PF_DIR[d][k][0], xx = x + sg * IS_PF_DIR[d][k][1];
                if (yy < 0 || xx < 0 || ((yy << sy) >> 2) >= f.MiRows || ((xx << sx) >> 2) >= f.MiCols) continue;
                const int p = src[(size_t)yy * stride + xx];
                if (t == 0) sum += (odd ? 3 : (k ? 2 : 4)) * pf_constrain(p - x0, c.pri, c.damping);
                else sum += (k ? 1 : 2) * pf_constrain(p - x0, c.sec, c.damping);
                mx = p > mx ? p : mx;
                mn = p < mn ? p : mn;
            }
    return pf_clip(mn, mx, x0 + ((8 + sum - (sum < 0)) >> 4));
}

}  // namespace is
