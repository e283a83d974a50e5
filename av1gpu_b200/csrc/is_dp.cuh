// is_dp.cuh - partition DP per 64x64 SB over the analysis J grids, then the leaves in decode order
// (the reference's k_dp, encoder/src/k_dp.cuh:72-297): bottom-up over the 85 square nodes, every partition type
// (8x8 nodes: NONE / HORZ / VERT / SPLIT), J + lambda * averaged partition bits; nodes cut by the frame edge keep
// HORZ / VERT / SPLIT as the syntax allows.  One thread per SB (the whole DP is ~1 k integer ops).
#pragma once
#include "is_dev.cuh"
#include "is_frame.cuh"

namespace is {

__device__ __forceinline__ i64 sat_add(i64 a, i64 b) { return (a >= INF || b >= INF) ? INF : min(a + b, INF); }
__device__ __forceinline__ int sq_bsize(int n) {
    return n == 4 ? AV1G_BLOCK_4X4 : n == 8 ? AV1G_BLOCK_8X8 : n == 16 ? AV1G_BLOCK_16X16 : n == 32 ? AV1G_BLOCK_32X32 : AV1G_BLOCK_64X64;
}
__device__ __forceinline__ int sub_bsize(int p, int n) { return ST(Partition_Subsize)[p][sq_bsize(n)]; }

__device__ __forceinline__ i64 dp_blockJ(const FrameDesc &F, int bs, int x, int y) {
    if (bs >= AV1G_BLOCK_INVALID || F.shNbx[bs] == 0) return INF;
    return F.blk[F.shOff[bs] + (uint32_t)(y / (4 * bh4(bs))) * F.shNbx[bs] + x / (4 * bw4(bs))].J;
}

__global__ void k_dp(const __grid_constant__ FrameDesc F, int nSb) {
    const int sb = blockIdx.x * blockDim.x + threadIdx.x;
    if (sb >= nSb) return;
    const int sbx = (sb % F.sbCols) * 64, sby = (sb / F.sbCols) * 64;
    const int FW = F.MiCols * 4, FH = F.MiRows * 4;
    const i64 lam = F.lam;
    i64 nJ[85];
    int8_t nP[85];
    const int lvBase[4] = {0, 1, 5, 21};
    for (int Lv = 3; Lv >= 0; Lv--) {
        const int n = 64 >> Lv, half = n >> 1, q4 = n >> 2, per = 1 << Lv;
        const int bsl = Lv == 3 ? 1 : Lv == 2 ? 2 : Lv == 1 ? 3 : 4;
        for (int ny = 0; ny < per; ny++)
            for (int nx = 0; nx < per; nx++) {
                const int ni = lvBase[Lv] + ny * per + nx;
                const int x = sbx + nx * n, y = sby + ny * n;
                if (x >= FW || y >= FH) { nJ[ni] = 0; nP[ni] = -1; continue; }
                const bool hasRows = (y + half) < FH, hasCols = (x + half) < FW;
                i64 splitJ = 0;
                if (n == 8) {
                    for (int k = 0; k < 4; k++) {
                        const int xx = x + (k & 1) * 4, yy = y + (k >> 1) * 4;
                        if (xx < FW && yy < FH) splitJ = sat_add(splitJ, dp_blockJ(F, AV1G_BLOCK_4X4, xx, yy));
                    }
                } else {
                    const int cb = lvBase[Lv + 1], cper = per * 2;
                    for (int k = 0; k < 4; k++) splitJ = sat_add(splitJ, nJ[cb + (ny * 2 + (k >> 1)) * cper + nx * 2 + (k & 1)]);
                }
                i64 best = INF;
                int bp = AV1G_PARTITION_SPLIT;
                auto consider = [&](int p, i64 J, int bits) {
                    const i64 t = sat_add(J, lam * bits);
                    if (t < best) { best = t; bp = p; }
                };
                if (hasRows && hasCols) {
                    const int *pb = c_avgPart[bsl];
                    consider(AV1G_PARTITION_SPLIT, splitJ, pb[AV1G_PARTITION_SPLIT]);
                    const int hz = sub_bsize(AV1G_PARTITION_HORZ, n), vt = sub_bsize(AV1G_PARTITION_VERT, n), sp = sub_bsize(AV1G_PARTITION_SPLIT, n);
                    const i64 jn = dp_blockJ(F, sq_bsize(n), x, y);
                    if (jn < INF) consider(AV1G_PARTITION_NONE, jn, pb[AV1G_PARTITION_NONE]);
                    consider(AV1G_PARTITION_HORZ, sat_add(dp_blockJ(F, hz, x, y), dp_blockJ(F, hz, x, y + half)), pb[AV1G_PARTITION_HORZ]);
                    consider(AV1G_PARTITION_VERT, sat_add(dp_blockJ(F, vt, x, y), dp_blockJ(F, vt, x + half, y)), pb[AV1G_PARTITION_VERT]);
                    if (n > 8) {
                        const i64 s00 = dp_blockJ(F, sp, x, y), s01 = dp_blockJ(F, sp, x + half, y);
                        const i64 s10 = dp_blockJ(F, sp, x, y + half), s11 = dp_blockJ(F, sp, x + half, y + half);
                        consider(AV1G_PARTITION_HORZ_A, sat_add(sat_add(s00, s01), dp_blockJ(F, hz, x, y + half)), pb[AV1G_PARTITION_HORZ_A]);
                        consider(AV1G_PARTITION_HORZ_B, sat_add(sat_add(dp_blockJ(F, hz, x, y), s10), s11), pb[AV1G_PARTITION_HORZ_B]);
                        consider(AV1G_PARTITION_VERT_A, sat_add(sat_add(s00, s10), dp_blockJ(F, vt, x + half, y)), pb[AV1G_PARTITION_VERT_A]);
                        consider(AV1G_PARTITION_VERT_B, sat_add(sat_add(dp_blockJ(F, vt, x, y), s01), s11), pb[AV1G_PARTITION_VERT_B]);
                        const int h4 = sub_bsize(AV1G_PARTITION_HORZ_4, n), v4 = sub_bsize(AV1G_PARTITION_VERT_4, n);
                        i64 Jh = 0, Jv = 0;
                        for (int i = 0; i < 4; i++) if (i < 3 || y + 3 * q4 < FH) Jh = sat_add(Jh, dp_blockJ(F, h4, x, y + i * q4));
                        consider(AV1G_PARTITION_HORZ_4, Jh, pb[AV1G_PARTITION_HORZ_4]);
                        for (int i = 0; i < 4; i++) if (i < 3 || x + 3 * q4 < FW) Jv = sat_add(Jv, dp_blockJ(F, v4, x + i * q4, y));
                        consider(AV1G_PARTITION_VERT_4, Jv, pb[AV1G_PARTITION_VERT_4]);
                    }
                } else if (hasCols) {
                    consider(AV1G_PARTITION_SPLIT, splitJ, 256);
                    consider(AV1G_PARTITION_HORZ, dp_blockJ(F, sub_bsize(AV1G_PARTITION_HORZ, n), x, y), 256);
                } else if (hasRows) {
                    consider(AV1G_PARTITION_SPLIT, splitJ, 256);
                    consider(AV1G_PARTITION_VERT, dp_blockJ(F, sub_bsize(AV1G_PARTITION_VERT, n), x, y), 256);
                } else {
                    consider(AV1G_PARTITION_SPLIT, splitJ, 0);
                }
                nJ[ni] = best;
                nP[ni] = (int8_t)bp;
            }
    }
    // leaves in decode order (pre-order walk of decode_partition)
    Leaf *out = F.leaves + (size_t)sb * SB_MAX_LEAVES;
    int nl = 0;
    auto leaf = [&](int bs, int x, int y) {
        if (x >= FW || y >= FH) return;
        Leaf l;
        l.bsize = (uint8_t)bs; l.x4 = (uint8_t)((x - sbx) >> 2); l.y4 = (uint8_t)((y - sby) >> 2); l.pad = 0;
        out[nl++] = l;
    };
    int stk[64][3], sp = 0;
    stk[0][0] = 0; stk[0][1] = 0; stk[0][2] = 0; sp = 1;
    while (sp > 0) {
        sp--;
        const int Lv = stk[sp][0], nx = stk[sp][1], ny = stk[sp][2];
        const int n = 64 >> Lv, half = n >> 1, q4 = n >> 2, per = 1 << Lv;
        const int ni = lvBase[Lv] + ny * per + nx;
        const int x = sbx + nx * n, y = sby + ny * n;
        if (nP[ni] < 0) continue;
        const int p = nP[ni], sub = sub_bsize(p, n), sp2 = sub_bsize(AV1G_PARTITION_SPLIT, n);
        const bool hasRows = (y + half) < FH, hasCols = (x + half) < FW;
        switch (p) {
        case AV1G_PARTITION_NONE: leaf(sub, x, y); break;
        case AV1G_PARTITION_HORZ: leaf(sub, x, y); if (hasRows) leaf(sub, x, y + half); break;
        case AV1G_PARTITION_VERT: leaf(sub, x, y); if (hasCols) leaf(sub, x + half, y); break;
        case AV1G_PARTITION_SPLIT:
            if (n == 8) {
                leaf(AV1G_BLOCK_4X4, x, y); leaf(AV1G_BLOCK_4X4, x + 4, y);
                leaf(AV1G_BLOCK_4X4, x, y + 4); leaf(AV1G_BLOCK_4X4, x + 4, y + 4);
            } else {
                for (int k = 3; k >= 0; k--) { stk[sp][0] = Lv + 1; stk[sp][1] = nx * 2 + (k & 1); stk[sp][2] = ny * 2 + (k >> 1); sp++; }
            }
            break;
        case AV1G_PARTITION_HORZ_A: leaf(sp2, x, y); leaf(sp2, x + half, y); leaf(sub, x, y + half); break;
        case AV1G_PARTITION_HORZ_B: leaf(sub, x, y); leaf(sp2, x, y + half); leaf(sp2, x + half, y + half); break;
        case AV1G_PARTITION_VERT_A: leaf(sp2, x, y); leaf(sp2, x, y + half); leaf(sub, x + half, y); break;
        case AV1G_PARTITION_VERT_B: leaf(sub, x, y); leaf(sp2, x + half, y); leaf(sp2, x + half, y + half); break;
        case AV1G_PARTITION_HORZ_4: for (int i = 0; i < 4; i++) if (i < 3 || y + 3 * q4 < FH) leaf(sub, x, y + i * q4); break;
        default: for (int i = 0; i < 4; i++) if (i < 3 || x + 3 * q4 < FW) leaf(sub, x + i * q4, y); break;
        }
    }
    F.nLeaves[sb] = (uint16_t)nl;
}

}  // namespace is
