// is_dp.cuh - the partition decision of every 64x64 SB over the analysis J grids, and its leaves in decode order (the
// step of the reference's k_dp, encoder/src/k_dp.cuh:72-297; the same decision rule, a different algorithm and thread
// mapping).
//
// One warp per SB.  The quadtree's 85 square nodes are decided level by level, bottom-up (8x8 nodes first): at each
// level every (node, candidate partition) pair is one lane task, its cost written to shared memory; then each node takes
// the cheapest of its candidates.  A partition is described by the table of its parts (the blocks it codes, in decode
// order); the same table gives both a candidate's cost and, after the decision, the node's leaves.
//
// The decision rule (what bit-exact decisions depend on):
//   - a node whose top-left sample lies outside the picture has no blocks (cost 0);
//   - the cost of a partition is the sum of the J of its parts whose top-left sample lies inside the picture (for
//     SPLIT above 8x8: the sum of the four child nodes' costs) plus lambda x its partition bits, saturating at INF;
//   - a node with both its lower and its right half inside the picture considers NONE, HORZ, VERT, SPLIT (8x8 nodes) or
//     all ten partitions, with the partition bits averaged over the contexts; a node with only its right half outside
//     considers SPLIT and VERT, one with only its lower half outside SPLIT and HORZ (256 = one bit each); a node with
//     both outside, SPLIT alone (no bits);
//   - candidates are taken in the order SPLIT, NONE, HORZ, VERT, HORZ_A, HORZ_B, VERT_A, VERT_B, HORZ_4, VERT_4: the
//     first of equal costs wins, and a node none of whose candidates has a finite cost is SPLIT.
// Leaves: the terminal nodes (reached from the root through SPLIT nodes) tile the SB, and the Z-order of their top-left
// 8x8 units is the decode order (pre-order of the partition tree).  Each lane looks at two 8x8 units in Z-order, finds
// the terminal node that holds them, counts the node's parts inside the picture if the unit is the node's top-left, and
// a warp prefix sum of the counts gives every node its first output slot.
#pragma once
#include "is_dev.cuh"
#include "is_frame.cuh"

namespace is {

constexpr int DP_WARPS = 4;
constexpr int DP_NODES = 85;   // 1 + 4 + 16 + 64 square nodes

// part kinds: the sub-size of a square node of side n that a part has (its Partition_Subsize row)
enum { PK_NONE = 0, PK_HORZ, PK_VERT, PK_SQ, PK_H4, PK_V4 };
// the parts of each partition (AV1 partition order), in decode order: (kind, x, y) with x, y in quarters of n
static __constant__ int8_t c_partCount[10] = {1, 2, 2, 4, 3, 3, 3, 3, 4, 4};
static __constant__ int8_t c_partParts[10][4][3] = {
    {{PK_NONE, 0, 0}},                                                  // NONE
    {{PK_HORZ, 0, 0}, {PK_HORZ, 0, 2}},                                 // HORZ
    {{PK_VERT, 0, 0}, {PK_VERT, 2, 0}},                                 // VERT
    {{PK_SQ, 0, 0}, {PK_SQ, 2, 0}, {PK_SQ, 0, 2}, {PK_SQ, 2, 2}},       // SPLIT (its blocks at 8x8: four 4x4)
    {{PK_SQ, 0, 0}, {PK_SQ, 2, 0}, {PK_HORZ, 0, 2}},                    // HORZ_A
    {{PK_HORZ, 0, 0}, {PK_SQ, 0, 2}, {PK_SQ, 2, 2}},                    // HORZ_B
    {{PK_SQ, 0, 0}, {PK_SQ, 0, 2}, {PK_VERT, 2, 0}},                    // VERT_A
    {{PK_VERT, 0, 0}, {PK_SQ, 2, 0}, {PK_SQ, 2, 2}},                    // VERT_B
    {{PK_H4, 0, 0}, {PK_H4, 0, 1}, {PK_H4, 0, 2}, {PK_H4, 0, 3}},       // HORZ_4
    {{PK_V4, 0, 0}, {PK_V4, 1, 0}, {PK_V4, 2, 0}, {PK_V4, 3, 0}}};      // VERT_4
// candidates in consideration order
static __constant__ int8_t c_partOrder[10] = {AV1G_PARTITION_SPLIT, AV1G_PARTITION_NONE, AV1G_PARTITION_HORZ,
                                              AV1G_PARTITION_VERT, AV1G_PARTITION_HORZ_A, AV1G_PARTITION_HORZ_B,
                                              AV1G_PARTITION_VERT_A, AV1G_PARTITION_VERT_B, AV1G_PARTITION_HORZ_4,
                                              AV1G_PARTITION_VERT_4};

__device__ __forceinline__ i64 sat_add(i64 a, i64 b) { return (a >= INF || b >= INF) ? INF : min(a + b, INF); }
// block size of a part kind in a square node of side n (log2 n = ln)
__device__ __forceinline__ int part_bsize(int kind, int ln) {
    const int sq = ln == 3 ? AV1G_BLOCK_8X8 : ln == 4 ? AV1G_BLOCK_16X16 : ln == 5 ? AV1G_BLOCK_32X32 : AV1G_BLOCK_64X64;
    const int p = kind == PK_NONE ? AV1G_PARTITION_NONE : kind == PK_HORZ ? AV1G_PARTITION_HORZ : kind == PK_VERT ? AV1G_PARTITION_VERT
                : kind == PK_SQ ? AV1G_PARTITION_SPLIT : kind == PK_H4 ? AV1G_PARTITION_HORZ_4 : AV1G_PARTITION_VERT_4;
    return ST(Partition_Subsize)[p][sq];
}
// the analysis J of a block of size bs at picture position (x, y) (INF: a size without analysis records)
__device__ __forceinline__ i64 analysis_J(const FrameDesc &F, int bs, int x, int y) {
    if (bs >= AV1G_BLOCK_INVALID || F.shNbx[bs] == 0) return INF;
    return F.blk[F.shOff[bs] + (uint32_t)(y / (4 * bh4(bs))) * F.shNbx[bs] + x / (4 * bw4(bs))].J;
}
__device__ __forceinline__ int level_base(int lv) { return lv == 0 ? 0 : lv == 1 ? 1 : lv == 2 ? 5 : 21; }

struct DpWarp {
    i64 J[DP_NODES];      // node costs
    i64 cost[256];        // the candidates' costs of the level being decided (node-major)
    int8_t P[DP_NODES];   // node partitions (-1: node outside the picture)
};

__global__ void __launch_bounds__(DP_WARPS * 32) k_dp(const __grid_constant__ FrameDesc F, int nSb) {
    __shared__ DpWarp sw[DP_WARPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sb = blockIdx.x * DP_WARPS + w;
    if (sb >= nSb) return;   // (whole warps: sb is uniform across the warp)
    DpWarp &S = sw[w];
    const int sbx = (sb % F.sbCols) * 64, sby = (sb / F.sbCols) * 64;
    const int FW = F.MiCols * 4, FH = F.MiRows * 4;
    for (int lv = 3; lv >= 0; lv--) {
        const int ln = 6 - lv, n = 1 << ln, per = 1 << lv, nNodes = per * per;
        const int nCand = lv == 3 ? 4 : 10, bsl = 4 - lv;   // bsl: the partition-bits row of this node size
        // one (node, candidate) pair per lane task
        for (int t = lane; t < nNodes * nCand; t += 32) {
            const int node = t / nCand, k = t % nCand;
            const int x = sbx + (node % per) * n, y = sby + (node / per) * n;
            i64 c = INF;
            if (x < FW && y < FH) {
                const bool rows = y + n / 2 < FH, cols = x + n / 2 < FW;
                const int p = c_partOrder[k];
                // the candidate set and bits of the node's edge case
                int bits = -1;
                if (rows && cols) bits = c_avgPart[bsl][p];
                else if (k == 0) bits = (rows || cols) ? 256 : 0;   // SPLIT
                else if (k == 2 && !rows && cols) bits = 256;       // HORZ
                else if (k == 3 && rows && !cols) bits = 256;       // VERT
                if (bits >= 0) {
                    i64 J = 0;
                    if (p == AV1G_PARTITION_SPLIT && lv < 3) {
                        const int cb = level_base(lv + 1), cper = per * 2, cx = (node % per) * 2, cy = (node / per) * 2;
                        for (int q = 0; q < 4; q++) J = sat_add(J, S.J[cb + (cy + (q >> 1)) * cper + cx + (q & 1)]);
                    } else {
                        for (int q = 0; q < c_partCount[p]; q++) {
                            const int px = x + c_partParts[p][q][1] * (n >> 2), py = y + c_partParts[p][q][2] * (n >> 2);
                            if (px < FW && py < FH) J = sat_add(J, analysis_J(F, part_bsize(c_partParts[p][q][0], ln), px, py));
                        }
                    }
                    c = sat_add(J, F.lam * bits);
                }
            }
            S.cost[t] = c;
        }
        __syncwarp();
        // each node: its cheapest candidate, the first of equal costs
        for (int node = lane; node < nNodes; node += 32) {
            const int x = sbx + (node % per) * n, y = sby + (node / per) * n;
            const int ni = level_base(lv) + node;
            if (x >= FW || y >= FH) { S.J[ni] = 0; S.P[ni] = -1; continue; }
            i64 best = INF;
            int bp = AV1G_PARTITION_SPLIT;
            for (int k = 0; k < nCand; k++) {
                const i64 c = S.cost[node * nCand + k];
                if (c < best) { best = c; bp = c_partOrder[k]; }
            }
            S.J[ni] = best;
            S.P[ni] = (int8_t)bp;
        }
        __syncwarp();
    }
    // ---- leaves: lane l looks at the 8x8 units 2 l and 2 l + 1 of the Z-order ----
    int cnt[2], tLv[2], tNode[2];
    for (int u = 0; u < 2; u++) {
        const int z = 2 * lane + u;
        const int ux = (z & 1) | ((z >> 1) & 2) | ((z >> 2) & 4), uy = ((z >> 1) & 1) | ((z >> 2) & 2) | ((z >> 3) & 4);
        int lv = 0, node = 0;
        while (lv < 3 && S.P[level_base(lv) + node] == AV1G_PARTITION_SPLIT) {
            lv++;
            node = (uy >> (3 - lv)) * (1 << lv) + (ux >> (3 - lv));
        }
        const int per = 1 << lv, sh = 3 - lv, p = S.P[level_base(lv) + node];
        const bool anchor = (ux >> sh) << sh == ux && (uy >> sh) << sh == uy;
        int c = 0;
        if (anchor && p >= 0) {
            const int n = 64 >> lv, x = sbx + (node % per) * n, y = sby + (node / per) * n;
            for (int q = 0; q < c_partCount[p]; q++)
                c += x + c_partParts[p][q][1] * (n >> 2) < FW && y + c_partParts[p][q][2] * (n >> 2) < FH;
        }
        cnt[u] = c;
        tLv[u] = lv;
        tNode[u] = node;
    }
    const int mine = cnt[0] + cnt[1];
    int incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    int at = incl - mine;
    Leaf *out = F.leaves + (size_t)sb * SB_MAX_LEAVES;
    for (int u = 0; u < 2; u++) {
        if (cnt[u]) {
            const int lv = tLv[u], node = tNode[u], per = 1 << lv, n = 64 >> lv, ln = 6 - lv;
            const int p = S.P[level_base(lv) + node], x = sbx + (node % per) * n, y = sby + (node / per) * n;
            for (int q = 0; q < c_partCount[p]; q++) {
                const int px = x + c_partParts[p][q][1] * (n >> 2), py = y + c_partParts[p][q][2] * (n >> 2);
                if (px >= FW || py >= FH) continue;
                Leaf l;
                l.bsize = (uint8_t)part_bsize(c_partParts[p][q][0], ln);
                l.x4 = (uint8_t)((px - sbx) >> 2);
                l.y4 = (uint8_t)((py - sby) >> 2);
                l.pad = 0;
                out[at++] = l;
            }
        }
    }
    if (lane == 31) F.nLeaves[sb] = (uint16_t)incl;
}

}  // namespace is
