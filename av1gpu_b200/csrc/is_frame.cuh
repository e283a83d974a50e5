// is_frame.cuh - the per-image descriptor shared by the host orchestration and the kernels, and the HBM layout.
//
// HBM layout of one image (all in one workspace, 256-byte aligned sub-buffers):
//   src[p], rec[p]   planes with a margin of SRC_MARGIN_Y rows above and SRC_MARGIN_X samples left of sample (0, 0),
//                    padded by edge replication to the 64x64 SB grid plus one SB column, pitch a multiple of 16 bytes,
//                    so a superblock tile and its edges are always in bounds for 128-bit loads.
//   blk              analysis records, shape-major: blk[shOff[s] + by * shNbx[s] + bx] (16 bytes)
//   leaves / nLeaves DP output, 256 slots per SB
//   mYMode, cLvl, cDc  4x4 context maps (luma MiRows x MiCols, chroma (MiRows >> ss) x (MiCols >> ss))
//   oBlocks / oTxb / oCoeffs  closed-loop output slots per SB (compacted into the DecisionRecord by k_pack)
#pragma once
#include <stdint.h>
#include "av1g/decisions.h"

namespace is {

constexpr int SRC_MARGIN_X = 16, SRC_MARGIN_Y = 1;
constexpr int SB_MAX_LEAVES = 256;
constexpr int SB_MAX_TXB = 768;      // luma 256 + chroma 2 x 256 (4:4:4 bound)
constexpr int SB_MAX_COEF = 12288;   // 3 x 64 x 64
// dependency entries per SB: a leaf of bw x bh luma 4x4 units has at most 2 bw + 1 + 2 bh luma dependencies (at most
// 5 bw bh) and, as a 4:2:0 chroma carrier narrower or lower than 8 samples, at most 5 more for its chroma strips; over
// the 2 x 2 (or 2 x 1) group of such leaves that is at most 8 per unit, so the leaves of one SB have at most 8 x 256
constexpr int REV_PER_SB = 2048;

struct BlockRes {      // analysis result of one (shape, position): 16 bytes
    long long J;       // best open-loop RD cost (J units)
    uint8_t cand[4];   // candidates (mode << 3 | delta + 3), best first
    uint8_t ncand;
    uint8_t tx;        // best tx type of cand[0]
    uint16_t txMask;   // tx types the closed loop's second pass may try for cand[0] (bit t: type t); 0: every type
};
// a block's learned shortlist (k_sl_select): its candidates, most probable first, and the tx types worth a try
struct SlCand {
    uint8_t c[8];      // (mode, delta) candidate codes
    uint16_t txMask;   // tx types (bit t) the analysis and the closed loop try beyond DCT_DCT; 0: every type
    uint8_t n;         // candidates; 0: the block falls back to the full search (top probability below conf)
    uint8_t pad[5];
};
struct Leaf { uint8_t bsize, x4, y4, pad; };
struct SbCount { uint32_t nBlocks, nTxb, nCoeffs, pad; };

struct __align__(16) FrameDesc {
    int W, H, MiCols, MiRows, sbCols, sbRows, ssx, ssy, bd, qidx, qctx;
    int tileCols, tileRows;
    int tileColStart[65], tileRowStart[65];   // mi units, [n] = MiCols / MiRows
    const uint8_t *src[3];                    // sample (0, 0); samples of the bit depth
    int spitch[3];                            // in samples
    uint8_t *rec[3];
    int rpitch[3];
    uint8_t *mYMode, *cLvl[3], *cDc[3];
    BlockRes *blk;
    uint32_t nRec;                            // analysis records (all shapes)
    SlCand *slCand;                           // learned shortlist of the scored records (compact order); null: none
    int slIdx[22];                            // first compact index of each scored shape, -1 for the others
    int slRdK;                                // RD candidates of a block with a learned shortlist
    int rdK;                                  // RD candidates of every other block (1 .. 4; the plain form: 4)
    int txKeep;                               // 0, or the tx types (best analysis cost first) a block's txMask keeps
    uint32_t shOff[22];
    int shNbx[22], shNby[22];
    long long lam, sqlam;                     // lambda, sqrt(lambda) in 1/256
    int dcQ, acQ;
    Leaf *leaves;                             // [nSb * 256]
    uint16_t *nLeaves;                        // [nSb]
    av1g_block *oBlocks;                      // [nSb * 256]
    uint16_t *oBlockTxb;                      // [nSb * 256] first txb (SB-local) of each block
    av1g_txb *oTxb;                           // [nSb * SB_MAX_TXB] (coeff_off SB-local)
    int16_t *oCoeffs;                         // [nSb * SB_MAX_COEF]
    SbCount *sbCount;                         // [nSb]
    const uint32_t *sbOrder;                  // [nSb] SBs sorted by wavefront step (tile-local c + 2 r)
    uint8_t *ordmap;                          // [nSb * 256] leaf index covering each luma 4x4 unit of an SB (255: none)
    uint16_t *leafTxb, *leafCoef;             // [nSb * 256] first tx block / coefficient (SB-local) of each leaf
    int *leafDone;                            // [nSb * 256] 1 once the leaf's luma (reconstruction, maps) is written, 2 once all is
    uint32_t *leafStart;                      // [nSb] first position of each SB's leaves in the wavefront order
    uint32_t *leafTotal;                      // [1] leaves of the image
    int *queue;                               // [4] [2]: next free entry of revList
    // the closed loop's ready queue, shared by every image of a batch: 1 + (image << 32 | sb << 8 | leaf) in the order
    // leaves became ready (0: slot not written yet); rq[0] next slot to take, rq[1] next slot to write
    unsigned long long *readyQ;
    int *rq;
    uint32_t readyCap;                        // positions of readyQ
    int img;                                  // the image's tag in the ready queue: its index in the descriptor array
                                              // (low 16 bits) and, in a serving session, the generation of its slot
    int *leafDoneCnt;                         // serving: leaves of the image finished (null in a batch)
    volatile int *doneFlag;                   // serving: host-mapped word of the image's slot, set to img once its last
                                              // leaf is done (null in a batch)
    int *depCnt;                              // [nSb * 256] luma dependencies of each leaf not yet published
    int *revCnt, *revFill;                    // [nSb * 256] dependents of each leaf; entries written so far
    uint32_t *revOff;                         // [nSb * 256] first entry of each leaf's dependents in revList
    uint32_t *revList;                        // [nSb * REV_PER_SB] dependents (sb << 8 | leaf), grouped per leaf
    int *err;                                 // [1] error status (0 = ok), shared by the images of a batch
    unsigned long long *leafTrace;            // [leaves * 4] optional (debug): claimed / ready / luma done / done (ns)
    // pack output (DecisionRecord arrays in decode order) and per-SB offsets
    uint32_t *sbDecodeOrder;                  // [nSb] SBs in decode order (tiles raster, SB raster inside a tile)
    uint32_t *offBlk, *offTxb;                // [nSb + 1] exclusive prefix sums in decode order
    uint64_t *offCoef;                        // [nSb + 1]
    av1g_block *recBlocks;
    uint32_t *recBlockTxb;
    av1g_txb *recTxb;
    int16_t *recCoeffs;
    // the closed loop's wait budgets (is_set_wait_limits): spins on a leaf flag, globaltimer ns on a ready-queue slot
    long long readyWaitNs;
    int waitIters;
    int poison;                               // fill shared memory with a pattern at kernel start (is_set_poison)
};

// error codes written to FrameDesc::err by the kernels
constexpr int KERR_WAIT_LEAF = 2;    // a leaf dependency wait of the closed loop ran out of its iteration budget
constexpr int KERR_CAPACITY = 3;     // per-SB output slots exceeded

}  // namespace is
