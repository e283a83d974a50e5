// is_api.cu - host orchestration of the B200 intra search and its C ABI (include/is_api.h).
//
// One encode = one stream-ordered sequence (the reference's GpEncoder::encode, encoder/src/pipeline.cpp:323-1180):
//   upload / pad   the caller's planes into the padded workspace planes (cudaMemcpy2DAsync + k_pad)
//   analysis       k_analysis: one CTA per SB, every shape and position
//   dp             k_dp: one thread per SB
//   closed loop    k_recon: persistent cooperative wavefront (one CTA per SM)
//   pack           k_pack_scan + k_pack: DecisionRecord arrays in decode order
// The workspace is one device allocation per handle, grown when a larger image arrives and reused otherwise.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "is_api.h"
#include "av1g/dsp.h"
#include "is_dev.cuh"
#include "is_frame.cuh"
#include "is_units.cuh"
#include "is_tiny.cuh"
#include "is_dp.cuh"
#include "is_sched.cuh"
#include "is_learn.cuh"

using namespace is;

namespace {

// ---------------------------------------------------------------------------------------------------------------
// fixed-point tables (the same definitions as the reference's gp_init_tables, k_misc.cu:505-621, in 1/256 bit)
// ---------------------------------------------------------------------------------------------------------------
struct HostTables {
    std::vector<uint16_t> cost[4];
    int avgY[13];
    int avgPart[5][10];
    int avgSkip0;
};

int bits_fx(double p) { return (int)llround(-std::log2(p) * 256.0); }

template <typename Arr>
void cost_of_field(const av1g_cdfs &c, const Arr &field, uint16_t *out) {
    typedef typename std::remove_reference<Arr>::type T;
    constexpr size_t L = std::extent<T, std::rank<T>::value - 1>::value;   // symbols + 1 (adaptation counter)
    const uint16_t *p = reinterpret_cast<const uint16_t *>(&field);
    const size_t base = (size_t)(p - reinterpret_cast<const uint16_t *>(&c));
    for (size_t b = 0; b < sizeof(T) / 2; b += L)
        for (size_t s = 0; s + 1 < L; s++) {
            const double lo = s ? p[b + s - 1] : 0.0, hi = p[b + s];
            out[base + b + s] = (uint16_t)bits_fx(std::max((hi - lo) / 32768.0, 1.0 / 32768.0));
        }
}

const HostTables &host_tables() {
    static HostTables T;
    static std::once_flag once;
    std::call_once(once, [] {
        const int qrep[4] = {20, 60, 120, 255};   // a base_q_idx of each coefficient-CDF q-context
        for (int qc = 0; qc < 4; qc++) {
            av1g_cdfs c;
            av1g_cdfs_init(&c, qrep[qc]);
            T.cost[qc].assign(NCDF, 0);
            uint16_t *o = T.cost[qc].data();
            cost_of_field(c, c.y_mode, o); cost_of_field(c, c.uv_mode_cfl_not_allowed, o); cost_of_field(c, c.uv_mode_cfl_allowed, o);
            cost_of_field(c, c.angle_delta, o); cost_of_field(c, c.partition_w8, o); cost_of_field(c, c.partition_w16, o);
            cost_of_field(c, c.partition_w32, o); cost_of_field(c, c.partition_w64, o); cost_of_field(c, c.tx_8x8, o);
            cost_of_field(c, c.tx_16x16, o); cost_of_field(c, c.tx_32x32, o); cost_of_field(c, c.tx_64x64, o);
            cost_of_field(c, c.skip, o); cost_of_field(c, c.filter_intra_mode, o); cost_of_field(c, c.filter_intra, o);
            cost_of_field(c, c.intra_tx_set1, o); cost_of_field(c, c.intra_tx_set2, o); cost_of_field(c, c.cfl_sign, o);
            cost_of_field(c, c.cfl_alpha, o); cost_of_field(c, c.txb_skip, o); cost_of_field(c, c.eob_pt_16, o);
            cost_of_field(c, c.eob_pt_32, o); cost_of_field(c, c.eob_pt_64, o); cost_of_field(c, c.eob_pt_128, o);
            cost_of_field(c, c.eob_pt_256, o); cost_of_field(c, c.eob_pt_512, o); cost_of_field(c, c.eob_pt_1024, o);
            cost_of_field(c, c.eob_extra, o); cost_of_field(c, c.dc_sign, o); cost_of_field(c, c.coeff_base_eob, o);
            cost_of_field(c, c.coeff_base, o); cost_of_field(c, c.coeff_br, o);
            if (qc) continue;
            for (int m = 0; m < 13; m++) {   // y_mode averaged over its 5 x 5 contexts
                double p = 0;
                for (int a = 0; a < 5; a++)
                    for (int l = 0; l < 5; l++) p += (c.y_mode[a][l][m] - (m ? c.y_mode[a][l][m - 1] : 0)) / 32768.0;
                T.avgY[m] = bits_fx(std::max(p / 25.0, 1e-6));
            }
            for (int b = 0; b < 5; b++)
                for (int p = 0; p < 10; p++) T.avgPart[b][p] = 20 * 256;
            for (int bsl = 1; bsl <= 4; bsl++) {   // partition averaged over its 4 contexts
                const int N = bsl == 1 ? 4 : 10;
                for (int p = 0; p < N; p++) {
                    double pr = 0;
                    for (int ctx = 0; ctx < 4; ctx++) {
                        const uint16_t *cd = bsl == 1 ? c.partition_w8[ctx] : bsl == 2 ? c.partition_w16[ctx]
                                           : bsl == 3 ? c.partition_w32[ctx] : c.partition_w64[ctx];
                        pr += (cd[p] - (p ? cd[p - 1] : 0)) / 32768.0;
                    }
                    T.avgPart[bsl][p] = bits_fx(std::max(pr / 4.0, 1e-6));
                }
            }
            double ps = 0;
            for (int ctx = 0; ctx < 3; ctx++) ps += c.skip[ctx][0] / 32768.0;
            T.avgSkip0 = bits_fx(ps / 3.0);
        }
    });
    return T;
}

// libaom-style lambda (the reference's gp_lambda, dev_common.cuh:99-107), fixed point 1/256
void lambda_fx(int qidx, int bd, long long *lam, long long *sq) {
    const int q = AV1G_T(Dc_Qlookup)[(bd - 8) >> 1][std::min(255, std::max(0, qidx))];
    double rd = (double)q * q * (3.3 + 0.0015 * q);
    int w = ((255 - qidx) * 3) / 4;
    w = w < 0 ? 0 : w > 72 ? 72 : w;
    rd = rd * (128 + w) / 128.0;
    const double l = rd / 2048.0;
    *lam = llround(l * 256.0);
    *sq = llround(std::sqrt(l) * 256.0);
}

// spec 5.9.15 tile_info with uniform spacing at the minimum legal tiling (the reference's compute_tiles,
// av1core/src/encoder.cpp:56-92): returns cols, rows and the starts in mi units
int tile_log2(int blk, int target) { int k = 0; while ((blk << k) < target) k++; return k; }
void min_tiles(int W, int H, std::vector<int> &cs, std::vector<int> &rs) {
    const int MiCols = 2 * ((W + 7) >> 3), MiRows = 2 * ((H + 7) >> 3);
    const int sbCols = (MiCols + 15) >> 4, sbRows = (MiRows + 15) >> 4;
    const int maxTileWidthSb = 4096 >> 6, maxTileAreaSb = (4096 * 2304) >> 12;
    const int minLog2TileCols = tile_log2(maxTileWidthSb, sbCols);
    const int maxLog2TileRows = tile_log2(1, std::min(sbRows, 64));
    const int minLog2Tiles = std::max(minLog2TileCols, tile_log2(maxTileAreaSb, sbRows * sbCols));
    const int colsLog2 = minLog2TileCols;
    const int tileWidthSb = (sbCols + (1 << colsLog2) - 1) >> colsLog2;
    cs.clear();
    for (int s = 0; s < sbCols; s += tileWidthSb) cs.push_back(s << 4);
    cs.push_back(MiCols);
    int rowsLog2 = std::max(minLog2Tiles - colsLog2, 0);
    for (;; rowsLog2++) {
        const int tileHeightSb = (sbRows + (1 << rowsLog2) - 1) >> rowsLog2;
        if (tileWidthSb * tileHeightSb <= maxTileAreaSb || rowsLog2 >= maxLog2TileRows) {
            rs.clear();
            for (int s = 0; s < sbRows; s += tileHeightSb) rs.push_back(s << 4);
            rs.push_back(MiRows);
            return;
        }
    }
}

// analysis task lists of one SB: (bsize, x4, y4) for every shape, largest area first; big = shapes with a 64 side
// the task list of an analysis kernel (an_task<LIST>): 0 the shapes up to 32 a side from 8x16 / 16x8 up, 1 the shapes
// with a 64-sample side (the six smallest, 4x4, 4x8, 8x4, 8x8, 4x16 and 16x4, have the per-thread kernels)
std::vector<uint8_t> an_tasks(int list) {
    std::vector<int> shapes;
    for (int s = 0; s < AV1G_BLOCK_INVALID; s++) {
        if (s >= 13 && s <= 15) continue;
        const bool b = AV1G_T(Num_4x4_Blocks_Wide)[s] == 16 || AV1G_T(Num_4x4_Blocks_High)[s] == 16;
        const bool small = s == AV1G_BLOCK_4X4 || s == AV1G_BLOCK_4X8 || s == AV1G_BLOCK_8X4 || s == AV1G_BLOCK_8X8 || s == AV1G_BLOCK_4X16 ||
                           s == AV1G_BLOCK_16X4;
        if (!small && b == (list == 1)) shapes.push_back(s);
    }
    std::stable_sort(shapes.begin(), shapes.end(), [](int a, int b) {
        return AV1G_T(Num_4x4_Blocks_Wide)[a] * AV1G_T(Num_4x4_Blocks_High)[a] > AV1G_T(Num_4x4_Blocks_Wide)[b] * AV1G_T(Num_4x4_Blocks_High)[b];
    });
    std::vector<uint8_t> t;
    for (int s : shapes) {
        const int w4 = AV1G_T(Num_4x4_Blocks_Wide)[s], h4 = AV1G_T(Num_4x4_Blocks_High)[s];
        for (int y = 0; y < 16; y += h4)
            for (int x = 0; x < 16; x += w4) { t.push_back((uint8_t)s); t.push_back((uint8_t)x); t.push_back((uint8_t)y); }
    }
    return t;
}

// pad kernel: replicate the last visible column / row of a plane over the padded area (right, then bottom)
template <typename Px>
__global__ void k_pad(Px *plane, int pitch, int vw, int vh, int pw, int ph) {
    const int y = blockIdx.y;
    if (y < vh) {
        const Px v = plane[(size_t)y * pitch + vw - 1];
        for (int x = vw + threadIdx.x; x < pw; x += blockDim.x) plane[(size_t)y * pitch + x] = v;
    } else if (y < ph) {   // below the picture: the last visible row, itself extended by its last sample
        const Px *s = plane + (size_t)(vh - 1) * pitch;
        for (int x = threadIdx.x; x < pw; x += blockDim.x) plane[(size_t)y * pitch + x] = s[min(x, vw - 1)];
    }
}

}  // namespace

// ---------------------------------------------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------------------------------------------
struct is_handle {
    is_params p;
    int device = 0, nSm = 0;
    cudaStream_t own = nullptr;
    std::string err;
    // workspace
    void *arena = nullptr;
    size_t arenaBytes = 0;
    FrameDesc F;                 // the descriptor (device pointers), passed by value to every kernel
    int nSb = 0;
    size_t smemRcG[4] = {0, 0, 0, 0};       // the closed loop per format group (fmt_group)
    int rcGridG[4] = {0, 0, 0, 0};
    int rcWarpsG[4] = {0, 0, 0, 0};         // its warps per CTA
    int reconWarps = 0;                     // warps per CTA the closed loop uses (0: all; is_set_closed_loop_warps)
    // last result
    bool have = false;
    uint32_t nBlocks = 0, nTxb = 0;
    uint64_t nCoeffs = 0;
    int qidx = 0;
    is_times times;
    bool trace = false;
    unsigned long long *traceBuf = nullptr;
    size_t traceCap = 0;
    cudaEvent_t ev[6];
    void *hostSmall = nullptr;   // pinned 64 bytes (unused by the batch path; kept for the test entry points)
    // ---- batch state: every encode is a batch (a single image is a batch of one); F / nSb / qidx above mirror
    //      image 0 of the last batch ----
    int bN = 0;
    std::vector<FrameDesc> bF;
    std::vector<int> bNsb, bQ;
    std::vector<uint32_t> bNb, bNt;
    std::vector<uint64_t> bNc;
    size_t bSlots = 0;                      // ready-queue slots (sum over images of SBs x 256)
    size_t bQBytes = 0;                     // bytes of the ready queues (all groups)
    FrameDesc *dFs = nullptr;               // the descriptors in device memory (for the closed loop)
    FrameDesc *hFs = nullptr;               // pinned staging of the descriptors
    size_t hFsCap = 0;
    uint32_t *hOrd = nullptr;               // pinned staging of every image's wavefront and decode orders
    size_t hOrdCap = 0;
    uint32_t *hCnt = nullptr;               // pinned readback: per image n_blocks, n_txb, n_coeffs (2 words), + err
    size_t hCntCap = 0;
    unsigned long long *bReadyQ = nullptr;  // the ready queues, one per format group of the batch (fmt_group order)
    int *bRq = nullptr, *bErr = nullptr;    // [2 g, 2 g + 1]: group g's head / tail
    std::vector<int> bBd, bC444;            // per image (batch order)
    std::vector<int> bPos;                  // per image: its position in the device descriptor array (groups in order)
    int bGrpStart[5] = {0, 0, 0, 0, 0};     // group g's descriptors: [bGrpStart[g], bGrpStart[g + 1])
    // multi-stream front end (upload, analysis, DP, dataflow graph of each image) and CUDA graph replay
    cudaStream_t aux[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t evFork = nullptr, evJoin[4] = {nullptr, nullptr, nullptr, nullptr};
    int frontStreams = 1;                   // 1, 2 or 4 (is_autotune_batch chooses)
    int reconCtas = 0;                      // CTAs of the closed loop (0: one per SM); fewer leave SMs to other streams
    bool useGraph = false;
    // error paths: the closed loop's wait budgets, the workspace budget, poison mode
    int waitIters = LEAF_WAIT_ITERS;
    long long readyWaitNs = READY_WAIT_NS;
    uint64_t wsLimit = 0;                   // 0: no limit
    bool poison = false;
    size_t bNeed = 0;                       // bytes of the arena the last batch uses
    // non-learned pruning (is_set_search_options): RD candidates per block, tx types the closed loop keeps per block
    int rdK = K_TOP, txKeep = 0;
    // learned shortlist (is_set_shortlist_model): the parameters (fp32) and their bf16 copies, the selection rule
    bool slOn = false;
    float *slParams = nullptr;
    SlNet slNet{};
    __nv_bfloat16 *slZ[4] = {nullptr, nullptr, nullptr, nullptr}, *slH[4] = {nullptr, nullptr, nullptr, nullptr};   // chunk buffers
    float *slS[4] = {nullptr, nullptr, nullptr, nullptr};                                                         // per front stream
    SlSel slSel{0.9f, 0.f, 0.9f, 8, 2};
    int slRdK = 4;
    int slVersion = 0;
    std::string graphKey;
    cudaGraphExec_t graphExec = nullptr;
    struct ServeSession *serve = nullptr;   // an open serving session (is_serve_open), or null
    // entropy coding of the records (is_encode_obu): device scratch, pinned result staging, timing events
    void *entScratch = nullptr;
    size_t entBytes = 0;
    void *pfScratch = nullptr;              // post-filters (is_postfilter)
    size_t pfBytes = 0;
    std::vector<av1g_frame_params> bPf;     // per image: the frame parameters of its post-filters (is_encode_obu codes them)
    std::vector<char> bPfSet;
    cudaEvent_t entEv[2] = {nullptr, nullptr};
    int setErr(int code, const char *fmt, ...) {
        char b[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(b, sizeof b, fmt, ap);
        va_end(ap);
        err = b;
        return code;
    }
};

#define IS_CK(call)                                                                                 \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return h->setErr(e_ == cudaErrorMemoryAllocation ? IS_ERR_OOM : IS_ERR_CUDA, \
                                                "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

namespace {

// per device: whether the tables are uploaded (a failed upload is retried by the next call)
std::mutex g_upload_mu;
bool g_uploaded[64];

// the search's tables into every compilation unit's copies on device dev (once per device)
int upload_tables(int dev) {
    if (dev < 0 || dev >= 64) return (int)cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_upload_mu);
    if (g_uploaded[dev]) return 0;
    {
        const HostTables &T = host_tables();
        TableBlob B;
        B.cost.assign((size_t)4 * NCDF, 0);
        for (int q = 0; q < 4; q++) memcpy(B.cost.data() + (size_t)q * NCDF, T.cost[q].data(), NCDF * 2);
        memcpy(B.avgY, T.avgY, sizeof B.avgY);
        memcpy(B.avgPart, T.avgPart, sizeof B.avgPart);
        B.avgSkip0 = T.avgSkip0;
        // scans packed per (tx size, class), one copy of each distinct table
        std::vector<const uint16_t *> seen;
        std::vector<uint16_t> seenOff;
        for (int t = 0; t < 19; t++) {
            const int n = std::min<int>(AV1G_T(Tx_Width)[t], 32) * std::min<int>(AV1G_T(Tx_Height)[t], 32);
            const bool oneD = AV1G_T(Tx_Width)[t] <= 16 && AV1G_T(Tx_Height)[t] <= 16;
            const int types[3] = {AV1G_DCT_DCT, AV1G_H_DCT, AV1G_V_DCT};   // class 2D, HORIZ, VERT
            for (int c = 0; c < 3; c++) {
                const uint16_t *sc = av1g_get_scan(t, (c == 0 || !oneD) ? AV1G_DCT_DCT : types[c]);
                size_t k = 0;
                while (k < seen.size() && seen[k] != sc) k++;
                if (k == seen.size()) {
                    seen.push_back(sc);
                    seenOff.push_back((uint16_t)B.scanPack.size());
                    B.scanPack.insert(B.scanPack.end(), sc, sc + n);
                }
                B.scanOff[t][c] = seenOff[k];
            }
        }
        cudaError_t e = cudaSuccess;
        // the compile-time copies of spec tables in the per-thread search must equal av1core's
        for (int c = 0; c < 3 && e == cudaSuccess; c++) {
            for (int k = 0; k < 5; k++)
                if (sig_ref(c, k, 0) != AV1G_T(Sig_Ref_Diff_Offset)[c][k][0] || sig_ref(c, k, 1) != AV1G_T(Sig_Ref_Diff_Offset)[c][k][1]) e = cudaErrorInvalidValue;
            for (int k = 0; k < 3; k++)
                if (mag_ref(c, k, 0) != AV1G_T(Mag_Ref_Offset_With_Tx_Class)[c][k][0] || mag_ref(c, k, 1) != AV1G_T(Mag_Ref_Offset_With_Tx_Class)[c][k][1])
                    e = cudaErrorInvalidValue;
        }
        if (kDr23 != AV1G_T(Dr_Intra_Derivative)[23] || kDr45 != AV1G_T(Dr_Intra_Derivative)[45] || kDr67 != AV1G_T(Dr_Intra_Derivative)[67]) e = cudaErrorInvalidValue;
        // the analysis task lists and where each shape's tasks start in them
        B.anTask = an_tasks(0);
        B.anTaskBig = an_tasks(1);
        auto starts = [](const std::vector<uint8_t> &t, int n, std::vector<int> &out) {
            out.assign(n + 1, 0);
            int k = 0;
            for (size_t i = 0; i < t.size() / 3; i++)
                if (i == 0 || t[3 * i] != t[3 * i - 3]) { if (k < n) out[k] = (int)i; k++; }
            out[n] = (int)(t.size() / 3);
            return k == n;
        };
        std::vector<int> stBig;
        bool okShapes = starts(B.anTask, AN_SHAPES, B.anShapeStart) && starts(B.anTaskBig, ANB_SHAPES, stBig);
        {   // the 64-sided list's groups: every shape of at least 2048 samples together, then one group per shape
            B.anShapeStartBig.assign(ANB_GROUPS + 1, 0);
            int g = 0;
            B.anShapeStartBig[g++] = 0;
            for (int k = 1; k < ANB_SHAPES && okShapes; k++) {
                const int bs = B.anTaskBig[3 * stBig[k]];
                if (AV1G_T(Num_4x4_Blocks_Wide)[bs] * AV1G_T(Num_4x4_Blocks_High)[bs] < 128) {
                    if (g >= ANB_GROUPS) okShapes = false;
                    else B.anShapeStartBig[g++] = stBig[k];
                }
            }
            if (g != ANB_GROUPS) okShapes = false;
            else B.anShapeStartBig[g] = stBig[ANB_SHAPES];
        }
        if (!okShapes) e = cudaErrorInvalidValue;
        if (e == cudaSuccess) e = upload_common(B);
        if (e == cudaSuccess) e = an_upload<8, 0>(B);
        if (e == cudaSuccess) e = an_upload<8, 1>(B);
        if (e == cudaSuccess) e = an_upload<10, 0>(B);
        if (e == cudaSuccess) e = an_upload<10, 1>(B);
        if (e == cudaSuccess) e = rc_upload<8, 1>(B);
        if (e == cudaSuccess) e = rc_upload<8, 0>(B);
        if (e == cudaSuccess) e = rc_upload<10, 1>(B);
        if (e == cudaSuccess) e = rc_upload<10, 0>(B);
        if (e == cudaSuccess) e = ent_upload(B);
        g_uploaded[dev] = e == cudaSuccess;
        return e == cudaSuccess ? 0 : (int)e;
    }
}

size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// format groups of a batch, each with its own closed-loop instance and ready queue: 0 8-bit 4:2:0, 1 8-bit 4:4:4,
// 2 10-bit 4:2:0, 3 10-bit 4:4:4
int fmt_group(int bd, int c444) { return (bd == 10 ? 2 : 0) + (c444 ? 1 : 0); }
// lay out the workspace for an image of W x H (bit depth bd, 4:4:4 or 4:2:0); returns bytes needed, fills F's
// pointers if base != 0.  Plane pitches are in samples (a multiple of 16).
size_t layout(int W, int H, int bd, int c444, uint8_t *base, FrameDesc &F, int &nSb) {
    F.W = W; F.H = H;
    F.MiCols = 2 * ((W + 7) >> 3); F.MiRows = 2 * ((H + 7) >> 3);
    F.sbCols = (F.MiCols + 15) >> 4; F.sbRows = (F.MiRows + 15) >> 4;
    F.ssx = F.ssy = c444 ? 0 : 1; F.bd = bd;
    nSb = F.sbCols * F.sbRows;
    const size_t px = bd > 8 ? 2 : 1;
    size_t at = 0;
    auto take = [&](size_t bytes) -> uint8_t * { uint8_t *p = base ? base + at : nullptr; at += align256(bytes); return p; };
    for (int p = 0; p < 3; p++) {
        const int ss = p ? F.ssx : 0;
        const int pw = (((F.sbCols + 1) * 64) >> ss) + SRC_MARGIN_X, ph = ((F.sbRows * 64) >> ss) + SRC_MARGIN_Y;
        const int pitch = (pw + 15) & ~15;
        uint8_t *s = take((size_t)pitch * ph * px), *r = take((size_t)pitch * ph * px);
        F.spitch[p] = F.rpitch[p] = pitch;
        F.src[p] = s ? s + ((size_t)SRC_MARGIN_Y * pitch + SRC_MARGIN_X) * px : nullptr;
        F.rec[p] = r ? r + ((size_t)SRC_MARGIN_Y * pitch + SRC_MARGIN_X) * px : nullptr;
    }
    F.mYMode = take((size_t)F.MiCols * F.MiRows);
    for (int p = 0; p < 3; p++) {
        const size_t n = (size_t)(F.MiCols >> (p ? F.ssx : 0)) * (F.MiRows >> (p ? F.ssy : 0));
        F.cLvl[p] = take(n);
        F.cDc[p] = take(n);
    }
    uint32_t off = 0;
    for (int s = 0; s < 22; s++) {
        F.shNbx[s] = F.shNby[s] = 0;
        F.shOff[s] = off;
        if (s >= AV1G_BLOCK_INVALID || (s >= 13 && s <= 15)) continue;
        const int w = 4 * AV1G_T(Num_4x4_Blocks_Wide)[s], h = 4 * AV1G_T(Num_4x4_Blocks_High)[s];
        F.shNbx[s] = (F.MiCols * 4 + w - 1) / w;
        F.shNby[s] = (F.MiRows * 4 + h - 1) / h;
        off += (uint32_t)(F.shNbx[s] * F.shNby[s]);
    }
    F.blk = (BlockRes *)take((size_t)off * sizeof(BlockRes));
    F.nRec = off;
    const uint32_t nScored = sl_scored_layout(F, F.slIdx);
    F.slCand = (SlCand *)take((size_t)nScored * sizeof(SlCand));   // kept only while a shortlist model is set (prepare_batch)
    F.leaves = (Leaf *)take((size_t)nSb * SB_MAX_LEAVES * sizeof(Leaf));
    F.nLeaves = (uint16_t *)take((size_t)nSb * 2);
    F.oBlocks = (av1g_block *)take((size_t)nSb * SB_MAX_LEAVES * sizeof(av1g_block));
    F.oBlockTxb = (uint16_t *)take((size_t)nSb * SB_MAX_LEAVES * 2);
    F.oTxb = (av1g_txb *)take((size_t)nSb * SB_MAX_TXB * sizeof(av1g_txb));
    F.oCoeffs = (int16_t *)take((size_t)nSb * SB_MAX_COEF * 2);
    F.sbCount = (SbCount *)take((size_t)nSb * sizeof(SbCount));
    F.sbOrder = (const uint32_t *)take((size_t)nSb * 4);
    F.ordmap = take((size_t)nSb * 256);
    F.leafTxb = (uint16_t *)take((size_t)nSb * SB_MAX_LEAVES * 2);
    F.leafCoef = (uint16_t *)take((size_t)nSb * SB_MAX_LEAVES * 2);
    F.leafDone = (int *)take((size_t)nSb * SB_MAX_LEAVES * 4);
    F.leafStart = (uint32_t *)take((size_t)nSb * 4);
    F.leafTotal = (uint32_t *)take(4);
    F.leafTrace = nullptr;   // set per encode when tracing is on (is_set_trace)
    F.queue = (int *)take(16);
    F.depCnt = (int *)take((size_t)nSb * SB_MAX_LEAVES * 4);
    F.revCnt = (int *)take((size_t)nSb * SB_MAX_LEAVES * 4);
    F.revFill = (int *)take((size_t)nSb * SB_MAX_LEAVES * 4);
    F.revOff = (uint32_t *)take((size_t)nSb * SB_MAX_LEAVES * 4);
    F.revList = (uint32_t *)take((size_t)nSb * REV_PER_SB * 4);
    F.err = (int *)take(4);
    F.sbDecodeOrder = (uint32_t *)take((size_t)nSb * 4);
    F.offBlk = (uint32_t *)take((size_t)(nSb + 1) * 4);
    F.offTxb = (uint32_t *)take((size_t)(nSb + 1) * 4);
    F.offCoef = (uint64_t *)take((size_t)(nSb + 1) * 8);
    F.recBlocks = (av1g_block *)take((size_t)nSb * SB_MAX_LEAVES * sizeof(av1g_block));
    F.recBlockTxb = (uint32_t *)take(((size_t)nSb * SB_MAX_LEAVES + 1) * 4);
    F.recTxb = (av1g_txb *)take((size_t)nSb * SB_MAX_TXB * sizeof(av1g_txb));
    F.recCoeffs = (int16_t *)take((size_t)nSb * SB_MAX_COEF * 2);
    return at;
}

}  // namespace

// ---------------------------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------------------------
extern "C" {

int is_create(const is_params *p, is_handle **out) {
    if (!p || !out) return IS_ERR_INVALID;
    if ((p->bit_depth != 8 && p->bit_depth != 10) || (p->chroma_444 != 0 && p->chroma_444 != 1)) return IS_ERR_INVALID;
    is_handle *h = new is_handle();
    h->p = *p;
    h->device = p->device;
    auto fail = [&](int rc) { is_destroy(h); *out = nullptr; return rc; };
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(IS_ERR_CUDA);
    if (upload_tables(h->device)) return fail(IS_ERR_CUDA);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, h->device) != cudaSuccess) return fail(IS_ERR_CUDA);
    h->nSm = prop.multiProcessorCount;
    if (an_setup<8, 0>() != cudaSuccess || an_setup<8, 1>() != cudaSuccess || an_setup<10, 0>() != cudaSuccess || an_setup<10, 1>() != cudaSuccess)
        return fail(IS_ERR_CUDA);
    for (int g = 0; g < 4; g++) {   // the closed loop of each format group: shared memory, warps, its cooperative grid
        int per = 0, nw = 0;
        size_t *sm = &h->smemRcG[g];
        const cudaError_t e = g == 0 ? rc_setup<8, 1>(sm, &per, &nw) : g == 1 ? rc_setup<8, 0>(sm, &per, &nw)
                            : g == 2 ? rc_setup<10, 1>(sm, &per, &nw) : rc_setup<10, 0>(sm, &per, &nw);
        if (e != cudaSuccess || per < 1) return fail(IS_ERR_CUDA);
        h->rcGridG[g] = per * h->nSm;
        h->rcWarpsG[g] = nw;
    }
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) return fail(IS_ERR_CUDA);
    for (auto &e : h->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return fail(IS_ERR_CUDA);
    if (cudaMallocHost(&h->hostSmall, 64) != cudaSuccess) return fail(IS_ERR_OOM);
    for (int k = 0; k < 4; k++) {
        if (cudaStreamCreateWithFlags(&h->aux[k], cudaStreamNonBlocking) != cudaSuccess) return fail(IS_ERR_CUDA);
        if (cudaEventCreateWithFlags(&h->evJoin[k], cudaEventDisableTiming) != cudaSuccess) return fail(IS_ERR_CUDA);
    }
    if (cudaEventCreateWithFlags(&h->evFork, cudaEventDisableTiming) != cudaSuccess) return fail(IS_ERR_CUDA);
    memset(&h->times, 0, sizeof h->times);
    *out = h;
    return IS_OK;
}

void is_destroy(is_handle *h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->serve) is_serve_close(h);
    if (h->own) cudaStreamSynchronize(h->own);
    if (h->arena) cudaFree(h->arena);
    if (h->entScratch) cudaFree(h->entScratch);
    if (h->pfScratch) cudaFree(h->pfScratch);
    for (auto &e : h->entEv)
        if (e) cudaEventDestroy(e);
    for (auto &e : h->ev)
        if (e) cudaEventDestroy(e);
    if (h->own) cudaStreamDestroy(h->own);
    if (h->hostSmall) cudaFreeHost(h->hostSmall);
    if (h->traceBuf) cudaFree(h->traceBuf);
    if (h->graphExec) cudaGraphExecDestroy(h->graphExec);
    for (int k = 0; k < 4; k++) {
        if (h->aux[k]) { cudaStreamSynchronize(h->aux[k]); cudaStreamDestroy(h->aux[k]); }
        if (h->evJoin[k]) cudaEventDestroy(h->evJoin[k]);
    }
    if (h->evFork) cudaEventDestroy(h->evFork);
    if (h->hFs) cudaFreeHost(h->hFs);
    void *sl[] = {h->slParams, h->slNet.c1, h->slNet.c2, h->slNet.c3, h->slNet.f1, h->slNet.f2, h->slZ[0], h->slZ[1], h->slZ[2], h->slZ[3],
                  h->slH[0], h->slH[1], h->slH[2], h->slH[3], h->slS[0], h->slS[1], h->slS[2], h->slS[3]};
    for (void *p : sl)
        if (p) cudaFree(p);
    if (h->hOrd) cudaFreeHost(h->hOrd);
    if (h->hCnt) cudaFreeHost(h->hCnt);
    delete h;
}

const char *is_last_error(const is_handle *h) { return h ? h->err.c_str() : "null handle"; }

// the wavefront order (SBs by tile-local step c + 2 r) and the decode order (tiles raster, SBs raster) of an image
static void sb_orders(const FrameDesc &F, const std::vector<int> &cs, const std::vector<int> &rs, uint32_t *order, uint32_t *dec) {
    struct J { uint32_t sb; int step; };
    std::vector<J> js;
    size_t nd = 0;
    for (int tr = 0; tr < F.tileRows; tr++)
        for (int tc = 0; tc < F.tileCols; tc++) {
            const int r0 = rs[tr] >> 4, r1 = (rs[tr + 1] + 15) >> 4, c0 = cs[tc] >> 4, c1 = (cs[tc + 1] + 15) >> 4;
            for (int r = r0; r < r1; r++)
                for (int c = c0; c < c1; c++) {
                    js.push_back(J{(uint32_t)(r * F.sbCols + c), (c - c0) + 2 * (r - r0)});
                    dec[nd++] = (uint32_t)(r * F.sbCols + c);
                }
        }
    std::stable_sort(js.begin(), js.end(), [](const J &a, const J &b) { return a.step < b.step; });
    for (size_t i = 0; i < js.size(); i++) order[i] = js[i].sb;
}

extern "C++" {
template <typename T> static int grow_pinned(is_handle *h, T **p, size_t *cap, size_t n) {
    if (n <= *cap) return IS_OK;
    if (*p) cudaFreeHost(*p);
    *p = nullptr;
    *cap = 0;
    IS_CK(cudaMallocHost((void **)p, n * sizeof(T)));
    *cap = n;
    return IS_OK;
}
}

// the format of a frame: its own (bit_depth 8 / 10) or the handle's (bit_depth 0)
static void frame_format(const is_handle *h, const is_frame *f, int *bd, int *c444) {
    *bd = f->bit_depth ? f->bit_depth : h->p.bit_depth;
    *c444 = f->bit_depth ? f->chroma_444 : h->p.chroma_444;
}

// Lay out a batch: every image's workspace, then the ready queues (one per format group), their counters, the error
// word and the device copy of the descriptors (grouped by format), in one arena; the descriptors and SB orders in
// pinned staging.
static int prepare_batch(is_handle *h, const is_frame *fr, int n) {
    if (!fr || n < 1 || n > 4096) return h->setErr(IS_ERR_INVALID, "invalid batch (%d images)", n);
    h->bBd.assign(n, 8);
    h->bC444.assign(n, 0);
    for (int i = 0; i < n; i++) {
        const is_frame *f = fr + i;
        if (f->width < 1 || f->height < 1 || f->width > 16384 || f->height > 16384 || f->qindex < 1 || f->qindex > 255)
            return h->setErr(IS_ERR_INVALID, "invalid frame %d (size %dx%d, qindex %d)", i, f->width, f->height, f->qindex);
        frame_format(h, f, &h->bBd[i], &h->bC444[i]);
        if ((h->bBd[i] != 8 && h->bBd[i] != 10) || (h->bC444[i] != 0 && h->bC444[i] != 1))
            return h->setErr(IS_ERR_INVALID, "invalid frame %d format (bit depth %d, chroma_444 %d)", i, h->bBd[i], h->bC444[i]);
        for (int p = 0; p < 3; p++) {   // every plane present, its rows at least as long as the plane is wide
            const int ss = (p && !h->bC444[i]) ? 1 : 0, vw = (f->width + ss) >> ss;
            if (!f->planes[p] || f->pitch[p] < vw)
                return h->setErr(IS_ERR_INVALID, "invalid frame %d plane %d (pointer %p, pitch %d for width %d)", i, p, f->planes[p], f->pitch[p], vw);
        }
    }
    std::vector<size_t> off(n + 1);
    std::vector<int> nsb(n), grp(n);
    size_t at = 0, slotsG[4] = {0, 0, 0, 0}, nOrd = 0;
    h->bPos.assign(n, 0);
    int cnt[4] = {0, 0, 0, 0};
    for (int i = 0; i < n; i++) cnt[grp[i] = fmt_group(h->bBd[i], h->bC444[i])]++;
    h->bGrpStart[0] = 0;
    for (int g = 0; g < 4; g++) h->bGrpStart[g + 1] = h->bGrpStart[g] + cnt[g];
    int fill[4] = {0, 0, 0, 0};
    for (int i = 0; i < n; i++) h->bPos[i] = h->bGrpStart[grp[i]] + fill[grp[i]]++;
    for (int i = 0; i < n; i++) {
        FrameDesc F;
        memset(&F, 0, sizeof F);
        off[i] = at;
        at += layout(fr[i].width, fr[i].height, h->bBd[i], h->bC444[i], nullptr, F, nsb[i]);
        slotsG[grp[i]] += (size_t)nsb[i] * SB_MAX_LEAVES;
        nOrd += 2 * (size_t)nsb[i];
    }
    const size_t slots = slotsG[0] + slotsG[1] + slotsG[2] + slotsG[3];
    size_t offQG[4];
    offQG[0] = at;
    for (int g = 1; g < 4; g++) offQG[g] = offQG[g - 1] + align256(slotsG[g - 1] * 8);
    const size_t offQ = at, offRq = offQG[3] + align256(slotsG[3] * 8), offErr = offRq + 256, offFs = offErr + 256;
    const size_t need = offFs + align256((size_t)n * sizeof(FrameDesc));
    if (h->wsLimit && need > h->wsLimit)
        return h->setErr(IS_ERR_OOM, "the batch needs %zu bytes of workspace, over the handle's limit of %llu", need,
                         (unsigned long long)h->wsLimit);
    h->bNeed = need;
    if (need > h->arenaBytes) {
        if (h->arena) { cudaStreamSynchronize(h->own); cudaDeviceSynchronize(); cudaFree(h->arena); h->arena = nullptr; h->arenaBytes = 0; }
        IS_CK(cudaMalloc(&h->arena, need));
        h->arenaBytes = need;
    }
    uint8_t *base = (uint8_t *)h->arena;
    h->bReadyQ = (unsigned long long *)(base + offQ);
    h->bRq = (int *)(base + offRq);
    h->bErr = (int *)(base + offErr);
    h->dFs = (FrameDesc *)(base + offFs);
    h->bSlots = slots;
    h->bQBytes = offRq - offQ;
    int rc = grow_pinned(h, &h->hFs, &h->hFsCap, (size_t)n);
    if (!rc) rc = grow_pinned(h, &h->hOrd, &h->hOrdCap, nOrd);
    if (!rc) rc = grow_pinned(h, &h->hCnt, &h->hCntCap, (size_t)n * 4 + 4);
    if (rc) return rc;
    if (h->trace) {
        const size_t needT = std::max(std::max(slotsG[0], slotsG[1]), std::max(slotsG[2], slotsG[3])) * TRACE_STAMPS;
        if (needT > h->traceCap) {
            if (h->traceBuf) cudaFree(h->traceBuf);
            h->traceBuf = nullptr;
            h->traceCap = 0;
            IS_CK(cudaMalloc(&h->traceBuf, needT * 8));
            h->traceCap = needT;
        }
    }
    h->bF.assign(n, FrameDesc());
    h->bPf.assign(n, av1g_frame_params());
    h->bPfSet.assign(n, 0);
    h->bNsb = nsb;
    h->bQ.assign(n, 0);
    h->bNb.assign(n, 0);
    h->bNt.assign(n, 0);
    h->bNc.assign(n, 0);
    size_t o = 0;
    for (int i = 0; i < n; i++) {
        const is_frame *f = fr + i;
        FrameDesc &F = h->bF[i];
        memset(&F, 0, sizeof F);
        int ns = 0;
        layout(f->width, f->height, h->bBd[i], h->bC444[i], base + off[i], F, ns);
        std::vector<int> cs, rs;
        min_tiles(f->width, f->height, cs, rs);
        if (cs.size() > 65 || rs.size() > 65) return h->setErr(IS_ERR_INVALID, "too many tiles");
        F.tileCols = (int)cs.size() - 1; F.tileRows = (int)rs.size() - 1;
        for (size_t k = 0; k < cs.size(); k++) F.tileColStart[k] = cs[k];
        for (size_t k = 0; k < rs.size(); k++) F.tileRowStart[k] = rs[k];
        F.qidx = f->qindex;
        F.qctx = av1g_coeff_cdf_q_ctx(f->qindex);
        const int bd = h->bBd[i], g10 = bd == 10;
        lambda_fx(f->qindex, bd, &F.lam, &F.sqlam);
        F.dcQ = AV1G_T(Dc_Qlookup)[g10][f->qindex];
        F.acQ = AV1G_T(Ac_Qlookup)[g10][f->qindex];
        // the image's format group: its ready queue and counters; img indexes the group's descriptors
        F.readyQ = (unsigned long long *)(base + offQG[grp[i]]);
        F.rq = h->bRq + 2 * grp[i];
        F.readyCap = (uint32_t)slotsG[grp[i]];
        F.err = h->bErr;
        F.img = h->bPos[i] - h->bGrpStart[grp[i]];
        F.leafTrace = (h->trace && i == 0 && F.img == 0) ? h->traceBuf : nullptr;   // image 0, when its group's first
        if (!h->slOn) F.slCand = nullptr;
        F.slRdK = h->slOn ? h->slRdK : 4;
        F.rdK = h->rdK;
        F.txKeep = h->txKeep;
        F.waitIters = h->waitIters;
        F.readyWaitNs = h->readyWaitNs;
        F.poison = h->poison ? 1 : 0;
        sb_orders(F, cs, rs, h->hOrd + o, h->hOrd + o + ns);
        o += 2 * (size_t)ns;
        h->hFs[h->bPos[i]] = F;
        h->bQ[i] = f->qindex;
    }
    h->bN = n;
    return IS_OK;
}

// The closed loop's working warps per CTA for a launch over n images of format group g: the handle's setting, else 4
// for one image (its loop is bound by its dependency chain, and fewer warps leave the SM a larger L1) and all the shared
// memory holds for a batch; and that launch's dynamic shared memory.
static int rc_warps_for(const is_handle *h, int g, int n) {
    const int all = h->rcWarpsG[g];
    return h->reconWarps > 0 ? std::min(h->reconWarps, all) : n == 1 ? std::min(4, all) : all;
}
static size_t rc_launch_smem(int g, int warps) {
    return g == 0 ? rc_smem<8, 1>(warps) : g == 1 ? rc_smem<8, 0>(warps) : g == 2 ? rc_smem<10, 1>(warps) : rc_smem<10, 0>(warps);
}

// The front end of one image on stream s: its planes into the padded workspace, the learned shortlist of every scored
// block (with a model set: the fused inference kernel), the analysis, the DP, the leaf maps and the dataflow graph,
// whose first ready leaves go to the image's ready queue.  ev1 / ev2 (optional) are recorded after the upload and after
// the analysis.
static int front_end(is_handle *h, const FrameDesc &F, const is_frame *f, int nSb, bool fromHost, cudaStream_t s, int k, cudaEvent_t ev1,
                     cudaEvent_t ev2) {
    const size_t px = F.bd > 8 ? 2 : 1;
    for (int p = 0; p < 3; p++) {
        const int ss = p ? F.ssx : 0;
        const int vw = (f->width + ss) >> ss, vh = (f->height + ss) >> ss;
        uint8_t *dst = const_cast<uint8_t *>(F.src[p]);
        IS_CK(cudaMemcpy2DAsync(dst, F.spitch[p] * px, f->planes[p], (size_t)f->pitch[p] * px, vw * px, vh,
                                fromHost ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
        const int pw = ((F.sbCols + 1) * 64) >> ss, ph = (F.sbRows * 64) >> ss;
        if (px == 1) k_pad<uint8_t><<<dim3(1, ph), 128, 0, s>>>(dst, F.spitch[p], vw, vh, pw, ph);
        else k_pad<uint16_t><<<dim3(1, ph), 128, 0, s>>>((uint16_t *)dst, F.spitch[p], vw, vh, pw, ph);
    }
    if (ev1) IS_CK(cudaEventRecord(ev1, s));
    if (h->slOn && F.slCand)   // the learned shortlist of every scored block (chunk buffers k)
        IS_CK(sl_infer_image(F, h->slNet, h->slSel, h->nSm, h->slZ[k], h->slH[k], h->slS[k], F.slCand, nullptr, s));
    IS_CK((F.bd == 8 ? an_launch<8, 0>(F, nSb, s) : an_launch<10, 0>(F, nSb, s)));
    IS_CK((F.bd == 8 ? an_launch<8, 1>(F, nSb, s) : an_launch<10, 1>(F, nSb, s)));
    IS_CK(cudaGetLastError());
    if (ev2) IS_CK(cudaEventRecord(ev2, s));
    k_dp<<<(nSb + DP_WARPS - 1) / DP_WARPS, DP_WARPS * 32, 0, s>>>(F, nSb);
    k_leaf_prep<<<nSb, 256, 0, s>>>(F, nSb);
    k_leaf_queue_scan<<<1, 1024, 0, s>>>(F, nSb);
    k_leaf_deps<0><<<nSb, 256, 0, s>>>(F, nSb);
    k_leaf_deps<1><<<nSb, 256, 0, s>>>(F, nSb);
    k_leaf_deps<2><<<nSb, 256, 0, s>>>(F, nSb);
    k_leaf_deps<3><<<nSb, 256, 0, s>>>(F, nSb);
    IS_CK(cudaGetLastError());
    return IS_OK;
}

// the launch sequence of a prepared batch on stream st (capturable: no host synchronisation inside)
static int launch_batch(is_handle *h, cudaStream_t st, const is_frame *fr, int n, bool fromHost, bool events) {
    if (events) IS_CK(cudaEventRecord(h->ev[0], st));
    // poison mode: every byte of the batch's workspace starts as garbage (whatever the launch sequence does not write
    // before it reads would change the results)
    if (h->poison) IS_CK(cudaMemsetAsync(h->arena, 0xA5, h->bNeed, st));
    IS_CK(cudaMemcpyAsync(h->dFs, h->hFs, (size_t)n * sizeof(FrameDesc), cudaMemcpyHostToDevice, st));
    {
        size_t o = 0;
        for (int i = 0; i < n; i++) {
            const FrameDesc &F = h->bF[i];
            const int ns = h->bNsb[i];
            IS_CK(cudaMemcpyAsync((void *)F.sbOrder, h->hOrd + o, (size_t)ns * 4, cudaMemcpyHostToDevice, st));
            IS_CK(cudaMemcpyAsync(F.sbDecodeOrder, h->hOrd + o + ns, (size_t)ns * 4, cudaMemcpyHostToDevice, st));
            IS_CK(cudaMemsetAsync(F.queue, 0, 16, st));
            o += 2 * (size_t)ns;
        }
    }
    IS_CK(cudaMemsetAsync(h->bReadyQ, 0, h->bQBytes, st));
    IS_CK(cudaMemsetAsync(h->bRq, 0, 32, st));
    IS_CK(cudaMemsetAsync(h->bErr, 0, 4, st));
    // front end of each image: planes, analysis, DP, leaf maps and the dataflow graph (its initial ready leaves go to
    // the shared queue); images spread over frontStreams streams
    const int K = n > 1 ? std::max(1, std::min(h->frontStreams, 4)) : 1;
    if (K > 1) {
        IS_CK(cudaEventRecord(h->evFork, st));
        for (int k = 0; k < K; k++) IS_CK(cudaStreamWaitEvent(h->aux[k], h->evFork, 0));
    }
    for (int i = 0; i < n; i++) {
        cudaStream_t s = K > 1 ? h->aux[i % K] : st;
        const int rc = front_end(h, h->bF[i], fr + i, h->bNsb[i], fromHost, s, K > 1 ? i % K : 0, (events && n == 1) ? h->ev[1] : nullptr,
                                 (events && n == 1) ? h->ev[2] : nullptr);
        if (rc) return rc;
    }
    if (K > 1) {
        for (int k = 0; k < K; k++) {
            IS_CK(cudaEventRecord(h->evJoin[k], h->aux[k]));
            IS_CK(cudaStreamWaitEvent(st, h->evJoin[k], 0));
        }
    }
    if (events) IS_CK(cudaEventRecord(h->ev[3], st));
    // the closed loop of every image of a format group at once (one cooperative launch per group)
    for (int g = 0; g < 4; g++) {
        const int gn = h->bGrpStart[g + 1] - h->bGrpStart[g];
        if (gn == 0) continue;
        const int grid = h->reconCtas > 0 && h->reconCtas < h->rcGridG[g] ? h->reconCtas : h->rcGridG[g];
        const FrameDesc *fs = h->dFs + h->bGrpStart[g];
        const FrameDesc &F0 = h->hFs[h->bGrpStart[g]];   // the group's first image: its queue, counters and trace
        RcCtl ctl;
        ctl.rq = F0.rq;
        ctl.readyQ = F0.readyQ;
        ctl.err = F0.err;
        ctl.serving = 0;
        ctl.cap = F0.readyCap;
        ctl.readyWaitNs = (unsigned long long)h->readyWaitNs;
        ctl.trace = F0.leafTrace;
        ctl.poison = h->poison ? 1 : 0;
        ctl.warps = rc_warps_for(h, g, gn);
        const size_t sm = rc_launch_smem(g, ctl.warps);
        IS_CK((g == 0 ? rc_launch<8, 1>(fs, gn, ctl, grid, sm, st) : g == 1 ? rc_launch<8, 0>(fs, gn, ctl, grid, sm, st)
               : g == 2 ? rc_launch<10, 1>(fs, gn, ctl, grid, sm, st) : rc_launch<10, 0>(fs, gn, ctl, grid, sm, st)));
    }
    if (events) IS_CK(cudaEventRecord(h->ev[4], st));
    for (int i = 0; i < n; i++) {
        const FrameDesc &F = h->bF[i];
        k_pack_scan<<<1, 1024, 0, st>>>(F, h->bNsb[i]);
        k_pack<<<h->bNsb[i], 256, 0, st>>>(F, h->bNsb[i]);
    }
    IS_CK(cudaGetLastError());
    if (events) IS_CK(cudaEventRecord(h->ev[5], st));
    // per image counts, then the error word
    for (int i = 0; i < n; i++) {
        const FrameDesc &F = h->bF[i];
        const int nSb = h->bNsb[i];
        IS_CK(cudaMemcpyAsync(h->hCnt + 4 * i, F.offBlk + nSb, 4, cudaMemcpyDeviceToHost, st));
        IS_CK(cudaMemcpyAsync(h->hCnt + 4 * i + 1, F.offTxb + nSb, 4, cudaMemcpyDeviceToHost, st));
        IS_CK(cudaMemcpyAsync(h->hCnt + 4 * i + 2, F.offCoef + nSb, 8, cudaMemcpyDeviceToHost, st));
    }
    IS_CK(cudaMemcpyAsync(h->hCnt + 4 * n, h->bErr, 4, cudaMemcpyDeviceToHost, st));
    return IS_OK;
}

static std::string batch_key(const is_handle *h, const is_frame *fr, int n, bool fromHost) {
    std::string k;
    char b[160];
    snprintf(b, sizeof b, "%p|%d|%d|%d|%d|%d|%d|%d|%lld|%d|%d|%d|", h->arena, n, (int)fromHost, h->frontStreams, h->reconCtas,
             h->slOn ? h->slVersion : -1, (int)h->poison, h->waitIters, h->readyWaitNs, h->rdK, h->txKeep, h->reconWarps);
    k += b;
    for (int i = 0; i < n; i++) {
        snprintf(b, sizeof b, "%d,%d,%d,%d,%d,%p,%p,%p,%d,%d,%d;", fr[i].width, fr[i].height, fr[i].qindex, fr[i].bit_depth, fr[i].chroma_444,
                 fr[i].planes[0], fr[i].planes[1], fr[i].planes[2], fr[i].pitch[0], fr[i].pitch[1], fr[i].pitch[2]);
        k += b;
    }
    return k;
}

static int run_batch(is_handle *h, cudaStream_t st, const is_frame *fr, int n, bool fromHost) {
    h->have = false;
    int rc = prepare_batch(h, fr, n);
    if (rc) return rc;
    if (h->useGraph) {
        // one CUDA graph per batch signature (sizes, qindex, plane addresses, workspace): captured once, then replayed
        const std::string key = batch_key(h, fr, n, fromHost);
        if (key != h->graphKey || !h->graphExec) {
            if (h->graphExec) { cudaGraphExecDestroy(h->graphExec); h->graphExec = nullptr; }
            h->graphKey.clear();
            IS_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            const int lrc = launch_batch(h, st, fr, n, fromHost, false);
            cudaGraph_t g = nullptr;
            const cudaError_t ec = cudaStreamEndCapture(st, &g);
            if (lrc) { if (g) cudaGraphDestroy(g); return lrc; }
            IS_CK(ec);
            const cudaError_t ei = cudaGraphInstantiate(&h->graphExec, g, 0);
            cudaGraphDestroy(g);
            IS_CK(ei);
            h->graphKey = key;
        }
        IS_CK(cudaEventRecord(h->ev[0], st));   // (events recorded inside a graph cannot be timed: the whole batch)
        IS_CK(cudaGraphLaunch(h->graphExec, st));
        IS_CK(cudaEventRecord(h->ev[5], st));
    } else {
        rc = launch_batch(h, st, fr, n, fromHost, true);
        if (rc) return rc;
    }
    IS_CK(cudaStreamSynchronize(st));
    if (h->hCnt[4 * n]) return h->setErr(IS_ERR_TIMEOUT, "closed loop reported error %u (dependency wait budget exhausted)", h->hCnt[4 * n]);
    for (int i = 0; i < n; i++) {
        h->bNb[i] = h->hCnt[4 * i];
        h->bNt[i] = h->hCnt[4 * i + 1];
        memcpy(&h->bNc[i], h->hCnt + 4 * i + 2, 8);
    }
    float ms[6] = {0, 0, 0, 0, 0, 0};
    memset(&h->times, 0, sizeof h->times);
    if (h->useGraph) {
        IS_CK(cudaEventElapsedTime(&ms[3], h->ev[0], h->ev[5]));
    } else {
        IS_CK(cudaEventElapsedTime(&ms[3], h->ev[0], h->ev[3]));
        IS_CK(cudaEventElapsedTime(&ms[4], h->ev[3], h->ev[4]));
        IS_CK(cudaEventElapsedTime(&ms[5], h->ev[4], h->ev[5]));
    }
    if (n == 1 && !h->useGraph) {   // single image on one stream: the front end split into its stages
        float up = 0, an = 0, dp = 0;
        IS_CK(cudaEventElapsedTime(&up, h->ev[0], h->ev[1]));
        IS_CK(cudaEventElapsedTime(&an, h->ev[1], h->ev[2]));
        IS_CK(cudaEventElapsedTime(&dp, h->ev[2], h->ev[3]));
        h->times.upload = up; h->times.analysis = an; h->times.dp = dp;
    } else {
        h->times.analysis = ms[3];   // upload + analysis + DP + dataflow graph of every image
    }
    h->times.recon = ms[4];
    h->times.pack = ms[5];
    h->times.total = ms[3] + ms[4] + ms[5];
    h->times.sbs = 0;
    h->times.blocks = 0;
    for (int i = 0; i < n; i++) { h->times.sbs += (uint32_t)h->bNsb[i]; h->times.blocks += h->bNb[i]; }
    // image 0 mirrored into the single-image fields
    h->F = h->bF[0];
    h->nSb = h->bNsb[0];
    h->qidx = h->bQ[0];
    h->nBlocks = h->bNb[0];
    h->nTxb = h->bNt[0];
    h->nCoeffs = h->bNc[0];
    h->have = true;
    return IS_OK;
}

int is_workspace_bytes_format(int width, int height, int bit_depth, int chroma_444, uint64_t *bytes) {
    if (width < 1 || height < 1 || width > 16384 || height > 16384 || !bytes || (bit_depth != 8 && bit_depth != 10) ||
        (chroma_444 != 0 && chroma_444 != 1))
        return IS_ERR_INVALID;
    FrameDesc F;
    memset(&F, 0, sizeof F);
    int nSb = 0;
    const size_t ws = layout(width, height, bit_depth, chroma_444, nullptr, F, nSb);
    *bytes = ws + align256((size_t)nSb * SB_MAX_LEAVES * 8) + align256(sizeof(FrameDesc)) + 768;
    return IS_OK;
}

int is_workspace_bytes(int width, int height, uint64_t *bytes) { return is_workspace_bytes_format(width, height, 8, 0, bytes); }

int is_encode_device(is_handle *h, const is_frame *f, void *stream) {
    if (!h) return IS_ERR_INVALID;
    IS_CK(cudaSetDevice(h->device));
    return run_batch(h, stream ? (cudaStream_t)stream : h->own, f, 1, false);
}

int is_encode_host(is_handle *h, const is_frame *f, void *stream) {
    if (!h) return IS_ERR_INVALID;
    IS_CK(cudaSetDevice(h->device));
    return run_batch(h, stream ? (cudaStream_t)stream : h->own, f, 1, true);
}

int is_encode_batch(is_handle *h, const is_frame *frames, int n, int from_host, void *stream) {
    if (!h) return IS_ERR_INVALID;
    IS_CK(cudaSetDevice(h->device));
    return run_batch(h, stream ? (cudaStream_t)stream : h->own, frames, n, from_host != 0);
}

int is_set_batch_options(is_handle *h, int use_graph, int front_streams, int recon_ctas) {
    if (!h || front_streams < 0 || front_streams > 4 || front_streams == 3 || recon_ctas < 0) return IS_ERR_INVALID;
    h->useGraph = use_graph != 0;
    if (front_streams) h->frontStreams = front_streams;
    h->reconCtas = recon_ctas;
    if (!h->useGraph && h->graphExec) { cudaGraphExecDestroy(h->graphExec); h->graphExec = nullptr; h->graphKey.clear(); }
    return IS_OK;
}

int is_set_wait_limits(is_handle *h, int leaf_wait_iters, long long ready_wait_ns) {
    if (!h || leaf_wait_iters < 0 || leaf_wait_iters > (1 << 24) || ready_wait_ns < 0 || ready_wait_ns > 60000000000ll) return IS_ERR_INVALID;
    h->waitIters = leaf_wait_iters ? leaf_wait_iters : LEAF_WAIT_ITERS;
    h->readyWaitNs = ready_wait_ns ? ready_wait_ns : READY_WAIT_NS;
    return IS_OK;
}

int is_set_workspace_limit(is_handle *h, uint64_t bytes) {
    if (!h) return IS_ERR_INVALID;
    h->wsLimit = bytes;
    return IS_OK;
}

int is_set_poison(is_handle *h, int on) {
    if (!h) return IS_ERR_INVALID;
    h->poison = on != 0;
    return IS_OK;
}

int is_set_search_options(is_handle *h, int rd_k, int tx_keep) {
    if (!h) return IS_ERR_INVALID;
    if (rd_k < 0 || rd_k > K_TOP || tx_keep < 0 || tx_keep > 3) return h->setErr(IS_ERR_INVALID, "invalid search options");
    h->rdK = rd_k ? rd_k : K_TOP;
    h->txKeep = tx_keep;
    return IS_OK;
}

int is_set_shortlist_model(is_handle *h, const float *params, float tau, int max_cand, float conf, int rd_k, float tx_tau, int max_tx) {
    if (!h) return IS_ERR_INVALID;
    IS_CK(cudaSetDevice(h->device));
    if (!params) { h->slOn = false; return IS_OK; }
    if (max_cand < 1 || max_cand > 8 || !(tau > 0.f) || tau > 1.f || !(conf >= 0.f) || conf > 1.f || rd_k < 1 || rd_k > 4 ||
        max_tx < 0 || max_tx > 16 || !(tx_tau > 0.f) || tx_tau > 1.f)
        return h->setErr(IS_ERR_INVALID, "invalid shortlist model");
    IS_CK(cudaStreamSynchronize(h->own));
    if (!h->slParams) {
        IS_CK(cudaMalloc(&h->slParams, SL_NPARAM * 4));
        IS_CK(cudaMalloc(&h->slNet.c1, SL_C1 * SL_K1P * 2));
        IS_CK(cudaMalloc(&h->slNet.c2, SL_C2 * SL_K2 * 2));
        IS_CK(cudaMalloc(&h->slNet.c3, SL_C3 * SL_K3 * 2));
        IS_CK(cudaMalloc(&h->slNet.f1, SL_HID * SL_Z * 2));
        IS_CK(cudaMalloc(&h->slNet.f2, SL_OUT * SL_HID * 2));
        h->slNet.b1 = h->slParams + SLP_C1B; h->slNet.b2 = h->slParams + SLP_C2B; h->slNet.b3 = h->slParams + SLP_C3B;
        h->slNet.bf1 = h->slParams + SLP_F1B; h->slNet.bf2 = h->slParams + SLP_F2B;
        for (int k = 0; k < 4; k++) {
            IS_CK(cudaMalloc(&h->slZ[k], (size_t)SL_CHUNK * SL_Z * 2));
            IS_CK(cudaMalloc(&h->slH[k], (size_t)SL_CHUNK * SL_HID * 2));
            IS_CK(cudaMalloc(&h->slS[k], (size_t)SL_CHUNK * SL_OUT * 4));
        }
        IS_CK(cudaFuncSetAttribute(k_sl_conv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SlcSmem)));
    }
    IS_CK(cudaMemcpy(h->slParams, params, SL_NPARAM * 4, cudaMemcpyHostToDevice));
    k_sl_weights<<<(SL_HID * SL_Z + 255) / 256, 256, 0, h->own>>>(h->slParams, h->slNet);
    IS_CK(cudaGetLastError());
    IS_CK(cudaStreamSynchronize(h->own));
    h->slSel = SlSel{tau, conf, tx_tau, max_cand, max_tx};
    h->slRdK = rd_k;
    h->slOn = true;
    h->slVersion++;
    return IS_OK;
}

int is_set_closed_loop_warps(is_handle *h, int warps) {
    if (!h || warps < 0 || warps > RC_MAX_WARPS) return IS_ERR_INVALID;
    h->reconWarps = warps;
    return IS_OK;
}

int is_autotune_batch(is_handle *h, const is_frame *frames, int n, int from_host, int *front_streams, int *recon_warps, float *ms) {
    if (!h || !frames || n < 1) return IS_ERR_INVALID;
    IS_CK(cudaSetDevice(h->device));
    const bool g = h->useGraph;
    h->useGraph = false;
    int best = 1, bestW = 0;
    float bestMs = 1e30f;
    const int cand[3] = {1, 2, 4}, wcand[3] = {4, 6, 0};   // front-end streams x closed-loop warps per CTA (0: all)
    for (int c = 0; c < 3; c++) {
        if (cand[c] > 1 && n < 2) break;
        for (int w = 0; w < 3; w++) {
            h->frontStreams = cand[c];
            h->reconWarps = wcand[w];
            float t = 0;
            for (int r = 0; r < 2; r++) {   // the second run is timed (the first warms the workspace)
                const int rc = run_batch(h, h->own, frames, n, from_host != 0);
                if (rc) { h->useGraph = g; return rc; }
                t = h->times.total;
            }
            if (t < bestMs) { bestMs = t; best = cand[c]; bestW = wcand[w]; }
        }
    }
    h->frontStreams = best;
    h->reconWarps = bestW;
    h->useGraph = g;
    if (front_streams) *front_streams = best;
    if (recon_warps) *recon_warps = bestW;
    if (ms) *ms = bestMs;
    return IS_OK;
}

int is_batch_counts(const is_handle *h, int i, uint32_t *nb, uint32_t *nt, uint64_t *nc) {
    if (!h || !h->have || i < 0 || i >= h->bN) return IS_ERR_STATE;
    if (nb) *nb = h->bNb[i];
    if (nt) *nt = h->bNt[i];
    if (nc) *nc = h->bNc[i];
    return IS_OK;
}

static void batch_fp(const is_handle *h, int i, av1g_frame_params *fp);

int is_batch_copy(is_handle *h, int i, av1g_frame_params *fp, av1g_block *blocks, uint32_t *block_txb, av1g_txb *txb, int16_t *coeffs,
                  void *recon[3], const int32_t recon_pitch[3]) {
    if (!h || !h->have || i < 0 || i >= h->bN) return IS_ERR_STATE;
    IS_CK(cudaSetDevice(h->device));
    const FrameDesc &F = h->bF[i];
    cudaStream_t st = h->own;
    if (fp) batch_fp(h, i, fp);
    if (blocks) IS_CK(cudaMemcpyAsync(blocks, F.recBlocks, (size_t)h->bNb[i] * sizeof(av1g_block), cudaMemcpyDeviceToHost, st));
    if (block_txb) IS_CK(cudaMemcpyAsync(block_txb, F.recBlockTxb, ((size_t)h->bNb[i] + 1) * 4, cudaMemcpyDeviceToHost, st));
    if (txb) IS_CK(cudaMemcpyAsync(txb, F.recTxb, (size_t)h->bNt[i] * sizeof(av1g_txb), cudaMemcpyDeviceToHost, st));
    if (coeffs) IS_CK(cudaMemcpyAsync(coeffs, F.recCoeffs, (size_t)h->bNc[i] * 2, cudaMemcpyDeviceToHost, st));
    const size_t px = F.bd > 8 ? 2 : 1;
    for (int p = 0; p < 3; p++) {
        if (!recon || !recon[p]) continue;
        const int ss = p ? F.ssx : 0;
        const int vw = (F.W + ss) >> ss, vh = (F.H + ss) >> ss;
        IS_CK(cudaMemcpy2DAsync(recon[p], (recon_pitch ? recon_pitch[p] : vw) * px, F.rec[p], F.rpitch[p] * px, vw * px, vh,
                                cudaMemcpyDeviceToHost, st));
    }
    IS_CK(cudaStreamSynchronize(st));
    return IS_OK;
}

int is_record_counts(const is_handle *h, uint32_t *nb, uint32_t *nt, uint64_t *nc) { return is_batch_counts(h, 0, nb, nt, nc); }

int is_record_copy(is_handle *h, av1g_frame_params *fp, av1g_block *blocks, uint32_t *block_txb, av1g_txb *txb, int16_t *coeffs,
                   void *recon[3], const int32_t recon_pitch[3]) {
    return is_batch_copy(h, 0, fp, blocks, block_txb, txb, coeffs, recon, recon_pitch);
}

int is_record_device(const is_handle *h, const av1g_block **blocks, const uint32_t **block_txb, const av1g_txb **txb, const int16_t **coeffs) {
    if (!h || !h->have) return IS_ERR_STATE;
    if (blocks) *blocks = h->F.recBlocks;
    if (block_txb) *block_txb = h->F.recBlockTxb;
    if (txb) *txb = h->F.recTxb;
    if (coeffs) *coeffs = h->F.recCoeffs;
    return IS_OK;
}

// the frame parameters of image i of the last batch (as is_batch_copy writes them; after is_postfilter, its parameters)
static void batch_fp(const is_handle *h, int i, av1g_frame_params *fp) {
    const FrameDesc &F = h->bF[i];
    if (i < (int)h->bPfSet.size() && h->bPfSet[i]) { *fp = h->bPf[i]; return; }
    memset(fp, 0, sizeof *fp);
    fp->version = AV1G_DECISIONS_VERSION;
    fp->width = (uint32_t)F.W; fp->height = (uint32_t)F.H;
    fp->base_q_idx = (uint8_t)h->bQ[i];
    fp->tile_cols_log2 = -1; fp->tile_rows_log2 = -1;
    fp->qm_y = fp->qm_u = fp->qm_v = 15;
    fp->chroma_format = F.ssx ? AV1G_CHROMA_420 : AV1G_CHROMA_444;
    fp->bit_depth = (uint8_t)F.bd;
}

int is_entropy_scratch_bytes(const is_ent_frame *frames, int n, uint64_t cap, uint64_t *bytes) {
    if (!bytes) return IS_ERR_INVALID;
    size_t b = 0;
    const int rc = ent_scratch(frames, n, cap, &b, nullptr);
    if (rc == IS_OK) *bytes = b;
    return rc;
}

int is_entropy_batch(int device, const is_ent_frame *frames, int n, uint64_t cap, void *scratch, uint64_t scratchBytes, void *stream,
                     is_ent_out *out, uint32_t *frameTile0) {
    if (!out) return IS_ERR_INVALID;
    int nDev = 0;
    if (cudaGetDeviceCount(&nDev) != cudaSuccess || device < 0 || device >= nDev) return IS_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess || upload_tables(device)) return IS_ERR_CUDA;
    return ent_launch(frames, n, cap, scratch, (size_t)scratchBytes, (cudaStream_t)stream, out, frameTile0, nullptr);
}

int is_obu_assemble(const av1g_frame_params *fp, const uint8_t *payload, const uint64_t *off, uint32_t nTiles, uint8_t *out, uint64_t cap,
                    uint64_t *size) {
    if (!fp || !payload || !off || !size || !nTiles) return IS_ERR_INVALID;
    std::vector<uint8_t> o;
    const int rc = obu_assemble(*fp, payload, off, nTiles, o, nullptr);
    if (rc != IS_OK) return rc;
    *size = o.size();
    if (!out || cap < o.size()) return IS_ERR_TOO_LARGE;
    memcpy(out, o.data(), o.size());
    return IS_OK;
}

int is_encode_obu(is_handle *h, int first, int n, uint8_t *out, uint64_t cap, uint64_t *offsets, float *device_ms) {
    if (!h || !h->have || first < 0 || n < 1 || first + n > h->bN) return h ? h->setErr(IS_ERR_STATE, "no such images") : IS_ERR_STATE;
    if (!offsets) return h->setErr(IS_ERR_INVALID, "offsets missing");
    IS_CK(cudaSetDevice(h->device));
    std::vector<is_ent_frame> fr(n);
    for (int k = 0; k < n; k++) {
        const int i = first + k;
        const FrameDesc &F = h->bF[i];
        batch_fp(h, i, &fr[k].fp);
        fr[k].blocks = F.recBlocks; fr[k].block_txb = F.recBlockTxb; fr[k].txb = F.recTxb; fr[k].coeffs = F.recCoeffs;
        fr[k].n_blocks = h->bNb[i]; fr[k].n_txb = h->bNt[i];
    }
    for (auto &e : h->entEv)
        if (!e) IS_CK(cudaEventCreate(&e));
    uint64_t cap0 = 0;
    std::vector<uint8_t> head;
    is_ent_out eo;
    std::vector<uint32_t> t0(n + 1);
    for (int attempt = 0; attempt < 2; attempt++) {
        size_t need = 0;
        int rc = ent_scratch(fr.data(), n, cap0, &need, &h->err);
        if (rc != IS_OK) return rc;
        if (need > h->entBytes) {
            if (h->entScratch) IS_CK(cudaFree(h->entScratch));
            h->entScratch = nullptr;
            h->entBytes = 0;
            IS_CK(cudaMalloc(&h->entScratch, need));
            h->entBytes = need;
        }
        IS_CK(cudaEventRecord(h->entEv[0], h->own));
        rc = ent_launch(fr.data(), n, cap0, h->entScratch, h->entBytes, h->own, &eo, t0.data(), &h->err);
        if (rc != IS_OK) return rc;
        IS_CK(cudaEventRecord(h->entEv[1], h->own));
        head.resize(eo.result_bytes);
        IS_CK(cudaMemcpyAsync(head.data(), eo.result, eo.result_bytes, cudaMemcpyDeviceToHost, h->own));
        IS_CK(cudaStreamSynchronize(h->own));
        const is_ent_status *st = (const is_ent_status *)head.data();
        if (st->error == IS_ENT_ERR_SYMBOLS && attempt == 0) { cap0 = st->symbols; continue; }
        if (st->error) return h->setErr(IS_ERR_INVALID, "entropy coding failed: error bits %d (symbols %llu)", st->error,
                                        (unsigned long long)st->symbols);
        break;
    }
    if (device_ms) IS_CK(cudaEventElapsedTime(device_ms, h->entEv[0], h->entEv[1]));
    const is_ent_status *st = (const is_ent_status *)head.data();
    const uint64_t *toff = (const uint64_t *)(head.data() + sizeof(is_ent_status));
    std::vector<uint8_t> pay(st->bytes);
    if (st->bytes) IS_CK(cudaMemcpy(pay.data(), eo.payload, st->bytes, cudaMemcpyDeviceToHost));
    uint64_t pos = 0;
    std::vector<uint8_t> obu;
    bool fits = true;
    for (int k = 0; k < n; k++) {
        std::vector<uint64_t> rel;
        for (uint32_t t = t0[k]; t <= t0[k + 1]; t++) rel.push_back(toff[t] - toff[t0[k]]);
        const int rc = obu_assemble(fr[k].fp, pay.data() + toff[t0[k]], rel.data(), t0[k + 1] - t0[k], obu, &h->err);
        if (rc != IS_OK) return rc;
        offsets[k] = pos;
        if (out && pos + obu.size() <= cap) memcpy(out + pos, obu.data(), obu.size());
        else fits = false;
        pos += obu.size();
    }
    offsets[n] = pos;
    return fits ? IS_OK : h->setErr(IS_ERR_TOO_LARGE, "the OBU streams need %llu bytes", (unsigned long long)pos);
}

int is_postfilter(is_handle *h, int i, const av1g_frame_params *fp, const int8_t *sb_cdef, float *device_ms) {
    if (!h || !h->have || i < 0 || i >= h->bN) return h ? h->setErr(IS_ERR_STATE, "no such image") : IS_ERR_STATE;
    const FrameDesc &F = h->bF[i];
    if (!fp || fp->width != (uint32_t)F.W || fp->height != (uint32_t)F.H || fp->monochrome || fp->base_q_idx == 0 ||
        (fp->chroma_format == AV1G_CHROMA_444) != (F.ssx == 0) || (fp->bit_depth == 10) != (F.bd == 10))
        return h->setErr(IS_ERR_INVALID, "frame parameters do not describe image %d", i);
    bool ok = fp->loop_filter_sharpness <= 7 && fp->enable_cdef <= 1 && fp->cdef_damping_minus_3 <= 3 && fp->cdef_bits <= 3;
    for (int k = 0; k < 4; k++) ok = ok && fp->loop_filter_level[k] <= 63;
    ok = ok && (fp->loop_filter_level[0] || fp->loop_filter_level[1] || (!fp->loop_filter_level[2] && !fp->loop_filter_level[3]));
    for (int k = 0; k < 8; k++) {
        auto sec = [](int v) { return v == 0 || v == 1 || v == 2 || v == 4; };
        ok = ok && fp->cdef_y_pri[k] <= 15 && fp->cdef_uv_pri[k] <= 15 && sec(fp->cdef_y_sec[k]) && sec(fp->cdef_uv_sec[k]);
    }
    const size_t nSb = (size_t)F.sbCols * F.sbRows;
    if (fp->enable_cdef && sb_cdef)
        for (size_t k = 0; k < nSb; k++) ok = ok && sb_cdef[k] >= 0 && sb_cdef[k] < (1 << fp->cdef_bits);
    if (!ok) return h->setErr(IS_ERR_INVALID, "post-filter parameters out of range");
    IS_CK(cudaSetDevice(h->device));
    const size_t need = pf_scratch_bytes(F.W, F.H, F.bd, F.ssx ? 0 : 1);
    if (need > h->pfBytes) {
        if (h->pfScratch) IS_CK(cudaFree(h->pfScratch));
        h->pfScratch = nullptr;
        h->pfBytes = 0;
        IS_CK(cudaMalloc(&h->pfScratch, need));
        h->pfBytes = need;
    }
    for (auto &e : h->entEv)
        if (!e) IS_CK(cudaEventCreate(&e));
    std::vector<int8_t> zero;
    if (fp->enable_cdef && !sb_cdef) { zero.assign(nSb, 0); sb_cdef = zero.data(); }
    IS_CK(cudaEventRecord(h->entEv[0], h->own));
    const int rc = pf_launch(*fp, h->bF[i].recBlocks, h->bNb[i], fp->enable_cdef ? sb_cdef : nullptr, F.rec, F.rpitch, h->pfScratch,
                             h->pfBytes, h->own, &h->err);
    if (rc != IS_OK) return rc;
    IS_CK(cudaEventRecord(h->entEv[1], h->own));
    IS_CK(cudaStreamSynchronize(h->own));
    if (device_ms) IS_CK(cudaEventElapsedTime(device_ms, h->entEv[0], h->entEv[1]));
    // the record now carries the filters: the bitstream is_encode_obu writes signals them
    av1g_frame_params q;
    batch_fp(h, i, &q);
    memcpy(q.loop_filter_level, fp->loop_filter_level, sizeof q.loop_filter_level);
    q.loop_filter_sharpness = fp->loop_filter_sharpness;
    q.enable_cdef = fp->enable_cdef;
    q.cdef_damping_minus_3 = fp->cdef_damping_minus_3;
    q.cdef_bits = fp->cdef_bits;
    memcpy(q.cdef_y_pri, fp->cdef_y_pri, 8); memcpy(q.cdef_y_sec, fp->cdef_y_sec, 8);
    memcpy(q.cdef_uv_pri, fp->cdef_uv_pri, 8); memcpy(q.cdef_uv_sec, fp->cdef_uv_sec, 8);
    h->bPf[i] = q;
    h->bPfSet[i] = 1;
    return IS_OK;
}

int is_avif_mux(const av1g_frame_params *fp, const uint8_t *obu, uint64_t obu_size, uint8_t *out, uint64_t cap, uint64_t *size) {
    if (!fp || !obu || !obu_size || !size) return IS_ERR_INVALID;
    std::vector<uint8_t> o;
    const int rc = avif_write(*fp, obu, (size_t)obu_size, o, nullptr);
    if (rc != IS_OK) return rc;
    *size = o.size();
    if (!out || cap < o.size()) return IS_ERR_TOO_LARGE;
    memcpy(out, o.data(), o.size());
    return IS_OK;
}

int is_postfilter_from_q(int qindex, int bit_depth, av1g_frame_params *fp) {
    if (!fp || qindex < 1 || qindex > 255 || (bit_depth != 8 && bit_depth != 10)) return IS_ERR_INVALID;
    // libaom av1_pick_filter_level, LPF_PICK_FROM_Q, key frame: a linear fit of the level to the ac quantizer step
    const int64_t ac = AV1G_T(Ac_Qlookup)[(bit_depth - 8) >> 1][qindex];
    int g = bit_depth == 8 ? (int)((ac * 17563 - 421574 + (1 << 17)) >> 18) : (int)((ac * 20723 + 4060632 + (1 << 19)) >> 20) - 4;
    g = std::min(std::max(g, 0), 63);
    // the effective level of an intra block: + the intra reference delta (1) scaled by 1 << (level >> 5)
    const int lvl = g ? std::min(g + (1 << (g >> 5)), 63) : 0;
    for (int i = 0; i < 4; i++) fp->loop_filter_level[i] = (uint8_t)lvl;
    fp->loop_filter_sharpness = (uint8_t)(qindex <= 120 ? 7 : qindex <= 160 ? 1 : 0);
    fp->cdef_damping_minus_3 = (uint8_t)(qindex >> 6);
    return IS_OK;
}

int is_times_get(const is_handle *h, is_times *t) {
    if (!h || !t) return IS_ERR_INVALID;
    *t = h->times;
    return IS_OK;
}

}  // extern "C"

#include "is_serve.cuh"
#include "is_testapi.cuh"
#include "is_noalloc.cuh"
#include "is_learn_api.cuh"
