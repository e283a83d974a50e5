// oracle/plain_search.cpp - CPU oracle of the plain-form intra RD search.  TEST INFRASTRUCTURE ONLY: loaded by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the product.
//
// A scalar restatement, in exact integer / fixed-point arithmetic, of maddog107/av1gpu's per-superblock intra search
// with the plain-form configuration (GpConfig defaults, encoder/src/pipeline.cpp:41-76: K 4, Krecheck 2, tx-type search
// open and closed loop, angle deltas, CfL, uvK 2, all 19 shapes, all partitions, no pruning / shortlists / filter
// intra / palette / QM / delta-q / edge filter).  Stages, each citing the reference code it restates:
//   tables    cost of every CDF symbol, averaged mode / partition / skip bits     k_misc.cu:505-517, 574-621
//   lambda    libaom-style lambda from dc_q                                       dev_common.cuh:99-107
//   analysis  open loop, every shape and aligned position                         k_analysis.cuh:496-689
//   dp        partition DP per 64x64 + leaves in decode order                     k_dp.cuh:72-297
//   closed    SB wavefront, luma re-check + tx search, chroma + CfL               k_recon.cuh:822-1214, 1220-1686, 1692-1808
//   rate      exact coefficient rate with all in-block contexts                   dev_tx.cuh:48-165
// What this restatement changes, on purpose, relative to the reference (identically in the CUDA kernels):
//   - the forward transform is the integer transpose of the spec's inverse butterfly network (the reference inverts
//     the exact inverse numerically in float, dev_tx.cuh:171-243);
//   - distortion, rate and J are integers: D in 2^-16 pixel-SSE units, R in 1/256 bit, lambda in 1/256, J = D + lambda R;
//   - CfL alpha and the quantiser use exact integer rounding; ties go to the first candidate in evaluation order.
// Prediction, edges, CfL, dequantisation and the inverse transform are av1core's own dsp.h functions; the
// reconstruction is checked against av1g_encode() of the produced DecisionRecord.
#include "oracle.h"
#include "av1g/av1g.h"
#include "av1g/dsp.h"
#include "av1g/blockinfo.h"
#include "av1g/cdfctx.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <functional>
#include <thread>
#include <vector>

// av1core has the dequantiser per template bit depth only; a run-time variant for the oracle
static inline int32_t av1g_dequant_coef_bd(int32_t quant, int q, int den, int bd) {
    return bd == 10 ? av1g_dequant_coef<10>(quant, q, den) : av1g_dequant_coef<8>(quant, q, den);
}

namespace orc {

typedef int64_t i64;
static const i64 INF = (i64)1 << 60;
static const int FB = 3;          // fractional bits of the forward-transform coefficients
static const int NCDF = (int)(sizeof(av1g_cdfs) / 2);

// plain-form knobs (pipeline.cpp:41-76)
static const int K_TOP = 4, K_RECHECK = 2, UV_K = 2;
// experiment switch (orc_set_uv_open_loop; the plain form is 0): the chroma screening reads its edges from the SOURCE
// with the closed loop's availability, as the reference's open-loop chroma shortlist (k_leafprep.cu:1-30) does, so it
// could run before the closed loop; its operations are then counted as open-loop work
static int g_uvOpenLoop = 0;
// experiment switch (orc_set_edge_filter; the plain form is 0): directional predictions with the intra edge filter and
// upsampling (spec 7.11.2.11-12, enable_intra_edge_filter = 1), filter type 0 in the open-loop analysis (no neighbour
// modes yet, as the reference's analysis) and from the neighbours' modes in the closed loop
static int g_edgeFilter = 0;
static const int UV_OVERHEAD = 384;     // uvOverheadBits 1.5, in 1/256 bit

static inline i64 sat_add(i64 a, i64 b) { return (a >= INF || b >= INF) ? INF : std::min(a + b, INF); }

// ---------------------------------------------------------------------------------------------------------------
// cost tables (k_misc.cu:505-517 cost_field, 574-621 averages), in 1/256 bit
// ---------------------------------------------------------------------------------------------------------------
struct Tables {
    std::vector<uint16_t> cost[4];
    int avgY[13];
    int avgPart[5][10];
    int avgSkip0;
};
static av1g_cdfs g_layout;   // only its addresses: the uint16 offset of a CDF entry in av1g_cdfs
#define COFF(expr) ((int)((const uint16_t *)&(g_layout.expr) - (const uint16_t *)&g_layout))

static inline int bits_fx(double p) { return (int)llround(-std::log2(p) * 256.0); }

template <typename Arr>
static void cost_field(const av1g_cdfs &c, const Arr &field, uint16_t *out) {
    typedef typename std::remove_reference<Arr>::type T;
    constexpr size_t L = std::extent<T, std::rank<T>::value - 1>::value;
    const uint16_t *p = (const uint16_t *)&field;
    const size_t off = (size_t)(p - (const uint16_t *)&c);
    const size_t total = sizeof(T) / 2;
    for (size_t b = 0; b < total; b += L)
        for (size_t s = 0; s + 1 < L; s++) {
            const double lo = s ? p[b + s - 1] : 0.0, hi = p[b + s];
            out[off + b + s] = (uint16_t)bits_fx(std::max((hi - lo) / 32768.0, 1.0 / 32768.0));
        }
}

static const Tables &tables() {
    static Tables T;
    static std::once_flag once;
    std::call_once(once, [] {
        const int qrep[4] = {20, 60, 120, 255};
        for (int qc = 0; qc < 4; qc++) {
            av1g_cdfs c;
            av1g_cdfs_init(&c, qrep[qc]);
            T.cost[qc].assign(NCDF, 0);
            uint16_t *o = T.cost[qc].data();
#define CF(f) cost_field(c, c.f, o)
            CF(y_mode); CF(uv_mode_cfl_not_allowed); CF(uv_mode_cfl_allowed); CF(angle_delta);
            CF(partition_w8); CF(partition_w16); CF(partition_w32); CF(partition_w64);
            CF(tx_8x8); CF(tx_16x16); CF(tx_32x32); CF(tx_64x64); CF(skip); CF(filter_intra_mode); CF(filter_intra);
            CF(intra_tx_set1); CF(intra_tx_set2); CF(cfl_sign); CF(cfl_alpha);
            CF(txb_skip); CF(eob_pt_16); CF(eob_pt_32); CF(eob_pt_64); CF(eob_pt_128);
            CF(eob_pt_256); CF(eob_pt_512); CF(eob_pt_1024); CF(eob_extra); CF(dc_sign); CF(coeff_base_eob); CF(coeff_base);
            CF(coeff_br);
#undef CF
            if (qc == 0) {
                for (int m = 0; m < 13; m++) {
                    double p = 0;
                    for (int a = 0; a < 5; a++)
                        for (int l = 0; l < 5; l++) {
                            const uint16_t *cd = c.y_mode[a][l];
                            p += (cd[m] - (m ? cd[m - 1] : 0)) / 32768.0;
                        }
                    T.avgY[m] = bits_fx(std::max(p / 25.0, 1e-6));
                }
                for (int b = 0; b < 5; b++)
                    for (int p = 0; p < 10; p++) T.avgPart[b][p] = 20 * 256;
                for (int bsl = 1; bsl <= 4; bsl++) {
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
        }
    });
    return T;
}

// lambda (dev_common.cuh:99-107): rdmult = dc_q^2 (3.3 + 0.0015 dc_q) (128 + w) / 128, lambda = rdmult / 2048
static void lambda_fx(int qidx, int bd, i64 *lam, i64 *sq) {
    const int q = av1g_dc_q_bd(qidx, bd);
    double rd = (double)q * q * (3.3 + 0.0015 * q);
    int w = ((255 - qidx) * 3) / 4;
    w = w < 0 ? 0 : w > 72 ? 72 : w;
    rd = rd * (128 + w) / 128.0;
    const double l = rd / 2048.0;
    *lam = llround(l * 256.0);
    *sq = llround(std::sqrt(l) * 256.0);
}

// ---------------------------------------------------------------------------------------------------------------
// forward transform: the transposed step lists of the spec's inverse 1-D transforms (spec 7.13.2), run in reverse.
// Integer, with the spec's Round2(., 12) per rotation.  Evaluated in 64 bits; an intermediate outside int32 aborts
// (the kernels evaluate in 32 bits, so agreement also proves their range).
// ---------------------------------------------------------------------------------------------------------------
struct Op { char t; int a, b, ang, flip; };
struct OpList { std::vector<Op> ops; std::vector<std::vector<int>> perms, sgns; };

static int brevn(int n, int x) { int t = 0; for (int i = 0; i < n; i++) t |= ((x >> i) & 1) << (n - 1 - i); return t; }

static void push_perm(OpList &L, const std::vector<int> &src, const std::vector<int> &sgn) {
    L.ops.push_back(Op{'P', (int)L.perms.size(), 0, 0, 0});
    L.perms.push_back(src);
    L.sgns.push_back(sgn);
}

// the av1g_idct step order (dsp.h:242-285), recorded instead of executed
static OpList idct_list(int n) {
    OpList L;
    const int n0 = 1 << n;
    std::vector<int> src(n0), one(n0, 1);
    for (int i = 0; i < n0; i++) src[i] = brevn(n, i);
    push_perm(L, src, one);
    auto B = [&](int a, int b, int ang, int fl) { L.ops.push_back(Op{'B', a, b, ang, fl}); };
    auto H = [&](int a, int b, int fl) { L.ops.push_back(Op{'H', a, b, 0, fl}); };
    if (n == 6) for (int i = 0; i < 16; i++) B(32 + i, 63 - i, 63 - 4 * brevn(4, i), 0);
    if (n >= 5) for (int i = 0; i < 8; i++) B(16 + i, 31 - i, 6 + (brevn(3, 7 - i) << 3), 0);
    if (n == 6) for (int i = 0; i < 16; i++) H(32 + i * 2, 33 + i * 2, i & 1);
    if (n >= 4) for (int i = 0; i < 4; i++) B(8 + i, 15 - i, 12 + (brevn(2, 3 - i) << 4), 0);
    if (n >= 5) for (int i = 0; i < 8; i++) H(16 + 2 * i, 17 + 2 * i, i & 1);
    if (n == 6) for (int i = 0; i < 4; i++) for (int j = 0; j < 2; j++) B(62 - i * 4 - j, 33 + i * 4 + j, 60 - 16 * brevn(2, i) + 64 * j, 1);
    if (n >= 3) for (int i = 0; i < 2; i++) B(4 + i, 7 - i, 56 - 32 * i, 0);
    if (n >= 4) for (int i = 0; i < 4; i++) H(8 + 2 * i, 9 + 2 * i, i & 1);
    if (n >= 5) for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) B(30 - 4 * i - j, 17 + 4 * i + j, 24 + (j << 6) + ((1 - i) << 5), 1);
    if (n == 6) for (int i = 0; i < 8; i++) for (int j = 0; j < 2; j++) H(32 + i * 4 + j, 35 + i * 4 - j, i & 1);
    for (int i = 0; i < 2; i++) B(2 * i, 2 * i + 1, 32 + 16 * i, 1 - i);
    if (n >= 3) for (int i = 0; i < 2; i++) H(4 + 2 * i, 5 + 2 * i, i);
    if (n >= 4) for (int i = 0; i < 2; i++) B(14 - i, 9 + i, 48 + 64 * i, 1);
    if (n >= 5) for (int i = 0; i < 4; i++) for (int j = 0; j < 2; j++) H(16 + 4 * i + j, 19 + 4 * i - j, i & 1);
    if (n == 6) for (int i = 0; i < 2; i++) for (int j = 0; j < 4; j++) B(61 - i * 8 - j, 34 + i * 8 + j, 56 - i * 32 + (j >> 1) * 64, 1);
    for (int i = 0; i < 2; i++) H(i, 3 - i, 0);
    if (n >= 3) B(6, 5, 32, 1);
    if (n >= 4) for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) H(8 + 4 * i + j, 11 + 4 * i - j, i);
    if (n >= 5) for (int i = 0; i < 4; i++) B(29 - i, 18 + i, 48 + (i >> 1) * 64, 1);
    if (n == 6) for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) H(32 + 8 * i + j, 39 + 8 * i - j, i & 1);
    if (n >= 3) for (int i = 0; i < 4; i++) H(i, 7 - i, 0);
    if (n >= 4) for (int i = 0; i < 2; i++) B(13 - i, 10 + i, 32, 1);
    if (n >= 5) for (int i = 0; i < 2; i++) for (int j = 0; j < 4; j++) H(16 + i * 8 + j, 23 + i * 8 - j, i);
    if (n == 6) for (int i = 0; i < 8; i++) B(59 - i, 36 + i, i < 4 ? 48 : 112, 1);
    if (n >= 4) for (int i = 0; i < 8; i++) H(i, 15 - i, 0);
    if (n >= 5) for (int i = 0; i < 4; i++) B(27 - i, 20 + i, 32, 1);
    if (n == 6) for (int i = 0; i < 8; i++) { H(32 + i, 47 - i, 0); H(48 + i, 63 - i, 1); }
    if (n >= 5) for (int i = 0; i < 16; i++) H(i, 31 - i, 0);
    if (n == 6) for (int i = 0; i < 8; i++) B(55 - i, 40 + i, 32, 1);
    if (n == 6) for (int i = 0; i < 32; i++) H(i, 63 - i, 0);
    return L;
}

// av1g_iadst_in_perm / out_perm (dsp.h:287-305)
static void adst_perms(int n, std::vector<int> &inSrc, std::vector<int> &outSrc, std::vector<int> &outSgn) {
    const int n0 = 1 << n;
    inSrc.resize(n0); outSrc.resize(n0); outSgn.resize(n0);
    for (int i = 0; i < n0; i++) {
        inSrc[i] = (i & 1) ? (i - 1) : (n0 - i - 1);
        const int a = (i >> 3) & 1, b = ((i >> 2) & 1) ^ ((i >> 3) & 1), c = ((i >> 1) & 1) ^ ((i >> 2) & 1), d = (i & 1) ^ ((i >> 1) & 1);
        outSrc[i] = ((d << 3) | (c << 2) | (b << 1) | a) >> (4 - n);
        outSgn[i] = (i & 1) ? -1 : 1;
    }
}

// av1g_iadst8 / av1g_iadst16 step order (dsp.h:343-367)
static OpList iadst_list(int n) {
    OpList L;
    std::vector<int> inSrc, outSrc, outSgn;
    adst_perms(n, inSrc, outSrc, outSgn);
    push_perm(L, inSrc, std::vector<int>(inSrc.size(), 1));
    auto B = [&](int a, int b, int ang, int fl) { L.ops.push_back(Op{'B', a, b, ang, fl}); };
    auto H = [&](int a, int b, int fl) { L.ops.push_back(Op{'H', a, b, 0, fl}); };
    if (n == 3) {
        for (int i = 0; i < 4; i++) B(2 * i, 2 * i + 1, 60 - 16 * i, 1);
        for (int i = 0; i < 4; i++) H(i, 4 + i, 0);
        for (int i = 0; i < 2; i++) B(4 + 3 * i, 5 + i, 48 - 32 * i, 1);
        for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) H(4 * j + i, 2 + 4 * j + i, 0);
        for (int i = 0; i < 2; i++) B(2 + 4 * i, 3 + 4 * i, 32, 1);
    } else {
        for (int i = 0; i < 8; i++) B(2 * i, 2 * i + 1, 62 - 8 * i, 1);
        for (int i = 0; i < 8; i++) H(i, 8 + i, 0);
        for (int i = 0; i < 2; i++) { B(8 + 2 * i, 9 + 2 * i, 56 - 32 * i, 1); B(13 + 2 * i, 12 + 2 * i, 8 + 32 * i, 1); }
        for (int i = 0; i < 4; i++) for (int j = 0; j < 2; j++) H(8 * j + i, 4 + 8 * j + i, 0);
        for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) B(4 + 8 * j + 3 * i, 5 + 8 * j + i, 48 - 32 * i, 1);
        for (int i = 0; i < 2; i++) for (int j = 0; j < 4; j++) H(4 * j + i, 2 + 4 * j + i, 0);
        for (int i = 0; i < 4; i++) B(2 + 4 * i, 3 + 4 * i, 32, 1);
    }
    push_perm(L, outSrc, outSgn);
    return L;
}

static inline i64 chk32(i64 v) {
    if (v < INT32_MIN || v > INT32_MAX) { fprintf(stderr, "oracle: forward transform left int32\n"); abort(); }
    return v;
}

// transpose of the recorded network, in reverse step order
static void run_transposed(const OpList &L, i64 *T) {
    for (int k = (int)L.ops.size() - 1; k >= 0; k--) {
        const Op &o = L.ops[k];
        if (o.t == 'P') {
            const std::vector<int> &src = L.perms[o.a], &sgn = L.sgns[o.a];
            i64 c[64];
            for (size_t i = 0; i < src.size(); i++) c[i] = T[i];
            for (size_t i = 0; i < src.size(); i++) T[src[i]] = sgn[i] * c[i];
        } else if (o.t == 'B') {
            const int ang = o.flip ? o.ang : -o.ang;
            const i64 c = av1g_cos128(ang), s = av1g_sin128(ang);
            const i64 p1 = chk32(T[o.a] * c), p2 = chk32(T[o.b] * s), p3 = chk32(T[o.a] * s), p4 = chk32(T[o.b] * c);
            const i64 x = (chk32(p1 - p2) + 2048) >> 12, y = (chk32(p3 + p4) + 2048) >> 12;
            if (o.flip) { T[o.a] = y; T[o.b] = x; } else { T[o.a] = x; T[o.b] = y; }
        } else {
            int a = o.a, b = o.b;
            if (o.flip) std::swap(a, b);
            const i64 x = T[a], y = T[b];
            T[a] = chk32(x + y);
            T[b] = chk32(x - y);
        }
    }
}

static void fwd1d(int kind, int n, i64 *T) {
    static std::vector<OpList> dct, adst;
    static std::once_flag once;
    std::call_once(once, [] {
        dct.resize(7); adst.resize(7);
        for (int k = 2; k <= 6; k++) dct[k] = idct_list(k);
        adst[3] = iadst_list(3);
        adst[4] = iadst_list(4);
    });
    if (kind == AV1G_K_DCT) { run_transposed(dct[n], T); return; }
    if (kind == AV1G_K_ADST) {
        if (n == 2) {   // transpose of the SINPI matrix of av1g_iadst4 (dsp.h:307-341)
            static const int S[4][4] = {{1321, 3344, 3803, 2482}, {2482, 3344, -1321, -3803}, {3344, 0, -3344, 3344},
                                        {3803, -3344, 2482, -1321}};
            i64 x[4] = {T[0], T[1], T[2], T[3]};
            for (int j = 0; j < 4; j++) {
                i64 s = 0;
                for (int i = 0; i < 4; i++) s = chk32(s + chk32(S[i][j] * x[i]));
                T[j] = (s + 2048) >> 12;
            }
            return;
        }
        run_transposed(adst[n], T);
        return;
    }
    // identity (av1g_iidentity, dsp.h:369-377): a diagonal, its own transpose
    for (int i = 0; i < (1 << n); i++) {
        if (n == 2) T[i] = (chk32(T[i] * 5793) + 2048) >> 12;
        else if (n == 3) T[i] = chk32(T[i] * 2);
        else if (n == 4) T[i] = (chk32(T[i] * 11586) + 2048) >> 12;
        else T[i] = chk32(T[i] * 4);
    }
}

// shifts of the 2-D forward transform (the design's range rule): input pre-shift s0 keeps every column value below
// 2^17 (sum of |inputs| bound), s1 = log2 W keeps the row inputs' sum below 2^17, s2 brings the result to the
// dequantisation domain with FB fractional bits: DQ = M_H^T R M_W 2^(rowShift + 4) / (H W / 4) / rect.
struct FwdShifts { int s0, s1, s2; };
static FwdShifts fwd_shifts(int txSz, int bd) {
    const int lw = AV1G_T(Tx_Width_Log2)[txSz], lh = AV1G_T(Tx_Height_Log2)[txSz];
    FwdShifts s;
    s.s0 = std::max(0, 17 - bd - lh);
    s.s1 = lw;
    const int E = AV1G_T(Transform_Row_Shift)[txSz] + 4 + FB - (lw + lh - 2);
    s.s2 = s.s0 - s.s1 - E;
    return s;
}
static inline i64 rshift_round(i64 v, int s) { return s > 0 ? (v + ((i64)1 << (s - 1))) >> s : (s < 0 ? v * ((i64)1 << -s) : v); }

static void fwd2d(const int32_t *res, int txSz, int txType, int bd, int32_t *out) {
    const int lw = AV1G_T(Tx_Width_Log2)[txSz], lh = AV1G_T(Tx_Height_Log2)[txSz];
    const int W = 1 << lw, H = 1 << lh, tw = std::min(W, 32), th = std::min(H, 32);
    const int rk = av1g_row_kind(txType), ck = av1g_col_kind(txType);
    const int fud = av1g_flip_ud(txType), flr = av1g_flip_lr(txType);
    const bool rect = (lw - lh == 1 || lh - lw == 1);
    const FwdShifts s = fwd_shifts(txSz, bd);
    std::vector<i64> tmp((size_t)th * W);
    i64 T[64];
    for (int j = 0; j < W; j++) {
        for (int i = 0; i < H; i++) T[i] = (i64)res[(fud ? H - 1 - i : i) * W + (flr ? W - 1 - j : j)] * ((i64)1 << s.s0);
        fwd1d(ck, lh, T);
        for (int i = 0; i < th; i++) tmp[(size_t)i * W + j] = rshift_round(T[i], s.s1);
    }
    for (int i = 0; i < th; i++) {
        for (int j = 0; j < W; j++) T[j] = tmp[(size_t)i * W + j];
        fwd1d(rk, lw, T);
        for (int j = 0; j < tw; j++) {
            i64 v = T[j];
            if (rect) v = (chk32(v * 5793) + 2048) >> 12;
            out[i * tw + j] = (int32_t)chk32(rshift_round(v, s.s2));
        }
    }
}

// ---------------------------------------------------------------------------------------------------------------
// quantisation, distortion, rate (dev_tx.cuh:48-165, 273-317)
// ---------------------------------------------------------------------------------------------------------------
static int tx_index_in_set(int set, int t) {
    if (set == AV1G_TX_SET_INTRA_1) { for (int i = 0; i < 7; i++) if (AV1G_T(Tx_Type_Intra_Inv_Set1)[i] == t) return i; }
    else { for (int i = 0; i < 5; i++) if (AV1G_T(Tx_Type_Intra_Inv_Set2)[i] == t) return i; }
    return 0;
}

// distortion scale: pixel SSE = sum (DQ - dequant)^2 2^-(2 FB + k), k = 2 (rowShift + 4) - (lw + lh - 2) + rect
static int dist_k(int txSz) {
    const int lw = AV1G_T(Tx_Width_Log2)[txSz], lh = AV1G_T(Tx_Height_Log2)[txSz];
    const int rect = (lw - lh == 1 || lh - lw == 1) ? 1 : 0;
    return 2 * (AV1G_T(Transform_Row_Shift)[txSz] + 4) - (lw + lh - 2) + rect;
}

struct EvalIn {
    int txSz, txType, plane, bd, dcQ, acQ, skipCtx, dcCtx, intraDir;
    const uint16_t *C;
    i64 resEnergy;   // sum r^2 of the residual (64-point sizes: the energy of the dropped coefficients)
};
struct EvalOut { i64 D, R; int eob; };

static i64 base_bits(const EvalIn &e, int eob) {
    const int txSz = e.txSz;
    const int txSzCtx = (AV1G_T(Tx_Size_Sqr)[txSz] + AV1G_T(Tx_Size_Sqr_Up)[txSz] + 1) >> 1;
    const uint16_t *C = e.C;
    if (eob == 0) return C[COFF(txb_skip[txSzCtx][e.skipCtx]) + 1];
    i64 b = C[COFF(txb_skip[txSzCtx][e.skipCtx]) + 0];
    const int ptype = e.plane > 0;
    if (e.plane == 0) {
        const int set = av1g_get_tx_set_intra(txSz, 0);
        if (set > 0) {
            const int sqr = AV1G_T(Tx_Size_Sqr)[txSz];
            const int idx = tx_index_in_set(set, e.txType);
            if (set == AV1G_TX_SET_INTRA_1) b += C[COFF(intra_tx_set1[sqr][e.intraDir]) + idx];
            else b += C[COFF(intra_tx_set2[sqr][e.intraDir]) + idx];
        }
    }
    const int txClass = av1g_tx_class(e.txType);
    const int eobMultisize = std::min((int)AV1G_T(Tx_Width_Log2)[txSz], 5) + std::min((int)AV1G_T(Tx_Height_Log2)[txSz], 5) - 4;
    int eobPt;
    if (eob <= 2) eobPt = eob;
    else { eobPt = 2; int v = eob - 1; while (v > 1) { v >>= 1; eobPt++; } }
    const int ectx = txClass == AV1G_TX_CLASS_2D ? 0 : 1;
    int c;
    switch (eobMultisize) {
    case 0: c = COFF(eob_pt_16[ptype][ectx]); break;
    case 1: c = COFF(eob_pt_32[ptype][ectx]); break;
    case 2: c = COFF(eob_pt_64[ptype][ectx]); break;
    case 3: c = COFF(eob_pt_128[ptype][ectx]); break;
    case 4: c = COFF(eob_pt_256[ptype][ectx]); break;
    case 5: c = COFF(eob_pt_512[ptype]); break;
    default: c = COFF(eob_pt_1024[ptype]); break;
    }
    b += C[c + eobPt - 1];
    if (eobPt >= 3) {
        const int rem = eob - ((1 << (eobPt - 2)) + 1);
        b += C[COFF(eob_extra[txSzCtx][ptype][eobPt - 3]) + ((rem >> (eobPt - 3)) & 1)];
        b += (i64)(eobPt - 3) * 256;
    }
    return b;
}

static i64 coeff_bits(int c, int eob, const int16_t *q, const uint16_t *scan, int txSz, int txClass, int ptype, int dcCtx,
                      const uint16_t *C) {
    const int txSzCtx = (AV1G_T(Tx_Size_Sqr)[txSz] + AV1G_T(Tx_Size_Sqr_Up)[txSz] + 1) >> 1;
    const int adj = AV1G_T(Adjusted_Tx_Size)[txSz];
    const int bwl = AV1G_T(Tx_Width_Log2)[adj];
    const int width = 1 << bwl, height = AV1G_T(Tx_Height)[adj];
    const int pos = scan[c];
    const int qv = q[pos];
    const int v = std::abs(qv);
    const int level = std::min(v, 15);
    const int row = pos >> bwl, col = pos - (row << bwl);
    i64 b;
    if (c == eob - 1) {
        const int bctx = c == 0 ? 0 : c <= (height << bwl) / 8 ? 1 : c <= (height << bwl) / 4 ? 2 : 3;
        b = C[COFF(coeff_base_eob[txSzCtx][ptype][bctx]) + std::min(level, 3) - 1];
    } else {
        int mag = 0;
        for (int idx = 0; idx < 5; idx++) {
            const int rr = row + AV1G_T(Sig_Ref_Diff_Offset)[txClass][idx][0];
            const int cc = col + AV1G_T(Sig_Ref_Diff_Offset)[txClass][idx][1];
            if (rr >= 0 && cc >= 0 && rr < height && cc < width) mag += std::min(std::abs((int)q[(rr << bwl) + cc]), 3);
        }
        int bctx = std::min((mag + 1) >> 1, 4);
        if (txClass == AV1G_TX_CLASS_2D) {
            if (row == 0 && col == 0) bctx = 0;
            else bctx += AV1G_T(Coeff_Base_Ctx_Offset)[txSz][std::min(row, 4)][std::min(col, 4)];
        } else {
            const int id = txClass == AV1G_TX_CLASS_VERT ? row : col;
            bctx += AV1G_T(Coeff_Base_Pos_Ctx_Offset)[std::min(id, 2)];
        }
        b = C[COFF(coeff_base[txSzCtx][ptype][bctx]) + std::min(level, 3)];
    }
    if (level > 2) {
        int mag = 0;
        for (int idx = 0; idx < 3; idx++) {
            const int rr = row + AV1G_T(Mag_Ref_Offset_With_Tx_Class)[txClass][idx][0];
            const int cc = col + AV1G_T(Mag_Ref_Offset_With_Tx_Class)[txClass][idx][1];
            if (rr >= 0 && cc >= 0 && rr < height && cc < width) mag += std::min(std::abs((int)q[rr * width + cc]), 15);
        }
        mag = std::min((mag + 1) >> 1, 6);
        int brctx;
        if (pos == 0) brctx = mag;
        else if (txClass == AV1G_TX_CLASS_2D) brctx = (row < 2 && col < 2) ? mag + 7 : mag + 14;
        else if (txClass == AV1G_TX_CLASS_HORIZ) brctx = col == 0 ? mag + 7 : mag + 14;
        else brctx = row == 0 ? mag + 7 : mag + 14;
        const int brsz = std::min(txSzCtx, (int)AV1G_TX_32X32);
        const int cid = COFF(coeff_br[brsz][ptype][brctx]);
        int rem = level - 3;
        for (int i = 0; i < 4; i++) {
            const int k = std::min(rem, 3);
            b += C[cid + k];
            rem -= k;
            if (k < 3) break;
        }
    }
    if (v) {
        if (c == 0) b += C[COFF(dc_sign[ptype][dcCtx]) + (qv < 0)];
        else b += 256;
        if (v > 14) {
            int xg = v - 14, len = 0;
            while (xg > 1) { xg >>= 1; len++; }
            b += (i64)(2 * len + 1) * 256;
        }
    }
    return b;
}

// dead-zone quantiser in integers: zbin 21/32 (0.65625), rounding 3/8 (0.375); dequantisation per spec 7.12.3
static void quant_rate(const int32_t *coef, const EvalIn &e, int16_t *q, EvalOut &o) {
    const int txSz = e.txSz;
    const int W = AV1G_T(Tx_Width)[txSz], H = AV1G_T(Tx_Height)[txSz];
    const int tw = std::min(W, 32), th = std::min(H, 32), n = tw * th;
    const int den = av1g_dq_denom(txSz);
    i64 dist = 0, kept = 0;
    for (int idx = 0; idx < n; idx++) {
        const int32_t v = coef[idx];
        const int step = idx == 0 ? e.dcQ : e.acQ;
        const i64 a = (i64)std::abs(v) * den;
        const i64 S = (i64)step << FB;
        int l = 0;
        if (a * 32 >= 21 * S) l = (int)std::min<i64>((8 * a + 3 * S) / (8 * S), 16383);
        const int qv = v < 0 ? -l : l;
        q[idx] = (int16_t)qv;
        const i64 dq = l ? (i64)av1g_dequant_coef_bd(qv, step, den, e.bd) << FB : 0;
        const i64 d = (i64)v - dq;
        dist += d * d;
        kept += (i64)v * v;
    }
    const uint16_t *scan = av1g_get_scan(txSz, e.txType);
    int eob = 0;
    for (int c = 0; c < n; c++) if (q[scan[c]]) eob = c + 1;
    i64 bits = base_bits(e, eob);
    const int txClass = av1g_tx_class(e.txType);
    for (int c = 0; c < eob; c++) bits += coeff_bits(c, eob, q, scan, txSz, txClass, e.plane > 0, e.dcCtx, e.C);
    const int sh = 16 - 2 * FB - dist_k(txSz);   // >= 0 for every size
    i64 D = dist << sh;
    if (W == 64 || H == 64) D += std::max<i64>(0, (e.resEnergy << 16) - (kept << sh));
    o.D = D;
    o.R = bits;
    o.eob = eob;
}




// ---------------------------------------------------------------------------------------------------------------
// algorithmic INT32 operation count (the roofline numerator): every unit of work the search does is counted, each with
// the integer operations (add / sub / mul / shift / min / max / abs / compare / select / table read) its definition
// takes, counted from this file's code: a residual sample = its prediction + 1; a 4x4 Hadamard = 111; a forward
// butterfly rotation = 10, an H step = 2, the ADST4 matrix = 36, an identity element = 2, plus 1 pre-shift and 2 for
// the rounding of every input / output; quantisation 18 per coefficient, the eob scan 2; the rate 40 per coefficient up
// to the eob (+25 when level > 2) and 60 per block; the inverse as the forward plus 6 per coefficient of dequantisation
// and 3 per sample of reconstruction.  ops[0]: open-loop analysis, ops[1]: closed loop.
// ---------------------------------------------------------------------------------------------------------------
struct OpCounter { std::atomic<uint64_t> ops[2]; };
static int pred_ops(int mode, int delta) {
    if (mode == AV1G_DC_PRED) return 1;
    if (mode == AV1G_PAETH_PRED) return 12;
    if (mode == AV1G_SMOOTH_PRED) return 12;
    if (mode == AV1G_SMOOTH_V_PRED || mode == AV1G_SMOOTH_H_PRED) return 7;
    const int pa = AV1G_T(Mode_To_Angle)[mode] + delta * AV1G_ANGLE_STEP;
    return (pa == 90 || pa == 180) ? 1 : 9;
}
static int fwd1d_ops(int kind, int n) {
    static int cache[3][7];
    static std::once_flag once;
    std::call_once(once, [] {
        for (int k = 0; k < 3; k++) for (int l = 2; l <= 6; l++) {
            int c = 0;
            if (k == AV1G_K_IDT) c = 2 * (1 << l);
            else if (k == AV1G_K_ADST && l == 2) c = 36;
            else if (k == AV1G_K_DCT || (k == AV1G_K_ADST && l <= 4)) {
                const OpList L = k == AV1G_K_DCT ? idct_list(l) : iadst_list(l);
                for (const Op &o : L.ops) c += o.t == 'B' ? 10 : o.t == 'H' ? 2 : 0;
            }
            cache[k][l] = c + 3 * (1 << l);
        }
    });
    return cache[kind][n];
}
static uint64_t fwd2d_ops(int txSz, int txType) {
    const int lw = AV1G_T(Tx_Width_Log2)[txSz], lh = AV1G_T(Tx_Height_Log2)[txSz];
    const int W = 1 << lw, H = 1 << lh, th = std::min(H, 32), tw = std::min(W, 32);
    return (uint64_t)W * fwd1d_ops(av1g_col_kind(txType), lh) + (uint64_t)th * fwd1d_ops(av1g_row_kind(txType), lw) + 3ull * tw * th;
}
static uint64_t eval_ops(int txSz, int txType, int eob, int nBig, int mode, int delta) {
    const int W = AV1G_T(Tx_Width)[txSz], H = AV1G_T(Tx_Height)[txSz], n = std::min(W, 32) * std::min(H, 32);
    return (uint64_t)W * H * (pred_ops(mode, delta) + 1) + fwd2d_ops(txSz, txType) + 20ull * n + 40ull * eob + 25ull * nBig + 60;
}

// ---------------------------------------------------------------------------------------------------------------
// the search engine of one image
// ---------------------------------------------------------------------------------------------------------------
struct BlockRes { i64 J; uint8_t cand[4]; uint8_t ncand; uint8_t tx; };
struct Leaf { uint8_t bsize, x4, y4; };
struct TileBox { int x0, y0, x1, y1; };   // pixels
struct TxbOut { av1g_txb t; std::vector<int16_t> q; };
struct SbOut { std::vector<av1g_block> blocks; std::vector<std::vector<TxbOut>> txb; };

static inline int cand_mode(int c) { return c >> 3; }
static inline int cand_delta(int c) { return (c & 7) - 3; }
static inline int cand_pack(int m, int d) { return (m << 3) | (d + 3); }
static inline int bw_px(int bs) { return 4 * av1g_bw4(bs); }
static inline int bh_px(int bs) { return 4 * av1g_bh4(bs); }
static inline int log2i(int v) { int l = 0; while ((1 << l) < v) l++; return l; }

// Z-order index of a 4x4 unit inside a 64x64 SB (dev_common.cuh:145-149)
static inline int zorder16(int x, int y) {
    int z = 0;
    for (int b = 0; b < 4; b++) z |= (((x >> b) & 1) << (2 * b)) | (((y >> b) & 1) << (2 * b + 1));
    return z;
}
// open-loop "decoded before (x, y)" guess for the analysis edges (dev_common.cuh:153-163), luma units
static bool ol_decoded(int px, int py, int x, int y, const TileBox &t) {
    if (px < t.x0 || py < t.y0 || px >= t.x1 || py >= t.y1) return false;
    const int S = 64, sbx = (x / S) * S, sby = (y / S) * S;
    if (py < sby) return true;
    if (px < sbx) return py < sby + S;
    if (px >= sbx + S || py >= sby + S) return false;
    return zorder16(((px - sbx) / 4) & 15, ((py - sby) / 4) & 15) < zorder16(((x - sbx) / 4) & 15, ((y - sby) / 4) & 15);
}

// sum |coefficients| of the 4x4 Hadamard transform of d (k_analysis.cuh:47-62)
static int hadamard4_sum(const int *d0) {
    int d[16];
    for (int k = 0; k < 16; k++) d[k] = d0[k];
    for (int i = 0; i < 4; i++) {
        int *r = d + 4 * i;
        const int s0 = r[0] + r[1], s1 = r[0] - r[1], s2 = r[2] + r[3], s3 = r[2] - r[3];
        r[0] = s0 + s2; r[1] = s1 + s3; r[2] = s0 - s2; r[3] = s1 - s3;
    }
    int sum = 0;
    for (int j = 0; j < 4; j++) {
        const int s0 = d[j] + d[4 + j], s1 = d[j] - d[4 + j], s2 = d[8 + j] + d[12 + j], s3 = d[8 + j] - d[12 + j];
        sum += std::abs(s0 + s2) + std::abs(s1 + s3) + std::abs(s0 - s2) + std::abs(s1 - s3);
    }
    return sum;
}

template <int BD>
struct Engine {
    typedef av1g_pixel_t(BD) Px;
    int W = 0, H = 0, MiCols = 0, MiRows = 0, sbCols = 0, sbRows = 0, ssx = 1, ssy = 1, qidx = 0, qctx = 0;
    av1g_tiles tiles;
    int pw[3], ph[3];                 // padded plane sizes (allocation), samples
    std::vector<Px> src[3], rec[3];
    i64 lam = 0, sqlam = 0;
    int dcQ[3], acQ[3];
    const uint16_t *C = nullptr;
    const Tables *T = nullptr;
    std::vector<BlockRes> blk[22];
    int shNbx[22], shNby[22];
    std::vector<std::vector<Leaf>> leaves;
    std::vector<uint8_t> mYMode, mUVMode, cLvl[3], cDc[3];
    std::vector<SbOut> sbo;
    OpCounter *ops = nullptr;

    TileBox tile_of(int x, int y) const {
        int c = 0, r = 0;
        while (c + 1 < (int)tiles.cols && x >= (int)tiles.mi_col_starts[c + 1] * 4) c++;
        while (r + 1 < (int)tiles.rows && y >= (int)tiles.mi_row_starts[r + 1] * 4) r++;
        return TileBox{(int)tiles.mi_col_starts[c] * 4, (int)tiles.mi_row_starts[r] * 4, (int)tiles.mi_col_starts[c + 1] * 4,
                       (int)tiles.mi_row_starts[r + 1] * 4};
    }

    void setup(const orc_image &img) {
        W = img.width; H = img.height;
        MiCols = av1g_mi_cols(W); MiRows = av1g_mi_rows(H);
        sbCols = (MiCols + 15) >> 4; sbRows = (MiRows + 15) >> 4;
        ssx = ssy = img.chroma_444 ? 0 : 1;
        qidx = img.qindex;
        qctx = av1g_coeff_cdf_q_ctx(qidx);
        av1g_tile_layout((uint32_t)W, (uint32_t)H, -1, -1, &tiles);
        T = &tables();
        C = T->cost[qctx].data();
        lambda_fx(qidx, BD, &lam, &sqlam);
        // block quantizers (spec set_block_q; no chroma delta-q in the plain form)
        for (int p = 0; p < 3; p++) { dcQ[p] = av1g_dc_q<BD>(qidx); acQ[p] = av1g_ac_q<BD>(qidx); }
        // source planes padded by edge replication to the SB grid (+ one SB column of slack)
        for (int p = 0; p < 3; p++) {
            const int sx = p ? ssx : 0, sy = p ? ssy : 0;
            pw[p] = ((sbCols + 1) * 64) >> sx;
            ph[p] = (sbRows * 64) >> sy;
            const int vw = (W + sx) >> sx, vh = (H + sy) >> sy;
            src[p].assign((size_t)pw[p] * ph[p], 0);
            rec[p].assign((size_t)pw[p] * ph[p], 0);
            const Px *in = (const Px *)img.planes[p];
            for (int y = 0; y < ph[p]; y++)
                for (int x = 0; x < pw[p]; x++)
                    src[p][(size_t)y * pw[p] + x] = in[(size_t)std::min(y, vh - 1) * img.stride[p] + std::min(x, vw - 1)];
        }
        for (int s = 0; s < 22; s++) {
            shNbx[s] = shNby[s] = 0;
            if (s >= AV1G_BLOCK_INVALID || (s >= 13 && s <= 15)) continue;
            shNbx[s] = (MiCols * 4 + bw_px(s) - 1) / bw_px(s);
            shNby[s] = (MiRows * 4 + bh_px(s) - 1) / bh_px(s);
            blk[s].assign((size_t)shNbx[s] * shNby[s], BlockRes{INF, {0, 0, 0, 0}, 0, 0});
        }
        mYMode.assign((size_t)MiCols * MiRows, 0);
        mUVMode.assign((size_t)MiCols * MiRows, 0);
        for (int p = 0; p < 3; p++) {
            const size_t n = (size_t)(MiCols >> (p ? ssx : 0)) * (MiRows >> (p ? ssy : 0));
            cLvl[p].assign(n, 0);
            cDc[p].assign(n, 0);
        }
        leaves.assign((size_t)sbCols * sbRows, {});
        sbo.assign((size_t)sbCols * sbRows, SbOut());
    }

    // ---- one evaluation: residual -> forward transform -> quantise / rate / distortion ----
    EvalOut eval(const int32_t *res, int txSz, int txType, int plane, int skipCtx, int dcCtx, int intraDir, i64 resE, int16_t *q,
                 int stage = -1, int mode = 0, int delta = 0) const {
        int32_t coef[1024];
        fwd2d(res, txSz, txType, BD, coef);
        EvalIn e{txSz, txType, plane, BD, dcQ[plane], acQ[plane], skipCtx, dcCtx, intraDir, C, resE};
        EvalOut o;
        quant_rate(coef, e, q, o);
        if (ops && stage >= 0) {
            const uint16_t *scan = av1g_get_scan(txSz, txType);
            int big = 0;
            for (int c = 0; c < o.eob; c++) big += std::abs((int)q[scan[c]]) > 2;
            ops->ops[stage].fetch_add(eval_ops(txSz, txType, o.eob, big, mode, delta), std::memory_order_relaxed);
        }
        return o;
    }
    void count(int stage, uint64_t n) const { if (ops) ops->ops[stage].fetch_add(n, std::memory_order_relaxed); }

    // ---- open-loop analysis of one block (k_analysis.cuh:496-689) ----
    void analyse(int bs, int bx, int by) {
        const int w = bw_px(bs), h = bh_px(bs), lw = log2i(w), lh = log2i(h);
        const int x = bx * w, y = by * h;
        BlockRes &out = blk[bs][(size_t)by * shNbx[bs] + bx];
        if (x >= MiCols * 4 || y >= MiRows * 4) { out.J = INF; out.ncand = 0; return; }
        const TileBox tb = tile_of(x, y);
        const int haveL = x > tb.x0, haveA = y > tb.y0;
        const int haveAR = ol_decoded(x + w, y - 1, x, y, tb), haveBL = ol_decoded(x - 1, y + h, x, y, tb);
        const int maxX = MiCols * 4 - 1, maxY = MiRows * 4 - 1;
        const int sp = pw[0];
        const Px *s = src[0].data() + (size_t)y * sp + x;
        Px ea[AV1G_EDGE_LEN], el[AV1G_EDGE_LEN];
        Px *A = ea + AV1G_EDGE_OFF, *L = el + AV1G_EDGE_OFF;
        av1g_build_edges<BD>(src[0].data(), sp, x, y, lw, lh, haveL, haveA, haveAR, haveBL, maxX, maxY, A, L);
        const int txSz = AV1G_T(Max_Tx_Size_Rect)[bs];
        const int set = av1g_get_tx_set_intra(txSz, 0);
        auto mbits = [&](int c) -> i64 {
            const int m = cand_mode(c);
            i64 b = T->avgY[m];
            if (bs >= AV1G_BLOCK_8X8 && av1g_is_directional(m)) b += C[COFF(angle_delta[m - AV1G_V_PRED]) + cand_delta(c) + 3];
            return b;
        };
        std::vector<Px> pred((size_t)w * h);
        auto predict = [&](int c) { predictx(0, cand_mode(c), cand_delta(c), haveL, haveA, lw, lh, x, y, 0, A, L, pred.data(), w); };
        // ---- SATD screening: 13 modes at delta 0, then +-1..3 around the two best directional modes ----
        int cands[32];
        i64 js[32];
        int nc = 13;
        for (int m = 0; m < 13; m++) cands[m] = cand_pack(m, 0);
        auto screen = [&](int c0, int c1) {
            for (int ci = c0; ci < c1; ci++) {
                predict(cands[ci]);
                i64 satd = 0;
                for (int sy = 0; sy < h; sy += 4)
                    for (int sx = 0; sx < w; sx += 4) {
                        int d[16];
                        for (int i = 0; i < 4; i++)
                            for (int j = 0; j < 4; j++)
                                d[i * 4 + j] = (int)s[(sy + i) * sp + sx + j] - (int)pred[(size_t)(sy + i) * w + sx + j];
                        satd += hadamard4_sum(d);
                    }
                js[ci] = (satd << 14) + sqlam * mbits(cands[ci]);
                count(0, (uint64_t)(w * h / 16) * (16 * (uint64_t)pred_ops(cand_mode(cands[ci]), cand_delta(cands[ci])) + 111) + 30);
            }
        };
        screen(0, 13);
        if (bs >= AV1G_BLOCK_8X8) {
            int b0 = -1, b1 = -1;
            for (int m = AV1G_V_PRED; m <= AV1G_D67_PRED; m++) if (b0 < 0 || js[m] < js[b0]) b0 = m;
            for (int m = AV1G_V_PRED; m <= AV1G_D67_PRED; m++) if (m != b0 && (b1 < 0 || js[m] < js[b1])) b1 = m;
            for (int k = 0; k < 12; k++) {
                const int m = k < 6 ? b0 : b1, kk = k % 6;
                cands[13 + k] = cand_pack(m, kk < 3 ? -(kk + 1) : (kk - 2));
            }
            nc = 25;
            screen(13, 25);
        }
        int top[K_TOP];
        int nK = 0;
        {
            bool used[32] = {false};
            for (int k = 0; k < K_TOP; k++) {
                int b = -1;
                for (int i = 0; i < nc; i++) if (!used[i] && (b < 0 || js[i] < js[b])) b = i;
                if (b < 0) break;
                used[b] = true;
                top[nK++] = b;
            }
        }
        // ---- RD of the top-K with DCT_DCT, then the tx types of the winner ----
        const int hasC = av1g_has_chroma(bs, y >> 2, x >> 2, 0, ssx, ssy);
        const i64 overhead = (hasC ? UV_OVERHEAD : 0) + T->avgSkip0;
        std::vector<int32_t> res((size_t)w * h);
        int16_t q[1024];
        i64 bestJ = INF, resE = 0;
        int bestK = 0, bestTx = AV1G_DCT_DCT, resK = -1;
        const int nSteps = nK + (set != AV1G_TX_SET_DCTONLY ? 15 : 0);
        for (int st = 0; st < nSteps; st++) {
            const int k = st < nK ? st : bestK, t = st < nK ? AV1G_DCT_DCT : st - nK + 1;
            if (t != AV1G_DCT_DCT && !av1g_tx_type_in_set_intra(set, t)) continue;
            const int c = cands[top[k]];
            if (k != resK) {
                predict(c);
                resE = 0;
                for (int i = 0; i < h; i++)
                    for (int j = 0; j < w; j++) {
                        const int r = (int)s[i * sp + j] - (int)pred[(size_t)i * w + j];
                        res[(size_t)i * w + j] = r;
                        resE += (i64)r * r;
                    }
                resK = k;
            }
            const EvalOut o = eval(res.data(), txSz, t, 0, 0, 0, cand_mode(c), resE, q, 0, cand_mode(c), cand_delta(c));
            const i64 J = o.D + lam * (o.R + mbits(c) + overhead);
            if (J < bestJ) {
                bestJ = J;
                if (st < nK) bestK = k; else bestTx = t;
            }
        }
        out.J = bestJ;
        out.tx = (uint8_t)bestTx;
        int n = 0;
        out.cand[n++] = (uint8_t)cands[top[bestK]];
        for (int k = 0; k < nK; k++) if (k != bestK) out.cand[n++] = (uint8_t)cands[top[k]];
        out.ncand = (uint8_t)n;
    }

    // ---- partition DP of one SB (k_dp.cuh:72-297) ----
    i64 dpJ(int bs, int x, int y) const {
        if (bs >= AV1G_BLOCK_INVALID || shNbx[bs] == 0) return INF;
        return blk[bs][(size_t)(y / bh_px(bs)) * shNbx[bs] + x / bw_px(bs)].J;
    }
    static int sq_bsize(int n) { return n == 4 ? AV1G_BLOCK_4X4 : n == 8 ? AV1G_BLOCK_8X8 : n == 16 ? AV1G_BLOCK_16X16 : n == 32 ? AV1G_BLOCK_32X32 : AV1G_BLOCK_64X64; }
    static int sub_bsize(int p, int n) { return AV1G_T(Partition_Subsize)[p][sq_bsize(n)]; }

    void dp(int sbr, int sbc) {
        const int sbx = sbc * 64, sby = sbr * 64, FW = MiCols * 4, FH = MiRows * 4;
        struct Node { i64 J; int p; } node[85];
        const int lvBase[4] = {0, 1, 5, 21};
        for (int Lv = 3; Lv >= 0; Lv--) {
            const int n = 64 >> Lv, half = n >> 1, q4 = n >> 2, per = 1 << Lv;
            const int bsl = Lv == 3 ? 1 : Lv == 2 ? 2 : Lv == 1 ? 3 : 4;
            const int pmask = n == 8 ? 0xF : 0x3FF;
            for (int ny = 0; ny < per; ny++)
                for (int nx = 0; nx < per; nx++) {
                    Node &nd = node[lvBase[Lv] + ny * per + nx];
                    const int x = sbx + nx * n, y = sby + ny * n;
                    if (x >= FW || y >= FH) { nd.J = 0; nd.p = -1; continue; }
                    const bool hasRows = (y + half) < FH, hasCols = (x + half) < FW;
                    i64 splitJ = 0;
                    if (n == 8) {
                        for (int k = 0; k < 4; k++) {
                            const int xx = x + (k & 1) * 4, yy = y + (k >> 1) * 4;
                            if (xx < FW && yy < FH) splitJ = sat_add(splitJ, dpJ(AV1G_BLOCK_4X4, xx, yy));
                        }
                    } else {
                        const int cb = lvBase[Lv + 1], cper = per * 2;
                        for (int k = 0; k < 4; k++) splitJ = sat_add(splitJ, node[cb + (ny * 2 + (k >> 1)) * cper + nx * 2 + (k & 1)].J);
                    }
                    i64 best = INF;
                    int bp = AV1G_PARTITION_SPLIT;
                    auto consider = [&](int p, i64 J, i64 bits) {
                        const i64 t = sat_add(J, lam * bits);
                        if (t < best) { best = t; bp = p; }
                    };
                    if (hasRows && hasCols) {
                        const int *pb = T->avgPart[bsl];
                        consider(AV1G_PARTITION_SPLIT, splitJ, pb[AV1G_PARTITION_SPLIT]);
                        const int hz = sub_bsize(AV1G_PARTITION_HORZ, n), vt = sub_bsize(AV1G_PARTITION_VERT, n);
                        const int sp = sub_bsize(AV1G_PARTITION_SPLIT, n);
                        if (pmask & (1 << AV1G_PARTITION_NONE)) {
                            const i64 jn = dpJ(sq_bsize(n), x, y);
                            if (jn < INF) consider(AV1G_PARTITION_NONE, jn, pb[AV1G_PARTITION_NONE]);
                        }
                        if (pmask & (1 << AV1G_PARTITION_HORZ)) consider(AV1G_PARTITION_HORZ, sat_add(dpJ(hz, x, y), dpJ(hz, x, y + half)), pb[AV1G_PARTITION_HORZ]);
                        if (pmask & (1 << AV1G_PARTITION_VERT)) consider(AV1G_PARTITION_VERT, sat_add(dpJ(vt, x, y), dpJ(vt, x + half, y)), pb[AV1G_PARTITION_VERT]);
                        if (n > 8) {
                            const i64 s00 = dpJ(sp, x, y), s01 = dpJ(sp, x + half, y), s10 = dpJ(sp, x, y + half), s11 = dpJ(sp, x + half, y + half);
                            consider(AV1G_PARTITION_HORZ_A, sat_add(sat_add(s00, s01), dpJ(hz, x, y + half)), pb[AV1G_PARTITION_HORZ_A]);
                            consider(AV1G_PARTITION_HORZ_B, sat_add(sat_add(dpJ(hz, x, y), s10), s11), pb[AV1G_PARTITION_HORZ_B]);
                            consider(AV1G_PARTITION_VERT_A, sat_add(sat_add(s00, s10), dpJ(vt, x + half, y)), pb[AV1G_PARTITION_VERT_A]);
                            consider(AV1G_PARTITION_VERT_B, sat_add(sat_add(dpJ(vt, x, y), s01), s11), pb[AV1G_PARTITION_VERT_B]);
                            const int h4 = sub_bsize(AV1G_PARTITION_HORZ_4, n), v4 = sub_bsize(AV1G_PARTITION_VERT_4, n);
                            i64 Jh = 0, Jv = 0;
                            for (int i = 0; i < 4; i++) if (i < 3 || y + 3 * q4 < FH) Jh = sat_add(Jh, dpJ(h4, x, y + i * q4));
                            consider(AV1G_PARTITION_HORZ_4, Jh, pb[AV1G_PARTITION_HORZ_4]);
                            for (int i = 0; i < 4; i++) if (i < 3 || x + 3 * q4 < FW) Jv = sat_add(Jv, dpJ(v4, x + i * q4, y));
                            consider(AV1G_PARTITION_VERT_4, Jv, pb[AV1G_PARTITION_VERT_4]);
                        }
                    } else if (hasCols) {
                        consider(AV1G_PARTITION_SPLIT, splitJ, 256);
                        consider(AV1G_PARTITION_HORZ, dpJ(sub_bsize(AV1G_PARTITION_HORZ, n), x, y), 256);
                    } else if (hasRows) {
                        consider(AV1G_PARTITION_SPLIT, splitJ, 256);
                        consider(AV1G_PARTITION_VERT, dpJ(sub_bsize(AV1G_PARTITION_VERT, n), x, y), 256);
                    } else {
                        consider(AV1G_PARTITION_SPLIT, splitJ, 0);
                    }
                    nd.J = best;
                    nd.p = bp;
                }
        }
        // leaves in decode order (pre-order walk)
        std::vector<Leaf> &out = leaves[(size_t)sbr * sbCols + sbc];
        out.clear();
        auto leaf = [&](int bs, int x, int y) {
            if (x >= FW || y >= FH) return;
            out.push_back(Leaf{(uint8_t)bs, (uint8_t)((x - sbx) >> 2), (uint8_t)((y - sby) >> 2)});
        };
        int stk[64][3], sp = 0;
        stk[sp][0] = 0; stk[sp][1] = 0; stk[sp][2] = 0; sp++;
        while (sp > 0) {
            sp--;
            const int Lv = stk[sp][0], nx = stk[sp][1], ny = stk[sp][2];
            const int n = 64 >> Lv, half = n >> 1, q4 = n >> 2, per = 1 << Lv;
            const Node &nd = node[lvBase[Lv] + ny * per + nx];
            const int x = sbx + nx * n, y = sby + ny * n;
            if (nd.p < 0) continue;
            const int p = nd.p, sub = sub_bsize(p, n), sp2 = sub_bsize(AV1G_PARTITION_SPLIT, n);
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
    }

    // ---- closed loop of one SB (k_recon.cuh:1692-1808) ----
    struct SbState {
        uint32_t bdm[3][18];   // BlockDecoded: row yy + 1, bit xx + 1 (yy, xx in -1 .. 16)
    };
    static bool bd_at(const SbState &S, int p, int yy, int xx) { return (S.bdm[p][yy + 1] >> (xx + 1)) & 1; }

    // coefficient contexts from the 4x4 maps (spec get_tx_size_context / the reference's txb_ctx, k_recon.cuh:204-238)
    void txb_ctx(int plane, int txSz, int x4, int y4, int bsize, const TileBox &tb, int *skipCtx, int *dcCtx) const {
        const int subX = plane ? ssx : 0, subY = plane ? ssy : 0;
        const int stride = MiCols >> subX, maxX4 = MiCols >> subX, maxY4 = MiRows >> subY;
        const uint8_t *Lv = cLvl[plane].data(), *Dc = cDc[plane].data();
        const bool hasAbove = y4 > ((tb.y0 >> 2) >> subY), hasLeft = x4 > ((tb.x0 >> 2) >> subX);
        const int w = AV1G_T(Tx_Width)[txSz], h = AV1G_T(Tx_Height)[txSz], w4 = w >> 2, h4 = h >> 2;
        bool nzA = false, nzL = false, gtA = false, gtL = false;
        int n2 = 0, n1 = 0;
        for (int k = 0; k < w4; k++)
            if (hasAbove && x4 + k < maxX4) {
                const int la = Lv[(size_t)(y4 - 1) * stride + x4 + k], da = Dc[(size_t)(y4 - 1) * stride + x4 + k];
                if (plane) nzA |= (la | da) != 0; else { nzA |= la != 0; gtA |= la > 3; }
                n2 += da == 2; n1 += da == 1;
            }
        for (int k = 0; k < h4; k++)
            if (hasLeft && y4 + k < maxY4) {
                const int ll = Lv[(size_t)(y4 + k) * stride + x4 - 1], dl = Dc[(size_t)(y4 + k) * stride + x4 - 1];
                if (plane) nzL |= (ll | dl) != 0; else { nzL |= ll != 0; gtL |= ll > 3; }
                n2 += dl == 2; n1 += dl == 1;
            }
        if (plane == 0) {
            const int bw = bw_px(bsize), bh = bh_px(bsize);
            if (bw == w && bh == h) *skipCtx = 0;
            else if (!nzA && !nzL) *skipCtx = 1;
            else if (!nzA || !nzL) *skipCtx = 2 + (gtA || gtL);
            else if (!gtA && !gtL) *skipCtx = 4;
            else if (!gtA || !gtL) *skipCtx = 5;
            else *skipCtx = 6;
        } else {
            const int ub = av1g_uv_bsize(bsize, ssx, ssy);
            *skipCtx = (int)nzA + (int)nzL + 7 + ((bw_px(ub) * bh_px(ub) > w * h) ? 3 : 0);
        }
        const int dcSign = n2 - n1;
        *dcCtx = dcSign < 0 ? 1 : dcSign > 0 ? 2 : 0;
    }

    // exact inverse + reconstruction with the conformance repair (levels halved until conformant, as
    // AV1G_ENC_FIX_RANGE / the reference's cta_inverse_add, k_recon.cuh:140-197); q may change
    void inverse_add(int16_t *q, int txSz, int txType, int plane, Px *dst, int pitch) const {
        const int W = AV1G_T(Tx_Width)[txSz], H = AV1G_T(Tx_Height)[txSz];
        const int n = std::min(W, 32) * std::min(H, 32);
        std::vector<int32_t> dq(n), res((size_t)W * H);
        for (;;) {
            bool nz = false;
            for (int i = 0; i < n; i++) nz |= q[i] != 0;
            if (!nz) return;
            av1g_dequant<BD>(q, dq.data(), txSz, dcQ[plane], acQ[plane], nullptr);
            uint32_t err = 0;
            av1g_inv_txfm2d<BD>(dq.data(), txSz, txType, res.data(), &err);
            if (!err) break;
            for (int i = 0; i < n; i++) q[i] = (int16_t)(q[i] / 2);
        }
        av1g_add_residual<BD>(dst, pitch, res.data(), txSz, txType);
        count(1, fwd2d_ops(txSz, txType) + 6ull * n + 3ull * W * H + (uint64_t)W * H * 4);
    }

    // record a finished tx block: eob, context maps, BlockDecoded, the txb entry (k_recon.cuh:686-730)
    int record_txb(SbState &S, std::vector<TxbOut> &out, const int16_t *q, int plane, int txSz, int txType, int x4, int y4,
                   int sbr4, int sbc4) {
        const int W = AV1G_T(Tx_Width)[txSz], H = AV1G_T(Tx_Height)[txSz];
        const int n = std::min(W, 32) * std::min(H, 32);
        const uint16_t *scan = av1g_get_scan(txSz, txType);
        int eob = 0;
        for (int c = 0; c < n; c++) if (q[scan[c]]) eob = c + 1;
        int cul = 0;
        for (int c = 0; c < eob; c++) cul += std::abs((int)q[scan[c]]);
        cul = std::min(cul, 63);
        const int dcCat = q[0] < 0 ? 1 : q[0] > 0 ? 2 : 0;
        const int subX = plane ? ssx : 0, subY = plane ? ssy : 0;
        const int stride = MiCols >> subX, rows = MiRows >> subY;
        for (int yy = y4; yy < y4 + (H >> 2); yy++)
            for (int xx = x4; xx < x4 + (W >> 2); xx++)
                if (yy < rows && xx < stride) {
                    cLvl[plane][(size_t)yy * stride + xx] = (uint8_t)(eob ? cul : 0);
                    cDc[plane][(size_t)yy * stride + xx] = (uint8_t)(eob ? dcCat : 0);
                }
        for (int r = 0; r < (H >> 2); r++)
            for (int c = 0; c < (W >> 2); c++) S.bdm[plane][sbr4 + r + 1] |= 1u << (sbc4 + c + 1);
        TxbOut t;
        memset(&t.t, 0, sizeof t.t);
        t.t.x4 = (uint16_t)x4; t.t.y4 = (uint16_t)y4;
        t.t.plane = (uint8_t)plane; t.t.tx_size = (uint8_t)txSz;
        t.t.tx_type = (uint8_t)(plane == 0 && eob == 0 ? AV1G_DCT_DCT : txType);
        t.t.eob = (uint16_t)eob;
        t.q.assign(q, q + n);
        out.push_back(std::move(t));
        return eob;
    }

    void closed_loop_sb(int sbr, int sbc) {
        const int sbx = sbc * 64, sby = sbr * 64;
        const TileBox tb = tile_of(sbx, sby);
        const int miRowEnd = tb.y1 >> 2, miColEnd = tb.x1 >> 2;
        SbState S;
        for (int p = 0; p < 3; p++) {   // clear_block_decoded_flags (spec)
            const int subX = p ? ssx : 0, subY = p ? ssy : 0;
            const int sbW4 = (miColEnd - sbc * 16) >> subX, sbH4 = (miRowEnd - sbr * 16) >> subY;
            for (int yy = -1; yy <= 16; yy++) {
                uint32_t w = 0;
                for (int xx = -1; xx <= 16; xx++) {
                    int v = (yy < 0 && xx < sbW4) ? 1 : (xx < 0 && yy < sbH4) ? 1 : 0;
                    if (yy == (16 >> subY) && xx == -1) v = 0;
                    w |= (uint32_t)v << (xx + 1);
                }
                S.bdm[p][yy + 1] = w;
            }
        }
        SbOut &so = sbo[(size_t)sbr * sbCols + sbc];
        so.blocks.clear();
        so.txb.clear();
        const std::vector<Leaf> &lv = leaves[(size_t)sbr * sbCols + sbc];
        for (const Leaf &lf : lv) {
            const int bsize = lf.bsize, x = sbx + lf.x4 * 4, y = sby + lf.y4 * 4;
            const int mi_row = y >> 2, mi_col = x >> 2;
            int availU, availL, availUC, availLC;
            av1g_block_avail(bsize, mi_row, mi_col, 0, ssx, ssy, tb.y0 >> 2, miRowEnd, tb.x0 >> 2, miColEnd, &availU, &availL, &availUC, &availLC);
            const int hasChroma = av1g_has_chroma(bsize, mi_row, mi_col, 0, ssx, ssy);
            so.txb.emplace_back();
            std::vector<TxbOut> &txbs = so.txb.back();
            int yMode = 0, yDelta = 0, eobY = 0;
            luma(S, txbs, bsize, x, y, availU, availL, tb, &yMode, &yDelta, &eobY);
            int uv = 0, duv = 0, aU = 0, aV = 0, eobU = 0, eobV = 0;
            if (hasChroma) chroma(S, txbs, bsize, mi_row, mi_col, yMode, availUC, availLC, tb, &uv, &duv, &aU, &aV, &eobU, &eobV);
            const int skip = (eobY == 0 && eobU == 0 && eobV == 0) ? 1 : 0;
            for (int r = mi_row; r < mi_row + av1g_bh4(bsize) && r < MiRows; r++)
                for (int c = mi_col; c < mi_col + av1g_bw4(bsize) && c < MiCols; c++) {
                    mYMode[(size_t)r * MiCols + c] = (uint8_t)yMode;
                    if (hasChroma) mUVMode[(size_t)r * MiCols + c] = (uint8_t)uv;
                }
            av1g_block b;
            memset(&b, 0, sizeof b);
            b.mi_row = (uint16_t)mi_row; b.mi_col = (uint16_t)mi_col;
            b.bsize = (uint8_t)bsize; b.skip = (uint8_t)skip; b.tx_depth = 0;
            b.y_mode = (uint8_t)yMode;
            b.angle_delta_y = (int8_t)(bsize >= AV1G_BLOCK_8X8 && av1g_is_directional(yMode) ? yDelta : 0);
            b.uv_mode = (uint8_t)(hasChroma ? uv : 0);
            b.angle_delta_uv = (int8_t)(hasChroma && bsize >= AV1G_BLOCK_8X8 && av1g_is_directional(uv) ? duv : 0);
            b.cfl_alpha_u = (int8_t)aU; b.cfl_alpha_v = (int8_t)aV;
            so.blocks.push_back(b);
        }
    }

    // build the edges of a tx block from the reconstruction (luma or chroma plane units)
    void rec_edges(int plane, int px, int py, int lw, int lh, int haveL, int haveA, int haveAR, int haveBL, Px *A, Px *L) const {
        const int maxX = ((MiCols * 4) >> (plane ? ssx : 0)) - 1, maxY = ((MiRows * 4) >> (plane ? ssy : 0)) - 1;
        av1g_build_edges<BD>(rec[plane].data(), pw[plane], px, py, lw, lh, haveL, haveA, haveAR, haveBL, maxX, maxY, A, L);
    }
    // prediction of a tx block at plane position (px, py): av1core's plain predictor, or with the edge-filter switch its
    // predictor with the intra edge filter (on copies of the edges, which it filters in place)
    void predictx(int plane, int mode, int delta, int haveL, int haveA, int lw, int lh, int px, int py, int filterType, const Px *A,
                  const Px *L, Px *dst, int stride) const {
        if (!g_edgeFilter) { av1g_predict_intra<BD>(mode, delta, haveL, haveA, lw, lh, A, L, dst, stride); return; }
        Px ea[AV1G_EDGE_LEN], el[AV1G_EDGE_LEN];
        memcpy(ea, A - AV1G_EDGE_OFF, sizeof ea);
        memcpy(el, L - AV1G_EDGE_OFF, sizeof el);
        const int maxX = ((MiCols * 4) >> (plane ? ssx : 0)) - 1, maxY = ((MiRows * 4) >> (plane ? ssy : 0)) - 1;
        av1g_predict_intra_ex<BD>(mode, delta, -1, 1, filterType, haveL, haveA, lw, lh, px, py, maxX, maxY, ea + AV1G_EDGE_OFF,
                                  el + AV1G_EDGE_OFF, dst, stride);
    }
    int filter_type(int plane, int mi_row, int mi_col, int availU, int availL) const {
        return av1g_get_filter_type(plane, mi_row, mi_col, availU, availL, mYMode.data(), mUVMode.data(), MiCols, ssx, ssy);
    }
    // the same from the source planes (the open-loop chroma screening of the experiment switch)
    void src_edges(int plane, int px, int py, int lw, int lh, int haveL, int haveA, int haveAR, int haveBL, Px *A, Px *L) const {
        const int maxX = ((MiCols * 4) >> (plane ? ssx : 0)) - 1, maxY = ((MiRows * 4) >> (plane ? ssy : 0)) - 1;
        av1g_build_edges<BD>(src[plane].data(), pw[plane], px, py, lw, lh, haveL, haveA, haveAR, haveBL, maxX, maxY, A, L);
    }

    // ---- luma of one block (k_recon.cuh:822-1214, tx_depth 0) ----
    void luma(SbState &S, std::vector<TxbOut> &txbs, int bsize, int x, int y, int availU, int availL, const TileBox &tb, int *outMode,
              int *outDelta, int *outEob) {
        const int txSz = AV1G_T(Max_Tx_Size_Rect)[bsize];
        const int Wt = AV1G_T(Tx_Width)[txSz], Ht = AV1G_T(Tx_Height)[txSz], lw = log2i(Wt), lh = log2i(Ht);
        const int sbr4 = (y >> 2) & 15, sbc4 = (x >> 2) & 15;
        const int haveAR = bd_at(S, 0, sbr4 - 1, sbc4 + (Wt >> 2)), haveBL = bd_at(S, 0, sbr4 + (Ht >> 2), sbc4 - 1);
        Px ea[AV1G_EDGE_LEN], el[AV1G_EDGE_LEN];
        Px *A = ea + AV1G_EDGE_OFF, *L = el + AV1G_EDGE_OFF;
        rec_edges(0, x, y, lw, lh, availL, availU, haveAR, haveBL, A, L);
        const BlockRes &br = blk[bsize][(size_t)(y / Ht) * shNbx[bsize] + x / Wt];
        int skipCtx, dcCtx;
        txb_ctx(0, txSz, x >> 2, y >> 2, bsize, tb, &skipCtx, &dcCtx);
        const int mi_row = y >> 2, mi_col = x >> 2;
        const int am = AV1G_T(Intra_Mode_Context)[availU ? mYMode[(size_t)(mi_row - 1) * MiCols + mi_col] : AV1G_DC_PRED];
        const int lm = AV1G_T(Intra_Mode_Context)[availL ? mYMode[(size_t)mi_row * MiCols + mi_col - 1] : AV1G_DC_PRED];
        auto mbits = [&](int c) -> i64 {
            const int m = cand_mode(c);
            i64 b = C[COFF(y_mode[am][lm]) + m];
            if (bsize >= AV1G_BLOCK_8X8 && av1g_is_directional(m)) b += C[COFF(angle_delta[m - AV1G_V_PRED]) + cand_delta(c) + 3];
            return b;
        };
        const int sp = pw[0];
        const Px *s = src[0].data() + (size_t)y * sp + x;
        const int set = av1g_get_tx_set_intra(txSz, 0);
        std::vector<Px> pred((size_t)Wt * Ht);
        std::vector<int32_t> res((size_t)Wt * Ht);
        const int fType = g_edgeFilter ? filter_type(0, mi_row, mi_col, availU, availL) : 0;
        auto residual = [&](int c) -> i64 {
            predictx(0, cand_mode(c), cand_delta(c), availL, availU, lw, lh, x, y, fType, A, L, pred.data(), Wt);
            i64 e = 0;
            for (int i = 0; i < Ht; i++)
                for (int j = 0; j < Wt; j++) {
                    const int r = (int)s[i * sp + j] - (int)pred[(size_t)i * Wt + j];
                    res[(size_t)i * Wt + j] = r;
                    e += (i64)r * r;
                }
            return e;
        };
        struct Task { int c, t; };
        std::vector<Task> tasks;
        const int nc = std::max(1, std::min((int)br.ncand, K_RECHECK));
        const bool pass2 = set != AV1G_TX_SET_DCTONLY;
        int bestC = br.cand[0], bestT = br.tx;
        i64 bestJ = INF;
        int16_t q[1024], bestQ[1024];
        bool have = false;
        auto run = [&](const std::vector<Task> &ts) {
            for (const Task &tk : ts) {
                const i64 e = residual(tk.c);
                const EvalOut o = eval(res.data(), txSz, tk.t, 0, skipCtx, dcCtx, cand_mode(tk.c), e, q, 1, cand_mode(tk.c), cand_delta(tk.c));
                const i64 J = o.D + lam * (o.R + mbits(tk.c));
                if (J < bestJ) {
                    bestJ = J; bestC = tk.c; bestT = tk.t; have = true;
                    memcpy(bestQ, q, sizeof q);
                }
            }
        };
        // pass 1: the re-checked candidates with DCT_DCT (+ the analysis winner with its tx type)
        for (int k = 0; k < nc; k++) tasks.push_back(Task{br.cand[k], AV1G_DCT_DCT});
        if (br.tx != AV1G_DCT_DCT) tasks.push_back(Task{br.cand[0], br.tx});
        const bool skip1 = tasks.size() == 1;
        if (!skip1) run(tasks);
        else { bestC = tasks[0].c; bestT = tasks[0].t; }
        // pass 2: the tx types of the winner
        if (pass2) {
            std::vector<Task> t2;
            for (int t = 0; t < 16; t++) {
                if (!av1g_tx_type_in_set_intra(set, t)) continue;
                if (!skip1 && (t == AV1G_DCT_DCT || (bestC == br.cand[0] && t == br.tx))) continue;
                t2.push_back(Task{bestC, t});
            }
            run(t2);
        }
        if (!have) {   // a single candidate, DCT only: its levels
            const i64 e = residual(bestC);
            eval(res.data(), txSz, bestT, 0, skipCtx, dcCtx, cand_mode(bestC), e, bestQ, 1, cand_mode(bestC), cand_delta(bestC));
        }
        // final: prediction + exact inverse into the reconstruction, record
        Px *dst = rec[0].data() + (size_t)y * pw[0] + x;
        predictx(0, cand_mode(bestC), cand_delta(bestC), availL, availU, lw, lh, x, y, fType, A, L, dst, pw[0]);
        inverse_add(bestQ, txSz, bestT, 0, dst, pw[0]);
        *outEob = record_txb(S, txbs, bestQ, 0, txSz, bestT, x >> 2, y >> 2, sbr4, sbc4);
        *outMode = cand_mode(bestC);
        *outDelta = cand_delta(bestC);
    }

    // ---- chroma of one block (k_recon.cuh:1220-1686) ----
    void chroma(SbState &S, std::vector<TxbOut> &txbs, int bsize, int mi_row, int mi_col, int yMode, int availUC, int availLC,
                const TileBox &tb, int *outUv, int *outDuv, int *outAu, int *outAv, int *outEobU, int *outEobV) {
        const int txSz = av1g_uv_tx_size(bsize, ssx, ssy);
        const int Wt = AV1G_T(Tx_Width)[txSz], Ht = AV1G_T(Tx_Height)[txSz], lw = log2i(Wt), lh = log2i(Ht);
        const int cx = (mi_col >> ssx) * 4, cy = (mi_row >> ssy) * 4;
        const int x4 = cx >> 2, y4 = cy >> 2;
        const int sbr4 = (mi_row & 15) >> ssy, sbc4 = (mi_col & 15) >> ssx;
        Px ea[3][AV1G_EDGE_LEN], el[3][AV1G_EDGE_LEN], oa[3][AV1G_EDGE_LEN], ol[3][AV1G_EDGE_LEN];
        Px *A[3], *L[3], *OA[3], *OL[3];   // OA / OL: the screening's edges (the source's with the experiment switch)
        int dcv[3];
        for (int pl = 1; pl <= 2; pl++) {
            A[pl] = ea[pl] + AV1G_EDGE_OFF; L[pl] = el[pl] + AV1G_EDGE_OFF;
            const int haveAR = bd_at(S, pl, sbr4 - 1, sbc4 + (Wt >> 2)), haveBL = bd_at(S, pl, sbr4 + (Ht >> 2), sbc4 - 1);
            rec_edges(pl, cx, cy, lw, lh, availLC, availUC, haveAR, haveBL, A[pl], L[pl]);
            dcv[pl] = av1g_dc_value<BD>(A[pl], L[pl], availLC, availUC, lw, lh);
            OA[pl] = A[pl]; OL[pl] = L[pl];
            if (g_uvOpenLoop) {
                OA[pl] = oa[pl] + AV1G_EDGE_OFF; OL[pl] = ol[pl] + AV1G_EDGE_OFF;
                src_edges(pl, cx, cy, lw, lh, availLC, availUC, haveAR, haveBL, OA[pl], OL[pl]);
            }
        }
        const int fTypeC = g_edgeFilter ? filter_type(1, mi_row, mi_col, availUC, availLC) : 0;
        const Px *sU = src[1].data() + (size_t)cy * pw[1] + cx, *sV = src[2].data() + (size_t)cy * pw[2] + cx;
        const Px *sP[3] = {nullptr, sU, sV};
        const int spP[3] = {0, pw[1], pw[2]};
        const bool cflAllowed = av1g_cfl_allowed(bsize);
        auto uvbits = [&](int m) -> i64 {
            return cflAllowed ? C[COFF(uv_mode_cfl_allowed[yMode]) + m] : C[COFF(uv_mode_cfl_not_allowed[yMode]) + m];
        };
        auto uvcbits = [&](int c) -> i64 {
            const int m = cand_mode(c);
            i64 b = uvbits(m);
            if (bsize >= AV1G_BLOCK_8X8 && av1g_is_directional(m)) b += C[COFF(angle_delta[m - AV1G_V_PRED]) + cand_delta(c) + 3];
            return b;
        };
        const int npx = Wt * Ht;
        // ---- CfL: luma values from the reconstruction (spec 7.11.5), least-squares alpha, +-1 refinement ----
        std::vector<int> cflL(npx);
        int cflAvg = 0, alpha[3] = {0, 0, 0};
        if (cflAllowed) {
            const int lumaTx = av1g_luma_tx_size(bsize, 0);
            const int tw = AV1G_T(Tx_Width)[lumaTx], th = AV1G_T(Tx_Height)[lumaTx];
            int maxLumaW = 0, maxLumaH = 0;
            for (int ly = mi_row * 4; ly < mi_row * 4 + bh_px(bsize); ly += th)
                for (int lx = mi_col * 4; lx < mi_col * 4 + bw_px(bsize); lx += tw)
                    if (lx < MiCols * 4 && ly < MiRows * 4) { maxLumaW = lx + tw; maxLumaH = ly + th; }
            const Px *luma = rec[0].data();
            const int lp = pw[0];
            i64 sum = 0;
            for (int i = 0; i < Ht; i++)
                for (int j = 0; j < Wt; j++) {
                    int v;
                    if (ssx) {
                        int lumaY = (cy + i) << 1, lumaX = (cx + j) << 1;
                        if (lumaY > maxLumaH - 2) lumaY = maxLumaH - 2;
                        if (lumaX > maxLumaW - 2) lumaX = maxLumaW - 2;
                        v = (luma[(size_t)lumaY * lp + lumaX] + luma[(size_t)lumaY * lp + lumaX + 1] + luma[(size_t)(lumaY + 1) * lp + lumaX] +
                             luma[(size_t)(lumaY + 1) * lp + lumaX + 1]) << 1;
                    } else {
                        const int lumaY = std::min(cy + i, maxLumaH - 1), lumaX = std::min(cx + j, maxLumaW - 1);
                        v = luma[(size_t)lumaY * lp + lumaX] << 3;
                    }
                    cflL[i * Wt + j] = v;
                    sum += v;
                }
            cflAvg = (int)((sum + ((i64)1 << (lw + lh - 1))) >> (lw + lh));
            count(1, (uint64_t)npx * (8 + 8 + 2 * 3 * 9));
            i64 den = 0, num[3] = {0, 0, 0};
            for (int i = 0; i < Ht; i++)
                for (int j = 0; j < Wt; j++) {
                    const i64 l = cflL[i * Wt + j] - cflAvg;
                    for (int pl = 1; pl <= 2; pl++) num[pl] += l * ((int)sP[pl][i * spP[pl] + j] - dcv[pl]);
                    den += l * l;
                }
            for (int pl = 1; pl <= 2; pl++) {
                int a = 0;
                if (den > 0) {   // round(64 num / den), halves away from zero
                    const i64 n = 64 * num[pl];
                    a = (int)(n >= 0 ? (2 * n + den) / (2 * den) : -((-2 * n + den) / (2 * den)));
                }
                a = std::max(-16, std::min(16, a));
                i64 sse[3] = {0, 0, 0};
                for (int k = 0; k < 3; k++) {
                    const int ak = std::max(-16, std::min(16, a + k - 1));
                    for (int i = 0; i < Ht; i++)
                        for (int j = 0; j < Wt; j++) {
                            const int pr = av1g_clip1<BD>(dcv[pl] + av1g_round2signed(ak * (cflL[i * Wt + j] - cflAvg), 6));
                            const i64 d = (int)sP[pl][i * spP[pl] + j] - pr;
                            sse[k] += d * d;
                        }
                }
                int bk = 1;
                for (int k = 0; k < 3; k++) if (sse[k] < sse[bk]) bk = k;
                alpha[pl] = std::max(-16, std::min(16, a + bk - 1));
            }
        }
        // ---- SATD screening of the 13 UV modes (U + V), then +-1..3 around the best directional one ----
        std::vector<Px> pred((size_t)npx);
        int uvc[32];
        i64 satd[32];
        for (int m = 0; m < 13; m++) uvc[m] = cand_pack(m, 0);
        int nuv = 13;
        const i64 lamS = sqlam;
        auto screen = [&](int c0, int c1) {
            for (int ci = c0; ci < c1; ci++) {
                i64 t = 0;
                for (int pl = 1; pl <= 2; pl++) {
                    predictx(pl, cand_mode(uvc[ci]), cand_delta(uvc[ci]), availLC, availUC, lw, lh, cx, cy, fTypeC, OA[pl], OL[pl], pred.data(), Wt);
                    for (int sy = 0; sy < Ht; sy += 4)
                        for (int sx = 0; sx < Wt; sx += 4) {
                            int d[16];
                            for (int i = 0; i < 4; i++)
                                for (int j = 0; j < 4; j++)
                                    d[i * 4 + j] = (int)sP[pl][(sy + i) * spP[pl] + sx + j] - (int)pred[(size_t)(sy + i) * Wt + sx + j];
                            t += hadamard4_sum(d);
                        }
                }
                satd[ci] = t << 14;
                count(g_uvOpenLoop ? 0 : 1, 2 * (uint64_t)(npx / 16) * (16 * (uint64_t)pred_ops(cand_mode(uvc[ci]), cand_delta(uvc[ci])) + 111) + 30);
            }
        };
        screen(0, 13);
        if (bsize >= AV1G_BLOCK_8X8) {
            int bm = -1;
            i64 bj = INF;
            for (int m = AV1G_V_PRED; m <= AV1G_D67_PRED; m++) {
                const i64 j = satd[m] + lamS * uvcbits(uvc[m]);
                if (j < bj) { bj = j; bm = m; }
            }
            for (int k = 0; k < 6; k++) uvc[13 + k] = cand_pack(bm, k < 3 ? -(k + 1) : (k - 2));
            nuv = 19;
            screen(13, 19);
        }
        // top uvK by SATD cost, then CfL
        std::vector<int> chosen;
        {
            bool used[32] = {false};
            for (int k = 0; k < UV_K; k++) {
                int b = -1;
                i64 bj = INF;
                for (int i = 0; i < nuv; i++) {
                    if (used[i]) continue;
                    const i64 j = satd[i] + lamS * uvcbits(uvc[i]);
                    if (j < bj) { bj = j; b = i; }
                }
                if (b < 0) break;
                used[b] = true;
                chosen.push_back(uvc[b]);
            }
        }
        const bool cflTask = cflAllowed && (alpha[1] || alpha[2]);
        if (cflTask) chosen.push_back(255);
        int skipCtx[3], dcCtx[3];
        for (int pl = 1; pl <= 2; pl++) txb_ctx(pl, txSz, x4, y4, bsize, tb, &skipCtx[pl], &dcCtx[pl]);
        std::vector<int32_t> res((size_t)npx);
        auto residual = [&](int pl, int c) {
            if (c == 255) {
                for (int i = 0; i < Ht; i++)
                    for (int j = 0; j < Wt; j++) {
                        const int pr = av1g_clip1<BD>(dcv[pl] + av1g_round2signed(alpha[pl] * (cflL[i * Wt + j] - cflAvg), 6));
                        res[(size_t)i * Wt + j] = (int)sP[pl][i * spP[pl] + j] - pr;
                    }
                return;
            }
            predictx(pl, cand_mode(c), cand_delta(c), availLC, availUC, lw, lh, cx, cy, fTypeC, A[pl], L[pl], pred.data(), Wt);
            for (int i = 0; i < Ht; i++)
                for (int j = 0; j < Wt; j++) res[(size_t)i * Wt + j] = (int)sP[pl][i * spP[pl] + j] - (int)pred[(size_t)i * Wt + j];
        };
        i64 bJ = INF;
        int bestC = cand_pack(AV1G_DC_PRED, 0);
        int16_t q[1024], bestQ[3][1024];
        for (int c : chosen) {
            const int mode = c == 255 ? AV1G_UV_CFL_PRED : cand_mode(c);
            const int txType = av1g_chroma_tx_type(txSz, mode, 0);
            i64 J = 0;
            int16_t qq[3][1024];
            for (int pl = 1; pl <= 2; pl++) {
                residual(pl, c);
                const EvalOut o = eval(res.data(), txSz, txType, pl, skipCtx[pl], dcCtx[pl], 0, 0, q, 1, c == 255 ? AV1G_SMOOTH_V_PRED : cand_mode(c),
                                       c == 255 ? 0 : cand_delta(c));
                J += o.D + lam * o.R;
                memcpy(qq[pl], q, sizeof q);
            }
            i64 b;
            if (c == 255) {
                const int a1 = alpha[1], a2 = alpha[2];
                const int sU = a1 == 0 ? 0 : a1 < 0 ? 1 : 2, sV = a2 == 0 ? 0 : a2 < 0 ? 1 : 2;
                b = uvbits(AV1G_UV_CFL_PRED) + C[COFF(cfl_sign) + sU * 3 + sV - 1];
                if (sU) b += C[COFF(cfl_alpha[(sU - 1) * 3 + sV]) + std::abs(a1) - 1];
                if (sV) b += C[COFF(cfl_alpha[(sV - 1) * 3 + sU]) + std::abs(a2) - 1];
            } else {
                b = uvcbits(c);
            }
            J += lam * b;
            if (J < bJ) {
                bJ = J; bestC = c;
                memcpy(bestQ[1], qq[1], sizeof q); memcpy(bestQ[2], qq[2], sizeof q);
            }
        }
        const bool cfl = bestC == 255;
        const int bestUv = cfl ? AV1G_UV_CFL_PRED : cand_mode(bestC);
        const int uvTxType = av1g_chroma_tx_type(txSz, bestUv, 0);
        // chroma tx blocks per plane (k_recon.cuh:1588-1680): one in 4:2:0 and in 4:4:4 up to 32x32; 2 or 4 in raster
        // order for a 4:4:4 block with a 64-sample side, the mode chosen on the first.  A further tx block takes its
        // edges from the reconstruction (the block's earlier tx blocks included), its own coefficient contexts and a
        // closed-loop quantisation of the chosen mode; tx blocks that start outside the coded area are not coded.
        const int ub = av1g_uv_bsize(bsize, ssx, ssy);
        const int nTxX = ssx ? 1 : std::max(1, bw_px(ub) / Wt), nTxY = ssy ? 1 : std::max(1, bh_px(ub) / Ht);
        const int cCols4 = MiCols >> ssx, cRows4 = MiRows >> ssy;
        int eobs[3] = {0, 0, 0};
        for (int pl = 1; pl <= 2; pl++) {
            Px *dst = rec[pl].data() + (size_t)cy * pw[pl] + cx;
            if (cfl) {
                for (int i = 0; i < Ht; i++)
                    for (int j = 0; j < Wt; j++)
                        dst[(size_t)i * pw[pl] + j] = (Px)av1g_clip1<BD>(dcv[pl] + av1g_round2signed(alpha[pl] * (cflL[i * Wt + j] - cflAvg), 6));
            } else {
                predictx(pl, cand_mode(bestC), cand_delta(bestC), availLC, availUC, lw, lh, cx, cy, fTypeC, A[pl], L[pl], dst, pw[pl]);
            }
            inverse_add(bestQ[pl], txSz, uvTxType, pl, dst, pw[pl]);
            eobs[pl] = record_txb(S, txbs, bestQ[pl], pl, txSz, uvTxType, x4, y4, sbr4, sbc4);
            for (int ty = 0; ty < nTxY; ty++)
                for (int tx = 0; tx < nTxX; tx++) {
                    if (tx == 0 && ty == 0) continue;
                    const int ox = tx * Wt, oy = ty * Ht;
                    if (x4 + (ox >> 2) >= cCols4 || y4 + (oy >> 2) >= cRows4) continue;
                    const int r4 = sbr4 + (oy >> 2), c4 = sbc4 + (ox >> 2);
                    const int haveL = availLC || tx > 0, haveA = availUC || ty > 0;
                    const int haveAR = bd_at(S, pl, r4 - 1, c4 + (Wt >> 2)), haveBL = bd_at(S, pl, r4 + (Ht >> 2), c4 - 1);
                    Px ea2[AV1G_EDGE_LEN], el2[AV1G_EDGE_LEN];
                    Px *A2 = ea2 + AV1G_EDGE_OFF, *L2 = el2 + AV1G_EDGE_OFF;
                    rec_edges(pl, cx + ox, cy + oy, lw, lh, haveL, haveA, haveAR, haveBL, A2, L2);
                    int sc, dc;
                    txb_ctx(pl, txSz, x4 + (ox >> 2), y4 + (oy >> 2), bsize, tb, &sc, &dc);
                    Px *d2 = rec[pl].data() + (size_t)(cy + oy) * pw[pl] + cx + ox;
                    predictx(pl, cand_mode(bestC), cand_delta(bestC), haveL, haveA, lw, lh, cx + ox, cy + oy, fTypeC, A2, L2, d2, pw[pl]);
                    const Px *s2 = sP[pl] + (size_t)oy * spP[pl] + ox;
                    for (int i = 0; i < Ht; i++)
                        for (int j = 0; j < Wt; j++) res[(size_t)i * Wt + j] = (int)s2[(size_t)i * spP[pl] + j] - (int)d2[(size_t)i * pw[pl] + j];
                    int16_t q2[1024];
                    eval(res.data(), txSz, uvTxType, pl, sc, dc, 0, 0, q2, 1, cand_mode(bestC), cand_delta(bestC));
                    inverse_add(q2, txSz, uvTxType, pl, d2, pw[pl]);
                    eobs[pl] |= record_txb(S, txbs, q2, pl, txSz, uvTxType, x4 + (ox >> 2), y4 + (oy >> 2), r4, c4);
                }
        }
        *outUv = bestUv;
        *outDuv = cfl ? 0 : cand_delta(bestC);
        *outAu = cfl ? alpha[1] : 0;
        *outAv = cfl ? alpha[2] : 0;
        *outEobU = eobs[1];
        *outEobV = eobs[2];
    }

    // ---- whole image ----
    void run(int threads) {
        threads = std::max(1, threads);
        auto par = [&](size_t n, const std::function<void(size_t)> &fn) {
            std::atomic<size_t> next{0};
            auto work = [&] { for (;;) { const size_t i = next.fetch_add(1); if (i >= n) break; fn(i); } };
            std::vector<std::thread> th;
            for (int t = 1; t < threads; t++) th.emplace_back(work);
            work();
            for (auto &t : th) t.join();
        };
        // analysis: every shape, every position (rows of blocks as work items)
        std::vector<std::pair<int, int>> rows;
        for (int s = 0; s < 22; s++) for (int r = 0; r < shNby[s]; r++) rows.emplace_back(s, r);
        par(rows.size(), [&](size_t i) {
            const int s = rows[i].first, r = rows[i].second;
            for (int c = 0; c < shNbx[s]; c++) analyse(s, c, r);
        });
        par((size_t)sbCols * sbRows, [&](size_t i) { dp((int)(i / sbCols), (int)(i % sbCols)); });
        // closed loop: SBs ordered by (tile, wavefront step c + 2 r); each waits for its left and above-right SBs
        struct Job { int r, c, step, tile; };
        std::vector<Job> jobs;
        for (uint32_t tr = 0; tr < tiles.rows; tr++)
            for (uint32_t tc = 0; tc < tiles.cols; tc++) {
                const int r0 = tiles.mi_row_starts[tr] >> 4, r1 = (tiles.mi_row_starts[tr + 1] + 15) >> 4;
                const int c0 = tiles.mi_col_starts[tc] >> 4, c1 = (tiles.mi_col_starts[tc + 1] + 15) >> 4;
                for (int r = r0; r < r1; r++)
                    for (int c = c0; c < c1; c++) jobs.push_back(Job{r, c, (c - c0) + 2 * (r - r0), (int)(tr * tiles.cols + tc)});
            }
        std::stable_sort(jobs.begin(), jobs.end(), [](const Job &a, const Job &b) { return a.step < b.step; });
        std::unique_ptr<std::atomic<int>[]> done(new std::atomic<int>[(size_t)sbCols * sbRows]);
        for (size_t i = 0; i < (size_t)sbCols * sbRows; i++) done[i].store(0);
        par(jobs.size(), [&](size_t i) {
            const Job &j = jobs[i];
            const TileBox tb = tile_of(j.c * 64, j.r * 64);
            const int c0 = tb.x0 / 64, r0 = tb.y0 / 64, c1 = (tb.x1 + 63) / 64;
            auto wait = [&](int r, int c) { while (!done[(size_t)r * sbCols + c].load(std::memory_order_acquire)) std::this_thread::yield(); };
            if (j.c > c0) wait(j.r, j.c - 1);
            if (j.r > r0) wait(j.r - 1, std::min(j.c + 1, c1 - 1));
            closed_loop_sb(j.r, j.c);
            done[(size_t)j.r * sbCols + j.c].store(1, std::memory_order_release);
        });
    }
};

}  // namespace orc

// ---------------------------------------------------------------------------------------------------------------
// C API
// ---------------------------------------------------------------------------------------------------------------
struct orc_result {
    int bd = 8, W = 0, H = 0, ssx = 1, ssy = 1;
    av1g_frame_params fp;
    std::vector<av1g_block> blocks;
    std::vector<uint32_t> block_txb;
    std::vector<av1g_txb> txb;
    std::vector<int16_t> coeffs;
    std::vector<uint8_t> recon[3];   // cropped, bytes (8-bit) or uint16 pairs
    std::vector<orc::BlockRes> blk[22];
    std::vector<std::vector<orc::Leaf>> leaves;
    uint64_t ops[2] = {0, 0};
};

template <int BD>
static int encode_bd(const orc_image *img, int threads, orc_result *R) {
    typedef av1g_pixel_t(BD) Px;
    std::unique_ptr<orc::Engine<BD>> E(new orc::Engine<BD>());
    orc::OpCounter cnt;
    cnt.ops[0] = 0;
    cnt.ops[1] = 0;
    E->ops = &cnt;
    E->setup(*img);
    E->run(threads);
    R->ops[0] = cnt.ops[0].load();
    R->ops[1] = cnt.ops[1].load();
    memset(&R->fp, 0, sizeof R->fp);
    R->fp.version = AV1G_DECISIONS_VERSION;
    R->fp.width = (uint32_t)img->width;
    R->fp.height = (uint32_t)img->height;
    R->fp.base_q_idx = (uint8_t)img->qindex;
    R->fp.tile_cols_log2 = -1;
    R->fp.tile_rows_log2 = -1;
    R->fp.qm_y = R->fp.qm_u = R->fp.qm_v = 15;
    R->fp.chroma_format = img->chroma_444 ? AV1G_CHROMA_444 : AV1G_CHROMA_420;
    R->fp.bit_depth = (uint8_t)BD;
    R->bd = BD; R->W = img->width; R->H = img->height; R->ssx = E->ssx; R->ssy = E->ssy;
    // decode order: tiles raster, SBs raster inside the tile, leaves
    const av1g_tiles &t = E->tiles;
    R->block_txb.assign(1, 0);
    for (uint32_t tr = 0; tr < t.rows; tr++)
        for (uint32_t tc = 0; tc < t.cols; tc++)
            for (uint32_t r = t.mi_row_starts[tr]; r < t.mi_row_starts[tr + 1]; r += 16)
                for (uint32_t c = t.mi_col_starts[tc]; c < t.mi_col_starts[tc + 1]; c += 16) {
                    const orc::SbOut &so = E->sbo[(size_t)(r >> 4) * E->sbCols + (c >> 4)];
                    for (size_t b = 0; b < so.blocks.size(); b++) {
                        R->blocks.push_back(so.blocks[b]);
                        for (const orc::TxbOut &x : so.txb[b]) {
                            av1g_txb tt = x.t;
                            tt.coeff_off = (uint32_t)R->coeffs.size();
                            R->txb.push_back(tt);
                            R->coeffs.insert(R->coeffs.end(), x.q.begin(), x.q.end());
                        }
                        R->block_txb.push_back((uint32_t)R->txb.size());
                    }
                }
    for (int p = 0; p < 3; p++) {
        const int sx = p ? E->ssx : 0, sy = p ? E->ssy : 0;
        const int w = (img->width + sx) >> sx, h = (img->height + sy) >> sy;
        R->recon[p].assign((size_t)w * h * sizeof(Px), 0);
        Px *d = (Px *)R->recon[p].data();
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) d[(size_t)y * w + x] = E->rec[p][(size_t)y * E->pw[p] + x];
    }
    for (int s = 0; s < 22; s++) R->blk[s] = E->blk[s];
    R->leaves = E->leaves;
    return 0;
}

extern "C" {

int orc_encode(const orc_image *img, int threads, orc_result **out) {
    if (!img || !out || img->width < 1 || img->height < 1 || img->qindex < 1 || img->qindex > 255) return -1;
    if (img->bit_depth != 8 && img->bit_depth != 10) return -1;
    orc_result *R = new orc_result();
    const int rc = img->bit_depth == 8 ? encode_bd<8>(img, threads, R) : encode_bd<10>(img, threads, R);
    if (rc) { delete R; return rc; }
    *out = R;
    return 0;
}

void orc_free(orc_result *r) { delete r; }

void orc_counts(const orc_result *r, uint32_t *nb, uint32_t *nt, uint64_t *nc) {
    if (nb) *nb = (uint32_t)r->blocks.size();
    if (nt) *nt = (uint32_t)r->txb.size();
    if (nc) *nc = r->coeffs.size();
}

void orc_copy_record(const orc_result *r, av1g_frame_params *fp, av1g_block *blocks, uint32_t *block_txb, av1g_txb *txb, int16_t *coeffs) {
    if (fp) *fp = r->fp;
    if (blocks) memcpy(blocks, r->blocks.data(), r->blocks.size() * sizeof(av1g_block));
    if (block_txb) memcpy(block_txb, r->block_txb.data(), r->block_txb.size() * sizeof(uint32_t));
    if (txb) memcpy(txb, r->txb.data(), r->txb.size() * sizeof(av1g_txb));
    if (coeffs) memcpy(coeffs, r->coeffs.data(), r->coeffs.size() * sizeof(int16_t));
}

void orc_copy_recon(const orc_result *r, int p, void *dst) { memcpy(dst, r->recon[p].data(), r->recon[p].size()); }

uint32_t orc_analysis(const orc_result *r, int bs, int64_t *J, uint8_t *cand, uint8_t *ncand, uint8_t *tx) {
    if (bs < 0 || bs >= 22) return 0;
    const auto &v = r->blk[bs];
    for (size_t i = 0; i < v.size(); i++) {
        if (J) J[i] = v[i].J;
        if (cand) memcpy(cand + 4 * i, v[i].cand, 4);
        if (ncand) ncand[i] = v[i].ncand;
        if (tx) tx[i] = v[i].tx;
    }
    return (uint32_t)v.size();
}

int orc_leaves(const orc_result *r, uint32_t sb, uint8_t *bsize, uint8_t *x4, uint8_t *y4) {
    if (sb >= r->leaves.size()) return 0;
    const auto &v = r->leaves[sb];
    for (size_t i = 0; i < v.size(); i++) {
        if (bsize) bsize[i] = v[i].bsize;
        if (x4) x4[i] = v[i].x4;
        if (y4) y4[i] = v[i].y4;
    }
    return (int)v.size();
}

int orc_av1g_recon(av1g_decision_record *rec, void *recon[3], char *err, size_t errlen, uint64_t *obu_bytes) {
    // layout must reproduce the record's own offsets; av1g_layout resets tx_type / eob, so keep copies
    std::vector<av1g_txb> keep(rec->txb, rec->txb + rec->n_txb);
    std::vector<uint32_t> bt(rec->n_blocks + 1);
    std::vector<av1g_txb> lt(rec->n_txb + 1);
    av1g_decision_record L = *rec;
    L.block_txb = bt.data();
    L.txb = lt.data();
    int rc = av1g_layout(&L, (uint32_t)lt.size(), rec->n_coeffs + 1);
    if (rc != AV1G_OK) { if (err) snprintf(err, errlen, "av1g_layout %d", rc); return rc; }
    if (L.n_txb != rec->n_txb || L.n_coeffs != rec->n_coeffs) { if (err) snprintf(err, errlen, "layout counts differ"); return -100; }
    for (uint32_t i = 0; i < rec->n_txb; i++) {
        const av1g_txb &a = lt[i], &b = keep[i];
        if (a.coeff_off != b.coeff_off || a.x4 != b.x4 || a.y4 != b.y4 || a.plane != b.plane || a.tx_size != b.tx_size) {
            if (err) snprintf(err, errlen, "layout of txb %u differs", i);
            return -101;
        }
    }
    for (uint32_t i = 0; i <= rec->n_blocks; i++)
        if (bt[i] != rec->block_txb[i]) { if (err) snprintf(err, errlen, "block_txb %u differs", i); return -102; }
    av1g_encode_opts o = {0, -1};
    av1g_output out;
    memset(&out, 0, sizeof out);
    rc = av1g_encode(rec, &o, &out);
    if (rc != AV1G_OK) { if (err) snprintf(err, errlen, "%s", out.error); av1g_output_free(&out); return rc; }
    for (int p = 0; p < 3; p++)
        if (recon[p] && out.recon[p])
            memcpy(recon[p], out.recon[p], (size_t)out.recon_w[p] * out.recon_h[p] * (rec->fp.bit_depth == 10 ? 2 : 1));
    if (obu_bytes) *obu_bytes = out.obu_size;
    av1g_output_free(&out);
    return 0;
}

void orc_fwd2d(const int32_t *res, int txSz, int txType, int bd, int32_t *coef) { orc::fwd2d(res, txSz, txType, bd, coef); }

uint32_t orc_inv2d(const int16_t *levels, int txSz, int txType, int bd, int dcQ, int acQ, int32_t *res) {
    int32_t dq[1024];
    uint32_t err = 0;
    if (bd == 10) { av1g_dequant<10>(levels, dq, txSz, dcQ, acQ, nullptr); av1g_inv_txfm2d<10>(dq, txSz, txType, res, &err); }
    else { av1g_dequant<8>(levels, dq, txSz, dcQ, acQ, nullptr); av1g_inv_txfm2d<8>(dq, txSz, txType, res, &err); }
    return err;
}

void orc_quant_rate(const int32_t *coef, int txSz, int txType, int plane, int bd, int dcQ, int acQ, int skipCtx, int dcCtx,
                    int intraDir, int qctx, int64_t resEnergy, int16_t *levels, int64_t *D, int64_t *R, int *eob) {
    orc::EvalIn e{txSz, txType, plane, bd, dcQ, acQ, skipCtx, dcCtx, intraDir, orc::tables().cost[qctx].data(), resEnergy};
    orc::EvalOut o;
    orc::quant_rate(coef, e, levels, o);
    *D = o.D; *R = o.R; *eob = o.eob;
}

size_t orc_cost_table(int qctx, uint16_t *out, size_t cap) {
    const auto &v = orc::tables().cost[qctx & 3];
    if (out) memcpy(out, v.data(), std::min(cap, v.size()) * 2);
    return v.size();
}

void orc_avg_bits(int32_t *avgY, int32_t *avgPart, int32_t *avgSkip0) {
    const orc::Tables &T = orc::tables();
    for (int i = 0; i < 13; i++) avgY[i] = T.avgY[i];
    for (int i = 0; i < 50; i++) avgPart[i] = T.avgPart[i / 10][i % 10];
    *avgSkip0 = T.avgSkip0;
}

void orc_lambda(int qindex, int bd, int64_t *lam, int64_t *sqrtlam) { orc::lambda_fx(qindex, bd, lam, sqrtlam); }

void orc_predict(const uint8_t *plane, int stride, int x, int y, int log2W, int log2H, int haveLeft, int haveAbove, int haveAR,
                 int haveBL, int maxX, int maxY, int mode, int delta, uint8_t *dst) {
    uint8_t ea[AV1G_EDGE_LEN], el[AV1G_EDGE_LEN];
    uint8_t *A = ea + AV1G_EDGE_OFF, *L = el + AV1G_EDGE_OFF;
    av1g_build_edges<8>(plane, stride, x, y, log2W, log2H, haveLeft, haveAbove, haveAR, haveBL, maxX, maxY, A, L);
    av1g_predict_intra<8>(mode, delta, haveLeft, haveAbove, log2W, log2H, A, L, dst, 1 << log2W);
}

}  // extern "C"

extern "C" int orc_av1g_recon_arrays(int width, int height, int qindex, int bd, int chroma_444, uint32_t n_blocks, av1g_block *blocks,
                                     uint32_t *block_txb, uint32_t n_txb, av1g_txb *txb, uint64_t n_coeffs, int16_t *coeffs,
                                     void *recon[3], char *err, size_t errlen, uint64_t *obu_bytes) {
    av1g_decision_record rec;
    memset(&rec, 0, sizeof rec);
    rec.fp.version = AV1G_DECISIONS_VERSION;
    rec.fp.width = (uint32_t)width;
    rec.fp.height = (uint32_t)height;
    rec.fp.base_q_idx = (uint8_t)qindex;
    rec.fp.tile_cols_log2 = -1;
    rec.fp.tile_rows_log2 = -1;
    rec.fp.qm_y = rec.fp.qm_u = rec.fp.qm_v = 15;
    rec.fp.chroma_format = chroma_444 ? AV1G_CHROMA_444 : AV1G_CHROMA_420;
    rec.fp.bit_depth = (uint8_t)bd;
    rec.n_blocks = n_blocks;
    rec.blocks = blocks;
    rec.block_txb = block_txb;
    rec.n_txb = n_txb;
    rec.txb = txb;
    rec.n_coeffs = n_coeffs;
    rec.coeffs = coeffs;
    return orc_av1g_recon(&rec, recon, err, errlen, obu_bytes);
}

extern "C" int orc_av1g_obu_fp(const av1g_frame_params *fp, uint32_t n_blocks, av1g_block *blocks, uint32_t *block_txb, uint32_t n_txb,
                               av1g_txb *txb, uint64_t n_coeffs, int16_t *coeffs, uint8_t *obu, uint64_t cap, uint64_t *size,
                               uint32_t *n_tiles, uint64_t *tile_off, uint32_t *tile_bytes, uint32_t tile_cap, uint64_t *n_symbols,
                               char *err, size_t errlen);

// av1g_encode()'s OBU stream of a record (the bitstream only) and, from av1g_parse() of it, where each tile payload lies
extern "C" int orc_av1g_obu_arrays(int width, int height, int qindex, int bd, int chroma_444, uint32_t n_blocks, av1g_block *blocks,
                                   uint32_t *block_txb, uint32_t n_txb, av1g_txb *txb, uint64_t n_coeffs, int16_t *coeffs, uint8_t *obu,
                                   uint64_t cap, uint64_t *size, uint32_t *n_tiles, uint64_t *tile_off, uint32_t *tile_bytes, uint32_t tile_cap,
                                   uint64_t *n_symbols, char *err, size_t errlen) {
    av1g_frame_params fp;
    memset(&fp, 0, sizeof fp);
    fp.version = AV1G_DECISIONS_VERSION;
    fp.width = (uint32_t)width;
    fp.height = (uint32_t)height;
    fp.base_q_idx = (uint8_t)qindex;
    fp.tile_cols_log2 = -1;
    fp.tile_rows_log2 = -1;
    fp.qm_y = fp.qm_u = fp.qm_v = 15;
    fp.chroma_format = chroma_444 ? AV1G_CHROMA_444 : AV1G_CHROMA_420;
    fp.bit_depth = (uint8_t)bd;
    return orc_av1g_obu_fp(&fp, n_blocks, blocks, block_txb, n_txb, txb, n_coeffs, coeffs, obu, cap, size, n_tiles, tile_off, tile_bytes,
                           tile_cap, n_symbols, err, errlen);
}

// the same with the record's frame parameters given (header fields: delta_q, quantizer matrices, loop-filter levels,
// colour description, ...)
extern "C" int orc_av1g_obu_fp(const av1g_frame_params *fp, uint32_t n_blocks, av1g_block *blocks, uint32_t *block_txb, uint32_t n_txb,
                               av1g_txb *txb, uint64_t n_coeffs, int16_t *coeffs, uint8_t *obu, uint64_t cap, uint64_t *size,
                               uint32_t *n_tiles, uint64_t *tile_off, uint32_t *tile_bytes, uint32_t tile_cap, uint64_t *n_symbols,
                               char *err, size_t errlen) {
    av1g_decision_record rec;
    memset(&rec, 0, sizeof rec);
    rec.fp = *fp;
    rec.n_blocks = n_blocks;
    rec.blocks = blocks;
    rec.block_txb = block_txb;
    rec.n_txb = n_txb;
    rec.txb = txb;
    rec.n_coeffs = n_coeffs;
    rec.coeffs = coeffs;
    av1g_encode_opts o = {AV1G_ENC_BITSTREAM_ONLY, -1};
    av1g_output out;
    memset(&out, 0, sizeof out);
    int rc = av1g_encode(&rec, &o, &out);
    if (rc != AV1G_OK) { if (err) snprintf(err, errlen, "%s", out.error); av1g_output_free(&out); return rc; }
    *size = out.obu_size;
    if (n_symbols) *n_symbols = out.n_symbols;
    if (obu && cap >= out.obu_size) memcpy(obu, out.obu, out.obu_size);
    av1g_parsed *ps = nullptr;
    rc = av1g_parse(out.obu, out.obu_size, &ps);
    av1g_output_free(&out);
    if (rc != AV1G_OK) { if (err) snprintf(err, errlen, "av1g_parse %d: %s", rc, ps ? ps->error : ""); av1g_parsed_free(ps); return rc; }
    *n_tiles = ps->n_tiles;
    for (uint32_t i = 0; i < ps->n_tiles && i < tile_cap; i++) { tile_off[i] = ps->tile_offsets[i]; tile_bytes[i] = ps->tile_bytes[i]; }
    av1g_parsed_free(ps);
    return 0;
}

// av1g_encode() of a record with the given frame parameters (e.g. post-filter fields) and flags; its reconstruction
// planes copied out (cropped, or with AV1G_ENC_PREFILTER_RECON the unfiltered coded area)
extern "C" int orc_av1g_encode_fp(const av1g_frame_params *fp, uint32_t flags, uint32_t n_blocks, av1g_block *blocks, uint32_t *block_txb,
                                  uint32_t n_txb, av1g_txb *txb, uint64_t n_coeffs, int16_t *coeffs, void *recon[3], char *err, size_t errlen) {
    av1g_decision_record rec;
    memset(&rec, 0, sizeof rec);
    rec.fp = *fp;
    rec.n_blocks = n_blocks;
    rec.blocks = blocks;
    rec.block_txb = block_txb;
    rec.n_txb = n_txb;
    rec.txb = txb;
    rec.n_coeffs = n_coeffs;
    rec.coeffs = coeffs;
    av1g_encode_opts o = {flags, -1};
    av1g_output out;
    memset(&out, 0, sizeof out);
    const int rc = av1g_encode(&rec, &o, &out);
    if (rc != AV1G_OK) { if (err) snprintf(err, errlen, "%s", out.error); av1g_output_free(&out); return rc; }
    for (int p = 0; p < 3; p++)
        if (recon[p] && out.recon[p])
            memcpy(recon[p], out.recon[p], (size_t)out.recon_w[p] * out.recon_h[p] * (fp->bit_depth == 10 ? 2 : 1));
    av1g_output_free(&out);
    return 0;
}

// av1core's post-filters (av1g_postfilter / av1g_postfilter16) in place on the planes, for the record's blocks and fp
extern "C" int orc_av1g_postfilter(const av1g_frame_params *fp, uint32_t n_blocks, av1g_block *blocks, void *planes[3], const int stride[3]) {
    av1g_decision_record rec;
    memset(&rec, 0, sizeof rec);
    rec.fp = *fp;
    rec.n_blocks = n_blocks;
    rec.blocks = blocks;
    if (fp->bit_depth == 10) return av1g_postfilter16(&rec, (uint16_t *const *)planes, stride);
    return av1g_postfilter(&rec, (uint8_t *const *)planes, stride);
}

// av1core's AVIF muxer around an OBU stream (cap 0: only the size)
extern "C" int orc_mux_avif(const uint8_t *obu, uint64_t n, uint32_t w, uint32_t h, uint8_t *out, uint64_t cap, uint64_t *size) {
    uint8_t *a = nullptr;
    size_t an = 0;
    const int rc = av1g_mux_avif(obu, (size_t)n, w, h, &a, &an);
    if (rc != AV1G_OK) return rc;
    *size = an;
    if (out && cap >= an) memcpy(out, a, an);
    free(a);
    return 0;
}

extern "C" void orc_set_uv_open_loop(int on) { orc::g_uvOpenLoop = on ? 1 : 0; }
extern "C" void orc_set_edge_filter(int on) { orc::g_edgeFilter = on ? 1 : 0; }

extern "C" void orc_qstep(int qindex, int bd, int *dcq, int *acq) {
    *dcq = av1g_dc_q_bd(qindex, bd);
    *acq = av1g_ac_q_bd(qindex, bd);
}

extern "C" void orc_op_counts(const orc_result *r, uint64_t *analysis, uint64_t *closed) {
    *analysis = r->ops[0];
    *closed = r->ops[1];
}
