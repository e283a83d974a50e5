// oracle/ref_gpu.cpp - C entry points around the reference's own GPU search (maddog107/av1gpu GpEncoder::encode,
// encoder/src/pipeline.h:191-211), built from the reference's sources by oracle/refgpu.mk into oracle/_ref/libref_gpu.so.
// Measurement infrastructure only: the speed bar the B200 build is compared with, and a source of the reference's own
// decisions for BD-rate comparisons.  Nothing in the product links or calls it.
//
// The configuration is the plain knob set: GpConfig's defaults (encoder/src/pipeline.cpp:41-76: all 19 shapes and 10
// partitions, K 4 / Krecheck 2, tx-type search in both loops, angle deltas, CfL, uvK 2, no pruning or staged analysis)
// with palette off, the intra edge filter off (the default), minimum legal tiling (tileMinMp 0) and no post-filters.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "av1g/av1g.h"
#include "pipeline.h"

namespace {
GpEncoder *g_enc = nullptr;
int g_q = -1;
GpFrameOut g_out;
std::string g_err;
uint8_t *g_dev[3] = {nullptr, nullptr, nullptr};
size_t g_devBytes[3] = {0, 0, 0};
}  // namespace

extern "C" {

const char *ref_gpu_error() { return g_err.c_str(); }

// One search of an 8-bit 4:2:0 picture (host planes y w x h, u / v ((w+1)/2) x ((h+1)/2), row-contiguous) at qindex, run
// reps times; times[0..5] = the last run's GpTimes setup, analysis, dp, recon, pack, total (ms, CUDA events); the
// counts of the record.  The planes are padded (edge replication) to the 64-multiple the encoder takes and uploaded
// before the runs; the record stays for ref_gpu_copy.
int ref_gpu_search(int w, int h, int qindex, const uint8_t *y, const uint8_t *u, const uint8_t *v, int reps, float *times, uint32_t *nb,
                   uint32_t *nt, uint64_t *nc) {
    if (w < 1 || h < 1 || qindex < 1 || qindex > 255 || !y || !u || !v || reps < 1) { g_err = "bad arguments"; return -1; }
    if (!g_enc || g_q != qindex) {
        delete g_enc;
        g_enc = new GpEncoder();
        GpConfig cfg;
        cfg.qindex = qindex;
        cfg.palette = 0;
        cfg.edgeFilter = 0;
        cfg.tileMinMp = 0;
        cfg.wantRecon = true;
        if (g_enc->init(cfg, g_err)) { delete g_enc; g_enc = nullptr; return -1; }
        g_q = qindex;
    }
    const int MiW = 2 * ((w + 7) >> 3) * 4, MiH = 2 * ((h + 7) >> 3) * 4;
    const int aw = (MiW + 63) & ~63, ah = (MiH + 63) & ~63;
    const int cw = (w + 1) / 2, ch = (h + 1) / 2, caw = aw / 2, cah = ah / 2;
    const uint8_t *src[3] = {y, u, v};
    const int pw[3] = {w, cw, cw}, ph[3] = {h, ch, ch}, paw[3] = {aw, caw, caw}, pah[3] = {ah, cah, cah};
    GpFrameIn in;
    in.W = w; in.H = h; in.aw = aw; in.ah = ah; in.bitDepth = 8; in.yuv444 = 0;
    for (int p = 0; p < 3; p++) {
        std::vector<uint8_t> pad((size_t)paw[p] * pah[p]);
        for (int r = 0; r < pah[p]; r++)
            for (int c = 0; c < paw[p]; c++) pad[(size_t)r * paw[p] + c] = src[p][(size_t)std::min(r, ph[p] - 1) * pw[p] + std::min(c, pw[p] - 1)];
        if (g_devBytes[p] < pad.size()) {
            if (g_dev[p]) cudaFree(g_dev[p]);
            if (cudaMalloc(&g_dev[p], pad.size()) != cudaSuccess) { g_err = "cudaMalloc"; g_dev[p] = nullptr; g_devBytes[p] = 0; return -1; }
            g_devBytes[p] = pad.size();
        }
        if (cudaMemcpy(g_dev[p], pad.data(), pad.size(), cudaMemcpyHostToDevice) != cudaSuccess) { g_err = "upload"; return -1; }
        in.dsrc[p] = g_dev[p];
        in.spitch[p] = paw[p];
    }
    std::vector<GpFrameIn> ins(1, in);
    GpTimes t;
    for (int r = 0; r < reps; r++) {
        std::vector<GpFrameOut> outs;
        t = GpTimes();
        if (g_enc->encode(ins, outs, t, g_err, 0, nullptr)) return -1;
        g_out = std::move(outs[0]);
    }
    if (times) {
        times[0] = t.setup; times[1] = t.analysis; times[2] = t.dp; times[3] = t.recon; times[4] = t.pack; times[5] = t.total;
    }
    if (nb) *nb = (uint32_t)g_out.blocks.size();
    if (nt) *nt = (uint32_t)g_out.txb.size();
    if (nc) *nc = (uint64_t)g_out.coeffs.size();
    return 0;
}

// The last record: blocks, block_txb (n_blocks + 1), txb, coeffs and the cropped reconstruction planes.
int ref_gpu_copy(av1g_block *blocks, uint32_t *block_txb, av1g_txb *txb, int16_t *coeffs, uint8_t *ry, uint8_t *ru, uint8_t *rv) {
    if (g_out.blocks.empty()) { g_err = "no result"; return -1; }
    memcpy(blocks, g_out.blocks.data(), g_out.blocks.size() * sizeof(av1g_block));
    memcpy(block_txb, g_out.block_txb.data(), g_out.block_txb.size() * sizeof(uint32_t));
    memcpy(txb, g_out.txb.data(), g_out.txb.size() * sizeof(av1g_txb));
    memcpy(coeffs, g_out.coeffs.data(), g_out.coeffs.size() * sizeof(int16_t));
    uint8_t *r[3] = {ry, ru, rv};
    for (int p = 0; p < 3; p++)
        if (r[p]) memcpy(r[p], g_out.recon[p].data(), g_out.recon[p].size());
    return 0;
}

// av1g_encode of the last record with its own frame parameters (the reference's --check, encoder/apps/av1gpu.cpp:932-961):
// the OBU size, whether av1core's reconstruction equals the search's sample for sample, and the frame parameters.
int ref_gpu_check(uint64_t *obu_bytes, int *recon_equal, av1g_frame_params *fp) {
    if (g_out.blocks.empty()) { g_err = "no result"; return -1; }
    GpFrameOut copy = g_out;   // av1g_encode writes eobs / chroma tx types into the record
    av1g_decision_record rec = copy.record();
    if (fp) *fp = rec.fp;
    av1g_encode_opts o = {0, -1};
    av1g_output out;
    memset(&out, 0, sizeof out);
    const int rc = av1g_encode(&rec, &o, &out);
    if (rc != AV1G_OK) { g_err = out.error; av1g_output_free(&out); return -1; }
    int eq = 1;
    for (int p = 0; p < 3; p++) {
        const size_t n = (size_t)out.recon_w[p] * out.recon_h[p];
        if (!out.recon[p] || n != g_out.recon[p].size() || memcmp(out.recon[p], g_out.recon[p].data(), n)) eq = 0;
    }
    *obu_bytes = out.obu_size;
    *recon_equal = eq;
    av1g_output_free(&out);
    return 0;
}

}  // extern "C"
