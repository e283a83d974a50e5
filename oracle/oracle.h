/* oracle/oracle.h - C API of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The oracle is a scalar CPU restatement of the plain-form intra RD search of maddog107/av1gpu
 * (encoder/src: k_analysis.cuh, k_dp.cuh, k_recon.cuh, dev_tx.cuh, k_misc.cu) in exact integer / fixed-point
 * arithmetic.  It is linked with av1core (built from the reference's own sources) and calls av1core's dsp.h for
 * prediction, edges, CfL, dequantisation and the inverse transform, and av1g_encode() for the reconstruction check.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the product never does.
 */
#ifndef ORACLE_H
#define ORACLE_H
#include <stdint.h>
#include <stddef.h>
#include "av1g/decisions.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_image {
    int width, height;       /* visible size */
    int bit_depth;           /* 8 or 10 */
    int chroma_444;          /* 0: 4:2:0, 1: 4:4:4 */
    int qindex;              /* base_q_idx 1..255 */
    const void *planes[3];   /* visible planes (uint8_t or uint16_t samples), chroma per chroma_444 */
    int stride[3];           /* in samples */
} orc_image;

typedef struct orc_result orc_result;

/* Run the plain-form search.  threads >= 1: superblocks in the 2:1 wavefront over that many host threads
 * (results do not depend on it).  Returns 0 or a negative error. */
int orc_encode(const orc_image *img, int threads, orc_result **out);
void orc_free(orc_result *r);

/* Record access: counts, then copies into caller arrays (any pointer may be NULL). */
void orc_counts(const orc_result *r, uint32_t *n_blocks, uint32_t *n_txb, uint64_t *n_coeffs);
void orc_copy_record(const orc_result *r, av1g_frame_params *fp, av1g_block *blocks, uint32_t *block_txb, av1g_txb *txb,
                     int16_t *coeffs);
/* Cropped reconstruction of plane p (samples of the bit depth, width x height of the plane). */
void orc_copy_recon(const orc_result *r, int p, void *dst);
/* Analysis records of shape bsize (raster over the shape's grid): J (int64, J units), cand[4] (mode << 3 | delta + 3),
 * ncand, tx.  Returns the number of blocks of the shape. */
uint32_t orc_analysis(const orc_result *r, int bsize, int64_t *J, uint8_t *cand, uint8_t *ncand, uint8_t *tx);
/* Leaves of superblock sb (raster over the image's SB grid): bsize, x4, y4 (SB-relative); returns the count. */
int orc_leaves(const orc_result *r, uint32_t sb, uint8_t *bsize, uint8_t *x4, uint8_t *y4);

/* av1core's reconstruction of a record (av1g_layout + av1g_encode, no post-filters): cropped planes into
 * recon[p] (plane widths x heights).  Returns av1g_encode's status, message in err. */
int orc_av1g_recon(av1g_decision_record *rec, void *recon[3], char *err, size_t errlen, uint64_t *obu_bytes);

/* Primitives for the kernel tests. */
/* Forward 2-D transform of a residual (H x W row-major int32) into tw x th fixed-point coefficients. */
void orc_fwd2d(const int32_t *res, int txSz, int txType, int bd, int32_t *coef);
/* Exact inverse (av1core av1g_dequant + av1g_inv_txfm2d) of levels: residual H x W; returns the error flags. */
uint32_t orc_inv2d(const int16_t *levels, int txSz, int txType, int bd, int dcQ, int acQ, int32_t *res);
/* Quantise + rate + distortion of coefficients (tw x th); levels out; D (J units), R (1/256 bit), eob. */
void orc_quant_rate(const int32_t *coef, int txSz, int txType, int plane, int bd, int dcQ, int acQ, int skipCtx, int dcCtx,
                    int intraDir, int qctx, int64_t resEnergy, int16_t *levels, int64_t *D, int64_t *R, int *eob);
/* Fixed-point tables: the coefficient-CDF cost table of q-context qctx (1/256 bit, uint16 per CDF entry of
 * av1g_cdfs), n = entries; the averaged mode / partition / skip bits. */
size_t orc_cost_table(int qctx, uint16_t *out, size_t cap);
void orc_avg_bits(int32_t *avgY13, int32_t *avgPart50, int32_t *avgSkip0);
/* lambda (1/256 units of lambda) and sqrt(lambda) (1/256 units) of a qindex / bit depth */
void orc_lambda(int qindex, int bd, int64_t *lam, int64_t *sqrtlam);
/* Intra prediction of one block through av1core (mode, delta, edges from a plane), for the kernel tests. */
void orc_predict(const uint8_t *plane, int stride, int x, int y, int log2W, int log2H, int haveLeft, int haveAbove,
                 int haveAR, int haveBL, int maxX, int maxY, int mode, int delta, uint8_t *dst);

/* The reference's own CPU decision engine (av1core/src/ref_engine.cpp, a different and simpler algorithm):
 * 8-bit 4:2:0 only; returns decide seconds and encode seconds. */
int orc_ref_engine(const orc_image *img, double *sec_decide, double *sec_encode);

/* Algorithmic INT32 operations of the last search (the roofline numerator, cost model in plain_search.cpp):
 * open-loop analysis and closed loop. */
void orc_op_counts(const orc_result *r, uint64_t *analysis, uint64_t *closed);

/* dc_q / ac_q of a qindex (spec 7.12.2 Dc_Qlookup / Ac_Qlookup). */
void orc_qstep(int qindex, int bd, int *dcq, int *acq);

/* orc_av1g_recon of a record given as arrays; the frame parameters are the plain form's for that picture. */
int orc_av1g_recon_arrays(int width, int height, int qindex, int bd, int chroma_444, uint32_t n_blocks, av1g_block *blocks,
                          uint32_t *block_txb, uint32_t n_txb, av1g_txb *txb, uint64_t n_coeffs, int16_t *coeffs,
                          void *recon[3], char *err, size_t errlen, uint64_t *obu_bytes);

/* av1g_encode()'s OBU stream of such a record (bitstream only; obu may be NULL to ask for the size), its symbol count, and
 * where av1g_parse() finds each tile payload in it (offsets from the start of the stream, byte counts; tile_cap entries at
 * most). */
int orc_av1g_obu_arrays(int width, int height, int qindex, int bd, int chroma_444, uint32_t n_blocks, av1g_block *blocks,
                        uint32_t *block_txb, uint32_t n_txb, av1g_txb *txb, uint64_t n_coeffs, int16_t *coeffs, uint8_t *obu,
                        uint64_t cap, uint64_t *size, uint32_t *n_tiles, uint64_t *tile_off, uint32_t *tile_bytes, uint32_t tile_cap,
                        uint64_t *n_symbols, char *err, size_t errlen);

/* orc_av1g_obu_arrays with the record's frame parameters given. */
int orc_av1g_obu_fp(const av1g_frame_params *fp, uint32_t n_blocks, av1g_block *blocks, uint32_t *block_txb, uint32_t n_txb,
                    av1g_txb *txb, uint64_t n_coeffs, int16_t *coeffs, uint8_t *obu, uint64_t cap, uint64_t *size,
                    uint32_t *n_tiles, uint64_t *tile_off, uint32_t *tile_bytes, uint32_t tile_cap, uint64_t *n_symbols,
                    char *err, size_t errlen);
/* av1g_encode() of a record with the given frame parameters and flags (AV1G_ENC_*); recon planes as av1g_output describes
 * them (cropped, or the unfiltered coded area with AV1G_ENC_PREFILTER_RECON). */
int orc_av1g_encode_fp(const av1g_frame_params *fp, uint32_t flags, uint32_t n_blocks, av1g_block *blocks, uint32_t *block_txb,
                       uint32_t n_txb, av1g_txb *txb, uint64_t n_coeffs, int16_t *coeffs, void *recon[3], char *err, size_t errlen);
/* av1core's post-filters in place on planes of at least the coded area (strides in samples). */
int orc_av1g_postfilter(const av1g_frame_params *fp, uint32_t n_blocks, av1g_block *blocks, void *planes[3], const int stride[3]);

/* av1core's AVIF muxer (av1g_mux_avif) around an OBU stream; out may be NULL to ask for the size. */
int orc_mux_avif(const uint8_t *obu, uint64_t n, uint32_t w, uint32_t h, uint8_t *out, uint64_t cap, uint64_t *size);
/* Experiment switch (0 = the plain form): the chroma screening on source edges (the reference's open-loop chroma
 * shortlist), its operations counted as open-loop work.  Process-wide; set it before orc_encode. */
void orc_set_uv_open_loop(int on);
/* Experiment switch (0 = the plain form): the search with the intra edge filter (its records need
 * enable_intra_edge_filter = 1).  Process-wide; set it before orc_encode. */
void orc_set_edge_filter(int on);
/* The reference's default frame-level post-filter decisions for a base qindex (ref_shim.cpp). */
void orc_ref_lf_from_q(int base, int bd, int *level, int *sharpness, int *damping);

#ifdef __cplusplus
}
#endif
#endif
