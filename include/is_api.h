/* include/is_api.h - C ABI of the B200 intra RD search (libisearch.so).
 *
 * The drop-in boundary for maddog107/av1gpu's per-superblock intra search.  The reference's boundary is the C++ class
 * GpEncoder (encoder/src/pipeline.h:191-211): init(const GpConfig&, err) and encode(frames, out records, times, err,
 * stream).  These entry points replace it with plain pointers and sizes:
 *   is_create / is_destroy    <- GpEncoder::GpEncoder + GpEncoder::init            (pipeline.h:193-196, pipeline.cpp:221-298)
 *   is_encode_device          <- GpEncoder::encode, device planes in              (pipeline.h:197-199, pipeline.cpp:323-1180)
 *   is_encode_host            <- the same, host planes in (upload inside)          (av1gpu.cpp:690-843 upload + encode)
 *   is_record_counts / _copy  <- GpFrameOut::record() + the record download       (pipeline.h:165-178, pipeline.cpp:829-1010)
 *   is_record_device          <- GpDevRecords (records stay on the GPU)            (pipeline.h:197-199 `dev`)
 * The output is av1core's DecisionRecord (av1core/include/av1g/decisions.h): blocks in decode order, the tx-block
 * layout of av1g_layout(), quantised levels, plus the exact reconstruction, so av1g_encode() of the record reproduces
 * the reconstruction sample for sample.
 *
 * Plain form only: the reference GpConfig defaults without the speed switches (all 19 shapes, all partitions,
 * K 4 / Krecheck 2, tx-type search open and closed loop, angle deltas, CfL, uvK 2; edge filter, filter intra,
 * palette, QM, delta-q off; minimum legal tiling; tx_mode_select 0).  8- and 10-bit samples, 4:2:0 and 4:4:4, chosen per
 * frame (is_frame.bit_depth / chroma_444) or per handle (is_params).
 *
 * Status codes: IS_OK or a negative IS_ERR_*; is_last_error() returns the message of the last failure of a handle.
 * A handle serves one host thread at a time (several handles may run concurrently on different streams).
 */
#ifndef IS_API_H
#define IS_API_H
#include <stddef.h>
#include <stdint.h>
#include "av1g/decisions.h"

#ifdef __cplusplus
extern "C" {
#endif

#define IS_OK 0
#define IS_ERR_INVALID -1   /* bad argument (size, qindex, bit depth, format) */
#define IS_ERR_CUDA -2      /* a CUDA call failed (message in is_last_error) */
#define IS_ERR_OOM -3       /* device allocation failed */
#define IS_ERR_TIMEOUT -4   /* a wavefront dependency wait of the closed loop ran out of its budget (no hang) */
#define IS_ERR_STATE -5     /* no encode result to read */
#define IS_ERR_TOO_LARGE -6 /* the request does not fit the fixed scratch of is_fwd_quant_static, or an output buffer */
#define IS_ERR_BUSY -7      /* a serving session has no room for the image now: poll, copy finished images, retry */

typedef struct is_params {
    int32_t bit_depth;      /* 8 or 10: the format of frames whose own bit_depth is 0 */
    int32_t chroma_444;     /* 0 (4:2:0) or 1 (4:4:4), likewise */
    int32_t device;         /* CUDA device ordinal */
    int32_t reserved[5];    /* 0 */
} is_params;

typedef struct is_handle is_handle;

/* One image.  planes: Y, U, V of width x height (4:2:0 chroma ((width+1)/2) x ((height+1)/2), 4:4:4 chroma width x
 * height), samples uint8_t (8-bit) or uint16_t (10-bit), pitch in samples.  bit_depth 0 takes the handle's format
 * (is_params); 8 or 10 with chroma_444 0 / 1 gives the frame's own, so one batch may mix formats.
 * is_encode_device: device pointers; is_encode_host: host pointers (pinned memory gives the fastest upload). */
typedef struct is_frame {
    int32_t width, height;
    int32_t qindex;         /* base_q_idx 1..255 */
    int32_t bit_depth;      /* 0 (the handle's), 8 or 10 */
    const void *planes[3];
    int32_t pitch[3];
    int32_t chroma_444;     /* with bit_depth 8 / 10: 0 (4:2:0) or 1 (4:4:4) */
} is_frame;

/* Stage times of the last encode (ms, CUDA events on the handle's stream), cf. the reference's GpTimes
 * (pipeline.h:180-189). */
typedef struct is_times {
    float upload, analysis, dp, recon, pack, total;
    uint32_t sbs, blocks;
} is_times;

int is_create(const is_params *p, is_handle **out);
void is_destroy(is_handle *h);
const char *is_last_error(const is_handle *h);

/* Run the search on one image; stream: a cudaStream_t (NULL = the handle's own stream).  Returns after the work is
 * queued and the record sizes are known (one small device->host read). */
int is_encode_device(is_handle *h, const is_frame *f, void *stream);
int is_encode_host(is_handle *h, const is_frame *f, void *stream);

int is_record_counts(const is_handle *h, uint32_t *n_blocks, uint32_t *n_txb, uint64_t *n_coeffs);
/* Copy the last record (frame params, blocks, block_txb[n_blocks + 1], txb, coeffs) and the cropped
 * reconstruction planes to host memory; any pointer may be NULL. */
int is_record_copy(is_handle *h, av1g_frame_params *fp, av1g_block *blocks, uint32_t *block_txb, av1g_txb *txb,
                   int16_t *coeffs, void *recon[3], const int32_t recon_pitch[3]);
/* Device pointers of the last record (valid until the next encode on the handle). */
int is_record_device(const is_handle *h, const av1g_block **blocks, const uint32_t **block_txb, const av1g_txb **txb,
                     const int16_t **coeffs);
int is_times_get(const is_handle *h, is_times *t);

/* ---- batched form: many images (uneven sizes, mixed qindex) per call ----
 * One persistent closed-loop launch serves every image of the batch through one ready queue (the reference runs one
 * wavefront per image and step: encoder/src/batch.cpp:1005-1029 threads GpEncoders over images).  Each image's front
 * end (upload, analysis, DP, dataflow graph) runs on one of front_streams streams.  Results per image index; the
 * single-image record calls read image 0.  Timing of a batch: is_times_get (analysis = the whole front end). */
int is_encode_batch(is_handle *h, const is_frame *frames, int n, int from_host, void *stream);
int is_batch_counts(const is_handle *h, int i, uint32_t *n_blocks, uint32_t *n_txb, uint64_t *n_coeffs);
int is_batch_copy(is_handle *h, int i, av1g_frame_params *fp, av1g_block *blocks, uint32_t *block_txb, av1g_txb *txb,
                  int16_t *coeffs, void *recon[3], const int32_t recon_pitch[3]);
/* use_graph: capture each batch's launch sequence in a CUDA graph and replay it while the batch signature (sizes,
 * qindex, plane addresses, workspace) repeats; front_streams: 1, 2 or 4 (0 keeps the current value); recon_ctas: CTAs
 * of the closed loop, one per SM when 0 (fewer leave SMs to the work of other streams, e.g. another handle's batch). */
int is_set_batch_options(is_handle *h, int use_graph, int front_streams, int recon_ctas);
/* ---- error paths and checks ----
 * Closed-loop wait budgets of the handle's later encodes: spins of a wait on a neighbouring leaf's flag (each spin
 * sleeps about 64 ns) and nanoseconds a worker waits on an empty ready-queue slot; 0 restores the defaults (2^20 spins,
 * 4 s; at most 2^24 spins and 60 s).  A wait that runs out ends the closed loop (every worker abandons its leaf and the
 * kernel returns) and the encode returns IS_ERR_TIMEOUT; the handle stays usable.  The reference has no counterpart
 * (its wavefront steps are separate launches with no waits). */
int is_set_wait_limits(is_handle *h, int leaf_wait_iters, long long ready_wait_ns);
/* Device-memory budget of the handle's workspace in bytes (0: no limit): an encode or batch whose workspace would
 * exceed it returns IS_ERR_OOM before any allocation (admission by HBM budget; the reference fails in cudaMalloc,
 * pipeline.cpp:31-39). */
int is_set_workspace_limit(is_handle *h, uint64_t bytes);
/* Poison mode (the reference's GP_POISON / GP_POISON_SMEM, encoder/src/pipeline.cpp:311-313, k_recon.cuh:1705-1708):
 * before each encode every byte of the workspace is set to 0xA5, and every search kernel fills its shared memory with a
 * fixed pattern before it starts.  A read of anything the search did not write first would change the results; with
 * poison on they must equal those without. */
int is_set_poison(is_handle *h, int on);

/* Non-learned pruning of the handle's later encodes (the plain form: rd_k 4, tx_keep 0).  rd_k (1 .. 4; 0 = 4): every
 * analysed block takes its best rd_k screened candidates into the exact-rate RD (the reference's K, GpParams::K,
 * encoder/src/gp.h); tx_keep (0 .. 3): each analysed block keeps its tx_keep best tx types by open-loop RD cost, and the
 * closed loop's tx-type pass for that block's first candidate tries only those (with DCT_DCT and the analysis' type) -
 * the reference's open-loop tx shortlist (GpParams::txShortlist, encoder/src/k_leafprep.cu:292-360), ranked here by the
 * analysis' own exact-rate costs instead of a transform-domain L1 after the DP.  0 keeps every type.  Decisions change,
 * the reconstruction stays exact. */
int is_set_search_options(is_handle *h, int rd_k, int tx_keep);
/* Device workspace of one image of width x height in a batch (bytes; host only, no GPU needed): what admission by
 * HBM budget counts. */
int is_workspace_bytes(int width, int height, uint64_t *bytes);
/* the same for a frame of the given format (bit_depth 8 / 10, chroma_444 0 / 1) */
int is_workspace_bytes_format(int width, int height, int bit_depth, int chroma_444, uint64_t *bytes);
/* Warps per CTA the closed loop runs: 1 .. 8 caps it at the most the shared memory of a CTA holds (8 for 8-bit 4:2:0,
 * fewer for the larger formats); 0 (the default) takes 4 for a single image - its loop is bound by its dependency chain,
 * and fewer warps leave the SM a larger L1 - and all of them for a batch or a serving session. */
int is_set_closed_loop_warps(is_handle *h, int warps);
/* Autotuner: times the batch with 1, 2 and 4 front-end streams x 4, 6 and all closed-loop warps per CTA (two runs each,
 * the second timed) and keeps the fastest for the handle; returns the choice and its time (ms). */
int is_autotune_batch(is_handle *h, const is_frame *frames, int n, int from_host, int *front_streams, int *recon_warps, float *ms);

/* ---- serving: continuous admission of images into a running closed loop ----
 * A session (one per handle, one image format; is_serve_open allocates it, is_serve_start starts it) keeps one persistent
 * closed loop running on recon_ctas SMs (0: three
 * quarters of them; the rest run the front ends of arriving images and the packs of finished ones).  is_serve_submit
 * places an image in a free range of the session's workspace arena (arena_bytes; an image needs
 * is_workspace_bytes_format(...) bytes of it) and a free slot of max_images, and queues its front end (upload, analysis,
 * DP, dataflow graph) on a front-end stream; its first ready leaves go into the loop that is already running, so an image
 * submitted while others are in the closed loop is searched together with them.  Its last leaf signals the host:
 * is_serve_poll packs the records of the images whose loop has finished and returns the tickets of those whose records
 * are ready; is_serve_copy copies one out (as is_batch_copy) and frees its range and slot.  Each image's result is that of
 * the same image searched alone.  Limits: max_leaves bounds the leaf positions of the whole session (each image reserves
 * 256 per superblock; IS_ERR_STATE when used up: close and open a new session).  The loop ends by itself after 2 ms
 * without work, and is_serve_poll launches it again once a submitted image's front end has queued leaves: the caller
 * polls to make progress, and the loop holds its stream only while there is work.  is_serve_stop waits for the loop to
 * end (no new launch follows); is_serve_close stops and frees the session (images not read out are lost).  While a
 * session is open its loop occupies the device: host planes should be in pinned memory, and the process should not free
 * device or pinned memory (cudaFree / cudaFreeHost, e.g. another handle's workspace growing), which would wait for the
 * loop.  A running loop holds a hardware work queue: a process that opens sessions does best with more queues than the
 * default 8 (CUDA_DEVICE_MAX_CONNECTIONS=32, which the Python package sets on import), so that fewer streams share one
 * with a loop and wait for it to become idle.  The
 * reference runs whole batches per GpEncoder thread (encoder/src/batch.cpp:1005-1029) and has no counterpart. */
int is_serve_open(is_handle *h, int bit_depth, int chroma_444, uint64_t arena_bytes, int max_images, uint64_t max_leaves,
                  int recon_ctas);
/* starts the session's loop (allocates nothing: open every session of the process first, then start them) */
int is_serve_start(is_handle *h);
/* from_host: host planes (else device planes); IS_ERR_BUSY: no free slot or range now (poll / copy, then retry) */
int is_serve_submit(is_handle *h, const is_frame *f, int from_host, int *ticket);
int is_serve_poll(is_handle *h, int *tickets, int cap, int *n);
int is_serve_counts(is_handle *h, int ticket, uint32_t *n_blocks, uint32_t *n_txb, uint64_t *n_coeffs);
int is_serve_copy(is_handle *h, int ticket, av1g_frame_params *fp, av1g_block *blocks, uint32_t *block_txb, av1g_txb *txb,
                  int16_t *coeffs, void *recon[3], const int32_t recon_pitch[3]);
/* ends the loop without freeing (a process with several sessions stops them all, then closes them: frees wait for every
 * running kernel); is_serve_close stops if needed and frees the session */
int is_serve_stop(is_handle *h);
int is_serve_close(is_handle *h);

/* ---- entropy coding on the device: records -> AV1 bitstream ----
 * Replaces av1core's GPU entropy coder av1g_gpu::run_batch_device_scratch_bytes / run_batch_device
 * (av1core/include/av1g/gpu_entropy.h:73-147) and the OBU assembly after it (Encoder::write_headers,
 * av1core/src/encoder.cpp:1317-1441, and the framing of Encoder::run, :1571-1600).  The payloads are byte for byte those
 * of av1g_encode() on the same records.  Records of the search's toolset: lossy, 4:2:0 or 4:4:4, 8- or 10-bit, tx_depth
 * 0, no delta-q / palette / filter intra / reduced tx set (IS_ERR_INVALID otherwise), with or without CDEF (each SB's
 * cdef_idx is coded with its first non-skip block); header-only fields (tiling, delta_q_* of the planes, quantizer
 * matrices, loop-filter levels, colour description) are free. */
typedef struct is_ent_frame {
    av1g_frame_params fp;        /* host copy of the frame parameters */
    const av1g_block *blocks;    /* device: n_blocks blocks in decode order */
    const uint32_t *block_txb;   /* device: n_blocks + 1 entries (the av1g_layout() of the blocks) */
    const av1g_txb *txb;         /* device: n_txb tx blocks; the chroma tx_type and eob fields are not read (derived) */
    const int16_t *coeffs;       /* device: the levels, txb[].coeff_off relative to this pointer */
    uint32_t n_blocks, n_txb;
} is_ent_frame;
#define IS_ENT_ERR_SYMBOLS 1     /* more symbols than the capacity: status.symbols is the count needed (rerun with it) */
#define IS_ENT_ERR_OUTPUT 2      /* a tile's payload outgrew its buffer */
#define IS_ENT_ERR_RECORD 4      /* blocks out of decode order, a partition the syntax cannot code, a field out of range */
typedef struct is_ent_status {   /* the head of the device result */
    int32_t error;               /* 0 or IS_ENT_ERR_* bits; the payloads are valid only for 0 */
    int32_t reserved;
    uint64_t symbols;            /* symbols of the batch (also when it exceeded the capacity) */
    uint64_t capacity;
    uint64_t bytes;              /* payload bytes of every tile */
} is_ent_status;
typedef struct is_ent_out {
    const void *result;          /* device: is_ent_status, then uint64_t tile_offset[n_tiles + 1] (one download) */
    uint64_t result_bytes;
    const uint8_t *payload;      /* device: tile i of the batch = payload[tile_offset[i] .. tile_offset[i + 1]) */
    uint64_t payload_capacity;
    uint32_t n_tiles;            /* frame f owns tiles frame_tile0[f] .. frame_tile0[f + 1] - 1 (raster order) */
} is_ent_out;
/* Scratch the batch needs with a symbol capacity (0: a default bound from the frames' sizes). */
int is_entropy_scratch_bytes(const is_ent_frame *frames, int n, uint64_t symbol_capacity, uint64_t *bytes);
/* Enqueue the coding of n frames on stream (a cudaStream_t; NULL = the legacy default stream of device): no allocation,
 * no synchronisation.  scratch: device memory of at least is_entropy_scratch_bytes(), 256-byte aligned; it and the
 * out pointers belong to the call until the stream has passed it.  frame_tile0: n + 1 entries (host) or NULL. */
int is_entropy_batch(int device, const is_ent_frame *frames, int n, uint64_t symbol_capacity, void *scratch, uint64_t scratch_bytes,
                     void *stream, is_ent_out *out, uint32_t *frame_tile0);
/* The OBU stream of one frame (sequence header OBU + frame OBU, no temporal delimiter; av1g_encode()'s obu bytes) from
 * its tile payloads (host memory, tile i = payload[tile_offset[i] .. tile_offset[i + 1])).  *size gets the length;
 * IS_ERR_TOO_LARGE when cap is smaller (nothing written). */
int is_obu_assemble(const av1g_frame_params *fp, const uint8_t *payload, const uint64_t *tile_offset, uint32_t n_tiles, uint8_t *out,
                    uint64_t cap, uint64_t *size);
/* The AVIF file (still image, the layout libavif writes: ftyp, meta with hdlr / pitm / iinf / iloc / iprp (ispe, av1C,
 * pixi, colr nclx), mdat) around an OBU stream written for fp (is_obu_assemble / is_encode_obu): av1core's av1g_mux_avif
 * (av1core/include/av1g/av1g.h:128-131, av1core/src/avif.cpp) writes the same bytes.  Host only; IS_ERR_TOO_LARGE when
 * cap is smaller (*size = the bytes needed). */
int is_avif_mux(const av1g_frame_params *fp, const uint8_t *obu, uint64_t obu_size, uint8_t *out, uint64_t cap, uint64_t *size);
/* Images first .. first + n - 1 of the handle's last encode (batch order; a single image is image 0) coded on the device
 * in one batch and returned as OBU streams back to back: image k at out[offsets[k] .. offsets[k + 1]).  The handle keeps
 * the scratch; a symbol count above the default capacity reruns once with the exact count.  device_ms (may be NULL):
 * the device time of the coding kernels.  IS_ERR_TOO_LARGE when cap is smaller than the streams (offsets[n] = the bytes
 * needed). */
int is_encode_obu(is_handle *h, int first, int n, uint8_t *out, uint64_t cap, uint64_t *offsets, float *device_ms);

/* ---- post-filters on the device ----
 * Deblocking (spec 7.14) then CDEF (spec 7.15), as the decoder applies them, in place on image i's reconstruction of the
 * handle's last encode (is_batch_copy / is_record_copy then return the filtered planes); replaces av1core's
 * av1g_postfilter / av1g_postfilter16 (av1core/include/av1g/av1g.h:95-104, encoder.cpp:1998-2041) and its GPU
 * counterpart (av1core/src/gpu_postfilter.cu).  fp: the frame's parameters with the filter fields set (effective
 * loop_filter_level[4], loop_filter_sharpness, enable_cdef, cdef_damping_minus_3, cdef_bits and the strengths); its size and
 * format must be the image's.  sb_cdef: the cdef_idx of every 64x64 (raster, (MiCols + 15) / 16 per row; NULL = 0), written
 * into the record's blocks so that av1g_encode() of the record with fp reconstructs the filtered planes; from then on the
 * frame parameters is_batch_copy / is_record_copy return and the frame header is_encode_obu writes carry the filters (so
 * the decoded stream is the filtered picture).  device_ms (may be NULL): device time of the filters.  Not undone by
 * anything but a new encode. */
int is_postfilter(is_handle *h, int i, const av1g_frame_params *fp, const int8_t *sb_cdef, float *device_ms);
/* The reference's default deblocking decision for a base qindex (av1f LF_FROM_Q, av1f/include/av1f/lfsearch_gpu.h:19,
 * av1f/include/av1f/tuneiq.h:152-199: libaom's av1_pick_filter_level LPF_PICK_FROM_Q for a key frame plus the intra
 * delta, the tune=iq sharpness rule) into fp's loop_filter_level[4] and loop_filter_sharpness, and its CDEF damping
 * (cdef_damping_minus_3); enable_cdef and the presets are left as they are (the reference's CDEF preset search has no
 * counterpart here).  No GPU needed. */
int is_postfilter_from_q(int qindex, int bit_depth, av1g_frame_params *fp);

/* ---- kernel-level entry points for the parity tests (device primitives of av1core's dsp.h API) ---- */
/* Forward 2-D transform (this project's integer transform) + quantisation + rate of n residual blocks of one tx
 * size / type, host arrays: res [n][H*W] int32 -> coef [n][tw*th] (fixed point), levels [n][tw*th], D, R, eob per block.
 * plane 0 luma, 1/2 chroma; ctx = (skipCtx, dcCtx, intraDir). */
int is_test_fwd_quant(is_handle *h, int n, const int32_t *res, int tx_size, int tx_type, int plane, int qindex,
                      const int32_t ctx[3], int32_t *coef, int16_t *levels, int64_t *D, int64_t *R, int32_t *eob);
/* Exact inverse transform (av1g_dequant + av1g_inv_txfm2d semantics) of n level blocks: res [n][H*W], flags [n]. */
int is_test_inverse(is_handle *h, int n, const int16_t *levels, int tx_size, int tx_type, int qindex, int32_t *res,
                    uint32_t *flags);
/* Intra prediction (av1g_build_edges + av1g_predict_intra semantics) of n blocks on an 8-bit plane (host, w x h):
 * params [n][10] = {x, y, log2W, log2H, haveLeft, haveAbove, haveAR, haveBL, mode, delta}, out [n][64*64]. */
int is_test_predict(is_handle *h, int n, const uint8_t *plane, int w, int hgt, const int32_t *params, uint8_t *out);
/* Analysis records of one shape of the last encode: J, cand[4], ncand, tx and the closed loop's tx mask per block (0:
 * every type); returns the count or < 0. */
int is_debug_analysis(is_handle *h, int bsize, int64_t *J, uint8_t *cand, uint8_t *ncand, uint8_t *tx, uint16_t *tx_mask);
/* Leaves of SB sb of the last encode (bsize, x4, y4); returns the count or < 0. */
int is_debug_leaves(is_handle *h, uint32_t sb, uint8_t *bsize, uint8_t *x4, uint8_t *y4);
/* Fixed-point tables as uploaded: cost table of q-context qctx (n entries), averaged bits, lambda of a qindex.  Host
 * only: h may be NULL (no GPU needed).  Returns the cost-table size. */
int is_debug_tables(is_handle *h, int qctx, uint16_t *cost, size_t cap, int32_t *avgY13, int32_t *avgPart50,
                    int32_t *avgSkip0, int qindex, int64_t *lam, int64_t *sqrtlam);

/* Closed-loop trace (debug): is_set_trace(h, 1) before an encode records, per queued leaf (queue order), 10 values:
 * the globaltimer (ns) when a worker claimed its queue slot, read the slot, finished the luma prologue (loads, edges,
 * contexts), luma pass 1, luma pass 2, published the luma, finished its chroma waits, the chroma screening and RD, and
 * the leaf; then the queue entry (image << 32 | sb << 8 | leaf).  The queue is image 0's: in a batch, that of image 0's
 * format group (every image of the group).  is_get_trace copies up to cap / 10 leaves and sets n to the queue's leaves. */
int is_set_trace(is_handle *h, int on);
int is_get_trace(is_handle *h, unsigned long long *out, size_t cap, uint32_t *n);

/* ---- learned shortlist: a small BF16 conv / MLP network scoring (mode, angle delta, tx type) candidates per block,
 * trained on the GPU with the library's BF16 tensor-core kernels on labels the exhaustive search produces.  It plays the
 * role of the reference's external-screener hook (GpBatch::extCand / GpExtCand {J, mode, delta, tx},
 * encoder/src/gp.h:136-143,164-170, consumed in place of the SATD screening at encoder/src/k_analysis.cuh:586-606), which
 * nothing in the reference fills; its hand-made pruning is the staged analysis and the open-loop shortlists
 * (encoder/src/an_stage.h, k_leafprep.cu).
 * Scored blocks: the 16 shapes of at least 64 samples (8x8 .. 64x64, 4x16, 16x4; not 4x4, 4x8, 8x4), in the order
 * 8x8 8x16 16x8 16x16 16x32 32x16 32x32 32x64 64x32 64x64 4x16 16x4 8x32 32x8 16x64 64x16.  Input (IS_SL_FEAT bf16 per
 * block): a 32 x 32 luma patch resampled from the block and a margin of ceil(side / 8) samples above and left (box
 * averages, mean removed, / 64; 10-bit samples count a quarter), then 32 extras: an 8-bin gradient-orientation histogram
 * of the patch, the shape one-hot (16), qindex / 255, 1, zeros.  Layers: conv 3x3 stride 2 1 -> 8 (16 x 16), 8 -> 16
 * (8 x 8), 16 -> 16 (4 x 4), each ReLU; fc 288 (the 256 conv outputs, position-major, then the 32 extras) -> 160 ReLU;
 * fc 160 -> 80 scores: [0, 61) the (mode, delta) classes (DC, SMOOTH, SMOOTH_V, SMOOTH_H, PAETH, then V .. D67 x delta
 * -3 .. 3), [64, 80) the 16 tx types.  Parameters: IS_SL_PARAMS fp32 in the order conv1 w [8][9] b [8], conv2 w [16][72]
 * b [16], conv3 w [16][144] b [16], fc1 w [160][288] b [160], fc2 w [80][160] b [80] (a conv weight's column is
 * tap * in_channels + channel, tap = 3 ky + kx). */
#define IS_SL_FEAT 1056
#define IS_SL_OUT 80
#define IS_SL_PARAMS 62688
typedef struct is_learner is_learner;
int is_sl_create(int device, int max_batch, is_learner **out);   /* max_batch: a multiple of 32, at most 65536 */
void is_sl_destroy(is_learner *L);
int is_sl_set_params(is_learner *L, const float *params);   /* also resets the Adam state */
int is_sl_get_params(is_learner *L, float *params);
/* scores (device, n x IS_SL_OUT fp32) of n feature rows (device bf16, n x IS_SL_FEAT), through the GEMM path */
int is_sl_forward(is_learner *L, const void *X, int n, float *S, void *stream);
/* gradients (host, IS_SL_PARAMS floats in parameter order) of the mean loss of one batch (n a multiple of 32; device X,
 * labels y n x 3 int32: (mode, delta) class, tx type or -1, the tx set's types as a bit mask), its mean loss and the
 * count of rows whose best-scored class is the label; weights unchanged.  Loss: softmax cross-entropy of the (mode,
 * delta) head plus that of the tx head restricted to the block's set (no tx term where the tx label is -1). */
int is_sl_grads(is_learner *L, const void *X, const int32_t *y, int n, float *grads, float *loss, int *correct);
/* one Adam step (lr; beta 0.9 / 0.999) on a batch; the batch's mean loss and correct count */
int is_sl_train_step(is_learner *L, const void *X, const int32_t *y, int n, float lr, float *loss, int *correct);
/* C[M x N] = A[M x K] B[N x K]^T (+ bias, ReLU) on device bf16 operands, fp32 out (K, lda, ldb multiples of 8) */
int is_nn_gemm(int M, int N, int K, const void *A, int lda, const void *B, int ldb, float *C, int ldc, const float *bias,
               int relu, void *stream);
/* training rows of image i of the last search: features (device bf16, n x IS_SL_FEAT) and labels (device int32, n x 3)
 * of its scored records (shape by shape, records in analysis order; a record outside the frame has class -1 and zero
 * features), the labels being the analysis' choices (best (mode, delta), its tx type); *n = the number of records (also
 * when it exceeds cap: then nothing is written) */
int is_sl_dataset(is_handle *h, int i, void *X, int32_t *y, int cap, int *n);
/* the search's fused inference kernel (source plane -> candidates in one kernel) on image i of the last search with the
 * learner's weights: scores (device fp32, n x IS_SL_OUT) of the same rows as is_sl_dataset (rows outside the frame are
 * not written) */
int is_sl_infer(is_handle *h, is_learner *L, int i, float *S, int cap, int *n);

/* Use a trained shortlist in the search of this handle (params NULL: the plain form again).  Before each image's
 * analysis the fused kernel scores every scored block; a block whose most probable (mode, delta) has probability below
 * conf falls back to the full search; the others screen only the smallest set of most probable (mode, delta) candidates
 * whose probabilities add up to tau (at most max_cand, 1 .. 8), with no separate angle-delta search, take their best
 * rd_k (1 .. 4) into the exact-rate RD, and try beyond DCT_DCT only the tx types of the block's set that cover tx_tau of
 * the tx head's probability (at most max_tx; 0: none) - in the analysis and in the closed loop's tx-type pass.  The
 * chosen modes are still coded and reconstructed exactly. */
int is_set_shortlist_model(is_handle *h, const float *params, float tau, int max_cand, float conf, int rd_k, float tx_tau,
                           int max_tx);

/* INT32 issue-rate probe: the measured INT32 instruction throughput of the device (Gop/s, multiply-add + logic chains
 * over every SM) and the best kernel time, the roofline denominator of this integer path. */
int is_probe_int32(int device, double *gops, float *ms);

/* Forward transform + quantisation + rate of n residual blocks (the same computation and arguments as
 * is_test_fwd_quant) without any device allocation: no handle, and no cudaMalloc / cudaFree or other allocating call.
 * No counterpart in the reference.  For callers that may not allocate device memory (memory owned by a pool or
 * budgeted elsewhere, or code that must not meet the allocator's implicit synchronisation).  The kernel's buffers live
 * in one static scratch of IS_STATIC_SCRATCH_BYTES per device, reserved with the library's module.
 *  - The first call on a device does one-time setup (the search's tables, the scratch address): make it before any
 *    stream capture.  While the given stream is being captured, a call that would do the setup returns IS_ERR_INVALID
 *    without doing anything; a setup that failed is tried again by the next call.  Nothing is claimed about calls
 *    inside a capture.
 *  - ctx = (skipCtx 0..12, dcCtx 0..2, intraDir 0..12), and tx_type must be one of the intra set of tx_size
 *    (DCT_DCT alone for sizes with a 64-sample side and for 32x32, 16x32, 32x16, 8x32, 32x8); anything else returns
 *    IS_ERR_INVALID before any GPU work.
 *  - n blocks of W x H need n * (4 W H + 6 nc + 20) bytes, each of the six sections rounded up to 256 bytes
 *    (nc = min(W, 32) * min(H, 32)); a request that does not fit returns IS_ERR_TOO_LARGE before any GPU work (for
 *    example at most 186 blocks of 64x64, 1625 of 16x16).  Bad arguments return IS_ERR_INVALID, CUDA failures
 *    IS_ERR_CUDA (no message: there is no handle).
 *  - Nothing in the scratch has to start at zero: the call copies its residuals in before the launch and the kernel
 *    writes every output word the call reads back.
 *  - Calls on one device share the scratch: they must not overlap.  Two calls in flight at once on the same device
 *    (from other threads or streams) race on it and can return each other's results.
 * Host arrays in and out (as is_test_fwd_quant); stream: a cudaStream_t (NULL = the legacy default stream); returns
 * after the results are in the host arrays.  The calling thread's current device is restored. */
#define IS_STATIC_SCRATCH_BYTES (4u << 20)
int is_fwd_quant_static(int device, int n, const int32_t *res, int tx_size, int tx_type, int plane, int qindex,
                        const int32_t ctx[3], int32_t *coef, int16_t *levels, int64_t *D, int64_t *R, int32_t *eob,
                        void *stream);

#ifdef __cplusplus
}
#endif
#endif
