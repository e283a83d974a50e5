// is_serve.cuh - serving sessions: continuous admission of images into a running closed loop (included by is_api.cu).
//
// A session owns a workspace arena, a table of image descriptors, one ready queue and a persistent closed-loop kernel
// (k_recon in serving mode) on part of the SMs.  is_serve_submit lays an image out in a free range of the arena, writes
// its descriptor into a free table slot and queues its front end (upload, analysis, DP, dataflow graph) on a front-end
// stream; the front end's first ready leaves go into the queue of the kernel that is already running, so the image's
// closed loop starts while earlier images are still in theirs.  The image's last leaf sets the slot's word in
// host-mapped memory; is_serve_poll then packs that image's record on a pack stream, and once the pack is done reports
// the image, whose record is_serve_copy reads out (freeing its range and slot).  The reference has no counterpart: its
// batch front end threads one GpEncoder per stream (encoder/src/batch.cpp:1005-1029), each running whole batches.
#pragma once

struct ServeSlot {
    int state = 0;                 // 0 free, 1 searching, 2 packing, 3 record ready
    int gen = 0;                   // generation of the slot (the high bits of the image's tag)
    size_t off = 0, bytes = 0;     // its range of the arena
    FrameDesc F;
    int nSb = 0, qidx = 0, maxLeaves = 0;
    cudaEvent_t ev = nullptr;      // recorded after its pack and the download of its counts
    cudaEvent_t evFront = nullptr; // recorded after its front end (its first ready leaves are in the queue)
    uint32_t *hCnt = nullptr;      // pinned: n_blocks, n_txb, n_coeffs (2 words)
    uint32_t *hOrd = nullptr;      // pinned staging of its SB orders (room for the largest picture, 65536 SBs)
};

struct ServeSession {
    int bd = 8, c444 = 0, g = 0, grid = 0, warps = 0;   // format, its group; the loop's CTAs and warps per CTA
    uint8_t *arena = nullptr;
    size_t arenaBytes = 0;
    std::vector<std::pair<size_t, size_t>> freeList;   // (offset, bytes), sorted by offset
    std::vector<ServeSlot> slots;
    FrameDesc *dTable = nullptr, *hTable = nullptr;   // device table of descriptors, pinned staging
    unsigned long long *dQueue = nullptr;              // ready queue (positions are never reused within a session)
    size_t queueCap = 0, inflightLeaves = 0;           // positions; upper bound of the leaves of the images in the loop
    int *dCtl = nullptr;                               // [0] next slot to take, [1] next slot to write, [2] error
    volatile int *hFlags = nullptr;                    // host-mapped: per table slot, the tag of its finished image
    int *dFlags = nullptr;
    int *hErr = nullptr;                               // pinned: the loop's error word, read after a run
    cudaStream_t kst = nullptr, fst[2] = {nullptr, nullptr}, pst = nullptr;
    cudaEvent_t kdone = nullptr;                       // recorded after the kernel (it completes only when the loop ends)
    int nextFront = 0;
    bool started = false, stopped = false;
};

namespace {

constexpr int SERVE_MAX_SBS = 256 * 256;   // superblocks of the largest picture (16384 x 16384)
constexpr unsigned long long SERVE_IDLE_NS = 2000000ull;   // a session's loop ends after 2 ms without work

// the free range of the arena that fits bytes (first fit, 256-byte aligned); returns false if none does
bool serve_alloc(ServeSession *S, size_t bytes, size_t *off) {
    bytes = align256(bytes);
    for (size_t i = 0; i < S->freeList.size(); i++) {
        auto &r = S->freeList[i];
        if (r.second >= bytes) {
            *off = r.first;
            r.first += bytes;
            r.second -= bytes;
            if (!r.second) S->freeList.erase(S->freeList.begin() + (long)i);
            return true;
        }
    }
    return false;
}
void serve_free(ServeSession *S, size_t off, size_t bytes) {
    bytes = align256(bytes);
    auto it = S->freeList.begin();
    while (it != S->freeList.end() && it->first < off) ++it;
    it = S->freeList.insert(it, std::make_pair(off, bytes));
    if (it + 1 != S->freeList.end() && it->first + it->second == (it + 1)->first) {   // merge with the next range
        it->second += (it + 1)->second;
        S->freeList.erase(it + 1);
    }
    if (it != S->freeList.begin() && (it - 1)->first + (it - 1)->second == it->first) {   // and with the previous one
        (it - 1)->second += it->second;
        S->freeList.erase(it);
    }
}

void serve_release(ServeSession *S) {
    if (S->kst) cudaStreamSynchronize(S->kst);
    for (cudaStream_t s : {S->fst[0], S->fst[1], S->pst})
        if (s) cudaStreamSynchronize(s);
    for (auto &sl : S->slots) {
        if (sl.ev) cudaEventDestroy(sl.ev);
        if (sl.evFront) cudaEventDestroy(sl.evFront);
        if (sl.hCnt) cudaFreeHost(sl.hCnt);
        if (sl.hOrd) cudaFreeHost(sl.hOrd);
    }
    if (S->arena) cudaFree(S->arena);
    if (S->dTable) cudaFree(S->dTable);
    if (S->dQueue) cudaFree(S->dQueue);
    if (S->dCtl) cudaFree(S->dCtl);
    if (S->hTable) cudaFreeHost(S->hTable);
    if (S->hFlags) cudaFreeHost((void *)S->hFlags);
    if (S->hErr) cudaFreeHost(S->hErr);
    for (cudaStream_t s : {S->kst, S->fst[0], S->fst[1], S->pst})
        if (s) cudaStreamDestroy(s);
    if (S->kdone) cudaEventDestroy(S->kdone);
    delete S;
}

}  // namespace

#define IS_SCK(call)                                                                                                 \
    do {                                                                                                             \
        cudaError_t e_ = (call);                                                                                     \
        if (e_ != cudaSuccess) {                                                                                     \
            const int c_ = e_ == cudaErrorMemoryAllocation ? IS_ERR_OOM : IS_ERR_CUDA;                               \
            h->setErr(c_, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);                      \
            serve_release(S);                                                                                        \
            h->serve = nullptr;                                                                                      \
            return c_;                                                                                               \
        }                                                                                                            \
    } while (0)

extern "C" {

int is_serve_open(is_handle *h, int bit_depth, int chroma_444, uint64_t arena_bytes, int max_images, uint64_t max_leaves, int recon_ctas) {
    if (!h || h->serve || (bit_depth != 8 && bit_depth != 10) || (chroma_444 != 0 && chroma_444 != 1) || max_images < 1 ||
        max_images > 4096 || arena_bytes < (1u << 20) || max_leaves < 1 || recon_ctas < 0)
        return IS_ERR_INVALID;
    IS_CK(cudaSetDevice(h->device));
    ServeSession *S = new ServeSession();
    h->serve = S;
    S->bd = bit_depth;
    S->c444 = chroma_444;
    S->g = fmt_group(bit_depth, chroma_444);
    // the closed loop keeps part of the SMs free for the front ends of arriving images (a quarter when not given)
    const int full = h->rcGridG[S->g];
    S->grid = recon_ctas > 0 ? std::min(recon_ctas, full) : std::max(1, full * 3 / 4);
    S->arenaBytes = align256(arena_bytes);
    // queue positions: the leaves of every image the session will take, plus the slots idle workers give up (one per
    // worker each time the loop ends; max_leaves covers both, submit checks the leaves' share)
    S->warps = h->rcWarpsG[S->g];
    S->queueCap = (size_t)max_leaves + (size_t)S->grid * S->warps + 64;
    S->slots.resize(max_images);
    IS_SCK(cudaMalloc(&S->arena, S->arenaBytes));
    S->freeList.push_back(std::make_pair((size_t)0, S->arenaBytes));
    IS_SCK(cudaMalloc(&S->dTable, (size_t)max_images * sizeof(FrameDesc)));
    IS_SCK(cudaMalloc(&S->dQueue, S->queueCap * 8));
    IS_SCK(cudaMalloc(&S->dCtl, 64));
    IS_SCK(cudaMallocHost(&S->hTable, (size_t)max_images * sizeof(FrameDesc)));
    void *p = nullptr;
    IS_SCK(cudaHostAlloc(&p, (size_t)max_images * 4, cudaHostAllocMapped));
    S->hFlags = (volatile int *)p;
    IS_SCK(cudaHostGetDevicePointer((void **)&S->dFlags, p, 0));
    IS_SCK(cudaMallocHost(&S->hErr, 64));
    for (int i = 0; i < max_images; i++) S->hFlags[i] = 0;
    IS_SCK(cudaStreamCreateWithFlags(&S->kst, cudaStreamNonBlocking));
    for (auto &s : S->fst) IS_SCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    IS_SCK(cudaStreamCreateWithFlags(&S->pst, cudaStreamNonBlocking));
    IS_SCK(cudaEventCreateWithFlags(&S->kdone, cudaEventDisableTiming));
    // every host buffer of the session now: while its loop runs nothing may be freed (cudaFree / cudaFreeHost wait for
    // the device, which would wait for the loop)
    for (auto &sl : S->slots) {
        IS_SCK(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming));
        IS_SCK(cudaEventCreateWithFlags(&sl.evFront, cudaEventDisableTiming));
        IS_SCK(cudaMallocHost(&sl.hCnt, 16));
        IS_SCK(cudaMallocHost(&sl.hOrd, (size_t)2 * SERVE_MAX_SBS * 4));
    }
    IS_SCK(cudaMemsetAsync(S->dQueue, 0, S->queueCap * 8, S->kst));
    IS_SCK(cudaMemsetAsync(S->dCtl, 0, 64, S->kst));
    IS_SCK(cudaStreamSynchronize(S->kst));
    return IS_OK;
}

// (Re)launch the session's loop: it ends by itself after SERVE_IDLE_NS without work, so it holds its stream (and the
// hardware queue the stream runs on) only while there is work; an error the last run reported ends the session.
static int serve_launch(is_handle *h) {
    ServeSession *S = h->serve;
    RcCtl ctl;
    ctl.rq = S->dCtl;
    ctl.readyQ = S->dQueue;
    ctl.err = S->dCtl + 2;
    ctl.serving = 1;
    ctl.cap = (uint32_t)S->queueCap;
    ctl.readyWaitNs = SERVE_IDLE_NS;
    ctl.trace = nullptr;
    ctl.poison = h->poison ? 1 : 0;
    ctl.warps = rc_warps_for(h, S->g, 2);   // (a session's loop serves many images)
    const size_t sm = rc_launch_smem(S->g, ctl.warps);
    const FrameDesc *fs = S->dTable;
    const int g = S->g, grid = S->grid;
    IS_CK((g == 0 ? rc_launch<8, 1>(fs, 0, ctl, grid, sm, S->kst) : g == 1 ? rc_launch<8, 0>(fs, 0, ctl, grid, sm, S->kst)
           : g == 2 ? rc_launch<10, 1>(fs, 0, ctl, grid, sm, S->kst) : rc_launch<10, 0>(fs, 0, ctl, grid, sm, S->kst)));
    IS_CK(cudaEventRecord(S->kdone, S->kst));
    return IS_OK;
}
// the loop is running, or has ended cleanly and is launched again; IS_ERR_TIMEOUT if it ended with an error
static int serve_ensure_loop(is_handle *h) {
    ServeSession *S = h->serve;
    const cudaError_t q = cudaEventQuery(S->kdone);
    if (q == cudaErrorNotReady) return IS_OK;
    IS_CK(q);
    IS_CK(cudaMemcpyAsync(S->hErr, S->dCtl + 2, 4, cudaMemcpyDeviceToHost, S->kst));
    IS_CK(cudaStreamSynchronize(S->kst));
    if (*S->hErr) return h->setErr(IS_ERR_TIMEOUT, "the session's closed loop reported error %d", *S->hErr);
    return serve_launch(h);
}

// Starts the session's loop.  No allocation happens here or while the session is open (page-locked and device
// allocations and frees wait for running kernels: a process with several sessions opens them all, then starts them).
int is_serve_start(is_handle *h) {
    if (!h || !h->serve || h->serve->started) return IS_ERR_INVALID;
    IS_CK(cudaSetDevice(h->device));
    const int rc = serve_launch(h);
    if (!rc) h->serve->started = true;
    return rc;
}

// Nothing here allocates or frees device or pinned memory (the session's loop is running).
int is_serve_submit(is_handle *h, const is_frame *f, int from_host, int *ticket) {
    if (!h || !h->serve || !h->serve->started || !f || !ticket) return IS_ERR_INVALID;
    ServeSession *S = h->serve;
    IS_CK(cudaSetDevice(h->device));
    int bd = 0, c444 = 0;
    frame_format(h, f, &bd, &c444);
    if (f->width < 1 || f->height < 1 || f->width > 16384 || f->height > 16384 || f->qindex < 1 || f->qindex > 255)
        return h->setErr(IS_ERR_INVALID, "invalid frame (size %dx%d, qindex %d)", f->width, f->height, f->qindex);
    if (bd != S->bd || c444 != S->c444) return h->setErr(IS_ERR_INVALID, "the frame's format is not the session's");
    for (int p = 0; p < 3; p++) {
        const int ss = (p && !c444) ? 1 : 0, vw = (f->width + ss) >> ss;
        if (!f->planes[p] || f->pitch[p] < vw) return h->setErr(IS_ERR_INVALID, "invalid plane %d", p);
    }
    int slot = -1;
    for (int i = 0; i < (int)S->slots.size() && slot < 0; i++)
        if (S->slots[i].state == 0) slot = i;
    if (slot < 0) return h->setErr(IS_ERR_BUSY, "no free image slot");
    ServeSlot &sl = S->slots[slot];
    FrameDesc F;
    memset(&F, 0, sizeof F);
    int nSb = 0;
    const size_t bytes = layout(f->width, f->height, bd, c444, nullptr, F, nSb);
    const int maxLeaves = nSb * SB_MAX_LEAVES;
    // positions taken so far (leaves and given-up slots alike) plus this image's leaves and a full set of idle workers
    int64_t taken = 0;
    IS_CK(cudaMemcpyAsync(S->hErr + 4, S->dCtl, 8, cudaMemcpyDeviceToHost, S->pst));
    IS_CK(cudaStreamSynchronize(S->pst));
    taken = std::max<int64_t>(S->hErr[4], S->hErr[5]);
    if ((size_t)taken + S->inflightLeaves + (size_t)maxLeaves + 2 * (size_t)S->grid * S->warps + 64 > S->queueCap)
        return h->setErr(IS_ERR_STATE, "the session's queue positions are used up (close and open a new session)");
    size_t off = 0;
    if (!serve_alloc(S, bytes, &off)) return h->setErr(IS_ERR_BUSY, "no free workspace range of %zu bytes", bytes);
    memset(&F, 0, sizeof F);
    layout(f->width, f->height, bd, c444, S->arena + off, F, nSb);
    std::vector<int> cs, rs;
    min_tiles(f->width, f->height, cs, rs);
    if (cs.size() > 65 || rs.size() > 65) { serve_free(S, off, bytes); return h->setErr(IS_ERR_INVALID, "too many tiles"); }
    F.tileCols = (int)cs.size() - 1; F.tileRows = (int)rs.size() - 1;
    for (size_t k = 0; k < cs.size(); k++) F.tileColStart[k] = cs[k];
    for (size_t k = 0; k < rs.size(); k++) F.tileRowStart[k] = rs[k];
    F.qidx = f->qindex;
    F.qctx = av1g_coeff_cdf_q_ctx(f->qindex);
    lambda_fx(f->qindex, bd, &F.lam, &F.sqlam);
    F.dcQ = AV1G_T(Dc_Qlookup)[bd == 10][f->qindex];
    F.acQ = AV1G_T(Ac_Qlookup)[bd == 10][f->qindex];
    sl.gen = (sl.gen + 1) & 0x7FFF;
    F.readyQ = S->dQueue;
    F.readyCap = (uint32_t)S->queueCap;
    F.rq = S->dCtl;
    F.err = S->dCtl + 2;
    F.img = slot | (sl.gen << 16);
    F.leafDoneCnt = F.queue + 3;
    F.doneFlag = S->dFlags + slot;
    F.leafTrace = nullptr;
    if (!h->slOn) F.slCand = nullptr;
    F.slRdK = h->slOn ? h->slRdK : 4;
    F.rdK = h->rdK;
    F.txKeep = h->txKeep;
    F.waitIters = h->waitIters;
    F.readyWaitNs = h->readyWaitNs;
    F.poison = 0;
    sb_orders(F, cs, rs, sl.hOrd, sl.hOrd + nSb);
    S->hTable[slot] = F;
    S->hFlags[slot] = 0;
    // the front end on the next front stream: the descriptor first (the kernel reads it when it takes the image's first
    // leaf, which the front end's last kernels queue), the orders and counters, then the search's front kernels
    cudaStream_t st = S->fst[S->nextFront];
    const int k = S->nextFront;
    S->nextFront ^= 1;
    IS_CK(cudaMemcpyAsync(S->dTable + slot, S->hTable + slot, sizeof(FrameDesc), cudaMemcpyHostToDevice, st));
    IS_CK(cudaMemcpyAsync((void *)F.sbOrder, sl.hOrd, (size_t)nSb * 4, cudaMemcpyHostToDevice, st));
    IS_CK(cudaMemcpyAsync(F.sbDecodeOrder, sl.hOrd + nSb, (size_t)nSb * 4, cudaMemcpyHostToDevice, st));
    IS_CK(cudaMemsetAsync(F.queue, 0, 16, st));
    const int rc = front_end(h, F, f, nSb, from_host != 0, st, k, nullptr, nullptr);
    if (rc) return rc;   // (the slot stays taken: the session is not usable after a failed launch)
    IS_CK(cudaEventRecord(sl.evFront, st));
    sl.state = 1;
    sl.off = off;
    sl.bytes = bytes;
    sl.F = F;
    sl.nSb = nSb;
    sl.qidx = f->qindex;
    sl.maxLeaves = maxLeaves;
    S->inflightLeaves += (size_t)maxLeaves;
    *ticket = F.img;
    return IS_OK;   // (is_serve_poll starts the loop once the front end has queued leaves)
}

int is_serve_poll(is_handle *h, int *tickets, int cap, int *n) {
    if (!h || !h->serve || !n || (cap > 0 && !tickets)) return IS_ERR_INVALID;
    ServeSession *S = h->serve;
    IS_CK(cudaSetDevice(h->device));
    *n = 0;
    bool active = false;
    for (size_t i = 0; i < S->slots.size(); i++) {
        ServeSlot &sl = S->slots[i];
        if (sl.state == 1 && S->hFlags[i] == sl.F.img) {   // its last leaf is done: pack its record, download the counts
            const FrameDesc &F = sl.F;
            k_pack_scan<<<1, 1024, 0, S->pst>>>(F, sl.nSb);
            k_pack<<<sl.nSb, 256, 0, S->pst>>>(F, sl.nSb);
            IS_CK(cudaGetLastError());
            IS_CK(cudaMemcpyAsync(sl.hCnt, F.offBlk + sl.nSb, 4, cudaMemcpyDeviceToHost, S->pst));
            IS_CK(cudaMemcpyAsync(sl.hCnt + 1, F.offTxb + sl.nSb, 4, cudaMemcpyDeviceToHost, S->pst));
            IS_CK(cudaMemcpyAsync(sl.hCnt + 2, F.offCoef + sl.nSb, 8, cudaMemcpyDeviceToHost, S->pst));
            IS_CK(cudaEventRecord(sl.ev, S->pst));
            sl.state = 2;
            S->inflightLeaves -= (size_t)sl.maxLeaves;
        }
        if (sl.state == 2) {
            const cudaError_t q = cudaEventQuery(sl.ev);
            if (q == cudaSuccess) {
                sl.state = 3;
                if (*n < cap) tickets[(*n)++] = sl.F.img;
            } else if (q != cudaErrorNotReady) {
                IS_CK(q);
            }
        }
        // an image whose front end is done has leaves in the queue (or in progress): the loop must be running
        if (sl.state == 1 && !active) active = cudaEventQuery(sl.evFront) == cudaSuccess;
    }
    if (active) return serve_ensure_loop(h);
    return IS_OK;
}

static ServeSlot *serve_slot(is_handle *h, int ticket) {
    if (!h || !h->serve) return nullptr;
    const int slot = ticket & 0xFFFF;
    if (slot < 0 || slot >= (int)h->serve->slots.size()) return nullptr;
    ServeSlot &sl = h->serve->slots[slot];
    return (sl.state == 3 && sl.F.img == ticket) ? &sl : nullptr;
}

int is_serve_counts(is_handle *h, int ticket, uint32_t *n_blocks, uint32_t *n_txb, uint64_t *n_coeffs) {
    ServeSlot *sl = serve_slot(h, ticket);
    if (!sl) return IS_ERR_STATE;
    if (n_blocks) *n_blocks = sl->hCnt[0];
    if (n_txb) *n_txb = sl->hCnt[1];
    if (n_coeffs) memcpy(n_coeffs, sl->hCnt + 2, 8);
    return IS_OK;
}

int is_serve_copy(is_handle *h, int ticket, av1g_frame_params *fp, av1g_block *blocks, uint32_t *block_txb, av1g_txb *txb, int16_t *coeffs,
                  void *recon[3], const int32_t recon_pitch[3]) {
    ServeSlot *sl = serve_slot(h, ticket);
    if (!sl) return IS_ERR_STATE;
    ServeSession *S = h->serve;
    IS_CK(cudaSetDevice(h->device));
    const FrameDesc &F = sl->F;
    const uint32_t nb = sl->hCnt[0], nt = sl->hCnt[1];
    uint64_t nc = 0;
    memcpy(&nc, sl->hCnt + 2, 8);
    cudaStream_t st = S->pst;
    if (fp) {
        memset(fp, 0, sizeof *fp);
        fp->version = AV1G_DECISIONS_VERSION;
        fp->width = (uint32_t)F.W; fp->height = (uint32_t)F.H;
        fp->base_q_idx = (uint8_t)sl->qidx;
        fp->tile_cols_log2 = -1; fp->tile_rows_log2 = -1;
        fp->qm_y = fp->qm_u = fp->qm_v = 15;
        fp->chroma_format = F.ssx ? AV1G_CHROMA_420 : AV1G_CHROMA_444;
        fp->bit_depth = (uint8_t)F.bd;
    }
    if (blocks) IS_CK(cudaMemcpyAsync(blocks, F.recBlocks, (size_t)nb * sizeof(av1g_block), cudaMemcpyDeviceToHost, st));
    if (block_txb) IS_CK(cudaMemcpyAsync(block_txb, F.recBlockTxb, ((size_t)nb + 1) * 4, cudaMemcpyDeviceToHost, st));
    if (txb) IS_CK(cudaMemcpyAsync(txb, F.recTxb, (size_t)nt * sizeof(av1g_txb), cudaMemcpyDeviceToHost, st));
    if (coeffs) IS_CK(cudaMemcpyAsync(coeffs, F.recCoeffs, (size_t)nc * 2, cudaMemcpyDeviceToHost, st));
    const size_t px = F.bd > 8 ? 2 : 1;
    for (int p = 0; p < 3; p++) {
        if (!recon || !recon[p]) continue;
        const int ss = p ? F.ssx : 0;
        const int vw = (F.W + ss) >> ss, vh = (F.H + ss) >> ss;
        IS_CK(cudaMemcpy2DAsync(recon[p], (recon_pitch ? recon_pitch[p] : vw) * px, F.rec[p], F.rpitch[p] * px, vw * px, vh,
                                cudaMemcpyDeviceToHost, st));
    }
    IS_CK(cudaStreamSynchronize(st));
    serve_free(S, sl->off, sl->bytes);
    sl->state = 0;
    return IS_OK;
}

// Ends the session's loop without freeing anything (frees wait for every running kernel: a process with several
// sessions stops them all before it closes them).  Images whose leaves are in the running loop are completed, others are
// abandoned; none is read out.
int is_serve_stop(is_handle *h) {
    if (!h || !h->serve) return IS_ERR_INVALID;
    ServeSession *S = h->serve;
    if (!S->started || S->stopped) return IS_OK;
    cudaSetDevice(h->device);
    // the loop ends when it has no work (2 ms after its last leaf); no new launch follows
    for (auto &s : S->fst) cudaStreamSynchronize(s);
    cudaError_t e = cudaStreamSynchronize(S->kst);
    S->stopped = true;
    if (e == cudaSuccess) e = cudaMemcpyAsync(S->hErr, S->dCtl + 2, 4, cudaMemcpyDeviceToHost, S->kst);
    if (e == cudaSuccess) e = cudaStreamSynchronize(S->kst);
    if (e != cudaSuccess) return h->setErr(IS_ERR_CUDA, "closed loop: %s", cudaGetErrorString(e));
    if (*S->hErr) return h->setErr(IS_ERR_TIMEOUT, "the session's closed loop reported error %d", *S->hErr);
    return IS_OK;
}

int is_serve_close(is_handle *h) {
    if (!h || !h->serve) return IS_ERR_INVALID;
    const int rc = is_serve_stop(h);
    serve_release(h->serve);
    h->serve = nullptr;
    return rc;
}

}  // extern "C"
