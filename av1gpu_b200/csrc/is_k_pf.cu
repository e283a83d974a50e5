// is_k_pf.cu - the post-filters on the device: deblocking (one thread per filtered line, vertical edges of every plane,
// then horizontal ones) and CDEF (one thread per 8x8 luma block for the direction search, then one thread per output
// sample of each plane), applied to a reconstruction in device memory.  The arithmetic is is_postfilter.cuh's.
#include "is_units.cuh"
#include "is_postfilter.cuh"
#include <algorithm>

namespace is {

// the maps from the record's blocks; with sbCdef, every block's cdef_idx becomes its 64x64's entry (written back)
__global__ void k_pf_maps(PfFrame f, av1g_block *blocks, uint32_t n, const int8_t *sbCdef) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    av1g_block b = blocks[i];
    if (b.mi_row >= f.MiRows || b.mi_col >= f.MiCols || b.bsize >= 22) return;
    if (sbCdef) {
        b.cdef_idx = sbCdef[(b.mi_row >> 4) * f.sbCols + (b.mi_col >> 4)];
        blocks[i].cdef_idx = b.cdef_idx;
    }
    pf_mark_block(f, b);
}

struct PfPlanes {
    uint8_t *p[3];
    int pitch[3];   // samples
};

// pass 0: x = edge column (4x4 units), y = sample row; pass 1: x = sample column, y = edge row; z = plane
template <typename P>
__global__ void k_pf_deblock(PfFrame f, PfPlanes pl, int pass) {
    const int plane = blockIdx.z, sx = plane ? f.ssx : 0, sy = plane ? f.ssy : 0;
    const int rows = (f.MiRows * 4) >> sy, cols = (f.MiCols * 4) >> sx;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    P *base = reinterpret_cast<P *>(pl.p[plane]);
    const int pitch = pl.pitch[plane];
    PfEdge e;
    if (pass == 0) {
        if (x >= cols / 4 || y >= rows || !pf_edge(f, plane, 0, x, y >> 2, e)) return;
        pf_line(base + (size_t)y * pitch + 4 * x, 1, plane, e, f.bd);
    } else {
        if (x >= cols || y >= rows / 4 || !pf_edge(f, plane, 1, x >> 2, y, e)) return;
        pf_line(base + (size_t)(4 * y) * pitch + x, (ptrdiff_t)pitch, plane, e, f.bd);
    }
}

// per 8x8 luma block: -1 when CDEF leaves it, else var << 7 | direction << 4 | cdef_idx
template <typename P>
__global__ void k_pf_cdef_dir(PfFrame f, const P *y, int pitch, int32_t *info) {
    const int bx = blockIdx.x * blockDim.x + threadIdx.x, by = blockIdx.y * blockDim.y + threadIdx.y;
    const int nbx = f.MiCols / 2, nby = f.MiRows / 2;
    if (bx >= nbx || by >= nby) return;
    const int idx = pf_cdef_idx(f, 2 * by, 2 * bx);
    int32_t v = -1;
    if (idx >= 0) {
        int dir, var;
        pf_cdef_dir(y + (size_t)(8 * by) * pitch + 8 * bx, (ptrdiff_t)pitch, f.bd, dir, var);
        v = (var << 7) | (dir << 4) | idx;
    }
    info[(size_t)by * nbx + bx] = v;
}

// every sample of the coded area of each plane (z): CDEF of the deblocked plane src into dst
template <typename P>
__global__ void k_pf_cdef(PfFrame f, PfPlanes src, PfPlanes dst, const int32_t *info) {
    const int plane = blockIdx.z, sx = plane ? f.ssx : 0, sy = plane ? f.ssy : 0;
    const int rows = (f.MiRows * 4) >> sy, cols = (f.MiCols * 4) >> sx;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= cols || y >= rows) return;
    const P *s = reinterpret_cast<const P *>(src.p[plane]);
    const int sp = src.pitch[plane];
    const int32_t v = info[(size_t)((y << sy) >> 3) * (f.MiCols / 2) + ((x << sx) >> 3)];
    int out = s[(size_t)y * sp + x];
    if (v >= 0) out = pf_cdef_sample(f, s, (ptrdiff_t)sp, plane, x, y, pf_cdef_plane(f, plane, v & 15, (v >> 4) & 7, v >> 7));
    reinterpret_cast<P *>(dst.p[plane])[(size_t)y * dst.pitch[plane] + x] = (P)out;
}

// ---- host ----
size_t pf_scratch_bytes(int W, int H, int bd, int c444) {
    const int MiCols = 2 * ((W + 7) >> 3), MiRows = 2 * ((H + 7) >> 3), sbCols = (MiCols + 15) >> 4, sbRows = (MiRows + 15) >> 4;
    const size_t px = bd > 8 ? 2 : 1, mi = (size_t)MiCols * MiRows, cmi = c444 ? mi : mi / 4;
    auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
    return al(mi) + al(mi) + 2 * al(cmi) + al((size_t)sbCols * sbRows) * 2 + al(mi / 4 * 4) + al(mi * 16 * px) + 2 * al(cmi * 16 * px);
}

int pf_launch(const av1g_frame_params &fp, av1g_block *blocks, uint32_t nBlocks, const int8_t *sbCdefHost, uint8_t *const rec[3],
              const int rpitch[3], void *scratch, size_t scratchBytes, cudaStream_t s, std::string *err) {
    PfFrame f;
    pf_init(fp, f);
    const int sbRows = (f.MiRows + 15) >> 4;
    const size_t px = f.bd > 8 ? 2 : 1, mi = (size_t)f.MiCols * f.MiRows, cmi = f.ssx ? mi / 4 : mi;
    const int c444 = f.ssx ? 0 : 1;
    if (scratchBytes < pf_scratch_bytes(f.W, f.H, f.bd, c444)) { if (err) *err = "post-filter scratch too small"; return IS_ERR_INVALID; }
    auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
    uint8_t *S = (uint8_t *)scratch;
    size_t at = 0;
    auto take = [&](size_t b) { uint8_t *p = S + at; at += al(b); return p; };
    f.skip = take(mi);
    f.txs[0] = take(mi);
    f.txs[1] = take(cmi);
    f.txs[2] = take(cmi);
    f.cdefIdx = (int8_t *)take((size_t)f.sbCols * sbRows);
    int8_t *sbCdef = (int8_t *)take((size_t)f.sbCols * sbRows);
    int32_t *info = (int32_t *)take(mi / 4 * 4);
    PfPlanes tmp, recP;
    for (int p = 0; p < 3; p++) {
        const int sx = p ? f.ssx : 0, sy = p ? f.ssy : 0;
        tmp.pitch[p] = (f.MiCols * 4) >> sx;
        tmp.p[p] = take((size_t)tmp.pitch[p] * ((f.MiRows * 4) >> sy) * px);
        recP.p[p] = rec[p];
        recP.pitch[p] = rpitch[p];
    }
    cudaError_t e = cudaMemsetAsync(f.cdefIdx, 0xFF, (size_t)f.sbCols * sbRows, s);
    if (e == cudaSuccess && sbCdefHost) e = cudaMemcpyAsync(sbCdef, sbCdefHost, (size_t)f.sbCols * sbRows, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) { if (err) *err = cudaGetErrorString(e); return IS_ERR_CUDA; }
    k_pf_maps<<<(nBlocks + 255) / 256, 256, 0, s>>>(f, blocks, nBlocks, sbCdefHost ? sbCdef : nullptr);
    const bool deblock = f.lvl[0] || f.lvl[1];
    const dim3 tb(32, 8);
    const int rows = f.MiRows * 4, cols = f.MiCols * 4;
    if (deblock) {
        const dim3 g0((cols / 4 + 31) / 32, (rows + 7) / 8, 3), g1((cols + 31) / 32, (rows / 4 + 7) / 8, 3);
        if (px == 1) {
            k_pf_deblock<uint8_t><<<g0, tb, 0, s>>>(f, recP, 0);
            k_pf_deblock<uint8_t><<<g1, tb, 0, s>>>(f, recP, 1);
        } else {
            k_pf_deblock<uint16_t><<<g0, tb, 0, s>>>(f, recP, 0);
            k_pf_deblock<uint16_t><<<g1, tb, 0, s>>>(f, recP, 1);
        }
    }
    if (f.cdefOn) {
        const dim3 gd((f.MiCols / 2 + 31) / 32, (f.MiRows / 2 + 7) / 8), gc((cols + 31) / 32, (rows + 7) / 8, 3);
        if (px == 1) {
            k_pf_cdef_dir<uint8_t><<<gd, tb, 0, s>>>(f, rec[0], rpitch[0], info);
            k_pf_cdef<uint8_t><<<gc, tb, 0, s>>>(f, recP, tmp, info);
        } else {
            k_pf_cdef_dir<uint16_t><<<gd, tb, 0, s>>>(f, (const uint16_t *)rec[0], rpitch[0], info);
            k_pf_cdef<uint16_t><<<gc, tb, 0, s>>>(f, recP, tmp, info);
        }
        for (int p = 0; p < 3 && e == cudaSuccess; p++) {
            const int sx = p ? f.ssx : 0, sy = p ? f.ssy : 0;
            e = cudaMemcpy2DAsync(rec[p], rpitch[p] * px, tmp.p[p], tmp.pitch[p] * px, ((size_t)cols >> sx) * px, rows >> sy,
                                  cudaMemcpyDeviceToDevice, s);
        }
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) { if (err) *err = cudaGetErrorString(e); return IS_ERR_CUDA; }
    return IS_OK;
}

}  // namespace is
