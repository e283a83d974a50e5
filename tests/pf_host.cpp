// Host build of the library's post-filter arithmetic (av1gpu_b200/csrc/is_postfilter.cuh) for the CPU tests: the maps
// from the blocks, deblocking (vertical edges of every plane, then horizontal ones) and CDEF into a copy, in the order the
// device kernels use.  Test infrastructure only: the library itself runs these functions on the GPU.
#include "is_postfilter.cuh"
#include <cstring>
#include <vector>

using namespace is;

template <typename P>
static void run(PfFrame &f, void *planes[3], const int stride[3]) {
    if (f.lvl[0] || f.lvl[1])
        for (int pass = 0; pass < 2; pass++)
            for (int p = 0; p < 3; p++) {
                const int sx = p ? f.ssx : 0, sy = p ? f.ssy : 0;
                const int r4 = f.MiRows >> sy, c4 = f.MiCols >> sx;
                P *pl = (P *)planes[p];
                for (int y4 = 0; y4 < r4; y4++)
                    for (int x4 = 0; x4 < c4; x4++) {
                        PfEdge e;
                        if (!pf_edge(f, p, pass, x4, y4, e)) continue;
                        for (int i = 0; i < 4; i++) {
                            if (pass == 0) pf_line(pl + (size_t)(4 * y4 + i) * stride[p] + 4 * x4, 1, p, e, f.bd);
                            else pf_line(pl + (size_t)(4 * y4) * stride[p] + 4 * x4 + i, (ptrdiff_t)stride[p], p, e, f.bd);
                        }
                    }
            }
    if (!f.cdefOn) return;
    std::vector<P> out[3];
    for (int p = 0; p < 3; p++) {
        const int sy = p ? f.ssy : 0;
        const P *pl = (const P *)planes[p];
        out[p].assign(pl, pl + (size_t)stride[p] * ((f.MiRows * 4) >> sy));
    }
    for (int r = 0; r < f.MiRows; r += 2)
        for (int c = 0; c < f.MiCols; c += 2) {
            const int idx = pf_cdef_idx(f, r, c);
            if (idx < 0) continue;
            int dir, var;
            pf_cdef_dir((const P *)planes[0] + (size_t)(4 * r) * stride[0] + 4 * c, (ptrdiff_t)stride[0], f.bd, dir, var);
            for (int p = 0; p < 3; p++) {
                const int sx = p ? f.ssx : 0, sy = p ? f.ssy : 0;
                const PfCdef cp = pf_cdef_plane(f, p, idx, dir, var);
                for (int y = (4 * r) >> sy; y < (4 * r + 8) >> sy; y++)
                    for (int x = (4 * c) >> sx; x < (4 * c + 8) >> sx; x++)
                        out[p][(size_t)y * stride[p] + x] = (P)pf_cdef_sample(f, (const P *)planes[p], (ptrdiff_t)stride[p], p, x, y, cp);
            }
        }
    for (int p = 0; p < 3; p++) memcpy(planes[p], out[p].data(), out[p].size() * sizeof(P));
}

extern "C" int pfh_apply(const av1g_frame_params *fp, const av1g_block *blocks, uint32_t n, void *planes[3], const int stride[3]) {
    PfFrame f;
    pf_init(*fp, f);
    const size_t mi = (size_t)f.MiCols * f.MiRows, cmi = (size_t)(f.MiCols >> f.ssx) * (f.MiRows >> f.ssy);
    std::vector<uint8_t> skip(mi), t0(mi), t1(cmi), t2(cmi);
    std::vector<int8_t> cidx((size_t)f.sbCols * ((f.MiRows + 15) >> 4), -1);
    f.skip = skip.data();
    f.txs[0] = t0.data(); f.txs[1] = t1.data(); f.txs[2] = t2.data();
    f.cdefIdx = cidx.data();
    for (uint32_t i = 0; i < n; i++) pf_mark_block(f, blocks[i]);
    if (f.bd == 10) run<uint16_t>(f, planes, stride);
    else run<uint8_t>(f, planes, stride);
    return 0;
}
