// oracle/ref_shim.cpp - C entry to the reference's own CPU decision engine (av1core/src/ref_engine.cpp,
// ref_engine_encode at tools.h:66-77).  TEST / BASELINE INFRASTRUCTURE ONLY: bench.py times it beside the oracle as
// "the reference CPU engine".  It is a different, simpler algorithm than the search (NONE / SPLIT only,
// TX_MODE_LARGEST, at most 4 decide threads), so only its speed is reported, never its decisions.
#include "oracle.h"
#include "tools.h"
#include "av1f/tuneiq.h"

#include <cstring>
#include <string>

extern "C" int orc_ref_engine(const orc_image *img, double *sec_decide, double *sec_encode) {
    if (!img || img->bit_depth != 8 || img->chroma_444) return -1;
    av1g::Image im;
    im.W = img->width;
    im.H = img->height;
    im.mono = 0;
    for (int p = 0; p < 3; p++) {
        const int w = im.w(p), h = im.h(p);
        im.p[p].resize((size_t)w * h);
        const uint8_t *s = (const uint8_t *)img->planes[p];
        for (int y = 0; y < h; y++) memcpy(im.p[p].data() + (size_t)y * w, s + (size_t)y * img->stride[p], (size_t)w);
    }
    av1g::RefEngineOpts o;
    o.qindex = img->qindex;
    o.min_block = 4;
    av1g::OwnedRecord rec;
    av1g_output out;
    memset(&out, 0, sizeof out);
    av1g::RefEngineStats st;
    std::string err;
    const int rc = av1g::ref_engine_encode(im, o, rec, &out, &st, err);
    av1g_output_free(&out);
    if (sec_decide) *sec_decide = st.seconds_decide;
    if (sec_encode) *sec_encode = st.seconds_encode;
    return rc;
}

// The reference's frame-level post-filter decisions of its default (av1f/include/av1f/tuneiq.h av1f_tuneiq_frame_init:
// deblocking level from Q with the intra delta, sharpness, CDEF damping), the pin of the library's is_postfilter_from_q.
extern "C" void orc_ref_lf_from_q(int base, int bd, int *level, int *sharpness, int *damping) {
    av1f_tuneiq_frame t;
    av1f_tuneiq_frame_init(base, 1, 1, 0, &t, bd);
    *level = t.lf_level;
    *sharpness = t.lf_sharpness;
    *damping = t.cdef_damping;
}

