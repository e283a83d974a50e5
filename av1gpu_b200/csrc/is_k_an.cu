// is_k_an.cu - an analysis unit: two of the four open-loop analysis kernels of one sample bit depth (IS_BD 8 or 10;
// IS_AN_PART 0: the warp-path kernels k_analysis_big and k_analysis, 1: the per-thread kernels k_analysis_tiny and
// k_analysis_mid; both set on the compiler command line), their table upload and launches.
#include "is_units.cuh"
#include "is_analysis.cuh"
#include "is_tiny.cuh"

#if !defined(IS_BD) || !defined(IS_AN_PART)
#error "IS_BD (8 or 10) and IS_AN_PART (0 or 1) must be defined"
#endif

namespace is {

template <> cudaError_t an_upload<IS_BD, IS_AN_PART>(const TableBlob &B) {
    cudaError_t e = upload_common(B);
    const bool ok = B.anTask.size() == (size_t)AN_TASKS * 3 && B.anTaskBig.size() == (size_t)ANB_TASKS * 3 &&
                    B.anShapeStart.size() == (size_t)AN_SHAPES + 1 && B.anShapeStartBig.size() == (size_t)ANB_GROUPS + 1;
    if (e == cudaSuccess && !ok) e = cudaErrorInvalidValue;
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_anTask, B.anTask.data(), B.anTask.size());
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_anTaskBig, B.anTaskBig.data(), B.anTaskBig.size());
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_anShapeStart, B.anShapeStart.data(), B.anShapeStart.size() * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_anShapeStartBig, B.anShapeStartBig.data(), B.anShapeStartBig.size() * sizeof(int));
    return e;
}

typedef std::conditional<IS_BD == 8, uint8_t, uint16_t>::type AnPx;
static cudaError_t smem_attr(const void *k, size_t b) { return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b); }

#if IS_AN_PART == 0
static const size_t kSmemAn = sizeof(AnSmem<AnPx, AN_WARPS, AN_BUF_INTS>), kSmemAnBig = sizeof(AnSmem<AnPx, ANB_WARPS, ANB_BUF_INTS>);

template <> cudaError_t an_setup<IS_BD, 0>() {
    cudaError_t e = smem_attr((const void *)k_analysis<IS_BD>, kSmemAn);
    if (e == cudaSuccess) e = smem_attr((const void *)k_analysis_big<IS_BD>, kSmemAnBig);
    return e;
}

template <> cudaError_t an_launch<IS_BD, 0>(const FrameDesc &F, int nSb, cudaStream_t s) {
    k_analysis_big<IS_BD><<<ANB_GROUPS * nSb, ANB_WARPS * 32, kSmemAnBig, s>>>(F);
    k_analysis<IS_BD><<<AN_SHAPES * nSb, AN_WARPS * 32, kSmemAn, s>>>(F);
    return cudaGetLastError();
}
#else
template <> cudaError_t an_setup<IS_BD, 1>() {
    cudaError_t e = smem_attr((const void *)k_analysis_mid<IS_BD>, sizeof(MidSmem<AnPx>));
    if (e == cudaSuccess) e = smem_attr((const void *)k_analysis_tiny<IS_BD>, sizeof(TinySmem<AnPx>));
    return e;
}

template <> cudaError_t an_launch<IS_BD, 1>(const FrameDesc &F, int nSb, cudaStream_t s) {
    k_analysis_tiny<IS_BD><<<nSb, TINY_THREADS, sizeof(TinySmem<AnPx>), s>>>(F);
    k_analysis_mid<IS_BD><<<3 * ((nSb + MID_SBS - 1) / MID_SBS), MID_THREADS, sizeof(MidSmem<AnPx>), s>>>(F);
    return cudaGetLastError();
}
#endif

}  // namespace is
