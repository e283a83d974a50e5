// is_k_rc.cu - the closed-loop unit: k_recon of one format (IS_BD 8 / 10 and IS_SS 1 (4:2:0) / 0 (4:4:4), set on the
// compiler command line), its table upload, occupancy and cooperative launch.
#include "is_units.cuh"
#include "is_recon.cuh"

#if !defined(IS_BD) || !defined(IS_SS)
#error "IS_BD (8 or 10) and IS_SS (1 or 0) must be defined"
#endif

namespace is {

typedef RcPxOf<IS_BD> RcPx;
constexpr int RcNW = rc_warps_of<IS_BD, IS_SS>();

template <> cudaError_t rc_upload<IS_BD, IS_SS>(const TableBlob &B) { return upload_common(B); }

template <> size_t rc_smem<IS_BD, IS_SS>(int warps) { return rc_smem_bytes<RcPx, IS_SS>(warps); }

template <> cudaError_t rc_setup<IS_BD, IS_SS>(size_t *smem, int *ctasPerSm, int *warps) {
    const void *k = (const void *)k_recon<IS_BD, IS_SS>;
    *smem = sizeof(RcSmem<RcPx, IS_SS, RcNW>);
    *warps = RcNW;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctasPerSm, k, RcNW * 32, *smem);
    return e;
}

// A batch's loop is a cooperative launch (all CTAs resident at once), expressed with launch attributes so that it can be
// captured in a graph.  A serving session's loop is a plain launch: it runs next to other loops and front ends, and it
// needs no co-residency - a queue slot is only ever claimed by a warp that is running, and every wait is on a leaf that a
// running warp holds.
template <> cudaError_t rc_launch<IS_BD, IS_SS>(const FrameDesc *fs, int nImg, const RcCtl &ctl, int grid, size_t smem, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(RcNW * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = ctl.serving ? 0 : 1;
    return cudaLaunchKernelEx(&cfg, k_recon<IS_BD, IS_SS>, fs, nImg, ctl);
}

}  // namespace is
