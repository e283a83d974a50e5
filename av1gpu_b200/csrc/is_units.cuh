// is_units.cuh - the library's compilation units and what they export to the host orchestration (is_api.cu).
//
// The kernels are compiled in separate units so that they build in parallel: is_k_an.cu once per bit depth and kernel
// pair (the four analysis kernels), is_k_rc.cu once per format (the closed loop), is_k_ent.cu (entropy coding of the
// records), is_k_pf.cu (post-filters), is_api.cu (host API, DP, scheduling, pack, learned-shortlist and test kernels).  Device globals have internal linkage (static): every unit holds its own copy
// of the search's tables, and upload_tables() in is_api.cu fills each unit's copy from one host-built TableBlob.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "is_api.h"
#include "is_dev.cuh"
#include "is_frame.cuh"

namespace is {

// the host-built tables of the search (cost tables of the four q-contexts, averaged bits, packed scans, analysis task
// lists); the spec tables of av1core are copied by each unit from av1core's host arrays
struct TableBlob {
    std::vector<uint16_t> cost;            // 4 x NCDF
    int avgY[13];
    int avgPart[5][10];
    int avgSkip0;
    std::vector<uint16_t> scanPack;        // SCAN_PACK entries
    uint16_t scanOff[19][3];
    std::vector<uint8_t> anTask, anTaskBig;
    std::vector<int> anShapeStart, anShapeStartBig;
};

// the tables every unit indexes, into this unit's copies
static inline cudaError_t upload_common(const TableBlob &B) {
    cudaError_t e = B.cost.size() == (size_t)4 * NCDF && B.scanPack.size() == (size_t)SCAN_PACK ? cudaSuccess : cudaErrorInvalidValue;
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_cost, B.cost.data(), B.cost.size() * 2);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_avgY, B.avgY, sizeof B.avgY);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_avgPart, B.avgPart, sizeof B.avgPart);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_avgSkip0, &B.avgSkip0, sizeof B.avgSkip0);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_scanPack, B.scanPack.data(), B.scanPack.size() * 2);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_scanOff, B.scanOff, sizeof B.scanOff);
#define IS_UPLOAD_SPEC_TABLE(T, name, dims) \
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_##name, name##_host, sizeof(name##_host));
    IS_SPEC_TABLES(IS_UPLOAD_SPEC_TABLE)
#undef IS_UPLOAD_SPEC_TABLE
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_baseCtx, &AV1G_T(Coeff_Base_Ctx_Offset)[0][0][0], 19 * 25);
    return e;
}

// ---- analysis units (is_k_an.cu, BD 8 / 10 x PART 0: the warp-path kernels k_analysis_big and k_analysis, PART 1:
//      the per-thread kernels k_analysis_tiny and k_analysis_mid) ----
template <int BD, int PART> cudaError_t an_upload(const TableBlob &B);
template <int BD, int PART> cudaError_t an_setup();   // dynamic shared memory limits of the unit's kernels
template <int BD, int PART> cudaError_t an_launch(const FrameDesc &F, int nSb, cudaStream_t s);

// ---- closed-loop unit (is_k_rc.cu, BD 8 / 10 x SS 1 (4:2:0) / 0 (4:4:4)) ----
template <int BD, int SS> cudaError_t rc_upload(const TableBlob &B);
// shared memory of the kernel and its co-resident CTAs per SM (the cooperative grid is that times the SM count)
template <int BD, int SS> cudaError_t rc_setup(size_t *smem, int *ctasPerSm, int *warps);
template <int BD, int SS> size_t rc_smem(int warps);   // dynamic shared memory of a launch with that many working warps
struct RcCtl;
template <int BD, int SS> cudaError_t rc_launch(const FrameDesc *fs, int nImg, const RcCtl &ctl, int grid, size_t smem, cudaStream_t st);

// ---- entropy unit (is_k_ent.cu): records on the device -> tile payloads; OBU framing on the host ----
struct TileGeom {   // uniform tile spacing (spec 5.9.15): log2 counts, their legal ranges, tile sizes in SBs, counts
    int minLog2Cols, maxLog2Cols, minLog2Rows, maxLog2Rows, colsLog2, rowsLog2, wSb, hSb, cols, rows;
};
bool tile_info(int W, int H, int colsLog2, int rowsLog2, TileGeom &t);
cudaError_t ent_upload(const TableBlob &B);
int ent_scratch(const is_ent_frame *frames, int n, uint64_t cap, size_t *bytes, std::string *err);
int ent_launch(const is_ent_frame *frames, int n, uint64_t cap, void *scratch, size_t scratchBytes, cudaStream_t s, is_ent_out *out,
               uint32_t *frameTile0, std::string *err);
int obu_assemble(const av1g_frame_params &fp, const uint8_t *payload, const uint64_t *off, uint32_t nTiles, std::vector<uint8_t> &o,
                 std::string *err);
int avif_write(const av1g_frame_params &fp, const uint8_t *obu, size_t n, std::vector<uint8_t> &out, std::string *err);

// ---- post-filter unit (is_k_pf.cu): deblocking + CDEF of a reconstruction on the device ----
size_t pf_scratch_bytes(int W, int H, int bd, int c444);
int pf_launch(const av1g_frame_params &fp, av1g_block *blocks, uint32_t nBlocks, const int8_t *sbCdefHost, uint8_t *const rec[3],
              const int rpitch[3], void *scratch, size_t scratchBytes, cudaStream_t s, std::string *err);

}  // namespace is
