// GENERATED by gen_txfm.py from the AV1 inverse-transform step lists (spec 7.13.2). DO NOT EDIT.
// fwd_*: transposed networks (forward transforms of this project); inv_*: the spec inverse 1-D transforms
// with their conformance checks (return value: nonzero when a butterfly output left r bits).
#pragma once
#include <stdint.h>
#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif
__host__ __device__ __forceinline__ int32_t rnd12(int32_t x) { return (x + 2048) >> 12; }
__host__ __device__ __forceinline__ int32_t clampr(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

__host__ __device__ __forceinline__ void fwd_dct4(int32_t *T) {
    { const int32_t x_ = T[1], y_ = T[2]; T[1] = x_ + y_; T[2] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[3]; T[0] = x_ + y_; T[3] = x_ - y_; }
    { const int32_t x_ = rnd12(T[2] * 1567 - T[3] * -3784), y_ = rnd12(T[2] * -3784 + T[3] * 1567); T[2] = x_; T[3] = y_; }
    { const int32_t x_ = rnd12(T[0] * 2896 - T[1] * 2896), y_ = rnd12(T[0] * 2896 + T[1] * 2896); T[0] = y_; T[1] = x_; }
    {
        int32_t c_[4];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3];
        T[0] = c_[0];
        T[2] = c_[1];
        T[1] = c_[2];
        T[3] = c_[3];
    }
}
__host__ __device__ __forceinline__ uint32_t inv_dct4(int32_t *T, int r) {
    uint32_t e_ = 0;
    const int32_t lo_ = -(1 << (r - 1)), hi_ = (1 << (r - 1)) - 1;
    {
        int32_t c_[4];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3];
        T[0] = c_[0];
        T[1] = c_[2];
        T[2] = c_[1];
        T[3] = c_[3];
    }
    { const int32_t x_ = rnd12(T[0] * 2896 - T[1] * 2896), y_ = rnd12(T[0] * 2896 + T[1] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[1] = x_; T[0] = y_; }
    { const int32_t x_ = rnd12(T[2] * 1567 - T[3] * 3784), y_ = rnd12(T[2] * 3784 + T[3] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[2] = x_; T[3] = y_; }
    { const int32_t x_ = T[0], y_ = T[3]; T[0] = clampr(x_ + y_, lo_, hi_); T[3] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[2]; T[1] = clampr(x_ + y_, lo_, hi_); T[2] = clampr(x_ - y_, lo_, hi_); }
    return e_;
}
__host__ __device__ __forceinline__ void fwd_dct8(int32_t *T) {
    { const int32_t x_ = T[3], y_ = T[4]; T[3] = x_ + y_; T[4] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[5]; T[2] = x_ + y_; T[5] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[6]; T[1] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[7]; T[0] = x_ + y_; T[7] = x_ - y_; }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[5] * 2896), y_ = rnd12(T[6] * 2896 + T[5] * 2896); T[6] = y_; T[5] = x_; }
    { const int32_t x_ = T[1], y_ = T[2]; T[1] = x_ + y_; T[2] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[3]; T[0] = x_ + y_; T[3] = x_ - y_; }
    { const int32_t x_ = T[7], y_ = T[6]; T[7] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[5]; T[4] = x_ + y_; T[5] = x_ - y_; }
    { const int32_t x_ = rnd12(T[2] * 1567 - T[3] * -3784), y_ = rnd12(T[2] * -3784 + T[3] * 1567); T[2] = x_; T[3] = y_; }
    { const int32_t x_ = rnd12(T[0] * 2896 - T[1] * 2896), y_ = rnd12(T[0] * 2896 + T[1] * 2896); T[0] = y_; T[1] = x_; }
    { const int32_t x_ = rnd12(T[5] * 3406 - T[6] * -2276), y_ = rnd12(T[5] * -2276 + T[6] * 3406); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = rnd12(T[4] * 799 - T[7] * -4017), y_ = rnd12(T[4] * -4017 + T[7] * 799); T[4] = x_; T[7] = y_; }
    {
        int32_t c_[8];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7];
        T[0] = c_[0];
        T[4] = c_[1];
        T[2] = c_[2];
        T[6] = c_[3];
        T[1] = c_[4];
        T[5] = c_[5];
        T[3] = c_[6];
        T[7] = c_[7];
    }
}
__host__ __device__ __forceinline__ uint32_t inv_dct8(int32_t *T, int r) {
    uint32_t e_ = 0;
    const int32_t lo_ = -(1 << (r - 1)), hi_ = (1 << (r - 1)) - 1;
    {
        int32_t c_[8];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7];
        T[0] = c_[0];
        T[1] = c_[4];
        T[2] = c_[2];
        T[3] = c_[6];
        T[4] = c_[1];
        T[5] = c_[5];
        T[6] = c_[3];
        T[7] = c_[7];
    }
    { const int32_t x_ = rnd12(T[4] * 799 - T[7] * 4017), y_ = rnd12(T[4] * 4017 + T[7] * 799); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[4] = x_; T[7] = y_; }
    { const int32_t x_ = rnd12(T[5] * 3406 - T[6] * 2276), y_ = rnd12(T[5] * 2276 + T[6] * 3406); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = rnd12(T[0] * 2896 - T[1] * 2896), y_ = rnd12(T[0] * 2896 + T[1] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[1] = x_; T[0] = y_; }
    { const int32_t x_ = rnd12(T[2] * 1567 - T[3] * 3784), y_ = rnd12(T[2] * 3784 + T[3] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[2] = x_; T[3] = y_; }
    { const int32_t x_ = T[4], y_ = T[5]; T[4] = clampr(x_ + y_, lo_, hi_); T[5] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[7], y_ = T[6]; T[7] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[0], y_ = T[3]; T[0] = clampr(x_ + y_, lo_, hi_); T[3] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[2]; T[1] = clampr(x_ + y_, lo_, hi_); T[2] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[5] * 2896), y_ = rnd12(T[6] * 2896 + T[5] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = T[0], y_ = T[7]; T[0] = clampr(x_ + y_, lo_, hi_); T[7] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[6]; T[1] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[5]; T[2] = clampr(x_ + y_, lo_, hi_); T[5] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[4]; T[3] = clampr(x_ + y_, lo_, hi_); T[4] = clampr(x_ - y_, lo_, hi_); }
    return e_;
}
__host__ __device__ __forceinline__ void fwd_dct16(int32_t *T) {
    { const int32_t x_ = T[7], y_ = T[8]; T[7] = x_ + y_; T[8] = x_ - y_; }
    { const int32_t x_ = T[6], y_ = T[9]; T[6] = x_ + y_; T[9] = x_ - y_; }
    { const int32_t x_ = T[5], y_ = T[10]; T[5] = x_ + y_; T[10] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[11]; T[4] = x_ + y_; T[11] = x_ - y_; }
    { const int32_t x_ = T[3], y_ = T[12]; T[3] = x_ + y_; T[12] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[13]; T[2] = x_ + y_; T[13] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[14]; T[1] = x_ + y_; T[14] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[15]; T[0] = x_ + y_; T[15] = x_ - y_; }
    { const int32_t x_ = rnd12(T[12] * 2896 - T[11] * 2896), y_ = rnd12(T[12] * 2896 + T[11] * 2896); T[12] = y_; T[11] = x_; }
    { const int32_t x_ = rnd12(T[13] * 2896 - T[10] * 2896), y_ = rnd12(T[13] * 2896 + T[10] * 2896); T[13] = y_; T[10] = x_; }
    { const int32_t x_ = T[3], y_ = T[4]; T[3] = x_ + y_; T[4] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[5]; T[2] = x_ + y_; T[5] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[6]; T[1] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[7]; T[0] = x_ + y_; T[7] = x_ - y_; }
    { const int32_t x_ = T[14], y_ = T[13]; T[14] = x_ + y_; T[13] = x_ - y_; }
    { const int32_t x_ = T[15], y_ = T[12]; T[15] = x_ + y_; T[12] = x_ - y_; }
    { const int32_t x_ = T[9], y_ = T[10]; T[9] = x_ + y_; T[10] = x_ - y_; }
    { const int32_t x_ = T[8], y_ = T[11]; T[8] = x_ + y_; T[11] = x_ - y_; }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[5] * 2896), y_ = rnd12(T[6] * 2896 + T[5] * 2896); T[6] = y_; T[5] = x_; }
    { const int32_t x_ = T[1], y_ = T[2]; T[1] = x_ + y_; T[2] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[3]; T[0] = x_ + y_; T[3] = x_ - y_; }
    { const int32_t x_ = rnd12(T[13] * -3784 - T[10] * 1567), y_ = rnd12(T[13] * 1567 + T[10] * -3784); T[13] = y_; T[10] = x_; }
    { const int32_t x_ = rnd12(T[14] * 1567 - T[9] * 3784), y_ = rnd12(T[14] * 3784 + T[9] * 1567); T[14] = y_; T[9] = x_; }
    { const int32_t x_ = T[7], y_ = T[6]; T[7] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[5]; T[4] = x_ + y_; T[5] = x_ - y_; }
    { const int32_t x_ = rnd12(T[2] * 1567 - T[3] * -3784), y_ = rnd12(T[2] * -3784 + T[3] * 1567); T[2] = x_; T[3] = y_; }
    { const int32_t x_ = rnd12(T[0] * 2896 - T[1] * 2896), y_ = rnd12(T[0] * 2896 + T[1] * 2896); T[0] = y_; T[1] = x_; }
    { const int32_t x_ = T[15], y_ = T[14]; T[15] = x_ + y_; T[14] = x_ - y_; }
    { const int32_t x_ = T[12], y_ = T[13]; T[12] = x_ + y_; T[13] = x_ - y_; }
    { const int32_t x_ = T[11], y_ = T[10]; T[11] = x_ + y_; T[10] = x_ - y_; }
    { const int32_t x_ = T[8], y_ = T[9]; T[8] = x_ + y_; T[9] = x_ - y_; }
    { const int32_t x_ = rnd12(T[5] * 3406 - T[6] * -2276), y_ = rnd12(T[5] * -2276 + T[6] * 3406); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = rnd12(T[4] * 799 - T[7] * -4017), y_ = rnd12(T[4] * -4017 + T[7] * 799); T[4] = x_; T[7] = y_; }
    { const int32_t x_ = rnd12(T[11] * 3920 - T[12] * -1189), y_ = rnd12(T[11] * -1189 + T[12] * 3920); T[11] = x_; T[12] = y_; }
    { const int32_t x_ = rnd12(T[10] * 1931 - T[13] * -3612), y_ = rnd12(T[10] * -3612 + T[13] * 1931); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = rnd12(T[9] * 3166 - T[14] * -2598), y_ = rnd12(T[9] * -2598 + T[14] * 3166); T[9] = x_; T[14] = y_; }
    { const int32_t x_ = rnd12(T[8] * 401 - T[15] * -4076), y_ = rnd12(T[8] * -4076 + T[15] * 401); T[8] = x_; T[15] = y_; }
    {
        int32_t c_[16];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7]; c_[8] = T[8]; c_[9] = T[9]; c_[10] = T[10]; c_[11] = T[11]; c_[12] = T[12]; c_[13] = T[13]; c_[14] = T[14]; c_[15] = T[15];
        T[0] = c_[0];
        T[8] = c_[1];
        T[4] = c_[2];
        T[12] = c_[3];
        T[2] = c_[4];
        T[10] = c_[5];
        T[6] = c_[6];
        T[14] = c_[7];
        T[1] = c_[8];
        T[9] = c_[9];
        T[5] = c_[10];
        T[13] = c_[11];
        T[3] = c_[12];
        T[11] = c_[13];
        T[7] = c_[14];
        T[15] = c_[15];
    }
}
__host__ __device__ __forceinline__ uint32_t inv_dct16(int32_t *T, int r) {
    uint32_t e_ = 0;
    const int32_t lo_ = -(1 << (r - 1)), hi_ = (1 << (r - 1)) - 1;
    {
        int32_t c_[16];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7]; c_[8] = T[8]; c_[9] = T[9]; c_[10] = T[10]; c_[11] = T[11]; c_[12] = T[12]; c_[13] = T[13]; c_[14] = T[14]; c_[15] = T[15];
        T[0] = c_[0];
        T[1] = c_[8];
        T[2] = c_[4];
        T[3] = c_[12];
        T[4] = c_[2];
        T[5] = c_[10];
        T[6] = c_[6];
        T[7] = c_[14];
        T[8] = c_[1];
        T[9] = c_[9];
        T[10] = c_[5];
        T[11] = c_[13];
        T[12] = c_[3];
        T[13] = c_[11];
        T[14] = c_[7];
        T[15] = c_[15];
    }
    { const int32_t x_ = rnd12(T[8] * 401 - T[15] * 4076), y_ = rnd12(T[8] * 4076 + T[15] * 401); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[8] = x_; T[15] = y_; }
    { const int32_t x_ = rnd12(T[9] * 3166 - T[14] * 2598), y_ = rnd12(T[9] * 2598 + T[14] * 3166); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[9] = x_; T[14] = y_; }
    { const int32_t x_ = rnd12(T[10] * 1931 - T[13] * 3612), y_ = rnd12(T[10] * 3612 + T[13] * 1931); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = rnd12(T[11] * 3920 - T[12] * 1189), y_ = rnd12(T[11] * 1189 + T[12] * 3920); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[11] = x_; T[12] = y_; }
    { const int32_t x_ = rnd12(T[4] * 799 - T[7] * 4017), y_ = rnd12(T[4] * 4017 + T[7] * 799); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[4] = x_; T[7] = y_; }
    { const int32_t x_ = rnd12(T[5] * 3406 - T[6] * 2276), y_ = rnd12(T[5] * 2276 + T[6] * 3406); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = T[8], y_ = T[9]; T[8] = clampr(x_ + y_, lo_, hi_); T[9] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[11], y_ = T[10]; T[11] = clampr(x_ + y_, lo_, hi_); T[10] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[12], y_ = T[13]; T[12] = clampr(x_ + y_, lo_, hi_); T[13] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[15], y_ = T[14]; T[15] = clampr(x_ + y_, lo_, hi_); T[14] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[0] * 2896 - T[1] * 2896), y_ = rnd12(T[0] * 2896 + T[1] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[1] = x_; T[0] = y_; }
    { const int32_t x_ = rnd12(T[2] * 1567 - T[3] * 3784), y_ = rnd12(T[2] * 3784 + T[3] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[2] = x_; T[3] = y_; }
    { const int32_t x_ = T[4], y_ = T[5]; T[4] = clampr(x_ + y_, lo_, hi_); T[5] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[7], y_ = T[6]; T[7] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[14] * 1567 - T[9] * 3784), y_ = rnd12(T[14] * 3784 + T[9] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[9] = x_; T[14] = y_; }
    { const int32_t x_ = rnd12(T[13] * -3784 - T[10] * 1567), y_ = rnd12(T[13] * 1567 + T[10] * -3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = T[0], y_ = T[3]; T[0] = clampr(x_ + y_, lo_, hi_); T[3] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[2]; T[1] = clampr(x_ + y_, lo_, hi_); T[2] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[5] * 2896), y_ = rnd12(T[6] * 2896 + T[5] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = T[8], y_ = T[11]; T[8] = clampr(x_ + y_, lo_, hi_); T[11] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[9], y_ = T[10]; T[9] = clampr(x_ + y_, lo_, hi_); T[10] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[15], y_ = T[12]; T[15] = clampr(x_ + y_, lo_, hi_); T[12] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[14], y_ = T[13]; T[14] = clampr(x_ + y_, lo_, hi_); T[13] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[0], y_ = T[7]; T[0] = clampr(x_ + y_, lo_, hi_); T[7] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[6]; T[1] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[5]; T[2] = clampr(x_ + y_, lo_, hi_); T[5] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[4]; T[3] = clampr(x_ + y_, lo_, hi_); T[4] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[13] * 2896 - T[10] * 2896), y_ = rnd12(T[13] * 2896 + T[10] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = rnd12(T[12] * 2896 - T[11] * 2896), y_ = rnd12(T[12] * 2896 + T[11] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[11] = x_; T[12] = y_; }
    { const int32_t x_ = T[0], y_ = T[15]; T[0] = clampr(x_ + y_, lo_, hi_); T[15] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[14]; T[1] = clampr(x_ + y_, lo_, hi_); T[14] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[13]; T[2] = clampr(x_ + y_, lo_, hi_); T[13] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[12]; T[3] = clampr(x_ + y_, lo_, hi_); T[12] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[4], y_ = T[11]; T[4] = clampr(x_ + y_, lo_, hi_); T[11] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[5], y_ = T[10]; T[5] = clampr(x_ + y_, lo_, hi_); T[10] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[6], y_ = T[9]; T[6] = clampr(x_ + y_, lo_, hi_); T[9] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[7], y_ = T[8]; T[7] = clampr(x_ + y_, lo_, hi_); T[8] = clampr(x_ - y_, lo_, hi_); }
    return e_;
}
__host__ __device__ __forceinline__ void fwd_dct32(int32_t *T) {
    { const int32_t x_ = T[15], y_ = T[16]; T[15] = x_ + y_; T[16] = x_ - y_; }
    { const int32_t x_ = T[14], y_ = T[17]; T[14] = x_ + y_; T[17] = x_ - y_; }
    { const int32_t x_ = T[13], y_ = T[18]; T[13] = x_ + y_; T[18] = x_ - y_; }
    { const int32_t x_ = T[12], y_ = T[19]; T[12] = x_ + y_; T[19] = x_ - y_; }
    { const int32_t x_ = T[11], y_ = T[20]; T[11] = x_ + y_; T[20] = x_ - y_; }
    { const int32_t x_ = T[10], y_ = T[21]; T[10] = x_ + y_; T[21] = x_ - y_; }
    { const int32_t x_ = T[9], y_ = T[22]; T[9] = x_ + y_; T[22] = x_ - y_; }
    { const int32_t x_ = T[8], y_ = T[23]; T[8] = x_ + y_; T[23] = x_ - y_; }
    { const int32_t x_ = T[7], y_ = T[24]; T[7] = x_ + y_; T[24] = x_ - y_; }
    { const int32_t x_ = T[6], y_ = T[25]; T[6] = x_ + y_; T[25] = x_ - y_; }
    { const int32_t x_ = T[5], y_ = T[26]; T[5] = x_ + y_; T[26] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[27]; T[4] = x_ + y_; T[27] = x_ - y_; }
    { const int32_t x_ = T[3], y_ = T[28]; T[3] = x_ + y_; T[28] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[29]; T[2] = x_ + y_; T[29] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[30]; T[1] = x_ + y_; T[30] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[31]; T[0] = x_ + y_; T[31] = x_ - y_; }
    { const int32_t x_ = rnd12(T[24] * 2896 - T[23] * 2896), y_ = rnd12(T[24] * 2896 + T[23] * 2896); T[24] = y_; T[23] = x_; }
    { const int32_t x_ = rnd12(T[25] * 2896 - T[22] * 2896), y_ = rnd12(T[25] * 2896 + T[22] * 2896); T[25] = y_; T[22] = x_; }
    { const int32_t x_ = rnd12(T[26] * 2896 - T[21] * 2896), y_ = rnd12(T[26] * 2896 + T[21] * 2896); T[26] = y_; T[21] = x_; }
    { const int32_t x_ = rnd12(T[27] * 2896 - T[20] * 2896), y_ = rnd12(T[27] * 2896 + T[20] * 2896); T[27] = y_; T[20] = x_; }
    { const int32_t x_ = T[7], y_ = T[8]; T[7] = x_ + y_; T[8] = x_ - y_; }
    { const int32_t x_ = T[6], y_ = T[9]; T[6] = x_ + y_; T[9] = x_ - y_; }
    { const int32_t x_ = T[5], y_ = T[10]; T[5] = x_ + y_; T[10] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[11]; T[4] = x_ + y_; T[11] = x_ - y_; }
    { const int32_t x_ = T[3], y_ = T[12]; T[3] = x_ + y_; T[12] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[13]; T[2] = x_ + y_; T[13] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[14]; T[1] = x_ + y_; T[14] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[15]; T[0] = x_ + y_; T[15] = x_ - y_; }
    { const int32_t x_ = T[28], y_ = T[27]; T[28] = x_ + y_; T[27] = x_ - y_; }
    { const int32_t x_ = T[29], y_ = T[26]; T[29] = x_ + y_; T[26] = x_ - y_; }
    { const int32_t x_ = T[30], y_ = T[25]; T[30] = x_ + y_; T[25] = x_ - y_; }
    { const int32_t x_ = T[31], y_ = T[24]; T[31] = x_ + y_; T[24] = x_ - y_; }
    { const int32_t x_ = T[19], y_ = T[20]; T[19] = x_ + y_; T[20] = x_ - y_; }
    { const int32_t x_ = T[18], y_ = T[21]; T[18] = x_ + y_; T[21] = x_ - y_; }
    { const int32_t x_ = T[17], y_ = T[22]; T[17] = x_ + y_; T[22] = x_ - y_; }
    { const int32_t x_ = T[16], y_ = T[23]; T[16] = x_ + y_; T[23] = x_ - y_; }
    { const int32_t x_ = rnd12(T[12] * 2896 - T[11] * 2896), y_ = rnd12(T[12] * 2896 + T[11] * 2896); T[12] = y_; T[11] = x_; }
    { const int32_t x_ = rnd12(T[13] * 2896 - T[10] * 2896), y_ = rnd12(T[13] * 2896 + T[10] * 2896); T[13] = y_; T[10] = x_; }
    { const int32_t x_ = T[3], y_ = T[4]; T[3] = x_ + y_; T[4] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[5]; T[2] = x_ + y_; T[5] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[6]; T[1] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[7]; T[0] = x_ + y_; T[7] = x_ - y_; }
    { const int32_t x_ = rnd12(T[26] * -3784 - T[21] * 1567), y_ = rnd12(T[26] * 1567 + T[21] * -3784); T[26] = y_; T[21] = x_; }
    { const int32_t x_ = rnd12(T[27] * -3784 - T[20] * 1567), y_ = rnd12(T[27] * 1567 + T[20] * -3784); T[27] = y_; T[20] = x_; }
    { const int32_t x_ = rnd12(T[28] * 1567 - T[19] * 3784), y_ = rnd12(T[28] * 3784 + T[19] * 1567); T[28] = y_; T[19] = x_; }
    { const int32_t x_ = rnd12(T[29] * 1567 - T[18] * 3784), y_ = rnd12(T[29] * 3784 + T[18] * 1567); T[29] = y_; T[18] = x_; }
    { const int32_t x_ = T[14], y_ = T[13]; T[14] = x_ + y_; T[13] = x_ - y_; }
    { const int32_t x_ = T[15], y_ = T[12]; T[15] = x_ + y_; T[12] = x_ - y_; }
    { const int32_t x_ = T[9], y_ = T[10]; T[9] = x_ + y_; T[10] = x_ - y_; }
    { const int32_t x_ = T[8], y_ = T[11]; T[8] = x_ + y_; T[11] = x_ - y_; }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[5] * 2896), y_ = rnd12(T[6] * 2896 + T[5] * 2896); T[6] = y_; T[5] = x_; }
    { const int32_t x_ = T[1], y_ = T[2]; T[1] = x_ + y_; T[2] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[3]; T[0] = x_ + y_; T[3] = x_ - y_; }
    { const int32_t x_ = T[30], y_ = T[29]; T[30] = x_ + y_; T[29] = x_ - y_; }
    { const int32_t x_ = T[31], y_ = T[28]; T[31] = x_ + y_; T[28] = x_ - y_; }
    { const int32_t x_ = T[25], y_ = T[26]; T[25] = x_ + y_; T[26] = x_ - y_; }
    { const int32_t x_ = T[24], y_ = T[27]; T[24] = x_ + y_; T[27] = x_ - y_; }
    { const int32_t x_ = T[22], y_ = T[21]; T[22] = x_ + y_; T[21] = x_ - y_; }
    { const int32_t x_ = T[23], y_ = T[20]; T[23] = x_ + y_; T[20] = x_ - y_; }
    { const int32_t x_ = T[17], y_ = T[18]; T[17] = x_ + y_; T[18] = x_ - y_; }
    { const int32_t x_ = T[16], y_ = T[19]; T[16] = x_ + y_; T[19] = x_ - y_; }
    { const int32_t x_ = rnd12(T[13] * -3784 - T[10] * 1567), y_ = rnd12(T[13] * 1567 + T[10] * -3784); T[13] = y_; T[10] = x_; }
    { const int32_t x_ = rnd12(T[14] * 1567 - T[9] * 3784), y_ = rnd12(T[14] * 3784 + T[9] * 1567); T[14] = y_; T[9] = x_; }
    { const int32_t x_ = T[7], y_ = T[6]; T[7] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[5]; T[4] = x_ + y_; T[5] = x_ - y_; }
    { const int32_t x_ = rnd12(T[2] * 1567 - T[3] * -3784), y_ = rnd12(T[2] * -3784 + T[3] * 1567); T[2] = x_; T[3] = y_; }
    { const int32_t x_ = rnd12(T[0] * 2896 - T[1] * 2896), y_ = rnd12(T[0] * 2896 + T[1] * 2896); T[0] = y_; T[1] = x_; }
    { const int32_t x_ = rnd12(T[25] * -2276 - T[22] * 3406), y_ = rnd12(T[25] * 3406 + T[22] * -2276); T[25] = y_; T[22] = x_; }
    { const int32_t x_ = rnd12(T[26] * 3406 - T[21] * 2276), y_ = rnd12(T[26] * 2276 + T[21] * 3406); T[26] = y_; T[21] = x_; }
    { const int32_t x_ = rnd12(T[29] * -4017 - T[18] * 799), y_ = rnd12(T[29] * 799 + T[18] * -4017); T[29] = y_; T[18] = x_; }
    { const int32_t x_ = rnd12(T[30] * 799 - T[17] * 4017), y_ = rnd12(T[30] * 4017 + T[17] * 799); T[30] = y_; T[17] = x_; }
    { const int32_t x_ = T[15], y_ = T[14]; T[15] = x_ + y_; T[14] = x_ - y_; }
    { const int32_t x_ = T[12], y_ = T[13]; T[12] = x_ + y_; T[13] = x_ - y_; }
    { const int32_t x_ = T[11], y_ = T[10]; T[11] = x_ + y_; T[10] = x_ - y_; }
    { const int32_t x_ = T[8], y_ = T[9]; T[8] = x_ + y_; T[9] = x_ - y_; }
    { const int32_t x_ = rnd12(T[5] * 3406 - T[6] * -2276), y_ = rnd12(T[5] * -2276 + T[6] * 3406); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = rnd12(T[4] * 799 - T[7] * -4017), y_ = rnd12(T[4] * -4017 + T[7] * 799); T[4] = x_; T[7] = y_; }
    { const int32_t x_ = T[31], y_ = T[30]; T[31] = x_ + y_; T[30] = x_ - y_; }
    { const int32_t x_ = T[28], y_ = T[29]; T[28] = x_ + y_; T[29] = x_ - y_; }
    { const int32_t x_ = T[27], y_ = T[26]; T[27] = x_ + y_; T[26] = x_ - y_; }
    { const int32_t x_ = T[24], y_ = T[25]; T[24] = x_ + y_; T[25] = x_ - y_; }
    { const int32_t x_ = T[23], y_ = T[22]; T[23] = x_ + y_; T[22] = x_ - y_; }
    { const int32_t x_ = T[20], y_ = T[21]; T[20] = x_ + y_; T[21] = x_ - y_; }
    { const int32_t x_ = T[19], y_ = T[18]; T[19] = x_ + y_; T[18] = x_ - y_; }
    { const int32_t x_ = T[16], y_ = T[17]; T[16] = x_ + y_; T[17] = x_ - y_; }
    { const int32_t x_ = rnd12(T[11] * 3920 - T[12] * -1189), y_ = rnd12(T[11] * -1189 + T[12] * 3920); T[11] = x_; T[12] = y_; }
    { const int32_t x_ = rnd12(T[10] * 1931 - T[13] * -3612), y_ = rnd12(T[10] * -3612 + T[13] * 1931); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = rnd12(T[9] * 3166 - T[14] * -2598), y_ = rnd12(T[9] * -2598 + T[14] * 3166); T[9] = x_; T[14] = y_; }
    { const int32_t x_ = rnd12(T[8] * 401 - T[15] * -4076), y_ = rnd12(T[8] * -4076 + T[15] * 401); T[8] = x_; T[15] = y_; }
    { const int32_t x_ = rnd12(T[23] * 4052 - T[24] * -601), y_ = rnd12(T[23] * -601 + T[24] * 4052); T[23] = x_; T[24] = y_; }
    { const int32_t x_ = rnd12(T[22] * 2440 - T[25] * -3290), y_ = rnd12(T[22] * -3290 + T[25] * 2440); T[22] = x_; T[25] = y_; }
    { const int32_t x_ = rnd12(T[21] * 3513 - T[26] * -2106), y_ = rnd12(T[21] * -2106 + T[26] * 3513); T[21] = x_; T[26] = y_; }
    { const int32_t x_ = rnd12(T[20] * 995 - T[27] * -3973), y_ = rnd12(T[20] * -3973 + T[27] * 995); T[20] = x_; T[27] = y_; }
    { const int32_t x_ = rnd12(T[19] * 3857 - T[28] * -1380), y_ = rnd12(T[19] * -1380 + T[28] * 3857); T[19] = x_; T[28] = y_; }
    { const int32_t x_ = rnd12(T[18] * 1751 - T[29] * -3703), y_ = rnd12(T[18] * -3703 + T[29] * 1751); T[18] = x_; T[29] = y_; }
    { const int32_t x_ = rnd12(T[17] * 3035 - T[30] * -2751), y_ = rnd12(T[17] * -2751 + T[30] * 3035); T[17] = x_; T[30] = y_; }
    { const int32_t x_ = rnd12(T[16] * 201 - T[31] * -4091), y_ = rnd12(T[16] * -4091 + T[31] * 201); T[16] = x_; T[31] = y_; }
    {
        int32_t c_[32];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7]; c_[8] = T[8]; c_[9] = T[9]; c_[10] = T[10]; c_[11] = T[11]; c_[12] = T[12]; c_[13] = T[13]; c_[14] = T[14]; c_[15] = T[15]; c_[16] = T[16]; c_[17] = T[17]; c_[18] = T[18]; c_[19] = T[19]; c_[20] = T[20]; c_[21] = T[21]; c_[22] = T[22]; c_[23] = T[23]; c_[24] = T[24]; c_[25] = T[25]; c_[26] = T[26]; c_[27] = T[27]; c_[28] = T[28]; c_[29] = T[29]; c_[30] = T[30]; c_[31] = T[31];
        T[0] = c_[0];
        T[16] = c_[1];
        T[8] = c_[2];
        T[24] = c_[3];
        T[4] = c_[4];
        T[20] = c_[5];
        T[12] = c_[6];
        T[28] = c_[7];
        T[2] = c_[8];
        T[18] = c_[9];
        T[10] = c_[10];
        T[26] = c_[11];
        T[6] = c_[12];
        T[22] = c_[13];
        T[14] = c_[14];
        T[30] = c_[15];
        T[1] = c_[16];
        T[17] = c_[17];
        T[9] = c_[18];
        T[25] = c_[19];
        T[5] = c_[20];
        T[21] = c_[21];
        T[13] = c_[22];
        T[29] = c_[23];
        T[3] = c_[24];
        T[19] = c_[25];
        T[11] = c_[26];
        T[27] = c_[27];
        T[7] = c_[28];
        T[23] = c_[29];
        T[15] = c_[30];
        T[31] = c_[31];
    }
}
__host__ __device__ __forceinline__ uint32_t inv_dct32(int32_t *T, int r) {
    uint32_t e_ = 0;
    const int32_t lo_ = -(1 << (r - 1)), hi_ = (1 << (r - 1)) - 1;
    {
        int32_t c_[32];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7]; c_[8] = T[8]; c_[9] = T[9]; c_[10] = T[10]; c_[11] = T[11]; c_[12] = T[12]; c_[13] = T[13]; c_[14] = T[14]; c_[15] = T[15]; c_[16] = T[16]; c_[17] = T[17]; c_[18] = T[18]; c_[19] = T[19]; c_[20] = T[20]; c_[21] = T[21]; c_[22] = T[22]; c_[23] = T[23]; c_[24] = T[24]; c_[25] = T[25]; c_[26] = T[26]; c_[27] = T[27]; c_[28] = T[28]; c_[29] = T[29]; c_[30] = T[30]; c_[31] = T[31];
        T[0] = c_[0];
        T[1] = c_[16];
        T[2] = c_[8];
        T[3] = c_[24];
        T[4] = c_[4];
        T[5] = c_[20];
        T[6] = c_[12];
        T[7] = c_[28];
        T[8] = c_[2];
        T[9] = c_[18];
        T[10] = c_[10];
        T[11] = c_[26];
        T[12] = c_[6];
        T[13] = c_[22];
        T[14] = c_[14];
        T[15] = c_[30];
        T[16] = c_[1];
        T[17] = c_[17];
        T[18] = c_[9];
        T[19] = c_[25];
        T[20] = c_[5];
        T[21] = c_[21];
        T[22] = c_[13];
        T[23] = c_[29];
        T[24] = c_[3];
        T[25] = c_[19];
        T[26] = c_[11];
        T[27] = c_[27];
        T[28] = c_[7];
        T[29] = c_[23];
        T[30] = c_[15];
        T[31] = c_[31];
    }
    { const int32_t x_ = rnd12(T[16] * 201 - T[31] * 4091), y_ = rnd12(T[16] * 4091 + T[31] * 201); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[16] = x_; T[31] = y_; }
    { const int32_t x_ = rnd12(T[17] * 3035 - T[30] * 2751), y_ = rnd12(T[17] * 2751 + T[30] * 3035); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[17] = x_; T[30] = y_; }
    { const int32_t x_ = rnd12(T[18] * 1751 - T[29] * 3703), y_ = rnd12(T[18] * 3703 + T[29] * 1751); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[18] = x_; T[29] = y_; }
    { const int32_t x_ = rnd12(T[19] * 3857 - T[28] * 1380), y_ = rnd12(T[19] * 1380 + T[28] * 3857); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[19] = x_; T[28] = y_; }
    { const int32_t x_ = rnd12(T[20] * 995 - T[27] * 3973), y_ = rnd12(T[20] * 3973 + T[27] * 995); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[20] = x_; T[27] = y_; }
    { const int32_t x_ = rnd12(T[21] * 3513 - T[26] * 2106), y_ = rnd12(T[21] * 2106 + T[26] * 3513); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[21] = x_; T[26] = y_; }
    { const int32_t x_ = rnd12(T[22] * 2440 - T[25] * 3290), y_ = rnd12(T[22] * 3290 + T[25] * 2440); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[22] = x_; T[25] = y_; }
    { const int32_t x_ = rnd12(T[23] * 4052 - T[24] * 601), y_ = rnd12(T[23] * 601 + T[24] * 4052); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[23] = x_; T[24] = y_; }
    { const int32_t x_ = rnd12(T[8] * 401 - T[15] * 4076), y_ = rnd12(T[8] * 4076 + T[15] * 401); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[8] = x_; T[15] = y_; }
    { const int32_t x_ = rnd12(T[9] * 3166 - T[14] * 2598), y_ = rnd12(T[9] * 2598 + T[14] * 3166); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[9] = x_; T[14] = y_; }
    { const int32_t x_ = rnd12(T[10] * 1931 - T[13] * 3612), y_ = rnd12(T[10] * 3612 + T[13] * 1931); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = rnd12(T[11] * 3920 - T[12] * 1189), y_ = rnd12(T[11] * 1189 + T[12] * 3920); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[11] = x_; T[12] = y_; }
    { const int32_t x_ = T[16], y_ = T[17]; T[16] = clampr(x_ + y_, lo_, hi_); T[17] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[19], y_ = T[18]; T[19] = clampr(x_ + y_, lo_, hi_); T[18] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[20], y_ = T[21]; T[20] = clampr(x_ + y_, lo_, hi_); T[21] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[23], y_ = T[22]; T[23] = clampr(x_ + y_, lo_, hi_); T[22] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[24], y_ = T[25]; T[24] = clampr(x_ + y_, lo_, hi_); T[25] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[27], y_ = T[26]; T[27] = clampr(x_ + y_, lo_, hi_); T[26] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[28], y_ = T[29]; T[28] = clampr(x_ + y_, lo_, hi_); T[29] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[31], y_ = T[30]; T[31] = clampr(x_ + y_, lo_, hi_); T[30] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[4] * 799 - T[7] * 4017), y_ = rnd12(T[4] * 4017 + T[7] * 799); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[4] = x_; T[7] = y_; }
    { const int32_t x_ = rnd12(T[5] * 3406 - T[6] * 2276), y_ = rnd12(T[5] * 2276 + T[6] * 3406); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = T[8], y_ = T[9]; T[8] = clampr(x_ + y_, lo_, hi_); T[9] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[11], y_ = T[10]; T[11] = clampr(x_ + y_, lo_, hi_); T[10] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[12], y_ = T[13]; T[12] = clampr(x_ + y_, lo_, hi_); T[13] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[15], y_ = T[14]; T[15] = clampr(x_ + y_, lo_, hi_); T[14] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[30] * 799 - T[17] * 4017), y_ = rnd12(T[30] * 4017 + T[17] * 799); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[17] = x_; T[30] = y_; }
    { const int32_t x_ = rnd12(T[29] * -4017 - T[18] * 799), y_ = rnd12(T[29] * 799 + T[18] * -4017); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[18] = x_; T[29] = y_; }
    { const int32_t x_ = rnd12(T[26] * 3406 - T[21] * 2276), y_ = rnd12(T[26] * 2276 + T[21] * 3406); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[21] = x_; T[26] = y_; }
    { const int32_t x_ = rnd12(T[25] * -2276 - T[22] * 3406), y_ = rnd12(T[25] * 3406 + T[22] * -2276); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[22] = x_; T[25] = y_; }
    { const int32_t x_ = rnd12(T[0] * 2896 - T[1] * 2896), y_ = rnd12(T[0] * 2896 + T[1] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[1] = x_; T[0] = y_; }
    { const int32_t x_ = rnd12(T[2] * 1567 - T[3] * 3784), y_ = rnd12(T[2] * 3784 + T[3] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[2] = x_; T[3] = y_; }
    { const int32_t x_ = T[4], y_ = T[5]; T[4] = clampr(x_ + y_, lo_, hi_); T[5] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[7], y_ = T[6]; T[7] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[14] * 1567 - T[9] * 3784), y_ = rnd12(T[14] * 3784 + T[9] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[9] = x_; T[14] = y_; }
    { const int32_t x_ = rnd12(T[13] * -3784 - T[10] * 1567), y_ = rnd12(T[13] * 1567 + T[10] * -3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = T[16], y_ = T[19]; T[16] = clampr(x_ + y_, lo_, hi_); T[19] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[17], y_ = T[18]; T[17] = clampr(x_ + y_, lo_, hi_); T[18] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[23], y_ = T[20]; T[23] = clampr(x_ + y_, lo_, hi_); T[20] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[22], y_ = T[21]; T[22] = clampr(x_ + y_, lo_, hi_); T[21] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[24], y_ = T[27]; T[24] = clampr(x_ + y_, lo_, hi_); T[27] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[25], y_ = T[26]; T[25] = clampr(x_ + y_, lo_, hi_); T[26] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[31], y_ = T[28]; T[31] = clampr(x_ + y_, lo_, hi_); T[28] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[30], y_ = T[29]; T[30] = clampr(x_ + y_, lo_, hi_); T[29] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[0], y_ = T[3]; T[0] = clampr(x_ + y_, lo_, hi_); T[3] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[2]; T[1] = clampr(x_ + y_, lo_, hi_); T[2] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[5] * 2896), y_ = rnd12(T[6] * 2896 + T[5] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = T[8], y_ = T[11]; T[8] = clampr(x_ + y_, lo_, hi_); T[11] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[9], y_ = T[10]; T[9] = clampr(x_ + y_, lo_, hi_); T[10] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[15], y_ = T[12]; T[15] = clampr(x_ + y_, lo_, hi_); T[12] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[14], y_ = T[13]; T[14] = clampr(x_ + y_, lo_, hi_); T[13] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[29] * 1567 - T[18] * 3784), y_ = rnd12(T[29] * 3784 + T[18] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[18] = x_; T[29] = y_; }
    { const int32_t x_ = rnd12(T[28] * 1567 - T[19] * 3784), y_ = rnd12(T[28] * 3784 + T[19] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[19] = x_; T[28] = y_; }
    { const int32_t x_ = rnd12(T[27] * -3784 - T[20] * 1567), y_ = rnd12(T[27] * 1567 + T[20] * -3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[20] = x_; T[27] = y_; }
    { const int32_t x_ = rnd12(T[26] * -3784 - T[21] * 1567), y_ = rnd12(T[26] * 1567 + T[21] * -3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[21] = x_; T[26] = y_; }
    { const int32_t x_ = T[0], y_ = T[7]; T[0] = clampr(x_ + y_, lo_, hi_); T[7] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[6]; T[1] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[5]; T[2] = clampr(x_ + y_, lo_, hi_); T[5] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[4]; T[3] = clampr(x_ + y_, lo_, hi_); T[4] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[13] * 2896 - T[10] * 2896), y_ = rnd12(T[13] * 2896 + T[10] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = rnd12(T[12] * 2896 - T[11] * 2896), y_ = rnd12(T[12] * 2896 + T[11] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[11] = x_; T[12] = y_; }
    { const int32_t x_ = T[16], y_ = T[23]; T[16] = clampr(x_ + y_, lo_, hi_); T[23] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[17], y_ = T[22]; T[17] = clampr(x_ + y_, lo_, hi_); T[22] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[18], y_ = T[21]; T[18] = clampr(x_ + y_, lo_, hi_); T[21] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[19], y_ = T[20]; T[19] = clampr(x_ + y_, lo_, hi_); T[20] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[31], y_ = T[24]; T[31] = clampr(x_ + y_, lo_, hi_); T[24] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[30], y_ = T[25]; T[30] = clampr(x_ + y_, lo_, hi_); T[25] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[29], y_ = T[26]; T[29] = clampr(x_ + y_, lo_, hi_); T[26] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[28], y_ = T[27]; T[28] = clampr(x_ + y_, lo_, hi_); T[27] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[0], y_ = T[15]; T[0] = clampr(x_ + y_, lo_, hi_); T[15] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[14]; T[1] = clampr(x_ + y_, lo_, hi_); T[14] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[13]; T[2] = clampr(x_ + y_, lo_, hi_); T[13] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[12]; T[3] = clampr(x_ + y_, lo_, hi_); T[12] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[4], y_ = T[11]; T[4] = clampr(x_ + y_, lo_, hi_); T[11] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[5], y_ = T[10]; T[5] = clampr(x_ + y_, lo_, hi_); T[10] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[6], y_ = T[9]; T[6] = clampr(x_ + y_, lo_, hi_); T[9] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[7], y_ = T[8]; T[7] = clampr(x_ + y_, lo_, hi_); T[8] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[27] * 2896 - T[20] * 2896), y_ = rnd12(T[27] * 2896 + T[20] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[20] = x_; T[27] = y_; }
    { const int32_t x_ = rnd12(T[26] * 2896 - T[21] * 2896), y_ = rnd12(T[26] * 2896 + T[21] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[21] = x_; T[26] = y_; }
    { const int32_t x_ = rnd12(T[25] * 2896 - T[22] * 2896), y_ = rnd12(T[25] * 2896 + T[22] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[22] = x_; T[25] = y_; }
    { const int32_t x_ = rnd12(T[24] * 2896 - T[23] * 2896), y_ = rnd12(T[24] * 2896 + T[23] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[23] = x_; T[24] = y_; }
    { const int32_t x_ = T[0], y_ = T[31]; T[0] = clampr(x_ + y_, lo_, hi_); T[31] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[30]; T[1] = clampr(x_ + y_, lo_, hi_); T[30] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[29]; T[2] = clampr(x_ + y_, lo_, hi_); T[29] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[28]; T[3] = clampr(x_ + y_, lo_, hi_); T[28] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[4], y_ = T[27]; T[4] = clampr(x_ + y_, lo_, hi_); T[27] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[5], y_ = T[26]; T[5] = clampr(x_ + y_, lo_, hi_); T[26] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[6], y_ = T[25]; T[6] = clampr(x_ + y_, lo_, hi_); T[25] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[7], y_ = T[24]; T[7] = clampr(x_ + y_, lo_, hi_); T[24] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[8], y_ = T[23]; T[8] = clampr(x_ + y_, lo_, hi_); T[23] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[9], y_ = T[22]; T[9] = clampr(x_ + y_, lo_, hi_); T[22] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[10], y_ = T[21]; T[10] = clampr(x_ + y_, lo_, hi_); T[21] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[11], y_ = T[20]; T[11] = clampr(x_ + y_, lo_, hi_); T[20] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[12], y_ = T[19]; T[12] = clampr(x_ + y_, lo_, hi_); T[19] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[13], y_ = T[18]; T[13] = clampr(x_ + y_, lo_, hi_); T[18] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[14], y_ = T[17]; T[14] = clampr(x_ + y_, lo_, hi_); T[17] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[15], y_ = T[16]; T[15] = clampr(x_ + y_, lo_, hi_); T[16] = clampr(x_ - y_, lo_, hi_); }
    return e_;
}
__host__ __device__ __forceinline__ void fwd_dct64(int32_t *T) {
    { const int32_t x_ = T[31], y_ = T[32]; T[31] = x_ + y_; T[32] = x_ - y_; }
    { const int32_t x_ = T[30], y_ = T[33]; T[30] = x_ + y_; T[33] = x_ - y_; }
    { const int32_t x_ = T[29], y_ = T[34]; T[29] = x_ + y_; T[34] = x_ - y_; }
    { const int32_t x_ = T[28], y_ = T[35]; T[28] = x_ + y_; T[35] = x_ - y_; }
    { const int32_t x_ = T[27], y_ = T[36]; T[27] = x_ + y_; T[36] = x_ - y_; }
    { const int32_t x_ = T[26], y_ = T[37]; T[26] = x_ + y_; T[37] = x_ - y_; }
    { const int32_t x_ = T[25], y_ = T[38]; T[25] = x_ + y_; T[38] = x_ - y_; }
    { const int32_t x_ = T[24], y_ = T[39]; T[24] = x_ + y_; T[39] = x_ - y_; }
    { const int32_t x_ = T[23], y_ = T[40]; T[23] = x_ + y_; T[40] = x_ - y_; }
    { const int32_t x_ = T[22], y_ = T[41]; T[22] = x_ + y_; T[41] = x_ - y_; }
    { const int32_t x_ = T[21], y_ = T[42]; T[21] = x_ + y_; T[42] = x_ - y_; }
    { const int32_t x_ = T[20], y_ = T[43]; T[20] = x_ + y_; T[43] = x_ - y_; }
    { const int32_t x_ = T[19], y_ = T[44]; T[19] = x_ + y_; T[44] = x_ - y_; }
    { const int32_t x_ = T[18], y_ = T[45]; T[18] = x_ + y_; T[45] = x_ - y_; }
    { const int32_t x_ = T[17], y_ = T[46]; T[17] = x_ + y_; T[46] = x_ - y_; }
    { const int32_t x_ = T[16], y_ = T[47]; T[16] = x_ + y_; T[47] = x_ - y_; }
    { const int32_t x_ = T[15], y_ = T[48]; T[15] = x_ + y_; T[48] = x_ - y_; }
    { const int32_t x_ = T[14], y_ = T[49]; T[14] = x_ + y_; T[49] = x_ - y_; }
    { const int32_t x_ = T[13], y_ = T[50]; T[13] = x_ + y_; T[50] = x_ - y_; }
    { const int32_t x_ = T[12], y_ = T[51]; T[12] = x_ + y_; T[51] = x_ - y_; }
    { const int32_t x_ = T[11], y_ = T[52]; T[11] = x_ + y_; T[52] = x_ - y_; }
    { const int32_t x_ = T[10], y_ = T[53]; T[10] = x_ + y_; T[53] = x_ - y_; }
    { const int32_t x_ = T[9], y_ = T[54]; T[9] = x_ + y_; T[54] = x_ - y_; }
    { const int32_t x_ = T[8], y_ = T[55]; T[8] = x_ + y_; T[55] = x_ - y_; }
    { const int32_t x_ = T[7], y_ = T[56]; T[7] = x_ + y_; T[56] = x_ - y_; }
    { const int32_t x_ = T[6], y_ = T[57]; T[6] = x_ + y_; T[57] = x_ - y_; }
    { const int32_t x_ = T[5], y_ = T[58]; T[5] = x_ + y_; T[58] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[59]; T[4] = x_ + y_; T[59] = x_ - y_; }
    { const int32_t x_ = T[3], y_ = T[60]; T[3] = x_ + y_; T[60] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[61]; T[2] = x_ + y_; T[61] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[62]; T[1] = x_ + y_; T[62] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[63]; T[0] = x_ + y_; T[63] = x_ - y_; }
    { const int32_t x_ = rnd12(T[48] * 2896 - T[47] * 2896), y_ = rnd12(T[48] * 2896 + T[47] * 2896); T[48] = y_; T[47] = x_; }
    { const int32_t x_ = rnd12(T[49] * 2896 - T[46] * 2896), y_ = rnd12(T[49] * 2896 + T[46] * 2896); T[49] = y_; T[46] = x_; }
    { const int32_t x_ = rnd12(T[50] * 2896 - T[45] * 2896), y_ = rnd12(T[50] * 2896 + T[45] * 2896); T[50] = y_; T[45] = x_; }
    { const int32_t x_ = rnd12(T[51] * 2896 - T[44] * 2896), y_ = rnd12(T[51] * 2896 + T[44] * 2896); T[51] = y_; T[44] = x_; }
    { const int32_t x_ = rnd12(T[52] * 2896 - T[43] * 2896), y_ = rnd12(T[52] * 2896 + T[43] * 2896); T[52] = y_; T[43] = x_; }
    { const int32_t x_ = rnd12(T[53] * 2896 - T[42] * 2896), y_ = rnd12(T[53] * 2896 + T[42] * 2896); T[53] = y_; T[42] = x_; }
    { const int32_t x_ = rnd12(T[54] * 2896 - T[41] * 2896), y_ = rnd12(T[54] * 2896 + T[41] * 2896); T[54] = y_; T[41] = x_; }
    { const int32_t x_ = rnd12(T[55] * 2896 - T[40] * 2896), y_ = rnd12(T[55] * 2896 + T[40] * 2896); T[55] = y_; T[40] = x_; }
    { const int32_t x_ = T[15], y_ = T[16]; T[15] = x_ + y_; T[16] = x_ - y_; }
    { const int32_t x_ = T[14], y_ = T[17]; T[14] = x_ + y_; T[17] = x_ - y_; }
    { const int32_t x_ = T[13], y_ = T[18]; T[13] = x_ + y_; T[18] = x_ - y_; }
    { const int32_t x_ = T[12], y_ = T[19]; T[12] = x_ + y_; T[19] = x_ - y_; }
    { const int32_t x_ = T[11], y_ = T[20]; T[11] = x_ + y_; T[20] = x_ - y_; }
    { const int32_t x_ = T[10], y_ = T[21]; T[10] = x_ + y_; T[21] = x_ - y_; }
    { const int32_t x_ = T[9], y_ = T[22]; T[9] = x_ + y_; T[22] = x_ - y_; }
    { const int32_t x_ = T[8], y_ = T[23]; T[8] = x_ + y_; T[23] = x_ - y_; }
    { const int32_t x_ = T[7], y_ = T[24]; T[7] = x_ + y_; T[24] = x_ - y_; }
    { const int32_t x_ = T[6], y_ = T[25]; T[6] = x_ + y_; T[25] = x_ - y_; }
    { const int32_t x_ = T[5], y_ = T[26]; T[5] = x_ + y_; T[26] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[27]; T[4] = x_ + y_; T[27] = x_ - y_; }
    { const int32_t x_ = T[3], y_ = T[28]; T[3] = x_ + y_; T[28] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[29]; T[2] = x_ + y_; T[29] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[30]; T[1] = x_ + y_; T[30] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[31]; T[0] = x_ + y_; T[31] = x_ - y_; }
    { const int32_t x_ = T[56], y_ = T[55]; T[56] = x_ + y_; T[55] = x_ - y_; }
    { const int32_t x_ = T[39], y_ = T[40]; T[39] = x_ + y_; T[40] = x_ - y_; }
    { const int32_t x_ = T[57], y_ = T[54]; T[57] = x_ + y_; T[54] = x_ - y_; }
    { const int32_t x_ = T[38], y_ = T[41]; T[38] = x_ + y_; T[41] = x_ - y_; }
    { const int32_t x_ = T[58], y_ = T[53]; T[58] = x_ + y_; T[53] = x_ - y_; }
    { const int32_t x_ = T[37], y_ = T[42]; T[37] = x_ + y_; T[42] = x_ - y_; }
    { const int32_t x_ = T[59], y_ = T[52]; T[59] = x_ + y_; T[52] = x_ - y_; }
    { const int32_t x_ = T[36], y_ = T[43]; T[36] = x_ + y_; T[43] = x_ - y_; }
    { const int32_t x_ = T[60], y_ = T[51]; T[60] = x_ + y_; T[51] = x_ - y_; }
    { const int32_t x_ = T[35], y_ = T[44]; T[35] = x_ + y_; T[44] = x_ - y_; }
    { const int32_t x_ = T[61], y_ = T[50]; T[61] = x_ + y_; T[50] = x_ - y_; }
    { const int32_t x_ = T[34], y_ = T[45]; T[34] = x_ + y_; T[45] = x_ - y_; }
    { const int32_t x_ = T[62], y_ = T[49]; T[62] = x_ + y_; T[49] = x_ - y_; }
    { const int32_t x_ = T[33], y_ = T[46]; T[33] = x_ + y_; T[46] = x_ - y_; }
    { const int32_t x_ = T[63], y_ = T[48]; T[63] = x_ + y_; T[48] = x_ - y_; }
    { const int32_t x_ = T[32], y_ = T[47]; T[32] = x_ + y_; T[47] = x_ - y_; }
    { const int32_t x_ = rnd12(T[24] * 2896 - T[23] * 2896), y_ = rnd12(T[24] * 2896 + T[23] * 2896); T[24] = y_; T[23] = x_; }
    { const int32_t x_ = rnd12(T[25] * 2896 - T[22] * 2896), y_ = rnd12(T[25] * 2896 + T[22] * 2896); T[25] = y_; T[22] = x_; }
    { const int32_t x_ = rnd12(T[26] * 2896 - T[21] * 2896), y_ = rnd12(T[26] * 2896 + T[21] * 2896); T[26] = y_; T[21] = x_; }
    { const int32_t x_ = rnd12(T[27] * 2896 - T[20] * 2896), y_ = rnd12(T[27] * 2896 + T[20] * 2896); T[27] = y_; T[20] = x_; }
    { const int32_t x_ = T[7], y_ = T[8]; T[7] = x_ + y_; T[8] = x_ - y_; }
    { const int32_t x_ = T[6], y_ = T[9]; T[6] = x_ + y_; T[9] = x_ - y_; }
    { const int32_t x_ = T[5], y_ = T[10]; T[5] = x_ + y_; T[10] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[11]; T[4] = x_ + y_; T[11] = x_ - y_; }
    { const int32_t x_ = T[3], y_ = T[12]; T[3] = x_ + y_; T[12] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[13]; T[2] = x_ + y_; T[13] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[14]; T[1] = x_ + y_; T[14] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[15]; T[0] = x_ + y_; T[15] = x_ - y_; }
    { const int32_t x_ = rnd12(T[52] * -3784 - T[43] * 1567), y_ = rnd12(T[52] * 1567 + T[43] * -3784); T[52] = y_; T[43] = x_; }
    { const int32_t x_ = rnd12(T[53] * -3784 - T[42] * 1567), y_ = rnd12(T[53] * 1567 + T[42] * -3784); T[53] = y_; T[42] = x_; }
    { const int32_t x_ = rnd12(T[54] * -3784 - T[41] * 1567), y_ = rnd12(T[54] * 1567 + T[41] * -3784); T[54] = y_; T[41] = x_; }
    { const int32_t x_ = rnd12(T[55] * -3784 - T[40] * 1567), y_ = rnd12(T[55] * 1567 + T[40] * -3784); T[55] = y_; T[40] = x_; }
    { const int32_t x_ = rnd12(T[56] * 1567 - T[39] * 3784), y_ = rnd12(T[56] * 3784 + T[39] * 1567); T[56] = y_; T[39] = x_; }
    { const int32_t x_ = rnd12(T[57] * 1567 - T[38] * 3784), y_ = rnd12(T[57] * 3784 + T[38] * 1567); T[57] = y_; T[38] = x_; }
    { const int32_t x_ = rnd12(T[58] * 1567 - T[37] * 3784), y_ = rnd12(T[58] * 3784 + T[37] * 1567); T[58] = y_; T[37] = x_; }
    { const int32_t x_ = rnd12(T[59] * 1567 - T[36] * 3784), y_ = rnd12(T[59] * 3784 + T[36] * 1567); T[59] = y_; T[36] = x_; }
    { const int32_t x_ = T[28], y_ = T[27]; T[28] = x_ + y_; T[27] = x_ - y_; }
    { const int32_t x_ = T[29], y_ = T[26]; T[29] = x_ + y_; T[26] = x_ - y_; }
    { const int32_t x_ = T[30], y_ = T[25]; T[30] = x_ + y_; T[25] = x_ - y_; }
    { const int32_t x_ = T[31], y_ = T[24]; T[31] = x_ + y_; T[24] = x_ - y_; }
    { const int32_t x_ = T[19], y_ = T[20]; T[19] = x_ + y_; T[20] = x_ - y_; }
    { const int32_t x_ = T[18], y_ = T[21]; T[18] = x_ + y_; T[21] = x_ - y_; }
    { const int32_t x_ = T[17], y_ = T[22]; T[17] = x_ + y_; T[22] = x_ - y_; }
    { const int32_t x_ = T[16], y_ = T[23]; T[16] = x_ + y_; T[23] = x_ - y_; }
    { const int32_t x_ = rnd12(T[12] * 2896 - T[11] * 2896), y_ = rnd12(T[12] * 2896 + T[11] * 2896); T[12] = y_; T[11] = x_; }
    { const int32_t x_ = rnd12(T[13] * 2896 - T[10] * 2896), y_ = rnd12(T[13] * 2896 + T[10] * 2896); T[13] = y_; T[10] = x_; }
    { const int32_t x_ = T[3], y_ = T[4]; T[3] = x_ + y_; T[4] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[5]; T[2] = x_ + y_; T[5] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[6]; T[1] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[7]; T[0] = x_ + y_; T[7] = x_ - y_; }
    { const int32_t x_ = T[60], y_ = T[59]; T[60] = x_ + y_; T[59] = x_ - y_; }
    { const int32_t x_ = T[61], y_ = T[58]; T[61] = x_ + y_; T[58] = x_ - y_; }
    { const int32_t x_ = T[62], y_ = T[57]; T[62] = x_ + y_; T[57] = x_ - y_; }
    { const int32_t x_ = T[63], y_ = T[56]; T[63] = x_ + y_; T[56] = x_ - y_; }
    { const int32_t x_ = T[51], y_ = T[52]; T[51] = x_ + y_; T[52] = x_ - y_; }
    { const int32_t x_ = T[50], y_ = T[53]; T[50] = x_ + y_; T[53] = x_ - y_; }
    { const int32_t x_ = T[49], y_ = T[54]; T[49] = x_ + y_; T[54] = x_ - y_; }
    { const int32_t x_ = T[48], y_ = T[55]; T[48] = x_ + y_; T[55] = x_ - y_; }
    { const int32_t x_ = T[44], y_ = T[43]; T[44] = x_ + y_; T[43] = x_ - y_; }
    { const int32_t x_ = T[45], y_ = T[42]; T[45] = x_ + y_; T[42] = x_ - y_; }
    { const int32_t x_ = T[46], y_ = T[41]; T[46] = x_ + y_; T[41] = x_ - y_; }
    { const int32_t x_ = T[47], y_ = T[40]; T[47] = x_ + y_; T[40] = x_ - y_; }
    { const int32_t x_ = T[35], y_ = T[36]; T[35] = x_ + y_; T[36] = x_ - y_; }
    { const int32_t x_ = T[34], y_ = T[37]; T[34] = x_ + y_; T[37] = x_ - y_; }
    { const int32_t x_ = T[33], y_ = T[38]; T[33] = x_ + y_; T[38] = x_ - y_; }
    { const int32_t x_ = T[32], y_ = T[39]; T[32] = x_ + y_; T[39] = x_ - y_; }
    { const int32_t x_ = rnd12(T[26] * -3784 - T[21] * 1567), y_ = rnd12(T[26] * 1567 + T[21] * -3784); T[26] = y_; T[21] = x_; }
    { const int32_t x_ = rnd12(T[27] * -3784 - T[20] * 1567), y_ = rnd12(T[27] * 1567 + T[20] * -3784); T[27] = y_; T[20] = x_; }
    { const int32_t x_ = rnd12(T[28] * 1567 - T[19] * 3784), y_ = rnd12(T[28] * 3784 + T[19] * 1567); T[28] = y_; T[19] = x_; }
    { const int32_t x_ = rnd12(T[29] * 1567 - T[18] * 3784), y_ = rnd12(T[29] * 3784 + T[18] * 1567); T[29] = y_; T[18] = x_; }
    { const int32_t x_ = T[14], y_ = T[13]; T[14] = x_ + y_; T[13] = x_ - y_; }
    { const int32_t x_ = T[15], y_ = T[12]; T[15] = x_ + y_; T[12] = x_ - y_; }
    { const int32_t x_ = T[9], y_ = T[10]; T[9] = x_ + y_; T[10] = x_ - y_; }
    { const int32_t x_ = T[8], y_ = T[11]; T[8] = x_ + y_; T[11] = x_ - y_; }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[5] * 2896), y_ = rnd12(T[6] * 2896 + T[5] * 2896); T[6] = y_; T[5] = x_; }
    { const int32_t x_ = T[1], y_ = T[2]; T[1] = x_ + y_; T[2] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[3]; T[0] = x_ + y_; T[3] = x_ - y_; }
    { const int32_t x_ = rnd12(T[50] * -2276 - T[45] * 3406), y_ = rnd12(T[50] * 3406 + T[45] * -2276); T[50] = y_; T[45] = x_; }
    { const int32_t x_ = rnd12(T[51] * -2276 - T[44] * 3406), y_ = rnd12(T[51] * 3406 + T[44] * -2276); T[51] = y_; T[44] = x_; }
    { const int32_t x_ = rnd12(T[52] * 3406 - T[43] * 2276), y_ = rnd12(T[52] * 2276 + T[43] * 3406); T[52] = y_; T[43] = x_; }
    { const int32_t x_ = rnd12(T[53] * 3406 - T[42] * 2276), y_ = rnd12(T[53] * 2276 + T[42] * 3406); T[53] = y_; T[42] = x_; }
    { const int32_t x_ = rnd12(T[58] * -4017 - T[37] * 799), y_ = rnd12(T[58] * 799 + T[37] * -4017); T[58] = y_; T[37] = x_; }
    { const int32_t x_ = rnd12(T[59] * -4017 - T[36] * 799), y_ = rnd12(T[59] * 799 + T[36] * -4017); T[59] = y_; T[36] = x_; }
    { const int32_t x_ = rnd12(T[60] * 799 - T[35] * 4017), y_ = rnd12(T[60] * 4017 + T[35] * 799); T[60] = y_; T[35] = x_; }
    { const int32_t x_ = rnd12(T[61] * 799 - T[34] * 4017), y_ = rnd12(T[61] * 4017 + T[34] * 799); T[61] = y_; T[34] = x_; }
    { const int32_t x_ = T[30], y_ = T[29]; T[30] = x_ + y_; T[29] = x_ - y_; }
    { const int32_t x_ = T[31], y_ = T[28]; T[31] = x_ + y_; T[28] = x_ - y_; }
    { const int32_t x_ = T[25], y_ = T[26]; T[25] = x_ + y_; T[26] = x_ - y_; }
    { const int32_t x_ = T[24], y_ = T[27]; T[24] = x_ + y_; T[27] = x_ - y_; }
    { const int32_t x_ = T[22], y_ = T[21]; T[22] = x_ + y_; T[21] = x_ - y_; }
    { const int32_t x_ = T[23], y_ = T[20]; T[23] = x_ + y_; T[20] = x_ - y_; }
    { const int32_t x_ = T[17], y_ = T[18]; T[17] = x_ + y_; T[18] = x_ - y_; }
    { const int32_t x_ = T[16], y_ = T[19]; T[16] = x_ + y_; T[19] = x_ - y_; }
    { const int32_t x_ = rnd12(T[13] * -3784 - T[10] * 1567), y_ = rnd12(T[13] * 1567 + T[10] * -3784); T[13] = y_; T[10] = x_; }
    { const int32_t x_ = rnd12(T[14] * 1567 - T[9] * 3784), y_ = rnd12(T[14] * 3784 + T[9] * 1567); T[14] = y_; T[9] = x_; }
    { const int32_t x_ = T[7], y_ = T[6]; T[7] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[5]; T[4] = x_ + y_; T[5] = x_ - y_; }
    { const int32_t x_ = rnd12(T[2] * 1567 - T[3] * -3784), y_ = rnd12(T[2] * -3784 + T[3] * 1567); T[2] = x_; T[3] = y_; }
    { const int32_t x_ = rnd12(T[0] * 2896 - T[1] * 2896), y_ = rnd12(T[0] * 2896 + T[1] * 2896); T[0] = y_; T[1] = x_; }
    { const int32_t x_ = T[62], y_ = T[61]; T[62] = x_ + y_; T[61] = x_ - y_; }
    { const int32_t x_ = T[63], y_ = T[60]; T[63] = x_ + y_; T[60] = x_ - y_; }
    { const int32_t x_ = T[57], y_ = T[58]; T[57] = x_ + y_; T[58] = x_ - y_; }
    { const int32_t x_ = T[56], y_ = T[59]; T[56] = x_ + y_; T[59] = x_ - y_; }
    { const int32_t x_ = T[54], y_ = T[53]; T[54] = x_ + y_; T[53] = x_ - y_; }
    { const int32_t x_ = T[55], y_ = T[52]; T[55] = x_ + y_; T[52] = x_ - y_; }
    { const int32_t x_ = T[49], y_ = T[50]; T[49] = x_ + y_; T[50] = x_ - y_; }
    { const int32_t x_ = T[48], y_ = T[51]; T[48] = x_ + y_; T[51] = x_ - y_; }
    { const int32_t x_ = T[46], y_ = T[45]; T[46] = x_ + y_; T[45] = x_ - y_; }
    { const int32_t x_ = T[47], y_ = T[44]; T[47] = x_ + y_; T[44] = x_ - y_; }
    { const int32_t x_ = T[41], y_ = T[42]; T[41] = x_ + y_; T[42] = x_ - y_; }
    { const int32_t x_ = T[40], y_ = T[43]; T[40] = x_ + y_; T[43] = x_ - y_; }
    { const int32_t x_ = T[38], y_ = T[37]; T[38] = x_ + y_; T[37] = x_ - y_; }
    { const int32_t x_ = T[39], y_ = T[36]; T[39] = x_ + y_; T[36] = x_ - y_; }
    { const int32_t x_ = T[33], y_ = T[34]; T[33] = x_ + y_; T[34] = x_ - y_; }
    { const int32_t x_ = T[32], y_ = T[35]; T[32] = x_ + y_; T[35] = x_ - y_; }
    { const int32_t x_ = rnd12(T[25] * -2276 - T[22] * 3406), y_ = rnd12(T[25] * 3406 + T[22] * -2276); T[25] = y_; T[22] = x_; }
    { const int32_t x_ = rnd12(T[26] * 3406 - T[21] * 2276), y_ = rnd12(T[26] * 2276 + T[21] * 3406); T[26] = y_; T[21] = x_; }
    { const int32_t x_ = rnd12(T[29] * -4017 - T[18] * 799), y_ = rnd12(T[29] * 799 + T[18] * -4017); T[29] = y_; T[18] = x_; }
    { const int32_t x_ = rnd12(T[30] * 799 - T[17] * 4017), y_ = rnd12(T[30] * 4017 + T[17] * 799); T[30] = y_; T[17] = x_; }
    { const int32_t x_ = T[15], y_ = T[14]; T[15] = x_ + y_; T[14] = x_ - y_; }
    { const int32_t x_ = T[12], y_ = T[13]; T[12] = x_ + y_; T[13] = x_ - y_; }
    { const int32_t x_ = T[11], y_ = T[10]; T[11] = x_ + y_; T[10] = x_ - y_; }
    { const int32_t x_ = T[8], y_ = T[9]; T[8] = x_ + y_; T[9] = x_ - y_; }
    { const int32_t x_ = rnd12(T[5] * 3406 - T[6] * -2276), y_ = rnd12(T[5] * -2276 + T[6] * 3406); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = rnd12(T[4] * 799 - T[7] * -4017), y_ = rnd12(T[4] * -4017 + T[7] * 799); T[4] = x_; T[7] = y_; }
    { const int32_t x_ = rnd12(T[49] * -1189 - T[46] * 3920), y_ = rnd12(T[49] * 3920 + T[46] * -1189); T[49] = y_; T[46] = x_; }
    { const int32_t x_ = rnd12(T[50] * 3920 - T[45] * 1189), y_ = rnd12(T[50] * 1189 + T[45] * 3920); T[50] = y_; T[45] = x_; }
    { const int32_t x_ = rnd12(T[53] * -3612 - T[42] * 1931), y_ = rnd12(T[53] * 1931 + T[42] * -3612); T[53] = y_; T[42] = x_; }
    { const int32_t x_ = rnd12(T[54] * 1931 - T[41] * 3612), y_ = rnd12(T[54] * 3612 + T[41] * 1931); T[54] = y_; T[41] = x_; }
    { const int32_t x_ = rnd12(T[57] * -2598 - T[38] * 3166), y_ = rnd12(T[57] * 3166 + T[38] * -2598); T[57] = y_; T[38] = x_; }
    { const int32_t x_ = rnd12(T[58] * 3166 - T[37] * 2598), y_ = rnd12(T[58] * 2598 + T[37] * 3166); T[58] = y_; T[37] = x_; }
    { const int32_t x_ = rnd12(T[61] * -4076 - T[34] * 401), y_ = rnd12(T[61] * 401 + T[34] * -4076); T[61] = y_; T[34] = x_; }
    { const int32_t x_ = rnd12(T[62] * 401 - T[33] * 4076), y_ = rnd12(T[62] * 4076 + T[33] * 401); T[62] = y_; T[33] = x_; }
    { const int32_t x_ = T[31], y_ = T[30]; T[31] = x_ + y_; T[30] = x_ - y_; }
    { const int32_t x_ = T[28], y_ = T[29]; T[28] = x_ + y_; T[29] = x_ - y_; }
    { const int32_t x_ = T[27], y_ = T[26]; T[27] = x_ + y_; T[26] = x_ - y_; }
    { const int32_t x_ = T[24], y_ = T[25]; T[24] = x_ + y_; T[25] = x_ - y_; }
    { const int32_t x_ = T[23], y_ = T[22]; T[23] = x_ + y_; T[22] = x_ - y_; }
    { const int32_t x_ = T[20], y_ = T[21]; T[20] = x_ + y_; T[21] = x_ - y_; }
    { const int32_t x_ = T[19], y_ = T[18]; T[19] = x_ + y_; T[18] = x_ - y_; }
    { const int32_t x_ = T[16], y_ = T[17]; T[16] = x_ + y_; T[17] = x_ - y_; }
    { const int32_t x_ = rnd12(T[11] * 3920 - T[12] * -1189), y_ = rnd12(T[11] * -1189 + T[12] * 3920); T[11] = x_; T[12] = y_; }
    { const int32_t x_ = rnd12(T[10] * 1931 - T[13] * -3612), y_ = rnd12(T[10] * -3612 + T[13] * 1931); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = rnd12(T[9] * 3166 - T[14] * -2598), y_ = rnd12(T[9] * -2598 + T[14] * 3166); T[9] = x_; T[14] = y_; }
    { const int32_t x_ = rnd12(T[8] * 401 - T[15] * -4076), y_ = rnd12(T[8] * -4076 + T[15] * 401); T[8] = x_; T[15] = y_; }
    { const int32_t x_ = T[63], y_ = T[62]; T[63] = x_ + y_; T[62] = x_ - y_; }
    { const int32_t x_ = T[60], y_ = T[61]; T[60] = x_ + y_; T[61] = x_ - y_; }
    { const int32_t x_ = T[59], y_ = T[58]; T[59] = x_ + y_; T[58] = x_ - y_; }
    { const int32_t x_ = T[56], y_ = T[57]; T[56] = x_ + y_; T[57] = x_ - y_; }
    { const int32_t x_ = T[55], y_ = T[54]; T[55] = x_ + y_; T[54] = x_ - y_; }
    { const int32_t x_ = T[52], y_ = T[53]; T[52] = x_ + y_; T[53] = x_ - y_; }
    { const int32_t x_ = T[51], y_ = T[50]; T[51] = x_ + y_; T[50] = x_ - y_; }
    { const int32_t x_ = T[48], y_ = T[49]; T[48] = x_ + y_; T[49] = x_ - y_; }
    { const int32_t x_ = T[47], y_ = T[46]; T[47] = x_ + y_; T[46] = x_ - y_; }
    { const int32_t x_ = T[44], y_ = T[45]; T[44] = x_ + y_; T[45] = x_ - y_; }
    { const int32_t x_ = T[43], y_ = T[42]; T[43] = x_ + y_; T[42] = x_ - y_; }
    { const int32_t x_ = T[40], y_ = T[41]; T[40] = x_ + y_; T[41] = x_ - y_; }
    { const int32_t x_ = T[39], y_ = T[38]; T[39] = x_ + y_; T[38] = x_ - y_; }
    { const int32_t x_ = T[36], y_ = T[37]; T[36] = x_ + y_; T[37] = x_ - y_; }
    { const int32_t x_ = T[35], y_ = T[34]; T[35] = x_ + y_; T[34] = x_ - y_; }
    { const int32_t x_ = T[32], y_ = T[33]; T[32] = x_ + y_; T[33] = x_ - y_; }
    { const int32_t x_ = rnd12(T[23] * 4052 - T[24] * -601), y_ = rnd12(T[23] * -601 + T[24] * 4052); T[23] = x_; T[24] = y_; }
    { const int32_t x_ = rnd12(T[22] * 2440 - T[25] * -3290), y_ = rnd12(T[22] * -3290 + T[25] * 2440); T[22] = x_; T[25] = y_; }
    { const int32_t x_ = rnd12(T[21] * 3513 - T[26] * -2106), y_ = rnd12(T[21] * -2106 + T[26] * 3513); T[21] = x_; T[26] = y_; }
    { const int32_t x_ = rnd12(T[20] * 995 - T[27] * -3973), y_ = rnd12(T[20] * -3973 + T[27] * 995); T[20] = x_; T[27] = y_; }
    { const int32_t x_ = rnd12(T[19] * 3857 - T[28] * -1380), y_ = rnd12(T[19] * -1380 + T[28] * 3857); T[19] = x_; T[28] = y_; }
    { const int32_t x_ = rnd12(T[18] * 1751 - T[29] * -3703), y_ = rnd12(T[18] * -3703 + T[29] * 1751); T[18] = x_; T[29] = y_; }
    { const int32_t x_ = rnd12(T[17] * 3035 - T[30] * -2751), y_ = rnd12(T[17] * -2751 + T[30] * 3035); T[17] = x_; T[30] = y_; }
    { const int32_t x_ = rnd12(T[16] * 201 - T[31] * -4091), y_ = rnd12(T[16] * -4091 + T[31] * 201); T[16] = x_; T[31] = y_; }
    { const int32_t x_ = rnd12(T[47] * 4085 - T[48] * -301), y_ = rnd12(T[47] * -301 + T[48] * 4085); T[47] = x_; T[48] = y_; }
    { const int32_t x_ = rnd12(T[46] * 2675 - T[49] * -3102), y_ = rnd12(T[46] * -3102 + T[49] * 2675); T[46] = x_; T[49] = y_; }
    { const int32_t x_ = rnd12(T[45] * 3659 - T[50] * -1842), y_ = rnd12(T[45] * -1842 + T[50] * 3659); T[45] = x_; T[50] = y_; }
    { const int32_t x_ = rnd12(T[44] * 1285 - T[51] * -3889), y_ = rnd12(T[44] * -3889 + T[51] * 1285); T[44] = x_; T[51] = y_; }
    { const int32_t x_ = rnd12(T[43] * 3948 - T[52] * -1092), y_ = rnd12(T[43] * -1092 + T[52] * 3948); T[43] = x_; T[52] = y_; }
    { const int32_t x_ = rnd12(T[42] * 2019 - T[53] * -3564), y_ = rnd12(T[42] * -3564 + T[53] * 2019); T[42] = x_; T[53] = y_; }
    { const int32_t x_ = rnd12(T[41] * 3229 - T[54] * -2520), y_ = rnd12(T[41] * -2520 + T[54] * 3229); T[41] = x_; T[54] = y_; }
    { const int32_t x_ = rnd12(T[40] * 501 - T[55] * -4065), y_ = rnd12(T[40] * -4065 + T[55] * 501); T[40] = x_; T[55] = y_; }
    { const int32_t x_ = rnd12(T[39] * 4036 - T[56] * -700), y_ = rnd12(T[39] * -700 + T[56] * 4036); T[39] = x_; T[56] = y_; }
    { const int32_t x_ = rnd12(T[38] * 2359 - T[57] * -3349), y_ = rnd12(T[38] * -3349 + T[57] * 2359); T[38] = x_; T[57] = y_; }
    { const int32_t x_ = rnd12(T[37] * 3461 - T[58] * -2191), y_ = rnd12(T[37] * -2191 + T[58] * 3461); T[37] = x_; T[58] = y_; }
    { const int32_t x_ = rnd12(T[36] * 897 - T[59] * -3996), y_ = rnd12(T[36] * -3996 + T[59] * 897); T[36] = x_; T[59] = y_; }
    { const int32_t x_ = rnd12(T[35] * 3822 - T[60] * -1474), y_ = rnd12(T[35] * -1474 + T[60] * 3822); T[35] = x_; T[60] = y_; }
    { const int32_t x_ = rnd12(T[34] * 1660 - T[61] * -3745), y_ = rnd12(T[34] * -3745 + T[61] * 1660); T[34] = x_; T[61] = y_; }
    { const int32_t x_ = rnd12(T[33] * 2967 - T[62] * -2824), y_ = rnd12(T[33] * -2824 + T[62] * 2967); T[33] = x_; T[62] = y_; }
    { const int32_t x_ = rnd12(T[32] * 101 - T[63] * -4095), y_ = rnd12(T[32] * -4095 + T[63] * 101); T[32] = x_; T[63] = y_; }
    {
        int32_t c_[64];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7]; c_[8] = T[8]; c_[9] = T[9]; c_[10] = T[10]; c_[11] = T[11]; c_[12] = T[12]; c_[13] = T[13]; c_[14] = T[14]; c_[15] = T[15]; c_[16] = T[16]; c_[17] = T[17]; c_[18] = T[18]; c_[19] = T[19]; c_[20] = T[20]; c_[21] = T[21]; c_[22] = T[22]; c_[23] = T[23]; c_[24] = T[24]; c_[25] = T[25]; c_[26] = T[26]; c_[27] = T[27]; c_[28] = T[28]; c_[29] = T[29]; c_[30] = T[30]; c_[31] = T[31]; c_[32] = T[32]; c_[33] = T[33]; c_[34] = T[34]; c_[35] = T[35]; c_[36] = T[36]; c_[37] = T[37]; c_[38] = T[38]; c_[39] = T[39]; c_[40] = T[40]; c_[41] = T[41]; c_[42] = T[42]; c_[43] = T[43]; c_[44] = T[44]; c_[45] = T[45]; c_[46] = T[46]; c_[47] = T[47]; c_[48] = T[48]; c_[49] = T[49]; c_[50] = T[50]; c_[51] = T[51]; c_[52] = T[52]; c_[53] = T[53]; c_[54] = T[54]; c_[55] = T[55]; c_[56] = T[56]; c_[57] = T[57]; c_[58] = T[58]; c_[59] = T[59]; c_[60] = T[60]; c_[61] = T[61]; c_[62] = T[62]; c_[63] = T[63];
        T[0] = c_[0];
        T[32] = c_[1];
        T[16] = c_[2];
        T[48] = c_[3];
        T[8] = c_[4];
        T[40] = c_[5];
        T[24] = c_[6];
        T[56] = c_[7];
        T[4] = c_[8];
        T[36] = c_[9];
        T[20] = c_[10];
        T[52] = c_[11];
        T[12] = c_[12];
        T[44] = c_[13];
        T[28] = c_[14];
        T[60] = c_[15];
        T[2] = c_[16];
        T[34] = c_[17];
        T[18] = c_[18];
        T[50] = c_[19];
        T[10] = c_[20];
        T[42] = c_[21];
        T[26] = c_[22];
        T[58] = c_[23];
        T[6] = c_[24];
        T[38] = c_[25];
        T[22] = c_[26];
        T[54] = c_[27];
        T[14] = c_[28];
        T[46] = c_[29];
        T[30] = c_[30];
        T[62] = c_[31];
        T[1] = c_[32];
        T[33] = c_[33];
        T[17] = c_[34];
        T[49] = c_[35];
        T[9] = c_[36];
        T[41] = c_[37];
        T[25] = c_[38];
        T[57] = c_[39];
        T[5] = c_[40];
        T[37] = c_[41];
        T[21] = c_[42];
        T[53] = c_[43];
        T[13] = c_[44];
        T[45] = c_[45];
        T[29] = c_[46];
        T[61] = c_[47];
        T[3] = c_[48];
        T[35] = c_[49];
        T[19] = c_[50];
        T[51] = c_[51];
        T[11] = c_[52];
        T[43] = c_[53];
        T[27] = c_[54];
        T[59] = c_[55];
        T[7] = c_[56];
        T[39] = c_[57];
        T[23] = c_[58];
        T[55] = c_[59];
        T[15] = c_[60];
        T[47] = c_[61];
        T[31] = c_[62];
        T[63] = c_[63];
    }
}
__host__ __device__ __forceinline__ uint32_t inv_dct64(int32_t *T, int r) {
    uint32_t e_ = 0;
    const int32_t lo_ = -(1 << (r - 1)), hi_ = (1 << (r - 1)) - 1;
    {
        int32_t c_[64];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7]; c_[8] = T[8]; c_[9] = T[9]; c_[10] = T[10]; c_[11] = T[11]; c_[12] = T[12]; c_[13] = T[13]; c_[14] = T[14]; c_[15] = T[15]; c_[16] = T[16]; c_[17] = T[17]; c_[18] = T[18]; c_[19] = T[19]; c_[20] = T[20]; c_[21] = T[21]; c_[22] = T[22]; c_[23] = T[23]; c_[24] = T[24]; c_[25] = T[25]; c_[26] = T[26]; c_[27] = T[27]; c_[28] = T[28]; c_[29] = T[29]; c_[30] = T[30]; c_[31] = T[31]; c_[32] = T[32]; c_[33] = T[33]; c_[34] = T[34]; c_[35] = T[35]; c_[36] = T[36]; c_[37] = T[37]; c_[38] = T[38]; c_[39] = T[39]; c_[40] = T[40]; c_[41] = T[41]; c_[42] = T[42]; c_[43] = T[43]; c_[44] = T[44]; c_[45] = T[45]; c_[46] = T[46]; c_[47] = T[47]; c_[48] = T[48]; c_[49] = T[49]; c_[50] = T[50]; c_[51] = T[51]; c_[52] = T[52]; c_[53] = T[53]; c_[54] = T[54]; c_[55] = T[55]; c_[56] = T[56]; c_[57] = T[57]; c_[58] = T[58]; c_[59] = T[59]; c_[60] = T[60]; c_[61] = T[61]; c_[62] = T[62]; c_[63] = T[63];
        T[0] = c_[0];
        T[1] = c_[32];
        T[2] = c_[16];
        T[3] = c_[48];
        T[4] = c_[8];
        T[5] = c_[40];
        T[6] = c_[24];
        T[7] = c_[56];
        T[8] = c_[4];
        T[9] = c_[36];
        T[10] = c_[20];
        T[11] = c_[52];
        T[12] = c_[12];
        T[13] = c_[44];
        T[14] = c_[28];
        T[15] = c_[60];
        T[16] = c_[2];
        T[17] = c_[34];
        T[18] = c_[18];
        T[19] = c_[50];
        T[20] = c_[10];
        T[21] = c_[42];
        T[22] = c_[26];
        T[23] = c_[58];
        T[24] = c_[6];
        T[25] = c_[38];
        T[26] = c_[22];
        T[27] = c_[54];
        T[28] = c_[14];
        T[29] = c_[46];
        T[30] = c_[30];
        T[31] = c_[62];
        T[32] = c_[1];
        T[33] = c_[33];
        T[34] = c_[17];
        T[35] = c_[49];
        T[36] = c_[9];
        T[37] = c_[41];
        T[38] = c_[25];
        T[39] = c_[57];
        T[40] = c_[5];
        T[41] = c_[37];
        T[42] = c_[21];
        T[43] = c_[53];
        T[44] = c_[13];
        T[45] = c_[45];
        T[46] = c_[29];
        T[47] = c_[61];
        T[48] = c_[3];
        T[49] = c_[35];
        T[50] = c_[19];
        T[51] = c_[51];
        T[52] = c_[11];
        T[53] = c_[43];
        T[54] = c_[27];
        T[55] = c_[59];
        T[56] = c_[7];
        T[57] = c_[39];
        T[58] = c_[23];
        T[59] = c_[55];
        T[60] = c_[15];
        T[61] = c_[47];
        T[62] = c_[31];
        T[63] = c_[63];
    }
    { const int32_t x_ = rnd12(T[32] * 101 - T[63] * 4095), y_ = rnd12(T[32] * 4095 + T[63] * 101); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[32] = x_; T[63] = y_; }
    { const int32_t x_ = rnd12(T[33] * 2967 - T[62] * 2824), y_ = rnd12(T[33] * 2824 + T[62] * 2967); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[33] = x_; T[62] = y_; }
    { const int32_t x_ = rnd12(T[34] * 1660 - T[61] * 3745), y_ = rnd12(T[34] * 3745 + T[61] * 1660); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[34] = x_; T[61] = y_; }
    { const int32_t x_ = rnd12(T[35] * 3822 - T[60] * 1474), y_ = rnd12(T[35] * 1474 + T[60] * 3822); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[35] = x_; T[60] = y_; }
    { const int32_t x_ = rnd12(T[36] * 897 - T[59] * 3996), y_ = rnd12(T[36] * 3996 + T[59] * 897); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[36] = x_; T[59] = y_; }
    { const int32_t x_ = rnd12(T[37] * 3461 - T[58] * 2191), y_ = rnd12(T[37] * 2191 + T[58] * 3461); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[37] = x_; T[58] = y_; }
    { const int32_t x_ = rnd12(T[38] * 2359 - T[57] * 3349), y_ = rnd12(T[38] * 3349 + T[57] * 2359); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[38] = x_; T[57] = y_; }
    { const int32_t x_ = rnd12(T[39] * 4036 - T[56] * 700), y_ = rnd12(T[39] * 700 + T[56] * 4036); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[39] = x_; T[56] = y_; }
    { const int32_t x_ = rnd12(T[40] * 501 - T[55] * 4065), y_ = rnd12(T[40] * 4065 + T[55] * 501); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[40] = x_; T[55] = y_; }
    { const int32_t x_ = rnd12(T[41] * 3229 - T[54] * 2520), y_ = rnd12(T[41] * 2520 + T[54] * 3229); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[41] = x_; T[54] = y_; }
    { const int32_t x_ = rnd12(T[42] * 2019 - T[53] * 3564), y_ = rnd12(T[42] * 3564 + T[53] * 2019); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[42] = x_; T[53] = y_; }
    { const int32_t x_ = rnd12(T[43] * 3948 - T[52] * 1092), y_ = rnd12(T[43] * 1092 + T[52] * 3948); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[43] = x_; T[52] = y_; }
    { const int32_t x_ = rnd12(T[44] * 1285 - T[51] * 3889), y_ = rnd12(T[44] * 3889 + T[51] * 1285); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[44] = x_; T[51] = y_; }
    { const int32_t x_ = rnd12(T[45] * 3659 - T[50] * 1842), y_ = rnd12(T[45] * 1842 + T[50] * 3659); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[45] = x_; T[50] = y_; }
    { const int32_t x_ = rnd12(T[46] * 2675 - T[49] * 3102), y_ = rnd12(T[46] * 3102 + T[49] * 2675); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[46] = x_; T[49] = y_; }
    { const int32_t x_ = rnd12(T[47] * 4085 - T[48] * 301), y_ = rnd12(T[47] * 301 + T[48] * 4085); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[47] = x_; T[48] = y_; }
    { const int32_t x_ = rnd12(T[16] * 201 - T[31] * 4091), y_ = rnd12(T[16] * 4091 + T[31] * 201); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[16] = x_; T[31] = y_; }
    { const int32_t x_ = rnd12(T[17] * 3035 - T[30] * 2751), y_ = rnd12(T[17] * 2751 + T[30] * 3035); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[17] = x_; T[30] = y_; }
    { const int32_t x_ = rnd12(T[18] * 1751 - T[29] * 3703), y_ = rnd12(T[18] * 3703 + T[29] * 1751); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[18] = x_; T[29] = y_; }
    { const int32_t x_ = rnd12(T[19] * 3857 - T[28] * 1380), y_ = rnd12(T[19] * 1380 + T[28] * 3857); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[19] = x_; T[28] = y_; }
    { const int32_t x_ = rnd12(T[20] * 995 - T[27] * 3973), y_ = rnd12(T[20] * 3973 + T[27] * 995); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[20] = x_; T[27] = y_; }
    { const int32_t x_ = rnd12(T[21] * 3513 - T[26] * 2106), y_ = rnd12(T[21] * 2106 + T[26] * 3513); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[21] = x_; T[26] = y_; }
    { const int32_t x_ = rnd12(T[22] * 2440 - T[25] * 3290), y_ = rnd12(T[22] * 3290 + T[25] * 2440); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[22] = x_; T[25] = y_; }
    { const int32_t x_ = rnd12(T[23] * 4052 - T[24] * 601), y_ = rnd12(T[23] * 601 + T[24] * 4052); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[23] = x_; T[24] = y_; }
    { const int32_t x_ = T[32], y_ = T[33]; T[32] = clampr(x_ + y_, lo_, hi_); T[33] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[35], y_ = T[34]; T[35] = clampr(x_ + y_, lo_, hi_); T[34] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[36], y_ = T[37]; T[36] = clampr(x_ + y_, lo_, hi_); T[37] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[39], y_ = T[38]; T[39] = clampr(x_ + y_, lo_, hi_); T[38] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[40], y_ = T[41]; T[40] = clampr(x_ + y_, lo_, hi_); T[41] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[43], y_ = T[42]; T[43] = clampr(x_ + y_, lo_, hi_); T[42] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[44], y_ = T[45]; T[44] = clampr(x_ + y_, lo_, hi_); T[45] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[47], y_ = T[46]; T[47] = clampr(x_ + y_, lo_, hi_); T[46] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[48], y_ = T[49]; T[48] = clampr(x_ + y_, lo_, hi_); T[49] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[51], y_ = T[50]; T[51] = clampr(x_ + y_, lo_, hi_); T[50] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[52], y_ = T[53]; T[52] = clampr(x_ + y_, lo_, hi_); T[53] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[55], y_ = T[54]; T[55] = clampr(x_ + y_, lo_, hi_); T[54] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[56], y_ = T[57]; T[56] = clampr(x_ + y_, lo_, hi_); T[57] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[59], y_ = T[58]; T[59] = clampr(x_ + y_, lo_, hi_); T[58] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[60], y_ = T[61]; T[60] = clampr(x_ + y_, lo_, hi_); T[61] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[63], y_ = T[62]; T[63] = clampr(x_ + y_, lo_, hi_); T[62] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[8] * 401 - T[15] * 4076), y_ = rnd12(T[8] * 4076 + T[15] * 401); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[8] = x_; T[15] = y_; }
    { const int32_t x_ = rnd12(T[9] * 3166 - T[14] * 2598), y_ = rnd12(T[9] * 2598 + T[14] * 3166); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[9] = x_; T[14] = y_; }
    { const int32_t x_ = rnd12(T[10] * 1931 - T[13] * 3612), y_ = rnd12(T[10] * 3612 + T[13] * 1931); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = rnd12(T[11] * 3920 - T[12] * 1189), y_ = rnd12(T[11] * 1189 + T[12] * 3920); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[11] = x_; T[12] = y_; }
    { const int32_t x_ = T[16], y_ = T[17]; T[16] = clampr(x_ + y_, lo_, hi_); T[17] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[19], y_ = T[18]; T[19] = clampr(x_ + y_, lo_, hi_); T[18] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[20], y_ = T[21]; T[20] = clampr(x_ + y_, lo_, hi_); T[21] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[23], y_ = T[22]; T[23] = clampr(x_ + y_, lo_, hi_); T[22] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[24], y_ = T[25]; T[24] = clampr(x_ + y_, lo_, hi_); T[25] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[27], y_ = T[26]; T[27] = clampr(x_ + y_, lo_, hi_); T[26] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[28], y_ = T[29]; T[28] = clampr(x_ + y_, lo_, hi_); T[29] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[31], y_ = T[30]; T[31] = clampr(x_ + y_, lo_, hi_); T[30] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[62] * 401 - T[33] * 4076), y_ = rnd12(T[62] * 4076 + T[33] * 401); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[33] = x_; T[62] = y_; }
    { const int32_t x_ = rnd12(T[61] * -4076 - T[34] * 401), y_ = rnd12(T[61] * 401 + T[34] * -4076); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[34] = x_; T[61] = y_; }
    { const int32_t x_ = rnd12(T[58] * 3166 - T[37] * 2598), y_ = rnd12(T[58] * 2598 + T[37] * 3166); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[37] = x_; T[58] = y_; }
    { const int32_t x_ = rnd12(T[57] * -2598 - T[38] * 3166), y_ = rnd12(T[57] * 3166 + T[38] * -2598); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[38] = x_; T[57] = y_; }
    { const int32_t x_ = rnd12(T[54] * 1931 - T[41] * 3612), y_ = rnd12(T[54] * 3612 + T[41] * 1931); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[41] = x_; T[54] = y_; }
    { const int32_t x_ = rnd12(T[53] * -3612 - T[42] * 1931), y_ = rnd12(T[53] * 1931 + T[42] * -3612); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[42] = x_; T[53] = y_; }
    { const int32_t x_ = rnd12(T[50] * 3920 - T[45] * 1189), y_ = rnd12(T[50] * 1189 + T[45] * 3920); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[45] = x_; T[50] = y_; }
    { const int32_t x_ = rnd12(T[49] * -1189 - T[46] * 3920), y_ = rnd12(T[49] * 3920 + T[46] * -1189); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[46] = x_; T[49] = y_; }
    { const int32_t x_ = rnd12(T[4] * 799 - T[7] * 4017), y_ = rnd12(T[4] * 4017 + T[7] * 799); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[4] = x_; T[7] = y_; }
    { const int32_t x_ = rnd12(T[5] * 3406 - T[6] * 2276), y_ = rnd12(T[5] * 2276 + T[6] * 3406); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = T[8], y_ = T[9]; T[8] = clampr(x_ + y_, lo_, hi_); T[9] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[11], y_ = T[10]; T[11] = clampr(x_ + y_, lo_, hi_); T[10] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[12], y_ = T[13]; T[12] = clampr(x_ + y_, lo_, hi_); T[13] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[15], y_ = T[14]; T[15] = clampr(x_ + y_, lo_, hi_); T[14] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[30] * 799 - T[17] * 4017), y_ = rnd12(T[30] * 4017 + T[17] * 799); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[17] = x_; T[30] = y_; }
    { const int32_t x_ = rnd12(T[29] * -4017 - T[18] * 799), y_ = rnd12(T[29] * 799 + T[18] * -4017); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[18] = x_; T[29] = y_; }
    { const int32_t x_ = rnd12(T[26] * 3406 - T[21] * 2276), y_ = rnd12(T[26] * 2276 + T[21] * 3406); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[21] = x_; T[26] = y_; }
    { const int32_t x_ = rnd12(T[25] * -2276 - T[22] * 3406), y_ = rnd12(T[25] * 3406 + T[22] * -2276); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[22] = x_; T[25] = y_; }
    { const int32_t x_ = T[32], y_ = T[35]; T[32] = clampr(x_ + y_, lo_, hi_); T[35] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[33], y_ = T[34]; T[33] = clampr(x_ + y_, lo_, hi_); T[34] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[39], y_ = T[36]; T[39] = clampr(x_ + y_, lo_, hi_); T[36] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[38], y_ = T[37]; T[38] = clampr(x_ + y_, lo_, hi_); T[37] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[40], y_ = T[43]; T[40] = clampr(x_ + y_, lo_, hi_); T[43] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[41], y_ = T[42]; T[41] = clampr(x_ + y_, lo_, hi_); T[42] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[47], y_ = T[44]; T[47] = clampr(x_ + y_, lo_, hi_); T[44] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[46], y_ = T[45]; T[46] = clampr(x_ + y_, lo_, hi_); T[45] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[48], y_ = T[51]; T[48] = clampr(x_ + y_, lo_, hi_); T[51] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[49], y_ = T[50]; T[49] = clampr(x_ + y_, lo_, hi_); T[50] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[55], y_ = T[52]; T[55] = clampr(x_ + y_, lo_, hi_); T[52] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[54], y_ = T[53]; T[54] = clampr(x_ + y_, lo_, hi_); T[53] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[56], y_ = T[59]; T[56] = clampr(x_ + y_, lo_, hi_); T[59] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[57], y_ = T[58]; T[57] = clampr(x_ + y_, lo_, hi_); T[58] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[63], y_ = T[60]; T[63] = clampr(x_ + y_, lo_, hi_); T[60] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[62], y_ = T[61]; T[62] = clampr(x_ + y_, lo_, hi_); T[61] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[0] * 2896 - T[1] * 2896), y_ = rnd12(T[0] * 2896 + T[1] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[1] = x_; T[0] = y_; }
    { const int32_t x_ = rnd12(T[2] * 1567 - T[3] * 3784), y_ = rnd12(T[2] * 3784 + T[3] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[2] = x_; T[3] = y_; }
    { const int32_t x_ = T[4], y_ = T[5]; T[4] = clampr(x_ + y_, lo_, hi_); T[5] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[7], y_ = T[6]; T[7] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[14] * 1567 - T[9] * 3784), y_ = rnd12(T[14] * 3784 + T[9] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[9] = x_; T[14] = y_; }
    { const int32_t x_ = rnd12(T[13] * -3784 - T[10] * 1567), y_ = rnd12(T[13] * 1567 + T[10] * -3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = T[16], y_ = T[19]; T[16] = clampr(x_ + y_, lo_, hi_); T[19] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[17], y_ = T[18]; T[17] = clampr(x_ + y_, lo_, hi_); T[18] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[23], y_ = T[20]; T[23] = clampr(x_ + y_, lo_, hi_); T[20] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[22], y_ = T[21]; T[22] = clampr(x_ + y_, lo_, hi_); T[21] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[24], y_ = T[27]; T[24] = clampr(x_ + y_, lo_, hi_); T[27] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[25], y_ = T[26]; T[25] = clampr(x_ + y_, lo_, hi_); T[26] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[31], y_ = T[28]; T[31] = clampr(x_ + y_, lo_, hi_); T[28] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[30], y_ = T[29]; T[30] = clampr(x_ + y_, lo_, hi_); T[29] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[61] * 799 - T[34] * 4017), y_ = rnd12(T[61] * 4017 + T[34] * 799); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[34] = x_; T[61] = y_; }
    { const int32_t x_ = rnd12(T[60] * 799 - T[35] * 4017), y_ = rnd12(T[60] * 4017 + T[35] * 799); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[35] = x_; T[60] = y_; }
    { const int32_t x_ = rnd12(T[59] * -4017 - T[36] * 799), y_ = rnd12(T[59] * 799 + T[36] * -4017); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[36] = x_; T[59] = y_; }
    { const int32_t x_ = rnd12(T[58] * -4017 - T[37] * 799), y_ = rnd12(T[58] * 799 + T[37] * -4017); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[37] = x_; T[58] = y_; }
    { const int32_t x_ = rnd12(T[53] * 3406 - T[42] * 2276), y_ = rnd12(T[53] * 2276 + T[42] * 3406); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[42] = x_; T[53] = y_; }
    { const int32_t x_ = rnd12(T[52] * 3406 - T[43] * 2276), y_ = rnd12(T[52] * 2276 + T[43] * 3406); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[43] = x_; T[52] = y_; }
    { const int32_t x_ = rnd12(T[51] * -2276 - T[44] * 3406), y_ = rnd12(T[51] * 3406 + T[44] * -2276); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[44] = x_; T[51] = y_; }
    { const int32_t x_ = rnd12(T[50] * -2276 - T[45] * 3406), y_ = rnd12(T[50] * 3406 + T[45] * -2276); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[45] = x_; T[50] = y_; }
    { const int32_t x_ = T[0], y_ = T[3]; T[0] = clampr(x_ + y_, lo_, hi_); T[3] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[2]; T[1] = clampr(x_ + y_, lo_, hi_); T[2] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[5] * 2896), y_ = rnd12(T[6] * 2896 + T[5] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[6] = y_; }
    { const int32_t x_ = T[8], y_ = T[11]; T[8] = clampr(x_ + y_, lo_, hi_); T[11] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[9], y_ = T[10]; T[9] = clampr(x_ + y_, lo_, hi_); T[10] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[15], y_ = T[12]; T[15] = clampr(x_ + y_, lo_, hi_); T[12] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[14], y_ = T[13]; T[14] = clampr(x_ + y_, lo_, hi_); T[13] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[29] * 1567 - T[18] * 3784), y_ = rnd12(T[29] * 3784 + T[18] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[18] = x_; T[29] = y_; }
    { const int32_t x_ = rnd12(T[28] * 1567 - T[19] * 3784), y_ = rnd12(T[28] * 3784 + T[19] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[19] = x_; T[28] = y_; }
    { const int32_t x_ = rnd12(T[27] * -3784 - T[20] * 1567), y_ = rnd12(T[27] * 1567 + T[20] * -3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[20] = x_; T[27] = y_; }
    { const int32_t x_ = rnd12(T[26] * -3784 - T[21] * 1567), y_ = rnd12(T[26] * 1567 + T[21] * -3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[21] = x_; T[26] = y_; }
    { const int32_t x_ = T[32], y_ = T[39]; T[32] = clampr(x_ + y_, lo_, hi_); T[39] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[33], y_ = T[38]; T[33] = clampr(x_ + y_, lo_, hi_); T[38] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[34], y_ = T[37]; T[34] = clampr(x_ + y_, lo_, hi_); T[37] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[35], y_ = T[36]; T[35] = clampr(x_ + y_, lo_, hi_); T[36] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[47], y_ = T[40]; T[47] = clampr(x_ + y_, lo_, hi_); T[40] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[46], y_ = T[41]; T[46] = clampr(x_ + y_, lo_, hi_); T[41] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[45], y_ = T[42]; T[45] = clampr(x_ + y_, lo_, hi_); T[42] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[44], y_ = T[43]; T[44] = clampr(x_ + y_, lo_, hi_); T[43] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[48], y_ = T[55]; T[48] = clampr(x_ + y_, lo_, hi_); T[55] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[49], y_ = T[54]; T[49] = clampr(x_ + y_, lo_, hi_); T[54] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[50], y_ = T[53]; T[50] = clampr(x_ + y_, lo_, hi_); T[53] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[51], y_ = T[52]; T[51] = clampr(x_ + y_, lo_, hi_); T[52] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[63], y_ = T[56]; T[63] = clampr(x_ + y_, lo_, hi_); T[56] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[62], y_ = T[57]; T[62] = clampr(x_ + y_, lo_, hi_); T[57] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[61], y_ = T[58]; T[61] = clampr(x_ + y_, lo_, hi_); T[58] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[60], y_ = T[59]; T[60] = clampr(x_ + y_, lo_, hi_); T[59] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[0], y_ = T[7]; T[0] = clampr(x_ + y_, lo_, hi_); T[7] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[6]; T[1] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[5]; T[2] = clampr(x_ + y_, lo_, hi_); T[5] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[4]; T[3] = clampr(x_ + y_, lo_, hi_); T[4] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[13] * 2896 - T[10] * 2896), y_ = rnd12(T[13] * 2896 + T[10] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[10] = x_; T[13] = y_; }
    { const int32_t x_ = rnd12(T[12] * 2896 - T[11] * 2896), y_ = rnd12(T[12] * 2896 + T[11] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[11] = x_; T[12] = y_; }
    { const int32_t x_ = T[16], y_ = T[23]; T[16] = clampr(x_ + y_, lo_, hi_); T[23] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[17], y_ = T[22]; T[17] = clampr(x_ + y_, lo_, hi_); T[22] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[18], y_ = T[21]; T[18] = clampr(x_ + y_, lo_, hi_); T[21] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[19], y_ = T[20]; T[19] = clampr(x_ + y_, lo_, hi_); T[20] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[31], y_ = T[24]; T[31] = clampr(x_ + y_, lo_, hi_); T[24] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[30], y_ = T[25]; T[30] = clampr(x_ + y_, lo_, hi_); T[25] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[29], y_ = T[26]; T[29] = clampr(x_ + y_, lo_, hi_); T[26] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[28], y_ = T[27]; T[28] = clampr(x_ + y_, lo_, hi_); T[27] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[59] * 1567 - T[36] * 3784), y_ = rnd12(T[59] * 3784 + T[36] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[36] = x_; T[59] = y_; }
    { const int32_t x_ = rnd12(T[58] * 1567 - T[37] * 3784), y_ = rnd12(T[58] * 3784 + T[37] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[37] = x_; T[58] = y_; }
    { const int32_t x_ = rnd12(T[57] * 1567 - T[38] * 3784), y_ = rnd12(T[57] * 3784 + T[38] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[38] = x_; T[57] = y_; }
    { const int32_t x_ = rnd12(T[56] * 1567 - T[39] * 3784), y_ = rnd12(T[56] * 3784 + T[39] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[39] = x_; T[56] = y_; }
    { const int32_t x_ = rnd12(T[55] * -3784 - T[40] * 1567), y_ = rnd12(T[55] * 1567 + T[40] * -3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[40] = x_; T[55] = y_; }
    { const int32_t x_ = rnd12(T[54] * -3784 - T[41] * 1567), y_ = rnd12(T[54] * 1567 + T[41] * -3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[41] = x_; T[54] = y_; }
    { const int32_t x_ = rnd12(T[53] * -3784 - T[42] * 1567), y_ = rnd12(T[53] * 1567 + T[42] * -3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[42] = x_; T[53] = y_; }
    { const int32_t x_ = rnd12(T[52] * -3784 - T[43] * 1567), y_ = rnd12(T[52] * 1567 + T[43] * -3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[43] = x_; T[52] = y_; }
    { const int32_t x_ = T[0], y_ = T[15]; T[0] = clampr(x_ + y_, lo_, hi_); T[15] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[14]; T[1] = clampr(x_ + y_, lo_, hi_); T[14] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[13]; T[2] = clampr(x_ + y_, lo_, hi_); T[13] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[12]; T[3] = clampr(x_ + y_, lo_, hi_); T[12] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[4], y_ = T[11]; T[4] = clampr(x_ + y_, lo_, hi_); T[11] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[5], y_ = T[10]; T[5] = clampr(x_ + y_, lo_, hi_); T[10] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[6], y_ = T[9]; T[6] = clampr(x_ + y_, lo_, hi_); T[9] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[7], y_ = T[8]; T[7] = clampr(x_ + y_, lo_, hi_); T[8] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[27] * 2896 - T[20] * 2896), y_ = rnd12(T[27] * 2896 + T[20] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[20] = x_; T[27] = y_; }
    { const int32_t x_ = rnd12(T[26] * 2896 - T[21] * 2896), y_ = rnd12(T[26] * 2896 + T[21] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[21] = x_; T[26] = y_; }
    { const int32_t x_ = rnd12(T[25] * 2896 - T[22] * 2896), y_ = rnd12(T[25] * 2896 + T[22] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[22] = x_; T[25] = y_; }
    { const int32_t x_ = rnd12(T[24] * 2896 - T[23] * 2896), y_ = rnd12(T[24] * 2896 + T[23] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[23] = x_; T[24] = y_; }
    { const int32_t x_ = T[32], y_ = T[47]; T[32] = clampr(x_ + y_, lo_, hi_); T[47] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[63], y_ = T[48]; T[63] = clampr(x_ + y_, lo_, hi_); T[48] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[33], y_ = T[46]; T[33] = clampr(x_ + y_, lo_, hi_); T[46] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[62], y_ = T[49]; T[62] = clampr(x_ + y_, lo_, hi_); T[49] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[34], y_ = T[45]; T[34] = clampr(x_ + y_, lo_, hi_); T[45] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[61], y_ = T[50]; T[61] = clampr(x_ + y_, lo_, hi_); T[50] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[35], y_ = T[44]; T[35] = clampr(x_ + y_, lo_, hi_); T[44] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[60], y_ = T[51]; T[60] = clampr(x_ + y_, lo_, hi_); T[51] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[36], y_ = T[43]; T[36] = clampr(x_ + y_, lo_, hi_); T[43] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[59], y_ = T[52]; T[59] = clampr(x_ + y_, lo_, hi_); T[52] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[37], y_ = T[42]; T[37] = clampr(x_ + y_, lo_, hi_); T[42] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[58], y_ = T[53]; T[58] = clampr(x_ + y_, lo_, hi_); T[53] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[38], y_ = T[41]; T[38] = clampr(x_ + y_, lo_, hi_); T[41] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[57], y_ = T[54]; T[57] = clampr(x_ + y_, lo_, hi_); T[54] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[39], y_ = T[40]; T[39] = clampr(x_ + y_, lo_, hi_); T[40] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[56], y_ = T[55]; T[56] = clampr(x_ + y_, lo_, hi_); T[55] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[0], y_ = T[31]; T[0] = clampr(x_ + y_, lo_, hi_); T[31] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[30]; T[1] = clampr(x_ + y_, lo_, hi_); T[30] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[29]; T[2] = clampr(x_ + y_, lo_, hi_); T[29] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[28]; T[3] = clampr(x_ + y_, lo_, hi_); T[28] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[4], y_ = T[27]; T[4] = clampr(x_ + y_, lo_, hi_); T[27] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[5], y_ = T[26]; T[5] = clampr(x_ + y_, lo_, hi_); T[26] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[6], y_ = T[25]; T[6] = clampr(x_ + y_, lo_, hi_); T[25] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[7], y_ = T[24]; T[7] = clampr(x_ + y_, lo_, hi_); T[24] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[8], y_ = T[23]; T[8] = clampr(x_ + y_, lo_, hi_); T[23] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[9], y_ = T[22]; T[9] = clampr(x_ + y_, lo_, hi_); T[22] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[10], y_ = T[21]; T[10] = clampr(x_ + y_, lo_, hi_); T[21] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[11], y_ = T[20]; T[11] = clampr(x_ + y_, lo_, hi_); T[20] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[12], y_ = T[19]; T[12] = clampr(x_ + y_, lo_, hi_); T[19] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[13], y_ = T[18]; T[13] = clampr(x_ + y_, lo_, hi_); T[18] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[14], y_ = T[17]; T[14] = clampr(x_ + y_, lo_, hi_); T[17] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[15], y_ = T[16]; T[15] = clampr(x_ + y_, lo_, hi_); T[16] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[55] * 2896 - T[40] * 2896), y_ = rnd12(T[55] * 2896 + T[40] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[40] = x_; T[55] = y_; }
    { const int32_t x_ = rnd12(T[54] * 2896 - T[41] * 2896), y_ = rnd12(T[54] * 2896 + T[41] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[41] = x_; T[54] = y_; }
    { const int32_t x_ = rnd12(T[53] * 2896 - T[42] * 2896), y_ = rnd12(T[53] * 2896 + T[42] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[42] = x_; T[53] = y_; }
    { const int32_t x_ = rnd12(T[52] * 2896 - T[43] * 2896), y_ = rnd12(T[52] * 2896 + T[43] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[43] = x_; T[52] = y_; }
    { const int32_t x_ = rnd12(T[51] * 2896 - T[44] * 2896), y_ = rnd12(T[51] * 2896 + T[44] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[44] = x_; T[51] = y_; }
    { const int32_t x_ = rnd12(T[50] * 2896 - T[45] * 2896), y_ = rnd12(T[50] * 2896 + T[45] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[45] = x_; T[50] = y_; }
    { const int32_t x_ = rnd12(T[49] * 2896 - T[46] * 2896), y_ = rnd12(T[49] * 2896 + T[46] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[46] = x_; T[49] = y_; }
    { const int32_t x_ = rnd12(T[48] * 2896 - T[47] * 2896), y_ = rnd12(T[48] * 2896 + T[47] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[47] = x_; T[48] = y_; }
    { const int32_t x_ = T[0], y_ = T[63]; T[0] = clampr(x_ + y_, lo_, hi_); T[63] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[62]; T[1] = clampr(x_ + y_, lo_, hi_); T[62] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[61]; T[2] = clampr(x_ + y_, lo_, hi_); T[61] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[60]; T[3] = clampr(x_ + y_, lo_, hi_); T[60] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[4], y_ = T[59]; T[4] = clampr(x_ + y_, lo_, hi_); T[59] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[5], y_ = T[58]; T[5] = clampr(x_ + y_, lo_, hi_); T[58] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[6], y_ = T[57]; T[6] = clampr(x_ + y_, lo_, hi_); T[57] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[7], y_ = T[56]; T[7] = clampr(x_ + y_, lo_, hi_); T[56] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[8], y_ = T[55]; T[8] = clampr(x_ + y_, lo_, hi_); T[55] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[9], y_ = T[54]; T[9] = clampr(x_ + y_, lo_, hi_); T[54] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[10], y_ = T[53]; T[10] = clampr(x_ + y_, lo_, hi_); T[53] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[11], y_ = T[52]; T[11] = clampr(x_ + y_, lo_, hi_); T[52] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[12], y_ = T[51]; T[12] = clampr(x_ + y_, lo_, hi_); T[51] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[13], y_ = T[50]; T[13] = clampr(x_ + y_, lo_, hi_); T[50] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[14], y_ = T[49]; T[14] = clampr(x_ + y_, lo_, hi_); T[49] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[15], y_ = T[48]; T[15] = clampr(x_ + y_, lo_, hi_); T[48] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[16], y_ = T[47]; T[16] = clampr(x_ + y_, lo_, hi_); T[47] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[17], y_ = T[46]; T[17] = clampr(x_ + y_, lo_, hi_); T[46] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[18], y_ = T[45]; T[18] = clampr(x_ + y_, lo_, hi_); T[45] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[19], y_ = T[44]; T[19] = clampr(x_ + y_, lo_, hi_); T[44] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[20], y_ = T[43]; T[20] = clampr(x_ + y_, lo_, hi_); T[43] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[21], y_ = T[42]; T[21] = clampr(x_ + y_, lo_, hi_); T[42] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[22], y_ = T[41]; T[22] = clampr(x_ + y_, lo_, hi_); T[41] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[23], y_ = T[40]; T[23] = clampr(x_ + y_, lo_, hi_); T[40] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[24], y_ = T[39]; T[24] = clampr(x_ + y_, lo_, hi_); T[39] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[25], y_ = T[38]; T[25] = clampr(x_ + y_, lo_, hi_); T[38] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[26], y_ = T[37]; T[26] = clampr(x_ + y_, lo_, hi_); T[37] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[27], y_ = T[36]; T[27] = clampr(x_ + y_, lo_, hi_); T[36] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[28], y_ = T[35]; T[28] = clampr(x_ + y_, lo_, hi_); T[35] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[29], y_ = T[34]; T[29] = clampr(x_ + y_, lo_, hi_); T[34] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[30], y_ = T[33]; T[30] = clampr(x_ + y_, lo_, hi_); T[33] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[31], y_ = T[32]; T[31] = clampr(x_ + y_, lo_, hi_); T[32] = clampr(x_ - y_, lo_, hi_); }
    return e_;
}
__host__ __device__ __forceinline__ void fwd_adst8(int32_t *T) {
    {
        int32_t c_[8];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7];
        T[0] = c_[0];
        T[4] = -c_[1];
        T[6] = c_[2];
        T[2] = -c_[3];
        T[3] = c_[4];
        T[7] = -c_[5];
        T[5] = c_[6];
        T[1] = -c_[7];
    }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[7] * 2896), y_ = rnd12(T[6] * 2896 + T[7] * 2896); T[6] = y_; T[7] = x_; }
    { const int32_t x_ = rnd12(T[2] * 2896 - T[3] * 2896), y_ = rnd12(T[2] * 2896 + T[3] * 2896); T[2] = y_; T[3] = x_; }
    { const int32_t x_ = T[5], y_ = T[7]; T[5] = x_ + y_; T[7] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[3]; T[1] = x_ + y_; T[3] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[6]; T[4] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[2]; T[0] = x_ + y_; T[2] = x_ - y_; }
    { const int32_t x_ = rnd12(T[7] * 3784 - T[6] * 1567), y_ = rnd12(T[7] * 1567 + T[6] * 3784); T[7] = y_; T[6] = x_; }
    { const int32_t x_ = rnd12(T[4] * 1567 - T[5] * 3784), y_ = rnd12(T[4] * 3784 + T[5] * 1567); T[4] = y_; T[5] = x_; }
    { const int32_t x_ = T[3], y_ = T[7]; T[3] = x_ + y_; T[7] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[6]; T[2] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[5]; T[1] = x_ + y_; T[5] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[4]; T[0] = x_ + y_; T[4] = x_ - y_; }
    { const int32_t x_ = rnd12(T[6] * 3920 - T[7] * 1189), y_ = rnd12(T[6] * 1189 + T[7] * 3920); T[6] = y_; T[7] = x_; }
    { const int32_t x_ = rnd12(T[4] * 3166 - T[5] * 2598), y_ = rnd12(T[4] * 2598 + T[5] * 3166); T[4] = y_; T[5] = x_; }
    { const int32_t x_ = rnd12(T[2] * 1931 - T[3] * 3612), y_ = rnd12(T[2] * 3612 + T[3] * 1931); T[2] = y_; T[3] = x_; }
    { const int32_t x_ = rnd12(T[0] * 401 - T[1] * 4076), y_ = rnd12(T[0] * 4076 + T[1] * 401); T[0] = y_; T[1] = x_; }
    {
        int32_t c_[8];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7];
        T[7] = c_[0];
        T[0] = c_[1];
        T[5] = c_[2];
        T[2] = c_[3];
        T[3] = c_[4];
        T[4] = c_[5];
        T[1] = c_[6];
        T[6] = c_[7];
    }
}
__host__ __device__ __forceinline__ uint32_t inv_adst8(int32_t *T, int r) {
    uint32_t e_ = 0;
    const int32_t lo_ = -(1 << (r - 1)), hi_ = (1 << (r - 1)) - 1;
    {
        int32_t c_[8];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7];
        T[0] = c_[7];
        T[1] = c_[0];
        T[2] = c_[5];
        T[3] = c_[2];
        T[4] = c_[3];
        T[5] = c_[4];
        T[6] = c_[1];
        T[7] = c_[6];
    }
    { const int32_t x_ = rnd12(T[0] * 401 - T[1] * 4076), y_ = rnd12(T[0] * 4076 + T[1] * 401); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[1] = x_; T[0] = y_; }
    { const int32_t x_ = rnd12(T[2] * 1931 - T[3] * 3612), y_ = rnd12(T[2] * 3612 + T[3] * 1931); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[3] = x_; T[2] = y_; }
    { const int32_t x_ = rnd12(T[4] * 3166 - T[5] * 2598), y_ = rnd12(T[4] * 2598 + T[5] * 3166); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[4] = y_; }
    { const int32_t x_ = rnd12(T[6] * 3920 - T[7] * 1189), y_ = rnd12(T[6] * 1189 + T[7] * 3920); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[7] = x_; T[6] = y_; }
    { const int32_t x_ = T[0], y_ = T[4]; T[0] = clampr(x_ + y_, lo_, hi_); T[4] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[5]; T[1] = clampr(x_ + y_, lo_, hi_); T[5] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[6]; T[2] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[7]; T[3] = clampr(x_ + y_, lo_, hi_); T[7] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[4] * 1567 - T[5] * 3784), y_ = rnd12(T[4] * 3784 + T[5] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[4] = y_; }
    { const int32_t x_ = rnd12(T[7] * 3784 - T[6] * 1567), y_ = rnd12(T[7] * 1567 + T[6] * 3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[6] = x_; T[7] = y_; }
    { const int32_t x_ = T[0], y_ = T[2]; T[0] = clampr(x_ + y_, lo_, hi_); T[2] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[4], y_ = T[6]; T[4] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[3]; T[1] = clampr(x_ + y_, lo_, hi_); T[3] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[5], y_ = T[7]; T[5] = clampr(x_ + y_, lo_, hi_); T[7] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[2] * 2896 - T[3] * 2896), y_ = rnd12(T[2] * 2896 + T[3] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[3] = x_; T[2] = y_; }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[7] * 2896), y_ = rnd12(T[6] * 2896 + T[7] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[7] = x_; T[6] = y_; }
    {
        int32_t c_[8];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7];
        T[0] = c_[0];
        T[1] = -c_[4];
        T[2] = c_[6];
        T[3] = -c_[2];
        T[4] = c_[3];
        T[5] = -c_[7];
        T[6] = c_[5];
        T[7] = -c_[1];
    }
    return e_;
}
__host__ __device__ __forceinline__ void fwd_adst16(int32_t *T) {
    {
        int32_t c_[16];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7]; c_[8] = T[8]; c_[9] = T[9]; c_[10] = T[10]; c_[11] = T[11]; c_[12] = T[12]; c_[13] = T[13]; c_[14] = T[14]; c_[15] = T[15];
        T[0] = c_[0];
        T[8] = -c_[1];
        T[12] = c_[2];
        T[4] = -c_[3];
        T[6] = c_[4];
        T[14] = -c_[5];
        T[10] = c_[6];
        T[2] = -c_[7];
        T[3] = c_[8];
        T[11] = -c_[9];
        T[15] = c_[10];
        T[7] = -c_[11];
        T[5] = c_[12];
        T[13] = -c_[13];
        T[9] = c_[14];
        T[1] = -c_[15];
    }
    { const int32_t x_ = rnd12(T[14] * 2896 - T[15] * 2896), y_ = rnd12(T[14] * 2896 + T[15] * 2896); T[14] = y_; T[15] = x_; }
    { const int32_t x_ = rnd12(T[10] * 2896 - T[11] * 2896), y_ = rnd12(T[10] * 2896 + T[11] * 2896); T[10] = y_; T[11] = x_; }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[7] * 2896), y_ = rnd12(T[6] * 2896 + T[7] * 2896); T[6] = y_; T[7] = x_; }
    { const int32_t x_ = rnd12(T[2] * 2896 - T[3] * 2896), y_ = rnd12(T[2] * 2896 + T[3] * 2896); T[2] = y_; T[3] = x_; }
    { const int32_t x_ = T[13], y_ = T[15]; T[13] = x_ + y_; T[15] = x_ - y_; }
    { const int32_t x_ = T[9], y_ = T[11]; T[9] = x_ + y_; T[11] = x_ - y_; }
    { const int32_t x_ = T[5], y_ = T[7]; T[5] = x_ + y_; T[7] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[3]; T[1] = x_ + y_; T[3] = x_ - y_; }
    { const int32_t x_ = T[12], y_ = T[14]; T[12] = x_ + y_; T[14] = x_ - y_; }
    { const int32_t x_ = T[8], y_ = T[10]; T[8] = x_ + y_; T[10] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[6]; T[4] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[2]; T[0] = x_ + y_; T[2] = x_ - y_; }
    { const int32_t x_ = rnd12(T[15] * 3784 - T[14] * 1567), y_ = rnd12(T[15] * 1567 + T[14] * 3784); T[15] = y_; T[14] = x_; }
    { const int32_t x_ = rnd12(T[7] * 3784 - T[6] * 1567), y_ = rnd12(T[7] * 1567 + T[6] * 3784); T[7] = y_; T[6] = x_; }
    { const int32_t x_ = rnd12(T[12] * 1567 - T[13] * 3784), y_ = rnd12(T[12] * 3784 + T[13] * 1567); T[12] = y_; T[13] = x_; }
    { const int32_t x_ = rnd12(T[4] * 1567 - T[5] * 3784), y_ = rnd12(T[4] * 3784 + T[5] * 1567); T[4] = y_; T[5] = x_; }
    { const int32_t x_ = T[11], y_ = T[15]; T[11] = x_ + y_; T[15] = x_ - y_; }
    { const int32_t x_ = T[3], y_ = T[7]; T[3] = x_ + y_; T[7] = x_ - y_; }
    { const int32_t x_ = T[10], y_ = T[14]; T[10] = x_ + y_; T[14] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[6]; T[2] = x_ + y_; T[6] = x_ - y_; }
    { const int32_t x_ = T[9], y_ = T[13]; T[9] = x_ + y_; T[13] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[5]; T[1] = x_ + y_; T[5] = x_ - y_; }
    { const int32_t x_ = T[8], y_ = T[12]; T[8] = x_ + y_; T[12] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[4]; T[0] = x_ + y_; T[4] = x_ - y_; }
    { const int32_t x_ = rnd12(T[15] * 2276 - T[14] * 3406), y_ = rnd12(T[15] * 3406 + T[14] * 2276); T[15] = y_; T[14] = x_; }
    { const int32_t x_ = rnd12(T[10] * 3406 - T[11] * 2276), y_ = rnd12(T[10] * 2276 + T[11] * 3406); T[10] = y_; T[11] = x_; }
    { const int32_t x_ = rnd12(T[13] * 4017 - T[12] * 799), y_ = rnd12(T[13] * 799 + T[12] * 4017); T[13] = y_; T[12] = x_; }
    { const int32_t x_ = rnd12(T[8] * 799 - T[9] * 4017), y_ = rnd12(T[8] * 4017 + T[9] * 799); T[8] = y_; T[9] = x_; }
    { const int32_t x_ = T[7], y_ = T[15]; T[7] = x_ + y_; T[15] = x_ - y_; }
    { const int32_t x_ = T[6], y_ = T[14]; T[6] = x_ + y_; T[14] = x_ - y_; }
    { const int32_t x_ = T[5], y_ = T[13]; T[5] = x_ + y_; T[13] = x_ - y_; }
    { const int32_t x_ = T[4], y_ = T[12]; T[4] = x_ + y_; T[12] = x_ - y_; }
    { const int32_t x_ = T[3], y_ = T[11]; T[3] = x_ + y_; T[11] = x_ - y_; }
    { const int32_t x_ = T[2], y_ = T[10]; T[2] = x_ + y_; T[10] = x_ - y_; }
    { const int32_t x_ = T[1], y_ = T[9]; T[1] = x_ + y_; T[9] = x_ - y_; }
    { const int32_t x_ = T[0], y_ = T[8]; T[0] = x_ + y_; T[8] = x_ - y_; }
    { const int32_t x_ = rnd12(T[14] * 4052 - T[15] * 601), y_ = rnd12(T[14] * 601 + T[15] * 4052); T[14] = y_; T[15] = x_; }
    { const int32_t x_ = rnd12(T[12] * 3857 - T[13] * 1380), y_ = rnd12(T[12] * 1380 + T[13] * 3857); T[12] = y_; T[13] = x_; }
    { const int32_t x_ = rnd12(T[10] * 3513 - T[11] * 2106), y_ = rnd12(T[10] * 2106 + T[11] * 3513); T[10] = y_; T[11] = x_; }
    { const int32_t x_ = rnd12(T[8] * 3035 - T[9] * 2751), y_ = rnd12(T[8] * 2751 + T[9] * 3035); T[8] = y_; T[9] = x_; }
    { const int32_t x_ = rnd12(T[6] * 2440 - T[7] * 3290), y_ = rnd12(T[6] * 3290 + T[7] * 2440); T[6] = y_; T[7] = x_; }
    { const int32_t x_ = rnd12(T[4] * 1751 - T[5] * 3703), y_ = rnd12(T[4] * 3703 + T[5] * 1751); T[4] = y_; T[5] = x_; }
    { const int32_t x_ = rnd12(T[2] * 995 - T[3] * 3973), y_ = rnd12(T[2] * 3973 + T[3] * 995); T[2] = y_; T[3] = x_; }
    { const int32_t x_ = rnd12(T[0] * 201 - T[1] * 4091), y_ = rnd12(T[0] * 4091 + T[1] * 201); T[0] = y_; T[1] = x_; }
    {
        int32_t c_[16];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7]; c_[8] = T[8]; c_[9] = T[9]; c_[10] = T[10]; c_[11] = T[11]; c_[12] = T[12]; c_[13] = T[13]; c_[14] = T[14]; c_[15] = T[15];
        T[15] = c_[0];
        T[0] = c_[1];
        T[13] = c_[2];
        T[2] = c_[3];
        T[11] = c_[4];
        T[4] = c_[5];
        T[9] = c_[6];
        T[6] = c_[7];
        T[7] = c_[8];
        T[8] = c_[9];
        T[5] = c_[10];
        T[10] = c_[11];
        T[3] = c_[12];
        T[12] = c_[13];
        T[1] = c_[14];
        T[14] = c_[15];
    }
}
__host__ __device__ __forceinline__ uint32_t inv_adst16(int32_t *T, int r) {
    uint32_t e_ = 0;
    const int32_t lo_ = -(1 << (r - 1)), hi_ = (1 << (r - 1)) - 1;
    {
        int32_t c_[16];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7]; c_[8] = T[8]; c_[9] = T[9]; c_[10] = T[10]; c_[11] = T[11]; c_[12] = T[12]; c_[13] = T[13]; c_[14] = T[14]; c_[15] = T[15];
        T[0] = c_[15];
        T[1] = c_[0];
        T[2] = c_[13];
        T[3] = c_[2];
        T[4] = c_[11];
        T[5] = c_[4];
        T[6] = c_[9];
        T[7] = c_[6];
        T[8] = c_[7];
        T[9] = c_[8];
        T[10] = c_[5];
        T[11] = c_[10];
        T[12] = c_[3];
        T[13] = c_[12];
        T[14] = c_[1];
        T[15] = c_[14];
    }
    { const int32_t x_ = rnd12(T[0] * 201 - T[1] * 4091), y_ = rnd12(T[0] * 4091 + T[1] * 201); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[1] = x_; T[0] = y_; }
    { const int32_t x_ = rnd12(T[2] * 995 - T[3] * 3973), y_ = rnd12(T[2] * 3973 + T[3] * 995); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[3] = x_; T[2] = y_; }
    { const int32_t x_ = rnd12(T[4] * 1751 - T[5] * 3703), y_ = rnd12(T[4] * 3703 + T[5] * 1751); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[4] = y_; }
    { const int32_t x_ = rnd12(T[6] * 2440 - T[7] * 3290), y_ = rnd12(T[6] * 3290 + T[7] * 2440); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[7] = x_; T[6] = y_; }
    { const int32_t x_ = rnd12(T[8] * 3035 - T[9] * 2751), y_ = rnd12(T[8] * 2751 + T[9] * 3035); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[9] = x_; T[8] = y_; }
    { const int32_t x_ = rnd12(T[10] * 3513 - T[11] * 2106), y_ = rnd12(T[10] * 2106 + T[11] * 3513); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[11] = x_; T[10] = y_; }
    { const int32_t x_ = rnd12(T[12] * 3857 - T[13] * 1380), y_ = rnd12(T[12] * 1380 + T[13] * 3857); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[13] = x_; T[12] = y_; }
    { const int32_t x_ = rnd12(T[14] * 4052 - T[15] * 601), y_ = rnd12(T[14] * 601 + T[15] * 4052); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[15] = x_; T[14] = y_; }
    { const int32_t x_ = T[0], y_ = T[8]; T[0] = clampr(x_ + y_, lo_, hi_); T[8] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[9]; T[1] = clampr(x_ + y_, lo_, hi_); T[9] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[10]; T[2] = clampr(x_ + y_, lo_, hi_); T[10] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[11]; T[3] = clampr(x_ + y_, lo_, hi_); T[11] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[4], y_ = T[12]; T[4] = clampr(x_ + y_, lo_, hi_); T[12] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[5], y_ = T[13]; T[5] = clampr(x_ + y_, lo_, hi_); T[13] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[6], y_ = T[14]; T[6] = clampr(x_ + y_, lo_, hi_); T[14] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[7], y_ = T[15]; T[7] = clampr(x_ + y_, lo_, hi_); T[15] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[8] * 799 - T[9] * 4017), y_ = rnd12(T[8] * 4017 + T[9] * 799); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[9] = x_; T[8] = y_; }
    { const int32_t x_ = rnd12(T[13] * 4017 - T[12] * 799), y_ = rnd12(T[13] * 799 + T[12] * 4017); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[12] = x_; T[13] = y_; }
    { const int32_t x_ = rnd12(T[10] * 3406 - T[11] * 2276), y_ = rnd12(T[10] * 2276 + T[11] * 3406); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[11] = x_; T[10] = y_; }
    { const int32_t x_ = rnd12(T[15] * 2276 - T[14] * 3406), y_ = rnd12(T[15] * 3406 + T[14] * 2276); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[14] = x_; T[15] = y_; }
    { const int32_t x_ = T[0], y_ = T[4]; T[0] = clampr(x_ + y_, lo_, hi_); T[4] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[8], y_ = T[12]; T[8] = clampr(x_ + y_, lo_, hi_); T[12] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[5]; T[1] = clampr(x_ + y_, lo_, hi_); T[5] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[9], y_ = T[13]; T[9] = clampr(x_ + y_, lo_, hi_); T[13] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[2], y_ = T[6]; T[2] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[10], y_ = T[14]; T[10] = clampr(x_ + y_, lo_, hi_); T[14] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[3], y_ = T[7]; T[3] = clampr(x_ + y_, lo_, hi_); T[7] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[11], y_ = T[15]; T[11] = clampr(x_ + y_, lo_, hi_); T[15] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[4] * 1567 - T[5] * 3784), y_ = rnd12(T[4] * 3784 + T[5] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[5] = x_; T[4] = y_; }
    { const int32_t x_ = rnd12(T[12] * 1567 - T[13] * 3784), y_ = rnd12(T[12] * 3784 + T[13] * 1567); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[13] = x_; T[12] = y_; }
    { const int32_t x_ = rnd12(T[7] * 3784 - T[6] * 1567), y_ = rnd12(T[7] * 1567 + T[6] * 3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[6] = x_; T[7] = y_; }
    { const int32_t x_ = rnd12(T[15] * 3784 - T[14] * 1567), y_ = rnd12(T[15] * 1567 + T[14] * 3784); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[14] = x_; T[15] = y_; }
    { const int32_t x_ = T[0], y_ = T[2]; T[0] = clampr(x_ + y_, lo_, hi_); T[2] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[4], y_ = T[6]; T[4] = clampr(x_ + y_, lo_, hi_); T[6] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[8], y_ = T[10]; T[8] = clampr(x_ + y_, lo_, hi_); T[10] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[12], y_ = T[14]; T[12] = clampr(x_ + y_, lo_, hi_); T[14] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[1], y_ = T[3]; T[1] = clampr(x_ + y_, lo_, hi_); T[3] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[5], y_ = T[7]; T[5] = clampr(x_ + y_, lo_, hi_); T[7] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[9], y_ = T[11]; T[9] = clampr(x_ + y_, lo_, hi_); T[11] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = T[13], y_ = T[15]; T[13] = clampr(x_ + y_, lo_, hi_); T[15] = clampr(x_ - y_, lo_, hi_); }
    { const int32_t x_ = rnd12(T[2] * 2896 - T[3] * 2896), y_ = rnd12(T[2] * 2896 + T[3] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[3] = x_; T[2] = y_; }
    { const int32_t x_ = rnd12(T[6] * 2896 - T[7] * 2896), y_ = rnd12(T[6] * 2896 + T[7] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[7] = x_; T[6] = y_; }
    { const int32_t x_ = rnd12(T[10] * 2896 - T[11] * 2896), y_ = rnd12(T[10] * 2896 + T[11] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[11] = x_; T[10] = y_; }
    { const int32_t x_ = rnd12(T[14] * 2896 - T[15] * 2896), y_ = rnd12(T[14] * 2896 + T[15] * 2896); e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); T[15] = x_; T[14] = y_; }
    {
        int32_t c_[16];
        c_[0] = T[0]; c_[1] = T[1]; c_[2] = T[2]; c_[3] = T[3]; c_[4] = T[4]; c_[5] = T[5]; c_[6] = T[6]; c_[7] = T[7]; c_[8] = T[8]; c_[9] = T[9]; c_[10] = T[10]; c_[11] = T[11]; c_[12] = T[12]; c_[13] = T[13]; c_[14] = T[14]; c_[15] = T[15];
        T[0] = c_[0];
        T[1] = -c_[8];
        T[2] = c_[12];
        T[3] = -c_[4];
        T[4] = c_[6];
        T[5] = -c_[14];
        T[6] = c_[10];
        T[7] = -c_[2];
        T[8] = c_[3];
        T[9] = -c_[11];
        T[10] = c_[15];
        T[11] = -c_[7];
        T[12] = c_[5];
        T[13] = -c_[13];
        T[14] = c_[9];
        T[15] = -c_[1];
    }
    return e_;
}
__host__ __device__ __forceinline__ void fwd_adst4(int32_t *T) {
    const int32_t x0 = T[0], x1 = T[1], x2 = T[2], x3 = T[3];
    T[0] = rnd12(x0 * 1321 + x1 * 2482 + x2 * 3344 + x3 * 3803);
    T[1] = rnd12(x0 * 3344 + x1 * 3344 + x3 * -3344);
    T[2] = rnd12(x0 * 3803 + x1 * -1321 + x2 * -3344 + x3 * 2482);
    T[3] = rnd12(x0 * 2482 + x1 * -3803 + x2 * 3344 + x3 * -1321);
}

