#!/usr/bin/env python3
"""Generate straight-line integer 1-D transforms (txfm_gen.cuh) from the AV1 inverse-transform step lists.

The AV1 specification (7.13.2) defines only the INVERSE 1-D transforms, as ordered lists of butterfly steps:
    B(a, b, angle, flip)   rotation of T[a], T[b] by cos128/sin128(angle), Round2(., 12), range-checked
    H(a, b, flip)          T[a] + T[b] / T[a] - T[b] (flip swaps a, b), clamped to r bits
    permutations           bit reversal (DCT), the ADST input/output permutations (with negations)
(the same lists av1core/include/av1g/dsp.h:242-413 walks: av1g_idct, av1g_iadst8/16, av1g_iadst_in/out_perm).

The forward transforms of this project are the exact TRANSPOSES of those networks, run in reverse step order:
    B(a, b, angle, 0)^T = B(a, b, -angle, 0)      B(a, b, angle, 1)^T = B(a, b, angle, 1)   (symmetric)
    H(a, b, flip)^T     = H(a, b, flip)           (both forms are symmetric matrices)
    permutation^T       = the inverse permutation (negations stay on the same entries)
Each rotation keeps the spec's Round2(., 12); the forward network has no clamps (its input range is bounded by the
caller's pre-shift, see fwd_shifts() in is_tables.h).  Because every inverse 1-D transform M satisfies
M^T M = (n / 2) I (rotations are orthogonal, every H stage scales by sqrt 2), M^T is the inverse up to the known
scale n / 2, which the 2-D driver folds into its shifts.  ADST4 (spec 7.13.2.6) is a 4x4 integer matrix over
SINPI_k_9; its transpose is applied directly.

Run: python gen_txfm.py > txfm_gen.cuh   (the build does this when the header is missing or older than this file)
"""
import math
import sys

# Cos128_Lookup (spec 7.13.2.1): round(4096 * cos(i * pi / 128)), i = 0..64
COS128 = [int(math.floor(4096 * math.cos(i * math.pi / 128) + 0.5)) for i in range(65)]
SINPI = (1321, 2482, 3344, 3803)   # SINPI_1_9 .. SINPI_4_9 (spec 7.13.2.6)


def cos128(angle):
    a = angle & 255
    if a <= 64:
        return COS128[a]
    if a <= 128:
        return -COS128[128 - a]
    if a <= 192:
        return -COS128[a - 128]
    return COS128[256 - a]


def sin128(angle):
    return cos128(angle - 64)


def brev(nbits, x):
    t = 0
    for i in range(nbits):
        t |= ((x >> i) & 1) << (nbits - 1 - i)
    return t


def idct_ops(n):
    """Step list of the inverse DCT of 2^n points (spec 7.13.2.3), in execution order."""
    ops = []
    n0 = 1 << n
    ops.append(('P', [brev(n, i) for i in range(n0)], [1] * n0))   # T[i] = sgn[i] * old[src[i]]
    B = lambda a, b, ang, fl: ops.append(('B', a, b, ang, fl))
    H = lambda a, b, fl: ops.append(('H', a, b, fl))
    if n == 6:
        for i in range(16): B(32 + i, 63 - i, 63 - 4 * brev(4, i), 0)
    if n >= 5:
        for i in range(8): B(16 + i, 31 - i, 6 + (brev(3, 7 - i) << 3), 0)
    if n == 6:
        for i in range(16): H(32 + i * 2, 33 + i * 2, i & 1)
    if n >= 4:
        for i in range(4): B(8 + i, 15 - i, 12 + (brev(2, 3 - i) << 4), 0)
    if n >= 5:
        for i in range(8): H(16 + 2 * i, 17 + 2 * i, i & 1)
    if n == 6:
        for i in range(4):
            for j in range(2): B(62 - i * 4 - j, 33 + i * 4 + j, 60 - 16 * brev(2, i) + 64 * j, 1)
    if n >= 3:
        for i in range(2): B(4 + i, 7 - i, 56 - 32 * i, 0)
    if n >= 4:
        for i in range(4): H(8 + 2 * i, 9 + 2 * i, i & 1)
    if n >= 5:
        for i in range(2):
            for j in range(2): B(30 - 4 * i - j, 17 + 4 * i + j, 24 + (j << 6) + ((1 - i) << 5), 1)
    if n == 6:
        for i in range(8):
            for j in range(2): H(32 + i * 4 + j, 35 + i * 4 - j, i & 1)
    for i in range(2): B(2 * i, 2 * i + 1, 32 + 16 * i, 1 - i)
    if n >= 3:
        for i in range(2): H(4 + 2 * i, 5 + 2 * i, i)
    if n >= 4:
        for i in range(2): B(14 - i, 9 + i, 48 + 64 * i, 1)
    if n >= 5:
        for i in range(4):
            for j in range(2): H(16 + 4 * i + j, 19 + 4 * i - j, i & 1)
    if n == 6:
        for i in range(2):
            for j in range(4): B(61 - i * 8 - j, 34 + i * 8 + j, 56 - i * 32 + (j >> 1) * 64, 1)
    for i in range(2): H(i, 3 - i, 0)
    if n >= 3: B(6, 5, 32, 1)
    if n >= 4:
        for i in range(2):
            for j in range(2): H(8 + 4 * i + j, 11 + 4 * i - j, i)
    if n >= 5:
        for i in range(4): B(29 - i, 18 + i, 48 + (i >> 1) * 64, 1)
    if n == 6:
        for i in range(4):
            for j in range(4): H(32 + 8 * i + j, 39 + 8 * i - j, i & 1)
    if n >= 3:
        for i in range(4): H(i, 7 - i, 0)
    if n >= 4:
        for i in range(2): B(13 - i, 10 + i, 32, 1)
    if n >= 5:
        for i in range(2):
            for j in range(4): H(16 + i * 8 + j, 23 + i * 8 - j, i)
    if n == 6:
        for i in range(8): B(59 - i, 36 + i, 48 if i < 4 else 112, 1)
    if n >= 4:
        for i in range(8): H(i, 15 - i, 0)
    if n >= 5:
        for i in range(4): B(27 - i, 20 + i, 32, 1)
    if n == 6:
        for i in range(8):
            H(32 + i, 47 - i, 0)
            H(48 + i, 63 - i, 1)
    if n >= 5:
        for i in range(16): H(i, 31 - i, 0)
    if n == 6:
        for i in range(8): B(55 - i, 40 + i, 32, 1)
    if n == 6:
        for i in range(32): H(i, 63 - i, 0)
    return ops


def adst_in_perm(n):
    n0 = 1 << n
    return ('P', [(i - 1) if (i & 1) else (n0 - i - 1) for i in range(n0)], [1] * n0)


def adst_out_perm(n):
    n0 = 1 << n
    src, sgn = [], []
    for i in range(n0):
        a = (i >> 3) & 1
        b = ((i >> 2) & 1) ^ ((i >> 3) & 1)
        c = ((i >> 1) & 1) ^ ((i >> 2) & 1)
        d = (i & 1) ^ ((i >> 1) & 1)
        src.append(((d << 3) | (c << 2) | (b << 1) | a) >> (4 - n))
        sgn.append(-1 if (i & 1) else 1)
    return ('P', src, sgn)


def iadst8_ops():
    ops = [adst_in_perm(3)]
    for i in range(4): ops.append(('B', 2 * i, 2 * i + 1, 60 - 16 * i, 1))
    for i in range(4): ops.append(('H', i, 4 + i, 0))
    for i in range(2): ops.append(('B', 4 + 3 * i, 5 + i, 48 - 32 * i, 1))
    for i in range(2):
        for j in range(2): ops.append(('H', 4 * j + i, 2 + 4 * j + i, 0))
    for i in range(2): ops.append(('B', 2 + 4 * i, 3 + 4 * i, 32, 1))
    ops.append(adst_out_perm(3))
    return ops


def iadst16_ops():
    ops = [adst_in_perm(4)]
    for i in range(8): ops.append(('B', 2 * i, 2 * i + 1, 62 - 8 * i, 1))
    for i in range(8): ops.append(('H', i, 8 + i, 0))
    for i in range(2):
        ops.append(('B', 8 + 2 * i, 9 + 2 * i, 56 - 32 * i, 1))
        ops.append(('B', 13 + 2 * i, 12 + 2 * i, 8 + 32 * i, 1))
    for i in range(4):
        for j in range(2): ops.append(('H', 8 * j + i, 4 + 8 * j + i, 0))
    for i in range(2):
        for j in range(2): ops.append(('B', 4 + 8 * j + 3 * i, 5 + 8 * j + i, 48 - 32 * i, 1))
    for i in range(2):
        for j in range(4): ops.append(('H', 4 * j + i, 2 + 4 * j + i, 0))
    for i in range(4): ops.append(('B', 2 + 4 * i, 3 + 4 * i, 32, 1))
    ops.append(adst_out_perm(4))
    return ops


def adst4_matrix():
    """S with inverse ADST4 output x[i] = Round2(sum_j S[i][j] T[j], 12) (spec 7.13.2.6 without its Round2)."""
    s1, s2, s3, s4 = SINPI
    return [[s1, s3, s4, s2],
            [s2, s3, -s1, -s4],
            [s3, 0, -s3, s3],
            [s4, -s3, s2, -s1]]


# ------------------------------------------------------------------------------------------------------------------
# code emission
# ------------------------------------------------------------------------------------------------------------------
def emit_perm(out, src, sgn, inverse):
    n0 = len(src)
    out.append('    {')
    out.append('        int32_t c_[%d];' % n0)
    out.append('        ' + ' '.join('c_[%d] = T[%d];' % (i, i) for i in range(n0)))
    if not inverse:   # T[i] = sgn[i] * c[src[i]]
        for i in range(n0):
            out.append('        T[%d] = %sc_[%d];' % (i, '-' if sgn[i] < 0 else '', src[i]))
    else:             # transpose: T[src[i]] = sgn[i] * c[i]
        for i in range(n0):
            out.append('        T[%d] = %sc_[%d];' % (src[i], '-' if sgn[i] < 0 else '', i))
    out.append('    }')


def emit_fwd(name, ops, n0):
    out = ['__host__ __device__ __forceinline__ void %s(int32_t *T) {' % name]
    for op in reversed(ops):
        if op[0] == 'P':
            emit_perm(out, op[1], op[2], inverse=True)
        elif op[0] == 'B':
            _, a, b, ang, fl = op
            if not fl:
                ang = -ang
            c, s = cos128(ang), sin128(ang)
            x = 'rnd12(T[%d] * %d - T[%d] * %d)' % (a, c, b, s)
            y = 'rnd12(T[%d] * %d + T[%d] * %d)' % (a, s, b, c)
            if fl:
                out.append('    { const int32_t x_ = %s, y_ = %s; T[%d] = y_; T[%d] = x_; }' % (x, y, a, b))
            else:
                out.append('    { const int32_t x_ = %s, y_ = %s; T[%d] = x_; T[%d] = y_; }' % (x, y, a, b))
        else:
            _, a, b, fl = op
            if fl:
                a, b = b, a
            out.append('    { const int32_t x_ = T[%d], y_ = T[%d]; T[%d] = x_ + y_; T[%d] = x_ - y_; }' % (a, b, a, b))
    out.append('}')
    return out


def emit_inv(name, ops, n0):
    """Inverse with the spec's checks: B outputs must fit r bits (flag 1), H results are clamped to r bits.

    32-bit arithmetic is exact for every transform that ends with the flag clear: its inputs are within r bits
    (dequantised values are clipped to BitDepth + 8 bits, the column inputs to the column clamp range), so while no
    rotation has left r bits every rotation input is within r bits (H results are clamped; a permutation negation
    adds at most 1) and |T[a] c - T[b] s| + 2048 < 2^(r + 13) <= 2^31 for r <= 18 (bit depth <= 10).  After the
    first out-of-range rotation the flag is set and the caller discards the values."""
    out = ['__host__ __device__ __forceinline__ uint32_t %s(int32_t *T, int r) {' % name,
           '    uint32_t e_ = 0;',
           '    const int32_t lo_ = -(1 << (r - 1)), hi_ = (1 << (r - 1)) - 1;']
    for op in ops:
        if op[0] == 'P':
            emit_perm(out, op[1], op[2], inverse=False)
        elif op[0] == 'B':
            _, a, b, ang, fl = op
            c, s = cos128(ang), sin128(ang)
            x = 'rnd12(T[%d] * %d - T[%d] * %d)' % (a, c, b, s)
            y = 'rnd12(T[%d] * %d + T[%d] * %d)' % (a, s, b, c)
            dst = (b, a) if fl else (a, b)
            out.append('    { const int32_t x_ = %s, y_ = %s; e_ |= (x_ < lo_ || x_ > hi_ || y_ < lo_ || y_ > hi_); '
                       'T[%d] = x_; T[%d] = y_; }' % (x, y, dst[0], dst[1]))
        else:
            _, a, b, fl = op
            if fl:
                a, b = b, a
            out.append('    { const int32_t x_ = T[%d], y_ = T[%d]; T[%d] = clampr(x_ + y_, lo_, hi_); '
                       'T[%d] = clampr(x_ - y_, lo_, hi_); }' % (a, b, a, b))
    out.append('    return e_;')
    out.append('}')
    return out


def main():
    out = ['// GENERATED by gen_txfm.py from the AV1 inverse-transform step lists (spec 7.13.2). DO NOT EDIT.',
           '// fwd_*: transposed networks (forward transforms of this project); inv_*: the spec inverse 1-D transforms',
           '// with their conformance checks (return value: nonzero when a butterfly output left r bits).',
           '#pragma once',
           '#include <stdint.h>',
           '#ifndef __CUDACC__',
           '#define __host__',
           '#define __device__',
           '#define __forceinline__ inline',
           '#endif',
           '__host__ __device__ __forceinline__ int32_t rnd12(int32_t x) { return (x + 2048) >> 12; }',
           '__host__ __device__ __forceinline__ int32_t clampr(int32_t v, int32_t lo, int32_t hi) '
           '{ return v < lo ? lo : (v > hi ? hi : v); }',
           '']
    for n in range(2, 7):
        out += emit_fwd('fwd_dct%d' % (1 << n), idct_ops(n), 1 << n)
        out += emit_inv('inv_dct%d' % (1 << n), idct_ops(n), 1 << n)
    out += emit_fwd('fwd_adst8', iadst8_ops(), 8)
    out += emit_inv('inv_adst8', iadst8_ops(), 8)
    out += emit_fwd('fwd_adst16', iadst16_ops(), 16)
    out += emit_inv('inv_adst16', iadst16_ops(), 16)
    S = adst4_matrix()
    # forward ADST4: y_j = Round2(sum_i S[i][j] x_i, 12)
    out.append('__host__ __device__ __forceinline__ void fwd_adst4(int32_t *T) {')
    out.append('    const int32_t x0 = T[0], x1 = T[1], x2 = T[2], x3 = T[3];')
    for j in range(4):
        terms = ' + '.join('x%d * %d' % (i, S[i][j]) for i in range(4) if S[i][j] != 0)
        out.append('    T[%d] = rnd12(%s);' % (j, terms))
    out.append('}')
    out.append('')
    sys.stdout.write('\n'.join(out) + '\n')


if __name__ == '__main__':
    main()
