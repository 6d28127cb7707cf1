// bitslice.cuh -- bit-sliced ("plane") representation of GF(2^16) symbols.
//
// A group of 32 symbols is held as 16 32-bit plane words: plane b holds bit b
// of every symbol.  Multiplication by a constant c is then GF(2)-linear on the
// planes: out_plane[j] = XOR_b M_c[j][b] * in_plane[b], with column b of M_c
// equal to c * x^b in GF(2^16) (poly 0x1100B, par2-rs galois/core.rs:12).
//
// Bit p of a plane word belongs to symbol sigma(p) of the group: even symbols
// (2p) in bits 0..15 and odd symbols (2(p-16)+1) in bits 16..31.  That is the
// order a 32-bit load of two little-endian u16 symbols gives for free.
#pragma once
#include <stdint.h>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace p2g {

constexpr uint32_t kPoly = 0x1100Bu;

// Transposes two 16x16 bit matrices packed side by side in 16 words (low
// halves: matrix A, high halves: matrix B): afterwards bit j of half h of
// x[b] is what bit b of half h of x[j] was.  Four butterfly stages of
// block-swaps (the classic recursive transpose); the operation is its own
// inverse, so it converts 32 symbols <-> 16 planes in both directions.
__host__ __device__ __forceinline__ void transpose16x2(uint32_t x[16])
{
#define P2G_SWAP(j, h, m)                                   \
    {                                                       \
        uint32_t t_ = ((x[j] >> (h)) ^ x[(j) + (h)]) & (m); \
        x[(j) + (h)] ^= t_;                                 \
        x[j] ^= t_ << (h);                                  \
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
        P2G_SWAP(j, 8, 0x00FF00FFu);
#pragma unroll
    for (int j0 = 0; j0 < 16; j0 += 8)
#pragma unroll
        for (int j = j0; j < j0 + 4; ++j)
            P2G_SWAP(j, 4, 0x0F0F0F0Fu);
#pragma unroll
    for (int j0 = 0; j0 < 16; j0 += 4)
#pragma unroll
        for (int j = j0; j < j0 + 2; ++j)
            P2G_SWAP(j, 2, 0x33333333u);
#pragma unroll
    for (int j0 = 0; j0 < 16; j0 += 2)
        P2G_SWAP(j0, 1, 0x55555555u);
#undef P2G_SWAP
}

// c * x in GF(2^16) (one doubling step of galois/core.rs:58-63).
__host__ __device__ __forceinline__ uint32_t gf_times_x(uint32_t v)
{
    v <<= 1;
    return (v & 0x10000u) ? (v ^ kPoly) : v;
}

// Row stride of a lookup table in shared memory: one 32-bit word per lane.
constexpr uint32_t kRowBytes = 128;

// The 8-word "record" of a coefficient c.  The 16 input planes are split in
// two halves of 8; for each half a 256-row table holds every XOR combination
// of its planes (row n = XOR of the planes whose bit is set in n; rows of 128
// bytes: one word per lane).  Output plane j is then
//   T0[n0_j] ^ T1[n1_j],  n0_j = sum_{b<8} bit_j(c x^b) << b,
//                         n1_j = sum_{b<8} bit_j(c x^{b+8}) << b.
// The rows are fetched four at a time with ldmatrix.x4 (matrix m's eight
// 16-byte row pointers come from lanes 8m..8m+7).  For plane pair p (planes
// 2p, 2p+1) the four rows are
//   class 0: T0[n0_2p]   class 1: T1[n1_2p]   class 2: T0[n0_2p+1]   class 3: T1[n1_2p+1]
// and byte p of record words 2m, 2m + 1 (little-endian, 8 bytes) holds the
// row index of class m for plane pair p, so a lane reads the 8 bytes of its
// class and needs no other record data.  Odd classes index T1, even T0: the
// reader folds the table into its lane's base address.
__host__ __device__ __forceinline__ uint32_t row_index(int m, const uint32_t n0[16],
                                                       const uint32_t n1[16], int p)
{
    const int j = 2 * p + (m >> 1);
    return (m & 1) ? n1[j] : n0[j];
}

__host__ __device__ __forceinline__ void make_record(uint32_t c, uint32_t w[8])
{
    uint32_t col[16];
    uint32_t v = c & 0xFFFFu;
#pragma unroll
    for (int b = 0; b < 16; ++b) {
        col[b] = v;
        v = gf_times_x(v);
    }
    uint32_t n0[16], n1[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        uint32_t a = 0, b1 = 0;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            a |= ((col[b] >> j) & 1u) << b;
            b1 |= ((col[b + 8] >> j) & 1u) << b;
        }
        n0[j] = a;
        n1[j] = b1;
    }
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            uint32_t x = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                x |= row_index(m, n0, n1, 4 * h + q) << (8 * q);
            w[2 * m + h] = x;
        }
}

// Words per record of the two table forms.
constexpr int kRecordWords = 8;
constexpr int kRecordWordsSmall = 24;

// The small-output form (6 + 5 + 5 planes): three tables of 64, 32 and 32
// rows over planes 0-5, 6-10 and 11-15 (T1 from row 64, T2 from row 96), 16
// KiB per input instead of 64, built with 128 row stores instead of 512 --
// cheaper when few outputs share an input's tables, at 48 row reads per
// coefficient instead of 32.  Output plane j is
//   T0[a_j] ^ T1[b_j] ^ T2[c_j],  a_j = sum_{b<6} bit_j(c x^b) << b,
//   b_j = sum_{b<5} bit_j(c x^{6+b}) << b,  c_j = sum_{b<5} bit_j(c x^{11+b}) << b.
// The 48 rows form the sequence s = 3j + t (t = 0, 1, 2 for T0, T1, T2),
// fetched four at a time: ldmatrix k reads s = 4k..4k+3, lane group m
// (lanes 8m..8m+7) pointing at row 4k + m.  Words 6m..6m+5 of the 24-word
// record hold lane group m's twelve byte offsets: k = 2i in the low half of
// word 6m + i, k = 2i + 1 in the high half.
__host__ __device__ __forceinline__ void make_record_small(uint32_t c, uint32_t w[24])
{
    uint32_t col[16];
    uint32_t v = c & 0xFFFFu;
#pragma unroll
    for (int b = 0; b < 16; ++b) {
        col[b] = v;
        v = gf_times_x(v);
    }
    uint32_t off[48];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        uint32_t a = 0, b1 = 0, c1 = 0;
#pragma unroll
        for (int b = 0; b < 6; ++b)
            a |= ((col[b] >> j) & 1u) << b;
#pragma unroll
        for (int b = 0; b < 5; ++b) {
            b1 |= ((col[6 + b] >> j) & 1u) << b;
            c1 |= ((col[11 + b] >> j) & 1u) << b;
        }
        off[3 * j] = a * kRowBytes;
        off[3 * j + 1] = (64u + b1) * kRowBytes;
        off[3 * j + 2] = (96u + c1) * kRowBytes;
    }
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int i = 0; i < 6; ++i)
            w[6 * m + i] = off[8 * i + m] | (off[8 * i + 4 + m] << 16);
}

#ifdef __CUDACC__
// Writes record idx of coefficient c in the small (24-word) or the 8 + 8
// (8-word) form; records are 16-byte aligned in both.
__device__ __forceinline__ void write_record(uint32_t *recs, size_t idx, uint32_t c, bool small)
{
    if (small) {
        uint32_t w[kRecordWordsSmall];
        make_record_small(c, w);
        uint4 *R = reinterpret_cast<uint4 *>(recs + idx * kRecordWordsSmall);
#pragma unroll
        for (int q = 0; q < kRecordWordsSmall / 4; ++q)
            R[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
        return;
    }
    uint32_t w[kRecordWords];
    make_record(c, w);
    uint4 *R = reinterpret_cast<uint4 *>(recs + idx * kRecordWords);
#pragma unroll
    for (int q = 0; q < kRecordWords / 4; ++q)
        R[q] = make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
}
#endif

}  // namespace p2g
