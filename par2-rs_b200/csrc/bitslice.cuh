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

// The 16-word "record" of a coefficient c.  The 16 input planes are split in
// two halves of 8; for each half a 256-row table holds every XOR combination
// of its planes (row n = XOR of the planes whose bit is set in n; T1 follows
// T0, rows of 128 bytes: one word per lane).  Output plane j is then
//   T0[n0_j] ^ T1[n1_j],  n0_j = sum_{b<8} bit_j(c x^b) << b,
//                         n1_j = sum_{b<8} bit_j(c x^{b+8}) << b.
// The rows are fetched four at a time with ldmatrix.x4 (matrix m's eight
// 16-byte row pointers come from lanes 8m..8m+7, so lane L receives word L of
// each of the four rows).  For plane pair p (planes 2p, 2p+1) the four rows are
//   m = 0: T0[n0_2p]   m = 1: T1[n1_2p]   m = 2: T0[n0_2p+1]   m = 3: T1[n1_2p+1]
// and word 4m + i of the record holds the byte offsets of matrix m's rows for
// p = 2i (low half) and p = 2i+1 (high half), so lane L reads the 16 bytes at
// word 4*(L/8) and needs no other record data.
__host__ __device__ __forceinline__ uint32_t row_offset(int m, uint32_t n0[16], uint32_t n1[16],
                                                        int p)
{
    const int j = 2 * p + (m >> 1);
    return (m & 1) ? (256u + n1[j]) * kRowBytes : n0[j] * kRowBytes;
}

__host__ __device__ __forceinline__ void make_record(uint32_t c, uint32_t w[16])
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
        for (int i = 0; i < 4; ++i)
            w[4 * m + i] = row_offset(m, n0, n1, 2 * i) | (row_offset(m, n0, n1, 2 * i + 1) << 16);
}

}  // namespace p2g
