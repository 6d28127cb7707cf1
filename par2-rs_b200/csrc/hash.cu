// hash.cu -- per-slice MD5 + CRC32 (the IFSC checksums of a PAR2 set).
//
// Replaces the per-slice hashing of par2-rs: verify_file_blocks
// (verify.rs:548-654: CRC32 first, MD5 when the CRC matches) and the IFSC
// computation of the creator (creator.rs:397-409).  par2-rs takes both from
// crates (md-5 0.10.6, crc32fast 1.5.0); here they are written from their
// definitions:
//   * MD5 from RFC 1321 (four rounds of 16 steps over 64-byte blocks, padding
//     0x80, zeros, 64-bit little-endian bit length);
//   * CRC-32/ISO-HDLC: reflected polynomial 0xEDB88320, initial value and
//     final XOR 0xFFFFFFFF, computed four bytes at a time with four 256-entry
//     tables ("slicing by 4").
//
// One thread owns one slice (MD5 is a serial chain over the slice).  The four
// CRC tables are replicated 32 times in shared memory so that lane L always
// reads bank L: data-dependent table reads never conflict.
#include "hash.cuh"

namespace p2g {

// RFC 1321 section 3.4: T[i] = floor(2^32 * |sin(i + 1)|)
__constant__ uint32_t kMd5T[64] = {
    0xd76aa478, 0xe8c7b756, 0x242070db, 0xc1bdceee, 0xf57c0faf, 0x4787c62a, 0xa8304613,
    0xfd469501, 0x698098d8, 0x8b44f7af, 0xffff5bb1, 0x895cd7be, 0x6b901122, 0xfd987193,
    0xa679438e, 0x49b40821, 0xf61e2562, 0xc040b340, 0x265e5a51, 0xe9b6c7aa, 0xd62f105d,
    0x02441453, 0xd8a1e681, 0xe7d3fbc8, 0x21e1cde6, 0xc33707d6, 0xf4d50d87, 0x455a14ed,
    0xa9e3e905, 0xfcefa3f8, 0x676f02d9, 0x8d2a4c8a, 0xfffa3942, 0x8771f681, 0x6d9d6122,
    0xfde5380c, 0xa4beea44, 0x4bdecfa9, 0xf6bb4b60, 0xbebfbc70, 0x289b7ec6, 0xeaa127fa,
    0xd4ef3085, 0x04881d05, 0xd9d4d039, 0xe6db99e5, 0x1fa27cf8, 0xc4ac5665, 0xf4292244,
    0x432aff97, 0xab9423a7, 0xfc93a039, 0x655b59c3, 0x8f0ccc92, 0xffeff47d, 0x85845dd1,
    0x6fa87e4f, 0xfe2ce6e0, 0xa3014314, 0x4e0811a1, 0xf7537e82, 0xbd3af235, 0x2ad7d2bb,
    0xeb86d391};

__device__ __forceinline__ uint32_t rotl(uint32_t x, int s) { return __funnelshift_l(x, x, s); }

// One RFC 1321 block transform of the 16 little-endian words x.
__device__ __forceinline__ void md5_block(uint32_t st[4], const uint32_t x[16])
{
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3];
#define P2G_STEP(f, a, b, c, d, k, s, i)              \
    {                                                 \
        a = b + rotl(a + (f) + x[k] + kMd5T[i], s);   \
    }
#pragma unroll
    for (int i = 0; i < 16; i += 4) {
        P2G_STEP((b & c) | (~b & d), a, b, c, d, i, 7, i);
        P2G_STEP((a & b) | (~a & c), d, a, b, c, i + 1, 12, i + 1);
        P2G_STEP((d & a) | (~d & b), c, d, a, b, i + 2, 17, i + 2);
        P2G_STEP((c & d) | (~c & a), b, c, d, a, i + 3, 22, i + 3);
    }
#pragma unroll
    for (int i = 16; i < 32; i += 4) {
        P2G_STEP((b & d) | (c & ~d), a, b, c, d, (5 * i + 1) & 15, 5, i);
        P2G_STEP((a & c) | (b & ~c), d, a, b, c, (5 * (i + 1) + 1) & 15, 9, i + 1);
        P2G_STEP((d & b) | (a & ~b), c, d, a, b, (5 * (i + 2) + 1) & 15, 14, i + 2);
        P2G_STEP((c & a) | (d & ~a), b, c, d, a, (5 * (i + 3) + 1) & 15, 20, i + 3);
    }
#pragma unroll
    for (int i = 32; i < 48; i += 4) {
        P2G_STEP(b ^ c ^ d, a, b, c, d, (3 * i + 5) & 15, 4, i);
        P2G_STEP(a ^ b ^ c, d, a, b, c, (3 * (i + 1) + 5) & 15, 11, i + 1);
        P2G_STEP(d ^ a ^ b, c, d, a, b, (3 * (i + 2) + 5) & 15, 16, i + 2);
        P2G_STEP(c ^ d ^ a, b, c, d, a, (3 * (i + 3) + 5) & 15, 23, i + 3);
    }
#pragma unroll
    for (int i = 48; i < 64; i += 4) {
        P2G_STEP(c ^ (b | ~d), a, b, c, d, (7 * i) & 15, 6, i);
        P2G_STEP(b ^ (a | ~c), d, a, b, c, (7 * (i + 1)) & 15, 10, i + 1);
        P2G_STEP(a ^ (d | ~b), c, d, a, b, (7 * (i + 2)) & 15, 15, i + 2);
        P2G_STEP(d ^ (c | ~a), b, c, d, a, (7 * (i + 3)) & 15, 21, i + 3);
    }
#undef P2G_STEP
    st[0] += a;
    st[1] += b;
    st[2] += c;
    st[3] += d;
}

constexpr int kHashThreads = 256;
constexpr int kCrcTabWords = 4 * 256 * 32;  // 4 tables x 256 entries x 32 bank copies

// table t, entry e, for this lane
__device__ __forceinline__ uint32_t crc_tab(const uint32_t *stab, int t, uint32_t e, int lane)
{
    return stab[((t << 8) + e) * 32 + lane];
}

__device__ __forceinline__ uint32_t crc_word(const uint32_t *stab, uint32_t crc, uint32_t w, int lane)
{
    crc ^= w;
    return crc_tab(stab, 3, crc & 0xFF, lane) ^ crc_tab(stab, 2, (crc >> 8) & 0xFF, lane) ^
           crc_tab(stab, 1, (crc >> 16) & 0xFF, lane) ^ crc_tab(stab, 0, crc >> 24, lane);
}

__device__ __forceinline__ uint32_t crc_byte(const uint32_t *stab, uint32_t crc, uint32_t b, int lane)
{
    return crc_tab(stab, 0, (crc ^ b) & 0xFF, lane) ^ (crc >> 8);
}

__global__ void __launch_bounds__(kHashThreads, 1)
    hash_slices_kernel(const uint8_t *const *__restrict__ slices, int n, size_t S,
                       const uint32_t *__restrict__ crc_tables, uint8_t *__restrict__ md5_out,
                       uint32_t *__restrict__ crc_out)
{
    extern __shared__ uint32_t stab[];
    for (int idx = threadIdx.x; idx < kCrcTabWords; idx += blockDim.x)
        stab[idx] = crc_tables[idx >> 5];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int lane = threadIdx.x & 31;
    const uint8_t *p = slices[i];
    uint32_t st[4] = {0x67452301u, 0xefcdab89u, 0x98badcfeu, 0x10325476u};
    uint32_t crc = 0xFFFFFFFFu;
    const size_t full = S / 64;
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
    for (size_t blk = 0; blk < full; ++blk) {
        uint32_t x[16];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            uint4 u = __ldg(q + blk * 4 + v);
            x[4 * v] = u.x;
            x[4 * v + 1] = u.y;
            x[4 * v + 2] = u.z;
            x[4 * v + 3] = u.w;
        }
#pragma unroll
        for (int j = 0; j < 16; ++j)
            crc = crc_word(stab, crc, x[j], lane);
        md5_block(st, x);
    }
    // tail: remaining bytes, 0x80, zeros, 64-bit bit length (RFC 1321 3.1-3.2)
    const size_t rem = S - full * 64;
    const uint8_t *t = p + full * 64;
    uint32_t x[16];
#pragma unroll
    for (int j = 0; j < 16; ++j)
        x[j] = 0;
    for (size_t b = 0; b < rem; ++b) {
        uint32_t v = t[b];
        crc = crc_byte(stab, crc, v, lane);
        x[b >> 2] |= v << (8 * (b & 3));
    }
    x[rem >> 2] |= 0x80u << (8 * (rem & 3));
    const uint64_t bits = static_cast<uint64_t>(S) * 8;
    if (rem >= 56) {
        md5_block(st, x);
#pragma unroll
        for (int j = 0; j < 16; ++j)
            x[j] = 0;
    }
    x[14] = static_cast<uint32_t>(bits);
    x[15] = static_cast<uint32_t>(bits >> 32);
    md5_block(st, x);
    uint4 *o = reinterpret_cast<uint4 *>(md5_out + static_cast<size_t>(i) * 16);
    *o = make_uint4(st[0], st[1], st[2], st[3]);
    crc_out[i] = crc ^ 0xFFFFFFFFu;
}

void crc32_tables(uint32_t tab[4][256])
{
    for (uint32_t b = 0; b < 256; ++b) {
        uint32_t c = b;
        for (int k = 0; k < 8; ++k)
            c = (c & 1) ? (c >> 1) ^ 0xEDB88320u : c >> 1;
        tab[0][b] = c;
    }
    for (int t = 1; t < 4; ++t)
        for (uint32_t b = 0; b < 256; ++b)
            tab[t][b] = (tab[t - 1][b] >> 8) ^ tab[0][tab[t - 1][b] & 0xFF];
}

size_t hash_smem_bytes() { return kCrcTabWords * sizeof(uint32_t); }

int hash_run(p2g_ctx *ctx, const uint8_t *const *d_slices, int n, size_t S, uint8_t *d_md5,
             uint32_t *d_crc)
{
    if (n <= 0)
        return P2G_OK;
    const size_t smem = hash_smem_bytes();
    P2G_CUDA(cudaFuncSetAttribute(hash_slices_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    const int grid = (n + kHashThreads - 1) / kHashThreads;
    hash_slices_kernel<<<grid, kHashThreads, smem, ctx->stream>>>(d_slices, n, S, ctx->d_crc,
                                                                  d_md5, d_crc);
    P2G_CUDA(cudaGetLastError());
    ++ctx->launches;
    return P2G_OK;
}

}  // namespace p2g
