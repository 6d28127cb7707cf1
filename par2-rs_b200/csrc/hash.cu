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
// One lane owns one slice (MD5 is a serial chain over the slice) and computes
// both checksums from the same registers.  The 32 slices of a warp stream
// through a 3-stage shared-memory ring filled by cp.async: eight lanes copy
// 128 contiguous bytes of one slice (coalesced), the 16-byte units of each
// slice row are XOR-swizzled by the slice index so that the lanes' 16-byte
// reads of their own rows never conflict, and the copy of chunk c+2 is in
// flight while chunk c is hashed.  The four CRC tables are replicated 32 times
// in shared memory so that lane L always reads bank L: data-dependent table
// reads never conflict.
#include <algorithm>

#include "async.cuh"
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
constexpr int kHashWarps = kHashThreads / 32;
constexpr int kCrcTabWords = 4 * 256 * 32;  // 4 tables x 256 entries x 32 bank copies
constexpr int kChunk = 128;                 // bytes of every slice per ring stage
constexpr int kStages = 3;
constexpr int kStageBytes = 32 * kChunk;    // one warp's 32 slices
constexpr size_t kHashSmem =
    static_cast<size_t>(kCrcTabWords) * 4 + static_cast<size_t>(kHashWarps) * kStages * kStageBytes;

// CRC table layout in shared memory: tables 2p and 2p+1 share a 64 KiB
// region p, whose row e (256 bytes) holds entry e of table 2p in its first
// 128 bytes and of table 2p+1 in its second, 32 copies each -- copy L for
// lane L, so every lane reads its own bank.  The byte offset of (table T,
// entry e, lane L) is then base_T(L) with e placed in its byte 1, one PRMT.
__device__ __forceinline__ uint32_t crc_base(int T, int lane)
{
    return static_cast<uint32_t>((T >> 1) << 16 | (T & 1) << 7 | lane << 2);
}
__device__ __forceinline__ uint32_t crc_at(const uint32_t *stab, uint32_t off)
{
    return *reinterpret_cast<const uint32_t *>(reinterpret_cast<const uint8_t *>(stab) + off);
}

struct CrcLanes {
    uint32_t b0, b1, b2, b3;  // crc_base(T, lane) for T = 0..3
};

// slicing by 4: crc' = T3[t.b0] ^ T2[t.b1] ^ T1[t.b2] ^ T0[t.b3], t = crc ^ w
__device__ __forceinline__ uint32_t crc_word(const uint32_t *stab, uint32_t crc, uint32_t w,
                                             const CrcLanes &L)
{
    const uint32_t t = crc ^ w;
    return crc_at(stab, __byte_perm(t, L.b3, 0x7604)) ^ crc_at(stab, __byte_perm(t, L.b2, 0x7614)) ^
           crc_at(stab, __byte_perm(t, L.b1, 0x7624)) ^ crc_at(stab, __byte_perm(t, L.b0, 0x7634));
}

__device__ __forceinline__ uint32_t crc_byte(const uint32_t *stab, uint32_t crc, uint32_t b,
                                             const CrcLanes &L)
{
    return crc_at(stab, __byte_perm(crc ^ b, L.b0, 0x7604)) ^ (crc >> 8);
}

// byte offset of 16-byte unit u of slice row s inside a stage
__device__ __forceinline__ int stage_pos(int s, int u) { return s * kChunk + ((u ^ (s & 7)) << 4); }

// Copies bytes [off, off + kChunk) of the warp's slices into a stage: lane L
// moves unit L % 8 of slices L / 8, 4 + L / 8, ... (null pointer: no slice).
__device__ __forceinline__ void stage_chunk(uint8_t *stage, const uint8_t *const ptr[8], size_t off,
                                            int lane)
{
    const int u = lane & 7;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int s = 4 * i + (lane >> 3);
        if (ptr[i])
            cp_async16(stage + stage_pos(s, u), ptr[i] + off + u * 16);
    }
}

__device__ __forceinline__ void hash_block(const uint32_t *stab, uint32_t st[4], uint32_t &crc,
                                           const uint32_t x[16], const CrcLanes &L)
{
#pragma unroll
    for (int j = 0; j < 16; ++j)
        crc = crc_word(stab, crc, x[j], L);
    md5_block(st, x);
}

__global__ void __launch_bounds__(kHashThreads, 1)
    hash_slices_kernel(const uint8_t *const *__restrict__ slices, int n, int per_cta, size_t S,
                       const uint32_t *__restrict__ crc_tables, uint8_t *__restrict__ md5_out,
                       uint32_t *__restrict__ crc_out)
{
    extern __shared__ __align__(16) uint32_t stab[];
    for (int idx = threadIdx.x; idx < kCrcTabWords; idx += blockDim.x) {
        const int L = idx & 31, e = (idx >> 5) & 255, T = idx >> 13;
        stab[(crc_base(T, L) | e << 8) >> 2] = crc_tables[T * 256 + e];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    // this CTA hashes slices [blockIdx * per_cta, end), 32 to a warp
    const int first = blockIdx.x * per_cta + warp * 32;
    const int end = min(n, (blockIdx.x + 1) * per_cta);
    if (first >= end)
        return;
    const CrcLanes CL{crc_base(0, lane), crc_base(1, lane), crc_base(2, lane), crc_base(3, lane)};
    uint8_t *ring = reinterpret_cast<uint8_t *>(stab + kCrcTabWords) +
                    static_cast<size_t>(warp) * kStages * kStageBytes;
    const uint8_t *ptr[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int g = first + 4 * i + (lane >> 3);
        ptr[i] = g < end ? slices[g] : nullptr;
    }
    const int me = first + lane;
    const bool active = me < end;
    uint32_t st[4] = {0x67452301u, 0xefcdab89u, 0x98badcfeu, 0x10325476u};
    uint32_t crc = 0xFFFFFFFFu;
    const size_t nch = S / kChunk;
#pragma unroll
    for (int c = 0; c < kStages - 1; ++c) {
        if (static_cast<size_t>(c) < nch)
            stage_chunk(ring + c * kStageBytes, ptr, static_cast<size_t>(c) * kChunk, lane);
        cp_async_commit();
    }
    int cur = 0;
    for (size_t c = 0; c < nch; ++c) {
        cp_async_wait<kStages - 2>();  // this lane's copies of chunk c have landed
        __syncwarp();                  // ... and every other lane's; chunk c-1 is consumed
        const size_t pre = c + kStages - 1;
        const int pst = cur == 0 ? kStages - 1 : cur - 1;
        if (pre < nch)
            stage_chunk(ring + pst * kStageBytes, ptr, pre * kChunk, lane);
        cp_async_commit();
        if (active) {
            const uint8_t *row = ring + cur * kStageBytes;
#pragma unroll
            for (int b = 0; b < kChunk / 64; ++b) {
                uint32_t x[16];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    const uint4 q = *reinterpret_cast<const uint4 *>(row + stage_pos(lane, 4 * b + v));
                    x[4 * v] = q.x;
                    x[4 * v + 1] = q.y;
                    x[4 * v + 2] = q.z;
                    x[4 * v + 3] = q.w;
                }
                hash_block(stab, st, crc, x, CL);
            }
        }
        cur = cur == kStages - 1 ? 0 : cur + 1;
    }
    cp_async_wait<0>();
    if (!active)
        return;
    // the last S % 128 bytes: one more full 64-byte block if there is one,
    // then the remaining bytes, 0x80, zeros, 64-bit bit length (RFC 1321 3.1-3.2)
    const uint8_t *t = slices[me] + nch * kChunk;
    size_t rem = S - nch * kChunk;
    uint32_t x[16];
    if (rem >= 64) {
        const uint4 *q = reinterpret_cast<const uint4 *>(t);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const uint4 u = __ldg(q + v);
            x[4 * v] = u.x;
            x[4 * v + 1] = u.y;
            x[4 * v + 2] = u.z;
            x[4 * v + 3] = u.w;
        }
        hash_block(stab, st, crc, x, CL);
        t += 64;
        rem -= 64;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j)
        x[j] = 0;
    for (size_t b = 0; b < rem; ++b) {
        uint32_t v = t[b];
        crc = crc_byte(stab, crc, v, CL);
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
    uint4 *o = reinterpret_cast<uint4 *>(md5_out + static_cast<size_t>(me) * 16);
    *o = make_uint4(st[0], st[1], st[2], st[3]);
    crc_out[me] = crc ^ 0xFFFFFFFFu;
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

size_t hash_smem_bytes() { return kHashSmem; }

int hash_run(p2g_ctx *ctx, const uint8_t *const *d_slices, int n, size_t S, uint8_t *d_md5,
             uint32_t *d_crc)
{
    if (n <= 0)
        return P2G_OK;
    const size_t smem = hash_smem_bytes();
    P2G_CUDA(cudaFuncSetAttribute(hash_slices_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    // spread the slices over every SM (one CTA per SM fits), at most 256 per CTA
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    const int per_cta = std::min(kHashThreads, std::max(1, (n + sms - 1) / sms));
    const int grid = (n + per_cta - 1) / per_cta;
    hash_slices_kernel<<<grid, kHashThreads, smem, ctx->stream>>>(d_slices, n, per_cta, S,
                                                                  ctx->d_crc, d_md5, d_crc);
    P2G_CUDA(cudaGetLastError());
    ++ctx->launches;
    return P2G_OK;
}

}  // namespace p2g
