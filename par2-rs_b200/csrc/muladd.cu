// muladd.cu -- GF(2^16) region multiply-accumulate on sm_100a.
//
// Replaces the per-strategy region kernels of par2-rs (galois/simd/x86/
// avx2.rs:686-821 behind galois/region/mod.rs:90-131, and the column path
// galois/mod.rs:328-349 used by par2_rs.rs:816-870) for both recovery-slice
// creation and repair:
//
//     dst[o][x] (^)= XOR_i  coeff(i, o) * src[i][x]      (GF(2^16), 0x1100B)
//
// Design (bit-sliced tables, "method of four Russians" over GF(2)):
//   * Inputs are first converted to 16 bit planes per group of 32 symbols
//     (slices_to_planes).  Multiplication by a constant is GF(2)-linear on the
//     planes (bitslice.cuh).
//   * A CTA owns one column tile of 1024 symbols (2 KiB of every slice) and a
//     block of up to 8*EREG outputs; each warp keeps EREG outputs x 16 planes
//     in registers, lane L owning symbol group L of the tile.
//   * Per input slice the CTA builds, in shared memory, two 256-row tables of
//     every XOR combination of planes 0-7 and of planes 8-15 (64 KiB, lane L's
//     column in bank L).  One output plane of one coefficient is then two
//     table rows XORed; the rows to read are the coefficient's "record" (32
//     row-index bytes), the same for all 32 lanes.  ldmatrix.x4 serves as a
//     4-row gather: one instruction hands every lane its own word of four
//     rows, so a coefficient costs 8 ldmatrix + 1 record load + 16 XORs per
//     lane.
//   * The next input's planes and records stream into a 4-slot shared-memory
//     ring with cp.async while the current table is consumed; the table is
//     double-buffered, one CTA barrier per input slice.
//   * Few tiles / outputs: the input range is split across CTAs and the
//     partial sums are folded into the output with atomic XOR.
//   * Problems of at most 24 outputs use three tables instead (planes 0-5,
//     6-10, 11-15: 64 + 32 + 32 rows, 16 KiB), built with 128 row stores per
//     input instead of 512 at 48 row reads per coefficient instead of 32;
//     with few outputs to share an input's tables the build dominates, and
//     the smaller tables let two CTAs share an SM.
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "async.cuh"
#include "bitslice.cuh"
#include "muladd.cuh"

namespace p2g {

constexpr int kTileBytes = 2048;             // 1024 symbols
constexpr int kTableWords = 512 * 32;        // T0 and T1, 128 B per row
constexpr int kTableBytes = kTableWords * 4; // 64 KiB
constexpr int kSmallTableWords = 128 * 32;   // T0, T1, T2 of the small-output form
constexpr int kSmallTableBytes = kSmallTableWords * 4;  // 16 KiB
constexpr int kRing = 4;
constexpr int kPairTileBytes = 1024;          // 512 symbols (paired form)
constexpr int kPairTableWords = 256 * 32;     // 256 combined rows of 128 B
// ring slots of the paired form with one / two inputs per CTA barrier
__host__ __device__ constexpr int pair_ring_slots(int stage) { return stage == 1 ? 4 : 8; }

// Four 8x8 b16 matrices from shared memory: lanes 8m..8m+7 give the row
// addresses of matrix m, lane L receives word L % 4 of row L / 4 of each.
__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t &d0, uint32_t &d1, uint32_t &d2,
                                        uint32_t &d3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(d0), "=r"(d1), "=r"(d2), "=r"(d3)
                 : "r"(addr));
}

// 32 little-endian u16 symbols at byte offset `off` of a 16-byte aligned
// slice of S bytes (zero beyond S), as 16 words of two symbols each.
__device__ __forceinline__ void load_group(const uint8_t *base, size_t S, size_t off,
                                           uint32_t x[16])
{
    if (off + 64 <= S) {
        const uint4 *p = reinterpret_cast<const uint4 *>(base + off);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint4 v = __ldg(p + q);
            x[4 * q] = v.x;
            x[4 * q + 1] = v.y;
            x[4 * q + 2] = v.z;
            x[4 * q + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            size_t o = off + 4 * j;
            uint32_t v = 0;
            if (o + 4 <= S)
                v = *reinterpret_cast<const uint32_t *>(base + o);
            else if (o + 2 <= S)
                v = *reinterpret_cast<const uint16_t *>(base + o);
            x[j] = v;
        }
    }
}

// Writes (mode 0), XORs (mode 1) or atomically XORs (mode 2) 32 symbols.
__device__ __forceinline__ void store_group(uint8_t *base, size_t S, size_t off,
                                            const uint32_t x[16], int mode)
{
    if (mode == 2) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            size_t o = off + 4 * j;
            if (o + 4 <= S) {
                atomicXor(reinterpret_cast<unsigned int *>(base + o), x[j]);
            } else if (o + 2 <= S) {
                // o is 4-byte aligned: the low half of the aligned word
                atomicXor(reinterpret_cast<unsigned int *>(base + o), x[j] & 0xFFFFu);
            }
        }
        return;
    }
    if (off + 64 <= S) {
        uint4 *p = reinterpret_cast<uint4 *>(base + off);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint4 v = make_uint4(x[4 * q], x[4 * q + 1], x[4 * q + 2], x[4 * q + 3]);
            if (mode == 1) {
                uint4 old = p[q];
                v.x ^= old.x;
                v.y ^= old.y;
                v.z ^= old.z;
                v.w ^= old.w;
            }
            p[q] = v;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            size_t o = off + 4 * j;
            if (o + 4 <= S) {
                uint32_t *p = reinterpret_cast<uint32_t *>(base + o);
                *p = mode == 1 ? (*p ^ x[j]) : x[j];
            } else if (o + 2 <= S) {
                uint16_t *p = reinterpret_cast<uint16_t *>(base + o);
                uint16_t v = static_cast<uint16_t>(x[j]);
                *p = mode == 1 ? static_cast<uint16_t>(*p ^ v) : v;
            }
        }
    }
}

// LE symbols -> planes[i][t][b][lane]; one thread per group of 32 symbols.
__global__ void slices_to_planes(const uint8_t *const *__restrict__ src, int nin, int T,
                                 size_t S, uint32_t *__restrict__ planes)
{
    size_t gid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    size_t total = static_cast<size_t>(nin) * T * 32;
    if (gid >= total)
        return;
    int lane = static_cast<int>(gid & 31);
    size_t it = gid >> 5;
    int t = static_cast<int>(it % T);
    int i = static_cast<int>(it / T);
    uint32_t x[16];
    load_group(src[i], S, static_cast<size_t>(t) * kTileBytes + lane * 64, x);
    transpose16x2(x);
    uint32_t *P = planes + it * 512 + lane;
#pragma unroll
    for (int b = 0; b < 16; ++b)
        P[b * 32] = x[b];
}

__global__ void records_matrix_kernel(const uint16_t *__restrict__ coeff, int nin, int nout,
                                      uint32_t *__restrict__ recs)
{
    size_t gid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (gid >= static_cast<size_t>(nin) * nout)
        return;
    int o = static_cast<int>(gid % nout);
    size_t i = gid / nout;
    write_record(recs, gid, coeff[static_cast<size_t>(o) * nin + i], nout <= kSmallOutputs);
}

// c_i^e by the log / antilog tables: (log c * e) mod 65535 (galois/core.rs:242-258)
__global__ void records_par2_kernel(const uint16_t *__restrict__ consts,
                                    const uint32_t *__restrict__ exps,
                                    const uint16_t *__restrict__ glog,
                                    const uint16_t *__restrict__ gexp, int nin, int nout,
                                    uint32_t *__restrict__ recs)
{
    size_t gid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (gid >= static_cast<size_t>(nin) * nout)
        return;
    int o = static_cast<int>(gid % nout);
    int i = static_cast<int>(gid / nout);
    uint32_t base = consts[i];
    uint32_t e = exps[o];
    uint32_t c;
    if (base == 0)
        c = e == 0 ? 1u : 0u;
    else if (e == 0)
        c = 1u;
    else
        c = gexp[static_cast<uint32_t>((static_cast<uint64_t>(glog[base]) * e) % 65535u)];
    write_record(recs, gid, c, nout <= kSmallOutputs);
}

// WARPS warps per CTA; each output group of EREG outputs is held by PSPLIT
// warps, each keeping 16 / PSPLIT of the 16 planes (PSPLIT = 2 doubles the
// warps per SM at the same number of outputs per table).  SMALL selects the
// small-output tables (6 + 5 + 5 planes, 24-word records; 8 warps, PSPLIT 1).
// One work item: column tile t, output block ob, inputs [i0, i1).  smode:
// 0 store, 1 XOR into the outputs, 2 atomic XOR (input ranges of one tile
// and block handled by several CTAs).
template <int WARPS, int EREG, int PSPLIT, bool SMALL = false>
__device__ __forceinline__ void muladd_item(uint8_t *smem, const uint32_t *__restrict__ planes,
                                            const uint32_t *__restrict__ recs, int nin, int nout,
                                            int T, int t, int ob, int i0, int i1,
                                            uint8_t *const *__restrict__ dst, size_t S, int smode)
{
    static_assert(!SMALL || (WARPS == 8 && PSPLIT == 1), "small tables: 8 warps, no plane split");
    constexpr int THREADS = WARPS * 32;
    constexpr int GROUPS = WARPS / PSPLIT;   // output groups
    constexpr int NPL = 16 / PSPLIT;         // planes per warp
    constexpr int EBLK = GROUPS * EREG;
    constexpr int RW = SMALL ? kRecordWordsSmall : kRecordWords;  // words per record
    constexpr int TW = SMALL ? kSmallTableWords : kTableWords;   // words per table buffer
    constexpr int SLOT = kTileBytes + EBLK * RW * 4;
    uint32_t *tab = reinterpret_cast<uint32_t *>(smem);
    uint8_t *ring = smem + 2 * TW * 4;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int obase = ob * EBLK;
    const int nb = min(EBLK, nout - obase);
    const int ph = warp % PSPLIT;            // which planes: [ph*NPL, ph*NPL + NPL)
    // a partial block's outputs are spread evenly over the groups
    const int per = (nb + GROUPS - 1) / GROUPS;
    const int my0 = (warp / PSPLIT) * per;
    const int myn = max(0, min(per, nb - my0));

    auto issue = [&](int i) {
        if (i < i1) {
            uint8_t *s = ring + (i & (kRing - 1)) * SLOT;
            const uint8_t *gp = reinterpret_cast<const uint8_t *>(
                planes + (static_cast<size_t>(i) * T + t) * 512);
            const uint8_t *gr = reinterpret_cast<const uint8_t *>(
                recs + (static_cast<size_t>(i) * nout + obase) * RW);
            const int nchunk = 128 + nb * (RW / 4);
            for (int c = threadIdx.x; c < nchunk; c += THREADS) {
                if (c < 128)
                    cp_async16(s + c * 16, gp + c * 16);
                else
                    cp_async16(s + kTileBytes + (c - 128) * 16, gr + (c - 128) * 16);
            }
        }
        cp_async_commit();
    };

    // The 512 table rows form 32 groups of 16 (half = g / 16 selects planes
    // 0-7 or 8-15; h = g % 16 is the pattern of the half's planes 4-7, the
    // row's low nibble the pattern of its planes 0-3).  Warp w builds groups
    // [32w/WARPS, 32(w+1)/WARPS), which never straddle the two halves for
    // WARPS in {8, 12, 16}.
    // Small form: warp w builds 16 rows -- warps 0-3 the four quarters of T0
    // (planes 0-3 vary, planes 4-5 fixed by w), warps 4-5 the halves of T1
    // (planes 6-9 vary, plane 10 fixed), warps 6-7 those of T2 (planes 11-14,
    // plane 15).
    auto build_small = [&](int i, int buf) {
        const uint32_t *P = reinterpret_cast<const uint32_t *>(ring + (i & (kRing - 1)) * SLOT);
        int b0, row0;
        uint32_t H;
        if (warp < 4) {
            b0 = 0;
            row0 = 16 * warp;
            H = ((warp & 1) ? P[4 * 32 + lane] : 0u) ^ ((warp & 2) ? P[5 * 32 + lane] : 0u);
        } else if (warp < 6) {
            b0 = 6;
            row0 = 64 + 16 * (warp - 4);
            H = (warp & 1) ? P[10 * 32 + lane] : 0u;
        } else {
            b0 = 11;
            row0 = 96 + 16 * (warp - 6);
            H = (warp & 1) ? P[15 * 32 + lane] : 0u;
        }
        uint32_t p[4];
#pragma unroll
        for (int b = 0; b < 4; ++b)
            p[b] = P[(b0 + b) * 32 + lane];
        uint32_t L[16];
        L[0] = 0;
        L[1] = p[0];
        L[2] = p[1];
        L[3] = p[0] ^ p[1];
        L[4] = p[2];
        L[5] = L[4] ^ p[0];
        L[6] = L[4] ^ p[1];
        L[7] = L[6] ^ p[0];
#pragma unroll
        for (int x = 0; x < 8; ++x)
            L[8 + x] = L[x] ^ p[3];
        uint32_t *T0 = tab + buf * TW + row0 * 32 + lane;
#pragma unroll
        for (int x = 0; x < 16; ++x)
            T0[x * 32] = H ^ L[x];
    };

    auto build = [&](int i, int buf) {
        if constexpr (SMALL) {
            build_small(i, buf);
            return;
        }
        const uint32_t *P = reinterpret_cast<const uint32_t *>(ring + (i & (kRing - 1)) * SLOT);
        const int g0 = warp * 32 / WARPS, g1 = (warp + 1) * 32 / WARPS;
        const int half = g0 >> 4;
        uint32_t p[8];
#pragma unroll
        for (int b = 0; b < 8; ++b)
            p[b] = P[(half * 8 + b) * 32 + lane];
        uint32_t L[16];
        L[0] = 0;
        L[1] = p[0];
        L[2] = p[1];
        L[3] = p[0] ^ p[1];
        L[4] = p[2];
        L[5] = L[4] ^ p[0];
        L[6] = L[4] ^ p[1];
        L[7] = L[6] ^ p[0];
#pragma unroll
        for (int x = 0; x < 8; ++x)
            L[8 + x] = L[x] ^ p[3];
        constexpr int GMAX = (32 + WARPS - 1) / WARPS;
        const int h0 = g0 & 15;
        uint32_t *T0 = tab + buf * TW + (half * 256 + h0 * 16) * 32 + lane;
#pragma unroll
        for (int gg = 0; gg < GMAX; ++gg) {
            if (GMAX * WARPS == 32 || g0 + gg < g1) {
                const int h = h0 + gg;
                const uint32_t H = ((h & 1) ? p[4] : 0u) ^ ((h & 2) ? p[5] : 0u) ^
                                   ((h & 4) ? p[6] : 0u) ^ ((h & 8) ? p[7] : 0u);
#pragma unroll
                for (int x = 0; x < 16; ++x)
                    T0[(gg * 16 + x) * 32] = H ^ L[x];
            }
        }
    };

    uint32_t acc[EREG][NPL];
#pragma unroll
    for (int e = 0; e < EREG; ++e)
#pragma unroll
        for (int j = 0; j < NPL; ++j)
            acc[e][j] = 0;

    // Lane L fetches, per plane pair, word L of four table rows with one
    // ldmatrix.x4; it supplies the address of 16-byte chunk (L % 8) of the
    // row of class L / 8, read from its class's 8 record bytes (bitslice.cuh
    // make_record).  Odd classes read T1, whose rows follow T0's 256: their
    // lanes' base address carries the 32 KiB.
    const uint32_t tab_s = static_cast<uint32_t>(__cvta_generic_to_shared(tab)) + (lane & 7) * 16 +
                           ((!SMALL && ((lane >> 3) & 1)) ? 256u * 128u : 0u);
    auto consume_small = [&](int i, int buf) {
        // lane group m's six record words: 3 x 8 bytes at word 6m of each record
        const uint2 *R = reinterpret_cast<const uint2 *>(ring + (i & (kRing - 1)) * SLOT +
                                                         kTileBytes) +
                         my0 * (RW / 2) + (lane >> 3) * 3;
        const uint32_t tb = tab_s + buf * TW * 4;
#pragma unroll
        for (int e = 0; e < EREG; ++e) {
            if (e < myn) {
                uint32_t w[6];
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const uint2 r = R[e * (RW / 2) + q];
                    w[2 * q] = r.x;
                    w[2 * q + 1] = r.y;
                }
                // ldmatrix k: rows 4k..4k+3 of the sequence s = 3j + t
#pragma unroll
                for (int k = 0; k < 12; ++k) {
                    const uint32_t off = (k & 1) ? (w[k >> 1] >> 16) : (w[k >> 1] & 0xFFFFu);
                    uint32_t d[4];
                    ldsm_x4(tb + off, d[0], d[1], d[2], d[3]);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        acc[e][(4 * k + q) / 3] ^= d[q];
                }
            }
        }
    };

    auto consume = [&](int i, int buf) {
        if constexpr (SMALL) {
            consume_small(i, buf);
            return;
        }
        // lane group m's 8 record bytes: words 2m, 2m + 1
        const uint2 *R = reinterpret_cast<const uint2 *>(ring + (i & (kRing - 1)) * SLOT +
                                                         kTileBytes) +
                         my0 * 4 + (lane >> 3);
        const uint32_t tb = tab_s + buf * kTableBytes;
        // the next output's record is loaded before this output's lookups, so
        // it does not wait behind them in the shared-memory queue
        uint2 nxt = make_uint2(0, 0);
        if constexpr (PSPLIT == 1)
            if (myn > 0)
                nxt = R[0];
#pragma unroll
        for (int e = 0; e < EREG; ++e) {
            if (e < myn) {
                uint32_t w[2];
                if constexpr (PSPLIT == 1) {
                    const uint2 r = nxt;
                    if (e + 1 < myn)
                        nxt = R[(e + 1) * 4];
                    w[0] = r.x;
                    w[1] = r.y;
                } else {
                    // plane pairs [4ph, 4ph+4): record word 2m + ph
                    w[0] = reinterpret_cast<const uint32_t *>(R + e * 4)[ph];
                    w[1] = 0;
                }
#pragma unroll
                for (int p = 0; p < NPL / 2; ++p) {
                    const uint32_t row = __byte_perm(w[p >> 2], 0u, 0x4440u | (p & 3));
                    uint32_t d0, d1, d2, d3;
                    ldsm_x4(tb + (row << 7), d0, d1, d2, d3);
                    acc[e][2 * p] ^= d0 ^ d1;
                    acc[e][2 * p + 1] ^= d2 ^ d3;
                }
            }
        }
    };

    if (i0 < i1) {
        issue(i0);
        issue(i0 + 1);
        issue(i0 + 2);
        cp_async_wait<1>();
        __syncthreads();
        build(i0, 0);
        __syncthreads();
        for (int i = i0; i < i1; ++i) {
            issue(i + 3);
            consume(i, (i - i0) & 1);
            if (i + 1 < i1)
                build(i + 1, (i + 1 - i0) & 1);
            cp_async_wait<1>();
            __syncthreads();
        }
    }
    cp_async_wait<0>();

    if constexpr (PSPLIT == 1) {
#pragma unroll
        for (int e = 0; e < EREG; ++e) {
            if (e < myn) {
                uint32_t x[16];
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    x[j] = acc[e][j];
                transpose16x2(x);
                store_group(dst[obase + my0 + e], S,
                            static_cast<size_t>(t) * kTileBytes + lane * 64, x, smode);
            }
        }
    } else {
        // the odd warp of each pair hands its planes 8-15 to the even warp
        // through shared memory (the tables are no longer needed)
        uint32_t *xch = tab + (warp / 2) * (8 * 32);
#pragma unroll
        for (int e = 0; e < EREG; ++e) {
            __syncthreads();
            if (ph == 1 && e < myn)
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    xch[j * 32 + lane] = acc[e][j];
            __syncthreads();
            if (ph == 0 && e < myn) {
                uint32_t x[16];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    x[j] = acc[e][j];
                    x[8 + j] = xch[j * 32 + lane];
                }
                transpose16x2(x);
                store_group(dst[obase + my0 + e], S,
                            static_cast<size_t>(t) * kTileBytes + lane * 64, x, smode);
            }
        }
    }
}

template <int WARPS, int EREG, int PSPLIT, bool SMALL = false>
__global__ void __launch_bounds__(WARPS * 32, SMALL ? 2 : 1)
    muladd_bitsliced(const uint32_t *__restrict__ planes, const uint32_t *__restrict__ recs,
                     int nin, int nout, int T, int nblk, int nsplit,
                     uint8_t *const *__restrict__ dst, size_t S, int mode)
{
    extern __shared__ __align__(128) uint8_t smem[];
    int bid = blockIdx.x;
    const int split = bid % nsplit;
    bid /= nsplit;
    const int ob = bid % nblk;
    const int t = bid / nblk;
    const int i0 = static_cast<int>(static_cast<long long>(nin) * split / nsplit);
    const int i1 = static_cast<int>(static_cast<long long>(nin) * (split + 1) / nsplit);
    muladd_item<WARPS, EREG, PSPLIT, SMALL>(smem, planes, recs, nin, nout, T, t, ob, i0, i1,
                                            dst, S, nsplit > 1 ? 2 : mode);
}

// The paired form: a CTA owns a column tile of 512 symbols (half of a plane
// tile) and each warp accumulates TWO outputs per table lookup, lanes 0-15 one
// and lanes 16-31 the other (lane L owning symbol group L % 16).  Both halves
// share the input's tables, so one table build serves up to 16 * EREG
// outputs per warp pair count -- 208 for EREG = 13, which covers r = 205 in
// one output block where the 1024-symbol form needs two blocks, each
// building the same tables.  The table build halves with the tile (256
// combined rows per input instead of 512 rows), the lookups per output do
// not change.
//
// Table: 256 combined rows of 128 bytes, row n = [T0 row n | T1 row n] with
// T0 row n (words 0-15) the XOR of planes {b < 8 : bit b of n} for groups
// 0-15 and T1 row n (words 16-31) that of planes {8 + b}.  One ldmatrix.x4
// serves a plane pair of both outputs: in each of its four 8x8 matrices one
// half-warp reads a T0 half-row and the other a T1 half-row (64 bytes each,
// disjoint banks), so every matrix is one conflict-free wavefront:
//   matrix 0: lanes 0-15 T0[n0_2k(A)], lanes 16-31 T1[n1_2k(B)]
//   matrix 1: lanes 0-15 T1[n1_2k(A)], lanes 16-31 T0[n0_2k(B)]
//   matrix 2, 3: the same for plane 2k + 1
// (A, B: the outputs of the two halves).  Records are the 8-word records of
// the 1024-symbol form (bitslice.cuh make_record): record words 2m, 2m + 1
// hold the class-m row indices, and the lanes that give matrix m's addresses
// for output B read class m ^ 1, whose T0 / T1 roles are swapped.
template <int WARPS, int EREG, int STAGE>
__device__ __forceinline__ void muladd_item_paired(uint8_t *smem, const uint32_t *__restrict__ planes,
                                                   const uint32_t *__restrict__ recs, int nout,
                                                   int T, int u, int ob, int i0, int i1,
                                                   uint8_t *const *__restrict__ dst, size_t S,
                                                   int smode)
{
    static_assert(STAGE == 1 || STAGE == 2, "one or two inputs per barrier");
    constexpr int THREADS = WARPS * 32;
    constexpr int EBLK = WARPS * EREG * 2;                 // outputs per block
    constexpr int TW = kPairTableWords;                    // words per table buffer
    constexpr int SLOT = kPairTileBytes + EBLK * kRecordWords * 4;
    constexpr int RING = pair_ring_slots(STAGE);
    uint32_t *tab = reinterpret_cast<uint32_t *>(smem);
    uint8_t *ring = smem + 2 * STAGE * TW * 4;
    // ring slot of input i (RING is a power of two: any RING consecutive
    // inputs take distinct slots)
    static_assert((RING & (RING - 1)) == 0, "ring slots: a power of two");
    auto slot = [&](int i) { return ring + (i & (RING - 1)) * SLOT; };

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int half = lane >> 4;
    const int grp = lane & 15;
    const int obase = ob * EBLK;
    const int nb = min(EBLK, nout - obase);
    const int npairs = (nb + 1) >> 1;
    // a partial block's pairs are spread evenly over the warps
    const int per = (npairs + WARPS - 1) / WARPS;
    const int q0 = warp * per;
    const int myq = max(0, min(per, npairs - q0));
    const int t = u >> 1, hsel = u & 1;  // plane tile and its half

    auto issue = [&](int i) {
        if (i < i1) {
            uint8_t *s = slot(i);
            // planes b = 0..15, groups 16 hsel .. 16 hsel + 15: 64 bytes each
            const uint8_t *gp = reinterpret_cast<const uint8_t *>(
                planes + (static_cast<size_t>(i) * T + t) * 512 + hsel * 16);
            const uint8_t *gr = reinterpret_cast<const uint8_t *>(
                recs + (static_cast<size_t>(i) * nout + obase) * kRecordWords);
            // an odd block's last record is copied twice, so that the
            // second output of its last pair reads valid offsets
            const int nchunk = 64 + (nb + (nb & 1)) * (kRecordWords / 4);
            for (int c = threadIdx.x; c < nchunk; c += THREADS) {
                // plane b goes to position 2 (b % 8) + b / 8, so that planes
                // b and b + 8, read together by the two halves of a warp in
                // the build, share one 128-byte row of banks
                if (c < 64) {
                    cp_async16(s + (((c >> 2) & 7) * 2 + (c >> 5)) * 64 + (c & 3) * 16,
                               gp + (c >> 2) * 128 + (c & 3) * 16);
                } else {
                    const int rc = c - 64;
                    cp_async16(s + kPairTileBytes + rc * 16,
                               gr + (rc < nb * (kRecordWords / 4) ? rc : rc - kRecordWords / 4) * 16);
                }
            }
        }
        cp_async_commit();
    };

    // Lane L writes word L of the combined rows: lanes 0-15 T0 (planes 0-7 of
    // group L), lanes 16-31 T1 (planes 8-15 of group L - 16).  The 256 rows
    // form 16 groups of 16 (low nibble: planes 0-3 of the half, high nibble
    // h: planes 4-7); warp w builds groups [16w/WARPS, 16(w+1)/WARPS).
    auto build = [&](int i, int buf) {
        const uint32_t *P = reinterpret_cast<const uint32_t *>(slot(i));
        uint32_t p[8];
#pragma unroll
        for (int b = 0; b < 8; ++b)
            p[b] = P[(b * 2 + half) * 16 + grp];
        uint32_t L[16];
        L[0] = 0;
        L[1] = p[0];
        L[2] = p[1];
        L[3] = p[0] ^ p[1];
        L[4] = p[2];
        L[5] = L[4] ^ p[0];
        L[6] = L[4] ^ p[1];
        L[7] = L[6] ^ p[0];
#pragma unroll
        for (int x = 0; x < 8; ++x)
            L[8 + x] = L[x] ^ p[3];
        const int g0 = warp * 16 / WARPS, g1 = (warp + 1) * 16 / WARPS;
        constexpr int GMAX = (16 + WARPS - 1) / WARPS;
        uint32_t *Tp = tab + buf * TW + g0 * 16 * 32 + lane;
#pragma unroll
        for (int gg = 0; gg < GMAX; ++gg) {
            if (GMAX * WARPS == 16 || g0 + gg < g1) {
                const int h = g0 + gg;
                const uint32_t H = ((h & 1) ? p[4] : 0u) ^ ((h & 2) ? p[5] : 0u) ^
                                   ((h & 4) ? p[6] : 0u) ^ ((h & 8) ? p[7] : 0u);
#pragma unroll
                for (int x = 0; x < 16; ++x)
                    Tp[(gg * 16 + x) * 32] = H ^ L[x];
            }
        }
    };

    uint32_t acc[EREG][16];
#pragma unroll
    for (int e = 0; e < EREG; ++e)
#pragma unroll
        for (int j = 0; j < 16; ++j)
            acc[e][j] = 0;

    // As an address giver, lane L serves matrix m = L / 8 for output s =
    // (L / 4) & 1 of the pair (chunk L % 4 of that output's half-row) and
    // reads the 8 record bytes of class m ^ s of output s.  Odd classes index
    // T1, whose half-row of combined row n sits at n * 128 + 64: their lanes'
    // base address carries the 64.  The second output of an odd block's last
    // pair reads the duplicated last record (its sums are never stored).
    const int gs = (lane >> 2) & 1;
    const int gcls = (lane >> 3) ^ gs;
    const uint32_t tab_s = static_cast<uint32_t>(__cvta_generic_to_shared(tab)) + (lane & 3) * 16 +
                           (gcls & 1) * 64;
    auto consume = [&](int i, int buf) {
        const uint2 *R = reinterpret_cast<const uint2 *>(slot(i) + kPairTileBytes) +
                         (2 * q0 + gs) * 4 + gcls;
        const uint32_t tb = tab_s + buf * TW * 4;
        // the next pair's record is loaded before this pair's lookups
        uint2 nxt = myq > 0 ? R[0] : make_uint2(0, 0);
#pragma unroll
        for (int e = 0; e < EREG; ++e) {
            if (e < myq) {
                const uint2 r = nxt;
                if (e + 1 < myq)
                    nxt = R[(e + 1) * 8];
                const uint32_t w[2] = {r.x, r.y};
#pragma unroll
                for (int p = 0; p < 8; ++p) {
                    const uint32_t row = __byte_perm(w[p >> 2], 0u, 0x4440u | (p & 3));
                    uint32_t d0, d1, d2, d3;
                    ldsm_x4(tb + (row << 7), d0, d1, d2, d3);
                    acc[e][2 * p] ^= d0 ^ d1;
                    acc[e][2 * p + 1] ^= d2 ^ d3;
                }
            }
        }
    };

    if constexpr (STAGE == 1) {
        // one input per barrier: consume input i, then build input i + 1
        // (lookups first: 2 % faster than building first)
        if (i0 < i1) {
            issue(i0);
            issue(i0 + 1);
            issue(i0 + 2);
            cp_async_wait<1>();
            __syncthreads();
            build(i0, 0);
            __syncthreads();
            for (int i = i0; i < i1; ++i) {
                issue(i + 3);
                consume(i, (i - i0) & 1);
                if (i + 1 < i1)
                    build(i + 1, (i + 1 - i0) & 1);
                cp_async_wait<1>();
                __syncthreads();
            }
        }
    } else {
        // two inputs per barrier (four table buffers, eight ring slots):
        // stage s consumes inputs s, s + 1 from one table pair, then builds
        // s + 2, s + 3 into the other (lookups first: 1 % faster than
        // building first), and fetches s + 6, s + 7, whose copies may still
        // be in flight at the barrier that ends the stage (s + 4, s + 5,
        // fetched a stage earlier, must have landed by then)
        if (i0 < i1) {
#pragma unroll
            for (int q = 0; q < 6; ++q)
                issue(i0 + q);
            cp_async_wait<4>();
            __syncthreads();
            build(i0, 0);
            if (i0 + 1 < i1)
                build(i0 + 1, 1);
            cp_async_wait<2>();
            __syncthreads();
            for (int s = i0; s < i1; s += 2) {
                const int tp = ((s - i0) >> 1) & 1;
                issue(s + 6);
                issue(s + 7);
                consume(s, 2 * tp);
                if (s + 1 < i1)
                    consume(s + 1, 2 * tp + 1);
                if (s + 2 < i1)
                    build(s + 2, 2 * (tp ^ 1));
                if (s + 3 < i1)
                    build(s + 3, 2 * (tp ^ 1) + 1);
                cp_async_wait<2>();
                __syncthreads();
            }
        }
    }
    cp_async_wait<0>();

#pragma unroll
    for (int e = 0; e < EREG; ++e) {
        const int o = 2 * (q0 + e) + half;
        if (e < myq && o < nb) {
            uint32_t x[16];
#pragma unroll
            for (int j = 0; j < 16; ++j)
                x[j] = acc[e][j];
            transpose16x2(x);
            store_group(dst[obase + o], S, static_cast<size_t>(u) * kPairTileBytes + grp * 64, x,
                        smode);
        }
    }
}

template <int WARPS, int EREG, int STAGE>
__global__ void __launch_bounds__(WARPS * 32, 1)
    muladd_paired(const uint32_t *__restrict__ planes, const uint32_t *__restrict__ recs,
                  int nin, int nout, int T, int nblk, int nsplit,
                  uint8_t *const *__restrict__ dst, size_t S, int mode)
{
    extern __shared__ __align__(128) uint8_t smem[];
    int bid = blockIdx.x;
    const int split = bid % nsplit;
    bid /= nsplit;
    const int ob = bid % nblk;
    const int u = bid / nblk;
    const int i0 = static_cast<int>(static_cast<long long>(nin) * split / nsplit);
    const int i1 = static_cast<int>(static_cast<long long>(nin) * (split + 1) / nsplit);
    muladd_item_paired<WARPS, EREG, STAGE>(smem, planes, recs, nout, T, u, ob, i0, i1, dst, S,
                                           nsplit > 1 ? 2 : mode);
}

// Persistent form for batches of independent problems: one CTA per SM takes
// items (problem, tile, output block, input split) from a queue ordered
// longest first and runs each in its problem's form as muladd_bitsliced /
// muladd_paired would.
__global__ void __launch_bounds__(kBatchWarps * 32, 1)
    muladd_persistent(const BatchProb *__restrict__ probs, const BatchItem *__restrict__ items,
                      int nitems, int *__restrict__ counter, const volatile int *abort)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ int cur;
    int stop = 0, fetches = 0;  // the abort flag as read during an earlier item
    while (true) {
        // a raised abort flag stops the CTA before its next item
        if (threadIdx.x == 0)
            cur = stop ? nitems : atomicAdd(counter, 1);
        __syncthreads();
        const int it = cur;
        if (it >= nitems)
            break;
        // poll the flag on every 4th item, used at a later fetch so that the
        // read overlaps the item's work
        if (threadIdx.x == 0 && (fetches++ & 3) == 0)
            stop = *abort;
        const BatchItem item = items[it];
        const BatchProb p = probs[item.prob];
        const int i0 = static_cast<int>(static_cast<long long>(p.nin) * item.split / p.nsplit);
        const int i1 =
            static_cast<int>(static_cast<long long>(p.nin) * (item.split + 1) / p.nsplit);
        const int smode = p.nsplit > 1 ? 2 : p.mode;
        if (p.form == kFormPaired)
            muladd_item_paired<kBatchWarps, 13, 2>(smem, p.planes, p.recs, p.nout, p.T, item.t,
                                                   item.ob, i0, i1, p.dst, p.S, smode);
        else if (p.form == kFormSmall)
            muladd_item<kBatchWarps, 3, 1, true>(smem, p.planes, p.recs, p.nin, p.nout, p.T,
                                                 item.t, item.ob, i0, i1, p.dst, p.S, smode);
        else
            muladd_item<kBatchWarps, 13, 1>(smem, p.planes, p.recs, p.nin, p.nout, p.T, item.t,
                                            item.ob, i0, i1, p.dst, p.S, smode);
        __syncthreads();
    }
}

// Zeroes nout slices before a split (atomic-XOR) run in store mode.
__global__ void zero_slices(uint8_t *const *__restrict__ dst, int nout, size_t S)
{
    int o = blockIdx.y;
    if (o >= nout)
        return;
    uint8_t *d = dst[o];
    for (size_t x = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) * 16; x < S;
         x += static_cast<size_t>(gridDim.x) * blockDim.x * 16) {
        if (x + 16 <= S)
            *reinterpret_cast<uint4 *>(d + x) = make_uint4(0, 0, 0, 0);
        else
            for (size_t y = x; y < S; y += 2)
                *reinterpret_cast<uint16_t *>(d + y) = 0;
    }
}

using KernelFn = void (*)(const uint32_t *, const uint32_t *, int, int, int, int, int,
                          uint8_t *const *, size_t, int);

struct Variant {
    int warps, ereg, psplit;
    bool small;   // small-output tables (problems of at most kSmallOutputs outputs)
    bool paired;  // 512-symbol tiles, two outputs per warp lookup (muladd_paired)
    int stage;    // inputs per CTA barrier (paired form: 1 or 2)
    KernelFn fn;
};

// Compiled tile shapes: warps per CTA x outputs per warp.  The register
// budget (64K per SM, one CTA per SM) caps EREG at 13 / 8 / 5 for 8 / 12 / 16
// warps without spills; the paired form holds EREG pairs of outputs per warp
// (2 x EREG outputs, EREG x 16 accumulator registers per lane).
#define P2G_V(W, E, P) {W, E, P, false, false, 1, muladd_bitsliced<W, E, P>}
#define P2G_VS(E) {8, E, 1, true, false, 1, muladd_bitsliced<8, E, 1, true>}
#define P2G_VP(W, E, G) {W, E, 1, false, true, G, muladd_paired<W, E, G>}
static const Variant kVariants[] = {
    P2G_VS(1),        P2G_VS(2),        P2G_VS(3),
    P2G_V(8, 1, 1),   P2G_V(8, 2, 1),   P2G_V(8, 3, 1),   P2G_V(8, 4, 1),   P2G_V(8, 5, 1),
    P2G_V(8, 6, 1),   P2G_V(8, 7, 1),   P2G_V(8, 8, 1),   P2G_V(8, 9, 1),   P2G_V(8, 10, 1),
    P2G_V(8, 11, 1),  P2G_V(8, 12, 1),  P2G_V(8, 13, 1),  P2G_V(12, 4, 1),  P2G_V(12, 6, 1),
    P2G_V(12, 7, 1),  P2G_V(12, 8, 1),  P2G_V(16, 2, 1),  P2G_V(16, 3, 1),  P2G_V(16, 4, 1),
    P2G_V(16, 5, 1),  P2G_V(16, 8, 2),  P2G_V(16, 10, 2), P2G_V(16, 12, 2),
    P2G_VP(8, 7, 1),  P2G_VP(8, 8, 1),  P2G_VP(8, 9, 1),  P2G_VP(8, 10, 1), P2G_VP(8, 11, 1),
    P2G_VP(8, 12, 1), P2G_VP(8, 13, 1), P2G_VP(12, 8, 1), P2G_VP(8, 7, 2),  P2G_VP(8, 9, 2),
    P2G_VP(8, 11, 2), P2G_VP(8, 13, 2), P2G_VP(12, 8, 2),
};
#undef P2G_V
#undef P2G_VS
#undef P2G_VP

static KernelFn kernel_for(int warps, int ereg, int psplit, bool small, bool paired, int stage)
{
    for (const Variant &v : kVariants)
        if (v.warps == warps && v.ereg == ereg && v.psplit == psplit && v.small == small &&
            v.paired == paired && v.stage == stage)
            return v.fn;
    return nullptr;
}
static KernelFn kernel_for(const MuladdPlan &p)
{
    return kernel_for(p.warps, p.ereg, p.psplit, p.small, p.paired, p.stage);
}

// The 8 + 8 shapes (the small-output form reuses 8-warp shapes of 1-3
// outputs per warp).
int muladd_variants(int *warps, int *eregs, int *psplits, int cap)
{
    int n = 0;
    for (const Variant &v : kVariants) {
        if (v.small || v.paired)
            continue;
        if (n < cap) {
            warps[n] = v.warps;
            eregs[n] = v.ereg;
            psplits[n] = v.psplit;
        }
        ++n;
    }
    return n;
}

// outputs one CTA of this shape covers
static int block_outputs(const MuladdPlan &p)
{
    return p.paired ? p.warps * p.ereg * 2 : p.warps / p.psplit * p.ereg;
}

int plan_tiles(const MuladdPlan &p, size_t S)
{
    const size_t tb = p.paired ? kPairTileBytes : kTileBytes;
    return static_cast<int>((S + tb - 1) / tb);
}

static size_t smem_bytes(const MuladdPlan &p)
{
    if (p.paired)
        return 2 * p.stage * kPairTableWords * 4 +
               pair_ring_slots(p.stage) * (kPairTileBytes + block_outputs(p) * kRecordWords * 4);
    if (p.small)
        return 2 * kSmallTableBytes + kRing * (kTileBytes + block_outputs(p) * kRecordWordsSmall * 4);
    return 2 * kTableBytes + kRing * (kTileBytes + block_outputs(p) * kRecordWords * 4);
}

// CTAs of plan p that fit on one SM at once (registers and shared memory),
// from the occupancy calculator; cached per compiled shape.
static int resident_ctas(const MuladdPlan &p)
{
    static std::mutex mu;
    static std::map<std::tuple<int, int, int, bool, bool, int>, int> cache;
    const auto key = std::make_tuple(p.warps, p.ereg, p.psplit, p.small, p.paired, p.stage);
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end())
        return it->second;
    int n = 0;
    KernelFn fn = kernel_for(p);
    const size_t smem = smem_bytes(p);
    if (!fn ||
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, p.warps * 32, smem) != cudaSuccess ||
        n < 1) {
        cudaGetLastError();
        n = 1;
    }
    cache[key] = n;
    return n;
}

int plan_slots(const p2g_ctx *ctx, const MuladdPlan &p)
{
    const int sms = ctx && ctx->sm_count > 0 ? ctx->sm_count : 148;
    return sms * resident_ctas(p);
}

MuladdPlan choose_plan(const p2g_ctx *ctx, int nin, int nout, size_t S)
{
    if (ctx) {
        auto it = ctx->plans.find(plan_key(nin, nout, S));
        if (it != ctx->plans.end())
            return it->second;
    }
    MuladdPlan p;
    p.warps = 8;
    p.small = nout <= kSmallOutputs;
    if (nout > 8 * 13) {
        // more outputs than one 1024-symbol block holds: the paired form
        // (up to 208 outputs per block) builds each input's tables half as
        // often per output
        p.paired = true;
        p.nblk = (nout + 8 * 13 * 2 - 1) / (8 * 13 * 2);
        const int pairs = ((nout + p.nblk - 1) / p.nblk + 1) / 2;
        // two inputs per barrier (compiled for odd pair counts 7-13 per warp)
        p.ereg = std::max(7, (pairs + 7) / 8) | 1;
        p.stage = 2;
    } else {
        p.nblk = (nout + 8 * 13 - 1) / (8 * 13);
        p.ereg = std::max(1, (nout + 8 * p.nblk - 1) / (8 * p.nblk));
    }
    const int T = plan_tiles(p, S);
    // Input splits (atomic-XOR folds, whole aligned words: S % 4 == 0) for
    // grids that would leave SMs idle.  A CTA costs its inputs plus a fixed
    // prologue/epilogue of ~17 input tiles (~20 when it folds atomically),
    // and a launch takes ceil(CTAs / resident slots) waves; the split count
    // minimising waves x per-CTA cost wins.  Fitted on 205 outputs, 148 SMs:
    // it picks the fastest measured split for 2048 and 256 inputs at 16, 32,
    // 64 and 128 KiB (e.g. 2048 x 64 KiB: 1 split 5.09 ms, 2 splits 2.63,
    // 9 splits 2.50; 256 x 128 KiB: 1 split 0.68 ms, 8 splits 0.96).
    if (S % 4 == 0 && nin >= 16) {
        const int sms = ctx && ctx->sm_count > 0 ? ctx->sm_count : 148;
        const long long slots = static_cast<long long>(sms) * resident_ctas(p);
        const long long ctas = static_cast<long long>(T) * p.nblk;
        const int cap = std::min(64, nin / 8);
        double best = 0;
        for (int sp = 1; sp <= cap; ++sp) {
            const long long waves = (ctas * sp + slots - 1) / slots;
            const double cost = static_cast<double>(waves) *
                                (static_cast<double>(nin) / sp + (sp == 1 ? 17.0 : 20.0));
            if (sp == 1 || cost < best * 0.999) {
                best = cost;
                p.nsplit = sp;
            }
        }
    }
    return p;
}

bool plan_valid(const MuladdPlan &p, int nin, int nout, size_t S)
{
    if (p.psplit < 1 || p.small != (nout <= kSmallOutputs) || (p.paired && p.small) ||
        (!p.paired && p.stage != 1) || kernel_for(p) == nullptr || p.nblk < 1)
        return false;
    const long long eb = block_outputs(p);
    return p.nblk * eb >= nout && (p.nblk - 1) * eb < nout && p.nsplit >= 1 &&
           (p.nsplit == 1 || (S % 4 == 0 && p.nsplit <= std::max(1, nin)));
}

int records_from_matrix(p2g_ctx *ctx, const uint16_t *d_coeff, int nin, int nout,
                        uint32_t *d_recs)
{
    size_t n = static_cast<size_t>(nin) * nout;
    if (n == 0)
        return P2G_OK;
    records_matrix_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, ctx->stream>>>(
        d_coeff, nin, nout, d_recs);
    P2G_CUDA(cudaGetLastError());
    ++ctx->launches;
    return P2G_OK;
}

int records_par2(p2g_ctx *ctx, const uint16_t *d_consts, const uint32_t *d_exps, int nin,
                 int nout, uint32_t *d_recs)
{
    size_t n = static_cast<size_t>(nin) * nout;
    if (n == 0)
        return P2G_OK;
    records_par2_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, ctx->stream>>>(
        d_consts, d_exps, ctx->d_log, ctx->d_exp, nin, nout, d_recs);
    P2G_CUDA(cudaGetLastError());
    ++ctx->launches;
    return P2G_OK;
}

static int launch_kernel(cudaStream_t stream, const MuladdPlan &p, const uint32_t *planes,
                         const uint32_t *d_recs, int nin, int nout, int T,
                         uint8_t *const *d_dst, size_t S, int mode)
{
    KernelFn fn = kernel_for(p);
    size_t smem = smem_bytes(p);
    P2G_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    // T counts 1024-symbol plane tiles; the paired form runs 512-symbol tiles
    long long grid = static_cast<long long>(p.paired ? plan_tiles(p, S) : T) * p.nblk * p.nsplit;
    if (grid > 0x7fffffffLL) {
        set_error("muladd grid too large");
        return P2G_ERANGE;
    }
    fn<<<static_cast<unsigned>(grid), p.warps * 32, smem, stream>>>(
        planes, d_recs, nin, nout, T, p.nblk, p.nsplit, d_dst, S, mode);
    P2G_CUDA(cudaGetLastError());
    return P2G_OK;
}

int muladd_run(p2g_ctx *ctx, const uint8_t *const *d_src, int nin, uint8_t *const *d_dst,
               int nout, size_t S, const uint32_t *d_recs, int mode, const MuladdPlan *plan)
{
    if (nout <= 0)
        return P2G_OK;
    const int T = static_cast<int>((S + kTileBytes - 1) / kTileBytes);
    MuladdPlan p = plan ? *plan : choose_plan(ctx, nin, nout, S);
    if (!plan_valid(p, nin, nout, S)) {
        set_error("invalid muladd plan warps=%d ereg=%d nblk=%d nsplit=%d for %d outputs",
                  p.warps, p.ereg, p.nblk, p.nsplit, nout);
        return P2G_EINVAL;
    }
    if (nin == 0) {
        if (mode == 0) {
            dim3 g(static_cast<unsigned>(std::min<size_t>((S + 4095) / 4096, 1024)), nout);
            zero_slices<<<g, 256, 0, ctx->stream>>>(d_dst, nout, S);
            P2G_CUDA(cudaGetLastError());
            ++ctx->launches;
        }
        return P2G_OK;
    }
    size_t plane_bytes = static_cast<size_t>(nin) * T * kTileBytes;
    P2G_TRY(ctx->planes.ensure(plane_bytes));
    uint32_t *planes = ctx->planes.as<uint32_t>();
    size_t groups = static_cast<size_t>(nin) * T * 32;
    ctx->mark(1);
    slices_to_planes<<<static_cast<unsigned>((groups + 255) / 256), 256, 0, ctx->stream>>>(
        d_src, nin, T, S, planes);
    P2G_CUDA(cudaGetLastError());
    ++ctx->launches;
    if (p.nsplit > 1 && mode == 0) {
        dim3 g(static_cast<unsigned>(std::min<size_t>((S + 4095) / 4096, 1024)), nout);
        zero_slices<<<g, 256, 0, ctx->stream>>>(d_dst, nout, S);
        P2G_CUDA(cudaGetLastError());
        ++ctx->launches;
    }
    ctx->mark(2);
    P2G_TRY(launch_kernel(ctx->stream, p, planes, d_recs, nin, nout, T, d_dst, S, mode));
    ++ctx->launches;
    ctx->mark(3);
    return P2G_OK;
}

// Deterministic pseudo-random bytes for the tuner's synthetic slices.
__global__ void fill_pattern(uint32_t *p, size_t words, uint32_t seed)
{
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < words;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        uint32_t x = static_cast<uint32_t>(i) * 0x9E3779B9u ^ seed;
        x ^= x >> 16;
        x *= 0x7FEB352Du;
        x ^= x >> 15;
        x *= 0x846CA68Bu;
        x ^= x >> 16;
        p[i] = x;
    }
}

int fill_synthetic(cudaStream_t st, void *p, size_t bytes, uint32_t seed)
{
    if (bytes < 4)
        return P2G_OK;
    fill_pattern<<<1024, 256, 0, st>>>(static_cast<uint32_t *>(p), bytes / 4, seed);
    P2G_CUDA(cudaGetLastError());
    return P2G_OK;
}

int muladd_autotune(p2g_ctx *ctx, int nin, int nout, size_t S, int reps, MuladdPlan *best,
                    float *best_ms, int *tried)
{
    if (nin <= 0 || nout <= 0 || S == 0 || S % 2) {
        set_error("p2g_autotune: empty or odd-sized problem");
        return P2G_EINVAL;
    }
    reps = std::max(1, reps);
    const int T = static_cast<int>((S + kTileBytes - 1) / kTileBytes);
    const size_t slot = (S + 15) & ~static_cast<size_t>(15);
    // synthetic sources, outputs, coefficients, records, planes in context scratch
    P2G_TRY(ctx->in_copy.ensure(slot * nin));
    P2G_TRY(ctx->out_copy.ensure(slot * nout));
    P2G_TRY(ctx->coeffs.ensure(static_cast<size_t>(nin) * nout * 2 + 16));
    P2G_TRY(ctx->recs.ensure(record_bytes(nin, nout)));
    P2G_TRY(ctx->planes.ensure(static_cast<size_t>(nin) * T * kTileBytes));
    fill_pattern<<<1024, 256, 0, ctx->stream>>>(ctx->in_copy.as<uint32_t>(), slot * nin / 4, 1u);
    fill_pattern<<<256, 256, 0, ctx->stream>>>(ctx->coeffs.as<uint32_t>(),
                                               static_cast<size_t>(nin) * nout / 2, 7u);
    P2G_CUDA(cudaGetLastError());
    std::vector<const uint8_t *> sp(nin);
    std::vector<uint8_t *> dp(nout);
    for (int i = 0; i < nin; ++i)
        sp[i] = ctx->in_copy.as<uint8_t>() + i * slot;
    for (int o = 0; o < nout; ++o)
        dp[o] = ctx->out_copy.as<uint8_t>() + o * slot;
    const size_t ptr_bytes = (static_cast<size_t>(nin) + nout) * sizeof(void *);
    P2G_TRY(ctx->params.ensure(ptr_bytes));
    uint8_t *d_ptrs = ctx->params.as<uint8_t>();
    P2G_CUDA(cudaMemcpyAsync(d_ptrs, sp.data(), nin * sizeof(void *), cudaMemcpyHostToDevice,
                             ctx->stream));
    P2G_CUDA(cudaMemcpyAsync(d_ptrs + nin * sizeof(void *), dp.data(), nout * sizeof(void *),
                             cudaMemcpyHostToDevice, ctx->stream));
    const uint8_t *const *d_src = reinterpret_cast<const uint8_t *const *>(d_ptrs);
    uint8_t *const *d_dst = reinterpret_cast<uint8_t *const *>(d_ptrs + nin * sizeof(void *));
    P2G_TRY(records_from_matrix(ctx, ctx->coeffs.as<uint16_t>(), nin, nout, ctx->recs.as<uint32_t>()));
    size_t groups = static_cast<size_t>(nin) * T * 32;
    slices_to_planes<<<static_cast<unsigned>((groups + 255) / 256), 256, 0, ctx->stream>>>(
        d_src, nin, T, S, ctx->planes.as<uint32_t>());
    P2G_CUDA(cudaGetLastError());

    // candidates: each compiled (warps, ereg) shape at the fewest output blocks
    // it allows and the next two, times input splits that keep the grid
    // within a few waves
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    const bool small = nout <= kSmallOutputs;  // the table form is fixed by nout
    std::vector<MuladdPlan> cands;
    auto add = [&](const MuladdPlan &p) {
        if (!plan_valid(p, nin, nout, S))
            return;
        for (const MuladdPlan &q : cands)
            if (q.warps == p.warps && q.ereg == p.ereg && q.nblk == p.nblk &&
                q.nsplit == p.nsplit && q.psplit == p.psplit && q.paired == p.paired &&
                q.stage == p.stage)
                return;
        cands.push_back(p);
    };
    // the heuristic's own plan is always a candidate
    add(choose_plan(nullptr, nin, nout, S));
    for (const Variant &v0 : kVariants) {
        if (v0.small != small)
            continue;
        // one pass per (warps, psplit, form) family: its largest compiled ereg
        // sets the fewest output blocks; then the next two block counts, each
        // with the smallest compiled ereg that covers nout
        auto same = [&](const Variant &v) {
            return v.warps == v0.warps && v.psplit == v0.psplit && v.small == small &&
                   v.paired == v0.paired && v.stage == v0.stage;
        };
        bool first = true;
        int emax = 0;
        for (const Variant &v : kVariants) {
            if (same(v)) {
                emax = std::max(emax, v.ereg);
                if (&v < &v0)
                    first = false;
            }
        }
        if (!first)
            continue;
        // outputs per block for each unit of ereg
        const int G = v0.paired ? v0.warps * 2 : v0.warps / v0.psplit;
        const int nmin = (nout + G * emax - 1) / (G * emax);
        for (int nblk = nmin; nblk <= nmin + 2; ++nblk) {
            const int need = (nout + G * nblk - 1) / (G * nblk);
            int ereg = 0;
            for (const Variant &v : kVariants)
                if (same(v) && v.ereg >= need && (ereg == 0 || v.ereg < ereg))
                    ereg = v.ereg;
            if (ereg == 0)
                continue;
            MuladdPlan p;
            p.warps = v0.warps;
            p.psplit = v0.psplit;
            p.small = small;
            p.paired = v0.paired;
            p.stage = v0.stage;
            p.ereg = ereg;
            p.nblk = nblk;
            const int tiles = plan_tiles(p, S);
            for (int ns : {1, 2, 3, 4, 6, 8, 12, 16}) {
                p.nsplit = ns;
                const long long ctas = static_cast<long long>(tiles) * nblk * ns;
                if (ns > 1 && (nin / ns < 8 || ctas > 8LL * sms))
                    continue;
                add(p);
            }
        }
    }
    cudaEvent_t e0, e1;
    P2G_CUDA(cudaEventCreate(&e0));
    P2G_CUDA(cudaEventCreate(&e1));
    float best_t = 1e30f;
    MuladdPlan best_p = choose_plan(nullptr, nin, nout, S);
    int rc = P2G_OK;
    for (const MuladdPlan &p : cands) {
        // warm-up launch, then the best of `reps` timed launches
        rc = launch_kernel(ctx->stream, p, ctx->planes.as<uint32_t>(), ctx->recs.as<uint32_t>(),
                           nin, nout, T, d_dst, S, 1);
        if (rc != P2G_OK)
            break;
        float t = 1e30f;
        for (int r = 0; r < reps && rc == P2G_OK; ++r) {
            cudaEventRecord(e0, ctx->stream);
            rc = launch_kernel(ctx->stream, p, ctx->planes.as<uint32_t>(),
                               ctx->recs.as<uint32_t>(), nin, nout, T, d_dst, S, 1);
            cudaEventRecord(e1, ctx->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                set_error("p2g_autotune: %s", cudaGetErrorString(cudaGetLastError()));
                rc = P2G_ECUDA;
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            t = std::min(t, ms);
        }
        if (rc != P2G_OK)
            break;
        if (t < best_t) {
            best_t = t;
            best_p = p;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    P2G_TRY(rc);
    ctx->plans[plan_key(nin, nout, S)] = best_p;
    *best = best_p;
    *best_ms = best_t;
    *tried = static_cast<int>(cands.size());
    return P2G_OK;
}

// ---- batches of independent problems -----------------------------------

template <class P>
__device__ __forceinline__ int find_prob(const P *probs, int np, unsigned long long gid)
{
    int lo = 0, hi = np - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (probs[mid].first <= gid)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__global__ void batch_planes_kernel(const PlanesProb *__restrict__ probs, int np,
                                    unsigned long long total)
{
    const unsigned long long gid = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (gid >= total)
        return;
    const PlanesProb p = probs[find_prob(probs, np, gid)];
    const unsigned long long local = gid - p.first;
    const int lane = static_cast<int>(local & 31);
    const unsigned long long it = local >> 5;
    const int t = static_cast<int>(it % p.T);
    const int i = static_cast<int>(it / p.T);
    uint32_t x[16];
    load_group(p.src[i], p.S, static_cast<size_t>(t) * kTileBytes + lane * 64, x);
    transpose16x2(x);
    uint32_t *P = p.planes + it * 512 + lane;
#pragma unroll
    for (int b = 0; b < 16; ++b)
        P[b * 32] = x[b];
}

__global__ void batch_records_kernel(const RecProb *__restrict__ probs, int np,
                                     unsigned long long total, const uint16_t *__restrict__ glog,
                                     const uint16_t *__restrict__ gexp)
{
    const unsigned long long gid = static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (gid >= total)
        return;
    const RecProb p = probs[find_prob(probs, np, gid)];
    const unsigned long long local = gid - p.first;
    const int o = static_cast<int>(local % p.nout);
    const int i = static_cast<int>(local / p.nout);
    uint32_t c;
    if (p.coeff) {
        c = p.coeff[static_cast<size_t>(o) * p.nin + i];
    } else {
        const uint32_t base = p.consts[i], e = p.exps[o];
        if (base == 0)
            c = e == 0 ? 1u : 0u;
        else if (e == 0)
            c = 1u;
        else
            c = gexp[static_cast<uint32_t>((static_cast<uint64_t>(glog[base]) * e) % 65535u)];
    }
    write_record(p.recs, local, c, p.small != 0);
}

__global__ void batch_zero_kernel(uint8_t *const *__restrict__ ptrs,
                                  const unsigned long long *__restrict__ bytes, int n)
{
    for (int j = blockIdx.y; j < n; j += gridDim.y) {
        uint8_t *d = ptrs[j];
        const size_t S = bytes[j];
        for (size_t x = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) * 16; x < S;
             x += static_cast<size_t>(gridDim.x) * blockDim.x * 16) {
            if (x + 16 <= S)
                *reinterpret_cast<uint4 *>(d + x) = make_uint4(0, 0, 0, 0);
            else
                for (size_t y = x; y < S; y += 2)
                    *reinterpret_cast<uint16_t *>(d + y) = 0;
        }
    }
}

__global__ void batch_copy_kernel(const uint8_t *const *__restrict__ src,
                                  uint8_t *const *__restrict__ dst,
                                  const unsigned long long *__restrict__ bytes, int n)
{
    for (int j = blockIdx.y; j < n; j += gridDim.y) {
        const uint8_t *s = src[j];
        uint8_t *d = dst[j];
        const size_t S = bytes[j];
        for (size_t x = (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) * 16; x < S;
             x += static_cast<size_t>(gridDim.x) * blockDim.x * 16) {
            if (x + 16 <= S)
                *reinterpret_cast<uint4 *>(d + x) = *reinterpret_cast<const uint4 *>(s + x);
            else
                for (size_t y = x; y < S; y += 2)
                    *reinterpret_cast<uint16_t *>(d + y) = *reinterpret_cast<const uint16_t *>(s + y);
        }
    }
}

static unsigned grid_for(unsigned long long n)
{
    return static_cast<unsigned>((n + 255) / 256);
}

int batch_planes(cudaStream_t st, const PlanesProb *d, int np, unsigned long long total)
{
    if (!total)
        return P2G_OK;
    batch_planes_kernel<<<grid_for(total), 256, 0, st>>>(d, np, total);
    P2G_CUDA(cudaGetLastError());
    return P2G_OK;
}

int batch_records(cudaStream_t st, const uint16_t *glog, const uint16_t *gexp, const RecProb *d,
                  int np, unsigned long long total)
{
    if (!total)
        return P2G_OK;
    batch_records_kernel<<<grid_for(total), 256, 0, st>>>(d, np, total, glog, gexp);
    P2G_CUDA(cudaGetLastError());
    return P2G_OK;
}

int batch_zero(cudaStream_t st, uint8_t *const *ptrs, const unsigned long long *bytes, int n)
{
    if (n <= 0)
        return P2G_OK;
    batch_zero_kernel<<<dim3(16, std::min(n, 4096)), 256, 0, st>>>(ptrs, bytes, n);
    P2G_CUDA(cudaGetLastError());
    return P2G_OK;
}

int batch_copy(cudaStream_t st, const uint8_t *const *src, uint8_t *const *dst,
               const unsigned long long *bytes, int n)
{
    if (n <= 0)
        return P2G_OK;
    batch_copy_kernel<<<dim3(16, std::min(n, 4096)), 256, 0, st>>>(src, dst, bytes, n);
    P2G_CUDA(cudaGetLastError());
    return P2G_OK;
}

// Shared memory of the persistent kernel: the largest of its forms'.
static size_t batch_smem_bytes()
{
    MuladdPlan w, sm, pr;
    w.warps = sm.warps = pr.warps = kBatchWarps;
    w.ereg = 13;
    sm.ereg = 3;
    sm.small = true;
    pr.ereg = 13;
    pr.paired = true;
    pr.stage = 2;
    return std::max({smem_bytes(w), smem_bytes(sm), smem_bytes(pr)});
}

int batch_muladd(cudaStream_t st, int grid, const BatchProb *probs, const BatchItem *items,
                 int nitems, int *counter, const volatile int *abort)
{
    if (nitems <= 0)
        return P2G_OK;
    const size_t smem = batch_smem_bytes();
    P2G_CUDA(cudaFuncSetAttribute(muladd_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    muladd_persistent<<<grid, kBatchWarps * 32, smem, st>>>(probs, items, nitems, counter, abort);
    P2G_CUDA(cudaGetLastError());
    return P2G_OK;
}

size_t planes_bytes_fixed(int nin, size_t S)
{
    return static_cast<size_t>(nin) * ((S + kTileBytes - 1) / kTileBytes) * kTileBytes;
}

int records_matrix_fixed(cudaStream_t stream, const uint16_t *d_coeff, int nin, int nout,
                         uint32_t *d_recs)
{
    size_t n = static_cast<size_t>(nin) * nout;
    if (n == 0)
        return P2G_OK;
    records_matrix_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0, stream>>>(
        d_coeff, nin, nout, d_recs);
    P2G_CUDA(cudaGetLastError());
    return P2G_OK;
}

int muladd_run_fixed(cudaStream_t stream, int sm_count, const uint8_t *const *d_src, int nin,
                     uint8_t *const *d_dst, int nout, size_t S, const uint32_t *d_recs,
                     uint32_t *d_planes)
{
    if (nout <= 0)
        return P2G_OK;
    p2g_ctx probe;  // choose_plan reads only sm_count
    probe.sm_count = sm_count;
    const MuladdPlan p = choose_plan(&probe, nin, nout, S);
    const int T = static_cast<int>((S + kTileBytes - 1) / kTileBytes);
    dim3 zg(static_cast<unsigned>(std::min<size_t>((S + 4095) / 4096, 1024)), nout);
    if (nin == 0 || p.nsplit > 1) {
        zero_slices<<<zg, 256, 0, stream>>>(d_dst, nout, S);
        P2G_CUDA(cudaGetLastError());
        if (nin == 0)
            return P2G_OK;
    }
    size_t groups = static_cast<size_t>(nin) * T * 32;
    slices_to_planes<<<static_cast<unsigned>((groups + 255) / 256), 256, 0, stream>>>(
        d_src, nin, T, S, d_planes);
    P2G_CUDA(cudaGetLastError());
    return launch_kernel(stream, p, d_planes, d_recs, nin, nout, T, d_dst, S, 0);
}

}  // namespace p2g
