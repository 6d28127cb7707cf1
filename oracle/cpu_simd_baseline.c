/*
 * cpu_simd_baseline.c -- TEST / MEASUREMENT INFRASTRUCTURE ONLY.
 *
 * The par2-rs CPU fast path restated in C so that it can be timed on the host
 * cores next to the CUDA library (the Rust reference cannot be built here:
 * no cargo/rustc in this image).  It is the strategy par2-rs selects on an
 * AVX2 host -- "AVX2-Shuffle", priority Optimal, registered before
 * AVX2-PCLMUL (galois/simd/x86/mod.rs:13-26, galois/simd/mod.rs:171-189):
 *
 *   - data in the "shuffle2x" split layout: in every 32-byte block of 16
 *     symbols the 16 low bytes occupy the first 128-bit lane and the 16 high
 *     bytes the second (galois/simd/x86/avx2.rs:571-625);
 *   - per coefficient, four 32-byte nibble tables built from the
 *     lo/hi-byte products of the four nibble positions
 *     (galois/core.rs:116-163, avx2.rs:222-250);
 *   - per 16 symbols: 4 byte shuffles, one lane swap, 3 XORs
 *     (avx2.rs:632-677);
 *   - encode threading as StreamingEncoder::flush_batch: recovery slices in
 *     batches of 4..8 per task, data slices in batches of 16..128
 *     (par2_rs.rs:88-126, :816-870);
 *   - region kernel with 4 destinations x 4 sources per pass
 *     (avx2.rs:686-821).
 *
 * Results are checked against par2_oracle.c by the tests; bench.py times it.
 */
#include <immintrin.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define POLY 0x1100Bu

static uint16_t gl[65536];
static uint16_t ge[131072];
static int ready = 0;

static void tables_init(void)
{
    if (ready)
        return;
    uint32_t b = 1;
    for (uint32_t l = 0; l < 65535; ++l) {
        ge[l] = ge[l + 65535] = (uint16_t)b;
        gl[b] = (uint16_t)l;
        b <<= 1;
        if (b & 0x10000u)
            b ^= POLY;
    }
    ready = 1;
}

static inline uint16_t mul(uint16_t a, uint16_t b)
{
    return (a && b) ? ge[(uint32_t)gl[a] + gl[b]] : 0;
}

/* Split-layout nibble tables for one coefficient.  t0/t1 are applied to the
 * low/high nibble of every byte; in the low-byte lane they hold the products'
 * low bytes ("same lane"), in the high-byte lane the products' high bytes;
 * s0/s1 hold the bytes that must cross to the other lane. */
typedef struct {
    __m256i t0, t1, s0, s1;
} split_tables;

static split_tables make_tables(uint16_t c)
{
    uint8_t lo[4][16], hi[4][16];
    for (int pos = 0; pos < 4; ++pos)
        for (int x = 0; x < 16; ++x) {
            uint16_t p = mul((uint16_t)(x << (4 * pos)), c);
            lo[pos][x] = (uint8_t)p;
            hi[pos][x] = (uint8_t)(p >> 8);
        }
    uint8_t t0[32], t1[32], s0[32], s1[32];
    /* lane 0 (low bytes): nibble positions 0 (low nibble) and 1 (high nibble)
     * lane 1 (high bytes): nibble positions 2 and 3 */
    memcpy(t0, lo[0], 16); memcpy(t0 + 16, hi[2], 16);
    memcpy(t1, lo[1], 16); memcpy(t1 + 16, hi[3], 16);
    memcpy(s0, hi[0], 16); memcpy(s0 + 16, lo[2], 16);
    memcpy(s1, hi[1], 16); memcpy(s1 + 16, lo[3], 16);
    split_tables t;
    t.t0 = _mm256_loadu_si256((const __m256i *)t0);
    t.t1 = _mm256_loadu_si256((const __m256i *)t1);
    t.s0 = _mm256_loadu_si256((const __m256i *)s0);
    t.s1 = _mm256_loadu_si256((const __m256i *)s1);
    return t;
}

static inline __m256i mul_split(const split_tables *t, __m256i d, __m256i mask)
{
    __m256i nl = _mm256_and_si256(d, mask);
    __m256i nh = _mm256_and_si256(_mm256_srli_epi16(d, 4), mask);
    __m256i same = _mm256_xor_si256(_mm256_shuffle_epi8(t->t0, nl), _mm256_shuffle_epi8(t->t1, nh));
    __m256i cross = _mm256_xor_si256(_mm256_shuffle_epi8(t->s0, nl), _mm256_shuffle_epi8(t->s1, nh));
    cross = _mm256_permute2x128_si256(cross, cross, 0x01);
    return _mm256_xor_si256(same, cross);
}

/* interleaved LE u16 -> split layout, per 32-byte block (in place) */
static void to_split(uint8_t *p, size_t bytes)
{
    const __m256i sep = _mm256_setr_epi8(0, 2, 4, 6, 8, 10, 12, 14, 1, 3, 5, 7, 9, 11, 13, 15,
                                         0, 2, 4, 6, 8, 10, 12, 14, 1, 3, 5, 7, 9, 11, 13, 15);
    for (size_t o = 0; o + 32 <= bytes; o += 32) {
        __m256i v = _mm256_loadu_si256((const __m256i *)(p + o));
        v = _mm256_shuffle_epi8(v, sep);
        v = _mm256_permute4x64_epi64(v, 0xD8);
        _mm256_storeu_si256((__m256i *)(p + o), v);
    }
}

static void from_split(uint8_t *p, size_t bytes)
{
    const __m256i join = _mm256_setr_epi8(0, 8, 1, 9, 2, 10, 3, 11, 4, 12, 5, 13, 6, 14, 7, 15,
                                          0, 8, 1, 9, 2, 10, 3, 11, 4, 12, 5, 13, 6, 14, 7, 15);
    for (size_t o = 0; o + 32 <= bytes; o += 32) {
        __m256i v = _mm256_loadu_si256((const __m256i *)(p + o));
        v = _mm256_permute4x64_epi64(v, 0xD8);
        v = _mm256_shuffle_epi8(v, join);
        _mm256_storeu_si256((__m256i *)(p + o), v);
    }
}

/* dst ^= c * src over split-layout data; a ragged tail (< 32 bytes) stays
 * interleaved and is done with scalar products, as avx2.rs:670-676 does. */
static void muladd_split(uint8_t *dst, const uint8_t *src, size_t bytes, uint16_t c)
{
    if (!c)
        return;
    split_tables t = make_tables(c);
    const __m256i mask = _mm256_set1_epi8(0x0f);
    size_t o = 0;
    for (; o + 32 <= bytes; o += 32) {
        __m256i d = _mm256_loadu_si256((const __m256i *)(src + o));
        __m256i a = _mm256_loadu_si256((const __m256i *)(dst + o));
        _mm256_storeu_si256((__m256i *)(dst + o), _mm256_xor_si256(a, mul_split(&t, d, mask)));
    }
    for (; o + 2 <= bytes; o += 2) {
        uint16_t s = (uint16_t)(src[o] | (src[o + 1] << 8));
        uint16_t p = mul(s, c);
        dst[o] ^= (uint8_t)p;
        dst[o + 1] ^= (uint8_t)(p >> 8);
    }
}

typedef struct {
    const uint8_t *src;     /* k split-layout slices */
    const uint16_t *coeff;  /* [k][r] */
    uint8_t *rec;           /* r split-layout slices */
    size_t k, r, bytes, rbatch, dbatch;
    size_t task_lo, task_hi; /* recovery-batch index range of this thread */
} enc_job;

static void *enc_worker(void *arg)
{
    enc_job *j = (enc_job *)arg;
    for (size_t d0 = 0; d0 < j->k; d0 += j->dbatch) {
        size_t d1 = d0 + j->dbatch < j->k ? d0 + j->dbatch : j->k;
        for (size_t t = j->task_lo; t < j->task_hi; ++t) {
            size_t e0 = t * j->rbatch, e1 = e0 + j->rbatch < j->r ? e0 + j->rbatch : j->r;
            for (size_t i = d0; i < d1; ++i)
                for (size_t e = e0; e < e1; ++e)
                    muladd_split(j->rec + e * j->bytes, j->src + i * j->bytes, j->bytes,
                                 j->coeff[i * j->r + e]);
        }
    }
    return NULL;
}

static size_t clampz(size_t v, size_t lo, size_t hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* Encode k contiguous slices into r recovery slices with exponents 0..r-1
 * (par2_rs.rs:687-902) on `nthreads` threads.  `src` is not modified (it is
 * copied into split-layout batch buffers as process_block does). */
void pb_encode(const uint8_t *src, size_t k, size_t bytes, size_t r, uint8_t *out, int nthreads)
{
    tables_init();
    if (nthreads < 1)
        nthreads = 1;
    /* constants and coefficient matrix c_i^e by repeated multiplication */
    uint16_t *c = (uint16_t *)malloc(k * 2);
    size_t have = 0;
    for (uint64_t n = 1; have < k; ++n)
        if (n % 3 && n % 5 && n % 17 && n % 257)
            c[have++] = ge[n % 65535];
    uint16_t *coeff = (uint16_t *)malloc(k * r * 2);
    for (size_t i = 0; i < k; ++i) {
        uint16_t v = 1;
        for (size_t e = 0; e < r; ++e) {
            coeff[i * r + e] = v;
            v = mul(v, c[i]);
        }
    }
    uint8_t *split = (uint8_t *)aligned_alloc(64, ((k * bytes + 63) / 64) * 64);
    memcpy(split, src, k * bytes);
    for (size_t i = 0; i < k; ++i)
        to_split(split + i * bytes, bytes);
    memset(out, 0, r * bytes);
    /* batch sizes: par2_rs.rs:88-126 */
    size_t ncpu = (size_t)nthreads;
    size_t base = r >= 100 ? ncpu * 8 : (r >= 50 ? ncpu * 4 : ncpu * 2);
    size_t dbatch = clampz(base, 16, 128);
    size_t rbatch = clampz(r / ncpu ? r / ncpu : 1, 4, 8);
    size_t ntasks = (r + rbatch - 1) / rbatch;
    pthread_t *th = (pthread_t *)malloc(ncpu * sizeof(pthread_t));
    enc_job *jobs = (enc_job *)malloc(ncpu * sizeof(enc_job));
    for (size_t t = 0; t < ncpu; ++t) {
        jobs[t] = (enc_job){split, coeff, out, k, r, bytes, rbatch, dbatch,
                            ntasks * t / ncpu, ntasks * (t + 1) / ncpu};
        pthread_create(&th[t], NULL, enc_worker, &jobs[t]);
    }
    for (size_t t = 0; t < ncpu; ++t)
        pthread_join(th[t], NULL);
    for (size_t e = 0; e < r; ++e)
        from_split(out + e * bytes, bytes);
    free(th);
    free(jobs);
    free(split);
    free(coeff);
    free(c);
}

typedef struct {
    uint8_t *const *dst;
    const uint8_t *const *src;
    const uint16_t *coeff; /* [ndst][nsrc] */
    size_t ndst, nsrc, lo, hi;
} reg_job;

/* One thread's byte range [lo, hi) of every slice, processed in 128 KiB
 * regions with 4 destinations x 4 sources per pass (avx2.rs:686-821,
 * region/mod.rs:40). */
static void *reg_worker(void *arg)
{
    reg_job *j = (reg_job *)arg;
    const __m256i mask = _mm256_set1_epi8(0x0f);
    const size_t REGION = 128 * 1024;
    for (size_t r0 = j->lo; r0 < j->hi; r0 += REGION) {
        size_t r1 = r0 + REGION < j->hi ? r0 + REGION : j->hi;
        for (size_t d0 = 0; d0 < j->ndst; d0 += 4) {
            size_t dn = j->ndst - d0 < 4 ? j->ndst - d0 : 4;
            for (size_t s0 = 0; s0 < j->nsrc; s0 += 4) {
                size_t sn = j->nsrc - s0 < 4 ? j->nsrc - s0 : 4;
                split_tables tb[4][4];
                int nz[4][4], any = 0;
                for (size_t a = 0; a < dn; ++a)
                    for (size_t b = 0; b < sn; ++b) {
                        uint16_t c = j->coeff[(d0 + a) * j->nsrc + s0 + b];
                        nz[a][b] = c != 0;
                        any |= nz[a][b];
                        if (c)
                            tb[a][b] = make_tables(c);
                    }
                if (!any)
                    continue;
                for (size_t o = r0; o + 32 <= r1; o += 32) {
                    __m256i d[4];
                    for (size_t b = 0; b < sn; ++b)
                        d[b] = _mm256_loadu_si256((const __m256i *)(j->src[s0 + b] + o));
                    for (size_t a = 0; a < dn; ++a) {
                        __m256i acc = _mm256_loadu_si256((const __m256i *)(j->dst[d0 + a] + o));
                        for (size_t b = 0; b < sn; ++b)
                            if (nz[a][b])
                                acc = _mm256_xor_si256(acc, mul_split(&tb[a][b], d[b], mask));
                        _mm256_storeu_si256((__m256i *)(j->dst[d0 + a] + o), acc);
                    }
                }
            }
        }
    }
    return NULL;
}

/* Region multiply-accumulate over split-layout slices of `bytes` (multiple of
 * 32), byte range split statically across threads as repair.rs:907-970 does
 * with its chunk ranges. */
void pb_muladd_region_split(uint8_t *const *dst, size_t ndst, const uint8_t *const *src,
                            size_t nsrc, const uint16_t *coeff, size_t bytes, int nthreads)
{
    tables_init();
    if (nthreads < 1)
        nthreads = 1;
    size_t blocks = bytes / 32;
    pthread_t *th = (pthread_t *)malloc(nthreads * sizeof(pthread_t));
    reg_job *jobs = (reg_job *)malloc(nthreads * sizeof(reg_job));
    for (int t = 0; t < nthreads; ++t) {
        jobs[t] = (reg_job){dst, src, coeff, ndst, nsrc, blocks * t / nthreads * 32,
                            blocks * (t + 1) / nthreads * 32};
        pthread_create(&th[t], NULL, reg_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t)
        pthread_join(th[t], NULL);
    free(th);
    free(jobs);
}

/* Layout converters exposed for the tests. */
void pb_to_split(uint8_t *p, size_t bytes) { to_split(p, bytes); }
void pb_from_split(uint8_t *p, size_t bytes) { from_split(p, bytes); }
