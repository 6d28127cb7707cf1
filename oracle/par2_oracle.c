/*
 * par2_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the par2-rs erasure-coding path: the parity
 * reference the CUDA library's results are compared with (tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py).  Nothing in
 * the product links or calls it.
 *
 * Parity pinning: the restatement is checked against the QuickPar fixture set
 * bundled with par2-rs (tests/data/testdata*.par2): all 60 recovery slices,
 * all 200 IFSC (MD5, CRC32) entries and the byte-exact repair scenarios of
 * tests/external_multiblock_repair.rs.  The derived vectors live in
 * tests/golden/ together with the script that extracted them.
 *
 * Every function cites the par2-rs source it restates (paths relative to the
 * par2-rs repository root).
 *
 * MD5 and CRC-32 come from OpenSSL libcrypto and zlib.  par2-rs itself uses
 * the crates md-5 0.10.6 and crc32fast 1.5.0 (Cargo.lock); both compute
 * RFC 1321 MD5 and CRC-32/ISO-HDLC (reflected poly 0xEDB88320, init and
 * xorout 0xFFFFFFFF), which is exactly what libcrypto MD5() and zlib crc32()
 * compute.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <openssl/md5.h>
#include <zlib.h>

#define PO_GF_SIZE 65536u
#define PO_POLY 0x1100Bu

static uint16_t po_log[PO_GF_SIZE];
static uint16_t po_exp[PO_GF_SIZE * 2];
static int po_ready = 0;

/* galois/core.rs:49-91 init_tables: generator 2, poly 0x1100B, exp table
 * doubled so exp[log a + log b] needs no reduction, log(0) stored as 0. */
void po_init(void)
{
    if (po_ready)
        return;
    uint32_t b = 1;
    for (uint32_t l = 0; l < PO_GF_SIZE - 1; ++l) {
        po_exp[l] = (uint16_t)b;
        po_exp[l + PO_GF_SIZE - 1] = (uint16_t)b;
        po_log[b] = (uint16_t)l;
        b <<= 1;
        if (b & 0x10000u)
            b ^= PO_POLY;
    }
    po_log[0] = 0;
    po_ready = 1;
}

/* galois/core.rs:175-189 gf_mul */
uint16_t po_gf_mul(uint16_t a, uint16_t b)
{
    po_init();
    if (a == 0 || b == 0)
        return 0;
    return po_exp[(uint32_t)po_log[a] + po_log[b]];
}

/* galois/core.rs:205-230 gf_div; returns -1 for a zero divisor (the
 * reference's None), 0 otherwise. */
int po_gf_div(uint16_t a, uint16_t b, uint16_t *out)
{
    po_init();
    if (b == 0)
        return -1;
    if (a == 0) {
        *out = 0;
        return 0;
    }
    uint32_t la = po_log[a], lb = po_log[b];
    uint32_t l = la >= lb ? la - lb : la + (PO_GF_SIZE - 1) - lb;
    *out = po_exp[l];
    return 0;
}

/* galois/core.rs:242-258 gf_pow: (log a * n) mod 65535, 0^0 = 1. */
uint16_t po_gf_pow(uint16_t a, uint64_t n)
{
    po_init();
    if (a == 0)
        return n == 0 ? 1 : 0;
    if (n == 0)
        return 1;
    uint64_t l = ((uint64_t)po_log[a] * n) % (PO_GF_SIZE - 1);
    return po_exp[l];
}

/* The erasure matrix of par2_rs.rs:346-353 (and V of :404-412):
 * out[row][col] = gf_pow(bases[col], exps[row]) for ne rows x nb columns. */
void po_power_matrix(const uint16_t *bases, size_t nb, const uint32_t *exps, size_t ne,
                     uint16_t *out)
{
    po_init();
    for (size_t e = 0; e < ne; ++e)
        for (size_t j = 0; j < nb; ++j)
            out[e * nb + j] = po_gf_pow(bases[j], exps[e]);
}

/* par2_rs.rs:64-76 generate_par2_constants: c_i = 2^n for the i-th n >= 1
 * with n not divisible by 3, 5, 17 or 257. */
void po_par2_constants(size_t k, uint16_t *out)
{
    po_init();
    size_t have = 0;
    uint64_t n = 1;
    while (have < k) {
        if (n % 3 && n % 5 && n % 17 && n % 257)
            out[have++] = po_gf_pow(2, n);
        ++n;
    }
}

static inline uint16_t rd16(const uint8_t *p) { return (uint16_t)(p[0] | (p[1] << 8)); }
static inline void wr16(uint8_t *p, uint16_t v) { p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); }

/* dst[x] ^= c * src[x] over n LE u16 symbols (galois/scalar.rs:22-29). */
static void muladd_bytes(uint8_t *dst, const uint8_t *src, size_t nsym, uint16_t c)
{
    if (c == 0)
        return;
    uint32_t lc = po_log[c];
    for (size_t x = 0; x < nsym; ++x) {
        uint16_t s = rd16(src + 2 * x);
        if (s)
            wr16(dst + 2 * x, rd16(dst + 2 * x) ^ po_exp[po_log[s] + lc]);
    }
}

/* Encode: rec_e = sum_i c_i^{exp_e} * D_i over k contiguous slices of
 * slice_bytes (even).  Restates the math of the streaming encoder,
 * par2_rs.rs:687-772 (coefficients c_i^e) and :816-870 (accumulation);
 * finalize (:880-902) writes the u16 symbols back little-endian.  `out`
 * receives r contiguous slices. */
void po_encode(const uint8_t *src, size_t k, size_t slice_bytes,
               const uint32_t *exps, size_t r, uint8_t *out)
{
    po_init();
    uint16_t *c = (uint16_t *)malloc(k * sizeof(uint16_t));
    po_par2_constants(k, c);
    memset(out, 0, r * slice_bytes);
    size_t nsym = slice_bytes / 2;
    for (size_t e = 0; e < r; ++e)
        for (size_t i = 0; i < k; ++i)
            muladd_bytes(out + e * slice_bytes, src + i * slice_bytes, nsym,
                         po_gf_pow(c[i], exps[e]));
    free(c);
}

/* Region multiply-accumulate with the semantics of
 * galois/scalar.rs:82-113 gf_muladd_region_scalar:
 * dsts[d][off..off+len] ^= sum_s coeffs[d*nsrc+s] * srcs[s][off..off+len]. */
void po_muladd_region(uint16_t *const *dsts, size_t ndst,
                      const uint16_t *const *srcs, size_t nsrc,
                      const uint16_t *coeffs, size_t off, size_t len)
{
    po_init();
    for (size_t d = 0; d < ndst; ++d)
        for (size_t s = 0; s < nsrc; ++s) {
            uint16_t c = coeffs[d * nsrc + s];
            if (!c)
                continue;
            uint32_t lc = po_log[c];
            for (size_t x = off; x < off + len; ++x) {
                uint16_t v = srcs[s][x];
                if (v)
                    dsts[d][x] ^= po_exp[po_log[v] + lc];
            }
        }
}

/* The elimination record of par2_rs.rs:319-422
 * compute_reconstruction_transform. */
typedef struct {
    size_t m;
    size_t *row_order;   /* m */
    uint16_t *scale;     /* m */
    uint16_t *elim;      /* m*m, row-major [r][k] */
} po_transform;

static void transform_free(po_transform *t)
{
    free(t->row_order);
    free(t->scale);
    free(t->elim);
}

/* Gauss-Jordan on A (m x m, row-major, destroyed), recording row swaps,
 * pivots and factors exactly as par2_rs.rs:355-401 does: a row swap only when
 * the pivot is zero (first non-zero row below), the pivot row divided by the
 * pivot, every other row reduced.  Returns -1 for "Singular matrix". */
static int eliminate(uint16_t *A, size_t m, po_transform *t)
{
    t->m = m;
    t->row_order = (size_t *)malloc(m * sizeof(size_t));
    t->scale = (uint16_t *)malloc(m * sizeof(uint16_t));
    t->elim = (uint16_t *)calloc(m * m, sizeof(uint16_t));
    for (size_t i = 0; i < m; ++i) {
        t->row_order[i] = i;
        t->scale[i] = 1;
    }
    uint16_t *tmp = (uint16_t *)malloc(m * sizeof(uint16_t));
    for (size_t k = 0; k < m; ++k) {
        if (A[k * m + k] == 0) {
            size_t r = k + 1;
            while (r < m && A[r * m + k] == 0)
                ++r;
            if (r == m) {
                free(tmp);
                return -1;
            }
            memcpy(tmp, A + k * m, m * 2);
            memcpy(A + k * m, A + r * m, m * 2);
            memcpy(A + r * m, tmp, m * 2);
            size_t so = t->row_order[k];
            t->row_order[k] = t->row_order[r];
            t->row_order[r] = so;
            uint16_t ss = t->scale[k];
            t->scale[k] = t->scale[r];
            t->scale[r] = ss;
            memcpy(tmp, t->elim + k * m, m * 2);
            memcpy(t->elim + k * m, t->elim + r * m, m * 2);
            memcpy(t->elim + r * m, tmp, m * 2);
        }
        uint16_t pivot = A[k * m + k];
        t->scale[k] = pivot;
        if (pivot != 1)
            for (size_t j = k; j < m; ++j)
                if (A[k * m + j])
                    po_gf_div(A[k * m + j], pivot, &A[k * m + j]);
        for (size_t r = 0; r < m; ++r) {
            if (r == k)
                continue;
            uint16_t f = A[r * m + k];
            t->elim[r * m + k] = f;
            if (!f)
                continue;
            for (size_t j = k; j < m; ++j)
                if (A[k * m + j])
                    A[r * m + j] ^= po_gf_mul(A[k * m + j], f);
        }
    }
    free(tmp);
    return 0;
}

/* Replays the recorded elimination on m row vectors of nsym symbols
 * (par2_rs.rs:618-655): acc[k] /= pivot_k, then acc[r] ^= f[r][k]*acc[k]
 * for r < k and r > k. */
static void replay(const po_transform *t, uint16_t **acc, size_t nsym)
{
    size_t m = t->m;
    for (size_t k = 0; k < m; ++k) {
        uint16_t p = t->scale[k];
        if (p != 1)
            for (size_t s = 0; s < nsym; ++s)
                if (acc[k][s])
                    po_gf_div(acc[k][s], p, &acc[k][s]);
        for (size_t r = 0; r < m; ++r) {
            if (r == k)
                continue;
            uint16_t f = t->elim[r * m + k];
            if (!f)
                continue;
            uint32_t lf = po_log[f];
            for (size_t s = 0; s < nsym; ++s)
                if (acc[k][s])
                    acc[r][s] ^= po_exp[po_log[acc[k][s]] + lf];
        }
    }
}

/* Inverse of an m x m matrix by the reference's elimination: the recorded
 * row operations applied to the identity (the same replay the repair path
 * applies to data).  Returns -1 when singular. */
int po_invert(size_t m, const uint16_t *A_in, uint16_t *Ainv)
{
    po_init();
    uint16_t *A = (uint16_t *)malloc(m * m * 2);
    memcpy(A, A_in, m * m * 2);
    po_transform t;
    int rc = eliminate(A, m, &t);
    free(A);
    if (rc) {
        transform_free(&t);
        return rc;
    }
    /* acc rows start as the identity rows permuted by row_order
     * (par2_rs.rs:486-498 places recovery row `o` at the position where
     * row_order holds `o`). */
    uint16_t **acc = (uint16_t **)malloc(m * sizeof(uint16_t *));
    for (size_t i = 0; i < m; ++i)
        acc[i] = Ainv + i * m;
    memset(Ainv, 0, m * m * 2);
    for (size_t pos = 0; pos < m; ++pos)
        acc[pos][t.row_order[pos]] = 1;
    replay(&t, acc, m);
    free(acc);
    transform_free(&t);
    return 0;
}

/* Repair, restating par2_rs.rs:319-422 (transform) and :442-675
 * (reconstruct_streaming_chunk over the whole slice):
 *   - k data slices of slice_bytes, contiguous in `data`; the slices listed in
 *     `missing` (m of them, ascending global index) are ignored;
 *   - m recovery slices in `rec` (contiguous) with exponents rec_exps, in the
 *     order repair.rs:585-604 chooses them (lowest exponents first);
 *   - A[row][col] = c_{missing[col]}^{rec_exps[row]}, V[row][j] =
 *     c_{present[j]}^{rec_exps[row]};
 *   - acc = R (row-permuted), acc ^= V * present, replay elimination;
 *   - out (m contiguous slices) receives missing[row] in row order.
 * Returns 0, or -1 for "Singular matrix". */
int po_reconstruct(size_t k, size_t slice_bytes, const uint64_t *missing, size_t m,
                   const uint8_t *data, const uint32_t *rec_exps, const uint8_t *rec,
                   uint8_t *out, int ref_row_quirk, uint64_t *nswaps)
{
    po_init();
    size_t nsym = slice_bytes / 2;
    uint16_t *c = (uint16_t *)malloc(k * 2);
    po_par2_constants(k, c);
    uint16_t *A = (uint16_t *)malloc(m * m * 2);
    for (size_t row = 0; row < m; ++row)
        for (size_t col = 0; col < m; ++col)
            A[row * m + col] = po_gf_pow(c[missing[col]], rec_exps[row]);
    po_transform t;
    int rc = eliminate(A, m, &t);
    free(A);
    if (rc) {
        transform_free(&t);
        free(c);
        return rc;
    }
    uint16_t **acc = (uint16_t **)malloc(m * sizeof(uint16_t *));
    for (size_t i = 0; i < m; ++i)
        acc[i] = (uint16_t *)calloc(nsym, 2);
    for (size_t orig = 0; orig < m; ++orig) {
        size_t pos = 0;
        while (t.row_order[pos] != orig)
            ++pos;
        for (size_t s = 0; s < nsym; ++s)
            acc[pos][s] = rd16(rec + orig * slice_bytes + 2 * s);
    }
    /* acc[pos] ^= V[row][j] * present_j over the present data slices in
     * ascending index order.  Mathematically row = row_order[pos] (the
     * recovery equation whose R sits at pos).  The reference multiplies
     * accumulators[pos] by vandermonde_coeffs[pos] instead
     * (par2_rs.rs:561-599 against :486-498), which differs only when the
     * elimination swapped rows; ref_row_quirk=1 restates that behaviour.
     * *nswaps reports how many positions moved. */
    uint64_t moved = 0;
    for (size_t pos = 0; pos < m; ++pos)
        moved += t.row_order[pos] != pos;
    if (nswaps)
        *nswaps = moved;
    uint8_t *is_missing = (uint8_t *)calloc(k, 1);
    for (size_t i = 0; i < m; ++i)
        is_missing[missing[i]] = 1;
    for (size_t pos = 0; pos < m; ++pos)
        for (size_t i = 0; i < k; ++i) {
            if (is_missing[i])
                continue;
            size_t row = ref_row_quirk ? pos : t.row_order[pos];
            uint16_t v = po_gf_pow(c[i], rec_exps[row]);
            if (!v)
                continue;
            uint32_t lv = po_log[v];
            const uint8_t *src = data + i * slice_bytes;
            for (size_t s = 0; s < nsym; ++s) {
                uint16_t d = rd16(src + 2 * s);
                if (d)
                    acc[pos][s] ^= po_exp[po_log[d] + lv];
            }
        }
    replay(&t, acc, nsym);
    for (size_t row = 0; row < m; ++row)
        for (size_t s = 0; s < nsym; ++s)
            wr16(out + row * slice_bytes + 2 * s, acc[row][s]);
    for (size_t i = 0; i < m; ++i)
        free(acc[i]);
    free(acc);
    free(is_missing);
    transform_free(&t);
    free(c);
    return 0;
}

/* hash/mod.rs:22-27 compute_md5 (md-5 crate == RFC 1321). */
void po_md5(const uint8_t *data, size_t n, uint8_t out[16])
{
    MD5(data, n, out);
}

/* crc32fast::hash == CRC-32/ISO-HDLC == zlib crc32. */
uint32_t po_crc32(const uint8_t *data, size_t n)
{
    uLong c = crc32(0L, Z_NULL, 0);
    while (n) {
        uInt chunk = n > (1u << 30) ? (1u << 30) : (uInt)n;
        c = crc32(c, data, chunk);
        data += chunk;
        n -= chunk;
    }
    return (uint32_t)c;
}

/* Per-slice MD5 + CRC32 of n contiguous, already zero-padded slices, the
 * IFSC entries of creator.rs:397-409 and the checks of verify.rs:610-648. */
void po_hash_slices(const uint8_t *data, size_t n, size_t slice_bytes,
                    uint8_t *md5s, uint32_t *crcs)
{
    for (size_t i = 0; i < n; ++i) {
        po_md5(data + i * slice_bytes, slice_bytes, md5s + 16 * i);
        crcs[i] = po_crc32(data + i * slice_bytes, slice_bytes);
    }
}

/* creator.rs:30-67 calculate_block_size. */
uint64_t po_calculate_block_size(uint64_t total)
{
    const uint64_t MINB = 2048, MAXB = 4ull * 1024 * 1024, TARGET = 2000, MAXN = 65535;
    if (total == 0)
        return MINB;
    uint64_t bs = total / TARGET;
    uint64_t min_field = (total + MAXN - 1) / MAXN;
    if (bs % 4)
        bs = (bs / 4 + 1) * 4;
    uint64_t min_block = min_field > MINB ? min_field : MINB;
    if (min_block % 4)
        min_block = (min_block / 4 + 1) * 4;
    if (min_block > MAXB) {
        bs = min_block;
    } else {
        if (bs < MINB)
            bs = MINB;
        if (bs > MAXB)
            bs = MAXB;
        if (bs < min_block)
            bs = min_block;
    }
    return bs;
}

/* creator.rs:324-331: recovery_bytes = floor(data_bytes * (pct_f32 as f64 /
 * 100)); r = ceil(recovery_bytes / block_size). */
uint64_t po_recovery_count(uint64_t data_blocks, uint64_t block_size, float pct)
{
    double rb = (double)(data_blocks * block_size) * ((double)pct / 100.0);
    uint64_t recovery_bytes = (uint64_t)rb;
    return (recovery_bytes + block_size - 1) / block_size;
}
