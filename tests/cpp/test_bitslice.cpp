// Host check of the coefficient records the multiply-accumulate kernel reads
// (par2-rs_b200/csrc/bitslice.cuh), both table forms, without a GPU.
//
// For a group of 32 random symbols and a coefficient c, the tables are built
// from the symbols' 16 bit planes as the kernel builds them, the record's row
// offsets are followed in the order the kernel's ldmatrix.x4 lookups use them
// (lane group m supplies the row of matrix m), and the XOR of the rows must
// be the bit planes of c * symbol for every symbol (GF(2^16), 0x1100B, the
// multiplication of galois/core.rs:175-200 written as shift-and-add).
// Prints "ok <cases>" and exits 0, or the first mismatch and exits 1.
#include <stdio.h>

#include <random>

#include "../../par2-rs_b200/csrc/bitslice.cuh"

using namespace p2g;

static uint32_t gf_mul(uint32_t a, uint32_t b)
{
    uint32_t r = 0;
    for (int i = 0; i < 16; ++i) {
        if (b & (1u << i))
            r ^= a;
        a = gf_times_x(a);
    }
    return r;
}

// 32 symbols -> 16 plane words (and back: transpose16x2 is an involution)
static void to_planes(const uint16_t sym[32], uint32_t planes[16])
{
    for (int j = 0; j < 16; ++j)
        planes[j] = static_cast<uint32_t>(sym[2 * j]) | (static_cast<uint32_t>(sym[2 * j + 1]) << 16);
    transpose16x2(planes);
}

// rows[r] = XOR of planes base + b for every bit b set in r (r < 2^bits)
static void fill(uint32_t *rows, const uint32_t *planes, int base, int bits)
{
    for (uint32_t r = 0; r < (1u << bits); ++r) {
        uint32_t v = 0;
        for (int b = 0; b < bits; ++b)
            if (r & (1u << b))
                v ^= planes[base + b];
        rows[r] = v;
    }
}

// The 8 + 8 form: T0 rows 0-255 over planes 0-7, T1 rows 256-511 over 8-15;
// lookup p (0..7) fetches rows {T0, T1} of planes 2p and 2p + 1.
static void apply_wide(const uint32_t planes[16], uint32_t c, uint32_t out[16])
{
    uint32_t tab[512], w[kRecordWords];
    fill(tab, planes, 0, 8);
    fill(tab + 256, planes, 8, 8);
    make_record(c, w);
    for (int j = 0; j < 16; ++j)
        out[j] = 0;
    for (int p = 0; p < 8; ++p) {
        uint32_t d[4];
        for (int m = 0; m < 4; ++m) {
            // byte p of class m's two record words; odd classes index T1
            const uint32_t row = (w[2 * m + (p >> 2)] >> (8 * (p & 3))) & 0xFFu;
            d[m] = tab[row + ((m & 1) ? 256u : 0u)];
        }
        out[2 * p] ^= d[0] ^ d[1];
        out[2 * p + 1] ^= d[2] ^ d[3];
    }
}

// The small form: T0 rows 0-63 over planes 0-5, T1 rows 64-95 over 6-10, T2
// rows 96-127 over 11-15; lookup k (0..11) fetches rows 4k..4k+3 of the
// sequence s = 3j + t, row s going to output plane s / 3.
static void apply_small(const uint32_t planes[16], uint32_t c, uint32_t out[16])
{
    uint32_t tab[128], w[kRecordWordsSmall];
    fill(tab, planes, 0, 6);
    fill(tab + 64, planes, 6, 5);
    fill(tab + 96, planes, 11, 5);
    make_record_small(c, w);
    for (int j = 0; j < 16; ++j)
        out[j] = 0;
    for (int k = 0; k < 12; ++k)
        for (int m = 0; m < 4; ++m) {
            const uint32_t word = w[6 * m + (k >> 1)];
            const uint32_t off = (k & 1) ? (word >> 16) : (word & 0xFFFFu);
            if (off % kRowBytes || off / kRowBytes >= 128) {
                printf("small record of %u: offset %u out of the table\n", c, off);
                return;
            }
            out[(4 * k + m) / 3] ^= tab[off / kRowBytes];
        }
}

int main()
{
    std::mt19937 rng(20261204);
    int cases = 0;
    for (int it = 0; it < 4000; ++it) {
        uint32_t c = rng() & 0xFFFFu;
        if (it < 6)
            c = (const uint32_t[]){0u, 1u, 2u, 3u, 0x8000u, 0xFFFFu}[it];
        uint16_t sym[32], prod[32];
        for (int i = 0; i < 32; ++i) {
            sym[i] = static_cast<uint16_t>(rng());
            prod[i] = static_cast<uint16_t>(gf_mul(sym[i], c));
        }
        uint32_t planes[16], want[16];
        to_planes(sym, planes);
        to_planes(prod, want);
        for (int form = 0; form < 2; ++form) {
            uint32_t got[16];
            (form ? apply_small : apply_wide)(planes, c, got);
            for (int j = 0; j < 16; ++j)
                if (got[j] != want[j]) {
                    printf("%s record of c=%u: plane %d is %08x, want %08x\n",
                           form ? "small" : "wide", c, j, got[j], want[j]);
                    return 1;
                }
            ++cases;
        }
    }
    printf("ok %d\n", cases);
    return 0;
}
