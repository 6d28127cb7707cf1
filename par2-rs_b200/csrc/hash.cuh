// hash.cuh -- per-slice MD5 + CRC32 launcher.
#pragma once
#include "common.cuh"

namespace p2g {

// The four slicing-by-4 tables of CRC-32/ISO-HDLC (reflected 0xEDB88320).
void crc32_tables(uint32_t tab[4][256]);
size_t hash_smem_bytes();

// MD5 (16 bytes per slice, d_md5) and CRC32 (d_crc) of n slices of S bytes;
// d_slices is a DEVICE array of 16-byte aligned device pointers.
int hash_run(p2g_ctx *ctx, const uint8_t *const *d_slices, int n, size_t S, uint8_t *d_md5,
             uint32_t *d_crc);

}  // namespace p2g
