// invert.cuh -- device Gauss-Jordan over GF(2^16).
#pragma once
#include "common.cuh"

namespace p2g {

// Scratch of one inversion: the augmented matrix and a status word.
struct GjWork {
    DevBuf &M;
    DevBuf &status;
};

// Inverts the m x m matrix given either as PAR2 constants of the missing
// slices and recovery exponents (A[row][col] = cmiss[col]^exps[row]) or, when
// d_A is non-null, as a dense row-major device matrix.  d_inv receives A^-1
// (row-major m x m).  h_exps (optional) is a host copy of the exponents: when
// they are a permutation of consecutive values, the closed-form Vandermonde
// inverse replaces the elimination.  Singularity is reported by gj_status.
int gj_invert(p2g_ctx *ctx, GjWork &w, int m, const uint16_t *d_cmiss, const uint32_t *d_exps,
              const uint32_t *h_exps, const uint16_t *d_A, uint16_t *d_inv);

// Waits for the inversion and reads its status (1 = singular).
int gj_status(p2g_ctx *ctx, GjWork &w, int *singular);

}  // namespace p2g
