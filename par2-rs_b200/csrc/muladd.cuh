// muladd.cuh -- host launchers of the GF(2^16) region multiply-accumulate.
#pragma once
#include "common.cuh"

namespace p2g {

// The plan for a problem: the context's tuned plan for this shape if there
// is one, else a heuristic (8 warps, as many outputs per warp as fit).
MuladdPlan choose_plan(const p2g_ctx *ctx, int nin, int nout, size_t slice_bytes);
bool plan_valid(const MuladdPlan &p, int nin, int nout, size_t slice_bytes);
// The compiled (warps, outputs per group, warps per group) shapes; returns
// their number.
int muladd_variants(int *warps, int *eregs, int *psplits, int cap);

// Times every candidate plan for (nin, nout, S) on synthetic data in the
// context's scratch, caches the fastest in ctx->plans and returns it.
int muladd_autotune(p2g_ctx *ctx, int nin, int nout, size_t S, int reps, MuladdPlan *best,
                    float *best_ms, int *tried);

// Coefficient records [nin][nout][16 words] from a row-major matrix
// coeff[nout][nin] (coefficients[dst][src] of galois/region/mod.rs:78-82).
int records_from_matrix(p2g_ctx *ctx, const uint16_t *d_coeff, int nin, int nout,
                        uint32_t *d_recs);

// Records of the PAR2 encoding matrix: coefficient (i, o) = consts[i]^exps[o]
// (par2_rs.rs:707-719).
int records_par2(p2g_ctx *ctx, const uint16_t *d_consts, const uint32_t *d_exps, int nin,
                 int nout, uint32_t *d_recs);

// dst[o] (^)= sum_i coeff(i, o) * src[i] over slices of slice_bytes.
// d_src / d_dst are DEVICE arrays of 16-byte aligned device pointers.
// mode 0 stores, mode 1 XORs into the existing contents.
int muladd_run(p2g_ctx *ctx, const uint8_t *const *d_src, int nin, uint8_t *const *d_dst,
               int nout, size_t slice_bytes, const uint32_t *d_recs, int mode,
               const MuladdPlan *plan = nullptr);

// The same work as records_from_matrix / muladd_run (store mode) on a given
// stream with caller-provided scratch: nothing is allocated.  d_planes must
// hold planes_bytes_fixed(nin, S) bytes.
size_t planes_bytes_fixed(int nin, size_t S);
int records_matrix_fixed(cudaStream_t stream, const uint16_t *d_coeff, int nin, int nout,
                         uint32_t *d_recs);
int muladd_run_fixed(cudaStream_t stream, int sm_count, const uint8_t *const *d_src, int nin,
                     uint8_t *const *d_dst, int nout, size_t S, const uint32_t *d_recs,
                     uint32_t *d_planes);

}  // namespace p2g
