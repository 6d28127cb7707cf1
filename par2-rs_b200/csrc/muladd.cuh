// muladd.cuh -- host launchers of the GF(2^16) region multiply-accumulate.
#pragma once
#include "bitslice.cuh"
#include "common.cuh"

namespace p2g {

// Problems of at most this many outputs use the small-output tables (6 + 5 +
// 5 planes: 128 table rows per input instead of 512, 48 row reads per
// coefficient instead of 32; cheaper below ~24 outputs) and 24-word records;
// larger ones the 8 + 8 tables and 8-word records.  The form follows from
// the output count alone, so records built for a problem always match the
// kernel that reads them.
constexpr int kSmallOutputs = 24;
inline int record_words(int nout) { return nout <= kSmallOutputs ? kRecordWordsSmall : kRecordWords; }
// Bytes of the records of an nin x nout problem.
inline size_t record_bytes(size_t nin, int nout)
{
    return nin * static_cast<size_t>(nout) * record_words(nout) * 4;
}

// Tile forms of the persistent batch kernel, chosen per problem: the 8 + 8
// tables over 1024-symbol tiles (8 warps x 13 outputs, 104 per item), the
// small-output tables (8 warps x 3, 24 per item) and the paired form over
// 512-symbol tiles (8 warps x 13 output pairs, 208 per item, two inputs per
// barrier).
enum BatchForm : int { kFormWide = 0, kFormSmall = 1, kFormPaired = 2, kBatchForms = 3 };
inline int batch_block(int form)
{
    return form == kFormSmall ? 24 : form == kFormPaired ? 208 : 104;
}
// column bytes one item covers
inline size_t batch_tile_bytes(int form) { return form == kFormPaired ? 1024 : 2048; }
inline int batch_record_words(int form)
{
    return form == kFormSmall ? kRecordWordsSmall : kRecordWords;
}
// Shared-memory wavefronts one input of an item of nb outputs costs: table
// rows built plus plane reads, then table reads and record loads per output.
inline double batch_item_cost(int form, int nb)
{
    if (form == kFormSmall)
        return 144.0 + 50.0 * nb;
    if (form == kFormPaired)
        return 320.0 + 17.0 * nb;
    return 576.0 + 34.0 * nb;
}
// The problem classes the batch autotuner keys on: outputs 1-24, 25-104,
// 105-208, more; slices up to 16 KiB or larger.
inline int batch_class(int nout, size_t S)
{
    const int c = nout <= 24 ? 0 : nout <= 104 ? 1 : nout <= 208 ? 2 : 3;
    return 2 * c + (S > (16u << 10) ? 1 : 0);
}
// A form's validity for a problem: the small tables take at most 24 outputs.
inline bool batch_form_valid(int form, int nout)
{
    return form >= 0 && form < kBatchForms && (form != kFormSmall || nout <= 24);
}

// One multiply-accumulate problem of a batch (device-resident description).
struct BatchProb {
    const uint32_t *planes;  // [nin][T][512]
    const uint32_t *recs;    // [nin][nout][batch_record_words(form)]
    uint8_t *const *dst;     // nout device pointers
    size_t S;                // bytes per slice
    int nin, nout, T, nblk, nsplit, mode, form;
};
// One work item of a batch: (problem, column tile of the problem's form,
// output block, input split).
struct BatchItem {
    int prob, t, ob, split;
};
constexpr int kBatchWarps = 8;

// Bit-plane conversion of one problem of a batch; `first` is the problem's
// first thread in the batched grid (nin * T * 32 threads each).
struct PlanesProb {
    const uint8_t *const *src;
    uint32_t *planes;
    size_t S;
    int nin, T;
    unsigned long long first;
};
// Records of one problem: coefficient (i, o) from a [nout][nin] matrix, or
// consts[i]^exps[o]; nin * nout threads each.
struct RecProb {
    const uint16_t *consts;
    const uint32_t *exps;
    const uint16_t *coeff;
    uint32_t *recs;
    int nin, nout;
    int small;  // small-output (24-word) records
    unsigned long long first;
};

int batch_planes(cudaStream_t st, const PlanesProb *d, int np, unsigned long long total);
int batch_records(cudaStream_t st, const uint16_t *glog, const uint16_t *gexp, const RecProb *d,
                  int np, unsigned long long total);
int batch_zero(cudaStream_t st, uint8_t *const *ptrs, const unsigned long long *bytes, int n);
int batch_copy(cudaStream_t st, const uint8_t *const *src, uint8_t *const *dst,
               const unsigned long long *bytes, int n);
// The persistent kernel over `nitems` items (longest first) with `grid` CTAs,
// each item run in its problem's form; *counter must be zero.  A CTA takes no further item once it has seen the
// device word *abort non-zero (polled every 4th item).
int batch_muladd(cudaStream_t st, int grid, const BatchProb *probs, const BatchItem *items,
                 int nitems, int *counter, const volatile int *abort);

// The plan for a problem: the context's tuned plan for this shape if there
// is one, else a heuristic (8 warps, as many outputs per warp as fit).
MuladdPlan choose_plan(const p2g_ctx *ctx, int nin, int nout, size_t slice_bytes);
// Column tiles of plan p over slices of S bytes (1024 symbols each, 512 in
// the paired form); a launch runs tiles x output blocks x input splits CTAs.
int plan_tiles(const MuladdPlan &p, size_t S);
// CTAs of plan p the device runs at once (SMs x CTAs resident per SM).
int plan_slots(const p2g_ctx *ctx, const MuladdPlan &p);
bool plan_valid(const MuladdPlan &p, int nin, int nout, size_t slice_bytes);
// The compiled (warps, outputs per group, warps per group) shapes; returns
// their number.
int muladd_variants(int *warps, int *eregs, int *psplits, int cap);

// Deterministic pseudo-random words over bytes / 4 words at p (device).
int fill_synthetic(cudaStream_t st, void *p, size_t bytes, uint32_t seed);

// Times every candidate plan for (nin, nout, S) on synthetic data in the
// context's scratch, caches the fastest in ctx->plans and returns it.
int muladd_autotune(p2g_ctx *ctx, int nin, int nout, size_t S, int reps, MuladdPlan *best,
                    float *best_ms, int *tried);

// Coefficient records [nin][nout][record_words(nout)] from a row-major matrix
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
