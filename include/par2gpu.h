/*
 * par2gpu.h -- C ABI of the B200 (sm_100a) GF(2^16) erasure-coding library.
 *
 * The entry points are what a par2-rs backend binds through FFI.  Each one
 * names the par2-rs interface it stands in for (paths are relative to the
 * par2-rs repository root).  All symbols are plain C: pointers, sizes and
 * integer status codes, no C++ or torch types.
 *
 * Conventions
 *   - Slices are byte arrays; a GF(2^16) symbol is a little-endian u16
 *     (par2-rs galois/mod.rs:178-223).  Slice lengths in bytes must be even.
 *   - Every call returns P2G_OK (0) or a negative P2G_E* code; the message of
 *     the last failure on the calling thread is p2g_last_error().
 *   - Pointers are host pointers unless P2G_DEVICE_PTRS is passed, in which
 *     case every slice pointer (not the pointer arrays themselves, which are
 *     always host arrays) is a device pointer on the context's device.
 *   - The caller owns all buffers.  A context serialises its calls with an
 *     internal lock, so one context may be shared by threads (as par2-rs
 *     shares its Send + Sync strategy object, galois/simd/mod.rs:24); for
 *     concurrency give each thread its own context.
 */
#ifndef PAR2GPU_H
#define PAR2GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define P2G_OK 0
#define P2G_EINVAL (-1)     /* bad argument (odd length, null pointer, k = 0 ...) */
#define P2G_ENOMEM (-2)     /* device or pinned allocation failed */
#define P2G_ECUDA (-3)      /* a CUDA runtime call failed */
#define P2G_ESINGULAR (-4)  /* "Singular matrix" (par2_rs.rs:361-370) */
#define P2G_ETIMEOUT (-5)   /* a bounded device wait gave up */
#define P2G_ENODEV (-6)     /* no usable sm_100 device */
#define P2G_ERANGE (-7)     /* a size beyond a documented maximum */
#define P2G_ECANCELED (-8)  /* the batch was cancelled (p2g_batch_cancel) */

/* flags */
#define P2G_DEVICE_PTRS 0x1u /* slice pointers are device pointers */

/* strategy priority values, par2-rs galois/simd/mod.rs:14-21 */
#define P2G_PRIORITY_FALLBACK 0
#define P2G_PRIORITY_BASIC 10
#define P2G_PRIORITY_ENHANCED 20
#define P2G_PRIORITY_ADVANCED 30
#define P2G_PRIORITY_OPTIMAL 40

typedef struct p2g_ctx p2g_ctx;

/* Message of the last failed call on this thread ("" if none). */
const char *p2g_last_error(void);

/* Library / device context.  Replaces the lazily initialised global state of
 * par2-rs (galois/core.rs:49-91 tables, galois/simd/mod.rs:237-242 registry)
 * with an explicit handle bound to one CUDA device. */
int p2g_create(int device, p2g_ctx **out);
int p2g_destroy(p2g_ctx *ctx);

/* Runs the context's work on a caller-supplied CUDA stream (a cudaStream_t
 * passed as void*; NULL restores the context's own non-blocking stream, so
 * pass cudaStreamLegacy to mean the legacy default stream).  Calls still
 * return only when their work is complete.  No counterpart in par2-rs: it is
 * the device-side plumbing a host integration needs. */
int p2g_set_stream(p2g_ctx *ctx, void *cuda_stream);

/* Per-phase device times of the last call, measured with CUDA events on the
 * stream the kernels run on when timing is enabled.  No counterpart in
 * par2-rs (its tracing is host-side, par2_rs.rs:220-226). */
typedef struct {
    float ms_records;  /* coefficient records */
    float ms_planes;   /* slices -> bit planes */
    float ms_kernel;   /* the main kernel: multiply-accumulate, or hashing */
    float ms_total;    /* first to last event of the call */
    int launches;      /* kernels launched by the call */
} p2g_timing;
int p2g_set_timing(p2g_ctx *ctx, int enable);
int p2g_last_timing(p2g_ctx *ctx, p2g_timing *out);

/* Tile shape of the multiply-accumulate kernel for one problem shape:
 * warps per CTA; warps_per_group warps share one group of outputs_per_group
 * outputs (each holding 16 / warps_per_group of the 16 bit planes); output
 * blocks of (warps / warps_per_group) * outputs_per_group outputs; input
 * splits (partial sums folded with atomic XOR); the kernel time it measured
 * at (ms, set by p2g_autotune); the column tile: 1024 symbols (0 means the
 * same), or 512 for the paired form, in which each warp accumulates
 * outputs_per_group outputs (an even number), half a warp per output, and a
 * CTA builds each input's lookup tables once for up to 208 outputs; and the
 * inputs a CTA takes between two of its barriers (0 or 1; 2 in the paired
 * form, which then holds four tables).  No counterpart in par2-rs, whose
 * strategies fix their blocking (avx2.rs:700-701 DEST_BATCH / SRC_BATCH). */
typedef struct {
    int warps;
    int outputs_per_group;
    int warps_per_group;
    int output_blocks;
    int input_splits;
    float ms;
    int tile_symbols;
    int inputs_per_stage;
} p2g_plan;

/* Autotuner: times every compiled tile shape (and output-block / input-split
 * choice) of the multiply-accumulate kernel for nin inputs x nout outputs of
 * slice_bytes on synthetic data in the context's scratch (best of `reps`
 * launches each) and makes the fastest the context's plan for that shape.
 * Untuned shapes use a heuristic plan. */
int p2g_autotune(p2g_ctx *ctx, size_t nin, size_t nout, size_t slice_bytes, int reps,
                 p2g_plan *best);

/* Pins the plan for one shape (P2G_EINVAL if the shape is not compiled or
 * does not cover nout outputs).  Problems of at most 24 outputs run the
 * small-output kernel (three smaller lookup tables per input), compiled for
 * 8 warps x 1-3 outputs per group, warps_per_group 1; larger problems the
 * 8 + 8 table kernel (8 warps x 1-13, 12 warps x 4/6/7/8, 16 warps x 2-5,
 * and 16 warps x 8/10/12 with warps_per_group 2) or its paired form
 * (tile_symbols 512: 8 warps x 14-26 even, 12 warps x 16 outputs per
 * warp; with inputs_per_stage 2: 8 warps x 14/18/22/26, 12 warps x 16). */
int p2g_set_plan(p2g_ctx *ctx, size_t nin, size_t nout, size_t slice_bytes,
                 const p2g_plan *plan);

/* GaloisSimdStrategy::{name, is_available, priority}
 * (galois/simd/mod.rs:26-33): "CUDA-sm100a", available iff an sm_100 device
 * is present, priority P2G_PRIORITY_OPTIMAL. */
int p2g_strategy_info(const char **name, int *priority, int *available);

/* GaloisSimdStrategy::mul_slice (galois/simd/mod.rs:39): data[i] = c * data[i]
 * over n u16 symbols. */
int p2g_mul_slice(p2g_ctx *ctx, uint16_t c, uint16_t *data, size_t n, uint32_t flags);

/* GaloisSimdStrategy::muladd (galois/simd/mod.rs:45):
 * dst[i] ^= c * src[i] over n u16 symbols. */
int p2g_muladd(p2g_ctx *ctx, uint16_t *dst, const uint16_t *src, size_t n, uint16_t c,
               uint32_t flags);

/* GaloisSimdStrategy::muladd_region (galois/simd/mod.rs:51-58), also the
 * target of gf_muladd_block_regions (galois/region/mod.rs:195-242):
 *   dsts[d][off .. off+len) ^= sum_s coeff_rows[d][s] * srcs[s][off .. off+len)
 * with coeff_rows[d] an array of nsrc coefficients (coefficients[dst][src]),
 * off and len in u16 units. */
int p2g_muladd_region(p2g_ctx *ctx, uint16_t *const *dsts, size_t ndst,
                      const uint16_t *const *srcs, size_t nsrc,
                      const uint16_t *const *coeff_rows, size_t off_u16, size_t len_u16,
                      uint32_t flags);

/* GaloisSimdStrategy's shuffle2x hooks (galois/simd/mod.rs:68-127), which
 * par2-rs calls around its accumulation loops: prepare_shuffle2x on every
 * accumulator and buffered source (par2_rs.rs:727-731, :792-800, :503-506,
 * :540-553), muladd_shuffle2x / muladd_region_shuffle2x inside the loops
 * (par2_rs.rs:859-864 via galois/mod.rs:328-349; :588-599 via
 * galois/region/mod.rs:195-242) and finish_shuffle2x before an accumulator
 * is read (par2_rs.rs:884-888, :610-613).  Between its prepare and its finish
 * a buffer's contents belong to the strategy: here a device copy holds them
 * (prepare uploads the buffer and does not modify it), the multiply-
 * accumulates are recorded and run as multi-output kernel launches -- at a
 * prepare once about 3 ms of kernel work or 1 GiB of sources is waiting, and
 * at every finish -- and finish writes the accumulator's result back into the
 * caller's buffer.  Buffers are identified by their start address and must
 * cover off + len symbols.  A call whose destination was not prepared runs at
 * once (after the recorded work), as the interface's default would.  Safe
 * from many threads at once (the recording calls take no context lock);
 * recorded work runs on the context's stream. */
int p2g_supports_shuffle2x(void);
int p2g_prepare_shuffle2x(p2g_ctx *ctx, uint16_t *data, size_t n);
int p2g_muladd_shuffle2x(p2g_ctx *ctx, uint16_t *dst, const uint16_t *src, size_t n, uint16_t c);
int p2g_muladd_region_shuffle2x(p2g_ctx *ctx, uint16_t *const *dsts, size_t ndst,
                                const uint16_t *const *srcs, size_t nsrc,
                                const uint16_t *const *coeff_rows, size_t off_u16,
                                size_t len_u16);
int p2g_finish_shuffle2x(p2g_ctx *ctx, uint16_t *data, size_t n);

/* PAR2 input-slice constants (par2_rs.rs:64-76 generate_par2_constants):
 * out[i] = 2^n_i, n_i the i-th n >= 1 not divisible by 3, 5, 17 or 257. */
int p2g_par2_constants(size_t k, uint16_t *out);

/* Recovery-slice creation, the work of Par2ReedSolomon::create_streaming_encoder
 * + StreamingEncoder::{process_block, flush_batch, finalize}
 * (par2_rs.rs:687-902): out[e] = sum_i c_i^{exps[e]} * src[i] for k input
 * slices of slice_bytes (the caller zero-pads the last slice of a file, as
 * creator.rs:386-395 does).  out receives r recovery slice bodies. */
int p2g_encode(p2g_ctx *ctx, const uint8_t *const *src, size_t k, size_t slice_bytes,
               const uint32_t *exps, size_t r, uint8_t *const *out, uint32_t flags);

/* Exact GF(2^16) inverse of an m x m matrix (row-major host arrays), by
 * Gauss-Jordan on the device -- the elimination par2-rs performs in
 * Par2ReedSolomon::compute_reconstruction_transform (par2_rs.rs:355-401).
 * Returns P2G_ESINGULAR ("Singular matrix", :361-370) when A has no inverse. */
int p2g_invert(p2g_ctx *ctx, size_t m, const uint16_t *A, uint16_t *inv);

/* The repair decode matrix A^-1 (m x m, row-major) for
 * A[row][col] = c_{missing[col]}^{exps[row]}, c_i the PAR2 constants of k
 * input slices (par2_rs.rs:346-353). */
int p2g_reconstruction_matrix(p2g_ctx *ctx, size_t k, const uint64_t *missing, size_t m,
                              const uint32_t *exps, uint16_t *inv);

/* Repair: Par2ReedSolomon::compute_reconstruction_transform +
 * reconstruct_streaming_chunk over whole slices (par2_rs.rs:319-675).
 *   k           input slices in the set (fixes the constants c_i)
 *   missing[m]  strictly ascending global indices of the slices to rebuild
 *   present     the k - m other input slices, ascending index order
 *   exps[m], recovery[m]  the recovery slices used; par2-rs takes the m
 *               lowest exponents (repair.rs:585-604)
 *   out[m]      out[j] receives slice missing[j]
 * Computes out = A^-1 (R ^ V * present) with V[row][j] = c_{present_j}^{exps[row]}.
 * Returns P2G_ESINGULAR when A is singular. */
int p2g_repair(p2g_ctx *ctx, size_t k, size_t slice_bytes, const uint64_t *missing, size_t m,
               const uint8_t *const *present, const uint32_t *exps,
               const uint8_t *const *recovery, uint8_t *const *out, uint32_t flags);

/* Per-slice MD5 (RFC 1321) and CRC-32/ISO-HDLC of n slices of slice_bytes
 * each, the IFSC checksums par2-rs computes with the md-5 and crc32fast
 * crates (creator.rs:397-409, hash/md5_crc32_fused.rs:28-88).  md5_out
 * receives 16 bytes per slice, crc_out one value per slice (host arrays). */
int p2g_hash_slices(p2g_ctx *ctx, const uint8_t *const *slices, size_t n, size_t slice_bytes,
                    uint8_t *md5_out, uint32_t *crc_out, uint32_t flags);

/* Slice verification of verify_file_blocks (verify.rs:610-648): ok_out[i] = 1
 * when slice i has the expected CRC32 and the expected MD5, else 0 (the
 * reference rejects on CRC before computing MD5; the verdict is the same). */
int p2g_verify_slices(p2g_ctx *ctx, const uint8_t *const *slices, size_t n, size_t slice_bytes,
                      const uint8_t *md5_expect, const uint32_t *crc_expect, uint8_t *ok_out,
                      uint32_t flags);

/* ---- batches of independent jobs ---------------------------------------
 * Many recovery sets of uneven sizes in one execution: per phase ONE
 * persistent kernel takes (job, column tile, output block, input split)
 * items, longest first, from a device queue -- instead of per-set launches
 * that leave most SMs idle for small sets.  No counterpart in par2-rs (it
 * handles one set per process); the per-job work is that of p2g_encode,
 * p2g_repair and p2g_verify_slices. */
#define P2G_JOB_CREATE 1
#define P2G_JOB_REPAIR 2
#define P2G_JOB_VERIFY 3

typedef struct {
    int kind;                    /* P2G_JOB_* */
    size_t k;                    /* input slices of the recovery set (fixes the constants) */
    size_t slice_bytes;
    size_t col_begin, col_end;   /* byte range of every slice this job covers; col_end = 0
                                    means the whole slice; col_begin a multiple of 2048
                                    (column ranges are independent: the work is
                                    column-separable).  VERIFY jobs take whole slices. */
    const uint8_t *const *src;   /* CREATE, VERIFY: k slices; REPAIR: the k - n present ones */
    size_t n;                    /* CREATE: recovery slices; REPAIR: missing slices */
    const uint32_t *exps;        /* CREATE, REPAIR: n exponents */
    const uint64_t *missing;     /* REPAIR: n ascending slice indices */
    const uint8_t *const *recovery; /* REPAIR: n recovery slices */
    const uint16_t *inverse;     /* REPAIR: optional host n x n decode matrix
                                    (p2g_reconstruction_matrix); NULL: computed here */
    uint8_t *const *out;         /* CREATE, REPAIR: n output slices */
    uint8_t *md5_out;            /* VERIFY: host, 16 bytes per slice */
    uint32_t *crc_out;           /* VERIFY: host, one per slice */
    int status;                  /* set by p2g_batch_run: P2G_OK, P2G_ESINGULAR, ... */
} p2g_job;

typedef struct p2g_batch p2g_batch;

#define P2G_BATCH_GRAPH 0x2u /* capture the device work into a CUDA graph for replay */

/* Prepares a batch: validates the jobs, computes the decode matrices of
 * REPAIR jobs (a singular one marks that job P2G_ESINGULAR and drops it),
 * sizes and allocates the batch's scratch, uploads its work tables and, with
 * P2G_BATCH_GRAPH, captures the device work into a CUDA graph.  Slice
 * pointers are device pointers; `jobs` must outlive the batch. */
int p2g_batch_create(p2g_ctx *ctx, p2g_job *jobs, size_t njobs, uint32_t flags,
                     p2g_batch **out);
/* Runs (or replays) the batch and waits for it; fills statuses and hashes. */
int p2g_batch_run(p2g_batch *batch);
/* Starts the batch without waiting; p2g_batch_wait completes it. */
int p2g_batch_launch(p2g_batch *batch);
int p2g_batch_poll(p2g_batch *batch, int *done);
int p2g_batch_wait(p2g_batch *batch);
/* Cancels a launched batch from any thread: a copy engine raises a device
 * word that the persistent kernels poll, so they take no further work items
 * (those running finish; nothing waits), and p2g_batch_wait returns
 * P2G_ECANCELED with every job's status P2G_ECANCELED and its outputs
 * unspecified (a cancel that lands before the batch starts may let it run to
 * the end; it is reported cancelled all the same).  The context stays usable;
 * the next p2g_batch_launch clears the word.  No counterpart in par2-rs (its
 * Cancelled error, error.rs:34-35, stops host loops between chunks). */
int p2g_batch_cancel(p2g_batch *batch);
int p2g_batch_destroy(p2g_batch *batch);

/* Tile forms of the persistent batch kernel; each problem of a batch runs in
 * the form chosen for its class.  No counterpart in par2-rs, which runs one
 * recovery set per process (par2_rs.rs:816-870) with the blocking its
 * strategy fixes (avx2.rs:700-701). */
#define P2G_FORM_WIDE 0   /* 8 + 8 tables over 1024-symbol tiles, 104 outputs per item */
#define P2G_FORM_SMALL 1  /* 6 + 5 + 5 tables, at most 24 outputs */
#define P2G_FORM_PAIRED 2 /* 8 + 8 tables over 512-symbol tiles, 208 outputs per item */
/* Problem classes: 2 * (outputs 1-24: 0, 25-104: 1, 105-208: 2, more: 3)
 * + (slice_bytes > 16 KiB ? 1 : 0). */
#define P2G_BATCH_CLASSES 8

/* Batch autotuner: times each form valid for a class on one synthetic
 * problem of that class (8, 64, 160 or 420 outputs of ten times as many
 * inputs; slices of 8 KiB or 256 KiB; up to 64 copies of a small problem in
 * one launch, as many as make about 2e9 symbol multiply-accumulates; best
 * of `reps` launches of the persistent kernel after a warm-up) and keeps per
 * class, for this context's later batches, the default form (small tables up
 * to 24 outputs, paired above 104, wide between) unless another is at least
 * 3 % faster.  forms_out / ms_out (optional,
 * P2G_BATCH_CLASSES entries) receive the chosen forms and their times. */
int p2g_batch_autotune(p2g_ctx *ctx, int reps, int *forms_out, float *ms_out);
/* Pins the form per class (P2G_BATCH_CLASSES entries; -1, or forms NULL,
 * restores the heuristic: small tables up to 24 outputs, paired above 104,
 * wide between).  P2G_EINVAL for the small form on a class above 24
 * outputs. */
int p2g_batch_set_forms(p2g_ctx *ctx, const int *forms);

/* Size of the fixed device scratch array behind p2g_encode_noalloc. */
#define P2G_NOALLOC_SCRATCH_BYTES (64u << 20)

/* Recovery-slice creation (the work of p2g_encode) for callers that cannot
 * allocate device memory at call time: services that reserved a fixed
 * device-memory budget up front, latency paths that cannot take cudaMalloc's
 * implicit synchronisation, hosts that forbid allocation after start-up.  No
 * counterpart in par2-rs.
 *   - Allocates nothing: its scratch is one static device array of
 *     P2G_NOALLOC_SCRATCH_BYTES on every GPU that loads this library, held
 *     until the process exits.  A problem's scratch is about k*r*98 bytes
 *     when r <= 24 (2-byte coefficient + 96-byte record per pair) or
 *     k*r*34 bytes when r > 24 (32-byte records), plus k*slice_bytes rounded
 *     up to 2 KiB tiles, plus the pointer tables; a problem that needs more
 *     than the array returns P2G_ERANGE.
 *   - src[k] / out[r] are 16-byte aligned DEVICE pointers on the current
 *     device; the pointer arrays and exps are host arrays, pinned or not,
 *     read before the call returns (the caller may reuse them at once).
 *   - The work is enqueued on cuda_stream (a cudaStream_t; NULL is the legacy
 *     default stream) and the call returns without waiting for it;
 *     synchronise the stream before reading the outputs.
 *   - The first call on a device sets that device up (it looks up the device
 *     address of the scratch array, which loads the module); make that first
 *     call before any stream capture.
 *   - All calls on a device share the array: calls whose work overlaps on the
 *     GPU race, and the caller must serialise them. */
int p2g_encode_noalloc(void *cuda_stream, const uint8_t *const *src, size_t k,
                       size_t slice_bytes, const uint32_t *exps, size_t r, uint8_t *const *out);

#ifdef __cplusplus
}
#endif

#endif /* PAR2GPU_H */
