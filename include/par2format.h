/* par2format.h -- create and repair of PAR2 sets from files on one GPU.
 *
 * The top-level operations of par2-rs over the GPU codec (libpar2gpu):
 *   p2f_create  Par2Creator::new(..).with_*(..).create()   creator.rs:148-521
 *   p2f_repair  Par2Repairer::repair                       lib.rs:132-351
 * Files are written with par2-rs's packets, packet order, volume names and
 * creator text.  Every call returns P2F_OK (0) or a negative code; the
 * message of the last failure on this thread is p2f_last_error().
 * Built as par2-rs_b200/lib/libpar2format.so (needs libpar2gpu.so). */
#ifndef PAR2FORMAT_H
#define PAR2FORMAT_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define P2F_OK 0
#define P2F_ERROR (-1)          /* Par2Error::InvalidFormat / Io: see p2f_last_error */
#define P2F_ESINGULAR (-4)      /* Par2Error::RepairFailed("Singular matrix") */
#define P2F_EINSUFFICIENT (-8)  /* Par2Error::InsufficientRecovery (error.rs:5-39) */
#define P2F_ECANCELLED (-9)     /* Par2Error::Cancelled: "PAR2 operation cancelled" */
#define P2F_EDAMAGED (-10)      /* RepairFailed("Files are damaged and repair was not requested") */

#define P2F_SCHEME_SINGLE 0       /* VolumeScheme::Single (volumes.rs:27-31) */
#define P2F_SCHEME_EXPONENTIAL 1  /* VolumeScheme::Exponential: 1, 2, 4 ... slices per file */

/* Phase times of one call (milliseconds) and what it processed. */
typedef struct p2f_stats {
    double ms_scan, ms_ingest, ms_gpu, ms_write, ms_total;
    uint64_t block_size, data_blocks, recovery_blocks, bytes_read;
    uint64_t damaged_blocks, files_written;
} p2f_stats;

/* Creates the set of `inputs` (n paths) at `output` (the index .par2; NULL:
 * the first input with its extensions replaced by .par2, creator.rs:170).
 * block_size 0 picks it as par2-rs does (creator.rs:30-67); otherwise it
 * must be a multiple of 4 and at least 2048.  The paths of the written files
 * are not returned: they follow volumes.rs:65-78.  stats may be NULL. */
int p2f_create(const char *const *inputs, size_t n, const char *output, uint64_t block_size,
               float redundancy_percent, int scheme, p2f_stats *stats);

/* Verifies the files of the set `par2_path` (with its volumes, found by
 * recovery set ID) in directory `dir` and rebuilds damaged or missing slices
 * in place.  *rebuilt (may be NULL) receives the number of slices rebuilt,
 * 0 when every slice was intact. */
int p2f_repair(const char *par2_path, const char *dir, uint64_t *rebuilt, p2f_stats *stats);

/* Par2Operation (lib.rs:76-81) passed to the progress callback */
#define P2F_OP_SCANNING 0
#define P2F_OP_LOADING 1
#define P2F_OP_VERIFYING 2
#define P2F_OP_REPAIRING 3
typedef void (*p2f_progress_fn)(void *user, int operation, uint64_t current, uint64_t total);

/* p2f_create with Par2Creator::with_progress_callback (creator.rs:245-253):
 * progress, if not NULL, is called on this thread with P2F_OP_REPAIRING
 * (the reference's name for encoding progress), current = data slices
 * encoded and total = data slices: 0 before the files are read, total once
 * the recovery slices exist. */
int p2f_create_ex(const char *const *inputs, size_t n, const char *output, uint64_t block_size,
                  float redundancy_percent, int scheme, p2f_progress_fn progress, void *user,
                  p2f_stats *stats);

/* Par2Repairer::repair_with_callbacks_cancellable (lib.rs:196-351):
 *   do_repair  0: verify only -- any damage returns P2F_EDAMAGED
 *   purge      1: delete the set's .par2 files after a verified or repaired set
 *   progress   optional (operation, current, total) callback, called on this thread
 *   cancel     optional flag; set it non-zero from any thread to stop at the next
 *              safe point (P2F_ECANCELLED).  Rebuilt files are written to
 *              <name>.par2tmp and renamed into place only after all of them are
 *              written, so a cancellation or an error before that leaves every
 *              data file unchanged; a cancellation after it skips the purge. */
int p2f_repair_ex(const char *par2_path, const char *dir, int do_repair, int purge,
                  p2f_progress_fn progress, void *user, const volatile int32_t *cancel,
                  uint64_t *rebuilt, p2f_stats *stats);

/* Recovery slices through par2-rs's streaming encoder path with the callers
 * unchanged: Par2ReedSolomon::create_streaming_encoder + process_block per
 * data block + finalize (par2_rs.rs:687-902), restated on the host over the
 * selected galois strategy (the CUDA strategy, or the one named by
 * PAR2_SIMD_STRATEGY).  Data blocks are buffered in batches of 16-128 and
 * each full batch is multiplied into the recovery accumulators by `threads`
 * worker threads (0: the host's thread count), recovery batches of 4-8 at a
 * time, one strategy call per (recovery block, data block) pair -- through
 * the shuffle2x hooks when the strategy supports them, as par2-rs does.
 *   src[k]  host data blocks of block_size bytes (even)
 *   out[r]  host buffers receiving the recovery slices, exponents 0..r-1 */
int p2f_streaming_encode(const uint8_t *const *src, size_t k, size_t block_size, size_t r,
                         uint8_t *const *out, int threads);

const char *p2f_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
