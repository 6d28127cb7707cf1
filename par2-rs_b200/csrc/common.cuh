// common.cuh -- context, scratch buffers and error plumbing shared by the
// CUDA translation units of libpar2gpu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/par2gpu.h"

namespace p2g {

// Thread-local message behind p2g_last_error().
void set_error(const char *fmt, ...);
void clear_error();

// PAR2 input-slice constants (par2_rs.rs:64-76) on the host.
void par2_constants(size_t k, uint16_t *out);

// Growable device (or pinned host) buffer owned by a context.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    bool pinned = false;
    int ensure(size_t n);  // P2G_OK / P2G_ENOMEM; contents not preserved
    void release();
    template <class T>
    T *as() const { return static_cast<T *>(p); }
};

// How one multiply-accumulate problem is cut into CTAs: warps per CTA,
// outputs per output group (16 / psplit accumulator registers per warp each),
// output blocks of (warps / psplit) * ereg outputs, input ranges folded with
// atomic XOR.
struct MuladdPlan {
    int warps = 8;
    int ereg = 1;
    int nblk = 1;
    int nsplit = 1;
    int psplit = 1;  // warps sharing one output group (each holds 16/psplit planes)
    bool small = false;  // small-output tables (set for problems of <= kSmallOutputs outputs)
    bool paired = false; // 512-symbol tiles, two outputs per warp lookup (more than 104 outputs)
    int stage = 1;       // inputs per CTA barrier (2: paired form only)
};

using PlanKey = std::tuple<int, int, size_t>;  // inputs, outputs, slice bytes

// Device mirrors and recorded products of the shuffle2x hooks (deferred.cu).
struct Deferred;
inline PlanKey plan_key(int nin, int nout, size_t S) { return PlanKey(nin, nout, S); }

}  // namespace p2g

struct p2g_ctx {
    // tuned plans (p2g_autotune); choose_plan falls back to a heuristic
    std::map<p2g::PlanKey, p2g::MuladdPlan> plans;
    // tile form of the persistent batch kernel per problem class
    // (p2g_batch_autotune / p2g_batch_set_forms); -1: the heuristic's
    int batch_forms[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
    int device = 0;
    int sm_count = 0;
    cudaStream_t own_stream = nullptr;  // created with the context
    cudaStream_t stream = nullptr;      // where work runs (own or caller's)
    // host-to-device copies that overlap the kernels (p2g_encode from host)
    cudaStream_t copy_stream = nullptr;
    // device-to-host read-back of finished output slabs (p2g_encode to host)
    cudaStream_t d2h_stream = nullptr;
    // the copy that raises a running batch's abort word (p2g_batch_cancel)
    cudaStream_t cancel_stream = nullptr;
    static constexpr int kPipe = 16;        // input groups of a host encode
    static constexpr int kPipeEvents = 56;  // group events + slab events
    cudaEvent_t pipe_ev[kPipeEvents] = {};
    std::mutex mu;
    // optional per-phase timing (p2g_set_timing / p2g_last_timing)
    bool timing = false;
    cudaEvent_t ev[5] = {};
    bool ev_marked[5] = {};
    int launches = 0;
    p2g_timing last = {};
    // Records event `idx` (0 call start, 1 records done, 2 planes done,
    // 3 muladd done, 4 call end) when timing is enabled.
    void mark(int idx)
    {
        if (timing && ev[idx]) {
            cudaEventRecord(ev[idx], stream);
            ev_marked[idx] = true;
        }
    }
    // GF(2^16) log / antilog tables on the device (galois/core.rs:49-91)
    uint16_t *d_log = nullptr;
    uint16_t *d_exp = nullptr;
    // CRC-32 slicing-by-4 tables on the device (4 x 256 words)
    uint32_t *d_crc = nullptr;
    // scratch
    p2g::DevBuf planes;    // bit-sliced inputs
    p2g::DevBuf recs;      // coefficient records
    p2g::DevBuf in_copy;   // device copies of host / misaligned inputs
    p2g::DevBuf out_copy;  // device copies of host / misaligned outputs
    p2g::DevBuf params;    // small device parameter block (pointer arrays ...)
    p2g::DevBuf hparams;   // pinned host mirror of `params`
    p2g::DevBuf coeffs;    // coefficient matrices
    p2g::DevBuf recs2;     // records of a second pass (repair)
    p2g::DevBuf rhs;       // repair right-hand sides
    p2g::DevBuf inv;       // decode matrix
    p2g::DevBuf gj_M;      // Gauss-Jordan augmented matrix
    p2g::DevBuf gj_status; // Gauss-Jordan status + pivots
    p2g::DevBuf hash_out;  // MD5 + CRC results
    p2g::DevBuf wb;        // decode matrices by Woodbury correction
    // Scratch buffers of destroyed batches, kept for the next batch: freeing
    // device or pinned memory synchronises the whole device, which would stall
    // a batch being prepared while another one runs.  Guarded by `mu`.
    std::vector<p2g::DevBuf> spare;
    // the shuffle2x hooks' state, created on first use (read without the
    // context lock by the recording calls)
    std::atomic<p2g::Deferred *> deferred{nullptr};
};

namespace p2g {
// Frees the shuffle2x state (mirrors, staging, pool) of a context.
void deferred_release(p2g_ctx *ctx);
}  // namespace p2g

#define P2G_CUDA(call)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) {                                                        \
            p2g::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),      \
                           __FILE__, __LINE__);                                         \
            return P2G_ECUDA;                                                           \
        }                                                                               \
    } while (0)

#define P2G_TRY(expr)           \
    do {                        \
        int rc_ = (expr);       \
        if (rc_ != P2G_OK)      \
            return rc_;         \
    } while (0)
