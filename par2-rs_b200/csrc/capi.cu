// capi.cu -- the C ABI of libpar2gpu (include/par2gpu.h): contexts, staging
// of host / misaligned buffers, argument checking and error reporting.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "hash.cuh"
#include "invert.cuh"
#include "muladd.cuh"

namespace p2g {

static thread_local std::string g_last_error;

void set_error(const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
}

void clear_error() { g_last_error.clear(); }

int DevBuf::ensure(size_t n)
{
    if (n <= cap)
        return P2G_OK;
    release();
    size_t want = n < 4096 ? 4096 : n;
    cudaError_t e = pinned ? cudaMallocHost(&p, want) : cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        cap = 0;
        (void)cudaGetLastError();
        set_error("%s of %zu bytes failed: %s", pinned ? "cudaMallocHost" : "cudaMalloc", want,
                  cudaGetErrorString(e));
        return P2G_ENOMEM;
    }
    cap = want;
    return P2G_OK;
}

void DevBuf::release()
{
    if (p) {
        if (pinned)
            cudaFreeHost(p);
        else
            cudaFree(p);
    }
    p = nullptr;
    cap = 0;
}

static size_t round16(size_t n) { return (n + 15) & ~static_cast<size_t>(15); }

// PAR2 constants (par2_rs.rs:64-76), with the GF tables of galois/core.rs:49-91.
struct HostTables {
    uint16_t log[65536];
    uint16_t exp[65535];
    HostTables()
    {
        uint32_t b = 1;
        for (uint32_t l = 0; l < 65535; ++l) {
            exp[l] = static_cast<uint16_t>(b);
            log[b] = static_cast<uint16_t>(l);
            b <<= 1;
            if (b & 0x10000u)
                b ^= 0x1100Bu;
        }
        log[0] = 0;
    }
};

static const HostTables &tables()
{
    static HostTables t;
    return t;
}

void par2_constants(size_t k, uint16_t *out)
{
    const HostTables &t = tables();
    size_t have = 0;
    for (uint64_t n = 1; have < k; ++n)
        if (n % 3 && n % 5 && n % 17 && n % 257)
            out[have++] = t.exp[n % 65535];
}

// Layout of the per-call parameter block (device + pinned mirror).
struct ParamLayout {
    size_t src_off, dst_off, a_off, b_off, total;
    ParamLayout(size_t nsrc, size_t ndst, size_t a_bytes, size_t b_bytes)
    {
        src_off = 0;
        dst_off = round16(nsrc * sizeof(void *));
        a_off = dst_off + round16(ndst * sizeof(void *));
        b_off = a_off + round16(a_bytes);
        total = b_off + round16(b_bytes);
    }
};

static int upload_params(p2g_ctx *ctx, const ParamLayout &L)
{
    P2G_CUDA(cudaMemcpyAsync(ctx->params.p, ctx->hparams.p, L.total, cudaMemcpyHostToDevice,
                             ctx->stream));
    return P2G_OK;
}

constexpr int kTailGroups = 2;     // input groups processed slab by slab (host outputs)
constexpr int kMaxTailSlabs = 16;  // column slabs of those groups, at most
constexpr int kSlabEvents = p2g_ctx::kPipe;  // pipe_ev index of the first slab event
static_assert(kSlabEvents + 2 * kMaxTailSlabs + 1 <= p2g_ctx::kPipeEvents, "slab events");

static bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Copies n slices of `bytes` each, src[i] -> dst[i], on `stream`.  Runs of
// slices whose source and destination addresses both advance by constant
// strides (slices cut from one buffer) become one 2D copy: one DMA transfer
// instead of one per slice.
static int copy_slices(uint8_t *const *dst, const uint8_t *const *src, size_t n, size_t bytes,
                       cudaMemcpyKind kind, cudaStream_t stream)
{
    constexpr ptrdiff_t kMaxPitch = ptrdiff_t(1) << 30;
    size_t i = 0;
    while (i < n) {
        size_t j = i + 1;
        if (j < n) {
            const ptrdiff_t hs = src[j] - src[i], ds = dst[j] - dst[i];
            if (hs >= static_cast<ptrdiff_t>(bytes) && ds >= static_cast<ptrdiff_t>(bytes) &&
                hs <= kMaxPitch && ds <= kMaxPitch) {
                while (j + 1 < n && src[j + 1] - src[j] == hs && dst[j + 1] - dst[j] == ds)
                    ++j;
                ++j;  // [i, j) has constant strides
                P2G_CUDA(cudaMemcpy2DAsync(dst[i], static_cast<size_t>(ds), src[i],
                                           static_cast<size_t>(hs), bytes, j - i, kind, stream));
                i = j;
                continue;
            }
        }
        P2G_CUDA(cudaMemcpyAsync(dst[i], src[i], bytes, kind, stream));
        ++i;
    }
    return P2G_OK;
}

// Resolves the slice pointers a kernel will use: device pointers that are
// 16-byte aligned are used in place; host pointers (or misaligned device
// pointers) are staged through `buf` (one padded slot per slice).  `copy_in`
// copies the current contents in.
static int stage(p2g_ctx *ctx, p2g::DevBuf &buf, const uint8_t *const *ptrs, size_t n,
                 size_t bytes, bool device, bool copy_in, std::vector<uint8_t *> &out,
                 bool &staged)
{
    out.resize(n);
    bool all_ok = device;
    if (device)
        for (size_t i = 0; i < n; ++i)
            if (!aligned16(ptrs[i]))
                all_ok = false;
    staged = !all_ok;
    if (all_ok) {
        for (size_t i = 0; i < n; ++i)
            out[i] = const_cast<uint8_t *>(ptrs[i]);
        return P2G_OK;
    }
    size_t slot = round16(bytes);
    P2G_TRY(buf.ensure(slot * (n ? n : 1)));
    for (size_t i = 0; i < n; ++i)
        out[i] = buf.as<uint8_t>() + i * slot;
    if (copy_in)
        P2G_TRY(copy_slices(out.data(), ptrs, n, bytes,
                            device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            ctx->stream));
    return P2G_OK;
}

// Copies results back to the caller's slices.  If a copy fails, the ones
// already enqueued land before the error is returned (the caller may free
// its buffers as soon as the call returns).
static int unstage(p2g_ctx *ctx, uint8_t *const *user, const std::vector<uint8_t *> &dev,
                   size_t n, size_t bytes, bool device)
{
    const int rc = copy_slices(user, dev.data(), n, bytes,
                               device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                               ctx->stream);
    if (rc != P2G_OK)
        cudaStreamSynchronize(ctx->stream);
    return rc;
}

// Starts a call: resets the launch counter and the timing marks.
static void begin(p2g_ctx *ctx)
{
    ctx->launches = 0;
    for (bool &m : ctx->ev_marked)
        m = false;
    ctx->mark(0);
}

static float elapsed(p2g_ctx *ctx, int a, int b)
{
    float ms = 0.f;
    if (ctx->ev_marked[a] && ctx->ev_marked[b] &&
        cudaEventElapsedTime(&ms, ctx->ev[a], ctx->ev[b]) != cudaSuccess) {
        (void)cudaGetLastError();
        ms = 0.f;
    }
    return ms;
}

// Ends a call: waits for its work and collects the timing.
static int finish(p2g_ctx *ctx)
{
    ctx->mark(4);
    P2G_CUDA(cudaStreamSynchronize(ctx->stream));
    P2G_CUDA(cudaGetLastError());
    ctx->last = p2g_timing{};
    ctx->last.launches = ctx->launches;
    if (ctx->timing) {
        ctx->last.ms_records = elapsed(ctx, 0, 1);
        ctx->last.ms_planes = elapsed(ctx, 1, 2);
        ctx->last.ms_kernel = elapsed(ctx, 2, 3);
        ctx->last.ms_total = elapsed(ctx, 0, 4);
    }
    return P2G_OK;
}

// Generic coefficient-matrix muladd over resolved device slices:
// dst[o] (^)= sum_i coeff[o][i] * src[i]; coeff is a host [nout][nin] matrix.
static int matrix_muladd(p2g_ctx *ctx, const std::vector<uint8_t *> &src,
                         const std::vector<uint8_t *> &dst, const uint16_t *coeff,
                         size_t bytes, int mode)
{
    size_t nin = src.size(), nout = dst.size();
    ParamLayout L(nin, nout, nin * nout * 2, 0);
    P2G_TRY(ctx->hparams.ensure(L.total));
    P2G_TRY(ctx->params.ensure(L.total));
    uint8_t *h = ctx->hparams.as<uint8_t>();
    memcpy(h + L.src_off, src.data(), nin * sizeof(void *));
    memcpy(h + L.dst_off, dst.data(), nout * sizeof(void *));
    memcpy(h + L.a_off, coeff, nin * nout * 2);
    P2G_TRY(upload_params(ctx, L));
    uint8_t *d = ctx->params.as<uint8_t>();
    P2G_TRY(ctx->recs.ensure(record_bytes(nin, static_cast<int>(nout))));
    P2G_TRY(records_from_matrix(ctx, reinterpret_cast<const uint16_t *>(d + L.a_off),
                                static_cast<int>(nin), static_cast<int>(nout),
                                ctx->recs.as<uint32_t>()));
    P2G_TRY(muladd_run(ctx, reinterpret_cast<const uint8_t *const *>(d + L.src_off),
                       static_cast<int>(nin), reinterpret_cast<uint8_t *const *>(d + L.dst_off),
                       static_cast<int>(nout), bytes, ctx->recs.as<uint32_t>(), mode));
    return P2G_OK;
}

}  // namespace p2g

using namespace p2g;

extern "C" {

const char *p2g_last_error(void) { return g_last_error.c_str(); }

int p2g_strategy_info(const char **name, int *priority, int *available)
{
    if (name)
        *name = "CUDA-sm100a";
    if (priority)
        *priority = P2G_PRIORITY_OPTIMAL;
    if (available) {
        int n = 0, ok = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            (void)cudaGetLastError();
            n = 0;
        }
        for (int d = 0; d < n; ++d) {
            int major = 0;
            if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d) ==
                    cudaSuccess &&
                major == 10)
                ok = 1;
        }
        *available = ok;
    }
    return P2G_OK;
}

int p2g_create(int device, p2g_ctx **out)
{
    clear_error();
    if (!out) {
        set_error("p2g_create: null output pointer");
        return P2G_EINVAL;
    }
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        (void)cudaGetLastError();
        set_error("p2g_create: no CUDA device %d", device);
        return P2G_ENODEV;
    }
    cudaDeviceProp prop;
    P2G_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        set_error("p2g_create: device %d is sm_%d%d, the library is compiled for sm_100a", device,
                  prop.major, prop.minor);
        return P2G_ENODEV;
    }
    P2G_CUDA(cudaSetDevice(device));
    p2g_ctx *ctx = new p2g_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    ctx->hparams.pinned = true;
    int rc = P2G_OK;
    do {
        if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
            set_error("cudaStreamCreate failed");
            rc = P2G_ECUDA;
            break;
        }
        ctx->stream = ctx->own_stream;
        if (cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&ctx->d2h_stream, cudaStreamNonBlocking) != cudaSuccess) {
            set_error("cudaStreamCreate failed");
            rc = P2G_ECUDA;
            break;
        }
        bool ev_ok = true;
        for (cudaEvent_t &e : ctx->ev)
            ev_ok = ev_ok && cudaEventCreate(&e) == cudaSuccess;
        for (cudaEvent_t &e : ctx->pipe_ev)
            ev_ok = ev_ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
        if (!ev_ok) {
            set_error("cudaEventCreate failed");
            rc = P2G_ECUDA;
            break;
        }
        const HostTables &t = tables();
        if (cudaMalloc(&ctx->d_log, sizeof t.log) != cudaSuccess ||
            cudaMalloc(&ctx->d_exp, sizeof t.exp) != cudaSuccess ||
            cudaMemcpy(ctx->d_log, t.log, sizeof t.log, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(ctx->d_exp, t.exp, sizeof t.exp, cudaMemcpyHostToDevice) != cudaSuccess) {
            set_error("p2g_create: GF table upload failed");
            rc = P2G_ENOMEM;
            break;
        }
        static uint32_t crc_tab[4][256];
        crc32_tables(crc_tab);
        if (cudaMalloc(&ctx->d_crc, sizeof crc_tab) != cudaSuccess ||
            cudaMemcpy(ctx->d_crc, crc_tab, sizeof crc_tab, cudaMemcpyHostToDevice) != cudaSuccess) {
            set_error("p2g_create: CRC table upload failed");
            rc = P2G_ENOMEM;
            break;
        }
    } while (0);
    if (rc != P2G_OK) {
        (void)cudaGetLastError();
        p2g_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return P2G_OK;
}

int p2g_destroy(p2g_ctx *ctx)
{
    if (!ctx)
        return P2G_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream)
        cudaStreamSynchronize(ctx->own_stream);
    p2g::deferred_release(ctx);
    ctx->planes.release();
    ctx->recs.release();
    ctx->in_copy.release();
    ctx->out_copy.release();
    ctx->params.release();
    ctx->hparams.release();
    ctx->coeffs.release();
    ctx->recs2.release();
    ctx->rhs.release();
    ctx->inv.release();
    ctx->gj_M.release();
    ctx->gj_status.release();
    if (ctx->d_log)
        cudaFree(ctx->d_log);
    if (ctx->d_exp)
        cudaFree(ctx->d_exp);
    if (ctx->d_crc)
        cudaFree(ctx->d_crc);
    ctx->hash_out.release();
    ctx->wb.release();
    for (p2g::DevBuf &d : ctx->spare)
        d.release();
    ctx->spare.clear();
    for (cudaEvent_t e : ctx->ev)
        if (e)
            cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->pipe_ev)
        if (e)
            cudaEventDestroy(e);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    if (ctx->d2h_stream) {
        cudaStreamSynchronize(ctx->d2h_stream);
        cudaStreamDestroy(ctx->d2h_stream);
    }
    if (ctx->cancel_stream) {
        cudaStreamSynchronize(ctx->cancel_stream);
        cudaStreamDestroy(ctx->cancel_stream);
    }
    if (ctx->own_stream)
        cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return P2G_OK;
}

int p2g_set_stream(p2g_ctx *ctx, void *cuda_stream)
{
    clear_error();
    if (!ctx) {
        set_error("p2g_set_stream: null context");
        return P2G_EINVAL;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ctx->own_stream;
    return P2G_OK;
}

int p2g_set_timing(p2g_ctx *ctx, int enable)
{
    clear_error();
    if (!ctx) {
        set_error("p2g_set_timing: null context");
        return P2G_EINVAL;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->timing = enable != 0;
    return P2G_OK;
}

int p2g_last_timing(p2g_ctx *ctx, p2g_timing *out)
{
    clear_error();
    if (!ctx || !out) {
        set_error("p2g_last_timing: null argument");
        return P2G_EINVAL;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    *out = ctx->last;
    return P2G_OK;
}

int p2g_autotune(p2g_ctx *ctx, size_t nin, size_t nout, size_t slice_bytes, int reps,
                 p2g_plan *best)
{
    clear_error();
    if (!ctx || !best) {
        set_error("p2g_autotune: null argument");
        return P2G_EINVAL;
    }
    if (nin > 65535 || nout > 65535) {
        set_error("p2g_autotune: %zu x %zu beyond 65535", nin, nout);
        return P2G_ERANGE;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    MuladdPlan p;
    float ms = 0.f;
    int tried = 0;
    P2G_TRY(muladd_autotune(ctx, static_cast<int>(nin), static_cast<int>(nout), slice_bytes,
                            reps, &p, &ms, &tried));
    *best = p2g_plan{p.warps, p.paired ? 2 * p.ereg : p.ereg, p.psplit, p.nblk, p.nsplit, ms,
                     p.paired ? 512 : 1024, p.stage};
    return P2G_OK;
}

int p2g_set_plan(p2g_ctx *ctx, size_t nin, size_t nout, size_t slice_bytes,
                 const p2g_plan *plan)
{
    clear_error();
    if (!ctx || !plan) {
        set_error("p2g_set_plan: null argument");
        return P2G_EINVAL;
    }
    MuladdPlan p;
    p.warps = plan->warps;
    p.ereg = plan->outputs_per_group;
    p.psplit = plan->warps_per_group;
    p.nblk = plan->output_blocks;
    p.nsplit = plan->input_splits;
    p.small = nout <= static_cast<size_t>(p2g::kSmallOutputs);  // the table form follows nout
    // 512-symbol tiles: a warp accumulates outputs_per_group outputs, two per
    // lookup (an even count)
    p.paired = plan->tile_symbols == 512;
    if (p.paired)
        p.ereg = plan->outputs_per_group % 2 ? -1 : plan->outputs_per_group / 2;
    p.stage = plan->inputs_per_stage == 0 ? 1 : plan->inputs_per_stage;
    if ((plan->tile_symbols != 0 && plan->tile_symbols != 512 && plan->tile_symbols != 1024) ||
        nin > 65535 || nout > 65535 ||
        !plan_valid(p, static_cast<int>(nin), static_cast<int>(nout), slice_bytes)) {
        set_error("p2g_set_plan: warps=%d outputs_per_group=%d warps_per_group=%d blocks=%d "
                  "splits=%d tile_symbols=%d inputs_per_stage=%d is not a compiled shape "
                  "covering %zu outputs",
                  plan->warps, plan->outputs_per_group, plan->warps_per_group,
                  plan->output_blocks, plan->input_splits, plan->tile_symbols,
                  plan->inputs_per_stage, nout);
        return P2G_EINVAL;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->plans[plan_key(static_cast<int>(nin), static_cast<int>(nout), slice_bytes)] = p;
    return P2G_OK;
}

int p2g_par2_constants(size_t k, uint16_t *out)
{
    clear_error();
    if (!out && k) {
        set_error("p2g_par2_constants: null output");
        return P2G_EINVAL;
    }
    par2_constants(k, out);
    return P2G_OK;
}

int p2g_encode(p2g_ctx *ctx, const uint8_t *const *src, size_t k, size_t slice_bytes,
               const uint32_t *exps, size_t r, uint8_t *const *out, uint32_t flags)
{
    clear_error();
    if (!ctx || (k && !src) || (r && (!out || !exps))) {
        set_error("p2g_encode: null argument");
        return P2G_EINVAL;
    }
    if (slice_bytes == 0 || slice_bytes % 2) {
        set_error("p2g_encode: slice size %zu must be even and non-zero "
                  "(\"Block size must be multiple of 2\", par2_rs.rs:697-699)",
                  slice_bytes);
        return P2G_EINVAL;
    }
    if (k > 65535 || r > 65535) {
        set_error("p2g_encode: %zu inputs / %zu outputs exceed the GF(2^16) limit of 65535", k,
                  r);
        return P2G_ERANGE;
    }
    if (r == 0)
        return P2G_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    begin(ctx);
    const bool dev = flags & P2G_DEVICE_PTRS;
    // Host sources are copied in groups on the copy stream while the kernel
    // accumulates the groups already on the device (XOR into the outputs).
    const int groups = (!dev && k >= 128) ? static_cast<int>(std::min<size_t>(p2g_ctx::kPipe, k / 64)) : 1;
    std::vector<uint8_t *> s, d;
    bool s_staged = false, d_staged = false;
    P2G_TRY(stage(ctx, ctx->in_copy, src, k, slice_bytes, dev, groups == 1, s, s_staged));
    P2G_TRY(stage(ctx, ctx->out_copy, out, r, slice_bytes, dev, false, d, d_staged));
    // With host outputs, the last kTailGroups input groups run slab by slab
    // (column ranges): a slab's inputs go up, its outputs are then final and
    // go back on their own stream while the next slab goes up -- both PCIe
    // directions busy -- instead of reading all outputs back after the end.
    // Slabs are sized to whole waves: one slab's launch (slab tiles x output
    // blocks CTAs) about fills the device, so none leaves SMs idle.
    const size_t tiles = (slice_bytes + 2047) / 2048;
    int slabs = 1;
    if (groups >= 4 && d_staged) {
        const p2g::MuladdPlan tp = p2g::choose_plan(ctx, static_cast<int>(k / groups * kTailGroups),
                                                    static_cast<int>(r), slice_bytes);
        const double waves = static_cast<double>(p2g::plan_tiles(tp, slice_bytes)) * tp.nblk /
                             p2g::plan_slots(ctx, tp);
        slabs = static_cast<int>(std::min<double>(kMaxTailSlabs, std::floor(waves + 0.5)));
        if (static_cast<size_t>(slabs) > tiles)
            slabs = 1;
    }
    const bool tail = slabs >= 2;
    const size_t t0 = tail ? k * (groups - kTailGroups) / groups : k, ntail = k - t0;
    std::vector<size_t> cut(slabs + 1);
    for (int q = 0; q <= slabs; ++q)
        cut[q] = q == slabs ? slice_bytes : tiles * q / slabs * 2048;
    // The last slab's compute and read-back are what remains after the last
    // upload: it goes in two halves, the first computed and read back while
    // the second uploads.
    if (tail && slabs < kMaxTailSlabs) {
        const size_t a = cut[slabs - 1] / 2048, b = tiles;
        if (b - a >= 2)
            cut.insert(cut.end() - 1, (a + (b - a) / 2) * 2048);
    }
    slabs = static_cast<int>(cut.size()) - 1;
    const size_t tail_bytes = tail ? slabs * (ntail + r) * sizeof(void *) : 0;
    ParamLayout L(k, r, k * 2, round16(r * 4) + tail_bytes);
    P2G_TRY(ctx->hparams.ensure(L.total));
    P2G_TRY(ctx->params.ensure(L.total));
    uint8_t *h = ctx->hparams.as<uint8_t>();
    memcpy(h + L.src_off, s.data(), k * sizeof(void *));
    memcpy(h + L.dst_off, d.data(), r * sizeof(void *));
    par2_constants(k, reinterpret_cast<uint16_t *>(h + L.a_off));
    memcpy(h + L.b_off, exps, r * 4);
    const size_t tail_off = L.b_off + round16(r * 4);
    if (tail) {
        // per slab: the tail inputs, then the outputs, offset to the slab
        uint8_t **t = reinterpret_cast<uint8_t **>(h + tail_off);
        for (int q = 0; q < slabs; ++q) {
            for (size_t i = 0; i < ntail; ++i)
                *t++ = s[t0 + i] + cut[q];
            for (size_t e = 0; e < r; ++e)
                *t++ = d[e] + cut[q];
        }
    }
    // the copy stream starts after everything already queued on the compute
    // stream (earlier users of the staging buffers), not after this call's
    // records
    if (groups > 1) {
        P2G_CUDA(cudaEventRecord(ctx->pipe_ev[0], ctx->stream));
        P2G_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->pipe_ev[0], 0));
    }
    P2G_TRY(upload_params(ctx, L));
    uint8_t *dp = ctx->params.as<uint8_t>();
    P2G_TRY(ctx->recs.ensure(record_bytes(k, static_cast<int>(r))));
    const size_t rw = static_cast<size_t>(record_words(static_cast<int>(r)));  // per record
    P2G_TRY(records_par2(ctx, reinterpret_cast<const uint16_t *>(dp + L.a_off),
                         reinterpret_cast<const uint32_t *>(dp + L.b_off), static_cast<int>(k),
                         static_cast<int>(r), ctx->recs.as<uint32_t>()));
    const uint8_t *const *d_src = reinterpret_cast<const uint8_t *const *>(dp + L.src_off);
    uint8_t *const *d_dst = reinterpret_cast<uint8_t *const *>(dp + L.dst_off);
    if (groups == 1) {
        P2G_TRY(muladd_run(ctx, d_src, static_cast<int>(k), d_dst, static_cast<int>(r),
                           slice_bytes, ctx->recs.as<uint32_t>(), 0));
    } else {
        // The copies run on the context's side streams.  If a step below
        // fails, the ones already enqueued (some into the caller's host
        // buffers) finish before the error is returned.
        const int rc = [&]() -> int {
            const int full = tail ? groups - kTailGroups : groups;
            for (int g = 0; g < full; ++g) {
                const size_t i0 = k * g / groups, i1 = k * (g + 1) / groups;
                P2G_TRY(copy_slices(s.data() + i0, src + i0, i1 - i0, slice_bytes,
                                    cudaMemcpyHostToDevice, ctx->copy_stream));
                P2G_CUDA(cudaEventRecord(ctx->pipe_ev[g], ctx->copy_stream));
                P2G_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->pipe_ev[g], 0));
                P2G_TRY(muladd_run(ctx, d_src + i0, static_cast<int>(i1 - i0), d_dst,
                                   static_cast<int>(r), slice_bytes,
                                   ctx->recs.as<uint32_t>() + i0 * r * rw, g == 0 ? 0 : 1));
            }
            if (tail) {
                uint8_t *const *tab = reinterpret_cast<uint8_t *const *>(dp + tail_off);
                std::vector<const uint8_t *> hs(ntail);
                std::vector<uint8_t *> ds(ntail), uo(r), so(r);
                cudaEvent_t *up = ctx->pipe_ev + kSlabEvents, *done = up + slabs;
                for (int q = 0; q < slabs; ++q) {
                    const size_t w = cut[q + 1] - cut[q];
                    for (size_t i = 0; i < ntail; ++i) {
                        hs[i] = src[t0 + i] + cut[q];
                        ds[i] = s[t0 + i] + cut[q];
                    }
                    P2G_TRY(copy_slices(ds.data(), hs.data(), ntail, w, cudaMemcpyHostToDevice,
                                        ctx->copy_stream));
                    P2G_CUDA(cudaEventRecord(up[q], ctx->copy_stream));
                    P2G_CUDA(cudaStreamWaitEvent(ctx->stream, up[q], 0));
                    uint8_t *const *qt = tab + q * (ntail + r);
                    P2G_TRY(muladd_run(ctx, reinterpret_cast<const uint8_t *const *>(qt),
                                       static_cast<int>(ntail), qt + ntail, static_cast<int>(r), w,
                                       ctx->recs.as<uint32_t>() + t0 * r * rw, 1));
                    P2G_CUDA(cudaEventRecord(done[q], ctx->stream));
                    P2G_CUDA(cudaStreamWaitEvent(ctx->d2h_stream, done[q], 0));
                    for (size_t e = 0; e < r; ++e) {
                        uo[e] = out[e] + cut[q];
                        so[e] = d[e] + cut[q];
                    }
                    P2G_TRY(copy_slices(uo.data(), so.data(), r, w, cudaMemcpyDeviceToHost,
                                        ctx->d2h_stream));
                }
                // the call ends when the last read-back has landed
                P2G_CUDA(cudaEventRecord(done[slabs], ctx->d2h_stream));
                P2G_CUDA(cudaStreamWaitEvent(ctx->stream, done[slabs], 0));
            }
            return P2G_OK;
        }();
        if (rc != P2G_OK) {
            cudaStreamSynchronize(ctx->copy_stream);
            cudaStreamSynchronize(ctx->d2h_stream);
            cudaStreamSynchronize(ctx->stream);
            return rc;
        }
    }
    if (d_staged && !tail)
        P2G_TRY(unstage(ctx, out, d, r, slice_bytes, dev));
    return finish(ctx);
}

int p2g_muladd_region(p2g_ctx *ctx, uint16_t *const *dsts, size_t ndst,
                      const uint16_t *const *srcs, size_t nsrc,
                      const uint16_t *const *coeff_rows, size_t off_u16, size_t len_u16,
                      uint32_t flags)
{
    clear_error();
    if (!ctx || (ndst && (!dsts || !coeff_rows)) || (nsrc && !srcs)) {
        set_error("p2g_muladd_region: null argument");
        return P2G_EINVAL;
    }
    if (ndst > 65535 || nsrc > 65535) {
        set_error("p2g_muladd_region: too many slices");
        return P2G_ERANGE;
    }
    if (ndst == 0 || nsrc == 0 || len_u16 == 0)
        return P2G_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    begin(ctx);
    const bool dev = flags & P2G_DEVICE_PTRS;
    const size_t bytes = len_u16 * 2;
    std::vector<const uint8_t *> sp(nsrc);
    std::vector<uint8_t *> dp(ndst);
    for (size_t i = 0; i < nsrc; ++i)
        sp[i] = reinterpret_cast<const uint8_t *>(srcs[i] + off_u16);
    for (size_t o = 0; o < ndst; ++o)
        dp[o] = reinterpret_cast<uint8_t *>(dsts[o] + off_u16);
    std::vector<uint16_t> coeff(ndst * nsrc);
    for (size_t o = 0; o < ndst; ++o)
        memcpy(&coeff[o * nsrc], coeff_rows[o], nsrc * 2);
    std::vector<uint8_t *> s, d;
    bool s_staged = false, d_staged = false;
    P2G_TRY(stage(ctx, ctx->in_copy, sp.data(), nsrc, bytes, dev, true, s, s_staged));
    P2G_TRY(stage(ctx, ctx->out_copy, dp.data(), ndst, bytes, dev, true, d, d_staged));
    P2G_TRY(matrix_muladd(ctx, s, d, coeff.data(), bytes, 1));
    if (d_staged)
        P2G_TRY(unstage(ctx, dp.data(), d, ndst, bytes, dev));
    return finish(ctx);
}

int p2g_muladd(p2g_ctx *ctx, uint16_t *dst, const uint16_t *src, size_t n, uint16_t c,
               uint32_t flags)
{
    if (c == 0 || n == 0) {
        clear_error();
        return ctx ? P2G_OK : P2G_EINVAL;
    }
    const uint16_t *row = &c;
    return p2g_muladd_region(ctx, &dst, 1, &src, 1, &row, 0, n, flags);
}

int p2g_mul_slice(p2g_ctx *ctx, uint16_t c, uint16_t *data, size_t n, uint32_t flags)
{
    clear_error();
    if (!ctx || (n && !data)) {
        set_error("p2g_mul_slice: null argument");
        return P2G_EINVAL;
    }
    if (n == 0)
        return P2G_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    begin(ctx);
    const bool dev = flags & P2G_DEVICE_PTRS;
    const size_t bytes = n * 2;
    const uint8_t *in = reinterpret_cast<const uint8_t *>(data);
    std::vector<uint8_t *> s;
    bool staged = false;
    P2G_TRY(stage(ctx, ctx->in_copy, &in, 1, bytes, dev, true, s, staged));
    // in place: the planes are taken before the product is stored
    P2G_TRY(matrix_muladd(ctx, s, s, &c, bytes, 0));
    if (staged) {
        uint8_t *user = reinterpret_cast<uint8_t *>(data);
        P2G_TRY(unstage(ctx, &user, s, 1, bytes, dev));
    }
    return finish(ctx);
}

int p2g_invert(p2g_ctx *ctx, size_t m, const uint16_t *A, uint16_t *inv)
{
    clear_error();
    if (!ctx || (m && (!A || !inv))) {
        set_error("p2g_invert: null argument");
        return P2G_EINVAL;
    }
    if (m > 65535) {
        set_error("p2g_invert: m = %zu beyond 65535", m);
        return P2G_ERANGE;
    }
    if (m == 0)
        return P2G_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    begin(ctx);
    P2G_TRY(ctx->coeffs.ensure(m * m * 2));
    P2G_TRY(ctx->inv.ensure(m * m * 2));
    P2G_CUDA(cudaMemcpyAsync(ctx->coeffs.p, A, m * m * 2, cudaMemcpyHostToDevice, ctx->stream));
    GjWork w{ctx->gj_M, ctx->gj_status};
    P2G_TRY(gj_invert(ctx, w, static_cast<int>(m), nullptr, nullptr, nullptr, ctx->coeffs.as<uint16_t>(),
                      ctx->inv.as<uint16_t>()));
    int singular = 0;
    P2G_TRY(gj_status(ctx, w, &singular));
    if (singular) {
        set_error("Singular matrix");
        return P2G_ESINGULAR;
    }
    P2G_CUDA(cudaMemcpyAsync(inv, ctx->inv.p, m * m * 2, cudaMemcpyDeviceToHost, ctx->stream));
    return finish(ctx);
}

static int check_missing(size_t k, const uint64_t *missing, size_t m)
{
    for (size_t j = 0; j < m; ++j) {
        if (missing[j] >= k || (j && missing[j] <= missing[j - 1])) {
            set_error("missing indices must be strictly ascending and below k = %zu", k);
            return P2G_EINVAL;
        }
    }
    return P2G_OK;
}

int p2g_reconstruction_matrix(p2g_ctx *ctx, size_t k, const uint64_t *missing, size_t m,
                              const uint32_t *exps, uint16_t *inv)
{
    clear_error();
    if (!ctx || (m && (!missing || !exps || !inv))) {
        set_error("p2g_reconstruction_matrix: null argument");
        return P2G_EINVAL;
    }
    if (k > 65535 || m > k) {
        set_error("p2g_reconstruction_matrix: k = %zu, m = %zu out of range", k, m);
        return P2G_ERANGE;
    }
    P2G_TRY(check_missing(k, missing, m));
    if (m == 0)
        return P2G_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    begin(ctx);
    std::vector<uint16_t> c(k);
    par2_constants(k, c.data());
    ParamLayout L(0, 0, m * 2, m * 4);
    P2G_TRY(ctx->hparams.ensure(L.total));
    P2G_TRY(ctx->params.ensure(L.total));
    uint8_t *h = ctx->hparams.as<uint8_t>();
    for (size_t j = 0; j < m; ++j)
        reinterpret_cast<uint16_t *>(h + L.a_off)[j] = c[missing[j]];
    memcpy(h + L.b_off, exps, m * 4);
    P2G_TRY(upload_params(ctx, L));
    uint8_t *dp = ctx->params.as<uint8_t>();
    P2G_TRY(ctx->inv.ensure(m * m * 2));
    GjWork w{ctx->gj_M, ctx->gj_status};
    P2G_TRY(gj_invert(ctx, w, static_cast<int>(m), reinterpret_cast<const uint16_t *>(dp + L.a_off),
                      reinterpret_cast<const uint32_t *>(dp + L.b_off), exps, nullptr,
                      ctx->inv.as<uint16_t>()));
    int singular = 0;
    P2G_TRY(gj_status(ctx, w, &singular));
    if (singular) {
        set_error("Singular matrix");
        return P2G_ESINGULAR;
    }
    P2G_CUDA(cudaMemcpyAsync(inv, ctx->inv.p, m * m * 2, cudaMemcpyDeviceToHost, ctx->stream));
    return finish(ctx);
}

// Column slabs of a host-buffer repair's last input groups: each slab's
// present columns go up, both passes run on the slab, and its finished
// output columns go back while the next slab uploads.
struct RepairTail {
    int slabs = 0;             // 0: no slabs
    int groups = 0;            // upload groups in the tail
    size_t t0 = 0, ntail = 0;  // the tail's present slices [t0, t0 + ntail)
    std::vector<size_t> cut;   // slab q: columns [cut[q], cut[q + 1])
    size_t tab_off = 0;        // per slab: ntail inputs, m RHS, m outputs (device pointers)
    const uint8_t *const *present = nullptr;  // the caller's host slices
    const std::vector<uint8_t *> *ps = nullptr;  // their device copies
};

static int repair_passes(p2g_ctx *ctx, size_t m, size_t np, size_t slice_bytes, int groups,
                         uint8_t *dp, const ParamLayout &L, size_t exps_off,
                         const uint32_t *exps, uint8_t *const *out,
                         const std::vector<uint8_t *> &os, bool o_st, bool dev,
                         const RepairTail &tail);

int p2g_repair(p2g_ctx *ctx, size_t k, size_t slice_bytes, const uint64_t *missing, size_t m,
               const uint8_t *const *present, const uint32_t *exps,
               const uint8_t *const *recovery, uint8_t *const *out, uint32_t flags)
{
    clear_error();
    if (!ctx || (m && (!missing || !exps || !recovery || !out)) || (k > m && !present)) {
        set_error("p2g_repair: null argument");
        return P2G_EINVAL;
    }
    if (slice_bytes == 0 || slice_bytes % 2) {
        set_error("p2g_repair: slice size %zu must be even and non-zero", slice_bytes);
        return P2G_EINVAL;
    }
    if (k > 65535 || m > k) {
        set_error("p2g_repair: k = %zu, m = %zu out of range", k, m);
        return P2G_ERANGE;
    }
    P2G_TRY(check_missing(k, missing, m));
    if (m == 0)
        return P2G_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    begin(ctx);
    const bool dev = flags & P2G_DEVICE_PTRS;
    const size_t np = k - m;
    std::vector<uint16_t> c(k);
    par2_constants(k, c.data());
    std::vector<uint16_t> cpres, cmiss(m);
    cpres.reserve(np);
    {
        size_t j = 0;
        for (size_t i = 0; i < k; ++i) {
            if (j < m && missing[j] == i)
                cmiss[j++] = c[i];
            else
                cpres.push_back(c[i]);
        }
    }
    // slices: present data and recovery inputs, outputs.  Host present
    // slices (128 or more) go up in groups on the copy stream instead, while
    // the inversion and the earlier groups' multiply-accumulate run.
    const int groups =
        (!dev && np >= 128) ? static_cast<int>(std::min<size_t>(p2g_ctx::kPipe, np / 64)) : 1;
    std::vector<uint8_t *> ps, os;
    bool p_st = false, o_st = false;
    P2G_TRY(stage(ctx, ctx->in_copy, present, np, slice_bytes, dev, groups == 1, ps, p_st));
    // the right-hand sides start as copies of the recovery slices
    const size_t slot = round16(slice_bytes);
    P2G_TRY(ctx->rhs.ensure(slot * m));
    std::vector<uint8_t *> rhs(m);
    for (size_t j = 0; j < m; ++j)
        rhs[j] = ctx->rhs.as<uint8_t>() + j * slot;
    P2G_TRY(copy_slices(rhs.data(), recovery, m, slice_bytes,
                        dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
    P2G_TRY(stage(ctx, ctx->out_copy, out, m, slice_bytes, dev, false, os, o_st));
    // With host outputs, the last groups of present slices run slab by slab
    // (as in p2g_encode): what remains after the last upload is one slab's
    // passes and read-back instead of the whole second pass and the
    // read-back of every output.  Slabs about fill the device each.
    RepairTail tail;
    const size_t tiles = (slice_bytes + 2047) / 2048;
    if (groups >= 4 && o_st) {
        // the last kTailGroups groups (measured on 2048 x 1 MiB, m = 205:
        // 45.1 ms with 2, 46.7 with 4, 47.7 with 6; 48.8 without slabs)
        const int tg = std::min(kTailGroups, groups - 1);
        const p2g::MuladdPlan tp = p2g::choose_plan(
            ctx, static_cast<int>(np / groups * tg), static_cast<int>(m), slice_bytes);
        const double waves = static_cast<double>(p2g::plan_tiles(tp, slice_bytes)) * tp.nblk /
                             p2g::plan_slots(ctx, tp);
        int slabs = static_cast<int>(std::min<double>(kMaxTailSlabs - 1, std::floor(waves + 0.5)));
        if (slabs >= 2 && static_cast<size_t>(slabs) <= tiles) {
            for (int q = 0; q <= slabs; ++q)
                tail.cut.push_back(q == slabs ? slice_bytes : tiles * q / slabs * 2048);
            // the last slab in two halves (see p2g_encode)
            const size_t a = tail.cut[slabs - 1] / 2048;
            if (tiles - a >= 2)
                tail.cut.insert(tail.cut.end() - 1, (a + (tiles - a) / 2) * 2048);
            tail.slabs = static_cast<int>(tail.cut.size()) - 1;
            tail.groups = tg;
            tail.t0 = np * (groups - tg) / groups;
            tail.ntail = np - tail.t0;
            tail.present = present;
            tail.ps = &ps;
        }
    }
    const size_t tail_bytes =
        tail.slabs ? tail.slabs * (tail.ntail + 2 * m) * sizeof(void *) : 0;
    // parameter block: [present ptrs][rhs ptrs | out ptrs][cmiss | exps | cpres | slab tables]
    ParamLayout L(np, 2 * m, m * 2 + m * 4 + 16, round16(np * 2) + tail_bytes);
    P2G_TRY(ctx->hparams.ensure(L.total));
    P2G_TRY(ctx->params.ensure(L.total));
    uint8_t *h = ctx->hparams.as<uint8_t>();
    memcpy(h + L.src_off, ps.data(), np * sizeof(void *));
    memcpy(h + L.dst_off, rhs.data(), m * sizeof(void *));
    memcpy(h + L.dst_off + m * sizeof(void *), os.data(), m * sizeof(void *));
    const size_t exps_off = L.a_off + round16(m * 2);
    memcpy(h + L.a_off, cmiss.data(), m * 2);
    memcpy(h + exps_off, exps, m * 4);
    if (np)
        memcpy(h + L.b_off, cpres.data(), np * 2);
    if (tail.slabs) {
        tail.tab_off = L.b_off + round16(np * 2);
        uint8_t **t = reinterpret_cast<uint8_t **>(h + tail.tab_off);
        for (int q = 0; q < tail.slabs; ++q) {
            for (size_t i = 0; i < tail.ntail; ++i)
                *t++ = ps[tail.t0 + i] + tail.cut[q];
            for (size_t j = 0; j < m; ++j)
                *t++ = rhs[j] + tail.cut[q];
            for (size_t j = 0; j < m; ++j)
                *t++ = os[j] + tail.cut[q];
        }
    }
    P2G_TRY(upload_params(ctx, L));
    uint8_t *dp = ctx->params.as<uint8_t>();
    if (groups > 1) {
        // after everything already queued on the compute stream (earlier
        // users of the staging buffers); the tail groups go up slab by slab
        // in repair_passes
        P2G_CUDA(cudaEventRecord(ctx->pipe_ev[0], ctx->stream));
        P2G_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->pipe_ev[0], 0));
        for (int g = 0; g < (tail.slabs ? groups - tail.groups : groups); ++g) {
            const size_t i0 = np * g / groups, i1 = np * (g + 1) / groups;
            const int rc = copy_slices(ps.data() + i0, present + i0, i1 - i0, slice_bytes,
                                       cudaMemcpyHostToDevice, ctx->copy_stream);
            if (rc != P2G_OK || cudaEventRecord(ctx->pipe_ev[g], ctx->copy_stream) != cudaSuccess) {
                cudaStreamSynchronize(ctx->copy_stream);
                if (rc == P2G_OK)
                    set_error("cudaEventRecord failed");
                return rc != P2G_OK ? rc : P2G_ECUDA;
            }
        }
    }
    // every return below waits for the uploads still reading the caller's
    // present slices
    const int rc = repair_passes(ctx, m, np, slice_bytes, groups, dp, L, exps_off, exps, out, os,
                                 o_st, dev, tail);
    if (groups > 1) {
        cudaStreamSynchronize(ctx->copy_stream);
        if (tail.slabs)
            cudaStreamSynchronize(ctx->d2h_stream);
    }
    return rc;
}

// Steps 1-3 of p2g_repair once its slices and parameters are in place.
static int repair_passes(p2g_ctx *ctx, size_t m, size_t np, size_t slice_bytes, int groups,
                         uint8_t *dp, const ParamLayout &L, size_t exps_off,
                         const uint32_t *exps, uint8_t *const *out,
                         const std::vector<uint8_t *> &os, bool o_st, bool dev,
                         const RepairTail &tail)
{
    const uint32_t *d_exps = reinterpret_cast<const uint32_t *>(dp + exps_off);
    // 1. A^-1 on the device
    P2G_TRY(ctx->inv.ensure(m * m * 2));
    GjWork w{ctx->gj_M, ctx->gj_status};
    P2G_TRY(gj_invert(ctx, w, static_cast<int>(m), reinterpret_cast<const uint16_t *>(dp + L.a_off),
                      d_exps, exps, nullptr, ctx->inv.as<uint16_t>()));
    int singular = 0;
    P2G_TRY(gj_status(ctx, w, &singular));
    if (singular) {
        set_error("Singular matrix");
        return P2G_ESINGULAR;
    }
    // 2. RHS = R ^ V * present (by input groups as their uploads land)
    if (np) {
        P2G_TRY(ctx->recs.ensure(record_bytes(np, static_cast<int>(m))));
        P2G_TRY(records_par2(ctx, reinterpret_cast<const uint16_t *>(dp + L.b_off), d_exps,
                             static_cast<int>(np), static_cast<int>(m), ctx->recs.as<uint32_t>()));
        const uint8_t *const *d_src = reinterpret_cast<const uint8_t *const *>(dp + L.src_off);
        const size_t rw = static_cast<size_t>(record_words(static_cast<int>(m)));
        const int full = tail.slabs ? groups - tail.groups : groups;
        for (int g = 0; g < full; ++g) {
            const size_t i0 = np * g / groups, i1 = np * (g + 1) / groups;
            if (groups > 1)
                P2G_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->pipe_ev[g], 0));
            P2G_TRY(muladd_run(ctx, d_src + i0, static_cast<int>(i1 - i0),
                               reinterpret_cast<uint8_t *const *>(dp + L.dst_off),
                               static_cast<int>(m), slice_bytes,
                               ctx->recs.as<uint32_t>() + i0 * m * rw, 1));
        }
    }
    // 3. missing = A^-1 * RHS
    P2G_TRY(ctx->recs2.ensure(record_bytes(m, static_cast<int>(m))));
    P2G_TRY(records_from_matrix(ctx, ctx->inv.as<uint16_t>(), static_cast<int>(m),
                                static_cast<int>(m), ctx->recs2.as<uint32_t>()));
    if (!tail.slabs) {
        P2G_TRY(muladd_run(ctx, reinterpret_cast<const uint8_t *const *>(dp + L.dst_off),
                           static_cast<int>(m),
                           reinterpret_cast<uint8_t *const *>(dp + L.dst_off + m * sizeof(void *)),
                           static_cast<int>(m), slice_bytes, ctx->recs2.as<uint32_t>(), 0));
        if (o_st)
            P2G_TRY(unstage(ctx, out, os, m, slice_bytes, dev));
        return finish(ctx);
    }
    // Tail slabs: the slab's present columns go up, step 2 finishes the
    // slab's right-hand sides, step 3 forms its missing columns, which go
    // back on the read-back stream while the next slab uploads.  (A failed
    // step returns after the copies already enqueued, see p2g_repair.)
    const size_t rw = static_cast<size_t>(record_words(static_cast<int>(m)));
    uint8_t *const *tab = reinterpret_cast<uint8_t *const *>(dp + tail.tab_off);
    const size_t per = tail.ntail + 2 * m;
    std::vector<const uint8_t *> hs(tail.ntail);
    std::vector<uint8_t *> ds(tail.ntail), uo(m), so(m);
    cudaEvent_t *up = ctx->pipe_ev + kSlabEvents, *done = up + tail.slabs;
    for (int q = 0; q < tail.slabs; ++q) {
        const size_t c0 = tail.cut[q], w = tail.cut[q + 1] - c0;
        for (size_t i = 0; i < tail.ntail; ++i) {
            hs[i] = tail.present[tail.t0 + i] + c0;
            ds[i] = (*tail.ps)[tail.t0 + i] + c0;
        }
        P2G_TRY(copy_slices(ds.data(), hs.data(), tail.ntail, w, cudaMemcpyHostToDevice,
                            ctx->copy_stream));
        P2G_CUDA(cudaEventRecord(up[q], ctx->copy_stream));
        P2G_CUDA(cudaStreamWaitEvent(ctx->stream, up[q], 0));
        uint8_t *const *qt = tab + q * per;
        P2G_TRY(muladd_run(ctx, reinterpret_cast<const uint8_t *const *>(qt),
                           static_cast<int>(tail.ntail), qt + tail.ntail, static_cast<int>(m), w,
                           ctx->recs.as<uint32_t>() + tail.t0 * m * rw, 1));
        P2G_TRY(muladd_run(ctx, reinterpret_cast<const uint8_t *const *>(qt + tail.ntail),
                           static_cast<int>(m), qt + tail.ntail + m, static_cast<int>(m), w,
                           ctx->recs2.as<uint32_t>(), 0));
        P2G_CUDA(cudaEventRecord(done[q], ctx->stream));
        P2G_CUDA(cudaStreamWaitEvent(ctx->d2h_stream, done[q], 0));
        for (size_t j = 0; j < m; ++j) {
            uo[j] = out[j] + c0;
            so[j] = os[j] + c0;
        }
        P2G_TRY(copy_slices(uo.data(), so.data(), m, w, cudaMemcpyDeviceToHost, ctx->d2h_stream));
    }
    // the call ends when the last read-back has landed
    P2G_CUDA(cudaEventRecord(done[tail.slabs], ctx->d2h_stream));
    P2G_CUDA(cudaStreamWaitEvent(ctx->stream, done[tail.slabs], 0));
    return finish(ctx);
}

static int hash_common(p2g_ctx *ctx, const uint8_t *const *slices, size_t n, size_t S,
                       uint32_t flags, std::vector<uint8_t> &md5, std::vector<uint32_t> &crc)
{
    const bool dev = flags & P2G_DEVICE_PTRS;
    std::vector<uint8_t *> sp;
    bool staged = false;
    P2G_TRY(stage(ctx, ctx->in_copy, slices, n, S, dev, true, sp, staged));
    ParamLayout L(n, 0, 0, 0);
    P2G_TRY(ctx->hparams.ensure(L.total));
    P2G_TRY(ctx->params.ensure(L.total));
    memcpy(ctx->hparams.p, sp.data(), n * sizeof(void *));
    P2G_TRY(upload_params(ctx, L));
    P2G_TRY(ctx->hash_out.ensure(round16(n * 16) + n * 4));
    uint8_t *d_md5 = ctx->hash_out.as<uint8_t>();
    uint32_t *d_crc = reinterpret_cast<uint32_t *>(d_md5 + round16(n * 16));
    ctx->mark(1);
    ctx->mark(2);
    P2G_TRY(hash_run(ctx, reinterpret_cast<const uint8_t *const *>(ctx->params.p),
                     static_cast<int>(n), S, d_md5, d_crc));
    ctx->mark(3);
    md5.resize(n * 16);
    crc.resize(n);
    P2G_CUDA(cudaMemcpyAsync(md5.data(), d_md5, n * 16, cudaMemcpyDeviceToHost, ctx->stream));
    P2G_CUDA(cudaMemcpyAsync(crc.data(), d_crc, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    return finish(ctx);
}

int p2g_hash_slices(p2g_ctx *ctx, const uint8_t *const *slices, size_t n, size_t slice_bytes,
                    uint8_t *md5_out, uint32_t *crc_out, uint32_t flags)
{
    clear_error();
    if (!ctx || (n && (!slices || !md5_out || !crc_out))) {
        set_error("p2g_hash_slices: null argument");
        return P2G_EINVAL;
    }
    if (n > 0x7fffffff) {
        set_error("p2g_hash_slices: too many slices");
        return P2G_ERANGE;
    }
    if (n == 0)
        return P2G_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    begin(ctx);
    std::vector<uint8_t> md5;
    std::vector<uint32_t> crc;
    P2G_TRY(hash_common(ctx, slices, n, slice_bytes, flags, md5, crc));
    memcpy(md5_out, md5.data(), n * 16);
    memcpy(crc_out, crc.data(), n * 4);
    return P2G_OK;
}

int p2g_verify_slices(p2g_ctx *ctx, const uint8_t *const *slices, size_t n, size_t slice_bytes,
                      const uint8_t *md5_expect, const uint32_t *crc_expect, uint8_t *ok_out,
                      uint32_t flags)
{
    clear_error();
    if (!ctx || (n && (!slices || !md5_expect || !crc_expect || !ok_out))) {
        set_error("p2g_verify_slices: null argument");
        return P2G_EINVAL;
    }
    if (n > 0x7fffffff) {
        set_error("p2g_verify_slices: too many slices");
        return P2G_ERANGE;
    }
    if (n == 0)
        return P2G_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    begin(ctx);
    std::vector<uint8_t> md5;
    std::vector<uint32_t> crc;
    P2G_TRY(hash_common(ctx, slices, n, slice_bytes, flags, md5, crc));
    for (size_t i = 0; i < n; ++i)
        ok_out[i] = crc[i] == crc_expect[i] && memcmp(&md5[i * 16], md5_expect + i * 16, 16) == 0;
    return P2G_OK;
}

}  // extern "C"
