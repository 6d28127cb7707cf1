// batch.cu -- batches of independent create / repair / verify jobs.
//
// Many recovery sets of uneven file sizes, slice sizes and redundancy run
// together: every REPAIR job's decode matrix is formed first (K2), then two
// phases of multiply-accumulate work each run as ONE persistent kernel over a
// queue of (problem, column tile, output block, input split) items sorted
// longest first:
//   phase A: CREATE jobs (sources -> recovery slices) and the first REPAIR
//            pass (RHS = recovery ^ V * present, into scratch);
//   phase B: the second REPAIR pass (missing = A^-1 * RHS).
// VERIFY jobs are hashed by one launch per distinct slice size.  The device
// work can be captured once into a CUDA graph and replayed.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "hash.cuh"
#include "invert.cuh"
#include "muladd.cuh"

using namespace p2g;

namespace {

size_t al256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }
size_t al16(size_t n) { return (n + 15) & ~static_cast<size_t>(15); }

// Host image of the batch's device tables, laid out with 256-byte alignment.
struct Image {
    std::vector<uint8_t> bytes;
    size_t put(const void *p, size_t n)
    {
        const size_t off = al256(bytes.size());
        bytes.resize(off + al256(n ? n : 1));
        if (p && n)
            memcpy(bytes.data() + off, p, n);
        return off;
    }
};

struct HashGroup {
    size_t ptr_off;  // device table of slice pointers
    size_t S;
    int n;
    size_t out_off;  // into hash buffer: md5 (n*16), then crc (n*4)
    std::vector<std::pair<int, int>> slices;  // (job, slice index) of each entry
};

struct Phase {
    size_t planes_off = 0, rec_off = 0, prob_off = 0, item_off = 0, zero_ptr_off = 0,
           zero_len_off = 0;
    int nplanes = 0, nrec = 0, nitems = 0, nzero = 0, grid = 0;
    unsigned long long planes_total = 0, rec_total = 0;
};

}  // namespace

struct p2g_batch {
    p2g_ctx *ctx = nullptr;
    p2g_job *jobs = nullptr;
    size_t njobs = 0;
    DevBuf params, hparams, planes, recs, rhs, inv, hashbuf;
    Phase A, B;
    size_t copy_src_off = 0, copy_dst_off = 0, copy_len_off = 0, counter_off = 0;
    int ncopy = 0;
    std::vector<HashGroup> hash;
    size_t hash_bytes = 0;  // MD5 + CRC results of all groups
    DevBuf hash_host;  // pinned
    DevBuf abort_buf;  // device word the persistent kernels poll (p2g_batch_cancel)
    int *abort_dev = nullptr;
    std::atomic<bool> cancelled{false};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t done = nullptr;
    bool launched = false;
    bool recorded = false;  // `done` has been recorded at least once
};

namespace {

uint8_t *dp(p2g_batch *b, size_t off) { return b->params.as<uint8_t>() + off; }

constexpr size_t kMaxSpare = 32;

// Gives `d` (empty on entry) at least `need` bytes: the smallest spare buffer
// of the context that fits, else a new allocation with 25 % headroom so that
// batches of similar size reuse it.  ctx->mu must be held.
int take(p2g_ctx *ctx, DevBuf &d, size_t need)
{
    if (need <= d.cap)
        return P2G_OK;
    size_t best = ctx->spare.size();
    for (size_t i = 0; i < ctx->spare.size(); ++i) {
        const DevBuf &x = ctx->spare[i];
        if (x.pinned == d.pinned && x.cap >= need &&
            (best == ctx->spare.size() || x.cap < ctx->spare[best].cap))
            best = i;
    }
    if (best < ctx->spare.size()) {
        d.release();
        d = ctx->spare[best];
        ctx->spare.erase(ctx->spare.begin() + static_cast<long>(best));
        return P2G_OK;
    }
    return d.ensure(need + need / 4);
}

// Returns `d` to the context's spares (the GPU no longer uses it); beyond
// kMaxSpare buffers the smallest ones are freed.  ctx->mu must be held.
void give(p2g_ctx *ctx, DevBuf &d)
{
    if (d.p)
        ctx->spare.push_back(d);
    d = DevBuf{};
    while (ctx->spare.size() > kMaxSpare) {
        size_t small = 0;
        for (size_t i = 1; i < ctx->spare.size(); ++i)
            if (ctx->spare[i].cap < ctx->spare[small].cap)
                small = i;
        ctx->spare[small].release();
        ctx->spare.erase(ctx->spare.begin() + static_cast<long>(small));
    }
}

// Frees a batch.  Its buffers go back to the context only once every
// operation that touches them has completed (b->done is recorded after the
// create-time uploads and again after each launch).  ctx->mu must be held.
void batch_free(p2g_batch *b)
{
    if (b->done && b->recorded)
        cudaEventSynchronize(b->done);
    if (b->exec)
        cudaGraphExecDestroy(b->exec);
    if (b->graph)
        cudaGraphDestroy(b->graph);
    if (b->done)
        cudaEventDestroy(b->done);
    DevBuf *bufs[] = {&b->params, &b->hparams, &b->planes,    &b->recs,     &b->rhs,
                      &b->inv,    &b->hashbuf, &b->hash_host, &b->abort_buf};
    for (DevBuf *d : bufs) {
        if (b->ctx)
            give(b->ctx, *d);
        else
            d->release();
    }
    delete b;
}

int enqueue(p2g_batch *b)
{
    p2g_ctx *ctx = b->ctx;
    cudaStream_t st = ctx->stream;
    P2G_CUDA(cudaMemsetAsync(dp(b, b->counter_off), 0, 2 * sizeof(int), st));
    P2G_CUDA(cudaMemsetAsync(b->abort_dev, 0, sizeof(int), st));
    P2G_TRY(batch_copy(st, reinterpret_cast<const uint8_t *const *>(dp(b, b->copy_src_off)),
                       reinterpret_cast<uint8_t *const *>(dp(b, b->copy_dst_off)),
                       reinterpret_cast<const unsigned long long *>(dp(b, b->copy_len_off)),
                       b->ncopy));
    Phase *ph[2] = {&b->A, &b->B};
    for (int x = 0; x < 2; ++x) {
        Phase &P = *ph[x];
        if (!P.nitems)
            continue;
        P2G_TRY(batch_planes(st, reinterpret_cast<const PlanesProb *>(dp(b, P.planes_off)),
                             P.nplanes, P.planes_total));
        P2G_TRY(batch_records(st, ctx->d_log, ctx->d_exp,
                              reinterpret_cast<const RecProb *>(dp(b, P.rec_off)), P.nrec,
                              P.rec_total));
        P2G_TRY(batch_zero(st, reinterpret_cast<uint8_t *const *>(dp(b, P.zero_ptr_off)),
                           reinterpret_cast<const unsigned long long *>(dp(b, P.zero_len_off)),
                           P.nzero));
        if (x == 0)
            ctx->mark(2);
        P2G_TRY(batch_muladd(st, P.grid, reinterpret_cast<const BatchProb *>(dp(b, P.prob_off)),
                             reinterpret_cast<const BatchItem *>(dp(b, P.item_off)), P.nitems,
                             reinterpret_cast<int *>(dp(b, b->counter_off)) + x, b->abort_dev));
        ctx->launches += 4;
    }
    ctx->mark(3);
    for (const HashGroup &g : b->hash) {
        uint8_t *out = b->hashbuf.as<uint8_t>() + g.out_off;
        P2G_TRY(hash_run(ctx, reinterpret_cast<const uint8_t *const *>(dp(b, g.ptr_off)), g.n, g.S,
                         out, reinterpret_cast<uint32_t *>(out + al16(static_cast<size_t>(g.n) * 16))));
    }
    return P2G_OK;
}

// Per-problem description gathered while scanning the jobs.
struct Prob {
    int phase;
    size_t src_off, dst_off;        // param offsets of the pointer arrays
    int nin, nout;
    size_t S;
    int mode;
    // records: par2 (consts/exps offsets) or matrix (coeff device pointer)
    size_t consts_off, exps_off;
    const uint16_t *coeff;  // device
    int form;               // tile form of the persistent kernel (BatchForm)
};

// The tile form for a problem: the context's tuned form for its class if
// there is one, else small tables up to 24 outputs, the paired form above
// 104 (one table build per input serves up to 208 outputs) and the 8 + 8
// tables over 1024-symbol tiles between.
// Input splits of an item of `unit` cost when the queue aims at items of
// `target` cost (whole aligned words: S % 4 == 0; at least 16 inputs each).
int split_for(double unit, double target, int nin, size_t S)
{
    if (unit <= target || S % 4)
        return 1;
    const double ns = std::min<double>({std::ceil(unit / target), std::max(1.0, nin / 16.0), 64.0});
    return std::max(1, static_cast<int>(ns));
}

int form_for(const p2g_ctx *ctx, int nout, size_t S)
{
    const int f = ctx->batch_forms[batch_class(nout, S)];
    if (batch_form_valid(f, nout))
        return f;
    return nout <= 24 ? kFormSmall : nout > 104 ? kFormPaired : kFormWide;
}

// Times each valid form of the persistent kernel on `copies` synthetic
// problems of class `cls` in one launch (nin x nout each, slices of S bytes,
// shared sources and coefficients from a random matrix, outputs of their own,
// XORed into) and returns in *best_form the default form for nout unless
// another is at least 3 % faster.
int tune_class(p2g_ctx *ctx, int cls, int nin, int nout, size_t S, int copies, int reps,
               cudaEvent_t e0, cudaEvent_t e1, int *best_form, float *best_ms)
{
    cudaStream_t st = ctx->stream;
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    const int T = static_cast<int>((S + 2047) / 2048);
    P2G_TRY(ctx->in_copy.ensure(S * nin));
    P2G_TRY(ctx->out_copy.ensure(S * nout * copies));
    P2G_TRY(ctx->coeffs.ensure(static_cast<size_t>(nin) * nout * 2 + 16));
    P2G_TRY(ctx->recs.ensure(static_cast<size_t>(nin) * nout * kRecordWordsSmall * 4));
    P2G_TRY(ctx->planes.ensure(static_cast<size_t>(nin) * T * 2048));
    P2G_TRY(fill_synthetic(st, ctx->in_copy.p, S * nin, 11u + cls));
    P2G_TRY(fill_synthetic(st, ctx->coeffs.p, (static_cast<size_t>(nin) * nout * 2) & ~size_t(3),
                           29u + cls));
    std::vector<const uint8_t *> sp(nin);
    std::vector<uint8_t *> dv(static_cast<size_t>(nout) * copies);
    for (int i = 0; i < nin; ++i)
        sp[i] = ctx->in_copy.as<uint8_t>() + i * S;
    for (size_t o = 0; o < dv.size(); ++o)
        dv[o] = ctx->out_copy.as<uint8_t>() + o * S;
    float times[kBatchForms];
    for (float &t : times)
        t = 1e30f;
    for (int f = 0; f < kBatchForms; ++f) {
        if (!batch_form_valid(f, nout))
            continue;
        const int blk = batch_block(f);
        const int nblk = (nout + blk - 1) / blk;
        const int tiles = static_cast<int>((S + batch_tile_bytes(f) - 1) / batch_tile_bytes(f));
        const double unit = static_cast<double>(nin) * batch_item_cost(f, std::min(nout, blk));
        const double target = std::max(1.0, unit * tiles * nblk * copies / (4.0 * sms));
        const int ns = split_for(unit, target, nin, S);
        std::vector<BatchItem> items;
        for (int c = 0; c < copies; ++c)
            for (int t = 0; t < tiles; ++t)
                for (int ob = 0; ob < nblk; ++ob)
                    for (int x = 0; x < ns; ++x)
                        items.push_back(BatchItem{c, t, ob, x});
        // upload image: pointer tables, counter + abort word, problem tables, items
        Image img;
        const size_t src_off = img.put(sp.data(), nin * sizeof(void *));
        const size_t dst_off = img.put(dv.data(), dv.size() * sizeof(void *));
        const size_t ctr_off = img.put(nullptr, 64);
        const size_t pl_off = img.put(nullptr, sizeof(PlanesProb));
        const size_t rc_off = img.put(nullptr, sizeof(RecProb));
        const size_t bp_off = img.put(nullptr, copies * sizeof(BatchProb));
        const size_t it_off = img.put(items.data(), items.size() * sizeof(BatchItem));
        P2G_TRY(ctx->params.ensure(img.bytes.size()));
        uint8_t *base = ctx->params.as<uint8_t>();
        PlanesProb pp{};
        pp.src = reinterpret_cast<const uint8_t *const *>(base + src_off);
        pp.planes = ctx->planes.as<uint32_t>();
        pp.S = S;
        pp.nin = nin;
        pp.T = T;
        RecProb rp{};
        rp.coeff = ctx->coeffs.as<uint16_t>();
        rp.recs = ctx->recs.as<uint32_t>();
        rp.nin = nin;
        rp.nout = nout;
        rp.small = f == kFormSmall;
        BatchProb bp{};
        bp.planes = pp.planes;
        bp.recs = rp.recs;
        bp.dst = reinterpret_cast<uint8_t *const *>(base + dst_off);
        bp.S = S;
        bp.nin = nin;
        bp.nout = nout;
        bp.T = T;
        bp.nblk = nblk;
        bp.nsplit = ns;
        bp.mode = 1;
        bp.form = f;
        memcpy(img.bytes.data() + pl_off, &pp, sizeof pp);
        memcpy(img.bytes.data() + rc_off, &rp, sizeof rp);
        for (int c = 0; c < copies; ++c) {
            bp.dst = reinterpret_cast<uint8_t *const *>(base + dst_off) +
                     static_cast<size_t>(c) * nout;
            memcpy(img.bytes.data() + bp_off + c * sizeof bp, &bp, sizeof bp);
        }
        // a pageable source: the copy has read it when the call returns
        P2G_CUDA(cudaMemcpyAsync(base, img.bytes.data(), img.bytes.size(), cudaMemcpyHostToDevice, st));
        P2G_CUDA(cudaMemsetAsync(base + ctr_off, 0, 64, st));
        P2G_TRY(batch_planes(st, reinterpret_cast<const PlanesProb *>(base + pl_off), 1,
                             static_cast<unsigned long long>(nin) * T * 32));
        P2G_TRY(batch_records(st, ctx->d_log, ctx->d_exp,
                              reinterpret_cast<const RecProb *>(base + rc_off), 1,
                              static_cast<unsigned long long>(nin) * nout));
        int *counter = reinterpret_cast<int *>(base + ctr_off);
        const volatile int *abort_word = counter + 8;
        const int grid = static_cast<int>(std::min<size_t>(items.size(), sms));
        float t_best = 1e30f;
        for (int r = 0; r <= reps; ++r) {  // the first launch warms up
            P2G_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), st));
            P2G_CUDA(cudaEventRecord(e0, st));
            P2G_TRY(batch_muladd(st, grid, reinterpret_cast<const BatchProb *>(base + bp_off),
                                 reinterpret_cast<const BatchItem *>(base + it_off),
                                 static_cast<int>(items.size()), counter, abort_word));
            P2G_CUDA(cudaEventRecord(e1, st));
            P2G_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            P2G_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (r > 0)
                t_best = std::min(t_best, ms);
        }
        times[f] = t_best;
    }
    // the default form for this output count stays unless another is at
    // least 3 % faster (a closer margin is within the timing noise)
    const int dflt = nout <= 24 ? kFormSmall : nout > 104 ? kFormPaired : kFormWide;
    *best_form = dflt;
    *best_ms = times[dflt];
    for (int f = 0; f < kBatchForms; ++f)
        if (times[f] < 0.97f * times[dflt] && times[f] < *best_ms) {
            *best_form = f;
            *best_ms = times[f];
        }
    return P2G_OK;
}

}  // namespace

extern "C" {

int p2g_batch_create(p2g_ctx *ctx, p2g_job *jobs, size_t njobs, uint32_t flags, p2g_batch **out)
{
    clear_error();
    if (!ctx || !out || (njobs && !jobs)) {
        set_error("p2g_batch_create: null argument");
        return P2G_EINVAL;
    }
    *out = nullptr;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    ctx->launches = 0;
    for (bool &m : ctx->ev_marked)
        m = false;
    // ---- validation ----
    for (size_t j = 0; j < njobs; ++j) {
        p2g_job &J = jobs[j];
        J.status = P2G_OK;
        const size_t cb = J.col_begin, ce = J.col_end ? J.col_end : J.slice_bytes;
        bool bad = J.slice_bytes == 0 || J.slice_bytes % 2 || cb % 2048 || ce > J.slice_bytes ||
                   cb >= ce || ce % 2 || J.k == 0 || J.k > 65535 || !J.src;
        if (J.kind == P2G_JOB_CREATE)
            bad = bad || J.n > 65535 || (J.n && (!J.exps || !J.out));
        else if (J.kind == P2G_JOB_REPAIR)
            bad = bad || J.n == 0 || J.n > J.k || !J.exps || !J.missing || !J.recovery || !J.out;
        else if (J.kind == P2G_JOB_VERIFY)
            bad = bad || cb != 0 || ce != J.slice_bytes || !J.md5_out || !J.crc_out;
        else
            bad = true;
        if (J.kind == P2G_JOB_REPAIR && !bad)
            for (size_t q = 0; q < J.n; ++q)
                bad = bad || J.missing[q] >= J.k || (q && J.missing[q] <= J.missing[q - 1]);
        if (bad) {
            set_error("p2g_batch_create: job %zu is malformed", j);
            return P2G_EINVAL;
        }
        // the kernels move 16-byte vectors: every slice must start 16-byte aligned
        auto al = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
        bool aligned = true;
        const size_t nsrc = J.kind == P2G_JOB_REPAIR ? J.k - J.n : J.k;
        for (size_t i = 0; i < nsrc; ++i)
            aligned = aligned && J.src[i] && al(J.src[i]);
        if (J.kind != P2G_JOB_VERIFY)
            for (size_t e = 0; e < J.n; ++e)
                aligned = aligned && J.out[e] && al(J.out[e]) &&
                          (J.kind != P2G_JOB_REPAIR || (J.recovery[e] && al(J.recovery[e])));
        if (!aligned) {
            set_error("p2g_batch_create: job %zu has a null or non-16-byte-aligned slice pointer",
                      j);
            return P2G_EINVAL;
        }
    }
    p2g_batch *b = new p2g_batch();
    b->ctx = ctx;
    b->jobs = jobs;
    b->njobs = njobs;
    b->hparams.pinned = true;
    b->hash_host.pinned = true;
    if (cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess) {
        (void)cudaGetLastError();
        delete b;
        set_error("p2g_batch_create: cudaEventCreate failed");
        return P2G_ECUDA;
    }
    // on failure, wait for the uploads already queued before reusing buffers
    auto fail = [&](int rc) {
        if (cudaEventRecord(b->done, ctx->stream) == cudaSuccess)
            b->recorded = true;
        (void)cudaGetLastError();
        batch_free(b);
        return rc;
    };
    // the abort word (device memory), cleared by every launch
    if (int rc = take(ctx, b->abort_buf, 64))
        return fail(rc);
    b->abort_dev = b->abort_buf.as<int>();
    // ---- decode matrices of REPAIR jobs ----
    std::vector<size_t> inv_off(njobs, 0);
    size_t inv_bytes = 0;
    for (size_t j = 0; j < njobs; ++j)
        if (jobs[j].kind == P2G_JOB_REPAIR) {
            inv_off[j] = inv_bytes;
            inv_bytes += al256(jobs[j].n * jobs[j].n * 2);
        }
    if (int rc = take(ctx, b->inv, inv_bytes + 256))
        return fail(rc);
    std::vector<int> singular(njobs, 0);
    {
        std::vector<int> pending;
        DevBuf stat;
        if (int rc = take(ctx, stat, njobs * sizeof(int) + 16))
            return fail(rc);
        std::vector<uint8_t> h;
        for (size_t j = 0; j < njobs; ++j) {
            p2g_job &J = jobs[j];
            if (J.kind != P2G_JOB_REPAIR)
                continue;
            uint16_t *d_inv = reinterpret_cast<uint16_t *>(b->inv.as<uint8_t>() + inv_off[j]);
            if (J.inverse) {
                if (cudaMemcpyAsync(d_inv, J.inverse, J.n * J.n * 2, cudaMemcpyHostToDevice,
                                    ctx->stream) != cudaSuccess) {
                    set_error("p2g_batch_create: decode matrix upload failed");
                    give(ctx, stat);
                    return fail(P2G_ECUDA);
                }
                continue;
            }
            // constants of the missing slices and the exponents
            std::vector<uint16_t> c(J.k);
            par2_constants(J.k, c.data());
            const size_t m = J.n;
            h.assign(al256(m * 2) + m * 4, 0);
            for (size_t q = 0; q < m; ++q)
                reinterpret_cast<uint16_t *>(h.data())[q] = c[J.missing[q]];
            memcpy(h.data() + al256(m * 2), J.exps, m * 4);
            int rc = ctx->coeffs.ensure(h.size() + 16);
            if (rc == P2G_OK &&
                cudaMemcpyAsync(ctx->coeffs.p, h.data(), h.size(), cudaMemcpyHostToDevice,
                                ctx->stream) != cudaSuccess)
                rc = P2G_ECUDA;
            GjWork w{ctx->gj_M, ctx->gj_status};
            if (rc == P2G_OK)
                rc = gj_invert(ctx, w, static_cast<int>(m), ctx->coeffs.as<uint16_t>(),
                               reinterpret_cast<const uint32_t *>(ctx->coeffs.as<uint8_t>() +
                                                                  al256(m * 2)),
                               J.exps, nullptr, d_inv);
            if (rc == P2G_OK &&
                cudaMemcpyAsync(stat.as<int>() + j, ctx->gj_status.p, sizeof(int),
                                cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
                rc = P2G_ECUDA;
            // the pageable host source is consumed before the next iteration
            // reuses `h`, and ctx->coeffs before the next upload (stream order)
            if (rc != P2G_OK) {
                give(ctx, stat);
                return fail(rc);
            }
            pending.push_back(static_cast<int>(j));
        }
        if (!pending.empty()) {
            std::vector<int> st(njobs, 0);
            if (cudaMemcpyAsync(st.data(), stat.p, njobs * sizeof(int), cudaMemcpyDeviceToHost,
                                ctx->stream) != cudaSuccess ||
                cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
                set_error("p2g_batch_create: inversion failed: %s",
                          cudaGetErrorString(cudaGetLastError()));
                give(ctx, stat);
                return fail(P2G_ECUDA);
            }
            for (int j : pending)
                if (st[j]) {
                    singular[j] = 1;
                    jobs[j].status = P2G_ESINGULAR;
                }
        }
        give(ctx, stat);
    }
    // ---- problems ----
    Image img;
    std::vector<Prob> probs;
    std::vector<uint8_t *> copy_src, copy_dst;
    std::vector<unsigned long long> copy_len;
    size_t rhs_bytes = 0;
    std::vector<size_t> rhs_off(njobs, 0);
    for (size_t j = 0; j < njobs; ++j)
        if (jobs[j].kind == P2G_JOB_REPAIR && !singular[j]) {
            const size_t S = (jobs[j].col_end ? jobs[j].col_end : jobs[j].slice_bytes) - jobs[j].col_begin;
            rhs_off[j] = rhs_bytes;
            rhs_bytes += al256(jobs[j].n * al16(S));
        }
    if (int rc = take(ctx, b->rhs, rhs_bytes + 256))
        return fail(rc);
    std::vector<HashGroup> hg;
    for (size_t j = 0; j < njobs; ++j) {
        p2g_job &J = jobs[j];
        const size_t cb = J.col_begin;
        const size_t S = (J.col_end ? J.col_end : J.slice_bytes) - cb;
        if (J.kind == P2G_JOB_VERIFY) {
            HashGroup *g = nullptr;
            for (HashGroup &x : hg)
                if (x.S == S)
                    g = &x;
            if (!g) {
                hg.push_back(HashGroup());
                g = &hg.back();
                g->S = S;
                g->n = 0;
            }
            for (size_t i = 0; i < J.k; ++i)
                g->slices.push_back({static_cast<int>(j), static_cast<int>(i)});
            continue;
        }
        if (J.kind == P2G_JOB_CREATE) {
            if (J.n == 0)
                continue;
            std::vector<const uint8_t *> s(J.k);
            std::vector<uint8_t *> d(J.n);
            for (size_t i = 0; i < J.k; ++i)
                s[i] = J.src[i] + cb;
            for (size_t e = 0; e < J.n; ++e)
                d[e] = J.out[e] + cb;
            std::vector<uint16_t> c(J.k);
            par2_constants(J.k, c.data());
            Prob p{};
            p.phase = 0;
            p.src_off = img.put(s.data(), s.size() * sizeof(void *));
            p.dst_off = img.put(d.data(), d.size() * sizeof(void *));
            p.consts_off = img.put(c.data(), c.size() * 2);
            p.exps_off = img.put(J.exps, J.n * 4);
            p.nin = static_cast<int>(J.k);
            p.nout = static_cast<int>(J.n);
            p.S = S;
            p.mode = 0;
            probs.push_back(p);
            continue;
        }
        // REPAIR
        if (singular[j])
            continue;
        const size_t m = J.n, np = J.k - m;
        std::vector<uint16_t> c(J.k), cp;
        par2_constants(J.k, c.data());
        {
            size_t q = 0;
            for (size_t i = 0; i < J.k; ++i) {
                if (q < m && J.missing[q] == i)
                    ++q;
                else
                    cp.push_back(c[i]);
            }
        }
        std::vector<uint8_t *> rh(m), o(m);
        for (size_t q = 0; q < m; ++q) {
            rh[q] = b->rhs.as<uint8_t>() + rhs_off[j] + q * al16(S);
            o[q] = J.out[q] + cb;
            copy_src.push_back(const_cast<uint8_t *>(J.recovery[q]) + cb);
            copy_dst.push_back(rh[q]);
            copy_len.push_back(S);
        }
        const size_t rh_off = img.put(rh.data(), m * sizeof(void *));
        if (np) {
            std::vector<const uint8_t *> s(np);
            for (size_t i = 0; i < np; ++i)
                s[i] = J.src[i] + cb;
            Prob p{};
            p.phase = 0;
            p.src_off = img.put(s.data(), np * sizeof(void *));
            p.dst_off = rh_off;
            p.consts_off = img.put(cp.data(), np * 2);
            p.exps_off = img.put(J.exps, m * 4);
            p.nin = static_cast<int>(np);
            p.nout = static_cast<int>(m);
            p.S = S;
            p.mode = 1;
            probs.push_back(p);
        }
        Prob p{};
        p.phase = 1;
        p.src_off = rh_off;
        p.dst_off = img.put(o.data(), m * sizeof(void *));
        p.coeff = reinterpret_cast<const uint16_t *>(b->inv.as<uint8_t>() + inv_off[j]);
        p.nin = static_cast<int>(m);
        p.nout = static_cast<int>(m);
        p.S = S;
        p.mode = 0;
        probs.push_back(p);
    }
    // ---- scratch and work tables per phase ----
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    for (Prob &p : probs)
        p.form = form_for(ctx, p.nout, p.S);
    size_t plane_need = 0, rec_need = 0;
    for (int x = 0; x < 2; ++x) {
        size_t pl = 0, rc = 0;
        for (const Prob &p : probs)
            if (p.phase == x) {
                pl += static_cast<size_t>(p.nin) * ((p.S + 2047) / 2048) * 2048;
                rc += static_cast<size_t>(p.nin) * p.nout * batch_record_words(p.form) * 4;
            }
        plane_need = std::max(plane_need, pl);
        rec_need = std::max(rec_need, rc);
    }
    if (int rc = take(ctx, b->planes, plane_need + 256))
        return fail(rc);
    if (int rc = take(ctx, b->recs, rec_need + 256))
        return fail(rc);
    b->copy_src_off = img.put(copy_src.data(), copy_src.size() * sizeof(void *));
    b->copy_dst_off = img.put(copy_dst.data(), copy_dst.size() * sizeof(void *));
    b->copy_len_off = img.put(copy_len.data(), copy_len.size() * 8);
    b->ncopy = static_cast<int>(copy_src.size());
    b->counter_off = img.put(nullptr, 2 * sizeof(int));
    // The device addresses of the image are only known after the upload
    // buffer exists: size it first (tables below reference image offsets).
    struct Pending {
        std::vector<PlanesProb> pl;
        std::vector<RecProb> rc;
        std::vector<BatchProb> bp;
        std::vector<BatchItem> items;
        std::vector<uint8_t *> zptr;
        std::vector<unsigned long long> zlen;
    } ph[2];
    // the params buffer must exist before pointers into it are formed: the
    // image grows below, so reserve generously and fix the base afterwards
    std::vector<std::pair<size_t, int>> fixups;  // (image offset of a pointer field, kind)
    for (int x = 0; x < 2; ++x) {
        Pending &P = ph[x];
        size_t pl_off = 0, rc_off = 0;
        unsigned long long pl_first = 0, rc_first = 0;
        double total_cost = 0;
        for (const Prob &p : probs)
            if (p.phase == x) {
                const int blk = batch_block(p.form);
                const size_t tb = batch_tile_bytes(p.form);
                total_cost += static_cast<double>(p.nin) * ((p.S + tb - 1) / tb) *
                              ((p.nout + blk - 1) / blk) *
                              batch_item_cost(p.form, std::min(p.nout, blk));
            }
        const double target = std::max(1.0, total_cost / (4.0 * sms));
        for (size_t pi = 0; pi < probs.size(); ++pi) {
            const Prob &p = probs[pi];
            if (p.phase != x)
                continue;
            const int T = static_cast<int>((p.S + 2047) / 2048);
            PlanesProb pp{};
            pp.S = p.S;
            pp.nin = p.nin;
            pp.T = T;
            pp.first = pl_first;
            // pointer fields hold image offsets for now; rebased after upload
            pp.src = reinterpret_cast<const uint8_t *const *>(p.src_off);
            pp.planes = reinterpret_cast<uint32_t *>(b->planes.as<uint8_t>() + pl_off);
            P.pl.push_back(pp);
            RecProb rp{};
            rp.nin = p.nin;
            rp.nout = p.nout;
            rp.first = rc_first;
            rp.coeff = p.coeff;
            rp.consts = p.coeff ? nullptr : reinterpret_cast<const uint16_t *>(p.consts_off);
            rp.exps = p.coeff ? nullptr : reinterpret_cast<const uint32_t *>(p.exps_off);
            rp.recs = reinterpret_cast<uint32_t *>(b->recs.as<uint8_t>() + rc_off);
            rp.small = p.form == kFormSmall;
            P.rc.push_back(rp);
            BatchProb bp{};
            bp.planes = pp.planes;
            bp.recs = rp.recs;
            bp.dst = reinterpret_cast<uint8_t *const *>(p.dst_off);
            bp.S = p.S;
            bp.nin = p.nin;
            bp.nout = p.nout;
            bp.T = T;
            const int blk = batch_block(p.form);
            bp.nblk = (p.nout + blk - 1) / blk;
            bp.mode = p.mode;
            bp.form = p.form;
            const double unit = static_cast<double>(p.nin) *
                                batch_item_cost(p.form, std::min(p.nout, blk));
            bp.nsplit = split_for(unit, target, p.nin, p.S);
            const int bpi = static_cast<int>(P.bp.size());
            P.bp.push_back(bp);
            const int tiles = static_cast<int>((p.S + batch_tile_bytes(p.form) - 1) /
                                               batch_tile_bytes(p.form));
            for (int t = 0; t < tiles; ++t)
                for (int ob = 0; ob < bp.nblk; ++ob)
                    for (int sp = 0; sp < bp.nsplit; ++sp)
                        P.items.push_back(BatchItem{bpi, t, ob, sp});
            if (bp.nsplit > 1 && bp.mode == 0) {
                // outputs are folded with atomic XOR: start them at zero
                for (int e = 0; e < p.nout; ++e) {
                    uint8_t *ptr;
                    memcpy(&ptr, img.bytes.data() + p.dst_off + e * sizeof(void *), sizeof ptr);
                    P.zptr.push_back(ptr);
                    P.zlen.push_back(p.S);
                }
            }
            pl_off += static_cast<size_t>(p.nin) * T * 2048;
            rc_off += static_cast<size_t>(p.nin) * p.nout * batch_record_words(p.form) * 4;
            pl_first += static_cast<unsigned long long>(p.nin) * T * 32;
            rc_first += static_cast<unsigned long long>(p.nin) * p.nout;
        }
        // longest items first
        std::vector<double> cost(P.items.size());
        for (size_t i = 0; i < P.items.size(); ++i) {
            const BatchItem &it = P.items[i];
            const BatchProb &bp = P.bp[it.prob];
            const int blk = batch_block(bp.form);
            const int nb = std::min(blk, bp.nout - it.ob * blk);
            cost[i] = static_cast<double>(bp.nin) / bp.nsplit * batch_item_cost(bp.form, nb);
        }
        std::vector<size_t> order(P.items.size());
        for (size_t i = 0; i < order.size(); ++i)
            order[i] = i;
        std::stable_sort(order.begin(), order.end(),
                         [&](size_t a, size_t c) { return cost[a] > cost[c]; });
        std::vector<BatchItem> sorted(order.size());
        for (size_t i = 0; i < order.size(); ++i)
            sorted[i] = P.items[order[i]];
        P.items.swap(sorted);
        Phase &D = x == 0 ? b->A : b->B;
        D.nplanes = static_cast<int>(P.pl.size());
        D.nrec = static_cast<int>(P.rc.size());
        D.nitems = static_cast<int>(P.items.size());
        D.nzero = static_cast<int>(P.zptr.size());
        D.grid = std::min(D.nitems, sms);
        D.planes_total = pl_first;
        D.rec_total = rc_first;
    }
    // tables go at the end of the image; pointer fields that hold image
    // offsets are rebased to device addresses once the buffer exists
    for (int x = 0; x < 2; ++x) {
        Phase &D = x == 0 ? b->A : b->B;
        D.planes_off = img.put(nullptr, ph[x].pl.size() * sizeof(PlanesProb));
        D.rec_off = img.put(nullptr, ph[x].rc.size() * sizeof(RecProb));
        D.prob_off = img.put(nullptr, ph[x].bp.size() * sizeof(BatchProb));
        D.item_off = img.put(ph[x].items.data(), ph[x].items.size() * sizeof(BatchItem));
        D.zero_ptr_off = img.put(ph[x].zptr.data(), ph[x].zptr.size() * sizeof(void *));
        D.zero_len_off = img.put(ph[x].zlen.data(), ph[x].zlen.size() * 8);
    }
    for (HashGroup &g : hg) {
        g.n = static_cast<int>(g.slices.size());
        std::vector<const uint8_t *> ptrs(g.n);
        for (int i = 0; i < g.n; ++i)
            ptrs[i] = jobs[g.slices[i].first].src[g.slices[i].second];
        g.ptr_off = img.put(ptrs.data(), ptrs.size() * sizeof(void *));
    }
    if (int rc = take(ctx, b->params, img.bytes.size() + 256))
        return fail(rc);
    uint8_t *base = b->params.as<uint8_t>();
    auto rebase = [&](const void *off) { return base + reinterpret_cast<uintptr_t>(off); };
    for (int x = 0; x < 2; ++x) {
        Phase &D = x == 0 ? b->A : b->B;
        for (PlanesProb &q : ph[x].pl)
            q.src = reinterpret_cast<const uint8_t *const *>(rebase(q.src));
        for (RecProb &q : ph[x].rc) {
            if (!q.coeff) {
                q.consts = reinterpret_cast<const uint16_t *>(rebase(q.consts));
                q.exps = reinterpret_cast<const uint32_t *>(rebase(q.exps));
            }
        }
        for (BatchProb &q : ph[x].bp)
            q.dst = reinterpret_cast<uint8_t *const *>(rebase(q.dst));
        memcpy(img.bytes.data() + D.planes_off, ph[x].pl.data(), ph[x].pl.size() * sizeof(PlanesProb));
        memcpy(img.bytes.data() + D.rec_off, ph[x].rc.data(), ph[x].rc.size() * sizeof(RecProb));
        memcpy(img.bytes.data() + D.prob_off, ph[x].bp.data(), ph[x].bp.size() * sizeof(BatchProb));
    }
    // verify outputs
    size_t hbytes = 0;
    for (HashGroup &g : hg) {
        g.out_off = hbytes;
        hbytes += al256(al16(static_cast<size_t>(g.n) * 16) + static_cast<size_t>(g.n) * 4);
    }
    if (int rc = take(ctx, b->hashbuf, hbytes + 256))
        return fail(rc);
    if (hbytes)
        if (int rc = take(ctx, b->hash_host, hbytes + 256))
            return fail(rc);
    b->hash = hg;
    b->hash_bytes = hbytes;
    if (int rc = take(ctx, b->hparams, img.bytes.size() + 256))
        return fail(rc);
    memcpy(b->hparams.p, img.bytes.data(), img.bytes.size());
    if (cudaMemcpyAsync(b->params.p, b->hparams.p, img.bytes.size(), cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess ||
        cudaEventRecord(b->done, ctx->stream) != cudaSuccess) {
        set_error("p2g_batch_create: table upload failed");
        return fail(P2G_ECUDA);
    }
    b->recorded = true;
    if (flags & P2G_BATCH_GRAPH) {
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
            set_error("p2g_batch_create: %s", cudaGetErrorString(cudaGetLastError()));
            return fail(P2G_ECUDA);
        }
        // capture on the context's own stream (the caller's may be the legacy
        // default stream, which cannot be captured); replays go to ctx->stream
        const bool timing = ctx->timing;
        cudaStream_t caller = ctx->stream;
        ctx->timing = false;  // no event records inside the graph
        ctx->stream = ctx->own_stream;
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
        int rc = e == cudaSuccess ? enqueue(b) : P2G_ECUDA;
        cudaError_t e2 = cudaStreamEndCapture(ctx->stream, &b->graph);
        ctx->stream = caller;
        ctx->timing = timing;
        if (rc != P2G_OK || e2 != cudaSuccess ||
            cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) {
            (void)cudaGetLastError();
            set_error("p2g_batch_create: graph capture failed");
            return fail(rc != P2G_OK ? rc : P2G_ECUDA);
        }
    }
    *out = b;
    return P2G_OK;
}

int p2g_batch_launch(p2g_batch *b)
{
    clear_error();
    if (!b) {
        set_error("p2g_batch_launch: null batch");
        return P2G_EINVAL;
    }
    p2g_ctx *ctx = b->ctx;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    ctx->launches = 0;
    for (bool &m : ctx->ev_marked)
        m = false;
    ctx->mark(0);
    b->cancelled = false;
    for (size_t j = 0; j < b->njobs; ++j)  // a cancelled run's statuses (singular jobs keep theirs)
        if (b->jobs[j].status == P2G_ECANCELED)
            b->jobs[j].status = P2G_OK;
    if (b->exec) {
        P2G_CUDA(cudaGraphLaunch(b->exec, ctx->stream));
        ctx->launches = 1;
    } else {
        P2G_TRY(enqueue(b));
    }
    if (b->hash_bytes)
        P2G_CUDA(cudaMemcpyAsync(b->hash_host.p, b->hashbuf.p, b->hash_bytes,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    ctx->mark(4);
    P2G_CUDA(cudaEventRecord(b->done, ctx->stream));
    b->launched = true;
    return P2G_OK;
}

int p2g_batch_poll(p2g_batch *b, int *done)
{
    clear_error();
    if (!b || !done) {
        set_error("p2g_batch_poll: null argument");
        return P2G_EINVAL;
    }
    cudaError_t e = cudaEventQuery(b->done);
    if (e == cudaErrorNotReady) {
        (void)cudaGetLastError();
        *done = 0;
        return P2G_OK;
    }
    P2G_CUDA(e);
    *done = 1;
    return P2G_OK;
}

int p2g_batch_wait(p2g_batch *b)
{
    clear_error();
    if (!b || !b->launched) {
        set_error("p2g_batch_wait: batch not launched");
        return P2G_EINVAL;
    }
    p2g_ctx *ctx = b->ctx;
    P2G_CUDA(cudaSetDevice(ctx->device));
    P2G_CUDA(cudaEventSynchronize(b->done));
    P2G_CUDA(cudaGetLastError());
    b->launched = false;
    if (b->cancelled) {
        for (size_t j = 0; j < b->njobs; ++j)
            b->jobs[j].status = P2G_ECANCELED;
        set_error("p2g_batch_wait: batch cancelled");
        return P2G_ECANCELED;
    }
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        ctx->last = p2g_timing{};
        ctx->last.launches = ctx->launches;
        if (ctx->timing) {
            auto el = [&](int a, int c) {
                float ms = 0.f;
                if (ctx->ev_marked[a] && ctx->ev_marked[c])
                    cudaEventElapsedTime(&ms, ctx->ev[a], ctx->ev[c]);
                return ms;
            };
            ctx->last.ms_kernel = el(2, 3);
            ctx->last.ms_total = el(0, 4);
        }
    }
    for (const HashGroup &g : b->hash) {
        const uint8_t *md5 = b->hash_host.as<uint8_t>() + g.out_off;
        const uint32_t *crc = reinterpret_cast<const uint32_t *>(md5 + al16(static_cast<size_t>(g.n) * 16));
        for (int i = 0; i < g.n; ++i) {
            p2g_job &J = b->jobs[g.slices[i].first];
            const int s = g.slices[i].second;
            memcpy(J.md5_out + 16 * s, md5 + 16 * i, 16);
            J.crc_out[s] = crc[i];
        }
    }
    return P2G_OK;
}

int p2g_batch_run(p2g_batch *b)
{
    P2G_TRY(p2g_batch_launch(b));
    return p2g_batch_wait(b);
}

int p2g_batch_cancel(p2g_batch *b)
{
    clear_error();
    if (!b || !b->abort_dev) {
        set_error("p2g_batch_cancel: null batch");
        return P2G_EINVAL;
    }
    p2g_ctx *ctx = b->ctx;
    // a copy engine writes the word while the persistent kernel occupies the
    // SMs (a memset kernel could not start before it ends)
    static const int one = 1;
    {
        std::lock_guard<std::mutex> lock(ctx->mu);
        P2G_CUDA(cudaSetDevice(ctx->device));
        if (!ctx->cancel_stream)
            P2G_CUDA(cudaStreamCreateWithFlags(&ctx->cancel_stream, cudaStreamNonBlocking));
        P2G_CUDA(cudaMemcpyAsync(b->abort_dev, &one, sizeof one, cudaMemcpyHostToDevice,
                                 ctx->cancel_stream));
    }
    b->cancelled = true;
    return P2G_OK;
}

int p2g_batch_destroy(p2g_batch *b)
{
    if (!b)
        return P2G_OK;
    if (!b->ctx) {
        batch_free(b);
        return P2G_OK;
    }
    cudaSetDevice(b->ctx->device);
    // wait outside the lock: other batches of the context may be created meanwhile
    if (b->done && b->recorded)
        cudaEventSynchronize(b->done);
    std::lock_guard<std::mutex> lock(b->ctx->mu);
    batch_free(b);
    return P2G_OK;
}

int p2g_batch_set_forms(p2g_ctx *ctx, const int *forms)
{
    clear_error();
    if (!ctx) {
        set_error("p2g_batch_set_forms: null context");
        return P2G_EINVAL;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    for (int c = 0; c < 8; ++c) {
        const int f = forms ? forms[c] : -1;
        if (f != -1 && !batch_form_valid(f, c < 2 ? 24 : 25)) {
            set_error("p2g_batch_set_forms: form %d is not valid for class %d", f, c);
            return P2G_EINVAL;
        }
    }
    for (int c = 0; c < 8; ++c)
        ctx->batch_forms[c] = forms ? forms[c] : -1;
    return P2G_OK;
}

int p2g_batch_autotune(p2g_ctx *ctx, int reps, int *forms_out, float *ms_out)
{
    clear_error();
    if (!ctx) {
        set_error("p2g_batch_autotune: null context");
        return P2G_EINVAL;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    reps = std::max(1, reps);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0)
            cudaEventDestroy(e0);
        (void)cudaGetLastError();
        set_error("p2g_batch_autotune: cudaEventCreate failed");
        return P2G_ECUDA;
    }
    // representative outputs per class pair, ten inputs per output (a set
    // of 10 % redundancy)
    static const int kOut[4] = {8, 64, 160, 420};
    int rc = P2G_OK;
    for (int c = 0; c < 8 && rc == P2G_OK; ++c) {
        const int nout = kOut[c / 2];
        const size_t S = (c & 1) ? (256u << 10) : (8u << 10);
        int form = -1;
        float ms = 0.f;
        // as many problems in one launch as give about 2e9 symbol
        // multiply-accumulates (small sets run many to a batch), at most 64
        const double macs = 10.0 * nout * nout * (S / 2.0);
        const int copies = static_cast<int>(std::min(64.0, std::max(1.0, std::ceil(2e9 / macs))));
        rc = tune_class(ctx, c, 10 * nout, nout, S, copies, reps, e0, e1, &form, &ms);
        if (rc == P2G_OK) {
            ctx->batch_forms[c] = form;
            if (forms_out)
                forms_out[c] = form;
            if (ms_out)
                ms_out[c] = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

}  // extern "C"
