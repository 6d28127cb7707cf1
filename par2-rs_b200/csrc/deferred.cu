// deferred.cu -- the strategy interface's shuffle2x hooks as deferred,
// device-resident multiply-accumulate.
//
// par2-rs brackets its accumulation loops with the selected strategy's
// shuffle2x hooks (galois/simd/mod.rs:68-127; dispatch galois/mod.rs:248-349):
//   * prepare_shuffle2x on every accumulator before the loop and on every
//     source block as it is buffered (par2_rs.rs:727-731, :792-800 for
//     creation; :503-506, :540-553 for reconstruction);
//   * muladd_shuffle2x / muladd_region_shuffle2x inside it (par2_rs.rs:859-864
//     through gf_muladd_column_shuffle2x; :588-599 through
//     gf_muladd_block_regions_shuffle2x);
//   * finish_shuffle2x before any accumulator is read (par2_rs.rs:884-888,
//     :610-613).
// Between prepare and finish a buffer's contents are the strategy's own
// representation.  This strategy's representation is a device copy (a
// "mirror") of the buffer: prepare uploads the buffer (through a pinned
// staging ring, on the copy stream) and leaves the host memory untouched;
// each multiply-accumulate between prepared buffers is recorded, not run; the
// recorded work runs as multi-output kernel launches -- at a prepare once
// enough has accumulated (the callers prepare between their batches, when no
// worker is adding work) and at every finish -- and finish copies the
// accumulator's mirror back into the caller's buffer.  Recorded products of
// the same (destination, source, region) add up in GF(2^16) (c1 s + c2 s =
// (c1 ^ c2) s), so a launch carries one coefficient per pair.
//
// Lifetimes: a mirror lives while it is the current mirror of its host
// address and while recorded work refers to it.  A new prepare of the same
// address (a reused batch buffer) or a finish retires it; once no prepared
// destination is left, the remaining source mirrors are retired too (their
// host buffers still hold the data, so a later use uploads them again).
// Device memory comes from a stream-ordered pool owned by the context.
//
// Calls on unprepared buffers stay correct: an unprepared source is uploaded
// for the recorded work that uses it; an unprepared destination makes the
// call synchronous (pending work is run first and a prepared source is read
// back from its mirror).
//
// Cost per call: the callers make one multiply-accumulate call per
// (destination, source) pair from many threads (par2_rs.rs:832-866), so a
// recorded product takes one uncontended lock: the mirror map and the
// pending products are split over shards, a thread records into its own
// shard, and prepare / finish / flush take every shard.  Prepare copies the
// caller's buffer into the pinned staging ring with helper threads, and
// device blocks of retired mirrors are kept for reuse once the work that
// used them has completed.
#include <string.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "muladd.cuh"

namespace p2g {

namespace {

constexpr size_t kStageChunk = 8u << 20;  // pinned staging chunk
constexpr int kStageChunks = 4;
// pending work that triggers a launch at the next prepare: symbol-MACs
// (about 3 ms of kernel time) or bytes of source mirrors waiting to be used
constexpr double kFlushMacs = 17179869184.0;  // 2^34
constexpr size_t kFlushSourceBytes = size_t(1) << 30;

struct Mirror {
    uint8_t *dev = nullptr;
    size_t bytes = 0;
    uintptr_t host = 0;  // the address it mirrors while current
    int refs = 0;        // recorded products that read or write it (atomic)
    bool current = false;
    bool dst = false;    // written by recorded products (atomic)
};

struct Product {
    uint32_t dst, src;
    size_t off, len;  // u16 units
    uint16_t c;
};

constexpr int kShards = 16;

// One lock of the sharded map lock, with the products recorded under it.
struct alignas(64) Shard {
    std::mutex mu;
    std::vector<Product> pending;
    double macs = 0;
    size_t src_bytes = 0;
};

// A device block of a retired mirror, reusable once `ev` has completed.
struct FreeBlock {
    uint8_t *dev;
    size_t bytes;
    cudaEvent_t ev;
};
constexpr size_t kMaxFreeBytes = size_t(2) << 30;

// Helper threads copying a staged chunk in parts: prepare must have read the
// caller's buffer when it returns, and one thread copies ~13 GB/s.
class CopyPool {
  public:
    explicit CopyPool(int helpers)
    {
        for (int i = 0; i < helpers; ++i)
            th_.emplace_back([this] { loop(); });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> l(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (std::thread &t : th_)
            t.join();
    }
    // n bytes from src to dst in up to helpers + 1 parts of at least 128 KiB
    void copy(uint8_t *dst, const uint8_t *src, size_t n)
    {
        const size_t parts = std::min<size_t>(th_.size() + 1, std::max<size_t>(1, n >> 17));
        if (parts <= 1) {
            memcpy(dst, src, n);
            return;
        }
        const size_t step = ((n + parts - 1) / parts + 63) & ~size_t(63);
        {
            std::lock_guard<std::mutex> l(mu_);
            dst_ = dst;
            src_ = src;
            n_ = n;
            step_ = step;
            parts_ = (n + step - 1) / step;
            next_ = 1;
            left_ = parts_ - 1;
        }
        cv_.notify_all();
        memcpy(dst, src, std::min(step, n));  // part 0 on the calling thread
        std::unique_lock<std::mutex> l(mu_);
        done_.wait(l, [&] { return left_ == 0; });
    }

  private:
    void loop()
    {
        std::unique_lock<std::mutex> l(mu_);
        while (true) {
            cv_.wait(l, [&] { return stop_ || next_ < parts_; });
            if (stop_)
                return;
            const size_t p = next_++;
            const size_t a = p * step_, b = std::min(n_, a + step_);
            uint8_t *dst = dst_;
            const uint8_t *src = src_;
            l.unlock();
            memcpy(dst + a, src + a, b - a);
            l.lock();
            if (--left_ == 0)
                done_.notify_one();
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    uint8_t *dst_ = nullptr;
    const uint8_t *src_ = nullptr;
    size_t n_ = 0, step_ = 0, parts_ = 0, next_ = 0, left_ = 0;
    bool stop_ = false;
};

}  // namespace

struct Deferred {
    // The map lock: shard[j].mu for the recording threads of shard j, all
    // of them (in index order) for everything that changes the map.
    Shard shard[kShards];
    std::vector<Mirror> mirrors;
    std::vector<uint32_t> free_ids;
    std::unordered_map<uintptr_t, uint32_t> by_host;
    int live_dsts = 0;  // current mirrors that recorded products write (atomic)

    std::mutex stage_mu;  // staging ring
    uint8_t *stage[kStageChunks] = {};
    cudaEvent_t stage_ev[kStageChunks] = {};
    int stage_next = 0;
    cudaEvent_t upload_ev = nullptr;  // after the latest upload on the copy stream
    bool uploads = false;
    CopyPool *copier = nullptr;

    // device blocks of retired mirrors (oldest first) and idle events
    std::vector<FreeBlock> free_blocks;
    size_t free_bytes = 0;
    std::vector<cudaEvent_t> spare_events;

    // kernel parameters of a launch: pinned, two slots, each reused only after
    // the copy that read it has run
    DevBuf hpar[2], dpar[2];
    cudaEvent_t par_ev[2] = {};
    int par_next = 0;

    cudaMemPool_t pool = nullptr;
};

namespace {

// The shard of the calling thread (threads take shards round robin).
Shard &my_shard(Deferred *d)
{
    static std::atomic<unsigned> next{0};
    thread_local unsigned mine = next.fetch_add(1) % kShards;
    return d->shard[mine];
}

// Every shard's lock: the map may change.
struct MapWriteLock {
    Deferred *d;
    bool held = true;
    explicit MapWriteLock(Deferred *dd) : d(dd)
    {
        for (Shard &s : d->shard)
            s.mu.lock();
    }
    void unlock()
    {
        if (held)
            for (int j = kShards - 1; j >= 0; --j)
                d->shard[j].mu.unlock();
        held = false;
    }
    ~MapWriteLock() { unlock(); }
};

// ctx->mu held.
int setup(p2g_ctx *ctx, Deferred *&out)
{
    if ((out = ctx->deferred.load()) != nullptr)
        return P2G_OK;
    Deferred *d = new Deferred();
    int rc = P2G_OK;
    for (int i = 0; i < kStageChunks && rc == P2G_OK; ++i) {
        if (cudaMallocHost(&d->stage[i], kStageChunk) != cudaSuccess ||
            cudaEventCreateWithFlags(&d->stage_ev[i], cudaEventDisableTiming) != cudaSuccess)
            rc = P2G_ENOMEM;
    }
    for (int i = 0; i < 2 && rc == P2G_OK; ++i) {
        d->hpar[i].pinned = true;
        if (cudaEventCreateWithFlags(&d->par_ev[i], cudaEventDisableTiming) != cudaSuccess)
            rc = P2G_ECUDA;
    }
    if (rc == P2G_OK &&
        cudaEventCreateWithFlags(&d->upload_ev, cudaEventDisableTiming) != cudaSuccess)
        rc = P2G_ECUDA;
    if (rc == P2G_OK) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = ctx->device;
        if (cudaMemPoolCreate(&d->pool, &props) != cudaSuccess) {
            rc = P2G_ECUDA;
        } else {
            // keep freed mirror memory for the next mirrors instead of
            // returning it at every synchronisation
            uint64_t keep = ~uint64_t(0);
            cudaMemPoolSetAttribute(d->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    if (rc == P2G_OK) {
        // helpers for the staging copies: up to 7 more threads (the callers
        // prepare between their batches, when their workers are idle)
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        d->copier = new CopyPool(static_cast<int>(std::min(7u, hw / 2)));
    }
    if (rc != P2G_OK) {
        (void)cudaGetLastError();
        set_error("shuffle2x: setting up the device mirrors failed");
        ctx->deferred = d;  // released by deferred_release
        deferred_release(ctx);
        return rc;
    }
    ctx->deferred = d;
    out = d;
    return P2G_OK;
}

// Retires the device block of mirror `id`: it is kept for a later mirror
// once every launch that used it and every upload enqueued so far have run
// (an event on the compute stream after both); beyond kMaxFreeBytes of kept
// blocks the oldest go back to the pool.  Map write-locked.
int drop_mirror(p2g_ctx *ctx, Deferred *d, uint32_t id)
{
    Mirror &m = d->mirrors[id];
    if (m.dev) {
        if (d->uploads)
            P2G_CUDA(cudaStreamWaitEvent(ctx->stream, d->upload_ev, 0));
        cudaEvent_t ev = nullptr;
        if (!d->spare_events.empty()) {
            ev = d->spare_events.back();
            d->spare_events.pop_back();
        } else {
            P2G_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        }
        P2G_CUDA(cudaEventRecord(ev, ctx->stream));
        d->free_blocks.push_back(FreeBlock{m.dev, m.bytes, ev});
        d->free_bytes += m.bytes;
        while (d->free_bytes > kMaxFreeBytes) {
            const FreeBlock b = d->free_blocks.front();
            d->free_blocks.erase(d->free_blocks.begin());
            d->free_bytes -= b.bytes;
            d->spare_events.push_back(b.ev);
            P2G_CUDA(cudaFreeAsync(b.dev, ctx->stream));
        }
    }
    m = Mirror{};
    d->free_ids.push_back(id);
    return P2G_OK;
}

// A device block of at least `bytes` for a new mirror: a kept block of the
// same size whose last use has completed, else one from the pool (on the
// copy stream, which uploads into it).  Map write-locked.
int take_block(p2g_ctx *ctx, Deferred *d, size_t bytes, uint8_t *&dev)
{
    const size_t want = std::max<size_t>(bytes, 16);
    for (size_t j = 0; j < d->free_blocks.size(); ++j) {
        FreeBlock &b = d->free_blocks[j];
        if (b.bytes != want)
            continue;
        const cudaError_t q = cudaEventQuery(b.ev);
        if (q == cudaErrorNotReady) {
            // blocks are kept oldest first and their events complete in
            // stream order: no younger block is free yet either
            (void)cudaGetLastError();
            break;
        }
        P2G_CUDA(q);
        dev = b.dev;
        d->free_bytes -= b.bytes;
        d->spare_events.push_back(b.ev);
        d->free_blocks.erase(d->free_blocks.begin() + static_cast<long>(j));
        return P2G_OK;
    }
    P2G_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void **>(&dev), want, d->pool,
                                     ctx->copy_stream));
    return P2G_OK;
}

// A new mirror of `bytes` holding a copy of host[0, bytes).  Map
// write-locked.
int new_mirror(p2g_ctx *ctx, Deferred *d, const void *host, size_t bytes, uint32_t &id)
{
    uint8_t *dev = nullptr;
    P2G_TRY(take_block(ctx, d, bytes, dev));
    {
        std::lock_guard<std::mutex> lock(d->stage_mu);
        const uint8_t *h = static_cast<const uint8_t *>(host);
        for (size_t off = 0; off < bytes; off += kStageChunk) {
            const size_t n = std::min(kStageChunk, bytes - off);
            const int c = d->stage_next;
            d->stage_next = (c + 1) % kStageChunks;
            P2G_CUDA(cudaEventSynchronize(d->stage_ev[c]));
            d->copier->copy(d->stage[c], h + off, n);
            P2G_CUDA(cudaMemcpyAsync(dev + off, d->stage[c], n, cudaMemcpyHostToDevice,
                                     ctx->copy_stream));
            P2G_CUDA(cudaEventRecord(d->stage_ev[c], ctx->copy_stream));
        }
        P2G_CUDA(cudaEventRecord(d->upload_ev, ctx->copy_stream));
        d->uploads = true;
    }
    if (d->free_ids.empty()) {
        id = static_cast<uint32_t>(d->mirrors.size());
        d->mirrors.emplace_back();
    } else {
        id = d->free_ids.back();
        d->free_ids.pop_back();
    }
    Mirror &m = d->mirrors[id];
    m.dev = dev;
    m.bytes = bytes;
    return P2G_OK;
}

// Makes mirror `id` no longer current; frees it when no recorded product
// uses it.  Map write-locked (no product is being recorded).
int retire(p2g_ctx *ctx, Deferred *d, uint32_t id)
{
    Mirror &m = d->mirrors[id];
    if (m.current) {
        d->by_host.erase(m.host);
        if (m.dst)
            --d->live_dsts;
        m.current = false;
    }
    return m.refs == 0 ? drop_mirror(ctx, d, id) : P2G_OK;
}

// Pointer arrays and coefficient matrix of one launch in a parameter slot.
int launch_group(p2g_ctx *ctx, Deferred *d, const std::vector<uint8_t *> &srcs,
                 const std::vector<uint8_t *> &dsts, const std::vector<uint16_t> &coeff,
                 size_t bytes)
{
    const size_t nin = srcs.size(), nout = dsts.size();
    const size_t so = 0, dso = ((nin * sizeof(void *)) + 15) & ~size_t(15);
    const size_t co = dso + (((nout * sizeof(void *)) + 15) & ~size_t(15));
    const size_t total = co + nin * nout * 2;
    const int slot = d->par_next;
    d->par_next ^= 1;
    P2G_CUDA(cudaEventSynchronize(d->par_ev[slot]));
    P2G_TRY(d->hpar[slot].ensure(total));
    P2G_TRY(d->dpar[slot].ensure(total));
    uint8_t *h = d->hpar[slot].as<uint8_t>();
    memcpy(h + so, srcs.data(), nin * sizeof(void *));
    memcpy(h + dso, dsts.data(), nout * sizeof(void *));
    memcpy(h + co, coeff.data(), nin * nout * 2);
    uint8_t *dp = d->dpar[slot].as<uint8_t>();
    P2G_CUDA(cudaMemcpyAsync(dp, h, total, cudaMemcpyHostToDevice, ctx->stream));
    P2G_CUDA(cudaEventRecord(d->par_ev[slot], ctx->stream));
    P2G_TRY(ctx->recs.ensure(record_bytes(nin, static_cast<int>(nout))));
    P2G_TRY(records_from_matrix(ctx, reinterpret_cast<const uint16_t *>(dp + co),
                                static_cast<int>(nin), static_cast<int>(nout),
                                ctx->recs.as<uint32_t>()));
    return muladd_run(ctx, reinterpret_cast<const uint8_t *const *>(dp + so),
                      static_cast<int>(nin), reinterpret_cast<uint8_t *const *>(dp + dso),
                      static_cast<int>(nout), bytes, ctx->recs.as<uint32_t>(), 1);
}

// Runs every recorded product.  ctx->mu held, map write-locked.
int flush(p2g_ctx *ctx, Deferred *d)
{
    std::vector<Product> work;
    for (Shard &sh : d->shard) {
        if (work.empty())
            work.swap(sh.pending);
        else
            work.insert(work.end(), sh.pending.begin(), sh.pending.end());
        sh.pending.clear();
        sh.macs = 0;
        sh.src_bytes = 0;
    }
    if (work.empty())
        return P2G_OK;
    if (d->uploads)
        P2G_CUDA(cudaStreamWaitEvent(ctx->stream, d->upload_ev, 0));
    std::sort(work.begin(), work.end(), [](const Product &a, const Product &b) {
        if (a.off != b.off)
            return a.off < b.off;
        if (a.len != b.len)
            return a.len < b.len;
        if (a.src != b.src)
            return a.src < b.src;
        return a.dst < b.dst;
    });
    int rc = P2G_OK;
    std::vector<int> dix(d->mirrors.size(), -1);
    size_t g0 = 0;
    while (g0 < work.size() && rc == P2G_OK) {
        size_t g1 = g0;
        while (g1 < work.size() && work[g1].off == work[g0].off && work[g1].len == work[g0].len)
            ++g1;
        const size_t off = work[g0].off, len = work[g0].len;
        // sources of the group in chunks of at most 65535, all destinations
        // (dix: a destination mirror's row in the coefficient matrix)
        std::vector<uint8_t *> dsts;
        for (size_t q = g0; q < g1; ++q) {
            if (dix[work[q].dst] < 0) {
                dix[work[q].dst] = static_cast<int>(dsts.size());
                dsts.push_back(d->mirrors[work[q].dst].dev + off * 2);
            }
        }
        size_t q = g0;
        while (q < g1 && rc == P2G_OK) {
            std::vector<uint8_t *> srcs;
            std::vector<size_t> col;  // per product of this chunk: its source column
            size_t q1 = q;
            uint32_t last = UINT32_MAX;
            while (q1 < g1) {
                if (work[q1].src != last) {
                    if (srcs.size() == 65535)
                        break;
                    last = work[q1].src;
                    srcs.push_back(d->mirrors[last].dev + off * 2);
                }
                col.push_back(srcs.size() - 1);
                ++q1;
            }
            std::vector<uint16_t> coeff(dsts.size() * srcs.size(), 0);
            for (size_t t = q; t < q1; ++t)
                coeff[dix[work[t].dst] * srcs.size() + col[t - q]] ^= work[t].c;
            bool aligned = (off * 2) % 16 == 0;
            if (aligned) {
                rc = launch_group(ctx, d, srcs, dsts, coeff, len * 2);
            } else {
                // a region that does not start on a 16-byte boundary: staged
                // through aligned scratch, computed, copied back
                const size_t slot = (len * 2 + 15) & ~size_t(15);
                rc = ctx->in_copy.ensure(slot * srcs.size());
                if (rc == P2G_OK)
                    rc = ctx->out_copy.ensure(slot * dsts.size());
                std::vector<uint8_t *> s2(srcs.size()), d2(dsts.size());
                for (size_t i = 0; i < srcs.size() && rc == P2G_OK; ++i) {
                    s2[i] = ctx->in_copy.as<uint8_t>() + i * slot;
                    if (cudaMemcpyAsync(s2[i], srcs[i], len * 2, cudaMemcpyDeviceToDevice,
                                        ctx->stream) != cudaSuccess)
                        rc = P2G_ECUDA;
                }
                for (size_t o = 0; o < dsts.size() && rc == P2G_OK; ++o) {
                    d2[o] = ctx->out_copy.as<uint8_t>() + o * slot;
                    if (cudaMemcpyAsync(d2[o], dsts[o], len * 2, cudaMemcpyDeviceToDevice,
                                        ctx->stream) != cudaSuccess)
                        rc = P2G_ECUDA;
                }
                if (rc == P2G_OK)
                    rc = launch_group(ctx, d, s2, d2, coeff, len * 2);
                for (size_t o = 0; o < dsts.size() && rc == P2G_OK; ++o)
                    if (cudaMemcpyAsync(dsts[o], d2[o], len * 2, cudaMemcpyDeviceToDevice,
                                        ctx->stream) != cudaSuccess)
                        rc = P2G_ECUDA;
                if (rc == P2G_ECUDA)
                    set_error("shuffle2x: staging a misaligned region failed");
            }
            q = q1;
        }
        for (size_t q = g0; q < g1; ++q)
            dix[work[q].dst] = -1;
        g0 = g1;
    }
    // the products have been enqueued: release their references
    std::vector<uint32_t> dead;
    for (const Product &p : work) {
        if (--d->mirrors[p.dst].refs == 0 && !d->mirrors[p.dst].current)
            dead.push_back(p.dst);
        if (--d->mirrors[p.src].refs == 0 && !d->mirrors[p.src].current)
            dead.push_back(p.src);
    }
    std::sort(dead.begin(), dead.end());
    dead.erase(std::unique(dead.begin(), dead.end()), dead.end());
    for (uint32_t id : dead)
        if (rc == P2G_OK)
            rc = drop_mirror(ctx, d, id);
    return rc;
}

// The current mirror of host address p covering at least `bytes`, or -1.
// A shard lock or the map write lock held.
long find(Deferred *d, const void *p, size_t bytes)
{
    auto it = d->by_host.find(reinterpret_cast<uintptr_t>(p));
    if (it == d->by_host.end() || d->mirrors[it->second].bytes < bytes)
        return -1;
    return static_cast<long>(it->second);
}

// One recorded product into shard `sh`.  sh.mu held (or the map write
// lock); mirror reference counts and flags change atomically, as other
// shards record products on the same mirrors.
void add_product(Deferred *d, Shard &sh, uint32_t dst, uint32_t src, size_t off, size_t len,
                 uint16_t c)
{
    Mirror &md = d->mirrors[dst];
    Mirror &ms = d->mirrors[src];
    if (__atomic_fetch_add(&ms.refs, 1, __ATOMIC_RELAXED) == 0 &&
        !__atomic_load_n(&ms.dst, __ATOMIC_RELAXED))
        sh.src_bytes += ms.bytes;
    __atomic_fetch_add(&md.refs, 1, __ATOMIC_RELAXED);
    if (!__atomic_load_n(&md.dst, __ATOMIC_RELAXED) &&
        !__atomic_exchange_n(&md.dst, true, __ATOMIC_RELAXED) && md.current)
        __atomic_fetch_add(&d->live_dsts, 1, __ATOMIC_RELAXED);
    sh.pending.push_back(Product{dst, src, off, len, c});
    sh.macs += static_cast<double>(len);
}

// Records dsts[o][off, off+len) ^= coeff(o, i) * srcs[i][off, off+len).
// `coeff(o, i)` gives the coefficient.
template <class Coeff>
int record(p2g_ctx *ctx, uint16_t *const *dsts, size_t ndst, const uint16_t *const *srcs,
           size_t nsrc, Coeff coeff, size_t off, size_t len)
{
    Deferred *d = ctx->deferred.load();
    if (!d) {
        std::lock_guard<std::mutex> lock(ctx->mu);
        P2G_CUDA(cudaSetDevice(ctx->device));
        P2G_TRY(setup(ctx, d));
    }
    const size_t need = (off + len) * 2;
    // mirror ids of the call's buffers (on the stack for small calls)
    constexpr size_t kSmall = 16;
    long dm_s[kSmall], sm_s[kSmall];
    std::vector<long> dm_v, sm_v;
    long *dm = dm_s, *sm = sm_s;
    if (ndst > kSmall) {
        dm_v.resize(ndst);
        dm = dm_v.data();
    }
    if (nsrc > kSmall) {
        sm_v.resize(nsrc);
        sm = sm_v.data();
    }
    {
        // every buffer prepared: record under this thread's shard lock
        Shard &sh = my_shard(d);
        std::lock_guard<std::mutex> lock(sh.mu);
        bool all = true;
        for (size_t o = 0; o < ndst && all; ++o)
            all = (dm[o] = find(d, dsts[o], need)) >= 0;
        for (size_t i = 0; i < nsrc && all; ++i)
            all = (sm[i] = find(d, srcs[i], need)) >= 0;
        if (all) {
            for (size_t o = 0; o < ndst; ++o)
                for (size_t i = 0; i < nsrc; ++i) {
                    const uint16_t c = coeff(o, i);
                    if (c)
                        add_product(d, sh, static_cast<uint32_t>(dm[o]),
                                    static_cast<uint32_t>(sm[i]), off, len, c);
                }
            return P2G_OK;
        }
    }
    // Some buffer is not prepared.
    std::unique_lock<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    MapWriteLock wlock(d);
    std::vector<size_t> prep, unprep;  // destinations with / without a mirror
    for (size_t o = 0; o < ndst; ++o) {
        dm[o] = find(d, dsts[o], need);
        (dm[o] >= 0 ? prep : unprep).push_back(o);
    }
    if (!prep.empty()) {
        // recorded for the prepared destinations; unprepared sources are
        // uploaded for them (not current: freed once these products have run)
        for (size_t i = 0; i < nsrc; ++i) {
            if ((sm[i] = find(d, srcs[i], need)) >= 0)
                continue;
            uint32_t id;
            P2G_TRY(new_mirror(ctx, d, srcs[i], need, id));
            sm[i] = id;
        }
        for (size_t o : prep)
            for (size_t i = 0; i < nsrc; ++i) {
                const uint16_t c = coeff(o, i);
                if (c)
                    add_product(d, d->shard[0], static_cast<uint32_t>(dm[o]),
                                static_cast<uint32_t>(sm[i]), off, len, c);
            }
        // temporaries that ended up unused (all-zero coefficients) go now
        for (size_t i = 0; i < nsrc; ++i)
            if (!d->mirrors[sm[i]].current && d->mirrors[sm[i]].refs == 0 &&
                d->mirrors[sm[i]].dev)
                P2G_TRY(drop_mirror(ctx, d, static_cast<uint32_t>(sm[i])));
    }
    if (unprep.empty())
        return P2G_OK;
    // Unprepared destinations: their products run now, on host buffers,
    // after the recorded work; prepared sources are read back from their
    // mirrors (recorded products may have written them).
    P2G_TRY(flush(ctx, d));
    std::vector<std::vector<uint16_t>> back(nsrc);
    std::vector<const uint16_t *> sp(srcs, srcs + nsrc);
    for (size_t i = 0; i < nsrc; ++i) {
        const long id = find(d, srcs[i], need);
        if (id < 0)
            continue;
        back[i].resize(off + len);
        P2G_CUDA(cudaMemcpyAsync(back[i].data(), d->mirrors[id].dev, need,
                                 cudaMemcpyDeviceToHost, ctx->stream));
        sp[i] = back[i].data();
    }
    P2G_CUDA(cudaStreamSynchronize(ctx->stream));
    wlock.unlock();
    lock.unlock();
    std::vector<uint16_t> rows(unprep.size() * nsrc);
    std::vector<const uint16_t *> rp(unprep.size());
    std::vector<uint16_t *> dp(unprep.size());
    for (size_t q = 0; q < unprep.size(); ++q) {
        for (size_t i = 0; i < nsrc; ++i)
            rows[q * nsrc + i] = coeff(unprep[q], i);
        rp[q] = rows.data() + q * nsrc;
        dp[q] = dsts[unprep[q]];
    }
    return p2g_muladd_region(ctx, dp.data(), dp.size(), sp.data(), nsrc, rp.data(), off, len, 0);
}

}  // namespace

void deferred_release(p2g_ctx *ctx)
{
    Deferred *d = ctx->deferred.load();
    if (!d)
        return;
    cudaStreamSynchronize(ctx->stream);
    cudaStreamSynchronize(ctx->copy_stream);
    delete d->copier;
    for (Mirror &m : d->mirrors)
        if (m.dev)
            cudaFree(m.dev);
    for (FreeBlock &b : d->free_blocks) {
        cudaFree(b.dev);
        cudaEventDestroy(b.ev);
    }
    for (cudaEvent_t ev : d->spare_events)
        cudaEventDestroy(ev);
    if (d->pool)
        cudaMemPoolDestroy(d->pool);
    for (int i = 0; i < kStageChunks; ++i) {
        if (d->stage[i])
            cudaFreeHost(d->stage[i]);
        if (d->stage_ev[i])
            cudaEventDestroy(d->stage_ev[i]);
    }
    for (int i = 0; i < 2; ++i) {
        d->hpar[i].release();
        d->dpar[i].release();
        if (d->par_ev[i])
            cudaEventDestroy(d->par_ev[i]);
    }
    if (d->upload_ev)
        cudaEventDestroy(d->upload_ev);
    (void)cudaGetLastError();
    delete d;
    ctx->deferred = nullptr;
}

}  // namespace p2g

using namespace p2g;

extern "C" {

int p2g_supports_shuffle2x(void) { return 1; }

int p2g_prepare_shuffle2x(p2g_ctx *ctx, uint16_t *data, size_t n)
{
    clear_error();
    if (!ctx || (n && !data)) {
        set_error("p2g_prepare_shuffle2x: null argument");
        return P2G_EINVAL;
    }
    if (n == 0)
        return P2G_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    Deferred *d = nullptr;
    P2G_TRY(setup(ctx, d));
    MapWriteLock wlock(d);
    // between the caller's batches: run what has accumulated
    double macs = 0;
    size_t src_bytes = 0;
    for (const Shard &sh : d->shard) {
        macs += sh.macs;
        src_bytes += sh.src_bytes;
    }
    const bool due = macs >= kFlushMacs || src_bytes >= kFlushSourceBytes;
    if (due)
        P2G_TRY(flush(ctx, d));
    const long old = find(d, data, 0);
    if (old >= 0)
        P2G_TRY(retire(ctx, d, static_cast<uint32_t>(old)));
    uint32_t id;
    P2G_TRY(new_mirror(ctx, d, data, n * 2, id));
    Mirror &m = d->mirrors[id];
    m.host = reinterpret_cast<uintptr_t>(data);
    m.current = true;
    d->by_host[m.host] = id;
    return P2G_OK;
}

int p2g_muladd_shuffle2x(p2g_ctx *ctx, uint16_t *dst, const uint16_t *src, size_t n, uint16_t c)
{
    clear_error();
    if (!ctx || (n && (!dst || !src))) {
        set_error("p2g_muladd_shuffle2x: null argument");
        return P2G_EINVAL;
    }
    if (n == 0 || c == 0)
        return P2G_OK;
    return record(ctx, &dst, 1, &src, 1, [c](size_t, size_t) { return c; }, 0, n);
}

int p2g_muladd_region_shuffle2x(p2g_ctx *ctx, uint16_t *const *dsts, size_t ndst,
                                const uint16_t *const *srcs, size_t nsrc,
                                const uint16_t *const *coeff_rows, size_t off_u16,
                                size_t len_u16)
{
    clear_error();
    if (!ctx || (ndst && (!dsts || !coeff_rows)) || (nsrc && !srcs)) {
        set_error("p2g_muladd_region_shuffle2x: null argument");
        return P2G_EINVAL;
    }
    if (ndst > 65535 || nsrc > 65535) {
        set_error("p2g_muladd_region_shuffle2x: too many slices");
        return P2G_ERANGE;
    }
    if (ndst == 0 || nsrc == 0 || len_u16 == 0)
        return P2G_OK;
    return record(ctx, dsts, ndst, srcs, nsrc,
                  [coeff_rows](size_t o, size_t i) { return coeff_rows[o][i]; }, off_u16,
                  len_u16);
}

int p2g_finish_shuffle2x(p2g_ctx *ctx, uint16_t *data, size_t n)
{
    clear_error();
    if (!ctx || (n && !data)) {
        set_error("p2g_finish_shuffle2x: null argument");
        return P2G_EINVAL;
    }
    if (n == 0)
        return P2G_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    P2G_CUDA(cudaSetDevice(ctx->device));
    Deferred *d = nullptr;
    P2G_TRY(setup(ctx, d));
    MapWriteLock wlock(d);
    const long id = find(d, data, 0);
    if (id < 0)
        return P2G_OK;  // never prepared: the buffer already holds its data
    P2G_TRY(flush(ctx, d));
    Mirror &m = d->mirrors[id];
    P2G_CUDA(cudaMemcpyAsync(data, m.dev, std::min(n * 2, m.bytes), cudaMemcpyDeviceToHost,
                             ctx->stream));
    P2G_CUDA(cudaStreamSynchronize(ctx->stream));
    P2G_TRY(retire(ctx, d, static_cast<uint32_t>(id)));
    if (d->live_dsts == 0) {
        // no accumulator left: the remaining sources' mirrors go too
        std::vector<uint32_t> rest;
        for (const auto &kv : d->by_host)
            rest.push_back(kv.second);
        for (uint32_t r : rest)
            P2G_TRY(retire(ctx, d, r));
    }
    return P2G_OK;
}

}  // extern "C"
