// par2_pipeline.hpp -- create and repair of PAR2 sets from files, with the
// slices resident on the GPU:
//
//   Par2Creator::create      creator.rs:261-521  (new, with_* options 148-253)
//   Par2Repairer::repair     lib.rs:132-351, repair.rs:537-604 (verify, lowest
//                            exponents, rebuild, write back)
//
// Files stream through pinned host buffers straight into one device buffer of
// zero-padded slices: a pool of reader threads each reads a file in 8 MiB
// chunks, folds every chunk into the file's MD5 on the host (whole-file MD5 is
// a serial chain) and uploads it on its own stream while reading the next
// chunk.  The IFSC checksums, the slice verification and the recovery slices
// are computed from that buffer by libpar2gpu (P2G_DEVICE_PTRS); only the
// recovery slices come back to the host.
#pragma once
#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <functional>
#include <memory>
#include <mutex>
#include <set>
#include <thread>

#include "par2_format.hpp"

namespace par2 {

struct PipelineStats {
    double ms_scan = 0;    // sizes, first-16-KiB MD5s, File IDs, order
    double ms_ingest = 0;  // read + whole-file MD5 + upload of every file
    double ms_gpu = 0;     // IFSC / verification + encode / repair on the device
    double ms_write = 0;   // packets and files (create) / repaired files (repair)
    double ms_total = 0;
    uint64_t block_size = 0, data_blocks = 0, recovery_blocks = 0, bytes_read = 0;
    uint64_t damaged_blocks = 0, files_written = 0;
};

namespace detail {

inline double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

inline void cuda_check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw Par2Error(std::string(what) + ": " + cudaGetErrorString(e));
    }
}

// Device buffer of k zero-padded slices of bs bytes.  The zero fill has
// finished when the constructor returns: the buffer is then written from
// non-blocking streams (the readers', the codec context's), which do not
// order themselves after work on the default stream.
class DeviceSlices {
  public:
    DeviceSlices(uint64_t k, uint64_t bs) : k_(k), bs_(bs)
    {
        if (k && bs) {
            cuda_check(cudaMalloc(&p_, k * bs), "cudaMalloc (slices)");
            cudaStream_t st = nullptr;
            cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
            const cudaError_t e1 = cudaMemsetAsync(p_, 0, k * bs, st);
            const cudaError_t e2 = cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
            cuda_check(e1 != cudaSuccess ? e1 : e2, "cudaMemsetAsync (slices)");
        }
    }
    ~DeviceSlices()
    {
        if (p_)
            cudaFree(p_);
    }
    DeviceSlices(const DeviceSlices &) = delete;
    DeviceSlices &operator=(const DeviceSlices &) = delete;
    uint8_t *slice(uint64_t i) const { return static_cast<uint8_t *>(p_) + i * bs_; }
    std::vector<const uint8_t *> ptrs(uint64_t first, uint64_t n) const
    {
        std::vector<const uint8_t *> v(n);
        for (uint64_t i = 0; i < n; ++i)
            v[i] = slice(first + i);
        return v;
    }

  private:
    void *p_ = nullptr;
    uint64_t k_, bs_;
};

// Process-wide pool of pinned 8 MiB host chunks for the pipelines' copies.
// Pinning is far slower than the copies it serves (tens of ms for the ~100
// MiB a create uses), so chunks are pinned once, on first demand, and reused
// by every later ingest and read-back; they live until the process exits.
constexpr size_t kPinnedChunk = 8u << 20;

class PinnedPool {
  public:
    static PinnedPool &get()
    {
        static PinnedPool *p = new PinnedPool;  // never destroyed: see above
        return *p;
    }
    uint8_t *take()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (!free_.empty()) {
                uint8_t *b = free_.back();
                free_.pop_back();
                return b;
            }
        }
        void *b = nullptr;
        cuda_check(cudaMallocHost(&b, kPinnedChunk), "cudaMallocHost");
        return static_cast<uint8_t *>(b);
    }
    void give(uint8_t *b)
    {
        if (!b)
            return;
        std::lock_guard<std::mutex> lk(mu_);
        free_.push_back(b);
    }

  private:
    std::mutex mu_;
    std::vector<uint8_t *> free_;
};

struct IngestJob {
    std::filesystem::path path;
    uint8_t *dst = nullptr;   // device: the file's first slice
    uint64_t length = 0;      // bytes to read (file length)
    bool hash = true;         // fold the bytes into md5
    FileHash md5{};           // out: MD5 of what was read
    bool ok = false;          // out: the file existed and had `length` bytes
};

// true when the caller asked to stop (polled between phases and read chunks)
using CancelFn = std::function<bool()>;

// Reads every job's file into device memory with whole-file MD5s, `threads`
// files at a time.  Per file, a read-ahead thread fills a ring of three
// pinned 8 MiB chunks while the worker folds the previous chunk into the MD5
// and uploads it on its own stream, so reading, hashing and uploading
// overlap (a chunk is refilled only after its upload has finished).
inline uint64_t ingest(std::vector<IngestJob> &jobs, unsigned threads,
                       const CancelFn *cancel = nullptr)
{
    auto cancelled = [&] { return cancel && *cancel && (*cancel)(); };
    constexpr size_t kChunk = kPinnedChunk;
    constexpr int kSlots = 3;
    std::atomic<size_t> next{0};
    std::atomic<uint64_t> total{0};
    std::vector<std::string> errors(threads);
    auto worker = [&](unsigned t) {
        cudaStream_t st = nullptr;
        uint8_t *buf[kSlots] = {};
        cudaEvent_t ev[kSlots] = {};
        try {
            cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
            for (int b = 0; b < kSlots; ++b) {
                buf[b] = PinnedPool::get().take();
                cuda_check(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming), "cudaEventCreate");
            }
            for (size_t j; !cancelled() && (j = next.fetch_add(1)) < jobs.size();) {
                IngestJob &job = jobs[j];
                FILE *f = fopen(job.path.string().c_str(), "rb");
                if (!f)
                    continue;  // missing file: its slices stay zero
                std::mutex mu;
                std::condition_variable cv;
                size_t len[kSlots] = {};
                bool full[kSlots] = {}, stop = false;
                std::thread reader([&] {
                    uint64_t roff = 0;
                    for (size_t i = 0;; ++i) {
                        const int s = static_cast<int>(i % kSlots);
                        {
                            std::unique_lock<std::mutex> lk(mu);
                            cv.wait(lk, [&] { return !full[s] || stop; });
                            if (stop)
                                return;
                        }
                        cudaEventSynchronize(ev[s]);  // the slot's last upload is done
                        size_t n = 0;
                        if (roff < job.length && !cancelled())
                            n = fread(buf[s], 1, std::min<uint64_t>(kChunk, job.length - roff), f);
                        roff += n;
                        {
                            std::lock_guard<std::mutex> lk(mu);
                            len[s] = n;
                            full[s] = true;
                        }
                        cv.notify_all();
                        if (n == 0)
                            return;
                    }
                });
                Md5 h;
                uint64_t off = 0;
                try {
                    for (size_t i = 0;; ++i) {
                        const int s = static_cast<int>(i % kSlots);
                        size_t n;
                        {
                            std::unique_lock<std::mutex> lk(mu);
                            cv.wait(lk, [&] { return full[s]; });
                            n = len[s];
                        }
                        if (n == 0)
                            break;
                        if (job.hash)
                            h.update(buf[s], n);
                        cuda_check(cudaMemcpyAsync(job.dst + off, buf[s], n, cudaMemcpyHostToDevice, st),
                                   "cudaMemcpyAsync");
                        cuda_check(cudaEventRecord(ev[s], st), "cudaEventRecord");
                        off += n;
                        {
                            std::lock_guard<std::mutex> lk(mu);
                            full[s] = false;
                        }
                        cv.notify_all();
                    }
                } catch (...) {
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        stop = true;
                    }
                    cv.notify_all();
                    reader.join();
                    fclose(f);
                    throw;
                }
                reader.join();
                uint8_t extra;
                job.ok = off == job.length && fread(&extra, 1, 1, f) == 0;
                fclose(f);
                job.md5 = h.finalize();
                total += off;
            }
            cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        } catch (const std::exception &e) {
            errors[t] = e.what();
        }
        if (st)
            cudaStreamSynchronize(st);
        for (int b = 0; b < kSlots; ++b) {
            if (ev[b])
                cudaEventDestroy(ev[b]);
            PinnedPool::get().give(buf[b]);
        }
        if (st)
            cudaStreamDestroy(st);
    };
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < threads; ++t)
        pool.emplace_back(worker, t);
    for (auto &th : pool)
        th.join();
    for (const std::string &e : errors)
        if (!e.empty())
            throw Par2Error(e);
    return total;
}

inline unsigned reader_threads(size_t files)
{
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    return static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(files, hw)));
}

inline std::vector<uint8_t> read_head(const std::filesystem::path &p, size_t n)
{
    std::vector<uint8_t> d(n);
    FILE *f = fopen(p.string().c_str(), "rb");
    if (!f)
        throw Par2Error("Failed to open " + p.string());
    const size_t got = n ? fread(d.data(), 1, n, f) : 0;
    fclose(f);
    d.resize(got);
    return d;
}

// Runs sink(chunk bytes, offset, length) over n bytes of device memory cut
// into 8 MiB chunks: up to 8 host threads each copy chunks down through their
// own pooled pinned buffer and stream and hand them to the sink, so the
// copies and the sinks (file writes, page faults of the destination) run side
// by side.  Returns false when a copy or a sink failed.
template <class Sink> bool drain_device(const uint8_t *d, size_t n, Sink sink)
{
    constexpr size_t kChunk = kPinnedChunk;
    const size_t chunks = (n + kChunk - 1) / kChunk;
    const size_t nt = std::min<size_t>(
        chunks, std::min(8u, std::max(1u, std::thread::hardware_concurrency())));
    std::atomic<size_t> next{0};
    std::atomic<bool> failed{false};
    auto worker = [&] {
        uint8_t *buf = nullptr;
        cudaStream_t st = nullptr;
        try {
            buf = PinnedPool::get().take();
        } catch (const Par2Error &) {
            failed = true;
        }
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
            failed = true;
        for (size_t c; !failed && (c = next.fetch_add(1)) < chunks;) {
            const size_t off = c * kChunk, len = std::min(kChunk, n - off);
            if (cudaMemcpyAsync(buf, d + off, len, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess ||
                !sink(static_cast<const uint8_t *>(buf), off, len))
                failed = true;
        }
        if (st)
            cudaStreamDestroy(st);
        PinnedPool::get().give(buf);
    };
    std::vector<std::thread> pool;
    for (size_t t = 0; t < nt; ++t)
        pool.emplace_back(worker);
    for (auto &th : pool)
        th.join();
    if (failed)
        (void)cudaGetLastError();
    return !failed;
}

// Uploads n pieces: fill(i, pinned host chunk) writes piece i (at most
// kPinnedChunk bytes) into the chunk and returns {device destination, bytes}.
// Up to 8 host threads each run fills and copies through their own pooled
// chunk and stream, so the reads of several pieces and their uploads overlap.
template <class Fill> void fill_device(size_t n, Fill fill)
{
    const size_t nt = std::min<size_t>(n, std::min(8u, std::max(1u, std::thread::hardware_concurrency())));
    std::atomic<size_t> next{0};
    std::vector<std::string> errors(nt);
    auto worker = [&](size_t t) {
        uint8_t *buf = nullptr;
        cudaStream_t st = nullptr;
        try {
            buf = PinnedPool::get().take();
            cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
            for (size_t i; errors[t].empty() && (i = next.fetch_add(1)) < n;) {
                const std::pair<uint8_t *, size_t> dst = fill(i, buf);
                cuda_check(cudaMemcpyAsync(dst.first, buf, dst.second, cudaMemcpyHostToDevice, st),
                           "cudaMemcpyAsync");
                cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
            }
        } catch (const std::exception &e) {
            errors[t] = e.what();
            next = n;  // the other threads stop too
        }
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        PinnedPool::get().give(buf);
    };
    std::vector<std::thread> pool;
    for (size_t t = 0; t < nt; ++t)
        pool.emplace_back(worker, t);
    for (auto &th : pool)
        th.join();
    for (const std::string &e : errors)
        if (!e.empty())
            throw Par2Error(e);
}

// MD5 of n bytes of device memory, copied down in order through one pooled
// pinned chunk (whole-file hashes are one serial chain).
inline FileHash md5_of_device(const uint8_t *d, size_t n)
{
    uint8_t *buf = PinnedPool::get().take();
    Md5 h;
    cudaError_t e = cudaSuccess;
    for (size_t off = 0; off < n && e == cudaSuccess; off += kPinnedChunk) {
        const size_t len = std::min(kPinnedChunk, n - off);
        e = cudaMemcpy(buf, d + off, len, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            h.update(buf, len);
    }
    PinnedPool::get().give(buf);
    cuda_check(e, "cudaMemcpy (file hash)");
    return h.finalize();
}

// Copies n bytes of device memory into host memory h (any, pageable).
inline void copy_to_host(uint8_t *h, const uint8_t *d, size_t n)
{
    if (!drain_device(d, n, [&](const uint8_t *b, size_t off, size_t len) {
            memcpy(h + off, b, len);
            return true;
        }))
        throw Par2Error("cudaMemcpy (device to host) failed");
}

// Writes n bytes of device memory to a new file at p (pwrite at each chunk's
// offset).
inline void write_file_from_device(const std::filesystem::path &p, const uint8_t *d, size_t n)
{
    const int fd = ::open(p.string().c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0)
        throw Par2Error("Failed to write " + p.string());
    const bool ok = drain_device(d, n, [&](const uint8_t *b, size_t off, size_t len) {
        for (size_t w = 0; w < len;) {
            const ssize_t x = ::pwrite(fd, b + w, len - w, static_cast<off_t>(off + w));
            if (x <= 0)
                return false;
            w += static_cast<size_t>(x);
        }
        return true;
    });
    if (::close(fd) != 0 || !ok)
        throw Par2Error("Failed to write " + p.string());
}

// fn(i) for i in [0, n) on the host's threads
template <class F> void parallel_for(size_t n, F fn)
{
    const size_t nt = std::min<size_t>(n, std::max(1u, std::thread::hardware_concurrency()));
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (size_t t = 0; t < nt; ++t)
        pool.emplace_back([&] {
            for (size_t i; (i = next.fetch_add(1)) < n;)
                fn(i);
        });
    for (auto &th : pool)
        th.join();
}

}  // namespace detail

// Par2Operation of lib.rs:76-81 and the progress callback (operation,
// current, total)
enum class Par2Operation { Scanning = 0, Loading = 1, Verifying = 2, Repairing = 3 };
using ProgressCallback = std::function<void(Par2Operation, uint64_t, uint64_t)>;

class Par2Creator {
  public:
    explicit Par2Creator(std::vector<std::filesystem::path> input_files)
        : inputs_(std::move(input_files))
    {
        if (inputs_.empty())
            throw Par2Error("No input files");
        for (const auto &f : inputs_)
            if (!std::filesystem::exists(f))
                throw Par2Error("Input file does not exist: " + f.string());
        // first input with its extensions replaced: a.b.c -> a.par2 (creator.rs:170)
        output_ = inputs_[0];
        output_.replace_extension("");
        output_.replace_extension("par2");
    }
    Par2Creator &with_block_size(uint64_t size)
    {
        if (size == 0)
            throw Par2Error("Block size cannot be zero");
        if (size < 2048)
            throw Par2Error("Block size must be at least 2048 bytes (got " + std::to_string(size) + ")");
        if (size % 4)
            throw Par2Error("Block size must be multiple of 4");
        block_size_ = size;
        return *this;
    }
    Par2Creator &with_redundancy(float percent)
    {
        if (percent != percent || percent - percent != 0)
            throw Par2Error("Redundancy percentage must be a finite number");
        if (percent < 0)
            throw Par2Error("Redundancy percentage cannot be negative");
        percent_ = percent;
        return *this;
    }
    Par2Creator &with_output_path(std::filesystem::path p)
    {
        output_ = std::move(p);
        return *this;
    }
    Par2Creator &with_volume_scheme(VolumeScheme s)
    {
        scheme_ = s;
        return *this;
    }
    Par2Creator &with_creator_text(std::string t)
    {
        creator_ = std::move(t);
        return *this;
    }
    // creator.rs:245-253: encoding progress as (Repairing, slices done, data
    // slices), called on the creating thread -- 0 before the files stream in,
    // all of them once the recovery slices exist
    Par2Creator &with_progress(ProgressCallback cb)
    {
        progress_ = std::move(cb);
        return *this;
    }
    const PipelineStats &stats() const { return stats_; }

    // Writes the index file and the volumes; returns their paths.
    std::vector<std::filesystem::path> create()
    {
        using detail::ms_since;
        const auto t0 = std::chrono::steady_clock::now();
        stats_ = PipelineStats();
        // File IDs need only the first 16 KiB; the order fixes the slice layout
        std::vector<FileInfo> infos(inputs_.size());
        for (size_t i = 0; i < inputs_.size(); ++i) {
            FileInfo &fi = infos[i];
            fi.name = inputs_[i].filename().string();
            fi.length = std::filesystem::file_size(inputs_[i]);
            const std::vector<uint8_t> head = detail::read_head(inputs_[i], 16384);
            fi.hash_16k = Md5::of(head.data(), head.size());
            fi.file_id = compute_file_id(fi.hash_16k, fi.length, fi.name);
        }
        std::vector<size_t> order(infos.size());
        for (size_t i = 0; i < order.size(); ++i)
            order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
            return file_id_less(infos[a].file_id, infos[b].file_id);
        });
        uint64_t total = 0;
        for (const FileInfo &f : infos)
            total += f.length;
        const uint64_t bs = block_size_ ? block_size_ : calculate_block_size(total);
        std::vector<uint64_t> first(infos.size()), nblk(infos.size());
        uint64_t k = 0;
        for (size_t i : order) {
            first[i] = k;
            nblk[i] = (infos[i].length + bs - 1) / bs;
            k += nblk[i];
        }
        if (k > 65535)
            throw Par2Error("Total data blocks (" + std::to_string(k) + ") exceed GF(2^16) limit (65535)");
        const uint64_t r = recovery_block_count(k, bs, percent_);
        if (r > 65535)
            throw Par2Error("Recovery blocks (" + std::to_string(r) + ") exceed GF(2^16) limit (65535)");
        if (k + r > 65535)
            throw Par2Error("Total blocks (data + recovery) exceed GF(2^16) limit (65535)");
        stats_.block_size = bs;
        stats_.data_blocks = k;
        stats_.recovery_blocks = r;
        stats_.ms_scan = ms_since(t0);
        if (progress_)
            progress_(Par2Operation::Repairing, 0, k);
        // every file once: whole-file MD5 on the host, slices to the device
        const auto t1 = std::chrono::steady_clock::now();
        codec_ctx();  // the device context exists before the readers start
        detail::DeviceSlices dev(k, bs);
        std::vector<detail::IngestJob> jobs(infos.size());
        for (size_t i = 0; i < infos.size(); ++i) {
            jobs[i].path = inputs_[i];
            jobs[i].dst = k ? dev.slice(first[i]) : nullptr;
            jobs[i].length = infos[i].length;
        }
        stats_.bytes_read = detail::ingest(jobs, detail::reader_threads(jobs.size()));
        for (size_t i = 0; i < infos.size(); ++i) {
            if (!jobs[i].ok)
                throw Par2Error("Failed to read " + inputs_[i].string());
            infos[i].hash = jobs[i].md5;
        }
        stats_.ms_ingest = ms_since(t1);
        // IFSC checksums and recovery slices from the device-resident slices
        const auto t2 = std::chrono::steady_clock::now();
        std::vector<uint8_t> md5(k * 16);
        // filled by the copy below (not zero-initialised first)
        std::unique_ptr<uint8_t[]> rec(new uint8_t[static_cast<size_t>(r * bs)]);
        std::vector<uint32_t> crc(k);
        if (k) {
            std::vector<const uint8_t *> sp = dev.ptrs(0, k);
            check(p2g_hash_slices(codec_ctx(), sp.data(), k, bs, md5.data(), crc.data(),
                                  P2G_DEVICE_PTRS));
            if (r) {
                detail::DeviceSlices out(r, bs);
                std::vector<uint8_t *> op(r);
                std::vector<uint32_t> exps(r);
                for (uint64_t e = 0; e < r; ++e) {
                    op[e] = out.slice(e);
                    exps[e] = static_cast<uint32_t>(e);
                }
                check(p2g_encode(codec_ctx(), sp.data(), k, bs, exps.data(), r, op.data(),
                                 P2G_DEVICE_PTRS));
                detail::copy_to_host(rec.get(), out.slice(0), r * bs);
            }
        }
        stats_.ms_gpu = ms_since(t2);
        if (progress_)
            progress_(Par2Operation::Repairing, k, k);
        // packets shared by every file, then one file per volume (creator.rs:441-521)
        const auto t3 = std::chrono::steady_clock::now();
        std::vector<FileHash> ids;
        for (size_t i : order)
            ids.push_back(infos[i].file_id);
        const FileHash set_id = compute_recovery_set_id(build_main_packet_body(bs, ids));
        std::vector<uint8_t> common;
        write_packet(common, packet_types::CREATOR, set_id,
                     std::vector<uint8_t>(creator_.begin(), creator_.end()));
        write_packet(common, packet_types::MAIN, set_id, build_main_packet_body(bs, ids));
        for (size_t i : order)
            write_packet(common, packet_types::FILE_DESC, set_id, file_desc_body(infos[i]));
        for (size_t i : order) {
            std::vector<SliceChecksum> cs(nblk[i]);
            for (uint64_t b = 0; b < nblk[i]; ++b) {
                memcpy(cs[b].md5.data(), md5.data() + (first[i] + b) * 16, 16);
                cs[b].crc32 = crc[first[i] + b];
            }
            write_packet(common, packet_types::IFSC, set_id, ifsc_body(infos[i].file_id, cs));
        }
        std::vector<uint32_t> all(r);
        for (uint64_t e = 0; e < r; ++e)
            all[e] = static_cast<uint32_t>(e);
        std::vector<VolumeInfo> vols = split_into_volumes(all, scheme_, output_);
        if (scheme_ == VolumeScheme::Single && !vols.empty()) {
            vols[0].path = output_;
        } else {
            VolumeInfo index;
            index.path = output_;
            vols.insert(vols.begin(), index);
        }
        // RecvSlic packets (header, exponent, slice; bs is a multiple of 4, so
        // no padding): the headers' MD5s in parallel, the bodies written from
        // the recovery buffer in place
        std::vector<std::array<uint8_t, 68>> head(r);
        detail::parallel_for(r, [&](size_t e) {
            uint8_t *hd = head[e].data();
            const uint8_t ex[4] = {static_cast<uint8_t>(e), static_cast<uint8_t>(e >> 8),
                                   static_cast<uint8_t>(e >> 16), static_cast<uint8_t>(e >> 24)};
            Md5 h;
            h.update(set_id.data(), 16);
            h.update(packet_types::RECV_SLICE.data(), 16);
            h.update(ex, 4);
            h.update(rec.get() + e * bs, bs);
            const FileHash md5 = h.finalize();
            const uint64_t len = 64 + 4 + bs;
            memcpy(hd, kPar2Magic, 8);
            for (int i = 0; i < 8; ++i)
                hd[8 + i] = static_cast<uint8_t>(len >> (8 * i));
            memcpy(hd + 16, md5.data(), 16);
            memcpy(hd + 32, set_id.data(), 16);
            memcpy(hd + 48, packet_types::RECV_SLICE.data(), 16);
            memcpy(hd + 64, ex, 4);
        });
        // the volumes are independent files: written side by side
        std::vector<uint8_t> vol_ok(vols.size(), 0);
        detail::parallel_for(vols.size(), [&](size_t i) {
            const VolumeInfo &v = vols[i];
            FILE *f = fopen(v.path.string().c_str(), "wb");
            bool ok = f && fwrite(common.data(), 1, common.size(), f) == common.size();
            for (uint32_t e : v.exponents)
                ok = ok && fwrite(head[e].data(), 1, 68, f) == 68 &&
                     fwrite(rec.get() + static_cast<size_t>(e) * bs, 1, bs, f) == bs;
            if (f)
                ok = fclose(f) == 0 && ok;
            vol_ok[i] = ok;
        });
        std::vector<std::filesystem::path> written;
        for (size_t i = 0; i < vols.size(); ++i) {
            if (!vol_ok[i])
                throw Par2Error("Failed to write " + vols[i].path.string());
            written.push_back(vols[i].path);
        }
        stats_.files_written = written.size();
        stats_.ms_write = ms_since(t3);
        stats_.ms_total = ms_since(t0);
        return written;
    }

  private:
    std::vector<std::filesystem::path> inputs_;
    std::filesystem::path output_;
    uint64_t block_size_ = 0;
    float percent_ = 5.0f;
    VolumeScheme scheme_ = VolumeScheme::Exponential;
    ProgressCallback progress_;
    std::string creator_ = kReferenceCreator;
    PipelineStats stats_;
};

// Par2Operation (lib.rs:76-81) and the progress callback (operation, current, total)

struct Cancelled : Par2Error {
    Cancelled() : Par2Error("PAR2 operation cancelled") {}
};

// Verification and repair of the files of a set in `dir`
// (Par2Repairer::repair_with_callbacks_cancellable, lib.rs:196-351): every
// slice is checked against its IFSC entry on the GPU (a missing or short file
// counts as damaged where it lacks data); without do_repair any damage is an
// error; otherwise the damaged slices are rebuilt from the m lowest recovery
// exponents (repair.rs:537-604) and checked again against their IFSC
// entries, every touched file is written to `<name>.par2tmp` and only then
// are all of them renamed into place (repair.rs:54-110), so that an error or
// a cancellation before the commit leaves every data file as it was.  With
// purge, the set's .par2 files are deleted after a verified or repaired set.
// The cancel flag is checked between phases and between read chunks.
class Par2Repairer {
  public:
    Par2Repairer(std::filesystem::path par2, std::filesystem::path dir)
        : par2_(std::move(par2)), dir_(std::move(dir))
    {
    }
    Par2Repairer &with_repair(bool do_repair)
    {
        do_repair_ = do_repair;
        return *this;
    }
    Par2Repairer &with_purge(bool purge)
    {
        purge_ = purge;
        return *this;
    }
    Par2Repairer &with_progress(ProgressCallback cb)
    {
        progress_ = std::move(cb);
        return *this;
    }
    Par2Repairer &with_cancel(detail::CancelFn is_cancelled)
    {
        cancel_ = std::move(is_cancelled);
        return *this;
    }
    const PipelineStats &stats() const { return stats_; }

    // returns the number of slices rebuilt (0: nothing was damaged)
    uint64_t repair()
    {
        using detail::ms_since;
        const auto t0 = std::chrono::steady_clock::now();
        stats_ = PipelineStats();
        check_cancel();
        report(Par2Operation::Loading, 0, 100);
        Par2File p = Par2File::load(par2_);
        report(Par2Operation::Loading, 100, 100);
        // the files the set names, in slice order (lib.rs:232-241 reports its
        // directory scan here)
        report(Par2Operation::Scanning, 0, 100);
        const uint64_t bs = p.block_size;
        std::vector<uint64_t> first, nblk;
        uint64_t k = 0;
        for (const FileInfo &f : p.files_in_order) {
            first.push_back(k);
            nblk.push_back((f.length + bs - 1) / bs);
            k += nblk.back();
        }
        if (k > 65535)
            throw Par2Error("Total data blocks exceed GF(2^16) limit (65535)");
        stats_.block_size = bs;
        stats_.data_blocks = k;
        stats_.recovery_blocks = p.recovery_blocks.size();
        stats_.ms_scan = ms_since(t0);
        report(Par2Operation::Scanning, 100, 100);
        check_cancel();
        // Files whose IFSC entries cover every slice are verified slice by
        // slice on the device; the others by their whole-file MD5, computed
        // while they are read (the full-file fallback of verify.rs:522-540).
        std::vector<char> has_ifsc(p.files_in_order.size(), 0);
        for (size_t i = 0; i < p.files_in_order.size(); ++i) {
            const auto it = p.slice_checksums.find(p.files_in_order[i].file_id);
            has_ifsc[i] = it != p.slice_checksums.end() && it->second.size() >= nblk[i];
        }
        // the files into device slices
        const auto t1 = std::chrono::steady_clock::now();
        report(Par2Operation::Verifying, 0, 100);
        codec_ctx();
        detail::DeviceSlices dev(k, bs);
        std::vector<detail::IngestJob> jobs(p.files_in_order.size());
        for (size_t i = 0; i < jobs.size(); ++i) {
            jobs[i].path = dir_ / p.files_in_order[i].name;
            jobs[i].dst = k ? dev.slice(first[i]) : nullptr;
            jobs[i].length = p.files_in_order[i].length;
            jobs[i].hash = !has_ifsc[i];
        }
        stats_.bytes_read = detail::ingest(jobs, detail::reader_threads(jobs.size()), &cancel_);
        check_cancel();
        stats_.ms_ingest = ms_since(t1);
        // per-slice verification on the device
        const auto t2 = std::chrono::steady_clock::now();
        std::vector<uint64_t> damaged;
        std::vector<uint8_t> md5(k * 16, 0);
        std::vector<uint32_t> crc(k, 0);
        if (k) {
            std::vector<uint8_t> ok(k, 0);
            for (size_t i = 0; i < p.files_in_order.size(); ++i) {
                if (!has_ifsc[i])
                    continue;
                const auto &cs = p.slice_checksums.find(p.files_in_order[i].file_id)->second;
                for (uint64_t b = 0; b < nblk[i]; ++b) {
                    memcpy(md5.data() + (first[i] + b) * 16, cs[b].md5.data(), 16);
                    crc[first[i] + b] = cs[b].crc32;
                }
            }
            std::vector<const uint8_t *> sp = dev.ptrs(0, k);
            check(p2g_verify_slices(codec_ctx(), sp.data(), k, bs, md5.data(), crc.data(), ok.data(),
                                    P2G_DEVICE_PTRS));
            for (size_t i = 0; i < p.files_in_order.size(); ++i) {
                // without IFSC a file is intact or, as a whole, damaged
                const bool file_ok = !has_ifsc[i] && jobs[i].ok && jobs[i].md5 == p.files_in_order[i].hash;
                for (uint64_t b = 0; b < nblk[i]; ++b)
                    if (has_ifsc[i] ? !ok[first[i] + b] : !file_ok)
                        damaged.push_back(first[i] + b);
            }
        }
        // a file longer than its FileDesc length: its last slice is rebuilt so
        // that the file is rewritten at its length
        for (size_t i = 0; i < jobs.size(); ++i) {
            std::error_code ec;
            const uint64_t sz = std::filesystem::file_size(jobs[i].path, ec);
            const uint64_t last = first[i] + nblk[i] - 1;
            if (!ec && nblk[i] && sz > p.files_in_order[i].length &&
                !std::binary_search(damaged.begin(), damaged.end(), last))
                damaged.insert(std::lower_bound(damaged.begin(), damaged.end(), last), last);
        }
        report(Par2Operation::Verifying, 100, 100);
        stats_.damaged_blocks = damaged.size();
        stats_.ms_gpu = ms_since(t2);
        if (damaged.empty()) {
            finish(p, t0);
            return 0;
        }
        if (!do_repair_)
            throw Par2Error("Files are damaged and repair was not requested");
        check_cancel();
        report(Par2Operation::Repairing, 0, 100);
        const auto t3 = std::chrono::steady_clock::now();
        std::vector<RecoveryRef> recs = p.recovery_blocks;
        std::stable_sort(recs.begin(), recs.end(),
                         [](const RecoveryRef &a, const RecoveryRef &b) { return a.exponent < b.exponent; });
        recs.erase(std::unique(recs.begin(), recs.end(),
                               [](const RecoveryRef &a, const RecoveryRef &b) { return a.exponent == b.exponent; }),
                   recs.end());
        const uint64_t m = damaged.size();
        if (recs.size() < m)
            throw Par2Error("Insufficient recovery blocks: need " + std::to_string(m) + ", have " +
                            std::to_string(recs.size()));
        // the m lowest exponents' slices to the device, then the repair there
        detail::DeviceSlices rdev(m, bs), out(m, bs);
        std::vector<uint32_t> exps(m);
        for (uint64_t q = 0; q < m; ++q)
            exps[q] = recs[q].exponent;
        // pieces of up to one pinned chunk, read and uploaded by several threads
        const uint64_t parts = (bs + detail::kPinnedChunk - 1) / detail::kPinnedChunk;
        detail::fill_device(m * parts, [&](size_t i, uint8_t *host) {
            const uint64_t q = i / parts, off = (i % parts) * detail::kPinnedChunk;
            const size_t len = static_cast<size_t>(std::min<uint64_t>(detail::kPinnedChunk, bs - off));
            p.read_recovery_into(recs[q], off, len, host);
            return std::make_pair(rdev.slice(q) + off, len);
        });
        check_cancel();
        std::set<uint64_t> dset(damaged.begin(), damaged.end());
        std::vector<const uint8_t *> present;
        for (uint64_t g = 0; g < k; ++g)
            if (!dset.count(g))
                present.push_back(dev.slice(g));
        std::vector<const uint8_t *> rp = rdev.ptrs(0, m);
        std::vector<uint8_t *> op(m);
        for (uint64_t q = 0; q < m; ++q)
            op[q] = out.slice(q);
        const int rc = p2g_repair(codec_ctx(), k, bs, damaged.data(), m, present.data(), exps.data(),
                                  rp.data(), op.data(), P2G_DEVICE_PTRS);
        if (rc == P2G_ESINGULAR)
            throw Par2Error("Singular matrix");
        check(rc);
        for (uint64_t q = 0; q < m; ++q)
            detail::cuda_check(cudaMemcpy(dev.slice(damaged[q]), out.slice(q), bs, cudaMemcpyDeviceToDevice),
                               "cudaMemcpy (rebuilt slice)");
        // device-to-device copies return before they finish; the check below
        // runs on the codec context's own stream
        detail::cuda_check(cudaStreamSynchronize(cudaStreamLegacy), "cudaStreamSynchronize");
        // the rebuilt slices against their IFSC entries, and files without
        // them by their whole-file MD5 (the post-repair verification of
        // lib.rs:302-325)
        {
            std::vector<uint64_t> slices;  // rebuilt slices of files with IFSC
            std::set<size_t> whole;        // touched files without
            size_t fi = 0;
            for (uint64_t g : damaged) {
                while (g >= first[fi] + nblk[fi])
                    ++fi;
                if (has_ifsc[fi])
                    slices.push_back(g);
                else
                    whole.insert(fi);
            }
            const size_t n = slices.size();
            std::vector<uint8_t> wmd5(n * 16), ok(n, 0);
            std::vector<uint32_t> wcrc(n);
            std::vector<const uint8_t *> rp2(n);
            for (size_t q = 0; q < n; ++q) {
                memcpy(wmd5.data() + q * 16, md5.data() + slices[q] * 16, 16);
                wcrc[q] = crc[slices[q]];
                rp2[q] = dev.slice(slices[q]);
            }
            if (n)
                check(p2g_verify_slices(codec_ctx(), rp2.data(), n, bs, wmd5.data(), wcrc.data(),
                                        ok.data(), P2G_DEVICE_PTRS));
            bool good = std::all_of(ok.begin(), ok.end(), [](uint8_t v) { return v != 0; });
            for (size_t i : whole)
                good = good && detail::md5_of_device(dev.slice(first[i]), p.files_in_order[i].length) ==
                                   p.files_in_order[i].hash;
            if (!good)
                throw Par2Error("Repair completed but verification failed - files may still be damaged");
        }
        stats_.ms_gpu += ms_since(t3);
        // write every touched file to <name>.par2tmp, then commit them all
        const auto t4 = std::chrono::steady_clock::now();
        std::vector<std::pair<std::filesystem::path, std::filesystem::path>> commits;
        try {
            for (size_t i = 0; i < p.files_in_order.size(); ++i) {
                const FileInfo &f = p.files_in_order[i];
                bool touched = false;
                for (uint64_t b = 0; b < nblk[i] && !touched; ++b)
                    touched = dset.count(first[i] + b) > 0;
                if (!touched)
                    continue;
                check_cancel();
                const std::filesystem::path fin = dir_ / f.name;
                std::filesystem::path tmp = fin;
                tmp += ".par2tmp";
                commits.emplace_back(tmp, fin);
                detail::write_file_from_device(tmp, dev.slice(first[i]), f.length);
            }
            check_cancel();
        } catch (...) {
            for (const auto &c : commits) {
                std::error_code ec;
                std::filesystem::remove(c.first, ec);
            }
            throw;
        }
        for (const auto &c : commits) {
            std::filesystem::rename(c.first, c.second);
            ++stats_.files_written;
        }
        report(Par2Operation::Repairing, 100, 100);
        stats_.ms_write = ms_since(t4);
        finish(p, t0);
        return m;
    }

  private:
    void check_cancel() const
    {
        if (cancel_ && cancel_())
            throw Cancelled();
    }
    void report(Par2Operation op, uint64_t cur, uint64_t total) const
    {
        if (progress_)
            progress_(op, cur, total);
    }
    // cancellation after the commit skips the purge (lib.rs:338-347)
    void finish(const Par2File &p, std::chrono::steady_clock::time_point t0)
    {
        check_cancel();
        if (purge_)
            for (const auto &f : p.set_files) {
                std::error_code ec;
                std::filesystem::remove(f, ec);
            }
        stats_.ms_total = detail::ms_since(t0);
    }

    std::filesystem::path par2_, dir_;
    bool do_repair_ = true, purge_ = false;
    ProgressCallback progress_;
    detail::CancelFn cancel_;
    PipelineStats stats_;
};

}  // namespace par2
