// par2_codec.hpp -- C++ mirror of par2-rs's Reed-Solomon codec API over
// libpar2gpu (par2-rs src/par2_rs.rs):
//
//   Par2ReedSolomon::new / encode            par2_rs.rs:160-313
//   compute_reconstruction_transform         par2_rs.rs:319-422
//   reconstruct_streaming_chunk              par2_rs.rs:442-675
//   create_streaming_encoder                 par2_rs.rs:687-772
//   StreamingEncoder::{process_block, flush_batch, finalize}  par2_rs.rs:775-902
//   galois dispatch (supports / prepare / finish_shuffle2x,
//     gf_muladd_column[_shuffle2x])          galois/mod.rs:118-142, :248-349
//
// Same names, argument meaning and error strings.  The transform holds the
// decode matrix A^-1 formed on the GPU (the reference records the elimination
// steps instead; A^-1 is what those steps apply), so a singular set is
// reported when the transform is computed, as in the reference.
// Reconstruction runs as the two multiply-accumulate passes of p2g_repair.
#pragma once
#include <string.h>

#include <algorithm>
#include <atomic>
#include <exception>
#include <functional>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "galois_strategy.hpp"

namespace par2 {

// Errors carry the reference's message text (String errors of par2_rs.rs).
struct Par2Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

using RecoveryBlocks = std::vector<std::pair<uint32_t, std::vector<uint8_t>>>;

// The decode matrix of one set of missing blocks, in ascending missing order.
struct ReconstructionTransform {
    std::vector<uint64_t> missing;        // missing data block indices, ascending
    std::vector<uint32_t> exponents;      // exponents of the m recovery blocks used
    std::vector<uint16_t> inverse;        // m x m, row-major
};

// The device context shared by the codec objects of this process.
inline p2g_ctx *codec_ctx()
{
    static CudaSm100aStrategy strategy;
    return strategy.ctx();
}

// Scalar GF(2^16) on the host (galois/core.rs:49-91, :175-193): the codec's
// coefficient matrix needs c_i^e for every input i and exponent e.
namespace gf {
struct Tables {
    uint16_t log[65536];
    uint16_t exp[131070];
    Tables()
    {
        uint32_t b = 1;
        for (uint32_t l = 0; l < 65535; ++l) {
            exp[l] = exp[l + 65535] = static_cast<uint16_t>(b);
            log[b] = static_cast<uint16_t>(l);
            b <<= 1;
            if (b & 0x10000u)
                b ^= 0x1100Bu;
        }
        log[0] = 0;
    }
};
inline const Tables &tables()
{
    static const Tables *t = new Tables();
    return *t;
}
inline uint16_t mul(uint16_t a, uint16_t b)
{
    if (!a || !b)
        return 0;
    const Tables &t = tables();
    return t.exp[t.log[a] + t.log[b]];
}
}  // namespace gf

// The galois/mod.rs entry points the codec calls, dispatched to the selected
// strategy.  With no strategy selected they throw (the reference falls back
// to its scalar code; this library has no CPU path).
namespace galois {
inline const GaloisSimdStrategy &selected()
{
    const GaloisSimdStrategy *s = get_registry().get_selected();
    if (!s)
        throw std::runtime_error("no galois strategy is available (no sm_100 device)");
    return *s;
}
// galois/mod.rs:255-260
inline bool supports_shuffle2x()
{
    const GaloisSimdStrategy *s = get_registry().get_selected();
    return s && s->supports_shuffle2x();
}
// galois/mod.rs:274-282, :288-296
inline void prepare_shuffle2x(uint16_t *data, size_t n)
{
    const GaloisSimdStrategy *s = get_registry().get_selected();
    if (s && s->supports_shuffle2x())
        s->prepare_shuffle2x(data, n);
}
inline void finish_shuffle2x(uint16_t *data, size_t n)
{
    const GaloisSimdStrategy *s = get_registry().get_selected();
    if (s && s->supports_shuffle2x())
        s->finish_shuffle2x(data, n);
}
// galois/mod.rs:118-142: dst[i] ^= source * coefficients[i], one strategy
// call per non-zero coefficient
inline void gf_muladd_column(uint16_t *const *dsts, size_t ndst, const uint16_t *src, size_t n,
                             const uint16_t *coeffs)
{
    const GaloisSimdStrategy &s = selected();
    for (size_t i = 0; i < ndst; ++i)
        if (coeffs[i])
            s.muladd(dsts[i], src, n, coeffs[i]);
}
// galois/mod.rs:328-349
inline void gf_muladd_column_shuffle2x(uint16_t *const *dsts, size_t ndst, const uint16_t *src,
                                       size_t n, const uint16_t *coeffs)
{
    const GaloisSimdStrategy &s = selected();
    if (!s.supports_shuffle2x()) {
        gf_muladd_column(dsts, ndst, src, n, coeffs);
        return;
    }
    for (size_t i = 0; i < ndst; ++i)
        if (coeffs[i])
            s.muladd_shuffle2x(dsts[i], src, n, coeffs[i]);
}
}  // namespace galois

// par2_rs.rs:88-126 (num_cpus: the host's thread count, or `threads`)
inline size_t optimal_data_batch_size(size_t recovery_blocks, size_t num_cpus)
{
    const size_t base = recovery_blocks >= 100 ? num_cpus * 8
                        : recovery_blocks >= 50 ? num_cpus * 4
                                                : num_cpus * 2;
    return std::min<size_t>(std::max<size_t>(base, 16), 128);
}
inline size_t optimal_recovery_batch_size(size_t recovery_blocks, size_t num_cpus)
{
    const size_t max_batch = std::max<size_t>(recovery_blocks / num_cpus, 1);
    return std::min<size_t>(std::max<size_t>(max_batch, 4), 8);
}

// StreamingEncoder (par2_rs.rs:775-902), restated over the strategy
// interface: data blocks are copied into reusable batch buffers (and
// prepared when the strategy uses shuffle2x); a full batch is multiplied into
// the recovery accumulators by worker threads, each taking recovery batches
// of 4-8 blocks and calling the column multiply-accumulate once per buffered
// data block (flush_batch, :816-870); finalize flushes the rest, finishes the
// accumulators and returns them as little-endian bytes.  Worker threads take
// recovery batches from a shared counter (the reference's rayon
// par_chunks_mut).
class StreamingEncoder {
  public:
    StreamingEncoder(const std::vector<uint16_t> &constants, size_t recovery_blocks,
                     size_t block_size, size_t threads = 0)
        : k_(constants.size()), r_(recovery_blocks), bs_(block_size), spb_(block_size / 2)
    {
        threads_ = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
        // par2_rs.rs:707-719: coeff[i][e] = c_i^e by repeated multiplication
        coeff_.assign(k_, std::vector<uint16_t>(r_));
        for (size_t i = 0; i < k_; ++i) {
            uint16_t c = 1;
            for (size_t e = 0; e < r_; ++e) {
                coeff_[i][e] = c;
                c = gf::mul(c, constants[i]);
            }
        }
        recovery_.assign(r_, std::vector<uint16_t>(spb_, 0));
        use_shuffle2x_ = galois::supports_shuffle2x();
        if (use_shuffle2x_)
            for (auto &rb : recovery_)
                galois::prepare_shuffle2x(rb.data(), rb.size());
        data_batch_size_ = optimal_data_batch_size(r_, threads_);
        recovery_batch_size_ = optimal_recovery_batch_size(r_, threads_);
        batch_buffers_.assign(data_batch_size_, std::vector<uint16_t>(spb_, 0));
        batch_indices_.reserve(data_batch_size_);
    }
    size_t data_batch_size() const { return data_batch_size_; }
    size_t recovery_batch_size() const { return recovery_batch_size_; }

    // par2_rs.rs:785-807; indices beyond the data block count are ignored
    void process_block(size_t data_block_idx, const uint16_t *block_data_u16, size_t nsym)
    {
        if (data_block_idx >= k_)
            return;
        const size_t slot = batch_indices_.size();
        std::vector<uint16_t> &buffer = batch_buffers_[slot];
        const size_t n = std::min(nsym, spb_);
        memcpy(buffer.data(), block_data_u16, n * 2);
        if (use_shuffle2x_)
            galois::prepare_shuffle2x(buffer.data(), n);
        batch_indices_.push_back(data_block_idx);
        if (batch_indices_.size() >= data_batch_size_)
            flush_batch();
    }

    // (exponent, bytes) for exponents 0..r-1 (par2_rs.rs:880-902)
    RecoveryBlocks finalize()
    {
        flush_batch();
        if (use_shuffle2x_)
            for (auto &rb : recovery_)
                galois::finish_shuffle2x(rb.data(), rb.size());
        RecoveryBlocks out(r_);
        for (size_t e = 0; e < r_; ++e) {
            out[e].first = static_cast<uint32_t>(e);
            out[e].second.resize(bs_ - bs_ % 2);
#if defined(__BYTE_ORDER__) && __BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__
            // the symbols' little-endian bytes are their memory image here
            memcpy(out[e].second.data(), recovery_[e].data(), spb_ * 2);
#else
            for (size_t x = 0; x < spb_; ++x) {
                out[e].second[2 * x] = static_cast<uint8_t>(recovery_[e][x]);
                out[e].second[2 * x + 1] = static_cast<uint8_t>(recovery_[e][x] >> 8);
            }
#endif
        }
        return out;
    }

  private:
    // par2_rs.rs:816-870
    void flush_batch()
    {
        if (batch_indices_.empty())
            return;
        const size_t ntasks = (r_ + recovery_batch_size_ - 1) / recovery_batch_size_;
        std::atomic<size_t> next{0};
        std::exception_ptr err;
        std::mutex err_mu;
        auto worker = [&] {
            std::vector<uint16_t *> dsts;
            std::vector<uint16_t> coeffs;
            for (size_t t; (t = next.fetch_add(1)) < ntasks;) {
                const size_t b0 = t * recovery_batch_size_;
                const size_t b1 = std::min(r_, b0 + recovery_batch_size_);
                try {
                    for (size_t slot = 0; slot < batch_indices_.size(); ++slot) {
                        const uint16_t *data_block = batch_buffers_[slot].data();
                        const std::vector<uint16_t> &c = coeff_[batch_indices_[slot]];
                        dsts.clear();
                        coeffs.clear();
                        for (size_t e = b0; e < b1; ++e) {
                            dsts.push_back(recovery_[e].data());
                            coeffs.push_back(c[e]);
                        }
                        if (use_shuffle2x_)
                            galois::gf_muladd_column_shuffle2x(dsts.data(), dsts.size(),
                                                               data_block, spb_, coeffs.data());
                        else
                            galois::gf_muladd_column(dsts.data(), dsts.size(), data_block, spb_,
                                                     coeffs.data());
                    }
                } catch (...) {
                    std::lock_guard<std::mutex> lock(err_mu);
                    if (!err)
                        err = std::current_exception();
                }
            }
        };
        const size_t nthreads = std::min(threads_, ntasks);
        std::vector<std::thread> pool;
        for (size_t w = 1; w < nthreads; ++w)
            pool.emplace_back(worker);
        worker();
        for (auto &th : pool)
            th.join();
        batch_indices_.clear();
        if (err)
            std::rethrow_exception(err);
    }

    size_t k_, r_, bs_, spb_, threads_;
    std::vector<std::vector<uint16_t>> coeff_;
    std::vector<std::vector<uint16_t>> recovery_;
    bool use_shuffle2x_ = false;
    std::vector<std::vector<uint16_t>> batch_buffers_;
    std::vector<size_t> batch_indices_;
    size_t data_batch_size_ = 16, recovery_batch_size_ = 4;
};

class Par2ReedSolomon {
  public:
    Par2ReedSolomon(size_t data_blocks, size_t /*recovery_blocks*/) : data_blocks_(data_blocks)
    {
        constants_.resize(data_blocks);
        if (data_blocks)
            check(p2g_par2_constants(data_blocks, constants_.data()));
    }
    const std::vector<uint16_t> &constants() const { return constants_; }

    RecoveryBlocks encode(const std::vector<std::vector<uint8_t>> &data_blocks,
                          size_t num_recovery, size_t block_size) const
    {
        if (data_blocks.size() != data_blocks_)
            throw Par2Error("Expected " + std::to_string(data_blocks_) + " data blocks, got " +
                            std::to_string(data_blocks.size()));
        if (block_size % 2 != 0)
            throw Par2Error("Block size must be multiple of 2");
        for (const auto &b : data_blocks)
            if (b.size() != block_size)
                throw Par2Error("Data block size mismatch: expected " + std::to_string(block_size) +
                                ", got " + std::to_string(b.size()));
        // the streaming encoder's batched path (the reference's encode makes
        // one strategy call per data x recovery block pair instead)
        StreamingEncoder enc(constants_, num_recovery, block_size);
        for (size_t i = 0; i < data_blocks.size(); ++i)
            enc.process_block(i, reinterpret_cast<const uint16_t *>(data_blocks[i].data()),
                              block_size / 2);
        return enc.finalize();
    }

    StreamingEncoder create_streaming_encoder(size_t recovery_blocks, size_t block_size,
                                              size_t chunk_size) const
    {
        if (block_size % 2 != 0)
            throw Par2Error("Block size must be multiple of 2");
        if (chunk_size % 2 != 0)
            throw Par2Error("Chunk size must be multiple of 2");
        if (chunk_size > block_size)
            throw Par2Error("Chunk size cannot exceed block size");
        return StreamingEncoder(constants_, recovery_blocks, block_size);
    }

    // present_recovery_indices are block indices >= data_blocks (recovery
    // block i has exponent recovery_exponents[i - data_blocks]); the first m
    // of them are used, as in the reference (par2_rs.rs:348-353).
    ReconstructionTransform compute_reconstruction_transform(
        const std::vector<size_t> &missing_indices, const std::vector<size_t> &present_data_indices,
        const std::vector<size_t> &present_recovery_indices,
        const std::vector<uint32_t> &recovery_exponents) const
    {
        (void)present_data_indices;
        const size_t m = missing_indices.size();
        if (m == 0)
            throw Par2Error("No missing blocks to reconstruct");
        if (present_recovery_indices.size() < m)
            throw Par2Error("Need " + std::to_string(m) + " recovery blocks, have " +
                            std::to_string(present_recovery_indices.size()));
        ReconstructionTransform t;
        t.missing.assign(missing_indices.begin(), missing_indices.end());
        std::sort(t.missing.begin(), t.missing.end());
        for (size_t q = 0; q < m; ++q)
            t.exponents.push_back(recovery_exponents[present_recovery_indices[q] - data_blocks_]);
        t.inverse.assign(m * m, 0);
        const int rc = p2g_reconstruction_matrix(codec_ctx(), data_blocks_, t.missing.data(), m,
                                                 t.exponents.data(), t.inverse.data());
        if (rc == P2G_ESINGULAR)
            throw Par2Error("Singular matrix");
        check(rc);
        return t;
    }

    // read_block(block_idx, offset, size) -> bytes; write_result(missing_idx, bytes).
    // Recovery chunks are read first, then the present data chunks, and the
    // results are written in missing_indices order (par2_rs.rs:487-499,
    // 540-553, 653-669).  A data block neither missing nor present adds
    // nothing, as in the reference.
    void reconstruct_streaming_chunk(
        const std::vector<size_t> &missing_indices, const std::vector<size_t> &present_data_indices,
        const std::vector<size_t> &present_recovery_indices, const ReconstructionTransform &transform,
        size_t chunk_offset, size_t chunk_size,
        const std::function<std::vector<uint8_t>(size_t, size_t, size_t)> &read_block,
        const std::function<void(size_t, std::vector<uint8_t>)> &write_result) const
    {
        const size_t m = missing_indices.size();
        if (m == 0)
            return;
        if (present_recovery_indices.size() < m)
            throw Par2Error("Need " + std::to_string(m) + " recovery blocks, have " +
                            std::to_string(present_recovery_indices.size()));
        if (transform.missing.size() != m)
            throw Par2Error("Transform does not match the missing blocks");
        auto fetch = [&](size_t idx) {
            std::vector<uint8_t> b = read_block(idx, chunk_offset, chunk_size);
            if (b.size() != chunk_size)
                throw Par2Error("Chunk size mismatch for block " + std::to_string(idx));
            return b;
        };
        std::vector<std::vector<uint8_t>> rec(m), slot(data_blocks_);
        for (size_t q = 0; q < m; ++q)
            rec[q] = fetch(present_recovery_indices[q]);
        for (size_t idx : present_data_indices)
            if (idx < data_blocks_ &&
                !std::binary_search(transform.missing.begin(), transform.missing.end(), idx))
                slot[idx] = fetch(idx);
        const std::vector<uint8_t> zero(chunk_size, 0);
        std::vector<const uint8_t *> dp, rp;
        for (size_t i = 0; i < data_blocks_; ++i)
            if (!std::binary_search(transform.missing.begin(), transform.missing.end(), i))
                dp.push_back(slot[i].empty() ? zero.data() : slot[i].data());
        for (auto &r : rec)
            rp.push_back(r.data());
        std::vector<std::vector<uint8_t>> out(m, std::vector<uint8_t>(chunk_size));
        std::vector<uint8_t *> op;
        for (auto &o : out)
            op.push_back(o.data());
        if (chunk_size) {
            const int rc = p2g_repair(codec_ctx(), data_blocks_, chunk_size, transform.missing.data(),
                                      m, dp.data(), transform.exponents.data(), rp.data(), op.data(),
                                      0);
            if (rc == P2G_ESINGULAR)
                throw Par2Error("Singular matrix");
            check(rc);
        }
        for (size_t idx : missing_indices) {
            const size_t j = static_cast<size_t>(
                std::lower_bound(transform.missing.begin(), transform.missing.end(), idx) -
                transform.missing.begin());
            write_result(idx, std::move(out[j]));
        }
    }

  private:
    size_t data_blocks_;
    std::vector<uint16_t> constants_;
};

}  // namespace par2
