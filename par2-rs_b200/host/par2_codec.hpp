// par2_codec.hpp -- C++ mirror of par2-rs's Reed-Solomon codec API over
// libpar2gpu (par2-rs src/par2_rs.rs):
//
//   Par2ReedSolomon::new / encode            par2_rs.rs:160-313
//   compute_reconstruction_transform         par2_rs.rs:319-422
//   reconstruct_streaming_chunk              par2_rs.rs:442-675
//   create_streaming_encoder                 par2_rs.rs:687-772
//   StreamingEncoder::{process_block, finalize}  par2_rs.rs:775-902
//
// Same names, argument meaning and error strings.  The transform holds the
// decode matrix A^-1 formed on the GPU (the reference records the elimination
// steps instead; A^-1 is what those steps apply), so a singular set is
// reported when the transform is computed, as in the reference.
// Reconstruction runs as the two multiply-accumulate passes of p2g_repair.
#pragma once
#include <string.h>

#include <algorithm>
#include <functional>
#include <numeric>
#include <string>
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

class StreamingEncoder {
  public:
    StreamingEncoder(size_t data_blocks, size_t recovery_blocks, size_t block_size)
        : k_(data_blocks), r_(recovery_blocks), bs_(block_size), data_(k_ * bs_, 0)
    {
    }
    // block_data_u16: the block as u16 symbols; indices beyond the data block
    // count are ignored (par2_rs.rs:785-788).  Blocks never given count as zero.
    void process_block(size_t data_block_idx, const uint16_t *block_data_u16, size_t nsym)
    {
        if (data_block_idx >= k_)
            return;
        const size_t n = std::min(nsym * 2, bs_);
        memcpy(data_.data() + data_block_idx * bs_, block_data_u16, n);
    }
    // (exponent, bytes) for exponents 0..r-1 (par2_rs.rs:880-902)
    RecoveryBlocks finalize()
    {
        RecoveryBlocks out(r_);
        std::vector<const uint8_t *> src(k_);
        std::vector<uint8_t *> dst(r_);
        std::vector<uint32_t> exps(r_);
        for (size_t i = 0; i < k_; ++i)
            src[i] = data_.data() + i * bs_;
        for (size_t e = 0; e < r_; ++e) {
            out[e].first = static_cast<uint32_t>(e);
            out[e].second.assign(bs_, 0);
            dst[e] = out[e].second.data();
            exps[e] = static_cast<uint32_t>(e);
        }
        if (r_ && k_ && bs_)
            check(p2g_encode(codec_ctx(), src.data(), k_, bs_, exps.data(), r_, dst.data(), 0));
        return out;
    }

  private:
    size_t k_, r_, bs_;
    std::vector<uint8_t> data_;
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
        StreamingEncoder enc(data_blocks_, num_recovery, block_size);
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
        return StreamingEncoder(data_blocks_, recovery_blocks, block_size);
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
