// format_capi.cpp -- the C ABI of par2format.h over par2_pipeline.hpp.
#include "../../include/par2format.h"

#include <string.h>

#include <string>

#include "par2_codec.hpp"
#include "par2_pipeline.hpp"

namespace {

thread_local std::string g_error;

int fail(const std::exception &e)
{
    g_error = e.what();
    if (dynamic_cast<const par2::Cancelled *>(&e))
        return P2F_ECANCELLED;
    if (g_error.find("repair was not requested") != std::string::npos)
        return P2F_EDAMAGED;
    if (g_error.find("Singular matrix") != std::string::npos)
        return P2F_ESINGULAR;
    if (g_error.find("Insufficient recovery") != std::string::npos)
        return P2F_EINSUFFICIENT;
    return P2F_ERROR;
}

void fill(p2f_stats *out, const par2::PipelineStats &s)
{
    if (!out)
        return;
    out->ms_scan = s.ms_scan;
    out->ms_ingest = s.ms_ingest;
    out->ms_gpu = s.ms_gpu;
    out->ms_write = s.ms_write;
    out->ms_total = s.ms_total;
    out->block_size = s.block_size;
    out->data_blocks = s.data_blocks;
    out->recovery_blocks = s.recovery_blocks;
    out->bytes_read = s.bytes_read;
    out->damaged_blocks = s.damaged_blocks;
    out->files_written = s.files_written;
}

}  // namespace

extern "C" {

int p2f_create(const char *const *inputs, size_t n, const char *output, uint64_t block_size,
               float redundancy_percent, int scheme, p2f_stats *stats)
{
    return p2f_create_ex(inputs, n, output, block_size, redundancy_percent, scheme, nullptr,
                         nullptr, stats);
}

int p2f_create_ex(const char *const *inputs, size_t n, const char *output, uint64_t block_size,
                  float redundancy_percent, int scheme, p2f_progress_fn progress, void *user,
                  p2f_stats *stats)
{
    g_error.clear();
    try {
        if (!inputs && n)
            throw par2::Par2Error("p2f_create: null input list");
        std::vector<std::filesystem::path> in;
        for (size_t i = 0; i < n; ++i) {
            if (!inputs[i])
                throw par2::Par2Error("p2f_create: null input path");
            in.emplace_back(inputs[i]);
        }
        if (scheme != P2F_SCHEME_SINGLE && scheme != P2F_SCHEME_EXPONENTIAL)
            throw par2::Par2Error("p2f_create: unknown volume scheme");
        par2::Par2Creator c(in);
        c.with_redundancy(redundancy_percent)
            .with_volume_scheme(scheme == P2F_SCHEME_SINGLE ? par2::VolumeScheme::Single
                                                            : par2::VolumeScheme::Exponential);
        if (output)
            c.with_output_path(output);
        if (block_size)
            c.with_block_size(block_size);
        if (progress)
            c.with_progress([progress, user](par2::Par2Operation op, uint64_t cur, uint64_t tot) {
                progress(user, static_cast<int>(op), cur, tot);
            });
        c.create();
        fill(stats, c.stats());
        return P2F_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int p2f_repair(const char *par2_path, const char *dir, uint64_t *rebuilt, p2f_stats *stats)
{
    g_error.clear();
    try {
        if (!par2_path || !dir)
            throw par2::Par2Error("p2f_repair: null path");
        par2::Par2Repairer r(par2_path, dir);
        const uint64_t n = r.repair();
        if (rebuilt)
            *rebuilt = n;
        fill(stats, r.stats());
        return P2F_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int p2f_repair_ex(const char *par2_path, const char *dir, int do_repair, int purge,
                  p2f_progress_fn progress, void *user, const volatile int32_t *cancel,
                  uint64_t *rebuilt, p2f_stats *stats)
{
    g_error.clear();
    try {
        if (!par2_path || !dir)
            throw par2::Par2Error("p2f_repair_ex: null path");
        par2::Par2Repairer r(par2_path, dir);
        r.with_repair(do_repair != 0).with_purge(purge != 0);
        if (progress)
            r.with_progress([progress, user](par2::Par2Operation op, uint64_t cur, uint64_t tot) {
                progress(user, static_cast<int>(op), cur, tot);
            });
        if (cancel)
            r.with_cancel([cancel] { return *cancel != 0; });
        const uint64_t n = r.repair();
        if (rebuilt)
            *rebuilt = n;
        fill(stats, r.stats());
        return P2F_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

int p2f_streaming_encode(const uint8_t *const *src, size_t k, size_t block_size, size_t r,
                         uint8_t *const *out, int threads)
{
    g_error.clear();
    try {
        if ((k && !src) || (r && !out))
            throw par2::Par2Error("p2f_streaming_encode: null argument");
        if (block_size % 2 != 0)
            throw par2::Par2Error("Block size must be multiple of 2");
        par2::Par2ReedSolomon codec(k, r);
        par2::StreamingEncoder enc(codec.constants(), r, block_size,
                                   threads > 0 ? static_cast<size_t>(threads) : 0);
        for (size_t i = 0; i < k; ++i)
            enc.process_block(i, reinterpret_cast<const uint16_t *>(src[i]), block_size / 2);
        par2::RecoveryBlocks rec = enc.finalize();
        for (size_t e = 0; e < r; ++e)
            memcpy(out[e], rec[e].second.data(), rec[e].second.size());
        return P2F_OK;
    } catch (const std::exception &e) {
        return fail(e);
    }
}

const char *p2f_last_error(void) { return g_error.c_str(); }

}  // extern "C"
