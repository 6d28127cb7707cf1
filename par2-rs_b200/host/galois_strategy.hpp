// galois_strategy.hpp -- C++ mirror of par2-rs's GF(2^16) strategy plugin
// interface, with the CUDA strategy that drives libpar2gpu through its C ABI.
//
//   trait GaloisSimdStrategy        src/galois/simd/mod.rs:24-128
//   enum Priority                   src/galois/simd/mod.rs:14-21
//   struct SimdRegistry             src/galois/simd/mod.rs:131-229
//   get_registry / PAR2_SIMD_STRATEGY  src/galois/simd/mod.rs:237-253,
//                                      src/galois/mod.rs:230-235
//
// Same names, argument meaning and behaviour: register() keeps only
// available strategies, select_best() keeps the FIRST strategy of the highest
// priority (a later one needs a strictly higher priority), select_by_name()
// overrides, and the methods are infallible (a failing CUDA call throws, as a
// panicking Rust strategy would abort the caller).
#pragma once
#include <stdint.h>
#include <stdlib.h>

#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/par2gpu.h"

namespace par2 {

enum class Priority : int {
    Fallback = 0,
    Basic = 10,
    Enhanced = 20,
    Advanced = 30,
    Optimal = 40,
};

class GaloisSimdStrategy {
  public:
    virtual ~GaloisSimdStrategy() = default;
    virtual const char *name() const = 0;
    virtual bool is_available() const = 0;
    virtual Priority priority() const = 0;
    // data[i] = scalar * data[i]
    virtual void mul_slice(uint16_t scalar, uint16_t *data, size_t n) const = 0;
    // dst[i] ^= src[i] * scalar
    virtual void muladd(uint16_t *dst, const uint16_t *src, size_t n, uint16_t scalar) const = 0;
    // dsts[d][off..off+len) ^= sum_s coeffs[d][s] * srcs[s][off..off+len)
    virtual void muladd_region(uint16_t *const *dsts, size_t ndst, const uint16_t *const *srcs,
                               size_t nsrc, const uint16_t *const *coeffs, size_t region_offset,
                               size_t region_size) const = 0;
    // shuffle2x hooks with the trait's defaults (mod.rs:68-127)
    virtual bool supports_shuffle2x() const { return false; }
    virtual void prepare_shuffle2x(uint16_t *, size_t) const {}
    virtual void finish_shuffle2x(uint16_t *, size_t) const {}
    virtual void muladd_shuffle2x(uint16_t *dst, const uint16_t *src, size_t n,
                                  uint16_t scalar) const
    {
        muladd(dst, src, n, scalar);
    }
    virtual void muladd_region_shuffle2x(uint16_t *const *dsts, size_t ndst,
                                         const uint16_t *const *srcs, size_t nsrc,
                                         const uint16_t *const *coeffs, size_t region_offset,
                                         size_t region_size) const
    {
        muladd_region(dsts, ndst, srcs, nsrc, coeffs, region_offset, region_size);
    }
};

class SimdRegistry {
  public:
    void register_strategy(std::unique_ptr<GaloisSimdStrategy> s)
    {
        if (s && s->is_available())
            strategies_.push_back(std::move(s));
    }
    void select_best()
    {
        if (strategies_.empty())
            return;
        size_t best = 0;
        for (size_t i = 1; i < strategies_.size(); ++i)
            if (strategies_[i]->priority() > strategies_[best]->priority())
                best = i;
        selected_ = static_cast<long>(best);
    }
    const GaloisSimdStrategy *get_selected() const
    {
        return selected_ < 0 ? nullptr : strategies_[selected_].get();
    }
    bool select_by_name(const std::string &name)
    {
        for (size_t i = 0; i < strategies_.size(); ++i)
            if (name == strategies_[i]->name()) {
                selected_ = static_cast<long>(i);
                return true;
            }
        return false;
    }
    std::vector<std::pair<std::string, Priority>> list_available() const
    {
        std::vector<std::pair<std::string, Priority>> out;
        for (const auto &s : strategies_)
            out.emplace_back(s->name(), s->priority());
        return out;
    }

  private:
    std::vector<std::unique_ptr<GaloisSimdStrategy>> strategies_;
    long selected_ = -1;
};

// Throws with p2g_last_error() when a C ABI call fails.
inline void check(int rc)
{
    if (rc != P2G_OK)
        throw std::runtime_error(std::string("libpar2gpu: ") + p2g_last_error());
}

// The GPU strategy: "CUDA-sm100a", Optimal, available iff an sm_100 device is
// present.  One device context per strategy object; the context serialises
// concurrent callers (the trait is Send + Sync).
class CudaSm100aStrategy final : public GaloisSimdStrategy {
  public:
    explicit CudaSm100aStrategy(int device = 0) : device_(device) {}
    ~CudaSm100aStrategy() override
    {
        if (ctx_)
            p2g_destroy(ctx_);
    }
    const char *name() const override { return "CUDA-sm100a"; }
    bool is_available() const override
    {
        int avail = 0;
        p2g_strategy_info(nullptr, nullptr, &avail);
        return avail != 0;
    }
    Priority priority() const override { return Priority::Optimal; }
    void mul_slice(uint16_t scalar, uint16_t *data, size_t n) const override
    {
        check(p2g_mul_slice(ctx(), scalar, data, n, 0));
    }
    void muladd(uint16_t *dst, const uint16_t *src, size_t n, uint16_t scalar) const override
    {
        check(p2g_muladd(ctx(), dst, src, n, scalar, 0));
    }
    void muladd_region(uint16_t *const *dsts, size_t ndst, const uint16_t *const *srcs,
                       size_t nsrc, const uint16_t *const *coeffs, size_t region_offset,
                       size_t region_size) const override
    {
        check(p2g_muladd_region(ctx(), dsts, ndst, srcs, nsrc, coeffs, region_offset,
                                region_size, 0));
    }
    // shuffle2x: prepared buffers live on the device while the callers'
    // loops record multiply-accumulates; finish runs them and copies back
    bool supports_shuffle2x() const override { return p2g_supports_shuffle2x() != 0; }
    void prepare_shuffle2x(uint16_t *data, size_t n) const override
    {
        check(p2g_prepare_shuffle2x(ctx(), data, n));
    }
    void finish_shuffle2x(uint16_t *data, size_t n) const override
    {
        check(p2g_finish_shuffle2x(ctx(), data, n));
    }
    void muladd_shuffle2x(uint16_t *dst, const uint16_t *src, size_t n,
                          uint16_t scalar) const override
    {
        check(p2g_muladd_shuffle2x(ctx(), dst, src, n, scalar));
    }
    void muladd_region_shuffle2x(uint16_t *const *dsts, size_t ndst, const uint16_t *const *srcs,
                                 size_t nsrc, const uint16_t *const *coeffs, size_t region_offset,
                                 size_t region_size) const override
    {
        check(p2g_muladd_region_shuffle2x(ctx(), dsts, ndst, srcs, nsrc, coeffs, region_offset,
                                          region_size));
    }
    p2g_ctx *ctx() const
    {
        std::call_once(once_, [this] { check(p2g_create(device_, &ctx_)); });
        return ctx_;
    }

  private:
    int device_;
    mutable std::once_flag once_;
    mutable p2g_ctx *ctx_ = nullptr;
};

// The global registry: the CUDA strategy registered first (it wins the
// priority tie against any CPU strategy registered after it), then best
// selection, then the PAR2_SIMD_STRATEGY name override.
inline SimdRegistry &get_registry()
{
    static SimdRegistry reg = [] {
        SimdRegistry r;
        r.register_strategy(std::make_unique<CudaSm100aStrategy>());
        r.select_best();
        if (const char *forced = getenv("PAR2_SIMD_STRATEGY"))
            r.select_by_name(forced);
        return r;
    }();
    return reg;
}

}  // namespace par2
