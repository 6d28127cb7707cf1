// Tests of the C++ mirror of par2-rs's strategy interface and codec API
// (par2-rs_b200/host/), written after par2-rs's own tests:
//   src/galois/tests.rs:482-553   test_each_simd_strategy
//   src/par2_rs.rs:909-971        test_encode_basic / wrong count / wrong size / odd size
//   src/galois/simd/mod.rs:131-229  registry selection rules
// `test_host registry` needs no GPU; `test_host gpu` drives the CUDA strategy.
#include <stdio.h>
#include <string.h>

#include <map>
#include <mutex>
#include <random>
#include <string>
#include <thread>

#include "../../par2-rs_b200/host/par2_codec.hpp"

using namespace par2;

static int failures = 0;
#define CHECK(cond, ...)                                         \
    do {                                                         \
        if (!(cond)) {                                           \
            ++failures;                                          \
            fprintf(stderr, "FAIL %s:%d: ", __FILE__, __LINE__); \
            fprintf(stderr, __VA_ARGS__);                        \
            fprintf(stderr, "\n");                               \
        }                                                        \
    } while (0)

// scalar GF(2^16) for the checks (poly 0x1100B, generator 2)
static uint16_t glog[65536], gexp[131070];
static void tables()
{
    uint32_t b = 1;
    for (uint32_t l = 0; l < 65535; ++l) {
        gexp[l] = gexp[l + 65535] = static_cast<uint16_t>(b);
        glog[b] = static_cast<uint16_t>(l);
        b <<= 1;
        if (b & 0x10000)
            b ^= 0x1100B;
    }
}
static uint16_t gf_mul(uint16_t a, uint16_t b)
{
    return (a && b) ? gexp[glog[a] + glog[b]] : 0;
}
static uint16_t gf_pow(uint16_t a, uint32_t n)
{
    if (n == 0)
        return 1;
    if (!a)
        return 0;
    return gexp[(static_cast<uint64_t>(glog[a]) * n) % 65535];
}

struct Fake final : GaloisSimdStrategy {
    std::string nm;
    Priority pr;
    bool av;
    Fake(const char *n, Priority p, bool a) : nm(n), pr(p), av(a) {}
    const char *name() const override { return nm.c_str(); }
    bool is_available() const override { return av; }
    Priority priority() const override { return pr; }
    void mul_slice(uint16_t, uint16_t *, size_t) const override {}
    void muladd(uint16_t *, const uint16_t *, size_t, uint16_t) const override {}
    void muladd_region(uint16_t *const *, size_t, const uint16_t *const *, size_t,
                       const uint16_t *const *, size_t, size_t) const override {}
};

static void test_registry()
{
    SimdRegistry r;
    r.register_strategy(std::make_unique<Fake>("SSE2", Priority::Basic, true));
    r.register_strategy(std::make_unique<Fake>("SSSE3", Priority::Enhanced, true));
    r.register_strategy(std::make_unique<Fake>("AVX2-Shuffle", Priority::Optimal, true));
    r.register_strategy(std::make_unique<Fake>("Missing", Priority::Optimal, false));
    r.register_strategy(std::make_unique<Fake>("AVX2-PCLMUL", Priority::Optimal, true));
    CHECK(r.get_selected() == nullptr, "nothing selected before select_best");
    r.select_best();
    CHECK(r.list_available().size() == 4, "unavailable strategies are not registered");
    CHECK(std::string(r.get_selected()->name()) == "AVX2-Shuffle",
          "the first strategy of the highest priority wins a tie");
    CHECK(r.select_by_name("SSSE3") && std::string(r.get_selected()->name()) == "SSSE3",
          "select_by_name");
    CHECK(!r.select_by_name("NEON") && std::string(r.get_selected()->name()) == "SSSE3",
          "an unknown name is refused and keeps the selection");
    SimdRegistry empty;
    empty.select_best();
    CHECK(empty.get_selected() == nullptr, "an empty registry selects nothing");
    // the CUDA strategy ranks Optimal and is registered first, so it wins
    SimdRegistry g;
    g.register_strategy(std::make_unique<Fake>("CUDA-sm100a", Priority::Optimal, true));
    g.register_strategy(std::make_unique<Fake>("AVX2-Shuffle", Priority::Optimal, true));
    g.select_best();
    CHECK(std::string(g.get_selected()->name()) == "CUDA-sm100a", "CUDA strategy selected");
    CudaSm100aStrategy cuda;
    CHECK(std::string(cuda.name()) == "CUDA-sm100a" && cuda.priority() == Priority::Optimal,
          "strategy identity");
    CHECK(cuda.supports_shuffle2x(), "the GPU strategy takes the shuffle2x hooks");
}

// A CPU strategy for the streaming encoder's call sequence: prepare_shuffle2x
// changes the buffer in place (XOR with a mask) and finish_shuffle2x undoes
// it, so a buffer used without a prepare or read without a finish gives wrong
// results; the hooks also check that every multiply-accumulate names prepared
// buffers and count the calls and the threads that made them.
struct ShuffleFake final : GaloisSimdStrategy {
    static constexpr uint16_t kMask = 0x5A5A;
    mutable std::mutex mu;
    mutable std::map<const uint16_t *, size_t> prepared;  // address -> symbols
    mutable size_t calls = 0, violations = 0;
    mutable std::map<std::thread::id, size_t> threads;
    const char *name() const override { return "TestShuffle"; }
    bool is_available() const override { return true; }
    Priority priority() const override { return Priority::Optimal; }
    void mul_slice(uint16_t c, uint16_t *d, size_t n) const override
    {
        for (size_t i = 0; i < n; ++i)
            d[i] = gf_mul(d[i], c);
    }
    void muladd(uint16_t *dst, const uint16_t *src, size_t n, uint16_t c) const override
    {
        for (size_t i = 0; i < n; ++i)
            dst[i] ^= gf_mul(src[i], c);
    }
    void muladd_region(uint16_t *const *, size_t, const uint16_t *const *, size_t,
                       const uint16_t *const *, size_t, size_t) const override {}
    bool supports_shuffle2x() const override { return true; }
    void prepare_shuffle2x(uint16_t *d, size_t n) const override
    {
        for (size_t i = 0; i < n; ++i)
            d[i] ^= kMask;
        std::lock_guard<std::mutex> lock(mu);
        prepared[d] = n;
    }
    void finish_shuffle2x(uint16_t *d, size_t n) const override
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!prepared.count(d))
            ++violations;
        prepared.erase(d);
        for (size_t i = 0; i < n; ++i)
            d[i] ^= kMask;
    }
    void muladd_shuffle2x(uint16_t *dst, const uint16_t *src, size_t n, uint16_t c) const override
    {
        {
            std::lock_guard<std::mutex> lock(mu);
            ++calls;
            ++threads[std::this_thread::get_id()];
            auto a = prepared.find(dst), b = prepared.find(src);
            if (a == prepared.end() || b == prepared.end() || a->second < n || b->second < n)
                ++violations;
        }
        for (size_t i = 0; i < n; ++i)
            dst[i] = static_cast<uint16_t>(
                ((dst[i] ^ kMask) ^ gf_mul(static_cast<uint16_t>(src[i] ^ kMask), c)) ^ kMask);
    }
};

// StreamingEncoder (par2_rs.rs:775-902) over a strategy with shuffle2x: the
// reference's batch sizes (par2_rs.rs:88-126), every data block prepared,
// every accumulator prepared and finished, one call per (recovery block, data
// block) pair from several worker threads, and the recovery slices of the
// scalar definition.
static void test_streaming_encoder()
{
    SimdRegistry &reg = get_registry();
    auto owned = std::make_unique<ShuffleFake>();
    const ShuffleFake *fake = owned.get();
    reg.register_strategy(std::move(owned));
    CHECK(reg.select_by_name("TestShuffle"), "select the test strategy");
    CHECK(optimal_data_batch_size(205, 16) == 128 && optimal_data_batch_size(37, 4) == 16 &&
              optimal_data_batch_size(60, 8) == 32,
          "data batch sizes");
    CHECK(optimal_recovery_batch_size(205, 16) == 8 && optimal_recovery_batch_size(37, 4) == 8 &&
              optimal_recovery_batch_size(13, 8) == 4,
          "recovery batch sizes");
    const size_t k = 300, r = 37, bs = 96;
    std::mt19937 rng(11);
    std::vector<std::vector<uint8_t>> data(k, std::vector<uint8_t>(bs));
    for (auto &b : data)
        for (auto &x : b)
            x = static_cast<uint8_t>(rng());
    Par2ReedSolomon codec(k, r);
    StreamingEncoder enc(codec.constants(), r, bs, 4);
    CHECK(enc.data_batch_size() == 16 && enc.recovery_batch_size() == 8, "encoder batch sizes");
    for (size_t i = 0; i < k; ++i)
        enc.process_block(i, reinterpret_cast<const uint16_t *>(data[i].data()), bs / 2);
    enc.process_block(k + 5, reinterpret_cast<const uint16_t *>(data[0].data()), bs / 2);
    RecoveryBlocks rec = enc.finalize();
    bool ok = rec.size() == r;
    for (size_t e = 0; e < r && ok; ++e) {
        ok = rec[e].first == e && rec[e].second.size() == bs;
        for (size_t x = 0; x < bs / 2 && ok; ++x) {
            uint16_t want = 0;
            for (size_t i = 0; i < k; ++i) {
                const uint16_t v = static_cast<uint16_t>(data[i][2 * x] | (data[i][2 * x + 1] << 8));
                want ^= gf_mul(gf_pow(codec.constants()[i], static_cast<uint32_t>(e)), v);
            }
            ok = want == static_cast<uint16_t>(rec[e].second[2 * x] | (rec[e].second[2 * x + 1] << 8));
        }
    }
    CHECK(ok, "recovery slices equal sum_i c_i^e D_i");
    CHECK(fake->calls == k * r, "one call per (recovery, data) pair: %zu", fake->calls);
    CHECK(fake->violations == 0, "every call on prepared buffers, every finish after a prepare");
    CHECK(fake->threads.size() > 1, "the batches ran on several threads (%zu)", fake->threads.size());
    reg.select_best();
}

static void test_each_simd_strategy()
{
    const GaloisSimdStrategy *s = get_registry().get_selected();
    CHECK(s && std::string(s->name()) == "CUDA-sm100a", "registry selects the CUDA strategy");
    if (!s)
        return;
    const size_t sizes[] = {7, 8, 15, 16, 31, 32, 100, 1024};
    const uint16_t scalars[] = {0, 1, 2, 12345, 65535};
    for (size_t n : sizes)
        for (uint16_t c : scalars) {
            std::vector<uint16_t> d(n), want(n), src(n), dst(n), want2(n);
            for (size_t i = 0; i < n; ++i) {
                d[i] = static_cast<uint16_t>(i * 97 + 1);
                want[i] = gf_mul(d[i], c);
                src[i] = static_cast<uint16_t>(i * 13 + 7);
                dst[i] = static_cast<uint16_t>(i * 17 + 3);
                want2[i] = dst[i] ^ gf_mul(src[i], c);
            }
            s->mul_slice(c, d.data(), n);
            CHECK(d == want, "mul_slice size=%zu scalar=%u", n, c);
            s->muladd(dst.data(), src.data(), n, c);
            CHECK(dst == want2, "muladd size=%zu scalar=%u", n, c);
            std::vector<uint16_t> dst2 = dst;
            s->muladd_shuffle2x(dst2.data(), src.data(), n, c);  // trait default = muladd
            for (size_t i = 0; i < n; ++i)
                want2[i] = dst[i] ^ gf_mul(src[i], c);
            CHECK(dst2 == want2, "muladd_shuffle2x size=%zu scalar=%u", n, c);
        }
    // muladd_region over a sub-region, one zero coefficient
    std::mt19937 rng(3);
    const size_t len = 3000, nd = 5, ns = 7, off = 77, rs = 2500;
    std::vector<std::vector<uint16_t>> D(nd, std::vector<uint16_t>(len)),
        S(ns, std::vector<uint16_t>(len)), C(nd, std::vector<uint16_t>(ns));
    for (auto &v : D)
        for (auto &x : v) x = static_cast<uint16_t>(rng());
    for (auto &v : S)
        for (auto &x : v) x = static_cast<uint16_t>(rng());
    for (auto &v : C)
        for (auto &x : v) x = static_cast<uint16_t>(rng());
    C[1][2] = 0;
    auto W = D;
    for (size_t d = 0; d < nd; ++d)
        for (size_t t = 0; t < ns; ++t)
            for (size_t x = off; x < off + rs; ++x)
                W[d][x] ^= gf_mul(S[t][x], C[d][t]);
    std::vector<uint16_t *> dp;
    std::vector<const uint16_t *> sp, cp;
    for (auto &v : D) dp.push_back(v.data());
    for (auto &v : S) sp.push_back(v.data());
    for (auto &v : C) cp.push_back(v.data());
    s->muladd_region(dp.data(), nd, sp.data(), ns, cp.data(), off, rs);
    CHECK(D == W, "muladd_region");
}

template <class F> static bool throws_with(F f, const char *text)
{
    try {
        f();
    } catch (const Par2Error &e) {
        return strstr(e.what(), text) != nullptr;
    }
    return false;
}

static void test_codec()
{
    // test_encode_basic (par2_rs.rs:909-935)
    Par2ReedSolomon rs(3, 2);
    std::vector<std::vector<uint8_t>> blocks = {{1, 0, 2, 0, 3, 0, 4, 0},
                                                {5, 0, 6, 0, 7, 0, 8, 0},
                                                {9, 0, 10, 0, 11, 0, 12, 0}};
    RecoveryBlocks res = rs.encode(blocks, 2, 8);
    CHECK(res.size() == 2 && res[0].first == 0 && res[1].first == 1, "two recovery blocks");
    CHECK(res[0].second.size() == 8 && res[1].second.size() == 8, "8-byte recovery blocks");
    for (int e = 0; e < 2; ++e)
        for (int x = 0; x < 4; ++x) {
            uint16_t acc = 0;
            for (int i = 0; i < 3; ++i) {
                const uint16_t v = blocks[i][2 * x] | (blocks[i][2 * x + 1] << 8);
                acc ^= gf_mul(v, gf_pow(rs.constants()[i], e));
            }
            const uint16_t got = res[e].second[2 * x] | (res[e].second[2 * x + 1] << 8);
            CHECK(got == acc, "recovery value e=%d x=%d", e, x);
        }
    // error cases (par2_rs.rs:937-971)
    CHECK(throws_with([&] { rs.encode({blocks[0], blocks[1]}, 2, 8); },
                      "Expected 3 data blocks, got 2"),
          "wrong block count");
    CHECK(throws_with([] { Par2ReedSolomon(2, 1).encode({{1, 0, 2, 0, 3, 0, 4, 0}, {5, 0, 6, 0}}, 1, 8); },
                      "Data block size mismatch: expected 8, got 4"),
          "mismatched block sizes");
    CHECK(throws_with([] { Par2ReedSolomon(2, 1).encode({{1, 2, 3}, {4, 5, 6}}, 1, 3); },
                      "Block size must be multiple of 2"),
          "odd block size");
    CHECK(throws_with([&] { rs.create_streaming_encoder(2, 8, 3); },
                      "Chunk size must be multiple of 2"),
          "odd chunk size");
    CHECK(throws_with([&] { rs.create_streaming_encoder(2, 8, 16); },
                      "Chunk size cannot exceed block size"),
          "chunk larger than block");

    // streaming encoder == encode; then rebuild three blocks in two chunks
    std::mt19937 rng(9);
    const size_t k = 50, bs = 8192, r = 6, chunk = 4096;
    std::vector<std::vector<uint8_t>> data(k, std::vector<uint8_t>(bs));
    for (auto &b : data)
        for (auto &x : b) x = static_cast<uint8_t>(rng());
    Par2ReedSolomon codec(k, r);
    RecoveryBlocks rec = codec.encode(data, r, bs);
    StreamingEncoder enc = codec.create_streaming_encoder(r, bs, chunk);
    for (size_t i = 0; i < k; ++i)
        enc.process_block(i, reinterpret_cast<const uint16_t *>(data[i].data()), bs / 2);
    enc.process_block(k + 3, reinterpret_cast<const uint16_t *>(data[0].data()), bs / 2);
    CHECK(enc.finalize() == rec, "streaming encoder equals encode");

    const std::vector<size_t> missing = {40, 3, 17};   // any order, as the caller has them
    std::vector<size_t> present;
    for (size_t i = 0; i < k; ++i)
        if (i != 3 && i != 17 && i != 40)
            present.push_back(i);
    const std::vector<size_t> prec = {k + 1, k + 2, k + 4, k + 5};   // first m used
    std::vector<uint32_t> exps(r);
    for (size_t e = 0; e < r; ++e) exps[e] = static_cast<uint32_t>(e);
    ReconstructionTransform t = codec.compute_reconstruction_transform(missing, present, prec, exps);
    CHECK(t.inverse.size() == 9 && t.exponents == std::vector<uint32_t>({1, 2, 4}),
          "transform uses the first m recovery blocks");
    std::map<size_t, std::vector<uint8_t>> rebuilt;
    std::vector<size_t> write_order;
    for (size_t off = 0; off < bs; off += chunk) {
        codec.reconstruct_streaming_chunk(
            missing, present, prec, t, off, chunk,
            [&](size_t idx, size_t o, size_t n) {
                const std::vector<uint8_t> &b = idx < k ? data[idx] : rec[idx - k].second;
                return std::vector<uint8_t>(b.begin() + o, b.begin() + o + n);
            },
            [&](size_t idx, std::vector<uint8_t> bytes) {
                write_order.push_back(idx);
                rebuilt[idx].insert(rebuilt[idx].end(), bytes.begin(), bytes.end());
            });
    }
    for (size_t idx : missing)
        CHECK(rebuilt[idx] == data[idx], "block %zu rebuilt", idx);
    CHECK(write_order.size() == 6 && write_order[0] == 40 && write_order[1] == 3 &&
              write_order[2] == 17,
          "results written in missing_indices order");
    CHECK(throws_with([&] { codec.compute_reconstruction_transform({}, present, prec, exps); },
                      "No missing blocks to reconstruct"),
          "no missing blocks");
    CHECK(throws_with([&] { codec.compute_reconstruction_transform(missing, present, {k}, exps); },
                      "Need 3 recovery blocks, have 1"),
          "insufficient recovery");
    CHECK(throws_with(
              [&] {
                  codec.compute_reconstruction_transform(missing, present, {k + 1, k + 1, k + 2},
                                                         exps);
              },
              "Singular matrix"),
          "singular matrix");
}

int main(int argc, char **argv)
{
    tables();
    const std::string what = argc > 1 ? argv[1] : "registry";
    try {
        if (what == "registry") {
            test_registry();
            test_streaming_encoder();
        } else {
            test_each_simd_strategy();
            test_codec();
        }
    } catch (const std::exception &e) {
        fprintf(stderr, "exception: %s\n", e.what());
        ++failures;
    }
    printf("%s: %s\n", what.c_str(), failures ? "FAILED" : "ok");
    return failures ? 1 : 0;
}
