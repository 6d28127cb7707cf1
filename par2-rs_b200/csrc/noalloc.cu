// noalloc.cu -- recovery-slice creation that allocates no memory.
//
// Some callers cannot allocate device memory at the moment they want to
// encode: a service that reserved its whole device-memory budget up front and
// admits work against it, a latency-critical path where cudaMalloc's implicit
// device synchronisation is not acceptable, or a host that forbids allocation
// after start-up.  p2g_encode_noalloc serves them.  Its scratch is one
// file-scope __device__ array of fixed size (P2G_NOALLOC_SCRATCH_BYTES) that
// every GPU loading this library holds until the process exits; inputs and
// outputs are the caller's device buffers.  It calls no cudaMalloc / cudaFree
// and no allocating library routine.
//
// The array is shared by every call on a device and keeps the previous call's
// contents.  Every region a call reads is written earlier in the same call
// (pointer tables, coefficients, records, bit planes), so nothing has to start
// at zero.  Calls whose work overlaps on the GPU (different streams, or host
// threads sharing a device) race on the array; callers must serialise them.
#include <mutex>
#include <vector>

#include "common.cuh"
#include "muladd.cuh"

namespace p2g {

static __device__ __align__(256) uint8_t g_noalloc_scratch[P2G_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;

struct DeviceSetup {
    std::once_flag once;
    int rc = P2G_OK;
    uint8_t *scratch = nullptr;  // device address of g_noalloc_scratch
    int sm_count = 0;
};

DeviceSetup g_setup[kMaxDevices];

// Once per device, with that device current: the device address of the
// scratch array (in host code the symbol is only a stand-in, never a device
// address) and the SM count.
void setup_device(int dev)
{
    DeviceSetup &s = g_setup[dev];
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        set_error("p2g_encode_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        s.rc = P2G_ECUDA;
        return;
    }
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        set_error("p2g_encode_noalloc: cudaDeviceGetAttribute failed: %s", cudaGetErrorString(e));
        s.rc = P2G_ECUDA;
        return;
    }
    s.scratch = static_cast<uint8_t *>(ptr);
    s.sm_count = sms;
}

size_t align256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }

// PAR2 constants and their powers c_i^e on the host (par2_rs.rs:64-76, :707-719),
// as a [r][k] matrix (coefficients[dst][src]).
void coefficient_matrix(size_t k, const uint32_t *exps, size_t r, std::vector<uint16_t> &out)
{
    static uint16_t lg[65536], ex[65535];
    static std::once_flag tables;
    std::call_once(tables, [] {
        uint32_t b = 1;
        for (uint32_t l = 0; l < 65535; ++l) {
            ex[l] = static_cast<uint16_t>(b);
            lg[b] = static_cast<uint16_t>(l);
            b <<= 1;
            if (b & 0x10000u)
                b ^= 0x1100Bu;
        }
    });
    std::vector<uint16_t> c(k);
    size_t have = 0;
    for (uint64_t n = 1; have < k; ++n)
        if (n % 3 && n % 5 && n % 17 && n % 257)
            c[have++] = ex[n % 65535];
    out.resize(k * r);
    for (size_t e = 0; e < r; ++e)
        for (size_t i = 0; i < k; ++i)
            out[e * k + i] =
                exps[e] == 0
                    ? 1
                    : ex[static_cast<uint32_t>((static_cast<uint64_t>(lg[c[i]]) * exps[e]) % 65535u)];
}

}  // namespace

}  // namespace p2g

using namespace p2g;

extern "C" int p2g_encode_noalloc(void *cuda_stream, const uint8_t *const *src, size_t k,
                                  size_t slice_bytes, const uint32_t *exps, size_t r,
                                  uint8_t *const *out)
{
    clear_error();
    if ((k && !src) || (r && (!out || !exps))) {
        set_error("p2g_encode_noalloc: null argument");
        return P2G_EINVAL;
    }
    if (slice_bytes == 0 || slice_bytes % 2) {
        set_error("p2g_encode_noalloc: slice size %zu must be even and non-zero", slice_bytes);
        return P2G_EINVAL;
    }
    if (k > 65535 || r > 65535) {
        set_error("p2g_encode_noalloc: %zu inputs / %zu outputs exceed 65535", k, r);
        return P2G_ERANGE;
    }
    for (size_t i = 0; i < k; ++i)
        if (reinterpret_cast<uintptr_t>(src[i]) & 15) {
            set_error("p2g_encode_noalloc: input slice %zu is not 16-byte aligned", i);
            return P2G_EINVAL;
        }
    for (size_t e = 0; e < r; ++e)
        if (reinterpret_cast<uintptr_t>(out[e]) & 15) {
            set_error("p2g_encode_noalloc: output slice %zu is not 16-byte aligned", e);
            return P2G_EINVAL;
        }
    // scratch layout: [src ptrs][dst ptrs][coefficients r x k][records][planes]
    const size_t off_dst = align256(k * sizeof(void *));
    const size_t off_coef = off_dst + align256(r * sizeof(void *));
    const size_t off_rec = off_coef + align256(k * r * 2);
    const size_t off_pl = off_rec + align256(record_bytes(k, static_cast<int>(r)));
    const size_t need = off_pl + planes_bytes_fixed(static_cast<int>(k), slice_bytes);
    if (need > P2G_NOALLOC_SCRATCH_BYTES) {
        set_error("p2g_encode_noalloc: k=%zu, r=%zu, slice=%zu bytes needs %zu bytes of scratch; "
                  "the static maximum is %zu bytes",
                  k, r, slice_bytes, need, static_cast<size_t>(P2G_NOALLOC_SCRATCH_BYTES));
        return P2G_ERANGE;
    }
    if (r == 0)
        return P2G_OK;
    int dev = 0;
    P2G_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("p2g_encode_noalloc: device %d out of range", dev);
        return P2G_ERANGE;
    }
    DeviceSetup &s = g_setup[dev];
    std::call_once(s.once, setup_device, dev);
    if (s.rc != P2G_OK) {
        set_error("p2g_encode_noalloc: set-up of device %d failed", dev);
        return s.rc;
    }
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    uint8_t *base = s.scratch;
    std::vector<uint16_t> coef;
    coefficient_matrix(k, exps, r, coef);
    // The caller's pointer tables may be pinned, and a copy from pinned memory
    // runs after the call returns; copies of them in pageable memory (staged
    // by the driver before cudaMemcpyAsync returns) leave the caller free to
    // reuse its tables as soon as the call is back.
    std::vector<const uint8_t *> src_tab(src, src + k);
    std::vector<uint8_t *> out_tab(out, out + r);
    P2G_CUDA(cudaMemcpyAsync(base, src_tab.data(), k * sizeof(void *), cudaMemcpyHostToDevice,
                             stream));
    P2G_CUDA(cudaMemcpyAsync(base + off_dst, out_tab.data(), r * sizeof(void *),
                             cudaMemcpyHostToDevice, stream));
    P2G_CUDA(cudaMemcpyAsync(base + off_coef, coef.data(), k * r * 2, cudaMemcpyHostToDevice,
                             stream));
    uint32_t *recs = reinterpret_cast<uint32_t *>(base + off_rec);
    P2G_TRY(records_matrix_fixed(stream, reinterpret_cast<const uint16_t *>(base + off_coef),
                                 static_cast<int>(k), static_cast<int>(r), recs));
    P2G_TRY(muladd_run_fixed(stream, s.sm_count, reinterpret_cast<const uint8_t *const *>(base),
                             static_cast<int>(k), reinterpret_cast<uint8_t *const *>(base + off_dst),
                             static_cast<int>(r), slice_bytes, recs,
                             reinterpret_cast<uint32_t *>(base + off_pl)));
    return P2G_OK;
}
