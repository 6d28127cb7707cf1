// probe_int_peak.cu -- measures the 32-bit logic-op issue rate (LOP3) of the
// device: the denominator of the integer roofline of the GF(2^16) kernels
// (2 LOP3 per symbol multiply-accumulate in the bit-sliced form).  Built as a
// separate library used only by bench.py.
#include <cuda_runtime.h>
#include <stdint.h>


#define LOP3(d, a, b, c, imm) asm volatile("lop3.b32 %0, %1, %2, %3, " #imm ";" : "=r"(d) : "r"(a), "r"(b), "r"(c))

__global__ void lop3_loop(uint32_t *out, int iters, uint32_t seed)
{
    uint32_t a = seed ^ (blockIdx.x * blockDim.x + threadIdx.x);
    uint32_t b = a * 3u, c = a * 5u, d = a * 7u, e = a * 11u, f = a * 13u, g = a * 17u,
             h = a * 19u;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            LOP3(a, a, b, c, 0x96);
            LOP3(b, b, c, d, 0xE8);
            LOP3(c, c, d, e, 0x96);
            LOP3(d, d, e, f, 0xE8);
            LOP3(e, e, f, g, 0x96);
            LOP3(f, f, g, h, 0xE8);
            LOP3(g, g, h, a, 0x96);
            LOP3(h, h, a, b, 0xE8);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = a ^ b ^ c ^ d ^ e ^ f ^ g ^ h;
}

extern "C" int p2g_probe_lop3(int device, double *ops_per_s, double *ms_out, int *sms)
{
    if (cudaSetDevice(device) != cudaSuccess)
        return -1;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return -1;
    const int threads = 256, blocks = prop.multiProcessorCount * 8, iters = 4096;
    uint32_t *out = nullptr;
    if (cudaMalloc(&out, sizeof(uint32_t) * threads * blocks) != cudaSuccess)
        return -2;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    lop3_loop<<<blocks, threads>>>(out, iters, 1u);  // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        lop3_loop<<<blocks, threads>>>(out, iters, rep + 2u);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best)
            best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess)
        return -3;
    double ops = 32.0 * iters * (double)threads * blocks;
    *ops_per_s = ops / (best * 1e-3);
    *ms_out = best;
    *sms = prop.multiProcessorCount;
    return 0;
}

// The binary tensor-core rate (mma.sync m16n8k256 b1 with AND + POPC): the
// GF(2) bit-matrix formulation of the multiply-accumulate computes every
// output bit as the parity of an AND-popcount over 16 x (inputs) bits, 256
// bit-MACs per symbol multiply-accumulate.  Register operands only; each warp
// runs 8 independent accumulator chains.
__global__ void bmma_loop(uint32_t *out, int iters, uint32_t seed)
{
    const uint32_t a0 = seed ^ (blockIdx.x * blockDim.x + threadIdx.x), a1 = a0 * 3u,
                   a2 = a0 * 5u, a3 = a0 * 7u, b0 = a0 * 11u, b1 = a0 * 13u;
    int acc[8][4] = {};
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < 8; ++c)
            asm volatile("mma.sync.aligned.m16n8k256.row.col.s32.b1.b1.s32.and.popc "
                         "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                         : "+r"(acc[c][0]), "+r"(acc[c][1]), "+r"(acc[c][2]), "+r"(acc[c][3])
                         : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    }
    uint32_t x = 0;
    for (int c = 0; c < 8; ++c)
        x ^= static_cast<uint32_t>(acc[c][0] ^ acc[c][1] ^ acc[c][2] ^ acc[c][3]);
    out[blockIdx.x * blockDim.x + threadIdx.x] = x;
}

// bit-MACs per second of binary MMA (16 x 8 x 256 per instruction)
extern "C" int p2g_probe_bmma(int device, double *bitmacs_per_s, double *ms_out)
{
    if (cudaSetDevice(device) != cudaSuccess)
        return -1;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return -1;
    const int threads = 256, blocks = sms * 4, iters = 4096;
    uint32_t *out = nullptr;
    if (cudaMalloc(&out, sizeof(uint32_t) * threads * blocks) != cudaSuccess)
        return -2;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    bmma_loop<<<blocks, threads>>>(out, iters, 1u);  // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0);
        bmma_loop<<<blocks, threads>>>(out, iters, rep + 2u);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best)
            best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess)
        return -3;
    const double mmas = static_cast<double>(blocks) * (threads / 32) * iters * 8;
    *bitmacs_per_s = mmas * 16 * 8 * 256 / (best * 1e-3);
    *ms_out = best;
    return 0;
}

// Tensor memory as a second lookup-table store: the table lookups of the
// multiply-accumulate read one table row for all 32 lanes of a warp (the row
// index comes from the coefficient), which is what tcgen05.ld.32x32b.x1 reads
// from a TMEM column.  This measures TMEM column loads alone, ldmatrix.x4
// row-chunk loads from shared memory alone, and both interleaved, in bytes per
// SM-clock.  One 512-thread CTA per SM (150 KB dynamic shared memory); warp 0
// allocates all 512 columns and frees them before the CTA exits; every loop is
// of fixed length.
__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

template <int MODE>  // 0 TMEM, 1 shared memory, 2 both
__global__ void __launch_bounds__(512, 1) tmem_loop(uint32_t *out, int iters)
{
    extern __shared__ __align__(16) uint8_t sm[];
    __shared__ uint32_t tbase;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t *tab = reinterpret_cast<uint32_t *>(sm);  // 512 rows x 128 B
    for (int i = threadIdx.x; i < 512 * 32; i += blockDim.x)
        tab[i] = i * 2654435761u;
    if (MODE != 1 && warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_addr(&tbase)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tb = tbase + (static_cast<uint32_t>(32 * (warp & 3)) << 16);  // this warp's lane quarter
    if (MODE != 1) {
        for (int c = warp >> 2; c < 512; c += 4) {
            const uint32_t v = c * 7u + lane;
            asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(tb + c), "r"(v));
        }
        asm volatile("tcgen05.wait::st.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    uint32_t acc = 0;
    // lanes 8m..8m+7 give the eight 16-byte chunks of one 128-byte row
    const uint32_t row_addr = smem_addr(tab) + (lane & 7) * 16 + (lane >> 3) * 128 * 97;
    for (int it = 0; it < iters; ++it) {
        uint32_t t[32];
        if (MODE != 1) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const uint32_t col = static_cast<uint32_t>(it * 37 + j * 29) & 511u;
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(t[j]) : "r"(tb + col));
            }
        }
        if (MODE != 0) {
            uint32_t q[8][4];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint32_t off = (static_cast<uint32_t>(it * 5 + j * 3) & 63u) * 128;
                asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                             : "=r"(q[j][0]), "=r"(q[j][1]), "=r"(q[j][2]), "=r"(q[j][3])
                             : "r"(row_addr + off));
            }
#pragma unroll
            for (int j = 0; j < 8; ++j)
                acc ^= q[j][0] ^ q[j][1] ^ q[j][2] ^ q[j][3];
        }
        if (MODE != 1) {
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int j = 0; j < 32; ++j)
                asm volatile("" : "+r"(t[j]));  // the values are valid after the wait
#pragma unroll
            for (int j = 0; j < 32; ++j)
                acc ^= t[j];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (MODE != 1 && warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tbase));
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

template <int MODE>
static float time_tmem(uint32_t *out, int sms, int iters)
{
    const size_t smem = 150 * 1024;
    if (cudaFuncSetAttribute(tmem_loop<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) != cudaSuccess)
        return -1.f;
    tmem_loop<MODE><<<sms, 512, smem>>>(out, iters);
    if (cudaDeviceSynchronize() != cudaSuccess)
        return -1.f;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0);
        tmem_loop<MODE><<<sms, 512, smem>>>(out, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best)
            best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

// bytes per SM-clock (at clock_hz): out[0] TMEM alone, out[1] shared memory
// alone, out[2] / out[3] TMEM / shared memory when interleaved
extern "C" int p2g_probe_tmem(int device, double clock_hz, double out[4])
{
    if (cudaSetDevice(device) != cudaSuccess)
        return -1;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return -1;
    const int iters = 2048;
    uint32_t *buf = nullptr;
    if (cudaMalloc(&buf, sizeof(uint32_t) * 512 * sms) != cudaSuccess)
        return -2;
    const float t0 = time_tmem<0>(buf, sms, iters), t1 = time_tmem<1>(buf, sms, iters),
                t2 = time_tmem<2>(buf, sms, iters);
    cudaFree(buf);
    if (t0 < 0 || t1 < 0 || t2 < 0)
        return -3;
    const double per = 16.0 * iters / clock_hz;  // warps per CTA x iterations / clock
    out[0] = per * 32 * 128 / (t0 * 1e-3);
    out[1] = per * 8 * 512 / (t1 * 1e-3);
    out[2] = per * 32 * 128 / (t2 * 1e-3);
    out[3] = per * 8 * 512 / (t2 * 1e-3);
    return 0;
}
