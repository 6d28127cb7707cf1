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
