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
