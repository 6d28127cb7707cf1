// invert.cu -- exact GF(2^16) Gauss-Jordan inversion of the erasure matrix.
//
// Replaces Par2ReedSolomon::compute_reconstruction_transform
// (par2-rs par2_rs.rs:319-422) and, together with the muladd kernels, the
// elimination replay of reconstruct_streaming_chunk (:618-655): instead of
// recording row operations and replaying them on every chunk, the inverse
// A^-1 itself is formed once on the device and applied as one more
// multiply-accumulate pass.  A is invertible exactly when the reference's
// elimination finds a pivot in every column, so "Singular matrix" is reported
// for the same inputs.
//
// The augmented matrix [A | I] (m x 2m u16, row-major, row stride W) lives in
// device memory.  Each column step is two launches: gj_pivot (one CTA: find a
// non-zero pivot at or below the diagonal -- swapping rows only when the
// diagonal entry is zero, as the reference does -- and scale the pivot row by
// the pivot's inverse) and gj_eliminate (one CTA per row: row ^= f * pivot
// row).  A status word turns the remaining steps into no-ops once a column has
// no pivot.
#include "invert.cuh"

namespace p2g {

// a * b with the log / antilog tables (galois/core.rs:175-189)
__device__ __forceinline__ uint32_t gmul(uint32_t a, uint32_t b, const uint16_t *__restrict__ glog,
                                         const uint16_t *__restrict__ gexp)
{
    if (a == 0 || b == 0)
        return 0;
    uint32_t l = glog[a] + glog[b];
    if (l >= 65535u)
        l -= 65535u;
    return gexp[l];
}

__global__ void gj_build_par2(uint16_t *__restrict__ M, int m, int W,
                              const uint16_t *__restrict__ cmiss, const uint32_t *__restrict__ exps,
                              const uint16_t *__restrict__ glog, const uint16_t *__restrict__ gexp)
{
    int row = blockIdx.y;
    for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < 2 * m;
         col += gridDim.x * blockDim.x) {
        uint32_t v;
        if (col < m) {
            uint32_t c = cmiss[col], e = exps[row];
            if (c == 0)
                v = e == 0 ? 1u : 0u;
            else if (e == 0)
                v = 1u;
            else
                v = gexp[static_cast<uint32_t>((static_cast<uint64_t>(glog[c]) * e) % 65535u)];
        } else {
            v = (col - m == row) ? 1u : 0u;
        }
        M[static_cast<size_t>(row) * W + col] = static_cast<uint16_t>(v);
    }
}

__global__ void gj_build_from(uint16_t *__restrict__ M, int m, int W, const uint16_t *__restrict__ A)
{
    int row = blockIdx.y;
    for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < 2 * m;
         col += gridDim.x * blockDim.x)
        M[static_cast<size_t>(row) * W + col] =
            col < m ? A[static_cast<size_t>(row) * m + col] : static_cast<uint16_t>(col - m == row);
}

__global__ void gj_pivot(uint16_t *__restrict__ M, int m, int W, int k,
                         const uint16_t *__restrict__ glog, const uint16_t *__restrict__ gexp,
                         int *__restrict__ status, uint16_t *__restrict__ pivots)
{
    __shared__ int found;
    if (*status != 0)
        return;
    uint16_t *rowk = M + static_cast<size_t>(k) * W;
    if (threadIdx.x == 0)
        found = rowk[k] != 0 ? k : m;
    __syncthreads();
    if (found == m) {
        // first row below k with a non-zero entry in column k (par2_rs.rs:361-370)
        for (int r = k + 1 + threadIdx.x; r < m; r += blockDim.x)
            if (M[static_cast<size_t>(r) * W + k] != 0)
                atomicMin(&found, r);
        __syncthreads();
        if (found == m) {
            if (threadIdx.x == 0)
                *status = 1;  // singular
            return;
        }
        uint16_t *rowr = M + static_cast<size_t>(found) * W;
        for (int j = threadIdx.x; j < 2 * m; j += blockDim.x) {
            uint16_t t = rowk[j];
            rowk[j] = rowr[j];
            rowr[j] = t;
        }
        __syncthreads();
    }
    const uint32_t p = rowk[k];
    __syncthreads();
    if (threadIdx.x == 0)
        pivots[k] = static_cast<uint16_t>(p);
    // p^-1 = 2^(65535 - log p)
    const uint32_t lp = glog[p];
    const uint32_t pinv = gexp[lp == 0 ? 0 : 65535u - lp];
    for (int j = k + threadIdx.x; j < 2 * m; j += blockDim.x)
        rowk[j] = static_cast<uint16_t>(gmul(rowk[j], pinv, glog, gexp));
}

__global__ void gj_eliminate(uint16_t *__restrict__ M, int m, int W, int k,
                             const uint16_t *__restrict__ glog, const uint16_t *__restrict__ gexp,
                             const int *__restrict__ status)
{
    const int r = blockIdx.x;
    if (*status != 0 || r == k)
        return;
    __shared__ uint32_t f;
    uint16_t *row = M + static_cast<size_t>(r) * W;
    const uint16_t *rowk = M + static_cast<size_t>(k) * W;
    if (threadIdx.x == 0)
        f = row[k];
    __syncthreads();
    const uint32_t fr = f;
    if (fr == 0)
        return;
    const uint32_t lf = glog[fr];
    for (int j = k + threadIdx.x; j < 2 * m; j += blockDim.x) {
        uint32_t x = rowk[j];
        if (x) {
            uint32_t l = glog[x] + lf;
            if (l >= 65535u)
                l -= 65535u;
            row[j] ^= gexp[l];
        }
    }
}

// Copies the right half of [I | A^-1] into a dense m x m matrix.
__global__ void gj_extract(const uint16_t *__restrict__ M, int m, int W, uint16_t *__restrict__ inv)
{
    int row = blockIdx.y;
    for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < m; col += gridDim.x * blockDim.x)
        inv[static_cast<size_t>(row) * m + col] = M[static_cast<size_t>(row) * W + m + col];
}

int gj_invert(p2g_ctx *ctx, GjWork &w, int m, const uint16_t *d_cmiss, const uint32_t *d_exps,
              const uint16_t *d_A, uint16_t *d_inv)
{
    if (m <= 0)
        return P2G_OK;
    const int W = (2 * m + 7) & ~7;
    P2G_TRY(w.M.ensure(static_cast<size_t>(m) * W * 2));
    P2G_TRY(w.status.ensure(sizeof(int) + static_cast<size_t>(m) * 2 + 16));
    uint16_t *M = w.M.as<uint16_t>();
    int *status = w.status.as<int>();
    uint16_t *pivots = reinterpret_cast<uint16_t *>(w.status.as<uint8_t>() + 16);
    P2G_CUDA(cudaMemsetAsync(status, 0, sizeof(int), ctx->stream));
    dim3 g(static_cast<unsigned>((2 * m + 255) / 256 < 64 ? (2 * m + 255) / 256 : 64),
           static_cast<unsigned>(m));
    if (d_A)
        gj_build_from<<<g, 256, 0, ctx->stream>>>(M, m, W, d_A);
    else
        gj_build_par2<<<g, 256, 0, ctx->stream>>>(M, m, W, d_cmiss, d_exps, ctx->d_log, ctx->d_exp);
    P2G_CUDA(cudaGetLastError());
    ++ctx->launches;
    for (int k = 0; k < m; ++k) {
        gj_pivot<<<1, 256, 0, ctx->stream>>>(M, m, W, k, ctx->d_log, ctx->d_exp, status, pivots);
        gj_eliminate<<<m, 128, 0, ctx->stream>>>(M, m, W, k, ctx->d_log, ctx->d_exp, status);
        ctx->launches += 2;
    }
    P2G_CUDA(cudaGetLastError());
    gj_extract<<<g, 256, 0, ctx->stream>>>(M, m, W, d_inv);
    P2G_CUDA(cudaGetLastError());
    ++ctx->launches;
    return P2G_OK;
}

int gj_status(p2g_ctx *ctx, GjWork &w, int *singular)
{
    int h = 0;
    P2G_CUDA(cudaMemcpyAsync(&h, w.status.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    P2G_CUDA(cudaStreamSynchronize(ctx->stream));
    *singular = h != 0;
    return P2G_OK;
}

}  // namespace p2g
