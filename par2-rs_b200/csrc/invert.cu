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
#include <algorithm>
#include <vector>

#include "bitslice.cuh"
#include "invert.cuh"
#include "muladd.cuh"

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

// a * b without tables: carry-less shift-and-add with reduction by
// x^16 + x^12 + x^3 + x + 1 at every step (no memory latency on the
// sequential paths of the pivot search).
__device__ __forceinline__ uint32_t gmul_alu(uint32_t a, uint32_t b)
{
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        r ^= a & (0u - ((b >> i) & 1u));
        a = (a << 1) ^ ((a & 0x8000u) ? 0x1100Bu : 0u);
    }
    return r & 0xFFFFu;
}

__device__ __forceinline__ uint32_t ginv(uint32_t p, const uint16_t *__restrict__ glog,
                                         const uint16_t *__restrict__ gexp)
{
    // p^-1 = 2^(65535 - log p)
    const uint32_t lp = glog[p];
    return gexp[lp == 0 ? 0 : 65535u - lp];
}

constexpr int kSmallM = 96;   // matrices up to this size: one CTA, all in shared memory
constexpr int kPanel = 64;    // panel width of the blocked elimination
constexpr int kGjThreads = 256;

constexpr uint32_t kLogZero = 0xFFFFu;  // marks log(0)

__device__ __forceinline__ uint32_t glog_or_zero(uint32_t v, const uint16_t *__restrict__ glog)
{
    return v ? __ldg(glog + v) : kLogZero;
}

// product from logs (either kLogZero: 0) with the antilog table in shared memory
__device__ __forceinline__ uint32_t gmul_logs_s(uint32_t la, uint32_t lb, const uint16_t *sexp)
{
    if (la == kLogZero || lb == kLogZero)
        return 0;
    uint32_t l = la + lb;
    if (l >= 65535u)
        l -= 65535u;
    return sexp[l];
}

constexpr size_t kExpSmem = 65535 * sizeof(uint16_t);  // antilog table in shared memory

// Copies the antilog table into shared memory (all threads; ends with a barrier).
__device__ void load_exp_table(uint16_t *sexp, const uint16_t *__restrict__ gexp)
{
    const uint32_t *g = reinterpret_cast<const uint32_t *>(gexp);
    uint32_t *d = reinterpret_cast<uint32_t *>(sexp);
    for (int i = threadIdx.x; i < 65535 / 2; i += blockDim.x)
        d[i] = __ldg(g + i);
    if (threadIdx.x == 0)
        sexp[65534] = gexp[65534];
    __syncthreads();
}

// Gauss-Jordan on [A | I] (n x 2n, row stride ld) in shared memory by one
// CTA, with the reference's pivot rule: rows are swapped only when the
// diagonal entry is zero (first non-zero row below).  Returns false (for every
// thread) when A is singular.  Each elimination step takes the logs of the
// pivot row (lrow, 2n entries) and of the row factors (fcol) once, so every
// product of the row updates is one lookup in the shared antilog table sexp.
__device__ bool cta_gauss_jordan(uint16_t *S, int n, int ld, uint32_t *fcol, uint32_t *lrow,
                                 const uint16_t *sexp, const uint16_t *__restrict__ glog,
                                 const uint16_t *__restrict__ gexp)
{
    __shared__ int piv;
    const int tid = threadIdx.x, nt = blockDim.x, w2 = 2 * n;
    for (int k = 0; k < n; ++k) {
        if (tid == 0)
            piv = n;
        __syncthreads();
        // first row r >= k with a non-zero entry in column k
        for (int r0 = k; r0 < n; r0 += nt) {
            const int r = r0 + tid;
            const bool nz = r < n && S[r * ld + k] != 0;
            const unsigned ball = __ballot_sync(0xffffffffu, nz);
            if (ball && (tid & 31) == 0)
                atomicMin(&piv, r0 + (tid & ~31) + __ffs(ball) - 1);
            __syncthreads();
            if (piv < n)
                break;
        }
        if (tid == 0 && piv == n)
            piv = -1;
        __syncthreads();
        const int p = piv;
        if (p < 0)
            return false;
        if (p != k) {
            for (int j = tid; j < w2; j += nt) {
                uint16_t t = S[k * ld + j];
                S[k * ld + j] = S[p * ld + j];
                S[p * ld + j] = t;
            }
            __syncthreads();
        }
        // scale the pivot row by 1/pivot and keep the logs of its entries
        const uint32_t pinv = ginv(S[k * ld + k], glog, gexp);
        __syncthreads();
        for (int j = tid; j < w2; j += nt) {
            const uint32_t v = gmul_alu(S[k * ld + j], pinv);
            S[k * ld + j] = static_cast<uint16_t>(v);
            lrow[j] = glog_or_zero(v, glog);
        }
        for (int r = tid; r < n; r += nt)
            fcol[r] = r == k ? kLogZero : glog_or_zero(S[r * ld + k], glog);
        __syncthreads();
        // S[r][j] ^= f_r * S[k][j] over the n x 2n block, no division per entry
        int r = tid / w2, j = tid - r * w2;
        const int dr = nt / w2, dj = nt - dr * w2;
        for (; r < n;) {
            const uint32_t lf = fcol[r];
            if (lf != kLogZero)
                S[r * ld + j] ^= static_cast<uint16_t>(gmul_logs_s(lf, lrow[j], sexp));
            r += dr;
            j += dj;
            if (j >= w2) {
                j -= w2;
                ++r;
            }
        }
        __syncthreads();
    }
    return true;
}

// Whole inversion of a small matrix (m <= kSmallM) by one CTA.
__global__ void __launch_bounds__(kGjThreads)
    gj_small(const uint16_t *__restrict__ M, int m, int W, uint16_t *__restrict__ inv,
             int *__restrict__ status, const uint16_t *__restrict__ glog,
             const uint16_t *__restrict__ gexp)
{
    extern __shared__ __align__(16) uint16_t dyn[];  // antilog table, then S (m x 2m)
    uint16_t *sexp = dyn, *S = dyn + 65536;
    __shared__ uint32_t fcol[kSmallM];
    __shared__ uint32_t lrow[2 * kSmallM];
    load_exp_table(sexp, gexp);
    for (int idx = threadIdx.x; idx < m * 2 * m; idx += blockDim.x) {
        const int r = idx / (2 * m), j = idx - r * 2 * m;
        S[idx] = M[static_cast<size_t>(r) * W + j];
    }
    __syncthreads();
    if (!cta_gauss_jordan(S, m, 2 * m, fcol, lrow, sexp, glog, gexp)) {
        if (threadIdx.x == 0)
            *status = 1;
        return;
    }
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
        const int r = idx / m, j = idx - r * m;
        inv[idx] = S[r * 2 * m + m + j];
    }
}

// Scratch of the blocked elimination (device).
struct PanelBufs {
    uint16_t *akk_inv;  // kPanel x kPanel inverse of the pivot block
    int *used;          // m: row already a pivot row
    int *kall;          // m: pivot row of each column
    int *orow;          // m: the rows that are not this panel's pivots
    const uint8_t **kptr;  // kPanel row pointers of the pivot rows
    uint8_t **optr;        // m row pointers of the other rows
};

// One panel [c0, c0+b) of the blocked Gauss-Jordan, by one CTA: choose b
// pivot rows among the rows not yet used (incremental row reduction,
// smallest row index first), invert their b x b block A_KK, and list
// the pivot rows (K) and the other rows (O) for the two multiply-accumulate
// passes that follow:  X = A_KK^-1 M[K,:];  M[O,:] ^= M[O, panel] X;  M[K,:] = X.
// On a singular matrix (or after an earlier failure) it sets *status and
// still writes valid row lists so the passes stay in bounds.
__global__ void __launch_bounds__(kGjThreads)
    gj_panel(uint16_t *__restrict__ M, int m, int W, int c0, int b, PanelBufs pb,
             int *__restrict__ status, const uint16_t *__restrict__ glog,
             const uint16_t *__restrict__ gexp)
{
    extern __shared__ __align__(16) uint16_t sexp[];  // antilog table
    __shared__ uint16_t S[kPanel * 2 * kPanel];
    __shared__ uint32_t fcol[kPanel];
    __shared__ uint32_t lrow[2 * kPanel];
    __shared__ int ksel[kPanel];
    __shared__ int failed, fast;
    __shared__ int scan[kGjThreads];
    // used[] as a bitmap (m <= 65535 rows)
    __shared__ uint32_t used_bits[65536 / 32];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int nwords = (m + 31) / 32;
    if (tid == 0) {
        failed = *status != 0;
        fast = 0;
    }
    for (int w = tid; w < nwords; w += nt) {
        uint32_t bits = 0;
        for (int i = 0; i < 32 && w * 32 + i < m; ++i)
            bits |= pb.used[w * 32 + i] ? (1u << i) : 0u;
        used_bits[w] = bits;
    }
    load_exp_table(sexp, gexp);
    // Fast path: the first b unused rows as the pivot rows.  Any rows whose
    // b x b block is invertible give the same inverse; for an invertible A
    // this block is singular only by accident (then the search below runs).
    if (!failed) {
        if (tid == 0) {
            int n = 0;
            for (int w = 0; w < nwords && n < b; ++w) {
                uint32_t free_bits = ~used_bits[w];
                while (free_bits && n < b) {
                    const int r = w * 32 + __ffs(free_bits) - 1;
                    free_bits &= free_bits - 1;
                    if (r < m)
                        ksel[n++] = r;
                }
            }
            if (n < b)
                failed = 1;
        }
        __syncthreads();
        if (!failed) {
            for (int idx = tid; idx < b * 2 * b; idx += nt) {
                const int r = idx / (2 * b), j = idx - r * 2 * b;
                S[r * 2 * kPanel + j] = j < b ? M[static_cast<size_t>(ksel[r]) * W + c0 + j]
                                              : static_cast<uint16_t>(j - b == r);
            }
            __syncthreads();
            if (cta_gauss_jordan(S, b, 2 * kPanel, fcol, lrow, sexp, glog, gexp)) {
                for (int j = tid; j < b; j += nt)
                    pb.used[ksel[j]] = 1;
                if (tid == 0)
                    fast = 1;
            }
            __syncthreads();
        }
    }
    if (!failed && !fast) {
        // Incremental row reduction: candidate rows (unused, ascending) are
        // reduced against the pivot rows found so far (kept in reduced echelon
        // form, pivot entries 1); a candidate with a non-zero remainder
        // becomes the pivot of its first non-zero column.  Stops after b
        // pivots, so only about b rows are touched per panel.
        uint16_t *piv_rows = S;           // b x kPanel (reuses the A_KK buffer)
        __shared__ uint16_t vec[kPanel];
        __shared__ uint16_t coef[kPanel];                // f_q or g_q of the current step
        __shared__ uint16_t part[kGjThreads / kPanel][kPanel];
        __shared__ int piv_col[kPanel];
        __shared__ int nk, cand, lead;
        constexpr int QG = kGjThreads / kPanel;          // pivot groups summed in parallel
        const int col = tid % kPanel, qg = tid / kPanel;
        if (tid == 0) {
            nk = 0;
            cand = -1;
        }
        __syncthreads();
        while (true) {
            if (tid == 0) {
                // next row after cand whose used bit is clear
                int r = cand + 1, found = m;
                for (int w = r >> 5; w < nwords; ++w) {
                    uint32_t free_bits = ~used_bits[w];
                    if (w == (r >> 5))
                        free_bits &= ~0u << (r & 31);
                    if (free_bits) {
                        found = min(m, w * 32 + __ffs(free_bits) - 1);
                        break;
                    }
                }
                cand = found;
            }
            __syncthreads();
            const int r = cand;
            if (r >= m || nk >= b)
                break;
            const int n0 = nk;
            if (tid < b)
                vec[tid] = M[static_cast<size_t>(r) * W + c0 + tid];
            __syncthreads();
            // The pivot rows are reduced (zero in every other pivot column), so
            // the coefficients of all reductions are the candidate's own
            // entries in the pivot columns: one dot product, no chain.
            if (tid < n0)
                coef[tid] = vec[piv_col[tid]];
            __syncthreads();
            {
                uint32_t acc = 0;
                if (col < b)
                    for (int q = qg; q < n0; q += QG)
                        acc ^= gmul_alu(coef[q], piv_rows[q * kPanel + col]);
                part[qg][col] = static_cast<uint16_t>(acc);
            }
            __syncthreads();
            if (tid < b) {
                uint32_t x = vec[tid];
#pragma unroll
                for (int g2 = 0; g2 < QG; ++g2)
                    x ^= part[g2][tid];
                vec[tid] = static_cast<uint16_t>(x);
            }
            __syncthreads();
            if (tid < 64) {
                const unsigned ball = __ballot_sync(0xffffffffu, tid < b && vec[tid] != 0);
                if ((tid & 31) == 0)
                    part[0][tid >> 5] = static_cast<uint16_t>(ball ? (tid + __ffs(ball) - 1) : 0xFFFF);
            }
            __syncthreads();
            if (tid == 0) {
                const int a0 = part[0][0], a1 = part[0][1];
                lead = a0 != 0xFFFF ? a0 : (a1 != 0xFFFF ? a1 : b);
            }
            __syncthreads();
            const int j = lead;
            if (j < b) {
                const uint32_t inv = ginv(vec[j], glog, gexp);
                if (tid < n0)
                    coef[tid] = piv_rows[tid * kPanel + j];
                __syncthreads();
                if (tid < b)
                    vec[tid] = static_cast<uint16_t>(gmul_alu(vec[tid], inv));
                __syncthreads();
                // keep the earlier pivot rows reduced in the new pivot column
                for (int idx = tid; idx < n0 * kPanel; idx += nt) {
                    const int q = idx / kPanel, c = idx - q * kPanel;
                    if (c < b && coef[q])
                        piv_rows[q * kPanel + c] ^= static_cast<uint16_t>(gmul_alu(coef[q], vec[c]));
                }
                if (tid < b)
                    piv_rows[n0 * kPanel + tid] = vec[tid];
                if (tid == 0) {
                    piv_col[n0] = j;
                    ksel[n0] = r;
                    pb.used[r] = 1;
                    used_bits[r >> 5] |= 1u << (r & 31);
                    nk = n0 + 1;
                }
            }
            __syncthreads();
        }
        if (nk < b) {
            if (tid == 0)
                failed = 1;
            __syncthreads();
        }
    }
    if (failed) {
        // valid but meaningless row lists
        for (int j = tid; j < b; j += nt)
            ksel[j] = j;
        if (tid == 0)
            *status = 1;
        __syncthreads();
    } else {
        if (!fast) {
            // A_KK^-1 from the current values of the pivot rows' panel columns
            for (int idx = tid; idx < b * 2 * b; idx += nt) {
                const int r = idx / (2 * b), j = idx - r * 2 * b;
                S[r * 2 * kPanel + j] =
                    j < b ? M[static_cast<size_t>(ksel[r]) * W + c0 + j]
                          : static_cast<uint16_t>(j - b == r);
            }
            __syncthreads();
            if (!cta_gauss_jordan(S, b, 2 * kPanel, fcol, lrow, sexp, glog, gexp)) {
                // cannot happen when every column found a pivot; guarded anyway
                if (tid == 0)
                    *status = 1;
            }
        }
        for (int idx = tid; idx < b * b; idx += nt) {
            const int r = idx / b, j = idx - r * b;
            pb.akk_inv[idx] = S[r * 2 * kPanel + b + j];
        }
    }
    for (int j = tid; j < b; j += nt) {
        pb.kptr[j] = reinterpret_cast<const uint8_t *>(M + static_cast<size_t>(ksel[j]) * W);
        pb.kall[c0 + j] = ksel[j];
    }
    // O = rows not in K, ascending: block-wide exclusive scan of the flags
    const int per = (m + nt - 1) / nt, r0 = tid * per, r1 = min(m, r0 + per);
    auto in_k = [&](int r) {
        for (int j = 0; j < b; ++j)
            if (ksel[j] == r)
                return true;
        return false;
    };
    int cnt = 0;
    for (int r = r0; r < r1; ++r)
        cnt += !in_k(r);
    scan[tid] = cnt;
    __syncthreads();
    if (tid == 0) {
        int acc = 0;
        for (int t = 0; t < nt; ++t) {
            int c = scan[t];
            scan[t] = acc;
            acc += c;
        }
    }
    __syncthreads();
    int o = scan[tid];
    for (int r = r0; r < r1; ++r) {
        if (!in_k(r)) {
            pb.orow[o] = r;
            pb.optr[o] = reinterpret_cast<uint8_t *>(M + static_cast<size_t>(r) * W);
            ++o;
        }
    }
}

// Records for the row update: coefficient (i, o) = M[orow[o]][c0 + i].
__global__ void gj_records_rows(const uint16_t *__restrict__ M, int W, const int *__restrict__ orow,
                                int c0, int nin, int nout, uint32_t *__restrict__ recs)
{
    size_t gid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (gid >= static_cast<size_t>(nin) * nout)
        return;
    const int o = static_cast<int>(gid % nout), i = static_cast<int>(gid / nout);
    write_record(recs, gid, M[static_cast<size_t>(orow[o]) * W + c0 + i], nout <= kSmallOutputs);
}

// M[K_j, :] = X_j
__global__ void gj_copy_rows(const uint8_t *const *__restrict__ xptr,
                             const uint8_t *const *__restrict__ kptr, int b, size_t bytes)
{
    const int j = blockIdx.y;
    if (j >= b)
        return;
    const uint4 *x = reinterpret_cast<const uint4 *>(xptr[j]);
    uint4 *k = reinterpret_cast<uint4 *>(const_cast<uint8_t *>(kptr[j]));
    for (size_t q = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < bytes / 16;
         q += static_cast<size_t>(gridDim.x) * blockDim.x)
        k[q] = x[q];
}

// inv[c][:] = right half of row kall[c]
__global__ void gj_extract_perm(const uint16_t *__restrict__ M, int m, int W,
                                const int *__restrict__ kall, uint16_t *__restrict__ inv)
{
    const int c = blockIdx.y;
    const uint16_t *row = M + static_cast<size_t>(kall[c]) * W + m;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x)
        inv[static_cast<size_t>(c) * m + j] = row[j];
}

// ---- consecutive exponents: the inverse of a Vandermonde matrix ----------
//
// When the recovery exponents are a permutation of s, s+1, ..., s+m-1 (the m
// lowest exponents of an undamaged recovery set), A[r][j] = x_j^(s + e_r) with
// x_j the constants of the missing slices, i.e. A = V D with V[e][j] = x_j^e
// (a transposed Vandermonde matrix) and D = diag(x_j^s).  Row j of V^-1 holds
// the coefficients of the Lagrange polynomial
//     L_j(z) = Q_j(z) / Q_j(x_j),   Q_j(z) = P(z) / (z + x_j),   P(z) = prod_k (z + x_k),
// since L_j(x_k) = [j == k].  So inv[j][r] = x_j^-s coef_{e_r - s}(L_j): O(m^2)
// work in place of the elimination's O(m^3), and the same matrix (the inverse
// is unique).  A is singular exactly when two x_j are equal (Q_j(x_j) = 0),
// or when some x_j = 0 and s > 0; both are reported like a failed
// elimination.

constexpr uint16_t kNoLog = 0xFFFF;  // log of 0

// level 0 of the product tree: the factors z + x_k (leading 1 implicit)
__global__ void vdm_leaves(const uint16_t *__restrict__ x, int m, uint16_t *__restrict__ P,
                           uint16_t *__restrict__ LP, const uint16_t *__restrict__ glog)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) {
        P[k] = x[k];
        LP[k] = x[k] ? glog[x[k]] : kNoLog;
    }
}

// One level of the product tree.  Pin holds monic polynomials of degree G
// (the last one shorter), each as its G low coefficients at offset g*G;
// pairs are multiplied into Pout (degree 2G at offset q*2G).  One thread per
// output coefficient; LP/LPout are the logs of the coefficients.
__global__ void vdm_level(const uint16_t *__restrict__ Pin, const uint16_t *__restrict__ LPin,
                          uint16_t *__restrict__ Pout, uint16_t *__restrict__ LPout, int m, int G,
                          const uint16_t *__restrict__ glog, const uint16_t *__restrict__ gexp)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m)
        return;
    const int base = (t / (2 * G)) * 2 * G, u = t - base;
    const int a = min(G, m - base), b = max(0, min(G, m - base - G));
    if (b == 0) {
        Pout[t] = Pin[t];
        LPout[t] = LPin[t];
        return;
    }
    // c_u = sum_{i+j=u} A_i B_j with A_a = B_b = 1 (u < a + b)
    const uint16_t *LA = LPin + base, *LB = LPin + base + G;
    uint32_t acc = 0;
    for (int i = max(0, u - b); i <= min(u, a); ++i) {
        const int j = u - i;
        const uint32_t la = i == a ? 0u : LA[i], lb = j == b ? 0u : LB[j];
        if (la != kNoLog && lb != kNoLog) {
            uint32_t l = la + lb;
            if (l >= 65535u)
                l -= 65535u;
            acc ^= gexp[l];
        }
    }
    Pout[t] = static_cast<uint16_t>(acc);
    LPout[t] = acc ? glog[acc] : kNoLog;
}

// y * q for a fixed y given as X[i] = y * 2^i (i < 16): the XOR of the X[i]
// selected by the bits of q, summed in four independent chains.
__device__ __forceinline__ uint32_t gmul_fixed(const uint32_t X[16], uint32_t q)
{
    uint32_t r[4] = {0, 0, 0, 0};
#pragma unroll
    for (int i = 0; i < 16; ++i)
        r[i & 3] ^= X[i] & (0u - ((q >> i) & 1u));
    return (r[0] ^ r[1]) ^ (r[2] ^ r[3]);
}

// Thread j: Q_j = P / (z + x_j) by synthetic division (q_{m-1} = 1,
// q_{i-1} = p_i + x_j q_i), written transposed (QT[i][j]), and Q_j(x_j) by
// Horner in the same pass; scale[j] = x_j^-s / Q_j(x_j).
__global__ void vdm_quotients(const uint16_t *__restrict__ P, const uint16_t *__restrict__ x,
                              int m, uint32_t s, uint16_t *__restrict__ QT,
                              uint16_t *__restrict__ scale, int *__restrict__ status,
                              const uint16_t *__restrict__ glog, const uint16_t *__restrict__ gexp)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m)
        return;
    const uint32_t xj = x[j];
    uint32_t X[16];
    X[0] = xj;
#pragma unroll
    for (int i = 1; i < 16; ++i)
        X[i] = ((X[i - 1] << 1) ^ ((X[i - 1] & 0x8000u) ? 0x1100Bu : 0u)) & 0xFFFFu;
    uint32_t q = 1, h = 1;
    QT[static_cast<size_t>(m - 1) * m + j] = 1;
    for (int i = m - 1; i >= 1; --i) {
        q = __ldg(P + i) ^ gmul_fixed(X, q);
        QT[static_cast<size_t>(i - 1) * m + j] = static_cast<uint16_t>(q);
        h = gmul_fixed(X, h) ^ q;
    }
    if (h == 0 || (xj == 0 && s != 0)) {
        atomicExch(status, 1);
        scale[j] = 0;
        return;
    }
    // x_j^-s / h = 2^(-(s log x_j) - log h)  (mod 65535)
    const uint64_t lx = xj ? glog[xj] : 0;
    const uint64_t neg = (lx * s + glog[h]) % 65535u;
    scale[j] = gexp[neg == 0 ? 0 : 65535u - neg];
}

// inv[j][r] (row stride ld) = scale[j] * QT[e_r - s][j], through a 32 x 32 shared-memory tile
// so that both the reads (along j) and the writes (along r) are coalesced.
__global__ void vdm_finish(const uint16_t *__restrict__ QT, const uint16_t *__restrict__ scale,
                           const uint32_t *__restrict__ exps, uint32_t s, int m, int ld,
                           uint16_t *__restrict__ inv, const uint16_t *__restrict__ glog,
                           const uint16_t *__restrict__ gexp)
{
    __shared__ uint16_t tile[32][33];
    const int j0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int rr = ty; rr < 32; rr += blockDim.y) {
        const int r = r0 + rr, j = j0 + tx;
        tile[rr][tx] = (r < m && j < m) ? QT[static_cast<size_t>(exps[r] - s) * m + j] : 0;
    }
    __syncthreads();
    for (int jj = ty; jj < 32; jj += blockDim.y) {
        const int j = j0 + jj, r = r0 + tx;
        if (j < m && r < m)
            inv[static_cast<size_t>(j) * ld + r] =
                static_cast<uint16_t>(gmul(scale[j], tile[tx][jj], glog, gexp));
    }
}

// true when exps[0..m) is a permutation of s .. s+m-1
static bool exps_are_run(const uint32_t *exps, int m, uint32_t *s)
{
    uint32_t lo = exps[0], hi = exps[0];
    for (int r = 1; r < m; ++r) {
        lo = std::min(lo, exps[r]);
        hi = std::max(hi, exps[r]);
    }
    if (static_cast<uint64_t>(hi) - lo + 1 != static_cast<uint64_t>(m))
        return false;
    std::vector<char> seen(m, 0);
    for (int r = 0; r < m; ++r) {
        if (seen[exps[r] - lo])
            return false;
        seen[exps[r] - lo] = 1;
    }
    *s = lo;
    return true;
}

static int vdm_invert(p2g_ctx *ctx, GjWork &w, int m, const uint16_t *d_x, const uint32_t *d_exps,
                      uint32_t s, uint16_t *d_inv, int ld)
{
    const size_t vec = (static_cast<size_t>(m) * 2 + 255) & ~static_cast<size_t>(255);
    P2G_TRY(w.status.ensure(256 + 5 * vec));
    P2G_TRY(w.M.ensure(static_cast<size_t>(m) * m * 2 + 16));
    uint8_t *aux = w.status.as<uint8_t>();
    int *status = reinterpret_cast<int *>(aux);
    uint16_t *P[2] = {reinterpret_cast<uint16_t *>(aux + 256),
                      reinterpret_cast<uint16_t *>(aux + 256 + vec)};
    uint16_t *LP[2] = {reinterpret_cast<uint16_t *>(aux + 256 + 2 * vec),
                       reinterpret_cast<uint16_t *>(aux + 256 + 3 * vec)};
    uint16_t *scale = reinterpret_cast<uint16_t *>(aux + 256 + 4 * vec);
    P2G_CUDA(cudaMemsetAsync(status, 0, sizeof(int), ctx->stream));
    const int tb = 256, nb = (m + tb - 1) / tb;
    vdm_leaves<<<nb, tb, 0, ctx->stream>>>(d_x, m, P[0], LP[0], ctx->d_log);
    P2G_CUDA(cudaGetLastError());
    ++ctx->launches;
    int cur = 0;
    for (int G = 1; G < m; G *= 2) {
        vdm_level<<<nb, tb, 0, ctx->stream>>>(P[cur], LP[cur], P[cur ^ 1], LP[cur ^ 1], m, G,
                                              ctx->d_log, ctx->d_exp);
        P2G_CUDA(cudaGetLastError());
        ++ctx->launches;
        cur ^= 1;
    }
    uint16_t *QT = w.M.as<uint16_t>();
    vdm_quotients<<<(m + 31) / 32, 32, 0, ctx->stream>>>(P[cur], d_x, m, s, QT, scale, status,
                                                         ctx->d_log, ctx->d_exp);
    P2G_CUDA(cudaGetLastError());
    ++ctx->launches;
    const dim3 g2((m + 31) / 32, (m + 31) / 32), b2(32, 8);
    vdm_finish<<<g2, b2, 0, ctx->stream>>>(QT, scale, d_exps, s, m, ld, d_inv, ctx->d_log,
                                           ctx->d_exp);
    P2G_CUDA(cudaGetLastError());
    ++ctx->launches;
    return P2G_OK;
}

static size_t al256(size_t n) { return (n + 255) & ~static_cast<size_t>(255); }
// ---- a few exponents outside a run: Woodbury correction --------------------
//
// When g of the m exponents fall outside the window [s, s+m) that holds the
// most of them (recovery slices inside the window were lost), give each of
// those rows one of the window's unused exponents: the result V is a permuted
// Vandermonde matrix (closed-form inverse above) and A = V + U W differs from
// it in g rows, U selecting the rows Q and W[q][j] = x_j^e_q + x_j^h_q.  Then
//     A^-1 = V^-1 + V^-1 U C^-1 W V^-1,   C = I_g + W V^-1 U     (char 2: + = -)
// costs O(g m^2): three multiply-accumulate passes and a g x g inversion.  A
// is singular exactly when V or C is.

struct WoodburyPlan {
    uint32_t s = 0;
    std::vector<uint32_t> vexps;    // exponents of V (a permutation of s..s+m-1)
    std::vector<int> rows;          // Q: rows whose exponent lies outside the window
    std::vector<uint32_t> e, h;     // their exponents in A and in V
};

// false when the exponents repeat or more than kSmallM lie outside the best window
static bool plan_woodbury(const uint32_t *exps, int m, WoodburyPlan *wp)
{
    std::vector<uint32_t> sorted(exps, exps + m);
    std::sort(sorted.begin(), sorted.end());
    for (int i = 1; i < m; ++i)
        if (sorted[i] == sorted[i - 1])
            return false;
    int best = 0, bi = 0;
    for (int i = 0, j = 0; i < m; ++i) {
        while (j < m && static_cast<uint64_t>(sorted[j]) < static_cast<uint64_t>(sorted[i]) + m)
            ++j;
        if (j - i > best) {
            best = j - i;
            bi = i;
        }
    }
    const int g = m - best;
    if (g == 0 || g > kSmallM)
        return false;
    wp->s = sorted[bi];
    std::vector<char> taken(m, 0);
    for (int r = 0; r < m; ++r)
        if (exps[r] >= wp->s && exps[r] - wp->s < static_cast<uint32_t>(m))
            taken[exps[r] - wp->s] = 1;
    std::vector<uint32_t> holes;
    for (int t = 0; t < m; ++t)
        if (!taken[t])
            holes.push_back(wp->s + t);
    wp->vexps.assign(exps, exps + m);
    for (int r = 0; r < m; ++r)
        if (!(exps[r] >= wp->s && exps[r] - wp->s < static_cast<uint32_t>(m))) {
            wp->rows.push_back(r);
            wp->e.push_back(exps[r]);
            wp->h.push_back(holes[wp->rows.size() - 1]);
            wp->vexps[r] = wp->h.back();
        }
    return static_cast<int>(wp->rows.size()) == g && static_cast<int>(holes.size()) == g;
}

__device__ __forceinline__ uint32_t gpow(uint32_t x, uint32_t e, const uint16_t *__restrict__ glog,
                                         const uint16_t *__restrict__ gexp)
{
    if (x == 0)
        return e == 0 ? 1u : 0u;
    return gexp[static_cast<uint32_t>((static_cast<uint64_t>(glog[x]) * e) % 65535u)];
}

// Wm[q][j] = x_j^e_q + x_j^h_q  (g x m)
__global__ void wb_w_kernel(const uint16_t *__restrict__ x, int m, int g,
                            const uint32_t *__restrict__ e, const uint32_t *__restrict__ h,
                            uint16_t *__restrict__ Wm, const uint16_t *__restrict__ glog,
                            const uint16_t *__restrict__ gexp)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x, q = blockIdx.y;
    if (j < m && q < g)
        Wm[static_cast<size_t>(q) * m + j] =
            static_cast<uint16_t>(gpow(x[j], e[q], glog, gexp) ^ gpow(x[j], h[q], glog, gexp));
}

// [C | I] for gj_small: C[q][q'] = [q == q'] + Y[q][rows[q']]  (row stride ldc)
__global__ void wb_c_kernel(const uint16_t *__restrict__ Y, int ldy, const int *__restrict__ rows,
                            int g, uint16_t *__restrict__ Caug, int ldc)
{
    const int q = blockIdx.x;
    for (int c = threadIdx.x; c < 2 * g; c += blockDim.x) {
        uint32_t v = c < g ? (Y[static_cast<size_t>(q) * ldy + rows[c]] ^ (c == q ? 1u : 0u))
                           : (c - g == q ? 1u : 0u);
        Caug[static_cast<size_t>(q) * ldc + c] = static_cast<uint16_t>(v);
    }
}

// Vc[j][q] = Vinv[j][rows[q]]  (m x g)
__global__ void wb_cols_kernel(const uint16_t *__restrict__ Vinv, int ldv, const int *__restrict__ rows,
                               int m, int g, uint16_t *__restrict__ Vc)
{
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx < static_cast<size_t>(m) * g) {
        const size_t j = idx / g;
        const int q = static_cast<int>(idx - j * g);
        Vc[idx] = Vinv[j * ldv + rows[q]];
    }
}

static int woodbury_invert(p2g_ctx *ctx, GjWork &w, int m, const uint16_t *d_x,
                           const WoodburyPlan &wp, uint16_t *d_inv)
{
    const int g = static_cast<int>(wp.rows.size());
    const int ld = (m + 7) & ~7;                 // u16 per row: rows 16-byte aligned
    const int ldc = (2 * g + 7) & ~7;
    const size_t row = static_cast<size_t>(ld) * 2;
    // scratch: [vexps | e | h | rows | ptrs] then Vinv, Y, Z, Wm, Caug, Cinv, Vc
    const size_t o_e = al256(m * 4), o_h = o_e + al256(g * 4), o_rows = o_h + al256(g * 4),
                 o_ptr = o_rows + al256(g * 4), o_v = o_ptr + al256((m + 2 * g) * 8),
                 o_y = o_v + al256(m * row), o_z = o_y + al256(g * row),
                 o_w = o_z + al256(g * row), o_c = o_w + al256(static_cast<size_t>(g) * m * 2),
                 o_ci = o_c + al256(static_cast<size_t>(g) * ldc * 2),
                 o_vc = o_ci + al256(static_cast<size_t>(g) * g * 2),
                 total = o_vc + al256(static_cast<size_t>(m) * g * 2);
    P2G_TRY(ctx->wb.ensure(total));
    uint8_t *b = ctx->wb.as<uint8_t>();
    uint16_t *Vinv = reinterpret_cast<uint16_t *>(b + o_v), *Y = reinterpret_cast<uint16_t *>(b + o_y),
             *Wm = reinterpret_cast<uint16_t *>(b + o_w),
             *Caug = reinterpret_cast<uint16_t *>(b + o_c), *Cinv = reinterpret_cast<uint16_t *>(b + o_ci),
             *Vc = reinterpret_cast<uint16_t *>(b + o_vc);
    // host tables: V's exponents, e, h, rows and the row pointers of Vinv, Y, Z
    std::vector<uint8_t> hb(o_v, 0);
    memcpy(hb.data(), wp.vexps.data(), m * 4);
    memcpy(hb.data() + o_e, wp.e.data(), g * 4);
    memcpy(hb.data() + o_h, wp.h.data(), g * 4);
    memcpy(hb.data() + o_rows, wp.rows.data(), g * 4);
    uint8_t **ptr = reinterpret_cast<uint8_t **>(hb.data() + o_ptr);
    for (int j = 0; j < m; ++j)
        ptr[j] = b + o_v + j * row;
    for (int q = 0; q < g; ++q) {
        ptr[m + q] = b + o_y + q * row;
        ptr[m + g + q] = b + o_z + q * row;
    }
    // pageable source: consumed before the call returns
    P2G_CUDA(cudaMemcpyAsync(b, hb.data(), o_v, cudaMemcpyHostToDevice, ctx->stream));
    uint8_t *const *pv = reinterpret_cast<uint8_t *const *>(b + o_ptr);
    uint8_t *const *py = pv + m, *const *pz = pv + m + g;
    const int *d_rows = reinterpret_cast<const int *>(b + o_rows);
    // V^-1 (status cleared; set when V is singular)
    P2G_TRY(vdm_invert(ctx, w, m, d_x, reinterpret_cast<const uint32_t *>(b), wp.s, Vinv, ld));
    int *status = w.status.as<int>();
    // Y = W V^-1
    wb_w_kernel<<<dim3((m + 255) / 256, g), 256, 0, ctx->stream>>>(
        d_x, m, g, reinterpret_cast<const uint32_t *>(b + o_e),
        reinterpret_cast<const uint32_t *>(b + o_h), Wm, ctx->d_log, ctx->d_exp);
    P2G_CUDA(cudaGetLastError());
    // the three products' records (g, g and m outputs) share one buffer
    const size_t nrec = std::max({record_bytes(m, g), record_bytes(g, g), record_bytes(g, m)});
    P2G_TRY(ctx->recs2.ensure(nrec));
    uint32_t *recs = ctx->recs2.as<uint32_t>();
    const size_t bytes = static_cast<size_t>(m) * 2;
    P2G_TRY(records_from_matrix(ctx, Wm, m, g, recs));
    P2G_TRY(muladd_run(ctx, const_cast<const uint8_t *const *>(pv), m, py, g, bytes, recs, 0));
    // C = I + Y U, C^-1 by one CTA (status set when C is singular)
    wb_c_kernel<<<g, 128, 0, ctx->stream>>>(Y, ld, d_rows, g, Caug, ldc);
    P2G_CUDA(cudaGetLastError());
    const size_t smem = 65536 * 2 + static_cast<size_t>(g) * 2 * g * 2;
    P2G_CUDA(cudaFuncSetAttribute(gj_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    gj_small<<<1, kGjThreads, smem, ctx->stream>>>(Caug, g, ldc, Cinv, status, ctx->d_log,
                                                  ctx->d_exp);
    P2G_CUDA(cudaGetLastError());
    // Z = C^-1 Y
    P2G_TRY(records_from_matrix(ctx, Cinv, g, g, recs));
    P2G_TRY(muladd_run(ctx, const_cast<const uint8_t *const *>(py), g, pz, g, bytes, recs, 0));
    // V^-1 += (V^-1 U) Z
    const size_t nvc = static_cast<size_t>(m) * g;
    wb_cols_kernel<<<static_cast<unsigned>((nvc + 255) / 256), 256, 0, ctx->stream>>>(Vinv, ld, d_rows,
                                                                                   m, g, Vc);
    P2G_CUDA(cudaGetLastError());
    P2G_TRY(records_from_matrix(ctx, Vc, g, m, recs));
    P2G_TRY(muladd_run(ctx, const_cast<const uint8_t *const *>(pz), g, pv, m, bytes, recs, 1));
    P2G_CUDA(cudaMemcpy2DAsync(d_inv, bytes, Vinv, row, bytes, m, cudaMemcpyDeviceToDevice,
                               ctx->stream));
    ctx->launches += 6;
    return P2G_OK;
}


int gj_invert(p2g_ctx *ctx, GjWork &w, int m, const uint16_t *d_cmiss, const uint32_t *d_exps,
              const uint32_t *h_exps, const uint16_t *d_A, uint16_t *d_inv)
{
    if (m <= 0)
        return P2G_OK;
    uint32_t s = 0;
    if (!d_A && h_exps && exps_are_run(h_exps, m, &s))
        return vdm_invert(ctx, w, m, d_cmiss, d_exps, s, d_inv, m);
    WoodburyPlan wp;
    if (!d_A && h_exps && m > kSmallM && plan_woodbury(h_exps, m, &wp))
        return woodbury_invert(ctx, w, m, d_cmiss, wp, d_inv);
    const int W = (2 * m + 7) & ~7;  // row stride in u16: rows are 16-byte aligned
    const size_t row_bytes = static_cast<size_t>(W) * 2;
    P2G_TRY(w.M.ensure(static_cast<size_t>(m) * row_bytes));
    // aux layout: status | used | kall | orow | kptr | optr | xptr | akk_inv | X
    const size_t o_used = 256, o_kall = o_used + al256(m * 4), o_orow = o_kall + al256(m * 4),
                 o_kptr = o_orow + al256(m * 4), o_optr = o_kptr + al256(kPanel * 8),
                 o_xptr = o_optr + al256(static_cast<size_t>(m) * 8),
                 o_akk = o_xptr + al256(kPanel * 8),
                 o_X = o_akk + al256(kPanel * kPanel * 2), total = o_X + kPanel * row_bytes;
    P2G_TRY(w.status.ensure(total));
    uint8_t *aux = w.status.as<uint8_t>();
    uint16_t *M = w.M.as<uint16_t>();
    int *status = reinterpret_cast<int *>(aux);
    P2G_CUDA(cudaMemsetAsync(aux, 0, o_kall, ctx->stream));  // status + used
    dim3 g(static_cast<unsigned>((2 * m + 255) / 256 < 64 ? (2 * m + 255) / 256 : 64),
           static_cast<unsigned>(m));
    if (d_A)
        gj_build_from<<<g, 256, 0, ctx->stream>>>(M, m, W, d_A);
    else
        gj_build_par2<<<g, 256, 0, ctx->stream>>>(M, m, W, d_cmiss, d_exps, ctx->d_log, ctx->d_exp);
    P2G_CUDA(cudaGetLastError());
    ++ctx->launches;
    if (m <= kSmallM) {
        const size_t smem = 65536 * 2 + static_cast<size_t>(m) * 2 * m * 2;
        P2G_CUDA(cudaFuncSetAttribute(gj_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(smem)));
        gj_small<<<1, kGjThreads, smem, ctx->stream>>>(M, m, W, d_inv, status, ctx->d_log,
                                                      ctx->d_exp);
        P2G_CUDA(cudaGetLastError());
        ++ctx->launches;
        return P2G_OK;
    }
    PanelBufs pb;
    pb.used = reinterpret_cast<int *>(aux + o_used);
    pb.kall = reinterpret_cast<int *>(aux + o_kall);
    pb.orow = reinterpret_cast<int *>(aux + o_orow);
    pb.kptr = reinterpret_cast<const uint8_t **>(aux + o_kptr);
    pb.optr = reinterpret_cast<uint8_t **>(aux + o_optr);
    uint8_t **xptr = reinterpret_cast<uint8_t **>(aux + o_xptr);
    pb.akk_inv = reinterpret_cast<uint16_t *>(aux + o_akk);
    uint8_t *X = aux + o_X;
    {
        std::vector<uint8_t *> xp(kPanel);
        for (int j = 0; j < kPanel; ++j)
            xp[j] = X + j * row_bytes;
        P2G_CUDA(cudaMemcpyAsync(xptr, xp.data(), kPanel * sizeof(void *), cudaMemcpyHostToDevice,
                                 ctx->stream));
        // pageable source: consumed before the call returns
    }
    P2G_CUDA(cudaFuncSetAttribute(gj_panel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(kExpSmem)));
    // per panel: the b x b pivot block's records, then the b x (m - b) row
    // update's, each in the form for its output count (b, m - b <= m)
    const size_t recA_bytes = std::max(record_bytes(kPanel, kPanel),
                                       record_bytes(kSmallOutputs, kSmallOutputs));
    P2G_TRY(ctx->recs2.ensure(recA_bytes +
                              std::max(record_bytes(kPanel, m), record_bytes(kPanel, kSmallOutputs))));
    uint32_t *recsA = ctx->recs2.as<uint32_t>();
    uint32_t *recsO = recsA + recA_bytes / 4;
    for (int c0 = 0; c0 < m; c0 += kPanel) {
        const int b = std::min(kPanel, m - c0);
        gj_panel<<<1, kGjThreads, kExpSmem, ctx->stream>>>(M, m, W, c0, b, pb, status,
                                                           ctx->d_log, ctx->d_exp);
        P2G_CUDA(cudaGetLastError());
        ++ctx->launches;
        P2G_TRY(records_from_matrix(ctx, pb.akk_inv, b, b, recsA));
        const int no = m - b;
        if (no > 0) {
            size_t n = static_cast<size_t>(b) * no;
            gj_records_rows<<<static_cast<unsigned>((n + 255) / 256), 256, 0, ctx->stream>>>(
                M, W, pb.orow, c0, b, no, recsO);
            P2G_CUDA(cudaGetLastError());
            ++ctx->launches;
        }
        P2G_TRY(muladd_run(ctx, pb.kptr, b, xptr, b, row_bytes, recsA, 0));
        if (no > 0)
            P2G_TRY(muladd_run(ctx, const_cast<const uint8_t *const *>(xptr), b, pb.optr, no,
                               row_bytes, recsO, 1));
        gj_copy_rows<<<dim3(8, b), 256, 0, ctx->stream>>>(
            const_cast<const uint8_t *const *>(xptr), pb.kptr, b, row_bytes);
        P2G_CUDA(cudaGetLastError());
        ++ctx->launches;
    }
    gj_extract_perm<<<g, 256, 0, ctx->stream>>>(M, m, W, pb.kall, d_inv);
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
