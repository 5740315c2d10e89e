// Kernels of the restarted GMRES that solves the dense influence system
// (an addition to the reference's A\b, src/SlipCalculator3D.jl:22): the
// matrix-vector product with the 3N x 3N matrix -- the HBM-bound part, one
// pass over A per iteration -- and classical Gram-Schmidt with
// re-orthogonalisation, fused so that each pass over the Krylov basis also
// produces the next reduction's partial sums.
//
// Every reduction runs in a fixed order (per-block partials, then a fixed
// sum), so results are reproducible run to run.  Blocks own 256 consecutive
// rows; a block's partial dot products cover only its rows, which it also
// updates, so the fused passes need no grid-wide barrier.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "krylov.h"

namespace cad {

namespace {

constexpr int kRows = 256;     // rows per block
constexpr int kCols = 256;     // columns of x staged in shared memory at a time

// part[c][i] = sum over the columns of chunk c of A[i, j] x[j]
template <typename TA>
__global__ void __launch_bounds__(kRows) gemv_part_kernel(const TA* __restrict__ A, int64_t lda, int n,
                                                          const double* __restrict__ x, int chunk,
                                                          double* __restrict__ part)
{
    __shared__ double sx[kCols];
    const int i = blockIdx.x * kRows + threadIdx.x;
    const int c0 = blockIdx.y * chunk;
    const int c1 = c0 + chunk < n ? c0 + chunk : n;
    const bool live = i < n;
    const TA* a = A + (live ? i : 0);
    double acc0 = 0.0, acc1 = 0.0;
    for (int cb = c0; cb < c1; cb += kCols) {
        const int nc = c1 - cb < kCols ? c1 - cb : kCols;
        __syncthreads();
        if ((int)threadIdx.x < nc) sx[threadIdx.x] = x[cb + threadIdx.x];
        __syncthreads();
        if (!live) continue;
        const TA* ac = a + (int64_t)cb * lda;
        int j = 0;
        for (; j + 8 <= nc; j += 8) {
            TA v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = __ldcs(ac + (int64_t)(j + u) * lda);   // streamed once
#pragma unroll
            for (int u = 0; u < 8; u += 2) {
                acc0 = fma((double)v[u], sx[j + u], acc0);
                acc1 = fma((double)v[u + 1], sx[j + u + 1], acc1);
            }
        }
        for (; j < nc; ++j) acc0 = fma((double)ac[(int64_t)j * lda], sx[j], acc0);
    }
    if (live) part[(int64_t)blockIdx.y * n + i] = acc0 + acc1;
}

// The same with VEC consecutive rows per thread read as one 16-byte vector
// per column (A 16-byte aligned, lda a multiple of VEC): four times the bytes
// in flight per load instruction.  Rows past n are skipped per vector.
template <typename TA, typename TV, int VEC>
__global__ void __launch_bounds__(kRows) gemv_part_vec_kernel(const TA* __restrict__ A, int64_t lda, int n,
                                                              const double* __restrict__ x, int chunk,
                                                              double* __restrict__ part)
{
    __shared__ double sx[kCols];
    const int r0 = (blockIdx.x * kRows + threadIdx.x) * VEC;
    const int c0 = blockIdx.y * chunk;
    const int c1 = c0 + chunk < n ? c0 + chunk : n;
    const bool live = r0 < n;
    const bool full = r0 + VEC <= n;
    double acc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) acc[v] = 0.0;
    for (int cb = c0; cb < c1; cb += kCols) {
        const int nc = c1 - cb < kCols ? c1 - cb : kCols;
        __syncthreads();
        if ((int)threadIdx.x < nc) sx[threadIdx.x] = x[cb + threadIdx.x];
        __syncthreads();
        if (!live) continue;
        const TA* ac = A + r0 + (int64_t)cb * lda;
        if (full) {
            int j = 0;
            for (; j + 8 <= nc; j += 8) {
                TV w[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) w[u] = __ldcs(reinterpret_cast<const TV*>(ac + (int64_t)(j + u) * lda));
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const TA* e = reinterpret_cast<const TA*>(&w[u]);
#pragma unroll
                    for (int v = 0; v < VEC; ++v) acc[v] = fma((double)e[v], sx[j + u], acc[v]);
                }
            }
            for (; j < nc; ++j) {
                const TV w = *reinterpret_cast<const TV*>(ac + (int64_t)j * lda);
                const TA* e = reinterpret_cast<const TA*>(&w);
#pragma unroll
                for (int v = 0; v < VEC; ++v) acc[v] = fma((double)e[v], sx[j], acc[v]);
            }
        } else {
            for (int j = 0; j < nc; ++j)
#pragma unroll
                for (int v = 0; v < VEC; ++v)
                    if (r0 + v < n) acc[v] = fma((double)ac[(int64_t)j * lda + v], sx[j], acc[v]);
        }
    }
    if (!live) return;
#pragma unroll
    for (int v = 0; v < VEC; ++v)
        if (r0 + v < n) part[(int64_t)blockIdx.y * n + r0 + v] = acc[v];
}

__device__ __forceinline__ double block_sum(double v, double* sred)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) sred[warp] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kRows / 32; ++w) s += sred[w];
    return s;
}

// y[i] = (b ? b[i] : 0) + alpha * sum_c part[c][i]; with V set (nv columns,
// ldv) also dots[blockIdx.x][q] = sum over this block's rows of V[i, q] y[i]
__global__ void __launch_bounds__(kRows) gemv_reduce_kernel(const double* __restrict__ part, int nchunk, int n,
                                                            double alpha, const double* __restrict__ b,
                                                            double* __restrict__ y, const double* __restrict__ V,
                                                            int64_t ldv, int nv, double* __restrict__ dots)
{
    __shared__ double sred[kRows / 32];
    const int i = blockIdx.x * kRows + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        double s = 0.0;
        for (int c = 0; c < nchunk; ++c) s += part[(int64_t)c * n + i];
        v = (b ? b[i] : 0.0) + alpha * s;
        y[i] = v;
    }
    for (int q = 0; q < nv; ++q) {
        const double t = block_sum(i < n ? V[i + (int64_t)q * ldv] * v : 0.0, sred);
        if (threadIdx.x == 0) dots[(int64_t)blockIdx.x * nv + q] = t;
    }
}

// One classical Gram-Schmidt pass: h = sum over blocks of dots (fixed
// order), w -= V h on this block's rows; then, on the updated rows, either
// the next pass's dots (norm == false) or the partial squared norm.  Block 0
// stores h.
__global__ void __launch_bounds__(kRows) cgs_pass_kernel(const double* __restrict__ V, int64_t ldv, int n, int nv,
                                                         const double* __restrict__ dots, int nblk,
                                                         double* __restrict__ w, double* __restrict__ h_out,
                                                         bool norm, double* __restrict__ next)
{
    __shared__ double sh[kMaxBasis];
    __shared__ double sred[kRows / 32];
    for (int q = threadIdx.x; q < nv; q += kRows) {
        double s = 0.0;
        for (int bk = 0; bk < nblk; ++bk) s += dots[(int64_t)bk * nv + q];
        sh[q] = s;
        if (blockIdx.x == 0) h_out[q] = s;
    }
    __syncthreads();
    const int i = blockIdx.x * kRows + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        v = w[i];
        for (int q = 0; q < nv; ++q) v -= V[i + (int64_t)q * ldv] * sh[q];
        w[i] = v;
    }
    if (norm) {
        const double t = block_sum(v * v, sred);
        if (threadIdx.x == 0) next[blockIdx.x] = t;
    } else {
        for (int q = 0; q < nv; ++q) {
            const double t = block_sum(i < n ? V[i + (int64_t)q * ldv] * v : 0.0, sred);
            if (threadIdx.x == 0) next[(int64_t)blockIdx.x * nv + q] = t;
        }
    }
}

// hcol[q] = h1[q] + h2[q] (q < nv), hcol[nv] = sqrt(sum of the partial norms)
__global__ void cgs_finish_kernel(const double* __restrict__ h1, const double* __restrict__ h2, int nv,
                                  const double* __restrict__ norms, int nblk, double* __restrict__ hcol)
{
    __shared__ double s[256];
    double a = 0.0;
    for (int bk = threadIdx.x; bk < nblk; bk += blockDim.x) a += norms[bk];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int hh = blockDim.x / 2; hh > 0; hh >>= 1) {
        if ((int)threadIdx.x < hh) s[threadIdx.x] += s[threadIdx.x + hh];
        __syncthreads();
    }
    for (int q = threadIdx.x; q < nv; q += blockDim.x) hcol[q] = h1[q] + h2[q];
    if (threadIdx.x == 0) hcol[nv] = sqrt(s[0]);
}

// out = w / *hn (out = w untouched when hn is 0)
__global__ void scale_by_kernel(const double* __restrict__ w, int n, const double* __restrict__ hn,
                                double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double d = *hn;
    if (i < n) out[i] = d > 0.0 ? w[i] / d : w[i];
}

// partial squared norms of x per block
__global__ void __launch_bounds__(kRows) norm_part_kernel(const double* __restrict__ x, int n,
                                                          double* __restrict__ part)
{
    __shared__ double sred[kRows / 32];
    const int i = blockIdx.x * kRows + threadIdx.x;
    const double v = i < n ? x[i] : 0.0;
    const double t = block_sum(v * v, sred);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// out = sqrt(sum of part) (one block, fixed order)
__global__ void norm_finish_kernel(const double* __restrict__ part, int nblk, double* __restrict__ out)
{
    __shared__ double s[256];
    double a = 0.0;
    for (int bk = threadIdx.x; bk < nblk; bk += blockDim.x) a += part[bk];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int hh = blockDim.x / 2; hh > 0; hh >>= 1) {
        if ((int)threadIdx.x < hh) s[threadIdx.x] += s[threadIdx.x + hh];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sqrt(s[0]);
}

// out[i] = sum_q V[i, q] y[q]   (y: device, nv values)
__global__ void basis_combine_kernel(const double* __restrict__ V, int64_t ldv, int n, int nv,
                                     const double* __restrict__ y, double* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int q = 0; q < nv; ++q) s += V[i + (int64_t)q * ldv] * y[q];
    out[i] = s;
}

__global__ void axpy_kernel(double a, const double* __restrict__ x, int n, double* __restrict__ y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += a * x[i];
}

__global__ void cast_to_f32_kernel(const double* __restrict__ A, int64_t lda, int64_t n, float* __restrict__ B,
                                   int64_t ldb)
{
    for (int64_t c = blockIdx.y; c < n; c += gridDim.y)
        for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
            B[r + c * ldb] = (float)A[r + c * lda];
}

// y[j] = sum_i A[i + j lda] x[i] (j < cols, i < rows): one warp per column,
// lane-strided partial sums combined by a fixed shuffle tree
__global__ void gemv_t_kernel(const double* __restrict__ A, int64_t lda, int64_t rows, int64_t cols,
                              const double* __restrict__ x, double* __restrict__ y)
{
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t j = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); j < cols; j += warps) {
        const double* a = A + j * lda;
        double s = 0.0;
        for (int64_t i = lane; i < rows; i += 32) s = fma(a[i], x[i], s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) y[j] = s;
    }
}

// At[j + i ldt] = -A[i + j lda] through 32 x 32 shared-memory tiles
__global__ void transpose_neg_kernel(const double* __restrict__ A, int64_t lda, int64_t rows, int64_t cols,
                                     double* __restrict__ At, int64_t ldt)
{
    __shared__ double t[32][33];
    const int64_t i0 = (int64_t)blockIdx.x * 32, j0 = (int64_t)blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8 threads
    for (int r = ty; r < 32; r += 8)
        if (i0 + tx < rows && j0 + r < cols) t[r][tx] = A[(i0 + tx) + (j0 + r) * lda];
    __syncthreads();
    for (int r = ty; r < 32; r += 8)
        if (j0 + tx < cols && i0 + r < rows) At[(j0 + tx) + (i0 + r) * ldt] = -t[tx][r];
}

inline unsigned nb(int n) { return (unsigned)((n + kRows - 1) / kRows); }

}  // namespace

int krylov_blocks(int64_t n) { return (int)((n + kRows - 1) / kRows); }

size_t krylov_work_doubles(int64_t n)
{
    // gemv partials (kMaxGemvChunks x n), two dot buffers, norms, two h vectors
    const size_t nblk = (size_t)krylov_blocks(n);
    return (size_t)kMaxGemvChunks * (size_t)n + 2 * nblk * kMaxBasis + nblk + 2 * kMaxBasis + 64;
}

KrylovWork krylov_carve(double* base, int64_t n)
{
    const size_t nblk = (size_t)krylov_blocks(n);
    KrylovWork k;
    k.part = base;
    k.dots1 = k.part + (size_t)kMaxGemvChunks * (size_t)n;
    k.dots2 = k.dots1 + nblk * kMaxBasis;
    k.norms = k.dots2 + nblk * kMaxBasis;
    k.h1 = k.norms + nblk;
    k.h2 = k.h1 + kMaxBasis;
    k.scalar = k.h2 + kMaxBasis;
    return k;
}

template <typename TA>
cudaError_t krylov_gemv(cudaStream_t st, const TA* A, int64_t lda, int n, const double* x, double alpha,
                        const double* b, double* y, const KrylovWork& k, const double* V, int64_t ldv, int nv,
                        int64_t* launches, int nchunks)
{
    if (n <= 0) return cudaSuccess;
    if (nchunks < 1 || nchunks > kMaxGemvChunks) nchunks = kGemvChunks;
    const int chunk = (n + nchunks - 1) / nchunks;
    const int nchunk = (n + chunk - 1) / chunk;
    constexpr int VEC = 16 / (int)sizeof(TA);
    if (((uintptr_t)A & 15u) == 0 && lda % VEC == 0) {
        using TV = typename std::conditional<sizeof(TA) == 4, float4, double2>::type;
        const unsigned gx = (unsigned)((n + kRows * VEC - 1) / (kRows * VEC));
        gemv_part_vec_kernel<TA, TV, VEC><<<dim3(gx, (unsigned)nchunk), kRows, 0, st>>>(A, lda, n, x, chunk, k.part);
    } else {
        gemv_part_kernel<TA><<<dim3(nb(n), (unsigned)nchunk), kRows, 0, st>>>(A, lda, n, x, chunk, k.part);
    }
    gemv_reduce_kernel<<<nb(n), kRows, 0, st>>>(k.part, nchunk, n, alpha, b, y, V, ldv, V ? nv : 0, k.dots1);
    if (launches) *launches += 2;
    return cudaGetLastError();
}
template cudaError_t krylov_gemv<double>(cudaStream_t, const double*, int64_t, int, const double*, double,
                                         const double*, double*, const KrylovWork&, const double*, int64_t, int,
                                         int64_t*, int);
template cudaError_t krylov_gemv<float>(cudaStream_t, const float*, int64_t, int, const double*, double, const double*,
                                        double*, const KrylovWork&, const double*, int64_t, int, int64_t*, int);

cudaError_t krylov_orthogonalise(cudaStream_t st, const double* V, int64_t ldv, int n, int nv, double* w,
                                 double* hcol, double* vnext, const KrylovWork& k, int64_t* launches)
{
    if (nv > kMaxBasis) return cudaErrorInvalidValue;
    const int nblk = krylov_blocks(n);
    cgs_pass_kernel<<<nb(n), kRows, 0, st>>>(V, ldv, n, nv, k.dots1, nblk, w, k.h1, false, k.dots2);
    cgs_pass_kernel<<<nb(n), kRows, 0, st>>>(V, ldv, n, nv, k.dots2, nblk, w, k.h2, true, k.norms);
    cgs_finish_kernel<<<1, 256, 0, st>>>(k.h1, k.h2, nv, k.norms, nblk, hcol);
    scale_by_kernel<<<nb(n), kRows, 0, st>>>(w, n, hcol + nv, vnext);
    if (launches) *launches += 4;
    return cudaGetLastError();
}

cudaError_t krylov_norm(cudaStream_t st, const double* x, int n, double* out, const KrylovWork& k, int64_t* launches)
{
    const int nblk = krylov_blocks(n);
    norm_part_kernel<<<nb(n), kRows, 0, st>>>(x, n, k.norms);
    norm_finish_kernel<<<1, 256, 0, st>>>(k.norms, nblk, out);
    if (launches) *launches += 2;
    return cudaGetLastError();
}

cudaError_t krylov_scale(cudaStream_t st, const double* x, int n, const double* by, double* out, int64_t* launches)
{
    scale_by_kernel<<<nb(n), kRows, 0, st>>>(x, n, by, out);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t krylov_combine(cudaStream_t st, const double* V, int64_t ldv, int n, int nv, const double* y, double* out,
                           int64_t* launches)
{
    basis_combine_kernel<<<nb(n), kRows, 0, st>>>(V, ldv, n, nv, y, out);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t krylov_axpy(cudaStream_t st, double a, const double* x, int n, double* y, int64_t* launches)
{
    axpy_kernel<<<nb(n), kRows, 0, st>>>(a, x, n, y);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t krylov_cast_f32(cudaStream_t st, const double* A, int64_t lda, int64_t n, float* B, int64_t ldb,
                            int64_t* launches)
{
    if (n <= 0) return cudaSuccess;
    const int64_t rb = (n + 255) / 256;
    cast_to_f32_kernel<<<dim3((unsigned)(rb < 8 ? rb : 8), (unsigned)(n < 8192 ? n : 8192)), 256, 0, st>>>(A, lda, n,
                                                                                                      B, ldb);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t krylov_gemv_t(cudaStream_t st, const double* A, int64_t lda, int64_t rows, int64_t cols, const double* x,
                          double* y, int64_t* launches)
{
    if (cols <= 0) return cudaSuccess;
    if (rows <= 0) return cudaMemsetAsync(y, 0, (size_t)cols * sizeof(double), st);
    const int64_t blocks = (cols + 7) / 8;
    gemv_t_kernel<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, st>>>(A, lda, rows, cols, x, y);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t krylov_transpose_neg(cudaStream_t st, const double* A, int64_t lda, int64_t rows, int64_t cols, double* At,
                                 int64_t ldt, int64_t* launches)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    if ((rows + 31) / 32 > INT32_MAX || (cols + 31) / 32 > 65535) return cudaErrorInvalidValue;
    transpose_neg_kernel<<<dim3((unsigned)((rows + 31) / 32), (unsigned)((cols + 31) / 32)), 256, 0, st>>>(
        A, lda, rows, cols, At, ldt);
    if (launches) ++*launches;
    return cudaGetLastError();
}

}  // namespace cad
