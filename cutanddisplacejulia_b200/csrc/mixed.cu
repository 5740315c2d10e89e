// Mixed-precision solve of the 3N x 3N influence system (an addition to the
// reference's `A\b`, src/SlipCalculator3D.jl:22): the FP64 matrix is cast to
// FP32 and factorised by the blocked LU of csrc/lu.cu (TF32 tensor-core
// trailing updates), and restarted GMRES in FP64, right-preconditioned by that
// factorisation, drives the FP64 residual b - A x down to the requested
// relative tolerance.  FP64 is kept for the matrix-vector product, the Krylov
// basis and the solution; FP32 only inside the preconditioner.
//
// The preconditioner's triangular solves are one launch per triangle: each
// CTA owns a 128-row block, takes its place in the dependency order from an
// atomic ticket (so every block it waits for has already started), streams
// its off-diagonal blocks against the solved pieces as they are published
// (flag per block, release/acquire), and finishes with a GEMV against the
// explicitly inverted diagonal block.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <math.h>
#include <cstdint>
#include <vector>

#include "lu.h"
#include "mixed.h"
#include "gemm.h"
#include "krylov.h"
#include "mlp.h"

namespace cad {

namespace {

constexpr int kRB = 128;            // row block of the triangular solves
constexpr int kChainThreads = 512;  // four threads per row: quarters of each 128-column block

// B (n x n, leading dimension ldb) = (float) A (n x n, lda); columns strided over grid.y
__global__ void cast_f32_kernel(const double* __restrict__ A, int64_t lda, int64_t n, float* __restrict__ B,
                                int64_t ldb)
{
    for (int64_t c = blockIdx.y; c < n; c += gridDim.y)
        for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
            B[r + c * ldb] = (float)A[r + c * lda];
}

// Inverse of diagonal block i (kRB x kRB, zero-padded to the identity past n)
// of the unit lower (UPPER false) or the non-unit upper triangle of the LU
// factors, column-major into D + i * kRB * kRB.  Thread j computes column j of
// the inverse by substitution; the block and the inverse sit in shared memory
// (the inverse row-major with a pad, so the threads' columns are conflict-free).
// sum over k in [k0, k1) of a[k kRB] x[k (kRB + 1)]: four accumulators over
// consecutive k (added in a fixed order), the last k1 - k0 mod 4 terms into
// the first
__device__ __forceinline__ float dot_range(const float* a, const float* x, int k0, int k1)
{
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    int k = k0;
    for (; k + 4 <= k1; k += 4) {
        s0 = fmaf(a[k * kRB], x[k * (kRB + 1)], s0);
        s1 = fmaf(a[(k + 1) * kRB], x[(k + 1) * (kRB + 1)], s1);
        s2 = fmaf(a[(k + 2) * kRB], x[(k + 2) * (kRB + 1)], s2);
        s3 = fmaf(a[(k + 3) * kRB], x[(k + 3) * (kRB + 1)], s3);
    }
    for (; k < k1; ++k) s0 = fmaf(a[k * kRB], x[k * (kRB + 1)], s0);
    return (s0 + s1) + (s2 + s3);
}

template <bool UPPER>
__device__ __forceinline__ void invert_diag_body(const float* __restrict__ A, int64_t lda, int n,
                                                 float* __restrict__ D, int i)
{
    extern __shared__ float sm[];
    float* s_a = sm;                  // [kRB][kRB] column-major
    float* s_x = sm + kRB * kRB;      // [kRB][kRB + 1] row-major: s_x[r * (kRB + 1) + j]
    const int j = threadIdx.x;
    const int r0 = i * kRB;
    const int b = n - r0 < kRB ? n - r0 : kRB;
    for (int e = j; e < kRB * kRB; e += kRB) {
        const int r = e % kRB, c = e / kRB;
        float v = (r < b && c < b) ? A[(int64_t)(r0 + r) + (int64_t)(r0 + c) * lda] : 0.f;
        if (r == c && r >= b) v = 1.f;
        s_a[e] = v;
    }
    __syncthreads();
    // The k loops run over the warp's common range (the column's own entries
    // outside [j, r) are the zeros written above), so every read of the
    // triangle is a broadcast; four accumulators (k mod 4, added in a fixed
    // order) keep four multiply-adds in flight.
    const int jw0 = j & ~31, jw1 = j | 31;
    if (!UPPER) {
        for (int r = 0; r < kRB; ++r) {
            float v;
            const float sum = dot_range(s_a + r, s_x + j, jw0, r);
            if (r < j) v = 0.f;
            else if (r == j) v = 1.f;
            else v = -sum;
            s_x[r * (kRB + 1) + j] = v;
        }
    } else {
        for (int r = kRB - 1; r >= 0; --r) {
            float v;
            const float sum = dot_range(s_a + r, s_x + j, r + 1, jw1 + 1);
            if (r > j) v = 0.f;
            else if (r == j) v = 1.f / s_a[r + r * kRB];
            else v = -sum / s_a[r + r * kRB];
            s_x[r * (kRB + 1) + j] = v;
        }
    }
    __syncthreads();
    float* out = D + (int64_t)i * kRB * kRB;
    for (int e = j; e < kRB * kRB; e += kRB) {
        const int r = e % kRB, c = e / kRB;
        out[e] = s_x[r * (kRB + 1) + c];
    }
}

template <bool UPPER>
__global__ void __launch_bounds__(kRB) invert_diag_kernel(const float* __restrict__ A, int64_t lda, int n,
                                                         float* __restrict__ D)
{
    invert_diag_body<UPPER>(A, lda, n, D, blockIdx.x);
}

__device__ __forceinline__ int ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int* p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// One triangle of M^-1 v with M = P^T L U in FP32.  Lower (UPPER false):
// y = L^-1 (P v), v FP64 gathered through perm.  Upper: x = U^-1 y, written
// as FP64 to out.  x32 holds the solved blocks for the other CTAs; flags[i]
// is set once block i is published; ticket orders the CTAs (a CTA waits only
// on blocks whose CTAs took earlier tickets, so they are running).
// Thread (q, r): row r of the CTA's 128-row block, column quarter q of every
// 128-column block.  The quarter's 32 values of the next block are loaded
// before its flag is awaited, so the memory latency overlaps the wait.
template <bool UPPER>
__device__ __forceinline__ void trsv_chain_body(const float* __restrict__ A, int64_t lda, int n, int nblk,
                                                const float* __restrict__ Dinv, const double* __restrict__ v_in,
                                                const int* __restrict__ perm, const float* y_in, float* x32,
                                                double* __restrict__ out, int* flags, int* ticket, int* fail,
                                                long wait_limit)
{
    constexpr int kQ = kChainThreads / kRB;   // column quarters
    constexpr int kC = kRB / kQ;              // columns per quarter
    __shared__ float s_x[kRB];
    __shared__ float s_part[kQ][kRB];
    __shared__ int s_t;
    const int tid = threadIdx.x, rr = tid % kRB, q = tid / kRB;
    if (tid == 0) s_t = atomicAdd(ticket, 1);
    __syncthreads();
    const int t = s_t;
    const int i = UPPER ? nblk - 1 - t : t;
    const int r0 = i * kRB;
    const int rows = n - r0 < kRB ? n - r0 : kRB;
    const int row = r0 + rr;
    const bool rok = rr < rows;
    float acc = 0.f;
    if (q == 0 && rok) acc = UPPER ? __ldcg(y_in + row) : (float)v_in[perm[row]];
    for (int s = 0; s < t; ++s) {
        const int j = UPPER ? nblk - 1 - s : s;
        const int c0 = j * kRB + q * kC;
        float a[kC];
#pragma unroll
        for (int c = 0; c < kC; ++c) a[c] = (rok && c0 + c < n) ? __ldg(A + row + (int64_t)(c0 + c) * lda) : 0.f;
        if (tid == 0) {
            long spins = 0;
            while (ld_acquire(flags + j) == 0) {
                if (++spins > wait_limit) {
                    atomicExch(fail, 1);
                    break;
                }
                __nanosleep(32);
            }
        }
        __syncthreads();
        if (tid < kRB) s_x[tid] = j * kRB + tid < n ? __ldcg(x32 + j * kRB + tid) : 0.f;
        __syncthreads();
        float p0 = 0.f, p1 = 0.f;
#pragma unroll
        for (int c = 0; c < kC; c += 2) {
            p0 = fmaf(a[c], s_x[q * kC + c], p0);
            p1 = fmaf(a[c + 1], s_x[q * kC + c + 1], p1);
        }
        acc -= p0 + p1;
    }
    // right-hand side of the diagonal block, then its explicit inverse
    s_part[q][rr] = acc;
    __syncthreads();
    if (tid < kRB) {
        float sum = 0.f;
#pragma unroll
        for (int k = 0; k < kQ; ++k) sum += s_part[k][tid];
        s_x[tid] = sum;
    }
    __syncthreads();
    const float* d = Dinv + (int64_t)i * kRB * kRB + rr + (int64_t)(q * kC) * kRB;
    float p0 = 0.f, p1 = 0.f;
#pragma unroll
    for (int c = 0; c < kC; c += 2) {
        p0 = fmaf(d[(int64_t)c * kRB], s_x[q * kC + c], p0);
        p1 = fmaf(d[(int64_t)(c + 1) * kRB], s_x[q * kC + c + 1], p1);
    }
    s_part[q][rr] = p0 + p1;
    __syncthreads();
    if (tid < rows) {
        float x = 0.f;
#pragma unroll
        for (int k = 0; k < kQ; ++k) x += s_part[k][tid];
        x32[r0 + tid] = x;
        if (UPPER) out[r0 + tid] = (double)x;
    }
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        st_release(flags + i, 1);
    }
}

template <bool UPPER>
__global__ void __launch_bounds__(kChainThreads) trsv_chain_kernel(
    const float* __restrict__ A, int64_t lda, int n, int nblk, const float* __restrict__ Dinv,
    const double* __restrict__ v_in, const int* __restrict__ perm, const float* y_in, float* x32,
    double* __restrict__ out, int* flags, int* ticket, int* fail, long wait_limit)
{
    trsv_chain_body<UPPER>(A, lda, n, nblk, Dinv, v_in, perm, y_in, x32, out, flags, ticket, fail, wait_limit);
}

}  // namespace

int mixed_prepare(const LuStreams& ls, const double* A, int64_t lda, int64_t n, float* A32, float* Dinv, int* ipiv,
                  int* perm, int* info, int nb, bool inverses)
{
    if (n <= 0) return LU_OK;
    const int64_t rb = (n + 255) / 256;
    const int64_t ld = mixed_ld(n);
    cast_f32_kernel<<<dim3((unsigned)(rb < 8 ? rb : 8), (unsigned)(n < 4096 ? n : 4096)), 256, 0, ls.main>>>(A, lda, n,
                                                                                                     A32, ld);
    if (cudaGetLastError() != cudaSuccess) return LU_CUDA_ERROR;
    if (ls.launches) ++*ls.launches;
    int rc = lu_factor_solve<float>(ls, A32, n, ld, nullptr, 0, 0, nullptr, 0, ipiv, perm, info, nb, true, false);
    if (rc != LU_OK) return rc;
    rc = lu_pivots_to_perm(ls, ipiv, n, perm);
    if (rc != LU_OK || !inverses) return rc;
    const int nblk = (int)((n + kRB - 1) / kRB);
    const size_t smem = (size_t)(kRB * kRB + kRB * (kRB + 1)) * sizeof(float);
    if (cudaFuncSetAttribute(invert_diag_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(invert_diag_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
        return LU_CUDA_ERROR;
    invert_diag_kernel<false><<<nblk, kRB, smem, ls.main>>>(A32, ld, (int)n, Dinv);
    invert_diag_kernel<true><<<nblk, kRB, smem, ls.main>>>(A32, ld, (int)n, Dinv + (int64_t)nblk * kRB * kRB);
    if (cudaGetLastError() != cudaSuccess) return LU_CUDA_ERROR;
    if (ls.launches) *ls.launches += 2;
    return LU_OK;
}

int64_t mixed_ld(int64_t n) { return (n + 3) / 4 * 4; }

size_t mixed_dinv_floats(int64_t n) { return (size_t)2 * ((n + kRB - 1) / kRB) * kRB * kRB; }
size_t mixed_sync_ints(int64_t n) { return (size_t)2 * ((n + kRB - 1) / kRB) + 4; }

namespace {

struct Precond {
    const float* A32;
    const float* Dinv;
    const int* perm;
    int n, nblk;
    float* y32;
    float* x32;
    int* sync;   // [2 * nblk flags][2 tickets][fail]
    cudaStream_t st;
    int64_t* launches;
    const int* spai_nbr;
    const float* spai_blocks;
    int spai_k;
    long wait_limit;

    // z = M^-1 v (FP64 in and out, FP32 inside)
    bool apply(const double* v, double* z) const
    {
        if (spai_nbr) {
            if (launches) ++*launches;
            return spai_apply(st, spai_nbr, spai_blocks, spai_k, v, n / 3, z) == cudaSuccess;
        }
        if (cudaMemsetAsync(sync, 0, (size_t)(2 * nblk + 2) * sizeof(int), st) != cudaSuccess) return false;
        int* fl = sync;
        int* fu = sync + nblk;
        int* tk = sync + 2 * nblk;
        int* fail = sync + 2 * nblk + 2;
        const float* DL = Dinv;
        const float* DU = Dinv + (int64_t)nblk * kRB * kRB;
        trsv_chain_kernel<false><<<nblk, kChainThreads, 0, st>>>(A32, mixed_ld(n), n, nblk, DL, v, perm, nullptr, y32, nullptr,
                                                                 fl, tk, fail, wait_limit);
        trsv_chain_kernel<true><<<nblk, kChainThreads, 0, st>>>(A32, mixed_ld(n), n, nblk, DU, nullptr, nullptr, y32, x32, z, fu,
                                                                tk + 1, fail, wait_limit);
        if (launches) *launches += 2;
        return cudaGetLastError() == cudaSuccess;
    }
};

}  // namespace

int gmres_ir_solve(const GmresArgs& a, GmresResult* res)
{
    const int64_t n = a.n;
    const int m = a.restart;
    cudaStream_t st = a.stream;
    res->iterations = 0;
    res->rel_residual = 0.0;
    res->status = GMRES_OK;
    if (m < 1 || m + 1 > kMaxBasis || n > INT32_MAX || !a.kwork) return GMRES_CUDA_ERROR;
    const int nn = (int)n;
    const int nblk = (int)((n + kRB - 1) / kRB);
    Precond M{a.A32, a.Dinv, a.perm, (int)n, nblk, a.y32, a.x32, a.sync, st, a.launches, a.spai_nbr, a.spai_blocks,
              a.spai_k, a.wait_limit > 0 ? a.wait_limit : kDefaultWaitLimit};
    const KrylovWork kw = krylov_carve(a.kwork, n);
    double* V = a.V;        // n x (m + 1)
    double* w = a.w;
    double* z = a.z;
    double* r = a.r;
    double* hd = a.hd;      // 2 (m + 1) device scratch: the Hessenberg column, then y
    double* x = a.x;
    int64_t* L = a.launches;
#define GM_CK(e)                                  \
    do {                                          \
        if ((e) != cudaSuccess) return GMRES_CUDA_ERROR; \
    } while (0)

    GM_CK(cudaMemsetAsync(a.sync + 2 * nblk + 2, 0, sizeof(int), st));
    double bnorm = 0.0;
    GM_CK(krylov_norm(st, a.b, nn, kw.scalar, kw, L));
    GM_CK(cudaMemcpyAsync(&bnorm, kw.scalar, sizeof(double), cudaMemcpyDeviceToHost, st));
    GM_CK(cudaMemsetAsync(x, 0, n * sizeof(double), st));
    GM_CK(cudaStreamSynchronize(st));
    if (bnorm == 0.0) return GMRES_OK;

    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), hcol(m + 2), y(m);
    int total = 0;
    while (true) {
        // true residual r = b - A x, in FP64
        GM_CK(krylov_gemv<double>(st, a.A, a.lda, nn, x, -1.0, a.b, r, kw, nullptr, 0, 0, L));
        GM_CK(krylov_norm(st, r, nn, kw.scalar + 1, kw, L));
        double beta = 0.0;
        GM_CK(cudaMemcpyAsync(&beta, kw.scalar + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
        GM_CK(cudaStreamSynchronize(st));
        res->rel_residual = beta / bnorm;
        res->iterations = total;
        if (res->rel_residual <= a.tol) return GMRES_OK;
        if (total >= a.max_iter) {
            res->status = GMRES_NOT_CONVERGED;
            return GMRES_NOT_CONVERGED;
        }
        GM_CK(krylov_scale(st, r, nn, kw.scalar + 1, V, L));
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int kend = 0;
        for (int k = 0; k < m; ++k) {
            double* vk = V + (int64_t)k * n;
            if (!M.apply(vk, z)) return GMRES_CUDA_ERROR;
            // w = A z (the FP32 copy of A when one is given: the Arnoldi
            // matrix only needs to be accurate to the restart's reduction),
            // with the first Gram-Schmidt pass's dot products
            const int gc = a.gemv_chunks > 0 ? a.gemv_chunks : kGemvChunks;
            if (a.A32mv)
                GM_CK(krylov_gemv<float>(st, a.A32mv, a.ld32, nn, z, 1.0, nullptr, w, kw, V, n, k + 1, L, gc));
            else
                GM_CK(krylov_gemv<double>(st, a.A, a.lda, nn, z, 1.0, nullptr, w, kw, V, n, k + 1, L, gc));
            GM_CK(krylov_orthogonalise(st, V, n, nn, k + 1, w, hd, V + (int64_t)(k + 1) * n, kw, L));
            GM_CK(cudaMemcpyAsync(hcol.data(), hd, (k + 2) * sizeof(double), cudaMemcpyDeviceToHost, st));
            GM_CK(cudaStreamSynchronize(st));
            double* Hk = H.data() + (size_t)k * (m + 1);
            for (int q = 0; q <= k + 1; ++q) Hk[q] = hcol[q];
            const double hn = hcol[k + 1];
            // previous rotations, then a new one zeroing H[k+1][k]
            for (int q = 0; q < k; ++q) {
                const double t0 = cs[q] * Hk[q] + sn[q] * Hk[q + 1];
                Hk[q + 1] = -sn[q] * Hk[q] + cs[q] * Hk[q + 1];
                Hk[q] = t0;
            }
            const double den = std::hypot(Hk[k], Hk[k + 1]);
            cs[k] = den > 0.0 ? Hk[k] / den : 1.0;
            sn[k] = den > 0.0 ? Hk[k + 1] / den : 0.0;
            Hk[k] = den;
            Hk[k + 1] = 0.0;
            g[k + 1] = -sn[k] * g[k];
            g[k] = cs[k] * g[k];
            ++total;
            kend = k + 1;
            // the rotated g estimates the residual; stop a little below the
            // tolerance so the true residual checked next is within it
            if (std::fabs(g[k + 1]) <= 0.5 * a.tol * bnorm || total >= a.max_iter || hn == 0.0) break;
        }
        // y = H^-1 g (upper triangular kend x kend), x += M^-1 (V y)
        for (int q = kend - 1; q >= 0; --q) {
            double s = g[q];
            for (int c = q + 1; c < kend; ++c) s -= H[(size_t)c * (m + 1) + q] * y[c];
            y[q] = s / H[(size_t)q * (m + 1) + q];
        }
        GM_CK(cudaMemcpyAsync(hd, y.data(), kend * sizeof(double), cudaMemcpyHostToDevice, st));
        GM_CK(krylov_combine(st, V, n, nn, kend, hd, w, L));
        if (!M.apply(w, z)) return GMRES_CUDA_ERROR;
        GM_CK(krylov_axpy(st, 1.0, z, nn, x, L));
        int fail = 0;
        GM_CK(cudaMemcpyAsync(&fail, a.sync + 2 * nblk + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
        GM_CK(cudaStreamSynchronize(st));
        if (fail) return GMRES_TIMEOUT;
    }
#undef GM_CK
}


// ------------------------------------------------- batched iterative refinement
namespace {

// Y (n x ncol, ldy) = (float) X (ldx)
__global__ void d2f_kernel(const double* __restrict__ X, int64_t ldx, int64_t n, float* __restrict__ Y, int64_t ldy)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t c = blockIdx.y;
    if (i < n) Y[i + c * ldy] = (float)X[i + c * ldx];
}

// X (ldx) += (double) Y (ldy)
__global__ void add_f2d_kernel(const float* __restrict__ Y, int64_t ldy, int64_t n, double* __restrict__ X,
                               int64_t ldx)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t c = blockIdx.y;
    if (i < n) X[i + c * ldx] += (double)Y[i + c * ldy];
}

// out[c] = || X[:, c] ||_2, one block per column, fixed summation order
__global__ void __launch_bounds__(256) col_norms_kernel(const double* __restrict__ X, int64_t ldx, int64_t n,
                                                        double* __restrict__ out)
{
    __shared__ double s[256];
    const int64_t c = blockIdx.x;
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += 256) {
        const double v = X[i + c * ldx];
        acc = fma(v, v, acc);
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = sqrt(s[0]);
}

}  // namespace

namespace {

// R = B - A X (n x nrhs): one column as a matrix-vector product, several as
// the library's FP64 tensor-core GEMM
cudaError_t ir_residual(const IrArgs& a, cudaStream_t st)
{
    const int64_t n = a.n;
    if (a.nrhs == 1 && a.kwork)
        return krylov_gemv<double>(st, a.A, a.lda, (int)n, a.X, -1.0, a.B, a.R, krylov_carve(a.kwork, n), nullptr,
                                   0, 0, a.ls.launches);
    cudaError_t e = cudaMemcpy2DAsync(a.R, n * sizeof(double), a.B, a.ldb * sizeof(double), n * sizeof(double),
                                      a.nrhs, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    if (a.ls.launches) ++*a.ls.launches;
    return gemm_sub(st, (int)n, a.nrhs, (int)n, a.A, a.lda, a.X, n, a.R, n, nullptr);
}

}  // namespace

int ir_solve_batched(const IrArgs& a, IrResult* res, std::vector<char>& converged)
{
    const int64_t n = a.n;
    const int nrhs = a.nrhs;
    cudaStream_t st = a.ls.main;
    res->status = GMRES_OK;
    res->iterations = 0;
    res->max_rel_residual = 0.0;
    converged.assign(nrhs, 0);
    if (n == 0 || nrhs == 0) return GMRES_OK;
    int64_t* launches = a.ls.launches;
    const dim3 g((unsigned)((n + 255) / 256), (unsigned)nrhs);
    std::vector<double> hn(2 * (size_t)nrhs);
    col_norms_kernel<<<nrhs, 256, 0, st>>>(a.B, a.ldb, n, a.norms);
    if (cudaMemsetAsync(a.X, 0, (size_t)n * nrhs * sizeof(double), st) != cudaSuccess ||
        cudaMemcpy2DAsync(a.R, n * sizeof(double), a.B, a.ldb * sizeof(double), n * sizeof(double), nrhs,
                          cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return GMRES_CUDA_ERROR;
    if (launches) ++*launches;
    double prev = INFINITY;
    for (int it = 1; it <= a.max_iter; ++it) {
        d2f_kernel<<<g, 256, 0, st>>>(a.R, n, n, a.R32, n);
        if (launches) ++*launches;
        if (cudaGetLastError() != cudaSuccess) return GMRES_CUDA_ERROR;
        const int rc = lu_factor_solve<float>(a.ls, a.A32, n, mixed_ld(n), a.R32, n, nrhs, a.X32, n, a.ipiv, a.perm, a.info,
                                              a.nb, false, true);
        if (rc != LU_OK) return GMRES_CUDA_ERROR;
        add_f2d_kernel<<<g, 256, 0, st>>>(a.X32, n, n, a.X, n);
        if (launches) ++*launches;
        if (ir_residual(a, st) != cudaSuccess) return GMRES_CUDA_ERROR;
        col_norms_kernel<<<nrhs, 256, 0, st>>>(a.R, n, n, a.norms + nrhs);
        if (launches) ++*launches;
        if (cudaMemcpyAsync(hn.data(), a.norms, 2 * (size_t)nrhs * sizeof(double), cudaMemcpyDeviceToHost, st) !=
                cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return GMRES_CUDA_ERROR;
        res->iterations = it;
        double worst = 0.0;
        bool all = true;
        for (int c = 0; c < nrhs; ++c) {
            const double rr = hn[c] > 0.0 ? hn[nrhs + c] / hn[c] : 0.0;
            converged[c] = rr <= a.tol;
            all = all && converged[c];
            worst = rr > worst || rr != rr ? rr : worst;
        }
        res->max_rel_residual = worst;
        if (all || !(worst < 0.5 * prev)) break;   // done, or refinement stopped converging (or NaN)
        prev = worst;
    }
    return GMRES_OK;
}


namespace {
// out[0] = max_c norms[nrhs + c] / norms[c] (0 where norms[c] == 0; NaN kept)
__global__ void relres_kernel(const double* __restrict__ norms, int nrhs, double* __restrict__ out)
{
    double worst = 0.0;
    for (int c = 0; c < nrhs; ++c) {
        const double r = norms[c] > 0.0 ? norms[nrhs + c] / norms[c] : 0.0;
        worst = (r > worst || r != r) ? r : worst;
    }
    out[0] = worst;
}
}  // namespace

int ir_solve_fixed(const IrArgs& a, int iters, double* rel_out)
{
    const int64_t n = a.n;
    const int nrhs = a.nrhs;
    cudaStream_t st = a.ls.main;
    if (n == 0 || nrhs == 0) return GMRES_OK;
    int64_t* launches = a.ls.launches;
    const dim3 g((unsigned)((n + 255) / 256), (unsigned)nrhs);
    col_norms_kernel<<<nrhs, 256, 0, st>>>(a.B, a.ldb, n, a.norms);
    if (launches) ++*launches;
    if (cudaMemsetAsync(a.X, 0, (size_t)n * nrhs * sizeof(double), st) != cudaSuccess ||
        cudaMemcpy2DAsync(a.R, n * sizeof(double), a.B, a.ldb * sizeof(double), n * sizeof(double), nrhs,
                          cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return GMRES_CUDA_ERROR;
    const bool chain = nrhs == 1 && a.Dinv && a.sync && a.Z;
    const int nblk = (int)((n + kRB - 1) / kRB);
    Precond M{a.A32, a.Dinv, a.perm, (int)n, nblk, a.R32, a.X32, a.sync, st, launches, nullptr, nullptr, 0,
              a.wait_limit > 0 ? a.wait_limit : kDefaultWaitLimit};
    for (int it = 0; it < iters; ++it) {
        if (chain) {
            // X += LU32 \ R: two chain launches, FP64 in and out
            if (!M.apply(a.R, a.Z)) return GMRES_CUDA_ERROR;
            if (krylov_axpy(st, 1.0, a.Z, (int)n, a.X, launches) != cudaSuccess) return GMRES_CUDA_ERROR;
        } else {
            d2f_kernel<<<g, 256, 0, st>>>(a.R, n, n, a.R32, n);
            if (launches) ++*launches;
            if (cudaGetLastError() != cudaSuccess) return GMRES_CUDA_ERROR;
            const int rc = lu_factor_solve<float>(a.ls, a.A32, n, mixed_ld(n), a.R32, n, nrhs, a.X32, n, a.ipiv, a.perm, a.info,
                                                  a.nb, false, true);
            if (rc != LU_OK) return GMRES_CUDA_ERROR;
            add_f2d_kernel<<<g, 256, 0, st>>>(a.X32, n, n, a.X, n);
            if (launches) ++*launches;
        }
        if (ir_residual(a, st) != cudaSuccess) return GMRES_CUDA_ERROR;
    }
    col_norms_kernel<<<nrhs, 256, 0, st>>>(a.R, n, n, a.norms + nrhs);
    relres_kernel<<<1, 1, 0, st>>>(a.norms, nrhs, rel_out);
    if (launches) *launches += 2;
    return cudaGetLastError() == cudaSuccess ? GMRES_OK : GMRES_CUDA_ERROR;
}

// ------------------------------------------------ grouped many-crack solve
namespace {

constexpr int kCrackGroupMax = 256;   // cracks per grouped launch
struct CrackGroup {
    int count, pad;
    CrackRec rec[kCrackGroupMax];
};
static_assert(sizeof(CrackGroup) <= 32000, "grouped solve records exceed the kernel parameter space");

// A32 (n_pad x n_pad, leading dimension n_pad) = (float) A, the identity past n
__global__ void __launch_bounds__(256) cast_pad_group_kernel(const __grid_constant__ CrackGroup g)
{
    const CrackRec& r = g.rec[blockIdx.y];
    for (int c = blockIdx.x; c < r.n_pad; c += gridDim.x) {
        float* dst = r.A32 + (int64_t)c * r.n_pad;
        const double* src = r.A + (int64_t)c * r.lda;
        for (int i = threadIdx.x; i < r.n_pad; i += blockDim.x)
            dst[i] = (i < r.n && c < r.n) ? (float)src[i] : (i == c ? 1.f : 0.f);
    }
}

// inverses of the diagonal blocks: z = 0 unit lower, z = 1 upper
__global__ void __launch_bounds__(kRB) invert_group_kernel(const __grid_constant__ CrackGroup g)
{
    const CrackRec& r = g.rec[blockIdx.y];
    const int nblk = r.n_pad / kRB;
    if ((int)blockIdx.x >= nblk) return;
    if (blockIdx.z == 0)
        invert_diag_body<false>(r.A32, r.n_pad, r.n_pad, r.Dinv, blockIdx.x);
    else
        invert_diag_body<true>(r.A32, r.n_pad, r.n_pad, r.Dinv + (int64_t)nblk * kRB * kRB, blockIdx.x);
}

// one triangle of z = (LU)^-1 P r for every crack (per-crack tickets and
// flags in its sync words: [nblk lower flags][nblk upper flags][2 tickets][fail])
template <bool UPPER>
__global__ void __launch_bounds__(kChainThreads) chain_group_kernel(const __grid_constant__ CrackGroup g,
                                                                    long wait_limit)
{
    const CrackRec& r = g.rec[blockIdx.y];
    const int nblk = r.n_pad / kRB;
    if ((int)blockIdx.x >= nblk) return;   // before any ticket is taken
    int* sync = r.sync;
    if (!UPPER)
        trsv_chain_body<false>(r.A32, r.n_pad, r.n_pad, nblk, r.Dinv, r.r, r.perm, nullptr, r.y32, nullptr, sync,
                               sync + 2 * nblk, sync + 2 * nblk + 2, wait_limit);
    else
        trsv_chain_body<true>(r.A32, r.n_pad, r.n_pad, nblk, r.Dinv + (int64_t)nblk * kRB * kRB, nullptr, nullptr,
                              r.y32, r.x32, r.z, sync + nblk, sync + 2 * nblk + 1, sync + 2 * nblk + 2, wait_limit);
}

// x = 0, r = b (zero past n)
__global__ void __launch_bounds__(256) init_group_kernel(const __grid_constant__ CrackGroup g)
{
    const CrackRec& r = g.rec[blockIdx.y];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.n_pad; i += gridDim.x * blockDim.x) {
        if (i < r.n) r.x[i] = 0.0;
        r.r[i] = i < r.n ? r.b[i] : 0.0;
    }
}

// x += z
__global__ void __launch_bounds__(256) axpy_group_kernel(const __grid_constant__ CrackGroup g)
{
    const CrackRec& r = g.rec[blockIdx.y];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < r.n; i += gridDim.x * blockDim.x) r.x[i] += r.z[i];
}

// r = b - A x in FP64: thread per row (coalesced down each column), x staged
// through shared memory, eight column loads in flight per thread into four
// accumulators (column c to accumulator c % 4, combined in a fixed order);
// rows past n zero
__global__ void __launch_bounds__(128) residual_group_kernel(const __grid_constant__ CrackGroup g)
{
    __shared__ double s_x[1024];
    const CrackRec& r = g.rec[blockIdx.y];
    const int i = blockIdx.x * 128 + threadIdx.x;
    if ((int)blockIdx.x * 128 >= r.n_pad) return;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c0 = 0; c0 < r.n; c0 += 1024) {
        const int cn = r.n - c0 < 1024 ? r.n - c0 : 1024;
        __syncthreads();
        for (int c = threadIdx.x; c < cn; c += 128) s_x[c] = r.x[c0 + c];
        __syncthreads();
        if (i < r.n) {
            const double* a = r.A + i + (int64_t)c0 * r.lda;
            int c = 0;
            for (; c + 8 <= cn; c += 8) {
                double v[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) v[u] = a[(int64_t)(c + u) * r.lda];
#pragma unroll
                for (int u = 0; u < 8; ++u) acc[u & 3] = fma(v[u], s_x[c + u], acc[u & 3]);
            }
            for (; c < cn; ++c) acc[c & 3] = fma(a[(int64_t)c * r.lda], s_x[c], acc[c & 3]);
        }
    }
    if (i < r.n_pad) r.r[i] = i < r.n ? r.b[i] - ((acc[0] + acc[1]) + (acc[2] + acc[3])) : 0.0;
}

// rel = ||r|| / ||b|| per crack (fixed-order block reduction)
__global__ void __launch_bounds__(256) relres_group_kernel(const __grid_constant__ CrackGroup g)
{
    __shared__ double s_b[256], s_r[256];
    const CrackRec& r = g.rec[blockIdx.x];
    double bb = 0.0, rr = 0.0;
    for (int i = threadIdx.x; i < r.n; i += 256) {
        bb = fma(r.b[i], r.b[i], bb);
        rr = fma(r.r[i], r.r[i], rr);
    }
    s_b[threadIdx.x] = bb;
    s_r[threadIdx.x] = rr;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            s_b[threadIdx.x] += s_b[threadIdx.x + h];
            s_r[threadIdx.x] += s_r[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *r.rel = s_b[0] > 0.0 ? sqrt(s_r[0]) / sqrt(s_b[0]) : 0.0;
}

}  // namespace

namespace {

// every grouped launch over the cracks, kCrackGroupMax at a time
template <class F>
bool each_group(const std::vector<CrackRec>& cracks, int64_t* launches, F&& launch)
{
    CrackGroup g{};
    int nmax = 0;
    for (size_t p = 0; p <= cracks.size(); ++p) {
        if (g.count == kCrackGroupMax || (p == cracks.size() && g.count > 0)) {
            launch(g, nmax);
            if (launches) ++*launches;
            if (cudaGetLastError() != cudaSuccess) return false;
            g.count = 0;
            nmax = 0;
        }
        if (p < cracks.size()) {
            g.rec[g.count++] = cracks[p];
            nmax = cracks[p].n_pad > nmax ? cracks[p].n_pad : nmax;
        }
    }
    return true;
}

}  // namespace

int mixed_group_sweeps(const LuStreams& ls, const std::vector<CrackRec>& cracks, int* sync_all, size_t sync_ints,
                       int sweeps)
{
    if (cracks.empty()) return GMRES_OK;
    cudaStream_t st = ls.main;
    int64_t* L = ls.launches;
    const long wl = ls.wait_limit > 0 ? ls.wait_limit : kDefaultWaitLimit;
    for (int it = 0; it < sweeps; ++it) {
        if (cudaMemsetAsync(sync_all, 0, sync_ints * sizeof(int), st) != cudaSuccess) return GMRES_CUDA_ERROR;
        if (!each_group(cracks, L, [&](const CrackGroup& g, int nmax) {
                chain_group_kernel<false><<<dim3((unsigned)(nmax / kRB), g.count), kChainThreads, 0, st>>>(g, wl);
            }) ||
            !each_group(cracks, L, [&](const CrackGroup& g, int nmax) {
                chain_group_kernel<true><<<dim3((unsigned)(nmax / kRB), g.count), kChainThreads, 0, st>>>(g, wl);
            }) ||
            !each_group(cracks, L, [&](const CrackGroup& g, int nmax) {
                axpy_group_kernel<<<dim3((unsigned)((nmax + 255) / 256), g.count), 256, 0, st>>>(g);
            }) ||
            !each_group(cracks, L, [&](const CrackGroup& g, int nmax) {
                residual_group_kernel<<<dim3((unsigned)((nmax + 127) / 128), g.count), 128, 0, st>>>(g);
            }))
            return GMRES_CUDA_ERROR;
    }
    if (!each_group(cracks, L, [&](const CrackGroup& g, int) { relres_group_kernel<<<g.count, 256, 0, st>>>(g); }))
        return GMRES_CUDA_ERROR;
    return GMRES_OK;
}

int mixed_group_solve(const LuStreams& ls, const std::vector<CrackRec>& cracks, const std::vector<GroupSystem>& sys,
                      const CUtensorMap* dev_maps, int* infos, int* status, int* sync_all, size_t sync_ints,
                      int sweeps, int nb)
{
    if (cracks.empty()) return GMRES_OK;
    if (cracks.size() != sys.size()) return GMRES_CUDA_ERROR;
    cudaStream_t st = ls.main;
    int64_t* L = ls.launches;
    for (const auto& c : cracks)
        if (c.n_pad % kRB || c.n_pad < c.n) return GMRES_CUDA_ERROR;
    if (!each_group(cracks, L,
                    [&](const CrackGroup& g, int) { cast_pad_group_kernel<<<dim3(32, g.count), 256, 0, st>>>(g); }))
        return GMRES_CUDA_ERROR;
    if (lu_factor_group(ls, sys, dev_maps, infos, status, nb) != LU_OK) return GMRES_CUDA_ERROR;
    std::vector<int*> perms;
    for (const auto& c : cracks) perms.push_back(c.perm);
    if (lu_pivots_to_perm_group(st, sys, perms, L) != LU_OK) return GMRES_CUDA_ERROR;
    const size_t ismem = (size_t)(kRB * kRB + kRB * (kRB + 1)) * sizeof(float);
    if (cudaFuncSetAttribute(invert_group_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ismem) !=
        cudaSuccess)
        return GMRES_CUDA_ERROR;
    if (!each_group(cracks, L, [&](const CrackGroup& g, int nmax) {
            invert_group_kernel<<<dim3((unsigned)(nmax / kRB), g.count, 2), kRB, ismem, st>>>(g);
        }))
        return GMRES_CUDA_ERROR;
    if (!each_group(cracks, L, [&](const CrackGroup& g, int nmax) {
            init_group_kernel<<<dim3((unsigned)((nmax + 255) / 256), g.count), 256, 0, st>>>(g);
        }))
        return GMRES_CUDA_ERROR;
    return mixed_group_sweeps(ls, cracks, sync_all, sync_ints, sweeps);
}

}  // namespace cad
