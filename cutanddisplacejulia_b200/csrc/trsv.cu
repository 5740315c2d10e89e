// Single-right-hand-side FP64 solve with the LU factors (the solve half of
// the `A\b` of src/SlipCalculator3D.jl:22): x = U^-1 L^-1 P b as one launch
// per triangle instead of a 64-row diagonal solve plus a GEMV per block.
//
// Each CTA owns a 64-row block and takes its place in the dependency order
// from an atomic ticket (every block it waits for belongs to a CTA that took
// an earlier ticket, so it is already running).  It loads its diagonal block
// into shared memory and, for every block already solved, issues the loads of
// its off-diagonal 64 x 64 piece before waiting on that block's flag
// (release / acquire), then one warp solves the diagonal block by
// substitution -- the same operations as a row-block TRSV, no explicit
// inverse.  A wait that runs out sets info to -1 (reported as a timeout).
#include <cuda_runtime.h>

#include <cstdint>

#include "lu.h"

namespace cad {

namespace {

constexpr int kB = 64;            // rows per block
constexpr int kThreads = 256;     // four threads per row: quarters of each 64-column block
constexpr int kQ = kThreads / kB;
constexpr int kC = kB / kQ;       // 16 columns per quarter

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

// Lower (UPPER false): y = L^-1 (P b), b gathered through perm, pieces to y.
// Upper: x = U^-1 y, pieces to x.
template <bool UPPER>
__global__ void __launch_bounds__(kThreads) trsv_chain_f64_kernel(const double* __restrict__ A, int64_t lda, int n,
                                                                  int nblk, const double* __restrict__ b,
                                                                  const int* __restrict__ perm, double* y, double* x,
                                                                  int* flags, int* ticket, int* info,
                                                                  long wait_limit)
{
    __shared__ double s_d[kB][kB + 1];
    __shared__ double s_x[kB];
    __shared__ double s_part[kQ][kB];
    __shared__ double s_rinv[kB];
    __shared__ int s_t;
    const int tid = threadIdx.x, rr = tid % kB, q = tid / kB;
    if (tid == 0) s_t = atomicAdd(ticket, 1);
    __syncthreads();
    const int t = s_t;
    const int i = UPPER ? nblk - 1 - t : t;
    const int r0 = i * kB;
    const int rows = n - r0 < kB ? n - r0 : kB;
    const int row = r0 + rr;
    const bool rok = rr < rows;
    // the diagonal block (identity past n)
    for (int e = tid; e < kB * kB; e += kThreads) {
        const int r = e % kB, c = e / kB;
        s_d[r][c] = (r < rows && c < rows) ? A[(int64_t)(r0 + r) + (int64_t)(r0 + c) * lda] : (r == c ? 1.0 : 0.0);
    }
    __syncthreads();   // s_d complete before any thread reads it (a first block runs no waiting loop)
    double acc = 0.0;
    if (q == 0 && rok) acc = UPPER ? __ldcg(y + row) : b[perm[row]];
    const double* src = UPPER ? x : y;   // solved pieces of the other blocks
    for (int s = 0; s < t; ++s) {
        const int j = UPPER ? nblk - 1 - s : s;
        const int c0 = j * kB + q * kC;
        double a[kC];
#pragma unroll
        for (int c = 0; c < kC; ++c) a[c] = (rok && c0 + c < n) ? __ldg(A + row + (int64_t)(c0 + c) * lda) : 0.0;
        if (tid == 0) {
            long spins = 0;
            while (ld_acquire(flags + j) == 0) {
                if (++spins > wait_limit) {
                    atomicMin(info, -1);
                    break;
                }
                __nanosleep(32);
            }
        }
        __syncthreads();
        if (tid < kB) s_x[tid] = j * kB + tid < n ? __ldcg(src + j * kB + tid) : 0.0;
        __syncthreads();
        double p0 = 0.0, p1 = 0.0;
#pragma unroll
        for (int c = 0; c < kC; c += 2) {
            p0 = fma(a[c], s_x[q * kC + c], p0);
            p1 = fma(a[c + 1], s_x[q * kC + c + 1], p1);
        }
        acc -= p0 + p1;
    }
    s_part[q][rr] = acc;
    if (UPPER && tid < kB) s_rinv[tid] = 1.0 / s_d[tid][tid];
    __syncthreads();
    if (tid < 32) {
        const int l = tid;
        double v0 = 0.0, v1 = 0.0;
#pragma unroll
        for (int k = 0; k < kQ; ++k) {
            v0 += s_part[k][l];
            v1 += s_part[k][l + 32];
        }
        if (!UPPER) {
            for (int c = 0; c < kB; ++c) {   // unit lower: row c is final once reached
                const double xc = __shfl_sync(0xffffffffu, c < 32 ? v0 : v1, c & 31);
                if (l > c) v0 -= s_d[l][c] * xc;
                if (l + 32 > c) v1 -= s_d[l + 32][c] * xc;
            }
        } else {
            for (int c = kB - 1; c >= 0; --c) {
                const double xc = __shfl_sync(0xffffffffu, c < 32 ? v0 : v1, c & 31) * s_rinv[c];
                if (l == (c & 31)) {
                    if (c < 32) v0 = xc;
                    else v1 = xc;
                }
                if (l < c) v0 -= s_d[l][c] * xc;
                if (l + 32 < c) v1 -= s_d[l + 32][c] * xc;
            }
        }
        double* out = UPPER ? x : y;
        if (l < rows) out[r0 + l] = v0;
        if (l + 32 < rows) out[r0 + l + 32] = v1;
    }
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        st_release(flags + i, 1);
    }
}

}  // namespace

size_t lu_chain_sync_ints(int64_t n) { return (size_t)2 * ((n + kB - 1) / kB) + 2; }

cudaError_t lu_solve_chain_f64(cudaStream_t st, const double* A, int64_t lda, int64_t n, const int* perm,
                               const double* b, double* y, double* x, int* sync, int* info, int64_t* launches,
                               long wait_limit)
{
    if (wait_limit <= 0) wait_limit = kDefaultWaitLimit;
    if (n <= 0) return cudaSuccess;
    const int nblk = (int)((n + kB - 1) / kB);
    cudaError_t e = cudaMemsetAsync(sync, 0, lu_chain_sync_ints(n) * sizeof(int), st);
    if (e != cudaSuccess) return e;
    int* fl = sync;
    int* fu = sync + nblk;
    int* tk = sync + 2 * nblk;
    trsv_chain_f64_kernel<false><<<nblk, kThreads, 0, st>>>(A, lda, (int)n, nblk, b, perm, y, x, fl, tk, info,
                                                            wait_limit);
    trsv_chain_f64_kernel<true><<<nblk, kThreads, 0, st>>>(A, lda, (int)n, nblk, b, perm, y, x, fu, tk + 1, info,
                                                           wait_limit);
    if (launches) *launches += 2;
    return cudaGetLastError();
}

__global__ void set_ticket_kernel(int* ticket, int v) { *ticket = v; }

cudaError_t lu_chain_timeout_probe(cudaStream_t st, const double* A, int64_t lda, int64_t n, const int* perm,
                                   const double* b, double* y, double* x, int* sync, int* info, long wait_limit)
{
    const int nblk = (int)((n + kB - 1) / kB);
    if (nblk < 2 || wait_limit <= 0) return cudaErrorInvalidValue;
    cudaError_t e = cudaMemsetAsync(sync, 0, lu_chain_sync_ints(n) * sizeof(int), st);
    if (e != cudaSuccess) return e;
    int* tk = sync + 2 * nblk;
    set_ticket_kernel<<<1, 1, 0, st>>>(tk, 1);
    // tickets 1 .. nblk - 1: blocks 1 .. nblk - 1, none of which is block 0
    trsv_chain_f64_kernel<false><<<nblk - 1, kThreads, 0, st>>>(A, lda, (int)n, nblk, b, perm, y, x, sync, tk, info,
                                                                wait_limit);
    return cudaGetLastError();
}

}  // namespace cad
