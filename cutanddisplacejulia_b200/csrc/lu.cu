// Dense LU with partial pivoting and triangular solves (the `A\b` of
// SlipCalculator3D, src/SlipCalculator3D.jl:22) for sm_100a.
//
// Right-looking blocked LU (outer block nb).  Each nb-wide panel is factorised
// recursively: the left half, then a row swap, a triangular solve and a GEMM
// update of the right half, then the right half.  The recursion stops at
// narrow leaves that one thread-block cluster factorises with its rows held in
// distributed shared memory: per column, every CTA proposes its largest
// |entry|, the cluster agrees on the pivot through DSMEM, the pivot row and the
// displaced row are exchanged through DSMEM, and every CTA updates its own rows
// -- two hardware cluster barriers per column, no global-memory spin.  Rank-nb
// trailing updates and the intra-panel updates are the library's own tensor-
// core GEMMs (csrc/gemm.cu: DMMA tiles in FP64; tcgen05 TF32 with TMA-staged
// operands for the single-precision factorisation).
//
// Pivot choice is LAPACK's: the first row of largest magnitude; scaling by the
// reciprocal pivot; ipiv[k] = absolute row swapped with row k.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <mutex>
#include <cstdint>
#include <vector>

#include "gemm.h"
#include "lu.h"

namespace cg = cooperative_groups;

namespace cad {

namespace {

constexpr int kLeafThreads = 512;
constexpr int kLeafWarps = kLeafThreads / 32;
constexpr int kMaxCluster = 16;
constexpr int kLeafRegs = 32;   // row values one leaf thread keeps in registers (RPT * W)
constexpr int kMaxSwaps = 256;   // pivots one row-swap launch applies
constexpr int kMaxBlock = 1024;  // widest outer block of lu_factor_solve
constexpr int kMaxDevices = 64;  // devices whose leaf cluster size is remembered

// ---------------------------------------------- records of grouped launches
// One launch of a grouped factorisation (many independent FP32 systems) takes
// its per-system arguments by value as a kernel parameter (up to 32 KB), one
// record per system; grid dimension y selects the record.
constexpr int kGroupMax = 512;   // records per grouped launch
struct LeafRec {
    float* A;     // panel top
    int* piv;     // pivots of the panel's columns
    int* info;
    int lda, m, piv_base, col_base;
};
struct LeafGroup {
    int count, w;
    long wait_limit;
    LeafRec rec[kGroupMax];
};
struct LaswpRec {
    float *A1, *A2;
    const int* piv;
    int lda, ncol1, ncol2, row_base;
};
struct LaswpGroup {
    int count, npiv;
    LaswpRec rec[kGroupMax];
};
struct TrsmRec {
    const float* L;
    float* B;
    int ldl, ldb, ncol, pad;
};
struct TrsmGroup {
    int count, b;
    TrsmRec rec[kGroupMax];
};
static_assert(sizeof(LeafGroup) <= 32000 && sizeof(LaswpGroup) <= 32000 && sizeof(TrsmGroup) <= 32000,
              "grouped launch records exceed the kernel parameter space");

// A pivot candidate as integers: |value| orders like the bit pattern of the
// non-negative double, so hi = 1 + its high word (0: no candidate), lo = its
// low word; ties go to the smaller position (LAPACK's first largest entry).
struct __align__(16) Key {
    unsigned hi, lo, pos, who;
};
__device__ __forceinline__ bool key_better(const Key& a, const Key& b)
{
    return a.hi > b.hi || (a.hi == b.hi && (a.lo > b.lo || (a.lo == b.lo && a.pos < b.pos)));
}
__device__ __forceinline__ Key key_of(double v, int pos, unsigned who)
{
    const unsigned long long bits = (unsigned long long)__double_as_longlong(fabs(v));
    return Key{(unsigned)(bits >> 32) + 1u, (unsigned)bits, (unsigned)pos, who};
}
// the warp's best key in every lane: three integer warp reductions instead of
// a shuffle tree of double compares
__device__ __forceinline__ Key warp_key_max(const Key& k)
{
    const unsigned full = 0xffffffffu;
    const unsigned mhi = __reduce_max_sync(full, k.hi);
    const unsigned mlo = __reduce_max_sync(full, k.hi == mhi ? k.lo : 0u);
    const bool tie = k.hi == mhi && k.lo == mlo;
    const unsigned mpos = __reduce_min_sync(full, tie ? k.pos : 0xffffffffu);
    const unsigned win = __ballot_sync(full, tie && k.pos == mpos);
    return Key{mhi, mlo, mpos, __shfl_sync(full, k.who, __ffs(win) - 1)};
}

// ------------------------------------------------------------ leaf (cluster)
// DSMEM pushes: st.async stores into another CTA's shared memory that count
// their bytes on that CTA's mbarrier, so a receiver waits on its own barrier
// for exactly the bytes it expects -- no cluster-wide barrier (whose
// release/acquire fence costs about a microsecond) per column.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned cluster_map(unsigned addr, unsigned rank)
{
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
    return r;
}
__device__ __forceinline__ void st_async_b64(unsigned addr, unsigned long long v, unsigned mbar)
{
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b64 [%0], %1, [%2];" ::"r"(addr), "l"(v), "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void st_async_b32(unsigned addr, unsigned v, unsigned mbar)
{
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];" ::"r"(addr), "r"(v), "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void st_async_word(unsigned addr, double v, unsigned mbar)
{
    st_async_b64(addr, (unsigned long long)__double_as_longlong(v), mbar);
}
__device__ __forceinline__ void st_async_word(unsigned addr, float v, unsigned mbar)
{
    st_async_b32(addr, __float_as_uint(v), mbar);
}
__device__ __forceinline__ void st_async_v4(unsigned addr, unsigned a, unsigned b, unsigned c, unsigned d, unsigned mbar)
{
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(addr),
                 "r"(a), "r"(b), "r"(c), "r"(d), "r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void mbar_init(unsigned mbar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect(unsigned mbar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned mbar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0u;
}

// Factorises the m x w panel at A (leading dimension lda, w <= W) in place.
// CTA q of the cluster owns panel rows [q*R, (q+1)*R), R = 512 * RPT; thread t
// keeps rows t + 512*k (k < RPT) in registers for the whole leaf and never
// moves them -- each row carries its current logical position.  Per column j:
// every warp reduces its candidates, every warp then reduces the 16 warp
// results, and one warp pushes the CTA's best row, the reciprocal of its pivot
// entry and its key into slot [j & 1][q] of every CTA of the cluster; each CTA
// waits on its own barrier for the C payloads, picks the pivot and updates its
// rows from the pivot row in shared memory.  Two slots suffice: a CTA pushes
// column j + 2 only after every CTA's column j + 1 payload reached it, and a
// CTA sends that payload only once all its threads are done with column j.
// Rows are stored to their final positions at the end.  piv[c] = piv_base +
// position swapped with c (LAPACK order); info: smallest zero-pivot column
// (1-based, + col_base), or -1 if a wait ran out.
template <typename T, int W, int RPT>
__device__ __forceinline__ void leaf_body(T* __restrict__ A, int64_t lda, int m, int w, int* __restrict__ piv,
                                          int piv_base, int* __restrict__ info, int col_base, long wait_limit)
{
    static_assert(W * RPT <= kLeafRegs && W <= 32, "leaf tile exceeds its register budget");
    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank();
    const int C = (int)cluster.num_blocks();
    __shared__ __align__(16) T s_row[2][kMaxCluster][W];
    __shared__ __align__(16) T s_rinv[2][kMaxCluster];
    __shared__ __align__(16) Key s_ckey[2][kMaxCluster];
    __shared__ __align__(8) unsigned long long s_bar[2];
    __shared__ Key s_wkey[2][kLeafWarps];   // by column parity: a fast warp may write column j + 1's
                                            // while a slow one still reads column j's
    __shared__ int s_hist[W];
    __shared__ int s_fail;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // bytes one column delivers to each CTA: C rows, reciprocals and keys
    const unsigned col_bytes = (unsigned)C * (unsigned)(W * sizeof(T) + sizeof(T) + sizeof(Key));
    if (tid == 0) {
        s_fail = 0;
        mbar_init(smem_u32(&s_bar[0]), 1);
        mbar_init(smem_u32(&s_bar[1]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        mbar_arrive_expect(smem_u32(&s_bar[0]), col_bytes);
        if (w > 1) mbar_arrive_expect(smem_u32(&s_bar[1]), col_bytes);
    }
    T x[RPT][W];
    int pos[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
        const int row = crank * (kLeafThreads * RPT) + k * kLeafThreads + tid;
        pos[k] = row < m ? row : INT_MAX;
#pragma unroll
        for (int c = 0; c < W; ++c)
            x[k][c] = (row < m && c < w) ? A[(int64_t)row + (int64_t)c * lda] : (T)0;
    }
    cluster.sync();   // barriers initialised and every CTA running before the first push

#pragma unroll
    for (int j = 0; j < W; ++j) {
        if (j >= w) break;
        const int par = j & 1;
        Key key{0u, 0u, 0xffffffffu, 0u};
        T piv_val = (T)0;
#pragma unroll
        for (int k = 0; k < RPT; ++k)
            if (pos[k] != INT_MAX && pos[k] >= j) {
                const Key kk = key_of((double)x[k][j], pos[k], (unsigned)((k << 10) | tid));
                if (key_better(kk, key)) {
                    key = kk;
                    piv_val = x[k][j];
                }
            }
        const T inv_c = piv_val != (T)0 ? (T)1 / piv_val : (T)0;
        const Key wk = warp_key_max(key);
        if (lane == 0) s_wkey[par][warp] = wk;
        __syncthreads();
        const Key b = warp_key_max(lane < kLeafWarps ? s_wkey[par][lane] : Key{0u, 0u, 0xffffffffu, 0u});
        // one warp pushes this CTA's payload for column j to every CTA: the
        // best row (zeros if none), its reciprocal and its key
        const int pusher = b.hi != 0u ? (int)((b.who & 1023u) >> 5) : 0;
        if (warp == pusher) {
            const int src = (int)(b.who & 31u), kk = (int)(b.who >> 10);
            T mine = (T)0;
#pragma unroll
            for (int cc = 0; cc < W; ++cc) {
                T v = x[0][cc];
#pragma unroll
                for (int k = 1; k < RPT; ++k)
                    if (k == kk) v = x[k][cc];
                v = __shfl_sync(0xffffffffu, v, src);
                if (lane == cc) mine = v;
            }
            T rinv = __shfl_sync(0xffffffffu, inv_c, src);
            if (b.hi == 0u) mine = rinv = (T)0;
            const unsigned bar = smem_u32(&s_bar[par]);
            const unsigned row_addr = smem_u32(&s_row[par][crank][lane]);
            const unsigned rinv_addr = smem_u32(&s_rinv[par][crank]);
            const unsigned key_addr = smem_u32(&s_ckey[par][crank]);
            for (int q = 0; q < C; ++q) {
                const unsigned rbar = cluster_map(bar, (unsigned)q);
                if (lane < W)
                    st_async_word(cluster_map(row_addr, (unsigned)q), mine, rbar);
            }
            if (lane < C) {
                const unsigned rbar = cluster_map(bar, (unsigned)lane);
                st_async_word(cluster_map(rinv_addr, (unsigned)lane), rinv, rbar);
                st_async_v4(cluster_map(key_addr, (unsigned)lane), b.hi, b.lo, b.pos, b.who, rbar);
            }
        }
        // wait for the C payloads of column j
        {
            const unsigned bar = smem_u32(&s_bar[par]);
            const unsigned parity = (unsigned)((j >> 1) & 1);
            long spins = 0;
            while (!mbar_try_wait(bar, parity))
                if (++spins > (wait_limit >> 2)) {   // a try_wait round may suspend briefly
                    s_fail = 1;
                    break;
                }
        }
        __syncwarp();
        if (tid == 0 && j + 2 < w) mbar_arrive_expect(smem_u32(&s_bar[par]), col_bytes);
        Key g = lane < C ? s_ckey[par][lane] : Key{0u, 0u, 0xffffffffu, 0u};
        g.who = (unsigned)lane;
        g = warp_key_max(g);
        const bool ok = g.hi > 1u || (g.hi == 1u && g.lo != 0u);
        const int p = ok ? (int)g.pos : j;
        if (tid == 0) {
            s_hist[j] = p;
            if (!ok && crank == 0) atomicMin(info, col_base + j + 1);
        }
        if (ok) {
            const T* u = s_row[par][g.who];
            const T inv = s_rinv[par][g.who];
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                int ps = pos[k];
                if (ps == p) ps = j;
                else if (ps == j) ps = p;
                pos[k] = ps;
                if (ps != INT_MAX && ps > j) {
                    const T l = x[k][j] * inv;
                    x[k][j] = l;
#pragma unroll
                    for (int cc = j + 1; cc < W; ++cc) x[k][cc] -= l * u[cc];
                }
            }
        }
    }
    cluster.sync();   // every push has landed and been read before any CTA exits
#pragma unroll
    for (int k = 0; k < RPT; ++k)
        if (pos[k] != INT_MAX)
#pragma unroll
            for (int c = 0; c < W; ++c)
                if (c < w) A[(int64_t)pos[k] + (int64_t)c * lda] = x[k][c];
    __syncthreads();
    if (crank == 0 && tid < w) piv[tid] = piv_base + s_hist[tid];
    if (tid == 0 && s_fail) atomicMin(info, -1);
}

template <typename T, int W, int RPT>
__global__ void __launch_bounds__(kLeafThreads, 1) leaf_lu_kernel(T* __restrict__ A, int64_t lda, int m, int w,
                                                                int* __restrict__ piv, int piv_base,
                                                                int* __restrict__ info, int col_base,
                                                                long wait_limit)
{
    leaf_body<T, W, RPT>(A, lda, m, w, piv, piv_base, info, col_base, wait_limit);
}

// The leaves of many systems in one launch: cluster y of the grid factorises
// the panel of record y (every cluster of the launch has the same size, so the
// records of one launch need the same number of CTAs).
template <int W, int RPT>
__global__ void __launch_bounds__(kLeafThreads, 1) leaf_group_kernel(const __grid_constant__ LeafGroup g)
{
    const LeafRec& r = g.rec[blockIdx.y];
    leaf_body<float, W, RPT>(r.A, r.lda, r.m, g.w, r.piv, r.piv_base, r.info, r.col_base, g.wait_limit);
}

// ------------------------------------------------------------ row swaps
// Applies the swaps row k <-> row piv[k] - row_base (k = 0..npiv-1, in order,
// rows relative to the block top) to columns [0, ncol1) of A1 and [0, ncol2)
// of A2.  Every CTA first derives the net movement: each touched row follows
// its content through the swap sequence, giving at most 2 * npiv (dst, src)
// pairs; then one warp per column gathers the sources and stores them.
template <typename T>
__device__ __forceinline__ void laswp_body(T* __restrict__ A1, int ncol1, T* __restrict__ A2, int ncol2, int64_t lda,
                                           const int* __restrict__ piv, int npiv, int row_base, int cta, int ncta)
{
    constexpr int kPer = 2 * kMaxSwaps / 32;
    __shared__ int s_piv[kMaxSwaps];
    __shared__ int s_dst[2 * kMaxSwaps], s_src[2 * kMaxSwaps];
    __shared__ int s_count;
    for (int k = threadIdx.x; k < npiv; k += blockDim.x) s_piv[k] = piv[k] - row_base;
    if (threadIdx.x == 0) s_count = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < 2 * npiv; t += blockDim.x) {
        int row = t;
        bool track = true;
        if (t >= npiv) {   // a pivot row below the block's first npiv rows, tracked once
            const int kk = t - npiv;
            row = s_piv[kk];
            track = row >= npiv;
            for (int k = 0; k < kk && track; ++k) track = s_piv[k] != row;
        }
        if (!track) continue;
        int at = row;
        for (int k = 0; k < npiv; ++k) {
            const int q = s_piv[k];
            at = at == k ? q : (at == q ? k : at);
        }
        if (at != row) {
            const int slot = atomicAdd(&s_count, 1);
            s_dst[slot] = at;
            s_src[slot] = row;
        }
    }
    __syncthreads();
    const int count = s_count;
    if (count == 0) return;
    const int lane = threadIdx.x & 31;
    int dst[kPer], src[kPer];
#pragma unroll
    for (int t = 0; t < kPer; ++t) {
        const int e = lane + 32 * t;
        dst[t] = e < count ? s_dst[e] : -1;
        src[t] = e < count ? s_src[e] : 0;
    }
    const int wid = (cta * blockDim.x + threadIdx.x) >> 5;
    const int nw = (ncta * blockDim.x) >> 5;
    for (int col = wid; col < ncol1 + ncol2; col += nw) {
        T* a = col < ncol1 ? A1 + (int64_t)col * lda : A2 + (int64_t)(col - ncol1) * lda;
        T v[kPer];
#pragma unroll
        for (int t = 0; t < kPer; ++t) v[t] = dst[t] >= 0 ? a[src[t]] : (T)0;
        __syncwarp();
#pragma unroll
        for (int t = 0; t < kPer; ++t)
            if (dst[t] >= 0) a[dst[t]] = v[t];
        __syncwarp();
    }
}

template <typename T>
__global__ void __launch_bounds__(256) laswp_kernel(T* __restrict__ A1, int ncol1, T* __restrict__ A2, int ncol2,
                                                    int64_t lda, const int* __restrict__ piv, int npiv, int row_base)
{
    laswp_body<T>(A1, ncol1, A2, ncol2, lda, piv, npiv, row_base, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(256) laswp_group_kernel(const __grid_constant__ LaswpGroup g)
{
    const LaswpRec& r = g.rec[blockIdx.y];
    laswp_body<float>(r.A1, r.ncol1, r.A2, r.ncol2, r.lda, r.piv, g.npiv, r.row_base, blockIdx.x, gridDim.x);
}

// ------------------------------------------------- triangular diagonal blocks
// B (b x ncol, ldb) := L^-1 B with L the b x b unit lower triangle at L (ldl),
// or U^-1 B with U upper, non-unit; b <= 64.  A CTA of 4 warps takes 32
// columns (8 per warp); lane l holds rows l and l + 32; the solved row c is
// broadcast from its lane by shuffles.
template <typename T, bool UPPER>
__device__ __forceinline__ void trsm_diag_body(const T* __restrict__ L, int64_t ldl, int b, T* __restrict__ B,
                                               int64_t ldb, int ncol, int cta)
{
    __shared__ T s_L[64 * 64];
    __shared__ T s_inv[64];   // UPPER: reciprocal diagonal
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int col0 = cta * 32 + warp * 8;
    if (cta * 32 >= ncol) return;   // CTA-uniform: a grouped launch sizes x for its widest record
    {
        // every load of the block and of the right-hand sides in flight at once
        T t[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int e = threadIdx.x + 128 * i, r = e & 63, c = e >> 6;
            t[i] = (r < b && c < b) ? L[r + (int64_t)c * ldl] : (T)0;
        }
#pragma unroll
        for (int i = 0; i < 32; ++i) s_L[threadIdx.x + 128 * i] = t[i];
    }
    T x[2][8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = lane + 32 * h, col = col0 + k;
            x[h][k] = (r < b && col < ncol) ? B[r + (int64_t)col * ldb] : (T)0;
        }
    __syncthreads();
    if (UPPER && threadIdx.x < 64) s_inv[threadIdx.x] = threadIdx.x < b ? (T)1 / s_L[threadIdx.x * 65] : (T)1;
    if (UPPER) __syncthreads();
    // row c = 32 * hc + cc is solved, then broadcast from lane cc; the loop
    // over cc stays rolled (a fully unrolled 64-step solve overflows the
    // instruction cache), the register half hc is static
    if (!UPPER) {
#pragma unroll
        for (int hc = 0; hc < 2; ++hc)
#pragma unroll 2
            for (int cc = 0; cc < 32; ++cc) {
                const int c = 32 * hc + cc;
                if (c >= b) break;
                const T l0 = s_L[c * 64 + lane], l1 = s_L[c * 64 + 32 + lane];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const T xc = __shfl_sync(0xffffffffu, x[hc][k], cc);
                    if (hc == 0 && lane > c) x[0][k] -= l0 * xc;
                    if (32 + lane > c) x[1][k] -= l1 * xc;
                }
            }
    } else {
#pragma unroll
        for (int hc = 1; hc >= 0; --hc)
#pragma unroll 2
            for (int cc = 31; cc >= 0; --cc) {
                const int c = 32 * hc + cc;
                if (c >= b) continue;
                const T d = s_inv[c], u0 = s_L[c * 64 + lane], u1 = s_L[c * 64 + 32 + lane];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const T xc = __shfl_sync(0xffffffffu, x[hc][k], cc) * d;
                    if (lane == cc) x[hc][k] = xc;
                    if (lane < c) x[0][k] -= u0 * xc;
                    if (hc == 1 && 32 + lane < c) x[1][k] -= u1 * xc;
                }
            }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = lane + 32 * h, col = col0 + k;
            if (r < b && col < ncol) B[r + (int64_t)col * ldb] = x[h][k];
        }
}

template <typename T, bool UPPER>
__global__ void __launch_bounds__(128) trsm_diag_kernel(const T* __restrict__ L, int64_t ldl, int b, T* __restrict__ B,
                                                        int64_t ldb, int ncol)
{
    trsm_diag_body<T, UPPER>(L, ldl, b, B, ldb, ncol, blockIdx.x);
}

__global__ void __launch_bounds__(128) trsm_group_kernel(const __grid_constant__ TrsmGroup g)
{
    const TrsmRec& r = g.rec[blockIdx.y];
    trsm_diag_body<float, false>(r.L, r.ldl, g.b, r.B, r.ldb, r.ncol, blockIdx.x);
}

// perm[i] = source row of row i after all n pivots (ipiv applied in order),
// built by one thread in shared memory.
__global__ void pivots_to_perm_kernel(const int* __restrict__ ipiv, int n, int* __restrict__ perm)
{
    extern __shared__ int s_perm[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_perm[i] = i;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < n; ++k) {
            const int q = ipiv[k];
            const int t = s_perm[k];
            s_perm[k] = s_perm[q];
            s_perm[q] = t;
        }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = s_perm[i];
}

// The same in global memory, for n beyond what shared memory holds.
__global__ void pivots_to_perm_global_kernel(const int* __restrict__ ipiv, int n, int* __restrict__ perm)
{
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = i;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < n; ++k) {
            const int q = ipiv[k];
            const int t = perm[k];
            perm[k] = perm[q];
            perm[q] = t;
        }
}

// perm from ipiv on stream st (shared-memory kernel where n ints fit)
cudaError_t launch_pivots_to_perm(cudaStream_t st, const int* ipiv, int64_t n, int* perm)
{
    if (n <= 0) return cudaSuccess;
    int dev = 0, smem_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t psmem = (size_t)n * sizeof(int);
    if (psmem <= (size_t)smem_optin) {
        cudaError_t e = cudaFuncSetAttribute(pivots_to_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)psmem);
        if (e != cudaSuccess) return e;
        pivots_to_perm_kernel<<<1, 1024, psmem, st>>>(ipiv, (int)n, perm);
    } else {
        pivots_to_perm_global_kernel<<<1, 1024, 0, st>>>(ipiv, (int)n, perm);
    }
    return cudaGetLastError();
}

// Y[i, c] = X[perm[i], c]
template <typename T>
__global__ void permute_rows_kernel(const T* __restrict__ X, int64_t ldx, const int* __restrict__ perm, int n,
                                    int ncol, T* __restrict__ Y, int64_t ldy)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (i < n && c < ncol) Y[i + (int64_t)c * ldy] = X[perm[i] + (int64_t)c * ldx];
}

__global__ void set_int_kernel(int* p, int v) { *p = v; }

template <typename T>
struct Lu {
    cudaStream_t st;   // the stream the next launches go to
    cudaStream_t main_st, side_st;
    int* ipiv;    // absolute pivots, device
    int* info;
    int cluster;  // largest leaf cluster (16 where the device co-schedules it, else 8)
    long wait_limit = kDefaultWaitLimit;   // try_wait rounds before a leaf gives up on a push
    int min_rpt = 1;        // fewest rows per leaf thread (wider leaves with fewer rows each)
    int64_t launches = 0;   // own kernels launched
    cudaError_t err = cudaSuccess;

    bool ok() const { return err == cudaSuccess; }

    // C (m x n) -= A (m x k) * B (k x n) on the current stream
    void gemm(int m, int n, int k, const T* A, int64_t lda, const T* B, int64_t ldb, T* C, int64_t ldc)
    {
        if (!ok() || m <= 0 || n <= 0 || k <= 0) return;
        err = gemm_sub(st, m, n, k, A, lda, B, ldb, C, ldc, info);
        ++launches;
    }

    // rows per leaf thread for an m-row panel: the fewest that fit one cluster
    int leaf_rpt(int m) const
    {
        int rpt = min_rpt;
        while (rpt < 8 && (int64_t)cluster * kLeafThreads * rpt < m) rpt *= 2;
        return rpt;
    }
    int leaf_width(int m) const { return kLeafRegs / leaf_rpt(m); }

    // swaps rows k <-> piv[k] - row_base (k < npiv, in order) of the column
    // blocks (A1, ncol1) and (A2, ncol2), both relative to the same block top
    void laswp(const int* piv, int npiv, int row_base, T* A1, int ncol1, T* A2, int ncol2, int64_t lda)
    {
        if (npiv <= 0 || ncol1 + ncol2 <= 0 || !ok()) return;
        if (npiv > kMaxSwaps) {   // in order, kMaxSwaps swaps per launch (block tops moved down)
            for (int c0 = 0; c0 < npiv; c0 += kMaxSwaps)
                laswp(piv + c0, npiv - c0 < kMaxSwaps ? npiv - c0 : kMaxSwaps, row_base + c0, A1 ? A1 + c0 : nullptr,
                      ncol1, A2 ? A2 + c0 : nullptr, ncol2, lda);
            return;
        }
        const int ncol = ncol1 + ncol2;
        const int blocks = (ncol + 7) / 8 < 148 * 2 ? (ncol + 7) / 8 : 148 * 2;
        laswp_kernel<T><<<blocks, 256, 0, st>>>(A1, ncol1, A2, ncol2, lda, piv, npiv, row_base);
        ++launches;
        err = cudaGetLastError();
    }

    // B (b x ncol) := L^-1 B, L unit lower b x b (b arbitrary): 64-row blocks + GEMM
    void trsm_lower(const T* L, int64_t ldl, int b, T* B, int64_t ldb, int ncol)
    {
        for (int d = 0; d < b && ok(); d += 64) {
            const int db = b - d < 64 ? b - d : 64;
            trsm_diag_kernel<T, false><<<(ncol + 31) / 32, 128, 0, st>>>(L + d + d * ldl, ldl, db, B + d, ldb, ncol);
            ++launches;
            err = cudaGetLastError();
            if (d + db < b) gemm(b - d - db, ncol, db, L + (d + db) + d * ldl, ldl, B + d, ldb, B + d + db, ldb);
        }
    }

    template <int W, int RPT>
    void leaf_launch(T* A, int64_t lda, int m, int w, int* piv, int piv_base, int col_base)
    {
        const int C = (m + kLeafThreads * RPT - 1) / (kLeafThreads * RPT);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(C);
        cfg.blockDim = dim3(kLeafThreads);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = C;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        err = cudaLaunchKernelEx(&cfg, leaf_lu_kernel<T, W, RPT>, A, lda, m, w, piv, piv_base, info, col_base,
                                 wait_limit);
        ++launches;
    }

    void leaf(T* A, int64_t lda, int m, int w, int* piv, int piv_base, int col_base)
    {
        if (!ok()) return;
        switch (leaf_rpt(m)) {
            case 1: leaf_launch<32, 1>(A, lda, m, w, piv, piv_base, col_base); break;
            case 2: leaf_launch<16, 2>(A, lda, m, w, piv, piv_base, col_base); break;
            case 4: leaf_launch<8, 4>(A, lda, m, w, piv, piv_base, col_base); break;
            default: leaf_launch<4, 8>(A, lda, m, w, piv, piv_base, col_base); break;
        }
    }

    // m x w panel at A; its pivots (relative to the panel top, + piv_base) go to piv[0..w)
    void panel(T* A, int64_t lda, int m, int w, int* piv, int piv_base, int col_base)
    {
        if (!ok()) return;
        const int lw = leaf_width(m);
        if (w <= lw) {
            leaf(A, lda, m, w, piv, piv_base, col_base);
            return;
        }
        int w1 = w / 2;
        w1 = (w1 + lw - 1) / lw * lw;
        if (w1 >= w) w1 = w - lw;
        panel(A, lda, m, w1, piv, piv_base, col_base);
        laswp(piv, w1, piv_base, A + w1 * lda, w - w1, nullptr, 0, lda);
        trsm_lower(A, lda, w1, A + w1 * lda, lda, w - w1);
        if (m > w1) gemm(m - w1, w - w1, w1, A + w1, lda, A + w1 * lda, lda, A + w1 + w1 * lda, lda);
        panel(A + w1 + w1 * lda, lda, m - w1, w - w1, piv + w1, piv_base + w1, col_base + w1);
        // the right half's pivots (rows w1.. of the panel) applied to the left half's columns
        laswp(piv + w1, w - w1, piv_base + w1, A + w1, w1, nullptr, 0, lda);
    }

    void use(bool side) { st = side ? side_st : main_st; }

    // Right-looking blocked LU with a look-ahead of one block column.  Block
    // b's update is split: the main stream swaps, solves and updates block
    // column b + 1 only, then factorises it as the next panel; the side stream
    // meanwhile swaps, solves and updates the remaining columns.  The panel is
    // latency-bound on a few SMs, the trailing GEMM fills the rest.  Events:
    // panel[b] (block column b factorised; its pivots exist), rest[b] (side
    // work of block b done -- the main stream waits for it before touching
    // block column b + 2 or swapping rows of the L columns the side GEMM reads).
    void factor(T* A, int64_t n, int64_t lda, int nb)
    {
        use(false);
        set_int_kernel<<<1, 1, 0, st>>>(info, INT_MAX);
        ++launches;
        err = cudaGetLastError();
        const int nblk = (int)((n + nb - 1) / nb);
        if (nblk == 0 || !ok()) return;
        std::vector<cudaEvent_t> ev_panel(nblk, nullptr), ev_rest(nblk, nullptr);
        for (int b = 0; b < nblk && ok(); ++b) {
            err = cudaEventCreateWithFlags(&ev_panel[b], cudaEventDisableTiming);
            if (ok()) err = cudaEventCreateWithFlags(&ev_rest[b], cudaEventDisableTiming);
        }
        if (ok()) {
            const int kb0 = (int)(n < nb ? n : nb);
            panel(A, lda, (int)n, kb0, ipiv, 0, 0);
            if (ok()) err = cudaEventRecord(ev_panel[0], main_st);
        }
        for (int b = 0; b < nblk && ok(); ++b) {
            const int64_t k = (int64_t)b * nb;
            const int kb = (int)(n - k < nb ? n - k : nb);
            const int64_t k1 = k + kb;                                  // next block column
            const int kb1 = (int)(n - k1 < nb ? n - k1 : nb);
            const int64_t k2 = k1 + kb1;                                // the rest
            const int nr2 = (int)(n - k2);
            T* Akk = A + k + k * lda;
            // main: swaps left of the panel and in the next block column, its
            // solve and update, then the next panel
            use(false);
            if (b > 0) err = cudaStreamWaitEvent(main_st, ev_rest[b - 1], 0);
            laswp(ipiv + k, kb, (int)k, A + k, (int)k, A + k + k1 * lda, kb1, lda);
            if (kb1 > 0) {
                trsm_lower(Akk, lda, kb, A + k + k1 * lda, lda, kb1);
                gemm((int)(n - k1), kb1, kb, A + k1 + k * lda, lda, A + k + k1 * lda, lda, A + k1 + k1 * lda, lda);
                panel(A + k1 + k1 * lda, lda, (int)(n - k1), kb1, ipiv + k1, (int)k1, (int)k1);
                if (ok()) err = cudaEventRecord(ev_panel[b + 1], main_st);
            }
            // side: the same for the remaining block columns
            use(true);
            if (nr2 > 0 && ok()) {
                err = cudaStreamWaitEvent(side_st, ev_panel[b], 0);
                laswp(ipiv + k, kb, (int)k, A + k + k2 * lda, nr2, nullptr, 0, lda);
                trsm_lower(Akk, lda, kb, A + k + k2 * lda, lda, nr2);
                gemm((int)(n - k1), nr2, kb, A + k1 + k * lda, lda, A + k + k2 * lda, lda, A + k1 + k2 * lda, lda);
            }
            if (ok()) err = cudaEventRecord(ev_rest[b], side_st);
        }
        use(false);
        if (ok()) err = cudaStreamWaitEvent(main_st, ev_rest[nblk - 1], 0);
        for (int b = 0; b < nblk; ++b) {
            if (ev_panel[b]) cudaEventDestroy(ev_panel[b]);
            if (ev_rest[b]) cudaEventDestroy(ev_rest[b]);
        }
    }

    // X (n x nrhs) := A^-1 B with the factors in A; perm: n ints
    void solve(const T* A, int64_t n, int64_t lda, const T* B, int64_t ldb, int nrhs, T* X, int64_t ldx, int* perm)
    {
        if (!ok()) return;
        err = launch_pivots_to_perm(st, ipiv, n, perm);
        ++launches;
        if (!ok()) return;
        permute_rows_kernel<T><<<dim3((unsigned)((n + 255) / 256), nrhs), 256, 0, st>>>(B, ldb, perm, (int)n, nrhs, X,
                                                                                        ldx);
        ++launches;
        err = cudaGetLastError();
        // forward: L y = P b (unit lower), 64-row blocks
        for (int64_t d = 0; d < n && ok(); d += 64) {
            const int db = (int)(n - d < 64 ? n - d : 64);
            trsm_diag_kernel<T, false><<<(nrhs + 31) / 32, 128, 0, st>>>(A + d + d * lda, lda, db, X + d, ldx, nrhs);
            ++launches;
            err = cudaGetLastError();
            if (d + db < n) gemm((int)(n - d - db), nrhs, db, A + (d + db) + d * lda, lda, X + d, ldx, X + d + db, ldx);
        }
        // backward: U x = y, 64-row blocks from the bottom
        for (int64_t e = n; e > 0 && ok(); e -= 64) {
            const int64_t d = e - 64 > 0 ? e - 64 : 0;
            const int db = (int)(e - d);
            trsm_diag_kernel<T, true><<<(nrhs + 31) / 32, 128, 0, st>>>(A + d + d * lda, lda, db, X + d, ldx, nrhs);
            ++launches;
            err = cudaGetLastError();
            if (d > 0) gemm((int)d, nrhs, db, A + d * lda, lda, X + d, ldx, X, ldx);
        }
    }
};

template <typename T, int W, int RPT>
void allow_wide_clusters()
{
    cudaFuncSetAttribute(leaf_lu_kernel<T, W, RPT>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

// largest leaf cluster the device co-schedules: 16 CTAs (non-portable) or 8;
// worked out once per device and precision
template <typename T>
int configure(Lu<T>& lu)
{
    static std::atomic<int> known[kMaxDevices];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) dev = -1;
    if (dev >= 0) {
        const int c = known[dev].load();
        if (c) {
            lu.cluster = c;
            return 0;
        }
    }
    allow_wide_clusters<T, 32, 1>();
    allow_wide_clusters<T, 16, 2>();
    allow_wide_clusters<T, 8, 4>();
    allow_wide_clusters<T, 4, 8>();
    lu.cluster = 16;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16);
    cfg.blockDim = dim3(kLeafThreads);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 16;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, leaf_lu_kernel<T, 32, 1>, &cfg) != cudaSuccess || nclusters < 1) {
        cudaGetLastError();
        lu.cluster = 8;
    }
    if (dev >= 0) known[dev].store(lu.cluster);
    return 0;
}

// ------------------------------------------------------------ graph cache
struct LuGraphKey {
    int type;   // sizeof(T)
    const void *A, *B, *X;
    int64_t n, lda, ldb, ldx;
    int nrhs, nb;
    const int *ipiv, *perm, *info;
    bool factor, solve;
    cudaStream_t main, side;
    long wait_limit;
    int min_rpt;
    bool same(const LuGraphKey& o) const
    {
        return type == o.type && A == o.A && B == o.B && X == o.X && n == o.n && lda == o.lda && ldb == o.ldb &&
               ldx == o.ldx && nrhs == o.nrhs && nb == o.nb && ipiv == o.ipiv && perm == o.perm && info == o.info &&
               factor == o.factor && solve == o.solve && main == o.main && side == o.side &&
               wait_limit == o.wait_limit && min_rpt == o.min_rpt;
    }
};

struct LuGraphEntry {
    LuGraphKey key;
    cudaGraphExec_t exec = nullptr;   // null: seen once, not captured yet
    int64_t launches = 0;             // own kernels inside the graph
    uint64_t stamp = 0;
};

}  // namespace

struct LuGraphCache {
    static constexpr int kMax = 8;
    std::vector<LuGraphEntry> entries;
    uint64_t clock = 0;

    LuGraphEntry* find(const LuGraphKey& k)
    {
        for (auto& e : entries)
            if (e.key.same(k)) {
                e.stamp = ++clock;
                return &e;
            }
        return nullptr;
    }
    LuGraphEntry* insert(const LuGraphKey& k)
    {
        if ((int)entries.size() >= kMax) {
            size_t old = 0;
            for (size_t i = 1; i < entries.size(); ++i)
                if (entries[i].stamp < entries[old].stamp) old = i;
            if (entries[old].exec) cudaGraphExecDestroy(entries[old].exec);
            entries.erase(entries.begin() + (long)old);
        }
        LuGraphEntry e;
        e.key = k;
        e.stamp = ++clock;
        entries.push_back(e);
        return &entries.back();
    }
    ~LuGraphCache()
    {
        for (auto& e : entries)
            if (e.exec) cudaGraphExecDestroy(e.exec);
    }
};

LuGraphCache* lu_graph_cache_create() { return new LuGraphCache(); }
void lu_graph_cache_destroy(LuGraphCache* c) { delete c; }

namespace {

template <typename T>
void lu_body(Lu<T>& lu, T* A, int64_t n, int64_t lda, const T* B, int64_t ldb, int nrhs, T* X, int64_t ldx,
             int* perm, int nb, bool factor, bool solve)
{
    if (factor) lu.factor(A, n, lda, nb);
    lu.use(false);
    if (solve && nrhs > 0) lu.solve(A, n, lda, B, ldb, nrhs, X, ldx, perm);
}

// Captures lu_body on the main stream (the side stream joins through a fork
// event and is joined back before the capture ends) and instantiates it.
template <typename T>
cudaError_t lu_capture(Lu<T>& lu, T* A, int64_t n, int64_t lda, const T* B, int64_t ldb, int nrhs, T* X, int64_t ldx,
                       int* perm, int nb, bool factor, bool solve, cudaGraphExec_t* exec)
{
    *exec = nullptr;
    const bool two = lu.side_st != lu.main_st;
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (fork) cudaEventDestroy(fork);
        return e;
    }
    e = cudaStreamBeginCapture(lu.main_st, cudaStreamCaptureModeRelaxed);
    if (e == cudaSuccess) {
        if (two) {
            lu.err = cudaEventRecord(fork, lu.main_st);
            if (lu.ok()) lu.err = cudaStreamWaitEvent(lu.side_st, fork, 0);
        }
        if (lu.ok()) lu_body(lu, A, n, lda, B, ldb, nrhs, X, ldx, perm, nb, factor, solve);
        if (two) {
            const cudaError_t e1 = cudaEventRecord(join, lu.side_st);
            const cudaError_t e2 = cudaStreamWaitEvent(lu.main_st, join, 0);
            if (lu.err == cudaSuccess) lu.err = e1 != cudaSuccess ? e1 : e2;
        }
        cudaGraph_t graph = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(lu.main_st, &graph);
        if (lu.err == cudaSuccess) lu.err = ee;
        // the nodes keep the priorities of the streams they were captured on
        // (panel chain high, side-stream updates low); by default a graph
        // would run every node at the priority of the stream it is launched on
        if (lu.ok() && graph) lu.err = cudaGraphInstantiate(exec, graph, cudaGraphInstantiateFlagUseNodePriority);
        if (graph) cudaGraphDestroy(graph);
        e = lu.err;
        if (!lu.ok() && *exec) {
            cudaGraphExecDestroy(*exec);
            *exec = nullptr;
        }
    }
    cudaEventDestroy(fork);
    cudaEventDestroy(join);
    return e;
}

}  // namespace

template <typename T>
int lu_factor_solve(const LuStreams& s, T* A, int64_t n, int64_t lda, const T* B, int64_t ldb, int nrhs, T* X,
                    int64_t ldx, int* ipiv, int* perm, int* info, int nb, bool factor, bool solve)
{
    Lu<T> lu;
    lu.main_st = s.main;
    // without a side stream the look-ahead degenerates to one in-order stream
    lu.side_st = s.side ? s.side : s.main;
    lu.use(false);
    lu.ipiv = ipiv;
    lu.info = info;
    lu.wait_limit = s.wait_limit > 0 ? s.wait_limit : kDefaultWaitLimit;
    lu.min_rpt = (s.min_leaf_rpt == 2 || s.min_leaf_rpt == 4) ? s.min_leaf_rpt : 1;
    configure(lu);
    // a leaf cluster holds at most cluster * 512 * 8 rows
    if (nb < 1 || nb > kMaxBlock || n > (int64_t)lu.cluster * kLeafThreads * 8 || n > INT32_MAX)
        return LU_TOO_LARGE;
    LuGraphEntry* entry = nullptr;
    // graphs are captured from the caller's stream: not from CUDA's legacy
    // default stream (it cannot be captured) nor from a stream the caller is
    // capturing already (the work then lands in the caller's graph)
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    const bool cacheable = s.graphs && n > 0 && s.main != nullptr &&
                           cudaStreamIsCapturing(s.main, &cap) == cudaSuccess && cap == cudaStreamCaptureStatusNone;
    if (cacheable) {
        const LuGraphKey key{(int)sizeof(T), A, B, X, n, lda, ldb, ldx, nrhs, nb, ipiv, perm, info, factor, solve,
                             lu.main_st, lu.side_st, lu.wait_limit, lu.min_rpt};
        entry = s.graphs->find(key);
        if (entry && entry->exec) {   // replay
            if (cudaGraphLaunch(entry->exec, lu.main_st) != cudaSuccess) return LU_CUDA_ERROR;
            if (s.launches) *s.launches += entry->launches;
            return LU_OK;
        }
        if (!entry) {                 // first sighting: eager, remembered
            s.graphs->insert(key);
            entry = nullptr;
        }
    }
    if (entry) {                      // second sighting: capture, then launch
        cudaGraphExec_t exec = nullptr;
        lu_capture(lu, A, n, lda, B, ldb, nrhs, X, ldx, perm, nb, factor, solve, &exec);
        if (lu.err != cudaSuccess || !exec) return LU_CUDA_ERROR;
        entry->exec = exec;
        entry->launches = lu.launches;
        if (cudaGraphLaunch(exec, lu.main_st) != cudaSuccess) return LU_CUDA_ERROR;
        if (s.launches) *s.launches += lu.launches;
        return LU_OK;
    }
    lu_body(lu, A, n, lda, B, ldb, nrhs, X, ldx, perm, nb, factor, solve);
    if (s.launches) *s.launches += lu.launches;
    if (lu.err != cudaSuccess) return LU_CUDA_ERROR;
    return LU_OK;
}

// ------------------------------------------------- grouped factorisation
namespace {

__global__ void set_ints_kernel(int* p, int n, int v)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// perm of every system from its pivots: one CTA per system, in shared memory
struct PermRec {
    const int* ipiv;
    int* perm;
    int n, pad;
};
struct PermGroup {
    int count, pad;
    PermRec rec[kGroupMax];
};
__global__ void __launch_bounds__(1024) perm_group_kernel(const __grid_constant__ PermGroup g)
{
    extern __shared__ int s_perm[];
    const PermRec& r = g.rec[blockIdx.x];
    for (int i = threadIdx.x; i < r.n; i += blockDim.x) s_perm[i] = i;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < r.n; ++k) {
            const int q = r.ipiv[k];
            const int t = s_perm[k];
            s_perm[k] = s_perm[q];
            s_perm[q] = t;
        }
    __syncthreads();
    for (int i = threadIdx.x; i < r.n; i += blockDim.x) r.perm[i] = s_perm[i];
}

// The blocked right-looking LU of csrc/lu.cu's Lu::factor over many systems
// at once: every launch covers the systems still active at its step (a system
// of n_pad rows takes part in block steps k < n_pad).  Panels of nb columns
// split recursively down to 32-column cluster leaves; trailing updates are
// grouped TF32 tcgen05 products.  Look-ahead of one block column on a side
// stream, as in the single-system factorisation.
struct GroupLu {
    cudaStream_t st, main_st, side_st;
    cudaStream_t* aux = nullptr;   // leaf streams
    int naux = 0;
    cudaEvent_t ev_fork = nullptr;
    std::vector<cudaEvent_t> ev_join;
    const std::vector<GroupSystem>* sys;
    const CUtensorMap* maps;
    int* status;
    int cluster = 8;
    long wait_limit = kDefaultWaitLimit;
    int64_t launches = 0;
    cudaError_t err = cudaSuccess;
    bool ok() const { return err == cudaSuccess; }
    const GroupSystem& S(int p) const { return (*sys)[p]; }
    static float* at(const GroupSystem& g, int r, int c) { return g.A + r + (int64_t)c * g.lda; }

    // systems with n_pad > rows
    std::vector<int> active(const std::vector<int>& from, int rows) const
    {
        std::vector<int> a;
        for (int p : from)
            if (S(p).n_pad > rows) a.push_back(p);
        return a;
    }

    void gemm(std::vector<GemmGroupRec>& recs)
    {
        if (!ok() || recs.empty()) return;
        err = gemm_sub_group(st, maps, recs, status, &launches);
    }

    // rows [o, o + npiv) swapped with ipiv[o ..] in the column ranges given by f
    template <class F>
    void laswp(const std::vector<int>& act, int npiv, F f)
    {
        if (!ok() || act.empty()) return;
        LaswpGroup g{};
        g.npiv = npiv;
        int widest = 0;
        auto flush = [&]() {
            if (g.count == 0 || !ok()) return;
            const int blocks = (widest + 7) / 8 < 64 ? (widest + 7) / 8 : 64;
            laswp_group_kernel<<<dim3((unsigned)(blocks > 0 ? blocks : 1), (unsigned)g.count), 256, 0, st>>>(g);
            ++launches;
            err = cudaGetLastError();
            g.count = 0;
            widest = 0;
        };
        for (int p : act) {
            LaswpRec r{};
            f(S(p), r);
            if (r.ncol1 + r.ncol2 <= 0) continue;
            if (g.count == kGroupMax) flush();
            widest = r.ncol1 + r.ncol2 > widest ? r.ncol1 + r.ncol2 : widest;
            g.rec[g.count++] = r;
        }
        flush();
    }

    // B (b x ncol) := L^-1 B, L unit lower at diagonal position o, B columns
    // [c1, c1 + ncol(p)): 64-row blocks and grouped products
    template <class NC>
    void trsm_lower(const std::vector<int>& act, int o, int b, int c1, NC ncol)
    {
        for (int d = 0; d < b && ok(); d += 64) {
            const int db = b - d < 64 ? b - d : 64;
            TrsmGroup g{};
            g.b = db;
            int widest = 0;
            auto flush = [&]() {
                if (g.count == 0 || !ok()) return;
                trsm_group_kernel<<<dim3((unsigned)((widest + 31) / 32), (unsigned)g.count), 128, 0, st>>>(g);
                ++launches;
                err = cudaGetLastError();
                g.count = 0;
                widest = 0;
            };
            std::vector<GemmGroupRec> recs;
            for (int p : act) {
                const GroupSystem& y = S(p);
                const int nc = ncol(y);
                if (nc <= 0) continue;
                if (g.count == kGroupMax) flush();
                g.rec[g.count++] = TrsmRec{at(y, o + d, o + d), at(y, o + d, c1), y.lda, y.lda, nc, 0};
                widest = nc > widest ? nc : widest;
                if (d + db < b)
                    recs.push_back(GemmGroupRec{at(y, o + d + db, c1), y.lda, b - d - db, nc, db, o + d + db, o + d,
                                                o + d, c1, y.map, 0});
            }
            flush();
            gemm(recs);
        }
    }

    // 32-column leaves of the panel at diagonal position o, one launch per
    // cluster size (CTAs of 512 rows); the launches of different sizes run
    // side by side on the auxiliary streams when there are any
    void leaf(const std::vector<int>& act, int o, int w)
    {
        if (!ok()) return;
        std::vector<int> sizes;
        for (int p : act) {
            const int m = S(p).n_pad - o;
            const int C = (m + kLeafThreads - 1) / kLeafThreads;
            if (m > 0 && std::find(sizes.begin(), sizes.end(), C) == sizes.end()) sizes.push_back(C);
        }
        const bool fan = naux > 0 && sizes.size() > 1;
        cudaStream_t home = st;
        if (fan) {
            err = cudaEventRecord(ev_fork, home);
            for (int q = 0; q < naux && ok(); ++q) err = cudaStreamWaitEvent(aux[q], ev_fork, 0);
        }
        int used = 0;
        for (int C = 1; C <= cluster && ok(); ++C) {
            if (std::find(sizes.begin(), sizes.end(), C) == sizes.end()) continue;
            if (fan) st = aux[used++ % naux];
            LeafGroup g{};
            g.w = w;
            g.wait_limit = wait_limit;
            auto flush = [&]() {
                if (g.count == 0 || !ok()) return;
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3((unsigned)C, (unsigned)g.count);
                cfg.blockDim = dim3(kLeafThreads);
                cfg.stream = st;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeClusterDimension;
                attr[0].val.clusterDim.x = (unsigned)C;
                attr[0].val.clusterDim.y = 1;
                attr[0].val.clusterDim.z = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                err = cudaLaunchKernelEx(&cfg, leaf_group_kernel<32, 1>, g);
                ++launches;
                g.count = 0;
            };
            for (int p : act) {
                const GroupSystem& y = S(p);
                const int m = y.n_pad - o;
                if (m <= 0 || (m + kLeafThreads - 1) / kLeafThreads != C) continue;
                if (g.count == kGroupMax) flush();
                g.rec[g.count++] = LeafRec{at(y, o, o), y.ipiv + o, y.info, y.lda, m, o, o};
            }
            flush();
        }
        st = home;
        if (fan)   // the home stream continues once every size's leaves are done
            for (int q = 0; q < (used < naux ? used : naux) && ok(); ++q) {
                err = cudaEventRecord(ev_join[q], aux[q]);
                if (ok()) err = cudaStreamWaitEvent(home, ev_join[q], 0);
            }
    }

    void panel(const std::vector<int>& act, int o, int w)
    {
        if (!ok() || act.empty()) return;
        if (w <= 32) {
            leaf(act, o, w);
            return;
        }
        int w1 = w / 2;
        w1 = (w1 + 31) / 32 * 32;
        if (w1 >= w) w1 = w - 32;
        panel(act, o, w1);
        laswp(act, w1, [&](const GroupSystem& y, LaswpRec& r) {
            r = LaswpRec{at(y, o, o + w1), nullptr, y.ipiv + o, y.lda, w - w1, 0, o};
        });
        trsm_lower(act, o, w1, o + w1, [&](const GroupSystem&) { return w - w1; });
        std::vector<GemmGroupRec> recs;
        for (int p : act) {
            const GroupSystem& y = S(p);
            if (y.n_pad - o > w1)
                recs.push_back(GemmGroupRec{at(y, o + w1, o + w1), y.lda, y.n_pad - o - w1, w - w1, w1, o + w1, o, o,
                                            o + w1, y.map, 0});
        }
        gemm(recs);
        panel(active(act, o + w1), o + w1, w - w1);
        laswp(act, w - w1, [&](const GroupSystem& y, LaswpRec& r) {
            r = LaswpRec{at(y, o + w1, o), nullptr, y.ipiv + o + w1, y.lda, w1, 0, o + w1};
        });
    }

    void use(bool side) { st = side ? side_st : main_st; }

    void factor(int nb)
    {
        use(false);
        int nmax = 0;
        std::vector<int> all;
        for (int p = 0; p < (int)sys->size(); ++p) {
            all.push_back(p);
            nmax = S(p).n_pad > nmax ? S(p).n_pad : nmax;
        }
        const int nblk = (nmax + nb - 1) / nb;
        if (nblk == 0) return;
        std::vector<cudaEvent_t> ev_panel(nblk, nullptr), ev_rest(nblk, nullptr);
        cudaEvent_t fork = nullptr;
        err = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
        for (int b = 0; b < nblk && ok(); ++b) {
            err = cudaEventCreateWithFlags(&ev_panel[b], cudaEventDisableTiming);
            if (ok()) err = cudaEventCreateWithFlags(&ev_rest[b], cudaEventDisableTiming);
        }
        // the side stream follows the main stream from here on (and joins a
        // stream capture of it) even where it gets no work
        if (ok() && side_st != main_st) {
            err = cudaEventRecord(fork, main_st);
            if (ok()) err = cudaStreamWaitEvent(side_st, fork, 0);
        }
        if (ok()) {
            panel(all, 0, nb);
            if (ok()) err = cudaEventRecord(ev_panel[0], main_st);
        }
        for (int b = 0; b < nblk && ok(); ++b) {
            const int k = b * nb, k1 = k + nb, k2 = k1 + nb;
            const std::vector<int> act = active(all, k), act1 = active(all, k1), act2 = active(all, k2);
            use(false);
            if (b > 0) err = cudaStreamWaitEvent(main_st, ev_rest[b - 1], 0);
            laswp(act, nb, [&](const GroupSystem& y, LaswpRec& r) {
                r = LaswpRec{at(y, k, 0), at(y, k, k1), y.ipiv + k, y.lda, k, y.n_pad > k1 ? nb : 0, k};
            });
            if (!act1.empty()) {
                trsm_lower(act1, k, nb, k1, [&](const GroupSystem&) { return nb; });
                std::vector<GemmGroupRec> recs;
                for (int p : act1) {
                    const GroupSystem& y = S(p);
                    recs.push_back(GemmGroupRec{at(y, k1, k1), y.lda, y.n_pad - k1, nb, nb, k1, k, k, k1, y.map, 0});
                }
                gemm(recs);
                panel(act1, k1, nb);
                if (ok()) err = cudaEventRecord(ev_panel[b + 1], main_st);
            }
            use(true);
            if (!act2.empty() && ok()) {
                err = cudaStreamWaitEvent(side_st, ev_panel[b], 0);
                laswp(act2, nb, [&](const GroupSystem& y, LaswpRec& r) {
                    r = LaswpRec{at(y, k, k2), nullptr, y.ipiv + k, y.lda, y.n_pad - k2, 0, k};
                });
                trsm_lower(act2, k, nb, k2, [&](const GroupSystem& y) { return y.n_pad - k2; });
                std::vector<GemmGroupRec> recs;
                for (int p : act2) {
                    const GroupSystem& y = S(p);
                    recs.push_back(
                        GemmGroupRec{at(y, k1, k2), y.lda, y.n_pad - k1, y.n_pad - k2, nb, k1, k, k, k2, y.map, 0});
                }
                gemm(recs);
            }
            if (ok()) err = cudaEventRecord(ev_rest[b], side_st);
        }
        use(false);
        if (ok()) err = cudaStreamWaitEvent(main_st, ev_rest[nblk - 1], 0);
        for (int b = 0; b < nblk; ++b) {
            if (ev_panel[b]) cudaEventDestroy(ev_panel[b]);
            if (ev_rest[b]) cudaEventDestroy(ev_rest[b]);
        }
        if (fork) cudaEventDestroy(fork);
    }
};

}  // namespace

int lu_factor_group(const LuStreams& s, const std::vector<GroupSystem>& sys, const CUtensorMap* dev_maps,
                    int* infos, int* status, int nb)
{
    if (sys.empty()) return LU_OK;
    GroupLu g;
    g.main_st = s.main;
    g.side_st = s.side ? s.side : s.main;
    g.use(false);
    g.sys = &sys;
    g.maps = dev_maps;
    g.status = status;
    g.wait_limit = s.wait_limit > 0 ? s.wait_limit : kDefaultWaitLimit;
    g.aux = s.aux;
    g.naux = s.aux ? s.naux : 0;
    if (g.naux > 0) {
        g.err = cudaEventCreateWithFlags(&g.ev_fork, cudaEventDisableTiming);
        g.ev_join.assign((size_t)g.naux, nullptr);
        for (auto& e : g.ev_join)
            if (g.ok()) g.err = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    }
    struct Cleanup {   // the events of the leaf fan-out
        GroupLu& g;
        ~Cleanup()
        {
            if (g.ev_fork) cudaEventDestroy(g.ev_fork);
            for (auto e : g.ev_join)
                if (e) cudaEventDestroy(e);
        }
    } cleanup{g};
    if (!g.ok()) return LU_CUDA_ERROR;
    {
        Lu<float> probe;
        configure(probe);
        g.cluster = probe.cluster;
        static std::once_flag once;
        std::call_once(once, [] {
            cudaFuncSetAttribute(leaf_group_kernel<32, 1>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        });
    }
    if (nb < 32 || nb > kMaxSwaps || nb % 32) return LU_TOO_LARGE;
    for (const auto& y : sys)
        if (y.n_pad % nb || y.n_pad > g.cluster * kLeafThreads || y.lda < y.n_pad) return LU_TOO_LARGE;
    set_ints_kernel<<<(unsigned)((sys.size() + 255) / 256), 256, 0, s.main>>>(infos, (int)sys.size(), INT_MAX);
    ++g.launches;
    g.err = cudaGetLastError();
    if (g.ok()) g.factor(nb);
    if (s.launches) *s.launches += g.launches;
    return g.ok() ? LU_OK : LU_CUDA_ERROR;
}

int lu_group_max_rows()
{
    Lu<float> probe;
    configure(probe);
    return probe.cluster * kLeafThreads;
}

int lu_pivots_to_perm_group(cudaStream_t st, const std::vector<GroupSystem>& sys, const std::vector<int*>& perms,
                            int64_t* launches)
{
    int nmax = 0;
    for (const auto& y : sys) nmax = y.n_pad > nmax ? y.n_pad : nmax;
    const size_t smem = (size_t)nmax * sizeof(int);
    if (cudaFuncSetAttribute(perm_group_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return LU_CUDA_ERROR;
    PermGroup g{};
    for (size_t p = 0; p <= sys.size(); ++p) {
        if (g.count == kGroupMax || (p == sys.size() && g.count > 0)) {
            perm_group_kernel<<<(unsigned)g.count, 1024, smem, st>>>(g);
            if (launches) ++*launches;
            if (cudaGetLastError() != cudaSuccess) return LU_CUDA_ERROR;
            g.count = 0;
        }
        if (p < sys.size()) g.rec[g.count++] = PermRec{sys[p].ipiv, perms[p], sys[p].n_pad, 0};
    }
    return LU_OK;
}

int lu_pivots_to_perm(const LuStreams& s, const int* ipiv, int64_t n, int* perm)
{
    if (n <= 0) return LU_OK;
    if (launch_pivots_to_perm(s.main, ipiv, n, perm) != cudaSuccess) return LU_CUDA_ERROR;
    if (s.launches) ++*s.launches;
    return LU_OK;
}

template int lu_factor_solve<double>(const LuStreams&, double*, int64_t, int64_t, const double*, int64_t, int, double*,
                                     int64_t, int*, int*, int*, int, bool, bool);
template int lu_factor_solve<float>(const LuStreams&, float*, int64_t, int64_t, const float*, int64_t, int, float*,
                                    int64_t, int*, int*, int*, int, bool, bool);

}  // namespace cad
