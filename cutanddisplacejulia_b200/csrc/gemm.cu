// The dense LU's matrix products, C -= A * B (column-major, no transposes),
// written for sm_100a:
//
// * FP64 (the plain FP64 solve, A\b of src/SlipCalculator3D.jl:22): DMMA
//   tensor-core tiles (mma.sync m8n8k4 f64).  A 128 x 64 block of C per CTA,
//   4 warps of 64 x 32, three CTAs per SM, k-steps of 16 through a 3-deep
//   cp.async ring (8-byte copies: any leading dimension and any row offset).
//   Shared-memory words are XOR-swizzled by row so that every fragment load is
//   free of bank conflicts.
// * FP32 with TF32 tensor cores (the mixed solve's FP32 factorisation):
//   tcgen05.mma kind::tf32 with operands staged by TMA in 128-byte-swizzled
//   tiles (the MN-major A in 32-byte swizzle atoms, the only layout MN-major
//   32-bit operands take) and the 128 x 128 FP32 accumulator in tensor memory.  One warp
//   issues the TMA loads, one the MMAs, four run the epilogue (tensor memory
//   -> registers, C -= product with coalesced column accesses); a 3-stage
//   ring of 32 KB stages, two CTAs per SM so that one CTA's epilogue overlaps
//   the other's loads.  TMA needs 16-byte aligned operand starts and leading
//   dimensions that are multiples of 4 floats; other FP32 calls take a CUDA-
//   core FP32 kernel.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "gemm.h"
#include "sm100.cuh"

namespace cad {

namespace {

// ------------------------------------------------------------------ FP64 DMMA
// CTA tile BM x BN (128 x 64 for large products, 64 x 32 where the large
// tiles would not fill the GPU), 4 warps of BM/2 x BN/2 as DMMA tiles of
// 8 x 8; k-steps of 16; several CTAs per SM (the large tile: three, 72 KB of
// shared memory each -- 3 stages of unpadded, swizzled tiles) so that the
// DMMA latency is hidden and one CTA's prologue and epilogue overlap the
// others' main loops.
constexpr int DBK = 16, DSTAGES = 3, DTHREADS = 128;
constexpr int DLDB = DBK;       // shared row (one n) of the B tile, doubles
template <int BM, int BN>
struct DTile {
    static constexpr int STAGE_A = DBK * BM;
    static constexpr int STAGE_B = BN * DLDB;
    static constexpr int MT = BM / 16;         // 8-row DMMA tiles per warp
    static constexpr int NT = BN / 16;         // 8-column DMMA tiles per warp
    static constexpr size_t SMEM = (size_t)DSTAGES * (STAGE_A + STAGE_B) * sizeof(double);
};
// Unpadded rows with the 8-byte words XOR-swizzled by the row index: a
// fragment load (4 rows x 4 (A) or 4 x 4 (B) words per half warp) then hits 16
// distinct banks pairs.  Element (row, col) of a tile with rows of `ld` words
// sits at row * ld + (col ^ (4 * (row & 3))).
__device__ __forceinline__ int swz(int row, int col, int ld) { return row * ld + (col ^ ((row & 3) << 2)); }

__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src, bool pred)
{
    // src-size 0 writes zeros (rows or columns outside the operand)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(dst), "l"(src), "r"(pred ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// 16 x 8 x MK DMMA (MK = 8 or 16).  Thread (g = lane / 4, t = lane % 4) holds
// A elements (row g + 8 (r & 1), k t + 4 (r >> 1)) for r < MK / 2, B elements
// (k t + 4 r, column g) for r < MK / 4, and C elements (row g, columns 2t,
// 2t + 1) in c0, c1 and (row g + 8, the same columns) in c2, c3.
template <int MK>
__device__ __forceinline__ void dmma16(double& c0, double& c1, double& c2, double& c3, const double* a,
                                       const double* b);
template <>
__device__ __forceinline__ void dmma16<8>(double& c0, double& c1, double& c2, double& c3, const double* a,
                                          const double* b)
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+d"(c0), "+d"(c1), "+d"(c2), "+d"(c3)
                 : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}
template <>
__device__ __forceinline__ void dmma16<16>(double& c0, double& c1, double& c2, double& c3, const double* a,
                                           const double* b)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7,%8,%9,%10,%11}, "
                 "{%12,%13,%14,%15}, {%0,%1,%2,%3};"
                 : "+d"(c0), "+d"(c1), "+d"(c2), "+d"(c3)
                 : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
                   "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// Stage s of the ring <- k-step kt: the A tile (BM rows x 16 columns, stored
// k-major: row k holds BM consecutive m) and the B tile (16 rows x BN
// columns, stored n-major: row n holds 16 consecutive k).
template <int BM, int BN>
__device__ __forceinline__ void dgemm_load_stage(double* sA, double* sB, const double* __restrict__ A, int64_t lda,
                                                 const double* __restrict__ B, int64_t ldb, int m, int n, int k,
                                                 int m0, int n0, int kt)
{
    const int tid = threadIdx.x;
    const int k0 = kt * DBK;
#pragma unroll
    for (int i = 0; i < (BM * DBK) / DTHREADS; ++i) {
        const int e = tid + DTHREADS * i;
        const int kk = e / BM, mm = e % BM;
        const bool ok = (m0 + mm < m) && (k0 + kk < k);
        const double* src = ok ? A + (int64_t)(m0 + mm) + (int64_t)(k0 + kk) * lda : A;
        cp_async8(sm100::smem_addr(sA + swz(kk, mm, BM)), src, ok);
    }
#pragma unroll
    for (int i = 0; i < (BN * DBK) / DTHREADS; ++i) {
        const int e = tid + DTHREADS * i;
        const int nn = e / DBK, kk = e % DBK;
        const bool ok = (n0 + nn < n) && (k0 + kk < k);
        const double* src = ok ? B + (int64_t)(k0 + kk) + (int64_t)(n0 + nn) * ldb : B;
        cp_async8(sm100::smem_addr(sB + swz(nn, kk, DLDB)), src, ok);
    }
}

// MK: k-extent of one DMMA (4: m8n8k4 tiles; 8 or 16: m16n8k8 / m16n8k16)
template <int MK, int BM, int BN, int MINB>
__global__ void __launch_bounds__(DTHREADS, MINB) dgemm_sub_kernel(int m, int n, int k, const double* __restrict__ A,
                                                               int64_t lda, const double* __restrict__ B, int64_t ldb,
                                                               double* __restrict__ C, int64_t ldc)
{
    using TL = DTile<BM, BN>;
    constexpr int MT = TL::MT, NT = TL::NT;
    extern __shared__ __align__(16) double dsm[];
    double* sA = dsm;
    double* sB = dsm + DSTAGES * TL::STAGE_A;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = (warp & 1) * (BM / 2), wn = (warp >> 1) * (BN / 2);   // 2 x 2 warps
    const int g = lane >> 2, t = lane & 3;
    double acc[MT][NT][2];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    const int nk = (k + DBK - 1) / DBK;
#pragma unroll
    for (int s = 0; s < DSTAGES - 1; ++s) {
        if (s < nk)
            dgemm_load_stage<BM, BN>(sA + s * TL::STAGE_A, sB + s * TL::STAGE_B, A, lda, B, ldb, m, n, k, m0, n0, s);
        cp_async_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<DSTAGES - 2>();
        __syncthreads();
        // refill the stage consumed one step ago (every warp is past it)
        const int kn = kt + DSTAGES - 1;
        if (kn < nk)
            dgemm_load_stage<BM, BN>(sA + (kn % DSTAGES) * TL::STAGE_A, sB + (kn % DSTAGES) * TL::STAGE_B, A, lda, B,
                                     ldb, m, n, k, m0, n0, kn);
        cp_async_commit();
        const double* a_s = sA + (kt % DSTAGES) * TL::STAGE_A;
        const double* b_s = sB + (kt % DSTAGES) * TL::STAGE_B;
        if constexpr (MK == 4) {
#pragma unroll
            for (int kk = 0; kk < DBK; kk += 4) {
                double af[MT], bf[NT];
#pragma unroll
                for (int i = 0; i < MT; ++i) af[i] = a_s[swz(kk + t, wm + 8 * i + g, BM)];
#pragma unroll
                for (int j = 0; j < NT; ++j) bf[j] = b_s[swz(wn + 8 * j + g, kk + t, DLDB)];
#pragma unroll
                for (int i = 0; i < MT; ++i)
#pragma unroll
                    for (int j = 0; j < NT; ++j) dmma(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
            }
        } else {
            // 16-row blocks: acc[2I] holds rows wm + 16I + g, acc[2I + 1]
            // rows wm + 16I + 8 + g (the 8-row layout of the m8n8k4 path)
#pragma unroll
            for (int kk = 0; kk < DBK; kk += MK) {
                double af[MT / 2][MK / 2], bf[NT][MK / 4];
#pragma unroll
                for (int I = 0; I < MT / 2; ++I)
#pragma unroll
                    for (int r = 0; r < MK / 2; ++r)
                        af[I][r] = a_s[swz(kk + t + 4 * (r >> 1), wm + 16 * I + 8 * (r & 1) + g, BM)];
#pragma unroll
                for (int j = 0; j < NT; ++j)
#pragma unroll
                    for (int r = 0; r < MK / 4; ++r) bf[j][r] = b_s[swz(wn + 8 * j + g, kk + t + 4 * r, DLDB)];
#pragma unroll
                for (int I = 0; I < MT / 2; ++I)
#pragma unroll
                    for (int j = 0; j < NT; ++j)
                        dmma16<MK>(acc[2 * I][j][0], acc[2 * I][j][1], acc[2 * I + 1][j][0], acc[2 * I + 1][j][1],
                                   af[I], bf[j]);
            }
        }
    }
    cp_async_wait<0>();
    // C -= acc: thread holds rows wm + 8i + g, columns wn + 8j + 2t + {0, 1}.
    // Per column pair, all loads are issued before any store (the compiler
    // cannot reorder a load of C past a store to C), so their latencies overlap.
#pragma unroll
    for (int j = 0; j < NT; ++j) {
        double c[2][MT];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int col = n0 + wn + 8 * j + 2 * t + h;
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                const int row = m0 + wm + 8 * i + g;
                c[h][i] = (col < n && row < m) ? C[(int64_t)col * ldc + row] : 0.0;
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int col = n0 + wn + 8 * j + 2 * t + h;
            if (col >= n) continue;
            double* cc = C + (int64_t)col * ldc;
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                const int row = m0 + wm + 8 * i + g;
                if (row < m) cc[row] = c[h][i] - acc[i][j][h];
            }
        }
    }
}

// ------------------------------------------------------- FP32: tcgen05 + TMA
constexpr int TBM = 128, TBN = 128, TBK = 32, TSTAGES = 3, TTHREADS = 192;
constexpr uint32_t TSTAGE_A = TBM * TBK * 4;   // 4 boxes of 32 m x 32 k, 4 KB each
constexpr uint32_t TSTAGE_B = TBN * TBK * 4;   // one box of 32 k x 128 n
constexpr uint32_t TSTAGE = TSTAGE_A + TSTAGE_B;
constexpr size_t TSMEM = (size_t)TSTAGES * TSTAGE + 1024 /* alignment slack */ + 256 /* barriers */;
constexpr uint32_t TIDESC = sm100::instr_desc(TBM, TBN, 2, 2, 1 /* A MN-major */, 0 /* B K-major */);
constexpr long kTcWaitLimit = 1L << 24;
constexpr uint32_t kRoundBytes = TSTAGE;   // bytes of each stage rounded to TF32 (A and B tiles)

struct GemmGroup {
    int count, pad;
    const CUtensorMap* maps;
    int* status;
    GemmGroupRec rec[kGemmGroupMax];
};
static_assert(sizeof(GemmGroup) <= 32000, "grouped GEMM records exceed the kernel parameter space");

// A: dims {m, k}, box {32, 32}, 128-byte rows swizzled in 32-byte chunks;
// B: dims {k, n}, box {32, 128}, 128-byte swizzle; both FP32, out-of-range
// elements read as zero.
// One 128 x 128 tile (m0, n0) of C -= A B: A is rows [ax, ax + m), columns
// [ay, ay + k) of the tensor behind mapA, B rows [bx, bx + k), columns [by, by
// + n) of mapB's.  Rows and columns of the boxes past m, n are computed and
// dropped; k must be a multiple of TBK where the tensors continue past it.
__device__ __forceinline__ void tf32_tile(const CUtensorMap* mapA, const CUtensorMap* mapB, int ax, int ay, int bx,
                                          int by, int m, int n, int k, float* __restrict__ C, int64_t ldc, int m0,
                                          int n0, int* __restrict__ status)
{
    extern __shared__ uint8_t tsm_raw[];
    uint8_t* tsm = (uint8_t*)(((uintptr_t)tsm_raw + 1023) & ~(uintptr_t)1023);   // swizzle atoms: 1024-byte aligned
    uint64_t* bars = (uint64_t*)(tsm + TSTAGES * TSTAGE);
    // bars[0..S): stage full (TMA -> rounding warps); bars[S..2S): stage empty
    // (MMA -> TMA); bars[2S]: accumulator ready (MMA -> epilogue);
    // bars[2S+1..3S+1): stage rounded to TF32 (the four epilogue warps -> MMA)
    uint64_t* rounded = bars + 2 * TSTAGES + 1;
    uint32_t* tmem_slot = (uint32_t*)(bars + 3 * TSTAGES + 1);
    __shared__ int s_fail;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nk = (k + TBK - 1) / TBK;

    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int s = 0; s < 2 * TSTAGES + 1; ++s) sm100::mbar_init(sm100::smem_addr(&bars[s]), 1);
        for (int s = 0; s < TSTAGES; ++s) sm100::mbar_init(sm100::smem_addr(&rounded[s]), 4);
        sm100::fence_barrier_init();
        sm100::prefetch_tensormap(mapA);
        sm100::prefetch_tensormap(mapB);
    }
    if (warp == 1) {
        sm100::tmem_alloc(sm100::smem_addr(tmem_slot), TBN);
        sm100::tmem_relinquish();
    }
    sm100::tc_fence_before();
    __syncthreads();
    sm100::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // producer: stage s gets k-step kt once the MMAs of k-step kt - S are done
        int issued = 0;
        for (int kt = 0; kt < nk; ++kt) {
            const int s = kt % TSTAGES;
            const uint32_t ph = (uint32_t)((kt / TSTAGES) & 1);
            if (!sm100::mbar_wait(sm100::smem_addr(&bars[TSTAGES + s]), ph ^ 1u, kTcWaitLimit)) {
                s_fail = 1;
                break;
            }
            const uint32_t full = sm100::smem_addr(&bars[s]);
            sm100::mbar_arrive_expect_tx(full, TSTAGE);
            const uint32_t sa = sm100::smem_addr(tsm + s * TSTAGE);
#pragma unroll
            for (int mb = 0; mb < TBM / 32; ++mb)
                sm100::tma_load_2d(sa + mb * 4096, mapA, ax + m0 + 32 * mb, ay + kt * TBK, full);
            sm100::tma_load_2d(sa + TSTAGE_A, mapB, bx + kt * TBK, by + n0, full);
            issued = kt + 1;
        }
        // no copy may still be landing when the CTA exits (a no-op unless a wait
        // above ran out)
        for (int kt = issued > TSTAGES ? issued - TSTAGES : 0; kt < issued; ++kt)
            if (!sm100::mbar_wait(sm100::smem_addr(&bars[kt % TSTAGES]), (uint32_t)((kt / TSTAGES) & 1), kTcWaitLimit))
                s_fail = 1;
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: 4 MMAs (K = 8 each) per stage once the stage is rounded,
        // accumulator in tensor memory
        bool ok = true;
        for (int kt = 0; kt < nk && ok; ++kt) {
            const int s = kt % TSTAGES;
            const uint32_t ph = (uint32_t)((kt / TSTAGES) & 1);
            if (!sm100::mbar_wait(sm100::smem_addr(&rounded[s]), ph, kTcWaitLimit)) {
                s_fail = 1;
                ok = false;
                break;
            }
            sm100::tc_fence_after();
            const uint32_t sa = sm100::smem_addr(tsm + s * TSTAGE);
            const uint32_t sb = sa + TSTAGE_A;
#pragma unroll
            for (int kk = 0; kk < TBK / 8; ++kk) {
                // A (MN-major, 32-bit): k-rows of 128 bytes swizzled in 32-byte
                // chunks, 4 rows per atom (512 bytes apart: stride byte offset),
                // +1 KB per K = 8; the four 32-row m boxes 4 KB apart (leading
                // byte offset).  B (K-major): rows of 32 k -> +32 bytes per K =
                // 8; 8-row atoms 1 KB apart (stride byte offset).
                const uint64_t da = sm100::smem_desc(sa + kk * 1024, 4096, 512, sm100::kLayoutSW128Atom32);
                const uint64_t db = sm100::smem_desc_sw128(sb + kk * 32, 16, 1024);
                sm100::mma_tf32(tmem, da, db, TIDESC, kt > 0 || kk > 0);
            }
            sm100::mma_commit(sm100::smem_addr(&bars[TSTAGES + s]));   // stage s free once these MMAs finish
        }
        sm100::mma_commit(sm100::smem_addr(&bars[2 * TSTAGES]));        // accumulator complete
        // every MMA done before tensor memory is released at the end
        if (!sm100::mbar_wait(sm100::smem_addr(&bars[2 * TSTAGES]), 0, kTcWaitLimit)) s_fail = 1;
    } else if (warp >= 2) {
        // main loop: round every landed stage to TF32 in place (the tensor
        // cores would truncate the FP32 operands' low mantissa bits, a biased
        // error that builds up over the factorisation's many updates)
        const int te = threadIdx.x - 64;   // 0..127
        bool fine = true;
        for (int kt = 0; kt < nk && fine; ++kt) {
            const int s = kt % TSTAGES;
            const uint32_t ph = (uint32_t)((kt / TSTAGES) & 1);
            if (!sm100::mbar_wait(sm100::smem_addr(&bars[s]), ph, kTcWaitLimit)) {
                s_fail = 1;
                fine = false;
                break;
            }
            uint4* st4 = reinterpret_cast<uint4*>(tsm + s * TSTAGE);
#pragma unroll 4
            for (int j = 0; j < (int)(kRoundBytes / 16) / 128; ++j) {
                uint4 v = st4[te + 128 * j];
                v.x = sm100::tf32_rna(__uint_as_float(v.x));
                v.y = sm100::tf32_rna(__uint_as_float(v.y));
                v.z = sm100::tf32_rna(__uint_as_float(v.z));
                v.w = sm100::tf32_rna(__uint_as_float(v.w));
                st4[te + 128 * j] = v;
            }
            sm100::fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) sm100::mbar_arrive(sm100::smem_addr(&rounded[s]));
        }
        // epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31 = tile rows
        const int q = warp & 3;
        const int row = m0 + 32 * q + lane;
        const bool got = sm100::mbar_wait(sm100::smem_addr(&bars[2 * TSTAGES]), 0, kTcWaitLimit);
        sm100::tc_fence_after();
        if (!got) {
            s_fail = 1;
        } else if (nk > 0) {
#pragma unroll 1
            for (int c0 = 0; c0 < TBN; c0 += 32) {
                if (n0 + c0 >= n) break;   // warp-uniform
                uint32_t v[32];
                float cv[32];
                const int ncol = n - (n0 + c0) < 32 ? n - (n0 + c0) : 32;
                float* cc = C + (int64_t)(n0 + c0) * ldc + row;
#pragma unroll
                for (int c = 0; c < 32; ++c) cv[c] = (row < m && c < ncol) ? cc[(int64_t)c * ldc] : 0.f;
                sm100::tmem_ld_32x32b_x32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
                sm100::tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < 32; ++c)
                    if (row < m && c < ncol) cc[(int64_t)c * ldc] = cv[c] - __uint_as_float(v[c]);
            }
        }
    }
    sm100::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        sm100::tc_fence_after();
        sm100::tmem_dealloc(tmem, TBN);
    }
    if (threadIdx.x == 0 && s_fail) atomicMin(status, -1);
}

__global__ void __launch_bounds__(TTHREADS, 2) sgemm_tf32_sub_kernel(const __grid_constant__ CUtensorMap mapA,
                                                                     const __grid_constant__ CUtensorMap mapB, int m,
                                                                     int n, int k, float* __restrict__ C, int64_t ldc,
                                                                     int* __restrict__ status)
{
    tf32_tile(&mapA, &mapB, 0, 0, 0, 0, m, n, k, C, ldc, blockIdx.x * TBM, blockIdx.y * TBN, status);
}

// Many products in one launch: CTA x takes tile x of the flattened tile list
// (records in order, each record's tiles m-fastest).
__global__ void __launch_bounds__(TTHREADS, 2) sgemm_tf32_group_kernel(const __grid_constant__ GemmGroup g)
{
    const int t = blockIdx.x;
    int lo = 0, hi = g.count - 1;
    while (lo < hi) {   // last record whose first tile is at or before t
        const int mid = (lo + hi + 1) >> 1;
        if (g.rec[mid].tile0 <= t) lo = mid;
        else hi = mid - 1;
    }
    const GemmGroupRec& r = g.rec[lo];
    const int mt = (r.m + TBM - 1) / TBM;
    const int local = t - r.tile0;
    tf32_tile(g.maps + 2 * r.map, g.maps + 2 * r.map + 1, r.ax, r.ay, r.bx, r.by, r.m, r.n, r.k, r.C, r.ldc,
              (local % mt) * TBM, (local / mt) * TBN, g.status);
}

// ------------------------------------------- FP32 on CUDA cores (any layout)
constexpr int SBM = 64, SBN = 64, SBK = 16;
__global__ void __launch_bounds__(256) sgemm_sub_simt_kernel(int m, int n, int k, const float* __restrict__ A,
                                                             int64_t lda, const float* __restrict__ B, int64_t ldb,
                                                             float* __restrict__ C, int64_t ldc)
{
    __shared__ float sA[SBK][SBM + 4];
    __shared__ float sB[SBN][SBK + 1];
    const int m0 = blockIdx.x * SBM, n0 = blockIdx.y * SBN;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // 4 x 4 outputs each
    float acc[4][4] = {};
    for (int k0 = 0; k0 < k; k0 += SBK) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = threadIdx.x + 256 * i;
            const int kk = e / SBM, mm = e % SBM;
            sA[kk][mm] = (m0 + mm < m && k0 + kk < k) ? A[(int64_t)(m0 + mm) + (int64_t)(k0 + kk) * lda] : 0.f;
            const int nn = e / SBK, k2 = e % SBK;
            sB[nn][k2] = (n0 + nn < n && k0 + k2 < k) ? B[(int64_t)(k0 + k2) + (int64_t)(n0 + nn) * ldb] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < SBK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sA[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sB[ty + 16 * j][kk];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int col = n0 + ty + 16 * j;
        if (col >= n) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int row = m0 + tx + 16 * i;
            if (row < m) C[(int64_t)row + (int64_t)col * ldc] -= acc[i][j];
        }
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// Column-major FP32 matrix (rows x cols, ld) as a 2-D tensor map with
// box {box_rows, box_cols} and 128-byte swizzle.
bool encode_f32(CUtensorMap* map, const float* base, int rows, int cols, int64_t ld, int box_rows, int box_cols,
                CUtensorMapSwizzle swizzle)
{
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)box_rows, (cuuint32_t)box_cols};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool tma_ok(const float* p, int64_t ld)
{
    return ((uintptr_t)p & 15u) == 0 && (ld % 4) == 0 && ld > 0 && ld * 4 < ((int64_t)1 << 40);
}

}  // namespace

namespace {
template <int MK, int BM, int BN, int MINB>
cudaError_t launch_dgemm_tile(cudaStream_t st, int m, int n, int k, const double* A, int64_t lda, const double* B,
                              int64_t ldb, double* C, int64_t ldc)
{
    constexpr size_t smem = DTile<BM, BN>::SMEM;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaFuncSetAttribute(dgemm_sub_kernel<MK, BM, BN, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        cudaFuncSetAttribute(dgemm_sub_kernel<MK, BM, BN, MINB>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    });
    const dim3 grid((unsigned)((m + BM - 1) / BM), (unsigned)((n + BN - 1) / BN));
    dgemm_sub_kernel<MK, BM, BN, MINB><<<grid, DTHREADS, smem, st>>>(m, n, k, A, lda, B, ldb, C, ldc);
    return cudaGetLastError();
}

// the large tile where it gives at least two CTAs per SM, else the small one
template <int MK>
cudaError_t launch_dgemm(cudaStream_t st, int m, int n, int k, const double* A, int64_t lda, const double* B,
                         int64_t ldb, double* C, int64_t ldc)
{
    const int64_t big = (int64_t)((m + 127) / 128) * ((n + 63) / 64);
    if (big >= 2 * 148) return launch_dgemm_tile<MK, 128, 64, 3>(st, m, n, k, A, lda, B, ldb, C, ldc);
    return launch_dgemm_tile<MK, 64, 32, 6>(st, m, n, k, A, lda, B, ldb, C, ldc);
}
}  // namespace

cudaError_t gemm_sub(cudaStream_t st, int m, int n, int k, const double* A, int64_t lda, const double* B, int64_t ldb,
                     double* C, int64_t ldc, int* status, int dmma_k)
{
    (void)status;   // the FP64 kernel has no waits
    if (m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
    switch (dmma_k > 0 ? dmma_k : kDefaultDmmaK) {
    case 4: return launch_dgemm<4>(st, m, n, k, A, lda, B, ldb, C, ldc);
    case 8: return launch_dgemm<8>(st, m, n, k, A, lda, B, ldb, C, ldc);
    case 16: return launch_dgemm<16>(st, m, n, k, A, lda, B, ldb, C, ldc);
    default: return cudaErrorInvalidValue;
    }
}

bool gemm_group_maps(CUtensorMap* out, const float* base, int rows, int cols, int64_t ld)
{
    return tma_ok(base, ld) && encode_f32(&out[0], base, rows, cols, ld, 32, 32, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B) &&
           encode_f32(&out[1], base, rows, cols, ld, 32, TBN, CU_TENSOR_MAP_SWIZZLE_128B);
}

cudaError_t gemm_sub_group(cudaStream_t st, const CUtensorMap* dev_maps, std::vector<GemmGroupRec>& recs,
                           int* status, int64_t* launches)
{
    static std::once_flag once;
    std::call_once(once, [] {
        cudaFuncSetAttribute(sgemm_tf32_group_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TSMEM);
    });
    GemmGroup g{};
    g.maps = dev_maps;
    g.status = status;
    int64_t tiles = 0;
    auto flush = [&]() -> cudaError_t {
        if (g.count == 0) return cudaSuccess;
        sgemm_tf32_group_kernel<<<(unsigned)tiles, TTHREADS, TSMEM, st>>>(g);
        if (launches) ++*launches;
        g.count = 0;
        tiles = 0;
        return cudaGetLastError();
    };
    for (auto& r : recs) {
        if (r.m <= 0 || r.n <= 0 || r.k <= 0) continue;
        if (r.k % TBK || r.ax % 4 || r.bx % 4) return cudaErrorInvalidValue;
        if (g.count == kGemmGroupMax) {
            if (cudaError_t e = flush()) return e;
        }
        r.tile0 = (int)tiles;
        g.rec[g.count++] = r;
        tiles += (int64_t)((r.m + TBM - 1) / TBM) * ((r.n + TBN - 1) / TBN);
    }
    return flush();
}

cudaError_t gemm_sub(cudaStream_t st, int m, int n, int k, const float* A, int64_t lda, const float* B, int64_t ldb,
                     float* C, int64_t ldc, int* status)
{
    if (m <= 0 || n <= 0 || k <= 0) return cudaSuccess;
    CUtensorMap ma, mb;
    // A column-major (m contiguous: MN-major, 32-byte swizzle atoms); B
    // column-major (k contiguous: K-major, 16-byte atoms)
    if (status && tma_ok(A, lda) && tma_ok(B, ldb) &&
        encode_f32(&ma, A, m, k, lda, 32, 32, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B) &&
        encode_f32(&mb, B, k, n, ldb, 32, TBN, CU_TENSOR_MAP_SWIZZLE_128B)) {
        static std::once_flag once;
        std::call_once(once, [] {
            cudaFuncSetAttribute(sgemm_tf32_sub_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TSMEM);
        });
        const dim3 grid((unsigned)((m + TBM - 1) / TBM), (unsigned)((n + TBN - 1) / TBN));
        sgemm_tf32_sub_kernel<<<grid, TTHREADS, TSMEM, st>>>(ma, mb, m, n, k, C, ldc, status);
        return cudaGetLastError();
    }
    const dim3 grid((unsigned)((m + SBM - 1) / SBM), (unsigned)((n + SBN - 1) / SBN));
    sgemm_sub_simt_kernel<<<grid, 256, 0, st>>>(m, n, k, A, lda, B, ldb, C, ldc);
    return cudaGetLastError();
}

}  // namespace cad
