// Learned preconditioner (an addition to the reference, whose only solver is
// the dense A\b of src/SlipCalculator3D.jl:22): a per-element MLP maps the
// local geometry of an element's 16 nearest elements to 16 3x3 blocks of a
// sparse approximate inverse, which right-preconditions FP64 GMRES.
//
// The network is 112 -> 256 -> 256 -> 144 (ReLU), BF16 weights and
// activations with FP32 accumulation and FP32 master weights (Adam).  All of
// it -- forward, backward, loss, optimiser -- is this file's kernels: a BF16
// GEMM on the 5th-generation tensor cores (tcgen05.mma kind::f16 with
// TMA-staged 128-byte-swizzled operand tiles and the FP32 accumulator in
// tensor memory; K-major or MN-major operands, so one kernel serves the six
// GEMM shapes of a training step without transposing anything), bias + ReLU
// forward / backward, column sums, MSE, Adam.  A tiled mma.sync kernel takes
// operands whose strides TMA cannot describe.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "mlp.h"
#include "sm100.cuh"

namespace cad {

namespace {

constexpr int kTile = 64;    // CTA tile (M and N)
constexpr int kKStep = 16;   // K per mma
constexpr int kGemmThreads = 128;

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// C (M x N, row-major, ldc, FP32) = op(A) op(B) (+ C if accumulate), A and B
// BF16 row-major: op(A) is M x K (A stored M x K, or K x M when TA), op(B) is
// K x N (B stored K x N, or N x K when TB).  4 warps, each a 32 x 32 piece of
// the 64 x 64 tile as 2 x 4 mma tiles of 16 x 8.
template <bool TA, bool TB>
__global__ void __launch_bounds__(kGemmThreads) gemm_bf16_kernel(const __nv_bfloat16* __restrict__ A, int64_t lda,
                                                                 const __nv_bfloat16* __restrict__ B, int64_t ldb,
                                                                 float* __restrict__ C, int64_t ldc, int M, int N,
                                                                 int K, int accumulate)
{
    __shared__ __nv_bfloat16 As[kTile][kKStep + 2];
    __shared__ __nv_bfloat16 Bs[kKStep][kTile + 2];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;
    const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int k0 = 0; k0 < K; k0 += kKStep) {
        for (int e = tid; e < kTile * kKStep; e += kGemmThreads) {
            const int r = e / kKStep, k = e % kKStep;
            const int gm = m0 + r, gk = k0 + k;
            As[r][k] = (gm < M && gk < K) ? (TA ? A[(int64_t)gk * lda + gm] : A[(int64_t)gm * lda + gk]) : zero;
            const int kk = e / kTile, c = e % kTile;
            const int gn = n0 + c, gk2 = k0 + kk;
            Bs[kk][c] = (gn < N && gk2 < K) ? (TB ? B[(int64_t)gn * ldb + gk2] : B[(int64_t)gk2 * ldb + gn]) : zero;
        }
        __syncthreads();
        uint32_t a[2][4], b[4][2];
        const int g = lane >> 2, q = (lane & 3) * 2;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int r = wm * 32 + i * 16 + g;
            a[i][0] = pack_bf16(As[r][q], As[r][q + 1]);
            a[i][1] = pack_bf16(As[r + 8][q], As[r + 8][q + 1]);
            a[i][2] = pack_bf16(As[r][q + 8], As[r][q + 9]);
            a[i][3] = pack_bf16(As[r + 8][q + 8], As[r + 8][q + 9]);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = wn * 32 + j * 8 + g;
            b[j][0] = pack_bf16(Bs[q][c], Bs[q + 1][c]);
            b[j][1] = pack_bf16(Bs[q + 8][c], Bs[q + 9][c]);
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                    "{%8, %9}, {%0, %1, %2, %3};\n"
                    : "+f"(acc[i][j][0]), "+f"(acc[i][j][1]), "+f"(acc[i][j][2]), "+f"(acc[i][j][3])
                    : "r"(a[i][0]), "r"(a[i][1]), "r"(a[i][2]), "r"(a[i][3]), "r"(b[j][0]), "r"(b[j][1]));
        __syncthreads();
    }
    const int g = lane >> 2, q = (lane & 3) * 2;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = m0 + wm * 32 + i * 16 + g + (e >= 2 ? 8 : 0);
                const int c = n0 + wn * 32 + j * 8 + q + (e & 1);
                if (r < M && c < N) {
                    float* p = C + (int64_t)r * ldc + c;
                    *p = accumulate ? *p + acc[i][j][e] : acc[i][j][e];
                }
            }
}

// ------------------------------------------------------ tcgen05 BF16 GEMM
// C (M x N, row-major FP32) (+)= op(A) op(B) with BF16 operands.  One CTA per
// 128 x BN tile of C; k-steps of 64 (128 bytes of BF16 = one swizzle row)
// through a 4-stage TMA ring; warp 0 issues the loads, warp 1 the MMAs (K = 16
// each) into tensor memory, warps 2-5 read the accumulator back and write C.
// A K-major operand (K contiguous) is one box {64 k, rows} per stage; an
// MN-major one (M or N contiguous) is boxes {64 mn, 64 k}, 8 KB apart.
constexpr int GBM = 128, GBK = 64, GSTAGES = 4, GTHREADS = 192, GBN_MAX = 256;
constexpr uint32_t GSTAGE_A = GBM * GBK * 2;
constexpr uint32_t GSTAGE_B = GBN_MAX * GBK * 2;
constexpr uint32_t GSTAGE = GSTAGE_A + GSTAGE_B;
constexpr size_t GSMEM = (size_t)GSTAGES * GSTAGE + 1024 + 256;
constexpr long kGemmWaitLimit = 1L << 24;

template <bool A_MN, bool B_MN>
__global__ void __launch_bounds__(GTHREADS, 1) gemm_bf16_tc_kernel(const __grid_constant__ CUtensorMap mapA,
                                                                   const __grid_constant__ CUtensorMap mapB, int M,
                                                                   int N, int K, int BN, float* __restrict__ C,
                                                                   int64_t ldc, int accumulate, int* __restrict__ status)
{
    extern __shared__ uint8_t gsm_raw[];
    uint8_t* gsm = (uint8_t*)(((uintptr_t)gsm_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* bars = (uint64_t*)(gsm + GSTAGES * GSTAGE);
    uint32_t* tmem_slot = (uint32_t*)(bars + 2 * GSTAGES + 1);
    __shared__ int s_fail;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * GBM, n0 = blockIdx.y * BN;
    const int nk = (K + GBK - 1) / GBK;
    const int nbox_b = (BN + 63) / 64;
    const uint32_t bytes = GSTAGE_A + (B_MN ? (uint32_t)nbox_b * 8192u : (uint32_t)BN * 128u);
    const uint32_t idesc = sm100::instr_desc(GBM, BN, 1, 1, A_MN ? 1u : 0u, B_MN ? 1u : 0u);

    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int q = 0; q < 2 * GSTAGES + 1; ++q) sm100::mbar_init(sm100::smem_addr(&bars[q]), 1);
        sm100::fence_barrier_init();
        sm100::prefetch_tensormap(&mapA);
        sm100::prefetch_tensormap(&mapB);
    }
    if (warp == 1) {
        sm100::tmem_alloc(sm100::smem_addr(tmem_slot), GBN_MAX);
        sm100::tmem_relinquish();
    }
    sm100::tc_fence_before();
    __syncthreads();
    sm100::tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        int issued = 0;
        for (int kt = 0; kt < nk; ++kt) {
            const int q = kt % GSTAGES;
            const uint32_t ph = (uint32_t)((kt / GSTAGES) & 1);
            if (!sm100::mbar_wait(sm100::smem_addr(&bars[GSTAGES + q]), ph ^ 1u, kGemmWaitLimit)) {
                s_fail = 1;
                break;
            }
            const uint32_t full = sm100::smem_addr(&bars[q]);
            sm100::mbar_arrive_expect_tx(full, bytes);
            const uint32_t sa = sm100::smem_addr(gsm + q * GSTAGE);
            const uint32_t sb = sa + GSTAGE_A;
            if (A_MN) {
                sm100::tma_load_2d(sa, &mapA, m0, kt * GBK, full);
                sm100::tma_load_2d(sa + 8192, &mapA, m0 + 64, kt * GBK, full);
            } else {
                sm100::tma_load_2d(sa, &mapA, kt * GBK, m0, full);
            }
            if (B_MN) {
                for (int j = 0; j < nbox_b; ++j) sm100::tma_load_2d(sb + j * 8192, &mapB, n0 + 64 * j, kt * GBK, full);
            } else {
                sm100::tma_load_2d(sb, &mapB, kt * GBK, n0, full);
            }
            issued = kt + 1;
        }
        for (int kt = issued > GSTAGES ? issued - GSTAGES : 0; kt < issued; ++kt)
            if (!sm100::mbar_wait(sm100::smem_addr(&bars[kt % GSTAGES]), (uint32_t)((kt / GSTAGES) & 1), kGemmWaitLimit))
                s_fail = 1;
    } else if (warp == 1 && lane == 0) {
        bool ok = true;
        for (int kt = 0; kt < nk && ok; ++kt) {
            const int q = kt % GSTAGES;
            const uint32_t ph = (uint32_t)((kt / GSTAGES) & 1);
            if (!sm100::mbar_wait(sm100::smem_addr(&bars[q]), ph, kGemmWaitLimit)) {
                s_fail = 1;
                ok = false;
                break;
            }
            sm100::tc_fence_after();
            const uint32_t sa = sm100::smem_addr(gsm + q * GSTAGE);
            const uint32_t sb = sa + GSTAGE_A;
#pragma unroll
            for (int kk = 0; kk < GBK / 16; ++kk) {
                // K-major: +32 bytes per K = 16 inside the 128-byte row, 8-row atoms 1 KB apart.
                // MN-major: one 128-byte row per k, K = 16 = two 8-row atoms (1 KB apart),
                // 64-element MN groups in boxes 8 KB apart.
                const uint64_t da = A_MN ? sm100::smem_desc_sw128(sa + kk * 2048, 8192, 1024)
                                         : sm100::smem_desc_sw128(sa + kk * 32, 16, 1024);
                const uint64_t db = B_MN ? sm100::smem_desc_sw128(sb + kk * 2048, 8192, 1024)
                                         : sm100::smem_desc_sw128(sb + kk * 32, 16, 1024);
                sm100::mma_f16(tmem, da, db, idesc, kt > 0 || kk > 0);
            }
            sm100::mma_commit(sm100::smem_addr(&bars[GSTAGES + q]));
        }
        sm100::mma_commit(sm100::smem_addr(&bars[2 * GSTAGES]));
        if (!sm100::mbar_wait(sm100::smem_addr(&bars[2 * GSTAGES]), 0, kGemmWaitLimit)) s_fail = 1;
    } else if (warp >= 2) {
        const int qd = warp & 3;
        const int row = m0 + 32 * qd + lane;
        const bool got = sm100::mbar_wait(sm100::smem_addr(&bars[2 * GSTAGES]), 0, kGemmWaitLimit);
        sm100::tc_fence_after();
        if (!got) {
            s_fail = 1;
        } else if (nk > 0) {
#pragma unroll 1
            for (int c0 = 0; c0 < BN; c0 += 32) {
                if (n0 + c0 >= N) break;
                uint32_t v[32];
                sm100::tmem_ld_32x32b_x32(tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)c0, v);
                sm100::tmem_wait_ld();
                if (row < M) {
                    float* cr = C + (int64_t)row * ldc + n0 + c0;
                    const int ncol = N - (n0 + c0) < 32 ? N - (n0 + c0) : 32;
#pragma unroll
                    for (int c = 0; c < 32; ++c)
                        if (c < ncol) cr[c] = (accumulate ? cr[c] : 0.f) + __uint_as_float(v[c]);
                }
            }
        }
    }
    sm100::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        sm100::tc_fence_after();
        sm100::tmem_dealloc(tmem, GBN_MAX);
    }
    if (threadIdx.x == 0 && s_fail) atomicExch(status, 1);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_tiled()
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

// Row-major BF16 matrix (rows x cols, ld elements) as a 2-D tensor map:
// dimension 0 = cols (contiguous), box {box_c, box_r}, 128-byte swizzle.
bool encode_bf16(CUtensorMap* map, const __nv_bfloat16* base, int rows, int cols, int64_t ld, int box_c, int box_r)
{
    auto fn = encode_tiled();
    if (!fn || ((uintptr_t)base & 15u) || (ld * 2) % 16 != 0) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    const cuuint32_t box[2] = {(cuuint32_t)box_c, (cuuint32_t)box_r};
    const cuuint32_t estr[2] = {1, 1};
    return fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)base, dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The device word the tcgen05 GEMMs raise when a pipeline wait runs out.
__device__ int g_mlp_gemm_status;

// pre = C + bias (kept, FP32), act = relu(pre) (BF16) -- or, for the output
// layer (relu false), out = C + bias.
__global__ void bias_act_kernel(const float* __restrict__ C, const float* __restrict__ bias, int64_t rows, int cols,
                                bool relu, float* __restrict__ pre, __nv_bfloat16* __restrict__ act)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= rows * cols) return;
    const float v = C[i] + bias[i % cols];
    pre[i] = v;
    if (act) act[i] = __float2bfloat16(relu ? fmaxf(v, 0.f) : v);
}

// d = 2 w (out - target) / count, BF16 (the output gradient); sq[i] = w (out - target)^2
__global__ void mse_grad_kernel(const float* __restrict__ out, const float* __restrict__ target, int64_t n,
                                float scale, __nv_bfloat16* __restrict__ d, float* __restrict__ dfp,
                                float* __restrict__ sq)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float e = out[i] - target[i];
    const float g = 2.f * e * scale;
    d[i] = __float2bfloat16(g);
    dfp[i] = g;
    sq[i] = e * e;
}

// dpre = dact * (pre > 0), as BF16 and FP32
__global__ void relu_back_kernel(const float* __restrict__ dact, const float* __restrict__ pre, int64_t n,
                                 __nv_bfloat16* __restrict__ d, float* __restrict__ dfp)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = pre[i] > 0.f ? dact[i] : 0.f;
    d[i] = __float2bfloat16(g);
    dfp[i] = g;
}

// out[c] = sum over rows of X[r][c] in a fixed order: a block of 32 x 32
// threads takes 32 columns; thread (x, y) sums rows y, y + 32, ... of column
// x (coalesced rows), then the 32 partial sums are added in order of y.
__global__ void __launch_bounds__(1024) colsum_kernel(const float* __restrict__ X, int64_t rows, int cols,
                                                      float* __restrict__ out)
{
    __shared__ float part[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int c = blockIdx.x * 32 + tx;
    float s = 0.f;
    if (c < cols)
        for (int64_t r = ty; r < rows; r += 32) s += X[r * cols + c];
    part[ty][tx] = s;
    __syncthreads();
    if (ty == 0 && c < cols) {
        float t = 0.f;
        for (int y = 0; y < 32; ++y) t += part[y][tx];
        out[c] = t;
    }
}

// sum of x, one block, fixed order
__global__ void __launch_bounds__(1024) sum_kernel(const float* __restrict__ x, int64_t n, float* __restrict__ out)
{
    __shared__ float s[1024];
    float a = 0.f;
    for (int64_t i = threadIdx.x; i < n; i += 1024) a += x[i];
    s[threadIdx.x] = a;
    __syncthreads();
    for (int h = 512; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

__global__ void f2bf_kernel(const float* __restrict__ x, int64_t n, __nv_bfloat16* __restrict__ y)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

// Adam (bias-corrected) on the FP32 master weights; BF16 copy refreshed
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2, __nv_bfloat16* __restrict__ wb)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16(wi);
}

// Block-sparse right preconditioner: for element i (unknowns i, N + i,
// 2N + i), z_i = sum_k blocks[i][k] v_{nbr[i][k]} with 3 x 3 FP32 blocks
// (row-major), FP64 in and out.
__global__ void spai_apply_kernel(const int* __restrict__ nbr, const float* __restrict__ blocks, int k,
                                  const double* __restrict__ v, int64_t N, double* __restrict__ z)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int q = 0; q < k; ++q) {
        const int64_t j = nbr[i * k + q];
        const float* b = blocks + (i * k + q) * 9;
        const double v0 = v[j], v1 = v[N + j], v2 = v[2 * N + j];
        a0 += (double)b[0] * v0 + (double)b[1] * v1 + (double)b[2] * v2;
        a1 += (double)b[3] * v0 + (double)b[4] * v1 + (double)b[5] * v2;
        a2 += (double)b[6] * v0 + (double)b[7] * v1 + (double)b[8] * v2;
    }
    z[i] = a0;
    z[N + i] = a1;
    z[2 * N + i] = a2;
}

// Block-Jacobi preconditioner: the inverse of each element's own 3 x 3 block
// of A (rows and columns i, N + i, 2N + i; A column-major, lda), by cofactors
// in FP64, stored FP32 row-major; nbr[i] = i.
__global__ void block_jacobi_kernel(const double* __restrict__ A, int64_t lda, int64_t N, int* __restrict__ nbr,
                                    float* __restrict__ blocks)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    double m[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) m[r][c] = A[(i + r * N) + lda * (i + c * N)];
    const double c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    const double c01 = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    const double c02 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    const double det = m[0][0] * c00 + m[0][1] * c01 + m[0][2] * c02;
    const double id = det != 0.0 ? 1.0 / det : 0.0;
    double inv[3][3];
    inv[0][0] = c00 * id;
    inv[1][0] = c01 * id;
    inv[2][0] = c02 * id;
    inv[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id;
    inv[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id;
    inv[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id;
    inv[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
    inv[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
    inv[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
    nbr[i] = (int)i;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) blocks[i * 9 + r * 3 + c] = (float)inv[r][c];
}

inline unsigned blocks_for(int64_t n) { return (unsigned)((n + 255) / 256); }

}  // namespace

cudaError_t block_jacobi(cudaStream_t st, const double* A, int64_t lda, int64_t N, int* nbr, float* blocks)
{
    if (N <= 0) return cudaSuccess;
    block_jacobi_kernel<<<blocks_for(N), 256, 0, st>>>(A, lda, N, nbr, blocks);
    return cudaGetLastError();
}

template <bool A_MN, bool B_MN>
cudaError_t launch_gemm_tc(cudaStream_t st, const CUtensorMap& ma, const CUtensorMap& mb, int M, int N, int K, int BN,
                           float* C, int64_t ldc, bool accumulate)
{
    static std::once_flag once;
    std::call_once(once, [] {
        cudaFuncSetAttribute(gemm_bf16_tc_kernel<A_MN, B_MN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GSMEM);
    });
    int* status = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void**)&status, g_mlp_gemm_status);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)((M + GBM - 1) / GBM), (unsigned)((N + BN - 1) / BN));
    gemm_bf16_tc_kernel<A_MN, B_MN><<<grid, GTHREADS, GSMEM, st>>>(ma, mb, M, N, K, BN, C, ldc, accumulate ? 1 : 0,
                                                                   status);
    return cudaGetLastError();
}

cudaError_t mlp_gemm(cudaStream_t st, bool ta, bool tb, const __nv_bfloat16* A, int64_t lda, const __nv_bfloat16* B,
                     int64_t ldb, float* C, int64_t ldc, int M, int N, int K, bool accumulate)
{
    if (M <= 0 || N <= 0) return cudaSuccess;
    if (K > 0) {
        // tensor-core path: N tile of 256, or 144 / 128 columns when N is one of those
        const int BN = N <= 128 ? 128 : (N <= 144 ? 144 : 256);
        CUtensorMap ma, mb;
        // op(A) = A (M x K, row-major: K-major) or A^T (A stored K x M: M-major);
        // op(B) = B (K x N row-major: N-major) or B^T (B stored N x K: K-major)
        const bool okA = ta ? encode_bf16(&ma, A, K, M, lda, 64, 64) : encode_bf16(&ma, A, M, K, lda, 64, GBM);
        const bool okB = tb ? encode_bf16(&mb, B, N, K, ldb, 64, BN) : encode_bf16(&mb, B, K, N, ldb, 64, 64);
        if (okA && okB) {
            if (!ta && !tb) return launch_gemm_tc<false, true>(st, ma, mb, M, N, K, BN, C, ldc, accumulate);
            if (ta && !tb) return launch_gemm_tc<true, true>(st, ma, mb, M, N, K, BN, C, ldc, accumulate);
            if (!ta && tb) return launch_gemm_tc<false, false>(st, ma, mb, M, N, K, BN, C, ldc, accumulate);
            return launch_gemm_tc<true, false>(st, ma, mb, M, N, K, BN, C, ldc, accumulate);
        }
    }
    dim3 grid((unsigned)((N + kTile - 1) / kTile), (unsigned)((M + kTile - 1) / kTile));
    if (!ta && !tb) gemm_bf16_kernel<false, false><<<grid, kGemmThreads, 0, st>>>(A, lda, B, ldb, C, ldc, M, N, K, accumulate);
    else if (ta && !tb) gemm_bf16_kernel<true, false><<<grid, kGemmThreads, 0, st>>>(A, lda, B, ldb, C, ldc, M, N, K, accumulate);
    else if (!ta && tb) gemm_bf16_kernel<false, true><<<grid, kGemmThreads, 0, st>>>(A, lda, B, ldb, C, ldc, M, N, K, accumulate);
    else gemm_bf16_kernel<true, true><<<grid, kGemmThreads, 0, st>>>(A, lda, B, ldb, C, ldc, M, N, K, accumulate);
    return cudaGetLastError();
}

// Parameter layout in the FP32 master vector: W1 (in x h), b1, W2 (h x h), b2, W3 (h x out), b3.
size_t mlp_param_count() { return (size_t)kMlpIn * kMlpHidden + kMlpHidden + (size_t)kMlpHidden * kMlpHidden +
                                  kMlpHidden + (size_t)kMlpHidden * kMlpOut + kMlpOut; }

namespace {
struct Views {
    float *W1, *b1, *W2, *b2, *W3, *b3;
};
Views views(float* p)
{
    Views v;
    v.W1 = p;
    v.b1 = v.W1 + (size_t)kMlpIn * kMlpHidden;
    v.W2 = v.b1 + kMlpHidden;
    v.b2 = v.W2 + (size_t)kMlpHidden * kMlpHidden;
    v.W3 = v.b2 + kMlpHidden;
    v.b3 = v.W3 + (size_t)kMlpHidden * kMlpOut;
    return v;
}
}  // namespace

size_t mlp_workspace_bytes(int64_t rows)
{
    const size_t r = (size_t)rows;
    // bf16: X, A1, A2, dOut, dH2, dH1, W bf16 copy; fp32: C, pre1, pre2, out, dfp x3, dA, sq, loss
    return r * (kMlpIn + 2 * kMlpHidden + kMlpOut + 2 * kMlpHidden) * 2 + mlp_param_count() * 2 +
           r * (kMlpHidden * 2 + kMlpHidden * 2 + kMlpOut * 3 + kMlpHidden * 2) * 4 + 4096;
}

int mlp_step(const MlpStep& s)
{
    cudaStream_t st = s.stream;
    const int64_t R = s.rows;
    int64_t nl = 0;
    // carve the workspace
    char* w = (char*)s.workspace;
    auto take = [&](size_t bytes) {
        char* p = w;
        w += (bytes + 255) / 256 * 256;
        return p;
    };
    __nv_bfloat16* Xb = (__nv_bfloat16*)take(R * kMlpIn * 2);
    __nv_bfloat16* A1 = (__nv_bfloat16*)take(R * kMlpHidden * 2);
    __nv_bfloat16* A2 = (__nv_bfloat16*)take(R * kMlpHidden * 2);
    __nv_bfloat16* dOb = (__nv_bfloat16*)take(R * kMlpOut * 2);
    __nv_bfloat16* dH2b = (__nv_bfloat16*)take(R * kMlpHidden * 2);
    __nv_bfloat16* dH1b = (__nv_bfloat16*)take(R * kMlpHidden * 2);
    __nv_bfloat16* Wb = (__nv_bfloat16*)take(mlp_param_count() * 2);
    float* C = (float*)take(R * (kMlpHidden > kMlpOut ? kMlpHidden : kMlpOut) * 4);
    float* pre1 = (float*)take(R * kMlpHidden * 4);
    float* pre2 = (float*)take(R * kMlpHidden * 4);
    float* out = (float*)take(R * kMlpOut * 4);
    float* dOf = (float*)take(R * kMlpOut * 4);
    float* dAf = (float*)take(R * kMlpHidden * 4);
    float* dHf = (float*)take(R * kMlpHidden * 4);
    float* sq = (float*)take(R * kMlpOut * 4);
    (void)C;
    const Views P = views(s.params);
    __nv_bfloat16* W1b = Wb;
    __nv_bfloat16* W2b = W1b + (P.W2 - P.W1);
    __nv_bfloat16* W3b = W1b + (P.W3 - P.W1);
    cudaError_t e;
#define MLP_CK(x)                          \
    do {                                   \
        e = (x);                           \
        if (e != cudaSuccess) return (int)e; \
    } while (0)
    // BF16 copies of the weights and the input
    f2bf_kernel<<<blocks_for((int64_t)mlp_param_count()), 256, 0, st>>>(s.params, (int64_t)mlp_param_count(), Wb);
    f2bf_kernel<<<blocks_for(R * kMlpIn), 256, 0, st>>>(s.X, R * kMlpIn, Xb);
    nl += 2;
    // forward
    MLP_CK(mlp_gemm(st, false, false, Xb, kMlpIn, W1b, kMlpHidden, C, kMlpHidden, (int)R, kMlpHidden, kMlpIn, false));
    bias_act_kernel<<<blocks_for(R * kMlpHidden), 256, 0, st>>>(C, P.b1, R, kMlpHidden, true, pre1, A1);
    MLP_CK(mlp_gemm(st, false, false, A1, kMlpHidden, W2b, kMlpHidden, C, kMlpHidden, (int)R, kMlpHidden, kMlpHidden,
                    false));
    bias_act_kernel<<<blocks_for(R * kMlpHidden), 256, 0, st>>>(C, P.b2, R, kMlpHidden, true, pre2, A2);
    MLP_CK(mlp_gemm(st, false, false, A2, kMlpHidden, W3b, kMlpOut, C, kMlpOut, (int)R, kMlpOut, kMlpHidden, false));
    bias_act_kernel<<<blocks_for(R * kMlpOut), 256, 0, st>>>(C, P.b3, R, kMlpOut, false, out, nullptr);
    nl += 6;
    if (s.out) MLP_CK(cudaMemcpyAsync(s.out, out, R * kMlpOut * 4, cudaMemcpyDeviceToDevice, st));
    if (!s.grads) {
        if (s.launches) *s.launches += nl;
        return (int)cudaGetLastError();
    }
    // loss and backward
    const Views Gd = views(s.grads);
    mse_grad_kernel<<<blocks_for(R * kMlpOut), 256, 0, st>>>(out, s.T, R * kMlpOut, 1.f / (float)(R * kMlpOut), dOb,
                                                             dOf, sq);
    if (s.loss) sum_kernel<<<1, 1024, 0, st>>>(sq, R * kMlpOut, s.loss);
    MLP_CK(mlp_gemm(st, true, false, A2, kMlpHidden, dOb, kMlpOut, Gd.W3, kMlpOut, kMlpHidden, kMlpOut, (int)R, false));
    colsum_kernel<<<(kMlpOut + 31) / 32, 1024, 0, st>>>(dOf, R, kMlpOut, Gd.b3);
    MLP_CK(mlp_gemm(st, false, true, dOb, kMlpOut, W3b, kMlpOut, dAf, kMlpHidden, (int)R, kMlpHidden, kMlpOut, false));
    relu_back_kernel<<<blocks_for(R * kMlpHidden), 256, 0, st>>>(dAf, pre2, R * kMlpHidden, dH2b, dHf);
    MLP_CK(mlp_gemm(st, true, false, A1, kMlpHidden, dH2b, kMlpHidden, Gd.W2, kMlpHidden, kMlpHidden, kMlpHidden, (int)R,
                    false));
    colsum_kernel<<<(kMlpHidden + 31) / 32, 1024, 0, st>>>(dHf, R, kMlpHidden, Gd.b2);
    MLP_CK(mlp_gemm(st, false, true, dH2b, kMlpHidden, W2b, kMlpHidden, dAf, kMlpHidden, (int)R, kMlpHidden,
                    kMlpHidden, false));
    relu_back_kernel<<<blocks_for(R * kMlpHidden), 256, 0, st>>>(dAf, pre1, R * kMlpHidden, dH1b, dHf);
    MLP_CK(mlp_gemm(st, true, false, Xb, kMlpIn, dH1b, kMlpHidden, Gd.W1, kMlpHidden, kMlpIn, kMlpHidden, (int)R,
                    false));
    colsum_kernel<<<(kMlpHidden + 31) / 32, 1024, 0, st>>>(dHf, R, kMlpHidden, Gd.b1);
    nl += 13 + (s.loss ? 1 : 0);
    if (s.adam_m) {
        const int64_t n = (int64_t)mlp_param_count();
        adam_kernel<<<blocks_for(n), 256, 0, st>>>(s.params, s.grads, s.adam_m, s.adam_v, n, s.lr, 0.9f, 0.999f, 1e-8f,
                                                   s.bias_c1, s.bias_c2, nullptr);
        ++nl;
    }
#undef MLP_CK
    if (s.launches) *s.launches += nl;
    return (int)cudaGetLastError();
}

cudaError_t spai_apply(cudaStream_t st, const int* nbr, const float* blocks, int k, const double* v, int64_t N,
                       double* z)
{
    if (N <= 0) return cudaSuccess;
    spai_apply_kernel<<<blocks_for(N), 256, 0, st>>>(nbr, blocks, k, v, N, z);
    return cudaGetLastError();
}

}  // namespace cad
