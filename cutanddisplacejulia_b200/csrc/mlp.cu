// Learned preconditioner (an addition to the reference, whose only solver is
// the dense A\b of src/SlipCalculator3D.jl:22): a per-element MLP maps the
// local geometry of an element's 16 nearest elements to 16 3x3 blocks of a
// sparse approximate inverse, which right-preconditions FP64 GMRES.
//
// The network is 112 -> 256 -> 256 -> 144 (ReLU), BF16 weights and
// activations with FP32 accumulation and FP32 master weights (Adam).  All of
// it -- forward, backward, loss, optimiser -- is this file's kernels: a tiled
// BF16 GEMM on the tensor cores (mma.sync m16n8k16, FP32 accumulate; the
// network is small, so one general kernel serves the six GEMM shapes of a
// training step), bias + ReLU forward / backward, column sums, MSE, Adam.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "mlp.h"

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

// out[c] = sum over rows of X[r][c] (fixed order); one thread per column
__global__ void colsum_kernel(const float* __restrict__ X, int64_t rows, int cols, float* __restrict__ out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int64_t r = 0; r < rows; ++r) s += X[r * cols + c];
    out[c] = s;
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

cudaError_t mlp_gemm(cudaStream_t st, bool ta, bool tb, const __nv_bfloat16* A, int64_t lda, const __nv_bfloat16* B,
                     int64_t ldb, float* C, int64_t ldc, int M, int N, int K, bool accumulate)
{
    if (M <= 0 || N <= 0) return cudaSuccess;
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
    colsum_kernel<<<(kMlpOut + 127) / 128, 128, 0, st>>>(dOf, R, kMlpOut, Gd.b3);
    MLP_CK(mlp_gemm(st, false, true, dOb, kMlpOut, W3b, kMlpOut, dAf, kMlpHidden, (int)R, kMlpHidden, kMlpOut, false));
    relu_back_kernel<<<blocks_for(R * kMlpHidden), 256, 0, st>>>(dAf, pre2, R * kMlpHidden, dH2b, dHf);
    MLP_CK(mlp_gemm(st, true, false, A1, kMlpHidden, dH2b, kMlpHidden, Gd.W2, kMlpHidden, kMlpHidden, kMlpHidden, (int)R,
                    false));
    colsum_kernel<<<(kMlpHidden + 127) / 128, 128, 0, st>>>(dHf, R, kMlpHidden, Gd.b2);
    MLP_CK(mlp_gemm(st, false, true, dH2b, kMlpHidden, W2b, kMlpHidden, dAf, kMlpHidden, (int)R, kMlpHidden,
                    kMlpHidden, false));
    relu_back_kernel<<<blocks_for(R * kMlpHidden), 256, 0, st>>>(dAf, pre1, R * kMlpHidden, dH1b, dHf);
    MLP_CK(mlp_gemm(st, true, false, Xb, kMlpIn, dH1b, kMlpHidden, Gd.W1, kMlpHidden, kMlpIn, kMlpHidden, (int)R,
                    false));
    colsum_kernel<<<(kMlpHidden + 127) / 128, 128, 0, st>>>(dHf, R, kMlpHidden, Gd.b1);
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
