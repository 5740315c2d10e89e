// Device pieces of the frictional slip solve (src/SlipCalculator3D.jl:36-238)
// and of a Fischer-Burmeister Newton method for the linear complementarity
// problem it poses (the reference calls FischerNewton.fischer_newton,
// src/SlipCalculator3D.jl:196, an external package; the method here is the
// published one, written from its mathematics).
//
// The 5m x 5m friction matrix is never stored: its products are one 3m x 3m
// GEMV with C plus O(m) element-wise work, and the Newton matrix
// J = diag(Da) + diag(Db) M is written entry by entry straight from C.
// Reductions run on a fixed grid of kRedBlocks blocks with per-block partials
// summed in a fixed order by one block, so every result is reproducible.
// Where the oracle's float arithmetic is element-wise (Fischer-Burmeister
// values, Jacobian diagonals, trial points, the Newton matrix entries), the
// same operations are written with round-to-nearest intrinsics so that no
// multiply-add is contracted.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "lcp.h"

namespace cad {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kStat = kRedBlocks * (kLsSteps + 1);   // offset of the reduced results in part

// Fischer-Burmeister phi(a, b) = sqrt(a^2 + b^2) - a - b, cancellation-free
// where a + b > 0 (there it equals -2ab / (sqrt(a^2 + b^2) + a + b)).
__device__ __forceinline__ double fb(double a, double b)
{
    const double r = sqrt(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
    const double s = __dadd_rn(a, b);
    if (s > 0.0) return __ddiv_rn(__dmul_rn(__dmul_rn(-2.0, a), b), __dadd_rn(r, s));
    return __dsub_rn(r, s);
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Entry (i, j) of the friction matrix (layout in lcp.h).
__device__ __forceinline__ double friction_entry(const double* __restrict__ C, int64_t ldc,
                                                 const double* __restrict__ mu, int64_t m, int64_t i, int64_t j)
{
    const int64_t cb = j / m, jj = j - cb * m;
    if (i < 3 * m) {
        if (cb == 0) {
            const double w = mu[jj];
            const double c1 = C[i + jj * ldc], c2 = C[i + (m + jj) * ldc], c3 = C[i + (2 * m + jj) * ldc];
            return __dsub_rn(__dsub_rn(c1, __dmul_rn(c2, w)), __dmul_rn(c3, w));
        }
        if (cb <= 2) return C[i + j * ldc];
        if (cb == 3) return (i - m == jj) ? 1.0 : 0.0;
        return (i - 2 * m == jj) ? 1.0 : 0.0;
    }
    const int64_t ii = i - 3 * m, rb = ii / m, r = ii - rb * m;
    if (r != jj) return 0.0;
    if (cb == 0) return __dmul_rn(2.0, mu[jj]);
    if (cb == 1) return rb == 0 ? -1.0 : 0.0;
    if (cb == 2) return rb == 1 ? -1.0 : 0.0;
    return 0.0;
}

template <bool FRICTION>
__global__ void __launch_bounds__(kThreads) jacobian_kernel(const double* __restrict__ M, int64_t ldm,
                                                           const double* __restrict__ mu, int64_t m, int64_t n,
                                                           const double* __restrict__ Da,
                                                           const double* __restrict__ Db, double* __restrict__ J,
                                                           int64_t ldj)
{
    const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
    if (i >= n) return;
    const double da = Da[i], db = Db[i];
    for (int64_t j = blockIdx.y; j < n; j += gridDim.y) {
        const double v = FRICTION ? friction_entry(M, ldm, mu, m, i, j) : M[i + j * ldm];
        const double e = __dmul_rn(db, v);
        J[i + j * ldj] = (i == j) ? __dadd_rn(e, da) : e;
    }
}

// u = [v1; v2 - mu v1; v3 - mu v1] so that C u is the top 3m rows of M v
__global__ void friction_pre_kernel(const double* __restrict__ v, const double* __restrict__ mu, int64_t m,
                                    double* __restrict__ u)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
        const double v1 = v[r], w = __dmul_rn(mu[r], v1);
        u[r] = v1;
        u[m + r] = __dsub_rn(v[m + r], w);
        u[2 * m + r] = __dsub_rn(v[2 * m + r], w);
    }
}

// out[0:3m] holds C u on entry; completes M v (+ q)
__global__ void friction_post_kernel(const double* __restrict__ v, const double* __restrict__ mu,
                                     const double* __restrict__ q, int64_t m, double* __restrict__ out)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
        const double v1 = v[r], tw = __dmul_rn(__dmul_rn(2.0, mu[r]), v1);
        double o[5] = {out[r], __dadd_rn(out[m + r], v[3 * m + r]), __dadd_rn(out[2 * m + r], v[4 * m + r]),
                       __dsub_rn(tw, v[m + r]), __dsub_rn(tw, v[2 * m + r])};
#pragma unroll
        for (int k = 0; k < 5; ++k) out[k * m + r] = q ? __dadd_rn(o[k], q[k * m + r]) : o[k];
    }
}

// s = C^T v_top in s (3m); out = M^T v
__global__ void friction_post_t_kernel(const double* __restrict__ v, const double* __restrict__ mu,
                                       const double* __restrict__ s, int64_t m, double* __restrict__ out)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
        const double w = mu[r], v4 = v[3 * m + r], v5 = v[4 * m + r];
        double o0 = __dsub_rn(__dsub_rn(s[r], __dmul_rn(w, s[m + r])), __dmul_rn(w, s[2 * m + r]));
        o0 = __dadd_rn(o0, __dmul_rn(__dmul_rn(2.0, w), v4));
        o0 = __dadd_rn(o0, __dmul_rn(__dmul_rn(2.0, w), v5));
        out[r] = o0;
        out[m + r] = __dsub_rn(s[m + r], v4);
        out[2 * m + r] = __dsub_rn(s[2 * m + r], v5);
        out[3 * m + r] = v[m + r];
        out[4 * m + r] = v[2 * m + r];
    }
}

// Per-block partials of (max |phi|, sum phi^2, degenerate count) at part[3 b + k]
__global__ void __launch_bounds__(kThreads) fb_eval_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                                          int64_t n, double* __restrict__ phi, double* __restrict__ z,
                                                          double* __restrict__ part)
{
    double mx = 0.0, sq = 0.0, deg = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        const double a = x[i], b = y[i];
        const double p = fb(a, b);
        const bool d = (a == 0.0 && b == 0.0);
        phi[i] = p;
        z[i] = d ? 1.0 : 0.0;
        mx = fmax(mx, fabs(p));
        sq += p * p;
        deg += d ? 1.0 : 0.0;
    }
    __shared__ double s[3][kWarps];
    mx = warp_max(mx);
    sq = warp_sum(sq);
    deg = warp_sum(deg);
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
    if (l == 0) {
        s[0][w] = mx;
        s[1][w] = sq;
        s[2][w] = deg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0, c = 0.0;
        for (int k = 0; k < kWarps; ++k) {
            a = fmax(a, s[0][k]);
            b += s[1][k];
            c += s[2][k];
        }
        part[3 * blockIdx.x + 0] = a;
        part[3 * blockIdx.x + 1] = b;
        part[3 * blockIdx.x + 2] = c;
    }
}

// max |v| partials at part[3 b]
__global__ void __launch_bounds__(kThreads) max_abs_kernel(const double* __restrict__ v, int64_t n,
                                                          double* __restrict__ part)
{
    double mx = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads)
        mx = fmax(mx, fabs(v[i]));
    __shared__ double s[kWarps];
    mx = warp_max(mx);
    if (threadIdx.x % 32 == 0) s[threadIdx.x / 32] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int k = 0; k < kWarps; ++k) a = fmax(a, s[k]);
        part[3 * blockIdx.x + 0] = a;
        part[3 * blockIdx.x + 1] = 0.0;
        part[3 * blockIdx.x + 2] = 0.0;
    }
}

// stats[k] for k < 3 from the kRedBlocks partial triples (k = 0 max, else sum)
__global__ void reduce3_kernel(const double* __restrict__ part, double* __restrict__ stats)
{
    const int k = threadIdx.x;
    if (k >= 3) return;
    double a = 0.0;
    for (int b = 0; b < kRedBlocks; ++b) a = (k == 0) ? fmax(a, part[3 * b + k]) : a + part[3 * b + k];
    stats[k] = a;
}

__global__ void fb_diag_kernel(const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, const double* __restrict__ w,
                               const double* __restrict__ phi, int64_t n, double* __restrict__ Da,
                               double* __restrict__ Db, double* __restrict__ d)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool deg = z[i] != 0.0;
        const double a = deg ? z[i] : x[i], b = deg ? w[i] : y[i];
        const double r = sqrt(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
        Da[i] = __dsub_rn(__ddiv_rn(a, r), 1.0);
        Db[i] = __dsub_rn(__ddiv_rn(b, r), 1.0);
        d[i] = -phi[i];
    }
}

__global__ void scale_vec_kernel(const double* __restrict__ Db, const double* __restrict__ phi, int64_t n,
                                 double* __restrict__ v)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = __dmul_rn(Db[i], phi[i]);
}

// d = -(Da phi + d); partial sums of d^2 at part[3 b + 1]
__global__ void __launch_bounds__(kThreads) grad_dir_kernel(const double* __restrict__ Da,
                                                           const double* __restrict__ phi, int64_t n,
                                                           double* __restrict__ d, double* __restrict__ part)
{
    double sq = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        const double g = __dadd_rn(__dmul_rn(Da[i], phi[i]), d[i]);
        d[i] = -g;
        sq += g * g;
    }
    __shared__ double s[kWarps];
    sq = warp_sum(sq);
    if (threadIdx.x % 32 == 0) s[threadIdx.x / 32] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int k = 0; k < kWarps; ++k) a += s[k];
        part[3 * blockIdx.x + 0] = 0.0;
        part[3 * blockIdx.x + 1] = a;
        part[3 * blockIdx.x + 2] = 0.0;
    }
}

// Per-block partials of psi at every trial step, plus the non-finite count of
// d, at part[(kLsSteps + 1) b + k]
__global__ void __launch_bounds__(kThreads) line_search_kernel(const double* __restrict__ x,
                                                              const double* __restrict__ d,
                                                              const double* __restrict__ y,
                                                              const double* __restrict__ Md, int64_t n,
                                                              double* __restrict__ part)
{
    double acc[kLsSteps + 1];
#pragma unroll
    for (int k = 0; k <= kLsSteps; ++k) acc[k] = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
        const double xi = x[i], di = d[i], yi = y[i], mi = Md[i];
        acc[kLsSteps] += (isfinite(di) && isfinite(mi)) ? 0.0 : 1.0;
        double t = 1.0;
#pragma unroll
        for (int k = 0; k < kLsSteps; ++k) {
            const double p = fb(__dadd_rn(xi, __dmul_rn(t, di)), __dadd_rn(yi, __dmul_rn(t, mi)));
            acc[k] += p * p;
            t *= 0.5;
        }
    }
    __shared__ double s[kLsSteps + 1][kWarps];
    const int w = threadIdx.x / 32, l = threadIdx.x % 32;
#pragma unroll
    for (int k = 0; k <= kLsSteps; ++k) {
        const double v = warp_sum(acc[k]);
        if (l == 0) s[k][w] = v;
    }
    __syncthreads();
    if (threadIdx.x <= kLsSteps) {
        double a = 0.0;
        for (int q = 0; q < kWarps; ++q) a += s[threadIdx.x][q];
        part[(kLsSteps + 1) * blockIdx.x + threadIdx.x] = a;
    }
}

__global__ void line_search_reduce_kernel(const double* __restrict__ part, double* __restrict__ psi)
{
    const int k = threadIdx.x;
    if (k > kLsSteps) return;
    double a = 0.0;
    for (int b = 0; b < kRedBlocks; ++b) a += part[(kLsSteps + 1) * b + k];
    psi[k] = (k < kLsSteps) ? 0.5 * a : a;
}

__global__ void step_kernel(double* __restrict__ x, const double* __restrict__ d, double t, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = __dadd_rn(x[i], __dmul_rn(t, d[i]));
}

__global__ void friction_rhs_kernel(const double* __restrict__ b, const double* __restrict__ Sf, int64_t m,
                                    double* __restrict__ r, double* __restrict__ q)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const double s = Sf[i];
        r[i] = b[i];
        r[m + i] = __dsub_rn(b[m + i], s);
        r[2 * m + i] = __dsub_rn(b[2 * m + i], s);
        q[3 * m + i] = __dmul_rn(2.0, s);
        q[4 * m + i] = __dmul_rn(2.0, s);
    }
}

__global__ void friction_slip_kernel(const double* __restrict__ x, const double* __restrict__ y, int64_t m,
                                     double scl, double* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        out[i] = __dmul_rn(y[i], scl);
        out[m + i] = __dmul_rn(__dsub_rn(y[m + i], x[3 * m + i]), scl);
        out[2 * m + i] = __dmul_rn(__dsub_rn(y[2 * m + i], x[4 * m + i]), scl);
    }
}

__global__ void scale_identity_kernel(double* __restrict__ A, int64_t lda, int64_t n, double s,
                                      double* __restrict__ I)
{
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    for (int64_t c = blockIdx.y; c < n; c += gridDim.y) {
        A[r + c * lda] = __dmul_rn(A[r + c * lda], s);
        I[r + c * n] = (r == c) ? 1.0 : 0.0;
    }
}

// coef layout: field f of element r at coef[f * m + r]
enum { CF_A2, CF_B2, CF_C2, CF_A4, CF_B4, CF_C4, CF_A3, CF_B3, CF_C3, CF_A5, CF_B5, CF_C5, CF_L21, CF_L22, CF_L31,
       CF_L33, CF_COUNT };

__global__ void reduce_prep_kernel(const double* __restrict__ Da, const double* __restrict__ Db,
                                   const double* __restrict__ r, const double* __restrict__ mu, int64_t m,
                                   double* __restrict__ coef, double* __restrict__ u0)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
        const double w2 = __dmul_rn(2.0, mu[e]);
        u0[e] = 0.0;
#pragma unroll
        for (int h = 0; h < 2; ++h) {   // h = 0: blocks 2 / 4, h = 1: blocks 3 / 5
            const int64_t s = (1 + h) * m + e, t = (3 + h) * m + e;
            const double da = Da[t], db = Db[t], rt = r[t];
            double as, bs, cs, at, bt, ct;
            if (fabs(da) >= fabs(db)) {   // row t solved for d_t
                as = 0.0; bs = 0.0; cs = 1.0;
                at = __ddiv_rn(rt, da);
                bt = -__ddiv_rn(__dmul_rn(w2, db), da);
                ct = __ddiv_rn(db, da);
            } else {                      // row t solved for d_s; d_t becomes the unknown
                as = -__ddiv_rn(rt, db);
                bs = w2;
                cs = __ddiv_rn(da, db);
                at = 0.0; bt = 0.0; ct = 1.0;
            }
            double* c = coef + (int64_t)(6 * h) * m + e;
            c[0 * m] = as; c[1 * m] = bs; c[2 * m] = cs;
            c[3 * m] = at; c[4 * m] = bt; c[5 * m] = ct;
            const double das = Da[s], dbs = Db[s];
            coef[(int64_t)(CF_L21 + 2 * h) * m + e] = __dadd_rn(__dmul_rn(das, bs), __dmul_rn(dbs, bt));
            coef[(int64_t)(CF_L22 + 2 * h) * m + e] = __dadd_rn(__dmul_rn(das, cs), __dmul_rn(dbs, ct));
            u0[(1 + h) * m + e] = as;
        }
    }
}

__global__ void reduced_rhs_kernel(const double* __restrict__ r, const double* __restrict__ Da,
                                   const double* __restrict__ Db, const double* __restrict__ cu0,
                                   const double* __restrict__ coef, int64_t m, double* __restrict__ rhs)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 3 * m;
         i += (int64_t)gridDim.x * blockDim.x) {
        double v = __dsub_rn(r[i], __dmul_rn(Db[i], cu0[i]));
        if (i >= m) {
            const int64_t h = i / m - 1, e = i - (1 + h) * m;
            const double as = coef[(int64_t)(CF_A2 + 6 * h) * m + e], at = coef[(int64_t)(CF_A4 + 6 * h) * m + e];
            v = __dsub_rn(v, __dadd_rn(__dmul_rn(Da[i], as), __dmul_rn(Db[i], at)));
        }
        rhs[i] = v;
    }
}

__global__ void __launch_bounds__(kThreads) reduced_jacobian_kernel(const double* __restrict__ C, int64_t ldc,
                                                                   const double* __restrict__ mu,
                                                                   const double* __restrict__ Da,
                                                                   const double* __restrict__ Db,
                                                                   const double* __restrict__ coef, int64_t m,
                                                                   double* __restrict__ R, int64_t ldr)
{
    const int64_t n3 = 3 * m;
    const int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
    if (i >= n3) return;
    const double db = Db[i];
    const int64_t rb = i / m, ri = i - rb * m;
    for (int64_t col = blockIdx.y; col < n3; col += gridDim.y) {
        const int64_t cb = col / m, e = col - cb * m;
        double v;
        if (cb == 0) {
            const double g2 = __dsub_rn(coef[(int64_t)CF_B2 * m + e], mu[e]);
            const double g3 = __dsub_rn(coef[(int64_t)CF_B3 * m + e], mu[e]);
            v = __dadd_rn(__dadd_rn(C[i + e * ldc], __dmul_rn(g2, C[i + (m + e) * ldc])),
                          __dmul_rn(g3, C[i + (2 * m + e) * ldc]));
        } else {
            v = __dmul_rn(coef[(int64_t)(cb == 1 ? CF_C2 : CF_C3) * m + e], C[i + col * ldc]);
        }
        double out = __dmul_rn(db, v);
        if (ri == e) {
            double loc = 0.0;
            if (rb == 0 && cb == 0) loc = Da[i];
            else if (rb == 1 && cb == 0) loc = coef[(int64_t)CF_L21 * m + e];
            else if (rb == 1 && cb == 1) loc = coef[(int64_t)CF_L22 * m + e];
            else if (rb == 2 && cb == 0) loc = coef[(int64_t)CF_L31 * m + e];
            else if (rb == 2 && cb == 2) loc = coef[(int64_t)CF_L33 * m + e];
            out = __dadd_rn(out, loc);
        }
        R[i + col * ldr] = out;
    }
}

__global__ void recover_kernel(const double* __restrict__ v, const double* __restrict__ coef, int64_t m,
                               double* __restrict__ d)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
        const double v1 = v[e];
        d[e] = v1;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const double vs = v[(1 + h) * m + e];
            const double* c = coef + (int64_t)(6 * h) * m + e;
            d[(1 + h) * m + e] = __dadd_rn(__dadd_rn(c[0 * m], __dmul_rn(c[1 * m], v1)), __dmul_rn(c[2 * m], vs));
            d[(3 + h) * m + e] = __dadd_rn(__dadd_rn(c[3 * m], __dmul_rn(c[4 * m], v1)), __dmul_rn(c[5 * m], vs));
        }
    }
}

int grid_for(int64_t n)
{
    const int64_t g = (n + kThreads - 1) / kThreads;
    return (int)(g < 1 ? 1 : (g > 4 * kRedBlocks ? 4 * kRedBlocks : g));
}

unsigned cols_grid(int64_t n) { return (unsigned)(n < 32768 ? (n < 1 ? 1 : n) : 32768); }

}  // namespace

size_t lcp_partial_doubles() { return (size_t)kStat + 64; }

int lcp_matvec(const LcpOperator& op, const KrylovWork& kw, cudaStream_t st, const double* v, const double* q,
               double* out, double* u, int64_t* launches)
{
    if (!op.friction) {
        if (krylov_gemv<double>(st, op.M, op.ldm, (int)op.n, v, 1.0, q, out, kw, nullptr, 0, 0, launches) !=
            cudaSuccess)
            return 1;
        return 0;
    }
    const int64_t m = op.m;
    friction_pre_kernel<<<grid_for(m), kThreads, 0, st>>>(v, op.mu, m, u);
    if (launches) ++*launches;
    if (krylov_gemv<double>(st, op.C, op.ldc, (int)(3 * m), u, 1.0, nullptr, out, kw, nullptr, 0, 0, launches) !=
        cudaSuccess)
        return 1;
    friction_post_kernel<<<grid_for(m), kThreads, 0, st>>>(v, op.mu, q, m, out);
    if (launches) ++*launches;
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

int lcp_matvec_t(const LcpOperator& op, cudaStream_t st, const double* v, double* out, double* u, int64_t* launches)
{
    if (!op.friction) return krylov_gemv_t(st, op.M, op.ldm, op.n, op.n, v, out, launches) == cudaSuccess ? 0 : 1;
    const int64_t m = op.m;
    if (krylov_gemv_t(st, op.C, op.ldc, 3 * m, 3 * m, v, u, launches) != cudaSuccess) return 1;
    friction_post_t_kernel<<<grid_for(m), kThreads, 0, st>>>(v, op.mu, u, m, out);
    if (launches) ++*launches;
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

cudaError_t lcp_build_jacobian(const LcpOperator& op, const double* Da, const double* Db, double* J, int64_t ldj,
                               cudaStream_t st)
{
    if (op.n <= 0) return cudaSuccess;
    const dim3 grid((unsigned)((op.n + kThreads - 1) / kThreads), cols_grid(op.n));
    if (op.friction)
        jacobian_kernel<true><<<grid, kThreads, 0, st>>>(op.C, op.ldc, op.mu, op.m, op.n, Da, Db, J, ldj);
    else
        jacobian_kernel<false><<<grid, kThreads, 0, st>>>(op.M, op.ldm, nullptr, 0, op.n, Da, Db, J, ldj);
    return cudaGetLastError();
}

cudaError_t lcp_fb_eval(const double* x, const double* y, int64_t n, double* phi, double* z, double* part,
                        double* stats, cudaStream_t st, int64_t* launches)
{
    fb_eval_kernel<<<kRedBlocks, kThreads, 0, st>>>(x, y, n, phi, z, part);
    reduce3_kernel<<<1, 32, 0, st>>>(part, stats);
    if (launches) *launches += 2;
    return cudaGetLastError();
}

cudaError_t lcp_max_abs(const double* v, int64_t n, double* part, double* stats, cudaStream_t st, int64_t* launches)
{
    max_abs_kernel<<<kRedBlocks, kThreads, 0, st>>>(v, n, part);
    reduce3_kernel<<<1, 32, 0, st>>>(part, stats);
    if (launches) *launches += 2;
    return cudaGetLastError();
}

cudaError_t lcp_fb_diag(const double* x, const double* y, const double* z, const double* w, const double* phi,
                        int64_t n, double* Da, double* Db, double* d, cudaStream_t st, int64_t* launches)
{
    fb_diag_kernel<<<grid_for(n), kThreads, 0, st>>>(x, y, z, w, phi, n, Da, Db, d);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t lcp_scale(const double* Db, const double* phi, int64_t n, double* v, cudaStream_t st, int64_t* launches)
{
    scale_vec_kernel<<<grid_for(n), kThreads, 0, st>>>(Db, phi, n, v);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t lcp_grad_dir(const double* Da, const double* phi, int64_t n, double* d, double* part, double* stats,
                         cudaStream_t st, int64_t* launches)
{
    grad_dir_kernel<<<kRedBlocks, kThreads, 0, st>>>(Da, phi, n, d, part);
    reduce3_kernel<<<1, 32, 0, st>>>(part, stats);
    if (launches) *launches += 2;
    return cudaGetLastError();
}

cudaError_t lcp_line_search(const double* x, const double* d, const double* y, const double* Md, int64_t n,
                            double* part, double* psi, cudaStream_t st, int64_t* launches)
{
    line_search_kernel<<<kRedBlocks, kThreads, 0, st>>>(x, d, y, Md, n, part);
    line_search_reduce_kernel<<<1, 64, 0, st>>>(part, psi);
    if (launches) *launches += 2;
    return cudaGetLastError();
}

cudaError_t lcp_step(double* x, const double* d, double t, int64_t n, cudaStream_t st, int64_t* launches)
{
    step_kernel<<<grid_for(n), kThreads, 0, st>>>(x, d, t, n);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t friction_rhs(const double* b, const double* Sf, int64_t m, double* r, double* q, cudaStream_t st,
                         int64_t* launches)
{
    friction_rhs_kernel<<<grid_for(m), kThreads, 0, st>>>(b, Sf, m, r, q);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t friction_slip(const double* x, const double* y, int64_t m, double scl, double* out, cudaStream_t st,
                          int64_t* launches)
{
    friction_slip_kernel<<<grid_for(m), kThreads, 0, st>>>(x, y, m, scl, out);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t friction_reduce_prep(const double* Da, const double* Db, const double* r, const double* mu, int64_t m,
                                 double* coef, double* u0, cudaStream_t st, int64_t* launches)
{
    reduce_prep_kernel<<<grid_for(m), kThreads, 0, st>>>(Da, Db, r, mu, m, coef, u0);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t friction_reduced_rhs(const double* r, const double* Da, const double* Db, const double* cu0,
                                 const double* coef, int64_t m, double* rhs, cudaStream_t st, int64_t* launches)
{
    reduced_rhs_kernel<<<grid_for(3 * m), kThreads, 0, st>>>(r, Da, Db, cu0, coef, m, rhs);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t friction_reduced_jacobian(const double* C, int64_t ldc, const double* mu, const double* Da,
                                      const double* Db, const double* coef, int64_t m, double* R, int64_t ldr,
                                      cudaStream_t st)
{
    if (m <= 0) return cudaSuccess;
    const dim3 grid((unsigned)((3 * m + kThreads - 1) / kThreads), cols_grid(3 * m));
    reduced_jacobian_kernel<<<grid, kThreads, 0, st>>>(C, ldc, mu, Da, Db, coef, m, R, ldr);
    return cudaGetLastError();
}

cudaError_t friction_recover(const double* v, const double* coef, int64_t m, double* d, cudaStream_t st,
                             int64_t* launches)
{
    recover_kernel<<<grid_for(m), kThreads, 0, st>>>(v, coef, m, d);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t scale_and_identity(double* A, int64_t lda, int64_t n, double s, double* I, cudaStream_t st,
                               int64_t* launches)
{
    if (n <= 0) return cudaSuccess;
    const dim3 grid((unsigned)((n + kThreads - 1) / kThreads), cols_grid(n));
    scale_identity_kernel<<<grid, kThreads, 0, st>>>(A, lda, n, s, I);
    if (launches) ++*launches;
    return cudaGetLastError();
}

}  // namespace cad
