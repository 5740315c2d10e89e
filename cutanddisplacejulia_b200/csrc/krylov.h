// GMRES building blocks on the device (csrc/krylov.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace cad {

constexpr int kMaxBasis = 64;     // Krylov basis vectors one orthogonalisation handles
constexpr int kGemvChunks = 16;    // default column chunks of the matrix-vector product
constexpr int kMaxGemvChunks = 32;

// Device scratch of the kernels below (krylov_work_doubles(n) doubles).
struct KrylovWork {
    double* part;    // kMaxGemvChunks x n partial products
    double* dots1;   // blocks x kMaxBasis
    double* dots2;
    double* norms;   // blocks
    double* h1;      // kMaxBasis
    double* h2;
    double* scalar;  // a few device scalars for the caller
};
size_t krylov_work_doubles(int64_t n);
KrylovWork krylov_carve(double* base, int64_t n);
int krylov_blocks(int64_t n);

// y = (b ? b : 0) + alpha * A x (A column-major n x n, lda; FP64 or FP32
// storage, FP64 arithmetic).  With V set, also the first Gram-Schmidt pass's
// partial dot products of y with V's nv columns (consumed by
// krylov_orthogonalise).
template <typename TA>
cudaError_t krylov_gemv(cudaStream_t st, const TA* A, int64_t lda, int n, const double* x, double alpha,
                        const double* b, double* y, const KrylovWork& k, const double* V, int64_t ldv, int nv,
                        int64_t* launches, int nchunks = kGemvChunks);
// w := w - V h twice (classical Gram-Schmidt with re-orthogonalisation, the
// first pass's dots from krylov_gemv); hcol[0..nv) = h, hcol[nv] = ||w||;
// vnext = w / ||w||.  All on the device.
cudaError_t krylov_orthogonalise(cudaStream_t st, const double* V, int64_t ldv, int n, int nv, double* w,
                                 double* hcol, double* vnext, const KrylovWork& k, int64_t* launches);
// *out (device) = ||x||_2
cudaError_t krylov_norm(cudaStream_t st, const double* x, int n, double* out, const KrylovWork& k, int64_t* launches);
// out = x / *by (device scalar)
cudaError_t krylov_scale(cudaStream_t st, const double* x, int n, const double* by, double* out, int64_t* launches);
// out = V y (y: nv device values)
cudaError_t krylov_combine(cudaStream_t st, const double* V, int64_t ldv, int n, int nv, const double* y, double* out,
                           int64_t* launches);
// y += a x
cudaError_t krylov_axpy(cudaStream_t st, double a, const double* x, int n, double* y, int64_t* launches);
// B (ldb) = (float) A (n x n, lda)
cudaError_t krylov_cast_f32(cudaStream_t st, const double* A, int64_t lda, int64_t n, float* B, int64_t ldb,
                            int64_t* launches);

// y = A^T x (A column-major rows x cols, lda; FP64), cols outputs
cudaError_t krylov_gemv_t(cudaStream_t st, const double* A, int64_t lda, int64_t rows, int64_t cols, const double* x,
                          double* y, int64_t* launches);
// At (cols x rows, ldt) = -A^T (A rows x cols, lda)
cudaError_t krylov_transpose_neg(cudaStream_t st, const double* A, int64_t lda, int64_t rows, int64_t cols, double* At,
                                 int64_t ldt, int64_t* launches);

}  // namespace cad
