// Mixed-precision solve: FP32/TF32 LU preconditioner + FP64 GMRES (csrc/mixed.cu).
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "lu.h"

namespace cad {

// Casts A (FP64, n x n, lda) to A32 (n x n, leading dimension n), factorises
// A32 in place (partial pivoting; TF32 tensor-core trailing updates), forms
// the row permutation and inverts the 128-row diagonal blocks of both
// triangles into Dinv (mixed_dinv_floats(n) floats).  Returns an LU_* code;
// info as lu_factor_solve.
int mixed_prepare(const LuStreams& ls, const double* A, int64_t lda, int64_t n, float* A32, float* Dinv, int* ipiv,
                  int* perm, int* info, int nb);
size_t mixed_dinv_floats(int64_t n);
size_t mixed_sync_ints(int64_t n);   // flags, tickets and the failure word of one preconditioner apply

enum { GMRES_OK = 0, GMRES_NOT_CONVERGED = 1, GMRES_CUDA_ERROR = 2, GMRES_BLAS_ERROR = 3, GMRES_TIMEOUT = 4 };

struct GmresArgs {
    cublasHandle_t blas;
    cudaStream_t stream;
    int64_t n;
    const double* A;   // FP64 system matrix (n x n, lda)
    int64_t lda;
    const double* b;   // right-hand side (n)
    double* x;         // solution (n)
    const float* A32;  // FP32 LU factors from mixed_prepare
    const float* Dinv;
    const int* perm;
    double tol;        // relative residual ||b - A x|| / ||b||
    int max_iter;      // total GMRES iterations
    int restart;       // Krylov dimension per cycle
    // workspace
    double* V;         // n x (restart + 1)
    double* w;         // n
    double* z;         // n
    double* r;         // n
    double* hd;        // 2 (restart + 1)
    float* y32;        // n
    float* x32;        // n
    int* sync;         // mixed_sync_ints(n)
    int64_t* launches;
};

struct GmresResult {
    int status;
    int iterations;
    double rel_residual;   // of the returned x, recomputed in FP64
};

int gmres_ir_solve(const GmresArgs& a, GmresResult* res);

}  // namespace cad
