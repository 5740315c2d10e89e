// Mixed-precision solve: FP32/TF32 LU preconditioner + FP64 GMRES (csrc/mixed.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "lu.h"

namespace cad {

// Casts A (FP64, n x n, lda) to A32 (n x n, leading dimension mixed_ld(n)), factorises
// A32 in place (partial pivoting; TF32 tensor-core trailing updates), forms
// the row permutation and inverts the 128-row diagonal blocks of both
// triangles into Dinv (mixed_dinv_floats(n) floats).  Returns an LU_* code;
// info as lu_factor_solve.
int mixed_prepare(const LuStreams& ls, const double* A, int64_t lda, int64_t n, float* A32, float* Dinv, int* ipiv,
                  int* perm, int* info, int nb, bool inverses = true);
size_t mixed_dinv_floats(int64_t n);
// Leading dimension of the FP32 factors: n rounded up to a multiple of 4
// floats, so the TF32 trailing updates can stage them with TMA.
int64_t mixed_ld(int64_t n);
size_t mixed_sync_ints(int64_t n);   // flags, tickets and the failure word of one preconditioner apply

enum { GMRES_OK = 0, GMRES_NOT_CONVERGED = 1, GMRES_CUDA_ERROR = 2, GMRES_TIMEOUT = 4 };

struct GmresArgs {
    cudaStream_t stream;
    int64_t n;
    const double* A;   // FP64 system matrix (n x n, lda): the true residual of every restart
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
    // block-sparse preconditioner instead of the FP32 factors (when set):
    // n / 3 elements x spai_k 3 x 3 blocks at the neighbours spai_nbr
    const int* spai_nbr = nullptr;
    const float* spai_blocks = nullptr;
    int spai_k = 0;
    long wait_limit = 0;   // polls of a triangular-solve flag wait (0: kDefaultWaitLimit)
    double* kwork = nullptr;       // krylov_work_doubles(n) doubles of device scratch
    const float* A32mv = nullptr;  // if set, an FP32 copy of A (ld32) for the Arnoldi products
    int64_t ld32 = 0;
    int gemv_chunks = 0;           // column chunks of the Arnoldi product (0: the default)
};

struct GmresResult {
    int status;
    int iterations;
    double rel_residual;   // of the returned x, recomputed in FP64
};

int gmres_ir_solve(const GmresArgs& a, GmresResult* res);

// Many right-hand sides at once: classical iterative refinement on the FP32
// factors -- X += LU32 \ (float)(B - A X), the residual of every column from
// one FP64 GEMM, the corrections from one multi-column FP32 triangular solve
// -- until every column's ||b - A x|| / ||b|| <= tol, or until the largest
// ratio stops halving or max_iter is reached.  converged[c] (host) tells
// which columns made it; the caller finishes the others with GMRES.
struct IrArgs {
    LuStreams ls;
    int64_t n;
    const double* A;    // FP64 system matrix (n x n, lda)
    int64_t lda;
    const double* B;    // n x nrhs, ldb
    int64_t ldb;
    int nrhs;
    double* X;          // n x nrhs (leading dimension n), the solution
    float* A32;         // FP32 LU factors and pivots from mixed_prepare
    int* ipiv;
    int* perm;
    int* info;
    int nb;
    double tol;
    int max_iter;
    // workspace
    double* R;          // n x nrhs
    float* R32;         // n x nrhs
    float* X32;         // n x nrhs
    double* norms;      // 2 nrhs
    double* kwork = nullptr;   // krylov_work_doubles(n): one-column residuals as a GEMV (else a GEMM)
    // one column with these set: each correction LU32 \ R is two ticket-
    // ordered chain launches on the factors (explicit inverses of the
    // diagonal blocks from mixed_prepare) instead of a blocked triangular solve
    const float* Dinv = nullptr;   // mixed_dinv_floats(n)
    int* sync = nullptr;           // mixed_sync_ints(n)
    double* Z = nullptr;           // n doubles
    long wait_limit = 0;
};

struct IrResult {
    int status;         // GMRES_OK / GMRES_CUDA_ERROR / GMRES_TIMEOUT
    int iterations;
    double max_rel_residual;
};

int ir_solve_batched(const IrArgs& a, IrResult* res, std::vector<char>& converged);

// `iters` refinement sweeps with no host synchronisation (capturable in a
// CUDA graph); rel_out (device, 1 double) = the largest final column ratio
// ||b - A x|| / ||b||.  Returns a GMRES_* status (launch errors only).
int ir_solve_fixed(const IrArgs& a, int iters, double* rel_out);

// One crack of a grouped many-crack solve (device pointers): the FP64 system
// A (n x n, lda), right-hand side b and solution x (n); its FP32 factors A32
// (n_pad x n_pad, leading dimension n_pad, n_pad a multiple of 128, the
// identity past n), Dinv (mixed_dinv_floats(n_pad)), perm (n_pad), sync
// (mixed_sync_ints(n_pad), inside the caller's contiguous sync array), r, z
// (n_pad doubles), y32, x32 (n_pad floats) and where its relative residual
// goes.
struct CrackRec {
    const double* A;
    const double* b;
    double* x;
    float* A32;
    float* Dinv;
    int* perm;
    int* sync;
    double* r;
    double* z;
    float* y32;
    float* x32;
    double* rel;
    int lda, n, n_pad, pad;
};
// Every crack: A32 = (float) A padded, grouped FP32 LU (sys[p] describes
// cracks[p]'s A32, see lu_factor_group), then `sweeps` refinement sweeps x +=
// (LU)^-1 (b - A x) with FP64 residuals, all cracks in each launch; *rel of
// every crack at the end.  sync_all (sync_ints ints) holds every crack's sync
// words and is cleared before each sweep.  Returns a GMRES_* code.
int mixed_group_solve(const LuStreams& ls, const std::vector<CrackRec>& cracks, const std::vector<GroupSystem>& sys,
                      const CUtensorMap* dev_maps, int* infos, int* status, int* sync_all, size_t sync_ints,
                      int sweeps, int nb);
// `sweeps` more refinement sweeps of the given cracks (factors, x and r from
// an earlier mixed_group_solve), then their *rel.
int mixed_group_sweeps(const LuStreams& ls, const std::vector<CrackRec>& cracks, int* sync_all, size_t sync_ints,
                       int sweeps);

}  // namespace cad
