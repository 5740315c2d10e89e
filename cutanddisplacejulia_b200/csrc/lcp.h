// Linear complementarity problems on the device (csrc/lcp.cu): the operator
// of the frictional slip problem (src/SlipCalculator3D.jl:90-175) or a dense
// matrix, and the element-wise pieces of a Fischer-Burmeister Newton method.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "krylov.h"

namespace cad {

// The LCP matrix.  Dense: M (n x n, ldm).  Friction: M is never stored; it
// is the 5m x 5m matrix of src/SlipCalculator3D.jl:141-151 built from
// C = inv(A * Scl) (3m x 3m, ldc) and the friction coefficients mu (m):
//   [C11 - C12 dmu - C13 dmu   C12  C13  0  0]
//   [C21 - C22 dmu - C23 dmu   C22  C23  I  0]
//   [C31 - C32 dmu - C33 dmu   C32  C33  0  I]
//   [2 dmu                     -I   0    0  0]
//   [2 dmu                      0  -I    0  0]
struct LcpOperator {
    bool friction = false;
    int64_t n = 0;              // LCP dimension (5m for friction)
    const double* M = nullptr;  // dense
    int64_t ldm = 0;
    const double* C = nullptr;  // friction
    int64_t ldc = 0;
    const double* mu = nullptr;
    int64_t m = 0;
};

// Number of per-block partial slots the reductions below use, and the number
// of trial steps of one line-search launch (t = 1, 1/2, ..., 2^-(kLsSteps-1)).
constexpr int kRedBlocks = 148;
constexpr int kLsSteps = 40;
size_t lcp_partial_doubles();   // device workspace of the reductions

// out = M v (+ q when q is set).  u: 3m doubles of workspace (friction).
// (krylov work: krylov_work_doubles(n) of device scratch, n = the operator's
// size: 3m for friction)
int lcp_matvec(const LcpOperator& op, const KrylovWork& kw, cudaStream_t st, const double* v, const double* q,
               double* out, double* u, int64_t* launches);
// out = M^T v.  u: 3m doubles of workspace (friction).
int lcp_matvec_t(const LcpOperator& op, cudaStream_t st, const double* v, double* out, double* u, int64_t* launches);

// J (n x n, ldj) = diag(Da) + diag(Db) M.
cudaError_t lcp_build_jacobian(const LcpOperator& op, const double* Da, const double* Db, double* J, int64_t ldj,
                               cudaStream_t st);

// phi = FB(x, y), z = 1 where x_i = y_i = 0 (else 0); stats[0..2] = max |phi|,
// sum phi^2, number of such rows.  part: lcp_partial_doubles().
cudaError_t lcp_fb_eval(const double* x, const double* y, int64_t n, double* phi, double* z, double* part,
                        double* stats, cudaStream_t st, int64_t* launches);
// max |v| into stats[0] (the scale of q).
cudaError_t lcp_max_abs(const double* v, int64_t n, double* part, double* stats, cudaStream_t st,
                        int64_t* launches);
// Da, Db of the generalized Jacobian (rows with z set use (1, w_i)) and
// d = -phi (the Newton right-hand side).
cudaError_t lcp_fb_diag(const double* x, const double* y, const double* z, const double* w, const double* phi,
                        int64_t n, double* Da, double* Db, double* d, cudaStream_t st, int64_t* launches);
// Steepest descent on psi = |phi|^2 / 2: d = -(Da phi + s) where s = M^T (Db phi)
// already sits in d; stats[0] = |d|^2.  v: Db phi on entry is not needed.
cudaError_t lcp_grad_dir(const double* Da, const double* phi, int64_t n, double* d, double* part, double* stats,
                         cudaStream_t st, int64_t* launches);
// v = Db phi (operand of the gradient's M^T product).
cudaError_t lcp_scale(const double* Db, const double* phi, int64_t n, double* v, cudaStream_t st,
                      int64_t* launches);
// psi[k] = |FB(x + t_k d, y + t_k Md)|^2 / 2 for t_k = 2^-k, k < kLsSteps;
// psi[kLsSteps] = number of non-finite entries of d.
cudaError_t lcp_line_search(const double* x, const double* d, const double* y, const double* Md, int64_t n,
                            double* part, double* psi, cudaStream_t st, int64_t* launches);
// x += t d
cudaError_t lcp_step(double* x, const double* d, double t, int64_t n, cudaStream_t st, int64_t* launches);

// Frictional slip problem set-up and read-out (src/SlipCalculator3D.jl:158-175,
// :190-237): r = b - [0; Sf; Sf] (3m), whose product with C is the top of q;
// q_bottom = 2 Sf.
cudaError_t friction_rhs(const double* b, const double* Sf, int64_t m, double* r, double* q, cudaStream_t st,
                         int64_t* launches);
// Dn = y1 Scl, Dss = (y2 - x4) Scl, Dds = (y3 - x5) Scl into out (3m).
cudaError_t friction_slip(const double* x, const double* y, int64_t m, double scl, double* out, cudaStream_t st,
                          int64_t* launches);
// Newton direction of the friction LCP through a 3m x 3m system instead of
// the 5m x 5m one.  Rows L4 / L5 of J = diag(Da) + diag(Db) M couple only d4
// (d5), d2 (d3) and d1 of the same element; each such row is solved for d4_r
// when |Da4_r| >= |Db4_r|, else for d2_r (Da, Db lie on the circle
// (Da+1)^2 + (Db+1)^2 = 1, so the divisor is at least 1 - 1/sqrt(2)), and the
// result substituted into rows L1..L3.  The unknowns of the reduced system
// are v = [d1; d2 or d4; d3 or d5] per element; coef (16m) holds, per
// element, d2 = a2 + b2 v1 + c2 v2, d4 = a4 + b4 v1 + c4 v2, the same for
// 3 / 5, and the four local diagonal entries.  u0 (3m) = [0; a2; a3].
cudaError_t friction_reduce_prep(const double* Da, const double* Db, const double* r, const double* mu, int64_t m,
                                 double* coef, double* u0, cudaStream_t st, int64_t* launches);
// rhs (3m) = r_top - Db_top (C u0) - the local constants; cu0 = C u0.
cudaError_t friction_reduced_rhs(const double* r, const double* Da, const double* Db, const double* cu0,
                                 const double* coef, int64_t m, double* rhs, cudaStream_t st, int64_t* launches);
// R (3m x 3m, ldr): the reduced Newton matrix, entry by entry from C.
cudaError_t friction_reduced_jacobian(const double* C, int64_t ldc, const double* mu, const double* Da,
                                      const double* Db, const double* coef, int64_t m, double* R, int64_t ldr,
                                      cudaStream_t st);
// d (5m) from the reduced solution v (3m).
cudaError_t friction_recover(const double* v, const double* coef, int64_t m, double* d, cudaStream_t st,
                             int64_t* launches);

// A *= s (n x n, lda); I = identity (n x n, n).
cudaError_t scale_and_identity(double* A, int64_t lda, int64_t n, double s, double* I, cudaStream_t st,
                               int64_t* launches);

}  // namespace cad
