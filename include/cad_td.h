/*
 * cad_td.h -- C ABI of the B200 triangular-dislocation library (libcad_td.so).
 *
 * Drop-in boundary for the hot path of CutAndDisplaceJulia: the bodies of the
 * Threads.@threads loops of TD (src/TD.jl:146-214 and :273-384), TD_sum
 * (src/TD_sum.jl:1-41), the traction assembly of CalculateInfluenceMatrices3D
 * (src/CalculateInfluenceMatrices3D.jl:2-48, :73-114) and the dense solve
 * D = A\b of SlipCalculator3D (src/SlipCalculator3D.jl:1-33).  Julia binds
 * these with ccall; every argument is a plain pointer or number, nothing here
 * depends on any framework type.
 *
 * Conventions (all follow the reference's Julia layout):
 *   - FP64 everywhere.
 *   - Vertex lists P1, P2, P3 are N x 3 column-major (x of all triangles, then
 *     y, then z), exactly like Julia's P1List.
 *   - An influence matrix is M x N column-major: row = observation point,
 *     column = triangle.
 *   - Slip arguments are in the reference's order: Dss, Dds, Dn.
 *   - Host-pointer entry points take caller-owned host arrays (the library
 *     copies in and out); *_dev entry points take device pointers on the
 *     context's device and run asynchronously on the context's stream.
 *   - Every function returns a status code; cad_last_error() gives the message.
 *
 * Status codes mirror the reference's errors:
 *   CAD_ERR_DIMS             "Element size inputs must be the same dimensions"   (src/TD.jl:424)
 *   CAD_ERR_HS_ABOVE_SURFACE "Half-space solution: Z coordinates must be negative!" (src/TD.jl:617)
 * NaN outputs for observation points that lie on a triangle edge in the
 * triangle's plane are data, not errors (src/TD.jl:808-818, :1572-1595).
 */
#ifndef CAD_TD_H
#define CAD_TD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CAD_OK 0
#define CAD_ERR_DIMS 1
#define CAD_ERR_HS_ABOVE_SURFACE 2
#define CAD_ERR_UNSUPPORTED 3
#define CAD_ERR_CUDA 4
#define CAD_ERR_OOM 5
#define CAD_ERR_TIMEOUT 6
#define CAD_ERR_NOT_CONVERGED 7
#define CAD_ERR_SINGULAR 8
#define CAD_ERR_ARG 9
#define CAD_ERR_TOO_LARGE 10

/* Solvers for the dense system (cad_set_solver). */
#define CAD_SOLVER_LU64 0  /* FP64 LU with partial pivoting: the reference's A\b (default) */
#define CAD_SOLVER_MIXED 1 /* FP32 LU (TF32 tensor-core updates) preconditioning FP64 GMRES */
#define CAD_SOLVER_GMRES_SPAI 2 /* FP64 GMRES, block-sparse preconditioner of cad_set_preconditioner */
#define CAD_SOLVER_GMRES_LEARNED 3 /* as GMRES_SPAI; cad_slip_calculator first installs the context
                                      network's preconditioner for its mesh (cad_lpc_install_dev) */
#define CAD_SOLVER_GMRES_BLOCK_JACOBI 4 /* FP64 GMRES, inverses of A's 3 x 3 element self blocks */
#define CAD_SOLVER_GMRES 5 /* FP64 GMRES with no preconditioner */

/* Precision of the system-matrix assembly (cad_set_assembly). */
#define CAD_ASSEMBLY_FP64 0  /* every pair in FP64, as the reference (default) */
#define CAD_ASSEMBLY_MIXED 1 /* far-field pairs in FP32, near-field pairs in FP64 */

typedef struct cad_ctx cad_ctx;

/* Context: one device, one stream, its own workspace.  A context is used by
 * one host thread at a time; separate contexts may run concurrently. */
int cad_init(int device, cad_ctx** ctx);
int cad_destroy(cad_ctx* ctx);
const char* cad_last_error(const cad_ctx* ctx);
/* Run on an existing cudaStream_t (passed as void*; NULL is CUDA's default
 * stream).  The context starts on its own stream: cad_get_stream() before the
 * first cad_set_stream() returns it, for switching back. */
int cad_set_stream(cad_ctx* ctx, void* stream);
void* cad_get_stream(const cad_ctx* ctx);
/* Device time (ms, CUDA events on the context stream) of the most recent
 * launch of: 0 = the TD kernels of the last assembly or evaluation (with
 * shared edges: the edge kernels and the pair kernel together), 1 = dense
 * factorisation + solve, 2 = the
 * factorisation part of the last mixed-precision solve (cast to FP32, FP32 LU,
 * diagonal-block inverses; -1 after an FP64 LU solve). */
double cad_last_time_ms(const cad_ctx* ctx, int which);
/* Library version string. */
const char* cad_version(void);
/* Number of the library's own CUDA kernels launched through this context so
 * far.  No counterpart in the reference (an
 * accounting utility). */
int64_t cad_kernel_launches(const cad_ctx* ctx);
/* Solver of the dense 3N x 3N system used by cad_slip_calculator, cad_solve and
 * cad_solve_dev from now on.  CAD_SOLVER_LU64 (default) factorises in FP64 as
 * the reference's A\b (src/SlipCalculator3D.jl:22) does.  CAD_SOLVER_MIXED has
 * no counterpart in the reference: A is cast to FP32 and factorised with
 * TF32 tensor-core trailing updates; restarted GMRES in FP64, right-
 * preconditioned by that factorisation, iterates until ||b - A x|| / ||b|| <=
 * tol (computed in FP64) or max_iter iterations (then CAD_ERR_NOT_CONVERGED,
 * with the last iterate returned).  Several right-hand sides are first
 * refined together (FP64 residuals of all columns from one GEMM, corrections
 * from the FP32 factors); GMRES finishes any column the refinement leaves.
 * The TF32 updates make the FP32 factors accurate to ~1e-3 relative, so the
 * mixed solver suits condition numbers up to ~1e3-1e4 (the influence systems
 * are ~1e2); take the FP64 LU for ill-conditioned systems.  In mixed mode
 * cad_solve_dev leaves A unchanged. */
int cad_set_solver(cad_ctx* ctx, int mode, double tol, int max_iter);
/* Precision of the 3N x 3N system matrix built by cad_assemble_dev and
 * cad_slip_calculator from now on.  CAD_ASSEMBLY_FP64 (default) evaluates
 * every pair in FP64 like the reference (src/CalculateInfluenceMatrices3D.jl).
 * CAD_ASSEMBLY_MIXED has no counterpart in the reference: pairs are evaluated
 * in FP32 (coordinates relative to each triangle origin formed in FP64), then
 * every 128-element tile that holds a collocation point within near_factor
 * mean edge lengths of a source triangle's centroid is evaluated again in
 * FP64 for that triangle (the near field, where the log and atan terms
 * cancel).  The matrix is stored in FP64 either way.  The traction influence
 * matrices of cad_influence_traction are always FP64. */
int cad_set_assembly(cad_ctx* ctx, int mode, double near_factor);
/* GMRES iterations (summed over right-hand sides) and the largest final
 * relative residual of the last mixed solve. */
int cad_last_solve_stats(const cad_ctx* ctx, int* iterations, double* rel_residual);
/* Autotuning of launch shapes (no counterpart in the reference): mode 0
 * (default) uses fixed shapes; 1 uses the shapes stored in cache_path (a text
 * file of "key value" lines, may be NULL) and times the candidates of any key
 * not there on its first use, adding the winner to the file; 2 uses stored
 * shapes only.  Keys are (kernel, size class = the power of two at or above
 * the size, precision): the pair kernel's triangles per block for the FP64
 * system matrix, the Arnoldi product's column chunks, and the FP64 LU's leaf
 * width (timed on a scratch copy of A, systems up to 12288 unknowns).  A call
 * that meets a new key in mode 1 runs each candidate twice first.
 * cad_autotune_entries: the number of stored keys (and, in tuned_here, how many
 * this process timed). */
int cad_set_autotune(cad_ctx* ctx, int mode, const char* cache_path);
int64_t cad_autotune_entries(const cad_ctx* ctx, int64_t* tuned_here);
/* Arnoldi products of the preconditioned-GMRES solvers (CAD_SOLVER_GMRES_*):
 * fp32 = 1 (default) multiplies with an FP32 copy of A (half the bytes per
 * iteration; the solve keeps an extra n x n FP32 array), every restart still
 * forming the residual b - A x in FP64, so the tolerance is met in FP64;
 * fp32 = 0 multiplies with the FP64 A.  No counterpart in the reference. */
int cad_set_gmres_matvec(cad_ctx* ctx, int fp32);
/* How cad_slip_calculator_batched* factorises and refines its cracks (every
 * mode gives the same slips to the refinement tolerance; no counterpart in
 * the reference, whose cracks are solved one SlipCalculator3D call at a
 * time):
 *   CAD_BATCH_GROUPED (default): after each crack's assembly, one launch per
 *     step and kind covers every crack -- the FP32 blocked LU (cluster leaves,
 *     row swaps, triangular blocks, TF32 tcgen05 products) and the FP64
 *     refinement sweeps (ticket-ordered triangular chains, FP64 residuals);
 *     cracks above 3N = 512 x the largest leaf cluster take the lanes path;
 *   CAD_BATCH_LANES: every crack's own factorisation and sweeps on 32 stream
 *     lanes, triangular solves in 64-row blocks;
 *   CAD_BATCH_LANES_CHAIN: the lanes with ticket-ordered chain solves. */
/* Outer block width of the dense LU of a single system (the FP64 solve, the
 * mixed solve's FP32 factorisation): 32..1024 columns, 0 = the library's
 * defaults (256 for FP64, 512 for FP32).  Wider blocks give the trailing-
 * update products a longer inner dimension and the panels more work.  Same factors and pivots up to
 * the order of the products' sums.  No counterpart in the reference. */
int cad_set_lu_block(cad_ctx* ctx, int nb);
/* Krylov dimension of one restarted-GMRES cycle (the mixed and the
 * preconditioned GMRES solvers): 1..63, 0 = the default 30.  Every cycle
 * starts from the FP64 residual b - A x.  No counterpart in the reference. */
int cad_set_gmres_restart(cad_ctx* ctx, int m);
/* Half-space work on meshes whose triangles share edges (fewer edges than
 * 0.9 x the triangle sides; other meshes always take the per-side path).
 * 1 (default): the FP64 system matrix and traction influence fields
 * (cad_assemble*, cad_slip_calculator*, cad_influence_traction with hs_flag
 * 1) evaluate the free-surface correction of each mesh edge once per
 * collocation point, and the triangles that share the edge reuse it
 * with the sign of their side's direction, and so do the influence fields
 * (cad_td_inf*, strain and displacement maps per edge); the summed evaluations
 * (cad_td_sum_eval*) evaluate it once per edge for the net Burgers vector of
 * the sides on it.  0: per triangle side, as the reference does.  Same
 * results to rounding.  No counterpart in the reference. */
int cad_set_shared_edges(cad_ctx* ctx, int enable);
#define CAD_BATCH_GROUPED 0
#define CAD_BATCH_LANES 1
#define CAD_BATCH_LANES_CHAIN 2
int cad_set_batch_solve(cad_ctx* ctx, int mode);
/* Device waits (a leaf's pivot exchange, a triangular-solve chain flag) poll
 * at most `polls` times (default 4194304, a few seconds at worst) before the
 * kernel records the failure and returns; the call then reports
 * CAD_ERR_TIMEOUT and the context stays usable.  No counterpart in the
 * reference (its waits are CPU thread joins). */
int cad_set_wait_limit(cad_ctx* ctx, int64_t polls);
/* Exercises that timeout path on an n x n zero system (128 <= n <= 8192): the
 * lower chain of the one-right-hand-side solve is launched with its order
 * counter started past block 0, so every block waits for a flag that no block
 * sets.  Returns CAD_ERR_TIMEOUT once the waits run out (the kernels end
 * normally; nothing faults or hangs). */
int cad_wait_timeout_probe(cad_ctx* ctx, int64_t n);
/* Measured FP64 fused-multiply-add throughput of the device (TFLOP/s, 2 flops
 * per FMA), the denominator of the TD kernels' roofline.  No counterpart in
 * the reference (a measurement utility). */
int cad_fp64_fma_probe(cad_ctx* ctx, int64_t iters, double* tflops);

/* ---------------------------------------------------------------- TD ----
 * TD influence-matrix overloads (replaces src/TD.jl:77-133 allocation and the
 * loop body of src/TD.jl:135-216).  strain_out: 18 pointers to M x N arrays in
 * StrainInf field order (exxDn, eyyDn, ezzDn, exyDn, exzDn, eyzDn, then the
 * same for Dss and Dds); disp_out: 9 pointers in DispInf order (DnUx, DnUy,
 * DnUz, DssUx, ..., DdsUz).  A flag of 0 leaves the matching pointer array
 * unused (it may be NULL).  G is accepted for signature parity; the reference
 * does not use it for strain or displacement. */
int cad_td_inf(cad_ctx* ctx, const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
               const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds,
               const double* Dn, double nu, double G, int disp_flag, int strain_flag, int hs_flag,
               double* const* strain_out, double* const* disp_out);

/* TD summing overload (replaces the loop of src/TD.jl:219-410): strain_out 6
 * pointers (exx, eyy, ezz, exy, exz, eyz), disp_out 3 pointers (Ux, Uy, Uz),
 * each of length M: the sum over triangles and slip modes.  Deterministic
 * (fixed summation order), unlike the reference's shared accumulation. */
int cad_td_sum_eval(cad_ctx* ctx, const double* X, const double* Y, const double* Z, int64_t M,
                    const double* P1, const double* P2, const double* P3, int64_t N, const double* Dss,
                    const double* Dds, const double* Dn, double nu, double G, int disp_flag, int strain_flag,
                    int hs_flag, double* const* strain_out, double* const* disp_out);

/* TD_sum (src/TD_sum.jl:1-41): sum 18 strain / 9 displacement influence
 * matrices (M x N, field orders as above) over modes and columns.  Either
 * input array may be NULL (then its outputs are untouched). */
int cad_td_sum(cad_ctx* ctx, int64_t M, int64_t N, const double* const* strain_in, const double* const* disp_in,
               double* const* strain_out, double* const* disp_out);

/* ------------------------------------------------------------ assembly ---
 * CalculateInfluenceMatrices3D (src/CalculateInfluenceMatrices3D.jl:2-48):
 * normals and midpoints N x 3 (FaceNormalVector, MidPoint), vertex lists
 * N x 3; trac_out: 9 pointers to N x N arrays in TractionInf order (DnTn,
 * DnTss, DnTds, DssTn, DssTss, DssTds, DdsTn, DdsTss, DdsTds).  fixed_els
 * (N values, may be NULL): with elements marked 1, the rows of those elements
 * hold the displacement influence at their collocation points (DnUx in DnTn,
 * DnUy in DnTss, DnUz in DnTds, and so on by field) and only the columns of
 * the other n_free elements are kept (ConcatInfMats / PutDispInfsIntoInfMat,
 * src/CalculateInfluenceMatrices3D.jl:145-199): each trac_out field is then
 * N x n_free. */
int cad_influence_traction(cad_ctx* ctx, const double* normals, const double* midpoints, const double* P1,
                           const double* P2, const double* P3, int64_t N, double nu, double G, double lambda,
                           const double* fixed_els, int hs_flag, double* const* trac_out);

/* SlipCalculator3D for traction-vector boundary conditions
 * (src/SlipCalculator3D.jl:1-33): assembles A = -[Atn;Atss;Atds] (3N x 3N) and
 * solves A D = [Tn; Tss; Tds] by LU with partial pivoting.  Outputs Dn, Dss,
 * Dds (N each); A_out (3N x 3N) and b_out (3N) may be NULL. */
int cad_slip_calculator(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, double nu,
                        double G, double lambda, const double* midpoints, const double* normals, int hs_flag,
                        const double* Tn, const double* Tss, const double* Tds, double* Dn, double* Dss,
                        double* Dds, double* A_out, double* b_out);

/* SlipCalculator3D with fixed elements (src/SlipCalculator3D.jl:1-33 with
 * FixedEls, src/KnockOutFixedRows.jl): the tractions of fixed elements are set
 * to zero, A (3N x 3 n_free) has displacement rows for them and no columns,
 * and A D = b is solved in the least-squares sense (the reference's `\` on a
 * tall matrix) through the normal equations and the FP64 LU.  Dn, Dss, Dds:
 * n_free values each (elements not fixed, in order); A_out (3N x 3 n_free)
 * and b_out (3N) may be NULL.  Without fixed elements this is
 * cad_slip_calculator. */
int cad_slip_calculator_fixed(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N,
                              double nu, double G, double lambda, const double* midpoints, const double* normals,
                              int hs_flag, const double* Tn, const double* Tss, const double* Tds,
                              const double* fixed_els, double* Dn, double* Dss, double* Dds, double* A_out,
                              double* b_out);

/* SlipCalculator3D with friction (MixedBoundaryConditionsFriction,
 * src/SlipCalculator3D.jl:36-238).  Tn, Tss, Tds: element tractions of the
 * boundary conditions (remote stress resolved on the elements plus applied
 * tractions, as the frictionless call takes them); mu, Sf: friction
 * coefficient and cohesion per element (N each).  When no element can
 * overcome its frictional resistance Tn*mu on both shear components
 * (:46-55) the slip is zero.  Otherwise A (3N x 3N, as cad_slip_calculator)
 * is scaled by Scl = mean half-perimeter / G, C = inv(A Scl), and the 5N x 5N
 * linear complementarity problem of :90-175 is solved by a Fischer-Burmeister
 * Newton method (the reference calls FischerNewton.fischer_newton, :196) to
 * max|Phi| <= tol max|q| within max_iter Newton steps; Dn = y1 Scl,
 * Dss = (y2 - x4) Scl, Dds = (y3 - x5) Scl (:197-237).  The results are
 * written also when the tolerance is not met, which returns
 * CAD_ERR_NOT_CONVERGED; cad_last_solve_stats() gives the Newton steps and
 * the final max|Phi| / max|q|. */
int cad_slip_calculator_friction(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N,
                                 double nu, double G, double lambda, const double* midpoints, const double* normals,
                                 int hs_flag, const double* Tn, const double* Tss, const double* Tds,
                                 const double* mu, const double* Sf, double tol, int max_iter, double* Dn,
                                 double* Dss, double* Dds);

/* The two halves of cad_slip_calculator_friction, for many loads on one
 * geometry (the reference prepares the LCP once, src/SlipCalculator3D.jl:90-175,
 * and solves it per load, :177-238, as its fluid-volume search does).
 * cad_friction_prepare assembles A and keeps C = inv(A Scl) in the context;
 * cad_friction_solve solves the LCP for one set of element tractions and
 * friction parameters with it (no early exit: the caller decides, as the
 * reference's prepared overloads do).  The prepared system stays valid until
 * the next cad_friction_prepare, cad_slip_calculator_friction or
 * cad_fischer_newton call on the context; cad_friction_solve returns
 * CAD_ERR_ARG when there is none of N elements. */
int cad_friction_prepare(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, double nu,
                         double G, double lambda, const double* midpoints, const double* normals, int hs_flag);
int cad_friction_solve(cad_ctx* ctx, int64_t N, const double* Tn, const double* Tss, const double* Tds,
                       const double* mu, const double* Sf, double tol, int max_iter, double* Dn, double* Dss,
                       double* Dds);

/* Linear complementarity problem x >= 0, y = A x + b >= 0, x'y = 0 for a dense
 * A (n x n, column-major) and b (n): the call FischerNewton.fischer_newton(A, b)
 * makes at src/SlipCalculator3D.jl:196, solved by the same Fischer-Burmeister
 * Newton method as cad_slip_calculator_friction, from x = 0.  x: n values
 * (written also when CAD_ERR_NOT_CONVERGED is returned). */
int cad_fischer_newton(cad_ctx* ctx, int64_t n, const double* A, const double* b, double tol, int max_iter,
                       double* x);

/* Dense solve A X = B (the `\` of src/SlipCalculator3D.jl:22): A n x n, B n x
 * nrhs, both column-major host arrays; X n x nrhs. */
int cad_solve(cad_ctx* ctx, int64_t n, const double* A, const double* B, int64_t nrhs, double* X);

/* ------------------------------------------------ device-pointer variants ---
 * Same semantics, device pointers, asynchronous on the context stream (the
 * half-space argument check synchronises once).  Multi-field outputs are one
 * contiguous buffer: field f of an M x N result starts at out + f*M*N. */
int cad_td_inf_dev(cad_ctx* ctx, const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
                   const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds,
                   const double* Dn, double nu, int disp_flag, int strain_flag, int hs_flag, double* strain_out,
                   double* disp_out);
int cad_td_sum_eval_dev(cad_ctx* ctx, const double* X, const double* Y, const double* Z, int64_t M,
                        const double* P1, const double* P2, const double* P3, int64_t N, const double* Dss,
                        const double* Dds, const double* Dn, double nu, int disp_flag, int strain_flag,
                        int hs_flag, double* strain_out, double* disp_out);
/* Assemble A = -[Atn;Atss;Atds] (3N x 3N, leading dimension lda >= 3N). */
int cad_assemble_dev(cad_ctx* ctx, const double* normals, const double* midpoints, const double* P1,
                     const double* P2, const double* P3, int64_t N, double nu, double G, double lambda, int hs_flag,
                     double* A, int64_t lda);
/* Incremental re-assembly (no counterpart in the reference, whose
 * propagation loop re-assembles the whole system every step,
 * test/test_PropagationTest.jl:398): after the geometry of the k elements
 * `changed` (host, indices < N) changed, recompute their rows and columns of
 * an A built by cad_assemble_dev for the same N (FP64, every other entry kept);
 * the arguments are the updated geometry. */
int cad_assemble_update_dev(cad_ctx* ctx, const double* normals, const double* midpoints, const double* P1,
                            const double* P2, const double* P3, int64_t N, double nu, double G, double lambda,
                            int hs_flag, const int64_t* changed, int64_t k, double* A, int64_t lda);
/* A column block of the system matrix of cad_assemble_dev: the columns of
 * elements j0 .. j1-1 (all 3N rows), for sharding the assembly across GPUs
 * with no exchange (the reference fills whole columns per thread,
 * src/CalculateInfluenceMatrices3D.jl:84-112).  A_block (3N x 3(j1-j0), lda
 * >= 3N) holds the Dn columns of the block, then its Dss columns, then its
 * Dds columns, each as in A = -[Atn;Atss;Atds]. */
int cad_assemble_columns_dev(cad_ctx* ctx, const double* normals, const double* midpoints, const double* P1,
                             const double* P2, const double* P3, int64_t N, double nu, double G, double lambda,
                             int hs_flag, int64_t j0, int64_t j1, double* A_block, int64_t lda);
/* In-place LU solve: A (n x n, lda) is overwritten by its LU factors, B
 * (n x nrhs, ldb) by the solution. */
int cad_solve_dev(cad_ctx* ctx, int64_t n, double* A, int64_t lda, double* B, int64_t ldb, int64_t nrhs);
/* C (m x n, ldc) -= A (m x k, lda) * B (k x n, ldb), column-major device
 * arrays, precision 0 = FP64 (DMMA tensor cores), 1 = FP32 (TF32 tensor cores
 * through tcgen05 when A and B start on 16-byte boundaries and lda, ldb are
 * multiples of 4; FP32 CUDA cores otherwise); 2, 3, 4 = FP64 with the DMMA
 * shape m8n8k4, m16n8k8 or m16n8k16 (precision 0 takes the library's
 * default shape).  The trailing-update product of
 * the dense LU that replaces the reference's A\b (src/SlipCalculator3D.jl:22),
 * exposed on its own for testing and measurement; synchronises the context
 * stream. */
int cad_gemm_sub_dev(cad_ctx* ctx, int precision, int64_t m, int64_t n, int64_t k, const void* A, int64_t lda,
                     const void* B, int64_t ldb, void* C, int64_t ldc);

/* ---------------------------------------------- learned preconditioner ---
 * No counterpart in the reference (its only solver is the dense A\b).  A
 * block-sparse approximate inverse M (N elements x k blocks of 3 x 3, FP32,
 * row-major; block q of element i acts on the unknowns of element
 * nbr[i*k + q], unknown order [Dn; Dss; Dds] as in SlipCalculator3D)
 * right-preconditions FP64 restarted GMRES when the solver is
 * CAD_SOLVER_GMRES_SPAI.  The device arrays are used in place: keep them
 * alive while the setting stands.  cad_block_jacobi_dev fills the k = 1
 * block-Jacobi preconditioner (inverses of the 3 x 3 self blocks of A). */
int cad_set_preconditioner(cad_ctx* ctx, int64_t N, int k, const int* nbr, const float* blocks);
int cad_block_jacobi_dev(cad_ctx* ctx, int64_t N, const double* A, int64_t lda, int* nbr, float* blocks);
/* The network that predicts M's blocks from each element's 16 nearest
 * elements: 112 inputs (per neighbour: centroid offset and normal in the
 * element's own frame, area ratio), two hidden layers of 256 (ReLU), 144
 * outputs (16 blocks of 9), BF16 weights and activations, FP32 accumulation,
 * FP32 master weights (cad_lpc_param_count floats: W1, b1, W2, b2, W3, b3,
 * each W in x out, row-major).  cad_lpc_step runs one pass over `rows`
 * samples (device X rows x 112, T rows x 144): the output to `out` if set;
 * with grads set, the gradient of the mean squared error against T and, with
 * loss set, the sum of squared errors (device float); with adam_m and adam_v
 * set, one Adam step (step number t >= 1, step size lr) on params. */
int64_t cad_lpc_param_count(void);
int cad_lpc_step(cad_ctx* ctx, float* params, const float* X, const float* T, int64_t rows, float* out, float* grads,
                 float* loss, float* adam_m, float* adam_v, int64_t t, float lr);
/* The learned path without any host-side numerics (no counterpart in the
 * reference):
 * - cad_lpc_features_dev: device vertex lists (N x 3 column-major) -> the
 *   network inputs X (N x 112), the 16 nearest elements of each element by
 *   centroid distance, itself first (nbr, N x 16), and h = sqrt(2 area)
 *   (N, may be NULL); all device arrays.
 * - cad_lpc_set_network / cad_lpc_get_network: the context's network weights
 *   (host, cad_lpc_param_count floats); setting them resets the Adam state.
 * - cad_lpc_dataset_add: appends one mesh to the context's training set
 *   (host arrays as cad_slip_calculator): the library assembles its FP64
 *   system, inverts it with the FP64 LU and keeps, per element, its features
 *   and the 16 3 x 3 blocks of A^-1 toward its neighbours divided by h / G.
 *   cad_lpc_dataset_rows / _clear: its size (elements) / empty it.
 * - cad_lpc_train: `steps` Adam steps (cosine step size from lr) on
 *   minibatches of `batch` rows drawn from the training set by a seeded hash;
 *   loss_hist (host, ceil(steps / 100) floats, may be NULL) gets the mean
 *   squared error of every 100th minibatch.
 * - cad_lpc_install_dev / cad_lpc_install (host vertex lists): runs the
 *   network on a mesh and installs the blocks (x h / G) as the context's
 *   preconditioner for CAD_SOLVER_GMRES_SPAI / _LEARNED solves; the arrays
 *   belong to the context. */
int cad_lpc_features_dev(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, float* X,
                         int* nbr, double* h);
int cad_lpc_set_network(cad_ctx* ctx, const float* params);
int cad_lpc_get_network(cad_ctx* ctx, float* params);
int cad_lpc_dataset_add(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, double nu,
                        double G, double lambda, const double* midpoints, const double* normals, int hs_flag);
int64_t cad_lpc_dataset_rows(const cad_ctx* ctx);
int cad_lpc_dataset_clear(cad_ctx* ctx);
/* Host-array forms: cad_lpc_dataset_set replaces the training set by `rows`
 * host rows (X rows x 112, T rows x 144); cad_lpc_dataset_get copies rows
 * row0 .. row0 + rows - 1 of it out; cad_lpc_forward_backward runs the
 * context's network over host rows X and returns its outputs (out, rows x
 * 144, may be NULL) and, with T set, the gradient of the mean squared error
 * (grads, cad_lpc_param_count floats) and the sum of squared errors (loss). */
int cad_lpc_dataset_set(cad_ctx* ctx, const float* X, const float* T, int64_t rows);
int cad_lpc_dataset_get(cad_ctx* ctx, int64_t row0, int64_t rows, float* X, float* T);
int cad_lpc_forward_backward(cad_ctx* ctx, const float* X, const float* T, int64_t rows, float* out, float* grads,
                             float* loss);
int cad_lpc_train(cad_ctx* ctx, int64_t steps, int64_t batch, float lr, uint64_t seed, float* loss_hist);
int cad_lpc_install_dev(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, double G);
int cad_lpc_install(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, double G);

/* Batched SlipCalculator3D over independent cracks (no counterpart in the
 * reference, which solves one crack per call; src/SlipCalculator3D.jl:1-33 per
 * crack).  Device pointers; crack c has N_c = offsets[c+1] - offsets[c]
 * triangles (offsets: host array of nbatch + 1, offsets[0] = 0) and its
 * arrays start at 3 * offsets[c]: its N_c x 3 column-major P1, P2, P3,
 * normals and midpoints, its traction vector [Tn; Tss; Tds] in T and its
 * slip [Dn; Dss; Dds] in D.  Each crack is assembled at the context's
 * assembly precision (cad_set_assembly) and solved by FP32 LU (TF32
 * updates) with FP64 refinement to the context's tolerance (cad_set_solver),
 * GMRES finishing any crack the refinement leaves.  The cracks run
 * concurrently on 32 stream lanes inside one CUDA graph, captured on the first
 * call with these arguments and replayed by identical calls.  Needs device
 * memory for every crack's 3N_c x 3N_c matrix at once.  rel_residual (host,
 * nbatch, may be NULL): each crack's final ||b - A D|| / ||b||. */
int cad_slip_calculator_batched_dev(cad_ctx* ctx, int64_t nbatch, const int64_t* offsets, const double* P1,
                                    const double* P2, const double* P3, const double* normals,
                                    const double* midpoints, double nu, double G, double lambda, int hs_flag,
                                    const double* T, double* D, double* rel_residual);

/* The same with host arrays (copied in and out by the library). */
int cad_slip_calculator_batched(cad_ctx* ctx, int64_t nbatch, const int64_t* offsets, const double* P1,
                                const double* P2, const double* P3, const double* normals, const double* midpoints,
                                double nu, double G, double lambda, int hs_flag, const double* T, double* D,
                                double* rel_residual);

/* -------------------------------------------------- no-allocation variant ---
 * Summing-overload evaluation that allocates no device memory, for callers
 * that cannot allow a library to call cudaMalloc: hosts whose device memory is
 * owned by their own pool and budget (a hidden allocation can fail under
 * memory pressure or break the pool's accounting), and services that fix each
 * tenant's device memory at start-up.  No counterpart in the reference.
 *
 * Same arguments and results as cad_td_sum_eval_dev (device pointers: X, Y, Z
 * of length M; P1, P2, P3 N x 3; slips of length N; strain_out 6 x M;
 * disp_out 3 x M), but no context: it runs on `stream` (NULL is CUDA's
 * default stream) and returns only a status code.  Its intermediates live in
 * one fixed device array of about 25 MiB that every GPU loading the library
 * reserves until the process exits; limits are N <= 1024 triangles and
 * M <= 16384 points (CAD_ERR_TOO_LARGE beyond).  Calls share that array, so
 * calls that overlap on the GPU race; order them on one stream.  The first
 * call on a device looks up the array's address with that device current:
 * make it before any stream capture.  With hs_flag = 1 every call
 * synchronises `stream`: the half-space check reads its flag back to the
 * host before the evaluation starts, as in the other entry points. */
int cad_td_sum_eval_noalloc(void* stream, const double* X, const double* Y, const double* Z, int64_t M,
                            const double* P1, const double* P2, const double* P3, int64_t N, const double* Dss,
                            const double* Dds, const double* Dn, double nu, int disp_flag, int strain_flag,
                            int hs_flag, double* strain_out, double* disp_out);

#ifdef __cplusplus
}
#endif

#endif /* CAD_TD_H */
