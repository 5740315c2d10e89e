// Dense LU with partial pivoting + solve (csrc/lu.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace cad {

enum { LU_OK = 0, LU_CUDA_ERROR = 1, LU_TOO_LARGE = 3 };

// Executable CUDA graphs of lu_factor_solve calls, one per call signature
// (precision, sizes, every pointer and the streams).  The factorisation
// is thousands of dependent launches -- leaves, row swaps, triangular blocks,
// GEMMs -- whose launch gaps dominate at moderate n; a signature seen a second
// time is captured once and replayed from then on as a single graph launch.
// The first call of a signature runs eagerly (no capture cost for one-off
// calls).  Owned by one context (not thread-safe).
struct LuGraphCache;
LuGraphCache* lu_graph_cache_create();
void lu_graph_cache_destroy(LuGraphCache* c);

// Where the factorisation runs: the caller's stream, plus an optional side
// stream for the look-ahead's trailing updates (side null: everything on the
// main stream).  The result is ordered on the main stream.
struct LuStreams {
    cudaStream_t main;
    cudaStream_t side;
    int64_t* launches;       // if set, incremented by the number of own kernel launches
    LuGraphCache* graphs;    // if set, repeated call signatures replay a captured graph
    long wait_limit = 0;     // polls a device wait makes before it gives up (0: kDefaultWaitLimit)
    int min_leaf_rpt = 1;    // fewest rows per leaf thread (1, 2, 4): leaves of 32 / rpt columns
    // grouped factorisations: streams on which the leaf launches of different
    // cluster sizes run side by side (none: one after the other on main)
    cudaStream_t* aux = nullptr;
    int naux = 0;
};

// Polls of a device-side wait (a pivot exchange, a chain flag) before the
// kernel gives up, records the failure in the info word and returns.
constexpr long kDefaultWaitLimit = 1L << 22;

// Factorise A (n x n, lda, column-major) in place (if factor) and / or solve
// A X = B with the factors (if solve).  ipiv (n ints), perm (n ints) and info
// (1 int) are device memory; info ends as INT_MAX when every pivot is
// non-zero, else the 1-based column of the first zero pivot.  nb: outer block
// width (1..1024).
// The single-precision variant runs its GEMMs on TF32 tensor cores.
template <typename T>
int lu_factor_solve(const LuStreams& s, T* A, int64_t n, int64_t lda, const T* B, int64_t ldb, int nrhs, T* X,
                    int64_t ldx, int* ipiv, int* perm, int* info, int nb, bool factor, bool solve);

// x = U^-1 L^-1 P b for one right-hand side with the FP64 factors in A
// (lda), perm from lu_pivots_to_perm: two ticket-ordered chain launches
// (csrc/trsv.cu).  y: n doubles of workspace; sync: lu_chain_sync_ints(n)
// ints; a dependency wait that runs out sets *info to -1.
cudaError_t lu_solve_chain_f64(cudaStream_t st, const double* A, int64_t lda, int64_t n, const int* perm,
                               const double* b, double* y, double* x, int* sync, int* info, int64_t* launches,
                               long wait_limit);
// The lower chain launch with its ticket counter started at 1: every block
// waits for block 0's flag, which no block publishes, so each wait runs out
// after wait_limit polls and *info ends at -1 (exercises the timeout path).
cudaError_t lu_chain_timeout_probe(cudaStream_t st, const double* A, int64_t lda, int64_t n, const int* perm,
                                   const double* b, double* y, double* x, int* sync, int* info, long wait_limit);
size_t lu_chain_sync_ints(int64_t n);

// perm[i] = row of the original matrix that the factorisation's row i came
// from (the pivots applied in order); perm: n ints, device.
int lu_pivots_to_perm(const LuStreams& s, const int* ipiv, int64_t n, int* perm);

// One FP32 system of a grouped factorisation: A (n_pad x n_pad, lda), n_pad a
// multiple of the block width (the caller pads a system with the identity),
// tensor maps 2 map, 2 map + 1 of gemm_group_maps for A in the device array
// the factorisation is given; ipiv (n_pad ints); info points into the infos
// array (one int per system: INT_MAX, the first zero-pivot column or -1).
struct GroupSystem {
    float* A;
    int n_pad, lda;
    int* ipiv;
    int* info;
    int map;
};
// Factorises every system in place with grouped launches (one launch per
// step and kind covers every system still active; leaves grouped by cluster
// size).  n_pad may not exceed 512 x the largest leaf cluster.  status:
// device int, lowered to -1 when a tensor-core pipeline wait ran out.
int lu_factor_group(const LuStreams& s, const std::vector<GroupSystem>& sys, const CUtensorMap* dev_maps,
                    int* infos, int* status, int nb);
// the largest n_pad lu_factor_group takes on this device
int lu_group_max_rows();
// perms[p] (n_pad ints) from system p's pivots, one launch per 512 systems
int lu_pivots_to_perm_group(cudaStream_t st, const std::vector<GroupSystem>& sys, const std::vector<int*>& perms,
                            int64_t* launches);

}  // namespace cad
