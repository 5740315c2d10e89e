// Learned preconditioner: features, targets, minibatches (csrc/lpc.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace cad {

constexpr int kLpcK = 16;      // neighbours per element, itself first
constexpr int kLpcIn = 7 * kLpcK;
constexpr int kLpcOut = 9 * kLpcK;

// doubles of the per-mesh geometry workspace: centroids, frames, areas, h
size_t lpc_geom_doubles(int64_t N);
// h = sqrt(2 area) inside that workspace
const double* lpc_geom_h(const double* geom, int64_t N);

// Element geometry into geom (lpc_geom_doubles(N)), the 16 nearest elements
// (nbr, N x 16, itself first) and the network inputs X (N x 112).
cudaError_t lpc_features(cudaStream_t st, const double* P1, const double* P2, const double* P3, int64_t N,
                         double* geom, int* nbr, float* X, int64_t* launches);
// Training targets T (N x 144) from the exact inverse Ainv (3N x 3N, ld).
cudaError_t lpc_targets(cudaStream_t st, const double* Ainv, int64_t ld, const int* nbr, const double* h, double G,
                        int64_t N, float* T, int64_t* launches);
// Minibatch `step` of `batch` rows drawn (seeded hash) from the training set.
cudaError_t lpc_gather(cudaStream_t st, const float* X, const float* T, int64_t rows, int64_t batch, uint64_t seed,
                       int64_t step, float* xb, float* tb, int64_t* launches);
// Network outputs (N x 144) -> preconditioner blocks in the system's units.
cudaError_t lpc_scale_blocks(cudaStream_t st, const float* out, const double* h, double G, int64_t N, float* blocks,
                             int64_t* launches);
// n x n identity (column-major, ld).
cudaError_t lpc_identity(cudaStream_t st, double* I, int64_t ld, int64_t n, int64_t* launches);
// Identity 3 x 3 blocks (k = 1) for N elements: GMRES with no preconditioning.
cudaError_t lpc_identity_blocks(cudaStream_t st, int64_t N, int* nbr, float* blocks, int64_t* launches);

}  // namespace cad
