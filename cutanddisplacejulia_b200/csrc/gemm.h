// The dense LU's matrix products on the tensor cores (csrc/gemm.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace cad {

// C (m x n, ldc) -= A (m x k, lda) * B (k x n, ldb), column-major, on stream
// st.  FP64: DMMA tensor-core tiles, any leading dimensions.  FP32: TF32
// tensor cores through tcgen05 with TMA-staged operands when A and B start on
// 16-byte boundaries and lda, ldb are multiples of 4 (else FP32 CUDA cores).
// status (device int, may be null for FP64): a pipeline wait of the tcgen05
// kernel that runs out lowers it to -1 (the LU's info word convention); a
// null status selects the CUDA-core kernel for FP32.
// dmma_k: k-extent of the FP64 DMMA instruction (4: m8n8k4, 8: m16n8k8, 16:
// m16n8k16; 0 = kDefaultDmmaK); every shape gives the same products up to the
// order of the k-sums.
constexpr int kDefaultDmmaK = 4;
cudaError_t gemm_sub(cudaStream_t st, int m, int n, int k, const double* A, int64_t lda, const double* B, int64_t ldb,
                     double* C, int64_t ldc, int* status, int dmma_k = 0);
cudaError_t gemm_sub(cudaStream_t st, int m, int n, int k, const float* A, int64_t lda, const float* B, int64_t ldb,
                     float* C, int64_t ldc, int* status);

}  // namespace cad
