// The dense LU's matrix products on the tensor cores (csrc/gemm.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

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

// One product C -= A B of a grouped FP32 launch (many independent systems):
// A is rows [ax, ax + m), columns [ay, ay + k) of the matrix behind tensor
// maps 2 map (A boxes) and B rows [bx, bx + k), columns [by, by + n) of the
// matrix behind map 2 map + 1 (B boxes); C (ldc) points at the product's
// first element.  k, ax and bx must be multiples of 32, 4 and 4.
struct GemmGroupRec {
    float* C;
    int ldc, m, n, k;
    int ax, ay, bx, by;
    int map;
    int tile0;   // first tile of the record in its launch (set by gemm_sub_group)
};
constexpr int kGemmGroupMax = 512;   // records per launch

// The two tensor maps (out[0]: A-operand boxes, out[1]: B-operand boxes) of a
// column-major FP32 matrix (rows x cols, ld; 16-byte aligned base, ld a
// multiple of 4) for grouped products.
bool gemm_group_maps(CUtensorMap* out, const float* base, int rows, int cols, int64_t ld);

// C -= A B for every record (records with an empty product are skipped) on
// TF32 tcgen05 tensor cores, kGemmGroupMax records per launch; dev_maps holds
// the records' tensor maps in device memory.  status as gemm_sub.
cudaError_t gemm_sub_group(cudaStream_t st, const CUtensorMap* dev_maps, std::vector<GemmGroupRec>& recs,
                           int* status, int64_t* launches);

}  // namespace cad
