// Learned preconditioner network (csrc/mlp.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace cad {

constexpr int kMlpIn = 112;      // 16 neighbours x (offset 3, normal 3, area 1)
constexpr int kMlpHidden = 256;
constexpr int kMlpOut = 144;     // 16 blocks x 9

size_t mlp_param_count();
size_t mlp_workspace_bytes(int64_t rows);

// One pass over `rows` samples: forward (out, if set, gets the network output
// rows x kMlpOut); with grads set also the MSE loss against T (loss: device
// float, the sum of squared errors, if set) and the gradient of the mean
// squared error; with adam_m / adam_v set also one Adam update of params.
struct MlpStep {
    cudaStream_t stream;
    float* params;            // FP32 master weights (mlp_param_count)
    const float* X;           // rows x kMlpIn
    const float* T;           // rows x kMlpOut
    int64_t rows;
    float* out;
    float* grads;
    float* loss;
    float* adam_m;
    float* adam_v;
    float lr, bias_c1, bias_c2;   // Adam step size and bias corrections 1 - beta^t
    void* workspace;          // mlp_workspace_bytes(rows)
    int64_t* launches;
};
int mlp_step(const MlpStep& s);   // 0 or a cudaError_t

cudaError_t mlp_gemm(cudaStream_t st, bool ta, bool tb, const __nv_bfloat16* A, int64_t lda, const __nv_bfloat16* B,
                     int64_t ldb, float* C, int64_t ldc, int M, int N, int K, bool accumulate);

// z = M v with M block-sparse: N elements x k blocks of 3 x 3 (FP32,
// row-major) at the neighbour elements nbr (N x k)
cudaError_t spai_apply(cudaStream_t st, const int* nbr, const float* blocks, int k, const double* v, int64_t N,
                       double* z);

// The inverses of the 3 x 3 self blocks of the 3N x 3N system A (k = 1).
cudaError_t block_jacobi(cudaStream_t st, const double* A, int64_t lda, int64_t N, int* nbr, float* blocks);

}  // namespace cad
