// Learned preconditioner, device side of its data path (an addition to the
// reference, whose only solver is the dense A\b of src/SlipCalculator3D.jl:22):
// element frames and the 16 nearest elements of each element, the network's
// input features, training targets gathered from an exact inverse, minibatch
// gathers for training and the scaling of predicted blocks into the system's
// units.  Together with csrc/mlp.cu (the network) this keeps the whole
// learned path -- features, training, prediction, preconditioning -- on the
// device behind the C ABI.
//
// Feature definition (per element i, neighbour q = 0..15, itself first):
// the neighbour's centroid offset and normal in i's (normal, strike, dip)
// frame, the offset divided by h_i = sqrt(2 area_i), and the area ratio
// area_j / area_i; 7 floats per neighbour, 112 per element.  Targets: the
// 3 x 3 blocks (A^-1)[i, nbr(i, q)] (rows i, N + i, 2N + i; columns the
// neighbour's) divided by h_i / G.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "lpc.h"

namespace cad {

namespace {

inline unsigned grid_for(int64_t n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// centroid (3 x N), frame rows n, ss, ds (9 x N), area, h (N each); vertex
// lists N x 3 column-major
__global__ void elem_geom_kernel(const double* __restrict__ P1, const double* __restrict__ P2,
                                 const double* __restrict__ P3, int64_t N, double* __restrict__ cen,
                                 double* __restrict__ R, double* __restrict__ area, double* __restrict__ h)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    double a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) {
        a[k] = P1[i + k * N];
        b[k] = P2[i + k * N];
        c[k] = P3[i + k * N];
    }
    const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    const double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    const double w[3] = {u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0]};
    const double len = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    const double cx = w[0] / len, cy = w[1] / len, cz = w[2] / len;
    // strike and dip directions of the normal (as CalculateSSandDSDirs)
    const double nrm = sqrt(cx * cx + cy * cy);
    double ss[3] = {-(cy / nrm), cx / nrm, 0.0};
    const double dsz = cos(acos(cz) - M_PI / 2.0);
    double L = sin(acos(dsz));
    if (cz < 0.0) L = -L;
    const double ang = atan2(cy, cx);
    double ds[3] = {-(cos(ang) * L), -(sin(ang) * L), dsz};
    if (cx == 0.0 && cy == 0.0) {
        ds[0] = -1.0; ds[1] = 0.0; ds[2] = 0.0;
        ss[0] = 0.0; ss[1] = cz < 1.0 ? -1.0 : 1.0; ss[2] = 0.0;
    }
    for (int k = 0; k < 3; ++k) cen[i + k * N] = (a[k] + b[k] + c[k]) / 3.0;
    const double nn[3] = {cx, cy, cz};
    for (int k = 0; k < 3; ++k) {
        R[i + k * N] = nn[k];
        R[i + (3 + k) * N] = ss[k];
        R[i + (6 + k) * N] = ds[k];
    }
    area[i] = 0.5 * len;
    h[i] = sqrt(len);   // sqrt(2 area)
}

// (distance^2, index) ordering: nearer first, ties to the smaller index
__device__ __forceinline__ bool nearer(double d, int j, double e, int k) { return d < e || (d == e && j < k); }

// The kLpcK nearest centroids of each element by brute force over tiles of
// 256 centroids in shared memory; the sorted list lives in registers and a
// closer candidate bubbles in from the end.  Meshes of fewer than kLpcK
// elements repeat the farthest neighbour.
__global__ void __launch_bounds__(256) knn_kernel(const double* __restrict__ cen, int64_t N, int* __restrict__ nbr)
{
    __shared__ double sx[256], sy[256], sz[256];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool live = i < N;
    const double qx = live ? cen[i] : 0.0, qy = live ? cen[i + N] : 0.0, qz = live ? cen[i + 2 * N] : 0.0;
    double bd[kLpcK];
    int bi[kLpcK];
#pragma unroll
    for (int q = 0; q < kLpcK; ++q) {
        bd[q] = INFINITY;
        bi[q] = 0x7fffffff;
    }
    for (int64_t j0 = 0; j0 < N; j0 += 256) {
        const int64_t j = j0 + threadIdx.x;
        __syncthreads();
        sx[threadIdx.x] = j < N ? cen[j] : 0.0;
        sy[threadIdx.x] = j < N ? cen[j + N] : 0.0;
        sz[threadIdx.x] = j < N ? cen[j + 2 * N] : 0.0;
        __syncthreads();
        const int cnt = N - j0 < 256 ? (int)(N - j0) : 256;
        for (int t = 0; t < cnt; ++t) {
            const double dx = sx[t] - qx, dy = sy[t] - qy, dz = sz[t] - qz;
            const double d = dx * dx + dy * dy + dz * dz;
            const int jj = (int)(j0 + t);
            if (nearer(d, jj, bd[kLpcK - 1], bi[kLpcK - 1])) {
                bd[kLpcK - 1] = d;
                bi[kLpcK - 1] = jj;
#pragma unroll
                for (int q = kLpcK - 1; q > 0; --q)
                    if (nearer(bd[q], bi[q], bd[q - 1], bi[q - 1])) {
                        const double td = bd[q];
                        bd[q] = bd[q - 1];
                        bd[q - 1] = td;
                        const int ti = bi[q];
                        bi[q] = bi[q - 1];
                        bi[q - 1] = ti;
                    }
            }
        }
    }
    if (!live) return;
    const int have = N < kLpcK ? (int)N : kLpcK;
#pragma unroll
    for (int q = 0; q < kLpcK; ++q) nbr[i * kLpcK + q] = q < have ? bi[q] : bi[have - 1];
}

// X[i, q*7 + c]: offset (3, in i's frame, / h_i), normal (3, in i's frame),
// area ratio; one thread per (element, neighbour)
__global__ void features_kernel(const double* __restrict__ cen, const double* __restrict__ R,
                                const double* __restrict__ area, const double* __restrict__ h,
                                const int* __restrict__ nbr, int64_t N, float* __restrict__ X)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= N * kLpcK) return;
    const int64_t i = t / kLpcK;
    const int q = (int)(t % kLpcK);
    const int64_t j = nbr[t];
    const double d[3] = {cen[j] - cen[i], cen[j + N] - cen[i + N], cen[j + 2 * N] - cen[i + 2 * N]};
    const double nj[3] = {R[j], R[j + N], R[j + 2 * N]};
    const double hi = h[i];
    float* x = X + i * kLpcIn + q * 7;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double r0 = R[i + (3 * a) * N], r1 = R[i + (3 * a + 1) * N], r2 = R[i + (3 * a + 2) * N];
        x[a] = (float)((r0 * d[0] + r1 * d[1] + r2 * d[2]) / hi);
        x[3 + a] = (float)(r0 * nj[0] + r1 * nj[1] + r2 * nj[2]);
    }
    x[6] = (float)(area[j] / area[i]);
}

// T[i, q*9 + r*3 + c] = Ainv[r*N + i, c*N + nbr(i, q)] / (h_i / G)
__global__ void targets_kernel(const double* __restrict__ Ainv, int64_t ld, const int* __restrict__ nbr,
                               const double* __restrict__ h, double G, int64_t N, float* __restrict__ T)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= N * kLpcOut) return;
    const int64_t i = t / kLpcOut;
    const int e = (int)(t % kLpcOut);
    const int q = e / 9, r = (e % 9) / 3, c = e % 3;
    const int64_t j = nbr[i * kLpcK + q];
    T[t] = (float)(Ainv[(r * N + i) + ld * (c * N + j)] / (h[i] / G));
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// minibatch row b of training step `step` = row splitmix64(seed, step, b) mod rows
__global__ void gather_kernel(const float* __restrict__ X, const float* __restrict__ T, int64_t rows, int64_t batch,
                              uint64_t seed, int64_t step, float* __restrict__ xb, float* __restrict__ tb)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    constexpr int W = kLpcIn + kLpcOut;
    if (t >= batch * W) return;
    const int64_t b = t / W;
    const int c = (int)(t % W);
    const uint64_t key = splitmix64(seed ^ splitmix64((uint64_t)step * 0x100000001B3ull + (uint64_t)b));
    const int64_t r = (int64_t)(key % (uint64_t)rows);
    if (c < kLpcIn) xb[b * kLpcIn + c] = X[r * kLpcIn + c];
    else tb[b * kLpcOut + (c - kLpcIn)] = T[r * kLpcOut + (c - kLpcIn)];
}

__global__ void scale_blocks_kernel(const float* __restrict__ out, const double* __restrict__ h, double G, int64_t N,
                                    float* __restrict__ blocks)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= N * kLpcOut) return;
    blocks[t] = out[t] * (float)(h[t / kLpcOut] / G);
}

// columns c0 .. c0 + gridDim.y - 1 of the n x n identity (I points at column c0)
__global__ void identity_kernel(double* __restrict__ I, int64_t ld, int64_t n, int64_t c0)
{
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t c = blockIdx.y;
    if (r < n) I[r + c * ld] = r == c0 + c ? 1.0 : 0.0;
}

__global__ void identity_blocks_kernel(int64_t N, int* __restrict__ nbr, float* __restrict__ blocks)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    nbr[i] = (int)i;
    for (int e = 0; e < 9; ++e) blocks[i * 9 + e] = (e % 4 == 0) ? 1.f : 0.f;
}

}  // namespace

size_t lpc_geom_doubles(int64_t N) { return (size_t)15 * (size_t)N; }

cudaError_t lpc_features(cudaStream_t st, const double* P1, const double* P2, const double* P3, int64_t N,
                         double* geom, int* nbr, float* X, int64_t* launches)
{
    if (N <= 0) return cudaSuccess;
    double* cen = geom;
    double* R = geom + 3 * N;
    double* area = geom + 12 * N;
    double* h = geom + 13 * N;
    elem_geom_kernel<<<grid_for(N, 128), 128, 0, st>>>(P1, P2, P3, N, cen, R, area, h);
    knn_kernel<<<grid_for(N, 256), 256, 0, st>>>(cen, N, nbr);
    features_kernel<<<grid_for(N * kLpcK, 256), 256, 0, st>>>(cen, R, area, h, nbr, N, X);
    if (launches) *launches += 3;
    return cudaGetLastError();
}

const double* lpc_geom_h(const double* geom, int64_t N) { return geom + 13 * N; }

cudaError_t lpc_targets(cudaStream_t st, const double* Ainv, int64_t ld, const int* nbr, const double* h, double G,
                        int64_t N, float* T, int64_t* launches)
{
    if (N <= 0) return cudaSuccess;
    targets_kernel<<<grid_for(N * kLpcOut, 256), 256, 0, st>>>(Ainv, ld, nbr, h, G, N, T);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t lpc_gather(cudaStream_t st, const float* X, const float* T, int64_t rows, int64_t batch, uint64_t seed,
                       int64_t step, float* xb, float* tb, int64_t* launches)
{
    if (batch <= 0 || rows <= 0) return cudaSuccess;
    gather_kernel<<<grid_for(batch * (kLpcIn + kLpcOut), 256), 256, 0, st>>>(X, T, rows, batch, seed, step, xb, tb);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t lpc_scale_blocks(cudaStream_t st, const float* out, const double* h, double G, int64_t N, float* blocks,
                             int64_t* launches)
{
    if (N <= 0) return cudaSuccess;
    scale_blocks_kernel<<<grid_for(N * kLpcOut, 256), 256, 0, st>>>(out, h, G, N, blocks);
    if (launches) ++*launches;
    return cudaGetLastError();
}

cudaError_t lpc_identity(cudaStream_t st, double* I, int64_t ld, int64_t n, int64_t* launches)
{
    for (int64_t c0 = 0; c0 < n; c0 += 65535) {   // grid.y limit
        const int64_t nc = n - c0 < 65535 ? n - c0 : 65535;
        identity_kernel<<<dim3(grid_for(n, 256), (unsigned)nc), 256, 0, st>>>(I + c0 * ld, ld, n, c0);
        if (launches) ++*launches;
    }
    return cudaGetLastError();
}

cudaError_t lpc_identity_blocks(cudaStream_t st, int64_t N, int* nbr, float* blocks, int64_t* launches)
{
    if (N <= 0) return cudaSuccess;
    identity_blocks_kernel<<<grid_for(N, 256), 256, 0, st>>>(N, nbr, blocks);
    if (launches) ++*launches;
    return cudaGetLastError();
}

}  // namespace cad
