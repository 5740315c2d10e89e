// TD pair kernels for sm_100a (FP64 CUDA-core work; no tensor-core shape).
//
// Work decomposition: one thread per observation point, one block per
// (128-point tile, chunk of triangles).  The block stages one triangle's
// precomputed record (TriDev) at a time in shared memory; every thread reads
// it as a broadcast, evaluates its pair and writes the pair's outputs
// (consecutive threads = consecutive rows of a column-major M x N influence
// matrix, so every store is coalesced).
//
// Output modes:
//   OUT_INF   18 strain and / or 9 displacement influence matrices (TD overload
//             src/TD.jl:135-216)
//   OUT_SUM   per-chunk partial sums over triangles of strain (6) and
//             displacement (3) (TD summing overload src/TD.jl:219-410); a
//             second kernel adds the chunks in index order (deterministic)
//   OUT_TRAC  9 traction influence matrices, strain converted in registers
//             (ConvertStrainInfMatsToTraction, src/CalculateInfluenceMatrices3D.jl:73-114)
//   OUT_AMAT  the 3N x 3N system matrix -[Atn;Atss;Atds] (src/SlipCalculator3D.jl:13-16)
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "td_device.cuh"
#include "td_kernels.h"

namespace cad {

// ------------------------------------------------------------ setup kernel
__global__ void td_setup_kernel(const double* __restrict__ P1, const double* __restrict__ P2,
                                const double* __restrict__ P3, int64_t N, const double* __restrict__ Dss,
                                const double* __restrict__ Dds, const double* __restrict__ Dn, int64_t slip_stride,
                                double nu, int hs, TriDev* __restrict__ out)
{
    const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (j >= N) return;
    TriDev& t = out[j];
    const double a[3] = {P1[j], P1[j + N], P1[j + 2 * N]};
    const double b[3] = {P2[j], P2[j + N], P2[j + 2 * N]};
    const double c[3] = {P3[j], P3[j + N], P3[j + 2 * N]};
    build_triangle(a, b, c, Dss ? Dss[j * slip_stride] : 1.0, Dds ? Dds[j * slip_stride] : 1.0,
                   Dn ? Dn[j * slip_stride] : 1.0, nu, hs != 0, t);
}

// ------------------------------------------------ half-space argument check
// flag |= 1 when any vertex or observation z > 0 (src/TD.jl:606-619).
// With nz set, the observation z is Z - 1e-12 nz (collocation points from
// midpoints and normals, as SetupCollationPoints forms them).
__global__ void hs_check_kernel(const double* __restrict__ Z, const double* __restrict__ nz, int64_t M,
                                const double* __restrict__ P1, const double* __restrict__ P2,
                                const double* __restrict__ P3, int64_t N, int* __restrict__ flag)
{
    int bad = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M + N; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < M) bad |= (nz ? Z[i] - nz[i] * 1e-12 : Z[i]) > 0.0;
        else {
            const int64_t j = i - M;
            bad |= (P1[j + 2 * N] > 0.0) | (P2[j + 2 * N] > 0.0) | (P3[j + 2 * N] > 0.0);
        }
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

// ---------------------------------------------------- collocation points
// obs = incentre - 1e-12 * normal (SetupCollationPoints,
// src/CalculateInfluenceMatrices3D.jl:52-71) and the strike / dip directions
// of every element (CalculateSSandDSDirs, src/CalculateSSandDSDirs.jl:417-481).
__global__ void colloc_kernel(const double* __restrict__ normals, const double* __restrict__ mid, int64_t N,
                              double* __restrict__ X, double* __restrict__ Y, double* __restrict__ Z,
                              double* __restrict__ dirs /* 9 x N: n, ss, ds */)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double cx = normals[i], cy = normals[i + N], cz = normals[i + 2 * N];
    X[i] = mid[i] - cx * 1e-12;
    Y[i] = mid[i + N] - cy * 1e-12;
    Z[i] = mid[i + 2 * N] - cz * 1e-12;
    const double inv = 1.0 / sqrt(cx * cx + cy * cy);
    double ss[3] = {-(cy * inv), cx * inv, 0.0};
    const double dsz = cos(acos(cz) - M_PI / 2.0);
    double L = sin(acos(dsz));
    if (cz < 0.0) L = -L;
    const double a = atan2(cy, cx);
    double ds[3] = {-(cos(a) * L), -(sin(a) * L), dsz};
    if (cx == 0.0 && cy == 0.0) {
        ds[0] = -1.0; ds[1] = 0.0; ds[2] = 0.0;
        ss[0] = 0.0; ss[1] = cz < 1.0 ? -1.0 : 1.0; ss[2] = 0.0;
    }
    dirs[i] = cx; dirs[i + N] = cy; dirs[i + 2 * N] = cz;
    for (int k = 0; k < 3; ++k) { dirs[i + (3 + k) * N] = ss[k]; dirs[i + (6 + k) * N] = ds[k]; }
}

// Unit-mode strain -> (Tn, Tss, Tds) on the element with normal n, strike ss,
// dip ds (Hooke, CalculateNormalTraction3D!, TractionVectorCartesianComponents3D!,
// CalculateTractionInChosenDirection3D!).
template <typename R>
__device__ __forceinline__ void strain_to_traction(const R e[6], R lam, R G2, const R n[3], const R ss[3],
                                                   const R ds[3], R out[3])
{
    const R cons = lam * (e[0] + e[1] + e[2]);
    const R Sxx = G2 * e[0] + cons, Syy = G2 * e[1] + cons, Szz = G2 * e[2] + cons;
    const R Sxy = G2 * e[3], Sxz = G2 * e[4], Syz = G2 * e[5];
    const R cx = n[0], cy = n[1], cz = n[2];
    const R two = R(2.0);
    out[0] = Sxx * (cx * cx) + Syy * (cy * cy) + Szz * (cz * cz) + two * Sxy * (cx * cy) + two * Syz * (cy * cz) +
             two * Sxz * (cz * cx);
    const R Tx = Sxx * cx + Sxy * cy + Sxz * cz;
    const R Ty = Sxy * cx + Syy * cy + Syz * cz;
    const R Tz = Sxz * cx + Syz * cy + Szz * cz;
    // traction projected onto the plane: t - (t.n) n
    const R tn = Tx * cx + Ty * cy + Tz * cz;
    const R px = Tx - tn * cx, py = Ty - tn * cy, pz = Tz - tn * cz;
    out[1] = px * ss[0] + py * ss[1] + pz * ss[2];
    out[2] = px * ds[0] + py * ds[1] + pz * ds[2];
}

// ------------------------------------------------------------- pair kernel
// NEAR: rewrite only the triangles whose centroid lies within the near
// radius of some point of the block (the FP64 pass of the mixed assembly).
// LIST (OUT_AMAT only): incremental re-assembly through a.tri_list /
// a.obs_list into a system of a.Ntot elements.
// MINB > 1: compiled for MINB resident blocks per SM (fewer registers per
// thread, more warps to hide the FP64 latency, some spilling) -- a launch
// shape the autotuner may pick for the half-space system matrix.
// EDGE (half space): the free-surface corrections are left to per-edge work;
// the staged record is the two frames only.  OUT_AMAT, OUT_TRAC (strain) and
// OUT_INF: they come from the per-edge maps a.fscG (fsc_edge_kernel).
// OUT_SUM: they are left out here, and fsc_sum_kernel adds each edge's once.
template <bool HS, bool STRAIN, bool DISP, int OUT, bool NEAR = false, bool LIST = false, int MINB = 1,
          bool EDGE = false>
__global__ void __launch_bounds__(kPairThreads, MINB) td_pair_kernel(PairArgs a)
{
    static_assert(!EDGE || (HS && !LIST && !NEAR &&
                            (((OUT == OUT_AMAT || OUT == OUT_TRAC) && STRAIN && !DISP) || OUT == OUT_SUM ||
                             OUT == OUT_INF)),
                  "shared edges: HS system matrix, traction or influence fields, or sums only");
    constexpr bool EDGE_MAPS = EDGE && OUT != OUT_SUM;
    // values per (edge, point) in the maps: strain 18, then displacement 9
    constexpr int64_t kQ = (STRAIN ? 18 : 0) + (DISP ? 9 : 0);
    extern __shared__ double smem[];
    constexpr int words = HS ? (EDGE ? kTriWordsImg : kTriWordsHS) : kTriWordsFS;
    const TriDev& t = *reinterpret_cast<const TriDev*>(smem);
    const int64_t i = (int64_t)blockIdx.x * kPairThreads + threadIdx.x;
    const bool active = i < a.M;
    // LIST: this thread's point (system row) and the full system's size
    const int64_t io = (LIST && a.obs_list && active) ? (int64_t)a.obs_list[i] : i;
    const int64_t NS = LIST ? a.Ntot : a.N;
    const int64_t MD = (LIST || EDGE_MAPS) ? a.Ntot : a.M;
    double X = 0.0, Y = 0.0, Z = 0.0;
    if (active) { X = a.X[io]; Y = a.Y[io]; Z = a.Z[io]; }
    const int64_t j0 = (int64_t)blockIdx.y * a.tri_chunk;
    const int64_t j1 = min(a.N, j0 + a.tri_chunk);
    // row stride of the M x N output fields: a block of an Ntot-point system
    // with the edge maps
    const int64_t MR = EDGE_MAPS ? MD : a.M;
    const int64_t MN = MR * a.N;
    double sumE[6] = {0, 0, 0, 0, 0, 0}, sumU[3] = {0, 0, 0};
    double n[3] = {0, 0, 0}, ss[3] = {0, 0, 0}, ds[3] = {0, 0, 0};
    if ((OUT == OUT_TRAC || OUT == OUT_AMAT) && active) {
        for (int k = 0; k < 3; ++k) {
            n[k] = a.dirs[io + k * MD];
            ss[k] = a.dirs[io + (3 + k) * MD];
            ds[k] = a.dirs[io + (6 + k) * MD];
        }
    }
    const double near_r2 = NEAR ? a.near[3 * a.N] : 0.0;
    for (int64_t j = j0; j < j1; ++j) {
        if (NEAR) {
            bool nr = false;
            if (active) {
                const double dx = X - a.near[j], dy = Y - a.near[j + a.N], dz = Z - a.near[j + 2 * a.N];
                nr = dx * dx + dy * dy + dz * dz < near_r2;
            }
            if (!__syncthreads_or(nr)) continue;   // also the barrier before restaging
        } else {
            __syncthreads();
        }
        const int64_t jt = (LIST && a.tri_list) ? (int64_t)a.tri_list[j] : j;   // system column
        const double* src = reinterpret_cast<const double*>(a.tri + jt);
        for (int w = threadIdx.x; w < words; w += kPairThreads) smem[w] = src[w];
        __syncthreads();
        if (!active) continue;
        if (STRAIN) {
            double E[3][6];
            if constexpr (EDGE_MAPS)
                pair_strain_edges(t, X, Y, Z, a.fscG + i, a.M, kQ * a.M, a.side_edge + 3 * jt, E);
            else if constexpr (EDGE)
                pair_strain_fs_image(t, X, Y, Z, E);
            else
                pair_strain<HS>(t, X, Y, Z, E);
            if (OUT == OUT_INF) {
#pragma unroll
                for (int m = 0; m < 3; ++m)
#pragma unroll
                    for (int k = 0; k < 6; ++k) a.strain[(6 * m + k) * MN + i + MR * j] = E[m][k];
            } else if (OUT == OUT_SUM) {
#pragma unroll
                for (int k = 0; k < 6; ++k) sumE[k] += (E[0][k] + E[1][k]) + E[2][k];
            } else {
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    double tr[3];
                    strain_to_traction(E[m], a.lambda, 2.0 * a.G, n, ss, ds, tr);
                    if (OUT == OUT_TRAC) {
#pragma unroll
                        for (int r = 0; r < 3; ++r) a.trac[(3 * m + r) * MN + i + MR * j] = tr[r];
                    } else {
#pragma unroll
                        for (int r = 0; r < 3; ++r)
                            a.A[(int64_t)(r * MD + io) + a.lda * (int64_t)(m * NS + jt)] = -tr[r];
                    }
                }
            }
        }
        if (DISP) {
            double U[3][3];
            if constexpr (EDGE_MAPS)
                pair_disp_edges(t, X, Y, Z, a.fscG + i + (STRAIN ? 18 : 0) * a.M, a.M, kQ * a.M, a.side_edge + 3 * jt,
                                U);
            else if constexpr (EDGE)
                pair_disp_fs_image(t, X, Y, Z, U);
            else
                pair_disp<HS>(t, X, Y, Z, U);
            if (OUT == OUT_INF) {
#pragma unroll
                for (int m = 0; m < 3; ++m)
#pragma unroll
                    for (int c = 0; c < 3; ++c) a.disp[(3 * m + c) * MN + i + MR * j] = U[m][c];
            } else if (OUT == OUT_SUM) {
#pragma unroll
                for (int c = 0; c < 3; ++c) sumU[c] += (U[0][c] + U[1][c]) + U[2][c];
            }
        }
    }
    if (OUT == OUT_SUM && active) {
        double* p = a.partial + (int64_t)blockIdx.y * 9 * a.M;
#pragma unroll
        for (int k = 0; k < 6; ++k) p[k * a.M + i] = sumE[k];
#pragma unroll
        for (int c = 0; c < 3; ++c) p[(6 + c) * a.M + i] = sumU[c];
    }
}

// Adds the per-chunk partial sums in chunk order: out[f][i] = sum_c partial[c][f][i].
__global__ void sum_chunks_kernel(const double* __restrict__ partial, int64_t nchunk, int64_t M, int fields_mask,
                                  double* __restrict__ out)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (i >= M || !((fields_mask >> f) & 1)) return;
    double s = 0.0;
    for (int64_t c = 0; c < nchunk; ++c) s += partial[(c * 9 + f) * M + i];
    out[f * M + i] = s;
}

// As sum_chunks_kernel, with strain fields (0-5) and displacement fields
// (6-8) written to two separate outputs (6 x M and 3 x M).
__global__ void sum_chunks_split_kernel(const double* __restrict__ partial, int64_t nchunk, int64_t M,
                                        int fields_mask, double* __restrict__ strain_out,
                                        double* __restrict__ disp_out)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (i >= M || !((fields_mask >> f) & 1)) return;
    double s = 0.0;
    for (int64_t c = 0; c < nchunk; ++c) s += partial[(c * 9 + f) * M + i];
    if (f < 6) strain_out[f * M + i] = s;
    else disp_out[(f - 6) * M + i] = s;
}

// TD_sum (src/TD_sum.jl:1-41): sum the three modes, then across the N columns.
// in: nf*3 matrices M x N (field f of mode m at in + (m*nf + f)*M*N), out: nf x M.
__global__ void td_sum_kernel(const double* __restrict__ in, int64_t M, int64_t N, int nf, double* __restrict__ out)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (i >= M) return;
    const int64_t MN = M * N;
    double s = 0.0;
    for (int64_t j = 0; j < N; ++j) {
        const int64_t o = i + M * j;
        s += (in[(0 * nf + f) * MN + o] + in[(1 * nf + f) * MN + o]) + in[(2 * nf + f) * MN + o];
    }
    out[f * M + i] = s;
}

// ------------------------------------------------------- fixed elements
// Splice of CalculateInfluenceMatrices3D with fixed elements (ConcatInfMats,
// PutDispInfsIntoInfMat, src/CalculateInfluenceMatrices3D.jl:145-199): field
// f's row i is the displacement influence disp[f] (nfix x N) of fixed row
// fixrow[i] when i is fixed (fixrow[i] >= 0), else the traction influence
// trac[f] (N x N); only the columns freecol[0..nf) are kept.  amat = 0:
// out + f * N * nf holds field f (N x nf, column-major); amat = 1: out is the
// system A (3N x 3nf, lda) = -[[F0 F3 F6]; [F1 F4 F7]; [F2 F5 F8]].
__global__ void splice_fixed_kernel(const double* __restrict__ trac, const double* __restrict__ disp, int64_t N,
                                    int64_t nfix, const int* __restrict__ fixrow, const int* __restrict__ freecol,
                                    int64_t nf, int amat, double* __restrict__ out, int64_t lda)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t jf = blockIdx.y;
    const int f = blockIdx.z;
    if (i >= N || jf >= nf) return;
    const int64_t j = freecol[jf];
    const int fr = fixrow[i];
    const double v = fr >= 0 ? disp[(int64_t)f * nfix * N + fr + nfix * j] : trac[(int64_t)f * N * N + i + N * j];
    if (!amat) {
        out[(int64_t)f * N * nf + i + N * jf] = v;
    } else {
        const int m = f / 3, r = f % 3;   // field 3m + r: slip mode m (column block), traction row r
        out[(r * N + i) + lda * (m * nf + jf)] = -v;
    }
}

// out[k] = (X, Y, Z)[idx[k]] as three SoA arrays of length n
__global__ void gather_points_kernel(const double* __restrict__ X, const double* __restrict__ Y,
                                     const double* __restrict__ Z, const int* __restrict__ idx, int64_t n,
                                     double* __restrict__ out)
{
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int64_t i = idx[k];
    out[k] = X[i];
    out[k + n] = Y[i];
    out[k + 2 * n] = Z[i];
}

// ----------------------------------------------- mixed-precision assembly
// Centroids of the triangles (near + [0, 3N)) and the squared near-field
// radius (near[3N]) = (factor x mean edge length)^2; one block, fixed
// summation order.
__global__ void __launch_bounds__(1024) near_setup_kernel(const double* __restrict__ P1, const double* __restrict__ P2,
                                                          const double* __restrict__ P3, int64_t N, double factor,
                                                          double* __restrict__ near)
{
    __shared__ double s_sum[1024];
    double acc = 0.0;
    for (int64_t j = threadIdx.x; j < N; j += blockDim.x) {
        double e = 0.0;
        for (int c = 0; c < 3; ++c) near[j + c * N] = (P1[j + c * N] + P2[j + c * N] + P3[j + c * N]) / 3.0;
        const double* P[3] = {P1, P2, P3};
        for (int v = 0; v < 3; ++v) {
            const double* p = P[v];
            const double* q = P[(v + 1) % 3];
            const double dx = q[j] - p[j], dy = q[j + N] - p[j + N], dz = q[j + 2 * N] - p[j + 2 * N];
            e += sqrt(dx * dx + dy * dy + dz * dz);
        }
        acc += e;
    }
    s_sum[threadIdx.x] = acc;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s_sum[threadIdx.x] += s_sum[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double r = factor * (N > 0 ? s_sum[0] / (3.0 * (double)N) : 0.0);
        near[3 * N] = r * r;
    }
}

// FP32 copy of the first `words` values of each triangle record (records
// `stride` values apart in both copies): element-wise, then the origins' low
// parts (an FP32 record keeps each origin as hi + lo).
__global__ void tri_to_f32_kernel(const double* __restrict__ in, int64_t N, int words, int stride,
                                  float* __restrict__ out)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N * words) return;
    const int64_t j = i / words;
    const int w = (int)(i - j * words);
    const int64_t at = j * stride + w;
    constexpr int kReal = (int)((offsetof(TriDev, real) + offsetof(Frame, P2lo)) / sizeof(double));
    constexpr int kImage = (int)((offsetof(TriDev, image) + offsetof(Frame, P2lo)) / sizeof(double));
    constexpr int kSide0 = (int)((offsetof(TriDev, side) + offsetof(FscSide, PAlo)) / sizeof(double));
    constexpr int kSideW = (int)(sizeof(FscSide) / sizeof(double));
    bool lo = (w >= kReal && w < kReal + 3) || (w >= kImage && w < kImage + 3);
    for (int sd = 0; sd < 3; ++sd) lo = lo || (w >= kSide0 + sd * kSideW && w < kSide0 + sd * kSideW + 3);
    if (lo) {
        const double hi = in[at - 3];
        out[at] = (float)(hi - (double)(float)hi);
    } else {
        out[at] = (float)in[at];
    }
}

// Far-field pass: the system-matrix kernel with FP32 records and FP32
// arithmetic (coordinates relative to each origin formed in FP64).
template <bool HS>
__global__ void __launch_bounds__(kPairThreads) td_pair_f32_kernel(PairArgs a)
{
    extern __shared__ float smem32[];
    constexpr int words = HS ? kTriWordsHS : kTriWordsFS;
    const TriDevT<float>& t = *reinterpret_cast<const TriDevT<float>*>(smem32);
    const int64_t i = (int64_t)blockIdx.x * kPairThreads + threadIdx.x;
    const bool active = i < a.M;
    double X = 0.0, Y = 0.0, Z = 0.0;
    if (active) { X = a.X[i]; Y = a.Y[i]; Z = a.Z[i]; }
    const int64_t j0 = (int64_t)blockIdx.y * a.tri_chunk;
    const int64_t j1 = min(a.N, j0 + a.tri_chunk);
    float n[3] = {0, 0, 0}, ss[3] = {0, 0, 0}, ds[3] = {0, 0, 0};
    if (active) {
        for (int k = 0; k < 3; ++k) {
            n[k] = (float)a.dirs[i + k * a.M];
            ss[k] = (float)a.dirs[i + (3 + k) * a.M];
            ds[k] = (float)a.dirs[i + (6 + k) * a.M];
        }
    }
    const float* recs = reinterpret_cast<const float*>(a.tri32);
    const float lam = (float)a.lambda, G2 = (float)(2.0 * a.G);
    for (int64_t j = j0; j < j1; ++j) {
        __syncthreads();
        const float* src = recs + j * (int64_t)kTriWordsHS;   // records keep the FP64 stride
        for (int w = threadIdx.x; w < words; w += kPairThreads) smem32[w] = src[w];
        __syncthreads();
        if (!active) continue;
        float E[3][6];
        pair_strain<HS>(t, X, Y, Z, E);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            float tr[3];
            strain_to_traction(E[m], lam, G2, n, ss, ds, tr);
#pragma unroll
            for (int r = 0; r < 3; ++r) a.A[(int64_t)(r * a.N + i) + a.lda * (int64_t)(m * a.N + j)] = -(double)tr[r];
        }
    }
}

// ------------------------------------------------------------ launchers
template <bool HS, bool STRAIN, bool DISP, int OUT, int MINB = 1>
static cudaError_t launch_pair(const PairArgs& a, cudaStream_t st)
{
    const size_t smem = (HS ? kTriWordsHS : kTriWordsFS) * sizeof(double);
    auto kern = td_pair_kernel<HS, STRAIN, DISP, OUT, false, false, MINB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int64_t ntile = (a.M + kPairThreads - 1) / kPairThreads;
    const int64_t nchunk = (a.N + a.tri_chunk - 1) / a.tri_chunk;
    if (ntile == 0 || nchunk == 0) return cudaSuccess;
    dim3 grid((unsigned)ntile, (unsigned)nchunk);
    kern<<<grid, kPairThreads, smem, st>>>(a);
    return cudaGetLastError();
}

#define CAD_DISPATCH_FLAGS(OUTK)                                                              \
    if (hs) {                                                                                 \
        if (strain && disp) return launch_pair<true, true, true, OUTK>(a, st);                \
        if (strain) return launch_pair<true, true, false, OUTK>(a, st);                       \
        if (disp) return launch_pair<true, false, true, OUTK>(a, st);                         \
    } else {                                                                                  \
        if (strain && disp) return launch_pair<false, true, true, OUTK>(a, st);               \
        if (strain) return launch_pair<false, true, false, OUTK>(a, st);                      \
        if (disp) return launch_pair<false, false, true, OUTK>(a, st);                        \
    }                                                                                         \
    return cudaSuccess;

cudaError_t launch_td_pairs(const PairArgs& a, int out, bool hs, bool strain, bool disp, cudaStream_t st)
{
    switch (out) {
        case OUT_INF: { CAD_DISPATCH_FLAGS(OUT_INF) }
        case OUT_SUM: { CAD_DISPATCH_FLAGS(OUT_SUM) }
        case OUT_TRAC:
            if (hs) return launch_pair<true, true, false, OUT_TRAC>(a, st);
            return launch_pair<false, true, false, OUT_TRAC>(a, st);
        case OUT_AMAT:
            if (hs) {
                if (a.min_blocks == 3) return launch_pair<true, true, false, OUT_AMAT, 3>(a, st);
                if (a.min_blocks == 4) return launch_pair<true, true, false, OUT_AMAT, 4>(a, st);
                return launch_pair<true, true, false, OUT_AMAT>(a, st);
            }
            return launch_pair<false, true, false, OUT_AMAT>(a, st);
    }
    return cudaErrorInvalidValue;
}

// ------------------------------------------------ shared-edge half space
// One mesh edge's free-surface record (geometry only) per thread; edge e's
// endpoints PA, PB at pts[6 e ..].
__global__ void edge_setup_kernel(const double* __restrict__ pts, int64_t E, double nu, FscSide* __restrict__ out)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= E) return;
    const double PA[3] = {pts[6 * e], pts[6 * e + 1], pts[6 * e + 2]};
    const double PB[3] = {pts[6 * e + 3], pts[6 * e + 4], pts[6 * e + 5]};
    build_side_geom(PA, PB, nu, out[e]);
}

// G[(e * Q + q) M + i] = value q of edge e's free-surface maps at point i:
// the strain map (fsc_strain_map, 18 values) when STRAIN, then the
// displacement map (fsc_disp_map, 9) when DISP; zero for an edge the beta test
// drops.  Block = 128 points x a chunk of edges, each edge record staged in
// shared memory.
template <bool STRAIN, bool DISP>
__global__ void __launch_bounds__(kPairThreads, 1) fsc_edge_kernel(const FscSide* __restrict__ edges, int64_t E,
                                                                 int64_t echunk, const double* __restrict__ X,
                                                                 const double* __restrict__ Y,
                                                                 const double* __restrict__ Z, int64_t M,
                                                                 double* __restrict__ G)
{
    extern __shared__ double smem[];
    const FscSide& s = *reinterpret_cast<const FscSide*>(smem);
    const int64_t i = (int64_t)blockIdx.x * kPairThreads + threadIdx.x;
    const bool active = i < M;
    double x = 0.0, y = 0.0, z = 0.0;
    if (active) { x = X[i]; y = Y[i]; z = Z[i]; }
    const int64_t e0 = (int64_t)blockIdx.y * echunk;
    const int64_t e1 = min(E, e0 + echunk);
    for (int64_t e = e0; e < e1; ++e) {
        __syncthreads();
        const double* src = reinterpret_cast<const double*>(edges + e);
        for (int w = threadIdx.x; w < kSideWords; w += kPairThreads) smem[w] = src[w];
        __syncthreads();
        if (!active) continue;
        constexpr int64_t Q = (STRAIN ? 18 : 0) + (DISP ? 9 : 0);
        if (STRAIN) {
            double Gm[3][6];
            if (s.skip != 0.0) {
#pragma unroll
                for (int q = 0; q < 18; ++q) Gm[q / 6][q % 6] = 0.0;
            } else {
                fsc_strain_map(s, x, y, z, Gm);
            }
#pragma unroll
            for (int q = 0; q < 18; ++q) G[(e * Q + q) * M + i] = Gm[q / 6][q % 6];
        }
        if (DISP) {
            double Gu[3][3];
            if (s.skip != 0.0) {
#pragma unroll
                for (int q = 0; q < 9; ++q) Gu[q / 3][q % 3] = 0.0;
            } else {
                fsc_disp_map(s, x, y, z, Gu);
            }
            constexpr int64_t q0 = STRAIN ? 18 : 0;
#pragma unroll
            for (int q = 0; q < 9; ++q) G[(e * Q + q0 + q) * M + i] = Gu[q / 3][q % 3];
        }
    }
}

size_t edge_record_bytes() { return sizeof(FscSide); }

cudaError_t launch_assemble_edges(PairArgs a, int out_kind, bool strain, bool disp, const double* edge_pts,
                                  int64_t E, const int* side_edge, void* edge_rec, double* G, int64_t Mc, double nu,
                                  cudaStream_t st, int64_t* launches)
{
    if (out_kind == OUT_AMAT || out_kind == OUT_TRAC) {
        strain = true;
        disp = false;
    } else if (out_kind != OUT_INF || !(strain || disp)) {
        return cudaErrorInvalidValue;
    }
    if (a.M == 0 || a.N == 0) return cudaSuccess;
    if (E > 0) {
        edge_setup_kernel<<<(unsigned)((E + 127) / 128), 128, 0, st>>>(edge_pts, E, nu, (FscSide*)edge_rec);
        if (launches) ++*launches;
        if (cudaError_t e = cudaGetLastError()) return e;
    }
    // a.min_blocks 3: three resident blocks per SM (168 registers, 308 B of
    // spills), 69.8 ms against 73.9 ms with the full register file (1) at
    // 10 000 triangles (system matrix; the influence fields keep 1)
    using PairKernel = void (*)(PairArgs);
    using EdgeKernel = void (*)(const FscSide*, int64_t, int64_t, const double*, const double*, const double*,
                                int64_t, double*);
    PairKernel pk;
    EdgeKernel ek = fsc_edge_kernel<true, false>;
    if (out_kind == OUT_TRAC) {
        pk = a.min_blocks == 1 ? td_pair_kernel<true, true, false, OUT_TRAC, false, false, 1, true>
                               : td_pair_kernel<true, true, false, OUT_TRAC, false, false, 3, true>;
    } else if (out_kind == OUT_AMAT) {
        pk = a.min_blocks == 1 ? td_pair_kernel<true, true, false, OUT_AMAT, false, false, 1, true>
                               : td_pair_kernel<true, true, false, OUT_AMAT, false, false, 3, true>;
    } else if (strain && disp) {
        pk = td_pair_kernel<true, true, true, OUT_INF, false, false, 1, true>;
        ek = fsc_edge_kernel<true, true>;
    } else if (strain) {
        pk = td_pair_kernel<true, true, false, OUT_INF, false, false, 1, true>;
    } else {
        pk = td_pair_kernel<true, false, true, OUT_INF, false, false, 1, true>;
        ek = fsc_edge_kernel<false, true>;
    }
    const size_t psmem = (size_t)kTriWordsImg * sizeof(double);
    const size_t esmem = (size_t)kSideWords * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(ek, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)esmem);
    if (e != cudaSuccess) return e;
    const int64_t echunk = 32;
    for (int64_t c0 = 0; c0 < a.M; c0 += Mc) {
        const int64_t mc = a.M - c0 < Mc ? a.M - c0 : Mc;
        const unsigned tiles = (unsigned)((mc + kPairThreads - 1) / kPairThreads);
        if (E > 0) {
            ek<<<dim3(tiles, (unsigned)((E + echunk - 1) / echunk)), kPairThreads, esmem, st>>>(
                (const FscSide*)edge_rec, E, echunk, a.X + c0, a.Y + c0, a.Z + c0, mc, G);
            if (launches) ++*launches;
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        PairArgs b = a;
        b.X = a.X + c0;
        b.Y = a.Y + c0;
        b.Z = a.Z + c0;
        b.dirs = a.dirs ? a.dirs + c0 : nullptr;
        b.A = a.A ? a.A + c0 : nullptr;
        b.trac = a.trac ? a.trac + c0 : nullptr;
        b.strain = a.strain ? a.strain + c0 : nullptr;
        b.disp = a.disp ? a.disp + c0 : nullptr;
        b.M = mc;
        b.Ntot = a.M;   // the output fields' row stride
        b.fscG = G;
        b.side_edge = side_edge;
        pk<<<dim3(tiles, (unsigned)((a.N + a.tri_chunk - 1) / a.tri_chunk)), kPairThreads, psmem, st>>>(b);
        if (launches) ++*launches;
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Net Burgers vector of each mesh edge: the signed sum over the triangle sides
// on it (edge_tris[edge_ptr[e] .. edge_ptr[e + 1]) = +-(triangle + 1), in
// triangle order) of Dn Vn + Dss Vs + Dds Vd, then the edge's record for it.
__global__ void edge_burgers_kernel(const double* __restrict__ pts, int64_t E, const int* __restrict__ edge_ptr,
                                    const int* __restrict__ edge_tris, const TriDev* __restrict__ tri, double nu,
                                    FscSide* __restrict__ out)
{
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= E) return;
    double B[3] = {0.0, 0.0, 0.0};
    for (int k = edge_ptr[e]; k < edge_ptr[e + 1]; ++k) {
        const int c = edge_tris[k];
        const TriDev& t = tri[(c > 0 ? c : -c) - 1];
        const double sg = c > 0 ? 1.0 : -1.0;
        const double slip[3] = {t.Dn, t.Dss, t.Dds};
        const double* axes[3] = {t.real.Vn, t.real.Vs, t.real.Vd};
        for (int m = 0; m < 3; ++m)
            for (int i = 0; i < 3; ++i) B[i] = add_rn(B[i], sg * mul_rn(axes[m][i], slip[m]));
    }
    const double PA[3] = {pts[6 * e], pts[6 * e + 1], pts[6 * e + 2]};
    const double PB[3] = {pts[6 * e + 3], pts[6 * e + 4], pts[6 * e + 5]};
    build_side_burgers(PA, PB, B, nu, out[e]);
}

// partial[(blockIdx.y * 9 + f) M + i] = the free-surface strain (f 0-5) and
// displacement (f 6-8) at point i of the edges of chunk blockIdx.y, summed in
// edge order (each edge record staged in shared memory).
template <bool STRAIN, bool DISP>
__global__ void __launch_bounds__(kPairThreads, 1) fsc_sum_kernel(const FscSide* __restrict__ edges, int64_t E,
                                                                int64_t echunk, const double* __restrict__ X,
                                                                const double* __restrict__ Y,
                                                                const double* __restrict__ Z, int64_t M,
                                                                double* __restrict__ partial)
{
    extern __shared__ double smem[];
    const FscSide& s = *reinterpret_cast<const FscSide*>(smem);
    const int64_t i = (int64_t)blockIdx.x * kPairThreads + threadIdx.x;
    const bool active = i < M;
    double x = 0.0, y = 0.0, z = 0.0;
    if (active) { x = X[i]; y = Y[i]; z = Z[i]; }
    double Es[3][6] = {}, Us[3][3] = {};
    const int64_t e0 = (int64_t)blockIdx.y * echunk;
    const int64_t e1 = min(E, e0 + echunk);
    for (int64_t e = e0; e < e1; ++e) {
        __syncthreads();
        const double* src = reinterpret_cast<const double*>(edges + e);
        for (int w = threadIdx.x; w < kSideWords; w += kPairThreads) smem[w] = src[w];
        __syncthreads();
        if (!active || s.skip != 0.0) continue;
        if (STRAIN) fsc_strain(s, x, y, z, 0.0, 0.0, 1.0, Es);
        if (DISP) fsc_disp(s, x, y, z, 0.0, 0.0, 1.0, Us);
    }
    if (!active) return;
    double* p = partial + (int64_t)blockIdx.y * 9 * M;
#pragma unroll
    for (int k = 0; k < 6; ++k) p[k * M + i] = STRAIN ? Es[0][k] : 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) p[(6 + c) * M + i] = DISP ? Us[0][c] : 0.0;
}

cudaError_t launch_td_sum_edges(PairArgs a, bool strain, bool disp, const double* edge_pts, int64_t E,
                                const int* edge_ptr, const int* edge_tris, void* edge_rec, double nu, int64_t echunk,
                                double* edge_partial, cudaStream_t st, int64_t* launches)
{
    if (a.M == 0 || a.N == 0 || !(strain || disp)) return cudaSuccess;
    const size_t psmem = (size_t)kTriWordsImg * sizeof(double);
    const size_t esmem = (size_t)kSideWords * sizeof(double);
    const unsigned tiles = (unsigned)((a.M + kPairThreads - 1) / kPairThreads);
    auto pairs = [&](auto kern) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem);
        if (e != cudaSuccess) return e;
        kern<<<dim3(tiles, (unsigned)((a.N + a.tri_chunk - 1) / a.tri_chunk)), kPairThreads, psmem, st>>>(a);
        if (launches) ++*launches;
        return cudaGetLastError();
    };
    auto sums = [&](auto kern) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)esmem);
        if (e != cudaSuccess) return e;
        kern<<<dim3(tiles, (unsigned)((E + echunk - 1) / echunk)), kPairThreads, esmem, st>>>(
            (const FscSide*)edge_rec, E, echunk, a.X, a.Y, a.Z, a.M, edge_partial);
        if (launches) ++*launches;
        return cudaGetLastError();
    };
    cudaError_t e = strain && disp ? pairs(td_pair_kernel<true, true, true, OUT_SUM, false, false, 1, true>)
                    : strain       ? pairs(td_pair_kernel<true, true, false, OUT_SUM, false, false, 1, true>)
                                   : pairs(td_pair_kernel<true, false, true, OUT_SUM, false, false, 1, true>);
    if (e != cudaSuccess || E == 0) return e;
    edge_burgers_kernel<<<(unsigned)((E + 127) / 128), 128, 0, st>>>(edge_pts, E, edge_ptr, edge_tris, a.tri, nu,
                                                                      (FscSide*)edge_rec);
    if (launches) ++*launches;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return strain && disp ? sums(fsc_sum_kernel<true, true>)
           : strain       ? sums(fsc_sum_kernel<true, false>)
                          : sums(fsc_sum_kernel<false, true>);
}

cudaError_t launch_splice_fixed(const double* trac, const double* disp, int64_t N, int64_t nfix, const int* fixrow,
                                const int* freecol, int64_t nf, bool amat, double* out, int64_t lda, cudaStream_t st)
{
    if (N == 0 || nf == 0) return cudaSuccess;
    dim3 grid((unsigned)((N + 127) / 128), (unsigned)nf, 9);
    splice_fixed_kernel<<<grid, 128, 0, st>>>(trac, disp, N, nfix, fixrow, freecol, nf, amat ? 1 : 0, out, lda);
    return cudaGetLastError();
}

cudaError_t launch_gather_points(const double* X, const double* Y, const double* Z, const int* idx, int64_t n,
                                 double* out, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    gather_points_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(X, Y, Z, idx, n, out);
    return cudaGetLastError();
}

cudaError_t launch_assemble_mixed(PairArgs a, bool hs, const double* P1, const double* P2, const double* P3,
                                  double near_factor, void* tri32, double* near, cudaStream_t st, int64_t* launches)
{
    if (a.N == 0 || a.M == 0) return cudaSuccess;
    near_setup_kernel<<<1, 1024, 0, st>>>(P1, P2, P3, a.N, near_factor, near);
    const int words = hs ? kTriWordsHS : kTriWordsFS;
    const int64_t total = a.N * words;
    tri_to_f32_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(reinterpret_cast<const double*>(a.tri), a.N,
                                                                         words, kTriWordsHS, (float*)tri32);
    *launches += 2;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    a.tri32 = tri32;
    a.near = near;
    const int64_t ntile = (a.M + kPairThreads - 1) / kPairThreads;
    const int64_t nchunk = (a.N + a.tri_chunk - 1) / a.tri_chunk;
    dim3 grid((unsigned)ntile, (unsigned)nchunk);
    {
        auto kern = hs ? td_pair_f32_kernel<true> : td_pair_f32_kernel<false>;
        const size_t smem = (size_t)words * sizeof(float);
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, kPairThreads, smem, st>>>(a);
        ++*launches;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    {
        auto kern = hs ? td_pair_kernel<true, true, false, OUT_AMAT, true>
                       : td_pair_kernel<false, true, false, OUT_AMAT, true>;
        const size_t smem = (size_t)words * sizeof(double);
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kern<<<grid, kPairThreads, smem, st>>>(a);
        ++*launches;
    }
    return cudaGetLastError();
}

size_t tri_record_bytes_f32() { return sizeof(TriDevT<float>); }

cudaError_t launch_assemble_update(PairArgs a, bool hs, const int* list, int64_t k, cudaStream_t st,
                                   int64_t* launches)
{
    if (k == 0 || a.N == 0) return cudaSuccess;
    const int words = hs ? kTriWordsHS : kTriWordsFS;
    const size_t smem = (size_t)words * sizeof(double);
    auto kern = hs ? td_pair_kernel<true, true, false, OUT_AMAT, false, true>
                   : td_pair_kernel<false, true, false, OUT_AMAT, false, true>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int64_t Ntot = a.N;
    a.Ntot = Ntot;
    // columns of the listed triangles, every point
    PairArgs c = a;
    c.tri_list = list;
    c.obs_list = nullptr;
    c.M = Ntot;
    c.N = k;
    c.tri_chunk = k < 8 ? k : 8;
    dim3 gc((unsigned)((Ntot + kPairThreads - 1) / kPairThreads), (unsigned)((k + c.tri_chunk - 1) / c.tri_chunk));
    kern<<<gc, kPairThreads, smem, st>>>(c);
    // rows of the listed points, every triangle
    PairArgs r = a;
    r.tri_list = nullptr;
    r.obs_list = list;
    r.M = k;
    r.N = Ntot;
    r.tri_chunk = 8;
    dim3 gr((unsigned)((k + kPairThreads - 1) / kPairThreads), (unsigned)((Ntot + 7) / 8));
    kern<<<gr, kPairThreads, smem, st>>>(r);
    *launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_td_setup(const double* P1, const double* P2, const double* P3, int64_t N, const double* Dss,
                            const double* Dds, const double* Dn, int64_t slip_stride, double nu, bool hs,
                            TriDev* out, cudaStream_t st)
{
    if (N == 0) return cudaSuccess;
    const int bs = 64;
    td_setup_kernel<<<(unsigned)((N + bs - 1) / bs), bs, 0, st>>>(P1, P2, P3, N, Dss, Dds, Dn, slip_stride, nu,
                                                                  hs ? 1 : 0, out);
    return cudaGetLastError();
}

cudaError_t launch_hs_check(const double* Z, int64_t M, const double* P1, const double* P2, const double* P3,
                            int64_t N, int* flag, cudaStream_t st, const double* nz, bool clear)
{
    cudaError_t e = clear ? cudaMemsetAsync(flag, 0, sizeof(int), st) : cudaSuccess;
    if (e != cudaSuccess || M + N == 0) return e;
    const int bs = 256;
    int64_t nb = (M + N + bs - 1) / bs;
    if (nb > 1184) nb = 1184;
    hs_check_kernel<<<(unsigned)nb, bs, 0, st>>>(Z, nz, M, P1, P2, P3, N, flag);
    return cudaGetLastError();
}

cudaError_t launch_colloc(const double* normals, const double* mid, int64_t N, double* X, double* Y, double* Z,
                          double* dirs, cudaStream_t st)
{
    if (N == 0) return cudaSuccess;
    const int bs = 128;
    colloc_kernel<<<(unsigned)((N + bs - 1) / bs), bs, 0, st>>>(normals, mid, N, X, Y, Z, dirs);
    return cudaGetLastError();
}

cudaError_t launch_sum_chunks(const double* partial, int64_t nchunk, int64_t M, int fields_mask, double* out,
                              cudaStream_t st)
{
    if (M == 0) return cudaSuccess;
    const int bs = 256;
    dim3 grid((unsigned)((M + bs - 1) / bs), 9);
    sum_chunks_kernel<<<grid, bs, 0, st>>>(partial, nchunk, M, fields_mask, out);
    return cudaGetLastError();
}

cudaError_t launch_sum_chunks_split(const double* partial, int64_t nchunk, int64_t M, int fields_mask,
                                    double* strain_out, double* disp_out, cudaStream_t st)
{
    if (M == 0) return cudaSuccess;
    const int bs = 256;
    dim3 grid((unsigned)((M + bs - 1) / bs), 9);
    sum_chunks_split_kernel<<<grid, bs, 0, st>>>(partial, nchunk, M, fields_mask, strain_out, disp_out);
    return cudaGetLastError();
}

cudaError_t launch_td_sum(const double* in, int64_t M, int64_t N, int nf, double* out, cudaStream_t st)
{
    if (M == 0) return cudaSuccess;
    const int bs = 256;
    dim3 grid((unsigned)((M + bs - 1) / bs), (unsigned)nf);
    td_sum_kernel<<<grid, bs, 0, st>>>(in, M, N, nf, out);
    return cudaGetLastError();
}

}  // namespace cad
