// Internal launch interface of the TD pair kernels (host side of td_kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace cad {

template <typename T>
struct TriDevT;
using TriDev = TriDevT<double>;

constexpr int kPairThreads = 128;
constexpr int kEdgeMinBlocks = 3;   // default build of the shared-edge pair kernel

enum OutKind { OUT_INF = 0, OUT_SUM = 1, OUT_TRAC = 2, OUT_AMAT = 3 };

struct PairArgs {
    const double* X;
    const double* Y;
    const double* Z;
    int64_t M;
    const TriDev* tri;
    int64_t N;
    int64_t tri_chunk;   // triangles per block (grid.y = ceil(N / tri_chunk))
    double lambda, G;
    double* strain;      // OUT_INF: 18 x M x N
    double* disp;        // OUT_INF: 9 x M x N
    double* partial;     // OUT_SUM: nchunk x 9 x M
    double* trac;        // OUT_TRAC: 9 x M x N
    double* A;           // OUT_AMAT: 3M x 3N column-major, leading dimension lda (row r*M + i,
                         // column m*N + j; a column block of a system when N < M)
    int64_t lda;
    const double* dirs;  // OUT_TRAC / OUT_AMAT: 9 x M (normal, strike, dip of each observed element)
    // mixed-precision assembly (OUT_AMAT): FP32 records of the triangles, and
    // the near field -- centroids (3 x N) followed by the squared radius
    const void* tri32;
    const double* near;
    // incremental re-assembly (OUT_AMAT): only the triangles tri_list[0..N)
    // (columns) or only the points obs_list[0..M) (rows) of a system of Ntot
    // elements; X, Y, Z, dirs and tri then cover all Ntot elements
    const int* tri_list;
    const int* obs_list;
    int64_t Ntot;
    // half-space system matrix: the kernel variant compiled for this many
    // resident blocks per SM (1: the full register file; 3 or 4)
    int min_blocks = 1;
    // half-space system matrix with shared-edge free-surface maps: the maps
    // of this launch's points (18 x M per edge, fsc_edge_kernel) and each
    // triangle's three side codes (+-(edge + 1), 0: none); rows are then a
    // block of an Ntot-point system (X, Y, Z, dirs and A or trac start at the
    // block; the output fields keep the system's row stride)
    const double* fscG = nullptr;
    const int* side_edge = nullptr;
};

// Half-space system matrix (out_kind OUT_AMAT), traction fields (OUT_TRAC) or
// influence fields (OUT_INF, strain and / or displacement), FP64, with the
// free-surface correction evaluated once per mesh edge at each point:
// edge_pts holds E edges (PA, PB: 6 doubles each), side_edge each triangle's
// three side codes; edge_rec (edge_record_bytes() x E) and G (Q x Mc x E
// doubles, Q = 18 for strain + 9 for displacement) are workspaces; the points
// are processed in blocks of Mc.  OUT_AMAT / OUT_TRAC: a.M == a.N (the
// collocation points).  a.min_blocks selects the system-matrix and traction
// kernels' build: 1 (the full register file) or anything else for three
// resident blocks per SM (kEdgeMinBlocks).
cudaError_t launch_assemble_edges(PairArgs a, int out_kind, bool strain, bool disp, const double* edge_pts,
                                  int64_t E, const int* side_edge, void* edge_rec, double* G, int64_t Mc, double nu,
                                  cudaStream_t st, int64_t* launches);
size_t edge_record_bytes();

// Half-space sums (OUT_SUM) with the free-surface correction evaluated once
// per mesh edge for the net Burgers vector of the triangle sides on it:
// a.partial receives the real + image terms of each triangle chunk (as
// launch_td_pairs), edge_partial the corrections of each chunk of echunk
// edges (9 x a.M each).  edge_ptr / edge_tris list each edge's sides as
// +-(triangle + 1), + for a side running the edge's way.  a.tri must hold the
// records of launch_td_setup (with the triangles' slip).
cudaError_t launch_td_sum_edges(PairArgs a, bool strain, bool disp, const double* edge_pts, int64_t E,
                                const int* edge_ptr, const int* edge_tris, void* edge_rec, double nu, int64_t echunk,
                                double* edge_partial, cudaStream_t st, int64_t* launches);

// Mixed-precision system matrix: every pair in FP32 (far field), then the
// pairs of every 128-point tile that has a point within the near radius of
// the source centroid again in FP64.  near_factor: radius in mean edge lengths.
cudaError_t launch_assemble_mixed(PairArgs a, bool hs, const double* P1, const double* P2, const double* P3,
                                  double near_factor, void* tri32, double* near, cudaStream_t st, int64_t* launches);
size_t tri_record_bytes_f32();

// Rows and columns of the k elements `list` (device) of an assembled system
// matrix recomputed in FP64 (a: the full system's points, directions and
// triangle records; a.N = a.M = the full size).
cudaError_t launch_assemble_update(PairArgs a, bool hs, const int* list, int64_t k, cudaStream_t st,
                                   int64_t* launches);

// Fixed-element splice (see td_kernels.cu) and a gather of points by index.
cudaError_t launch_splice_fixed(const double* trac, const double* disp, int64_t N, int64_t nfix, const int* fixrow,
                                const int* freecol, int64_t nf, bool amat, double* out, int64_t lda, cudaStream_t st);
cudaError_t launch_gather_points(const double* X, const double* Y, const double* Z, const int* idx, int64_t n,
                                 double* out, cudaStream_t st);

size_t tri_record_bytes();

cudaError_t launch_td_setup(const double* P1, const double* P2, const double* P3, int64_t N, const double* Dss,
                            const double* Dds, const double* Dn, int64_t slip_stride, double nu, bool hs,
                            TriDev* out, cudaStream_t st);
cudaError_t launch_td_pairs(const PairArgs& a, int out, bool hs, bool strain, bool disp, cudaStream_t st);
// flag |= 1 when an observation z or a vertex z is above 0 (nz set: the
// observation z is Z - 1e-12 nz); clear: zero the flag first.
cudaError_t launch_hs_check(const double* Z, int64_t M, const double* P1, const double* P2, const double* P3,
                            int64_t N, int* flag, cudaStream_t st, const double* nz = nullptr, bool clear = true);
cudaError_t launch_colloc(const double* normals, const double* mid, int64_t N, double* X, double* Y, double* Z,
                          double* dirs, cudaStream_t st);
cudaError_t launch_sum_chunks(const double* partial, int64_t nchunk, int64_t M, int fields_mask, double* out,
                              cudaStream_t st);
cudaError_t launch_sum_chunks_split(const double* partial, int64_t nchunk, int64_t M, int fields_mask,
                                    double* strain_out, double* disp_out, cudaStream_t st);
cudaError_t launch_td_sum(const double* in, int64_t M, int64_t N, int nf, double* out, cudaStream_t st);

}  // namespace cad
