// TD summing evaluation for callers that cannot allocate device memory.
//
// Some hosts must not have a library call cudaMalloc behind their back: a
// Julia or Python process whose device memory is owned by its own pool and
// budget (an allocation outside it can fail under memory pressure or push the
// pool into an out-of-memory state), or a service that gives each tenant a
// fixed slice of the GPU and forbids growth after start-up.  cudaMalloc and
// cudaFree also synchronise the device, which such callers want to avoid.
//
// cad_td_sum_eval_noalloc runs the same kernels as cad_td_sum_eval_dev but
// keeps every intermediate (the per-triangle records and the per-chunk partial
// sums) in one file-scope device array of fixed size, so the call itself
// allocates nothing: no context, no cudaMalloc / cudaFree, no library routine
// that allocates.  The caller passes device inputs and outputs and a stream.
//
// Limits: at most kMaxTri triangles and kMaxObs observation points per call
// (CAD_ERR_TOO_LARGE beyond that).  The array (about 25 MiB) is reserved on
// every GPU that loads the library, until the process exits.  All calls share
// it and it keeps the previous call's contents, so two calls whose work
// overlaps on the GPU (different streams, or different host threads on one
// device) race on it; order them on one stream.  The first call on a device
// looks up the array's device address (cudaGetSymbolAddress) with that device
// current; make that first call before any stream capture.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/cad_td.h"
#include "td_device.cuh"
#include "td_kernels.h"

namespace {

constexpr int64_t kMaxTri = 1024;
constexpr int64_t kMaxObs = 16384;
constexpr int64_t kMaxChunks = 8;
constexpr size_t kFlagBytes = 256;
constexpr size_t kTriBytes = (size_t)kMaxTri * sizeof(cad::TriDev);
constexpr size_t kPartBytes = (size_t)kMaxChunks * 9 * kMaxObs * sizeof(double);
constexpr size_t kScratchBytes = kFlagBytes + ((kTriBytes + 255) / 256) * 256 + kPartBytes;

// The scratch array.  Host code must not use its name as a device address;
// the address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the array on the current device (looked up once per device).
int scratch_address(void** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CAD_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CAD_ERR_CUDA;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return CAD_OK;
}

}  // namespace

extern "C" int cad_td_sum_eval_noalloc(void* stream, const double* X, const double* Y, const double* Z, int64_t M,
                                       const double* P1, const double* P2, const double* P3, int64_t N,
                                       const double* Dss, const double* Dds, const double* Dn, double nu,
                                       int disp_flag, int strain_flag, int hs_flag, double* strain_out,
                                       double* disp_out)
{
    using namespace cad;
    if (M < 0 || N < 0 || (disp_flag != 0 && disp_flag != 1) || (strain_flag != 0 && strain_flag != 1) ||
        (hs_flag != 0 && hs_flag != 1))
        return CAD_ERR_ARG;
    if ((strain_flag == 1 && !strain_out) || (disp_flag == 1 && !disp_out)) return CAD_ERR_ARG;
    if (M > kMaxObs || N > kMaxTri) return CAD_ERR_TOO_LARGE;
    // with no points there is nothing to evaluate, but half-space triangles
    // are still checked, as cad_td_sum_eval_dev and the reference do
    if (M == 0 && (hs_flag == 0 || N == 0)) return CAD_OK;
    cudaStream_t st = (cudaStream_t)stream;
    void* base = nullptr;
    if (int r = scratch_address(&base)) return r;
    unsigned char* b = (unsigned char*)base;
    int* flag = (int*)b;
    TriDev* tri = (TriDev*)(b + kFlagBytes);
    double* part = (double*)(b + kFlagBytes + ((kTriBytes + 255) / 256) * 256);

    if (hs_flag == 1 && N > 0) {
        // the flag must start at zero: the array keeps the last call's contents
        if (launch_hs_check(Z, M, P1, P2, P3, N, flag, st) != cudaSuccess) return CAD_ERR_CUDA;
        int h = 0;
        if (cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return CAD_ERR_CUDA;
        if (h) return CAD_ERR_HS_ABOVE_SURFACE;
    }
    if (M == 0) return CAD_OK;
    if (N == 0) {
        if (strain_flag == 1 && cudaMemsetAsync(strain_out, 0, 6 * M * sizeof(double), st) != cudaSuccess)
            return CAD_ERR_CUDA;
        if (disp_flag == 1 && cudaMemsetAsync(disp_out, 0, 3 * M * sizeof(double), st) != cudaSuccess)
            return CAD_ERR_CUDA;
        return CAD_OK;
    }
    if (launch_td_setup(P1, P2, P3, N, Dss, Dds, Dn, 1, nu, hs_flag == 1, tri, st) != cudaSuccess)
        return CAD_ERR_CUDA;
    PairArgs a{};
    a.X = X; a.Y = Y; a.Z = Z; a.M = M; a.tri = tri; a.N = N;
    const int64_t tiles = (M + kPairThreads - 1) / kPairThreads;
    int64_t nchunk = (148 * 16 + tiles - 1) / tiles;
    if (nchunk > kMaxChunks) nchunk = kMaxChunks;
    if (nchunk > N) nchunk = N;
    a.tri_chunk = (N + nchunk - 1) / nchunk;
    nchunk = (N + a.tri_chunk - 1) / a.tri_chunk;
    a.partial = part;   // every (chunk, field, row < M) entry is written before it is read
    if (launch_td_pairs(a, OUT_SUM, hs_flag == 1, strain_flag == 1, disp_flag == 1, st) != cudaSuccess)
        return CAD_ERR_CUDA;
    const int mask = (strain_flag == 1 ? 0x3f : 0) | (disp_flag == 1 ? 0x1c0 : 0);
    if (launch_sum_chunks_split(part, nchunk, M, mask, strain_out, disp_out, st) != cudaSuccess) return CAD_ERR_CUDA;
    return CAD_OK;
}
