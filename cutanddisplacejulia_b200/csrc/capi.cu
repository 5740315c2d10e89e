// C ABI of libcad_td.so (declared in include/cad_td.h).
//
// Each context owns its CUDA streams (the caller-visible one, a low-priority
// side stream for the LU's look-ahead updates, four leaf streams for grouped
// factorisations) and a set of device workspaces that grow on demand and are
// reused across calls (no allocation in steady state).  Host-pointer entry points copy inputs in,
// run the device path and copy results out; *_dev entry points run the device
// path directly on caller-provided device memory.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/cad_td.h"
#include "gemm.h"
#include "krylov.h"
#include "lcp.h"
#include "lpc.h"
#include "tune.h"
#include "lu.h"
#include "mixed.h"
#include "mlp.h"
#include "td_device.cuh"
#include "td_kernels.h"

using namespace cad;

namespace cad {
size_t tri_record_bytes() { return sizeof(TriDev); }
}

namespace {

enum Slot {
    S_OBS, S_GEOM, S_SLIP, S_TRI, S_OUT, S_PART, S_DIRS, S_FLAG, S_A, S_B, S_WORK, S_PIV, S_INFO, S_PERM,
    S_A32, S_DINV, S_KRYLOV, S_VEC32, S_SYNC, S_TRI32, S_NEAR, S_IR, S_IR32, S_NORMS, S_REL, S_BGEOM, S_BTD, S_MLP,
    S_FIX, S_FOBS, S_FDISP, S_ATA, S_LIST, S_CHAIN, S_LCPJ, S_LCPC, S_LCPV, S_LCPP, S_GEMM, S_LPC_NET, S_LPC_WS, S_LPC_GEOM, S_LPC_TNBR, S_LPC_FEAT, S_LPC_OUT,
    S_LPC_NBR, S_LPC_BLK, S_LPC_MAT, S_LPC_PGEOM, S_BJ_NBR, S_BJ_BLK, S_KWORK, S_A32MV, S_TUNE, S_AT, S_G_A32, S_G_INT, S_G_F32, S_G_F64, S_G_MAPS,
    S_EDGE_PTS, S_EDGE_CODE, S_EDGE_REC, S_EDGE_G, S_EDGE_PTR, S_EDGE_TRIS, S_COUNT
};

constexpr int kGmresRestart = 30; // default Krylov dimension of a GMRES cycle
constexpr int kLuBlock = 256;     // outer block width of the FP64 LU
constexpr int kLuBlock32 = 512;   // of the FP32 factorisation (its TF32 products gain more from a long k)
constexpr size_t kEdgeMapBytes = size_t(8) << 30;   // cap on the shared-edge free-surface maps of one chunk

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// One lane of the batched solve: its own streams and workspaces, so cracks
// on different lanes run concurrently.
enum LaneSlot { L_OBS, L_DIRS, L_TRI, L_TRI32, L_NEAR, L_A32, L_PIV, L_PERM, L_INFO, L_IR, L_IR32, L_NORMS,
                L_KWORK, L_DINV, L_SYNC, L_Z, L_COUNT };
struct Lane {
    cudaStream_t main = nullptr, side = nullptr;
    cudaEvent_t done = nullptr;
    DevBuf buf[L_COUNT];
};
constexpr int kLanes = 32;           // cracks of a batch in flight at once
constexpr int kBatchSweeps = 4;      // refinement sweeps per crack inside the batch graph
constexpr int kGroupBlock = 128;     // block width of the grouped FP32 factorisation (systems padded to it)
constexpr int kGroupExtraRounds = 3; // rounds of two more grouped sweeps for cracks still above the tolerance
constexpr int kLeafAux = 4;          // streams for the grouped leaves of different cluster sizes

// The captured graph of the last batched call and what it was captured for.
struct BatchGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<int64_t> offsets;
    const void* ptrs[9] = {};
    double params[5] = {};
    int flags[3] = {};
    int64_t launches = 0;
};

}  // namespace

struct cad_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t side_stream = nullptr;   // the LU's look-ahead trailing updates
    LuGraphCache* graphs = nullptr;       // captured LU factorisations, replayed for repeated calls
    std::vector<Lane> lanes;              // batched solve (created on first use)
    BatchGraph batch;
    DevBuf buf[S_COUNT];
    // event pairs: [0,1] TD pair kernel, [2,3] dense solve, [2,4] its
    // factorisation (mixed solver: cast + FP32 LU + block inverses)
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    bool timed[3] = {false, false, false};
    int64_t launches = 0;   // own kernel launches issued through this context
    int solver = CAD_SOLVER_LU64;   // cad_set_solver
    int assembly = CAD_ASSEMBLY_FP64;   // cad_set_assembly
    const int* spai_nbr = nullptr;      // cad_set_preconditioner (caller's device memory)
    const float* spai_blocks = nullptr;
    int64_t spai_N = 0;
    int spai_k = 0;
    double near_factor = 3.0;
    long wait_limit = kDefaultWaitLimit;   // cad_set_wait_limit
    int gmres_matvec32 = 1;                // cad_set_gmres_matvec: FP32 copy of A for the Arnoldi products
    int batch_mode = CAD_BATCH_GROUPED;    // cad_set_batch_solve
    int lu_block = 0;                      // cad_set_lu_block: outer block width of single-system LUs (0: default)
    int gmres_restart = kGmresRestart;          // cad_set_gmres_restart: Krylov dimension of a cycle
    std::vector<CUtensorMap> gmaps_host;   // tensor maps of the grouped batch's FP32 systems
    cudaStream_t leaf_aux[kLeafAux] = {};  // grouped leaves of different cluster sizes, side by side
    cudaEvent_t side_fork = nullptr, side_join = nullptr;   // work forked onto the side stream
    Tuner tuner;                           // cad_set_autotune
    int shared_edges = 1;                  // cad_set_shared_edges
    // mesh-edge table of the last half-space assembly: the vertices it was
    // built from (P1, P2, P3, 3 N each), its edges' endpoints (6 per edge)
    // and each triangle side's signed edge number (0 for none); per edge, the
    // signed triangles on it (edge_ptr offsets into edge_tris)
    std::vector<double> edge_geom, edge_pts;
    std::vector<int> edge_code, edge_ptr, edge_tris;
    int64_t edge_n = -1;
    double tol = 1e-10;
    int max_iter = 200;
    bool fric_ready = false;      // cad_friction_prepare: C = inv(A Scl) of fric_N elements in S_LCPC
    int64_t fric_N = 0;
    double fric_scl = 0.0;
    int last_iters = 0;           // of the last mixed solve (all right-hand sides)
    double last_relres = 0.0;     // largest over its right-hand sides
    // learned preconditioner: network weights, Adam moments and gradients in
    // S_LPC_NET (4 x mlp_param_count floats), Adam step count, training set
    bool lpc_net = false;
    int64_t lpc_t = 0;
    float* lpc_X = nullptr;       // lpc_rows x 112 network inputs
    float* lpc_T = nullptr;       // lpc_rows x 144 exact-inverse targets
    int64_t lpc_rows = 0, lpc_cap = 0;
    std::string err;
};

namespace {

// One NVTX range per C-ABI call, named after the entry point: a profiler's
// timeline shows which call each kernel belongs to (no cost without a tool).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
#define CAD_NVTX_RANGE() NvtxRange nvtx_range_(__func__)

// outer block width of a single-system factorisation
int lu_nb(const cad_ctx* c, bool fp32) { return c->lu_block > 0 ? c->lu_block : (fp32 ? kLuBlock32 : kLuBlock); }

int fail(cad_ctx* c, int code, const std::string& msg)
{
    if (c) c->err = msg;
    return code;
}

int cuda_fail(cad_ctx* c, cudaError_t e, const char* what)
{
    const int code = (e == cudaErrorMemoryAllocation) ? CAD_ERR_OOM : CAD_ERR_CUDA;
    return fail(c, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(expr)                                                        \
    do {                                                                \
        cudaError_t e_ = (expr);                                        \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #expr);        \
    } while (0)

int ensure(cad_ctx* ctx, Slot s, size_t bytes, void** out)
{
    DevBuf& b = ctx->buf[s];
    if (bytes == 0) bytes = 16;
    if (b.bytes < bytes) {
        if (b.p) {
            CK(cudaStreamSynchronize(ctx->stream));
            CK(cudaFree(b.p));
            b.p = nullptr;
            b.bytes = 0;
        }
        const size_t grown = bytes + bytes / 8;
        CK(cudaMalloc(&b.p, grown));
        b.bytes = grown;
    }
    *out = b.p;
    return CAD_OK;
}

int set_device(cad_ctx* ctx)
{
    if (!ctx) return CAD_ERR_ARG;
    CK(cudaSetDevice(ctx->device));
    return CAD_OK;
}

// Triangles per block along grid.y: enough blocks to fill every SM several
// times while keeping each block's triangle loop long enough to amortise the
// shared-memory staging.
int64_t pick_chunk(int64_t M, int64_t N, bool sum_mode)
{
    if (N <= 0) return 1;
    const int64_t tiles = (M + kPairThreads - 1) / kPairThreads;
    const int64_t target_blocks = 148 * 16;
    int64_t nchunk = (target_blocks + tiles - 1) / tiles;
    if (!sum_mode) nchunk = nchunk < (N + 7) / 8 ? (N + 7) / 8 : nchunk;   // at most 8 triangles per block
    if (nchunk > N) nchunk = N;
    if (nchunk < 1) nchunk = 1;
    return (N + nchunk - 1) / nchunk;
}

int hs_check(cad_ctx* ctx, const double* Z, int64_t M, const double* P1, const double* P2, const double* P3,
             int64_t N)
{
    void* flag;
    if (int r = ensure(ctx, S_FLAG, sizeof(int), &flag)) return r;
    ++ctx->launches;
    CK(launch_hs_check(Z, M, P1, P2, P3, N, (int*)flag, ctx->stream));
    int h = 0;
    CK(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h) return fail(ctx, CAD_ERR_HS_ABOVE_SURFACE, "Half-space solution: Z coordinates must be negative!");
    return CAD_OK;
}

// Number the mesh's distinct triangle sides (edges).  Side s of triangle j
// runs P1->P2, P2->P3, P3->P1; its code is e + 1 when it runs the way edge e
// was first seen, -(e + 1) when it runs the other way.  Endpoints match when
// their coordinates are equal (-0.0 taken as 0.0).  The table is rebuilt only
// when the vertices differ from the last call's; the device copies of the
// edge endpoints and codes are uploaded with it.
struct EdgeKey {
    double v[6];
    bool operator==(const EdgeKey& o) const { return std::memcmp(v, o.v, sizeof v) == 0; }
};
struct EdgeKeyHash {
    size_t operator()(const EdgeKey& k) const
    {
        uint64_t h = 1469598103934665603ull;
        for (double d : k.v) {
            uint64_t u;
            std::memcpy(&u, &d, sizeof u);
            h = (h ^ u) * 1099511628211ull;
            h ^= h >> 29;
        }
        return (size_t)h;
    }
};

struct EdgeTable {
    int64_t E = 0;
    double* pts = nullptr;   // device: 6 doubles per edge
    int* code = nullptr;     // device: 3 per triangle
    int* ptr = nullptr;      // device: E + 1 offsets into tris
    int* tris = nullptr;     // device: +-(triangle + 1) per side, by edge
};

// Shared-edge work pays when the mesh's edges are clearly fewer than its
// triangle sides (a manifold mesh has about half); a soup of unconnected
// triangles stays on the per-side kernels.
bool edges_pay(int64_t E, int64_t N) { return 10 * E < 9 * 3 * N; }

int edge_table(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, EdgeTable* out)
{
    if (3 * N > INT32_MAX) {   // side codes are ints: such meshes stay on the per-side path
        out->E = 3 * N;
        return CAD_OK;
    }
    std::vector<double> geom((size_t)9 * N);
    CK(cudaMemcpyAsync(geom.data(), P1, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(geom.data() + 3 * N, P2, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(geom.data() + 6 * N, P3, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    void *pts, *code, *eptr, *etris;
    const bool same = ctx->edge_n == N && ctx->edge_geom == geom;
    if (!same) {
        std::unordered_map<EdgeKey, int, EdgeKeyHash> seen;
        seen.reserve((size_t)3 * N);
        ctx->edge_pts.clear();
        ctx->edge_code.assign((size_t)3 * N, 0);
        for (int64_t j = 0; j < N; ++j)
            for (int sd = 0; sd < 3; ++sd) {
                const double* va = geom.data() + 3 * N * sd + j;
                const double* vb = geom.data() + 3 * N * ((sd + 1) % 3) + j;
                // + 0.0 turns -0.0 into 0.0
                const EdgeKey fwd{{va[0] + 0.0, va[N] + 0.0, va[2 * N] + 0.0, vb[0] + 0.0, vb[N] + 0.0, vb[2 * N] + 0.0}};
                const EdgeKey rev{{fwd.v[3], fwd.v[4], fwd.v[5], fwd.v[0], fwd.v[1], fwd.v[2]}};
                int c;
                auto it = seen.find(fwd);
                if (it != seen.end()) {
                    c = it->second + 1;
                } else if ((it = seen.find(rev)) != seen.end()) {
                    c = -(it->second + 1);
                } else {
                    const int e = (int)seen.size();
                    seen.emplace(fwd, e);
                    ctx->edge_pts.insert(ctx->edge_pts.end(), fwd.v, fwd.v + 6);
                    c = e + 1;
                }
                ctx->edge_code[(size_t)3 * j + sd] = c;
            }
        // edge -> sides, in triangle order (counting sort on the edge number)
        const size_t E = ctx->edge_pts.size() / 6;
        ctx->edge_ptr.assign(E + 1, 0);
        for (int c : ctx->edge_code) ++ctx->edge_ptr[(size_t)(c > 0 ? c : -c)];
        for (size_t e = 0; e < E; ++e) ctx->edge_ptr[e + 1] += ctx->edge_ptr[e];
        ctx->edge_tris.assign((size_t)3 * N, 0);
        std::vector<int> fill(ctx->edge_ptr.begin(), ctx->edge_ptr.end() - 1);
        for (int64_t k = 0; k < 3 * N; ++k) {
            const int c = ctx->edge_code[(size_t)k];
            const int t = (int)(k / 3) + 1;
            ctx->edge_tris[(size_t)fill[(size_t)((c > 0 ? c : -c) - 1)]++] = c > 0 ? t : -t;
        }
        ctx->edge_n = -1;
        if (int r = ensure(ctx, S_EDGE_PTS, ctx->edge_pts.size() * sizeof(double), &pts)) return r;
        if (int r = ensure(ctx, S_EDGE_CODE, ctx->edge_code.size() * sizeof(int), &code)) return r;
        if (int r = ensure(ctx, S_EDGE_PTR, ctx->edge_ptr.size() * sizeof(int), &eptr)) return r;
        if (int r = ensure(ctx, S_EDGE_TRIS, ctx->edge_tris.size() * sizeof(int), &etris)) return r;
        CK(cudaMemcpyAsync(eptr, ctx->edge_ptr.data(), ctx->edge_ptr.size() * sizeof(int), cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(cudaMemcpyAsync(etris, ctx->edge_tris.data(), ctx->edge_tris.size() * sizeof(int),
                           cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(pts, ctx->edge_pts.data(), ctx->edge_pts.size() * sizeof(double),
                           cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(code, ctx->edge_code.data(), ctx->edge_code.size() * sizeof(int),
                           cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->edge_geom.swap(geom);
        ctx->edge_n = N;
    } else {
        pts = ctx->buf[S_EDGE_PTS].p;
        code = ctx->buf[S_EDGE_CODE].p;
        eptr = ctx->buf[S_EDGE_PTR].p;
        etris = ctx->buf[S_EDGE_TRIS].p;
    }
    out->E = (int64_t)(ctx->edge_pts.size() / 6);
    out->pts = (double*)pts;
    out->code = (int*)code;
    out->ptr = (int*)eptr;
    out->tris = (int*)etris;
    return CAD_OK;
}

// Device path shared by the TD entry points (inputs already on the device).
int td_device(cad_ctx* ctx, const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
              const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds, const double* Dn,
              double nu, int disp, int strain, int hs, int out_kind, double* strain_out, double* disp_out,
              double* sum_out /* 9 x M for OUT_SUM */)
{
    if (hs == 1 && N > 0)
        if (int r = hs_check(ctx, Z, M, P1, P2, P3, N)) return r;
    if (M == 0 || N == 0) {
        if (out_kind == OUT_SUM && sum_out) CK(cudaMemsetAsync(sum_out, 0, 9 * M * sizeof(double), ctx->stream));
        return CAD_OK;
    }
    void* tri;
    if (int r = ensure(ctx, S_TRI, (size_t)N * tri_record_bytes(), &tri)) return r;
    ++ctx->launches;
    CK(launch_td_setup(P1, P2, P3, N, Dss, Dds, Dn, 1, nu, hs == 1, (TriDev*)tri, ctx->stream));
    PairArgs a{};
    a.X = X; a.Y = Y; a.Z = Z; a.M = M; a.tri = (const TriDev*)tri; a.N = N;
    a.tri_chunk = pick_chunk(M, N, out_kind == OUT_SUM);
    a.strain = strain_out; a.disp = disp_out;
    const int64_t nchunk = (N + a.tri_chunk - 1) / a.tri_chunk;
    EdgeTable et;
    const bool edge_kind = (out_kind == OUT_SUM || out_kind == OUT_INF) && hs == 1 && ctx->shared_edges &&
                           (strain == 1 || disp == 1);
    if (edge_kind)
        if (int r = edge_table(ctx, P1, P2, P3, N, &et)) return r;
    if (edge_kind && out_kind == OUT_INF && edges_pay(et.E, N)) {
        // per-edge free-surface maps at the points (strain 18, displacement
        // 9 values), read by the triangles that share each edge
        void *rec, *gmap;
        if (int r = ensure(ctx, S_EDGE_REC, (size_t)et.E * edge_record_bytes(), &rec)) return r;
        const int64_t per_point = (18 * (strain == 1) + 9 * (disp == 1)) * et.E * (int64_t)sizeof(double);
        int64_t Mc = (int64_t)(kEdgeMapBytes / per_point) / kPairThreads * kPairThreads;
        if (Mc < kPairThreads) Mc = kPairThreads;
        if (Mc > M) Mc = M;
        if (int r = ensure(ctx, S_EDGE_G, (size_t)Mc * per_point, &gmap)) return r;
        CK(cudaEventRecord(ctx->ev[0], ctx->stream));
        CK(launch_assemble_edges(a, OUT_INF, strain == 1, disp == 1, et.pts, et.E, et.code, rec, (double*)gmap, Mc,
                                 nu, ctx->stream, &ctx->launches));
        CK(cudaEventRecord(ctx->ev[1], ctx->stream));
        ctx->timed[0] = true;
        return CAD_OK;
    }
    if (edge_kind && out_kind == OUT_SUM && edges_pay(et.E, N)) {
        // real + image terms per triangle chunk, then each mesh edge's
        // free-surface correction once, for the net Burgers vector of the
        // sides on it; all partials summed in one fixed order
        const int64_t echunk = pick_chunk(M, et.E, true);
        const int64_t nechunk = (et.E + echunk - 1) / echunk;
        void *part, *rec;
        if (int r = ensure(ctx, S_PART, (size_t)(nchunk + nechunk) * 9 * M * sizeof(double), &part)) return r;
        if (int r = ensure(ctx, S_EDGE_REC, (size_t)et.E * edge_record_bytes(), &rec)) return r;
        a.partial = (double*)part;
        CK(cudaEventRecord(ctx->ev[0], ctx->stream));
        CK(launch_td_sum_edges(a, strain == 1, disp == 1, et.pts, et.E, et.ptr, et.tris, rec, nu, echunk,
                               a.partial + (size_t)nchunk * 9 * M, ctx->stream, &ctx->launches));
        CK(cudaEventRecord(ctx->ev[1], ctx->stream));
        ctx->timed[0] = true;
        const int mask = (strain == 1 ? 0x3f : 0) | (disp == 1 ? 0x1c0 : 0);
        ++ctx->launches;
        CK(launch_sum_chunks(a.partial, nchunk + nechunk, M, mask, sum_out, ctx->stream));
        return CAD_OK;
    }
    if (out_kind == OUT_SUM) {
        void* part;
        if (int r = ensure(ctx, S_PART, (size_t)nchunk * 9 * M * sizeof(double), &part)) return r;
        a.partial = (double*)part;
    }
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    ++ctx->launches;
    CK(launch_td_pairs(a, out_kind, hs == 1, strain == 1, disp == 1, ctx->stream));
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    ctx->timed[0] = true;
    if (out_kind == OUT_SUM) {
        const int mask = (strain == 1 ? 0x3f : 0) | (disp == 1 ? 0x1c0 : 0);
        ++ctx->launches;
    CK(launch_sum_chunks(a.partial, nchunk, M, mask, sum_out, ctx->stream));
    }
    return CAD_OK;
}

int assemble_device(cad_ctx* ctx, const double* normals, const double* mid, const double* P1, const double* P2,
                    const double* P3, int64_t N, double nu, double G, double lambda, int hs, int out_kind,
                    double* trac_out, double* A, int64_t lda)
{
    void* obs;
    void* dirs;
    if (int r = ensure(ctx, S_OBS, (size_t)3 * N * sizeof(double), &obs)) return r;
    if (int r = ensure(ctx, S_DIRS, (size_t)9 * N * sizeof(double), &dirs)) return r;
    double* X = (double*)obs;
    ++ctx->launches;
    CK(launch_colloc(normals, mid, N, X, X + N, X + 2 * N, (double*)dirs, ctx->stream));
    if (hs == 1 && N > 0)
        if (int r = hs_check(ctx, X + 2 * N, N, P1, P2, P3, N)) return r;
    if (N == 0) return CAD_OK;
    void* tri;
    if (int r = ensure(ctx, S_TRI, (size_t)N * tri_record_bytes(), &tri)) return r;
    ++ctx->launches;
    CK(launch_td_setup(P1, P2, P3, N, nullptr, nullptr, nullptr, 1, nu, hs == 1, (TriDev*)tri, ctx->stream));
    PairArgs a{};
    a.X = X; a.Y = X + N; a.Z = X + 2 * N; a.M = N; a.tri = (const TriDev*)tri; a.N = N;
    a.tri_chunk = pick_chunk(N, N, false);
    a.lambda = lambda; a.G = G; a.dirs = (const double*)dirs;
    a.trac = trac_out; a.A = A; a.lda = lda;
    if (out_kind == OUT_AMAT && ctx->assembly == CAD_ASSEMBLY_MIXED) {
        void *tri32, *near;
        if (int r = ensure(ctx, S_TRI32, (size_t)N * tri_record_bytes_f32(), &tri32)) return r;
        if (int r = ensure(ctx, S_NEAR, (size_t)(3 * N + 1) * sizeof(double), &near)) return r;
        CK(cudaEventRecord(ctx->ev[0], ctx->stream));
        CK(launch_assemble_mixed(a, hs == 1, P1, P2, P3, ctx->near_factor, tri32, (double*)near, ctx->stream,
                                 &ctx->launches));
        CK(cudaEventRecord(ctx->ev[1], ctx->stream));
        ctx->timed[0] = true;
        return CAD_OK;
    }
    EdgeTable et;
    const bool edge_kind = (out_kind == OUT_AMAT && ctx->assembly != CAD_ASSEMBLY_MIXED) || out_kind == OUT_TRAC;
    if (edge_kind && hs == 1 && ctx->shared_edges)
        if (int r = edge_table(ctx, P1, P2, P3, N, &et)) return r;
    if (edge_kind && hs == 1 && ctx->shared_edges && edges_pay(et.E, N)) {
        // each mesh edge's free-surface map evaluated once, then read by the
        // (one or two) triangles that share the edge
        const int64_t E = et.E;
        double* pts = et.pts;
        int* codes = et.code;
        void *rec, *gmap;
        if (int r = ensure(ctx, S_EDGE_REC, (size_t)(E > 0 ? E : 1) * edge_record_bytes(), &rec)) return r;
        const int64_t per_point = 18 * (E > 0 ? E : 1) * (int64_t)sizeof(double);
        int64_t Mc = (int64_t)(kEdgeMapBytes / per_point) / kPairThreads * kPairThreads;
        if (Mc < kPairThreads) Mc = kPairThreads;
        if (Mc > N) Mc = N;
        if (int r = ensure(ctx, S_EDGE_G, (size_t)Mc * per_point, &gmap)) return r;
        a.min_blocks = kEdgeMinBlocks;
        if (ctx->tuner.mode != TUNE_OFF && out_kind == OUT_AMAT) {
            // triangles per block of the edge pair kernel, then its build
            // (resident blocks per SM); each candidate runs the whole path
            char key[96];
            auto run = [&](const PairArgs& t) {
                return launch_assemble_edges(t, out_kind, true, false, pts, E, codes, rec, (double*)gmap, Mc, nu, ctx->stream,
                                             &ctx->launches);
            };
            std::snprintf(key, sizeof key, "pair_amat_f64_hs1_edge_N%lld", (long long)tune_class(N));
            PairArgs t = a;
            a.tri_chunk = tune_choice(ctx->tuner, key, ctx->stream, {2, 4, 8, 16, 32}, (int)a.tri_chunk, [&](int c) {
                t.tri_chunk = c;
                return run(t);
            });
            std::snprintf(key, sizeof key, "pair_amat_f64_hs1_edge_minblocks_N%lld", (long long)tune_class(N));
            t = a;
            a.min_blocks = tune_choice(ctx->tuner, key, ctx->stream, {kEdgeMinBlocks, 1}, kEdgeMinBlocks, [&](int c) {
                t.min_blocks = c;
                return run(t);
            });
        }
        CK(cudaEventRecord(ctx->ev[0], ctx->stream));
        CK(launch_assemble_edges(a, out_kind, true, false, pts, E, codes, rec, (double*)gmap, Mc, nu, ctx->stream, &ctx->launches));
        CK(cudaEventRecord(ctx->ev[1], ctx->stream));
        ctx->timed[0] = true;
        return CAD_OK;
    }
    if (out_kind == OUT_AMAT && ctx->tuner.mode != TUNE_OFF) {
        // triangles per block of the pair kernel (each block stages one
        // triangle record at a time into shared memory)
        char key[96];
        std::snprintf(key, sizeof key, "pair_amat_f64_hs%d_N%lld", hs, (long long)tune_class(N));
        PairArgs t = a;
        a.tri_chunk = tune_choice(ctx->tuner, key, ctx->stream, {2, 4, 8, 16, 32}, (int)a.tri_chunk, [&](int c) {
            t.tri_chunk = c;
            ++ctx->launches;
            return launch_td_pairs(t, out_kind, hs == 1, true, false, ctx->stream);
        });
        if (hs == 1) {
            // then the half-space kernel's occupancy variant at that chunk
            std::snprintf(key, sizeof key, "pair_amat_f64_hs1_minblocks_N%lld", (long long)tune_class(N));
            t = a;
            a.min_blocks = tune_choice(ctx->tuner, key, ctx->stream, {1, 3, 4}, 1, [&](int c) {
                t.min_blocks = c;
                ++ctx->launches;
                return launch_td_pairs(t, out_kind, true, true, false, ctx->stream);
            });
        }
    }
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    ++ctx->launches;
    CK(launch_td_pairs(a, out_kind, hs == 1, true, false, ctx->stream));
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    ctx->timed[0] = true;
    return CAD_OK;
}

constexpr int kIrMaxIter = 20; // refinement sweeps of a multi-column mixed solve before GMRES takes over

int read_info(cad_ctx* ctx, int* info);

// FP32/TF32 LU + FP64 GMRES: B := A^-1 B, A left unchanged.  Sets *info from
// the FP32 factorisation's pivots (0: all non-zero).
int solve_mixed_device(cad_ctx* ctx, int64_t n, const double* A, int64_t lda, double* B, int64_t ldb, int64_t nrhs,
                       int* info_out)
{
    void *a32, *dinv, *piv, *perm, *info, *kry, *v32, *sync, *work;
    if (int r = ensure(ctx, S_A32, (size_t)mixed_ld(n) * n * sizeof(float), &a32)) return r;
    if (int r = ensure(ctx, S_DINV, mixed_dinv_floats(n) * sizeof(float), &dinv)) return r;
    if (int r = ensure(ctx, S_PIV, (size_t)n * sizeof(int), &piv)) return r;
    if (int r = ensure(ctx, S_PERM, (size_t)n * sizeof(int), &perm)) return r;
    if (int r = ensure(ctx, S_INFO, sizeof(int), &info)) return r;
    const int rs = ctx->gmres_restart;
    if (int r = ensure(ctx, S_KRYLOV, ((size_t)n * (rs + 1) + 3 * (size_t)n + 2 * (rs + 1)) * sizeof(double),
                       &kry))
        return r;
    if (int r = ensure(ctx, S_VEC32, 2 * (size_t)n * sizeof(float), &v32)) return r;
    if (int r = ensure(ctx, S_SYNC, mixed_sync_ints(n) * sizeof(int), &sync)) return r;
    if (int r = ensure(ctx, S_WORK, (size_t)n * sizeof(double), &work)) return r;
    CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    const LuStreams ls{ctx->stream, ctx->side_stream, &ctx->launches,
                        ctx->graphs, ctx->wait_limit};
    ctx->timed[1] = ctx->timed[2] = false;
    int rc = mixed_prepare(ls, A, lda, n, (float*)a32, (float*)dinv, (int*)piv, (int*)perm, (int*)info,
                           lu_nb(ctx, true));
    if (rc == LU_TOO_LARGE) return fail(ctx, CAD_ERR_ARG, "matrix too large for the dense LU");
    if (rc != LU_OK) return fail(ctx, CAD_ERR_CUDA, "FP32 LU failed (CUDA error)");
    CK(cudaEventRecord(ctx->ev[4], ctx->stream));
    ctx->timed[2] = true;
    if (int r = read_info(ctx, info_out)) return r;
    if (*info_out > 0) return CAD_OK;
    double* V = (double*)kry;
    double* w = V + (size_t)n * (rs + 1);
    GmresArgs g{};
    g.stream = ctx->stream;
    g.n = n;
    g.A = A;
    g.lda = lda;
    g.A32 = (const float*)a32;
    g.Dinv = (const float*)dinv;
    g.perm = (const int*)perm;
    g.tol = ctx->tol;
    g.max_iter = ctx->max_iter;
    g.restart = rs;
    g.V = V;
    g.w = w;
    g.z = w + n;
    g.r = w + 2 * n;
    g.hd = w + 3 * n;
    g.y32 = (float*)v32;
    g.x32 = (float*)v32 + n;
    g.sync = (int*)sync;
    g.launches = &ctx->launches;
    g.wait_limit = ctx->wait_limit;
    {
        void* kw;
        if (int r = ensure(ctx, S_KWORK, krylov_work_doubles(n) * sizeof(double), &kw)) return r;
        g.kwork = (double*)kw;
    }
    ctx->last_iters = 0;
    ctx->last_relres = 0.0;
    bool converged = true;
    // several right-hand sides: batched refinement first; GMRES finishes the
    // columns it leaves (their solutions go to the refinement's X, which is
    // copied to B at the end, so GMRES still reads the original B)
    std::vector<char> done((size_t)nrhs, 0);
    double* X = nullptr;
    if (nrhs > 1) {
        void *ir, *ir32, *norms;
        if (int r = ensure(ctx, S_IR, 2 * (size_t)n * nrhs * sizeof(double), &ir)) return r;
        if (int r = ensure(ctx, S_IR32, 2 * (size_t)n * nrhs * sizeof(float), &ir32)) return r;
        if (int r = ensure(ctx, S_NORMS, 2 * (size_t)nrhs * sizeof(double), &norms)) return r;
        X = (double*)ir;
        IrArgs ia{ls, n, A, lda, B, ldb, (int)nrhs, X, (float*)a32, (int*)piv, (int*)perm, (int*)info, lu_nb(ctx, true),
                  ctx->tol, kIrMaxIter, X + (size_t)n * nrhs, (float*)ir32, (float*)ir32 + (size_t)n * nrhs,
                  (double*)norms};
        IrResult res{};
        const int st = ir_solve_batched(ia, &res, done);
        if (st != GMRES_OK) return fail(ctx, CAD_ERR_CUDA, "mixed solve: CUDA error in the refinement");
        ctx->last_iters += res.iterations;
        for (int64_t c = 0; c < nrhs; ++c)
            if (done[c]) ctx->last_relres = res.max_rel_residual > ctx->last_relres ? res.max_rel_residual
                                                                                    : ctx->last_relres;
    }
    for (int64_t c = 0; c < nrhs; ++c) {
        if (done[c]) continue;
        g.b = B + c * ldb;
        g.x = X ? X + c * n : (double*)work;
        GmresResult res{};
        const int st = gmres_ir_solve(g, &res);
        if (st == GMRES_TIMEOUT) return fail(ctx, CAD_ERR_TIMEOUT, "mixed solve: a triangular-solve wait ran out");
        if (st == GMRES_CUDA_ERROR)
            return fail(ctx, CAD_ERR_CUDA, "mixed solve: CUDA error in GMRES");
        converged = converged && st == GMRES_OK;
        ctx->last_iters += res.iterations;
        ctx->last_relres = res.rel_residual > ctx->last_relres ? res.rel_residual : ctx->last_relres;
        if (!X) CK(cudaMemcpyAsync(B + c * ldb, work, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    if (X)
        CK(cudaMemcpy2DAsync(B, ldb * sizeof(double), X, n * sizeof(double), n * sizeof(double), nrhs,
                             cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    ctx->timed[1] = true;
    if (!converged)
        return fail(ctx, CAD_ERR_NOT_CONVERGED, "mixed solve: GMRES did not reach the residual tolerance");
    return CAD_OK;
}

// FP64 GMRES right-preconditioned by the block-sparse preconditioner of
// cad_set_preconditioner (no factorisation); B := A^-1 B, A unchanged.
int solve_spai_device(cad_ctx* ctx, int64_t n, const double* A, int64_t lda, double* B, int64_t ldb, int64_t nrhs)
{
    if (!ctx->spai_nbr || 3 * ctx->spai_N != n)
        return fail(ctx, CAD_ERR_ARG, "no preconditioner for this system size (cad_set_preconditioner)");
    void *kry, *sync, *work;
    const int rs = ctx->gmres_restart;
    if (int r = ensure(ctx, S_KRYLOV, ((size_t)n * (rs + 1) + 3 * (size_t)n + 2 * (rs + 1)) * sizeof(double),
                       &kry))
        return r;
    if (int r = ensure(ctx, S_SYNC, mixed_sync_ints(n) * sizeof(int), &sync)) return r;
    if (int r = ensure(ctx, S_WORK, (size_t)n * sizeof(double), &work)) return r;
    CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    ctx->timed[1] = ctx->timed[2] = false;
    double* V = (double*)kry;
    double* w = V + (size_t)n * (rs + 1);
    GmresArgs g{};
    g.stream = ctx->stream;
    g.n = n;
    g.A = A;
    g.lda = lda;
    g.tol = ctx->tol;
    g.max_iter = ctx->max_iter;
    g.restart = rs;
    g.V = V;
    g.w = w;
    g.z = w + n;
    g.r = w + 2 * n;
    g.hd = w + 3 * n;
    g.sync = (int*)sync;
    g.launches = &ctx->launches;
    g.wait_limit = ctx->wait_limit;
    {
        void* kw;
        if (int r = ensure(ctx, S_KWORK, krylov_work_doubles(n) * sizeof(double), &kw)) return r;
        g.kwork = (double*)kw;
    }
    g.spai_nbr = ctx->spai_nbr;
    g.spai_blocks = ctx->spai_blocks;
    g.spai_k = ctx->spai_k;
    if (ctx->gmres_matvec32) {
        // FP32 copy of A for the Arnoldi products (half the bytes per
        // iteration); every restart's residual b - A x stays FP64
        const int64_t ld32 = (n + 31) / 32 * 32;
        void* a32;
        if (int r = ensure(ctx, S_A32MV, (size_t)ld32 * n * sizeof(float), &a32)) return r;
        CK(krylov_cast_f32(ctx->stream, A, lda, n, (float*)a32, ld32, &ctx->launches));
        g.A32mv = (const float*)a32;
        g.ld32 = ld32;
    }
    if (ctx->tuner.mode != TUNE_OFF && n > 0 && n <= INT32_MAX) {
        // column chunks of the Arnoldi product (y = A b into the work vector)
        char key[64];
        std::snprintf(key, sizeof key, "gemv_%s_n%lld", g.A32mv ? "f32" : "f64", (long long)tune_class(n));
        const KrylovWork kw = krylov_carve(g.kwork, n);
        g.gemv_chunks = tune_choice(ctx->tuner, key, ctx->stream, {8, 16, 32}, kGemvChunks, [&](int c) {
            return g.A32mv ? krylov_gemv<float>(ctx->stream, g.A32mv, g.ld32, (int)n, B, 1.0, nullptr, g.w, kw,
                                                nullptr, 0, 0, &ctx->launches, c)
                           : krylov_gemv<double>(ctx->stream, A, lda, (int)n, B, 1.0, nullptr, g.w, kw, nullptr, 0,
                                                 0, &ctx->launches, c);
        });
    }
    ctx->last_iters = 0;
    ctx->last_relres = 0.0;
    bool converged = true;
    for (int64_t c = 0; c < nrhs; ++c) {
        g.b = B + c * ldb;
        g.x = (double*)work;
        GmresResult res{};
        const int st = gmres_ir_solve(g, &res);
        if (st == GMRES_CUDA_ERROR || st == GMRES_TIMEOUT)
            return fail(ctx, CAD_ERR_CUDA, "preconditioned GMRES: CUDA error");
        converged = converged && st == GMRES_OK;
        ctx->last_iters += res.iterations;
        ctx->last_relres = res.rel_residual > ctx->last_relres ? res.rel_residual : ctx->last_relres;
        CK(cudaMemcpyAsync(B + c * ldb, work, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    ctx->timed[1] = true;
    if (!converged)
        return fail(ctx, CAD_ERR_NOT_CONVERGED, "preconditioned GMRES did not reach the residual tolerance");
    return CAD_OK;
}

int solve_device(cad_ctx* ctx, int64_t n, double* A, int64_t lda, double* B, int64_t ldb, int64_t nrhs)
{
    if (n == 0 || nrhs == 0) return CAD_OK;
    if (ctx->solver == CAD_SOLVER_GMRES_SPAI || ctx->solver == CAD_SOLVER_GMRES_LEARNED ||
        ctx->solver == CAD_SOLVER_GMRES_BLOCK_JACOBI || ctx->solver == CAD_SOLVER_GMRES) {
        if (n > INT32_MAX || lda > INT32_MAX || ldb > INT32_MAX || nrhs > INT32_MAX)
            return fail(ctx, CAD_ERR_ARG, "matrix dimension exceeds 2^31-1");
        if (ctx->solver == CAD_SOLVER_GMRES_BLOCK_JACOBI || ctx->solver == CAD_SOLVER_GMRES) {
            // the element-diagonal preconditioner of this A (or identity blocks)
            if (n % 3 != 0) return fail(ctx, CAD_ERR_ARG, "system size is not 3N");
            const int64_t N = n / 3;
            void *nbr, *blk;
            if (int r = ensure(ctx, S_BJ_NBR, (size_t)N * sizeof(int), &nbr)) return r;
            if (int r = ensure(ctx, S_BJ_BLK, (size_t)N * 9 * sizeof(float), &blk)) return r;
            ++ctx->launches;
            if (ctx->solver == CAD_SOLVER_GMRES_BLOCK_JACOBI)
                CK(block_jacobi(ctx->stream, A, lda, N, (int*)nbr, (float*)blk));
            else
                CK(lpc_identity_blocks(ctx->stream, N, (int*)nbr, (float*)blk, nullptr));
            const int* keep_nbr = ctx->spai_nbr;
            const float* keep_blk = ctx->spai_blocks;
            const int64_t keep_N = ctx->spai_N;
            const int keep_k = ctx->spai_k;
            ctx->spai_nbr = (const int*)nbr;
            ctx->spai_blocks = (const float*)blk;
            ctx->spai_N = N;
            ctx->spai_k = 1;
            const int r = solve_spai_device(ctx, n, A, lda, B, ldb, nrhs);
            ctx->spai_nbr = keep_nbr;
            ctx->spai_blocks = keep_blk;
            ctx->spai_N = keep_N;
            ctx->spai_k = keep_k;
            return r;
        }
        return solve_spai_device(ctx, n, A, lda, B, ldb, nrhs);
    }
    if (ctx->solver == CAD_SOLVER_MIXED) {
        if (n > INT32_MAX || lda > INT32_MAX || ldb > INT32_MAX || nrhs > INT32_MAX)
            return fail(ctx, CAD_ERR_ARG, "matrix dimension exceeds 2^31-1");
        int info = 0;
        return solve_mixed_device(ctx, n, A, lda, B, ldb, nrhs, &info);
    }
    if (n > INT32_MAX || lda > INT32_MAX || ldb > INT32_MAX || nrhs > INT32_MAX)
        return fail(ctx, CAD_ERR_ARG, "matrix dimension exceeds 2^31-1");
    void *work, *piv, *info, *perm;
    if (int r = ensure(ctx, S_WORK, (size_t)n * nrhs * sizeof(double), &work)) return r;
    if (int r = ensure(ctx, S_PIV, (size_t)n * sizeof(int), &piv)) return r;
    if (int r = ensure(ctx, S_PERM, (size_t)n * sizeof(int), &perm)) return r;
    if (int r = ensure(ctx, S_INFO, sizeof(int), &info)) return r;
    CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    ctx->timed[1] = ctx->timed[2] = false;
    LuStreams ls{ctx->stream, ctx->side_stream, &ctx->launches,
                 ctx->graphs, ctx->wait_limit};
    if (ctx->tuner.mode != TUNE_OFF) {
        // leaf width of the panel factorisation (rows per leaf thread), timed
        // on a scratch copy of A for systems up to 12288 unknowns
        char key[64];
        std::snprintf(key, sizeof key, "lu_leaf_f64_n%lld", (long long)tune_class(n));
        if (ctx->tuner.find(key) >= 0 || (ctx->tuner.mode == TUNE_ON && n <= 12288)) {
            void* scratch = nullptr;
            if (ctx->tuner.find(key) < 0)
                if (int r = ensure(ctx, S_TUNE, (size_t)n * n * sizeof(double), &scratch)) return r;
            LuStreams lt = ls;
            lt.graphs = nullptr;
            ls.min_leaf_rpt = tune_choice(ctx->tuner, key, ctx->stream, {1, 2, 4}, 1, [&](int c) {
                cudaError_t e = cudaMemcpy2DAsync(scratch, n * sizeof(double), A, lda * sizeof(double),
                                                  n * sizeof(double), n, cudaMemcpyDeviceToDevice, ctx->stream);
                if (e != cudaSuccess) return e;
                lt.min_leaf_rpt = c;
                return lu_factor_solve<double>(lt, (double*)scratch, n, n, nullptr, 0, 0, nullptr, 0, (int*)piv,
                                               (int*)perm, (int*)info, lu_nb(ctx, false), true, false) == LU_OK
                           ? cudaSuccess
                           : cudaErrorUnknown;
            });
        }
    }
    if (nrhs == 1) {   // one right-hand side: factorise, then the two chain launches
        void* chain;
        if (int r = ensure(ctx, S_CHAIN, (size_t)n * sizeof(double) + lu_chain_sync_ints(n) * sizeof(int), &chain))
            return r;
        int rc = lu_factor_solve<double>(ls, A, n, lda, nullptr, 0, 0, nullptr, 0, (int*)piv, (int*)perm, (int*)info,
                                         lu_nb(ctx, false), true, false);
        if (rc == LU_OK) rc = lu_pivots_to_perm(ls, (const int*)piv, n, (int*)perm);
        if (rc == LU_TOO_LARGE) return fail(ctx, CAD_ERR_ARG, "matrix too large for the dense LU");
        if (rc != LU_OK) return fail(ctx, CAD_ERR_CUDA, "dense LU failed (CUDA error)");
        double* y = (double*)chain;
        CK(lu_solve_chain_f64(ctx->stream, A, lda, n, (const int*)perm, B, y, (double*)work, (int*)(y + n),
                              (int*)info, &ctx->launches, ctx->wait_limit));
        CK(cudaMemcpyAsync(B, work, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaEventRecord(ctx->ev[3], ctx->stream));
        ctx->timed[1] = true;
        return CAD_OK;
    }
    const int rc = lu_factor_solve<double>(ls, A, n, lda, B, ldb, (int)nrhs, (double*)work, n, (int*)piv, (int*)perm,
                                           (int*)info, lu_nb(ctx, false), true, true);
    if (rc == LU_TOO_LARGE) return fail(ctx, CAD_ERR_ARG, "matrix too large for the dense LU");
    if (rc != LU_OK) return fail(ctx, CAD_ERR_CUDA, "dense LU failed (CUDA error)");
    CK(cudaMemcpy2DAsync(B, ldb * sizeof(double), work, n * sizeof(double), n * sizeof(double), nrhs,
                         cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    ctx->timed[1] = true;
    return CAD_OK;
}

// info of the last factorisation: 0 when every pivot was non-zero (and when
// the solver factorises nothing)
int read_info(cad_ctx* ctx, int* info)
{
    *info = 0;
    if (ctx->solver == CAD_SOLVER_GMRES_SPAI || !ctx->buf[S_INFO].p) return CAD_OK;
    int h = 0;
    CK(cudaMemcpyAsync(&h, ctx->buf[S_INFO].p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    // negative: a leaf of the factorisation gave up waiting on a pivot exchange
    if (h < 0) return fail(ctx, CAD_ERR_TIMEOUT, "LU factorisation: a pivot exchange wait ran out");
    *info = (h == INT32_MAX) ? 0 : h;
    return CAD_OK;
}

int copy_fields_out(cad_ctx* ctx, const double* dev, int nfield, int64_t count, double* const* host)
{
    for (int f = 0; f < nfield; ++f)
        if (host[f])
            CK(cudaMemcpyAsync(host[f], dev + f * count, count * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    return CAD_OK;
}

int upload(cad_ctx* ctx, double* dst, const double* src, int64_t count)
{
    if (count > 0) CK(cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    return CAD_OK;
}

bool bad_flag(int f) { return f != 0 && f != 1; }

}  // namespace


// ------------------------------------------------------------- batched solve
int lane_ensure(cad_ctx* ctx, Lane& l, LaneSlot slot, size_t bytes, void** out)
{
    DevBuf& b = l.buf[slot];
    if (bytes == 0) bytes = 16;
    if (b.bytes < bytes) {
        if (b.p) {
            CK(cudaStreamSynchronize(l.main));
            CK(cudaStreamSynchronize(l.side));
            CK(cudaFree(b.p));
            b.p = nullptr;
            b.bytes = 0;
        }
        CK(cudaMalloc(&b.p, bytes));
        b.bytes = bytes;
    }
    *out = b.p;
    return CAD_OK;
}

int make_lanes(cad_ctx* ctx)
{
    if (!ctx->lanes.empty()) return CAD_OK;
    int prio_low = 0, prio_high = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    ctx->lanes.resize(kLanes);
    for (auto& l : ctx->lanes) {
        CK(cudaStreamCreateWithPriority(&l.main, cudaStreamNonBlocking, prio_high));
        CK(cudaStreamCreateWithPriority(&l.side, cudaStreamNonBlocking, prio_low));
        CK(cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming));
    }
    return CAD_OK;
}

// One crack's system matrix on the lane's main stream with the lane's buffers.
cudaError_t assemble_on_lane(Lane& l, int64_t* launches, const double* normals, const double* mid, const double* P1,
                             const double* P2, const double* P3, int64_t N, double nu, double G, double lambda,
                             int hs, bool mixed, double near_factor, double* A, int64_t lda)
{
    double* X = (double*)l.buf[L_OBS].p;
    cudaError_t e = launch_colloc(normals, mid, N, X, X + N, X + 2 * N, (double*)l.buf[L_DIRS].p, l.main);
    if (e != cudaSuccess) return e;
    e = launch_td_setup(P1, P2, P3, N, nullptr, nullptr, nullptr, 1, nu, hs == 1, (TriDev*)l.buf[L_TRI].p, l.main);
    if (e != cudaSuccess) return e;
    *launches += 2;
    PairArgs a{};
    a.X = X; a.Y = X + N; a.Z = X + 2 * N; a.M = N; a.tri = (const TriDev*)l.buf[L_TRI].p; a.N = N;
    a.tri_chunk = pick_chunk(N, N, false);
    a.lambda = lambda; a.G = G; a.dirs = (const double*)l.buf[L_DIRS].p;
    a.A = A; a.lda = lda;
    if (mixed)
        return launch_assemble_mixed(a, hs == 1, P1, P2, P3, near_factor, l.buf[L_TRI32].p, (double*)l.buf[L_NEAR].p,
                                     l.main, launches);
    ++*launches;
    return launch_td_pairs(a, OUT_AMAT, hs == 1, true, false, l.main);
}

struct BatchArgs {
    int64_t nbatch;
    const int64_t* offsets;
    const double *P1, *P2, *P3, *normals, *midpoints, *T;
    double* D;
    double nu, G, lambda;
    int hs;
    double* Aall;                   // every crack's 3N x 3N matrix, back to back
    const std::vector<int64_t>* aoff;
    const std::vector<int>* lane_of;
    const std::vector<int64_t>* order;   // issue order
    double* rel;                    // device, nbatch
    // grouped solve (when set): every crack's records, FP32 systems, tensor
    // maps, info words and the GEMM status word, sync words
    const std::vector<CrackRec>* crecs = nullptr;
    const std::vector<GroupSystem>* gsys = nullptr;
    const CUtensorMap* maps = nullptr;
    int* ginfo = nullptr;
    int* gstatus = nullptr;
    int* gsync = nullptr;
    size_t gsync_ints = 0;
};

// Issues the whole batch: fork the lanes off the context stream, every
// crack's assembly on its lane -- with the lanes path also its FP32 LU and
// fixed refinement sweeps -- join; with the grouped path then every crack's
// cast, FP32 LU and sweeps in grouped launches on the context stream.
int batch_body(cad_ctx* ctx, const BatchArgs& b, cudaEvent_t fork)
{
    CK(cudaEventRecord(fork, ctx->stream));
    for (auto& l : ctx->lanes) {
        CK(cudaStreamWaitEvent(l.main, fork, 0));
        CK(cudaStreamWaitEvent(l.side, fork, 0));
    }
    const bool mixed = ctx->assembly == CAD_ASSEMBLY_MIXED;
    for (int64_t c : *b.order) {
        Lane& l = ctx->lanes[(*b.lane_of)[c]];
        const int64_t o = b.offsets[c], N = b.offsets[c + 1] - o, n3 = 3 * N;
        if (N == 0) continue;
        double* A = b.Aall + (*b.aoff)[c];
        CK(assemble_on_lane(l, &ctx->launches, b.normals + 3 * o, b.midpoints + 3 * o, b.P1 + 3 * o, b.P2 + 3 * o,
                            b.P3 + 3 * o, N, b.nu, b.G, b.lambda, b.hs, mixed, ctx->near_factor, A, n3));
        if (b.crecs) continue;
        const LuStreams ls{l.main, l.side, &ctx->launches, nullptr, ctx->wait_limit};
        const bool chain = ctx->batch_mode == CAD_BATCH_LANES_CHAIN;
        int rc = mixed_prepare(ls, A, n3, n3, (float*)l.buf[L_A32].p, (float*)l.buf[L_DINV].p,
                               (int*)l.buf[L_PIV].p, (int*)l.buf[L_PERM].p, (int*)l.buf[L_INFO].p, kLuBlock, chain);
        if (rc != LU_OK) return fail(ctx, CAD_ERR_CUDA, "batched solve: FP32 LU failed");
        float* r32 = (float*)l.buf[L_IR32].p;
        IrArgs ia{ls, n3, A, n3, b.T + 3 * o, n3, 1, b.D + 3 * o, (float*)l.buf[L_A32].p, (int*)l.buf[L_PIV].p,
                  (int*)l.buf[L_PERM].p, (int*)l.buf[L_INFO].p, kLuBlock, ctx->tol, kBatchSweeps,
                  (double*)l.buf[L_IR].p, r32, r32 + n3, (double*)l.buf[L_NORMS].p,
                  (double*)l.buf[L_KWORK].p, chain ? (const float*)l.buf[L_DINV].p : nullptr,
                  chain ? (int*)l.buf[L_SYNC].p : nullptr, chain ? (double*)l.buf[L_Z].p : nullptr, ctx->wait_limit};
        if (ir_solve_fixed(ia, kBatchSweeps, b.rel + c) != GMRES_OK)
            return fail(ctx, CAD_ERR_CUDA, "batched solve: refinement launch failed");
    }
    for (auto& l : ctx->lanes) {
        CK(cudaEventRecord(l.done, l.main));
        CK(cudaStreamWaitEvent(ctx->stream, l.done, 0));
    }
    if (b.crecs) {
        CK(cudaMemsetAsync(b.gstatus, 0, sizeof(int), ctx->stream));
        LuStreams ls{ctx->stream, ctx->side_stream, &ctx->launches, nullptr, ctx->wait_limit};
        ls.aux = ctx->leaf_aux;
        ls.naux = kLeafAux;
        if (mixed_group_solve(ls, *b.crecs, *b.gsys, b.maps, b.ginfo, b.gstatus, b.gsync, b.gsync_ints, kBatchSweeps,
                              kGroupBlock) != GMRES_OK)
            return fail(ctx, CAD_ERR_CUDA, "batched solve: grouped launch failed");
    }
    return CAD_OK;
}

int slip_batched(cad_ctx* ctx, int64_t nbatch, const int64_t* offsets, const double* P1, const double* P2,
                 const double* P3, const double* normals, const double* midpoints, double nu, double G, double lambda,
                 int hs, const double* T, double* D, double* rel_host)
{
    if (nbatch == 0) return CAD_OK;
    if (hs == 1) {   // every crack's vertices and collocation points at or below z = 0
        void* flag;
        if (int r = ensure(ctx, S_FLAG, sizeof(int), &flag)) return r;
        CK(cudaMemsetAsync(flag, 0, sizeof(int), ctx->stream));
        for (int64_t c = 0; c < nbatch; ++c) {
            const int64_t o = offsets[c], N = offsets[c + 1] - o;
            CK(launch_hs_check(midpoints + 3 * o + 2 * N, N, P1 + 3 * o, P2 + 3 * o, P3 + 3 * o, N, (int*)flag,
                               ctx->stream, normals + 3 * o + 2 * N, false));
        }
        ctx->launches += nbatch;
        int h = 0;
        CK(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (h) return fail(ctx, CAD_ERR_HS_ABOVE_SURFACE, "Half-space solution: Z coordinates must be negative!");
    }
    // sizes, matrix offsets, lanes (largest cracks first, each to the least
    // loaded lane), issue order (round robin over lanes)
    std::vector<int64_t> aoff((size_t)nbatch + 1, 0), byN((size_t)nbatch);
    int64_t maxN = 0;
    for (int64_t c = 0; c < nbatch; ++c) {
        const int64_t N = offsets[c + 1] - offsets[c];
        aoff[c + 1] = aoff[c] + 9 * N * N;
        maxN = N > maxN ? N : maxN;
        byN[c] = c;
    }
    std::sort(byN.begin(), byN.end(), [&](int64_t x, int64_t y) {
        return offsets[x + 1] - offsets[x] > offsets[y + 1] - offsets[y];
    });
    if (int r = make_lanes(ctx)) return r;
    std::vector<int> lane_of((size_t)nbatch, 0);
    std::vector<double> load(kLanes, 0.0);
    std::vector<std::vector<int64_t>> per_lane(kLanes);
    std::vector<int64_t> laneN(kLanes, 0);
    for (int64_t c : byN) {
        int best = 0;
        for (int k = 1; k < kLanes; ++k)
            if (load[k] < load[best]) best = k;
        const double N = (double)(offsets[c + 1] - offsets[c]);
        load[best] += N * N * N;
        lane_of[c] = best;
        per_lane[best].push_back(c);
        laneN[best] = std::max<int64_t>(laneN[best], offsets[c + 1] - offsets[c]);
    }
    std::vector<int64_t> order;
    for (size_t i = 0;; ++i) {
        bool any = false;
        for (int k = 0; k < kLanes; ++k)
            if (i < per_lane[k].size()) {
                order.push_back(per_lane[k][i]);
                any = true;
            }
        if (!any) break;
    }
    // the grouped path takes every crack when the largest fits one leaf cluster
    const int64_t pad_max = (3 * maxN + kGroupBlock - 1) / kGroupBlock * kGroupBlock;
    const bool group = ctx->batch_mode == CAD_BATCH_GROUPED && pad_max <= lu_group_max_rows();
    // workspaces sized before anything is captured
    void *Aall, *rel, *p;
    if (int r = ensure(ctx, S_A, (size_t)aoff[nbatch] * sizeof(double), &Aall)) return r;
    if (int r = ensure(ctx, S_REL, (size_t)nbatch * sizeof(double), &rel)) return r;
    for (int k = 0; k < kLanes; ++k) {
        Lane& l = ctx->lanes[k];
        const size_t N = (size_t)laneN[k], n3 = 3 * N;
        if (N == 0) continue;
        if (int r = lane_ensure(ctx, l, L_OBS, 3 * N * sizeof(double), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_DIRS, 9 * N * sizeof(double), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_TRI, N * tri_record_bytes(), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_TRI32, N * tri_record_bytes_f32(), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_NEAR, (3 * N + 1) * sizeof(double), &p)) return r;
        if (group) continue;   // the lanes only assemble
        if (int r = lane_ensure(ctx, l, L_A32, mixed_ld(n3) * n3 * sizeof(float), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_PIV, n3 * sizeof(int), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_PERM, n3 * sizeof(int), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_INFO, sizeof(int), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_IR, n3 * sizeof(double), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_IR32, 2 * n3 * sizeof(float), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_NORMS, 2 * sizeof(double), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_KWORK, krylov_work_doubles(n3) * sizeof(double), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_DINV, mixed_dinv_floats(n3) * sizeof(float), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_SYNC, mixed_sync_ints(n3) * sizeof(int), &p)) return r;
        if (int r = lane_ensure(ctx, l, L_Z, n3 * sizeof(double), &p)) return r;
    }
    BatchArgs b{nbatch, offsets, P1, P2, P3, normals, midpoints, T, D, nu, G, lambda, hs, (double*)Aall, &aoff,
                &lane_of, &order, (double*)rel};
    std::vector<CrackRec> crecs;
    std::vector<GroupSystem> gsys;
    void* ga32 = nullptr;
    if (group) {
        // group buffers: FP32 systems back to back; ints = [every crack's sync
        // words][info per crack][GEMM status][pivots and permutation per
        // crack]; floats = diagonal-block inverses, y32, x32 per crack;
        // doubles = r, z per crack
        std::vector<size_t> oa((size_t)nbatch), oi((size_t)nbatch), os((size_t)nbatch), of((size_t)nbatch),
            od((size_t)nbatch);
        size_t na = 0, ns = 0, ni = 0, nf = 0, nd = 0;
        for (int64_t c = 0; c < nbatch; ++c) {
            const size_t np = (size_t)((3 * (offsets[c + 1] - offsets[c]) + kGroupBlock - 1) / kGroupBlock) *
                              kGroupBlock;
            oa[c] = na;
            na += np * np;
            os[c] = ns;
            ns += mixed_sync_ints((int64_t)np);
            oi[c] = ni;
            ni += 2 * np;
            of[c] = nf;
            nf += mixed_dinv_floats((int64_t)np) + 2 * np;
            od[c] = nd;
            nd += 2 * np;
        }
        void *gint, *gf32, *gf64, *gmaps;
        if (int r = ensure(ctx, S_G_A32, na * sizeof(float) + 16, &ga32)) return r;
        if (int r = ensure(ctx, S_G_INT, (ns + (size_t)nbatch + 1 + ni) * sizeof(int), &gint)) return r;
        if (int r = ensure(ctx, S_G_F32, nf * sizeof(float) + 16, &gf32)) return r;
        if (int r = ensure(ctx, S_G_F64, nd * sizeof(double) + 16, &gf64)) return r;
        if (int r = ensure(ctx, S_G_MAPS, (size_t)nbatch * 2 * sizeof(CUtensorMap), &gmaps)) return r;
        int* sync_all = (int*)gint;
        int* infos = sync_all + ns;
        int* status = infos + nbatch;
        int* piv_all = status + 1;
        ctx->gmaps_host.assign((size_t)nbatch * 2, CUtensorMap{});
        for (int64_t c = 0; c < nbatch; ++c) {
            const int64_t o = offsets[c], n3 = 3 * (offsets[c + 1] - o);
            const int np = (int)((n3 + kGroupBlock - 1) / kGroupBlock * kGroupBlock);
            float* A32 = (float*)ga32 + oa[c];
            float* f = (float*)gf32 + of[c];
            double* d = (double*)gf64 + od[c];
            int* ip = piv_all + oi[c];
            if (!gemm_group_maps(&ctx->gmaps_host[2 * c], A32, np, np, np))
                return fail(ctx, CAD_ERR_CUDA, "batched solve: tensor map encoding failed");
            gsys.push_back(GroupSystem{A32, np, np, ip, infos + c, (int)c});
            crecs.push_back(CrackRec{(double*)Aall + aoff[c], T + 3 * o, D + 3 * o, A32, f, ip + np, sync_all + os[c],
                                     d, d + np, f + mixed_dinv_floats(np), f + mixed_dinv_floats(np) + np,
                                     (double*)rel + c, (int)n3, (int)n3, np, 0});
        }
        CK(cudaMemcpyAsync(gmaps, ctx->gmaps_host.data(), ctx->gmaps_host.size() * sizeof(CUtensorMap),
                           cudaMemcpyHostToDevice, ctx->stream));
        b.crecs = &crecs;
        b.gsys = &gsys;
        b.maps = (const CUtensorMap*)gmaps;
        b.ginfo = infos;
        b.gstatus = status;
        b.gsync = sync_all;
        b.gsync_ints = ns;
    }
    // the captured graph of an identical earlier call is replayed
    BatchGraph& g = ctx->batch;
    const void* ptrs[9] = {P1, P2, P3, normals, midpoints, T, D, Aall, ga32};
    const double params[5] = {nu, G, lambda, ctx->tol, ctx->near_factor};
    const int flags[3] = {hs, ctx->assembly, ctx->batch_mode};
    const bool same = g.exec && g.offsets.size() == (size_t)nbatch + 1 &&
                      std::equal(g.offsets.begin(), g.offsets.end(), offsets) &&
                      std::equal(ptrs, ptrs + 9, g.ptrs) && std::equal(params, params + 5, g.params) &&
                      std::equal(flags, flags + 3, g.flags);
    cudaEvent_t fork = nullptr;
    CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    int rc = CAD_OK;
    if (same) {
        CK(cudaGraphLaunch(g.exec, ctx->stream));
        ctx->launches += g.launches;
    } else if (ctx->stream == nullptr) {   // the legacy default stream cannot be captured: run directly
        rc = batch_body(ctx, b, fork);
    } else {
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
        const int64_t l0 = ctx->launches;
        cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed);
        if (e != cudaSuccess) {
            cudaEventDestroy(fork);
            return cuda_fail(ctx, e, "batched solve: stream capture");
        }
        rc = batch_body(ctx, b, fork);
        cudaGraph_t graph = nullptr;
        e = cudaStreamEndCapture(ctx->stream, &graph);
        if (rc == CAD_OK && e != cudaSuccess) rc = cuda_fail(ctx, e, "batched solve: stream capture");
        if (rc == CAD_OK) {
            e = cudaGraphInstantiate(&g.exec, graph, cudaGraphInstantiateFlagUseNodePriority);
            if (e != cudaSuccess) rc = cuda_fail(ctx, e, "batched solve: graph instantiation");
        }
        if (graph) cudaGraphDestroy(graph);
        if (rc == CAD_OK) {
            g.offsets.assign(offsets, offsets + nbatch + 1);
            std::copy(ptrs, ptrs + 9, g.ptrs);
            std::copy(params, params + 5, g.params);
            std::copy(flags, flags + 3, g.flags);
            g.launches = ctx->launches - l0;
            e = cudaGraphLaunch(g.exec, ctx->stream);
            if (e != cudaSuccess) rc = cuda_fail(ctx, e, "batched solve: graph launch");
        } else if (g.exec) {
            cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
    }
    cudaEventDestroy(fork);
    if (rc != CAD_OK) return rc;
    // every crack's residual; GMRES (on the context stream) for any crack the
    // refinement sweeps left above the tolerance
    std::vector<double> hrel((size_t)nbatch);
    std::vector<int> hinfo(group ? (size_t)nbatch + 1 : 0);
    CK(cudaMemcpyAsync(hrel.data(), rel, (size_t)nbatch * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (group)
        CK(cudaMemcpyAsync(hinfo.data(), b.ginfo, hinfo.size() * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    for (int v : hinfo)   // a leaf, chain or tensor-core pipeline wait that ran out
        if (v < 0) return fail(ctx, CAD_ERR_TIMEOUT, "batched solve: a device wait ran out");
    if (group) {
        // cracks the graph's sweeps left above the tolerance: more grouped
        // sweeps on their factors, two at a time
        for (int round = 0; round < kGroupExtraRounds; ++round) {
            std::vector<CrackRec> left;
            for (int64_t c = 0; c < nbatch; ++c)
                if (!(hrel[c] <= ctx->tol) && std::isfinite(hrel[c])) left.push_back(crecs[c]);
            if (left.empty()) break;
            const LuStreams ls{ctx->stream, ctx->side_stream, &ctx->launches, nullptr, ctx->wait_limit};
            if (mixed_group_sweeps(ls, left, b.gsync, b.gsync_ints, 2) != GMRES_OK)
                return fail(ctx, CAD_ERR_CUDA, "batched solve: grouped launch failed");
            CK(cudaMemcpyAsync(hrel.data(), rel, (size_t)nbatch * sizeof(double), cudaMemcpyDeviceToHost,
                               ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
        }
    }
    bool converged = true;
    for (int64_t c = 0; c < nbatch; ++c) {
        if (hrel[c] <= ctx->tol) continue;
        const int64_t o = offsets[c], n3 = 3 * (offsets[c + 1] - o);
        CK(cudaMemcpyAsync(D + 3 * o, T + 3 * o, n3 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        int info = 0;
        const int r = solve_mixed_device(ctx, n3, (double*)Aall + aoff[c], n3, D + 3 * o, n3, 1, &info);
        if (r == CAD_ERR_NOT_CONVERGED) converged = false;
        else if (r != CAD_OK) return r;
        if (info > 0) return fail(ctx, CAD_ERR_SINGULAR, "matrix is singular to working precision");
        hrel[c] = ctx->last_relres;
    }
    if (rel_host) std::copy(hrel.begin(), hrel.end(), rel_host);
    if (!converged) return fail(ctx, CAD_ERR_NOT_CONVERGED, "batched solve: a crack did not reach the tolerance");
    return CAD_OK;
}

extern "C" {

const char* cad_version(void) { return "cad_td 1.0 (sm_100a, FP64)"; }

int cad_init(int device, cad_ctx** out)
{
    if (!out) return CAD_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return CAD_ERR_CUDA;
    cad_ctx* ctx = new cad_ctx();
    ctx->device = device;
    // the context stream carries the LU's latency-bound panel chain: highest
    // priority, so its small launches get SMs ahead of the side stream's
    // trailing-update GEMMs (lowest priority)
    int prio_low = 0, prio_high = 0;
    if (cudaSetDevice(device) != cudaSuccess || cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high) != cudaSuccess ||
        cudaStreamCreateWithPriority(&ctx->own_stream, cudaStreamNonBlocking, prio_high) != cudaSuccess) {
        delete ctx;
        return CAD_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    for (auto& e : ctx->ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            cad_destroy(ctx);
            return CAD_ERR_CUDA;
        }
    if (cudaStreamCreateWithPriority(&ctx->side_stream, cudaStreamNonBlocking, prio_low) != cudaSuccess) {
        cad_destroy(ctx);
        return CAD_ERR_CUDA;
    }
    for (auto& a : ctx->leaf_aux)
        if (cudaStreamCreateWithPriority(&a, cudaStreamNonBlocking, prio_high) != cudaSuccess) {
            cad_destroy(ctx);
            return CAD_ERR_CUDA;
        }
    if (cudaEventCreateWithFlags(&ctx->side_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->side_join, cudaEventDisableTiming) != cudaSuccess) {
        cad_destroy(ctx);
        return CAD_ERR_CUDA;
    }
    ctx->graphs = lu_graph_cache_create();
    *out = ctx;
    return CAD_OK;
}

int cad_destroy(cad_ctx* ctx)
{
    if (!ctx) return CAD_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& b : ctx->buf)
        if (b.p) cudaFree(b.p);
    if (ctx->lpc_X) cudaFree(ctx->lpc_X);
    if (ctx->lpc_T) cudaFree(ctx->lpc_T);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->side_stream) cudaStreamSynchronize(ctx->side_stream);
    lu_graph_cache_destroy(ctx->graphs);
    if (ctx->batch.exec) cudaGraphExecDestroy(ctx->batch.exec);
    for (auto& l : ctx->lanes) {
        if (l.main) cudaStreamSynchronize(l.main);
        if (l.side) cudaStreamSynchronize(l.side);
        for (auto& b : l.buf)
            if (b.p) cudaFree(b.p);
        if (l.main) cudaStreamDestroy(l.main);
        if (l.side) cudaStreamDestroy(l.side);
        if (l.done) cudaEventDestroy(l.done);
    }
    if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
    for (auto a : ctx->leaf_aux)
        if (a) cudaStreamDestroy(a);
    if (ctx->side_fork) cudaEventDestroy(ctx->side_fork);
    if (ctx->side_join) cudaEventDestroy(ctx->side_join);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return CAD_OK;
}

const char* cad_last_error(const cad_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int64_t cad_kernel_launches(const cad_ctx* ctx) { return ctx ? ctx->launches : 0; }

int cad_set_assembly(cad_ctx* ctx, int mode, double near_factor)
{
    if (!ctx) return CAD_ERR_ARG;
    if ((mode != CAD_ASSEMBLY_FP64 && mode != CAD_ASSEMBLY_MIXED) || !(near_factor >= 0.0))
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->assembly = mode;
    ctx->near_factor = near_factor;
    return CAD_OK;
}

int cad_set_solver(cad_ctx* ctx, int mode, double tol, int max_iter)
{
    if (!ctx) return CAD_ERR_ARG;
    if (mode < CAD_SOLVER_LU64 || mode > CAD_SOLVER_GMRES || !(tol > 0.0) || max_iter < 1)
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->solver = mode;
    ctx->tol = tol;
    ctx->max_iter = max_iter;
    return CAD_OK;
}

int cad_set_autotune(cad_ctx* ctx, int mode, const char* cache_path)
{
    if (!ctx) return CAD_ERR_ARG;
    if (mode < TUNE_OFF || mode > TUNE_CACHED) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->tuner.mode = mode;
    ctx->tuner.load(cache_path ? std::string(cache_path) : std::string());
    return CAD_OK;
}

int64_t cad_autotune_entries(const cad_ctx* ctx, int64_t* tuned_here)
{
    if (!ctx) return 0;
    if (tuned_here) *tuned_here = ctx->tuner.tuned;
    return (int64_t)ctx->tuner.table.size();
}

int cad_set_gmres_matvec(cad_ctx* ctx, int fp32)
{
    if (!ctx) return CAD_ERR_ARG;
    if (fp32 != 0 && fp32 != 1) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->gmres_matvec32 = fp32;
    return CAD_OK;
}

int cad_set_gmres_restart(cad_ctx* ctx, int m)
{
    if (!ctx) return CAD_ERR_ARG;
    if (m != 0 && (m < 1 || m + 1 > kMaxBasis)) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->gmres_restart = m == 0 ? kGmresRestart : m;
    return CAD_OK;
}

int cad_set_shared_edges(cad_ctx* ctx, int enable)
{
    if (!ctx) return CAD_ERR_ARG;
    if (enable != 0 && enable != 1) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->shared_edges = enable;
    return CAD_OK;
}

int cad_set_lu_block(cad_ctx* ctx, int nb)
{
    if (!ctx) return CAD_ERR_ARG;
    if (nb != 0 && (nb < 32 || nb > 1024)) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->lu_block = nb;
    return CAD_OK;
}

int cad_set_batch_solve(cad_ctx* ctx, int mode)
{
    if (!ctx) return CAD_ERR_ARG;
    if (mode != CAD_BATCH_GROUPED && mode != CAD_BATCH_LANES && mode != CAD_BATCH_LANES_CHAIN)
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->batch_mode = mode;
    return CAD_OK;
}

int cad_set_wait_limit(cad_ctx* ctx, int64_t polls)
{
    if (!ctx) return CAD_ERR_ARG;
    if (polls < 1) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->wait_limit = (long)polls;
    return CAD_OK;
}

int cad_wait_timeout_probe(cad_ctx* ctx, int64_t n)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (n < 128 || n > 8192) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    void *a, *vec, *perm, *chain, *info;
    if (int r = ensure(ctx, S_WORK, (size_t)n * n * sizeof(double), &a)) return r;
    if (int r = ensure(ctx, S_B, 3 * (size_t)n * sizeof(double), &vec)) return r;
    if (int r = ensure(ctx, S_PERM, (size_t)n * sizeof(int), &perm)) return r;
    if (int r = ensure(ctx, S_CHAIN, lu_chain_sync_ints(n) * sizeof(int), &chain)) return r;
    if (int r = ensure(ctx, S_INFO, sizeof(int), &info)) return r;
    CK(cudaMemsetAsync(a, 0, (size_t)n * n * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(vec, 0, 3 * (size_t)n * sizeof(double), ctx->stream));
    CK(cudaMemsetAsync(perm, 0, (size_t)n * sizeof(int), ctx->stream));
    const int big = INT_MAX;
    CK(cudaMemcpyAsync(info, &big, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    double* v = (double*)vec;
    CK(lu_chain_timeout_probe(ctx->stream, (const double*)a, n, n, (const int*)perm, v, v + n, v + 2 * n, (int*)chain,
                              (int*)info, ctx->wait_limit));
    ctx->launches += 2;
    int h = 0;
    CK(cudaMemcpyAsync(&h, info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h < 0) return fail(ctx, CAD_ERR_TIMEOUT, "a device wait ran out (triangular-solve chain flag)");
    return CAD_OK;
}

int cad_last_solve_stats(const cad_ctx* ctx, int* iterations, double* rel_residual)
{
    if (!ctx) return CAD_ERR_ARG;
    if (iterations) *iterations = ctx->last_iters;
    if (rel_residual) *rel_residual = ctx->last_relres;
    return CAD_OK;
}

int cad_set_stream(cad_ctx* ctx, void* stream)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    ctx->stream = (cudaStream_t)stream;   // NULL is CUDA's default stream, as everywhere in CUDA
    return CAD_OK;
}

void* cad_get_stream(const cad_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

double cad_last_time_ms(const cad_ctx* ctx, int which)
{
    if (!ctx || which < 0 || which > 2 || !ctx->timed[which]) return -1.0;
    static const int from[3] = {0, 2, 2}, to[3] = {1, 3, 4};
    float ms = 0.f;
    if (cudaEventSynchronize(ctx->ev[to[which]]) != cudaSuccess) return -1.0;
    if (cudaEventElapsedTime(&ms, ctx->ev[from[which]], ctx->ev[to[which]]) != cudaSuccess) return -1.0;
    return ms;
}

// ------------------------------------------------------------------- TD
static int td_host(cad_ctx* ctx, bool sum_mode, const double* X, const double* Y, const double* Z, int64_t M,
                   const double* P1, const double* P2, const double* P3, int64_t N, const double* Dss,
                   const double* Dds, const double* Dn, double nu, int disp, int strain, int hs,
                   double* const* strain_out, double* const* disp_out)
{
    if (int r = set_device(ctx)) return r;
    if (M < 0 || N < 0 || bad_flag(disp) || bad_flag(strain) || bad_flag(hs))
        return fail(ctx, CAD_ERR_ARG, "invalid size or flag");
    if ((M > 0 && (!X || !Y || !Z)) || (N > 0 && (!P1 || !P2 || !P3 || !Dss || !Dds || !Dn)))
        return fail(ctx, CAD_ERR_ARG, "null input pointer");
    const int ns = sum_mode ? 6 : 18, nd = sum_mode ? 3 : 9;
    if ((strain == 1 && !strain_out) || (disp == 1 && !disp_out)) return fail(ctx, CAD_ERR_ARG, "null output list");
    void *obs, *geom, *slip, *out;
    if (int r = ensure(ctx, S_OBS, (size_t)3 * M * sizeof(double), &obs)) return r;
    if (int r = ensure(ctx, S_GEOM, (size_t)9 * N * sizeof(double), &geom)) return r;
    if (int r = ensure(ctx, S_SLIP, (size_t)3 * N * sizeof(double), &slip)) return r;
    double* o = (double*)obs;
    double* g = (double*)geom;
    double* s = (double*)slip;
    if (int r = upload(ctx, o, X, M)) return r;
    if (int r = upload(ctx, o + M, Y, M)) return r;
    if (int r = upload(ctx, o + 2 * M, Z, M)) return r;
    if (int r = upload(ctx, g, P1, 3 * N)) return r;
    if (int r = upload(ctx, g + 3 * N, P2, 3 * N)) return r;
    if (int r = upload(ctx, g + 6 * N, P3, 3 * N)) return r;
    if (int r = upload(ctx, s, Dss, N)) return r;
    if (int r = upload(ctx, s + N, Dds, N)) return r;
    if (int r = upload(ctx, s + 2 * N, Dn, N)) return r;
    const int64_t per = sum_mode ? M : M * N;
    const size_t out_words = sum_mode ? (size_t)9 * M : (size_t)((strain == 1 ? ns : 0) + (disp == 1 ? nd : 0)) * per;
    if (int r = ensure(ctx, S_OUT, out_words * sizeof(double), &out)) return r;
    double* ob = (double*)out;
    double* so = ob;
    double* dout = sum_mode ? ob + 6 * M : ob + (strain == 1 ? ns * per : 0);
    int r = td_device(ctx, o, o + M, o + 2 * M, M, g, g + 3 * N, g + 6 * N, N, s, s + N, s + 2 * N, nu, disp, strain,
                      hs, sum_mode ? OUT_SUM : OUT_INF, so, dout, sum_mode ? ob : nullptr);
    if (r) return r;
    if (strain == 1)
        if (int rr = copy_fields_out(ctx, so, ns, per, strain_out)) return rr;
    if (disp == 1)
        if (int rr = copy_fields_out(ctx, dout, nd, per, disp_out)) return rr;
    CK(cudaStreamSynchronize(ctx->stream));
    return CAD_OK;
}

int cad_td_inf(cad_ctx* ctx, const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
               const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds,
               const double* Dn, double nu, double G, int disp_flag, int strain_flag, int hs_flag,
               double* const* strain_out, double* const* disp_out)
{
    CAD_NVTX_RANGE();
    (void)G;
    return td_host(ctx, false, X, Y, Z, M, P1, P2, P3, N, Dss, Dds, Dn, nu, disp_flag, strain_flag, hs_flag,
                   strain_out, disp_out);
}

int cad_td_sum_eval(cad_ctx* ctx, const double* X, const double* Y, const double* Z, int64_t M,
                    const double* P1, const double* P2, const double* P3, int64_t N, const double* Dss,
                    const double* Dds, const double* Dn, double nu, double G, int disp_flag, int strain_flag,
                    int hs_flag, double* const* strain_out, double* const* disp_out)
{
    CAD_NVTX_RANGE();
    (void)G;
    return td_host(ctx, true, X, Y, Z, M, P1, P2, P3, N, Dss, Dds, Dn, nu, disp_flag, strain_flag, hs_flag,
                   strain_out, disp_out);
}

int cad_td_sum(cad_ctx* ctx, int64_t M, int64_t N, const double* const* strain_in, const double* const* disp_in,
               double* const* strain_out, double* const* disp_out)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (M < 0 || N < 0) return fail(ctx, CAD_ERR_ARG, "invalid size");
    const int64_t MN = M * N;
    for (int kind = 0; kind < 2; ++kind) {
        const double* const* in = kind == 0 ? strain_in : disp_in;
        double* const* out = kind == 0 ? strain_out : disp_out;
        if (!in) continue;
        if (!out) return fail(ctx, CAD_ERR_ARG, "null output list");
        const int nf = kind == 0 ? 6 : 3;
        void *dev_in, *dev_out;
        if (int r = ensure(ctx, S_A, (size_t)3 * nf * MN * sizeof(double), &dev_in)) return r;
        if (int r = ensure(ctx, S_OUT, (size_t)nf * M * sizeof(double), &dev_out)) return r;
        for (int f = 0; f < 3 * nf; ++f)
            if (int r = upload(ctx, (double*)dev_in + f * MN, in[f], MN)) return r;
        ++ctx->launches;
    CK(launch_td_sum((const double*)dev_in, M, N, nf, (double*)dev_out, ctx->stream));
        if (int r = copy_fields_out(ctx, (const double*)dev_out, nf, M, out)) return r;
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return CAD_OK;
}

// ------------------------------------------------------------- assembly
static int upload_geometry(cad_ctx* ctx, const double* normals, const double* mid, const double* P1,
                           const double* P2, const double* P3, int64_t N, double** g)
{
    void* geom;
    if (int r = ensure(ctx, S_GEOM, (size_t)15 * N * sizeof(double), &geom)) return r;
    *g = (double*)geom;
    if (int r = upload(ctx, *g, P1, 3 * N)) return r;
    if (int r = upload(ctx, *g + 3 * N, P2, 3 * N)) return r;
    if (int r = upload(ctx, *g + 6 * N, P3, 3 * N)) return r;
    if (int r = upload(ctx, *g + 9 * N, normals, 3 * N)) return r;
    if (int r = upload(ctx, *g + 12 * N, mid, 3 * N)) return r;
    return CAD_OK;
}

// Fixed elements of a FixedEls vector (value 1): row map (fixed row index or
// -1) and the kept columns.
struct FixedSplit {
    std::vector<int> fixrow, freecol, fixidx;
};
static FixedSplit split_fixed(const double* fixed_els, int64_t N)
{
    FixedSplit f;
    f.fixrow.assign((size_t)N, -1);
    for (int64_t i = 0; i < N; ++i) {
        if (fixed_els && fixed_els[i] == 1.0) {
            f.fixrow[i] = (int)f.fixidx.size();
            f.fixidx.push_back((int)i);
        } else {
            f.freecol.push_back((int)i);
        }
    }
    return f;
}

// CalculateInfluenceMatrices3D with fixed elements
// (src/CalculateInfluenceMatrices3D.jl:10-33, :145-199) on the device: the
// traction fields of every pair, the displacement fields at the fixed
// elements' collocation points (unit slips), spliced -- either the nine
// N x nf fields (amat false) or A = -[Atn; Atss; Atds] (3N x 3nf, lda).
static int assemble_fixed_device(cad_ctx* ctx, const double* g, int64_t N, double nu, double G, double lambda, int hs,
                                 const FixedSplit& fs, bool amat, double* out, int64_t lda)
{
    const int64_t nfix = (int64_t)fs.fixidx.size(), nf = (int64_t)fs.freecol.size();
    void *trac, *idx, *fobs, *fdisp;
    if (int r = ensure(ctx, S_OUT, (size_t)9 * N * N * sizeof(double), &trac)) return r;
    if (int r = assemble_device(ctx, g + 9 * N, g + 12 * N, g, g + 3 * N, g + 6 * N, N, nu, G, lambda, hs, OUT_TRAC,
                                (double*)trac, nullptr, 0))
        return r;
    if (int r = ensure(ctx, S_FIX, (size_t)(N + nf + nfix) * sizeof(int), &idx)) return r;
    if (int r = ensure(ctx, S_FOBS, (size_t)3 * nfix * sizeof(double), &fobs)) return r;
    if (int r = ensure(ctx, S_FDISP, (size_t)9 * nfix * N * sizeof(double), &fdisp)) return r;
    int* fixrow = (int*)idx;
    int* freecol = fixrow + N;
    int* fixidx = freecol + nf;
    CK(cudaMemcpyAsync(fixrow, fs.fixrow.data(), N * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    if (nf) CK(cudaMemcpyAsync(freecol, fs.freecol.data(), nf * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    if (nfix) {
        CK(cudaMemcpyAsync(fixidx, fs.fixidx.data(), nfix * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        const double* X = (const double*)ctx->buf[S_OBS].p;   // collocation points of assemble_device
        ++ctx->launches;
        CK(launch_gather_points(X, X + N, X + 2 * N, fixidx, nfix, (double*)fobs, ctx->stream));
        PairArgs a{};
        const double* fo = (const double*)fobs;
        a.X = fo; a.Y = fo + nfix; a.Z = fo + 2 * nfix; a.M = nfix;
        a.tri = (const TriDev*)ctx->buf[S_TRI].p; a.N = N;   // unit-slip records of assemble_device
        a.tri_chunk = pick_chunk(nfix, N, false);
        a.disp = (double*)fdisp;
        ++ctx->launches;
        CK(launch_td_pairs(a, OUT_INF, hs == 1, false, true, ctx->stream));
    }
    ++ctx->launches;
    CK(launch_splice_fixed((const double*)trac, (const double*)fdisp, N, nfix, fixrow, freecol, nf, amat, out, lda,
                           ctx->stream));
    // the host vectors of fs are read by the copies above: finish before they go
    CK(cudaStreamSynchronize(ctx->stream));
    return CAD_OK;
}

int cad_influence_traction(cad_ctx* ctx, const double* normals, const double* midpoints, const double* P1,
                           const double* P2, const double* P3, int64_t N, double nu, double G, double lambda,
                           const double* fixed_els, int hs_flag, double* const* trac_out)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 0 || bad_flag(hs_flag) || !trac_out) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    double* g;
    if (int r = upload_geometry(ctx, normals, midpoints, P1, P2, P3, N, &g)) return r;
    const FixedSplit fs = split_fixed(fixed_els, N);
    if (!fs.fixidx.empty()) {
        const int64_t nf = (int64_t)fs.freecol.size();
        void* out;
        if (int r = ensure(ctx, S_A, (size_t)9 * N * nf * sizeof(double) + 16, &out)) return r;
        if (int r = assemble_fixed_device(ctx, g, N, nu, G, lambda, hs_flag, fs, false, (double*)out, 0)) return r;
        if (int rr = copy_fields_out(ctx, (const double*)out, 9, N * nf, trac_out)) return rr;
        CK(cudaStreamSynchronize(ctx->stream));
        return CAD_OK;
    }
    void* out;
    if (int r = ensure(ctx, S_OUT, (size_t)9 * N * N * sizeof(double), &out)) return r;
    int r = assemble_device(ctx, g + 9 * N, g + 12 * N, g, g + 3 * N, g + 6 * N, N, nu, G, lambda, hs_flag, OUT_TRAC,
                            (double*)out, nullptr, 0);
    if (r) return r;
    if (int rr = copy_fields_out(ctx, (const double*)out, 9, N * N, trac_out)) return rr;
    CK(cudaStreamSynchronize(ctx->stream));
    return CAD_OK;
}

int cad_slip_calculator(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, double nu,
                        double G, double lambda, const double* midpoints, const double* normals, int hs_flag,
                        const double* Tn, const double* Tss, const double* Tds, double* Dn, double* Dss,
                        double* Dds, double* A_out, double* b_out)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 0 || bad_flag(hs_flag) || !Tn || !Tss || !Tds || !Dn || !Dss || !Dds)
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    double* g;
    if (int r = upload_geometry(ctx, normals, midpoints, P1, P2, P3, N, &g)) return r;
    const int64_t n3 = 3 * N;
    void *A, *b;
    if (int r = ensure(ctx, S_A, (size_t)n3 * n3 * sizeof(double), &A)) return r;
    if (int r = ensure(ctx, S_B, (size_t)n3 * sizeof(double), &b)) return r;
    double* bd = (double*)b;
    if (int r = upload(ctx, bd, Tn, N)) return r;
    if (int r = upload(ctx, bd + N, Tss, N)) return r;
    if (int r = upload(ctx, bd + 2 * N, Tds, N)) return r;
    // the learned preconditioner depends on the geometry only: it is built
    // on the side stream while the system matrix is assembled
    const bool learned = ctx->solver == CAD_SOLVER_GMRES_LEARNED && N > 0;
    int r = CAD_OK;
    if (learned) {
        CK(cudaEventRecord(ctx->side_fork, ctx->stream));
        CK(cudaStreamWaitEvent(ctx->side_stream, ctx->side_fork, 0));
        cudaStream_t home = ctx->stream;
        ctx->stream = ctx->side_stream;
        r = cad_lpc_install_dev(ctx, g, g + 3 * N, g + 6 * N, N, G);
        ctx->stream = home;
        if (r) return r;
        CK(cudaEventRecord(ctx->side_join, ctx->side_stream));
    }
    r = assemble_device(ctx, g + 9 * N, g + 12 * N, g, g + 3 * N, g + 6 * N, N, nu, G, lambda, hs_flag, OUT_AMAT,
                        nullptr, (double*)A, n3);
    if (learned) CK(cudaStreamWaitEvent(ctx->stream, ctx->side_join, 0));
    if (r) return r;
    if (A_out) CK(cudaMemcpyAsync(A_out, A, (size_t)n3 * n3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (b_out) CK(cudaMemcpyAsync(b_out, bd, (size_t)n3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if ((r = solve_device(ctx, n3, (double*)A, n3, bd, n3, 1))) return r;
    int info = 0;
    if (n3 > 0)
        if ((r = read_info(ctx, &info))) return r;
    CK(cudaMemcpyAsync(Dn, bd, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(Dss, bd + N, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(Dds, bd + 2 * N, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (info > 0) return fail(ctx, CAD_ERR_SINGULAR, "SingularException: the system matrix is singular");
    return CAD_OK;
}

int cad_solve(cad_ctx* ctx, int64_t n, const double* A, const double* B, int64_t nrhs, double* X)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (n < 0 || nrhs < 0 || (n > 0 && (!A || !B || !X))) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    void *Ad, *Bd;
    if (int r = ensure(ctx, S_A, (size_t)n * n * sizeof(double), &Ad)) return r;
    if (int r = ensure(ctx, S_B, (size_t)n * nrhs * sizeof(double), &Bd)) return r;
    if (int r = upload(ctx, (double*)Ad, A, n * n)) return r;
    if (int r = upload(ctx, (double*)Bd, B, n * nrhs)) return r;
    if (int r = solve_device(ctx, n, (double*)Ad, n, (double*)Bd, n, nrhs)) return r;
    int info = 0;
    if (n > 0 && nrhs > 0) {
        if (int r = read_info(ctx, &info)) return r;
        CK(cudaMemcpyAsync(X, Bd, (size_t)n * nrhs * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    if (info > 0) return fail(ctx, CAD_ERR_SINGULAR, "SingularException: the system matrix is singular");
    return CAD_OK;
}

// ------------------------------------------------------------ device API
int cad_td_inf_dev(cad_ctx* ctx, const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
                   const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds,
                   const double* Dn, double nu, int disp_flag, int strain_flag, int hs_flag, double* strain_out,
                   double* disp_out)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (M < 0 || N < 0 || bad_flag(disp_flag) || bad_flag(strain_flag) || bad_flag(hs_flag))
        return fail(ctx, CAD_ERR_ARG, "invalid size or flag");
    return td_device(ctx, X, Y, Z, M, P1, P2, P3, N, Dss, Dds, Dn, nu, disp_flag, strain_flag, hs_flag, OUT_INF,
                     strain_out, disp_out, nullptr);
}

int cad_td_sum_eval_dev(cad_ctx* ctx, const double* X, const double* Y, const double* Z, int64_t M,
                        const double* P1, const double* P2, const double* P3, int64_t N, const double* Dss,
                        const double* Dds, const double* Dn, double nu, int disp_flag, int strain_flag,
                        int hs_flag, double* strain_out, double* disp_out)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (M < 0 || N < 0 || bad_flag(disp_flag) || bad_flag(strain_flag) || bad_flag(hs_flag))
        return fail(ctx, CAD_ERR_ARG, "invalid size or flag");
    void* out;
    if (int r = ensure(ctx, S_OUT, (size_t)9 * M * sizeof(double), &out)) return r;
    int r = td_device(ctx, X, Y, Z, M, P1, P2, P3, N, Dss, Dds, Dn, nu, disp_flag, strain_flag, hs_flag, OUT_SUM,
                      nullptr, nullptr, (double*)out);
    if (r) return r;
    if (strain_flag == 1 && strain_out)
        CK(cudaMemcpyAsync(strain_out, out, 6 * M * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    if (disp_flag == 1 && disp_out)
        CK(cudaMemcpyAsync(disp_out, (double*)out + 6 * M, 3 * M * sizeof(double), cudaMemcpyDeviceToDevice,
                           ctx->stream));
    return CAD_OK;
}

int cad_assemble_dev(cad_ctx* ctx, const double* normals, const double* midpoints, const double* P1,
                     const double* P2, const double* P3, int64_t N, double nu, double G, double lambda, int hs_flag,
                     double* A, int64_t lda)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 0 || bad_flag(hs_flag) || lda < 3 * N) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    return assemble_device(ctx, normals, midpoints, P1, P2, P3, N, nu, G, lambda, hs_flag, OUT_AMAT, nullptr, A, lda);
}

int cad_assemble_columns_dev(cad_ctx* ctx, const double* normals, const double* midpoints, const double* P1,
                             const double* P2, const double* P3, int64_t N, double nu, double G, double lambda,
                             int hs_flag, int64_t j0, int64_t j1, double* A_block, int64_t lda)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 0 || bad_flag(hs_flag) || j0 < 0 || j1 < j0 || j1 > N || lda < 3 * N || (j1 > j0 && !A_block))
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    const int64_t nb = j1 - j0;
    void *obs, *dirs, *tri;
    if (int r = ensure(ctx, S_OBS, (size_t)3 * N * sizeof(double), &obs)) return r;
    if (int r = ensure(ctx, S_DIRS, (size_t)9 * N * sizeof(double), &dirs)) return r;
    double* X = (double*)obs;
    ++ctx->launches;
    CK(launch_colloc(normals, midpoints, N, X, X + N, X + 2 * N, (double*)dirs, ctx->stream));
    if (hs_flag == 1 && N > 0)
        if (int r = hs_check(ctx, X + 2 * N, N, P1, P2, P3, N)) return r;
    if (nb == 0) return CAD_OK;
    // every triangle record (one thread each, cheap); the pair kernel reads the block's
    if (int r = ensure(ctx, S_TRI, (size_t)N * tri_record_bytes(), &tri)) return r;
    ++ctx->launches;
    CK(launch_td_setup(P1, P2, P3, N, nullptr, nullptr, nullptr, 1, nu, hs_flag == 1, (TriDev*)tri, ctx->stream));
    PairArgs a{};
    a.X = X; a.Y = X + N; a.Z = X + 2 * N; a.M = N;
    a.tri = (const TriDev*)tri + j0; a.N = nb;
    a.tri_chunk = pick_chunk(N, nb, false);
    a.lambda = lambda; a.G = G; a.dirs = (const double*)dirs;
    a.A = A_block; a.lda = lda;
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    ++ctx->launches;
    CK(launch_td_pairs(a, OUT_AMAT, hs_flag == 1, true, false, ctx->stream));
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    ctx->timed[0] = true;
    return CAD_OK;
}

int cad_solve_dev(cad_ctx* ctx, int64_t n, double* A, int64_t lda, double* B, int64_t ldb, int64_t nrhs)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (n < 0 || nrhs < 0 || lda < n || ldb < n) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (int r = solve_device(ctx, n, A, lda, B, ldb, nrhs)) return r;
    int info = 0;
    if (n > 0 && nrhs > 0)
        if (int r = read_info(ctx, &info)) return r;
    if (info > 0) return fail(ctx, CAD_ERR_SINGULAR, "SingularException: the system matrix is singular");
    return CAD_OK;
}

int cad_gemm_sub_dev(cad_ctx* ctx, int precision, int64_t m, int64_t n, int64_t k, const void* A, int64_t lda,
                     const void* B, int64_t ldb, void* C, int64_t ldc)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (m < 0 || n < 0 || k < 0 || m > INT32_MAX || n > INT32_MAX || k > INT32_MAX || lda < (m > 0 ? m : 1) ||
        ldb < (k > 0 ? k : 1) || ldc < (m > 0 ? m : 1) || precision < 0 || precision > 4)
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (m == 0 || n == 0 || k == 0) return CAD_OK;
    void* st;
    if (int r = ensure(ctx, S_GEMM, sizeof(int), &st)) return r;
    CK(cudaMemsetAsync(st, 0, sizeof(int), ctx->stream));
    if (precision != 1) {
        static const int dmma_k[5] = {0, 0, 4, 8, 16};
        CK(gemm_sub(ctx->stream, (int)m, (int)n, (int)k, (const double*)A, lda, (const double*)B, ldb, (double*)C, ldc,
                    (int*)st, dmma_k[precision]));
    } else
        CK(gemm_sub(ctx->stream, (int)m, (int)n, (int)k, (const float*)A, lda, (const float*)B, ldb, (float*)C, ldc,
                    (int*)st));
    ++ctx->launches;
    int h = 0;
    CK(cudaMemcpyAsync(&h, st, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (h < 0) return fail(ctx, CAD_ERR_TIMEOUT, "GEMM: a pipeline wait ran out");
    return CAD_OK;
}

int cad_slip_calculator_batched_dev(cad_ctx* ctx, int64_t nbatch, const int64_t* offsets, const double* P1,
                                    const double* P2, const double* P3, const double* normals,
                                    const double* midpoints, double nu, double G, double lambda, int hs_flag,
                                    const double* T, double* D, double* rel_residual)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (nbatch < 0 || bad_flag(hs_flag) || (nbatch > 0 && !offsets)) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (nbatch > 0 && offsets[0] != 0) return fail(ctx, CAD_ERR_ARG, "offsets[0] must be 0");
    for (int64_t c = 0; c < nbatch; ++c)
        if (offsets[c + 1] < offsets[c]) return fail(ctx, CAD_ERR_DIMS, "Element size inputs must be the same dimensions");
    if (nbatch > 0 && offsets[nbatch] > 0 && (!P1 || !P2 || !P3 || !normals || !midpoints || !T || !D))
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    return slip_batched(ctx, nbatch, offsets, P1, P2, P3, normals, midpoints, nu, G, lambda, hs_flag, T, D,
                        rel_residual);
}

int cad_slip_calculator_batched(cad_ctx* ctx, int64_t nbatch, const int64_t* offsets, const double* P1,
                                const double* P2, const double* P3, const double* normals, const double* midpoints,
                                double nu, double G, double lambda, int hs_flag, const double* T, double* D,
                                double* rel_residual)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (nbatch < 0 || (nbatch > 0 && !offsets)) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    const int64_t ntot = nbatch > 0 ? offsets[nbatch] : 0;
    if (ntot < 0) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (ntot > 0 && (!P1 || !P2 || !P3 || !normals || !midpoints || !T || !D))
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    void *geom, *td;
    if (int r = ensure(ctx, S_BGEOM, (size_t)15 * ntot * sizeof(double), &geom)) return r;
    if (int r = ensure(ctx, S_BTD, (size_t)6 * ntot * sizeof(double), &td)) return r;
    double* g = (double*)geom;
    double* t = (double*)td;
    const double* src[5] = {P1, P2, P3, normals, midpoints};
    for (int k = 0; k < 5; ++k)
        if (int r = upload(ctx, g + k * 3 * ntot, src[k], 3 * ntot)) return r;
    if (int r = upload(ctx, t, T, 3 * ntot)) return r;
    if (int r = cad_slip_calculator_batched_dev(ctx, nbatch, offsets, g, g + 3 * ntot, g + 6 * ntot, g + 9 * ntot,
                                                g + 12 * ntot, nu, G, lambda, hs_flag, t, t + 3 * ntot, rel_residual))
        return r;
    if (ntot > 0) {
        CK(cudaMemcpyAsync(D, t + 3 * ntot, (size_t)3 * ntot * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return CAD_OK;
}

int cad_set_preconditioner(cad_ctx* ctx, int64_t N, int k, const int* nbr, const float* blocks)
{
    if (!ctx) return CAD_ERR_ARG;
    if (N < 0 || k < 0 || (N > 0 && (k < 1 || !nbr || !blocks))) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->spai_N = N;
    ctx->spai_k = k;
    ctx->spai_nbr = N > 0 ? nbr : nullptr;
    ctx->spai_blocks = N > 0 ? blocks : nullptr;
    return CAD_OK;
}

int cad_block_jacobi_dev(cad_ctx* ctx, int64_t N, const double* A, int64_t lda, int* nbr, float* blocks)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 0 || lda < 3 * N || (N > 0 && (!A || !nbr || !blocks))) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ++ctx->launches;
    CK(block_jacobi(ctx->stream, A, lda, N, nbr, blocks));
    return CAD_OK;
}

int64_t cad_lpc_param_count(void) { return (int64_t)mlp_param_count(); }

int cad_lpc_features_dev(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, float* X,
                         int* nbr, double* h)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 0 || (N > 0 && (!P1 || !P2 || !P3 || !X || !nbr))) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (N > INT32_MAX) return fail(ctx, CAD_ERR_ARG, "too many elements");
    if (N == 0) return CAD_OK;
    void* geom;
    if (int r = ensure(ctx, S_LPC_GEOM, lpc_geom_doubles(N) * sizeof(double), &geom)) return r;
    CK(lpc_features(ctx->stream, P1, P2, P3, N, (double*)geom, nbr, X, &ctx->launches));
    if (h)
        CK(cudaMemcpyAsync(h, lpc_geom_h((const double*)geom, N), (size_t)N * sizeof(double), cudaMemcpyDeviceToDevice,
                           ctx->stream));
    return CAD_OK;
}

static float* lpc_net_ptr(cad_ctx* ctx) { return (float*)ctx->buf[S_LPC_NET].p; }

int cad_lpc_set_network(cad_ctx* ctx, const float* params)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (!params) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    const size_t P = mlp_param_count();
    void* net;
    if (int r = ensure(ctx, S_LPC_NET, 4 * P * sizeof(float), &net)) return r;
    CK(cudaMemcpyAsync(net, params, P * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync((float*)net + P, 0, 3 * P * sizeof(float), ctx->stream));   // Adam moments, gradients
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->lpc_net = true;
    ctx->lpc_t = 0;
    return CAD_OK;
}

int cad_lpc_get_network(cad_ctx* ctx, float* params)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (!params) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (!ctx->lpc_net) return fail(ctx, CAD_ERR_ARG, "no network set (cad_lpc_set_network)");
    CK(cudaMemcpyAsync(params, lpc_net_ptr(ctx), mlp_param_count() * sizeof(float), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CAD_OK;
}

int cad_lpc_dataset_clear(cad_ctx* ctx)
{
    if (!ctx) return CAD_ERR_ARG;
    ctx->lpc_rows = 0;
    return CAD_OK;
}

int64_t cad_lpc_dataset_rows(const cad_ctx* ctx) { return ctx ? ctx->lpc_rows : 0; }

// room for `need` rows in the training set, keeping the rows already there
static int lpc_grow(cad_ctx* ctx, int64_t need)
{
    if (need <= ctx->lpc_cap) return CAD_OK;
    int64_t cap = ctx->lpc_cap * 2 > need ? ctx->lpc_cap * 2 : need;
    if (cap < 4096) cap = 4096;
    float *X = nullptr, *T = nullptr;
    CK(cudaMalloc(&X, (size_t)cap * kLpcIn * sizeof(float)));
    if (cudaMalloc(&T, (size_t)cap * kLpcOut * sizeof(float)) != cudaSuccess) {
        cudaFree(X);
        return fail(ctx, CAD_ERR_OOM, "training set: out of device memory");
    }
    if (ctx->lpc_rows > 0) {
        CK(cudaMemcpyAsync(X, ctx->lpc_X, (size_t)ctx->lpc_rows * kLpcIn * sizeof(float), cudaMemcpyDeviceToDevice,
                           ctx->stream));
        CK(cudaMemcpyAsync(T, ctx->lpc_T, (size_t)ctx->lpc_rows * kLpcOut * sizeof(float), cudaMemcpyDeviceToDevice,
                           ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->lpc_X) cudaFree(ctx->lpc_X);
    if (ctx->lpc_T) cudaFree(ctx->lpc_T);
    ctx->lpc_X = X;
    ctx->lpc_T = T;
    ctx->lpc_cap = cap;
    return CAD_OK;
}

int cad_lpc_dataset_add(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, double nu,
                        double G, double lambda, const double* midpoints, const double* normals, int hs_flag)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 1 || bad_flag(hs_flag) || !P1 || !P2 || !P3 || !midpoints || !normals)
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (3 * N > 46000) return fail(ctx, CAD_ERR_ARG, "training meshes are limited to 15333 elements");
    double* g;
    if (int r = upload_geometry(ctx, normals, midpoints, P1, P2, P3, N, &g)) return r;
    const int64_t n3 = 3 * N;
    void *mat, *geom, *nbr;
    if (int r = ensure(ctx, S_LPC_MAT, 2 * (size_t)n3 * n3 * sizeof(double), &mat)) return r;
    if (int r = ensure(ctx, S_LPC_GEOM, lpc_geom_doubles(N) * sizeof(double), &geom)) return r;
    if (int r = ensure(ctx, S_LPC_TNBR, (size_t)N * kLpcK * sizeof(int), &nbr)) return r;
    if (int r = lpc_grow(ctx, ctx->lpc_rows + N)) return r;
    double* A = (double*)mat;
    double* Ainv = A + n3 * n3;
    // the exact inverse the targets come from: FP64 assembly, FP64 LU
    const int keep_asm = ctx->assembly, keep_solver = ctx->solver;
    ctx->assembly = CAD_ASSEMBLY_FP64;
    ctx->solver = CAD_SOLVER_LU64;
    int r = assemble_device(ctx, g + 9 * N, g + 12 * N, g, g + 3 * N, g + 6 * N, N, nu, G, lambda, hs_flag, OUT_AMAT,
                            nullptr, A, n3);
    if (!r) {
        const cudaError_t e = lpc_identity(ctx->stream, Ainv, n3, n3, &ctx->launches);
        r = e != cudaSuccess ? cuda_fail(ctx, e, "identity") : solve_device(ctx, n3, A, n3, Ainv, n3, n3);
    }
    ctx->assembly = keep_asm;
    ctx->solver = keep_solver;
    if (r) return r;
    int info = 0;
    if (int rr = read_info(ctx, &info)) return rr;
    if (info > 0) return fail(ctx, CAD_ERR_SINGULAR, "SingularException: the system matrix is singular");
    CK(lpc_features(ctx->stream, g, g + 3 * N, g + 6 * N, N, (double*)geom, (int*)nbr,
                    ctx->lpc_X + ctx->lpc_rows * kLpcIn, &ctx->launches));
    CK(lpc_targets(ctx->stream, Ainv, n3, (const int*)nbr, lpc_geom_h((const double*)geom, N), G, N,
                   ctx->lpc_T + ctx->lpc_rows * kLpcOut, &ctx->launches));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->lpc_rows += N;
    return CAD_OK;
}

int cad_lpc_dataset_set(cad_ctx* ctx, const float* X, const float* T, int64_t rows)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (rows < 0 || (rows > 0 && (!X || !T))) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->lpc_rows = 0;
    if (rows == 0) return CAD_OK;
    if (int r = lpc_grow(ctx, rows)) return r;
    CK(cudaMemcpyAsync(ctx->lpc_X, X, (size_t)rows * kLpcIn * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->lpc_T, T, (size_t)rows * kLpcOut * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->lpc_rows = rows;
    return CAD_OK;
}

// One pass of the context's network over host rows: outputs (out) and, with
// T set, the gradient of the mean squared error (grads) and the sum of
// squared errors (loss); host arrays in and out.
int cad_lpc_forward_backward(cad_ctx* ctx, const float* X, const float* T, int64_t rows, float* out, float* grads,
                             float* loss)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (rows < 1 || !X || (T && !grads) || (!T && (grads || loss))) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (rows > INT32_MAX) return fail(ctx, CAD_ERR_ARG, "too many rows");
    if (!ctx->lpc_net) return fail(ctx, CAD_ERR_ARG, "no network set (cad_lpc_set_network)");
    const size_t P = mlp_param_count();
    const size_t mlpws = (mlp_workspace_bytes(rows) + 255) / 256 * 256;
    const size_t io = (size_t)rows * (kLpcIn + 2 * kLpcOut) + P + 1;
    void* ws;
    if (int r = ensure(ctx, S_LPC_WS, mlpws + io * sizeof(float), &ws)) return r;
    float* xd = (float*)((char*)ws + mlpws);
    float* td = xd + rows * kLpcIn;
    float* od = td + rows * kLpcOut;
    float* gd = od + rows * kLpcOut;
    float* ld = gd + P;
    CK(cudaMemcpyAsync(xd, X, (size_t)rows * kLpcIn * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    if (T) CK(cudaMemcpyAsync(td, T, (size_t)rows * kLpcOut * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    MlpStep st{};
    st.stream = ctx->stream;
    st.params = lpc_net_ptr(ctx);
    st.X = xd;
    st.T = T ? td : nullptr;
    st.rows = rows;
    st.out = out ? od : nullptr;
    st.grads = T ? gd : nullptr;
    st.loss = T ? ld : nullptr;
    st.workspace = ws;
    st.launches = &ctx->launches;
    const int e = mlp_step(st);
    if (e != 0) return cuda_fail(ctx, (cudaError_t)e, "learned-preconditioner network");
    if (out) CK(cudaMemcpyAsync(out, od, (size_t)rows * kLpcOut * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (grads) CK(cudaMemcpyAsync(grads, gd, P * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (loss) CK(cudaMemcpyAsync(loss, ld, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CAD_OK;
}

int cad_lpc_dataset_get(cad_ctx* ctx, int64_t row0, int64_t rows, float* X, float* T)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (row0 < 0 || rows < 0 || row0 + rows > ctx->lpc_rows || (rows > 0 && (!X || !T)))
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (rows == 0) return CAD_OK;
    CK(cudaMemcpyAsync(X, ctx->lpc_X + row0 * kLpcIn, (size_t)rows * kLpcIn * sizeof(float), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK(cudaMemcpyAsync(T, ctx->lpc_T + row0 * kLpcOut, (size_t)rows * kLpcOut * sizeof(float),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CAD_OK;
}

int cad_lpc_train(cad_ctx* ctx, int64_t steps, int64_t batch, float lr, uint64_t seed, float* loss_hist)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (steps < 0 || batch < 1 || !(lr > 0.f)) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (!ctx->lpc_net) return fail(ctx, CAD_ERR_ARG, "no network set (cad_lpc_set_network)");
    if (ctx->lpc_rows < 1) return fail(ctx, CAD_ERR_ARG, "empty training set (cad_lpc_dataset_add)");
    const int64_t b = batch < ctx->lpc_rows ? batch : ctx->lpc_rows;
    if (b > INT32_MAX) return fail(ctx, CAD_ERR_ARG, "batch too large");
    const int64_t nhist = (steps + 99) / 100;
    const size_t mlpws = (mlp_workspace_bytes(b) + 255) / 256 * 256;
    const size_t xbytes = ((size_t)b * (kLpcIn + kLpcOut) * sizeof(float) + 255) / 256 * 256;
    void* ws;
    if (int r = ensure(ctx, S_LPC_WS, mlpws + xbytes + (size_t)(nhist + 1) * sizeof(float), &ws)) return r;
    float* xb = (float*)((char*)ws + mlpws);
    float* tb = xb + b * kLpcIn;
    float* hist = (float*)((char*)ws + mlpws + xbytes);
    const size_t P = mlp_param_count();
    float* net = lpc_net_ptr(ctx);
    for (int64_t s = 0; s < steps; ++s) {
        CK(lpc_gather(ctx->stream, ctx->lpc_X, ctx->lpc_T, ctx->lpc_rows, b, seed, ctx->lpc_t, xb, tb,
                      &ctx->launches));
        ++ctx->lpc_t;
        MlpStep st{};
        st.stream = ctx->stream;
        st.params = net;
        st.X = xb;
        st.T = tb;
        st.rows = b;
        st.grads = net + 3 * P;
        st.loss = (s % 100 == 0) ? hist + s / 100 : nullptr;
        st.adam_m = net + P;
        st.adam_v = net + 2 * P;
        // cosine step size over this call's steps
        st.lr = (float)(lr * 0.5 * (1.0 + cos(M_PI * (double)s / (double)steps)));
        st.bias_c1 = 1.f - powf(0.9f, (float)ctx->lpc_t);
        st.bias_c2 = 1.f - powf(0.999f, (float)ctx->lpc_t);
        st.workspace = ws;
        st.launches = &ctx->launches;
        const int e = mlp_step(st);
        if (e != 0) return cuda_fail(ctx, (cudaError_t)e, "learned-preconditioner training step");
    }
    if (loss_hist && nhist > 0) {
        CK(cudaMemcpyAsync(loss_hist, hist, (size_t)nhist * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        for (int64_t k = 0; k < nhist; ++k) loss_hist[k] /= (float)(b * kLpcOut);
    }
    return CAD_OK;
}

int cad_lpc_install_dev(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, double G)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 1 || !P1 || !P2 || !P3) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (N > INT32_MAX) return fail(ctx, CAD_ERR_ARG, "too many elements");
    if (!ctx->lpc_net) return fail(ctx, CAD_ERR_ARG, "no network set (cad_lpc_set_network)");
    void *geom, *nbr, *feat, *out, *blk, *ws;
    if (int r = ensure(ctx, S_LPC_GEOM, lpc_geom_doubles(N) * sizeof(double), &geom)) return r;
    if (int r = ensure(ctx, S_LPC_NBR, (size_t)N * kLpcK * sizeof(int), &nbr)) return r;
    if (int r = ensure(ctx, S_LPC_FEAT, (size_t)N * kLpcIn * sizeof(float), &feat)) return r;
    if (int r = ensure(ctx, S_LPC_OUT, (size_t)N * kLpcOut * sizeof(float), &out)) return r;
    if (int r = ensure(ctx, S_LPC_BLK, (size_t)N * kLpcOut * sizeof(float), &blk)) return r;
    if (int r = ensure(ctx, S_MLP, mlp_workspace_bytes(N), &ws)) return r;
    CK(lpc_features(ctx->stream, P1, P2, P3, N, (double*)geom, (int*)nbr, (float*)feat, &ctx->launches));
    MlpStep st{};
    st.stream = ctx->stream;
    st.params = lpc_net_ptr(ctx);
    st.X = (const float*)feat;
    st.rows = N;
    st.out = (float*)out;
    st.workspace = ws;
    st.launches = &ctx->launches;
    const int e = mlp_step(st);
    if (e != 0) return cuda_fail(ctx, (cudaError_t)e, "learned-preconditioner network");
    CK(lpc_scale_blocks(ctx->stream, (const float*)out, lpc_geom_h((const double*)geom, N), G, N, (float*)blk,
                        &ctx->launches));
    ctx->spai_N = N;
    ctx->spai_k = kLpcK;
    ctx->spai_nbr = (const int*)nbr;
    ctx->spai_blocks = (const float*)blk;
    return CAD_OK;
}

int cad_lpc_install(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, double G)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 1 || !P1 || !P2 || !P3) return fail(ctx, CAD_ERR_ARG, "invalid argument");
    void* pg;
    if (int r = ensure(ctx, S_LPC_PGEOM, (size_t)9 * N * sizeof(double), &pg)) return r;
    double* g = (double*)pg;
    if (int r = upload(ctx, g, P1, 3 * N)) return r;
    if (int r = upload(ctx, g + 3 * N, P2, 3 * N)) return r;
    if (int r = upload(ctx, g + 6 * N, P3, 3 * N)) return r;
    return cad_lpc_install_dev(ctx, g, g + 3 * N, g + 6 * N, N, G);
}

int cad_lpc_step(cad_ctx* ctx, float* params, const float* X, const float* T, int64_t rows, float* out, float* grads,
                 float* loss, float* adam_m, float* adam_v, int64_t t, float lr)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (rows < 0 || !params || (rows > 0 && !X) || (grads && !T) || ((adam_m || adam_v) && (!adam_m || !adam_v ||
                                                                                             !grads || t < 1)))
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (rows == 0) return CAD_OK;
    if (rows > INT32_MAX) return fail(ctx, CAD_ERR_ARG, "too many rows");
    void* ws;
    if (int r = ensure(ctx, S_MLP, mlp_workspace_bytes(rows), &ws)) return r;
    MlpStep st{};
    st.stream = ctx->stream;
    st.params = params;
    st.X = X;
    st.T = T;
    st.rows = rows;
    st.out = out;
    st.grads = grads;
    st.loss = loss;
    st.adam_m = adam_m;
    st.adam_v = adam_v;
    st.lr = lr;
    st.bias_c1 = 1.f - powf(0.9f, (float)t);
    st.bias_c2 = 1.f - powf(0.999f, (float)t);
    st.workspace = ws;
    st.launches = &ctx->launches;
    const int e = mlp_step(st);
    if (e != 0) return cuda_fail(ctx, (cudaError_t)e, "learned-preconditioner network step");
    return CAD_OK;
}

int cad_slip_calculator_fixed(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N,
                              double nu, double G, double lambda, const double* midpoints, const double* normals,
                              int hs_flag, const double* Tn, const double* Tss, const double* Tds,
                              const double* fixed_els, double* Dn, double* Dss, double* Dds, double* A_out,
                              double* b_out)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 0 || bad_flag(hs_flag) || !Tn || !Tss || !Tds || !Dn || !Dss || !Dds)
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    const FixedSplit fs = split_fixed(fixed_els, N);
    if (fs.fixidx.empty())
        return cad_slip_calculator(ctx, P1, P2, P3, N, nu, G, lambda, midpoints, normals, hs_flag, Tn, Tss, Tds, Dn,
                                   Dss, Dds, A_out, b_out);
    const int64_t nf = (int64_t)fs.freecol.size(), n3 = 3 * N, m3 = 3 * nf;
    double* g;
    if (int r = upload_geometry(ctx, normals, midpoints, P1, P2, P3, N, &g)) return r;
    // tractions with the fixed rows knocked out (src/KnockOutFixedRows.jl)
    std::vector<double> hb((size_t)n3);
    for (int64_t i = 0; i < N; ++i) {
        const bool fx = fs.fixrow[i] >= 0;
        hb[i] = fx ? 0.0 : Tn[i];
        hb[N + i] = fx ? 0.0 : Tss[i];
        hb[2 * N + i] = fx ? 0.0 : Tds[i];
    }
    void *A, *b, *ata;
    if (int r = ensure(ctx, S_A, (size_t)n3 * m3 * sizeof(double) + 16, &A)) return r;
    if (int r = ensure(ctx, S_B, (size_t)n3 * sizeof(double), &b)) return r;
    if (int r = ensure(ctx, S_ATA, ((size_t)m3 * m3 + m3) * sizeof(double), &ata)) return r;
    if (int r = upload(ctx, (double*)b, hb.data(), n3)) return r;
    if (int r = assemble_fixed_device(ctx, g, N, nu, G, lambda, hs_flag, fs, true, (double*)A, n3)) return r;
    if (A_out) CK(cudaMemcpyAsync(A_out, A, (size_t)n3 * m3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (b_out) CK(cudaMemcpyAsync(b_out, b, (size_t)n3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    // the tall system in the least-squares sense (Julia's backslash on a 3N x 3nf
    // matrix): normal equations A^T A D = A^T b, solved by the FP64 LU
    double* AtA = (double*)ata;
    double* Atb = AtA + (size_t)m3 * m3;
    // A^T A = 0 - (-A^T) A through the library's DMMA product; A^T b by a
    // column-wise reduction
    void* atv;
    if (int r = ensure(ctx, S_AT, (size_t)m3 * n3 * sizeof(double) + 16, &atv)) return r;
    CK(krylov_transpose_neg(ctx->stream, (const double*)A, n3, n3, m3, (double*)atv, m3, &ctx->launches));
    CK(cudaMemsetAsync(AtA, 0, (size_t)m3 * m3 * sizeof(double), ctx->stream));
    CK(gemm_sub(ctx->stream, (int)m3, (int)m3, (int)n3, (const double*)atv, m3, (const double*)A, n3, AtA, m3,
                nullptr));
    ++ctx->launches;
    CK(krylov_gemv_t(ctx->stream, (const double*)A, n3, n3, m3, (const double*)b, Atb, &ctx->launches));
    const int solver = ctx->solver;
    ctx->solver = CAD_SOLVER_LU64;
    int r = solve_device(ctx, m3, AtA, m3, Atb, m3, 1);
    int info = 0;
    if (r == CAD_OK) r = read_info(ctx, &info);
    ctx->solver = solver;
    if (r) return r;
    if (info > 0) return fail(ctx, CAD_ERR_SINGULAR, "SingularException: the system matrix is rank deficient");
    CK(cudaMemcpyAsync(Dn, Atb, nf * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(Dss, Atb + nf, nf * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(Dds, Atb + 2 * nf, nf * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return CAD_OK;
}

int cad_assemble_update_dev(cad_ctx* ctx, const double* normals, const double* midpoints, const double* P1,
                            const double* P2, const double* P3, int64_t N, double nu, double G, double lambda,
                            int hs_flag, const int64_t* changed, int64_t k, double* A, int64_t lda)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 0 || k < 0 || bad_flag(hs_flag) || lda < 3 * N || (k > 0 && !changed) || N > INT32_MAX)
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    std::vector<int> list((size_t)k);
    for (int64_t q = 0; q < k; ++q) {
        if (changed[q] < 0 || changed[q] >= N) return fail(ctx, CAD_ERR_ARG, "changed element index out of range");
        list[q] = (int)changed[q];
    }
    if (k == 0 || N == 0) return CAD_OK;
    void *obs, *dirs, *tri, *dl;
    if (int r = ensure(ctx, S_OBS, (size_t)3 * N * sizeof(double), &obs)) return r;
    if (int r = ensure(ctx, S_DIRS, (size_t)9 * N * sizeof(double), &dirs)) return r;
    if (int r = ensure(ctx, S_TRI, (size_t)N * tri_record_bytes(), &tri)) return r;
    if (int r = ensure(ctx, S_LIST, (size_t)k * sizeof(int), &dl)) return r;
    double* X = (double*)obs;
    ++ctx->launches;
    CK(launch_colloc(normals, midpoints, N, X, X + N, X + 2 * N, (double*)dirs, ctx->stream));
    if (hs_flag == 1)
        if (int r = hs_check(ctx, X + 2 * N, N, P1, P2, P3, N)) return r;
    ++ctx->launches;
    CK(launch_td_setup(P1, P2, P3, N, nullptr, nullptr, nullptr, 1, nu, hs_flag == 1, (TriDev*)tri, ctx->stream));
    CK(cudaMemcpyAsync(dl, list.data(), k * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    PairArgs a{};
    a.X = X; a.Y = X + N; a.Z = X + 2 * N; a.M = N; a.tri = (const TriDev*)tri; a.N = N;
    a.lambda = lambda; a.G = G; a.dirs = (const double*)dirs;
    a.A = A; a.lda = lda;
    CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    CK(launch_assemble_update(a, hs_flag == 1, (const int*)dl, k, ctx->stream, &ctx->launches));
    CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    ctx->timed[0] = true;
    CK(cudaStreamSynchronize(ctx->stream));   // the host list is read by the copy above
    return CAD_OK;
}


// ---------------------------------------------------------------- LCP solve ---

namespace {

// Fischer-Burmeister Newton method for the LCP x >= 0, y = M x + q >= 0,
// x'y = 0 (the job of FischerNewton.fischer_newton, src/SlipCalculator3D.jl:196):
// from x = 0, Newton steps on Phi(x) = FB(x, M x + q) = 0 with the generalized
// Jacobian diag(Da) + diag(Db) M (rows with x_i = y_i = 0 taken along
// z = e_beta), each solved by the FP64 LU and chain solve, and an Armijo
// backtracking line search on psi = |Phi|^2 / 2 (all kLsSteps trial steps in
// one launch).  A singular Newton matrix or a non-finite direction falls back
// to steepest descent on psi.  Stops when max|Phi| <= tol max|q|, after
// max_iter steps, or when no trial step decreases psi.  x (device, n) is the
// solution; y (device, n) holds M x + q at exit; rel = max|Phi| / max|q|.
int lcp_newton_device(cad_ctx* ctx, const LcpOperator& op, const double* q, double* x, double* y, double tol,
                      int max_iter, int* iters_out, double* rel_out)
{
    const int64_t n = op.n;
    constexpr double kSigma = 1e-4;
    // the friction problem's Newton systems are solved in reduced form (3m unknowns)
    const int64_t nj = op.friction ? 3 * op.m : n;
    void *jv, *vv;
    if (int r = ensure(ctx, S_LCPJ, (size_t)nj * nj * sizeof(double), &jv)) return r;
    if (int r = ensure(ctx, S_LCPV, ((size_t)13 * n + lcp_partial_doubles()) * sizeof(double), &vv)) return r;
    double* J = (double*)jv;
    double* V = (double*)vv;
    double *phi = V, *z = V + n, *w = V + 2 * n, *Da = V + 3 * n, *Db = V + 4 * n, *d = V + 5 * n, *Md = V + 6 * n,
           *u = V + 7 * n, *part = V + 13 * n;
    // friction: coef (16m), u0 (3m), C u0 (3m), reduced right-hand side (3m) = 5n doubles
    double *coef = V + 8 * n, *u0 = coef + 16 * op.m, *cu0 = u0 + 3 * op.m, *rhs = cu0 + 3 * op.m;
    double* stats = part + (size_t)kRedBlocks * (kLsSteps + 1);
    double* psi_dev = stats + 8;
    void* kwv;
    if (int r = ensure(ctx, S_KWORK, krylov_work_doubles(n) * sizeof(double), &kwv)) return r;
    const KrylovWork kw = krylov_carve((double*)kwv, n);
    cudaStream_t st = ctx->stream;
    CK(cudaMemsetAsync(x, 0, n * sizeof(double), st));
    CK(cudaMemsetAsync(w, 0, n * sizeof(double), st));
    double hs[kLsSteps + 1];
    CK(lcp_max_abs(q, n, part, stats, st, &ctx->launches));
    CK(cudaMemcpyAsync(hs, stats, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const double qscale = hs[0] > 0.0 ? hs[0] : 1.0;
    const int saved_solver = ctx->solver;
    struct Restore {
        cad_ctx* c;
        int s;
        ~Restore() { c->solver = s; }
    } restore{ctx, saved_solver};
    ctx->solver = CAD_SOLVER_LU64;
    int it = 0;
    bool stalled = false;
    double rel = 0.0;
    for (;;) {
        if (lcp_matvec(op, kw, st, x, q, y, u, &ctx->launches))
            return fail(ctx, CAD_ERR_CUDA, "LCP: matrix-vector product failed");
        CK(lcp_fb_eval(x, y, n, phi, z, part, stats, st, &ctx->launches));
        CK(cudaMemcpyAsync(hs, stats, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        rel = hs[0] / qscale;
        const double psi = 0.5 * hs[1];
        if (!(rel > tol) || it >= max_iter || stalled) break;
        if (hs[2] > 0.0)   // rows with x_i = y_i = 0: w = M z
            if (lcp_matvec(op, kw, st, z, nullptr, w, u, &ctx->launches))
                return fail(ctx, CAD_ERR_CUDA, "LCP: matrix-vector product failed");
        CK(lcp_fb_diag(x, y, z, w, phi, n, Da, Db, d, st, &ctx->launches));
        int info = 0;
        if (op.friction) {   // J d = -phi through the 3m x 3m reduced system
            const int64_t m = op.m, m3 = 3 * m;
            CK(friction_reduce_prep(Da, Db, d, op.mu, m, coef, u0, st, &ctx->launches));
            if (krylov_gemv<double>(st, op.C, op.ldc, (int)m3, u0, 1.0, nullptr, cu0, kw, nullptr, 0, 0,
                                    &ctx->launches) != cudaSuccess)
                return fail(ctx, CAD_ERR_CUDA, "LCP: matrix-vector product failed");
            CK(friction_reduced_rhs(d, Da, Db, cu0, coef, m, rhs, st, &ctx->launches));
            CK(friction_reduced_jacobian(op.C, op.ldc, op.mu, Da, Db, coef, m, J, m3, st));
            ++ctx->launches;
            if (int r = solve_device(ctx, m3, J, m3, rhs, m3, 1)) return r;
            if (int r = read_info(ctx, &info)) return r;
            CK(friction_recover(rhs, coef, m, d, st, &ctx->launches));
        } else {
            CK(lcp_build_jacobian(op, Da, Db, J, n, st));
            ++ctx->launches;
            if (int r = solve_device(ctx, n, J, n, d, n, 1)) return r;
            if (int r = read_info(ctx, &info)) return r;
        }
        double slope = -2.0 * psi;
        bool newton = info == 0;
        if (newton) {
            if (lcp_matvec(op, kw, st, d, nullptr, Md, u, &ctx->launches))
                return fail(ctx, CAD_ERR_CUDA, "LCP: matrix-vector product failed");
            CK(lcp_line_search(x, d, y, Md, n, part, psi_dev, st, &ctx->launches));
            CK(cudaMemcpyAsync(hs, psi_dev, (kLsSteps + 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (hs[kLsSteps] > 0.0) newton = false;   // a non-finite direction
        }
        if (!newton) {   // steepest descent: d = -(Da phi + M^T (Db phi))
            CK(lcp_scale(Db, phi, n, Md, st, &ctx->launches));
            if (lcp_matvec_t(op, st, Md, d, u, &ctx->launches))
                return fail(ctx, CAD_ERR_CUDA, "LCP: matrix-vector product failed");
            CK(lcp_grad_dir(Da, phi, n, d, part, stats, st, &ctx->launches));
            CK(cudaMemcpyAsync(hs, stats + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            slope = -hs[0];
            if (lcp_matvec(op, kw, st, d, nullptr, Md, u, &ctx->launches))
                return fail(ctx, CAD_ERR_CUDA, "LCP: matrix-vector product failed");
            CK(lcp_line_search(x, d, y, Md, n, part, psi_dev, st, &ctx->launches));
            CK(cudaMemcpyAsync(hs, psi_dev, (kLsSteps + 1) * sizeof(double), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
        double step = 0.0, t = 1.0;
        for (int k = 0; k < kLsSteps; ++k) {
            if (hs[k] <= psi + kSigma * t * slope) {
                step = t;
                break;
            }
            t *= 0.5;
        }
        ++it;
        if (step == 0.0) {
            stalled = true;   // no decrease left at rounding level: re-evaluate and stop
            continue;
        }
        CK(lcp_step(x, d, step, n, st, &ctx->launches));
    }
    ctx->last_iters = it;
    ctx->last_relres = rel;
    *iters_out = it;
    *rel_out = rel;
    return CAD_OK;
}

int lcp_status(cad_ctx* ctx, int iters, double rel, double tol)
{
    if (rel > tol || !(rel == rel)) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "Fischer-Newton stopped at max|Phi|/max|q| = %.3e after %d iterations", rel,
                      iters);
        return fail(ctx, CAD_ERR_NOT_CONVERGED, msg);
    }
    return CAD_OK;
}

}  // namespace

int cad_fischer_newton(cad_ctx* ctx, int64_t n, const double* A, const double* b, double tol, int max_iter,
                       double* x)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (n < 0 || !(tol > 0.0) || max_iter < 0 || (n > 0 && (!A || !b || !x)) || n > INT32_MAX)
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    if (n == 0) return CAD_OK;
    void *Mv, *pv;
    ctx->fric_ready = false;   // the dense matrix takes the prepared frictional system's place
    if (int r = ensure(ctx, S_LCPC, (size_t)n * n * sizeof(double), &Mv)) return r;
    if (int r = ensure(ctx, S_LCPP, (size_t)3 * n * sizeof(double), &pv)) return r;
    double* P = (double*)pv;
    double *q = P, *xd = P + n, *y = P + 2 * n;
    if (int r = upload(ctx, (double*)Mv, A, n * n)) return r;
    if (int r = upload(ctx, q, b, n)) return r;
    LcpOperator op;
    op.n = n;
    op.M = (const double*)Mv;
    op.ldm = n;
    int iters = 0;
    double rel = 0.0;
    if (int r = lcp_newton_device(ctx, op, q, xd, y, tol, max_iter, &iters, &rel)) return r;
    CK(cudaMemcpyAsync(x, xd, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return lcp_status(ctx, iters, rel, tol);
}

}  // extern "C"

namespace {

// The set-up half of the frictional solve (src/SlipCalculator3D.jl:56-61 and
// :90-92): A assembled as the plain path does, Scl = mean(HalfPerimeter) / G
// (AreaOfTriangle3D), C = inv(A Scl) from the FP64 LU solved against the
// identity, kept in the context for friction_solve_device.
int friction_prepare_device(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, double nu,
                            double G, double lambda, const double* midpoints, const double* normals, int hs_flag)
{
    ctx->fric_ready = false;
    double hp = 0.0;
    for (int64_t i = 0; i < N; ++i) {
        double e[3];
        const double* V[4] = {P1, P2, P3, P1};
        for (int k = 0; k < 3; ++k) {
            const double dx = V[k][i] - V[k + 1][i], dy = V[k][i + N] - V[k + 1][i + N],
                         dz = V[k][i + 2 * N] - V[k + 1][i + 2 * N];
            e[k] = std::sqrt(dx * dx + dy * dy + dz * dz);
        }
        hp += (e[0] + e[1] + e[2]) / 2.0;
    }
    const double scl = (hp / (double)N) / G;
    double* g;
    if (int r = upload_geometry(ctx, normals, midpoints, P1, P2, P3, N, &g)) return r;
    const int64_t n3 = 3 * N;
    void *A, *Cv;
    if (int r = ensure(ctx, S_A, (size_t)n3 * n3 * sizeof(double), &A)) return r;
    if (int r = ensure(ctx, S_LCPC, (size_t)n3 * n3 * sizeof(double), &Cv)) return r;
    int r = assemble_device(ctx, g + 9 * N, g + 12 * N, g, g + 3 * N, g + 6 * N, N, nu, G, lambda, hs_flag, OUT_AMAT,
                            nullptr, (double*)A, n3);
    if (r) return r;
    double* C = (double*)Cv;
    CK(scale_and_identity((double*)A, n3, n3, scl, C, ctx->stream, &ctx->launches));
    const int solver = ctx->solver;
    ctx->solver = CAD_SOLVER_LU64;
    r = solve_device(ctx, n3, (double*)A, n3, C, n3, n3);
    int info = 0;
    if (r == CAD_OK) r = read_info(ctx, &info);
    ctx->solver = solver;
    if (r) return r;
    if (info > 0) return fail(ctx, CAD_ERR_SINGULAR, "SingularException: the system matrix is singular");
    ctx->fric_ready = true;
    ctx->fric_N = N;
    ctx->fric_scl = scl;
    return CAD_OK;
}

// The solve half (src/SlipCalculator3D.jl:90-175 for q, :177-237 for the
// solve and the read-out) with the prepared C: q = [C (b - [0; Sf; Sf]); 2 Sf;
// 2 Sf], the LCP by the Fischer-Burmeister Newton method, slip from x and y.
int friction_solve_device(cad_ctx* ctx, const double* Tn, const double* Tss, const double* Tds, const double* mu,
                          const double* Sf, double tol, int max_iter, double* Dn, double* Dss, double* Dds)
{
    const int64_t N = ctx->fric_N, n3 = 3 * N, n5 = 5 * N;
    const double scl = ctx->fric_scl;
    double* C = (double*)ctx->buf[S_LCPC].p;
    void* pv;
    if (int r = ensure(ctx, S_LCPP, ((size_t)2 * N + n3 + n3 + 3 * n5) * sizeof(double), &pv)) return r;
    double* P = (double*)pv;
    double *dmu = P, *dsf = P + N, *b = P + 2 * N, *rr = b + n3, *q = rr + n3, *xd = q + n5, *y = xd + n5;
    double* slip = rr;   // r is dead once q is formed
    if (int r = upload(ctx, dmu, mu, N)) return r;
    if (int r = upload(ctx, dsf, Sf, N)) return r;
    if (int r = upload(ctx, b, Tn, N)) return r;
    if (int r = upload(ctx, b + N, Tss, N)) return r;
    if (int r = upload(ctx, b + 2 * N, Tds, N)) return r;
    // q = [C (b - [0; Sf; Sf]); 2 Sf; 2 Sf] (src/SlipCalculator3D.jl:158-163, :190-193)
    CK(friction_rhs(b, dsf, N, rr, q, ctx->stream, &ctx->launches));
    {
        void* kwv;
        if (int r = ensure(ctx, S_KWORK, krylov_work_doubles(n3) * sizeof(double), &kwv)) return r;
        CK(krylov_gemv<double>(ctx->stream, C, n3, (int)n3, rr, 1.0, nullptr, q, krylov_carve((double*)kwv, n3),
                               nullptr, 0, 0, &ctx->launches));
    }
    LcpOperator op;
    op.friction = true;
    op.n = n5;
    op.C = C;
    op.ldc = n3;
    op.mu = dmu;
    op.m = N;
    int iters = 0;
    double rel = 0.0;
    if (int r = lcp_newton_device(ctx, op, q, xd, y, tol, max_iter, &iters, &rel)) return r;
    CK(friction_slip(xd, y, N, scl, slip, ctx->stream, &ctx->launches));
    CK(cudaMemcpyAsync(Dn, slip, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(Dss, slip + N, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(Dds, slip + 2 * N, N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return lcp_status(ctx, iters, rel, tol);
}

bool friction_geometry_args_ok(int64_t N, int hs_flag, double G, const double* P1, const double* P2,
                               const double* P3, const double* midpoints, const double* normals)
{
    return N >= 0 && !bad_flag(hs_flag) && G != 0.0 && 5 * N <= INT32_MAX &&
           (N == 0 || (P1 && P2 && P3 && midpoints && normals));
}

bool friction_load_args_ok(int64_t N, double tol, int max_iter, const double* Tn, const double* Tss,
                           const double* Tds, const double* mu, const double* Sf, const double* Dn, const double* Dss,
                           const double* Dds)
{
    return tol > 0.0 && max_iter >= 0 && (N == 0 || (Tn && Tss && Tds && mu && Sf && Dn && Dss && Dds));
}

}  // namespace

extern "C" {

int cad_slip_calculator_friction(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N,
                                 double nu, double G, double lambda, const double* midpoints, const double* normals,
                                 int hs_flag, const double* Tn, const double* Tss, const double* Tds,
                                 const double* mu, const double* Sf, double tol, int max_iter, double* Dn,
                                 double* Dss, double* Dds)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (!friction_geometry_args_ok(N, hs_flag, G, P1, P2, P3, midpoints, normals) ||
        !friction_load_args_ok(N, tol, max_iter, Tn, Tss, Tds, mu, Sf, Dn, Dss, Dds))
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->last_iters = 0;
    ctx->last_relres = 0.0;
    if (N == 0) return CAD_OK;
    // no element can overcome its frictional resistance: no slip
    // (src/SlipCalculator3D.jl:46-55; FricRes = Tn mu, negative is compression)
    bool all_ss = true, all_ds = true;
    for (int64_t i = 0; i < N; ++i) {
        const double fr = Tn[i] * mu[i];
        all_ss = all_ss && (-std::fabs(Tss[i]) > fr);
        all_ds = all_ds && (-std::fabs(Tds[i]) > fr);
    }
    if (all_ss && all_ds) {
        std::fill(Dn, Dn + N, 0.0);
        std::fill(Dss, Dss + N, 0.0);
        std::fill(Dds, Dds + N, 0.0);
        return CAD_OK;
    }
    if (int r = friction_prepare_device(ctx, P1, P2, P3, N, nu, G, lambda, midpoints, normals, hs_flag)) return r;
    return friction_solve_device(ctx, Tn, Tss, Tds, mu, Sf, tol, max_iter, Dn, Dss, Dds);
}

int cad_friction_prepare(cad_ctx* ctx, const double* P1, const double* P2, const double* P3, int64_t N, double nu,
                         double G, double lambda, const double* midpoints, const double* normals, int hs_flag)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (!friction_geometry_args_ok(N, hs_flag, G, P1, P2, P3, midpoints, normals))
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->fric_ready = false;
    if (N == 0) return CAD_OK;
    return friction_prepare_device(ctx, P1, P2, P3, N, nu, G, lambda, midpoints, normals, hs_flag);
}

int cad_friction_solve(cad_ctx* ctx, int64_t N, const double* Tn, const double* Tss, const double* Tds,
                       const double* mu, const double* Sf, double tol, int max_iter, double* Dn, double* Dss,
                       double* Dds)
{
    CAD_NVTX_RANGE();
    if (int r = set_device(ctx)) return r;
    if (N < 0 || !friction_load_args_ok(N, tol, max_iter, Tn, Tss, Tds, mu, Sf, Dn, Dss, Dds))
        return fail(ctx, CAD_ERR_ARG, "invalid argument");
    ctx->last_iters = 0;
    ctx->last_relres = 0.0;
    if (N == 0) return CAD_OK;
    if (!ctx->fric_ready || ctx->fric_N != N)
        return fail(ctx, CAD_ERR_ARG, "cad_friction_solve: no prepared frictional system of this size "
                                      "(call cad_friction_prepare first)");
    return friction_solve_device(ctx, Tn, Tss, Tds, mu, Sf, tol, max_iter, Dn, Dss, Dds);
}

}  // extern "C"
