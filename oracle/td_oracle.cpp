// CPU oracle entry points (extern "C", loaded by oracle/oracle.py through ctypes).
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA library and the timed CPU
// baseline.  Restates, per (observation, triangle) pair and in the reference's
// operation order:
//   TD influence-matrix overload  src/TD.jl:77-216
//   TD summing overload           src/TD.jl:219-410 (race-free: one thread owns
//                                 each observation point; triangles are summed in
//                                 index order as a single Julia thread does)
//   ConvertStrainInfMatsToTraction + helpers
//                                 src/CalculateInfluenceMatrices3D.jl:73-114,
//                                 src/HookesLaw3DStrain2Stress!.jl:160-184,
//                                 src/CalculateNormalTraction3D!.jl:229-255,
//                                 src/TractionVectorCartesianComponents3D!.jl:298-309,
//                                 src/CalculateTractionInChosenDirection3D!.jl:358-381,
//                                 src/CalculateSSandDSDirs.jl:417-481
//   SetupCollationPoints          src/CalculateInfluenceMatrices3D.jl:52-71
//   A = -[Atn;Atss;Atds]          src/SlipCalculator3D.jl:13-16
//
// Layouts follow Julia: vertex lists are N x 3 column-major (P[i + N*c]); an
// influence matrix is M x N column-major (observation = row, triangle = column).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <atomic>
#include <thread>
#include <vector>

#include "td_oracle.hpp"

using namespace cad_oracle;

namespace {

enum { OK = 0, ERR_DIMS = 1, ERR_HS_ABOVE = 2 };

// Dynamic parallel loop over [0, n) in chunks, on nthreads std::threads.
template <class F>
void parallel_for(int64_t n, int nthreads, int64_t chunk, F body)
{
    if (nthreads <= 1 || n <= chunk) {
        for (int64_t i = 0; i < n; ++i) body(i);
        return;
    }
    std::atomic<int64_t> next(0);
    auto worker = [&]() {
        for (;;) {
            const int64_t s = next.fetch_add(chunk);
            if (s >= n) break;
            const int64_t e = s + chunk < n ? s + chunk : n;
            for (int64_t i = s; i < e; ++i) body(i);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
}

bool hs_violation(const double* Z, int64_t M, const double* P1, const double* P2, const double* P3, int64_t N)
{
    // src/TD.jl:606-619 (checked for every triangle; any triangle fails them all)
    if (N == 0) return false;
    for (int64_t j = 0; j < N; ++j)
        if (P1[j + 2 * N] > 0.0 || P2[j + 2 * N] > 0.0 || P3[j + 2 * N] > 0.0) return true;
    for (int64_t i = 0; i < M; ++i)
        if (Z[i] > 0.0) return true;
    return false;
}

void tri_vertices(const double* P1, const double* P2, const double* P3, int64_t N, int64_t j, double a[3],
                  double b[3], double c[3])
{
    for (int k = 0; k < 3; ++k) {
        a[k] = P1[j + N * k];
        b[k] = P2[j + N * k];
        c[k] = P3[j + N * k];
    }
}

// Strike-slip and dip-slip direction cosines of one element normal
// (CalculateSSandDSDirs, src/CalculateSSandDSDirs.jl:417-481).
void ss_ds_dirs(double cx, double cy, double cz, double ss[3], double ds[3])
{
    const double nrm = std::sqrt(cx * cx + cy * cy);
    const double inv = 1.0 / nrm;
    const double r1 = cx * inv, r2 = cy * inv;
    ss[0] = -r2; ss[1] = r1; ss[2] = 0.0;
    const double DSCosAz = std::cos(std::acos(cz) - (M_PI / 2.0));
    double L = std::sin(std::acos(DSCosAz));
    if (cz < 0.0) L = -L;
    const double a = std::atan2(cy, cx);
    const double DSCosAx = std::cos(a) * L;
    const double DSCosAy = std::sin(a) * L;
    ds[0] = -DSCosAx; ds[1] = -DSCosAy; ds[2] = DSCosAz;
    // cross(eZ, n) == 0  <=>  normal is vertical
    if (cx == 0.0 && cy == 0.0) {
        if (cz < 1.0) {
            ds[0] = -1.0; ds[1] = 0.0; ds[2] = 0.0;
            ss[0] = 0.0; ss[1] = -1.0; ss[2] = 0.0;
        } else {
            ds[0] = -1.0; ds[1] = 0.0; ds[2] = 0.0;
            ss[0] = 0.0; ss[1] = 1.0; ss[2] = 0.0;
        }
    }
}

// Strain (one slip mode) -> (Tn, Tss, Tds) on the element with normal n.
void strain_to_traction(const double e[6], double lambda, double G, const double n[3], const double ss[3],
                        const double ds[3], double out[3])
{
    // Hooke (src/HookesLaw3DStrain2Stress!.jl:169-180)
    const double G2 = 2.0 * G;
    const double cons = lambda * ((e[0] + e[1]) + e[2]);
    const double Sxx = (G2 * e[0]) + cons, Syy = (G2 * e[1]) + cons, Szz = (G2 * e[2]) + cons;
    const double Sxy = G2 * e[3], Sxz = G2 * e[4], Syz = G2 * e[5];
    const double cx = n[0], cy = n[1], cz = n[2];
    // normal traction
    const double AA = Sxx * (cx * cx), BB = Syy * (cy * cy), CC = Szz * (cz * cz);
    const double DD = (2.0 * Sxy) * (cx * cy), EE = (2.0 * Syz) * (cy * cz), FF = (2.0 * Sxz) * (cz * cx);
    out[0] = ((((AA + BB) + CC) + DD) + EE) + FF;
    // traction vector, projected onto the plane and onto strike / dip
    const double Tx = ((Sxx * cx) + (Sxy * cy)) + (Sxz * cz);
    const double Ty = ((Sxy * cx) + (Syy * cy)) + (Syz * cz);
    const double Tz = ((Sxz * cx) + (Syz * cy)) + (Szz * cz);
    const double X2 = 1.0 - (cx * cx), Y2 = 1.0 - (cy * cy), Z2 = 1.0 - (cz * cz);
    const double XY = cx * cy, YZ = cy * cz, ZX = cz * cx;
    const double* dirs[2] = {ss, ds};
    for (int d = 0; d < 2; ++d) {
        const double* D = dirs[d];
        const double A = (((Tx * X2) - (Ty * XY)) - (Tz * ZX)) * D[0];
        const double B = (((Tx * (-XY)) + (Ty * Y2)) - (Tz * YZ)) * D[1];
        const double C = (((Tx * (-ZX)) - (Ty * YZ)) + (Tz * Z2)) * D[2];
        out[1 + d] = (A + B) + C;
    }
}

}  // namespace

namespace cad_oracle {
inline long double sq(long double x) { return x * x; }
inline long double cube(long double x) { return x * x * x; }
inline long double ipow(long double x, int n) { return std::pow(x, (long double)n); }
}  // namespace cad_oracle

extern "C" {

// TD influence-matrix overload.  strain_out: 18 fields x (M x N), StrainInf
// field order; disp_out: 9 fields x (M x N), DispInf field order.  Either may
// be null when its flag is 0.
int cado_td_inf(const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
                const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds,
                const double* Dn, double nu, double G, int disp, int strain, int hs, int nthreads,
                double* strain_out, double* disp_out)
{
    (void)G;
    if (hs == 1 && hs_violation(Z, M, P1, P2, P3, N)) return ERR_HS_ABOVE;
    const int64_t MN = M * N;
    parallel_for(N, nthreads, 1, [&](int64_t j) {
        double a[3], b[3], c[3];
        tri_vertices(P1, P2, P3, N, j, a, b, c);
        TriangleState<double> t;
        build_triangle(a, b, c, t);
        for (int64_t i = 0; i < M; ++i) {
            if (strain == 1) {
                double E[3][6];
                pair_strain(t, X[i], Y[i], Z[i], Dss[j], Dds[j], Dn[j], nu, hs == 1, E);
                for (int m = 0; m < 3; ++m)
                    for (int k = 0; k < 6; ++k) strain_out[(6 * m + k) * MN + i + M * j] = E[m][k];
            }
            if (disp == 1) {
                double U[3][3];
                pair_disp(t, X[i], Y[i], Z[i], Dss[j], Dds[j], Dn[j], nu, hs == 1, U);
                for (int m = 0; m < 3; ++m)
                    for (int cc = 0; cc < 3; ++cc) disp_out[(3 * m + cc) * MN + i + M * j] = U[m][cc];
            }
        }
    });
    return OK;
}

// The same influence-matrix computation carried out in long double (x87
// extended precision): an accuracy referee that tells how far any FP64
// evaluation of the closed form (this oracle's or the GPU's) is from the
// mathematically exact value on a given geometry.  Results rounded to double.
int cado_td_inf_ld(const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
                   const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds,
                   const double* Dn, double nu, int disp, int strain, int hs, int nthreads, double* strain_out,
                   double* disp_out)
{
    if (hs == 1 && hs_violation(Z, M, P1, P2, P3, N)) return ERR_HS_ABOVE;
    const int64_t MN = M * N;
    parallel_for(N, nthreads, 1, [&](int64_t j) {
        long double a[3], b[3], c[3];
        for (int k = 0; k < 3; ++k) {
            a[k] = P1[j + N * k];
            b[k] = P2[j + N * k];
            c[k] = P3[j + N * k];
        }
        TriangleState<long double> t;
        build_triangle(a, b, c, t);
        for (int64_t i = 0; i < M; ++i) {
            if (strain == 1) {
                long double E[3][6];
                pair_strain<long double>(t, X[i], Y[i], Z[i], Dss[j], Dds[j], Dn[j], nu, hs == 1, E);
                for (int m = 0; m < 3; ++m)
                    for (int k = 0; k < 6; ++k) strain_out[(6 * m + k) * MN + i + M * j] = (double)E[m][k];
            }
            if (disp == 1) {
                long double U[3][3];
                pair_disp<long double>(t, X[i], Y[i], Z[i], Dss[j], Dds[j], Dn[j], nu, hs == 1, U);
                for (int m = 0; m < 3; ++m)
                    for (int cc = 0; cc < 3; ++cc) disp_out[(3 * m + cc) * MN + i + M * j] = (double)U[m][cc];
            }
        }
    });
    return OK;
}

// TD summing overload: strain_out 6 x M (xx,yy,zz,xy,xz,yz), disp_out 3 x M.
int cado_td_sum_eval(const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
                     const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds,
                     const double* Dn, double nu, double G, int disp, int strain, int hs, int nthreads,
                     double* strain_out, double* disp_out)
{
    (void)G;
    if (hs == 1 && hs_violation(Z, M, P1, P2, P3, N)) return ERR_HS_ABOVE;
    std::vector<TriangleState<double>> tris(N);
    for (int64_t j = 0; j < N; ++j) {
        double a[3], b[3], c[3];
        tri_vertices(P1, P2, P3, N, j, a, b, c);
        build_triangle(a, b, c, tris[j]);
    }
    parallel_for(M, nthreads, 16, [&](int64_t i) {
        double es[6] = {0, 0, 0, 0, 0, 0}, us[3] = {0, 0, 0};
        for (int64_t j = 0; j < N; ++j) {
            if (strain == 1) {
                double E[3][6];
                pair_strain(tris[j], X[i], Y[i], Z[i], Dss[j], Dds[j], Dn[j], nu, hs == 1, E);
                for (int k = 0; k < 6; ++k) es[k] = es[k] + ((E[0][k] + E[1][k]) + E[2][k]);
            }
            if (disp == 1) {
                double U[3][3];
                pair_disp(tris[j], X[i], Y[i], Z[i], Dss[j], Dds[j], Dn[j], nu, hs == 1, U);
                for (int cc = 0; cc < 3; ++cc) us[cc] = us[cc] + ((U[0][cc] + U[1][cc]) + U[2][cc]);
            }
        }
        if (strain == 1)
            for (int k = 0; k < 6; ++k) strain_out[k * M + i] = es[k];
        if (disp == 1)
            for (int cc = 0; cc < 3; ++cc) disp_out[cc * M + i] = us[cc];
    });
    return OK;
}

// ConvertStrainInfMatsToTraction applied to given strain influence matrices:
// strain_in 18 x (M x N); normals M x 3; trac_out 9 x (M x N) in TractionInf
// order (DnTn,DnTss,DnTds,DssTn,DssTss,DssTds,DdsTn,DdsTss,DdsTds).
int cado_strain_to_traction(const double* strain_in, int64_t M, int64_t N, const double* normals, double lambda,
                            double G, int nthreads, double* trac_out)
{
    const int64_t MN = M * N;
    parallel_for(M, nthreads, 64, [&](int64_t i) {
        const double n[3] = {normals[i], normals[i + M], normals[i + 2 * M]};
        double ss[3], ds[3];
        ss_ds_dirs(n[0], n[1], n[2], ss, ds);
        for (int64_t j = 0; j < N; ++j)
            for (int m = 0; m < 3; ++m) {
                double e[6], t[3];
                for (int k = 0; k < 6; ++k) e[k] = strain_in[(6 * m + k) * MN + i + M * j];
                strain_to_traction(e, lambda, G, n, ss, ds, t);
                for (int r = 0; r < 3; ++r) trac_out[(3 * m + r) * MN + i + M * j] = t[r];
            }
    });
    return OK;
}

// CalculateInfluenceMatrices3D without fixed elements, fused per pair:
// collocation at incentre - 1e-12 * normal, unit slip in every mode, strain
// then traction.  Either trac_out (9 x N x N) or A_out (3N x 3N, the matrix
// -[Atn;Atss;Atds] of src/SlipCalculator3D.jl:13-16) may be null.
int cado_influence_traction(const double* normals, const double* midpoints, const double* P1, const double* P2,
                            const double* P3, int64_t N, double nu, double G, double lambda, int hs,
                            int nthreads, double* trac_out, double* A_out)
{
    std::vector<double> X(N), Y(N), Z(N);
    for (int64_t i = 0; i < N; ++i) {
        X[i] = midpoints[i] - (normals[i] * 1e-12);
        Y[i] = midpoints[i + N] - (normals[i + N] * 1e-12);
        Z[i] = midpoints[i + 2 * N] - (normals[i + 2 * N] * 1e-12);
    }
    if (hs == 1 && hs_violation(Z.data(), N, P1, P2, P3, N)) return ERR_HS_ABOVE;
    std::vector<double> SS(3 * N), DS(3 * N);
    for (int64_t i = 0; i < N; ++i) ss_ds_dirs(normals[i], normals[i + N], normals[i + 2 * N], &SS[3 * i], &DS[3 * i]);
    const int64_t NN = N * N, n3 = 3 * N;
    parallel_for(N, nthreads, 1, [&](int64_t j) {
        double a[3], b[3], c[3];
        tri_vertices(P1, P2, P3, N, j, a, b, c);
        TriangleState<double> t;
        build_triangle(a, b, c, t);
        for (int64_t i = 0; i < N; ++i) {
            double E[3][6];
            pair_strain(t, X[i], Y[i], Z[i], 1.0, 1.0, 1.0, nu, hs == 1, E);
            const double n[3] = {normals[i], normals[i + N], normals[i + 2 * N]};
            for (int m = 0; m < 3; ++m) {
                double tr[3];
                strain_to_traction(E[m], lambda, G, n, &SS[3 * i], &DS[3 * i], tr);
                if (trac_out)
                    for (int r = 0; r < 3; ++r) trac_out[(3 * m + r) * NN + i + N * j] = tr[r];
                if (A_out)
                    for (int r = 0; r < 3; ++r) A_out[(r * N + i) + n3 * (m * N + j)] = -tr[r];
            }
        }
    });
    return OK;
}

// CalculateNormalAndShearTractions3D (src/CalculateNormalAndShearTractions3D.jl:91-115)
// for a remote stress given per element: out Tn, Tds, Tss (each N).
void cado_normal_shear_tractions(const double* sxx, const double* syy, const double* szz, const double* sxy,
                                 const double* sxz, const double* syz, const double* normals, int64_t N,
                                 double* Tn, double* Tds, double* Tss)
{
    for (int64_t i = 0; i < N; ++i) {
        const double n[3] = {normals[i], normals[i + N], normals[i + 2 * N]};
        double ss[3], ds[3];
        ss_ds_dirs(n[0], n[1], n[2], ss, ds);
        const double Sxx = sxx[i], Syy = syy[i], Szz = szz[i], Sxy = sxy[i], Sxz = sxz[i], Syz = syz[i];
        const double cx = n[0], cy = n[1], cz = n[2];
        const double AA = Sxx * (cx * cx), BB = Syy * (cy * cy), CC = Szz * (cz * cz);
        const double DD = (2.0 * Sxy) * (cx * cy), EE = (2.0 * Syz) * (cy * cz), FF = (2.0 * Sxz) * (cz * cx);
        Tn[i] = ((((AA + BB) + CC) + DD) + EE) + FF;
        const double Tx = ((Sxx * cx) + (Sxy * cy)) + (Sxz * cz);
        const double Ty = ((Sxy * cx) + (Syy * cy)) + (Syz * cz);
        const double Tz = ((Sxz * cx) + (Syz * cy)) + (Szz * cz);
        const double X2 = 1.0 - (cx * cx), Y2 = 1.0 - (cy * cy), Z2 = 1.0 - (cz * cz);
        const double XY = cx * cy, YZ = cy * cz, ZX = cz * cx;
        const double* dirs[2] = {ss, ds};
        double out[2];
        for (int d = 0; d < 2; ++d) {
            const double* D = dirs[d];
            const double A = (((Tx * X2) - (Ty * XY)) - (Tz * ZX)) * D[0];
            const double B = (((Tx * (-XY)) + (Ty * Y2)) - (Tz * YZ)) * D[1];
            const double C = (((Tx * (-ZX)) - (Ty * YZ)) + (Tz * Z2)) * D[2];
            out[d] = (A + B) + C;
        }
        Tss[i] = out[0];
        Tds[i] = out[1];
    }
}

}  // extern "C"
