// Test-only host build of the device pair code (csrc/td_device.cuh compiled by a
// plain C++ compiler), so the kernels' arithmetic can be checked against the
// oracle on a machine without a GPU.  Not part of the library.
#include <cmath>
#include <cstdint>
#include "td_device.cuh"
using namespace cad;
extern "C" int host_td_inf(const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
                           const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds,
                           const double* Dn, double nu, int disp, int strain, int hs, double* so, double* dout) {
  const int64_t MN = M * N;
  static TriDev t;  // ~13 KB; one record at a time
  for (int64_t j = 0; j < N; ++j) {
    double a[3] = {P1[j], P1[j + N], P1[j + 2 * N]}, b[3] = {P2[j], P2[j + N], P2[j + 2 * N]},
           c[3] = {P3[j], P3[j + N], P3[j + 2 * N]};
    build_triangle(a, b, c, Dss[j], Dds[j], Dn[j], nu, hs != 0, t);
    for (int64_t i = 0; i < M; ++i) {
      if (strain) {
        double E[3][6];
        if (hs) pair_strain<true>(t, X[i], Y[i], Z[i], E); else pair_strain<false>(t, X[i], Y[i], Z[i], E);
        for (int m = 0; m < 3; ++m) for (int k = 0; k < 6; ++k) so[(6 * m + k) * MN + i + M * j] = E[m][k];
      }
      if (disp) {
        double U[3][3];
        if (hs) pair_disp<true>(t, X[i], Y[i], Z[i], U); else pair_disp<false>(t, X[i], Y[i], Z[i], U);
        for (int m = 0; m < 3; ++m) for (int k = 0; k < 3; ++k) dout[(3 * m + k) * MN + i + M * j] = U[m][k];
      }
    }
  }
  return 0;
}

// The shared-edge half-space paths on the host, laid out as the kernels do.
// side_code: 3 per triangle, +-(edge + 1); edge_pts: 6 per edge (PA, PB).
// Influence fields: per-edge strain and displacement maps at every point,
// G[(e Q + q) M + i], read by pair_strain_edges / pair_disp_edges.
extern "C" int host_td_inf_edges(const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
                                 const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds,
                                 const double* Dn, double nu, const int* side_code, const double* edge_pts, int64_t E,
                                 double* so, double* dout) {
  const int64_t MN = M * N, Q = 27;
  double* G = new double[(size_t)(E * Q * M)];
  static FscSide s;
  for (int64_t e = 0; e < E; ++e) {
    build_side_geom(edge_pts + 6 * e, edge_pts + 6 * e + 3, nu, s);
    for (int64_t i = 0; i < M; ++i) {
      double Gm[3][6] = {}, Gu[3][3] = {};
      if (s.skip == 0.0) { fsc_strain_map(s, X[i], Y[i], Z[i], Gm); fsc_disp_map(s, X[i], Y[i], Z[i], Gu); }
      for (int q = 0; q < 18; ++q) G[(e * Q + q) * M + i] = Gm[q / 6][q % 6];
      for (int q = 0; q < 9; ++q) G[(e * Q + 18 + q) * M + i] = Gu[q / 3][q % 3];
    }
  }
  static TriDev t;
  for (int64_t j = 0; j < N; ++j) {
    double a[3] = {P1[j], P1[j + N], P1[j + 2 * N]}, b[3] = {P2[j], P2[j + N], P2[j + 2 * N]},
           c[3] = {P3[j], P3[j + N], P3[j + 2 * N]};
    build_triangle(a, b, c, Dss[j], Dds[j], Dn[j], nu, true, t);
    for (int64_t i = 0; i < M; ++i) {
      double Es[3][6], U[3][3];
      pair_strain_edges(t, X[i], Y[i], Z[i], G + i, M, Q * M, side_code + 3 * j, Es);
      pair_disp_edges(t, X[i], Y[i], Z[i], G + 18 * M + i, M, Q * M, side_code + 3 * j, U);
      for (int m = 0; m < 3; ++m) for (int k = 0; k < 6; ++k) so[(6 * m + k) * MN + i + M * j] = Es[m][k];
      for (int m = 0; m < 3; ++m) for (int k = 0; k < 3; ++k) dout[(3 * m + k) * MN + i + M * j] = U[m][k];
    }
  }
  delete[] G;
  return 0;
}

// Sums: real + image terms per triangle, plus each edge's correction once for
// the net Burgers vector of the sides on it (edge_tris[edge_ptr[e] ..
// edge_ptr[e + 1]) = +-(triangle + 1)).  so: 6 x M, dout: 3 x M.
extern "C" int host_td_sum_edges(const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
                                 const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds,
                                 const double* Dn, double nu, const int* edge_ptr, const int* edge_tris,
                                 const double* edge_pts, int64_t E, double* so, double* dout) {
  TriDev* T = new TriDev[(size_t)N];
  for (int64_t j = 0; j < N; ++j) {
    double a[3] = {P1[j], P1[j + N], P1[j + 2 * N]}, b[3] = {P2[j], P2[j + N], P2[j + 2 * N]},
           c[3] = {P3[j], P3[j + N], P3[j + 2 * N]};
    build_triangle(a, b, c, Dss[j], Dds[j], Dn[j], nu, true, T[j]);
  }
  FscSide* S = new FscSide[(size_t)E];
  for (int64_t e = 0; e < E; ++e) {
    double B[3] = {0.0, 0.0, 0.0};
    for (int k = edge_ptr[e]; k < edge_ptr[e + 1]; ++k) {
      const int cc = edge_tris[k];
      const TriDev& t = T[(cc > 0 ? cc : -cc) - 1];
      const double sg = cc > 0 ? 1.0 : -1.0;
      const double slip[3] = {t.Dn, t.Dss, t.Dds};
      const double* axes[3] = {t.real.Vn, t.real.Vs, t.real.Vd};
      for (int m = 0; m < 3; ++m)
        for (int q = 0; q < 3; ++q) B[q] = add_rn(B[q], sg * mul_rn(axes[m][q], slip[m]));
    }
    build_side_burgers(edge_pts + 6 * e, edge_pts + 6 * e + 3, B, nu, S[e]);
  }
  for (int64_t i = 0; i < M; ++i) {
    double Es[6] = {}, Us[3] = {};
    for (int64_t j = 0; j < N; ++j) {
      double E6[3][6], U3[3][3];
      pair_strain_fs_image(T[j], X[i], Y[i], Z[i], E6);
      pair_disp_fs_image(T[j], X[i], Y[i], Z[i], U3);
      for (int k = 0; k < 6; ++k) Es[k] += (E6[0][k] + E6[1][k]) + E6[2][k];
      for (int k = 0; k < 3; ++k) Us[k] += (U3[0][k] + U3[1][k]) + U3[2][k];
    }
    double Ee[3][6] = {}, Ue[3][3] = {};
    for (int64_t e = 0; e < E; ++e)
      if (S[e].skip == 0.0) { fsc_strain(S[e], X[i], Y[i], Z[i], 0.0, 0.0, 1.0, Ee); fsc_disp(S[e], X[i], Y[i], Z[i], 0.0, 0.0, 1.0, Ue); }
    for (int k = 0; k < 6; ++k) so[k * M + i] = Es[k] + Ee[0][k];
    for (int k = 0; k < 3; ++k) dout[k * M + i] = Us[k] + Ue[0][k];
  }
  delete[] S;
  delete[] T;
  return 0;
}
