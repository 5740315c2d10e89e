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
