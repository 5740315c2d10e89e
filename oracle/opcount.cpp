// Algorithmic work per (observation, triangle) pair: runs the oracle's literal
// restatement of src/TD.jl on a counting scalar.
//
// TEST INFRASTRUCTURE ONLY (used by bench.py to state the algorithmic FLOPs per
// pair that the roofline figure divides by time).
//
// Counting rule: every binary +, -, *, / on FP64 values is 1; sqrt, log, atan,
// atan2, acos, sin, cos, tan are 1 each; x^2 is 1 multiply, x^3 is 2, x^n is
// n-1; negation and comparisons are free.  Per-triangle work (frames, side
// constants) is reported separately so that callers can amortise it.
#include <cstdint>

#include "td_oracle.hpp"

namespace cad_oracle {

struct Counters {
    int64_t add = 0, mul = 0, div = 0, sqrt = 0, tr = 0;
};
static thread_local Counters g_cnt;

struct Flop {
    double v;
    Flop() : v(0.0) {}
    Flop(double x) : v(x) {}
};
inline Flop operator+(Flop a, Flop b) { ++g_cnt.add; return Flop(a.v + b.v); }
inline Flop operator-(Flop a, Flop b) { ++g_cnt.add; return Flop(a.v - b.v); }
inline Flop operator*(Flop a, Flop b) { ++g_cnt.mul; return Flop(a.v * b.v); }
inline Flop operator/(Flop a, Flop b) { ++g_cnt.div; return Flop(a.v / b.v); }
inline Flop operator-(Flop a) { return Flop(-a.v); }
inline bool operator==(Flop a, Flop b) { return a.v == b.v; }
inline bool operator!=(Flop a, Flop b) { return a.v != b.v; }
inline bool operator<(Flop a, Flop b) { return a.v < b.v; }
inline bool operator<=(Flop a, Flop b) { return a.v <= b.v; }
inline bool operator>(Flop a, Flop b) { return a.v > b.v; }
inline bool operator>=(Flop a, Flop b) { return a.v >= b.v; }
inline Flop sq(Flop x) { ++g_cnt.mul; return Flop(x.v * x.v); }
inline Flop cube(Flop x) { g_cnt.mul += 2; return Flop(x.v * x.v * x.v); }
inline Flop ipow(Flop x, int n) { g_cnt.mul += n - 1; return Flop(std::pow(x.v, (double)n)); }
inline Flop sqrt(Flop x) { ++g_cnt.sqrt; return Flop(std::sqrt(x.v)); }
inline Flop log(Flop x) { ++g_cnt.tr; return Flop(std::log(x.v)); }
inline Flop atan(Flop x) { ++g_cnt.tr; return Flop(std::atan(x.v)); }
inline Flop atan2(Flop y, Flop x) { ++g_cnt.tr; return Flop(std::atan2(y.v, x.v)); }
inline Flop acos(Flop x) { ++g_cnt.tr; return Flop(std::acos(x.v)); }
inline Flop cos(Flop x) { ++g_cnt.tr; return Flop(std::cos(x.v)); }
inline Flop sin(Flop x) { ++g_cnt.tr; return Flop(std::sin(x.v)); }
inline Flop tan(Flop x) { ++g_cnt.tr; return Flop(std::tan(x.v)); }
inline Flop fabs(Flop x) { return Flop(std::fabs(x.v)); }

}  // namespace cad_oracle

using namespace cad_oracle;

extern "C" {

// Counts for one pair of each kind over the given points and triangles
// (averaged over all M x N pairs).  out[0..4] = add, mul, div, sqrt,
// transcendental per pair for the pair work, out[5..9] the same for the
// per-triangle setup (per triangle).  kind: 0 strain, 1 displacement.
int cado_opcount(const double* X, const double* Y, const double* Z, int64_t M, const double* P1,
                 const double* P2, const double* P3, int64_t N, const double* Dss, const double* Dds,
                 const double* Dn, double nu, int kind, int hs, double* out)
{
    Counters pair_tot, setup_tot;
    for (int64_t j = 0; j < N; ++j) {
        Flop a[3], b[3], c[3];
        for (int k = 0; k < 3; ++k) {
            a[k] = P1[j + N * k];
            b[k] = P2[j + N * k];
            c[k] = P3[j + N * k];
        }
        g_cnt = Counters();
        TriangleState<Flop> t;
        build_triangle(a, b, c, t);
        Counters s = g_cnt;
        setup_tot.add += s.add; setup_tot.mul += s.mul; setup_tot.div += s.div;
        setup_tot.sqrt += s.sqrt; setup_tot.tr += s.tr;
        for (int64_t i = 0; i < M; ++i) {
            g_cnt = Counters();
            if (kind == 0) {
                Flop E[3][6];
                pair_strain(t, Flop(X[i]), Flop(Y[i]), Flop(Z[i]), Flop(Dss[j]), Flop(Dds[j]), Flop(Dn[j]),
                            Flop(nu), hs == 1, E);
            } else {
                Flop U[3][3];
                pair_disp(t, Flop(X[i]), Flop(Y[i]), Flop(Z[i]), Flop(Dss[j]), Flop(Dds[j]), Flop(Dn[j]),
                          Flop(nu), hs == 1, U);
            }
            pair_tot.add += g_cnt.add; pair_tot.mul += g_cnt.mul; pair_tot.div += g_cnt.div;
            pair_tot.sqrt += g_cnt.sqrt; pair_tot.tr += g_cnt.tr;
        }
    }
    const double np = (double)(M * N), nt = (double)N;
    out[0] = pair_tot.add / np; out[1] = pair_tot.mul / np; out[2] = pair_tot.div / np;
    out[3] = pair_tot.sqrt / np; out[4] = pair_tot.tr / np;
    out[5] = setup_tot.add / nt; out[6] = setup_tot.mul / nt; out[7] = setup_tot.div / nt;
    out[8] = setup_tot.sqrt / nt; out[9] = setup_tot.tr / nt;
    return 0;
}

}  // extern "C"
