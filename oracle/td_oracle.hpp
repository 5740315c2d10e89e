// CPU oracle for the triangular-dislocation (TD) hot path.
//
// TEST INFRASTRUCTURE ONLY.  A scalar FP64 restatement of the reference's
// algorithm (src/TD.jl of CutAndDisplaceJulia), used as the checker by tests/,
// by the smoke check and as the benchmark's CPU baseline.  The CUDA product
// never includes or links this file.  Parity unpinned: the reference (Julia)
// cannot run here and stores no golden vectors, so this restatement is pinned
// only by the reference's analytic known-answer tests (Okada, Mogi, Eshelby,
// traction-free surface, Savage, Burgmann).
//
// The reference evaluates one triangle at a time and makes several passes over
// all observation points (src/TD.jl:146-214, :735-867, :1499-1620).  Every pass
// is element-wise in the observation index, so the arithmetic applied to one
// (observation, triangle) pair is a fixed sequence of operations; this oracle
// applies that sequence pair by pair, in the reference's order, with the
// reference's association of every sum and product.
//
// Templated on the scalar type so that the same code can run on `double`
// (checker, CPU baseline) and on an operation-counting scalar (algorithmic
// work per pair; see opcount.cpp).
#pragma once
#include <cmath>
#include <cstdint>
#include <limits>

#include "tde_closed_form.hpp"

namespace cad_oracle {

// ---------------------------------------------------------------- helpers
// cross! (src/cross!.jl:2-14) and LinearAlgebra.cross: same component formulas.
template <class T>
inline void cross3(const T a[3], const T b[3], T c[3])
{
    c[0] = (a[1] * b[2]) - (a[2] * b[1]);
    c[1] = (a[2] * b[0]) - (a[0] * b[2]);
    c[2] = (a[0] * b[1]) - (a[1] * b[0]);
}

// RotateObject3DNewCoords! (src/RotateObject3DNewCoords!.jl:45-55):
//   out_i = Ax1[i]*(X-Pa) + Ax2[i]*(Y-Pb) + Ax3[i]*(Z-Pc)
template <class T>
inline void rot3(T X, T Y, T Z, T Pa, T Pb, T Pc, const T ax1[3], const T ax2[3], const T ax3[3],
                 T& x, T& y, T& z)
{
    const T dX = X - Pa, dY = Y - Pb, dZ = Z - Pc;
    const T xo = ((ax1[0] * dX) + (ax2[0] * dY)) + (ax3[0] * dZ);
    const T yo = ((ax1[1] * dX) + (ax2[1] * dY)) + (ax3[1] * dZ);
    const T zo = ((ax1[2] * dX) + (ax2[2] * dY)) + (ax3[2] * dZ);
    x = xo; y = yo; z = zo;
}

// RotateObject3DNewCoords (allocating form, src/RotateObject3DNewCoords.jl:73-131)
// with Pa=Pb=Pc=0 (no shift):  out_i = (Ax1[i]*X + Ax2[i]*Y) + Ax3[i]*Z
template <class T>
inline void rot3_noshift(T X, T Y, T Z, const T ax1[3], const T ax2[3], const T ax3[3],
                         T& x, T& y, T& z)
{
    const T xo = ((ax1[0] * X) + (ax2[0] * Y)) + (ax3[0] * Z);
    const T yo = ((ax1[1] * X) + (ax2[1] * Y)) + (ax3[1] * Z);
    const T zo = ((ax1[2] * X) + (ax2[2] * Y)) + (ax3[2] * Z);
    x = xo; y = yo; z = zo;
}

// TensorTransformation3D! scalar form (src/TensorTransformation3D!.jl:35-53).
// A is the 3x3 matrix stored column-major as 9 numbers (A[0]..A[8] = A[1]..A[9]).
template <class T>
inline void tensor_rot(T t[6], const T A[9])
{
    const T Txx = t[0], Tyy = t[1], Tzz = t[2], Txy = t[3], Txz = t[4], Tyz = t[5];
    const T txx = (((((sq(A[0]) * Txx) + (((2.0 * A[0]) * A[3]) * Txy)) + (((2.0 * A[0]) * A[6]) * Txz)) +
                    (((2.0 * A[3]) * A[6]) * Tyz)) + (sq(A[3]) * Tyy)) + (sq(A[6]) * Tzz);
    const T tyy = (((((sq(A[1]) * Txx) + (((2.0 * A[1]) * A[4]) * Txy)) + (((2.0 * A[1]) * A[7]) * Txz)) +
                    (((2.0 * A[4]) * A[7]) * Tyz)) + (sq(A[4]) * Tyy)) + (sq(A[7]) * Tzz);
    const T tzz = (((((sq(A[2]) * Txx) + (((2.0 * A[2]) * A[5]) * Txy)) + (((2.0 * A[2]) * A[8]) * Txz)) +
                    (((2.0 * A[5]) * A[8]) * Tyz)) + (sq(A[5]) * Tyy)) + (sq(A[8]) * Tzz);
    const T txy = ((((((A[0] * A[1]) * Txx) + (((A[0] * A[4]) + (A[1] * A[3])) * Txy)) +
                     (((A[0] * A[7]) + (A[1] * A[6])) * Txz)) + (((A[3] * A[7]) + (A[4] * A[6])) * Tyz)) +
                   ((A[3] * A[4]) * Tyy)) + ((A[6] * A[7]) * Tzz);
    const T txz = ((((((A[0] * A[2]) * Txx) + (((A[0] * A[5]) + (A[2] * A[3])) * Txy)) +
                     (((A[0] * A[8]) + (A[2] * A[6])) * Txz)) + (((A[3] * A[8]) + (A[5] * A[6])) * Tyz)) +
                   ((A[3] * A[5]) * Tyy)) + ((A[6] * A[8]) * Tzz);
    const T tyz = ((((((A[1] * A[2]) * Txx) + (((A[2] * A[4]) + (A[1] * A[5])) * Txy)) +
                     (((A[2] * A[7]) + (A[1] * A[8])) * Txz)) + (((A[5] * A[7]) + (A[4] * A[8])) * Tyz)) +
                   ((A[4] * A[5]) * Tyy)) + ((A[7] * A[8]) * Tzz);
    t[0] = txx; t[1] = tyy; t[2] = tzz; t[3] = txy; t[4] = txz; t[5] = tyz;
}

// --------------------------------------------------------- triangle frame
// One triangle (real or image) in TDCS, as built by CalculateLocalTriCoords!
// (src/TD.jl:712-732), GlobalToTDECoords (:870-908) and CalcTDVectsAndAngles
// (:962-1008).  p2 is the TDCS origin (0,0,0).
template <class T>
struct TdFrame {
    T P1[3], P2[3], P3[3];
    T Vn[3], Vs[3], Vd[3];
    T p1[3], p2[3], p3[3];
    T e12[3], e13[3], e23[3];
    T A, B, C;
    // trimodefinder constants (src/TD.jl:1025-1030) on the (y,z) TDCS plane
    T t23y, t32x, t13x, t13y, t31y, base;
    bool flat;   // all three vertex z exactly 0 (the ImageFlag sign-flip branch)
};

template <class T>
void build_frame(const T P1[3], const T P2[3], const T P3[3], TdFrame<T>& f)
{
    for (int i = 0; i < 3; ++i) { f.P1[i] = P1[i]; f.P2[i] = P2[i]; f.P3[i] = P3[i]; }
    // CalculateLocalTriCoords!
    T a[3], b[3];
    for (int i = 0; i < 3; ++i) { a[i] = P2[i] - P1[i]; b[i] = P3[i] - P1[i]; }
    cross3(a, b, f.Vn);
    const T nn = sqrt((sq(f.Vn[0]) + sq(f.Vn[1])) + sq(f.Vn[2]));
    for (int i = 0; i < 3; ++i) f.Vn[i] = f.Vn[i] / nn;
    const T eZ[3] = {T(0.0), T(0.0), T(1.0)};
    cross3(eZ, f.Vn, f.Vs);
    if (f.Vs[0] == 0.0 && f.Vs[1] == 0.0 && f.Vs[2] == 0.0) {
        f.Vs[0] = T(0.0) * f.Vn[2];
        f.Vs[1] = T(1.0) * f.Vn[2];
        f.Vs[2] = T(0.0) * f.Vn[2];
    }
    const T ns = sqrt((sq(f.Vs[0]) + sq(f.Vs[1])) + sq(f.Vs[2]));
    for (int i = 0; i < 3; ++i) f.Vs[i] = f.Vs[i] / ns;
    cross3(f.Vn, f.Vs, f.Vd);

    // GlobalToTDECoords: Vx=(Vn1,Vs1,Vd1), Vy=(Vn2,Vs2,Vd2), Vz=(Vn3,Vs3,Vd3)
    const T Vx[3] = {f.Vn[0], f.Vs[0], f.Vd[0]};
    const T Vy[3] = {f.Vn[1], f.Vs[1], f.Vd[1]};
    const T Vz[3] = {f.Vn[2], f.Vs[2], f.Vd[2]};
    rot3(P1[0], P1[1], P1[2], P2[0], P2[1], P2[2], Vx, Vy, Vz, f.p1[0], f.p1[1], f.p1[2]);
    rot3(P3[0], P3[1], P3[2], P2[0], P2[1], P2[2], Vx, Vy, Vz, f.p3[0], f.p3[1], f.p3[2]);
    f.p2[0] = T(0.0); f.p2[1] = T(0.0); f.p2[2] = T(0.0);

    // CalcTDVectsAndAngles
    for (int i = 0; i < 3; ++i) f.e12[i] = f.p2[i] - f.p1[i];
    T nrm = sqrt((sq(f.e12[0]) + sq(f.e12[1])) + sq(f.e12[2]));
    for (int i = 0; i < 3; ++i) f.e12[i] = f.e12[i] / nrm;
    for (int i = 0; i < 3; ++i) f.e13[i] = f.p3[i] - f.p1[i];
    nrm = sqrt((sq(f.e13[0]) + sq(f.e13[1])) + sq(f.e13[2]));
    for (int i = 0; i < 3; ++i) f.e13[i] = f.e13[i] / nrm;
    for (int i = 0; i < 3; ++i) f.e23[i] = f.p3[i] - f.p2[i];
    nrm = sqrt((sq(f.e23[0]) + sq(f.e23[1])) + sq(f.e23[2]));
    for (int i = 0; i < 3; ++i) f.e23[i] = f.e23[i] / nrm;
    using std::acos;
    f.A = acos(((f.e12[0] * f.e13[0]) + (f.e12[1] * f.e13[1])) + (f.e12[2] * f.e13[2]));
    f.B = acos((((-f.e12[0]) * f.e23[0]) + ((-f.e12[1]) * f.e23[1])) + ((-f.e12[2]) * f.e23[2]));
    f.C = acos(((f.e23[0] * f.e13[0]) + (f.e23[1] * f.e13[1])) + (f.e23[2] * f.e13[2]));

    // trimodefinder(y, z, x, p1[2:3], p2[2:3], p3[2:3]) constants
    f.t23y = f.p2[2] - f.p3[2];   // p2_2_m_p3_2
    f.t32x = f.p3[1] - f.p2[1];   // p3_1_m_p2_1
    f.t13x = f.p1[1] - f.p3[1];   // p1_1_m_p3_1
    f.t13y = f.p1[2] - f.p3[2];   // p1_2_m_p3_2
    f.t31y = f.p3[2] - f.p1[2];   // p3_2_m_p1_2
    f.base = (f.t23y * f.t13x) + (f.t32x * f.t13y);
    f.flat = (P1[2] == 0.0 && P2[2] == 0.0 && P3[2] == 0.0);
}

// Observation point into TDCS of frame f (GlobalToTDECoords, src/TD.jl:891).
template <class T>
inline void to_tdcs(const TdFrame<T>& f, T X, T Y, T Z, T& x, T& y, T& z)
{
    const T Vx[3] = {f.Vn[0], f.Vs[0], f.Vd[0]};
    const T Vy[3] = {f.Vn[1], f.Vs[1], f.Vd[1]};
    const T Vz[3] = {f.Vn[2], f.Vs[2], f.Vd[2]};
    rot3(X, Y, Z, f.P2[0], f.P2[1], f.P2[2], Vx, Vy, Vz, x, y, z);
}

// trimodefinder (src/TD.jl:1010-1079): +1 configuration I, -1 configuration
// II, 0 on a TD side and in the TD plane.  Called with (y, z, x) of TDCS.
template <class T>
inline int trimode(const TdFrame<T>& f, T x, T y, T z)
{
    // x <- TDCS y, y <- TDCS z, z <- TDCS x (argument order of the caller)
    const T px = f.p3[1], py = f.p3[2];
    const T a = ((f.t23y * (y - px)) + (f.t32x * (z - py))) / f.base;
    const T b = ((f.t31y * (y - px)) + (f.t13x * (z - py))) / f.base;
    const T c = (T(1.0) - a) - b;
    bool casen = false, casez = false;
    if (a <= 0.0 && b > c && c > a) casen = true;
    else if (b <= 0.0 && c > a && a > b) casen = true;
    else if (c <= 0.0 && a > b && b > c) casen = true;
    else if (a == 0.0 && b >= 0.0 && c >= 0.0) casez = true;
    else if (a >= 0.0 && b == 0.0 && c >= 0.0) casez = true;
    else if (a >= 0.0 && b >= 0.0 && c == 0.0) casez = true;
    if (casez && x != 0.0) casez = false;   // -> casep
    if (casez) return 0;
    if (casen) return -1;
    return 1;
}

// ------------------------------------------------------ full-space strain
// TDSetupS for one point (src/TD.jl:1623-1750).  E[m][k]: m = Dn, Dss, Dds;
// k = xx, yy, zz, xy, xz, yz.
template <class T>
void td_setup_s(T x, T y, T z, T alpha, T Dn, T Dss, T Dds, T nu, const T tv[3], const T side[3],
                T E[3][6])
{
    const T CosT = side[2];
    const T SinT = side[1];
    // RotateObject2D(Dss,0,0,0,CosT,SinT) and RotateObject2D(0,Dds,0,0,CosT,SinT)
    const T Dss1 = (CosT * Dss) + ((-SinT) * 0.0);
    const T Dds0 = (SinT * Dss) + (CosT * 0.0);
    const T Dss0 = (CosT * 0.0) + ((-SinT) * Dds);
    const T Dds1 = (SinT * 0.0) + (CosT * Dds);
    using std::cos;
    using std::sin;
    const T Ang = T(-M_PI) + alpha;
    const T cosA = cos(Ang);
    const T sinA = sin(Ang);
    const T E1 = T(1.0) - nu;
    const T E2 = (2.0 * nu) + 1.0;
    const T sinADE1 = ((sinA / 8.0) / T(M_PI)) / (T(1.0) - nu);
    const T E3 = ((Dn / 8.0) / T(M_PI)) / E1;
    const T E5Dss1 = ((Dss1 / 8.0) / T(M_PI)) / E1;
    const T E5Dss0 = ((Dss0 / 8.0) / T(M_PI)) / E1;
    const T Bm[9] = {T(1.0), T(0.0), T(0.0), T(0.0), CosT, -SinT, T(0.0), SinT, CosT};

    // RotateObject2D!(y, z, tv2, tv3, CosT, SinT)
    const T Y = (CosT * (y - tv[1])) + ((-SinT) * (z - tv[2]));
    const T Z = (SinT * (y - tv[1])) + (CosT * (z - tv[2]));
    T o[21];
    ang_dis_strain(x, Y, Z, cosA, sinA, nu, E2, sinADE1, o);
    const T exxBx = o[0], exxBy = o[1], exxBz = o[2];
    const T eyyBx = o[3], eyyBy = o[4], eyyBz = o[5];
    const T ezzBx = o[6], ezzBy = o[7], ezzBz = o[8];
    const T exyBx = o[9], exyBy = o[10], exyBz = o[11];
    const T exzBx = o[12], exzBy = o[13], exzBz = o[14];
    const T eyzBx = o[15], eyzBy = o[16], eyzBz = o[17];
    const T rFi_rx = o[18], rFi_ry = o[19], rFi_rz = o[20];

    if (Dn != 0.0) {
        T t[6];
        t[0] = (Dn * rFi_rx) + (E3 * exxBx);
        t[1] = E3 * eyyBx;
        t[2] = E3 * ezzBx;
        t[3] = ((Dn * rFi_ry) / 2.0) - (E3 * exyBx);
        t[4] = ((Dn * rFi_rz) / 2.0) - (E3 * exzBx);
        t[5] = E3 * eyzBx;
        tensor_rot(t, Bm);
        for (int k = 0; k < 6; ++k) E[0][k] = E[0][k] + t[k];
    }
    // Dss and Dds modes share one form with (Dss1,Dds0,E5Dss1) or (Dss0,Dds1,E5Dss0)
    const T Ds_[2] = {Dss1, Dss0};
    const T Dd_[2] = {Dds0, Dds1};
    const T E5_[2] = {E5Dss1, E5Dss0};
    const T slip[2] = {Dss, Dds};
    for (int q = 0; q < 2; ++q) {
        if (!(slip[q] != 0.0)) continue;
        const T Ds = Ds_[q], Dd = Dd_[q], E5 = E5_[q];
        const T E4 = (((Ds * x) / 8.0) / T(M_PI)) / E1;
        T t[6];
        t[0] = ((-E4) * exxBy) + (((Dd * x) * sinADE1) * exxBz);
        t[1] = ((Ds * rFi_ry) - (E4 * eyyBy)) + (((Dd * x) * sinADE1) * eyyBz);
        t[2] = ((-E4) * ezzBy) + ((Dd * rFi_rz) + (((Dd * x) * sinADE1) * ezzBz));
        t[3] = (((Ds * rFi_rx) / 2.0) + (E5 * exyBy)) - ((Dd * sinADE1) * exyBz);
        t[4] = (E5 * exzBy) + (((Dd * rFi_rx) / 2.0) - ((Dd * sinADE1) * exzBz));
        t[5] = (((Ds * rFi_rz) / 2.0) - (E4 * eyzBy)) + (((Dd * rFi_ry) / 2.0) - (((Dd * x) * sinADE1) * eyzBz));
        tensor_rot(t, Bm);
        for (int k = 0; k < 6; ++k) E[1 + q][k] = E[1 + q][k] + t[k];
    }
}

// TDstrainFS (src/TD.jl:1499-1620) for one point.  E holds the accumulated
// EFCS strain of this (point, triangle) pair on entry (zero for the real TD;
// real + harmonic for the image TD) and the result on exit.
template <class T>
void td_strain_fs(const TdFrame<T>& f, T X, T Y, T Z, T Dss, T Dds, T Dn, T nu, bool image,
                  T E[3][6])
{
    T x, y, z;
    to_tdcs(f, X, Y, Z, x, y, z);
    const int mode = trimode(f, x, y, z);

    // Caller-visible components (k = 4, 5) that the flat-image branch detaches.
    T keep_xz[3], keep_yz[3];
    const bool detach = image && f.flat;
    if (image) {
        const T RotInv[9] = {f.Vn[0], f.Vs[0], f.Vd[0], f.Vn[1], f.Vs[1], f.Vd[1], f.Vn[2], f.Vs[2], f.Vd[2]};
        for (int m = 0; m < 3; ++m) tensor_rot(E[m], RotInv);
        if (detach) {
            // src/TD.jl:1518-1525: `exz = -exz` rebinds a local copy; the caller
            // keeps the TDCS-rotated value for the xz and yz components.
            for (int m = 0; m < 3; ++m) {
                keep_xz[m] = E[m][4];
                keep_yz[m] = E[m][5];
                E[m][4] = -E[m][4];
                E[m][5] = -E[m][5];
            }
        }
    }
    T ne13[3], ne12[3], ne23[3];
    for (int i = 0; i < 3; ++i) { ne13[i] = -f.e13[i]; ne12[i] = -f.e12[i]; ne23[i] = -f.e23[i]; }
    if (mode == 1) {
        td_setup_s(x, y, z, f.A, Dn, Dss, Dds, nu, f.p1, ne13, E);
        td_setup_s(x, y, z, f.B, Dn, Dss, Dds, nu, f.p2, f.e12, E);
        td_setup_s(x, y, z, f.C, Dn, Dss, Dds, nu, f.p3, f.e23, E);
    } else if (mode == -1) {
        td_setup_s(x, y, z, f.A, Dn, Dss, Dds, nu, f.p1, f.e13, E);
        td_setup_s(x, y, z, f.B, Dn, Dss, Dds, nu, f.p2, ne12, E);
        td_setup_s(x, y, z, f.C, Dn, Dss, Dds, nu, f.p3, ne23, E);
    } else {
        const T nan = T(std::numeric_limits<double>::quiet_NaN());
        for (int m = 0; m < 3; ++m)
            for (int k = 0; k < 6; ++k) E[m][k] = nan;
    }
    const T Rot[9] = {f.Vn[0], f.Vn[1], f.Vn[2], f.Vs[0], f.Vs[1], f.Vs[2], f.Vd[0], f.Vd[1], f.Vd[2]};
    for (int m = 0; m < 3; ++m) tensor_rot(E[m], Rot);
    if (detach) {
        for (int m = 0; m < 3; ++m) {
            E[m][4] = keep_xz[m];
            E[m][5] = keep_yz[m];
        }
    }
}

// -------------------------------------------------- full-space displacement
// TDSetupD for one point (src/TD.jl:1081-1173).  U[m][c]: m = Dn, Dss, Dds.
template <class T>
void td_setup_d(T x, T y, T z, T alpha, T Dn, T Dss, T Dds, T nu, const T tv[3], const T side[3],
                T U[3][3])
{
    const T CosT = side[2];
    const T SinT = side[1];
    const T Dss1 = (CosT * Dss) + ((-SinT) * 0.0);
    const T Dds0 = (SinT * Dss) + (CosT * 0.0);
    const T Dss0 = (CosT * 0.0) + ((-SinT) * Dds);
    const T Dds1 = (SinT * 0.0) + (CosT * Dds);
    using std::cos;
    using std::sin;
    const T Ang = T(-M_PI) + alpha;
    const T cosA = cos(Ang);
    const T sinA = sin(Ang);
    const T E1 = T(1.0) - nu;
    const T E2 = T(1.0) - (2.0 * nu);
    const T cosA2 = sq(cosA);
    const T sinADE1 = ((sinA / 8.0) / T(M_PI)) / (T(1.0) - nu);
    const T Dn8p = (Dn / 8.0) / T(M_PI);

    const T Y = (CosT * (y - tv[1])) + ((-SinT) * (z - tv[2]));
    const T Z = (SinT * (y - tv[1])) + (CosT * (z - tv[2]));
    T o[9];
    ang_dis_disp(x, Y, Z, cosA, sinA, E1, E2, cosA2, sinADE1, o);
    const T ux = o[0], uy = o[1], uz = o[2], vx = o[3], vy = o[4], vz = o[5], wx = o[6], wy = o[7], wz = o[8];

    // RotateObject2D!(u, w, 0, 0, CosT, -SinT)
    auto back = [&](T a, T b, T& ra, T& rb) {
        ra = (CosT * (a - 0.0)) + (SinT * (b - 0.0));
        rb = ((-SinT) * (a - 0.0)) + (CosT * (b - 0.0));
    };
    if (Dn != 0.0) {
        U[0][0] = U[0][0] + ((Dn8p / E1) * ux);
        T a = (Dn8p / E1) * vx, b = (Dn8p / E1) * wx, ra, rb;
        back(a, b, ra, rb);
        U[0][1] = U[0][1] + ra;
        U[0][2] = U[0][2] + rb;
    }
    const T Ds_[2] = {Dss1, Dss0};
    const T Dd_[2] = {Dds0, Dds1};
    const T slip[2] = {Dss, Dds};
    for (int q = 0; q < 2; ++q) {
        if (!(slip[q] != 0.0)) continue;
        const T Ds = Ds_[q], Dd = Dd_[q];
        U[1 + q][0] = (U[1 + q][0] + ((((Ds / 8.0) / T(M_PI)) / E1) * uy)) + ((Dd * sinADE1) * uz);
        T a = (((((Ds * x) / 8.0) / T(M_PI)) / E1) * vy) + (((Dd * x) * sinADE1) * vz);
        T b = (((((Ds * x) / 8.0) / T(M_PI)) / E1) * wy) + (((Dd * x) * sinADE1) * wz);
        T ra, rb;
        back(a, b, ra, rb);
        U[1 + q][1] = U[1 + q][1] + ra;
        U[1 + q][2] = U[1 + q][2] + rb;
    }
}

// TDdispFS (src/TD.jl:735-867) for one point.
template <class T>
void td_disp_fs(const TdFrame<T>& f, T X, T Y, T Z, T Dss, T Dds, T Dn, T nu, bool image, T U[3][3])
{
    T x, y, z;
    to_tdcs(f, X, Y, Z, x, y, z);
    const int mode = trimode(f, x, y, z);
    const bool detach = image && f.flat;
    T keep_z[3];
    if (image) {
        const T VxR[3] = {f.Vn[0], f.Vs[0], f.Vd[0]};
        const T VyR[3] = {f.Vn[1], f.Vs[1], f.Vd[1]};
        const T VzR[3] = {f.Vn[2], f.Vs[2], f.Vd[2]};
        for (int m = 0; m < 3; ++m)
            rot3(U[m][0], U[m][1], U[m][2], T(0.0), T(0.0), T(0.0), VxR, VyR, VzR, U[m][0], U[m][1], U[m][2]);
        if (detach) {
            // src/TD.jl:759-763: `UzDn = -UzDn` rebinds a local copy; the caller
            // keeps the TDCS-rotated z component.
            for (int m = 0; m < 3; ++m) {
                keep_z[m] = U[m][2];
                U[m][2] = -U[m][2];
            }
        }
    }
    T ne13[3], ne12[3], ne23[3];
    for (int i = 0; i < 3; ++i) { ne13[i] = -f.e13[i]; ne12[i] = -f.e12[i]; ne23[i] = -f.e23[i]; }
    if (mode == 1) {
        td_setup_d(x, y, z, f.A, Dn, Dss, Dds, nu, f.p1, ne13, U);
        td_setup_d(x, y, z, f.B, Dn, Dss, Dds, nu, f.p2, f.e12, U);
        td_setup_d(x, y, z, f.C, Dn, Dss, Dds, nu, f.p3, f.e23, U);
    } else if (mode == -1) {
        td_setup_d(x, y, z, f.A, Dn, Dss, Dds, nu, f.p1, f.e13, U);
        td_setup_d(x, y, z, f.B, Dn, Dss, Dds, nu, f.p2, ne12, U);
        td_setup_d(x, y, z, f.C, Dn, Dss, Dds, nu, f.p3, ne23, U);
    } else {
        const T nan = T(std::numeric_limits<double>::quiet_NaN());
        for (int m = 0; m < 3; ++m)
            for (int c = 0; c < 3; ++c) U[m][c] = nan;
    }
    // Burgers' function (solid angle) contribution, src/TD.jl:820-840
    {
        using std::atan2;
        const T a1 = -x, a2 = f.p1[1] - y, a3 = f.p1[2] - z;
        const T b1 = -x, b2 = -y, b3 = -z;
        const T c1 = -x, c2 = f.p3[1] - y, c3 = f.p3[2] - z;
        const T a12 = sq(a1);
        const T na = sqrt((a12 + sq(a2)) + sq(a3));
        const T nb = sqrt((a12 + sq(b2)) + sq(b3));
        const T nc = sqrt((a12 + sq(c2)) + sq(c3));
        const T one = ((a1 * ((b2 * c3) - (b3 * c2))) - (a2 * ((b1 * c3) - (b3 * c1)))) + (a3 * ((b1 * c2) - (b2 * c1)));
        const T ab = ((a1 * b1) + (a2 * b2)) + (a3 * b3);
        const T ac = ((a1 * c1) + (a2 * c2)) + (a3 * c3);
        const T bc = ((b1 * c1) + (b2 * c2)) + (b3 * c3);
        const T two = (((((na * nb) * nc) + (ab * nc)) + (ac * nb)) + (bc * na));
        const T Fi = (((-2.0) * atan2(one, two)) / 4.0) / T(M_PI);
        U[0][0] = (Dn * Fi) + U[0][0];
        U[1][1] = (Dss * Fi) + U[1][1];
        U[2][2] = (Dds * Fi) + U[2][2];
    }
    for (int m = 0; m < 3; ++m)
        rot3(U[m][0], U[m][1], U[m][2], T(0.0), T(0.0), T(0.0), f.Vn, f.Vs, f.Vd, U[m][0], U[m][1], U[m][2]);
    if (detach)
        for (int m = 0; m < 3; ++m) U[m][2] = keep_z[m];
}

// ------------------------------------------------- half-space corrections
// One TD side (PA -> PB) of the free-surface correction: side frame and
// skip test (CalcSideVec src/TD.jl:935-960, AngSetup*FSC :1267-1293, :1876-1908).
template <class T>
struct FscSide {
    bool skip;
    T beta, ey1[3], ey2[3], ey3[3], y1B, y2B, y3B, PA[3], PB[3];
};

template <class T>
void build_side(const T PA[3], const T PB[3], FscSide<T>& s)
{
    using std::acos;
    using std::fabs;
    using std::tan;
    for (int i = 0; i < 3; ++i) { s.PA[i] = PA[i]; s.PB[i] = PB[i]; }
    T S[3];
    for (int i = 0; i < 3; ++i) S[i] = PB[i] - PA[i];
    const T Sv = sqrt((sq(S[0]) + sq(S[1])) + sq(S[2]));
    T beta = (((-S[0]) * 0.0) - (S[1] * 0.0)) - (S[2] * 1.0);
    beta = acos(beta / Sv);
    s.beta = beta;
    const double eps = std::numeric_limits<double>::epsilon();
    s.skip = (fabs(beta) < eps) || (fabs(T(M_PI) - beta) < eps) || (fabs(T(1.0) / tan(beta)) > 5e3);
    if (s.skip) return;
    s.ey1[0] = S[0]; s.ey1[1] = S[1]; s.ey1[2] = T(0.0);
    const T nrm = sqrt((sq(s.ey1[0]) + sq(s.ey1[1])) + sq(s.ey1[2]));
    for (int i = 0; i < 3; ++i) s.ey1[i] = s.ey1[i] / nrm;
    s.ey3[0] = T(-0.0); s.ey3[1] = T(-0.0); s.ey3[2] = T(-1.0);
    cross3(s.ey3, s.ey1, s.ey2);
    rot3(S[0], S[1], S[2], T(0.0), T(0.0), T(0.0), s.ey1, s.ey2, s.ey3, s.y1B, s.y2B, s.y3B);
}

// AngSetupStrainFSC (src/TD.jl:1867-2081) for one point.
template <class T>
void fsc_strain_side(const FscSide<T>& s, const TdFrame<T>& f, T X, T Y, T Z, T Dss, T Dds, T Dn, T nu,
                     T E[3][6])
{
    if (s.skip) return;
    using std::cos;
    using std::sin;
    using std::tan;
    const T AFlip[9] = {s.ey1[0], s.ey1[1], s.ey1[2], s.ey2[0], s.ey2[1], s.ey2[2], s.ey3[0], s.ey3[1], s.ey3[2]};
    // slip TDCS -> EFCS -> ADCS, three unit modes
    T Dn1i, Dss0ni, Dds0n, Dn0ssi, Dss1i, Dds1ss, Dn0dsi, Dss0dsi, Dds1;
    rot3_noshift(Dn, T(0.0), T(0.0), f.Vn, f.Vs, f.Vd, Dn1i, Dss0ni, Dds0n);
    rot3_noshift(T(0.0), Dss, T(0.0), f.Vn, f.Vs, f.Vd, Dn0ssi, Dss1i, Dds1ss);
    rot3_noshift(T(0.0), T(0.0), Dds, f.Vn, f.Vs, f.Vd, Dn0dsi, Dss0dsi, Dds1);
    rot3_noshift(Dn1i, Dss0ni, Dds0n, s.ey1, s.ey2, s.ey3, Dn1i, Dss0ni, Dds0n);
    rot3_noshift(Dn0ssi, Dss1i, Dds1ss, s.ey1, s.ey2, s.ey3, Dn0ssi, Dss1i, Dds1ss);
    rot3_noshift(Dn0dsi, Dss0dsi, Dds1, s.ey1, s.ey2, s.ey3, Dn0dsi, Dss0dsi, Dds1);
    const T pib = T(M_PI) - s.beta;
    const T sinPib = sin(pib), cosPib = cos(pib), cotPib = T(1.0) / tan(pib);
    const T sinB = sin(s.beta), cosB = cos(s.beta), cotB = T(1.0) / tan(s.beta);

    T x, y, z;
    rot3(X, Y, Z, s.PA[0], s.PA[1], s.PA[2], s.ey1, s.ey2, s.ey3, x, y, z);
    const T Bx = s.beta * x;
    const bool flip = (Bx >= 0.0);
    T vA[18], vB[18];
    T c[3][3];   // c[m] = (first, second, third) ADCS slip for mode m
    if (flip) {
        ang_dis_strain_fsc(-x, -y, z, cosPib, sinPib, cotPib, nu, -s.PA[2], vA);
        for (int g = 0; g < 3; ++g) { vA[6 * g + 4] = -vA[6 * g + 4]; vA[6 * g + 5] = -vA[6 * g + 5]; }
        c[0][0] = -Dn1i;   c[0][1] = -Dss0ni;  c[0][2] = Dds0n;
        c[1][0] = -Dn0ssi; c[1][1] = -Dss1i;   c[1][2] = Dds1ss;
        c[2][0] = -Dn0dsi; c[2][1] = -Dss0dsi; c[2][2] = Dds1;
        ang_dis_strain_fsc((-x) + s.y1B, (-y) + s.y2B, z - s.y3B, cosPib, sinPib, cotPib, nu, -s.PB[2], vB);
        for (int g = 0; g < 3; ++g) { vB[6 * g + 4] = -vB[6 * g + 4]; vB[6 * g + 5] = -vB[6 * g + 5]; }
    } else {
        ang_dis_strain_fsc(x, y, z, cosB, sinB, cotB, nu, -s.PA[2], vA);
        c[0][0] = Dn1i;   c[0][1] = Dss0ni;  c[0][2] = Dds0n;
        c[1][0] = Dn0ssi; c[1][1] = Dss1i;   c[1][2] = Dds1ss;
        c[2][0] = Dn0dsi; c[2][1] = Dss0dsi; c[2][2] = Dds1;
        ang_dis_strain_fsc(x - s.y1B, y - s.y2B, z - s.y3B, cosB, sinB, cotB, nu, -s.PB[2], vB);
    }
    const T slip[3] = {Dn, Dss, Dds};
    for (int m = 0; m < 3; ++m) {
        if (!(slip[m] != 0.0)) continue;
        T t[6];
        // v arrays: index 6*g + k, g = slip component (x,y,z), k = 11,22,33,12,13,23
        for (int k = 0; k < 3; ++k)
            t[k] = -(((c[m][0] * vA[k]) + (c[m][1] * vA[6 + k])) + (c[m][2] * vA[12 + k]));
        for (int k = 3; k < 6; ++k)
            t[k] = -((((c[m][0] / 2.0) * vA[k]) + ((c[m][1] / 2.0) * vA[6 + k])) + ((c[m][2] / 2.0) * vA[12 + k]));
        for (int k = 0; k < 3; ++k)
            t[k] = t[k] + (((c[m][0] * vB[k]) + (c[m][1] * vB[6 + k])) + (c[m][2] * vB[12 + k]));
        for (int k = 3; k < 6; ++k)
            t[k] = t[k] + ((((c[m][0] / 2.0) * vB[k]) + ((c[m][1] / 2.0) * vB[6 + k])) + ((c[m][2] / 2.0) * vB[12 + k]));
        tensor_rot(t, AFlip);
        for (int k = 0; k < 6; ++k) E[m][k] = E[m][k] + t[k];
    }
}

// AngSetupDispFSC (src/TD.jl:1258-1409) for one point.
template <class T>
void fsc_disp_side(const FscSide<T>& s, const TdFrame<T>& f, T X, T Y, T Z, T Dss, T Dds, T Dn, T nu,
                   T U[3][3])
{
    if (s.skip) return;
    using std::cos;
    using std::sin;
    using std::tan;
    const T VxR[3] = {s.ey1[0], s.ey2[0], s.ey3[0]};
    const T VyR[3] = {s.ey1[1], s.ey2[1], s.ey3[1]};
    const T VzR[3] = {s.ey1[2], s.ey2[2], s.ey3[2]};
    T c[3][3];
    rot3_noshift(Dn, T(0.0), T(0.0), f.Vn, f.Vs, f.Vd, c[0][0], c[0][1], c[0][2]);
    rot3_noshift(T(0.0), Dss, T(0.0), f.Vn, f.Vs, f.Vd, c[1][0], c[1][1], c[1][2]);
    rot3_noshift(T(0.0), T(0.0), Dds, f.Vn, f.Vs, f.Vd, c[2][0], c[2][1], c[2][2]);
    for (int m = 0; m < 3; ++m)
        rot3(c[m][0], c[m][1], c[m][2], T(0.0), T(0.0), T(0.0), s.ey1, s.ey2, s.ey3, c[m][0], c[m][1], c[m][2]);
    const T pib = T(-M_PI) + s.beta;
    const T sinPib = sin(pib), cosPib = cos(pib), cotPib = T(1.0) / tan(pib), cotPib2 = T(1.0) / tan(pib / 2.0);
    const T b = s.beta;
    const T sinB = sin(b), cosB = cos(b), cotB = T(1.0) / tan(b), cotB2 = T(1.0) / tan(b / 2.0);

    T x, y, z;
    rot3(X, Y, Z, s.PA[0], s.PA[1], s.PA[2], s.ey1, s.ey2, s.ey3, x, y, z);
    const T Bx = s.beta * x;
    T uA[9], uB[9];
    if (Bx >= 0.0) {
        ang_dis_disp_fsc(x, y, z, cosPib, sinPib, cotPib, cotPib2, nu, -s.PA[2], uA);
        ang_dis_disp_fsc(x - s.y1B, y - s.y2B, z - s.y3B, cosPib, sinPib, cotPib, cotPib2, nu, -s.PB[2], uB);
    } else {
        ang_dis_disp_fsc(x, y, z, cosB, sinB, cotB, cotB2, nu, -s.PA[2], uA);
        ang_dis_disp_fsc(x - s.y1B, y - s.y2B, z - s.y3B, cosB, sinB, cotB, cotB2, nu, -s.PB[2], uB);
    }
    // returned order: ux,uy,uz,vx,vy,vz,wx,wy,wz; the slip component g scales
    // (u,v,w)_g and the displacement component is u (0), v (1), w (2).
    const T slip[3] = {Dn, Dss, Dds};
    for (int m = 0; m < 3; ++m) {
        if (!(slip[m] != 0.0)) continue;
        T k3[3];
        for (int g = 0; g < 3; ++g) k3[g] = ((c[m][g] / 4.0) / T(M_PI)) / (T(1.0) - nu);
        T u[3];
        for (int d = 0; d < 3; ++d)
            u[d] = -(((k3[0] * uA[3 * d + 0]) + (k3[1] * uA[3 * d + 1])) + (k3[2] * uA[3 * d + 2]));
        for (int d = 0; d < 3; ++d)
            u[d] = u[d] + (((k3[0] * uB[3 * d + 0]) + (k3[1] * uB[3 * d + 1])) + (k3[2] * uB[3 * d + 2]));
        rot3(u[0], u[1], u[2], T(0.0), T(0.0), T(0.0), VxR, VyR, VzR, u[0], u[1], u[2]);
        for (int d = 0; d < 3; ++d) U[m][d] = U[m][d] + u[d];
    }
}

// -------------------------------------------------------- per-pair drivers
// All of one triangle: real frame, image frame, three FSC sides.
template <class T>
struct TriangleState {
    TdFrame<T> real, image;
    FscSide<T> side[3];
};

template <class T>
void build_triangle(const T P1[3], const T P2[3], const T P3[3], TriangleState<T>& t)
{
    build_frame(P1, P2, P3, t.real);
    const T P1i[3] = {P1[0], P1[1], -P1[2]};
    const T P2i[3] = {P2[0], P2[1], -P2[2]};
    const T P3i[3] = {P3[0], P3[1], -P3[2]};
    build_frame(P1i, P2i, P3i, t.image);
    build_side(P1, P2, t.side[0]);
    build_side(P2, P3, t.side[1]);
    build_side(P3, P1, t.side[2]);
}

// ComputeStrainInfluences (src/TD.jl:670-708) for one pair: E[m][k] on exit.
template <class T>
void pair_strain(const TriangleState<T>& t, T X, T Y, T Z, T Dss, T Dds, T Dn, T nu, bool hs, T E[3][6])
{
    for (int m = 0; m < 3; ++m)
        for (int k = 0; k < 6; ++k) E[m][k] = T(0.0);
    td_strain_fs(t.real, X, Y, Z, Dss, Dds, Dn, nu, false, E);
    if (hs) {
        for (int s = 0; s < 3; ++s) fsc_strain_side(t.side[s], t.real, X, Y, Z, Dss, Dds, Dn, nu, E);
        td_strain_fs(t.image, X, Y, Z, Dss, Dds, Dn, nu, true, E);
    }
}

// ComputeDispInfluences (src/TD.jl:631-668) for one pair: U[m][c] on exit.
template <class T>
void pair_disp(const TriangleState<T>& t, T X, T Y, T Z, T Dss, T Dds, T Dn, T nu, bool hs, T U[3][3])
{
    for (int m = 0; m < 3; ++m)
        for (int c = 0; c < 3; ++c) U[m][c] = T(0.0);
    td_disp_fs(t.real, X, Y, Z, Dss, Dds, Dn, nu, false, U);
    if (hs) {
        for (int s = 0; s < 3; ++s) fsc_disp_side(t.side[s], t.real, X, Y, Z, Dss, Dds, Dn, nu, U);
        td_disp_fs(t.image, X, Y, Z, Dss, Dds, Dn, nu, true, U);
    }
}

}  // namespace cad_oracle
