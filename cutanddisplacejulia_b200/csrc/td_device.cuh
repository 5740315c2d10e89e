// Device-side triangular dislocation (TD) evaluation for one (observation,
// triangle) pair: full-space strain / displacement, the half-space free-surface
// correction and the image dislocation.
//
// Semantics follow the reference's per-point arithmetic in src/TD.jl:
//   frame + TDCS coordinates       CalculateLocalTriCoords! :712-732, GlobalToTDECoords :870-908
//   interior angles, side vectors  CalcTDVectsAndAngles :962-1008
//   configuration selection        trimodefinder :1010-1079
//   full-space strain / disp       TDstrainFS :1499-1620 + TDSetupS :1623-1750,
//                                  TDdispFS :735-867 + TDSetupD :1081-1173
//   free-surface correction        AngSetupStrainFSC :1867-2081, AngSetupDispFSC :1258-1409
//   image dislocation              ComputeStrainInfluences :670-708, ComputeDispInfluences :631-668
// The closed-form angular-dislocation terms come from tde_closed_form.cuh.
//
// Data layout: everything that depends only on the triangle (frames, angles,
// per-dislocation constants of every closed-form term, slip rotations) is
// computed once per triangle by td_setup_kernel into a TriDev record; the pair
// kernels stage one TriDev at a time in shared memory and every thread of the
// block (one observation point each) reads it as a broadcast.
#pragma once
#include <cfloat>
#include <cstddef>
#include <cstdint>

#include "tde_closed_form.cuh"

namespace cad {

// ------------------------------------------------------------------ records
// Every field of a record has the record's type T, so a record is a plain
// array of T: the FP32 copy used for far-field pairs is an element-wise
// conversion of the FP64 record (flags are stored as 0 / 1 values).
template <typename T>
struct AngDisT {         // one angular dislocation of a TD frame (configuration I)
    T cosT, sinT;        // side-vector z and y components; configuration II negates both
    T tv1, tv2;          // vertex y, z in TDCS
    T sinADE1;           // sin(alpha - pi) / (8 pi (1 - nu))
    ang_dis_strain_k<T> ks;
    ang_dis_disp_k<T> kd;
};

template <typename T>
struct FrameT {          // a TD (real or image) in its own coordinate system
    T P2[3];
    T P2lo[3];           // FP32 records: P2 - (double)(float)P2 (0 in FP64 records)
    T Vn[3], Vs[3], Vd[3];
    T p1y, p1z, p3y, p3z;           // TDCS (y, z) of P1 and P3; P2 is the origin
    T t23y, t32x, t31y, t13x, base; // configuration-test constants
    AngDisT<T> v[3];                // at P1 (side -e13), P2 (e12), P3 (e23)
    T flat;                         // 1: all vertex z exactly 0
};

template <typename T>
struct FscSideT {        // one TD side PA -> PB of the free-surface correction
    T skip;              // 1: the side adds nothing (beta test)
    T ey1[3], ey2[3], ey3[3];
    T PA[3];
    T PAlo[3];           // as P2lo
    T y1B, y2B, y3B;
    T beta;
    T cs[3][3];          // ADCS slip of each unit mode m (Dn, Dss, Dds), component g
    T cd[3][3];          // the same scaled by 1 / (4 pi (1 - nu)) for displacements
    ang_dis_strain_fsc_k<T> ks[2][2];   // [0: beta, 1: pi - beta][0: at PA, 1: at PB]
    ang_dis_disp_fsc_k<T> kd[2][2];     // [0: beta, 1: beta - pi][0: at PA, 1: at PB]
};

template <typename T>
struct TriDevT {
    T Dss, Dds, Dn;
    T K8;                // 1 / (8 pi (1 - nu))
    FrameT<T> real;
    FrameT<T> image;
    FscSideT<T> side[3];
};

using AngDis = AngDisT<double>;
using Frame = FrameT<double>;
using FscSide = FscSideT<double>;
using TriDev = TriDevT<double>;
static_assert(sizeof(TriDevT<float>) * 2 == sizeof(TriDevT<double>), "records are plain arrays of their type");

// Number of values of a record needed by a full-space-only kernel / in all.
constexpr int kTriWordsFS = (int)(offsetof(TriDev, image) / sizeof(double));
constexpr int kTriWordsHS = (int)(sizeof(TriDev) / sizeof(double));
constexpr int kTriWordsImg = (int)(offsetof(TriDev, side) / sizeof(double));   // real + image frames
constexpr int kSideWords = (int)(sizeof(FscSide) / sizeof(double));

// ------------------------------------------------------------------ helpers
template <typename R>
CAD_HD R qnan()
{
#ifdef __CUDA_ARCH__
    return (R)__longlong_as_double(0x7ff8000000000000LL);
#else
    return (R)__builtin_nan("");
#endif
}

// Unfused arithmetic for the quantities that feed exact comparisons (TDCS
// coordinates, barycentric configuration test, side test), so that those
// decisions match an unfused FP64 evaluation bit for bit.
CAD_HD double mul_rn(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    double r = a * b;
#if !defined(__CUDACC__) && defined(__GNUC__) && defined(__x86_64__)
    asm("" : "+x"(r));   // plain C++ test build: keep the product out of any fused multiply-add
#endif
    return r;
#endif
}
CAD_HD double add_rn(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
CAD_HD double sub_rn(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
CAD_HD float mul_rn(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    float r = a * b;
#if !defined(__CUDACC__) && defined(__GNUC__) && defined(__x86_64__)
    asm("" : "+x"(r));
#endif
    return r;
#endif
}
CAD_HD float add_rn(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
CAD_HD float sub_rn(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
template <typename R>
CAD_HD R dot3_rn(R a0, R a1, R a2, R b0, R b1, R b2)
{
    return add_rn(add_rn(mul_rn(a0, b0), mul_rn(a1, b1)), mul_rn(a2, b2));
}
CAD_HD double cad_atan2(double y, double x) { return atan2(y, x); }
CAD_HD float cad_atan2(float y, float x) { return atan2f(y, x); }

// Observation point minus a record origin, in R.  FP64 records subtract
// unfused; FP32 records subtract their origin's two float parts in FP64 and
// round the difference once.
template <typename R>
CAD_HD void rel_origin(const R* o, const R* olo, double X, double Y, double Z, R& dX, R& dY, R& dZ)
{
    if constexpr (sizeof(R) == sizeof(double)) {
        dX = sub_rn(X, (double)o[0]);
        dY = sub_rn(Y, (double)o[1]);
        dZ = sub_rn(Z, (double)o[2]);
    } else {
        dX = (R)((X - (double)o[0]) - (double)olo[0]);
        dY = (R)((Y - (double)o[1]) - (double)olo[1]);
        dZ = (R)((Z - (double)o[2]) - (double)olo[2]);
    }
}

// Symmetric tensor t (xx,yy,zz,xy,xz,yz) -> A-rotated, A column-major 3x3
// (TensorTransformation3D! form).
template <typename R>
CAD_HD void tensor_rot(R t[6], const R* A)
{
    const R two = R(2.0);
    const R Txx = t[0], Tyy = t[1], Tzz = t[2], Txy = t[3], Txz = t[4], Tyz = t[5];
    t[0] = A[0] * A[0] * Txx + two * A[0] * A[3] * Txy + two * A[0] * A[6] * Txz + two * A[3] * A[6] * Tyz +
           A[3] * A[3] * Tyy + A[6] * A[6] * Tzz;
    t[1] = A[1] * A[1] * Txx + two * A[1] * A[4] * Txy + two * A[1] * A[7] * Txz + two * A[4] * A[7] * Tyz +
           A[4] * A[4] * Tyy + A[7] * A[7] * Tzz;
    t[2] = A[2] * A[2] * Txx + two * A[2] * A[5] * Txy + two * A[2] * A[8] * Txz + two * A[5] * A[8] * Tyz +
           A[5] * A[5] * Tyy + A[8] * A[8] * Tzz;
    t[3] = A[0] * A[1] * Txx + (A[0] * A[4] + A[1] * A[3]) * Txy + (A[0] * A[7] + A[1] * A[6]) * Txz +
           (A[3] * A[7] + A[4] * A[6]) * Tyz + A[3] * A[4] * Tyy + A[6] * A[7] * Tzz;
    t[4] = A[0] * A[2] * Txx + (A[0] * A[5] + A[2] * A[3]) * Txy + (A[0] * A[8] + A[2] * A[6]) * Txz +
           (A[3] * A[8] + A[5] * A[6]) * Tyz + A[3] * A[5] * Tyy + A[6] * A[8] * Tzz;
    t[5] = A[1] * A[2] * Txx + (A[2] * A[4] + A[1] * A[5]) * Txy + (A[2] * A[7] + A[1] * A[8]) * Txz +
           (A[5] * A[7] + A[4] * A[8]) * Tyz + A[4] * A[5] * Tyy + A[7] * A[8] * Tzz;
}

// Rotation of a tensor about the TDCS x axis by the side angle (the B matrix
// [1 0 0; 0 c -s; 0 s c] of TDSetupS, stored column-major), written out.
template <typename R>
CAD_HD void tensor_rot_x(R t[6], R c, R s)
{
    const R Tyy = t[1], Tzz = t[2], Txy = t[3], Txz = t[4], Tyz = t[5];
    const R cc = c * c, ss = s * s, cs = c * s;
    t[1] = R(2.0) * cs * Tyz + cc * Tyy + ss * Tzz;
    t[2] = R(-2.0) * cs * Tyz + ss * Tyy + cc * Tzz;
    t[3] = c * Txy + s * Txz;
    t[4] = -s * Txy + c * Txz;
    t[5] = (cc - ss) * Tyz + cs * (Tzz - Tyy);
}

// Observation point -> TDCS of frame f.
template <typename R>
CAD_HD void to_tdcs(const FrameT<R>& f, double X, double Y, double Z, R& x, R& y, R& z)
{
    R dX, dY, dZ;
    rel_origin(f.P2, f.P2lo, X, Y, Z, dX, dY, dZ);
    x = dot3_rn(f.Vn[0], f.Vn[1], f.Vn[2], dX, dY, dZ);
    y = dot3_rn(f.Vs[0], f.Vs[1], f.Vs[2], dX, dY, dZ);
    z = dot3_rn(f.Vd[0], f.Vd[1], f.Vd[2], dX, dY, dZ);
}

// Artefact-free configuration: +1 (I), -1 (II), 0 (on a side, in the TD plane).
template <typename R>
CAD_HD int trimode(const FrameT<R>& f, R x, R y, R z)
{
    const R dy = sub_rn(y, f.p3y), dz = sub_rn(z, f.p3z);
    const R a = add_rn(mul_rn(f.t23y, dy), mul_rn(f.t32x, dz)) / f.base;
    const R b = add_rn(mul_rn(f.t31y, dy), mul_rn(f.t13x, dz)) / f.base;
    const R c = sub_rn(sub_rn(R(1.0), a), b);
    bool casen = false, casez = false;
    if (a <= 0.0 && b > c && c > a) casen = true;
    else if (b <= 0.0 && c > a && a > b) casen = true;
    else if (c <= 0.0 && a > b && b > c) casen = true;
    else if (a == 0.0 && b >= 0.0 && c >= 0.0) casez = true;
    else if (a >= 0.0 && b == 0.0 && c >= 0.0) casez = true;
    else if (a >= 0.0 && b >= 0.0 && c == 0.0) casez = true;
    if (casez && x != 0.0) casez = false;
    return casez ? 0 : (casen ? -1 : 1);
}

// ------------------------------------------------------ full-space strain
// One angular dislocation's contribution for all three unit modes, added to
// E[m][k] (TDCS).  sgn = +1 for configuration I, -1 for II.
template <typename R>
CAD_HD void ad_strain(const AngDisT<R>& v, R sgn, R x, R y, R z, R Dss, R Dds, R Dn, R K8, R E[3][6])
{
    const R CosT = sgn * v.cosT, SinT = sgn * v.sinT;
    const R dy = y - v.tv1, dz = z - v.tv2;
    const R Yr = CosT * dy - SinT * dz;
    const R Zr = SinT * dy + CosT * dz;
    R o[21];
    ang_dis_strain(v.ks, x, Yr, Zr, o);
    const R exxBx = o[0], exxBy = o[1], exxBz = o[2];
    const R eyyBx = o[3], eyyBy = o[4], eyyBz = o[5];
    const R ezzBx = o[6], ezzBy = o[7], ezzBz = o[8];
    const R exyBx = o[9], exyBy = o[10], exyBz = o[11];
    const R exzBx = o[12], exzBy = o[13], exzBz = o[14];
    const R eyzBx = o[15], eyzBy = o[16], eyzBz = o[17];
    const R rFx = o[18], rFy = o[19], rFz = o[20];
    const R sinADE1 = v.sinADE1;
    if (Dn != 0.0) {
        const R E3 = Dn * K8;
        R t[6];
        t[0] = Dn * rFx + E3 * exxBx;
        t[1] = E3 * eyyBx;
        t[2] = E3 * ezzBx;
        t[3] = R(0.5) * Dn * rFy - E3 * exyBx;
        t[4] = R(0.5) * Dn * rFz - E3 * exzBx;
        t[5] = E3 * eyzBx;
        tensor_rot_x(t, CosT, SinT);
#pragma unroll
        for (int k = 0; k < 6; ++k) E[0][k] += t[k];
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const R slip = q == 0 ? Dss : Dds;
        if (!(slip != 0.0)) continue;
        // in-plane slip (strike, dip) of this mode in ADCS
        const R Ds = q == 0 ? CosT * Dss : -SinT * Dds;
        const R Dd = q == 0 ? SinT * Dss : CosT * Dds;
        const R E5 = Ds * K8;
        const R E4 = E5 * x;
        const R dsa = Dd * sinADE1;
        const R dsax = dsa * x;
        R t[6];
        t[0] = -E4 * exxBy + dsax * exxBz;
        t[1] = Ds * rFy - E4 * eyyBy + dsax * eyyBz;
        t[2] = -E4 * ezzBy + Dd * rFz + dsax * ezzBz;
        t[3] = R(0.5) * Ds * rFx + E5 * exyBy - dsa * exyBz;
        t[4] = E5 * exzBy + R(0.5) * Dd * rFx - dsa * exzBz;
        t[5] = R(0.5) * Ds * rFz - E4 * eyzBy + R(0.5) * Dd * rFy - dsax * eyzBz;
        tensor_rot_x(t, CosT, SinT);
#pragma unroll
        for (int k = 0; k < 6; ++k) E[1 + q][k] += t[k];
    }
}

// Full-space strain of frame f at one point, added into E (EFCS).  For the
// image frame the accumulated value is first carried into the image TDCS and
// the result carried back, as the reference does; a flat (z = 0) image
// triangle keeps the reference's detached xz / yz components.
template <bool IMAGE, typename R>
CAD_HD void strain_fs(const FrameT<R>& f, double X, double Y, double Z, R Dss, R Dds, R Dn, R K8, R E[3][6])
{
    R x, y, z;
    to_tdcs(f, X, Y, Z, x, y, z);
    const int mode = trimode(f, x, y, z);
    R keep_xz[3], keep_yz[3];
    const bool detach = IMAGE && f.flat != R(0);
    if (IMAGE) {
        const R RotInv[9] = {f.Vn[0], f.Vs[0], f.Vd[0], f.Vn[1], f.Vs[1], f.Vd[1], f.Vn[2], f.Vs[2], f.Vd[2]};
#pragma unroll
        for (int m = 0; m < 3; ++m) tensor_rot(E[m], RotInv);
        if (detach) {
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                keep_xz[m] = E[m][4];
                keep_yz[m] = E[m][5];
                E[m][4] = -E[m][4];
                E[m][5] = -E[m][5];
            }
        }
    }
    const R sgn = mode == -1 ? R(-1.0) : R(1.0);
#pragma unroll 1
    for (int a = 0; a < 3; ++a) ad_strain(f.v[a], sgn, x, y, z, Dss, Dds, Dn, K8, E);
    if (mode == 0) {
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int k = 0; k < 6; ++k) E[m][k] = qnan<R>();
    }
    const R Rot[9] = {f.Vn[0], f.Vn[1], f.Vn[2], f.Vs[0], f.Vs[1], f.Vs[2], f.Vd[0], f.Vd[1], f.Vd[2]};
#pragma unroll
    for (int m = 0; m < 3; ++m) tensor_rot(E[m], Rot);
    if (detach) {
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            E[m][4] = keep_xz[m];
            E[m][5] = keep_yz[m];
        }
    }
}

// -------------------------------------------------- full-space displacement
template <typename R>
CAD_HD void ad_disp(const AngDisT<R>& v, R sgn, R x, R y, R z, R Dss, R Dds, R Dn, R K8, R U[3][3])
{
    const R CosT = sgn * v.cosT, SinT = sgn * v.sinT;
    const R dy = y - v.tv1, dz = z - v.tv2;
    const R Yr = CosT * dy - SinT * dz;
    const R Zr = SinT * dy + CosT * dz;
    R o[9];
    ang_dis_disp(v.kd, x, Yr, Zr, o);
    const R ux = o[0], uy = o[1], uz = o[2], vx = o[3], vy = o[4], vz = o[5], wx = o[6], wy = o[7], wz = o[8];
    const R sinADE1 = v.sinADE1;
    // back-rotation of (y, z) components: (c u + s w, -s u + c w)
    if (Dn != 0.0) {
        const R c = Dn * K8;
        const R a = c * vx, b = c * wx;
        U[0][0] += c * ux;
        U[0][1] += CosT * a + SinT * b;
        U[0][2] += -SinT * a + CosT * b;
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const R slip = q == 0 ? Dss : Dds;
        if (!(slip != 0.0)) continue;
        const R Ds = q == 0 ? CosT * Dss : -SinT * Dds;
        const R Dd = q == 0 ? SinT * Dss : CosT * Dds;
        const R cs = Ds * K8, cd = Dd * sinADE1;
        const R a = x * (cs * vy + cd * vz);
        const R b = x * (cs * wy + cd * wz);
        U[1 + q][0] += cs * uy + cd * uz;
        U[1 + q][1] += CosT * a + SinT * b;
        U[1 + q][2] += -SinT * a + CosT * b;
    }
}

template <bool IMAGE, typename R>
CAD_HD void disp_fs(const FrameT<R>& f, double X, double Y, double Z, R Dss, R Dds, R Dn, R K8, R U[3][3])
{
    R x, y, z;
    to_tdcs(f, X, Y, Z, x, y, z);
    const int mode = trimode(f, x, y, z);
    const bool detach = IMAGE && f.flat != R(0);
    R keep_z[3];
    if (IMAGE) {
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            const R a = U[m][0], b = U[m][1], c = U[m][2];
            U[m][0] = f.Vn[0] * a + f.Vn[1] * b + f.Vn[2] * c;
            U[m][1] = f.Vs[0] * a + f.Vs[1] * b + f.Vs[2] * c;
            U[m][2] = f.Vd[0] * a + f.Vd[1] * b + f.Vd[2] * c;
        }
        if (detach) {
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                keep_z[m] = U[m][2];
                U[m][2] = -U[m][2];
            }
        }
    }
    const R sgn = mode == -1 ? R(-1.0) : R(1.0);
#pragma unroll 1
    for (int a = 0; a < 3; ++a) ad_disp(f.v[a], sgn, x, y, z, Dss, Dds, Dn, K8, U);
    if (mode == 0) {
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
            for (int c = 0; c < 3; ++c) U[m][c] = qnan<R>();
    }
    {   // Burgers' function (solid angle of the TD seen from the point)
        const R a1 = -x, a2 = f.p1y - y, a3 = f.p1z - z;
        const R b2 = -y, b3 = -z;
        const R c2 = f.p3y - y, c3 = f.p3z - z;
        const R a12 = a1 * a1;
        const R na = cad_sqrt(a12 + a2 * a2 + a3 * a3);
        const R nb = cad_sqrt(a12 + b2 * b2 + b3 * b3);
        const R nc = cad_sqrt(a12 + c2 * c2 + c3 * c3);
        const R one = a1 * (b2 * c3 - b3 * c2) - a2 * (a1 * c3 - b3 * a1) + a3 * (a1 * c2 - b2 * a1);
        const R ab = a1 * a1 + a2 * b2 + a3 * b3;
        const R ac = a1 * a1 + a2 * c2 + a3 * c3;
        const R bc = a1 * a1 + b2 * c2 + b3 * c3;
        const R two = na * nb * nc + ab * nc + ac * nb + bc * na;
        const R Fi = R(-0.5) * R(M_1_PI) * cad_atan2(one, two);
        U[0][0] += Dn * Fi;
        U[1][1] += Dss * Fi;
        U[2][2] += Dds * Fi;
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const R a = U[m][0], b = U[m][1], c = U[m][2];
        U[m][0] = f.Vn[0] * a + f.Vs[0] * b + f.Vd[0] * c;
        U[m][1] = f.Vn[1] * a + f.Vs[1] * b + f.Vd[1] * c;
        U[m][2] = f.Vn[2] * a + f.Vs[2] * b + f.Vd[2] * c;
    }
    if (detach) {
#pragma unroll
        for (int m = 0; m < 3; ++m) U[m][2] = keep_z[m];
    }
}

// --------------------------------------------------- free-surface correction
// Observation point -> ADCS of a side, relative to PA.
template <typename R>
CAD_HD void to_adcs(const FscSideT<R>& s, double X, double Y, double Z, R& x, R& y, R& z)
{
    R dX, dY, dZ;
    rel_origin(s.PA, s.PAlo, X, Y, Z, dX, dY, dZ);
    x = add_rn(add_rn(mul_rn(s.ey1[0], dX), mul_rn(s.ey2[0], dY)), mul_rn(s.ey3[0], dZ));
    y = add_rn(add_rn(mul_rn(s.ey1[1], dX), mul_rn(s.ey2[1], dY)), mul_rn(s.ey3[1], dZ));
    z = add_rn(add_rn(mul_rn(s.ey1[2], dX), mul_rn(s.ey2[2], dY)), mul_rn(s.ey3[2], dZ));
}

// The FP64 free-surface strain groups are called out of line: each then gets
// the whole register file, which spills far less than one inlined body (the
// FP32 groups fit inline).
#ifdef __CUDACC__
#define CAD_OUTLINE static __host__ __device__ __noinline__
#else
#define CAD_OUTLINE static inline
#endif
CAD_OUTLINE void fsc_strain_g0_f64(const ang_dis_strain_fsc_k<double>& k, double y1, double y2, double y3, double* v)
{
    ang_dis_strain_fsc_g0(k, y1, y2, y3, v);
}
CAD_OUTLINE void fsc_strain_g1_f64(const ang_dis_strain_fsc_k<double>& k, double y1, double y2, double y3, double* v)
{
    ang_dis_strain_fsc_g1(k, y1, y2, y3, v);
}
CAD_OUTLINE void fsc_strain_g2_f64(const ang_dis_strain_fsc_k<double>& k, double y1, double y2, double y3, double* v)
{
    ang_dis_strain_fsc_g2(k, y1, y2, y3, v);
}

template <typename R>
CAD_HD void fsc_strain_eval(const ang_dis_strain_fsc_k<R>& k, R y1, R y2, R y3, R v[18])
{
    if constexpr (sizeof(R) == sizeof(double)) {
        fsc_strain_g0_f64(k, y1, y2, y3, v);
        fsc_strain_g1_f64(k, y1, y2, y3, v + 6);
        fsc_strain_g2_f64(k, y1, y2, y3, v + 12);
    } else {
        ang_dis_strain_fsc_g0(k, y1, y2, y3, v);
        ang_dis_strain_fsc_g1(k, y1, y2, y3, v + 6);
        ang_dis_strain_fsc_g2(k, y1, y2, y3, v + 12);
    }
}

// One side's harmonic correction to the strain, added into E (EFCS).
template <typename R>
CAD_HD void fsc_strain(const FscSideT<R>& s, double X, double Y, double Z, R Dss, R Dds, R Dn, R E[3][6])
{
    R x, y, z;
    to_adcs(s, X, Y, Z, x, y, z);
    const bool flip = mul_rn(s.beta, x) >= 0.0;
    const int c = flip ? 1 : 0;
    const R f = flip ? R(-1.0) : R(1.0);
    // d = (term at PB) - (term at PA), formed before any slip product: far
    // from the side the two terms nearly cancel, and differencing them first
    // keeps the products from rounding the two halves differently.
    R d[18];
    fsc_strain_eval(s.ks[c][0], f * x, f * y, z, d);
#pragma unroll
    for (int q = 0; q < 18; ++q) d[q] = -d[q];
    {
        R v[18];
        fsc_strain_eval(s.ks[c][1], f * (x - s.y1B), f * (y - s.y2B), z - s.y3B, v);
#pragma unroll
        for (int q = 0; q < 18; ++q) d[q] += v[q];
    }
    R T[3][6];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        // configuration flip negates the first two ADCS slip components and
        // the 13 / 23 strain components
        const R c0 = f * s.cs[m][0], c1 = f * s.cs[m][1], c2 = s.cs[m][2];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const R fk = (k >= 4) ? f : R(1.0);
            const R h = (k >= 3) ? R(0.5) : R(1.0);
            T[m][k] = h * fk * (c0 * d[k] + c1 * d[6 + k] + c2 * d[12 + k]);
        }
    }
    const R AFlip[9] = {s.ey1[0], s.ey1[1], s.ey1[2], s.ey2[0], s.ey2[1], s.ey2[2], s.ey3[0], s.ey3[1], s.ey3[2]};
    const R slip[3] = {Dn, Dss, Dds};
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        if (!(slip[m] != 0.0)) continue;
        tensor_rot(T[m], AFlip);
#pragma unroll
        for (int k = 0; k < 6; ++k) E[m][k] += T[m][k];
    }
}

// The same correction as a linear map of the side's Burgers vector: G[j] is
// the EFCS strain of a unit Burgers vector along EFCS axis j.  A side shared
// by two triangles is traversed in opposite directions, and the reversed
// side's map is the negative of this one (the two dislocation segments
// cancel), so one evaluation per mesh edge serves both triangles.
template <typename R>
CAD_HD void fsc_strain_map(const FscSideT<R>& s, double X, double Y, double Z, R G[3][6])
{
    R x, y, z;
    to_adcs(s, X, Y, Z, x, y, z);
    const bool flip = mul_rn(s.beta, x) >= 0.0;
    const int c = flip ? 1 : 0;
    const R f = flip ? R(-1.0) : R(1.0);
    R d[18];
    fsc_strain_eval(s.ks[c][0], f * x, f * y, z, d);
#pragma unroll
    for (int q = 0; q < 18; ++q) d[q] = -d[q];
    {
        R v[18];
        fsc_strain_eval(s.ks[c][1], f * (x - s.y1B), f * (y - s.y2B), z - s.y3B, v);
#pragma unroll
        for (int q = 0; q < 18; ++q) d[q] += v[q];
    }
    const R AFlip[9] = {s.ey1[0], s.ey1[1], s.ey1[2], s.ey2[0], s.ey2[1], s.ey2[2], s.ey3[0], s.ey3[1], s.ey3[2]};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        // ADCS slip components of a unit Burgers vector along EFCS axis j (as
        // build_side forms them: the j-th frame vector ey(j+1))
        const R c0 = f * AFlip[3 * j], c1 = f * AFlip[3 * j + 1], c2 = AFlip[3 * j + 2];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const R fk = (k >= 4) ? f : R(1.0);
            const R h = (k >= 3) ? R(0.5) : R(1.0);
            G[j][k] = h * fk * (c0 * d[k] + c1 * d[6 + k] + c2 * d[12 + k]);
        }
        tensor_rot(G[j], AFlip);
    }
}

// E[m] += sign * (the map G applied to the EFCS Burgers vector of unit mode m
// of the triangle with frame `real`), for the modes with non-zero slip.
template <typename R>
CAD_HD void fsc_apply_map(const R G[3][6], R sign, const FrameT<R>& real, R Dss, R Dds, R Dn, R E[3][6])
{
    const R slip[3] = {Dn, Dss, Dds};
    const R* axes[3] = {real.Vn, real.Vs, real.Vd};
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        if (!(slip[m] != 0.0)) continue;
        const R w0 = sign * axes[m][0] * slip[m], w1 = sign * axes[m][1] * slip[m], w2 = sign * axes[m][2] * slip[m];
#pragma unroll
        for (int k = 0; k < 6; ++k) E[m][k] += w0 * G[0][k] + w1 * G[1][k] + w2 * G[2][k];
    }
}

// One side's harmonic correction to the displacement, added into U (EFCS).
template <typename R>
CAD_HD void fsc_disp(const FscSideT<R>& s, double X, double Y, double Z, R Dss, R Dds, R Dn, R U[3][3])
{
    R x, y, z;
    to_adcs(s, X, Y, Z, x, y, z);
    const int c = mul_rn(s.beta, x) >= 0.0 ? 1 : 0;
    R uA[9], uB[9];
    ang_dis_disp_fsc(s.kd[c][0], x, y, z, uA);
    ang_dis_disp_fsc(s.kd[c][1], x - s.y1B, y - s.y2B, z - s.y3B, uB);
    const R slip[3] = {Dn, Dss, Dds};
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        if (!(slip[m] != 0.0)) continue;
        R u[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            u[d] = s.cd[m][0] * (uB[3 * d] - uA[3 * d]) + s.cd[m][1] * (uB[3 * d + 1] - uA[3 * d + 1]) +
                   s.cd[m][2] * (uB[3 * d + 2] - uA[3 * d + 2]);
        // ADCS -> EFCS: rows (ey1, ey2, ey3) as in the reference's VxR, VyR, VzR
        U[m][0] += s.ey1[0] * u[0] + s.ey1[1] * u[1] + s.ey1[2] * u[2];
        U[m][1] += s.ey2[0] * u[0] + s.ey2[1] * u[1] + s.ey2[2] * u[2];
        U[m][2] += s.ey3[0] * u[0] + s.ey3[1] * u[1] + s.ey3[2] * u[2];
    }
}

// The free-surface displacement of side s at (X, Y, Z) for a unit Burgers
// vector along EFCS axis j, without the factor 1 / (4 pi (1 - nu)):
// Gu[j][c] = sum_d ey_c[d] sum_g ey_j[g] (uB - uA)[3 d + g] (fsc_disp with
// cs = ey_j).  As for the strain map, the reversed side's map is the
// negative of this one.
template <typename R>
CAD_HD void fsc_disp_map(const FscSideT<R>& s, double X, double Y, double Z, R Gu[3][3])
{
    R x, y, z;
    to_adcs(s, X, Y, Z, x, y, z);
    const int c = mul_rn(s.beta, x) >= 0.0 ? 1 : 0;
    R uA[9], uB[9];
    ang_dis_disp_fsc(s.kd[c][0], x, y, z, uA);
    ang_dis_disp_fsc(s.kd[c][1], x - s.y1B, y - s.y2B, z - s.y3B, uB);
    const R* ey[3] = {s.ey1, s.ey2, s.ey3};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        R u[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            u[d] = ey[j][0] * (uB[3 * d] - uA[3 * d]) + ey[j][1] * (uB[3 * d + 1] - uA[3 * d + 1]) +
                   ey[j][2] * (uB[3 * d + 2] - uA[3 * d + 2]);
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) Gu[j][cc] = ey[cc][0] * u[0] + ey[cc][1] * u[1] + ey[cc][2] * u[2];
    }
}

// U[m] += sign * 2 K8 * (the map Gu applied to the EFCS Burgers vector of
// unit mode m of the triangle with frame `real`), for the modes with
// non-zero slip (2 K8 = 1 / (4 pi (1 - nu))).
template <typename R>
CAD_HD void fsc_apply_disp_map(const R Gu[3][3], R sign, const FrameT<R>& real, R Dss, R Dds, R Dn, R K8, R U[3][3])
{
    const R slip[3] = {Dn, Dss, Dds};
    const R* axes[3] = {real.Vn, real.Vs, real.Vd};
    const R f = sign * (K8 + K8);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        if (!(slip[m] != 0.0)) continue;
        const R w0 = axes[m][0] * slip[m], w1 = axes[m][1] * slip[m], w2 = axes[m][2] * slip[m];
#pragma unroll
        for (int c = 0; c < 3; ++c) U[m][c] += f * (w0 * Gu[0][c] + w1 * Gu[1][c] + w2 * Gu[2][c]);
    }
}

// -------------------------------------------------------- triangle setup
// The per-triangle setup uses unfused arithmetic throughout: it is negligible
// work, and the half-space terms of the two ends of a side cancel far from the
// side, which amplifies any inconsistency between the side angle beta and the
// side vector (fused rounding of |S| alone is enough to show).
CAD_HD double sq_rn(double a) { return mul_rn(a, a); }
CAD_HD double norm3_rn(double a, double b, double c) { return sqrt(add_rn(add_rn(sq_rn(a), sq_rn(b)), sq_rn(c))); }
CAD_HD void cross3_rn(const double a[3], const double b[3], double c[3])
{
    c[0] = sub_rn(mul_rn(a[1], b[2]), mul_rn(a[2], b[1]));
    c[1] = sub_rn(mul_rn(a[2], b[0]), mul_rn(a[0], b[2]));
    c[2] = sub_rn(mul_rn(a[0], b[1]), mul_rn(a[1], b[0]));
}

CAD_HD void build_frame(const double P1[3], const double P2[3], const double P3[3], double nu, Frame& f)
{
    double a[3], b[3], Vn[3], Vs[3], Vd[3];
    for (int i = 0; i < 3; ++i) { a[i] = sub_rn(P2[i], P1[i]); b[i] = sub_rn(P3[i], P1[i]); }
    cross3_rn(a, b, Vn);
    const double nn = norm3_rn(Vn[0], Vn[1], Vn[2]);
    for (int i = 0; i < 3; ++i) Vn[i] = Vn[i] / nn;
    const double eZ[3] = {0.0, 0.0, 1.0};
    cross3_rn(eZ, Vn, Vs);
    if (Vs[0] == 0.0 && Vs[1] == 0.0 && Vs[2] == 0.0) {   // horizontal TD
        Vs[0] = mul_rn(0.0, Vn[2]);
        Vs[1] = mul_rn(1.0, Vn[2]);
        Vs[2] = mul_rn(0.0, Vn[2]);
    }
    const double ns = norm3_rn(Vs[0], Vs[1], Vs[2]);
    for (int i = 0; i < 3; ++i) Vs[i] = Vs[i] / ns;
    cross3_rn(Vn, Vs, Vd);
    for (int i = 0; i < 3; ++i) { f.P2[i] = P2[i]; f.Vn[i] = Vn[i]; f.Vs[i] = Vs[i]; f.Vd[i] = Vd[i]; }

    double p1[3], p3[3];
    {
        const double d1[3] = {sub_rn(P1[0], P2[0]), sub_rn(P1[1], P2[1]), sub_rn(P1[2], P2[2])};
        const double d3[3] = {sub_rn(P3[0], P2[0]), sub_rn(P3[1], P2[1]), sub_rn(P3[2], P2[2])};
        p1[0] = dot3_rn(Vn[0], Vn[1], Vn[2], d1[0], d1[1], d1[2]);
        p1[1] = dot3_rn(Vs[0], Vs[1], Vs[2], d1[0], d1[1], d1[2]);
        p1[2] = dot3_rn(Vd[0], Vd[1], Vd[2], d1[0], d1[1], d1[2]);
        p3[0] = dot3_rn(Vn[0], Vn[1], Vn[2], d3[0], d3[1], d3[2]);
        p3[1] = dot3_rn(Vs[0], Vs[1], Vs[2], d3[0], d3[1], d3[2]);
        p3[2] = dot3_rn(Vd[0], Vd[1], Vd[2], d3[0], d3[1], d3[2]);
    }
    f.p1y = p1[1]; f.p1z = p1[2]; f.p3y = p3[1]; f.p3z = p3[2];
    double e12[3], e13[3], e23[3];
    for (int i = 0; i < 3; ++i) { e12[i] = sub_rn(0.0, p1[i]); e13[i] = sub_rn(p3[i], p1[i]); e23[i] = sub_rn(p3[i], 0.0); }
    const double n12 = norm3_rn(e12[0], e12[1], e12[2]);
    const double n13 = norm3_rn(e13[0], e13[1], e13[2]);
    const double n23 = norm3_rn(e23[0], e23[1], e23[2]);
    for (int i = 0; i < 3; ++i) { e12[i] /= n12; e13[i] /= n13; e23[i] /= n23; }
    const double A = acos(dot3_rn(e12[0], e12[1], e12[2], e13[0], e13[1], e13[2]));
    const double B = acos(dot3_rn(-e12[0], -e12[1], -e12[2], e23[0], e23[1], e23[2]));
    const double C = acos(dot3_rn(e23[0], e23[1], e23[2], e13[0], e13[1], e13[2]));

    // configuration test constants (trimodefinder on the TDCS (y, z) plane)
    f.t23y = sub_rn(0.0, p3[2]);
    f.t32x = sub_rn(p3[1], 0.0);
    f.t13x = sub_rn(p1[1], p3[1]);
    const double t13y = sub_rn(p1[2], p3[2]);
    f.t31y = sub_rn(p3[2], p1[2]);
    f.base = add_rn(mul_rn(f.t23y, f.t13x), mul_rn(f.t32x, t13y));

    const double alpha[3] = {A, B, C};
    const double side_y[3] = {-e13[1], e12[1], e23[1]};
    const double side_z[3] = {-e13[2], e12[2], e23[2]};
    const double tv1[3] = {p1[1], 0.0, p3[1]};
    const double tv2[3] = {p1[2], 0.0, p3[2]};
    for (int v = 0; v < 3; ++v) {
        AngDis& d = f.v[v];
        d.cosT = side_z[v];
        d.sinT = side_y[v];
        d.tv1 = tv1[v];
        d.tv2 = tv2[v];
        const double Ang = -M_PI + alpha[v];
        const double cosA = cos(Ang), sinA = sin(Ang);
        d.sinADE1 = sinA / 8.0 / M_PI / sub_rn(1.0, nu);
        ang_dis_strain_setup(cosA, sinA, nu, add_rn(mul_rn(2.0, nu), 1.0), d.sinADE1, d.ks);
        ang_dis_disp_setup(cosA, sinA, sub_rn(1.0, nu), sub_rn(1.0, mul_rn(2.0, nu)), mul_rn(cosA, cosA), d.sinADE1,
                           d.kd);
    }
    f.flat = (P1[2] == 0.0 && P2[2] == 0.0 && P3[2] == 0.0) ? 1.0 : 0.0;
    for (int i = 0; i < 3; ++i) f.P2lo[i] = 0.0;
}

// The geometry of side PA -> PB (frame, beta test, closed-form constants);
// its slip coefficients cs, cd are left zero.
CAD_HD void build_side_geom(const double PA[3], const double PB[3], double nu, FscSide& s)
{
    for (int m = 0; m < 3; ++m)
        for (int g = 0; g < 3; ++g) s.cs[m][g] = s.cd[m][g] = 0.0;
    const double S[3] = {sub_rn(PB[0], PA[0]), sub_rn(PB[1], PA[1]), sub_rn(PB[2], PA[2])};
    const double Sv = norm3_rn(S[0], S[1], S[2]);
    const double beta = acos(-S[2] / Sv);
    s.beta = beta;
    s.skip = ((fabs(beta) < DBL_EPSILON) || (fabs(M_PI - beta) < DBL_EPSILON) || (fabs(1.0 / tan(beta)) > 5e3)) ? 1.0 : 0.0;
    for (int i = 0; i < 3; ++i) { s.PA[i] = PA[i]; s.PAlo[i] = 0.0; }
    if (s.skip != 0.0) return;
    const double n1 = norm3_rn(S[0], S[1], 0.0);
    const double e1[3] = {S[0] / n1, S[1] / n1, 0.0 / n1};
    const double e3[3] = {-0.0, -0.0, -1.0};
    double e2[3];
    cross3_rn(e3, e1, e2);
    for (int i = 0; i < 3; ++i) { s.ey1[i] = e1[i]; s.ey2[i] = e2[i]; s.ey3[i] = e3[i]; }
    s.y1B = add_rn(add_rn(mul_rn(e1[0], S[0]), mul_rn(e2[0], S[1])), mul_rn(e3[0], S[2]));
    s.y2B = add_rn(add_rn(mul_rn(e1[1], S[0]), mul_rn(e2[1], S[1])), mul_rn(e3[1], S[2]));
    s.y3B = add_rn(add_rn(mul_rn(e1[2], S[0]), mul_rn(e2[2], S[1])), mul_rn(e3[2], S[2]));
    const double a_end[2] = {-PA[2], -PB[2]};
    const double pibs = M_PI - beta, pibd = -M_PI + beta;
    for (int e = 0; e < 2; ++e) {
        ang_dis_strain_fsc_setup(cos(beta), sin(beta), 1.0 / tan(beta), nu, a_end[e], s.ks[0][e]);
        ang_dis_strain_fsc_setup(cos(pibs), sin(pibs), 1.0 / tan(pibs), nu, a_end[e], s.ks[1][e]);
        ang_dis_disp_fsc_setup(cos(beta), sin(beta), 1.0 / tan(beta), 1.0 / tan(beta / 2.0), nu, a_end[e],
                               s.kd[0][e]);
        ang_dis_disp_fsc_setup(cos(pibd), sin(pibd), 1.0 / tan(pibd), 1.0 / tan(pibd / 2.0), nu, a_end[e],
                               s.kd[1][e]);
    }
}

CAD_HD void build_side(const double PA[3], const double PB[3], const Frame& real, double Dss, double Dds,
                       double Dn, double nu, FscSide& s)
{
    build_side_geom(PA, PB, nu, s);
    if (s.skip != 0.0) return;
    // unit-mode slip vectors: TDCS (n, s, d) -> EFCS -> ADCS
    const double slip[3] = {Dn, Dss, Dds};
    const double* axes[3] = {real.Vn, real.Vs, real.Vd};
    for (int m = 0; m < 3; ++m) {
        double w[3];
        for (int i = 0; i < 3; ++i) w[i] = mul_rn(axes[m][i], slip[m]);
        for (int g = 0; g < 3; ++g) {
            s.cs[m][g] = add_rn(add_rn(mul_rn(s.ey1[g], w[0]), mul_rn(s.ey2[g], w[1])), mul_rn(s.ey3[g], w[2]));
            s.cd[m][g] = s.cs[m][g] / 4.0 / M_PI / sub_rn(1.0, nu);
        }
    }
}

// Side PA -> PB carrying the net Burgers vector B (EFCS) of every triangle side
// on that mesh edge, as unit mode 0 (evaluate with Dn = 1, Dss = Dds = 0).  The
// slip coefficients follow build_side's for w = B.
CAD_HD void build_side_burgers(const double PA[3], const double PB[3], const double B[3], double nu, FscSide& s)
{
    build_side_geom(PA, PB, nu, s);
    if (s.skip != 0.0) return;
    for (int g = 0; g < 3; ++g) {
        s.cs[0][g] = add_rn(add_rn(mul_rn(s.ey1[g], B[0]), mul_rn(s.ey2[g], B[1])), mul_rn(s.ey3[g], B[2]));
        s.cd[0][g] = s.cs[0][g] / 4.0 / M_PI / sub_rn(1.0, nu);
    }
}

// ------------------------------------------------------------ pair drivers
template <bool HS, typename R>
CAD_HD void pair_strain(const TriDevT<R>& t, double X, double Y, double Z, R E[3][6])
{
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int k = 0; k < 6; ++k) E[m][k] = R(0.0);
    strain_fs<false>(t.real, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, E);
    if (HS) {
#pragma unroll 1
        for (int sd = 0; sd < 3; ++sd)
            if (t.side[sd].skip == R(0)) fsc_strain(t.side[sd], X, Y, Z, t.Dss, t.Dds, t.Dn, E);
        strain_fs<true>(t.image, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, E);
    }
}

// Half-space strain with the free-surface corrections of the triangle's sides
// read from per-edge maps (fsc_strain_map): entry (edge e, value q) of this
// observation point at G[e * ge + q * gq]; code[sd] = +-(e + 1) for side sd
// traversed along / against edge e's direction, 0 for no correction.
CAD_HD void pair_strain_edges(const TriDev& t, double X, double Y, double Z, const double* G, int64_t gq, int64_t ge,
                              const int* code, double E[3][6])
{
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int k = 0; k < 6; ++k) E[m][k] = 0.0;
    strain_fs<false>(t.real, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, E);
#pragma unroll 1
    for (int sd = 0; sd < 3; ++sd) {
        const int c = code[sd];
        if (c == 0) continue;
        const int64_t e = (int64_t)(c > 0 ? c : -c) - 1;
        double Gm[3][6];
#pragma unroll
        for (int q = 0; q < 18; ++q) Gm[q / 6][q % 6] = G[e * ge + q * gq];
        fsc_apply_map(Gm, c > 0 ? 1.0 : -1.0, t.real, t.Dss, t.Dds, t.Dn, E);
    }
    strain_fs<true>(t.image, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, E);
}

// Half-space strain and displacement without the free-surface corrections
// (real and image full-space terms only): the shared-edge sums add the
// corrections once per mesh edge.
CAD_HD void pair_strain_fs_image(const TriDev& t, double X, double Y, double Z, double E[3][6])
{
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int k = 0; k < 6; ++k) E[m][k] = 0.0;
    strain_fs<false>(t.real, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, E);
    strain_fs<true>(t.image, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, E);
}

CAD_HD void pair_disp_fs_image(const TriDev& t, double X, double Y, double Z, double U[3][3])
{
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int c = 0; c < 3; ++c) U[m][c] = 0.0;
    disp_fs<false>(t.real, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, U);
    disp_fs<true>(t.image, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, U);
}

// Half-space displacement with the free-surface corrections of the triangle's
// sides read from per-edge maps (fsc_disp_map), addressed as in
// pair_strain_edges.
CAD_HD void pair_disp_edges(const TriDev& t, double X, double Y, double Z, const double* G, int64_t gq, int64_t ge,
                            const int* code, double U[3][3])
{
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int c = 0; c < 3; ++c) U[m][c] = 0.0;
    disp_fs<false>(t.real, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, U);
#pragma unroll 1
    for (int sd = 0; sd < 3; ++sd) {
        const int c = code[sd];
        if (c == 0) continue;
        const int64_t e = (int64_t)(c > 0 ? c : -c) - 1;
        double Gu[3][3];
#pragma unroll
        for (int q = 0; q < 9; ++q) Gu[q / 3][q % 3] = G[e * ge + q * gq];
        fsc_apply_disp_map(Gu, c > 0 ? 1.0 : -1.0, t.real, t.Dss, t.Dds, t.Dn, t.K8, U);
    }
    disp_fs<true>(t.image, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, U);
}

template <bool HS, typename R>
CAD_HD void pair_disp(const TriDevT<R>& t, double X, double Y, double Z, R U[3][3])
{
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
        for (int c = 0; c < 3; ++c) U[m][c] = R(0.0);
    disp_fs<false>(t.real, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, U);
    if (HS) {
#pragma unroll 1
        for (int sd = 0; sd < 3; ++sd)
            if (t.side[sd].skip == R(0)) fsc_disp(t.side[sd], X, Y, Z, t.Dss, t.Dds, t.Dn, U);
        disp_fs<true>(t.image, X, Y, Z, t.Dss, t.Dds, t.Dn, t.K8, U);
    }
}

CAD_HD void build_triangle(const double a[3], const double b[3], const double c[3], double Dss, double Dds,
                           double Dn, double nu, bool hs, TriDev& t)
{
    t.Dss = Dss;
    t.Dds = Dds;
    t.Dn = Dn;
    t.K8 = 1.0 / (8.0 * M_PI * (1.0 - nu));
    build_frame(a, b, c, nu, t.real);
    if (!hs) return;
    const double ai[3] = {a[0], a[1], -a[2]}, bi[3] = {b[0], b[1], -b[2]}, ci[3] = {c[0], c[1], -c[2]};
    build_frame(ai, bi, ci, nu, t.image);
    build_side(a, b, t.real, t.Dss, t.Dds, t.Dn, nu, t.side[0]);
    build_side(b, c, t.real, t.Dss, t.Dds, t.Dn, nu, t.side[1]);
    build_side(c, a, t.real, t.Dss, t.Dds, t.Dn, nu, t.side[2]);
}

}  // namespace cad
