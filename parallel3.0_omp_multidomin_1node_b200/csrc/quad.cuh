// Device-side dynamic fundamental solutions and element quadrature for the
// constant 8-node quadrilateral element (FP64).
//
// Point kernels follow DSquareElement::GetDynaUij / GetDynaT1ij /
// GetDynaT2ij (DBEM1/dsquareelement.cpp:1238-1582) with the auxiliary
// tensors GetAij..GetHij (DBEM1/dsquareelement.h:648-893), the wave-front
// indicators Fai (:896-903) and the I/J series (DBEM1/dsquareelement.cpp:
// 1070-1154).  Element integrals are evaluated by one warp: each lane takes
// quadrature points and the warp sums the weighted integrands.
#pragma once

#include "tdbem_common.cuh"

namespace tdbem {

__device__ __forceinline__ double qwarp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// X(s1, s2) from the coordinate polynomial (GetFromLocal, DBEM1/dsquareelement.h:363-375)
__device__ __forceinline__ void q_from_local(const double* cc, double s1, double s2, double* pt)
{
    const double s12 = s1 * s1, s22 = s2 * s2, s1s22 = s1 * s22, s12s2 = s12 * s2;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double* k = cc + 8 * c;
        pt[c] = k[0] + k[1] * s1 + k[2] * s2 + k[3] * s1 * s2 + k[4] * s12 + k[5] * s22 + k[6] * s12s2 + k[7] * s1s22;
    }
}

__device__ __forceinline__ void q_rdiff1(const double* cc, double s1, double s2, double* r)
{
    const double s1_2 = 2.0 * s1, s1s2_2 = 2.0 * s1 * s2, s22 = s2 * s2;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double* k = cc + 8 * c;
        r[c] = k[1] + k[3] * s2 + k[4] * s1_2 + k[6] * s1s2_2 + k[7] * s22;
    }
}

__device__ __forceinline__ void q_rdiff2(const double* cc, double s1, double s2, double* r)
{
    const double s2_2 = 2.0 * s2, s1s2_2 = 2.0 * s1 * s2, s12 = s1 * s1;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double* k = cc + 8 * c;
        r[c] = k[2] + k[3] * s1 + k[5] * s2_2 + k[6] * s12 + k[7] * s1s2_2;
    }
}

// Unit normal and surface Jacobian at (s1, s2) (Normal / Jacobi, DBEM1/dsquareelement.h:433-484)
__device__ __forceinline__ void q_normal_jacobi(const double* cc, double s1, double s2, double* n, double* jac)
{
    double r1[3], r2[3];
    q_rdiff1(cc, s1, s2, r1);
    q_rdiff2(cc, s1, s2, r2);
    n[0] = r1[1] * r2[2] - r2[1] * r1[2];
    n[1] = r1[2] * r2[0] - r2[2] * r1[0];
    n[2] = r1[0] * r2[1] - r2[0] * r1[1];
    const double t = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    n[0] = n[0] / t;
    n[1] = n[1] / t;
    n[2] = n[2] / t;
    const double E = r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2];
    const double F = r1[0] * r2[0] + r1[1] * r2[1] + r1[2] * r2[2];
    const double G = r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2];
    *jac = sqrt(fabs(E * G - F * F));
}

__device__ __forceinline__ double q_jacobi(const double* cc, double s1, double s2)
{
    double r1[3], r2[3];
    q_rdiff1(cc, s1, s2, r1);
    q_rdiff2(cc, s1, s2, r2);
    const double E = r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2];
    const double F = r1[0] * r2[0] + r1[1] * r2[1] + r1[2] * r2[2];
    const double G = r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2];
    return sqrt(fabs(E * G - F * F));
}

__device__ __forceinline__ double q_dist(const double* a, const double* b)
{
    return sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
}

// Distance powers R[1..5] = r..r^5 and the separation RI[1..3] = x - source.
struct QR {
    double R[6];
    double RI[4];
};

__device__ __forceinline__ void q_get_r(const double* src, const double* pt, QR& r)
{
    r.RI[1] = pt[0] - src[0];
    r.RI[2] = pt[1] - src[1];
    r.RI[3] = pt[2] - src[2];
    r.R[1] = sqrt(r.RI[1] * r.RI[1] + r.RI[2] * r.RI[2] + r.RI[3] * r.RI[3]);
    r.R[2] = r.R[1] * r.R[1];
    r.R[3] = r.R[2] * r.R[1];
    r.R[4] = r.R[3] * r.R[1];
    r.R[5] = r.R[4] * r.R[1];
}

// The kernels below are templates over the material type: DynaMat gives the
// FP64 values, DynaMatD (QDual fields) the same values with their
// derivatives with respect to the domain's E.  Wave-front windows and
// rule choices are decided on the values, so the derivative is that of the
// smooth piece the quadrature sits on.
template <class S>
__device__ __forceinline__ bool q_fai(double n, double dt, double r, const S& c)
{
    const double ndt = n * dt, roc = r / qv(c);
    return (roc >= ndt) && (roc < (ndt + dt));
}

__device__ __forceinline__ QDual qwarp_sum(const QDual& v) { return {qwarp_sum(v.v), qwarp_sum(v.e)}; }

// I(n+1) - I(n) and J(n+1) - J(n) of the time integration (ISeries / JSeries)
template <class MT, class S = typename MT::Scalar>
__device__ __forceinline__ bool q_iseries(const MT& M, double n, const double* R, S& res)
{
    const double ndt = n * M.Dt, np1dt = ndt + M.Dt;
    const double r1 = R[1] / qv(M.C1), r2 = R[1] / qv(M.C2);
    if (np1dt <= r1 || ndt >= r2) { res = 0.0; return false; }
    if (ndt >= r1 && np1dt <= r2) { res = (n + 0.5) * M.Dt_2 / R[2]; return true; }
    if (ndt <= r1 && (np1dt >= r1 && np1dt <= r2)) { const double t = np1dt / R[1]; res = 0.5 * (t * t - M.OneOverC1_2); return true; }
    if (ndt <= r1 && np1dt >= r2) { res = M.Half_1OC22_1OC12; return true; }
    if (np1dt >= r2 && (ndt >= r1 && ndt <= r2)) { const double t = ndt / R[1]; res = 0.5 * (M.OneOverC2_2 - t * t); return true; }
    res = 0.0;
    return false;
}

template <class MT, class S = typename MT::Scalar>
__device__ __forceinline__ void q_jseries(const MT& M, double n, const double* R, S& res)
{
    const double ndt = n * M.Dt, np1dt = ndt + M.Dt;
    const double r1 = R[1] / qv(M.C1), r2 = R[1] / qv(M.C2);
    if (np1dt <= r1 || ndt >= r2) { res = 0.0; return; }
    if (ndt >= r1 && np1dt <= r2) { res = (n * n + n + 0.33333333333333333) * (M.Dt_3 / R[3]); return; }
    if (ndt <= r1 && (np1dt >= r1 && np1dt <= r2)) { const double t = np1dt / R[1]; res = 0.33333333333333 * (t * t * t - M.OneOverC1_3); return; }
    if (ndt <= r1 && np1dt >= r2) { res = M.Third_1OC23_1OC13; return; }
    if (np1dt >= r2 && (ndt >= r1 && ndt <= r2)) { const double t = ndt / R[1]; res = 0.333333333333333 * (M.OneOverC2_3 - t * t * t); return; }
    res = 0.0;
}

// Displacement kernel U(n): sum of the A, B and C tensor terms.  Returns the
// number of active terms (0 means U is zero).
template <class MT, class S = typename MT::Scalar>
__device__ __forceinline__ int q_dyna_u(const MT& M, S* U, double n, const QR& r)
{
    const double* R = r.R;
    const double* RI = r.RI;
    const double q0 = RI[1] * RI[1], q1 = RI[1] * RI[2], q2 = RI[1] * RI[3], q3 = RI[2] * RI[2], q4 = RI[2] * RI[3],
                 q5 = RI[3] * RI[3];
    S u0 = 0.0, u1 = 0.0, u2 = 0.0, u4 = 0.0, u5 = 0.0, u8 = 0.0;
    int flag = 0;
    const S k = M.OneOverFourPaiRou;
    if (q_fai(n, M.Dt, R[1], M.C1)) {
        ++flag;
        const S c = M.OneOverC1_2 / R[3];
        u0 += c * q0 * k; u1 += c * q1 * k; u2 += c * q2 * k; u4 += c * q3 * k; u5 += c * q4 * k; u8 += c * q5 * k;
    }
    if (q_fai(n, M.Dt, R[1], M.C2)) {
        ++flag;
        const S c = M.OneOverC2_2;
        u0 += c * (1.0 / R[1] - q0 / R[3]) * k;
        u1 += c * (-q1 / R[3]) * k;
        u2 += c * (-q2 / R[3]) * k;
        u4 += c * (1.0 / R[1] - q3 / R[3]) * k;
        u5 += c * (-q4 / R[3]) * k;
        u8 += c * (1.0 / R[1] - q5 / R[3]) * k;
    }
    S res;
    if (q_iseries(M, n, R, res)) {
        ++flag;
        const double C1 = 3.0 / R[3], C2 = 1.0 / R[1];
        const S t = k * res;
        u0 += (C1 * q0 - C2) * t; u1 += (C1 * q1) * t; u2 += (C1 * q2) * t;
        u4 += (C1 * q3 - C2) * t; u5 += (C1 * q4) * t; u8 += (C1 * q5 - C2) * t;
    }
    U[0] = u0; U[1] = u1; U[2] = u2; U[3] = u1; U[4] = u4; U[5] = u5; U[6] = u2; U[7] = u5; U[8] = u8;
    return flag;
}

// Traction kernel: type 1 = T1(n), type 2 = T2(n) (evaluated at n - 1).
template <class MT, class S = typename MT::Scalar>
__device__ __forceinline__ int q_dyna_t(const MT& M, int type, S* T, double n, const QR& r, const double* N)
{
    const double* R = r.R;
    const double* RI = r.RI;
    const double q0 = RI[1] * RI[1], q1 = RI[1] * RI[2], q2 = RI[1] * RI[3], q3 = RI[2] * RI[2], q4 = RI[2] * RI[3],
                 q5 = RI[3] * RI[3];
    const double RmNm = RI[1] * N[0] + RI[2] * N[1] + RI[3] * N[2];
    const double m = type == 1 ? n : n - 1;
#pragma unroll
    for (int i = 0; i < 9; ++i) T[i] = 0.0;
    int flag = 0;
    if (q_fai(m, M.Dt, R[1], M.C1)) {
        ++flag;
        const double C1 = (4.0 * M.C2_2OverC1_2 - 1.0) / R[3];
        const double C2 = M.C2_2OverC1_2 * 12.0 * RmNm / R[5];
        const double C3 = M.C2_2OverC1_2 * 2.0 / R[3];
        const S G1 = -2.0 * M.C2_2OverC1_3 * RmNm / R[4];
        const S G2 = 1.0 / M.C1 * (2.0 * M.C2_2OverC1_2 - 1.0) / R[2];
        S t1;
        double t2;
        if (type == 1) { t1 = kOneOver4Pi * (n + 1.0 - R[1] / M.C1Dt); t2 = kOneOver4Pi / M.Dt; }
        else { t1 = kOneOver4Pi * (1.0 - n + R[1] / M.C1Dt); t2 = -kOneOver4Pi / M.Dt; }
        const double d[9] = {C1 * RI[1] * N[0] - (C2 * q0 - C3 * (RI[1] * N[0] + RmNm)),
                             C1 * RI[2] * N[0] - (C2 * q1 - C3 * (RI[1] * N[1])),
                             C1 * RI[3] * N[0] - (C2 * q2 - C3 * (RI[1] * N[2])),
                             C1 * RI[1] * N[1] - (C2 * q1 - C3 * (RI[2] * N[0])),
                             C1 * RI[2] * N[1] - (C2 * q3 - C3 * (RI[2] * N[1] + RmNm)),
                             C1 * RI[3] * N[1] - (C2 * q4 - C3 * (RI[2] * N[2])),
                             C1 * RI[1] * N[2] - (C2 * q2 - C3 * (RI[3] * N[0])),
                             C1 * RI[2] * N[2] - (C2 * q4 - C3 * (RI[3] * N[1])),
                             C1 * RI[3] * N[2] - (C2 * q5 - C3 * (RI[3] * N[2] + RmNm))};
        const S g[9] = {G1 * q0 + G2 * RI[1] * N[0], G1 * q1 + G2 * RI[2] * N[0], G1 * q2 + G2 * RI[3] * N[0],
                        G1 * q1 + G2 * RI[1] * N[1], G1 * q3 + G2 * RI[2] * N[1], G1 * q4 + G2 * RI[3] * N[1],
                        G1 * q2 + G2 * RI[1] * N[2], G1 * q4 + G2 * RI[2] * N[2], G1 * q5 + G2 * RI[3] * N[2]};
#pragma unroll
        for (int i = 0; i < 9; ++i) T[i] += d[i] * t1 + g[i] * t2;
    }
    if (q_fai(m, M.Dt, R[1], M.C2)) {
        ++flag;
        const double E1 = 12.0 * RmNm / R[5], E2 = 2.0 / R[3], E3 = 3.0 / R[3];
        const S H1 = 2.0 / M.C2 * RmNm / R[4], H2 = -1.0 / M.C2 / R[2];
        S t1;
        double t2;
        if (type == 1) { t1 = kOneOver4Pi * (n + 1.0 - R[1] / M.C2Dt); t2 = kOneOver4Pi / M.Dt; }
        else { t1 = kOneOver4Pi * (1.0 - n + R[1] / M.C2Dt); t2 = -kOneOver4Pi / M.Dt; }
        const double e[9] = {E1 * q0 - E2 * RI[1] * N[0] - E3 * (RI[1] * N[0] + RmNm),
                             E1 * q1 - E2 * RI[2] * N[0] - E3 * (RI[1] * N[1]),
                             E1 * q2 - E2 * RI[3] * N[0] - E3 * (RI[1] * N[2]),
                             E1 * q1 - E2 * RI[1] * N[1] - E3 * (RI[2] * N[0]),
                             E1 * q3 - E2 * RI[2] * N[1] - E3 * (RI[2] * N[1] + RmNm),
                             E1 * q4 - E2 * RI[3] * N[1] - E3 * (RI[2] * N[2]),
                             E1 * q2 - E2 * RI[1] * N[2] - E3 * (RI[3] * N[0]),
                             E1 * q4 - E2 * RI[2] * N[2] - E3 * (RI[3] * N[1]),
                             E1 * q5 - E2 * RI[3] * N[2] - E3 * (RI[3] * N[2] + RmNm)};
        const S h[9] = {H1 * q0 + H2 * (RI[1] * N[0] + RmNm), H1 * q1 + H2 * RI[1] * N[1],
                        H1 * q2 + H2 * RI[1] * N[2], H1 * q1 + H2 * RI[2] * N[0],
                        H1 * q3 + H2 * (RI[2] * N[1] + RmNm), H1 * q4 + H2 * RI[2] * N[2],
                        H1 * q2 + H2 * RI[3] * N[0], H1 * q4 + H2 * RI[3] * N[1],
                        H1 * q5 + H2 * (RI[3] * N[2] + RmNm)};
#pragma unroll
        for (int i = 0; i < 9; ++i) T[i] += e[i] * t1 + h[i] * t2;
    }
    S resI;
    if (q_iseries(M, m, R, resI)) {
        ++flag;
        S resJ;
        q_jseries(M, m, R, resJ);
        const S F1 = -6.0 * M.C2_2;
        const double F2 = 5.0 * RmNm / R[5];
        const S f[9] = {F1 * (F2 * q0 - (RI[1] * N[0] + RI[1] * N[0] + RmNm) / R[3]),
                        F1 * (F2 * q1 - (RI[2] * N[0] + RI[1] * N[1]) / R[3]),
                        F1 * (F2 * q2 - (RI[3] * N[0] + RI[1] * N[2]) / R[3]),
                        0.0,
                        F1 * (F2 * q3 - (RI[2] * N[1] + RI[2] * N[1] + RmNm) / R[3]),
                        F1 * (F2 * q4 - (RI[3] * N[1] + RI[2] * N[2]) / R[3]),
                        0.0,
                        0.0,
                        F1 * (F2 * q5 - (RI[3] * N[2] + RI[3] * N[2] + RmNm) / R[3])};
        const S t1 = type == 1 ? kOneOver4Pi * ((n + 1.0) * resI - R[1] * resJ / M.Dt)
                               : kOneOver4Pi * ((1.0 - n) * resI + R[1] * resJ / M.Dt);
        T[0] += f[0] * t1; T[1] += f[1] * t1; T[2] += f[2] * t1;
        T[3] += f[1] * t1; T[4] += f[4] * t1; T[5] += f[5] * t1;
        T[6] += f[2] * t1; T[7] += f[5] * t1; T[8] += f[8] * t1;
    }
    return flag;
}

// Static traction kernel (GetTij, DBEM1/dsquareelement.cpp:496-543); R[0]=r, R[1..3]=d.
// Depends on the Poisson ratio only.
template <class MT>
__device__ __forceinline__ void q_static_t(const MT& M, double* T, const double* R, const double* n)
{
    const double t1 = R[0] * R[0];
    const double t2 = M.STCoef1 / t1;
    const double t3 = M.STCoef2 / R[0];
    const double drdn = (R[1] * n[0] + R[2] * n[1] + R[3] * n[2]) / R[0];
    const double t5 = t3 * (R[2] * n[0] - R[1] * n[1]);
    const double t6 = t3 * (R[3] * n[0] - R[1] * n[2]);
    const double t7 = t3 * (R[3] * n[1] - R[2] * n[2]);
    const double t8 = t2 * drdn;
    const double t9 = t8 * M.STCoef2;
    const double t10 = t8 * 3.0 / t1;
    double t4 = t10 * R[1];
    T[0] = t9 + t4 * R[1];
    T[1] = t4 * R[2] - t2 * t5;
    T[2] = t4 * R[3] - t2 * t6;
    T[3] = t4 * R[2] + t2 * t5;
    T[4] = t9 + t10 * R[2] * R[2];
    t4 = t10 * R[3];
    T[5] = t4 * R[2] - t2 * t7;
    T[6] = t4 * R[1] + t2 * t6;
    T[7] = t4 * R[2] + t2 * t7;
    T[8] = t9 + t10 * R[3] * R[3];
}

// Wave-front classification of (field element, source point) for time
// index n: 0 skip, 1 patch-wise rule, 2 regular rule (NeedCal,
// DBEM1/dsquareelement.cpp:1156-1201).
template <class MT>
__device__ __forceinline__ int q_need_cal(const MT& M, const double* center, double radius, int type, double n,
                                          const double* o)
{
    const double nn = type == 2 ? n - 1 : n;
    const double ndt = nn * M.Dt, np1dt = (nn + 1) * M.Dt;
    const double r = q_dist(center, o);
    const double Rmax = r + radius;
    double Rmin = r - radius;
    if (Rmin < 0.0) Rmin = 0.0;
    const double a1 = Rmax / qv(M.C1), a2 = Rmax / qv(M.C2), b1 = Rmin / qv(M.C1), b2 = Rmin / qv(M.C2);
    if (ndt >= a2 || np1dt <= b1) return 0;
    if (ndt <= b1 && (np1dt >= a1 && np1dt <= b2)) return 2;
    if (ndt <= b1 && np1dt >= a2) return 2;
    if (ndt >= a1 && np1dt <= b2) return 2;
    if ((ndt >= a1 && ndt <= b2) && np1dt >= a2) return 2;
    return 1;
}

template <class MT>
__device__ __forceinline__ bool q_pw_need_cal(const MT& M, double rpw, int type, double n, const double* pc,
                                              const double* o)
{
    const double nn = type == 2 ? n - 1 : n;
    const double c2ndt = nn * qv(M.C2Dt), c1np1dt = (nn + 1) * qv(M.C1Dt);
    const double r = q_dist(pc, o);
    return !((r - rpw) >= c1np1dt || (r + rpw) < c2ndt);
}

// Field element data a warp needs for its integrals.
struct QElem {
    const double* cc;   // [24] (global)
    const double* rcen; // [36*3] (global)
    double center[3];
    double radius, rpw;
};

// ---- warp-cooperative element integrals (result in out[9] on every lane) ----

// regular 4x4 rule for U(n) (IntDynaUij, DBEM1/dsquareelement.cpp:1955-2009)
template <class MT, class S = typename MT::Scalar>
__device__ __forceinline__ void w_int_u_regular(const QuadRules& q, const MT& M, const QElem& e,
                                                const double* src, double n, S* out)
{
    const int lane = threadIdx.x & 31;
    S c[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (lane < 16) {
        double pt[3];
        S U[9];
        QR r;
        q_from_local(e.cc, q.rp[lane][0], q.rp[lane][1], pt);
        q_get_r(src, pt, r);
        if (q_dyna_u(M, U, n, r)) {
            const double t = q.nrgv0[lane] * q_jacobi(e.cc, q.rp[lane][0], q.rp[lane][1]);
            c[0] = U[0] * t; c[1] = U[1] * t; c[2] = U[2] * t; c[3] = U[4] * t; c[4] = U[5] * t; c[5] = U[8] * t;
        }
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) c[i] = qwarp_sum(c[i]);
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = c[1]; out[4] = c[3]; out[5] = c[4];
    out[6] = c[2]; out[7] = c[4]; out[8] = c[5];
}

// regular rule for T: T1(n) + T2(n) at every point, whatever the requested
// type (IntDynaTij(typeT, ..., T_ID), DBEM1/dsquareelement.cpp:2233-2290)
template <class MT, class S = typename MT::Scalar>
__device__ __forceinline__ void w_int_t_regular(const QuadRules& q, const MT& M, const QElem& e,
                                                const double* src, double n, S* out)
{
    const int lane = threadIdx.x & 31;
    S c[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) c[i] = 0.0;
    if (lane < 16) {
        double pt[3], nor[3], jac;
        S T1[9], T2[9];
        QR r;
        q_from_local(e.cc, q.rp[lane][0], q.rp[lane][1], pt);
        q_get_r(src, pt, r);
        q_normal_jacobi(e.cc, q.rp[lane][0], q.rp[lane][1], nor, &jac);
        int flag = q_dyna_t(M, 1, T1, n, r, nor);
        flag += q_dyna_t(M, 2, T2, n, r, nor);
        if (flag) {
            const double t = q.nrgv0[lane] * jac;
#pragma unroll
            for (int i = 0; i < 9; ++i) c[i] = (T1[i] + T2[i]) * t;
        }
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) out[i] = qwarp_sum(c[i]);
}

// patch-wise 6x6 x 3x3 rule for U(n) (IntDynaUijPW, DBEM1/dsquareelementdyna.cpp:794-848)
template <class MT, class S = typename MT::Scalar>
__device__ __forceinline__ void w_int_u_pw(const QuadRules& q, const MT& M, const QElem& e, const double* src,
                                           double n, S* out)
{
    const int lane = threadIdx.x & 31;
    S c[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int it = lane; it < kNumPW2 * 9; it += 32) {
        const int p = it / 9, j = it - 9 * (it / 9);
        if (!q_pw_need_cal(M, e.rpw, 1, n, e.rcen + 3 * p, src)) continue;
        double pt[3];
        S U[9];
        QR r;
        q_from_local(e.cc, q.lpospw[p][j][0], q.lpospw[p][j][1], pt);
        q_get_r(src, pt, r);
        q_dyna_u(M, U, n, r);
        const double t = q.pwgv[p][j] * q_jacobi(e.cc, q.lpospw[p][j][0], q.lpospw[p][j][1]);
        c[0] += U[0] * t; c[1] += U[1] * t; c[2] += U[2] * t; c[3] += U[4] * t; c[4] += U[5] * t; c[5] += U[8] * t;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) c[i] = qwarp_sum(c[i]);
    out[0] = c[0]; out[1] = c[1]; out[2] = c[2]; out[3] = c[1]; out[4] = c[3]; out[5] = c[4];
    out[6] = c[2]; out[7] = c[4]; out[8] = c[5];
}

// patch-wise rule for T1 or T2 (IntDynaTijPW(typeT, ..., T_ID), DBEM1/dsquareelementdyna.cpp:940-994)
template <class MT, class S = typename MT::Scalar>
__device__ __forceinline__ void w_int_t_pw(const QuadRules& q, const MT& M, const QElem& e, int type,
                                           const double* src, double n, S* out)
{
    const int lane = threadIdx.x & 31;
    S c[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) c[i] = 0.0;
    for (int it = lane; it < kNumPW2 * 9; it += 32) {
        const int p = it / 9, j = it - 9 * (it / 9);
        if (!q_pw_need_cal(M, e.rpw, type, n, e.rcen + 3 * p, src)) continue;
        double pt[3], nor[3], jac;
        S T[9];
        QR r;
        q_from_local(e.cc, q.lpospw[p][j][0], q.lpospw[p][j][1], pt);
        q_get_r(src, pt, r);
        q_normal_jacobi(e.cc, q.lpospw[p][j][0], q.lpospw[p][j][1], nor, &jac);
        q_dyna_t(M, type, T, n, r, nor);
        const double t = q.pwgv[p][j] * jac;
#pragma unroll
        for (int i = 0; i < 9; ++i) c[i] += T[i] * t;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) out[i] = qwarp_sum(c[i]);
}

// IntDynaUijJudge / IntDynaTijJudge(typeT, ..., T_ID)
// (DBEM1/dsquareelementdyna.cpp:1603-1616, 1677-1690)
template <class MT, class S = typename MT::Scalar>
__device__ __forceinline__ int w_judge_u(const QuadRules& q, const MT& M, const QElem& e, const double* src,
                                         double n, S* out)
{
    const int f = q_need_cal(M, e.center, e.radius, 1, n, src);
    if (f == 1) w_int_u_pw(q, M, e, src, n, out);
    else if (f == 2) w_int_u_regular(q, M, e, src, n, out);
    return f;
}

template <class MT, class S = typename MT::Scalar>
__device__ __forceinline__ int w_judge_t(const QuadRules& q, const MT& M, const QElem& e, int type,
                                         const double* src, double n, S* out)
{
    const int f = q_need_cal(M, e.center, e.radius, type, n, src);
    if (f == 1) w_int_t_pw(q, M, e, type, src, n, out);
    else if (f == 2) w_int_t_regular(q, M, e, src, n, out);
    return f;
}

}  // namespace tdbem
