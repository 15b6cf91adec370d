// Shared device-side definitions of the B200 multi-domain TDBEM library.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tdbem {

constexpr double kPi = 3.141592653589793239;           // DBEM1/precompiler.h:7
constexpr double kOneOver4Pi = 0.0795774715459476679;  // DBEM1/precompiler.h:8
constexpr int kNumPW = 6;                              // patch grid per element side
constexpr int kNumPW2 = 36;
constexpr int kSinNumPW = 20;                          // polar sub-patches per sector side
constexpr int kSinNumPW2 = 400;
constexpr int kMaxDomains = 64;

// Per-domain material constants, the fields of the reference's DynaMat
// (DBEM1/dsquareelement.h:22-56) computed as BuildDynaMat does.
struct DynaMat {
    using Scalar = double;
    double G, v, Rou, C1, C2, Dt, Dt2, Dt_2, Dt_3, C1_2, C2_2, OneOverC1_2, OneOverC2_2, OneOverC1_3,
        OneOverC2_3, C2_2OverC1_2, C2_2OverC1_3, C1Dt, C2Dt, OneOverFourPaiRou, Third_1OC23_1OC13,
        Half_1OC22_1OC12, STCoef1, STCoef2;
};

// A quantity with its derivative with respect to the Young's modulus of one
// domain (forward-mode differentiation of the quadrature; geometry, time
// indices and the Poisson ratio carry none).  The density derivative follows
// by homogeneity: every kernel depends on E and rho through the wave speeds
// (proportional to sqrt(E/rho)) and, for the displacement kernel only, a
// factor 1/rho, so dF/drho = -(E/rho) dF/dE - [F is a displacement-kernel
// block] F/rho.
struct QDual {
    double v, e;
    QDual() = default;
    __host__ __device__ constexpr QDual(double x) : v(x), e(0.0) {}
    __host__ __device__ constexpr QDual(double x, double de) : v(x), e(de) {}
};

__host__ __device__ __forceinline__ double qv(double x) { return x; }
__host__ __device__ __forceinline__ double qv(const QDual& x) { return x.v; }

__host__ __device__ __forceinline__ QDual operator+(const QDual& a, const QDual& b) { return {a.v + b.v, a.e + b.e}; }
__host__ __device__ __forceinline__ QDual operator+(const QDual& a, double b) { return {a.v + b, a.e}; }
__host__ __device__ __forceinline__ QDual operator+(double a, const QDual& b) { return {a + b.v, b.e}; }
__host__ __device__ __forceinline__ QDual operator-(const QDual& a, const QDual& b) { return {a.v - b.v, a.e - b.e}; }
__host__ __device__ __forceinline__ QDual operator-(const QDual& a, double b) { return {a.v - b, a.e}; }
__host__ __device__ __forceinline__ QDual operator-(double a, const QDual& b) { return {a - b.v, -b.e}; }
__host__ __device__ __forceinline__ QDual operator-(const QDual& a) { return {-a.v, -a.e}; }
__host__ __device__ __forceinline__ QDual operator*(const QDual& a, const QDual& b)
{
    return {a.v * b.v, a.e * b.v + a.v * b.e};
}
__host__ __device__ __forceinline__ QDual operator*(const QDual& a, double b) { return {a.v * b, a.e * b}; }
__host__ __device__ __forceinline__ QDual operator*(double a, const QDual& b) { return {a * b.v, a * b.e}; }
__host__ __device__ __forceinline__ QDual operator/(const QDual& a, const QDual& b)
{
    const double q = a.v / b.v;
    return {q, (a.e - q * b.e) / b.v};
}
__host__ __device__ __forceinline__ QDual operator/(const QDual& a, double b) { return {a.v / b, a.e / b}; }
__host__ __device__ __forceinline__ QDual operator/(double a, const QDual& b)
{
    const double q = a / b.v;
    return {q, -q * b.e / b.v};
}
__host__ __device__ __forceinline__ QDual& operator+=(QDual& a, const QDual& b) { return a = a + b; }
__host__ __device__ __forceinline__ QDual& operator-=(QDual& a, const QDual& b) { return a = a - b; }

// DynaMat with the fields that depend on E as QDual (the Poisson-ratio-only
// fields and the time step stay plain).  A field that scales as
// (E/rho)^(p/2) rho^q has d/dE = (p/2) X/E.
struct DynaMatD {
    using Scalar = QDual;
    QDual G;
    double v;
    QDual Rou, C1, C2;
    double Dt, Dt2, Dt_2, Dt_3;
    QDual C1_2, C2_2, OneOverC1_2, OneOverC2_2, OneOverC1_3, OneOverC2_3;
    double C2_2OverC1_2;
    QDual C2_2OverC1_3, C1Dt, C2Dt, OneOverFourPaiRou, Third_1OC23_1OC13, Half_1OC22_1OC12;
    double STCoef1, STCoef2;
};

// Quadrature rules for the constant element (the subset of quadinfo,
// DBEM1/quadinfo.cpp:83-171, the constant-element SecInfo/FValue entries of
// :200-398 are in global memory, see SingularTables).
struct QuadRules {
    double gap;
    double lc0[2];           // local coordinates of node 0: (-gap, -gap)
    double rp[16][2];        // 4x4 Gauss-Legendre points
    double nrgv0[16];        // corner shape function N0 x weight (reference's regular weight)
    double lpospw[36][9][2]; // 6x6 patches x 3x3 points
    double pwgv[36][9];      // patch weights (no shape function)
    double cenpw[36][2];     // patch centres
    double sec_pos[4][2][16];
    double sec_val[4][16];
    double line_pos[4][4];
    double fm1_sec[4][16];
    double fm1_line[4][4];
};

// Device pointers of the per-element geometry (structure of arrays).
struct ElemGeom {
    double* cc;      // [E][3][8] coordinate polynomial coefficients
    double* center;  // [E][3]
    double* radius;  // [E]
    double* rpw;     // [E] patch radius
    double* rcen;    // [E][36][3] patch centres
    double* node;    // [E][3] collocation point (element centre)
    double* trans;   // [E][9] local frame rows t1, t2, n
    double* on_u1;   // [E][9] singular self blocks
    double* on_t1;
    double* on_t2;
    int32_t* bcid;
    int32_t* domain;
    int32_t* surface; // 1 = interface element
};

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace tdbem
