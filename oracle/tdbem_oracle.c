/*
 * TEST INFRASTRUCTURE ONLY -- parity oracle for the multi-domain TDBEM march.
 * Not part of the product; see tdbem_oracle.h.  Each routine names the
 * reference routine (file:line under DBEM1/) whose arithmetic it restates,
 * keeping the reference's operation order so the results agree to rounding.
 */
#include "tdbem_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PI_REF 3.141592653589793239           /* DBEM1/precompiler.h:7 */
#define ONE_OVER_4PI_REF 0.0795774715459476679 /* DBEM1/precompiler.h:8 */
#define NUMPW 6
#define NUMPW2 36
#define SINNUMPW 20
#define SINNUMPW2 400

static char g_err[256];
const char* orc_last_error(void) { return g_err; }

/* ------------------------------------------------------------------ */
/* Material constants: BuildDynaMat, DBEM1/dsquareelement.cpp:63-97    */
/* ------------------------------------------------------------------ */
typedef struct {
    double G, v, Rou, C1, C2, Dt, Dt2, Dt_2, Dt_3, C1_2, C2_2, OneOverC1_2, OneOverC2_2, OneOverC1_3,
        OneOverC2_3, C2_2OverC1_2, C2_2OverC1_3, C1Dt, C2Dt, OneOverFourPaiRou, Third_1OC23_1OC13,
        Half_1OC22_1OC12, STCoef1, STCoef2;
} mat_t;

static mat_t build_mat(double v, double G, double rho, double dt)
{
    mat_t m;
    m.v = v;
    m.G = G;
    m.Rou = rho;
    m.C1 = sqrt((2.0 - 2.0 * v) / (1.0 - 2.0 * v) * G / rho);
    m.C2 = sqrt(G / rho);
    m.Dt = dt;
    m.Dt2 = 2.0 * dt;
    m.Dt_2 = dt * dt;
    m.Dt_3 = dt * dt * dt;
    m.OneOverFourPaiRou = ONE_OVER_4PI_REF / rho;
    m.C1_2 = m.C1 * m.C1;
    m.C2_2 = m.C2 * m.C2;
    m.OneOverC1_2 = 1.0 / m.C1_2;
    m.OneOverC2_2 = 1.0 / m.C2_2;
    m.OneOverC1_3 = 1.0 / m.C1_2 / m.C1;
    m.OneOverC2_3 = 1.0 / m.C2_2 / m.C2;
    m.C2_2OverC1_2 = m.C2_2 / m.C1_2;
    m.C2_2OverC1_3 = m.C2_2OverC1_2 / m.C1;
    m.C1Dt = m.C1 * m.Dt;
    m.C2Dt = m.C2 * m.Dt;
    m.STCoef1 = -1.0 / (8.0 * PI_REF * (1.0 - m.v));
    m.STCoef2 = 1.0 - 2.0 * m.v;
    m.Third_1OC23_1OC13 = 1.0 / 3.0 * (m.OneOverC2_3 - m.OneOverC1_3);
    m.Half_1OC22_1OC12 = 0.5 * (m.OneOverC2_2 - m.OneOverC1_2);
    return m;
}

/* ------------------------------------------------------------------ */
/* Quadrature tables: GaussNumeMatrix (DBEM1/gaussnumematrix.cpp:4-86) */
/* with the 15-decimal Gauss-Legendre values of DBEM1/gaussposition    */
/* and gaussweight, and quadinfo::init / AssignSecInfo / AssignFValue  */
/* (DBEM1/quadinfo.cpp:83-398) restricted to the constant element.     */
/* ------------------------------------------------------------------ */
static const double GP3[3] = {-0.774596669241484, 0.0, 0.774596669241484};
static const double GW3[3] = {0.555555555555555, 0.888888888888889, 0.555555555555555};
static const double GP4[4] = {-0.861136311594052, -0.339981043584856, 0.339981043584856, 0.861136311594052};
static const double GW4[4] = {0.347854845137454, 0.652145154862546, 0.652145154862546, 0.347854845137454};

typedef struct {
    double gap;
    double lc[8][2];          /* m_LocalCoord */
    double rp[16][2];         /* regular points */
    double nrgv0[16];         /* m_NRGV[0][i] */
    double lpospw[36][9][2];  /* m_LPOSPW */
    double pwgv[36][9];       /* m_PWGV */
    double cenpw[36][2];
    double sec_pos[4][2][16]; /* m_SecConstPos */
    double sec_val[4][16];    /* m_SecConstVal */
    double line_pos[4][4];    /* m_ConstLinePos */
    double fm1_sec[4][16];    /* m_ConstFMinusOneSecVal */
    double fm1_line[4][4];    /* m_ConstFMinusOneLineVal */
    double (*secpw_pos)[2][SINNUMPW2][9]; /* m_SecConstPosPW [4] */
    double (*secpw_val)[SINNUMPW2][9];    /* m_SecConstValPW [4] */
} quad_t;

/* quadinfo::N, DBEM1/quadinfo.h:153-176 */
static void quad_N(const quad_t* q, double s1, double s2, double* res)
{
    const double(*L)[2] = q->lc;
    double lx = L[1][0] - L[0][0];
    double ly = L[3][1] - L[0][1];
    double lxly = lx * ly;
    double hx = 0.25 * lx * lxly;
    double hy = 0.25 * ly * lxly;
    res[0] = (s1 - L[1][0]) * (s2 - L[3][1]) / lxly;
    res[1] = (s1 - L[0][0]) * (s2 - L[2][1]) / (-lxly);
    res[2] = (s1 - L[3][0]) * (s2 - L[1][1]) / (lxly);
    res[3] = (s1 - L[2][0]) * (s2 - L[0][1]) / (-lxly);
    res[4] = (s1 - L[0][0]) * (s1 - L[1][0]) * (s2 - L[6][1]) / (hx);
    res[5] = (s1 - L[7][0]) * (s2 - L[1][1]) * (s2 - L[2][1]) / (-hy);
    res[6] = (s1 - L[2][0]) * (s1 - L[3][0]) * (s2 - L[4][1]) / (-hx);
    res[7] = (s1 - L[5][0]) * (s2 - L[0][1]) * (s2 - L[3][1]) / (hy);
    res[0] -= 0.5 * (res[4] + res[7]);
    res[1] -= 0.5 * (res[4] + res[5]);
    res[2] -= 0.5 * (res[5] + res[6]);
    res[3] -= 0.5 * (res[6] + res[7]);
}

/* anonymous-namespace helpers, DBEM1/quadinfo.cpp:3-50 */
static double c_theta_start(int a)
{
    switch (a) {
    case 0: return -0.75 * PI_REF;
    case 1: return -0.25 * PI_REF;
    case 2: return 0.25 * PI_REF;
    case 3: return 0.75 * PI_REF;
    }
    return 0.0;
}
static double c_theta_diff(void) { return 0.5 * PI_REF; }
static double c_theta_from_local(double lt, int a) { return c_theta_start(a) + 0.5 * (lt + 1.0) * c_theta_diff(); }
static double c_alpha(double t, int a)
{
    switch (a) {
    case 0: return -1.0 / sin(t);
    case 1: return 1.0 / cos(t);
    case 2: return 1.0 / sin(t);
    case 3: return -1.0 / cos(t);
    }
    return 0.0;
}
static double c_polar(double lr, double t, int a) { return 0.5 * (lr + 1.0) * c_alpha(t, a); }

static void quad_init(quad_t* q, double gap)
{
    int i, j, m, p, a;
    double res[8];
    q->gap = gap;
    /* quadinfo::GetLocalCoord, DBEM1/quadinfo.h:64-90 */
    double lc[8][2] = {{-gap, -gap}, {gap, -gap}, {gap, gap}, {-gap, gap},
                       {0.0, -gap}, {gap, 0.0}, {0.0, gap}, {-gap, 0.0}};
    memcpy(q->lc, lc, sizeof lc);
    double sp[16][2], sa[16], pwrp[9][2], pwra[9];
    for (i = 0; i < 4; ++i)
        for (j = 0; j < 4; ++j) {
            m = i * 4 + j;
            q->rp[m][0] = GP4[j];
            q->rp[m][1] = GP4[i];
            sp[m][0] = GP4[j];
            sp[m][1] = GP4[i];
            sa[m] = GW4[j] * GW4[i];
        }
    for (i = 0; i < 3; ++i)
        for (j = 0; j < 3; ++j) {
            m = i * 3 + j;
            pwrp[m][0] = GP3[j];
            pwrp[m][1] = GP3[i];
            pwra[m] = GW3[j] * GW3[i];
        }
    for (m = 0; m < 16; ++m) {
        quad_N(q, q->rp[m][0], q->rp[m][1], res);
        q->nrgv0[m] = res[0] * sa[m]; /* ra == sa for the 4-point rule */
    }
    double L = 2.0 / NUMPW;
    for (i = 0; i < NUMPW; ++i)
        for (j = 0; j < NUMPW; ++j) {
            p = i * NUMPW + j;
            q->cenpw[p][0] = -1.0 + L / 2.0 + L * j;
            q->cenpw[p][1] = -1.0 + L / 2.0 + L * i;
            for (m = 0; m < 9; ++m) {
                q->lpospw[p][m][0] = q->cenpw[p][0] + pwrp[m][0] / NUMPW;
                q->lpospw[p][m][1] = q->cenpw[p][1] + pwrp[m][1] / NUMPW;
            }
        }
    for (i = 0; i < NUMPW2; ++i)
        for (m = 0; m < 9; ++m) q->pwgv[i][m] = pwra[m] * (L / 2.0) * (L / 2.0);

    double Ls = 2.0 / SINNUMPW;
    static double sinlpos[SINNUMPW2][9][2];
    double sinnpwgv[9];
    for (i = 0; i < SINNUMPW; ++i)
        for (j = 0; j < SINNUMPW; ++j) {
            p = i * SINNUMPW + j;
            double c0 = -1.0 + Ls / 2.0 + Ls * j, c1 = -1.0 + Ls / 2.0 + Ls * i;
            for (m = 0; m < 9; ++m) {
                sinlpos[p][m][0] = c0 + pwrp[m][0] / SINNUMPW;
                sinlpos[p][m][1] = c1 + pwrp[m][1] / SINNUMPW;
            }
        }
    for (m = 0; m < 9; ++m) sinnpwgv[m] = pwra[m] * (Ls / 2.0) * (Ls / 2.0);

    for (a = 0; a < 4; ++a)
        for (m = 0; m < 16; ++m) {
            double th = c_theta_from_local(sp[m][0], a);
            double fa = 0.25 * c_alpha(th, a) * c_theta_diff();
            double rou = c_polar(sp[m][1], th, a);
            q->sec_pos[a][0][m] = rou * cos(th);
            q->sec_pos[a][1][m] = rou * sin(th);
            q->sec_val[a][m] = rou * fa * sa[m];
            double temp = rou * fa * sa[m];
            q->fm1_sec[a][m] = temp / rou / rou;
        }
    for (a = 0; a < 4; ++a)
        for (m = 0; m < 4; ++m) {
            double th = c_theta_from_local(GP4[m], a);
            q->line_pos[a][m] = th;
            double rou = c_polar(1.0, th, a);
            q->fm1_line[a][m] = 0.5 * c_theta_diff() * log(rou) * GW4[m];
        }
    q->secpw_pos = malloc(sizeof(double[2][SINNUMPW2][9]) * 4);
    q->secpw_val = malloc(sizeof(double[SINNUMPW2][9]) * 4);
    for (a = 0; a < 4; ++a)
        for (p = 0; p < SINNUMPW2; ++p)
            for (m = 0; m < 9; ++m) {
                double th = c_theta_from_local(sinlpos[p][m][0], a);
                double fa = 0.25 * c_alpha(th, a) * c_theta_diff();
                double rou = c_polar(sinlpos[p][m][1], th, a);
                q->secpw_pos[a][0][p][m] = rou * cos(th);
                q->secpw_pos[a][1][p][m] = rou * sin(th);
                q->secpw_val[a][p][m] = rou * fa * sinnpwgv[m];
            }
}

/* ------------------------------------------------------------------ */
/* Element geometry: DSquareElement::GetCoef / GetFromLocal / RDiffs / */
/* Normal / Jacobi / TranslateMatrix (DBEM1/dsquareelement.h:363-611), */
/* GeoInit (DBEM1/dsquareelement.cpp:332-382)                         */
/* ------------------------------------------------------------------ */
typedef struct {
    double cc[3][8];
    double center[3];
    double radius, radius_pw;
    double rcen[NUMPW2][3];
    double node[3];
    double trans[9];
    double on_u1[9], on_t1[9], on_t2[9];
    int bcid, domain, surface;
} elem_t;

static void get_coef(double* c, const double* v)
{
    c[0] = 0.25 * (-v[0] - v[3] + 2 * v[5] - v[2] - v[1] + 2 * v[4] + 2 * v[7] + 2 * v[6]);
    c[1] = 0.5 * (v[5] - v[7]);
    c[2] = 0.5 * (-v[4] + v[6]);
    c[3] = 0.25 * (v[0] - v[1] + v[2] - v[3]);
    c[4] = 0.25 * (-2 * v[4] + v[3] + v[2] - 2 * v[6] + v[1] + v[0]);
    c[5] = 0.25 * (-2 * v[5] + v[1] - 2 * v[7] + v[2] + v[0] + v[3]);
    c[6] = 0.25 * (2 * v[4] + v[3] + v[2] - 2 * v[6] - v[1] - v[0]);
    c[7] = 0.25 * (2 * v[7] - 2 * v[5] + v[1] - v[3] + v[2] - v[0]);
}

static void from_local(const elem_t* e, double s1, double s2, double* pt)
{
    double s12 = s1 * s1, s22 = s2 * s2, s1s22 = s1 * s22, s12s2 = s12 * s2;
    for (int c = 0; c < 3; ++c) {
        const double* k = e->cc[c];
        pt[c] = k[0] + k[1] * s1 + k[2] * s2 + k[3] * s1 * s2 + k[4] * s12 + k[5] * s22 + k[6] * s12s2 + k[7] * s1s22;
    }
}

static void rdiff1(const elem_t* e, double s1, double s2, double* r)
{
    double s1_2 = 2.0 * s1, s1s2_2 = 2.0 * s1 * s2, s22 = s2 * s2;
    for (int c = 0; c < 3; ++c) {
        const double* k = e->cc[c];
        r[c] = k[1] + k[3] * s2 + k[4] * s1_2 + k[6] * s1s2_2 + k[7] * s22;
    }
}

static void rdiff2(const elem_t* e, double s1, double s2, double* r)
{
    double s2_2 = 2.0 * s2, s1s2_2 = 2.0 * s1 * s2, s12 = s1 * s1;
    for (int c = 0; c < 3; ++c) {
        const double* k = e->cc[c];
        r[c] = k[2] + k[3] * s1 + k[5] * s2_2 + k[6] * s12 + k[7] * s1s2_2;
    }
}

static void normal_at(const elem_t* e, double s1, double s2, double* n)
{
    double r1[3], r2[3];
    rdiff1(e, s1, s2, r1);
    rdiff2(e, s1, s2, r2);
    n[0] = r1[1] * r2[2] - r2[1] * r1[2];
    n[1] = r1[2] * r2[0] - r2[2] * r1[0];
    n[2] = r1[0] * r2[1] - r2[0] * r1[1];
    double t = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    n[0] = n[0] / t;
    n[1] = n[1] / t;
    n[2] = n[2] / t;
}

static double jacobi_at(const elem_t* e, double s1, double s2)
{
    double ru[3], rv[3];
    rdiff1(e, s1, s2, ru);
    rdiff2(e, s1, s2, rv);
    double E = ru[0] * ru[0] + ru[1] * ru[1] + ru[2] * ru[2];
    double F = ru[0] * rv[0] + ru[1] * rv[1] + ru[2] * rv[2];
    double G = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
    return sqrt(fabs(E * G - F * F));
}

static void unit3(const double* r, double* t)
{
    double l = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    t[0] = r[0] / l;
    t[1] = r[1] / l;
    t[2] = r[2] / l;
}

static void translate_matrix(const elem_t* e, double s1, double s2, double* T)
{
    double r[3];
    rdiff1(e, s1, s2, r);
    unit3(r, T);
    rdiff2(e, s1, s2, r);
    unit3(r, T + 3);
    T[6] = T[1] * T[5] - T[4] * T[2];
    T[7] = T[3] * T[2] - T[0] * T[5];
    T[8] = T[0] * T[4] - T[3] * T[1];
    double t = sqrt(T[6] * T[6] + T[7] * T[7] + T[8] * T[8]);
    T[6] /= t;
    T[7] /= t;
    T[8] /= t;
    T[3] = T[7] * T[2] - T[8] * T[1];
    T[4] = T[8] * T[0] - T[6] * T[2];
    T[5] = T[6] * T[1] - T[7] * T[0];
}

static double dist3(const double* a, const double* b)
{
    return sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
}

/* ------------------------------------------------------------------ */
/* Dynamic fundamental solution at one point: GetAij..GetHij           */
/* (DBEM1/dsquareelement.h:648-893), Fai (:896-903), ISeries/JSeries   */
/* (DBEM1/dsquareelement.cpp:1070-1154), GetDynaUij/T1ij/T2ij          */
/* (:1238-1582), static GetTij (:496-543)                              */
/* ------------------------------------------------------------------ */
typedef struct {
    double R[6];  /* R[1]=r .. R[5]=r^5 */
    double RI[4]; /* RI[1..3] = x - source */
} rvec_t;

static void get_r(const double* src, const double* pt, rvec_t* r)
{
    r->RI[1] = pt[0] - src[0];
    r->RI[2] = pt[1] - src[1];
    r->RI[3] = pt[2] - src[2];
    r->R[1] = sqrt(r->RI[1] * r->RI[1] + r->RI[2] * r->RI[2] + r->RI[3] * r->RI[3]);
    r->R[2] = r->R[1] * r->R[1];
    r->R[3] = r->R[2] * r->R[1];
    r->R[4] = r->R[3] * r->R[1];
    r->R[5] = r->R[4] * r->R[1];
    r->RI[0] = r->R[1];
}

static int fai(double n, double dt, double r, double c)
{
    double ndt = n * dt;
    double roc = r / c;
    return (roc >= ndt) && (roc < (ndt + dt));
}

static int iseries(const mat_t* M, double n, const double* R, double* res)
{
    double ndt = n * M->Dt, np1dt = ndt + M->Dt;
    double r1 = R[1] / M->C1, r2 = R[1] / M->C2, t1;
    if (np1dt <= r1 || ndt >= r2) { *res = 0.0; return 0; }
    else if (ndt >= r1 && np1dt <= r2) { *res = (n + 0.5) * M->Dt_2 / R[2]; return 1; }
    else if (ndt <= r1 && (np1dt >= r1 && np1dt <= r2)) { t1 = np1dt / R[1]; *res = 0.5 * (t1 * t1 - M->OneOverC1_2); return 1; }
    else if (ndt <= r1 && np1dt >= r2) { *res = M->Half_1OC22_1OC12; return 1; }
    else if (np1dt >= r2 && (ndt >= r1 && ndt <= r2)) { t1 = ndt / R[1]; *res = 0.5 * (M->OneOverC2_2 - t1 * t1); return 1; }
    *res = 0.0;
    return 0;
}

static int jseries(const mat_t* M, double n, const double* R, double* res)
{
    double ndt = n * M->Dt, np1dt = ndt + M->Dt;
    double r1 = R[1] / M->C1, r2 = R[1] / M->C2, t1;
    if (np1dt <= r1 || ndt >= r2) { *res = 0.0; return 0; }
    else if (ndt >= r1 && np1dt <= r2) { t1 = M->Dt_3 / R[3]; *res = (n * n + n + 0.33333333333333333) * t1; return 1; }
    else if (ndt <= r1 && (np1dt >= r1 && np1dt <= r2)) { t1 = np1dt / R[1]; *res = 0.33333333333333 * (t1 * t1 * t1 - M->OneOverC1_3); return 1; }
    else if (ndt <= r1 && np1dt >= r2) { *res = M->Third_1OC23_1OC13; return 1; }
    else if (np1dt >= r2 && (ndt >= r1 && ndt <= r2)) { t1 = ndt / R[1]; *res = 0.333333333333333 * (M->OneOverC2_3 - t1 * t1 * t1); return 1; }
    *res = 0.0;
    return 0;
}

static void rirj_of(const double* RI, double* q)
{
    q[0] = RI[1] * RI[1];
    q[1] = RI[1] * RI[2];
    q[2] = RI[1] * RI[3];
    q[3] = RI[2] * RI[2];
    q[4] = RI[2] * RI[3];
    q[5] = RI[3] * RI[3];
}

static void k_aij(const mat_t* M, double* a, const double* R, const double* q)
{
    double C1 = M->OneOverC1_2 / R[3];
    a[0] = C1 * q[0]; a[1] = C1 * q[1]; a[2] = C1 * q[2]; a[3] = a[1]; a[4] = C1 * q[3];
    a[5] = C1 * q[4]; a[6] = a[2]; a[7] = a[5]; a[8] = C1 * q[5];
}

static void k_bij(const mat_t* M, double* b, const double* R, const double* q)
{
    double k = M->OneOverC2_2;
    b[0] = k * (1.0 / R[1] - q[0] / R[3]);
    b[1] = k * (-q[1] / R[3]);
    b[2] = k * (-q[2] / R[3]);
    b[3] = b[1];
    b[4] = k * (1.0 / R[1] - q[3] / R[3]);
    b[5] = k * (-q[4] / R[3]);
    b[6] = b[2];
    b[7] = b[5];
    b[8] = k * (1.0 / R[1] - q[5] / R[3]);
}

static void k_cij(double* c, const double* R, const double* q)
{
    double C1 = 3.0 / R[3], C2 = 1.0 / R[1];
    c[0] = C1 * q[0] - C2; c[1] = C1 * q[1]; c[2] = C1 * q[2]; c[3] = c[1]; c[4] = C1 * q[3] - C2;
    c[5] = C1 * q[4]; c[6] = c[2]; c[7] = c[5]; c[8] = C1 * q[5] - C2;
}

static void k_dij(const mat_t* M, double* d, const double* R, const double* RI, const double* N, const double* q)
{
    double RmNm = RI[1] * N[0] + RI[2] * N[1] + RI[3] * N[2];
    double C1 = (4.0 * M->C2_2OverC1_2 - 1.0) / R[3];
    double C2 = M->C2_2OverC1_2 * 12.0 * RmNm / R[5];
    double C3 = M->C2_2OverC1_2 * 2.0 / R[3];
    d[0] = C1 * RI[1] * N[0] - (C2 * q[0] - C3 * (RI[1] * N[0] + RmNm));
    d[1] = C1 * RI[2] * N[0] - (C2 * q[1] - C3 * (RI[1] * N[1]));
    d[2] = C1 * RI[3] * N[0] - (C2 * q[2] - C3 * (RI[1] * N[2]));
    d[3] = C1 * RI[1] * N[1] - (C2 * q[1] - C3 * (RI[2] * N[0]));
    d[4] = C1 * RI[2] * N[1] - (C2 * q[3] - C3 * (RI[2] * N[1] + RmNm));
    d[5] = C1 * RI[3] * N[1] - (C2 * q[4] - C3 * (RI[2] * N[2]));
    d[6] = C1 * RI[1] * N[2] - (C2 * q[2] - C3 * (RI[3] * N[0]));
    d[7] = C1 * RI[2] * N[2] - (C2 * q[4] - C3 * (RI[3] * N[1]));
    d[8] = C1 * RI[3] * N[2] - (C2 * q[5] - C3 * (RI[3] * N[2] + RmNm));
}

static void k_eij(double* e, const double* R, const double* RI, const double* N, const double* q)
{
    double RmNm = RI[1] * N[0] + RI[2] * N[1] + RI[3] * N[2];
    double C1 = 12.0 * RmNm / R[5], C2 = 2.0 / R[3], C3 = 3.0 / R[3];
    e[0] = C1 * q[0] - C2 * RI[1] * N[0] - C3 * (RI[1] * N[0] + RmNm);
    e[1] = C1 * q[1] - C2 * RI[2] * N[0] - C3 * (RI[1] * N[1]);
    e[2] = C1 * q[2] - C2 * RI[3] * N[0] - C3 * (RI[1] * N[2]);
    e[3] = C1 * q[1] - C2 * RI[1] * N[1] - C3 * (RI[2] * N[0]);
    e[4] = C1 * q[3] - C2 * RI[2] * N[1] - C3 * (RI[2] * N[1] + RmNm);
    e[5] = C1 * q[4] - C2 * RI[3] * N[1] - C3 * (RI[2] * N[2]);
    e[6] = C1 * q[2] - C2 * RI[1] * N[2] - C3 * (RI[3] * N[0]);
    e[7] = C1 * q[4] - C2 * RI[2] * N[2] - C3 * (RI[3] * N[1]);
    e[8] = C1 * q[5] - C2 * RI[3] * N[2] - C3 * (RI[3] * N[2] + RmNm);
}

static void k_fij(const mat_t* M, double* f, const double* R, const double* RI, const double* N, const double* q)
{
    double RmNm = RI[1] * N[0] + RI[2] * N[1] + RI[3] * N[2];
    double C1 = -6.0 * M->C2_2, C2 = 5.0 * RmNm / R[5];
    f[0] = C1 * (C2 * q[0] - (RI[1] * N[0] + RI[1] * N[0] + RmNm) / R[3]);
    f[1] = C1 * (C2 * q[1] - (RI[2] * N[0] + RI[1] * N[1]) / R[3]);
    f[2] = C1 * (C2 * q[2] - (RI[3] * N[0] + RI[1] * N[2]) / R[3]);
    f[3] = f[1];
    f[4] = C1 * (C2 * q[3] - (RI[2] * N[1] + RI[2] * N[1] + RmNm) / R[3]);
    f[5] = C1 * (C2 * q[4] - (RI[3] * N[1] + RI[2] * N[2]) / R[3]);
    f[6] = f[2];
    f[7] = f[5];
    f[8] = C1 * (C2 * q[5] - (RI[3] * N[2] + RI[3] * N[2] + RmNm) / R[3]);
}

static void k_gij(const mat_t* M, double* g, const double* R, const double* RI, const double* N, const double* q)
{
    double RmNm = RI[1] * N[0] + RI[2] * N[1] + RI[3] * N[2];
    double C1 = -2.0 * M->C2_2OverC1_3 * RmNm / R[4];
    double C2 = 1.0 / M->C1 * (2.0 * M->C2_2OverC1_2 - 1.0) / R[2];
    g[0] = C1 * q[0] + C2 * RI[1] * N[0];
    g[1] = C1 * q[1] + C2 * RI[2] * N[0];
    g[2] = C1 * q[2] + C2 * RI[3] * N[0];
    g[3] = C1 * q[1] + C2 * RI[1] * N[1];
    g[4] = C1 * q[3] + C2 * RI[2] * N[1];
    g[5] = C1 * q[4] + C2 * RI[3] * N[1];
    g[6] = C1 * q[2] + C2 * RI[1] * N[2];
    g[7] = C1 * q[4] + C2 * RI[2] * N[2];
    g[8] = C1 * q[5] + C2 * RI[3] * N[2];
}

static void k_hij(const mat_t* M, double* h, const double* R, const double* RI, const double* N, const double* q)
{
    double RmNm = RI[1] * N[0] + RI[2] * N[1] + RI[3] * N[2];
    double C1 = 2.0 / M->C2 * RmNm / R[4];
    double C2 = -1.0 / M->C2 / R[2];
    h[0] = C1 * q[0] + C2 * (RI[1] * N[0] + RmNm);
    h[1] = C1 * q[1] + C2 * RI[1] * N[1];
    h[2] = C1 * q[2] + C2 * RI[1] * N[2];
    h[3] = C1 * q[1] + C2 * RI[2] * N[0];
    h[4] = C1 * q[3] + C2 * (RI[2] * N[1] + RmNm);
    h[5] = C1 * q[4] + C2 * RI[2] * N[2];
    h[6] = C1 * q[2] + C2 * RI[3] * N[0];
    h[7] = C1 * q[4] + C2 * RI[3] * N[1];
    h[8] = C1 * q[5] + C2 * (RI[3] * N[2] + RmNm);
}

static int dyna_u(const mat_t* M, double* U, double n, const rvec_t* r)
{
    double T[9], q[6], res, t1;
    int flag = 0, k;
    for (k = 0; k < 9; ++k) U[k] = 0.0;
    rirj_of(r->RI, q);
    if (fai(n, M->Dt, r->R[1], M->C1)) {
        flag++;
        k_aij(M, T, r->R, q);
        t1 = M->OneOverFourPaiRou;
        for (k = 0; k < 9; ++k) U[k] += T[k] * t1;
    }
    if (fai(n, M->Dt, r->R[1], M->C2)) {
        flag++;
        k_bij(M, T, r->R, q);
        t1 = M->OneOverFourPaiRou;
        for (k = 0; k < 9; ++k) U[k] += T[k] * t1;
    }
    if (iseries(M, n, r->R, &res)) {
        flag++;
        k_cij(T, r->R, q);
        t1 = M->OneOverFourPaiRou * res;
        for (k = 0; k < 9; ++k) U[k] += T[k] * t1;
    }
    return flag;
}

/* type 1: GetDynaT1ij(n); type 2: GetDynaT2ij(n) (which evaluates at n-1) */
static int dyna_t(const mat_t* M, int type, double* T, double n, const rvec_t* r, const double* N)
{
    double A[9], B[9], q[6], resI, resJ, t1, t2;
    int flag = 0, k;
    const double* R = r->R;
    const double* RI = r->RI;
    double m = type == 1 ? n : n - 1;
    for (k = 0; k < 9; ++k) T[k] = 0.0;
    rirj_of(RI, q);
    if (fai(m, M->Dt, R[1], M->C1)) {
        flag++;
        k_dij(M, A, R, RI, N, q);
        k_gij(M, B, R, RI, N, q);
        if (type == 1) {
            t1 = ONE_OVER_4PI_REF * (n + 1.0 - R[1] / M->C1Dt);
            t2 = ONE_OVER_4PI_REF / M->Dt;
        } else {
            t1 = ONE_OVER_4PI_REF * (1.0 - n + R[1] / M->C1Dt);
            t2 = -ONE_OVER_4PI_REF / M->Dt;
        }
        for (k = 0; k < 9; ++k) T[k] += A[k] * t1 + B[k] * t2;
    }
    if (fai(m, M->Dt, R[1], M->C2)) {
        flag++;
        k_eij(A, R, RI, N, q);
        k_hij(M, B, R, RI, N, q);
        if (type == 1) {
            t1 = ONE_OVER_4PI_REF * (n + 1.0 - R[1] / M->C2Dt);
            t2 = ONE_OVER_4PI_REF / M->Dt;
        } else {
            t1 = ONE_OVER_4PI_REF * (1.0 - n + R[1] / M->C2Dt);
            t2 = -ONE_OVER_4PI_REF / M->Dt;
        }
        for (k = 0; k < 9; ++k) T[k] += A[k] * t1 + B[k] * t2;
    }
    if (iseries(M, m, R, &resI)) {
        flag++;
        jseries(M, m, R, &resJ);
        k_fij(M, A, R, RI, N, q);
        if (type == 1)
            t1 = ONE_OVER_4PI_REF * ((n + 1.0) * resI - R[1] * resJ / M->Dt);
        else
            t1 = ONE_OVER_4PI_REF * ((1.0 - n) * resI + R[1] * resJ / M->Dt);
        for (k = 0; k < 9; ++k) T[k] += A[k] * t1;
    }
    return flag;
}

/* static traction kernel GetTij, R[0]=r, R[1..3]=d (DBEM1/dsquareelement.cpp:496-543) */
static void static_t(const mat_t* M, double* T, const double* R, const double* n)
{
    double t1 = R[0] * R[0];
    double t2 = M->STCoef1 / t1;
    double t3 = M->STCoef2 / R[0];
    double drdn = (R[1] * n[0] + R[2] * n[1] + R[3] * n[2]) / R[0];
    double t4, t5, t6, t7, t8, t9, t10;
    t5 = t3 * (R[2] * n[0] - R[1] * n[1]);
    t6 = t3 * (R[3] * n[0] - R[1] * n[2]);
    t7 = t3 * (R[3] * n[1] - R[2] * n[2]);
    t8 = t2 * drdn;
    t9 = t8 * M->STCoef2;
    t10 = t8 * 3.0 / t1;
    t4 = t10 * R[1];
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

/* GetFijMinusOne, DBEM1/dsquareelement.cpp:609-640 */
static void fij_minus_one(double* F, const double* A, const double* J, double c1, double c2)
{
    double AkJk0 = A[1] * J[0] + A[2] * J[1] + A[3] * J[2];
    double t1 = 3.0 * A[1] * AkJk0 / A[5];
    double t2 = c2 * (A[2] * J[0] - A[1] * J[1]) / A[4];
    double t3 = c2 * (A[3] * J[0] - A[1] * J[2]) / A[4];
    double t4 = c2 * (A[3] * J[1] - A[2] * J[2]) / A[4];
    double temp = c2 * AkJk0 / A[4];
    F[0] = c1 * (temp + t1 * A[1]);
    F[1] = c1 * (t1 * A[2] - t2);
    F[2] = c1 * (t1 * A[3] - t3);
    F[3] = c1 * (t1 * A[2] + t2);
    F[4] = c1 * (temp + 3.0 * A[2] * A[2] * AkJk0 / A[5]);
    t1 = 3.0 * A[3] * AkJk0 / A[5];
    F[5] = c1 * (t1 * A[2] - t4);
    F[6] = c1 * (t1 * A[1] + t3);
    F[7] = c1 * (t1 * A[2] + t4);
    F[8] = c1 * (temp + t1 * A[3]);
}

/* ------------------------------------------------------------------ */
/* Element integrals                                                   */
/* ------------------------------------------------------------------ */

/* NeedCal, DBEM1/dsquareelement.cpp:1156-1201 */
static int need_cal(const mat_t* M, const elem_t* e, int type, double n, const double* o)
{
    double nn = type == 2 ? n - 1 : n;
    double ndt = nn * M->Dt, np1dt = (nn + 1) * M->Dt;
    double r = dist3(e->center, o);
    double Rmax = r + e->radius, Rmin = r - e->radius;
    if (Rmin < 0.0) Rmin = 0.0;
    double a1 = Rmax / M->C1, a2 = Rmax / M->C2, b1 = Rmin / M->C1, b2 = Rmin / M->C2;
    if (ndt >= a2 || np1dt <= b1) return 0;
    else if (ndt <= b1 && (np1dt >= a1 && np1dt <= b2)) return 2;
    else if (ndt <= b1 && np1dt >= a2) return 2;
    else if (ndt >= a1 && np1dt <= b2) return 2;
    else if ((ndt >= a1 && ndt <= b2) && np1dt >= a2) return 2;
    return 1;
}

/* PWNeedCal, DBEM1/dsquareelement.h:926-943 */
static int pw_need_cal(const mat_t* M, const elem_t* e, int type, double n, const double* pc, const double* o)
{
    double nn = type == 2 ? n - 1 : n;
    double c2ndt = nn * M->C2Dt, c1np1dt = (nn + 1) * M->C1Dt;
    double r = dist3(pc, o);
    double rpr = r + e->radius_pw, rmr = r - e->radius_pw;
    return (rmr >= c1np1dt || rpr < c2ndt) ? 0 : 1;
}

/* IntDynaUij(..., T_ID), DBEM1/dsquareelement.cpp:1955-2009 */
static void int_u_regular(const quad_t* q, const mat_t* M, const elem_t* e, const double* src, double n, double* out)
{
    double U[9], pt[3];
    rvec_t r;
    int i, k;
    for (k = 0; k < 9; ++k) out[k] = 0.0;
    for (i = 0; i < 16; ++i) {
        from_local(e, q->rp[i][0], q->rp[i][1], pt);
        get_r(src, pt, &r);
        if (dyna_u(M, U, n, &r)) {
            double temp = q->nrgv0[i] * jacobi_at(e, q->rp[i][0], q->rp[i][1]);
            out[0] += U[0] * temp; out[1] += U[1] * temp; out[2] += U[2] * temp;
            out[4] += U[4] * temp; out[5] += U[5] * temp; out[8] += U[8] * temp;
        }
    }
    out[3] = out[1]; out[6] = out[2]; out[7] = out[5];
}

/* IntDynaTij(typeT, ..., T_ID), DBEM1/dsquareelement.cpp:2233-2290: the
 * regular rule adds T1(n)+T2(n) at every point whatever typeT is. */
static void int_t_regular(const quad_t* q, const mat_t* M, const elem_t* e, const double* src, double n, double* out)
{
    double T1[9], T2[9], pt[3], nor[3];
    rvec_t r;
    int i, k;
    for (k = 0; k < 9; ++k) out[k] = 0.0;
    for (i = 0; i < 16; ++i) {
        from_local(e, q->rp[i][0], q->rp[i][1], pt);
        get_r(src, pt, &r);
        normal_at(e, q->rp[i][0], q->rp[i][1], nor);
        int flag = dyna_t(M, 1, T1, n, &r, nor);
        flag += dyna_t(M, 2, T2, n, &r, nor);
        if (flag) {
            double temp = q->nrgv0[i] * jacobi_at(e, q->rp[i][0], q->rp[i][1]);
            for (k = 0; k < 9; ++k) out[k] += (T1[k] + T2[k]) * temp;
        }
    }
}

/* IntDynaUijPW(..., T_ID), DBEM1/dsquareelementdyna.cpp:794-848 */
static void int_u_pw(const quad_t* q, const mat_t* M, const elem_t* e, const double* src, double n, double* out)
{
    double U[9], pt[3];
    rvec_t r;
    int i, j, k;
    for (k = 0; k < 9; ++k) out[k] = 0.0;
    for (i = 0; i < NUMPW2; ++i) {
        if (!pw_need_cal(M, e, 1, n, e->rcen[i], src)) continue;
        for (j = 0; j < 9; ++j) {
            from_local(e, q->lpospw[i][j][0], q->lpospw[i][j][1], pt);
            get_r(src, pt, &r);
            dyna_u(M, U, n, &r);
            double temp = q->pwgv[i][j] * jacobi_at(e, q->lpospw[i][j][0], q->lpospw[i][j][1]);
            out[0] += U[0] * temp; out[1] += U[1] * temp; out[2] += U[2] * temp;
            out[4] += U[4] * temp; out[5] += U[5] * temp; out[8] += U[8] * temp;
        }
    }
    out[3] = out[1]; out[6] = out[2]; out[7] = out[5];
}

/* IntDynaTijPW(typeT, ..., T_ID), DBEM1/dsquareelementdyna.cpp:940-994 */
static void int_t_pw(const quad_t* q, const mat_t* M, const elem_t* e, int type, const double* src, double n,
                     double* out)
{
    double T[9], pt[3], nor[3];
    rvec_t r;
    int i, j, k;
    for (k = 0; k < 9; ++k) out[k] = 0.0;
    for (i = 0; i < NUMPW2; ++i) {
        if (!pw_need_cal(M, e, type, n, e->rcen[i], src)) continue;
        for (j = 0; j < 9; ++j) {
            from_local(e, q->lpospw[i][j][0], q->lpospw[i][j][1], pt);
            get_r(src, pt, &r);
            normal_at(e, q->lpospw[i][j][0], q->lpospw[i][j][1], nor);
            dyna_t(M, type, T, n, &r, nor);
            double temp = q->pwgv[i][j] * jacobi_at(e, q->lpospw[i][j][0], q->lpospw[i][j][1]);
            for (k = 0; k < 9; ++k) out[k] += T[k] * temp;
        }
    }
}

/* IntDynaUijJudge / IntDynaTijJudge(typeT, ..., T_ID),
 * DBEM1/dsquareelementdyna.cpp:1603-1616, 1677-1690 */
static int judge_u(const quad_t* q, const mat_t* M, const elem_t* e, const double* src, double n, double* out)
{
    int f = need_cal(M, e, 1, n, src);
    if (f == 1) int_u_pw(q, M, e, src, n, out);
    else if (f == 2) int_u_regular(q, M, e, src, n, out);
    return f;
}

static int judge_t(const quad_t* q, const mat_t* M, const elem_t* e, int type, const double* src, double n, double* out)
{
    int f = need_cal(M, e, type, n, src);
    if (f == 1) int_t_pw(q, M, e, type, src, n, out);
    else if (f == 2) int_t_regular(q, M, e, src, n, out);
    return f;
}

/* Singular self-element integrals: InElementStaticTij()
 * (DBEM1/dsquareelement.cpp:2292-2427) and PthInElementIntDynamic
 * (DBEM1/dsquareelementdyna.cpp:239-490). */
static void self_integrals(const quad_t* q, const mat_t* M, elem_t* e)
{
    double ST[9], UT[9], temp, s1, s2, pt[3], nor[3], SR[4];
    int a, j, k, l;
    const double* src = e->node;
    /* static strongly singular part */
    double stat[9] = {0};
    double coef1 = -1.0 / (8.0 * PI_REF * (1.0 - M->v));
    double coef2 = 1.0 - 2.0 * M->v;
    double onJ[4][16], onN[4][16][3], onR[4][16][4];
    for (a = 0; a < 4; ++a)
        for (j = 0; j < 16; ++j) {
            s1 = q->sec_pos[a][0][j];
            s2 = q->sec_pos[a][1][j];
            onJ[a][j] = jacobi_at(e, s1, s2);
            normal_at(e, s1, s2, onN[a][j]);
            from_local(e, s1, s2, pt);
            onR[a][j][1] = pt[0] - src[0];
            onR[a][j][2] = pt[1] - src[1];
            onR[a][j][3] = pt[2] - src[2];
            onR[a][j][0] = sqrt(onR[a][j][1] * onR[a][j][1] + onR[a][j][2] * onR[a][j][2] + onR[a][j][3] * onR[a][j][3]);
        }
    double Jh[3], d1[3], d2[3];
    {
        double tJ = jacobi_at(e, q->lc[0][0], q->lc[0][1]);
        double n0[3];
        normal_at(e, q->lc[0][0], q->lc[0][1], n0);
        Jh[0] = tJ * n0[0];
        Jh[1] = tJ * n0[1];
        Jh[2] = tJ * n0[2];
        rdiff1(e, 0.0, 0.0, d1);
        rdiff2(e, 0.0, 0.0, d2);
    }
    for (a = 0; a < 4; ++a)
        for (j = 0; j < 16; ++j) {
            static_t(M, UT, onR[a][j], onN[a][j]);
            temp = q->sec_val[a][j] * onJ[a][j];
            for (l = 0; l < 9; ++l) stat[l] += UT[l] * temp;
        }
    for (a = 0; a < 4; ++a)
        for (j = 0; j < 4; ++j) {
            double A[6], F[9], th = q->line_pos[a][j];
            A[1] = d1[0] * cos(th) + d2[0] * sin(th);
            A[2] = d1[1] * cos(th) + d2[1] * sin(th);
            A[3] = d1[2] * cos(th) + d2[2] * sin(th);
            A[0] = sqrt(A[1] * A[1] + A[2] * A[2] + A[3] * A[3]);
            A[4] = A[0] * A[0] * A[0];
            A[5] = A[4] * A[0] * A[0];
            fij_minus_one(F, A, Jh, coef1, coef2);
            for (l = 0; l < 4; ++l) {
                double fvs = q->fm1_sec[a][l * 4 + j];
                for (k = 0; k < 9; ++k) stat[k] -= F[k] * fvs;
            }
            double fvl = q->fm1_line[a][j];
            for (k = 0; k < 9; ++k) stat[k] += F[k] * fvl;
        }
    /* dynamic parts in polar sub-patches */
    double u1[9] = {0}, t1[9] = {0}, t2[9] = {0};
    for (a = 0; a < 4; ++a)
        for (k = 0; k < SINNUMPW2; ++k)
            for (l = 0; l < 9; ++l) {
                rvec_t r;
                s1 = q->secpw_pos[a][0][k][l];
                s2 = q->secpw_pos[a][1][k][l];
                double Jac = jacobi_at(e, s1, s2);
                from_local(e, s1, s2, pt);
                get_r(src, pt, &r);
                dyna_u(M, UT, 0.0, &r);
                temp = q->secpw_val[a][k][l] * Jac;
                u1[0] += UT[0] * temp; u1[1] += UT[1] * temp; u1[2] += UT[2] * temp;
                u1[4] += UT[4] * temp; u1[5] += UT[5] * temp; u1[8] += UT[8] * temp;
            }
    u1[3] = u1[1]; u1[6] = u1[2]; u1[7] = u1[5];
    for (a = 0; a < 4; ++a)
        for (k = 0; k < SINNUMPW2; ++k)
            for (l = 0; l < 9; ++l) {
                rvec_t r;
                double D1[9], D2[9];
                s1 = q->secpw_pos[a][0][k][l];
                s2 = q->secpw_pos[a][1][k][l];
                double Jac = jacobi_at(e, s1, s2);
                normal_at(e, s1, s2, nor);
                from_local(e, s1, s2, pt);
                get_r(src, pt, &r);
                dyna_t(M, 1, D1, 0.0, &r, nor);
                dyna_t(M, 2, D2, 1.0, &r, nor);
                SR[0] = r.R[1]; SR[1] = r.RI[1]; SR[2] = r.RI[2]; SR[3] = r.RI[3];
                static_t(M, ST, SR, nor);
                temp = q->secpw_val[a][k][l] * Jac;
                for (j = 0; j < 9; ++j) {
                    t1[j] += (D1[j] - ST[j]) * temp;
                    t2[j] += (D2[j] - ST[j]) * temp;
                }
            }
    for (j = 0; j < 9; ++j) {
        t1[j] += stat[j];
        t2[j] += stat[j];
    }
    t1[0] += 0.5; t1[4] += 0.5; t1[8] += 0.5;
    memcpy(e->on_u1, u1, sizeof u1);
    memcpy(e->on_t1, t1, sizeof t1);
    memcpy(e->on_t2, t2, sizeof t2);
}

/* ConvertUnknownCoef / ConvertKnownCoef(long T_ID) for BCID 123 and 456
 * (DBEM1/dsquareelement.cpp:2756-2868, 3281-3394):
 * out[3m+i] = sign * sum_j K[3j+i] * R[3m+j], sign -1 for U on 123-unknown /
 * T on 123-known, +1 for T on 456-unknown / U on 456-known. */
static void convert_block(const double* K, const double* R, double sign, double* out)
{
    int i, j, m;
    for (i = 0; i < 9; ++i) out[i] = 0.0;
    for (i = 0; i < 3; ++i)
        for (j = 0; j < 3; ++j)
            for (m = 0; m < 3; ++m) {
                if (sign < 0)
                    out[3 * j + i] -= K[3 * m + i] * R[3 * j + m];
                else
                    out[3 * j + i] += K[3 * m + i] * R[3 * j + m];
            }
}

/* Step0 coefficient block for (source point, field element) with the
 * field element's effective BCID, FlagDynaMethod 2:
 * RegularIntUnknownCoef / RegularIntKnownCoef (DBEM1/dsquareelement.cpp:
 * 4215-4550, 5157-5492), InElementIntUnknownCoef / InElementIntKnownCoef
 * (:5922-6078, 6476-6632).  unknown = 1: the kernel multiplying the
 * unknown (T for 456, U for 123); unknown = 0: the known kernel.
 * Returns 0 when the pair contributes nothing. */
static int step0_block(const quad_t* q, const mat_t* M, const elem_t* e, int self, const double* src, int bcid,
                       int unknown, double* out)
{
    int useU = unknown ? (bcid == 123) : (bcid == 456);
    double K[9], tmp[9];
    int i;
    for (i = 0; i < 9; ++i) K[i] = 0.0;
    if (self) {
        if (useU) {
            for (i = 0; i < 9; ++i) K[i] += 4.0 * e->on_u1[i];
            int_u_pw(q, M, e, src, 1.0, tmp);
            for (i = 0; i < 9; ++i) K[i] += tmp[i];
        } else {
            for (i = 0; i < 9; ++i) {
                K[i] += 4.0 * e->on_t1[i];
                K[i] += e->on_t2[i];
            }
            int_t_pw(q, M, e, 1, src, 1.0, tmp);
            for (i = 0; i < 9; ++i) K[i] += tmp[i];
        }
    } else {
        int f0 = need_cal(M, e, 1, 0.0, src);
        int fsum = f0;
        if (f0 == 1 || f0 == 2) {
            if (useU) {
                if (f0 == 1) int_u_pw(q, M, e, src, 0.0, tmp);
                else int_u_regular(q, M, e, src, 0.0, tmp);
                for (i = 0; i < 9; ++i) K[i] += 4.0 * tmp[i];
            } else {
                if (f0 == 1) int_t_pw(q, M, e, 1, src, 0.0, tmp);
                else int_t_regular(q, M, e, src, 0.0, tmp);
                for (i = 0; i < 9; ++i) K[i] += 4.0 * tmp[i];
                if (f0 == 1) int_t_pw(q, M, e, 2, src, 1.0, tmp);
                else int_t_regular(q, M, e, src, 1.0, tmp);
                for (i = 0; i < 9; ++i) K[i] += tmp[i];
            }
        }
        int f1 = need_cal(M, e, 1, 1.0, src);
        fsum += f1;
        if (f1 == 1 || f1 == 2) {
            if (useU) {
                if (f1 == 1) int_u_pw(q, M, e, src, 1.0, tmp);
                else int_u_regular(q, M, e, src, 1.0, tmp);
            } else {
                if (f1 == 1) int_t_pw(q, M, e, 1, src, 1.0, tmp);
                else int_t_regular(q, M, e, src, 1.0, tmp);
            }
            for (i = 0; i < 9; ++i) K[i] += tmp[i];
        }
        if (!fsum) return 0;
    }
    double sign = unknown ? (bcid == 123 ? -1.0 : 1.0) : (bcid == 456 ? 1.0 : -1.0);
    convert_block(K, e->trans, sign, out);
    return 1;
}

/* ------------------------------------------------------------------ */
/* Block builder: MultiDomainCCSRBuilder::AddBlock / Build             */
/* (DBEM1/multidomain.cpp:1120-1214).  Keys are unique per assembly    */
/* pass except MTS, where T2 then T1 land on the same key; entries are */
/* kept per row in insertion order and sorted by column on build.      */
/* ------------------------------------------------------------------ */
typedef struct {
    int32_t col;
    double v[9];
} entry_t;

typedef struct {
    int64_t rows, cols;
    int64_t* n;
    int64_t* cap;
    entry_t** e;
} builder_t;

static void b_init(builder_t* b, int64_t rows, int64_t cols)
{
    b->rows = rows;
    b->cols = cols;
    b->n = calloc(rows, sizeof(int64_t));
    b->cap = calloc(rows, sizeof(int64_t));
    b->e = calloc(rows, sizeof(entry_t*));
}

static void b_free(builder_t* b)
{
    for (int64_t i = 0; i < b->rows; ++i) free(b->e[i]);
    free(b->n);
    free(b->cap);
    free(b->e);
    memset(b, 0, sizeof *b);
}

static double maxabs9(const double* v)
{
    double m = 0.0;
    for (int i = 0; i < 9; ++i)
        if (fabs(v[i]) > m) m = fabs(v[i]);
    return m;
}

/* block9 in the element routines' column-major form; stored transposed */
static void b_add(builder_t* b, int64_t row, int64_t col, double sign, const double* block9)
{
    int i, r, c;
    if (row < 0 || row >= b->rows || col < 0 || col >= b->cols) return;
    int zero = 1, finite = 1;
    for (i = 0; i < 9; ++i) {
        if (block9[i] != 0.0) zero = 0;
        if (!(block9[i] == block9[i]) || fabs(block9[i]) > 1.7976931348623157e308) finite = 0;
    }
    if (sign == 0.0 || zero || maxabs9(block9) <= 1.0e-14 || !finite) return;
    entry_t* t = 0;
    for (int64_t k = 0; k < b->n[row]; ++k)
        if (b->e[row][k].col == col) { t = &b->e[row][k]; break; }
    if (!t) {
        if (b->n[row] == b->cap[row]) {
            b->cap[row] = b->cap[row] ? 2 * b->cap[row] : 16;
            b->e[row] = realloc(b->e[row], b->cap[row] * sizeof(entry_t));
        }
        t = &b->e[row][b->n[row]++];
        t->col = (int32_t)col;
        for (i = 0; i < 9; ++i) t->v[i] = 0.0;
    }
    for (r = 0; r < 3; ++r)
        for (c = 0; c < 3; ++c) t->v[r * 3 + c] += sign * block9[c * 3 + r];
    if (maxabs9(t->v) <= 1.0e-14) {
        int64_t k = t - b->e[row];
        memmove(&b->e[row][k], &b->e[row][k + 1], (b->n[row] - k - 1) * sizeof(entry_t));
        b->n[row]--;
    }
}

typedef struct {
    int64_t n_rows, nnz;
    int32_t* row_ptr;
    int32_t* col;
    double* val;
} ccsr_t;

static int cmp_entry(const void* a, const void* b)
{
    return ((const entry_t*)a)->col - ((const entry_t*)b)->col;
}

static void b_build(builder_t* b, ccsr_t* out)
{
    int64_t nnz = 0, r, k;
    for (r = 0; r < b->rows; ++r) nnz += b->n[r];
    out->n_rows = b->rows;
    out->nnz = nnz;
    out->row_ptr = malloc((b->rows + 1) * sizeof(int32_t));
    out->col = malloc((nnz ? nnz : 1) * sizeof(int32_t));
    out->val = malloc((nnz ? nnz : 1) * 9 * sizeof(double));
    out->row_ptr[0] = 0;
    int64_t p = 0;
    for (r = 0; r < b->rows; ++r) {
        qsort(b->e[r], b->n[r], sizeof(entry_t), cmp_entry);
        for (k = 0; k < b->n[r]; ++k, ++p) {
            out->col[p] = b->e[r][k].col;
            memcpy(out->val + 9 * p, b->e[r][k].v, 9 * sizeof(double));
        }
        out->row_ptr[r + 1] = (int32_t)p;
    }
}

static void ccsr_free(ccsr_t* m)
{
    free(m->row_ptr);
    free(m->col);
    free(m->val);
    memset(m, 0, sizeof *m);
}

/* SparseMul(CCSRMat&), DBEM1/mat_vec.cpp:2273-2300 (0-based vectors) */
static void spmv(const ccsr_t* M, const double* x, double* b)
{
    for (int64_t i = 0; i < M->n_rows; ++i) {
        double b0 = 0.0, b1 = 0.0, b2 = 0.0;
        for (int32_t j = M->row_ptr[i]; j < M->row_ptr[i + 1]; ++j) {
            const double* v = M->val + 9 * (int64_t)j;
            const double* xc = x + 3 * (int64_t)M->col[j];
            b0 += v[0] * xc[0] + v[1] * xc[1] + v[2] * xc[2];
            b1 += v[3] * xc[0] + v[4] * xc[1] + v[5] * xc[2];
            b2 += v[6] * xc[0] + v[7] * xc[1] + v[8] * xc[2];
        }
        b[3 * i] = b0;
        b[3 * i + 1] = b1;
        b[3 * i + 2] = b2;
    }
}

/* ------------------------------------------------------------------ */
/* Problem, DOF map (GlobalDofMap::Build, DBEM1/multidomain.cpp:777-900) */
/* ------------------------------------------------------------------ */
typedef struct {
    int64_t block;
    double sign;
    int known;
} vref_t;

struct orc_problem {
    int64_t E, D, I;
    int32_t nstep, restart, max_leaf;
    double tol, dt, max_length;
    quad_t q;
    mat_t* mats;
    elem_t* el;
    int64_t* itf; /* I*5 */
    int64_t* dom_begin;
    int64_t* dom_count;
    /* dof map */
    vref_t *uref, *tref, *hu, *ht;
    int64_t* pref;
    int64_t n_unknown, n_known, n_hist;
    /* matrices */
    int assembled;
    ccsr_t A, K;
    int32_t n_hist_k;
    int32_t n_hist_alloc; /* history steps assembled (>= n_hist_k; the rest are empty) */
    ccsr_t* mts; /* [n_hist_alloc], index k-1 */
    ccsr_t* mgs;
    /* preconditioner */
    int64_t n_leaves;
    int64_t *repid, *leaf_begin, *leaf_count;
    double** leaf_inv;
};

static int build_dofmap(orc_problem* p)
{
    int64_t E = p->E, i;
    p->uref = calloc(E, sizeof(vref_t));
    p->tref = calloc(E, sizeof(vref_t));
    p->hu = calloc(E, sizeof(vref_t));
    p->ht = calloc(E, sizeof(vref_t));
    p->pref = malloc(E * sizeof(int64_t));
    char* side = calloc(E, 1);
    int64_t nu = 0, nk = 0, nh = 0;
    for (i = 0; i < E; ++i) p->pref[i] = -1;
    for (i = 0; i < p->I; ++i) {
        int64_t a = p->itf[5 * i + 1], b = p->itf[5 * i + 3];
        double s = p->itf[5 * i + 4] == 0 ? -1.0 : (double)p->itf[5 * i + 4];
        int64_t ub = nu++, tb = nu++;
        p->uref[a] = (vref_t){ub, 1.0, 0};
        p->uref[b] = (vref_t){ub, 1.0, 0};
        p->tref[a] = (vref_t){tb, 1.0, 0};
        p->tref[b] = (vref_t){tb, s, 0};
        p->pref[a] = ub;
        p->pref[b] = tb;
        p->hu[a] = (vref_t){nh, 1.0, 0};
        p->hu[b] = (vref_t){nh, 1.0, 0};
        p->ht[a] = (vref_t){nh, 1.0, 0};
        p->ht[b] = (vref_t){nh, s, 0};
        nh++;
        side[a] = side[b] = 1;
    }
    for (i = 0; i < E; ++i) {
        if (side[i]) continue;
        if (p->el[i].bcid == 123) {
            int64_t tb = nu++;
            p->uref[i] = (vref_t){nk++, 1.0, 1};
            p->tref[i] = (vref_t){tb, 1.0, 0};
            p->pref[i] = tb;
        } else {
            int64_t ub = nu++;
            p->uref[i] = (vref_t){ub, 1.0, 0};
            p->tref[i] = (vref_t){nk++, 1.0, 1};
            p->pref[i] = ub;
        }
        p->hu[i] = (vref_t){nh, 1.0, 0};
        p->ht[i] = (vref_t){nh, 1.0, 0};
        nh++;
    }
    free(side);
    p->n_unknown = nu;
    p->n_known = nk;
    p->n_hist = nh;
    if (nu != E) {
        snprintf(g_err, sizeof g_err, "unknown blocks %lld != equation blocks %lld", (long long)nu, (long long)E);
        return 0;
    }
    return 1;
}

orc_problem* orc_create(int64_t n_points, const double* points, int64_t n_elements, const int64_t* elements,
                        const int32_t* bcid, int32_t n_domains, const double* materials,
                        int64_t n_interfaces, const int64_t* interfaces, double card_E, double card_nu,
                        double card_rho, double beta, double gap, int32_t n_steps, int32_t restart, double tol,
                        int32_t max_leaf, double max_length)
{
    int64_t i, d;
    g_err[0] = 0;
    if (n_elements <= 0 || n_domains <= 0 || n_domains > n_elements || n_steps < 0 || restart <= 0) {
        snprintf(g_err, sizeof g_err, "invalid sizes");
        return NULL;
    }
    for (i = 0; i < n_elements; ++i) {
        if (bcid[i] != 123 && bcid[i] != 456) {
            snprintf(g_err, sizeof g_err, "element %lld has BCID %d; only 123 and 456 are supported",
                     (long long)i, bcid[i]);
            return NULL;
        }
        for (int c = 0; c < 8; ++c)
            if (elements[8 * i + c] < 0 || elements[8 * i + c] >= n_points) {
                snprintf(g_err, sizeof g_err, "element %lld references point out of range", (long long)i);
                return NULL;
            }
    }
    orc_problem* p = calloc(1, sizeof *p);
    p->E = n_elements;
    p->D = n_domains;
    p->I = n_interfaces;
    p->nstep = n_steps;
    p->restart = restart;
    p->tol = tol;
    p->max_leaf = max_leaf;
    p->max_length = max_length;
    quad_init(&p->q, gap);
    /* dt = Beta * AveEleSize / c1 (DBEM1/DBEM.cpp:909-914, GetEleSize :2383-2396) */
    double ave = 0.0;
    for (i = 0; i < n_elements; ++i)
        ave += dist3(points + 3 * elements[8 * i], points + 3 * elements[8 * i + 1]);
    ave /= n_elements;
    double G = card_E / 2.0 / (1 + card_nu);
    double c1 = sqrt((2.0 - 2.0 * card_nu) / (1.0 - 2.0 * card_nu) * G / card_rho);
    p->dt = beta * ave / c1;
    p->mats = malloc(n_domains * sizeof(mat_t));
    for (d = 0; d < n_domains; ++d) {
        double Gd = materials[3 * d] / 2.0 / (1.0 + materials[3 * d + 1]);
        p->mats[d] = build_mat(materials[3 * d + 1], Gd, materials[3 * d + 2], p->dt);
    }
    /* contiguous equal element ranges, DBEM1/multidomain.cpp:1413-1436 */
    p->dom_begin = malloc(n_domains * sizeof(int64_t));
    p->dom_count = malloc(n_domains * sizeof(int64_t));
    p->el = calloc(n_elements, sizeof(elem_t));
    int64_t b = 0;
    for (d = 0; d < n_domains; ++d) {
        int64_t c = n_elements / n_domains + (d < n_elements % n_domains ? 1 : 0);
        p->dom_begin[d] = b;
        p->dom_count[d] = c;
        for (i = b; i < b + c; ++i) p->el[i].domain = (int)d;
        b += c;
    }
    p->itf = malloc((n_interfaces ? n_interfaces : 1) * 5 * sizeof(int64_t));
    memcpy(p->itf, interfaces, n_interfaces * 5 * sizeof(int64_t));
    char* used = calloc(n_elements, 1);
    for (i = 0; i < n_interfaces; ++i) {
        int64_t dA = interfaces[5 * i], eA = interfaces[5 * i + 1], dB = interfaces[5 * i + 2],
                eB = interfaces[5 * i + 3];
        if (dA < 0 || dA >= n_domains || dB < 0 || dB >= n_domains || dA == dB || eA < 0 || eA >= n_elements ||
            eB < 0 || eB >= n_elements || p->el[eA].domain != dA || p->el[eB].domain != dB || used[eA] ||
            used[eB]) {
            snprintf(g_err, sizeof g_err, "invalid interface %lld", (long long)i);
            free(used);
            orc_destroy(p);
            return NULL;
        }
        used[eA] = used[eB] = 1;
        if (p->itf[5 * i + 4] == 0) p->itf[5 * i + 4] = -1;
    }
    for (i = 0; i < n_elements; ++i) {
        elem_t* e = &p->el[i];
        e->bcid = bcid[i];
        e->surface = used[i];
        /* GeoInit, DBEM1/dsquareelement.cpp:332-382 */
        for (int c = 0; c < 3; ++c) {
            double v[8];
            for (int k = 0; k < 8; ++k) v[k] = points[3 * elements[8 * i + k] + c];
            get_coef(e->cc[c], v);
        }
        for (int k = 0; k < NUMPW2; ++k) from_local(e, p->q.cenpw[k][0], p->q.cenpw[k][1], e->rcen[k]);
        from_local(e, 0.0, 0.0, e->center);
        e->radius = -1.0;
        for (int k = 0; k < 8; ++k) {
            double dd = dist3(e->center, points + 3 * elements[8 * i + k]);
            if (e->radius < dd) e->radius = dd;
        }
        e->radius_pw = e->radius / NUMPW;
        /* GetNodeInfo (DBEM1/DBEM.cpp:1409-1427): node at the centre */
        from_local(e, 0.0, 0.0, e->node);
        /* PthPhyInit, DBEM1/dsquareelement.cpp:402-418 */
        translate_matrix(e, p->q.lc[0][0], p->q.lc[0][1], e->trans);
        self_integrals(&p->q, &p->mats[e->domain], e);
    }
    free(used);
    if (!build_dofmap(p)) {
        orc_destroy(p);
        return NULL;
    }
    return p;
}

void orc_destroy(orc_problem* p)
{
    if (!p) return;
    free(p->q.secpw_pos);
    free(p->q.secpw_val);
    free(p->mats);
    free(p->el);
    free(p->itf);
    free(p->dom_begin);
    free(p->dom_count);
    free(p->uref);
    free(p->tref);
    free(p->hu);
    free(p->ht);
    free(p->pref);
    ccsr_free(&p->A);
    ccsr_free(&p->K);
    for (int32_t k = 0; k < p->n_hist_alloc; ++k) {
        ccsr_free(&p->mts[k]);
        ccsr_free(&p->mgs[k]);
    }
    free(p->mts);
    free(p->mgs);
    free(p->repid);
    free(p->leaf_begin);
    free(p->leaf_count);
    if (p->leaf_inv)
        for (int64_t l = 0; l < p->n_leaves; ++l) free(p->leaf_inv[l]);
    free(p->leaf_inv);
    free(p);
}

double orc_dt(const orc_problem* p) { return p->dt; }

void orc_dof_counts(const orc_problem* p, int64_t out[3])
{
    out[0] = p->n_unknown;
    out[1] = p->n_known;
    out[2] = p->n_hist;
}

void orc_geometry(const orc_problem* p, double* coordcoef, double* center, double* radius, double* radius_pw,
                  double* rcen_pw, double* transmat, double* on_u1, double* on_t1, double* on_t2)
{
    for (int64_t i = 0; i < p->E; ++i) {
        const elem_t* e = &p->el[i];
        if (coordcoef) memcpy(coordcoef + 24 * i, e->cc, 24 * sizeof(double));
        if (center) memcpy(center + 3 * i, e->center, 3 * sizeof(double));
        if (radius) radius[i] = e->radius;
        if (radius_pw) radius_pw[i] = e->radius_pw;
        if (rcen_pw) memcpy(rcen_pw + 108 * i, e->rcen, 108 * sizeof(double));
        if (transmat) memcpy(transmat + 9 * i, e->trans, 9 * sizeof(double));
        if (on_u1) memcpy(on_u1 + 9 * i, e->on_u1, 9 * sizeof(double));
        if (on_t1) memcpy(on_t1 + 9 * i, e->on_t1, 9 * sizeof(double));
        if (on_t2) memcpy(on_t2 + 9 * i, e->on_t2, 9 * sizeof(double));
    }
}

/* ------------------------------------------------------------------ */
/* Assembly                                                            */
/* ------------------------------------------------------------------ */

/* Interface transform of the B side: BuildLocalTransformFromReference
 * (DBEM1/multidomain.cpp:1603-1645) and TransformColumnBlock9 (:1668-1680) */
static void interface_transform(const orc_problem* p, int64_t ele, double* T)
{
    int i;
    for (i = 0; i < 9; ++i) T[i] = 0.0;
    T[0] = T[4] = T[8] = 1.0;
    for (int64_t k = 0; k < p->I; ++k) {
        if (p->itf[5 * k + 1] == ele) return;
        if (p->itf[5 * k + 3] == ele) {
            const double* sb = p->el[ele].trans;
            const double* sa = p->el[p->itf[5 * k + 1]].trans;
            for (int s = 0; s < 3; ++s)
                for (int r = 0; r < 3; ++r) {
                    double dot = 0.0;
                    for (int ax = 0; ax < 3; ++ax) dot += sb[s * 3 + ax] * sa[r * 3 + ax];
                    T[s * 3 + r] = dot;
                }
            return;
        }
    }
}

static void transform_block(const double* b9, const double* T, double* out)
{
    for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q) {
            double v = 0.0;
            for (int c = 0; c < 3; ++c) v += b9[c * 3 + r] * T[c * 3 + q];
            out[q * 3 + r] = v;
        }
}

/* AssembleMultiDomainStep0 (DBEM1/multidomain.cpp:2256-2327); the pthread
 * variant the solver uses gives the same blocks because every (row, col)
 * key receives exactly one contribution. */
static void assemble_step0(orc_problem* p, builder_t* ub, builder_t* kb)
{
    double blk[9], tb[9], T[9];
    for (int64_t d = 0; d < p->D; ++d) {
        const mat_t* M = &p->mats[d];
        for (int64_t s = p->dom_begin[d]; s < p->dom_begin[d] + p->dom_count[d]; ++s) {
            const double* src = p->el[s].node;
            for (int64_t f = p->dom_begin[d]; f < p->dom_begin[d] + p->dom_count[d]; ++f) {
                const elem_t* e = &p->el[f];
                int self = f == s;
                if (e->surface) {
                    interface_transform(p, f, T);
                    if (step0_block(&p->q, M, e, self, src, 456, 1, blk)) {
                        transform_block(blk, T, tb);
                        b_add(ub, s, p->uref[f].block, p->uref[f].sign, tb);
                    }
                    if (step0_block(&p->q, M, e, self, src, 123, 1, blk)) {
                        transform_block(blk, T, tb);
                        b_add(ub, s, p->tref[f].block, p->tref[f].sign, tb);
                    }
                } else {
                    const vref_t* ru = e->bcid == 123 ? &p->tref[f] : &p->uref[f];
                    const vref_t* rk = e->bcid == 123 ? &p->uref[f] : &p->tref[f];
                    if (step0_block(&p->q, M, e, self, src, e->bcid, 1, blk) && !ru->known)
                        b_add(ub, s, ru->block, ru->sign, blk);
                    if (step0_block(&p->q, M, e, self, src, e->bcid, 0, blk) && rk->known)
                        b_add(kb, s, rk->block, rk->sign, blk);
                }
            }
        }
    }
}

/* AssembleMultiDomainHistoryStep (DBEM1/multidomain.cpp:2329-2378) with
 * ComputeT2Block / ComputeT1Block / ComputeUBlock (:1739-1813) */
static void assemble_history(orc_problem* p, int k, builder_t* tb, builder_t* gb)
{
    double blk[9];
    for (int64_t d = 0; d < p->D; ++d) {
        const mat_t* M = &p->mats[d];
        for (int64_t s = p->dom_begin[d]; s < p->dom_begin[d] + p->dom_count[d]; ++s) {
            const double* src = p->el[s].node;
            for (int64_t f = p->dom_begin[d]; f < p->dom_begin[d] + p->dom_count[d]; ++f) {
                const elem_t* e = &p->el[f];
                if (k <= 1 && f == s) {
                    b_add(tb, s, p->hu[f].block, p->hu[f].sign, e->on_t2);
                } else if (judge_t(&p->q, M, e, 2, src, (double)k, blk)) {
                    b_add(tb, s, p->hu[f].block, p->hu[f].sign, blk);
                }
                if (judge_t(&p->q, M, e, 1, src, (double)k, blk)) b_add(tb, s, p->hu[f].block, p->hu[f].sign, blk);
                if (judge_u(&p->q, M, e, src, (double)k, blk)) b_add(gb, s, p->ht[f].block, p->ht[f].sign, blk);
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Mapped-leaf preconditioner: octree of element centres (AssignCubeSize, */
/* InitRoot, CreateTree, CreateLeafPointer, RenumberPointID;            */
/* DBEM1/geo.cpp:6-39,109-137, DBEM1/tree.cpp:12-325) and              */
/* BuildMappedLeafPreConditioner (DBEM1/multidomain.cpp:3493-3565).     */
/* A node's point list is a linked list built by head insertion, so a  */
/* child's points are in reverse order of arrival.                      */
/* ------------------------------------------------------------------ */
typedef struct {
    double c[3];
    double len;
} cube_t;

static int cube_isin(const double* pt, const cube_t* cb)
{
    double l = 0.5 * cb->len;
    for (int i = 0; i < 3; i++) {
        double ds = cb->c[i] - pt[i];
        if (ds * ds > l * l * 1.0001) return 0;
    }
    return 1;
}

static void sub_cube(const cube_t* f, cube_t* ch, int pos)
{
    ch->len = 0.5 * f->len;
    double half = 0.5 * ch->len;
    int bit = 1;
    for (int i = 0; i < 3; i++) {
        ch->c[i] = f->c[i] + ((bit & pos) == 0 ? -1 : 1) * half;
        bit <<= 1;
    }
}

static void tree_split(const orc_problem* p, const cube_t* cb, const int64_t* list, int64_t n, int64_t max_point,
                       int64_t* repid, int64_t* pos, int64_t* lb, int64_t* lc, int64_t* nleaf)
{
    if (n <= max_point) {
        lb[*nleaf] = *pos;
        lc[*nleaf] = n;
        (*nleaf)++;
        for (int64_t i = 0; i < n; ++i) repid[(*pos)++] = list[i];
        return;
    }
    cube_t ch[8];
    int64_t* arrive[8];
    int64_t cnt[8];
    for (int i = 0; i < 8; ++i) {
        sub_cube(cb, &ch[i], i);
        arrive[i] = malloc(n * sizeof(int64_t));
        cnt[i] = 0;
    }
    for (int64_t k = 0; k < n; ++k) {
        const double* pt = p->el[list[k]].node;
        int near = -1;
        for (int i = 0; i < 8; ++i)
            if (cube_isin(pt, &ch[i])) { near = i; break; }
        if (near < 0) {
            double best = dist3(pt, ch[0].c);
            near = 0;
            for (int i = 1; i < 8; ++i) {
                double dd = dist3(pt, ch[i].c);
                if (best > dd) { best = dd; near = i; }
            }
        }
        arrive[near][cnt[near]++] = list[k];
    }
    for (int i = 0; i < 8; ++i) {
        if (cnt[i]) {
            /* head insertion reverses the arrival order */
            for (int64_t a = 0, b = cnt[i] - 1; a < b; ++a, --b) {
                int64_t t = arrive[i][a];
                arrive[i][a] = arrive[i][b];
                arrive[i][b] = t;
            }
            tree_split(p, &ch[i], arrive[i], cnt[i], max_point, repid, pos, lb, lc, nleaf);
        }
        free(arrive[i]);
    }
}

/* inv_mat: full-pivot Gauss-Jordan in place, DBEM1/lin_comp.cpp:83-183.
 * a is n x n row-major; returns 0 when a pivot is <= 1e-10 (the reference
 * ignores this and keeps the partially inverted matrix). */
static int inv_mat(double* a, int64_t n)
{
#define AA(i, j) a[((i)-1) * n + ((j)-1)]
    int64_t k, i, j;
    int64_t* is = malloc((n + 1) * sizeof(int64_t));
    int64_t* js = malloc((n + 1) * sizeof(int64_t));
    double t, d, temp;
    for (k = 1; k <= n; k++) {
        d = 0.0;
        for (i = k; i <= n; i++)
            for (j = k; j <= n; j++) {
                t = sqrt(AA(i, j) * AA(i, j));
                if (t > d) { d = t; is[k] = i; js[k] = j; }
            }
        if (d <= 0.0000000001) {
            free(is);
            free(js);
            return 0;
        }
        for (j = 1; j <= n; j++) { i = is[k]; temp = AA(k, j); AA(k, j) = AA(i, j); AA(i, j) = temp; }
        for (i = 1; i <= n; i++) { j = js[k]; temp = AA(i, k); AA(i, k) = AA(i, j); AA(i, j) = temp; }
        AA(k, k) = 1.0 / AA(k, k);
        for (j = 1; j <= n; j++)
            if (j != k) AA(k, j) *= AA(k, k);
        for (i = 1; i <= n; i++)
            if (i != k)
                for (j = 1; j <= n; j++)
                    if (j != k) AA(i, j) -= AA(i, k) * AA(k, j);
        for (i = 1; i <= n; i++)
            if (i != k) AA(i, k) *= -1.0 * AA(k, k);
    }
    for (k = n; k >= 1; k--) {
        for (j = 1; j <= n; j++) { i = js[k]; temp = AA(k, j); AA(k, j) = AA(i, j); AA(i, j) = temp; }
        for (i = 1; i <= n; i++) { j = is[k]; temp = AA(i, k); AA(i, k) = AA(i, j); AA(i, j) = temp; }
    }
    free(is);
    free(js);
    return 1;
#undef AA
}

static const double* find_block(const ccsr_t* M, int64_t row, int64_t col)
{
    for (int32_t j = M->row_ptr[row]; j < M->row_ptr[row + 1]; ++j)
        if (M->col[j] == col) return M->val + 9 * (int64_t)j;
    return NULL;
}

static void build_precond(orc_problem* p)
{
    int64_t N = p->E, i;
    double rmin[3], rmax[3], ml;
    for (i = 0; i < 3; ++i) rmin[i] = rmax[i] = p->el[0].node[i];
    for (int64_t k = 1; k < N; ++k)
        for (i = 0; i < 3; ++i) {
            if (rmin[i] > p->el[k].node[i]) rmin[i] = p->el[k].node[i];
            if (rmax[i] < p->el[k].node[i]) rmax[i] = p->el[k].node[i];
        }
    cube_t root;
    ml = rmax[0] - rmin[0];
    for (i = 0; i < 3; ++i) {
        if (ml < rmax[i] - rmin[i]) ml = rmax[i] - rmin[i];
        root.c[i] = rmin[i] + 0.5 * (rmax[i] - rmin[i]);
    }
    root.len = 1.02 * ml;
    int64_t* list = malloc(N * sizeof(int64_t));
    for (i = 0; i < N; ++i) list[i] = i;
    p->repid = malloc(N * sizeof(int64_t));
    p->leaf_begin = malloc(N * sizeof(int64_t));
    p->leaf_count = malloc(N * sizeof(int64_t));
    int64_t pos = 0, nleaf = 0;
    tree_split(p, &root, list, N, p->max_leaf, p->repid, &pos, p->leaf_begin, p->leaf_count, &nleaf);
    free(list);
    p->n_leaves = nleaf;
    p->leaf_inv = malloc(nleaf * sizeof(double*));
    for (int64_t l = 0; l < nleaf; ++l) {
        int64_t L = p->leaf_count[l], b = p->leaf_begin[l], n3 = 3 * L;
        double* m = calloc(n3 * n3, sizeof(double));
        for (int64_t r = 0; r < L; ++r) {
            int64_t row = p->repid[b + r];
            for (int64_t c = 0; c < L; ++c) {
                int64_t col = p->pref[p->repid[b + c]];
                const double* blk = find_block(&p->A, row, col);
                if (!blk) continue;
                for (int a = 0; a < 3; ++a)
                    for (int e = 0; e < 3; ++e) m[(3 * r + a) * n3 + 3 * c + e] = blk[3 * a + e];
            }
        }
        inv_mat(m, n3);
        p->leaf_inv[l] = m;
    }
}

/* GMRES_M_X, DBEM1/pre_gmres.cpp:837-895 */
static void precond_apply(const orc_problem* p, const double* X, double* B)
{
    int64_t n = 3 * p->E;
    for (int64_t i = 0; i < n; ++i) B[i] = 0.0;
    for (int64_t l = 0; l < p->n_leaves; ++l) {
        int64_t L = p->leaf_count[l], b = p->leaf_begin[l], n3 = 3 * L;
        const double* m = p->leaf_inv[l];
        for (int64_t j = 0; j < L; ++j) {
            int64_t a1 = 3 * p->pref[p->repid[b + j]];
            for (int64_t k = 0; k < L; ++k) {
                int64_t a2 = 3 * p->repid[b + k];
                for (int mm = 0; mm < 3; ++mm)
                    for (int nn = 0; nn < 3; ++nn) B[a1 + mm] += m[(3 * j + mm) * n3 + 3 * k + nn] * X[a2 + nn];
            }
        }
    }
}

static double norm2(const double* a, int64_t n)
{
    double r = 0.0;
    for (int64_t i = 0; i < n; ++i) r += a[i] * a[i];
    return sqrt(r);
}

/* gmres(..., CCSRMat&, ...), DBEM1/pre_gmres.cpp:1369-1605, maxit = 1 */
static void gmres(orc_problem* p, const double* b, double* x, int* flag, int* iter)
{
    int64_t n = 3 * p->E, k, l;
    int64_t rs = p->restart;
    double* r = calloc(n, sizeof(double));
    double* vh = calloc(n, sizeof(double));
    double* u = calloc(n, sizeof(double));
    double* u2 = calloc(n, sizeof(double));
    double* V = calloc(n * (rs + 1), sizeof(double)); /* column j at V + j*n */
    double* W = calloc(n * rs, sizeof(double));
    double* h = calloc(rs + 2, sizeof(double));
    double* q = calloc(rs + 2, sizeof(double));
    double* f = calloc(rs + 2, sizeof(double));
    double* QT = calloc((rs + 2) * (rs + 2), sizeof(double));
    double* R = calloc((rs + 1) * (rs + 1), sizeof(double));
#define QTm(i, j) QT[(i) * (rs + 2) + (j)]
#define Rm(i, j) R[(i) * (rs + 1) + (j)]
    double n2b = norm2(b, n);
    iter[0] = iter[1] = 0;
    for (k = 0; k < n; ++k) x[k] = 0.0;
    if (n2b == 0.0) { *flag = 0; goto done; }
    *flag = 1;
    double tolb = p->tol * n2b;
    spmv(&p->A, x, r);
    for (k = 0; k < n; ++k) r[k] = b[k] - r[k];
    if (norm2(r, n) <= tolb) { *flag = 0; goto done; }
    int stag = 0;
    precond_apply(p, r, vh);
    h[1] = norm2(vh, n);
    for (k = 0; k < n; ++k) V[k] = vh[k] / h[1];
    QTm(1, 1) = 1.0;
    double phibar = h[1];
    int64_t j;
    for (j = 1; j <= rs; ++j) {
        double* Vj = V + (j - 1) * n;
        spmv(&p->A, Vj, u2);
        precond_apply(p, u2, u);
        for (k = 1; k <= j; ++k) {
            double* Vk = V + (k - 1) * n;
            h[k] = 0.0;
            for (l = 0; l < n; ++l) h[k] += Vk[l] * u[l];
            for (l = 0; l < n; ++l) u[l] -= h[k] * Vk[l];
        }
        h[j + 1] = norm2(u, n);
        double* Vn = V + j * n;
        if (h[j + 1] <= 1.0e-12)
            for (k = 0; k < n; ++k) Vn[k] = 0.0;
        else
            for (k = 0; k < n; ++k) Vn[k] = u[k] / h[j + 1];
        for (k = 1; k <= j; ++k) {
            Rm(k, j) = 0.0;
            for (l = 1; l <= j; ++l) Rm(k, j) += QTm(k, l) * h[l];
        }
        double rt = Rm(j, j), c, s, temp;
        if (h[j + 1] == 0.0) { c = 1.0; s = 0.0; }
        else if (h[j + 1] * h[j + 1] > rt * rt) {
            temp = rt / h[j + 1];
            s = 1.0 / sqrt(1.0 + fabs(temp) * fabs(temp));
            c = -temp * s;
        } else {
            temp = h[j + 1] / rt;
            c = 1.0 / sqrt(1.0 + fabs(temp) * fabs(temp));
            s = -temp * c;
        }
        Rm(j, j) = c * rt - s * h[j + 1];
        for (k = 1; k <= j; ++k) q[k] = QTm(j, k);
        for (k = 1; k <= j; ++k) QTm(j, k) = c * q[k];
        for (k = 1; k <= j; ++k) QTm(j + 1, k) = s * q[k];
        QTm(j, j + 1) = -s;
        QTm(j + 1, j + 1) = c;
        f[j] = c * phibar;
        phibar = s * phibar;
        if (j < rs) {
            if (f[j] == 0.0) stag = 1;
            double* Wj = W + (j - 1) * n;
            for (k = 0; k < n; ++k) {
                Wj[k] = Vj[k] / Rm(j, j);
                for (l = 1; l <= j - 1; ++l) Wj[k] -= W[(l - 1) * n + k] * Rm(l, j) / Rm(j, j);
            }
            for (k = 0; k < n; ++k) x[k] += f[j] * Wj[k];
        } else {
            /* final restart column: x = x0 + V R^-1 f (x0 = 0) */
            double* Ri = calloc(rs * rs, sizeof(double));
            for (k = 0; k < rs; ++k)
                for (l = 0; l < rs; ++l) Ri[k * rs + l] = Rm(k + 1, l + 1);
            inv_mat(Ri, rs);
            for (k = 0; k < rs; ++k) {
                q[k + 1] = 0.0;
                for (l = 0; l < rs; ++l) q[k + 1] += Ri[k * rs + l] * f[l + 1];
            }
            free(Ri);
            for (k = 0; k < n; ++k) {
                double acc = 0.0;
                for (l = 1; l <= rs; ++l) acc += V[(l - 1) * n + k] * q[l];
                x[k] = acc;
            }
        }
        spmv(&p->A, x, vh);
        for (k = 0; k < n; ++k) vh[k] = b[k] - vh[k];
        if (norm2(vh, n) <= tolb) { *flag = 0; iter[0] = 1; iter[1] = (int)j; goto done; }
        if (stag) { *flag = 3; iter[0] = 1; iter[1] = (int)j; goto done; }
    }
    iter[0] = 1;
    iter[1] = (int)j;
done:
#undef QTm
#undef Rm
    free(r); free(vh); free(u); free(u2); free(V); free(W); free(h); free(q); free(f); free(QT); free(R);
}

/* ------------------------------------------------------------------ */
/* Public entry points                                                 */
/* ------------------------------------------------------------------ */
/* Replay of MultiDomainCCSRBuilder::AddBlock calls (DBEM1/multidomain.cpp:
 * 1120-1144) then Build (:1186-1210): call i adds sign[i] * blocks[9 i..]
 * (column-major) at (row[i], col[i]).  Returns the number of stored blocks;
 * fills row_ptr [rows + 1], col and val [nnz][9] (row-major) when given. */
int64_t orc_builder_replay(int64_t rows, int64_t cols, int64_t n, const int64_t* row, const int64_t* col,
                           const double* sign, const double* blocks, int32_t* row_ptr, int32_t* col_out,
                           double* val_out)
{
    builder_t b;
    ccsr_t m;
    b_init(&b, rows, cols);
    for (int64_t i = 0; i < n; ++i) b_add(&b, row[i], col[i], sign[i], blocks + 9 * i);
    b_build(&b, &m);
    b_free(&b);
    const int64_t nnz = m.nnz;
    if (row_ptr) memcpy(row_ptr, m.row_ptr, sizeof(int32_t) * (size_t)(rows + 1));
    if (col_out && nnz) memcpy(col_out, m.col, sizeof(int32_t) * (size_t)nnz);
    if (val_out && nnz) memcpy(val_out, m.val, sizeof(double) * 9 * (size_t)nnz);
    ccsr_free(&m);
    return nnz;
}

/* Last history step whose blocks can be nonzero: every kernel of step k is
 * skipped by NeedCal (DBEM1/dsquareelement.cpp:1156-1190) once
 * (k - 1) Dt >= (|c_e - s| + radius_e) / C2 for all source nodes s and field
 * elements e of a domain (T2 uses nn = k - 1, U and T1 nn = k); one step is
 * added against rounding in that comparison. */
static int32_t history_step_bound(const orc_problem* p)
{
    double steps = 0.0;
    for (int64_t d = 0; d < p->D; ++d) {
        const int64_t b = p->dom_begin[d], n = p->dom_count[d];
        double dmax = 0.0;
        for (int64_t e = b; e < b + n; ++e)
            for (int64_t q = b; q < b + n; ++q) {
                const double* c = p->el[e].center;
                const double* s = p->el[q].node;
                const double r = sqrt((c[0] - s[0]) * (c[0] - s[0]) + (c[1] - s[1]) * (c[1] - s[1]) +
                                      (c[2] - s[2]) * (c[2] - s[2])) + p->el[e].radius;
                if (r > dmax) dmax = r;
            }
        const double v = 1.0 + dmax / (p->mats[d].C2 * p->dt);
        if (v > steps) steps = v;
    }
    return (int32_t)(ceil(steps) + 1.0);
}

int32_t orc_history_step_bound(const orc_problem* p) { return history_step_bound(p); }

int32_t orc_assemble(orc_problem* p, int32_t kmax)
{
    builder_t ub, kb;
    b_init(&ub, p->E, p->n_unknown);
    b_init(&kb, p->E, p->n_known);
    assemble_step0(p, &ub, &kb);
    b_build(&ub, &p->A);
    b_build(&kb, &p->K);
    b_free(&ub);
    b_free(&kb);
    /* MaxN (DBEM1/multidomain.cpp:3718-3740) */
    int32_t maxn = p->nstep;
    double minc2dt = 1.0e308;
    for (int64_t d = 0; d < p->D; ++d)
        if (p->mats[d].C2Dt > 0.0 && p->mats[d].C2Dt < minc2dt) minc2dt = p->mats[d].C2Dt;
    for (int32_t i = 0; i <= p->nstep; ++i)
        if (minc2dt * i > p->max_length) { maxn = i; break; }
    if (kmax > 0 && kmax < maxn) maxn = kmax;
    if (kmax <= 0) {
        const int32_t kb = history_step_bound(p);
        if (kb < maxn) maxn = kb;
    }
    p->mts = calloc(maxn > 0 ? maxn : 1, sizeof(ccsr_t));
    p->mgs = calloc(maxn > 0 ? maxn : 1, sizeof(ccsr_t));
    int32_t last = 0, k;
    for (k = 1; k <= maxn; ++k) {
        builder_t tb, gb;
        b_init(&tb, p->E, p->n_hist);
        b_init(&gb, p->E, p->n_hist);
        assemble_history(p, k, &tb, &gb);
        b_build(&tb, &p->mts[k - 1]);
        b_build(&gb, &p->mgs[k - 1]);
        b_free(&tb);
        b_free(&gb);
        if (p->mts[k - 1].nnz || p->mgs[k - 1].nnz) last = k;
    }
    /* empty steps add exact zeros: keep steps 1..last (all maxn with kmax > 0) */
    p->n_hist_alloc = k - 1;
    p->n_hist_k = kmax > 0 ? k - 1 : last;
    build_precond(p);
    p->assembled = 1;
    return p->n_hist_k;
}

int32_t orc_matrix(const orc_problem* p, int32_t which, int32_t k, orc_ccsr* out)
{
    const ccsr_t* m = NULL;
    if (!p->assembled) return 0;
    if (which == 0) m = &p->A;
    else if (which == 1) m = &p->K;
    else if ((which == 2 || which == 3) && k >= 1 && k <= p->n_hist_k) m = which == 2 ? &p->mts[k - 1] : &p->mgs[k - 1];
    if (!m) return 0;
    out->n_rows = m->n_rows;
    out->nnz = m->nnz;
    out->row_ptr = m->row_ptr;
    out->col = m->col;
    out->val = m->val;
    return 1;
}

int64_t orc_precond_layout(const orc_problem* p, int64_t* repid, int64_t* leaf_begin, int64_t* leaf_count)
{
    if (!p->assembled) return 0;
    if (repid) memcpy(repid, p->repid, p->E * sizeof(int64_t));
    if (leaf_begin) memcpy(leaf_begin, p->leaf_begin, p->n_leaves * sizeof(int64_t));
    if (leaf_count) memcpy(leaf_count, p->leaf_count, p->n_leaves * sizeof(int64_t));
    return p->n_leaves;
}

/* The time loop of DynaGMRESSolverMultiDomainCCSR
 * (DBEM1/multidomain.cpp:3811-3893) with BuildKnownInputVectorFromBoundary
 * (:3047-3084), BuildConvolutionVector (:3201-3225), ScatterUnknownToBoundary
 * (:3086-3144), BoundaryValue::AllLocToAbs (DBEM1/dsquareelement.h:88-125)
 * and BuildPhysicalStateFromBoundary (:3162-3200). */
int32_t orc_march(orc_problem* p, const double* known, double* bd_lu, double* bd_lt, double* rhs_out,
                  double* x_out, int32_t* flags)
{
    if (!p->assembled) orc_assemble(p, 0);
    int64_t E = p->E, n = 3 * E, nh3 = 3 * p->n_hist, nk3 = 3 * p->n_known, i, s;
    int32_t N = p->nstep;
    memcpy(bd_lu, known, (N + 1) * n * sizeof(double));
    memset(bd_lt, 0, (N + 1) * n * sizeof(double));
    /* bd[0]: Convert (456 swaps lu/lt) then local -> global */
    for (i = 0; i < E; ++i)
        if (p->el[i].bcid == 456)
            for (int c = 0; c < 3; ++c) {
                double t = bd_lt[3 * i + c];
                bd_lt[3 * i + c] = bd_lu[3 * i + c];
                bd_lu[3 * i + c] = t;
            }
    double* XU = calloc((N + 1) * nh3, sizeof(double));
    double* XT = calloc((N + 1) * nh3, sizeof(double));
    double* kv = calloc(nk3 ? nk3 : 1, sizeof(double));
    double* rhs = calloc(n, sizeof(double));
    double* tmp = calloc(n, sizeof(double));
    double* cv = calloc(nh3 ? nh3 : 1, sizeof(double));
    double* x = calloc(n, sizeof(double));
    int32_t solved = 0;
    for (s = 0; s <= N; ++s) {
        double* lu = bd_lu + s * n;
        double* lt = bd_lt + s * n;
        if (s > 0) {
            /* known vector from bd[s].lu */
            memset(kv, 0, nk3 * sizeof(double));
            for (i = 0; i < E; ++i) {
                if (p->el[i].surface) continue;
                const vref_t* r = p->el[i].bcid == 123 ? &p->uref[i] : &p->tref[i];
                if (!r->known) continue;
                for (int c = 0; c < 3; ++c) kv[3 * r->block + c] = r->sign * known[s * n + 3 * i + c];
            }
            spmv(&p->K, kv, rhs);
            for (int64_t k = 1; s > 1 && k <= s; ++k) {
                if (k > p->n_hist_k) break;
                for (int type = 1; type >= 0; --type) {
                    const double* X = type ? XT : XU;
                    int64_t ids[3] = {s - k + 1, s - k, s - k - 1};
                    double cf[3] = {1.0, 2.0, 1.0};
                    memset(cv, 0, nh3 * sizeof(double));
                    for (int t = 0; t < 3; ++t)
                        if (ids[t] > 0 && ids[t] < s)
                            for (i = 0; i < nh3; ++i) cv[i] += cf[t] * X[ids[t] * nh3 + i];
                    spmv(type ? &p->mgs[k - 1] : &p->mts[k - 1], cv, tmp);
                    if (type)
                        for (i = 0; i < n; ++i) rhs[i] += 1.0 * tmp[i];
                    else
                        for (i = 0; i < n; ++i) rhs[i] += -1.0 * tmp[i];
                }
            }
            if (rhs_out) memcpy(rhs_out + (s - 1) * n, rhs, n * sizeof(double));
            int flag = 1, iter[2];
            gmres(p, rhs, x, &flag, iter);
            if (flags) {
                flags[3 * (s - 1)] = flag;
                flags[3 * (s - 1) + 1] = iter[0];
                flags[3 * (s - 1) + 2] = iter[1];
            }
            if (x_out) memcpy(x_out + (s - 1) * n, x, n * sizeof(double));
            solved++;
            if (flag != 0) break;
            /* scatter: unknowns (interface B side through the transform), knowns from input lu */
            for (i = 0; i < E; ++i) {
                double T[9], in[3] = {lu[3 * i], lu[3 * i + 1], lu[3 * i + 2]};
                interface_transform(p, i, T);
                const vref_t* ru = &p->uref[i];
                const vref_t* rt = &p->tref[i];
                if (!ru->known) {
                    const double* v = x + 3 * ru->block;
                    for (int r = 0; r < 3; ++r)
                        lu[3 * i + r] = ru->sign * (T[r * 3] * v[0] + T[r * 3 + 1] * v[1] + T[r * 3 + 2] * v[2]);
                }
                if (!rt->known) {
                    const double* v = x + 3 * rt->block;
                    for (int r = 0; r < 3; ++r)
                        lt[3 * i + r] = rt->sign * (T[r * 3] * v[0] + T[r * 3 + 1] * v[1] + T[r * 3 + 2] * v[2]);
                }
                if (ru->known)
                    for (int r = 0; r < 3; ++r) lu[3 * i + r] = ru->sign * in[r];
                if (rt->known)
                    for (int r = 0; r < 3; ++r) lt[3 * i + r] = rt->sign * in[r];
            }
        }
        /* local -> global: x_abs[c] = sum_r Trans[3r+c] x_loc[r] */
        for (i = 0; i < E; ++i) {
            const double* Tr = p->el[i].trans;
            double a[3], b[3];
            for (int c = 0; c < 3; ++c) {
                a[c] = Tr[c] * lu[3 * i] + Tr[3 + c] * lu[3 * i + 1] + Tr[6 + c] * lu[3 * i + 2];
                b[c] = Tr[c] * lt[3 * i] + Tr[3 + c] * lt[3 * i + 1] + Tr[6 + c] * lt[3 * i + 2];
            }
            memcpy(lu + 3 * i, a, sizeof a);
            memcpy(lt + 3 * i, b, sizeof b);
        }
        /* physical history state from the reference (A) side */
        double* xu = XU + s * nh3;
        double* xt = XT + s * nh3;
        for (i = 0; i < E; ++i) {
            int skip = 0;
            if (p->el[i].surface)
                for (int64_t k = 0; k < p->I; ++k)
                    if (p->itf[5 * k + 3] == i) { skip = 1; break; }
            if (skip) continue;
            for (int c = 0; c < 3; ++c) {
                xu[3 * p->hu[i].block + c] = p->hu[i].sign * lu[3 * i + c];
                xt[3 * p->ht[i].block + c] = p->ht[i].sign * lt[3 * i + c];
            }
        }
    }
    free(XU); free(XT); free(kv); free(rhs); free(tmp); free(cv); free(x);
    return solved;
}
