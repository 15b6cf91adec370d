// On-device element geometry, singular self-element integrals, Step0 and
// history block quadrature, block-CCSR compaction, history stacking and the
// mapped-leaf preconditioner inverses.
#include "assemble.cuh"
#include "quad.cuh"

namespace tdbem {

__constant__ DynaMat c_mats[kMaxDomains];

__constant__ DynaMatD c_dmats[kMaxDomains];

cudaError_t upload_materials(const DynaMat* mats, int n, cudaStream_t s)
{
    return cudaMemcpyToSymbolAsync(c_mats, mats, sizeof(DynaMat) * n, 0, cudaMemcpyHostToDevice, s);
}

cudaError_t upload_materials_dual(const DynaMatD* mats, int n, cudaStream_t s)
{
    return cudaMemcpyToSymbolAsync(c_dmats, mats, sizeof(DynaMatD) * n, 0, cudaMemcpyHostToDevice, s);
}

namespace {

__device__ __forceinline__ double ws(double v) { return qwarp_sum(v); }

__device__ void load_rules(const QuadRules* g, QuadRules* s)
{
    const double* src = reinterpret_cast<const double*>(g);
    double* dst = reinterpret_cast<double*>(s);
    for (int i = threadIdx.x; i < (int)(sizeof(QuadRules) / sizeof(double)); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}

__device__ __forceinline__ void load_elem(const ElemGeom& g, int f, QElem& e)
{
    e.cc = g.cc + 24 * (int64_t)f;
    e.rcen = g.rcen + 108 * (int64_t)f;
    e.center[0] = g.center[3 * f];
    e.center[1] = g.center[3 * f + 1];
    e.center[2] = g.center[3 * f + 2];
    e.radius = g.radius[f];
    e.rpw = g.rpw[f];
}

// Builder semantics of MultiDomainCCSRBuilder::AddBlock
// (DBEM1/multidomain.cpp:1120-1144): skip all-zero, near-zero (<= 1e-14)
// or non-finite blocks, store sign * block transposed.  Decided on the values.
template <class S>
__device__ __forceinline__ bool admit(const S* b9)
{
    bool zero = true, finite = true;
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const double b = qv(b9[i]);
        if (b != 0.0) zero = false;
        if (!(b == b) || fabs(b) > 1.7976931348623157e308) finite = false;
        m = fmax(m, fabs(b));
    }
    return !zero && finite && m > 1.0e-14;
}

template <class S>
__device__ __forceinline__ double maxabs9(const S* v)
{
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < 9; ++i) m = fmax(m, fabs(qv(v[i])));
    return m;
}

// out = convert(K): out[3j+i] = sign * sum_m K[3m+i] R[3j+m]
// (ConvertUnknownCoef / ConvertKnownCoef(long), DBEM1/dsquareelement.cpp:2756-2868, 3281-3394)
template <class S>
__device__ __forceinline__ void convert_block(const S* K, const double* R, double sign, S* out)
{
#pragma unroll
    for (int i = 0; i < 9; ++i) out[i] = 0.0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int m = 0; m < 3; ++m) {
                if (sign < 0)
                    out[3 * j + i] -= K[3 * m + i] * R[3 * j + m];
                else
                    out[3 * j + i] += K[3 * m + i] * R[3 * j + m];
            }
}

// Singular self-element blocks of one element: on_u1, on_t1, on_t2 (9 each).
template <class S>
struct SelfBlocks {
    const S* u1;
    const S* t1;
    const S* t2;
};

// Step0 coefficient block with the effective BCID (RegularInt*Coef /
// InElementInt*Coef with FlagDynaMethod 2); unknown = 1 for the kernel that
// multiplies the unknown.  Warp-uniform; result valid on every lane.
template <class MT, class S = typename MT::Scalar>
__device__ bool step0_block(const QuadRules& q, const MT& M, const QElem& e, const double* trans9, bool self,
                            const SelfBlocks<S>& sb, const double* src, int bcid, int unknown, S* out)
{
    const bool useU = unknown ? (bcid == 123) : (bcid == 456);
    S K[9], t[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) K[i] = 0.0;
    if (self) {
        if (useU) {
            for (int i = 0; i < 9; ++i) K[i] += 4.0 * sb.u1[i];
            w_int_u_pw(q, M, e, src, 1.0, t);
        } else {
            for (int i = 0; i < 9; ++i) {
                K[i] += 4.0 * sb.t1[i];
                K[i] += sb.t2[i];
            }
            w_int_t_pw(q, M, e, 1, src, 1.0, t);
        }
#pragma unroll
        for (int i = 0; i < 9; ++i) K[i] += t[i];
    } else {
        const int f0 = q_need_cal(M, e.center, e.radius, 1, 0.0, src);
        int fsum = f0;
        if (f0) {
            if (useU) {
                if (f0 == 1) w_int_u_pw(q, M, e, src, 0.0, t);
                else w_int_u_regular(q, M, e, src, 0.0, t);
#pragma unroll
                for (int i = 0; i < 9; ++i) K[i] += 4.0 * t[i];
            } else {
                if (f0 == 1) w_int_t_pw(q, M, e, 1, src, 0.0, t);
                else w_int_t_regular(q, M, e, src, 0.0, t);
#pragma unroll
                for (int i = 0; i < 9; ++i) K[i] += 4.0 * t[i];
                if (f0 == 1) w_int_t_pw(q, M, e, 2, src, 1.0, t);
                else w_int_t_regular(q, M, e, src, 1.0, t);
#pragma unroll
                for (int i = 0; i < 9; ++i) K[i] += t[i];
            }
        }
        const int f1 = q_need_cal(M, e.center, e.radius, 1, 1.0, src);
        fsum += f1;
        if (f1) {
            if (useU) {
                if (f1 == 1) w_int_u_pw(q, M, e, src, 1.0, t);
                else w_int_u_regular(q, M, e, src, 1.0, t);
            } else {
                if (f1 == 1) w_int_t_pw(q, M, e, 1, src, 1.0, t);
                else w_int_t_regular(q, M, e, src, 1.0, t);
            }
#pragma unroll
            for (int i = 0; i < 9; ++i) K[i] += t[i];
        }
        if (!fsum) return false;
    }
    const double sign = unknown ? (bcid == 123 ? -1.0 : 1.0) : (bcid == 456 ? 1.0 : -1.0);
    convert_block(K, trans9, sign, out);
    return true;
}

// The Step0 blocks of one (source s, field f) pair of a domain
// (AssembleMultiDomainStep0 with the interface field treatment of
// DBEM1/multidomain.cpp:2256-2327, 1594-1691): up to two A blocks (out0,
// out1) and one KnownM block (out1 for outer elements), transposed and
// signed; returns flags bit0 A0, bit1 A1, bit2 K.
template <class MT, class S = typename MT::Scalar>
__device__ uint8_t step0_pair(const QuadRules& q, const MT& M, const QElem& e, const ElemGeom& g, const DofRefs& dr,
                              int f, bool self, const SelfBlocks<S>& sb, const double* src, S* out0, S* out1)
{
    const double* tr = g.trans + 9 * (int64_t)f;
    S blk[9];
    uint8_t fl = 0;
    if (g.surface[f]) {
        const double* T = dr.itf_trans + 9 * (int64_t)f;
        for (int pass = 0; pass < 2; ++pass) {
            const int bc = pass == 0 ? 456 : 123;
            const double sign = pass == 0 ? dr.uref_sign[f] : dr.tref_sign[f];
            if (step0_block(q, M, e, tr, self, sb, src, bc, 1, blk)) {
                // TransformColumnBlock9 then AddBlock's transpose
                S tb[9];
                for (int r = 0; r < 3; ++r)
                    for (int qq = 0; qq < 3; ++qq) {
                        S v = 0.0;
                        for (int c = 0; c < 3; ++c) v += blk[c * 3 + r] * T[c * 3 + qq];
                        tb[qq * 3 + r] = v;
                    }
                if (sign != 0.0 && admit(tb)) {
                    S* o = pass == 0 ? out0 : out1;
                    for (int r = 0; r < 3; ++r)
                        for (int c = 0; c < 3; ++c) o[r * 3 + c] = 0.0 + sign * tb[c * 3 + r];
                    if (maxabs9(o) > 1.0e-14) fl |= (uint8_t)(pass == 0 ? 1 : 2);
                }
            }
        }
    } else {
        const int bc = g.bcid[f];
        if (step0_block(q, M, e, tr, self, sb, src, bc, 1, blk)) {
            const double sign = bc == 123 ? dr.tref_sign[f] : dr.uref_sign[f];
            if (sign != 0.0 && admit(blk)) {
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) out0[r * 3 + c] = 0.0 + sign * blk[c * 3 + r];
                if (maxabs9(out0) > 1.0e-14) fl |= 1;
            }
        }
        if (step0_block(q, M, e, tr, self, sb, src, bc, 0, blk)) {
            const double sign = bc == 123 ? dr.uref_sign[f] : dr.tref_sign[f];
            if (sign != 0.0 && admit(blk)) {
                for (int r = 0; r < 3; ++r)
                    for (int c = 0; c < 3; ++c) out1[r * 3 + c] = 0.0 + sign * blk[c * 3 + r];
                if (maxabs9(out1) > 1.0e-14) fl |= 4;
            }
        }
    }
    return fl;
}

// History step k blocks of one pair (AssembleMultiDomainHistoryStep,
// DBEM1/multidomain.cpp:2329-2378, ComputeT2Block / T1Block / UBlock
// :1739-1813): acc = MTS (T2 then T1 accumulated), mgs = MGS (U), both
// transposed and signed; returns flags bit0 MTS, bit1 MGS.  self_t2 is the
// field element's singular T2 block (used at k <= 1 when s == f).
template <class MT, class S = typename MT::Scalar>
__device__ uint8_t history_pair(const QuadRules& q, const MT& M, const QElem& e, const DofRefs& dr, int f, bool self,
                                const S* self_t2, const double* src, int k, S* acc, S* mgs)
{
    const double n = (double)k;
    const bool self_k = (k <= 1 && self);
    const int c2 = self_k ? 3 : q_need_cal(M, e.center, e.radius, 2, n, src);
    const int c1 = q_need_cal(M, e.center, e.radius, 1, n, src);
    uint8_t fl = 0;
    S blk[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) acc[i] = 0.0;
    bool present = false;
    const double su = dr.hu_sign[f], st = dr.ht_sign[f];
    if (c2 || c1) {
        // T2 block
        if (self_k) {
            for (int i = 0; i < 9; ++i) blk[i] = self_t2[i];
        } else if (c2 == 1) {
            w_int_t_pw(q, M, e, 2, src, n, blk);
        } else if (c2 == 2) {
            w_int_t_regular(q, M, e, src, n, blk);
        }
        if (c2 && su != 0.0 && admit(blk)) {
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) acc[r * 3 + c] += su * blk[c * 3 + r];
            present = true;
            if (maxabs9(acc) <= 1.0e-14) {
                present = false;
                for (int i = 0; i < 9; ++i) acc[i] = 0.0;
            }
        }
        // T1 block
        if (c1 == 1) w_int_t_pw(q, M, e, 1, src, n, blk);
        else if (c1 == 2) w_int_t_regular(q, M, e, src, n, blk);
        if (c1 && su != 0.0 && admit(blk)) {
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) acc[r * 3 + c] += su * blk[c * 3 + r];
            present = true;
            if (maxabs9(acc) <= 1.0e-14) {
                present = false;
                for (int i = 0; i < 9; ++i) acc[i] = 0.0;
            }
        }
        if (present) fl |= 1;
    }
    if (c1) {
        if (c1 == 1) w_int_u_pw(q, M, e, src, n, blk);
        else w_int_u_regular(q, M, e, src, n, blk);
        if (st != 0.0 && admit(blk)) {
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) mgs[r * 3 + c] = 0.0 + st * blk[c * 3 + r];
            if (maxabs9(mgs) > 1.0e-14) fl |= 2;
        }
    }
    return fl;
}

__device__ __forceinline__ void decode_pair(const PairSpace& ps, int64_t p, int& d, int& s, int& f)
{
    d = 0;
    while (d + 1 < ps.n_domains && p >= ps.pair_off[d + 1]) ++d;
    const int64_t loc = p - ps.pair_off[d];
    const int nd = ps.dom_count[d];
    s = ps.dom_begin[d] + (int)(loc / nd);
    f = ps.dom_begin[d] + (int)(loc - (loc / nd) * nd);
}

}  // namespace

// ---------------------------------------------------------------------------
// Element geometry (GeoInit, DBEM1/dsquareelement.cpp:332-382; node at the
// centre, GetNodeInfo, DBEM1/DBEM.cpp:1409-1427; local frame at node 0,
// TranslateMatrix, DBEM1/dsquareelement.h:488-507).  One thread per element.
__global__ void geometry_kernel(int E, const double* points, const int64_t* elements, const QuadRules* rules,
                                ElemGeom g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= E) return;
    double* cc = g.cc + 24 * (int64_t)i;
    double pts[8][3];
    for (int k = 0; k < 8; ++k)
        for (int c = 0; c < 3; ++c) pts[k][c] = points[3 * elements[8 * (int64_t)i + k] + c];
    for (int c = 0; c < 3; ++c) {
        const double v[8] = {pts[0][c], pts[1][c], pts[2][c], pts[3][c], pts[4][c], pts[5][c], pts[6][c], pts[7][c]};
        double* k = cc + 8 * c;
        // GetCoef, DBEM1/dsquareelement.h:582-611
        k[0] = 0.25 * (-v[0] - v[3] + 2 * v[5] - v[2] - v[1] + 2 * v[4] + 2 * v[7] + 2 * v[6]);
        k[1] = 0.5 * (v[5] - v[7]);
        k[2] = 0.5 * (-v[4] + v[6]);
        k[3] = 0.25 * (v[0] - v[1] + v[2] - v[3]);
        k[4] = 0.25 * (-2 * v[4] + v[3] + v[2] - 2 * v[6] + v[1] + v[0]);
        k[5] = 0.25 * (-2 * v[5] + v[1] - 2 * v[7] + v[2] + v[0] + v[3]);
        k[6] = 0.25 * (2 * v[4] + v[3] + v[2] - 2 * v[6] - v[1] - v[0]);
        k[7] = 0.25 * (2 * v[7] - 2 * v[5] + v[1] - v[3] + v[2] - v[0]);
    }
    for (int p = 0; p < kNumPW2; ++p) q_from_local(cc, rules->cenpw[p][0], rules->cenpw[p][1], g.rcen + 108 * (int64_t)i + 3 * p);
    double ctr[3];
    q_from_local(cc, 0.0, 0.0, ctr);
    double rad = -1.0;
    for (int k = 0; k < 8; ++k) {
        const double dd = q_dist(ctr, pts[k]);
        if (rad < dd) rad = dd;
    }
    for (int c = 0; c < 3; ++c) {
        g.center[3 * i + c] = ctr[c];
        g.node[3 * i + c] = ctr[c];
    }
    g.radius[i] = rad;
    g.rpw[i] = rad / kNumPW;
    double T[9], r[3], l;
    const double s1 = rules->lc0[0], s2 = rules->lc0[1];
    q_rdiff1(cc, s1, s2, r);
    l = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    T[0] = r[0] / l; T[1] = r[1] / l; T[2] = r[2] / l;
    q_rdiff2(cc, s1, s2, r);
    l = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    T[3] = r[0] / l; T[4] = r[1] / l; T[5] = r[2] / l;
    T[6] = T[1] * T[5] - T[4] * T[2];
    T[7] = T[3] * T[2] - T[0] * T[5];
    T[8] = T[0] * T[4] - T[3] * T[1];
    const double t = sqrt(T[6] * T[6] + T[7] * T[7] + T[8] * T[8]);
    T[6] /= t; T[7] /= t; T[8] /= t;
    T[3] = T[7] * T[2] - T[8] * T[1];
    T[4] = T[8] * T[0] - T[6] * T[2];
    T[5] = T[6] * T[1] - T[7] * T[0];
    for (int k = 0; k < 9; ++k) g.trans[9 * (int64_t)i + k] = T[k];
}

// ---------------------------------------------------------------------------
// Singular self-element integrals, one CTA per element: the static strongly
// singular part (InElementStaticTij(), DBEM1/dsquareelement.cpp:2292-2427)
// and the dynamic polar sub-patch sums (PthInElementIntDynamic,
// DBEM1/dsquareelementdyna.cpp:239-490).
__global__ void __launch_bounds__(256) singular_kernel(int E, const QuadRules* rules, const double* secpw_pos,
                                                       const double* secpw_val, ElemGeom g)
{
    const int i = blockIdx.x;
    if (i >= E) return;
    __shared__ double red[24][8];
    __shared__ double stat[9];
    const DynaMat& M = c_mats[g.domain[i]];
    const double* cc = g.cc + 24 * (int64_t)i;
    const double src[3] = {g.node[3 * i], g.node[3 * i + 1], g.node[3 * i + 2]};
    double acc[24];
#pragma unroll
    for (int k = 0; k < 24; ++k) acc[k] = 0.0;
    const int n_items = 4 * kSinNumPW2 * 9;
    for (int it = threadIdx.x; it < n_items; it += blockDim.x) {
        const int a = it / (kSinNumPW2 * 9), rem = it - a * (kSinNumPW2 * 9);
        const double s1 = secpw_pos[(a * 2 + 0) * kSinNumPW2 * 9 + rem];
        const double s2 = secpw_pos[(a * 2 + 1) * kSinNumPW2 * 9 + rem];
        const double w = secpw_val[a * kSinNumPW2 * 9 + rem];
        double pt[3], nor[3], jac, U[9], D1[9], D2[9], ST[9];
        QR r;
        q_from_local(cc, s1, s2, pt);
        q_get_r(src, pt, r);
        q_normal_jacobi(cc, s1, s2, nor, &jac);
        q_dyna_u(M, U, 0.0, r);
        q_dyna_t(M, 1, D1, 0.0, r, nor);
        q_dyna_t(M, 2, D2, 1.0, r, nor);
        const double SR[4] = {r.R[1], r.RI[1], r.RI[2], r.RI[3]};
        q_static_t(M, ST, SR, nor);
        const double t = w * jac;
        acc[0] += U[0] * t; acc[1] += U[1] * t; acc[2] += U[2] * t;
        acc[3] += U[4] * t; acc[4] += U[5] * t; acc[5] += U[8] * t;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            acc[6 + k] += (D1[k] - ST[k]) * t;
            acc[15 + k] += (D2[k] - ST[k]) * t;
        }
    }
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 24; ++k) {
        const double v = ws(acc[k]);
        if (lane == 0) red[k][wp] = v;
    }
    // static strongly singular part by warp 0
    if (wp == 0) {
        const QuadRules& q = *rules;
        double st[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) st[k] = 0.0;
        const double coef1 = -1.0 / (8.0 * kPi * (1.0 - M.v));
        const double coef2 = 1.0 - 2.0 * M.v;
        for (int it = lane; it < 64; it += 32) {
            const int a = it / 16, j = it % 16;
            const double s1 = q.sec_pos[a][0][j], s2 = q.sec_pos[a][1][j];
            double pt[3], nor[3], jac, T[9];
            q_from_local(cc, s1, s2, pt);
            q_normal_jacobi(cc, s1, s2, nor, &jac);
            double R[4];
            R[1] = pt[0] - src[0];
            R[2] = pt[1] - src[1];
            R[3] = pt[2] - src[2];
            R[0] = sqrt(R[1] * R[1] + R[2] * R[2] + R[3] * R[3]);
            q_static_t(M, T, R, nor);
            const double t = q.sec_val[a][j] * jac;
#pragma unroll
            for (int k = 0; k < 9; ++k) st[k] += T[k] * t;
        }
        if (lane < 16) {
            const int a = lane / 4, j = lane % 4;
            double Jh[3], d1[3], d2[3], n0[3], tJ;
            q_normal_jacobi(cc, q.lc0[0], q.lc0[1], n0, &tJ);
            Jh[0] = tJ * n0[0]; Jh[1] = tJ * n0[1]; Jh[2] = tJ * n0[2];
            q_rdiff1(cc, 0.0, 0.0, d1);
            q_rdiff2(cc, 0.0, 0.0, d2);
            const double th = q.line_pos[a][j];
            double A[6];
            A[1] = d1[0] * cos(th) + d2[0] * sin(th);
            A[2] = d1[1] * cos(th) + d2[1] * sin(th);
            A[3] = d1[2] * cos(th) + d2[2] * sin(th);
            A[0] = sqrt(A[1] * A[1] + A[2] * A[2] + A[3] * A[3]);
            A[4] = A[0] * A[0] * A[0];
            A[5] = A[4] * A[0] * A[0];
            // GetFijMinusOne, DBEM1/dsquareelement.cpp:609-640
            const double AkJk0 = A[1] * Jh[0] + A[2] * Jh[1] + A[3] * Jh[2];
            double t1 = 3.0 * A[1] * AkJk0 / A[5];
            const double t2 = coef2 * (A[2] * Jh[0] - A[1] * Jh[1]) / A[4];
            const double t3 = coef2 * (A[3] * Jh[0] - A[1] * Jh[2]) / A[4];
            const double t4 = coef2 * (A[3] * Jh[1] - A[2] * Jh[2]) / A[4];
            const double temp = coef2 * AkJk0 / A[4];
            double F[9];
            F[0] = coef1 * (temp + t1 * A[1]);
            F[1] = coef1 * (t1 * A[2] - t2);
            F[2] = coef1 * (t1 * A[3] - t3);
            F[3] = coef1 * (t1 * A[2] + t2);
            F[4] = coef1 * (temp + 3.0 * A[2] * A[2] * AkJk0 / A[5]);
            t1 = 3.0 * A[3] * AkJk0 / A[5];
            F[5] = coef1 * (t1 * A[2] - t4);
            F[6] = coef1 * (t1 * A[1] + t3);
            F[7] = coef1 * (t1 * A[2] + t4);
            F[8] = coef1 * (temp + t1 * A[3]);
            double fvs = 0.0;
            for (int l = 0; l < 4; ++l) fvs += q.fm1_sec[a][l * 4 + j];
            const double fvl = q.fm1_line[a][j];
#pragma unroll
            for (int k = 0; k < 9; ++k) st[k] += F[k] * (fvl - fvs);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const double v = ws(st[k]);
            if (lane == 0) stat[k] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < 24) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
        const int k = threadIdx.x;
        if (k < 6) {
            const int map[6] = {0, 1, 2, 4, 5, 8};
            g.on_u1[9 * (int64_t)i + map[k]] = s;
            if (k == 1) g.on_u1[9 * (int64_t)i + 3] = s;
            if (k == 2) g.on_u1[9 * (int64_t)i + 6] = s;
            if (k == 4) g.on_u1[9 * (int64_t)i + 7] = s;
        } else if (k < 15) {
            const int c = k - 6;
            g.on_t1[9 * (int64_t)i + c] = s + stat[c] + ((c == 0 || c == 4 || c == 8) ? 0.5 : 0.0);
        } else {
            const int c = k - 15;
            g.on_t2[9 * (int64_t)i + c] = s + stat[c];
        }
    }
}

// ---------------------------------------------------------------------------
// Step0 blocks, one warp per (source row, field element) pair of a domain:
// up to two A blocks (slot 0, 1) and one KnownM block (slot 1 for outer
// elements), already transposed and signed; flags bit0 A0, bit1 A1, bit2 K.
__global__ void __launch_bounds__(128) step0_kernel(PairSpace ps, const QuadRules* rules, ElemGeom g, DofRefs dr,
                                                    double* blocks, uint8_t* flags)
{
    __shared__ QuadRules q;
    load_rules(rules, &q);
    const int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (p >= ps.n_pairs) return;
    const int lane = threadIdx.x & 31;
    int d, s, f;
    decode_pair(ps, p, d, s, f);
    const DynaMat& M = c_mats[d];
    QElem e;
    load_elem(g, f, e);
    const double src[3] = {g.node[3 * s], g.node[3 * s + 1], g.node[3 * s + 2]};
    const SelfBlocks<double> sb{g.on_u1 + 9 * (int64_t)f, g.on_t1 + 9 * (int64_t)f, g.on_t2 + 9 * (int64_t)f};
    double out0[9], out1[9];
    const uint8_t fl = step0_pair(q, M, e, g, dr, f, s == f, sb, src, out0, out1);
    if (lane < 9) {
        blocks[(p * 2 + 0) * 9 + lane] = (fl & 1) ? out0[lane] : 0.0;
        blocks[(p * 2 + 1) * 9 + lane] = (fl & 6) ? out1[lane] : 0.0;
    }
    if (lane == 0) flags[p] = fl;
}

// History step k blocks, one warp per pair: slot 0 = MTS, slot 1 = MGS.
__global__ void __launch_bounds__(128) history_kernel(PairSpace ps, const QuadRules* rules, ElemGeom g, DofRefs dr,
                                                      int k, double* blocks, uint8_t* flags)
{
    __shared__ QuadRules q;
    load_rules(rules, &q);
    const int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (p >= ps.n_pairs) return;
    const int lane = threadIdx.x & 31;
    int d, s, f;
    decode_pair(ps, p, d, s, f);
    const DynaMat& M = c_mats[d];
    QElem e;
    load_elem(g, f, e);
    const double src[3] = {g.node[3 * s], g.node[3 * s + 1], g.node[3 * s + 2]};
    double acc[9], mgs[9];
    const uint8_t fl = history_pair(q, M, e, dr, f, s == f, g.on_t2 + 9 * (int64_t)f, src, k, acc, mgs);
    if (lane < 9) {
        blocks[(p * 2 + 0) * 9 + lane] = (fl & 1) ? acc[lane] : 0.0;
        blocks[(p * 2 + 1) * 9 + lane] = (fl & 2) ? mgs[lane] : 0.0;
    }
    if (lane == 0) flags[p] = fl;
}

// Count the blocks each row receives from a pair buffer: mask selects the
// flag bits counted.
__global__ void count_rows_kernel(PairSpace ps, const uint8_t* flags, int mask, int E, int* counts)
{
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= E) return;
    int d = 0;
    while (d + 1 < ps.n_domains && row >= ps.dom_begin[d + 1]) ++d;
    const int nd = ps.dom_count[d];
    const int64_t base = ps.pair_off[d] + (int64_t)(row - ps.dom_begin[d]) * nd;
    int c = 0;
    for (int j = lane; j < nd; j += 32) c += __popc(flags[base + j] & mask);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) counts[row] = c;
}

// Scatter a pair buffer into compacted per-row storage (field order within a
// row).  For each set bit b of (flag & mask), block slot slot_of_bit[b] goes
// to column col_of_bit[b][field] with values from blocks[pair][slot].
__global__ void scatter_rows_kernel(PairSpace ps, const uint8_t* flags, const double* blocks, int mask, int E,
                                    const int64_t* row_start, ScatterCols sc, int32_t* out_col, double* out_val)
{
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= E) return;
    int d = 0;
    while (d + 1 < ps.n_domains && row >= ps.dom_begin[d + 1]) ++d;
    const int nd = ps.dom_count[d];
    const int64_t base = ps.pair_off[d] + (int64_t)(row - ps.dom_begin[d]) * nd;
    int64_t pos = row_start[row];
    for (int j0 = 0; j0 < nd; j0 += 32) {
        const int j = j0 + lane;
        const uint8_t fl = j < nd ? (uint8_t)(flags[base + j] & mask) : (uint8_t)0;
        const int mine = __popc(fl);
        int incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        int64_t at = pos + incl - mine;
        if (fl) {
            const int f = ps.dom_begin[d] + j;
            for (int b = 0; b < 3; ++b) {
                if (!(fl & (1 << b))) continue;
                const int slot = sc.slot_of_bit[b];
                out_col[at] = (int32_t)sc.col_of_bit[b][f];
                const double* src = blocks + ((base + j) * 2 + slot) * 9;
                for (int c = 0; c < 9; ++c) out_val[at * 9 + c] = src[c];
                ++at;
            }
        }
        pos += total;
    }
}

// Stack the per-k history matrices into one row-major structure:
// row r = [k=1: MGS_1 (type 1), MTS_1 negated (type 0)] [k=2: ...] ...
// each part in ascending column order, with values as 9 planes (structure
// of arrays) and packed columns.
__global__ void stack_history_kernel(int E, int K, const HistK* hk, const int64_t* kptr, uint32_t* col, double* val,
                                     int64_t nnz)
{
    const int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= (int64_t)E * K) return;
    const int row = (int)(t / K), k = (int)(t % K) + 1;
    int64_t pos = kptr[(int64_t)row * (K + 1) + (k - 1)];
    const HistK& h = hk[k - 1];
    for (int type = 1; type >= 0; --type) {
        const int64_t* rp = type ? h.mgs_rp : h.mts_rp;
        const int32_t* cc = type ? h.mgs_col : h.mts_col;
        const double* vv = type ? h.mgs_val : h.mts_val;
        const int64_t b = rp[row], e = rp[row + 1];
        const double sg = type ? 1.0 : -1.0;
        for (int64_t j = b + lane; j < e; j += 32) {
            // ascending columns within the segment (the assembled rows come in
            // pair order; columns of one row are distinct)
            const int cj = cc[j];
            int64_t rank = 0;
            for (int64_t q = b; q < e; ++q) rank += cc[q] < cj;
            const int64_t o = pos + rank;
            col[o] = ((uint32_t)k << 21) | ((uint32_t)type << 20) | (uint32_t)cj;
            for (int c = 0; c < 9; ++c) val[c * nnz + o] = sg * vv[j * 9 + c];
        }
        pos += e - b;
    }
}

__global__ void to_float_kernel(const double* in, float* out, int64_t n)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// ---------------------------------------------------------------------------
// Mapped-leaf preconditioner: gather each leaf's dense (3L x 3L) block of A'
// and invert it by full-pivot Gauss-Jordan (inv_mat, DBEM1/lin_comp.cpp:83-183,
// pivot = first largest |a| in row-major scan, singular if <= 1e-10).
// One CTA per leaf; the matrix lives in shared memory.
__global__ void __launch_bounds__(256) leaf_inverse_kernel(int n_leaves, const int32_t* leaf_begin,
                                                           const int32_t* leaf_count, const int64_t* leaf_off,
                                                           const int32_t* a_rp, const int32_t* a_col,
                                                           const double* a_val, double* pinv, int* singular)
{
    extern __shared__ double sa[];
    __shared__ int piv_i[1], piv_j[1];
    __shared__ double wv[32];
    __shared__ int wi[32];
    const int L = blockIdx.x;
    if (L >= n_leaves) return;
    const int b = leaf_begin[L], cnt = leaf_count[L], n = 3 * cnt;
    int* is = reinterpret_cast<int*>(sa + (int64_t)n * n);
    int* js = is + n + 1;
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) sa[t] = 0.0;
    __syncthreads();
    for (int r = threadIdx.x; r < cnt; r += blockDim.x) {
        const int p = b + r;
        for (int j = a_rp[p]; j < a_rp[p + 1]; ++j) {
            const int c = a_col[j] - b;
            if (c < 0 || c >= cnt) continue;
            for (int x = 0; x < 3; ++x)
                for (int y = 0; y < 3; ++y) sa[(3 * r + x) * n + 3 * c + y] = a_val[9 * (int64_t)j + 3 * x + y];
        }
    }
    __syncthreads();
#define AA(i, j) sa[((i)-1) * n + ((j)-1)]
    bool bad = false;
    for (int k = 1; k <= n; ++k) {
        // first maximum in row-major order over i, j >= k
        double best = 0.0;
        int bidx = 0x7fffffff;
        const int m = n - k + 1;
        for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
            const int i = k + t / m, j = k + t % m;
            const double v = sqrt(AA(i, j) * AA(i, j));
            const int idx = (i - 1) * n + (j - 1);
            if (v > best || (v == best && v > 0.0 && idx < bidx)) {
                best = v;
                bidx = idx;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
            if (ov > best || (ov == best && oi < bidx)) {
                best = ov;
                bidx = oi;
            }
        }
        if ((threadIdx.x & 31) == 0) {
            wv[threadIdx.x >> 5] = best;
            wi[threadIdx.x >> 5] = bidx;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double bb = 0.0;
            int bi = 0x7fffffff;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
                if (wv[w] > bb || (wv[w] == bb && wi[w] < bi)) {
                    bb = wv[w];
                    bi = wi[w];
                }
            if (bb <= 0.0000000001) {
                piv_i[0] = -1;
            } else {
                piv_i[0] = bi / n + 1;
                piv_j[0] = bi % n + 1;
            }
            is[k] = piv_i[0];
            js[k] = piv_j[0];
        }
        __syncthreads();
        if (piv_i[0] < 0) {
            bad = true;
            break;
        }
        const int pi = piv_i[0], pj = piv_j[0];
        for (int j = 1 + threadIdx.x; j <= n; j += blockDim.x) {
            const double tmp = AA(k, j);
            AA(k, j) = AA(pi, j);
            AA(pi, j) = tmp;
        }
        __syncthreads();
        for (int i = 1 + threadIdx.x; i <= n; i += blockDim.x) {
            const double tmp = AA(i, k);
            AA(i, k) = AA(i, pj);
            AA(i, pj) = tmp;
        }
        __syncthreads();
        if (threadIdx.x == 0) AA(k, k) = 1.0 / AA(k, k);
        __syncthreads();
        const double akk = AA(k, k);
        for (int j = 1 + threadIdx.x; j <= n; j += blockDim.x)
            if (j != k) AA(k, j) *= akk;
        __syncthreads();
        for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
            const int i = t / n + 1, j = t % n + 1;
            if (i != k && j != k) AA(i, j) -= AA(i, k) * AA(k, j);
        }
        __syncthreads();
        for (int i = 1 + threadIdx.x; i <= n; i += blockDim.x)
            if (i != k) AA(i, k) *= -1.0 * akk;
        __syncthreads();
    }
    if (bad) {
        if (threadIdx.x == 0) atomicExch(singular, L + 1);
    } else {
        for (int k = n; k >= 1; --k) {
            const int ik = js[k], jk = is[k];
            for (int j = 1 + threadIdx.x; j <= n; j += blockDim.x) {
                const double tmp = AA(k, j);
                AA(k, j) = AA(ik, j);
                AA(ik, j) = tmp;
            }
            __syncthreads();
            for (int i = 1 + threadIdx.x; i <= n; i += blockDim.x) {
                const double tmp = AA(i, k);
                AA(i, k) = AA(i, jk);
                AA(i, jk) = tmp;
            }
            __syncthreads();
        }
    }
#undef AA
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) pinv[leaf_off[L] + t] = sa[t];
}

// ---------------------------------------------------------------------------
// Material gradient: dJ/dE_d and dJ/drho_d of J = <cot, march outputs> by the
// adjoint identity dJ/dtheta = sum_n lam_n^T (db_n/dtheta - dA/dtheta x_n),
// with the derivative blocks recomputed by the quadrature in QDual form
// (never stored) and contracted at once with the adjoint vectors and the
// saved forward states.  Every block belongs to one domain, so a pair adds
// to its own domain only.  Per pair the kernels return (gE, gU): gE the
// contraction of the E-derivative blocks, gU that of the values of the
// displacement-kernel blocks; then dJ/dE = sum gE and
// dJ/drho = -(E/rho) sum gE - sum gU / rho.

// E-derivatives of the singular self-element blocks on_u1, on_t1, on_t2: the
// dynamic polar sub-patch sums of singular_kernel in QDual form (the static
// strongly singular part depends on the Poisson ratio only).  Values are
// copied from the FP64 blocks.  One CTA per element.
__global__ void __launch_bounds__(256) singular_grad_kernel(int E, const double* secpw_pos, const double* secpw_val,
                                                            ElemGeom g, QDual* self_d)
{
    const int i = blockIdx.x;
    if (i >= E) return;
    __shared__ double red[27][8];
    const DynaMatD& M = c_dmats[g.domain[i]];
    const double* cc = g.cc + 24 * (int64_t)i;
    const double src[3] = {g.node[3 * i], g.node[3 * i + 1], g.node[3 * i + 2]};
    double ae[27];
#pragma unroll
    for (int k = 0; k < 27; ++k) ae[k] = 0.0;
    const int n_items = 4 * kSinNumPW2 * 9;
    for (int it = threadIdx.x; it < n_items; it += blockDim.x) {
        const int a = it / (kSinNumPW2 * 9), rem = it - a * (kSinNumPW2 * 9);
        const double s1 = secpw_pos[(a * 2 + 0) * kSinNumPW2 * 9 + rem];
        const double s2 = secpw_pos[(a * 2 + 1) * kSinNumPW2 * 9 + rem];
        const double w = secpw_val[a * kSinNumPW2 * 9 + rem];
        double pt[3], nor[3], jac;
        QR r;
        q_from_local(cc, s1, s2, pt);
        q_get_r(src, pt, r);
        q_normal_jacobi(cc, s1, s2, nor, &jac);
        const double t = w * jac;
        QDual K[9];
        q_dyna_u(M, K, 0.0, r);
#pragma unroll
        for (int k = 0; k < 9; ++k) ae[k] += K[k].e * t;
        q_dyna_t(M, 1, K, 0.0, r, nor);
#pragma unroll
        for (int k = 0; k < 9; ++k) ae[9 + k] += K[k].e * t;
        q_dyna_t(M, 2, K, 1.0, r, nor);
#pragma unroll
        for (int k = 0; k < 9; ++k) ae[18 + k] += K[k].e * t;
    }
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 27; ++k) {
        const double ve = ws(ae[k]);
        if (lane == 0) red[k][wp] = ve;
    }
    __syncthreads();
    if (threadIdx.x < 27) {
        const int k = threadIdx.x;
        double se = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) se += red[k][w];
        const double* val = k < 9 ? g.on_u1 : (k < 18 ? g.on_t1 : g.on_t2);
        self_d[27 * (int64_t)i + k] = QDual(val[9 * (int64_t)i + k % 9], se);
    }
}

// History states X_m of the saved march, as the write-back stores them in the
// state ring: X_m[0][hb] = hu_sign * lu_m, X_m[1][hb] = ht_sign * lt_m
// (global frame) of the owner element of history block hb, m = 1..N.
__global__ void history_states_kernel(int N, int E, int nh, const int32_t* hist_owner, const int64_t* hist_block,
                                      const double* hu_sign, const double* ht_sign, const double* out_lu,
                                      const double* out_lt, double* xh)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < (int64_t)N * E;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = 1 + t / E, i = t % E;
        if (!hist_owner[i]) continue;
        const int64_t hb = hist_block[i];
        const double* lu = out_lu + (m * E + i) * 3;
        const double* lt = out_lt + (m * E + i) * 3;
        double* xu = xh + ((m * 2 + 0) * nh + hb) * 3;
        double* xt = xh + ((m * 2 + 1) * nh + hb) * 3;
        for (int c = 0; c < 3; ++c) {
            xu[c] = hu_sign[i] * lu[c];
            xt[c] = ht_sign[i] * lt[c];
        }
    }
}

namespace {

// ge += sg * l^T dB/dE v; gu += sg * l^T B v when B is a displacement-kernel
// block (B row-major 3x3)
__device__ __forceinline__ void contract_add(const QDual* B, const double* l, const double* v, double sg, bool ublock,
                                             double& ge, double& gu)
{
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double li = sg * l[i];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            ge += li * B[3 * i + j].e * v[j];
            if (ublock) gu += li * B[3 * i + j].v * v[j];
        }
    }
}

}  // namespace

// Step0 part, one warp per pair: A blocks add -lam_n^T dA x_n, the KnownM
// block adds lam_n^T dK k_n, n = 1..N (lanes take the steps).  Displacement-
// kernel blocks: an interface element's T column (slot 1), an outer
// element's unknown column when its BCID is 123 and its known column when
// it is 456.  part[2p], part[2p+1] = the pair's gE and gU.
__global__ void __launch_bounds__(128) grad_step0_kernel(PairSpace ps, const QuadRules* rules, ElemGeom g, DofRefs dr,
                                                         const QDual* self_d, GradState gs, double* part)
{
    __shared__ QuadRules q;
    load_rules(rules, &q);
    const int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (p >= ps.n_pairs) return;
    const int lane = threadIdx.x & 31;
    int d, s, f;
    decode_pair(ps, p, d, s, f);
    const DynaMatD& M = c_dmats[d];
    QElem e;
    load_elem(g, f, e);
    const double src[3] = {g.node[3 * s], g.node[3 * s + 1], g.node[3 * s + 2]};
    const QDual* sd = self_d + 27 * (int64_t)f;
    const SelfBlocks<QDual> sb{sd, sd + 9, sd + 18};
    QDual out0[9], out1[9];
    const uint8_t fl = step0_pair(q, M, e, g, dr, f, s == f, sb, src, out0, out1);
    const bool surf = g.surface[f] != 0;
    const bool u0 = !surf && g.bcid[f] == 123, uk = !surf && g.bcid[f] == 456;
    double ge = 0.0, gu = 0.0;
    if (fl) {
        const int64_t E3 = 3 * (int64_t)gs.E;
        for (int n = 1 + lane; n <= gs.N; n += 32) {
            const double* l = gs.lam + n * E3 + 3 * (int64_t)s;
            const double* xn = gs.x + (int64_t)(n - 1) * E3;
            if (fl & 1) contract_add(out0, l, xn + 3 * gs.col_a0[f], -1.0, u0, ge, gu);
            if (fl & 2) contract_add(out1, l, xn + 3 * gs.col_a1[f], -1.0, true, ge, gu);
            if (fl & 4) {
                const int64_t kb = gs.col_k[f];
                const double* kv = gs.known + ((int64_t)n * gs.E + gs.known_elem[kb]) * 3;
                contract_add(out1, l, kv, gs.known_sign[kb], uk, ge, gu);
            }
        }
    }
    ge = qwarp_sum(ge);
    gu = qwarp_sum(gu);
    if (lane == 0) {
        part[2 * p] = ge;
        part[2 * p + 1] = gu;
    }
}

// History part, one warp per pair over k = 1..K: the stacked -MTS_k
// (traction kernel) and MGS_k (displacement kernel) blocks add
// lam_n^T (-dMTS_k W0 + dMGS_k W1) with the convolution vector the march
// used at step n >= 2, W_m = [m+1 < n] X_{m+1} + 2 X_m + X_{m-1},
// m = n - k (X_0 = X_-1 = 0).
__global__ void __launch_bounds__(128) grad_history_kernel(PairSpace ps, const QuadRules* rules, ElemGeom g,
                                                           DofRefs dr, const QDual* self_d, GradState gs,
                                                           double* part)
{
    __shared__ QuadRules q;
    load_rules(rules, &q);
    const int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (p >= ps.n_pairs) return;
    const int lane = threadIdx.x & 31;
    int d, s, f;
    decode_pair(ps, p, d, s, f);
    const DynaMatD& M = c_dmats[d];
    QElem e;
    load_elem(g, f, e);
    const double src[3] = {g.node[3 * s], g.node[3 * s + 1], g.node[3 * s + 2]};
    const QDual* self_t2 = self_d + 27 * (int64_t)f + 18;
    const int64_t hb = gs.col_h[f];
    const int64_t E3 = 3 * (int64_t)gs.E, X3 = 3 * (int64_t)gs.nh;
    double ge = 0.0, gu = 0.0;
    for (int k = 1; k <= gs.K; ++k) {
        QDual acc[9], mgs[9];
        const uint8_t fl = history_pair(q, M, e, dr, f, s == f, self_t2, src, k, acc, mgs);
        if (!fl) continue;
        for (int n = (k > 2 ? k : 2) + lane; n <= gs.N; n += 32) {
            const int m = n - k;
            const double* l = gs.lam + n * E3 + 3 * (int64_t)s;
            for (int type = 0; type < 2; ++type) {
                if (!(fl & (1 << type))) continue;
                const double* xm = gs.xh + ((int64_t)m * 2 + type) * X3 + 3 * hb;
                double w[3] = {2.0 * xm[0], 2.0 * xm[1], 2.0 * xm[2]};
                if (m + 1 < n) {
                    const double* xp = gs.xh + ((int64_t)(m + 1) * 2 + type) * X3 + 3 * hb;
                    for (int c = 0; c < 3; ++c) w[c] += xp[c];
                }
                if (m >= 1) {
                    const double* xq = gs.xh + ((int64_t)(m - 1) * 2 + type) * X3 + 3 * hb;
                    for (int c = 0; c < 3; ++c) w[c] += xq[c];
                }
                contract_add(type ? mgs : acc, l, w, type ? 1.0 : -1.0, type == 1, ge, gu);
            }
        }
    }
    ge = qwarp_sum(ge);
    gu = qwarp_sum(gu);
    if (lane == 0) {
        part[2 * p] = ge;
        part[2 * p + 1] = gu;
    }
}

}  // namespace tdbem
