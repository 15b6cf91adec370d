// Host runtime and C ABI of the B200 multi-domain TDBEM library
// (include/tdbem.h).  The host side owns the integer bookkeeping the
// reference does in C++ (model validation, GlobalDofMap numbering, the
// octree leaf partition of the preconditioner, index permutations); every
// floating-point stage of the path runs in the CUDA kernels of
// assemble.cu and march.cu.
#include "../../include/tdbem.h"
#include "assemble.cuh"
#include "host_error.h"
#include "march.cuh"
#include "tdbem_common.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>
#include <limits>

using namespace tdbem;

namespace {

thread_local std::string g_error;

tdbem_status fail(tdbem_status s, const std::string& msg)
{
    g_error = msg;
    return s;
}

}  // namespace

namespace tdbem {
void set_last_error(const std::string& message) { g_error = message; }
}  // namespace tdbem

namespace {

#define CUDA_TRY(expr)                                                                                       \
    do {                                                                                                     \
        cudaError_t e_ = (expr);                                                                             \
        if (e_ != cudaSuccess)                                                                               \
            return fail(e_ == cudaErrorMemoryAllocation ? TDBEM_OUT_OF_MEMORY : TDBEM_CUDA_ERROR,            \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));                                 \
    } while (0)

// Owning device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t alloc(size_t n)
    {
        release();
        bytes = n;
        if (n == 0) return cudaSuccess;
        return cudaMalloc(&p, n);
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
    void adopt(void* q, size_t n)
    {
        release();
        p = q;
        bytes = n;
    }
};

template <class T>
cudaError_t upload(DevBuf& b, const std::vector<T>& v, cudaStream_t s)
{
    cudaError_t e = b.alloc(std::max<size_t>(v.size(), 1) * sizeof(T));
    if (e != cudaSuccess) return e;
    if (v.empty()) return cudaSuccess;
    return cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

template <class T>
cudaError_t download(std::vector<T>& v, const DevBuf& b, size_t n, cudaStream_t s)
{
    v.resize(n);
    if (n == 0) return cudaSuccess;
    cudaError_t e = cudaMemcpyAsync(v.data(), b.p, n * sizeof(T), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s);
}

// ---------------------------------------------------------------------------
// Quadrature rules (GaussNumeMatrix + quadinfo for the constant element,
// DBEM1/gaussnumematrix.cpp:4-86, DBEM1/quadinfo.cpp:83-398).  The Gauss-
// Legendre nodes and weights are the 15-decimal values of the reference's
// gaussposition / gaussweight tables.
const double kGP3[3] = {-0.774596669241484, 0.0, 0.774596669241484};
const double kGW3[3] = {0.555555555555555, 0.888888888888889, 0.555555555555555};
const double kGP4[4] = {-0.861136311594052, -0.339981043584856, 0.339981043584856, 0.861136311594052};
const double kGW4[4] = {0.347854845137454, 0.652145154862546, 0.652145154862546, 0.347854845137454};

double c_theta_start(int a) { return a == 0 ? -0.75 * kPi : a == 1 ? -0.25 * kPi : a == 2 ? 0.25 * kPi : 0.75 * kPi; }
double c_theta_diff() { return 0.5 * kPi; }
double c_theta_from_local(double lt, int a) { return c_theta_start(a) + 0.5 * (lt + 1.0) * c_theta_diff(); }
double c_alpha(double t, int a)
{
    return a == 0 ? -1.0 / std::sin(t) : a == 1 ? 1.0 / std::cos(t) : a == 2 ? 1.0 / std::sin(t) : -1.0 / std::cos(t);
}
double c_polar(double lr, double t, int a) { return 0.5 * (lr + 1.0) * c_alpha(t, a); }

void build_rules(double gap, QuadRules& q, std::vector<double>& secpw_pos, std::vector<double>& secpw_val)
{
    std::memset(&q, 0, sizeof q);
    q.gap = gap;
    q.lc0[0] = -gap;
    q.lc0[1] = -gap;
    const double lc[8][2] = {{-gap, -gap}, {gap, -gap}, {gap, gap}, {-gap, gap},
                             {0.0, -gap}, {gap, 0.0}, {0.0, gap}, {-gap, 0.0}};
    double sp[16][2], sa[16], pwrp[9][2], pwra[9];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
            const int m = i * 4 + j;
            q.rp[m][0] = sp[m][0] = kGP4[j];
            q.rp[m][1] = sp[m][1] = kGP4[i];
            sa[m] = kGW4[j] * kGW4[i];
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const int m = i * 3 + j;
            pwrp[m][0] = kGP3[j];
            pwrp[m][1] = kGP3[i];
            pwra[m] = kGW3[j] * kGW3[i];
        }
    // m_NRGV[0] = quadinfo::N(s)[0] * weight (DBEM1/quadinfo.h:153-176)
    for (int m = 0; m < 16; ++m) {
        const double s1 = q.rp[m][0], s2 = q.rp[m][1];
        const double lx = lc[1][0] - lc[0][0], ly = lc[3][1] - lc[0][1], lxly = lx * ly;
        const double hx = 0.25 * lx * lxly, hy = 0.25 * ly * lxly;
        double r0 = (s1 - lc[1][0]) * (s2 - lc[3][1]) / lxly;
        const double r4 = (s1 - lc[0][0]) * (s1 - lc[1][0]) * (s2 - lc[6][1]) / (hx);
        const double r7 = (s1 - lc[5][0]) * (s2 - lc[0][1]) * (s2 - lc[3][1]) / (hy);
        r0 -= 0.5 * (r4 + r7);
        q.nrgv0[m] = r0 * sa[m];
    }
    const double L = 2.0 / kNumPW;
    for (int i = 0; i < kNumPW; ++i)
        for (int j = 0; j < kNumPW; ++j) {
            const int p = i * kNumPW + j;
            q.cenpw[p][0] = -1.0 + L / 2.0 + L * j;
            q.cenpw[p][1] = -1.0 + L / 2.0 + L * i;
            for (int m = 0; m < 9; ++m) {
                q.lpospw[p][m][0] = q.cenpw[p][0] + pwrp[m][0] / kNumPW;
                q.lpospw[p][m][1] = q.cenpw[p][1] + pwrp[m][1] / kNumPW;
                q.pwgv[p][m] = pwra[m] * (L / 2.0) * (L / 2.0);
            }
        }
    for (int a = 0; a < 4; ++a)
        for (int m = 0; m < 16; ++m) {
            const double th = c_theta_from_local(sp[m][0], a);
            const double fa = 0.25 * c_alpha(th, a) * c_theta_diff();
            const double rou = c_polar(sp[m][1], th, a);
            q.sec_pos[a][0][m] = rou * std::cos(th);
            q.sec_pos[a][1][m] = rou * std::sin(th);
            q.sec_val[a][m] = rou * fa * sa[m];
            const double temp = rou * fa * sa[m];
            q.fm1_sec[a][m] = temp / rou / rou;
        }
    for (int a = 0; a < 4; ++a)
        for (int m = 0; m < 4; ++m) {
            const double th = c_theta_from_local(kGP4[m], a);
            q.line_pos[a][m] = th;
            q.fm1_line[a][m] = 0.5 * c_theta_diff() * std::log(c_polar(1.0, th, a)) * kGW4[m];
        }
    const double Ls = 2.0 / kSinNumPW;
    secpw_pos.assign(4 * 2 * kSinNumPW2 * 9, 0.0);
    secpw_val.assign(4 * kSinNumPW2 * 9, 0.0);
    for (int a = 0; a < 4; ++a)
        for (int i = 0; i < kSinNumPW; ++i)
            for (int j = 0; j < kSinNumPW; ++j) {
                const int p = i * kSinNumPW + j;
                const double c0 = -1.0 + Ls / 2.0 + Ls * j, c1 = -1.0 + Ls / 2.0 + Ls * i;
                for (int m = 0; m < 9; ++m) {
                    const double l0 = c0 + pwrp[m][0] / kSinNumPW, l1 = c1 + pwrp[m][1] / kSinNumPW;
                    const double th = c_theta_from_local(l0, a);
                    const double fa = 0.25 * c_alpha(th, a) * c_theta_diff();
                    const double rou = c_polar(l1, th, a);
                    secpw_pos[((a * 2 + 0) * kSinNumPW2 + p) * 9 + m] = rou * std::cos(th);
                    secpw_pos[((a * 2 + 1) * kSinNumPW2 + p) * 9 + m] = rou * std::sin(th);
                    secpw_val[(a * kSinNumPW2 + p) * 9 + m] = rou * fa * (pwra[m] * (Ls / 2.0) * (Ls / 2.0));
                }
            }
}

DynaMat build_mat(double v, double G, double rho, double dt)
{
    DynaMat m;
    m.v = v;
    m.G = G;
    m.Rou = rho;
    m.C1 = std::sqrt((2.0 - 2.0 * v) / (1.0 - 2.0 * v) * G / rho);
    m.C2 = std::sqrt(G / rho);
    m.Dt = dt;
    m.Dt2 = 2.0 * dt;
    m.Dt_2 = dt * dt;
    m.Dt_3 = dt * dt * dt;
    m.OneOverFourPaiRou = kOneOver4Pi / rho;
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
    m.STCoef1 = -1.0 / (8.0 * kPi * (1.0 - m.v));
    m.STCoef2 = 1.0 - 2.0 * m.v;
    m.Third_1OC23_1OC13 = 1.0 / 3.0 * (m.OneOverC2_3 - m.OneOverC1_3);
    m.Half_1OC22_1OC12 = 0.5 * (m.OneOverC2_2 - m.OneOverC1_2);
    return m;
}

// The material constants with their derivatives with respect to E (G = E /
// (2 (1 + v)), wave speeds proportional to sqrt(E / rho)); rho, v and the
// time step are held fixed.
DynaMatD build_mat_dual(const DynaMat& m)
{
    const double E = 2.0 * m.G * (1.0 + m.v);
    // X proportional to E^(p/2)
    auto sd = [&](double x, double p) { return QDual(x, 0.5 * p * x / E); };
    DynaMatD d;
    d.G = QDual(m.G, m.G / E);
    d.v = m.v;
    d.Rou = QDual(m.Rou);
    d.C1 = sd(m.C1, 1);
    d.C2 = sd(m.C2, 1);
    d.Dt = m.Dt;
    d.Dt2 = m.Dt2;
    d.Dt_2 = m.Dt_2;
    d.Dt_3 = m.Dt_3;
    d.C1_2 = sd(m.C1_2, 2);
    d.C2_2 = sd(m.C2_2, 2);
    d.OneOverC1_2 = sd(m.OneOverC1_2, -2);
    d.OneOverC2_2 = sd(m.OneOverC2_2, -2);
    d.OneOverC1_3 = sd(m.OneOverC1_3, -3);
    d.OneOverC2_3 = sd(m.OneOverC2_3, -3);
    d.C2_2OverC1_2 = m.C2_2OverC1_2;
    d.C2_2OverC1_3 = sd(m.C2_2OverC1_3, -1);
    d.C1Dt = sd(m.C1Dt, 1);
    d.C2Dt = sd(m.C2Dt, 1);
    d.OneOverFourPaiRou = QDual(m.OneOverFourPaiRou);
    d.Third_1OC23_1OC13 = sd(m.Third_1OC23_1OC13, -3);
    d.Half_1OC22_1OC12 = sd(m.Half_1OC22_1OC12, -2);
    d.STCoef1 = m.STCoef1;
    d.STCoef2 = m.STCoef2;
    return d;
}

double dist3(const double* a, const double* b)
{
    return std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) + (a[2] - b[2]) * (a[2] - b[2]));
}

// Octree of element centres (AssignCubeSize, InitRoot, CreateTree,
// CreateLeafPointer, RenumberPointID; DBEM1/geo.cpp:6-39, 109-137,
// DBEM1/tree.cpp:12-325).  A node's point list is built by head insertion,
// so each child's points come out in reverse order of arrival.
struct Cube {
    double c[3];
    double len;
};

bool cube_isin(const double* pt, const Cube& cb)
{
    const double l = 0.5 * cb.len;
    for (int i = 0; i < 3; i++) {
        const double ds = cb.c[i] - pt[i];
        if (ds * ds > l * l * 1.0001) return false;
    }
    return true;
}

void tree_split(const std::vector<double>& node, const Cube& cb, std::vector<int64_t>& list, int64_t max_point,
                std::vector<int64_t>& repid, std::vector<int64_t>& lb, std::vector<int64_t>& lc, int depth)
{
    if ((int64_t)list.size() <= max_point || depth > 60) {
        lb.push_back((int64_t)repid.size());
        lc.push_back((int64_t)list.size());
        repid.insert(repid.end(), list.begin(), list.end());
        return;
    }
    Cube ch[8];
    std::vector<int64_t> arrive[8];
    for (int i = 0; i < 8; ++i) {
        ch[i].len = 0.5 * cb.len;
        const double half = 0.5 * ch[i].len;
        int bit = 1;
        for (int a = 0; a < 3; a++) {
            ch[i].c[a] = cb.c[a] + ((bit & i) == 0 ? -1 : 1) * half;
            bit <<= 1;
        }
    }
    for (int64_t pid : list) {
        const double* pt = &node[3 * pid];
        int near = -1;
        for (int i = 0; i < 8; ++i)
            if (cube_isin(pt, ch[i])) {
                near = i;
                break;
            }
        if (near < 0) {
            double best = dist3(pt, ch[0].c);
            near = 0;
            for (int i = 1; i < 8; ++i) {
                const double dd = dist3(pt, ch[i].c);
                if (best > dd) {
                    best = dd;
                    near = i;
                }
            }
        }
        arrive[near].push_back(pid);
    }
    for (int i = 0; i < 8; ++i)
        if (!arrive[i].empty()) {
            std::reverse(arrive[i].begin(), arrive[i].end());
            tree_split(node, ch[i], arrive[i], max_point, repid, lb, lc, depth + 1);
        }
}

}  // namespace

// ---------------------------------------------------------------------------
// Transposed operators and scratch of the adjoint march (built by the first
// tdbem_md_march_vjp of a handle).
struct AdjointState {
    DevBuf at_rp, at_col, at_val, pinvT;            // A'^T (perm space) and its leaf inverses
    DevBuf tptr, trow, tval;                        // history blocks by (type, column), then k
    DevBuf lam, adj, g, gp;                         // adjoint right-hand sides, state adjoint, solve rhs
    DevBuf b, bp, x, rv, u, V, W, AW, givens, status, flags, audit, xring, wring, known, out_lu, out_lt;
    DevBuf unk_of, perm_of_row;
    DevBuf unk_src, kt_ptr, kt_row, kt_blk;         // write-back sources per unknown; KnownM by columns
    DevBuf cot_u, cot_t, gk, contrib, flags_all;    // per-call cotangents, gradient, scratch, per-step flags
};

// CUDA events a handle reuses from march to march (a march records seven
// per time step, the host-buffer march two per copy chunk): created on first
// need, grown on demand, destroyed with the handle.
struct EventPool {
    std::vector<cudaEvent_t> ev;
    unsigned flags = cudaEventDefault;
    // the first n events of the pool (created as needed)
    cudaError_t take(size_t n, std::vector<cudaEvent_t>& out)
    {
        while (ev.size() < n) {
            cudaEvent_t e = nullptr;
            const cudaError_t r = cudaEventCreateWithFlags(&e, flags);
            if (r != cudaSuccess) return r;
            ev.push_back(e);
        }
        out.assign(ev.begin(), ev.begin() + (std::ptrdiff_t)n);
        return cudaSuccess;
    }
    ~EventPool()
    {
        for (auto& e : ev) cudaEventDestroy(e);
    }
};

struct tdbem_handle {
    int device = 0;
    EventPool ev_timed;                                   // MarchRun's step events
    EventPool ev_order{{}, cudaEventDisableTiming};       // ordering-only events (copy chunks, grouped march)
    cudaStream_t s0 = nullptr;    // default stream of the handle
    cudaStream_t hp = nullptr;    // high-priority stream of the per-step chain
    cudaStream_t side = nullptr;  // low-priority stream of the overlapped history part
    cudaStream_t cin = nullptr, cout = nullptr;  // host march: input and output copies beside the steps
    // model
    int64_t E = 0, P = 0, I = 0;
    int D = 0;
    int nstep = 0, restart = 0, max_leaf = 0, precision = 0, R = 1;
    double tol = 0, dt = 0, gap = 0, max_length = 1000.0;
    std::vector<double> points;
    std::vector<int64_t> elements;
    std::vector<int32_t> bcid, domain_of, surface;
    std::vector<int64_t> itf;  // I*5
    std::vector<int32_t> dom_begin, dom_count;
    std::vector<DynaMat> mats;
    // dof map
    std::vector<int64_t> uref_block, tref_block, hist_block, pref;
    std::vector<double> uref_sign, tref_sign, hu_sign, ht_sign;
    std::vector<int32_t> uref_known, tref_known, hist_owner;
    int64_t n_unknown = 0, n_known = 0, n_hist = 0;
    std::vector<int32_t> known_elem;
    std::vector<double> known_sign;
    // geometry (host copies of device results)
    std::vector<double> node, trans, itf_trans;
    // preconditioner layout
    std::vector<int64_t> repid, leaf_begin, leaf_count;
    // matrices (host copies in reference layout)
    std::vector<int32_t> a_rp, a_col, k_rp, k_col;
    std::vector<double> a_val, k_val;
    int K = 0;
    int64_t h_nnz = 0;
    int64_t hist_mts_blocks = 0, hist_mgs_blocks = 0;  // all MTS_k, all MGS_k
    double assembly_s = 0.0;                         // host wall time of the last assemble / load
    std::vector<int64_t> h_kptr;
    bool assembled = false;
    bool record = false;
    bool saved_forward = false;  // the last march was tdbem_md_march_forward (states kept)
    bool diag_ready = false;     // the last march was a recorded host march (rhs diagnostics)
    int cluster = 1;
    int dsm_rows = 0;   // GMRES Krylov copies in shared memory for owned ranges of this many rows (0: off)
    int groups = 1;
    int rhs_cpt = 0;              // history pass: load cases per thread (0 = the default for R)
    std::vector<int32_t> ap_col;  // A' columns (perm space), for re-laying the GMRES clusters
    // device buffers
    DevBuf d_rules, d_secpw_pos, d_secpw_val, d_points, d_elements;
    DevBuf g_cc, g_center, g_radius, g_rpw, g_rcen, g_node, g_trans, g_u1, g_t1, g_t2, g_bcid, g_domain, g_surface;
    DevBuf d_uref_sign, d_tref_sign, d_hu_sign, d_ht_sign, d_itf_trans, d_uref_block, d_tref_block, d_hist_block;
    DevBuf d_uref_known, d_tref_known, d_hist_owner, d_known_elem, d_known_sign, d_itf_pairs, d_itf_sign;
    DevBuf d_h_kptr, d_h_col, d_h_val, d_h_val32;
    DevBuf d_r_ptr, d_r_meta, d_r_off, d_r_val;  // run layout of steps k >= run_k (T-step history pass)
    int64_t r_nb = 0, r_runs = 0;
    int run_k = 0;
    DevBuf d_k_rp, d_k_col, d_k_val, d_k_elem, d_k_sgn;
    DevBuf d_a_rp, d_a_col, d_a_val, d_a_val32, d_row_of, d_unk_of, d_perm_of_unk;
    DevBuf d_leaf_begin, d_leaf_count, d_leaf_of_perm, d_leaf_off, d_pinv, d_pinv32, d_cta_leaf, d_a_colx;
    DevBuf d_xring, d_wring, d_bulk, d_b, d_bp, d_x, d_rv, d_u, d_V, d_W, d_AW, d_givens, d_status,
        d_flags, d_audit;
    DevBuf d_known, d_out_lu, d_out_lt, d_rec_rhs, d_rec_x, d_xold;
    std::unique_ptr<AdjointState> adjoint;

    ElemGeom geom() const
    {
        ElemGeom g;
        g.cc = g_cc.as<double>();
        g.center = g_center.as<double>();
        g.radius = g_radius.as<double>();
        g.rpw = g_rpw.as<double>();
        g.rcen = g_rcen.as<double>();
        g.node = g_node.as<double>();
        g.trans = g_trans.as<double>();
        g.on_u1 = g_u1.as<double>();
        g.on_t1 = g_t1.as<double>();
        g.on_t2 = g_t2.as<double>();
        g.bcid = g_bcid.as<int32_t>();
        g.domain = g_domain.as<int32_t>();
        g.surface = g_surface.as<int32_t>();
        return g;
    }
};

namespace {

tdbem_status build_dofmap(tdbem_handle* h)
{
    const int64_t E = h->E;
    h->uref_block.assign(E, -1);
    h->tref_block.assign(E, -1);
    h->hist_block.assign(E, -1);
    h->pref.assign(E, -1);
    h->uref_sign.assign(E, 1.0);
    h->tref_sign.assign(E, 1.0);
    h->hu_sign.assign(E, 1.0);
    h->ht_sign.assign(E, 1.0);
    h->uref_known.assign(E, 0);
    h->tref_known.assign(E, 0);
    h->hist_owner.assign(E, 1);
    std::vector<char> side(E, 0);
    int64_t nu = 0, nk = 0, nh = 0;
    // GlobalDofMap::Build, DBEM1/multidomain.cpp:777-900: interface pairs
    // first (U block, T block; B-side T sign = normalSign), then outer
    // elements in element order.
    for (int64_t i = 0; i < h->I; ++i) {
        const int64_t a = h->itf[5 * i + 1], b = h->itf[5 * i + 3];
        const double s = h->itf[5 * i + 4] == 0 ? -1.0 : (double)h->itf[5 * i + 4];
        const int64_t ub = nu++, tb = nu++;
        h->uref_block[a] = h->uref_block[b] = ub;
        h->tref_block[a] = h->tref_block[b] = tb;
        h->tref_sign[b] = s;
        h->pref[a] = ub;
        h->pref[b] = tb;
        h->hist_block[a] = h->hist_block[b] = nh;
        h->ht_sign[b] = s;
        h->hist_owner[b] = 0;
        ++nh;
        side[a] = side[b] = 1;
    }
    h->known_elem.clear();
    h->known_sign.clear();
    for (int64_t i = 0; i < E; ++i) {
        if (side[i]) continue;
        if (h->bcid[i] == 123) {
            h->uref_block[i] = nk++;
            h->uref_known[i] = 1;
            h->tref_block[i] = nu;
            h->pref[i] = nu++;
        } else {
            h->uref_block[i] = nu;
            h->pref[i] = nu++;
            h->tref_block[i] = nk++;
            h->tref_known[i] = 1;
        }
        h->known_elem.push_back((int32_t)i);
        h->known_sign.push_back(1.0);
        h->hist_block[i] = nh++;
    }
    h->n_unknown = nu;
    h->n_known = nk;
    h->n_hist = nh;
    if (nu != E)
        return fail(TDBEM_DOFMAP_INVALID, "unknown blocks " + std::to_string(nu) + " != equation blocks " +
                                              std::to_string(E));
    std::vector<int> used(E, 0);
    for (int64_t i = 0; i < E; ++i) used[h->pref[i]]++;
    for (int64_t u = 0; u < E; ++u)
        if (used[u] != 1) return fail(TDBEM_DOFMAP_INVALID, "preferred unknown block used " + std::to_string(used[u]) + " times");
    return TDBEM_OK;
}

template <class T>
cudaError_t up(DevBuf& b, const std::vector<T>& v, cudaStream_t s)
{
    return upload(b, v, s);
}

}  // namespace

extern "C" {

const char* tdbem_status_string(tdbem_status s)
{
    switch (s) {
    case TDBEM_OK: return "ok";
    case TDBEM_INVALID_INPUT: return "invalid input";
    case TDBEM_DOFMAP_INVALID: return "dof map invalid";
    case TDBEM_SINGULAR_BLOCK: return "singular preconditioner block";
    case TDBEM_NOT_CONVERGED: return "GMRES did not converge";
    case TDBEM_CUDA_ERROR: return "CUDA error";
    case TDBEM_OUT_OF_MEMORY: return "out of device memory";
    case TDBEM_NOT_ASSEMBLED: return "matrices not assembled";
    }
    return "unknown status";
}

const char* tdbem_last_error(void) { return g_error.c_str(); }
int32_t tdbem_abi_version(void) { return TDBEM_ABI_VERSION; }

tdbem_status tdbem_md_create(const tdbem_problem* pr, int32_t device, tdbem_handle** out)
{
    g_error.clear();
    if (!pr || !out) return fail(TDBEM_INVALID_INPUT, "null argument");
    *out = nullptr;
    if (pr->n_elements <= 0 || pr->n_points <= 0 || pr->n_domains <= 0 || pr->n_domains > kMaxDomains ||
        pr->n_domains > pr->n_elements || pr->n_steps < 0 || pr->restart <= 0 || pr->restart > 480 ||
        pr->max_leaf <= 0 || pr->n_loads < 1 || pr->n_interfaces < 0 || !pr->points || !pr->elements ||
        !pr->bcid || !pr->materials || (pr->n_interfaces > 0 && !pr->interfaces))
        return fail(TDBEM_INVALID_INPUT, "invalid sizes or null arrays in tdbem_problem");
    if (!march_supported_loads(pr->n_loads))
        return fail(TDBEM_INVALID_INPUT, "n_loads must be 1, 2, 4, 8, 16 or 32");
    if (!(pr->tol > 0.0) || !(pr->beta > 0.0) || !(pr->gap > 0.0 && pr->gap <= 1.0))
        return fail(TDBEM_INVALID_INPUT, "tol, beta and gap must be positive (gap <= 1)");
    auto h = std::make_unique<tdbem_handle>();
    h->device = device;
    h->E = pr->n_elements;
    h->P = pr->n_points;
    h->D = pr->n_domains;
    h->I = pr->n_interfaces;
    h->nstep = pr->n_steps;
    h->restart = pr->restart;
    h->tol = pr->tol;
    h->gap = pr->gap;
    h->max_leaf = pr->max_leaf;
    h->max_length = pr->max_length > 0 ? pr->max_length : 1000.0;
    h->precision = pr->precision;
    h->R = pr->n_loads;
    const int64_t E = h->E;
    h->points.assign(pr->points, pr->points + 3 * h->P);
    h->elements.assign(pr->elements, pr->elements + 8 * E);
    h->bcid.assign(pr->bcid, pr->bcid + E);
    for (int64_t i = 0; i < E; ++i) {
        if (h->bcid[i] != 123 && h->bcid[i] != 456)
            return fail(TDBEM_INVALID_INPUT, "element " + std::to_string(i) + " has BCID " +
                                                 std::to_string(h->bcid[i]) + "; only 123 and 456 are supported");
        for (int c = 0; c < 8; ++c)
            if (h->elements[8 * i + c] < 0 || h->elements[8 * i + c] >= h->P)
                return fail(TDBEM_INVALID_INPUT, "element " + std::to_string(i) + " references a point out of range");
    }
    // dt = beta * mean|P0 - P1| / c1(card) (DBEM1/DBEM.cpp:909-914)
    double ave = 0.0;
    for (int64_t i = 0; i < E; ++i)
        ave += dist3(&h->points[3 * h->elements[8 * i]], &h->points[3 * h->elements[8 * i + 1]]);
    ave /= (double)E;
    const double G = pr->card_E / 2.0 / (1 + pr->card_nu);
    const double c1 = std::sqrt((2.0 - 2.0 * pr->card_nu) / (1.0 - 2.0 * pr->card_nu) * G / pr->card_rho);
    if (!(c1 > 0.0) || !std::isfinite(c1)) return fail(TDBEM_INVALID_INPUT, "card material gives no wave speed");
    if (!(pr->dt >= 0.0) || !std::isfinite(pr->dt)) return fail(TDBEM_INVALID_INPUT, "dt must be finite and >= 0");
    h->dt = pr->dt > 0.0 ? pr->dt : pr->beta * ave / c1;
    for (int d = 0; d < h->D; ++d) {
        const double Ed = pr->materials[3 * d], nu = pr->materials[3 * d + 1], rho = pr->materials[3 * d + 2];
        if (!(Ed > 0.0) || !(rho > 0.0) || !(nu > -1.0 && nu < 0.5))
            return fail(TDBEM_INVALID_INPUT, "domain " + std::to_string(d) + " has an invalid material");
        h->mats.push_back(build_mat(nu, Ed / 2.0 / (1.0 + nu), rho, h->dt));
    }
    // contiguous equal element ranges (DBEM1/multidomain.cpp:1413-1436)
    h->domain_of.assign(E, 0);
    int64_t b = 0;
    for (int d = 0; d < h->D; ++d) {
        const int64_t c = E / h->D + (d < E % h->D ? 1 : 0);
        h->dom_begin.push_back((int32_t)b);
        h->dom_count.push_back((int32_t)c);
        for (int64_t i = b; i < b + c; ++i) h->domain_of[i] = d;
        b += c;
    }
    h->surface.assign(E, 0);
    h->itf.assign(pr->interfaces, pr->interfaces + 5 * h->I);
    for (int64_t i = 0; i < h->I; ++i) {
        const int64_t dA = h->itf[5 * i], eA = h->itf[5 * i + 1], dB = h->itf[5 * i + 2], eB = h->itf[5 * i + 3];
        if (dA < 0 || dA >= h->D || dB < 0 || dB >= h->D || dA == dB || eA < 0 || eA >= E || eB < 0 || eB >= E ||
            h->domain_of[eA] != dA || h->domain_of[eB] != dB || h->surface[eA] || h->surface[eB])
            return fail(TDBEM_INVALID_INPUT, "invalid interface " + std::to_string(i));
        h->surface[eA] = h->surface[eB] = 1;
        if (h->itf[5 * i + 4] == 0) h->itf[5 * i + 4] = -1;
    }
    tdbem_status st = build_dofmap(h.get());
    if (st != TDBEM_OK) return st;

    CUDA_TRY(cudaSetDevice(device));
    CUDA_TRY(cudaStreamCreateWithFlags(&h->s0, cudaStreamNonBlocking));
    {
        int least = 0, greatest = 0;
        CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CUDA_TRY(cudaStreamCreateWithPriority(&h->hp, cudaStreamNonBlocking, greatest));
        CUDA_TRY(cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, least));
        CUDA_TRY(cudaStreamCreateWithFlags(&h->cin, cudaStreamNonBlocking));
        CUDA_TRY(cudaStreamCreateWithFlags(&h->cout, cudaStreamNonBlocking));
    }
    cudaStream_t s = h->s0;
    QuadRules rules;
    std::vector<double> secpos, secval;
    build_rules(h->gap, rules, secpos, secval);
    CUDA_TRY(h->d_rules.alloc(sizeof(QuadRules)));
    CUDA_TRY(cudaMemcpyAsync(h->d_rules.p, &rules, sizeof rules, cudaMemcpyHostToDevice, s));
    CUDA_TRY(up(h->d_secpw_pos, secpos, s));
    CUDA_TRY(up(h->d_secpw_val, secval, s));
    CUDA_TRY(up(h->d_points, h->points, s));
    CUDA_TRY(up(h->d_elements, h->elements, s));
    CUDA_TRY(upload_materials(h->mats.data(), h->D, s));
    CUDA_TRY(h->g_cc.alloc(E * 24 * 8));
    CUDA_TRY(h->g_center.alloc(E * 3 * 8));
    CUDA_TRY(h->g_radius.alloc(E * 8));
    CUDA_TRY(h->g_rpw.alloc(E * 8));
    CUDA_TRY(h->g_rcen.alloc(E * 108 * 8));
    CUDA_TRY(h->g_node.alloc(E * 3 * 8));
    CUDA_TRY(h->g_trans.alloc(E * 9 * 8));
    CUDA_TRY(h->g_u1.alloc(E * 9 * 8));
    CUDA_TRY(h->g_t1.alloc(E * 9 * 8));
    CUDA_TRY(h->g_t2.alloc(E * 9 * 8));
    CUDA_TRY(up(h->g_bcid, h->bcid, s));
    CUDA_TRY(up(h->g_domain, h->domain_of, s));
    CUDA_TRY(up(h->g_surface, h->surface, s));
    ElemGeom g = h->geom();
    geometry_kernel<<<ceil_div(E, 128), 128, 0, s>>>((int)E, h->d_points.as<double>(), h->d_elements.as<int64_t>(),
                                                      h->d_rules.as<QuadRules>(), g);
    CUDA_TRY(cudaGetLastError());
    singular_kernel<<<(unsigned)E, 256, 0, s>>>((int)E, h->d_rules.as<QuadRules>(), h->d_secpw_pos.as<double>(),
                                                h->d_secpw_val.as<double>(), g);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(download(h->node, h->g_node, 3 * E, s));
    CUDA_TRY(download(h->trans, h->g_trans, 9 * E, s));
    // interface B-side transform T_B T_A^T (BuildLocalTransformFromReference,
    // DBEM1/multidomain.cpp:1603-1645)
    h->itf_trans.assign(9 * E, 0.0);
    for (int64_t i = 0; i < E; ++i) h->itf_trans[9 * i] = h->itf_trans[9 * i + 4] = h->itf_trans[9 * i + 8] = 1.0;
    for (int64_t k = 0; k < h->I; ++k) {
        const int64_t a = h->itf[5 * k + 1], bb = h->itf[5 * k + 3];
        for (int si = 0; si < 3; ++si)
            for (int r = 0; r < 3; ++r) {
                double dot = 0.0;
                for (int ax = 0; ax < 3; ++ax) dot += h->trans[9 * bb + si * 3 + ax] * h->trans[9 * a + r * 3 + ax];
                h->itf_trans[9 * bb + si * 3 + r] = dot;
            }
    }
    std::vector<int32_t> pairs;
    std::vector<double> isign;
    for (int64_t k = 0; k < h->I; ++k) {
        pairs.push_back((int32_t)h->itf[5 * k + 1]);
        pairs.push_back((int32_t)h->itf[5 * k + 3]);
        isign.push_back((double)h->itf[5 * k + 4]);
    }
    CUDA_TRY(up(h->d_itf_pairs, pairs, s));
    CUDA_TRY(up(h->d_itf_sign, isign, s));
    CUDA_TRY(up(h->d_uref_sign, h->uref_sign, s));
    CUDA_TRY(up(h->d_tref_sign, h->tref_sign, s));
    CUDA_TRY(up(h->d_hu_sign, h->hu_sign, s));
    CUDA_TRY(up(h->d_ht_sign, h->ht_sign, s));
    CUDA_TRY(up(h->d_itf_trans, h->itf_trans, s));
    CUDA_TRY(up(h->d_uref_block, h->uref_block, s));
    CUDA_TRY(up(h->d_tref_block, h->tref_block, s));
    CUDA_TRY(up(h->d_hist_block, h->hist_block, s));
    CUDA_TRY(up(h->d_uref_known, h->uref_known, s));
    CUDA_TRY(up(h->d_tref_known, h->tref_known, s));
    CUDA_TRY(up(h->d_hist_owner, h->hist_owner, s));
    CUDA_TRY(up(h->d_known_elem, h->known_elem, s));
    CUDA_TRY(up(h->d_known_sign, h->known_sign, s));
    // preconditioner leaf partition
    {
        double rmin[3], rmax[3];
        for (int i = 0; i < 3; ++i) rmin[i] = rmax[i] = h->node[i];
        for (int64_t k = 1; k < E; ++k)
            for (int i = 0; i < 3; ++i) {
                rmin[i] = std::min(rmin[i], h->node[3 * k + i]);
                rmax[i] = std::max(rmax[i], h->node[3 * k + i]);
            }
        Cube root;
        double ml = rmax[0] - rmin[0];
        for (int i = 0; i < 3; ++i) {
            if (ml < rmax[i] - rmin[i]) ml = rmax[i] - rmin[i];
            root.c[i] = rmin[i] + 0.5 * (rmax[i] - rmin[i]);
        }
        root.len = 1.02 * ml;
        std::vector<int64_t> list(E);
        std::iota(list.begin(), list.end(), 0);
        tree_split(h->node, root, list, h->max_leaf, h->repid, h->leaf_begin, h->leaf_count, 0);
    }
    CUDA_TRY(cudaStreamSynchronize(s));
    *out = h.release();
    return TDBEM_OK;
}

void tdbem_md_destroy(tdbem_handle* h)
{
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->s0) cudaStreamSynchronize(h->s0);
    cudaStream_t s = h->s0, a = h->hp, b = h->side, ci = h->cin, co = h->cout;
    delete h;
    if (s) cudaStreamDestroy(s);
    if (a) cudaStreamDestroy(a);
    if (b) cudaStreamDestroy(b);
    if (ci) cudaStreamDestroy(ci);
    if (co) cudaStreamDestroy(co);
}

}  // extern "C"

namespace {

// Compact a pair buffer into CSR rows: returns row pointers (E+1) and
// device col/val arrays sized to the block count.
tdbem_status compact(tdbem_handle* h, const PairSpace& ps, const DevBuf& flags, const DevBuf& blocks, int mask,
                     ScatterCols sc, std::vector<int64_t>& rp, DevBuf& d_rp, DevBuf& col, DevBuf& val, cudaStream_t s)
{
    const int E = (int)h->E;
    DevBuf counts;
    CUDA_TRY(counts.alloc(sizeof(int) * E));
    count_rows_kernel<<<ceil_div(E, 8), 256, 0, s>>>(ps, flags.as<uint8_t>(), mask, E, counts.as<int>());
    CUDA_TRY(cudaGetLastError());
    std::vector<int> c;
    CUDA_TRY(download(c, counts, E, s));
    rp.assign(E + 1, 0);
    for (int i = 0; i < E; ++i) rp[i + 1] = rp[i] + c[i];
    CUDA_TRY(up(d_rp, rp, s));
    CUDA_TRY(col.alloc(sizeof(int32_t) * std::max<int64_t>(rp[E], 1)));
    CUDA_TRY(val.alloc(sizeof(double) * 9 * std::max<int64_t>(rp[E], 1)));
    scatter_rows_kernel<<<ceil_div(E, 8), 256, 0, s>>>(ps, flags.as<uint8_t>(), blocks.as<double>(), mask, E,
                                                        d_rp.as<int64_t>(), sc, col.as<int32_t>(), val.as<double>());
    CUDA_TRY(cudaGetLastError());
    return TDBEM_OK;
}

// Run layout of the history steps k >= 2T + 1 for the T-step history pass
// (two or more load cases; T = 2, or 3 with TDBEM_HISTORY_STEPS=3 and at
// least 7 history steps; off with TDBEM_RUNS=0).  Left out, and the march
// keeps the one-step pass, when the build would not fit in free device
// memory.  On the 3,072-element bar with 32 load cases T = 3 makes the
// history pass 15% faster but doubles the head pass on the GMRES chain
// (k <= 6): the march is 1% faster in mixed precision and 7% slower in FP64,
// so T = 2 is the default.
tdbem_status build_runs(tdbem_handle* h, cudaStream_t s)
{
    int steps = 2;
    if (const char* v = std::getenv("TDBEM_HISTORY_STEPS"))
        if (std::atoi(v) == 3) steps = 3;
    if (h->K < 2 * steps + 1) steps = 2;
    const int kRunK = 2 * steps + 1;
    h->d_r_ptr.release();
    h->d_r_meta.release();
    h->d_r_off.release();
    h->d_r_val.release();
    h->r_nb = h->r_runs = 0;
    h->run_k = 0;
    const int E = (int)h->E, K = h->K;
    if (K < kRunK || h->R < 2 || h->h_nnz == 0) return TDBEM_OK;
    if (const char* v = std::getenv("TDBEM_RUNS"))
        if (std::atoi(v) == 0) return TDBEM_OK;
    int64_t nb = 0;
    for (int r = 0; r < E; ++r)
        nb += h->h_kptr[(size_t)r * (K + 1) + K] - h->h_kptr[(size_t)r * (K + 1) + kRunK - 1];
    const bool mixed = h->precision == TDBEM_PRECISION_MIXED;
    size_t free_b = 0, total_b = 0;
    CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    if ((double)history_runs_bytes(nb, mixed) * 1.1 + (double)(1ull << 30) > (double)free_b) return TDBEM_OK;
    HistoryRuns hr;
    const void* vals = mixed ? static_cast<const void*>(h->d_h_val32.p) : static_cast<const void*>(h->d_h_val.p);
    cudaError_t e = build_history_runs(E, K, kRunK, h->h_kptr, h->d_h_kptr.as<int64_t>(), h->d_h_col.as<uint32_t>(),
                                       vals, h->h_nnz, mixed, hr, s);
    const size_t vs = mixed ? sizeof(float) : sizeof(double);
    h->d_r_ptr.adopt(hr.ptr, sizeof(int64_t) * (E + 1));
    h->d_r_meta.adopt(hr.meta, sizeof(uint2) * (size_t)hr.runs);
    h->d_r_off.adopt(hr.off, sizeof(int64_t) * (size_t)hr.runs);
    h->d_r_val.adopt(hr.val, vs * 9 * (size_t)hr.nb);
    if (e == cudaErrorMemoryAllocation) {
        // out of device memory part way: march with the one-step pass
        cudaGetLastError();
        h->d_r_ptr.release();
        h->d_r_meta.release();
        h->d_r_off.release();
        h->d_r_val.release();
        return TDBEM_OK;
    }
    CUDA_TRY(e);
    h->r_nb = hr.nb;
    h->r_runs = hr.runs;
    h->run_k = hr.kr;
    return TDBEM_OK;
}

// Build the stacked history structure from per-k device matrices.
tdbem_status stack_history(tdbem_handle* h, std::vector<std::vector<int64_t>>& mts_rp,
                           std::vector<std::vector<int64_t>>& mgs_rp, std::vector<HistK>& hk, cudaStream_t s)
{
    const int E = (int)h->E, K = h->K;
    h->hist_mts_blocks = h->hist_mgs_blocks = 0;
    for (int k = 0; k < K; ++k) {
        h->hist_mts_blocks += mts_rp[k][E];
        h->hist_mgs_blocks += mgs_rp[k][E];
    }
    h->h_kptr.assign((size_t)E * (K + 1), 0);
    int64_t pos = 0;
    for (int r = 0; r < E; ++r) {
        h->h_kptr[(size_t)r * (K + 1)] = pos;
        for (int k = 1; k <= K; ++k) {
            pos += (mts_rp[k - 1][r + 1] - mts_rp[k - 1][r]) + (mgs_rp[k - 1][r + 1] - mgs_rp[k - 1][r]);
            h->h_kptr[(size_t)r * (K + 1) + k] = pos;
        }
    }
    h->h_nnz = pos;
    if (h->n_hist >= (1 << 20) || K >= (1 << 11))
        return fail(TDBEM_INVALID_INPUT, "history columns or steps exceed the packed column format");
    CUDA_TRY(up(h->d_h_kptr, h->h_kptr, s));
    CUDA_TRY(h->d_h_col.alloc(sizeof(uint32_t) * std::max<int64_t>(pos, 1)));
    CUDA_TRY(h->d_h_val.alloc(sizeof(double) * 9 * std::max<int64_t>(pos, 1)));
    if (K > 0 && pos > 0) {
        DevBuf d_hk;
        CUDA_TRY(d_hk.alloc(sizeof(HistK) * K));
        CUDA_TRY(cudaMemcpyAsync(d_hk.p, hk.data(), sizeof(HistK) * K, cudaMemcpyHostToDevice, s));
        const int64_t tasks = (int64_t)E * K;
        stack_history_kernel<<<ceil_div(tasks, 8), 256, 0, s>>>(E, K, d_hk.as<HistK>(), h->d_h_kptr.as<int64_t>(),
                                                                 h->d_h_col.as<uint32_t>(), h->d_h_val.as<double>(), pos);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (h->precision == TDBEM_PRECISION_MIXED) {
        CUDA_TRY(h->d_h_val32.alloc(sizeof(float) * 9 * std::max<int64_t>(pos, 1)));
        to_float_kernel<<<1184, 256, 0, s>>>(h->d_h_val.as<double>(), h->d_h_val32.as<float>(), 9 * pos);
        CUDA_TRY(cudaGetLastError());
    }
    return TDBEM_OK;
}

// Last history step that can hold a nonzero block, from the reference's own
// skip rule.  A history block of step k integrates the kernels U(k), T1(k)
// and T2(k) of field element e at source node s of the same domain; each is
// skipped (NeedCal returns 0, DBEM1/dsquareelement.cpp:1156-1190) when
// nn * Dt >= (|c_e - s| + radius_e) / C2 of the domain, with nn = k for U and
// T1 and k - 1 for T2 (type 2).  So every block of step k is zero once
// (k - 1) Dt >= D / C2 with D the largest |c_e - s| + radius_e over the
// domain's (source, field) pairs: steps k >= 1 + D / (C2 Dt) are empty.  The
// bound adds one step against rounding in that comparison.
tdbem_status history_step_bound(tdbem_handle* h, cudaStream_t s, int& kb)
{
    const int64_t E = h->E;
    std::vector<double> center, radius;
    CUDA_TRY(download(center, h->g_center, 3 * (size_t)E, s));
    CUDA_TRY(download(radius, h->g_radius, (size_t)E, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    double steps = 0.0;
    for (int d = 0; d < h->D; ++d) {
        const int64_t b = h->dom_begin[d], n = h->dom_count[d];
        double dmax = 0.0;
        for (int64_t e = b; e < b + n; ++e)
            for (int64_t q = b; q < b + n; ++q)
                dmax = std::max(dmax, dist3(&center[3 * e], &h->node[3 * q]) + radius[e]);
        const double c2dt = h->mats[d].C2 * h->dt;
        if (!(c2dt > 0.0)) return fail(TDBEM_INVALID_INPUT, "domain " + std::to_string(d) + " has no shear wave speed");
        steps = std::max(steps, 1.0 + dmax / c2dt);
    }
    kb = (int)std::min(std::ceil(steps) + 1.0, 1.0e9);
    return TDBEM_OK;
}

// Permuted system matrix A', leaf inverses, GMRES partition and march state.
// GMRES launch layout: G clusters (load-case groups) of C CTAs; within a
// cluster every CTA owns a contiguous range of leaves of about equal point
// count, and the A' columns are tagged with their owner CTA and row within
// it so the products read Krylov vectors from the owners' shared memory
// when the per-CTA copies fit.
tdbem_status gmres_layout(tdbem_handle* h, int G, int C, cudaStream_t s)
{
    const int64_t E = h->E;
    const int R = h->R;
    const int nl = (int)h->leaf_begin.size();
    C = std::max(1, std::min(C, nl));
    h->groups = G;
    std::vector<int32_t> cta(C + 1, nl);
    {
        int L = 0;
        for (int c = 0; c < C; ++c) {
            cta[c] = L;
            const int64_t target = (E * (c + 1)) / C;
            while (L < nl && (h->leaf_begin[L] + h->leaf_count[L] <= target || L == cta[c])) ++L;
            if (nl - L < C - c - 1) L = nl - (C - c - 1);
        }
        cta[0] = 0;
        cta[C] = nl;
    }
    h->cluster = C;
    CUDA_TRY(up(h->d_cta_leaf, cta, s));
    {
        std::vector<int32_t> owner((size_t)E, 0), local((size_t)E, 0);
        int rows_max = 0;
        for (int c = 0; c < C; ++c) {
            if (cta[c] >= cta[c + 1]) continue;
            const int lo = (int)h->leaf_begin[cta[c]];
            const int hi = (int)(h->leaf_begin[cta[c + 1] - 1] + h->leaf_count[cta[c + 1] - 1]);
            rows_max = std::max(rows_max, hi - lo);
            for (int p = lo; p < hi; ++p) {
                owner[p] = c;
                local[p] = p - lo;
            }
        }
        std::vector<int32_t> colx(h->ap_col.size());
        for (size_t j = 0; j < h->ap_col.size(); ++j) colx[j] = (owner[h->ap_col[j]] << 24) | local[h->ap_col[j]];
        CUDA_TRY(up(h->d_a_colx, colx, s));
        h->dsm_rows = gmres_dsm_bytes(rows_max, R / G, h->precision == TDBEM_PRECISION_MIXED) <= kGmresDsmMax
                          ? rows_max
                          : 0;
        if (const char* off = std::getenv("TDBEM_GMRES_DSM"))
            if (std::atoi(off) == 0) h->dsm_rows = 0;  // tuning override: vectors from global memory
    }
    CUDA_TRY(h->d_givens.alloc(sizeof(double) * (size_t)C * R * kGivensArrays * (h->restart + 2)));
    return TDBEM_OK;
}

tdbem_status finish_setup(tdbem_handle* h, cudaStream_t s)
{
    const int64_t E = h->E;
    std::vector<int32_t> row_of(E), unk_of(E), perm_of_unk(E);
    for (int64_t p = 0; p < E; ++p) {
        row_of[p] = (int32_t)h->repid[p];
        unk_of[p] = (int32_t)h->pref[h->repid[p]];
        perm_of_unk[unk_of[p]] = (int32_t)p;
    }
    std::vector<int32_t> arp(E + 1, 0), acol;
    std::vector<double> aval;
    for (int64_t p = 0; p < E; ++p) {
        const int r = row_of[p];
        for (int j = h->a_rp[r]; j < h->a_rp[r + 1]; ++j) {
            acol.push_back(perm_of_unk[h->a_col[j]]);
            aval.insert(aval.end(), &h->a_val[9 * (int64_t)j], &h->a_val[9 * (int64_t)j] + 9);
        }
        arp[p + 1] = (int32_t)acol.size();
    }
    CUDA_TRY(up(h->d_a_rp, arp, s));
    CUDA_TRY(up(h->d_a_col, acol, s));
    h->ap_col = acol;
    CUDA_TRY(up(h->d_a_val, aval, s));
    CUDA_TRY(up(h->d_row_of, row_of, s));
    CUDA_TRY(up(h->d_unk_of, unk_of, s));
    CUDA_TRY(up(h->d_perm_of_unk, perm_of_unk, s));
    const int nl = (int)h->leaf_begin.size();
    std::vector<int32_t> lb(nl), lc(nl);
    std::vector<int64_t> loff(nl + 1, 0);
    int maxn = 0;
    for (int l = 0; l < nl; ++l) {
        lb[l] = (int32_t)h->leaf_begin[l];
        lc[l] = (int32_t)h->leaf_count[l];
        loff[l + 1] = loff[l] + 9LL * lc[l] * lc[l];
        maxn = std::max(maxn, 3 * lc[l]);
    }
    CUDA_TRY(up(h->d_leaf_begin, lb, s));
    CUDA_TRY(up(h->d_leaf_count, lc, s));
    std::vector<int32_t> lop(E, 0);
    for (int l = 0; l < nl; ++l)
        for (int q = 0; q < lc[l]; ++q) lop[lb[l] + q] = l;
    CUDA_TRY(up(h->d_leaf_of_perm, lop, s));
    CUDA_TRY(up(h->d_leaf_off, loff, s));
    CUDA_TRY(h->d_pinv.alloc(sizeof(double) * std::max<int64_t>(loff[nl], 1)));
    DevBuf sing;
    CUDA_TRY(sing.alloc(sizeof(int)));
    CUDA_TRY(cudaMemsetAsync(sing.p, 0, sizeof(int), s));
    const size_t smem = sizeof(double) * (size_t)maxn * maxn + sizeof(int) * 2 * (maxn + 2);
    if (smem > 48 * 1024)
        CUDA_TRY(cudaFuncSetAttribute(leaf_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    leaf_inverse_kernel<<<nl, 256, smem, s>>>(nl, h->d_leaf_begin.as<int32_t>(), h->d_leaf_count.as<int32_t>(),
                                             h->d_leaf_off.as<int64_t>(), h->d_a_rp.as<int32_t>(),
                                             h->d_a_col.as<int32_t>(), h->d_a_val.as<double>(),
                                             h->d_pinv.as<double>(), sing.as<int>());
    CUDA_TRY(cudaGetLastError());
    int singular = 0;
    CUDA_TRY(cudaMemcpyAsync(&singular, sing.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (singular)
        return fail(TDBEM_SINGULAR_BLOCK, "preconditioner leaf " + std::to_string(singular - 1) +
                                              " has a pivot <= 1e-10");
    if (h->precision == TDBEM_PRECISION_MIXED) {
        CUDA_TRY(h->d_pinv32.alloc(sizeof(float) * std::max<int64_t>(loff[nl], 1)));
        to_float_kernel<<<148, 256, 0, s>>>(h->d_pinv.as<double>(), h->d_pinv32.as<float>(), loff[nl]);
        CUDA_TRY(h->d_a_val32.alloc(sizeof(float) * std::max<size_t>(aval.size(), 1)));
        to_float_kernel<<<148, 256, 0, s>>>(h->d_a_val.as<double>(), h->d_a_val32.as<float>(), (int64_t)aval.size());
        CUDA_TRY(cudaGetLastError());
    }
    // GMRES: `groups` clusters of C CTAs, each solving R / groups load cases;
    // within a cluster every CTA owns contiguous leaf ranges of about equal
    // point count.  Most groups whose clusters fit on half the SMs when the
    // bulk history pass (k >= 3) runs beside GMRES and needs the other half
    // (measured on the 3072-element bar with 32 loads: 4 clusters of 16
    // 9% faster per step than 8), on all of them otherwise.
    const int R = h->R;
    int sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    const bool mixed = h->precision == TDBEM_PRECISION_MIXED;
    // batched small models: clusters of at most E / 24 rows' worth of CTAs
    // (a power of two), and every SM for GMRES when the history is short
    // (the bulk pass beside it has little to do); measured on the
    // 120-element rod with 32 loads, where the autotuner found 32 clusters of
    // 4 CTAs 18% faster than 4 of 16.  The 3072-element bar (K = 39) and
    // single-load handles keep the layout below.
    const bool small = R >= 2 && (E < 24 * 16 || h->K < 16);
    int c_rows = 1;
    while (c_rows * 2 <= std::max<int64_t>(1, E / 24)) c_rows *= 2;
    const int gmres_sms = h->K >= 3 && !(R >= 2 && h->K < 16) ? sms / 2 : sms;
    int G = 1, C = gmres_cluster_size(h->device, R, mixed);
    for (int g = R; g >= 1; g /= 2) {
        if (R % g) continue;
        int c = gmres_cluster_size(h->device, R / g, mixed);
        if (small) c = std::min(c, c_rows);
        if (g * c <= gmres_sms) {
            G = g;
            C = c;
            break;
        }
    }
    if (const char* force = std::getenv("TDBEM_GMRES_GROUPS")) {
        const int f = std::atoi(force);
        if (f >= 1 && R % f == 0 && (f & (f - 1)) == 0) {
            G = f;
            C = gmres_cluster_size(h->device, R / G, mixed);
        }
    }
    if (const char* force = std::getenv("TDBEM_GMRES_CLUSTER")) {
        const int f = std::atoi(force);
        if (f >= 1 && f <= C) C = f;  // tuning override, never above the schedulable size
    }
    if (tdbem_status st = gmres_layout(h, G, C, s); st != TDBEM_OK) return st;
    const int rs = h->restart;
    const size_t vec = sizeof(double) * 3 * (size_t)E * R;
    CUDA_TRY(h->d_V.alloc(vec * (rs + 1)));
    CUDA_TRY(h->d_W.alloc(vec * (rs + 1)));
    CUDA_TRY(h->d_AW.alloc(vec * (rs + 1)));
    CUDA_TRY(h->d_b.alloc(vec));
    CUDA_TRY(h->d_bp.alloc(vec));
    CUDA_TRY(h->d_x.alloc(vec));
    if (h->precision == TDBEM_PRECISION_MIXED) CUDA_TRY(h->d_xold.alloc(vec));
    CUDA_TRY(h->d_rv.alloc(vec));
    CUDA_TRY(h->d_u.alloc(vec));
    CUDA_TRY(h->d_bulk.alloc(8 * vec));
    CUDA_TRY(h->d_status.alloc(sizeof(int) * 4));
    const int SW = h->K + 1;
    const int64_t nhm = std::max<int64_t>(h->n_hist, 1);
    CUDA_TRY(h->d_xring.alloc(sizeof(double) * 3 * 2 * nhm * 3 * R));
    CUDA_TRY(h->d_wring.alloc(sizeof(double) * SW * 2 * nhm * 3 * R));
    // known KnownM upload, with each block's known element and sign
    CUDA_TRY(up(h->d_k_rp, h->k_rp, s));
    CUDA_TRY(up(h->d_k_col, h->k_col, s));
    CUDA_TRY(up(h->d_k_val, h->k_val, s));
    {
        std::vector<int32_t> ke(h->k_col.size());
        std::vector<double> ks(h->k_col.size());
        for (size_t j = 0; j < h->k_col.size(); ++j) {
            ke[j] = h->known_elem[h->k_col[j]];
            ks[j] = h->known_sign[h->k_col[j]];
        }
        CUDA_TRY(up(h->d_k_elem, ke, s));
        CUDA_TRY(up(h->d_k_sgn, ks, s));
    }
    CUDA_TRY(cudaStreamSynchronize(s));
    h->assembled = true;
    return TDBEM_OK;
}

// Append to a diagnostic CSV, writing the header when the file is new
// (OpenDiagnosticCsv, DBEM1/multidomain.cpp:130-144).
FILE* open_diagnostic_csv(const std::string& path, const char* header)
{
    FILE* t = std::fopen(path.c_str(), "r");
    const bool fresh = t == nullptr;
    if (t) std::fclose(t);
    FILE* f = std::fopen(path.c_str(), "a");
    if (f && fresh) std::fprintf(f, "%s\n", header);
    return f;
}

// Pair space over the domains, the GlobalDofMap references and the
// per-field-element column maps of the Step0 and history blocks (device
// copies), shared by the assembly and the material gradient.
struct PairSetup {
    std::vector<int64_t> poff;
    DevBuf dom_begin, dom_count, pair_off, col_a0, col_a1, col_k, col_h;
    PairSpace ps{};
    DofRefs dr{};
};

tdbem_status pair_setup(tdbem_handle* h, PairSetup& P, cudaStream_t s)
{
    const int64_t E = h->E;
    P.poff.assign(h->D + 1, 0);
    for (int d = 0; d < h->D; ++d) P.poff[d + 1] = P.poff[d] + (int64_t)h->dom_count[d] * h->dom_count[d];
    CUDA_TRY(up(P.dom_begin, h->dom_begin, s));
    CUDA_TRY(up(P.dom_count, h->dom_count, s));
    CUDA_TRY(up(P.pair_off, P.poff, s));
    P.ps = PairSpace{h->D, P.poff[h->D], P.dom_begin.as<int32_t>(), P.dom_count.as<int32_t>(),
                     P.pair_off.as<int64_t>()};
    P.dr = DofRefs{h->d_uref_sign.as<double>(), h->d_tref_sign.as<double>(), h->d_hu_sign.as<double>(),
                   h->d_ht_sign.as<double>(), h->d_itf_trans.as<double>()};
    // A slot 0: the interface element's U unknown or the outer element's
    // unknown; A slot 1: the interface T unknown; KnownM: the known block
    std::vector<int64_t> a0(E), a1(E), kc(E), hc(E);
    for (int64_t i = 0; i < E; ++i) {
        a0[i] = h->surface[i] ? h->uref_block[i] : (h->bcid[i] == 123 ? h->tref_block[i] : h->uref_block[i]);
        a1[i] = h->tref_block[i];
        kc[i] = h->bcid[i] == 123 ? h->uref_block[i] : h->tref_block[i];
        hc[i] = h->hist_block[i];
    }
    CUDA_TRY(up(P.col_a0, a0, s));
    CUDA_TRY(up(P.col_a1, a1, s));
    CUDA_TRY(up(P.col_k, kc, s));
    CUDA_TRY(up(P.col_h, hc, s));
    return TDBEM_OK;
}

// One march of one handle, split so that several handles' marches can be
// interleaved step by step (tdbem_md_march_many): begin enqueues the set-up,
// step enqueues one time step, end enqueues the join with the caller's
// stream, finish waits and builds the report.
struct MarchRun {
    tdbem_handle* h = nullptr;
    MarchData d{};
    std::vector<cudaEvent_t> ev;
    bool overlap = false;
    // TDBEM_OVERLAP=0: the history part k >= 3 runs on the chain stream
    // after each step's GMRES instead of beside it (same results; its
    // events then time the history kernel alone, for measurement)
    bool serial_history = false;
    bool grouped = false;             // stepped by the several-models launches (no per-phase times)
    cudaStream_t us = nullptr, s = nullptr;
    int N = 0, R = 1;
    int64_t E = 0;

    MarchRun() = default;
    MarchRun(const MarchRun&) = delete;
    MarchRun& operator=(const MarchRun&) = delete;
    cudaEvent_t E7(int step, int j) const { return ev[3 + 7 * (size_t)(step - 1) + j]; }

    tdbem_status begin(tdbem_handle* hh, const double* d_known_lu, double* d_out_lu, double* d_out_lt, void* stream)
    {
        h = hh;
        if (!h || !d_known_lu || !d_out_lu || !d_out_lt) return fail(TDBEM_INVALID_INPUT, "null argument");
        if (!h->assembled) return fail(TDBEM_NOT_ASSEMBLED, "call tdbem_md_assemble or tdbem_md_load_matrices first");
        CUDA_TRY(cudaSetDevice(h->device));
        us = stream ? (cudaStream_t)stream : h->s0;
        s = h->hp;
        E = h->E;
        N = h->nstep;
        R = h->R;
        h->saved_forward = false;
        h->diag_ready = false;
        CUDA_TRY(h->d_flags.alloc(sizeof(int) * 3 * std::max(N, 1) * R));
        CUDA_TRY(h->d_audit.alloc(sizeof(double) * 2 * std::max(N, 1)));
        if (h->record) {
            CUDA_TRY(h->d_rec_rhs.alloc(sizeof(double) * 3 * E * std::max(N, 1)));
            CUDA_TRY(h->d_rec_x.alloc(sizeof(double) * 3 * E * std::max(N, 1)));
        } else {
            h->d_rec_rhs.release();
            h->d_rec_x.release();
        }
        d.E = (int)E;
        d.n_known = (int)h->n_known;
        d.nh = (int)h->n_hist;
        d.K = h->K;
        d.R = R;
        d.nstep = N;
        d.SW = h->K + 1;
        d.mixed = h->precision == TDBEM_PRECISION_MIXED;
        d.h_kptr = h->d_h_kptr.as<int64_t>();
        d.h_col = h->d_h_col.as<uint32_t>();
        d.h_val = h->d_h_val.as<double>();
        d.h_val32 = h->d_h_val32.as<float>();
        d.h_nnz = h->h_nnz;
        d.r_ptr = h->d_r_ptr.as<int64_t>();
        d.r_meta = h->d_r_meta.as<uint2>();
        d.r_off = h->d_r_off.as<int64_t>();
        d.r_val = h->d_r_val.as<double>();
        d.r_val32 = h->d_r_val.as<float>();
        d.r_nb = h->r_nb;
        d.kr = h->run_k;
        d.k_rp = h->d_k_rp.as<int32_t>();
        d.k_col = h->d_k_col.as<int32_t>();
        d.k_val = h->d_k_val.as<double>();
        d.k_elem = h->d_k_elem.as<int32_t>();
        d.k_sgn = h->d_k_sgn.as<double>();
        d.known_elem = h->d_known_elem.as<int32_t>();
        d.known_sign = h->d_known_sign.as<double>();
        d.a_rp = h->d_a_rp.as<int32_t>();
        d.a_col = h->d_a_col.as<int32_t>();
        d.a_val = h->d_a_val.as<double>();
        d.a_val32 = h->d_a_val32.as<float>();
        d.row_of = h->d_row_of.as<int32_t>();
        d.perm_of_unk = h->d_perm_of_unk.as<int32_t>();
        d.leaf_begin = h->d_leaf_begin.as<int32_t>();
        d.leaf_count = h->d_leaf_count.as<int32_t>();
        d.leaf_of_perm = h->d_leaf_of_perm.as<int32_t>();
        d.leaf_off = h->d_leaf_off.as<int64_t>();
        d.pinv = h->d_pinv.as<double>();
        d.pinv32 = h->d_pinv32.as<float>();
        d.cta_leaf = h->d_cta_leaf.as<int32_t>();
        d.a_colx = h->d_a_colx.as<int32_t>();
        d.dsm_rows = h->dsm_rows;
        d.uref_block = h->d_uref_block.as<int64_t>();
        d.uref_sign = h->d_uref_sign.as<double>();
        d.uref_known = h->d_uref_known.as<int32_t>();
        d.tref_block = h->d_tref_block.as<int64_t>();
        d.tref_sign = h->d_tref_sign.as<double>();
        d.tref_known = h->d_tref_known.as<int32_t>();
        d.hist_block = h->d_hist_block.as<int64_t>();
        d.hu_sign = h->d_hu_sign.as<double>();
        d.ht_sign = h->d_ht_sign.as<double>();
        d.hist_owner = h->d_hist_owner.as<int32_t>();
        d.itf_trans = h->d_itf_trans.as<double>();
        d.trans = h->g_trans.as<double>();
        d.bcid = h->g_bcid.as<int32_t>();
        d.itf_pairs = h->d_itf_pairs.as<int32_t>();
        d.itf_sign = h->d_itf_sign.as<double>();
        d.n_itf = (int)h->I;
        d.xring = h->d_xring.as<double>();
        d.wring = h->d_wring.as<double>();
        d.bulk = h->d_bulk.as<double>();
        d.b = h->d_b.as<double>();
        d.groups = h->groups;
        d.bp = h->d_bp.as<double>();
        d.x = h->d_x.as<double>();
        d.xold = h->d_xold.as<double>();
        d.rv = h->d_rv.as<double>();
        d.u = h->d_u.as<double>();
        d.V = h->d_V.as<double>();
        d.W = h->d_W.as<double>();
        d.AW = h->d_AW.as<double>();
        d.givens = h->d_givens.as<double>();
        d.status = h->d_status.as<int>();
        d.step_flags = h->d_flags.as<int>();
        d.audit = h->d_audit.as<double>();
        d.known_lu = d_known_lu;
        d.out_lu = d_out_lu;
        d.out_lt = d_out_lt;
        d.rec_rhs = h->record ? h->d_rec_rhs.as<double>() : nullptr;
        d.rec_x = h->record ? h->d_rec_x.as<double>() : nullptr;
        d.restart = h->restart;
        d.tol = h->tol;
        d.cluster = h->cluster;
        d.rhs_cpt = h->rhs_cpt;
        d.givens_stride = (int64_t)kGivensArrays * (h->restart + 2);

        overlap = h->K >= 3;
        if (const char* v = std::getenv("TDBEM_OVERLAP")) serial_history = std::atoi(v) == 0;
        // the chain runs on the handle's high-priority stream, ordered after
        // the caller's stream and followed by it
        const int NS = std::max(N, 1);
        CUDA_TRY(h->ev_timed.take(7 * (size_t)NS + 3, ev));
        CUDA_TRY(cudaEventRecord(ev[0], us));
        CUDA_TRY(cudaStreamWaitEvent(s, ev[0], 0));
        CUDA_TRY(cudaStreamWaitEvent(h->side, ev[0], 0));
        CUDA_TRY(cudaEventRecord(ev[1], s));
        CUDA_TRY(cudaMemsetAsync(d_out_lu, 0, sizeof(double) * R * (N + 1) * E * 3, s));
        CUDA_TRY(cudaMemsetAsync(d_out_lt, 0, sizeof(double) * R * (N + 1) * E * 3, s));
        CUDA_TRY(cudaMemsetAsync(h->d_flags.p, 0, h->d_flags.bytes, s));
        CUDA_TRY(march_prepare(d, s));
        return TDBEM_OK;
    }

    tdbem_status step(int k)
    {
        CUDA_TRY(cudaSetDevice(h->device));
        const int T = h->run_k >= 5 ? (h->run_k - 1) / 2 : 2;  // steps per history pass
        StepEvents se{E7(k, 0), E7(k, 1), E7(k, 2), E7(k, 3), E7(k, 4), E7(k, 5), E7(k, 6),
                      k == 1 ? ev[1] : E7(k - 1, 3), k > T ? E7(k - T, 6) : nullptr};
        CUDA_TRY(march_step(d, k, s, serial_history ? s : h->side, se, overlap));
        return TDBEM_OK;
    }

    tdbem_status end()
    {
        CUDA_TRY(cudaSetDevice(h->device));
        CUDA_TRY(cudaEventRecord(ev[2], s));
        CUDA_TRY(cudaStreamWaitEvent(us, ev[2], 0));
        return TDBEM_OK;
    }

    tdbem_status finish(tdbem_report* report)
    {
        CUDA_TRY(cudaSetDevice(h->device));
        CUDA_TRY(cudaEventSynchronize(ev[2]));
        std::vector<int> flags(3 * std::max(N, 1) * R, 0);
        CUDA_TRY(cudaMemcpy(flags.data(), h->d_flags.p, sizeof(int) * flags.size(), cudaMemcpyDeviceToHost));
        std::vector<double> audit(2 * std::max(N, 1), 0.0);
        CUDA_TRY(cudaMemcpy(audit.data(), h->d_audit.p, sizeof(double) * audit.size(), cudaMemcpyDeviceToHost));
        tdbem_report rep{};
        float ms = 0.0f;
        double ms_rhs = 0.0, ms_gm = 0.0, ms_hist = 0.0;
        for (int step = 1; step <= N && !grouped; ++step) {
            float a = 0.0f, b = 0.0f, c = 0.0f;
            cudaEventElapsedTime(&a, E7(step, 0), E7(step, 1));
            cudaEventElapsedTime(&b, E7(step, 2), E7(step, 3));
            if (overlap && step < N) cudaEventElapsedTime(&c, E7(step, 4), E7(step, 5));
            ms_rhs += a + c;
            ms_gm += b;
            ms_hist += c;
        }

        cudaEventElapsedTime(&ms, ev[1], ev[2]);
        rep.ms_total = ms;
        rep.gmres_cluster = h->cluster;
        rep.gmres_groups = h->groups;
        rep.ms_rhs = ms_rhs;
        rep.ms_gmres = ms_gm;
        rep.ms_history = ms_hist;
        rep.history_steps = h->K;
        rep.history_blocks = h->h_nnz;
        rep.a_blocks = h->a_rp.empty() ? 0 : h->a_rp[h->E];
        // algorithmic bytes of the right-hand side: each launch reads every
        // block it applies once (9 values, FP32 in mixed mode, plus the packed
        // column of the step-major passes; the run headers of the T-step
        // pass) and every distinct combined history vector it meets once (3 x R
        // FP64 per history column and type); the head pass also reads KnownM
        // and the known values and writes the right-hand side, a history pass
        // writes its steps' parts
        double bytes = 0.0;
        {
            const int K = h->K, kr = h->run_k;
            const bool pair = overlap && !grouped && kr >= 5;
            const int T = pair ? (kr - 1) / 2 : 1;  // steps per history pass
            std::vector<int64_t> cum(K + 1, 0);
            for (int64_t r = 0; r < E; ++r)
                for (int k = 0; k <= K; ++k) cum[k] += h->h_kptr[r * (K + 1) + k] - h->h_kptr[r * (K + 1)];
            const double vs = h->precision == TDBEM_PRECISION_MIXED ? 4.0 : 8.0;
            const double knz = h->k_rp.empty() ? 0.0 : (double)h->k_rp[E];
            const double slot_b = 2.0 * h->n_hist * 3.0 * 8.0 * R;
            // KnownM . known_s: blocks (9 values, known element and sign) and
            // the known values; computed by the pass that covers the step
            const double known_b = knz * (72.0 + 4.0 + 8.0) + (double)h->n_known * 24.0 * R;
            const double head_fixed = (double)E * (24.0 * R + 16.0 + 4.0);
            for (int step = 1; step <= N; ++step) {
                const int kc = step > 1 ? std::min(step, K) : 0;
                rep.rhs_block_reads += (double)cum[kc];
                const int kh = !overlap ? kc : std::min(kc, pair ? kr - 1 : 2);
                const bool covered = overlap && step >= (pair ? 2 + T : 3);
                bytes += (double)cum[kh] * (9.0 * vs + 4.0) + (double)kh * slot_b + head_fixed +
                         (covered ? 0.0 : known_b);
                if (!overlap) continue;
                double hb = 0.0;
                if (pair) {
                    const int t0 = step + T, klast = std::min(t0 + T - 1, K);
                    if (step >= 2 && (step - 2) % T == 0 && t0 <= N) {
                        // distinct W slots: t0 + h - k over the launch's (h, k)
                        const int slots = (t0 + T - 1 - kr) - std::max(t0 - klast, 0) + 1;
                        const int steps_out = std::min(T, N - t0 + 1);
                        hb = (double)(cum[klast] - cum[kr - 1]) * 9.0 * vs + (double)h->r_runs * 16.0 +
                             std::max(slots, 0) * slot_b + (double)E * 24.0 * R * steps_out + steps_out * known_b;
                        for (int hh = 0; hh < T; ++hh)
                            rep.history_block_steps +=
                                (double)std::max<int64_t>(cum[std::min(t0 + hh, K)] - cum[kr - 1], 0);
                        rep.history_vector_loads +=
                            (double)(cum[std::min(t0, K)] > cum[kr - 1] ? cum[std::min(t0, K)] - cum[kr - 1] : 0) +
                            (double)(T - 1) * h->r_runs;
                        ++rep.history_launches;
                    }
                } else if (step + 1 <= N) {
                    const int kc1 = std::min(step + 1, K);
                    if (kc1 >= 3) {
                        hb = (double)(cum[kc1] - cum[2]) * (9.0 * vs + 4.0) + (kc1 - 2) * slot_b +
                             (double)E * 24.0 * R + known_b;
                        rep.history_block_steps += (double)(cum[kc1] - cum[2]);
                        rep.history_vector_loads += (double)(cum[kc1] - cum[2]);
                        ++rep.history_launches;
                    }
                }
                rep.history_bytes += hb;
                bytes += hb;
            }
        }
        rep.rhs_bytes = bytes;
        tdbem_status result = TDBEM_OK;
        for (int step = 1; step <= N; ++step) {
            for (int r = 0; r < R; ++r) {
                const int* f = &flags[3 * ((size_t)(step - 1) * R + r)];
                rep.total_inner += f[2];
                rep.max_refinements = std::max(rep.max_refinements, f[1]);
                if (f[0] != 0 && result == TDBEM_OK) {
                    rep.failed_step = step;
                    rep.gmres_flag = f[0];
                    result = TDBEM_NOT_CONVERGED;
                }
            }
            if (result != TDBEM_OK) break;
            rep.steps_solved = step;
            rep.max_interface_jump = std::max(rep.max_interface_jump, audit[2 * (step - 1)]);
            rep.max_interface_balance = std::max(rep.max_interface_balance, audit[2 * (step - 1) + 1]);
        }
        if (report) *report = rep;
        if (result != TDBEM_OK)
            g_error = "GMRES flag " + std::to_string(rep.gmres_flag) + " at step " + std::to_string(rep.failed_step);
        return result;
    }
};

}  // namespace

extern "C" {

tdbem_status tdbem_md_assemble(tdbem_handle* h, void* stream)
{
    g_error.clear();
    if (!h) return fail(TDBEM_INVALID_INPUT, "null handle");
    const auto t_start = std::chrono::steady_clock::now();
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : h->s0;
    const int E = (int)h->E;
    PairSetup P;
    if (tdbem_status st = pair_setup(h, P, s); st != TDBEM_OK) return st;
    const PairSpace ps = P.ps;
    const DofRefs dr = P.dr;
    DevBuf blocks, flags;
    CUDA_TRY(blocks.alloc(sizeof(double) * 18 * ps.n_pairs));
    CUDA_TRY(flags.alloc(ps.n_pairs));
    ElemGeom g = h->geom();
    const int warps_per_cta = 4;
    step0_kernel<<<ceil_div(ps.n_pairs, warps_per_cta), 32 * warps_per_cta, 0, s>>>(
        ps, h->d_rules.as<QuadRules>(), g, dr, blocks.as<double>(), flags.as<uint8_t>());
    CUDA_TRY(cudaGetLastError());
    {
        ScatterCols sa{{0, 1, 1}, {P.col_a0.as<int64_t>(), P.col_a1.as<int64_t>(), P.col_k.as<int64_t>()}};
        std::vector<int64_t> rp;
        DevBuf drp, col, val;
        tdbem_status st = compact(h, ps, flags, blocks, 3, sa, rp, drp, col, val, s);
        if (st != TDBEM_OK) return st;
        // host copy in the reference's (row, col) order
        std::vector<int32_t> c;
        std::vector<double> v;
        CUDA_TRY(download(c, col, rp[E], s));
        CUDA_TRY(download(v, val, 9 * rp[E], s));
        h->a_rp.assign(E + 1, 0);
        h->a_col.clear();
        h->a_val.clear();
        for (int r = 0; r < E; ++r) {
            std::vector<int64_t> idx(rp[r + 1] - rp[r]);
            std::iota(idx.begin(), idx.end(), rp[r]);
            std::sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return c[a] < c[b]; });
            for (int64_t j : idx) {
                h->a_col.push_back(c[j]);
                h->a_val.insert(h->a_val.end(), &v[9 * j], &v[9 * j] + 9);
            }
            h->a_rp[r + 1] = (int32_t)h->a_col.size();
        }
        std::vector<int64_t> rpk;
        DevBuf drpk, colk, valk;
        st = compact(h, ps, flags, blocks, 4, sa, rpk, drpk, colk, valk, s);
        if (st != TDBEM_OK) return st;
        CUDA_TRY(download(c, colk, rpk[E], s));
        CUDA_TRY(download(v, valk, 9 * rpk[E], s));
        h->k_rp.assign(E + 1, 0);
        h->k_col.clear();
        h->k_val.clear();
        for (int r = 0; r < E; ++r) {
            std::vector<int64_t> idx(rpk[r + 1] - rpk[r]);
            std::iota(idx.begin(), idx.end(), rpk[r]);
            std::sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return c[a] < c[b]; });
            for (int64_t j : idx) {
                h->k_col.push_back(c[j]);
                h->k_val.insert(h->k_val.end(), &v[9 * j], &v[9 * j] + 9);
            }
            h->k_rp[r + 1] = (int32_t)h->k_col.size();
        }
    }
    // history steps: MaxN (DBEM1/multidomain.cpp:3718-3740), and no further
    // than the last step any block can be nonzero (history_step_bound)
    int maxn = h->nstep;
    double minc2dt = 1.0e308;
    for (const DynaMat& m : h->mats)
        if (m.C2Dt > 0.0 && m.C2Dt < minc2dt) minc2dt = m.C2Dt;
    for (int i = 0; i <= h->nstep; ++i)
        if (minc2dt * i > h->max_length) {
            maxn = i;
            break;
        }
    {
        int kb = 0;
        if (tdbem_status st = history_step_bound(h, s, kb); st != TDBEM_OK) return st;
        maxn = std::min(maxn, kb);
    }
    std::vector<std::unique_ptr<DevBuf>> keep;
    std::vector<std::vector<int64_t>> mts_rp, mgs_rp;
    std::vector<HistK> hk;
    int last = 0;
    for (int k = 1; k <= maxn; ++k) {
        history_kernel<<<ceil_div(ps.n_pairs, warps_per_cta), 32 * warps_per_cta, 0, s>>>(
            ps, h->d_rules.as<QuadRules>(), g, dr, k, blocks.as<double>(), flags.as<uint8_t>());
        CUDA_TRY(cudaGetLastError());
        ScatterCols sh{{0, 1, 1}, {P.col_h.as<int64_t>(), P.col_h.as<int64_t>(), P.col_h.as<int64_t>()}};
        std::vector<int64_t> rt, rg;
        auto trp = std::make_unique<DevBuf>(), tcol = std::make_unique<DevBuf>(), tval = std::make_unique<DevBuf>();
        auto grp = std::make_unique<DevBuf>(), gcol = std::make_unique<DevBuf>(), gval = std::make_unique<DevBuf>();
        tdbem_status st = compact(h, ps, flags, blocks, 1, sh, rt, *trp, *tcol, *tval, s);
        if (st != TDBEM_OK) return st;
        st = compact(h, ps, flags, blocks, 2, sh, rg, *grp, *gcol, *gval, s);
        if (st != TDBEM_OK) return st;
        const bool empty = rt[E] == 0 && rg[E] == 0;
        if (!empty) last = k;
        mts_rp.push_back(rt);
        mgs_rp.push_back(rg);
        hk.push_back(HistK{trp->as<int64_t>(), tcol->as<int32_t>(), tval->as<double>(), grp->as<int64_t>(),
                           gcol->as<int32_t>(), gval->as<double>()});
        keep.push_back(std::move(trp));
        keep.push_back(std::move(tcol));
        keep.push_back(std::move(tval));
        keep.push_back(std::move(grp));
        keep.push_back(std::move(gcol));
        keep.push_back(std::move(gval));
    }
    h->K = last;
    mts_rp.resize(last);
    mgs_rp.resize(last);
    hk.resize(last);
    blocks.release();
    flags.release();
    tdbem_status st = stack_history(h, mts_rp, mgs_rp, hk, s);
    if (st != TDBEM_OK) return st;
    keep.clear();  // the per-step matrices, before the run layout takes its memory
    if ((st = build_runs(h, s)) != TDBEM_OK) return st;
    const tdbem_status done = finish_setup(h, s);
    h->assembly_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    return done;
}

tdbem_status tdbem_md_load_matrices(tdbem_handle* h, const int32_t* a_rowptr, const int32_t* a_col,
                                    const double* a_val, const int32_t* k_rowptr, const int32_t* k_col,
                                    const double* k_val, int32_t n_hist, const int32_t* mts_rowptr,
                                    const int32_t* mts_col, const double* mts_val, const int32_t* mgs_rowptr,
                                    const int32_t* mgs_col, const double* mgs_val, void* stream)
{
    const auto t_start = std::chrono::steady_clock::now();
    g_error.clear();
    if (!h || !a_rowptr || !k_rowptr || n_hist < 0) return fail(TDBEM_INVALID_INPUT, "null argument");
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : h->s0;
    const int E = (int)h->E;
    h->a_rp.assign(a_rowptr, a_rowptr + E + 1);
    h->a_col.assign(a_col, a_col + h->a_rp[E]);
    h->a_val.assign(a_val, a_val + 9 * (int64_t)h->a_rp[E]);
    h->k_rp.assign(k_rowptr, k_rowptr + E + 1);
    h->k_col.assign(k_col, k_col + h->k_rp[E]);
    h->k_val.assign(k_val, k_val + 9 * (int64_t)h->k_rp[E]);
    for (int64_t j = 0; j < h->a_rp[E]; ++j)
        if (h->a_col[j] < 0 || h->a_col[j] >= h->n_unknown) return fail(TDBEM_INVALID_INPUT, "A column out of range");
    for (int64_t j = 0; j < h->k_rp[E]; ++j)
        if (h->k_col[j] < 0 || h->k_col[j] >= h->n_known) return fail(TDBEM_INVALID_INPUT, "KnownM column out of range");
    h->K = n_hist;
    std::vector<std::vector<int64_t>> mts_rp(n_hist), mgs_rp(n_hist);
    std::vector<HistK> hk(n_hist);
    std::vector<std::unique_ptr<DevBuf>> keep;
    int64_t ot = 0, og = 0;
    for (int k = 0; k < n_hist; ++k) {
        const int32_t* rt = mts_rowptr + (int64_t)k * (E + 1);
        const int32_t* rg = mgs_rowptr + (int64_t)k * (E + 1);
        mts_rp[k].assign(rt, rt + E + 1);
        mgs_rp[k].assign(rg, rg + E + 1);
        const int64_t nt = rt[E], ng = rg[E];
        for (int64_t j = 0; j < nt; ++j)
            if (mts_col[ot + j] < 0 || mts_col[ot + j] >= h->n_hist) return fail(TDBEM_INVALID_INPUT, "MTS column out of range");
        for (int64_t j = 0; j < ng; ++j)
            if (mgs_col[og + j] < 0 || mgs_col[og + j] >= h->n_hist) return fail(TDBEM_INVALID_INPUT, "MGS column out of range");
        std::vector<int32_t> ct(mts_col + ot, mts_col + ot + nt), cg(mgs_col + og, mgs_col + og + ng);
        std::vector<double> vt(mts_val + 9 * ot, mts_val + 9 * (ot + nt)), vg(mgs_val + 9 * og, mgs_val + 9 * (og + ng));
        for (int i = 0; i < 6; ++i) keep.push_back(std::make_unique<DevBuf>());
        const size_t base = keep.size() - 6;
        CUDA_TRY(up(*keep[base], mts_rp[k], s));
        CUDA_TRY(up(*keep[base + 1], ct, s));
        CUDA_TRY(up(*keep[base + 2], vt, s));
        CUDA_TRY(up(*keep[base + 3], mgs_rp[k], s));
        CUDA_TRY(up(*keep[base + 4], cg, s));
        CUDA_TRY(up(*keep[base + 5], vg, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        hk[k] = HistK{keep[base]->as<int64_t>(), keep[base + 1]->as<int32_t>(), keep[base + 2]->as<double>(),
                      keep[base + 3]->as<int64_t>(), keep[base + 4]->as<int32_t>(), keep[base + 5]->as<double>()};
        ot += nt;
        og += ng;
    }
    tdbem_status st = stack_history(h, mts_rp, mgs_rp, hk, s);
    if (st != TDBEM_OK) return st;
    keep.clear();  // the per-step matrices, before the run layout takes its memory
    if ((st = build_runs(h, s)) != TDBEM_OK) return st;
    const tdbem_status done = finish_setup(h, s);
    h->assembly_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    return done;
}

tdbem_status tdbem_md_set_record(tdbem_handle* h, int32_t on)
{
    if (!h) return fail(TDBEM_INVALID_INPUT, "null handle");
    h->record = on != 0;
    return TDBEM_OK;
}

tdbem_status tdbem_md_march_device(tdbem_handle* h, const double* d_known_lu, double* d_out_lu, double* d_out_lt,
                                   tdbem_report* report, void* stream)
{
    g_error.clear();
    MarchRun run;
    if (tdbem_status st = run.begin(h, d_known_lu, d_out_lu, d_out_lt, stream); st != TDBEM_OK) return st;
    for (int step = 1; step <= run.N; ++step)
        if (tdbem_status st = run.step(step); st != TDBEM_OK) return st;
    if (tdbem_status st = run.end(); st != TDBEM_OK) return st;
    return run.finish(report);
}

tdbem_status tdbem_md_march_many(tdbem_handle* const* handles, int32_t n, const double* const* d_known_lu,
                                 double* const* d_out_lu, double* const* d_out_lt, tdbem_report* reports, void* stream)
{
    g_error.clear();
    if (!handles || n <= 0 || !d_known_lu || !d_out_lu || !d_out_lt) return fail(TDBEM_INVALID_INPUT, "null argument");
    for (int i = 0; i < n; ++i) {
        if (!handles[i]) return fail(TDBEM_INVALID_INPUT, "null handle");
        for (int j = 0; j < i; ++j)
            if (handles[j] == handles[i]) return fail(TDBEM_INVALID_INPUT, "a handle appears twice");
    }
    // Default: each model's steps go to its own streams, interleaved step by
    // step.  With TDBEM_MARCH_MANY=grouped, models that share the device, the
    // load-case count (1, 2, 4 or 8) and the precision are marched grouped:
    // each time step of all models is two launches, every model's head
    // right-hand side and then one GMRES cluster per model, while one launch
    // on a side stream computes every model's history bulk (k >= 3) of the
    // next step, as a single march does.  The models are laid out for one
    // cluster size: the largest power of two that keeps all models' clusters
    // within half the SMs (the bulk pass takes the rest).  Grouped, every
    // step waits for the slowest model; on 16 rods of 480 to 3,630 elements
    // it measured 2,240 model-steps/s against 2,640 with streams (FP64).
    bool grouped = n >= 2;
    {
        const char* mode = std::getenv("TDBEM_MARCH_MANY");
        grouped = grouped && mode && std::strcmp(mode, "grouped") == 0;
    }
    for (int i = 0; i < n && grouped; ++i) {
        const tdbem_handle* hi = handles[i];
        grouped = hi->assembled && hi->device == handles[0]->device && hi->R == handles[0]->R &&
                  hi->precision == handles[0]->precision &&
                  (hi->R == 1 || hi->R == 2 || hi->R == 4 || hi->R == 8);
    }
    std::vector<std::pair<int, int>> layout((size_t)n);
    int gC = 1;
    if (grouped) {
        const tdbem_handle* h0 = handles[0];
        CUDA_TRY(cudaSetDevice(h0->device));
        int sms = 0;
        CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h0->device));
        const int cap = gmres_cluster_size(h0->device, h0->R, h0->precision == TDBEM_PRECISION_MIXED);
        int maxK = 0;
        for (int i = 0; i < n; ++i) maxK = std::max(maxK, handles[i]->K);
        // GMRES of all models on half the SMs when the history bulk pass runs
        // beside it, on all of them otherwise
        const int budget = maxK >= 3 ? sms / 2 : sms;
        int lim = std::max(1, std::min(cap, budget / n));
        for (int i = 0; i < n; ++i) lim = std::min(lim, (int)handles[i]->leaf_begin.size());
        while (gC * 2 <= lim) gC *= 2;
        for (int i = 0; i < n; ++i) {
            tdbem_handle* hi = handles[i];
            layout[i] = {hi->groups, hi->cluster};
            if (tdbem_status st = gmres_layout(hi, 1, gC, hi->s0); st != TDBEM_OK) return st;
            CUDA_TRY(cudaStreamSynchronize(hi->s0));
        }
    }
    auto restore_layouts = [&]() {
        if (!grouped) return;
        for (int i = 0; i < n; ++i) {
            gmres_layout(handles[i], layout[i].first, layout[i].second, handles[i]->s0);
            cudaStreamSynchronize(handles[i]->s0);
        }
    };
    std::vector<MarchRun> runs((size_t)n);
    int steps = 0;
    for (int i = 0; i < n; ++i) {
        if (tdbem_status st = runs[i].begin(handles[i], d_known_lu[i], d_out_lu[i], d_out_lt[i], stream); st != TDBEM_OK) {
            restore_layouts();
            return st;
        }
        steps = std::max(steps, runs[i].N);
    }
    if (grouped) {
        tdbem_handle* h0 = handles[0];
        cudaStream_t gs = h0->hp;
        std::vector<MarchData> ds((size_t)n);
        std::vector<int32_t> row_off((size_t)n + 1, 0);
        size_t dsm = 0;
        int max_K = 0;
        for (int i = 0; i < n; ++i) {
            ds[i] = runs[i].d;
            ds[i].k_lo = 1;
            ds[i].k_hi = 0;
            row_off[i + 1] = row_off[i] + runs[i].d.E;
            dsm = std::max(dsm, gmres_dsm_bytes(runs[i].d.dsm_rows, h0->R, h0->precision == TDBEM_PRECISION_MIXED));
            max_K = std::max(max_K, runs[i].d.K);
        }
        DevBuf d_ds, d_off;
        CUDA_TRY(d_ds.alloc(sizeof(MarchData) * (size_t)n));
        CUDA_TRY(cudaMemcpy(d_ds.p, ds.data(), sizeof(MarchData) * (size_t)n, cudaMemcpyHostToDevice));
        CUDA_TRY(up(d_off, row_off, gs));
        // the grouped launches follow every model's set-up; every model's
        // stream then follows them.  gm[s]: GMRES of step s done; bk[s]: bulk
        // of step s done
        cudaStream_t bs = h0->side;
        const bool overlap = max_K >= 3;
        std::vector<cudaEvent_t> ev;
        CUDA_TRY(h0->ev_order.take((size_t)n + 2 + 2 * ((size_t)steps + 2), ev));
        cudaEvent_t* gm = &ev[(size_t)n + 1];
        cudaEvent_t* bk = gm + (steps + 2);
        for (int i = 0; i < n; ++i) {
            CUDA_TRY(cudaEventRecord(ev[i], runs[i].s));
            CUDA_TRY(cudaStreamWaitEvent(gs, ev[i], 0));
            CUDA_TRY(cudaStreamWaitEvent(bs, ev[i], 0));
        }
        const bool mixed = h0->precision == TDBEM_PRECISION_MIXED;
        tdbem_status st = TDBEM_OK;
        auto launch = [&](int step, int phase, cudaStream_t on) {
            const cudaError_t e = march_models_step(d_ds.as<MarchData>(), d_off.as<int32_t>(), n, row_off[n], h0->R,
                                                    mixed, gC, dsm, max_K, step, phase, on);
            if (e != cudaSuccess && st == TDBEM_OK)
                st = fail(TDBEM_CUDA_ERROR, std::string("grouped march: ") + cudaGetErrorString(e));
        };
        for (int step = 1; step <= steps && st == TDBEM_OK; ++step) {
            if (overlap && step >= 3) CUDA_TRY(cudaStreamWaitEvent(gs, bk[step], 0));
            launch(step, overlap ? 1 : 0, gs);
            CUDA_TRY(cudaEventRecord(gm[step], gs));
            if (overlap && step + 1 <= steps && step + 1 >= 3) {
                // bulk of step + 1 needs the states up to step - 1
                CUDA_TRY(cudaStreamWaitEvent(bs, gm[step - 1], 0));
                launch(step + 1, 2, bs);
                CUDA_TRY(cudaEventRecord(bk[step + 1], bs));
            }
        }
        CUDA_TRY(cudaEventRecord(ev[n], bs));
        CUDA_TRY(cudaStreamWaitEvent(gs, ev[n], 0));
        CUDA_TRY(cudaEventRecord(ev.back(), gs));
        for (int i = 0; i < n; ++i) {
            CUDA_TRY(cudaStreamWaitEvent(runs[i].s, ev.back(), 0));
            runs[i].grouped = true;
        }
        CUDA_TRY(cudaEventSynchronize(ev.back()));
        if (st != TDBEM_OK) {
            restore_layouts();
            return st;
        }
    } else {
        // step by step across the models: each model's kernels go to its own
        // streams, so the models' time steps run side by side on the GPU
        for (int step = 1; step <= steps; ++step)
            for (int i = 0; i < n; ++i)
                if (step <= runs[i].N)
                    if (tdbem_status st = runs[i].step(step); st != TDBEM_OK) return st;
    }
    for (int i = 0; i < n; ++i)
        if (tdbem_status st = runs[i].end(); st != TDBEM_OK) {
            restore_layouts();
            return st;
        }
    tdbem_status result = TDBEM_OK;
    std::string first_error;
    for (int i = 0; i < n; ++i) {
        tdbem_report rep{};
        const tdbem_status st = runs[i].finish(&rep);
        if (reports) reports[i] = rep;
        if (st != TDBEM_OK && result == TDBEM_OK) {
            result = st;
            first_error = "model " + std::to_string(i) + ": " + g_error;
        }
    }
    restore_layouts();
    if (result != TDBEM_OK) g_error = first_error;
    return result;
}

}  // extern "C"

namespace {

bool pinned(const void* p)
{
    if (!p) return true;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

extern "C" {

tdbem_status tdbem_md_march(tdbem_handle* h, const double* known_lu, double* out_lu, double* out_lt,
                            tdbem_report* report, void* stream)
{
    g_error.clear();
    if (!h || !known_lu) return fail(TDBEM_INVALID_INPUT, "null argument");
    if (!h->assembled) return fail(TDBEM_NOT_ASSEMBLED, "call tdbem_md_assemble or tdbem_md_load_matrices first");
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : h->s0;
    const int N = h->nstep, R = h->R;
    const size_t step_doubles = (size_t)h->E * 3;
    const size_t n = sizeof(double) * (size_t)R * (N + 1) * step_doubles;
    if (h->d_known.bytes != n) {
        CUDA_TRY(h->d_known.alloc(n));
        CUDA_TRY(h->d_out_lu.alloc(n));
        CUDA_TRY(h->d_out_lt.alloc(n));
    }
    tdbem_status st = TDBEM_OK;
    if (!(pinned(known_lu) && pinned(out_lu) && pinned(out_lt))) {
        CUDA_TRY(cudaMemcpyAsync(h->d_known.p, known_lu, n, cudaMemcpyDefault, s));
        st = tdbem_md_march_device(h, h->d_known.as<double>(), h->d_out_lu.as<double>(), h->d_out_lt.as<double>(),
                                   report, s);
        if (st != TDBEM_OK && st != TDBEM_NOT_CONVERGED) return st;
        if (out_lu) CUDA_TRY(cudaMemcpyAsync(out_lu, h->d_out_lu.p, n, cudaMemcpyDefault, s));
        if (out_lt) CUDA_TRY(cudaMemcpyAsync(out_lt, h->d_out_lt.p, n, cudaMemcpyDefault, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        h->diag_ready = h->record;
        return st;
    }
    // Pinned host buffers: the copies run beside the march by chunks of
    // steps.  Chunk 0's inputs go ahead of the set-up on the caller's stream,
    // the later chunks' on the input stream, each waited for by the first
    // step that reads it; each chunk's boundary values go back on the output
    // stream once its last step's GMRES (which writes them) is done.
    const int chunks = std::max(1, std::min(N + 1, 32));
    std::vector<int> bound((size_t)chunks + 1);
    for (int c = 0; c <= chunks; ++c) bound[c] = (int)((int64_t)(N + 1) * c / chunks);
    auto copy_chunk = [&](int c, bool in, cudaStream_t on) -> cudaError_t {
        const size_t off = (size_t)bound[c] * step_doubles, cnt = (size_t)(bound[c + 1] - bound[c]) * step_doubles;
        for (int r = 0; r < R; ++r) {
            const size_t o = (size_t)r * (N + 1) * step_doubles + off;
            cudaError_t e = cudaSuccess;
            if (in) {
                e = cudaMemcpyAsync(h->d_known.as<double>() + o, known_lu + o, sizeof(double) * cnt,
                                    cudaMemcpyHostToDevice, on);
            } else {
                if (out_lu)
                    e = cudaMemcpyAsync(out_lu + o, h->d_out_lu.as<double>() + o, sizeof(double) * cnt,
                                        cudaMemcpyDeviceToHost, on);
                if (e == cudaSuccess && out_lt)
                    e = cudaMemcpyAsync(out_lt + o, h->d_out_lt.as<double>() + o, sizeof(double) * cnt,
                                        cudaMemcpyDeviceToHost, on);
            }
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    std::vector<cudaEvent_t> ev;
    CUDA_TRY(h->ev_order.take(2 * (size_t)chunks + 2, ev));
    cudaEvent_t* in_done = ev.data();
    cudaEvent_t* out_ready = ev.data() + chunks;
    CUDA_TRY(copy_chunk(0, true, s));
    CUDA_TRY(cudaEventRecord(ev[2 * chunks], s));  // the input stream follows the caller's stream
    CUDA_TRY(cudaStreamWaitEvent(h->cin, ev[2 * chunks], 0));
    for (int c = 1; c < chunks; ++c) {
        CUDA_TRY(copy_chunk(c, true, h->cin));
        CUDA_TRY(cudaEventRecord(in_done[c], h->cin));
    }
    MarchRun run;
    if ((st = run.begin(h, h->d_known.as<double>(), h->d_out_lu.as<double>(), h->d_out_lt.as<double>(), s)) !=
        TDBEM_OK) {
        cudaStreamSynchronize(h->cin);
        return st;
    }
    int c = 0;
    for (int step = 1; step <= N && st == TDBEM_OK; ++step) {
        while (c + 1 < chunks && step >= bound[c + 1]) {
            // chunk c's boundary values are complete: steps < bound[c + 1] are done
            if (cudaEventRecord(out_ready[c], run.s) != cudaSuccess ||
                cudaStreamWaitEvent(h->cout, out_ready[c], 0) != cudaSuccess || copy_chunk(c, false, h->cout) != cudaSuccess)
                st = fail(TDBEM_CUDA_ERROR, "output copy");
            ++c;
            if (cudaStreamWaitEvent(run.s, in_done[c], 0) != cudaSuccess) st = fail(TDBEM_CUDA_ERROR, "input wait");
        }
        if (st == TDBEM_OK) st = run.step(step);
    }
    if (st == TDBEM_OK) st = run.end();
    if (st == TDBEM_OK) {
        // the remaining chunks after the last step, on the caller's stream
        // (which follows the march), then the caller's stream follows the
        // output stream
        for (; c < chunks; ++c) CUDA_TRY(copy_chunk(c, false, s));
        CUDA_TRY(cudaEventRecord(ev[2 * chunks + 1], h->cout));
        CUDA_TRY(cudaStreamWaitEvent(s, ev[2 * chunks + 1], 0));
        st = run.finish(report);
    }
    CUDA_TRY(cudaStreamSynchronize(s));
    CUDA_TRY(cudaStreamSynchronize(h->cout));
    CUDA_TRY(cudaStreamSynchronize(h->cin));
    if (st != TDBEM_OK && st != TDBEM_NOT_CONVERGED) return st;
    h->diag_ready = h->record;
    return st;
}

tdbem_status tdbem_md_step_record(tdbem_handle* h, double* rhs, double* x, int32_t* flags)
{
    if (!h) return fail(TDBEM_INVALID_INPUT, "null handle");
    const size_t n = sizeof(double) * 3 * h->E * h->nstep;
    if ((rhs || x) && !h->d_rec_rhs.p) return fail(TDBEM_INVALID_INPUT, "no record: call tdbem_md_set_record(h, 1) before the march");
    if (rhs) CUDA_TRY(cudaMemcpy(rhs, h->d_rec_rhs.p, n, cudaMemcpyDeviceToHost));
    if (x) CUDA_TRY(cudaMemcpy(x, h->d_rec_x.p, n, cudaMemcpyDeviceToHost));
    if (flags && h->d_flags.p) CUDA_TRY(cudaMemcpy(flags, h->d_flags.p, sizeof(int) * 3 * h->nstep, cudaMemcpyDeviceToHost));
    return TDBEM_OK;
}

tdbem_status tdbem_md_export_matrix(tdbem_handle* h, int32_t which, int32_t k, int64_t* n_rows, int64_t* nnz,
                                    int32_t* row_ptr, int32_t* col, double* val)
{
    if (!h) return fail(TDBEM_INVALID_INPUT, "null handle");
    if (!h->assembled) return fail(TDBEM_NOT_ASSEMBLED, "nothing assembled");
    const int64_t E = h->E;
    if (n_rows) *n_rows = E;
    if (which == 0 || which == 1) {
        const auto& rp = which == 0 ? h->a_rp : h->k_rp;
        const auto& cc = which == 0 ? h->a_col : h->k_col;
        const auto& vv = which == 0 ? h->a_val : h->k_val;
        if (nnz) *nnz = rp[E];
        if (row_ptr) std::copy(rp.begin(), rp.end(), row_ptr);
        if (col) std::copy(cc.begin(), cc.end(), col);
        if (val) std::copy(vv.begin(), vv.end(), val);
        return TDBEM_OK;
    }
    if ((which != 2 && which != 3) || k < 1 || k > h->K) return fail(TDBEM_INVALID_INPUT, "no such matrix");
    const int type = which == 3 ? 1 : 0;
    const int K = h->K;
    std::vector<uint32_t> hc;
    std::vector<double> hv;
    CUDA_TRY(download(hc, h->d_h_col, h->h_nnz, h->s0));
    std::vector<int32_t> rp(E + 1, 0), cc;
    std::vector<double> vv;
    const bool want_vals = val != nullptr;
    if (want_vals) CUDA_TRY(download(hv, h->d_h_val, 9 * h->h_nnz, h->s0));
    for (int64_t r = 0; r < E; ++r) {
        std::vector<std::pair<int32_t, int64_t>> row;
        for (int64_t j = h->h_kptr[r * (K + 1) + k - 1]; j < h->h_kptr[r * (K + 1) + k]; ++j) {
            const uint32_t c = hc[j];
            if ((int)((c >> 20) & 1u) == type) row.push_back({(int32_t)(c & 0xFFFFFu), j});
        }
        std::sort(row.begin(), row.end());
        for (auto& e : row) {
            cc.push_back(e.first);
            if (want_vals)
                for (int q = 0; q < 9; ++q) vv.push_back((type ? 1.0 : -1.0) * hv[q * h->h_nnz + e.second]);
        }
        rp[r + 1] = (int32_t)cc.size();
    }
    if (nnz) *nnz = (int64_t)cc.size();
    if (row_ptr) std::copy(rp.begin(), rp.end(), row_ptr);
    if (col) std::copy(cc.begin(), cc.end(), col);
    if (val) std::copy(vv.begin(), vv.end(), val);
    return TDBEM_OK;
}

tdbem_status tdbem_md_geometry(tdbem_handle* h, double* coordcoef, double* center, double* radius, double* radius_pw,
                               double* transmat, double* on_u1, double* on_t1, double* on_t2)
{
    if (!h) return fail(TDBEM_INVALID_INPUT, "null handle");
    CUDA_TRY(cudaSetDevice(h->device));
    const int64_t E = h->E;
    struct {
        double* dst;
        DevBuf* src;
        int64_t n;
    } items[] = {{coordcoef, &h->g_cc, 24 * E}, {center, &h->g_center, 3 * E}, {radius, &h->g_radius, E},
                 {radius_pw, &h->g_rpw, E},     {transmat, &h->g_trans, 9 * E}, {on_u1, &h->g_u1, 9 * E},
                 {on_t1, &h->g_t1, 9 * E},      {on_t2, &h->g_t2, 9 * E}};
    for (auto& it : items)
        if (it.dst) CUDA_TRY(cudaMemcpy(it.dst, it.src->p, sizeof(double) * it.n, cudaMemcpyDeviceToHost));
    return TDBEM_OK;
}

tdbem_status tdbem_md_info(tdbem_handle* h, double* dt, int64_t* n_unknown, int64_t* n_known, int64_t* n_history,
                           int64_t* n_leaves)
{
    if (!h) return fail(TDBEM_INVALID_INPUT, "null handle");
    if (dt) *dt = h->dt;
    if (n_unknown) *n_unknown = h->n_unknown;
    if (n_known) *n_known = h->n_known;
    if (n_history) *n_history = h->n_hist;
    if (n_leaves) *n_leaves = (int64_t)h->leaf_begin.size();
    return TDBEM_OK;
}

tdbem_status tdbem_md_precond_layout(tdbem_handle* h, int64_t* repid, int64_t* leaf_begin, int64_t* leaf_count)
{
    if (!h) return fail(TDBEM_INVALID_INPUT, "null handle");
    if (repid) std::copy(h->repid.begin(), h->repid.end(), repid);
    if (leaf_begin) std::copy(h->leaf_begin.begin(), h->leaf_begin.end(), leaf_begin);
    if (leaf_count) std::copy(h->leaf_count.begin(), h->leaf_count.end(), leaf_count);
    return TDBEM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Solve without device allocation.  The storage of one FP64 single-load
// GMRES solve lives in one static device array per device, found once with
// cudaGetSymbolAddress; the call itself only enqueues a memset, three kernels
// and (optionally) a copy of three flags.
namespace {

// Capacity of the static scratch.  One solve needs, in doubles,
//   (15 + 9 (restart + 1)) E + 5 C (restart + 2) + 32
// plus 256-byte alignment of each region (C = GMRES cluster CTAs): at
// restart 30 about 2.35 KB per element, so roughly 14,000 elements.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
struct NoAllocDevice {
    bool ready = false;
    unsigned char* scratch = nullptr;
    int max_cluster = 0;  // schedulable cluster size of the FP64 single-load GMRES kernel
};
NoAllocDevice g_noalloc[kMaxDevices];
std::mutex g_noalloc_mutex;

// Scratch regions of one solve, each 256-byte aligned.  The head (status
// word and flags) starts at zero on every call.  The GMRES kernel runs with
// solve_only set, so the march's write-back targets (boundary values,
// history states, audit) need no storage here.
struct NoAllocLayout {
    size_t head = 0, b = 0, bp = 0, x = 0, rv = 0, u = 0, V = 0, W = 0, AW = 0, givens = 0, zero_bytes = 0, total = 0;
};

NoAllocLayout noalloc_layout(int64_t E, int rs, int C)
{
    NoAllocLayout L;
    size_t at = 0;
    auto take = [&](size_t doubles) {
        const size_t o = at;
        at += (doubles * sizeof(double) + 255) / 256 * 256;
        return o;
    };
    const size_t e3 = 3 * (size_t)E;
    L.head = take(32);
    L.zero_bytes = at;
    L.b = take(e3);
    L.bp = take(e3);
    L.x = take(e3);
    L.rv = take(e3);
    L.u = take(e3);
    L.V = take((size_t)(rs + 1) * e3);
    L.W = take((size_t)(rs + 1) * e3);
    L.AW = take((size_t)(rs + 1) * e3);
    L.givens = take((size_t)C * kGivensArrays * (rs + 2));
    L.total = at;
    return L;
}

// Natural equation-row order -> leaf (perm) order.
__global__ void noalloc_rows_to_perm(int E, const int32_t* row_of, const double* rhs, double* b)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 3LL * E; t += (int64_t)gridDim.x * blockDim.x)
        b[t] = rhs[3LL * row_of[t / 3] + t % 3];
}

// Leaf (perm) order -> natural unknown order.
__global__ void noalloc_perm_to_unknowns(int E, const int32_t* perm_of_unk, const double* x, double* out)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 3LL * E; t += (int64_t)gridDim.x * blockDim.x)
        out[t] = x[3LL * perm_of_unk[t / 3] + t % 3];
}

// First call on a device (that device current): the scratch address and the
// largest cluster the single-load kernel can be scheduled with.
tdbem_status noalloc_setup(int device, NoAllocDevice** out)
{
    if (device < 0 || device >= kMaxDevices) return fail(TDBEM_INVALID_INPUT, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoAllocDevice& nd = g_noalloc[device];
    if (!nd.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return fail(TDBEM_CUDA_ERROR, std::string("cudaGetSymbolAddress of the static scratch: ") +
                                              cudaGetErrorString(e));
        nd.scratch = static_cast<unsigned char*>(p);
        nd.max_cluster = gmres_cluster_size(device, 1, false);
        nd.ready = true;
    }
    *out = &nd;
    return TDBEM_OK;
}

}  // namespace

extern "C" {

tdbem_status tdbem_md_solve_noalloc(tdbem_handle* h, const double* d_rhs, double* d_x, int32_t* flags,
                                    void* stream)
{
    g_error.clear();
    if (!h || !d_rhs || !d_x) return fail(TDBEM_INVALID_INPUT, "null argument");
    if (!h->assembled) return fail(TDBEM_NOT_ASSEMBLED, "call tdbem_md_assemble or tdbem_md_load_matrices first");
    CUDA_TRY(cudaSetDevice(h->device));
    NoAllocDevice* nd = nullptr;
    if (tdbem_status st = noalloc_setup(h->device, &nd); st != TDBEM_OK) return st;
    const int64_t E = h->E;
    const int rs = h->restart, C = h->cluster;
    if (C > nd->max_cluster)
        return fail(TDBEM_INVALID_INPUT, "the handle's GMRES cluster of " + std::to_string(C) +
                                             " CTAs exceeds the " + std::to_string(nd->max_cluster) +
                                             " the single-load solver can be scheduled with");
    const NoAllocLayout L = noalloc_layout(E, rs, C);
    if (L.total > kNoAllocScratchBytes)
        return fail(TDBEM_INVALID_INPUT, "tdbem_md_solve_noalloc needs " + std::to_string(L.total) +
                                             " bytes of scratch for " + std::to_string(E) +
                                             " elements at restart " + std::to_string(rs) +
                                             "; its static scratch holds " +
                                             std::to_string(kNoAllocScratchBytes) + " bytes");
    cudaStream_t s = stream ? (cudaStream_t)stream : h->s0;
    unsigned char* base = nd->scratch;
    auto dbl = [&](size_t off) { return reinterpret_cast<double*>(base + off); };
    MarchData d{};
    d.E = (int)E;
    d.nh = (int)h->n_hist;
    d.R = 1;
    d.nstep = 1;
    d.SW = 1;
    d.mixed = 0;
    d.a_rp = h->d_a_rp.as<int32_t>();
    d.a_col = h->d_a_col.as<int32_t>();
    d.a_val = h->d_a_val.as<double>();
    d.row_of = h->d_row_of.as<int32_t>();
    d.perm_of_unk = h->d_perm_of_unk.as<int32_t>();
    d.leaf_begin = h->d_leaf_begin.as<int32_t>();
    d.leaf_count = h->d_leaf_count.as<int32_t>();
    d.leaf_of_perm = h->d_leaf_of_perm.as<int32_t>();
    d.leaf_off = h->d_leaf_off.as<int64_t>();
    d.pinv = h->d_pinv.as<double>();
    d.cta_leaf = h->d_cta_leaf.as<int32_t>();
    d.a_colx = h->d_a_colx.as<int32_t>();
    d.dsm_rows = h->dsm_rows;
    d.uref_block = h->d_uref_block.as<int64_t>();
    d.uref_sign = h->d_uref_sign.as<double>();
    d.uref_known = h->d_uref_known.as<int32_t>();
    d.tref_block = h->d_tref_block.as<int64_t>();
    d.tref_sign = h->d_tref_sign.as<double>();
    d.tref_known = h->d_tref_known.as<int32_t>();
    d.hist_block = h->d_hist_block.as<int64_t>();
    d.hu_sign = h->d_hu_sign.as<double>();
    d.ht_sign = h->d_ht_sign.as<double>();
    d.hist_owner = h->d_hist_owner.as<int32_t>();
    d.itf_trans = h->d_itf_trans.as<double>();
    d.trans = h->g_trans.as<double>();
    d.bcid = h->g_bcid.as<int32_t>();
    d.itf_pairs = h->d_itf_pairs.as<int32_t>();
    d.itf_sign = h->d_itf_sign.as<double>();
    d.n_itf = (int)h->I;
    d.status = reinterpret_cast<int*>(base + L.head);
    d.step_flags = reinterpret_cast<int*>(base + L.head + 16);
    d.solve_only = 1;
    d.b = dbl(L.b);
    d.groups = 1;
    d.bp = dbl(L.bp);
    d.x = dbl(L.x);
    d.rv = dbl(L.rv);
    d.u = dbl(L.u);
    d.V = dbl(L.V);
    d.W = dbl(L.W);
    d.AW = dbl(L.AW);
    d.givens = dbl(L.givens);
    d.restart = rs;
    d.tol = h->tol;
    d.cluster = C;
    d.givens_stride = (int64_t)kGivensArrays * (rs + 2);
    const int grid = (int)std::min<int64_t>(ceil_div(3 * E, 256), 4 * 148);
    CUDA_TRY(cudaMemsetAsync(base, 0, L.zero_bytes, s));
    noalloc_rows_to_perm<<<grid, 256, 0, s>>>((int)E, d.row_of, d_rhs, d.b);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(gmres_solve_single(d, s));
    noalloc_perm_to_unknowns<<<grid, 256, 0, s>>>((int)E, d.perm_of_unk, d.x, d_x);
    CUDA_TRY(cudaGetLastError());
    if (flags) {
        CUDA_TRY(cudaMemcpyAsync(flags, d.step_flags, 3 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        if (flags[0] != 0) return fail(TDBEM_NOT_CONVERGED, "GMRES flag " + std::to_string(flags[0]));
    }
    return TDBEM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Validation output in the reference's formats (WriteValidationOutputs,
// DBEM1/DBEM.cpp:434-561; WriteMultiDomainValidationMetrics and the matrix
// structure diagnosis, DBEM1/multidomain.cpp:387-416, 3314-3420): the same
// files, columns and keys, so tools written against the reference read them.
namespace {

// 3x3 full-pivot Gauss-Jordan singularity test with the 1e-10 pivot bound of
// the reference's inv_mat (DBEM1/lin_comp.cpp:83-117); true when invertible
// with a finite inverse.
bool block_invertible(const double* b9)
{
    double a[3][6] = {};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            if (!std::isfinite(b9[3 * i + j])) return false;
            a[i][j] = b9[3 * i + j];
        }
    for (int i = 0; i < 3; ++i) a[i][3 + i] = 1.0;
    int colperm[3] = {0, 1, 2};
    for (int k = 0; k < 3; ++k) {
        int pi = k, pj = k;
        double best = 0.0;
        for (int i = k; i < 3; ++i)
            for (int j = k; j < 3; ++j)
                if (std::fabs(a[i][j]) > best) {
                    best = std::fabs(a[i][j]);
                    pi = i;
                    pj = j;
                }
        if (best <= 1.0e-10) return false;
        for (int j = 0; j < 6; ++j) std::swap(a[k][j], a[pi][j]);
        for (int i = 0; i < 3; ++i) std::swap(a[i][k], a[i][pj]);
        std::swap(colperm[k], colperm[pj]);
        const double piv = a[k][k];
        for (int j = 0; j < 6; ++j) a[k][j] /= piv;
        for (int i = 0; i < 3; ++i)
            if (i != k) {
                const double f = a[i][k];
                for (int j = 0; j < 6; ++j) a[i][j] -= f * a[k][j];
            }
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 3; j < 6; ++j)
            if (!std::isfinite(a[i][j])) return false;
    return true;
}

}  // namespace

extern "C" {

tdbem_status tdbem_md_write_validation(tdbem_handle* h, const char* directory, int32_t load, const double* out_lu,
                                       const double* out_lt, const tdbem_report* report)
{
    g_error.clear();
    if (!h || !directory || !out_lu || !out_lt || !report) return fail(TDBEM_INVALID_INPUT, "null argument");
    if (load < 0 || load >= h->R) return fail(TDBEM_INVALID_INPUT, "load case out of range");
    if (!h->assembled) return fail(TDBEM_NOT_ASSEMBLED, "no matrices");
    const int64_t E = h->E;
    const int N = h->nstep, R = h->R;
    const double* lu = out_lu + (size_t)load * (N + 1) * E * 3;
    const double* lt = out_lt + (size_t)load * (N + 1) * E * 3;
    const std::string dir(directory);
    FILE* f = std::fopen((dir + "/validation_state.csv").c_str(), "w");
    if (!f) return fail(TDBEM_INVALID_INPUT, "cannot open " + dir + "/validation_state.csv");
    std::fprintf(f, "step,element,localNode,nodeId,domain,surfaceType,bcid,x,y,z,ux,uy,uz,tx,ty,tz\n");
    for (int step = 0; step <= N; ++step)
        for (int64_t e = 0; e < E; ++e) {
            const double* u = lu + ((size_t)step * E + e) * 3;
            const double* t = lt + ((size_t)step * E + e) * 3;
            const double* x = &h->node[3 * e];
            std::fprintf(f, "%d,%lld,0,%lld,%d,%d,%d,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g\n", step,
                         (long long)e, (long long)e, h->domain_of[e], h->surface[e], h->bcid[e], x[0], x[1], x[2],
                         u[0], u[1], u[2], t[0], t[1], t[2]);
        }
    std::fclose(f);

    // interface transfer audit per solved step (WriteInterfaceTransferAuditCsv,
    // DBEM1/multidomain.cpp:329-379; one node per constant element)
    {
        FILE* fa = open_diagnostic_csv(dir + "/interface_transfer_audit.csv",
                                       "solver,step,interfaceId,domainA,domainB,normalSign,localNode,nodeA,nodeB,eleA,"
                                       "eleB,component,uA,uB,uJump,tA,tB,tResidual");
        if (!fa) return fail(TDBEM_INVALID_INPUT, "cannot open " + dir + "/interface_transfer_audit.csv");
        const char comp[3] = {'x', 'y', 'z'};
        for (int step = 1; step <= std::min(N, report->steps_solved); ++step)
            for (int64_t i = 0; i < h->I; ++i) {
                const int64_t* it = &h->itf[5 * i];
                const int sgn = it[4] == 0 ? -1 : (int)it[4];
                const int64_t a = it[1], b = it[3];
                for (int k = 0; k < 3; ++k) {
                    const size_t ia = ((size_t)step * E + a) * 3 + k, ib = ((size_t)step * E + b) * 3 + k;
                    std::fprintf(fa, "multidomain,%d,%lld,%d,%d,%d,0,%lld,%lld,%lld,%lld,%c,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g\n",
                                 step, (long long)i, (int)it[0], (int)it[2], sgn, (long long)a, (long long)b,
                                 (long long)a, (long long)b, comp[k], lu[ia], lu[ib], lu[ia] - lu[ib], lt[ia], lt[ib],
                                 lt[ib] - (double)sgn * lt[ia]);
                }
            }
        std::fclose(fa);
    }

    // per-step GMRES counts of this load case
    std::vector<int> flags(3 * (size_t)std::max(N, 1) * R, 0);
    if (h->d_flags.p)
        CUDA_TRY(cudaMemcpy(flags.data(), h->d_flags.p, std::min(h->d_flags.bytes, sizeof(int) * flags.size()),
                            cudaMemcpyDeviceToHost));
    long outer = 0, inner = 0;
    int final_flag = 0;
    const int solved = report->steps_solved;
    for (int step = 1; step <= std::min(N, solved + (report->failed_step ? 1 : 0)); ++step) {
        const int* fl = &flags[3 * ((size_t)(step - 1) * R + load)];
        outer += fl[1];
        inner += fl[2];
        final_flag = fl[0];
    }
    f = std::fopen((dir + "/validation_metrics.txt").c_str(), "w");
    if (!f) return fail(TDBEM_INVALID_INPUT, "cannot open " + dir + "/validation_metrics.txt");
    std::fprintf(f, "ValidationOutput=1\nSolver=2\nNStep=%d\nDt=%.17g\nElementCount=%lld\nNodeCount=%lld\n", N, h->dt,
                 (long long)E, (long long)E);
    std::fprintf(f, "MultiDomainActive=1\nDomainCount=%d\nInterfaceCount=%lld\n", h->D, (long long)h->I);
    for (int d = 0; d < h->D; ++d)
        std::fprintf(f, "DomainMaterial[%d]=C1 %.17g C2 %.17g C1Dt %.17g C2Dt %.17g\n", d, h->mats[d].C1, h->mats[d].C2,
                     h->mats[d].C1Dt, h->mats[d].C2Dt);
    double all_u = 0.0, all_t = 0.0;
    for (int step = 0; step <= N; ++step) {
        double mu = 0.0, mt = 0.0;
        for (int64_t i = 0; i < h->I; ++i) {
            const int64_t a = h->itf[5 * i + 1], b = h->itf[5 * i + 3];
            const double sg = h->itf[5 * i + 4] == 0 ? -1.0 : (double)h->itf[5 * i + 4];
            for (int k = 0; k < 3; ++k) {
                const size_t ia = ((size_t)step * E + a) * 3 + k, ib = ((size_t)step * E + b) * 3 + k;
                mu = std::max(mu, std::fabs(lu[ia] - lu[ib]));
                mt = std::max(mt, std::fabs(lt[ib] - sg * lt[ia]));
            }
        }
        all_u = std::max(all_u, mu);
        all_t = std::max(all_t, mt);
        std::fprintf(f, "InterfaceStep[%d].MaxAbsU=%.17g\nInterfaceStep[%d].MaxAbsTBalance=%.17g\n", step, mu, step, mt);
    }
    std::fprintf(f, "InterfaceOverallMaxAbsU=%.17g\nInterfaceOverallMaxAbsTBalance=%.17g\n", all_u, all_t);
    // structure of A (natural order)
    long zero_rows = 0, zero_cols = 0, nonfinite = 0, diag = 0, diag_inv = 0;
    std::vector<long> colc((size_t)E, 0);
    for (int64_t r = 0; r < E; ++r) {
        const int b = h->a_rp[r], e = h->a_rp[r + 1];
        if (b == e) ++zero_rows;
        for (int p = b; p < e; ++p) {
            const int c = h->a_col[p];
            if (c < 0 || c >= E) {
                ++nonfinite;
                continue;
            }
            ++colc[c];
            const double* v = &h->a_val[9 * (size_t)p];
            bool fin = true;
            for (int q = 0; q < 9; ++q) fin = fin && std::isfinite(v[q]);
            if (!fin) ++nonfinite;
            if (c == r) {
                ++diag;
                if (block_invertible(v)) ++diag_inv;
            }
        }
    }
    for (int64_t c = 0; c < E; ++c) zero_cols += colc[c] == 0;
    const double steps = std::max(N, 1);
    std::fprintf(f, "MultiDomainMetricsValid=1\nMultiDomainFinalFlag=%d\nMultiDomainSolvedSteps=%d\n", final_flag, solved);
    std::fprintf(f, "MultiDomainTotalOuterIterations=%ld\nMultiDomainTotalInnerIterations=%ld\n", outer, inner);
    std::fprintf(f, "MultiDomainAverageOuterIterations=%lf\nMultiDomainAverageInnerIterations=%lf\n",
                 solved > 0 ? (double)outer / solved : 0.0, solved > 0 ? (double)inner / solved : 0.0);
    std::fprintf(f, "MultiDomainDomainCount=%d\nMultiDomainGlobalUnknownBlocks=%lld\n", h->D, (long long)h->n_unknown);
    std::fprintf(f, "MultiDomainMTS0NonZeroBlocks=%lld\n", (long long)(h->a_rp.empty() ? 0 : h->a_rp[E]));
    std::fprintf(f, "MultiDomainMTSAverageBlocks=%lf\nMultiDomainMGSAverageBlocks=%lf\n",
                 N > 0 ? (double)h->hist_mts_blocks / steps : 0.0, N > 0 ? (double)h->hist_mgs_blocks / steps : 0.0);
    std::fprintf(f, "MultiDomainMatrixAssemblyTime=%lf\nMultiDomainGMRESTime=%lf\n", h->assembly_s,
                 report->ms_gmres / 1000.0);
    std::fprintf(f, "MultiDomainMatrixStructureValid=%d\n", zero_rows == 0 && zero_cols == 0 && nonfinite == 0);
    std::fprintf(f, "MultiDomainMatrixZeroRows=%ld\nMultiDomainMatrixZeroCols=%ld\nMultiDomainMatrixNonFiniteBlocks=%ld\n",
                 zero_rows, zero_cols, nonfinite);
    std::fprintf(f, "MultiDomainMatrixDiagonalBlocks=%ld\nMultiDomainMatrixInvertibleDiagonalBlocks=%ld\n", diag,
                 diag_inv);
    // the DOF-map invariants are checked when the handle is created, which
    // fails on any violation
    std::fprintf(f, "MultiDomainInterfaceDofInvariantValid=1\nMultiDomainInterfaceDofInvariantFailures=0\n");
    std::fclose(f);
    return TDBEM_OK;
}

tdbem_status tdbem_md_write_rhs_diagnostics(tdbem_handle* h, const char* directory, const tdbem_report* report)
{
    g_error.clear();
    if (!h || !directory || !report) return fail(TDBEM_INVALID_INPUT, "null argument");
    if (!h->diag_ready)
        return fail(TDBEM_INVALID_INPUT,
                    "no recorded march: call tdbem_md_set_record(h, 1) and then tdbem_md_march (or "
                    "tdbem_md_march_forward)");
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t s = h->s0;
    const int64_t E = h->E, nh = std::max<int64_t>(h->n_hist, 1);
    const int N = h->nstep;
    const int solved = std::min(N, report->steps_solved);
    const std::string dir(directory);
    // history states of load 0 and A in equation-row order
    DevBuf xh, arp, acol, aval, out;
    CUDA_TRY(xh.alloc(sizeof(double) * 6 * (size_t)(N + 1) * nh));
    CUDA_TRY(cudaMemsetAsync(xh.p, 0, xh.bytes, s));
    if (h->n_hist > 0 && N > 0) {
        const int grid = (int)std::min<int64_t>(ceil_div((int64_t)N * E, 256), 4 * 148);
        history_states_kernel<<<grid, 256, 0, s>>>(N, (int)E, (int)h->n_hist, h->d_hist_owner.as<int32_t>(),
                                                   h->d_hist_block.as<int64_t>(), h->d_hu_sign.as<double>(),
                                                   h->d_ht_sign.as<double>(), h->d_out_lu.as<double>(),
                                                   h->d_out_lt.as<double>(), xh.as<double>());
        CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(up(arp, h->a_rp, s));
    CUDA_TRY(up(acol, h->a_col, s));
    CUDA_TRY(up(aval, h->a_val, s));
    CUDA_TRY(out.alloc(sizeof(double) * 12 * (size_t)E));
    std::vector<double> center, parts(12 * (size_t)E), rhs(3 * (size_t)E), x(3 * (size_t)E);
    CUDA_TRY(download(center, h->g_center, 3 * (size_t)E, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    FILE* fb = open_diagnostic_csv(dir + "/rhs_breakdown.csv",
                                   "solver,step,rowNode,rowElement,localNode,domain,surfaceType,bcid,cx,cy,cz,"
                                   "component,knownRhs,historyG,historyT,totalRhs,Ax,residual,solution");
    if (!fb) return fail(TDBEM_INVALID_INPUT, "cannot open " + dir + "/rhs_breakdown.csv");
    FILE* fr = open_diagnostic_csv(dir + "/residual_probe.csv",
                                   "solver,step,maxAbsResidual,l2Residual,l2Rhs,relativeResidual");
    if (!fr) {
        std::fclose(fb);
        return fail(TDBEM_INVALID_INPUT, "cannot open " + dir + "/residual_probe.csv");
    }
    const char comp[3] = {'x', 'y', 'z'};
    for (int n = 1; n <= solved; ++n) {
        RhsSplitArgs a{};
        a.E = (int)E;
        a.K = h->K;
        a.nh = (int)nh;
        a.n = n;
        a.h_kptr = h->d_h_kptr.as<int64_t>();
        a.h_col = h->d_h_col.as<uint32_t>();
        a.h_val = h->d_h_val.as<double>();
        a.h_nnz = h->h_nnz;
        a.xh = xh.as<double>();
        a.k_rp = h->d_k_rp.as<int32_t>();
        a.k_col = h->d_k_col.as<int32_t>();
        a.k_val = h->d_k_val.as<double>();
        a.known_elem = h->d_known_elem.as<int32_t>();
        a.known_sign = h->d_known_sign.as<double>();
        a.known = h->d_known.as<double>();
        a.a_rp = arp.as<int32_t>();
        a.a_col = acol.as<int32_t>();
        a.a_val = aval.as<double>();
        a.x = h->d_rec_x.as<double>() + (size_t)(n - 1) * 3 * E;
        a.out = out.as<double>();
        CUDA_TRY(rhs_split(a, s));
        CUDA_TRY(cudaMemcpyAsync(parts.data(), out.p, sizeof(double) * 12 * E, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyAsync(rhs.data(), h->d_rec_rhs.as<double>() + (size_t)(n - 1) * 3 * E,
                                 sizeof(double) * 3 * E, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyAsync(x.data(), a.x, sizeof(double) * 3 * E, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        const double* pk = parts.data();
        const double* pg = pk + 3 * E;
        const double* pt = pg + 3 * E;
        const double* ax = pt + 3 * E;
        double max_res = 0.0, res2 = 0.0, rhs2 = 0.0;
        for (int64_t r = 0; r < E; ++r)
            for (int c = 0; c < 3; ++c) {
                const size_t p = 3 * (size_t)r + c;
                const double res = ax[p] - rhs[p];
                // the solution column is x in unknown order read at the row's
                // index, as the reference prints it
                std::fprintf(fb, "multidomain,%d,%lld,%lld,0,%d,%d,%d,%.17g,%.17g,%.17g,%c,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g\n",
                             n, (long long)r, (long long)r, h->domain_of[r], h->surface[r], h->bcid[r], center[3 * r],
                             center[3 * r + 1], center[3 * r + 2], comp[c], pk[p], pg[p], pt[p], rhs[p], ax[p], res,
                             x[p]);
                max_res = std::max(max_res, std::fabs(res));
                res2 += res * res;
                rhs2 += rhs[p] * rhs[p];
            }
        const double l2r = std::sqrt(res2), l2b = std::sqrt(rhs2);
        std::fprintf(fr, "multidomain,%d,%.17g,%.17g,%.17g,%.17g\n", n, max_res, l2r, l2b, l2b > 0.0 ? l2r / l2b : l2r);
    }
    std::fclose(fb);
    std::fclose(fr);
    return TDBEM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Matrix cache file: the assembled A, KnownM, MTS_k and MGS_k of a handle,
// saved once and loaded by later runs of the same model instead of
// assembling.  Each matrix is stored like the reference's
// CCSRMat::WriteBinary (DBEM1/mat_vec.cpp:1690-1707: n, nnz, row_ptr, col,
// 9 values per block, with 64-bit counts) behind a header and an entry table
// as in its single-domain gmres_ccsr_cache.bin (DBEM1/pre_gmres.cpp:316-488).
// The header carries a fingerprint of the model (geometry, BCIDs, domains,
// materials, interfaces, dt, gap): a cache is only loaded into the same model.
namespace {

struct MatCacheHeader {
    char magic[16];
    int32_t version, matrix_count;
    int64_t E, n_unknown, n_known, n_hist, n_steps, K;
    double dt, gap;
    uint64_t fingerprint;
};
struct MatCacheEntry {
    int32_t type, step;  // 1 A, 2 MTS_k, 3 MGS_k, 4 KnownM
    int64_t offset, bytes;
};
constexpr char kMatCacheMagic[16] = "TDBEMMDCACHE";

uint64_t fnv(uint64_t h, const void* p, size_t n)
{
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}

uint64_t model_fingerprint(const tdbem_handle* h)
{
    uint64_t f = 1469598103934665603ull;
    f = fnv(f, h->points.data(), sizeof(double) * h->points.size());
    f = fnv(f, h->elements.data(), sizeof(int64_t) * h->elements.size());
    f = fnv(f, h->bcid.data(), sizeof(int32_t) * h->bcid.size());
    f = fnv(f, h->domain_of.data(), sizeof(int32_t) * h->domain_of.size());
    f = fnv(f, h->itf.data(), sizeof(int64_t) * h->itf.size());
    for (const DynaMat& m : h->mats) f = fnv(f, &m, sizeof(DynaMat));
    f = fnv(f, &h->dt, sizeof(double));
    f = fnv(f, &h->gap, sizeof(double));
    return f;
}

bool write_ccsr(FILE* f, const std::vector<int32_t>& rp, const std::vector<int32_t>& col, const std::vector<double>& val)
{
    const int64_t n = (int64_t)rp.size() - 1, nnz = (int64_t)col.size();
    return std::fwrite(&n, 8, 1, f) == 1 && std::fwrite(&nnz, 8, 1, f) == 1 &&
           std::fwrite(rp.data(), 4, rp.size(), f) == rp.size() &&
           (nnz == 0 || std::fwrite(col.data(), 4, col.size(), f) == col.size()) &&
           (nnz == 0 || std::fwrite(val.data(), 8, val.size(), f) == val.size());
}

bool read_ccsr(FILE* f, int64_t E, std::vector<int32_t>& rp, std::vector<int32_t>& col, std::vector<double>& val)
{
    int64_t n = 0, nnz = 0;
    if (std::fread(&n, 8, 1, f) != 1 || std::fread(&nnz, 8, 1, f) != 1 || n != E || nnz < 0) return false;
    rp.resize((size_t)n + 1);
    col.resize((size_t)nnz);
    val.resize(9 * (size_t)nnz);
    return std::fread(rp.data(), 4, rp.size(), f) == rp.size() &&
           (nnz == 0 || std::fread(col.data(), 4, col.size(), f) == col.size()) &&
           (nnz == 0 || std::fread(val.data(), 8, val.size(), f) == val.size()) && rp[(size_t)n] == nnz;
}

}  // namespace

extern "C" {

tdbem_status tdbem_md_save_matrices(tdbem_handle* h, const char* path)
{
    g_error.clear();
    if (!h || !path) return fail(TDBEM_INVALID_INPUT, "null argument");
    if (!h->assembled) return fail(TDBEM_NOT_ASSEMBLED, "nothing assembled");
    CUDA_TRY(cudaSetDevice(h->device));
    const int64_t E = h->E;
    const int K = h->K;
    // the stacked history matrix, once, split back into MTS_k and MGS_k
    std::vector<uint32_t> hc;
    std::vector<double> hv;
    CUDA_TRY(download(hc, h->d_h_col, (size_t)h->h_nnz, h->s0));
    CUDA_TRY(download(hv, h->d_h_val, 9 * (size_t)h->h_nnz, h->s0));
    CUDA_TRY(cudaStreamSynchronize(h->s0));
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(TDBEM_INVALID_INPUT, std::string("cannot open ") + path);
    MatCacheHeader hd{};
    std::memcpy(hd.magic, kMatCacheMagic, sizeof(hd.magic));
    hd.version = 1;
    hd.matrix_count = 2 + 2 * K;
    hd.E = E;
    hd.n_unknown = h->n_unknown;
    hd.n_known = h->n_known;
    hd.n_hist = h->n_hist;
    hd.n_steps = h->nstep;
    hd.K = K;
    hd.dt = h->dt;
    hd.gap = h->gap;
    hd.fingerprint = model_fingerprint(h);
    std::vector<MatCacheEntry> ent((size_t)hd.matrix_count);
    bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1 && std::fwrite(ent.data(), sizeof(MatCacheEntry), ent.size(), f) == ent.size();
    size_t idx = 0;
    auto put = [&](int type, int step, const std::vector<int32_t>& rp, const std::vector<int32_t>& col,
                   const std::vector<double>& val) {
        if (!ok) return;
        ent[idx].type = type;
        ent[idx].step = step;
        ent[idx].offset = (int64_t)std::ftell(f);
        ok = write_ccsr(f, rp, col, val);
        ent[idx].bytes = (int64_t)std::ftell(f) - ent[idx].offset;
        ++idx;
    };
    put(1, 0, h->a_rp, h->a_col, h->a_val);
    put(4, 0, h->k_rp, h->k_col, h->k_val);
    for (int type = 0; type <= 1 && ok; ++type)
        for (int k = 1; k <= K && ok; ++k) {
            std::vector<int32_t> rp((size_t)E + 1, 0), cc;
            std::vector<double> vv;
            for (int64_t r = 0; r < E; ++r) {
                for (int64_t j = h->h_kptr[r * (K + 1) + k - 1]; j < h->h_kptr[r * (K + 1) + k]; ++j) {
                    const uint32_t c = hc[(size_t)j];
                    if ((int)((c >> 20) & 1u) != type) continue;  // ascending columns within the segment
                    cc.push_back((int32_t)(c & 0xFFFFFu));
                    for (int q = 0; q < 9; ++q) vv.push_back((type ? 1.0 : -1.0) * hv[(size_t)q * h->h_nnz + j]);
                }
                rp[(size_t)r + 1] = (int32_t)cc.size();
            }
            put(type ? 3 : 2, k, rp, cc, vv);
        }
    ok = ok && std::fseek(f, (long)sizeof(hd), SEEK_SET) == 0 &&
         std::fwrite(ent.data(), sizeof(MatCacheEntry), ent.size(), f) == ent.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(TDBEM_INVALID_INPUT, std::string("writing ") + path + " failed");
    return TDBEM_OK;
}

tdbem_status tdbem_md_load_matrix_cache(tdbem_handle* h, const char* path, void* stream)
{
    g_error.clear();
    if (!h || !path) return fail(TDBEM_INVALID_INPUT, "null argument");
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(TDBEM_INVALID_INPUT, std::string("cannot open ") + path);
    MatCacheHeader hd{};
    std::string why;
    if (std::fread(&hd, sizeof(hd), 1, f) != 1 || std::memcmp(hd.magic, kMatCacheMagic, sizeof(hd.magic)) != 0 ||
        hd.version != 1)
        why = "not a matrix cache of this library";
    else if (hd.E != h->E || hd.n_unknown != h->n_unknown || hd.n_known != h->n_known || hd.n_hist != h->n_hist)
        why = "element or DOF counts differ";
    else if (hd.n_steps != h->nstep)
        why = "NStep differs";
    else if (hd.fingerprint != model_fingerprint(h))
        why = "model fingerprint differs (geometry, boundary types, domains, materials, interfaces, dt or gap)";
    std::vector<MatCacheEntry> ent;
    if (why.empty()) {
        ent.resize((size_t)std::max(hd.matrix_count, 0));
        if (hd.matrix_count != 2 + 2 * hd.K ||
            std::fread(ent.data(), sizeof(MatCacheEntry), ent.size(), f) != ent.size())
            why = "entry table damaged";
    }
    std::vector<int32_t> arp, acol, krp, kcol, trp, tcol, grp, gcol;
    std::vector<double> aval, kval, tval, gval;
    const int K = (int)hd.K;
    for (size_t i = 0; why.empty() && i < ent.size(); ++i) {
        std::vector<int32_t> rp, col;
        std::vector<double> val;
        if (std::fseek(f, (long)ent[i].offset, SEEK_SET) != 0 || !read_ccsr(f, hd.E, rp, col, val)) {
            why = "matrix " + std::to_string(i) + " damaged";
            break;
        }
        if (ent[i].type == 1) {
            arp = rp; acol = col; aval = val;
        } else if (ent[i].type == 4) {
            krp = rp; kcol = col; kval = val;
        } else {
            auto& R = ent[i].type == 2 ? trp : grp;
            auto& C = ent[i].type == 2 ? tcol : gcol;
            auto& V = ent[i].type == 2 ? tval : gval;
            R.insert(R.end(), rp.begin(), rp.end());
            C.insert(C.end(), col.begin(), col.end());
            V.insert(V.end(), val.begin(), val.end());
        }
    }
    std::fclose(f);
    if (!why.empty()) return fail(TDBEM_INVALID_INPUT, std::string(path) + ": " + why);
    if (trp.size() != (size_t)K * (hd.E + 1) || grp.size() != trp.size())
        return fail(TDBEM_INVALID_INPUT, std::string(path) + ": history matrices incomplete");
    if (tcol.empty()) { tcol.push_back(0); tval.resize(9); }
    if (gcol.empty()) { gcol.push_back(0); gval.resize(9); }
    if (trp.empty()) { trp.push_back(0); grp.push_back(0); }
    return tdbem_md_load_matrices(h, arp.data(), acol.data(), aval.data(), krp.data(), kcol.data(), kval.data(), K,
                                  trp.data(), tcol.data(), tval.data(), grp.data(), gcol.data(), gval.data(), stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Adjoint of the FP64 march: the vector-Jacobian product of
//   known_lu -> (out_lu, out_lt)
// for one load case, run as a reverse time march with transposed operators
// (the forward operations of DBEM1/multidomain.cpp:3819-3893, transposed):
//   lam_n = A^-T g_n,  g_n = (write-back)^T (cotangent_n + state adjoint_n),
//   state adjoint_n = sum_k H_k^T (lam_{n+k-1} + 2 lam_{n+k} + lam_{n+k+1}),
//   d/dknown_n = (write-back)^T_known (...) + KnownM^T lam_n.
// The march is linear in the prescribed values, so no forward state is kept.
namespace {

__global__ void gather_blocks(int E, const int32_t* idx, const double* in, double* out)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 3LL * E; t += (int64_t)gridDim.x * blockDim.x)
        out[t] = in[3LL * idx[t / 3] + t % 3];
}

tdbem_status adjoint_setup(tdbem_handle* h, cudaStream_t s)
{
    auto A = std::make_unique<AdjointState>();
    const int64_t E = h->E;
    const int K = h->K;
    const int64_t nh = std::max<int64_t>(h->n_hist, 1);
    std::vector<int32_t> row_of((size_t)E), unk_of((size_t)E), perm_of_unk((size_t)E), perm_of_row((size_t)E);
    for (int64_t p = 0; p < E; ++p) {
        row_of[p] = (int32_t)h->repid[p];
        unk_of[p] = (int32_t)h->pref[h->repid[p]];
    }
    for (int64_t p = 0; p < E; ++p) {
        perm_of_unk[unk_of[p]] = (int32_t)p;
        perm_of_row[row_of[p]] = (int32_t)p;
    }
    // A'^T: A(r, c) sits at A'(perm_of_row[r], perm_of_unk[c]); transposed,
    // row perm_of_unk[c], column perm_of_row[r], block B^T
    std::vector<std::vector<std::pair<int32_t, int64_t>>> rows((size_t)E);
    for (int64_t r = 0; r < E; ++r)
        for (int j = h->a_rp[r]; j < h->a_rp[r + 1]; ++j) rows[perm_of_unk[h->a_col[j]]].push_back({perm_of_row[r], j});
    std::vector<int32_t> rp((size_t)E + 1, 0), col;
    std::vector<double> val;
    for (int64_t q = 0; q < E; ++q) {
        std::sort(rows[q].begin(), rows[q].end());
        for (auto& e : rows[q]) {
            col.push_back(e.first);
            const double* B = &h->a_val[9 * (size_t)e.second];
            for (int i = 0; i < 3; ++i)
                for (int k = 0; k < 3; ++k) val.push_back(B[3 * k + i]);
        }
        rp[q + 1] = (int32_t)col.size();
    }
    CUDA_TRY(up(A->at_rp, rp, s));
    CUDA_TRY(up(A->at_col, col, s));
    CUDA_TRY(up(A->at_val, val, s));
    // transposed leaf inverses
    const int nl = (int)h->leaf_begin.size();
    int64_t total = 0;
    for (int l = 0; l < nl; ++l) total += 9 * h->leaf_count[l] * h->leaf_count[l];
    std::vector<double> pinv;
    CUDA_TRY(download(pinv, h->d_pinv, (size_t)total, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    std::vector<double> pinvT(pinv.size());
    int64_t off = 0;
    for (int l = 0; l < nl; ++l) {
        const int64_t n3 = 3 * h->leaf_count[l];
        for (int64_t i = 0; i < n3; ++i)
            for (int64_t j = 0; j < n3; ++j) pinvT[off + i * n3 + j] = pinv[off + j * n3 + i];
        off += n3 * n3;
    }
    CUDA_TRY(up(A->pinvT, pinvT, s));
    // history blocks by (type, column) and k, regrouped on the device
    const int64_t hn = std::max<int64_t>(h->h_nnz, 1);
    CUDA_TRY(A->tptr.alloc(sizeof(int64_t) * 2 * (size_t)nh * (K + 1)));
    CUDA_TRY(A->trow.alloc(sizeof(int32_t) * (size_t)hn));
    CUDA_TRY(A->tval.alloc(sizeof(double) * 9 * (size_t)hn));
    CUDA_TRY(adjoint_history_groups((int)E, K, (int)nh, h->h_nnz, h->d_h_kptr.as<int64_t>(), h->d_h_col.as<uint32_t>(),
                                    h->d_h_val.as<double>(), A->tptr.as<int64_t>(), A->trow.as<int32_t>(),
                                    A->tval.as<double>(), s));
    CUDA_TRY(up(A->unk_of, unk_of, s));
    CUDA_TRY(up(A->perm_of_row, perm_of_row, s));
    // sources (element * 2 + U/T) of every unknown in element order, and
    // KnownM by columns in row order, for the device-side transposed write-back
    {
        std::vector<int32_t> src(2 * (size_t)E, -1);
        for (int64_t i = 0; i < E; ++i)
            for (int which = 0; which < 2; ++which) {
                if (which ? h->tref_known[i] : h->uref_known[i]) continue;
                const int64_t u = which ? h->tref_block[i] : h->uref_block[i];
                int32_t* slot = &src[2 * (size_t)u];
                if (slot[0] < 0) slot[0] = (int32_t)(2 * i + which);
                else if (slot[1] < 0) slot[1] = (int32_t)(2 * i + which);
                else return fail(TDBEM_DOFMAP_INVALID, "an unknown block has more than two references");
            }
        CUDA_TRY(up(A->unk_src, src, s));
        const int64_t nk = h->n_known;
        std::vector<int32_t> ptr((size_t)nk + 1, 0), row, blk;
        for (int64_t r = 0; r < E; ++r)
            for (int j = h->k_rp[r]; j < h->k_rp[r + 1]; ++j) ++ptr[h->k_col[j] + 1];
        for (int64_t k = 0; k < nk; ++k) ptr[k + 1] += ptr[k];
        row.assign((size_t)ptr[nk], 0);
        blk.assign((size_t)ptr[nk], 0);
        std::vector<int32_t> fill(ptr.begin(), ptr.end() - 1);
        for (int64_t r = 0; r < E; ++r)
            for (int j = h->k_rp[r]; j < h->k_rp[r + 1]; ++j) {
                const int32_t o = fill[h->k_col[j]]++;
                row[o] = (int32_t)r;
                blk[o] = j;
            }
        CUDA_TRY(up(A->kt_ptr, ptr, s));
        CUDA_TRY(up(A->kt_row, row, s));
        CUDA_TRY(up(A->kt_blk, blk, s));
        const size_t per = 3 * (size_t)E;
        for (DevBuf* b : {&A->cot_u, &A->cot_t, &A->gk}) CUDA_TRY(b->alloc(sizeof(double) * per * (h->nstep + 1)));
        CUDA_TRY(A->contrib.alloc(sizeof(double) * 2 * per));
        CUDA_TRY(A->flags_all.alloc(sizeof(int) * 3 * (size_t)std::max(h->nstep, 1)));
    }
    // GMRES storage for one load case
    const size_t vec = sizeof(double) * 3 * (size_t)E;
    const int rs = h->restart;
    for (DevBuf* b : {&A->b, &A->bp, &A->x, &A->rv, &A->u, &A->g, &A->gp}) CUDA_TRY(b->alloc(vec));
    for (DevBuf* b : {&A->V, &A->W, &A->AW}) CUDA_TRY(b->alloc(vec * (rs + 1)));
    CUDA_TRY(A->givens.alloc(sizeof(double) * (size_t)h->cluster * kGivensArrays * (rs + 2)));
    CUDA_TRY(A->status.alloc(sizeof(int) * 4));
    CUDA_TRY(A->flags.alloc(sizeof(int) * 4));
    CUDA_TRY(A->audit.alloc(sizeof(double) * 2));
    CUDA_TRY(A->xring.alloc(sizeof(double) * 18 * nh));
    CUDA_TRY(A->wring.alloc(sizeof(double) * 6 * nh));
    for (DevBuf* b : {&A->known, &A->out_lu, &A->out_lt}) CUDA_TRY(b->alloc(2 * vec));
    CUDA_TRY(cudaMemsetAsync(A->known.p, 0, 2 * vec, s));
    CUDA_TRY(A->lam.alloc(sizeof(double) * 3 * (size_t)E * (h->nstep + 2)));
    CUDA_TRY(A->adj.alloc(sizeof(double) * 6 * (size_t)nh));
    CUDA_TRY(cudaStreamSynchronize(s));
    h->adjoint = std::move(A);
    return TDBEM_OK;
}

}  // namespace

extern "C" {

tdbem_status tdbem_md_march_vjp(tdbem_handle* h, const double* cot_lu, const double* cot_lt, double* grad_known,
                                tdbem_report* report, void* stream)
{
    g_error.clear();
    if (!h || !grad_known) return fail(TDBEM_INVALID_INPUT, "null argument");
    if (!h->assembled) return fail(TDBEM_NOT_ASSEMBLED, "call tdbem_md_assemble or tdbem_md_load_matrices first");
    if (h->R != 1) return fail(TDBEM_INVALID_INPUT, "the adjoint march takes handles of one load case");
    CUDA_TRY(cudaSetDevice(h->device));
    if (gmres_cluster_size(h->device, 1, false) < h->cluster)
        return fail(TDBEM_INVALID_INPUT, "the handle's GMRES cluster is too large for the one-load solver");
    cudaStream_t s = stream ? (cudaStream_t)stream : h->s0;
    if (!h->adjoint)
        if (tdbem_status st = adjoint_setup(h, s); st != TDBEM_OK) return st;
    AdjointState& A = *h->adjoint;
    const int64_t E = h->E, nh = h->n_hist;
    const int N = h->nstep, K = h->K;
    const size_t per = 3 * (size_t)E;
    MarchData d{};
    d.E = (int)E;
    d.nh = (int)nh;
    d.R = 1;
    d.nstep = 1;
    d.SW = 1;
    d.a_rp = A.at_rp.as<int32_t>();
    d.a_col = A.at_col.as<int32_t>();
    d.a_val = A.at_val.as<double>();
    d.pinv = A.pinvT.as<double>();
    d.row_of = h->d_row_of.as<int32_t>();
    d.perm_of_unk = h->d_perm_of_unk.as<int32_t>();
    d.leaf_begin = h->d_leaf_begin.as<int32_t>();
    d.leaf_count = h->d_leaf_count.as<int32_t>();
    d.leaf_of_perm = h->d_leaf_of_perm.as<int32_t>();
    d.leaf_off = h->d_leaf_off.as<int64_t>();
    d.cta_leaf = h->d_cta_leaf.as<int32_t>();
    d.dsm_rows = 0;
    d.uref_block = h->d_uref_block.as<int64_t>();
    d.uref_sign = h->d_uref_sign.as<double>();
    d.uref_known = h->d_uref_known.as<int32_t>();
    d.tref_block = h->d_tref_block.as<int64_t>();
    d.tref_sign = h->d_tref_sign.as<double>();
    d.tref_known = h->d_tref_known.as<int32_t>();
    d.hist_block = h->d_hist_block.as<int64_t>();
    d.hu_sign = h->d_hu_sign.as<double>();
    d.ht_sign = h->d_ht_sign.as<double>();
    d.hist_owner = h->d_hist_owner.as<int32_t>();
    d.itf_trans = h->d_itf_trans.as<double>();
    d.trans = h->g_trans.as<double>();
    d.bcid = h->g_bcid.as<int32_t>();
    d.itf_pairs = h->d_itf_pairs.as<int32_t>();
    d.itf_sign = h->d_itf_sign.as<double>();
    d.n_itf = (int)h->I;
    d.status = A.status.as<int>();
    d.step_flags = A.flags.as<int>();
    d.audit = A.audit.as<double>();
    d.xring = A.xring.as<double>();
    d.wring = A.wring.as<double>();
    d.known_lu = A.known.as<double>();
    d.out_lu = A.out_lu.as<double>();
    d.out_lt = A.out_lt.as<double>();
    d.b = A.gp.as<double>();
    d.groups = 1;
    d.bp = A.bp.as<double>();
    d.x = A.x.as<double>();
    d.rv = A.rv.as<double>();
    d.u = A.u.as<double>();
    d.V = A.V.as<double>();
    d.W = A.W.as<double>();
    d.AW = A.AW.as<double>();
    d.givens = A.givens.as<double>();
    d.restart = h->restart;
    d.tol = h->tol;
    d.cluster = h->cluster;
    d.givens_stride = (int64_t)kGivensArrays * (h->restart + 2);
    CUDA_TRY(cudaMemsetAsync(A.lam.p, 0, A.lam.bytes, s));
    // the reverse march runs on the device without host round trips:
    // cotangents in, transposed write-back, A'^T solve, KnownM^T, history
    // adjoint; GMRES flags per step are read once at the end
    const size_t all = per * (size_t)(N + 1);
    if (cot_lu) CUDA_TRY(cudaMemcpyAsync(A.cot_u.p, cot_lu, sizeof(double) * all, cudaMemcpyDefault, s));
    if (cot_lt) CUDA_TRY(cudaMemcpyAsync(A.cot_t.p, cot_lt, sizeof(double) * all, cudaMemcpyDefault, s));
    CUDA_TRY(cudaMemsetAsync(A.gk.p, 0, A.gk.bytes, s));
    CUDA_TRY(cudaMemsetAsync(A.flags_all.p, 0, A.flags_all.bytes, s));
    AdjWriteBack wb{};
    wb.E = (int)E;
    wb.nh = (int)nh;
    wb.cot_lu = cot_lu ? A.cot_u.as<double>() : nullptr;
    wb.cot_lt = cot_lt ? A.cot_t.as<double>() : nullptr;
    wb.hist_owner = h->d_hist_owner.as<int32_t>();
    wb.hist_block = h->d_hist_block.as<int64_t>();
    wb.hu_sign = h->d_hu_sign.as<double>();
    wb.ht_sign = h->d_ht_sign.as<double>();
    wb.trans = h->g_trans.as<double>();
    wb.itf_trans = h->d_itf_trans.as<double>();
    wb.uref_sign = h->d_uref_sign.as<double>();
    wb.tref_sign = h->d_tref_sign.as<double>();
    wb.uref_known = h->d_uref_known.as<int32_t>();
    wb.tref_known = h->d_tref_known.as<int32_t>();
    wb.gk = A.gk.as<double>();
    wb.contrib = A.contrib.as<double>();
    tdbem_report rep{};
    const int grid = (int)std::min<int64_t>(ceil_div(3 * E, 256), 4 * 148);
    for (int n = N; n >= 1; --n) {
        wb.adj = nullptr;
        if (n < N && nh > 0) {
            CUDA_TRY(adj_history(N, n, K, (int)nh, (int)E, A.tptr.as<int64_t>(), A.trow.as<int32_t>(),
                                 A.tval.as<double>(), A.lam.as<double>(), A.adj.as<double>(), s));
            wb.adj = A.adj.as<double>();
        }
        // lam_n = A^-T g: write-back transposed into A'^T rows, solve, equation rows
        CUDA_TRY(adjoint_writeback(wb, n, A.unk_src.as<int32_t>(), A.unk_of.as<int32_t>(), A.gp.as<double>(), s));
        CUDA_TRY(cudaMemsetAsync(A.status.p, 0, A.status.bytes, s));
        d.step_flags = A.flags_all.as<int>() + 3 * (size_t)(n - 1);
        CUDA_TRY(gmres_solve_single(d, s));
        double* lam_n = A.lam.as<double>() + (size_t)n * per;
        gather_blocks<<<grid, 256, 0, s>>>((int)E, A.perm_of_row.as<int32_t>(), A.x.as<double>(), lam_n);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(adjoint_known((int)h->n_known, A.kt_ptr.as<int32_t>(), A.kt_row.as<int32_t>(),
                               A.kt_blk.as<int32_t>(), h->d_k_val.as<double>(), h->d_known_elem.as<int32_t>(),
                               h->d_known_sign.as<double>(), lam_n, A.gk.as<double>() + (size_t)n * per, s));
    }
    // step 0: bd[0] converted to the global frame (lu for BCID 123, lt for 456)
    CUDA_TRY(adjoint_step0((int)E, h->g_trans.as<double>(), h->g_bcid.as<int32_t>(), wb.cot_lu, wb.cot_lt,
                           A.gk.as<double>(), s));
    std::vector<int> fl(3 * (size_t)std::max(N, 1), 0);
    CUDA_TRY(cudaMemcpyAsync(fl.data(), A.flags_all.p, sizeof(int) * fl.size(), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(grad_known, A.gk.p, sizeof(double) * all, cudaMemcpyDefault, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    for (int n = N; n >= 1; --n) {
        const int* f = &fl[3 * (size_t)(n - 1)];
        rep.total_inner += f[2];
        if (f[0] != 0) {
            rep.failed_step = n;
            rep.gmres_flag = f[0];
            if (report) *report = rep;
            return fail(TDBEM_NOT_CONVERGED, "adjoint GMRES flag " + std::to_string(f[0]) + " at step " +
                                                 std::to_string(n));
        }
        rep.steps_solved = N - n + 1;
    }
    if (report) *report = rep;
    return TDBEM_OK;
}

}  // extern "C"

namespace {

// grad[2d], grad[2d+1] = dJ/dE_d, dJ/drho_d from the adjoint vectors of the
// last tdbem_md_march_vjp and the state kept by tdbem_md_march_forward.
tdbem_status material_gradient(tdbem_handle* h, cudaStream_t s, double* grad)
{
    AdjointState& A = *h->adjoint;
    const int64_t E = h->E, nh = h->n_hist;
    const int N = h->nstep;
    std::vector<DynaMatD> dm;
    for (const DynaMat& m : h->mats) dm.push_back(build_mat_dual(m));
    CUDA_TRY(upload_materials_dual(dm.data(), (int)dm.size(), s));
    PairSetup P;
    if (tdbem_status st = pair_setup(h, P, s); st != TDBEM_OK) return st;
    const int64_t np = P.ps.n_pairs;
    ElemGeom g = h->geom();
    DevBuf self_d, xh, part;
    CUDA_TRY(self_d.alloc(sizeof(QDual) * 27 * (size_t)E));
    CUDA_TRY(xh.alloc(sizeof(double) * 6 * (size_t)(N + 1) * (size_t)std::max<int64_t>(nh, 1)));
    CUDA_TRY(part.alloc(sizeof(double) * 2 * (size_t)std::max<int64_t>(np, 1)));
    singular_grad_kernel<<<(unsigned)E, 256, 0, s>>>((int)E, h->d_secpw_pos.as<double>(), h->d_secpw_val.as<double>(),
                                                     g, self_d.as<QDual>());
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemsetAsync(xh.p, 0, xh.bytes, s));
    if (nh > 0 && N > 0) {
        const int grid = (int)std::min<int64_t>(ceil_div((int64_t)N * E, 256), 4 * 148);
        history_states_kernel<<<grid, 256, 0, s>>>(N, (int)E, (int)nh, h->d_hist_owner.as<int32_t>(),
                                                   h->d_hist_block.as<int64_t>(), h->d_hu_sign.as<double>(),
                                                   h->d_ht_sign.as<double>(), h->d_out_lu.as<double>(),
                                                   h->d_out_lt.as<double>(), xh.as<double>());
        CUDA_TRY(cudaGetLastError());
    }
    const GradState gs{N,
                       (int)E,
                       h->K,
                       (int)nh,
                       A.lam.as<double>(),
                       h->d_rec_x.as<double>(),
                       h->d_known.as<double>(),
                       xh.as<double>(),
                       h->d_known_elem.as<int32_t>(),
                       h->d_known_sign.as<double>(),
                       P.col_a0.as<int64_t>(),
                       P.col_a1.as<int64_t>(),
                       P.col_k.as<int64_t>(),
                       P.col_h.as<int64_t>()};
    std::fill(grad, grad + 2 * (size_t)h->D, 0.0);
    std::vector<double> pv;
    const int warps = 4;
    for (int pass = 0; pass < 2 && np > 0; ++pass) {
        if (pass == 0)
            grad_step0_kernel<<<ceil_div(np, warps), 32 * warps, 0, s>>>(P.ps, h->d_rules.as<QuadRules>(), g, P.dr,
                                                                         self_d.as<QDual>(), gs, part.as<double>());
        else
            grad_history_kernel<<<ceil_div(np, warps), 32 * warps, 0, s>>>(P.ps, h->d_rules.as<QuadRules>(), g, P.dr,
                                                                           self_d.as<QDual>(), gs, part.as<double>());
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(download(pv, part, 2 * (size_t)np, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        // fixed summation order per domain: gE, gU
        for (int d = 0; d < h->D; ++d)
            for (int64_t p = P.poff[d]; p < P.poff[d + 1]; ++p) {
                grad[2 * d] += pv[2 * p];
                grad[2 * d + 1] += pv[2 * p + 1];
            }
    }
    // dJ/drho = -(E/rho) dJ/dE - gU / rho
    for (int d = 0; d < h->D; ++d) {
        const DynaMat& m = h->mats[d];
        const double E = 2.0 * m.G * (1.0 + m.v), rho = m.Rou;
        grad[2 * d + 1] = -(E / rho) * grad[2 * d] - grad[2 * d + 1] / rho;
    }
    return TDBEM_OK;
}

}  // namespace

extern "C" {

tdbem_status tdbem_md_march_forward(tdbem_handle* h, const double* known_lu, double* out_lu, double* out_lt,
                                    tdbem_report* report, void* stream)
{
    g_error.clear();
    if (!h || !known_lu) return fail(TDBEM_INVALID_INPUT, "null argument");
    if (h->R != 1) return fail(TDBEM_INVALID_INPUT, "the forward/backward pair takes handles of one load case");
    const bool rec = h->record;
    h->record = true;
    const tdbem_status st = tdbem_md_march(h, known_lu, out_lu, out_lt, report, stream);
    h->record = rec;
    h->saved_forward = st == TDBEM_OK;
    return st;
}

tdbem_status tdbem_md_march_backward(tdbem_handle* h, const double* cot_lu, const double* cot_lt, double* grad_known,
                                     double* grad_material, tdbem_report* report, void* stream)
{
    g_error.clear();
    if (!h || !grad_known) return fail(TDBEM_INVALID_INPUT, "null argument");
    if (!h->saved_forward)
        return fail(TDBEM_INVALID_INPUT, "no saved forward state: call tdbem_md_march_forward on this handle first");
    const tdbem_status st = tdbem_md_march_vjp(h, cot_lu, cot_lt, grad_known, report, stream);
    if (st != TDBEM_OK || !grad_material) return st;
    CUDA_TRY(cudaSetDevice(h->device));
    return material_gradient(h, stream ? (cudaStream_t)stream : h->s0, grad_material);
}

}  // extern "C"

namespace {

// One timed march of the first `steps` steps on the handle's current launch
// configuration (after a warm-up march of the first `warm` steps, laid out
// for that length in known_w); +inf when it fails to converge.
tdbem_status time_prefix(tdbem_handle* h, int steps, int warm, const DevBuf& known, const DevBuf& known_w,
                         DevBuf& out_u, DevBuf& out_t, cudaStream_t s, double& ms)
{
    const int n_keep = h->nstep;
    tdbem_report rep{};
    h->nstep = warm;
    tdbem_status st = tdbem_md_march_device(h, known_w.as<double>(), out_u.as<double>(), out_t.as<double>(), &rep, s);
    if (st == TDBEM_OK) {
        h->nstep = steps;
        st = tdbem_md_march_device(h, known.as<double>(), out_u.as<double>(), out_t.as<double>(), &rep, s);
    }
    h->nstep = n_keep;
    ms = st == TDBEM_OK ? rep.ms_total / steps : std::numeric_limits<double>::infinity();
    return st == TDBEM_NOT_CONVERGED ? TDBEM_OK : st;
}

}  // namespace

extern "C" {

tdbem_status tdbem_md_autotune(tdbem_handle* h, const double* known_lu, int32_t steps, tdbem_tuning* out,
                               void* stream)
{
    g_error.clear();
    if (!h || !known_lu) return fail(TDBEM_INVALID_INPUT, "null argument");
    if (!h->assembled) return fail(TDBEM_NOT_ASSEMBLED, "call tdbem_md_assemble or tdbem_md_load_matrices first");
    if (h->nstep < 1) return fail(TDBEM_INVALID_INPUT, "the model has no time steps");
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t s = stream ? (cudaStream_t)stream : h->s0;
    const int N = h->nstep, R = h->R;
    const int64_t E = h->E;
    steps = std::max(1, std::min<int32_t>(steps, N));
    // the first `steps` steps of every load case, laid out for a march of that length
    const size_t per = (size_t)(steps + 1) * E * 3, full = (size_t)(N + 1) * E * 3;
    const int warm = std::min(3, steps);
    const size_t per_w = (size_t)(warm + 1) * E * 3;
    DevBuf known, known_w, out_u, out_t;
    CUDA_TRY(known.alloc(sizeof(double) * per * R));
    CUDA_TRY(known_w.alloc(sizeof(double) * per_w * R));
    CUDA_TRY(out_u.alloc(sizeof(double) * per * R));
    CUDA_TRY(out_t.alloc(sizeof(double) * per * R));
    for (int r = 0; r < R; ++r) {
        CUDA_TRY(cudaMemcpyAsync(known.as<double>() + r * per, known_lu + r * full, sizeof(double) * per,
                                 cudaMemcpyHostToDevice, s));
        CUDA_TRY(cudaMemcpyAsync(known_w.as<double>() + r * per_w, known_lu + r * full, sizeof(double) * per_w,
                                 cudaMemcpyHostToDevice, s));
    }
    const bool rec = h->record;
    h->record = false;
    const bool mixed = h->precision == TDBEM_PRECISION_MIXED;
    int sms = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    struct Conf {
        int G, C, cpt;
    };
    tdbem_tuning t{};
    const Conf start{h->groups, h->cluster, h->rhs_cpt};
    auto run = [&](const Conf& c, double& ms) -> tdbem_status {
        if (tdbem_status st = gmres_layout(h, c.G, c.C, s); st != TDBEM_OK) return st;
        h->rhs_cpt = c.cpt;
        ++t.candidates;
        return time_prefix(h, steps, warm, known, known_w, out_u, out_t, s, ms);
    };
    auto restore = [&](const Conf& c) {
        gmres_layout(h, c.G, c.C, s);
        h->rhs_cpt = c.cpt;
        h->record = rec;
    };
    double best_ms = 0.0;
    tdbem_status st = run(start, best_ms);
    if (st != TDBEM_OK) {
        restore(start);
        return st;
    }
    t.ms_per_step_default = best_ms;
    Conf best = start;
    // stage 1: load-case groups x cluster size (GMRES), default history tiling
    for (int G = 1; G <= R; G *= 2) {
        if (R % G) continue;
        const int cmax = gmres_cluster_size(h->device, R / G, mixed);
        for (int C = cmax; C >= std::max(1, cmax / 4); C /= 2) {
            if (G * C > sms || (G == start.G && C == start.C)) continue;
            double ms = 0.0;
            if ((st = run(Conf{G, C, start.cpt}, ms)) != TDBEM_OK) {
                restore(start);
                return st;
            }
            if (ms < best_ms) {
                best_ms = ms;
                best = Conf{G, C, start.cpt};
            }
        }
    }
    // stage 2: load cases per thread of the history pass at the best GMRES layout
    std::vector<int> cpts;
    if (R >= 4) cpts = {4, 2};
    else if (R == 2) cpts = {2, 1};
    for (int c : cpts) {
        const int cur = best.cpt ? best.cpt : (R >= 4 ? 4 : R);
        if (c == cur) continue;
        double ms = 0.0;
        if ((st = run(Conf{best.G, best.C, c}, ms)) != TDBEM_OK) {
            restore(start);
            return st;
        }
        if (ms < best_ms) {
            best_ms = ms;
            best.cpt = c;
        }
    }
    restore(best);
    CUDA_TRY(cudaStreamSynchronize(s));
    t.gmres_groups = h->groups;
    t.gmres_cluster = h->cluster;
    t.rhs_cases_per_thread = h->rhs_cpt ? h->rhs_cpt : (R >= 4 ? 4 : R);
    t.steps = steps;
    t.ms_per_step = best_ms;
    if (out) *out = t;
    return TDBEM_OK;
}

}  // extern "C"
