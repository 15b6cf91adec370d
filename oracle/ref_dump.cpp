// Golden-data harness around the reference solver (test infrastructure only).
//
// Linked against the unchanged reference objects (DBEM1/*.cpp, with main()
// renamed to dbem_reference_main).  The linker wraps two calls that cross
// reference object files:
//   * DynaGMRESSolverMultiDomainCCSR (DBEM1/multidomain.h:214-223): before the
//     real solver runs, this harness records the element geometry, singular
//     self-element blocks, per-domain materials and the Step0 / history
//     matrices assembled by the reference's own AssembleMultiDomainStep0 and
//     AssembleMultiDomainHistoryStep (DBEM1/multidomain.cpp:2256-2378); after it
//     returns, the final boundary values bd[0..NStep].
//   * gmres(..., CCSRMat&, ...) (DBEM1/pre_gmres.cpp:1369-1605): records the
//     right-hand side, solution, flag and iteration counts of every step, and
//     the mapped-leaf preconditioner layout on the first call.
// Records go to the file named by TDBEM_DUMP (default ref_dump.bin) in a
// simple tagged binary format read by tests/golden/refdump.py.
// TDBEM_DUMP_MATRICES=0 skips the serial re-assembly of the matrices (the
// DOF counts, geometry, per-step records and final boundary values are still
// written): on the 3072-element bar that re-assembly would take longer than
// the reference's own threaded run and the records would hold gigabytes.

#include "multidomain.h"
#include "pre_gmres.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

int dbem_reference_main();

extern "C" int __real__Z30DynaGMRESSolverMultiDomainCCSRP14DSquareElementP13BoundaryValueRK16MultiDomainModelldlldPPlS7_(
    DSquareElement*, BoundaryValue*, const MultiDomainModel&, long, double, long, long, double, long**, long**);
extern "C" int __real__Z5gmresP14DSquareElementR7CCSRMatR7WvectorR14PreConditionerldlS4_S4_RiPi(
    DSquareElement*, CCSRMat&, Wvector&, PreConditioner&, long, double, long, Wvector&, Wvector&, int&, int*);

namespace {

FILE* g_out = nullptr;
long g_step = 0;
bool g_preDumped = false;

void open_out()
{
    if (g_out) return;
    const char* path = getenv("TDBEM_DUMP");
    g_out = fopen(path ? path : "ref_dump.bin", "wb");
    if (!g_out) { perror("TDBEM_DUMP"); exit(3); }
    fwrite("TDBD", 1, 4, g_out);
}

// dtype: 0 = float64, 1 = int32, 2 = int64
void put(const std::string& name, int dtype, const std::vector<uint64_t>& dims, const void* data)
{
    open_out();
    uint32_t n = (uint32_t)name.size();
    fwrite(&n, 4, 1, g_out);
    fwrite(name.data(), 1, n, g_out);
    uint8_t dt = (uint8_t)dtype;
    fwrite(&dt, 1, 1, g_out);
    uint32_t nd = (uint32_t)dims.size();
    fwrite(&nd, 4, 1, g_out);
    uint64_t count = 1;
    for (uint64_t d : dims) { fwrite(&d, 8, 1, g_out); count *= d; }
    size_t es = dtype == 1 ? 4 : 8;
    if (count) fwrite(data, es, count, g_out);
}

void put_f64(const std::string& name, const std::vector<double>& v, std::vector<uint64_t> dims = {})
{
    if (dims.empty()) dims = {v.size()};
    put(name, 0, dims, v.data());
}

void put_i64(const std::string& name, const std::vector<int64_t>& v, std::vector<uint64_t> dims = {})
{
    if (dims.empty()) dims = {v.size()};
    put(name, 2, dims, v.data());
}

void put_ccsr(const std::string& name, const CCSRMat& m)
{
    long nnz = m.n > 0 ? m.row_ptr[m.n] : 0;
    put(name + ".row_ptr", 1, {(uint64_t)m.n + 1}, m.row_ptr);
    put(name + ".col", 1, {(uint64_t)nnz}, nnz ? (const void*)m.col_index : (const void*)"");
    put(name + ".val", 0, {(uint64_t)nnz, 9}, nnz ? (const void*)m.value : (const void*)"");
}

void put_mat(const std::string& name, const DynaMat& m)
{
    std::vector<double> v = {m.G, m.v, m.Rou, m.C1, m.C2, m.Dt, m.Dt2, m.Dt_2, m.Dt_3,
                             m.C1_2, m.C2_2, m.OneOverC1_2, m.OneOverC2_2, m.OneOverC1_3, m.OneOverC2_3,
                             m.C2_2OverC1_2, m.C2_2OverC1_3, m.C1Dt, m.C2Dt, m.OneOverFourPaiRou,
                             m.OneOverThree_1OC23_1OC13, m.Half_1OC22_1OC12, m.STCoef1, m.STCoef2};
    put_f64(name, v);
}

} // namespace

extern "C" int __wrap__Z30DynaGMRESSolverMultiDomainCCSRP14DSquareElementP13BoundaryValueRK16MultiDomainModelldlldPPlS7_(
    DSquareElement* elements, BoundaryValue* bd, const MultiDomainModel& model, long iterations, double error,
    long maxleafpointnum, long NStep, double MaxLength, long** infElePid, long** elePid)
{
    const long E = model.elementCount;
    const long D = model.DomainCount();
    const long I = (long)model.interfaces.size();

    put_i64("meta", {E, D, I, NStep, iterations, maxleafpointnum});
    put_f64("error", {error});
    put_f64("max_length", {MaxLength});
    for (long d = 0; d < D; ++d)
        put_mat("mat" + std::to_string(d), model.domains[(size_t)d].mat);
    std::vector<int64_t> itf;
    for (const InterfacePair& p : model.interfaces) {
        itf.push_back(p.domainA); itf.push_back(p.eleA); itf.push_back(p.domainB); itf.push_back(p.eleB);
        itf.push_back(p.normalSign);
    }
    put_i64("interfaces", itf, {(uint64_t)I, 5});

    std::vector<double> coef, center, radius, radiusPW, rcen, node, trans, u1, t1, t2;
    std::vector<int64_t> bcid, dom, surf, pts;
    for (long e = 0; e < E; ++e) {
        const DSquareElement& el = elements[e];
        for (int c = 0; c < 3; ++c) for (int j = 0; j < 8; ++j) coef.push_back(el.m_CoordCoef[c][j]);
        for (int c = 0; c < 3; ++c) center.push_back(el.m_center.pt[c]);
        radius.push_back(el.m_radius);
        radiusPW.push_back(el.m_radiusPW);
        for (int p = 0; p < NUMPW2; ++p) for (int c = 0; c < 3; ++c) rcen.push_back(el.m_rcenPW[p].pt[c]);
        for (int c = 0; c < 3; ++c) node.push_back(el.m_nodelist[el.m_nodeID[0]].pt[c]);
        for (int k = 0; k < 9; ++k) trans.push_back(DSquareElement::m_transmat[el.m_nodeID[0]][k]);
        for (int k = 0; k < 9; ++k) u1.push_back(el.m_OnElementU1ij[0][0][k]);
        for (int k = 0; k < 9; ++k) t1.push_back(el.m_OnElementT1ij[0][0][k]);
        for (int k = 0; k < 9; ++k) t2.push_back(el.m_OnElementT2ij[0][0][k]);
        bcid.push_back(el.BCID);
        dom.push_back(el.DomainID);
        surf.push_back(el.SurfaceType);
        for (int j = 0; j < 8; ++j) pts.push_back(el.m_pointID[j]);
    }
    put_f64("coordcoef", coef, {(uint64_t)E, 3, 8});
    put_f64("center", center, {(uint64_t)E, 3});
    put_f64("radius", radius);
    put_f64("radius_pw", radiusPW);
    put_f64("rcen_pw", rcen, {(uint64_t)E, NUMPW2, 3});
    put_f64("node", node, {(uint64_t)E, 3});
    put_f64("transmat", trans, {(uint64_t)E, 9});
    put_f64("on_u1", u1, {(uint64_t)E, 9});
    put_f64("on_t1", t1, {(uint64_t)E, 9});
    put_f64("on_t2", t2, {(uint64_t)E, 9});
    put_i64("bcid", bcid);
    put_i64("domain", dom);
    put_i64("surface", surf);
    put_i64("point_ids", pts, {(uint64_t)E, 8});

    // Matrices from the reference's serial assembly routines (the pthread
    // routines used by the solver are checked equal to these by the
    // reference itself when DBEM_MULTIDOMAIN_GMRES_PTHREAD_CHECK=1).
    GlobalDofMap dofMap;
    const char* want = getenv("TDBEM_DUMP_MATRICES");
    const bool matrices = !(want && atoi(want) == 0);
    const bool built = dofMap.Build(model, elements, E);
    if (built)
        put_i64("dof_counts", {dofMap.unknownBlockCount, dofMap.knownBlockCount, dofMap.historyUBlockCount,
                               dofMap.historyTBlockCount});
    if (built && matrices) {
        MultiDomainCCSRBuilder ub(dofMap.equationBlockCount, dofMap.unknownBlockCount);
        MultiDomainCCSRBuilder kb(dofMap.equationBlockCount, dofMap.knownBlockCount);
        if (AssembleMultiDomainStep0(elements, model, dofMap, infElePid, elePid, ub, kb)) {
            CCSRMat A, K;
            ub.Build(A);
            kb.Build(K);
            put_ccsr("A", A);
            put_ccsr("KnownM", K);
        }
        long kmax = NStep;
        const char* lim = getenv("TDBEM_DUMP_KMAX");
        if (lim && atol(lim) > 0 && atol(lim) < kmax) kmax = atol(lim);
        long lastNonEmpty = 0;
        for (long k = 1; k <= kmax; ++k) {
            MultiDomainCCSRBuilder mts(dofMap.equationBlockCount, dofMap.historyUBlockCount);
            MultiDomainCCSRBuilder mgs(dofMap.equationBlockCount, dofMap.historyTBlockCount);
            if (!AssembleMultiDomainHistoryStep(elements, model, dofMap, k, mts, mgs)) break;
            if (mts.NonZeroBlocks() == 0 && mgs.NonZeroBlocks() == 0) {
                if (k > lastNonEmpty + 3) break;   // the wave has left every domain
                continue;
            }
            lastNonEmpty = k;
            CCSRMat T, G;
            mts.Build(T);
            mgs.Build(G);
            put_ccsr("MTS" + std::to_string(k), T);
            put_ccsr("MGS" + std::to_string(k), G);
        }
        put_i64("history_last_nonempty", {lastNonEmpty});
    }
    fflush(g_out);

    int rc = __real__Z30DynaGMRESSolverMultiDomainCCSRP14DSquareElementP13BoundaryValueRK16MultiDomainModelldlldPPlS7_(
        elements, bd, model, iterations, error, maxleafpointnum, NStep, MaxLength, infElePid, elePid);

    std::vector<double> lu, lt;
    for (long s = 0; s <= NStep; ++s) {
        for (long i = 0; i < 3 * E; ++i) lu.push_back(bd[s].lu.b[i]);
        for (long i = 0; i < 3 * E; ++i) lt.push_back(bd[s].lt.b[i]);
    }
    put_f64("bd_lu", lu, {(uint64_t)NStep + 1, (uint64_t)(3 * E)});
    put_f64("bd_lt", lt, {(uint64_t)NStep + 1, (uint64_t)(3 * E)});
    put_i64("solver_return", {rc});
    put_i64("steps_recorded", {g_step});
    fclose(g_out);
    g_out = nullptr;
    return rc;
}

extern "C" int __wrap__Z5gmresP14DSquareElementR7CCSRMatR7WvectorR14PreConditionerldlS4_S4_RiPi(
    DSquareElement* elements, CCSRMat& A, Wvector& b, PreConditioner& pre, long restart, double tol, long maxit,
    Wvector& x0, Wvector& x, int& flag, int* iter)
{
    if (!g_preDumped) {
        g_preDumped = true;
        long P = A.n;
        // the legacy one-domain preconditioner (GMRESPreConditioner,
        // DBEM1/pre_gmres.cpp:635-720, taken when DomainCount == 1) leaves
        // the output ids unset: its columns are its rows' own points
        std::vector<int64_t> rep(pre.m_RePID, pre.m_RePID + P);
        std::vector<int64_t> outp = pre.m_OutputPID ? std::vector<int64_t>(pre.m_OutputPID, pre.m_OutputPID + P) : rep;
        std::vector<int64_t> lb(pre.m_LeafBeginID, pre.m_LeafBeginID + pre.m_LeafCount);
        std::vector<int64_t> lc(pre.m_LeafPointCount, pre.m_LeafPointCount + pre.m_LeafCount);
        put_i64("pre.repid", rep);
        put_i64("pre.outpid", outp);
        put_i64("pre.leaf_begin", lb);
        put_i64("pre.leaf_count", lc);
        std::vector<double> inv;
        for (long l = 0; l < pre.m_LeafCount; ++l)
            for (long i = 1; i <= pre.m_PreM[l].m; ++i)
                for (long j = 1; j <= pre.m_PreM[l].n; ++j) inv.push_back(pre.m_PreM[l](i, j));
        put_f64("pre.inverse", inv);
    }
    ++g_step;
    std::vector<double> rhs(b.b, b.b + b.n);
    put_f64("rhs" + std::to_string(g_step), rhs);
    int rc = __real__Z5gmresP14DSquareElementR7CCSRMatR7WvectorR14PreConditionerldlS4_S4_RiPi(
        elements, A, b, pre, restart, tol, maxit, x0, x, flag, iter);
    std::vector<double> sol(x.b, x.b + x.n);
    put_f64("x" + std::to_string(g_step), sol);
    put_i64("flag" + std::to_string(g_step), {flag, iter[0], iter[1]});
    return rc;
}

int main()
{
    return dbem_reference_main();
}
