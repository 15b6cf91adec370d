// The reference's multi-domain solver entry point over the B200 library.
//
//   int DynaGMRESSolverMultiDomainCCSR(DSquareElement* elements,
//       BoundaryValue* bd, const MultiDomainModel& model, long iterations,
//       double error, long maxleafpointnum, long NStep, double MaxLength,
//       long** infElePid, long** elePid)          (DBEM1/multidomain.h:214-223)
//
// Compiled together with the reference's own headers (dsquareelement.h,
// multidomain.h) and linked against libtdbem_b200.so and libcudart.  It
// marshals the reference's element and boundary objects into the flat
// tdbem_problem of include/tdbem.h, runs create / assemble / march on GPU 0
// in FP64, and writes the solved steps back into bd[0..NStep] in the global
// frame, as the reference's march does (DBEM1/multidomain.cpp:3819-3893).
// Return value: 1 when every step converged, -1 otherwise (the reference's
// convention); the library's message is printed on failure.
//
// With TDBEM_SHIM_DEFINE_ENTRY defined, the file also defines the entry
// point itself, for builds that drop the reference's definition
// (DBEM1/multidomain.cpp:3664-3926).
#include "dsquareelement.h"
#include "multidomain.h"
#include "tdbem.h"

#include <cmath>
#include <cstdio>
#include <vector>

int tdbem_legacy_solve(DSquareElement* elements, BoundaryValue* bd, const MultiDomainModel& model, long iterations,
                       double error, long maxleafpointnum, long NStep, double MaxLength)
{
    const long E = model.elementCount;
    // the 8 geometric nodes of each element, evaluated from its coordinate
    // coefficients at the natural coordinates of the reference's shape
    // functions (corners, then mid-sides; DBEM1/dsquareelement.h:270-295)
    static const double nat[8][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}, {0, -1}, {1, 0}, {0, 1}, {-1, 0}};
    std::vector<double> points((size_t)24 * E);
    std::vector<int64_t> ele((size_t)8 * E);
    std::vector<int32_t> bcid((size_t)E);
    double size_sum = 0.0;
    for (long i = 0; i < E; ++i) {
        for (int j = 0; j < 8; ++j) {
            const double s1 = nat[j][0], s2 = nat[j][1];
            const double basis[8] = {1.0, s1, s2, s1 * s2, s1 * s1, s2 * s2, s1 * s1 * s2, s1 * s2 * s2};
            for (int c = 0; c < 3; ++c) {
                double v = 0.0;
                for (int q = 0; q < 8; ++q) v += elements[i].m_CoordCoef[c][q] * basis[q];
                points[(size_t)(8 * i + j) * 3 + c] = v;
            }
            ele[(size_t)8 * i + j] = 8 * i + j;
        }
        const double* p0 = &points[(size_t)24 * i];
        const double* p1 = p0 + 3;
        size_sum += std::sqrt((p0[0] - p1[0]) * (p0[0] - p1[0]) + (p0[1] - p1[1]) * (p0[1] - p1[1]) +
                              (p0[2] - p1[2]) * (p0[2] - p1[2]));
        bcid[(size_t)i] = elements[i].BCID;
    }
    std::vector<double> mats;
    for (const Domain& d : model.domains) {
        mats.push_back(2.0 * d.mat.G * (1.0 + d.mat.v));  // E from the shear modulus
        mats.push_back(d.mat.v);
        mats.push_back(d.mat.Rou);
    }
    std::vector<int64_t> itf;
    for (const InterfacePair& p : model.interfaces) {
        itf.push_back(p.domainA);
        itf.push_back(p.eleA);
        itf.push_back(p.domainB);
        itf.push_back(p.eleB);
        itf.push_back(p.normalSign);
    }
    // the card material and its time step (DBEM1/DBEM.cpp:912-914): dt is
    // passed as the reference holds it, bit for bit; beta is given for
    // completeness (the library uses dt when it is set)
    const DynaMat& card = DSquareElement::m_DMat;
    tdbem_problem p{};
    p.n_points = 8 * E;
    p.points = points.data();
    p.n_elements = E;
    p.elements = ele.data();
    p.bcid = bcid.data();
    p.n_domains = (int32_t)model.domains.size();
    p.materials = mats.data();
    p.n_interfaces = (int64_t)model.interfaces.size();
    p.interfaces = itf.data();
    p.card_E = 2.0 * card.G * (1.0 + card.v);
    p.card_nu = card.v;
    p.card_rho = card.Rou;
    p.beta = card.Dt * card.C1 / (size_sum / (double)E);
    p.gap = DSquareElement::m_gap;
    p.n_steps = (int32_t)NStep;
    p.restart = (int32_t)iterations;
    p.tol = error;
    p.max_leaf = (int32_t)maxleafpointnum;
    p.max_length = MaxLength;
    p.precision = TDBEM_PRECISION_FP64;
    p.n_loads = 1;
    p.dt = card.Dt;

    tdbem_handle* h = nullptr;
    if (tdbem_md_create(&p, 0, &h) != TDBEM_OK) {
        std::printf("tdbem_md_create: %s\n", tdbem_last_error());
        return -1;
    }
    if (tdbem_md_assemble(h, nullptr) != TDBEM_OK) {
        std::printf("tdbem_md_assemble: %s\n", tdbem_last_error());
        tdbem_md_destroy(h);
        return -1;
    }
    // prescribed values are read from bd[n].lu at the element's node
    // (DBEM1/multidomain.cpp:3047-3084)
    const size_t per = (size_t)E * 3;
    std::vector<double> known((size_t)(NStep + 1) * per), lu(known.size()), lt(known.size());
    for (long n = 0; n <= NStep; ++n)
        for (long i = 0; i < E; ++i)
            for (int c = 0; c < 3; ++c)
                known[(size_t)n * per + 3 * i + c] = bd[n].lu.b[3 * elements[i].m_nodeID[0] + c];
    tdbem_report rep{};
    const tdbem_status st = tdbem_md_march(h, known.data(), lu.data(), lt.data(), &rep, nullptr);
    if (st != TDBEM_OK && st != TDBEM_NOT_CONVERGED) {
        std::printf("tdbem_md_march: %s\n", tdbem_last_error());
        tdbem_md_destroy(h);
        return -1;
    }
    // bd[0] (converted to the global frame) and every solved step
    const long solved = st == TDBEM_OK ? NStep : rep.steps_solved;
    for (long n = 0; n <= solved; ++n)
        for (long i = 0; i < E; ++i)
            for (int c = 0; c < 3; ++c) {
                const long node = elements[i].m_nodeID[0];
                bd[n].lu.b[3 * node + c] = lu[(size_t)n * per + 3 * i + c];
                bd[n].lt.b[3 * node + c] = lt[(size_t)n * per + 3 * i + c];
            }
    if (st != TDBEM_OK)
        std::printf("MultiDomain GMRES Solver: step %d did not converge (%s)\n", rep.failed_step, tdbem_last_error());
    tdbem_md_destroy(h);
    return st == TDBEM_OK ? 1 : -1;
}

#ifdef TDBEM_SHIM_DEFINE_ENTRY
int DynaGMRESSolverMultiDomainCCSR(DSquareElement* elements, BoundaryValue* bd, const MultiDomainModel& model,
                                   long iterations, double error, long maxleafpointnum, long NStep, double MaxLength,
                                   long** /*infElePid*/, long** /*elePid*/)
{
    return tdbem_legacy_solve(elements, bd, model, iterations, error, maxleafpointnum, NStep, MaxLength);
}
#endif
