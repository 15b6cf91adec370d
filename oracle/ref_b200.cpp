// The reference driver with its multi-domain solver replaced by the B200
// library through the legacy-signature shim (test infrastructure only).
//
// Linked against the unchanged reference objects, including its main(); the
// linker wraps DynaGMRESSolverMultiDomainCCSR (DBEM1/multidomain.h:214-223)
// so the reference's own input readers, element set-up and datacard handling
// run as usual and only the solver call goes to tdbem_legacy_solve
// (parallel3.0_omp_multidomin_1node_b200/shim/tdbem_legacy_shim.cpp).  After
// it returns, bd[0..NStep] are written to the file named by TDBEM_BD_OUT
// (default bd_b200.bin): int64 NStep, int64 node count, int32 return value,
// then per step lu[3*nodes] and lt[3*nodes] as float64.

#include "multidomain.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>

int tdbem_legacy_solve(DSquareElement* elements, BoundaryValue* bd, const MultiDomainModel& model, long iterations,
                       double error, long maxleafpointnum, long NStep, double MaxLength);

extern "C" int __wrap__Z30DynaGMRESSolverMultiDomainCCSRP14DSquareElementP13BoundaryValueRK16MultiDomainModelldlldPPlS7_(
    DSquareElement* elements, BoundaryValue* bd, const MultiDomainModel& model, long iterations, double error,
    long maxleafpointnum, long NStep, double MaxLength, long** /*infElePid*/, long** /*elePid*/)
{
    const int rc = tdbem_legacy_solve(elements, bd, model, iterations, error, maxleafpointnum, NStep, MaxLength);
    const char* path = getenv("TDBEM_BD_OUT");
    FILE* f = fopen(path ? path : "bd_b200.bin", "wb");
    if (!f) {
        perror("TDBEM_BD_OUT");
        exit(3);
    }
    const int64_t n = NStep, nodes = model.nodeCount;
    const int32_t r = rc;
    fwrite(&n, 8, 1, f);
    fwrite(&nodes, 8, 1, f);
    fwrite(&r, 4, 1, f);
    for (long s = 0; s <= NStep; ++s) {
        fwrite(bd[s].lu.b, sizeof(double), (size_t)(3 * nodes), f);
        fwrite(bd[s].lt.b, sizeof(double), (size_t)(3 * nodes), f);
    }
    fclose(f);
    return rc;
}
