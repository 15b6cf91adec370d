/*
 * TEST INFRASTRUCTURE ONLY -- the parity oracle, never linked into or called
 * by the product library.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load it.
 *
 * A plain-C, single-threaded restatement of the reference multi-domain TDBEM
 * time march (DynaGMRESSolverMultiDomainCCSR, DBEM1/multidomain.cpp:3664-3926)
 * for constant elements and the constant-velocity scheme (FlagDynaMethod 2):
 * element geometry, dynamic fundamental-solution quadrature, Step0 and
 * history assembly, GlobalDofMap numbering, block-CCSR building, the
 * mapped-leaf preconditioner, GMRES and the boundary write-back.
 * Parity is pinned against fixtures recorded from the reference itself
 * (tests/golden, made by tests/golden/make_golden.py).
 */
#ifndef TDBEM_ORACLE_H
#define TDBEM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_problem orc_problem;

/* Block-CCSR view (rows = equation blocks, 9 doubles per block, row-major
 * 3x3, column order ascending), owned by the problem. */
typedef struct {
    int64_t n_rows;
    int64_t nnz;
    const int32_t* row_ptr;
    const int32_t* col;
    const double* val;
} orc_ccsr;

/* points [P*3], elements [E*8] (0-based point ids), bcid [E] (123 or 456),
 * materials [D*3] (E, nu, rho), interfaces [I*5] (domainA, eleA, domainB,
 * eleB, normalSign; 0-based).  card_* is the global material that sets dt.
 * Returns NULL on invalid input (message in orc_last_error()). */
orc_problem* orc_create(int64_t n_points, const double* points, int64_t n_elements, const int64_t* elements,
                        const int32_t* bcid, int32_t n_domains, const double* materials,
                        int64_t n_interfaces, const int64_t* interfaces, double card_E, double card_nu,
                        double card_rho, double beta, double gap, int32_t n_steps, int32_t restart, double tol,
                        int32_t max_leaf, double max_length);
void orc_destroy(orc_problem* p);
const char* orc_last_error(void);

double orc_dt(const orc_problem* p);
/* dof counts: unknown, known, history */
void orc_dof_counts(const orc_problem* p, int64_t out[3]);

/* Per-element geometry as the reference stores it after GeoInit/PthPhyInit:
 * coordcoef [E*24], center [E*3], radius [E], radius_pw [E], rcen_pw
 * [E*36*3], transmat [E*9], on_u1/on_t1/on_t2 [E*9].  Any pointer may be NULL. */
void orc_geometry(const orc_problem* p, double* coordcoef, double* center, double* radius, double* radius_pw,
                  double* rcen_pw, double* transmat, double* on_u1, double* on_t1, double* on_t2);

/* Assemble Step0 (A, KnownM) and history steps 1..kmax (kmax <= 0: up to
 * orc_history_step_bound, keeping steps up to the last non-empty one).
 * Returns the number of history steps kept. */
int32_t orc_assemble(orc_problem* p, int32_t kmax);
/* Replay of builder calls: call i adds sign[i] * blocks[9 i..] (column-major)
 * at (row[i], col[i]) as MultiDomainCCSRBuilder::AddBlock; returns the stored
 * block count and fills row_ptr [rows + 1], col, val [nnz][9] when given. */
int64_t orc_builder_replay(int64_t rows, int64_t cols, int64_t n, const int64_t* row, const int64_t* col,
                           const double* sign, const double* blocks, int32_t* row_ptr, int32_t* col_out,
                           double* val_out);
/* Last history step whose blocks can be nonzero (the NeedCal skip rule). */
int32_t orc_history_step_bound(const orc_problem* p);
/* which: 0 = A, 1 = KnownM, 2 = MTS_k, 3 = MGS_k */
int32_t orc_matrix(const orc_problem* p, int32_t which, int32_t k, orc_ccsr* out);

/* Mapped-leaf preconditioner layout (after orc_assemble): repid [nb],
 * leaf_begin/leaf_count [n_leaves]; returns n_leaves. */
int64_t orc_precond_layout(const orc_problem* p, int64_t* repid, int64_t* leaf_begin, int64_t* leaf_count);

/* Run the march for one load case.  known: [(n_steps+1)*E*3] element-local
 * prescribed values (bd[n].lu as read from the .bd file).  Outputs
 * bd_lu/bd_lt: [(n_steps+1)*E*3] global-frame values as the reference leaves
 * them; rhs/x (may be NULL): [n_steps*3*nb]; flags (may be NULL):
 * [n_steps*3] = gmres flag, outer, inner.  Returns the number of steps solved
 * (the march stops at the first non-converged step, like the reference). */
int32_t orc_march(orc_problem* p, const double* known, double* bd_lu, double* bd_lt, double* rhs, double* x,
                  int32_t* flags);

#ifdef __cplusplus
}
#endif
#endif
