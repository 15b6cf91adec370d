/*
 * tdbem.h -- C ABI of the B200-native multi-domain TDBEM time march.
 *
 * One handle holds one multi-domain model on one GPU: element geometry,
 * per-domain materials, the GlobalDofMap numbering, the assembled block-CCSR
 * matrices (A, KnownM, history MTS_k / MGS_k) and the mapped-leaf
 * preconditioner, all resident in device memory.  Host buffers are owned by
 * the caller; device memory is owned by the library.  Every call that does
 * GPU work takes a cudaStream_t (passed as void*, NULL = default stream).
 * A handle is used by one host thread at a time.
 *
 * The entry points replace the reference's
 *   int DynaGMRESSolverMultiDomainCCSR(DSquareElement* elements,
 *       BoundaryValue* bd, const MultiDomainModel& model, long iterations,
 *       double error, long maxleafpointnum, long NStep, double MaxLength,
 *       long** infElePid, long** elePid)        (DBEM1/multidomain.h:214-223)
 * split into create (model + DOF map, DBEM1/multidomain.cpp:3664-3710),
 * assemble (Step0 + history + preconditioner, :3742-3809) and march
 * (the time loop, :3811-3893).  A C++ shim with the legacy signature
 * marshals DSquareElement / BoundaryValue into tdbem_problem and the known
 * values, calls these three, and copies out_lu / out_lt back into bd.
 */
#ifndef TDBEM_H
#define TDBEM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TDBEM_ABI_VERSION 3

typedef enum {
    TDBEM_OK = 0,
    TDBEM_INVALID_INPUT = 1,   /* bad sizes, BCID other than 123/456, bad interface */
    TDBEM_DOFMAP_INVALID = 2,  /* GlobalDofMap::Build/Validate failure */
    TDBEM_SINGULAR_BLOCK = 3,  /* a preconditioner leaf block could not be inverted */
    TDBEM_NOT_CONVERGED = 4,   /* GMRES flag != 0 at report.failed_step */
    TDBEM_CUDA_ERROR = 5,
    TDBEM_OUT_OF_MEMORY = 6,
    TDBEM_NOT_ASSEMBLED = 7    /* march before assemble / load_matrices */
} tdbem_status;

typedef enum {
    TDBEM_PRECISION_FP64 = 0,  /* reference arithmetic: FP64 everywhere */
    TDBEM_PRECISION_MIXED = 1  /* FP32 history blocks + FP32 Krylov SpMV in FP64 refinement */
} tdbem_precision;

typedef struct {
    int64_t n_points;
    const double* points;       /* [n_points*3] */
    int64_t n_elements;
    const int64_t* elements;    /* [n_elements*8] 0-based point ids, corners then mid-sides */
    const int32_t* bcid;        /* [n_elements] 123 or 456 */
    int32_t n_domains;          /* elements split into contiguous equal ranges */
    const double* materials;    /* [n_domains*3] E, nu, rho */
    int64_t n_interfaces;
    const int64_t* interfaces;  /* [n_interfaces*5] domainA, eleA, domainB, eleB, normalSign (0-based) */
    double card_E, card_nu, card_rho; /* global card material: sets dt */
    double beta;                /* dt = beta * mean|P0-P1| / c1(card) */
    double gap;                 /* discontinuous-element node offset (datacard gap) */
    int32_t n_steps;            /* NStep */
    int32_t restart;            /* GMRES restart = datacard iterations */
    double tol;                 /* GMRES relative tolerance = datacard error */
    int32_t max_leaf;           /* preconditioner leaf size = premaxleafpointnum */
    double max_length;          /* MaxLength (1000 in the reference driver) */
    int32_t precision;          /* tdbem_precision */
    int32_t n_loads;            /* R load cases marched together (>= 1) */
    double dt;                  /* > 0: the time step as the caller holds it (the reference's
                                   card DynaMat Dt, DBEM1/DBEM.cpp:912-914), used as given;
                                   0: dt = beta * mean|P0-P1| / c1(card) */
} tdbem_problem;

typedef struct {
    int32_t steps_solved;       /* steps completed (== n_steps on success) */
    int32_t failed_step;        /* first step whose GMRES did not converge, or 0 */
    int32_t gmres_flag;         /* last flag: 0 converged, 1 not converged, 3 stagnation */
    int64_t total_inner;        /* GMRES inner iterations summed over steps and loads */
    int32_t max_refinements;    /* mixed precision: most refinement cycles in one step */
    int32_t history_steps;      /* active history steps K (matrices MTS_1..MTS_K) */
    int64_t history_blocks;     /* nonzero 3x3 blocks in all MTS_k and MGS_k */
    int64_t a_blocks;           /* nonzero blocks in A */
    double max_interface_jump;  /* max |uA - uB| over interface pairs and steps */
    double max_interface_balance; /* max |tB - s tA| over interface pairs and steps */
    double rhs_bytes;           /* algorithmic bytes moved by the right-hand-side kernel over the march */
    double ms_rhs;              /* device time in the history right-hand side */
    double ms_gmres;            /* device time in GMRES + write-back */
    double ms_total;            /* device time of the march */
    int32_t gmres_cluster;      /* CTAs of each thread-block cluster running GMRES */
    int32_t gmres_groups;       /* clusters (load-case groups) running GMRES side by side */
    double rhs_block_reads;     /* 3x3 history blocks applied by the right-hand-side kernel over the march
                                   (each to all load cases) */
    int32_t history_launches;   /* history passes launched beside GMRES over the march: steps k >= 3 of
                                   one time step, or k >= 2T + 1 of T time steps from the run layout
                                   (two or more load cases; T = 2 by default) */
    double ms_history;          /* device time of those passes (part of ms_rhs) */
    double history_bytes;       /* their algorithmic bytes (part of rhs_bytes) */
    double history_block_steps; /* their block applications, one per block and time step (part of
                                   rhs_block_reads) */
    double history_vector_loads; /* combined history vectors (3 x n_loads FP64) they load: one per block
                                    in the one-step pass, one per block plus T - 1 per run in the T-step pass */
} tdbem_report;

typedef struct tdbem_handle tdbem_handle;

/* Launch configuration chosen by tdbem_md_autotune. */
typedef struct {
    int32_t gmres_groups;          /* GMRES thread-block clusters side by side (load-case groups) */
    int32_t gmres_cluster;         /* CTAs per cluster */
    int32_t rhs_cases_per_thread;  /* history pass R-tile; a warp takes 32 / (R / this) block rows per iteration */
    int32_t candidates;            /* configurations timed */
    int32_t steps;                 /* time steps each timing marched */
    double ms_per_step;            /* device time per step of the chosen configuration */
    double ms_per_step_default;    /* the same for the configuration the handle had before */
} tdbem_tuning;

const char* tdbem_status_string(tdbem_status s);
/* Last error message of the calling thread (empty when none). */
const char* tdbem_last_error(void);
int32_t tdbem_abi_version(void);

/* Validate the model, build element geometry and singular self-element
 * integrals on the GPU, and number the unknowns like GlobalDofMap::Build
 * (DBEM1/multidomain.cpp:777-900).  Copies every input array. */
tdbem_status tdbem_md_create(const tdbem_problem* problem, int32_t device, tdbem_handle** out);
void tdbem_md_destroy(tdbem_handle* h);

/* Dynamic fundamental-solution quadrature for Step0 (A, KnownM) and history
 * steps 1..K on the GPU (AssembleMultiDomainStep0 / HistoryStep,
 * DBEM1/multidomain.cpp:2256-2378), block-CCSR build, and the mapped-leaf
 * preconditioner (DBEM1/multidomain.cpp:3493-3565). */
tdbem_status tdbem_md_assemble(tdbem_handle* h, void* stream);

/* Load already-assembled matrices (reference block-CCSR layout, 9 doubles
 * per block row-major, ascending columns) instead of assembling: the
 * matrix-cache path.  hist_rowptr: [K*(E+1)], hist_col/hist_val: the K
 * matrices concatenated (MTS_1..MTS_K, resp. MGS_1..MGS_K). */
tdbem_status tdbem_md_load_matrices(tdbem_handle* h, const int32_t* a_rowptr, const int32_t* a_col,
                                    const double* a_val, const int32_t* k_rowptr, const int32_t* k_col,
                                    const double* k_val, int32_t n_hist, const int32_t* mts_rowptr,
                                    const int32_t* mts_col, const double* mts_val, const int32_t* mgs_rowptr,
                                    const int32_t* mgs_col, const double* mgs_val, void* stream);

/* Time march from host buffers (copies in and out inside the call).
 * known_lu: [n_loads][n_steps+1][n_elements][3] prescribed element-local
 * values (bd[n].lu as the .bd file gives them).  out_lu/out_lt (may be
 * NULL): [n_loads][n_steps+1][n_elements][3], the reference's final bd[n].lu
 * and bd[n].lt (global frame).  Returns TDBEM_NOT_CONVERGED with
 * report->failed_step set when a step's GMRES fails, like the reference's
 * march, which stops there.  With page-locked (pinned) host buffers the
 * copies run beside the march, chunk by chunk of steps; with pageable
 * buffers they are whole copies before and after it.  Device pointers are
 * accepted too (copied device to device). */
tdbem_status tdbem_md_march(tdbem_handle* h, const double* known_lu, double* out_lu, double* out_lt,
                            tdbem_report* report, void* stream);

/* Same, with device-resident buffers of the same shapes (no host copies). */
tdbem_status tdbem_md_march_device(tdbem_handle* h, const double* d_known_lu, double* d_out_lu,
                                   double* d_out_lt, tdbem_report* report, void* stream);

/* Several independent models marched together: the same as one
 * tdbem_md_march_device per handle, with the time steps of all handles
 * enqueued in turn on each handle's own streams, so the models' kernels run
 * side by side (models of different sizes and step counts; no counterpart in
 * the reference, which solves one model per run).  Handle i takes its own
 * device buffers d_known_lu[i], d_out_lu[i], d_out_lt[i] and fills
 * reports[i]; the first failure's status is returned.  A handle may appear
 * only once. */
tdbem_status tdbem_md_march_many(tdbem_handle* const* handles, int32_t n, const double* const* d_known_lu,
                                 double* const* d_out_lu, double* const* d_out_lt, tdbem_report* reports,
                                 void* stream);

/* Adjoint march (vector-Jacobian product) of a one-load FP64 handle: given
 * the cotangents of the march outputs, cot_lu and cot_lt ([n_steps+1]
 * [n_elements][3], global frame; either may be NULL for zero), returns in
 * grad_known the gradient with respect to the prescribed values known_lu
 * ([n_steps+1][n_elements][3], element-local as the march takes them).  The
 * march is linear in known_lu, so the product needs no saved forward state:
 * it runs the time march in reverse with A^T solves (the GMRES kernel on
 * the transposed permuted system with transposed leaf inverses) and the
 * transposed history convolution.  No counterpart in the reference.
 * report: steps_solved, total_inner, failed_step / gmres_flag of the solves.
 * For a sensor misfit J = sum_n sum_s |u_n(e_s) - obs|^2 pass
 * cot_lu = 2 (u - obs) at the sensors and 0 elsewhere. */
tdbem_status tdbem_md_march_vjp(tdbem_handle* h, const double* cot_lu, const double* cot_lt, double* grad_known,
                                tdbem_report* report, void* stream);

/* Forward/backward pair with saved state, for gradients with respect to the
 * domains' materials as well as the loads (no counterpart in the reference).
 * tdbem_md_march_forward is tdbem_md_march on a one-load handle that also
 * keeps on the device what the backward needs: the unknowns of every step,
 * the prescribed values and the boundary values.  Any later march of the
 * handle discards that state.
 * tdbem_md_march_backward then takes the cotangents as tdbem_md_march_vjp
 * does and returns grad_known as it does, plus (if grad_material is not
 * NULL) grad_material [n_domains][2] = dJ/dE_d, dJ/drho_d of
 * J = <cot_lu, out_lu> + <cot_lt, out_lt>.  Each domain's Young's modulus
 * and density enter through its wave speeds and the displacement kernel's
 * 1/rho; the Poisson ratio and dt (set by the card material) are held fixed.
 * The derivative blocks dA/dtheta, dKnownM/dtheta, dMTS_k/dtheta and
 * dMGS_k/dtheta are recomputed by the quadrature kernels in forward-mode
 * form and contracted at once with the adjoint vectors and the saved states
 * (sum_n lam_n^T (db_n/dtheta - dA/dtheta x_n)); none is stored.  Wave-front
 * windows and quadrature-rule choices are taken at the given materials, so
 * the result is the derivative of the piece of the discrete model the
 * materials sit on.  Fails with TDBEM_INVALID_INPUT when the last march of
 * the handle was not tdbem_md_march_forward.  known_lu, out_lu, out_lt,
 * cot_lu, cot_lt and grad_known may be host or device pointers;
 * grad_material is a host array. */
tdbem_status tdbem_md_march_forward(tdbem_handle* h, const double* known_lu, double* out_lu, double* out_lt,
                                    tdbem_report* report, void* stream);
tdbem_status tdbem_md_march_backward(tdbem_handle* h, const double* cot_lu, const double* cot_lt, double* grad_known,
                                     double* grad_material, tdbem_report* report, void* stream);

/* Launch-configuration autotuner (no counterpart in the reference, whose
 * CPU solver has no launch parameters): times marches of the first `steps`
 * time steps of known_lu (host, laid out as for tdbem_md_march) under
 * candidate configurations and keeps the fastest on the handle for its
 * later marches.  Stage 1 tries every power-of-two number of GMRES
 * load-case groups with the three largest schedulable cluster sizes;
 * stage 2 the history pass's load cases per thread (4 or 2 for R >= 4, 2 or
 * 1 for R = 2) at the best GMRES layout.  Each timing is a device-timed march
 * after a three-step warm-up.  The configuration the handle had (the set-up
 * heuristic) is timed first and kept unless a candidate is faster.  Choose
 * `steps` of at least the history length (report.history_steps) so the
 * timed steps carry the full history pass.  Results of later marches differ
 * from those of the default configuration by rounding only. */
tdbem_status tdbem_md_autotune(tdbem_handle* h, const double* known_lu, int32_t steps, tdbem_tuning* out,
                               void* stream);

/* Per-step diagnostics of the last march, load case 0, host buffers of
 * [n_steps][3*n_elements] (rhs in equation-row order, x in unknown order)
 * and [n_steps][3] (flag, refinements, inner iterations).  Any may be NULL.
 * Only recorded when tdbem_md_set_record(h, 1) preceded the march. */
tdbem_status tdbem_md_set_record(tdbem_handle* h, int32_t on);
tdbem_status tdbem_md_step_record(tdbem_handle* h, double* rhs, double* x, int32_t* flags);

/* Export an assembled matrix in the reference's block-CCSR layout.
 * which: 0 = A, 1 = KnownM, 2 = MTS_k, 3 = MGS_k (k in 1..history_steps).
 * Call with NULL arrays to get n_rows / nnz; then with buffers of
 * n_rows+1, nnz and 9*nnz entries. */
tdbem_status tdbem_md_export_matrix(tdbem_handle* h, int32_t which, int32_t k, int64_t* n_rows, int64_t* nnz,
                                    int32_t* row_ptr, int32_t* col, double* val);

/* Element geometry as the reference stores it (see orc_geometry in the
 * oracle): coordcoef [E*24], center [E*3], radius, radius_pw [E],
 * transmat [E*9], on_u1/on_t1/on_t2 [E*9].  Any pointer may be NULL. */
tdbem_status tdbem_md_geometry(tdbem_handle* h, double* coordcoef, double* center, double* radius,
                               double* radius_pw, double* transmat, double* on_u1, double* on_t1, double* on_t2);

/* Model facts: dt, unknown/known/history block counts, leaves. */
tdbem_status tdbem_md_info(tdbem_handle* h, double* dt, int64_t* n_unknown, int64_t* n_known, int64_t* n_history,
                           int64_t* n_leaves);

/* Preconditioner layout: repid [E] (leaf-order point ids), leaf_begin and
 * leaf_count [n_leaves]. */
tdbem_status tdbem_md_precond_layout(tdbem_handle* h, int64_t* repid, int64_t* leaf_begin, int64_t* leaf_count);

/* Matrix cache file: save the assembled A, KnownM, MTS_k and MGS_k of a
 * handle, and load them into a later handle of the same model instead of
 * assembling (the reference's matrix cache, gmres_ccsr_cache.bin of its
 * single-domain path, DBEM1/pre_gmres.cpp:16-545, extended to the
 * multi-domain matrices).  Each matrix is stored in the layout of
 * CCSRMat::WriteBinary (DBEM1/mat_vec.cpp:1690-1707) with 64-bit counts; the
 * header holds the counts, NStep and a fingerprint of the model (geometry,
 * BCIDs, domains, materials, interfaces, dt, gap), and loading into a
 * different model fails with TDBEM_INVALID_INPUT and the reason. */
tdbem_status tdbem_md_save_matrices(tdbem_handle* h, const char* path);
tdbem_status tdbem_md_load_matrix_cache(tdbem_handle* h, const char* path, void* stream);

/* Validation output of one load case of the last march in the reference's
 * formats (WriteValidationOutputs, DBEM1/DBEM.cpp:434-561, with the
 * multi-domain metrics of DBEM1/multidomain.cpp:387-416 and the structure
 * diagnosis of A, :3314-3420): <directory>/validation_state.csv and
 * <directory>/validation_metrics.txt, same columns and keys, and the
 * per-step interface audit <directory>/interface_transfer_audit.csv
 * (WriteInterfaceTransferAuditCsv, DBEM1/multidomain.cpp:329-379; appended
 * to, with the header written when the file is new, as the reference does).
 * out_lu / out_lt and report are the march's outputs (host buffers, all load
 * cases). */
tdbem_status tdbem_md_write_validation(tdbem_handle* h, const char* directory, int32_t load, const double* out_lu,
                                       const double* out_lt, const tdbem_report* report);

/* Right-hand-side diagnostics of every solved step of load case 0 of the
 * last march (WriteRhsBreakdownCsv, DBEM1/multidomain.cpp:247-327, written by
 * the reference when DBEM_RHS_DIAGNOSTIC=1): <directory>/rhs_breakdown.csv
 * (per equation row and component: the KnownM part, the MGS and -MTS history
 * parts, the total right-hand side, A x, A x - rhs and the solution column as
 * the reference prints it) and <directory>/residual_probe.csv (per step: max
 * and l2 residual, l2 rhs, relative residual), appended to like the
 * reference's.  The parts are recomputed on the device in FP64 from the
 * march's saved states.  Needs a recorded host march: tdbem_md_set_record(h,
 * 1) before tdbem_md_march, or tdbem_md_march_forward; otherwise
 * TDBEM_INVALID_INPUT.  report: that march's report. */
tdbem_status tdbem_md_write_rhs_diagnostics(tdbem_handle* h, const char* directory, const tdbem_report* report);

/* ---- Reference input files ------------------------------------------
 * Read a reference case directory the way the reference driver does:
 * BEM_DATACARD.DAT (the GMRES solver card, solvers = 2, with the optional
 * multi-domain tail of domain materials and interface pairs;
 * DBEM1/DBEM.cpp:637-791, DBEM1/multidomain.cpp:1305-1362, 1363-1477) and
 * input/<title>.model and input/<title>.bd as text or, by the card's input
 * mode, in the DBEMBIN binary form <file>.bin (DBEM1/DBEM.cpp:89-343,
 * 826-1085).  The card's batch boundary modes 1 and 2 name one boundary
 * file per load case; they become the case's load cases (n_loads), where
 * the reference's multi-domain path refuses them (DBEM1/DBEM.cpp:1226-1231).
 * Domain materials not on the card default to the card material; interface
 * and material ids may be 0- or 1-based as the reference accepts. */
typedef struct tdbem_case tdbem_case;
tdbem_status tdbem_case_read(const char* directory, tdbem_case** out);
/* The problem for tdbem_md_create: pointers into the case (valid until
 * tdbem_case_destroy), precision FP64, n_loads = the case's load cases,
 * max_length 1000 as the reference driver passes. */
tdbem_status tdbem_case_problem(const tdbem_case* c, tdbem_problem* problem);
/* Prescribed values bd[n].lu of every load case: [n_loads][n_steps+1][n_elements][3]. */
tdbem_status tdbem_case_known(const tdbem_case* c, double* known);
const char* tdbem_case_title(const tdbem_case* c);
void tdbem_case_destroy(tdbem_case* c);

/* Solve without device allocation.  This entry point has no counterpart in
 * the reference; it exists for callers that must not allocate device memory
 * while they run.  cudaMalloc and cudaFree may synchronise the whole device,
 * stalling the work such a caller keeps in flight on other streams, and they
 * fail once another allocator (a framework's caching pool, say) has reserved
 * the free memory; a solver called from inside such a loop needs its storage
 * to exist before the loop starts.
 *
 * It performs one FP64 GMRES solve A x = rhs for a single load case on an
 * assembled handle, with the kernel, preconditioner, restart and tolerance of
 * a march step (FP64 whatever the handle's precision).  All working storage
 * comes from one 32 MiB array the library declares in device memory; the
 * call enqueues a memset, three kernels and, with flags, one 12-byte copy,
 * and calls no allocating routine.
 *   rhs: device [3*n_elements] doubles in equation-row order (the order of
 *        the rhs tdbem_md_step_record returns);
 *   x:   device [3*n_elements] doubles, written in unknown order;
 *   flags: optional host int32[3] (GMRES flag, refinements, inner
 *        iterations).  Given, the call waits for the stream and returns
 *        TDBEM_NOT_CONVERGED on a nonzero flag; NULL, it returns TDBEM_OK
 *        once the work is enqueued, and a solve that does not converge is
 *        not reported (x then holds GMRES's last iterate): a caller that
 *        cannot wait must check the solution itself.
 * Limit: the solve needs 8 * ((15 + 9 * (restart + 1)) * E
 * + 5 * C * (restart + 2) + 32) bytes plus alignment (C = the handle's GMRES
 * cluster size), about 14,000 elements at restart 30.  Larger problems are
 * rejected with TDBEM_INVALID_INPUT and a message giving the bytes needed.
 * The first call on each device sets up, with that device current, the
 * array's address and the cluster size the kernel can be scheduled with;
 * make that first call before any stream capture begins.  One array serves
 * every handle of a device, so calls that overlap in time on one device
 * (from any handle, stream or thread) race on it: serialise them. */
tdbem_status tdbem_md_solve_noalloc(tdbem_handle* h, const double* rhs, double* x, int32_t* flags, void* stream);

#ifdef __cplusplus
}
#endif
#endif
