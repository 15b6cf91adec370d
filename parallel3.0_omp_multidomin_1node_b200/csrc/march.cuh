// Time-march kernels: history right-hand side (batched over load cases),
// cluster-resident GMRES and the boundary write-back (host-side launch
// wrappers).
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

namespace tdbem {

// Everything the per-step kernels read or write, all device pointers.
// Index spaces: "perm" = leaf order of the mapped-leaf preconditioner
// (row p is equation row row_of[p]; unknown p is unknown block
// unk_of[p] = preferred unknown of row_of[p]), so the preconditioner is
// block diagonal and every GMRES CTA owns one contiguous perm range.
// Vectors over the 3E unknowns are stored [3E][R], load case fastest.
struct MarchData {
    int E;            // elements = equation rows = unknown blocks
    int n_known;      // known blocks
    int nh;           // history blocks
    int K;            // history steps
    int R;            // load cases
    int nstep;
    int SW;           // W-ring slots (K + 1)
    int mixed;        // FP32 history + mixed-precision GMRES
    int k_lo, k_hi;   // right-hand side split: k in [k_lo, k_hi] (see march_step)
    // stacked history matrix: per equation row, blocks of k = 1..K, each k
    // with MGS_k (type 1, traction history) then MTS_k (type 0, negated)
    const int64_t* h_kptr;  // [E][K+1]: entry k = first block with step > k; entry 0 = row start
    const uint32_t* h_col;  // packed (k << 21) | (type << 20) | history column
    const double* h_val;    // SoA [9][nnz]
    const float* h_val32;   // SoA [9][nnz] (mixed)
    int64_t h_nnz;
    // run layout of the blocks of steps k >= kr = 2T + 1, for the T-step
    // history pass: per equation row, runs of one (type, column) pair over
    // consecutive steps, longest first; kr = 0 when there is none
    const int64_t* r_ptr;   // [E+1] first run of each equation row
    const uint2* r_meta;    // x = (type << 20) | column, y = (first step << 16) | length
    const int64_t* r_off;   // block of the run's first step in r_val / r_val32
    const double* r_val;    // SoA [9][r_nb] (FP64 mode)
    const float* r_val32;   // SoA [9][r_nb] (mixed)
    int64_t r_nb;
    int kr;
    // KnownM (natural rows), known blocks map to (element, sign)
    const int32_t* k_rp;
    const int32_t* k_col;
    const double* k_val;    // [nnz][9]
    const int32_t* known_elem;
    const double* known_sign;
    const int32_t* k_elem;  // per KnownM block: known_elem of its column
    const double* k_sgn;    // per KnownM block: known_sign of its column
    // permuted system matrix A' and preconditioner
    const int32_t* a_rp;
    const int32_t* a_col;
    const double* a_val;    // [nnz][9]
    const float* a_val32;
    const int32_t* row_of;  // perm -> equation row
    const int32_t* perm_of_unk; // unknown block -> perm
    const int32_t* leaf_begin;
    const int32_t* leaf_count;
    const int32_t* leaf_of_perm;  // perm index -> leaf
    const int64_t* leaf_off;  // offset of each leaf's dense inverse
    const double* pinv;       // dense (3L x 3L) leaf inverses, row-major
    const float* pinv32;
    const int32_t* cta_leaf;  // [C+1] leaf range per GMRES CTA of the cluster
    // A' columns as (owner CTA rank << 24) | row within the owner's range,
    // for Krylov vectors read from the cluster's shared memory
    const int32_t* a_colx;
    int dsm_rows;             // rows of the largest owned range; 0 = vectors read from global memory
    // per-element write-back data
    const int64_t* uref_block; const double* uref_sign; const int32_t* uref_known;
    const int64_t* tref_block; const double* tref_sign; const int32_t* tref_known;
    const int64_t* hist_block; const double* hu_sign; const double* ht_sign;
    const int32_t* hist_owner;  // 1 when the element feeds the history state (not an interface B side)
    const double* itf_trans;    // [E][9] local transform of interface B sides (identity elsewhere)
    const double* trans;        // [E][9] element frames
    const int32_t* bcid;
    const int32_t* itf_pairs;   // [I][2] eleA, eleB
    const double* itf_sign;     // [I]
    int n_itf;
    // state
    double* xring;    // [3][2][nh][3][R] physical history states X_s (type 0 = U, 1 = T)
    double* wring;    // [SW][2][nh][3][R] combined history vectors
    double* bulk;     // [8][3E][R] part of the right-hand side of step s at s % 8 computed
                      // ahead beside GMRES: history k >= 3 (k >= kr with the run layout), KnownM
    double* b;        // [3E][R] perm right-hand side
    // GMRES: `groups` clusters, cluster g solves load cases [g*Rg, (g+1)*Rg)
    // with private Krylov storage ([3E][Rg] per vector) at offset g
    int groups;
    double* bp;       // [groups][3E][Rg] right-hand side copy
    double* x;        // [groups][3E][Rg] perm solution
    double* xold;     // [groups][3E][Rg] solution of the step before (mixed-mode start vector), or null
    double* rv;       // [groups][3E][Rg] residual
    double* u;        // [groups][3E][Rg] Arnoldi work vector
    double* V;        // [groups][restart+1][3E][Rg]
    double* W;        // [groups][restart+1][3E][Rg] (last column keeps the refinement start x)
    double* AW;       // [groups][restart+1][3E][Rg] A W_j (mixed: residual recurrence)
    double* givens;   // [groups][C][Rg] cs, sn, h, rcol, c ([restart+2] each, kGivensArrays)
    int* status;      // [0] abort
    int* step_flags;  // [nstep][R][3] flag, refinements, inner iterations
    double* audit;    // [nstep][2] max interface jump, balance
    const double* known_lu; // [R][nstep+1][E][3] device input
    double* out_lu;          // [R][nstep+1][E][3]
    double* out_lt;
    double* rec_rhs;         // optional [nstep][E*3] (load 0, natural row order)
    double* rec_x;           // optional [nstep][E*3] (load 0, natural unknown order)
    int restart;
    double tol;
    int cluster;             // CTAs in the GMRES cluster
    int rhs_cpt;             // history pass: load cases per thread (0 = default: min(R, 4))
    int64_t givens_stride;   // doubles per (CTA, case) in givens
    int solve_only;          // 1: GMRES alone, no write-back, history update or audit (bare solve)
};

// Arrays of restart+2 doubles per (GMRES CTA, load case) in MarchData::givens:
// rotation cosines and sines, the Hessenberg column, its rotated copy and the
// second Gram-Schmidt pass's coefficients.
constexpr int kGivensArrays = 5;

// Run layout of the stacked history blocks of steps k >= kr (MarchData r_*),
// built on the device from the stacked arrays (kptr on the host and the
// device, packed columns, values FP32 when mixed, else FP64).  The arrays are
// the caller's (cudaFree each); kr = 0 on return when there is nothing to
// lay out or the sizes exceed the 32-bit sort indices.
struct HistoryRuns {
    int64_t* ptr = nullptr;   // [E+1]
    uint2* meta = nullptr;    // [runs]
    int64_t* off = nullptr;   // [runs]
    void* val = nullptr;      // SoA [9][nb]
    int64_t nb = 0, runs = 0;
    int kr = 0;
};
cudaError_t build_history_runs(int E, int K, int kr, const std::vector<int64_t>& kptr, const int64_t* d_kptr,
                               const uint32_t* d_col, const void* d_val, int64_t nnz, bool mixed, HistoryRuns& out,
                               cudaStream_t s);
// Device memory the build takes at most for nb blocks (outputs included).
size_t history_runs_bytes(int64_t nb, bool mixed);

// Sizes of the R template instantiations.
bool march_supported_loads(int R);
cudaError_t march_prepare(const MarchData& d, cudaStream_t s);
// One time step.  With `overlap`, the history part k >= 3 of step+1 is
// launched on `side` concurrently with this step's GMRES (it only needs
// states up to step-1), and this step's right-hand side adds the part
// computed during the previous step.  With the run layout (d.kr = 2T + 1,
// T = 2 or 3) steps 2, 2 + T, 2 + 2T, ... instead launch the part k >= kr of
// the T steps step+T .. step+2T-1 in one pass (it needs states up to step-1
// as well and has the GMRES of step .. step+T-1 to run beside), and the head
// covers k < kr.
// Events of one step: head0/head1 bracket the right-hand-side kernel on the
// chain stream, gm0/gm1 the GMRES kernel, bulk0/bulk1 the overlapped bulk
// kernel on the side stream; sync orders a later head after the bulk;
// prev_gm is gm1 of the previous step (the side stream waits on it);
// prev_pass is sync of step-T (the first step a T-step pass covers waits on
// it).
struct StepEvents {
    cudaEvent_t head0, head1, gm0, gm1, bulk0, bulk1, sync, prev_gm, prev_pass;
};
cudaError_t march_step(const MarchData& d, int step, cudaStream_t s, cudaStream_t side, const StepEvents& ev,
                       bool overlap);
int gmres_cluster_size(int device, int R, bool mixed);
// Launches of one time step of several models of R load cases each (R in 1,
// 2, 4, 8).  phase 0: every model's right-hand side over all history steps,
// then one GMRES cluster of `cluster` CTAs per model; phase 1: the same with
// the head right-hand side (KnownM, k <= 2, plus the bulk computed ahead);
// phase 2: only the bulk (history steps k >= 3) of `step` into the models'
// bulk buffers.  ds: device array of the models' MarchData (each laid out for
// `cluster`); row_off: [n_models + 1] prefix sums of their element counts;
// gmres_dsm: the largest dynamic shared memory any model's GMRES needs;
// max_K: the largest history length.
cudaError_t march_models_step(const MarchData* ds, const int* row_off, int n_models, int total_rows, int R,
                              bool mixed, int cluster, size_t gmres_dsm, int max_K, int step, int phase,
                              cudaStream_t s);
// The FP64 single-load GMRES step kernel on caller-supplied storage: d.R = 1,
// d.groups = 1, d.nstep = 1, step 1.  Every pointer it writes (b, bp, x, rv,
// u, V, W, AW, givens, status, step_flags, and unless d.solve_only the
// write-back targets out_lu, out_lt, xring, wring, audit) must be sized for
// that shape.
cudaError_t gmres_solve_single(const MarchData& d, cudaStream_t s);
// Adjoint march, step n: adj[type][col][3] (type 0 = U, 1 = T) = the
// transposed history convolution of the adjoint right-hand sides
// lam[0..N+1][E][3]; tptr [2 nh][K+1] gives each (type, column)'s blocks of
// step k, trow their equation rows, tval their 9 stacked values.
// One recorded step's right-hand side split into its parts (diagnostics):
// out [4][3E] = KnownM k_n, sum MGS_k W1, -sum MTS_k W0 and A x_n, rows in
// equation order.  xh: [N+1][2][nh][3] history states (X_0 = 0); known:
// [N+1][E][3]; a_*: A in equation-row order with 9 doubles per block; x: x_n
// in unknown order.
struct RhsSplitArgs {
    int E, K, nh, n;
    const int64_t* h_kptr;
    const uint32_t* h_col;
    const double* h_val;
    int64_t h_nnz;
    const double* xh;
    const int32_t* k_rp;
    const int32_t* k_col;
    const double* k_val;
    const int32_t* known_elem;
    const double* known_sign;
    const int32_t* k_elem;  // per KnownM block: known_elem of its column
    const double* k_sgn;    // per KnownM block: known_sign of its column
    const double* known;
    const int32_t* a_rp;
    const int32_t* a_col;
    const double* a_val;
    const double* x;
    double* out;
};
cudaError_t rhs_split(const RhsSplitArgs& a, cudaStream_t s);

// The stacked history blocks regrouped for adj_history: tptr [2 nh (K+1)]
// group ends, group (type * nh + column) * (K + 1) + k in ascending row order;
// trow, tval [nnz] and [nnz][9].  Synchronises the stream.
cudaError_t adjoint_history_groups(int E, int K, int nh, int64_t nnz, const int64_t* kptr, const uint32_t* hcol,
                                   const double* hval, int64_t* tptr, int32_t* trow, double* tval, cudaStream_t s);
// Transposed write-back of one reverse step (adjoint march), device arrays.
struct AdjWriteBack {
    int E, nh;
    const double* cot_lu;      // [N+1][E][3] or null
    const double* cot_lt;      // [N+1][E][3] or null
    const double* adj;         // [2][nh][3] history adjoint of this step, or null
    const int32_t* hist_owner;
    const int64_t* hist_block;
    const double* hu_sign;
    const double* ht_sign;
    const double* trans;       // [E][9] local frames
    const double* itf_trans;   // [E][9] interface transforms
    const double* uref_sign;
    const double* tref_sign;
    const int32_t* uref_known;
    const int32_t* tref_known;
    double* gk;                // [N+1][E][3] prescribed-value gradient (added to)
    double* contrib;           // [E][2][3] scratch
};
// Write-back of step n, then the transposed solve's right-hand side gp in
// perm order (unk_src: [E][2] (element * 2 + U/T) sources of each unknown,
// -1 for none; unk_of: unknown of each perm row).
cudaError_t adjoint_writeback(const AdjWriteBack& a, int n, const int32_t* unk_src, const int32_t* unk_of, double* gp,
                              cudaStream_t s);
// gk (step 0) += the cotangent of bd[0] through the local frame (lu for BCID
// 123, lt for 456); cot_* are the device cotangents of step 0 (or null).
cudaError_t adjoint_step0(int E, const double* trans, const int32_t* bcid, const double* cot_lu, const double* cot_lt,
                          double* gk, cudaStream_t s);
// gk (one step) += KnownM^T lam by columns: kt_ptr [n_known+1], kt_row and
// kt_blk (block index into k_val, 9 doubles row-major) in row order.
cudaError_t adjoint_known(int n_known, const int32_t* kt_ptr, const int32_t* kt_row, const int32_t* kt_blk,
                          const double* k_val, const int32_t* known_elem, const double* known_sign, const double* lam,
                          double* gk, cudaStream_t s);
cudaError_t adj_history(int N, int n, int K, int nh, int E, const int64_t* tptr, const int32_t* trow,
                        const double* tval, const double* lam, double* adj, cudaStream_t s);
// Dynamic shared memory of the GMRES kernel for Rg load cases per cluster
// and owned ranges of at most `rows` rows (0 when rows == 0).
size_t gmres_dsm_bytes(int rows, int Rg, bool mixed);
// Largest dynamic shared memory the GMRES kernel takes for the shared-memory
// Krylov path; owned ranges needing more fall back to global memory.
constexpr size_t kGmresDsmMax = 200 * 1024;

}  // namespace tdbem
