// Assembly kernels (geometry, singular integrals, Step0 / history blocks,
// compaction, stacking, preconditioner inverses).
#pragma once

#include "tdbem_common.cuh"

namespace tdbem {

// (source row, field element) pairs of every domain: pair p of domain d is
// row dom_begin[d] + loc / n_d, field dom_begin[d] + loc % n_d.
struct PairSpace {
    int n_domains;
    int64_t n_pairs;
    const int32_t* dom_begin;
    const int32_t* dom_count;
    const int64_t* pair_off;  // [n_domains + 1]
};

// GlobalDofMap references per element, device arrays.
struct DofRefs {
    const double* uref_sign;
    const double* tref_sign;
    const double* hu_sign;
    const double* ht_sign;
    const double* itf_trans;  // [E][9]
};

struct ScatterCols {
    int slot_of_bit[3];
    const int64_t* col_of_bit[3];
};

// One history step's compacted matrices (rows = equation rows).
struct HistK {
    const int64_t* mts_rp;
    const int32_t* mts_col;
    const double* mts_val;  // [nnz][9]
    const int64_t* mgs_rp;
    const int32_t* mgs_col;
    const double* mgs_val;
};

// Saved forward state and adjoint vectors read by the material-gradient
// contraction (one load case).
struct GradState {
    int N, E, K, nh;
    const double* lam;         // [N+2][E][3] adjoint vectors, equation-row order (steps 1..N)
    const double* x;           // [N][E][3] unknowns of step n at n-1, unknown order
    const double* known;       // [N+1][E][3] prescribed element-local values
    const double* xh;          // [N+1][2][nh][3] history states X_m (U, T); X_0 = 0
    const int32_t* known_elem;
    const double* known_sign;
    const int64_t* col_a0;     // per field element: column of A slot 0, A slot 1,
    const int64_t* col_a1;     // KnownM and the history matrices
    const int64_t* col_k;
    const int64_t* col_h;
};

cudaError_t upload_materials(const DynaMat* mats, int n, cudaStream_t s);
cudaError_t upload_materials_dual(const DynaMatD* mats, int n, cudaStream_t s);

__global__ void geometry_kernel(int E, const double* points, const int64_t* elements, const QuadRules* rules,
                                ElemGeom g);
__global__ void singular_kernel(int E, const QuadRules* rules, const double* secpw_pos, const double* secpw_val,
                                ElemGeom g);
__global__ void step0_kernel(PairSpace ps, const QuadRules* rules, ElemGeom g, DofRefs dr, double* blocks,
                             uint8_t* flags);
__global__ void history_kernel(PairSpace ps, const QuadRules* rules, ElemGeom g, DofRefs dr, int k, double* blocks,
                               uint8_t* flags);
__global__ void count_rows_kernel(PairSpace ps, const uint8_t* flags, int mask, int E, int* counts);
__global__ void scatter_rows_kernel(PairSpace ps, const uint8_t* flags, const double* blocks, int mask, int E,
                                    const int64_t* row_start, ScatterCols sc, int32_t* out_col, double* out_val);
__global__ void stack_history_kernel(int E, int K, const HistK* hk, const int64_t* kptr, uint32_t* col, double* val,
                                     int64_t nnz);
__global__ void singular_grad_kernel(int E, const double* secpw_pos, const double* secpw_val, ElemGeom g,
                                     QDual* self_d);
__global__ void history_states_kernel(int N, int E, int nh, const int32_t* hist_owner, const int64_t* hist_block,
                                      const double* hu_sign, const double* ht_sign, const double* out_lu,
                                      const double* out_lt, double* xh);
__global__ void grad_step0_kernel(PairSpace ps, const QuadRules* rules, ElemGeom g, DofRefs dr, const QDual* self_d,
                                  GradState gs, double* part);
__global__ void grad_history_kernel(PairSpace ps, const QuadRules* rules, ElemGeom g, DofRefs dr,
                                    const QDual* self_d, GradState gs, double* part);
__global__ void to_float_kernel(const double* in, float* out, int64_t n);
__global__ void leaf_inverse_kernel(int n_leaves, const int32_t* leaf_begin, const int32_t* leaf_count,
                                    const int64_t* leaf_off, const int32_t* a_rp, const int32_t* a_col,
                                    const double* a_val, double* pinv, int* singular);

}  // namespace tdbem
