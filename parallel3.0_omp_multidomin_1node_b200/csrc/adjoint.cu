// Device-side set-up of the adjoint march: the stacked history blocks
// regrouped by (type, column) and step for the transposed convolution
// (adj_history_kernel), by a stable radix sort so that each group keeps the
// ascending-row order of the stacked matrix.
#include <cub/cub.cuh>

#include "march.cuh"
#include "tdbem_common.cuh"

namespace tdbem {

namespace {

// One warp per equation row: group key of every block of the row,
// group = (type * nh + column) * (K + 1) + k, its row, and the group sizes.
__global__ void hist_keys_kernel(int E, int K, int nh, const int64_t* kptr, const uint32_t* hcol, uint32_t* key,
                                 uint32_t* idx, int32_t* rowof, unsigned long long* counts)
{
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= E) return;
    const int64_t b = kptr[(int64_t)row * (K + 1)], e = kptr[(int64_t)row * (K + 1) + K];
    for (int64_t j = b + lane; j < e; j += 32) {
        const uint32_t c = hcol[j];
        const uint32_t seg = ((c >> 20) & 1u) * (uint32_t)nh + (c & 0xFFFFFu);
        const uint32_t g = seg * (uint32_t)(K + 1) + (c >> 21);
        key[j] = g;
        idx[j] = (uint32_t)j;
        rowof[j] = row;
        atomicAdd(counts + g, 1ull);
    }
}

// Gather rows and values (9 planes -> 9 consecutive doubles) in group order.
__global__ void hist_gather_kernel(int64_t nnz, const uint32_t* order, const int32_t* rowof, const double* hval,
                                   int32_t* trow, double* tval)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = order[i];
        trow[i] = rowof[j];
#pragma unroll
        for (int q = 0; q < 9; ++q) tval[9 * i + q] = hval[(int64_t)q * nnz + j];
    }
}

struct Scratch {
    void* p = nullptr;
    ~Scratch()
    {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 1); }
};

#define ADJ_TRY(x)                                 \
    do {                                           \
        const cudaError_t e_ = (x);                \
        if (e_ != cudaSuccess) return e_;          \
    } while (0)

}  // namespace

cudaError_t adjoint_history_groups(int E, int K, int nh, int64_t nnz, const int64_t* kptr, const uint32_t* hcol,
                                   const double* hval, int64_t* tptr, int32_t* trow, double* tval, cudaStream_t s)
{
    const int64_t groups = 2LL * nh * (K + 1);
    if (nnz >= (1LL << 31) || groups >= (1LL << 31)) return cudaErrorInvalidValue;
    int end_bit = 1;
    while (end_bit < 32 && (1LL << end_bit) < groups) ++end_bit;
    const size_t n = (size_t)std::max<int64_t>(nnz, 1);
    Scratch keys, keys2, idx, idx2, rowof, counts;
    ADJ_TRY(keys.alloc(4 * n));
    ADJ_TRY(keys2.alloc(4 * n));
    ADJ_TRY(idx.alloc(4 * n));
    ADJ_TRY(idx2.alloc(4 * n));
    ADJ_TRY(rowof.alloc(4 * n));
    ADJ_TRY(counts.alloc(8 * (size_t)groups));
    auto* k1 = static_cast<uint32_t*>(keys.p);
    auto* k2 = static_cast<uint32_t*>(keys2.p);
    auto* i1 = static_cast<uint32_t*>(idx.p);
    auto* i2 = static_cast<uint32_t*>(idx2.p);
    auto* cnt = static_cast<unsigned long long*>(counts.p);
    ADJ_TRY(cudaMemsetAsync(cnt, 0, 8 * (size_t)groups, s));
    hist_keys_kernel<<<ceil_div(E, 8), 256, 0, s>>>(E, K, nh, kptr, hcol, k1, i1, static_cast<int32_t*>(rowof.p), cnt);
    ADJ_TRY(cudaGetLastError());
    // group ends (the layout adj_history_kernel reads)
    size_t scan_bytes = 0, sort_bytes = 0;
    ADJ_TRY(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, cnt, reinterpret_cast<unsigned long long*>(tptr),
                                          (int)groups, s));
    ADJ_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, k1, k2, i1, i2, (int)nnz, 0, end_bit, s));
    Scratch temp;
    ADJ_TRY(temp.alloc(std::max(scan_bytes, sort_bytes)));
    ADJ_TRY(cub::DeviceScan::InclusiveSum(temp.p, scan_bytes, cnt, reinterpret_cast<unsigned long long*>(tptr),
                                          (int)groups, s));
    if (nnz > 0) {
        ADJ_TRY(cub::DeviceRadixSort::SortPairs(temp.p, sort_bytes, k1, k2, i1, i2, (int)nnz, 0, end_bit, s));
        const int grid = (int)std::min<int64_t>(ceil_div(nnz, 256), 8 * 148);
        hist_gather_kernel<<<grid, 256, 0, s>>>(nnz, i2, static_cast<int32_t*>(rowof.p), hval, trow, tval);
        ADJ_TRY(cudaGetLastError());
    }
    // the scratch is released when this returns: wait for its last use
    return cudaStreamSynchronize(s);
}

}  // namespace tdbem

namespace tdbem {

namespace {

// Transposed write-back of reverse step n: the cotangents of the global-frame
// outputs of step n plus the history adjoint go back through LocToAbs and the
// GlobalDofMap references; prescribed entries add to gk, unknown entries are
// left per (element, U/T) in contrib for adj_unknown_kernel.
__global__ void adj_writeback_kernel(AdjWriteBack a, int n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.E) return;
    const int64_t o = ((int64_t)n * a.E + i) * 3;
    double cu[3], ct[3];
    for (int c = 0; c < 3; ++c) {
        cu[c] = a.cot_lu ? a.cot_lu[o + c] : 0.0;
        ct[c] = a.cot_lt ? a.cot_lt[o + c] : 0.0;
    }
    if (a.adj && a.hist_owner[i]) {
        const int64_t hb = a.hist_block[i];
        for (int c = 0; c < 3; ++c) {
            cu[c] += a.hu_sign[i] * a.adj[3 * hb + c];
            ct[c] += a.ht_sign[i] * a.adj[3 * (a.nh + hb) + c];
        }
    }
    const double* F = a.trans + 9 * i;
    const double* T = a.itf_trans + 9 * i;
    for (int which = 0; which < 2; ++which) {
        const double* cg = which ? ct : cu;
        double cl[3];  // gu = F^T l  ->  dl = F dgu
        for (int j = 0; j < 3; ++j) cl[j] = F[3 * j] * cg[0] + F[3 * j + 1] * cg[1] + F[3 * j + 2] * cg[2];
        const bool known = which ? a.tref_known[i] : a.uref_known[i];
        const double sg = which ? a.tref_sign[i] : a.uref_sign[i];
        double* cv = a.contrib + (2 * i + which) * 3;
        if (known) {
            for (int c = 0; c < 3; ++c) a.gk[o + c] += sg * cl[c];
            for (int c = 0; c < 3; ++c) cv[c] = 0.0;
        } else {
            for (int j = 0; j < 3; ++j) cv[j] = sg * (T[j] * cl[0] + T[3 + j] * cl[1] + T[6 + j] * cl[2]);
        }
    }
}

// Right-hand side of the transposed solve in perm (A' column) order: unknown
// u = unk_of[p] sums its (at most two) sources in element order.
__global__ void adj_unknown_kernel(int E, const int32_t* unk_src, const int32_t* unk_of, const double* contrib,
                                   double* gp)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= E) return;
    const int64_t u = unk_of[p];
    double g[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < 2; ++k) {
        const int src = unk_src[2 * u + k];
        if (src < 0) continue;
        for (int c = 0; c < 3; ++c) g[c] += contrib[3 * (int64_t)src + c];
    }
    for (int c = 0; c < 3; ++c) gp[3 * p + c] = g[c];
}

// KnownM^T lam_n into the prescribed-value gradient: known block kb sums its
// column's blocks in row order.
__global__ void adj_known_kernel(int n_known, const int32_t* kt_ptr, const int32_t* kt_row, const int32_t* kt_blk,
                                 const double* k_val, const int32_t* known_elem, const double* known_sign,
                                 const double* lam, double* gk)
{
    const int kb = blockIdx.x * blockDim.x + threadIdx.x;
    if (kb >= n_known) return;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int j = kt_ptr[kb]; j < kt_ptr[kb + 1]; ++j) {
        const double* B = k_val + 9 * (int64_t)kt_blk[j];
        const double* l = lam + 3 * (int64_t)kt_row[j];
        for (int c = 0; c < 3; ++c) acc[c] += B[c] * l[0] + B[3 + c] * l[1] + B[6 + c] * l[2];
    }
    const double sg = known_sign[kb];
    double* g = gk + 3 * (int64_t)known_elem[kb];
    for (int c = 0; c < 3; ++c) g[c] += sg * acc[c];
}

// Step 0 of the gradient: bd[0] is the prescribed value converted to the
// global frame (lu for BCID 123, lt for 456), so its cotangent goes back
// through the frame: gk[0][i] = F_i^T-applied cotangent.
__global__ void adj_step0_kernel(int E, const double* trans, const int32_t* bcid, const double* cot_lu,
                                 const double* cot_lt, double* gk)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= E) return;
    const double* c = bcid[i] == 456 ? cot_lt : cot_lu;
    if (!c) return;
    const double* F = trans + 9 * i;
    for (int j = 0; j < 3; ++j)
        gk[3 * i + j] += F[3 * j] * c[3 * i] + F[3 * j + 1] * c[3 * i + 1] + F[3 * j + 2] * c[3 * i + 2];
}

}  // namespace

cudaError_t adjoint_step0(int E, const double* trans, const int32_t* bcid, const double* cot_lu, const double* cot_lt,
                          double* gk, cudaStream_t s)
{
    adj_step0_kernel<<<ceil_div(E, 128), 128, 0, s>>>(E, trans, bcid, cot_lu, cot_lt, gk);
    return cudaGetLastError();
}

cudaError_t adjoint_writeback(const AdjWriteBack& a, int n, const int32_t* unk_src, const int32_t* unk_of, double* gp,
                              cudaStream_t s)
{
    adj_writeback_kernel<<<ceil_div(a.E, 128), 128, 0, s>>>(a, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    adj_unknown_kernel<<<ceil_div(a.E, 128), 128, 0, s>>>(a.E, unk_src, unk_of, a.contrib, gp);
    return cudaGetLastError();
}

cudaError_t adjoint_known(int n_known, const int32_t* kt_ptr, const int32_t* kt_row, const int32_t* kt_blk,
                          const double* k_val, const int32_t* known_elem, const double* known_sign, const double* lam,
                          double* gk, cudaStream_t s)
{
    if (n_known <= 0) return cudaSuccess;
    adj_known_kernel<<<ceil_div(n_known, 128), 128, 0, s>>>(n_known, kt_ptr, kt_row, kt_blk, k_val, known_elem,
                                                            known_sign, lam, gk);
    return cudaGetLastError();
}

}  // namespace tdbem
