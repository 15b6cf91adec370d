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
