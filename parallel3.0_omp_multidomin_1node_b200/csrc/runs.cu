// Run layout of the stacked history blocks, read by the T-step history pass
// (bulk_steps_kernel in march.cu).
//
// The stacked layout keeps each equation row's blocks step-major (k = 1..K,
// then type and column), which suits a pass over one step.  The blocks of one
// (row, type, column) pair form an unbroken run of consecutive steps (the
// wave front passes a source-field pair during a window of steps), so the
// T-step pass walks runs instead: block k of a run meets the combined
// history vectors W_{s-k} .. W_{s+T-1-k} for steps s .. s + T - 1, and all but
// W_{s-k} are vectors its predecessor met, kept in registers.
//
// Built on the device from the stacked arrays: sort the blocks of steps
// k >= kr by (row, type, column, k), cut runs where the pair changes or k
// jumps, order each row's runs longest first (so the lane groups of one warp
// walk runs of similar length), and gather the block values into that order.
#include "march.cuh"

#include <climits>
#include <vector>

#include <cub/cub.cuh>

namespace tdbem {

namespace {

// one warp per row: sort keys row << 32 | type << 31 | column << 11 | k of the
// row's blocks of steps k >= kr, with their stacked index
__global__ void run_keys_kernel(int E, int K, int kr, const int64_t* __restrict__ kptr,
                                const int64_t* __restrict__ qoff, const uint32_t* __restrict__ col,
                                unsigned long long* __restrict__ key, uint32_t* __restrict__ idx)
{
    const int r = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (r >= E) return;
    const int64_t beg = kptr[(int64_t)r * (K + 1) + kr - 1], end = kptr[(int64_t)r * (K + 1) + K];
    const int64_t q0 = qoff[r] - beg;
    for (int64_t i = beg + lane; i < end; i += 32) {
        const uint32_t cp = col[i];
        const unsigned long long k = cp >> 21, type = (cp >> 20) & 1u, c = cp & 0xFFFFFu;
        key[q0 + i] = ((unsigned long long)r << 32) | (type << 31) | (c << 11) | k;
        idx[q0 + i] = (uint32_t)i;
    }
}

// 1 where sorted block q starts a run: a new (row, type, column) or a gap in k
__global__ void run_flags_kernel(int64_t nb, const unsigned long long* __restrict__ key, int* __restrict__ flag)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nb; q += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long a = key[q];
        int f = 1;
        if (q > 0) {
            const unsigned long long b = key[q - 1];
            f = (b >> 11) != (a >> 11) || (b & 0x7FFull) + 1 != (a & 0x7FFull);
        }
        flag[q] = f;
    }
}

// run j (inclusive scan of the flags minus one) starts at sorted block q
__global__ void run_starts_kernel(int64_t nb, const int* __restrict__ flag, const int* __restrict__ runid,
                                  int* __restrict__ start)
{
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nb; q += (int64_t)gridDim.x * blockDim.x)
        if (flag[q]) start[runid[q] - 1] = (int)q;
}

// order key of run j: row << 16 | (0xFFFF - length), so a stable sort puts each
// row's runs longest first; counts the row's runs
__global__ void run_order_keys_kernel(int n_runs, int64_t nb, const int* __restrict__ start,
                                      const unsigned long long* __restrict__ key, unsigned long long* __restrict__ okey,
                                      int* __restrict__ oval, int* __restrict__ row_count)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n_runs; j += gridDim.x * blockDim.x) {
        const int q = start[j];
        const int len = (j + 1 < n_runs ? start[j + 1] : (int)nb) - q;
        const unsigned long long row = key[q] >> 32;
        okey[j] = (row << 16) | (unsigned long long)(0xFFFF - len);
        oval[j] = j;
        atomicAdd(row_count + row, 1);
    }
}

__global__ void run_lengths_kernel(int n_runs, const unsigned long long* __restrict__ okey, int64_t* __restrict__ len)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_runs; i += gridDim.x * blockDim.x)
        len[i] = 0xFFFF - (int64_t)(okey[i] & 0xFFFFull);
}

// one warp per run (in final order): header, then the 9 values of each block
template <class T>
__global__ void run_gather_kernel(int n_runs, int64_t nb, int64_t nnz, const int* __restrict__ order,
                                  const int* __restrict__ start, const int64_t* __restrict__ len,
                                  const int64_t* __restrict__ off, const unsigned long long* __restrict__ key,
                                  const uint32_t* __restrict__ idx, const T* __restrict__ val, uint2* __restrict__ meta,
                                  int64_t* __restrict__ r_off, T* __restrict__ out)
{
    const int i = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (i >= n_runs) return;
    const int q = start[order[i]];
    const int n = (int)len[i];
    const int64_t o = off[i];
    if (lane == 0) {
        const unsigned long long a = key[q];
        const unsigned type = (unsigned)((a >> 31) & 1u), c = (unsigned)((a >> 11) & 0xFFFFFu),
                       kf = (unsigned)(a & 0x7FFu);
        meta[i] = make_uint2((type << 20) | c, (kf << 16) | (unsigned)n);
        r_off[i] = o;
    }
    for (int t = lane; t < n; t += 32) {
        const int64_t src = idx[q + t];
#pragma unroll
        for (int c = 0; c < 9; ++c) out[c * nb + o + t] = val[c * nnz + src];
    }
}

struct Tmp {
    void* p = nullptr;
    Tmp() = default;
    Tmp(const Tmp&) = delete;
    Tmp& operator=(const Tmp&) = delete;
    ~Tmp() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
    }
    cudaError_t alloc(size_t n)
    {
        release();
        return cudaMalloc(&p, n ? n : 1);
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

int bits_for(unsigned long long v)
{
    int b = 0;
    while (b < 64 && (v >> b) != 0) ++b;
    return b;
}

}  // namespace

#define RUN_TRY(x)                          \
    do {                                    \
        cudaError_t e_ = (x);               \
        if (e_ != cudaSuccess) return e_;   \
    } while (0)

size_t history_runs_bytes(int64_t nb, bool mixed)
{
    // per block: sort keys and indices (double-buffered), flags, run ids and
    // the radix sort's scratch; per run (about nine blocks on the models
    // measured; counted as four): start, order keys and values
    // (double-buffered), length, offset and header; the output values.  An
    // estimate: the caller falls back to the one-step pass when an
    // allocation fails all the same.
    const size_t per_block = 2 * 8 + 2 * 4 + 4 + 4 + 16;
    const size_t per_run = 4 + 2 * 8 + 2 * 4 + 8 + 8 + 8 + 8;
    return (size_t)nb * (per_block + 9 * (mixed ? sizeof(float) : sizeof(double))) + (size_t)nb / 4 * per_run;
}

cudaError_t build_history_runs(int E, int K, int kr, const std::vector<int64_t>& kptr, const int64_t* d_kptr,
                               const uint32_t* d_col, const void* d_val, int64_t nnz, bool mixed, HistoryRuns& out,
                               cudaStream_t s)
{
    out = HistoryRuns{};
    if (kr < 1 || kr > K) return cudaSuccess;
    std::vector<int64_t> qoff(E + 1, 0);
    for (int r = 0; r < E; ++r)
        qoff[r + 1] = qoff[r] + kptr[(size_t)r * (K + 1) + K] - kptr[(size_t)r * (K + 1) + kr - 1];
    const int64_t nb = qoff[E];
    if (nb <= 0 || nb > INT_MAX || nnz >= (int64_t)UINT_MAX) return cudaSuccess;
    const int n = (int)nb;
    Tmp d_qoff, k1, k2, i1, i2, flag, runid;
    RUN_TRY(d_qoff.alloc(sizeof(int64_t) * (E + 1)));
    RUN_TRY(cudaMemcpyAsync(d_qoff.p, qoff.data(), sizeof(int64_t) * (E + 1), cudaMemcpyHostToDevice, s));
    RUN_TRY(k1.alloc(8 * (size_t)nb));
    RUN_TRY(k2.alloc(8 * (size_t)nb));
    RUN_TRY(i1.alloc(4 * (size_t)nb));
    RUN_TRY(i2.alloc(4 * (size_t)nb));
    run_keys_kernel<<<(E + 7) / 8, 256, 0, s>>>(E, K, kr, d_kptr, d_qoff.as<int64_t>(), d_col,
                                               k1.as<unsigned long long>(), i1.as<uint32_t>());
    RUN_TRY(cudaGetLastError());
    const int end_bit = 32 + bits_for((unsigned long long)E);
    size_t sort_bytes = 0;
    RUN_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, k1.as<unsigned long long>(),
                                            k2.as<unsigned long long>(), i1.as<uint32_t>(), i2.as<uint32_t>(), n, 0,
                                            end_bit, s));
    {
        Tmp temp;
        RUN_TRY(temp.alloc(sort_bytes));
        RUN_TRY(cub::DeviceRadixSort::SortPairs(temp.p, sort_bytes, k1.as<unsigned long long>(),
                                                k2.as<unsigned long long>(), i1.as<uint32_t>(), i2.as<uint32_t>(), n,
                                                0, end_bit, s));
    }
    // k2 / i2: blocks in (row, type, column, k) order
    RUN_TRY(flag.alloc(4 * (size_t)nb));
    RUN_TRY(runid.alloc(4 * (size_t)nb));
    run_flags_kernel<<<1184, 256, 0, s>>>(nb, k2.as<unsigned long long>(), flag.as<int>());
    RUN_TRY(cudaGetLastError());
    size_t scan_bytes = 0;
    RUN_TRY(cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, flag.as<int>(), runid.as<int>(), n, s));
    {
        Tmp temp;
        RUN_TRY(temp.alloc(scan_bytes));
        RUN_TRY(cub::DeviceScan::InclusiveSum(temp.p, scan_bytes, flag.as<int>(), runid.as<int>(), n, s));
    }
    int n_runs = 0;
    RUN_TRY(cudaMemcpyAsync(&n_runs, runid.as<int>() + (nb - 1), sizeof(int), cudaMemcpyDeviceToHost, s));
    RUN_TRY(cudaStreamSynchronize(s));
    k1.release();  // not needed past the sort
    i1.release();
    Tmp start, okey1, okey2, ov1, ov2, lens, offs;
    RUN_TRY(start.alloc(4 * (size_t)n_runs));
    run_starts_kernel<<<1184, 256, 0, s>>>(nb, flag.as<int>(), runid.as<int>(), start.as<int>());
    RUN_TRY(cudaGetLastError());
    RUN_TRY(okey1.alloc(8 * (size_t)n_runs));
    RUN_TRY(okey2.alloc(8 * (size_t)n_runs));
    RUN_TRY(ov1.alloc(4 * (size_t)n_runs));
    RUN_TRY(ov2.alloc(4 * (size_t)n_runs));
    // runs per row (E + 1 entries, the last one stays zero)
    Tmp rcnt32;
    RUN_TRY(rcnt32.alloc(sizeof(int) * (E + 1)));
    RUN_TRY(cudaMemsetAsync(rcnt32.p, 0, sizeof(int) * (E + 1), s));
    run_order_keys_kernel<<<1184, 256, 0, s>>>(n_runs, nb, start.as<int>(), k2.as<unsigned long long>(),
                                               okey1.as<unsigned long long>(), ov1.as<int>(), rcnt32.as<int>());
    RUN_TRY(cudaGetLastError());
    const int end2 = 16 + bits_for((unsigned long long)E);
    RUN_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, okey1.as<unsigned long long>(),
                                            okey2.as<unsigned long long>(), ov1.as<int>(), ov2.as<int>(), n_runs, 0,
                                            end2, s));
    {
        Tmp temp;
        RUN_TRY(temp.alloc(sort_bytes));
        RUN_TRY(cub::DeviceRadixSort::SortPairs(temp.p, sort_bytes, okey1.as<unsigned long long>(),
                                                okey2.as<unsigned long long>(), ov1.as<int>(), ov2.as<int>(), n_runs,
                                                0, end2, s));
    }
    RUN_TRY(lens.alloc(8 * (size_t)n_runs));
    RUN_TRY(offs.alloc(8 * (size_t)n_runs));
    run_lengths_kernel<<<1184, 256, 0, s>>>(n_runs, okey2.as<unsigned long long>(), lens.as<int64_t>());
    RUN_TRY(cudaGetLastError());
    RUN_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, lens.as<int64_t>(), offs.as<int64_t>(), n_runs, s));
    {
        Tmp temp;
        RUN_TRY(temp.alloc(scan_bytes));
        RUN_TRY(cub::DeviceScan::ExclusiveSum(temp.p, scan_bytes, lens.as<int64_t>(), offs.as<int64_t>(), n_runs,
                                              s));
    }
    // row pointers: exclusive sum of the per-row run counts (E + 1 entries,
    // the last count is zero)
    Tmp ptr32;
    RUN_TRY(ptr32.alloc(sizeof(int) * (E + 1)));
    RUN_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, rcnt32.as<int>(), ptr32.as<int>(), E + 1, s));
    {
        Tmp temp;
        RUN_TRY(temp.alloc(scan_bytes));
        RUN_TRY(cub::DeviceScan::ExclusiveSum(temp.p, scan_bytes, rcnt32.as<int>(), ptr32.as<int>(), E + 1, s));
    }
    std::vector<int> hp(E + 1);
    RUN_TRY(cudaMemcpyAsync(hp.data(), ptr32.p, sizeof(int) * (E + 1), cudaMemcpyDeviceToHost, s));
    RUN_TRY(cudaStreamSynchronize(s));
    std::vector<int64_t> hp64(hp.begin(), hp.end());
    const size_t vs = mixed ? sizeof(float) : sizeof(double);
    RUN_TRY(cudaMalloc(reinterpret_cast<void**>(&out.ptr), sizeof(int64_t) * (E + 1)));
    RUN_TRY(cudaMemcpyAsync(out.ptr, hp64.data(), sizeof(int64_t) * (E + 1), cudaMemcpyHostToDevice, s));
    RUN_TRY(cudaMalloc(reinterpret_cast<void**>(&out.meta), sizeof(uint2) * (size_t)n_runs));
    RUN_TRY(cudaMalloc(reinterpret_cast<void**>(&out.off), sizeof(int64_t) * (size_t)n_runs));
    RUN_TRY(cudaMalloc(&out.val, vs * 9 * (size_t)nb));
    const int gb = (int)(((int64_t)n_runs * 32 + 255) / 256);
    if (mixed)
        run_gather_kernel<float><<<gb, 256, 0, s>>>(n_runs, nb, nnz, ov2.as<int>(), start.as<int>(),
                                                    lens.as<int64_t>(), offs.as<int64_t>(),
                                                    k2.as<unsigned long long>(), i2.as<uint32_t>(),
                                                    static_cast<const float*>(d_val), out.meta, out.off,
                                                    static_cast<float*>(out.val));
    else
        run_gather_kernel<double><<<gb, 256, 0, s>>>(n_runs, nb, nnz, ov2.as<int>(), start.as<int>(),
                                                     lens.as<int64_t>(), offs.as<int64_t>(),
                                                     k2.as<unsigned long long>(), i2.as<uint32_t>(),
                                                     static_cast<const double*>(d_val), out.meta, out.off,
                                                     static_cast<double*>(out.val));
    RUN_TRY(cudaGetLastError());
    RUN_TRY(cudaStreamSynchronize(s));
    out.nb = nb;
    out.runs = n_runs;
    out.kr = kr;
    return cudaSuccess;
}

}  // namespace tdbem
