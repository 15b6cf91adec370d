// Per-step right-hand-side breakdown for the diagnostic CSV files
// (WriteRhsBreakdownCsv, DBEM1/multidomain.cpp:247-327): the KnownM part,
// the MGS (history G) and -MTS (history T) convolution parts and A x of one
// recorded step, recomputed in FP64 from the saved states.
#include "march.cuh"
#include "tdbem_common.cuh"

namespace tdbem {

namespace {

// One warp per equation row r; out[0..3][3E] = known, historyG, historyT, Ax.
__global__ void rhs_split_kernel(RhsSplitArgs a)
{
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= a.E) return;
    double acc[4][3];
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[p][c] = 0.0;
    // KnownM k_n
    const double* kn = a.known + (int64_t)a.n * a.E * 3;
    for (int j = a.k_rp[r] + lane; j < a.k_rp[r + 1]; j += 32) {
        const int kb = a.k_col[j];
        const double sg = a.known_sign[kb];
        const double* kv = kn + 3 * (int64_t)a.known_elem[kb];
        const double* B = a.k_val + 9 * (int64_t)j;
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[0][c] += B[3 * c] * (sg * kv[0]) + B[3 * c + 1] * (sg * kv[1]) + B[3 * c + 2] * (sg * kv[2]);
    }
    // history steps k = 1..min(n, K), for n >= 2: stacked MGS_k (type 1) and
    // -MTS_k (type 0) times the convolution vector of step n
    const int kmax = a.n >= 2 ? (a.n < a.K ? a.n : a.K) : 0;
    if (kmax > 0) {
        const int64_t beg = a.h_kptr[(int64_t)r * (a.K + 1)], end = a.h_kptr[(int64_t)r * (a.K + 1) + kmax];
        const int64_t X3 = 3 * (int64_t)a.nh;
        for (int64_t j = beg + lane; j < end; j += 32) {
            const uint32_t cp = a.h_col[j];
            const int k = (int)(cp >> 21), type = (int)((cp >> 20) & 1u), col = (int)(cp & 0xFFFFFu);
            const int m = a.n - k;
            const double* xm = a.xh + ((int64_t)m * 2 + type) * X3 + 3 * (int64_t)col;
            double w[3] = {2.0 * xm[0], 2.0 * xm[1], 2.0 * xm[2]};
            if (m + 1 < a.n) {
                const double* xp = a.xh + ((int64_t)(m + 1) * 2 + type) * X3 + 3 * (int64_t)col;
                for (int c = 0; c < 3; ++c) w[c] = xp[c] + w[c];
            }
            if (m >= 1) {
                const double* xq = a.xh + ((int64_t)(m - 1) * 2 + type) * X3 + 3 * (int64_t)col;
                for (int c = 0; c < 3; ++c) w[c] += xq[c];
            }
            double B[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) B[q] = a.h_val[(int64_t)q * a.h_nnz + j];
            const int p = type ? 1 : 2;
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[p][c] += B[3 * c] * w[0] + B[3 * c + 1] * w[1] + B[3 * c + 2] * w[2];
        }
    }
    // A x_n (row-order A, unknown-order x)
    for (int j = a.a_rp[r] + lane; j < a.a_rp[r + 1]; j += 32) {
        const double* xv = a.x + 3 * (int64_t)a.a_col[j];
        const double* B = a.a_val + 9 * (int64_t)j;
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[3][c] += B[3 * c] * xv[0] + B[3 * c + 1] * xv[1] + B[3 * c + 2] * xv[2];
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[p][c] += __shfl_xor_sync(0xffffffffu, acc[p][c], o);
    if (lane < 12) {
        const int p = lane / 3, c = lane % 3;
        a.out[(int64_t)p * 3 * a.E + 3 * r + c] = acc[p][c];
    }
}

}  // namespace

cudaError_t rhs_split(const RhsSplitArgs& a, cudaStream_t s)
{
    rhs_split_kernel<<<ceil_div(a.E, 8), 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace tdbem
