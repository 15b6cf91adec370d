// Per-step kernels of the multi-domain TDBEM time march on B200.
//
//   rhs_kernel          history-convolution right-hand side for R load
//                       cases at once (one CTA per equation row): each 3x3
//                       history block is read from HBM once and applied to
//                       all R combined history vectors (block SpMM),
//                       DBEM1/multidomain.cpp:3843-3866; the head pass on
//                       the GMRES chain and the one-step pass beside it
//   bulk_steps_kernel   the history steps k >= 2T + 1 of T time steps in
//                       one pass over the run layout (two or more load
//                       cases): each block read once for the T steps, each
//                       history vector of a run once, kept in registers
//   gmres_cluster_kernel left-preconditioned GMRES(restart) for the R load
//                       cases in lockstep on one thread-block cluster:
//                       hardware cluster barriers, reductions through
//                       distributed shared memory, one SpMM of A' per
//                       Arnoldi step shared by all cases,
//                       DBEM1/pre_gmres.cpp:1369-1605; then the boundary
//                       write-back and history-state update,
//                       DBEM1/multidomain.cpp:3086-3225
#include "march.cuh"

#include <atomic>
#include "tdbem_common.cuh"

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace tdbem {

namespace {

constexpr int kRhsThreads = 256;
constexpr int kMaxDevices = 64;        // launch attributes are kept per device
constexpr int kGmresThreads = 512;
constexpr int kGmresWarps = kGmresThreads / 32;
constexpr int kDotChunk = 8;                // basis vectors per Gram-Schmidt reduction
constexpr int kDotMax = kDotChunk + 1;      // values per cluster reduction

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }

template <int R, int kCpt = (R >= 4 ? 4 : R)>
struct Lanes {
    static constexpr int CPT = kCpt;            // load cases per thread
    static constexpr int TPB = R / CPT;         // threads sharing one block
    static constexpr int BPW = 32 / TPB;        // blocks per warp iteration
};

// CPT consecutive values (16-byte aligned when CPT = 4 and R % 4 == 0)
template <int CPT>
__device__ __forceinline__ void load_cases(const float* p, float* v)
{
    if constexpr (CPT == 4) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
    } else if constexpr (CPT == 2) {
        const float2 t = *reinterpret_cast<const float2*>(p);
        v[0] = t.x; v[1] = t.y;
    } else {
        v[0] = *p;
    }
}

template <int CPT>
__device__ __forceinline__ void load_cases(const double* p, double* v)
{
    if constexpr (CPT == 4) {
        const double2 a = *reinterpret_cast<const double2*>(p);
        const double2 b = *reinterpret_cast<const double2*>(p + 2);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else if constexpr (CPT == 2) {
        const double2 a = *reinterpret_cast<const double2*>(p);
        v[0] = a.x; v[1] = a.y;
    } else {
        v[0] = *p;
    }
}

template <int CPT>
__device__ __forceinline__ void ldcg_cases(const double* p, double* v)
{
    if constexpr (CPT == 4) {
        const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldcg(reinterpret_cast<const double2*>(p + 2));
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    } else if constexpr (CPT == 2) {
        const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
        v[0] = a.x; v[1] = a.y;
    } else {
        v[0] = __ldcg(p);
    }
}

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v)
{
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

}  // namespace

// ---------------------------------------------------------------------------
// bd[0] conversion (BoundaryValue::Convert + AllLocToAbs,
// DBEM1/multidomain.cpp:3819-3821) and zeroed history rings.
__global__ void prepare_kernel(MarchData d)
{
    const int E = d.E;
    const long long n0 = (long long)d.R * E;
    const long long g0 = blockIdx.x * (long long)blockDim.x + threadIdx.x, gs = gridDim.x * (long long)blockDim.x;
    for (long long t = g0; t < n0; t += gs) {
        const int r = (int)(t / E), i = (int)(t % E);
        const double* in = d.known_lu + ((long long)r * (d.nstep + 1) * E + i) * 3;
        double lu[3], lt[3];
        for (int c = 0; c < 3; ++c) {
            lu[c] = d.bcid[i] == 456 ? 0.0 : in[c];
            lt[c] = d.bcid[i] == 456 ? in[c] : 0.0;
        }
        const double* T = d.trans + 9 * i;
        double* ou = d.out_lu + ((long long)r * (d.nstep + 1) * E + i) * 3;
        double* ot = d.out_lt + ((long long)r * (d.nstep + 1) * E + i) * 3;
        for (int c = 0; c < 3; ++c) {
            ou[c] = T[c] * lu[0] + T[3 + c] * lu[1] + T[6 + c] * lu[2];
            ot[c] = T[c] * lt[0] + T[3 + c] * lt[1] + T[6 + c] * lt[2];
        }
    }
    const long long nx = 3LL * 2 * d.nh * 3 * d.R;
    for (long long t = g0; t < nx; t += gs) d.xring[t] = 0.0;
    const long long nw = (long long)d.SW * 2 * d.nh * 3 * d.R;
    for (long long t = g0; t < nw; t += gs) d.wring[t] = 0.0;
    for (long long t = g0; t < 8LL * 3 * d.E * d.R; t += gs) d.bulk[t] = 0.0;
    for (long long t = g0; t < 2LL * d.nstep; t += gs) d.audit[t] = 0.0;
    if (g0 < 4) d.status[g0] = 0;
}

// ---------------------------------------------------------------------------
// This warp's share of KnownM . known_step for equation row `row`
// (DBEM1/multidomain.cpp:3843-3846): known blocks j = first + w, first + w +
// NW, ... of the row; lane r < R takes load case r.  The warps' shares are
// summed with the history sums.
template <int R, int NW>
__device__ __forceinline__ void known_share(const MarchData& d, int row, int step, int w, int lane, double (&ka)[3])
{
    ka[0] = ka[1] = ka[2] = 0.0;
    if (lane >= R) return;
    const double* kv0 = d.known_lu + ((int64_t)lane * (d.nstep + 1) + step) * d.E * 3;
    const int je = d.k_rp[row + 1];
    for (int j = d.k_rp[row] + w; j < je; j += NW) {
        const double sg = d.k_sgn[j];
        const double* kv = kv0 + 3 * (int64_t)d.k_elem[j];
        const double x0 = sg * kv[0], x1 = sg * kv[1], x2 = sg * kv[2];
        const double* v = d.k_val + 9 * (int64_t)j;
        ka[0] += v[0] * x0 + v[1] * x1 + v[2] * x2;
        ka[1] += v[3] * x0 + v[4] * x1 + v[5] * x2;
        ka[2] += v[6] * x0 + v[7] * x1 + v[8] * x2;
    }
}

// ---------------------------------------------------------------------------
// Right-hand side of perm row p for steps k in [k_lo, k_hi]:
//   sum_k MGS_k . wT(s-k) - MTS_k . wU(s-k)     (MTS blocks stored negated)
// kBulk: write KnownM . known_s + sum to the bulk buffer of `step`.
// Otherwise write b = sum + the bulk buffer of `step` when add_bulk, else
// b = KnownM . known_s + sum.  Each block's 9 values are read once
// (streaming loads) and applied to the R load cases; a thread handles CPT
// cases.
template <int R, bool kMixed, bool kBulk, int kCpt>
__device__ __forceinline__ void rhs_row(const MarchData& d, const int p, const int step, const int add_bulk,
                                        const int k_lo, const int k_hi)
{
    // blocks in flight per lane group: measured best 6 (two CTAs per SM) for
    // 32 load cases, 4 (three CTAs per SM) for one
    constexpr int kUnroll = R >= 8 ? 6 : 4;
    using L = Lanes<R, kCpt>;
    constexpr int CPT = L::CPT, TPB = L::TPB, BPW = L::BPW;
    constexpr int NW = kRhsThreads / 32;
    // The head pass runs on the chain stream after the previous step's GMRES,
    // the only writer of the status word, so all its threads read one value.
    // The bulk pass runs beside a GMRES launch that may set the word at any
    // time: thread 0's reading is OR-ed across the CTA by the barrier itself,
    // so every thread takes the same branch.  (A form that broadcast the
    // reading through a shared variable made the 32-load mixed march 8%
    // slower, measured: the hot loop compiled differently.)
    if constexpr (!kBulk)
        if (*(volatile int*)d.status) return;
    extern __shared__ int slot_of_k[];
    __shared__ double red[NW][3][R];
    const int row = d.row_of[p];
    const int K = d.K, SW = d.SW;
    for (int k = threadIdx.x; k <= K; k += blockDim.x) slot_of_k[k] = (((step - k) % SW) + SW) % SW;
    if (__syncthreads_or(kBulk && threadIdx.x == 0 && *(volatile int*)d.status)) return;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sub = lane / TPB, cgp = lane % TPB;
    double acc[3][CPT];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int q = 0; q < CPT; ++q) acc[c][q] = 0.0;
    if (k_hi >= k_lo) {
        const int64_t beg = d.h_kptr[(int64_t)row * (K + 1) + k_lo - 1];
        const int64_t end = d.h_kptr[(int64_t)row * (K + 1) + k_hi];
        const int64_t nnz = d.h_nnz;
        const int nh = d.nh;
#pragma unroll kUnroll
        for (int64_t i = beg + w * BPW + sub; i < end; i += NW * BPW) {
            const uint32_t cp = __ldcs(d.h_col + i);
            const int k = (int)(cp >> 21), type = (int)((cp >> 20) & 1u), col = (int)(cp & 0xFFFFFu);
            const int64_t wi = (((int64_t)slot_of_k[k] * 2 + type) * nh + col) * 3 * R + cgp * CPT;
            if constexpr (kMixed) {
                // FP32 block values (exact in FP64), FP64 history state and
                // products: rounding the state to FP32 instead costs ~10x the
                // displacement error of rounding the blocks
                const float* v = d.h_val32 + i;
                double m[9];
#pragma unroll
                for (int c = 0; c < 9; ++c) m[c] = (double)__ldcs(v + c * nnz);
                double w0[CPT], w1[CPT], w2[CPT];
                load_cases<CPT>(d.wring + wi, w0);
                load_cases<CPT>(d.wring + wi + R, w1);
                load_cases<CPT>(d.wring + wi + 2 * R, w2);
#pragma unroll
                for (int q = 0; q < CPT; ++q) {
                    acc[0][q] += m[0] * w0[q] + m[1] * w1[q] + m[2] * w2[q];
                    acc[1][q] += m[3] * w0[q] + m[4] * w1[q] + m[5] * w2[q];
                    acc[2][q] += m[6] * w0[q] + m[7] * w1[q] + m[8] * w2[q];
                }
            } else {
                const double* v = d.h_val + i;
                double m[9];
#pragma unroll
                for (int c = 0; c < 9; ++c) m[c] = __ldcs(v + c * nnz);
                double w0[CPT], w1[CPT], w2[CPT];
                load_cases<CPT>(d.wring + wi, w0);
                load_cases<CPT>(d.wring + wi + R, w1);
                load_cases<CPT>(d.wring + wi + 2 * R, w2);
#pragma unroll
                for (int q = 0; q < CPT; ++q) {
                    acc[0][q] += m[0] * w0[q] + m[1] * w1[q] + m[2] * w2[q];
                    acc[1][q] += m[3] * w0[q] + m[4] * w1[q] + m[5] * w2[q];
                    acc[2][q] += m[6] * w0[q] + m[7] * w1[q] + m[8] * w2[q];
                }
            }
        }
    }
    // sum the lanes that share a case group, then the warps
#pragma unroll
    for (int o = 16; o >= TPB && o > 0; o >>= 1)
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int q = 0; q < CPT; ++q) acc[c][q] += __shfl_xor_sync(0xffffffffu, acc[c][q], o);
    if (sub == 0)
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int q = 0; q < CPT; ++q) red[w][c][cgp * CPT + q] = acc[c][q];
    // the KnownM term goes with the pass that covers the step: the history
    // pass beside GMRES when there is one (the head then adds its buffer),
    // else the head
    if (kBulk || !add_bulk) {
        double ka[3];
        known_share<R, NW>(d, row, step, w, lane, ka);
        __syncwarp();
        if (lane < R)
#pragma unroll
            for (int c = 0; c < 3; ++c) red[w][c][lane] += ka[c];
    }
    __syncthreads();
    const int E = d.E;
    if (threadIdx.x < 3 * R) {
        const int c = threadIdx.x / R, r = threadIdx.x % R;
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < NW; ++q) s += red[q][c][r];
        const int64_t o = (int64_t)(3 * p + c) * R + r;
        double* bulk = d.bulk + (int64_t)(step & 7) * 3 * E * R;
        if constexpr (kBulk) {
            bulk[o] = s;
        } else {
            if (add_bulk) s += bulk[o];
            d.b[o] = s;
            if (d.rec_rhs && r == 0) d.rec_rhs[(int64_t)(step - 1) * 3 * E + 3 * row + c] = s;
        }
    }
}

template <int R, bool kMixed, bool kBulk, int kCpt>
__global__ void __launch_bounds__(kRhsThreads, R >= 8 ? 2 : 3) rhs_kernel(MarchData d, int step, int add_bulk)
{
    rhs_row<R, kMixed, kBulk, kCpt>(d, blockIdx.x, step, add_bulk, d.k_lo, d.k_hi);
}

// ---------------------------------------------------------------------------
// History part k >= kr of the right-hand sides of the T steps t0 .. t0+T-1
// in one pass over the run layout (perm row blockIdx.x; the sums of
// DBEM1/multidomain.cpp:3843-3866 restricted to k >= kr, plus KnownM of each
// step).  Every block is read once for the T steps.  A lane group walks one
// run (one (type, column) pair, steps kf..kl) in increasing k keeping the
// window win[h] = W_{t0+h-k}, h < T, in registers: block k applies win[h] to
// step t0 + h, and moving to k + 1 shifts the window by one and loads only
// W_{t0-k-1}, so a run of n blocks loads n + T - 1 history vectors for T n
// products.  Needs the W slots up to t0 + T - 1 - kr, complete once the GMRES
// of step t0 + T - kr has run: kr = 2T + 1 leaves the T GMRES launches of
// steps t0 - T .. t0 - 1 to run beside.  Window entries of steps not yet
// reached (t0 + h - k < 0, only while t0 < K) are zero.
template <int R, bool kMixed, int kCpt, int T, int kUnroll = T>
__global__ void __launch_bounds__(kRhsThreads, 2) bulk_steps_kernel(MarchData d, int t0)
{
    using L = Lanes<R, kCpt>;
    constexpr int CPT = L::CPT, TPB = L::TPB, BPW = L::BPW;
    constexpr int NW = kRhsThreads / 32, NG = NW * BPW;
    __shared__ double red[NW][T][3][R];
    // runs beside GMRES launches that may set the status word: thread 0's
    // reading is OR-ed across the CTA by the barrier
    if (__syncthreads_or(threadIdx.x == 0 && *(volatile int*)d.status)) return;
    const int row = d.row_of[blockIdx.x];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int sub = lane / TPB, cgp = lane % TPB;
    const int K = d.K, SW = d.SW;
    const int klast = t0 + T - 1 < K ? t0 + T - 1 : K;  // last step of the last sum
    const int64_t nb = d.r_nb;
    const int64_t slot_len = 2LL * d.nh * 3 * R;
    double a[T][3][CPT];
#pragma unroll
    for (int h = 0; h < T; ++h)
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int q = 0; q < CPT; ++q) a[h][c][q] = 0.0;
    const int64_t rb = d.r_ptr[row], re = d.r_ptr[row + 1];
    for (int64_t r = rb + w * BPW + sub; r < re; r += NG) {
        const uint2 mt = __ldg(d.r_meta + r);
        const int kf = (int)(mt.y >> 16);
        const int kl = min(kf + (int)(mt.y & 0xFFFFu) - 1, klast);
        if (kl < kf) continue;
        const int64_t vb = __ldg(d.r_off + r) - kf;  // block of step k at vb + k
        const double* wc = d.wring + ((int64_t)(mt.x >> 20) * d.nh + (mt.x & 0xFFFFFu)) * 3 * R + cgp * CPT;
        double win[T][3][CPT];
        int slot = ((t0 - kf) % SW + SW) % SW;  // slot of W_{t0-k}, k = kf
#pragma unroll
        for (int h = 1; h < T; ++h) {
            if (t0 + h - kf >= 0) {
                const int sh = (slot + h) % SW;
#pragma unroll
                for (int c = 0; c < 3; ++c) load_cases<CPT>(wc + sh * slot_len + c * R, win[h][c]);
            } else {
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int q = 0; q < CPT; ++q) win[h][c][q] = 0.0;
            }
        }
        // steps k <= t0: every window entry is a stored vector
        const int kb = kl < t0 ? kl : t0;
#pragma unroll kUnroll
        for (int k = kf; k <= kb; ++k) {
            double m[9];
            if constexpr (kMixed) {
#pragma unroll
                for (int c = 0; c < 9; ++c) m[c] = (double)__ldg(d.r_val32 + c * nb + vb + k);
            } else {
#pragma unroll
                for (int c = 0; c < 9; ++c) m[c] = __ldg(d.r_val + c * nb + vb + k);
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) load_cases<CPT>(wc + slot * slot_len + c * R, win[0][c]);
            slot = slot == 0 ? SW - 1 : slot - 1;
#pragma unroll
            for (int h = 0; h < T; ++h)
#pragma unroll
                for (int q = 0; q < CPT; ++q)
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        a[h][c][q] += m[3 * c] * win[h][0][q] + m[3 * c + 1] * win[h][1][q] +
                                      m[3 * c + 2] * win[h][2][q];
#pragma unroll
            for (int h = T - 1; h > 0; --h)
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int q = 0; q < CPT; ++q) win[h][c][q] = win[h - 1][c][q];
        }
        // steps t0 < k <= t0 + T - 1 (only while t0 < K): W_{t0-k} does not
        // exist yet, the later steps' sums take the remaining entries
        for (int k = kb + 1 > kf ? kb + 1 : kf; k <= kl; ++k) {
            double m[9];
            if constexpr (kMixed) {
#pragma unroll
                for (int c = 0; c < 9; ++c) m[c] = (double)__ldg(d.r_val32 + c * nb + vb + k);
            } else {
#pragma unroll
                for (int c = 0; c < 9; ++c) m[c] = __ldg(d.r_val + c * nb + vb + k);
            }
#pragma unroll
            for (int h = 1; h < T; ++h)
#pragma unroll
                for (int q = 0; q < CPT; ++q)
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        a[h][c][q] += m[3 * c] * win[h][0][q] + m[3 * c + 1] * win[h][1][q] +
                                      m[3 * c + 2] * win[h][2][q];
#pragma unroll
            for (int h = T - 1; h > 1; --h)
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int q = 0; q < CPT; ++q) win[h][c][q] = win[h - 1][c][q];
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int q = 0; q < CPT; ++q) win[1][c][q] = 0.0;
        }
    }
    // sum the lanes that share a case group, then the warps
#pragma unroll
    for (int o = 16; o >= TPB && o > 0; o >>= 1)
#pragma unroll
        for (int h = 0; h < T; ++h)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int q = 0; q < CPT; ++q) a[h][c][q] += __shfl_xor_sync(0xffffffffu, a[h][c][q], o);
    if (sub == 0)
#pragma unroll
        for (int h = 0; h < T; ++h)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int q = 0; q < CPT; ++q) red[w][h][c][cgp * CPT + q] = a[h][c][q];
    // the KnownM terms of the T steps
    __syncwarp();
#pragma unroll 1
    for (int h = 0; h < T; ++h) {
        if (t0 + h > d.nstep) break;
        double ka[3];
        known_share<R, NW>(d, row, t0 + h, w, lane, ka);
        if (lane < R)
#pragma unroll
            for (int c = 0; c < 3; ++c) red[w][h][c][lane] += ka[c];
    }
    __syncthreads();
    const int64_t E3R = 3LL * d.E * R;
    for (int t = threadIdx.x; t < 3 * T * R; t += blockDim.x) {
        const int h = t / (3 * R), c = (t / R) % 3, r = t % R;
        if (t0 + h > d.nstep) continue;
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < NW; ++q) s += red[q][h][c][r];
        d.bulk[(int64_t)((t0 + h) & 7) * E3R + (int64_t)(3 * blockIdx.x + c) * R + r] = s;
    }
}

// Copy one model's MarchData into shared memory (several models per launch).
__device__ __forceinline__ void load_model(const MarchData* ds, int m, MarchData& sd)
{
    const int* src = reinterpret_cast<const int*>(ds + m);
    int* dst = reinterpret_cast<int*>(&sd);
    for (int i = threadIdx.x; i < (int)(sizeof(MarchData) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
}

// Several models' right-hand sides of one step in one launch: CTA b serves
// perm row b - row_off[m] of model m (row_off[m] <= b < row_off[m+1]); models
// whose march is shorter skip.  With kBulk the history steps 3..min(step, K_m)
// and KnownM go to the model's bulk buffer (computed one step ahead, beside
// GMRES); otherwise the head: k <= min(step, K_m, kmax_head) plus that bulk
// when k = 3.. applies (kmax_head = 2; KnownM itself before that), or KnownM
// and every history step (kmax_head = K_m).
template <int R, bool kMixed, bool kBulk, int kCpt>
__global__ void __launch_bounds__(kRhsThreads, R >= 8 ? 2 : 3) rhs_models_kernel(const MarchData* ds, const int* row_off,
                                                                                  int n_models, int step, int split)
{
    int lo = 0, hi = n_models - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((int)blockIdx.x >= row_off[mid]) lo = mid;
        else hi = mid - 1;
    }
    __shared__ MarchData sd;
    load_model(ds, lo, sd);
    if (step > sd.nstep) return;
    const int kcap = step > 1 ? (step < sd.K ? step : sd.K) : 0;
    const int p = (int)blockIdx.x - row_off[lo];
    if constexpr (kBulk) {
        if (kcap >= 3) rhs_row<R, kMixed, true, kCpt>(sd, p, step, 0, 3, kcap);
    } else if (split) {
        rhs_row<R, kMixed, false, kCpt>(sd, p, step, kcap >= 3 ? 1 : 0, 1, kcap < 2 ? kcap : 2);
    } else {
        rhs_row<R, kMixed, false, kCpt>(sd, p, step, 0, 1, kcap);
    }
}

// ---------------------------------------------------------------------------
// Transposed history convolution of the adjoint march at step n:
//   adj[type][c] = sum_k sum_r B(r, k, type, c)^T Omega_{n,k}[r]
//   Omega_{n,k} = lam_{n+k-1} (k >= 2) + 2 lam_{n+k} + lam_{n+k+1}, steps <= N,
// the transpose of the forward sum over k of B . (X_{s-k+1} + 2 X_{s-k} +
// X_{s-k-1}) (DBEM1/multidomain.cpp:3201-3225, 3843-3866) with B the stacked
// blocks (MTS negated).  Column-major view: one warp per (type, column), its
// blocks ordered by k.
__global__ void __launch_bounds__(256) adj_history_kernel(int N, int n, int K, int nh, int E, const int64_t* tptr,
                                                          const int32_t* trow, const double* tval, const double* lam,
                                                          double* adj)
{
    const int64_t seg = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (seg >= 2LL * nh) return;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int k = 1; k <= K; ++k) {
        const int64_t b = tptr[seg * (K + 1) + k - 1], e = tptr[seg * (K + 1) + k];
        if (b == e) continue;
        const int m0 = n + k - 1, m1 = n + k, m2 = n + k + 1;
        const double c0 = (k >= 2 && m0 <= N) ? 1.0 : 0.0, c1 = m1 <= N ? 2.0 : 0.0, c2 = m2 <= N ? 1.0 : 0.0;
        if (c0 == 0.0 && c1 == 0.0 && c2 == 0.0) continue;
        for (int64_t j = b + lane; j < e; j += 32) {
            const int64_t r = trow[j];
            double w[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double v = 0.0;
                if (c0 != 0.0) v += lam[((int64_t)m0 * E + r) * 3 + c];
                if (c1 != 0.0) v += c1 * lam[((int64_t)m1 * E + r) * 3 + c];
                if (c2 != 0.0) v += lam[((int64_t)m2 * E + r) * 3 + c];
                w[c] = v;
            }
            const double* B = tval + 9 * j;  // row-major B; B^T w
            a0 += B[0] * w[0] + B[3] * w[1] + B[6] * w[2];
            a1 += B[1] * w[0] + B[4] * w[1] + B[7] * w[2];
            a2 += B[2] * w[0] + B[5] * w[1] + B[8] * w[2];
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if (lane == 0) {
        adj[3 * seg] = a0;
        adj[3 * seg + 1] = a1;
        adj[3 * seg + 2] = a2;
    }
}

cudaError_t adj_history(int N, int n, int K, int nh, int E, const int64_t* tptr, const int32_t* trow,
                        const double* tval, const double* lam, double* adj, cudaStream_t s)
{
    const int64_t segs = 2LL * nh;
    adj_history_kernel<<<(int)((segs + 7) / 8), 256, 0, s>>>(N, n, K, nh, E, tptr, trow, tval, lam, adj);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
namespace {

// Per-CTA shared state of the cluster GMRES.
template <int R>
struct GShared {
    double part[2][kDotMax][R];          // this CTA's partial sums (read by peers)
    double wred[kGmresWarps][kDotMax][R];
    double vals[kDotMax][R];             // cluster-reduced values of a vector reduction
    double val[R];                       // cluster-reduced value of a scalar reduction
    double h1[R], phibar[R], f[R], n2b[R], normr[R], nn[R], hn[R];
    int run[R], flag[R], inner[R], cycles[R], stag[R], check[R], exact[R];
    int any, any_exact;
    int abort_src;  // the status word as cluster rank 0 read it
    int abort;      // rank 0's reading, copied by every CTA of the cluster
};

// Cluster-wide sums of m values per load case (m <= M <= kDotMax): thread t
// contributes v[q] to value q of case t % R.  Every CTA adds the C partials
// in rank order, so all hold the same results, in vals[q][case].  One
// cluster barrier; the two partial slots alternate so a peer still reading
// the previous reduction's slot is never overwritten.
template <int R, int M>
__device__ void cluster_sum_vec(double (&v)[M], int m, int& slot, GShared<R>& s, cg::cluster_group& cl)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < M; ++q) {
        if (q < m) {
#pragma unroll
            for (int o = 16; o >= R && o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
            if (lane < R) s.wred[w][q][lane] = v[q];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < m * R; i += blockDim.x) {
        const int q = i / R, r = i % R;
        double t = 0.0;
#pragma unroll
        for (int ww = 0; ww < kGmresWarps; ++ww) t += s.wred[ww][q][r];
        s.part[slot][q][r] = t;
    }
    cl.sync();
    const int C = (int)cl.num_blocks();
    for (int i = threadIdx.x; i < m * R; i += blockDim.x) {
        const int q = i / R, r = i % R;
        double t = 0.0;
        for (int c = 0; c < C; ++c) t += *cl.map_shared_rank(&s.part[slot][q][r], c);
        s.vals[q][r] = t;
    }
    __syncthreads();
    slot ^= 1;
}

// Cluster-wide sum per load case of one value, in val[case].
template <int R>
__device__ void cluster_sum(double v, int& slot, GShared<R>& s, cg::cluster_group& cl)
{
    double a[1] = {v};
    cluster_sum_vec<R, 1>(a, 1, slot, s, cl);
    if (threadIdx.x < R) s.val[threadIdx.x] = s.vals[0][threadIdx.x];
    __syncthreads();
}

// y[(3p+c)R + r] = (A' v)[p] for the owned perm rows p in [lo, hi), all cases.
// A warp works on RPW rows at once, LPR lanes per row (BPR blocks of a row
// in flight, TPB lanes per block for the load cases).
template <int R, bool kF32>
__device__ void spmm_owned(const MarchData& d, const double* v, int lo, int hi, double* y)
{
    using L = Lanes<R>;
    constexpr int CPT = L::CPT, TPB = L::TPB;
    constexpr int BPR = TPB >= 8 ? 1 : 8 / TPB;
    constexpr int LPR = TPB * BPR;
    constexpr int RPW = 32 / LPR;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int rsub = lane / LPR, l2 = lane % LPR;
    const int bsub = l2 / TPB, cgp = l2 % TPB;
    for (int p0 = lo + w * RPW; p0 < hi; p0 += kGmresWarps * RPW) {
        const int p = p0 + rsub;
        double acc[3][CPT];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int q = 0; q < CPT; ++q) acc[c][q] = 0.0;
        if (p < hi) {
            const int jb = d.a_rp[p], je = d.a_rp[p + 1];
#pragma unroll 2
            for (int j = jb + bsub; j < je; j += BPR) {
                const int col = d.a_col[j];
                double x0[CPT], x1[CPT], x2[CPT];
                ldcg_cases<CPT>(v + (int64_t)(3 * col) * R + cgp * CPT, x0);
                ldcg_cases<CPT>(v + (int64_t)(3 * col + 1) * R + cgp * CPT, x1);
                ldcg_cases<CPT>(v + (int64_t)(3 * col + 2) * R + cgp * CPT, x2);
                if constexpr (kF32) {
                    const float* a = d.a_val32 + 9 * (int64_t)j;
#pragma unroll
                    for (int q = 0; q < CPT; ++q) {
                        const float f0 = (float)x0[q], f1 = (float)x1[q], f2 = (float)x2[q];
                        acc[0][q] += (double)(a[0] * f0 + a[1] * f1 + a[2] * f2);
                        acc[1][q] += (double)(a[3] * f0 + a[4] * f1 + a[5] * f2);
                        acc[2][q] += (double)(a[6] * f0 + a[7] * f1 + a[8] * f2);
                    }
                } else {
                    const double* a = d.a_val + 9 * (int64_t)j;
#pragma unroll
                    for (int q = 0; q < CPT; ++q) {
                        acc[0][q] += a[0] * x0[q] + a[1] * x1[q] + a[2] * x2[q];
                        acc[1][q] += a[3] * x0[q] + a[4] * x1[q] + a[5] * x2[q];
                        acc[2][q] += a[6] * x0[q] + a[7] * x1[q] + a[8] * x2[q];
                    }
                }
            }
        }
        // sum the BPR lane groups of a row (lanes differing in the bsub bits)
#pragma unroll
        for (int o = TPB; o < LPR; o <<= 1)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int q = 0; q < CPT; ++q) acc[c][q] += __shfl_xor_sync(0xffffffffu, acc[c][q], o);
        if (p < hi && bsub == 0)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int q = 0; q < CPT; ++q) y[(int64_t)(3 * p + c) * R + cgp * CPT + q] = acc[c][q];
    }
    __syncthreads();
}

// out = M^-1 in on the owned leaves (block-diagonal leaf inverses,
// GMRES_M_X, DBEM1/pre_gmres.cpp:837-895; sum over k then n as the
// reference).  One thread per owned output value and load case.
template <int R, bool kF32>
__device__ void precond_owned(const MarchData& d, int lo, int hi, const double* in, double* out)
{
    const int64_t nout = 3LL * (hi - lo) * R;
    for (int64_t t = threadIdx.x; t < nout; t += blockDim.x) {
        const int r = (int)(t % R);
        const int e = (int)(t / R);           // owned value index
        const int p = lo + e / 3, c = e % 3;  // perm row and component
        const int L = d.leaf_of_perm[p];
        const int b = d.leaf_begin[L], n3 = 3 * d.leaf_count[L];
        const int rr = 3 * (p - b) + c;
        const double* src = in + (int64_t)(3 * b) * R + r;
        double s = 0.0;
        if constexpr (kF32) {
            const float* m = d.pinv32 + d.leaf_off[L] + (int64_t)rr * n3;
            for (int q = 0; q < n3; ++q) s += (double)(m[q] * (float)src[(int64_t)q * R]);
        } else {
            const double* m = d.pinv + d.leaf_off[L] + (int64_t)rr * n3;
            for (int q = 0; q < n3; ++q) s += m[q] * src[(int64_t)q * R];
        }
        out[(int64_t)(3 * lo) * R + t] = s;
    }
    __syncthreads();
}

// spmm_owned with v read from the cluster's shared-memory copies: vs is this
// CTA's copy of its owned values ([3][R] per row, from its first row); the
// owner and the row within the owner's range come packed in a_colx.  The
// result goes to y (global) and, when ys is not null, to this CTA's
// shared-memory copy.
template <int R, bool kF32>
__device__ void spmm_owned_dsm(const MarchData& d, const double* vs, int lo, int hi, double* y, double* ys,
                               cg::cluster_group& cl)
{
    using L = Lanes<R>;
    constexpr int CPT = L::CPT, TPB = L::TPB;
    constexpr int BPR = TPB >= 8 ? 1 : 8 / TPB;
    constexpr int LPR = TPB * BPR;
    constexpr int RPW = 32 / LPR;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int rsub = lane / LPR, l2 = lane % LPR;
    const int bsub = l2 / TPB, cgp = l2 % TPB;
    for (int p0 = lo + w * RPW; p0 < hi; p0 += kGmresWarps * RPW) {
        const int p = p0 + rsub;
        double acc[3][CPT];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int q = 0; q < CPT; ++q) acc[c][q] = 0.0;
        if (p < hi) {
            const int jb = d.a_rp[p], je = d.a_rp[p + 1];
#pragma unroll 2
            for (int j = jb + bsub; j < je; j += BPR) {
                const int cx = d.a_colx[j];
                const double* src = cl.map_shared_rank(vs, cx >> 24) + (int64_t)(3 * (cx & 0xFFFFFF)) * R + cgp * CPT;
                double x0[CPT], x1[CPT], x2[CPT];
                load_cases<CPT>(src, x0);
                load_cases<CPT>(src + R, x1);
                load_cases<CPT>(src + 2 * R, x2);
                if constexpr (kF32) {
                    const float* a = d.a_val32 + 9 * (int64_t)j;
#pragma unroll
                    for (int q = 0; q < CPT; ++q) {
                        const float f0 = (float)x0[q], f1 = (float)x1[q], f2 = (float)x2[q];
                        acc[0][q] += (double)(a[0] * f0 + a[1] * f1 + a[2] * f2);
                        acc[1][q] += (double)(a[3] * f0 + a[4] * f1 + a[5] * f2);
                        acc[2][q] += (double)(a[6] * f0 + a[7] * f1 + a[8] * f2);
                    }
                } else {
                    const double* a = d.a_val + 9 * (int64_t)j;
#pragma unroll
                    for (int q = 0; q < CPT; ++q) {
                        acc[0][q] += a[0] * x0[q] + a[1] * x1[q] + a[2] * x2[q];
                        acc[1][q] += a[3] * x0[q] + a[4] * x1[q] + a[5] * x2[q];
                        acc[2][q] += a[6] * x0[q] + a[7] * x1[q] + a[8] * x2[q];
                    }
                }
            }
        }
#pragma unroll
        for (int o = TPB; o < LPR; o <<= 1)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int q = 0; q < CPT; ++q) acc[c][q] += __shfl_xor_sync(0xffffffffu, acc[c][q], o);
        if (p < hi && bsub == 0)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int q = 0; q < CPT; ++q) {
                    y[(int64_t)(3 * p + c) * R + cgp * CPT + q] = acc[c][q];
                    if (ys) ys[(int64_t)(3 * (p - lo) + c) * R + cgp * CPT + q] = acc[c][q];
                }
    }
    __syncthreads();
}

// precond_owned reading its input from this CTA's shared-memory copy
// (owned values relative to the first owned row): every leaf lies inside
// one CTA's range.
template <int R, bool kF32>
__device__ void precond_owned_smem(const MarchData& d, int lo, int hi, const double* in_s, double* out)
{
    const int64_t nout = 3LL * (hi - lo) * R;
    for (int64_t t = threadIdx.x; t < nout; t += blockDim.x) {
        const int r = (int)(t % R);
        const int e = (int)(t / R);
        const int p = lo + e / 3, c = e % 3;
        const int L = d.leaf_of_perm[p];
        const int b = d.leaf_begin[L], n3 = 3 * d.leaf_count[L];
        const int rr = 3 * (p - b) + c;
        const double* src = in_s + (int64_t)(3 * (b - lo)) * R + r;
        double s0 = 0.0, s1 = 0.0;
        if constexpr (kF32) {
            const float* m = d.pinv32 + d.leaf_off[L] + (int64_t)rr * n3;
            int q = 0;
            for (; q + 1 < n3; q += 2) {
                s0 += (double)(m[q] * (float)src[(int64_t)q * R]);
                s1 += (double)(m[q + 1] * (float)src[(int64_t)(q + 1) * R]);
            }
            if (q < n3) s0 += (double)(m[q] * (float)src[(int64_t)q * R]);
        } else {
            const double* m = d.pinv + d.leaf_off[L] + (int64_t)rr * n3;
            // the reference's order: one running sum over the leaf's columns
            for (int q = 0; q < n3; ++q) s0 += m[q] * src[(int64_t)q * R];
        }
        out[(int64_t)(3 * lo) * R + t] = s0 + s1;
    }
    __syncthreads();
}

// Mixed-precision forms of the two products above for the Arnoldi step: the
// Krylov vector V_j and the product A' V_j are mirrored in shared memory as
// FP32, the FP32 blocks and leaf inverses multiply them with FP32
// accumulation, and each output is converted to FP64 once.  (Converting
// every FP64 operand to FP32 and every FP32 product back, as the FP64
// mirrors needed, cost about as much as the products.)  The Arnoldi
// iteration only preconditions the FP64 refinement, which checks every
// solution on the FP64 residual.
template <int R>
__device__ void spmm_owned_dsm32(const MarchData& d, const float* vs, int lo, int hi, double* y, float* ys,
                                 cg::cluster_group& cl)
{
    using L = Lanes<R>;
    constexpr int CPT = L::CPT, TPB = L::TPB;
    constexpr int BPR = TPB >= 8 ? 1 : 8 / TPB;
    constexpr int LPR = TPB * BPR;
    constexpr int RPW = 32 / LPR;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int rsub = lane / LPR, l2 = lane % LPR;
    const int bsub = l2 / TPB, cgp = l2 % TPB;
    for (int p0 = lo + w * RPW; p0 < hi; p0 += kGmresWarps * RPW) {
        const int p = p0 + rsub;
        float acc[3][CPT];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int q = 0; q < CPT; ++q) acc[c][q] = 0.0f;
        if (p < hi) {
            const int jb = d.a_rp[p], je = d.a_rp[p + 1];
#pragma unroll 2
            for (int j = jb + bsub; j < je; j += BPR) {
                const int cx = d.a_colx[j];
                const float* src = cl.map_shared_rank(vs, cx >> 24) + (int64_t)(3 * (cx & 0xFFFFFF)) * R + cgp * CPT;
                float x0[CPT], x1[CPT], x2[CPT];
                load_cases<CPT>(src, x0);
                load_cases<CPT>(src + R, x1);
                load_cases<CPT>(src + 2 * R, x2);
                const float* a = d.a_val32 + 9 * (int64_t)j;
#pragma unroll
                for (int q = 0; q < CPT; ++q) {
                    acc[0][q] += a[0] * x0[q] + a[1] * x1[q] + a[2] * x2[q];
                    acc[1][q] += a[3] * x0[q] + a[4] * x1[q] + a[5] * x2[q];
                    acc[2][q] += a[6] * x0[q] + a[7] * x1[q] + a[8] * x2[q];
                }
            }
        }
#pragma unroll
        for (int o = TPB; o < LPR; o <<= 1)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int q = 0; q < CPT; ++q) acc[c][q] += __shfl_xor_sync(0xffffffffu, acc[c][q], o);
        if (p < hi && bsub == 0)
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int q = 0; q < CPT; ++q) {
                    y[(int64_t)(3 * p + c) * R + cgp * CPT + q] = (double)acc[c][q];
                    ys[(int64_t)(3 * (p - lo) + c) * R + cgp * CPT + q] = acc[c][q];
                }
    }
    __syncthreads();
}

template <int R>
__device__ void precond_owned_smem32(const MarchData& d, int lo, int hi, const float* in_s, double* out)
{
    const int64_t nout = 3LL * (hi - lo) * R;
    for (int64_t t = threadIdx.x; t < nout; t += blockDim.x) {
        const int r = (int)(t % R);
        const int e = (int)(t / R);
        const int p = lo + e / 3, c = e % 3;
        const int L = d.leaf_of_perm[p];
        const int b = d.leaf_begin[L], n3 = 3 * d.leaf_count[L];
        const int rr = 3 * (p - b) + c;
        const float* src = in_s + (int64_t)(3 * (b - lo)) * R + r;
        const float* m = d.pinv32 + d.leaf_off[L] + (int64_t)rr * n3;
        float s0 = 0.0f, s1 = 0.0f;
        int q = 0;
        for (; q + 1 < n3; q += 2) {
            s0 += m[q] * src[(int64_t)q * R];
            s1 += m[q + 1] * src[(int64_t)(q + 1) * R];
        }
        if (q < n3) s0 += m[q] * src[(int64_t)q * R];
        out[(int64_t)(3 * lo) * R + t] = (double)(s0 + s1);
    }
    __syncthreads();
}

}  // namespace

// GMRES for the R load cases of one step on one thread-block cluster, then
// the write-back.  Case r stops updating once converged; the cluster stops
// when every case has.  FP64 mode checks the true residual b - A x after
// every inner step (maxit = 1, as the reference).  Mixed mode runs the
// Arnoldi SpMM and the preconditioner in FP32, keeps orthogonalisation,
// Givens and the residual recurrence r -= f_j A W_j in FP64, and restarts
// from the explicit FP64 residual until it meets the tolerance.
template <int R, bool kMixed>
__device__ __forceinline__ void gmres_body(const MarchData& d, const int step, const int grp)
{
    cg::cluster_group cl = cg::this_cluster();
    __shared__ GShared<R> s;
    // Another cluster of the same launch (another load-case group) may set
    // the status word at any time, so CTAs reading it separately could
    // disagree and leave peers waiting at a cluster barrier.  Rank 0 reads it
    // once; every CTA copies that reading through distributed shared memory;
    // the second barrier keeps rank 0 resident until all copies are taken.
    if (threadIdx.x == 0 && cl.block_rank() == 0) s.abort_src = *(volatile int*)d.status;
    cl.sync();
    if (threadIdx.x == 0) s.abort = *cl.map_shared_rank(&s.abort_src, 0);
    cl.sync();
    if (s.abort) return;  // uniform over the cluster
    const int cq = (int)cl.block_rank();
    const int C = (int)cl.num_blocks();
    // grp: cluster = group of load cases
    const int RT = d.R, roff = grp * R;          // total cases, first case of this group
    const int E = d.E, rs = d.restart;
    const int64_t n = 3LL * E * R;           // elements of one private vector
    const int L0 = d.cta_leaf[cq], L1 = d.cta_leaf[cq + 1];
    const int lo = L0 < L1 ? d.leaf_begin[L0] : 0;
    const int hi = L0 < L1 ? d.leaf_begin[L1 - 1] + d.leaf_count[L1 - 1] : 0;
    const int64_t ob = 3LL * lo * R, oe = 3LL * hi * R;  // owned element range
    double* G = d.givens + ((int64_t)grp * C + cq) * R * d.givens_stride;
    auto gcs = [&](int r) { return G + (int64_t)r * d.givens_stride; };
    // givens layout per case: cs[rs+2], sn[rs+2], h[rs+2], rcol[rs+2]
    const int gl = rs + 2;
    int slot = 0;
    double* b = d.bp + (int64_t)grp * n;
    double* x = d.x + (int64_t)grp * n;
    double* rv = d.rv + (int64_t)grp * n;
    double* u = d.u + (int64_t)grp * n;
    double* const Vb = d.V + (int64_t)grp * (rs + 1) * n;
    double* const Wb = d.W + (int64_t)grp * (rs + 1) * n;
    double* const AWb = d.AW + (int64_t)grp * (rs + 1) * n;
    // Krylov vector copies in shared memory (when d.dsm_rows > 0): V_j and
    // V_{j+1} alternate in vs[0], vs[1]; xsm mirrors x; aws holds A V_j for
    // the preconditioner.  Peers read vs and xsm through distributed shared
    // memory in the sparse products.
    extern __shared__ __align__(16) double dsm[];
    const bool use_dsm = d.dsm_rows > 0;
    const int64_t S = 3LL * d.dsm_rows * R;
    // FP64 mode: vs[0], vs[1], xsm, aws, all FP64; mixed mode: xsm in FP64,
    // then FP32 mirrors vs32[0], vs32[1] of V_j and aws32 of A' V_j (mirror i
    // at base + i S: offsets, not pointer arrays, which would live in local
    // memory)
    double* const vs64 = dsm;
    double* const xsm = kMixed ? dsm : dsm + 2 * S;
    double* const aws = dsm + 3 * S;
    float* const vs32 = reinterpret_cast<float*>(dsm + S);
    float* const aws32 = vs32 + 2 * S;
    // private copy of this group's right-hand side columns
    for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x)
        b[t] = d.b[(t / R) * RT + roff + (t % R)];
    __syncthreads();

    double part = 0.0;
    // mixed mode starts from the solutions of the previous steps extrapolated
    // linearly (x_{s-1} at step 2); the FP64 path starts from zero as the
    // reference does (DBEM1/multidomain.cpp:3869-3870)
    const bool warm = kMixed && d.xold != nullptr && step >= 2;
    double* xold = warm ? d.xold + (int64_t)grp * n : nullptr;
    if (!warm) {
        for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x) {
            x[t] = 0.0;
            if (use_dsm) xsm[t - ob] = 0.0;
            if (kMixed && d.xold) d.xold[(int64_t)grp * n + t] = 0.0;
            const double bb = b[t];
            rv[t] = bb;
            part += bb * bb;
        }
        cluster_sum<R>(part, slot, s, cl);
        if (threadIdx.x < R) {
            const int r = threadIdx.x;
            s.n2b[r] = sqrt(s.val[r]);
            const double tolb = d.tol * s.n2b[r];
            s.flag[r] = (s.n2b[r] == 0.0 || s.n2b[r] <= tolb) ? 0 : 1;
            s.inner[r] = 0;
            s.cycles[r] = 0;
        }
        __syncthreads();
    } else {
        for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x) {
            const double x1 = x[t], x2 = xold[t];
            const double x0 = step == 2 ? x1 : 2.0 * x1 - x2;
            xold[t] = x1;
            x[t] = x0;
            if (use_dsm) xsm[t - ob] = x0;
        }
        cl.sync();  // the start vector is complete in every CTA
        if (use_dsm)
            spmm_owned_dsm<R, false>(d, xsm, lo, hi, u, nullptr, cl);
        else
            spmm_owned<R, false>(d, x, lo, hi, u);
        double acc[2] = {0.0, 0.0};
        for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x) {
            const double bb = b[t], rr = bb - u[t];
            rv[t] = rr;
            acc[0] += bb * bb;
            acc[1] += rr * rr;
        }
        cluster_sum_vec<R, 2>(acc, 2, slot, s, cl);
        if (threadIdx.x < R) {
            const int r = threadIdx.x;
            s.n2b[r] = sqrt(s.vals[0][r]);
            const double tolb = d.tol * s.n2b[r];
            s.flag[r] = (s.n2b[r] == 0.0 || sqrt(s.vals[1][r]) <= tolb) ? 0 : 1;
            s.inner[r] = 0;
            s.cycles[r] = 0;
        }
        __syncthreads();
    }
    const int max_cycles = kMixed ? 8 : 1;
    for (int cycle = 0; cycle < max_cycles; ++cycle) {
        if (threadIdx.x == 0) {
            int a = 0;
            for (int r = 0; r < R; ++r) a |= s.flag[r] == 1;
            s.any = a;
        }
        __syncthreads();
        if (!s.any) break;
        // vh = M^-1 r, V_1 = vh / |vh|, x0 kept in W's last column
        precond_owned<R, kMixed>(d, lo, hi, rv, u);
        part = 0.0;
        for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x) part += u[t] * u[t];
        cluster_sum<R>(part, slot, s, cl);
        if (threadIdx.x < R) {
            const int r = threadIdx.x;
            s.h1[r] = sqrt(s.val[r]);
            s.phibar[r] = s.h1[r];
            s.run[r] = s.flag[r] == 1;
            s.stag[r] = 0;
            if (s.run[r]) s.cycles[r]++;
        }
        __syncthreads();
        double* X0 = Wb + (int64_t)rs * n;
        static_assert(kGmresThreads % R == 0, "a thread's values all belong to one case");
        const int tr0 = (int)((ob + threadIdx.x) % R);  // the case of every value this thread owns
        const bool run0 = s.run[tr0] != 0;
        const double inv_h1 = run0 ? 1.0 / s.h1[tr0] : 0.0;
        for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x) {
            const double v1 = run0 ? u[t] * inv_h1 : 0.0;
            Vb[t] = v1;
            if (use_dsm) {
                if constexpr (kMixed) vs32[t - ob] = (float)v1;
                else vs64[t - ob] = v1;
            }
            X0[t] = x[t];
        }
        cl.sync();  // V_1 complete
        for (int j = 1; j <= rs; ++j) {
            if (threadIdx.x == 0) {
                int a = 0;
                for (int r = 0; r < R; ++r) a |= s.run[r];
                s.any = a;
            }
            __syncthreads();
            if (!s.any) break;
            const double* Vj = Vb + (int64_t)(j - 1) * n;
            double* AWj = AWb + (int64_t)(j - 1) * n;
            if (use_dsm) {
                if constexpr (kMixed) {
                    spmm_owned_dsm32<R>(d, vs32 + ((j - 1) & 1) * S, lo, hi, AWj, aws32, cl);  // A V_j
                    precond_owned_smem32<R>(d, lo, hi, aws32, u);                             // u = M^-1 A V_j
                } else {
                    spmm_owned_dsm<R, false>(d, vs64 + ((j - 1) & 1) * S, lo, hi, AWj, aws, cl);
                    precond_owned_smem<R, false>(d, lo, hi, aws, u);
                }
            } else {
                spmm_owned<R, kMixed>(d, Vj, lo, hi, AWj);
                precond_owned<R, kMixed>(d, lo, hi, AWj, u);
            }
            // Classical Gram-Schmidt applied twice (CGS2): each sweep over the
            // owned values handles up to kDotChunk basis vectors and ends in
            // one cluster reduction, instead of one reduction per basis
            // vector as in MGS (DBEM1/pre_gmres.cpp:1462-1485).  The basis
            // and the Hessenberg column are MGS's up to rounding.
            const int tr = (int)((ob + threadIdx.x) % R);  // the case of every value this thread owns
            const double* hcol = gcs(tr) + 2 * gl;
            const double* ccol = gcs(tr) + 4 * gl;
            // sweep 1: h_k = V_k . u
            for (int k0 = 1; k0 <= j; k0 += kDotChunk) {
                const int nk = min(kDotChunk, j - k0 + 1);
                double acc[kDotChunk];
#pragma unroll
                for (int q = 0; q < kDotChunk; ++q) acc[q] = 0.0;
                for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x) {
                    const double ut = u[t];
#pragma unroll
                    for (int q = 0; q < kDotChunk; ++q)
                        if (q < nk) acc[q] += Vb[(int64_t)(k0 - 1 + q) * n + t] * ut;
                }
                cluster_sum_vec<R, kDotChunk>(acc, nk, slot, s, cl);
                for (int i = threadIdx.x; i < nk * R; i += blockDim.x)
                    gcs(i % R)[2 * gl + k0 + i / R] = s.vals[i / R][i % R];
                __syncthreads();
            }
            // sweep 2: u' = u - sum_k h_k V_k (kept in u), c_k = V_k . u',
            // and |u'|^2 with the first chunk
            for (int k0 = 1; k0 <= j; k0 += kDotChunk) {
                const int nk = min(kDotChunk, j - k0 + 1);
                double acc[kDotMax];
#pragma unroll
                for (int q = 0; q < kDotMax; ++q) acc[q] = 0.0;
                for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x) {
                    double ut = u[t];
                    if (k0 == 1) {
#pragma unroll 4
                        for (int k = 1; k <= j; ++k) ut -= hcol[k] * Vb[(int64_t)(k - 1) * n + t];
                        u[t] = ut;
                        acc[kDotChunk] += ut * ut;
                    }
#pragma unroll
                    for (int q = 0; q < kDotChunk; ++q)
                        if (q < nk) acc[q] += Vb[(int64_t)(k0 - 1 + q) * n + t] * ut;
                }
                cluster_sum_vec<R, kDotMax>(acc, k0 == 1 ? kDotMax : nk, slot, s, cl);
                for (int i = threadIdx.x; i < nk * R; i += blockDim.x)
                    gcs(i % R)[4 * gl + k0 + i / R] = s.vals[i / R][i % R];
                if (k0 == 1 && threadIdx.x < R) s.nn[threadIdx.x] = s.vals[kDotChunk][threadIdx.x];
                __syncthreads();
            }
            // h(k, j) = h_k + c_k; |u''|^2 = |u'|^2 - sum c_k^2 unless that
            // cancels (near breakdown): then u'' and its norm explicitly
            if (threadIdx.x < R) {
                const int r = threadIdx.x;
                double* h = gcs(r) + 2 * gl;
                const double* c = gcs(r) + 4 * gl;
                double cc = 0.0;
                for (int k = 1; k <= j; ++k) {
                    cc += c[k] * c[k];
                    h[k] += c[k];
                }
                const double est = s.nn[r] - cc;
                s.exact[r] = !(est > 1.0e-4 * s.nn[r]);
                s.hn[r] = s.exact[r] ? 0.0 : sqrt(est);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                int a = 0;
                for (int r = 0; r < R; ++r) a |= s.exact[r];
                s.any_exact = a;
            }
            __syncthreads();
            if (s.any_exact) {
                part = 0.0;
                for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x) {
                    double ut = u[t];
                    for (int k = 1; k <= j; ++k) ut -= ccol[k] * Vb[(int64_t)(k - 1) * n + t];
                    u[t] = ut;
                    part += ut * ut;
                }
                cluster_sum<R>(part, slot, s, cl);
                if (threadIdx.x < R) s.hn[threadIdx.x] = sqrt(s.val[threadIdx.x]);
                __syncthreads();
            }
            // Givens: R(1:j, j) = G_{j-1}..G_1 h(1:j), new rotation from (R(j,j), h(j+1))
            if (threadIdx.x < R) {
                const int r = threadIdx.x;
                double* cs = gcs(r);
                double* sn = cs + gl;
                double* h = sn + gl;
                double* rc = h + gl;
                const double hn = s.hn[r];
                h[j + 1] = hn;
                for (int k = 1; k <= j; ++k) rc[k] = h[k];
                for (int i = 1; i < j; ++i) {
                    const double a = rc[i], bb = rc[i + 1];
                    rc[i] = cs[i] * a - sn[i] * bb;
                    rc[i + 1] = sn[i] * a + cs[i] * bb;
                }
                const double rt = rc[j];
                double c, sv, temp;
                if (hn == 0.0) {
                    c = 1.0;
                    sv = 0.0;
                } else if (hn * hn > rt * rt) {
                    temp = rt / hn;
                    sv = 1.0 / sqrt(1.0 + fabs(temp) * fabs(temp));
                    c = -temp * sv;
                } else {
                    temp = hn / rt;
                    c = 1.0 / sqrt(1.0 + fabs(temp) * fabs(temp));
                    sv = -temp * c;
                }
                rc[j] = c * rt - sv * hn;
                cs[j] = c;
                sn[j] = sv;
                s.f[r] = c * s.phibar[r];
                s.phibar[r] = sv * s.phibar[r];
                if (s.run[r] && s.f[r] == 0.0) s.stag[r] = 1;
            }
            __syncthreads();
            // sweep 3: V_{j+1} = (u' - sum_k c_k V_k) / h(j+1, j) (zero when
            // h(j+1, j) <= 1e-12, DBEM1/pre_gmres.cpp:1481-1485);
            // W_j = (V_j - sum_l W_l R(l,j)) / R(j,j); x += f_j W_j; the same
            // recurrence on A V_j gives A W_j and the residual r -= f_j A W_j
            double* Vn = Vb + (int64_t)j * n;
            double* const vsn = vs64 + (j & 1) * S;
            float* const vsn32 = vs32 + (j & 1) * S;
            double* Wj = Wb + (int64_t)(j - 1) * n;
            const bool sub = !s.any_exact;
            const double hn_t = s.hn[tr];
            const bool run_t = s.run[tr] != 0;
            const double f_t = s.f[tr];
            const double* rc_t = gcs(tr) + 3 * gl;
            // one reciprocal per case and step: every value this thread owns
            // belongs to case tr, so the loops below multiply instead of
            // dividing (FP64 division is a long instruction sequence)
            const double inv_rjj = 1.0 / rc_t[j];
            const bool vzero = hn_t <= 1.0e-12;
            const double inv_hn = vzero ? 0.0 : 1.0 / hn_t;
            part = 0.0;
            for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x) {
                double ut = u[t];
                if (sub) {
#pragma unroll 4
                    for (int k = 1; k <= j; ++k) ut -= ccol[k] * Vb[(int64_t)(k - 1) * n + t];
                }
                const double vn = vzero ? 0.0 : ut * inv_hn;
                Vn[t] = vn;
                if (use_dsm) {
                    if constexpr (kMixed) vsn32[t - ob] = (float)vn;
                    else vsn[t - ob] = vn;
                }
                if (!run_t) {
                    Wj[t] = 0.0;
                    AWj[t] = 0.0;
                } else {
                    double wv = Vj[t];
                    double aw = AWj[t];
#pragma unroll 4
                    for (int l = 1; l <= j - 1; ++l) {
                        wv -= Wb[(int64_t)(l - 1) * n + t] * rc_t[l];
                        aw -= AWb[(int64_t)(l - 1) * n + t] * rc_t[l];
                    }
                    wv *= inv_rjj;
                    aw *= inv_rjj;
                    Wj[t] = wv;
                    AWj[t] = aw;
                    const double xn = x[t] + f_t * wv;
                    x[t] = xn;
                    if (use_dsm) xsm[t - ob] = xn;
                    rv[t] -= f_t * aw;
                }
                part += rv[t] * rv[t];
            }
            cluster_sum<R>(part, slot, s, cl);  // also orders V_{j+1} and x for the next step
            if (threadIdx.x < R) {
                const int r = threadIdx.x;
                s.check[r] = 0;
                if (s.run[r]) {
                    s.inner[r]++;
                    const double normr = sqrt(s.val[r]);
                    const double tolb = d.tol * s.n2b[r];
                    if (normr <= tolb) {
                        s.check[r] = 1;            // verify with the true residual
                    } else if (s.stag[r]) {
                        s.run[r] = 0;
                        s.flag[r] = 3;
                    } else if (kMixed && fabs(s.phibar[r]) <= 1.0e-5 * s.h1[r]) {
                        s.run[r] = 0;              // FP32 Krylov space exhausted: refine
                    }
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                int a = 0;
                for (int r = 0; r < R; ++r) a |= s.check[r];
                s.any = a;
            }
            __syncthreads();
            if (s.any) {
                // the reference's stopping test is on b - A x (DBEM1/pre_gmres.cpp:1566-1578)
                cl.sync();
                if (use_dsm)
                    spmm_owned_dsm<R, false>(d, xsm, lo, hi, u, nullptr, cl);
                else
                    spmm_owned<R, false>(d, x, lo, hi, u);
                part = 0.0;
                for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x) {
                    const double tr = b[t] - u[t];
                    if (s.check[t % R]) rv[t] = tr;
                    part += tr * tr;
                }
                cluster_sum<R>(part, slot, s, cl);
                if (threadIdx.x < R) {
                    const int r = threadIdx.x;
                    if (s.check[r] && sqrt(s.val[r]) <= d.tol * s.n2b[r]) {
                        s.run[r] = 0;
                        s.flag[r] = 0;
                    } else if (s.check[r] && kMixed) {
                        s.run[r] = 0;              // refine from the FP64 residual
                    }
                }
                __syncthreads();
            }
        }
        if constexpr (kMixed) {
            // explicit FP64 residual of the refined x
            cl.sync();
            if (use_dsm)
                spmm_owned_dsm<R, false>(d, xsm, lo, hi, rv, nullptr, cl);
            else
                spmm_owned<R, false>(d, x, lo, hi, rv);
            part = 0.0;
            for (int64_t t = ob + threadIdx.x; t < oe; t += blockDim.x) {
                rv[t] = b[t] - rv[t];
                part += rv[t] * rv[t];
            }
            cluster_sum<R>(part, slot, s, cl);
            if (threadIdx.x < R) {
                const int r = threadIdx.x;
                if (s.flag[r] == 1 && sqrt(s.val[r]) <= d.tol * s.n2b[r]) s.flag[r] = 0;
            }
            __syncthreads();
        }
    }
    if (threadIdx.x < R && cq == 0) {
        const int r = threadIdx.x;
        int* fl = d.step_flags + ((int64_t)(step - 1) * RT + roff + r) * 3;
        fl[0] = s.flag[r];
        fl[1] = s.cycles[r];
        fl[2] = s.inner[r];
        if (s.flag[r] != 0) atomicExch(d.status, 1);
    }
    if (threadIdx.x == 0) {
        int a = 0;
        for (int r = 0; r < R; ++r) a |= s.flag[r] != 0;
        s.any = a;
    }
    cl.sync();  // x complete; the failure decision is uniform
    if (s.any || d.solve_only) {
        cl.sync();
        return;
    }

    // ---- write-back (ScatterUnknownToBoundary + AllLocToAbs +
    //      BuildPhysicalStateFromBoundary) ----
    const int nh = d.nh;
    const int xs = step % 3;
    const int64_t gtid = (int64_t)cq * blockDim.x + threadIdx.x, gstride = (int64_t)C * blockDim.x;
    for (int64_t t = gtid; t < (int64_t)E * R; t += gstride) {
        const int64_t i = t / R;
        const int r = (int)(t % R), rg = roff + r;
        const double* T = d.itf_trans + 9 * i;
        const double* in = d.known_lu + (((int64_t)rg * (d.nstep + 1) + step) * E + i) * 3;
        double lu[3], lt[3];
        if (d.uref_known[i]) {
            for (int c = 0; c < 3; ++c) lu[c] = d.uref_sign[i] * in[c];
        } else {
            const int64_t pb = d.perm_of_unk[d.uref_block[i]];
            const double v0 = ldcg(x + (3 * pb) * R + r), v1 = ldcg(x + (3 * pb + 1) * R + r),
                         v2 = ldcg(x + (3 * pb + 2) * R + r);
            for (int c = 0; c < 3; ++c) lu[c] = d.uref_sign[i] * (T[3 * c] * v0 + T[3 * c + 1] * v1 + T[3 * c + 2] * v2);
        }
        if (d.tref_known[i]) {
            for (int c = 0; c < 3; ++c) lt[c] = d.tref_sign[i] * in[c];
        } else {
            const int64_t pb = d.perm_of_unk[d.tref_block[i]];
            const double v0 = ldcg(x + (3 * pb) * R + r), v1 = ldcg(x + (3 * pb + 1) * R + r),
                         v2 = ldcg(x + (3 * pb + 2) * R + r);
            for (int c = 0; c < 3; ++c) lt[c] = d.tref_sign[i] * (T[3 * c] * v0 + T[3 * c + 1] * v1 + T[3 * c + 2] * v2);
        }
        const double* F = d.trans + 9 * i;
        double gu[3], gt[3];
        for (int c = 0; c < 3; ++c) {
            gu[c] = F[c] * lu[0] + F[3 + c] * lu[1] + F[6 + c] * lu[2];
            gt[c] = F[c] * lt[0] + F[3 + c] * lt[1] + F[6 + c] * lt[2];
        }
        double* ou = d.out_lu + (((int64_t)rg * (d.nstep + 1) + step) * E + i) * 3;
        double* ot = d.out_lt + (((int64_t)rg * (d.nstep + 1) + step) * E + i) * 3;
        for (int c = 0; c < 3; ++c) {
            ou[c] = gu[c];
            ot[c] = gt[c];
        }
        if (d.hist_owner[i]) {
            const int64_t hb = d.hist_block[i];
            double* XU = d.xring + (((int64_t)xs * 2 + 0) * nh + hb) * 3 * RT + rg;
            double* XT = d.xring + (((int64_t)xs * 2 + 1) * nh + hb) * 3 * RT + rg;
            for (int c = 0; c < 3; ++c) {
                XU[c * RT] = d.hu_sign[i] * gu[c];
                XT[c * RT] = d.ht_sign[i] * gt[c];
            }
        }
    }
    if (d.rec_x && grp == 0)
        for (int64_t uu = gtid; uu < E; uu += gstride) {
            const int64_t pb = d.perm_of_unk[uu];
            for (int c = 0; c < 3; ++c) d.rec_x[(int64_t)(step - 1) * 3 * E + 3 * uu + c] = ldcg(x + (3 * pb + c) * R);
        }
    cl.sync();  // X_s complete
    // W_{s-1} = (X_s + 2 X_{s-1}) + X_{s-2};  W_s = 2 X_s + X_{s-1}
    // (BuildConvolutionVector's coefficients 1, 2, 1 and summation order;
    //  X_0 and unsolved states are zero, DBEM1/multidomain.cpp:3201-3225)
    const int SW = d.SW;
    const int x1 = (step + 2) % 3, x2 = (step + 1) % 3;
    const int wa = (step - 1) % SW, wb = step % SW;
    const int64_t per_type = (int64_t)nh * 3 * RT;
    for (int64_t tt = gtid; tt < 2LL * nh * 3 * R; tt += gstride) {
        // this group's cases only: (type, history column, component, case)
        const int64_t type = tt / ((int64_t)nh * 3 * R);
        const int64_t nc = (tt / R) % ((int64_t)nh * 3);
        const int64_t rest = nc * RT + roff + (tt % R);
        const double Xs = ldcg(d.xring + ((int64_t)xs * 2 + type) * per_type + rest);
        const double Xm1 = ldcg(d.xring + ((int64_t)x1 * 2 + type) * per_type + rest);
        const double Xm2 = ldcg(d.xring + ((int64_t)x2 * 2 + type) * per_type + rest);
        const double wcomplete = (Xs + 2.0 * Xm1) + Xm2;
        const double wpartial = 2.0 * Xs + Xm1;
        d.wring[((int64_t)wa * 2 + type) * per_type + rest] = wcomplete;
        d.wring[((int64_t)wb * 2 + type) * per_type + rest] = wpartial;
    }
    // interface audit (PrintInterfaceError, DBEM1/multidomain.cpp:3227-3257)
    for (int64_t t = gtid; t < (int64_t)d.n_itf * R; t += gstride) {
        const int64_t pi = t / R;
        const int r = roff + (int)(t % R);
        const int a = d.itf_pairs[2 * pi], bb = d.itf_pairs[2 * pi + 1];
        const int64_t base = ((int64_t)r * (d.nstep + 1) + step) * E;
        const double* ua = d.out_lu + (base + a) * 3;
        const double* ub = d.out_lu + (base + bb) * 3;
        const double* ta = d.out_lt + (base + a) * 3;
        const double* tb = d.out_lt + (base + bb) * 3;
        double jump = 0.0, bal = 0.0;
        for (int c = 0; c < 3; ++c) {
            jump = fmax(jump, fabs(ua[c] - ub[c]));
            bal = fmax(bal, fabs(tb[c] - d.itf_sign[pi] * ta[c]));
        }
        atomic_max_nonneg(d.audit + 2 * (step - 1), jump);
        atomic_max_nonneg(d.audit + 2 * (step - 1) + 1, bal);
    }
    cl.sync();  // no CTA leaves while a peer may still read its shared memory
}

template <int R, bool kMixed>
__global__ void __launch_bounds__(kGmresThreads, 1) gmres_cluster_kernel(MarchData d, int step)
{
    gmres_body<R, kMixed>(d, step, (int)(blockIdx.x / cg::this_cluster().num_blocks()));
}

// Several models' GMRES of one step in one launch: cluster m solves model m
// (one group of R load cases each; every model laid out for the launch's
// cluster size); models whose march is shorter skip.
template <int R, bool kMixed>
__global__ void __launch_bounds__(kGmresThreads, 1) gmres_models_kernel(const MarchData* ds, int step)
{
    __shared__ MarchData sd;
    load_model(ds, (int)(blockIdx.x / cg::this_cluster().num_blocks()), sd);
    if (step > sd.nstep) return;
    gmres_body<R, kMixed>(sd, step, 0);
}

// ---------------------------------------------------------------------------
namespace {

template <int R, bool kMixed>
cudaError_t launch_gmres(const MarchData& d, int step, cudaStream_t s)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(d.cluster * d.groups);
    cfg.blockDim = dim3(kGmresThreads);
    cfg.dynamicSmemBytes = gmres_dsm_bytes(d.dsm_rows, R, kMixed);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = d.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // the function attributes are set once per device, to the most the device
    // allows: changing them between launches (models of different sizes
    // marched side by side) would be a host-side attribute change per launch
    static std::atomic<int> dyn_max[kMaxDevices];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    int cap = dyn_max[dev].load();
    if (cap == 0) {
        cudaFuncAttributes fa{};
        int optin = 0;
        if ((e = cudaFuncGetAttributes(&fa, gmres_cluster_kernel<R, kMixed>)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
        cap = optin - (int)fa.sharedSizeBytes;
        if ((e = cudaFuncSetAttribute(gmres_cluster_kernel<R, kMixed>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      cap)) != cudaSuccess)
            return e;
        if ((e = cudaFuncSetAttribute(gmres_cluster_kernel<R, kMixed>,
                                      cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess)
            return e;
        dyn_max[dev].store(cap);
    }
    if (cfg.dynamicSmemBytes > (size_t)cap) return cudaErrorInvalidValue;
    return cudaLaunchKernelEx(&cfg, gmres_cluster_kernel<R, kMixed>, d, step);
}

template <int R, bool kMixed>
int cluster_size_for(int device)
{
    (void)device;
    for (int c : {16, 8, 4, 2, 1}) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(c);
        cfg.blockDim = dim3(kGmresThreads);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = c;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        if (c > 8 && cudaFuncSetAttribute(gmres_cluster_kernel<R, kMixed>,
                                          cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            cudaGetLastError();
            continue;
        }
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, gmres_cluster_kernel<R, kMixed>, &cfg) == cudaSuccess && n >= 1)
            return c;
        cudaGetLastError();
    }
    return 1;
}

template <int R, bool kMixed, int kCpt>
cudaError_t launch_rhs_cpt(const MarchData& d, int step, bool bulk, int add_bulk, cudaStream_t s)
{
    const size_t smem = sizeof(int) * (size_t)(d.K + 1);
    if (bulk)
        rhs_kernel<R, kMixed, true, kCpt><<<d.E, kRhsThreads, smem, s>>>(d, step, 0);
    else
        rhs_kernel<R, kMixed, false, kCpt><<<d.E, kRhsThreads, smem, s>>>(d, step, add_bulk);
    return cudaGetLastError();
}

// d.rhs_cpt selects the load cases per thread (the R-tile; with it the blocks
// a warp takes per iteration, 32 / (R / cpt)): 4 or 2 for R >= 4, 2 or 1 for
// R = 2; 0 is the default, min(R, 4)
template <int R, bool kMixed>
cudaError_t launch_rhs(const MarchData& d, int step, bool bulk, int add_bulk, cudaStream_t s)
{
    if constexpr (R >= 4) {
        if (d.rhs_cpt == 2) return launch_rhs_cpt<R, kMixed, 2>(d, step, bulk, add_bulk, s);
        return launch_rhs_cpt<R, kMixed, 4>(d, step, bulk, add_bulk, s);
    } else if constexpr (R == 2) {
        if (d.rhs_cpt == 1) return launch_rhs_cpt<R, kMixed, 1>(d, step, bulk, add_bulk, s);
        return launch_rhs_cpt<R, kMixed, 2>(d, step, bulk, add_bulk, s);
    } else {
        return launch_rhs_cpt<R, kMixed, 1>(d, step, bulk, add_bulk, s);
    }
}

// T-step history pass (T = (kr - 1) / 2, 2 or 3): two load cases per thread
// (the registers hold the T steps' sums and the window of T history
// vectors), one for R = 1.  Measured against the two-step form on the 32-load
// bar and kept out: staging the history vectors and block values through
// shared memory with cp.async (72% more instructions, 1.5x slower) and L1
// prefetches of the coming vectors (slower at every distance tried).
template <int R, bool kMixed>
cudaError_t launch_bulk_steps(const MarchData& d, int t0, cudaStream_t s)
{
    constexpr int kC = R >= 2 ? 2 : 1;
    if (d.kr >= 7) bulk_steps_kernel<R, kMixed, kC, 3><<<d.E, kRhsThreads, 0, s>>>(d, t0);
    else bulk_steps_kernel<R, kMixed, kC, 2><<<d.E, kRhsThreads, 0, s>>>(d, t0);
    return cudaGetLastError();
}

template <int R>
cudaError_t step_r(const MarchData& d0, int step, cudaStream_t s, cudaStream_t side, const StepEvents& ev, bool overlap)
{
    MarchData d = d0;
    const int kcap = step > 1 ? (step < d.K ? step : d.K) : 0;
    // T-step history passes: launched at steps 2, 2 + T, 2 + 2T, ..., the one
    // launched at step e covers steps e + T .. e + 2T - 1
    const int T = d.kr >= 5 ? (d.kr - 1) / 2 : 0;
    const bool pair = overlap && T >= 2;
    const bool launches = pair && step >= 2 && (step - 2) % T == 0;
    cudaError_t e;
    // the first step a pass covers waits for it
    if (pair && step >= 2 + T && (step - 2) % T == 0 && ev.prev_pass) cudaStreamWaitEvent(s, ev.prev_pass, 0);
    cudaEventRecord(ev.head0, s);
    if (!overlap) {
        d.k_lo = 1;
        d.k_hi = kcap;
        e = d.mixed ? launch_rhs<R, true>(d, step, false, 0, s) : launch_rhs<R, false>(d, step, false, 0, s);
    } else if (pair) {
        // head: k < kr, plus the part k >= kr and KnownM computed beside the
        // GMRES launches before this step (every step from 2 + T on)
        d.k_lo = 1;
        d.k_hi = kcap < d.kr - 1 ? kcap : d.kr - 1;
        const int add = step >= 2 + T ? 1 : 0;
        e = d.mixed ? launch_rhs<R, true>(d, step, false, add, s) : launch_rhs<R, false>(d, step, false, add, s);
    } else {
        // head: k in {1, 2}, plus the bulk (k >= 3 and KnownM) computed during
        // the previous step (every step from 3 on)
        d.k_lo = 1;
        d.k_hi = kcap < 2 ? kcap : 2;
        const int add = kcap >= 3 ? 1 : 0;
        e = d.mixed ? launch_rhs<R, true>(d, step, false, add, s) : launch_rhs<R, false>(d, step, false, add, s);
    }
    if (e != cudaSuccess) return e;
    cudaEventRecord(ev.head1, s);
    cudaEventRecord(ev.gm0, s);
    switch (d.R / d.groups) {
    case 1: e = d.mixed ? launch_gmres<1, true>(d, step, s) : launch_gmres<1, false>(d, step, s); break;
    case 2: e = d.mixed ? launch_gmres<2, true>(d, step, s) : launch_gmres<2, false>(d, step, s); break;
    case 4: e = d.mixed ? launch_gmres<4, true>(d, step, s) : launch_gmres<4, false>(d, step, s); break;
    case 8: e = d.mixed ? launch_gmres<8, true>(d, step, s) : launch_gmres<8, false>(d, step, s); break;
    case 16: e = d.mixed ? launch_gmres<16, true>(d, step, s) : launch_gmres<16, false>(d, step, s); break;
    case 32: e = d.mixed ? launch_gmres<32, true>(d, step, s) : launch_gmres<32, false>(d, step, s); break;
    default: e = cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    cudaEventRecord(ev.gm1, s);
    if (pair) {
        // part k >= kr of steps step+T .. step+2T-1 needs the states up to
        // step-1 only: it runs beside the GMRES of this step and the T - 1
        // after it
        if (ev.prev_gm) cudaStreamWaitEvent(side, ev.prev_gm, 0);
        cudaEventRecord(ev.bulk0, side);
        const int t0 = step + T;
        if (launches && t0 <= d.nstep) {
            e = d.mixed ? launch_bulk_steps<R, true>(d0, t0, side) : launch_bulk_steps<R, false>(d0, t0, side);
            if (e != cudaSuccess) return e;
        }
        cudaEventRecord(ev.bulk1, side);
        cudaEventRecord(ev.sync, side);
    } else if (overlap && step + 1 <= d.nstep) {
        // bulk of step+1 (k >= 3) needs the states up to step-1 only: run it on
        // the side stream while this step's GMRES runs; the next head waits.
        const int kc1 = step + 1 < d.K ? step + 1 : d.K;
        if (ev.prev_gm) cudaStreamWaitEvent(side, ev.prev_gm, 0);
        cudaEventRecord(ev.bulk0, side);
        if (kc1 >= 3) {
            MarchData db = d0;
            db.k_lo = 3;
            db.k_hi = kc1;
            e = d.mixed ? launch_rhs<R, true>(db, step + 1, true, 0, side)
                        : launch_rhs<R, false>(db, step + 1, true, 0, side);
            if (e != cudaSuccess) return e;
        }
        cudaEventRecord(ev.bulk1, side);
        cudaEventRecord(ev.sync, side);
        cudaStreamWaitEvent(s, ev.sync, 0);
    }
    return cudaSuccess;
}

}  // namespace

bool march_supported_loads(int R) { return R == 1 || R == 2 || R == 4 || R == 8 || R == 16 || R == 32; }

cudaError_t march_prepare(const MarchData& d, cudaStream_t s)
{
    prepare_kernel<<<296, 256, 0, s>>>(d);
    return cudaGetLastError();
}

cudaError_t march_step(const MarchData& d, int step, cudaStream_t s, cudaStream_t side, const StepEvents& ev,
                       bool overlap)
{
    switch (d.R) {
    case 1: return step_r<1>(d, step, s, side, ev, overlap);
    case 2: return step_r<2>(d, step, s, side, ev, overlap);
    case 4: return step_r<4>(d, step, s, side, ev, overlap);
    case 8: return step_r<8>(d, step, s, side, ev, overlap);
    case 16: return step_r<16>(d, step, s, side, ev, overlap);
    case 32: return step_r<32>(d, step, s, side, ev, overlap);
    }
    return cudaErrorInvalidValue;
}

cudaError_t gmres_solve_single(const MarchData& d, cudaStream_t s) { return launch_gmres<1, false>(d, 1, s); }

size_t gmres_dsm_bytes(int rows, int Rg, bool mixed)
{
    // FP64: four FP64 vectors; mixed: one FP64 vector and three FP32 ones
    const size_t per = mixed ? sizeof(double) + 3 * sizeof(float) : 4 * sizeof(double);
    return rows > 0 ? per * 3 * (size_t)rows * Rg : 0;
}

namespace {

// One step of several models (one launch per phase): the right-hand sides of
// every model, then one GMRES cluster of C CTAs per model.
template <int R, bool kMixed>
cudaError_t models_step_r(const MarchData* ds, const int* row_off, int n_models, int total_rows, int cluster,
                          size_t gmres_dsm, int max_K, int step, int phase, cudaStream_t s)
{
    constexpr int kC = R >= 4 ? 4 : R;
    const size_t smem = sizeof(int) * (size_t)(max_K + 1);
    if (phase == 2) {
        rhs_models_kernel<R, kMixed, true, kC><<<total_rows, kRhsThreads, smem, s>>>(ds, row_off, n_models, step, 1);
        return cudaGetLastError();
    }
    rhs_models_kernel<R, kMixed, false, kC><<<total_rows, kRhsThreads, smem, s>>>(ds, row_off, n_models, step, phase);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    static std::atomic<int> dyn_max[kMaxDevices];
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    int cap = dyn_max[dev].load();
    if (cap == 0) {
        cudaFuncAttributes fa{};
        int optin = 0;
        if ((e = cudaFuncGetAttributes(&fa, gmres_models_kernel<R, kMixed>)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
        cap = optin - (int)fa.sharedSizeBytes;
        if ((e = cudaFuncSetAttribute(gmres_models_kernel<R, kMixed>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      cap)) != cudaSuccess)
            return e;
        if ((e = cudaFuncSetAttribute(gmres_models_kernel<R, kMixed>,
                                      cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess)
            return e;
        dyn_max[dev].store(cap);
    }
    if (gmres_dsm > (size_t)cap) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster * n_models);
    cfg.blockDim = dim3(kGmresThreads);
    cfg.dynamicSmemBytes = gmres_dsm;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, gmres_models_kernel<R, kMixed>, ds, step);
}

}  // namespace

cudaError_t march_models_step(const MarchData* ds, const int* row_off, int n_models, int total_rows, int R,
                              bool mixed, int cluster, size_t gmres_dsm, int max_K, int step, int phase, cudaStream_t s)
{
#define TDBEM_MODELS_CASE(RR)                                                                                      \
    case RR:                                                                                                       \
        return mixed ? models_step_r<RR, true>(ds, row_off, n_models, total_rows, cluster, gmres_dsm, max_K, step, \
                                               phase, s)                                                           \
                     : models_step_r<RR, false>(ds, row_off, n_models, total_rows, cluster, gmres_dsm, max_K, step, \
                                                phase, s);
    switch (R) {
        TDBEM_MODELS_CASE(1)
        TDBEM_MODELS_CASE(2)
        TDBEM_MODELS_CASE(4)
        TDBEM_MODELS_CASE(8)
    }
#undef TDBEM_MODELS_CASE
    return cudaErrorInvalidValue;
}

int gmres_cluster_size(int device, int R, bool mixed)
{
    switch (R) {
    case 1: return mixed ? cluster_size_for<1, true>(device) : cluster_size_for<1, false>(device);
    case 2: return mixed ? cluster_size_for<2, true>(device) : cluster_size_for<2, false>(device);
    case 4: return mixed ? cluster_size_for<4, true>(device) : cluster_size_for<4, false>(device);
    case 8: return mixed ? cluster_size_for<8, true>(device) : cluster_size_for<8, false>(device);
    case 16: return mixed ? cluster_size_for<16, true>(device) : cluster_size_for<16, false>(device);
    case 32: return mixed ? cluster_size_for<32, true>(device) : cluster_size_for<32, false>(device);
    }
    return 1;
}

}  // namespace tdbem
