// Per-step kernels of the multi-domain TDBEM time march on B200.
//
//   rhs_kernel    the history-convolution right-hand side (one CTA per
//                 equation row, HBM-bound block SpMV over the stacked
//                 history matrix), DBEM1/multidomain.cpp:3843-3866
//   gmres_kernel  left-preconditioned GMRES(restart) with the reference's
//                 true-residual stop, one persistent cooperative grid with a
//                 bounded software grid barrier, DBEM1/pre_gmres.cpp:1369-1605,
//                 followed by the boundary write-back and the history-state
//                 update, DBEM1/multidomain.cpp:3086-3225
#include "march.cuh"
#include "tdbem_common.cuh"

#include <cooperative_groups.h>

namespace tdbem {

namespace {

constexpr int kRhsThreads = 256;
constexpr int kGmresThreads = 512;
constexpr long long kBarrierTimeoutCycles = 4000000000LL;  // about 2 s at 2 GHz

__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the CTA, result broadcast to every thread.  red: >= 33 doubles.
__device__ double block_sum(double v, double* red)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        double t = lane < nw ? red[lane] : 0.0;
        t = warp_sum(t);
        if (lane == 0) red[32] = t;
    }
    __syncthreads();
    return red[32];
}

// Software grid barrier with a bounded wait.  Returns false (and sets
// status[1]) when the wait exceeds its bound; callers then leave the kernel.
// All CTAs of the cooperative launch are co-resident, so every wait ends
// unless a CTA has already left after a timeout.
__device__ bool grid_barrier(unsigned* bar, int* status, int* sflag)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned* vgen = bar + 1;
        const unsigned gen = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(bar, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const long long t0 = clock64();
            while (*vgen == gen) {
                if (clock64() - t0 > kBarrierTimeoutCycles || *(volatile int*)(status + 1)) {
                    atomicExch(status + 1, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        *sflag = ok;
    }
    __syncthreads();
    return *sflag != 0;
}

// Deterministic grid-wide sum: every CTA adds the per-CTA partials in the
// same fixed order, so all CTAs hold the identical value.
__device__ bool grid_sum(double v, int slot, const MarchData& d, double* red, int* sflag, double* out)
{
    double s = block_sum(v, red);
    if (threadIdx.x == 0) d.partials[slot * gridDim.x + blockIdx.x] = s;
    if (!grid_barrier(d.bar, d.status, sflag)) return false;
    if (threadIdx.x < 32) {
        double t = 0.0;
        for (int c = threadIdx.x; c < (int)gridDim.x; c += 32) t += ldcg(d.partials + slot * gridDim.x + c);
        t = warp_sum(t);
        if (threadIdx.x == 0) red[32] = t;
    }
    __syncthreads();
    *out = red[32];
    __syncthreads();
    return true;
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
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n0; t += gridDim.x * (long long)blockDim.x) {
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
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nx; t += gridDim.x * (long long)blockDim.x)
        d.xring[t] = 0.0;
    const long long nw = (long long)d.SW * 2 * d.nh * 3 * d.R;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nw; t += gridDim.x * (long long)blockDim.x) {
        d.wring[t] = 0.0;
        if (d.wring32) d.wring32[t] = 0.0f;
    }
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 2LL * d.nstep; t += gridDim.x * (long long)blockDim.x)
        d.audit[t] = 0.0;
    if (blockIdx.x == 0 && threadIdx.x < 4) d.status[threadIdx.x] = 0;
    if (blockIdx.x == 0 && threadIdx.x < 2) d.bar[threadIdx.x] = 0;
}

// ---------------------------------------------------------------------------
// rhs_p = KnownM.known_s + sum_{k<=min(s,K)} MGS_k.wT(s-k) - MTS_k.wU(s-k)
// for perm row p (the MTS blocks are stored negated).  One CTA per row.
template <bool kMixed>
__global__ void __launch_bounds__(kRhsThreads) rhs_kernel(MarchData d, int step)
{
    if (*(volatile int*)d.status) return;
    extern __shared__ int slot_of_k[];
    __shared__ double red[3][kRhsThreads / 32];
    const int p = blockIdx.x;
    const int row = d.row_of[p];
    const int K = d.K, SW = d.SW;
    for (int k = threadIdx.x; k <= K; k += blockDim.x) slot_of_k[k] = (((step - k) % SW) + SW) % SW;
    __syncthreads();
    const int kcap = step > 1 ? min(step, K) : 0;
    const int64_t beg = d.h_kptr[(int64_t)row * (K + 1)];
    const int64_t end = d.h_kptr[(int64_t)row * (K + 1) + kcap];
    const int64_t nnz = d.h_nnz;
    const int nh = d.nh;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int64_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
        const uint32_t cp = __ldg(d.h_col + i);
        const int k = (int)(cp >> 21), type = (int)((cp >> 20) & 1u), col = (int)(cp & 0xFFFFFu);
        const int64_t wi = (((int64_t)slot_of_k[k] * 2 + type) * nh + col) * 3;
        if (kMixed) {
            const float* v = d.h_val32 + i;
            const float w0 = d.wring32[wi], w1 = d.wring32[wi + 1], w2 = d.wring32[wi + 2];
            // FP32 3x3 block product, FP64 accumulation across blocks
            const float r0 = __ldg(v) * w0 + __ldg(v + nnz) * w1 + __ldg(v + 2 * nnz) * w2;
            const float r1 = __ldg(v + 3 * nnz) * w0 + __ldg(v + 4 * nnz) * w1 + __ldg(v + 5 * nnz) * w2;
            const float r2 = __ldg(v + 6 * nnz) * w0 + __ldg(v + 7 * nnz) * w1 + __ldg(v + 8 * nnz) * w2;
            a0 += (double)r0;
            a1 += (double)r1;
            a2 += (double)r2;
        } else {
            const double* v = d.h_val + i;
            const double w0 = d.wring[wi], w1 = d.wring[wi + 1], w2 = d.wring[wi + 2];
            a0 += __ldg(v) * w0 + __ldg(v + nnz) * w1 + __ldg(v + 2 * nnz) * w2;
            a1 += __ldg(v + 3 * nnz) * w0 + __ldg(v + 4 * nnz) * w1 + __ldg(v + 5 * nnz) * w2;
            a2 += __ldg(v + 6 * nnz) * w0 + __ldg(v + 7 * nnz) * w1 + __ldg(v + 8 * nnz) * w2;
        }
    }
    const int E = d.E;
    for (int j = d.k_rp[row] + threadIdx.x; j < d.k_rp[row + 1]; j += blockDim.x) {
        const int kb = d.k_col[j];
        const int e = d.known_elem[kb];
        const double sg = d.known_sign[kb];
        const double* kv = d.known_lu + ((int64_t)step * E + e) * 3;
        const double k0 = sg * kv[0], k1 = sg * kv[1], k2 = sg * kv[2];
        const double* v = d.k_val + 9 * (int64_t)j;
        a0 += v[0] * k0 + v[1] * k1 + v[2] * k2;
        a1 += v[3] * k0 + v[4] * k1 + v[5] * k2;
        a2 += v[6] * k0 + v[7] * k1 + v[8] * k2;
    }
    a0 = warp_sum(a0);
    a1 = warp_sum(a1);
    a2 = warp_sum(a2);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][w] = a0;
        red[1][w] = a1;
        red[2][w] = a2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int q = 0; q < kRhsThreads / 32; ++q) s += red[threadIdx.x][q];
        d.b[3 * p + threadIdx.x] = s;
        if (d.rec_rhs) d.rec_rhs[(int64_t)(step - 1) * 3 * E + 3 * row + threadIdx.x] = s;
    }
}

// ---------------------------------------------------------------------------
namespace {

// y[0..3*nown) = (A' v)[lo..hi) into shared memory; v read through L2.
template <bool kF32>
__device__ void spmv_owned(const MarchData& d, const double* v, int lo, int hi, double* y)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int p = lo + w; p < hi; p += nw) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int j = d.a_rp[p] + lane; j < d.a_rp[p + 1]; j += 32) {
            const int c = d.a_col[j];
            const double x0 = ldcg(v + 3 * c), x1 = ldcg(v + 3 * c + 1), x2 = ldcg(v + 3 * c + 2);
            if (kF32) {
                const float* a = d.a_val32 + 9 * (int64_t)j;
                const float f0 = (float)x0, f1 = (float)x1, f2 = (float)x2;
                s0 += (double)(a[0] * f0 + a[1] * f1 + a[2] * f2);
                s1 += (double)(a[3] * f0 + a[4] * f1 + a[5] * f2);
                s2 += (double)(a[6] * f0 + a[7] * f1 + a[8] * f2);
            } else {
                const double* a = d.a_val + 9 * (int64_t)j;
                s0 += a[0] * x0 + a[1] * x1 + a[2] * x2;
                s1 += a[3] * x0 + a[4] * x1 + a[5] * x2;
                s2 += a[6] * x0 + a[7] * x1 + a[8] * x2;
            }
        }
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        s2 = warp_sum(s2);
        if (lane == 0) {
            y[3 * (p - lo)] = s0;
            y[3 * (p - lo) + 1] = s1;
            y[3 * (p - lo) + 2] = s2;
        }
    }
    __syncthreads();
}

// out[owned] = M^-1 in[owned]: block-diagonal leaf inverses (GMRES_M_X,
// DBEM1/pre_gmres.cpp:837-895), summation order k then n as the reference.
template <bool kF32>
__device__ void precond_owned(const MarchData& d, int L0, int L1, int lo, const double* in, double* out)
{
    for (int L = L0; L < L1; ++L) {
        const int b = d.leaf_begin[L], c = d.leaf_count[L], n3 = 3 * c;
        for (int r = threadIdx.x; r < n3; r += blockDim.x) {
            double s = 0.0;
            if (kF32) {
                const float* m = d.pinv32 + d.leaf_off[L] + (int64_t)r * n3;
                for (int q = 0; q < n3; ++q) s += (double)(m[q] * (float)in[3 * (b - lo) + q]);
            } else {
                const double* m = d.pinv + d.leaf_off[L] + (int64_t)r * n3;
                for (int q = 0; q < n3; ++q) s += m[q] * in[3 * (b - lo) + q];
            }
            out[3 * (b - lo) + r] = s;
        }
    }
    __syncthreads();
}

}  // namespace

// Persistent GMRES for one step (load case 0 .. R-1 handled one after the
// other), then the boundary write-back and history update.
// kMixed: Arnoldi SpMV and preconditioner in FP32, orthogonalisation,
// Givens and the true residual b - A x in FP64, restarted (iterative
// refinement) until the FP64 residual meets the tolerance.
template <bool kMixed>
__global__ void __launch_bounds__(kGmresThreads, 1) gmres_kernel(MarchData d, int step)
{
    if (*(volatile int*)d.status) return;
    extern __shared__ double sm[];
    __shared__ double red[40];
    __shared__ int sflag;
    __shared__ double s_c, s_s, s_phibar, s_f, s_h1;
    __shared__ int s_stag;

    const int cta = blockIdx.x;
    const int E = d.E, n = 3 * E, rs = d.restart;
    const int L0 = d.cta_leaf[cta], L1 = d.cta_leaf[cta + 1];
    const int lo = L0 < L1 ? d.leaf_begin[L0] : 0;
    const int hi = L0 < L1 ? d.leaf_begin[L1 - 1] + d.leaf_count[L1 - 1] : 0;
    const int n3 = 3 * (hi - lo);
    double* su2 = sm;
    double* su = sm + 3 * d.max_owned;
    double* sb = su + 3 * d.max_owned;
    double* QT = d.cta_scratch + (int64_t)cta * d.scratch_stride;
    const int ldq = rs + 2;
    double* Rm = QT + (int64_t)ldq * ldq;
    const int ldr = rs + 1;
    double* h = Rm + (int64_t)ldr * ldr;
    double* f = h + ldq;
    double* q = f + ldq;
#define QTM(i, j) QT[(int64_t)(i) * ldq + (j)]
#define RM(i, j) Rm[(int64_t)(i) * ldr + (j)]
    int slot = 0;
    double val;

    for (int t = threadIdx.x; t < n3; t += blockDim.x) sb[t] = d.b[3 * lo + t];
    for (int t = threadIdx.x; t < n3; t += blockDim.x) d.x[3 * lo + t] = 0.0;
    __syncthreads();

    double part = 0.0;
    for (int t = threadIdx.x; t < n3; t += blockDim.x) part += sb[t] * sb[t];
    if (!grid_sum(part, slot, d, red, &sflag, &val)) return;
    slot ^= 1;
    const double n2b = sqrt(val);
    const double tolb = d.tol * n2b;
    int flag = 1, inner = 0, cycles = 0;
    if (n2b == 0.0 || n2b <= tolb) {
        flag = 0;
    } else {
        // residual of the current x (zero at entry) kept in su2 for the cycle
        for (int t = threadIdx.x; t < n3; t += blockDim.x) su2[t] = sb[t];
        __syncthreads();
        const int max_cycles = kMixed ? 8 : 1;
        double normr = n2b;
        while (flag != 0 && cycles < max_cycles) {
            ++cycles;
            // vh = M^-1 r, V_1 = vh / |vh|
            precond_owned<kMixed>(d, L0, L1, lo, su2, su);
            part = 0.0;
            for (int t = threadIdx.x; t < n3; t += blockDim.x) part += su[t] * su[t];
            if (!grid_sum(part, slot, d, red, &sflag, &val)) return;
            slot ^= 1;
            const double h1 = sqrt(val);
            // V_1; the cycle's starting x (x0) is kept in W's last column,
            // which the incremental update never uses (it stops at restart-1)
            double* X0 = d.W + (int64_t)(rs - 1) * n + 3 * lo;
            for (int t = threadIdx.x; t < n3; t += blockDim.x) {
                d.V[3 * lo + t] = su[t] / h1;
                X0[t] = d.x[3 * lo + t];
            }
            if (threadIdx.x == 0) {
                QTM(1, 1) = 1.0;
                s_phibar = h1;
                s_h1 = h1;
                s_stag = 0;
            }
            if (!grid_barrier(d.bar, d.status, &sflag)) return;
            int j;
            for (j = 1; j <= rs; ++j) {
                const double* Vj = d.V + (int64_t)(j - 1) * n;
                spmv_owned<kMixed>(d, Vj, lo, hi, su2);
                precond_owned<kMixed>(d, L0, L1, lo, su2, su);
                // modified Gram-Schmidt
                for (int k = 1; k <= j; ++k) {
                    const double* Vk = d.V + (int64_t)(k - 1) * n + 3 * lo;
                    part = 0.0;
                    for (int t = threadIdx.x; t < n3; t += blockDim.x) part += ldcg(Vk + t) * su[t];
                    if (!grid_sum(part, slot, d, red, &sflag, &val)) return;
                    slot ^= 1;
                    if (threadIdx.x == 0) h[k] = val;
                    for (int t = threadIdx.x; t < n3; t += blockDim.x) su[t] -= val * ldcg(Vk + t);
                    __syncthreads();
                }
                part = 0.0;
                for (int t = threadIdx.x; t < n3; t += blockDim.x) part += su[t] * su[t];
                if (!grid_sum(part, slot, d, red, &sflag, &val)) return;
                slot ^= 1;
                const double hn = sqrt(val);
                double* Vn = d.V + (int64_t)j * n + 3 * lo;
                for (int t = threadIdx.x; t < n3; t += blockDim.x) Vn[t] = hn <= 1.0e-12 ? 0.0 : su[t] / hn;
                if (threadIdx.x == 0) h[j + 1] = hn;
                // Givens (every CTA computes the same small update)
                // column j+1 above the rotation rows must read as zero
                for (int k = 1 + threadIdx.x; k <= j - 1; k += blockDim.x) QTM(k, j + 1) = 0.0;
                __syncthreads();
                for (int k = 1 + threadIdx.x; k <= j; k += blockDim.x) {
                    double s = 0.0;
                    for (int l = 1; l <= j; ++l) s += QTM(k, l) * h[l];
                    RM(k, j) = s;
                }
                __syncthreads();
                if (threadIdx.x == 0) {
                    const double rt = RM(j, j), hj1 = h[j + 1];
                    double c, s, temp;
                    if (hj1 == 0.0) {
                        c = 1.0;
                        s = 0.0;
                    } else if (hj1 * hj1 > rt * rt) {
                        temp = rt / hj1;
                        s = 1.0 / sqrt(1.0 + fabs(temp) * fabs(temp));
                        c = -temp * s;
                    } else {
                        temp = hj1 / rt;
                        c = 1.0 / sqrt(1.0 + fabs(temp) * fabs(temp));
                        s = -temp * c;
                    }
                    RM(j, j) = c * rt - s * hj1;
                    s_c = c;
                    s_s = s;
                    f[j] = c * s_phibar;
                    s_f = f[j];
                    s_phibar = s * s_phibar;
                }
                __syncthreads();
                for (int k = 1 + threadIdx.x; k <= j; k += blockDim.x) {
                    const double qk = QTM(j, k);
                    QTM(j, k) = s_c * qk;
                    QTM(j + 1, k) = s_s * qk;
                }
                __syncthreads();
                if (threadIdx.x == 0) {
                    QTM(j, j + 1) = -s_s;
                    QTM(j + 1, j + 1) = s_c;
                }
                const double Rjj = RM(j, j);
                if (j < rs) {
                    if (threadIdx.x == 0 && s_f == 0.0) s_stag = 1;
                    double* Wj = d.W + (int64_t)(j - 1) * n + 3 * lo;
                    for (int t = threadIdx.x; t < n3; t += blockDim.x) {
                        double wv = ldcg(Vj + 3 * lo + t) / Rjj;
                        for (int l = 1; l <= j - 1; ++l) wv -= ldcg(d.W + (int64_t)(l - 1) * n + 3 * lo + t) * RM(l, j) / Rjj;
                        Wj[t] = wv;
                        d.x[3 * lo + t] += s_f * wv;
                    }
                } else {
                    // restart exhausted: x = x0 + V R^-1 f (back substitution)
                    if (threadIdx.x == 0) {
                        for (int k = j; k >= 1; --k) {
                            double s = f[k];
                            for (int l = k + 1; l <= j; ++l) s -= RM(k, l) * q[l];
                            q[k] = s / RM(k, k);
                        }
                    }
                    __syncthreads();
                    for (int t = threadIdx.x; t < n3; t += blockDim.x) {
                        double acc = 0.0;
                        for (int l = 1; l <= j; ++l) acc += ldcg(d.V + (int64_t)(l - 1) * n + 3 * lo + t) * q[l];
                        d.x[3 * lo + t] = acc + X0[t];
                    }
                }
                if (!grid_barrier(d.bar, d.status, &sflag)) return;
                // true residual r = b - A x (FP64 always)
                spmv_owned<false>(d, d.x, lo, hi, su2);
                part = 0.0;
                for (int t = threadIdx.x; t < n3; t += blockDim.x) {
                    su2[t] = sb[t] - su2[t];
                    part += su2[t] * su2[t];
                }
                if (!grid_sum(part, slot, d, red, &sflag, &val)) return;
                slot ^= 1;
                normr = sqrt(val);
                ++inner;
                if (normr <= tolb) {
                    flag = 0;
                    break;
                }
                if (s_stag) {
                    flag = 3;
                    break;
                }
                // mixed precision: the FP32 Krylov space has reached its
                // accuracy; restart from the FP64 residual held in su2
                if (kMixed && fabs(s_phibar) <= 1.0e-5 * s_h1) break;
            }
            if (flag == 3) break;
        }
    }
    if (cta == 0 && threadIdx.x == 0) {
        int* fl = d.step_flags + (int64_t)(step - 1) * d.R * 3;
        fl[0] = flag;
        fl[1] = cycles;
        fl[2] = inner;
        if (flag != 0) atomicExch(d.status, 1);
    }
    if (flag != 0) return;

    // ---- write-back (ScatterUnknownToBoundary + AllLocToAbs +
    //      BuildPhysicalStateFromBoundary) ----
    const int nh = d.nh;
    const int xs = step % 3;
    const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, gstride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = gtid; i < E; i += gstride) {
        const double* T = d.itf_trans + 9 * i;
        const double* in = d.known_lu + ((int64_t)step * E + i) * 3;
        double lu[3], lt[3];
        if (d.uref_known[i]) {
            for (int c = 0; c < 3; ++c) lu[c] = d.uref_sign[i] * in[c];
        } else {
            const int64_t pb = d.perm_of_unk[d.uref_block[i]];
            const double v0 = ldcg(d.x + 3 * pb), v1 = ldcg(d.x + 3 * pb + 1), v2 = ldcg(d.x + 3 * pb + 2);
            for (int c = 0; c < 3; ++c) lu[c] = d.uref_sign[i] * (T[3 * c] * v0 + T[3 * c + 1] * v1 + T[3 * c + 2] * v2);
        }
        if (d.tref_known[i]) {
            for (int c = 0; c < 3; ++c) lt[c] = d.tref_sign[i] * in[c];
        } else {
            const int64_t pb = d.perm_of_unk[d.tref_block[i]];
            const double v0 = ldcg(d.x + 3 * pb), v1 = ldcg(d.x + 3 * pb + 1), v2 = ldcg(d.x + 3 * pb + 2);
            for (int c = 0; c < 3; ++c) lt[c] = d.tref_sign[i] * (T[3 * c] * v0 + T[3 * c + 1] * v1 + T[3 * c + 2] * v2);
        }
        const double* F = d.trans + 9 * i;
        double gu[3], gt[3];
        for (int c = 0; c < 3; ++c) {
            gu[c] = F[c] * lu[0] + F[3 + c] * lu[1] + F[6 + c] * lu[2];
            gt[c] = F[c] * lt[0] + F[3 + c] * lt[1] + F[6 + c] * lt[2];
        }
        double* ou = d.out_lu + ((int64_t)step * E + i) * 3;
        double* ot = d.out_lt + ((int64_t)step * E + i) * 3;
        for (int c = 0; c < 3; ++c) {
            ou[c] = gu[c];
            ot[c] = gt[c];
        }
        if (d.hist_owner[i]) {
            const int64_t hb = d.hist_block[i];
            double* XU = d.xring + (((int64_t)xs * 2 + 0) * nh + hb) * 3;
            double* XT = d.xring + (((int64_t)xs * 2 + 1) * nh + hb) * 3;
            for (int c = 0; c < 3; ++c) {
                XU[c] = d.hu_sign[i] * gu[c];
                XT[c] = d.ht_sign[i] * gt[c];
            }
        }
    }
    if (d.rec_x)
        for (int64_t u = gtid; u < E; u += gstride) {
            const int64_t pb = d.perm_of_unk[u];
            for (int c = 0; c < 3; ++c) d.rec_x[(int64_t)(step - 1) * n + 3 * u + c] = ldcg(d.x + 3 * pb + c);
        }
    if (!grid_barrier(d.bar, d.status, &sflag)) return;
    // W_{s-1} = (X_s + 2 X_{s-1}) + X_{s-2};  W_s = 2 X_s + X_{s-1}
    // (BuildConvolutionVector's coefficients 1, 2, 1 and summation order;
    //  X_0 and unsolved states are zero, DBEM1/multidomain.cpp:3201-3225)
    const int SW = d.SW;
    const int x1 = (step + 2) % 3, x2 = (step + 1) % 3;
    const int wa = (step - 1) % SW, wb = step % SW;
    for (int64_t t = gtid; t < (int64_t)2 * nh * 3; t += gstride) {
        const int64_t type = t / (nh * 3), rest = t % (nh * 3);
        const double Xs = ldcg(d.xring + ((int64_t)xs * 2 + type) * nh * 3 + rest);
        const double Xm1 = ldcg(d.xring + ((int64_t)x1 * 2 + type) * nh * 3 + rest);
        const double Xm2 = ldcg(d.xring + ((int64_t)x2 * 2 + type) * nh * 3 + rest);
        const double wcomplete = (Xs + 2.0 * Xm1) + Xm2;
        const double wpartial = 2.0 * Xs + Xm1;
        d.wring[((int64_t)wa * 2 + type) * nh * 3 + rest] = wcomplete;
        d.wring[((int64_t)wb * 2 + type) * nh * 3 + rest] = wpartial;
        if (d.wring32) {
            d.wring32[((int64_t)wa * 2 + type) * nh * 3 + rest] = (float)wcomplete;
            d.wring32[((int64_t)wb * 2 + type) * nh * 3 + rest] = (float)wpartial;
        }
    }
    // interface audit (PrintInterfaceError, DBEM1/multidomain.cpp:3227-3257)
    for (int64_t t = gtid; t < d.n_itf; t += gstride) {
        const int a = d.itf_pairs[2 * t], b = d.itf_pairs[2 * t + 1];
        const double* ua = d.out_lu + ((int64_t)step * E + a) * 3;
        const double* ub = d.out_lu + ((int64_t)step * E + b) * 3;
        const double* ta = d.out_lt + ((int64_t)step * E + a) * 3;
        const double* tb = d.out_lt + ((int64_t)step * E + b) * 3;
        double jump = 0.0, bal = 0.0;
        for (int c = 0; c < 3; ++c) {
            jump = fmax(jump, fabs(ua[c] - ub[c]));
            bal = fmax(bal, fabs(tb[c] - d.itf_sign[t] * ta[c]));
        }
        atomic_max_nonneg(d.audit + 2 * (step - 1), jump);
        atomic_max_nonneg(d.audit + 2 * (step - 1) + 1, bal);
    }
#undef QTM
#undef RM
}

cudaError_t march_prepare(const MarchData& d, cudaStream_t s)
{
    prepare_kernel<<<296, 256, 0, s>>>(d);
    return cudaGetLastError();
}

cudaError_t march_step(const MarchData& d, int step, cudaStream_t s, cudaEvent_t ev_mid)
{
    const size_t rhs_smem = sizeof(int) * (size_t)(d.K + 1);
    if (d.mixed)
        rhs_kernel<true><<<d.E, kRhsThreads, rhs_smem, s>>>(d, step);
    else
        rhs_kernel<false><<<d.E, kRhsThreads, rhs_smem, s>>>(d, step);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (ev_mid) cudaEventRecord(ev_mid, s);
    const size_t smem = sizeof(double) * (size_t)(9 * d.max_owned);
    MarchData dd = d;
    int st = step;
    void* args[] = {&dd, &st};
    const void* fn = d.mixed ? (const void*)gmres_kernel<true> : (const void*)gmres_kernel<false>;
    return cudaLaunchCooperativeKernel(fn, dim3(d.grid), dim3(kGmresThreads), args, smem, s);
}

int gmres_max_grid(int device, int threads)
{
    (void)threads;
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, gmres_kernel<false>, kGmresThreads, 0);
    return sms * (per > 0 ? 1 : 0);
}

}  // namespace tdbem
