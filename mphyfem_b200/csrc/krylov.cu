// krylov.cu -- K4/K5: SpMV over the SELL-32 3x3 layout, preconditioned CG, FP64 iterative
// refinement, vector kernels.
//
// Replaces KSPSolve with KSPCG (SolverPetsc.cpp:250-314; -ksp_type cg -pc_type jacobi for the
// plain method). The iteration follows PETSc's documented KSPCG (Hestenes-Stiefel,
// preconditioned-residual norm, KSPConvergedDefault): x0 = 0, converged when
// ||z_k|| <= max(rtol ||z_0||, abstol), diverged when ||z_k|| >= dtol ||z_0||, indefinite when
// p.Ap <= 0, its = iterations performed.
//
// One CG iteration is three kernels with Jacobi (SpMV + fused p.q; x/r/z update + fused (r,z),
// (z,z); p update) or five with the factorised preconditioner M = G^T G (the update splits into
// the x/r update and two SpMVs, the second fusing the reductions). Reductions are
// deterministic: every CTA writes a partial sum, and the CTA that finishes last (an atomic
// ticket, no waiting) adds the partials in a fixed order and advances the shared scalar state.
// Chunks of iterations are replayed from a captured CUDA graph; kernels return immediately once
// the state says done. FP32 vectors keep every reduction in FP64.
#include <algorithm>
#include <cmath>

#include <mutex>
#include <unordered_map>

#include "krylov.cuh"

namespace mphy {

constexpr int kThreads = 256;

unsigned stride_grid(int64_t n, int threads, int sm_count, int per_sm) {
    const int64_t want = (n + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count * per_sm;
    return (unsigned)(want < 1 ? 1 : (want > cap ? cap : want));
}

// Grid of a grid-stride kernel sized to what the SMs hold at once (the kernel's occupancy), so
// that no second partial wave of CTAs runs at low occupancy after the first: a kernel with 40
// registers per thread holds 6 CTAs of 256 per SM, and 8 CTAs per SM would leave a quarter of
// the grid for a tail.
namespace {
std::mutex g_occ_mu;
std::unordered_map<const void*, int> g_occ;
}  // namespace

unsigned resident_grid(const void* kernel, int64_t n, int threads, int sm_count) {
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lk(g_occ_mu);
        auto it = g_occ.find(kernel);
        if (it != g_occ.end()) {
            per_sm = it->second;
        } else {
            MPHY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0));
            if (per_sm < 1) per_sm = 1;
            g_occ.emplace(kernel, per_sm);
        }
    }
    return stride_grid(n, threads, sm_count, per_sm);
}

namespace {

template <typename T>
struct AccOf {
    using type = T;
};

// matrix value -> arithmetic (FP64 / FP32 values as they are, BF16 factor values widened)
__device__ __forceinline__ double mval(double x) { return x; }
__device__ __forceinline__ float mval(float x) { return x; }
__device__ __forceinline__ float mval(__nv_bfloat16 x) { return __bfloat162float(x); }

// Matrix values and column indices are read once per product: evict-first loads, so that the
// streamed matrix does not push the Krylov vectors (gathered and re-read through L2) out.
template <typename T>
__device__ __forceinline__ T ld_once(const T* p) {
    return __ldcs(p);
}

// two consecutive vector entries as one 8- or 16-byte access
template <typename T>
struct Pair;
template <>
struct Pair<double> {
    using type = double2;
};
template <>
struct Pair<float> {
    using type = float2;
};
// every pointer aligned for the paired access (16 bytes covers both types)
__device__ __forceinline__ bool aligned16(const void* a, const void* b, const void* c, const void* d) {
    return ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) | reinterpret_cast<uintptr_t>(c) |
             reinterpret_cast<uintptr_t>(d)) & 15) == 0;
}

// Deterministic block sum (fixed butterfly per warp, fixed order across warps); valid in all
// threads of warp 0.
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();  // sh may still be read from a previous call
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

// True in every thread of the CTA that arrives last. The partial sums must have been written
// (by thread 0) before the call.
__device__ __forceinline__ bool arrive_last(uint32_t* counter) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    return last;
}

// Fixed-order sum of partials[0..n) by one CTA (L1 bypassed: written by other CTAs).
__device__ __forceinline__ double reduce_partials(const double* partials, int n, double* sh) {
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += __ldcg(partials + i);
    return block_sum(v, sh);
}

// State after the initial residual (KSPConvergedDefault at n = 0).
__device__ void finish_init(PcgState* st, double rz, double zz, double rtol, double abstol, double dtol, int maxit,
                            int norm_type) {
    const double dp = sqrt(zz);
    st->norm_type = norm_type;
    st->rz = rz;
    st->dp = dp;
    st->dp0 = dp;
    st->ttol = fmax(rtol * dp, abstol);
    st->dtol = dtol;
    st->maxit = maxit;
    st->its = 0;
    st->status = MPHY_OK;
    st->done = 0;
    if (dp != dp) {
        st->status = MPHY_ERR_DIVERGED;
        st->done = 1;
    } else if (dp <= st->ttol) {
        st->done = 1;
    } else if (rz == 0.0) {
        st->its = 1;
        st->done = 1;
    } else if (maxit <= 0) {
        st->status = MPHY_ERR_NOT_CONVERGED;
        st->done = 1;
    }
}

// State after iteration its+1 (convergence, divergence, limit, next beta).
__device__ void finish_iter(PcgState* st, double rz, double zz) {
    st->its += 1;
    const double dp = sqrt(zz);
    st->dp = dp;
    if (dp != dp) {
        st->status = MPHY_ERR_DIVERGED;
        st->done = 1;
    } else if (dp <= st->ttol) {
        st->status = MPHY_OK;
        st->done = 1;
    } else if (dp >= st->dtol * st->dp0) {
        st->status = MPHY_ERR_DIVERGED;
        st->done = 1;
    } else if (st->its >= st->maxit) {
        st->status = MPHY_ERR_NOT_CONVERGED;
        st->done = 1;
    } else if (rz == 0.0) {
        // the next iteration would stop at once with beta == 0 (KSP_CONVERGED_ATOL)
        st->its += 1;
        st->status = MPHY_OK;
        st->done = 1;
    } else {
        st->beta = rz / st->rz;
        st->rz = rz;
    }
}

// ---------------------------------------------------------------- SpMV
// One thread per block row; a warp is one 32-row slice, so every value load is 32 consecutive
// entries. DOT: fuse p.q (x = p, y = q) and, in the last CTA, alpha = (r,z) / p.q.
template <typename VT, typename XT, bool DOT>
__global__ void __launch_bounds__(kThreads) spmv_kernel(SellView A, const VT* __restrict__ val,
                                                        const XT* __restrict__ x, XT* __restrict__ y,
                                                        double* __restrict__ partials, PcgState* st) {
    using Acc = typename AccOf<XT>::type;
    __shared__ double sh[32];
    if (st && st->done) return;  // inside a CG iteration: nothing left to do
    double acc = 0.0;
    const int64_t rows = (int64_t)A.n_slices * 32;
    for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < rows;
         row += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = row >> 5;
        const int lane = (int)(row & 31);
        const int64_t base = A.slice_base[s];
        const int w = A.slice_width[s];
        Acc y0 = 0, y1 = 0, y2 = 0;
        // FP32 storage (off-diagonal blocks only): the row's diagonal block is minus the FP64 sum
        // of its stored blocks, summed here in storage order while the row streams past
        RowSum<VT> S;
        const int32_t* cp = A.col + base + lane;
        const VT* vp = val + 9 * base + lane;
#pragma unroll 2
        for (int k = 0; k < w; ++k) {
            const int64_t c = ld_once(cp + 32 * k);
            const Acc x0 = (Acc)x[3 * c], x1 = (Acc)x[3 * c + 1], x2 = (Acc)x[3 * c + 2];
            const VT* v = vp + 288 * (int64_t)k;
            Acc b[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) b[q] = (Acc)mval(ld_once(v + 32 * q));
            S.add(b);
            y0 += b[0] * x0 + b[1] * x1 + b[2] * x2;
            y1 += b[3] * x0 + b[4] * x1 + b[5] * x2;
            y2 += b[6] * x0 + b[7] * x1 + b[8] * x2;
        }
        if (row < A.n_node) {
            if (S.on(A)) {
                const double x0 = (double)x[3 * row], x1 = (double)x[3 * row + 1], x2 = (double)x[3 * row + 2];
                y0 = (Acc)((double)y0 + S.d(0) * x0 + S.d(1) * x1 + S.d(2) * x2);
                y1 = (Acc)((double)y1 + S.d(3) * x0 + S.d(4) * x1 + S.d(5) * x2);
                y2 = (Acc)((double)y2 + S.d(6) * x0 + S.d(7) * x1 + S.d(8) * x2);
            }
            if (A.fixed) {
                if (A.fixed[3 * row]) y0 = (Acc)x[3 * row];
                if (A.fixed[3 * row + 1]) y1 = (Acc)x[3 * row + 1];
                if (A.fixed[3 * row + 2]) y2 = (Acc)x[3 * row + 2];
            }
            y[3 * row] = (XT)y0;
            y[3 * row + 1] = (XT)y1;
            y[3 * row + 2] = (XT)y2;
            if (DOT)
                acc += (double)x[3 * row] * (double)(XT)y0 + (double)x[3 * row + 1] * (double)(XT)y1 +
                       (double)x[3 * row + 2] * (double)(XT)y2;
        }
    }
    if (!DOT) return;
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc;
    if (!arrive_last(&st->counter)) return;
    const double pq = reduce_partials(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
        st->counter = 0;
        st->pq = pq;
        if (!(pq > 0.0)) {
            // KSP_DIVERGED_INDEFINITE_MAT (or NaN); the iteration counts
            st->its += 1;
            st->status = pq != pq ? MPHY_ERR_DIVERGED : MPHY_ERR_INDEFINITE;
            st->done = 1;
        } else {
            st->alpha = st->rz / pq;
        }
    }
}

// z = G^T t with the fused (r, z), (z, z); INIT also sets p = z and the initial state.
template <typename XT, bool INIT>
__global__ void __launch_bounds__(kThreads) factor_apply_kernel(SellView A, CoarseView cv, const FactorT* __restrict__ val,
                                                                const XT* __restrict__ t, XT* __restrict__ z,
                                                                const XT* __restrict__ r, XT* __restrict__ p,
                                                                double* __restrict__ part_rz,
                                                                double* __restrict__ part_zz, PcgState* st,
                                                                double rtol, double abstol, double dtol, int maxit,
                                                                int norm_type) {
    using Acc = typename AccOf<XT>::type;
    __shared__ double sh[32];
    if (!INIT && st->done) return;
    const bool unprec = INIT ? norm_type == 1 : st->norm_type == 1;
    double a1 = 0.0, a2 = 0.0;
    const int64_t rows = (int64_t)A.n_slices * 32;
    for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < rows;
         row += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = row >> 5;
        const int lane = (int)(row & 31);
        const int64_t base = A.slice_base[s];
        const int w = A.slice_width[s];
        Acc y0 = 0, y1 = 0, y2 = 0;
        const int32_t* cp = A.col + base + lane;
        const FactorT* vp = val + 9 * base + lane;
#pragma unroll 2
        for (int k = 0; k < w; ++k) {
            const int64_t c = cp[32 * k];
            const Acc x0 = t[3 * c], x1 = t[3 * c + 1], x2 = t[3 * c + 2];
            const FactorT* v = vp + 288 * (int64_t)k;
            y0 += (Acc)mval(v[0]) * x0 + (Acc)mval(v[32]) * x1 + (Acc)mval(v[64]) * x2;
            y1 += (Acc)mval(v[96]) * x0 + (Acc)mval(v[128]) * x1 + (Acc)mval(v[160]) * x2;
            y2 += (Acc)mval(v[192]) * x0 + (Acc)mval(v[224]) * x1 + (Acc)mval(v[256]) * x2;
        }
        if (row < A.n_node) {
            if (cv.n_agg > 0) {  // two-level: + Z c
                double zc[3];
                coarse_node_value(cv, row, zc);
                if (!cv.fixed[3 * row]) y0 += (Acc)zc[0];
                if (!cv.fixed[3 * row + 1]) y1 += (Acc)zc[1];
                if (!cv.fixed[3 * row + 2]) y2 += (Acc)zc[2];
            }
            const XT zz[3] = {(XT)y0, (XT)y1, (XT)y2};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                z[3 * row + c] = zz[c];
                if (INIT) p[3 * row + c] = zz[c];
                a1 += (double)r[3 * row + c] * (double)zz[c];
                a2 += unprec ? (double)r[3 * row + c] * (double)r[3 * row + c] : (double)zz[c] * (double)zz[c];
            }
        }
    }
    a1 = block_sum(a1, sh);
    if (threadIdx.x == 0) part_rz[blockIdx.x] = a1;
    a2 = block_sum(a2, sh);
    if (threadIdx.x == 0) part_zz[blockIdx.x] = a2;
    if (!arrive_last(&st->counter)) return;
    const double rz = reduce_partials(part_rz, gridDim.x, sh);
    const double zz = reduce_partials(part_zz, gridDim.x, sh);
    if (threadIdx.x == 0) {
        st->counter = 0;
        if (INIT) finish_init(st, rz, zz, rtol, abstol, dtol, maxit, norm_type);
        else finish_iter(st, rz, zz);
    }
}

// r = b - A x in FP64 with the fused ||r||^2
template <typename VT>
__global__ void __launch_bounds__(kThreads) residual_kernel(SellView A, const VT* __restrict__ val,
                                                            const double* __restrict__ x, const double* __restrict__ b,
                                                            double* __restrict__ r, double* __restrict__ partials,
                                                            uint32_t* counter, double* out) {
    __shared__ double sh[32];
    double acc = 0.0;
    const int64_t rows = (int64_t)A.n_slices * 32;
    for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < rows;
         row += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = row >> 5;
        const int lane = (int)(row & 31);
        const int64_t base = A.slice_base[s];
        const int w = A.slice_width[s];
        double y0 = 0, y1 = 0, y2 = 0;
        RowSum<VT> S;  // as in spmv_kernel
        const int32_t* cp = A.col + base + lane;
        const VT* vp = val + 9 * base + lane;
#pragma unroll 2
        for (int k = 0; k < w; ++k) {
            const int64_t c = cp[32 * k];
            const double x0 = x[3 * c], x1 = x[3 * c + 1], x2 = x[3 * c + 2];
            const VT* v = vp + 288 * (int64_t)k;
            double b[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) b[q] = (double)v[32 * q];
            S.add(b);
            y0 += b[0] * x0 + b[1] * x1 + b[2] * x2;
            y1 += b[3] * x0 + b[4] * x1 + b[5] * x2;
            y2 += b[6] * x0 + b[7] * x1 + b[8] * x2;
        }
        if (row < A.n_node) {
            if (S.on(A)) {
                const double x0 = x[3 * row], x1 = x[3 * row + 1], x2 = x[3 * row + 2];
                y0 += S.d(0) * x0 + S.d(1) * x1 + S.d(2) * x2;
                y1 += S.d(3) * x0 + S.d(4) * x1 + S.d(5) * x2;
                y2 += S.d(6) * x0 + S.d(7) * x1 + S.d(8) * x2;
            }
            if (A.fixed) {
                if (A.fixed[3 * row]) y0 = x[3 * row];
                if (A.fixed[3 * row + 1]) y1 = x[3 * row + 1];
                if (A.fixed[3 * row + 2]) y2 = x[3 * row + 2];
            }
            const double ri[3] = {b[3 * row] - y0, b[3 * row + 1] - y1, b[3 * row + 2] - y2};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                r[3 * row + c] = ri[c];
                acc += ri[c] * ri[c];
            }
        }
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc;
    if (!arrive_last(counter)) return;
    const double t = reduce_partials(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
        *counter = 0;
        *out = t;
    }
}

// x += alpha p, r -= alpha q; JAC: z = D^-1 r and the fused (r, z), (z, z)
template <typename XT, bool JAC>
__global__ void __launch_bounds__(kThreads) pcg_update_kernel(int64_t n, XT* __restrict__ x, XT* __restrict__ r,
                                                              XT* __restrict__ z, const XT* __restrict__ p,
                                                              const XT* __restrict__ q, const XT* __restrict__ dinv,
                                                              double* __restrict__ part_rz,
                                                              double* __restrict__ part_zz, PcgState* st) {
    __shared__ double sh[32];
    if (st->done) return;
    const XT alpha = (XT)st->alpha;
    if (!JAC && aligned16(x, r, p, q)) {
        // no reduction: 16-byte pairs, the same arithmetic per element
        using V = typename Pair<XT>::type;
        const int64_t n2 = n >> 1;
        V* x2 = reinterpret_cast<V*>(x);
        V* r2 = reinterpret_cast<V*>(r);
        const V* p2 = reinterpret_cast<const V*>(p);
        const V* q2 = reinterpret_cast<const V*>(q);
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n2; i += (int64_t)gridDim.x * blockDim.x) {
            V xv = ld_once(x2 + i), rv = r2[i];
            const V pv = p2[i], qv = ld_once(q2 + i);
            xv.x = xv.x + alpha * pv.x;
            xv.y = xv.y + alpha * pv.y;
            rv.x = rv.x - alpha * qv.x;
            rv.y = rv.y - alpha * qv.y;
            __stcs(x2 + i, xv);
            r2[i] = rv;
        }
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
            x[n - 1] = x[n - 1] + alpha * p[n - 1];
            r[n - 1] = r[n - 1] - alpha * q[n - 1];
        }
        return;
    }
    const bool unprec = st->norm_type == 1;
    double a1 = 0.0, a2 = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        // x is next read in the next iteration's update and q is dead after this read: both
        // leave L2 first
        __stcs(x + i, ld_once(x + i) + alpha * p[i]);
        const XT ri = r[i] - alpha * ld_once(q + i);
        r[i] = ri;
        if (JAC) {
            const XT zi = dinv[i] * ri;
            z[i] = zi;
            a1 += (double)ri * (double)zi;
            a2 += unprec ? (double)ri * (double)ri : (double)zi * (double)zi;
        }
    }
    if (!JAC) return;
    a1 = block_sum(a1, sh);
    if (threadIdx.x == 0) part_rz[blockIdx.x] = a1;
    a2 = block_sum(a2, sh);
    if (threadIdx.x == 0) part_zz[blockIdx.x] = a2;
    if (!arrive_last(&st->counter)) return;
    const double rz = reduce_partials(part_rz, gridDim.x, sh);
    const double zz = reduce_partials(part_zz, gridDim.x, sh);
    if (threadIdx.x == 0) {
        st->counter = 0;
        finish_iter(st, rz, zz);
    }
}

// Two-level iteration with the ||r|| test: x += alpha p, r -= alpha q and the fused
// (r, D^-1 r), (r, r), left in the state for the coarse GEMV (coarse_gemv_kernel<true>), which
// adds (Z^T r, c) = (r, Z c) to complete (r, z); z = D^-1 r + Z c is then formed only inside the
// direction update (coarse_final_dir_kernel).
template <typename XT>
__global__ void __launch_bounds__(kThreads) pcg_update_rdr_kernel(int64_t n, XT* __restrict__ x, XT* __restrict__ r,
                                                                  const XT* __restrict__ p, const XT* __restrict__ q,
                                                                  const float* __restrict__ dinv,
                                                                  double* __restrict__ part_a,
                                                                  double* __restrict__ part_b, PcgState* st) {
    __shared__ double sh[32];
    if (st->done) return;
    const XT alpha = (XT)st->alpha;
    double a1 = 0.0, a2 = 0.0;
    if (aligned16(x, r, p, q) && (reinterpret_cast<uintptr_t>(dinv) & 7) == 0) {
        using V = typename Pair<XT>::type;
        const int64_t n2 = n >> 1;
        V* x2 = reinterpret_cast<V*>(x);
        V* r2 = reinterpret_cast<V*>(r);
        const V* p2 = reinterpret_cast<const V*>(p);
        const V* q2 = reinterpret_cast<const V*>(q);
        const float2* d2 = reinterpret_cast<const float2*>(dinv);
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n2; i += (int64_t)gridDim.x * blockDim.x) {
            V xv = ld_once(x2 + i), rv = r2[i];
            const V pv = p2[i], qv = ld_once(q2 + i);
            const float2 dv = d2[i];
            xv.x = xv.x + alpha * pv.x;
            xv.y = xv.y + alpha * pv.y;
            rv.x = rv.x - alpha * qv.x;
            rv.y = rv.y - alpha * qv.y;
            __stcs(x2 + i, xv);
            r2[i] = rv;
            a1 += (double)rv.x * ((double)dv.x * (double)rv.x) + (double)rv.y * ((double)dv.y * (double)rv.y);
            a2 += (double)rv.x * (double)rv.x + (double)rv.y * (double)rv.y;
        }
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
            x[n - 1] = x[n - 1] + alpha * p[n - 1];
            const XT ri = r[n - 1] - alpha * q[n - 1];
            r[n - 1] = ri;
            a1 += (double)ri * ((double)dinv[n - 1] * (double)ri);
            a2 += (double)ri * (double)ri;
        }
    } else {
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
            __stcs(x + i, ld_once(x + i) + alpha * p[i]);
            const XT ri = r[i] - alpha * ld_once(q + i);
            r[i] = ri;
            a1 += (double)ri * ((double)dinv[i] * (double)ri);
            a2 += (double)ri * (double)ri;
        }
    }
    a1 = block_sum(a1, sh);
    if (threadIdx.x == 0) part_a[blockIdx.x] = a1;
    a2 = block_sum(a2, sh);
    if (threadIdx.x == 0) part_b[blockIdx.x] = a2;
    if (!arrive_last(&st->counter)) return;
    const double rdr = reduce_partials(part_a, gridDim.x, sh);
    const double rr = reduce_partials(part_b, gridDim.x, sh);
    if (threadIdx.x == 0) {
        st->counter = 0;
        st->rdr = rdr;
        st->rr = rr;
    }
}

template <typename XT>
__global__ void __launch_bounds__(kThreads) pcg_direction_kernel(int64_t n, XT* __restrict__ p, const XT* __restrict__ z,
                                                                 const PcgState* st) {
    if (st->done) return;
    const XT beta = (XT)st->beta;
    if (aligned16(p, z, p, z)) {
        // 16-byte pairs, the same arithmetic per element
        using V = typename Pair<XT>::type;
        const int64_t n2 = n >> 1;
        V* p2 = reinterpret_cast<V*>(p);
        const V* z2 = reinterpret_cast<const V*>(z);
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n2; i += (int64_t)gridDim.x * blockDim.x) {
            const V zv = ld_once(z2 + i);
            V pv = p2[i];
            pv.x = zv.x + beta * pv.x;
            pv.y = zv.y + beta * pv.y;
            p2[i] = pv;
        }
        if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) p[n - 1] = z[n - 1] + beta * p[n - 1];
        return;
    }
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = ld_once(z + i) + beta * p[i];
}

// r = b, x = 0; JAC: z = D^-1 b, p = z, the fused (r, z), (z, z) and the initial state
template <typename XT, bool JAC>
__global__ void __launch_bounds__(kThreads) pcg_init_kernel(int64_t n, const XT* __restrict__ b, XT* __restrict__ x,
                                                            XT* __restrict__ r, XT* __restrict__ z, XT* __restrict__ p,
                                                            const XT* __restrict__ dinv, double* __restrict__ part_rz,
                                                            double* __restrict__ part_zz, PcgState* st, double rtol,
                                                            double abstol, double dtol, int maxit, int norm_type) {
    __shared__ double sh[32];
    double a1 = 0.0, a2 = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const XT ri = b[i];
        x[i] = 0;
        r[i] = ri;
        if (JAC) {
            const XT zi = dinv[i] * ri;
            z[i] = zi;
            p[i] = zi;
            a1 += (double)ri * (double)zi;
            a2 += norm_type == 1 ? (double)ri * (double)ri : (double)zi * (double)zi;
        }
    }
    if (!JAC) return;
    a1 = block_sum(a1, sh);
    if (threadIdx.x == 0) part_rz[blockIdx.x] = a1;
    a2 = block_sum(a2, sh);
    if (threadIdx.x == 0) part_zz[blockIdx.x] = a2;
    if (!arrive_last(&st->counter)) return;
    const double rz = reduce_partials(part_rz, gridDim.x, sh);
    const double zz = reduce_partials(part_zz, gridDim.x, sh);
    if (threadIdx.x == 0) {
        st->counter = 0;
        finish_init(st, rz, zz, rtol, abstol, dtol, maxit, norm_type);
    }
}

// ---------------------------------------------------------------- two-level (coarse) apply
// Z^T r of one node added to w (fixed DOFs carry no residual). Rigid-body modes: translations
// and the rotations about z, x, y; linear modes: translations and r_c d_k (u = a + B d).
__device__ __forceinline__ void restrict_node(bool lin, const double rr[3], const double dd[3], double w[12]) {
    w[0] += rr[0];
    w[1] += rr[1];
    w[2] += rr[2];
    if (lin) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 3; ++k) w[3 + 3 * c + k] += rr[c] * dd[k];
    } else {
        w[3] += -dd[1] * rr[0] + dd[0] * rr[1];
        w[4] += -dd[2] * rr[1] + dd[1] * rr[2];
        w[5] += dd[2] * rr[0] - dd[0] * rr[2];
    }
}

// w = Z^T r per aggregate. Work item (a, part) sums a contiguous part of aggregate a's node
// list, kRestrictNodes nodes per thread and step with every load issued before the arithmetic
// (offsets and mask from copies in node-list order, coalesced; only r is gathered); the CTA
// that finishes an aggregate's last part adds the parts' sums in part order, so w does not
// depend on which CTA ran which part. The CTAs walk the items in a grid-stride loop. NM (modes per
// aggregate) is a template parameter, so the rigid-body form keeps six accumulators and fits
// four CTAs per SM.
constexpr int kRestrictNodes = 2;     // nodes per thread and step, all loads issued first
constexpr int kRestrictThreads = 128;  // small CTAs: about one aggregate each at the default coarse size
template <typename XT, int NM>
__global__ void __launch_bounds__(kRestrictThreads, NM == 6 ? 8 : 6) coarse_restrict_kernel(CoarseView cv, int parts,
                                                                                   const XT* __restrict__ r,
                                                                                   const PcgState* st) {
    __shared__ double sh[kRestrictThreads / 32][NM];
    __shared__ bool last;
    if (st && st->done) return;
    constexpr bool lin = NM == 12;
    constexpr int nm = NM;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int items = cv.n_agg * parts;
    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int a = item / parts, part = item - a * parts;
        const int64_t b0 = cv.agg_ptr[a], len = cv.agg_ptr[a + 1] - b0;
        const int64_t lo = b0 + len * part / parts, hi = b0 + len * (part + 1) / parts;
        double w[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int64_t i = lo + threadIdx.x; i < hi; i += kRestrictNodes * (int64_t)blockDim.x) {
            int64_t li[kRestrictNodes], nd[kRestrictNodes];  // positions in the node list, nodes
#pragma unroll
            for (int k = 0; k < kRestrictNodes; ++k) {
                li[k] = i + k * (int64_t)blockDim.x < hi ? i + k * (int64_t)blockDim.x : i;
                nd[k] = cv.agg_nodes[li[k]];
            }
            XT rv[kRestrictNodes][3];
            double dv[kRestrictNodes][3];
            uint8_t fx[kRestrictNodes][3];
#pragma unroll
            for (int k = 0; k < kRestrictNodes; ++k)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    dv[k][c] = cv.dperm[3 * li[k] + c];
                    fx[k][c] = cv.fperm[3 * li[k] + c];
                    rv[k][c] = r[3 * nd[k] + c];
                }
#pragma unroll
            for (int k = 0; k < kRestrictNodes; ++k) {
                if (i + k * (int64_t)blockDim.x >= hi) break;
                double rr[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) rr[c] = fx[k][c] ? 0.0 : (double)rv[k][c];
                restrict_node(lin, rr, dv[k], w);
            }
        }
        // item sum: butterfly per warp, warps added in order
        __syncthreads();  // sh and last of the previous item are no longer read
#pragma unroll
        for (int m = 0; m < 12; ++m) {
            if (m < nm) {
                double v = w[m];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) sh[warp][m] = v;
            }
        }
        __syncthreads();
        double t = 0.0;
        if (threadIdx.x < nm)
            for (int k = 0; k < kRestrictThreads / 32; ++k) t += sh[k][threadIdx.x];
        if (parts == 1) {
            if (threadIdx.x < nm) cv.w[nm * a + threadIdx.x] = t;
            continue;
        }
        if (threadIdx.x < nm) cv.wpart[((int64_t)a * parts + part) * nm + threadIdx.x] = t;
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) last = atomicAdd(cv.wcount + a, 1u) == (uint32_t)parts - 1;
        __syncthreads();
        if (last) {
            if (threadIdx.x < nm) {
                double sum = 0.0;
                for (int k = 0; k < parts; ++k)
                    sum += __ldcg(cv.wpart + ((int64_t)a * parts + k) * nm + threadIdx.x);
                cv.w[nm * a + threadIdx.x] = sum;
            }
            if (threadIdx.x == 0) cv.wcount[a] = 0;
        }
    }
}

// Grid of the restriction: at most one work item per resident CTA (whole aggregates when there
// are about as many aggregates as resident CTAs), so every CTA pays the item's reduction, fence
// and ticket once.
template <typename XT, int NM>
void launch_restrict_nm(const CoarseView& cv, const XT* r, const PcgState* st, cudaStream_t s, int sm) {
    const unsigned grid = resident_grid((const void*)coarse_restrict_kernel<XT, NM>, (int64_t)1 << 40, kRestrictThreads, sm);
    int parts = (int)((int64_t)grid / cv.n_agg);
    parts = std::max(1, std::min(parts, kMaxRestrictParts));
    const unsigned g = (unsigned)std::min<int64_t>(grid, (int64_t)cv.n_agg * parts);
    coarse_restrict_kernel<XT, NM><<<g, kRestrictThreads, 0, s>>>(cv, parts, r, st);
}
template <typename XT>
void launch_restrict(const CoarseView& cv, const XT* r, const PcgState* st, cudaStream_t s, int sm) {
    if (cv.nm == 12) launch_restrict_nm<XT, 12>(cv, r, st, s, sm);
    else launch_restrict_nm<XT, 6>(cv, r, st, s, sm);
}

// c = E^{-1} w = W~^T (W~ w), W~ the FP32 lower tiles of W = L^{-1} (coarse_view.cuh), in two
// passes of two kernels each. A tile kernel has one CTA per stored tile (I, J), J <= I, reading
// it once (a 16 x 16 thread grid, each thread a 4 x 4 patch: one 16-byte load per patch row);
// it writes its 64 partial sums to the tile's slot of gpart: pass 1 W_IJ w_J (rows of I, summed
// across the half warp), pass 2 W_IJ^T y_I (rows of J, summed across the warps in warp order).
// A row kernel then adds each tile row's slots in tile order, so y and c do not depend on which
// CTA ran which tile: pass 1 y_X = sum_{J <= X}, with the row's share of y^T y; pass 2
// c_X = sum_{I >= X}. FIN (two-level iteration with the ||r|| test): the second row kernel has
// one more CTA, which adds the rows' shares of y^T y = w^T E^{-1} w in row order and ends the
// iteration: (r, z) = (r, D^-1 r) + (w, c). The kernel boundaries replace fences and tickets.
__device__ __forceinline__ int64_t lower_tile(int i, int j) { return (int64_t)i * (i + 1) / 2 + j; }

template <int PASS>
__global__ void __launch_bounds__(256) coarse_wtile_kernel(CoarseView cv, const PcgState* st) {
    __shared__ double v[64];
    __shared__ double colp[8][64];
    if (st && st->done) return;
    const int t = blockIdx.x;
    int I = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while (I * (I + 1) / 2 > t) --I;  // the float root, made exact
    while ((I + 1) * (I + 2) / 2 <= t) ++I;
    const int J = t - I * (I + 1) / 2;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tx = lane & 15, ty = 2 * warp + (lane >> 4);
    const float* W = cv.w32 + (int64_t)t * 4096;
    float4 ev[4];
    // the tile's loads first: they do not wait for the vector
#pragma unroll
    for (int a = 0; a < 4; ++a) ev[a] = ld_once(reinterpret_cast<const float4*>(W + 64 * (4 * ty + a) + 4 * tx));
    if (tid < 64) v[tid] = PASS == 0 ? cv.w[64 * J + tid] : cv.y[64 * I + tid];
    __syncthreads();
    double* gp = cv.gpart + (int64_t)t * 128;
    if (PASS == 0) {
        double rp[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            rp[a] = (double)ev[a].x * v[4 * tx] + (double)ev[a].y * v[4 * tx + 1] + (double)ev[a].z * v[4 * tx + 2] +
                    (double)ev[a].w * v[4 * tx + 3];
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) rp[a] += __shfl_xor_sync(0xffffffffu, rp[a], o);
        }
        if (tx == 0)
#pragma unroll
            for (int a = 0; a < 4; ++a) gp[4 * ty + a] = rp[a];
    } else {
        double cp[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double va = v[4 * ty + a];
            cp[0] += (double)ev[a].x * va;
            cp[1] += (double)ev[a].y * va;
            cp[2] += (double)ev[a].z * va;
            cp[3] += (double)ev[a].w * va;
        }
        // column sums: the two half warps, then the warps in order
#pragma unroll
        for (int b = 0; b < 4; ++b) cp[b] += __shfl_xor_sync(0xffffffffu, cp[b], 16);
        if (lane < 16)
#pragma unroll
            for (int b = 0; b < 4; ++b) colp[warp][4 * tx + b] = cp[b];
        __syncthreads();
        if (tid < 64) {
            double x = 0.0;
#pragma unroll
            for (int q = 0; q < 8; ++q) x += colp[q][tid];
            gp[64 + tid] = x;
        }
    }
}

// Row kernel of a pass: CTA X < nb adds tile row X's slots in tile order (kFinishGroups groups
// of 64 threads each take a contiguous share, added in order, so each thread waits for only a
// few loads). Pass 1: y_X = sum_{J <= X} slot(X, J), and FIN: y_X . y_X into rowyy[X]. Pass 2:
// c_X = sum_{I >= X} slot(I, X), and FIN: CTA nb adds rowyy in row order and ends the iteration.
constexpr int kFinishGroups = 16;
template <int PASS, bool FIN>
__global__ void __launch_bounds__(64 * kFinishGroups) coarse_wrow_kernel(CoarseView cv, PcgState* st) {
    __shared__ double part[kFinishGroups][64];
    __shared__ double sh[32];
    if (st && st->done) return;
    const int tid = threadIdx.x;
    const int X = blockIdx.x;
    if (PASS == 1 && FIN && X == cv.nb) {
        double x = tid < cv.nb ? cv.rowyy[tid] : 0.0;  // nb <= 1024: one row each, in row order
        x = block_sum(x, sh);
        if (tid == 0) finish_iter(st, st->rdr + x, st->rr);
        return;
    }
    const int g = tid >> 6, i = tid & 63;
    const int k_lo = PASS == 0 ? 0 : X, k_hi = PASS == 0 ? X + 1 : cv.nb;  // tiles (X, K) / (K, X)
    const int per = (k_hi - k_lo + kFinishGroups - 1) / kFinishGroups;
    const int k0 = k_lo + g * per, k1 = min(k_hi, k0 + per);
    double x = 0.0;
#pragma unroll 4
    for (int K = k0; K < k1; ++K)
        x += PASS == 0 ? cv.gpart[lower_tile(X, K) * 128 + i] : cv.gpart[lower_tile(K, X) * 128 + 64 + i];
    part[g][i] = x;
    __syncthreads();
    if (tid < 64) {
        double c = 0.0;
#pragma unroll
        for (int q = 0; q < kFinishGroups; ++q) c += part[q][tid];
        if (PASS == 0) {
            cv.y[64 * X + tid] = c;
            if (FIN) {
                double yy = c * c;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) yy += __shfl_xor_sync(0xffffffffu, yy, o);
                if ((tid & 31) == 0) sh[tid >> 5] = yy;
            }
        } else {
            cv.c[64 * X + tid] = c;
        }
    }
    if (PASS == 0 && FIN) {
        __syncthreads();
        if (tid == 0) cv.rowyy[X] = sh[0] + sh[1];
    }
}

// the coarse GEMV c = W~^T (W~ w): per pass, one CTA per stored tile, then one per tile row (FIN:
// and one for the end of the iteration)
template <bool FIN>
void launch_gemv(const CoarseView& cv, PcgState* st, cudaStream_t s) {
    const unsigned tiles = (unsigned)((int64_t)cv.nb * (cv.nb + 1) / 2);
    coarse_wtile_kernel<0><<<tiles, 256, 0, s>>>(cv, st);
    coarse_wrow_kernel<0, FIN><<<(unsigned)cv.nb, 64 * kFinishGroups, 0, s>>>(cv, st);
    coarse_wtile_kernel<1><<<tiles, 256, 0, s>>>(cv, st);
    coarse_wrow_kernel<1, FIN><<<(unsigned)(cv.nb + (FIN ? 1 : 0)), 64 * kFinishGroups, 0, s>>>(cv, st);
}

// z = D^{-1} r + Z c with the fused (r, z), (z, z); INIT also sets p = z and the initial state
template <typename XT, bool INIT>
__global__ void __launch_bounds__(kThreads) coarse_final_kernel(int32_t n_node, CoarseView cv, const XT* __restrict__ r,
                                                                XT* __restrict__ z, XT* __restrict__ p,
                                                                const float* __restrict__ dinv,
                                                                double* __restrict__ part_rz,
                                                                double* __restrict__ part_zz, PcgState* st,
                                                                double rtol, double abstol, double dtol, int maxit,
                                                                int norm_type) {
    __shared__ double sh[32];
    if (!INIT && st->done) return;
    const bool unprec = INIT ? norm_type == 1 : st->norm_type == 1;
    double a1 = 0.0, a2 = 0.0;
    // a thread takes the adjacent nodes 2t and 2t + 1: their six DOFs of r, D^-1, z (and p) and
    // their six offsets are three paired accesses each; every load comes before the first store
    using V = typename Pair<XT>::type;
    const bool paired = aligned16(r, z, INIT ? (const void*)p : (const void*)z, z);
    const int64_t npair = ((int64_t)n_node + 1) >> 1;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < npair; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n0 = 2 * t;
        const int cnt = n0 + 1 < n_node ? 2 : 1;
        XT rv[6];
        float dv[6];
        double od[6];
        uint8_t fx[6];
        int32_t ag[2];
        if (cnt == 2 && paired) {
            const V* r2 = reinterpret_cast<const V*>(r + 3 * n0);
            const float2* v2 = reinterpret_cast<const float2*>(dinv + 3 * n0);
            const float2* o2 = reinterpret_cast<const float2*>(cv.d + 3 * n0);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const V a = r2[q];
                const float2 b = v2[q];
                const float2 o = o2[q];
                rv[2 * q] = a.x;
                rv[2 * q + 1] = a.y;
                dv[2 * q] = b.x;
                dv[2 * q + 1] = b.y;
                od[2 * q] = o.x;
                od[2 * q + 1] = o.y;
            }
        } else {
#pragma unroll
            for (int e = 0; e < 6; ++e) {
                const bool in = e < 3 * cnt;
                rv[e] = in ? r[3 * n0 + e] : XT(0);
                dv[e] = in ? dinv[3 * n0 + e] : 0.0f;
                od[e] = in ? (double)cv.d[3 * n0 + e] : 0.0;
            }
        }
#pragma unroll
        for (int e = 0; e < 6; ++e) fx[e] = e < 3 * cnt ? cv.fixed[3 * n0 + e] : (uint8_t)1;
        ag[0] = cv.agg[n0];
        ag[1] = cnt == 2 ? cv.agg[n0 + 1] : ag[0];
        XT zv[6];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            double zc[3];
            coarse_node_value(cv, ag[k], od[3 * k], od[3 * k + 1], od[3 * k + 2], zc);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int e = 3 * k + a;
                zv[e] = (XT)((double)dv[e] * (double)rv[e] + (fx[e] ? 0.0 : zc[a]));
            }
        }
        if (cnt == 2 && paired) {
            V* z2 = reinterpret_cast<V*>(z + 3 * n0);
            V* p2 = reinterpret_cast<V*>(p + 3 * n0);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                V v;
                v.x = zv[2 * q];
                v.y = zv[2 * q + 1];
                z2[q] = v;
                if (INIT) p2[q] = v;
            }
        } else {
#pragma unroll
            for (int e = 0; e < 6; ++e)
                if (e < 3 * cnt) {
                    z[3 * n0 + e] = zv[e];
                    if (INIT) p[3 * n0 + e] = zv[e];
                }
        }
#pragma unroll
        for (int e = 0; e < 6; ++e)
            if (e < 3 * cnt) {
                a1 += (double)rv[e] * (double)zv[e];
                a2 += unprec ? (double)rv[e] * (double)rv[e] : (double)zv[e] * (double)zv[e];
            }
    }
    a1 = block_sum(a1, sh);
    if (threadIdx.x == 0) part_rz[blockIdx.x] = a1;
    a2 = block_sum(a2, sh);
    if (threadIdx.x == 0) part_zz[blockIdx.x] = a2;
    if (!arrive_last(&st->counter)) return;
    const double rz = reduce_partials(part_rz, gridDim.x, sh);
    const double zz = reduce_partials(part_zz, gridDim.x, sh);
    if (threadIdx.x == 0) {
        st->counter = 0;
        if (INIT) finish_init(st, rz, zz, rtol, abstol, dtol, maxit, norm_type);
        else finish_iter(st, rz, zz);
    }
}

// p = z + beta p with z = D^{-1} r + Z c formed in registers only (the two-level iteration with
// the ||r|| test: (r, z) is already known from the update and the GEMV). Same node-pair layout and
// the same arithmetic per entry as coarse_final_kernel followed by pcg_direction_kernel.
template <typename XT>
__global__ void __launch_bounds__(kThreads) coarse_final_dir_kernel(int32_t n_node, CoarseView cv,
                                                                    const XT* __restrict__ r, XT* __restrict__ p,
                                                                    const float* __restrict__ dinv, const PcgState* st) {
    if (st->done) return;
    const XT beta = (XT)st->beta;
    using V = typename Pair<XT>::type;
    const bool paired = aligned16(r, p, r, p);
    const int64_t npair = ((int64_t)n_node + 1) >> 1;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < npair; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n0 = 2 * t;
        const int cnt = n0 + 1 < n_node ? 2 : 1;
        XT rv[6], pv[6];
        float dv[6];
        double od[6];
        uint8_t fx[6];
        int32_t ag[2];
        if (cnt == 2 && paired) {
            const V* r2 = reinterpret_cast<const V*>(r + 3 * n0);
            const float2* v2 = reinterpret_cast<const float2*>(dinv + 3 * n0);
            const V* p2 = reinterpret_cast<const V*>(p + 3 * n0);
            const float2* o2 = reinterpret_cast<const float2*>(cv.d + 3 * n0);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const V a = r2[q], c = p2[q];
                const float2 b = v2[q];
                const float2 o = o2[q];
                rv[2 * q] = a.x;
                rv[2 * q + 1] = a.y;
                dv[2 * q] = b.x;
                dv[2 * q + 1] = b.y;
                pv[2 * q] = c.x;
                pv[2 * q + 1] = c.y;
                od[2 * q] = o.x;
                od[2 * q + 1] = o.y;
            }
        } else {
#pragma unroll
            for (int e = 0; e < 6; ++e) {
                const bool in = e < 3 * cnt;
                rv[e] = in ? r[3 * n0 + e] : XT(0);
                dv[e] = in ? dinv[3 * n0 + e] : 0.0f;
                pv[e] = in ? p[3 * n0 + e] : XT(0);
                od[e] = in ? (double)cv.d[3 * n0 + e] : 0.0;
            }
        }
#pragma unroll
        for (int e = 0; e < 6; ++e) fx[e] = e < 3 * cnt ? cv.fixed[3 * n0 + e] : (uint8_t)1;
        ag[0] = cv.agg[n0];
        ag[1] = cnt == 2 ? cv.agg[n0 + 1] : ag[0];
        XT nv[6];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            double zc[3];
            coarse_node_value(cv, ag[k], od[3 * k], od[3 * k + 1], od[3 * k + 2], zc);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const int e = 3 * k + a;
                const XT z = (XT)((double)dv[e] * (double)rv[e] + (fx[e] ? 0.0 : zc[a]));
                nv[e] = z + beta * pv[e];
            }
        }
        if (cnt == 2 && paired) {
            V* p2 = reinterpret_cast<V*>(p + 3 * n0);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                V v;
                v.x = nv[2 * q];
                v.y = nv[2 * q + 1];
                p2[q] = v;
            }
        } else {
#pragma unroll
            for (int e = 0; e < 6; ++e)
                if (e < 3 * cnt) p[3 * n0 + e] = nv[e];
        }
    }
}

// PCJACOBI: inverse diagonal, a zero diagonal entry (or a node without blocks) gives 1
template <typename VT, typename XT>
__global__ void jacobi_kernel(SellView A, const VT* __restrict__ val, XT* __restrict__ dinv) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < A.n_node; n += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t o = A.dvoff[n];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double d = A.diag64 ? A.diag64[9 * n + 4 * a] : (o != 0xffffffffu ? (double)val[o + 32u * (4 * a)] : 0.0);
            if (A.fixed && A.fixed[3 * n + a]) d = 1.0;
            dinv[3 * n + a] = (XT)(d != 0.0 ? 1.0 / d : 1.0);
        }
    }
}

__global__ void diag_rowsum_kernel(SellView A, const float* __restrict__ val, double* __restrict__ D) {
    const int64_t rows = (int64_t)A.n_slices * 32;
    for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < rows;
         row += (int64_t)gridDim.x * blockDim.x) {
        if (row >= A.n_node) continue;
        const int64_t s = row >> 5;
        const int lane = (int)(row & 31);
        const int64_t base = A.slice_base[s];
        const int w = A.slice_width[s];
        double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const float* vp = val + 9 * base + lane;
        for (int k = 0; k < w; ++k) {
            const float* v = vp + 288 * (int64_t)k;
#pragma unroll
            for (int q = 0; q < 9; ++q) acc[q] += (double)v[32 * q];
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) D[9 * row + q] = -acc[q];
    }
}

__global__ void export_fix_diag_kernel(const double* __restrict__ D, const int64_t* __restrict__ rowptr,
                                       const int32_t* __restrict__ col, const int32_t* __restrict__ assy, int32_t n_free,
                                       double* __restrict__ out) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n_free; r += (int64_t)gridDim.x * blockDim.x) {
        const int32_t dr = assy[r];
        const int32_t n = dr / 3, a = dr % 3;
        for (int64_t k = rowptr[r]; k < rowptr[r + 1]; ++k) {
            const int32_t dc = assy[col[k]];
            if (dc / 3 == n) out[k] = D[9 * (int64_t)n + 3 * a + dc % 3];
        }
    }
}

__global__ void dot_kernel(const double* __restrict__ a, const double* __restrict__ b, int64_t n,
                           double* __restrict__ partials, uint32_t* counter, double* out) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += a[i] * b[i];
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc;
    if (!arrive_last(counter)) return;
    const double t = reduce_partials(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
        *counter = 0;
        *out = t;
    }
}

// Minimal-residual step of a refinement sweep: with q = r_old - r_new (= A d), the dot products
// q.r_old and q.q into out[0], out[1]; deterministic (fixed-order partial sums, last CTA adds).
__global__ void mr_dots_kernel(int64_t n, const double* __restrict__ rold, const double* __restrict__ rnew,
                               double* __restrict__ part1, double* __restrict__ part2, uint32_t* counter,
                               double* out) {
    __shared__ double sh[32];
    double a1 = 0.0, a2 = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double ro = rold[i], q = ro - rnew[i];
        a1 += q * ro;
        a2 += q * q;
    }
    a1 = block_sum(a1, sh);
    if (threadIdx.x == 0) part1[blockIdx.x] = a1;
    a2 = block_sum(a2, sh);
    if (threadIdx.x == 0) part2[blockIdx.x] = a2;
    if (!arrive_last(counter)) return;
    const double t1 = reduce_partials(part1, gridDim.x, sh);
    const double t2 = reduce_partials(part2, gridDim.x, sh);
    if (threadIdx.x == 0) {
        *counter = 0;
        out[0] = t1;
        out[1] = t2;
    }
}

// x += (alpha - 1) d and r = r_old + alpha (r_new - r_old) (the residual of x_old + alpha d) in
// place of r_new, with ||r||^2 into *out.
template <typename XT>
__global__ void mr_combine_kernel(int64_t n, double alpha, double* __restrict__ x, const XT* __restrict__ d,
                                  const double* __restrict__ rold, double* __restrict__ r,
                                  double* __restrict__ partials, uint32_t* counter, double* out) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += (alpha - 1.0) * (double)d[i];
        const double ro = rold[i];
        const double ri = ro + alpha * (r[i] - ro);
        r[i] = ri;
        acc += ri * ri;
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc;
    if (!arrive_last(counter)) return;
    const double t = reduce_partials(partials, gridDim.x, sh);
    if (threadIdx.x == 0) {
        *counter = 0;
        *out = t;
    }
}

template <typename VT>
__global__ void prescribed_diag_kernel(SellView A, const uint8_t* __restrict__ fixed, VT* __restrict__ val) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < A.n_node; n += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t o = A.dvoff[n];
        if (o == 0xffffffffu) continue;
#pragma unroll
        for (int a = 0; a < 3; ++a)
            if (fixed[3 * n + a]) val[o + 32u * (4 * a)] = (VT)1;
    }
}

__global__ void add_scaled_free_kernel(const uint8_t* __restrict__ fixed, const double* __restrict__ f, double scale,
                                       double* __restrict__ rhs, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!fixed[i]) rhs[i] += scale * f[i];
}

template <typename XT>
__global__ void axpy_kernel(double* __restrict__ y, const XT* __restrict__ x, double a, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] += a * (double)x[i];
}

__global__ void to_f32_kernel(const double* __restrict__ in, float* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

template <typename VT>
__global__ void gather_values_kernel(const VT* __restrict__ val, const int64_t* __restrict__ src,
                                     double* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)val[src[i]];
}

__global__ void gather_free_kernel(const double* __restrict__ v, const int32_t* __restrict__ assy,
                                   double* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = v[assy[i]];
}

}  // namespace

// ---------------------------------------------------------------- host wrappers
template <typename VT, typename XT>
void spmv(const SellView& A, const VT* val, const XT* x, XT* y, cudaStream_t s, int sm) {
    const unsigned g = resident_grid((const void*)spmv_kernel<VT, XT, false>, (int64_t)A.n_slices * 32, kThreads, sm);
    spmv_kernel<VT, XT, false><<<g, kThreads, 0, s>>>(A, val, x, y, nullptr, nullptr);
    MPHY_CUDA(cudaGetLastError());
}
template void spmv<double, double>(const SellView&, const double*, const double*, double*, cudaStream_t, int);
template void spmv<float, float>(const SellView&, const float*, const float*, float*, cudaStream_t, int);
template void spmv<float, double>(const SellView&, const float*, const double*, double*, cudaStream_t, int);

template <typename VT, typename XT>
void spmv_dot(const SellView& A, const VT* val, const XT* x, XT* y, double* partials, PcgState* st, cudaStream_t s,
              int sm) {
    MPHY_CUDA(cudaMemsetAsync(st, 0, sizeof(PcgState), s));
    const unsigned g = resident_grid((const void*)spmv_kernel<VT, XT, true>, (int64_t)A.n_slices * 32, kThreads, sm);
    spmv_kernel<VT, XT, true><<<g, kThreads, 0, s>>>(A, val, x, y, partials, st);
    MPHY_CUDA(cudaGetLastError());
}
template void spmv_dot<double, double>(const SellView&, const double*, const double*, double*, double*, PcgState*,
                                       cudaStream_t, int);
template void spmv_dot<float, double>(const SellView&, const float*, const double*, double*, double*, PcgState*,
                                      cudaStream_t, int);

template <typename VT>
void residual_fp64(const SellView& A, const VT* val, const double* x, const double* b, double* r, double* partials,
                   uint32_t* counter, double* out_dev, cudaStream_t s, int sm) {
    residual_kernel<VT><<<resident_grid((const void*)residual_kernel<VT>, (int64_t)A.n_slices * 32, kThreads, sm), kThreads, 0, s>>>(
        A, val, x, b, r, partials, counter, out_dev);
    MPHY_CUDA(cudaGetLastError());
}
template void residual_fp64<double>(const SellView&, const double*, const double*, const double*, double*, double*,
                                    uint32_t*, double*, cudaStream_t, int);
template void residual_fp64<float>(const SellView&, const float*, const double*, const double*, double*, double*,
                                   uint32_t*, double*, cudaStream_t, int);

namespace {
// z_u += Z c on the free displacement DOFs (the prolongation of the coarse correction)
__global__ void __launch_bounds__(kThreads) coarse_prolong_add_kernel(int32_t n_node, CoarseView cv, double* z) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        double zc[3];
        coarse_node_value(cv, n, zc);
#pragma unroll
        for (int a = 0; a < 3; ++a)
            if (!cv.fixed[3 * n + a]) z[3 * n + a] += zc[a];
    }
}
}  // namespace

void coarse_apply_add(const CoarseView& cv, int32_t n_node, const double* r, double* z, cudaStream_t s, int sm) {
    launch_restrict<double>(cv, r, nullptr, s, sm);
    launch_gemv<false>(cv, nullptr, s);
    coarse_prolong_add_kernel<<<stride_grid(n_node, kThreads, sm), kThreads, 0, s>>>(n_node, cv, z);
    MPHY_CUDA(cudaGetLastError());
}

void diag_from_offdiag(const SellView& A, const float* val, double* diag64, cudaStream_t s, int sm) {
    diag_rowsum_kernel<<<stride_grid((int64_t)A.n_slices * 32, kThreads, sm), kThreads, 0, s>>>(A, val, diag64);
    MPHY_CUDA(cudaGetLastError());
}

void export_fix_diagonal(const double* diag64, const int64_t* rowptr, const int32_t* col, const int32_t* assy,
                         int32_t n_free, double* out, cudaStream_t s, int sm) {
    if (n_free <= 0) return;
    export_fix_diag_kernel<<<stride_grid(n_free, kThreads, sm), kThreads, 0, s>>>(diag64, rowptr, col, assy, n_free,
                                                                                  out);
    MPHY_CUDA(cudaGetLastError());
}

void dot_fp64(const double* a, const double* b, int64_t n, double* partials, uint32_t* counter, double* out_dev,
              cudaStream_t s, int sm) {
    dot_kernel<<<resident_grid((const void*)dot_kernel, n, kThreads, sm), kThreads, 0, s>>>(a, b, n, partials, counter, out_dev);
    MPHY_CUDA(cudaGetLastError());
}

template <typename VT>
void set_prescribed_diagonal(const SellView& A, const uint8_t* fixed, VT* val, cudaStream_t s, int sm) {
    prescribed_diag_kernel<VT><<<stride_grid(A.n_node, kThreads, sm), kThreads, 0, s>>>(A, fixed, val);
    MPHY_CUDA(cudaGetLastError());
}
template void set_prescribed_diagonal<double>(const SellView&, const uint8_t*, double*, cudaStream_t, int);
template void set_prescribed_diagonal<float>(const SellView&, const uint8_t*, float*, cudaStream_t, int);

__global__ void prescribed_increment_kernel(const uint8_t* __restrict__ fixed, const double* __restrict__ ramp,
                                            const double* __restrict__ cst, double t, const double* __restrict__ disp,
                                            double* __restrict__ lift, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        lift[i] = fixed[i] ? t * ramp[i] + cst[i] - disp[i] : 0.0;
}

void prescribed_increment(const uint8_t* fixed, const double* ramp, const double* cst, double t, const double* disp,
                          double* lift, int64_t n, cudaStream_t s, int sm) {
    prescribed_increment_kernel<<<stride_grid(n, kThreads, sm), kThreads, 0, s>>>(fixed, ramp, cst, t, disp, lift, n);
    MPHY_CUDA(cudaGetLastError());
}

void add_scaled_free(const uint8_t* fixed, const double* f, double scale, double* rhs, int64_t n, cudaStream_t s,
                     int sm) {
    add_scaled_free_kernel<<<stride_grid(n, kThreads, sm), kThreads, 0, s>>>(fixed, f, scale, rhs, n);
    MPHY_CUDA(cudaGetLastError());
}

void axpy_inplace(double* y, const double* x, double a, int64_t n, cudaStream_t s, int sm) {
    axpy_kernel<double><<<resident_grid((const void*)axpy_kernel<double>, n, kThreads, sm), kThreads, 0, s>>>(y, x, a, n);
    MPHY_CUDA(cudaGetLastError());
}

template <typename VT>
void gather_values(const VT* val, const int64_t* src, double* out, int64_t n, cudaStream_t s, int sm) {
    if (n <= 0) return;
    gather_values_kernel<VT><<<stride_grid(n, kThreads, sm), kThreads, 0, s>>>(val, src, out, n);
    MPHY_CUDA(cudaGetLastError());
}
template void gather_values<double>(const double*, const int64_t*, double*, int64_t, cudaStream_t, int);
template void gather_values<float>(const float*, const int64_t*, double*, int64_t, cudaStream_t, int);

void gather_free(const double* v, const int32_t* assy, double* out, int64_t n_free, cudaStream_t s, int sm) {
    if (n_free <= 0) return;
    gather_free_kernel<<<stride_grid(n_free, kThreads, sm), kThreads, 0, s>>>(v, assy, out, n_free);
    MPHY_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------- PCG driver
template <typename VT, typename XT>
void Pcg<VT, XT>::init(const SellView& A, int sm_count, int chunk) {
    A_ = A;
    sm_ = sm_count;
    chunk_ = chunk > 0 ? chunk : 32;
    n_ = 3 * (int64_t)A.n_node;
    r_.alloc(n_);
    z_.alloc(n_);
    p_.alloc(n_);
    q_.alloc(n_);
    t_.alloc(n_);
    dinv_.alloc(n_);
    dinv32_.alloc(n_);
    const size_t np = (size_t)sm_ * 8 + 8;
    partials_.alloc(np);
    partials2_.alloc(np);
    st_.alloc(1);
    MPHY_CUDA(cudaMemset(st_.p, 0, sizeof(PcgState)));
}

template <typename VT, typename XT>
Pcg<VT, XT>::~Pcg() {
    if (graph_) cudaGraphExecDestroy(graph_);
}

template <typename VT, typename XT>
void Pcg<VT, XT>::record_iterations(const VT* val, XT* x, cudaStream_t s, int n_iter) {
    const unsigned gs = resident_grid((const void*)spmv_kernel<VT, XT, true>, (int64_t)A_.n_slices * 32, kThreads, sm_);
    const unsigned gv = resident_grid((const void*)pcg_update_kernel<XT, true>, n_, kThreads, sm_);
    for (int it = 0; it < n_iter; ++it) {
        spmv_kernel<VT, XT, true><<<gs, kThreads, 0, s>>>(A_, val, p_.p, q_.p, partials_.p, st_.p);
        if (kind_ == PcKind::Jacobi) {
            pcg_update_kernel<XT, true><<<gv, kThreads, 0, s>>>(n_, x, r_.p, z_.p, p_.p, q_.p, dinv_.p, partials_.p,
                                                                 partials2_.p, st_.p);
        } else if (kind_ == PcKind::JacobiCoarse && norm_type == 1) {
            // (r, z) from (r, D^-1 r) and (Z^T r, c): z is formed only inside the direction update
            const unsigned gu = resident_grid((const void*)pcg_update_rdr_kernel<XT>, n_, kThreads, sm_);
            pcg_update_rdr_kernel<XT><<<gu, kThreads, 0, s>>>(n_, x, r_.p, p_.p, q_.p, dinv32_.p, partials_.p,
                                                               partials2_.p, st_.p);
            launch_restrict<XT>(coarse_, r_.p, st_.p, s, sm_);
            launch_gemv<true>(coarse_, st_.p, s);
            coarse_final_dir_kernel<XT><<<resident_grid((const void*)coarse_final_dir_kernel<XT>, A_.n_node, kThreads, sm_),
                                          kThreads, 0, s>>>(A_.n_node, coarse_, r_.p, p_.p, dinv32_.p, st_.p);
            continue;
        } else if (kind_ == PcKind::JacobiCoarse) {
            pcg_update_kernel<XT, false><<<gv, kThreads, 0, s>>>(n_, x, r_.p, z_.p, p_.p, q_.p, nullptr, nullptr,
                                                                  nullptr, st_.p);
            launch_restrict<XT>(coarse_, r_.p, st_.p, s, sm_);
            launch_gemv<false>(coarse_, st_.p, s);
            coarse_final_kernel<XT, false><<<resident_grid((const void*)coarse_final_kernel<XT, false>, A_.n_node, kThreads, sm_), kThreads, 0, s>>>(
                A_.n_node, coarse_, r_.p, z_.p, p_.p, dinv32_.p, partials_.p, partials2_.p, st_.p, 0, 0, 0, 0, norm_type);
        } else {
            pcg_update_kernel<XT, false><<<gv, kThreads, 0, s>>>(n_, x, r_.p, z_.p, p_.p, q_.p, nullptr, nullptr,
                                                                  nullptr, st_.p);
            const unsigned gg = resident_grid((const void*)factor_apply_kernel<XT, false>,
                                              (int64_t)factor_.G.n_slices * 32, kThreads, sm_);
            spmv_kernel<FactorT, XT, false><<<gg, kThreads, 0, s>>>(factor_.G, factor_.gval, r_.p, t_.p, nullptr, st_.p);
            if (kind_ == PcKind::FactorCoarse) {
                launch_restrict<XT>(coarse_, r_.p, st_.p, s, sm_);
                launch_gemv<false>(coarse_, st_.p, s);
            }
            factor_apply_kernel<XT, false><<<gg, kThreads, 0, s>>>(factor_.GT, kind_ == PcKind::FactorCoarse ? coarse_ : CoarseView{},
                                                                    factor_.gtval, t_.p, z_.p, r_.p, p_.p,
                                                                    partials_.p, partials2_.p, st_.p, 0, 0, 0, 0, norm_type);
        }
        pcg_direction_kernel<XT><<<gv, kThreads, 0, s>>>(n_, p_.p, z_.p, st_.p);
    }
}

template <typename VT, typename XT>
int Pcg<VT, XT>::solve(const VT* val, const XT* b, XT* x, double rtol, double abstol, double dtol, int maxit,
                       cudaStream_t s, int32_t* its, double* final_norm) {
    const unsigned gv = stride_grid(n_, kThreads, sm_);
    launches = 0;
    if (kind_ == PcKind::Jacobi) {
        jacobi_kernel<VT, XT><<<stride_grid(A_.n_node, kThreads, sm_), kThreads, 0, s>>>(A_, val, dinv_.p);
        pcg_init_kernel<XT, true><<<gv, kThreads, 0, s>>>(n_, b, x, r_.p, z_.p, p_.p, dinv_.p, partials_.p,
                                                           partials2_.p, st_.p, rtol, abstol, dtol, maxit, norm_type);
        launches += 2;
    } else if (kind_ == PcKind::JacobiCoarse) {
        // the two-level kernels read D^-1 in FP32: a rounded Jacobi preconditioner, the same in
        // every application
        jacobi_kernel<VT, float><<<stride_grid(A_.n_node, kThreads, sm_), kThreads, 0, s>>>(A_, val, dinv32_.p);
        pcg_init_kernel<XT, false><<<gv, kThreads, 0, s>>>(n_, b, x, r_.p, z_.p, p_.p, nullptr, nullptr, nullptr,
                                                            st_.p, rtol, abstol, dtol, maxit, norm_type);
        launch_restrict<XT>(coarse_, r_.p, nullptr, s, sm_);
        launch_gemv<false>(coarse_, nullptr, s);
        coarse_final_kernel<XT, true><<<resident_grid((const void*)coarse_final_kernel<XT, true>, A_.n_node, kThreads, sm_), kThreads, 0, s>>>(
            A_.n_node, coarse_, r_.p, z_.p, p_.p, dinv32_.p, partials_.p, partials2_.p, st_.p, rtol, abstol, dtol,
            maxit, norm_type);
        launches += 8;
    } else {
        pcg_init_kernel<XT, false><<<gv, kThreads, 0, s>>>(n_, b, x, r_.p, z_.p, p_.p, nullptr, nullptr, nullptr,
                                                            st_.p, rtol, abstol, dtol, maxit, norm_type);
        const unsigned gg = stride_grid((int64_t)factor_.G.n_slices * 32, kThreads, sm_);
        spmv_kernel<FactorT, XT, false><<<gg, kThreads, 0, s>>>(factor_.G, factor_.gval, r_.p, t_.p, nullptr, nullptr);
        if (kind_ == PcKind::FactorCoarse) {
            launch_restrict<XT>(coarse_, r_.p, nullptr, s, sm_);
            launch_gemv<false>(coarse_, nullptr, s);
            launches += 5;
        }
        factor_apply_kernel<XT, true><<<gg, kThreads, 0, s>>>(factor_.GT, kind_ == PcKind::FactorCoarse ? coarse_ : CoarseView{},
                                                               factor_.gtval, t_.p, z_.p, r_.p, p_.p,
                                                               partials_.p, partials2_.p, st_.p, rtol, abstol, dtol,
                                                               maxit, norm_type);
        launches += 3;
    }
    MPHY_CUDA(cudaGetLastError());
    if (!graph_ || graph_val_ != (const void*)val || graph_x_ != (void*)x || graph_stream_ != s ||
        graph_kind_ != kind_ || graph_norm_ != norm_type) {
        if (graph_) {
            cudaGraphExecDestroy(graph_);
            graph_ = nullptr;
        }
        cudaGraph_t g;
        MPHY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        record_iterations(val, x, s, chunk_);
        MPHY_CUDA(cudaStreamEndCapture(s, &g));
        MPHY_CUDA(cudaGraphInstantiate(&graph_, g, 0));
        cudaGraphDestroy(g);
        graph_val_ = val;
        graph_x_ = x;
        graph_stream_ = s;
        graph_kind_ = kind_;
        graph_norm_ = norm_type;
    }
    const int per_iter = kind_ == PcKind::Jacobi ? 3
                         : kind_ == PcKind::Factor ? 5
                         : kind_ == PcKind::FactorCoarse ? 10
                         : norm_type == 1 ? 8 : 9;
    PcgState h{};
    // every replay advances at most chunk_ iterations; the device stops at maxit
    const int64_t max_replays = (int64_t)(maxit > 0 ? maxit : 0) / chunk_ + 2;
    for (int64_t rep = 0;; ++rep) {
        MPHY_CUDA(cudaMemcpyAsync(&h, st_.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
        MPHY_CUDA(cudaStreamSynchronize(s));
        if (h.done) break;
        MPHY_REQUIRE(rep < max_replays, MPHY_ERR_CUDA, "internal: CG state never reached done");
        MPHY_CUDA(cudaGraphLaunch(graph_, s));
        launches += (int64_t)per_iter * chunk_;
    }
    if (its) *its = h.its;
    if (final_norm) *final_norm = h.dp;
    return h.status;
}

template class Pcg<double, double>;
template class Pcg<float, float>;

// ---------------------------------------------------------------- iterative refinement
namespace {
__global__ void copy_f64_kernel(const double* __restrict__ in, double* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[i];
}
void to_inner(const double* in, float* out, int64_t n, unsigned g, cudaStream_t s) {
    to_f32_kernel<<<g, kThreads, 0, s>>>(in, out, n);
}
void to_inner(const double* in, double* out, int64_t n, unsigned g, cudaStream_t s) {
    copy_f64_kernel<<<g, kThreads, 0, s>>>(in, out, n);
}
}  // namespace

template <typename XT>
void IterativeRefinement<XT>::init(const SellView& A, int sm_count, int chunk) {
    A_ = A;
    sm_ = sm_count;
    n_ = 3 * (int64_t)A.n_node;
    inner_.init(A, sm_count, chunk);
    r64_.alloc(n_);
    rold_.alloc(n_);
    rin_.alloc(n_);
    d_.alloc(n_);
    partials_.alloc((size_t)sm_count * 8 + 8);
    partials2_.alloc((size_t)sm_count * 8 + 8);
    scalars_.alloc(3);
    counter_.alloc(1);
    MPHY_CUDA(cudaMemset(counter_.p, 0, sizeof(uint32_t)));
}

template <typename XT>
int IterativeRefinement<XT>::solve(const float* val, const double* b, double* x, double rtol, double inner_rtol,
                                   int max_outer, int maxit, cudaStream_t s, int32_t* its, int32_t* sweeps,
                                   double* relres) {
    const unsigned gv = stride_grid(n_, kThreads, sm_);
    launches = 0;
    MPHY_CUDA(cudaMemsetAsync(x, 0, n_ * sizeof(double), s));
    MPHY_CUDA(cudaMemcpyAsync(r64_.p, b, n_ * sizeof(double), cudaMemcpyDeviceToDevice, s));
    dot_fp64(b, b, n_, partials_.p, counter_.p, scalars_.p, s, sm_);
    double bb = 0.0;
    MPHY_CUDA(cudaMemcpyAsync(&bb, scalars_.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    MPHY_CUDA(cudaStreamSynchronize(s));
    launches += 1;
    const double bnorm = std::sqrt(bb);
    int total = 0, k = 0, status = MPHY_OK, inner_status = MPHY_OK;
    bool broke_down = false;
    double rel = bnorm > 0.0 ? 1.0 : 0.0;
    while (rel > rtol && k < max_outer && total < maxit) {
        to_inner(r64_.p, rin_.p, n_, gv, s);
        int32_t it = 0;
        double dn = 0.0;
        // default inner tolerance: what this sweep must remove to reach rtol ||b|| (with a factor
        // 2 to spare), never tighter than rtol: the first sweep solves to rtol, later sweeps only
        // correct the drift of the recurrence residual
        const double tol_in = inner_rtol > 0.0 ? inner_rtol : std::fmin(0.5, std::fmax(rtol, 0.5 * rtol / rel));
        const int st = inner_.solve(val, rin_.p, d_.p, tol_in, 0.0, 1e5, maxit - total, s, &it, &dn);
        inner_status = st;
        launches += inner_.launches + 1;
        total += it;
        ++k;
        if (st == MPHY_ERR_DIVERGED) {  // NaN in the inner solve: the correction is unusable
            status = st;
            break;
        }
        // x += d, then the FP64 residual r_new = b - A x; with q = A d = r_old - r_new the sweep
        // keeps the multiple alpha = (q.r_old)/(q.q) of d that minimises ||b - A (x_old + alpha d)||
        // (alpha = 1 for an accurate correction). A correction cut short by a CG breakdown on the
        // FP32 operator (p.Ap <= 0: the stored operator can be indefinite along directions of
        // near-zero stiffness) then cannot raise the residual, and the next sweep restarts CG.
        MPHY_CUDA(cudaMemcpyAsync(rold_.p, r64_.p, n_ * sizeof(double), cudaMemcpyDeviceToDevice, s));
        axpy_kernel<XT><<<gv, kThreads, 0, s>>>(x, d_.p, 1.0, n_);
        residual_fp64<float>(A_, val, x, b, r64_.p, partials_.p, counter_.p, scalars_.p, s, sm_);
        mr_dots_kernel<<<gv, kThreads, 0, s>>>(n_, rold_.p, r64_.p, partials_.p, partials2_.p, counter_.p,
                                               scalars_.p + 1);
        launches += 3;
        double h3[3] = {0.0, 0.0, 0.0};  // ||r_new||^2, q.r_old, q.q
        MPHY_CUDA(cudaMemcpyAsync(h3, scalars_.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
        MPHY_CUDA(cudaStreamSynchronize(s));
        double rr = h3[0];
        const double alpha = h3[2] > 0.0 ? h3[1] / h3[2] : 1.0;
        if (alpha == alpha && std::fabs(alpha - 1.0) > 1e-12) {
            mr_combine_kernel<XT><<<gv, kThreads, 0, s>>>(n_, alpha, x, d_.p, rold_.p, r64_.p, partials_.p,
                                                          counter_.p, scalars_.p);
            launches += 1;
            MPHY_CUDA(cudaMemcpyAsync(&rr, scalars_.p, sizeof(double), cudaMemcpyDeviceToHost, s));
            MPHY_CUDA(cudaStreamSynchronize(s));
        }
        rel = std::sqrt(rr) / bnorm;
        if (st == MPHY_ERR_INDEFINITE) broke_down = true;
    }
    // one sweep: the inner solve's KSP status decides (its stopping rule is PETSc's); more sweeps:
    // the FP64 true residual does (an unconverged solve that met a breakdown reports it)
    if (status == MPHY_OK)
        status = max_outer <= 1 ? inner_status
                                : (rel > rtol ? (broke_down ? MPHY_ERR_INDEFINITE : MPHY_ERR_NOT_CONVERGED) : MPHY_OK);
    if (its) *its = total;
    if (sweeps) *sweeps = k;
    if (relres) *relres = rel;
    return status;
}

template class Pcg<float, double>;
template class IterativeRefinement<double>;
template class IterativeRefinement<float>;

}  // namespace mphy
