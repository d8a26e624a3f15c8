// krylov.cu -- K4/K5: SpMV over the SELL-32 3x3 layout, Jacobi-PCG, FP64 vector kernels.
//
// Replaces KSPSolve with KSPCG + PCJACOBI (SolverPetsc.cpp:250-314 with the options
// -ksp_type cg -pc_type jacobi). The iteration follows PETSc's documented KSPCG
// (Hestenes-Stiefel, preconditioned-residual norm, KSPConvergedDefault): x0 = 0,
// converged when ||z_k|| <= max(rtol ||z_0||, abstol), diverged when ||z_k|| >= dtol ||z_0||,
// indefinite when p.Ap <= 0, its = iterations performed.
//
// One CG iteration is three kernels: SpMV with the fused p.q reduction; the x/r/z update with
// the fused (r,z) and (z,z) reductions; the p update. Reductions are deterministic: every CTA
// writes a partial sum, and the CTA that finishes last (an atomic ticket, no waiting) adds the
// partials in a fixed order and advances the shared scalar state. Chunks of iterations are
// replayed from a captured CUDA graph; kernels return immediately once the state says done.
#include "krylov.cuh"

namespace mphy {

constexpr int kThreads = 256;

unsigned stride_grid(int64_t n, int threads, int sm_count, int per_sm) {
    const int64_t want = (n + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count * per_sm;
    return (unsigned)(want < 1 ? 1 : (want > cap ? cap : want));
}

namespace {

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

// ---------------------------------------------------------------- SpMV
template <bool DOT>
__global__ void __launch_bounds__(kThreads) spmv_fp64_kernel(SellView A, const double* __restrict__ val,
                                                             const double* __restrict__ x, double* __restrict__ y,
                                                             double* __restrict__ partials, PcgState* st) {
    __shared__ double sh[32];
    if (DOT && st->done) return;
    double acc = 0.0;
    const int64_t rows = (int64_t)A.n_slices * 32;
    for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < rows;
         row += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = row >> 5;
        const int lane = (int)(row & 31);
        const int64_t base = A.slice_base[s];
        const int w = A.slice_width[s];
        double y0 = 0.0, y1 = 0.0, y2 = 0.0;
        const int32_t* cp = A.col + base + lane;
        const double* vp = val + 9 * base + lane;
#pragma unroll 2
        for (int k = 0; k < w; ++k) {
            const int64_t c = cp[32 * k];
            const double x0 = x[3 * c], x1 = x[3 * c + 1], x2 = x[3 * c + 2];
            const double* v = vp + 288 * (int64_t)k;
            y0 += v[0] * x0 + v[32] * x1 + v[64] * x2;
            y1 += v[96] * x0 + v[128] * x1 + v[160] * x2;
            y2 += v[192] * x0 + v[224] * x1 + v[256] * x2;
        }
        if (row < A.n_node) {
            y[3 * row] = y0;
            y[3 * row + 1] = y1;
            y[3 * row + 2] = y2;
            if (DOT) acc += x[3 * row] * y0 + x[3 * row + 1] * y1 + x[3 * row + 2] * y2;
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

// x += alpha p, r -= alpha q, z = D^-1 r, then (r, z) and (z, z)
__global__ void __launch_bounds__(kThreads) pcg_update_kernel(int64_t n, double* __restrict__ x, double* __restrict__ r,
                                                              double* __restrict__ z, const double* __restrict__ p,
                                                              const double* __restrict__ q,
                                                              const double* __restrict__ dinv,
                                                              double* __restrict__ part_rz, double* __restrict__ part_zz,
                                                              PcgState* st) {
    __shared__ double sh[32];
    if (st->done) return;
    const double alpha = st->alpha;
    double a1 = 0.0, a2 = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * q[i];
        r[i] = ri;
        const double zi = dinv[i] * ri;
        z[i] = zi;
        a1 += ri * zi;
        a2 += zi * zi;
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
}

__global__ void __launch_bounds__(kThreads) pcg_direction_kernel(int64_t n, double* __restrict__ p,
                                                                 const double* __restrict__ z, const PcgState* st) {
    if (st->done) return;
    const double beta = st->beta;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// r = b, x = 0, z = D^-1 b, p = z; then (r, z), (z, z) and the initial state
__global__ void __launch_bounds__(kThreads) pcg_init_kernel(int64_t n, const double* __restrict__ b, double* __restrict__ x,
                                                            double* __restrict__ r, double* __restrict__ z,
                                                            double* __restrict__ p, const double* __restrict__ dinv,
                                                            double* __restrict__ part_rz, double* __restrict__ part_zz,
                                                            PcgState* st, double rtol, double abstol, double dtol,
                                                            int maxit) {
    __shared__ double sh[32];
    double a1 = 0.0, a2 = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double ri = b[i];
        const double zi = dinv[i] * ri;
        x[i] = 0.0;
        r[i] = ri;
        z[i] = zi;
        p[i] = zi;
        a1 += ri * zi;
        a2 += zi * zi;
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
        const double dp = sqrt(zz);
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
}

// PCJACOBI: inverse diagonal, a zero diagonal entry is replaced by 1
__global__ void jacobi_kernel(SellView A, const double* __restrict__ val, double* __restrict__ dinv) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < A.n_node; n += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t o = A.dvoff[n];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double d = o != 0xffffffffu ? val[o + 32u * (4 * a)] : 0.0;
            dinv[3 * n + a] = d != 0.0 ? 1.0 / d : 1.0;
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

__global__ void prescribed_diag_kernel(SellView A, const uint8_t* __restrict__ fixed, double* __restrict__ val) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < A.n_node; n += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t o = A.dvoff[n];
        if (o == 0xffffffffu) continue;
#pragma unroll
        for (int a = 0; a < 3; ++a)
            if (fixed[3 * n + a]) val[o + 32u * (4 * a)] = 1.0;
    }
}

__global__ void add_scaled_free_kernel(const uint8_t* __restrict__ fixed, const double* __restrict__ f, double scale,
                                       double* __restrict__ rhs, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (!fixed[i]) rhs[i] += scale * f[i];
}

__global__ void axpy_kernel(double* __restrict__ y, const double* __restrict__ x, double a, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] += a * x[i];
}

__global__ void gather_values_kernel(const double* __restrict__ val, const int64_t* __restrict__ src,
                                     double* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = val[src[i]];
}

__global__ void gather_free_kernel(const double* __restrict__ v, const int32_t* __restrict__ assy,
                                   double* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = v[assy[i]];
}

}  // namespace

void spmv_fp64(const SellView& A, const double* val, const double* x, double* y, cudaStream_t s, int sm) {
    spmv_fp64_kernel<false><<<stride_grid((int64_t)A.n_slices * 32, kThreads, sm), kThreads, 0, s>>>(
        A, val, x, y, nullptr, nullptr);
    MPHY_CUDA(cudaGetLastError());
}

void dot_fp64(const double* a, const double* b, int64_t n, double* partials, uint32_t* counter, double* out_dev,
              cudaStream_t s, int sm) {
    dot_kernel<<<stride_grid(n, kThreads, sm), kThreads, 0, s>>>(a, b, n, partials, counter, out_dev);
    MPHY_CUDA(cudaGetLastError());
}

void set_prescribed_diagonal(const SellView& A, const uint8_t* fixed, double* val, cudaStream_t s, int sm) {
    prescribed_diag_kernel<<<stride_grid(A.n_node, kThreads, sm), kThreads, 0, s>>>(A, fixed, val);
    MPHY_CUDA(cudaGetLastError());
}

void add_scaled_free(const uint8_t* fixed, const double* f, double scale, double* rhs, int64_t n, cudaStream_t s,
                     int sm) {
    add_scaled_free_kernel<<<stride_grid(n, kThreads, sm), kThreads, 0, s>>>(fixed, f, scale, rhs, n);
    MPHY_CUDA(cudaGetLastError());
}

void axpy_inplace(double* y, const double* x, double a, int64_t n, cudaStream_t s, int sm) {
    axpy_kernel<<<stride_grid(n, kThreads, sm), kThreads, 0, s>>>(y, x, a, n);
    MPHY_CUDA(cudaGetLastError());
}

void gather_values(const double* val, const int64_t* src, double* out, int64_t n, cudaStream_t s, int sm) {
    if (n <= 0) return;
    gather_values_kernel<<<stride_grid(n, kThreads, sm), kThreads, 0, s>>>(val, src, out, n);
    MPHY_CUDA(cudaGetLastError());
}

void gather_free(const double* v, const int32_t* assy, double* out, int64_t n_free, cudaStream_t s, int sm) {
    if (n_free <= 0) return;
    gather_free_kernel<<<stride_grid(n_free, kThreads, sm), kThreads, 0, s>>>(v, assy, out, n_free);
    MPHY_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------- PCG driver
void PcgFp64::init(const SellView& A, int sm_count, int chunk) {
    A_ = A;
    sm_ = sm_count;
    chunk_ = chunk > 0 ? chunk : 32;
    n_ = 3 * (int64_t)A.n_node;
    r_.alloc(n_);
    z_.alloc(n_);
    p_.alloc(n_);
    q_.alloc(n_);
    dinv_.alloc(n_);
    const size_t np = (size_t)sm_ * 8 + 8;
    partials_.alloc(np);
    partials2_.alloc(np);
    st_.alloc(1);
    MPHY_CUDA(cudaMemset(st_.p, 0, sizeof(PcgState)));
}

PcgFp64::~PcgFp64() {
    if (graph_) cudaGraphExecDestroy(graph_);
}

void PcgFp64::record_iterations(const double* val, double* x, cudaStream_t s, int n_iter) {
    const unsigned gs = stride_grid((int64_t)A_.n_slices * 32, kThreads, sm_);
    const unsigned gv = stride_grid(n_, kThreads, sm_);
    for (int it = 0; it < n_iter; ++it) {
        spmv_fp64_kernel<true><<<gs, kThreads, 0, s>>>(A_, val, p_.p, q_.p, partials_.p, st_.p);
        pcg_update_kernel<<<gv, kThreads, 0, s>>>(n_, x, r_.p, z_.p, p_.p, q_.p, dinv_.p, partials_.p, partials2_.p,
                                                   st_.p);
        pcg_direction_kernel<<<gv, kThreads, 0, s>>>(n_, p_.p, z_.p, st_.p);
    }
}

int PcgFp64::solve(const double* val, const double* b, double* x, double rtol, double abstol, double dtol, int maxit,
                   cudaStream_t s, int32_t* its, double* final_norm) {
    jacobi_kernel<<<stride_grid(A_.n_node, kThreads, sm_), kThreads, 0, s>>>(A_, val, dinv_.p);
    pcg_init_kernel<<<stride_grid(n_, kThreads, sm_), kThreads, 0, s>>>(n_, b, x, r_.p, z_.p, p_.p, dinv_.p,
                                                                        partials_.p, partials2_.p, st_.p, rtol, abstol,
                                                                        dtol, maxit);
    MPHY_CUDA(cudaGetLastError());
    if (!graph_ || graph_val_ != val || graph_x_ != x || graph_stream_ != s) {
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
    }
    launches = 2;
    PcgState h{};
    // every replay advances at most chunk_ iterations; the device stops at maxit
    const int64_t max_replays = (int64_t)maxit / chunk_ + 2;
    for (int64_t rep = 0;; ++rep) {
        MPHY_CUDA(cudaMemcpyAsync(&h, st_.p, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
        MPHY_CUDA(cudaStreamSynchronize(s));
        if (h.done) break;
        MPHY_REQUIRE(rep < max_replays, MPHY_ERR_CUDA, "internal: CG state never reached done");
        MPHY_CUDA(cudaGraphLaunch(graph_, s));
        launches += 3 * (int64_t)chunk_;
    }
    if (its) *its = h.its;
    if (final_norm) *final_norm = h.dp;
    return h.status;
}

}  // namespace mphy
