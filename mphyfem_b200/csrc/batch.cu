// batch.cu -- the batched form: many independent problems solved together.
//
// The instances are one block-diagonal union mesh: instance i owns the contiguous nodes
// [node_ptr[i], node_ptr[i+1]) and only elements among them. Assembly therefore runs over the
// union in the single-problem kernels (one element launch for all instances), and the SELL
// operator is block diagonal by construction.
//
// The linear solves of all instances run in ONE persistent launch (batch_pcg_kernel): a
// thread-block cluster takes instances from a work queue (largest first), splits each
// instance's block rows over its CTAs and runs Jacobi-PCG on it with KSPCG semantics per
// instance (SolverPetsc.cpp:250-330 with -ksp_type cg -pc_type jacobi). The two reductions of an
// iteration are cluster-wide: every CTA sums its rows, the partials meet in distributed shared
// memory and every CTA adds them in rank order, so all CTAs hold bitwise the same scalars and
// take the same branches. No grid-wide synchronisation, no per-iteration launches, and an
// instance's iteration count does not hold up the others.
//
// Newton control is per instance and stays on the device (batch_check_kernel applies the
// load-step loop's test of femSolidmechanics2.cpp:762-816 / femSolidmechanics1.cpp:616-636 to
// every instance), so one Newton iteration of the whole batch -- assembly, forces, checks, solves,
// update -- is a single CUDA graph replay with one small read-back.
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "solver.cuh"

namespace cg = cooperative_groups;

namespace mphy {
namespace {

// Deterministic block sum (fixed butterfly per warp, fixed order across warps); valid in all
// threads of warp 0.
__device__ __forceinline__ double bsum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

// Two sums over the whole cluster, returned identically in every thread of every CTA: each
// CTA's partial goes to its shared slot, and after the cluster barrier every thread adds the
// CTAs' slots in rank order. Slots alternate so that a slot is rewritten only after the next
// barrier, by which time every CTA has read it.
__device__ __forceinline__ void cluster_sum2(cg::cluster_group& cl, double& a, double& b, double (*slot)[2], int& par,
                                             double* sh) {
    a = bsum(a, sh);
    b = bsum(b, sh);
    if (threadIdx.x == 0) {
        slot[par][0] = a;
        slot[par][1] = b;
    }
    cl.sync();
    double sa = 0.0, sb = 0.0;
    const unsigned nb = cl.num_blocks();
    for (unsigned c = 0; c < nb; ++c) {
        const double* rs = cl.map_shared_rank(&slot[par][0], c);
        sa += rs[0];
        sb += rs[1];
    }
    par ^= 1;
    a = sa;
    b = sb;
}

struct BatchView {
    const int32_t* node_ptr;  // [n_inst+1]
    const int32_t* order;     // [n_inst] instances, largest first
    int32_t n_inst;
    const uint8_t* active;    // [n_inst] or null (all)
    const double* b;
    double *x, *r, *z, *p, *q, *dinv;
    int32_t* its;             // [n_inst]
    int32_t* status;
    double* dp;               // final and initial residual norms of the convergence test
    double* dp0;
    int32_t* its_total;       // [n_inst] running sum over solves, or null
    uint32_t* work;           // work-queue head, zero at launch
    double rtol, abstol, dtol;
    int32_t maxit, norm_type;
    // two-level variant: ns slabs per instance along its long axis, 6 rigid-body modes each
    int32_t ns;
    const double* slab_geo;   // [n_inst][4]: long axis, lo, hi, length scale of the offsets
    const double* slab_cent;  // [n_inst][kMaxSlabs][3] slab centroids (reference coordinates)
    const double* coords;     // [n_node][3] reference coordinates
    const uint8_t* fixed;     // [3 n_node] prescribed DOFs (zero rows of Z)
    const uint8_t* slab;      // [n_node] slab of every node within its instance
    // E = Z^T A Z without atomics: node n's row sums T_{n,s} (3 x 6 each, own slab first, then
    // every other slab its row reaches, in slab order) at tbuf[18 toff[n] ..]; per (instance,
    // slab pair sn * 8 + sm) the entries of its nodes in slab sn that reach slab sm, in node order
    const uint8_t* omask;     // [n_node] other slabs the row reaches
    const int32_t* toff;      // [n_node]
    const int64_t* lptr;      // [n_inst * 64 + 1]
    const int32_t* lent;      // entry of every list item
    const int32_t* lnode;     // node of every list item
    double* tbuf;             // [entries][18]
};

constexpr int kMaxSlabs = 8;
constexpr int kMaxCoarse = 6 * kMaxSlabs;
constexpr int kMaxWarps = 16;

// Shared workspace of the two-level variant (dynamic shared memory, per CTA).
struct CoarseSmem {
    double Epart[kMaxCoarse * kMaxCoarse];  // this CTA's rows' share of E = Z^T A Z
    double E[kMaxCoarse * kMaxCoarse];      // E, then E^{-1} (Gauss-Jordan in place)
    double wacc[kMaxWarps][kMaxCoarse];     // per-warp partials of Z^T r
    double vec[2][kMaxCoarse + 1];          // cluster-reduction slots (w and r.r)
    double w[kMaxCoarse + 1];               // reduced Z^T r (and r.r)
    double c[kMaxCoarse];                   // E^{-1} Z^T r
    double col[kMaxCoarse];
    int drop[kMaxCoarse];
};

// Z_n (3 x 6): translations and rotations about the slab centroid, zero rows on prescribed DOFs
__device__ __forceinline__ void slab_modes(const BatchView& v, int inst, int64_t n, int s, double Z[3][6]) {
    const double* cen = v.slab_cent + 3 * ((int64_t)inst * kMaxSlabs + s);
    const double h = v.slab_geo[4 * inst + 3];
    const double dx = (v.coords[3 * n] - cen[0]) / h, dy = (v.coords[3 * n + 1] - cen[1]) / h,
                 dz = (v.coords[3 * n + 2] - cen[2]) / h;
    const double m[3][6] = {{1, 0, 0, -dy, 0, dz}, {0, 1, 0, dx, -dz, 0}, {0, 0, 1, 0, dy, -dx}};
    for (int i = 0; i < 3; ++i) {
        const bool fx = v.fixed[3 * n + i] != 0;
        for (int j = 0; j < 6; ++j) Z[i][j] = fx ? 0.0 : m[i][j];
    }
}

// Column i of Z_n: z[r] = Z_n[r][i]
__device__ __forceinline__ void slab_mode_col(const BatchView& v, int inst, int64_t n, int s, int i, double z[3]) {
    const double* cen = v.slab_cent + 3 * ((int64_t)inst * kMaxSlabs + s);
    const double h = v.slab_geo[4 * inst + 3];
    const double dx = (v.coords[3 * n] - cen[0]) / h, dy = (v.coords[3 * n + 1] - cen[1]) / h,
                 dz = (v.coords[3 * n + 2] - cen[2]) / h;
    // the columns of [[1, 0, 0, -dy, 0, dz], [0, 1, 0, dx, -dz, 0], [0, 0, 1, 0, dy, -dx]]
    const double c0 = i == 0 ? 1.0 : i == 3 ? -dy : i == 5 ? dz : 0.0;
    const double c1 = i == 1 ? 1.0 : i == 3 ? dx : i == 4 ? -dz : 0.0;
    const double c2 = i == 2 ? 1.0 : i == 4 ? dy : i == 5 ? -dx : 0.0;
    z[0] = v.fixed[3 * n] ? 0.0 : c0;
    z[1] = v.fixed[3 * n + 1] ? 0.0 : c1;
    z[2] = v.fixed[3 * n + 2] ? 0.0 : c2;
}

// first position in lnode[lo, hi) whose node is >= n (the lists are in node order)
__device__ __forceinline__ int64_t list_lower_bound(const int32_t* __restrict__ lnode, int64_t lo, int64_t hi,
                                                    int64_t n) {
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo) / 2;
        if (lnode[mid] < n) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// The slabs other than its own that every row reaches (the pattern decides them, not the values)
__global__ void slab_mask_kernel(SellView A, const uint8_t* __restrict__ slab, uint8_t* __restrict__ omask) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < A.n_node;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int64_t sl = n >> 5;
        const int lane = (int)(n & 31);
        const int64_t base = A.slice_base[sl];
        const int w = A.slice_width[sl], s = slab[n];
        uint32_t mask = 0;
        for (int k = 0; k < w; ++k) {
            const int sm = slab[A.col[base + 32 * (int64_t)k + lane]];
            if (sm != s) mask |= 1u << sm;
        }
        omask[n] = (uint8_t)mask;
    }
}

// Sum of the per-CTA vectors vec[par][0..len) over the cluster in rank order into w[0..len),
// identical in every CTA.
__device__ __forceinline__ void cluster_sum_vec(cg::cluster_group& cl, CoarseSmem& cs, int len, int& par) {
    cl.sync();
    const unsigned nb = cl.num_blocks();
    for (int t = threadIdx.x; t < len; t += blockDim.x) {
        double acc = 0.0;
        for (unsigned c = 0; c < nb; ++c) acc += cl.map_shared_rank(&cs.vec[par][0], c)[t];
        cs.w[t] = acc;
    }
    par ^= 1;
    __syncthreads();
}

// This CTA's rows' Z^T r and r.r into vec[par]; then the cluster sum into w. No atomics: per
// step of 32 rows a warp sums each slab's six values with a fixed butterfly and lane 0 adds them
// to the warp's own accumulators; the warps' accumulators are then added in warp order.
__device__ __forceinline__ void coarse_restrict(cg::cluster_group& cl, CoarseSmem& cs, const BatchView& v, int inst,
                                                int64_t a0, int64_t a1, double rr, double* sh, int& par) {
    const int K = 6 * v.ns, warp = threadIdx.x >> 5, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
    for (int t = threadIdx.x; t < kMaxWarps * kMaxCoarse; t += blockDim.x) (&cs.wacc[0][0])[t] = 0.0;
    __syncthreads();
    for (int64_t base = a0; base < a1; base += blockDim.x) {  // the same trip count in every thread
        const int64_t n = base + threadIdx.x;
        const bool in = n < a1;
        int s = 0;
        double t[6] = {0, 0, 0, 0, 0, 0};
        if (in) {
            s = v.slab[n];
            double Z[3][6];
            slab_modes(v, inst, n, s, Z);
            const double r0 = v.r[3 * n], r1 = v.r[3 * n + 1], r2 = v.r[3 * n + 2];
#pragma unroll
            for (int j = 0; j < 6; ++j) t[j] = Z[0][j] * r0 + Z[1][j] * r1 + Z[2][j] * r2;
        }
        for (uint32_t present = __reduce_or_sync(0xffffffffu, in ? 1u << s : 0u); present; present &= present - 1) {
            const int sl = __ffs(present) - 1;
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                double x = in && s == sl ? t[j] : 0.0;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                if (lane == 0) cs.wacc[warp][6 * sl + j] += x;
            }
        }
    }
    rr = bsum(rr, sh);
    __syncthreads();
    for (int t = threadIdx.x; t < K; t += blockDim.x) {
        double acc = 0.0;
        for (int w = 0; w < nw; ++w) acc += cs.wacc[w][t];
        cs.vec[par][t] = acc;
    }
    if (threadIdx.x == 0) cs.vec[par][K] = rr;
    cluster_sum_vec(cl, cs, K + 1, par);
}

// c = E^{-1} w (every CTA, from its own copy of E^{-1}); 8 threads per row. The loop runs over
// whole warps (8 K rounded up to 32, blockDim a multiple of 32) so every lane of a warp takes
// part in the shuffles; lanes past the last row add zeros.
__device__ __forceinline__ void coarse_solve(CoarseSmem& cs, int K) {
    const int T8 = (8 * K + 31) & ~31;
    for (int t = threadIdx.x; t < T8; t += blockDim.x) {
        const int row = t >> 3, part = t & 7;
        double acc = 0.0;
        if (row < K)
            for (int j = part; j < K; j += 8) acc += cs.E[row * kMaxCoarse + j] * cs.w[j];
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        acc += __shfl_xor_sync(0xffffffffu, acc, 4);
        if (part == 0 && row < K) cs.c[row] = acc;
    }
    __syncthreads();
}

// E = Z^T A Z of the instance (this CTA's rows, then the cluster sum), its inverse in place.
// No atomics, every sum in a fixed order: each row's sums per slab go to the row's entries, then
// every value of this CTA's share of E is one thread's sum over its list in node order.
template <typename VT>
__device__ void coarse_setup(cg::cluster_group& cl, CoarseSmem& cs, const SellView& A, const VT* __restrict__ val,
                             const BatchView& v, int inst, int64_t a0, int64_t a1) {
    const int K = 6 * v.ns;
    for (int t = threadIdx.x; t < kMaxCoarse * kMaxCoarse; t += blockDim.x) cs.Epart[t] = 0.0;
    for (int64_t n = a0 + threadIdx.x; n < a1; n += blockDim.x) {
        const int sn = v.slab[n];
        const int64_t sl = n >> 5;
        const int lane = (int)(n & 31);
        const int64_t base = A.slice_base[sl];
        const int w = A.slice_width[sl];
        double* out = v.tbuf + 18 * (int64_t)v.toff[n];
        uint32_t todo = v.omask[n];
        for (int want = sn;;) {
            double T[3][6] = {{0}};
            double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // FP32 storage: the row's sum, in storage order
            for (int k = 0; k <= w; ++k) {
                double blk[9];
                int64_t m;
                if (k < w) {
                    m = A.col[base + 32 * (int64_t)k + lane];
                    const VT* p = val + 9 * (base + 32 * (int64_t)k) + lane;
                    bool any = false;
                    for (int q = 0; q < 9; ++q) {
                        blk[q] = (double)p[32 * q];
                        S[q] += blk[q];
                        any |= blk[q] != 0.0;
                    }
                    if (!any) continue;
                } else {
                    // the FP32 storage's diagonal block, minus the row's sum: the own slab's pass
                    if (!A.diag64 || want != sn) break;
                    m = n;
                    for (int q = 0; q < 9; ++q) blk[q] = -S[q];
                }
                const int sm = v.slab[m];
                if (sm != want) continue;
                if (A.fixed)
                    for (int q = 0; q < 9; ++q)
                        if (A.fixed[3 * n + q / 3] || A.fixed[3 * m + q % 3]) blk[q] = 0.0;
                double Zm[3][6];
                slab_modes(v, inst, m, sm, Zm);
                for (int r = 0; r < 3; ++r)
                    for (int j = 0; j < 6; ++j)
                        T[r][j] += blk[3 * r] * Zm[0][j] + blk[3 * r + 1] * Zm[1][j] + blk[3 * r + 2] * Zm[2][j];
            }
            for (int r = 0; r < 3; ++r)
                for (int j = 0; j < 6; ++j) out[6 * r + j] = T[r][j];
            out += 18;
            if (!todo) break;
            want = __ffs(todo) - 1;
            todo &= todo - 1;
        }
    }
    __syncthreads();  // the entries and the zeroed share are visible to the whole CTA
    const int64_t* lp = v.lptr + 64 * (int64_t)inst;
    for (int t = threadIdx.x; t < 64 * 36; t += blockDim.x) {
        const int key = t / 36, val_ = t % 36, sn = key >> 3, sm = key & 7;
        if (sn >= v.ns || sm >= v.ns || lp[key] == lp[key + 1]) continue;
        const int64_t lo = list_lower_bound(v.lnode, lp[key], lp[key + 1], a0);
        const int64_t hi = list_lower_bound(v.lnode, lo, lp[key + 1], a1);
        const int i = val_ / 6, j = val_ % 6;
        double acc = 0.0;
        for (int64_t q = lo; q < hi; ++q) {
            const int64_t n = v.lnode[q];
            const double* T = v.tbuf + 18 * (int64_t)v.lent[q];
            double z[3];
            slab_mode_col(v, inst, n, sn, i, z);
            acc += z[0] * T[j] + z[1] * T[6 + j] + z[2] * T[12 + j];
        }
        cs.Epart[(6 * sn + i) * kMaxCoarse + 6 * sm + j] = acc;
    }
    cl.sync();
    const unsigned nb = cl.num_blocks();
    for (int t = threadIdx.x; t < K * K; t += blockDim.x) {
        const int i = t / K, j = t % K;
        double acc = 0.0;
        for (unsigned c = 0; c < nb; ++c) acc += cl.map_shared_rank(cs.Epart, c)[i * kMaxCoarse + j];
        cs.E[i * kMaxCoarse + j] = acc;
    }
    __syncthreads();
    // modes without free DOFs (a slab of prescribed nodes) become identity rows, dropped below
    if (threadIdx.x == 0) {
        double mx = 0.0;
        for (int i = 0; i < K; ++i) mx = fmax(mx, fabs(cs.E[i * kMaxCoarse + i]));
        for (int i = 0; i < K; ++i) cs.drop[i] = !(cs.E[i * kMaxCoarse + i] > 1e-13 * mx);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < K * K; t += blockDim.x) {
        const int i = t / K, j = t % K;
        if (cs.drop[i] || cs.drop[j]) cs.E[i * kMaxCoarse + j] = i == j ? 1.0 : 0.0;
    }
    __syncthreads();
    // Gauss-Jordan inversion without pivoting (E is symmetric positive definite)
    for (int k = 0; k < K; ++k) {
        for (int i = threadIdx.x; i < K; i += blockDim.x) cs.col[i] = cs.E[i * kMaxCoarse + k];
        __syncthreads();
        const double piv = 1.0 / cs.col[k];
        for (int j = threadIdx.x; j < K; j += blockDim.x)
            cs.E[k * kMaxCoarse + j] = (j == k ? 1.0 : cs.E[k * kMaxCoarse + j]) * piv;
        __syncthreads();
        for (int t = threadIdx.x; t < K * K; t += blockDim.x) {
            const int i = t / K, j = t % K;
            if (i == k) continue;
            const double e = j == k ? 0.0 : cs.E[i * kMaxCoarse + j];
            cs.E[i * kMaxCoarse + j] = e - cs.col[i] * cs.E[k * kMaxCoarse + j];
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < K * K; t += blockDim.x) {
        const int i = t / K, j = t % K;
        if (cs.drop[i] || cs.drop[j]) cs.E[i * kMaxCoarse + j] = 0.0;
    }
    __syncthreads();
}

// y = (A p)_row, FP64 accumulation; p is read through L2 (written by other CTAs of the cluster)
template <typename VT>
__device__ __forceinline__ void row_apply(const SellView& A, const VT* __restrict__ val, const double* p, int64_t row,
                                          double& y0, double& y1, double& y2) {
    const int64_t s = row >> 5;
    const int lane = (int)(row & 31);
    const int64_t base = A.slice_base[s];
    const int w = A.slice_width[s];
    const int32_t* cp = A.col + base + lane;
    const VT* vp = val + 9 * base + lane;
    y0 = y1 = y2 = 0.0;
    RowSum<VT> S;  // FP32 storage: the row's diagonal block, minus the sum of its stored blocks
#pragma unroll 2
    for (int k = 0; k < w; ++k) {
        const int64_t c = cp[32 * k];
        const double x0 = __ldcg(p + 3 * c), x1 = __ldcg(p + 3 * c + 1), x2 = __ldcg(p + 3 * c + 2);
        const VT* v = vp + 288 * (int64_t)k;
        double b[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) b[q] = (double)v[32 * q];
        S.add(b);
        y0 += b[0] * x0 + b[1] * x1 + b[2] * x2;
        y1 += b[3] * x0 + b[4] * x1 + b[5] * x2;
        y2 += b[6] * x0 + b[7] * x1 + b[8] * x2;
    }
    if (S.on(A)) {
        const double x0 = __ldcg(p + 3 * row), x1 = __ldcg(p + 3 * row + 1), x2 = __ldcg(p + 3 * row + 2);
        y0 += S.d(0) * x0 + S.d(1) * x1 + S.d(2) * x2;
        y1 += S.d(3) * x0 + S.d(4) * x1 + S.d(5) * x2;
        y2 += S.d(6) * x0 + S.d(7) * x1 + S.d(8) * x2;
    }
    if (A.fixed) {
        if (A.fixed[3 * row]) y0 = __ldcg(p + 3 * row);
        if (A.fixed[3 * row + 1]) y1 = __ldcg(p + 3 * row + 1);
        if (A.fixed[3 * row + 2]) y2 = __ldcg(p + 3 * row + 2);
    }
}

// COARSE: the two-level preconditioner z = D^{-1} r + Z E^{-1} Z^T r on the instance's slabs (one
// more cluster reduction per iteration: Z^T r together with r.r).
template <typename VT, bool COARSE>
__global__ void __launch_bounds__(512) batch_pcg_kernel(SellView A, const VT* __restrict__ val, BatchView v) {
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank(), nb = (int)cl.num_blocks();
    __shared__ int job[2];
    __shared__ double slot[2][2];
    __shared__ double sh[32];
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    CoarseSmem& cs = *reinterpret_cast<CoarseSmem*>(dyn_smem);  // COARSE only
    const int K = COARSE ? 6 * v.ns : 0;
    int jpar = 0, rpar = 0, vpar = 0;
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) job[jpar] = (int)atomicAdd(v.work, 1u);
        cl.sync();
        const int k = *cl.map_shared_rank(&job[jpar], 0);
        jpar ^= 1;
        if (k >= v.n_inst) break;
        const int inst = v.order[k];
        const int64_t n0 = v.node_ptr[inst], n1 = v.node_ptr[inst + 1];
        // this CTA's rows: a multiple of 32 each, so a warp's rows are one slice where possible
        const int64_t per = (((n1 - n0) + nb - 1) / nb + 31) & ~(int64_t)31;
        const int64_t a0 = min(n1, n0 + per * rank), a1 = min(n1, a0 + per);
        const int64_t d0 = 3 * a0, d1 = 3 * a1;
        if (v.active && !v.active[inst]) {
            for (int64_t i = d0 + threadIdx.x; i < d1; i += blockDim.x) v.x[i] = 0.0;
            if (rank == 0 && threadIdx.x == 0) {
                v.its[inst] = 0;
                v.status[inst] = MPHY_OK;
                v.dp[inst] = 0.0;
                v.dp0[inst] = 0.0;
            }
            continue;
        }
        if constexpr (COARSE) coarse_setup<VT>(cl, cs, A, val, v, inst, a0, a1);
        // x = 0, r = b, z = D^-1 r (+ Z E^-1 Z^T r), p = z (PCJACOBI: a zero diagonal entry gives 1)
        double rz = 0.0, nn = 0.0, rr0 = 0.0;
        for (int64_t n = a0 + threadIdx.x; n < a1; n += blockDim.x) {
            const uint32_t o = A.dvoff[n];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double d = A.diag64 ? A.diag64[9 * n + 4 * c] : (o != 0xffffffffu ? (double)val[o + 32u * (4 * c)] : 0.0);
                if (A.fixed && A.fixed[3 * n + c]) d = 1.0;
                const double di = d != 0.0 ? 1.0 / d : 1.0;
                const double bi = v.b[3 * n + c];
                const double zi = di * bi;
                v.dinv[3 * n + c] = di;
                v.x[3 * n + c] = 0.0;
                v.r[3 * n + c] = bi;
                rr0 += bi * bi;
                if constexpr (!COARSE) {
                    v.z[3 * n + c] = zi;
                    v.p[3 * n + c] = zi;
                    rz += bi * zi;
                    nn += v.norm_type ? bi * bi : zi * zi;
                }
            }
        }
        if constexpr (COARSE) {
            coarse_restrict(cl, cs, v, inst, a0, a1, rr0, sh, vpar);
            coarse_solve(cs, K);
            for (int64_t n = a0 + threadIdx.x; n < a1; n += blockDim.x) {
                const int sl = v.slab[n];
                double Z[3][6];
                slab_modes(v, inst, n, sl, Z);
                const double* cc = cs.c + 6 * sl;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    double zc = 0.0;
                    for (int j = 0; j < 6; ++j) zc += Z[c][j] * cc[j];
                    const double ri = v.r[3 * n + c], zi = v.dinv[3 * n + c] * ri + zc;
                    v.z[3 * n + c] = zi;
                    v.p[3 * n + c] = zi;
                    rz += ri * zi;
                    nn += zi * zi;
                }
            }
        }
        cluster_sum2(cl, rz, nn, slot, rpar, sh);  // also publishes p to the cluster
        if constexpr (COARSE) {
            if (v.norm_type) nn = cs.w[K];
        }
        double dp = sqrt(nn);
        const double dp0 = dp, ttol = fmax(v.rtol * dp, v.abstol);
        int its = 0, status = MPHY_OK;
        bool done = false;
        if (dp != dp) {
            status = MPHY_ERR_DIVERGED;
            done = true;
        } else if (dp <= ttol) {
            done = true;
        } else if (rz == 0.0) {
            its = 1;
            done = true;
        } else if (v.maxit <= 0) {
            status = MPHY_ERR_NOT_CONVERGED;
            done = true;
        }
        while (!done) {
            double pq = 0.0, unused = 0.0;
            for (int64_t n = a0 + threadIdx.x; n < a1; n += blockDim.x) {
                double y0, y1, y2;
                row_apply<VT>(A, val, v.p, n, y0, y1, y2);
                v.q[3 * n] = y0;
                v.q[3 * n + 1] = y1;
                v.q[3 * n + 2] = y2;
                pq += v.p[3 * n] * y0 + v.p[3 * n + 1] * y1 + v.p[3 * n + 2] * y2;
            }
            cluster_sum2(cl, pq, unused, slot, rpar, sh);
            if (!(pq > 0.0)) {  // KSP_DIVERGED_INDEFINITE_MAT (or NaN); the iteration counts
                its += 1;
                status = pq != pq ? MPHY_ERR_DIVERGED : MPHY_ERR_INDEFINITE;
                break;
            }
            const double alpha = rz / pq;
            double rz1 = 0.0, nn1 = 0.0;
            if constexpr (!COARSE) {
                for (int64_t i = d0 + threadIdx.x; i < d1; i += blockDim.x) {
                    const double ri = v.r[i] - alpha * v.q[i];
                    const double zi = v.dinv[i] * ri;
                    v.x[i] += alpha * v.p[i];
                    v.r[i] = ri;
                    v.z[i] = zi;
                    rz1 += ri * zi;
                    nn1 += v.norm_type ? ri * ri : zi * zi;
                }
                cluster_sum2(cl, rz1, nn1, slot, rpar, sh);
            } else {
                double rr1 = 0.0;
                for (int64_t i = d0 + threadIdx.x; i < d1; i += blockDim.x) {
                    const double ri = v.r[i] - alpha * v.q[i];
                    v.x[i] += alpha * v.p[i];
                    v.r[i] = ri;
                    rr1 += ri * ri;
                }
                coarse_restrict(cl, cs, v, inst, a0, a1, rr1, sh, vpar);
                coarse_solve(cs, K);
                for (int64_t n = a0 + threadIdx.x; n < a1; n += blockDim.x) {
                    const int sl = v.slab[n];
                    double Z[3][6];
                    slab_modes(v, inst, n, sl, Z);
                    const double* cc = cs.c + 6 * sl;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        double zc = 0.0;
                        for (int j = 0; j < 6; ++j) zc += Z[c][j] * cc[j];
                        const double ri = v.r[3 * n + c], zi = v.dinv[3 * n + c] * ri + zc;
                        v.z[3 * n + c] = zi;
                        rz1 += ri * zi;
                        nn1 += zi * zi;
                    }
                }
                cluster_sum2(cl, rz1, nn1, slot, rpar, sh);
                if (v.norm_type) nn1 = cs.w[K];
            }
            its += 1;
            dp = sqrt(nn1);
            if (dp != dp) {
                status = MPHY_ERR_DIVERGED;
                break;
            }
            if (dp <= ttol) break;
            if (dp >= v.dtol * dp0) {
                status = MPHY_ERR_DIVERGED;
                break;
            }
            if (its >= v.maxit) {
                status = MPHY_ERR_NOT_CONVERGED;
                break;
            }
            if (rz1 == 0.0) {  // the next iteration would stop at once with beta == 0
                its += 1;
                break;
            }
            const double beta = rz1 / rz;
            rz = rz1;
            for (int64_t i = d0 + threadIdx.x; i < d1; i += blockDim.x) v.p[i] = v.z[i] + beta * v.p[i];
            cl.sync();  // the new direction, visible to every CTA of the cluster
        }
        if (rank == 0 && threadIdx.x == 0) {
            v.its[inst] = its;
            v.status[inst] = status;
            v.dp[inst] = dp;
            v.dp0[inst] = dp0;
            if (v.its_total) v.its_total[inst] += its;
        }
    }
    cl.sync();  // no CTA leaves while another may still read its shared memory
}

// Per-instance load stepping, one CTA per instance: the loop of femSolidmechanics2.cpp:730-851
// (as mphy_newton_run runs it) as a state machine advanced once per batch Newton iteration.
//   RUNNING, iteration it of the step at load factor t:
//     forces: R += t Fext (free DOFs); ||R||
//     it > max_newton, det F < 0 in an element, or divergence (it > 3, NaN or ratio > 1e7)
//         -> failed step: disp = last converged state, t -= dt, dt /= 2 (MyTime::cut), below
//            1% of the first dt the instance stops with MPHY_ERR_TIME_STEP; else retry at t + dt
//     ||R|| < max(tol_abs, tol_rel ||R||_it=1)  -> converged step: the next one starts at t + dt
//            while t <= t_final - 1e-10 and fewer than max_steps steps are done
//     otherwise                                 -> solve this iteration (active)
enum : int32_t { kRunning = 0, kDone = 1, kFailed = 2 };

struct NewtonView {
    const int32_t* node_ptr;
    const int32_t* elem_ptr;
    const uint8_t* fixed;
    const double* fext;
    double* rhs;
    double* disp;
    double* disp_prev;
    const uint8_t* bad_elem;
    double* t;             // load factor of the current step
    double* dt;
    int32_t* steps_done;   // starts at 1, as the reference's counter
    int32_t* it;           // Newton iterations solved in the current step
    int32_t* phase;
    int32_t* status;
    double* tol;
    double* norm;
    int32_t* newton_total;
    int32_t* cuts;
    int32_t* step_rec;     // [max_steps][n_inst] solves of each completed step
    uint8_t* active;
    uint32_t* n_running;
    uint32_t* n_active;
    int32_t n_inst;
    double dt0, t_final, tol_rel, tol_abs;
    int32_t max_steps, max_newton;
};

__global__ void __launch_bounds__(256) batch_step_kernel(NewtonView v) {
    __shared__ double sh[32];
    __shared__ int action;  // 0 solve, 1 converged, 2 failed, 3 inactive
    const int i = blockIdx.x;
    if (v.phase[i] != kRunning) {
        if (threadIdx.x == 0) v.active[i] = 0;
        return;
    }
    const int64_t d0 = 3 * (int64_t)v.node_ptr[i], d1 = 3 * (int64_t)v.node_ptr[i + 1];
    const double ti = v.t[i];
    double s = 0.0;
    for (int64_t k = d0 + threadIdx.x; k < d1; k += blockDim.x) {
        const double r = v.fixed[k] ? v.rhs[k] : v.rhs[k] + ti * v.fext[k];
        v.rhs[k] = r;
        s += r * r;
    }
    int bad = 0;
    for (int64_t e = v.elem_ptr[i] + threadIdx.x; e < v.elem_ptr[i + 1]; e += blockDim.x) bad |= v.bad_elem[e];
    bad = __syncthreads_or(bad);
    s = bsum(s, sh);
    if (threadIdx.x == 0) {
        const double norm = sqrt(s);
        const int it = v.it[i] + 1;
        const double prev = it == 1 ? -1.0 : v.norm[i];
        v.norm[i] = norm;
        int act;
        if (it > v.max_newton || bad) {
            act = 2;
        } else {
            if (it == 1) v.tol[i] = fmax(v.tol_abs, v.tol_rel * norm);
            if (norm < v.tol[i]) act = 1;
            else if (it > 3 && (norm != norm || (prev > -0.1 && norm / prev > 1.0e7))) act = 2;
            else act = 0;
        }
        action = act;
        if (act == 0) {
            v.it[i] = it;
            v.newton_total[i] += 1;
        } else if (act == 1) {
            const int done = v.steps_done[i];
            if (done - 1 < v.max_steps) v.step_rec[(int64_t)(done - 1) * v.n_inst + i] = it - 1;
            v.steps_done[i] = done + 1;
            if (ti <= v.t_final - 1.0e-10 && done + 1 <= v.max_steps) {
                v.t[i] = ti + v.dt[i];
                v.it[i] = 0;
            } else {
                v.phase[i] = kDone;
                action = 3;
            }
        } else {
            const double dt_old = v.dt[i], dt = 0.5 * dt_old;
            v.cuts[i] += 1;
            v.dt[i] = dt;
            if (dt < v.dt0 * 0.01) {
                v.phase[i] = kFailed;
                v.status[i] = MPHY_ERR_TIME_STEP;
                action = 4;  // restore the last converged state and stop
            } else {
                v.t[i] = (ti - dt_old) + dt;  // t -= dt; dt *= 0.5; then the next try's t += dt
                v.it[i] = 0;
            }
        }
        v.active[i] = act == 0;
        if (act == 0) atomicAdd(v.n_active, 1u);
        if (v.phase[i] == kRunning) atomicAdd(v.n_running, 1u);
    }
    __syncthreads();
    const int act = action;
    if (act == 1) {  // a new step starts from the converged state (saveSolution)
        for (int64_t k = d0 + threadIdx.x; k < d1; k += blockDim.x) v.disp_prev[k] = v.disp[k];
    } else if (act == 2 || act == 4) {  // SolutionDataSolid::reset
        for (int64_t k = d0 + threadIdx.x; k < d1; k += blockDim.x) v.disp[k] = v.disp_prev[k];
    }
}

}  // namespace
}  // namespace mphy

// ------------------------------------------------------------------------------- batch handle
struct mphy_batch {
    mphy_solver* s = nullptr;
    int32_t n_inst = 0;
    std::vector<int32_t> node_ptr_host;
    DevBuf<int32_t> node_ptr, order;
    DevBuf<double> r, z, p, q, dinv;
    DevBuf<int32_t> its, status, its_total;
    DevBuf<double> dp, dp0;
    DevBuf<uint32_t> work;
    // load-stepping state (NewtonView)
    DevBuf<int32_t> steps_done, it, phase, nstatus, newton_total, cuts, step_rec;
    DevBuf<double> t, dt, tol, norm;
    DevBuf<uint8_t> active, bad_elem;
    DevBuf<uint32_t> counters;  // [0] running, [1] active
    DevBuf<double> disp, disp_prev, fext;
    DevBuf<int32_t> elem_ptr;
    int32_t rec_steps = 0;
    int32_t cluster = 1, threads = 256;
    int32_t ns = 0;                          // slabs per instance of the two-level variant (0: off)
    DevBuf<double> slab_geo, slab_cent;
    DevBuf<uint8_t> slab_node, omask;  // slab of every node; other slabs its row reaches
    DevBuf<int32_t> toff, lent, lnode;
    DevBuf<int64_t> lptr;
    DevBuf<double> tbuf;
    cudaGraphExec_t graph = nullptr;
    int graph_cluster = 0, graph_threads = 0, graph_ns = 0;
    double graph_key[6] = {0, 0, 0, 0, 0, 0};
    int64_t launches = 0;
    uint32_t* pinned = nullptr;  // [0] instances still running, [1] instances solved in the last iteration
};

namespace {

using namespace mphy;

BatchView batch_view(mphy_batch* b, const uint8_t* active, bool totals, int maxit) {
    mphy_solver* s = b->s;
    BatchView v{};
    v.node_ptr = b->node_ptr.p;
    v.order = b->order.p;
    v.n_inst = b->n_inst;
    v.active = active;
    v.b = s->rhs.p;
    v.x = s->x.p;
    v.r = b->r.p;
    v.z = b->z.p;
    v.p = b->p.p;
    v.q = b->q.p;
    v.dinv = b->dinv.p;
    v.its = b->its.p;
    v.status = b->status.p;
    v.dp = b->dp.p;
    v.dp0 = b->dp0.p;
    v.its_total = totals ? b->its_total.p : nullptr;
    v.work = b->work.p;
    v.rtol = s->opts.rtol;
    v.abstol = s->opts.abstol;
    v.dtol = s->opts.dtol;
    v.maxit = maxit;
    v.norm_type = s->opts.norm_type;
    v.ns = b->ns;
    v.slab_geo = b->slab_geo.p;
    v.slab_cent = b->slab_cent.p;
    v.coords = s->mesh->coords.p;
    v.fixed = s->mesh->fixed.p;
    v.slab = b->slab_node.p;
    v.omask = b->omask.p;
    v.toff = b->toff.p;
    v.lptr = b->lptr.p;
    v.lent = b->lent.p;
    v.lnode = b->lnode.p;
    v.tbuf = b->tbuf.p;
    return v;
}

template <typename VT, bool COARSE>
void launch_pcg(mphy_batch* b, const VT* val, const BatchView& v, cudaStream_t st, int cluster, int threads) {
    const size_t dyn = COARSE ? sizeof(CoarseSmem) : 0;
    static std::atomic<uint64_t> smem_set{0};
    if (COARSE && first_use_on_device(smem_set)) {
        MPHY_CUDA(cudaFuncSetAttribute(batch_pcg_kernel<VT, COARSE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)dyn));
    }
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = dyn;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(cluster);
    int max_clusters = 0;
    MPHY_CUDA(cudaOccupancyMaxActiveClusters(&max_clusters, batch_pcg_kernel<VT, COARSE>, &cfg));
    MPHY_REQUIRE(max_clusters > 0, MPHY_ERR_UNSUPPORTED, "batched solve: this cluster shape cannot be resident");
    const int n_clusters = std::min(max_clusters, b->n_inst);
    cfg.gridDim = dim3((unsigned)(n_clusters * cluster));
    MPHY_CUDA(cudaMemsetAsync(b->work.p, 0, sizeof(uint32_t), st));
    MPHY_CUDA(cudaLaunchKernelEx(&cfg, batch_pcg_kernel<VT, COARSE>, b->s->A, val, v));
    b->launches += 1;
}

void run_pcg(mphy_batch* b, const uint8_t* active, bool totals, int maxit, cudaStream_t st, int cluster, int threads) {
    const BatchView v = batch_view(b, active, totals, maxit);
    if (b->s->mixed) {
        if (b->ns > 0) launch_pcg<float, true>(b, b->s->valf.p, v, st, cluster, threads);
        else launch_pcg<float, false>(b, b->s->valf.p, v, st, cluster, threads);
    } else {
        if (b->ns > 0) launch_pcg<double, true>(b, b->s->val.p, v, st, cluster, threads);
        else launch_pcg<double, false>(b, b->s->val.p, v, st, cluster, threads);
    }
}

bool schedule_ok(int cluster, int threads) {
    return (cluster == 1 || cluster == 2 || cluster == 4 || cluster == 8) && (threads == 128 || threads == 256 || threads == 512);
}

// One Newton iteration of every instance: assembly, per-instance forces / tests / step
// control, the persistent solve of the active instances, disp += x.
void newton_body(mphy_batch* b, const NewtonView& nv, cudaStream_t st) {
    mphy_solver* s = b->s;
    const int64_t nd = 3 * (int64_t)s->mesh->n_node;
    MPHY_CUDA(cudaMemsetAsync(b->bad_elem.p, 0, b->bad_elem.bytes(), st));
    solver_assemble(s, b->disp.p, b->bad_elem.p);
    MPHY_CUDA(cudaMemsetAsync(b->counters.p, 0, 2 * sizeof(uint32_t), st));
    batch_step_kernel<<<b->n_inst, 256, 0, st>>>(nv);
    run_pcg(b, b->active.p, true, s->opts.max_it, st, b->cluster, b->threads);
    axpy_inplace(b->disp.p, s->x.p, 1.0, nd, st, s->ctx->sm_count);
    MPHY_CUDA(cudaGetLastError());
}

}  // namespace

extern "C" {

int mphy_batch_create(mphy_solver* s, int32_t n_inst, const int32_t* node_ptr, mphy_batch** out) {
    return guarded([&] {
        MPHY_REQUIRE(s && node_ptr && out, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(n_inst > 0, MPHY_ERR_INVALID_ARG, "no instances");
        MPHY_REQUIRE(!s->mesh->has_presc && !s->p0, MPHY_ERR_UNSUPPORTED,
                     "the batched form takes clamped displacement elements");
        MPHY_REQUIRE(s->opts.pc_type == MPHY_PC_JACOBI && s->opts.coarse_aggregates <= 0 &&
                         s->opts.precision != MPHY_PREC_MIXED_F32VEC,
                     MPHY_ERR_UNSUPPORTED, "batched solves use Jacobi-PCG with FP64 vectors");
        MPHY_REQUIRE(s->mesh->n_node < INT32_MAX / 3, MPHY_ERR_UNSUPPORTED, "union mesh too large");
        MPHY_REQUIRE(node_ptr[0] == 0 && node_ptr[n_inst] == s->mesh->n_node, MPHY_ERR_INVALID_ARG,
                     "node_ptr must start at 0 and end at the node count");
        for (int32_t i = 0; i < n_inst; ++i)
            MPHY_REQUIRE(node_ptr[i + 1] > node_ptr[i], MPHY_ERR_INVALID_ARG, "empty or unordered instance");
        // every element's nodes lie in one instance (the operator is block diagonal)
        MPHY_CUDA(cudaSetDevice(s->device));
        const mphy_mesh* m = s->mesh;
        {
            std::vector<int32_t> conn((size_t)m->n_elem * m->npe);
            MPHY_CUDA(cudaMemcpy(conn.data(), m->conn.p, conn.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
            std::vector<int32_t> inst_of(m->n_node);
            for (int32_t i = 0; i < n_inst; ++i)
                for (int32_t n = node_ptr[i]; n < node_ptr[i + 1]; ++n) inst_of[n] = i;
            for (int64_t e = 0; e < m->n_elem; ++e) {
                const int32_t i0 = inst_of[conn[e * m->npe]];
                for (int a = 1; a < m->npe; ++a)
                    MPHY_REQUIRE(inst_of[conn[e * m->npe + a]] == i0, MPHY_ERR_INVALID_ARG,
                                 "an element couples two instances");
            }
        }
        auto* b = new mphy_batch;
        try {
            b->s = s;
            b->n_inst = n_inst;
            b->node_ptr_host.assign(node_ptr, node_ptr + n_inst + 1);
            std::vector<int32_t> order(n_inst);
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t c) {
                return node_ptr[a + 1] - node_ptr[a] > node_ptr[c + 1] - node_ptr[c];
            });
            cudaStream_t st = s->ctx->stream;
            const size_t nd = 3 * (size_t)m->n_node, ni = (size_t)n_inst;
            b->node_ptr.alloc(ni + 1);
            b->node_ptr.upload(node_ptr, ni + 1, st);
            b->order.alloc(ni);
            b->order.upload(order.data(), ni, st);
            for (DevBuf<double>* v : {&b->r, &b->z, &b->p, &b->q, &b->dinv}) v->alloc(nd);
            for (DevBuf<int32_t>* v : {&b->its, &b->status, &b->its_total, &b->steps_done, &b->it, &b->phase,
                                       &b->nstatus, &b->newton_total, &b->cuts})
                v->alloc(ni);
            for (DevBuf<double>* v : {&b->dp, &b->dp0, &b->t, &b->dt, &b->tol, &b->norm}) v->alloc(ni);
            b->active.alloc(ni);
            b->bad_elem.alloc((size_t)m->n_elem);
            b->work.alloc(1);
            b->counters.alloc(2);
            {
                // element ranges of the instances (elements of an instance need not be contiguous
                // in general; the union generator makes them so, and the check below enforces it)
                std::vector<int32_t> conn((size_t)m->n_elem * m->npe), eptr(ni + 1, 0);
                MPHY_CUDA(cudaMemcpy(conn.data(), m->conn.p, conn.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
                int32_t cur = 0;
                for (int64_t e = 0; e < m->n_elem; ++e) {
                    const int32_t n = conn[e * m->npe];
                    while (cur < n_inst && n >= node_ptr[cur + 1]) eptr[++cur] = (int32_t)e;
                    MPHY_REQUIRE(n >= node_ptr[cur], MPHY_ERR_INVALID_ARG,
                                 "the elements of an instance must be contiguous and in instance order");
                }
                while (cur < n_inst) eptr[++cur] = m->n_elem;
                b->elem_ptr.alloc(ni + 1);
                b->elem_ptr.upload(eptr.data(), ni + 1, st);
            }
            MPHY_CUDA(cudaMemsetAsync(b->its_total.p, 0, ni * sizeof(int32_t), st));
            MPHY_CUDA(cudaMallocHost(&b->pinned, 4 * sizeof(uint32_t)));
            MPHY_CUDA(cudaStreamSynchronize(st));
        } catch (...) {
            if (b->pinned) cudaFreeHost(b->pinned);
            delete b;
            throw;
        }
        *out = b;
        return (int)MPHY_OK;
    });
}

int mphy_batch_destroy(mphy_batch* b) {
    if (!b) return MPHY_OK;
    cudaSetDevice(b->s->device);
    cudaDeviceSynchronize();
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->pinned) cudaFreeHost(b->pinned);
    delete b;
    return MPHY_OK;
}

int mphy_batch_set_schedule(mphy_batch* b, int32_t cluster, int32_t threads) {
    if (!b) return MPHY_ERR_INVALID_ARG;
    if (!schedule_ok(cluster, threads)) {
        set_error("schedule: cluster in {1,2,4,8}, threads in {128,256,512}");
        return MPHY_ERR_INVALID_ARG;
    }
    b->cluster = cluster;
    b->threads = threads;
    return MPHY_OK;
}

int mphy_batch_set_coarse(mphy_batch* b, int32_t slabs) {
    return guarded([&] {
        MPHY_REQUIRE(b, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(slabs >= 0 && slabs <= kMaxSlabs, MPHY_ERR_INVALID_ARG,
                     "batched coarse space: 0 (off) to 8 slabs per instance");
        if (b->graph) {  // the recorded Newton iteration refers to the coarse buffers replaced here
            MPHY_CUDA(cudaGraphExecDestroy(b->graph));
            b->graph = nullptr;
        }
        if (slabs == 0) {
            b->ns = 0;
            return (int)MPHY_OK;
        }
        const mphy_mesh* m = b->s->mesh;
        const std::vector<double>& X = m->coords_host;
        const size_t ni = (size_t)b->n_inst;
        std::vector<double> geo(4 * ni), cen(3 * ni * kMaxSlabs, 0.0);
        std::vector<uint8_t> slab(m->n_node, 0);
        for (size_t i = 0; i < ni; ++i) {
            const int32_t n0 = b->node_ptr_host[i], n1 = b->node_ptr_host[i + 1];
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
            for (int32_t n = n0; n < n1; ++n)
                for (int d = 0; d < 3; ++d) {
                    lo[d] = std::min(lo[d], X[3 * (size_t)n + d]);
                    hi[d] = std::max(hi[d], X[3 * (size_t)n + d]);
                }
            int ax = 0;
            for (int d = 1; d < 3; ++d)
                if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
            const double len = std::max(hi[ax] - lo[ax], 1e-300);
            // offsets scaled by a slab's diagonal: the rotation modes are O(1) like the translations
            double diag = 0.0;
            for (int d = 0; d < 3; ++d) diag += std::pow(d == ax ? len / slabs : hi[d] - lo[d], 2);
            geo[4 * i] = ax;
            geo[4 * i + 1] = lo[ax];
            geo[4 * i + 2] = lo[ax] + len;
            geo[4 * i + 3] = std::sqrt(std::max(diag, 1e-300));
            std::vector<double> cnt(slabs, 0.0);
            for (int32_t n = n0; n < n1; ++n) {
                int sl = (int)std::floor((X[3 * (size_t)n + ax] - lo[ax]) / len * slabs);
                sl = sl < 0 ? 0 : (sl >= slabs ? slabs - 1 : sl);
                slab[n] = (uint8_t)sl;
                cnt[sl] += 1.0;
                for (int d = 0; d < 3; ++d) cen[3 * (i * kMaxSlabs + sl) + d] += X[3 * (size_t)n + d];
            }
            for (int sl = 0; sl < slabs; ++sl)
                for (int d = 0; d < 3; ++d)
                    if (cnt[sl] > 0.0) cen[3 * (i * kMaxSlabs + sl) + d] /= cnt[sl];
        }
        MPHY_CUDA(cudaSetDevice(b->s->device));
        cudaStream_t st = b->s->ctx->stream;
        b->slab_geo.alloc(geo.size());
        b->slab_geo.upload(geo.data(), geo.size(), st);
        b->slab_cent.alloc(cen.size());
        b->slab_cent.upload(cen.data(), cen.size(), st);
        const int32_t nn = m->n_node;
        b->slab_node.alloc(nn);
        b->slab_node.upload(slab.data(), nn, st);
        b->omask.alloc(nn);
        slab_mask_kernel<<<stride_grid(nn, 256, b->s->ctx->sm_count), 256, 0, st>>>(b->s->A, b->slab_node.p,
                                                                                   b->omask.p);
        MPHY_CUDA(cudaGetLastError());
        std::vector<uint8_t> om(nn);
        MPHY_CUDA(cudaMemcpyAsync(om.data(), b->omask.p, nn, cudaMemcpyDeviceToHost, st));
        MPHY_CUDA(cudaStreamSynchronize(st));
        // entries: own slab first, then the other slabs in slab order; lists per (instance, slab
        // pair) in node order
        std::vector<int32_t> toff(nn);
        int64_t entries = 0;
        for (int32_t n = 0; n < nn; ++n) {
            toff[n] = (int32_t)entries;
            entries += 1 + __builtin_popcount(om[n]);
            MPHY_REQUIRE(entries < INT32_MAX, MPHY_ERR_UNSUPPORTED, "batched coarse space: too many row entries");
        }
        std::vector<int64_t> lptr(64 * ni + 1, 0);
        std::vector<int32_t> lent, lnode;
        lent.reserve(entries);
        lnode.reserve(entries);
        std::vector<std::vector<int32_t>> be(64), bn(64);
        for (size_t i = 0; i < ni; ++i) {
            for (int k = 0; k < 64; ++k) {
                be[k].clear();
                bn[k].clear();
            }
            for (int32_t n = b->node_ptr_host[i]; n < b->node_ptr_host[i + 1]; ++n) {
                const int sn = slab[n];
                const uint32_t o = om[n];
                be[8 * sn + sn].push_back(toff[n]);
                bn[8 * sn + sn].push_back(n);
                for (int sm = 0; sm < slabs; ++sm)
                    if (o >> sm & 1u) {
                        be[8 * sn + sm].push_back(toff[n] + 1 + __builtin_popcount(o & ((1u << sm) - 1u)));
                        bn[8 * sn + sm].push_back(n);
                    }
            }
            for (int k = 0; k < 64; ++k) {
                lent.insert(lent.end(), be[k].begin(), be[k].end());
                lnode.insert(lnode.end(), bn[k].begin(), bn[k].end());
                lptr[64 * i + k + 1] = (int64_t)lent.size();
            }
        }
        b->toff.alloc(nn);
        b->toff.upload(toff.data(), nn, st);
        b->lptr.alloc(lptr.size());
        b->lptr.upload(lptr.data(), lptr.size(), st);
        b->lent.alloc(lent.size());
        b->lent.upload(lent.data(), lent.size(), st);
        b->lnode.alloc(lnode.size());
        b->lnode.upload(lnode.data(), lnode.size(), st);
        b->tbuf.alloc((size_t)entries * 18);
        MPHY_CUDA(cudaStreamSynchronize(st));
        b->ns = slabs;
        return (int)MPHY_OK;
    });
}

int mphy_batch_get_schedule(const mphy_batch* b, int32_t* cluster, int32_t* threads) {
    if (!b) return MPHY_ERR_INVALID_ARG;
    if (cluster) *cluster = b->cluster;
    if (threads) *threads = b->threads;
    return MPHY_OK;
}

int mphy_batch_solve(mphy_batch* b, int32_t maxit, int32_t* its, int32_t* status, double* relres, float* ms) {
    return guarded([&] {
        MPHY_REQUIRE(b, MPHY_ERR_INVALID_ARG, "null argument");
        mphy_solver* s = b->s;
        MPHY_REQUIRE(s->state == MPHY_ASSEMBLY_OK || s->state == MPHY_FACTORISE_OK, MPHY_ERR_STATE,
                     "batched solve: assemble first");
        MPHY_CUDA(cudaSetDevice(s->device));
        cudaStream_t st = s->ctx->stream;
        MPHY_CUDA(cudaEventRecord(s->ctx->ev0, st));
        run_pcg(b, nullptr, false, maxit > 0 ? maxit : s->opts.max_it, st, b->cluster, b->threads);
        MPHY_CUDA(cudaEventRecord(s->ctx->ev1, st));
        MPHY_CUDA(cudaEventSynchronize(s->ctx->ev1));
        s->state = MPHY_FACTORISE_OK;
        if (ms) cudaEventElapsedTime(ms, s->ctx->ev0, s->ctx->ev1);
        const size_t ni = (size_t)b->n_inst;
        if (its) b->its.download(its, ni, st);
        if (status) b->status.download(status, ni, st);
        if (relres) {
            std::vector<double> dp(ni), dp0(ni);
            b->dp.download(dp.data(), ni, st);
            b->dp0.download(dp0.data(), ni, st);
            MPHY_CUDA(cudaStreamSynchronize(st));
            for (size_t i = 0; i < ni; ++i) relres[i] = dp0[i] > 0.0 ? dp[i] / dp0[i] : 0.0;
        }
        MPHY_CUDA(cudaStreamSynchronize(st));
        return (int)MPHY_OK;
    });
}

int mphy_batch_autotune(mphy_batch* b, int32_t maxit, int32_t max_candidates, int32_t* n_candidates,
                        int32_t* clusters, int32_t* threads, float* ms) {
    return guarded([&] {
        MPHY_REQUIRE(b, MPHY_ERR_INVALID_ARG, "null argument");
        mphy_solver* s = b->s;
        MPHY_REQUIRE(s->state == MPHY_ASSEMBLY_OK || s->state == MPHY_FACTORISE_OK, MPHY_ERR_STATE,
                     "autotune: assemble first (the candidates are timed on the assembled system)");
        MPHY_CUDA(cudaSetDevice(s->device));
        cudaStream_t st = s->ctx->stream;
        const int cand_cl[4] = {1, 2, 4, 8}, cand_th[3] = {128, 256, 512};
        float best = 1e30f;
        int bc = b->cluster, bt = b->threads, k = 0;
        for (int ci = 0; ci < 4; ++ci)
            for (int ti = 0; ti < 3; ++ti) {
                const int c = cand_cl[ci], t = cand_th[ti];
                float t_ms = 0.f;
                const int mi = maxit > 0 ? maxit : s->opts.max_it;
                run_pcg(b, nullptr, false, mi, st, c, t);  // warm-up
                MPHY_CUDA(cudaEventRecord(s->ctx->ev0, st));
                run_pcg(b, nullptr, false, mi, st, c, t);
                MPHY_CUDA(cudaEventRecord(s->ctx->ev1, st));
                MPHY_CUDA(cudaEventSynchronize(s->ctx->ev1));
                cudaEventElapsedTime(&t_ms, s->ctx->ev0, s->ctx->ev1);
                if (k < max_candidates) {
                    if (clusters) clusters[k] = c;
                    if (threads) threads[k] = t;
                    if (ms) ms[k] = t_ms;
                }
                ++k;
                if (t_ms < best) {
                    best = t_ms;
                    bc = c;
                    bt = t;
                }
            }
        if (n_candidates) *n_candidates = k;
        b->cluster = bc;
        b->threads = bt;
        s->state = MPHY_FACTORISE_OK;
        return (int)MPHY_OK;
    });
}

int mphy_batch_newton_run(mphy_batch* b, const double* fext_host, const mphy_newton_opts* o, double* disp_host,
                          int32_t* newton_its, int32_t* krylov_its, int32_t* status, mphy_batch_stats* stats) {
    return guarded([&] {
        MPHY_REQUIRE(b && fext_host && o && disp_host, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(o->dt > 0.0 && o->max_steps > 0 && o->max_newton > 0, MPHY_ERR_INVALID_ARG, "bad Newton options");
        mphy_solver* s = b->s;
        MPHY_CUDA(cudaSetDevice(s->device));
        cudaStream_t st = s->ctx->stream;
        const size_t nd = 3 * (size_t)s->mesh->n_node, ni = (size_t)b->n_inst;
        if (!b->disp.p) {
            b->disp.alloc(nd);
            b->disp_prev.alloc(nd);
            b->fext.alloc(nd);
        }
        if (b->rec_steps != o->max_steps) {
            b->step_rec.alloc((size_t)o->max_steps * ni);
            b->rec_steps = o->max_steps;
        }
        b->disp.upload(disp_host, nd, st);
        b->fext.upload(fext_host, nd, st);
        MPHY_CUDA(cudaMemcpyAsync(b->disp_prev.p, b->disp.p, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
        {
            // every instance starts its first step: t = dt, steps_done = 1
            const std::vector<double> t0(ni, o->dt);
            const std::vector<int32_t> one(ni, 1);
            b->t.upload(t0.data(), ni, st);
            b->dt.upload(t0.data(), ni, st);
            b->steps_done.upload(one.data(), ni, st);
            MPHY_CUDA(cudaStreamSynchronize(st));  // the host vectors above are about to go
        }
        const int32_t first_phase = o->t_final >= 1.0e-10 ? kRunning : kDone;
        {
            const std::vector<int32_t> ph(ni, first_phase);
            b->phase.upload(ph.data(), ni, st);
            MPHY_CUDA(cudaStreamSynchronize(st));
        }
        for (DevBuf<int32_t>* v : {&b->it, &b->nstatus, &b->newton_total, &b->cuts, &b->its_total})
            MPHY_CUDA(cudaMemsetAsync(v->p, 0, ni * sizeof(int32_t), st));
        MPHY_CUDA(cudaMemsetAsync(b->step_rec.p, 0, b->step_rec.bytes(), st));
        NewtonView nv{};
        nv.node_ptr = b->node_ptr.p;
        nv.elem_ptr = b->elem_ptr.p;
        nv.fixed = s->mesh->fixed.p;
        nv.fext = b->fext.p;
        nv.rhs = s->rhs.p;
        nv.disp = b->disp.p;
        nv.disp_prev = b->disp_prev.p;
        nv.bad_elem = b->bad_elem.p;
        nv.t = b->t.p;
        nv.dt = b->dt.p;
        nv.steps_done = b->steps_done.p;
        nv.it = b->it.p;
        nv.phase = b->phase.p;
        nv.status = b->nstatus.p;
        nv.tol = b->tol.p;
        nv.norm = b->norm.p;
        nv.newton_total = b->newton_total.p;
        nv.cuts = b->cuts.p;
        nv.step_rec = b->step_rec.p;
        nv.active = b->active.p;
        nv.n_running = b->counters.p;
        nv.n_active = b->counters.p + 1;
        nv.n_inst = b->n_inst;
        nv.dt0 = o->dt;
        nv.t_final = o->t_final;
        nv.tol_rel = o->tol_rel;
        nv.tol_abs = o->tol_abs;
        nv.max_steps = o->max_steps;
        nv.max_newton = o->max_newton;
        const double key[6] = {o->dt, o->t_final, o->tol_rel, o->tol_abs, (double)o->max_steps, (double)o->max_newton};
        // the graph of one batch Newton iteration (rebuilt when the schedule or the options change)
        if (b->graph && (b->graph_cluster != b->cluster || b->graph_threads != b->threads || b->graph_ns != b->ns ||
                         std::memcmp(b->graph_key, key, sizeof(key)) != 0)) {
            MPHY_CUDA(cudaGraphExecDestroy(b->graph));
            b->graph = nullptr;
        }
        if (!b->graph) {
            solver_assemble(s, b->disp.p, b->bad_elem.p);  // outside the capture: first-use kernel attributes
            cudaGraph_t g = nullptr;
            MPHY_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            try {
                newton_body(b, nv, st);
            } catch (...) {
                cudaStreamEndCapture(st, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            MPHY_CUDA(cudaStreamEndCapture(st, &g));
            const cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            MPHY_CUDA(e);
            b->graph_cluster = b->cluster;
            b->graph_threads = b->threads;
            b->graph_ns = b->ns;
            std::memcpy(b->graph_key, key, sizeof(key));
        }
        // prescribed diagonal (FP64) or diagonal rebuild (mixed), element, step control, solve, update
        const int64_t body_launches = 5;
        // every instance needs at most max_steps converged steps and 7 consecutive cuts per step,
        // each costing at most max_newton + 1 iterations
        const int64_t cap = 8LL * o->max_steps * (o->max_newton + 1) + 8;
        mphy_batch_stats bs{};
        int rc = MPHY_OK;
        MPHY_CUDA(cudaEventRecord(s->ctx->ev0, st));
        if (first_phase == kRunning) {
            for (int64_t round = 0;; ++round) {
                if (round >= cap) {
                    rc = MPHY_ERR_NOT_CONVERGED;
                    set_error("batched load stepping: iteration cap reached");
                    break;
                }
                MPHY_CUDA(cudaGraphLaunch(b->graph, st));
                bs.graph_replays += 1;
                bs.kernel_launches += body_launches;
                MPHY_CUDA(cudaMemcpyAsync(b->pinned, b->counters.p, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
                MPHY_CUDA(cudaStreamSynchronize(st));
                if (b->pinned[0] == 0) break;
            }
        }
        MPHY_CUDA(cudaEventRecord(s->ctx->ev1, st));
        MPHY_CUDA(cudaEventSynchronize(s->ctx->ev1));
        cudaEventElapsedTime(&bs.t_ms, s->ctx->ev0, s->ctx->ev1);
        b->disp.download(disp_host, nd, st);
        if (newton_its) b->step_rec.download(newton_its, (size_t)o->max_steps * ni, st);
        if (krylov_its) b->its_total.download(krylov_its, ni, st);
        if (status) b->nstatus.download(status, ni, st);
        std::vector<int32_t> sd(ni);
        b->steps_done.download(sd.data(), ni, st);
        MPHY_CUDA(cudaStreamSynchronize(st));
        bs.steps = sd.empty() ? 0 : *std::max_element(sd.begin(), sd.end()) - 1;
        s->state = MPHY_FACTORISE_OK;
        if (stats) *stats = bs;
        return rc;
    });
}

int mphy_batch_instance_info(mphy_batch* b, int32_t* newton_total, int32_t* cuts, int32_t* steps_done, double* t) {
    return guarded([&] {
        MPHY_REQUIRE(b, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_CUDA(cudaSetDevice(b->s->device));
        cudaStream_t st = b->s->ctx->stream;
        const size_t ni = (size_t)b->n_inst;
        if (newton_total) b->newton_total.download(newton_total, ni, st);
        if (cuts) b->cuts.download(cuts, ni, st);
        if (steps_done) {
            b->steps_done.download(steps_done, ni, st);
            MPHY_CUDA(cudaStreamSynchronize(st));
            for (size_t i = 0; i < ni; ++i) steps_done[i] -= 1;
        }
        if (t) b->t.download(t, ni, st);
        MPHY_CUDA(cudaStreamSynchronize(st));
        return (int)MPHY_OK;
    });
}

}  // extern "C"
