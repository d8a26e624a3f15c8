// coarse.cu -- rigid-body coarse space on geometric aggregates (setup side; the per-iteration
// restriction, coarse GEMV and prolongation live in krylov.cu next to the CG state).
//
// Setup per operator:
//   1. centroids of the current coordinates per aggregate and scaled offsets d_n = (x_n - c_a)/H;
//   2. E = Z^T A Z, lower triangle (the factorisation reads no other): one thread per matrix row
//      sums the row's blocks per neighbour aggregate into per-node entries, then one CTA per
//      (aggregate, neighbour) adds the entries in a fixed order -- no atomics, so E is bitwise
//      the same on every run;
//   3. E = L L^T by a right-looking blocked Cholesky (64x64 tiles, FP64), W = L^{-1} by blocked
//      forward substitution, then W rounded to FP32 for the per-iteration E^{-1} w = W~^T (W~ w)
//      (W~^T W~ is symmetric positive definite whatever the rounding, where an FP32 copy of E^{-1}
//      itself can be indefinite when E is ill-conditioned). The aggregates are numbered with the
//      longest box axis slowest, so E is banded; L stays inside the band and the Cholesky and
//      forward-substitution steps touch only the tiles inside it.
#include <algorithm>
#include <array>
#include <cmath>
#include <vector>

#include "coarse.cuh"

namespace mphy {
namespace {

constexpr int T = 64;   // dense tile
constexpr int TP = 65;  // padded shared-memory row

// ---------------------------------------------------------------- modes
__global__ void centroid_kernel(int32_t n_agg, const int64_t* __restrict__ agg_ptr, const int32_t* __restrict__ nodes,
                                const double* __restrict__ X, const double* __restrict__ u, double* __restrict__ cent) {
    __shared__ double sh[3][256];
    for (int a = blockIdx.x; a < n_agg; a += gridDim.x) {
        double s[3] = {0, 0, 0};
        for (int64_t i = agg_ptr[a] + threadIdx.x; i < agg_ptr[a + 1]; i += blockDim.x) {
            const int64_t n = nodes[i];
            for (int d = 0; d < 3; ++d) s[d] += X[3 * n + d] + (u ? u[3 * n + d] : 0.0);
        }
        for (int d = 0; d < 3; ++d) sh[d][threadIdx.x] = s[d];
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if ((int)threadIdx.x < o)
                for (int d = 0; d < 3; ++d) sh[d][threadIdx.x] += sh[d][threadIdx.x + o];
            __syncthreads();
        }
        const double cnt = (double)(agg_ptr[a + 1] - agg_ptr[a]);
        if (threadIdx.x == 0)
            for (int d = 0; d < 3; ++d) cent[3 * a + d] = cnt > 0 ? sh[d][0] / cnt : 0.0;
        __syncthreads();
    }
}

// d_n = (x_n - c_a) / H, stored in FP32: the offsets only choose the coarse basis Z, and every
// kernel (E = Z^T A Z, restriction, prolongation) reads the same rounded values, so Z stays one
// basis while the per-iteration kernels read half the bytes
__global__ void offsets_kernel(int32_t n_node, const int32_t* __restrict__ agg, const double* __restrict__ X,
                               const double* __restrict__ u, const double* __restrict__ cent, double inv_h,
                               float* __restrict__ d) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        const int a = agg[n];
        for (int k = 0; k < 3; ++k)
            d[3 * n + k] = (float)((X[3 * n + k] + (u ? u[3 * n + k] : 0.0) - cent[3 * a + k]) * inv_h);
    }
}

// d and the prescribed-DOF mask in the order of the aggregates' node lists, so that the
// per-iteration restriction reads them coalesced and without waiting for the node index
__global__ void permute_offsets_kernel(int32_t n_node, const int32_t* __restrict__ nodes, const float* __restrict__ d,
                                       float* __restrict__ dperm) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_node; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = nodes[i];
        for (int k = 0; k < 3; ++k) dperm[3 * i + k] = d[3 * n + k];
    }
}

__global__ void permute_mask_kernel(int32_t n_node, const int32_t* __restrict__ nodes,
                                    const uint8_t* __restrict__ fixed, uint8_t* __restrict__ fperm) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_node; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = nodes[i];
        for (int k = 0; k < 3; ++k) fperm[3 * i + k] = fixed[3 * n + k];
    }
}

// ---------------------------------------------------------------- E = Z^T A Z
// E = Z^T A Z, lower triangle only (the blocked Cholesky reads tiles (i, j) with i >= j and the
// lower half of the diagonal tiles): for aggregate a the blocks E[a][b] with b < a (neighbour
// slots 0..12 of the 3x3x3 box stencil, z slowest) and the lower half of E[a][a] (slot 13).
// Two kernels, no atomics, every sum in a fixed order, so E is bitwise the same on every run:
//   1. one thread per matrix row n, in SELL order (coalesced like the SpMV): the row's blocks
//      are summed per neighbour box, T_{n,b} = sum_{m in b} A_nm Z_m (3 x NM), and stored as the
//      node's entries: T_{n,a} for its own box, then one per lower neighbour box its row reaches
//      (slot order);
//   2. one CTA per (aggregate, slot): E[a][b] = sum_n Z_n^T T_{n,b} over a fixed list of the
//      aggregate's nodes (node-list order), each thread one output value over a contiguous part
//      of the list, the parts added in order.
// Rigid-body modes: Z_n = [I | R(d_n)] with R(d) = [[-dy, 0, dz], [dx, -dz, 0], [0, dy, -dx]]
// (translations, then rotations about z, x, y). Linear modes: u = a + B d, columns a_0..a_2
// then B_ck at 3 + 3c + k. Rows of prescribed DOFs are zero in Z.
constexpr int kRowThreads = 128;
constexpr int kSumThreads = 256;
constexpr int kSlots = 14;  // 13 lower neighbour slots and the own box

__device__ __forceinline__ int box_slot(int pb, int ax, int ay, int az) {
    const int dx = (pb & 1023) - ax, dy = ((pb >> 10) & 1023) - ay, dz = (pb >> 20) - az;
    if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) return -1;
    return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1);
}

// The lower neighbour slots every row reaches (the pattern and the boxes only: computed once per
// layout). err = 1: a row reaches a box that is not a neighbour of its own.
__global__ void row_slots_kernel(SellView A, const int32_t* __restrict__ aggbox, uint16_t* __restrict__ lmask,
                                 int32_t* __restrict__ err) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < A.n_node;
         n += (int64_t)gridDim.x * blockDim.x) {
        const int64_t sl = n >> 5;
        const int lane = (int)(n & 31);
        const int64_t base = A.slice_base[sl];
        const int w = A.slice_width[sl];
        const int pn = aggbox[n];
        const int ax = pn & 1023, ay = (pn >> 10) & 1023, az = pn >> 20;
        uint32_t mask = 0;
        for (int k = 0; k < w; ++k) {
            const int slot = box_slot(aggbox[A.col[base + 32 * (int64_t)k + lane]], ax, ay, az);
            if (slot < 0)
                atomicExch(err, 1);
            else if (slot < 13)
                mask |= 1u << slot;
        }
        lmask[n] = (uint16_t)mask;
    }
}

// T += A_nm Z_m for one 3x3 block (column masks of m's prescribed DOFs applied)
template <int NM>
__device__ __forceinline__ void add_block_z(double (&T)[3][NM], const double blk[9], const float* __restrict__ d,
                                            const uint8_t* __restrict__ fixed, int64_t m) {
    const double dmx = d[3 * m], dmy = d[3 * m + 1], dmz = d[3 * m + 2];
    const double km0 = fixed[3 * m] ? 0.0 : 1.0, km1 = fixed[3 * m + 1] ? 0.0 : 1.0, km2 = fixed[3 * m + 2] ? 0.0 : 1.0;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const double c0 = km0 * blk[3 * r], c1 = km1 * blk[3 * r + 1], c2 = km2 * blk[3 * r + 2];
        T[r][0] += c0;
        T[r][1] += c1;
        T[r][2] += c2;
        if constexpr (NM == 6) {
            T[r][3] += -dmy * c0 + dmx * c1;
            T[r][4] += -dmz * c1 + dmy * c2;
            T[r][5] += dmz * c0 - dmx * c2;
        } else {
            const double dm[3] = {dmx, dmy, dmz};
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                T[r][3 + k] += c0 * dm[k];
                T[r][6 + k] += c1 * dm[k];
                T[r][9 + k] += c2 * dm[k];
            }
        }
    }
}

// Kernel 1: row n's entries (3 x NM each, row-major) at tbuf[toff[n] ..]: own box first, then
// the lower slots of lmask[n] in slot order. Rigid-body modes sum the own box and the first
// lower slot in one walk of the row; every further slot (rows at box edges and corners) walks
// the row again. The FP32 storage's diagonal block is minus the row's stored blocks, summed in
// storage order as the SpMV forms it.
template <typename VT, int NM>
__global__ void __launch_bounds__(kRowThreads, 4) coarse_rows_kernel(SellView A, const VT* __restrict__ aval, CoarseView cv,
                                                                  const int32_t* __restrict__ aggbox,
                                                                  const uint16_t* __restrict__ lmask,
                                                                  const int32_t* __restrict__ toff,
                                                                  double* __restrict__ tbuf) {
    constexpr bool kDual = NM == 6;
    const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (n >= A.n_node) return;
    const int64_t sl = n >> 5;
    const int lane = (int)(n & 31);
    const int64_t base = A.slice_base[sl];
    const int w = A.slice_width[sl];
    const int32_t* cp = A.col + base + lane;
    const VT* vp = aval + 9 * base + lane;
    const int pn = aggbox[n];
    const int ax = pn & 1023, ay = (pn >> 10) & 1023, az = pn >> 20;
    uint32_t todo = lmask[n];
    double* out = tbuf + (int64_t)toff[n] * (3 * NM);
    int want = 13, want2 = -1;
    if (kDual && todo) {
        want2 = __ffs(todo) - 1;
        todo &= todo - 1;
    }
    for (bool first = true;; first = false) {
        double T[3][NM], U[3][NM];  // U: the second slot of a rigid-body walk
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int j = 0; j < NM; ++j) {
                T[r][j] = 0.0;
                U[r][j] = 0.0;
            }
        double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = 0; k <= w; ++k) {
            double blk[9];
            int64_t m;
            if (k < w) {
                m = cp[32 * (int64_t)k];
                const VT* v = vp + 288 * (int64_t)k;
                bool any = false;
#pragma unroll
                for (int q = 0; q < 9; ++q) {
                    blk[q] = (double)v[32 * q];
                    S[q] += blk[q];
                    any |= blk[q] != 0.0;
                }
                if (!any) continue;  // SELL padding, zero blocks
            } else {
                if (!first || !A.diag64) break;  // the diagonal block belongs to the own box
                m = n;
#pragma unroll
                for (int q = 0; q < 9; ++q) blk[q] = -S[q];
            }
            const int slot = box_slot(aggbox[m], ax, ay, az);
            if (slot == want) {
                add_block_z<NM>(T, blk, cv.d, cv.fixed, m);
            } else if constexpr (kDual) {
                if (slot == want2) add_block_z<NM>(U, blk, cv.d, cv.fixed, m);
            }
        }
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int j = 0; j < NM; ++j) out[NM * r + j] = T[r][j];
        out += 3 * NM;
        if (want2 >= 0) {
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int j = 0; j < NM; ++j) out[NM * r + j] = U[r][j];
            out += 3 * NM;
        }
        if (!todo) break;
        want = __ffs(todo) - 1;
        todo &= todo - 1;
        want2 = -1;
    }
}

// Kernel 2, rigid-body modes: one CTA per (aggregate a, slot s); list[lptr[a 14 + s] ..) holds
// the entries of the nodes of a that reach slot s (node-list order) and their nodes. Each thread
// takes every kSumRigidThreads-th list item and adds its whole block Z_n^T T_{n,b} (36 values)
// in registers; the block is then summed over the CTA (butterfly per warp, warps in order).
constexpr int kSumRigidThreads = 128;
__global__ void __launch_bounds__(kSumRigidThreads) coarse_sum_rigid_kernel(CoarseView cv, int ngx, int ngy,
                                                                            const int64_t* __restrict__ lptr,
                                                                            const int32_t* __restrict__ lent,
                                                                            const int32_t* __restrict__ lnode,
                                                                            const double* __restrict__ tbuf,
                                                                            double* __restrict__ E) {
    __shared__ double red[kSumRigidThreads / 32][36];
    const int a = blockIdx.x / kSlots, s = blockIdx.x % kSlots;
    const int64_t b0 = lptr[blockIdx.x], b1 = lptr[blockIdx.x + 1];
    if (b0 == b1) return;
    double acc[36];
#pragma unroll
    for (int v = 0; v < 36; ++v) acc[v] = 0.0;
    for (int64_t q = b0 + threadIdx.x; q < b1; q += kSumRigidThreads) {
        const int64_t n = lnode[q];
        const double2* t2 = reinterpret_cast<const double2*>(tbuf + 18 * (int64_t)lent[q]);
        double T[18];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const double2 v = t2[k];
            T[2 * k] = v.x;
            T[2 * k + 1] = v.y;
        }
        const double dx = cv.d[3 * n], dy = cv.d[3 * n + 1], dz = cv.d[3 * n + 2];
        const double k0 = cv.fixed[3 * n] ? 0.0 : 1.0, k1 = cv.fixed[3 * n + 1] ? 0.0 : 1.0,
                     k2 = cv.fixed[3 * n + 2] ? 0.0 : 1.0;
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const double t0 = k0 * T[j], t1 = k1 * T[6 + j], t2v = k2 * T[12 + j];
            acc[j] += t0;
            acc[6 + j] += t1;
            acc[12 + j] += t2v;
            acc[18 + j] += -dy * t0 + dx * t1;
            acc[24 + j] += -dz * t1 + dy * t2v;
            acc[30 + j] += dz * t0 - dx * t2v;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < 36; ++v) {
        double x = acc[v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp][v] = x;
    }
    __syncthreads();
    if (threadIdx.x >= 36) return;
    const int i = threadIdx.x / 6, j = threadIdx.x % 6;
    const bool own = s == 13;
    if (own && j > i) return;  // E's lower triangle
    double x = 0.0;
#pragma unroll
    for (int w = 0; w < kSumRigidThreads / 32; ++w) x += red[w][threadIdx.x];
    const int ax = a % ngx, ay = (a / ngx) % ngy, az = a / (ngx * ngy);
    const int b = own ? a : (ax + s % 3 - 1) + ngx * ((ay + (s / 3) % 3 - 1) + ngy * (az + s / 9 - 1));
    E[(int64_t)(6 * a + i) * cv.kp + 6 * b + j] = x;
}

// Kernel 2, linear modes (144 values per block, too many for registers): thread (g, v) sums
// output value v over part g of the list; the parts are added in order.
template <int NM>
__global__ void __launch_bounds__(kSumThreads) coarse_sum_kernel(CoarseView cv, int ngx, int ngy,
                                                                 const int64_t* __restrict__ lptr,
                                                                 const int32_t* __restrict__ lent,
                                                                 const int32_t* __restrict__ lnode,
                                                                 const double* __restrict__ tbuf,
                                                                 double* __restrict__ E) {
    __shared__ double part[kSumThreads];
    const int a = blockIdx.x / kSlots, s = blockIdx.x % kSlots;
    const int64_t b0 = lptr[blockIdx.x], len = lptr[blockIdx.x + 1] - b0;
    if (len == 0) return;
    const bool own = s == 13;
    const int nval = own ? NM * (NM + 1) / 2 : NM * NM;
    const int groups = kSumThreads / nval;
    const int v = threadIdx.x % nval, g = threadIdx.x / nval;
    int i, j;
    if (own) {
        i = 0;
        while ((i + 1) * (i + 2) / 2 <= v) ++i;
        j = v - i * (i + 1) / 2;
    } else {
        i = v / NM;
        j = v % NM;
    }
    double acc = 0.0;
    if (g < groups) {
        // (Z_n^T T)[i][j] = c1 T[r1][j] + c2 T[r2][j]
        int r1 = i, r2 = 0, dk1 = -1, dk2 = -1;
        double s1 = 1.0, s2 = 0.0;
        if (NM == 6) {
            // i = 3: -dy T0 + dx T1; i = 4: -dz T1 + dy T2; i = 5: dz T0 - dx T2
            if (i >= 3) {
                r1 = i == 4 ? 1 : 0;
                r2 = i == 3 ? 1 : 2;
                dk1 = i == 3 ? 1 : 2;
                dk2 = i == 4 ? 1 : 0;
                s1 = i == 5 ? 1.0 : -1.0;
                s2 = -s1;
            }
        } else if (i >= 3) {
            r1 = (i - 3) / 3;
            dk1 = (i - 3) % 3;
        }
        const int64_t lo = b0 + len * g / groups, hi = b0 + len * (g + 1) / groups;
        for (int64_t q = lo; q < hi; ++q) {
            const int64_t n = lnode[q];
            const double* t = tbuf + (int64_t)lent[q] * (3 * NM);
            double c1 = cv.fixed[3 * n + r1] ? 0.0 : s1;
            if (dk1 >= 0) c1 *= (double)cv.d[3 * n + dk1];
            double x = c1 * t[NM * r1 + j];
            if (dk2 >= 0) {
                const double c2 = cv.fixed[3 * n + r2] ? 0.0 : s2 * (double)cv.d[3 * n + dk2];
                x += c2 * t[NM * r2 + j];
            }
            acc += x;
        }
    }
    part[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x >= nval) return;
    double x = 0.0;
    for (int q = 0; q < groups; ++q) x += part[q * nval + v];
    const int ax = a % ngx, ay = (a / ngx) % ngy, az = a / (ngx * ngy);
    const int b = own ? a : (ax + s % 3 - 1) + ngx * ((ay + (s / 3) % 3 - 1) + ngy * (az + s / 9 - 1));
    E[(int64_t)(NM * a + i) * cv.kp + NM * b + j] = x;
}

__global__ void drop_null_modes(double* __restrict__ E, int kp, int k) {
    __shared__ double red[32];
    // largest diagonal entry: per-thread maxima, then per warp and across warps
    double m = 0.0;
    for (int j = threadIdx.x; j < k; j += blockDim.x) m = fmax(m, fabs(E[(int64_t)j * kp + j]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) red[0] = m;
    }
    __syncthreads();
    const double mx = red[0];
    for (int j = threadIdx.x; j < kp; j += blockDim.x) {
        const bool drop = j >= k || !(E[(int64_t)j * kp + j] > 1e-13 * mx);
        if (!drop) continue;
        for (int i = 0; i < kp; ++i) {
            E[(int64_t)j * kp + i] = 0.0;
            E[(int64_t)i * kp + j] = 0.0;
        }
    }
    __syncthreads();
    for (int j = threadIdx.x; j < kp; j += blockDim.x)
        if (E[(int64_t)j * kp + j] == 0.0) E[(int64_t)j * kp + j] = 1.0;
}

// ---------------------------------------------------------------- dense Cholesky + inverse
__device__ __forceinline__ void load_tile(double (*S)[TP], const double* M, int kp, int ti, int tj) {
    for (int t = threadIdx.x; t < T * T; t += blockDim.x) S[t / T][t % T] = M[(int64_t)(ti * T + t / T) * kp + tj * T + t % T];
}

// Factor the diagonal tile (j, j) in place (lower triangle; upper zeroed), and write its inverse
// W_jj = L_jj^{-1} to W: the panel below becomes a tile product with W_jj (gemm_panel_tiles) and
// the triangular inverse reuses W_jj. The tile's lower triangle is cut into 4x4 patches, one per
// thread (136 patches), held in registers for the whole kernel with every patch index known at
// compile time.
//   Cholesky: right-looking over the 16 patch columns (blocked by 4), two barriers per step.
//   Inverse: L and the patches' inverses go to shared memory (dynamic, two padded tiles), and
//   X = L^{-1} is formed by recursive doubling (four levels, below).
constexpr int kPotrfPatches = (T / 4) * (T / 4 + 1) / 2;  // 136
constexpr int kPotrfThreads = 160;                          // five warps, the last 24 threads idle

__global__ void __launch_bounds__(kPotrfThreads) potrf_inv_tile(double* E, double* W, int kp, int j, int32_t* err) {
    __shared__ double pinv[4][4];      // inverse of the current step's diagonal patch
    __shared__ double panel[2][T][4];  // the current step's L_Pc, double-buffered
    __shared__ double rd[T];           // 1 / L(c, c)
    const int tid = threadIdx.x;
    const bool owner = tid < kPotrfPatches;
    // patch (P, Q), Q <= P, from the row-major triangular index
    int P = (int)((sqrtf(8.0f * (float)tid + 1.0f) - 1.0f) * 0.5f);
    while (P * (P + 1) / 2 > tid) --P;  // the float root, made exact
    while ((P + 1) * (P + 2) / 2 <= tid) ++P;
    const int Q = owner ? tid - P * (P + 1) / 2 : -1;
    if (!owner) P = -1;
    const int r0 = 4 * P, c0 = 4 * Q;
    double A[4][4];
    const double* Et = E + (int64_t)(j * T) * kp + j * T;
    if (owner) {
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const double2* row = reinterpret_cast<const double2*>(Et + (int64_t)(r0 + a) * kp + c0);
            const double2 v0 = row[0], v1 = row[1];
            A[a][0] = v0.x;
            A[a][1] = v0.y;
            A[a][2] = v1.x;
            A[a][3] = v1.y;
        }
    }
    // ---- Cholesky, right-looking in steps of one patch column cq (16 steps, two barriers each):
    // the owner of the diagonal patch factors it in registers and publishes its inverse; the
    // owners of the patches below form L_Pc = A_Pc L_cc^{-T} and publish them; every patch
    // (P, Q) with P >= Q > cq subtracts L_Pc L_Qc^T
    for (int cq = 0; cq < T / 4; ++cq) {
        const int buf = cq & 1;
        if (P == cq && Q == cq) {
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                double p = A[kk][kk];
                if (!(p > 0.0)) {
                    atomicExch(err, 2);
                    p = 1e-300;
                }
                const double il = rsqrt(p);
                rd[4 * cq + kk] = il;
#pragma unroll
                for (int a = 0; a < 4; ++a)
                    if (a >= kk) A[a][kk] *= il;
#pragma unroll
                for (int bb = 0; bb < 4; ++bb)
#pragma unroll
                    for (int a = 0; a < 4; ++a)
                        if (bb > kk && a >= bb) A[a][bb] = fma(-A[a][kk], A[bb][kk], A[a][bb]);
            }
            // the patch's inverse (forward substitution, 1 / L(i,i) = rd)
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const double di = rd[4 * cq + a];
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) {
                    double t = 0.0;
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (k >= bb && k < a) t = fma(A[a][k], pinv[k][bb], t);
                    pinv[a][bb] = bb < a ? -di * t : (bb == a ? di : 0.0);
                }
            }
        }
        __syncthreads();
        if (owner && Q == cq && P > cq) {
            double l[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) {
                    double t = 0.0;
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (k <= bb) t = fma(A[a][k], pinv[bb][k], t);  // (L_cc^{-T})[k][bb]
                    l[a][bb] = t;
                }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int bb = 0; bb < 4; ++bb) {
                    A[a][bb] = l[a][bb];
                    panel[buf][r0 + a][bb] = l[a][bb];
                }
        }
        __syncthreads();
        if (owner && Q > cq) {
            double lp[4][4], lq[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    lp[a][k] = panel[buf][r0 + a][k];
                    lq[a][k] = panel[buf][c0 + a][k];
                }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int bb = 0; bb < 4; ++bb)
#pragma unroll
                    for (int k = 0; k < 4; ++k) A[a][bb] = fma(-lp[a][k], lq[bb][k], A[a][bb]);
        }
    }
    // ---- inverse X = L^{-1} by recursive doubling over the 4x4 patches: the diagonal patches
    // first (forward substitution in registers, 1 / L(i,i) = rd[i]), then for half sizes of
    // 1, 2, 4, 8 patches every pair of diagonal blocks [A 0; C B] gets its lower block
    // X_BA = -X_B (L_BA X_A). Patch (P, Q), P > Q, belongs to the level of the highest bit in
    // which P and Q differ, so each owner works at one level; four barriers per level.
    extern __shared__ double dsm[];
    double (*Ls)[TP] = reinterpret_cast<double (*)[TP]>(dsm);
    double (*Xs)[TP] = reinterpret_cast<double (*)[TP]>(dsm + T * TP);
    __syncthreads();  // rd complete
    if (owner) {
        double x[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) x[a][b] = 0.0;
        if (P == Q) {
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const double di = rd[r0 + a];
                x[a][a] = di;
#pragma unroll
                for (int b = 0; b < a; ++b) {
                    double t = 0.0;
#pragma unroll
                    for (int k = b; k < a; ++k) t = fma(A[a][k], x[k][b], t);
                    x[a][b] = -di * t;
                }
            }
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                Ls[r0 + a][c0 + b] = c0 + b <= r0 + a ? A[a][b] : 0.0;
                Xs[r0 + a][c0 + b] = x[a][b];
            }
    }
    const int lvl = owner && P != Q ? 31 - __clz(P ^ Q) : -1;
    for (int lv = 0; lv < 4; ++lv) {
        const bool act = lvl == lv;
        const int mid = 4 * (((P >> (lv + 1)) << (lv + 1)) + (1 << lv));  // first row of block B
        double t[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) t[a][b] = 0.0;
        __syncthreads();  // the previous level's X (and the patches above) are in Xs
        if (act) {
            // T = L_BA X_A over the rows of block A from this patch's column on (X_A is lower)
            for (int k = c0; k < mid; ++k) {
                double l[4], xa[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) l[a] = Ls[r0 + a][k];
#pragma unroll
                for (int b = 0; b < 4; ++b) xa[b] = Xs[k][c0 + b];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) t[a][b] = fma(l[a], xa[b], t[a][b]);
            }
        }
        __syncthreads();
        if (act)
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) Xs[r0 + a][c0 + b] = t[a][b];  // T in X_BA's place
        __syncthreads();
        if (act) {
            // X_BA = -X_B T over the rows of block B up to this patch's last row (X_B is lower)
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) t[a][b] = 0.0;
            for (int k = mid; k < r0 + 4; ++k) {
                double xb[4], tt[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) xb[a] = Xs[r0 + a][k];
#pragma unroll
                for (int b = 0; b < 4; ++b) tt[b] = Xs[k][c0 + b];
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) t[a][b] = fma(-xb[a], tt[b], t[a][b]);
            }
        }
        __syncthreads();
        if (act)
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) Xs[r0 + a][c0 + b] = t[a][b];
    }
    __syncthreads();
    if (!owner) return;
    double* Eo = E + (int64_t)(j * T) * kp + j * T;
    double* Wo = W + (int64_t)(j * T) * kp + j * T;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        double l[4], x[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const bool lower = c0 + b <= r0 + a;
            l[b] = lower ? A[a][b] : 0.0;
            x[b] = lower ? Xs[r0 + a][c0 + b] : 0.0;
        }
        double2* er = reinterpret_cast<double2*>(Eo + (int64_t)(r0 + a) * kp + c0);
        double2* wr = reinterpret_cast<double2*>(Wo + (int64_t)(r0 + a) * kp + c0);
        er[0] = make_double2(l[0], l[1]);
        er[1] = make_double2(l[2], l[3]);
        wr[0] = make_double2(x[0], x[1]);
        wr[1] = make_double2(x[2], x[3]);
        if (P != Q) {
            // the mirrored upper patch (Q, P) is zero in both
            double2* eu = reinterpret_cast<double2*>(Eo + (int64_t)(c0 + a) * kp + r0);
            double2* wu = reinterpret_cast<double2*>(Wo + (int64_t)(c0 + a) * kp + r0);
            eu[0] = eu[1] = wu[0] = wu[1] = make_double2(0.0, 0.0);
        }
    }
}

// C (tile ci, cj of M) += alpha * sum_t A[r][t] * B[c][t]  with A, B 64x64 tiles in shared memory
__device__ __forceinline__ void tile_abt(const double (*A)[TP], const double (*B)[TP], double acc[4][4]) {
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
    for (int t = 0; t < T; ++t) {
        double a[4], b[4];
        for (int q = 0; q < 4; ++q) {
            a[q] = A[ty + 16 * q][t];
            b[q] = B[tx + 16 * q][t];
        }
        for (int q = 0; q < 4; ++q)
            for (int r = 0; r < 4; ++r) acc[q][r] += a[q] * b[r];
    }
}

// trailing update A_ik -= L_ij L_kj^T of step j. col_only: the tile column k = j + 1 (one CTA
// per tile i > j), which the next diagonal factorisation and panel need first; otherwise the
// rest, j + 2 <= k <= i (one CTA per tile of that triangle).
__global__ void __launch_bounds__(256) syrk_tiles(double* E, int kp, int j, int col_only) {
    extern __shared__ double sm[];
    double (*Li)[TP] = reinterpret_cast<double (*)[TP]>(sm);
    double (*Lk)[TP] = reinterpret_cast<double (*)[TP]>(sm + T * TP);
    int i, k;
    if (col_only) {
        i = j + 1 + (int)blockIdx.x;
        k = j + 1;
    } else {
        const int idx = blockIdx.x;
        const int ii = (int)((sqrt(8.0 * idx + 1.0) - 1.0) / 2.0);
        int a = ii, b = idx - ii * (ii + 1) / 2;
        if (b > a) { ++a; b = idx - a * (a + 1) / 2; }  // guard the float square root
        if (b < 0) { --a; b = idx - a * (a + 1) / 2; }
        i = j + 2 + a;
        k = j + 2 + b;
    }
    load_tile(Li, E, kp, i, j);
    load_tile(Lk, E, kp, k, j);
    __syncthreads();
    double acc[4][4] = {{0}};
    tile_abt(Li, Lk, acc);
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
    for (int q = 0; q < 4; ++q)
        for (int r = 0; r < 4; ++r) E[(int64_t)(i * T + ty + 16 * q) * kp + k * T + tx + 16 * r] -= acc[q][r];
}

// tiles below the diagonal as tile products: L_ij = A_ij L_jj^{-T} = A_ij W_jj^T
__global__ void __launch_bounds__(256) gemm_panel_tiles(double* E, const double* W, int kp, int j) {
    extern __shared__ double sm[];
    double (*A)[TP] = reinterpret_cast<double (*)[TP]>(sm);
    double (*B)[TP] = reinterpret_cast<double (*)[TP]>(sm + T * TP);
    const int i = j + 1 + blockIdx.x;
    load_tile(A, E, kp, i, j);
    load_tile(B, W, kp, j, j);
    __syncthreads();
    double acc[4][4] = {{0}};
    tile_abt(A, B, acc);  // sum_t A_ij[r][t] W_jj[c][t]
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
    for (int q = 0; q < 4; ++q)
        for (int r = 0; r < 4; ++r) E[(int64_t)(i * T + ty + 16 * q) * kp + j * T + tx + 16 * r] = acc[q][r];
}

// Right-looking W = L^{-1}: the strictly lower tiles of W first accumulate
// S_ij = sum_{k < i} L_ik W_kj; once tile row i is complete, W_ij = -W_ii S_ij. Step k finalises
// tile row k (k CTAs, one tile product each) and adds L_ik W_kj to every S_ij with i > k, j <= k
// (one CTA per tile, all independent), so no CTA runs a chain of products.
__global__ void __launch_bounds__(256) trtri_finalize(double* W, int kp, int k) {
    extern __shared__ double sm[];
    double (*A)[TP] = reinterpret_cast<double (*)[TP]>(sm);
    double (*B)[TP] = reinterpret_cast<double (*)[TP]>(sm + T * TP);
    const int j = blockIdx.x;
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
    load_tile(A, W, kp, k, k);  // W_kk
    for (int t = threadIdx.x; t < T * T; t += blockDim.x) B[t % T][t / T] = W[(int64_t)(k * T + t / T) * kp + j * T + t % T];
    __syncthreads();
    double acc[4][4] = {{0}};
    tile_abt(A, B, acc);  // W_kk S_kj
    for (int q = 0; q < 4; ++q)
        for (int r = 0; r < 4; ++r) W[(int64_t)(k * T + ty + 16 * q) * kp + j * T + tx + 16 * r] = -acc[q][r];
}

// rows: the tile rows i = k + 1 .. k + rows whose L_ik can be nonzero (E's band)
__global__ void __launch_bounds__(256) trtri_update(const double* E, double* W, int kp, int k, int rows) {
    extern __shared__ double sm[];
    double (*A)[TP] = reinterpret_cast<double (*)[TP]>(sm);
    double (*B)[TP] = reinterpret_cast<double (*)[TP]>(sm + T * TP);
    const int i = k + 1 + (int)(blockIdx.x % rows), j = (int)(blockIdx.x / rows);
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
    load_tile(A, E, kp, i, k);  // L_ik
    for (int t = threadIdx.x; t < T * T; t += blockDim.x) B[t % T][t / T] = W[(int64_t)(k * T + t / T) * kp + j * T + t % T];
    __syncthreads();
    double acc[4][4] = {{0}};
    tile_abt(A, B, acc);  // L_ik W_kj
    for (int q = 0; q < 4; ++q)
        for (int r = 0; r < 4; ++r) W[(int64_t)(i * T + ty + 16 * q) * kp + j * T + tx + 16 * r] += acc[q][r];
}

// The lower tiles of W = L^{-1} rounded to FP32, packed (tile (i, j), j <= i, row-major at
// tile index i (i + 1) / 2 + j) for the per-iteration W~^T (W~ w)
__global__ void __launch_bounds__(256) pack_w32_tiles(const double* __restrict__ W, float* __restrict__ w32, int kp) {
    const int t = blockIdx.x;
    int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while (i * (i + 1) / 2 > t) --i;  // the float root, made exact
    while ((i + 1) * (i + 2) / 2 <= t) ++i;
    const int j = t - i * (i + 1) / 2;
    float* o = w32 + (int64_t)t * T * T;
    for (int q = threadIdx.x; q < T * T; q += blockDim.x)
        o[q] = (float)W[(int64_t)(i * T + q / T) * kp + j * T + q % T];
}

}  // namespace

void CoarseSpace::init(mphy_ctx* ctx, const mphy_mesh* mesh, const mphy_pattern* pat, int target, int modes) {
    MPHY_REQUIRE(modes == 6 || modes == 12, MPHY_ERR_INVALID_ARG,
                 "coarse space: 6 (rigid-body) or 12 (linear) modes per aggregate");
    nm_ = modes;
    if (fact_graph_) {  // a new layout: the recorded factorisation refers to the old buffers
        MPHY_CUDA(cudaGraphExecDestroy(fact_graph_));
        fact_graph_ = nullptr;
    }
    boxd_ = 0.0;
    ctx_ = ctx;
    mesh_ = mesh;
    pat_ = pat;
    const int32_t nn = mesh->n_node;
    const std::vector<double>& X = mesh->coords_host;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int32_t n = 0; n < nn; ++n)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], X[3 * n + d]);
            hi[d] = std::max(hi[d], X[3 * n + d]);
        }
    double L[3], vol = 1.0;
    for (int d = 0; d < 3; ++d) {
        L[d] = std::max(hi[d] - lo[d], 1e-30);
        vol *= L[d];
    }
    // boxes as close to cubes as the bounding box allows, never thinner than ~2 elements
    const double h = std::cbrt(vol / std::max(target, 1));
    const double helem = std::cbrt(vol / std::max(mesh->n_elem, 1)) * 2.0;
    for (int d = 0; d < 3; ++d) {
        int g = (int)std::lround(L[d] / h);
        g = std::max(1, std::min(g, (int)(L[d] / helem)));
        ng_[d] = std::max(g, 1);
    }
    n_agg_ = ng_[0] * ng_[1] * ng_[2];
    kp_ = ((nm_ * n_agg_ + T - 1) / T) * T;
    // numbering: the axis with the most boxes varies slowest, so that E = Z^T A Z has the
    // narrowest band (neighbour boxes are at most 1 + n0 + n0 n1 apart in index). E's Cholesky
    // factor fills only inside that band, and the factorisation skips the tiles outside it.
    std::array<int, 3> ord = {0, 1, 2};
    std::stable_sort(ord.begin(), ord.end(), [&](int p, int q) { return ng_[p] < ng_[q]; });
    for (int k = 0; k < 3; ++k) ngl_[k] = ng_[ord[k]];
    {
        const int64_t reach = 1 + ngl_[0] + (int64_t)ngl_[0] * ngl_[1];
        const int64_t rows = reach * nm_ + nm_ - 1;  // largest row - column distance inside the band
        band_tiles_ = (int)std::min<int64_t>(kp_ / T - 1, (rows + T - 1) / T);
    }
    MPHY_REQUIRE(kp_ <= 16384, MPHY_ERR_UNSUPPORTED, "coarse space larger than 16384");
    std::vector<int32_t> agg(nn), cnt(n_agg_, 0);
    for (int32_t n = 0; n < nn; ++n) {
        int c[3];
        for (int d = 0; d < 3; ++d) c[d] = std::min(ng_[d] - 1, (int)((X[3 * n + d] - lo[d]) / L[d] * ng_[d]));
        agg[n] = c[ord[0]] + ngl_[0] * (c[ord[1]] + ngl_[1] * c[ord[2]]);
        ++cnt[agg[n]];
    }
    std::vector<int64_t> ptr(n_agg_ + 1, 0);
    for (int a = 0; a < n_agg_; ++a) ptr[a + 1] = ptr[a] + cnt[a];
    std::vector<int32_t> nodes(nn);
    std::vector<int64_t> cur(ptr.begin(), ptr.end() - 1);
    for (int32_t n = 0; n < nn; ++n) nodes[cur[agg[n]]++] = n;
    lists_ready_ = false;
    cudaStream_t s = ctx->stream;
    agg_.alloc(nn);
    agg_.upload(agg.data(), nn, s);
    // every node's aggregate box (bx, by, bz) packed in 10 bits each, for the E kernel
    MPHY_REQUIRE(ng_[0] <= 1024 && ng_[1] <= 1024 && ng_[2] <= 1024, MPHY_ERR_UNSUPPORTED,
                 "coarse space: more than 1024 aggregates along one axis");
    {
        std::vector<int32_t> box(nn);
        for (int32_t n = 0; n < nn; ++n) {
            const int a = agg[n];
            box[n] = (a % ngl_[0]) | (((a / ngl_[0]) % ngl_[1]) << 10) | ((a / (ngl_[0] * ngl_[1])) << 20);
        }
        aggbox_.alloc(nn);
        aggbox_.upload(box.data(), nn, s);
        MPHY_CUDA(cudaStreamSynchronize(s));  // box lives on the host stack until the copy ends
    }
    agg_ptr_.alloc(n_agg_ + 1);
    agg_ptr_.upload(ptr.data(), n_agg_ + 1, s);
    agg_nodes_.alloc(nn);
    agg_nodes_.upload(nodes.data(), nn, s);
    nodes_host_ = std::move(nodes);
    ptr_host_ = ptr;
    d_.alloc(3 * (size_t)nn);
    dperm_.alloc(3 * (size_t)nn);
    fperm_.alloc(3 * (size_t)nn);
    permute_mask_kernel<<<stride_grid(nn, 256, ctx->sm_count), 256, 0, s>>>(nn, agg_nodes_.p, mesh->fixed.p, fperm_.p);
    MPHY_CUDA(cudaGetLastError());
    cent_.alloc(3 * (size_t)n_agg_);
    E_.alloc((size_t)kp_ * kp_);
    W_.alloc((size_t)kp_ * kp_);
    const int nb = kp_ / T;
    const size_t tiles = (size_t)nb * (nb + 1) / 2;
    w32_.alloc(tiles * T * T);
    y_.alloc(kp_);
    gpart_.alloc(tiles * 2 * T);
    rowyy_.alloc(nb);
    w_.alloc(kp_);
    c_.alloc(kp_);
    wpart_.alloc((size_t)n_agg_ * kMaxRestrictParts * nm_);
    wcount_.alloc(n_agg_);
    err_.alloc(1);
    MPHY_CUDA(cudaMemsetAsync(w_.p, 0, w_.bytes(), s));
    MPHY_CUDA(cudaMemsetAsync(c_.p, 0, c_.bytes(), s));
    MPHY_CUDA(cudaMemsetAsync(wcount_.p, 0, wcount_.bytes(), s));
    MPHY_CUDA(cudaStreamSynchronize(s));
}

template <typename VT>
void CoarseSpace::setup(const SellView& A, const VT* aval, const double* disp, cudaStream_t s) {
    MPHY_CUDA(cudaEventRecord(ctx_->ev0, s));
    const int sm = ctx_->sm_count;
    launches = 0;
    centroid_kernel<<<std::min(n_agg_, sm * 8), 256, 0, s>>>(n_agg_, agg_ptr_.p, agg_nodes_.p, mesh_->coords.p, disp,
                                                             cent_.p);
    if (!(boxd_ > 0.0)) {
        // box diagonal of the reference grid: scales the rotation modes to O(1) (the reference
        // coordinates do not change, so it is computed once)
        const std::vector<double>& X = mesh_->coords_host;
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (size_t n = 0; n < X.size() / 3; ++n)
            for (int d = 0; d < 3; ++d) {
                lo[d] = std::min(lo[d], X[3 * n + d]);
                hi[d] = std::max(hi[d], X[3 * n + d]);
            }
        double b = 0.0;
        for (int d = 0; d < 3; ++d) b += std::pow((hi[d] - lo[d]) / ng_[d], 2);
        boxd_ = std::sqrt(std::max(b, 1e-300));
    }
    offsets_kernel<<<stride_grid(mesh_->n_node, 256, sm), 256, 0, s>>>(mesh_->n_node, agg_.p, mesh_->coords.p, disp,
                                                                      cent_.p, 1.0 / boxd_, d_.p);
    permute_offsets_kernel<<<stride_grid(mesh_->n_node, 256, sm), 256, 0, s>>>(mesh_->n_node, agg_nodes_.p, d_.p,
                                                                              dperm_.p);
    MPHY_CUDA(cudaMemsetAsync(E_.p, 0, E_.bytes(), s));
    MPHY_CUDA(cudaMemsetAsync(W_.p, 0, W_.bytes(), s));
    MPHY_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int32_t), s));
    if (!lists_ready_) build_entry_lists(A, s);
    CoarseView cv = view();
    const unsigned rows = (unsigned)((mesh_->n_node + kRowThreads - 1) / kRowThreads);
    if (nm_ == 12) {
        coarse_rows_kernel<VT, 12><<<rows, kRowThreads, 0, s>>>(A, aval, cv, aggbox_.p, lmask_.p, toff_.p, tbuf_.p);
        coarse_sum_kernel<12><<<n_agg_ * kSlots, kSumThreads, 0, s>>>(cv, ngl_[0], ngl_[1], lptr_.p, lent_.p, lnode_.p,
                                                                      tbuf_.p, E_.p);
    } else {
        coarse_rows_kernel<VT, 6><<<rows, kRowThreads, 0, s>>>(A, aval, cv, aggbox_.p, lmask_.p, toff_.p, tbuf_.p);
        coarse_sum_rigid_kernel<<<n_agg_ * kSlots, kSumRigidThreads, 0, s>>>(cv, ngl_[0], ngl_[1], lptr_.p, lent_.p,
                                                                             lnode_.p, tbuf_.p, E_.p);
    }
    MPHY_CUDA(cudaGetLastError());
    launches += 4;
    const int nb = kp_ / T;
    const size_t sm2 = 2 * (size_t)T * TP * sizeof(double);
    static std::atomic<uint64_t> attr{0};
    if (first_use_on_device(attr)) {
        MPHY_CUDA(cudaFuncSetAttribute(syrk_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
        MPHY_CUDA(cudaFuncSetAttribute(gemm_panel_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
        MPHY_CUDA(cudaFuncSetAttribute(trtri_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
        MPHY_CUDA(cudaFuncSetAttribute(trtri_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
        MPHY_CUDA(cudaFuncSetAttribute(potrf_inv_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
    }
    // The dense part (null modes, blocked Cholesky with tile inverses, triangular inverse,
    // W in FP32) is the same launch sequence on the same buffers every time: it is captured
    // once into a CUDA graph and replayed, so the short dependent launches run back to back.
    if (fact_graph_) {
        MPHY_CUDA(cudaGraphLaunch(fact_graph_, s));
        launches += fact_launches_;
    } else {
        const int64_t l0 = launches;
        cudaGraph_t g = nullptr;
        MPHY_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
            record_factorisation(s, nb, sm2);
        } catch (...) {
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        MPHY_CUDA(cudaStreamEndCapture(s, &g));
        const cudaError_t e = cudaGraphInstantiate(&fact_graph_, g, 0);
        cudaGraphDestroy(g);
        MPHY_CUDA(e);
        fact_launches_ = launches - l0;
        MPHY_CUDA(cudaGraphLaunch(fact_graph_, s));
    }
    MPHY_CUDA(cudaGetLastError());
    MPHY_CUDA(cudaEventRecord(ctx_->ev1, s));
    int32_t h = 0;
    MPHY_CUDA(cudaMemcpyAsync(&h, err_.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    MPHY_CUDA(cudaStreamSynchronize(s));
    cudaEventElapsedTime(&last_setup_ms, ctx_->ev0, ctx_->ev1);
    MPHY_REQUIRE(h != 2, MPHY_ERR_INDEFINITE, "coarse space: Z^T A Z is not positive definite");
}

// The lower slots of every row (device), then on the host the entry offsets and the
// per-(aggregate, slot) lists in node-list order. Once per layout: the pattern and the boxes
// decide them, not the values.
void CoarseSpace::build_entry_lists(const SellView& A, cudaStream_t s) {
    const int32_t nn = mesh_->n_node;
    lmask_.alloc(nn);
    MPHY_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int32_t), s));
    row_slots_kernel<<<stride_grid(nn, 256, ctx_->sm_count), 256, 0, s>>>(A, aggbox_.p, lmask_.p, err_.p);
    MPHY_CUDA(cudaGetLastError());
    std::vector<uint16_t> mask(nn);
    int32_t h = 0;
    MPHY_CUDA(cudaMemcpyAsync(mask.data(), lmask_.p, nn * sizeof(uint16_t), cudaMemcpyDeviceToHost, s));
    MPHY_CUDA(cudaMemcpyAsync(&h, err_.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    MPHY_CUDA(cudaStreamSynchronize(s));
    MPHY_REQUIRE(h == 0, MPHY_ERR_UNSUPPORTED, "coarse space: an element spans more than two aggregates");
    std::vector<int32_t> toff(nn);
    int64_t entries = 0;
    for (int32_t n = 0; n < nn; ++n) {
        toff[n] = (int32_t)entries;
        entries += 1 + __builtin_popcount(mask[n]);
        MPHY_REQUIRE(entries < INT32_MAX, MPHY_ERR_UNSUPPORTED, "coarse space: too many row entries");
    }
    std::vector<int64_t> lptr((size_t)n_agg_ * kSlots + 1, 0);
    std::vector<int32_t> lent, lnode;
    lent.reserve(entries);
    lnode.reserve(entries);
    for (int a = 0; a < n_agg_; ++a)
        for (int sl = 0; sl < kSlots; ++sl) {
            for (int64_t i = ptr_host_[a]; i < ptr_host_[a + 1]; ++i) {
                const int32_t n = nodes_host_[i];
                const uint32_t m = mask[n];
                if (sl == 13) {
                    lent.push_back(toff[n]);
                } else if (m >> sl & 1u) {
                    lent.push_back(toff[n] + 1 + __builtin_popcount(m & ((1u << sl) - 1u)));
                } else {
                    continue;
                }
                lnode.push_back(n);
            }
            lptr[(size_t)a * kSlots + sl + 1] = (int64_t)lent.size();
        }
    toff_.alloc(nn);
    toff_.upload(toff.data(), nn, s);
    lptr_.alloc(lptr.size());
    lptr_.upload(lptr.data(), lptr.size(), s);
    lent_.alloc(lent.size());
    lent_.upload(lent.data(), lent.size(), s);
    lnode_.alloc(lnode.size());
    lnode_.upload(lnode.data(), lnode.size(), s);
    tbuf_.alloc((size_t)entries * 3 * nm_);
    MPHY_CUDA(cudaStreamSynchronize(s));  // the host vectors end here
    lists_ready_ = true;
}

// Three streams inside the capture. Main: the diagonal factorisation and the panel of step j,
// then the update of tile column j + 1 (after the previous step's remaining update), so the next
// diagonal tile is ready as early as possible. Side 1: the rest of step j's trailing update.
// Side 2: the triangular inverse, step j as soon as column j of L and W_jj are final. Every
// tile is written by one stream at a time, in step order.
void CoarseSpace::record_factorisation(cudaStream_t s, int nb, size_t sm2) {
    if (!side_[0]) {
        for (auto& q : side_) MPHY_CUDA(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
        for (auto& e : ev_) MPHY_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    cudaStream_t s_rest = side_[0], s_tri = side_[1];
    cudaEvent_t ev_col = ev_[0], ev_rest = ev_[1], ev_tri = ev_[2];
    drop_null_modes<<<1, 1024, 0, s>>>(E_.p, kp_, nm_ * n_agg_);
    launches += 1;
    MPHY_CUDA(cudaEventRecord(ev_col, s));
    MPHY_CUDA(cudaStreamWaitEvent(s_rest, ev_col, 0));
    MPHY_CUDA(cudaStreamWaitEvent(s_tri, ev_col, 0));
    bool rest_pending = false;
    for (int j = 0; j < nb; ++j) {
        const int m = std::min(nb - j - 1, band_tiles_);  // tiles below (j, j) inside E's band
        potrf_inv_tile<<<1, kPotrfThreads, sm2, s>>>(E_.p, W_.p, kp_, j, err_.p);
        launches += 1;
        if (m > 0) {
            gemm_panel_tiles<<<m, 256, sm2, s>>>(E_.p, W_.p, kp_, j);
            launches += 1;
        }
        MPHY_CUDA(cudaEventRecord(ev_col, s));  // column j of L and W_jj are final
        MPHY_CUDA(cudaStreamWaitEvent(s_tri, ev_col, 0));
        if (j > 0) {
            trtri_finalize<<<j, 256, sm2, s_tri>>>(W_.p, kp_, j);
            launches += 1;
        }
        if (m > 0) {
            trtri_update<<<m * (j + 1), 256, sm2, s_tri>>>(E_.p, W_.p, kp_, j, m);
            launches += 1;
            if (m > 1) {
                MPHY_CUDA(cudaStreamWaitEvent(s_rest, ev_col, 0));
                syrk_tiles<<<(m - 1) * m / 2, 256, sm2, s_rest>>>(E_.p, kp_, j, 0);
                launches += 1;
            }
            // step j - 1's remaining update also covered tile column j + 1
            if (rest_pending) MPHY_CUDA(cudaStreamWaitEvent(s, ev_rest, 0));
            syrk_tiles<<<m, 256, sm2, s>>>(E_.p, kp_, j, 1);
            launches += 1;
            rest_pending = m > 1;
            if (rest_pending) MPHY_CUDA(cudaEventRecord(ev_rest, s_rest));
        }
    }
    // join both side streams before W is rounded to FP32
    MPHY_CUDA(cudaEventRecord(ev_rest, s_rest));
    MPHY_CUDA(cudaStreamWaitEvent(s, ev_rest, 0));
    MPHY_CUDA(cudaEventRecord(ev_tri, s_tri));
    MPHY_CUDA(cudaStreamWaitEvent(s, ev_tri, 0));
    pack_w32_tiles<<<nb * (nb + 1) / 2, 256, 0, s>>>(W_.p, w32_.p, kp_);
    launches += 1;
    MPHY_CUDA(cudaGetLastError());
}

CoarseSpace::~CoarseSpace() {
    if (fact_graph_) cudaGraphExecDestroy(fact_graph_);
    for (auto& e : ev_)
        if (e) cudaEventDestroy(e);
    for (auto& q : side_)
        if (q) cudaStreamDestroy(q);
}

template void CoarseSpace::setup<double>(const SellView&, const double*, const double*, cudaStream_t);
template void CoarseSpace::setup<float>(const SellView&, const float*, const double*, cudaStream_t);

CoarseView CoarseSpace::view() const {
    CoarseView v;
    v.n_agg = n_agg_;
    v.nm = nm_;
    v.k = nm_ * n_agg_;
    v.kp = kp_;
    v.agg = agg_.p;
    v.agg_ptr = agg_ptr_.p;
    v.agg_nodes = agg_nodes_.p;
    v.d = d_.p;
    v.fixed = mesh_->fixed.p;
    v.dperm = dperm_.p;
    v.fperm = fperm_.p;
    v.w32 = w32_.p;
    v.y = y_.p;
    v.nb = kp_ / T;
    v.gpart = gpart_.p;
    v.rowyy = rowyy_.p;
    v.w = w_.p;
    v.wpart = wpart_.p;
    v.wcount = wcount_.p;
    v.c = c_.p;
    return v;
}

}  // namespace mphy
