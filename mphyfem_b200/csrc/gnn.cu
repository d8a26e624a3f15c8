// gnn.cu -- learned FSAI: forward, backward and Adam kernels of a small message-passing network.
//
// Graph: the nodes of the mesh, the edges the 3x3 blocks of the assembled operator. With the
// Jacobi scaling A^ = D^{-1/2} A D^{-1/2} (D the diagonal; prescribed DOFs act as identity rows)
// every feature is dimensionless, and the exact FSAI of A^ is G^ = G D^{1/2}, so the network
// predicts G^ and the preconditioner uses G = G^ D^{-1/2}.
//
//   h0_n   = relu(W_in x_n + b_in)                       x_n: A^_nn (9), prescribed flags (3), deg/27
//   layer l (3 of them, width 64):
//     P    = h U^T
//     msg_n = (1/deg_n) sum_{m ~ n} relu(P_m + V e_nm + c)        e_nm = A^_nm (9)
//     q    = h S^T + msg T^T + d,   h <- h + relu(q)
//   lower edge (n, m), m <= n:  G^_nm = Wa h_n + Wb h_m + Wc e_nm + bo   (9 outputs; e_nn = A^_nn)
//   loss = mean over lower edges and entries of (G^ - G^_exact)^2
//
// Weights are stored FP32 (Adam) and used as BF16 by every kernel; accumulation is FP32. The
// backward pass recomputes each message from P, V and the edge features instead of storing one
// 64-vector per edge. Warps own nodes; each lane owns channels lane and lane + 32.
#include <cmath>

#include "gnn.cuh"

namespace mphy {
namespace {

constexpr int H = kGnnH;
constexpr int kWarpsPerCta = 8;

__device__ __forceinline__ float bf(const __nv_bfloat16* w, int i) { return __bfloat162float(w[i]); }

// Raw 3x3 block (a, b) of the stored operator at block slot k of row n (column m), with the
// prescribed DOFs of the FP32 storage turned into identity rows.
__device__ __forceinline__ void raw_block(const SellView& A, const void* aval, bool f32, int64_t n, int k, int64_t m,
                                          float out[9]) {
    if (m == n && A.diag64) {
        for (int v = 0; v < 9; ++v) out[v] = (float)A.diag64[9 * n + v];
    } else {
        const int64_t off = 9 * (A.slice_base[n >> 5] + 32 * (int64_t)k) + (n & 31);
        if (f32) {
            const float* p = static_cast<const float*>(aval) + off;
            for (int v = 0; v < 9; ++v) out[v] = p[32 * v];
        } else {
            const double* p = static_cast<const double*>(aval) + off;
            for (int v = 0; v < 9; ++v) out[v] = (float)p[32 * v];
        }
    }
    if (A.fixed) {
        for (int v = 0; v < 9; ++v)
            if (A.fixed[3 * n + v / 3] || A.fixed[3 * m + v % 3]) out[v] = (m == n && v / 3 == v % 3) ? 1.f : 0.f;
    }
}

__device__ __forceinline__ void scaled_block(const SellView& A, const void* aval, bool f32, const float* sqrt_s,
                                             int64_t n, int k, int64_t m, float e[9]) {
    raw_block(A, aval, f32, n, k, m, e);
    for (int v = 0; v < 9; ++v) e[v] /= sqrt_s[3 * n + v / 3] * sqrt_s[3 * m + v % 3];
}

// ---------------------------------------------------------------- graph features
__global__ void diag_scale_kernel(SellView A, const void* aval, bool f32, const int64_t* __restrict__ brow,
                                  const int32_t* __restrict__ bcol, float* __restrict__ sqrt_s, float* __restrict__ x,
                                  int32_t* __restrict__ deg) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < A.n_node; n += (int64_t)gridDim.x * blockDim.x) {
        int k = 0;
        const int64_t b = brow[n], e = brow[n + 1];
        while (b + k < e && bcol[b + k] != (int32_t)n) ++k;
        float D[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (b + k < e) raw_block(A, aval, f32, n, k, n, D);
        float s[3];
        for (int a = 0; a < 3; ++a) {
            const float d = fabsf(D[4 * a]);
            s[a] = d > 0.f ? sqrtf(d) : 1.f;
            sqrt_s[3 * n + a] = s[a];
        }
        for (int v = 0; v < 9; ++v) x[13 * n + v] = D[v] / (s[v / 3] * s[v % 3]);
        for (int a = 0; a < 3; ++a) x[13 * n + 9 + a] = 0.f;  // prescribed flags: fixed_flags_kernel
        const int dg = (int)(e - b) - 1;
        deg[n] = dg > 0 ? dg : 1;
        x[13 * n + 12] = (float)(e - b - 1) / 27.f;
    }
}

// Block-Jacobi FSAI in the network's scaled units: with only the diagonal block in the pattern,
// the block FSAI of fsai.cu is G_nn = L^T with L L^T = (A^_nn)^{-1}. The network predicts a
// correction to it, so an untrained (zero-output) network is block-Jacobi. A block that is not
// positive definite gives the identity (fsai.cu's fallback row, 1/sqrt|a_ii| unscaled).
__global__ void base_kernel(int32_t n_node, const float* __restrict__ x, float* __restrict__ base) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        double A[3][3];
        for (int v = 0; v < 9; ++v) A[v / 3][v % 3] = 0.5 * ((double)x[13 * n + v] + (double)x[13 * n + 3 * (v % 3) + v / 3]);
        const double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                           A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
        float out[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        if (det > 0.0) {
            const double r = 1.0 / det;
            double Y[3][3];  // (A^_nn)^{-1}, symmetric
            Y[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) * r;
            Y[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * r;
            Y[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * r;
            Y[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * r;
            Y[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * r;
            Y[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * r;
            const double l00s = Y[0][0];
            if (l00s > 0.0) {
                const double l00 = sqrt(l00s), l10 = Y[0][1] / l00, l20 = Y[0][2] / l00;
                const double l11s = Y[1][1] - l10 * l10;
                if (l11s > 0.0) {
                    const double l11 = sqrt(l11s), l21 = (Y[1][2] - l20 * l10) / l11;
                    const double l22s = Y[2][2] - l20 * l20 - l21 * l21;
                    if (l22s > 0.0) {
                        const double l22 = sqrt(l22s);
                        // G_nn = L^T (row-major)
                        const float g[9] = {(float)l00, (float)l10, (float)l20, 0.f, (float)l11, (float)l21,
                                            0.f, 0.f, (float)l22};
                        for (int v = 0; v < 9; ++v) out[v] = g[v];
                    }
                }
            }
        }
        for (int v = 0; v < 9; ++v) base[9 * n + v] = out[v];
    }
}

// prescribed flags for the FP64 storage (its rows are already identity): from the pattern's mask
__global__ void fixed_flags_kernel(int32_t n_node, const uint8_t* __restrict__ fixed, float* __restrict__ x) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x)
        for (int a = 0; a < 3; ++a) x[13 * n + 9 + a] = (float)fixed[3 * n + a];
}

__global__ void lower_slots_kernel(int32_t n_node, const int64_t* __restrict__ lrow, const int32_t* __restrict__ lcol,
                                   const int64_t* __restrict__ brow, const int32_t* __restrict__ bcol,
                                   int32_t* __restrict__ lslot, int32_t* __restrict__ lrow_of) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        for (int64_t j = lrow[n]; j < lrow[n + 1]; ++j) {
            const int32_t m = lcol[j];
            int64_t lo = brow[n], hi = brow[n + 1];
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (bcol[mid] < m) lo = mid + 1;
                else hi = mid;
            }
            lslot[j] = (int32_t)(lo - brow[n]);
            lrow_of[j] = (int32_t)n;
        }
    }
}

__global__ void upper_to_lower_kernel(int32_t n_node, const int64_t* __restrict__ urow, const int32_t* __restrict__ ucol,
                                      const int64_t* __restrict__ lrow, const int32_t* __restrict__ lcol,
                                      int64_t* __restrict__ u2l) {
    for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < n_node; m += (int64_t)gridDim.x * blockDim.x) {
        for (int64_t q = urow[m]; q < urow[m + 1]; ++q) {
            const int32_t n = ucol[q];
            int64_t lo = lrow[n], hi = lrow[n + 1];
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (lcol[mid] < (int32_t)m) lo = mid + 1;
                else hi = mid;
            }
            u2l[q] = lo;
        }
    }
}

// ---------------------------------------------------------------- training loss
// Kaporin's K-condition number of the preconditioned operator, whose minimiser over the pattern
// is exact FSAI and which bounds CG's iteration count:
//   K = (tr(G^ A^ G^T) / N) / det(G^ A^ G^T)^{1/N},
//   loss = log K + (1/N) log det A^ = log(tr(G^ A^ G^T) / N) - (2/N) sum_n log|det G^_nn|
// (N = 3 n_node; G^ lower block-triangular, so det G^ is the product of its diagonal blocks'
// determinants). The trace is a sum over block rows of local quadratic forms,
//   tr_n = sum_{j, j' in row n} tr(G^_j A^_{m_j m_j'} G^_j'^T),
// and d tr / d G^_j = 2 T_j with T_j = sum_{j'} G^_j' A^_{m_j' m_j}.
__device__ __forceinline__ int64_t slot_in_row(const int64_t* brow, const int32_t* bcol, int64_t r, int32_t c) {
    int64_t lo = brow[r], hi = brow[r + 1];
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (bcol[mid] < c) lo = mid + 1;
        else hi = mid;
    }
    return (lo < brow[r + 1] && bcol[lo] == c) ? lo - brow[r] : -1;
}

// One warp per block row; lane j of the row (at most 32 lower blocks) forms T_j.
__global__ void __launch_bounds__(256) kaporin_rows(SellView A, const void* aval, bool f32, int32_t n_node,
                                                    const int64_t* __restrict__ brow, const int32_t* __restrict__ bcol,
                                                    const int64_t* __restrict__ lrow, const int32_t* __restrict__ lcol,
                                                    const float* __restrict__ sqrt_s, const float* __restrict__ ghat,
                                                    float* __restrict__ tbuf, double* __restrict__ part_tr,
                                                    double* __restrict__ part_ld) {
    const int lane = threadIdx.x & 31;
    for (int64_t n = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; n < n_node;
         n += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t r0 = lrow[n], len = lrow[n + 1] - r0;
        double tr = 0.0, ld = 0.0;
        if (lane < len) {
            const int64_t j = r0 + lane;
            const int32_t m = lcol[j];
            float T[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int64_t jp = r0; jp < r0 + len; ++jp) {
                const int32_t mp = lcol[jp];
                const int64_t k = slot_in_row(brow, bcol, mp, m);
                if (k < 0) continue;  // m and m' are not neighbours: A^_{m' m} = 0
                float e[9];
                scaled_block(A, aval, f32, sqrt_s, mp, (int)k, m, e);
                const float* g = ghat + 9 * jp;
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c) T[3 * r + c] += g[3 * r] * e[c] + g[3 * r + 1] * e[3 + c] + g[3 * r + 2] * e[6 + c];
            }
            const float* gj = ghat + 9 * j;
#pragma unroll
            for (int v = 0; v < 9; ++v) {
                tbuf[9 * j + v] = T[v];
                tr += (double)T[v] * (double)gj[v];
            }
            if (m == (int32_t)n) {
                const double d = (double)gj[0] * ((double)gj[4] * gj[8] - (double)gj[5] * gj[7]) -
                                 (double)gj[1] * ((double)gj[3] * gj[8] - (double)gj[5] * gj[6]) +
                                 (double)gj[2] * ((double)gj[3] * gj[7] - (double)gj[4] * gj[6]);
                ld = log(fmax(fabs(d), 1e-300));
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            tr += __shfl_xor_sync(0xffffffffu, tr, o);
            ld += __shfl_xor_sync(0xffffffffu, ld, o);
        }
        if (lane == 0) {
            part_tr[n] = tr;
            part_ld[n] = ld;
        }
    }
}

// One CTA: fixed-order sums of the row partials; red = {tr, sum log|det|, loss}.
__global__ void __launch_bounds__(1024) kaporin_reduce(int32_t n_node, const double* __restrict__ part_tr,
                                                       const double* __restrict__ part_ld, double* __restrict__ red,
                                                       double* __restrict__ loss) {
    __shared__ double s1[1024], s2[1024];
    double a = 0.0, b = 0.0;
    for (int64_t i = threadIdx.x; i < n_node; i += blockDim.x) {
        a += part_tr[i];
        b += part_ld[i];
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s1[threadIdx.x] += s1[threadIdx.x + o];
            s2[threadIdx.x] += s2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double N = 3.0 * n_node;
        red[0] = s1[0];
        red[1] = s2[0];
        red[2] = log(s1[0] / N) - 2.0 / N * s2[0];
        *loss = red[2];
    }
}

// dL/dG^_j = (2 / tr) T_j - (2 / N) [m == n] G^_nn^{-T}, zero on entries fixed to the identity;
// dout_j = dL/dP_j = base_n^T dL/dG^_j (the decoder's P, see dec_fwd).
__global__ void kaporin_grad(int64_t n_lower, int32_t n_node, const int32_t* __restrict__ lrow_of,
                             const int32_t* __restrict__ lcol, const uint8_t* __restrict__ fixed,
                             const float* __restrict__ base, const float* __restrict__ ghat,
                             const float* __restrict__ tbuf, const double* __restrict__ red, float* __restrict__ dout) {
    const double tr = red[0], N = 3.0 * n_node;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n_lower; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = lrow_of[j], m = lcol[j];
        float dg[9];
        for (int v = 0; v < 9; ++v) dg[v] = (float)(2.0 / tr * tbuf[9 * j + v]);
        if (m == n) {
            const float* g = ghat + 9 * j;
            const double d = (double)g[0] * ((double)g[4] * g[8] - (double)g[5] * g[7]) -
                             (double)g[1] * ((double)g[3] * g[8] - (double)g[5] * g[6]) +
                             (double)g[2] * ((double)g[3] * g[7] - (double)g[4] * g[6]);
            if (fabs(d) > 1e-300) {
                // G^{-T}[r][c] = cof(G)[r][c] / det
                const double cof[9] = {g[4] * g[8] - g[5] * g[7], g[5] * g[6] - g[3] * g[8], g[3] * g[7] - g[4] * g[6],
                                       g[2] * g[7] - g[1] * g[8], g[0] * g[8] - g[2] * g[6], g[1] * g[6] - g[0] * g[7],
                                       g[1] * g[5] - g[2] * g[4], g[2] * g[3] - g[0] * g[5], g[0] * g[4] - g[1] * g[3]};
                for (int v = 0; v < 9; ++v) dg[v] -= (float)(2.0 / N * cof[v] / d);
            }
        }
        if (fixed)
            for (int v = 0; v < 9; ++v)
                if (fixed[3 * n + v / 3] || fixed[3 * m + v % 3]) dg[v] = 0.f;
        const float* B = base + 9 * n;
        for (int o = 0; o < 9; ++o) {
            const int k = o / 3, c = o % 3;
            dout[9 * j + o] = B[k] * dg[c] + B[3 + k] * dg[3 + c] + B[6 + k] * dg[6 + c];
        }
    }
}

// ---------------------------------------------------------------- dense node maps
// Y[n][o] = sum_k W[o][k] X[n][k] (+ b[o]) (+ relu); W at w (bf16 [O][K]), b at bias (or null)
template <int K, int O, bool RELU>
__global__ void __launch_bounds__(256) lin_fwd(int32_t n, const float* __restrict__ X, const __nv_bfloat16* __restrict__ w,
                                               const __nv_bfloat16* __restrict__ bias, float* __restrict__ Y) {
    __shared__ float W[O][K + 1];
    __shared__ float B[O];
    __shared__ float xs[kWarpsPerCta][K];
    for (int i = threadIdx.x; i < O * K; i += blockDim.x) W[i / K][i % K] = bf(w, i);
    for (int i = threadIdx.x; i < O; i += blockDim.x) B[i] = bias ? bf(bias, i) : 0.f;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t node = (int64_t)blockIdx.x * kWarpsPerCta + warp; node < n; node += (int64_t)gridDim.x * kWarpsPerCta) {
        for (int k = lane; k < K; k += 32) xs[warp][k] = X[node * K + k];
        __syncwarp();
        for (int o = lane; o < O; o += 32) {
            float acc = B[o];
#pragma unroll 8
            for (int k = 0; k < K; ++k) acc += W[o][k] * xs[warp][k];
            Y[node * O + o] = RELU ? fmaxf(acc, 0.f) : acc;
        }
        __syncwarp();
    }
}

// dX[n][k] (+)= sum_o W[o][k] dY[n][o]
template <int K, int O, bool ACC>
__global__ void __launch_bounds__(256) lin_bwd_data(int32_t n, const float* __restrict__ dY, const __nv_bfloat16* __restrict__ w,
                                                    float* __restrict__ dX) {
    __shared__ float W[O][K + 1];
    __shared__ float ys[kWarpsPerCta][O];
    for (int i = threadIdx.x; i < O * K; i += blockDim.x) W[i / K][i % K] = bf(w, i);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t node = (int64_t)blockIdx.x * kWarpsPerCta + warp; node < n; node += (int64_t)gridDim.x * kWarpsPerCta) {
        for (int o = lane; o < O; o += 32) ys[warp][o] = dY[node * O + o];
        __syncwarp();
        for (int k = lane; k < K; k += 32) {
            float acc = 0.f;
#pragma unroll 8
            for (int o = 0; o < O; ++o) acc += W[o][k] * ys[warp][o];
            if (ACC) dX[node * K + k] += acc;
            else dX[node * K + k] = acc;
        }
        __syncwarp();
    }
}

// gW[o][k] += sum_n dY[n][o] X[n][k]; gb[o] += sum_n dY[n][o] (gb may be null)
template <int K, int O>
__global__ void __launch_bounds__(256) lin_bwd_weight(int32_t n, const float* __restrict__ dY, const float* __restrict__ X,
                                                      float* __restrict__ gW, float* __restrict__ gb) {
    constexpr int NB = 32;
    __shared__ float ys[NB][O];
    __shared__ float xs[NB][K];
    constexpr int PER = (O * K + 255) / 256;
    float acc[PER];
    float bacc = 0.f;
    for (int i = 0; i < PER; ++i) acc[i] = 0.f;
    const int64_t chunk = ((int64_t)n + gridDim.x - 1) / gridDim.x;
    const int64_t n0 = blockIdx.x * chunk, n1 = min((int64_t)n, n0 + chunk);
    for (int64_t base = n0; base < n1; base += NB) {
        const int cnt = (int)min((int64_t)NB, n1 - base);
        for (int i = threadIdx.x; i < cnt * O; i += blockDim.x) ys[i / O][i % O] = dY[(base + i / O) * O + i % O];
        for (int i = threadIdx.x; i < cnt * K; i += blockDim.x) xs[i / K][i % K] = X[(base + i / K) * K + i % K];
        __syncthreads();
        for (int i = 0; i < PER; ++i) {
            const int idx = threadIdx.x + 256 * i;
            if (idx < O * K) {
                const int o = idx / K, k = idx % K;
                float s = 0.f;
                for (int t = 0; t < cnt; ++t) s += ys[t][o] * xs[t][k];
                acc[i] += s;
            }
        }
        if (gb && threadIdx.x < O)
            for (int t = 0; t < cnt; ++t) bacc += ys[t][threadIdx.x];
        __syncthreads();
    }
    for (int i = 0; i < PER; ++i) {
        const int idx = threadIdx.x + 256 * i;
        if (idx < O * K) atomicAdd(&gW[idx], acc[i]);
    }
    if (gb && threadIdx.x < O) atomicAdd(&gb[threadIdx.x], bacc);
}

// q = h S^T + msg T^T + d;  h_next = h + relu(q)
__global__ void __launch_bounds__(256) update_fwd(int32_t n, const float* __restrict__ h, const float* __restrict__ msg,
                                                  const __nv_bfloat16* __restrict__ S, const __nv_bfloat16* __restrict__ T,
                                                  const __nv_bfloat16* __restrict__ d, float* __restrict__ q,
                                                  float* __restrict__ hn) {
    extern __shared__ float sm[];
    float(*Ws)[H + 1] = reinterpret_cast<float(*)[H + 1]>(sm);
    float(*Wt)[H + 1] = reinterpret_cast<float(*)[H + 1]>(sm + H * (H + 1));
    float* D = sm + 2 * H * (H + 1);
    float(*hs)[2 * H] = reinterpret_cast<float(*)[2 * H]>(D + H);
    for (int i = threadIdx.x; i < H * H; i += blockDim.x) {
        Ws[i / H][i % H] = bf(S, i);
        Wt[i / H][i % H] = bf(T, i);
    }
    for (int i = threadIdx.x; i < H; i += blockDim.x) D[i] = bf(d, i);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t node = (int64_t)blockIdx.x * kWarpsPerCta + warp; node < n; node += (int64_t)gridDim.x * kWarpsPerCta) {
        hs[warp][lane] = h[node * H + lane];
        hs[warp][lane + 32] = h[node * H + lane + 32];
        hs[warp][H + lane] = msg[node * H + lane];
        hs[warp][H + lane + 32] = msg[node * H + lane + 32];
        __syncwarp();
        for (int o = lane; o < H; o += 32) {
            float acc = D[o];
#pragma unroll 8
            for (int k = 0; k < H; ++k) acc += Ws[o][k] * hs[warp][k] + Wt[o][k] * hs[warp][H + k];
            q[node * H + o] = acc;
            hn[node * H + o] = hs[warp][o] + fmaxf(acc, 0.f);
        }
        __syncwarp();
    }
}

// msg_n = (1/deg_n) sum_{m ~ n} relu(P_m + V e_nm + c)
__global__ void __launch_bounds__(256) msg_fwd(SellView A, const void* aval, bool f32, const int64_t* __restrict__ brow,
                                               const int32_t* __restrict__ bcol, const float* __restrict__ sqrt_s,
                                               const int32_t* __restrict__ deg, const float* __restrict__ P,
                                               const __nv_bfloat16* __restrict__ V, const __nv_bfloat16* __restrict__ c,
                                               float* __restrict__ msg) {
    __shared__ float Vs[H][kGnnEdgeIn];
    __shared__ float Cs[H];
    for (int i = threadIdx.x; i < H * kGnnEdgeIn; i += blockDim.x) Vs[i / kGnnEdgeIn][i % kGnnEdgeIn] = bf(V, i);
    for (int i = threadIdx.x; i < H; i += blockDim.x) Cs[i] = bf(c, i);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t n = (int64_t)blockIdx.x * kWarpsPerCta + warp; n < A.n_node; n += (int64_t)gridDim.x * kWarpsPerCta) {
        float a0 = 0.f, a1 = 0.f;
        const int64_t b = brow[n];
        const int len = (int)(brow[n + 1] - b);
        for (int k = 0; k < len; ++k) {
            const int64_t m = bcol[b + k];
            if (m == n) continue;
            float e[9];
            scaled_block(A, aval, f32, sqrt_s, n, k, m, e);
            float p0 = P[m * H + lane] + Cs[lane], p1 = P[m * H + lane + 32] + Cs[lane + 32];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                p0 += Vs[lane][i] * e[i];
                p1 += Vs[lane + 32][i] * e[i];
            }
            a0 += fmaxf(p0, 0.f);
            a1 += fmaxf(p1, 0.f);
        }
        const float inv = 1.f / (float)deg[n];
        msg[n * H + lane] = a0 * inv;
        msg[n * H + lane + 32] = a1 * inv;
    }
}

// dP_m = sum_{n ~ m} (dmsg_n / deg_n) [P_m + V e_nm + c > 0], with dV, dc accumulated.
// e_nm = A^_nm = (A^_mn)^T, read from m's own row.
__global__ void __launch_bounds__(256) msg_bwd(SellView A, const void* aval, bool f32, const int64_t* __restrict__ brow,
                                               const int32_t* __restrict__ bcol, const float* __restrict__ sqrt_s,
                                               const int32_t* __restrict__ deg, const float* __restrict__ P,
                                               const __nv_bfloat16* __restrict__ V, const __nv_bfloat16* __restrict__ c,
                                               const float* __restrict__ dmsg, float* __restrict__ dP,
                                               float* __restrict__ gV, float* __restrict__ gc) {
    __shared__ float Vs[H][kGnnEdgeIn];
    __shared__ float Cs[H];
    __shared__ float gVs[H][kGnnEdgeIn];
    __shared__ float gcs[H];
    for (int i = threadIdx.x; i < H * kGnnEdgeIn; i += blockDim.x) {
        Vs[i / kGnnEdgeIn][i % kGnnEdgeIn] = bf(V, i);
        gVs[i / kGnnEdgeIn][i % kGnnEdgeIn] = 0.f;
    }
    for (int i = threadIdx.x; i < H; i += blockDim.x) {
        Cs[i] = bf(c, i);
        gcs[i] = 0.f;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float lv0[9], lv1[9], lc0 = 0.f, lc1 = 0.f;
    for (int i = 0; i < 9; ++i) lv0[i] = lv1[i] = 0.f;
    for (int64_t m = (int64_t)blockIdx.x * kWarpsPerCta + warp; m < A.n_node; m += (int64_t)gridDim.x * kWarpsPerCta) {
        const float pm0 = P[m * H + lane] + Cs[lane], pm1 = P[m * H + lane + 32] + Cs[lane + 32];
        float d0 = 0.f, d1 = 0.f;
        const int64_t b = brow[m];
        const int len = (int)(brow[m + 1] - b);
        for (int k = 0; k < len; ++k) {
            const int64_t n = bcol[b + k];
            if (n == m) continue;
            float emn[9], e[9];
            scaled_block(A, aval, f32, sqrt_s, m, k, n, emn);
            for (int v = 0; v < 9; ++v) e[v] = emn[3 * (v % 3) + v / 3];  // e_nm = (A^_mn)^T
            float p0 = pm0, p1 = pm1;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                p0 += Vs[lane][i] * e[i];
                p1 += Vs[lane + 32][i] * e[i];
            }
            const float inv = 1.f / (float)deg[n];
            const float g0 = p0 > 0.f ? dmsg[n * H + lane] * inv : 0.f;
            const float g1 = p1 > 0.f ? dmsg[n * H + lane + 32] * inv : 0.f;
            d0 += g0;
            d1 += g1;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                lv0[i] += g0 * e[i];
                lv1[i] += g1 * e[i];
            }
            lc0 += g0;
            lc1 += g1;
        }
        dP[m * H + lane] = d0;
        dP[m * H + lane + 32] = d1;
    }
    for (int i = 0; i < 9; ++i) {
        atomicAdd(&gVs[lane][i], lv0[i]);
        atomicAdd(&gVs[lane + 32][i], lv1[i]);
    }
    atomicAdd(&gcs[lane], lc0);
    atomicAdd(&gcs[lane + 32], lc1);
    __syncthreads();
    for (int i = threadIdx.x; i < H * kGnnEdgeIn; i += blockDim.x) atomicAdd(&gV[i], gVs[i / kGnnEdgeIn][i % kGnnEdgeIn]);
    for (int i = threadIdx.x; i < H; i += blockDim.x) atomicAdd(&gc[i], gcs[i]);
}

// dq = dh_next [q > 0]
__global__ void relu_mask_kernel(int64_t n, const float* __restrict__ dh, const float* __restrict__ q,
                                 float* __restrict__ dq) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dq[i] = q[i] > 0.f ? dh[i] : 0.f;
}

// decoder on lower edges: P = [m == n] I + an_n + bn_m + [m != n] Wc e_nm + bo, and the predicted
// block is
// G^_nm = base_n P (3x3 product): block-Jacobi FSAI times a learned factor, so an untrained
// network (P = I on the diagonal, 0 elsewhere) is block-Jacobi, and the structure of exact FSAI's
// off-diagonal blocks, G_nm ~ -G_nn A^_nm, is linear in the decoder. The loss kernels (kaporin_*) give
// dout = dL/dP.
// Entries whose row or column DOF is prescribed are not predicted: they take the identity (1 on a
// prescribed DOF's own diagonal, 0 elsewhere), the structure of the exact FSAI of an operator with
// identity rows and columns there. M = G^T G then leaves prescribed components of the residual
// alone, which the mixed operator (couplings to prescribed DOFs stored, masked in SpMV) requires.
__global__ void __launch_bounds__(256) dec_fwd(SellView A, const void* aval, bool f32, const uint8_t* __restrict__ fixed,
                                               const float* __restrict__ base, int64_t n_lower,
                                               const int32_t* __restrict__ lrow_of, const int32_t* __restrict__ lcol,
                                               const int32_t* __restrict__ lslot, const float* __restrict__ sqrt_s,
                                               const float* __restrict__ an, const float* __restrict__ bn,
                                               const __nv_bfloat16* __restrict__ Wc, const __nv_bfloat16* __restrict__ bo,
                                               float* __restrict__ ghat, float* __restrict__ pred) {
    __shared__ float W[81], B[9];
    for (int i = threadIdx.x; i < 81; i += blockDim.x) W[i] = bf(Wc, i);
    for (int i = threadIdx.x; i < 9; i += blockDim.x) B[i] = bf(bo, i);
    __syncthreads();
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n_lower; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = lrow_of[j], m = lcol[j];
        float e[9], P[9], Bn[9];
        scaled_block(A, aval, f32, sqrt_s, n, lslot[j], m, e);
        for (int o = 0; o < 9; ++o) {
            float v = an[9 * n + o] + bn[9 * m + o] + B[o];
            if (m != n)
                for (int i = 0; i < 9; ++i) v += W[9 * o + i] * e[i];
            P[o] = v + ((m == n && o / 3 == o % 3) ? 1.f : 0.f);
            Bn[o] = base[9 * n + o];
        }
        for (int o = 0; o < 9; ++o) {
            const int r = o / 3, c = o % 3;
            float v = Bn[3 * r] * P[c] + Bn[3 * r + 1] * P[3 + c] + Bn[3 * r + 2] * P[6 + c];
            const bool masked = fixed && (fixed[3 * n + r] || fixed[3 * m + c]);
            if (masked) v = (m == n && r == c) ? 1.f : 0.f;
            if (ghat) ghat[9 * j + o] = v;
            if (pred) pred[9 * j + o] = v / sqrt_s[3 * m + c];
        }
    }
}

// dan_n = sum over lower edges of row n; dbn_m = sum over lower edges with column m (via G^T rows)
__global__ void dec_bwd_nodes(int32_t n_node, const int64_t* __restrict__ lrow, const int64_t* __restrict__ urow,
                              const int64_t* __restrict__ u2l, const float* __restrict__ dout, float* __restrict__ dan,
                              float* __restrict__ dbn) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        float a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int64_t j = lrow[n]; j < lrow[n + 1]; ++j)
            for (int o = 0; o < 9; ++o) a[o] += dout[9 * j + o];
        for (int64_t q = urow[n]; q < urow[n + 1]; ++q) {
            const int64_t j = u2l[q];
            for (int o = 0; o < 9; ++o) b[o] += dout[9 * j + o];
        }
        for (int o = 0; o < 9; ++o) {
            dan[9 * n + o] = a[o];
            dbn[9 * n + o] = b[o];
        }
    }
}

// dWc += sum dout (x) e, dbo += sum dout
__global__ void __launch_bounds__(256) dec_bwd_weights(SellView A, const void* aval, bool f32, int64_t n_lower,
                                                       const int32_t* __restrict__ lrow_of, const int32_t* __restrict__ lcol,
                                                       const int32_t* __restrict__ lslot, const float* __restrict__ sqrt_s,
                                                       const float* __restrict__ dout, float* __restrict__ gWc,
                                                       float* __restrict__ gbo) {
    __shared__ float s[90];
    for (int i = threadIdx.x; i < 90; i += blockDim.x) s[i] = 0.f;
    __syncthreads();
    float acc[90];
    for (int i = 0; i < 90; ++i) acc[i] = 0.f;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n_lower; j += (int64_t)gridDim.x * blockDim.x) {
        float e[9];
        const bool self = lrow_of[j] == lcol[j];  // the edge term acts on off-diagonal blocks only
        scaled_block(A, aval, f32, sqrt_s, lrow_of[j], lslot[j], lcol[j], e);
        for (int o = 0; o < 9; ++o) {
            const float d = dout[9 * j + o];
            if (!self)
                for (int i = 0; i < 9; ++i) acc[9 * o + i] += d * e[i];
            acc[81 + o] += d;
        }
    }
    for (int i = 0; i < 90; ++i) atomicAdd(&s[i], acc[i]);
    __syncthreads();
    for (int i = threadIdx.x; i < 81; i += blockDim.x) atomicAdd(&gWc[i], s[i]);
    for (int i = threadIdx.x; i < 9; i += blockDim.x) atomicAdd(&gbo[i], s[81 + i]);
}

__global__ void to_bf16_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) wb[i] = __float2bfloat16(w[i]);
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                            __nv_bfloat16* __restrict__ wb, int n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        wb[i] = __float2bfloat16(w[i]);
    }
}

unsigned node_grid(int64_t n, int sm) {
    const int64_t want = (n + kWarpsPerCta - 1) / kWarpsPerCta;
    const int64_t cap = (int64_t)sm * 16;
    return (unsigned)(want < 1 ? 1 : (want > cap ? cap : want));
}

}  // namespace

void Gnn::init(mphy_ctx* ctx, const float* params) {
    ctx_ = ctx;
    const int n = GnnLayout::total;
    w_.alloc(n);
    grad_.alloc(n);
    m_.alloc(n);
    v_.alloc(n);
    wb_.alloc(n);
    loss_.alloc(1);
    MPHY_CUDA(cudaMemset(m_.p, 0, m_.bytes()));
    MPHY_CUDA(cudaMemset(v_.p, 0, v_.bytes()));
    MPHY_CUDA(cudaMemset(grad_.p, 0, grad_.bytes()));
    set_params(params);
}

void Gnn::set_params(const float* host) {
    cudaStream_t s = ctx_->stream;
    w_.upload(host, GnnLayout::total, s);
    to_bf16_kernel<<<64, 256, 0, s>>>(w_.p, wb_.p, GnnLayout::total);
    MPHY_CUDA(cudaGetLastError());
    MPHY_CUDA(cudaStreamSynchronize(s));
}

void Gnn::get_params(float* host) const {
    w_.download(host, GnnLayout::total, ctx_->stream);
    MPHY_CUDA(cudaStreamSynchronize(ctx_->stream));
}

void Gnn::get_grads(float* host) const {
    grad_.download(host, GnnLayout::total, ctx_->stream);
    MPHY_CUDA(cudaStreamSynchronize(ctx_->stream));
}

void Gnn::zero_grads(cudaStream_t s) { MPHY_CUDA(cudaMemsetAsync(grad_.p, 0, grad_.bytes(), s)); }

void Gnn::adam_step(float lr, float b1, float b2, float eps, cudaStream_t s) {
    ++adam_t_;
    const float c1 = 1.f - std::pow(b1, (float)adam_t_), c2 = 1.f - std::pow(b2, (float)adam_t_);
    adam_kernel<<<64, 256, 0, s>>>(w_.p, grad_.p, m_.p, v_.p, wb_.p, GnnLayout::total, lr, b1, b2, eps, c1, c2);
    MPHY_CUDA(cudaGetLastError());
}

void Gnn::ensure_workspace(int32_t nn, int64_t nl) {
    if (nn <= ws_nodes_ && nl <= ws_lower_) return;
    ws_nodes_ = nn;
    ws_lower_ = nl;
    const size_t nh = (size_t)nn * H;
    h_.alloc((kGnnLayers + 1) * nh);
    P_.alloc(kGnnLayers * nh);
    msg_.alloc(kGnnLayers * nh);
    q_.alloc(kGnnLayers * nh);
    dh_.alloc(nh);
    dP_.alloc(nh);
    dmsg_.alloc(nh);
    dq_.alloc(nh);
    an_.alloc(9 * (size_t)nn);
    bn_.alloc(9 * (size_t)nn);
    dan_.alloc(9 * (size_t)nn);
    dbn_.alloc(9 * (size_t)nn);
    dout_.alloc(9 * (size_t)nl);
    ghat_.alloc(9 * (size_t)nl);
    tbuf_.alloc(9 * (size_t)nl);
    part_tr_.alloc(nn);
    part_ld_.alloc(nn);
    red_.alloc(3);
}

void Gnn::build_graph(GnnGraph& g, const mphy_pattern* P, const Fsai& F, const SellView& A, const void* aval,
                      bool f32, const uint8_t* fixed, bool training, cudaStream_t s) {
    const int sm = ctx_->sm_count;
    const int32_t nn = P->n_node;
    const SellPattern& L = F.lower();
    const SellPattern& U = F.upper();
    g.n_node = nn;
    g.n_lower = L.n_blocks;
    if (g.sqrt_s.n != 3 * (size_t)nn) {
        g.sqrt_s.alloc(3 * (size_t)nn);
        g.xnode.alloc((size_t)kGnnNodeIn * nn);
        g.deg.alloc(nn);
        g.lslot.alloc(L.n_blocks);
        g.lrow_of.alloc(L.n_blocks);
        g.u2l.alloc(U.n_blocks);
    }
    diag_scale_kernel<<<stride_grid(nn, 256, sm), 256, 0, s>>>(A, aval, f32, P->brow_ptr.p, P->bcol.p, g.sqrt_s.p,
                                                               g.xnode.p, g.deg.p);
    fixed_flags_kernel<<<stride_grid(nn, 256, sm), 256, 0, s>>>(nn, fixed, g.xnode.p);
    if (g.base.n != 9 * (size_t)nn) g.base.alloc(9 * (size_t)nn);
    base_kernel<<<stride_grid(nn, 256, sm), 256, 0, s>>>(nn, g.xnode.p, g.base.p);
    lower_slots_kernel<<<stride_grid(nn, 256, sm), 256, 0, s>>>(nn, L.rowptr.p, L.col.p, P->brow_ptr.p, P->bcol.p,
                                                                g.lslot.p, g.lrow_of.p);
    upper_to_lower_kernel<<<stride_grid(nn, 256, sm), 256, 0, s>>>(nn, U.rowptr.p, U.col.p, L.rowptr.p, L.col.p,
                                                                   g.u2l.p);
    g.training = training;
    MPHY_CUDA(cudaGetLastError());
}

double Gnn::run(const GnnGraph& g, const mphy_pattern* Pt, const Fsai& F, const SellView& A, const void* aval,
                bool f32, const uint8_t* fixed, float* out_blocks, bool compute_grad, cudaStream_t s) {
    const int sm = ctx_->sm_count;
    const int32_t nn = g.n_node;
    const int64_t nl = g.n_lower;
    ensure_workspace(nn, nl);
    const size_t nh = (size_t)nn * H;
    const __nv_bfloat16* W = wb_.p;
    float* G = grad_.p;
    const unsigned gn = node_grid(nn, sm);
    const SellPattern& L = F.lower();
    const SellPattern& U = F.upper();
    const bool train = g.training;
    MPHY_REQUIRE(F.max_lower() <= 32, MPHY_ERR_UNSUPPORTED, "learned FSAI: at most 32 lower blocks per row");
    launches = 0;
    // forward
    lin_fwd<kGnnNodeIn, H, true><<<gn, 256, 0, s>>>(nn, g.xnode.p, W + GnnLayout::w_in, W + GnnLayout::b_in, h_.p);
    const size_t upd_smem = (2 * H * (H + 1) + H + kWarpsPerCta * 2 * H) * sizeof(float);
    static std::atomic<uint64_t> attr{0};
    if (first_use_on_device(attr)) {
        MPHY_CUDA(cudaFuncSetAttribute(update_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)upd_smem));
    }
    for (int l = 0; l < kGnnLayers; ++l) {
        const int o = GnnLayout::layer(l);
        float* hl = h_.p + l * nh;
        lin_fwd<H, H, false><<<gn, 256, 0, s>>>(nn, hl, W + o + GnnLayout::U, nullptr, P_.p + l * nh);
        msg_fwd<<<gn, 256, 0, s>>>(A, aval, f32, Pt->brow_ptr.p, Pt->bcol.p, g.sqrt_s.p, g.deg.p, P_.p + l * nh,
                                   W + o + GnnLayout::V, W + o + GnnLayout::c, msg_.p + l * nh);
        update_fwd<<<gn, 256, upd_smem, s>>>(nn, hl, msg_.p + l * nh, W + o + GnnLayout::S, W + o + GnnLayout::Tm,
                                             W + o + GnnLayout::d, q_.p + l * nh, h_.p + (l + 1) * nh);
        launches += 3;
    }
    float* hL = h_.p + kGnnLayers * nh;
    lin_fwd<H, 9, false><<<gn, 256, 0, s>>>(nn, hL, W + GnnLayout::Wa, nullptr, an_.p);
    lin_fwd<H, 9, false><<<gn, 256, 0, s>>>(nn, hL, W + GnnLayout::Wb, nullptr, bn_.p);
    dec_fwd<<<stride_grid(nl, 256, sm), 256, 0, s>>>(A, aval, f32, fixed, g.base.p, nl, g.lrow_of.p, L.col.p,
                                                     g.lslot.p, g.sqrt_s.p, an_.p, bn_.p, W + GnnLayout::Wc,
                                                     W + GnnLayout::bo, train ? ghat_.p : nullptr, out_blocks);
    launches += 4;
    if (train) {
        kaporin_rows<<<stride_grid((int64_t)nn * 32, 256, sm, 16), 256, 0, s>>>(
            A, aval, f32, nn, Pt->brow_ptr.p, Pt->bcol.p, L.rowptr.p, L.col.p, g.sqrt_s.p, ghat_.p, tbuf_.p,
            part_tr_.p, part_ld_.p);
        kaporin_reduce<<<1, 1024, 0, s>>>(nn, part_tr_.p, part_ld_.p, red_.p, loss_.p);
        launches += 2;
        if (compute_grad) {
            kaporin_grad<<<stride_grid(nl, 256, sm), 256, 0, s>>>(nl, nn, g.lrow_of.p, L.col.p, fixed, g.base.p,
                                                                  ghat_.p, tbuf_.p, red_.p, dout_.p);
            launches += 1;
        }
    }
    MPHY_CUDA(cudaGetLastError());
    double loss = 0.0;
    if (train && compute_grad) {
        // decoder backward
        dec_bwd_nodes<<<stride_grid(nn, 256, sm), 256, 0, s>>>(nn, L.rowptr.p, U.rowptr.p, g.u2l.p, dout_.p, dan_.p,
                                                               dbn_.p);
        dec_bwd_weights<<<stride_grid(nl, 256, sm, 2), 256, 0, s>>>(A, aval, f32, nl, g.lrow_of.p, L.col.p, g.lslot.p,
                                                                    g.sqrt_s.p, dout_.p, G + GnnLayout::Wc,
                                                                    G + GnnLayout::bo);
        const unsigned gw = std::max(1u, std::min((unsigned)sm * 2, (unsigned)((nn + 255) / 256)));
        lin_bwd_weight<H, 9><<<gw, 256, 0, s>>>(nn, dan_.p, hL, G + GnnLayout::Wa, nullptr);
        lin_bwd_weight<H, 9><<<gw, 256, 0, s>>>(nn, dbn_.p, hL, G + GnnLayout::Wb, nullptr);
        lin_bwd_data<H, 9, false><<<gn, 256, 0, s>>>(nn, dan_.p, W + GnnLayout::Wa, dh_.p);
        lin_bwd_data<H, 9, true><<<gn, 256, 0, s>>>(nn, dbn_.p, W + GnnLayout::Wb, dh_.p);
        launches += 6;
        for (int l = kGnnLayers - 1; l >= 0; --l) {
            const int o = GnnLayout::layer(l);
            float* hl = h_.p + l * nh;
            // h_{l+1} = h_l + relu(q): dq, then dh_l = dh + S^T dq + (message path)
            relu_mask_kernel<<<stride_grid(nh, 256, sm), 256, 0, s>>>((int64_t)nh, dh_.p, q_.p + l * nh, dq_.p);
            lin_bwd_weight<H, H><<<gw, 256, 0, s>>>(nn, dq_.p, hl, G + o + GnnLayout::S, G + o + GnnLayout::d);
            lin_bwd_weight<H, H><<<gw, 256, 0, s>>>(nn, dq_.p, msg_.p + l * nh, G + o + GnnLayout::Tm, nullptr);
            lin_bwd_data<H, H, true><<<gn, 256, 0, s>>>(nn, dq_.p, W + o + GnnLayout::S, dh_.p);   // residual kept in dh
            lin_bwd_data<H, H, false><<<gn, 256, 0, s>>>(nn, dq_.p, W + o + GnnLayout::Tm, dmsg_.p);
            msg_bwd<<<gn, 256, 0, s>>>(A, aval, f32, Pt->brow_ptr.p, Pt->bcol.p, g.sqrt_s.p, g.deg.p, P_.p + l * nh,
                                       W + o + GnnLayout::V, W + o + GnnLayout::c, dmsg_.p, dP_.p,
                                       G + o + GnnLayout::V, G + o + GnnLayout::c);
            lin_bwd_weight<H, H><<<gw, 256, 0, s>>>(nn, dP_.p, hl, G + o + GnnLayout::U, nullptr);
            lin_bwd_data<H, H, true><<<gn, 256, 0, s>>>(nn, dP_.p, W + o + GnnLayout::U, dh_.p);
            launches += 8;
        }
        // encoder: h0 = relu(W_in x + b_in) -> d pre = dh [h0 > 0]
        relu_mask_kernel<<<stride_grid(nh, 256, sm), 256, 0, s>>>((int64_t)nh, dh_.p, h_.p, dq_.p);
        lin_bwd_weight<kGnnNodeIn, H><<<gw, 256, 0, s>>>(nn, dq_.p, g.xnode.p, G + GnnLayout::w_in, G + GnnLayout::b_in);
        launches += 2;
        MPHY_CUDA(cudaGetLastError());
    }
    if (train) {
        MPHY_CUDA(cudaMemcpyAsync(&loss, loss_.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        MPHY_CUDA(cudaStreamSynchronize(s));
    }
    return loss;
}

}  // namespace mphy
