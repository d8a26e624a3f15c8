// fsai.cu -- K5: block factorised sparse approximate inverse (FSAI), M = G^T G.
//
// The reference's solver takes its preconditioner from PETSc options (SolverPetsc.cpp:117-140;
// PCILU by default, overridable). A triangular solve does not map to a GPU's parallelism; the
// factorised sparse approximate inverse of Kolotilina and Yeremin does: G is lower
// block-triangular on A's own lower block pattern, and applying M = G^T G costs two SpMVs.
//
// Block FSAI: for block row n with lower pattern P = {m <= n : m neighbour of n} (n last), solve
// A[P,P] Y = E_n (the three unit columns of node n), factor Y_nn = L_n L_n^T and set
// G[n, P] = L_n^{-1} Y^T. Then (G A G^T)_nn = I. One warp per block row gathers A[P,P] into
// shared memory, factors it by Cholesky in FP64 and writes its row of G and the mirrored
// blocks of G^T (each block written once: no atomics). A row whose local matrix is not
// positive definite (an indefinite tangent) falls back to the inverse square root of its
// diagonal, and is counted.
#include <climits>
#include <cmath>

#include "fsai.cuh"
#include "pattern.cuh"

namespace mphy {
namespace {

constexpr int kWarps = 4;

__device__ __forceinline__ int64_t find_in_row(const int32_t* col, int64_t lo, int64_t hi, int32_t key) {
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (col[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// lower row length of every node: its neighbours up to and including itself, capped
__global__ void lower_counts(int32_t n_node, const int64_t* __restrict__ browp, const int32_t* __restrict__ bcol,
                             int max_lower, int32_t* __restrict__ lc, int64_t* __restrict__ diagpos) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = find_in_row(bcol, browp[n], browp[n + 1], (int32_t)n);
        diagpos[n] = p;
        const int64_t c = p - browp[n] + 1;
        lc[n] = (int32_t)(c < max_lower ? c : max_lower);
    }
}

__global__ void lower_fill(int32_t n_node, const int64_t* __restrict__ diagpos, const int32_t* __restrict__ bcol,
                           const int64_t* __restrict__ lrow, int32_t* __restrict__ lcol, int32_t* __restrict__ ucnt) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = lrow[n + 1] - lrow[n];
        for (int64_t k = 0; k < c; ++k) {
            const int32_t m = bcol[diagpos[n] - (c - 1) + k];
            lcol[lrow[n] + k] = m;
            atomicAdd(&ucnt[m], 1);
        }
    }
}

// upper rows as the transpose of the lower rows: (n, m) lower -> (m, n) upper
__global__ void upper_fill(int32_t n_node, const int64_t* __restrict__ lrow, const int32_t* __restrict__ lcol,
                           const int64_t* __restrict__ urow, int32_t* __restrict__ cursor, int32_t* __restrict__ ucol) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        for (int64_t k = lrow[n]; k < lrow[n + 1]; ++k) {
            const int32_t m = lcol[k];
            const int32_t slot = atomicAdd(&cursor[m], 1);
            ucol[urow[m] + slot] = (int32_t)n;
        }
    }
}

__global__ void sort_rows(int32_t n_node, const int64_t* __restrict__ row, int32_t* __restrict__ col) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = row[n], e = row[n + 1];
        for (int64_t i = b + 1; i < e; ++i) {  // insertion sort: rows hold at most a few dozen entries
            const int32_t v = col[i];
            int64_t j = i - 1;
            while (j >= b && col[j] > v) {
                col[j + 1] = col[j];
                --j;
            }
            col[j + 1] = v;
        }
    }
}

__global__ void row_lengths(int32_t n_node, const int64_t* __restrict__ row, int32_t* __restrict__ len) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x)
        len[n] = (int32_t)(row[n + 1] - row[n]);
}

__global__ void slice_widths_k(const int32_t* __restrict__ len, int32_t n_node, int32_t n_slices,
                               int32_t* __restrict__ width, int64_t* __restrict__ width32) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < n_slices; s += (int64_t)gridDim.x * blockDim.x) {
        int w = 0;
        for (int l = 0; l < 32; ++l) {
            const int64_t n = s * 32 + l;
            if (n < n_node) w = max(w, len[n]);
        }
        width[s] = w;
        width32[s] = 32 * (int64_t)w;
    }
}

__global__ void sell_fill(int32_t n_node, int32_t n_slices, const int64_t* __restrict__ row,
                          const int32_t* __restrict__ col, const int64_t* __restrict__ sbase,
                          const int32_t* __restrict__ swidth, int32_t* __restrict__ scol) {
    const int64_t rows = (int64_t)n_slices * 32;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = r >> 5;
        const int ln = (int)(r & 31);
        const int w = swidth[s];
        const int64_t b = r < n_node ? row[r] : 0, c = r < n_node ? row[r + 1] - row[r] : 0;
        for (int k = 0; k < w; ++k)
            scol[sbase[s] + 32 * (int64_t)k + ln] = k < c ? col[b + k] : (r < n_node ? (int32_t)r : 0);
    }
}

// value offsets: lower block j -> G SELL; lower block (n, m) -> G^T SELL position of (m, n)
__global__ void lower_maps(int32_t n_node, const int64_t* __restrict__ lrow, const int32_t* __restrict__ lcol,
                           const int64_t* __restrict__ lsb, const int64_t* __restrict__ urow,
                           const int32_t* __restrict__ ucol, const int64_t* __restrict__ usb,
                           int64_t* __restrict__ l2s, int64_t* __restrict__ l2u) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        for (int64_t j = lrow[n]; j < lrow[n + 1]; ++j) {
            const int64_t k = j - lrow[n];
            l2s[j] = 9 * (lsb[n >> 5] + 32 * k) + (n & 31);
            const int32_t m = lcol[j];
            const int64_t q = find_in_row(ucol, urow[m], urow[m + 1], (int32_t)n) - urow[m];
            l2u[j] = 9 * (usb[m >> 5] + 32 * q) + (m & 31);
        }
    }
}

void build_sell(SellPattern& P, int32_t n_node, cudaStream_t s, int sm) {
    P.n_node = n_node;
    P.n_slices = (n_node + 31) / 32;
    DevBuf<int32_t> len(n_node);
    DevBuf<int64_t> w32(P.n_slices);
    P.slice_width.alloc(P.n_slices);
    P.slice_base.alloc(P.n_slices + 1);
    row_lengths<<<stride_grid(n_node, 256, sm), 256, 0, s>>>(n_node, P.rowptr.p, len.p);
    slice_widths_k<<<stride_grid(P.n_slices, 256, sm), 256, 0, s>>>(len.p, n_node, P.n_slices, P.slice_width.p, w32.p);
    P.stored_blocks = exclusive_scan<int64_t>(w32.p, P.slice_base.p, P.n_slices, s);
    P.sell_col.alloc(P.stored_blocks > 0 ? P.stored_blocks : 1);
    sell_fill<<<stride_grid((int64_t)P.n_slices * 32, 256, sm), 256, 0, s>>>(
        n_node, P.n_slices, P.rowptr.p, P.col.p, P.slice_base.p, P.slice_width.p, P.sell_col.p);
    MPHY_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------- setup: one warp per block row
template <typename VT>
struct SetupArgs {
    int32_t n_node;
    int max_lower;
    const int64_t* lrow;
    const int32_t* lcol;
    const int64_t* l2s;
    const int64_t* l2u;
    // A
    const int64_t* abrow;
    const int32_t* abcol;
    const int64_t* aslice;
    const VT* aval;
    const double* diag64;  // mixed storage: FP64 diagonal blocks
    const uint8_t* fixed;  // mixed storage: prescribed DOFs are identity rows / zero columns
    FactorT* gval;
    FactorT* gtval;
    int32_t* nfail;
};

template <typename VT>
__device__ __forceinline__ double a_block_entry(const SetupArgs<VT>& a, int32_t m1, int32_t m2, int v) {
    if (a.fixed && (a.fixed[3 * (int64_t)m1 + v / 3] || a.fixed[3 * (int64_t)m2 + v % 3]))
        return (m1 == m2 && v / 3 == v % 3) ? 1.0 : 0.0;
    if (a.diag64 && m1 == m2) return a.diag64[9 * (int64_t)m1 + v];
    const int64_t b = a.abrow[m1], e = a.abrow[m1 + 1];
    const int64_t q = find_in_row(a.abcol, b, e, m2);
    if (q >= e || a.abcol[q] != m2) return 0.0;
    return (double)a.aval[9 * (a.aslice[m1 >> 5] + 32 * (q - b)) + (m1 & 31) + 32 * v];
}

template <typename VT>
__global__ void __launch_bounds__(kWarps * 32) fsai_setup_kernel(SetupArgs<VT> a) {
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int NMAX = 3 * a.max_lower;
    double* M = smem + (size_t)warp * (NMAX * NMAX + 6 * NMAX + 16);
    double* Y = M + NMAX * NMAX;   // [NMAX][3]
    double* Gr = Y + 3 * NMAX;     // [3][NMAX]
    double* sm = Gr + 3 * NMAX;    // 16 scratch values
    for (int64_t n = (int64_t)blockIdx.x * kWarps + warp; n < a.n_node; n += (int64_t)gridDim.x * kWarps) {
        const int64_t r0 = a.lrow[n];
        const int p = (int)(a.lrow[n + 1] - r0);
        const int N = 3 * p;
        // gather A[P,P] (symmetric: fill the lower triangle, i >= j)
        for (int t = lane; t < p * p; t += 32) {
            const int k1 = t / p, k2 = t % p;
            if (k1 < k2) continue;
            const int32_t m1 = a.lcol[r0 + k1], m2 = a.lcol[r0 + k2];
            for (int aa = 0; aa < 3; ++aa)
                for (int bb = 0; bb < 3; ++bb) {
                    const int i = 3 * k1 + aa, j = 3 * k2 + bb;
                    if (i >= j) M[i * NMAX + j] = a_block_entry(a, m1, m2, 3 * aa + bb);
                }
        }
        __syncwarp();
        // Cholesky, lower triangle in place
        bool ok = true;
        for (int k = 0; k < N; ++k) {
            const double d = M[k * NMAX + k];
            if (!(d > 0.0)) {
                ok = false;
                break;
            }
            const double l = sqrt(d);
            __syncwarp();
            if (lane == 0) M[k * NMAX + k] = l;
            for (int i = k + 1 + lane; i < N; i += 32) M[i * NMAX + k] /= l;
            __syncwarp();
            const int rem = N - k - 1;
            for (int t = lane; t < rem * rem; t += 32) {
                const int i = k + 1 + t / rem, j = k + 1 + t % rem;
                if (j <= i) M[i * NMAX + j] -= M[i * NMAX + k] * M[j * NMAX + k];
            }
            __syncwarp();
        }
        ok = __all_sync(0xffffffffu, ok);
        if (ok) {
            // Z = L^{-1} E_n is zero above the last three rows; Y = L^{-T} Z by back substitution
            if (lane < 3) {
                const int c = lane;
                double z[3];
                for (int r = 0; r < 3; ++r) {
                    const int i = N - 3 + r;
                    double s = (r == c) ? 1.0 : 0.0;
                    for (int q = 0; q < r; ++q) s -= M[i * NMAX + (N - 3 + q)] * z[q];
                    z[r] = s / M[i * NMAX + i];
                }
                for (int i = N - 1; i >= 0; --i) {
                    double s = i >= N - 3 ? z[i - (N - 3)] : 0.0;
                    for (int j = i + 1; j < N; ++j) s -= M[j * NMAX + i] * Y[j * 3 + c];
                    Y[i * 3 + c] = s / M[i * NMAX + i];
                }
            }
            __syncwarp();
            if (lane == 0) {
                // Y_nn = Ln Ln^T (3x3 Cholesky), then W = Ln^{-1}
                double Ynn[3][3], Lc[3][3] = {{0}}, W[3][3] = {{0}};
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) Ynn[i][j] = 0.5 * (Y[(N - 3 + i) * 3 + j] + Y[(N - 3 + j) * 3 + i]);
                bool pd = true;
                for (int j = 0; j < 3; ++j) {
                    double s = Ynn[j][j];
                    for (int k = 0; k < j; ++k) s -= Lc[j][k] * Lc[j][k];
                    if (!(s > 0.0)) pd = false;
                    Lc[j][j] = sqrt(fmax(s, 1e-300));
                    for (int i = j + 1; i < 3; ++i) {
                        double t = Ynn[i][j];
                        for (int k = 0; k < j; ++k) t -= Lc[i][k] * Lc[j][k];
                        Lc[i][j] = t / Lc[j][j];
                    }
                }
                for (int c = 0; c < 3; ++c)
                    for (int i = 0; i < 3; ++i) {
                        double s = (i == c) ? 1.0 : 0.0;
                        for (int k = 0; k < i; ++k) s -= Lc[i][k] * W[k][c];
                        W[i][c] = s / Lc[i][i];
                    }
                for (int i = 0; i < 9; ++i) sm[i] = W[i / 3][i % 3];
                sm[9] = pd ? 1.0 : 0.0;
            }
            __syncwarp();
            ok = sm[9] != 0.0;
            if (ok) {
                for (int t = lane; t < 3 * N; t += 32) {
                    const int r = t / N, j = t % N;
                    Gr[r * NMAX + j] = sm[3 * r] * Y[j * 3] + sm[3 * r + 1] * Y[j * 3 + 1] + sm[3 * r + 2] * Y[j * 3 + 2];
                }
            }
            __syncwarp();
        }
        if (!ok) {
            // fallback row: zero off-diagonal blocks, diagonal 1/sqrt(|a_ii|)
            if (lane == 0) atomicAdd(a.nfail, 1);
            for (int t = lane; t < 3 * N; t += 32) {
                const int r = t / N, j = t % N;
                double v = 0.0;
                if (j == N - 3 + r) {
                    const double d = fabs(a_block_entry(a, (int32_t)n, (int32_t)n, 4 * r));
                    v = d > 0.0 ? 1.0 / sqrt(d) : 1.0;
                }
                Gr[r * NMAX + j] = v;
            }
            __syncwarp();
        }
        // write G[n, m_k] and G^T[m_k, n]
        for (int t = lane; t < 9 * p; t += 32) {
            const int k = t / 9, v = t % 9, r = v / 3, c = v % 3;
            const float g = (float)Gr[r * NMAX + 3 * k + c];
            a.gval[a.l2s[r0 + k] + 32 * (3 * r + c)] = __float2bfloat16_rn((float)g);
            a.gtval[a.l2u[r0 + k] + 32 * (3 * c + r)] = __float2bfloat16_rn((float)g);
        }
        __syncwarp();
    }
}

__global__ void set_lower_kernel(int64_t n_lower, const float* __restrict__ blocks, const int64_t* __restrict__ l2s,
                                 const int64_t* __restrict__ l2u, FactorT* __restrict__ gval, FactorT* __restrict__ gtval) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 9 * n_lower; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / 9;
        const int v = (int)(t % 9), r = v / 3, c = v % 3;
        const float g = blocks[t];
        gval[l2s[j] + 32 * (3 * r + c)] = __float2bfloat16_rn(g);
        gtval[l2u[j] + 32 * (3 * c + r)] = __float2bfloat16_rn(g);
    }
}

__global__ void get_lower_kernel(int64_t n_lower, const FactorT* __restrict__ gval, const int64_t* __restrict__ l2s,
                                 float* __restrict__ out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 9 * n_lower; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / 9;
        const int v = (int)(t % 9);
        out[t] = __bfloat162float(gval[l2s[j] + 32 * v]);
    }
}

}  // namespace

void Fsai::init(mphy_ctx* ctx, const mphy_pattern* A, int max_lower) {
    ctx_ = ctx;
    A_ = A;
    max_lower_ = max_lower;
    cudaStream_t s = ctx->stream;
    const int sm = ctx->sm_count;
    const int32_t nn = A->n_node;
    DevBuf<int32_t> lc(nn), ucnt(nn), cursor(nn);
    DevBuf<int64_t> diagpos(nn);
    lower_counts<<<stride_grid(nn, 256, sm), 256, 0, s>>>(nn, A->brow_ptr.p, A->bcol.p, max_lower, lc.p, diagpos.p);
    L_.rowptr.alloc(nn + 1);
    L_.n_blocks = exclusive_scan<int32_t>(lc.p, L_.rowptr.p, nn, s);
    L_.col.alloc(L_.n_blocks);
    MPHY_CUDA(cudaMemsetAsync(ucnt.p, 0, ucnt.bytes(), s));
    lower_fill<<<stride_grid(nn, 256, sm), 256, 0, s>>>(nn, diagpos.p, A->bcol.p, L_.rowptr.p, L_.col.p, ucnt.p);
    U_.rowptr.alloc(nn + 1);
    U_.n_blocks = exclusive_scan<int32_t>(ucnt.p, U_.rowptr.p, nn, s);
    U_.col.alloc(U_.n_blocks);
    MPHY_CUDA(cudaMemsetAsync(cursor.p, 0, cursor.bytes(), s));
    upper_fill<<<stride_grid(nn, 256, sm), 256, 0, s>>>(nn, L_.rowptr.p, L_.col.p, U_.rowptr.p, cursor.p, U_.col.p);
    sort_rows<<<stride_grid(nn, 256, sm), 256, 0, s>>>(nn, U_.rowptr.p, U_.col.p);
    MPHY_CUDA(cudaGetLastError());
    build_sell(L_, nn, s, sm);
    build_sell(U_, nn, s, sm);
    MPHY_REQUIRE(9 * L_.stored_blocks < (int64_t)UINT32_MAX && 9 * U_.stored_blocks < (int64_t)UINT32_MAX,
                 MPHY_ERR_UNSUPPORTED, "preconditioner too large for 32-bit value offsets");
    l2sell_.alloc(L_.n_blocks);
    l2usell_.alloc(L_.n_blocks);
    lower_maps<<<stride_grid(nn, 256, sm), 256, 0, s>>>(nn, L_.rowptr.p, L_.col.p, L_.slice_base.p, U_.rowptr.p,
                                                        U_.col.p, U_.slice_base.p, l2sell_.p, l2usell_.p);
    gval_.alloc(9 * (size_t)L_.stored_blocks);
    gtval_.alloc(9 * (size_t)U_.stored_blocks);
    MPHY_CUDA(cudaMemsetAsync(gval_.p, 0, gval_.bytes(), s));
    MPHY_CUDA(cudaMemsetAsync(gtval_.p, 0, gtval_.bytes(), s));
    err_.alloc(1);
    MPHY_CUDA(cudaStreamSynchronize(s));
}

template <typename VT>
void Fsai::compute(const VT* aval, const double* diag64, const uint8_t* fixed, cudaStream_t s) {
    SetupArgs<VT> a{};
    a.n_node = A_->n_node;
    a.max_lower = max_lower_;
    a.lrow = L_.rowptr.p;
    a.lcol = L_.col.p;
    a.l2s = l2sell_.p;
    a.l2u = l2usell_.p;
    a.abrow = A_->brow_ptr.p;
    a.abcol = A_->bcol.p;
    a.aslice = A_->slice_base.p;
    a.aval = aval;
    a.diag64 = diag64;
    a.fixed = fixed;
    a.gval = gval_.p;
    a.gtval = gtval_.p;
    a.nfail = err_.p;
    const int NMAX = 3 * max_lower_;
    const size_t smem = (size_t)kWarps * (NMAX * NMAX + 6 * NMAX + 16) * sizeof(double);
    MPHY_CUDA(cudaFuncSetAttribute(fsai_setup_kernel<VT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MPHY_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int32_t), s));
    const unsigned grid = stride_grid((int64_t)A_->n_node * 32, kWarps * 32, ctx_->sm_count, 4);
    fsai_setup_kernel<VT><<<grid, kWarps * 32, smem, s>>>(a);
    MPHY_CUDA(cudaGetLastError());
    launches = 1;
}

template void Fsai::compute<double>(const double*, const double*, const uint8_t*, cudaStream_t);
template void Fsai::compute<float>(const float*, const double*, const uint8_t*, cudaStream_t);

void Fsai::set_lower_values(const float* gblocks, cudaStream_t s) {
    set_lower_kernel<<<stride_grid(9 * L_.n_blocks, 256, ctx_->sm_count), 256, 0, s>>>(L_.n_blocks, gblocks,
                                                                                       l2sell_.p, l2usell_.p,
                                                                                       gval_.p, gtval_.p);
    MPHY_CUDA(cudaGetLastError());
}

void Fsai::get_lower_values(float* out, cudaStream_t s) const {
    get_lower_kernel<<<stride_grid(9 * L_.n_blocks, 256, ctx_->sm_count), 256, 0, s>>>(L_.n_blocks, gval_.p,
                                                                                       l2sell_.p, out);
    MPHY_CUDA(cudaGetLastError());
}

int32_t Fsai::fallback_rows(cudaStream_t s) const {
    int32_t h = 0;
    MPHY_CUDA(cudaMemcpyAsync(&h, err_.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    MPHY_CUDA(cudaStreamSynchronize(s));
    return h;
}

FactorView<FactorT> Fsai::view() const {
    FactorView<FactorT> f;
    f.G = L_.view();
    f.GT = U_.view();
    f.gval = gval_.p;
    f.gtval = gtval_.p;
    return f;
}

}  // namespace mphy
