// pattern.cu -- K2: DOF map and sparsity pattern on the device.
//
// Replaces femSolidmechanics::prepareMatrixPattern (femSolidmechanics2.cpp:121-478). The
// reference pushes, for every element, every free column into every free row
// (vector<vector<int>>, 576 pushes per hex8) and then sorts and uniquifies each row. Here the
// same set is built per node: the nodes that share an element with node n, found through a
// node -> element incidence list, sorted and uniquified by one warp in shared memory. Because
// free DOFs are numbered node-major (:142-152), the reference's scalar CSR row of DOF (n, a)
// is exactly the free DOFs of those nodes in ascending node order, so the exported CSR is
// bit-identical to the reference's pattern.
#include <climits>

#include "common.cuh"
#include "pattern.cuh"

namespace mphy {

// ------------------------------------------------------------------ exclusive scan (int64)
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__global__ void scan_tiles(const T* __restrict__ in, int64_t* __restrict__ out, int64_t n,
                           int64_t* __restrict__ tile_sums) {
    __shared__ int64_t warp_tot[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int64_t v[kScanItems];
    int64_t run = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const int64_t idx = base + i;
        v[i] = idx < n ? (int64_t)in[idx] : 0;
        run += v[i];
    }
    // warp inclusive scan of per-thread totals
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < kScanThreads / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < kScanThreads / 32) warp_tot[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    int64_t excl = incl - run + (warp > 0 ? warp_tot[warp - 1] : 0);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const int64_t idx = base + i;
        if (idx < n) out[idx] = excl;
        excl += v[i];
    }
    if (threadIdx.x == kScanThreads - 1) tile_sums[blockIdx.x] = excl;
}

__global__ void scan_add(int64_t* __restrict__ out, int64_t n, const int64_t* __restrict__ tile_off) {
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    const int64_t add = tile_off[blockIdx.x];
    for (int i = threadIdx.x; i < kScanTile; i += blockDim.x) {
        const int64_t idx = base + i;
        if (idx < n) out[idx] += add;
    }
}

__global__ void write_total(const int64_t* __restrict__ scanned_last, const int64_t* __restrict__ last_in,
                            int64_t* __restrict__ total) {
    *total = *scanned_last + *last_in;
}

}  // namespace

template <typename T>
int64_t exclusive_scan(const T* in, int64_t* out, int64_t n, cudaStream_t s) {
    // out has n+1 entries; out[n] = total. Returns the total (synchronous read-back).
    if (n == 0) {
        MPHY_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
        return 0;
    }
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    DevBuf<int64_t> sums(tiles + 1);
    scan_tiles<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, sums.p);
    MPHY_CUDA(cudaGetLastError());
    if (tiles > 1) {
        DevBuf<int64_t> sums_scan(tiles + 1);
        exclusive_scan<int64_t>(sums.p, sums_scan.p, tiles, s);
        scan_add<<<(unsigned)tiles, kScanThreads, 0, s>>>(out, n, sums_scan.p);
        MPHY_CUDA(cudaGetLastError());
        MPHY_CUDA(cudaMemcpyAsync(out + n, sums_scan.p + tiles, sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
        int64_t total = 0;
        MPHY_CUDA(cudaMemcpyAsync(&total, out + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        MPHY_CUDA(cudaStreamSynchronize(s));
        return total;
    }
    MPHY_CUDA(cudaMemcpyAsync(out + n, sums.p, sizeof(int64_t), cudaMemcpyDeviceToDevice, s));
    int64_t total = 0;
    MPHY_CUDA(cudaMemcpyAsync(&total, out + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    MPHY_CUDA(cudaStreamSynchronize(s));
    return total;
}

template int64_t exclusive_scan<int32_t>(const int32_t*, int64_t*, int64_t, cudaStream_t);
template int64_t exclusive_scan<int64_t>(const int64_t*, int64_t*, int64_t, cudaStream_t);
template int64_t exclusive_scan<uint8_t>(const uint8_t*, int64_t*, int64_t, cudaStream_t);

// ------------------------------------------------------------------ incidence
namespace {

__global__ void count_incidence(const int32_t* __restrict__ conn, int64_t n_entries, int32_t n_node,
                                int32_t* __restrict__ cnt, int32_t* __restrict__ err) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_entries;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t n = conn[i];
        if (n < 0 || n >= n_node) {
            atomicExch(err, 1);
            continue;
        }
        atomicAdd(&cnt[n], 1);
    }
}

__global__ void fill_incidence(const int32_t* __restrict__ conn, int64_t n_entries, int32_t npe,
                               const int64_t* __restrict__ ptr, int32_t* __restrict__ cursor,
                               int32_t* __restrict__ n2e) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_entries;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t n = conn[i];
        const int32_t slot = atomicAdd(&cursor[n], 1);
        n2e[ptr[n] + slot] = (int32_t)(i / npe);
    }
}

// One warp per node: gather the nodes of every incident element, bitonic-sort them in shared
// memory and keep the distinct ones. kMaxCand bounds the candidates (incident elements x npe);
// hex8 meshes need at most 64, the Kuhn tet10 split at most 240.
constexpr int kMaxCand = 512;
constexpr int kNbrWarps = 4;

// mode 0: count distinct neighbours into rlen; mode 1: write them into bcol / sell_col.
template <int MODE>
__global__ void __launch_bounds__(kNbrWarps * 32)
node_neighbours(int32_t n_node, int32_t npe, const int32_t* __restrict__ conn,
                const int64_t* __restrict__ n2e_ptr, const int32_t* __restrict__ n2e,
                int32_t* __restrict__ rlen, const int64_t* __restrict__ brow_ptr,
                int32_t* __restrict__ bcol, const int64_t* __restrict__ slice_base,
                const int32_t* __restrict__ slice_width, int32_t* __restrict__ sell_col,
                uint32_t* __restrict__ dvoff, int32_t* __restrict__ err) {
    __shared__ int32_t keys[kNbrWarps][kMaxCand];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int32_t* k = keys[warp];
    for (int64_t n = (int64_t)blockIdx.x * kNbrWarps + warp; n < n_node;
         n += (int64_t)gridDim.x * kNbrWarps) {
        const int64_t e0 = n2e_ptr[n];
        const int ne = (int)(n2e_ptr[n + 1] - e0);
        const int ncand = ne * npe;
        if (ncand > kMaxCand) {
            if (lane == 0) atomicExch(err, 2);
            continue;
        }
        int S = 32;
        while (S < ncand) S <<= 1;
        for (int i = lane; i < S; i += 32)
            k[i] = i < ncand ? conn[(int64_t)n2e[e0 + i / npe] * npe + i % npe] : INT_MAX;
        __syncwarp();
        for (int sz = 2; sz <= S; sz <<= 1) {
            for (int j = sz >> 1; j > 0; j >>= 1) {
                for (int i = lane; i < S; i += 32) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const int32_t a = k[i], b = k[ixj];
                        const bool up = (i & sz) == 0;
                        if ((a > b) == up) {
                            k[i] = b;
                            k[ixj] = a;
                        }
                    }
                }
                __syncwarp();
            }
        }
        // distinct values in ascending order
        int count = 0;
        const int64_t rb = MODE == 1 ? brow_ptr[n] : 0;
        const int64_t s = n >> 5;
        const int64_t sb = MODE == 1 ? slice_base[s] : 0;
        const int ln = (int)(n & 31);
        for (int c = 0; c < S; c += 32) {
            const int i = c + lane;
            const int32_t v = k[i];
            const bool keep = v != INT_MAX && (i == 0 || v != k[i - 1]);
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (MODE == 1 && keep) {
                const int pos = count + __popc(m & ((1u << lane) - 1u));
                bcol[rb + pos] = v;
                sell_col[sb + 32 * (int64_t)pos + ln] = v;
                if (v == (int32_t)n) dvoff[n] = (uint32_t)(9 * (sb + 32 * (int64_t)pos) + ln);
            }
            count += __popc(m);
        }
        if (MODE == 0) {
            if (lane == 0) rlen[n] = count;
        } else {
            // padding blocks of this row: own column, zero values
            const int w = slice_width[s];
            for (int pos = count + lane; pos < w; pos += 32) sell_col[sb + 32 * (int64_t)pos + ln] = (int32_t)n;
        }
        __syncwarp();
    }
}

__global__ void slice_widths(const int32_t* __restrict__ rlen, int32_t n_node, int32_t n_slices,
                             int32_t* __restrict__ width, int64_t* __restrict__ width32) {
    const int lane = threadIdx.x & 31;
    for (int64_t s = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; s < n_slices;
         s += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int64_t n = s * 32 + lane;
        int w = n < n_node ? rlen[n] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w = max(w, __shfl_xor_sync(0xffffffffu, w, o));
        if (lane == 0) {
            width[s] = w;
            width32[s] = 32 * (int64_t)w;
        }
    }
}

// Rows of the last, partial slice that do not exist: every column slot points at node 0 with
// zero values (the SpMV kernel skips rows >= n_node anyway).
__global__ void pad_missing_rows(int32_t n_node, int32_t n_slices, const int64_t* __restrict__ slice_base,
                                 const int32_t* __restrict__ slice_width, int32_t* __restrict__ sell_col) {
    const int64_t s = n_slices - 1;
    const int w = slice_width[s];
    for (int i = threadIdx.x; i < 32 * w; i += blockDim.x) {
        const int ln = i & 31;
        if (s * 32 + ln >= n_node) sell_col[slice_base[s] + i] = 0;
    }
}

// value offset of every element block (I, J): binary search of node J in node I's row
__global__ void element_block_offsets(int32_t n_elem, int32_t npe, const int32_t* __restrict__ conn,
                                      const int64_t* __restrict__ brow_ptr, const int32_t* __restrict__ bcol,
                                      const int64_t* __restrict__ slice_base, uint32_t* __restrict__ e2v,
                                      int32_t* __restrict__ err) {
    const int64_t total = (int64_t)n_elem * npe * npe;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / (npe * npe);
        const int r = (int)(t % (npe * npe));
        const int32_t ni = conn[e * npe + r / npe], nj = conn[e * npe + r % npe];
        int64_t lo = brow_ptr[ni], hi = brow_ptr[ni + 1];
        const int64_t first = lo;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (bcol[mid] < nj) lo = mid + 1;
            else hi = mid;
        }
        if (lo >= brow_ptr[ni + 1] || bcol[lo] != nj) {
            atomicExch(err, 3);
            continue;
        }
        const int64_t kpos = lo - first;
        e2v[t] = (uint32_t)(9 * (slice_base[ni >> 5] + 32 * kpos) + (ni & 31));
    }
}

__global__ void free_flags(const uint8_t* __restrict__ fixed, int64_t n, uint8_t* __restrict__ isfree) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        isfree[i] = fixed[i] ? 0 : 1;
}

__global__ void number_dofs(const uint8_t* __restrict__ fixed, const int64_t* __restrict__ scan, int64_t n,
                            int32_t* __restrict__ node_dof, int32_t* __restrict__ assy) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (fixed[i]) {
            node_dof[i] = -1;
        } else {
            node_dof[i] = (int32_t)scan[i];
            assy[scan[i]] = (int32_t)i;
        }
    }
}

// reference CSR row length of every free DOF: free DOFs of all neighbour nodes
__global__ void csr_row_lengths(int32_t n_node, const int64_t* __restrict__ brow_ptr,
                                const int32_t* __restrict__ bcol, const uint8_t* __restrict__ fixed,
                                const int32_t* __restrict__ node_dof, int64_t* __restrict__ len) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        int64_t c = 0;
        for (int64_t k = brow_ptr[n]; k < brow_ptr[n + 1]; ++k) {
            const int32_t m = bcol[k];
            c += 3 - (fixed[3 * m] + fixed[3 * m + 1] + fixed[3 * m + 2]);
        }
        for (int a = 0; a < 3; ++a) {
            const int32_t r = node_dof[3 * n + a];
            if (r >= 0) len[r] = c;
        }
    }
}

__global__ void csr_fill(int32_t n_node, const int64_t* __restrict__ brow_ptr, const int32_t* __restrict__ bcol,
                         const int64_t* __restrict__ slice_base, const int32_t* __restrict__ node_dof,
                         const int64_t* __restrict__ rowptr, int32_t* __restrict__ col, int64_t* __restrict__ src) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < 3 * (int64_t)n_node;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = t / 3;
        const int a = (int)(t % 3);
        const int32_t r = node_dof[t];
        if (r < 0) continue;
        int64_t pos = rowptr[r];
        const int64_t sb = slice_base[n >> 5];
        const int ln = (int)(n & 31);
        for (int64_t k = brow_ptr[n]; k < brow_ptr[n + 1]; ++k) {
            const int32_t m = bcol[k];
            const int64_t kpos = k - brow_ptr[n];
            for (int b = 0; b < 3; ++b) {
                const int32_t c = node_dof[3 * m + b];
                if (c < 0) continue;
                col[pos] = c;
                if (src) src[pos] = 9 * (sb + 32 * kpos) + ln + 32 * (3 * a + b);
                ++pos;
            }
        }
    }
}

__global__ void elem_dofs(int32_t n_elem, int32_t npe, const int32_t* __restrict__ conn,
                          const int32_t* __restrict__ node_dof, int32_t* __restrict__ fav) {
    const int64_t total = (int64_t)n_elem * npe * 3;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e = t / (3 * npe);
        const int r = (int)(t % (3 * npe));
        fav[t] = node_dof[3 * (int64_t)conn[e * npe + r / 3] + r % 3];
    }
}

unsigned grid_for(int64_t n, int threads, int sm_count) {
    const int64_t want = (n + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count * 16;
    return (unsigned)(want < 1 ? 1 : (want > cap ? cap : want));
}

void check_err(const DevBuf<int32_t>& err, cudaStream_t s) {
    int32_t h = 0;
    MPHY_CUDA(cudaMemcpyAsync(&h, err.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    MPHY_CUDA(cudaStreamSynchronize(s));
    MPHY_REQUIRE(h != 1, MPHY_ERR_INVALID_ARG, "connectivity references a node id outside [0, n_node)");
    MPHY_REQUIRE(h != 2, MPHY_ERR_UNSUPPORTED, "a node is shared by more than 512/npe elements");
    MPHY_REQUIRE(h != 3, MPHY_ERR_CUDA, "internal: element block missing from its row");
}

}  // namespace

void build_pattern(mphy_ctx* ctx, const mphy_mesh* mesh, mphy_pattern* P) {
    cudaStream_t s = ctx->stream;
    const int sm = ctx->sm_count;
    const int32_t nn = mesh->n_node, ne = mesh->n_elem, npe = mesh->npe;
    P->ctx = ctx;
    P->mesh = mesh;
    P->device = ctx->device;
    P->n_node = nn;
    P->n_elem = ne;
    P->npe = npe;
    const int64_t nent = (int64_t)ne * npe;
    DevBuf<int32_t> err(1);
    MPHY_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int32_t), s));

    // node -> element incidence
    DevBuf<int32_t> cnt(nn), cursor(nn), n2e(nent), rlen(nn);
    DevBuf<int64_t> n2e_ptr(nn + 1);
    MPHY_CUDA(cudaMemsetAsync(cnt.p, 0, cnt.bytes(), s));
    MPHY_CUDA(cudaMemsetAsync(cursor.p, 0, cursor.bytes(), s));
    count_incidence<<<grid_for(nent, 256, sm), 256, 0, s>>>(mesh->conn.p, nent, nn, cnt.p, err.p);
    check_err(err, s);
    exclusive_scan<int32_t>(cnt.p, n2e_ptr.p, nn, s);
    fill_incidence<<<grid_for(nent, 256, sm), 256, 0, s>>>(mesh->conn.p, nent, npe, n2e_ptr.p, cursor.p, n2e.p);
    MPHY_CUDA(cudaGetLastError());

    // pass 1: row lengths
    const unsigned nb_grid = grid_for((int64_t)nn * 32, kNbrWarps * 32, sm);
    node_neighbours<0><<<nb_grid, kNbrWarps * 32, 0, s>>>(nn, npe, mesh->conn.p, n2e_ptr.p, n2e.p, rlen.p, nullptr,
                                                          nullptr, nullptr, nullptr, nullptr, nullptr, err.p);
    check_err(err, s);
    P->brow_ptr.alloc(nn + 1);
    P->n_blocks = exclusive_scan<int32_t>(rlen.p, P->brow_ptr.p, nn, s);

    // SELL slices
    P->n_slices = (nn + 31) / 32;
    P->slice_width.alloc(P->n_slices);
    P->slice_base.alloc(P->n_slices + 1);
    DevBuf<int64_t> w32(P->n_slices);
    slice_widths<<<grid_for((int64_t)P->n_slices * 32, 256, sm), 256, 0, s>>>(rlen.p, nn, P->n_slices,
                                                                             P->slice_width.p, w32.p);
    P->sell_blocks = exclusive_scan<int64_t>(w32.p, P->slice_base.p, P->n_slices, s);
    MPHY_REQUIRE(9 * P->sell_blocks < (int64_t)UINT32_MAX, MPHY_ERR_UNSUPPORTED,
                 "matrix too large for 32-bit value offsets");

    // pass 2: columns
    P->bcol.alloc(P->n_blocks);
    P->sell_col.alloc(P->sell_blocks);
    P->dvoff.alloc(nn);
    // a node that no element touches has no diagonal block: its offset stays UINT32_MAX
    MPHY_CUDA(cudaMemsetAsync(P->dvoff.p, 0xff, P->dvoff.bytes(), s));
    node_neighbours<1><<<nb_grid, kNbrWarps * 32, 0, s>>>(nn, npe, mesh->conn.p, n2e_ptr.p, n2e.p, rlen.p,
                                                          P->brow_ptr.p, P->bcol.p, P->slice_base.p,
                                                          P->slice_width.p, P->sell_col.p, P->dvoff.p, err.p);
    pad_missing_rows<<<1, 256, 0, s>>>(nn, P->n_slices, P->slice_base.p, P->slice_width.p, P->sell_col.p);
    check_err(err, s);


    // element block offsets
    P->e2v.alloc((size_t)ne * npe * npe);
    element_block_offsets<<<grid_for((int64_t)ne * npe * npe, 256, sm), 256, 0, s>>>(
        ne, npe, mesh->conn.p, P->brow_ptr.p, P->bcol.p, P->slice_base.p, P->e2v.p, err.p);
    check_err(err, s);

    // free DOF numbering (NodeDofArray / assyForSoln)
    const int64_t nd = 3 * (int64_t)nn;
    DevBuf<uint8_t> isfree(nd);
    DevBuf<int64_t> fscan(nd + 1);
    free_flags<<<grid_for(nd, 256, sm), 256, 0, s>>>(mesh->fixed.p, nd, isfree.p);
    P->n_free = (int32_t)exclusive_scan<uint8_t>(isfree.p, fscan.p, nd, s);
    P->node_dof.alloc(nd);
    P->assy_for_soln.alloc(P->n_free > 0 ? P->n_free : 1);
    number_dofs<<<grid_for(nd, 256, sm), 256, 0, s>>>(mesh->fixed.p, fscan.p, nd, P->node_dof.p, P->assy_for_soln.p);

    // reference CSR row pointer (columns are materialised on export)
    DevBuf<int64_t> len(P->n_free > 0 ? P->n_free : 1);
    csr_row_lengths<<<grid_for(nn, 256, sm), 256, 0, s>>>(nn, P->brow_ptr.p, P->bcol.p, mesh->fixed.p,
                                                          P->node_dof.p, len.p);
    P->csr_rowptr.alloc(P->n_free + 1);
    P->nnz = exclusive_scan<int64_t>(len.p, P->csr_rowptr.p, P->n_free, s);
    MPHY_CUDA(cudaStreamSynchronize(s));
}

void pattern_csr_columns(mphy_pattern* P, bool with_src) {
    cudaStream_t s = P->ctx->stream;
    if (!P->csr_col.p && P->nnz > 0) P->csr_col.alloc(P->nnz);
    if (with_src && !P->csr_src.p && P->nnz > 0) P->csr_src.alloc(P->nnz);
    csr_fill<<<grid_for(3 * (int64_t)P->n_node, 256, P->ctx->sm_count), 256, 0, s>>>(
        P->n_node, P->brow_ptr.p, P->bcol.p, P->slice_base.p, P->node_dof.p, P->csr_rowptr.p, P->csr_col.p,
        with_src ? P->csr_src.p : nullptr);
    MPHY_CUDA(cudaGetLastError());
}

void pattern_elem_dofs(const mphy_pattern* P, const mphy_mesh* mesh, int32_t* fav_dev) {
    elem_dofs<<<grid_for((int64_t)P->n_elem * P->npe * 3, 256, P->ctx->sm_count), 256, 0, P->ctx->stream>>>(
        P->n_elem, P->npe, mesh->conn.p, P->node_dof.p, fav_dev);
    MPHY_CUDA(cudaGetLastError());
}

}  // namespace mphy
