// mixed.cu -- mixed u-p (tet10 / linear vertex pressure) problems: the two-field system, its
// assembly, a preconditioned MINRES solve and the Newton load stepping with pressure unknowns.
//
// Replaces, for MIXED_ELEMENT meshes of Elem_Solid_3D_Mixed1 (npElem = 10):
//   * femSolidmechanics::prepareDataForMixedElements (femSolidmechanics1.cpp:274-380): the
//     pressure DOFs are the elements' vertex nodes, numbered in ascending node order;
//   * the u-p and p-p entries of prepareMatrixPattern (femSolidmechanics2.cpp:327-371) and
//     SolverPetsc::assembleMatrixAndVector2field (SolverPetsc.cpp:434-502);
//   * solveWithNewtonRaphson / factoriseSolveAndUpdate with pressure updates
//     (femSolidmechanics2.cpp:730-851, 1127-1200).
//
// Storage. The displacement block Kuu is the displacement path's SELL-32 3x3 layout (FP64, rows
// and columns of prescribed DOFs left out, identity on their diagonal). The coupling blocks are
// compressed rows with 3 values per entry: B = Kup by node rows over pressure columns, B^T = Kpu
// by pressure rows over node columns (both stored, so that y = A x needs no atomics), and C = Kpp
// by pressure rows. The two-field vectors are [3 n_node displacement | n_pres pressure].
//
// Solve. The reference's sample inputs factorise the indefinite system with MUMPS LU
// (-ksp_type preonly -pc_type lu). Here: MINRES (Paige-Saunders recurrences in the preconditioned
// form of Elman, Silvester and Wathen) with the symmetric positive definite block-diagonal
// preconditioner P_u^-1 (+) S^-1: P_u^-1 = diag(Kuu)^-1, plus Z E^-1 Z^T with the rigid-body
// coarse space of the displacement solver when coarse_aggregates > 0; S_ii = sum_k (B^T_ik)^2 /
// Kuu_kk + |C_ii| (the diagonal of the Schur complement's approximation). All scalars stay on
// the device; the host reads the residual estimate every kCheck iterations.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "coarse.cuh"
#include "common.cuh"
#include "elem.cuh"
#include "krylov.cuh"
#include "mixed.cuh"
#include "solver.cuh"

using namespace mphy;

struct mphy_mixed {
    mphy_ctx* ctx = nullptr;
    const mphy_mesh* mesh = nullptr;
    const mphy_pattern* pat = nullptr;
    int device = 0;
    mphy_mixed_opts opts{};
    int32_t n_node = 0, n_elem = 0, n_pres = 0;
    int npe = 10, np_elem = 4;  // element nodes and pressure nodes per element (tet10: 4, hex27: 8)
    int64_t nb = 0, nc = 0;  // B (= B^T) and C entries
    int64_t launches = 0;
    SellView A{};
    DevBuf<int32_t> pres_id, pres_node;
    DevBuf<double> val;
    DevBuf<int64_t> b_ptr, bt_ptr, c_ptr;
    DevBuf<int32_t> b_col, bt_col, c_col;
    DevBuf<double> b_val, bt_val, c_val;
    DevBuf<uint32_t> e2b, e2bt, e2c;
    DevBuf<double> rhs, reac, dinv;
    DevBuf<double> v[3], w[3], z[2], x, az;
    DevBuf<double> sc, partials;
    DevBuf<uint32_t> counter;
    DevBuf<unsigned long long> bad;
    DevBuf<double> disp, disp_prev, pres, pres_prev, fext;
    std::vector<int32_t> pres_node_host;
    bool assembled = false;
    CoarseSpace coarse;  // opts.coarse_aggregates > 0: two-level displacement block
    bool use_coarse = false;
};

namespace {

constexpr int kCheck = 8;  // MINRES iterations between host reads of the residual estimate

// device scalar slots of the MINRES recurrences
enum : int {
    S_DOT1 = 0,   // (A z, z) with z unscaled
    S_DOT2,       // (z_new, v_new)
    S_GAMMA,      // gamma_j
    S_GAMMA_OLD,  // gamma_{j-1}
    S_C, S_C_OLD, S_S, S_S_OLD,
    S_ETA,
    S_A1, S_A2, S_A3, S_XCOEF, S_INVG,  // coefficients of the w / x update
    S_ETA0,
    S_DONE,       // 1: converged (or a zero right-hand side), 2: breakdown
    S_WSKIP,      // this iteration's w / x update is skipped (set by the scalar kernel)
    S_COUNT
};

std::vector<int32_t> download_i32(const int32_t* d, size_t n) {
    std::vector<int32_t> h(n);
    if (n) MPHY_CUDA(cudaMemcpy(h.data(), d, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    return h;
}

// Compressed rows from (row, col) pairs, sorted and unique; `key` = row * n_cols + col.
void build_rows(std::vector<int64_t>& keys, int64_t n_rows, int64_t n_cols, std::vector<int64_t>& ptr,
                std::vector<int32_t>& col) {
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    ptr.assign(n_rows + 1, 0);
    col.resize(keys.size());
    for (size_t k = 0; k < keys.size(); ++k) {
        ptr[keys[k] / n_cols + 1] += 1;
        col[k] = (int32_t)(keys[k] % n_cols);
    }
    for (int64_t r = 0; r < n_rows; ++r) ptr[r + 1] += ptr[r];
}

uint32_t find_entry(const std::vector<int64_t>& ptr, const std::vector<int32_t>& col, int64_t row, int32_t c) {
    const auto b = col.begin() + ptr[row], e = col.begin() + ptr[row + 1];
    const auto it = std::lower_bound(b, e, c);
    MPHY_REQUIRE(it != e && *it == c, MPHY_ERR_CUDA, "mixed pattern: missing entry");
    return (uint32_t)(it - col.begin());
}

// y_u += B x_p (node rows); y_p = B^T x_u + C x_p (pressure rows)
__global__ void coupling_apply_kernel(int32_t n_node, int32_t n_pres, const int64_t* __restrict__ b_ptr,
                                      const int32_t* __restrict__ b_col, const double* __restrict__ b_val,
                                      const int64_t* __restrict__ bt_ptr, const int32_t* __restrict__ bt_col,
                                      const double* __restrict__ bt_val, const int64_t* __restrict__ c_ptr,
                                      const int32_t* __restrict__ c_col, const double* __restrict__ c_val,
                                      const double* __restrict__ x, double* __restrict__ y) {
    const double* xp = x + 3 * (int64_t)n_node;
    const int64_t total = (int64_t)n_node + n_pres;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        if (t < n_node) {
            double s0 = 0.0, s1 = 0.0, s2 = 0.0;
            for (int64_t k = b_ptr[t]; k < b_ptr[t + 1]; ++k) {
                const double xv = xp[b_col[k]];
                s0 += b_val[3 * k] * xv;
                s1 += b_val[3 * k + 1] * xv;
                s2 += b_val[3 * k + 2] * xv;
            }
            y[3 * t] += s0;
            y[3 * t + 1] += s1;
            y[3 * t + 2] += s2;
        } else {
            const int64_t i = t - n_node;
            double acc = 0.0;
            for (int64_t k = bt_ptr[i]; k < bt_ptr[i + 1]; ++k) {
                const int64_t n = bt_col[k];
                acc += bt_val[3 * k] * x[3 * n] + bt_val[3 * k + 1] * x[3 * n + 1] + bt_val[3 * k + 2] * x[3 * n + 2];
            }
            for (int64_t k = c_ptr[i]; k < c_ptr[i + 1]; ++k) acc += c_val[k] * xp[c_col[k]];
            y[3 * (int64_t)n_node + i] = acc;
        }
    }
}

// dinv: 1 / diag(Kuu) on the displacement rows (prescribed rows hold 1), then the pressure rows
// 1 / (sum_k sum_a bt_ak^2 / Kuu_(3k+a) + |C_ii|)
__global__ void precond_u_kernel(int32_t n_node, const uint32_t* __restrict__ dvoff, const double* __restrict__ val,
                                 double* __restrict__ dinv) {
    for (int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; n < n_node; n += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t o = dvoff[n];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double d = o == UINT32_MAX ? 1.0 : val[o + 32u * (4 * a)];
            dinv[3 * n + a] = d != 0.0 ? 1.0 / d : 1.0;
        }
    }
}

__global__ void precond_p_kernel(int32_t n_node, int32_t n_pres, const int64_t* __restrict__ bt_ptr,
                                 const int32_t* __restrict__ bt_col, const double* __restrict__ bt_val,
                                 const int64_t* __restrict__ c_ptr, const int32_t* __restrict__ c_col,
                                 const double* __restrict__ c_val, double* __restrict__ dinv) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_pres; i += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int64_t k = bt_ptr[i]; k < bt_ptr[i + 1]; ++k) {
            const int64_t n = bt_col[k];
#pragma unroll
            for (int a = 0; a < 3; ++a) s += bt_val[3 * k + a] * bt_val[3 * k + a] * fabs(dinv[3 * n + a]);
        }
        for (int64_t k = c_ptr[i]; k < c_ptr[i + 1]; ++k)
            if (c_col[k] == i) s += fabs(c_val[k]);
        dinv[3 * (int64_t)n_node + i] = s > 0.0 ? 1.0 / s : 1.0;
    }
}

// MINRES, part 1: v_new = A z / g - (delta / g) v - (g / g_old) v_old with delta = (A z, z) / g^2,
// z_new = M^-1 v_new (z, A z unscaled by g)
__global__ void minres_v_kernel(int64_t n, const double* __restrict__ az, const double* __restrict__ v,
                                const double* __restrict__ v_old, const double* __restrict__ dinv,
                                const double* __restrict__ sc, double* __restrict__ v_new, double* __restrict__ z_new) {
    if (sc[S_DONE] != 0.0) return;
    const double g = sc[S_GAMMA], g_old = sc[S_GAMMA_OLD];
    const double delta = sc[S_DOT1] / (g * g);
    const double c1 = 1.0 / g, c2 = delta / g, c3 = g / g_old;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double vn = c1 * az[i] - c2 * v[i] - c3 * v_old[i];
        v_new[i] = vn;
        z_new[i] = dinv[i] * vn;
    }
}

// part 2 (one thread): the Givens rotation and the shift of the scalar state
__global__ void minres_scalar_kernel(double* sc, double rtol) {
    sc[S_WSKIP] = 1.0;
    if (sc[S_DONE] != 0.0) return;
    const double g = sc[S_GAMMA], c = sc[S_C], c_old = sc[S_C_OLD], s = sc[S_S], s_old = sc[S_S_OLD];
    const double delta = sc[S_DOT1] / (g * g);
    const double g_new = sqrt(fmax(sc[S_DOT2], 0.0));
    const double a0 = c * delta - c_old * s * g;
    const double a1 = sqrt(a0 * a0 + g_new * g_new);
    const double a2 = s * delta + c_old * c * g;
    const double a3 = s_old * g;
    if (!(a1 > 0.0)) {  // breakdown: the Krylov space is exhausted, x is the solution
        sc[S_DONE] = 2.0;
        return;
    }
    sc[S_WSKIP] = 0.0;
    const double c_new = a0 / a1, s_new = g_new / a1;
    sc[S_A1] = a1;
    sc[S_A2] = a2;
    sc[S_A3] = a3;
    sc[S_INVG] = 1.0 / g;
    sc[S_XCOEF] = c_new * sc[S_ETA];
    sc[S_ETA] = -s_new * sc[S_ETA];
    sc[S_GAMMA_OLD] = g;
    sc[S_GAMMA] = g_new > 0.0 ? g_new : 1.0;
    sc[S_C_OLD] = c;
    sc[S_C] = c_new;
    sc[S_S_OLD] = s;
    sc[S_S] = s_new;
    if (fabs(sc[S_ETA]) <= rtol * sc[S_ETA0] || !(g_new > 0.0)) sc[S_DONE] = 1.0;
}

// part 3: w_new = (z / g - a3 w_old - a2 w) / a1, x += c_new eta w_new
__global__ void minres_w_kernel(int64_t n, const double* __restrict__ z, const double* __restrict__ w,
                                const double* __restrict__ w_old, const double* __restrict__ sc,
                                double* __restrict__ w_new, double* __restrict__ x) {
    if (sc[S_WSKIP] != 0.0) return;
    const double ig = sc[S_INVG], a1 = sc[S_A1], a2 = sc[S_A2], a3 = sc[S_A3], xc = sc[S_XCOEF];
    const double r = 1.0 / a1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double wn = (z[i] * ig - a3 * w_old[i] - a2 * w[i]) * r;
        w_new[i] = wn;
        x[i] += xc * wn;
    }
}

__global__ void minres_init_kernel(double* sc, double eta0) {
    for (int i = 0; i < S_COUNT; ++i) sc[i] = 0.0;
    sc[S_GAMMA] = eta0 > 0.0 ? eta0 : 1.0;
    sc[S_GAMMA_OLD] = 1.0;
    sc[S_C] = sc[S_C_OLD] = 1.0;
    sc[S_ETA] = eta0;
    sc[S_ETA0] = eta0;
    if (!(eta0 > 0.0)) sc[S_DONE] = 1.0;
}

__global__ void scale_kernel(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                             double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] * b[i];
}

// pres[pres_node[i]] += xp[i]; disp += x_u
__global__ void mixed_update_kernel(int32_t n_node, int32_t n_pres, const int32_t* __restrict__ pres_node,
                                    const double* __restrict__ x, double* __restrict__ disp, double* __restrict__ pres) {
    const int64_t total = 3 * (int64_t)n_node + n_pres;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        if (t < 3 * (int64_t)n_node) disp[t] += x[t];
        else pres[pres_node[t - 3 * (int64_t)n_node]] += x[t];
    }
}

float event_ms(mphy_ctx* c) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    return ms;
}

void apply(mphy_mixed* m, const double* x, double* y, cudaStream_t st) {
    const int sm = m->ctx->sm_count;
    spmv<double, double>(m->A, m->val.p, x, y, st, sm);
    const int64_t total = (int64_t)m->n_node + m->n_pres;
    coupling_apply_kernel<<<resident_grid((const void*)coupling_apply_kernel, total, 256, sm), 256, 0, st>>>(
        m->n_node, m->n_pres, m->b_ptr.p, m->b_col.p, m->b_val.p, m->bt_ptr.p, m->bt_col.p, m->bt_val.p, m->c_ptr.p,
        m->c_col.p, m->c_val.p, x, y);
    MPHY_CUDA(cudaGetLastError());
    m->launches += 2;
}

MixedElemArgs elem_args(mphy_mixed* m, const double* disp, const double* disp_prev, const double* pres) {
    const mphy_mesh* me = m->mesh;
    MixedElemArgs a{};
    a.base.n_elem = me->n_elem;
    a.base.coords = me->coords.p;
    a.base.conn = me->conn.p;
    a.base.mat_id = me->mat_id.p;
    a.base.mats = me->mats.p;
    a.base.matx = me->matx.p;
    a.base.disp = disp;
    a.base.tangent = m->opts.tangent;
    a.base.bad = m->bad.p;
    a.base.fixed = me->fixed.p;
    a.disp_prev = disp_prev;
    a.pres = pres;
    a.pres_id = m->pres_id.p;
    return a;
}

// zero, element scatter, rhs_u += lambda fext (free DOFs), preconditioner; the first bad element
void assemble(mphy_mixed* m, const double* disp, const double* disp_prev, const double* pres, double lambda,
              const double* fext) {
    cudaStream_t st = m->ctx->stream;
    const int sm = m->ctx->sm_count;
    MPHY_CUDA(cudaMemsetAsync(m->val.p, 0, m->val.bytes(), st));
    set_prescribed_diagonal<double>(m->A, m->mesh->fixed.p, m->val.p, st, sm);
    MPHY_CUDA(cudaMemsetAsync(m->b_val.p, 0, m->b_val.bytes(), st));
    MPHY_CUDA(cudaMemsetAsync(m->bt_val.p, 0, m->bt_val.bytes(), st));
    MPHY_CUDA(cudaMemsetAsync(m->c_val.p, 0, m->c_val.bytes(), st));
    MPHY_CUDA(cudaMemsetAsync(m->rhs.p, 0, m->rhs.bytes(), st));
    MPHY_CUDA(cudaMemsetAsync(m->reac.p, 0, m->reac.bytes(), st));
    MPHY_CUDA(cudaMemsetAsync(m->bad.p, 0xff, sizeof(unsigned long long), st));
    MixedElemArgs a = elem_args(m, disp, disp_prev, pres);
    a.base.e2v = m->pat->e2v.p;
    a.base.val = m->val.p;
    a.base.rhs = m->rhs.p;
    a.base.reac = m->reac.p;
    a.e2b = m->e2b.p;
    a.e2bt = m->e2bt.p;
    a.e2c = m->e2c.p;
    a.bval = m->b_val.p;
    a.btval = m->bt_val.p;
    a.cval = m->c_val.p;
    a.rhs_p = m->rhs.p + 3 * (int64_t)m->n_node;
    launch_elem_mixed(a, m->npe, 2, st);
    if (fext) add_scaled_free(m->mesh->fixed.p, fext, lambda, m->rhs.p, 3 * (int64_t)m->n_node, st, sm);
    precond_u_kernel<<<stride_grid(m->n_node, 256, sm), 256, 0, st>>>(m->n_node, m->A.dvoff, m->val.p, m->dinv.p);
    precond_p_kernel<<<stride_grid(m->n_pres, 256, sm), 256, 0, st>>>(m->n_node, m->n_pres, m->bt_ptr.p, m->bt_col.p,
                                                                      m->bt_val.p, m->c_ptr.p, m->c_col.p, m->c_val.p,
                                                                      m->dinv.p);
    MPHY_CUDA(cudaGetLastError());
    m->launches += 10;
    if (m->use_coarse) {
        m->coarse.setup<double>(m->A, m->val.p, nullptr, st);
        m->launches += m->coarse.launches;
    }
    m->assembled = true;
}

// ||rhs|| and the first bad element (one synchronisation)
double norm_and_bad(mphy_mixed* m, int64_t* first_bad) {
    cudaStream_t st = m->ctx->stream;
    const int64_t n = 3 * (int64_t)m->n_node + m->n_pres;
    dot_fp64(m->rhs.p, m->rhs.p, n, m->partials.p, m->counter.p, m->sc.p + S_COUNT, st, m->ctx->sm_count);
    double h = 0.0;
    unsigned long long b = 0;
    MPHY_CUDA(cudaMemcpyAsync(&h, m->sc.p + S_COUNT, sizeof(double), cudaMemcpyDeviceToHost, st));
    MPHY_CUDA(cudaMemcpyAsync(&b, m->bad.p, sizeof(b), cudaMemcpyDeviceToHost, st));
    MPHY_CUDA(cudaStreamSynchronize(st));
    m->launches += 1;
    if (first_bad) *first_bad = b == ULLONG_MAX ? -1 : (int64_t)b;
    return std::sqrt(h);
}

// MINRES on rhs -> x from x = 0. *its: iterations; *relres: ||rhs - A x|| / ||rhs|| in FP64.
int minres(mphy_mixed* m, int32_t* its_out, double* relres) {
    cudaStream_t st = m->ctx->stream;
    const int sm = m->ctx->sm_count;
    const int64_t n = 3 * (int64_t)m->n_node + m->n_pres;
    const unsigned grid = resident_grid((const void*)minres_w_kernel, n, 256, sm);
    double* sc = m->sc.p;
    MPHY_CUDA(cudaMemsetAsync(m->x.p, 0, n * sizeof(double), st));
    for (int k = 0; k < 3; ++k) MPHY_CUDA(cudaMemsetAsync(m->w[k].p, 0, n * sizeof(double), st));
    MPHY_CUDA(cudaMemsetAsync(m->v[0].p, 0, n * sizeof(double), st));
    MPHY_CUDA(cudaMemcpyAsync(m->v[1].p, m->rhs.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    scale_kernel<<<grid, 256, 0, st>>>(n, m->dinv.p, m->v[1].p, m->z[0].p);
    if (m->use_coarse) {
        coarse_apply_add(m->coarse.view(), m->n_node, m->v[1].p, m->z[0].p, st, sm);
        m->launches += 6;
    }
    dot_fp64(m->z[0].p, m->v[1].p, n, m->partials.p, m->counter.p, sc + S_DOT2, st, sm);
    double g0sq = 0.0;
    MPHY_CUDA(cudaMemcpyAsync(&g0sq, sc + S_DOT2, sizeof(double), cudaMemcpyDeviceToHost, st));
    MPHY_CUDA(cudaStreamSynchronize(st));
    minres_init_kernel<<<1, 1, 0, st>>>(sc, std::sqrt(std::fmax(g0sq, 0.0)));
    m->launches += 3;
    int iv_old = 0, iv = 1, iv_new = 2, iw_old = 0, iw = 1, iw_new = 2, iz = 0, iz_new = 1;
    int its = 0, status = MPHY_ERR_NOT_CONVERGED;
    const int maxit = m->opts.max_it > 0 ? m->opts.max_it : 10000;
    while (its < maxit) {
        for (int k = 0; k < kCheck && its < maxit; ++k, ++its) {
            apply(m, m->z[iz].p, m->az.p, st);
            dot_fp64(m->az.p, m->z[iz].p, n, m->partials.p, m->counter.p, sc + S_DOT1, st, sm);
            minres_v_kernel<<<grid, 256, 0, st>>>(n, m->az.p, m->v[iv].p, m->v[iv_old].p, m->dinv.p, sc,
                                                  m->v[iv_new].p, m->z[iz_new].p);
            if (m->use_coarse) {
                coarse_apply_add(m->coarse.view(), m->n_node, m->v[iv_new].p, m->z[iz_new].p, st, sm);
                m->launches += 6;
            }
            dot_fp64(m->z[iz_new].p, m->v[iv_new].p, n, m->partials.p, m->counter.p, sc + S_DOT2, st, sm);
            minres_scalar_kernel<<<1, 1, 0, st>>>(sc, m->opts.rtol);
            minres_w_kernel<<<grid, 256, 0, st>>>(n, m->z[iz].p, m->w[iw].p, m->w[iw_old].p, sc, m->w[iw_new].p,
                                                  m->x.p);
            MPHY_CUDA(cudaGetLastError());
            m->launches += 5;
            int t = iv_old;
            iv_old = iv;
            iv = iv_new;
            iv_new = t;
            t = iw_old;
            iw_old = iw;
            iw = iw_new;
            iw_new = t;
            std::swap(iz, iz_new);
        }
        double done = 0.0;
        MPHY_CUDA(cudaMemcpyAsync(&done, sc + S_DONE, sizeof(double), cudaMemcpyDeviceToHost, st));
        MPHY_CUDA(cudaStreamSynchronize(st));
        if (done != 0.0) {
            status = MPHY_OK;
            break;
        }
    }
    // FP64 true residual ||rhs - A x|| / ||rhs||
    apply(m, m->x.p, m->az.p, st);
    axpy_inplace(m->az.p, m->rhs.p, -1.0, n, st, sm);
    dot_fp64(m->az.p, m->az.p, n, m->partials.p, m->counter.p, sc + S_DOT1, st, sm);
    dot_fp64(m->rhs.p, m->rhs.p, n, m->partials.p, m->counter.p, sc + S_DOT2, st, sm);
    double h[2];
    MPHY_CUDA(cudaMemcpyAsync(h, sc + S_DOT1, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    MPHY_CUDA(cudaStreamSynchronize(st));
    m->launches += 4;
    if (its_out) *its_out = its;
    if (relres) *relres = h[1] > 0.0 ? std::sqrt(h[0] / h[1]) : 0.0;
    return status;
}

}  // namespace

extern "C" {

void mphy_mixed_opts_default(mphy_mixed_opts* o) {
    if (!o) return;
    o->tangent = MPHY_TANGENT_REFERENCE;
    o->max_it = 20000;
    o->rtol = 1e-10;
    o->coarse_aggregates = 0;
    o->coarse_modes = 0;
}

int mphy_mixed_create(mphy_ctx* c, const mphy_mesh* mesh, const mphy_pattern* pat, const mphy_mixed_opts* o,
                      mphy_mixed** out) {
    return guarded([&] {
        MPHY_REQUIRE(c && mesh && pat && out, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(!mesh->has_presc, MPHY_ERR_UNSUPPORTED,
                     "mixed u-p elements with nonzero prescribed displacements");
        MPHY_REQUIRE(mesh->npe == 10 || mesh->npe == 27, MPHY_ERR_UNSUPPORTED,
                     "mixed u-p elements: tet10 with linear vertex pressure (npe = 10) or hex27 with trilinear "
                     "corner pressure (npe = 27)");
        MPHY_REQUIRE(pat->mesh == mesh, MPHY_ERR_INVALID_ARG, "the pattern belongs to another mesh");
        MPHY_CUDA(cudaSetDevice(c->device));
        auto* m = new mphy_mixed;
        try {
            m->ctx = c;
            m->mesh = mesh;
            m->pat = pat;
            m->device = c->device;
            if (o) m->opts = *o;
            else mphy_mixed_opts_default(&m->opts);
            m->n_node = mesh->n_node;
            m->n_elem = mesh->n_elem;
            const int32_t nn = mesh->n_node, ne = mesh->n_elem;
            const int npe = mesh->npe, NP = npe == 27 ? 8 : 4;  // pressure nodes: the first NP of each element
            m->npe = npe;
            m->np_elem = NP;
            if (npe == 27) {
                static std::atomic<uint64_t> tables{0};
                if (first_use_on_device(tables)) upload_hex27_tables();
            }
            const std::vector<int32_t> conn = download_i32(mesh->conn.p, (size_t)ne * npe);
            // pressure DOFs: vertex (corner) nodes in ascending order
            std::vector<int32_t> pid(nn, -1);
            for (int32_t e = 0; e < ne; ++e)
                for (int i = 0; i < NP; ++i) pid[conn[npe * (size_t)e + i]] = 0;
            int32_t np = 0;
            m->pres_node_host.clear();
            for (int32_t n = 0; n < nn; ++n)
                if (pid[n] == 0) {
                    pid[n] = np++;
                    m->pres_node_host.push_back(n);
                }
            m->n_pres = np;
            // B (node rows), B^T (pressure rows), C (pressure rows)
            std::vector<int64_t> kb, kbt, kc;
            kb.reserve((size_t)ne * npe * NP);
            kbt.reserve((size_t)ne * npe * NP);
            kc.reserve((size_t)ne * NP * NP);
            for (int32_t e = 0; e < ne; ++e) {
                const int32_t* cn = &conn[npe * (size_t)e];
                for (int j = 0; j < NP; ++j) {
                    const int64_t pj = pid[cn[j]];
                    for (int I = 0; I < npe; ++I) {
                        kb.push_back((int64_t)cn[I] * np + pj);
                        kbt.push_back(pj * nn + cn[I]);
                    }
                    for (int i = 0; i < NP; ++i) kc.push_back((int64_t)pid[cn[i]] * np + pj);
                }
            }
            std::vector<int64_t> bp, btp, cp;
            std::vector<int32_t> bc, btc, cc;
            build_rows(kb, nn, np, bp, bc);
            build_rows(kbt, np, nn, btp, btc);
            build_rows(kc, np, np, cp, cc);
            m->nb = (int64_t)bc.size();
            m->nc = (int64_t)cc.size();
            std::vector<uint32_t> e2b((size_t)ne * npe * NP), e2bt((size_t)ne * npe * NP), e2c((size_t)ne * NP * NP);
            for (int32_t e = 0; e < ne; ++e) {
                const int32_t* cn = &conn[npe * (size_t)e];
                for (int I = 0; I < npe; ++I)
                    for (int j = 0; j < NP; ++j) {
                        e2b[(npe * (size_t)e + I) * NP + j] = find_entry(bp, bc, cn[I], pid[cn[j]]);
                        e2bt[(NP * (size_t)e + j) * npe + I] = find_entry(btp, btc, pid[cn[j]], cn[I]);
                    }
                for (int i = 0; i < NP; ++i)
                    for (int j = 0; j < NP; ++j)
                        e2c[(NP * (size_t)e + i) * NP + j] = find_entry(cp, cc, pid[cn[i]], pid[cn[j]]);
            }
            cudaStream_t st = c->stream;
            auto up32 = [&](DevBuf<int32_t>& d, const std::vector<int32_t>& h) { d.alloc(std::max<size_t>(1, h.size())); d.upload(h.data(), h.size(), st); };
            auto up64 = [&](DevBuf<int64_t>& d, const std::vector<int64_t>& h) { d.alloc(h.size()); d.upload(h.data(), h.size(), st); };
            auto upu = [&](DevBuf<uint32_t>& d, const std::vector<uint32_t>& h) { d.alloc(std::max<size_t>(1, h.size())); d.upload(h.data(), h.size(), st); };
            up32(m->pres_id, pid);
            up32(m->pres_node, m->pres_node_host);
            up64(m->b_ptr, bp);
            up64(m->bt_ptr, btp);
            up64(m->c_ptr, cp);
            up32(m->b_col, bc);
            up32(m->bt_col, btc);
            up32(m->c_col, cc);
            upu(m->e2b, e2b);
            upu(m->e2bt, e2bt);
            upu(m->e2c, e2c);
            m->b_val.alloc(3 * (size_t)std::max<int64_t>(1, m->nb));
            m->bt_val.alloc(3 * (size_t)std::max<int64_t>(1, m->nb));
            m->c_val.alloc((size_t)std::max<int64_t>(1, m->nc));
            m->A = SellView{pat->n_node, pat->n_slices, pat->slice_base.p, pat->slice_width.p, pat->sell_col.p,
                            pat->dvoff.p};
            m->val.alloc(9 * (size_t)pat->sell_blocks);
            const size_t n = 3 * (size_t)nn + np;
            m->rhs.alloc(n);
            m->reac.alloc(3 * (size_t)nn);
            m->dinv.alloc(n);
            for (auto& b : m->v) b.alloc(n);
            for (auto& b : m->w) b.alloc(n);
            for (auto& b : m->z) b.alloc(n);
            m->x.alloc(n);
            m->az.alloc(n);
            m->sc.alloc(S_COUNT + 4);
            m->partials.alloc((size_t)c->sm_count * 8 + 8);
            m->counter.alloc(1);
            MPHY_CUDA(cudaMemsetAsync(m->counter.p, 0, sizeof(uint32_t), st));
            m->bad.alloc(1);
            if (m->opts.coarse_aggregates > 0) {
                m->coarse.init(c, mesh, pat, m->opts.coarse_aggregates,
                               m->opts.coarse_modes > 0 ? m->opts.coarse_modes : 6);
                m->use_coarse = true;
            }
            MPHY_CUDA(cudaStreamSynchronize(st));
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
        return (int)MPHY_OK;
    });
}

int mphy_mixed_destroy(mphy_mixed* m) {
    if (!m) return MPHY_OK;
    cudaSetDevice(m->device);
    cudaDeviceSynchronize();
    delete m;
    return MPHY_OK;
}

int mphy_mixed_info(mphy_mixed* m, int32_t* n_pres, int64_t* nnz_coupling, int64_t* nnz_pp) {
    return guarded([&] {
        MPHY_REQUIRE(m, MPHY_ERR_INVALID_ARG, "null argument");
        if (n_pres) *n_pres = m->n_pres;
        if (nnz_coupling) *nnz_coupling = m->nb;
        if (nnz_pp) *nnz_pp = m->nc;
        return (int)MPHY_OK;
    });
}

int mphy_mixed_pressure_nodes(mphy_mixed* m, int32_t* nodes_host) {
    return guarded([&] {
        MPHY_REQUIRE(m && nodes_host, MPHY_ERR_INVALID_ARG, "null argument");
        std::memcpy(nodes_host, m->pres_node_host.data(), m->pres_node_host.size() * sizeof(int32_t));
        return (int)MPHY_OK;
    });
}

int mphy_mixed_elem_eval(mphy_mixed* m, const double* disp, const double* disp_prev, const double* pres, double* Kuu,
                         double* FU, double* Kup, double* Kpp, double* FP, int64_t* first_bad) {
    return guarded([&] {
        MPHY_REQUIRE(m && disp && disp_prev && pres && Kuu && FU && Kup && Kpp && FP, MPHY_ERR_INVALID_ARG,
                     "null argument");
        cudaStream_t st = m->ctx->stream;
        MPHY_CUDA(cudaMemsetAsync(m->bad.p, 0xff, sizeof(unsigned long long), st));
        MixedElemArgs a = elem_args(m, disp, disp_prev, pres);
        a.base.Ke = Kuu;
        a.base.Re = FU;
        a.Kup = Kup;
        a.Kpp = Kpp;
        a.FP = FP;
        launch_elem_mixed(a, m->npe, 1, st);
        unsigned long long h = 0;
        MPHY_CUDA(cudaMemcpyAsync(&h, m->bad.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        MPHY_CUDA(cudaStreamSynchronize(st));
        const int64_t b = h == ULLONG_MAX ? -1 : (int64_t)h;
        if (first_bad) *first_bad = b;
        if (b >= 0) {
            set_error("negative Jacobian in element " + std::to_string(b));
            return (int)MPHY_ERR_NEG_JACOBIAN;
        }
        return (int)MPHY_OK;
    });
}

int mphy_mixed_assemble(mphy_mixed* m, const double* disp, const double* disp_prev, const double* pres,
                        double lambda, const double* fext, double* rhs_norm, int64_t* first_bad) {
    return guarded([&] {
        MPHY_REQUIRE(m && disp && disp_prev && pres, MPHY_ERR_INVALID_ARG, "null argument");
        assemble(m, disp, disp_prev, pres, lambda, fext);
        int64_t b = -1;
        const double nrm = norm_and_bad(m, &b);
        if (rhs_norm) *rhs_norm = nrm;
        if (first_bad) *first_bad = b;
        if (b >= 0) {
            m->assembled = false;
            set_error("negative Jacobian in element " + std::to_string(b));
            return (int)MPHY_ERR_NEG_JACOBIAN;
        }
        return (int)MPHY_OK;
    });
}

int mphy_mixed_apply(mphy_mixed* m, const double* x, double* y) {
    return guarded([&] {
        MPHY_REQUIRE(m && x && y, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(m->assembled, MPHY_ERR_STATE, "assemble the mixed system first");
        apply(m, x, y, m->ctx->stream);
        MPHY_CUDA(cudaStreamSynchronize(m->ctx->stream));
        return (int)MPHY_OK;
    });
}

int mphy_mixed_vectors(mphy_mixed* m, double* rhs, double* reac, double* solution) {
    return guarded([&] {
        MPHY_REQUIRE(m, MPHY_ERR_INVALID_ARG, "null argument");
        cudaStream_t st = m->ctx->stream;
        const size_t n = 3 * (size_t)m->n_node + m->n_pres;
        if (rhs) MPHY_CUDA(cudaMemcpyAsync(rhs, m->rhs.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        if (reac) MPHY_CUDA(cudaMemcpyAsync(reac, m->reac.p, 3 * (size_t)m->n_node * sizeof(double),
                                            cudaMemcpyDeviceToDevice, st));
        if (solution) MPHY_CUDA(cudaMemcpyAsync(solution, m->x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        MPHY_CUDA(cudaStreamSynchronize(st));
        return (int)MPHY_OK;
    });
}

int mphy_mixed_solve(mphy_mixed* m, int32_t* its, double* relres) {
    return guarded([&] {
        MPHY_REQUIRE(m, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(m->assembled, MPHY_ERR_STATE, "assemble the mixed system first");
        const int rc = minres(m, its, relres);
        if (rc != MPHY_OK) set_error("MINRES did not reach rtol within max_it iterations");
        return rc;
    });
}

int mphy_mixed_newton_run(mphy_mixed* m, const double* fext_host, const mphy_newton_opts* o, double* disp_host,
                          double* pres_host, mphy_iter_stats* hist, int32_t max_hist, int32_t* n_hist) {
    return guarded([&] {
        MPHY_REQUIRE(m && fext_host && o && disp_host && pres_host, MPHY_ERR_INVALID_ARG, "null argument");
        cudaStream_t st = m->ctx->stream;
        const size_t nd = 3 * (size_t)m->n_node, nn = (size_t)m->n_node;
        for (DevBuf<double>* b : {&m->disp, &m->disp_prev, &m->fext})
            if (!b->p) b->alloc(nd);
        for (DevBuf<double>* b : {&m->pres, &m->pres_prev})
            if (!b->p) b->alloc(nn);
        m->disp.upload(disp_host, nd, st);
        m->pres.upload(pres_host, nn, st);
        m->fext.upload(fext_host, nd, st);
        const int sm = m->ctx->sm_count;
        const int64_t ntot = (int64_t)nd + m->n_pres;
        double t = 0.0, dt = o->dt;
        const double dt0 = o->dt;
        int steps_done = 1, rows = 0, rc = MPHY_OK;
        while (t <= o->t_final - 1.0e-10 && steps_done <= o->max_steps) {
            t += dt;  // timeUpdate: myTime.update, saveSolution (dispPrev, presPrev)
            const double lambda = t;
            MPHY_CUDA(cudaMemcpyAsync(m->disp_prev.p, m->disp.p, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
            MPHY_CUDA(cudaMemcpyAsync(m->pres_prev.p, m->pres.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, st));
            bool converged = false;
            double norm = -1.0, norm_prev = -1.0, tol = o->tol_abs;
            for (int iter = 1; iter <= o->max_newton; ++iter) {
                mphy_iter_stats is{};
                const int64_t l0 = m->launches;
                MPHY_CUDA(cudaEventRecord(m->ctx->ev0, st));
                assemble(m, m->disp.p, m->disp_prev.p, m->pres.p, lambda, m->fext.p);
                MPHY_CUDA(cudaEventRecord(m->ctx->ev1, st));
                int64_t bad = -1;
                norm_prev = norm;
                norm = norm_and_bad(m, &bad);
                is.t_assembly_ms = event_ms(m->ctx);
                if (bad >= 0) break;  // "Negative Jacobian encountered": the iteration loop ends
                if (iter == 1) tol = std::fmax(o->tol_abs, o->tol_rel * norm);
                bool stop = false;
                if (norm < tol) {
                    converged = true;
                    stop = true;
                } else if (iter > 3 && (std::isnan(norm) || (norm_prev > -0.1 && norm / norm_prev > 1.0e7))) {
                    stop = true;
                } else {
                    MPHY_CUDA(cudaEventRecord(m->ctx->ev0, st));
                    int32_t its = 0;
                    double rr = 0.0;
                    is.status = minres(m, &its, &rr);
                    mixed_update_kernel<<<stride_grid(ntot, 256, sm), 256, 0, st>>>(m->n_node, m->n_pres,
                                                                                     m->pres_node.p, m->x.p,
                                                                                     m->disp.p, m->pres.p);
                    MPHY_CUDA(cudaGetLastError());
                    m->launches += 1;
                    MPHY_CUDA(cudaEventRecord(m->ctx->ev1, st));
                    MPHY_CUDA(cudaEventSynchronize(m->ctx->ev1));
                    is.t_solve_ms = event_ms(m->ctx);
                    is.krylov_its = its;
                }
                is.step = steps_done;
                is.iter = iter;
                is.rhs_norm = norm;
                is.kernel_launches = m->launches - l0;
                if (hist && rows < max_hist) hist[rows++] = is;
                if (stop) break;
            }
            if (converged) {
                ++steps_done;
            } else {
                // MyTime::cut + SolutionDataSolid::reset (displacements and pressures)
                t -= dt;
                dt *= 0.5;
                if (dt < dt0 * 0.01) {
                    rc = MPHY_ERR_TIME_STEP;
                    set_error(mphy_status_string(rc));
                    break;
                }
                MPHY_CUDA(cudaMemcpyAsync(m->disp.p, m->disp_prev.p, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
                MPHY_CUDA(cudaMemcpyAsync(m->pres.p, m->pres_prev.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, st));
            }
        }
        m->disp.download(disp_host, nd, st);
        m->pres.download(pres_host, nn, st);
        MPHY_CUDA(cudaStreamSynchronize(st));
        if (n_hist) *n_hist = rows;
        return rc;
    });
}

}  // extern "C"
