// elem.cu -- K1 element kernels (+ K3 scatter-add assembly fused into them) and the batched
// material call.
//
// Replaces Elem_Solid_3D_Disp::calcStiffnessAndResidual (Elem_Solid_3D_Disp.cpp:196-373), the
// Neo-Hookean MaterialBase::computeStressAndTangent (utilitiesmaterialHyperelastic.cpp:186-295)
// and the per-entry MatSetValue/VecSetValue(ADD_VALUES) scatter (SolverPetsc.cpp:357-378).
//
// The reference contracts K_IJ(a,b) = sum_gp sum_{m,n} dvol dN_I/dx_m C(a m, b n) dN_J/dx_n with
// a dense 9x9 tangent. Written out, the Neo-Hookean tangent of :232-292 is a combination of
// Kronecker deltas and b = F F^T, so the same sum collapses per Gauss point to
//   K_IJ(a,b) += c1 h_Ib h_Ja + c2 (b h_I)_a h_Jb + c3 h_Ia h_Jb + c2 h_Ia (b h_J)_b
//                + d_ab (f4 h_I.b h_J + f9 h_I.h_J)              (all scaled by dvol)
// with h = spatial shape-function gradients and
//   c1 = mu J^-5/3 Ib/3 - U',  c2 = -(2/3) mu J^-5/3,  c3 = (2/9) mu J^-5/3 Ib + J U'' + U',
//   f4 = mu J^-5/3,            f9 = -U' (reference tangent) or 0 (consistent tangent).
// That is 30 FMAs per 3x3 block per Gauss point instead of the dense contraction's 108.
#include "common.cuh"
#include "elem.cuh"
#include "elem_store.cuh"
#include "nh.cuh"

namespace mphy {

// ---------------------------------------------------------------- shape tables (constant memory)
// dN/dxi at the Gauss points: hex8 [8 gp][3][8], tet10 [4 gp][3][10]; weights per gp.
__constant__ double c_hex8_dN[8 * 3 * 8];
__constant__ double c_hex8_w[8];
__constant__ double c_tet10_dN[4 * 3 * 10];
__constant__ double c_tet10_w[4];

namespace {

// Gauss rules and shape-function derivatives, with the reference's literals:
// QuadratureUtil.cpp:24-25 (2-point abscissa), :481-492 (hex ordering), :690-712 (tet 4-point);
// BasisFunctionsLagrange.cpp:146-152, :1243-1279 (hex8), :870-956 (tet10).
void host_hex8_tables(double* dN, double* w) {
    const double g = 0.577350269189626;
    const int pat[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int q = 0; q < 8; ++q) {
        double xi[3], n1[3][2];
        for (int d = 0; d < 3; ++d) {
            xi[d] = pat[q][d] ? g : -g;
            n1[d][0] = 0.5 * (1.0 - xi[d]);
            n1[d][1] = 0.5 * (1.0 + xi[d]);
        }
        const double d1[2] = {-0.5, 0.5};
        for (int a = 0; a < 8; ++a) {
            const int i = pat[a][0], j = pat[a][1], k = pat[a][2];
            dN[(q * 3 + 0) * 8 + a] = d1[i] * n1[1][j] * n1[2][k];
            dN[(q * 3 + 1) * 8 + a] = n1[0][i] * d1[j] * n1[2][k];
            dN[(q * 3 + 2) * 8 + a] = n1[0][i] * n1[1][j] * d1[k];
        }
        w[q] = 1.0;
    }
}

void host_tet10_tables(double* dN, double* w) {
    const double a = 0.1381966011250105, b = 0.5854101966249685;
    const double pts[4][3] = {{a, a, a}, {b, a, a}, {a, b, a}, {a, a, b}};
    const int edge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {2, 3}, {1, 3}};
    for (int q = 0; q < 4; ++q) {
        const double* xi = pts[q];
        const double L[4] = {1.0 - xi[0] - xi[1] - xi[2], xi[0], xi[1], xi[2]};
        auto dL = [](int v, int d) { return v == 0 ? -1.0 : (v == d + 1 ? 1.0 : 0.0); };
        for (int d = 0; d < 3; ++d) {
            for (int v = 0; v < 4; ++v) dN[(q * 3 + d) * 10 + v] = (4.0 * L[v] - 1.0) * dL(v, d);
            for (int e = 0; e < 6; ++e) {
                const int p = edge[e][0], r = edge[e][1];
                dN[(q * 3 + d) * 10 + 4 + e] = 4.0 * (dL(p, d) * L[r] + L[p] * dL(r, d));
            }
        }
        w[q] = 0.25 * (1.0 / 6.0);
    }
}

}  // namespace

void upload_shape_tables() {
    double h8[8 * 3 * 8], w8[8], t10[4 * 3 * 10], w4[4];
    host_hex8_tables(h8, w8);
    host_tet10_tables(t10, w4);
    MPHY_CUDA(cudaMemcpyToSymbol(c_hex8_dN, h8, sizeof(h8)));
    MPHY_CUDA(cudaMemcpyToSymbol(c_hex8_w, w8, sizeof(w8)));
    MPHY_CUDA(cudaMemcpyToSymbol(c_tet10_dN, t10, sizeof(t10)));
    MPHY_CUDA(cudaMemcpyToSymbol(c_tet10_w, w4, sizeof(w4)));
    upload_shape_tables_tc(h8, w8, t10, w4);
    upload_shape_tables_gen(h8, w8, t10, w4);
    upload_shape_tables_f32(h8, w8, t10, w4);
}

__device__ __forceinline__ double det3(const double A[3][3]) {
    return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

__device__ __forceinline__ void inv3(const double A[3][3], double det, double Ai[3][3]) {
    const double r = 1.0 / det;
    Ai[0][0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) * r;
    Ai[0][1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * r;
    Ai[0][2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * r;
    Ai[1][0] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) * r;
    Ai[1][1] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * r;
    Ai[1][2] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * r;
    Ai[2][0] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) * r;
    Ai[2][1] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * r;
    Ai[2][2] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * r;
}

// Batched material contract: full sigma (9) and C (81) in the reference's index order.
__global__ void nh_eval_kernel(int n, const double* __restrict__ Fm, double mu, double Kinv, int utype,
                               int tangent, double* __restrict__ stre, double* __restrict__ C) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double F[3][3], b[3][3];
    for (int i = 0; i < 9; ++i) F[i / 3][i % 3] = Fm[9 * (int64_t)t + i];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
    const double J = det3(F);
    const NhFactors f = nh_factors(b, J, mu, Kinv, utype, tangent);
    // (i, j) of the 9-index q: i = q % 3, j = q / 3 (map_tensor4)
    for (int q = 0; q < 9; ++q) stre[9 * (int64_t)t + q] = f.s1 * b[q % 3][q / 3] + (q % 3 == q / 3 ? f.s2 : 0.0);
    // C_ijkl = c1' d_il d_jk + c2 (b_ij d_kl + d_ij b_kl) + c3 d_ij d_kl + f4 b_jl d_ik + f9 d_jl d_ik,
    // where c1' d_il d_jk collects (mu J^-5/3 Ib/3 - U') as in the reference
    for (int p = 0; p < 9; ++p) {
        const int i = p % 3, j = p / 3;
        for (int q = 0; q < 9; ++q) {
            const int k = q % 3, l = q / 3;
            const double dij = i == j, dkl = k == l, dil = i == l, djk = j == k, dik = i == k, djl = j == l;
            C[81 * (int64_t)t + 9 * p + q] = f.c1 * dil * djk + f.c2 * (b[i][j] * dkl + dij * b[k][l]) +
                                             f.c3 * dij * dkl + f.f4 * b[j][l] * dik + f.f9 * djl * dik;
        }
    }
}

// ---------------------------------------------------------------- FP64 element kernel
template <int NPE>
struct ElemTraits;
template <>
struct ElemTraits<8> {
    static constexpr int NGP = 8;
    __device__ static const double* dN(int gp) { return c_hex8_dN + gp * 3 * 8; }
    __device__ static double w(int gp) { return c_hex8_w[gp]; }
};
template <>
struct ElemTraits<10> {
    static constexpr int NGP = 4;
    __device__ static const double* dN(int gp) { return c_tet10_dN + gp * 3 * 10; }
    __device__ static double w(int gp) { return c_tet10_w[gp]; }
};

constexpr int kEpb = 16;  // elements per CTA

// Shared memory per element: nodal data, per-(gp, node) spatial gradients h and b h, per-gp
// dvol-scaled tangent factors, per-(gp, node) residual contributions.
template <int NPE, int NGP>
struct ElemSmem {
    double x0[NPE][3];
    double u[NPE][3];
    double h[NGP][NPE][3];
    double bh[NGP][NPE][3];
    double fac[NGP][5];  // dvol * {c1, c2, c3, f4, f9}
    double r[NGP][NPE][3];
};

// MODE bit 1: export Ke/Re; bit 2: scatter into the matrix / rhs / reactions.
template <int NPE, int MODE>
__global__ void __launch_bounds__(kEpb * NPE) elem_fp64_kernel(ElemArgs a) {
    using T = ElemTraits<NPE>;
    constexpr int NGP = T::NGP;
    constexpr int NS = 3 * NPE;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto* S = reinterpret_cast<ElemSmem<NPE, NGP>*>(smem_raw);
    const int el = threadIdx.x / NPE, loc = threadIdx.x % NPE;
    const int64_t e = (int64_t)blockIdx.x * kEpb + el;
    const bool live = e < a.n_elem;
    ElemSmem<NPE, NGP>& s = S[el];

    int32_t node = 0;
    if (live) {
        node = a.conn[e * NPE + loc];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            s.x0[loc][d] = a.coords[3 * (int64_t)node + d];
            s.u[loc][d] = a.disp[3 * (int64_t)node + d];
        }
    }
    __syncthreads();

    // ---- phase 1: one thread per Gauss point
    if (live && loc < NGP) {
        const int gp = loc;
        const double* dN = T::dN(gp);
        double G[3][3] = {{0}}, Gc[3][3] = {{0}};
#pragma unroll
        for (int I = 0; I < NPE; ++I)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const double d = dN[r * NPE + I];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    G[r][c] += s.x0[I][c] * d;
                    Gc[r][c] += (s.x0[I][c] + s.u[I][c]) * d;
                }
            }
        double Gi[3][3], Gci[3][3];
        inv3(G, det3(G), Gi);
        const double jac = det3(Gc);
        inv3(Gc, jac, Gci);
        const double dvol = T::w(gp) * jac;
        // F = I + sum_I u_I (x) grad0 N_I   (ElementBase.cpp:334-361)
        double F[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
        for (int I = 0; I < NPE; ++I) {
            double g0[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                g0[c] = dN[I] * Gi[c][0] + dN[NPE + I] * Gi[c][1] + dN[2 * NPE + I] * Gi[c][2];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int m = 0; m < 3; ++m) F[i][m] += s.u[I][i] * g0[m];
        }
        const double J = det3(F);
        if (J < 0.0) {
            atomicMin(a.bad, (unsigned long long)e);
            if (a.bad_elem) a.bad_elem[e] = 1;
        }
        double b[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
        const double* m = a.mats + 4 * (int64_t)a.mat_id[e];
        const NhFactors f = nh_factors(b, J, m[0], m[1], (int)m[2], a.tangent);
#pragma unroll
        for (int I = 0; I < NPE; ++I) {
            double h[3], bh[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                h[c] = dN[I] * Gci[c][0] + dN[NPE + I] * Gci[c][1] + dN[2 * NPE + I] * Gci[c][2];
#pragma unroll
            for (int c = 0; c < 3; ++c) bh[c] = b[c][0] * h[0] + b[c][1] * h[1] + b[c][2] * h[2];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                s.h[gp][I][c] = h[c];
                s.bh[gp][I][c] = bh[c];
                // R_I -= dvol sigma h_I  (Elem_Solid_3D_Disp.cpp:328-334)
                s.r[gp][I][c] = -dvol * (f.s1 * bh[c] + f.s2 * h[c]);
            }
        }
        s.fac[gp][0] = dvol * f.c1;
        s.fac[gp][1] = dvol * f.c2;
        s.fac[gp][2] = dvol * f.c3;
        s.fac[gp][3] = dvol * f.f4;
        s.fac[gp][4] = dvol * f.f9;
    }
    __syncthreads();
    if (!live) return;

    // ---- phase 2: one thread per row node I
    const int I = loc;
    bool freeI[3] = {true, true, true};
    if (MODE & 2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) freeI[c] = a.fixed[3 * (int64_t)node + c] == 0;
    }
    {
        double R[3] = {0, 0, 0};
#pragma unroll
        for (int gp = 0; gp < NGP; ++gp)
#pragma unroll
            for (int c = 0; c < 3; ++c) R[c] += s.r[gp][I][c];
        store_residual<NPE, MODE>(a, e, I, node, freeI, R);
    }
    constexpr int CH = 4;
    double rl[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
    for (int J0 = 0; J0 < NPE; J0 += CH) {
        double acc[CH][9];
#pragma unroll
        for (int j = 0; j < CH; ++j)
#pragma unroll
            for (int v = 0; v < 9; ++v) acc[j][v] = 0.0;
#pragma unroll 2
        for (int gp = 0; gp < NGP; ++gp) {
            const double c1 = s.fac[gp][0], c2 = s.fac[gp][1], c3 = s.fac[gp][2], f4 = s.fac[gp][3],
                         f9 = s.fac[gp][4];
            double r[3], p[3], q[3], sv[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double hI = s.h[gp][I][c], bhI = s.bh[gp][I][c];
                r[c] = c1 * hI;
                p[c] = c2 * bhI + c3 * hI;
                q[c] = c2 * hI;
                sv[c] = f4 * bhI + f9 * hI;
            }
#pragma unroll
            for (int j = 0; j < CH; ++j) {
                if (J0 + j < NPE) {
                    double hJ[3], bhJ[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        hJ[c] = s.h[gp][J0 + j][c];
                        bhJ[c] = s.bh[gp][J0 + j][c];
                    }
#pragma unroll
                    for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                        for (int bb = 0; bb < 3; ++bb)
                            acc[j][3 * aa + bb] += r[bb] * hJ[aa] + p[aa] * hJ[bb] + q[aa] * bhJ[bb];
                    const double d = sv[0] * hJ[0] + sv[1] * hJ[1] + sv[2] * hJ[2];
                    acc[j][0] += d;
                    acc[j][4] += d;
                    acc[j][8] += d;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < CH; ++j) {
            const int J = J0 + j;
            if (J >= NPE) break;
            lift_block<NPE, MODE>(a, e, J, acc[j], rl);
            store_block<NPE, MODE>(a, e, I, J, node, freeI, acc[j]);
        }
    }
    store_lift<NPE, MODE>(a, node, freeI, rl);
}

template <int NPE, int MODE>
void launch_fp64(const ElemArgs& a, cudaStream_t s) {
    const size_t smem = kEpb * sizeof(ElemSmem<NPE, ElemTraits<NPE>::NGP>);
    static std::atomic<uint64_t> configured{0};
    if (first_use_on_device(configured)) {
        MPHY_CUDA(cudaFuncSetAttribute(elem_fp64_kernel<NPE, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    }
    const unsigned grid = ceil_div((size_t)a.n_elem, kEpb);
    if (grid == 0) return;
    elem_fp64_kernel<NPE, MODE><<<grid, kEpb * NPE, smem, s>>>(a);
    MPHY_CUDA(cudaGetLastError());
}

void launch_elem_fp64(const ElemArgs& a, int npe, int mode, cudaStream_t s) {
    if (npe == 8) {
        if (mode == 1) launch_fp64<8, 1>(a, s);
        else if (mode == 2) launch_fp64<8, 2>(a, s);
        else launch_fp64<8, 3>(a, s);
    } else {
        if (mode == 1) launch_fp64<10, 1>(a, s);
        else if (mode == 2) launch_fp64<10, 2>(a, s);
        else launch_fp64<10, 3>(a, s);
    }
}

void launch_nh_eval(int n, const double* F, double mu, double Kinv, int utype, int tangent, double* stre,
                    double* C, cudaStream_t s) {
    if (n <= 0) return;
    nh_eval_kernel<<<ceil_div(n, 128), 128, 0, s>>>(n, F, mu, Kinv, utype, tangent, stre, C);
    MPHY_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------- batch scatter (assembleMatrixAndVector)
template <int NPE>
__global__ void scatter_batch_kernel(int32_t n, const int32_t* __restrict__ ids, const int32_t* __restrict__ conn,
                                     const uint32_t* __restrict__ e2v, const uint8_t* __restrict__ fixed,
                                     const double* __restrict__ Ke, const double* __restrict__ Re,
                                     double* __restrict__ val, float* __restrict__ valf, double* __restrict__ rhs,
                                     double* __restrict__ reac) {
    constexpr int NS = 3 * NPE;
    const int64_t total = (int64_t)n * NPE * NPE;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = t / (NPE * NPE);
        const int IJ = (int)(t % (NPE * NPE));
        const int I = IJ / NPE, J = IJ % NPE;
        const int64_t e = ids ? ids[k] : k;
        const int32_t nI = conn[e * NPE + I], nJ = conn[e * NPE + J];
        const uint32_t off = e2v[e * NPE * NPE + IJ];
        if (valf) {
            // FP32 storage: off-diagonal blocks, unmasked; the diagonal is rebuilt from them
            if (nI != nJ)
                for (int v = 0; v < 9; ++v)
                    atomicAdd(&valf[off + 32u * v], (float)Ke[(k * NS + 3 * I + v / 3) * NS + 3 * J + v % 3]);
        } else {
            for (int aa = 0; aa < 3; ++aa) {
                if (fixed[3 * (int64_t)nI + aa]) continue;
                for (int bb = 0; bb < 3; ++bb) {
                    if (fixed[3 * (int64_t)nJ + bb]) continue;
                    atomicAdd(&val[off + 32u * (3 * aa + bb)], Ke[(k * NS + 3 * I + aa) * NS + 3 * J + bb]);
                }
            }
        }
        if (J == 0) {
            for (int aa = 0; aa < 3; ++aa) {
                const double r = Re[k * NS + 3 * I + aa];
                if (reac) atomicAdd(&reac[3 * (int64_t)nI + aa], r);
                if (!fixed[3 * (int64_t)nI + aa]) atomicAdd(&rhs[3 * (int64_t)nI + aa], r);
            }
        }
    }
}

void launch_scatter_batch(int npe, int32_t n, const int32_t* ids, const mphy_mesh* mesh, const mphy_pattern* P,
                          const double* Ke, const double* Re, double* val, float* valf, double* rhs, double* reac,
                          cudaStream_t s, int sm_count) {
    if (n <= 0) return;
    const int64_t total = (int64_t)n * npe * npe;
    unsigned grid = ceil_div(total, 256);
    if (grid > (unsigned)sm_count * 16) grid = sm_count * 16;
    if (npe == 8)
        scatter_batch_kernel<8><<<grid, 256, 0, s>>>(n, ids, mesh->conn.p, P->e2v.p, mesh->fixed.p, Ke, Re, val, valf,
                                                     rhs, reac);
    else
        scatter_batch_kernel<10><<<grid, 256, 0, s>>>(n, ids, mesh->conn.p, P->e2v.p, mesh->fixed.p, Ke, Re, val, valf,
                                                      rhs, reac);
    MPHY_CUDA(cudaGetLastError());
}

}  // namespace mphy
