// elem_f32.cu -- the mixed-precision element kernel (MPHY_PREC_MIXED, Neo-Hookean, hex8/tet10):
// Elem_Solid_3D_Disp::calcStiffnessAndResidual (Elem_Solid_3D_Disp.cpp:196-373) with the
// kinematics, stress and residual in FP64 and the tangent blocks in FP32, fused with the
// ADD_VALUES scatter (SolverPetsc.cpp:357-378) into the FP32 off-diagonal storage.
//
// One CTA takes 32 consecutive elements, one per lane: every warp holds the same local node (or
// Gauss point) of 32 elements, so the scatter of a block (I, J) of 32 neighbouring elements --
// consecutive node numbers in a structured mesh -- lands on consecutive SELL values (the SELL
// value v of the k-th block of node n sits at 9 (slice_base + 32 k) + 32 v + n % 32) and the
// reductions coalesce into few L2 sectors.
//
//   phase 1  thread (element, Gauss point), FP64: both Jacobians, F = I + (G^-1 U)^T with
//            U = sum_I u_I dN_I (the same F as ElementBase.cpp:334-361), J = det F, b = F F^T,
//            the Neo-Hookean factors, dvol sigma and the dvol-scaled tangent factors.
//   phase 2  thread (element, node I), FP64: spatial gradients h_I at every Gauss point and the
//            residual R_I = -sum_gp dvol sigma h_I (Elem_Solid_3D_Disp.cpp:328-334), added to the
//            right-hand side and the reactions; h_I and b h_I rounded to FP32 for the tangent.
//   phase 3  thread (element, node I), FP32: the tangent blocks K_IJ of the closed form of
//            elem.cu for the unordered pairs {I, J} this thread owns (pairs (I, I + d mod npe),
//            d = 1 .. npe/2, the d = npe/2 pairs owned by the smaller node). K is symmetric
//            (K_JI = K_IJ^T), so every pair is formed once and scattered twice.
//   phase 4  thread (element, node I): the element's diagonal block D_I = -sum_{J != I} K_IJ in
//            FP64, added to the solver's FP64 diagonal blocks (only their diagonal entries when
//            Jacobi is the local preconditioner). Those serve the preconditioners (Jacobi, FSAI,
//            the network's features); the operator itself recomputes each row's diagonal from its
//            stored blocks, so the stored FP32 operator still maps rigid translations exactly to
//            zero.
#include <cuda_pipeline.h>

#include "common.cuh"
#include "elem.cuh"
#include "nh.cuh"

namespace mphy {
namespace {

constexpr int kE = 32;  // elements per CTA, one per lane

// arithmetic of the tangent blocks (phase 3)
#ifndef MPHY_TANGENT_T
#define MPHY_TANGENT_T float
#endif
using TT = MPHY_TANGENT_T;

__constant__ double c_f8_dN[8 * 3 * 8];
__constant__ double c_f8_w[8];
__constant__ double c_f10_dN[4 * 3 * 10];
__constant__ double c_f10_w[4];

template <int NPE>
struct F32Traits;
template <>
struct F32Traits<8> {
    static constexpr int NGP = 8;
    __device__ static const double* dN(int g) { return c_f8_dN + g * 24; }
    __device__ static double w(int g) { return c_f8_w[g]; }
};
template <>
struct F32Traits<10> {
    static constexpr int NGP = 4;
    __device__ static const double* dN(int g) { return c_f10_dN + g * 30; }
    __device__ static double w(int g) { return c_f10_w[g]; }
};

// Element index fastest in every array: a warp reads 32 consecutive words, no bank conflicts.
template <int NPE, int NGP>
struct F32Smem {
    static constexpr int MAXP = NPE / 2;  // pair slots per owner node
    union {
        struct {
            double x0[NPE][3][kE];
            double u[NPE][3][kE];
        } nod;  // phase 1
        struct {
            float h[NGP][NPE][3][kE];
            float bh[NGP][NPE][3][kE];
        } grad;                          // phases 2-3
        float blk[NPE][MAXP][9][kE];     // phase 4: the owners' blocks K_IJ
    } a;
    uint32_t off[NPE][MAXP][2][kE];  // SELL offsets of K_IJ and K_JI of every owned pair
    double gci[NGP][9][kE];  // inverse current Jacobian, Gci[c][r]
    double sig[NGP][6][kE];  // dvol sigma: xx yy zz xy yz xz
    float b32[NGP][6][kE];   // b = F F^T: xx yy zz xy yz xz
    float fac[NGP][5][kE];   // dvol {c1, c2, c3, f4, f9}
};

__device__ __forceinline__ double det3d(const double A[3][3]) {
    return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

__device__ __forceinline__ void inv3d(const double A[3][3], double det, double Ai[3][3]) {
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

template <int NPE>
__global__ void __launch_bounds__(kE * NPE, NPE == 8 ? 2 : 1) elem_f32_kernel(ElemArgs a) {
    using T = F32Traits<NPE>;
    constexpr int NGP = T::NGP;
    using Smem = F32Smem<NPE, NGP>;
    constexpr int MAXP = Smem::MAXP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& s = *reinterpret_cast<Smem*>(smem_raw);
    const int e = threadIdx.x % kE;   // lane: element of the CTA
    const int row = threadIdx.x / kE; // warp: node (phases 0, 2-4) or Gauss point (phase 1)
    const int64_t elem = (int64_t)blockIdx.x * kE + e;
    const bool live = elem < a.n_elem;

    // pairs owned by node `row` (phase 3): slot q < MAXP - 1 (and the last slot when npe is odd)
    // J = I + q + 1; the last slot when npe is even: J = I + npe/2, owned by I < npe/2 only
    constexpr bool kEven = (NPE % 2) == 0;
    const int nslots = kEven ? (row < NPE / 2 ? MAXP : MAXP - 1) : MAXP;

    // ---- phase 0: nodal coordinates and displacements of node `row` of every element; the
    // offsets of the owned pairs' blocks are copied to shared memory asynchronously (read in
    // phase 3), and the node's prescribed flags kept for phase 2
    int32_t node = 0;
    uint32_t fixed3 = 0;
    if (live) {
        node = a.conn[elem * NPE + row];
#pragma unroll
        for (int q = 0; q < MAXP; ++q) {
            if (q < nslots) {
                int J = row + q + 1;
                if (J >= NPE) J -= NPE;
                __pipeline_memcpy_async(&s.off[row][q][0][e], &a.e2v[(elem * NPE + row) * NPE + J], sizeof(uint32_t));
                __pipeline_memcpy_async(&s.off[row][q][1][e], &a.e2v[(elem * NPE + J) * NPE + row], sizeof(uint32_t));
            }
        }
        __pipeline_commit();
#pragma unroll
        for (int c = 0; c < 3; ++c) fixed3 |= (uint32_t)(a.fixed[3 * (int64_t)node + c] != 0) << c;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        s.a.nod.x0[row][c][e] = live ? a.coords[3 * (int64_t)node + c] : (c == row % 3 ? 1.0 : 0.0);
        s.a.nod.u[row][c][e] = live ? a.disp[3 * (int64_t)node + c] : 0.0;
    }
    __syncthreads();

    // ---- phase 1: one thread per (element, Gauss point), FP64
    if (row < NGP) {
        const int g = row;
        const double* dN = T::dN(g);
        double G[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, U[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
        for (int I = 0; I < NPE; ++I) {
            double x[3], uu[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                x[c] = s.a.nod.x0[I][c][e];
                uu[c] = s.a.nod.u[I][c][e];
            }
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const double d = dN[r * NPE + I];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    G[r][c] += x[c] * d;
                    U[r][c] += uu[c] * d;
                }
            }
        }
        double Gc[3][3], Gi[3][3], Gci[3][3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) Gc[r][c] = G[r][c] + U[r][c];
        inv3d(G, det3d(G), Gi);
        const double jac = det3d(Gc);
        inv3d(Gc, jac, Gci);
        const double dvol = T::w(g) * jac;
        // F_ij = d_ij + sum_r U[r][i] Gi[j][r]  (= I + sum_I u_I (x) grad0 N_I)
        double F[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
                F[i][j] = (i == j ? 1.0 : 0.0) + (U[0][i] * Gi[j][0] + U[1][i] * Gi[j][1] + U[2][i] * Gi[j][2]);
        const double J = det3d(F);
        if (live && J < 0.0) {
            atomicMin(a.bad, (unsigned long long)elem);
            if (a.bad_elem) a.bad_elem[elem] = 1;
        }
        double b[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
        const double* m = a.mats + 4 * (int64_t)(live ? a.mat_id[elem] : 0);
        const NhFactors f = nh_factors(b, J, m[0], m[1], (int)m[2], a.tangent);
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 3; ++r) s.gci[g][3 * c + r][e] = Gci[c][r];
        const double sv[6] = {b[0][0], b[1][1], b[2][2], b[0][1], b[1][2], b[0][2]};
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            s.sig[g][k][e] = dvol * (f.s1 * sv[k] + (k < 3 ? f.s2 : 0.0));
            s.b32[g][k][e] = (float)sv[k];
        }
        s.fac[g][0][e] = (float)(dvol * f.c1);
        s.fac[g][1][e] = (float)(dvol * f.c2);
        s.fac[g][2][e] = (float)(dvol * f.c3);
        s.fac[g][3][e] = (float)(dvol * f.f4);
        s.fac[g][4][e] = (float)(dvol * f.f9);
    }
    __syncthreads();

    // ---- phase 2: thread (element, node I): h_I per Gauss point, residual in FP64
    const int I = row;
    {
        double R[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int g = 0; g < NGP; ++g) {
            const double* dN = T::dN(g);
            const double d0 = dN[I], d1 = dN[NPE + I], d2 = dN[2 * NPE + I];
            double h[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                h[c] = d0 * s.gci[g][3 * c][e] + d1 * s.gci[g][3 * c + 1][e] + d2 * s.gci[g][3 * c + 2][e];
            const double sxx = s.sig[g][0][e], syy = s.sig[g][1][e], szz = s.sig[g][2][e], sxy = s.sig[g][3][e],
                         syz = s.sig[g][4][e], sxz = s.sig[g][5][e];
            R[0] -= sxx * h[0] + sxy * h[1] + sxz * h[2];
            R[1] -= sxy * h[0] + syy * h[1] + syz * h[2];
            R[2] -= sxz * h[0] + syz * h[1] + szz * h[2];
            const float hf[3] = {(float)h[0], (float)h[1], (float)h[2]};
            const float bxx = s.b32[g][0][e], byy = s.b32[g][1][e], bzz = s.b32[g][2][e], bxy = s.b32[g][3][e],
                        byz = s.b32[g][4][e], bxz = s.b32[g][5][e];
            s.a.grad.h[g][I][0][e] = hf[0];
            s.a.grad.h[g][I][1][e] = hf[1];
            s.a.grad.h[g][I][2][e] = hf[2];
            s.a.grad.bh[g][I][0][e] = bxx * hf[0] + bxy * hf[1] + bxz * hf[2];
            s.a.grad.bh[g][I][1][e] = bxy * hf[0] + byy * hf[1] + byz * hf[2];
            s.a.grad.bh[g][I][2][e] = bxz * hf[0] + byz * hf[1] + bzz * hf[2];
        }
        if (live) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                if (a.reac) atomicAdd(&a.reac[3 * (int64_t)node + c], R[c]);
                if (!((fixed3 >> c) & 1u)) atomicAdd(&a.rhs[3 * (int64_t)node + c], R[c]);
            }
        }
    }
    __syncthreads();

    // ---- phase 3: the tangent blocks of the pairs this thread owns, FP32
    TT acc[MAXP][9];
#pragma unroll
    for (int q = 0; q < MAXP; ++q)
#pragma unroll
        for (int v = 0; v < 9; ++v) acc[q][v] = TT(0);
#pragma unroll 1
    for (int g = 0; g < NGP; ++g) {
        const TT c1 = s.fac[g][0][e], c2 = s.fac[g][1][e], c3 = s.fac[g][2][e], f4 = s.fac[g][3][e],
                 f9 = s.fac[g][4][e];
        TT r[3], p[3], qv[3], sv[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const TT hI = s.a.grad.h[g][I][c][e], bhI = s.a.grad.bh[g][I][c][e];
            r[c] = c1 * hI;
            p[c] = c2 * bhI + c3 * hI;
            qv[c] = c2 * hI;
            sv[c] = f4 * bhI + f9 * hI;
        }
#pragma unroll
        for (int q = 0; q < MAXP; ++q) {
            if (q < nslots) {
                int J = I + q + 1;
                if (J >= NPE) J -= NPE;
                TT hJ[3], bhJ[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    hJ[c] = s.a.grad.h[g][J][c][e];
                    bhJ[c] = s.a.grad.bh[g][J][c][e];
                }
#pragma unroll
                for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                    for (int bb = 0; bb < 3; ++bb)
                        acc[q][3 * aa + bb] += r[bb] * hJ[aa] + p[aa] * hJ[bb] + qv[aa] * bhJ[bb];
                const TT d = sv[0] * hJ[0] + sv[1] * hJ[1] + sv[2] * hJ[2];
                acc[q][0] += d;
                acc[q][4] += d;
                acc[q][8] += d;
            }
        }
    }
    __syncthreads();  // the gradients are read; the block area reuses their space

    // scatter K_IJ and K_JI = K_IJ^T into the FP32 off-diagonal storage; keep K_IJ for phase 4
    if (live) __pipeline_wait_prior(0);  // this thread's offsets (its own copies) have landed
#pragma unroll
    for (int q = 0; q < MAXP; ++q) {
        if (q < nslots) {
#pragma unroll
            for (int v = 0; v < 9; ++v) s.a.blk[I][q][v][e] = (float)acc[q][v];
            if (live) {
                const uint32_t oIJ = s.off[I][q][0][e];
                const uint32_t oJI = s.off[I][q][1][e];
#pragma unroll
                for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                    for (int bb = 0; bb < 3; ++bb) {
                        const float kv = (float)acc[q][3 * aa + bb];
                        atomicAdd(&a.valf[oIJ + 32u * (3 * aa + bb)], kv);
                        atomicAdd(&a.valf[oJI + 32u * (3 * bb + aa)], kv);
                    }
            }
        }
    }
    __syncthreads();

    // ---- phase 4: the element's diagonal block of node I, -sum_{J != I} K_IJ, FP64
    if (live && a.diag_out) {
        double D[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int J = 0; J < NPE; ++J) {
            if (J == I) continue;
            int d = J - I;
            if (d < 0) d += NPE;
            int owner, q;
            if (2 * d < NPE) {
                owner = I;
                q = d - 1;
            } else if (2 * d == NPE) {
                owner = I < J ? I : J;
                q = MAXP - 1;
            } else {
                owner = J;
                q = NPE - d - 1;
            }
            if (owner == I) {
#pragma unroll
                for (int v = 0; v < 9; ++v) D[v] -= (double)s.a.blk[I][q][v][e];
            } else {
#pragma unroll
                for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                    for (int bb = 0; bb < 3; ++bb) D[3 * aa + bb] -= (double)s.a.blk[J][q][3 * bb + aa][e];
            }
        }
#pragma unroll
        for (int v = 0; v < 9; ++v)
            if (a.diag_full || v % 4 == 0) atomicAdd(&a.diag_out[9 * (int64_t)node + v], D[v]);
    }
    // the lift of prescribed increments (applyDirichletBCs): free rows get -sum_J K_IJ lift_J, with
    // K_II = D_I, i.e. -sum_{J != I} K_IJ (lift_J - lift_I)
    if (live && a.lift) {
        const double lI[3] = {a.lift[3 * (int64_t)node], a.lift[3 * (int64_t)node + 1], a.lift[3 * (int64_t)node + 2]};
        double rl[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int J = 0; J < NPE; ++J) {
            if (J == I) continue;
            const int64_t nJ = a.conn[elem * NPE + J];
            const double dl[3] = {a.lift[3 * nJ] - lI[0], a.lift[3 * nJ + 1] - lI[1], a.lift[3 * nJ + 2] - lI[2]};
            int d = J - I;
            if (d < 0) d += NPE;
            const bool own = 2 * d < NPE || (2 * d == NPE && I < J);
            const int q = 2 * d < NPE ? d - 1 : (2 * d == NPE ? MAXP - 1 : NPE - d - 1);
#pragma unroll
            for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                for (int bb = 0; bb < 3; ++bb)
                    rl[aa] += (double)(own ? s.a.blk[I][q][3 * aa + bb][e] : s.a.blk[J][q][3 * bb + aa][e]) * dl[bb];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if ((fixed3 >> c) & 1u) continue;
            atomicAdd(&a.rhs[3 * (int64_t)node + c], -rl[c]);
            if (a.reac) atomicAdd(&a.reac[3 * (int64_t)node + c], -rl[c]);
        }
    }
}

template <int NPE>
void launch_f32(const ElemArgs& a, cudaStream_t s) {
    const size_t smem = sizeof(F32Smem<NPE, F32Traits<NPE>::NGP>);
    static std::atomic<uint64_t> configured{0};
    if (first_use_on_device(configured)) {
        MPHY_CUDA(cudaFuncSetAttribute(elem_f32_kernel<NPE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    const unsigned grid = ceil_div((size_t)a.n_elem, kE);
    if (grid == 0) return;
    elem_f32_kernel<NPE><<<grid, kE * NPE, smem, s>>>(a);
    MPHY_CUDA(cudaGetLastError());
}

}  // namespace

void upload_shape_tables_f32(const double* h8, const double* w8, const double* t10, const double* w4) {
    MPHY_CUDA(cudaMemcpyToSymbol(c_f8_dN, h8, sizeof(double) * 8 * 3 * 8));
    MPHY_CUDA(cudaMemcpyToSymbol(c_f8_w, w8, sizeof(double) * 8));
    MPHY_CUDA(cudaMemcpyToSymbol(c_f10_dN, t10, sizeof(double) * 4 * 3 * 10));
    MPHY_CUDA(cudaMemcpyToSymbol(c_f10_w, w4, sizeof(double) * 4));
}

void launch_elem_f32(const ElemArgs& a, int npe, cudaStream_t s) {
    MPHY_REQUIRE(a.valf && a.rhs && a.e2v && a.fixed, MPHY_ERR_INVALID_ARG, "mixed element kernel: assembly only");
    if (npe == 8) launch_f32<8>(a, s);
    else launch_f32<10>(a, s);
}

}  // namespace mphy
