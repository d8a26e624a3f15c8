// elem_gen.cu -- element kernel for any hyperelastic model of the material table, and the batched
// material call over the same models.
//
// Replaces Elem_Solid_3D_Disp::calcStiffnessAndResidual (Elem_Solid_3D_Disp.cpp:196-373) with
// MaterialBase::computeStressAndTangent dispatched to Matl_NeoHookean, Matl_MooneyRivlin,
// Matl_Gent or Matl_ArrudaBoyce per element (utilitiesmaterialHyperelastic.cpp:186-677). The
// reference's contraction with the dense 9x9 tangent is kept:
//     K_IJ(a, b) = sum_gp dvol sum_{m,n} h_mI C(a + 3m, b + 3n) h_nJ
// evaluated per Gauss point as Gc_I(a, q) = sum_m h_mI C(a + 3m, q) (81 FMAs per row node), then
// K_IJ(a, b) += sum_n Gc_I(a, b + 3n) h_nJ (27 FMAs per block).
//
// Layout: one element per group of NPE * NCH threads. Phase 1: one thread per Gauss point builds
// F, the spatial gradients h and dvol * {sigma, C} in shared memory. Phase 2: thread (I, ch) owns
// row node I and the column nodes J of chunk ch (4 per chunk), so the 9 * 4 accumulators stay in
// registers; chunk 0 also forms the residual of node I.
#include <vector>

#include "common.cuh"
#include "elem.cuh"
#include "elem_store.cuh"
#include "mat.cuh"
#include "mixed.cuh"

namespace mphy {

namespace {

// This translation unit's copy of the shape tables (dN/dxi at the Gauss points and the weights),
// filled by upload_shape_tables_gen from the host tables of elem.cu.
__constant__ double g_hex8_dN[8 * 3 * 8];
__constant__ double g_hex8_w[8];
__constant__ double g_tet10_dN[4 * 3 * 10];
__constant__ double g_tet10_w[4];

template <int NPE>
struct GenTraits;
template <>
struct GenTraits<8> {
    static constexpr int NGP = 8;
    static constexpr int PAD = 2;  // element stride 962 doubles: two elements of a warp on distinct banks
    __device__ static const double* dN(int gp) { return g_hex8_dN + gp * 3 * 8; }
    __device__ static double w(int gp) { return g_hex8_w[gp]; }
};
template <>
struct GenTraits<10> {
    static constexpr int NGP = 4;
    static constexpr int PAD = 6;  // element stride 546 doubles
    __device__ static const double* dN(int gp) { return g_tet10_dN + gp * 3 * 10; }
    __device__ static double w(int gp) { return g_tet10_w[gp]; }
};

constexpr int kGenEpb = 8;  // elements per CTA
constexpr int kGenCh = 4;   // column nodes per thread

template <int NPE>
struct GenSmem {
    static constexpr int NGP = GenTraits<NPE>::NGP;
    double x0[NPE][3];
    double u[NPE][3];
    double h[NGP][NPE][3];
    double C[NGP][81];   // dvol * C
    double sig[NGP][9];  // dvol * sigma
    double pad[GenTraits<NPE>::PAD];
};

__device__ __forceinline__ double det3g(const double A[3][3]) {
    return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

__device__ __forceinline__ void inv3g(const double A[3][3], double det, double Ai[3][3]) {
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

__device__ __forceinline__ void square3(const double b[3][3], double b2[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) b2[i][j] = b[i][0] * b[0][j] + b[i][1] * b[1][j] + b[i][2] * b[2][j];
}

// MODE bit 1: export Ke/Re; bit 2: scatter into the matrix / rhs / reactions.
template <int NPE, int MODE>
__global__ void __launch_bounds__(kGenEpb * NPE * ((NPE + kGenCh - 1) / kGenCh))
    elem_gen_kernel(ElemArgs a) {
    using T = GenTraits<NPE>;
    constexpr int NGP = T::NGP;
    constexpr int NCH = (NPE + kGenCh - 1) / kGenCh;
    constexpr int TPE = NPE * NCH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto* S = reinterpret_cast<GenSmem<NPE>*>(smem_raw);
    const int el = threadIdx.x / TPE, loc = threadIdx.x % TPE;
    const int I = loc % NPE, ch = loc / NPE;
    const int64_t e = (int64_t)blockIdx.x * kGenEpb + el;
    const bool live = e < a.n_elem;
    GenSmem<NPE>& s = S[el];

    int32_t node = 0;
    if (live) {
        node = a.conn[e * NPE + I];
        if (ch == 0) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                s.x0[I][d] = a.coords[3 * (int64_t)node + d];
                s.u[I][d] = a.disp[3 * (int64_t)node + d];
            }
        }
    }
    __syncthreads();

    // ---- phase 1: one thread per Gauss point
    if (live && loc < NGP) {
        const int gp = loc;
        const double* dN = T::dN(gp);
        double G[3][3] = {{0}}, Gc[3][3] = {{0}};
#pragma unroll
        for (int n = 0; n < NPE; ++n)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const double d = dN[r * NPE + n];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    G[r][c] += s.x0[n][c] * d;
                    Gc[r][c] += (s.x0[n][c] + s.u[n][c]) * d;
                }
            }
        double Gi[3][3], Gci[3][3];
        inv3g(G, det3g(G), Gi);
        const double jac = det3g(Gc);
        inv3g(Gc, jac, Gci);
        const double dvol = T::w(gp) * jac;
        // F = I + sum_n u_n (x) grad0 N_n   (ElementBase.cpp:334-361)
        double F[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
        for (int n = 0; n < NPE; ++n) {
            double g0[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                g0[c] = dN[n] * Gi[c][0] + dN[NPE + n] * Gi[c][1] + dN[2 * NPE + n] * Gi[c][2];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int m = 0; m < 3; ++m) F[i][m] += s.u[n][i] * g0[m];
            double h[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                h[c] = dN[n] * Gci[c][0] + dN[NPE + n] * Gci[c][1] + dN[2 * NPE + n] * Gci[c][2];
                s.h[gp][n][c] = h[c];
            }
        }
        const double J = det3g(F);
        if (J < 0.0) {
            atomicMin(a.bad, (unsigned long long)e);
            if (a.bad_elem) a.bad_elem[e] = 1;
        }
        double b[3][3], b2[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
        square3(b, b2);
        double row[kMatRow];
#pragma unroll
        for (int q = 0; q < kMatRow; ++q) row[q] = a.matx[kMatRow * (int64_t)a.mat_id[e] + q];
        const MatScalars m = material_scalars(row, a.tangent, b, b2, J);
        material_fill(m, b, b2, dvol, s.sig[gp], s.C[gp]);
    }
    __syncthreads();
    if (!live) return;

    // ---- phase 2: thread (I, ch)
    bool freeI[3] = {true, true, true};
    if (MODE & 2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) freeI[c] = a.fixed[3 * (int64_t)node + c] == 0;
    }
    if (ch == 0) {
        // R_I(a) = -sum_gp dvol sum_m h_mI sigma(a, m)   (Elem_Solid_3D_Disp.cpp:328-334)
        double R[3] = {0, 0, 0};
#pragma unroll
        for (int gp = 0; gp < NGP; ++gp)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                R[c] -= s.h[gp][I][0] * s.sig[gp][c] + s.h[gp][I][1] * s.sig[gp][3 + c] +
                        s.h[gp][I][2] * s.sig[gp][6 + c];
        store_residual<NPE, MODE>(a, e, I, node, freeI, R);
    }
    const int J0 = ch * kGenCh;
    double acc[kGenCh][9];
#pragma unroll
    for (int j = 0; j < kGenCh; ++j)
#pragma unroll
        for (int v = 0; v < 9; ++v) acc[j][v] = 0.0;
#pragma unroll 1
    for (int gp = 0; gp < NGP; ++gp) {
        const double h0 = s.h[gp][I][0], h1 = s.h[gp][I][1], h2 = s.h[gp][I][2];
        const double* C = s.C[gp];
        double Gc[3][9];
#pragma unroll
        for (int aa = 0; aa < 3; ++aa)
#pragma unroll
            for (int q = 0; q < 9; ++q) Gc[aa][q] = h0 * C[9 * aa + q] + h1 * C[9 * (3 + aa) + q] + h2 * C[9 * (6 + aa) + q];
#pragma unroll
        for (int j = 0; j < kGenCh; ++j) {
            if (J0 + j < NPE) {
                const double g0 = s.h[gp][J0 + j][0], g1 = s.h[gp][J0 + j][1], g2 = s.h[gp][J0 + j][2];
#pragma unroll
                for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                    for (int bb = 0; bb < 3; ++bb)
                        acc[j][3 * aa + bb] += Gc[aa][bb] * g0 + Gc[aa][3 + bb] * g1 + Gc[aa][6 + bb] * g2;
            }
        }
    }
    double rl[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 0; j < kGenCh; ++j) {
        const int J = J0 + j;
        if (J < NPE) {
            lift_block<NPE, MODE>(a, e, J, acc[j], rl);
            store_block<NPE, MODE>(a, e, I, J, node, freeI, acc[j]);
        }
    }
    store_lift<NPE, MODE>(a, node, freeI, rl);
}

template <int NPE, int MODE>
void launch_gen(const ElemArgs& a, cudaStream_t s) {
    constexpr int TPE = NPE * ((NPE + kGenCh - 1) / kGenCh);
    const size_t smem = kGenEpb * sizeof(GenSmem<NPE>);
    static std::atomic<uint64_t> configured{0};
    if (first_use_on_device(configured)) {
        MPHY_CUDA(cudaFuncSetAttribute(elem_gen_kernel<NPE, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    }
    const unsigned grid = ceil_div((size_t)a.n_elem, kGenEpb);
    if (grid == 0) return;
    elem_gen_kernel<NPE, MODE><<<grid, kGenEpb * TPE, smem, s>>>(a);
    MPHY_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------- mixed u-p element (Mixed1)
// ElementBase::calcStiffnessAndResidualMixed3D (ElementBase2.cpp:278-553) for Elem_Solid_3D_Mixed1:
//   - tet10: quadratic displacement, linear pressure on the four vertex nodes (basis the
//     barycentric coordinates, LagrangeBasisFunsTetra(4)), the 4-point rule;
//   - hex27 (P2-P1): triquadratic displacement, trilinear pressure on the eight corner nodes
//     (LagrangeBasisFunsHexa(8)), the 3x3x3 rule that getGaussPoints3D gives a 27-node hex.
// Per Gauss point: F from u, Fn from the last converged step (Jn, then Jhat = Jn - U'(Jn)/U''(Jn),
// thetahat = 1/U''(Jn)), p = sum Np_i p_i, the mixed material branch, and
//   Kup(3I+a, j) = sum dvol h_aI Np_j = Kpu(j, 3I+a),   Kpp(i, j) = -sum dvol0 thetahat Np_i Np_j,
//   FP(i) = -sum dvol0 Np_i (J - Jhat - thetahat p),    Kuu and FU as the displacement element.

// hex27 tables in global memory (the 27 Gauss-point threads read different points at once, which
// the constant cache would serialise): dN/dxi [gp][3][27], weights [gp], trilinear Np [gp][8]
__device__ double g_hex27_dN[27 * 3 * 27];
__device__ double g_hex27_w[27];
__device__ double g_hex27_np[27 * 8];

// tet 4-point rule (QuadratureUtil.cpp:690-712) points in barycentric form: Np(gp, i)
__device__ __forceinline__ double tet4_np(int gp, int i) {
    const double a = 0.1381966011250105, b = 0.5854101966249685;
    if (i == 0) return gp == 0 ? 1.0 - 3.0 * a : 1.0 - b - 2.0 * a;
    return gp == i ? b : a;
}

template <int NPE>
struct MixedTraits;
template <>
struct MixedTraits<10> {
    static constexpr int NGP = 4, NP = 4, EPB = kGenEpb;
    static constexpr int PAD = 8;  // element stride 594 doubles
    __device__ static const double* dN(int gp) { return GenTraits<10>::dN(gp); }
    __device__ static double w(int gp) { return GenTraits<10>::w(gp); }
    __device__ static double np(int gp, int i) { return tet4_np(gp, i); }
};
template <>
struct MixedTraits<27> {
    static constexpr int NGP = 27, NP = 8, EPB = 1;  // one element (189 threads, 39 KB) per CTA
    static constexpr int PAD = 0;
    __device__ static const double* dN(int gp) { return g_hex27_dN + gp * 3 * 27; }
    __device__ static double w(int gp) { return g_hex27_w[gp]; }
    __device__ static double np(int gp, int i) { return g_hex27_np[gp * 8 + i]; }
};

template <int NPE>
struct MixedSmem {
    static constexpr int NGP = MixedTraits<NPE>::NGP;
    double x0[NPE][3];
    double u[NPE][3];
    double up[NPE][3];
    double h[NGP][NPE][3];
    double C[NGP][81];
    double sig[NGP][9];
    double dvol[NGP], dvol0[NGP], th[NGP], resip[NGP];
    double pad[MixedTraits<NPE>::PAD > 0 ? MixedTraits<NPE>::PAD : 1];
};

template <int NPE>
constexpr int mixed_tpe() { return NPE * ((NPE + kGenCh - 1) / kGenCh); }

template <int NPE, int MODE>
__global__ void __launch_bounds__(MixedTraits<NPE>::EPB * mixed_tpe<NPE>()) elem_mixed_kernel(MixedElemArgs ma) {
    const ElemArgs& a = ma.base;
    using T = MixedTraits<NPE>;
    constexpr int NGP = T::NGP, NP = T::NP, TPE = mixed_tpe<NPE>(), NS = 3 * NPE;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto* S = reinterpret_cast<MixedSmem<NPE>*>(smem_raw);
    const int el = threadIdx.x / TPE, loc = threadIdx.x % TPE;
    const int I = loc % NPE, ch = loc / NPE;
    const int64_t e = (int64_t)blockIdx.x * T::EPB + el;
    const bool live = e < a.n_elem;
    MixedSmem<NPE>& s = S[el];

    int32_t node = 0;
    if (live) {
        node = a.conn[e * NPE + I];
        if (ch == 0) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                s.x0[I][d] = a.coords[3 * (int64_t)node + d];
                s.u[I][d] = a.disp[3 * (int64_t)node + d];
                s.up[I][d] = ma.disp_prev[3 * (int64_t)node + d];
            }
        }
    }
    __syncthreads();

    if (live && loc < NGP) {
        const int gp = loc;
        const double* dN = T::dN(gp);
        double G[3][3] = {{0}}, Gc[3][3] = {{0}};
#pragma unroll
        for (int n = 0; n < NPE; ++n)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const double d = dN[r * NPE + n];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    G[r][c] += s.x0[n][c] * d;
                    Gc[r][c] += (s.x0[n][c] + s.u[n][c]) * d;
                }
            }
        double Gi[3][3], Gci[3][3];
        const double jac0 = det3g(G);
        inv3g(G, jac0, Gi);
        const double jac = det3g(Gc);
        inv3g(Gc, jac, Gci);
        const double dvol = T::w(gp) * jac, dvol0 = T::w(gp) * jac0;
        double F[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, Fn[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
        for (int n = 0; n < NPE; ++n) {
            double g0[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                g0[c] = dN[n] * Gi[c][0] + dN[NPE + n] * Gi[c][1] + dN[2 * NPE + n] * Gi[c][2];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    F[i][m] += s.u[n][i] * g0[m];
                    Fn[i][m] += s.up[n][i] * g0[m];
                }
#pragma unroll
            for (int c = 0; c < 3; ++c)
                s.h[gp][n][c] = dN[n] * Gci[c][0] + dN[NPE + n] * Gci[c][1] + dN[2 * NPE + n] * Gci[c][2];
        }
        const double J = det3g(F);
        if (J < 0.0) {
            atomicMin(a.bad, (unsigned long long)e);
            if (a.bad_elem) a.bad_elem[e] = 1;
        }
        double row[kMatRow];
#pragma unroll
        for (int q = 0; q < kMatRow; ++q) row[q] = a.matx[kMatRow * (int64_t)a.mat_id[e] + q];
        // compute_constants_volumetric_functions (utilitiesmaterialHyperelastic.cpp:144-173)
        double Jhat = 1.0, th = 0.0;
        const int utype = (int)row[6];
        if (utype != -1) {
            double d1, d2;
            const double Jn = det3g(Fn);
            vol_derivs(utype, 1.0 / row[5], Jn, d1, d2);
            Jhat = Jn - d1 / d2;
            th = 1.0 / d2;
        }
        double pres = 0.0;
#pragma unroll
        for (int i = 0; i < NP; ++i) pres += T::np(gp, i) * ma.pres[a.conn[e * NPE + i]];
        double b[3][3], b2[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
        square3(b, b2);
        const MatScalars m = material_scalars(row, a.tangent, b, b2, J, true, pres);
        material_fill(m, b, b2, dvol, s.sig[gp], s.C[gp]);
        s.dvol[gp] = dvol;
        s.dvol0[gp] = dvol0;
        s.th[gp] = th;
        s.resip[gp] = J - Jhat - th * pres;
    }
    __syncthreads();
    if (!live) return;

    bool freeI[3] = {true, true, true};
    if (MODE & 2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) freeI[c] = a.fixed[3 * (int64_t)node + c] == 0;
    }
    if (ch == 0) {
        double R[3] = {0, 0, 0};
        double kup[3][NP] = {{0}};
#pragma unroll
        for (int gp = 0; gp < NGP; ++gp) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                R[c] -= s.h[gp][I][0] * s.sig[gp][c] + s.h[gp][I][1] * s.sig[gp][3 + c] +
                        s.h[gp][I][2] * s.sig[gp][6 + c];
#pragma unroll
                for (int j = 0; j < NP; ++j) kup[c][j] += s.dvol[gp] * s.h[gp][I][c] * T::np(gp, j);
            }
        }
        store_residual<NPE, MODE>(a, e, I, node, freeI, R);
        if (MODE & 1) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int j = 0; j < NP; ++j) ma.Kup[(e * NS + 3 * I + c) * NP + j] = kup[c][j];
        }
        if (MODE & 2) {
#pragma unroll
            for (int j = 0; j < NP; ++j) {
                const uint32_t ib = ma.e2b[(e * NPE + I) * NP + j], it = ma.e2bt[(e * NP + j) * NPE + I];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    if (!freeI[c]) continue;
                    atomicAdd(&ma.bval[3 * (int64_t)ib + c], kup[c][j]);
                    atomicAdd(&ma.btval[3 * (int64_t)it + c], kup[c][j]);
                }
            }
        }
    } else if (ch == 1 && I < NP) {
        // pressure row i = I (a vertex / corner node)
        double fp = 0.0, kpp[NP] = {0};
#pragma unroll
        for (int gp = 0; gp < NGP; ++gp) {
            const double w = s.dvol0[gp] * T::np(gp, I);
            fp -= w * s.resip[gp];
#pragma unroll
            for (int j = 0; j < NP; ++j) kpp[j] -= w * s.th[gp] * T::np(gp, j);
        }
        if (MODE & 1) {
            ma.FP[e * NP + I] = fp;
#pragma unroll
            for (int j = 0; j < NP; ++j) ma.Kpp[(e * NP + I) * NP + j] = kpp[j];
        }
        if (MODE & 2) {
            atomicAdd(&ma.rhs_p[ma.pres_id[node]], fp);
#pragma unroll
            for (int j = 0; j < NP; ++j) atomicAdd(&ma.cval[ma.e2c[(e * NP + I) * NP + j]], kpp[j]);
        }
    }
    // Kuu: thread (I, ch), column nodes 4 ch .. 4 ch + 3
    const int J0 = ch * kGenCh;
    double acc[kGenCh][9];
#pragma unroll
    for (int j = 0; j < kGenCh; ++j)
#pragma unroll
        for (int v = 0; v < 9; ++v) acc[j][v] = 0.0;
#pragma unroll 1
    for (int gp = 0; gp < NGP; ++gp) {
        const double h0 = s.h[gp][I][0], h1 = s.h[gp][I][1], h2 = s.h[gp][I][2];
        const double* C = s.C[gp];
        double Gc[3][9];
#pragma unroll
        for (int aa = 0; aa < 3; ++aa)
#pragma unroll
            for (int q = 0; q < 9; ++q) Gc[aa][q] = h0 * C[9 * aa + q] + h1 * C[9 * (3 + aa) + q] + h2 * C[9 * (6 + aa) + q];
#pragma unroll
        for (int j = 0; j < kGenCh; ++j) {
            if (J0 + j < NPE) {
                const double g0 = s.h[gp][J0 + j][0], g1 = s.h[gp][J0 + j][1], g2 = s.h[gp][J0 + j][2];
#pragma unroll
                for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                    for (int bb = 0; bb < 3; ++bb)
                        acc[j][3 * aa + bb] += Gc[aa][bb] * g0 + Gc[aa][3 + bb] * g1 + Gc[aa][6 + bb] * g2;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < kGenCh; ++j) {
        const int J = J0 + j;
        if (J < NPE) store_block<NPE, MODE>(a, e, I, J, node, freeI, acc[j]);
    }
}

template <int NPE, int MODE>
void launch_mixed(const MixedElemArgs& a, cudaStream_t s) {
    using T = MixedTraits<NPE>;
    const size_t smem = T::EPB * sizeof(MixedSmem<NPE>);
    static std::atomic<uint64_t> configured{0};
    if (first_use_on_device(configured)) {
        MPHY_CUDA(cudaFuncSetAttribute(elem_mixed_kernel<NPE, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    }
    const unsigned grid = ceil_div((size_t)a.base.n_elem, T::EPB);
    if (grid == 0) return;
    elem_mixed_kernel<NPE, MODE><<<grid, T::EPB * mixed_tpe<NPE>(), smem, s>>>(a);
    MPHY_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------- constant-pressure u-p element
// Elem_Solid_3D_Mixed0: ElementBase::calcStiffnessAndResidualMixed3D with one pressure function
// (nlbfP = 1, Np = 1, p = the element's pressure; ElementBase2.cpp:385-389) on the hex8 or tet10
// displacement element, then the condensation of Elem_Solid_3D_Mixed0::calcStiffnessAndResidual
// (Elem_Solid_3D_Mixed0.cpp:93-101):
//   K = Kuu - Kup Kpu / Kpp,   F = FU - Kup FP / Kpp,
// with Kup(3I+a) = sum dvol h_aI = Kpu(3I+a), Kpp = -sum dvol0 thetahat and
// FP = -sum dvol0 (J - Jhat - thetahat p). Kup, Kpp and FP are kept per element for the pressure
// update after the solve (Elem_Solid_3D_Mixed0::solveForPressure, :112-200).
template <int NPE>
struct P0Smem {
    static constexpr int NGP = GenTraits<NPE>::NGP;
    double x0[NPE][3];
    double u[NPE][3];
    double up[NPE][3];
    double h[NGP][NPE][3];
    double C[NGP][81];   // dvol * C
    double sig[NGP][9];  // dvol * sigma
    double dvol[NGP], dvol0[NGP], th[NGP], resip[NGP];
    double kup[NPE][3];
    double kpp, fp;
    double pad[2];
};

template <int NPE, int MODE>
__global__ void __launch_bounds__(kGenEpb * NPE * ((NPE + kGenCh - 1) / kGenCh)) elem_mixed0_kernel(MixedElemArgs ma) {
    const ElemArgs& a = ma.base;
    using T = GenTraits<NPE>;
    constexpr int NGP = T::NGP, NCH = (NPE + kGenCh - 1) / kGenCh, TPE = NPE * NCH, NS = 3 * NPE;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto* S = reinterpret_cast<P0Smem<NPE>*>(smem_raw);
    const int el = threadIdx.x / TPE, loc = threadIdx.x % TPE;
    const int I = loc % NPE, ch = loc / NPE;
    const int64_t e = (int64_t)blockIdx.x * kGenEpb + el;
    const bool live = e < a.n_elem;
    P0Smem<NPE>& s = S[el];

    int32_t node = 0;
    if (live) {
        node = a.conn[e * NPE + I];
        if (ch == 0) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                s.x0[I][d] = a.coords[3 * (int64_t)node + d];
                s.u[I][d] = a.disp[3 * (int64_t)node + d];
                s.up[I][d] = ma.disp_prev[3 * (int64_t)node + d];
            }
        }
    }
    __syncthreads();

    if (live && loc < NGP) {
        const int gp = loc;
        const double* dN = T::dN(gp);
        double G[3][3] = {{0}}, Gc[3][3] = {{0}};
#pragma unroll
        for (int n = 0; n < NPE; ++n)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const double d = dN[r * NPE + n];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    G[r][c] += s.x0[n][c] * d;
                    Gc[r][c] += (s.x0[n][c] + s.u[n][c]) * d;
                }
            }
        double Gi[3][3], Gci[3][3];
        const double jac0 = det3g(G);
        inv3g(G, jac0, Gi);
        const double jac = det3g(Gc);
        inv3g(Gc, jac, Gci);
        const double dvol = T::w(gp) * jac, dvol0 = T::w(gp) * jac0;
        double F[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, Fn[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
        for (int n = 0; n < NPE; ++n) {
            double g0[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                g0[c] = dN[n] * Gi[c][0] + dN[NPE + n] * Gi[c][1] + dN[2 * NPE + n] * Gi[c][2];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int m = 0; m < 3; ++m) {
                    F[i][m] += s.u[n][i] * g0[m];
                    Fn[i][m] += s.up[n][i] * g0[m];
                }
#pragma unroll
            for (int c = 0; c < 3; ++c)
                s.h[gp][n][c] = dN[n] * Gci[c][0] + dN[NPE + n] * Gci[c][1] + dN[2 * NPE + n] * Gci[c][2];
        }
        const double J = det3g(F);
        if (J < 0.0) {
            atomicMin(a.bad, (unsigned long long)e);
            if (a.bad_elem) a.bad_elem[e] = 1;
        }
        double row[kMatRow];
#pragma unroll
        for (int q = 0; q < kMatRow; ++q) row[q] = a.matx[kMatRow * (int64_t)a.mat_id[e] + q];
        // compute_constants_volumetric_functions (utilitiesmaterialHyperelastic.cpp:144-173)
        double Jhat = 1.0, th = 0.0;
        const int utype = (int)row[6];
        if (utype != -1) {
            double d1, d2;
            const double Jn = det3g(Fn);
            vol_derivs(utype, 1.0 / row[5], Jn, d1, d2);
            Jhat = Jn - d1 / d2;
            th = 1.0 / d2;
        }
        const double pres = ma.pe[e];
        double b[3][3], b2[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
        square3(b, b2);
        const MatScalars m = material_scalars(row, a.tangent, b, b2, J, true, pres);
        material_fill(m, b, b2, dvol, s.sig[gp], s.C[gp]);
        s.dvol[gp] = dvol;
        s.dvol0[gp] = dvol0;
        s.th[gp] = th;
        s.resip[gp] = J - Jhat - th * pres;
    }
    __syncthreads();
    // the coupling column, Kpp and FP of the element (fixed Gauss-point order)
    if (live && ch == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double k = 0.0;
#pragma unroll
            for (int gp = 0; gp < NGP; ++gp) k += s.dvol[gp] * s.h[gp][I][c];
            s.kup[I][c] = k;
        }
        if (I == 0) {
            double kpp = 0.0, fp = 0.0;
#pragma unroll
            for (int gp = 0; gp < NGP; ++gp) {
                kpp -= s.dvol0[gp] * s.th[gp];
                fp -= s.dvol0[gp] * s.resip[gp];
            }
            s.kpp = kpp;
            s.fp = fp;
        }
    }
    __syncthreads();
    if (!live) return;

    bool freeI[3] = {true, true, true};
    if (MODE & 2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) freeI[c] = a.fixed[3 * (int64_t)node + c] == 0;
    }
    const double rkpp = 1.0 / s.kpp;
    if (ch == 0) {
        double R[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double r = 0.0;
#pragma unroll
            for (int gp = 0; gp < NGP; ++gp)
                r -= s.h[gp][I][0] * s.sig[gp][c] + s.h[gp][I][1] * s.sig[gp][3 + c] + s.h[gp][I][2] * s.sig[gp][6 + c];
            R[c] = r - s.kup[I][c] * (s.fp * rkpp);
            if (ma.kup_e) ma.kup_e[e * NS + 3 * I + c] = s.kup[I][c];
        }
        store_residual<NPE, MODE>(a, e, I, node, freeI, R);
        if (I == 0) {
            if (ma.kpp_e) ma.kpp_e[e] = s.kpp;
            if (ma.fp_e) ma.fp_e[e] = s.fp;
        }
    }
    // Kuu - Kup Kpu / Kpp: thread (I, ch), column nodes 4 ch .. 4 ch + 3
    const int J0 = ch * kGenCh;
    double acc[kGenCh][9];
#pragma unroll
    for (int j = 0; j < kGenCh; ++j)
#pragma unroll
        for (int v = 0; v < 9; ++v) acc[j][v] = 0.0;
#pragma unroll 1
    for (int gp = 0; gp < NGP; ++gp) {
        const double h0 = s.h[gp][I][0], h1 = s.h[gp][I][1], h2 = s.h[gp][I][2];
        const double* C = s.C[gp];
        double Gc[3][9];
#pragma unroll
        for (int aa = 0; aa < 3; ++aa)
#pragma unroll
            for (int q = 0; q < 9; ++q) Gc[aa][q] = h0 * C[9 * aa + q] + h1 * C[9 * (3 + aa) + q] + h2 * C[9 * (6 + aa) + q];
#pragma unroll
        for (int j = 0; j < kGenCh; ++j) {
            if (J0 + j < NPE) {
                const double g0 = s.h[gp][J0 + j][0], g1 = s.h[gp][J0 + j][1], g2 = s.h[gp][J0 + j][2];
#pragma unroll
                for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                    for (int bb = 0; bb < 3; ++bb)
                        acc[j][3 * aa + bb] += Gc[aa][bb] * g0 + Gc[aa][3 + bb] * g1 + Gc[aa][6 + bb] * g2;
            }
        }
    }
    double rl[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 0; j < kGenCh; ++j) {
        const int J = J0 + j;
        if (J < NPE) {
#pragma unroll
            for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                for (int bb = 0; bb < 3; ++bb) acc[j][3 * aa + bb] -= s.kup[I][aa] * s.kup[J][bb] * rkpp;
            lift_block<NPE, MODE>(a, e, J, acc[j], rl);
            store_block<NPE, MODE>(a, e, I, J, node, freeI, acc[j]);
        }
    }
    store_lift<NPE, MODE>(a, node, freeI, rl);
}

template <int NPE, int MODE>
void launch_mixed0(const MixedElemArgs& a, cudaStream_t s) {
    constexpr int TPE = NPE * ((NPE + kGenCh - 1) / kGenCh);
    const size_t smem = kGenEpb * sizeof(P0Smem<NPE>);
    static std::atomic<uint64_t> configured{0};
    if (first_use_on_device(configured)) {
        MPHY_CUDA(cudaFuncSetAttribute(elem_mixed0_kernel<NPE, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    }
    const unsigned grid = ceil_div((size_t)a.base.n_elem, kGenEpb);
    if (grid == 0) return;
    elem_mixed0_kernel<NPE, MODE><<<grid, kGenEpb * TPE, smem, s>>>(a);
    MPHY_CUDA(cudaGetLastError());
}

// p_e += (FP - Kpu du_e) / Kpp, one thread per element
template <int NPE>
__global__ void pressure_update_p0_kernel(int64_t n_elem, const int32_t* __restrict__ conn, const double* __restrict__ du,
                                          const double* __restrict__ kup_e, const double* __restrict__ kpp_e,
                                          const double* __restrict__ fp_e, double* __restrict__ pe) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n_elem; e += (int64_t)gridDim.x * blockDim.x) {
        double v = 0.0;
#pragma unroll
        for (int I = 0; I < NPE; ++I) {
            const int64_t n = conn[e * NPE + I];
#pragma unroll
            for (int c = 0; c < 3; ++c) v += kup_e[e * 3 * NPE + 3 * I + c] * du[3 * n + c];
        }
        pe[e] += (fp_e[e] - v) / kpp_e[e];
    }
}

// Batched material call: F [n][9] row-major -> sigma [n][9], C [n][81] (reference index order).
__global__ void material_eval_kernel(int n, const double* __restrict__ Fm, const double* __restrict__ row_in,
                                     int tangent, double* __restrict__ stre, double* __restrict__ Cout) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double F[3][3], b[3][3], b2[3][3];
#pragma unroll
    for (int i = 0; i < 9; ++i) F[i / 3][i % 3] = Fm[9 * (int64_t)t + i];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
    square3(b, b2);
    double row[kMatRow];
#pragma unroll
    for (int q = 0; q < kMatRow; ++q) row[q] = row_in[q];
    const MatScalars m = material_scalars(row, tangent, b, b2, det3g(F));
    material_fill(m, b, b2, 1.0, stre + 9 * (int64_t)t, Cout + 81 * (int64_t)t);
}

}  // namespace

void upload_shape_tables_gen(const double* h8, const double* w8, const double* t10, const double* w4) {
    MPHY_CUDA(cudaMemcpyToSymbol(g_hex8_dN, h8, sizeof(g_hex8_dN)));
    MPHY_CUDA(cudaMemcpyToSymbol(g_hex8_w, w8, sizeof(g_hex8_w)));
    MPHY_CUDA(cudaMemcpyToSymbol(g_tet10_dN, t10, sizeof(g_tet10_dN)));
    MPHY_CUDA(cudaMemcpyToSymbol(g_tet10_w, w4, sizeof(g_tet10_w)));
}

void launch_elem_gen(const ElemArgs& a, int npe, int mode, cudaStream_t s) {
    if (npe == 8) {
        if (mode == 1) launch_gen<8, 1>(a, s);
        else if (mode == 2) launch_gen<8, 2>(a, s);
        else launch_gen<8, 3>(a, s);
    } else {
        if (mode == 1) launch_gen<10, 1>(a, s);
        else if (mode == 2) launch_gen<10, 2>(a, s);
        else launch_gen<10, 3>(a, s);
    }
}

// The hex27 tables: the 27-node hex of BasisFunctionsLagrange.cpp:1300-1399 (1D quadratic
// Lagrange triple ordered -1, +1, 0; node a at the 1D indices kHex27Ijk[a]) and the 3x3x3 rule of
// QuadratureUtil.cpp:497-524 (point q at the 1D indices of node q, weights 5/9, 5/9, 8/9),
// with the trilinear pressure basis of the 8 corners at the same points.
void upload_hex27_tables() {
    static const int kHex27Ijk[27][3] = {
        {0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1},
        {2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 2, 0}, {1, 0, 2}, {2, 1, 0}, {1, 1, 2}, {0, 1, 2},
        {2, 0, 1}, {0, 2, 1}, {1, 2, 1}, {2, 1, 1}, {2, 2, 0}, {2, 0, 2}, {0, 2, 2}, {1, 2, 2},
        {2, 1, 2}, {2, 2, 1}, {2, 2, 2}};
    const double g[3] = {-0.774596669241483, 0.774596669241483, 0.0};
    const double wt[3] = {5.0 / 9.0, 5.0 / 9.0, 8.0 / 9.0};
    std::vector<double> dN(27 * 3 * 27), w(27), np(27 * 8);
    for (int q = 0; q < 27; ++q) {
        double xi[3], n1[3][3], d1[3][3], l1[3][2];
        for (int d = 0; d < 3; ++d) {
            const double x = g[kHex27Ijk[q][d]], x2 = x * x;
            xi[d] = x;
            n1[d][0] = 0.5 * (x2 - x);
            n1[d][1] = 0.5 * (x2 + x);
            n1[d][2] = 1.0 - x2;
            d1[d][0] = 0.5 * (2.0 * x - 1.0);
            d1[d][1] = 0.5 * (2.0 * x + 1.0);
            d1[d][2] = -2.0 * x;
            l1[d][0] = 0.5 * (1.0 - x);
            l1[d][1] = 0.5 * (1.0 + x);
        }
        w[q] = wt[kHex27Ijk[q][0]] * wt[kHex27Ijk[q][1]] * wt[kHex27Ijk[q][2]];
        for (int a = 0; a < 27; ++a) {
            const int i = kHex27Ijk[a][0], j = kHex27Ijk[a][1], k = kHex27Ijk[a][2];
            dN[(q * 3 + 0) * 27 + a] = d1[0][i] * n1[1][j] * n1[2][k];
            dN[(q * 3 + 1) * 27 + a] = n1[0][i] * d1[1][j] * n1[2][k];
            dN[(q * 3 + 2) * 27 + a] = n1[0][i] * n1[1][j] * d1[2][k];
        }
        for (int a = 0; a < 8; ++a) {
            const int i = kHex27Ijk[a][0], j = kHex27Ijk[a][1], k = kHex27Ijk[a][2];
            np[q * 8 + a] = l1[0][i] * l1[1][j] * l1[2][k];
        }
        (void)xi;
    }
    MPHY_CUDA(cudaMemcpyToSymbol(g_hex27_dN, dN.data(), dN.size() * sizeof(double)));
    MPHY_CUDA(cudaMemcpyToSymbol(g_hex27_w, w.data(), w.size() * sizeof(double)));
    MPHY_CUDA(cudaMemcpyToSymbol(g_hex27_np, np.data(), np.size() * sizeof(double)));
}

void launch_elem_mixed(const MixedElemArgs& a, int npe, int mode, cudaStream_t s) {
    if (npe == 27) {
        if (mode == 1) launch_mixed<27, 1>(a, s);
        else if (mode == 2) launch_mixed<27, 2>(a, s);
        else launch_mixed<27, 3>(a, s);
    } else {
        if (mode == 1) launch_mixed<10, 1>(a, s);
        else if (mode == 2) launch_mixed<10, 2>(a, s);
        else launch_mixed<10, 3>(a, s);
    }
}

void launch_elem_mixed0(const MixedElemArgs& a, int npe, int mode, cudaStream_t s) {
    if (npe == 8) {
        if (mode == 1) launch_mixed0<8, 1>(a, s);
        else if (mode == 2) launch_mixed0<8, 2>(a, s);
        else launch_mixed0<8, 3>(a, s);
    } else {
        if (mode == 1) launch_mixed0<10, 1>(a, s);
        else if (mode == 2) launch_mixed0<10, 2>(a, s);
        else launch_mixed0<10, 3>(a, s);
    }
}

void launch_pressure_update_p0(int64_t n_elem, int npe, const int32_t* conn, const double* du, const double* kup_e,
                               const double* kpp_e, const double* fp_e, double* pe, cudaStream_t s, int sm) {
    if (n_elem <= 0) return;
    unsigned grid = ceil_div((size_t)n_elem, 256);
    if (grid > (unsigned)sm * 8) grid = sm * 8;
    if (npe == 8) pressure_update_p0_kernel<8><<<grid, 256, 0, s>>>(n_elem, conn, du, kup_e, kpp_e, fp_e, pe);
    else pressure_update_p0_kernel<10><<<grid, 256, 0, s>>>(n_elem, conn, du, kup_e, kpp_e, fp_e, pe);
    MPHY_CUDA(cudaGetLastError());
}

void launch_material_eval(int n, const double* F, const double* row_dev, int tangent, double* stre, double* C,
                          cudaStream_t s) {
    if (n <= 0) return;
    material_eval_kernel<<<ceil_div(n, 128), 128, 0, s>>>(n, F, row_dev, tangent, stre, C);
    MPHY_CUDA(cudaGetLastError());
}

}  // namespace mphy
