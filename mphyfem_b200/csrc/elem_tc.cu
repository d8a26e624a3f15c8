// elem_tc.cu -- mixed-precision element kernel: FP64 kinematics, stress and residual; the
// tangent's contraction on tensor cores with split-BF16 operands and FP32 accumulation.
//
// Replaces the same reference code as elem.cu (Elem_Solid_3D_Disp.cpp:196-373 with the
// Neo-Hookean tangent of utilitiesmaterialHyperelastic.cpp:186-295 and the scatter of
// SolverPetsc.cpp:357-378) for the FP32-stored operator.
//
// The closed form of elem.cu,
//   K_IJ(a,b) = sum_gp c1 h_Ib h_Ja + c2 (b h_I)_a h_Jb + c3 h_Ia h_Jb + c2 h_Ia (b h_J)_b
//               + d_ab (f4 h_I.b h_J + f9 h_I.h_J),
// is a sum over (gp, j) of h_Ij times
//   H_a[(J,b), (gp,j)] = c2 b_aj h_Jb + d_jb c1 h_Ja + d_ja (c3 h_Jb + c2 (b h_J)_b)
//                        + d_ab (f4 (b h_J)_j + f9 h_Jj)            (gp's factors, dvol folded in)
// so for every a one element's tangent is a dense product
//   K[(I,a), (J,b)] = D_a[(J,b), I],   D_a = H_a (3 NPE x 3 NGP)  *  Hn (3 NGP x NPE),
// Hn[(gp,j), I] = h_Ij. hex8: 24 x 24 x 8 per a, tet10: 30 x 12 x 10. A warp computes one
// element's three products with mma.sync m16n8k16 (BF16 in, FP32 accumulate). Every operand x
// is split x = hi + lo with hi = bf16(x), lo = bf16(x - hi); the product keeps hi*hi + hi*lo +
// lo*hi (the dropped lo*lo term is below 2^-16 of the product), so each entry of K is accurate
// to about 1e-5 relative, against 1e-16 for the FP64 kernel and 6e-8 for FP32 storage alone.
// The lanes build their fragments of H_a directly from the per-Gauss-point data in shared
// memory: every entry of H is formed once, with a handful of FMAs.
#include <cuda_bf16.h>

#include "common.cuh"
#include "elem.cuh"
#include "nh.cuh"

namespace mphy {

// the shape tables of elem.cu, uploaded by upload_shape_tables (constant memory is per file)
__constant__ double c_tc_hex8_dN[8 * 3 * 8];
__constant__ double c_tc_hex8_w[8];
__constant__ double c_tc_tet10_dN[4 * 3 * 10];
__constant__ double c_tc_tet10_w[4];

void upload_shape_tables_tc(const double* h8, const double* w8, const double* t10, const double* w4) {
    MPHY_CUDA(cudaMemcpyToSymbol(c_tc_hex8_dN, h8, sizeof(double) * 8 * 3 * 8));
    MPHY_CUDA(cudaMemcpyToSymbol(c_tc_hex8_w, w8, sizeof(double) * 8));
    MPHY_CUDA(cudaMemcpyToSymbol(c_tc_tet10_dN, t10, sizeof(double) * 4 * 3 * 10));
    MPHY_CUDA(cudaMemcpyToSymbol(c_tc_tet10_w, w4, sizeof(double) * 4));
}

namespace {

template <int NPE>
struct TcTraits;
template <>
struct TcTraits<8> {
    static constexpr int NGP = 8;
    __device__ static const double* dN(int gp) { return c_tc_hex8_dN + gp * 3 * 8; }
    __device__ static double w(int gp) { return c_tc_hex8_w[gp]; }
};
template <>
struct TcTraits<10> {
    static constexpr int NGP = 4;
    __device__ static const double* dN(int gp) { return c_tc_tet10_dN + gp * 3 * 10; }
    __device__ static double w(int gp) { return c_tc_tet10_w[gp]; }
};

constexpr int kTcEpb = 16;       // elements per CTA
constexpr int kTcThreads = 256;  // 8 warps

template <int NPE, int NGP>
struct TcSmem {
    double x0[NPE][3];
    double u[NPE][3];
    double r[NGP][NPE][3];  // residual contributions (FP64)
    float h[NGP][NPE][3];   // spatial gradients
    float bh[NGP][NPE][3];  // b h
    float bm[NGP][9];       // b = F F^T
    float fac[NGP][5];      // dvol * {c1, c2, c3, f4, f9}
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

// x -> (hi, lo) BF16 pair; pack(first, second) puts `first` in the low 16 bits, the order of the
// mma fragments (lower column / row index first)
struct Split2 {
    uint32_t hi, lo;
};
__device__ __forceinline__ Split2 split_pack(float x0, float x1) {
    const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
    const __nv_bfloat16 l0 = __float2bfloat16_rn(x0 - __bfloat162float(h0));
    const __nv_bfloat16 l1 = __float2bfloat16_rn(x1 - __bfloat162float(h1));
    __nv_bfloat162 hh, ll;
    hh.x = h0;
    hh.y = h1;
    ll.x = l0;
    ll.y = l1;
    Split2 s;
    s.hi = *reinterpret_cast<uint32_t*>(&hh);
    s.lo = *reinterpret_cast<uint32_t*>(&ll);
    return s;
}

__device__ __forceinline__ void mma_bf16(float d[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// H_a[(J,b), (gp,j)] of the file header; zero outside the 3 NPE x 3 NGP range
template <int NPE, int NGP>
__device__ __forceinline__ float h_entry(const TcSmem<NPE, NGP>& s, int a, int m, int k) {
    if (m >= 3 * NPE || k >= 3 * NGP) return 0.f;
    const int J = m / 3, b = m - 3 * J, gp = k / 3, j = k - 3 * gp;
    const float* f = s.fac[gp];
    const float* hJ = s.h[gp][J];
    const float* bhJ = s.bh[gp][J];
    float v = f[1] * s.bm[gp][3 * a + j] * hJ[b];
    if (j == b) v += f[0] * hJ[a];
    if (j == a) v += f[2] * hJ[b] + f[1] * bhJ[b];
    if (a == b) v += f[3] * bhJ[j] + f[4] * hJ[j];
    return v;
}

template <int NPE, int NGP>
__device__ __forceinline__ float hn_entry(const TcSmem<NPE, NGP>& s, int k, int I) {
    if (k >= 3 * NGP || I >= NPE) return 0.f;
    const int gp = k / 3;
    return s.h[gp][I][k - 3 * gp];
}

// MODE bit 1: export Ke/Re (FP64 arrays); bit 2: scatter (FP32 off-diagonal blocks, FP64 rhs)
template <int NPE, int MODE>
__global__ void __launch_bounds__(kTcThreads, 2) elem_tc_kernel(ElemArgs a) {
    using T = TcTraits<NPE>;
    constexpr int NGP = T::NGP;
    constexpr int NS = 3 * NPE;
    constexpr int MT = (3 * NPE + 15) / 16;  // m tiles over (J, b)
    constexpr int NT = (NPE + 7) / 8;        // n tiles over I
    constexpr int KT = (3 * NGP + 15) / 16;  // k tiles over (gp, j)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto* S = reinterpret_cast<TcSmem<NPE, NGP>*>(smem_raw);
    const int64_t e0 = (int64_t)blockIdx.x * kTcEpb;

    for (int t = threadIdx.x; t < kTcEpb * NPE; t += blockDim.x) {
        const int el = t / NPE, I = t % NPE;
        const int64_t e = e0 + el;
        if (e >= a.n_elem) continue;
        const int32_t node = a.conn[e * NPE + I];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            S[el].x0[I][d] = a.coords[3 * (int64_t)node + d];
            S[el].u[I][d] = a.disp[3 * (int64_t)node + d];
        }
    }
    __syncthreads();

    // ---- phase 1: one thread per (element, Gauss point), FP64
    for (int t = threadIdx.x; t < kTcEpb * NGP; t += blockDim.x) {
        const int el = t / NGP, gp = t % NGP;
        const int64_t e = e0 + el;
        if (e >= a.n_elem) continue;
        TcSmem<NPE, NGP>& s = S[el];
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
        inv3d(G, det3d(G), Gi);
        const double jac = det3d(Gc);
        inv3d(Gc, jac, Gci);
        const double dvol = T::w(gp) * jac;
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
        const double J = det3d(F);
        if (J < 0.0) {
            atomicMin(a.bad, (unsigned long long)e);
            if (a.bad_elem) a.bad_elem[e] = 1;
        }
        double b[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
        const double* mt = a.mats + 4 * (int64_t)a.mat_id[e];
        const NhFactors nf = nh_factors(b, J, mt[0], mt[1], (int)mt[2], a.tangent);
        const double s1 = nf.s1, s2 = nf.s2;
        const double fac[5] = {nf.c1, nf.c2, nf.c3, nf.f4, nf.f9};
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
                s.h[gp][I][c] = (float)h[c];
                s.bh[gp][I][c] = (float)bh[c];
                s.r[gp][I][c] = -dvol * (s1 * bh[c] + s2 * h[c]);  // R_I -= dvol sigma h_I
            }
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) s.bm[gp][q] = (float)b[q / 3][q % 3];
#pragma unroll
        for (int q = 0; q < 5; ++q) s.fac[gp][q] = (float)(dvol * fac[q]);
    }
    __syncthreads();

    // ---- phase 2: one warp per element
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    for (int el = warp; el < kTcEpb; el += kTcThreads / 32) {
        const int64_t e = e0 + el;
        if (e >= a.n_elem) break;
        const TcSmem<NPE, NGP>& s = S[el];
        // residual: lane -> (I, c)
        for (int t = lane; t < NS; t += 32) {
            const int I = t / 3, c = t % 3;
            double R = 0.0;
#pragma unroll
            for (int gp = 0; gp < NGP; ++gp) R += s.r[gp][I][c];
            if (MODE & 1) a.Re[e * NS + t] = R;
            if (MODE & 2) {
                const int32_t node = a.conn[e * NPE + I];
                if (a.reac) atomicAdd(&a.reac[3 * (int64_t)node + c], R);
                if (!a.fixed[3 * (int64_t)node + c]) atomicAdd(&a.rhs[3 * (int64_t)node + c], R);
            }
        }
        // B fragments of Hn (k x n): b0 = rows 2 tig, 2 tig + 1; b1 = rows 2 tig + 8, + 9; column gid
        uint32_t bhi[KT][NT][2], blo[KT][NT][2];
#pragma unroll
        for (int kt = 0; kt < KT; ++kt)
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const int k = 16 * kt + 2 * tig, n = 8 * nt + gid;
                const Split2 p0 = split_pack(hn_entry(s, k, n), hn_entry(s, k + 1, n));
                const Split2 p1 = split_pack(hn_entry(s, k + 8, n), hn_entry(s, k + 9, n));
                bhi[kt][nt][0] = p0.hi;
                blo[kt][nt][0] = p0.lo;
                bhi[kt][nt][1] = p1.hi;
                blo[kt][nt][1] = p1.lo;
            }
#pragma unroll 1
        for (int aa = 0; aa < 3; ++aa) {
            float acc[MT][NT][4];
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
#pragma unroll
                for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                    for (int q = 0; q < 4; ++q) acc[mt][nt][q] = 0.f;
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
#pragma unroll
                for (int kt = 0; kt < KT; ++kt) {
                    // A fragment of H_a (m x k): regs (row gid, cols 2tig..), (row gid+8), (cols +8), (both)
                    const int m = 16 * mt + gid, k = 16 * kt + 2 * tig;
                    const Split2 q0 = split_pack(h_entry(s, aa, m, k), h_entry(s, aa, m, k + 1));
                    const Split2 q1 = split_pack(h_entry(s, aa, m + 8, k), h_entry(s, aa, m + 8, k + 1));
                    const Split2 q2 = split_pack(h_entry(s, aa, m, k + 8), h_entry(s, aa, m, k + 9));
                    const Split2 q3 = split_pack(h_entry(s, aa, m + 8, k + 8), h_entry(s, aa, m + 8, k + 9));
#pragma unroll
                    for (int nt = 0; nt < NT; ++nt) {
                        mma_bf16(acc[mt][nt], q0.hi, q1.hi, q2.hi, q3.hi, bhi[kt][nt][0], bhi[kt][nt][1]);
                        mma_bf16(acc[mt][nt], q0.hi, q1.hi, q2.hi, q3.hi, blo[kt][nt][0], blo[kt][nt][1]);
                        mma_bf16(acc[mt][nt], q0.lo, q1.lo, q2.lo, q3.lo, bhi[kt][nt][0], bhi[kt][nt][1]);
                    }
                }
            // D_a[(J,b), I]: c0, c1 at row gid, cols 2 tig, 2 tig + 1; c2, c3 at row gid + 8
#pragma unroll
            for (int mt = 0; mt < MT; ++mt)
#pragma unroll
                for (int nt = 0; nt < NT; ++nt)
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int m = 16 * mt + gid + (q >= 2 ? 8 : 0);
                        const int I = 8 * nt + 2 * tig + (q & 1);
                        if (m >= NS || I >= NPE) continue;
                        const int J = m / 3, bb = m - 3 * J;
                        const float v = acc[mt][nt][q];
                        if (MODE & 1) a.Ke[(e * NS + 3 * I + aa) * NS + 3 * J + bb] = (double)v;
                        if (MODE & 2) {
                            const int32_t nI = a.conn[e * NPE + I], nJ = a.conn[e * NPE + J];
                            // FP32 storage: off-diagonal blocks, unmasked; the diagonal is rebuilt from them
                            if (nI != nJ) {
                                const uint32_t off = a.e2v[(e * NPE + I) * NPE + J];
                                atomicAdd(&a.valf[off + 32u * (3 * aa + bb)], v);
                            }
                        }
                    }
        }
    }
}

template <int NPE, int MODE>
void launch_tc(const ElemArgs& a, cudaStream_t s) {
    const size_t smem = kTcEpb * sizeof(TcSmem<NPE, TcTraits<NPE>::NGP>);
    static std::atomic<uint64_t> configured{0};
    if (first_use_on_device(configured)) {
        MPHY_CUDA(cudaFuncSetAttribute(elem_tc_kernel<NPE, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem));
    }
    const unsigned grid = (unsigned)((a.n_elem + kTcEpb - 1) / kTcEpb);
    if (grid == 0) return;
    elem_tc_kernel<NPE, MODE><<<grid, kTcThreads, smem, s>>>(a);
    MPHY_CUDA(cudaGetLastError());
}

}  // namespace

void launch_elem_tc(const ElemArgs& a, int npe, int mode, cudaStream_t s) {
    MPHY_REQUIRE(mode == 1 || a.valf, MPHY_ERR_INVALID_ARG, "tensor-core element kernel: FP32 storage only");
    if (npe == 8) {
        if (mode == 1) launch_tc<8, 1>(a, s);
        else if (mode == 2) launch_tc<8, 2>(a, s);
        else launch_tc<8, 3>(a, s);
    } else {
        if (mode == 1) launch_tc<10, 1>(a, s);
        else if (mode == 2) launch_tc<10, 2>(a, s);
        else launch_tc<10, 3>(a, s);
    }
}

}  // namespace mphy
