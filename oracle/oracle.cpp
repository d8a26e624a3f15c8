// oracle.cpp -- CPU FP64 restatement of chennachaos/mphyfem's femSolidmechanics Newton step.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA product path and the timed CPU baseline.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference legs
// load it. Parity status: unpinned against the reference binary (unbuildable here: PETSc,
// Eigen, Boost, MPI and VTK are absent); pinned by the analytic and finite-difference checks
// in tests/test_oracle_*.py. Every function names the reference lines it restates.

#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int kMaxNpe = 27;
constexpr int kMaxGp = 27;

struct GaussRule {
    int ngp = 0;
    double xi[kMaxGp][3];
    double w[kMaxGp];
};

// 2-point Gauss-Legendre abscissa exactly as written in src/utilities/QuadratureUtil.cpp:24-25.
constexpr double kGauss2 = 0.577350269189626;

// Hex 2x2x2 rule, point ordering of QuadratureUtil.cpp:481-492 (xi1 fastest, then xi2, xi3,
// with the (+,+) point of each layer third, matching the hex8 node order).
void rule_hex8(GaussRule& r) {
    const double g[2] = {-kGauss2, kGauss2};
    const int pattern[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                               {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    r.ngp = 8;
    for (int q = 0; q < 8; ++q) {
        for (int d = 0; d < 3; ++d) r.xi[q][d] = g[pattern[q][d]];
        r.w[q] = 1.0;
    }
}

// Tetrahedron 4-point rule of QuadratureUtil.cpp:690-712 (weights 1/4 of the volume 1/6).
void rule_tet4(GaussRule& r) {
    const double a = 0.1381966011250105, b = 0.5854101966249685;
    const double pts[4][3] = {{a, a, a}, {b, a, a}, {a, b, a}, {a, a, b}};
    r.ngp = 4;
    for (int q = 0; q < 4; ++q) {
        for (int d = 0; d < 3; ++d) r.xi[q][d] = pts[q][d];
        r.w[q] = 0.25 * (1.0 / 6.0);
    }
}

// Trilinear hex: tensor product of the linear 1D Lagrange pair (BasisFunctionsLagrange.cpp:146-152)
// with the node order of :1243-1250: (-,-,-),(+,-,-),(+,+,-),(-,+,-),(-,-,+),(+,-,+),(+,+,+),(-,+,+).
void shape_hex8(const double* xi, double* N, double dN[3][kMaxNpe]) {
    double n1[3][2], d1[3][2];
    for (int d = 0; d < 3; ++d) {
        n1[d][0] = 0.5 * (1.0 - xi[d]);
        n1[d][1] = 0.5 * (1.0 + xi[d]);
        d1[d][0] = -0.5;
        d1[d][1] = 0.5;
    }
    const int corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                              {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
    for (int a = 0; a < 8; ++a) {
        const int i = corner[a][0], j = corner[a][1], k = corner[a][2];
        N[a] = n1[0][i] * n1[1][j] * n1[2][k];
        dN[0][a] = d1[0][i] * n1[1][j] * n1[2][k];
        dN[1][a] = n1[0][i] * d1[1][j] * n1[2][k];
        dN[2][a] = n1[0][i] * n1[1][j] * d1[2][k];
    }
}

// Quadratic tetrahedron (BasisFunctionsLagrange.cpp:870-956). Barycentric L0 = 1-x1-x2-x3,
// vertices 0..3 at L0, x1, x2, x3; mid-side nodes 4:(0,1) 5:(1,2) 6:(0,2) 7:(0,3) 8:(2,3) 9:(1,3).
void shape_tet10(const double* xi, double* N, double dN[3][kMaxNpe]) {
    const double L[4] = {1.0 - xi[0] - xi[1] - xi[2], xi[0], xi[1], xi[2]};
    // dL_v / dxi_d: L0 -> -1 in every direction, L_{d+1} -> 1 in direction d.
    auto dL = [](int v, int d) { return v == 0 ? -1.0 : (v == d + 1 ? 1.0 : 0.0); };
    for (int v = 0; v < 4; ++v) {
        N[v] = L[v] * (2.0 * L[v] - 1.0);
        for (int d = 0; d < 3; ++d) dN[d][v] = (4.0 * L[v] - 1.0) * dL(v, d);
    }
    const int edge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {2, 3}, {1, 3}};
    for (int e = 0; e < 6; ++e) {
        const int p = edge[e][0], q = edge[e][1];
        N[4 + e] = 4.0 * L[p] * L[q];
        for (int d = 0; d < 3; ++d) dN[d][4 + e] = 4.0 * (dL(p, d) * L[q] + L[p] * dL(q, d));
    }
}

// Triquadratic hex (BasisFunctionsLagrange.cpp:1202-1399): tensor product of the quadratic 1D
// Lagrange triple of :45-61, ordered (xi = -1, xi = +1, xi = 0), with the 27-node order of
// :1300-1399 -- corners as hex8, then the mid-edge nodes 8..19, the mid-face nodes 20..25 and
// the centre 26. Entry a of kHex27 holds the 1D indices (i, j, k) of node a.
constexpr int kHex27[27][3] = {
    {0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1},
    {2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 2, 0}, {1, 0, 2}, {2, 1, 0}, {1, 1, 2}, {0, 1, 2},
    {2, 0, 1}, {0, 2, 1}, {1, 2, 1}, {2, 1, 1}, {2, 2, 0}, {2, 0, 2}, {0, 2, 2}, {1, 2, 2},
    {2, 1, 2}, {2, 2, 1}, {2, 2, 2}};

void shape_hex27(const double* xi, double* N, double dN[3][kMaxNpe]) {
    double n1[3][3], d1[3][3];
    for (int d = 0; d < 3; ++d) {
        const double x = xi[d], x2 = x * x;
        n1[d][0] = 0.5 * (x2 - x);
        n1[d][1] = 0.5 * (x2 + x);
        n1[d][2] = 1.0 - x2;
        d1[d][0] = 0.5 * (2.0 * x - 1.0);
        d1[d][1] = 0.5 * (2.0 * x + 1.0);
        d1[d][2] = -2.0 * x;
    }
    for (int a = 0; a < 27; ++a) {
        const int i = kHex27[a][0], j = kHex27[a][1], k = kHex27[a][2];
        N[a] = n1[0][i] * n1[1][j] * n1[2][k];
        dN[0][a] = d1[0][i] * n1[1][j] * n1[2][k];
        dN[1][a] = n1[0][i] * d1[1][j] * n1[2][k];
        dN[2][a] = n1[0][i] * n1[1][j] * d1[2][k];
    }
}

// Hex 3x3x3 rule of QuadratureUtil.cpp:497-524: the 3-point 1D rule of :29-33 (-0.7746.., +0.7746..,
// 0; weights 5/9, 5/9, 8/9), point q at the 1D indices of hex27 node q (kHex27), weight
// w_i w_j w_k in that product order.
void rule_hex27(GaussRule& r) {
    const double g[3] = {-0.774596669241483, 0.774596669241483, 0.0};
    const double wt[3] = {5.0 / 9.0, 5.0 / 9.0, 8.0 / 9.0};
    r.ngp = 27;
    for (int q = 0; q < 27; ++q) {
        for (int d = 0; d < 3; ++d) r.xi[q][d] = g[kHex27[q][d]];
        r.w[q] = wt[kHex27[q][0]] * wt[kHex27[q][1]] * wt[kHex27[q][2]];
    }
}

// The quadrature of each element, getGaussPoints3D (QuadratureUtil.cpp:268-317): 2x2x2 for
// hex8, 4 points for tet10, 3x3x3 for the 27-node hex (which ElementBase::calcStiffnessAndResidualMixed3D
// uses for Elem_Solid_3D_Mixed1, ElementBase2.cpp:320, whatever nGP prepareElemData set).
bool element_rule(int npe, GaussRule& r) {
    if (npe == 8) { rule_hex8(r); return true; }
    if (npe == 10) { rule_tet4(r); return true; }
    if (npe == 27) { rule_hex27(r); return true; }
    return false;
}

void shape(int npe, const double* xi, double* N, double dN[3][kMaxNpe]) {
    if (npe == 8) shape_hex8(xi, N, dN);
    else if (npe == 27) shape_hex27(xi, N, dN);
    else shape_tet10(xi, N, dN);
}

double det3(const double A[3][3]) {
    return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
           A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

// Inverse by cofactors (stands in for Eigen's MatrixXd::inverse(); last-ulp differences only).
void inv3(const double A[3][3], double det, double Ai[3][3]) {
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

// computeBasisFunctions3D (GeomDataLagrange.cpp:349-458): the mapping gradient
// G(r, c) = sum_I x_I[c] dN_I/dxi_r, its determinant, and spatial gradients
// dN/dx_c = sum_r dN/dxi_r * Ginv(c, r).
double spatial_gradients(int npe, const double* x, const double dN[3][kMaxNpe],
                         double grad[3][kMaxNpe]) {
    double G[3][3] = {{0}};
    for (int I = 0; I < npe; ++I)
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) G[r][c] += x[3 * I + c] * dN[r][I];
    const double jac = det3(G);
    double Gi[3][3];
    inv3(G, jac, Gi);
    for (int I = 0; I < npe; ++I)
        for (int c = 0; c < 3; ++c)
            grad[c][I] = dN[0][I] * Gi[c][0] + dN[1][I] * Gi[c][1] + dN[2][I] * Gi[c][2];
    return jac;
}

// 9-index <-> (i, j) of src/material/utilitiesmaterialHyperelastic.cpp:192 (column-major 3x3).
constexpr int kPairI[9] = {0, 1, 2, 0, 1, 2, 0, 1, 2};
constexpr int kPairJ[9] = {0, 0, 0, 1, 1, 1, 2, 2, 2};

inline double kd(int a, int b) { return a == b ? 1.0 : 0.0; }

// 0: the reference's tangent (volumetric part without the geometric stress term,
// utilitiesmaterialHyperelastic.cpp:283-288); 1: the consistent tangent, which adds
// U'(J) d_ik d_jl back. Test-only switch for the consistency checks.
int g_consistent_tangent = 0;
// 0: pick the pattern construction by size; 1: always the literal per-element push_back
// restatement; 2: always the per-node construction. Test-only switch (both give one pattern).
int g_pattern_mode = 0;

struct CsrPattern {
    int n_free = 0;
    std::vector<int32_t> node_dof;       // [n_node*3] free id or -1 (NodeDofArray)
    std::vector<int32_t> assy_for_soln;  // [n_free]
    std::vector<int32_t> for_assy;       // [n_elem][3npe] (forAssyVec)
    std::vector<int64_t> rowptr;         // [n_free+1]
    std::vector<int32_t> col;            // [nnz]
};

}  // namespace

struct orc_problem {
    int n_node, n_elem, npe;
    std::vector<double> coords;
    std::vector<int32_t> conn, mat_id;
    std::vector<double> mats;  // [n_mat][3] = {mu, Kinv, Utype}
    std::vector<int32_t> model;  // [n_mat] ORC_MAT_* (Neo-Hookean unless set)
    std::vector<double> data;    // [n_mat][ORC_MAT_NDATA] model parameters (data[0] = mu by default)
    std::vector<uint8_t> fixed;
    CsrPattern pat;
    // position of each (element row i, element col j) entry in the CSR value array, -1 if
    // either DOF is prescribed (what MatSetValue's row search resolves, SolverPetsc.cpp:370-374)
    std::vector<int64_t> slot;  // [n_elem][nsize*nsize]
    // constant-pressure mixed element (Elem_Solid_3D_Mixed0): element pressures, their values at
    // the last converged step, that step's displacement (Jn), and the coupling terms of the last
    // element evaluation (for solveForPressure)
    bool p0 = false;
    mutable std::vector<double> pe, pe_prev, disp_prev, kup, kpp, fp;
    // prescribed displacements t * presc_ramp + presc_const (empty: all prescribed values zero)
    std::vector<double> presc_ramp, presc_const;
};

extern "C" {

double orc_vol_dU(int type, double K, double J) {
    switch (type) {
        case -1: return 0.0;
        case 1: return 0.1 * K * (std::pow(J, 4) - 1.0 / std::pow(J, 6));
        case 2: return 0.125 * K * (J * J - 1.0 / (J * J)) * (J + 1.0 / (J * J * J));
        case 3: return K * (J - 1.0);
        case 4: return 0.5 * K * (J - 1.0 / J);
        case 5: return 0.5 * K * (J - 1.0 + std::log(J) / J);
        case 6: return K * std::log(J);
        case 7: return K * (1.0 - 1.0 / J);
        case 8: return K * std::log(J) / J;
        default: return 0.0;
    }
}

double orc_vol_d2U(int type, double K, double J) {
    switch (type) {
        case -1: return 0.0;
        case 1: return 0.2 * K * (2.0 * J * J * J + 3.0 / std::pow(J, 7));
        case 2: return 0.125 * K * (3.0 * J * J + 5.0 / std::pow(J, 6));
        case 3: return K;
        case 4: return 0.5 * K * (1.0 + 1.0 / (J * J));
        case 5: return 0.5 * K * (J * J + 1.0 - std::log(J)) / (J * J);
        case 6: return K / std::log(J);
        case 7: return K / (J * J);
        case 8: return K * (1.0 - std::log(J)) / (J * J);
        default: return 0.0;
    }
}

// Compressible Neo-Hookean, utilitiesmaterialHyperelastic.cpp:186-295 with MIXED_ELEMENT false:
//   sigma = mu J^{-5/3} (b - Ib/3 I) + U'(J) I
//   C_{ijkl} = (mu J^{-5/3} Ib/3) d_il d_jk - (2/3) mu J^{-5/3} (b_ij d_kl + d_ij b_kl)
//            + (2/9) mu J^{-5/3} Ib d_ij d_kl + mu J^{-5/3} b_jl d_ik
//            + (J U'' + U') d_ij d_kl - U' d_il d_jk - U' d_jl d_ik
// Mixed (u-p) branch, :218-221 and :275-281: the pressure unknown p replaces U'(J) in the stress
// and p (d_ij d_kl - d_jk d_il) replaces the volumetric tangent.
static int nh_impl(const double* Fm, double mu, double Kinv, int Utype, bool mixed, double pres, double* stre,
                   double* C) {
    const double K = 1.0 / Kinv;
    double F[3][3], b[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) F[i][j] = Fm[3 * i + j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
    const double J = det3(F);
    const double Jm2d3 = std::pow(J, -2.0 / 3.0);
    const double Jm5d3 = Jm2d3 / J;
    const double Ib = b[0][0] + b[1][1] + b[2][2];
    const double dU = orc_vol_dU(Utype, K, J);
    const double d2U = orc_vol_d2U(Utype, K, J);

    const double s1 = mu * Jm5d3;
    const double s2 = -s1 * (1.0 / 3.0) * Ib + (mixed ? pres : dU);
    for (int q = 0; q < 9; ++q) {
        const int i = kPairI[q], j = kPairJ[q];
        stre[q] = s1 * b[i][j] + (i == j ? s2 : 0.0);
    }

    const double c_iljk = (1.0 / 3.0) * mu * Jm5d3 * Ib;  // with d_il d_jk
    const double c_bdd = -(2.0 / 3.0) * mu * Jm5d3;        // with b_ij d_kl + d_ij b_kl
    const double c_dd = (2.0 / 3.0) * (1.0 / 3.0) * mu * Jm5d3 * Ib;
    const double c_bjl = mu * Jm5d3;                       // with b_jl d_ik
    const double c_vol = J * d2U + dU;                     // with d_ij d_kl
    for (int p = 0; p < 9; ++p) {
        const int i = kPairI[p], j = kPairJ[p];
        for (int q = 0; q < 9; ++q) {
            const int k = kPairI[q], l = kPairJ[q];
            double v = 0.0;
            v += c_iljk * (kd(i, l) * kd(j, k));
            v += c_bdd * (b[i][j] * kd(k, l) + kd(i, j) * b[k][l]);
            v += c_dd * (kd(i, j) * kd(k, l));
            v += c_bjl * (b[j][l] * kd(i, k));
            if (mixed) {
                v += pres * (kd(i, j) * kd(k, l) - kd(j, k) * kd(i, l));
            } else {
                v += c_vol * (kd(i, j) * kd(k, l)) - dU * (kd(i, l) * kd(j, k)) - dU * (kd(j, l) * kd(i, k));
                if (g_consistent_tangent) v += dU * (kd(j, l) * kd(i, k));
            }
            C[9 * p + q] = v;
        }
    }
    return 0;
}

int orc_nh_stress_tangent(const double* Fm, double mu, double Kinv, int Utype, double* stre, double* C) {
    return nh_impl(Fm, mu, Kinv, Utype, false, 0.0, stre, C);
}

namespace {

// Shared pieces of the three b-invariant models below: b = F F^T, b^2, J, the trace, the
// deviatoric part of b, U'(J), U''(J).
struct Kin {
    double b[3][3], b2[3][3], bdev[3][3];
    double J, Ib, dU, d2U;
};

Kin kinematics(const double* Fm, double Kinv, int Utype) {
    Kin k;
    double F[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) F[i][j] = Fm[3 * i + j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) k.b[i][j] = F[i][0] * F[j][0] + F[i][1] * F[j][1] + F[i][2] * F[j][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            k.b2[i][j] = k.b[i][0] * k.b[0][j] + k.b[i][1] * k.b[1][j] + k.b[i][2] * k.b[2][j];
    k.J = det3(F);
    k.Ib = k.b[0][0] + k.b[1][1] + k.b[2][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) k.bdev[i][j] = k.b[i][j] - (i == j ? k.Ib / 3.0 : 0.0);
    const double K = 1.0 / Kinv;
    k.dU = orc_vol_dU(Utype, K, k.J);
    k.d2U = orc_vol_d2U(Utype, K, k.J);
    return k;
}

// Mooney-Rivlin, utilitiesmaterialHyperelastic.cpp:300-420, compressible branch. data = {c1, c2}.
// The reference sets r7d3 = 5.0/3.0 (:303), so its "J^{-7/3}" factor is J^{-5/3}; restated as
// written (the c2 terms of stress and tangent both carry J^{-5/3}). With that factor the c2 stress
// is J^{2/3} times an energy's stress, and its exact linearisation adds (2/3) sigma_c2 (x) I to
// the tangent below: a non-symmetric term that a CG solve cannot take, so both tangent modes
// give the symmetric tangent as written.
void mooney_rivlin(const double* Fm, const double* data, double Kinv, int Utype, bool mixed, double pres,
                   double* stre, double* C) {
    const Kin k = kinematics(Fm, Kinv, Utype);
    const double c1 = data[0], c2 = data[1];
    const double Jm5d3 = std::pow(k.J, -2.0 / 3.0) / k.J;
    const double Jm7d3 = std::pow(k.J, -5.0 / 3.0);
    const double I1 = k.Ib;
    const double I2 = 0.5 * (I1 * I1 - (k.b2[0][0] + k.b2[1][1] + k.b2[2][2]));
    const double s1 = 2.0 * c1 * Jm5d3 + 2.0 * c2 * Jm7d3 * I1;
    const double s2 = -c1 * (2.0 / 3.0) * Jm5d3 * I1 - c2 * (4.0 / 3.0) * Jm7d3 * I2 + (mixed ? pres : k.dU);
    const double s3 = -2.0 * c2 * Jm7d3;
    for (int q = 0; q < 9; ++q) {
        const int i = kPairI[q], j = kPairJ[q];
        stre[q] = s1 * k.b[i][j] + s3 * k.b2[i][j] + (i == j ? s2 : 0.0);
    }
    const double f1 = 2.0 * c1 * Jm5d3, f2 = 2.0 * c2 * Jm7d3, f3 = (4.0 / 3.0) * c2 * Jm7d3;
    const double f7 = k.J * k.d2U + k.dU, f8 = -k.dU;
    const auto& b = k.b;
    const auto& b2 = k.b2;
    for (int p = 0; p < 9; ++p) {
        const int i = kPairI[p], j = kPairJ[p];
        for (int q = 0; q < 9; ++q) {
            const int kk = kPairI[q], l = kPairJ[q];
            const double dij = kd(i, j), dik = kd(i, kk), dil = kd(i, l), djk = kd(j, kk), dkl = kd(kk, l);
            double v = f1 * (dik * b[j][l] + (1.0 / 3.0) * I1 * dil * djk + (2.0 / 9.0) * I1 * dij * dkl -
                             (2.0 / 3.0) * b[i][j] * dkl - (2.0 / 3.0) * b[kk][l] * dij);
            v += f2 * (2.0 * b[i][j] * b[kk][l] + I1 * dik * b[j][l] - b[i][kk] * b[j][l] - b[i][l] * b[kk][j] -
                       dik * b2[j][l]);
            v += f3 * (I2 * dil * djk + (4.0 / 3.0) * I2 * dkl * dij + 2.0 * dij * b2[kk][l] + 2.0 * dkl * b2[i][j] -
                       2.0 * I1 * dkl * b[i][j] - 2.0 * I1 * dij * b[kk][l]);
            v += mixed ? pres * (dij * dkl - djk * dil) : f7 * (dij * dkl) + f8 * (dil * djk);
            C[9 * p + q] = v;
        }
    }
}

// Gent, utilitiesmaterialHyperelastic.cpp:423-548, compressible branch. data = {mu, Im}.
void gent(const double* Fm, const double* data, double Kinv, int Utype, bool mixed, double pres, double* stre,
          double* C) {
    const Kin k = kinematics(Fm, Kinv, Utype);
    const double mu = data[0], Im = data[1];
    const double Jm2d3 = std::pow(k.J, -2.0 / 3.0);
    const double Jm5d3 = Jm2d3 / k.J;
    const double Jm7d3 = std::pow(k.J, -7.0 / 3.0);
    const double gf = 1.0 / (1.0 - (Jm2d3 * k.Ib - 3.0) / Im);
    const double s1 = mu * Jm5d3 * gf;
    const double s2 = -s1 * (1.0 / 3.0) * k.Ib + (mixed ? pres : k.dU);
    for (int q = 0; q < 9; ++q) {
        const int i = kPairI[q], j = kPairJ[q];
        stre[q] = s1 * k.b[i][j] + (i == j ? s2 : 0.0);
    }
    const double f1 = -(2.0 / 3.0) * mu * Jm5d3 * gf, f2 = 2.0 * mu * Jm7d3 * gf * gf / Im, f3 = mu * Jm5d3 * gf;
    const double f7 = k.J * k.d2U + k.dU, f8 = -k.dU;
    const auto& b = k.b;
    const auto& bd = k.bdev;
    for (int p = 0; p < 9; ++p) {
        const int i = kPairI[p], j = kPairJ[p];
        for (int q = 0; q < 9; ++q) {
            const int kk = kPairI[q], l = kPairJ[q];
            const double dij = kd(i, j), dik = kd(i, kk), dil = kd(i, l), djk = kd(j, kk), dkl = kd(kk, l);
            double v = f1 * (bd[i][j] * dkl);
            v += f2 * (bd[i][j] * bd[kk][l]);
            v += f3 * (dik * b[j][l] - (2.0 / 3.0) * b[kk][l] * dij + (1.0 / 3.0) * k.Ib * dil * djk);
            v += mixed ? pres * (dij * dkl - djk * dil) : f7 * (dij * dkl) + f8 * (dil * djk);
            C[9 * p + q] = v;
        }
    }
}

// Arruda-Boyce (five-term inverse-Langevin series), utilitiesmaterialHyperelastic.cpp:551-677,
// compressible branch. data = {mu, N}.
void arruda_boyce(const double* Fm, const double* data, double Kinv, int Utype, bool mixed, double pres,
                  double* stre, double* C) {
    const Kin k = kinematics(Fm, Kinv, Utype);
    const double mu = data[0], N = data[1];
    const double c1 = mu / 2.0, c2 = mu / 20.0 / N, c3 = mu * 11.0 / 1050.0 / N / N,
                 c4 = mu * 19.0 / 7000.0 / N / N / N, c5 = mu * 519.0 / 673750.0 / N / N / N / N;
    const double Jm2d3 = std::pow(k.J, -2.0 / 3.0);
    const double Jm5d3 = std::pow(k.J, -5.0 / 3.0);
    const double Jm7d3 = std::pow(k.J, -7.0 / 3.0);
    const double Ibb = Jm2d3 * k.Ib;
    const double a1 = c1 + 2.0 * c2 * Ibb + 3.0 * c3 * Ibb * Ibb + 4.0 * c4 * Ibb * Ibb * Ibb +
                      5.0 * c5 * Ibb * Ibb * Ibb * Ibb;
    const double a2 = 2.0 * c2 + 6.0 * c3 * Ibb + 12.0 * c4 * Ibb * Ibb + 20.0 * c5 * Ibb * Ibb * Ibb;
    const double s1 = 2.0 * a1 * Jm5d3;
    const double s2 = -s1 * (1.0 / 3.0) * k.Ib + (mixed ? pres : k.dU);
    for (int q = 0; q < 9; ++q) {
        const int i = kPairI[q], j = kPairJ[q];
        stre[q] = s1 * k.b[i][j] + (i == j ? s2 : 0.0);
    }
    const double f1 = 4.0 * Jm7d3 * a2, f2 = -4.0 * (1.0 / 3.0) * a1 * Jm5d3, f3 = (2.0 / 3.0) * a1 * Jm5d3 * k.Ib,
                 f4 = 4.0 * (1.0 / 3.0) * (1.0 / 3.0) * a1 * Jm5d3 * k.Ib;
    const double f7 = k.J * k.d2U + k.dU, f8 = -k.dU;
    const auto& b = k.b;
    const auto& bd = k.bdev;
    for (int p = 0; p < 9; ++p) {
        const int i = kPairI[p], j = kPairJ[p];
        for (int q = 0; q < 9; ++q) {
            const int kk = kPairI[q], l = kPairJ[q];
            const double dij = kd(i, j), dik = kd(i, kk), dil = kd(i, l), djk = kd(j, kk), djl = kd(j, l),
                         dkl = kd(kk, l);
            double v = f1 * (bd[i][j] * bd[kk][l]);
            v += f2 * (b[i][j] * dkl + b[kk][l] * dij);
            v += f3 * (dik * djl + dil * djk);
            v += f4 * (dij * dkl);
            // mixed: the pressure term as written at :661-664 (with d_jl d_ik, which the
            // consistent tangent drops); displacement form: the volumetric terms
            if (mixed) v += pres * (dij * dkl - djk * dil - (g_consistent_tangent ? 0.0 : djl * dik));
            else v += f7 * (dij * dkl) + f8 * (dil * djk);
            // The deviatoric part above is the symmetrised form "without stress terms" (:655-660):
            // it has (2/3) a1 J^{-5/3} Ib d_ik d_jl where the exact linearisation of the stress
            // has 2 a1 J^{-5/3} d_ik b_jl. The consistent tangent swaps them.
            if (g_consistent_tangent) v += 2.0 * a1 * Jm5d3 * dik * (b[j][l] - (1.0 / 3.0) * k.Ib * djl);
            C[9 * p + q] = v;
        }
    }
}

}  // namespace

static int material_impl(int model, const double* data, double Kinv, int Utype, const double* F, bool mixed,
                         double pres, double* stre, double* C) {
    switch (model) {
        case ORC_MAT_NEOHOOKEAN: return nh_impl(F, data[0], Kinv, Utype, mixed, pres, stre, C);
        case ORC_MAT_MOONEYRIVLIN: mooney_rivlin(F, data, Kinv, Utype, mixed, pres, stre, C); return 0;
        case ORC_MAT_GENT: gent(F, data, Kinv, Utype, mixed, pres, stre, C); return 0;
        case ORC_MAT_ARRUDABOYCE: arruda_boyce(F, data, Kinv, Utype, mixed, pres, stre, C); return 0;
        default: return 2;
    }
}

int orc_material_stress_tangent(int model, const double* data, double Kinv, int Utype, const double* F,
                                double* stre, double* C) {
    return material_impl(model, data, Kinv, Utype, F, false, 0.0, stre, C);
}

int orc_material_stress_tangent_mixed(int model, const double* data, double Kinv, int Utype, const double* F,
                                      double pres, double* stre, double* C) {
    return material_impl(model, data, Kinv, Utype, F, true, pres, stre, C);
}

void orc_set_consistent_tangent(int on) { g_consistent_tangent = on ? 1 : 0; }
void orc_set_pattern_mode(int mode) { g_pattern_mode = mode; }

int orc_gauss_rule(int npe, double* xi, double* w, double* N, double* dNdxi) {
    GaussRule r;
    if (!element_rule(npe, r)) return 0;
    for (int q = 0; q < r.ngp; ++q) {
        double n[kMaxNpe], dn[3][kMaxNpe];
        shape(npe, r.xi[q], n, dn);
        for (int d = 0; d < 3; ++d) xi[3 * q + d] = r.xi[q][d];
        w[q] = r.w[q];
        for (int a = 0; a < npe; ++a) {
            N[q * npe + a] = n[a];
            for (int d = 0; d < 3; ++d) dNdxi[(q * 3 + d) * npe + a] = dn[d][a];
        }
    }
    return r.ngp;
}

// Elem_Solid_3D_Disp::calcStiffnessAndResidual (Elem_Solid_3D_Disp.cpp:196-373), STATIC
// scheme: af = td[2] = 1, no inertia or body force. The two configurations are built as in
// the reference: F from the reference-configuration gradients (ElementBase.cpp:334-361),
// then gradients and volume in the current configuration x = X + u.
int orc_elem_stiffness_residual(int npe, const double* X, const double* u, double mu, double Kinv,
                                int Utype, double* K, double* R) {
    return orc_elem_stiffness_residual_mat(npe, X, u, ORC_MAT_NEOHOOKEAN, &mu, Kinv, Utype, K, R);
}

int orc_elem_stiffness_residual_mat(int npe, const double* X, const double* u, int model, const double* data,
                                    double Kinv, int Utype, double* K, double* R) {
    GaussRule rule;
    if (npe == 27 || !element_rule(npe, rule)) return 2;  // displacement element: hex8 and tet10
    const int ns = 3 * npe;
    std::fill(K, K + ns * ns, 0.0);
    std::fill(R, R + ns, 0.0);
    double x[3 * kMaxNpe];
    for (int a = 0; a < 3 * npe; ++a) x[a] = X[a] + u[a];
    int bad = 0;
    for (int q = 0; q < rule.ngp; ++q) {
        double N[kMaxNpe], dN[3][kMaxNpe], g0[3][kMaxNpe], g[3][kMaxNpe];
        shape(npe, rule.xi[q], N, dN);
        spatial_gradients(npe, X, dN, g0);
        double F[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        for (int I = 0; I < npe; ++I)
            for (int a = 0; a < 3; ++a)
                for (int m = 0; m < 3; ++m) F[3 * a + m] += u[3 * I + a] * g0[m][I];
        double Fa[3][3];
        for (int i = 0; i < 9; ++i) Fa[i / 3][i % 3] = F[i];
        if (det3(Fa) < 0.0) bad = 1;
        const double dvol = rule.w[q] * spatial_gradients(npe, x, dN, g);
        double stre[9], C[81];
        if (orc_material_stress_tangent(model, data, Kinv, Utype, F, stre, C) != 0) return 2;
        for (int I = 0; I < npe; ++I) {
            const double bb[3] = {dvol * g[0][I], dvol * g[1][I], dvol * g[2][I]};
            double Gc[3][9];
            for (int kk = 0; kk < 9; ++kk)
                for (int a = 0; a < 3; ++a)
                    Gc[a][kk] = bb[0] * C[9 * a + kk] + bb[1] * C[9 * (3 + a) + kk] + bb[2] * C[9 * (6 + a) + kk];
            for (int a = 0; a < 3; ++a)
                R[3 * I + a] -= bb[0] * stre[a] + bb[1] * stre[3 + a] + bb[2] * stre[6 + a];
            for (int J = 0; J < npe; ++J) {
                const double c[3] = {g[0][J], g[1][J], g[2][J]};
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        K[(3 * I + a) * ns + 3 * J + b] +=
                            Gc[a][b] * c[0] + Gc[a][3 + b] * c[1] + Gc[a][6 + b] * c[2];
            }
        }
    }
    return bad;
}

}  // extern "C"

namespace {

// prepareMatrixPattern (femSolidmechanics2.cpp:121-478), single-rank branch: free DOFs
// numbered node-major skipping prescribed ones (:142-152), assyForSoln (:155-165),
// forAssyVec (:248-280), and per row the sorted unique union of the free columns of every
// element that touches it (:294-324, :390, findUnique = sort + unique).
void build_pattern(orc_problem* p) {
    CsrPattern& P = p->pat;
    const int nd = 3 * p->n_node, ns = 3 * p->npe;
    P.node_dof.assign(nd, -1);
    P.n_free = 0;
    for (int n = 0; n < p->n_node; ++n)
        for (int d = 0; d < 3; ++d)
            if (!p->fixed[3 * n + d]) P.node_dof[3 * n + d] = P.n_free++;
    P.assy_for_soln.clear();
    for (int i = 0; i < nd; ++i)
        if (P.node_dof[i] != -1) P.assy_for_soln.push_back(i);
    P.for_assy.resize((size_t)p->n_elem * ns);
    for (int e = 0; e < p->n_elem; ++e)
        for (int I = 0; I < p->npe; ++I)
            for (int d = 0; d < 3; ++d)
                P.for_assy[(size_t)e * ns + 3 * I + d] = P.node_dof[3 * p->conn[(size_t)e * p->npe + I] + d];

    const double literal_entries = (double)p->n_elem * ns * ns;
    std::vector<std::vector<int32_t>> rows(P.n_free);
    const bool literal = g_pattern_mode == 1 || (g_pattern_mode == 0 && literal_entries < 6.0e7);
    if (literal) {
        // literal restatement: every element pushes every free column into every free row
        for (int e = 0; e < p->n_elem; ++e) {
            const int32_t* fa = &P.for_assy[(size_t)e * ns];
            for (int i = 0; i < ns; ++i) {
                if (fa[i] == -1) continue;
                for (int j = 0; j < ns; ++j)
                    if (fa[j] != -1) rows[fa[i]].push_back(fa[j]);
            }
        }
        for (auto& r : rows) {
            std::sort(r.begin(), r.end());
            r.erase(std::unique(r.begin(), r.end()), r.end());
        }
    } else {
        // same set, built per node to bound memory on large meshes: the free columns of row
        // (n, d) are the free DOFs of every node sharing an element with n, ascending
        std::vector<std::vector<int32_t>> adj(p->n_node);
        for (int e = 0; e < p->n_elem; ++e) {
            const int32_t* cn = &p->conn[(size_t)e * p->npe];
            for (int I = 0; I < p->npe; ++I)
                for (int J = 0; J < p->npe; ++J) adj[cn[I]].push_back(cn[J]);
        }
        for (int n = 0; n < p->n_node; ++n) {
            auto& a = adj[n];
            std::sort(a.begin(), a.end());
            a.erase(std::unique(a.begin(), a.end()), a.end());
            for (int d = 0; d < 3; ++d) {
                const int r = P.node_dof[3 * n + d];
                if (r == -1) continue;
                for (int m : a)
                    for (int c = 0; c < 3; ++c)
                        if (P.node_dof[3 * m + c] != -1) rows[r].push_back(P.node_dof[3 * m + c]);
            }
            std::vector<int32_t>().swap(a);
        }
    }
    P.rowptr.assign(P.n_free + 1, 0);
    for (int r = 0; r < P.n_free; ++r) P.rowptr[r + 1] = P.rowptr[r] + (int64_t)rows[r].size();
    P.col.resize(P.rowptr[P.n_free]);
    for (int r = 0; r < P.n_free; ++r) {
        std::copy(rows[r].begin(), rows[r].end(), P.col.begin() + P.rowptr[r]);
        std::vector<int32_t>().swap(rows[r]);
    }

    // value slot of every element entry (the AIJ row search MatSetValue performs)
    p->slot.assign((size_t)p->n_elem * ns * ns, -1);
    for (int e = 0; e < p->n_elem; ++e) {
        const int32_t* fa = &P.for_assy[(size_t)e * ns];
        for (int i = 0; i < ns; ++i) {
            if (fa[i] == -1) continue;
            const int32_t* b = &P.col[P.rowptr[fa[i]]];
            const int32_t* en = &P.col[P.rowptr[fa[i] + 1]];
            for (int j = 0; j < ns; ++j) {
                if (fa[j] == -1) continue;
                const int32_t* it = std::lower_bound(b, en, fa[j]);
                p->slot[((size_t)e * ns + i) * ns + j] = P.rowptr[fa[i]] + (it - b);
            }
        }
    }
}

inline void set_threads(int nthreads) {
#ifdef _OPENMP
    omp_set_num_threads(nthreads > 0 ? nthreads : 1);
#else
    (void)nthreads;
#endif
}

void gather_element(const orc_problem* p, int64_t e, const double* disp, double* X, double* u) {
    for (int I = 0; I < p->npe; ++I) {
        const int n = p->conn[e * p->npe + I];
        for (int d = 0; d < 3; ++d) {
            X[3 * I + d] = p->coords[3 * (size_t)n + d];
            u[3 * I + d] = disp[3 * (size_t)n + d];
        }
    }
}

void elem_eval(const orc_problem* p, int64_t e, const double* disp, double* K, double* R, int* bad) {
    double X[3 * kMaxNpe], u[3 * kMaxNpe];
    gather_element(p, e, disp, X, u);
    const size_t id = (size_t)p->mat_id[e];
    const double* m = &p->mats[3 * id];
    if (p->p0) {
        double X2[3 * kMaxNpe], up[3 * kMaxNpe];
        gather_element(p, e, p->disp_prev.data(), X2, up);
        const int ns = 3 * p->npe;
        *bad = orc_elem_mixed0(p->npe, X, u, up, p->pe[e], p->model[id], &p->data[ORC_MAT_NDATA * id], m[1],
                               (int)m[2], K, R, &p->kup[e * ns], &p->kpp[e], &p->fp[e]);
        return;
    }
    *bad = orc_elem_stiffness_residual_mat(p->npe, X, u, p->model[id], &p->data[ORC_MAT_NDATA * id], m[1], (int)m[2],
                                           K, R);
}

// Elem_Solid_3D_Mixed0::solveForPressure (Elem_Solid_3D_Mixed0.cpp:112-200) for every element:
// p += (FP - Kpu du_e) / Kpp with du the node-major solution increment.
void p0_pressure_update(const orc_problem* p, const double* du) {
    const int ns = 3 * p->npe;
    for (int64_t e = 0; e < p->n_elem; ++e) {
        double v = 0.0;
        for (int I = 0; I < p->npe; ++I)
            for (int c = 0; c < 3; ++c) v += p->kup[e * ns + 3 * I + c] * du[3 * (size_t)p->conn[e * p->npe + I] + c];
        p->pe[e] += (p->fp[e] - v) / p->kpp[e];
    }
}

}  // namespace

extern "C" {

orc_problem* orc_problem_create(int n_node, const double* coords, int n_elem, int npe,
                                const int32_t* conn, const int32_t* mat_id, int n_mat,
                                const double* mats, const uint8_t* fixed) {
    // 27-node hexes only for the mixed u-p element (orc_problem_elements_mixed)
    if (npe != 8 && npe != 10 && npe != 27) return nullptr;
    orc_problem* p = new orc_problem;
    p->n_node = n_node;
    p->n_elem = n_elem;
    p->npe = npe;
    p->coords.assign(coords, coords + 3 * (size_t)n_node);
    p->conn.assign(conn, conn + (size_t)n_elem * npe);
    p->mat_id.assign(mat_id, mat_id + n_elem);
    p->mats.assign(mats, mats + 3 * (size_t)n_mat);
    p->model.assign(n_mat, ORC_MAT_NEOHOOKEAN);
    p->data.assign(ORC_MAT_NDATA * (size_t)n_mat, 0.0);
    for (int k = 0; k < n_mat; ++k) p->data[ORC_MAT_NDATA * (size_t)k] = mats[3 * k];
    p->fixed.assign(fixed, fixed + 3 * (size_t)n_node);
    build_pattern(p);
    return p;
}

void orc_problem_destroy(orc_problem* p) { delete p; }

int orc_problem_set_materials(orc_problem* p, int n_mat, const int32_t* model, const double* data) {
    if (n_mat != (int)p->model.size()) return 1;
    for (int k = 0; k < n_mat; ++k)
        if (model[k] < ORC_MAT_NEOHOOKEAN || model[k] > ORC_MAT_ARRUDABOYCE) return 2;
    p->model.assign(model, model + n_mat);
    p->data.assign(data, data + ORC_MAT_NDATA * (size_t)n_mat);
    return 0;
}
int orc_problem_nfree(const orc_problem* p) { return p->pat.n_free; }
int64_t orc_problem_nnz(const orc_problem* p) { return p->pat.rowptr.back(); }

void orc_problem_export_pattern(const orc_problem* p, int32_t* assy_for_soln, int32_t* for_assy_vec,
                                int64_t* rowptr, int32_t* col) {
    const CsrPattern& P = p->pat;
    if (assy_for_soln) std::copy(P.assy_for_soln.begin(), P.assy_for_soln.end(), assy_for_soln);
    if (for_assy_vec) std::copy(P.for_assy.begin(), P.for_assy.end(), for_assy_vec);
    if (rowptr) std::copy(P.rowptr.begin(), P.rowptr.end(), rowptr);
    if (col) std::copy(P.col.begin(), P.col.end(), col);
}

int64_t orc_problem_elements(const orc_problem* p, const double* disp, double* Ke, double* Re,
                             int nthreads) {
    if (p->npe == 27) return -2;  // displacement element: hex8 and tet10 only
    const int ns = 3 * p->npe;
    // the first bad element in ascending order, as the reference's serial loop meets it
    int64_t first_bad = p->n_elem;
    set_threads(nthreads);
#pragma omp parallel for schedule(static) reduction(min : first_bad) if (nthreads > 1)
    for (int64_t e = 0; e < p->n_elem; ++e) {
        int bad = 0;
        elem_eval(p, e, disp, Ke + e * ns * ns, Re + e * ns, &bad);
        if (bad && e < first_bad) first_bad = e;
    }
    return first_bad == p->n_elem ? -1 : first_bad;
}

// Per element: Kuu [ns][ns], Kup [ns][NP], Kpp [NP][NP], FU [ns], FP [NP] with ns = 3 npe and
// NP = 4 (tet10) or 8 (hex27).
int64_t orc_problem_elements_mixed(const orc_problem* p, const double* disp, const double* disp_prev,
                                   const double* pres, double* Kuu, double* Kup, double* Kpp, double* FU, double* FP,
                                   int nthreads) {
    if (p->npe != 10 && p->npe != 27) return -2;
    const int npe = p->npe, NP = npe == 10 ? 4 : 8, ns = 3 * npe;
    int64_t first_bad = p->n_elem;
    set_threads(nthreads);
#pragma omp parallel for schedule(static) reduction(min : first_bad) if (nthreads > 1)
    for (int64_t e = 0; e < p->n_elem; ++e) {
        double X[3 * kMaxNpe], u[3 * kMaxNpe], up[3 * kMaxNpe], pn[8], Kpu[8 * 3 * kMaxNpe];
        gather_element(p, e, disp, X, u);
        gather_element(p, e, disp_prev, X, up);
        for (int i = 0; i < NP; ++i) pn[i] = pres[p->conn[e * npe + i]];
        const size_t id = (size_t)p->mat_id[e];
        const double* m = &p->mats[3 * id];
        const int bad = orc_elem_mixed(npe, X, u, up, pn, p->model[id], &p->data[ORC_MAT_NDATA * id], m[1], (int)m[2],
                                       Kuu + e * ns * ns, Kup + e * ns * NP, Kpu, Kpp + e * NP * NP, FU + e * ns,
                                       FP + e * NP);
        if (bad && e < first_bad) first_bad = e;
    }
    return first_bad == p->n_elem ? -1 : first_bad;
}

// femSolidmechanics::calcStiffnessAndResidual (femSolidmechanics2.cpp:1047-1120); lift (may be
// null): the prescribed increments dispApplied, lifted by ElementBase::applyDirichletBCs
// (ElementBase.cpp:567-594) into the free rows of every element before its scatter.
static int64_t assemble_impl(const orc_problem* p, const double* disp, double* val, double* rhs, double* reac,
                             int nthreads, const double* lift) {
    if (p->npe == 27) return -2;  // the displacement element's 27-point hex27 rule is not restated
    const CsrPattern& P = p->pat;
    const int ns = 3 * p->npe;
    if (val) std::fill(val, val + P.rowptr.back(), 0.0);
    if (rhs) std::fill(rhs, rhs + P.n_free, 0.0);
    if (reac) std::fill(reac, reac + 3 * (size_t)p->n_node, 0.0);
    int64_t first_bad = p->n_elem;
    set_threads(nthreads);
    const bool par = nthreads > 1;
#pragma omp parallel if (par)
    {
        std::vector<double> K(ns * ns), R(ns);
#pragma omp for schedule(static) reduction(min : first_bad)
        for (int64_t e = 0; e < p->n_elem; ++e) {
            int bad = 0;
            elem_eval(p, e, disp, K.data(), R.data(), &bad);
            if (bad && e < first_bad) first_bad = e;
            const int32_t* fa = &P.for_assy[e * ns];
            if (lift) {
                for (int ii = 0; ii < ns; ++ii) {
                    if (fa[ii] != -1) continue;  // a prescribed DOF: its increment lifts the free rows
                    const double fact = lift[3 * (size_t)p->conn[e * p->npe + ii / 3] + ii % 3];
                    for (int jj = 0; jj < ns; ++jj)
                        if (fa[jj] != -1) R[jj] -= K[jj * ns + ii] * fact;
                }
            }
            const int64_t* sl = &p->slot[e * ns * ns];
            for (int i = 0; i < ns; ++i) {
                if (fa[i] == -1) continue;
                if (rhs) {
                    if (par) {
#pragma omp atomic
                        rhs[fa[i]] += R[i];
                    } else {
                        rhs[fa[i]] += R[i];
                    }
                }
                if (val) {
                    for (int j = 0; j < ns; ++j) {
                        const int64_t s = sl[i * ns + j];
                        if (s < 0) continue;
                        if (par) {
#pragma omp atomic
                            val[s] += K[i * ns + j];
                        } else {
                            val[s] += K[i * ns + j];
                        }
                    }
                }
            }
            if (reac) {
                for (int I = 0; I < p->npe; ++I)
                    for (int d = 0; d < 3; ++d) {
                        const size_t g = 3 * (size_t)p->conn[e * p->npe + I] + d;
                        if (par) {
#pragma omp atomic
                            reac[g] += R[3 * I + d];
                        } else {
                            reac[g] += R[3 * I + d];
                        }
                    }
            }
        }
    }
    return first_bad == p->n_elem ? -1 : first_bad;
}

int64_t orc_problem_assemble(const orc_problem* p, const double* disp, double* val, double* rhs, double* reac,
                             int nthreads) {
    return assemble_impl(p, disp, val, rhs, reac, nthreads, nullptr);
}

int orc_problem_set_prescribed(orc_problem* p, const double* ramp, const double* cst) {
    const size_t nd = 3 * (size_t)p->n_node;
    p->presc_ramp.assign(nd, 0.0);
    p->presc_const.assign(nd, 0.0);
    bool any = false;
    for (size_t i = 0; i < nd; ++i) {
        if (!p->fixed[i]) continue;
        p->presc_ramp[i] = ramp ? ramp[i] : 0.0;
        p->presc_const[i] = cst ? cst[i] : 0.0;
        any |= p->presc_ramp[i] != 0.0 || p->presc_const[i] != 0.0;
    }
    if (!any) {
        p->presc_ramp.clear();
        p->presc_const.clear();
    }
    return 0;
}

// KSPCG (Hestenes-Stiefel) with PCJACOBI, restated from PETSc's documented algorithm as the
// reference's solver runs it (SolverPetsc.cpp:250-314: zero initial guess, KSPSolve).
// Norm type KSP_NORM_PRECONDITIONED; KSPConvergedDefault tests ||z_k|| against
// max(rtol * ||z_0||, abstol).
int orc_cg_jacobi(const orc_problem* p, const double* val, const double* b, double* x, double rtol,
                  double abstol, int maxit, int nthreads, int* its_out, double* final_norm) {
    return orc_cg_jacobi_norm(p, val, b, x, rtol, abstol, maxit, nthreads, 0, its_out, final_norm);
}

int orc_cg_jacobi_norm(const orc_problem* p, const double* val, const double* b, double* x, double rtol,
                       double abstol, int maxit, int nthreads, int norm_type, int* its_out, double* final_norm) {
    const CsrPattern& P = p->pat;
    const int n = P.n_free;
    set_threads(nthreads);
    const bool par = nthreads > 1;
    std::vector<double> dinv(n), r(b, b + n), z(n), pv(n), q(n);
#pragma omp parallel for if (par)
    for (int i = 0; i < n; ++i) {
        double d = 0.0;
        for (int64_t k = P.rowptr[i]; k < P.rowptr[i + 1]; ++k)
            if (P.col[k] == i) d = val[k];
        dinv[i] = d != 0.0 ? 1.0 / d : 1.0;  // PCJACOBI replaces a zero diagonal by 1
        x[i] = 0.0;
    }
    auto dot = [&](const std::vector<double>& a, const std::vector<double>& c) {
        double s = 0.0;
#pragma omp parallel for reduction(+ : s) if (par)
        for (int i = 0; i < n; ++i) s += a[i] * c[i];
        return s;
    };
#pragma omp parallel for if (par)
    for (int i = 0; i < n; ++i) z[i] = dinv[i] * r[i];
    double dp = std::sqrt(norm_type == 1 ? dot(r, r) : dot(z, z));
    const double ttol = std::max(rtol * dp, abstol);
    int its = 0, status = 1;
    if (final_norm) *final_norm = dp;
    if (dp <= ttol) {
        if (its_out) *its_out = 0;
        return 0;
    }
    double beta = dot(z, r), betaold = 0.0;
    for (int i = 0; i < maxit; ++i) {
        its = i + 1;
        if (beta == 0.0) { status = 0; break; }
        if (i == 0) {
            pv = z;
        } else {
            const double bk = beta / betaold;
#pragma omp parallel for if (par)
            for (int k = 0; k < n; ++k) pv[k] = z[k] + bk * pv[k];
        }
#pragma omp parallel for schedule(static) if (par)
        for (int row = 0; row < n; ++row) {
            double s = 0.0;
            for (int64_t k = P.rowptr[row]; k < P.rowptr[row + 1]; ++k) s += val[k] * pv[P.col[k]];
            q[row] = s;
        }
        const double dpi = dot(q, pv);
        betaold = beta;
        if (!(dpi > 0.0)) { status = std::isnan(dpi) ? 3 : 2; break; }
        const double a = beta / dpi;
#pragma omp parallel for if (par)
        for (int k = 0; k < n; ++k) {
            x[k] += a * pv[k];
            r[k] -= a * q[k];
            z[k] = dinv[k] * r[k];
        }
        dp = std::sqrt(norm_type == 1 ? dot(r, r) : dot(z, z));
        if (final_norm) *final_norm = dp;
        if (std::isnan(dp)) { status = 3; break; }
        if (dp <= ttol) { status = 0; break; }
        beta = dot(z, r);
    }
    if (its_out) *its_out = its;
    return status;
}

// solveWithNewtonRaphson (femSolidmechanics2.cpp:730-851) for the STATIC scheme with nodal
// forces (addExternalForces, femSolidmechanics1.cpp:1094-1113), the load factor of the time
// function "1 0 1000 0 1 0 0 0 0 0 0" (lambda(t) = t, TimeFunction.cpp:47-68), converged()
// and diverging(1e7) of femSolidmechanics1.cpp:616-636, and MyTime::cut/reset on failure
// (MyTime.cpp:41-58, SolutionDataSolid.cpp:157-167).
int orc_newton_run(const orc_problem* p, const double* fnodal, const orc_newton_opts* o,
                   double* disp, double* hist, int max_hist) {
    const CsrPattern& P = p->pat;
    const int n = P.n_free;
    const size_t nd = 3 * (size_t)p->n_node;
    std::vector<double> val(P.rowptr.back()), rhs(n), dx(n), disp_prev(nd);
    double t = 0.0, dt = o->dt;
    const double dt0 = o->dt;
    int steps_done = 1, rows = 0;
    while (t <= o->t_final - 1.0e-10 && steps_done <= o->max_steps) {
        t += dt;
        const double lambda = t;
        std::copy(disp, disp + nd, disp_prev.begin());
        if (p->p0) orc_problem_save_step(p, disp);
        // setBoundaryConditions (femSolidmechanics1.cpp:813-891): dispApplied = value(t) - disp
        const bool presc = !p->presc_ramp.empty();
        std::vector<double> lift;
        if (presc) {
            lift.assign(nd, 0.0);
            for (size_t i = 0; i < nd; ++i)
                if (p->fixed[i]) lift[i] = t * p->presc_ramp[i] + p->presc_const[i] - disp[i];
        }
        bool converged = false;
        double norm = -1.0, norm_prev = -1.0, tol = o->tol_abs;
        for (int iter = 1; iter <= o->max_newton; ++iter) {
            const int64_t bad = assemble_impl(p, disp, val.data(), rhs.data(), nullptr, o->nthreads,
                                              presc && iter == 1 ? lift.data() : nullptr);
            if (bad >= 0) break;  // "Negative Jacobian encountered": the iteration loop ends
            for (int i = 0; i < n; ++i) rhs[i] += lambda * fnodal[P.assy_for_soln[i]];
            norm_prev = norm;
            double s = 0.0;
            for (int i = 0; i < n; ++i) s += rhs[i] * rhs[i];
            norm = std::sqrt(s);
            if (iter == 1) tol = std::max(o->tol_abs, o->tol_rel * norm);
            int its = 0;
            bool stop = false;
            if (norm < tol) {
                converged = true;
                stop = true;
            } else if (iter > 3 && (std::isnan(norm) || (norm_prev > -0.1 && norm / norm_prev > 1.0e7))) {
                stop = true;
            } else {
                double fn = 0.0;
                orc_cg_jacobi(p, val.data(), rhs.data(), dx.data(), o->cg_rtol, 1.0e-50, o->cg_maxit,
                              o->nthreads, &its, &fn);
                for (int i = 0; i < n; ++i) disp[P.assy_for_soln[i]] += dx[i];
                // dispIncr[prescribed] += dispApplied in the first iteration (femSolidmechanics2.cpp:1137-1145)
                if (presc && iter == 1)
                    for (size_t i = 0; i < nd; ++i) disp[i] += lift[i];
                if (p->p0) {
                    std::vector<double> du(nd, 0.0);
                    for (int i = 0; i < n; ++i) du[P.assy_for_soln[i]] = dx[i];
                    p0_pressure_update(p, du.data());
                }
            }
            if (rows < max_hist && hist) {
                hist[4 * rows + 0] = steps_done;
                hist[4 * rows + 1] = iter;
                hist[4 * rows + 2] = norm;
                hist[4 * rows + 3] = its;
                ++rows;
            }
            if (stop) break;
        }
        if (converged) {
            ++steps_done;
        } else {
            t -= dt;
            dt *= 0.5;
            if (dt < dt0 * 0.01) return -1;
            std::copy(disp_prev.begin(), disp_prev.end(), disp);
            if (p->p0) p->pe = p->pe_prev;
        }
    }
    return rows;
}

// compute_constants_volumetric_functions (utilitiesmaterialHyperelastic.cpp:144-173), finite
// strain: Jhat = Jn - U'(Jn)/U''(Jn), thetahat = 1/U''(Jn) (Utype -1: 1 and 0).
void orc_mixed_constants(int Utype, double Jn, double K, double* Jhat, double* thetahat) {
    if (Utype == -1) {
        *Jhat = 1.0;
        *thetahat = 0.0;
        return;
    }
    const double d1 = orc_vol_dU(Utype, K, Jn), d2 = orc_vol_d2U(Utype, K, Jn);
    *Jhat = Jn - d1 / d2;
    *thetahat = 1.0 / d2;
}

// ElementBase::calcStiffnessAndResidualMixed3D (ElementBase2.cpp:278-553) for
// Elem_Solid_3D_Mixed1 with the tet10 displacement and the linear (vertex) pressure of
// Elem_Solid_3D_Mixed1.cpp:55-75, STATIC scheme (af = 1, no inertia or body force). X, u, u_prev:
// [10][3]; pn: the 4 vertex pressures. Kuu [30][30], Kup [30][4], Kpu [4][30], Kpp [4][4], FU [30],
// FP [4], row-major. Returns 0, 1 when some Gauss point has det F < 0, 2 for npe != 10.
// ElementBase::calcStiffnessAndResidualMixed3D (ElementBase2.cpp:278-553) for NP pressure
// functions: NP = 4, the tet10 vertex-linear pressure of Elem_Solid_3D_Mixed1 (pn: the vertex
// pressures), or NP = 1, the constant pressure of Elem_Solid_3D_Mixed0 (Np = 1, pn[0] = the
// element's pressure; :385-389), on the hex8 or tet10 displacement element.
static int mixed_blocks(int npe, int NP, const double* X, const double* u, const double* u_prev, const double* pn,
                        int model, const double* data, double Kinv, int Utype, double* Kuu, double* Kup, double* Kpu,
                        double* Kpp, double* FU, double* FP) {
    const int NS = 3 * npe;
    GaussRule rule;
    element_rule(npe, rule);
    std::fill(Kuu, Kuu + NS * NS, 0.0);
    std::fill(Kup, Kup + NS * NP, 0.0);
    std::fill(Kpu, Kpu + NP * NS, 0.0);
    std::fill(Kpp, Kpp + NP * NP, 0.0);
    std::fill(FU, FU + NS, 0.0);
    std::fill(FP, FP + NP, 0.0);
    const double BULK = 1.0 / Kinv;
    double x[3 * kMaxNpe];
    for (int a = 0; a < 3 * npe; ++a) x[a] = X[a] + u[a];
    int bad = 0;
    for (int q = 0; q < rule.ngp; ++q) {
        double N[kMaxNpe], dN[3][kMaxNpe], g0[3][kMaxNpe], g[3][kMaxNpe];
        shape(npe, rule.xi[q], N, dN);
        const double dvol0 = rule.w[q] * spatial_gradients(npe, X, dN, g0);
        double F[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, Fn[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        for (int I = 0; I < npe; ++I)
            for (int a = 0; a < 3; ++a)
                for (int m = 0; m < 3; ++m) {
                    F[3 * a + m] += u[3 * I + a] * g0[m][I];
                    Fn[3 * a + m] += u_prev[3 * I + a] * g0[m][I];
                }
        double Fa[3][3], Fna[3][3];
        for (int i = 0; i < 9; ++i) {
            Fa[i / 3][i % 3] = F[i];
            Fna[i / 3][i % 3] = Fn[i];
        }
        double Jhat, thetahat;
        orc_mixed_constants(Utype, det3(Fna), BULK, &Jhat, &thetahat);
        const double J = det3(Fa);
        if (J < 0.0) bad = 1;
        const double dvol = rule.w[q] * spatial_gradients(npe, x, dN, g);
        // pressure basis: LagrangeBasisFunsTetra(4) (the barycentric coordinates, vertex order),
        // LagrangeBasisFunsHexa(8) (trilinear, the hex27's corner nodes), or Np = 1
        const double* xi = rule.xi[q];
        double Np[8] = {1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (NP == 4) {
            Np[0] = 1.0 - xi[0] - xi[1] - xi[2];
            Np[1] = xi[0];
            Np[2] = xi[1];
            Np[3] = xi[2];
        } else if (NP == 8) {
            double dNp[3][kMaxNpe];
            shape_hex8(xi, Np, dNp);
        }
        double pres = 0.0;
        for (int i = 0; i < NP; ++i) pres += Np[i] * pn[i];
        double stre[9], C[81];
        if (orc_material_stress_tangent_mixed(model, data, Kinv, Utype, F, pres, stre, C) != 0) return 2;
        for (int I = 0; I < npe; ++I) {
            const double bb[3] = {dvol * g[0][I], dvol * g[1][I], dvol * g[2][I]};
            double Gc[3][9];
            for (int kk = 0; kk < 9; ++kk)
                for (int a = 0; a < 3; ++a)
                    Gc[a][kk] = bb[0] * C[9 * a + kk] + bb[1] * C[9 * (3 + a) + kk] + bb[2] * C[9 * (6 + a) + kk];
            for (int a = 0; a < 3; ++a)
                FU[3 * I + a] -= bb[0] * stre[a] + bb[1] * stre[3 + a] + bb[2] * stre[6 + a];
            for (int Jn = 0; Jn < npe; ++Jn) {
                const double c[3] = {g[0][Jn], g[1][Jn], g[2][Jn]};
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        Kuu[(3 * I + a) * NS + 3 * Jn + b] +=
                            Gc[a][b] * c[0] + Gc[a][3 + b] * c[1] + Gc[a][6 + b] * c[2];
            }
            for (int j = 0; j < NP; ++j)
                for (int a = 0; a < 3; ++a) Kup[(3 * I + a) * NP + j] += bb[a] * Np[j];
        }
        const double resip = J - Jhat - thetahat * pres;
        for (int i = 0; i < NP; ++i) {
            const double b4 = dvol * Np[i];
            FP[i] -= dvol0 * Np[i] * resip;
            for (int Jn = 0; Jn < npe; ++Jn)
                for (int b = 0; b < 3; ++b) Kpu[i * NS + 3 * Jn + b] += b4 * g[b][Jn];
            for (int j = 0; j < NP; ++j) Kpp[i * NP + j] -= dvol0 * Np[i] * thetahat * Np[j];
        }
    }
    return bad;
}

// Elem_Solid_3D_Mixed1 (Elem_Solid_3D_Mixed1.cpp:34-76): tet10 with 4 vertex pressures, or the
// 27-node hex with 8 corner pressures (P2-P1).
int orc_elem_mixed(int npe, const double* X, const double* u, const double* u_prev, const double* pn, int model,
                   const double* data, double Kinv, int Utype, double* Kuu, double* Kup, double* Kpu, double* Kpp,
                   double* FU, double* FP) {
    if (npe != 10 && npe != 27) return 2;
    return mixed_blocks(npe, npe == 10 ? 4 : 8, X, u, u_prev, pn, model, data, Kinv, Utype, Kuu, Kup, Kpu, Kpp, FU,
                        FP);
}

int orc_elem_mixed0(int npe, const double* X, const double* u, const double* u_prev, double pres, int model,
                    const double* data, double Kinv, int Utype, double* K, double* F, double* kup, double* kpp,
                    double* fp) {
    if (npe != 8 && npe != 10) return 2;
    const int ns = 3 * npe;
    double Kpu[3 * kMaxNpe], Kpp = 0.0, FP = 0.0;
    const int bad = mixed_blocks(npe, 1, X, u, u_prev, &pres, model, data, Kinv, Utype, K, kup, Kpu, &Kpp, F, &FP);
    if (bad == 2) return 2;
    // static condensation of the element pressure (Elem_Solid_3D_Mixed0.cpp:97-98)
    for (int i = 0; i < ns; ++i) {
        for (int j = 0; j < ns; ++j) K[i * ns + j] -= kup[i] * (Kpu[j] / Kpp);
        F[i] -= kup[i] * (FP / Kpp);
    }
    *kpp = Kpp;
    *fp = FP;
    return bad;
}

int orc_problem_set_mixed_p0(orc_problem* p, int enable) {
    for (size_t k = 0; k < p->mats.size() / 3; ++k)
        if (enable && (int)p->mats[3 * k + 2] == -1) return 2;
    p->p0 = enable != 0;
    const size_t ne = (size_t)p->n_elem;
    p->pe.assign(ne, 0.0);
    p->pe_prev.assign(ne, 0.0);
    p->kup.assign(ne * 3 * p->npe, 0.0);
    p->kpp.assign(ne, 0.0);
    p->fp.assign(ne, 0.0);
    p->disp_prev.assign(3 * (size_t)p->n_node, 0.0);
    return 0;
}

void orc_problem_p0_pressure(const orc_problem* p, const double* set, double* get) {
    if (set) std::copy(set, set + p->n_elem, p->pe.begin());
    if (get) std::copy(p->pe.begin(), p->pe.end(), get);
}

void orc_problem_save_step(const orc_problem* p, const double* disp) {
    p->disp_prev.assign(disp, disp + 3 * (size_t)p->n_node);
    p->pe_prev = p->pe;
}

// femSolidmechanics::solveWithArclength (femSolidmechanics2.cpp:855-1039) with
// SolverPetsc::solveArclengthSystem (SolverPetsc.cpp:671-757), psi = 1, static scheme.
// Per step: extrapolate disp and the load factor from the two last converged steps (after the
// first), then iterations 1..max_newton-1 of: assemble, R += lambda F, stop when ||R|| < tol;
// du2 = -K^{-1} R, du1 = K^{-1} F, dl = (a.du2 - A) / (b + a.du1) with the spherical constraint
// (A = Du.Du + Dl^2 F.F - Ds^2, a = 2 Du, b = 2 Dl F.F; step 1: A = 0, a = 0, b = 1, so dl = 0),
// disp += -du2 + dl du1, lambda += dl. F.F runs over every DOF (the full Fext), Du over the free
// ones. Arc length after step 1: Ds = sqrt(Du.Du + lambda^2 F.F), its bounds [Ds/1024, Ds];
// doubled after two converged steps in a row, halved (quartered after a failure) on failure.
// Returns the history rows, or -1 when the first step does not converge (the reference then
// reads its arc length before setting it).
int orc_arclength_run(const orc_problem* p, const double* fnodal, const orc_newton_opts* o, double* disp,
                      double* lambdas, int max_lambdas, int* n_lambdas, double* hist, int max_hist) {
    const CsrPattern& P = p->pat;
    const int n = P.n_free;
    const size_t nd = 3 * (size_t)p->n_node;
    std::vector<double> val(P.rowptr.back()), rhs(n), fshort(n), du1(n), x1(n), du_full(nd, 0.0);
    std::vector<double> disp_prev(disp, disp + nd), disp_prev2(disp, disp + nd);
    double FtF = 0.0;
    for (size_t i = 0; i < nd; ++i) FtF += fnodal[i] * fnodal[i];
    for (int i = 0; i < n; ++i) fshort[i] = fnodal[P.assy_for_soln[i]];
    auto dot_free = [&](const std::vector<double>& a_full, const std::vector<double>& b) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) s += a_full[P.assy_for_soln[i]] * b[i];
        return s;
    };
    double t = 0.0;
    double lam = o->dt, lam_prev = 0.0, lam_prev2 = 0.0;
    double ds = 0.0, ds_prev = 0.0, ds_max = 0.0, ds_min = 0.0;
    bool conv = false, conv_prev = false;
    int steps_done = 1, rows = 0, nl = 0;
    while (t <= o->t_final - 1.0e-10 && steps_done <= o->max_steps) {
        t += o->dt;  // timeUpdate: myTime.update
        conv_prev = conv;
        conv = false;
        if (steps_done > 1) {
            const double f = ds / ds_prev;
            for (size_t i = 0; i < nd; ++i) disp[i] = (1.0 + f) * disp_prev[i] - f * disp_prev2[i];
            lam = (1.0 + f) * lam_prev - f * lam_prev2;
        }
        for (size_t i = 0; i < nd; ++i) du_full[i] = disp[i] - disp_prev[i];
        double dlam = lam - lam_prev;
        double norm = -1.0, tol = o->tol_abs;
        for (int iter = 1; iter < o->max_newton; ++iter) {
            const int64_t bad = orc_problem_assemble(p, disp, val.data(), rhs.data(), nullptr, o->nthreads);
            if (bad >= 0) break;  // the element throws; the iteration loop ends
            for (int i = 0; i < n; ++i) rhs[i] += lam * fshort[i];
            double s2 = 0.0;
            for (int i = 0; i < n; ++i) s2 += rhs[i] * rhs[i];
            norm = std::sqrt(s2);
            if (iter == 1) tol = std::max(o->tol_abs, o->tol_rel * norm);
            int its1 = 0, its2 = 0;
            const bool done = norm < tol;
            if (!done) {
                double A = 0.0, b = 1.0, adu2 = 0.0, adu1 = 0.0, fn = 0.0;
                orc_cg_jacobi(p, val.data(), rhs.data(), x1.data(), o->cg_rtol, 1.0e-50, o->cg_maxit, o->nthreads,
                              &its1, &fn);  // du2 = -x1
                orc_cg_jacobi(p, val.data(), fshort.data(), du1.data(), o->cg_rtol, 1.0e-50, o->cg_maxit,
                              o->nthreads, &its2, &fn);
                if (steps_done > 1) {
                    double dd = 0.0;
                    for (int i = 0; i < n; ++i) dd += du_full[P.assy_for_soln[i]] * du_full[P.assy_for_soln[i]];
                    A = dd + dlam * dlam * FtF - ds * ds;
                    b = 2.0 * dlam * FtF;
                    adu2 = -2.0 * dot_free(du_full, x1);
                    adu1 = 2.0 * dot_free(du_full, du1);
                }
                const double dl = (adu2 - A) / (b + adu1);
                for (int i = 0; i < n; ++i) {
                    const double d = x1[i] + dl * du1[i];
                    disp[P.assy_for_soln[i]] += d;
                    du_full[P.assy_for_soln[i]] += d;
                }
                lam += dl;
                dlam += dl;
            }
            if (rows < max_hist && hist) {
                hist[5 * rows + 0] = steps_done;
                hist[5 * rows + 1] = iter;
                hist[5 * rows + 2] = norm;
                hist[5 * rows + 3] = its1 + its2;
                hist[5 * rows + 4] = lam;
                ++rows;
            }
            if (done) {
                conv = true;
                break;
            }
        }
        if (conv) {
            if (steps_done == 1) {
                double dd = 0.0;
                for (size_t i = 0; i < nd; ++i) dd += du_full[i] * du_full[i];
                ds = std::sqrt(dd + lam * lam * FtF);
                ds_max = ds;
                ds_min = ds / 1024.0;
            }
            lam_prev2 = lam_prev;
            lam_prev = lam;
            disp_prev2 = disp_prev;
            std::copy(disp, disp + nd, disp_prev.begin());
            ds_prev = ds;
            if (conv_prev) ds = std::min(std::max(2.0 * ds, ds_min), ds_max);
            if (nl < max_lambdas && lambdas) lambdas[nl] = lam;
            ++nl;
            ++steps_done;
        } else {
            if (steps_done == 1) {
                if (n_lambdas) *n_lambdas = nl;
                return -1;
            }
            ds = std::max(ds * (conv_prev ? 0.5 : 0.25), ds_min);
        }
    }
    if (n_lambdas) *n_lambdas = nl;
    return rows;
}

}  // extern "C"
