// mat.cuh -- the hyperelastic models of MaterialBase's family at a Gauss point: Cauchy stress
// and 9x9 spatial tangent in the reference's index order (map_tensor4: q -> (q % 3, q / 3)).
//
// Every model here (Matl_NeoHookean, Matl_MooneyRivlin, Matl_Gent, Matl_ArrudaBoyce, compressible
// branch of utilitiesmaterialHyperelastic.cpp) has a stress of the form
//     sigma = s1 b + s2 I + s3 b^2
// and a tangent that is a combination of twelve isotropic fourth-order terms in I, b = F F^T and
// b^2:
//     C_ijkl = k0 d_il d_jk + k1 b_ij d_kl + k2 d_ij b_kl + k3 d_ij d_kl + k4 d_ik b_jl + k5 d_ik d_jl
//            + k6 b_ij b_kl + k7 b_ik b_jl + k8 b_il b_kj + k9 d_ik b2_jl + k10 d_ij b2_kl + k11 b2_ij d_kl
// Each model computes its scalars (s, k); one unrolled fill writes the entries. The coefficient
// of each term is the reference's, collected: e.g. Gent's fact2 * bbdev_ij bbdev_kl expands into
// k6 += fact2, k1 += -fact2 Ib/3, k2 += -fact2 Ib/3, k3 += fact2 Ib^2/9.
#pragma once
#include "nh.cuh"

namespace mphy {

// Device row of the material table: {model, data0, data1, data2, data3, Kinv, Utype, 0}.
constexpr int kMatRow = 8;

struct MatScalars {
    double s[3];
    double k[12];
};

__device__ __forceinline__ double pow_m23(double J) {
    const double r = rcbrt(J);
    return r * r;
}

// Neo-Hookean (:186-295), the factors of the structured kernel (nh.cuh) with U'(J), U''(J) given:
// the mixed branch passes dU = p, d2U = 0 and has no d_jl d_ik term.
__device__ __forceinline__ void nh_scalars(const double b[3][3], double J, double mu, double dU, double d2U,
                                           double f9, MatScalars& m) {
    const double Ib = b[0][0] + b[1][1] + b[2][2];
    const double jm53 = pow_m23(J) / J;
    m.s[0] = mu * jm53;
    m.s[1] = -m.s[0] * (1.0 / 3.0) * Ib + dU;
    m.k[0] = (1.0 / 3.0) * mu * jm53 * Ib - dU;
    m.k[1] = -(2.0 / 3.0) * mu * jm53;
    m.k[2] = m.k[1];
    m.k[3] = (2.0 / 3.0) * (1.0 / 3.0) * mu * jm53 * Ib + (J * d2U + dU);
    m.k[4] = mu * jm53;
    m.k[5] = f9;
}

// Mooney-Rivlin (:300-420). The reference's r7d3 is 5/3 (:303), so its J^{-7/3} factor is
// J^{-5/3}; kept as written. Both tangent modes give the symmetric tangent as written: the exact
// linearisation of this stress adds a non-symmetric (2/3) sigma_c2 (x) I term.
__device__ __forceinline__ void mr_scalars(const double b[3][3], const double b2[3][3], double J, double Ib,
                                           double c1, double c2, double dU, double d2U, MatScalars& m) {
    const double jm53 = pow_m23(J) / J;
    const double jm73 = jm53;  // r7d3 = 5/3 in the reference
    const double I2 = 0.5 * (Ib * Ib - (b2[0][0] + b2[1][1] + b2[2][2]));
    m.s[0] = 2.0 * c1 * jm53 + 2.0 * c2 * jm73 * Ib;
    m.s[1] = -c1 * (2.0 / 3.0) * jm53 * Ib - c2 * (4.0 / 3.0) * jm73 * I2 + dU;
    m.s[2] = -2.0 * c2 * jm73;
    const double f1 = 2.0 * c1 * jm53, f2 = 2.0 * c2 * jm73, f3 = (4.0 / 3.0) * c2 * jm73;
    const double f7 = J * d2U + dU, f8 = -dU;
    m.k[0] = f1 * (1.0 / 3.0) * Ib + f3 * I2 + f8;
    m.k[1] = -(2.0 / 3.0) * f1 - 2.0 * f3 * Ib;
    m.k[2] = m.k[1];
    m.k[3] = f1 * (2.0 / 9.0) * Ib + f3 * (4.0 / 3.0) * I2 + f7;
    m.k[4] = f1 + f2 * Ib;
    m.k[6] = 2.0 * f2;
    m.k[7] = -f2;
    m.k[8] = -f2;
    m.k[9] = -f2;
    m.k[10] = 2.0 * f3;
    m.k[11] = 2.0 * f3;
}

// Gent (:423-548), data {mu, Im}.
__device__ __forceinline__ void gent_scalars(double J, double Ib, double mu, double Im, double dU, double d2U,
                                             MatScalars& m) {
    const double jm23 = pow_m23(J);
    const double jm53 = jm23 / J;
    const double jm73 = jm53 * jm23;
    const double gf = 1.0 / (1.0 - (jm23 * Ib - 3.0) / Im);
    m.s[0] = mu * jm53 * gf;
    m.s[1] = -m.s[0] * (1.0 / 3.0) * Ib + dU;
    const double f1 = -(2.0 / 3.0) * mu * jm53 * gf, f2 = 2.0 * mu * jm73 * gf * gf / Im, f3 = mu * jm53 * gf;
    const double f7 = J * d2U + dU, f8 = -dU;
    const double t = Ib * (1.0 / 3.0);
    // f1 bdev_ij d_kl + f2 bdev_ij bdev_kl + f3 (d_ik b_jl - (2/3) b_kl d_ij + (Ib/3) d_il d_jk)
    m.k[0] = f3 * t + f8;
    m.k[1] = f1 - f2 * t;
    m.k[2] = -f2 * t - (2.0 / 3.0) * f3;
    m.k[3] = -f1 * t + f2 * t * t + f7;
    m.k[4] = f3;
    m.k[6] = f2;
}

// Arruda-Boyce (:551-677), data {mu, N}: five-term series c1..c5, a1 = W'(Ibbar), a2 = W''(Ibbar).
// The deviatoric tangent as written is the symmetrised form; the consistent tangent replaces its
// (2/3) a1 J^{-5/3} Ib d_ik d_jl by 2 a1 J^{-5/3} d_ik b_jl.
__device__ __forceinline__ void ab_scalars(double J, double Ib, double mu, double N, double dU, double d2U,
                                           int tangent, MatScalars& m) {
    const double c1 = mu / 2.0, c2 = mu / 20.0 / N, c3 = mu * 11.0 / 1050.0 / N / N,
                 c4 = mu * 19.0 / 7000.0 / N / N / N, c5 = mu * 519.0 / 673750.0 / N / N / N / N;
    const double jm23 = pow_m23(J);
    const double jm53 = jm23 / J;
    const double jm73 = jm53 * jm23;
    const double x = jm23 * Ib;
    const double a1 = c1 + x * (2.0 * c2 + x * (3.0 * c3 + x * (4.0 * c4 + x * 5.0 * c5)));
    const double a2 = 2.0 * c2 + x * (6.0 * c3 + x * (12.0 * c4 + x * 20.0 * c5));
    m.s[0] = 2.0 * a1 * jm53;
    m.s[1] = -m.s[0] * (1.0 / 3.0) * Ib + dU;
    const double f1 = 4.0 * jm73 * a2, f2 = -4.0 * (1.0 / 3.0) * a1 * jm53, f3 = (2.0 / 3.0) * a1 * jm53 * Ib,
                 f4 = 4.0 * (1.0 / 9.0) * a1 * jm53 * Ib;
    const double f7 = J * d2U + dU, f8 = -dU;
    const double t = Ib * (1.0 / 3.0);
    // f1 bdev_ij bdev_kl + f2 (b_ij d_kl + b_kl d_ij) + f3 (d_ik d_jl + d_il d_jk) + f4 d_ij d_kl
    m.k[0] = f3 + f8;
    m.k[1] = -f1 * t + f2;
    m.k[2] = m.k[1];
    m.k[3] = f1 * t * t + f4 + f7;
    m.k[5] = f3;
    m.k[6] = f1;
    if (tangent == MPHY_TANGENT_CONSISTENT) {
        m.k[4] += 2.0 * a1 * jm53;
        m.k[5] -= 2.0 * a1 * jm53 * t;
    }
}

// Stress and tangent scalars of material row `row` at deformation gradient F. Mixed (u-p)
// elements pass mixed = true and the Gauss-point pressure: p replaces U'(J) in the stress and
// p (d_ij d_kl - d_jk d_il) replaces the volumetric tangent (the MIXED_ELEMENT branches), which
// is U' = p, U'' = 0 in the factors below; Arruda-Boyce's written branch adds -p d_jl d_ik
// (:661-664), which the consistent tangent leaves out.
__device__ __forceinline__ MatScalars material_scalars(const double* row, int tangent, const double b[3][3],
                                                       const double b2[3][3], double J, bool mixed = false,
                                                       double pres = 0.0) {
    MatScalars m;
#pragma unroll
    for (int i = 0; i < 3; ++i) m.s[i] = 0.0;
#pragma unroll
    for (int i = 0; i < 12; ++i) m.k[i] = 0.0;
    const int model = (int)row[0];
    const double Kinv = row[5];
    const int utype = (int)row[6];
    const double Ib = b[0][0] + b[1][1] + b[2][2];
    double dU = pres, d2U = 0.0;
    if (!mixed) vol_derivs(utype, 1.0 / Kinv, J, dU, d2U);
    if (model == MPHY_MAT_NEOHOOKEAN) {
        nh_scalars(b, J, row[1], dU, d2U, (mixed || tangent == MPHY_TANGENT_CONSISTENT) ? 0.0 : -dU, m);
    } else if (model == MPHY_MAT_MOONEYRIVLIN) {
        mr_scalars(b, b2, J, Ib, row[1], row[2], dU, d2U, m);
    } else if (model == MPHY_MAT_GENT) {
        gent_scalars(J, Ib, row[1], row[2], dU, d2U, m);
    } else {
        ab_scalars(J, Ib, row[1], row[2], dU, d2U, tangent, m);
        if (mixed && tangent != MPHY_TANGENT_CONSISTENT) m.k[5] -= pres;
    }
    return m;
}

// sig[q] = scale * sigma(q % 3, q / 3); C[9 p + q] = scale * C_ijkl, (i, j) = (p % 3, p / 3),
// (k, l) = (q % 3, q / 3). C may point to shared or global memory.
__device__ __forceinline__ void material_fill(const MatScalars& m, const double b[3][3], const double b2[3][3],
                                              double scale, double* sig, double* C) {
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int i = q % 3, j = q / 3;
        sig[q] = scale * (m.s[0] * b[i][j] + m.s[2] * b2[i][j] + (i == j ? m.s[1] : 0.0));
    }
    double k[12];
#pragma unroll
    for (int t = 0; t < 12; ++t) k[t] = scale * m.k[t];
#pragma unroll
    for (int p = 0; p < 9; ++p) {
        const int i = p % 3, j = p / 3;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const int kk = q % 3, l = q / 3;
            double v = 0.0;
            if (i == l && j == kk) v += k[0];
            if (kk == l) v += k[1] * b[i][j] + k[11] * b2[i][j];
            if (i == j) v += k[2] * b[kk][l] + k[10] * b2[kk][l];
            if (i == j && kk == l) v += k[3];
            if (i == kk) v += k[4] * b[j][l] + k[9] * b2[j][l];
            if (i == kk && j == l) v += k[5];
            v += k[6] * b[i][j] * b[kk][l] + k[7] * b[i][kk] * b[j][l] + k[8] * b[i][l] * b[kk][j];
            C[9 * p + q] = v;
        }
    }
}

}  // namespace mphy
