// nh.cuh -- the Neo-Hookean material at a Gauss point, shared by the element kernels.
#pragma once
#include "../../include/mphy.h"

namespace mphy {

// U'(J) and U''(J) of the volumetric energies (utilitiesmaterialHyperelastic.cpp:45-140).
__device__ __forceinline__ void vol_derivs(int type, double K, double J, double& d1, double& d2) {
    switch (type) {
        case 3: d1 = K * (J - 1.0); d2 = K; break;
        case 1: d1 = 0.1 * K * (J * J * J * J - 1.0 / (J * J * J * J * J * J));
                d2 = 0.2 * K * (2.0 * J * J * J + 3.0 / (J * J * J * J * J * J * J)); break;
        case 2: d1 = 0.125 * K * (J * J - 1.0 / (J * J)) * (J + 1.0 / (J * J * J));
                d2 = 0.125 * K * (3.0 * J * J + 5.0 / (J * J * J * J * J * J)); break;
        case 4: d1 = 0.5 * K * (J - 1.0 / J); d2 = 0.5 * K * (1.0 + 1.0 / (J * J)); break;
        case 5: d1 = 0.5 * K * (J - 1.0 + log(J) / J); d2 = 0.5 * K * (J * J + 1.0 - log(J)) / (J * J); break;
        case 6: d1 = K * log(J); d2 = K / log(J); break;
        case 7: d1 = K * (1.0 - 1.0 / J); d2 = K / (J * J); break;
        case 8: d1 = K * log(J) / J; d2 = K * (1.0 - log(J)) / (J * J); break;
        default: d1 = 0.0; d2 = 0.0; break;
    }
}

// Per-Gauss-point Neo-Hookean factors (see the file header). b is the symmetric F F^T.
struct NhFactors {
    double s1, s2;              // sigma = s1 b + s2 I
    double c1, c2, c3, f4, f9;  // tangent factors
};

__device__ __forceinline__ NhFactors nh_factors(const double b[3][3], double J, double mu, double Kinv,
                                                int utype, int tangent) {
    const double K = 1.0 / Kinv;
    const double Ib = b[0][0] + b[1][1] + b[2][2];
    const double jm13 = rcbrt(J);
    const double jm53 = jm13 * jm13 / J;  // J^{-5/3}
    double dU, d2U;
    vol_derivs(utype, K, J, dU, d2U);
    NhFactors f;
    f.s1 = mu * jm53;
    f.s2 = -f.s1 * (1.0 / 3.0) * Ib + dU;
    f.c1 = (1.0 / 3.0) * mu * jm53 * Ib - dU;
    f.c2 = -(2.0 / 3.0) * mu * jm53;
    f.c3 = (2.0 / 3.0) * (1.0 / 3.0) * mu * jm53 * Ib + (J * d2U + dU);
    f.f4 = mu * jm53;
    f.f9 = tangent == MPHY_TANGENT_CONSISTENT ? 0.0 : -dU;
    return f;
}

}  // namespace mphy
