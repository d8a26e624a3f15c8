// coarse_view.cuh -- device view of the geometric coarse space (see coarse.cuh).
#pragma once
#include <stdint.h>

namespace mphy {

// Most CTAs that share one aggregate's restriction sum (w = Z^T r).
constexpr int kMaxRestrictParts = 16;

struct CoarseView {
    int32_t n_agg;           // aggregates (boxes)
    int32_t nm;              // modes per aggregate: 6 (rigid body) or 12 (linear displacement)
    int32_t k;               // coarse size nm n_agg (padded to kp in storage)
    int32_t kp;              // padded size (multiple of 64)
    const int32_t* agg;      // [n_node] aggregate of every node
    const int64_t* agg_ptr;  // [n_agg+1] nodes of every aggregate (in agg_nodes)
    const int32_t* agg_nodes;
    const float* d;          // [n_node][3] (x_n - c_agg) / H_agg at setup, FP32 (one rounded basis)
    const uint8_t* fixed;    // [3 n_node]
    const float* dperm;      // [n_node][3] d in the order of agg_nodes (the restriction's loads)
    const uint8_t* fperm;    // [3 n_node] fixed in the order of agg_nodes
    int32_t nb;              // kp / 64 tiles per side
    // E^{-1} = W^T W with W = L^{-1} (E = L L^T), applied as W~^T (W~ w) with W~ the FP32
    // rounding of W: its lower 64x64 tiles (I, J), J <= I, at tile index I (I + 1) / 2 + J,
    // each row-major. W~^T W~ is symmetric positive definite whatever the rounding (W~ stays
    // nonsingular), so the coarse term keeps CG's guarantees even when E is ill-conditioned;
    // the rounding only perturbs it by about 2^-24 times the condition number of W, the square
    // root of E's
    const float* w32;
    double* w;               // [kp] restriction Z^T r
    double* wpart;           // [n_agg][kMaxRestrictParts][nm] partial restriction sums
    uint32_t* wcount;        // [n_agg] parts summed so far (zero between launches)
    double* c;               // [kp] coarse correction E^{-1} w
    double* y;               // [kp] W~ w
    double* gpart;           // [tiles][2][64] the per-tile products W_IJ w_J and W_IJ^T y_I
    double* rowyy;           // [nb] each tile row's share of y^T y = w^T E^{-1} w
};

#ifdef __CUDACC__
// The coarse field at node n, (Z c)_n, with d the node's scaled offset from its aggregate's
// centroid. Rigid-body modes: c = (translation t, rotations w) and u = t + w x d with the
// mode order of the restriction; linear modes: c = (a, B row-major) and u = a + B d.
// The same with the node's aggregate and offsets already loaded.
__device__ __forceinline__ void coarse_node_value(const CoarseView& cv, int32_t agg, double dx, double dy, double dz,
                                                  double zc[3]) {
    if (cv.nm == 12) {
        const double* c = cv.c + 12 * (int64_t)agg;
#pragma unroll
        for (int a = 0; a < 3; ++a) zc[a] = c[a] + c[3 + 3 * a] * dx + c[4 + 3 * a] * dy + c[5 + 3 * a] * dz;
    } else {
        const double* c = cv.c + 6 * (int64_t)agg;
        zc[0] = c[0] - dy * c[3] + dz * c[5];
        zc[1] = c[1] + dx * c[3] - dz * c[4];
        zc[2] = c[2] + dy * c[4] - dx * c[5];
    }
}
__device__ __forceinline__ void coarse_node_value(const CoarseView& cv, int64_t n, double zc[3]) {
    coarse_node_value(cv, cv.agg[n], cv.d[3 * n], cv.d[3 * n + 1], cv.d[3 * n + 2], zc);
}
#endif

}  // namespace mphy
