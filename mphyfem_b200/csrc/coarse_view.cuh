// coarse_view.cuh -- device view of the rigid-body coarse space (see coarse.cuh).
#pragma once
#include <stdint.h>

namespace mphy {

struct CoarseView {
    int32_t n_agg;           // aggregates (boxes)
    int32_t k;               // coarse size 6 n_agg (padded to kp in storage)
    int32_t kp;              // padded size (multiple of 64)
    const int32_t* agg;      // [n_node] aggregate of every node
    const int64_t* agg_ptr;  // [n_agg+1] nodes of every aggregate (in agg_nodes)
    const int32_t* agg_nodes;
    const double* d;         // [n_node][3] (x_n - c_agg) / H_agg at setup
    const uint8_t* fixed;    // [3 n_node]
    // [kp][kp] inverse of E (row-major), FP64: with a large stiffness contrast E is so
    // ill-conditioned that rounding its inverse to FP32 makes the coarse term indefinite, and CG
    // on an indefinite preconditioner stalls
    const double* einv;
    double* w;               // [kp] restriction Z^T r
    double* c;               // [kp] coarse correction E^{-1} w
};

}  // namespace mphy
