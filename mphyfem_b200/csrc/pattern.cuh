// pattern.cuh -- K2 entry points (DOF map, node-block sparsity, reference CSR export).
#pragma once
#include "common.cuh"

namespace mphy {

// Exclusive scan of n values into out[0..n]; out[n] = total, also returned (synchronises).
template <typename T>
int64_t exclusive_scan(const T* in, int64_t* out, int64_t n, cudaStream_t s);

// prepareMatrixPattern on the device: incidence, sorted-unique node neighbours, SELL layout,
// element block offsets, free-DOF numbering and the reference CSR row pointer.
void build_pattern(mphy_ctx* ctx, const mphy_mesh* mesh, mphy_pattern* P);

// Materialise the reference CSR columns (and, with_src, each entry's SELL value offset).
void pattern_csr_columns(mphy_pattern* P, bool with_src);

// forAssyVec of every element into fav_dev [n_elem][3npe].
void pattern_elem_dofs(const mphy_pattern* P, const mphy_mesh* mesh, int32_t* fav_dev);

}  // namespace mphy
