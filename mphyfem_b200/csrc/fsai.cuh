// fsai.cuh -- K5: factorised sparse approximate inverse M = G^T G on A's lower block pattern.
#pragma once
#include "common.cuh"
#include "krylov.cuh"

namespace mphy {

// SELL-32 3x3 layout of a block pattern given as sorted block-CSR rows (see mphy_pattern).
struct SellPattern {
    int32_t n_node = 0, n_slices = 0;
    int64_t n_blocks = 0, stored_blocks = 0;
    DevBuf<int64_t> rowptr;      // [n_node+1] compact block CSR
    DevBuf<int32_t> col;         // [n_blocks]
    DevBuf<int64_t> slice_base;  // [n_slices+1]
    DevBuf<int32_t> slice_width; // [n_slices]
    DevBuf<int32_t> sell_col;    // [stored_blocks]
    SellView view() const {
        return SellView{n_node, n_slices, slice_base.p, slice_width.p, sell_col.p, nullptr};
    }
};

// G (lower) and G^T (upper) patterns and values. The lower row of node n is n's neighbours
// m <= n ascending (n last); the upper row is m >= n (n first).
class Fsai {
  public:
    // Builds both patterns from the matrix pattern. Limits the lower row to max_lower blocks
    // (the nearest, i.e. largest indices, are kept) so the local systems fit shared memory.
    void init(mphy_ctx* ctx, const mphy_pattern* A, int max_lower = 16);
    // Exact block FSAI of the assembled operator (values VT: double or float), FP64 local
    // Cholesky per block row, G and G^T stored in BF16 (FactorT).
    // diag64 / fixed: the null-space-preserving storage of the mixed path (null for FP64).
    template <typename VT>
    void compute(const VT* aval, const double* diag64, const uint8_t* fixed, cudaStream_t s);
    // Install externally predicted G blocks (lower pattern order, [n_blocks][9] row-major FP32)
    // and mirror them into G^T.
    void set_lower_values(const float* gblocks, cudaStream_t s);
    // lower-pattern blocks of G in compact order [n_blocks][9] (for training and checks)
    void get_lower_values(float* out_dev, cudaStream_t s) const;
    FactorView<FactorT> view() const;
    const SellPattern& lower() const { return L_; }
    const SellPattern& upper() const { return U_; }
    int max_lower() const { return max_lower_; }
    int32_t fallback_rows(cudaStream_t s) const;
    int64_t launches = 0;

  private:
    mphy_ctx* ctx_ = nullptr;
    const mphy_pattern* A_ = nullptr;
    int max_lower_ = 16;
    SellPattern L_, U_;
    DevBuf<FactorT> gval_, gtval_;     // SELL values of G and G^T
    DevBuf<int64_t> l2sell_;           // compact lower block -> SELL value offset in G
    DevBuf<int64_t> l2usell_;          // compact lower block (n, m) -> SELL value offset of (m, n) in G^T
    DevBuf<int32_t> err_;
};

}  // namespace mphy
