// coarse.cuh -- two-level preconditioner: a rigid-body coarse space on geometric aggregates.
//
//   M^{-1} r = D^{-1} r + Z E^{-1} Z^T r,   E = Z^T A Z,
// Z holding, for every box of a regular grid of boxes over the mesh, the six rigid-body modes
// (three translations, three rotations about the box centroid) of its nodes, zero on prescribed
// DOFs. M^{-1} is symmetric positive definite, so CG keeps its guarantees; the coarse term takes
// care of the global, smooth modes (beam bending) that no local preconditioner reaches.
#pragma once
#include <vector>

#include "common.cuh"
#include "coarse_view.cuh"
#include "krylov.cuh"

namespace mphy {

class CoarseSpace {
  public:
    // Aggregates: a grid of boxes over the bounding box of the reference coordinates with about
    // target_aggregates boxes, as close to cubes as the box allows.
    // modes: 6 (rigid-body: translations and rotations about the box centroid) or 12 (linear
    // displacement u = a + B d: translations, stretches, shears and rotations)
    void init(mphy_ctx* ctx, const mphy_mesh* mesh, const mphy_pattern* pat, int target_aggregates, int modes = 6);
    // Modes from the current coordinates X + disp (disp may be null), E = Z^T A Z, its Cholesky
    // factor and inverse, all FP64.
    template <typename VT>
    void setup(const SellView& A, const VT* aval, const double* disp, cudaStream_t s);
    CoarseView view() const;
    int n_agg() const { return n_agg_; }
    int coarse_size() const { return nm_ * n_agg_; }
    int modes() const { return nm_; }
    const int* grid() const { return ng_; }
    int64_t launches = 0;
    float last_setup_ms = 0.f;

    ~CoarseSpace();

  private:
    void record_factorisation(cudaStream_t s, int nb, size_t sm2);
    void build_entry_lists(const SellView& A, cudaStream_t s);
    cudaGraphExec_t fact_graph_ = nullptr;
    cudaStream_t side_[2] = {nullptr, nullptr};  // captured side streams of the factorisation
    cudaEvent_t ev_[3] = {nullptr, nullptr, nullptr};
    int64_t fact_launches_ = 0;
    double boxd_ = 0.0;
    int nm_ = 6;
    mphy_ctx* ctx_ = nullptr;
    const mphy_mesh* mesh_ = nullptr;
    const mphy_pattern* pat_ = nullptr;
    int ng_[3] = {1, 1, 1};   // boxes along x, y, z
    int ngl_[3] = {1, 1, 1};  // boxes along the numbering's axes, fastest first (fewest boxes first)
    int band_tiles_ = 0;      // tiles of E's Cholesky factor below the diagonal tile that can be nonzero
    int n_agg_ = 0, kp_ = 0;
    DevBuf<int32_t> agg_, agg_nodes_, err_;
    DevBuf<int32_t> aggbox_;  // [n_node] aggregate box bx | by << 10 | bz << 20
    DevBuf<int64_t> agg_ptr_;
    DevBuf<float> d_;       // FP32 offsets (x_n - c_a) / H
    DevBuf<double> cent_, E_, W_, w_, c_;
    DevBuf<float> w32_;       // lower tiles of W = L^{-1}, FP32
    DevBuf<double> y_, gpart_, rowyy_;
    DevBuf<uint8_t> drop_;
    DevBuf<double> wpart_;
    DevBuf<uint32_t> wcount_;
    // E = Z^T A Z in two passes (built at the first setup of a layout): per node, the lower
    // neighbour slots its row reaches and the offset of its entries (T_{n,b} = sum_{m in b} A_nm
    // Z_m, own box first); per (aggregate, slot), the list of entries and nodes to add, in order
    bool lists_ready_ = false;
    std::vector<int32_t> nodes_host_;  // agg_nodes
    std::vector<int64_t> ptr_host_;    // agg_ptr
    DevBuf<uint16_t> lmask_;
    DevBuf<int32_t> toff_, lent_, lnode_;
    DevBuf<int64_t> lptr_;
    DevBuf<double> tbuf_;
    DevBuf<float> dperm_;   // d in agg_nodes order
    DevBuf<uint8_t> fperm_; // fixed in agg_nodes order
};

}  // namespace mphy
