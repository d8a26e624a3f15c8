// gnn.cuh -- learned factorised sparse approximate inverse: a message-passing network that predicts
// the FSAI blocks G on the lower block pattern of the assembled operator.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"
#include "fsai.cuh"
#include "krylov.cuh"

namespace mphy {

constexpr int kGnnH = 64;       // width
constexpr int kGnnLayers = 3;   // message-passing layers
constexpr int kGnnNodeIn = 13;  // scaled diagonal block (9), prescribed flags (3), degree / 27
constexpr int kGnnEdgeIn = 9;   // scaled off-diagonal block

// Offsets of the flat FP32 parameter vector (the order of the host-side arrays).
struct GnnLayout {
    static constexpr int w_in = 0, b_in = w_in + kGnnH * kGnnNodeIn;
    static constexpr int layer0 = b_in + kGnnH;
    // per layer: U [H][H], V [H][9], c [H], S [H][H], T [H][H], d [H]
    static constexpr int U = 0, V = U + kGnnH * kGnnH, c = V + kGnnH * kGnnEdgeIn, S = c + kGnnH,
                         Tm = S + kGnnH * kGnnH, d = Tm + kGnnH * kGnnH, layer_size = d + kGnnH;
    static constexpr int dec = layer0 + kGnnLayers * layer_size;
    // decoder: Wa [9][H], Wb [9][H], Wc [9][9], bo [9]
    static constexpr int Wa = dec, Wb = Wa + 9 * kGnnH, Wc = Wb + 9 * kGnnH, bo = Wc + 81, total = bo + 9;
    static constexpr int layer(int l) { return layer0 + l * layer_size; }
};

// Per-operator graph: features and targets in the network's scaled units.
struct GnnGraph {
    int32_t n_node = 0;
    int64_t n_lower = 0;
    DevBuf<float> sqrt_s;     // [3 n_node] sqrt of |diag| (1 on prescribed DOFs)
    DevBuf<float> xnode;      // [n_node][13]
    DevBuf<int32_t> deg;      // [n_node] neighbours other than itself
    DevBuf<int32_t> lslot;    // [n_lower] position of the lower block (n, m) in A's row n
    DevBuf<int32_t> lrow_of;  // [n_lower] row n of every lower block
    DevBuf<int64_t> u2l;      // [n_lower] compact lower index of the k-th upper entry (G^T rows)
    DevBuf<float> base;       // [n_node][9] block-Jacobi FSAI diagonal blocks (scaled units)
    bool training = false;    // run() evaluates the loss (and gradients)
};

class Gnn {
  public:
    void init(mphy_ctx* ctx, const float* params_host);
    void set_params(const float* host);
    void get_params(float* host) const;
    void get_grads(float* host) const;
    // Features of the assembled operator (training: run() also evaluates the loss).
    void build_graph(GnnGraph& g, const mphy_pattern* P, const Fsai& F, const SellView& A, const void* aval,
                     bool fp32_values, const uint8_t* fixed, bool training, cudaStream_t s);
    // Forward pass; writes predicted G blocks (unscaled, FP32) into out_blocks when non-null.
    // For a training graph, returns the Kaporin loss log K(G A G^T) - (1/N) log det A^ and
    // (compute_grad) accumulates its gradients.
    double run(const GnnGraph& g, const mphy_pattern* P, const Fsai& F, const SellView& A, const void* aval,
               bool fp32_values, const uint8_t* fixed, float* out_blocks, bool compute_grad, cudaStream_t s);
    void zero_grads(cudaStream_t s);
    void adam_step(float lr, float beta1, float beta2, float eps, cudaStream_t s);
    int64_t launches = 0;

  private:
    void ensure_workspace(int32_t n_node, int64_t n_lower);
    mphy_ctx* ctx_ = nullptr;
    DevBuf<float> w_, grad_, m_, v_;   // FP32 master weights, gradients, Adam moments
    DevBuf<__nv_bfloat16> wb_;         // BF16 copy used by the kernels
    DevBuf<double> loss_;
    int64_t adam_t_ = 0;
    int32_t ws_nodes_ = 0;
    int64_t ws_lower_ = 0;
    // activations: h_l for l = 0..L ([n][H] each), P, msg, q per layer, decoder partials
    DevBuf<float> h_, P_, msg_, q_, dh_, dP_, dmsg_, dq_, an_, bn_, dout_, dan_, dbn_;
    DevBuf<float> ghat_, tbuf_;        // predicted scaled blocks, T_j of the loss
    DevBuf<double> part_tr_, part_ld_, red_;
};

}  // namespace mphy
