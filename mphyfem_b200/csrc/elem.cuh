// elem.cuh -- K1 element kernels and the batched material call.
#pragma once
#include "common.cuh"

namespace mphy {

struct ElemArgs {
    int64_t n_elem;
    const double* coords;   // [n_node][3]
    const int32_t* conn;    // [n_elem][npe]
    const int32_t* mat_id;  // [n_elem]
    const double* mats;     // [n_mat][4] = mu, Kinv, Utype, 0 (Neo-Hookean kernels)
    const double* matx = nullptr;  // [n_mat][8] = model, data0..3, Kinv, Utype, 0 (general kernel)
    const double* disp;     // [n_node*3]
    int tangent;
    unsigned long long* bad;  // min element id with det F < 0 (init ULLONG_MAX)
    uint8_t* bad_elem = nullptr;  // optional per-element flag (set to 1) for det F < 0
    // export (mode bit 1)
    double* Ke;
    double* Re;
    // assembly (mode bit 2)
    const uint8_t* fixed;
    const uint32_t* e2v;
    double* val;   // SELL values (FP64), or
    float* valf;   // SELL values (FP32) when non-null; then the scatter stores off-diagonal blocks
                   // only, without Dirichlet masking (null-space-preserving storage)
    double* rhs;   // [n_node*3], prescribed DOFs untouched
    double* reac;  // [n_node*3] or null
    double* diag_out = nullptr;  // FP32 storage: [n_node][9] FP64 diagonal blocks accumulated per
                                 // element (elem_f32.cu), for the preconditioners
    int diag_full = 1;           // 0: only the blocks' diagonal entries (all that Jacobi reads)
    const double* lift = nullptr;  // [n_node*3] increments of prescribed displacements (zero on
                                   // free DOFs): free rows get -K lift (applyDirichletBCs)
};

void upload_shape_tables();
void upload_shape_tables_tc(const double* h8, const double* w8, const double* t10, const double* w4);
void launch_elem_fp64(const ElemArgs& a, int npe, int mode, cudaStream_t s);
// Mixed-precision element kernel (elem_tc.cu): FP64 residual, tangent contraction on tensor
// cores (split-BF16, FP32 accumulation), FP32 off-diagonal scatter (a.valf) or Ke export.
void launch_elem_tc(const ElemArgs& a, int npe, int mode, cudaStream_t s);
// Mixed-precision element kernel (elem_f32.cu): FP64 kinematics, stress and residual, FP32
// tangent blocks formed once per symmetric pair, coalesced FP32 scatter into a.valf, element
// diagonal blocks into a.diag_out. Assembly only (Neo-Hookean, hex8 / tet10).
void launch_elem_f32(const ElemArgs& a, int npe, cudaStream_t s);
void upload_shape_tables_f32(const double* h8, const double* w8, const double* t10, const double* w4);
// Element kernel for any material model of the table a.matx (elem_gen.cu).
void launch_elem_gen(const ElemArgs& a, int npe, int mode, cudaStream_t s);
void upload_shape_tables_gen(const double* h8, const double* w8, const double* t10, const double* w4);
void launch_material_eval(int n, const double* F, const double* row_dev, int tangent, double* stre, double* C,
                          cudaStream_t s);
void launch_nh_eval(int n, const double* F, double mu, double Kinv, int utype, int tangent, double* stre,
                    double* C, cudaStream_t s);
void launch_scatter_batch(int npe, int32_t n, const int32_t* ids, const mphy_mesh* mesh, const mphy_pattern* P,
                          const double* Ke, const double* Re, double* val, float* valf, double* rhs, double* reac,
                          cudaStream_t s, int sm_count);

}  // namespace mphy
