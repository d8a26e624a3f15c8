// mixed.cuh -- the mixed u-p (tet10 displacement, linear vertex pressure) element and its
// two-field system: pressure DOFs at the vertex nodes, the coupling blocks B = Kup (u rows),
// B^T = Kpu (pressure rows) and C = Kpp, each in compressed rows.
#pragma once
#include "elem.cuh"

namespace mphy {

// Element evaluation (elem_gen.cu). MODE bit 1 exports per element Ke (= Kuu), Re (= FU), Kup
// [30][4], Kpp [4][4], FP [4]; bit 2 scatters Kuu / FU / reactions through `base` (FP64 masked
// SELL) and the coupling blocks through the element maps.
struct MixedElemArgs {
    ElemArgs base;
    const double* disp_prev;  // [3 n_node] last converged step: Jn of compute_constants_volumetric_functions
    const double* pres;       // [n_node] nodal pressures (vertex nodes)
    const int32_t* pres_id;   // [n_node] pressure DOF or -1
    // export
    double* Kup = nullptr;
    double* Kpp = nullptr;
    double* FP = nullptr;
    // assembly: entry indices of element pairs, values (3 per B / B^T entry, 1 per C entry)
    const uint32_t* e2b = nullptr;   // [n_elem][npe][NP]  (NP pressure nodes: 4 tet10, 8 hex27)
    const uint32_t* e2bt = nullptr;  // [n_elem][NP][npe]
    const uint32_t* e2c = nullptr;   // [n_elem][NP][NP]
    double* bval = nullptr;
    double* btval = nullptr;
    double* cval = nullptr;
    double* rhs_p = nullptr;  // [n_pres]
    // constant-pressure element (Elem_Solid_3D_Mixed0): element pressures in, and per element the
    // coupling column Kup [n_elem][3 npe], Kpp [n_elem] and FP [n_elem] of the last evaluation out
    const double* pe = nullptr;
    double* kup_e = nullptr;
    double* kpp_e = nullptr;
    double* fp_e = nullptr;
};

// Elem_Solid_3D_Mixed1 element kernel: npe 10 (tet10, 4 vertex pressures) or 27 (hex27, 8
// corner pressures)
void launch_elem_mixed(const MixedElemArgs& a, int npe, int mode, cudaStream_t s);
// hex27 shape tables of the Mixed1 kernel (once per device before its first launch)
void upload_hex27_tables();
// Elem_Solid_3D_Mixed0 (hex8 or tet10, one pressure per element), condensed: the displacement
// element's outputs (Ke/Re export or the scatter of ElemArgs) plus kup_e, kpp_e, fp_e.
void launch_elem_mixed0(const MixedElemArgs& a, int npe, int mode, cudaStream_t s);
// Elem_Solid_3D_Mixed0::solveForPressure for every element: p_e += (FP - Kpu du_e) / Kpp, du the
// node-major solution increment.
void launch_pressure_update_p0(int64_t n_elem, int npe, const int32_t* conn, const double* du, const double* kup_e,
                               const double* kpp_e, const double* fp_e, double* pe, cudaStream_t s, int sm);

}  // namespace mphy
