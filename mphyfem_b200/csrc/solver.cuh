// solver.cuh -- the solver handle behind mphy_solver_* and the internals shared by the
// single-problem driver (api.cu) and the batched driver (batch.cu).
#pragma once
#include <new>

#include "coarse.cuh"
#include "common.cuh"
#include "elem.cuh"
#include "fsai.cuh"
#include "gnn.cuh"
#include "krylov.cuh"

namespace mphy {

template <typename F>
int guarded(F&& f) {
    try {
        return f();
    } catch (const Error& e) {
        set_error(e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return MPHY_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_error(e.what());
        return MPHY_ERR_CUDA;
    }
}

}  // namespace mphy

// ------------------------------------------------------------------------------- solver struct
// (global-scope handle types of the C ABI; their members use the mphy internals)
using namespace mphy;

struct mphy_solver {
    mphy_ctx* ctx = nullptr;
    int device = 0;
    const mphy_mesh* mesh = nullptr;
    mphy_pattern* pat = nullptr;
    mphy_solver_opts opts{};
    int state = MPHY_SOLVER_EMPTY;
    int64_t launches = 0;  // libmphy kernels launched (running count)
    SellView A{};
    bool mixed = false;          // MPHY_PREC_MIXED: FP32 values + FP64 iterative refinement
    DevBuf<double> val;          // SELL values, FP64 (plain method)
    DevBuf<float> valf;          // SELL values, FP32 (mixed precision): off-diagonal blocks, unmasked
    DevBuf<double> diag64;       // [n_node][9] FP64 diagonal blocks = -sum of the stored off-diagonals
    DevBuf<double> rhs, reac, x; // [3*n_node]
    DevBuf<unsigned long long> bad;
    DevBuf<double> partials, scalar;
    DevBuf<uint32_t> counter;
    DevBuf<double> disp_tmp, fext_tmp, disp_prev;
    DevBuf<double> disp_prev2, du_full, x_first, arc_dots;  // arc-length continuation
    DevBuf<double> ref_r, ref_d;          // FP64 refinement sweeps (max_outer > 1), true residual
    DevBuf<float> pred_blocks;            // network-predicted G blocks (learned FSAI)
    DevBuf<PcgState> dot_st;              // mphy_solver_spmv_dot scratch
    DevBuf<double> dot_part;
    PcgFp64 pcg;
    IterativeRefinement<double> ir;       // MIXED
    IterativeRefinement<float> ir32;      // MIXED_F32VEC
    Fsai fsai;                            // MPHY_PC_FSAI*
    CoarseSpace coarse;                   // coarse_aggregates > 0
    bool coarse_ready = false;            // coarse holds an operator formed by an earlier solve
    int coarse_age = 0;                   // solves since it was formed (coarse_lag)
    mphy_gnn* gnn = nullptr;              // MPHY_PC_FSAI_LEARNED: network run before every solve
    int32_t last_fallback = 0;            // the last solve fell back to Jacobi
    int32_t first_status = 0, first_its = 0;  // the learned attempt of the last solve
    double first_relres = 0.0;
    GnnGraph graph;
    bool use_coarse = false;
    bool use_fsai = false;
    double t_pc_ms = 0.0;                 // last preconditioner setup time
    int32_t last_sweeps = 0;
    double* pinned = nullptr;  // [0] norm, [1] bad as bits
    // constant-pressure mixed element (Elem_Solid_3D_Mixed0): element pressures (current and at
    // the last converged step) and the coupling terms of the last assembly
    bool p0 = false;
    DevBuf<double> pe, pe_prev, kup_e, kpp_e, fp_e;
    DevBuf<double> lift;  // [3 n_node] prescribed increments of the current load step
};

struct mphy_gnn {
    mphy_ctx* ctx = nullptr;
    int device = 0;
    Gnn net;
};

namespace mphy {
// Zero K and R, element kernel with scatter into the SELL values (femSolidmechanics2.cpp:1047-1120).
// bad_elem: optional per-element det F < 0 flags (zeroed by the caller).
void solver_assemble(mphy_solver* s, const double* disp, uint8_t* bad_elem = nullptr, const double* lift = nullptr);
// ||rhs|| and the first bad element (-1 if none), one synchronisation.
double solver_norm_and_bad(mphy_solver* s, int64_t* first_bad);
// disp += solution, and for the constant-pressure element the element pressures' update
// (factoriseSolveAndUpdate, femSolidmechanics2.cpp:1183-1212).
void solver_update(mphy_solver* s, double* disp);
}  // namespace mphy
