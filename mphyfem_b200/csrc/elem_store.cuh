// elem_store.cuh -- the element kernels' output stage: export of Ke/Re, or the scatter-add into
// the SELL matrix, the right-hand side and the reactions (MatSetValue / VecSetValue with
// ADD_VALUES, SolverPetsc.cpp:357-378).
#pragma once
#include "elem.cuh"

namespace mphy {

// Row node I of element e: residual R (3 values). MODE bit 1 exports it to Re; bit 2 adds it to
// the reactions (every DOF) and to the right-hand side (free DOFs).
template <int NPE, int MODE>
__device__ __forceinline__ void store_residual(const ElemArgs& a, int64_t e, int I, int32_t node, const bool freeI[3],
                                               const double R[3]) {
    constexpr int NS = 3 * NPE;
    if (MODE & 1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) a.Re[e * NS + 3 * I + c] = R[c];
    }
    if (MODE & 2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (a.reac) atomicAdd(&a.reac[3 * (int64_t)node + c], R[c]);
            if (freeI[c]) atomicAdd(&a.rhs[3 * (int64_t)node + c], R[c]);
        }
    }
}

// Block (I, J) of element e, acc row-major 3x3. MODE bit 1 exports it to Ke; bit 2 adds it to the
// matrix: FP64 values with prescribed rows and columns skipped, or (a.valf) FP32 off-diagonal
// blocks unmasked, the diagonal being rebuilt from them after assembly.
template <int NPE, int MODE>
__device__ __forceinline__ void store_block(const ElemArgs& a, int64_t e, int I, int J, int32_t node,
                                            const bool freeI[3], const double acc[9]) {
    constexpr int NS = 3 * NPE;
    if (MODE & 1) {
#pragma unroll
        for (int aa = 0; aa < 3; ++aa)
#pragma unroll
            for (int bb = 0; bb < 3; ++bb) a.Ke[(e * NS + 3 * I + aa) * NS + 3 * J + bb] = acc[3 * aa + bb];
    }
    if (MODE & 2) {
        const int32_t nJ = a.conn[e * NPE + J];
        const uint32_t off = a.e2v[(e * NPE + I) * NPE + J];
        if (a.valf) {
            if (nJ != node) {
#pragma unroll
                for (int v = 0; v < 9; ++v) atomicAdd(&a.valf[off + 32u * v], (float)acc[v]);
            }
        } else {
#pragma unroll
            for (int bb = 0; bb < 3; ++bb) {
                if (a.fixed[3 * (int64_t)nJ + bb]) continue;
#pragma unroll
                for (int aa = 0; aa < 3; ++aa)
                    if (freeI[aa]) atomicAdd(&a.val[off + 32u * (3 * aa + bb)], acc[3 * aa + bb]);
            }
        }
    }
}

// Lift of prescribed displacement increments, ElementBase::applyDirichletBCs
// (ElementBase.cpp:567-594), applied in the first Newton iteration of a step
// (femSolidmechanics2.cpp:1080-1095): the free rows of element e get -sum_J K_IJ lift_J. Block
// (I, J) adds K_IJ lift_J to the row node's accumulator rl (K as formed, before any masking).
template <int NPE, int MODE>
__device__ __forceinline__ void lift_block(const ElemArgs& a, int64_t e, int J, const double acc[9], double rl[3]) {
    if (!(MODE & 2) || !a.lift) return;
    const int64_t nJ = a.conn[e * NPE + J];
    const double l0 = a.lift[3 * nJ], l1 = a.lift[3 * nJ + 1], l2 = a.lift[3 * nJ + 2];
#pragma unroll
    for (int aa = 0; aa < 3; ++aa) rl[aa] += acc[3 * aa] * l0 + acc[3 * aa + 1] * l1 + acc[3 * aa + 2] * l2;
}

// The accumulated lift of row node I into the right-hand side and the reactions (free DOFs: the
// reference's reaction sum takes the element vector after the lift).
template <int NPE, int MODE>
__device__ __forceinline__ void store_lift(const ElemArgs& a, int32_t node, const bool freeI[3], const double rl[3]) {
    if (!(MODE & 2) || !a.lift) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (!freeI[c] || rl[c] == 0.0) continue;
        atomicAdd(&a.rhs[3 * (int64_t)node + c], -rl[c]);
        if (a.reac) atomicAdd(&a.reac[3 * (int64_t)node + c], -rl[c]);
    }
}

}  // namespace mphy
