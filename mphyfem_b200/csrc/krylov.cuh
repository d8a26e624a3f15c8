// krylov.cuh -- K4/K5: SELL-32 3x3 SpMV, preconditioned CG with PETSc KSPCG semantics (FP64, or
// FP32 vectors with FP64 reductions), FP64 iterative refinement, and the vector operations.
#pragma once
#include <type_traits>
#include <cuda_bf16.h>

#include "common.cuh"

#include "coarse_view.cuh"

namespace mphy {

// Device-side CG state. Written only by the last CTA of a kernel (after every CTA has
// finished its part), read by the following kernels: no spin-waits anywhere.
struct PcgState {
    double rz;     // (r, z)
    double alpha;
    double beta;
    double dp;     // ||z|| (KSP_NORM_PRECONDITIONED)
    double dp0;
    double ttol;   // max(rtol * dp0, abstol)
    double dtol;
    double pq;
    int32_t its;
    int32_t done;
    int32_t status;  // mphy_status of the solve
    int32_t maxit;
    uint32_t counter;  // last-CTA detection, reset by the last CTA
    int32_t norm_type; // 0: ||z|| (KSP_NORM_PRECONDITIONED), 1: ||r|| (KSP_NORM_UNPRECONDITIONED)
    // two-level iteration with ||r||: (r, D^-1 r) and (r, r) from the update, completed by the
    // coarse GEMV with (Z^T r, c), c = E^-1 Z^T r, into (r, z) (z itself is not formed)
    double rdr;
    double rr;
};

struct SellView {
    int32_t n_node;
    int32_t n_slices;
    const int64_t* slice_base;
    const int32_t* slice_width;
    const int32_t* col;
    const uint32_t* dvoff;
    // Null-space-preserving storage (mixed precision): when diag64 is set, the stored diagonal
    // blocks are zero and block row n adds diag64[n] (FP64, [9]) times x_n; when fixed is set,
    // prescribed DOFs are identity rows (the stored rows and columns are unmasked).
    const double* diag64 = nullptr;
    const uint8_t* fixed = nullptr;
};

// Factorised preconditioner M = G^T G: G lower block-triangular and G^T, both in SELL layout.
// The factor is stored in BF16: M = G^T G is symmetric positive definite for every nonsingular
// G, so rounding G changes the preconditioner's quality by its 2^-9 relative error, never its
// validity, and the two factor SpMVs of every iteration stream half the bytes of FP32.
using FactorT = __nv_bfloat16;
template <typename VT>
struct FactorView {
    SellView G, GT;
    const VT* gval;
    const VT* gtval;
};

// Grid of a grid-stride kernel over n items with the given block size.
unsigned stride_grid(int64_t n, int threads, int sm_count, int per_sm = 8);
// The same, capped at the CTAs the SMs hold at once for `kernel` (occupancy query, cached).
unsigned resident_grid(const void* kernel, int64_t n, int threads, int sm_count);

// y = A x.
template <typename VT, typename XT>
void spmv(const SellView& A, const VT* val, const XT* x, XT* y, cudaStream_t s, int sm);
// y = A x and st->pq = (x, y) in one pass: the SpMV kernel of the CG iteration, on a scratch
// state (zeroed first) and a partials buffer of at least 8 entries per SM
template <typename VT, typename XT>
void spmv_dot(const SellView& A, const VT* val, const XT* x, XT* y, double* partials, PcgState* st, cudaStream_t s,
              int sm);

// r = b - A x in FP64 (A in VT), and ||r||^2 into *out_dev; partials [sm*8+8], counter zeroed.
template <typename VT>
void residual_fp64(const SellView& A, const VT* val, const double* x, const double* b, double* r, double* partials,
                   uint32_t* counter, double* out_dev, cudaStream_t s, int sm);

// Deterministic FP64 dot product of two device vectors; result left in *out_dev.
void dot_fp64(const double* a, const double* b, int64_t n, double* partials, uint32_t* counter, double* out_dev,
              cudaStream_t s, int sm);

enum class PcKind { Jacobi, Factor, JacobiCoarse, FactorCoarse };

// Preconditioned CG, VT = matrix values, XT = vector precision (double, or float with FP64
// reductions). solve() runs from x = 0 on b (XT), PETSc KSPCG semantics.
template <typename VT, typename XT>
class Pcg {
  public:
    void init(const SellView& A, int sm_count, int chunk);
    void set_factor(const FactorView<FactorT>& f) { factor_ = f; kind_ = PcKind::Factor; }
    void set_jacobi() { kind_ = PcKind::Jacobi; }
    // the coarse correction adds to the current local part (Jacobi or G^T G)
    void set_coarse(const CoarseView& c) {
        coarse_ = c;
        kind_ = kind_ == PcKind::Factor ? PcKind::FactorCoarse : PcKind::JacobiCoarse;
    }
    int solve(const VT* val, const XT* b, XT* x, double rtol, double abstol, double dtol, int maxit, cudaStream_t s,
              int32_t* its, double* final_norm);
    ~Pcg();
    int norm_type = 0;  // KSP norm type of the convergence test (see PcgState)
    int64_t launches = 0;  // kernels launched by the last solve()

  private:
    void record_iterations(const VT* val, XT* x, cudaStream_t s, int n_iter);
    SellView A_{};
    PcKind kind_ = PcKind::Jacobi;
    FactorView<FactorT> factor_{};
    CoarseView coarse_{};
    int sm_ = 148, chunk_ = 32;
    int64_t n_ = 0;
    DevBuf<XT> r_, z_, p_, q_, t_, dinv_;
    DevBuf<float> dinv32_;  // D^-1 of the two-level (Jacobi + coarse) iteration
    DevBuf<double> partials_, partials2_;
    DevBuf<PcgState> st_;
    cudaGraphExec_t graph_ = nullptr;
    const void* graph_val_ = nullptr;
    void* graph_x_ = nullptr;
    cudaStream_t graph_stream_ = nullptr;
    PcKind graph_kind_ = PcKind::Jacobi;
    int graph_norm_ = -1;
};

using PcgFp64 = Pcg<double, double>;

// FP64 iterative refinement around a PCG on the FP32-stored operator A32:
//   x = 0, r = b; repeat { d = PCG(A32, r, inner_rtol); x += d; r = b - A32 x (FP64) }
// until ||r|| <= rtol ||b|| or max_outer sweeps. XT is the inner Krylov vector precision:
// double (FP32 values, FP64 vectors and reductions) or float (FP32 vectors, FP64 reductions).
// x: FP64 output. Returns an mphy_status.
template <typename XT>
class IterativeRefinement {
  public:
    void init(const SellView& A, int sm_count, int chunk);
    Pcg<float, XT>& inner() { return inner_; }
    int solve(const float* val, const double* b, double* x, double rtol, double inner_rtol, int max_outer, int maxit,
              cudaStream_t s, int32_t* its, int32_t* sweeps, double* relres);
    int64_t launches = 0;

  private:
    SellView A_{};
    int sm_ = 148;
    int64_t n_ = 0;
    Pcg<float, XT> inner_;
    DevBuf<double> r64_, rold_, partials_, partials2_, scalars_;
    DevBuf<XT> rin_, d_;
    DevBuf<uint32_t> counter_;
};

// D_n = -sum_{m != n} A_nm over the stored FP32 blocks (the stored diagonal blocks are zero):
// the diagonal that makes the stored operator exactly translation invariant.
void diag_from_offdiag(const SellView& A, const float* val, double* diag64, cudaStream_t s, int sm);
// CSR export fix-up for that storage: entries of diagonal blocks come from diag64.
void export_fix_diagonal(const double* diag64, const int64_t* rowptr, const int32_t* col, const int32_t* assy,
                         int32_t n_free, double* out, cudaStream_t s, int sm);

// z_u += Z E^{-1} Z^T r_u: the coarse correction of a set-up coarse space added to z over the
// first 3 n_node entries (restriction, coarse solve, prolongation; FP64).
void coarse_apply_add(const CoarseView& cv, int32_t n_node, const double* r, double* z, cudaStream_t s, int sm);

// small kernels of the solver surface
template <typename VT>
void set_prescribed_diagonal(const SellView& A, const uint8_t* fixed, VT* val, cudaStream_t s, int sm);
void add_scaled_free(const uint8_t* fixed, const double* f, double scale, double* rhs, int64_t n, cudaStream_t s,
                     int sm);
// dispApplied of a load step: lift = t ramp + cst - disp on prescribed DOFs, zero on free ones
void prescribed_increment(const uint8_t* fixed, const double* ramp, const double* cst, double t, const double* disp,
                          double* lift, int64_t n, cudaStream_t s, int sm);
void axpy_inplace(double* y, const double* x, double a, int64_t n, cudaStream_t s, int sm);
template <typename VT>
void gather_values(const VT* val, const int64_t* src, double* out, int64_t n, cudaStream_t s, int sm);
void gather_free(const double* v, const int32_t* assy, double* out, int64_t n_free, cudaStream_t s, int sm);

// The FP32 storage keeps no diagonal blocks: the operator's diagonal block of a row is minus the
// FP64 sum of the row's stored FP32 blocks, in storage order (k = 0 .. width-1), which makes the
// stored operator map rigid translations exactly to zero. Every kernel that applies the operator
// forms that sum while it streams the row (RowSum), with each value widened once. The FP64
// storage has its diagonal blocks in the rows (RowSum<double> does nothing).
template <typename VT>
constexpr bool kOffDiagStorage = std::is_same<VT, float>::value;

template <typename VT>
struct RowSum {
    template <typename T>
    __device__ __forceinline__ void add(const T*) {}
    template <typename V>
    __device__ __forceinline__ bool on(const V&) const { return false; }
    __device__ __forceinline__ double d(int) const { return 0.0; }
};
template <>
struct RowSum<float> {
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    template <typename T>
    __device__ __forceinline__ void add(const T* b) {
#pragma unroll
        for (int q = 0; q < 9; ++q) acc[q] += (double)b[q];
    }
    template <typename V>
    __device__ __forceinline__ bool on(const V& A) const { return A.diag64 != nullptr; }
    __device__ __forceinline__ double d(int q) const { return -acc[q]; }
};

}  // namespace mphy
