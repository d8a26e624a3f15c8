// krylov.cuh -- K4/K5: SELL-32 3x3 SpMV, Jacobi-preconditioned CG with PETSc KSPCG semantics,
// and the FP64 vector operations around it.
#pragma once
#include "common.cuh"

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
    uint32_t pad;
};

struct SellView {
    int32_t n_node;
    int32_t n_slices;
    const int64_t* slice_base;
    const int32_t* slice_width;
    const int32_t* col;
    const uint32_t* dvoff;
};

// Grid of a grid-stride kernel over n items with the given block size.
unsigned stride_grid(int64_t n, int threads, int sm_count, int per_sm = 8);

// y = A x (FP64 values and vectors).
void spmv_fp64(const SellView& A, const double* val, const double* x, double* y, cudaStream_t s, int sm);

// Deterministic FP64 dot product of two device vectors; result left in *out_dev.
void dot_fp64(const double* a, const double* b, int64_t n, double* partials, uint32_t* counter, double* out_dev,
              cudaStream_t s, int sm);

// Jacobi-PCG driver, FP64. Holds its work vectors; solve() runs from x = 0.
class PcgFp64 {
  public:
    void init(const SellView& A, int sm_count, int chunk);
    // b: [3*n_node] FP64 (prescribed DOFs zero). x: [3*n_node] output.
    int solve(const double* val, const double* b, double* x, double rtol, double abstol, double dtol, int maxit,
              cudaStream_t s, int32_t* its, double* final_norm);
    ~PcgFp64();
    int64_t launches = 0;  // kernels launched by the last solve()

  private:
    void record_iterations(const double* val, double* x, cudaStream_t s, int n_iter);
    SellView A_{};
    int sm_ = 148, chunk_ = 32;
    int64_t n_ = 0;
    DevBuf<double> r_, z_, p_, q_, dinv_, partials_, partials2_;
    DevBuf<PcgState> st_;
    cudaGraphExec_t graph_ = nullptr;
    const double* graph_val_ = nullptr;
    double* graph_x_ = nullptr;
    cudaStream_t graph_stream_ = nullptr;
};

// small kernels of the solver surface
void set_prescribed_diagonal(const SellView& A, const uint8_t* fixed, double* val, cudaStream_t s, int sm);
void add_scaled_free(const uint8_t* fixed, const double* f, double scale, double* rhs, int64_t n, cudaStream_t s,
                     int sm);
void axpy_inplace(double* y, const double* x, double a, int64_t n, cudaStream_t s, int sm);
void gather_values(const double* val, const int64_t* src, double* out, int64_t n, cudaStream_t s, int sm);
void gather_free(const double* v, const int32_t* assy, double* out, int64_t n_free, cudaStream_t s, int sm);

}  // namespace mphy
