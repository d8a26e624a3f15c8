// common.cuh -- shared internals of libmphy.so: status plumbing, device buffers, handle structs.
#pragma once

#include <atomic>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "../../include/mphy.h"

namespace mphy {

// Last error message of this host thread (mphy_last_error).
void set_error(const std::string& msg);

struct Error {
    int status;
    std::string msg;
};

#define MPHY_CUDA(call)                                                                       \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            throw ::mphy::Error{e_ == cudaErrorMemoryAllocation ? MPHY_ERR_OUT_OF_MEMORY      \
                                                                : MPHY_ERR_CUDA,              \
                                std::string(#call) + ": " + cudaGetErrorString(e_)};          \
    } while (0)

#define MPHY_REQUIRE(cond, status, msg)                                                       \
    do {                                                                                      \
        if (!(cond)) throw ::mphy::Error{(status), (msg)};                                    \
    } while (0)

// Owning device allocation (stream-ordered free is not needed: frees happen at destroy time
// after a synchronize).
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count) {
        release();
        n = count;
        if (count) MPHY_CUDA(cudaMalloc(&p, count * sizeof(T)));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
    void upload(const T* host, size_t count, cudaStream_t s) {
        if (count) MPHY_CUDA(cudaMemcpyAsync(p, host, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void download(T* host, size_t count, cudaStream_t s) const {
        if (count) MPHY_CUDA(cudaMemcpyAsync(host, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    void copy_from(const DevBuf& o, cudaStream_t s) {
        if (n) MPHY_CUDA(cudaMemcpyAsync(p, o.p, (n < o.n ? n : o.n) * sizeof(T), cudaMemcpyDeviceToDevice, s));
    }
};

inline unsigned ceil_div(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace mphy

// ---------------------------------------------------------------------------------------------
// Handle structs (opaque in the C ABI)
// ---------------------------------------------------------------------------------------------
namespace mphy {
// True the first time it is called for the current device with this mask: kernel attributes
// (cudaFuncSetAttribute) are per device, so a process that drives several GPUs sets them on each.
inline bool first_use_on_device(std::atomic<uint64_t>& mask) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return true;
    const uint64_t bit = 1ull << dev;
    return (mask.fetch_or(bit) & bit) == 0;
}
}  // namespace mphy

struct mphy_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

// Device-resident mesh: the SoA replacement of GeomDataLagrange / elems[] / MaterialBase objects.
struct mphy_mesh {
    mphy_ctx* ctx = nullptr;
    int device = 0;  // kept so that destroy never touches the context (it may be gone)
    int32_t n_node = 0, n_elem = 0, npe = 0, n_mat = 0;
    mphy::DevBuf<double> coords;   // [n_node][3]
    mphy::DevBuf<int32_t> conn;    // [n_elem][npe]
    mphy::DevBuf<int32_t> mat_id;  // [n_elem]
    mphy::DevBuf<double> mats;     // [n_mat][4] = mu, Kinv, Utype, 0
    mphy::DevBuf<double> matx;     // [n_mat][8] = model, data0..3, Kinv, Utype, 0
    std::vector<double> matx_host;
    bool general = false;          // some material is not Neo-Hookean: dense-tangent element kernel
    mphy::DevBuf<uint8_t> fixed;   // [n_node*3]
    std::vector<uint8_t> fixed_host;
    // prescribed displacement of every prescribed DOF at time t: t * presc_ramp + presc_const
    // (both [n_node*3]; allocated only once nonzero values are set)
    mphy::DevBuf<double> presc_ramp, presc_const;
    bool has_presc = false;
    std::vector<double> coords_host;  // reference coordinates (aggregation of the coarse space)
};

// Node-block sparsity. Block rows are nodes; a block row holds the nodes that share an element
// with it, ascending. Values live in a sliced-ELL layout of 3x3 blocks ("SELL-32 x 3x3"):
// slice s covers nodes [32s, 32s+32); its width W_s is the longest row in the slice; the value v
// (0..8, row-major in the block) of the k-th block of node n sits at
//     9 * (slice_base[s] + 32 k) + 32 v + (n % 32)
// so that a warp reading one (k, v) over its 32 rows reads 32 consecutive values. Columns sit at
//     slice_base[s] + 32 k + (n % 32).
// Padding blocks (k >= row length) carry column n and zero values.
struct mphy_pattern {
    mphy_ctx* ctx = nullptr;
    const mphy_mesh* mesh = nullptr;
    int device = 0;
    int32_t n_node = 0, n_elem = 0, npe = 0, n_free = 0;
    int64_t n_blocks = 0;       // true blocks (sum of row lengths)
    int64_t sell_blocks = 0;    // stored blocks incl. padding
    int64_t nnz = 0;            // scalar nonzeros over free DOFs (reference CSR)
    int32_t n_slices = 0;
    mphy::DevBuf<int64_t> brow_ptr;    // [n_node+1] compact block CSR
    mphy::DevBuf<int32_t> bcol;        // [n_blocks]
    mphy::DevBuf<int64_t> slice_base;  // [n_slices+1] in blocks
    mphy::DevBuf<int32_t> slice_width; // [n_slices]
    mphy::DevBuf<int32_t> sell_col;    // [sell_blocks]
    mphy::DevBuf<uint32_t> e2v;        // [n_elem][npe][npe] value offset of block (I,J), v = 0
    mphy::DevBuf<uint32_t> dvoff;      // [n_node] value offset of the diagonal block
    mphy::DevBuf<int32_t> node_dof;    // [n_node*3] free id or -1 (NodeDofArray)
    mphy::DevBuf<int32_t> assy_for_soln;  // [n_free]
    mphy::DevBuf<int64_t> csr_rowptr;  // [n_free+1] reference CSR over free DOFs
    mphy::DevBuf<int32_t> csr_col;     // [nnz]
    mphy::DevBuf<int64_t> csr_src;     // [nnz] SELL value offset of each CSR entry
};
