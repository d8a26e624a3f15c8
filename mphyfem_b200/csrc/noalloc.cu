// noalloc.cu -- element evaluation for callers that must not allocate device memory.
//
// Some callers cannot let a library call cudaMalloc: a finite-element code that already holds
// its mesh in device memory under its own arena allocator (every byte of the device is
// reserved up front, so an allocation behind its back can fail or fragment the arena), or a
// host application under a no-allocation policy in its time-stepping loop. mphy_elem_eval needs
// a mesh handle (which copies the mesh) and a small per-call scratch buffer for the
// first-bad-element flag; mphy_elem_eval_noalloc takes the caller's device arrays directly and
// keeps its scratch -- the flag, a validation flag and the material table widened to the
// kernel's 4-double rows -- in one file-scope __device__ array.
//
// That array (kNoAllocMaxMaterials materials, about 32 KB) is part of the library image: every
// GPU that loads libmphy.so holds it until the process exits. All calls share it and it keeps
// the last call's contents, so each call resets the flags it relies on; calls that overlap on
// the GPU (other streams, other host threads) race on it and must be serialised by the caller.
// The first call on a device looks up the array's device address (cudaGetSymbolAddress). Every
// call runs on the context's stream and blocks the calling host thread until its result is
// ready: it synchronises that stream twice, once after the input checks and once to read the
// first-bad-element flag.
#include <climits>
#include <mutex>

#include "common.cuh"
#include "elem.cuh"

namespace mphy {
namespace {

constexpr int kNoAllocMaxMaterials = 1024;
constexpr int kNoAllocMaxDevices = 64;

struct NoAllocScratch {
    unsigned long long first_bad;   // lowest element id with det F < 0 (reset to ULLONG_MAX)
    int32_t invalid;                // 1: a connectivity or material id is out of range (reset to 0)
    int32_t pad[61];
    double mats[kNoAllocMaxMaterials][4];  // mu, Kinv, Utype, unused
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

std::mutex g_setup_mu;
NoAllocScratch* g_scratch_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device. Host code only sees a host-side
// stand-in under the array's name, so the address is looked up once per device, with that
// device current.
NoAllocScratch* scratch_for_device(int device) {
    MPHY_REQUIRE(device >= 0 && device < kNoAllocMaxDevices, MPHY_ERR_UNSUPPORTED, "device id too large");
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[device]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        MPHY_REQUIRE(e == cudaSuccess, MPHY_ERR_CUDA,
                     std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
        g_scratch_ptr[device] = static_cast<NoAllocScratch*>(ptr);
    }
    return g_scratch_ptr[device];
}

// Checks the kernel itself does not make, the same ones mphy_mesh_create makes on the host:
// connectivity within [0, n_node), material ids within [0, n_mat), every material row's Kinv
// (column 1 of the [n_mat][3] table) positive.
__global__ void validate_ids(int64_t n_conn, const int32_t* __restrict__ conn, int32_t n_node, int32_t n_elem,
                             const int32_t* __restrict__ mat_id, int32_t n_mat, const double* __restrict__ mats,
                             int32_t* invalid) {
    const int64_t n = n_conn > n_mat ? n_conn : n_mat;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < n_conn && (conn[i] < 0 || conn[i] >= n_node)) *invalid = 1;
        if (i < n_elem && (mat_id[i] < 0 || mat_id[i] >= n_mat)) *invalid = 1;
        if (i < n_mat && !(mats[3 * i + 1] > 0.0)) *invalid = 1;
    }
}

}  // namespace
}  // namespace mphy

using namespace mphy;

extern "C" int mphy_elem_eval_noalloc(mphy_ctx* c, int32_t n_node, const double* coords_dev, int32_t n_elem,
                                      int32_t npe, const int32_t* conn_dev, const int32_t* mat_id_dev, int32_t n_mat,
                                      const double* mats_dev, const double* disp_dev, int32_t tangent, double* Ke_dev,
                                      double* Re_dev, int64_t* first_bad) {
    try {
        MPHY_REQUIRE(c && coords_dev && conn_dev && mat_id_dev && mats_dev && disp_dev && Ke_dev && Re_dev,
                     MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(npe == 8 || npe == 10, MPHY_ERR_UNSUPPORTED, "npe must be 8 (hex8) or 10 (tet10)");
        MPHY_REQUIRE(n_node > 0 && n_elem >= 0, MPHY_ERR_INVALID_ARG, "invalid mesh size");
        MPHY_REQUIRE(n_mat >= 1 && n_mat <= kNoAllocMaxMaterials, MPHY_ERR_INVALID_ARG,
                     "n_mat must be in [1, 1024]: the allocation-free scratch holds at most 1024 materials");
        MPHY_CUDA(cudaSetDevice(c->device));
        NoAllocScratch* ptr = scratch_for_device(c->device);
        cudaStream_t s = c->stream;
        // reset the flags this call reads; stage the [n_mat][3] table into 4-double rows
        MPHY_CUDA(cudaMemsetAsync(&ptr->first_bad, 0xff, sizeof(unsigned long long), s));
        MPHY_CUDA(cudaMemsetAsync(&ptr->invalid, 0, sizeof(int32_t), s));
        MPHY_CUDA(cudaMemcpy2DAsync(ptr->mats, 4 * sizeof(double), mats_dev, 3 * sizeof(double), 3 * sizeof(double),
                                    n_mat, cudaMemcpyDeviceToDevice, s));
        {
            const int64_t n_conn = (int64_t)n_elem * npe;
            unsigned grid = ceil_div(n_conn > n_mat ? n_conn : (int64_t)n_mat, 256);
            if (grid > (unsigned)c->sm_count * 8) grid = c->sm_count * 8;
            validate_ids<<<grid, 256, 0, s>>>(n_conn, conn_dev, n_node, n_elem, mat_id_dev, n_mat, mats_dev,
                                              &ptr->invalid);
            MPHY_CUDA(cudaGetLastError());
            int32_t invalid = 0;
            MPHY_CUDA(cudaMemcpyAsync(&invalid, &ptr->invalid, sizeof(invalid), cudaMemcpyDeviceToHost, s));
            MPHY_CUDA(cudaStreamSynchronize(s));
            MPHY_REQUIRE(invalid == 0, MPHY_ERR_INVALID_ARG,
                         "connectivity or material id out of range, or a material row with Kinv <= 0");
        }
        if (n_elem > 0) {
            ElemArgs a{};
            a.n_elem = n_elem;
            a.coords = coords_dev;
            a.conn = conn_dev;
            a.mat_id = mat_id_dev;
            a.mats = &ptr->mats[0][0];
            a.disp = disp_dev;
            a.tangent = tangent;
            a.bad = &ptr->first_bad;
            a.Ke = Ke_dev;
            a.Re = Re_dev;
            launch_elem_fp64(a, npe, 1, s);
        }
        unsigned long long h = ULLONG_MAX;
        MPHY_CUDA(cudaMemcpyAsync(&h, &ptr->first_bad, sizeof(h), cudaMemcpyDeviceToHost, s));
        MPHY_CUDA(cudaStreamSynchronize(s));
        const int64_t b = h == ULLONG_MAX ? -1 : (int64_t)h;
        if (first_bad) *first_bad = b;
        if (b >= 0) {
            set_error("negative Jacobian in element " + std::to_string(b));
            return MPHY_ERR_NEG_JACOBIAN;
        }
        return MPHY_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.status;
    }
}
