// api.cu -- the C ABI of libmphy.so and the host-side objects behind it.
//
// The host side mirrors the reference's interfaces: mphy_solver is the SolverPetsc surface
// (initialise / zeroMtx / assembleMatrixAndVector / factoriseAndSolve with its status machine,
// SolverPetsc.h:16-96, SolverEigen.h:11), and the Newton driver follows
// femSolidmechanics::solveWithNewtonRaphson (femSolidmechanics2.cpp:730-851). Every failure is
// a status code plus a thread-local message; nothing throws across the ABI.
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>

#include "common.cuh"
#include "coarse.cuh"
#include "elem.cuh"
#include "fsai.cuh"
#include "gnn.cuh"
#include "mat.cuh"
#include "krylov.cuh"
#include "pattern.cuh"
#include "solver.cuh"
#include "mixed.cuh"

namespace mphy {

thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

std::mutex g_tables_mu;
bool g_tables_done[64] = {false};

}  // namespace mphy

using namespace mphy;

namespace mphy {

void solver_zero(mphy_solver* s) {
    cudaStream_t st = s->ctx->stream;
    if (s->mixed) {
        MPHY_CUDA(cudaMemsetAsync(s->valf.p, 0, s->valf.bytes(), st));
        MPHY_CUDA(cudaMemsetAsync(s->diag64.p, 0, s->diag64.bytes(), st));
    } else {
        MPHY_CUDA(cudaMemsetAsync(s->val.p, 0, s->val.bytes(), st));
        set_prescribed_diagonal<double>(s->A, s->mesh->fixed.p, s->val.p, st, s->ctx->sm_count);
    }
    s->launches += 1;
    MPHY_CUDA(cudaMemsetAsync(s->rhs.p, 0, s->rhs.bytes(), st));
    MPHY_CUDA(cudaMemsetAsync(s->reac.p, 0, s->reac.bytes(), st));
    MPHY_CUDA(cudaMemsetAsync(s->bad.p, 0xff, sizeof(unsigned long long), st));
}

ElemArgs elem_args(const mphy_mesh* m, const double* disp, int tangent, unsigned long long* bad) {
    ElemArgs a{};
    a.n_elem = m->n_elem;
    a.coords = m->coords.p;
    a.conn = m->conn.p;
    a.mat_id = m->mat_id.p;
    a.mats = m->mats.p;
    a.matx = m->matx.p;
    a.disp = disp;
    a.tangent = tangent;
    a.bad = bad;
    a.fixed = m->fixed.p;
    return a;
}

void solver_assemble(mphy_solver* s, const double* disp, uint8_t* bad_elem, const double* lift) {
    solver_zero(s);
    ElemArgs a = elem_args(s->mesh, disp, s->opts.tangent, s->bad.p);
    a.bad_elem = bad_elem;
    a.lift = lift;
    a.e2v = s->pat->e2v.p;
    a.val = s->val.p;
    a.valf = s->mixed ? s->valf.p : nullptr;
    a.rhs = s->rhs.p;
    a.reac = s->reac.p;
    const bool f32_tangent = s->mixed && !s->p0 && !s->mesh->general && s->opts.precision != MPHY_PREC_MIXED_TC;
    if (s->p0) {
        MixedElemArgs ma{};
        ma.base = a;
        ma.disp_prev = s->disp_prev.p;
        ma.pe = s->pe.p;
        ma.kup_e = s->kup_e.p;
        ma.kpp_e = s->kpp_e.p;
        ma.fp_e = s->fp_e.p;
        launch_elem_mixed0(ma, s->mesh->npe, 2, s->ctx->stream);
    } else if (s->mesh->general) launch_elem_gen(a, s->mesh->npe, 2, s->ctx->stream);
    else if (s->opts.precision == MPHY_PREC_MIXED_TC) launch_elem_tc(a, s->mesh->npe, 2, s->ctx->stream);
    else if (f32_tangent) {
        // FP32 tangent blocks; the element kernel also sums the element diagonal blocks that the
        // preconditioners read (the operator forms its own diagonal from the stored rows)
        a.diag_out = s->diag64.p;
        a.diag_full = s->opts.pc_type != MPHY_PC_JACOBI;  // FSAI and the network read whole blocks
        launch_elem_f32(a, s->mesh->npe, s->ctx->stream);
    } else launch_elem_fp64(a, s->mesh->npe, 2, s->ctx->stream);
    s->launches += 1;
    if (s->mixed && !f32_tangent) {
        diag_from_offdiag(s->A, s->valf.p, s->diag64.p, s->ctx->stream, s->ctx->sm_count);
        s->launches += 1;
    }
    s->state = MPHY_ASSEMBLY_OK;
}

void solver_update(mphy_solver* s, double* disp) {
    mphy_ctx* c = s->ctx;
    axpy_inplace(disp, s->x.p, 1.0, 3 * (int64_t)s->mesh->n_node, c->stream, c->sm_count);
    s->launches += 1;
    if (s->p0) {
        launch_pressure_update_p0(s->mesh->n_elem, s->mesh->npe, s->mesh->conn.p, s->x.p, s->kup_e.p, s->kpp_e.p,
                                  s->fp_e.p, s->pe.p, c->stream, c->sm_count);
        s->launches += 1;
    }
}

// ||rhs|| and the first bad element, one synchronisation
double solver_norm_and_bad(mphy_solver* s, int64_t* first_bad) {
    cudaStream_t st = s->ctx->stream;
    const int64_t n = 3 * (int64_t)s->mesh->n_node;
    dot_fp64(s->rhs.p, s->rhs.p, n, s->partials.p, s->counter.p, s->scalar.p, st, s->ctx->sm_count);
    s->launches += 1;
    MPHY_CUDA(cudaMemcpyAsync(&s->pinned[0], s->scalar.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    MPHY_CUDA(cudaMemcpyAsync(&s->pinned[1], s->bad.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    MPHY_CUDA(cudaStreamSynchronize(st));
    unsigned long long b;
    std::memcpy(&b, &s->pinned[1], sizeof(b));
    if (first_bad) *first_bad = b == ULLONG_MAX ? -1 : (int64_t)b;
    return std::sqrt(s->pinned[0]);
}

}  // namespace mphy

namespace {

int solver_solve_once(mphy_solver* s, int32_t* its, double* fnorm);
double true_relres(mphy_solver* s);

// A learned preconditioner is checked by the FP64 true residual: a failed or useless solve is
// repeated with the Jacobi local part (the coarse correction, if any, kept).
int solver_solve(mphy_solver* s, int32_t* its, double* fnorm) {
    s->last_fallback = 0;
    const int rc = solver_solve_once(s, its, fnorm);
    if (!(s->use_fsai && s->opts.pc_type == MPHY_PC_FSAI_LEARNED)) return rc;
    const double rel = true_relres(s);
    s->first_status = rc;
    s->first_its = its ? *its : 0;
    s->first_relres = rel;
    // 100 rtol: room for the drift of the recurrence residual from the true one on stiff
    // operators; a poor prediction shows up as divergence or an order-of-magnitude miss.
    if (rc == MPHY_OK && rel == rel && rel <= 100.0 * s->opts.rtol) return rc;
    s->last_fallback = 1;
    auto local_jacobi = [&](auto& pcg) {
        pcg.set_jacobi();
        if (s->use_coarse) pcg.set_coarse(s->coarse.view());
    };
    auto local_factor = [&](auto& pcg) {
        pcg.set_factor(s->fsai.view());
        if (s->use_coarse) pcg.set_coarse(s->coarse.view());
    };
    if (s->opts.precision == MPHY_PREC_MIXED || s->opts.precision == MPHY_PREC_MIXED_TC) local_jacobi(s->ir.inner());
    else if (s->opts.precision == MPHY_PREC_MIXED_F32VEC) local_jacobi(s->ir32.inner());
    else local_jacobi(s->pcg);
    int32_t its2 = 0;
    const int rc2 = solver_solve_once(s, &its2, fnorm);
    if (its) *its += its2;
    if (s->opts.precision == MPHY_PREC_MIXED || s->opts.precision == MPHY_PREC_MIXED_TC) local_factor(s->ir.inner());
    else if (s->opts.precision == MPHY_PREC_MIXED_F32VEC) local_factor(s->ir32.inner());
    else local_factor(s->pcg);
    return rc2;
}

int solver_solve_once(mphy_solver* s, int32_t* its, double* fnorm) {
    MPHY_REQUIRE(s->state == MPHY_ASSEMBLY_OK || s->state == MPHY_FACTORISE_OK, MPHY_ERR_STATE,
                 "factoriseAndSolve: assemble matrix first");
    // The preconditioner follows the operator (KSPSetReusePreconditioner false): it is built by
    // the first solve after an assembly and reused by further solves with the same matrix
    // (PETSc's PCSetUp runs only when the operator has changed).
    const bool setup = s->state == MPHY_ASSEMBLY_OK;
    s->state = MPHY_FACTORISE_OK;
    if (setup && s->use_fsai && s->opts.pc_type == MPHY_PC_FSAI) {
        // the preconditioner follows the operator: rebuilt for every solve (KSPSetReusePreconditioner false)
        MPHY_CUDA(cudaEventRecord(s->ctx->ev0, s->ctx->stream));
        if (s->mixed) s->fsai.compute<float>(s->valf.p, s->diag64.p, s->mesh->fixed.p, s->ctx->stream);
        else s->fsai.compute<double>(s->val.p, nullptr, nullptr, s->ctx->stream);
        MPHY_CUDA(cudaEventRecord(s->ctx->ev1, s->ctx->stream));
        MPHY_CUDA(cudaEventSynchronize(s->ctx->ev1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, s->ctx->ev0, s->ctx->ev1);
        s->t_pc_ms = ms;
        s->launches += s->fsai.launches;
    }
    if (setup && s->use_fsai && s->opts.pc_type == MPHY_PC_FSAI_LEARNED && s->gnn) {
        float ms = 0.f;
        const int rc = mphy_gnn_predict(s->gnn, s, &ms);
        MPHY_REQUIRE(rc == MPHY_OK, rc, "learned preconditioner: prediction failed");
        s->t_pc_ms = ms;
    }
    if (setup && s->use_coarse) {
        // the coarse operator follows the assembled matrix, unless a lag is asked for and the
        // kept one is young enough
        if (s->coarse_ready && s->opts.coarse_lag > 0 && s->coarse_age < s->opts.coarse_lag) {
            ++s->coarse_age;
            s->coarse.last_setup_ms = 0.f;  // this solve formed nothing
        } else {
            if (s->mixed) s->coarse.setup<float>(s->A, s->valf.p, nullptr, s->ctx->stream);
            else s->coarse.setup<double>(s->A, s->val.p, nullptr, s->ctx->stream);
            s->launches += s->coarse.launches;
            s->coarse_ready = true;
            s->coarse_age = 0;
        }
    }
    if (s->mixed) {
        // FP32 inner PCG inside an FP64 refinement loop; *fnorm is ||b - A x|| / ||b|| in FP64
        if (s->opts.precision == MPHY_PREC_MIXED_F32VEC) {
            const int rc = s->ir32.solve(s->valf.p, s->rhs.p, s->x.p, s->opts.rtol, s->opts.inner_rtol,
                                         s->opts.max_outer, s->opts.max_it, s->ctx->stream, its, &s->last_sweeps,
                                         fnorm);
            s->launches += s->ir32.launches;
            return rc;
        }
        const int rc = s->ir.solve(s->valf.p, s->rhs.p, s->x.p, s->opts.rtol, s->opts.inner_rtol, s->opts.max_outer,
                                   s->opts.max_it, s->ctx->stream, its, &s->last_sweeps, fnorm);
        s->launches += s->ir.launches;
        return rc;
    }
    int rc = s->pcg.solve(s->val.p, s->rhs.p, s->x.p, s->opts.rtol, s->opts.abstol, s->opts.dtol,
                          s->opts.max_it, s->ctx->stream, its, fnorm);
    s->launches += s->pcg.launches;
    s->last_sweeps = 1;
    if (s->opts.max_outer <= 1 || rc == MPHY_ERR_INDEFINITE || rc == MPHY_ERR_DIVERGED) return rc;
    // FP64 refinement sweeps: the recurrence residual of a long CG run drifts away from b - A x;
    // x += PCG(A, b - A x) until the FP64 true residual meets rtol (the same loop as the mixed
    // path, on the FP64 operator)
    cudaStream_t st = s->ctx->stream;
    const int sm = s->ctx->sm_count;
    const int64_t n = 3 * (int64_t)s->mesh->n_node;
    if (s->ref_r.n != (size_t)n) s->ref_r.alloc(n);
    if (s->ref_d.n != (size_t)n) s->ref_d.alloc(n);
    double bb = 0.0, rr = 0.0;
    dot_fp64(s->rhs.p, s->rhs.p, n, s->partials.p, s->counter.p, s->scalar.p, st, sm);
    MPHY_CUDA(cudaMemcpyAsync(&bb, s->scalar.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    MPHY_CUDA(cudaStreamSynchronize(st));
    const double bnorm = std::sqrt(bb);
    int32_t total = its ? *its : 0;
    double rel = 0.0;
    for (int k = 1;; ++k) {
        residual_fp64<double>(s->A, s->val.p, s->x.p, s->rhs.p, s->ref_r.p, s->partials.p, s->counter.p, s->scalar.p,
                              st, sm);
        s->launches += 1;
        MPHY_CUDA(cudaMemcpyAsync(&rr, s->scalar.p, sizeof(double), cudaMemcpyDeviceToHost, st));
        MPHY_CUDA(cudaStreamSynchronize(st));
        rel = bnorm > 0.0 ? std::sqrt(rr) / bnorm : 0.0;
        if (!(rel > s->opts.rtol) || k >= s->opts.max_outer || total >= s->opts.max_it) break;
        const double tol_in = std::fmin(0.5, std::fmax(s->opts.rtol, 0.5 * s->opts.rtol / rel));
        int32_t it = 0;
        double dn = 0.0;
        const int rc2 = s->pcg.solve(s->val.p, s->ref_r.p, s->ref_d.p, tol_in, 0.0, s->opts.dtol,
                                     s->opts.max_it - total, st, &it, &dn);
        s->launches += s->pcg.launches + 1;
        total += it;
        axpy_inplace(s->x.p, s->ref_d.p, 1.0, n, st, sm);
        s->last_sweeps = k + 1;
        if (rc2 == MPHY_ERR_INDEFINITE || rc2 == MPHY_ERR_DIVERGED) {
            rc = rc2;
            break;
        }
    }
    if (its) *its = total;
    if (fnorm) *fnorm = rel;
    if (rc == MPHY_OK || rc == MPHY_ERR_NOT_CONVERGED) rc = rel > s->opts.rtol ? MPHY_ERR_NOT_CONVERGED : MPHY_OK;
    return rc;
}

double true_relres(mphy_solver* s) {
    cudaStream_t st = s->ctx->stream;
    const int sm = s->ctx->sm_count;
    const int64_t n = 3 * (int64_t)s->mesh->n_node;
    if (s->ref_r.n != (size_t)n) s->ref_r.alloc(n);  // kept: no allocation per check
    DevBuf<double>& r = s->ref_r;
    if (s->mixed)
        residual_fp64<float>(s->A, s->valf.p, s->x.p, s->rhs.p, r.p, s->partials.p, s->counter.p, s->scalar.p, st, sm);
    else
        residual_fp64<double>(s->A, s->val.p, s->x.p, s->rhs.p, r.p, s->partials.p, s->counter.p, s->scalar.p, st, sm);
    double rr = 0.0, bb = 0.0;
    MPHY_CUDA(cudaMemcpyAsync(&rr, s->scalar.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    MPHY_CUDA(cudaStreamSynchronize(st));
    dot_fp64(s->rhs.p, s->rhs.p, n, s->partials.p, s->counter.p, s->scalar.p, st, sm);
    MPHY_CUDA(cudaMemcpyAsync(&bb, s->scalar.p, sizeof(double), cudaMemcpyDeviceToHost, st));
    MPHY_CUDA(cudaStreamSynchronize(st));
    return bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
}

float elapsed_ms(mphy_ctx* c) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    return ms;
}

// One Newton iteration on device buffers (femSolidmechanics2.cpp:762-816).
int newton_iteration(mphy_solver* s, double* disp, const double* fext, double lambda, double tol_abs,
                     mphy_iter_stats* st_out, bool* solved) {
    mphy_ctx* c = s->ctx;
    mphy_iter_stats st{};
    st.status = MPHY_OK;
    const int64_t l0 = s->launches;
    MPHY_CUDA(cudaEventRecord(c->ev0, c->stream));
    solver_assemble(s, disp);
    if (fext && lambda != 0.0) {
        add_scaled_free(s->mesh->fixed.p, fext, lambda, s->rhs.p, 3 * (int64_t)s->mesh->n_node, c->stream, c->sm_count);
        s->launches += 1;
    }
    MPHY_CUDA(cudaEventRecord(c->ev1, c->stream));
    int64_t bad = -1;
    st.rhs_norm = solver_norm_and_bad(s, &bad);
    st.t_assembly_ms = elapsed_ms(c);
    *solved = false;
    if (bad >= 0) {
        set_error("negative Jacobian in element " + std::to_string(bad));
        if (st_out) *st_out = st;
        return MPHY_ERR_NEG_JACOBIAN;
    }
    if (!(st.rhs_norm < tol_abs)) {
        MPHY_CUDA(cudaEventRecord(c->ev0, c->stream));
        int32_t its = 0;
        double fn = 0.0;
        st.status = solver_solve(s, &its, &fn);
        solver_update(s, disp);
        MPHY_CUDA(cudaEventRecord(c->ev1, c->stream));
        MPHY_CUDA(cudaEventSynchronize(c->ev1));
        st.t_solve_ms = elapsed_ms(c);
        st.krylov_its = its;
        *solved = true;
    }
    st.kernel_launches = s->launches - l0;
    if (st_out) *st_out = st;
    return MPHY_OK;
}

}  // namespace

namespace {
int elem_eval(mphy_ctx* c, const mphy_mesh* m, const double* disp, int32_t tangent, double* Ke, double* Re,
              int64_t* first_bad, bool tc) {
    return guarded([&] {
        MPHY_REQUIRE(c && m && disp && Ke && Re, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(m->npe == 8 || m->npe == 10, MPHY_ERR_UNSUPPORTED,
                     "the displacement element is hex8 or tet10 (27-node hexes: mphy_mixed_elem_eval)");
        DevBuf<unsigned long long> bad(1);
        MPHY_CUDA(cudaMemsetAsync(bad.p, 0xff, sizeof(unsigned long long), c->stream));
        ElemArgs a = elem_args(m, disp, tangent, bad.p);
        a.Ke = Ke;
        a.Re = Re;
        MPHY_REQUIRE(!(tc && m->general), MPHY_ERR_UNSUPPORTED,
                     "the tensor-core element kernel supports Neo-Hookean materials only");
        if (m->general) launch_elem_gen(a, m->npe, 1, c->stream);
        else if (tc) launch_elem_tc(a, m->npe, 1, c->stream);
        else launch_elem_fp64(a, m->npe, 1, c->stream);
        unsigned long long h = 0;
        MPHY_CUDA(cudaMemcpyAsync(&h, bad.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
        MPHY_CUDA(cudaStreamSynchronize(c->stream));
        const int64_t b = h == ULLONG_MAX ? -1 : (int64_t)h;
        if (first_bad) *first_bad = b;
        if (b >= 0) {
            set_error("negative Jacobian in element " + std::to_string(b));
            return (int)MPHY_ERR_NEG_JACOBIAN;
        }
        return (int)MPHY_OK;
    });
}
}  // namespace

extern "C" {

const char* mphy_status_string(int status) {
    switch (status) {
        case MPHY_OK: return "ok";
        case MPHY_ERR_INVALID_ARG: return "invalid argument";
        case MPHY_ERR_CUDA: return "CUDA error";
        case MPHY_ERR_NO_DEVICE: return "no CUDA device";
        case MPHY_ERR_OUT_OF_MEMORY: return "out of memory";
        case MPHY_ERR_UNSUPPORTED: return "unsupported";
        case MPHY_ERR_STATE: return "call out of order";
        case MPHY_ERR_NEG_JACOBIAN: return "negative Jacobian in an element";
        case MPHY_ERR_NOT_CONVERGED: return "Krylov iteration limit reached";
        case MPHY_ERR_INDEFINITE: return "indefinite matrix met by CG";
        case MPHY_ERR_DIVERGED: return "diverged";
        case MPHY_ERR_TIME_STEP: return "time step size fell below 1% of the initial value";
        default: return "unknown status";
    }
}

const char* mphy_last_error(void) { return g_last_error.c_str(); }
int mphy_api_version(void) { return MPHY_API_VERSION; }

int mphy_ctx_create(int device, mphy_ctx** out) {
    return guarded([&] {
        MPHY_REQUIRE(out, MPHY_ERR_INVALID_ARG, "out is null");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            throw Error{MPHY_ERR_NO_DEVICE, "no CUDA device visible"};
        }
        MPHY_REQUIRE(device >= 0 && device < n, MPHY_ERR_INVALID_ARG, "device id out of range");
        MPHY_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        MPHY_CUDA(cudaGetDeviceProperties(&prop, device));
        MPHY_REQUIRE(prop.major == 10, MPHY_ERR_UNSUPPORTED, "libmphy.so is built for sm_100a (B200) only");
        auto* c = new mphy_ctx;
        c->device = device;
        c->sm_count = prop.multiProcessorCount;
        // a blocking stream: ordered with the legacy default stream other CUDA users of the process use
        MPHY_CUDA(cudaStreamCreate(&c->stream));
        MPHY_CUDA(cudaEventCreate(&c->ev0));
        MPHY_CUDA(cudaEventCreate(&c->ev1));
        {
            std::lock_guard<std::mutex> lk(g_tables_mu);
            if (device < 64 && !g_tables_done[device]) {
                upload_shape_tables();
                g_tables_done[device] = true;
            }
        }
        *out = c;
        return (int)MPHY_OK;
    });
}

int mphy_ctx_destroy(mphy_ctx* c) {
    if (!c) return MPHY_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    cudaEventDestroy(c->ev0);
    cudaEventDestroy(c->ev1);
    cudaStreamDestroy(c->stream);
    delete c;
    return MPHY_OK;
}

int mphy_ctx_synchronize(mphy_ctx* c) {
    return guarded([&] {
        MPHY_REQUIRE(c, MPHY_ERR_INVALID_ARG, "ctx is null");
        MPHY_CUDA(cudaStreamSynchronize(c->stream));
        return (int)MPHY_OK;
    });
}

void* mphy_ctx_stream(mphy_ctx* c) { return c ? (void*)c->stream : nullptr; }

int mphy_mesh_create(mphy_ctx* c, int32_t n_node, const double* coords, int32_t n_elem, int32_t npe,
                     const int32_t* conn, const int32_t* mat_id, int32_t n_mat, const double* mats,
                     const uint8_t* fixed, mphy_mesh** out) {
    return guarded([&] {
        MPHY_REQUIRE(c && out && coords && conn && mat_id && mats && fixed, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(npe == 8 || npe == 10 || npe == 27, MPHY_ERR_UNSUPPORTED,
                     "npe must be 8 (hex8), 10 (tet10) or 27 (hex27, mixed u-p meshes only)");
        MPHY_REQUIRE(n_node > 0 && n_elem > 0 && n_mat > 0, MPHY_ERR_INVALID_ARG, "empty mesh");
        for (int32_t e = 0; e < n_elem; ++e)
            MPHY_REQUIRE(mat_id[e] >= 0 && mat_id[e] < n_mat, MPHY_ERR_INVALID_ARG, "material id out of range");
        for (int64_t i = 0; i < (int64_t)n_elem * npe; ++i)
            MPHY_REQUIRE(conn[i] >= 0 && conn[i] < n_node, MPHY_ERR_INVALID_ARG, "connectivity references a missing node");
        for (int32_t m = 0; m < n_mat; ++m)
            MPHY_REQUIRE(mats[3 * m + 1] > 0.0, MPHY_ERR_INVALID_ARG, "Kinv must be positive");
        MPHY_CUDA(cudaSetDevice(c->device));
        auto* m = new mphy_mesh;
        try {
            m->ctx = c;
            m->device = c->device;
            m->n_node = n_node;
            m->n_elem = n_elem;
            m->npe = npe;
            m->n_mat = n_mat;
            cudaStream_t s = c->stream;
            m->coords.alloc(3 * (size_t)n_node);
            m->coords.upload(coords, 3 * (size_t)n_node, s);
            m->conn.alloc((size_t)n_elem * npe);
            m->conn.upload(conn, (size_t)n_elem * npe, s);
            m->mat_id.alloc(n_elem);
            m->mat_id.upload(mat_id, n_elem, s);
            std::vector<double> m4(4 * (size_t)n_mat, 0.0);
            for (int32_t k = 0; k < n_mat; ++k)
                for (int q = 0; q < 3; ++q) m4[4 * k + q] = mats[3 * k + q];
            m->mats.alloc(m4.size());
            m->mats.upload(m4.data(), m4.size(), s);
            m->matx_host.assign(kMatRow * (size_t)n_mat, 0.0);
            for (int32_t k = 0; k < n_mat; ++k) {
                double* r = &m->matx_host[kMatRow * (size_t)k];
                r[0] = MPHY_MAT_NEOHOOKEAN;
                r[1] = mats[3 * k];
                r[5] = mats[3 * k + 1];
                r[6] = mats[3 * k + 2];
            }
            m->matx.alloc(m->matx_host.size());
            m->matx.upload(m->matx_host.data(), m->matx_host.size(), s);
            m->fixed_host.assign(fixed, fixed + 3 * (size_t)n_node);
            m->coords_host.assign(coords, coords + 3 * (size_t)n_node);
            m->fixed.alloc(3 * (size_t)n_node);
            m->fixed.upload(fixed, 3 * (size_t)n_node, s);
            MPHY_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
        return (int)MPHY_OK;
    });
}

int mphy_mesh_destroy(mphy_mesh* m) {
    if (!m) return MPHY_OK;
    // objects may be destroyed in any order relative to their context: no ctx access here
    cudaSetDevice(m->device);
    cudaDeviceSynchronize();
    delete m;
    return MPHY_OK;
}

int mphy_mesh_set_prescribed(mphy_mesh* m, const double* ramp, const double* cst) {
    return guarded([&] {
        MPHY_REQUIRE(m, MPHY_ERR_INVALID_ARG, "null mesh");
        const size_t nd = 3 * (size_t)m->n_node;
        bool any = false;
        std::vector<double> r(nd, 0.0), c(nd, 0.0);
        for (size_t i = 0; i < nd; ++i) {
            if (!m->fixed_host[i]) continue;
            r[i] = ramp ? ramp[i] : 0.0;
            c[i] = cst ? cst[i] : 0.0;
            MPHY_REQUIRE(std::isfinite(r[i]) && std::isfinite(c[i]), MPHY_ERR_INVALID_ARG,
                         "prescribed displacement is not finite");
            any |= r[i] != 0.0 || c[i] != 0.0;
        }
        MPHY_CUDA(cudaSetDevice(m->device));
        if (!any) {
            m->presc_ramp.release();
            m->presc_const.release();
            m->has_presc = false;
            return (int)MPHY_OK;
        }
        m->presc_ramp.alloc(nd);
        m->presc_const.alloc(nd);
        cudaStream_t st = m->ctx->stream;
        m->presc_ramp.upload(r.data(), nd, st);
        m->presc_const.upload(c.data(), nd, st);
        MPHY_CUDA(cudaStreamSynchronize(st));
        m->has_presc = true;
        return (int)MPHY_OK;
    });
}

int mphy_mesh_set_materials(mphy_mesh* m, int32_t n_mat, const int32_t* model, const double* data) {
    return guarded([&] {
        MPHY_REQUIRE(m && model && data, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(n_mat == m->n_mat, MPHY_ERR_INVALID_ARG, "n_mat differs from the mesh's material count");
        for (int32_t k = 0; k < n_mat; ++k) {
            MPHY_REQUIRE(model[k] >= MPHY_MAT_NEOHOOKEAN && model[k] <= MPHY_MAT_ARRUDABOYCE, MPHY_ERR_INVALID_ARG,
                         "unknown material model");
            const double* d = data + MPHY_MAT_NDATA * (size_t)k;
            MPHY_REQUIRE(model[k] != MPHY_MAT_GENT || d[1] > 0.0, MPHY_ERR_INVALID_ARG, "Gent needs Im > 0");
            MPHY_REQUIRE(model[k] != MPHY_MAT_ARRUDABOYCE || d[1] > 0.0, MPHY_ERR_INVALID_ARG,
                         "Arruda-Boyce needs N > 0");
        }
        MPHY_CUDA(cudaSetDevice(m->device));
        std::vector<double> m4(4 * (size_t)n_mat);
        MPHY_CUDA(cudaMemcpy(m4.data(), m->mats.p, m4.size() * sizeof(double), cudaMemcpyDeviceToHost));
        bool general = false;
        for (int32_t k = 0; k < n_mat; ++k) {
            double* r = &m->matx_host[kMatRow * (size_t)k];
            r[0] = model[k];
            for (int q = 0; q < MPHY_MAT_NDATA; ++q) r[1 + q] = data[MPHY_MAT_NDATA * (size_t)k + q];
            m4[4 * (size_t)k] = data[MPHY_MAT_NDATA * (size_t)k];
            general = general || model[k] != MPHY_MAT_NEOHOOKEAN;
        }
        // ordered after every assembly already issued on the mesh's stream
        cudaStream_t s = m->ctx ? m->ctx->stream : nullptr;
        m->matx.upload(m->matx_host.data(), m->matx_host.size(), s);
        m->mats.upload(m4.data(), m4.size(), s);
        MPHY_CUDA(cudaStreamSynchronize(s));
        m->general = general;
        return (int)MPHY_OK;
    });
}

int mphy_material_eval(mphy_ctx* c, int32_t n, const double* F, int32_t model, const double* data, double Kinv,
                       int32_t utype, int32_t tangent, double* stre, double* cmat) {
    return guarded([&] {
        MPHY_REQUIRE(c && F && data && stre && cmat && n >= 0 && Kinv > 0.0, MPHY_ERR_INVALID_ARG,
                     "invalid argument");
        MPHY_REQUIRE(model >= MPHY_MAT_NEOHOOKEAN && model <= MPHY_MAT_ARRUDABOYCE, MPHY_ERR_INVALID_ARG,
                     "unknown material model");
        double row[kMatRow] = {(double)model, data[0], data[1], data[2], data[3], Kinv, (double)utype, 0.0};
        DevBuf<double> drow(kMatRow);
        drow.upload(row, kMatRow, c->stream);
        launch_material_eval(n, F, drow.p, tangent, stre, cmat, c->stream);
        MPHY_CUDA(cudaStreamSynchronize(c->stream));
        return (int)MPHY_OK;
    });
}

int mphy_material_nh_eval(mphy_ctx* c, int32_t n, const double* F, double mu, double Kinv, int32_t utype,
                          int32_t tangent, double* stre, double* cmat) {
    return guarded([&] {
        MPHY_REQUIRE(c && F && stre && cmat && n >= 0 && Kinv > 0.0, MPHY_ERR_INVALID_ARG, "invalid argument");
        launch_nh_eval(n, F, mu, Kinv, utype, tangent, stre, cmat, c->stream);
        MPHY_CUDA(cudaStreamSynchronize(c->stream));
        return (int)MPHY_OK;
    });
}


int mphy_elem_eval(mphy_ctx* c, const mphy_mesh* m, const double* disp, int32_t tangent, double* Ke, double* Re,
                   int64_t* first_bad) {
    return elem_eval(c, m, disp, tangent, Ke, Re, first_bad, false);
}

int mphy_elem_eval_tc(mphy_ctx* c, const mphy_mesh* m, const double* disp, int32_t tangent, double* Ke, double* Re,
                      int64_t* first_bad) {
    return elem_eval(c, m, disp, tangent, Ke, Re, first_bad, true);
}

int mphy_pattern_build(mphy_ctx* c, const mphy_mesh* m, mphy_pattern** out) {
    return guarded([&] {
        MPHY_REQUIRE(c && m && out, MPHY_ERR_INVALID_ARG, "null argument");
        auto* P = new mphy_pattern;
        try {
            build_pattern(c, m, P);
        } catch (...) {
            delete P;
            throw;
        }
        *out = P;
        return (int)MPHY_OK;
    });
}

int mphy_pattern_info(const mphy_pattern* P, int32_t* n_free, int64_t* nnz, int64_t* n_blocks, int64_t* stored) {
    if (!P) return MPHY_ERR_INVALID_ARG;
    if (n_free) *n_free = P->n_free;
    if (nnz) *nnz = P->nnz;
    if (n_blocks) *n_blocks = P->n_blocks;
    if (stored) *stored = P->sell_blocks;
    return MPHY_OK;
}

int mphy_pattern_export_csr(const mphy_pattern* Pc, int64_t* rowptr, int32_t* col) {
    return guarded([&] {
        MPHY_REQUIRE(Pc, MPHY_ERR_INVALID_ARG, "null pattern");
        auto* P = const_cast<mphy_pattern*>(Pc);
        cudaStream_t s = P->ctx->stream;
        if (rowptr) P->csr_rowptr.download(rowptr, P->n_free + 1, s);
        if (col) {
            pattern_csr_columns(P, false);
            P->csr_col.download(col, P->nnz, s);
        }
        MPHY_CUDA(cudaStreamSynchronize(s));
        return (int)MPHY_OK;
    });
}

int mphy_pattern_export_dofmap(const mphy_pattern* P, int32_t* assy, int32_t* fav) {
    return guarded([&] {
        MPHY_REQUIRE(P, MPHY_ERR_INVALID_ARG, "null pattern");
        cudaStream_t s = P->ctx->stream;
        if (assy) P->assy_for_soln.download(assy, P->n_free, s);
        if (fav) {
            DevBuf<int32_t> tmp((size_t)P->n_elem * P->npe * 3);
            pattern_elem_dofs(P, P->mesh, tmp.p);
            tmp.download(fav, tmp.n, s);
            MPHY_CUDA(cudaStreamSynchronize(s));
        }
        MPHY_CUDA(cudaStreamSynchronize(s));
        return (int)MPHY_OK;
    });
}

int mphy_pattern_destroy(mphy_pattern* P) {
    if (!P) return MPHY_OK;
    cudaSetDevice(P->device);
    cudaDeviceSynchronize();
    delete P;
    return MPHY_OK;
}

void mphy_solver_opts_default(mphy_solver_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->precision = MPHY_PREC_FP64;
    o->pc_type = MPHY_PC_JACOBI;
    o->tangent = MPHY_TANGENT_REFERENCE;
    o->max_it = 10000;
    o->rtol = 1e-12;
    o->abstol = 1e-50;
    o->dtol = 1e5;
    o->inner_rtol = 0.0;  // inner sweep uses rtol (PETSc semantics on the preconditioned norm)
    o->max_outer = 1;
    o->chunk = 0;
}

int mphy_solver_create(mphy_ctx* c, const mphy_mesh* m, const mphy_pattern* P, const mphy_solver_opts* opts,
                       mphy_solver** out) {
    return guarded([&] {
        MPHY_REQUIRE(c && m && P && out, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(P->n_node == m->n_node && P->n_elem == m->n_elem, MPHY_ERR_INVALID_ARG, "pattern/mesh mismatch");
        MPHY_REQUIRE(m->npe == 8 || m->npe == 10, MPHY_ERR_UNSUPPORTED,
                     "the displacement element is hex8 or tet10; a 27-node hex mesh is for mphy_mixed_create");
        mphy_solver_opts o;
        mphy_solver_opts_default(&o);
        if (opts) o = *opts;
        MPHY_REQUIRE(o.precision == MPHY_PREC_FP64 || o.precision == MPHY_PREC_MIXED ||
                         o.precision == MPHY_PREC_MIXED_F32VEC || o.precision == MPHY_PREC_MIXED_TC,
                     MPHY_ERR_INVALID_ARG, "unknown precision");
        MPHY_REQUIRE(o.pc_type == MPHY_PC_JACOBI || o.pc_type == MPHY_PC_FSAI || o.pc_type == MPHY_PC_FSAI_LEARNED,
                     MPHY_ERR_INVALID_ARG, "unknown preconditioner");
        MPHY_REQUIRE(o.coarse_lag >= 0, MPHY_ERR_INVALID_ARG, "coarse_lag must be >= 0");
        MPHY_CUDA(cudaSetDevice(c->device));
        auto* s = new mphy_solver;
        try {
            s->ctx = c;
            s->device = c->device;
            s->mesh = m;
            s->pat = const_cast<mphy_pattern*>(P);
            s->opts = o;
            s->A = SellView{P->n_node, P->n_slices, P->slice_base.p, P->slice_width.p, P->sell_col.p, P->dvoff.p};
            s->mixed = o.precision != MPHY_PREC_FP64;
            if (s->mixed) {
                s->valf.alloc(9 * (size_t)P->sell_blocks);
                s->diag64.alloc(9 * (size_t)P->n_node);
                s->A.diag64 = s->diag64.p;
                s->A.fixed = m->fixed.p;
            } else {
                s->val.alloc(9 * (size_t)P->sell_blocks);
            }
            const size_t nd = 3 * (size_t)m->n_node;
            s->rhs.alloc(nd);
            s->reac.alloc(nd);
            s->x.alloc(nd);
            s->bad.alloc(1);
            s->partials.alloc((size_t)c->sm_count * 8 + 8);
            s->scalar.alloc(1);
            s->counter.alloc(1);
            MPHY_CUDA(cudaMemset(s->counter.p, 0, sizeof(uint32_t)));
            if (o.precision == MPHY_PREC_MIXED || o.precision == MPHY_PREC_MIXED_TC) s->ir.init(s->A, c->sm_count, o.chunk);
            else if (o.precision == MPHY_PREC_MIXED_F32VEC) s->ir32.init(s->A, c->sm_count, o.chunk);
            else s->pcg.init(s->A, c->sm_count, o.chunk);
            if (o.pc_type != MPHY_PC_JACOBI) {
                s->use_fsai = true;
                s->fsai.init(c, P, 16);
                const FactorView<FactorT> fv = s->fsai.view();
                if (o.precision == MPHY_PREC_MIXED || o.precision == MPHY_PREC_MIXED_TC) s->ir.inner().set_factor(fv);
                else if (o.precision == MPHY_PREC_MIXED_F32VEC) s->ir32.inner().set_factor(fv);
                else s->pcg.set_factor(fv);
            }
            if (o.coarse_aggregates > 0) {
                s->use_coarse = true;
                s->coarse.init(c, m, P, o.coarse_aggregates, o.coarse_modes > 0 ? o.coarse_modes : 6);
                const CoarseView cv = s->coarse.view();
                if (o.precision == MPHY_PREC_MIXED || o.precision == MPHY_PREC_MIXED_TC) s->ir.inner().set_coarse(cv);
                else if (o.precision == MPHY_PREC_MIXED_F32VEC) s->ir32.inner().set_coarse(cv);
                else s->pcg.set_coarse(cv);
            }
            // a learned local part is judged by the true residual, so it also stops on it
            const int nt = o.pc_type == MPHY_PC_FSAI_LEARNED ? 1 : o.norm_type;
            s->pcg.norm_type = nt;
            s->ir.inner().norm_type = nt;
            s->ir32.inner().norm_type = nt;
            MPHY_CUDA(cudaMallocHost(&s->pinned, 4 * sizeof(double)));
            s->state = MPHY_PATTERN_OK;
            solver_zero(s);
            MPHY_CUDA(cudaStreamSynchronize(c->stream));
            s->state = MPHY_INIT_OK;
        } catch (...) {
            if (s->pinned) cudaFreeHost(s->pinned);
            delete s;
            throw;
        }
        *out = s;
        return (int)MPHY_OK;
    });
}

int mphy_solver_destroy(mphy_solver* s) {
    if (!s) return MPHY_OK;
    cudaSetDevice(s->device);
    cudaDeviceSynchronize();
    if (s->pinned) cudaFreeHost(s->pinned);
    delete s;
    return MPHY_OK;
}

int mphy_solver_get_state(const mphy_solver* s, int32_t* state) {
    if (!s || !state) return MPHY_ERR_INVALID_ARG;
    *state = s->state;
    return MPHY_OK;
}

int mphy_solver_zero(mphy_solver* s) {
    return guarded([&] {
        MPHY_REQUIRE(s, MPHY_ERR_INVALID_ARG, "null solver");
        solver_zero(s);
        MPHY_CUDA(cudaStreamSynchronize(s->ctx->stream));
        s->state = MPHY_INIT_OK;
        return (int)MPHY_OK;
    });
}

int mphy_solver_assemble(mphy_solver* s, const double* disp, int64_t* first_bad) {
    return guarded([&] {
        MPHY_REQUIRE(s && disp, MPHY_ERR_INVALID_ARG, "null argument");
        solver_assemble(s, disp);
        unsigned long long h = 0;
        MPHY_CUDA(cudaMemcpyAsync(&h, s->bad.p, sizeof(h), cudaMemcpyDeviceToHost, s->ctx->stream));
        MPHY_CUDA(cudaStreamSynchronize(s->ctx->stream));
        const int64_t b = h == ULLONG_MAX ? -1 : (int64_t)h;
        if (first_bad) *first_bad = b;
        if (b >= 0) {
            set_error("negative Jacobian in element " + std::to_string(b));
            return (int)MPHY_ERR_NEG_JACOBIAN;
        }
        return (int)MPHY_OK;
    });
}

int mphy_solver_assemble_batch(mphy_solver* s, int32_t n, const int32_t* ids, const double* Ke, const double* Re) {
    return guarded([&] {
        MPHY_REQUIRE(s && Ke && Re && n >= 0, MPHY_ERR_INVALID_ARG, "invalid argument");
        MPHY_REQUIRE(ids || n == s->mesh->n_elem, MPHY_ERR_INVALID_ARG, "without ids, n must equal n_elem");
        launch_scatter_batch(s->mesh->npe, n, ids, s->mesh, s->pat, Ke, Re, s->val.p, s->mixed ? s->valf.p : nullptr,
                             s->rhs.p, s->reac.p, s->ctx->stream, s->ctx->sm_count);
        if (s->mixed) diag_from_offdiag(s->A, s->valf.p, s->diag64.p, s->ctx->stream, s->ctx->sm_count);
        MPHY_CUDA(cudaStreamSynchronize(s->ctx->stream));
        s->state = MPHY_ASSEMBLY_OK;
        return (int)MPHY_OK;
    });
}

int mphy_solver_assemble_batch_host(mphy_solver* s, int32_t n, const int32_t* ids, const double* Ke,
                                    const double* Re) {
    return guarded([&] {
        MPHY_REQUIRE(s && Ke && Re && n >= 0, MPHY_ERR_INVALID_ARG, "invalid argument");
        MPHY_REQUIRE(ids || n == s->mesh->n_elem, MPHY_ERR_INVALID_ARG, "without ids, n must equal n_elem");
        if (ids)
            for (int32_t k = 0; k < n; ++k)
                MPHY_REQUIRE(ids[k] >= 0 && ids[k] < s->mesh->n_elem, MPHY_ERR_INVALID_ARG, "element id out of range");
        const int ns = 3 * s->mesh->npe;
        constexpr int32_t kChunk = 16384;  // elements staged per copy (75 MB of hex8 matrices)
        const int32_t m0 = n < kChunk ? n : kChunk;
        DevBuf<double> kd((size_t)m0 * ns * ns), rd((size_t)m0 * ns);
        DevBuf<int32_t> idd(m0);
        std::vector<int32_t> iota;
        cudaStream_t st = s->ctx->stream;
        for (int32_t off = 0; off < n; off += kChunk) {
            const int32_t m = n - off < kChunk ? n - off : kChunk;
            kd.upload(Ke + (size_t)off * ns * ns, (size_t)m * ns * ns, st);
            rd.upload(Re + (size_t)off * ns, (size_t)m * ns, st);
            if (ids) {
                idd.upload(ids + off, m, st);
            } else {
                iota.resize(m);
                for (int32_t k = 0; k < m; ++k) iota[k] = off + k;
                idd.upload(iota.data(), m, st);
            }
            launch_scatter_batch(s->mesh->npe, m, idd.p, s->mesh, s->pat, kd.p, rd.p, s->val.p,
                                 s->mixed ? s->valf.p : nullptr, s->rhs.p, s->reac.p, st, s->ctx->sm_count);
            // the staging buffers are reused by the next chunk
            MPHY_CUDA(cudaStreamSynchronize(st));
        }
        if (s->mixed) diag_from_offdiag(s->A, s->valf.p, s->diag64.p, st, s->ctx->sm_count);
        MPHY_CUDA(cudaStreamSynchronize(st));
        s->state = MPHY_ASSEMBLY_OK;
        return (int)MPHY_OK;
    });
}

int mphy_solver_add_nodal_forces_host(mphy_solver* s, const double* fext, double scale) {
    return guarded([&] {
        MPHY_REQUIRE(s && fext, MPHY_ERR_INVALID_ARG, "null argument");
        const size_t nd = 3 * (size_t)s->mesh->n_node;
        if (s->fext_tmp.n != nd) s->fext_tmp.alloc(nd);
        s->fext_tmp.upload(fext, nd, s->ctx->stream);
        add_scaled_free(s->mesh->fixed.p, s->fext_tmp.p, scale, s->rhs.p, (int64_t)nd, s->ctx->stream,
                        s->ctx->sm_count);
        MPHY_CUDA(cudaStreamSynchronize(s->ctx->stream));
        return (int)MPHY_OK;
    });
}

int mphy_solver_add_nodal_forces(mphy_solver* s, const double* fext, double scale) {
    return guarded([&] {
        MPHY_REQUIRE(s && fext, MPHY_ERR_INVALID_ARG, "null argument");
        add_scaled_free(s->mesh->fixed.p, fext, scale, s->rhs.p, 3 * (int64_t)s->mesh->n_node, s->ctx->stream,
                        s->ctx->sm_count);
        return (int)MPHY_OK;
    });
}

int mphy_solver_rhs_norm(mphy_solver* s, double* norm) {
    return guarded([&] {
        MPHY_REQUIRE(s && norm, MPHY_ERR_INVALID_ARG, "null argument");
        *norm = solver_norm_and_bad(s, nullptr);
        return (int)MPHY_OK;
    });
}

int mphy_solver_solve(mphy_solver* s, int32_t* its, double* fnorm) {
    return guarded([&] {
        MPHY_REQUIRE(s, MPHY_ERR_INVALID_ARG, "null solver");
        const int st = solver_solve(s, its, fnorm);
        if (st != MPHY_OK) set_error(mphy_status_string(st));
        return st;
    });
}

int mphy_solver_spmv(mphy_solver* s, const double* x, double* y) {
    return guarded([&] {
        MPHY_REQUIRE(s && x && y, MPHY_ERR_INVALID_ARG, "null argument");
        if (s->mixed) spmv<float, double>(s->A, s->valf.p, x, y, s->ctx->stream, s->ctx->sm_count);
        else spmv<double, double>(s->A, s->val.p, x, y, s->ctx->stream, s->ctx->sm_count);
        s->launches += 1;
        return (int)MPHY_OK;
    });
}

int mphy_solver_spmv_dot(mphy_solver* s, const double* x, double* y, double* xy_host) {
    return guarded([&] {
        MPHY_REQUIRE(s && x && y, MPHY_ERR_INVALID_ARG, "null argument");
        if (!s->dot_st.p) {
            s->dot_st.alloc(1);
            s->dot_part.alloc((size_t)s->ctx->sm_count * 8 + 8);
        }
        cudaStream_t st = s->ctx->stream;
        if (s->mixed)
            spmv_dot<float, double>(s->A, s->valf.p, x, y, s->dot_part.p, s->dot_st.p, st, s->ctx->sm_count);
        else spmv_dot<double, double>(s->A, s->val.p, x, y, s->dot_part.p, s->dot_st.p, st, s->ctx->sm_count);
        s->launches += 1;
        if (xy_host) {
            PcgState h{};
            MPHY_CUDA(cudaMemcpyAsync(&h, s->dot_st.p, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
            MPHY_CUDA(cudaStreamSynchronize(st));
            *xy_host = h.pq;
        }
        return (int)MPHY_OK;
    });
}

int mphy_solver_matrix_info(const mphy_solver* s, int64_t* stored, int64_t* true_blocks, int64_t* value_bytes) {
    if (!s) return MPHY_ERR_INVALID_ARG;
    if (stored) *stored = s->pat->sell_blocks;
    if (true_blocks) *true_blocks = s->pat->n_blocks;
    if (value_bytes) *value_bytes = (int64_t)(s->mixed ? s->valf.bytes() : s->val.bytes());
    return MPHY_OK;
}

int mphy_solver_pc_pattern(mphy_solver* s, int64_t* n_lower, int64_t* rowptr, int32_t* col) {
    return guarded([&] {
        MPHY_REQUIRE(s && s->use_fsai, MPHY_ERR_STATE, "the solver has no factorised preconditioner");
        const SellPattern& L = s->fsai.lower();
        if (n_lower) *n_lower = L.n_blocks;
        if (rowptr) L.rowptr.download(rowptr, (size_t)L.n_node + 1, s->ctx->stream);
        if (col) L.col.download(col, (size_t)L.n_blocks, s->ctx->stream);
        MPHY_CUDA(cudaStreamSynchronize(s->ctx->stream));
        return (int)MPHY_OK;
    });
}

int mphy_solver_pc_get_blocks(mphy_solver* s, float* blocks) {
    return guarded([&] {
        MPHY_REQUIRE(s && blocks, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(s->use_fsai, MPHY_ERR_STATE, "the solver has no factorised preconditioner");
        s->fsai.get_lower_values(blocks, s->ctx->stream);
        MPHY_CUDA(cudaStreamSynchronize(s->ctx->stream));
        return (int)MPHY_OK;
    });
}

int mphy_solver_pc_set_blocks(mphy_solver* s, const float* blocks) {
    return guarded([&] {
        MPHY_REQUIRE(s && blocks, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(s->use_fsai, MPHY_ERR_STATE, "the solver has no factorised preconditioner");
        s->fsai.set_lower_values(blocks, s->ctx->stream);
        MPHY_CUDA(cudaStreamSynchronize(s->ctx->stream));
        return (int)MPHY_OK;
    });
}

int mphy_solver_pc_setup(mphy_solver* s, int32_t* n_fallback) {
    return guarded([&] {
        MPHY_REQUIRE(s, MPHY_ERR_INVALID_ARG, "null solver");
        MPHY_REQUIRE(s->use_fsai, MPHY_ERR_STATE, "the solver has no factorised preconditioner");
        MPHY_REQUIRE(s->state == MPHY_ASSEMBLY_OK || s->state == MPHY_FACTORISE_OK, MPHY_ERR_STATE,
                     "assemble the matrix first");
        if (s->mixed) s->fsai.compute<float>(s->valf.p, s->diag64.p, s->mesh->fixed.p, s->ctx->stream);
        else s->fsai.compute<double>(s->val.p, nullptr, nullptr, s->ctx->stream);
        const int32_t nf = s->fsai.fallback_rows(s->ctx->stream);
        if (n_fallback) *n_fallback = nf;
        return (int)MPHY_OK;
    });
}

int mphy_solver_true_residual(mphy_solver* s, double* relres) {
    return guarded([&] {
        MPHY_REQUIRE(s && relres, MPHY_ERR_INVALID_ARG, "null argument");
        *relres = true_relres(s);
        return (int)MPHY_OK;
    });
}

int mphy_solver_pc_last(const mphy_solver* s, int32_t* fallback, float* setup_ms, int32_t* first_status,
                        int32_t* first_its, double* first_relres) {
    if (!s) return MPHY_ERR_INVALID_ARG;
    if (fallback) *fallback = s->last_fallback;
    if (setup_ms) *setup_ms = (float)s->t_pc_ms;
    if (first_status) *first_status = s->first_status;
    if (first_its) *first_its = s->first_its;
    if (first_relres) *first_relres = s->first_relres;
    return MPHY_OK;
}

int mphy_solver_coarse_info(const mphy_solver* s, int32_t* grid3, int32_t* k, float* setup_ms) {
    if (!s) return MPHY_ERR_INVALID_ARG;
    if (!s->use_coarse) {
        set_error("the solver has no coarse correction");
        return MPHY_ERR_STATE;
    }
    if (grid3)
        for (int d = 0; d < 3; ++d) grid3[d] = s->coarse.grid()[d];
    if (k) *k = s->coarse.coarse_size();
    if (setup_ms) *setup_ms = s->coarse.last_setup_ms;
    return MPHY_OK;
}

int mphy_solver_get_solution(mphy_solver* s, double* dx) {
    return guarded([&] {
        MPHY_REQUIRE(s && dx, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_CUDA(cudaMemcpyAsync(dx, s->x.p, s->x.bytes(), cudaMemcpyDeviceToDevice, s->ctx->stream));
        MPHY_CUDA(cudaStreamSynchronize(s->ctx->stream));
        return (int)MPHY_OK;
    });
}

int mphy_solver_get_solution_host(mphy_solver* s, double* dx) {
    return guarded([&] {
        MPHY_REQUIRE(s && dx, MPHY_ERR_INVALID_ARG, "null argument");
        s->x.download(dx, s->x.n, s->ctx->stream);
        MPHY_CUDA(cudaStreamSynchronize(s->ctx->stream));
        return (int)MPHY_OK;
    });
}

int mphy_solver_update_disp(mphy_solver* s, double* disp) {
    return guarded([&] {
        MPHY_REQUIRE(s && disp, MPHY_ERR_INVALID_ARG, "null argument");
        solver_update(s, disp);
        return (int)MPHY_OK;
    });
}

int mphy_solver_set_mixed_p0(mphy_solver* s, int32_t enable) {
    return guarded([&] {
        MPHY_REQUIRE(s, MPHY_ERR_INVALID_ARG, "null solver");
        if (!enable) {
            s->p0 = false;
            return (int)MPHY_OK;
        }
        const mphy_mesh* m = s->mesh;
        for (int32_t k = 0; k < m->n_mat; ++k)
            MPHY_REQUIRE((int)m->matx_host[kMatRow * (size_t)k + 6] != -1, MPHY_ERR_UNSUPPORTED,
                         "constant-pressure element: Utype -1 (incompressible) has Kpp = 0");
        MPHY_CUDA(cudaSetDevice(s->device));
        cudaStream_t st = s->ctx->stream;
        const size_t nd = 3 * (size_t)m->n_node, ne = (size_t)m->n_elem;
        s->pe.alloc(ne);
        s->pe_prev.alloc(ne);
        s->kup_e.alloc(ne * 3 * (size_t)m->npe);
        s->kpp_e.alloc(ne);
        s->fp_e.alloc(ne);
        if (s->disp_prev.n != nd) s->disp_prev.alloc(nd);
        for (DevBuf<double>* b : {&s->pe, &s->pe_prev, &s->disp_prev})
            MPHY_CUDA(cudaMemsetAsync(b->p, 0, b->bytes(), st));
        MPHY_CUDA(cudaStreamSynchronize(st));
        s->p0 = true;
        s->state = std::min(s->state, (int)MPHY_INIT_OK);
        return (int)MPHY_OK;
    });
}

int mphy_solver_p0_pressure(mphy_solver* s, const double* set_host, double* get_host) {
    return guarded([&] {
        MPHY_REQUIRE(s && s->p0, MPHY_ERR_STATE, "the constant-pressure element is not enabled");
        cudaStream_t st = s->ctx->stream;
        if (set_host) s->pe.upload(set_host, s->pe.n, st);
        if (get_host) s->pe.download(get_host, s->pe.n, st);
        MPHY_CUDA(cudaStreamSynchronize(st));
        return (int)MPHY_OK;
    });
}

int mphy_solver_save_step(mphy_solver* s, const double* disp) {
    return guarded([&] {
        MPHY_REQUIRE(s && disp, MPHY_ERR_INVALID_ARG, "null argument");
        const size_t nd = 3 * (size_t)s->mesh->n_node;
        cudaStream_t st = s->ctx->stream;
        if (s->disp_prev.n != nd) s->disp_prev.alloc(nd);
        MPHY_CUDA(cudaMemcpyAsync(s->disp_prev.p, disp, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
        if (s->p0) s->pe_prev.copy_from(s->pe, st);
        MPHY_CUDA(cudaStreamSynchronize(st));
        return (int)MPHY_OK;
    });
}

int mphy_solver_export(mphy_solver* s, double* val_host, double* rhs_host, double* reac_host) {
    return guarded([&] {
        MPHY_REQUIRE(s, MPHY_ERR_INVALID_ARG, "null solver");
        cudaStream_t st = s->ctx->stream;
        const int sm = s->ctx->sm_count;
        if (val_host && s->pat->nnz > 0) {
            pattern_csr_columns(s->pat, true);
            DevBuf<double> tmp(s->pat->nnz);
            if (s->mixed) {
                // the operator's diagonal blocks: minus the sums of the stored rows
                DevBuf<double> dex(9 * (size_t)s->mesh->n_node);
                diag_from_offdiag(s->A, s->valf.p, dex.p, st, sm);
                gather_values<float>(s->valf.p, s->pat->csr_src.p, tmp.p, s->pat->nnz, st, sm);
                export_fix_diagonal(dex.p, s->pat->csr_rowptr.p, s->pat->csr_col.p, s->pat->assy_for_soln.p,
                                    s->pat->n_free, tmp.p, st, sm);
            } else {
                gather_values<double>(s->val.p, s->pat->csr_src.p, tmp.p, s->pat->nnz, st, sm);
            }
            tmp.download(val_host, s->pat->nnz, st);
            MPHY_CUDA(cudaStreamSynchronize(st));
        }
        if (rhs_host && s->pat->n_free > 0) {
            DevBuf<double> tmp(s->pat->n_free);
            gather_free(s->rhs.p, s->pat->assy_for_soln.p, tmp.p, s->pat->n_free, st, sm);
            tmp.download(rhs_host, s->pat->n_free, st);
            MPHY_CUDA(cudaStreamSynchronize(st));
        }
        if (reac_host) s->reac.download(reac_host, s->reac.n, st);
        MPHY_CUDA(cudaStreamSynchronize(st));
        return (int)MPHY_OK;
    });
}

int mphy_newton_iteration(mphy_solver* s, double* disp, const double* fext, double lambda, double tol_abs,
                          mphy_iter_stats* stats) {
    return guarded([&] {
        MPHY_REQUIRE(s && disp, MPHY_ERR_INVALID_ARG, "null argument");
        bool solved = false;
        return newton_iteration(s, disp, fext, lambda, tol_abs, stats, &solved);
    });
}

int mphy_newton_iteration_host(mphy_solver* s, double* disp_host, const double* fext_host, double lambda,
                               double tol_abs, mphy_iter_stats* stats) {
    return guarded([&] {
        MPHY_REQUIRE(s && disp_host, MPHY_ERR_INVALID_ARG, "null argument");
        const size_t nd = 3 * (size_t)s->mesh->n_node;
        cudaStream_t st = s->ctx->stream;
        if (!s->disp_tmp.p) s->disp_tmp.alloc(nd);
        if (fext_host && !s->fext_tmp.p) s->fext_tmp.alloc(nd);
        s->disp_tmp.upload(disp_host, nd, st);
        if (fext_host) s->fext_tmp.upload(fext_host, nd, st);
        bool solved = false;
        const int rc = newton_iteration(s, s->disp_tmp.p, fext_host ? s->fext_tmp.p : nullptr, lambda, tol_abs, stats,
                                        &solved);
        s->disp_tmp.download(disp_host, nd, st);
        MPHY_CUDA(cudaStreamSynchronize(st));
        return rc;
    });
}

int mphy_newton_run(mphy_solver* s, const double* fext_host, const mphy_newton_opts* o, double* disp_host,
                    mphy_iter_stats* hist, int32_t max_hist, int32_t* n_hist) {
    return guarded([&] {
        MPHY_REQUIRE(s && fext_host && o && disp_host, MPHY_ERR_INVALID_ARG, "null argument");
        const size_t nd = 3 * (size_t)s->mesh->n_node;
        cudaStream_t st = s->ctx->stream;
        if (!s->disp_tmp.p) s->disp_tmp.alloc(nd);
        if (!s->fext_tmp.p) s->fext_tmp.alloc(nd);
        if (!s->disp_prev.p) s->disp_prev.alloc(nd);
        double* disp = s->disp_tmp.p;
        s->disp_tmp.upload(disp_host, nd, st);
        s->fext_tmp.upload(fext_host, nd, st);
        const bool presc = s->mesh->has_presc;
        MPHY_REQUIRE(!presc || s->opts.precision != MPHY_PREC_MIXED_TC, MPHY_ERR_UNSUPPORTED,
                     "prescribed displacements with the tensor-core tangent");
        if (presc && s->lift.n != nd) s->lift.alloc(nd);
        double t = 0.0, dt = o->dt;
        const double dt0 = o->dt;
        int steps_done = 1, rows = 0, rc = MPHY_OK;
        while (t <= o->t_final - 1.0e-10 && steps_done <= o->max_steps) {
            // timeUpdate: myTime.update, TimeFunction::update (lambda = t), saveSolution
            t += dt;
            const double lambda = t;
            MPHY_CUDA(cudaMemcpyAsync(s->disp_prev.p, disp, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
            if (s->p0) s->pe_prev.copy_from(s->pe, st);
            // setBoundaryConditions (femSolidmechanics1.cpp:813-891): dispApplied = value(t) - disp on
            // the prescribed DOFs, lifted in the first iteration and added with its solution
            if (presc)
                prescribed_increment(s->mesh->fixed.p, s->mesh->presc_ramp.p, s->mesh->presc_const.p, t, disp,
                                     s->lift.p, (int64_t)nd, st, s->ctx->sm_count);
            bool converged = false;
            double norm = -1.0, norm_prev = -1.0, tol = o->tol_abs;
            s->coarse_ready = false;  // a lagged coarse operator never outlives its load step
            for (int iter = 1; iter <= o->max_newton; ++iter) {
                mphy_iter_stats is{};
                const int64_t l0 = s->launches;
                MPHY_CUDA(cudaEventRecord(s->ctx->ev0, st));
                solver_assemble(s, disp, nullptr, presc && iter == 1 ? s->lift.p : nullptr);
                add_scaled_free(s->mesh->fixed.p, s->fext_tmp.p, lambda, s->rhs.p, (int64_t)nd, st, s->ctx->sm_count);
                MPHY_CUDA(cudaEventRecord(s->ctx->ev1, st));
                int64_t bad = -1;
                norm_prev = norm;
                norm = solver_norm_and_bad(s, &bad);
                is.t_assembly_ms = elapsed_ms(s->ctx);
                if (bad >= 0) break;  // "Negative Jacobian encountered": the iteration loop ends
                if (iter == 1) tol = std::fmax(o->tol_abs, o->tol_rel * norm);
                bool stop = false;
                if (norm < tol) {
                    converged = true;
                    stop = true;
                } else if (iter > 3 && (std::isnan(norm) || (norm_prev > -0.1 && norm / norm_prev > 1.0e7))) {
                    stop = true;  // diverging(1e7), femSolidmechanics1.cpp:627-636
                } else {
                    MPHY_CUDA(cudaEventRecord(s->ctx->ev0, st));
                    int32_t its = 0;
                    double fn = 0.0;
                    is.status = solver_solve(s, &its, &fn);  // KSP divergence is only reported
                    solver_update(s, disp);
                    // dispIncr[prescribed] += dispApplied in the first iteration (femSolidmechanics2.cpp:1137-1145)
                    if (presc && iter == 1) axpy_inplace(disp, s->lift.p, 1.0, (int64_t)nd, st, s->ctx->sm_count);
                    MPHY_CUDA(cudaEventRecord(s->ctx->ev1, st));
                    MPHY_CUDA(cudaEventSynchronize(s->ctx->ev1));
                    is.t_solve_ms = elapsed_ms(s->ctx);
                    is.krylov_its = its;
                }
                is.step = steps_done;
                is.iter = iter;
                is.rhs_norm = norm;
                is.kernel_launches = s->launches - l0;
                if (hist && rows < max_hist) hist[rows++] = is;
                if (stop) break;
            }
            if (converged) {
                ++steps_done;
            } else {
                // MyTime::cut + SolutionDataSolid::reset
                t -= dt;
                dt *= 0.5;
                if (dt < dt0 * 0.01) {
                    rc = MPHY_ERR_TIME_STEP;
                    set_error(mphy_status_string(rc));
                    break;
                }
                MPHY_CUDA(cudaMemcpyAsync(disp, s->disp_prev.p, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
                if (s->p0) s->pe.copy_from(s->pe_prev, st);
            }
        }
        s->disp_tmp.download(disp_host, nd, st);
        MPHY_CUDA(cudaStreamSynchronize(st));
        if (n_hist) *n_hist = rows;
        return rc;
    });
}


int mphy_arclength_run(mphy_solver* s, const double* fext_host, const mphy_newton_opts* o, double* disp_host,
                       double* step_lambda, int32_t max_steps_out, int32_t* n_steps, mphy_iter_stats* hist,
                       double* hist_lambda, int32_t max_hist, int32_t* n_hist) {
    return guarded([&] {
        MPHY_REQUIRE(s && fext_host && o && disp_host, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(o->dt > 0.0 && o->max_newton >= 2, MPHY_ERR_INVALID_ARG,
                     "arc-length needs dt > 0 and max_newton >= 2 (iterations 1..max_newton-1)");
        MPHY_REQUIRE(!s->p0, MPHY_ERR_UNSUPPORTED, "arc-length with the constant-pressure element");
        MPHY_REQUIRE(!s->mesh->has_presc, MPHY_ERR_UNSUPPORTED, "arc-length with nonzero prescribed displacements");
        const size_t nd = 3 * (size_t)s->mesh->n_node;
        const int64_t n = (int64_t)nd;
        cudaStream_t st = s->ctx->stream;
        const int sm = s->ctx->sm_count;
        for (DevBuf<double>* b : {&s->disp_tmp, &s->fext_tmp, &s->disp_prev, &s->disp_prev2, &s->du_full, &s->x_first})
            if (!b->p) b->alloc(nd);
        if (!s->arc_dots.p) s->arc_dots.alloc(4);
        double* disp = s->disp_tmp.p;
        s->disp_tmp.upload(disp_host, nd, st);
        s->fext_tmp.upload(fext_host, nd, st);
        MPHY_CUDA(cudaMemcpyAsync(s->disp_prev.p, disp, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
        MPHY_CUDA(cudaMemcpyAsync(s->disp_prev2.p, disp, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
        double h[4];
        // F.F over every DOF (the full Fext of SolverPetsc.cpp:674)
        dot_fp64(s->fext_tmp.p, s->fext_tmp.p, n, s->partials.p, s->counter.p, s->arc_dots.p, st, sm);
        s->arc_dots.download(h, 1, st);
        MPHY_CUDA(cudaStreamSynchronize(st));
        const double FtF = h[0];
        double t = 0.0;
        double lam = o->dt, lam_prev = 0.0, lam_prev2 = 0.0;  // femBase.cpp:65; loadFactor = myTime.dt
        double ds = 0.0, ds_prev = 0.0, ds_max = 0.0, ds_min = 0.0;
        bool conv = false, conv_prev = false;
        int steps_done = 1, rows = 0, nl = 0, rc = MPHY_OK;
        while (t <= o->t_final - 1.0e-10 && steps_done <= o->max_steps) {
            t += o->dt;  // timeUpdate: myTime.update
            conv_prev = conv;
            conv = false;
            if (steps_done > 1) {
                // disp = (1 + f) dispPrev - f dispPrev2, lambda likewise, f = Ds / Ds_prev
                const double f = ds / ds_prev;
                MPHY_CUDA(cudaMemcpyAsync(disp, s->disp_prev.p, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
                axpy_inplace(disp, s->disp_prev.p, f, n, st, sm);
                axpy_inplace(disp, s->disp_prev2.p, -f, n, st, sm);
                lam = (1.0 + f) * lam_prev - f * lam_prev2;
            }
            // DuFull = disp - dispPrev
            MPHY_CUDA(cudaMemcpyAsync(s->du_full.p, disp, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
            axpy_inplace(s->du_full.p, s->disp_prev.p, -1.0, n, st, sm);
            double dlam = lam - lam_prev;
            double norm = -1.0, tol = o->tol_abs;
            s->coarse_ready = false;  // a lagged coarse operator never outlives its load step
            for (int iter = 1; iter < o->max_newton; ++iter) {
                mphy_iter_stats is{};
                const int64_t l0 = s->launches;
                MPHY_CUDA(cudaEventRecord(s->ctx->ev0, st));
                solver_assemble(s, disp);
                add_scaled_free(s->mesh->fixed.p, s->fext_tmp.p, lam, s->rhs.p, n, st, sm);
                MPHY_CUDA(cudaEventRecord(s->ctx->ev1, st));
                int64_t bad = -1;
                norm = solver_norm_and_bad(s, &bad);
                is.t_assembly_ms = elapsed_ms(s->ctx);
                if (bad >= 0) break;  // the element throws; the iteration loop ends
                if (iter == 1) tol = std::fmax(o->tol_abs, o->tol_rel * norm);
                const bool done = norm < tol;
                if (!done) {
                    // SolverPetsc::solveArclengthSystem: x1 = K^-1 R (du2 = -x1), x2 = K^-1 F on one
                    // assembled K, dl from the linearised spherical constraint, soln = x1 + dl x2
                    MPHY_CUDA(cudaEventRecord(s->ctx->ev0, st));
                    int32_t its1 = 0, its2 = 0;
                    double fn = 0.0;
                    const int st1 = solver_solve(s, &its1, &fn);
                    MPHY_CUDA(cudaMemcpyAsync(s->x_first.p, s->x.p, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
                    MPHY_CUDA(cudaMemsetAsync(s->rhs.p, 0, nd * sizeof(double), st));
                    add_scaled_free(s->mesh->fixed.p, s->fext_tmp.p, 1.0, s->rhs.p, n, st, sm);
                    const int st2 = solver_solve(s, &its2, &fn);
                    double A = 0.0, b = 1.0, adu2 = 0.0, adu1 = 0.0;
                    if (steps_done > 1) {
                        dot_fp64(s->du_full.p, s->du_full.p, n, s->partials.p, s->counter.p, s->arc_dots.p, st, sm);
                        dot_fp64(s->du_full.p, s->x_first.p, n, s->partials.p, s->counter.p, s->arc_dots.p + 1, st, sm);
                        dot_fp64(s->du_full.p, s->x.p, n, s->partials.p, s->counter.p, s->arc_dots.p + 2, st, sm);
                        s->launches += 3;
                        s->arc_dots.download(h, 3, st);
                        MPHY_CUDA(cudaStreamSynchronize(st));
                        A = h[0] + dlam * dlam * FtF - ds * ds;
                        b = 2.0 * dlam * FtF;
                        adu2 = -2.0 * h[1];
                        adu1 = 2.0 * h[2];
                    }
                    const double dl = (adu2 - A) / (b + adu1);
                    axpy_inplace(disp, s->x_first.p, 1.0, n, st, sm);
                    axpy_inplace(disp, s->x.p, dl, n, st, sm);
                    axpy_inplace(s->du_full.p, s->x_first.p, 1.0, n, st, sm);
                    axpy_inplace(s->du_full.p, s->x.p, dl, n, st, sm);
                    s->launches += 4;
                    lam += dl;
                    dlam += dl;
                    MPHY_CUDA(cudaEventRecord(s->ctx->ev1, st));
                    MPHY_CUDA(cudaEventSynchronize(s->ctx->ev1));
                    is.t_solve_ms = elapsed_ms(s->ctx);
                    is.krylov_its = its1 + its2;
                    is.status = st1 != MPHY_OK ? st1 : st2;
                }
                is.step = steps_done;
                is.iter = iter;
                is.rhs_norm = norm;
                is.kernel_launches = s->launches - l0;
                if (rows < max_hist) {
                    if (hist) hist[rows] = is;
                    if (hist_lambda) hist_lambda[rows] = lam;
                    ++rows;
                }
                if (done) {
                    conv = true;
                    break;
                }
            }
            if (conv) {
                if (steps_done == 1) {
                    dot_fp64(s->du_full.p, s->du_full.p, n, s->partials.p, s->counter.p, s->arc_dots.p, st, sm);
                    s->arc_dots.download(h, 1, st);
                    MPHY_CUDA(cudaStreamSynchronize(st));
                    ds = std::sqrt(h[0] + lam * lam * FtF);
                    ds_max = ds;
                    ds_min = ds / 1024.0;
                }
                lam_prev2 = lam_prev;
                lam_prev = lam;
                MPHY_CUDA(cudaMemcpyAsync(s->disp_prev2.p, s->disp_prev.p, nd * sizeof(double),
                                          cudaMemcpyDeviceToDevice, st));
                MPHY_CUDA(cudaMemcpyAsync(s->disp_prev.p, disp, nd * sizeof(double), cudaMemcpyDeviceToDevice, st));
                ds_prev = ds;
                if (conv_prev) ds = std::fmin(std::fmax(2.0 * ds, ds_min), ds_max);
                if (step_lambda && nl < max_steps_out) step_lambda[nl] = lam;
                ++nl;
                ++steps_done;
            } else {
                if (steps_done == 1) {
                    // the reference reads its arc length before the first step sets it
                    rc = MPHY_ERR_NOT_CONVERGED;
                    set_error("arc-length: the first step (a Newton solve at lambda = dt) did not converge");
                    break;
                }
                ds = std::fmax(ds * (conv_prev ? 0.5 : 0.25), ds_min);
            }
        }
        s->disp_tmp.download(disp_host, nd, st);
        MPHY_CUDA(cudaStreamSynchronize(st));
        if (n_hist) *n_hist = rows;
        if (n_steps) *n_steps = nl;
        return rc;
    });
}

// ------------------------------------------------------------------------------- learned FSAI
int mphy_gnn_param_count(void) { return GnnLayout::total; }

int mphy_gnn_create(mphy_ctx* c, const float* params, mphy_gnn** out) {
    return guarded([&] {
        MPHY_REQUIRE(c && params && out, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_CUDA(cudaSetDevice(c->device));
        auto* g = new mphy_gnn;
        try {
            g->ctx = c;
            g->device = c->device;
            g->net.init(c, params);
        } catch (...) {
            delete g;
            throw;
        }
        *out = g;
        return (int)MPHY_OK;
    });
}

int mphy_gnn_destroy(mphy_gnn* g) {
    if (!g) return MPHY_OK;
    cudaSetDevice(g->device);
    cudaDeviceSynchronize();
    delete g;
    return MPHY_OK;
}

int mphy_gnn_get_params(mphy_gnn* g, float* p) {
    return guarded([&] {
        MPHY_REQUIRE(g && p, MPHY_ERR_INVALID_ARG, "null argument");
        g->net.get_params(p);
        return (int)MPHY_OK;
    });
}

int mphy_gnn_set_params(mphy_gnn* g, const float* p) {
    return guarded([&] {
        MPHY_REQUIRE(g && p, MPHY_ERR_INVALID_ARG, "null argument");
        g->net.set_params(p);
        return (int)MPHY_OK;
    });
}

namespace {
// features of the assembled operator, forward, the Kaporin loss and (grad) the backward pass
double gnn_loss(mphy_gnn* g, mphy_solver* s, bool grad) {
    MPHY_REQUIRE(s->use_fsai, MPHY_ERR_STATE, "the solver needs pc_type MPHY_PC_FSAI or MPHY_PC_FSAI_LEARNED");
    MPHY_REQUIRE(s->state == MPHY_ASSEMBLY_OK || s->state == MPHY_FACTORISE_OK, MPHY_ERR_STATE,
                 "assemble the matrix first");
    cudaStream_t st = s->ctx->stream;
    const void* aval = s->mixed ? (const void*)s->valf.p : (const void*)s->val.p;
    g->net.build_graph(s->graph, s->pat, s->fsai, s->A, aval, s->mixed, s->mesh->fixed.p, true, st);
    if (grad) g->net.zero_grads(st);
    const double loss = g->net.run(s->graph, s->pat, s->fsai, s->A, aval, s->mixed, s->mesh->fixed.p, nullptr, grad, st);
    MPHY_CUDA(cudaStreamSynchronize(st));
    return loss;
}
}  // namespace

int mphy_gnn_loss_and_grads(mphy_gnn* g, mphy_solver* s, double* loss, float* grads) {
    return guarded([&] {
        MPHY_REQUIRE(g && s && loss, MPHY_ERR_INVALID_ARG, "null argument");
        *loss = gnn_loss(g, s, true);
        if (grads) g->net.get_grads(grads);
        return (int)MPHY_OK;
    });
}

int mphy_gnn_train_step(mphy_gnn* g, mphy_solver* s, float lr, double* loss) {
    return guarded([&] {
        MPHY_REQUIRE(g && s, MPHY_ERR_INVALID_ARG, "null argument");
        const double l = gnn_loss(g, s, true);
        g->net.adam_step(lr, 0.9f, 0.999f, 1e-8f, s->ctx->stream);
        MPHY_CUDA(cudaStreamSynchronize(s->ctx->stream));
        if (loss) *loss = l;
        return (int)MPHY_OK;
    });
}

int mphy_gnn_predict(mphy_gnn* g, mphy_solver* s, float* ms) {
    return guarded([&] {
        MPHY_REQUIRE(g && s, MPHY_ERR_INVALID_ARG, "null argument");
        MPHY_REQUIRE(s->use_fsai, MPHY_ERR_STATE, "the solver needs pc_type MPHY_PC_FSAI or MPHY_PC_FSAI_LEARNED");
        MPHY_REQUIRE(s->state == MPHY_ASSEMBLY_OK || s->state == MPHY_FACTORISE_OK, MPHY_ERR_STATE,
                     "assemble the matrix first");
        cudaStream_t st = s->ctx->stream;
        const void* aval = s->mixed ? (const void*)s->valf.p : (const void*)s->val.p;
        MPHY_CUDA(cudaEventRecord(s->ctx->ev0, st));
        g->net.build_graph(s->graph, s->pat, s->fsai, s->A, aval, s->mixed, s->mesh->fixed.p, false, st);
        const size_t nb = 9 * (size_t)s->fsai.lower().n_blocks;
        if (s->pred_blocks.n != nb) s->pred_blocks.alloc(nb);  // kept: no allocation per solve
        g->net.run(s->graph, s->pat, s->fsai, s->A, aval, s->mixed, s->mesh->fixed.p, s->pred_blocks.p, false, st);
        s->fsai.set_lower_values(s->pred_blocks.p, st);
        MPHY_CUDA(cudaEventRecord(s->ctx->ev1, st));
        MPHY_CUDA(cudaEventSynchronize(s->ctx->ev1));
        float t = 0.f;
        cudaEventElapsedTime(&t, s->ctx->ev0, s->ctx->ev1);
        if (ms) *ms = t;
        s->launches += g->net.launches + 5;
        return (int)MPHY_OK;
    });
}

int mphy_solver_attach_gnn(mphy_solver* s, mphy_gnn* g) {
    if (!s) return MPHY_ERR_INVALID_ARG;
    s->gnn = g;
    return MPHY_OK;
}
}  // extern "C"
