/*
 * mphy_solver_gpu.hpp -- SolverGpu, the C++ class a maintainer of mphyfem adds beside
 * SolverPetsc (src/mySolvers/SolverPetsc.h:16-96) so that femSolidmechanics runs its Newton step
 * on libmphy.so. Header-only; needs mphy.h and -lmphy, nothing else (no CUDA headers, no Eigen).
 *
 * Two ways in:
 *   - the reference's own call shapes, so that femSolidmechanics2.cpp needs no edits beyond
 *     creating this object: initialise(int, int, int*, int*) (SolverPetsc.h:56),
 *     zeroMtx(), assembleMatrixAndVector(row, col, Klocal, Flocal) and its (start1, start2, ...)
 *     overload (SolverPetsc.h:72-74, called once per element by femSolidmechanics2.cpp:1097),
 *     factoriseAndSolve() (-1 unless ASSEMBLY_OK, SolverPetsc.cpp:321-330). Element matrices
 *     arrive one by one from the CPU; they are buffered and scattered on the GPU in batches.
 *     Klocal / Flocal may be Eigen's MatrixXd / VectorXd or any type with (i, j) / (i) access.
 *   - the fused GPU path: calcStiffnessAndResidual(disp) evaluates and scatters every element on
 *     the GPU (femSolidmechanics2.cpp:1047-1120 in one call), and newtonIteration() is one whole
 *     iteration of solveWithNewtonRaphson's body (femSolidmechanics2.cpp:762-816).
 *
 * Errors of the library become std::runtime_error with mphy_last_error()'s message, as the
 * reference throws runtime_error; a negative Jacobian keeps the reference's message
 * "Negative Jacobian encountered" (femSolidmechanics2.cpp:1090).
 */
#ifndef MPHY_SOLVER_GPU_HPP
#define MPHY_SOLVER_GPU_HPP

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "mphy.h"

class SolverGpu {
  public:
    int currentStatus = MPHY_SOLVER_EMPTY;  // SolverEigen.h:11 enum order
    std::vector<int> assyForSoln;           // SolverPetsc::assyForSoln: free DOF -> global DOF
    std::vector<double> Fext;               // SolverPetsc::Fext, [3 n_node] (set by the caller)
    mphy_solver_opts opts;                  // setSolverAndParameters: KSPCG + PCJACOBI defaults
    int last_its = 0;                       // KSPGetIterationNumber of the last solve
    double last_norm = 0.0;

    SolverGpu() { mphy_solver_opts_default(&opts); }
    SolverGpu(const SolverGpu&) = delete;
    SolverGpu& operator=(const SolverGpu&) = delete;
    ~SolverGpu() { free(); }

    // femBase's mesh and boundary data (GeomData.NodePosOrig, elems[e]->nodeNums, MatlData: mu,
    // Kinv, Utype per material, NodeDofType flags), copied to the device. Call before initialise.
    int setMesh(int n_node, const double* xyz, int n_elem, int npe, const int* conn, const int* mat_id, int n_mat,
                const double* mats, const unsigned char* fixed, int device = 0) {
        check(mphy_ctx_create(device, &ctx_));
        check(mphy_mesh_create(ctx_, n_node, xyz, n_elem, npe, conn, mat_id, n_mat, mats, fixed, &mesh_));
        check(mphy_pattern_build(ctx_, mesh_, &pat_));  // prepareMatrixPattern on the GPU
        int32_t n_free = 0;
        int64_t nnz = 0, nb = 0, sb = 0;
        check(mphy_pattern_info(pat_, &n_free, &nnz, &nb, &sb));
        n_node_ = n_node;
        n_free_ = n_free;
        nnz_ = nnz;
        n_elem_ = n_elem;
        nsize_ = 3 * npe;
        assyForSoln.resize(n_free);
        for_assy_.resize((size_t)n_elem * nsize_);
        check(mphy_pattern_export_dofmap(pat_, assyForSoln.data(), for_assy_.data()));
        currentStatus = MPHY_PATTERN_OK;
        return 0;
    }

    // SolverPetsc::initialise(size_local, size_global, diag_nnz, offdiag_nnz) (SolverPetsc.h:56),
    // called by prepareMatrixPattern (femSolidmechanics2.cpp:414) with its own row counts. The
    // GPU pattern is already built by setMesh; the sizes and, when given, the per-row counts
    // (diag_nnz + offdiag_nnz, one process) must be the GPU pattern's. Then the solver is created.
    int initialise(int size_local, int size_global, int* diag_nnz, int* offdiag_nnz) {
        if (!pat_) throw std::runtime_error("SolverGpu::initialise: setMesh first");
        if (size_local != size_global || size_global != n_free_)
            throw std::runtime_error("SolverGpu::initialise: size " + std::to_string(size_global) +
                                     " differs from the pattern's " + std::to_string(n_free_) + " free DOFs");
        if (diag_nnz) {
            std::vector<int64_t> rowptr(n_free_ + 1);
            check(mphy_pattern_export_csr(pat_, rowptr.data(), nullptr));
            for (int i = 0; i < n_free_; ++i) {
                const int64_t want = (int64_t)diag_nnz[i] + (offdiag_nnz ? offdiag_nnz[i] : 0);
                if (rowptr[i + 1] - rowptr[i] != want)
                    throw std::runtime_error("SolverGpu::initialise: row " + std::to_string(i) +
                                             " has a different nonzero count in the GPU pattern");
            }
        }
        check(mphy_solver_create(ctx_, mesh_, pat_, &opts, &slv_));
        currentStatus = MPHY_INIT_OK;
        return 0;
    }

    int setSolverAndParameters() { return 0; }  // options live in `opts`, read by initialise

    int zeroMtx() {
        pending_.clear();
        pending_k_.clear();
        pending_f_.clear();
        check(mphy_solver_zero(slv_));
        return 0;
    }

    // SolverPetsc::assembleMatrixAndVector(row, col, Klocal, Flocal): element matrices from the
    // CPU element loop. The element is the one whose forAssyVec is `row` (the GPU pattern's
    // numbering is the reference's, so the reference's forAssyVec matches one element exactly);
    // an element with no free DOF adds nothing (PETSc ignores negative indices). Buffered.
    template <class Mat, class Vec>
    int assembleMatrixAndVector(std::vector<int>& row, std::vector<int>& col, Mat& Klocal, Vec& Flocal) {
        if (row != col) throw std::runtime_error("SolverGpu::assembleMatrixAndVector: row and col must be forAssyVec");
        if ((int)row.size() != nsize_) throw std::runtime_error("SolverGpu::assembleMatrixAndVector: wrong size");
        const int e = find_element(row);
        if (e < 0) return 0;
        pending_.push_back(e);
        for (int i = 0; i < nsize_; ++i)
            for (int j = 0; j < nsize_; ++j) pending_k_.push_back(Klocal(i, j));
        for (int i = 0; i < nsize_; ++i) pending_f_.push_back(Flocal(i));
        if ((int)pending_.size() >= kFlush) flush();
        currentStatus = MPHY_ASSEMBLY_OK;
        return 0;
    }

    // The (start1, start2, row, col, ...) overload femSolidmechanics::calcStiffnessAndResidual
    // calls with start1 = start2 = 0 (femSolidmechanics2.cpp:1097).
    template <class Mat, class Vec>
    int assembleMatrixAndVector(int start1, int start2, std::vector<int>& row, std::vector<int>& col, Mat& Klocal,
                                Vec& Flocal) {
        if (start1 != 0 || start2 != 0)
            throw std::runtime_error("SolverGpu::assembleMatrixAndVector: offsets other than 0 are not supported");
        return assembleMatrixAndVector(row, col, Klocal, Flocal);
    }

    // The fused path: every element evaluated and scattered on the GPU from the displacement
    // disp_dev (device, [3 n_node]); zeroes first.
    int calcStiffnessAndResidual(const double* disp_dev) {
        int64_t bad = -1;
        const int rc = mphy_solver_assemble(slv_, disp_dev, &bad);
        if (rc == MPHY_ERR_NEG_JACOBIAN) throw std::runtime_error("Negative Jacobian encountered");
        check(rc);
        currentStatus = MPHY_ASSEMBLY_OK;
        return 0;
    }

    // rhsVec[ii] += scale * Fext[assyForSoln[ii]] (femSolidmechanics2.cpp:785-789).
    int addExternalForces(double scale) {
        if (Fext.empty()) return 0;
        flush();
        check(mphy_solver_add_nodal_forces_host(slv_, Fext.data(), scale));
        return 0;
    }

    // VecNorm(rhsVec, NORM_2) (femSolidmechanics2.cpp:798-801).
    double rhsNorm() {
        flush();
        double n = 0.0;
        check(mphy_solver_rhs_norm(slv_, &n));
        return n;
    }

    // -1 unless ASSEMBLY_OK (SolverPetsc.cpp:321-330); a failed KSP solve is reported, not
    // thrown, as SolverPetsc::solve prints "Divergence in %d iterations" and returns 0.
    int factoriseAndSolve() {
        if (currentStatus != MPHY_ASSEMBLY_OK) {
            fprintf(stderr, "SolverGpu::factoriseAndSolve ... assemble matrix first!\n");
            return -1;
        }
        flush();
        int32_t its = 0;
        const int rc = mphy_solver_solve(slv_, &its, &last_norm);
        last_its = its;
        if (rc == MPHY_ERR_STATE) return -1;
        if (rc != MPHY_OK) fprintf(stderr, "\n Divergence in %d iterations.\n\n", its);
        currentStatus = MPHY_FACTORISE_OK;
        return 0;
    }

    // dispIncr[assyForSoln[i]] = soln[i] (femSolidmechanics2.cpp:1183-1186): [3 n_node] host.
    void getSolution(std::vector<double>& dispIncr) {
        dispIncr.resize(3 * (size_t)n_node_);
        check(mphy_solver_get_solution_host(slv_, dispIncr.data()));
    }

    // One iteration of the Newton body on host displacements: assemble, rhs += lambda Fext, norm,
    // solve, disp += dispIncr. Returns the residual norm before the update.
    double newtonIteration(std::vector<double>& disp, double lambda) {
        mphy_iter_stats st{};
        const int rc = mphy_newton_iteration_host(slv_, disp.data(), Fext.empty() ? nullptr : Fext.data(), lambda, 0.0,
                                                  &st);
        if (rc == MPHY_ERR_NEG_JACOBIAN) throw std::runtime_error("Negative Jacobian encountered");
        if (rc != MPHY_OK && rc != MPHY_ERR_NOT_CONVERGED && rc != MPHY_ERR_INDEFINITE) check(rc);
        last_its = st.krylov_its;
        return st.rhs_norm;
    }

    int free() {
        if (slv_) mphy_solver_destroy(slv_);
        if (pat_) mphy_pattern_destroy(pat_);
        if (mesh_) mphy_mesh_destroy(mesh_);
        if (ctx_) mphy_ctx_destroy(ctx_);
        slv_ = nullptr;
        pat_ = nullptr;
        mesh_ = nullptr;
        ctx_ = nullptr;
        currentStatus = MPHY_SOLVER_EMPTY;
        return 0;
    }

    int freeDofCount() const { return n_free_; }
    int64_t nonzeroCount() const { return nnz_; }
    const std::vector<int32_t>& forAssyVec() const { return for_assy_; }  // [n_elem][3 npe]
    mphy_solver* handle() const { return slv_; }

  private:
    static constexpr int kFlush = 16384;  // element matrices buffered before a GPU scatter
    mphy_ctx* ctx_ = nullptr;
    mphy_mesh* mesh_ = nullptr;
    mphy_pattern* pat_ = nullptr;
    mphy_solver* slv_ = nullptr;
    int n_node_ = 0, n_free_ = 0, n_elem_ = 0, nsize_ = 0;
    int64_t nnz_ = 0;
    std::vector<int32_t> for_assy_;
    std::unordered_multimap<uint64_t, int> by_row_;  // hash of forAssyVec -> element
    std::vector<int32_t> pending_;
    std::vector<double> pending_k_, pending_f_;

    static void check(int rc) {
        if (rc != MPHY_OK) throw std::runtime_error(std::string("libmphy: ") + mphy_last_error());
    }

    static uint64_t hash_row(const int* r, int n) {
        uint64_t h = 1469598103934665603ull;
        for (int i = 0; i < n; ++i) h = (h ^ (uint64_t)(uint32_t)r[i]) * 1099511628211ull;
        return h;
    }

    int find_element(const std::vector<int>& row) {
        bool any = false;
        for (int v : row) any |= v >= 0;
        if (!any) return -1;
        if (by_row_.empty())
            for (int e = 0; e < n_elem_; ++e) by_row_.emplace(hash_row(&for_assy_[(size_t)e * nsize_], nsize_), e);
        auto range = by_row_.equal_range(hash_row(row.data(), nsize_));
        for (auto it = range.first; it != range.second; ++it) {
            const int32_t* f = &for_assy_[(size_t)it->second * nsize_];
            bool same = true;
            for (int i = 0; i < nsize_ && same; ++i) same = f[i] == row[i];
            if (same) return it->second;
        }
        throw std::runtime_error("SolverGpu::assembleMatrixAndVector: forAssyVec matches no element of the mesh");
    }

    void flush() {
        if (pending_.empty()) return;
        check(mphy_solver_assemble_batch_host(slv_, (int32_t)pending_.size(), pending_.data(), pending_k_.data(),
                                              pending_f_.data()));
        pending_.clear();
        pending_k_.clear();
        pending_f_.clear();
    }
};

#endif  // MPHY_SOLVER_GPU_HPP
