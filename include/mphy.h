/*
 * mphy.h -- C ABI of libmphy.so, the B200 (sm_100a) implementation of mphyfem's
 * femSolidmechanics Newton-step hot path.
 *
 * Every entry point replaces one interface of the reference (paths relative to the
 * chennachaos/mphyfem source tree); the comment above each declaration names it.
 * Plain C types only: pointers, sizes, status codes. Arguments named *_dev are device
 * pointers on the context's device; *_host are host pointers. Calls on one context are
 * ordered on its CUDA stream; a context must be used by one host thread at a time. Meshes,
 * patterns and solvers may be destroyed in any order, before or after their context; no other
 * call may use an object after its context is destroyed.
 *
 * Layout conventions shared with the reference:
 *   - node-major DOF vectors: dof = 3*node + dim          (ElementBase.cpp:46-69)
 *   - element DOF order 3*local_node + dim; element matrices row-major [3npe][3npe]
 *   - 9-index of the material call: {(0,0),(1,0),(2,0),(0,1),(1,1),(2,1),(0,2),(1,2),(2,2)}
 *     (utilitiesmaterialHyperelastic.cpp:192)
 *   - free DOFs numbered node-major skipping prescribed ones (femSolidmechanics2.cpp:142-165)
 */
#ifndef MPHY_H
#define MPHY_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPHY_API_VERSION 1

typedef enum mphy_status {
    MPHY_OK = 0,
    MPHY_ERR_INVALID_ARG = 1,
    MPHY_ERR_CUDA = 2,
    MPHY_ERR_NO_DEVICE = 3,
    MPHY_ERR_OUT_OF_MEMORY = 4,
    MPHY_ERR_UNSUPPORTED = 5,
    /* call out of order; SolverPetsc::factoriseAndSolve returns -1 unless ASSEMBLY_OK
     * (SolverPetsc.cpp:321-330) */
    MPHY_ERR_STATE = 6,
    /* det F < 0 at a Gauss point; the reference throws (Elem_Solid_3D_Disp.cpp:275-278) */
    MPHY_ERR_NEG_JACOBIAN = 7,
    /* Krylov iteration limit reached (KSP_DIVERGED_ITS) */
    MPHY_ERR_NOT_CONVERGED = 8,
    /* p.Ap <= 0 met by CG (KSP_DIVERGED_INDEFINITE_MAT) */
    MPHY_ERR_INDEFINITE = 9,
    /* NaN residual or divergence-tolerance exceeded */
    MPHY_ERR_DIVERGED = 10,
    /* load step cut below 1% of the initial step (MyTime.cpp:41-58) */
    MPHY_ERR_TIME_STEP = 11
} mphy_status;

/* SolverEigen.h:11 status enum, mirrored for mphy_solver_state */
enum { MPHY_SOLVER_EMPTY = 0, MPHY_PATTERN_OK = 1, MPHY_INIT_OK = 2, MPHY_ASSEMBLY_OK = 3,
       MPHY_FACTORISE_OK = 4 };

/* arithmetic of the tangent and of the Krylov solve */
enum { MPHY_PREC_FP64 = 0,        /* FP64 element kernel, FP64 matrix, FP64 PCG (plain method) */
       MPHY_PREC_MIXED = 1,       /* FP32 tangent and matrix values; Krylov vectors, dot products,
                                   * residual and the iterative-refinement outer loop in FP64 */
       MPHY_PREC_MIXED_F32VEC = 2,/* as MIXED, with FP32 Krylov vectors (FP64 reductions) */
       MPHY_PREC_MIXED_TC = 3     /* as MIXED, with the element tangent's contraction on tensor
                                   * cores: split-BF16 operands, FP32 accumulation (about 1e-5
                                   * relative per entry); kinematics, stress and residual FP64 */ };
/* preconditioner (PCJACOBI, or factorised sparse approximate inverse M = G^T G) */
enum { MPHY_PC_JACOBI = 0, MPHY_PC_FSAI = 1, MPHY_PC_FSAI_LEARNED = 2 };
/* MPHY_TANGENT_REFERENCE reproduces utilitiesmaterialHyperelastic.cpp:232-292 exactly
 * (volumetric part without its geometric stress term); MPHY_TANGENT_CONSISTENT adds that
 * term, giving the exact derivative of the residual. */
enum { MPHY_TANGENT_REFERENCE = 0, MPHY_TANGENT_CONSISTENT = 1 };

typedef struct mphy_ctx mphy_ctx;
typedef struct mphy_mesh mphy_mesh;
typedef struct mphy_pattern mphy_pattern;
typedef struct mphy_solver mphy_solver;
typedef struct mphy_gnn mphy_gnn;

typedef struct mphy_solver_opts {
    int32_t precision;     /* MPHY_PREC_* */
    int32_t pc_type;       /* MPHY_PC_* */
    int32_t tangent;       /* MPHY_TANGENT_* */
    int32_t max_it;        /* KSP max_it (PETSc default 10000) */
    double rtol;           /* KSP rtol on the preconditioned residual norm */
    double abstol;         /* KSP abstol (PETSc default 1e-50) */
    double dtol;           /* KSP dtol (PETSc default 1e5) */
    double inner_rtol;     /* MIXED*: inner PCG rtol per refinement sweep (<= 0: rtol for the
                            * first sweep, then what the sweep must remove to reach rtol ||b||
                            * with a factor 2 to spare, capped at 0.5) */
    int32_t max_outer;     /* refinement sweeps, each ending with the FP64 residual b - A x
                            * (FP64 path too: against the drift of the CG recurrence residual);
                            * stops early once ||b - A x|| <= rtol ||b|| (default 1: the KSP
                            * solve alone, PETSc's behaviour) */
    int32_t chunk;         /* Krylov iterations per launched graph between host checks (0: auto) */
    int32_t coarse_aggregates; /* > 0: add the two-level rigid-body coarse correction
                                * M^{-1} = D^{-1} + Z (Z^T A Z)^{-1} Z^T over about this many
                                * geometric aggregates (6 modes each) to the local
                                * preconditioner (Jacobi: D^{-1}, FSAI: G^T G); the coarse
                                * inverse is applied as W^T W with W the inverse Cholesky
                                * factor rounded to FP32 (still SPD); about one
                                * aggregate per 1,300 nodes was the measured optimum on the
                                * 1.1 M-node hex8 and 1.8 M-node tet10 cantilevers */
    int32_t norm_type;     /* KSP norm of the convergence test: 0 = preconditioned ||z|| (PETSc's
                            * CG default), 1 = unpreconditioned ||r|| (true residual vs ||b||) */
    int32_t coarse_modes;  /* modes per aggregate of the coarse correction: 6 (0 = default:
                            * translations and rotations about the aggregate's centroid) or 12
                            * (linear displacement u = a + B (x - x_c): translations, stretches,
                            * shears and rotations; a richer space of the same size at half the
                            * aggregates) */
    int32_t coarse_lag;    /* > 0: the coarse operator (Z^T A Z)^{-1} formed by a solve is kept for
                            * up to this many further solves instead of being rebuilt from each
                            * new matrix; mphy_newton_run rebuilds it at the first iteration of
                            * every load step. The preconditioner lags, the convergence test does
                            * not. 0 (default): rebuilt for every new matrix, as PCSetUp is. */
} mphy_solver_opts;

typedef struct mphy_newton_opts {
    double dt;             /* Solver block timeStep */
    double t_final;        /* finalTime */
    int32_t max_steps;     /* maximumSteps */
    int32_t max_newton;    /* maximumIterations (femBase.cpp:57 default 10) */
    double tol_rel;        /* converged when ||R|| < max(tol_abs, tol_rel * ||R||_first) */
    double tol_abs;        /* the reference's absolute `tolerance` (femSolidmechanics1.cpp:616-622) */
} mphy_newton_opts;

/* One Newton iteration's statistics (femSolidmechanics2.cpp:803 prints the norm). */
typedef struct mphy_iter_stats {
    int32_t step, iter, krylov_its, status;
    double rhs_norm;
    double t_assembly_ms, t_solve_ms;
    int64_t kernel_launches;   /* libmphy kernels launched by this iteration */
} mphy_iter_stats;

const char* mphy_status_string(int status);
/* Message of the last failing call on this host thread. */
const char* mphy_last_error(void);
int mphy_api_version(void);

/* ---- context (replaces PetscInitialize + the MPI/PETSc communicator, femSolidmechanics.cpp:49) */
int mphy_ctx_create(int device, mphy_ctx** out);
int mphy_ctx_destroy(mphy_ctx* ctx);
int mphy_ctx_synchronize(mphy_ctx* ctx);
void* mphy_ctx_stream(mphy_ctx* ctx); /* the cudaStream_t all calls are ordered on */

/* ---- mesh: femBase::readInput's node/element/material/BC data, held on the device
 * (femBase.cpp:121-364, 571-614, 944-989; prescribed DOFs from setSpecifiedDOFs_Displacement,
 * femSolidmechanics1.cpp:1479-1543). mats: [n_mat][3] = {mu, Kinv, Utype} per material
 * (MaterialBase.cpp:91-116). fixed: [3*n_node], 1 = prescribed zero displacement.
 * npe: 8 (hex8) or 10 (tet10). All inputs are host pointers, copied. */
int mphy_mesh_create(mphy_ctx* ctx, int32_t n_node, const double* coords_host, int32_t n_elem,
                     int32_t npe, const int32_t* conn_host, const int32_t* mat_id_host,
                     int32_t n_mat, const double* mats_host, const uint8_t* fixed_host,
                     mphy_mesh** out);
int mphy_mesh_destroy(mphy_mesh* mesh);

/* Nonzero prescribed displacements ("specified" boundary conditions, femSolidmechanics1.cpp:813-891):
 * the DOFs flagged in `fixed` take t * ramp_host[i] + const_host[i] at time t of the load stepping
 * (a boundary condition with the time function lam = t, and one without a time function, which the
 * reference applies in full from the first step). Host arrays [3*n_node], either may be NULL (zero);
 * entries of free DOFs are ignored; all-zero values return the mesh to clamped DOFs. mphy_newton_run
 * lifts each step's increment dispApplied = value(t) - disp into the first iteration's right-hand
 * side (ElementBase::applyDirichletBCs, ElementBase.cpp:567-594) and adds it to the displacement
 * with that iteration's solution (femSolidmechanics2.cpp:1137-1145). Not available with the
 * MPHY_PREC_MIXED_TC tangent, the two-field mixed element, arc-length or the batched form. */
int mphy_mesh_set_prescribed(mphy_mesh* mesh, const double* ramp_host, const double* const_host);

/* ---- hyperelastic models (the compressible branch of utilitiesmaterialHyperelastic.cpp) and
 * their deviatoric parameters, as the reference's material blocks give them:
 *   MPHY_MAT_NEOHOOKEAN   Matl_NeoHookean    data_deviatoric : mu          (:186-295)
 *   MPHY_MAT_MOONEYRIVLIN Matl_MooneyRivlin  data_deviatoric : c1 c2       (:300-420)
 *   MPHY_MAT_GENT         Matl_Gent          data_deviatoric : mu Im       (:423-548)
 *   MPHY_MAT_ARRUDABOYCE  Matl_ArrudaBoyce   data            : mu N        (:551-677)
 * Each takes the volumetric energy Utype and Kinv = 1/K of data_volumetric.
 * Tangent modes: MPHY_TANGENT_REFERENCE gives each model's tangent as the reference writes it.
 * MPHY_TANGENT_CONSISTENT gives the exact derivative of the residual for Neo-Hookean, Gent and
 * Arruda-Boyce (whose reference tangent is a symmetrised form). Mooney-Rivlin keeps the written
 * tangent in both modes: the reference's stress carries J^{-5/3} where J^{-7/3} belongs (r7d3 =
 * 5/3, :303), and its exact derivative is not symmetric. */
enum { MPHY_MAT_NEOHOOKEAN = 0, MPHY_MAT_MOONEYRIVLIN = 1, MPHY_MAT_GENT = 2, MPHY_MAT_ARRUDABOYCE = 3 };
enum { MPHY_MAT_NDATA = 4 };

/* Sets the model and parameters of every material of the mesh (the Matl_* object that
 * MaterialBase's factory makes per material id). model: [n_mat] MPHY_MAT_*; data: [n_mat][4],
 * the model's parameters above, unused slots ignored. Kinv and Utype stay those of
 * mphy_mesh_create. n_mat must equal the mesh's; Gent needs Im > 0 and Arruda-Boyce N > 0
 * (MPHY_ERR_INVALID_ARG otherwise). Without this call every material is Neo-Hookean with mu =
 * mats[3k]. A mesh with any model other than Neo-Hookean assembles with the dense-tangent
 * element kernel (FP64; FP32 storage in the mixed precisions, MPHY_PREC_MIXED_TC included, whose
 * tensor-core kernel is Neo-Hookean only), and mphy_elem_eval_tc returns MPHY_ERR_UNSUPPORTED for
 * it. Host pointers, copied; affects assemblies issued after the call. */
int mphy_mesh_set_materials(mphy_mesh* mesh, int32_t n_mat, const int32_t* model_host, const double* data_host);

/* Batched stress and tangent of any model above at n deformation gradients (the material
 * contract of MaterialBase::computeStressAndTangent). data_host: [4]. Device arrays as in
 * mphy_material_nh_eval. */
int mphy_material_eval(mphy_ctx* ctx, int32_t n, const double* F_dev, int32_t model, const double* data_host,
                       double Kinv, int32_t utype, int32_t tangent, double* stre_dev, double* cmat_dev);

/* ---- material contract: MaterialBase::computeStressAndTangent (MaterialBase.h:94), Neo-Hookean
 * (Matl_NeoHookean.cpp:45-53 -> utilitiesmaterialHyperelastic.cpp:186-295), batched.
 * F_dev: [n][9] row-major F(i,j); stre_dev: [n][9]; cmat_dev: [n][81] row-major. */
int mphy_material_nh_eval(mphy_ctx* ctx, int32_t n, const double* F_dev, double mu, double Kinv,
                          int32_t utype, int32_t tangent, double* stre_dev, double* cmat_dev);

/* ---- element contract: ElementBase::calcStiffnessAndResidual (ElementBase.h:149, implemented by
 * Elem_Solid_3D_Disp.cpp:196-373), batched over every element of the mesh.
 * disp_dev: [3*n_node]. Ke_dev: [n_elem][3npe][3npe] row-major, Re_dev: [n_elem][3npe] (= -f_int).
 * *first_bad (host) receives the lowest element id with det F < 0, or -1; the call then returns
 * MPHY_ERR_NEG_JACOBIAN. */
int mphy_elem_eval(mphy_ctx* ctx, const mphy_mesh* mesh, const double* disp_dev, int32_t tangent,
                   double* Ke_dev, double* Re_dev, int64_t* first_bad);
/* The same contract computed by the MPHY_PREC_MIXED_TC element kernel: residual in FP64, tangent
 * contracted on tensor cores (split-BF16, FP32 accumulation), widened to FP64 on export. */
int mphy_elem_eval_tc(mphy_ctx* ctx, const mphy_mesh* mesh, const double* disp_dev, int32_t tangent,
                      double* Ke_dev, double* Re_dev, int64_t* first_bad);

/* Allocation-free variant of mphy_elem_eval for callers that cannot let the library call
 * cudaMalloc (their mesh already lives in device memory under their own arena allocator, or they
 * run under a no-allocation policy). No counterpart in the reference: it is the same element
 * evaluation taking the caller's device arrays directly -- coords_dev [n_node][3], conn_dev
 * [n_elem][npe], mat_id_dev [n_elem], mats_dev [n_mat][3] = {mu, Kinv, Utype}, disp_dev
 * [3*n_node] -- and writing Ke_dev / Re_dev as mphy_elem_eval does. Ids out of range and rows
 * with Kinv <= 0 return MPHY_ERR_INVALID_ARG. Its scratch is a fixed ~32 KB device array inside
 * libmphy.so (held by every GPU that loads it until exit), so n_mat is limited to 1024 (larger
 * values return MPHY_ERR_INVALID_ARG). The first call on a device looks up that array's device
 * address; make that first call before any stream capture. Every call blocks the calling host
 * thread until its result is ready (it synchronises the context's stream). Calls share the
 * scratch: calls that overlap on the GPU race and must be serialised by the caller. */
int mphy_elem_eval_noalloc(mphy_ctx* ctx, int32_t n_node, const double* coords_dev, int32_t n_elem,
                           int32_t npe, const int32_t* conn_dev, const int32_t* mat_id_dev,
                           int32_t n_mat, const double* mats_dev, const double* disp_dev,
                           int32_t tangent, double* Ke_dev, double* Re_dev, int64_t* first_bad);

/* ---- DOF map and sparsity: femSolidmechanics::prepareMatrixPattern (femSolidmechanics2.cpp:121-478),
 * built on the device. */
int mphy_pattern_build(mphy_ctx* ctx, const mphy_mesh* mesh, mphy_pattern** out);
int mphy_pattern_info(const mphy_pattern* pat, int32_t* n_free, int64_t* nnz, int64_t* n_blocks,
                      int64_t* stored_blocks);
/* CSR over free DOFs, rows sorted ascending (findUnique, util.h:41-45): rowptr [n_free+1], col [nnz]. */
int mphy_pattern_export_csr(const mphy_pattern* pat, int64_t* rowptr_host, int32_t* col_host);
/* assyForSoln [n_free] (femSolidmechanics2.cpp:155-165); forAssyVec [n_elem][3npe] (:248-280). */
int mphy_pattern_export_dofmap(const mphy_pattern* pat, int32_t* assy_for_soln_host,
                               int32_t* for_assy_vec_host);
int mphy_pattern_destroy(mphy_pattern* pat);

/* ---- solver surface: SolverPetsc (SolverPetsc.h:16-96) -------------------------------------- */
void mphy_solver_opts_default(mphy_solver_opts* opts);
/* initialise + setSolverAndParameters (SolverPetsc.cpp:33-140). */
int mphy_solver_create(mphy_ctx* ctx, const mphy_mesh* mesh, const mphy_pattern* pat,
                       const mphy_solver_opts* opts, mphy_solver** out);
int mphy_solver_destroy(mphy_solver* s);
int mphy_solver_get_state(const mphy_solver* s, int32_t* state);
/* zeroMtx (SolverPetsc.cpp:145-163): matrix, right-hand side and reactions to zero. */
int mphy_solver_zero(mphy_solver* s);
/* femSolidmechanics::calcStiffnessAndResidual (femSolidmechanics2.cpp:1047-1120): every element's
 * calcStiffnessAndResidual fused with the ADD_VALUES scatter of assembleMatrixAndVector
 * (SolverPetsc.cpp:357-378) and the reaction sum (:1106-1111). Zeroes first. Leaves ASSEMBLY_OK. */
int mphy_solver_assemble(mphy_solver* s, const double* disp_dev, int64_t* first_bad);
/* SolverPetsc::assembleMatrixAndVector for caller-supplied element matrices: element e scatters
 * Ke_dev[e] / Re_dev[e] through forAssyVec of element elem_ids[e] (all elements when elem_ids is
 * NULL; then n must equal n_elem). Adds to the current matrix; leaves ASSEMBLY_OK. */
int mphy_solver_assemble_batch(mphy_solver* s, int32_t n, const int32_t* elem_ids_dev,
                               const double* Ke_dev, const double* Re_dev);
/* The same with host arrays, for a caller that forms element matrices on the CPU one by one
 * (SolverPetsc::assembleMatrixAndVector(row, col, Klocal, Flocal), SolverPetsc.h:72-74, called
 * once per element by femSolidmechanics2.cpp:1097): elem_ids_host [n] (NULL: 0..n-1, n = n_elem),
 * Ke_host [n][3npe][3npe] row-major, Re_host [n][3npe]. Copied to the device in chunks;
 * ids outside [0, n_elem) return MPHY_ERR_INVALID_ARG. */
int mphy_solver_assemble_batch_host(mphy_solver* s, int32_t n, const int32_t* elem_ids_host,
                                    const double* Ke_host, const double* Re_host);
/* rhs += scale * Fext[assyForSoln] (femSolidmechanics2.cpp:785-789); fext_dev: [3*n_node]. */
int mphy_solver_add_nodal_forces(mphy_solver* s, const double* fext_dev, double scale);
/* The same with a host array, the reference's VecSetValue(rhsVec, ii, Fext[assyForSoln[ii]],
 * ADD_VALUES) loop (femSolidmechanics2.cpp:785-789) with Fext in host memory. */
int mphy_solver_add_nodal_forces_host(mphy_solver* s, const double* fext_host, double scale);
/* VecNorm(rhsVec, NORM_2) in FP64 (femSolidmechanics2.cpp:798-801). */
int mphy_solver_rhs_norm(mphy_solver* s, double* norm_host);
/* factoriseAndSolve (SolverPetsc.cpp:250-330): KSPSolve from x = 0. Returns MPHY_ERR_STATE unless
 * ASSEMBLY_OK; *its and *final_norm (preconditioned residual norm) on exit. */
int mphy_solver_solve(mphy_solver* s, int32_t* its, double* final_norm);
/* y = A x with the assembled matrix (MatMult), x_dev / y_dev: [3*n_node] FP64. */
int mphy_solver_spmv(mphy_solver* s, const double* x_dev, double* y_dev);
/* y = A x and (x, y) in one pass (MatMult followed by VecDot): the SpMV kernel that the CG
 * iteration runs. *xy_host (may be NULL: no copy and no host wait) receives (x, y). */
int mphy_solver_spmv_dot(mphy_solver* s, const double* x_dev, double* y_dev, double* xy_host);
/* Sizes of the assembled operator: stored 3x3 blocks (with padding), true blocks, value bytes. */
int mphy_solver_matrix_info(const mphy_solver* s, int64_t* stored_blocks, int64_t* true_blocks,
                            int64_t* value_bytes);
/* ---- factorised preconditioner M = G^T G (MPHY_PC_FSAI, MPHY_PC_FSAI_LEARNED). No counterpart
 * in the reference, whose PC comes from PETSc options (SolverPetsc.cpp:117-140). G is lower
 * block-triangular on the matrix's lower block pattern: block row n holds the neighbour nodes
 * m <= n ascending (n last, at most 16 blocks). Blocks are 3x3 row-major FP32. */
/* Lower pattern: rowptr [n_node+1], col [n_lower_blocks]. Either pointer may be NULL. */
int mphy_solver_pc_pattern(mphy_solver* s, int64_t* n_lower_blocks, int64_t* rowptr_host, int32_t* col_host);
/* Current G blocks in pattern order, [n_lower_blocks][9] FP32 device memory. With MPHY_PC_FSAI
 * they are the exact block FSAI of the last solved operator (or of the assembled one after
 * mphy_solver_pc_setup). */
int mphy_solver_pc_get_blocks(mphy_solver* s, float* blocks_dev);
/* Install G blocks (MPHY_PC_FSAI_LEARNED: the next solves use them as they are). */
int mphy_solver_pc_set_blocks(mphy_solver* s, const float* blocks_dev);
/* Exact block FSAI of the currently assembled operator; *n_fallback rows were not positive
 * definite and use the inverse square root of their diagonal. */
int mphy_solver_pc_setup(mphy_solver* s, int32_t* n_fallback);
/* ---- learned factorised preconditioner (MPHY_PC_FSAI_LEARNED). No counterpart in the reference.
 * A message-passing network (3 layers of width 64, BF16 weights, FP32 accumulation) predicts the
 * blocks of G from the Jacobi-scaled operator; it is trained on the GPU against the exact block
 * FSAI of operators the solver assembles. Parameters: a flat FP32 vector of
 * mphy_gnn_param_count() values. */
int mphy_gnn_param_count(void);
int mphy_gnn_create(mphy_ctx* ctx, const float* params_host, mphy_gnn** out);
int mphy_gnn_destroy(mphy_gnn* g);
int mphy_gnn_get_params(mphy_gnn* g, float* params_host);
int mphy_gnn_set_params(mphy_gnn* g, const float* params_host);
/* Loss and its gradient on the solver's assembled operator, without changing the parameters;
 * grads_host may be NULL. The loss is Kaporin's condition number of the preconditioned operator,
 * log( tr(G A G^T) / N ) - (2/N) sum_n log|det G_nn| in the Jacobi-scaled units (N = 3 n_node),
 * whose minimiser over the pattern is the exact block FSAI; it needs no target. */
int mphy_gnn_loss_and_grads(mphy_gnn* g, mphy_solver* s, double* loss, float* grads_host);
/* One Adam step on the solver's assembled operator; *loss before the step. */
int mphy_gnn_train_step(mphy_gnn* g, mphy_solver* s, float lr, double* loss);
/* Predict G for the solver's assembled operator and install it (then solves use it). */
int mphy_gnn_predict(mphy_gnn* g, mphy_solver* s, float* ms);
/* With MPHY_PC_FSAI_LEARNED, run the network before every solve (NULL detaches). Such solves stop
 * on the true residual (norm_type 1) and are accepted only with ||b - A x|| <= 100 rtol ||b|| in
 * FP64; otherwise they are repeated with the Jacobi local part (see mphy_solver_pc_last). */
int mphy_solver_attach_gnn(mphy_solver* s, mphy_gnn* g);
/* Last solve: *fallback = 1 when a learned preconditioner failed the FP64 true-residual check and
 * the solve was repeated with the Jacobi local part; *setup_ms = the local preconditioner's setup
 * time (exact FSAI or network inference; the coarse operator's is in mphy_solver_coarse_info);
 * first_*: status, iterations and true relative
 * residual of the learned attempt. Any pointer may be NULL. */
int mphy_solver_pc_last(const mphy_solver* s, int32_t* fallback, float* setup_ms, int32_t* first_status,
                        int32_t* first_its, double* first_relres);
/* Coarse space of the two-level correction: aggregate grid (boxes along x, y, z of the reference
 * bounding box) and coarse size (6 modes per box). *setup_ms: time of the E setup done by the
 * last solve (0 when it kept an earlier operator under coarse_lag).
 * No counterpart in the reference. */
int mphy_solver_coarse_info(const mphy_solver* s, int32_t* grid3, int32_t* coarse_size, float* setup_ms);
/* ||b - A x|| / ||b|| in FP64 for the last solve (A as stored: FP64, or the FP32 storage). */
int mphy_solver_true_residual(mphy_solver* s, double* relres);
/* Solution increment scattered to node-major layout (femSolidmechanics2.cpp:1183-1186):
 * dx_dev[assyForSoln[i]] = soln[i], prescribed DOFs 0. */
int mphy_solver_get_solution(mphy_solver* s, double* dx_dev);
/* The same into host memory (solnVec read back by factoriseSolveAndUpdate). */
int mphy_solver_get_solution_host(mphy_solver* s, double* dx_host);
/* disp_dev += solution (the update `SolnData.disp += SolnData.dispIncr`). */
int mphy_solver_update_disp(mphy_solver* s, double* disp_dev);
/* ---- constant-pressure mixed element: Elem_Solid_3D_Mixed0 (Elem_Solid_3D_Mixed0.cpp), hex8 or
 * tet10 displacement with one pressure per element, condensed in every element
 * (calcStiffnessAndResidual, :93-101), the element pressures updated after every solve
 * (solveForPressure, :112-200, called by factoriseSolveAndUpdate, femSolidmechanics2.cpp:1204-1212)
 * and, in mphy_newton_run, saved with each converged step and restored by a cut. The materials
 * take their mixed branch (the pressure replaces U'(J)); Utype -1 is refused (Kpp = 0).
 * enable = 1 turns it on for every later assembly with zero pressures and zero last-step
 * displacement; 0 turns it off. Not available with arc-length. */
int mphy_solver_set_mixed_p0(mphy_solver* s, int32_t enable);
/* Element pressures [n_elem], host: set_host (may be NULL) is copied in first, then get_host (may
 * be NULL) receives them. */
int mphy_solver_p0_pressure(mphy_solver* s, const double* set_host, double* get_host);
/* SolutionDataSolid::saveSolution for callers that drive mphy_newton_iteration themselves: disp_dev
 * becomes the last converged step (its J is the mixed element's Jn), with the element pressures. */
int mphy_solver_save_step(mphy_solver* s, const double* disp_dev);
/* Copies for checks: CSR values in mphy_pattern_export_csr order [nnz], rhs over free DOFs
 * [n_free], reactions [3*n_node]. Any pointer may be NULL. FP64 regardless of precision. */
int mphy_solver_export(mphy_solver* s, double* val_host, double* rhs_host, double* reac_host);

/* ---- Newton driver: femSolidmechanics::solveWithNewtonRaphson (femSolidmechanics2.cpp:730-851) ---- */
/* One Newton iteration at load factor lambda on device data: assemble, rhs += lambda*fext, norm,
 * and (unless the norm is already below tol_abs) solve and update disp_dev. */
int mphy_newton_iteration(mphy_solver* s, double* disp_dev, const double* fext_dev, double lambda,
                          double tol_abs, mphy_iter_stats* stats);
/* The same iteration with host buffers: disp_host is copied in, updated and copied back. */
int mphy_newton_iteration_host(mphy_solver* s, double* disp_host, const double* fext_host,
                               double lambda, double tol_abs, mphy_iter_stats* stats);
/* Full load stepping with cuts. fext_host: [3*n_node] nodal forces at lambda = 1 (lambda(t) = t);
 * disp_host in/out. hist_host: [max_hist] rows; *n_hist rows written. */
int mphy_newton_run(mphy_solver* s, const double* fext_host, const mphy_newton_opts* opts,
                    double* disp_host, mphy_iter_stats* hist_host, int32_t max_hist,
                    int32_t* n_hist);

/* ---- arc-length continuation: femSolidmechanics::solveWithArclength (femSolidmechanics2.cpp:855-1039)
 * with SolverPetsc::solveArclengthSystem (SolverPetsc.cpp:671-757), psi = 1.
 * opts: dt = the first step's load factor (loadFactor = myTime.dt) and the time increment of every
 * attempt; t_final; max_steps = converged steps; max_newton = iterationsMax (iterations
 * 1..max_newton-1 per step, the reference's bound); converged when ||R|| < max(tol_abs,
 * tol_rel ||R||_first of the step) (the reference: tol_abs = tolerance, tol_rel = 0).
 * Per iteration: assemble, R += lambda F, then two solves on the one assembled K (x1 = K^-1 R,
 * x2 = K^-1 F; the preconditioner is set up once), dl from the linearised spherical constraint
 * (Du.Du + Dl^2 F.F = Ds^2; dl = 0 in the first step, a Newton solve at lambda = dt), disp +=
 * x1 + dl x2, lambda += dl. Steps after the first start from the extrapolation of the two last
 * converged steps. Ds after the first step is sqrt(Du.Du + lambda^2 F.F), bounded to
 * [Ds/1024, Ds]; doubled after two converged steps in a row; halved on a failure after a
 * converged step, quartered after a failed one.
 * fext_host, disp_host (in/out): [3*n_node]. step_lambda_host: load factor of each converged
 * step [max_steps_out]; hist_host / hist_lambda_host: one row and the load factor after the
 * update per iteration [max_hist] (either may be NULL). Returns MPHY_ERR_NOT_CONVERGED when the
 * first step does not converge (the reference would go on with an unset arc length). */
int mphy_arclength_run(mphy_solver* s, const double* fext_host, const mphy_newton_opts* opts,
                       double* disp_host, double* step_lambda_host, int32_t max_steps_out,
                       int32_t* n_steps, mphy_iter_stats* hist_host, double* hist_lambda_host,
                       int32_t max_hist, int32_t* n_hist);

/* ---- mixed u-p elements: Elem_Solid_3D_Mixed1 with npElem = 10 (tet10 displacement, linear
 * pressure on the vertex nodes), ElementBase::calcStiffnessAndResidualMixed3D
 * (ElementBase2.cpp:278-553), STATIC scheme, every material model above through its mixed
 * branch. Pressure DOFs: the vertex nodes in ascending node order (prepareDataForMixedElements,
 * femSolidmechanics1.cpp:274-380), no prescribed pressures. The two-field vectors are
 * [3 n_node displacements | n_pres pressures]; prescribed displacement rows and columns are
 * left out of the coupling blocks and hold identity rows in Kuu (SolverPetsc.cpp:434-502 leaves
 * them out of the matrix). The solve is preconditioned MINRES (the reference's sample inputs run
 * MUMPS LU): relative tolerance rtol on the preconditioned residual, at most max_it iterations. */
typedef struct mphy_mixed mphy_mixed;
typedef struct mphy_mixed_opts {
    int32_t tangent;            /* MPHY_TANGENT_* */
    int32_t max_it;             /* MINRES iterations per solve */
    double rtol;                /* MINRES relative tolerance */
    int32_t coarse_aggregates;  /* > 0: the displacement block of the preconditioner adds the
                                 * coarse space over about this many aggregates */
    int32_t coarse_modes;       /* 6 (0 = default) or 12, as in mphy_solver_opts */
} mphy_mixed_opts;
void mphy_mixed_opts_default(mphy_mixed_opts* opts); /* reference tangent, 20000, 1e-10, 0 */
/* Elem_Solid_3D_Mixed1 meshes: tet10 (npe = 10, linear pressure on the 4 vertices) or the P2-P1
 * hex27 (npe = 27, trilinear pressure on the 8 corners; 3x3x3 rule); pattern: mphy_pattern_build
 * of the same mesh. opts may be NULL. */
int mphy_mixed_create(mphy_ctx* ctx, const mphy_mesh* mesh, const mphy_pattern* pattern,
                      const mphy_mixed_opts* opts, mphy_mixed** out);
int mphy_mixed_destroy(mphy_mixed* m);
/* pressure DOF count; entries of the coupling block B = Kup (node rows) and of C = Kpp */
int mphy_mixed_info(mphy_mixed* m, int32_t* n_pres, int64_t* nnz_coupling, int64_t* nnz_pp);
/* the global node of each pressure DOF (assyForSolnPres) [n_pres], host */
int mphy_mixed_pressure_nodes(mphy_mixed* m, int32_t* nodes_host);
/* calcStiffnessAndResidualMixed for every element. Device arrays: disp, disp_prev (the last
 * converged step, for Jn) [3 n_node], pres [n_node] nodal pressures (pressure nodes used);
 * with ns = 3 npe and NP pressure nodes per element (4 tet10, 8 hex27), outputs Kuu
 * [n_elem][ns][ns], FU [n_elem][ns], Kup [n_elem][ns][NP] (Kpu = Kup^T), Kpp [n_elem][NP][NP],
 * FP [n_elem][NP]. MPHY_ERR_NEG_JACOBIAN as mphy_elem_eval. */
int mphy_mixed_elem_eval(mphy_mixed* m, const double* disp_dev, const double* disp_prev_dev,
                         const double* pres_dev, double* Kuu_dev, double* FU_dev, double* Kup_dev,
                         double* Kpp_dev, double* FP_dev, int64_t* first_bad);
/* femSolidmechanics::calcStiffnessAndResidual for a mixed mesh plus rhs_u += lambda fext_dev on
 * the free DOFs (fext_dev may be NULL); *rhs_norm = ||rhs|| over both fields. */
int mphy_mixed_assemble(mphy_mixed* m, const double* disp_dev, const double* disp_prev_dev,
                        const double* pres_dev, double lambda, const double* fext_dev, double* rhs_norm,
                        int64_t* first_bad);
/* y = A x with the assembled two-field operator, device vectors [3 n_node + n_pres]. */
int mphy_mixed_apply(mphy_mixed* m, const double* x_dev, double* y_dev);
/* Copies (device, any may be NULL): rhs [3 n_node + n_pres], reactions [3 n_node], the last
 * solution [3 n_node + n_pres]. */
int mphy_mixed_vectors(mphy_mixed* m, double* rhs_dev, double* reac_dev, double* solution_dev);
/* MINRES on the assembled system from x = 0; *relres = ||rhs - A x|| / ||rhs|| (FP64). */
int mphy_mixed_solve(mphy_mixed* m, int32_t* its, double* relres);
/* solveWithNewtonRaphson for the mixed mesh (load stepping and cuts as mphy_newton_run; a cut
 * restores displacements and pressures). fext_host, disp_host: [3 n_node]; pres_host: [n_node]
 * nodal pressures; both in/out. hist: one row per Newton iteration (krylov_its = MINRES). */
int mphy_mixed_newton_run(mphy_mixed* m, const double* fext_host, const mphy_newton_opts* opts,
                          double* disp_host, double* pres_host, mphy_iter_stats* hist_host,
                          int32_t max_hist, int32_t* n_hist);

/* ------------------------------------------------------------------ batched form
 * Many independent problems as one block-diagonal union mesh: instance i owns the contiguous
 * nodes [node_ptr[i], node_ptr[i+1]) and only elements among them. The solver s (Jacobi-PCG,
 * FP64 or MPHY_PREC_MIXED values, FP64 vectors) is created on the union; assembly runs over the
 * union, and the linear solves of all instances run in one persistent launch: each thread-block
 * cluster takes instances from a work queue, largest first, and runs Jacobi-PCG (KSPCG semantics,
 * s's rtol / abstol / dtol / norm_type) on each with cluster-wide reductions in distributed
 * shared memory. The reference solves one problem per run (femSolidmechanics2.cpp:730-851); every
 * instance here follows that loop on its own. */
typedef struct mphy_batch mphy_batch;

typedef struct mphy_batch_stats {
    int32_t steps;            /* load steps completed */
    int32_t graph_replays;    /* batch Newton iterations (one CUDA graph replay each) */
    int64_t kernel_launches;  /* libmphy kernels in those replays */
    float t_ms;               /* device time of the load stepping */
} mphy_batch_stats;

/* node_ptr_host: [n_inst+1], 0 = node_ptr[0] < ... < node_ptr[n_inst] = n_node. Fails with
 * MPHY_ERR_INVALID_ARG when an element couples two instances. */
int mphy_batch_create(mphy_solver* s, int32_t n_inst, const int32_t* node_ptr_host, mphy_batch** out);
int mphy_batch_destroy(mphy_batch* b);
/* Schedule of the persistent solve: CTAs per cluster (1, 2, 4, 8) and threads per CTA (128, 256,
 * 512). The default is (1, 256); mphy_batch_autotune picks one by measurement. */
int mphy_batch_set_schedule(mphy_batch* b, int32_t cluster, int32_t threads);
int mphy_batch_get_schedule(const mphy_batch* b, int32_t* cluster, int32_t* threads);
/* Two-level variant of the persistent solve: every instance is cut into `slabs` (1..8; 0 turns
 * it off) slabs along its longest axis, and z = D^{-1} r + Z E^{-1} Z^T r with Z the six
 * rigid-body modes of every slab (zero on prescribed DOFs) and E = Z^T A Z assembled, summed over
 * the cluster and inverted in shared memory at the start of each instance's solve. */
int mphy_batch_set_coarse(mphy_batch* b, int32_t slabs);
/* Times every schedule on the assembled system (solves capped at maxit iterations; maxit <= 0:
 * complete solves, which also measures the load balance of the slowest instances) and keeps the
 * fastest. Writes up to max_candidates rows (cluster, threads, ms); *n_candidates = rows tried. */
int mphy_batch_autotune(mphy_batch* b, int32_t maxit, int32_t max_candidates, int32_t* n_candidates,
                        int32_t* clusters, int32_t* threads, float* ms);
/* Solve every instance on the assembled system (x = 0 start, solution in the solver's x) in one
 * launch. Per instance (host arrays, each may be NULL): iterations, status, final / initial norm
 * of the convergence test. maxit <= 0: the solver's max_it. *ms: device time. */
int mphy_batch_solve(mphy_batch* b, int32_t maxit, int32_t* its_host, int32_t* status_host,
                     double* relres_host, float* ms);
/* Load stepping of every instance (lambda = t, steps of o->dt up to o->t_final / o->max_steps),
 * each instance following mphy_newton_run on its own: its own load factor, Newton iterations,
 * step cuts (halving dt and restoring the last converged state after det F < 0, divergence or
 * max_newton iterations) and MPHY_ERR_TIME_STEP when dt falls below 1% of o->dt. One CUDA graph
 * replay per batch Newton iteration. fext_host, disp_host: [3*n_node] union vectors (disp
 * in/out). newton_its_host: [max_steps][n_inst] Newton solves of each converged step;
 * krylov_its_host, status_host: [n_inst]. Any output may be NULL. */
int mphy_batch_newton_run(mphy_batch* b, const double* fext_host, const mphy_newton_opts* o,
                          double* disp_host, int32_t* newton_its_host, int32_t* krylov_its_host,
                          int32_t* status_host, mphy_batch_stats* stats);
/* After mphy_batch_newton_run, per instance: Newton solves in all steps (failed tries included),
 * step cuts, converged steps, load factor reached. Any pointer may be NULL. */
int mphy_batch_instance_info(mphy_batch* b, int32_t* newton_total_host, int32_t* cuts_host,
                             int32_t* steps_done_host, double* t_host);

#ifdef __cplusplus
}
#endif

#endif /* MPHY_H */
