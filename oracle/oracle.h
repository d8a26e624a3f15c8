/*
 * oracle.h -- CPU FP64 restatement of chennachaos/mphyfem's femSolidmechanics Newton-step
 * hot path (element, Neo-Hookean material, DOF map / CSR pattern, assembly, PETSc-KSPCG
 * style Jacobi-preconditioned CG, Newton-Raphson load stepping).
 *
 * TEST INFRASTRUCTURE ONLY. Only the tests, the smoke check and the benchmark's CPU-baseline
 * leg load this library, and only as the checker / the timed CPU reference. The product path
 * (mphyfem_b200/libmphy.so) never links or calls it.
 *
 * Parity status: UNPINNED against the reference binary. The reference cannot be built here
 * (its hot path needs PETSc, Eigen, Boost, MPI and VTK, none of which is installed) and it
 * ships no tests, golden vectors or recorded outputs. The restatement is pinned instead by
 * independent checks in tests/: central-difference tangents (the stencil documented at
 * src/utilities/ElementBase.cpp:1519-1524), closed-form Neo-Hookean stresses, zero residual at
 * u = 0, rigid-rotation invariance, a linear patch test and symmetric element tangents.
 *
 * All matrices are row-major unless stated. Element DOF order is 3*node + dim
 * (src/utilities/ElementBase.cpp:46-69).
 */
#ifndef MPHY_ORACLE_H
#define MPHY_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Neo-Hookean Cauchy stress (9, column-major 3x3) and 9x9 spatial tangent, indices in the
 * map_tensor4 order {(0,0),(1,0),(2,0),(0,1),(1,1),(2,1),(0,2),(1,2),(2,2)}.
 * F is row-major F[3*i+j] = F(i,j). Cmat is row-major Cmat[9*i1+j1].
 * Follows src/material/utilitiesmaterialHyperelastic.cpp:186-295 (compressible branch).
 * Returns 0. */
int orc_nh_stress_tangent(const double* F, double mu, double Kinv, int Utype,
                          double* stre, double* Cmat);

/* Hyperelastic models of the reference's MaterialBase family and their parameters:
 *   ORC_MAT_NEOHOOKEAN   Matl_NeoHookean,   data_deviatoric = {mu}
 *   ORC_MAT_MOONEYRIVLIN Matl_MooneyRivlin, data_deviatoric = {c1, c2}
 *                        (utilitiesmaterialHyperelastic.cpp:300-420)
 *   ORC_MAT_GENT         Matl_Gent,         data_deviatoric = {mu, Im}  (:423-548)
 *   ORC_MAT_ARRUDABOYCE  Matl_ArrudaBoyce,  data = {mu, N}              (:551-677)
 * each with the volumetric energy Utype and Kinv = 1/K of data_volumetric. */
enum { ORC_MAT_NEOHOOKEAN = 0, ORC_MAT_MOONEYRIVLIN = 1, ORC_MAT_GENT = 2, ORC_MAT_ARRUDABOYCE = 3 };
enum { ORC_MAT_NDATA = 4 };

/* Stress and tangent of any model above, same conventions as orc_nh_stress_tangent.
 * Returns 0, or 2 for an unknown model. */
int orc_material_stress_tangent(int model, const double* data, double Kinv, int Utype, const double* F,
                                double* stre, double* Cmat);

/* Mixed (u-p) branch of the same models: the pressure pres replaces U'(J) in the stress and the
 * pressure term replaces the volumetric tangent (utilitiesmaterialHyperelastic.cpp, the
 * MIXED_ELEMENT branches). Returns 0, or 2 for an unknown model. */
int orc_material_stress_tangent_mixed(int model, const double* data, double Kinv, int Utype, const double* F,
                                      double pres, double* stre, double* Cmat);

/* compute_constants_volumetric_functions, finite strain (utilitiesmaterialHyperelastic.cpp:144-173). */
void orc_mixed_constants(int Utype, double Jn, double K, double* Jhat, double* thetahat);

/* Mixed u-p tet10 element with linear vertex pressure (Elem_Solid_3D_Mixed1 with npElem = 10,
 * ElementBase::calcStiffnessAndResidualMixed3D, ElementBase2.cpp:278-553), STATIC scheme.
 * X, u, u_prev (the last converged step's displacement, for Jn): [10][3]; pn: [4] vertex
 * pressures. Kuu [30][30], Kup [30][4], Kpu [4][30], Kpp [4][4], FU [30], FP [4], row-major.
 * Returns 0, 1 when some Gauss point has det F < 0, 2 for npe != 10 or an unknown model. */
int orc_elem_mixed(int npe, const double* X, const double* u, const double* u_prev, const double* pn, int model,
                   const double* data, double Kinv, int Utype, double* Kuu, double* Kup, double* Kpu, double* Kpp,
                   double* FU, double* FP);

/* Constant-pressure mixed element (Elem_Solid_3D_Mixed0, Elem_Solid_3D_Mixed0.cpp): hex8 or tet10
 * displacement, one pressure per element (nlbfP = 1, Np = 1, pres = the element's pressure), the
 * blocks of ElementBase::calcStiffnessAndResidualMixed3D condensed (:93-101):
 * K = Kuu - Kup Kpu / Kpp, F = FU - Kup FP / Kpp. Outputs K [3npe][3npe], F [3npe] and the
 * coupling column kup [3npe] (= Kpu), Kpp and FP for solveForPressure (:112-200).
 * Returns 0, 1 when some Gauss point has det F < 0, 2 for an unsupported npe or model. */
int orc_elem_mixed0(int npe, const double* X, const double* u, const double* u_prev, double pres, int model,
                    const double* data, double Kinv, int Utype, double* K, double* F, double* kup, double* kpp,
                    double* fp);

/* ---- see orc_problem_create below: every element of a tet10 problem as a mixed u-p element.
 * disp, disp_prev: [3*n_node]; pres: [n_node] nodal pressures (vertex nodes used). Outputs per
 * element: Kuu [30][30], Kup [30][4] (Kpu = Kup^T), Kpp [4][4], FU [30], FP [4]. Returns the
 * first element with det F < 0, -1, or -2 when the mesh is not tet10. */
typedef struct orc_problem orc_problem;
int64_t orc_problem_elements_mixed(const orc_problem* p, const double* disp, const double* disp_prev,
                                   const double* pres, double* Kuu, double* Kup, double* Kpp, double* FU, double* FP,
                                   int nthreads);

/* Test-only switch: 0 (default) = the reference's tangent; 1 = add the volumetric geometric
 * term U'(J) d_ik d_jl that the reference omits, giving the consistent tangent -dR/du. */
void orc_set_consistent_tangent(int on);

/* Test-only switch for the pattern builder: 0 = by size, 1 = literal per-element restatement,
 * 2 = per-node construction (bounded memory). Both produce the same CSR pattern. */
void orc_set_pattern_mode(int mode);

/* Volumetric energy derivatives U'(J), U''(J) for Utype 1..8
 * (src/material/utilitiesmaterialHyperelastic.cpp:45-140). */
double orc_vol_dU(int Utype, double K, double J);
double orc_vol_d2U(int Utype, double K, double J);

/* One displacement element (hex8: npe = 8, 2x2x2 Gauss; tet10: npe = 10, 4-point rule).
 * X, u: [npe][3]. K: [3npe][3npe] row-major, R: [3npe] (= -f_int, STATIC scheme).
 * Follows src/femSolidmechanics/Elem_Solid_3D_Disp.cpp:196-373. Returns 0, or 1 when some
 * Gauss point has det F < 0 (the reference throws there, :275-278). */
int orc_elem_stiffness_residual(int npe, const double* X, const double* u, double mu,
                                double Kinv, int Utype, double* K, double* R);

/* orc_elem_stiffness_residual with any material model (data: [ORC_MAT_NDATA]). */
int orc_elem_stiffness_residual_mat(int npe, const double* X, const double* u, int model, const double* data,
                                    double Kinv, int Utype, double* K, double* R);

/* Gauss points and shape functions used by the element (for cross-checks). Writes ngp and
 * xi[ngp][3], w[ngp]; N[ngp][npe]; dNdxi[ngp][3][npe]. Returns ngp. */
int orc_gauss_rule(int npe, double* xi, double* w, double* N, double* dNdxi);

/* ---- problem handle: mesh + DOF map + CSR pattern (prepareMatrixPattern) ---- */
typedef struct orc_problem orc_problem;

/* mats: [n_mat][3] = {mu, Kinv, Utype}. fixed: [n_node*3] (1 = prescribed DOF).
 * Builds the DOF map and the sorted-unique CSR pattern exactly as
 * src/femSolidmechanics/femSolidmechanics2.cpp:121-478 does. */
orc_problem* orc_problem_create(int n_node, const double* coords, int n_elem, int npe,
                                const int32_t* conn, const int32_t* mat_id, int n_mat,
                                const double* mats, const uint8_t* fixed);
void orc_problem_destroy(orc_problem* p);
/* Per-material model codes [n_mat] and parameters [n_mat][ORC_MAT_NDATA]; Kinv and Utype stay
 * those of orc_problem_create. Without this call every material is Neo-Hookean with mu =
 * mats[3k]. Returns 0, 1 when n_mat differs from the problem's, 2 for an unknown model. */
int orc_problem_set_materials(orc_problem* p, int n_mat, const int32_t* model, const double* data);
int orc_problem_nfree(const orc_problem* p);
/* Nonzero prescribed displacements: the DOFs flagged in `fixed` take t * ramp[i] + cst[i] at time t
 * (either array may be NULL: zero). The Newton run lifts each step's increment (value(t) - disp)
 * into the free rows of the first iteration (ElementBase::applyDirichletBCs, ElementBase.cpp:567-594)
 * and adds it to the displacement with that iteration's solution (femSolidmechanics2.cpp:1137-1145). */
int orc_problem_set_prescribed(orc_problem* p, const double* ramp, const double* cst);
/* Elem_Solid_3D_Mixed0 for every element (enable = 1; 0 = the displacement element): assembly,
 * elements and Newton use the condensed element; the Newton run updates the element pressures
 * after every solve (femSolidmechanics2.cpp:1204-1212), saves them with each converged step and
 * restores them on a cut. Pressures and the last-step displacement start at zero.
 * Returns 2 when a material has Utype -1 (Kpp = 0). */
int orc_problem_set_mixed_p0(orc_problem* p, int enable);
/* element pressures [n_elem]: set (may be NULL) copied in first, then get (may be NULL) filled */
void orc_problem_p0_pressure(const orc_problem* p, const double* set, double* get);
/* the last converged step: disp (its J is the mixed element's Jn) and the element pressures */
void orc_problem_save_step(const orc_problem* p, const double* disp);
int64_t orc_problem_nnz(const orc_problem* p);
/* assy_for_soln: [n_free]; for_assy_vec: [n_elem][3npe]; rowptr: [n_free+1]; col: [nnz] */
void orc_problem_export_pattern(const orc_problem* p, int32_t* assy_for_soln,
                                int32_t* for_assy_vec, int64_t* rowptr, int32_t* col);

/* Element matrices for every element at displacement disp [n_node*3].
 * Ke: [n_elem][3npe*3npe], Re: [n_elem][3npe]. Returns the first element with det F < 0, or -1. */
int64_t orc_problem_elements(const orc_problem* p, const double* disp, double* Ke, double* Re,
                             int nthreads);

/* calcStiffnessAndResidual (femSolidmechanics2.cpp:1047-1120) + the per-entry ADD_VALUES
 * scatter of SolverPetsc::assembleMatrixAndVector (SolverPetsc.cpp:357-378).
 * val: [nnz] CSR values, rhs: [n_free], reac: [n_node*3] (any may be NULL).
 * Returns the first element with det F < 0, or -1. nthreads > 1 uses OpenMP (atomic adds). */
int64_t orc_problem_assemble(const orc_problem* p, const double* disp, double* val, double* rhs,
                             double* reac, int nthreads);

/* PETSc KSPCG + PCJACOBI semantics: x0 = 0, preconditioned-residual norm, converged when
 * ||z_k|| <= max(rtol*||z_0||, abstol); divergence on non-positive p.Ap or its > maxit.
 * Returns 0 converged, 1 not converged within maxit, 2 indefinite, 3 NaN. */
int orc_cg_jacobi(const orc_problem* p, const double* val, const double* b, double* x,
                  double rtol, double abstol, int maxit, int nthreads, int* its,
                  double* final_norm);
/* The same with the norm type: 0 = KSP_NORM_PRECONDITIONED (||z||, PETSc's CG default),
 * 1 = KSP_NORM_UNPRECONDITIONED (||r||, the true residual relative to ||b||). */
int orc_cg_jacobi_norm(const orc_problem* p, const double* val, const double* b, double* x,
                       double rtol, double abstol, int maxit, int nthreads, int norm_type, int* its,
                       double* final_norm);

/* Newton-Raphson load stepping (femSolidmechanics2.cpp:730-851, STATIC scheme, nodal forces
 * scaled by the load factor lambda(t) = t).
 * fnodal: [n_node*3] reference nodal forces (lambda = 1). disp: [n_node*3] in/out.
 * Convergence when ||R|| < max(tol_abs, tol_rel * ||R||_first-iteration-of-step).
 * hist: [max_hist][4] = {step, iter, ||R||, cg its}; returns the number of rows written,
 * or -1 on time-step underflow. */
typedef struct {
    double dt;
    double t_final;
    int    max_steps;
    int    max_newton;
    double tol_rel;
    double tol_abs;
    double cg_rtol;
    int    cg_maxit;
    int    nthreads;
} orc_newton_opts;

int orc_newton_run(const orc_problem* p, const double* fnodal, const orc_newton_opts* opts,
                   double* disp, double* hist, int max_hist);

/* Arc-length continuation: femSolidmechanics::solveWithArclength (femSolidmechanics2.cpp:855-1039)
 * with SolverPetsc::solveArclengthSystem (SolverPetsc.cpp:671-757). opts: dt = the first load
 * factor and the time increment of every attempt, t_final, max_steps (converged steps),
 * max_newton = iterationsMax (iterations 1..max_newton-1), tol_abs / tol_rel as in
 * orc_newton_run. disp: [3*n_node] in/out. lambdas: load factor of each converged step.
 * hist rows: step, iter, ||R||, CG iterations of both solves, load factor after the update.
 * Returns the number of rows, or -1 when the first step does not converge. */
int orc_arclength_run(const orc_problem* p, const double* fnodal, const orc_newton_opts* opts,
                      double* disp, double* lambdas, int max_lambdas, int* n_lambdas, double* hist,
                      int max_hist);

#ifdef __cplusplus
}
#endif

#endif
