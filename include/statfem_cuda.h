/*
 * statfem_cuda.h -- C ABI of the B200-native statFEM forward-and-conditioning
 * path (element assembly, SPD sparse solves, GP forcing covariance and the
 * prior-to-posterior conditioning on sensor data).
 *
 * Plain C types only: host pointers, sizes, opaque handles.  Every function
 * returns SFC_OK (0) or a negative SFC_ERR_* code; sfc_last_error() gives the
 * message of the last failure on a context.  Calls on one context are issued
 * in order on that context's CUDA stream; a context is not thread-safe (one
 * context per host thread), like the reference's solver objects.  Pointer
 * arguments are HOST memory unless the name ends in _dev.
 *
 * Each declaration names the reference interface it replaces (file:line in
 * fcirak/statFEM).  The reference has no FFI of its own: it is a header-only
 * C++ library whose solver is selected by a typedef
 * (del2/apps/reference/laplaceRHSinfer/laplaceRHSinfer.cpp:99).  The C++
 * class corlib::SystemSolveCuda (include/corlib/SystemSolveCuda.hpp) wraps
 * this ABI with the method set of corlib::SystemSolveEigenSparse so that
 * changing that typedef is the whole integration.
 */
#ifndef STATFEM_CUDA_H
#define STATFEM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define SFC_OK                 0
#define SFC_ERR_CUDA          -1  /* a CUDA runtime call failed              */
#define SFC_ERR_BAD_ARG       -2  /* invalid argument / state                 */
#define SFC_ERR_NOT_SPD       -3  /* Cholesky or CG breakdown (p^T A p <= 0)  */
#define SFC_ERR_NOT_CONVERGED -4  /* iteration cap reached                    */
#define SFC_ERR_TIMEOUT       -5  /* a bounded device-side wait gave up       */
#define SFC_ERR_NO_MEMORY     -6  /* device or host allocation failed         */
#define SFC_ERR_NEG_JACOBIAN  -7  /* detJ <= 0 in an element (FTL_VERIFY in
                                     corlib/ElementBasic.ipp:199)             */
#define SFC_ERR_TOO_LARGE     -8  /* problem exceeds a fixed limit: a fixed-size
                                     scratch area, or the 32-bit index range
                                     (dofs < 2^31; element-matrix entries
                                     E * L^2 < 2^31, L = element dofs: about
                                     3.7 M hex8 elasticity elements, 33 M
                                     P1 triangles)                          */

/* ---- element kinds (element type + its integrand) ------------------------ */
#define SFC_ELEM_LINE2_POISSON  1 /* del2::fem::ElementPotential, 2-node line */
#define SFC_ELEM_TRI3_POISSON   2 /* ElementPotential, 3-node triangle        */
#define SFC_ELEM_HEX8_POISSON   3 /* ElementPotential, trilinear hexahedron   */
#define SFC_ELEM_HEX8_ELASTIC   4 /* solid::fem::ElementStatic + SVenant at
                                     F = I (isotropic linear elasticity)      */

/* ---- solver methods ------------------------------------------------------ */
#define SFC_SOLVER_PCG_FP64      0 /* plain FP64 Jacobi-PCG, one RHS at a time */
#define SFC_SOLVER_PCG_MIXED     1 /* FP32 block Jacobi-PCG (many RHS share the
                                      matrix) + FP64 residual refinement      */
#define SFC_SOLVER_FCG_MPNN      2 /* flexible CG (FP64) preconditioned by the
                                      learned message-passing network set with
                                      sfc_system_set_mpnn (forward solves)    */

typedef struct sfc_ctx sfc_ctx_t;
typedef struct sfc_mesh sfc_mesh_t;
typedef struct sfc_system sfc_system_t;
typedef struct sfc_covar_forcing sfc_covar_forcing_t;
typedef struct sfc_forward_gauss sfc_forward_gauss_t;
typedef struct sfc_koh sfc_koh_t;

typedef struct sfc_solver_options {
    int32_t method;        /* SFC_SOLVER_*                                     */
    int32_t max_iter;      /* inner iteration cap per right-hand side          */
    double tol;            /* relative residual ||b-Ax||/||b|| (true, FP64)    */
    double inner_tol;      /* FP32 inner reduction per refinement cycle        */
    int32_t block_width;   /* RHS per block for SFC_SOLVER_PCG_MIXED (0: auto) */
    int32_t check_every;   /* iterations between the host's convergence checks
                              (0: auto); the mixed block solver also tests
                              convergence on the device after every iteration
                              and skips the rest of an interval once all
                              columns are below their thresholds             */
    int32_t precond;       /* SFC_PRECOND_*                                    */
    int32_t coarse_size;   /* SFC_PRECOND_TWO_LEVEL: nodes per aggregate along
                              each axis (0: 8)                                */
} sfc_solver_options_t;

/* preconditioners.  JACOBI and BLOCK_JACOBI select the FP32 iteration's
 * preconditioner of SFC_SOLVER_PCG_MIXED (its FP64 solves use point Jacobi);
 * TWO_LEVEL applies to every PCG of the system, FP64 and mixed. */
#define SFC_PRECOND_JACOBI        0 /* point Jacobi                            */
#define SFC_PRECOND_BLOCK_JACOBI  1 /* nodal 3x3 block Jacobi on 3-dof meshes,
                                       point Jacobi otherwise                  */
#define SFC_PRECOND_TWO_LEVEL     2 /* Jacobi smoother plus an additive coarse
                                       correction on box aggregates of the
                                       mesh's nodes: nodal 3x3 block Jacobi and
                                       the six rigid-body modes per aggregate
                                       on 3-dof meshes, point Jacobi and the
                                       constant per aggregate on scalar ones
                                       (systems assembled from a mesh; the
                                       one-level preconditioner otherwise)    */

typedef struct sfc_solve_stats {
    int32_t iterations;       /* max over right-hand sides, inner iterations   */
    int32_t refinements;      /* FP64 refinement cycles (mixed solver)         */
    int32_t num_rhs;
    int32_t converged;        /* 1 when every RHS met tol                      */
    double max_rel_residual;  /* max over RHS of the true FP64 ||b-Ax||/||b||  */
    double device_ms;         /* device time of the last solve call            */
    int32_t fallback_columns; /* mixed solver: columns finished by FP64
                                 Jacobi-PCG after repeated FP32 breakdowns    */
    int32_t coarse_dofs;      /* size of the coarse space used (TWO_LEVEL),
                                 0 when the solve had none                    */
    int32_t spmm_kernel;      /* FP32 product of the mixed solver: 0 none (FP64
                                 solve), 1 CSR rows, 2 node blocks (3-dof
                                 meshes), 3 lattice bricks staged by TMA
                                 (SFC_SPMM=lattice), 4 streamed lattice
                                 x-lines (the default on 3-dof structured
                                 lattices)                                    */
    int32_t reserved;
} sfc_solve_stats_t;

/* Hyperparameters; the reference keeps them in std::map<std::string,double>
 * under these names (statX/infer/ExpKernel.hpp:63-64 with the prefixes set in
 * CovarianceForcing.hpp:73, MismatchCovariance.hpp:62-67 and
 * LikelihoodKOH.hpp:66). */
typedef struct sfc_hparams {
    double forcing_sigma;       /* "forcing.sigma"       */
    double forcing_length;      /* "forcing.length"      */
    double rho;                 /* "rho"                 */
    double mismatch_sigma;      /* "mismatch.sigma"      */
    double mismatch_length;     /* "mismatch.length"     */
    double mismatch_sensor_eps; /* "mismatch.sensorEps"  */
} sfc_hparams_t;

/* ---- context --------------------------------------------------------------- */
int32_t sfc_version(void);
/* No reference counterpart (the reference is host-only): owns the device and
 * the CUDA stream that every later call on it is issued on. */
int32_t sfc_ctx_create(int32_t device, sfc_ctx_t **out);
int32_t sfc_ctx_destroy(sfc_ctx_t *ctx);
const char *sfc_last_error(const sfc_ctx_t *ctx);
int32_t sfc_ctx_synchronize(sfc_ctx_t *ctx);
/* Number of kernels this library has launched on the context (kernels inside
 * a replayed CUDA graph included). */
int32_t sfc_ctx_kernel_launches(const sfc_ctx_t *ctx, int64_t *count);
/* Number of CUDA graphs this library has launched on the context (the mixed
 * block solver's captured check intervals, batch steps, dense inverses). */
int32_t sfc_ctx_graph_launches(const sfc_ctx_t *ctx, int64_t *count);
/* Device time between two markers recorded on the context stream. */
int32_t sfc_ctx_mark(sfc_ctx_t *ctx, int32_t slot);
int32_t sfc_ctx_marker_ms(sfc_ctx_t *ctx, int32_t slot_begin, int32_t slot_end, double *ms);

/* Kernel timing (no reference counterpart; the reference has no tracing):
 * when enabled, the hot kernels are bracketed by CUDA events on the context
 * stream.  The report writes one line per kernel name,
 * "name launches total_ms algorithmic_bytes", into buf (NUL-terminated) and
 * clears the records. */
int32_t sfc_ctx_set_profiling(sfc_ctx_t *ctx, int32_t enable);
int32_t sfc_ctx_profile_report(sfc_ctx_t *ctx, char *buf, int64_t buflen);

/* ---- mesh -------------------------------------------------------------- */
/* Replaces corlib::Mesh<Element>(std::istream& smf) (corlib/Mesh.ipp:63-102)
 * plus Node::numberDOFs (del2/fem/NodePotential.hpp:65,
 * solid/fem/NodeStatic.ipp:15-19): coords are num_nodes x 3 (an SMF node line
 * always has three columns), conn is num_elems x nodes_per_elem with 0-based
 * node ids, dof = node * dofs_per_node + component.  quad_points is the
 * reference's Quadrature<SHAPE,QPS> QPS (line: 1..5; triangle: 1 or 3;
 * hexahedron: 1, 8, 27, 64, 125).  Builds the CSR pattern and the
 * element-entry -> CSR-slot maps on the device (one-time symbolic phase). */
int32_t sfc_mesh_create(sfc_ctx_t *ctx, int32_t element_kind, int32_t quad_points,
                        const double *coords, int64_t num_nodes, const uint32_t *conn,
                        int64_t num_elems, sfc_mesh_t **out);
int32_t sfc_mesh_destroy(sfc_mesh_t *mesh);
/* Per-element coefficient: conductivity (ElementPotential::setConductivity,
 * del2/fem/ElementPotential.hpp:94-97) or Young's modulus (SVenant
 * "youngModulus", solid/material/svenant/SVenant.ipp:16); poisson_ratio is
 * used by the elastic kind.  values == NULL sets every element to uniform. */
int32_t sfc_mesh_set_coefficients(sfc_mesh_t *mesh, const double *values, double uniform,
                                  double poisson_ratio);
int64_t sfc_mesh_num_dofs(const sfc_mesh_t *mesh);
int64_t sfc_mesh_nnz(const sfc_mesh_t *mesh);

/* ---- system (corlib::SystemSolveEigenSparse replacement) ------------------ */
/* SystemSolveEigenSparse(numDofs), corlib/SystemSolveEigenSparse.hpp:54-60 */
int32_t sfc_system_create(sfc_ctx_t *ctx, int64_t num_dofs, sfc_system_t **out);
int32_t sfc_system_destroy(sfc_system_t *sys);
int32_t sfc_system_set_options(sfc_system_t *sys, const sfc_solver_options_t *opt);
int32_t sfc_system_get_options(const sfc_system_t *sys, sfc_solver_options_t *opt);
int32_t sfc_system_last_stats(const sfc_system_t *sys, sfc_solve_stats_t *stats);

/* insertToMatrix, SystemSolveEigenSparse.hpp:160-172 (called per element by
 * MatrixAssembler::operator(), corlib/MatrixAssembler.hpp:224-229).  Ke is
 * row-major n x m.  Entries are staged on the host and sorted / merged on the
 * GPU at the next finish, constraint or solve call, with the triplet
 * semantics of corlib/Triplet.hpp:126-170 (duplicates summed in insertion
 * order, explicit zeros kept). */
int32_t sfc_insert_matrix(sfc_system_t *sys, const double *Ke, const uint32_t *rows, uint32_t n,
                          const uint32_t *cols, uint32_t m);
/* insertToRhs, SystemSolveEigenSparse.hpp:176-184: F[dofs[i]] += fe[i]. */
int32_t sfc_insert_rhs(sfc_system_t *sys, const double *fe, const uint32_t *dofs, uint32_t n);
/* finishAssembly / finishMatAssembly / finishRhsAssembly,
 * SystemSolveEigenSparse.hpp:93-98 (no-ops there; here they flush the staged
 * host data to the device). */
int32_t sfc_finish_assembly(sfc_system_t *sys);

/* GPU assembler (corlib::MatrixComputeAndAssembleFun over all elements,
 * corlib/MatrixAssembler.hpp:43-100 + ComputeElementMatrix.hpp:62-77 with
 * Element::stiffnessIntegrand): computes every element matrix and sums them
 * into the system's CSR values, in element order per CSR slot.  Replaces any
 * previous matrix values (clearMatrix + full assembly). */
int32_t sfc_assemble_matrix(sfc_system_t *sys, const sfc_mesh_t *mesh);
/* GPU body-force load (Integrator<Quad,BodyForce> over elements +
 * VectorAssembler, corlib/Integrator.hpp:61-73, BodyForce.hpp:66-71,
 * VectorAssembler.hpp:101-114) for a constant force f[dofs_per_node]:
 * F += assembled nodal forces. */
int32_t sfc_assemble_load(sfc_system_t *sys, const sfc_mesh_t *mesh, const double *f);

/* applyConstraints, SystemSolveEigenSparse.hpp:197-215 (Triplet::zeroRow,
 * corlib/Triplet.hpp:219-260): for each (idx[t], value[t]) zero the row, put
 * `scalar` on its diagonal and set F[idx] = (factor*value)*scalar.
 * value == NULL means all zero. */
int32_t sfc_apply_constraints(sfc_system_t *sys, const uint32_t *idx, const double *value,
                              int64_t n, double factor, double scalar);
/* fixDOF, SystemSolveEigenSparse.hpp:219-226 */
int32_t sfc_fix_dof(sfc_system_t *sys, uint32_t idx, double scalar);

/* solveSystem() / solveSystem(bool reuse), SystemSolveEigenSparse.hpp:
 * 273-360: X = A^-1 F.  The row-zeroed matrix is solved through its symmetric
 * elimination (constrained columns lifted into the right-hand side) with the
 * configured PCG; `reuse` is accepted for interface parity (the iterative
 * solver keeps no factorisation). */
int32_t sfc_solve(sfc_system_t *sys, int32_t reuse);
/* solveSystemTranspose, SystemSolveEigenSparse.hpp:364-404: u = A^-T rhs
 * for num_rhs right-hand sides (rhs, u: num_rhs x num_dofs, row-major, host). */
int32_t sfc_solve_transpose(sfc_system_t *sys, const double *rhs, double *u, int32_t num_rhs,
                            int32_t reuse);
/* Many right-hand sides at once for A u = b, with A the reference's
 * row-zeroed system (solveSystem applied to each column; no single reference
 * counterpart, the reference solves one vector per call,
 * SystemSolveEigenSparse.hpp:273-310).  rhs, u: nrhs x num_dofs, host.
 * With SFC_SOLVER_PCG_MIXED the columns go through the FP32 block solver with
 * FP64 residual replacement, else FP64 Jacobi-PCG one column at a time. */
int32_t sfc_solve_multi(sfc_system_t *sys, const double *rhs, double *u, int32_t nrhs);
/* The same on device memory of the context's device, interleaved:
 * column a of row i at [i * ld + a] (ld >= nrhs); issued on the context
 * stream. */
int32_t sfc_solve_multi_device(sfc_system_t *sys, const double *rhs_dev, double *u_dev, int32_t nrhs,
                               int32_t ld);
/* giveSolution / giveForce, SystemSolveEigenSparse.hpp:408-428 */
int32_t sfc_give_solution(const sfc_system_t *sys, const uint32_t *dofs, int64_t n,
                          double *out);
int32_t sfc_give_force(const sfc_system_t *sys, const uint32_t *dofs, int64_t n, double *out);
/* clearMatrix / clearRhs, SystemSolveEigenSparse.hpp:104-107 */
int32_t sfc_clear_matrix(sfc_system_t *sys);
int32_t sfc_clear_rhs(sfc_system_t *sys);
/* numNonZeros / normMatrix / normRhs / norm1Rhs / normSol,
 * SystemSolveEigenSparse.hpp:78-83,118 */
int64_t sfc_num_nonzeros(const sfc_system_t *sys);
int32_t sfc_norms(const sfc_system_t *sys, double *frobenius_matrix, double *norm2_rhs,
                  double *norm1_rhs, double *norm2_sol);
/* Export of the assembled matrix in the reference's row-zeroed form (CSR of
 * the sorted, merged triplets; writeMatrix, SystemSolveEigenSparse.hpp:73). */
int32_t sfc_get_csr(const sfc_system_t *sys, int64_t *row_ptr, int32_t *col, double *val);

/* ---- statX: forcing covariance ------------------------------------------- */
/* CovarianceForcing<DOF,ExpKernel>(numNodes), statX/infer/CovarianceForcing.hpp:
 * 68-74, with coordinates inserted per node (insertToCoordinates, .ipp:27-34)
 * and phibar = int(phi_i) from the GPU unit load (inference.hpp:108-119). */
int32_t sfc_covar_forcing_create(sfc_ctx_t *ctx, const sfc_mesh_t *mesh,
                                 sfc_covar_forcing_t **out);
int32_t sfc_covar_forcing_destroy(sfc_covar_forcing_t *cf);
/* CovarianceForcing::applyConstraints, CovarianceForcing.hpp:101-114 */
int32_t sfc_covar_forcing_apply_constraints(sfc_covar_forcing_t *cf, const uint32_t *idx,
                                            int64_t n);
int32_t sfc_covar_forcing_get_phibar(const sfc_covar_forcing_t *cf, double *out);
/* giveProjectedCovar, CovarianceForcing.ipp:38-109: out = M C_f M^T for a
 * dense M (rows x num_dofs, row-major, host); out is rows x rows. */
int32_t sfc_covar_forcing_projected(sfc_covar_forcing_t *cf, const sfc_hparams_t *hp,
                                    const double *M, int64_t rows, double *out);

/* ---- statX: ForwardGaussRHS ------------------------------------------------ */
/* ForwardGaussRHS(solver, covarForcing, regEps), statX/infer/ForwardGaussRHS.hpp:61-64 */
int32_t sfc_forward_gauss_create(sfc_system_t *sys, sfc_covar_forcing_t *cf, double reg_eps,
                                 sfc_forward_gauss_t **out);
int32_t sfc_forward_gauss_destroy(sfc_forward_gauss_t *fg);
/* setProjectionMatrix, ForwardGaussRHS.hpp:71-74; P given as CSR
 * (num_sensors x num_dofs). */
int32_t sfc_forward_gauss_set_projection(sfc_forward_gauss_t *fg, int64_t num_sensors,
                                         const int64_t *indptr, const int32_t *indices,
                                         const double *data);
/* updateSolution, ForwardGaussRHS.hpp:95-139: R = P A^-1 from one block
 * adjoint solve, mean = R F, C_s = R C_f R^T + (sigma_f reg)^2 P P^T. */
int32_t sfc_forward_gauss_update(sfc_forward_gauss_t *fg, const sfc_hparams_t *hp);
/* giveProjectedMeanU / giveProjectedCovarU, ForwardGaussRHS.hpp:77-92 */
int32_t sfc_forward_gauss_mean(const sfc_forward_gauss_t *fg, double *out);
int32_t sfc_forward_gauss_covar(const sfc_forward_gauss_t *fg, double *out);

/* ---- statX: LikelihoodKOH ---------------------------------------------------- */
/* LikelihoodKOH(forwardGauss, mismatchCov) with MismatchCovariance(sensorCoords),
 * statX/infer/LikelihoodKOH.hpp:66-72, MismatchCovariance.hpp:62-67;
 * sensor_coords is num_sensors x dim. */
int32_t sfc_koh_create(sfc_forward_gauss_t *fg, const double *sensor_coords, int32_t dim,
                       sfc_koh_t **out);
int32_t sfc_koh_destroy(sfc_koh_t *koh);
/* setSensorValues, LikelihoodKOH.hpp:79-84: Y is num_sensors x num_readings,
 * row-major. */
int32_t sfc_koh_set_sensor_values(sfc_koh_t *koh, const double *Y, int32_t num_readings);
/* giveLogLikelihood, LikelihoodKOH.ipp:75-120 (FP64 sensor-space Cholesky) */
int32_t sfc_koh_log_likelihood(sfc_koh_t *koh, const sfc_hparams_t *hp, double *out);
/* giveProjFEconditionedData, LikelihoodKOH.ipp:311-361: posterior mean
 * (num_sensors) and covariance (num_sensors^2) at the sensors. */
int32_t sfc_koh_proj_conditioned(sfc_koh_t *koh, const sfc_hparams_t *hp, double *mean,
                                 double *cov);
/* giveFEconditionedDataWoodbury, LikelihoodKOH.ipp:442-508: full-field
 * posterior mean (num_dofs) and covariance (num_dofs^2; may be NULL).  Needs
 * num_dofs adjoint solves, so it is limited to num_dofs <= 8192. */
/* giveLogLikelihood (LikelihoodKOH.ipp:75-120) for n hyperparameter sets at
 * once against the forward model of the last sfc_forward_gauss_update: the
 * sets differ in rho and the mismatch parameters (their forcing parameters
 * are not used), one CTA each, one launch per chunk -- the inner loop of
 * hyperparameter MCMC (hyperParamLearning.hpp:90-249) over many proposals or
 * chains.  A set whose total covariance is not positive definite, or whose
 * quadratic term is not negative, gets NaN. */
int32_t sfc_koh_log_likelihood_batch(sfc_koh_t *koh, const sfc_hparams_t *hps, int32_t n, double *loglik);
int32_t sfc_koh_woodbury(sfc_koh_t *koh, const sfc_hparams_t *hp, double *mean, double *cov);
/* The posterior mean field of giveFEconditionedDataWoodbury
 * (LikelihoodKOH.ipp:442-508) for any mesh size: the same quantity as
 * sfc_koh_woodbury's mean, from the adjoint solution of the last
 * sfc_forward_gauss_update plus num_sensors + 1 forward solves (G = C_u P^T
 * = A^-1 C_f R^T + (sigma_f reg)^2 P^T, ubar = A^-1 F) and sensor-space FP64
 * Cholesky solves, instead of the num_dofs solves of the unprojected prior.
 * mean: num_dofs, host. */
int32_t sfc_koh_woodbury_mean(sfc_koh_t *koh, const sfc_hparams_t *hp, double *mean);

/* ---- first-order material uncertainty ------------------------------------------ */
/* Replaces statX::infer::ForwardPerturbation (ForwardPerturbation.hpp:109-195)
 * with CovarianceMaterial (CovarianceMaterial.hpp) and the stiffness
 * derivative of ElementPotential (ElementPotential.ipp:225-237), Poisson
 * element kinds.  Built on a ForwardGaussRHS object (its system, forcing
 * covariance and projection).  sfc_perturbation_update runs the forward
 * model (adjoint and forward solves) and forms
 *   C_s = R C_f R^T + sum_{e,d} C_m(e,d) R A'_e (A^-1 C_f A^-T + u u^T) A'_d^T R^T
 *         + (reg material_sigma)^2 P P^T,     mean = P u,
 * C_m the squared-exponential covariance ("material.sigma",
 * "material.length") of the element centroids, through a pivoted Cholesky
 * factor of C_m (stopped when the largest remaining diagonal is below
 * factor_tol * material_sigma^2, or at max_rank columns; rank returns the
 * columns used).  reg: the reference's regFactor (default 1e-4). */
typedef struct sfc_perturbation sfc_perturbation_t;
int32_t sfc_perturbation_create(sfc_forward_gauss_t *fg, double reg, sfc_perturbation_t **out);
int32_t sfc_perturbation_destroy(sfc_perturbation_t *pt);
int32_t sfc_perturbation_update(sfc_perturbation_t *pt, const sfc_hparams_t *hp, double material_sigma,
                                double material_length, double factor_tol, int32_t max_rank, int32_t *rank);
/* giveProjectedMeanU / giveProjectedCovarU: num_sensors, num_sensors^2. */
int32_t sfc_perturbation_mean(const sfc_perturbation_t *pt, double *mean);
int32_t sfc_perturbation_covar(const sfc_perturbation_t *pt, double *cov);

/* ---- allocation-free log-likelihood ----------------------------------------- */
/* No counterpart in the reference.  The same quantity as
 * sfc_koh_log_likelihood (LikelihoodKOH::giveLogLikelihood), for callers that
 * cannot allocate device memory while they run: an MCMC loop on a stream it
 * owns, where cudaMalloc / cudaFree would synchronise the whole device, or an
 * application that gives this library a fixed memory budget at start-up.
 * Everything is caller-owned DEVICE memory on the current device:
 *   mean_dev          num_sensors          prior mean at the sensors
 *   cov_dev           num_sensors^2        prior covariance C_s (row-major)
 *   sensor_coords_dev num_sensors x 3      sensor coordinates (first dim used)
 *   y_dev             num_sensors x num_readings readings (row-major)
 *   loglik_dev        1                    result
 *   info_dev          1                    0, k+1 if the Cholesky pivot k failed,
 *                                          -1 for a non-negative quadratic term
 * The kernel is launched on `stream` (a cudaStream_t, NULL = default stream)
 * and nothing is allocated: the scratch is a fixed device array of
 * 128*128 + 128*64 doubles (192 KiB, held by every device that loads the
 * library until exit), so num_sensors <= 128 and num_readings <= 64, else
 * SFC_ERR_TOO_LARGE.  Every call looks up that array's address in the
 * current context (a host-side lookup); under CUDA's lazy module loading the
 * first call in a context is the one that loads the library's kernels, which
 * allocates the array and the code and may synchronise: make one call at
 * start-up, before any stream capture and outside the loop that must not
 * allocate (and again after cudaDeviceReset).  All calls share the array:
 * calls that can overlap on the GPU race and must be ordered by the caller. */
int32_t sfc_koh_log_likelihood_noalloc(const double *mean_dev, const double *cov_dev,
                                       const double *sensor_coords_dev, int32_t dim,
                                       const double *y_dev, int32_t num_sensors,
                                       int32_t num_readings, const sfc_hparams_t *hp,
                                       double *loglik_dev, int32_t *info_dev, void *stream);

/* ---- learned preconditioner ------------------------------------------------- */
/* No counterpart in the reference (it factorises with Eigen::SparseLU,
 * SystemSolveEigenSparse.hpp).  A message-passing network on the matrix
 * graph: encoder (2 -> 64), 3 layers h' = relu(W [h ; Ahat h] + b) with
 * W 64 x 128 in BF16 on tensor cores (FP32 accumulate), linear decoder, where
 * Ahat = D^-1/2 S D^-1/2 is the unit-diagonal scaling of the system's
 * symmetric operator.  M(r) = D^-1 r + |D^-1/2 r| D^-1/2 y(r): Jacobi plus a
 * learned correction (the untrained network is exactly Jacobi).  Parameters
 * are FP32 masters of sfc_mpnn_num_params() floats, trained with Adam on
 * residual/error pairs (S e = r) from Jacobi-PCG iterates, loss = the S-norm
 * of the error of M(r), scaled by 1/|D^-1/2 r|^2.  The system passed to the
 * calls below must have its matrix assembled and constraints applied. */
typedef struct sfc_mpnn sfc_mpnn_t;
int64_t sfc_mpnn_num_params(void);
int32_t sfc_mpnn_create(sfc_ctx_t *ctx, uint64_t seed, sfc_mpnn_t **out);
int32_t sfc_mpnn_destroy(sfc_mpnn_t *net);
int32_t sfc_mpnn_get_params(const sfc_mpnn_t *net, float *params, int64_t n);
int32_t sfc_mpnn_set_params(sfc_mpnn_t *net, const float *params, int64_t n);
/* Checkpoint: parameters and Adam moments (binary, this library's format). */
int32_t sfc_mpnn_save(const sfc_mpnn_t *net, const char *path);
int32_t sfc_mpnn_load(sfc_mpnn_t *net, const char *path);
/* Loss and its parameter gradient (n = sfc_mpnn_num_params floats; grad may
 * be NULL) for one pair of host vectors r, e of length num_dofs. */
int32_t sfc_mpnn_loss_grad(sfc_mpnn_t *net, sfc_system_t *sys, const double *r, const double *e,
                           double *loss, float *grad);
/* z = M(r) for host vectors of length num_dofs, by the inference kernels
 * flexible CG uses (activations stored in BF16, the values the tensor-core
 * products round them to; training keeps them in FP32). */
int32_t sfc_mpnn_apply(sfc_mpnn_t *net, sfc_system_t *sys, const double *r, double *z);
/* Training on the GPU.  Pairs come from Jacobi-PCG on the system's current
 * right-hand side: the initial residual and the iterates after k iterations,
 * k spaced geometrically up to the iteration where |r_k|/|b| first drops
 * below pair_floor, against the solution converged to 1e-12 (later iterates
 * carry too few digits of their error).  Each Adam step sums the loss
 * gradients of `batch` pairs drawn at random (seeded); with normalize, a
 * pair's loss is divided by the loss of plain Jacobi on it, so the loss
 * reads as the fraction of Jacobi's error energy left (1.0 = no gain). */
typedef struct sfc_mpnn_train_options {
    int32_t steps;      /* Adam steps                                          */
    int32_t batch;      /* pairs per step                                      */
    int32_t max_pairs;  /* pairs from the PCG run (1..64)                      */
    int32_t normalize;  /* 1: loss relative to Jacobi's (see above)            */
    double lr;          /* Adam learning rate                                  */
    double pair_floor;  /* last iterate: |r_k|/|b| >= pair_floor, in (0, 1)    */
    uint64_t seed;      /* pair sampling                                       */
} sfc_mpnn_train_options_t;
int32_t sfc_mpnn_default_train_options(sfc_mpnn_train_options_t *opt);
/* loss_history (may be NULL): opt->steps doubles, the batch loss per step. */
int32_t sfc_mpnn_train(sfc_mpnn_t *net, sfc_system_t *sys, const sfc_mpnn_train_options_t *opt,
                       double *loss_history);
/* Attach (net != NULL) or detach the network used by SFC_SOLVER_FCG_MPNN. */
int32_t sfc_system_set_mpnn(sfc_system_t *sys, sfc_mpnn_t *net);

/* ---- batched instances (MCMC proposals) -------------------------------------- */
/* No single reference counterpart: the reference evaluates one statFEM
 * instance at a time (ForwardGaussRHS::updateSolution, ForwardGaussRHS.hpp:
 * 95-139; LikelihoodKOH::giveLogLikelihood and giveProjFEconditionedData,
 * LikelihoodKOH.ipp:75-120, 311-361), once per MCMC proposal
 * (hyperParamLearning.hpp:90-249).  Here num_instances 2-D Poisson statFEM
 * instances are one union mesh (SFC_ELEM_TRI3_POISSON): instance i owns dofs
 * [dof_offset[i], dof_offset[i+1]), the (grid_side[i]+1)^2 nodes of the unit
 * square grid, x fastest (checked).  bc_dofs: the homogeneous Dirichlet dofs
 * of all instances.  Sensors: num_sensors[i] <= 32 per instance, the rows of
 * P as num_instances x 32 x 3 global dofs (-1 = unused) and weights, and
 * num_instances x 32 x 2 coordinates (for the mismatch covariance).
 * forcing_mean: the constant body force f.  cluster_size: CTAs per instance
 * (0: 8; the largest size the device can co-schedule is used).
 * One sfc_batch_run assembles all instances (coefficients from
 * sfc_batch_set_coefficients, one value per element of the union mesh) and
 * runs one persistent kernel, captured once in a CUDA graph, that solves the
 * ns adjoint systems of every instance (FP32 block PCG, FP64 residual
 * refinement to the relative residual tol), forms mean and C_s at the
 * sensors (C_s with the Kronecker-factored forcing covariance) and evaluates
 * the log-likelihood and the posterior mean / covariance at the sensors in
 * FP64.  Per-instance status: SFC_OK, SFC_ERR_NOT_CONVERGED or
 * SFC_ERR_NOT_SPD (breakdown, NaN, Cholesky failure); a failing instance
 * does not stop the others. */
typedef struct sfc_batch sfc_batch_t;
int32_t sfc_batch_create(sfc_ctx_t *ctx, const sfc_mesh_t *mesh, int32_t num_instances,
                         const int64_t *dof_offset, const int32_t *grid_side, const uint32_t *bc_dofs,
                         int64_t num_bc, const int32_t *num_sensors, const int32_t *sensor_dofs,
                         const double *sensor_weights, const double *sensor_coords, double forcing_mean,
                         int32_t cluster_size, sfc_batch_t **out);
int32_t sfc_batch_destroy(sfc_batch_t *batch);
/* The launch shape in use: CTAs per cluster and CTAs in the grid. */
int32_t sfc_batch_cluster_size(const sfc_batch_t *batch, int32_t *cluster, int32_t *grid);
/* tol: true relative residual of every adjoint column (default 1e-8);
 * inner_tol: reduction of a column's FP32 recurrence residual between two
 * FP64 residual replacements (default 1e-2; the search direction is kept
 * across them); max_iter: inner iteration cap per instance. */
int32_t sfc_batch_set_solver(sfc_batch_t *batch, double tol, double inner_tol, int32_t max_iter);
int32_t sfc_batch_set_coefficients(sfc_batch_t *batch, const double *elem_coeff);
/* One sfc_hparams_t per instance (each proposal has its own), reg: the
 * ForwardGaussRHS regularisation (C_s += (sigma_f reg)^2 P P^T). */
int32_t sfc_batch_set_hparams(sfc_batch_t *batch, const sfc_hparams_t *hp, double reg);
/* y: num_instances x 32 x num_readings (rows past num_sensors ignored). */
int32_t sfc_batch_set_readings(sfc_batch_t *batch, const double *y, int32_t num_readings);
int32_t sfc_batch_run(sfc_batch_t *batch);
/* Autotuner: times the batch kernel with 1, 2, 4, 8 and 16 CTAs per
 * instance on the current inputs and keeps the fastest (cached per device
 * and shape class, see sfc_autotune_save; remeasure = 0 takes a cached
 * choice when there is one). */
int32_t sfc_batch_autotune(sfc_batch_t *batch, int32_t remeasure, int32_t *cluster);
/* Host copies of the last run's results (any pointer may be NULL):
 * loglik (n), mean_s (n x 32), cov_s (n x 32 x 32), post_mean (n x 32),
 * post_cov (n x 32 x 32), status (n), iterations (n, inner iterations). */
int32_t sfc_batch_results(sfc_batch_t *batch, double *loglik, double *mean_s, double *cov_s,
                          double *post_mean, double *post_cov, int32_t *status, int32_t *iterations);

/* ---- autotuner ----------------------------------------------------------------- */
/* No reference counterpart.  Launch shapes chosen by measurement on the
 * caller's problem and kept in a process-wide table keyed by device and
 * problem shape class (dof count, dofs per node, row length, right-hand
 * sides); remeasure = 0 reuses a stored choice for the same class.
 * sfc_autotune_spmv: lanes per row of the FP64 SpMV (4, 8, 16 or 32), set
 * on the system.  sfc_autotune_block_solver: block width and preconditioner
 * of SFC_SOLVER_PCG_MIXED, by the time to solution of the first
 * min(nrhs, 128) of the given right-hand sides (rhs: nrhs x num_dofs, host,
 * as sfc_solve_transpose), set on the system's options (tol and max_iter
 * kept) and returned in best. */
int32_t sfc_autotune_spmv(sfc_system_t *sys, int32_t remeasure, int32_t *lanes);
int32_t sfc_autotune_block_solver(sfc_system_t *sys, const double *rhs, int32_t nrhs, int32_t remeasure,
                                  sfc_solver_options_t *best);
/* The table as text, one "key value" line per shape class. */
int32_t sfc_autotune_save(const char *path);
int32_t sfc_autotune_load(const char *path);
int32_t sfc_autotune_clear(void);

/* ---- two-level preconditioner: the aggregation, on the host --------------- */
/* No reference counterpart (the reference factorises directly).  The box
 * aggregation that SFC_PRECOND_TWO_LEVEL builds for a mesh: a grid of about
 * `size` nodes per axis (0: 8) over the nodes' bounding box, about max_aggs
 * boxes at most (the library uses 512 on 3-dof meshes, 2048 on scalar ones),
 * halved per axis until every element's nodes lie in boxes at most one apart;
 * node_agg[num_nodes] receives each node's aggregate (non-empty boxes in box
 * order), boxes_per_axis[3] (nullable) the final grid.  Needs no device.
 * SFC_ERR_BAD_ARG when no grid satisfies the rule (degenerate input). */
int32_t sfc_coarse_boxes(const double *coords, int64_t num_nodes, const uint32_t *conn, int64_t num_elems,
                         int32_t nodes_per_elem, int32_t size, int32_t max_aggs, int32_t *node_agg,
                         int32_t *num_aggs, int32_t *boxes_per_axis);

#ifdef __cplusplus
}
#endif
#endif
