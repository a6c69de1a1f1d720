/* neon_b200.h -- C-ABI of the B200-native solid-mechanics Newton step.
 *
 * Drop-in for neon's nonlinear static solid path:
 *   mechanics::static_matrix<mechanics::solid::mesh<solid::submesh>>
 *     (src/assembler/mechanics/static_matrix.hpp:29-467),
 *   its element kernels and internal-variable update
 *     (src/mesh/mechanics/solid/submesh.cpp:66-269, mesh.cpp:56-76),
 *   the constitutive plugins on the path
 *     (src/constitutive/mechanics/solid/{isotropic_linear_elasticity,compressible_neohooke,
 *      small_strain_J2_plasticity,gaussian_affine_microsphere,affine_microsphere,
 *      nonaffine_microsphere}.cpp),
 *   and the linear_solver plugin (src/solver/linear/linear_solver.hpp:13-71).
 *
 * Plain C types only.  Every call returns an nb2_status; nothing throws across the boundary.
 * Host pointers are read (or written) only during the call.  A context is single-stream and not
 * thread-safe; several contexts may run on several streams.
 */
#ifndef NEON_B200_H
#define NEON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The recoverable numerical failures (1-6, 9) correspond to neon's
 * computational_error (src/exceptions.hpp:14-17), which static_matrix::solve answers with a
 * cutback (static_matrix.hpp:168-182).  NB2_E_INPUT corresponds to std::domain_error. */
typedef enum nb2_status {
    NB2_OK = 0,
    NB2_E_NEG_DETJ = 1,      /* negative det F (submesh.cpp:239-269) */
    NB2_E_NAN = 2,           /* FE_INVALID after an update / solve (submesh.cpp:196-207) */
    NB2_E_RETURN_MAP = 3,    /* radial return did not converge (small_strain_J2_plasticity.cpp:132-153) */
    NB2_E_CG_MAXIT = 4,      /* CG reached its iteration limit (linear_solver.cpp:104-108) */
    NB2_E_CG_BREAKDOWN = 5,  /* CG denominator not positive / not finite */
    NB2_E_TIMEOUT = 6,       /* a bounded device wait gave up */
    NB2_E_INPUT = 7,         /* invalid argument */
    NB2_E_CUDA = 8,          /* CUDA runtime error (message in nb2_last_error) */
    NB2_E_NEWTON_MAXIT = 9,  /* Newton iteration limit (static_matrix.hpp:451-454) */
    NB2_E_CUTBACK_LIMIT = 10 /* too many load cutbacks (adaptive_time_step.cpp:61-92) */
} nb2_status;

/* Constitutive models on the path (names as in constitutive_model_factory.cpp:26-161). */
typedef enum nb2_model {
    NB2_ISOTROPIC_LINEAR_ELASTICITY = 0, /* "isotropic_linear_elasticity" */
    NB2_NEOHOOKE = 1,                    /* "neohooke" */
    NB2_SMALL_STRAIN_J2_PLASTICITY = 2,  /* "J2_plasticity", "finite_strain": false */
    NB2_GAUSSIAN_AFFINE_MICROSPHERE = 3, /* "microsphere", "affine", "gaussian", "BO21"/"BO33" */
    NB2_LANGEVIN_AFFINE_MICROSPHERE = 4, /* "microsphere", "affine", "langevin", "BO21"
                                            (affine_microsphere.cpp:23-112) */
    NB2_NONAFFINE_MICROSPHERE = 5        /* "microsphere", "nonaffine", "BO21"
                                            (nonaffine_microsphere.cpp:29-175) */
} nb2_model;

/* Precision of the stiffness / inner linear solve. */
typedef enum nb2_precision {
    NB2_FP64 = 0,  /* everything FP64: parity path */
    NB2_MIXED = 1  /* FP32 tangent, SpMV and inner CG; FP64 residual, norms, dots, return map, det F */
} nb2_precision;

typedef struct nb2_ctx nb2_ctx;

/* Mesh: one element group (neon submesh).  Coordinates node-major [num_nodes][3]; DOF
 * 3*node + component (mesh/dof_allocator.hpp:39-47).  Connectivity element-major
 * [num_elements][nodes_per_element] in neon's local ordering (hex8: interpolations/hexahedron.cpp
 * corner order; tet4 after node_ordering_adapter.cpp:63-68).  hex8 uses the 8-point Gauss rule,
 * tet4 the 1-point rule (interpolation_factory.cpp:36-97). */
typedef struct nb2_mesh_desc {
    int32_t num_nodes;
    const double* coordinates;
    int32_t num_elements;
    int32_t nodes_per_element; /* 8 (hex8) or 4 (tet4) */
    const int32_t* connectivity;
} nb2_mesh_desc;

/* Material parameters as neon stores them: bulk modulus K and shear modulus G
 * (isotropic_elastic_property.cpp:10-43, lambda = K - 2G/3), yield stress and linear isotropic
 * hardening (isotropic_elastic_plastic.cpp:31-38), segments per chain
 * (micromechanical_elastomer.cpp:13-21; used by Langevin statistics and the non-affine model,
 * required but unused by Gaussian statistics), the non-affine stretch parameter p
 * (nonaffine_microsphere.cpp:17-25; non-affine model only). */
typedef struct nb2_material {
    int32_t model; /* nb2_model */
    double bulk_modulus;
    double shear_modulus;
    double yield_stress;
    double isotropic_hardening_modulus;
    double segments_per_chain;
    double nonaffine_stretch_parameter;
    int32_t unit_sphere_points; /* microsphere models: 21 (BO21; also when 0) or 33 (BO33),
                                   unit_sphere_quadrature.cpp:10-91 */
} nb2_material;

/* A time/value table applied to a DOF list: a Dirichlet boundary (mesh/boundary/nodal_value.cpp,
 * dirichlet.hpp) or a nodal force.  Values are interpolated linearly in time
 * (mesh/boundary/boundary.cpp:55-85).  weights (nullable, forces only) scales the value per DOF:
 * f_ext[dof[i]] += weights[i] * value(t). */
typedef struct nb2_dof_table {
    const int32_t* dofs;
    int32_t num_dofs;
    const double* times;
    const double* values;
    int32_t num_points;
    const double* weights;
} nb2_dof_table;

/* nonlinear_options (static_matrix.hpp:109-143), time/increments (adaptive_time_step.cpp),
 * linear_solver tolerance / maximum_iterations (linear_solver_factory.cpp:27-65). */
typedef struct nb2_solver_options {
    double residual_tolerance;
    double displacement_tolerance;
    int32_t linear_iterations; /* maximum Newton iterations per increment */
    int32_t absolute_tolerance;
    double period, initial_increment, minimum_increment, maximum_increment;
    int32_t adaptive;
    double cg_tolerance;
    int32_t cg_maximum_iterations;
    int32_t precision;         /* nb2_precision */
    double mixed_inner_tolerance; /* NB2_MIXED: the FP32 residual is replaced by the FP64 one
                                     after each reduction by this factor (1e-2 measured best) */
    int32_t use_graphs;        /* capture CG iteration blocks in CUDA graphs */
} nb2_solver_options;

typedef struct nb2_solve_report {
    int32_t status;
    int32_t load_steps;
    int64_t newton_iterations;
    int64_t cg_iterations;
    double seconds_total;           /* wall time of the load stepping, after the context's
                                       solver buffers are set up (once per context) */
    double seconds_update_assembly; /* device time of the element kernels */
    double seconds_solve;           /* device time of the linear solves */
    char message[256];
} nb2_solve_report;

/* One row per Newton iteration: step time, iteration, CG iterations, displacement norm,
 * residual norm (static_matrix.hpp:385-400). */
typedef struct nb2_newton_log {
    double step_time;
    int32_t iteration;
    int32_t cg_iterations;
    double displacement_norm;
    double force_norm;
} nb2_newton_log;

/* ---------------------------------------------------------------------------------------- */
/* Context                                                                                  */
/* ---------------------------------------------------------------------------------------- */

/* Builds the mesh on the device, the CSR pattern (sparsity_pattern.hpp:18-48: per row the sorted
 * unique coupled columns, explicit zeros kept), the element->block slot map and the
 * quadrature-point state (submesh.cpp:26-52).  Replaces solid::mesh / submesh construction. */
int nb2_create(const nb2_mesh_desc* mesh, const nb2_material* material, nb2_ctx** out);
int nb2_destroy(nb2_ctx* ctx);
/* Last error message of this context (or of the last failed nb2_create when ctx is NULL). */
int nb2_last_error(const nb2_ctx* ctx, char* buffer, size_t size);
/* Run all work of this context on a caller stream (cudaStream_t passed as void*). */
int nb2_set_stream(nb2_ctx* ctx, void* stream);

/* How element passes add element contributions into K and f_int (hex8, FP64).  No reference
 * counterpart: neon adds with OpenMP atomics (thread_safe_plugin.hpp:7-23), so its sums run in
 * a thread-dependent order.
 *   NB2_SCATTER_RED       (default for nb2_update_internal_variables / nb2_assemble /
 *                         nb2_update_assemble_device) every element in one launch, terms added
 *                         with red.global.add into zeroed arrays: the fastest; the order of the
 *                         additions, and so the last bits, can change from run to run.
 *   NB2_SCATTER_COLOURED  one launch per element colour (elements of a colour share no node),
 *                         so an entry receives at most one addition per launch and its sum runs
 *                         in colour order: the same inputs give bit-identical K and f_int.
 * nb2_static_solve always uses the coloured launches, whatever this setting: its Newton
 * iterates, CG and solution are then bit-reproducible (the element passes are ~1% of a Newton
 * step).  tet4 meshes, the anisotropic microsphere tangent, FP32 K and batched instances always
 * use one launch. */
#define NB2_SCATTER_RED 0
#define NB2_SCATTER_COLOURED 1
int nb2_set_scatter_mode(nb2_ctx* ctx, int32_t mode);
int nb2_get_sizes(const nb2_ctx* ctx, int32_t* num_dofs, int64_t* nnz, int64_t* num_blocks);
/* Number of kernels this library launched for the context so far. */
int nb2_launch_count(const nb2_ctx* ctx, int64_t* launches);

/* Per-element shear modulus (replaces the material G of the microsphere model per element). */
int nb2_set_element_shear_modulus(nb2_ctx* ctx, const double* shear_modulus);
/* Per-element bulk and shear modulus ([num_elements] each, either may be NULL) replacing the
 * material's K, G (lambda = K - 2G/3) for linear elasticity, neo-Hooke and the microsphere:
 * element groups of different materials (neon builds one submesh and one constitutive model per
 * group, mesh.cpp:36-42) in a single context, as the batched solves do. */
int nb2_set_element_moduli(nb2_ctx* ctx, const double* bulk_modulus, const double* shear_modulus);

/* ---------------------------------------------------------------------------------------- */
/* Element-level drop-ins (host buffers)                                                   */
/* ---------------------------------------------------------------------------------------- */

/* CSR export, bit-exact with neon's Eigen RowMajor pattern: rowptr[num_dofs+1], col[nnz]
 * (compute_sparsity_pattern, sparsity_pattern.hpp:18-48). */
int nb2_export_pattern(nb2_ctx* ctx, int32_t* rowptr, int32_t* col);

/* mesh.update_internal_variables(u, dt) (mesh.cpp:56-70): x = X + u, deformation measures,
 * det F check, constitutive update of the current (trial) state; stores stress and tangent
 * coefficients per quadrature point for the calls below. */
int nb2_update_internal_variables(nb2_ctx* ctx, const double* u, double time_step_size);

/* static_matrix::assemble_stiffness (static_matrix.hpp:243-277) into CSR values K[nnz] and
 * compute_internal_force (:189-203) into f_int[num_dofs], from the state of the last update.
 * Either pointer may be NULL. */
int nb2_assemble(nb2_ctx* ctx, double* K_values, double* f_int);

/* Matrix-free tangent product y = K v (host buffers, FP64) with the tangent of the last
 * nb2_update_internal_variables -- the same K nb2_assemble returns, applied element by element
 * without forming it (the defect residual of the mixed-precision solve). */
int nb2_apply_tangent(nb2_ctx* ctx, const double* v, double* y);
/* The same product with the FP32 matrix-free operator the mixed-precision PCG iterates with
 * (FP32 relative coordinates and tangent coefficients per quadrature point, node-ordered sums;
 * FP64 in and out).  Equals nb2_apply_tangent to FP32 rounding.  No reference counterpart. */
int nb2_apply_tangent_fp32(nb2_ctx* ctx, const double* v, double* y);

/* submesh::tangent_stiffness(element) (submesh.cpp:66-80): one element's tangent stiffness at
 * the state of the last nb2_update_internal_variables, dense, row-major, in neon's local DOF
 * order (3a + k for local node a): Ke [3 npe][3 npe] (576 doubles for hex8, 144 for tet4; host).
 * A per-element getter for checks and debugging; nb2_assemble is the batched path. */
int nb2_element_stiffness(nb2_ctx* ctx, int64_t element, double* Ke);

/* submesh::save_internal_variables (submesh.cpp:54-64): commit (1) or revert (0). */
int nb2_save_internal_variables(nb2_ctx* ctx, int32_t converged);

/* Quadrature-point outputs of the last update: which = 0 Cauchy stress [nqp][9] (row-major
 * 3x3), 1 det F [nqp], 2 plastic strain [nqp][9], 3 accumulated plastic strain [nqp]. */
int nb2_get_quadrature_values(nb2_ctx* ctx, int32_t which, double* out);

/* Quadrature values of the last update extrapolated to the nodes and averaged, the fields neon
 * writes to its .vtu output (submesh::nodal_averaged_variable, submesh.cpp:271-344, and
 * average_internal_variable, io/post/node_averaged_variables.hpp:18-41; extrapolation matrix
 * of shape_function.hpp:70-100).  which = 0 Cauchy stress [num_nodes][9], 1 det F [num_nodes],
 * 2 plastic strain [num_nodes][9], 3 accumulated plastic strain [num_nodes], 4 von Mises stress
 * [num_nodes].  Host output. */
int nb2_nodal_averaged_variable(nb2_ctx* ctx, int32_t which, double* out);

/* Non-follower loads (nonfollower_load_boundary, mechanics/solid/boundary/nonfollower_load.cpp:
 * 12-121): the nodal external-force vector of one load boundary per unit load value, in the
 * initial configuration, computed on the device.  The Newton driver scales it by the boundary's
 * time table (pass it as a weighted table in nb2_static_solve's nodal_forces).
 *   NB2_LOAD_TRACTION   surface_load::external_force (mesh/boundary/neumann.hpp:69-133): f[3a+k]
 *                       = sum_q w N_a |X,xi x X,eta| for the given component k;
 *   NB2_LOAD_PRESSURE   pressure::external_force (pressure.cpp:9-37): f[3a+i] = -sum_q w N_a n_i
 *                       |X,xi x X,eta|, n the unit normal X,xi x X,eta / |..| (positive pressure
 *                       compresses the surface; component is ignored);
 *   NB2_LOAD_BODY_FORCE volume_load::external_force (neumann.hpp:135-192) over the context's
 *                       elements: f[3a+k] = sum_q w N_a det(X dN).
 * faces [num_faces][nodes_per_face]: quad4 (4-point rule, or the 1-point rule when
 * reduced_quadrature is set) or tri3 (1-point rule) boundary faces in neon's local node order
 * (surface loads only; NULL for a body force).  f_out [num_dofs] (host) is overwritten. */
#define NB2_LOAD_TRACTION 0
#define NB2_LOAD_PRESSURE 1
#define NB2_LOAD_BODY_FORCE 2
int nb2_nonfollower_load(nb2_ctx* ctx, int32_t kind, int32_t component, const int32_t* faces,
                         int32_t num_faces, int32_t nodes_per_face, int32_t reduced_quadrature,
                         double* f_out);

/* static_matrix::enforce_dirichlet_conditions (static_matrix.hpp:279-320) on host CSR values
 * laid out as nb2_export_pattern: zero row and column of each listed DOF, keep the diagonal,
 * b[dof] = 0. */
int nb2_apply_dirichlet(nb2_ctx* ctx, const int32_t* dofs, int32_t num_dofs, double* K_values,
                        double* b);

/* ---------------------------------------------------------------------------------------- */
/* Linear solver plugin                                                                     */
/* ---------------------------------------------------------------------------------------- */

/* conjugate_gradient::solve (linear_solver.cpp:67-109) on a caller CSR (host buffers): Jacobi
 * PCG from x0 = 0, stop when ||r||^2 < max(tol^2 ||b||^2, DBL_MIN); NB2_E_CG_MAXIT when the
 * iteration count reaches maximum_iterations.  FP64 on the device. */
int nb2_pcg_solve(int32_t n, const int32_t* rowptr, const int32_t* col, const double* values,
                  const double* b, double* x, double tolerance, int32_t maximum_iterations,
                  int32_t* iterations, double* error);

/* Allocation-free variant of nb2_pcg_solve.  No counterpart in the reference: it exists for
 * callers that must not allocate device memory during a solve (codes that place every device
 * byte through their own pool or arena, or that must not trigger allocator growth mid-step).
 * The matrix (rowptr, col, values), b and x are DEVICE pointers the caller owns; the solver's
 * work vectors, reduction partials and scalars live in a fixed workspace inside the library
 * (NB2_NOALLOC_MAX_ROWS rows, about 4.2 MB, held by every GPU that loads the library until the
 * process exits).  n > NB2_NOALLOC_MAX_ROWS returns NB2_E_INPUT, as do row pointers that are not
 * monotone from 0 and column indices outside [0, n); the check cannot tell a rowptr[n] larger
 * than the caller's col/values buffers.  Each call looks the workspace up (cudaGetSymbolAddress)
 * with the caller's device current; the first call on a device loads the library there, so make
 * it before any stream capture.  The call allocates nothing but is not asynchronous: it blocks
 * the host on its stream after the input check and every few dozen iterations to read the
 * convergence flag, so it cannot run inside a stream capture.  Pass a stream created by the
 * caller (cudaStreamNonBlocking); NULL means the legacy default stream, which synchronises with
 * the device's other blocking streams.  All calls share the one workspace (it keeps the last
 * call's contents; the solver re-zeroes what must start at zero), so calls that overlap on the
 * GPU race: serialise them.  Same algorithm, stopping rule and status codes as nb2_pcg_solve. */
#define NB2_NOALLOC_MAX_ROWS 131072
int nb2_pcg_solve_noalloc(int32_t n, const int32_t* rowptr, const int32_t* col,
                          const double* values, const double* b, double* x, double tolerance,
                          int32_t maximum_iterations, void* stream, int32_t* iterations,
                          double* error);

/* ---------------------------------------------------------------------------------------- */
/* Newton driver: static_matrix                                                             */
/* ---------------------------------------------------------------------------------------- */

/* static_matrix::solve() (static_matrix.hpp:145-187): adaptive load stepping, full Newton with
 * Dirichlet lifting, device-resident PCG, commit/revert and cutback.  Dirichlet tables are taken
 * in the order neon iterates them (boundary names sorted, then x, y, z).  u_out (nullable,
 * [num_dofs]) receives the final displacement, log (nullable) up to max_log Newton rows. */
int nb2_static_solve(nb2_ctx* ctx, const nb2_solver_options* options,
                     const nb2_dof_table* dirichlet, int32_t num_dirichlet,
                     const nb2_dof_table* nodal_forces, int32_t num_nodal_forces, double* u_out,
                     nb2_solve_report* report, nb2_newton_log* log, int32_t max_log);

/* ---------------------------------------------------------------------------------------- */
/* Adjoint                                                                                  */
/* ---------------------------------------------------------------------------------------- */

/* Gradient of an objective J(u) with respect to the per-element shear modulus of the Gaussian
 * (gaussian_affine_microsphere.cpp:23-88) or Langevin (affine_microsphere.cpp:23-112) affine
 * microsphere model, at the equilibrium left by
 * the last nb2_static_solve on this context (its displacement and Dirichlet set).  dJdu: host
 * [num_dofs]; dJdG: host [num_elements].  Solves K lambda = dJ/du (K symmetric; precision
 * NB2_FP64 or NB2_MIXED, relative tolerance `tolerance`) and evaluates
 * dJ/dG_e = -lambda^T df_int/dG_e element by element, recomputing the quadrature-point state.
 * Extends the reference (neon has no sensitivities) for its material parameter G. */
int nb2_adjoint_shear_gradient(nb2_ctx* ctx, const double* dJdu, int32_t precision,
                               double tolerance, int32_t maximum_iterations, double* dJdG,
                               int32_t* iterations);

/* ---------------------------------------------------------------------------------------- */
/* Device-resident stepping (benchmarks and the batched / adjoint harnesses)                */
/* ---------------------------------------------------------------------------------------- */

/* Upload u (host) into the context's displacement. */
int nb2_set_displacement(nb2_ctx* ctx, const double* u);
int nb2_get_displacement(nb2_ctx* ctx, double* u);
/* One fused device pass at the context's displacement: constitutive update + tangent stiffness
 * (precision) + internal force, into device-resident K and f_int.  No host copies, no sync. */
int nb2_update_assemble_device(nb2_ctx* ctx, int32_t precision);
/* Copy device K (CSR order, FP64 path) / f_int to host. */
int nb2_download_system(nb2_ctx* ctx, double* K_values, double* f_int);
int nb2_synchronize(nb2_ctx* ctx);
/* Mark DOFs as active Dirichlet DOFs of the device solve (rows/columns treated as zeroed, the
 * enforce_dirichlet_conditions semantics of static_matrix.hpp:279-320). */
int nb2_set_dirichlet_mask(nb2_ctx* ctx, const int32_t* dofs, int32_t num_dofs);
/* Device PCG on the resident K (precision NB2_FP64: FP64 K; NB2_MIXED: FP32 K with FP64 dots)
 * with the context's internal force as right-hand side (masked DOFs zeroed), from x0 = 0.
 * tolerance 0 runs exactly maximum_iterations iterations (timing). */
int nb2_solve_device(nb2_ctx* ctx, int32_t precision, double tolerance, int32_t maximum_iterations,
                     int32_t* iterations, double* error);

/* ---------------------------------------------------------------------------------------- */
/* Batched solves: many independent problems of uneven size in one context                  */
/* ---------------------------------------------------------------------------------------- */

/* Static solves of num_instances independent problems that share one context (one model; each
 * instance's moduli set per element with nb2_set_element_moduli).  Instance i owns the nodes
 * [node_offsets[i], node_offsets[i+1]) and the elements on them (an element that couples two
 * instances is NB2_E_INPUT); its Dirichlet tables are dirichlet[dirichlet_offsets[i] ..
 * dirichlet_offsets[i+1]) and its nodal-force tables nodal_forces[force_offsets[i] ..
 * force_offsets[i+1]), DOFs global.  Every instance runs static_matrix::solve
 * (static_matrix.hpp:145-187, 402-467) with its own load stepping, Newton norms, cutbacks and
 * Jacobi-PCG (linear_solver.cpp:67-109), as if solved alone; one element pass, SpMV and vector
 * update serves all instances per launch.  options apply to every instance (precision NB2_FP64
 * or NB2_MIXED).  Models without history only (no J2 plasticity).  reports: [num_instances];
 * log (nullable): [num_instances][max_log].  Returns the first failing instance's status.
 * neon solves one mesh per simulation: no counterpart interface. */
int nb2_batch_static_solve(nb2_ctx* ctx, int32_t num_instances, const int32_t* node_offsets,
                           const nb2_solver_options* options, const nb2_dof_table* dirichlet,
                           const int32_t* dirichlet_offsets, const nb2_dof_table* nodal_forces,
                           const int32_t* force_offsets, double* u_out,
                           nb2_solve_report* reports, nb2_newton_log* log, int32_t max_log);
/* Autotuner of the batched PCG: times the SpMV over the instances' rows for each rows-per-chunk
 * (16, 32, 64, 128) and lanes-per-block-row (4, 8, 16, 32) candidate on this device and keeps
 * the fastest for the context's next nb2_batch_static_solve.  No counterpart in the reference. */
int nb2_batch_autotune(nb2_ctx* ctx, int32_t num_instances, const int32_t* node_offsets,
                       int32_t precision, int32_t* rows_per_chunk, int32_t* lanes_per_row,
                       double* ms_per_spmv);

#ifdef __cplusplus
}
#endif

#endif /* NEON_B200_H */
