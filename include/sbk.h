/*
 * sbk.h - C ABI of the B200 element loop of sparlab_form.
 *
 * The reference has no FFI for this path: its seam is the library-internal
 * class detail::NonlinearSystem (src/fem/NonlinearSystem.hpp:85-334), whose
 * evaluate/commit the forming driver calls every Newton iteration
 * (src/fem/Forming.cpp:692,766-783,1202), plus ToolContact
 * (include/sparlab/fem/RigidTool.hpp:248-320) for the penalty contact and
 * Assembler's node-block pattern (src/fem/Assembler.cpp:86-215). Every
 * entry point below replaces one member of those, with plain pointers and
 * sizes: no exceptions cross it (an int status is returned), buffers named
 * "_dev" are device pointers, everything else is host memory.
 *
 * Units and conventions are the reference's: SI, node-major DOFs (dof =
 * 3 node + k), Voigt order {11, 22, 33, 12, 23, 31} with engineering shear
 * strains and tensorial stresses, Hex8 nodes in VTK order.
 */
#ifndef SBK_H_
#define SBK_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference's exceptions) ------------------------ */
enum sbk_status {
  SBK_OK = 0,
  SBK_ERR_ARGUMENT = 1,    /* a null pointer, a bad size or option        */
  SBK_ERR_CONFIG = 2,      /* ConfigError: invalid material or rule       */
  SBK_ERR_MESH = 3,        /* MeshError: an element inverted at rest      */
  SBK_ERR_SOLVER = 4,      /* SolverError: see the failing element's code */
  SBK_ERR_CUDA = 5,        /* a CUDA call failed                          */
  SBK_ERR_UNSUPPORTED = 6, /* a rule or a size the library does not take */
  SBK_ERR_NO_EXTENSION = 7 /* no device: the library never falls back     */
};

/* ---- per-element codes (why an element's SolverError was thrown) ------- */
enum sbk_element_code {
  SBK_EL_OK = 0,
  SBK_EL_INVERTED_POINT = 1,     /* det F <= 0 (IncompatibleModes.cpp:214)         */
  SBK_EL_RETURN_NO_CONVERGE = 2, /* Plasticity.cpp:134-139, 356-359, 423-430       */
  SBK_EL_LOCAL_NO_CONVERGE = 3,  /* 25 local iterations (IncompatibleModes.cpp:470) */
  SBK_EL_LOCAL_SINGULAR = 4,     /* K_aa singular (IncompatibleModes.cpp:462)      */
  SBK_EL_LOCAL_NO_DESCENT = 5,   /* IncompatibleModes.cpp:537-545                  */
  SBK_EL_MESH_INVERTED = 6,      /* det J <= 0 (IncompatibleModes.cpp:159,176)     */
  SBK_EL_NONFINITE = 7,          /* LogarithmicStrain.cpp:110-112                  */
  SBK_EL_DEGENERATE = 8,         /* LogarithmicStrain.cpp:120-125                  */
  SBK_EL_BAD_NODE = 9            /* a device connectivity names a node out of range */
};

enum sbk_kinematics { SBK_SMALL_STRAIN = 0, SBK_FINITE = 1, SBK_FINITE_LOGARITHMIC = 2 };
enum sbk_criterion { SBK_VON_MISES = 0, SBK_HILL48 = 1 };
enum sbk_integration { SBK_EXPONENTIAL = 0, SBK_BACKWARD_EULER = 1 };

#define SBK_MAX_BACKSTRESSES 4
#define SBK_MAX_POINTS 32

/* The material block (include/sparlab/material/Material.hpp:103-257): E, nu,
 * sigma_y(a) = sy0 + H a + Q (1 - exp(-delta a)), Prager's H_kin, Hill48 from
 * r-values in the frame (rolling direction, sheet normal), Chaboche
 * backstresses (C_i, gamma_i). */
typedef struct sbk_material {
  double youngs_modulus, poisson_ratio;
  double yield_stress, hardening_modulus, kinematic_hardening_modulus;
  double saturation_stress, saturation_rate;
  int criterion;       /* sbk_criterion */
  int num_backstresses;
  int kinematic_integration; /* sbk_integration */
  int reserved;
  double backstress_modulus[SBK_MAX_BACKSTRESSES];
  double backstress_recovery[SBK_MAX_BACKSTRESSES];
  double r0, r45, r90, shear_l, shear_m;
  double rolling_direction[3], sheet_normal[3];
} sbk_material;

/* The stiffness rule (include/sparlab/elements/Element.hpp:56-71):
 * stiffness_points per direction (1..4), thickness_points (0: the cube
 * rule; else 1..7 along thickness_axis 0/1/2). The library takes rules of
 * at most SBK_MAX_POINTS points. */
typedef struct sbk_rule {
  int stiffness_points, thickness_points, thickness_axis, reserved;
} sbk_rule;

/* Number of points of a rule (0 for an invalid one). */
int sbk_rule_size(const sbk_rule* rule);

/* Doubles per integration point in the device state layout of a material:
 * plastic strain (6), whole back stress (6), one 6-vector per kinematic term
 * of the general return, accumulated plastic strain, loading flag (0/1). The
 * layout is field-major: field f of point q of element e at
 * state[f * (ne * nq) + e * nq + q]. PlasticState
 * (include/sparlab/material/Plasticity.hpp:185-201) minus its plane-stress
 * thickness strain. */
int sbk_state_fields(const sbk_material* material);

/* The yield matrix P (6x6, row-major, tensorial Voigt, global axes) the
 * material's criterion gives (Material.cpp:135-217); SBK_ERR_CONFIG for an
 * invalid material (Material::set_plasticity's checks). */
int sbk_yield_matrix(const sbk_material* material, double* p_out);

/* ---- one batch of independent elements ---------------------------------
 * incompatible_elastoplastic_element (src/fem/IncompatibleModes.cpp:577-600)
 * for ne elements at once, every pointer on the device:
 *   x_dev      ne x 24   reference coordinates, node-major (x0 y0 z0 x1 ...)
 *   u_dev      ne x 24   displacements, same order
 *   state_dev  committed points, field-major (sbk_state_fields)
 *   alpha_dev  ne x 9    committed mode parameters (NULL: zero)
 * outputs:
 *   force_dev  ne x 24   condensed force f*
 *   tangent_dev ne x 576 condensed tangent K* in node blocks: entry
 *              (3a+i, 3b+j) at e*576 + (8a+b)*9 + 3i + j; NULL: no tangent
 *   energy_dev ne, trial_dev (state layout), alpha_out_dev ne x 9,
 *   yield_dev  ne x nq (1 where the point's return was plastic),
 *   iterations_dev ne, code_dev ne (sbk_element_code).
 * stream: a cudaStream_t (NULL: the default stream). Returns SBK_OK or a
 * launch error; element failures are reported per element in code_dev. */
int sbk_element_batch(const sbk_material* material, const sbk_rule* rule, int kinematics, int64_t ne,
                      const double* x_dev, const double* u_dev, const double* state_dev,
                      const double* alpha_dev, double* force_dev, double* tangent_dev,
                      double* energy_dev, double* trial_dev, double* alpha_out_dev,
                      uint8_t* yield_dev, int32_t* iterations_dev, int32_t* code_dev, void* stream);

/* ---- the system: detail::NonlinearSystem ------------------------------- */
typedef struct sbk_system sbk_system;

typedef struct sbk_mesh {
  int32_t num_nodes, num_elements;
  const double* coords;        /* host, 3 per node                         */
  const int32_t* connectivity; /* host, 8 per element, VTK order           */
} sbk_mesh;

/* NonlinearSystem(model, assembler, options) (NonlinearSystem.hpp:95-101):
 * uploads the mesh, builds the node-block pattern (Assembler::build_pattern,
 * Assembler.cpp:86-173) and its gather maps, and starts every point virgin
 * and every element's modes at zero (initialise_history, :273-311). */
int sbk_system_create(const sbk_mesh* mesh, const sbk_material* material, const sbk_rule* rule,
                      int kinematics, sbk_system** out);
int sbk_system_destroy(sbk_system* sys);
/* All later launches go to this stream (a cudaStream_t; NULL: default). */
int sbk_system_set_stream(sbk_system* sys, void* stream);

/* The element formulation (the model's "element_formulation" and the forming
 * block's "mean_dilatation"; default: the incompatible-mode Hex8):
 * SBK_ELEMENT_STANDARD is elastoplastic_element for the standard Hex8
 * (src/fem/Elastoplastic.cpp:226-340) with B, B_NL or P B_NL per point,
 * averaged (mean dilatation, B-bar) under "auto" or "all" when the rule has
 * more than one point, as NonlinearSystem's constructor decides
 * (NonlinearSystem.hpp:283-309); the incompatible-mode Hex8 refuses "all"
 * (SBK_ERR_CONFIG). */
#define SBK_ELEMENT_INCOMPATIBLE_MODES 0
#define SBK_ELEMENT_STANDARD 1
#define SBK_MEAN_DILATATION_AUTO 0
#define SBK_MEAN_DILATATION_ALL 1
#define SBK_MEAN_DILATATION_NONE 2
int sbk_system_set_element(sbk_system* sys, int element, int mean_dilatation);
/* The formulation in use and whether it averages the dilatation. */
int sbk_system_element(const sbk_system* sys, int* element, int* averaged);

/* Where the evaluations with the tangent assemble its CSC values (nnz
 * doubles, device, the caller's; NULL: the system's own buffer). No
 * counterpart in the reference, whose Evaluation owns its matrix. A driver
 * that alternates two buffers can read one back to the host, or hand it to
 * its solver, while the next evaluation assembles into the other. The
 * buffer must stay valid while evaluations use it; node blocks and
 * stiffness_gross act on the current one. */
int sbk_system_set_values_buffer(sbk_system* sys, double* values_dev);

/* Launch shape of the element kernel: elements per thread block (0: the
 * default, 16 for rules of up to 8 points - four warps - and 8 for larger
 * rules - eight warps; at most what 227 KB of shared memory and 256 threads
 * hold; the batch autotuner sets it). */
int sbk_system_set_elements_per_block(sbk_system* sys, int elements_per_block);

/* How the incompatible-mode Hex8's local iteration runs on the GPU (no
 * counterpart in the reference; no result depends on it - both give the
 * same outputs to the bit). SBK_LOCAL_PHASES (the default): phase kernels
 * over the whole mesh - each round a pass over the elements still
 * iterating, then their element-level step - with the elements that need a
 * line search, the shifted direction or Levenberg-Marquardt handed to the
 * single kernel; rules of up to 8 points (the others always take the single
 * kernel). SBK_LOCAL_SINGLE_KERNEL: one kernel runs each element from start
 * to finish. The phase kernels keep per-element records on the device
 * (about 6.7 KB per element, allocated by the system when it is made or its
 * element changes). sbk_set_local_iteration sets what sbk_element_batch
 * uses and what new systems start with. */
#define SBK_LOCAL_PHASES 0
#define SBK_LOCAL_SINGLE_KERNEL 1
int sbk_set_local_iteration(int mode);
int sbk_system_set_local_iteration(sbk_system* sys, int mode);

/* The element schedule (no counterpart in the reference, whose OpenMP loop
 * takes the elements in mesh order): with by_cost = 1 (the default) every
 * evaluate after the first walks the elements grouped by the cost of their
 * last evaluation (local iterations, yielding points), so that the elements
 * sharing a warp take alike paths; 0 keeps the mesh order. No result depends
 * on it. */
int sbk_system_set_schedule(sbk_system* sys, int by_cost);

/* Sizes and the pattern (device pointers owned by the system). The values
 * array is the reference's column-major (CSC) layout; the pattern is
 * structurally symmetric, so the same arrays read as CSR hold K^T. */
typedef struct sbk_pattern {
  int64_t num_dofs, nnz;
  const int32_t* outer_dev; /* num_dofs + 1 */
  const int32_t* inner_dev; /* nnz          */
} sbk_pattern;
int sbk_system_pattern(const sbk_system* sys, sbk_pattern* out);

/* Evaluation (NonlinearSystem.hpp:27-47); device arrays owned by the system,
 * valid until the next evaluate. */
typedef struct sbk_evaluation {
  const double* internal_dev; /* f_int, num_dofs                          */
  const double* residual_dev; /* f_int - lambda f_dead = f_int (dead = 0) */
  const double* values_dev;   /* tangent CSC values, nnz (want_tangent)   */
  double energy;
  double gross;               /* |sum_e |f_e| per DOF|_2                   */
  int32_t yielding_points;
  int32_t failed_element;     /* -1, or the lowest failing element        */
  int32_t failure_code;       /* sbk_element_code of that element         */
  int32_t reserved;
} sbk_evaluation;

/* NonlinearSystem::evaluate(u, lambda, want_tangent)
 * (NonlinearSystem.hpp:192-268). u_dev: num_dofs doubles on the device.
 * Returns SBK_ERR_SOLVER (and fills failed_element, failure_code) where the
 * reference throws SolverError. */
int sbk_system_evaluate(sbk_system* sys, const double* u_dev, double lambda, int want_tangent,
                        sbk_evaluation* out);

/* sbk_system_evaluate without a synchronisation, for stream capture (a CUDA
 * graph of a Newton iteration, replayed every iteration): enqueues the
 * element kernel, the gathers and the schedule on the system's stream and
 * writes a 5-double summary to summary_dev (device): energy, gross,
 * yielding points, the lowest failing element (-1: none) and its code. The
 * schedule is used in the captured launch only if an evaluate ran before
 * the capture. The caller checks summary_dev[3] before it commits. (No
 * counterpart in the reference, whose evaluate returns its Evaluation.) */
int sbk_system_enqueue(sbk_system* sys, const double* u_dev, int want_tangent, double* summary_dev);

/* With stable = 1, sbk_system_commit copies the trial points and modes into
 * the committed buffers on the device instead of exchanging the two, so
 * that every device pointer of the system - and so a captured graph - stays
 * valid across commits. It then commits whatever the last evaluation left
 * in the trial buffers - an evaluate, an enqueue or a replay of a captured
 * enqueue, which the library does not see - so the caller checks that
 * evaluation's summary first. */
int sbk_system_set_stable_buffers(sbk_system* sys, int stable);

/* Device time of each phase of the last evaluate, in ms, recorded with CUDA
 * events on the system's stream when timing is on: [0] the element kernel,
 * [1] the force gather and reductions, [2] the tangent value gather (the
 * element_tangent / element_residual phases of the reference's TimingLedger,
 * src/fem/Forming.cpp:766-783, split by kernel). */
int sbk_system_set_timing(sbk_system* sys, int enable);
int sbk_system_last_timings(const sbk_system* sys, double* ms3);

/* NonlinearSystem::commit (NonlinearSystem.hpp:119-129): the trial points
 * and modes of the last successful evaluate become the committed ones. */
int sbk_system_commit(sbk_system* sys);

/* committed_all / set_committed (NonlinearSystem.hpp:161-182) and
 * internal_all / set_internal (:137-158) for restart and output: host
 * buffers, state in the field-major device layout, alpha ne x 9. */
int sbk_system_get_committed(const sbk_system* sys, double* state, double* alpha);
int sbk_system_set_committed(sbk_system* sys, const double* state, const double* alpha);
/* The trial state of the last evaluate (Evaluation::states / modes), and
 * its per-point yield flags (ne x nq). */
int sbk_system_get_trial(const sbk_system* sys, double* state, double* alpha, uint8_t* yield);
/* Device pointers of the committed and trial buffers (owned by the system). */
int sbk_system_buffers(const sbk_system* sys, const double** committed_state_dev,
                       const double** committed_alpha_dev, const double** trial_state_dev,
                       const double** trial_alpha_dev);
/* symmetric() and plastic() (NonlinearSystem.hpp:103-105). */
int sbk_system_symmetric(const sbk_system* sys);
int sbk_system_plastic(const sbk_system* sys);

/* add_node_block (src/fem/Forming.cpp:280-297) for n blocks (node, 3x3
 * row-major), all device pointers, added in list order into the tangent of
 * the last evaluate. */
int sbk_system_add_node_blocks(sbk_system* sys, int32_t n, const int32_t* nodes_dev,
                               const double* blocks_dev);

/* Stress recovery at the end of a step: elastoplastic_stress for every
 * element (IncompatibleModes.cpp:602-664; for the standard Hex8
 * Elastoplastic.cpp:342-430, the returns and the averaged measures at the
 * mean-dilatation strain; as the forming driver calls it at
 * Forming.cpp:1266-1281) at the displacement u_dev (num_dofs, device), from
 * the committed points and modes - call it after sbk_system_commit. out_dev
 * (device) receives 28 doubles per element: the point averages of the Cauchy
 * stress (6) and the second Piola-Kirchhoff stress (6), the von Mises stress
 * of the average Cauchy stress, the largest accumulated plastic strain, the
 * largest strain component, the smallest det F, the averages of the
 * Kirchhoff stress (6) and of the log strain (6, tensor components; zero
 * unless logarithmic). SBK_ERR_SOLVER names the lowest failing element.
 * The trial state of the last evaluate is overwritten. */
int sbk_system_stress(sbk_system* sys, const double* u_dev, double* out_dev);

/* stiffness_gross(K, u, free) (NonlinearSystem.hpp:49-67): the norm over the
 * free DOFs of |K| |u|, with K the tangent values of the last evaluate (with
 * any node blocks added since) and u_dev the displacement (num_dofs, device);
 * free_dev lists num_free DOF indices (device, int32). Every row sum is the
 * reference's to the bit (columns in ascending order); the squares of the
 * free rows are summed by a fixed tree. Needs an evaluate with the tangent
 * first (SBK_ERR_ARGUMENT otherwise). */
int sbk_system_stiffness_gross(sbk_system* sys, const double* u_dev, int32_t num_free, const int32_t* free_dev,
                               double* out);

/* The shape derivative of the internal force (the building block of an
 * adjoint with respect to the reference geometry): gx_dev (num_dofs, device)
 * = lambda^T d f_int / d X at the displacement u_dev, lambda_dev (num_dofs,
 * device) a cotangent on the DOFs, X the nodal reference coordinates, the
 * committed points and modes the history; every element's modes follow
 * through their local equilibrium (mu = -K_aa^-T K_ua^T lambda). frozen = 1
 * takes the committed plastic state as it is - the elastic response from the
 * committed plastic strain and back stresses, no return - as a release step
 * with the end-of-forming state frozen. The incompatible-mode Hex8 under
 * finite or logarithmic kinematics; the trial buffers of the last evaluate
 * are overwritten. SBK_ERR_SOLVER names the lowest failing element. */
int sbk_system_vjp_x(sbk_system* sys, const double* u_dev, const double* lambda_dev, int frozen, double* gx_dev);

/* Freeze the committed plastic state (frozen = 1): the evaluations, stress
 * recoveries and shape derivatives that follow take the committed plastic
 * strain and back stresses as they are and return no point - the release
 * step of the adjoint with the end-of-forming state frozen. The tangent is
 * then the elastic one and symmetric (sbk_system_symmetric says so); frozen =
 * 0 restores the material's own response. No counterpart in the reference,
 * whose release step always runs the returns. */
int sbk_system_set_frozen(sbk_system* sys, int frozen);

/* Replace the nodal reference coordinates (num_nodes x 3, device, row-major)
 * by a device-to-device copy on the system's stream; the connectivity,
 * pattern and history stay. The reference builds a new NonlinearSystem for a
 * new mesh; a shape optimisation or a finite-difference check moves the
 * nodes of one system instead. */
int sbk_system_set_coordinates(sbk_system* sys, const double* coords_dev);

/* ---- contact: ToolContact ---------------------------------------------- */
typedef struct sbk_contact sbk_contact;

/* One rigid tool (include/sparlab/fem/RigidTool.hpp:155-189) with its
 * piecewise-linear trajectory and its slave nodes (ascending), their
 * tributary areas and penalty stiffnesses kappa (ToolContact's constructor,
 * RigidTool.cpp:275-333, computes those once from the face geometry). */
typedef struct sbk_tool {
  int32_t shape; /* 0 sphere, 1 plane, 2 cylinder */
  int32_t num_knots;
  int32_t num_slaves;
  int32_t reserved;
  double radius, friction, tangential_ratio;
  double normal[3], axis[3];
  const double* times;     /* host, num_knots           */
  const double* points;    /* host, 3 per knot          */
  const int32_t* nodes;    /* host, num_slaves          */
  const double* area;      /* host                      */
  const double* kappa;     /* host                      */
} sbk_tool;

int sbk_contact_create(const sbk_mesh* mesh, int32_t num_tools, const sbk_tool* tools,
                       int friction_tangent /* 0 exact, 1 symmetric */, sbk_contact** out);
int sbk_contact_destroy(sbk_contact* c);
int sbk_contact_set_stream(sbk_contact* c, void* stream);

/* ToolContact::begin_increment (RigidTool.cpp:345-393); u0_dev on the
 * device, active one flag per tool (host). */
int sbk_contact_begin(sbk_contact* c, const double* u0_dev, double t0, double t1,
                      const uint8_t* active, double margin);

typedef struct sbk_contact_result {
  const double* residual_dev;  /* num_dofs: minus the contact forces          */
  const int32_t* block_nodes_dev; /* num_blocks, in tool then slave order     */
  const double* blocks_dev;    /* 9 per block, row-major, d(residual)/du      */
  int32_t num_blocks;
  int32_t symmetric;
  double gross, round_off, force_norm;
  int32_t failed;              /* 1: a node within half a radius (SolverError) */
  int32_t reserved;
} sbk_contact_result;

/* Per-tool resultants after evaluate: 9 doubles per tool, centre xyz,
 * force xyz, active nodes, slipping nodes, max penetration. */
int sbk_contact_resultants(const sbk_contact* c, double* out);

/* ToolContact::evaluate (RigidTool.cpp:398-555). */
int sbk_contact_evaluate(sbk_contact* c, const double* u_dev, double t, int want_tangent,
                         sbk_contact_result* out);
/* ToolContact::anticipate (RigidTool.cpp:557-603): adds to residual_dev and
 * appends to the block list of the last evaluate; returns the count added
 * in *added. */
int sbk_contact_anticipate(sbk_contact* c, const double* u_dev, const double* du_dev, double t,
                           double* residual_dev, int32_t* added, sbk_contact_result* out);
/* ToolContact::commit (RigidTool.cpp:605-611). */
int sbk_contact_commit(sbk_contact* c);
/* How begin finds an increment's candidates (no counterpart in the
 * reference, which scans every slave node, RigidTool.cpp:345-393; no result
 * depends on it - the same test, the same set, the same order).
 * SBK_SEARCH_GRID (the default): a spherical tool with a finite margin tests
 * only the slave nodes of a uniform-grid hash's cells (edge R + margin) near
 * its swept segment; other tools scan every slave. SBK_SEARCH_SCAN: every
 * tool scans every slave node. */
#define SBK_SEARCH_GRID 0
#define SBK_SEARCH_SCAN 1
int sbk_contact_set_search(sbk_contact* c, int mode);
/* The candidate count of tool k from the last begin (host). */
int sbk_contact_candidates(const sbk_contact* c, int32_t k, int32_t* count);

/* The committed history of tool k (host): count, then per slave node in
 * contact (node, force xyz, relative xyz). */
int sbk_contact_history(const sbk_contact* c, int32_t k, int32_t max_entries, double* out,
                        int32_t* count);

/* ---- the element loop of a small mesh, allocating nothing ---------------
 * No counterpart in the reference. For callers that cannot allocate device
 * memory - a solver working in a fixed device arena its host application
 * hands it, or code that must not call cudaMalloc while it runs - this
 * evaluates one mesh of at most SBK_NOALLOC_MAX_ELEMENTS elements and
 * SBK_NOALLOC_MAX_NODES nodes like sbk_system_evaluate, with every input and
 * output in the caller's device memory. The element tangents and forces
 * between the element kernel and the assembly live in one fixed file-scope
 * device array (about 10 MB), which every GPU that loads the library holds
 * until the process exits; larger meshes are refused (SBK_ERR_UNSUPPORTED).
 *   coords_dev 3 per node, connectivity_dev 8 per element, u_dev 3 per node,
 *   state_dev / alpha_dev the committed points and modes (sbk_element_batch
 *   layout; alpha NULL: zero), outer_dev / inner_dev / nnz the node-block
 *   CSC pattern of the mesh (as sbk_system_pattern gives it).
 * outputs: internal_dev (f_int, 3 per node), values_dev (nnz CSC values,
 *   summed element by element in element order; NULL: no tangent),
 *   trial_dev / alpha_out_dev / yield_dev (as sbk_element_batch), and
 *   summary_dev: 5 doubles - energy, gross, yielding points, the lowest
 *   failing element (-1 if none) and its sbk_element_code. An element that
 *   fails, for any reason, is left out of every sum (internal, values,
 *   gross, energy, yield count) and its yield_dev bytes are not written;
 *   an element whose connectivity names a node out of range fails with
 *   SBK_EL_BAD_NODE before anything of it is read. An element naming one
 *   node twice is added entry by entry, so both of its contributions to a
 *   shared entry count. A mesh block the pattern lacks gives -2 and
 *   SBK_EL_BAD_NODE.
 * The call only enqueues work on `stream`; read summary_dev after it. The
 * first call on a device looks up the array's device address (with that
 * device current), so make it before any stream capture. All calls share
 * the array: calls that overlap on the GPU race. */
#define SBK_NOALLOC_MAX_ELEMENTS 2048
#define SBK_NOALLOC_MAX_NODES 16384
int sbk_evaluate_noalloc(const sbk_material* material, const sbk_rule* rule, int kinematics,
                         int32_t num_nodes, int32_t num_elements, const double* coords_dev,
                         const int32_t* connectivity_dev, const double* u_dev, const double* state_dev,
                         const double* alpha_dev, const int32_t* outer_dev, const int32_t* inner_dev,
                         int64_t nnz, double* internal_dev, double* values_dev, double* trial_dev,
                         double* alpha_out_dev, uint8_t* yield_dev, double* summary_dev, void* stream);

/* ---- the free-free tangent: PartitionedFactor --------------------------- */
typedef struct sbk_partition sbk_partition;

/* A Dirichlet partition of an n-DOF model and its free-free block:
 * PartitionedFactor::reset (src/fem/Forming.cpp:73-84) and ::build
 * (Forming.cpp:213-241) on the full tangent's CSC pattern (outer_dev,
 * inner_dev: device, as sbk_system_pattern gives it; structurally
 * symmetric). free_host lists the num_free free DOFs, strictly ascending.
 * The block keeps the entries whose row and column are free, in the full
 * pattern's order. A fill-reducing order of the block for the sparse
 * factorisation is computed here too, once (METIS nested dissection). A new
 * pattern or a new free set is a new partition. */
int sbk_partition_create(int64_t num_dofs, const int32_t* outer_dev, const int32_t* inner_dev, int64_t nnz,
                         int32_t num_free, const int32_t* free_host, sbk_partition** out);
int sbk_partition_destroy(sbk_partition* part);
/* All later work goes to this stream (a cudaStream_t; NULL: default). */
int sbk_partition_set_stream(sbk_partition* part, void* stream);
/* The block's size and pattern: num_free + 1 column offsets and nnz_ff row
 * indices (CSC, free numbering), copied to caller device buffers (either may
 * be NULL). */
int sbk_partition_info(const sbk_partition* part, int32_t* num_free, int64_t* nnz_ff);
int sbk_partition_pattern(const sbk_partition* part, int32_t* outer_dev, int32_t* inner_dev);

/* PartitionedFactor::assemble (Forming.cpp:89-98): the free-free values of
 * the full tangent values_dev (nnz, device) into kff_dev (nnz_ff, device),
 * in the block's CSC order; every value is copied, none summed. */
int sbk_partition_assemble(sbk_partition* part, const double* values_dev, double* kff_dev);
/* restrict(v, free) (Forming.cpp:748,838): out_dev[i] = full_dev[free[i]];
 * add_to(full, free, v, alpha) (Forming.cpp:1036): full_dev[free[i]] +=
 * alpha v_dev[i]. Device arrays. */
int sbk_partition_restrict(sbk_partition* part, const double* full_dev, double* out_dev);
int sbk_partition_add_to(sbk_partition* part, double* full_dev, const double* v_dev, double alpha);

/* PartitionedFactor::factorize (Forming.cpp:100-160) of the free-free block
 * of values_dev (the full tangent, device), where the reference takes
 * CHOLMOD's supernodal Cholesky, then LDL^T, then LU (UMFPACK):
 *   symmetric: a sparse Cholesky on the device (cuSOLVER), its pattern
 *     analysed on the first call;
 *   not symmetric, or a Cholesky that meets a non-positive pivot or whose
 *     correction's backward error exceeds 1e-10: a dense LU with partial
 *     pivoting on the device while the block has at most the dense limit of
 *     rows (sbk_partition_set_dense_limit; default 20000, n^2 doubles);
 *   larger: restarted GMRES preconditioned by the Cholesky of the block's
 *     symmetric part, and a sparse QR on the device where that part is not
 *     positive definite or GMRES stalls.
 * SBK_ERR_SOLVER when the LU finds the block singular (a pivot below 1e-13
 * of the largest entry), as the reference's factorize returns false. kind
 * (may be NULL) receives the method of the next solve. */
#define SBK_FACTOR_CHOLESKY 1
#define SBK_FACTOR_QR 2
#define SBK_FACTOR_GMRES 3
#define SBK_FACTOR_LU 4
int sbk_partition_factorize(sbk_partition* part, const double* values_dev, int symmetric, int* kind);
/* Blocks of at most max_rows rows take the dense LU (0: never). */
int sbk_partition_set_dense_limit(sbk_partition* part, int32_t max_rows);
/* PartitionedFactor::solve (Forming.cpp:162-172): x_dev = K_ff^-1 b_dev
 * (num_free each, device, free numbering). SBK_ERR_SOLVER when the block is
 * singular (the QR's or LU's pivot below 1e-13 of the largest entry). */
int sbk_partition_solve(sbk_partition* part, const double* b_dev, double* x_dev);
/* x_dev = K_ff^-T b_dev with the same factorisation - the adjoint system of
 * a partition. A Cholesky (symmetric) or a dense LU factorisation;
 * SBK_ERR_UNSUPPORTED for the GMRES and QR solves. */
int sbk_partition_solve_transpose(sbk_partition* part, const double* b_dev, double* x_dev);
/* names() and failures() (Forming.cpp:174-181) as counts, since the
 * partition was made: factorisations solved by Cholesky, by preconditioned
 * GMRES, by dense LU, by QR; Choleskys and GMRES runs that fell back;
 * singular blocks; GMRES Krylov steps; solves. */
int sbk_partition_counts(const sbk_partition* part, int64_t counts[9]);

/* Last error message of this thread (never NULL). */
const char* sbk_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SBK_H_ */
