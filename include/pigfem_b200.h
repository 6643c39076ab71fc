/*
 * pigfem_b200.h -- C ABI of the B200 finite-element assembly path (libpigfem_b200.so).
 *
 * The reference's boundary for this path is
 *     PetscErrorCode Assembler::assemble(pmatrix& K, pvector& P_int, double delta_t,
 *                                        std::vector<std::vector<std::vector<double>>>& update_ISVs,
 *                                        NodalData* solution, bool assembleFunc, bool assembleJac)
 * (include/Assembler.h:46-48, src/Assembler.cpp:65-146), reached by every solver through a
 * non-virtual call.  The entry points below are what a host-side Assembler translation unit
 * forwards to (pigfem_b200/drop_in/Assembler_b200.cpp).  Plain pointers and sizes only; every call
 * returns 0 on success or one of the PG_ERR_* codes (never exits, never traps), with a message
 * available from pg_last_error().
 */
#ifndef PIGFEM_B200_H_
#define PIGFEM_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PG_OK 0
#define PG_ERR_INPUT 2        /* invalid description or argument */
#define PG_ERR_GEOMETRY 3     /* a node on an inclusion surface, a missing intersection, ... */
#define PG_ERR_UNSUPPORTED 4  /* a cut case outside the tables (the reference stops there too) */
#define PG_ERR_JACOBIAN 7     /* negative (sub-)element Jacobian */
#define PG_ERR_DEVICE 10      /* CUDA error or out of device memory */
#define PG_ERR_NONFINITE 11   /* a NaN/Inf produced in K or R */
#define PG_ERR_STATE 12       /* call out of order */
#define PG_ERR_CAPACITY 13    /* input larger than a fixed-size buffer allows (pg_norm2_noalloc) */

/* assembly flags */
#define PG_FUNC 1   /* assemble the internal-force vector P_int (assembleFunc) */
#define PG_JAC 2    /* assemble the stiffness K (assembleJac) */
#define PG_FP32 4   /* FP32-mixed element integration (FP64 accumulation in the scatter) */
/* pg_assemble only: the host K arrays still hold what this context's previous PG_JAC |
 * PG_KEEP_STATIC call with the same arrays and precision wrote there (the caller did not change
 * them), so only the values that can have changed since are copied back: the suffix of each
 * block from pg_changing_values on (the rows of the DOFs of nodes on cohesive elements; nothing
 * for a problem without cohesive elements).  The first such call copies everything. */
#define PG_KEEP_STATIC 8

/* background element types (Mesh::generate_mesh element types used by the reference drivers) */
#define PG_TRI3 0
#define PG_QUAD4 1
#define PG_TET4 2

/* cohesive laws: bilinear, Xu-Needleman, Ortiz-Pandolfi (plain, no-unloading "NU", augmented
 * "AUG"), trilinear and smoothed trilinear (plain and "NU") */
#define PG_COH_NONE 0
#define PG_COH_BL 1
#define PG_COH_BLNU 2
#define PG_COH_XN 3
#define PG_COH_XNNU 4
#define PG_COH_OP 5
#define PG_COH_OPNU 6
#define PG_COH_OPAUG 7
#define PG_COH_OPNUAUG 8
#define PG_COH_TL 9         /* TrilinearCohesiveMaterial (src/Material_TrilinearCohesive.cpp) */
#define PG_COH_TLNU 10      /* TrilinearCohesiveNUMaterial (src/Material_TrilinearCohesiveNU.cpp) */
#define PG_COH_STL 11       /* TrilinearSmoothedCohesiveMaterial (src/Material_SmoothedTrilinearCohesive.cpp) */
#define PG_COH_STLNU 12     /* TrilinearSmoothedCohesiveNUMaterial (src/Material_SmoothedTrilinearCohesiveNU.cpp) */

typedef struct pg_ctx pg_ctx;

/* Problem description: the inputs Tests/Main.cpp:150-648 gives Mesh / Problem / BoundaryObject. */
typedef struct {
  int32_t elem_type;            /* PG_TRI3, PG_QUAD4 or PG_TET4 */
  int32_t n[3];                 /* elements per direction (n[2] = 0 in 2D) */
  double lo[3], hi[3];          /* domain box */
  int32_t n_incl;               /* number of circles (2D) or spheres (3D) */
  const double* incl;           /* circles: cx, cy, r; spheres: cx, cy, cz, r */
  double E_matrix, nu_matrix, E_fiber, nu_fiber;
  int32_t coh_law;              /* PG_COH_*; applied to every fiber/matrix interface */
  double coh[4];                /* BL: sigma_c, delta_c1, delta_c2; XN: sigma_c, delta_cn, delta_ct, q; OP: sigma_c, delta_c, beta;
                                   TL, STL: sigma_c, delta_c1, delta_c2, delta_c3 (0 < delta_c1 <= delta_c2 <= delta_c3) */
  int32_t plane_strain;
  int32_t subscale;             /* 1: periodic mesh, macroscale strain eps_macro, node 0 pinned */
  double eps_macro[6];          /* Voigt (xx, yy, xy) or (xx, yy, zz, yz, xz, xy), engineering shear */
  double app_strain;            /* Dirichlet mode: u_x = app_strain * (hi[0]-lo[0]) on the right, 0 on the left, node 0 pinned */
  /* Bounding plies (Tests/Main.cpp:262-289, 343-360): the elements whose nodes all lie within
   * ply_frac * (hi[1]-lo[1]) of the top or of the bottom take a transversely isotropic material
   * (LinearElasticTransverselyIsotropicMaterial, src/material_leti.cpp; fibers along x) with
   * ply = {E1, E2, G12, G23, nu12}.  0: no plies.  As in the reference's Mesh::detection, an
   * element wholly inside an inclusion takes the fiber material even within a ply, and the
   * matrix-side sub-elements of a cut ply element take the ply material. */
  double ply_frac;
  double ply[5];
} pg_problem_desc;

typedef struct {
  int32_t dim, n_nodes, n_std_nodes, n_enrich_nodes, n_elem, n_cut_elem, n_coh_elem, n_coh_qp;
  int32_t n_free, n_const, n_isv;
  int64_t nnz[4];               /* K_ff, K_fp, K_pf, K_pp */
  int64_t cut_scratch_doubles;  /* element-matrix scratch the cut-element kernel uses */
} pg_sizes;

/* Set-up: Problem::init + Problem::setup equivalent (src/Problem.cpp:100-339): IGFEM detection,
 * enrichment, sub-element quadrature, DOF numbering, CSR preallocation; uploads to the device. */
int pg_create(const pg_problem_desc* desc, pg_ctx** out);
/* The two halves of pg_create: the host set-up alone (no device needed; pattern, nodes and
 * set-up tables can be read back) and the upload that makes the context assemble-ready. */
int pg_create_host(const pg_problem_desc* desc, pg_ctx** out);
int pg_upload(pg_ctx* ctx);
/* pg_create_host with the set-up's per-node, per-element and (PG_PREP_PATTERN) pattern passes on
 * the current CUDA device: node detection (Mesh::detect_node, src/Mesh.cpp:2727-2929), the all-equal element test
 * of the element detection (Tri3/Quad4/Tet4::detection), the enrichment nodes and their
 * intersection points (Mesh::add_enrichments, src/Mesh.cpp:3103-3252; Inclusion::
 * find_intersection, src/Inclusion.cpp:32-121), the standard nodes' DOF numbering (DofObject::
 * set_local_owned_normal_dofs, src/DofObject.cpp:336-385), and the DOF nodes' adjacency and the
 * CSR pattern of the four blocks (Solver::preallocate_matrix, src/Solver.cpp:426-490, 772-896).
 * The cut elements' case tables and sub-element quadrature stay on the host.  Every table is the
 * one pg_create_host forms (integers bit-exact, coordinates too); the context is host-only until
 * pg_upload.  Grids of fewer than 2 cells per direction run every pass on the host. */
int pg_create_prep_device(const pg_problem_desc* desc, int passes, pg_ctx** out);
/* passes of pg_create_prep_device: the per-node and per-element passes, and the adjacency and
 * pattern (the latter sorts every element's node pairs; a caller whose GPU is busy with other
 * work may keep it on the host threads) */
#define PG_PREP_NODES 1
#define PG_PREP_PATTERN 2
/* Device time in ms of the passes pg_create_prep_device ran (-1 when none ran). */
int pg_prep_device_ms(const pg_ctx* ctx, double* ms);
/* Read-only view of a set-up table by name (cut-element quadrature, topology); returns 1 for
 * int32, 2 for float64, 0 for an unknown name.  For tests and tools. */
int pg_debug_array(const pg_ctx* ctx, const char* name, int64_t* n, const void** ptr);
void pg_destroy(pg_ctx* ctx);
const char* pg_last_error(const pg_ctx* ctx);
int pg_get_sizes(const pg_ctx* ctx, pg_sizes* out);
/* Device memory the context holds now and the most it has held at once, in bytes: every
 * allocation of pg_upload, the solver workspaces and the homogenization partials, counted as
 * requested from the stream-ordered pool (0 for a host-only context).  Either pointer may be
 * NULL. */
int pg_device_bytes(const pg_ctx* ctx, int64_t* now, int64_t* peak);

/* CSR pattern of block b (0 ff, 1 fp, 2 pf, 3 pp): rowptr[nrows+1], cols[nnz]. */
int pg_get_pattern(const pg_ctx* ctx, int block, int32_t* rowptr, int32_t* cols);
/* Node coordinates (n_nodes*dim), node-major DOF map (n_nodes*dim), prescribed values of the
 * constrained DOFs at load fraction 1 (n_const). */
int pg_get_nodes(const pg_ctx* ctx, double* coords, int32_t* node_dofs, double* dirichlet);

/* Assembler::assemble.  U_node_major: displacement of every node (standard then enrichment),
 * n_nodes*dim, the reference's NodalData layout, in HOST memory.  t_frac scales eps_macro for
 * subscale problems (Assembler::assemble_new_load_step).  Outputs (host, may be NULL to skip):
 * the four K blocks' values in pattern order and P_f (n_free), P_p (n_const).  Internal variables:
 * trial = committed, updated by the cohesive laws (read with pg_get_isv). */
int pg_assemble(pg_ctx* ctx, const double* U_node_major, double t_frac, int flags,
                double* K_ff, double* K_fp, double* K_pf, double* K_pp, double* P_f, double* P_p);
/* Same, on device-resident data: d_U is a 16-byte aligned device pointer (n_nodes*dim); results
 * stay in the context's device buffers (pg_device_outputs). */
int pg_assemble_device(pg_ctx* ctx, const double* d_U, double t_frac, int flags);
/* Residuals of several macroscale strains in one pass, for subscale tri3 / tet4 problems
 * (PG_ERR_UNSUPPORTED for quad4): the load cases of a
 * homogenization, which the reference assembles one Assembler::assemble(assembleJac = false) at a
 * time after Assembler::assemble_new_load_step sets each case's macroscale value
 * (src/Assembler.cpp:65-146, 394-511).  Case k's strain is eps[6k .. 6k+5] * t_frac (Voigt; the 3D
 * entries are ignored in 2D); its residual parts go to d_Rf[k * n_free ...] and d_Rp[k * n_const
 * ...] (device arrays; d_Rp may be NULL when n_const = 0).  Each case's values are those of a
 * residual-only pg_assemble_device with that strain, up to the rounding of fused multiply-adds;
 * the openings, laws and internal variables of the cohesive points are evaluated once (they
 * depend on U only).  K and the context's own residual buffers are left as they are.
 * 1 <= n_cases <= 6.  Asynchronous on the context's stream. */
int pg_residual_strains(pg_ctx* ctx, const double* d_U, double t_frac, int n_cases, const double* eps,
                        double* d_Rf, double* d_Rp);
/* Device pointers of the outputs: K values (4 blocks), P_f, P_p. */
/* The first CSR value of each K block (ff, fp, pf, pp) from which a later assembly of this
 * context can change values; nnz of the block when none can.  Every bulk law is linear elastic,
 * so only the entries coupling DOFs of nodes on one cohesive element depend on the state, and
 * they lie in the rows from the smallest such DOF on. */
int pg_changing_values(const pg_ctx* ctx, int64_t* first);
int pg_device_outputs(pg_ctx* ctx, double** K_vals4, double** P_f, double** P_p);
/* Stream the context launches on (a cudaStream_t, 0 = legacy default). */
int pg_set_stream(pg_ctx* ctx, void* stream);

/* Device timing of the last assembly from CUDA events the context records on its streams:
 * ms[0] cohesive elements and element records, ms[1] stencil rows (2D: side stream, concurrent
 * with ms[0] and ms[2]; 3D: after ms[0]), ms[2] general rows (2D: after ms[0]; 3D: after ms[1]),
 * ms[3] the whole assembly (fork to join).  The event between ms[0] and ms[2] is recorded only
 * while timing is on (pg_set_timing(ctx, 1)): without it the general rows start early, while the
 * kernel before them finishes.  pg_kernel_times returns PG_ERR_STATE when the last assembly ran
 * with timing off. */
int pg_set_timing(pg_ctx* ctx, int on);
int pg_kernel_times(pg_ctx* ctx, float* ms);

/* Internal variables (InternalVars): committed <- values; read trial or committed; commit
 * (InternalVars::copy_data_in after a converged load step). */
int pg_set_isv(pg_ctx* ctx, const double* committed);
int pg_get_isv(const pg_ctx* ctx, int trial, double* out);
int pg_commit_isv(pg_ctx* ctx);
/* Damage zone of every cohesive quadrature point from the last assembly
 * (0 compression, 1 before the peak, 2 softening, 3 failed). */
int pg_get_damage_zones(const pg_ctx* ctx, uint8_t* zones);

/* Macroscale strain of a subscale problem (Voigt, 3 entries in 2D, 6 in 3D), the value that
 * Problem::setMacroscaleValue sets (src/Problem.cpp) and assemble_new_load_step scales by the load
 * fraction; later assemblies use eps * t_frac.  One K with several load cases is one assembly
 * with PG_JAC and one PG_FUNC assembly per strain. */
int pg_set_macro_strain(pg_ctx* ctx, const double* eps);

/* Residual norm ||F_ext,f - P_f||_2 on the device in FP64 with a fixed-order reduction
 * (SolverNonlinearKSP.cpp:81-84); F_ext is zero for the reference's drivers. */
int pg_residual_norm(pg_ctx* ctx, double* out);

/* Jacobi-preconditioned conjugate gradients on K_ff of the last assembly (FP64, on the device).
 * d_b: nrhs right-hand sides of n_free entries each, one after another; d_x: initial guesses in,
 * solutions out (same layout).  Stops each right-hand side at ||b - K x|| <= rtol ||b|| (checked
 * every iteration on the device; the host looks every 16 iterations, so at most max_it + 15
 * iterations run).  Inner products are fixed-order reductions: a right-hand side's result does not
 * depend on the others solved with it.  iters / relres (host, nrhs entries, may be NULL) get each
 * right-hand side's iteration count and final relative residual.  PG_ERR_STATE if any right-hand
 * side missed the tolerance.  The reference solves with a direct Cholesky factorisation (PETSc
 * KSPPREONLY + PCCHOLESKY through MUMPS, src/Solver.cpp:108-194); this is the device solver that
 * replaces it for linear requests and Newton corrections. */
int pg_pcg_solve(pg_ctx* ctx, const double* d_b, double* d_x, int nrhs, double rtol, int max_it, int* iters,
                 double* relres);

/* Volume average of the stress over the volumetric quadrature points (Problem::homogenize,
 * src/Problem.cpp:471-484): out[0..nv-1] = sum(J W sigma) / sum(J W), out[nv] = sum(J W), with
 * sigma from d_U (device, node-major) plus the macroscale strain eps_macro * t_frac. */
int pg_homogenize(pg_ctx* ctx, const double* d_U, double t_frac, double* out);

/* Material sensitivity of the internal force (SensitivityParameter::assemble_dPdd with a
 * SensitivityMaterialParameterStructural of a linear elastic isotropic material,
 * src/SensitivityParameter.cpp:110-153, src/SensitivityMaterialParameter.cpp:41-220): the
 * derivative of P_int at the node-major device displacements d_U by parameter `param` (0 E,
 * 1 lambda, 2 mu, 3 K, 4 nu) of `material` (0 matrix, 1 fiber), summed over the elements and
 * sub-elements of that material, into d_dPf (n_free) and d_dPp (n_const) on the context's stream
 * (returns once they are written).  The strain is that of d_U alone (no macroscale strain), as in
 * the reference.  Cohesive problems are PG_ERR_UNSUPPORTED (the cohesive laws' sensitivity
 * updates are not built). */
#define PG_SENS_E 0
#define PG_SENS_LAMBDA 1
#define PG_SENS_MU 2
#define PG_SENS_K 3
#define PG_SENS_NU 4
int pg_material_sensitivity(pg_ctx* ctx, const double* d_U, int material, int param, double* d_dPf, double* d_dPp);

/* ---- Batches: many contexts assembled by one set of persistent launches replayed from a CUDA
 * graph.  No counterpart in the reference (it assembles one mesh per process).  Each context's
 * results are bitwise those of pg_assemble_device on the same inputs. */
typedef struct pg_batch pg_batch;
/* The contexts must be uploaded and of one dimension; they stay owned by the caller and must
 * outlive the batch. */
int pg_batch_create(pg_ctx* const* ctxs, int n, pg_batch** out);
/* Enqueues one assembly of every context: d_U[i] (device, node-major) with load fraction
 * t_frac[i] (NULL: 1.0 for all) and the common flags (PG_FUNC | PG_JAC | PG_FP32).  Asynchronous
 * on the batch's own stream; outputs land in each context's device buffers. */
int pg_batch_assemble(pg_batch* b, const double* const* d_U, const double* t_frac, int flags);
/* Waits for the last pg_batch_assemble; ms (may be NULL) gets its device time. */
int pg_batch_wait(pg_batch* b, float* ms);
/* Autotuner: times every candidate launch shape (persistent blocks per SM; the stencil rows run
 * as fixed tiles, the general rows a thread per row block) over `reps` assemblies of this batch
 * and keeps the fastest; best[3] (may be NULL) gets {threads per stencil tile, 1, blocks per SM}.
 * Contexts must be tri3 or tet4 (PG_ERR_UNSUPPORTED for quad4). */
int pg_batch_tune(pg_batch* b, const double* const* d_U, int flags, int reps, int* best);
/* info[8]: contexts, elements, threads per stencil tile, 1, blocks per SM, cohesive-point chunks,
 * stencil chunks, general-row chunks. */
int pg_batch_info(const pg_batch* b, int64_t* info);
const char* pg_batch_last_error(const pg_batch* b);
void pg_batch_destroy(pg_batch* b);

/* ||x||_2 of a device vector of n doubles, written to the device double *d_out, enqueued on
 * `stream` (a cudaStream_t; NULL = legacy default stream).  No counterpart in the reference.
 * It allocates nothing: the block partials live in a fixed 32 KiB __device__ array (two
 * stream-ordered launches: the partials, then their sum), so n is limited to PG_NORM_NOALLOC_MAX_N (PG_ERR_CAPACITY beyond it).
 * For callers that must not allocate device memory: a request served against a fixed device
 * memory budget (an allocation would fall outside the admitted budget, and cudaFree
 * synchronises the whole device, stalling the other requests in flight), and a caller holding
 * a raw device vector without a pg_ctx whose scratch it could borrow.  The sum runs in a fixed
 * order, so the result is bitwise reproducible for the same n and data.  The first call on a
 * device looks up the scratch address (cudaGetSymbolAddress) and should come before any stream
 * capture.  Calls on one device share the scratch: calls that may overlap in time (different
 * streams without ordering, or host threads) race and must be serialised by the caller. */
#define PG_NORM_NOALLOC_MAX_N 33554432
int pg_norm2_noalloc(const double* d_x, int64_t n, double* d_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PIGFEM_B200_H_ */
