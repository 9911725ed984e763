/*
 * jfem_gpu.h -- C ABI of the B200 element hot path for OpenJFEM (SOL 101/105).
 *
 * The library replaces the two assembly calls of the reference solver:
 *
 *   Solver.assemble_stiffness(model; ...)             src/solver/assembly.jl:1953-4375
 *   Solver.assemble_geometric_stiffness(model, ...)   src/solver/assembly.jl:4382-6634
 *
 * called from _solve_sol105 / solve_model at src/JFEMSolver.jl:807-810 and
 * :1452-1457.  The caller keeps its own model build, SPC/MPC reduction,
 * factorization and eigensolve; this library only produces the same sparse
 * matrices (Julia SparseMatrixCSC{Float64,Int64} arrays: 1-based colptr,
 * rowval, nzval) that those two functions return.  On the same element
 * kernels it also serves the steps either side: the free-dof extraction,
 * shell-thickness sensitivities of K and KG, SOL 101 output recovery, and a
 * device-resident request loop.
 *
 * Every entry point takes plain pointers and sizes.  Host arrays are owned by
 * the caller; the library copies what it needs and keeps no pointer into
 * caller memory after a call returns.  Device state (mesh, property records,
 * CSR pattern, element-to-nonzero scatter map, staging) is owned by the
 * jfg_model handle until jfg_model_destroy.  Calls on one handle must not
 * overlap; different handles are independent.
 *
 * Errors: every entry returns a jfg_status.  On failure the handle keeps a
 * message (jfg_last_error), mirroring the reference's error(...) calls.
 */
#ifndef JFEM_GPU_H
#define JFEM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t jfg_status;
enum {
    JFG_OK = 0,
    JFG_ERR_INVALID = 1,      /* malformed input (bad index, size, null pointer) */
    JFG_ERR_UNSUPPORTED = 2,  /* deck leaves the reference's default branch */
    JFG_ERR_CUDA = 3,         /* CUDA runtime error */
    JFG_ERR_TIMEOUT = 4,      /* a bounded device wait expired */
    JFG_ERR_STATE = 5,        /* call order violated (e.g. no pattern yet) */
    JFG_ERR_NOMEM = 6,        /* device or host allocation failed */
    JFG_ERR_REFERENCE_RAISES = 7 /* the reference raises on this input (see message) */
};

/* Per-shell property record, 7 doubles per element, in this order:
 *   h      PSHELL T
 *   E, nu  MAT1 of MID (membrane/bending), G completed as extract_mats does
 *   G      MAT1 G of MID
 *   br     PSHELL 12I/T^3 (BEND_RATIO; 0 when MID2 is blank)
 *   tst    PSHELL TS/T (default 5/6)
 *   Gs     shear modulus of the MID3 material (MID when MID3 is blank)
 * Constitutive build: assembly.jl:2460-2469, shell_transverse_shear_matrix
 * assembly.jl:1808-1856. */
#define JFG_SHELL_PROP 7

/* Per-bar record (CBAR and CBEAM, identical in the reference), 18 doubles:
 *   A, I1, I2, I12, J, K1, K2   PBARL/PBAR section (extract_pbarl)
 *   E, G                        MAT1
 *   vx, vy, vz                  orientation vector in basic (G0 resolved by caller)
 *   wax, way, waz, wbx, wby, wbz  CBAR offsets WA, WB
 * Element: assembly.jl:3961-4092 (K), :6277-6424 (KG). */
#define JFG_BAR_PROP 18

typedef struct jfg_model_desc {
    int64_t n_nodes;            /* nodes in id_map order (sorted GRID IDs)           */
    const double *coords;       /* n_nodes*3, basic system                           */
    const double *node_R;       /* n_nodes*9 row-major CD frames, or NULL (all basic)*/
    int64_t n_quad4;
    const int32_t *quad4_nodes; /* n_quad4*4, 0-based node indices                   */
    const double *quad4_prop;   /* n_quad4*JFG_SHELL_PROP                           */
    int64_t n_tria3;
    const int32_t *tria3_nodes; /* n_tria3*3                                         */
    const double *tria3_prop;   /* n_tria3*JFG_SHELL_PROP                           */
    int64_t n_bar;
    const int32_t *bar_nodes;   /* n_bar*2 (GA, GB)                                  */
    const double *bar_prop;     /* n_bar*JFG_BAR_PROP                               */
    const int32_t *bar_pin;     /* n_bar*2 (PA, PB) or NULL                          */
    int64_t n_rbe2;
    const int32_t *rbe2_master; /* n_rbe2, GN node index                             */
    const int32_t *rbe2_cm;     /* n_rbe2, CM components as bit mask (bit0 = comp 1) */
    const int64_t *rbe2_slave_ptr; /* n_rbe2+1                                       */
    const int32_t *rbe2_slaves; /* GM node indices                                   */
    double k6rot;               /* PARAM K6ROT (reference default 100)               */
    double param_snorm;         /* PARAM SNORM; must be <= 0 (default branch)        */
} jfg_model_desc;

typedef struct jfg_model jfg_model;

/* Build a handle: validates the default-branch predicates, uploads the mesh,
 * builds the CSR pattern and the element-to-nonzero scatter map on the GPU.
 * Replaces the per-call node indexing, pre-extraction and sparse() pattern
 * work of assemble_stiffness (assembly.jl:1957-2536, :4371). */
jfg_status jfg_model_create(const jfg_model_desc *desc, jfg_model **out);

/* Size of the assembled matrices: ndof = 6*n_nodes and the structural
 * nonzero count of K (identical for KG on the supported element set). */
jfg_status jfg_pattern(jfg_model *m, int64_t *ndof, int64_t *nnz);

/* Fill caller-allocated CSC arrays (colptr: ndof+1, rowval: nnz), 1-based,
 * rows sorted within each column -- SparseArrays.sparse semantics with
 * explicit zeros kept (assembly.jl:4371, :6624). */
jfg_status jfg_pattern_fill(jfg_model *m, int64_t *colptr, int64_t *rowval);

/* Stiffness assembly (assemble_stiffness, assembly.jl:1953-4375).
 * nzval: nnz doubles in CSC order; max_elem_stiff: max |V| over element
 * triplets before constraints (:4353-4356); orig_diag: ndof doubles, sum of
 * element diagonal triplets before constraints (:4359-4364).  Any output
 * pointer may be NULL to skip it.  All pointers are host memory. */
jfg_status jfg_assemble_k(jfg_model *m, double *nzval, double *max_elem_stiff, double *orig_diag);

/* Geometric stiffness assembly (assemble_geometric_stiffness,
 * assembly.jl:4382-6634) from the static displacement u_global (ndof
 * doubles, node displacement systems).  Host pointers. */
jfg_status jfg_assemble_kg(jfg_model *m, const double *u_global, double *nzval);

/* Device-resident variants: the same work with all pointers in device
 * memory on the handle's stream (no host copies).  nzval_dev is nnz doubles;
 * orig_diag_dev (ndof) and max_elem_stiff_dev (1) may be NULL. */
jfg_status jfg_assemble_k_device(jfg_model *m, double *nzval_dev, double *max_elem_stiff_dev,
                                 double *orig_diag_dev);
jfg_status jfg_assemble_kg_device(jfg_model *m, const double *u_global_dev, double *nzval_dev);

/* Replace the per-element shell thicknesses (PSHELL T) in place; the mesh,
 * pattern and scatter map stay resident.  Semantics of the thickness update
 * of optimize_thickness.jl:209-240 / :307-313.  Host pointers, n_quad4 and
 * n_tria3 doubles (either may be NULL to keep the current values). */
jfg_status jfg_update_properties(jfg_model *m, const double *quad4_h, const double *tria3_h);

/* Multipoint-constraint map returned by assemble_stiffness as rbe3_map
 * (constraints.jl:319, merged at :319-322): dependent dof -> list of
 * (independent dof, coefficient), 1-based dofs.  Query the sizes with NULL
 * arrays first: n_dep entries, n_terms pairs in total. */
jfg_status jfg_constraint_map(jfg_model *m, int64_t *n_dep, int64_t *n_terms,
                              int64_t *dep_dof, int64_t *term_ptr, int64_t *ind_dof, double *coeff);

/* Set the CUDA stream (a cudaStream_t passed as void*) used by the handle;
 * NULL selects the handle's own stream.  A K / KG call also runs its RBE2-path
 * sums and orig_diag on an internal high-priority stream that forks from this
 * stream after the element kernels and joins it before the call's last
 * operation, so work queued after the call on this stream sees every output
 * (in a stream capture the fork and join become graph dependencies). */
jfg_status jfg_set_stream(jfg_model *m, void *stream);

/* Timing of the last assembly on the device (CUDA events around the element
 * kernels and the segmented reduction), milliseconds. */
jfg_status jfg_last_timing(jfg_model *m, double *element_ms, double *reduce_ms, double *total_ms);

/* Per-kernel device times of the last assembly, milliseconds, 6 doubles in
 * the order: quad4 elements, tria3 elements, bar elements, dof-level
 * (RBE2-expanded) reduction, node-pair block reduction, orig_diag reduction. */
jfg_status jfg_kernel_timing(jfg_model *m, double *ms6);

/* Per-kernel device times summed over all K (kind 0) or KG (kind 1)
 * assemblies since the last reset, with the number of calls; reset != 0
 * clears the sums after reading.  Waits for the recorded calls. */
jfg_status jfg_timing_accumulated(jfg_model *m, int kind, double *ms6_sum, int64_t *n_calls, int reset);

/* Sizes of the resident data: out8 = {staging values, global node-pair
 * blocks, CSC nonzeros, constraint-expanded contributions, raw values of
 * constraint-touching pairs, element node pairs (scatter-map length),
 * orig_diag entries, device bytes in use}. */
jfg_status jfg_model_stats(jfg_model *m, int64_t *out8);

/* KG entries moved to pageable host memory per jfg_assemble_kg: only the
 * entries KG can make nonzero cross the bus (the rest are +0.0 and written by
 * host threads).  *n_live = that count once the first such call has built the
 * live mask, -1 before (or when the model uses the plain copy). */
jfg_status jfg_kg_transfer_entries(jfg_model *m, int64_t *n_live);

/* Element and node counts of a handle: out4 = {n_nodes, n_quad4, n_tria3, n_bar}. */
jfg_status jfg_model_counts(jfg_model *m, int64_t *out4);

/* ---- Batched variants of one model ---------------------------------------
 * Design variants (one mesh, many property sets) and the requests of one
 * model family in the serving loop run as one launch per kernel: the
 * variants share the handle's mesh, CSC pattern and scatter maps; each has
 * its own shell thicknesses, optionally its own bar records, its own
 * displacement field and its own output values.  This is the batched form
 * of assemble_stiffness / assemble_geometric_stiffness
 * (src/solver/assembly.jl:1953-4375, 4382-6634) over n_var property sets;
 * the reference has no batched call (it assembles one model per call).
 */

/* Device bytes of batch workspace (block staging, raw RBE2 blocks, chunk
 * partials, diagonal staging) that n_var variants need. */
jfg_status jfg_batch_workspace_bytes(jfg_model *m, int32_t n_var, int64_t *bytes);

/* Grow the handle's batch workspace to hold n_var variants (1..65535).  It
 * allocates device memory, so call it before any stream capture. */
jfg_status jfg_batch_reserve(jfg_model *m, int32_t n_var);

/* Assemble K and/or KG for n_var variants (device pointers, the handle's
 * stream, returns without synchronising; n_var <= the reserved count):
 *   h_dev         [n_var][n_quad4 + n_tria3] shell thicknesses (> 0, not
 *                 checked on the device), or NULL for the handle's own;
 *   bar_prop_dev  [n_var][n_bar][JFG_BAR_PROP] bar records with the handle's
 *                 offsets and orientation vectors, or NULL for the handle's;
 *   u_dev         displacements for KG: [n_var][ndof] with u_stride = ndof,
 *                 or one field shared by every variant with u_stride = 0;
 *   nzk_dev       [n_var][nnz] K values, or NULL to skip K;
 *   max_dev       [n_var] max_elem_stiff, or NULL (needs nzk_dev);
 *   diag_dev      [n_var][ndof] orig_diag, or NULL (needs nzk_dev);
 *   nzkg_dev      [n_var][nnz] KG values, or NULL to skip KG.
 * Variant v's outputs equal, bit for bit, a single-model call with variant
 * v's properties.  KG refuses bars with offsets as jfg_assemble_kg does. */
jfg_status jfg_assemble_batch_device(jfg_model *m, int32_t n_var, const double *h_dev, const double *bar_prop_dev,
                                     const double *u_dev, int64_t u_stride, double *nzk_dev, double *max_dev,
                                     double *diag_dev, double *nzkg_dev);
/* The same with caller-provided batch workspace instead of the handle's
 * reserved one: workspace_dev, 256-byte aligned, at least
 * jfg_batch_workspace_bytes(m, n_var) bytes, used until the stream reaches
 * the end of the call's kernels.  Lets a server carve batches of any size out
 * of one device pool (no allocation inside the call). */
jfg_status jfg_assemble_batch_device_ws(jfg_model *m, int32_t n_var, void *workspace_dev, int64_t workspace_bytes,
                                        const double *h_dev, const double *bar_prop_dev, const double *u_dev,
                                        int64_t u_stride, double *nzk_dev, double *max_dev, double *diag_dev,
                                        double *nzkg_dev);

/* ---- Free-dof submatrices for the solver --------------------------------
 * The step right after assembly in the SOL 105 consumer: A_ff = A[free,
 * free] and its symmetric part 0.5 * (A_ff + A_ff') for K
 * (src/solver/boundary_conditions.jl:113-114) and Kg
 * (src/solver/solve_case.jl:1908-1927), with Kg's diagnostics max|Kg_ff| and
 * max|Kg_ff - Kg_ff'|.  As with Julia's sparse +, entries whose sum is
 * exactly zero are not stored.  Done on the device, so only the free-dof
 * matrices need to cross to the host. */

/* Set the free dofs (1-based, strictly increasing; the host computes them
 * from SPC, RBE2 dependents and AUTOSPC).  The first call also finds, once
 * per pattern, where each stored entry's transpose lives (allocates). */
jfg_status jfg_ff_set_free(jfg_model *m, const int64_t *free_dofs, int64_t n_free);

/* Extract from device values nz_dev (a K or KG of this handle, CSC order):
 * nnz of the symmetrised free-dof matrix, max|A_ff| and max|A_ff - A_ff'|.
 * Runs on the handle's stream and waits for it. */
jfg_status jfg_ff_extract_device(jfg_model *m, const double *nz_dev, int64_t *nnz_ff, double *max_abs,
                                 double *max_asym);

/* Host copies of the last extraction: 1-based CSC colptr (n_free + 1),
 * rowval and nzval (nnz_ff each). */
jfg_status jfg_ff_fetch(jfg_model *m, int64_t *colptr, int64_t *rowval, double *nzval);

/* Device pointers to the last extraction (valid until the next one). */
jfg_status jfg_ff_device_arrays(jfg_model *m, const int64_t **colptr, const int64_t **rowval, const double **nzval);

/* ---- Shell-thickness sensitivities dK/dh ---------------------------------
 * Replace the shell_thickness branch of compute_dKdx_u
 * (src/solver/dKdx.jl:193-250, _dKdx_u_shell_thickness_ad_forward and
 * _shell_thickness_dKe_forward_ad) and the per-element loop of
 * _compliance_and_sensitivity (src/solver/optimize_thickness.jl:420-441).
 * The element is the reference's sensitivity element, stiffness_quad4_generic
 * / stiffness_tria3_generic (src/FEMKernels.jl:1473-1656, :7113-7123: bend
 * ratio 1, TS/T 5/6, K6ROT 100, G = E / 2(1 + nu)), with each element's own
 * thickness, E and nu; the derivative is exact (what forward-mode AD gives),
 * not a difference quotient.  Vectors are ndof long (6 dofs per node, the
 * handle's node order); T_e holds the element frame and node CD frames.
 *
 * jfg_dkdh_contract: for every CQUAD4 e, c_q4[e] = a_e' T_e' dK_e/dh T_e b_e,
 * and likewise c_t3 for every CTRIA3 (a = b = u gives u' dK_e/dh u, the
 * compliance sensitivity -dC/dh_e; a = b = phi the buckling one).  Either
 * output may be NULL.
 * jfg_dkdh_load: the pseudo-load sum_e T_e' dK_e/dh T_e u_e over the elements
 * whose mask byte is nonzero (one byte per element; a NULL mask selects every
 * element of that type), summed per dof in a fixed order.
 * The _device forms take device pointers and run asynchronously on the
 * handle's stream (jfg_set_stream); jfg_dkdh_load_device reuses the handle's
 * orig_diag staging, so it must not overlap a K assembly of the same handle.
 * The host forms copy in and out and return when done. */
jfg_status jfg_dkdh_contract(jfg_model *m, const double *a, const double *b, double *c_q4, double *c_t3);
jfg_status jfg_dkdh_load(jfg_model *m, const double *u, const uint8_t *mask_q4, const uint8_t *mask_t3, double *load);
jfg_status jfg_dkdh_contract_device(jfg_model *m, const double *a_dev, const double *b_dev, double *c_q4_dev,
                                    double *c_t3_dev);
jfg_status jfg_dkdh_load_device(jfg_model *m, const double *u_dev, const uint8_t *mask_q4_dev, const uint8_t *mask_t3_dev,
                                double *load_dev);

/* ---- Per-element KG contractions (buckling sensitivities) ----------------
 * c_q4[e] = a_e' T_e' KG_e(u) T_e b_e for every CQUAD4, likewise c_t3, with KG_e
 * the element matrix of jfg_assemble_kg (before constraints).  With a = b =
 * phi and divided by the element thickness this is phi' dKG_e/dh phi, the
 * per-element term of _dKg_dx_phi_thickness (src/solver/adjoint_buckling.jl:
 * 2079-2150): at fixed u the membrane stress does not depend on h, and KG is
 * linear in h.  That function's flat-isotropic context uses the assembly's
 * KG formulation when the deck has line elements; for shell-only decks it
 * switches to the enhanced membrane modes (:930-951), which this library does
 * not build.  Decks whose KG assembly raises (offset bars) raise here too.
 * The _device form runs asynchronously on the handle's stream and uses the
 * handle's staging, so it must not overlap an assembly of the same handle. */
jfg_status jfg_kg_contract(jfg_model *m, const double *u_global, const double *a, const double *b, double *c_q4,
                           double *c_t3);
jfg_status jfg_kg_contract_device(jfg_model *m, const double *u_dev, const double *a_dev, const double *b_dev,
                                  double *c_q4_dev, double *c_t3_dev);

/* ---- SOL 101 output recovery ----------------------------------------------
 * Replace the per-element loops of recover_shell_stresses! and
 * recover_bar_stresses! (src/solver/stress_recovery.jl:163-430, :432-593) on
 * their default branch (isotropic PSHELL/MAT1, no SNORM, no curvature
 * membrane): stress_strain_quad4 + quad4_bilinear_corner_forces
 * (src/FEMKernels.jl:6003-6338) with the equilibrium-shear blend and the
 * pressure-moment scale of CQUAD4, stress_strain_tria3 (:7391-7432) with its
 * macro shear and the shared-edge macro-moment blend of CTRIA3, and
 * forces_frame3d (:215-229) with the four section points of CBAR/CBEAM.
 * u_global holds ndof values in the handle's dof order.
 *
 * Shell record, JFG_SHELL_REC doubles per element, CQUAD4s then CTRIA3s in
 * handle order (the results_json "forces", "stresses", "strains" and
 * "forces_bilin" entries):
 *   0-2   fx fy fxy          membrane forces N
 *   3-5   mx my mxy          bending moments M (CQUAD4: pressure scale applied)
 *   6-7   qx qy              transverse shear (CQUAD4: equilibrium blend applied)
 *   8-10  z1 stress          normal_x normal_y shear_xy at fibre -T/2
 *   11-13 z2 stress          at +T/2
 *   14-16 z1 strain, 17-19 z2 strain
 *   20    stresses[eid]      max principal of the z1 stress
 *   21    status             1 recovered; 0 where the reference's try block fails
 *   22-33 corner forces N    CQUAD4 GA..GD (3 each, bilinear rows); 0 for CTRIA3
 *   34-45 corner moments M   same layout, mxy constant across corners
 *   46-47 von Mises z1, z2
 * Bar record, JFG_BAR_REC doubles per CBAR/CBEAM in handle order:
 *   0-7   axial shear_1 shear_2 torque moment_a1 moment_a2 moment_b1 moment_b2
 *   8     axial stress (stresses[eid] is its absolute value)
 *   9-12  end A stress at section points C D E F, 13-16 end B
 *   17    status             1 recovered; 0 for a zero-length bar (skipped)
 * bar_points (may be NULL: section stresses 0) holds JFG_BAR_POINTS doubles
 * per bar: C1 C2 D1 D2 E1 E2 F1 F2 of the PBARL, then +1 for ROD/TUBE/TUBE2
 * sections and -1 otherwise (surface_stress_sign).
 * flags: JFG_RECOVER_PRESSURE_DECK declares that the deck has at least four
 * PLOAD4 cards and no RBE3, RSPLINE, MPC, CROD or CONROD and at least four
 * CSHELLs -- the model-level conditions of _quad4_pressure_resultant_moment_scale
 * (stress_recovery.jl:131-161) that the handle cannot see; the handle adds
 * "no bars, no RBE2" itself.  Either output may be NULL.  The _device form
 * takes device pointers and runs on the handle's stream without waiting. */
#define JFG_SHELL_REC 48
#define JFG_BAR_REC 18
#define JFG_BAR_POINTS 9
#define JFG_RECOVER_PRESSURE_DECK 1
jfg_status jfg_recover_stresses(jfg_model *m, const double *u_global, const double *bar_points, int32_t flags,
                                double *shell_out, double *bar_out);
jfg_status jfg_recover_stresses_device(jfg_model *m, const double *u_dev, const double *bar_points_dev, int32_t flags,
                                       double *shell_out_dev, double *bar_out_dev);

/* ---- Serving: a device-resident request loop over model families --------
 * Replaces the reference's optimisation worker loop
 * (tools/jfem_worker_jsonl.jl:132-148, manifest_batch_core.jl:283-409), which
 * reassembles a model per JSONL request: here each family's mesh, CSC pattern
 * and scatter maps stay on the GPU (its jfg_model handle), and a request
 * carries a new shell-thickness vector (n_quad4 + n_tria3 values, > 0) and
 * gets K and, when the family has a displacement field, KG of that family.
 * While a server lives it owns its families' handles (their streams are its
 * own); results stay on the device until released.
 *   JFG_SERVE_BATCHED  continuous batching: requests that wait when a result
 *                      slot frees up run together in one batched launch;
 *                      families run on their own streams and overlap.
 *   JFG_SERVE_SERIAL   one request per launch, in arrival order, each
 *                      finished before the next starts (the plain path).
 * Admission by HBM budget: one device pool of hbm_budget_bytes holds every
 * batch's workspace and results.  A batch takes both when it is formed (as
 * many queued requests as fit, at most max_batch); its workspace returns when
 * its kernels finish, its results when its last request is released.  A
 * request waits only while its launch unit has two batches in flight or the
 * pool lacks room.  Results of a batched request equal, bit for bit, the same
 * request served alone. */
#define JFG_SERVE_BATCHED 0
#define JFG_SERVE_SERIAL 1
typedef struct jfg_server jfg_server;

/* families[n_families] handles; u_host[n_families] displacement fields (ndof
 * each) for KG, or NULL entries / NULL array for K only. */
jfg_status jfg_server_create(jfg_model *const *families, const double *const *u_host, int32_t n_families,
                             int64_t hbm_budget_bytes, int32_t max_batch, int32_t policy, jfg_server **out);
/* Launch units: units[n_units] are handles, plain or group handles
 * (jfg_group_create), with u_host[n_units] displacement fields (ndof of the
 * unit, the group's concatenation for a group) or NULL entries.  Family f is
 * served by unit family_unit[f]: the whole handle when family_member[f] < 0
 * (one family per such unit), else member family_member[f] of the group.
 * Requests of a group's families share batches: variant v of a group batch
 * carries the v-th queued request of every member that has one, the members
 * without one are computed at the handle's current thickness and discarded.
 * A grouped family's max_elem_stiff result is the group's (max over its
 * members).  Group units need JFG_SERVE_BATCHED.  jfg_server_create is the
 * case of one plain unit per family. */
jfg_status jfg_server_create_units(jfg_model *const *units, const double *const *u_host, int32_t n_units,
                                   const int32_t *family_unit, const int32_t *family_member, int32_t n_families,
                                   int64_t hbm_budget_bytes, int32_t max_batch, int32_t policy, jfg_server **out);
/* Queue a request (the thickness vector is copied).  keep = 0 returns the
 * result slot as soon as the request is computed (timing only: its record
 * and times stay readable until jfg_server_release, its result pointers are
 * NULL). */
jfg_status jfg_server_submit(jfg_server *s, int32_t family, const double *h_host, int32_t keep, int64_t *ticket);
/* Wait until the request is done (timeout_s < 0: no limit); *done = 1 when finished. */
jfg_status jfg_server_wait(jfg_server *s, int64_t ticket, double timeout_s, int32_t *done);
/* Device pointers to a finished request's K values, KG values (NULL if the
 * family has no u) and max_elem_stiff, valid until jfg_server_release;
 * times3 = {submitted, launched, finished} in seconds since creation. */
jfg_status jfg_server_result(jfg_server *s, int64_t ticket, double **nzk_dev, double **nzkg_dev, double **max_dev,
                             double *times3);
/* A batch's results (all its variants) return to the pool when the last of
 * its requests is released: release results as they complete. */
jfg_status jfg_server_release(jfg_server *s, int64_t ticket);
/* out6 = {submitted, completed, batches launched, largest batch, most pool bytes in use at once, queued}. */
jfg_status jfg_server_stats(jfg_server *s, int64_t *out6);
jfg_status jfg_server_family_batch(jfg_server *s, int32_t family, int32_t *batch_limit);
/* hold != 0: queue new requests without launching them; hold = 0 admits the
 * queue (a burst submitted under hold is batched as a whole). */
jfg_status jfg_server_hold(jfg_server *s, int32_t hold);
const char *jfg_server_last_error(jfg_server *s);
void jfg_server_destroy(jfg_server *s);

/* Current shell thicknesses of the handle (PSHELL T after any update):
 * n_quad4 + n_tria3 doubles, CQUAD4s then CTRIA3s, the jfg_update_properties
 * layout. */
jfg_status jfg_shell_thickness(jfg_model *m, double *h_host);

/* ---- Launch-shape autotuner ------------------------------------------------
 * No counterpart in the reference, whose assembly loops are CPU threads.
 * jfg_autotune times the candidate CTA shapes of every element kernel on this
 * handle's model (K and, unless KG raises for the deck, KG assemblies, device
 * times from the handle's timing events) and keeps the fastest of each:
 *   cfg[0] warps per CQUAD4 CTA, 4 or 8 (12 or 24 elements per CTA)
 *   cfg[1] warps per CTRIA3-stiffness CTA, 2 or 4 (4 or 8 elements)
 *   cfg[2..4] elements per CTA of the CTRIA3 KG, bar K and bar KG kernels
 *          (one thread per CTRIA3, per bar node pair): 32, 64 or 128
 * The choice is stored per kernel and model-size class (floor(log2) of the
 * element count of the kernel's type) in a text file: JFG_TUNE_FILE, else
 * $HOME/.cache/jfem_b200/launch_tune.txt.  flags: JFG_TUNE_READ takes a stored
 * choice when every kernel's size class has one (no timing); JFG_TUNE_WRITE
 * stores the choice made.  The tuner overwrites the handle's work buffers
 * (its last K / KG values).  cfg_out (5 int32) may be NULL.
 * jfg_launch_config sets (cfg_in) and/or reads (cfg_out) the shapes. */
#define JFG_TUNE_READ 1
#define JFG_TUNE_WRITE 2
jfg_status jfg_autotune(jfg_model *m, int32_t flags, int32_t *cfg_out);
jfg_status jfg_launch_config(jfg_model *m, const int32_t *cfg_in, int32_t *cfg_out);

/* ---- Group handles: several models in one launch ------------------------
 * The reference assembles one model per call; its batch drivers loop over
 * models and design variants (tools/manifest_batch_core.jl:283-409,
 * src/solver/optimize_thickness.jl:209-240).  A group handle holds several
 * decks side by side as disjoint components: every element-kernel and
 * reduction launch takes bins from all members, of uneven sizes and mixed
 * element types, and jfg_assemble_batch_device runs design variants of every
 * member in the same launches (one CUDA graph when captured).  The handle is a
 * jfg_model: every entry point above works on it and jfg_model_destroy frees
 * it.  Members must share PARAM K6ROT; each is validated against its own
 * index ranges.  A member's dofs are [6 node_off, 6 (node_off + n_nodes)),
 * its CSC columns the same range and its nonzeros [nnz_off, nnz_off + nnz);
 * rows there are the member's own rows offset by 6 node_off.  Its values are
 * bit for bit those of the member on its own handle.  max_elem_stiff is the
 * group's (the max over members). */
jfg_status jfg_group_create(int32_t n, const jfg_model_desc *const *descs, jfg_model **out);
/* out8: n_nodes, node_off, nnz, nnz_off, CQUAD4 offset, CTRIA3 offset, bar
 * offset, element count of member i. */
jfg_status jfg_group_member(jfg_model *m, int32_t i, int64_t *out8);

/* ---- Allocation-free CQUAD4 stiffness assembly ---------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory where they need a stiffness matrix: a host framework that has
 * reserved all device memory up front and hands out only its own buffers,
 * or a real-time loop that forbids allocator calls because they may block or
 * synchronise the device.  Assembles K of a small patch of CQUAD4 elements
 * into a caller-provided CSR value array without allocating anything.
 *
 * All pointers are device memory: coords (n_nodes*3), node_R (n_nodes*9 or
 * NULL), quad4_nodes (n_quad4*4, 0-based), quad4_prop (n_quad4*JFG_SHELL_PROP),
 * and the 0-based symmetric CSR pattern rowptr (6*n_nodes+1) / colind that
 * holds every element entry -- the arrays jfg_pattern_fill returns, minus 1,
 * for a CQUAD4-only model.  nzval receives one value per stored entry in the
 * same order (entries no element touches are written as 0).  stream is a
 * cudaStream_t (NULL: the legacy default stream).  The call is synchronous:
 * it waits for the stream after its input checks and again before it
 * returns, to read the status back.
 *
 * Input checks are those of jfg_model_create for CQUAD4: a node index outside
 * [0, n_nodes), a repeated node, or thickness or E not positive give
 * JFG_ERR_INVALID; a non-flat quad (outside the flat default branch) gives
 * JFG_ERR_UNSUPPORTED.  These run on the device before the element kernel,
 * and nothing else is launched when one fails.
 *
 * Intermediate data lives in one fixed array in the library's device image
 * (about 6.3 MB, held by every GPU that loads the library until the process
 * exits).  Limits: n_quad4 <= JFG_NOALLOC_MAX_QUAD4, n_nodes <=
 * JFG_NOALLOC_MAX_NODES (both checked before any launch), at most
 * JFG_NOALLOC_MAX_VALENCE elements per node (checked on the device); larger
 * inputs give JFG_ERR_UNSUPPORTED.  Whenever the status is not JFG_OK the
 * contents of nzval are unspecified.  The first call on each device looks up
 * the array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  Every call reuses the same array, so calls that
 * overlap on the GPU (concurrent streams or threads) race and must be
 * serialised by the caller. */
#define JFG_NOALLOC_MAX_QUAD4 2048
#define JFG_NOALLOC_MAX_NODES 8192
#define JFG_NOALLOC_MAX_VALENCE 8
jfg_status jfg_assemble_k_quad4_noalloc(int64_t n_nodes, const double *coords_dev, const double *node_R_dev,
                                        int64_t n_quad4, const int32_t *quad4_nodes_dev, const double *quad4_prop_dev,
                                        double k6rot, const int64_t *rowptr_dev, const int64_t *colind_dev,
                                        double *nzval_dev, void *stream);

void jfg_model_destroy(jfg_model *m);
const char *jfg_last_error(jfg_model *m);
const char *jfg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* JFEM_GPU_H */
