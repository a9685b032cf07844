/*
 * libemfem — B200 (sm_100a) kernels for EMerge's Nedelec-2 FEM hot path, behind a C ABI.
 *
 * Every pointer argument named *_dev (or documented as "device") is a device pointer on the
 * handle's device; "host" arrays are plain host memory.  Complex numbers are interleaved
 * (re, im) float64 pairs, the memory layout of numpy/torch complex128.  Arrays follow the
 * reference's layouts: nodes (3, N_n) f64, tets (4, N_t) i64, tet_to_edge (6, N_t) i64,
 * tet_to_field (20, N_t) i64, er/ur (3, 3, N_t) c128 — all row-major, i.e. structure-of-arrays
 * over elements.  All calls are asynchronous on the handle's stream unless stated otherwise and
 * return an int status (EMFEM_OK = 0, negative on error); emfem_last_error() gives the text.
 *
 * Reference paths below are relative to the EMerge source tree; ASM/ =
 * src/emerge/_emerge/physics/microwave/assembly/.
 */
#ifndef EMFEM_H
#define EMFEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EMFEM_OK 0
#define EMFEM_ERR_INVALID_ARG -1   /* bad size, null pointer, unsupported option */
#define EMFEM_ERR_CUDA -2          /* a CUDA runtime call failed */
#define EMFEM_ERR_DEVICE_CHECK -3  /* a kernel's own bounds / consistency check fired */
#define EMFEM_ERR_WORKSPACE -4     /* caller-provided workspace too small */
#define EMFEM_ERR_NOT_CONVERGED -5 /* iterative solve hit its iteration cap or broke down */

/* Device status bits reported by emfem_device_status(). */
#define EMFEM_DEV_BAD_INDEX 1
#define EMFEM_DEV_DEGENERATE 2
#define EMFEM_DEV_NONFINITE 4
#define EMFEM_DEV_CAPACITY 8
#define EMFEM_DEV_BREAKDOWN 16

/* Limits and sizes of the auxiliary-space preconditioner (emfem_aux_*, emfem_mpnn_*). */
#define EMFEM_MAX_PORTS 8
#define EMFEM_MPNN_CHANNELS 32   /* complex channels = 64 real */
#define EMFEM_MPNN_LAYERS 4
#define EMFEM_MPNN_NPARAMS (2 * 32 + 4 * 4 * 32 * 32 + 2 * 32)

typedef struct emfem_handle_s *emfem_handle;
typedef struct emfem_plan_s *emfem_plan;
typedef struct emfem_aux_s *emfem_aux;
typedef struct emfem_conn_s *emfem_conn;

/* ---- library / handle ------------------------------------------------------------------- */
int emfem_version(void);
/* Copies the calling thread's last error message (NUL-terminated, truncated to len). */
int emfem_last_error(char *buf, size_t len);
/* stream: a cudaStream_t (NULL = legacy default stream). */
int emfem_create(emfem_handle *h, int device, void *stream);
int emfem_set_stream(emfem_handle h, void *stream);
int emfem_destroy(emfem_handle h);
/* Synchronises the stream, returns the sticky device status bits (EMFEM_DEV_*) and clears them. */
int emfem_device_status(emfem_handle h, int *status);

/* ---- per-element integrator -------------------------------------------------------------
 * Replaces the numeric part of _matrix_builder (ASM/curlcurl.py:419-466), i.e. per tet
 * ned2_tet_stiff_mass(..., matinv(ur), er) (ASM/curlcurl.py:180-412).  Writes, for every tet t,
 * the row-major 20x20 curl-curl matrix to E_out[400 t ...] and the mass matrix to B_out, exactly
 * the reference's dataE/dataB.  Local edge/face orientation is taken from the global node ids
 * of `tets`, which is what the reference's local_mapping of the sorted edge/triangle node lists
 * yields for a mesh in Mesh3D conventions (mesh3d.py:387-497).
 * All arrays device.  edge_lengths has n_edges entries (indexed through tet_to_edge). */
int emfem_ned2_tet_matrices(emfem_handle h, int64_t n_nodes, int64_t n_tets, int64_t n_edges,
                            const double *nodes, const int64_t *tets, const int64_t *tet_to_edge,
                            const double *edge_lengths, const void *ur, const void *er,
                            void *E_out, void *B_out);

/* COO row/column indices of _matrix_builder (ASM/curlcurl.py:459-465): for k = 20 i + j of tet t,
 * rows[400 t + k] = tet_to_field[i, t], cols[400 t + k] = tet_to_field[j, t].  Device arrays. */
int emfem_ned2_coo_indices(emfem_handle h, int64_t n_tets, const int64_t *tet_to_field,
                           int64_t *rows, int64_t *cols);

/* Mesh consistency check against the Mesh3D conventions the integrator relies on
 * (mesh3d.py:395-441): edges[:, tet_to_edge[e, t]] is the sorted pair of local vertices e and
 * tris[:, tet_to_tri[f, t]] the sorted triple of local face f.  Sets EMFEM_DEV_BAD_INDEX on a
 * mismatch or out-of-range id; read it with emfem_device_status().  Device arrays. */
int emfem_mesh_check(emfem_handle h, int64_t n_nodes, int64_t n_tets, int64_t n_edges, int64_t n_tris,
                     const int64_t *tets, const int64_t *edges, const int64_t *tris,
                     const int64_t *tet_to_edge, const int64_t *tet_to_tri);

/* ---- CSR plan (symbolic phase) + fused assembly -----------------------------------------
 * Replaces tet_mass_stiffness_matrices (ASM/curlcurl.py:145-173): the COO emission of
 * _matrix_builder plus coo_matrix(...).tocsr() with duplicate summation.  The plan is built once
 * per mesh on the device from tet_to_field (device, (20, n_tets) i64): the pattern is the union of
 * all tet DOF pairs, rows sorted, explicit zeros kept — bit-identical to SciPy's tocsr() of the
 * reference's COO.  n_field = 2 n_edges + 2 n_tris.  The plan owns its device memory. */
int emfem_plan_create(emfem_handle h, int64_t n_tets, int64_t n_edges, int64_t n_tris,
                      const int64_t *tet_to_field, emfem_plan *plan);
int emfem_plan_info(emfem_plan plan, int64_t *n_field, int64_t *nnz);
int emfem_plan_destroy(emfem_plan plan);
/* indptr (n_field + 1) and indices (nnz), int32, device. */
int emfem_plan_export_csr(emfem_plan plan, int32_t *indptr, int32_t *indices);
/* Fused integrate + deterministic segmented reduction: writes the CSR values of E (curl-curl) and
 * B (mass), nnz complex each, device.  Every CSR slot is the sum of its tets' contributions in
 * ascending tet order, so repeated calls are bit-identical.  Inputs as emfem_ned2_tet_matrices. */
int emfem_plan_assemble(emfem_plan plan, int64_t n_nodes, int64_t n_edges, const double *nodes,
                        const int64_t *tets, const int64_t *tet_to_edge, const double *edge_lengths,
                        const void *ur, const void *er, void *E_vals, void *B_vals);
/* Kernel variants of emfem_plan_assemble (chunk capacity x threads per CTA).  A project autotuner
 * (emerge_b200.assembly.CsrPlan.tune) times them on the device and selects the fastest; variants
 * whose chunk cannot hold the mesh's largest edge/face incidence are unavailable. */
int emfem_plan_variants(emfem_plan plan, int *n_variants, int *current);
int emfem_plan_set_variant(emfem_plan plan, int variant);
/* Variant v: chunk capacity (incidences), threads per CTA, and whether this mesh can use it. */
int emfem_plan_variant_info(emfem_plan plan, int variant, int *chunk, int *threads, int *available);
/* CSR slot of each (row, col) pair (device int64 arrays of length n), -1 where absent. */
int emfem_plan_find_slots(emfem_plan plan, int64_t n, const int64_t *rows, const int64_t *cols,
                          int32_t *slots);

/* ---- Robin / port triangles ----------------------------------------------------------------
 * Replaces ned2_tri_stiff_force / ned2_tri_stiff (ASM/robinbc.py:126-292, :314-427) for a batch of
 * boundary triangles.  tri_nodes: (3, n_sel) i64 global node ids of the selected triangles (the
 * reference's tris[:, surf_triangle_indices]); U: (3, npts, n_sel) c128 incident field at the
 * quadrature points as assemble_robin_bc_excited reshapes it (ASM/robinbc.py:445-463), or NULL;
 * dpts: (4, npts) f64 [W, L1, L2, L3] with npts <= 16.  Outputs: blocks (n_sel, 64) c128 — the
 * row-major 8x8 γ-scaled matrices — and, when U is given, bvec (n_sel, 8) c128.  Device arrays. */
int emfem_ned2_tri_robin(emfem_handle h, int64_t n_nodes, const double *nodes, int64_t n_sel,
                         const int64_t *tri_nodes, double gamma_re, double gamma_im,
                         const void *U, const double *dpts, int npts, void *blocks, void *bvec);

/* Deterministic segmented sum: out[i] = sum_{k=seg[i]}^{seg[i+1]-1} src[idx[k]] in k order
 * (complex128, device).  Used to scatter Robin blocks and port vectors onto CSR slots / DOFs. */
int emfem_segmented_gather_sum(emfem_handle h, int64_t n_out, const int32_t *seg, const int32_t *idx,
                               const void *src, void *out);

/* ---- frequency-sweep system ------------------------------------------------------------------
 * K = (E - k0^2 B) on the plan pattern (the product rounded first, as the reference's E - B*K0**2),
 * then K[patch_slot[i]] += gamma * patch_vals[i] (ASM/assembler.py:255 and :349-350).  The slots of one
 * call must be distinct (sum duplicates first, e.g. with emfem_segmented_gather_sum).  Device arrays;
 * nnz complex each. */
int emfem_sweep_combine(emfem_handle h, int64_t nnz, const void *E_vals, const void *B_vals, double k0sq,
                        int64_t n_patch, const int32_t *patch_slot, const void *patch_vals,
                        double gamma_re, double gamma_im, void *K_vals);

/* Exact zeros dropped from a CSR matrix, the other entries kept in order: the layout SciPy gives the
 * result of E - B*K0**2 and K + B_p (ASM/assembler.py:255, :350), whose sparse arithmetic stores only
 * nonzero results.  count: out_indptr (n + 1) i32 gets the compacted row pointers and *nnz_out (host)
 * the kept count (synchronises the stream); workspace (device) holds emfem_csr_drop_zeros_workspace()
 * bytes.  compact: out_indices (nnz_out) i32 and out_vals (nnz_out) c128.  Device arrays. */
int emfem_csr_drop_zeros_workspace(int64_t n, size_t *bytes);
int emfem_csr_count_nonzero(emfem_handle h, int64_t n, const int32_t *indptr, const void *vals, int32_t *out_indptr,
                            void *workspace, size_t workspace_bytes, int64_t *nnz_out);
int emfem_csr_compact_nonzero(emfem_handle h, int64_t n, const int32_t *indptr, const int32_t *indices,
                              const void *vals, const int32_t *out_indptr, int32_t *out_indices, void *out_vals);

/* ---- batched Krylov solver ------------------------------------------------------------------
 * Solves nsys systems A_s x_s = b_s on one CSR pattern, replacing the per-frequency direct solve
 * (SolverSuperLU, src/emerge/_emerge/solver.py:535-572, reached through SolveRoutine.solve
 * :1241-1326).  A_s = E - k0sq[s] * B + sum_p gamma[s, p] * R_p, where B may be NULL (then
 * A_s = E + ...), and the Robin terms R_p are given as a small row-compressed "patch"
 * (patch_rows, patch_rowptr (n_patch_rows + 1), patch_cols, patch_vals, patch_port).  Rows and
 * columns where free_mask == 0 are eliminated exactly as SolveRoutine's submatrix A[ids, ids]
 * (their solution entries are zero).  Vectors are (n, nsys) c128, DOF-major (entry (i, s) at
 * i * nsys + s).  x holds the initial guess on entry (zero for the reference's behaviour) and the
 * solution on exit.  k0sq (nsys) and gamma (nsys * n_ports complex) are host arrays.
 *   method:    0 = COCG (complex-symmetric A only), 1 = right-preconditioned BiCGStab (general A;
 *              the reference's mass matrix is not symmetric, so this is the default).
 *   precond:   0 none, 1 point Jacobi, 2 block Jacobi on DOF pairs (i, i + n/2) — the first- and
 *              second-kind DOFs of one edge/face (elements/nedelec2.py:42-58); 3 block Jacobi plus
 *              the auxiliary-space (discrete-gradient) correction with aux-space Jacobi, 4 block
 *              Jacobi plus the correction through the learned network.  3 and 4 need method 1 and
 *              `aux` (emfem_aux_create / _set_operator with the same ports / _reserve, and for 4
 *              _set_network); `aux` is ignored (may be NULL) for precond 0-2.  The reference has no
 *              preconditioner: it factorises directly.
 *   precision: 0 = FP64 Krylov; 1 = FP32 inner Krylov inside FP64 iterative refinement (FP64
 *              residual, solution update and convergence test).
 * Host outputs per system: status (0 converged, 1 iteration cap, 2 breakdown/stagnation), iters,
 * relres (FP64 true relative residual ||b - A x|| / ||b|| over free DOFs).  workspace (device)
 * must hold emfem_krylov_workspace_size() bytes.  Synchronises the stream.  Returns
 * EMFEM_ERR_NOT_CONVERGED when any system missed the tolerance (outputs still filled). */
int emfem_krylov_workspace_size(int64_t n, int64_t nnz, int nsys, int precision, size_t *bytes);
int emfem_krylov_solve(emfem_handle h, int method, int64_t n, int64_t nnz, const int32_t *indptr,
                       const int32_t *indices, const void *E_vals, const void *B_vals, int nsys,
                       const double *k0sq, int64_t n_patch_rows, const int32_t *patch_rows,
                       const int32_t *patch_rowptr, const int32_t *patch_cols, const void *patch_vals,
                       const int32_t *patch_port, int n_ports, const double *gamma,
                       const uint8_t *free_mask, const void *rhs, void *x, double tol, int maxit,
                       int precond, int precision, void *workspace, size_t workspace_bytes,
                       int *status, int *iters, double *relres, emfem_aux aux);

/* Many meshes in one batched solve.  The vectors hold G groups of nsys systems: row i (and i + n/2)
 * of column s belongs to system (pair_group[i], s), pair_group (n/2) i32 on the device, running
 * through 0..G-1 in order with every group starting at a multiple of 256 DOF pairs (pad a group's
 * rows with eliminated DOFs).  The CSR is block diagonal over the groups.  k0sq (G nsys), gamma
 * (G nsys n_ports complex) are host arrays; status / iters / relres have G nsys entries; rhs and x
 * are (n, nsys) c128.  precision 0 (FP64) or 1 (FP32 inner solves in FP64 refinement), precond 0-4 (3 and 4 with an aux space moved onto the grouped rows
 * by emfem_aux_set_rows, same ngroups; the network's weights are per node type, so one network serves
 * every mesh), method 0 or 1 (1 for precond 3-4); otherwise as emfem_krylov_solve.
 * One graph-captured iteration serves every system of every group; each system keeps its own
 * scalars and convergence test. */
int emfem_krylov_workspace_size_grouped(int64_t n, int64_t nnz, int nsys, int ngroups, int precision,
                                        size_t *bytes);
int emfem_krylov_solve_grouped(emfem_handle h, int method, int64_t n, int64_t nnz, const int32_t *indptr,
                               const int32_t *indices, const void *E_vals, const void *B_vals, int ngroups,
                               const int32_t *pair_group, int nsys, const double *k0sq, int64_t n_patch_rows,
                               const int32_t *patch_rows, const int32_t *patch_rowptr, const int32_t *patch_cols,
                               const void *patch_vals, const int32_t *patch_port, int n_ports, const double *gamma,
                               const uint8_t *free_mask, const void *rhs, void *x, double tol, int maxit, int precond,
                               int precision, void *workspace, size_t workspace_bytes, int *status, int *iters,
                               double *relres, emfem_aux aux);

/* y_s = A_s x_s for the operator of emfem_krylov_solve (FP64), eliminated rows/cols as there;
 * nsys a power of two <= 256; k0sq_dev and gamma_dev are device arrays. */
int emfem_sweep_spmv(emfem_handle h, int64_t n, const int32_t *indptr, const int32_t *indices,
                     const void *E_vals, const void *B_vals, int nsys, const double *k0sq_dev,
                     int64_t n_patch_rows, const int32_t *patch_rows, const int32_t *patch_rowptr,
                     const int32_t *patch_cols, const void *patch_vals, const int32_t *patch_port,
                     int n_ports, const double *gamma_dev, const uint8_t *free_mask,
                     const void *x, void *y);

/* Second-order absorbing-boundary correction: abc_order_2_matrix's per-triangle 8x8 blocks
 * (ASM/robin_abc_order2.py:192-373), cf * L_i L_j (int curl_t N_i curl_t N_j - int div_t N_i div_t N_j) |A|
 * in the triangle's plane frame with that module's 6-point rule.  tri_nodes (3, n_sel) i64 sorted
 * node ids; blocks (n_sel, 64) c128 row-major, DOF order of tri_to_field.  Device arrays. */
int emfem_ned2_tri_abc2(emfem_handle h, int64_t n_nodes, const double *nodes, int64_t n_sel,
                        const int64_t *tri_nodes, double cf_re, double cf_im, void *blocks);

/* ---- boundary-mode analysis (port modes) ----------------------------------------------------
 * Replaces generalized_matrix_GQ / _matrix_builder (ASM/generalized_eigen_hb.py:257-458), called by
 * Assembler.assemble_bma_matrices (ASM/assembler.py:110-187): the 14x14 blocks A ("E") and B ("B") of
 * the mixed Nedelec-2 / Lagrange-2 triangle element of every port-face triangle, DOF order
 * tri_to_field of NedelecLegrange2 (elements/nedleg2.py:140-150), for the eigenproblem
 * A e = -beta^2 B e.  local_nodes (2, n_nodes) f64: x then y in the port's local frame; tris (3, n_tris)
 * and tri_to_edge (3, n_tris) i64; edges (2, n_edges) i64 (any node order; it fixes the edge
 * orientation); er, ur (9, n_tris) c128 row-major 3x3 per triangle (the reference's (3,3,N) layout);
 * A, B (n_tris, 196) c128 row-major, i.e. the reference's dataE / dataB.  Device arrays. */
int emfem_ned2_bma_tri_matrices(emfem_handle h, int64_t n_nodes, const double *local_nodes, int64_t n_tris,
                                const int64_t *tris, int64_t n_edges, const int64_t *edges,
                                const int64_t *tri_to_edge, const void *er, const void *ur, double k0, void *A,
                                void *B);

/* A port-mode vector x (n_field) c128 of the NedelecLegrange2 field evaluated at points inside known
 * triangles: what = 0 gives E (ned2_tri_interp_full, elements/nedleg2.py -> elements/ned2_interp.py:616-685),
 * what = 1 the curl form of ned2_tri_interp_curl (:687-760) without its constant j/(k0 c0 mu0):
 * (d_y E_z - j beta E_y, -d_x E_z + j beta E_x, curl_t E_t), each component times the diagonal of
 * diadic (3, n_tris) c128 (ur^-1), or of the identity when diadic is NULL.  pts (2, npts, n_tris) f64
 * local coordinates, column t inside triangle t; tri_to_field (14, n_tris) i64; out (3, npts, n_tris)
 * c128 in the port's local frame.  Device arrays. */
int emfem_ned2_tri_field(emfem_handle h, int64_t n_nodes, const double *local_nodes, int64_t n_tris,
                         const int64_t *tris, int64_t n_edges, const int64_t *edges, const int64_t *tri_to_edge,
                         const int64_t *tri_to_field, int64_t n_field, const void *x, int npts, const double *pts,
                         int what, double beta_re, double beta_im, const void *diadic, void *out);

/* ---- S-parameter overlap integrals -------------------------------------------------------------
 * For the port triangles (tri_nodes (3, n_tri) i64, their owning tets tri_tet (n_tri) i64) and nsys
 * solutions x (n_field, nsys) c128, computes the port-mode overlap of every solution,
 *   overlap[s] = sum_t c_t A_t sum_p W_p E_s(x_p) . conj(shape(x_p)),
 * and the mode norm N = sum_t c_t A_t sum_p W_p |shape(x_p)|^2, with E interpolated in the owning
 * tet as ned2_tet_interp does (src/emerge/_emerge/elements/ned2_interp.py:142-300) and the integrals
 * of sparam_field_power / sparam_mode_power (src/emerge/_emerge/physics/microwave/sparam.py:71-138).
 * S[q, p] = (overlap / (scale_q(k0) N) - [q == p]) / sqrt(P_p), scale = the mode's amplitude factor.
 * shape: (3, npts, n_tri) c128 unit mode at the quadrature points; tri_const: (n_tri) c128 (TE:
 * 1/mean(diag ur)); dpts (4, npts) with npts <= 16; work: device scratch of 16 n_tri (nsys + 1)
 * bytes; overlap (nsys) and mode_norm (1) c128, device. */
int emfem_port_overlap(emfem_handle h, int64_t n_nodes, const double *nodes, int64_t n_tets, const int64_t *tets,
                       const int64_t *tet_to_field, int64_t n_field, int64_t n_tri, const int64_t *tri_tet,
                       const int64_t *tri_nodes, const double *dpts, int npts, const void *shape,
                       const void *tri_const, int nsys, const void *x, void *work, void *overlap, void *mode_norm);

/* E . dl at arbitrary points: for point p inside tet pt_tet[p] (the caller locates it), the Nedelec-2
 * field of each solution (ned2_tet_interp's formulas, elements/ned2_interp.py:230-295) dotted with
 * dl[3 p .. 3 p + 2]; out (npts, nsys) c128.  Used for lumped-port voltage lines
 * (physics/microwave/microwave_3d.py:1271-1291).  pts (3, npts) f64; x (n_field, nsys) c128; device. */
int emfem_point_field_dot(emfem_handle h, int64_t n_nodes, const double *nodes, int64_t n_tets, const int64_t *tets,
                          const int64_t *tet_to_field, int64_t n_field, int64_t npts, const int64_t *pt_tet,
                          const double *pts, const double *dl, int nsys, const void *x, void *out);

/* ---- mesh connectivity ---------------------------------------------------------------------
 * Replaces the connectivity part of Mesh3D._pre_update (src/emerge/_emerge/mesh3d.py:385-497):
 * the unique sorted edge / triangle node lists in lexicographic order (:386-406), tet_to_edge with
 * local pairs (1,2),(1,3),(1,4),(2,3),(4,2),(3,4) (:427), tet_to_tri with local triples
 * (1,2,3),(1,3,4),(1,4,2),(2,3,4) (:431), tri_to_tet with the tets in ascending order, padded with
 * EMFEM_MISSING_ID (:27, :437-447), tri_to_edge as (i1,i2),(i2,i3),(i1,i3) of the sorted triple (:470-481) and
 * edge_lengths (:497).  Ids are identical to the reference's.
 * create: tets (4, n_tets) i64, device; checks node ids are in range and distinct per tet
 * (EMFEM_ERR_DEVICE_CHECK otherwise), builds the per-node edge / triangle buckets and synchronises
 * the stream once to learn the counts.  info: the counts, host.  export: writes, all device,
 * edges (2, n_edges) i64, tris (3, n_tris) i64, tet_to_edge (6, n_tets), tet_to_tri (4, n_tets),
 * tri_to_edge (3, n_tris), tri_to_tet (2, n_tris) i64 and edge_lengths (n_edges) f64 from nodes
 * (3, n_nodes) f64; `tets` must be the array given to create.  A triangle shared by more than two
 * tets (a non-manifold mesh, which the reference rejects) keeps the two smallest tet ids and sets
 * EMFEM_DEV_CAPACITY. */
#define EMFEM_MISSING_ID (-1234)  /* Mesh3D's _MISSING_ID (mesh3d.py:27) */
int emfem_mesh_connect_create(emfem_handle h, int64_t n_nodes, int64_t n_tets, const int64_t *tets, emfem_conn *c);
int emfem_mesh_connect_info(emfem_conn c, int64_t *n_edges, int64_t *n_tris);
int emfem_mesh_connect_export(emfem_conn c, const double *nodes, const int64_t *tets, int64_t *edges, int64_t *tris,
                              int64_t *tet_to_edge, int64_t *tet_to_tri, int64_t *tri_to_edge, int64_t *tri_to_tet,
                              double *edge_lengths);
int emfem_mesh_connect_destroy(emfem_conn c);

/* ---- auxiliary nodal space and learned preconditioner -----------------------------------------
 * No counterpart in the reference (it factorises every system directly, solver.py:535-572).
 * The aux space has one node per mesh vertex (aux id v) and per mesh edge (aux id n_nodes + e); G
 * (n_field x n_aux) is the exact discrete gradient of the second-order nodal functions L_v and
 * L_a L_b in the reference's Nedelec-2 basis (elements/ned2_interp.py:248-295), built per entity
 * from edges (2, n_edges), tris (3, n_tris), tri_to_edge (3, n_tris) and edge_lengths (device,
 * Mesh3D layouts).  The preconditioner of precond 3/4 is M r = BJ r + G N(D_a^-1 G^T r) with
 * D_a = diag(G^T A_s G) per system and N the identity (3) or the network (4).
 * create: builds G (ELL, 6 per row), G^T (CSR) and the vertex-edge incidence graph; synchronises.
 * info: n_aux, nnz of G^T and of the graph.  export: device copies (any pointer may be NULL):
 *   gcol (n_field, 6) i32 (-1 = empty), gval (n_field, 6) f64, G^T ptr/row/val, graph ptr/nbr.
 * set_operator: the operator of emfem_krylov_solve (same arguments) -> diag(G^T E G), diag(G^T B G),
 *   diag(G^T R_p G) and the aux mask (1 where every DOF touched is free).  diag_out (optional,
 *   device): (2 + n_ports) * n_aux c128 [dE | dB | dR_0 ..]; mask_out (optional, device) n_aux u8.
 * reserve: allocates the solve-time buffers for up to nsys systems (call before emfem_krylov_solve).
 * set_network: device float params (EMFEM_MPNN_NPARAMS, layout below) used by precond 4; the
 *   caller keeps them alive.
 * dinv: dinv (n_aux, nsys) c128 = 1 / (dE - k0sq_s dB + sum_p gamma_{s,p} dR_p), 0 off the mask;
 *   k0sq_dev (nsys) and gamma_dev (nsys * n_ports complex) device.
 * restrict: x = dinv .* (G^T v) (dinv NULL: no scaling), v (n_field, nsys), x (n_aux, nsys) c128.
 * prolong: z (+)= G za on rows with free_mask (NULL: all rows), c128. */
int emfem_aux_create(emfem_handle h, int64_t n_nodes, int64_t n_edges, int64_t n_tris, const int64_t *edges,
                     const int64_t *tris, const int64_t *tri_to_edge, const double *edge_lengths, emfem_aux *aux);
int emfem_aux_info(emfem_aux aux, int64_t *n_aux, int64_t *nnz_gt, int64_t *nnz_graph);
int emfem_aux_export(emfem_aux aux, int32_t *gcol, double *gval, int32_t *gt_ptr, int32_t *gt_row, double *gt_val,
                     int32_t *graph_ptr, int32_t *graph_nbr);
int emfem_aux_set_operator(emfem_aux aux, int64_t n, const int32_t *indptr, const int32_t *indices,
                           const void *E_vals, const void *B_vals, int64_t n_patch_rows, const int32_t *patch_rows,
                           const int32_t *patch_rowptr, const int32_t *patch_cols, const void *patch_vals,
                           const int32_t *patch_port, int n_ports, const uint8_t *free_mask, void *diag_out,
                           uint8_t *mask_out);
/* Moves the aux space onto the rows of a grouped (multi-mesh) system: row r of its own numbering
 * becomes row new_of_old[r] (device i64, n_old entries) of an n_new-row system; aux_group (device i32,
 * n_aux entries) is the group of every aux node, null when ngroups is 1.  Call before
 * emfem_aux_set_operator with the grouped operator.  No counterpart in the reference. */
int emfem_aux_set_rows(emfem_aux aux, int64_t n_new, const int64_t *new_of_old, int ngroups, const int32_t *aux_group);
int emfem_aux_reserve(emfem_aux aux, int nsys);
int emfem_aux_set_network(emfem_aux aux, const float *params);
int emfem_aux_destroy(emfem_aux aux);
int emfem_aux_dinv(emfem_aux aux, int nsys, const double *k0sq_dev, const double *gamma_dev, void *dinv);
int emfem_aux_restrict(emfem_aux aux, int nsys, const void *dinv, const void *v, void *x);
int emfem_aux_prolong(emfem_aux aux, int nsys, const void *za, const uint8_t *free_mask, void *z, int accumulate);

/* The network (training and inference kernels).  Aux-space vectors x, za are (n_aux, nsys) c64
 * (FP32 complex); activations are FP32.  With t = 0 for vertex and 1 for edge aux nodes, N(y) the
 * incidence-graph neighbours and real weights:
 *   H_0 = x w_in[t];  H_{l+1,y} = H_{l,y} W_l[t_y] + (1/|N(y)|) sum_{j in N(y)} H_{l,j} U_l[t_y];
 *   za_y = x_y + H_{4,y} . w_out[t_y]           (linear in x, so M stays a fixed linear operator)
 * params (float): w_in[2][32] | (W_l[2][32][32] | U_l[2][32][32]) for l = 0..3 | w_out[2][32].
 * workspace_floats: sizes of act (forward output, all layers) and scratch (backward).
 * forward: za and act.  backward: grad (EMFEM_MPNN_NPARAMS floats, overwritten) of a real loss L
 *   given dza = dL/dRe(za) + i dL/dIm(za) (c64), from the act of the forward of the same x; the
 *   sums over nodes are fixed-order.  adam_step: one Adam update (bias-corrected, L2 weight decay
 *   added to the gradient) of params with moments m, v (device, n floats); step >= 1. */
int emfem_mpnn_nparams(void);
int emfem_mpnn_workspace_floats(emfem_aux aux, int nsys, int64_t *activation_floats, int64_t *scratch_floats);
int emfem_mpnn_forward(emfem_aux aux, int nsys, const float *params, const void *x, float *act, void *za);
/* Inference form used inside emfem_krylov_solve (precond 4): the same network on the tensor cores
 * (TF32 inputs, FP32 accumulation); work holds 2 * n_aux * nsys * 64 floats. */
int emfem_mpnn_infer(emfem_aux aux, int nsys, const float *params, const void *x, float *work, void *za);
int emfem_mpnn_backward(emfem_aux aux, int nsys, const float *params, const void *x, const float *act,
                        const void *dza, float *grad, float *scratch);
int emfem_adam_step(emfem_handle h, int64_t n, float *params, const float *grad, float *m, float *v, float lr,
                    float beta1, float beta2, float eps, float weight_decay, int step);

/* ---- multifrontal LU (device direct solve) ---------------------------------------------------
 * Replaces the reference's direct solve, SolverSuperLU (src/emerge/_emerge/solver.py:535-572, SuperLU
 * with MMD ordering), for the sweep system on a CSR pattern.  The host builds the symbolic structure
 * (emerge_b200/direct.py: nested dissection of the mesh's tets, fronts, assembly lists); the library
 * factors and solves on the device in complex64 (fronts) with FP64 input and output.
 * create (host arrays; allocates all device memory once): n_fronts fronts in postorder (children before
 *   parents, each front at most two children); e / b: eliminated and boundary DOFs per front (e + b <=
 *   46340); parent (-1 for the root), level (height, leaves 0; a parent's level exceeds its children's);
 *   fdof[fdof_ptr[v] .. fdof_ptr[v + 1]): the front's DOFs (own, then boundary, as CSR row numbers);
 *   ea: for every front in order, the position of each of its b boundary DOFs in its parent's front;
 *   asm_slot / asm_off (asm_ptr per front): the CSR slots assembled into each front and their local
 *   offsets row + col * (e + b).  The three assembly arrays may all be NULL; then
 *   emfem_mf_build_lists builds them on the device from the CSR pattern (device indptr (n + 1) and
 *   indices (nnz), int32), which must come before the first factorization.
 * info: device bytes held, factorization flops, number of levels.
 * factor: K_vals (nnz c128, device) on the CSR pattern the structure was built for; the factorization
 *   runs on the equilibrated D^-1/2 K D^-1/2 (D = |diag K|_1, 1 where the diagonal is zero), and solve
 *   undoes the scaling; *n_perturbed (host) gets the number of pivots raised to 1e-6 of their 32 x 32
 *   block's largest entry (pivoting is partial inside each 32-row diagonal block).  Synchronises the
 *   stream.
 * set_precision: bits = 64 (default) factors in complex64, 128 in complex128 (the level workspace and
 *   the update store double in size; the factor store stays complex64, rounded once at compaction).
 *   Reallocates the workspace and drops the factorization; on an allocation failure the handle stays
 *   complex64 and the call returns the error.
 * reserve: solve buffers for up to nrhs right-hand sides (<= 256).
 * solve: x = (LU)^-1 b for nrhs right-hand sides, b and x (n, nrhs) c128 DOF-major, device; x is zero on
 *   DOFs that belong to no front (PEC).
 * emfem_krylov_solve_lu: FP64 right-preconditioned BiCGStab of emfem_krylov_solve (same operator and
 *   arguments) with M = this factorization for every system; the factorization may belong to another
 *   frequency of the same mesh (a window of a sweep shares one).  Reserve the padded batch size
 *   (next power of two of nsys) first. */
typedef struct emfem_mf_s *emfem_mf;
int emfem_mf_create(emfem_handle h, int64_t n, int n_fronts, const int32_t *e, const int32_t *b, const int32_t *parent,
                    const int32_t *level, const int64_t *fdof_ptr, const int32_t *fdof, const int32_t *ea,
                    const int64_t *asm_ptr, const int32_t *asm_slot, const int32_t *asm_off, emfem_mf *out);
int emfem_mf_build_lists(emfem_mf lu, int64_t nnz, const int32_t *indptr, const int32_t *indices);
int emfem_mf_info(emfem_mf lu, size_t *device_bytes, double *flops, int *n_levels);
int emfem_mf_factor(emfem_mf lu, const void *K_vals, int *n_perturbed);
int emfem_mf_set_precision(emfem_mf lu, int bits);
int emfem_mf_reserve(emfem_mf lu, int nrhs);
int emfem_mf_solve(emfem_mf lu, int nrhs, const void *b, void *x);
int emfem_mf_destroy(emfem_mf lu);
int emfem_krylov_solve_lu(emfem_handle h, int64_t n, int64_t nnz, const int32_t *indptr, const int32_t *indices,
                          const void *E_vals, const void *B_vals, int nsys, const double *k0sq, int64_t n_patch_rows,
                          const int32_t *patch_rows, const int32_t *patch_rowptr, const int32_t *patch_cols,
                          const void *patch_vals, const int32_t *patch_port, int n_ports, const double *gamma,
                          const uint8_t *free_mask, const void *rhs, void *x, double tol, int maxit, emfem_mf lu,
                          void *workspace, size_t workspace_bytes, int *status, int *iters, double *relres);

/* ---- allocation-free sweep SpMV ------------------------------------------------------------
 * No counterpart in the reference.  The same y_s = A_s x_s as emfem_sweep_spmv, for callers that
 * cannot call cudaMalloc: applications whose device memory is owned up front by their own pool
 * allocator, and latency-critical loops that cannot afford an allocation's implicit device
 * synchronisation.  Its only scratch (one int per row: the row -> Robin-patch-row map) lives in a
 * fixed device array of EMFEM_NOALLOC_MAX_ROWS ints (16 MiB) inside the library, held by every GPU
 * that loads the library until the process exits; larger n is rejected with EMFEM_ERR_INVALID_ARG.
 * It calls no cudaMalloc/cudaFree.  The first call on a device resolves the array's device address
 * (cudaGetSymbolAddress) once per context (a new context after cudaDeviceReset resolves it again);
 * make that first call before any stream capture.  All calls share the
 * array (each call resets the rows it uses), so calls that overlap on the GPU race.  Arguments as
 * emfem_sweep_spmv. */
#define EMFEM_NOALLOC_MAX_ROWS 4194304
int emfem_sweep_spmv_noalloc(emfem_handle h, int64_t n, const int32_t *indptr, const int32_t *indices,
                             const void *E_vals, const void *B_vals, int nsys, const double *k0sq_dev,
                             int64_t n_patch_rows, const int32_t *patch_rows, const int32_t *patch_rowptr,
                             const int32_t *patch_cols, const void *patch_vals, const int32_t *patch_port,
                             int n_ports, const double *gamma_dev, const uint8_t *free_mask,
                             const void *x, void *y);

#ifdef __cplusplus
}
#endif
#endif
