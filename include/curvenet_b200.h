/* curvenet_b200.h -- C ABI of the B200 (sm_100a) sparse solve of the
 * profile-curves deformer: cut-mesh cotangent-Laplacian assembly into CSR,
 * IC(0) / Jacobi / HSC preconditioned CG in FP64 or FP32-with-FP64-refinement,
 * the deform (Stage 2) and harmonic solves, batched solves and the adjoint.
 *
 * The reference's C++ runtime headers (src/curvenet/sparse_linalg.h,
 * incomplete_cholesky.h, hierarchical_sparsify.h, cut_mesh_laplacian.h,
 * harmonic_solve.h, deform_solve.h, gpu_cg_solver.h, gpu_cg_multi_solver.h)
 * are not part of the reference snapshot; the Lean specification states that
 * it mirrors them 1:1 (lean/Curvenet/SparseLinAlg.lean:24,
 * lean/Curvenet/HalfedgeBuilder.lean:4).  Each entry point below cites the
 * Lean function whose behaviour it takes over.
 *
 * Conventions: plain pointers and sizes only; every array is row-major;
 * host arrays belong to the caller; a cn_handle owns its device memory, its
 * CUDA stream, the factor and the warm-start state.  A handle is not
 * thread-safe; distinct handles may be used from distinct threads.  Errors
 * are status codes, never aborts.
 */
#ifndef CURVENET_B200_H
#define CURVENET_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CN_OK = 0,
  CN_MAX_ITER = 1,            /* tolerance not reached within max_iter / max_refine */
  CN_SINGULAR_COMPONENT = 2,  /* a connected component of the cut mesh has no handle */
  CN_NONPOS_PIVOT = 3,        /* IC(0) pivot <= 0 and the diagonal-shift retries ran out */
  CN_NAN = 4,                 /* non-finite input or iterate */
  CN_BREAKDOWN = 5,           /* p.Ap <= 0 inside PCG */
  CN_TIMEOUT = 6,             /* a bounded device-side wait ran out */
  CN_BAD_INPUT = 7,
  CN_CUDA_ERROR = 8,
  CN_NO_DEVICE = 9
} cn_status;

typedef struct cn_system* cn_handle;
typedef struct cn_batch* cn_batch_handle;

/* Cut mesh: triangles on the cut vertex index space (seam vertices already
 * duplicated), CCW, and the Dirichlet handle vertices. */
typedef struct {
  int32_t n_verts;
  int32_t n_tris;
  const double* positions; /* n_verts x 3 rest positions */
  const int32_t* tris;     /* n_tris x 3 */
  int32_t n_handles;
  const int32_t* handles;  /* n_handles distinct vertex ids */
} cn_mesh_desc;

/* BSSOR: block SSOR, M = (D + L) D^-1 (D + U) over the rows each block of
 * the row-cached kernel owns (couplings between blocks dropped; L / U in the
 * order of a DSatur colouring inside the block, couplings between rows of one
 * colour dropped on both sides), applied by colour sweeps in shared memory;
 * no counterpart in the reference (its PCG takes Jacobi or IC(0)).  Fewer
 * iterations than Jacobi at the cost of a sweep per iteration. */
enum { CN_PRECOND_JACOBI = 0, CN_PRECOND_IC0 = 1, CN_PRECOND_HSC = 2, CN_PRECOND_BSSOR = 3 };
/* AUTO: COLOR with IC(0) (its levels), NATURAL otherwise (neighbouring
 * vertices stay neighbouring rows, so row gathers coalesce). */
enum { CN_ORDER_NATURAL = 0, CN_ORDER_COLOR = 1, CN_ORDER_AUTO = 2 };
enum { CN_LAPLACIAN_COT = 0, CN_LAPLACIAN_ROBUST = 1 };
enum { CN_PREC_FP64 = 0, CN_PREC_MIXED = 1 };
enum { CN_MODE_HARMONIC = 0, CN_MODE_DEFORM = 1, CN_MODE_RHS = 2 };
/* FUSED: one persistent launch.  With Jacobi: the row-cached kernel (rows
 * of A and each row's CG state in shared memory); in FP64 the pipelined CG
 * (one team barrier per iteration, falling back to the two-reduction form if
 * an inner solve stops reducing the residual), in mixed precision the
 * two-reduction CG (two barriers per iteration; FP32 pipelined recurrences
 * drift on ill-conditioned meshes).  With block SSOR: in mixed precision
 * the pipelined CG keeping u = M^-1 r and q = M^-1 s by recurrence, inner
 * solves of at most 1e-3 restarted by the FP64 refinement, with the same
 * fall-back; in FP64 the two-reduction CG.  With IC(0) and k = 1 or 3 on a
 * multi-block grid below 500,000 free rows, in mixed precision and in FP64
 * from 50,000 rows: the triangular sweeps without grid barriers (every
 * published value carries the number of the preconditioner application it
 * belongs to; block barriers between levels) under the single-reduction CG,
 * one grid barrier per iteration; otherwise (smaller FP64 systems, systems
 * from 500,000 rows, k = 9, one block) the level-scheduled kernel.  With
 * HSC: the level-scheduled kernel.  CLASSIC:
 * the two-reduction CG (row-cached kernel; IC(0): the level-scheduled
 * kernel).  PIPELINED: the pipelined CG without fall-back (Jacobi in both
 * precisions, block SSOR in mixed precision).  PLAIN: one kernel per
 * primitive, FP64 Jacobi.  SINGLE: the single-reduction CG (Chronopoulos
 * & Gear: alpha and beta from one reduction of (r, z), (z, A z), ||r||^2)
 * on the row-cached kernel, Jacobi or block SSOR: one grid barrier per
 * iteration, z exchanged with the neighbour blocks only; on IC(0) handles
 * (k = 1, 3) the sweeps without grid barriers in either precision. */
enum { CN_ALGO_FUSED = 0, CN_ALGO_PLAIN = 1, CN_ALGO_CLASSIC = 2, CN_ALGO_PIPELINED = 3, CN_ALGO_SINGLE = 4 };

typedef struct {
  int32_t precond;       /* CN_PRECOND_* (default IC0) */
  int32_t ordering;      /* CN_ORDER_* row order of A (default AUTO) */
  int32_t laplacian;     /* CN_LAPLACIAN_* (default COT) */
  double mollify_delta;  /* delta of the robust (mollified) Laplacian */
  int32_t device;        /* CUDA device ordinal */
  int32_t max_rhs;       /* largest k a solve will use (1..9), sizes the work vectors */
  int32_t tune;          /* 1: autotune the launch shape for this system (cached) */
  int32_t lanes;         /* 0: default/tuned; else lanes per row (1,2,4,8,16) */
  int32_t block;         /* 0: default/tuned; else threads per block */
  int32_t grid;          /* 0: default/tuned; else blocks of the persistent solve */
  int32_t hsc_tail_rows; /* HSC: levels with at most this many unknowns left run in one block (0 = 1024) */
  double hsc_theta;      /* HSC: fill kept when |S_ij| >= theta sqrt(S_ii S_jj) (0 = 0.01) */
} cn_build_opts;

typedef struct {
  int32_t precision;   /* CN_PREC_FP64 or CN_PREC_MIXED */
  int32_t mode;        /* CN_MODE_HARMONIC, CN_MODE_DEFORM (targets) or CN_MODE_RHS */
  int32_t algo;        /* CN_ALGO_FUSED, _CLASSIC, _PIPELINED, _SINGLE or _PLAIN */
  double tol;          /* relative residual ||b - A x|| / ||b|| per column */
  int32_t max_iter;    /* inner PCG iterations per refinement step */
  int32_t max_refine;  /* FP64 residual refinements (mixed precision) */
  double inner_tol;    /* mixed precision: inner relative tolerance */
  int32_t warm_start;  /* 1: start from this handle's previous solution */
  double wait_limit_ms;  /* bound of every device-side wait of a multi-block solve (its grid
                          * barriers), in ms; a wait that runs out ends the solve with
                          * CN_TIMEOUT and leaves the handle usable (0 = 2000 ms) */
} cn_solve_opts;

typedef struct {
  int32_t status;
  int32_t iterations;    /* inner PCG iterations summed over refinements */
  int32_t refinements;   /* FP64 residual evaluations after the first */
  int32_t k;
  double rel_residual[32]; /* final true relative residual of the first 32 columns */
  double max_rel_residual;
  double device_ms;      /* device time of the solve (CUDA events) */
} cn_solve_stats;

void cn_default_build_opts(cn_build_opts* o);
void cn_default_solve_opts(cn_solve_opts* o);
const char* cn_status_string(int32_t status);
/* Text of the last error on this thread ("" if none). */
const char* cn_last_error(void);

/* Seam cut of an uncut triangle mesh along closed vertex loops.  Each loop
 * vertex gets a copy (ids n_verts, n_verts+1, ... in loop order) and the
 * faces on the left of the loop at that vertex move to the copy.  Host only.
 * Replaces the cut-mesh construction of CutAlgorithm.lean:49-255 /
 * CutMesh.lean:39-79 for profile-curve seams along mesh edges.
 * tris_out: n_tris x 3; parent_out: capacity n_verts + total loop length. */
cn_status cn_cut_mesh(int32_t n_verts, int32_t n_tris, const int32_t* tris, int32_t n_loops,
                      const int32_t* loop_ptr, const int32_t* loop_verts, int32_t* tris_out,
                      int32_t* parent_out, int32_t* n_verts_out);

/* ---------------------------------------------------------------------------
 * Cut-mesh construction on the GPU (current device; host buffers in and
 * out).  Halfedge records are 4 int32 each: target, twin (-1 none), next,
 * face (-1 the outer face).
 *
 * cn_halfedges: HalfedgeBuilder.fromTriangles (HalfedgeBuilder.lean:34-90):
 * interior halfedges 3f, 3f+1, 3f+2 run t0->t1, t1->t2, t2->t0; a twin is the
 * lowest interior index with the reversed (source, target); each interior
 * halfedge without one gets a boundary halfedge, appended in interior index
 * order; a boundary halfedge's next is the lowest boundary index whose
 * source is its target (itself if none).  he_out capacity: 6 n_tris records.
 * Bit-exact with the specification on any triangle soup. */
cn_status cn_halfedges(int32_t n_verts, int32_t n_tris, const int32_t* tris, int32_t* he_out, int32_t* n_he_out);
/* The seam cut of cn_cut_mesh (same arguments and results) computed on the
 * GPU: the halfedges above, then one thread per loop vertex sweeping its fan
 * from the interior halfedge vertex -> next loop vertex by twin(prev(h)) up
 * to the halfedge vertex -> previous loop vertex. */
cn_status cn_cut_mesh_gpu(int32_t n_verts, int32_t n_tris, const int32_t* tris, int32_t n_loops,
                          const int32_t* loop_ptr, const int32_t* loop_verts, int32_t* tris_out,
                          int32_t* parent_out, int32_t* n_verts_out);
/* Batches of the cut surgery (CutAlgorithm.lean:49-100 subdivideEdge,
 * :125-170 splitFace, :225-251 insertCrack) on halfedge records `he`
 * (capacity counts[2] + 2m), counts = {vertices, faces, halfedges} updated in
 * place.  Operation k of a batch takes the new vertex counts[0] + k (or new
 * face counts[1] + k) and the new halfedges counts[2] + 2k, 2k + 1: the result
 * equals the operations applied one after another in batch order.  A batch
 * must touch disjoint records: subdivided halfedges and their twins distinct,
 * split pairs (a, b) in distinct faces, crack anchors distinct (otherwise
 * CN_BAD_INPUT). */
cn_status cn_subdivide_edges(int32_t* counts, int32_t* he, int32_t m, const int32_t* edges);
cn_status cn_split_faces(int32_t* counts, int32_t* he, int32_t m, const int32_t* a, const int32_t* b);
cn_status cn_insert_cracks(int32_t* counts, int32_t* he, int32_t m, const int32_t* anchors);

/* Assemble K = V^T L_h V (CutMeshLaplacian.lean:86-93) into CSR on the GPU,
 * reduce to the free unknowns, order, and factor (IncompleteCholesky.lean:30-33;
 * SlangCodegen/IncompleteCholesky.lean:9-12 for the level/colour schedule). */
cn_status cn_build(const cn_mesh_desc* mesh, const cn_build_opts* opts, cn_handle* out);
void cn_destroy(cn_handle h);

/* Solve for k right-hand sides with host buffers.  targets: n_handles x k
 * (modes HARMONIC/DEFORM) or, for CN_MODE_RHS, the free-row right-hand side
 * n_free x k in vertex order of cn_export_csr's free_of.  x0 (nullable):
 * n_verts x k initial guess.  x_out: n_verts x k with handles overlaid.
 * HARMONIC = HarmonicSolve.lean:51-66 solveMulti; DEFORM = DeformSolve.lean:
 * 123-135 Stage 2 with F_f = I; the PCG follows SparseLinAlg.lean:104-163. */
cn_status cn_solve(cn_handle h, int32_t k, const double* targets, const double* x0,
                   double* x_out, const cn_solve_opts* opts, cn_solve_stats* stats);

/* Same with device buffers, enqueued on the handle's stream.  With stats ==
 * NULL the call does not synchronise. */
cn_status cn_solve_device(cn_handle h, int32_t k, const double* d_targets, double* d_x_out,
                          const cn_solve_opts* opts, cn_solve_stats* stats);

/* The handle's cudaStream_t. */
void* cn_stream(cn_handle h);

/* info[0..11] = n_free, nnz_A, nnz_L(strict), n_levels, nnz_K, n_verts,
 * n_handles, grid, block, lanes, n_colors, device bytes held. */
cn_status cn_system_info(cn_handle h, int64_t* info);

/* Export the reduced matrix A = K[free, free] in solve order (free_of: row ->
 * vertex), the IC(0) factor (rows: strictly-lower entries then the diagonal,
 * the layout of IncompleteCholesky.lean factor3) and K over all vertices. */
cn_status cn_export_csr(cn_handle h, int32_t* free_of, int32_t* rowptr, int32_t* colidx,
                        double* vals);
cn_status cn_export_factor(cn_handle h, int32_t* rowptr, int32_t* colidx, double* vals);
cn_status cn_export_k(cn_handle h, int32_t* rowptr, int32_t* colidx, double* vals);

/* The full DeGoes22 two-stage solve (DeformSolve.lean:110-135): Stage 1
 * solves the 9 entries of the deformation gradient from F_c (n_handles x 9,
 * row-major 3x3 per handle), the Eq.(3) bridge averages them per face and
 * builds y_h = F_f rest, Stage 2 solves the positions from
 * -V^T L_h (C X_c - y_h).  X_c: n_handles x 3; x_out: n_verts x 3 with the
 * handles overlaid.  Needs a build with max_rhs = 9. */
cn_status cn_solve_deformation(cn_handle h, const double* Fc, const double* Xc, double* x_out,
                               const cn_solve_opts* opts, cn_solve_stats* stats);

/* y = A x on the handle's reduced matrix A in solve order (the rows of
 * cn_export_csr), on the handle's stream (cn_stream): the SpMV / SpMM of
 * SparseLinAlg.lean:44-60 with the multi-RHS layout of
 * SlangCodegen/SpmvMulti.lean:78-119.  precision CN_PREC_MIXED: FP32 values
 * and vectors; CN_PREC_FP64: FP64.  k in {1, 3, 9, 24}; d_x, d_y: device
 * pointers, [n_free][k] row-major, 16-byte aligned.  FP32 with k = 1 or 3
 * stages the rows of A through shared memory with bulk asynchronous copies;
 * its waits are bounded, and should one run out (not expected) the rows it
 * could not compute come back NaN. */
cn_status cn_spmv_device(cn_handle h, int32_t k, int32_t precision, const void* d_x, void* d_y);

/* ---------------------------------------------------------------------------
 * Direct Delta Mush.  Bind (DirectDeltaMushBind.lean:6-40): the influence of
 * handle i on every cut-mesh vertex is the harmonic solve with the unit
 * target on handle i (HarmonicSolve.lean:51-66); the weights are smoothed nu
 * times by w' = (1 - omega) w + omega * mean over the vertex's mesh
 * neighbours (:72-94), each vertex keeps the top_k of largest |w| (ties: the
 * lower handle index) and its kept weights are divided by their sum
 * (:104-133).  Output rows of take = min(top_k, n_handles) entries:
 * infl_idx / infl_w are n_verts x take (CSR start of vertex v = v * take).
 * Needs a build with max_rhs = 9; runs n_handles / 9 solves. */
cn_status cn_ddm_bind(cn_handle h, int32_t nu, double omega, int32_t top_k, const cn_solve_opts* opts,
                      int32_t* infl_idx, double* infl_w);
/* Runtime DDM (DirectDeltaMush.lean:84-102 lbsMatvec; the buffers of
 * SlangCodegen/DirectDeltaMush.lean:11-22): out[v] = sum over v's
 * influences of w * (T_i (rest[v], 1)).  Device pointers: rest and out
 * n_verts x 3, transforms n_handles x 16 (row-major 4x4), start n_verts + 1,
 * idx / w per influence; FP32 (CN_PREC_MIXED) or FP64; stream: a
 * cudaStream_t (NULL: the default stream). */
cn_status cn_lbs_matvec_device(int32_t n_verts, int32_t precision, const void* d_rest, const void* d_transforms,
                               const int32_t* d_start, const int32_t* d_idx, const void* d_w, void* d_out,
                               void* stream);

/* Launch shape of the persistent solve: lanes per row (1, 2, 4, 8, 16),
 * threads per block, blocks (1 = one block, __syncthreads barriers; more =
 * cooperative grid, clamped to the co-resident maximum). */
cn_status cn_set_launch(cn_handle h, int32_t lanes, int32_t block, int32_t grid);

/* The launch-shape autotuner: times every candidate shape (lanes per row x
 * threads per block x blocks) on k device right-hand sides with `reps`
 * timed solves each and keeps the fastest median.  results (nullable):
 * 5 doubles per candidate (lanes, block, grid, median ms, iterations);
 * capacity 120 candidates. */
cn_status cn_autotune(cn_handle h, int32_t k, const double* d_targets, const cn_solve_opts* opts,
                      int32_t reps, double* results, int32_t* n_results);

/* Structure of an HSC handle (CN_PRECOND_HSC; hierarchy built from the
 * elimination primitive of HierarchicalSparsifyCompensate.lean:97-125):
 * level count, first level solved by one block, coarse size, the n_levels+1
 * level offsets in HSC positions, and order[p] = row (natural free order,
 * i.e. free vertices by ascending id) at position p. */
cn_status cn_hsc_info(cn_handle h, int32_t* n_levels, int32_t* tail, int32_t* n_coarse,
                      int32_t* level_off, int32_t* order);

/* ---------------------------------------------------------------------------
 * Profile curves and the adjoint.  A curve is a composite cubic Bezier of
 * n_segments segments (3 n_segments + 1 control points, the cubic of
 * EndToEndExample.lean:52-60 per segment).  Handle h is bound at rest to curve
 * curve_of[h] (-1: none) at parameter tau[h] in [0, n_segments]; with per-curve
 * weight w_c its target is rest(h) + w_c (B_posed(tau_h) - B_rest(tau_h)).
 * The reference binds samples to curves by nearest-vertex projection
 * (SurfaceProjection.lean:46-64) and has no per-curve weights; this map is
 * the library's definition. */
cn_status cn_bind_curves(cn_handle h, int32_t n_curves, int32_t n_segments, const double* rest_cp,
                         const int32_t* curve_of, const double* tau);
/* Handle targets from the posed control points (n_curves x (3S+1) x 3) and
 * weights, then the deform solve (CN_MODE_DEFORM, k = 3); x_out: n_verts x 3. */
cn_status cn_deform(cn_handle h, const double* posed_cp, const double* weights, double* x_out,
                    const cn_solve_opts* opts, cn_solve_stats* stats);
/* Vector-Jacobian product of the last cn_deform: given dL/dx (n_verts x 3),
 * solves A lambda = (dL/dx)_free with the same factor (A = A^T), then
 * dL/dX_c(h) = -(K_{h,free} lambda) + dL/dx_h, chained to the control points
 * (dL_dcp, like posed_cp) and the weights (dL_dw, n_curves). */
cn_status cn_adjoint(cn_handle h, const double* dL_dx, double* dL_dcp, double* dL_dw,
                     const cn_solve_opts* opts, cn_solve_stats* stats);

/* ---------------------------------------------------------------------------
 * Curvenet: the curve side of the deformer on the GPU (DeGoes22 section 3 as
 * the reference specifies it in ScaledFrames.lean, SegmentGradient.lean,
 * IntersectionFrames.lean and CurveInterp.lean).  Each curve is a composite
 * cubic Bezier (EndToEndExample.lean:52-60 per segment) sampled at
 * n_samples fixed parameters; consecutive samples bound the polyline
 * segments (a closed curve's last segment joins its last sample to its
 * first).  Per segment and side the constraint gradient is
 *   isolated curve (closed, or no intersection at either end):
 *     F = (l / l_rest) R(t_rest, t)  (ScaledFrames.lean:71-98, both sides);
 *   curve with an intersection at one or both ends:
 *     F^+- = (B S)_posed (B S)_rest^-1  (ScaledFrames.lean:120-170) with the
 *     scaled frame B S = [t l | (n x t) w | n sqrt(l w)]
 *     (IntersectionFrames.lean:160-170), where the per-side normal n and
 *     width w come from the intersection frames of the curve's end segments
 *     (corner normals with the T-junction fallback, per-side widths:
 *     IntersectionFrames.lean:65-143) and are interpolated linearly along
 *     the curve (CurveInterp.lean:45-60), rest and posed separately.
 * The assembly rules are this library's definition (the reference states the
 * pieces): a curve end at an intersection leaves along its end segment (the
 * last segment reversed at the curve's end, where plus and minus swap); with
 * an intersection at one end only, that end's data hold along the whole
 * curve; a handle bound to (curve, sample i, side) takes F of the segment
 * starting at sample i (an open curve's last sample: the last segment) and
 * X_c = the posed curve point at sample i (EndToEndExample.lean:140-142);
 * handles bound to no curve keep F = I and X_c = their rest position.
 * Results equal the FP64 restatement bit for bit (no FMA contraction). */
typedef struct {
  int32_t n_curves;
  int32_t n_segments;          /* cubic segments per curve: 3 n_segments + 1 control points */
  int32_t n_samples;           /* samples per curve (>= 2) */
  const double* rest_cp;       /* n_curves x (3 n_segments + 1) x 3 */
  const double* sample_tau;    /* n_curves x n_samples, strictly rising in [0, n_segments] */
  const int32_t* closed;       /* n_curves (nullable: all open) */
  int32_t n_nodes;             /* intersections */
  const int32_t* node_ptr;     /* n_nodes + 1 */
  const int32_t* node_ends;    /* per intersection, counter-clockwise: 2 curve + (0 start, 1 end); 2..16 ends */
  const int32_t* handle_curve; /* per handle of the mesh: curve, or -1 */
  const int32_t* handle_sample;
  const int32_t* handle_side;  /* 0: plus side, 1: minus side */
} cn_curvenet_desc;

/* Bind a curvenet to the handles of h (copies the tables to the device). */
cn_status cn_bind_curvenet(cn_handle h, const cn_curvenet_desc* net);
/* F_c (n_poses x n_handles x 9, row-major 3x3) and X_c (n_poses x n_handles
 * x 3) from posed control points (n_poses x n_curves x (3S+1) x 3): device
 * pointers, enqueued on the handle's stream (no synchronisation). */
cn_status cn_curvenet_constraints_device(cn_handle h, int32_t n_poses, const double* d_posed_cp, double* d_Fc,
                                         double* d_Xc);
/* The same with host buffers (synchronous). */
cn_status cn_curvenet_constraints(cn_handle h, int32_t n_poses, const double* posed_cp, double* Fc, double* Xc);
/* Curves to positions for one pose: F_c and X_c on the GPU, then the
 * two-stage solve of cn_solve_deformation (DeformSolve.lean:110-135) without
 * leaving the device; x_out: n_verts x 3 with X_c overlaid.  Needs a build
 * with max_rhs = 9. */
cn_status cn_deform_curvenet(cn_handle h, const double* posed_cp, double* x_out, const cn_solve_opts* opts,
                             cn_solve_stats* stats);

/* ---------------------------------------------------------------------------
 * Batched solves: many meshes of uneven size, each with k right-hand sides
 * (k = 24: 8 poses x 3 coordinates, or k = 3), in ONE persistent,
 * CUDA-graph-captured launch.  Each thread-block cluster takes the next mesh
 * (largest first) and solves it with the algorithm of cn_solve; the hardware
 * cluster barrier synchronises the cluster.  The runtime's per-frame loop
 * over bound meshes and poses (HarmonicSolve.lean:51-66 per mesh;
 * SlangCodegen/SpmvMulti.lean:8-14 for the multi-RHS layout) becomes one
 * launch.  Targets are concatenated mesh by mesh (n_handles_m x k each),
 * positions likewise (n_verts_m x k each); cn_batch_offsets gives the
 * offsets. */
typedef struct {
  int32_t status;            /* worst mesh status */
  int32_t n_meshes;
  int32_t n_failed;          /* meshes not at CN_OK */
  int32_t max_iterations;    /* largest inner-iteration count of one mesh */
  int64_t total_iterations;
  double max_rel_residual;   /* over all meshes and columns */
  double device_ms;          /* device time of the launch (CUDA events) */
} cn_batch_stats;

/* cluster_size: blocks per cluster (0 = 4; up to 16); n_clusters: clusters of
 * the persistent grid (0 = all co-resident).  opts->block: threads per block
 * (0 = 512). */
cn_status cn_build_batch(const cn_mesh_desc* meshes, int32_t n_meshes, const cn_build_opts* opts,
                         int32_t k, int32_t cluster_size, int32_t n_clusters, cn_batch_handle* out);
void cn_destroy_batch(cn_batch_handle b);
cn_status cn_solve_batch(cn_batch_handle b, const double* targets, double* x_out,
                         const cn_solve_opts* opts, cn_batch_stats* stats);
/* Device buffers, enqueued on the batch's stream as one graph launch; with
 * stats == NULL the call does not synchronise. */
cn_status cn_solve_batch_device(cn_batch_handle b, const double* d_targets, double* d_x_out,
                                const cn_solve_opts* opts, cn_batch_stats* stats);
void* cn_batch_stream(cn_batch_handle b);
/* info[0..11] = n_meshes, k, total vertices, total handles, total free rows,
 * total nnz(A), total nnz(L strict), cluster size, clusters, block, max free
 * rows of one mesh, device bytes held. */
cn_status cn_batch_info(cn_batch_handle b, int64_t* info);
/* n_meshes + 1 offsets (in doubles) of each mesh's targets and positions. */
cn_status cn_batch_offsets(cn_batch_handle b, int64_t* tgt_off, int64_t* out_off);
/* Rows per warp of the batched launch, per size class of mesh: a mesh with
 * n free rows takes lanes[c] lanes per row for the first class c with
 * n <= class_max_rows[c] (the last class takes the rest); with k = 24 a lane
 * owns 24 / lanes columns, lanes 8 (4 rows per warp) or 4 (8 rows per warp);
 * k = 3 takes 1.  Chosen per size class by the autotuner
 * (tool_godot_curvenet_b200/tune.py); default 8.  The multi-RHS thread
 * mapping of SlangCodegen/SpmvMulti.lean:12-14 per mesh, in one launch. */
cn_status cn_batch_set_lanes(cn_batch_handle b, int32_t n_classes, const int32_t* class_max_rows,
                             const int32_t* lanes);
/* Lanes per row of each mesh (n_meshes entries). */
cn_status cn_batch_lanes(cn_batch_handle b, int32_t* lanes);
/* Per-mesh results of the last solve with stats (each array nullable,
 * n_meshes entries): status, inner iterations, largest relative residual
 * over the mesh's columns, FP64 residual evaluations after the first. */
cn_status cn_batch_mesh_stats(cn_batch_handle b, int32_t* status, int32_t* iterations,
                              double* max_rel_residual, int32_t* refinements);

/* FP64 Jacobi-preconditioned CG on a caller-owned device CSR matrix
 * (n rows, sorted columns, FP64 values) for k = 1, 3 or 9 right-hand sides,
 * that allocates no GPU memory.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc while they run: a real-time frame
 * loop with a fixed memory budget (an engine that pre-allocates at start-up
 * and forbids allocation per frame), code that records work into a CUDA
 * stream, or a host that owns all device memory itself.  The caller passes
 * the matrix (d_rowptr n+1, d_colidx, d_vals), the right-hand sides d_b
 * (n x k, row-major) and the solution d_x (n x k: initial guess in, solution
 * out); every temporary lives in one fixed device array inside the library
 * (about 14 MB per GPU, kept until the process exits).  The matrix is
 * trusted, not checked: row pointers non-decreasing from 0, every column
 * index in [0, n), columns sorted within a row, the matrix symmetric
 * positive definite.
 *
 * Limits: n <= 65,536 and n * k <= 196,608; larger systems return
 * CN_BAD_INPUT with the reason in cn_last_error().  The stopping test is the
 * relative residual ||b - A x|| <= tol ||b|| per column.  max_iter bounds the
 * CG iterations of one pass; after a pass the FP64 residual is recomputed
 * from b - A x and CG restarts from it, at most 4 passes, so a call runs at
 * most 4 * max_iter iterations.  A grid barrier that waits more than 2 s
 * ends the call with CN_TIMEOUT.
 *
 * The work is enqueued on `stream` (a cudaStream_t; NULL = the default
 * stream) of the current device.  With stats != NULL the call reads the
 * statistics back and synchronises the stream, and returns the solve's
 * status.  With stats == NULL it does neither and CN_OK only means the work
 * was enqueued; this is the form to use while a stream is being captured
 * (reading back and synchronising are not allowed during a capture).  The
 * results of the last call stay in the scratch: after synchronising, read
 * them with cn_pcg_csr_noalloc_last_stats.
 *
 * Every call shares the same scratch array, so calls that overlap on the GPU
 * (two streams or two threads at once) race and must be serialised by the
 * caller.  Each call looks up the array's device address on the current
 * device; the first lookup on a device loads the library's device code, so
 * make the first call on each device before any stream capture. */
cn_status cn_pcg_csr_noalloc(int32_t n, const int32_t* d_rowptr, const int32_t* d_colidx,
                             const double* d_vals, int32_t k, const double* d_b, double* d_x,
                             double tol, int32_t max_iter, void* stream, cn_solve_stats* stats);
/* Statistics of the last cn_pcg_csr_noalloc call on the current device
 * (status, iterations, FP64 residual passes after the first, k, per-column
 * relative residuals), read from the scratch with a blocking copy; call it
 * after synchronising the stream of that call.  Returns that call's status.
 * No counterpart in the reference. */
cn_status cn_pcg_csr_noalloc_last_stats(cn_solve_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* CURVENET_B200_H */
