// cn_internal.h -- shared between the host orchestration (cn_host.cpp) and the
// sm_100a kernels (cn_*.cu).  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/curvenet_b200.h"

namespace cn {

// Persistent-solve control block (reset by the host before every launch).
struct Control {
  unsigned bar_count;
  unsigned bar_gen;
  int abort;
  int status;
};

// Device-side statistics written by the persistent solve.
struct DevStats {
  int status;
  int iterations;
  int refinements;
  int pad;
  double rel_residual[32];
};

// Everything the persistent PCG kernel reads.  Arrays are device pointers;
// vectors are row-interleaved [rows][K].  T-typed arrays are passed as void*
// and cast inside the kernel (float for mixed precision, double for FP64).
struct SolveArgs {
  int n;        // free unknowns (rows of A)
  int nlev;     // level sets of the triangular solves
  const int* lev_ptr;
  // reduced matrix A in solve order
  const int* A_ptr;
  const int* A_col;
  const void* A_val;       // T
  const double* A_val64;
  // IC(0): strictly-lower L and its transpose U, and 1/L_ii
  const int* L_ptr;
  const int* L_col;
  const void* L_val;       // T
  const int* U_ptr;
  const int* U_col;
  const void* U_val;       // T
  const void* dinv;        // T
  // right-hand side assembly and output over all vertices
  int nv;
  int nh;
  const int* K_ptr;
  const int* K_col;
  const double* K_val;
  const int* free_of;      // row -> vertex
  const int* hidx;         // vertex -> handle index or -1
  const int* handles;      // handle -> vertex
  const double* pos;       // rest positions (deform mode)
  int mode;                // CN_MODE_*
  const double* targets;   // nh x K (or n x K for CN_MODE_RHS, solve order)
  double* x_out;           // nv x K (nullable)
  const double* x0;        // nv x K initial guess (nullable)
  int warm;                // keep x64 from the previous solve
  // vectors
  double* b64;
  double* x64;
  void* r;    // T
  void* y;    // T
  void* z;    // T
  void* p0;   // T
  void* p1;   // T
  void* Ap;   // T
  void* xin;  // T
  // pipelined Jacobi-PCG (cn_pipe.cu): the ping-pong copies of m = M^-1 w
  // that neighbouring rows gather ([rows][round_up(K, 16 B)])
  void* m0;   // T
  void* m1;   // T
  void* m2;   // T (the classic form's first records [z | p])
  int pipe_mode;           // 0 two-reduction, 1 pipelined, 2 pipelined with fall-back, 3 single-reduction
  unsigned* nbflag;        // single-reduction form: one z-publication count per block (zeroed per launch)
  double* pown;            // FP64 own-row state when it is not in shared memory: 7 x [rows][K]
  const double* dinv64;    // 1 / sqrt(A_ii), FP64
  int cache_bytes;         // dynamic shared memory (row cache, then own-row state)
  const unsigned char* bcolor;  // block SSOR: block-local colour of every row (null: Jacobi)
  int bncolor;                  // colours
  // block SSOR tables in global memory, for the blocks whose shared memory
  // cannot hold them (provided with every block-SSOR launch): list position
  // per row, the sweep vector (32 bytes a row), the neighbour lists (16 bytes
  // an entry) and each block's first entry in them
  int* bss_pos;
  void* bss_v;
  void* bss_lent;
  const long long* bss_loff;
  double* partials;        // [kSlots][grid][K]
  // HSC preconditioner (hsc != 0): rows are in HSC order; F_l = positions
  // [hsc_off[l], hsc_off[l + 1]); the coarse set starts at hsc_off[hsc_L];
  // levels >= hsc_tail (and the coarse solve) run in block 0 alone.
  int hsc, hsc_L, hsc_tail, hsc_nc;
  const int* hsc_off;
  const int* hsc_rlev;   // hsc_L + 1: R rows of level l
  const int* hsc_rrow;   // R row -> position of the C row
  const int* hsc_rptr;
  const int* hsc_rcol;
  const void* hsc_rval;  // T
  const int* hsc_pptr;   // over F positions [0, hsc_off[hsc_L])
  const int* hsc_pcol;
  const void* hsc_pval;  // T
  const void* hsc_dinv;  // T, over F positions
  const void* hsc_sinv;  // T, hsc_nc x hsc_nc
  // control
  double tol;
  double inner_tol;
  int max_iter;
  int max_refine;
  Control* ctl;
  DevStats* stats;
  long long timeout_ns;
};

constexpr int kSlots = 8;
// Row slices per thread that the pipelined solve's shared-memory row cache holds.
constexpr int kPipeSlices = 16;

// Sets the text cn_last_error() returns on this thread (cn_host.cpp).
void set_last_error_text(const char* msg);

// Launch the persistent solve; returns a cudaError_t.  precision: CN_PREC_*.
cudaError_t launch_persistent_solve(const SolveArgs& a, int precision, int K, int lanes,
                                    int block, int grid, cudaStream_t s);
// Largest co-resident grid of the persistent solve for this configuration.
int persistent_max_grid(int precision, int K, int lanes, int block);

// The IC(0) solve with synchronisation-free sweeps (cn_icsf.cu): tagged
// words of the forward and backward sweeps in a.m0 and a.m1 (FP32:
// round_up(K, 2) 64-bit words a row, FP64: 2K); precision CN_PREC_MIXED
// (FP32 inner solve) or CN_PREC_FP64; K = 1 or 3; at most icsf_max_levels()
// levels; a cooperative launch of `grid` blocks of `block` threads (block <= 512).
cudaError_t launch_icsf_solve(const SolveArgs& a, int precision, int K, int block, int grid, cudaStream_t s);
int icsf_max_grid(int precision, int K, int block);
int icsf_max_levels();

// dst[r * kd + d0 + c] = src[r * ks + s0 + c] for r < rows, c < ncols (cn_ddm.cu).
cudaError_t launch_copy_columns(const double* src, int rows, int ks, int s0, double* dst, int kd, int d0, int ncols,
                                cudaStream_t s);

// Direct Delta Mush (cn_ddm.cu).
cudaError_t launch_ddm_unit_targets(int nh, int c0, int kc, double* t, cudaStream_t s);
cudaError_t launch_ddm_smooth(int nv, const int* ptr, const int* col, const double* in, double* out, double omega,
                              cudaStream_t s);
cudaError_t launch_ddm_topk(int nv, int c0, int kc, int K, const double* W, int* bidx, double* bw, int* cnt,
                            cudaStream_t s);
cudaError_t launch_ddm_finish(int nv, int take, double* bw, cudaStream_t s);
cudaError_t launch_lbs_matvec(int nv, int precision, const void* rest, const void* tr, const int* start,
                              const int* idx, const void* w, void* out, cudaStream_t s);

// y = A x on a CSR matrix (cn_spmv.cu); k in {1, 3, 9, 24}, x and y
// [n][k] in T = float (CN_PREC_MIXED) or double, 16-byte aligned.  FP32 with
// k = 1 or 3 stages the CSR through shared memory with bulk copies: ptr, col
// and val then need 4 elements to spare past their ends, tile_ents is
// spmm_tile_entries of the host row pointers and err a device int raised if
// a bounded wait of that kernel runs out (tile_ents < 0 or err == null: the
// grid-stride kernel).
cudaError_t launch_spmm(int n, int k, int precision, const int* ptr, const int* col, const void* val,
                        const void* x, void* y, int tile_ents, int* err, cudaStream_t s);
int spmm_tile_entries(const int* hptr, int n);

// The row-cached Jacobi-PCG persistent solve (cn_pipe.cu).  a.cache_bytes of
// dynamic shared memory hold each block's rows of A and their CG state.
// qr: rows per thread gathered together (1: up to 1024 threads per block,
// 2: up to 512).  a.pipe_mode: 0 the classic two-reduction form (two
// barriers per iteration), 1 the pipelined form, 2 the pipelined form with a
// fall-back to the classic one when an inner solve stops reducing the FP64
// residual, 3 the single-reduction form, 4 the pipelined form with block
// SSOR (u = M^-1 r and q = M^-1 s kept by recurrence, FP32 only) with the
// same fall-back as 2, 5 the same without the fall-back; each form runs in a
// kernel compiled for it alone (pipe_mode is also needed by
// pipelined_max_grid).
cudaError_t launch_pipelined_solve(const SolveArgs& a, int precision, int K, int block, int grid, int qr,
                                   cudaStream_t s);
int pipelined_max_grid(int precision, int K, int block, int cache_bytes, int qr, int pipe_mode);
// Shared memory of the row-cached solve for this launch shape (the largest
// block's share), given A's pattern: *cache = the row cache alone, *full =
// the row cache and the own-row state of rec_vectors K + 1 values a row
// (and, for block SSOR, the colour lists); SIZE_MAX when a block holds more
// than kPipeSlices row slices.
void pipelined_smem_need(const int* A_ptr, const int* A_col, int n, int grid, int block, int precision, int K,
                         bool bssor, int rec_vectors, size_t* cache, size_t* full);
// Greedy colouring of the rows inside each block of rb consecutive rows, in
// row order, over the couplings inside the block (at most 64 colours);
// returns the number of colours.
int block_colours(const int* A_ptr, const int* A_col, int n, int rb, unsigned char* col);
// Entries of the block-SSOR lists of the block of rows [blk0, blk0 + rb_n)
// (per colour: rows x (widest lower + widest upper in-block neighbour count)).
long long block_list_entries(const int* A_ptr, const int* A_col, const unsigned char* col, long long blk0,
                             long long rb_n);

// Build-time kernels (cn_assemble.cu).
struct BuildArgs {
  int nv, nt, nnzK, n, nnzA, nnzL, nlev;
  const double* pos;
  const int* tris;
  int lap_kind;
  double delta;
  double* face_m;           // nt x 6
  const int* K_cptr;        // nnzK + 1
  const int* K_contrib;     // face*6 + slot, ascending face per entry
  double* K_val;
  const int* A_src;         // nnzA -> K entry
  double* A_val64;
  float* A_val32;
  const int* A_diag;        // n -> A entry of the diagonal
  const int* lev_ptr;
  const int* h_lev_ptr;     // host copy of lev_ptr (launch bounds)
  const int* L_ptr;         // strictly lower, n + 1
  const int* L_src;         // nnzL -> A entry
  const int* L_col;
  const int* T_ptr;         // nnzL + 1 task pointers
  const int* T_a;           // L entry of L_ik
  const int* T_b;           // L entry of L_jk
  double* L_val64;
  float* L_val32;
  double* Ld64;             // n
  double* dinv64;
  float* dinv32;
  const int* U_src;         // nnzL -> L entry
  double* U_val64;
  float* U_val32;
  int* status;              // -1 ok, else first failing row
  double shift;             // diagonal shift factor (Manteuffel): A_ii * (1 + shift)
  int precond;
};
cudaError_t launch_assemble(const BuildArgs& b, cudaStream_t s);
cudaError_t launch_factor(const BuildArgs& b, cudaStream_t s);

// Profile-curve binding of the handles (cn_adjoint.cu).
struct CurveArgs {
  int nh, ncurves, nseg;
  const int* handles;     // handle -> vertex
  const int* curve_of;    // handle -> curve or -1
  const double* tau;      // handle -> curve parameter in [0, nseg]
  const double* rest_cp;  // ncurves x (3 nseg + 1) x 3
  const double* posed_cp;
  const double* weights;  // ncurves
  const double* pos;      // rest positions
};
cudaError_t launch_curve_targets(const CurveArgs& c, double* targets, cudaStream_t s);
cudaError_t launch_adjoint_rhs(int n, const int* free_of, const double* dLdx, double* b, cudaStream_t s);
cudaError_t launch_adjoint_grad(const CurveArgs& c, const int* K_ptr, const int* K_col, const double* K_val,
                                const int* row_of, const double* lambda, const double* dLdx, double* dP,
                                double* dw, cudaStream_t s);

// The Stage 1 -> Stage 2 bridge of the DeGoes22 solve (cn_deform.cu).
struct DeformArgs {
  int nt, n;
  const int* tris;
  const double* pos;
  const double* face_m;   // nt x 6 (the face's 3x3 in faceLoop order)
  const int* hidx;
  const double* Fv;       // nv x 9 (Stage 1, handles overlaid with F_c)
  const double* Xc;       // nh x 3
  const int* free_of;
  const int* vf_ptr;      // vertex -> incident faces, ascending
  const int* vf_face;
  const int* vf_corner;
  double* contrib;        // 3 nt x 3
  double* b;              // n x 3 Stage-2 right-hand side (solve order)
};
cudaError_t launch_deform_bridge(const DeformArgs& d, cudaStream_t s);

// Profile curves on the GPU (cn_curvenet.cu): samples, segment tangents and
// lengths, intersection frames, per-handle F_c and X_c for many poses.
constexpr int kCnetMaxNodeDegree = 16;
struct CurvenetArgs {
  int n_curves, n_segments, n_samples;
  const double* rest_cp;     // n_curves x (3 n_segments + 1) x 3
  const double* sample_tau;  // n_curves x n_samples
  const int* seg_off;        // n_curves + 1: first polyline segment of each curve
  int total_segs;
  const int* curve_kind;     // 0 isolated, bit 0: start at a node, bit 1: end at a node
  int n_nodes;
  const int* node_ptr;       // n_nodes + 1
  const int* node_ends;      // 2 curve + end, counter-clockwise per node
  int nh;
  const int* h_curve;        // per handle: curve (-1: rest, F = I)
  const int* h_sample;
  const int* h_side;         // 0 plus, 1 minus
  const int* handles;        // handle -> vertex
  const double* pos;         // rest positions, n_verts x 3
  double* seg;               // scratch: poses x total_segs x 8
  double* ends;              // scratch: poses x n_curves x 2 x 16
};
cudaError_t launch_curvenet_constraints(const CurvenetArgs& a, int n_poses, const double* posed_cp, double* Fc,
                                        double* Xc, cudaStream_t s);
cudaError_t launch_curvenet_overlay(int nh, const int* handles, const double* Xc, double* x, cudaStream_t s);

// Plain FP64 Jacobi-PCG with one kernel per primitive and the scalars folded
// on the host each iteration (the reference's GPU orchestration).
struct PlainArgs {
  int n, K;
  const int* A_ptr;
  const int* A_col;
  const double* A_val;
  const int* A_diag;
  double *b, *x, *r, *z, *p, *Ap;
  double* partials;  // [blocks][K]
  int blocks;
};
cudaError_t plain_spmv(const PlainArgs& a, const double* x, double* y, cudaStream_t s);
cudaError_t plain_dot(const PlainArgs& a, const double* u, const double* v, cudaStream_t s);
cudaError_t plain_axpy2(const PlainArgs& a, const double* alpha, cudaStream_t s);
cudaError_t plain_jacobi(const PlainArgs& a, cudaStream_t s);
cudaError_t plain_saxpby(const PlainArgs& a, const double* beta, cudaStream_t s);
cudaError_t plain_rhs_and_init(const SolveArgs& sa, const PlainArgs& a, cudaStream_t s);
cudaError_t plain_residual(const PlainArgs& a, cudaStream_t s);
cudaError_t plain_output(const SolveArgs& sa, const PlainArgs& a, cudaStream_t s);
cudaError_t plain_set_scalars(double* d_dst, const double* h_src, int K, cudaStream_t s);

}  // namespace cn
