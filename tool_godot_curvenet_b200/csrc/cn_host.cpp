// cn_host.cpp -- the single-mesh handle of the C ABI: build (host structure,
// one device allocation, GPU assembly + IC(0)), solve dispatch (persistent
// fused solve or the plain per-primitive baseline), and the exports.  All
// floating-point work runs on the GPU; the host builds integer structure only.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <map>
#include <tuple>
#include <vector>

#include "cn_hsc.h"
#include "cn_mesh.h"

using cn::Control;
using cn::DevStats;
using cn::MeshDev;
using cn::MeshHost;
using cn::SolveArgs;
using cn::set_err;

#define CN_CUDA(call)                                                          \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      set_err("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                       \
      return CN_CUDA_ERROR;                                                    \
    }                                                                          \
  } while (0)

struct cn_system {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cn_build_opts opts{};
  MeshHost H;
  MeshDev D;
  int kmax = 3;
  int lanes = 2, block = 512, grid = 0;
  double shift_used = 0.0;
  char* buf = nullptr;   // the one device allocation
  size_t bytes = 0;
  // solve state (inside buf)
  double *d_b64 = nullptr, *d_x64 = nullptr, *d_partials = nullptr;
  double* d_w64[7] = {};
  float* d_w32[7] = {};
  Control* d_ctl = nullptr;
  DevStats* d_stats = nullptr;
  double *d_targets = nullptr, *d_xout = nullptr, *d_scal = nullptr;
  double *d_pown = nullptr, *d_m[3] = {};   // row-cached solve: own-row state, gather buffers
  double *d_split_t = nullptr, *d_split_x = nullptr;  // k = 9 as three k = 3 solves
  // block SSOR: block-local colours of the rows for blocks of bcolor_rb rows (own allocation)
  unsigned char* d_bcolor = nullptr;
  int bcolor_rb = -1, bncolor = 0;
  std::vector<unsigned char> h_bcolor;
  // block SSOR tables in global memory (own allocations): list positions,
  // sweep vector, lists and each block's first entry, for (bss_rb, bss_grid)
  int* d_bss_pos = nullptr;
  void* d_bss_v = nullptr;
  void* d_bss_lent = nullptr;
  long long* d_bss_loff = nullptr;
  long long bss_lent_cap = 0;
  int bss_loff_cap = 0, bss_rb = -1, bss_grid = -1;
  int* d_status = nullptr;
  unsigned* d_nbflag = nullptr;  // single-reduction form: per-block publication counts (inside buf)
  int* d_spmv_err = nullptr;     // raised by the staged SpMV if one of its bounded waits runs out (inside buf)
  int spmv_ents = -1;            // most entries of A in one SpMV tile (computed on first use)
  // pipelined solve: shared-memory needs of the last (grid, block, precision, k)
  // shared memory of the row-cached solve per launch shape (grid, block,
  // precision, k, record vectors) -> (row cache, full state): the sizing
  // colours the blocks on the host, so it is kept for every shape a handle
  // has launched
  std::map<std::tuple<int, int, int, int, int>, std::pair<size_t, size_t>> pipe_smem;
  int max_grid_alloc = 0;
  bool shape_set = false;   // cn_set_launch fixed the launch shape
  bool have_solution = false;
  // HSC preconditioner tables (own allocations)
  bool hsc = false;
  int hsc_L = 0, hsc_tail = 0, hsc_nc = 0;
  std::vector<int> hsc_order, hsc_off_h;
  std::vector<void*> hsc_mem;
  int *d_hoff = nullptr, *d_hrlev = nullptr, *d_hrrow = nullptr, *d_hrptr = nullptr, *d_hrcol = nullptr,
      *d_hpptr = nullptr, *d_hpcol = nullptr;
  double *d_hrval64 = nullptr, *d_hpval64 = nullptr, *d_hdinv64 = nullptr, *d_hsinv64 = nullptr;
  float *d_hrval32 = nullptr, *d_hpval32 = nullptr, *d_hdinv32 = nullptr, *d_hsinv32 = nullptr;
  // two-stage deform (cn_solve_deformation), own allocations
  int *d_vf_ptr = nullptr, *d_vf_face = nullptr, *d_vf_corner = nullptr;
  double *d_contrib = nullptr, *d_Xc = nullptr;
  // profile-curve binding (cn_bind_curves), own allocations
  int ncurves = 0, nseg = 0;
  bool have_forward = false;
  int *d_curve_of = nullptr, *d_row_of = nullptr;
  double *d_tau = nullptr, *d_rest_cp = nullptr, *d_posed_cp = nullptr, *d_weights = nullptr;
  double *d_dLdx = nullptr, *d_dP = nullptr, *d_dw = nullptr;
  // profile curvenet (cn_bind_curvenet): bound tables, per-pose scratch and
  // the host-call staging buffers, own allocations
  bool have_cnet = false;
  cn::CurvenetArgs cnet{};
  std::vector<void*> cnet_mem;
  int cnet_pose_cap = 0;
  double *d_cnet_posed = nullptr, *d_cnet_F = nullptr, *d_cnet_X = nullptr;
};

namespace {

// Jacobi and block SSOR run on the row-cached kernel
bool row_cached(const cn_system* S) {
  return !S->hsc && (S->opts.precond == CN_PRECOND_JACOBI || S->opts.precond == CN_PRECOND_BSSOR);
}

// The IC(0) solve without grid barriers in the sweeps (cn_icsf.cu) is used
// for IC(0) solves of k = 1 or 3 columns unless CLASSIC asks for the
// level-scheduled kernel: in mixed precision below 500,000 free rows, in
// FP64 from 50,000 to 500,000, and whenever SINGLE asks for it.  Measured on
// B200: the FP64 form (two words a value) beat the level-scheduled kernel on
// the 130k-row torus by 9 % and lost by 3-12 % on 5k-18k-row meshes; on the
// 1.05M-row torus the level-scheduled kernel with 1,024-thread blocks beat
// both forms (mixed 30.2 ms against 46.1 ms, FP64 46.7 against 64 ms).
// k = 9 stays on the level-scheduled kernel in one launch: both are bound by
// latency, and three k = 3 solves would take about three times one.
constexpr int kLargeRows = 500000;

bool icsf_wanted(const cn_system* S, int k, const cn_solve_opts& o) {
  if (S->hsc || S->opts.precond != CN_PRECOND_IC0 || (k != 1 && k != 3) || o.algo == CN_ALGO_CLASSIC ||
      o.algo == CN_ALGO_PLAIN || S->H.nlev > cn::icsf_max_levels())
    return false;
  if (o.algo == CN_ALGO_SINGLE) return true;
  const int n = S->H.n;
  return n < kLargeRows && (o.precision == CN_PREC_MIXED || n >= 50000);
}

// Launch shape of a level-scheduled or IC(0) solve: the handle's where the
// caller fixed it (build options, cn_set_launch, the tuner) or for a system
// of fewer than 1,024 rows (one block); otherwise sized by the system and
// the kernel, from measurements on B200 across 2k-1M-row tori and cylinders
// (one block took 1.3-5x longer than these grids from 2k rows on):
// * the IC(0) sweeps without grid barriers: about 600 rows a block (below
//   300,000 rows at most 7/8 of the SMs: fewer blocks keep more of a
//   level's rows in each), 256 threads a block below 20,000 rows, else 512;
// * the level-scheduled kernel, IC(0): about 120 rows a block, the same block
//   sizes, the handle's lanes per row; from 500,000 rows every SM with
//   1,024-thread blocks, one lane per row in mixed precision (two in FP64);
// * HSC: one lane per row (the V-cycle's R and P rows are short), 1,024-thread
//   blocks from 500,000 rows.
void solve_shape(const cn_system* S, int k, const cn_solve_opts& o, int* grid, int* block, int* lanes) {
  *grid = S->grid;
  *block = S->block;
  *lanes = S->lanes;
  if (S->shape_set || S->opts.grid > 0 || S->opts.block > 0 || S->H.n < 1024) return;
  const int n = S->H.n;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->device);
  if (S->hsc) {
    if (S->opts.lanes <= 0) *lanes = 1;
    if (n >= kLargeRows) *block = 1024;
    return;
  }
  if (S->opts.precond != CN_PRECOND_IC0) return;
  if (icsf_wanted(S, k, o)) {
    const int cap = n < 300000 ? std::max(8, sms * 7 / 8) : sms;
    *grid = std::min(cap, std::max(8, n / 600));
    *block = n >= 20000 ? 512 : 256;
  } else if (n >= kLargeRows) {
    *grid = sms;
    *block = 1024;
    if (S->opts.lanes <= 0) *lanes = o.precision == CN_PREC_MIXED ? 1 : 2;
  } else {
    *grid = std::min(sms, std::max(8, n / 120));
    *block = n >= 20000 ? 512 : 256;
  }
}

// ... on a multi-block grid
bool icsf_path(const cn_system* S, int k, const cn_solve_opts& o) {
  int grid = 0, block = 0, lanes = 0;
  solve_shape(S, k, o, &grid, &block, &lanes);
  return icsf_wanted(S, k, o) && grid > 1;
}

const char* kStatusText[] = {"ok", "max_iter", "singular_component", "nonpositive_pivot",
                             "nan", "breakdown", "timeout", "bad_input", "cuda_error",
                             "no_device"};

// Lay out the mesh tables and the solve state in one buffer.
void layout_all(cn::Bump& b, cn_system* S) {
  cn::layout(b, S->H, S->D);
  const size_t nk = (size_t)std::max(S->H.n, 1) * S->kmax;
  S->d_b64 = b.take<double>(nk);
  S->d_x64 = b.take<double>(nk);
  for (int i = 0; i < 7; ++i) {
    S->d_w64[i] = b.take<double>(nk);
    S->d_w32[i] = b.take<float>(nk);
  }
  S->d_pown = b.take<double>(7 * nk);
  if (S->kmax >= 9) {
    S->d_split_t = b.take<double>((size_t)std::max(S->H.nh, S->H.n) * 3 + 1);
    S->d_split_x = b.take<double>((size_t)S->H.nv * 3 + 1);
  }
  for (int i = 0; i < 3; ++i) S->d_m[i] = b.take<double>((size_t)std::max(S->H.n, 1) * (2 * S->kmax + 2));
  S->d_partials = b.take<double>((size_t)cn::kSlots * S->max_grid_alloc * S->kmax);
  S->d_scal = b.take<double>(64);
  S->d_ctl = b.take<Control>(1);
  S->d_stats = b.take<DevStats>(1);
  S->d_targets = b.take<double>((size_t)std::max(S->H.nh, S->H.n) * S->kmax + 1);
  S->d_xout = b.take<double>((size_t)S->H.nv * S->kmax + 1);
  S->d_status = b.take<int>(1);
  S->d_nbflag = b.take<unsigned>((size_t)S->max_grid_alloc);
  S->d_spmv_err = b.take<int>(1);
}

void choose_launch(cn_system* S) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->device);
  S->lanes = S->opts.lanes > 0 ? S->opts.lanes : 2;
  if (S->H.n <= 12288) {
    S->block = S->opts.block > 0 ? S->opts.block : 1024;
    S->grid = S->opts.grid > 0 ? S->opts.grid : 1;
  } else {
    S->block = S->opts.block > 0 ? S->opts.block : 512;
    S->grid = S->opts.grid > 0 ? S->opts.grid : sms;
  }
}

// Host -> device uploads go on the handle's stream: the stream is
// non-blocking, and a synchronous cudaMemcpy from pageable memory may return
// before its DMA lands, so a kernel on the handle's stream could otherwise
// read the destination before it holds the data.
template <class Tp>
cn_status up_new(cn_system* S, Tp** dst, const std::vector<Tp>& h) {
  const size_t bytes = sizeof(Tp) * std::max<size_t>(h.size(), 1);
  if (cudaMalloc((void**)dst, bytes) != cudaSuccess) {
    set_err("device allocation of %zu bytes failed", bytes);
    return CN_CUDA_ERROR;
  }
  S->hsc_mem.push_back(*dst);
  if (!h.empty() && cudaMemcpyAsync(*dst, h.data(), sizeof(Tp) * h.size(), cudaMemcpyHostToDevice, S->stream) != cudaSuccess) {
    set_err("upload failed");
    return CN_CUDA_ERROR;
  }
  return CN_OK;
}

std::vector<float> to_f32(const std::vector<double>& v) { return std::vector<float>(v.begin(), v.end()); }

// HSC: read A back, build the hierarchy on the host, move the rows into HSC
// order, reassemble A in that order and upload the level tables.
cn_status setup_hsc(cn_system* S, const cn_build_opts& ob) {
  MeshHost& H = S->H;
  std::vector<double> A(H.nnzA);
  if (H.nnzA && cudaMemcpy(A.data(), S->D.A64, sizeof(double) * H.nnzA, cudaMemcpyDeviceToHost) != cudaSuccess) {
    set_err("read-back of A failed");
    return CN_CUDA_ERROR;
  }
  cn::HscHost h;
  cn::HscParams prm;
  if (S->opts.hsc_theta > 0.0) prm.theta = S->opts.hsc_theta;
  cn_status st = cn::hsc_build(H.n, H.A_ptr.data(), H.A_col.data(), A.data(), prm, h);
  if (st != CN_OK) {
    set_err("HSC coarse matrix is not positive definite");
    return st;
  }
  cn::permute_solve_order(H, h.order);
  st = cn::upload(H, S->D, S->stream);
  if (st != CN_OK) return st;
  st = cn::assemble_factor(H, S->D, ob, S->d_status, S->stream, nullptr);
  if (st != CN_OK) return st;
  const int L = (int)h.levels.size();
  S->hsc_L = L;
  S->hsc_nc = h.nc;
  S->hsc_order = h.order;
  std::vector<int> off(L + 1), rlev(L + 1, 0), rrow, rptr(1, 0), rcol, pptr(1, 0), pcol;
  std::vector<double> rval, pval, dinv;
  for (int l = 0; l < L; ++l) {
    const auto& V = h.levels[l];
    off[l] = V.off;
    for (size_t k = 0; k < V.R_rows.size(); ++k) {
      rrow.push_back(V.R_rows[k]);
      for (int e = V.R_ptr[k]; e < V.R_ptr[k + 1]; ++e) {
        rcol.push_back(V.R_col[e]);
        rval.push_back(V.R_val[e]);
      }
      rptr.push_back((int)rcol.size());
    }
    rlev[l + 1] = (int)rrow.size();
    for (int k = 0; k < V.nf; ++k) {
      for (int e = V.P_ptr[k]; e < V.P_ptr[k + 1]; ++e) {
        pcol.push_back(V.P_col[e]);
        pval.push_back(V.P_val[e]);
      }
      pptr.push_back((int)pcol.size());
      dinv.push_back(V.dinv[k]);
    }
  }
  off[L] = h.coarse_off;
  S->hsc_off_h = off;
  // levels with at most this many remaining unknowns run in one block
  const int kTailRows = S->opts.hsc_tail_rows > 0 ? S->opts.hsc_tail_rows : 1024;
  int tail = L;
  for (int l = 0; l < L; ++l)
    if (H.n - off[l] <= kTailRows) { tail = l; break; }
  S->hsc_tail = tail;
  if ((st = up_new(S, &S->d_hoff, off)) || (st = up_new(S, &S->d_hrlev, rlev)) ||
      (st = up_new(S, &S->d_hrrow, rrow)) || (st = up_new(S, &S->d_hrptr, rptr)) ||
      (st = up_new(S, &S->d_hrcol, rcol)) || (st = up_new(S, &S->d_hpptr, pptr)) ||
      (st = up_new(S, &S->d_hpcol, pcol)) || (st = up_new(S, &S->d_hrval64, rval)) ||
      (st = up_new(S, &S->d_hpval64, pval)) || (st = up_new(S, &S->d_hdinv64, dinv)) ||
      (st = up_new(S, &S->d_hsinv64, h.Sinv)) || (st = up_new(S, &S->d_hrval32, to_f32(rval))) ||
      (st = up_new(S, &S->d_hpval32, to_f32(pval))) || (st = up_new(S, &S->d_hdinv32, to_f32(dinv))) ||
      (st = up_new(S, &S->d_hsinv32, to_f32(h.Sinv))))
    return st;
  return CN_OK;
}

}  // namespace

// ===========================================================================
extern "C" {

void cn_default_build_opts(cn_build_opts* o) {
  std::memset(o, 0, sizeof *o);
  o->precond = CN_PRECOND_IC0;
  o->ordering = CN_ORDER_AUTO;
  o->laplacian = CN_LAPLACIAN_COT;
  o->mollify_delta = 1e-4;
  o->device = 0;
  o->max_rhs = 3;
}

void cn_default_solve_opts(cn_solve_opts* o) {
  std::memset(o, 0, sizeof *o);
  o->precision = CN_PREC_MIXED;
  o->mode = CN_MODE_DEFORM;
  o->algo = CN_ALGO_FUSED;
  o->tol = 1e-8;
  o->max_iter = 2000;
  o->max_refine = 8;
  o->inner_tol = 1e-5;
  o->warm_start = 0;
  o->wait_limit_ms = 2000.0;
}

const char* cn_status_string(int32_t s) {
  if (s < 0 || s > 9) return "unknown";
  return kStatusText[s];
}

const char* cn_last_error(void) { return cn::last_err(); }

cn_status cn_cut_mesh(int32_t nv, int32_t nt, const int32_t* tris, int32_t nloops,
                      const int32_t* loop_ptr, const int32_t* loop_verts, int32_t* tris_out,
                      int32_t* parent_out, int32_t* nv_out) {
  if (nv < 0 || nt < 0 || nloops < 0 || !tris_out || !parent_out || !nv_out) {
    set_err("bad arguments");
    return CN_BAD_INPUT;
  }
  for (int i = 0; i < 3 * nt; ++i)
    if (tris[i] < 0 || tris[i] >= nv) {
      set_err("triangle vertex out of range");
      return CN_BAD_INPUT;
    }
  std::vector<int> vf_ptr, vf_face, vf_corner;
  cn::vertex_faces(nv, nt, tris, vf_ptr, vf_face, vf_corner);
  std::memcpy(tris_out, tris, sizeof(int32_t) * 3 * (size_t)nt);
  for (int v = 0; v < nv; ++v) parent_out[v] = v;
  std::vector<char> seen(nv, 0);
  int next_id = nv;
  for (int l = 0; l < nloops; ++l) {
    const int lo = loop_ptr[l], hi = loop_ptr[l + 1], m = hi - lo;
    if (m < 3) {
      set_err("loop %d has fewer than 3 vertices", l);
      return CN_BAD_INPUT;
    }
    for (int i = 0; i < m; ++i) {
      const int v = loop_verts[lo + i];
      const int vn = loop_verts[lo + (i + 1) % m], vp = loop_verts[lo + (i - 1 + m) % m];
      if (v < 0 || v >= nv || seen[v]) {
        set_err("loop vertex %d out of range or in two loops", v);
        return CN_BAD_INPUT;
      }
      seen[v] = 1;
      const int copy = next_id++;
      parent_out[copy] = v;
      // Sweep the fan of v counter-clockwise from the face with edge (v, vn):
      // in face (v, a, b) the next face is the one holding (v, b, .).
      int a = vn, guard = 0;
      const int deg = vf_ptr[v + 1] - vf_ptr[v];
      while (true) {
        int f = -1, cf = -1;
        for (int q = vf_ptr[v]; q < vf_ptr[v + 1]; ++q) {
          const int ff = vf_face[q], c = vf_corner[q];
          if (tris[3 * ff + (c + 1) % 3] == a) { f = ff; cf = c; break; }
        }
        if (f < 0 || ++guard > deg) {
          set_err("loop %d: the fan of vertex %d is open or not a disc", l, v);
          return CN_BAD_INPUT;
        }
        tris_out[3 * f + cf] = copy;
        const int b = tris[3 * f + (cf + 2) % 3];
        if (b == vp) break;
        a = b;
      }
    }
  }
  *nv_out = next_id;
  return CN_OK;
}

cn_status cn_build(const cn_mesh_desc* mesh, const cn_build_opts* opts, cn_handle* out) {
  cn::set_last_error_text("");
  if (!out) {
    set_err("out is NULL");
    return CN_BAD_INPUT;
  }
  *out = nullptr;
  cn_status st = cn::check_mesh(mesh);
  if (st != CN_OK) return st;
  cn_build_opts o;
  if (opts) o = *opts;
  else cn_default_build_opts(&o);
  if (o.max_rhs != 1 && o.max_rhs != 3 && o.max_rhs != 9) {
    set_err("max_rhs must be 1, 3 or 9");
    return CN_BAD_INPUT;
  }
  if (o.precond != CN_PRECOND_IC0 && o.precond != CN_PRECOND_JACOBI && o.precond != CN_PRECOND_HSC &&
      o.precond != CN_PRECOND_BSSOR) {
    set_err("unsupported preconditioner %d", o.precond);
    return CN_BAD_INPUT;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_err("no CUDA device");
    return CN_NO_DEVICE;
  }
  if (o.device < 0 || o.device >= ndev) {
    set_err("device %d out of range", o.device);
    return CN_BAD_INPUT;
  }
  if (cudaSetDevice(o.device) != cudaSuccess) {
    set_err("cudaSetDevice(%d) failed", o.device);
    return CN_CUDA_ERROR;
  }
  cn_system* S = new cn_system;
  S->opts = o;
  S->device = o.device;
  S->kmax = o.max_rhs;
  auto fail = [&](cn_status s) {
    cn_destroy(S);
    return s;
  };
  S->hsc = o.precond == CN_PRECOND_HSC;
  cn_build_opts ob = o;
  if (S->hsc) {  // the structure pass builds A in natural order without an IC(0) pattern
    ob.precond = CN_PRECOND_JACOBI;
    ob.ordering = CN_ORDER_NATURAL;
  }
  st = cn::build_host(mesh, ob, S->H);
  if (st != CN_OK) return fail(st);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->device);
  S->max_grid_alloc = std::max(sms * 8, 1024);
  if (cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&S->ev0) != cudaSuccess || cudaEventCreate(&S->ev1) != cudaSuccess) {
    set_err("stream/event creation failed");
    return fail(CN_CUDA_ERROR);
  }
  cn::Bump sizing;
  layout_all(sizing, S);
  if (cudaMalloc((void**)&S->buf, sizing.off) != cudaSuccess) {
    set_err("device allocation of %zu bytes failed", sizing.off);
    return fail(CN_CUDA_ERROR);
  }
  S->bytes = sizing.off;
  cn::Bump real;
  real.base = S->buf;
  layout_all(real, S);
  if (cudaMemsetAsync(S->buf, 0, S->bytes, S->stream) != cudaSuccess) {
    set_err("device memset failed");
    return fail(CN_CUDA_ERROR);
  }
  st = cn::upload(S->H, S->D, S->stream);
  if (st != CN_OK) return fail(st);
  st = cn::assemble_factor(S->H, S->D, ob, S->d_status, S->stream, &S->shift_used);
  if (st != CN_OK) return fail(st);
  if (S->hsc) {
    st = setup_hsc(S, ob);
    if (st != CN_OK) return fail(st);
  }
  choose_launch(S);
  *out = S;
  return CN_OK;
}

void cn_destroy(cn_handle S) {
  if (!S) return;
  cudaSetDevice(S->device);
  if (S->stream) cudaStreamSynchronize(S->stream);
  if (S->buf) cudaFree(S->buf);
  for (void* p : S->hsc_mem) cudaFree(p);
  for (void* p : S->cnet_mem) cudaFree(p);
  for (void* p : {(void*)S->cnet.seg, (void*)S->cnet.ends, (void*)S->d_cnet_posed, (void*)S->d_cnet_F,
                  (void*)S->d_cnet_X})
    if (p) cudaFree(p);
  for (void* p : {(void*)S->d_curve_of, (void*)S->d_row_of, (void*)S->d_tau, (void*)S->d_rest_cp,
                  (void*)S->d_posed_cp, (void*)S->d_weights, (void*)S->d_dLdx, (void*)S->d_dP, (void*)S->d_dw,
                  (void*)S->d_vf_ptr, (void*)S->d_vf_face, (void*)S->d_vf_corner, (void*)S->d_contrib,
                  (void*)S->d_Xc, (void*)S->d_bcolor, (void*)S->d_bss_pos, S->d_bss_v, S->d_bss_lent,
                  (void*)S->d_bss_loff})
    if (p) cudaFree(p);
  if (S->ev0) cudaEventDestroy(S->ev0);
  if (S->ev1) cudaEventDestroy(S->ev1);
  if (S->stream) cudaStreamDestroy(S->stream);
  delete S;
}

void* cn_stream(cn_handle S) { return S ? (void*)S->stream : nullptr; }

cn_status cn_system_info(cn_handle S, int64_t* info) {
  if (!S || !info) return CN_BAD_INPUT;
  const MeshHost& H = S->H;
  int64_t v[12] = {H.n, H.nnzA, H.nnzL, S->hsc ? S->hsc_L : H.nlev, H.nnzK, H.nv, H.nh,
                   S->grid, S->block, S->lanes, H.ncolors, (int64_t)S->bytes};
  std::memcpy(info, v, sizeof v);
  return CN_OK;
}

static cn_status solve_plain(cn_handle S, int k, const double* d_targets, double* d_xout,
                             const cn_solve_opts* o, cn_solve_stats* stats);

static cn_status fill_stats(cn_handle S, int k, cn_solve_stats* stats) {
  DevStats ds;
  CN_CUDA(cudaMemcpyAsync(&ds, S->d_stats, sizeof ds, cudaMemcpyDeviceToHost, S->stream));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, S->ev0, S->ev1);
  std::memset(stats, 0, sizeof *stats);
  stats->status = ds.status;
  stats->iterations = ds.iterations;
  stats->refinements = ds.refinements;
  stats->k = k;
  stats->device_ms = ms;
  double mx = 0.0;
  for (int c = 0; c < k && c < 32; ++c) {
    stats->rel_residual[c] = ds.rel_residual[c];
    mx = std::max(mx, ds.rel_residual[c]);
  }
  stats->max_rel_residual = mx;
  return (cn_status)ds.status;
}

cn_status cn_solve_device(cn_handle S, int32_t k, const double* d_targets, double* d_xout,
                          const cn_solve_opts* opts, cn_solve_stats* stats) {
  if (!S) return CN_BAD_INPUT;
  cn_solve_opts o;
  if (opts) o = *opts;
  else cn_default_solve_opts(&o);
  if (k != 1 && k != 3 && k != 9) {
    set_err("k must be 1, 3 or 9");
    return CN_BAD_INPUT;
  }
  if (k > S->kmax) {
    set_err("k = %d exceeds the build's max_rhs = %d", k, S->kmax);
    return CN_BAD_INPUT;
  }
  if (o.mode == CN_MODE_DEFORM && k % 3 != 0) {
    set_err("deform mode needs k a multiple of 3");
    return CN_BAD_INPUT;
  }
  // The row-cached Jacobi kernel runs k = 9 as three k = 3 solves on column
  // slices: its k = 9 state fits neither shared memory nor registers, and
  // three k = 3 solves take a third of the time of one k = 9 solve.
  if (k == 9 && row_cached(S) && o.algo != CN_ALGO_PLAIN && S->d_split_t &&
      o.tol > 0.0 && o.max_iter >= 0 && o.max_refine >= 1) {
    CN_CUDA(cudaSetDevice(S->device));
    const int rows_t = o.mode == CN_MODE_RHS ? S->H.n : S->H.nh;
    cn_solve_opts o3 = o;
    o3.warm_start = 0;
    cn_solve_stats acc;
    std::memset(&acc, 0, sizeof acc);
    cn_status worst = CN_OK;
    for (int g = 0; g < 3; ++g) {
      CN_CUDA(cn::launch_copy_columns(d_targets, rows_t, 9, 3 * g, S->d_split_t, 3, 0, 3, S->stream));
      cn_solve_stats s3;
      const cn_status st = cn_solve_device(S, 3, S->d_split_t, S->d_split_x, &o3, stats ? &s3 : nullptr);
      if (st != CN_OK && st != CN_MAX_ITER) return st;
      if (st != CN_OK) worst = st;
      CN_CUDA(cn::launch_copy_columns(S->d_split_x, S->H.nv, 3, 0, d_xout, 9, 3 * g, 3, S->stream));
      if (stats) {
        acc.iterations += s3.iterations;
        acc.refinements = std::max(acc.refinements, s3.refinements);
        acc.device_ms += s3.device_ms;
        for (int c = 0; c < 3; ++c) acc.rel_residual[3 * g + c] = s3.rel_residual[c];
        acc.max_rel_residual = std::max(acc.max_rel_residual, s3.max_rel_residual);
        if (s3.status != CN_OK) acc.status = s3.status;
      }
    }
    S->have_solution = false;
    if (stats) {
      acc.k = 9;
      *stats = acc;
    }
    return worst;
  }
  if (!(o.tol > 0.0) || o.max_iter < 0 || o.max_refine < 1 || o.algo < CN_ALGO_FUSED ||
      o.algo > CN_ALGO_SINGLE) {
    set_err("bad solve options");
    return CN_BAD_INPUT;
  }
  CN_CUDA(cudaSetDevice(S->device));
  if (o.algo == CN_ALGO_PLAIN) return solve_plain(S, k, d_targets, d_xout, &o, stats);
  const bool mixed = o.precision == CN_PREC_MIXED;
  SolveArgs a = cn::solve_args(S->H, S->D, mixed);
  a.mode = o.mode; a.targets = d_targets; a.x_out = d_xout; a.x0 = nullptr;
  a.warm = o.warm_start && S->have_solution ? 1 : 0;
  a.b64 = S->d_b64; a.x64 = S->d_x64;
  void** w = mixed ? (void**)S->d_w32 : (void**)S->d_w64;
  a.r = w[0]; a.y = w[1]; a.z = w[2]; a.p0 = w[3]; a.p1 = w[4]; a.Ap = w[5]; a.xin = w[6];
  a.partials = S->d_partials;
  if (S->hsc) {
    a.hsc = 1;
    a.hsc_L = S->hsc_L;
    a.hsc_tail = S->hsc_tail;
    a.hsc_nc = S->hsc_nc;
    a.hsc_off = S->d_hoff;
    a.hsc_rlev = S->d_hrlev;
    a.hsc_rrow = S->d_hrrow;
    a.hsc_rptr = S->d_hrptr;
    a.hsc_rcol = S->d_hrcol;
    a.hsc_rval = mixed ? (const void*)S->d_hrval32 : (const void*)S->d_hrval64;
    a.hsc_pptr = S->d_hpptr;
    a.hsc_pcol = S->d_hpcol;
    a.hsc_pval = mixed ? (const void*)S->d_hpval32 : (const void*)S->d_hpval64;
    a.hsc_dinv = mixed ? (const void*)S->d_hdinv32 : (const void*)S->d_hdinv64;
    a.hsc_sinv = mixed ? (const void*)S->d_hsinv32 : (const void*)S->d_hsinv64;
  }
  a.tol = o.tol;
  a.inner_tol = mixed ? o.inner_tol : 0.0;
  a.max_iter = o.max_iter;
  a.max_refine = o.max_refine;
  a.ctl = S->d_ctl; a.stats = S->d_stats;
  a.timeout_ns = o.wait_limit_ms > 0.0 ? (long long)(o.wait_limit_ms * 1e6) : 2000000000LL;
  a.m0 = S->d_m[0]; a.m1 = S->d_m[1]; a.m2 = S->d_m[2]; a.pown = S->d_pown; a.dinv64 = S->D.dinv64;
  if (o.algo == CN_ALGO_PIPELINED &&
      (!row_cached(S) || (S->opts.precond == CN_PRECOND_BSSOR && o.precision != CN_PREC_MIXED))) {
    set_err("the pipelined form needs the Jacobi preconditioner, or block SSOR in mixed precision");
    return CN_BAD_INPUT;
  }
  if (o.algo == CN_ALGO_SINGLE && !row_cached(S) && !(S->opts.precond == CN_PRECOND_IC0 && !S->hsc)) {
    set_err("the single-reduction form runs on Jacobi, block SSOR and IC(0) handles");
    return CN_BAD_INPUT;
  }
  if (row_cached(S)) {
    // Jacobi -- FP64: pipelined, falling back to the two-reduction form if
    // an inner solve stalls; mixed: the two-reduction form (the FP32
    // pipelined recurrences drift on ill-conditioned meshes), pipelined on
    // request.  Block SSOR -- mixed: pipelined with u = M^-1 r kept by
    // recurrence, with the same fall-back; FP64: the two-reduction form.
    const bool bssor = S->opts.precond == CN_PRECOND_BSSOR;
    if (!bssor)
      a.pipe_mode = o.algo == CN_ALGO_PIPELINED ? 1 : o.algo == CN_ALGO_CLASSIC ? 0
                  : o.precision == CN_PREC_FP64 ? 2 : 0;
    else
      a.pipe_mode = o.precision != CN_PREC_MIXED || o.algo == CN_ALGO_CLASSIC ? 0
                  : o.algo == CN_ALGO_PIPELINED ? 5 : 4;
    if (o.algo == CN_ALGO_SINGLE) a.pipe_mode = 3;
    int rec = a.pipe_mode == 4 || a.pipe_mode == 5 ? 8 : 6;
    a.nbflag = S->d_nbflag;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->device);
    // the grid: every SM, or fewer blocks of at least 256 rows for a small mesh
    int grid = S->shape_set ? S->grid
             : S->opts.grid > 0 ? S->opts.grid : std::min(sms, std::max(1, (S->H.n + 255) / 256));
    int block = S->block, qr = 1;
    a.cache_bytes = 0;
    const int grid0 = grid, block0 = block;
    // The block-SSOR pipelined default needs each block's whole state in
    // shared memory (its longer records and the lists); where that does not
    // fit (the 1M-row torus: 14 row slices a block) the two-reduction form
    // measured faster, so the default falls back to it before the launch.
    for (int attempt = 0; attempt < 2; ++attempt) {
      grid = grid0;
      block = block0;
      qr = 1;
      a.cache_bytes = 0;
      rec = a.pipe_mode == 4 || a.pipe_mode == 5 ? 8 : 6;
      int level = 2;  // 2: row cache and own state in shared memory, 1: row cache only, 0: none
      if (grid > 1) {
        grid = std::min(grid, S->max_grid_alloc);
        // two rows per thread, gathered together: block = n / (2 grid) rounded
        // up to a warp (an explicit block above 512 runs one row per thread)
        if (!S->shape_set && S->opts.block <= 0)
          block = std::min(512, std::max(128, ((S->H.n + 2 * grid - 1) / (2 * grid) + 31) / 32 * 32));
        qr = block <= 512 ? 2 : 1;
        const size_t cap = 220 * 1024;
        for (int tries = 0; tries < 6; ++tries) {
          const auto key = std::make_tuple(grid, block, (int)o.precision, k, rec);
          auto it = S->pipe_smem.find(key);
          if (it == S->pipe_smem.end()) {
            size_t cache = 0, full = 0;
            cn::pipelined_smem_need(S->H.A_ptr.data(), S->H.A_col.data(), S->H.n, grid, block, o.precision, k, bssor,
                                    rec, &cache, &full);
            it = S->pipe_smem.emplace(key, std::make_pair(cache, full)).first;
          }
          const size_t pipe_cache = it->second.first, pipe_full = it->second.second;
          if (level == 2 && pipe_full > cap) level = 1;
          if (level == 1 && pipe_cache > cap) level = 0;
          a.cache_bytes = level == 2 ? (int)pipe_full : level == 1 ? (int)pipe_cache : 0;
          const int mg = cn::pipelined_max_grid(o.precision, k, block, a.cache_bytes, qr, a.pipe_mode);
          if (mg >= grid) break;
          if (mg <= 0) {
            if (level == 0) {
              set_err("the pipelined solve does not fit on this device (block %d)", block);
              return CN_CUDA_ERROR;
            }
            --level;
            continue;
          }
          grid = mg;
        }
      }
      if (a.pipe_mode == 4 && grid > 1 && level < 2) {
        a.pipe_mode = 0;
        continue;
      }
      break;
    }
    a.bcolor = nullptr;
    a.bncolor = 0;
    if (bssor) {
      // block-local colours for the blocks of this launch (rb rows each)
      const long long tot = (long long)(grid > 1 ? grid : 1) * block;
      const int rb = (int)(((long long)S->H.n + tot - 1) / tot * block);
      const int n = S->H.n;
      if (S->bcolor_rb != rb) {
        S->h_bcolor.assign((size_t)std::max(n, 1), 0);
        S->bncolor = cn::block_colours(S->H.A_ptr.data(), S->H.A_col.data(), n, std::max(rb, 1), S->h_bcolor.data());
        if (!S->d_bcolor) CN_CUDA(cudaMalloc((void**)&S->d_bcolor, (size_t)std::max(n, 1)));
        if (n) CN_CUDA(cudaMemcpyAsync(S->d_bcolor, S->h_bcolor.data(), (size_t)n, cudaMemcpyHostToDevice, S->stream));
        S->bcolor_rb = rb;
      }
      a.bcolor = S->d_bcolor;
      a.bncolor = S->bncolor;
      // the global tables (used by the blocks whose shared memory cannot hold
      // them): each block's list entries, prefix-summed
      const int nb = grid > 1 ? grid : 1;
      if (S->bss_rb != rb || S->bss_grid != nb) {
        std::vector<long long> off((size_t)nb + 1, 0);
        for (int b = 0; b < nb; ++b) {
          const long long blk0 = (long long)b * rb;
          const long long rb_n = blk0 < n ? std::min<long long>(n - blk0, rb) : 0;
          off[b + 1] = off[b] + (rb_n > 0 ? cn::block_list_entries(S->H.A_ptr.data(), S->H.A_col.data(),
                                                                     S->h_bcolor.data(), blk0, rb_n)
                                          : 0);
        }
        if (!S->d_bss_pos) {
          CN_CUDA(cudaMalloc((void**)&S->d_bss_pos, sizeof(int) * (size_t)std::max(n, 1)));
          CN_CUDA(cudaMalloc(&S->d_bss_v, 32 * (size_t)std::max(n, 1)));
        }
        if (off[nb] > S->bss_lent_cap || !S->d_bss_lent) {
          if (S->d_bss_lent) CN_CUDA(cudaFree(S->d_bss_lent));
          S->d_bss_lent = nullptr;
          CN_CUDA(cudaMalloc(&S->d_bss_lent, 16 * (size_t)std::max<long long>(off[nb], 1)));
          S->bss_lent_cap = off[nb];
        }
        if (nb + 1 > S->bss_loff_cap) {
          if (S->d_bss_loff) CN_CUDA(cudaFree(S->d_bss_loff));
          S->d_bss_loff = nullptr;
          CN_CUDA(cudaMalloc((void**)&S->d_bss_loff, sizeof(long long) * (size_t)(nb + 1)));
          S->bss_loff_cap = nb + 1;
        }
        CN_CUDA(cudaMemcpyAsync(S->d_bss_loff, off.data(), sizeof(long long) * (size_t)(nb + 1), cudaMemcpyHostToDevice, S->stream));
        S->bss_rb = rb;
        S->bss_grid = nb;
      }
      a.bss_pos = S->d_bss_pos;
      a.bss_v = S->d_bss_v;
      a.bss_lent = S->d_bss_lent;
      a.bss_loff = S->d_bss_loff;
    }
    CN_CUDA(cudaMemsetAsync(S->d_ctl, 0, sizeof(Control), S->stream));
    if (a.pipe_mode == 3)
      CN_CUDA(cudaMemsetAsync(S->d_nbflag, 0, sizeof(unsigned) * (size_t)std::max(grid, 1), S->stream));
    CN_CUDA(cudaEventRecord(S->ev0, S->stream));
    CN_CUDA(cn::launch_pipelined_solve(a, o.precision, k, block, grid, qr, S->stream));
    CN_CUDA(cudaEventRecord(S->ev1, S->stream));
    S->have_solution = true;
    if (!stats) return CN_OK;
    return fill_stats(S, k, stats);
  }
  int grid = S->grid, lblock = S->block, llanes = S->lanes;
  solve_shape(S, k, o, &grid, &lblock, &llanes);
  // IC(0) on a multi-block grid: the sweeps without grid barriers (tagged
  // words) under the single-reduction CG (icsf_wanted: mixed precision, or
  // FP64 on a large system); otherwise the level-scheduled kernel
  if (icsf_path(S, k, o)) {
    const int block = std::min(lblock, 512);
    const int mg = cn::icsf_max_grid(o.precision, k, block);
    if (mg <= 0) {
      set_err("the IC(0) solve does not fit on this device (block %d)", block);
      return CN_CUDA_ERROR;
    }
    grid = std::min(std::min(grid, mg), S->max_grid_alloc);
    a.m0 = S->d_m[0];
    a.m1 = S->d_m[1];
    CN_CUDA(cudaMemsetAsync(S->d_ctl, 0, sizeof(Control), S->stream));
    CN_CUDA(cudaEventRecord(S->ev0, S->stream));
    CN_CUDA(cn::launch_icsf_solve(a, o.precision, k, block, grid, S->stream));
    CN_CUDA(cudaEventRecord(S->ev1, S->stream));
    S->have_solution = true;
    if (!stats) return CN_OK;
    return fill_stats(S, k, stats);
  }
  if (grid > 1) {
    const int mg = cn::persistent_max_grid(o.precision, k, llanes, lblock);
    if (mg <= 0) {
      set_err("the persistent solve does not fit on this device (lanes %d, block %d)", llanes, lblock);
      return CN_CUDA_ERROR;
    }
    grid = std::min(std::min(grid, mg), S->max_grid_alloc);
  }
  // one block: the sweeps' y and z in shared memory when both fit
  a.cache_bytes = 0;
  if (grid <= 1 && !S->hsc) {
    const size_t half = ((size_t)S->H.n * k * (mixed ? sizeof(float) : sizeof(double)) + 15) & ~(size_t)15;
    if (2 * half <= (size_t)220 * 1024) a.cache_bytes = (int)(2 * half);
  }
  CN_CUDA(cudaMemsetAsync(S->d_ctl, 0, sizeof(Control), S->stream));
  CN_CUDA(cudaEventRecord(S->ev0, S->stream));
  CN_CUDA(cn::launch_persistent_solve(a, o.precision, k, llanes, lblock, grid, S->stream));
  CN_CUDA(cudaEventRecord(S->ev1, S->stream));
  S->have_solution = true;
  if (!stats) return CN_OK;
  return fill_stats(S, k, stats);
}

cn_status cn_solve(cn_handle S, int32_t k, const double* targets, const double* x0,
                   double* x_out, const cn_solve_opts* opts, cn_solve_stats* stats) {
  if (!S || !x_out || (k > 0 && !targets)) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  if (k < 1 || k > S->kmax) {
    set_err("k out of range");
    return CN_BAD_INPUT;
  }
  cn_solve_opts o;
  if (opts) o = *opts;
  else cn_default_solve_opts(&o);
  CN_CUDA(cudaSetDevice(S->device));
  const MeshHost& H = S->H;
  const size_t nt = (size_t)(o.mode == CN_MODE_RHS ? H.n : H.nh) * k;
  for (size_t i = 0; i < nt; ++i)
    if (!std::isfinite(targets[i])) {
      set_err("target %zu is not finite", i);
      return CN_NAN;
    }
  if (nt) CN_CUDA(cudaMemcpyAsync(S->d_targets, targets, sizeof(double) * nt, cudaMemcpyHostToDevice, S->stream));
  if (x0) {
    // the initial guess enters as the warm-start state, gathered to solve order
    std::vector<double> xs((size_t)H.n * k);
    for (int i = 0; i < H.n; ++i)
      for (int c = 0; c < k; ++c) xs[(size_t)i * k + c] = x0[(size_t)H.free_of[i] * k + c];
    CN_CUDA(cudaMemcpyAsync(S->d_x64, xs.data(), sizeof(double) * xs.size(), cudaMemcpyHostToDevice,
                            S->stream));
    CN_CUDA(cudaStreamSynchronize(S->stream));
    S->have_solution = true;
    o.warm_start = 1;
  }
  cn_solve_stats local;
  cn_status st = cn_solve_device(S, k, S->d_targets, S->d_xout, &o, stats ? stats : &local);
  if (st != CN_OK && st != CN_MAX_ITER) return st;
  CN_CUDA(cudaMemcpyAsync(x_out, S->d_xout, sizeof(double) * (size_t)H.nv * k, cudaMemcpyDeviceToHost,
                          S->stream));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  return st;
}

// Plain FP64 Jacobi-PCG: one kernel per primitive, the dots folded on the host
// every iteration (SlangCodegen/SparseLinAlg.lean:11-15,
// SlangCodegen/DotReduceMulti.lean:8-11), absolute-to-relative test as cn_solve.
static cn_status solve_plain(cn_handle S, int k, const double* d_targets, double* d_xout,
                             const cn_solve_opts* o, cn_solve_stats* stats) {
  cn::PlainArgs p{};
  p.n = S->H.n; p.K = k;
  p.A_ptr = S->D.A_ptr; p.A_col = S->D.A_col; p.A_val = S->D.A64; p.A_diag = S->D.A_diag;
  p.b = S->d_b64; p.x = S->d_x64;
  p.r = S->d_w64[0]; p.z = S->d_w64[1]; p.p = S->d_w64[2]; p.Ap = S->d_w64[3];
  p.blocks = 120;
  p.partials = S->d_partials;
  double* d_scal = S->d_scal;
  SolveArgs sa{};
  sa.nv = S->H.nv; sa.nh = S->H.nh; sa.K_ptr = S->D.K_ptr; sa.K_col = S->D.K_col; sa.K_val = S->D.K_val;
  sa.free_of = S->D.free_of; sa.hidx = S->D.hidx; sa.handles = S->D.handles; sa.pos = S->D.pos;
  sa.mode = o->mode; sa.targets = d_targets; sa.x_out = d_xout; sa.x0 = nullptr;
  std::vector<double> part((size_t)p.blocks * k), alpha(k), beta(k), rz(k), bb(k), rr(k);
  std::vector<int> active(k, 1);
  auto host_dot = [&](const double* u, const double* v, std::vector<double>& out) -> cn_status {
    CN_CUDA(cn::plain_dot(p, u, v, S->stream));
    CN_CUDA(cudaMemcpyAsync(part.data(), p.partials, sizeof(double) * part.size(), cudaMemcpyDeviceToHost,
                            S->stream));
    CN_CUDA(cudaStreamSynchronize(S->stream));
    for (int c = 0; c < k; ++c) {
      double s = 0.0;
      for (int b = 0; b < p.blocks; ++b) s += part[(size_t)b * k + c];
      out[c] = s;
    }
    return CN_OK;
  };
  CN_CUDA(cudaEventRecord(S->ev0, S->stream));
  CN_CUDA(cn::plain_rhs_and_init(sa, p, S->stream));
  CN_CUDA(cn::plain_residual(p, S->stream));
  cn_status st;
  if ((st = host_dot(p.b, p.b, bb)) != CN_OK) return st;
  CN_CUDA(cn::plain_jacobi(p, S->stream));
  CN_CUDA(cudaMemcpyAsync(p.p, p.z, sizeof(double) * (size_t)p.n * k, cudaMemcpyDeviceToDevice, S->stream));
  if ((st = host_dot(p.r, p.z, rz)) != CN_OK) return st;
  int it = 0;
  for (; it < o->max_iter; ++it) {
    CN_CUDA(cn::plain_spmv(p, p.p, p.Ap, S->stream));
    std::vector<double> pap(k);
    if ((st = host_dot(p.p, p.Ap, pap)) != CN_OK) return st;
    for (int c = 0; c < k; ++c) {
      if (active[c] && !(pap[c] > 0.0)) active[c] = 0;
      alpha[c] = active[c] ? rz[c] / pap[c] : 0.0;
    }
    CN_CUDA(cn::plain_set_scalars(d_scal, alpha.data(), k, S->stream));
    CN_CUDA(cn::plain_axpy2(p, d_scal, S->stream));
    if ((st = host_dot(p.r, p.r, rr)) != CN_OK) return st;
    bool any = false;
    for (int c = 0; c < k; ++c) {
      if (active[c] && rr[c] < o->tol * o->tol * bb[c]) active[c] = 0;
      any = any || active[c];
    }
    if (!any) { ++it; break; }
    CN_CUDA(cn::plain_jacobi(p, S->stream));
    std::vector<double> rzn(k);
    if ((st = host_dot(p.r, p.z, rzn)) != CN_OK) return st;
    for (int c = 0; c < k; ++c) {
      beta[c] = active[c] ? (rz[c] == 0.0 ? 0.0 : rzn[c] / rz[c]) : 0.0;
      rz[c] = rzn[c];
    }
    CN_CUDA(cn::plain_set_scalars(d_scal + k, beta.data(), k, S->stream));
    CN_CUDA(cn::plain_saxpby(p, d_scal + k, S->stream));
  }
  CN_CUDA(cn::plain_residual(p, S->stream));
  if ((st = host_dot(p.r, p.r, rr)) != CN_OK) return st;
  CN_CUDA(cn::plain_output(sa, p, S->stream));
  CN_CUDA(cudaEventRecord(S->ev1, S->stream));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  S->have_solution = false;  // the plain path does not keep the warm-start layout
  CN_CUDA(cudaMemsetAsync(S->d_x64, 0, sizeof(double) * (size_t)S->H.n * S->kmax, S->stream));
  double mx = 0.0;
  cn_status res = CN_OK;
  cn_solve_stats local{};
  cn_solve_stats* out = stats ? stats : &local;
  std::memset(out, 0, sizeof *out);
  for (int c = 0; c < k; ++c) {
    const double rel = bb[c] > 0 ? std::sqrt(rr[c] / bb[c]) : std::sqrt(rr[c]);
    if (c < 32) out->rel_residual[c] = rel;
    mx = std::max(mx, rel);
    if (!(rel <= o->tol)) res = CN_MAX_ITER;
  }
  float ms = 0.f;
  cudaEventElapsedTime(&ms, S->ev0, S->ev1);
  out->status = res;
  out->iterations = it;
  out->refinements = 1;
  out->k = k;
  out->max_rel_residual = mx;
  out->device_ms = ms;
  return res;
}

// ---------------------------------------------------------------------------
// Profile curves -> handle targets, deform, adjoint (cn_adjoint.cu).
static cn::CurveArgs curve_args(cn_handle S) {
  cn::CurveArgs c{};
  c.nh = S->H.nh; c.ncurves = S->ncurves; c.nseg = S->nseg;
  c.handles = S->D.handles; c.curve_of = S->d_curve_of; c.tau = S->d_tau;
  c.rest_cp = S->d_rest_cp; c.posed_cp = S->d_posed_cp; c.weights = S->d_weights; c.pos = S->D.pos;
  return c;
}

cn_status cn_bind_curves(cn_handle S, int32_t n_curves, int32_t n_segments, const double* rest_cp,
                         const int32_t* curve_of, const double* tau) {
  if (!S || n_curves < 1 || n_segments < 1 || !rest_cp || !curve_of || !tau) {
    set_err("bad curve binding arguments");
    return CN_BAD_INPUT;
  }
  const MeshHost& H = S->H;
  for (int h = 0; h < H.nh; ++h)
    if (curve_of[h] >= n_curves || !std::isfinite(tau[h]) || tau[h] < 0.0 || tau[h] > n_segments) {
      set_err("handle %d: curve %d / parameter out of range", h, curve_of[h]);
      return CN_BAD_INPUT;
    }
  const size_t ncp = (size_t)n_curves * (3 * n_segments + 1) * 3;
  for (size_t i = 0; i < ncp; ++i)
    if (!std::isfinite(rest_cp[i])) {
      set_err("rest control point %zu is not finite", i);
      return CN_NAN;
    }
  CN_CUDA(cudaSetDevice(S->device));
  for (void* p : {(void*)S->d_curve_of, (void*)S->d_row_of, (void*)S->d_tau, (void*)S->d_rest_cp,
                  (void*)S->d_posed_cp, (void*)S->d_weights, (void*)S->d_dLdx, (void*)S->d_dP, (void*)S->d_dw})
    if (p) cudaFree(p);
  S->ncurves = n_curves;
  S->nseg = n_segments;
  S->have_forward = false;
  std::vector<int> row_of(H.nv, -1);
  for (int i = 0; i < H.n; ++i) row_of[H.free_of[i]] = i;
  CN_CUDA(cudaMalloc((void**)&S->d_curve_of, sizeof(int) * std::max(H.nh, 1)));
  CN_CUDA(cudaMalloc((void**)&S->d_row_of, sizeof(int) * std::max(H.nv, 1)));
  CN_CUDA(cudaMalloc((void**)&S->d_tau, sizeof(double) * std::max(H.nh, 1)));
  CN_CUDA(cudaMalloc((void**)&S->d_rest_cp, sizeof(double) * ncp));
  CN_CUDA(cudaMalloc((void**)&S->d_posed_cp, sizeof(double) * ncp));
  CN_CUDA(cudaMalloc((void**)&S->d_weights, sizeof(double) * n_curves));
  CN_CUDA(cudaMalloc((void**)&S->d_dLdx, sizeof(double) * 3 * std::max(H.nv, 1)));
  CN_CUDA(cudaMalloc((void**)&S->d_dP, sizeof(double) * ncp));
  CN_CUDA(cudaMalloc((void**)&S->d_dw, sizeof(double) * n_curves));
  if (H.nh) {
    CN_CUDA(cudaMemcpyAsync(S->d_curve_of, curve_of, sizeof(int) * H.nh, cudaMemcpyHostToDevice, S->stream));
    CN_CUDA(cudaMemcpyAsync(S->d_tau, tau, sizeof(double) * H.nh, cudaMemcpyHostToDevice, S->stream));
  }
  CN_CUDA(cudaMemcpyAsync(S->d_row_of, row_of.data(), sizeof(int) * H.nv, cudaMemcpyHostToDevice, S->stream));
  CN_CUDA(cudaMemcpyAsync(S->d_rest_cp, rest_cp, sizeof(double) * ncp, cudaMemcpyHostToDevice, S->stream));
  return CN_OK;
}

cn_status cn_deform(cn_handle S, const double* posed_cp, const double* weights, double* x_out,
                    const cn_solve_opts* opts, cn_solve_stats* stats) {
  if (!S || !posed_cp || !weights || !x_out) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  if (!S->ncurves) {
    set_err("no curves bound (cn_bind_curves)");
    return CN_BAD_INPUT;
  }
  const size_t ncp = (size_t)S->ncurves * (3 * S->nseg + 1) * 3;
  for (size_t i = 0; i < ncp; ++i)
    if (!std::isfinite(posed_cp[i])) {
      set_err("posed control point %zu is not finite", i);
      return CN_NAN;
    }
  for (int c = 0; c < S->ncurves; ++c)
    if (!std::isfinite(weights[c])) {
      set_err("weight %d is not finite", c);
      return CN_NAN;
    }
  cn_solve_opts o;
  if (opts) o = *opts;
  else cn_default_solve_opts(&o);
  o.mode = CN_MODE_DEFORM;
  CN_CUDA(cudaSetDevice(S->device));
  CN_CUDA(cudaMemcpyAsync(S->d_posed_cp, posed_cp, sizeof(double) * ncp, cudaMemcpyHostToDevice, S->stream));
  CN_CUDA(cudaMemcpyAsync(S->d_weights, weights, sizeof(double) * S->ncurves, cudaMemcpyHostToDevice, S->stream));
  CN_CUDA(cn::launch_curve_targets(curve_args(S), S->d_targets, S->stream));
  cn_solve_stats local;
  cn_status st = cn_solve_device(S, 3, S->d_targets, S->d_xout, &o, stats ? stats : &local);
  if (st != CN_OK && st != CN_MAX_ITER) return st;
  CN_CUDA(cudaMemcpyAsync(x_out, S->d_xout, sizeof(double) * 3 * (size_t)S->H.nv, cudaMemcpyDeviceToHost,
                          S->stream));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  S->have_forward = true;
  return st;
}

cn_status cn_adjoint(cn_handle S, const double* dL_dx, double* dL_dcp, double* dL_dw, const cn_solve_opts* opts,
                     cn_solve_stats* stats) {
  if (!S || !dL_dx || !dL_dcp || !dL_dw) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  if (!S->have_forward) {
    set_err("cn_adjoint needs a preceding cn_deform on this handle");
    return CN_BAD_INPUT;
  }
  const MeshHost& H = S->H;
  for (size_t i = 0; i < 3 * (size_t)H.nv; ++i)
    if (!std::isfinite(dL_dx[i])) {
      set_err("dL/dx %zu is not finite", i);
      return CN_NAN;
    }
  cn_solve_opts o;
  if (opts) o = *opts;
  else cn_default_solve_opts(&o);
  o.mode = CN_MODE_RHS;
  o.warm_start = 0;
  CN_CUDA(cudaSetDevice(S->device));
  CN_CUDA(cudaMemcpyAsync(S->d_dLdx, dL_dx, sizeof(double) * 3 * H.nv, cudaMemcpyHostToDevice, S->stream));
  CN_CUDA(cn::launch_adjoint_rhs(H.n, S->D.free_of, S->d_dLdx, S->d_targets, S->stream));
  // A lambda = g_f with the same factor (A is symmetric); lambda lands in x64.
  cn_solve_stats local;
  cn_status st = cn_solve_device(S, 3, S->d_targets, nullptr, &o, stats ? stats : &local);
  S->have_solution = false;  // x64 now holds lambda, not a warm start
  if (st != CN_OK && st != CN_MAX_ITER) return st;
  CN_CUDA(cn::launch_adjoint_grad(curve_args(S), S->D.K_ptr, S->D.K_col, S->D.K_val, S->d_row_of, S->d_x64,
                                  S->d_dLdx, S->d_dP, S->d_dw, S->stream));
  const size_t ncp = (size_t)S->ncurves * (3 * S->nseg + 1) * 3;
  CN_CUDA(cudaMemcpyAsync(dL_dcp, S->d_dP, sizeof(double) * ncp, cudaMemcpyDeviceToHost, S->stream));
  CN_CUDA(cudaMemcpyAsync(dL_dw, S->d_dw, sizeof(double) * S->ncurves, cudaMemcpyDeviceToHost, S->stream));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  return st;
}

// DeGoes22 two-stage solve (DeformSolve.lean:110-135): Stage 1 (k = 9
// harmonic solve of F), the bridge (cn_deform.cu), Stage 2 (k = 3).
// Device tables of the two-stage solve (vertex -> incident faces, per-face
// contributions, X_c), allocated on first use.
static cn_status ensure_deform_tables(cn_handle S) {
  const MeshHost& H = S->H;
  if (S->d_vf_ptr) return CN_OK;
  CN_CUDA(cudaMalloc((void**)&S->d_vf_ptr, sizeof(int) * H.vf_ptr.size()));
  CN_CUDA(cudaMalloc((void**)&S->d_vf_face, sizeof(int) * std::max<size_t>(H.vf_face.size(), 1)));
  CN_CUDA(cudaMalloc((void**)&S->d_vf_corner, sizeof(int) * std::max<size_t>(H.vf_corner.size(), 1)));
  CN_CUDA(cudaMalloc((void**)&S->d_contrib, sizeof(double) * 9 * std::max(H.nt, 1)));
  CN_CUDA(cudaMalloc((void**)&S->d_Xc, sizeof(double) * 3 * std::max(H.nh, 1)));
  CN_CUDA(cudaMemcpyAsync(S->d_vf_ptr, H.vf_ptr.data(), sizeof(int) * H.vf_ptr.size(), cudaMemcpyHostToDevice, S->stream));
  if (!H.vf_face.empty()) {
    CN_CUDA(cudaMemcpyAsync(S->d_vf_face, H.vf_face.data(), sizeof(int) * H.vf_face.size(), cudaMemcpyHostToDevice, S->stream));
    CN_CUDA(cudaMemcpyAsync(S->d_vf_corner, H.vf_corner.data(), sizeof(int) * H.vf_corner.size(),
                            cudaMemcpyHostToDevice, S->stream));
  }
  return CN_OK;
}

// DeformSolve.lean:110-135 from F_c in d_targets (n_handles x 9) and X_c in
// d_Xc (n_handles x 3), both on the device: Stage 1 (k = 9 harmonic solve),
// the Eq.(3) bridge, Stage 2 (k = 3); positions in d_xout, handle rows not
// yet overlaid.
static cn_status deform_stages(cn_handle S, const cn_solve_opts& o, cn_solve_stats* stats) {
  const MeshHost& H = S->H;
  cn_solve_opts o1 = o;
  o1.mode = CN_MODE_HARMONIC;
  o1.warm_start = 0;
  cn_solve_stats s1;
  cn_status st = cn_solve_device(S, 9, S->d_targets, S->d_xout, &o1, &s1);
  if (st != CN_OK) return st;
  cn::DeformArgs d{};
  d.nt = H.nt; d.n = H.n; d.tris = S->D.tris; d.pos = S->D.pos; d.face_m = S->D.face_m;
  d.hidx = S->D.hidx; d.Fv = S->d_xout; d.Xc = S->d_Xc; d.free_of = S->D.free_of;
  d.vf_ptr = S->d_vf_ptr; d.vf_face = S->d_vf_face; d.vf_corner = S->d_vf_corner;
  d.contrib = S->d_contrib; d.b = S->d_targets;
  CN_CUDA(cn::launch_deform_bridge(d, S->stream));
  cn_solve_opts o2 = o;
  o2.mode = CN_MODE_RHS;
  o2.warm_start = 0;
  cn_solve_stats s2;
  st = cn_solve_device(S, 3, S->d_targets, S->d_xout, &o2, stats ? stats : &s2);
  S->have_solution = false;
  if (stats) stats->iterations += s1.iterations;
  return st;
}

cn_status cn_solve_deformation(cn_handle S, const double* Fc, const double* Xc, double* x_out,
                               const cn_solve_opts* opts, cn_solve_stats* stats) {
  if (!S || !Fc || !Xc || !x_out) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  if (S->kmax < 9) {
    set_err("the two-stage solve needs a build with max_rhs = 9");
    return CN_BAD_INPUT;
  }
  const MeshHost& H = S->H;
  for (size_t i = 0; i < 9 * (size_t)H.nh; ++i)
    if (!std::isfinite(Fc[i])) {
      set_err("F_c %zu is not finite", i);
      return CN_NAN;
    }
  for (size_t i = 0; i < 3 * (size_t)H.nh; ++i)
    if (!std::isfinite(Xc[i])) {
      set_err("X_c %zu is not finite", i);
      return CN_NAN;
    }
  CN_CUDA(cudaSetDevice(S->device));
  cn_status st = ensure_deform_tables(S);
  if (st != CN_OK) return st;
  cn_solve_opts o;
  if (opts) o = *opts;
  else cn_default_solve_opts(&o);
  if (H.nh) CN_CUDA(cudaMemcpyAsync(S->d_targets, Fc, sizeof(double) * 9 * H.nh, cudaMemcpyHostToDevice, S->stream));
  CN_CUDA(cudaMemcpyAsync(S->d_Xc, Xc, sizeof(double) * 3 * std::max(H.nh, 0), cudaMemcpyHostToDevice, S->stream));
  st = deform_stages(S, o, stats);
  if (st != CN_OK && st != CN_MAX_ITER) return st;
  CN_CUDA(cudaMemcpyAsync(x_out, S->d_xout, sizeof(double) * 3 * (size_t)H.nv, cudaMemcpyDeviceToHost, S->stream));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  for (int h = 0; h < H.nh; ++h)
    for (int c = 0; c < 3; ++c) x_out[3 * (size_t)H.handles[h] + c] = Xc[3 * (size_t)h + c];
  return st;
}

// ---------------------------------------------------------------------------
// Profile curvenet (cn_curvenet.cu holds the kernels and the rules).

static cn_status cnet_upload_bytes(cn_system* S, void** dst, const void* h, size_t bytes) {
  void* d = nullptr;
  CN_CUDA(cudaMalloc(&d, std::max<size_t>(bytes, 8)));
  S->cnet_mem.push_back(d);
  if (bytes) CN_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, S->stream));
  *dst = d;
  return CN_OK;
}
static cn_status cnet_upload_i(cn_system* S, const int** dst, const int* h, size_t n) {
  return cnet_upload_bytes(S, (void**)dst, h, sizeof(int) * n);
}
static cn_status cnet_upload_d(cn_system* S, const double** dst, const double* h, size_t n) {
  return cnet_upload_bytes(S, (void**)dst, h, sizeof(double) * n);
}

cn_status cn_bind_curvenet(cn_handle S, const cn_curvenet_desc* net) {
  if (!S || !net || !net->rest_cp || !net->sample_tau || !net->handle_curve || !net->handle_sample ||
      !net->handle_side) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  const int C = net->n_curves, Sg = net->n_segments, M = net->n_samples, nn = net->n_nodes;
  if (C < 1 || Sg < 1 || M < 2 || nn < 0 || (nn > 0 && (!net->node_ptr || !net->node_ends))) {
    set_err("cn_bind_curvenet: need n_curves >= 1, n_segments >= 1, n_samples >= 2 and node tables");
    return CN_BAD_INPUT;
  }
  const size_t np = 3 * (size_t)Sg + 1;
  for (size_t i = 0; i < (size_t)C * np * 3; ++i)
    if (!std::isfinite(net->rest_cp[i])) {
      set_err("rest control point %zu is not finite", i);
      return CN_NAN;
    }
  for (int c = 0; c < C; ++c)
    for (int i = 0; i < M; ++i) {
      const double t = net->sample_tau[(size_t)c * M + i];
      if (!(t >= 0.0 && t <= (double)Sg) || (i > 0 && !(t > net->sample_tau[(size_t)c * M + i - 1]))) {
        set_err("sample parameters of curve %d must rise strictly inside [0, %d]", c, Sg);
        return CN_BAD_INPUT;
      }
    }
  std::vector<int> closed(C, 0), kind(C, 0), seg_off(C + 1, 0);
  for (int c = 0; c < C; ++c) closed[c] = net->closed ? (net->closed[c] != 0) : 0;
  std::vector<int> used(2 * (size_t)C, 0);
  if (nn > 0) {
    if (net->node_ptr[0] != 0) {
      set_err("node_ptr[0] must be 0");
      return CN_BAD_INPUT;
    }
    for (int j = 0; j < nn; ++j) {
      const int deg = net->node_ptr[j + 1] - net->node_ptr[j];
      if (deg < 2 || deg > cn::kCnetMaxNodeDegree) {
        set_err("intersection %d has %d curve ends (2..%d)", j, deg, cn::kCnetMaxNodeDegree);
        return CN_BAD_INPUT;
      }
      for (int q = net->node_ptr[j]; q < net->node_ptr[j + 1]; ++q) {
        const int e = net->node_ends[q];
        if (e < 0 || e >= 2 * C || closed[e >> 1] || used[e]) {
          set_err("intersection %d: curve end %d is out of range, on a closed curve or used twice", j, e);
          return CN_BAD_INPUT;
        }
        used[e] = 1;
        kind[e >> 1] |= (e & 1) ? 2 : 1;
      }
    }
  }
  for (int c = 0; c < C; ++c) seg_off[c + 1] = seg_off[c] + (closed[c] ? M : M - 1);
  const MeshHost& H = S->H;
  for (int h = 0; h < H.nh; ++h) {
    const int c = net->handle_curve[h];
    if (c < -1 || c >= C || (c >= 0 && (net->handle_sample[h] < 0 || net->handle_sample[h] >= M)) ||
        (c >= 0 && net->handle_side[h] != 0 && net->handle_side[h] != 1)) {
      set_err("handle %d: curve, sample or side out of range", h);
      return CN_BAD_INPUT;
    }
  }
  CN_CUDA(cudaSetDevice(S->device));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  for (void* p : S->cnet_mem) cudaFree(p);
  S->cnet_mem.clear();
  cn::CurvenetArgs& a = S->cnet;
  // the per-pose scratch is sized for the new binding on the next call
  for (void* p : {(void*)a.seg, (void*)a.ends, (void*)S->d_cnet_posed, (void*)S->d_cnet_F, (void*)S->d_cnet_X})
    if (p) cudaFree(p);
  S->d_cnet_posed = S->d_cnet_F = S->d_cnet_X = nullptr;
  S->cnet_pose_cap = 0;
  S->have_cnet = false;
  a = cn::CurvenetArgs{};
  a.n_curves = C; a.n_segments = Sg; a.n_samples = M; a.n_nodes = nn; a.total_segs = seg_off[C]; a.nh = H.nh;
  cn_status st;
  std::vector<int> zero1(1, 0);
  if ((st = cnet_upload_d(S, &a.rest_cp, net->rest_cp, (size_t)C * np * 3)) != CN_OK ||
      (st = cnet_upload_d(S, &a.sample_tau, net->sample_tau, (size_t)C * M)) != CN_OK ||
      (st = cnet_upload_i(S, &a.seg_off, seg_off.data(), seg_off.size())) != CN_OK ||
      (st = cnet_upload_i(S, &a.curve_kind, kind.data(), kind.size())) != CN_OK ||
      (st = cnet_upload_i(S, &a.node_ptr, nn > 0 ? net->node_ptr : zero1.data(), nn > 0 ? (size_t)nn + 1 : 1)) !=
          CN_OK ||
      (st = cnet_upload_i(S, &a.node_ends, net->node_ends, nn > 0 ? (size_t)net->node_ptr[nn] : 0)) != CN_OK ||
      (st = cnet_upload_i(S, &a.h_curve, net->handle_curve, (size_t)H.nh)) != CN_OK ||
      (st = cnet_upload_i(S, &a.h_sample, net->handle_sample, (size_t)H.nh)) != CN_OK ||
      (st = cnet_upload_i(S, &a.h_side, net->handle_side, (size_t)H.nh)) != CN_OK)
    return st;
  a.handles = S->D.handles;
  a.pos = S->D.pos;
  S->have_cnet = true;
  return CN_OK;
}

static cn_status cnet_scratch(cn_system* S, int n_poses) {
  if (n_poses <= S->cnet_pose_cap) return CN_OK;
  cn::CurvenetArgs& a = S->cnet;
  for (void* p : {(void*)a.seg, (void*)a.ends, (void*)S->d_cnet_posed, (void*)S->d_cnet_F, (void*)S->d_cnet_X})
    if (p) cudaFree(p);
  a.seg = a.ends = S->d_cnet_posed = S->d_cnet_F = S->d_cnet_X = nullptr;
  S->cnet_pose_cap = 0;
  const size_t np = 3 * (size_t)a.n_segments + 1;
  CN_CUDA(cudaMalloc((void**)&a.seg, sizeof(double) * 8 * std::max<size_t>((size_t)n_poses * a.total_segs, 1)));
  CN_CUDA(cudaMalloc((void**)&a.ends, sizeof(double) * 32 * (size_t)n_poses * a.n_curves));
  CN_CUDA(cudaMalloc((void**)&S->d_cnet_posed, sizeof(double) * (size_t)n_poses * a.n_curves * np * 3));
  CN_CUDA(cudaMalloc((void**)&S->d_cnet_F, sizeof(double) * 9 * std::max<size_t>((size_t)n_poses * a.nh, 1)));
  CN_CUDA(cudaMalloc((void**)&S->d_cnet_X, sizeof(double) * 3 * std::max<size_t>((size_t)n_poses * a.nh, 1)));
  // the intersection records of curve ends without a node stay zero
  CN_CUDA(cudaMemset(a.ends, 0, sizeof(double) * 32 * (size_t)n_poses * a.n_curves));
  S->cnet_pose_cap = n_poses;
  return CN_OK;
}

cn_status cn_curvenet_constraints_device(cn_handle S, int32_t n_poses, const double* d_posed_cp, double* d_Fc,
                                         double* d_Xc) {
  if (!S || !d_posed_cp || !d_Fc || !d_Xc || n_poses < 1) {
    set_err("null argument or n_poses < 1");
    return CN_BAD_INPUT;
  }
  if (!S->have_cnet) {
    set_err("no curvenet bound (cn_bind_curvenet)");
    return CN_BAD_INPUT;
  }
  CN_CUDA(cudaSetDevice(S->device));
  cn_status st = cnet_scratch(S, n_poses);
  if (st != CN_OK) return st;
  CN_CUDA(cn::launch_curvenet_constraints(S->cnet, n_poses, d_posed_cp, d_Fc, d_Xc, S->stream));
  return CN_OK;
}

cn_status cn_curvenet_constraints(cn_handle S, int32_t n_poses, const double* posed_cp, double* Fc, double* Xc) {
  if (!S || !posed_cp || !Fc || !Xc || n_poses < 1) {
    set_err("null argument or n_poses < 1");
    return CN_BAD_INPUT;
  }
  if (!S->have_cnet) {
    set_err("no curvenet bound (cn_bind_curvenet)");
    return CN_BAD_INPUT;
  }
  const cn::CurvenetArgs& a = S->cnet;
  const size_t ncp = (size_t)n_poses * a.n_curves * (3 * (size_t)a.n_segments + 1) * 3;
  for (size_t i = 0; i < ncp; ++i)
    if (!std::isfinite(posed_cp[i])) {
      set_err("posed control point %zu is not finite", i);
      return CN_NAN;
    }
  CN_CUDA(cudaSetDevice(S->device));
  cn_status st = cnet_scratch(S, n_poses);
  if (st != CN_OK) return st;
  CN_CUDA(cudaMemcpyAsync(S->d_cnet_posed, posed_cp, sizeof(double) * ncp, cudaMemcpyHostToDevice, S->stream));
  CN_CUDA(cn::launch_curvenet_constraints(S->cnet, n_poses, S->d_cnet_posed, S->d_cnet_F, S->d_cnet_X, S->stream));
  CN_CUDA(cudaMemcpyAsync(Fc, S->d_cnet_F, sizeof(double) * 9 * (size_t)n_poses * a.nh, cudaMemcpyDeviceToHost,
                          S->stream));
  CN_CUDA(cudaMemcpyAsync(Xc, S->d_cnet_X, sizeof(double) * 3 * (size_t)n_poses * a.nh, cudaMemcpyDeviceToHost,
                          S->stream));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  return CN_OK;
}

cn_status cn_deform_curvenet(cn_handle S, const double* posed_cp, double* x_out, const cn_solve_opts* opts,
                             cn_solve_stats* stats) {
  if (!S || !posed_cp || !x_out) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  if (!S->have_cnet) {
    set_err("no curvenet bound (cn_bind_curvenet)");
    return CN_BAD_INPUT;
  }
  if (S->kmax < 9) {
    set_err("the two-stage solve needs a build with max_rhs = 9");
    return CN_BAD_INPUT;
  }
  const MeshHost& H = S->H;
  const cn::CurvenetArgs& a = S->cnet;
  const size_t ncp = (size_t)a.n_curves * (3 * (size_t)a.n_segments + 1) * 3;
  for (size_t i = 0; i < ncp; ++i)
    if (!std::isfinite(posed_cp[i])) {
      set_err("posed control point %zu is not finite", i);
      return CN_NAN;
    }
  CN_CUDA(cudaSetDevice(S->device));
  cn_status st = ensure_deform_tables(S);
  if (st != CN_OK) return st;
  if ((st = cnet_scratch(S, 1)) != CN_OK) return st;
  cn_solve_opts o;
  if (opts) o = *opts;
  else cn_default_solve_opts(&o);
  CN_CUDA(cudaMemcpyAsync(S->d_cnet_posed, posed_cp, sizeof(double) * ncp, cudaMemcpyHostToDevice, S->stream));
  // F_c straight into the Stage-1 targets, X_c into the bridge's table
  CN_CUDA(cn::launch_curvenet_constraints(S->cnet, 1, S->d_cnet_posed, S->d_targets, S->d_Xc, S->stream));
  st = deform_stages(S, o, stats);
  if (st != CN_OK && st != CN_MAX_ITER) return st;
  CN_CUDA(cn::launch_curvenet_overlay(H.nh, S->D.handles, S->d_Xc, S->d_xout, S->stream));
  CN_CUDA(cudaMemcpyAsync(x_out, S->d_xout, sizeof(double) * 3 * (size_t)H.nv, cudaMemcpyDeviceToHost, S->stream));
  CN_CUDA(cudaStreamSynchronize(S->stream));
  return st;
}

// Direct Delta Mush bind (DirectDeltaMushBind.lean:6-40): W[:, i] is the
// harmonic solve with the unit target on handle i (chunks of 9 handles as
// one k = 9 solve), smoothed nu times over the cut-mesh adjacency, merged
// into each vertex's top-K list and renormalised.
cn_status cn_ddm_bind(cn_handle S, int32_t nu, double omega, int32_t top_k, const cn_solve_opts* opts,
                      int32_t* infl_idx, double* infl_w) {
  if (!S || !infl_idx || !infl_w) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  if (nu < 0 || !std::isfinite(omega) || top_k < 1 || top_k > 32) {
    set_err("cn_ddm_bind: need nu >= 0, a finite omega and 1 <= top_k <= 32");
    return CN_BAD_INPUT;
  }
  if (S->kmax < 9) {
    set_err("cn_ddm_bind needs a build with max_rhs = 9");
    return CN_BAD_INPUT;
  }
  const MeshHost& H = S->H;
  const int nv = H.nv, nh = H.nh;
  if (nh < 1) {
    set_err("cn_ddm_bind: the mesh has no handles");
    return CN_BAD_INPUT;
  }
  const int take = std::min(top_k, nh);
  cn_solve_opts o;
  if (opts) o = *opts;
  else cn_default_solve_opts(&o);
  o.mode = CN_MODE_HARMONIC;
  o.warm_start = 0;
  CN_CUDA(cudaSetDevice(S->device));
  int *d_bidx = nullptr, *d_cnt = nullptr;
  double *d_bw = nullptr, *d_tmp = nullptr;
  auto release = [&]() {
    for (void* p : {(void*)d_bidx, (void*)d_cnt, (void*)d_bw, (void*)d_tmp})
      if (p) cudaFree(p);
  };
  if (cudaMalloc((void**)&d_bidx, sizeof(int) * (size_t)nv * take) != cudaSuccess ||
      cudaMalloc((void**)&d_cnt, sizeof(int) * (size_t)nv) != cudaSuccess ||
      cudaMalloc((void**)&d_bw, sizeof(double) * (size_t)nv * take) != cudaSuccess ||
      cudaMalloc((void**)&d_tmp, sizeof(double) * (size_t)nv * 9) != cudaSuccess) {
    release();
    set_err("cn_ddm_bind: device allocation failed");
    return CN_CUDA_ERROR;
  }
  cn_status st = CN_OK;
  if (cudaMemsetAsync(d_cnt, 0, sizeof(int) * (size_t)nv, S->stream) != cudaSuccess) st = CN_CUDA_ERROR;
  for (int c0 = 0; c0 < nh && st == CN_OK; c0 += 9) {
    const int kc = std::min(9, nh - c0);
    if (cn::launch_ddm_unit_targets(nh, c0, kc, S->d_targets, S->stream) != cudaSuccess) { st = CN_CUDA_ERROR; break; }
    cn_solve_stats ss;
    st = cn_solve_device(S, 9, S->d_targets, S->d_xout, &o, &ss);
    if (st != CN_OK) break;
    double* cur = S->d_xout;
    double* nxt = d_tmp;
    for (int pass = 0; pass < nu; ++pass) {
      if (cn::launch_ddm_smooth(nv, S->D.K_ptr, S->D.K_col, cur, nxt, omega, S->stream) != cudaSuccess) {
        st = CN_CUDA_ERROR;
        break;
      }
      std::swap(cur, nxt);
    }
    if (st != CN_OK) break;
    if (cn::launch_ddm_topk(nv, c0, kc, take, cur, d_bidx, d_bw, d_cnt, S->stream) != cudaSuccess) st = CN_CUDA_ERROR;
  }
  if (st == CN_OK && cn::launch_ddm_finish(nv, take, d_bw, S->stream) != cudaSuccess) st = CN_CUDA_ERROR;
  if (st == CN_OK &&
      (cudaMemcpyAsync(infl_idx, d_bidx, sizeof(int) * (size_t)nv * take, cudaMemcpyDeviceToHost, S->stream) !=
           cudaSuccess ||
       cudaMemcpyAsync(infl_w, d_bw, sizeof(double) * (size_t)nv * take, cudaMemcpyDeviceToHost, S->stream) !=
           cudaSuccess ||
       cudaStreamSynchronize(S->stream) != cudaSuccess))
    st = CN_CUDA_ERROR;
  if (st == CN_CUDA_ERROR) set_err("cn_ddm_bind: %s", cudaGetErrorString(cudaGetLastError()));
  cudaStreamSynchronize(S->stream);
  release();
  S->have_solution = false;
  return st;
}

// Runtime DDM (DirectDeltaMush.lean:84-102): one thread per vertex.
cn_status cn_lbs_matvec_device(int32_t n_verts, int32_t precision, const void* d_rest, const void* d_transforms,
                               const int32_t* d_start, const int32_t* d_idx, const void* d_w, void* d_out,
                               void* stream) {
  if (n_verts < 0 || (n_verts > 0 && (!d_rest || !d_transforms || !d_start || !d_idx || !d_w || !d_out)) ||
      (precision != CN_PREC_MIXED && precision != CN_PREC_FP64)) {
    set_err("cn_lbs_matvec_device: bad arguments");
    return CN_BAD_INPUT;
  }
  CN_CUDA(cn::launch_lbs_matvec(n_verts, precision, d_rest, d_transforms, d_start, d_idx, d_w, d_out,
                                (cudaStream_t)stream));
  return CN_OK;
}

// SpMV / SpMM on the handle's reduced matrix (SparseLinAlg.lean:44-60,
// SlangCodegen/SpmvMulti.lean:78-119), on the handle's stream.
cn_status cn_spmv_device(cn_handle S, int32_t k, int32_t precision, const void* d_x, void* d_y) {
  if (!S || !d_x || !d_y) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  if ((k != 1 && k != 3 && k != 9 && k != 24) || (precision != CN_PREC_MIXED && precision != CN_PREC_FP64)) {
    set_err("cn_spmv_device: k must be 1, 3, 9 or 24 and precision CN_PREC_MIXED or CN_PREC_FP64");
    return CN_BAD_INPUT;
  }
  if (((uintptr_t)d_x | (uintptr_t)d_y) & 15) {
    set_err("cn_spmv_device: x and y must be 16-byte aligned");
    return CN_BAD_INPUT;
  }
  CN_CUDA(cudaSetDevice(S->device));
  const void* val = precision == CN_PREC_MIXED ? (const void*)S->D.A32 : (const void*)S->D.A64;
  if (S->spmv_ents < 0) S->spmv_ents = cn::spmm_tile_entries(S->H.A_ptr.data(), S->H.n);
  CN_CUDA(cn::launch_spmm(S->H.n, k, precision, S->D.A_ptr, S->D.A_col, val, d_x, d_y, S->spmv_ents,
                          S->d_spmv_err, S->stream));
  return CN_OK;
}

cn_status cn_set_launch(cn_handle S, int32_t lanes, int32_t block, int32_t grid) {
  if (!S || (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16) || block < 64 ||
      block > 1024 || block % 32 != 0 || grid < 1) {
    set_err("bad launch shape (lanes %d, block %d, grid %d)", lanes, block, grid);
    return CN_BAD_INPUT;
  }
  const bool rc = row_cached(S);  // clamps its grid per solve
  if (grid > 1 && !rc) {
    const int mg = std::min(cn::persistent_max_grid(CN_PREC_MIXED, S->kmax, lanes, block),
                            cn::persistent_max_grid(CN_PREC_FP64, S->kmax, lanes, block));
    if (mg < 1) {
      set_err("shape (lanes %d, block %d) does not fit as a cooperative grid", lanes, block);
      return CN_BAD_INPUT;
    }
    grid = std::min(grid, std::min(mg, S->max_grid_alloc));
  }
  if (rc) grid = std::min(grid, S->max_grid_alloc);
  S->lanes = lanes;
  S->block = block;
  S->grid = grid;
  S->shape_set = true;
  return CN_OK;
}

// The project's launch-shape autotuner: every candidate (lanes per row,
// threads per block, blocks) solves the caller's right-hand sides a few times
// on the device; the fastest median keeps.  results (nullable, 5 doubles per
// candidate): lanes, block, grid, median ms, iterations.
cn_status cn_autotune(cn_handle S, int32_t k, const double* d_targets, const cn_solve_opts* opts, int32_t reps,
                      double* results, int32_t* n_results) {
  if (!S || !d_targets) {
    set_err("null argument");
    return CN_BAD_INPUT;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->device);
  struct Cand { int lanes, block, grid; };
  std::vector<Cand> cands;
  const int lane_set[] = {1, 2, 4, 8};
  if (row_cached(S)) {
    // the row-cached kernel: one lane per row; blocks of up to 512 threads
    // take two rows per thread, larger ones one
    for (int g : {sms / 2, (3 * sms) / 4, sms}) {
      const int fit = std::min(512, std::max(128, ((S->H.n + 2 * g - 1) / (2 * g) + 31) / 32 * 32));
      cands.push_back({1, fit, g});
      for (int b : {256, 384, 512, 768, 1024})
        if (b != fit) cands.push_back({1, b, g});
    }
  } else {
    if (S->H.n <= 65536)
      for (int l : lane_set)
        for (int b : {256, 512, 1024}) cands.push_back({l, b, 1});
    if (S->H.n > 4096)
      for (int l : lane_set)
        for (int b : {256, 512, 1024})
          for (int g : {sms / 2, sms, 2 * sms}) cands.push_back({l, b, g});
  }
  const int old_l = S->lanes, old_b = S->block, old_g = S->grid;
  const bool old_set = S->shape_set;
  cn_solve_opts o;
  if (opts) o = *opts;
  else cn_default_solve_opts(&o);
  double best = 1e30;
  Cand pick{old_l, old_b, old_g};
  int nr = 0;
  reps = std::max(1, reps);
  for (const Cand& c : cands) {
    if (cn_set_launch(S, c.lanes, c.block, c.grid) != CN_OK) continue;
    std::vector<double> ms;
    int iters = 0;
    bool ok = true;
    for (int r = 0; r <= reps; ++r) {  // the first run warms up
      cn_solve_stats st;
      if (cn_solve_device(S, k, d_targets, S->d_xout, &o, &st) != CN_OK) { ok = false; break; }
      if (r) ms.push_back(st.device_ms);
      iters = st.iterations;
    }
    if (!ok) continue;
    std::sort(ms.begin(), ms.end());
    const double med = ms[ms.size() / 2];
    if (results) {
      double* R = results + 5 * nr;
      R[0] = c.lanes; R[1] = c.block; R[2] = S->grid; R[3] = med; R[4] = iters;
    }
    ++nr;
    if (med < best) { best = med; pick = {c.lanes, c.block, S->grid}; }
  }
  if (n_results) *n_results = nr;
  cn_set_launch(S, pick.lanes, pick.block, pick.grid);
  S->have_solution = false;
  if (nr == 0) {
    set_err("no launch shape ran");
    cn_set_launch(S, old_l, old_b, old_g);
    S->shape_set = old_set;
    return CN_CUDA_ERROR;
  }
  return CN_OK;
}

cn_status cn_hsc_info(cn_handle S, int32_t* n_levels, int32_t* tail, int32_t* n_coarse, int32_t* level_off,
                      int32_t* order) {
  if (!S || !S->hsc) {
    set_err("not an HSC handle");
    return CN_BAD_INPUT;
  }
  if (n_levels) *n_levels = S->hsc_L;
  if (tail) *tail = S->hsc_tail;
  if (n_coarse) *n_coarse = S->hsc_nc;
  if (level_off) std::memcpy(level_off, S->hsc_off_h.data(), sizeof(int) * S->hsc_off_h.size());
  if (order) std::memcpy(order, S->hsc_order.data(), sizeof(int) * S->hsc_order.size());
  return CN_OK;
}

cn_status cn_export_csr(cn_handle S, int32_t* free_of, int32_t* rowptr, int32_t* colidx,
                        double* vals) {
  if (!S) return CN_BAD_INPUT;
  CN_CUDA(cudaSetDevice(S->device));
  const MeshHost& H = S->H;
  if (free_of) std::memcpy(free_of, H.free_of.data(), sizeof(int) * H.n);
  if (rowptr) std::memcpy(rowptr, H.A_ptr.data(), sizeof(int) * (H.n + 1));
  if (colidx) std::memcpy(colidx, H.A_col.data(), sizeof(int) * H.nnzA);
  if (vals) CN_CUDA(cudaMemcpy(vals, S->D.A64, sizeof(double) * H.nnzA, cudaMemcpyDeviceToHost));
  return CN_OK;
}

cn_status cn_export_factor(cn_handle S, int32_t* rowptr, int32_t* colidx, double* vals) {
  if (!S) return CN_BAD_INPUT;
  CN_CUDA(cudaSetDevice(S->device));
  const MeshHost& H = S->H;
  std::vector<double> L(H.nnzL), d(H.n);
  if (H.nnzL) CN_CUDA(cudaMemcpy(L.data(), S->D.L64, sizeof(double) * H.nnzL, cudaMemcpyDeviceToHost));
  if (H.n) CN_CUDA(cudaMemcpy(d.data(), S->D.Ld64, sizeof(double) * H.n, cudaMemcpyDeviceToHost));
  int q = 0;
  if (rowptr) rowptr[0] = 0;
  for (int i = 0; i < H.n; ++i) {
    for (int e = H.L_ptr[i]; e < H.L_ptr[i + 1]; ++e, ++q) {
      if (colidx) colidx[q] = H.L_col[e];
      if (vals) vals[q] = L[e];
    }
    if (colidx) colidx[q] = i;
    if (vals) vals[q] = d[i];
    ++q;
    if (rowptr) rowptr[i + 1] = q;
  }
  return CN_OK;
}

cn_status cn_export_k(cn_handle S, int32_t* rowptr, int32_t* colidx, double* vals) {
  if (!S) return CN_BAD_INPUT;
  CN_CUDA(cudaSetDevice(S->device));
  const MeshHost& H = S->H;
  if (rowptr) std::memcpy(rowptr, H.K_ptr.data(), sizeof(int) * (H.nv + 1));
  if (colidx) std::memcpy(colidx, H.K_col.data(), sizeof(int) * H.nnzK);
  if (vals) CN_CUDA(cudaMemcpy(vals, S->D.K_val, sizeof(double) * H.nnzK, cudaMemcpyDeviceToHost));
  return CN_OK;
}

}  // extern "C"
