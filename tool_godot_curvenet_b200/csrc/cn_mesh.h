// cn_mesh.h -- per-mesh structure shared by the single-mesh handle
// (cn_host.cpp) and the batch (cn_batch_host.cpp): the integer structure
// built on the host, its device layout in one allocation, and the GPU
// assembly + IC(0) factor.  Not part of the public ABI.
#pragma once

#include <string>
#include <vector>

#include "cn_internal.h"

namespace cn {

// Thread-local error text behind cn_last_error().
void set_err(const char* fmt, ...);
const char* last_err();

// Integer structure of one cut mesh (host).  Row / column indices are local
// to the mesh.
struct MeshHost {
  int nv = 0, nt = 0, nh = 0, n = 0, nlev = 0, ncolors = 0;
  int nnzK = 0, nnzA = 0, nnzL = 0;
  std::vector<double> pos;
  std::vector<int> tris, handles, hidx;
  std::vector<int> K_ptr, K_col, K_cptr, K_contrib;   // K over all vertices
  std::vector<int> free_of, lev_ptr;                   // solve order
  std::vector<int> A_ptr, A_col, A_src, A_diag;        // A = K[free, free]
  std::vector<int> L_ptr, L_col, L_src, T_ptr, T_a, T_b;  // strictly-lower IC(0) pattern
  std::vector<int> U_ptr, U_col, U_src;                // U = L^T
  std::vector<int> vf_ptr, vf_face, vf_corner;         // vertex -> incident faces (ascending)
};

// Device arrays of one mesh (sub-allocations of one buffer).
struct MeshDev {
  double *pos = nullptr, *face_m = nullptr, *K_val = nullptr;
  int *tris = nullptr, *K_ptr = nullptr, *K_col = nullptr, *K_cptr = nullptr, *K_contrib = nullptr;
  int *hidx = nullptr, *free_of = nullptr, *handles = nullptr;
  int *A_ptr = nullptr, *A_col = nullptr, *A_src = nullptr, *A_diag = nullptr, *lev_ptr = nullptr;
  double* A64 = nullptr;
  float* A32 = nullptr;
  int *L_ptr = nullptr, *L_col = nullptr, *L_src = nullptr, *T_ptr = nullptr, *T_a = nullptr,
      *T_b = nullptr;
  int *U_ptr = nullptr, *U_col = nullptr, *U_src = nullptr;
  double *L64 = nullptr, *U64 = nullptr, *Ld64 = nullptr, *dinv64 = nullptr;
  float *L32 = nullptr, *U32 = nullptr, *dinv32 = nullptr;
};

// Bump allocator over one device buffer: a sizing pass (base == nullptr)
// counts bytes, the second pass hands out 256-byte aligned pointers.
struct Bump {
  char* base = nullptr;
  size_t off = 0;
  template <class T>
  T* take(size_t count) {
    const size_t bytes = (sizeof(T) * (count ? count : 1) + 255) & ~(size_t)255;
    T* p = base ? (T*)(base + off) : nullptr;
    off += bytes;
    return p;
  }
};

cn_status check_mesh(const cn_mesh_desc* m);
cn_status build_host(const cn_mesh_desc* m, const cn_build_opts& o, MeshHost& H);
void layout(Bump& b, const MeshHost& H, MeshDev& D);
cn_status upload(const MeshHost& H, const MeshDev& D, cudaStream_t s);
// Assembly of K and A and the IC(0) factor with diagonal-shift retries;
// d_status: one device int.  Synchronises the stream.
cn_status assemble_factor(const MeshHost& H, const MeshDev& D, const cn_build_opts& o, int* d_status,
                          cudaStream_t s, double* shift_used);
// Solve arguments of a mesh (matrix, maps, precision-dependent values);
// vectors, partials, control, targets and outputs are filled by the caller.
SolveArgs solve_args(const MeshHost& H, const MeshDev& D, bool mixed);

// Relabel the solve order: new row p is old row order[p] (A, its source map,
// the diagonal positions and free_of follow).  Only for a mesh without an
// IC(0) pattern (one level, empty L).
void permute_solve_order(MeshHost& H, const std::vector<int>& order);

// Vertex -> incident faces (ascending face id) with the vertex's corner.
void vertex_faces(int nv, int nt, const int* tris, std::vector<int>& ptr, std::vector<int>& face,
                  std::vector<int>& corner);

}  // namespace cn
