"""HSC (hierarchical sparsify and compensate) hierarchy and V-cycle, numpy /
scipy restatement.

TEST INFRASTRUCTURE ONLY: the checker of the product's HSC preconditioner
(tool_godot_curvenet_b200/csrc/cn_hsc.cpp and the HSC phases of the
persistent solve).  The reference specifies the elimination primitive
(HierarchicalSparsifyCompensate.lean:97-125: eliminating v adds
w_i w_j / deg(v) to the edge (i, j) of every pair of v's neighbours and drops
v's edges); the level structure, sparsification and coarse solve below are
the library's completion of it (Krishnan-Fattal-Szeliski 2013 is the
reference's citation):

1. M-matrix part: every positive off-diagonal a_ij of A is dropped and added
   to a_ii and a_jj (A + a_ij (e_i - e_j)(e_i - e_j)^T: still SPD).
2. Per level, F = greedy maximal independent set in index order; C = rest.
   Eliminating the independent set F is the spec's rule applied to each v in
   F: S = M_CC - M_CF D_F^{-1} M_FC (the diagonal of a graph Laplacian is
   deg(v), with Dirichlet excess it is M_vv).
3. Sparsify: a fill entry (i, j) of S absent from M_CC is kept when
   |S_ij| >= theta sqrt(S_ii S_jj) or when it is among the keep_k strongest
   off-diagonals of row i or of row j; a dropped entry is compensated into
   the diagonals (S_ii += S_ij, S_jj += S_ij), which keeps every row sum, so
   the operator's action on constants (and the Dirichlet excess) is
   unchanged, and no row loses all of its couplings.
4. Recurse until at most n_coarse unknowns; the coarsest matrix is inverted
   densely.
Apply (z = M^{-1} r): down the levels w_C -= M_CF D_F^{-1} w_F, the coarse
z_c = S^{-1} w_c, up the levels z_F = D_F^{-1} (w_F - M_FC z_C).
"""
import numpy as np
import scipy.sparse as sp


def m_matrix_part(A):
    A = sp.csr_matrix(A, dtype=np.float64)
    off = A - sp.diags(A.diagonal())
    pos = off.multiply(off > 0)
    if pos.nnz:
        A = A - pos + sp.diags(np.asarray(pos.sum(axis=1)).ravel())
    A = sp.csr_matrix(A)
    A.eliminate_zeros()
    A.sort_indices()
    return A


def greedy_mis(M):
    n = M.shape[0]
    sel = np.zeros(n, bool)
    blocked = np.zeros(n, bool)
    ptr, col = M.indptr, M.indices
    for v in range(n):
        if not blocked[v]:
            sel[v] = True
            blocked[col[ptr[v]:ptr[v + 1]]] = True
    return sel


def _top_k(row, col, mag, n, k):
    """Entries among the k largest magnitudes of their row or of their
    column's row (symmetric union); ties broken by the lower column."""
    order = np.lexsort((col, -mag, row))
    rank = np.empty(row.size, np.int64)
    starts = np.searchsorted(row[order], np.arange(n))
    rank[order] = np.arange(row.size) - starts[row[order]]
    in_row = (rank < k) & (mag >= 0)
    key = row.astype(np.int64) * n + col
    tkey = col.astype(np.int64) * n + row
    kept = set(key[in_row].tolist())
    return in_row | np.fromiter((t in kept for t in tkey), bool, count=tkey.size)


def build(A, theta=0.05, n_coarse=512, max_levels=64, keep_k=3):
    """Returns dict(order, levels=[(off, nf, R (CSR over C rows, cols F local),
    P (CSR F x C), dinv)], coarse_off, Sinv).  `order` maps HSC position ->
    row of A."""
    M = m_matrix_part(A)
    gid = np.arange(M.shape[0])
    order = []
    levels = []
    off = 0
    while M.shape[0] > n_coarse and len(levels) < max_levels:
        sel = greedy_mis(M)
        F = np.nonzero(sel)[0]
        Cc = np.nonzero(~sel)[0]
        if F.size < 0.02 * M.shape[0]:
            break
        d = M.diagonal()[F]
        MCF = M[Cc][:, F]
        MFC = M[F][:, Cc]
        levels.append(dict(off=off, nf=F.size, R=sp.csr_matrix(MCF @ sp.diags(1.0 / d)), P=sp.csr_matrix(MFC),
                           dinv=1.0 / d, C_gid=gid[Cc], F_gid=gid[F]))
        order.extend(gid[F].tolist())
        off += F.size
        S = sp.csr_matrix(M[Cc][:, Cc] - MCF @ sp.diags(1.0 / d) @ MFC)
        S.sort_indices()
        base = sp.csr_matrix(M[Cc][:, Cc])
        base.data[:] = 1.0
        # fill entries (absent from M_CC) below the threshold -> diagonal
        Sc = S.tocoo()
        diag = S.diagonal()
        is_base = np.asarray(base[Sc.row, Sc.col]).ravel() != 0
        off_diag = Sc.row != Sc.col
        weak = np.abs(Sc.data) < theta * np.sqrt(diag[Sc.row] * diag[Sc.col])
        top = _top_k(Sc.row, Sc.col, np.where(off_diag, np.abs(Sc.data), -1.0), S.shape[0], keep_k)
        drop = off_diag & ~is_base & weak & ~top
        comp = np.bincount(Sc.row[drop], weights=Sc.data[drop], minlength=S.shape[0])
        keep = ~drop
        S = sp.csr_matrix((Sc.data[keep], (Sc.row[keep], Sc.col[keep])), shape=S.shape)
        S = S + sp.diags(comp)
        S = sp.csr_matrix(S)
        S.sort_indices()
        M = S
        gid = gid[Cc]
    order.extend(gid.tolist())
    order = np.array(order)
    pos_of = np.empty(order.size, np.int64)
    pos_of[order] = np.arange(order.size)
    for L in levels:
        L["C_pos"] = pos_of[L["C_gid"]]  # HSC position of each C row of the level
    Sd = M.toarray()
    Sinv = np.linalg.inv(Sd)
    return dict(order=order, levels=levels, coarse_off=off, Sinv=Sinv, n=A.shape[0])


def apply(h, r):
    """z = M^{-1} r for r in A's row order (n,) or (n, k)."""
    n = h["n"]
    rr = np.asarray(r, dtype=np.float64)
    w = rr[h["order"]].copy()
    for L in h["levels"]:
        o, nf = L["off"], L["nf"]
        w[L["C_pos"]] -= L["R"] @ w[o:o + nf]
    co = h["coarse_off"]
    z = np.zeros_like(w)
    z[co:] = h["Sinv"] @ w[co:]
    for L in reversed(h["levels"]):
        o, nf = L["off"], L["nf"]
        dinv = L["dinv"][:, None] if w.ndim == 2 else L["dinv"]
        z[o:o + nf] = dinv * (w[o:o + nf] - L["P"] @ z[L["C_pos"]])
    out = np.empty_like(z)
    out[h["order"]] = z
    return out


def pcg(A, b, h, tol=1e-8, max_iter=1000):
    """HSC-PCG in FP64 (relative test ||r|| < tol ||b||); returns (x, iters)."""
    x = np.zeros_like(b)
    r = b.copy()
    z = apply(h, r)
    p = z.copy()
    rz = r @ z
    bb = b @ b
    for it in range(max_iter):
        Ap = A @ p
        a = rz / (p @ Ap)
        x += a * p
        r -= a * Ap
        if r @ r < tol * tol * bb:
            return x, it + 1
        z = apply(h, r)
        rzn = r @ z
        p = z + (rzn / rz) * p
        rz = rzn
    return x, max_iter
