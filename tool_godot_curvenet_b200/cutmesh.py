"""Cut-mesh construction on the GPU over the C ABI: the halfedge structure of
a triangle soup (HalfedgeBuilder.lean:34-90), the seam cut along profile-curve
loops, and batches of the cut surgery (CutAlgorithm.lean:49-255).  Halfedge
records are (target, twin, next, face) int32 rows; -1 marks no twin / the
outer face."""
import ctypes as C

import numpy as np

from . import _lib as L
from .solver import CnError, _i32, _ip


def halfedges(n_verts, tris):
    """(n_he, 4) halfedge records of HalfedgeMesh.fromTriangles, on the GPU."""
    tris = _i32(tris).reshape(-1, 3)
    out = np.empty((max(6 * tris.shape[0], 1), 4), np.int32)
    n = C.c_int32(0)
    st = L.lib().cn_halfedges(n_verts, tris.shape[0], _ip(tris), _ip(out), C.byref(n))
    if st != L.CN_OK:
        raise CnError(st, "cn_halfedges")
    return out[: n.value].copy()


def cut_mesh_gpu(n_verts, tris, loops):
    """cut_mesh computed on the GPU: (tris_cut, parent)."""
    tris = _i32(tris).reshape(-1, 3)
    ptr = np.zeros(len(loops) + 1, np.int32)
    for i, l in enumerate(loops):
        ptr[i + 1] = ptr[i] + len(l)
    verts = _i32(np.concatenate(loops)) if loops else np.zeros(1, np.int32)
    out = np.empty_like(tris)
    parent = np.empty(n_verts + int(ptr[-1]), np.int32)
    nv_out = C.c_int32(0)
    st = L.lib().cn_cut_mesh_gpu(n_verts, tris.shape[0], _ip(tris), len(loops), _ip(ptr), _ip(verts), _ip(out),
                                 _ip(parent), C.byref(nv_out))
    if st != L.CN_OK:
        raise CnError(st, "cn_cut_mesh_gpu")
    return out, parent[: nv_out.value]


def _surgery(fn, name, counts, he, m, *lists):
    counts = _i32(counts).copy()
    he = _i32(he).reshape(-1, 4)
    buf = np.empty((he.shape[0] + 2 * m, 4), np.int32)
    buf[: he.shape[0]] = he
    args = [_ip(_i32(x)) for x in lists]
    st = fn(_ip(counts), _ip(buf), m, *args)
    if st != L.CN_OK:
        raise CnError(st, name)
    return counts, buf


def subdivide_edges(counts, he, edges):
    """Batch of subdivideEdge: returns (counts, he) after the batch."""
    return _surgery(L.lib().cn_subdivide_edges, "cn_subdivide_edges", counts, he, len(edges), edges)


def split_faces(counts, he, a, b):
    """Batch of splitFace over (a[k], b[k]) pairs in distinct faces."""
    return _surgery(L.lib().cn_split_faces, "cn_split_faces", counts, he, len(a), a, b)


def insert_cracks(counts, he, anchors):
    """Batch of insertCrack at distinct anchor halfedges."""
    return _surgery(L.lib().cn_insert_cracks, "cn_insert_cracks", counts, he, len(anchors), anchors)
